// C ABI of the Relay-BP-S decoder (include/relaybp.h): graph preparation,
// decoder state, launch-shape selection and the decode launch.  The kernel
// itself is in relaybp_kernel.cuh.

#include "relaybp.h"
#include "relaybp_host.h"
#include "relaybp_kernel.cuh"
#include "relaybp_slots.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace {

using rbpk::DevArgs;
using rbpk::DevGraph;
using rbpk::KernelFn;
using rbph::align16;
using rbph::DevBuf;
using rbph::DeviceGuard;
using rbph::fail;

}  // namespace

namespace rbph {
std::string& err_slot() {
  thread_local std::string s;
  return s;
}
}  // namespace rbph

struct rbp_decoder {
  const rbp_graph* g = nullptr;
  rbp_params p{};
  int rows = 0;                // check slots per row in the layout (padded, multiple of VEC)
  DevBuf<uint16_t> var_pos;    // [vslots, V] slot index of variable v's k-th edge
  DevBuf<float> llr;
  DevBuf<float> gamma_legs;
  DevBuf<float> alpha;
  DevBuf<int> queue;
  int n_alpha = 0;
  // launch shapes: shape[0] for launches that skip the relay legs (pre-iterations
  // only, so a shot's latency is bounded by pre_iter), shape[1] for the others
  struct Shape {
    KernelFn kernel = nullptr;
    int group_threads = 0, groups = 0, blocks = 0, vpt = 0;
    int nshots = 1;            // shots a group decodes at once
    int slots_kernel = 0;      // 1: relaybp_slots_kernel (one group per block)
    int minb = 1;              // resident blocks per SM the kernel is compiled for
    int group_bytes = 0, block_bytes = 0;
  } shape[2];
  int sm_count = 0;
  size_t max_smem = 0;
};

namespace {

size_t msg_size(int t) { return t == RBP_MSG_F64 ? 8 : (t == RBP_MSG_F32 ? 4 : 2); }

struct Layout {
  int off_chk_deg, off_llr, off_first, off_group0;
  int g_msg, g_par, g_best, g_first, g_red, g_s1, group_bytes;
};

// Rows of the check-slot layout: the slot count the kernel holds in registers
// (8 or 16) or the exact maximum degree, rounded up to whole 16-byte chunks.
int layout_rows(int slots, int msg_type) {
  const int vec = 16 / (int)msg_size(msg_type);
  const int r = slots <= 8 ? 8 : (slots <= 16 ? 16 : slots);
  return (r + vec - 1) / vec * vec;
}

// Slot index of (slot j, check c) for the message type (slot_index<M> in the kernel).
int slot_index_host(int j, int c, int C, int msg_type) {
  switch (msg_type) {
    case RBP_MSG_F32: return rbpk::slot_index<float>(j, c, C);
    case RBP_MSG_F64: return rbpk::slot_index<double>(j, c, C);
    default: return rbpk::slot_index<__half>(j, c, C);
  }
}

// Block-wide tables first, then one region per group.  first_sums: the region also holds
// the shot's first-pass sums and the memory mixes a relay leg's first iteration keeps for its
// deferred stores, one accumulator each per owned-variable slot (the one-shot block-per-group
// kernel).
Layout make_layout(int C, int V, int rows, int msg_type, int group_threads, bool first_sums = false) {
  Layout L{};
  int o = 0;
  L.off_chk_deg = o;
  o = align16(o + C);
  L.off_llr = o;
  o = align16(o + 4 * V);
  L.off_first = o;  // first-pass table of the check rows (see build_first_pass_table)
  o = align16(o + (int)msg_size(msg_type) * rows * C);
  L.off_group0 = o;
  const int slots_total = rows * C + 1;  // + the dummy slot of absent variable edges
  const int W = (V + 31) / 32;
  int q = 0;
  L.g_msg = q;
  q = align16(q + (int)msg_size(msg_type) * slots_total);
  L.g_par = q;
  q = align16(q + 4 * ((C + 31) / 32));
  L.g_best = q;
  q = align16(q + 4 * W);
  L.g_first = q;
  q = align16(q + 4 * W);
  L.g_red = q;
  q = align16(q + 8 * (group_threads / 32 + 4));
  L.g_s1 = q;
  if (first_sums) {
    int vpt = 16;  // owned variables per thread (vpt_for)
    for (int v : rbpk::kVptChoices)
      if ((long long)v * group_threads >= V) {
        vpt = v;
        break;
      }
    q = align16(q + (msg_type == RBP_MSG_F64 ? 8 : 4) * 2 * vpt * group_threads);  // + memory mixes
  }
  L.group_bytes = q;
  return L;
}

KernelFn pick_kernel(int msg_type, int dc, int dv, int vpt) {
  switch (msg_type) {
    case RBP_MSG_F32: return rbpk::pick_f32(dc, dv, vpt);
    case RBP_MSG_F16: return rbpk::pick_f16(dc, dv, vpt);
    case RBP_MSG_BF16: return rbpk::pick_bf16(dc, dv, vpt);
    case RBP_MSG_F64: return rbpk::pick_f64(dc, dv, vpt);
    default: return nullptr;
  }
}

KernelFn pick_slots_kernel(int msg_type, int dc, int dv, int vpt, int ns, int minb) {
  switch (msg_type) {
    case RBP_MSG_F32: return rbpk::pick_slots_f32(dc, dv, vpt, ns, minb);
    case RBP_MSG_F16: return rbpk::pick_slots_f16(dc, dv, vpt, ns, minb);
    case RBP_MSG_BF16: return rbpk::pick_slots_bf16(dc, dv, vpt, ns, minb);
    case RBP_MSG_F64: return rbpk::pick_slots_f64(dc, dv, vpt, ns, minb);
    default: return nullptr;
  }
}

// Smallest supported owned-variable count covering V with G threads.
int vpt_for(int V, int G) {
  const int need = (V + G - 1) / G;
  for (int v : rbpk::kVptChoices)
    if (v >= need) return v;
  return -1;
}

// Default shape: the fewest owned variables per thread (from 3 up) whose group
// still fits the register budget of that count (of the one- or two-shot
// kernel, at one or two resident blocks per SM), so a shot's iteration is short.
int default_group_threads(int C, int V, int nshots = 1, int vslots = 8, int minb = 1) {
  for (int vpt : {3, 4, 6, 8, 12, 16}) {
    const int G = std::max(32, (V + vpt - 1) / vpt + 31) / 32 * 32;
    const int max_threads = minb == 2 ? rbpk::max_slots_block_threads2(vpt)
                                      : rbpk::max_slots_block_threads(vpt, nshots, vslots <= 3 ? 3 : 8);
    if (G <= max_threads && (C + G - 1) / G <= 32 && vpt_for(V, G) <= vpt) return G;
  }
  return 256;  // configure reports why no shape fits
}

// Allow a kernel the device's opt-in shared memory minus its static shared
// memory as dynamic shared memory.  The attribute belongs to the kernel
// function and is shared by every decoder using it, so it is set to that
// limit; occupancy queries use each launch's actual size.
cudaError_t set_max_dynamic_smem(const void* kernel, size_t max_smem, size_t* static_smem = nullptr) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
  if (e != cudaSuccess) return e;
  if (static_smem) *static_smem = fa.sharedSizeBytes;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)(max_smem - fa.sharedSizeBytes));
}

struct Launch {
  KernelFn kernel;
  int group_threads, groups, blocks;
  int nshots;        // shots a group decodes at once
  int slots_kernel;  // 1: relaybp_slots_kernel (one group per block, nshots shot regions)
  int minb;          // resident blocks per SM the kernel is compiled for
};

// Block-per-group shape: one group of G threads per block with nshots shot regions
// (relaybp_slots_kernel), compiled for minb (1 or 2) resident blocks per SM.
int choose_slots_launch(int C, int V, int slots, int vslots, int rows, int msg_type, int G, int nshots, int minb,
                        size_t max_smem, int sm_count, Launch* out, const std::string& w) {
  const int vpt = vpt_for(V, G);
  const int max_threads = minb == 2 ? rbpk::max_slots_block_threads2(vpt)
                                    : rbpk::max_slots_block_threads(vpt, nshots, vslots <= 3 ? 3 : 8);
  if (G > max_threads)
    return fail(RBP_ERR_UNSUPPORTED, w + ": " + std::to_string(G) + " threads with " + std::to_string(vpt) +
                                         " variables each exceed the register budget of " + std::to_string(nshots) +
                                         "-shot groups" + (minb == 2 ? " at two blocks per SM" : ""));
  KernelFn k = pick_slots_kernel(msg_type, slots, vslots, vpt, nshots, minb);
  if (!k)
    return fail(RBP_ERR_UNSUPPORTED,
                w + (minb == 2 ? ": no two-blocks-per-SM kernel for this shape (one shot per group, check "
                                 "degrees up to 16)"
                               : ": no block-per-group kernel for this degree / shape (check degrees "
                                 "above 16 run with several groups per block, one shot each)"));
  const Layout L = make_layout(C, V, rows, msg_type, G, nshots == 1);
  const size_t smem = (size_t)L.off_group0 + (size_t)nshots * L.group_bytes;
  if (smem > max_smem)
    return fail(RBP_ERR_UNSUPPORTED, w + ": " + std::to_string(nshots) + " shots' state (" +
                                         std::to_string(nshots * L.group_bytes) + " B) does not fit in shared memory");
  RBP_CUDA(set_max_dynamic_smem(reinterpret_cast<const void*>(k), max_smem));
  int per_sm = 0;
  RBP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, G, smem));
  if (per_sm < 1) return fail(RBP_ERR_UNSUPPORTED, w + ": launch shape has zero occupancy");
  *out = Launch{k, G, 1, per_sm * sm_count, nshots, 1, minb};
  return RBP_OK;
}

// Kernel and launch shape for G threads per group (groups_per_block 0: as many
// as fit) decoding `nshots` shots at once (1 or 2); blocks_per_sm 2 selects the
// block-per-group kernel compiled for two resident blocks per SM.
int choose_launch(int C, int V, int slots, int vslots, int rows, int msg_type, int G, int groups_per_block,
                  size_t max_smem, int sm_count, Launch* out, const char* who, int nshots = 1,
                  int blocks_per_sm = 1) {
  const std::string w(who);
  if (G % 32 != 0 || G > 1024)
    return fail(RBP_ERR_ARGUMENT, w + ": group_threads must be a multiple of 32, at most 1024");
  if (nshots != 1 && nshots != 2) return fail(RBP_ERR_ARGUMENT, w + ": shots_per_group must be 1 or 2");
  const int vpt = vpt_for(V, G);
  if (vpt < 0) return fail(RBP_ERR_UNSUPPORTED, w + ": more than 16 variables per thread; use more group threads");
  if ((C + G - 1) / G > 32) return fail(RBP_ERR_UNSUPPORTED, w + ": more than 32 checks per thread; use more group threads");
  if (blocks_per_sm != 1 && blocks_per_sm != 2)
    return fail(RBP_ERR_ARGUMENT, w + ": blocks_per_sm must be 0 (one), 1 or 2");
  if (blocks_per_sm == 2 && (nshots != 1 || groups_per_block != 1))
    return fail(RBP_ERR_UNSUPPORTED, w + ": two blocks per SM run the block-per-group kernel with one shot per "
                                         "group (groups_per_block 1, shots_per_group 1)");
  // groups_per_block 1, or two shots per group: the block-per-group kernel
  if (nshots == 2 || groups_per_block == 1) {
    if (groups_per_block > 1)
      return fail(RBP_ERR_UNSUPPORTED, w + ": two-shot groups run one group per block");
    return choose_slots_launch(C, V, slots, vslots, rows, msg_type, G, nshots, blocks_per_sm, max_smem, sm_count,
                               out, w);
  }
  const int max_threads = rbpk::max_block_threads(vpt);
  if (G > max_threads)
    return fail(RBP_ERR_UNSUPPORTED, w + ": " + std::to_string(G) + " threads with " + std::to_string(vpt) +
                                         " variables each exceed the register budget");
  KernelFn k = pick_kernel(msg_type, slots, vslots, vpt);
  if (!k) return fail(RBP_ERR_UNSUPPORTED, w + ": no kernel for this degree / shape");
  const Layout L = make_layout(C, V, rows, msg_type, G);
  const size_t block_fixed = (size_t)L.off_group0;
  if (block_fixed + L.group_bytes > max_smem)
    return fail(RBP_ERR_UNSUPPORTED,
                w + ": one shot's state (" + std::to_string(L.group_bytes) + " B) does not fit in shared memory");
  int max_groups = (int)((max_smem - block_fixed) / L.group_bytes);
  max_groups = std::min(max_groups, max_threads / G);
  if (G != 32) max_groups = std::min(max_groups, 15);  // named barriers 1..15
  const int NG = groups_per_block > 0 ? groups_per_block : max_groups;
  if (NG < 1 || NG > max_groups)
    return fail(RBP_ERR_UNSUPPORTED,
                w + ": groups_per_block must be in [1, " + std::to_string(max_groups) + "] for this shape");
  RBP_CUDA(set_max_dynamic_smem(reinterpret_cast<const void*>(k), max_smem));
  const size_t smem = block_fixed + (size_t)NG * L.group_bytes;
  int per_sm = 0;
  RBP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, G * NG, smem));
  if (per_sm < 1) return fail(RBP_ERR_UNSUPPORTED, w + ": launch shape has zero occupancy");
  *out = Launch{k, G, NG, per_sm * sm_count, 1, 0, 1};
  return RBP_OK;
}

int check_batch(const char* who, int64_t B, const rbp_batch* in, const rbp_outputs* out, const rbp_params& p,
                int n_alpha) {
  const std::string w(who);
  if (in->struct_size != sizeof(rbp_batch))
    return fail(RBP_ERR_ARGUMENT, w + ": rbp_batch.struct_size is " + std::to_string(in->struct_size) +
                                      ", this library's rbp_batch has " + std::to_string(sizeof(rbp_batch)) +
                                      " bytes (the caller's declaration differs from include/relaybp.h)");
  if (out->struct_size != sizeof(rbp_outputs))
    return fail(RBP_ERR_ARGUMENT, w + ": rbp_outputs.struct_size is " + std::to_string(out->struct_size) +
                                      ", this library's rbp_outputs has " + std::to_string(sizeof(rbp_outputs)) +
                                      " bytes (the caller's declaration differs from include/relaybp.h)");
  if (B < 0) return fail(RBP_ERR_ARGUMENT, w + ": negative batch");
  if (B > INT_MAX) return fail(RBP_ERR_UNSUPPORTED, w + ": batch exceeds 2^31-1 shots");
  if (B == 0) return RBP_OK;
  if (!in->syndromes || !out->found_count || !out->iterations)
    return fail(RBP_ERR_ARGUMENT, w + ": syndromes, found_count and iterations are required");
  if (in->pre_iter < 0) return fail(RBP_ERR_ARGUMENT, w + ": pre_iter must be >= 0");
  if (p.use_alpha && in->pre_iter > n_alpha) return fail(RBP_ERR_ARGUMENT, w + ": pre_iter exceeds the alpha table");
  if (in->n_shot_legs < 0 || (in->n_shot_legs > 0 && !in->gamma_legs_shot))
    return fail(RBP_ERR_ARGUMENT, w + ": gamma_legs_shot missing");
  if (in->shot_leg_rows < 0) return fail(RBP_ERR_ARGUMENT, w + ": shot_leg_rows must be >= 0");
  if (in->solved_legs < 0) return fail(RBP_ERR_ARGUMENT, w + ": solved_legs must be >= 0");
  if (in->parity_first < 0 || in->parity_first > 2) return fail(RBP_ERR_ARGUMENT, w + ": parity_first must be 0, 1 or 2");
  if (in->suspend_unsolved && !in->suspend_state)
    return fail(RBP_ERR_ARGUMENT, w + ": suspend_unsolved needs suspend_state");
  if (in->resume_state && (in->legs_begin < 0 || in->legs_begin > p.num_sets))
    return fail(RBP_ERR_ARGUMENT, w + ": legs_begin out of range");
  if ((reinterpret_cast<uintptr_t>(in->resume_state) | reinterpret_cast<uintptr_t>(in->suspend_state)) % 16)
    return fail(RBP_ERR_ARGUMENT, w + ": resume_state and suspend_state must be 16-byte aligned");
  return RBP_OK;
}

// Fill the kernel arguments and launch (memset of the work counter + kernel) on `st`.
int launch_decode(const DevGraph& dgph, const rbp_params& p, const Layout& L, const Launch& lc, const float* llr,
                  const float* gamma_legs, const float* alpha, int* queue, int64_t B,
                  const rbp_batch* in, const rbp_outputs* out, cudaStream_t st, const char* who) {
  DevArgs a{};
  a.pre_iter = in->pre_iter;
  a.num_sets = p.num_sets;
  a.set_max_iter = p.set_max_iter;
  a.stop_nconv = p.stop_nconv;
  a.last_leg = p.last_leg;
  a.use_alpha = p.use_alpha;
  a.use_beta = p.use_beta;
  a.mix_mode = p.mix_mode;
  a.skip_legs = in->skip_relay_legs;
  a.beta = p.beta;
  a.gamma0 = in->gamma0;
  a.llr = llr;
  a.gamma_legs = gamma_legs;
  a.alpha = alpha;
  a.B = B;
  a.syn = in->syndromes;
  a.llr_shot = in->llr_per_shot;
  a.gamma_pre = in->gamma_pre;
  a.gamma_legs_shot = in->gamma_legs_shot;
  a.n_shot_legs = in->n_shot_legs;
  a.shot_leg_rows = in->shot_leg_rows > 0 ? in->shot_leg_rows : std::max(1, in->n_shot_legs);
  a.order = in->shot_order;
  a.queue_len = in->queue_len;
  a.solved_gamma = in->solved_gamma;
  a.solved_legs = in->solved_legs;
  a.suspend_unsolved = in->suspend_unsolved;
  a.parity_first = in->parity_first;
  a.init_post = in->init_posterior;
  a.errors = out->errors;
  a.errors_packed = out->errors_packed;
  a.weights = out->weights;
  a.wfixed = reinterpret_cast<long long*>(out->weight_fixed);
  a.found = out->found_count;
  a.iters = out->iterations;
  a.last_post = out->last_posterior;
  a.legs_begin = in->legs_begin;
  a.legs_end = in->legs_end;
  a.resume = static_cast<const unsigned char*>(in->resume_state);
  a.suspend = static_cast<unsigned char*>(in->suspend_state);
  a.state_stride = rbpk::state_stride(dgph.V, p.msg_type == RBP_MSG_F64 ? 8 : 4);
  a.queue = queue;
  a.group_threads = lc.group_threads;
  a.groups = lc.groups;
  a.off_chk_deg = L.off_chk_deg;
  a.off_llr = L.off_llr;
  a.off_first = L.off_first;
  a.first_table = 1;
  a.off_group0 = L.off_group0;
  a.group_bytes = L.group_bytes;
  a.g_msg = L.g_msg;
  a.g_par = L.g_par;
  a.g_best = L.g_best;
  a.g_first = L.g_first;
  a.g_red = L.g_red;
  a.g_s1 = L.g_s1;
  const long long per_block = (long long)lc.groups * lc.nshots;  // shots a block decodes at once
  const long long need_blocks = (B + per_block - 1) / per_block;
  const int blocks = (int)std::min<long long>(lc.blocks, need_blocks);
  const size_t smem = (size_t)L.off_group0 + (size_t)per_block * L.group_bytes;
  cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(int), st);
  if (e != cudaSuccess) return fail(RBP_ERR_CUDA, std::string(who) + ": cudaMemsetAsync: " + cudaGetErrorString(e));
  lc.kernel<<<blocks, lc.group_threads * lc.groups, smem, st>>>(dgph, a);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(RBP_ERR_CUDA, std::string(who) + ": launch: " + cudaGetErrorString(e));
  return RBP_OK;
}

// Scratch of rbp_decode_static: the work counter and the graph tables of the
// current call.  Every device that loads the library holds it until exit.
static __device__ __align__(256) unsigned char g_static_scratch[RBP_STATIC_SCRATCH_BYTES];

// Device address of g_static_scratch on `device` (the current device), looked
// up on the first call per device and cached.  Host threads may race on a
// device's first lookup: both store the same address, and the atomics make
// that race well defined.
int static_scratch(int device, unsigned char** out) {
  static std::atomic<void*> cached[64];
  if (device < 0 || device >= 64) return fail(RBP_ERR_UNSUPPORTED, "rbp_decode_static: device ordinal above 63");
  void* ptr = cached[device].load(std::memory_order_relaxed);
  if (!ptr) {
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_scratch);
    if (e != cudaSuccess)
      return fail(RBP_ERR_CUDA, std::string("rbp_decode_static: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    cached[device].store(ptr, std::memory_order_relaxed);
  }
  *out = static_cast<unsigned char*>(ptr);
  return RBP_OK;
}

}  // namespace

extern "C" {

const char* rbp_last_error(void) { return rbph::err_slot().c_str(); }

const char* rbp_version(void) { return "relaybp-b200 0.2 (sm_100a)"; }

int rbp_graph_create(int32_t C, int32_t V, int32_t E, const int32_t* chk_ptr,
                     const int32_t* edge_var, const int32_t* var_ptr, const int32_t* var_edges,
                     int32_t device, rbp_graph** out) {
  if (!out) return fail(RBP_ERR_ARGUMENT, "rbp_graph_create: out is null");
  *out = nullptr;
  if (C <= 0 || V <= 0 || E <= 0) return fail(RBP_ERR_ARGUMENT, "rbp_graph_create: C, V and E must be positive");
  if (!chk_ptr || !edge_var || !var_ptr || !var_edges)
    return fail(RBP_ERR_ARGUMENT, "rbp_graph_create: null graph array");
  if (chk_ptr[0] != 0 || chk_ptr[C] != E || var_ptr[0] != 0 || var_ptr[V] != E)
    return fail(RBP_ERR_ARGUMENT, "rbp_graph_create: chk_ptr/var_ptr must start at 0 and end at E");
  int slots = 0, vslots = 0;
  std::vector<int> edge_chk(E), edge_slot(E);
  for (int c = 0; c < C; ++c) {
    if (chk_ptr[c + 1] < chk_ptr[c]) return fail(RBP_ERR_ARGUMENT, "rbp_graph_create: chk_ptr not monotone");
    slots = std::max(slots, chk_ptr[c + 1] - chk_ptr[c]);
    for (int e = chk_ptr[c]; e < chk_ptr[c + 1]; ++e) {
      edge_chk[e] = c;
      edge_slot[e] = e - chk_ptr[c];
    }
  }
  for (int e = 0; e < E; ++e)
    if (edge_var[e] < 0 || edge_var[e] >= V) return fail(RBP_ERR_ARGUMENT, "rbp_graph_create: edge_var out of range");
  std::vector<int> seen(E, 0);
  for (int v = 0; v < V; ++v) {
    if (var_ptr[v + 1] < var_ptr[v]) return fail(RBP_ERR_ARGUMENT, "rbp_graph_create: var_ptr not monotone");
    vslots = std::max(vslots, var_ptr[v + 1] - var_ptr[v]);
    for (int k = var_ptr[v]; k < var_ptr[v + 1]; ++k) {
      const int e = var_edges[k];
      if (e < 0 || e >= E || edge_var[e] != v || seen[e])
        return fail(RBP_ERR_ARGUMENT,
                    "rbp_graph_create: var_edges is not the variable-major permutation of edge_var");
      seen[e] = 1;
    }
  }
  if (vslots > 8)
    return fail(RBP_ERR_UNSUPPORTED, "rbp_graph_create: variable degree " + std::to_string(vslots) +
                                         " exceeds 8 (edge slots are held in registers)");
  if ((long long)layout_rows(slots, RBP_MSG_F64) * C >= 65535)
    return fail(RBP_ERR_UNSUPPORTED,
                "rbp_graph_create: padded_check_degree * C must be below 65535 message slots; this decoder keeps a "
                "shot's messages in shared memory");
  std::vector<uint8_t> h_chk_deg(C);
  for (int c = 0; c < C; ++c) h_chk_deg[c] = (uint8_t)std::min(255, chk_ptr[c + 1] - chk_ptr[c]);
  DeviceGuard dg(device);
  if (!dg.ok) return fail(RBP_ERR_CUDA, "rbp_graph_create: cannot select the CUDA device");
  rbp_graph* g = new rbp_graph();
  g->device = device;
  g->C = C;
  g->V = V;
  g->E = E;
  g->slots = slots;
  g->vslots = vslots;
  g->edge_chk = std::move(edge_chk);
  g->edge_slot = std::move(edge_slot);
  g->var_ptr.assign(var_ptr, var_ptr + V + 1);
  g->var_edges.assign(var_edges, var_edges + E);
  int rc;
  if ((rc = g->chk_deg.upload(h_chk_deg.data(), C)) || (rc = g->chk_ptr.upload(chk_ptr, (size_t)C + 1))) {
    delete g;
    return rc;
  }
  *out = g;
  return RBP_OK;
}

int rbp_graph_destroy(rbp_graph* g) {
  if (!g) return RBP_OK;
  DeviceGuard dg(g->device);
  delete g;
  return RBP_OK;
}

int rbp_decoder_configure(rbp_decoder* d, int32_t group_threads, int32_t groups_per_block,
                          int32_t shots_per_group) {
  return rbp_decoder_configure_kind(d, RBP_LAUNCH_ALL, group_threads, groups_per_block, shots_per_group, 0);
}

int rbp_decoder_configure_kind(rbp_decoder* d, int32_t kind, int32_t group_threads, int32_t groups_per_block,
                               int32_t shots_per_group, int32_t blocks_per_sm) {
  if (!d) return fail(RBP_ERR_ARGUMENT, "rbp_decoder_configure: null decoder");
  if (kind < RBP_LAUNCH_ALL || kind > RBP_LAUNCH_LEGS)
    return fail(RBP_ERR_ARGUMENT, "rbp_decoder_configure: kind must be RBP_LAUNCH_ALL, _PRE or _LEGS");
  if (blocks_per_sm < 0 || blocks_per_sm > 2)
    return fail(RBP_ERR_ARGUMENT, "rbp_decoder_configure: blocks_per_sm must be 0 (one), 1 or 2");
  const int minb = blocks_per_sm == 2 ? 2 : 1;
  const rbp_graph* g = d->g;
  const int nshots = shots_per_group > 0 ? shots_per_group : 1;
  // groups_per_block 0 (default) or -1: the multi-group kernel with as many one-shot groups
  // per block as fit; 1, or two shots per group: the block-per-group kernel
  if (groups_per_block < 0) {
    if (nshots != 1) return fail(RBP_ERR_ARGUMENT, "rbp_decoder_configure: groups_per_block -1 runs one shot per group");
    groups_per_block = 0;
  }
  const bool block_per_group = nshots == 2 || groups_per_block == 1;
  // default group size within the register budget of the kernel family that runs it
  const int G = group_threads > 0 ? group_threads
                                  : default_group_threads(g->C, g->V, nshots, block_per_group ? g->vslots : 8, minb);
  DeviceGuard dg(g->device);
  Launch lc{};
  const int rc = choose_launch(g->C, g->V, g->slots, g->vslots, d->rows, d->p.msg_type, G, groups_per_block,
                               d->max_smem, d->sm_count, &lc, "rbp_decoder_configure", nshots, minb);
  if (rc != RBP_OK) return rc;
  const Layout L = make_layout(g->C, g->V, d->rows, d->p.msg_type, G, lc.slots_kernel && lc.nshots == 1);
  rbp_decoder::Shape sh;
  sh.kernel = lc.kernel;
  sh.vpt = vpt_for(g->V, G);
  sh.group_threads = lc.group_threads;
  sh.groups = lc.groups;
  sh.blocks = lc.blocks;
  sh.nshots = lc.nshots;
  sh.slots_kernel = lc.slots_kernel;
  sh.minb = lc.minb;
  sh.group_bytes = L.group_bytes;
  sh.block_bytes = L.off_group0;
  if (kind != RBP_LAUNCH_LEGS) d->shape[0] = sh;
  if (kind != RBP_LAUNCH_PRE) d->shape[1] = sh;
  return RBP_OK;
}

int rbp_decoder_create(const rbp_graph* g, const rbp_params* p, const float* llr, const float* gamma_legs,
                       const float* alpha, int32_t n_alpha, rbp_decoder** out) {
  if (!out) return fail(RBP_ERR_ARGUMENT, "rbp_decoder_create: out is null");
  *out = nullptr;
  if (!g || !p || !llr) return fail(RBP_ERR_ARGUMENT, "rbp_decoder_create: null graph, params or llr");
  if (p->pre_iter < 0 || p->num_sets < 0 || p->set_max_iter < 0)
    return fail(RBP_ERR_ARGUMENT, "rbp_decoder_create: iteration counts must be >= 0");
  if (p->msg_type < RBP_MSG_F32 || p->msg_type > RBP_MSG_F64)
    return fail(RBP_ERR_ARGUMENT, "rbp_decoder_create: unknown msg_type");
  if (p->mix_mode < RBP_MIX_SEPARATE || p->mix_mode > RBP_MIX_FMA_LP)
    return fail(RBP_ERR_ARGUMENT, "rbp_decoder_create: unknown mix_mode");
  if (p->num_sets > 0 && !gamma_legs) return fail(RBP_ERR_ARGUMENT, "rbp_decoder_create: gamma_legs is null");
  if (p->use_alpha && (!alpha || n_alpha < std::max(p->pre_iter, p->set_max_iter)))
    return fail(RBP_ERR_ARGUMENT, "rbp_decoder_create: alpha table shorter than max(pre_iter, set_max_iter)");
  DeviceGuard dg(g->device);
  if (!dg.ok) return fail(RBP_ERR_CUDA, "rbp_decoder_create: cannot select the CUDA device");
  rbp_decoder* d = new rbp_decoder();
  d->g = g;
  d->p = *p;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, g->device) != cudaSuccess) {
    delete d;
    return fail(RBP_ERR_CUDA, "rbp_decoder_create: cudaGetDeviceProperties failed");
  }
  d->sm_count = prop.multiProcessorCount;
  d->max_smem = prop.sharedMemPerBlockOptin;
  d->rows = layout_rows(g->slots, p->msg_type);
  if ((long long)d->rows * g->C >= 65535) {
    delete d;
    return fail(RBP_ERR_UNSUPPORTED, "rbp_decoder_create: message layout exceeds 65535 slots");
  }
  {
    std::vector<uint16_t> h_var_pos((size_t)g->vslots * g->V, rbpk::kNoSlot);
    for (int v = 0; v < g->V; ++v)
      for (int k = g->var_ptr[v]; k < g->var_ptr[v + 1]; ++k) {
        const int e = g->var_edges[k];
        h_var_pos[(size_t)(k - g->var_ptr[v]) * g->V + v] =
            (uint16_t)slot_index_host(g->edge_slot[e], g->edge_chk[e], g->C, p->msg_type);
      }
    int rc0;
    if ((rc0 = d->var_pos.upload(h_var_pos.data(), h_var_pos.size()))) {
      delete d;
      return rc0;
    }
  }
  std::vector<float> a_host;
  if (p->use_alpha) a_host.assign(alpha, alpha + n_alpha);
  else a_host.assign(1, 1.0f);
  d->n_alpha = (int)a_host.size();
  int zero = 0, rc;
  if ((rc = d->gamma_legs.upload(gamma_legs, (size_t)p->num_sets * g->V)) ||
      (rc = d->alpha.upload(a_host.data(), a_host.size())) || (rc = d->queue.upload(&zero, 1)) ||
      (rc = rbp_decoder_set_llr(d, llr)) || (rc = rbp_decoder_configure(d, 0, 0, 0))) {
    delete d;
    return rc;
  }
  *out = d;
  return RBP_OK;
}

int rbp_decoder_set_llr(rbp_decoder* d, const float* llr) {
  if (!d || !llr) return fail(RBP_ERR_ARGUMENT, "rbp_decoder_set_llr: null argument");
  const int V = d->g->V;
  DeviceGuard dg(d->g->device);
  return d->llr.upload(llr, V);
}

int rbp_decoder_destroy(rbp_decoder* d) {
  if (!d) return RBP_OK;
  DeviceGuard dg(d->g->device);
  delete d;
  return RBP_OK;
}

int rbp_state_bytes(const rbp_decoder* d, int64_t* bytes_per_shot) {
  if (!d || !bytes_per_shot) return fail(RBP_ERR_ARGUMENT, "rbp_state_bytes: null argument");
  *bytes_per_shot = rbpk::state_stride(d->g->V, d->p.msg_type == RBP_MSG_F64 ? 8 : 4);
  return RBP_OK;
}

int rbp_state_posterior_offset(const rbp_decoder* d, int64_t* offset) {
  if (!d || !offset) return fail(RBP_ERR_ARGUMENT, "rbp_state_posterior_offset: null argument");
  *offset = rbpk::state_post_offset(d->g->V);
  return RBP_OK;
}

int rbp_decoder_query(const rbp_decoder* d, int64_t* group_smem, int64_t* block_smem, int32_t* group_threads,
                      int32_t* groups_per_block, int32_t* blocks, int32_t* shots_per_group) {
  if (!d) return fail(RBP_ERR_ARGUMENT, "rbp_decoder_query: null decoder");
  if (group_smem) *group_smem = d->shape[1].group_bytes;
  if (block_smem) *block_smem = d->shape[1].block_bytes;
  return rbp_decoder_query_kind(d, RBP_LAUNCH_LEGS, group_threads, groups_per_block, shots_per_group, nullptr,
                                blocks);
}

int rbp_decoder_query_kind(const rbp_decoder* d, int32_t kind, int32_t* group_threads, int32_t* groups_per_block,
                           int32_t* shots_per_group, int32_t* blocks_per_sm, int32_t* blocks) {
  if (!d) return fail(RBP_ERR_ARGUMENT, "rbp_decoder_query: null decoder");
  if (kind != RBP_LAUNCH_PRE && kind != RBP_LAUNCH_LEGS)
    return fail(RBP_ERR_ARGUMENT, "rbp_decoder_query: kind must be RBP_LAUNCH_PRE or RBP_LAUNCH_LEGS");
  const rbp_decoder::Shape& sh = d->shape[kind == RBP_LAUNCH_PRE ? 0 : 1];
  if (group_threads) *group_threads = sh.group_threads;
  if (groups_per_block) *groups_per_block = sh.groups;
  if (shots_per_group) *shots_per_group = sh.nshots;
  if (blocks_per_sm) *blocks_per_sm = sh.minb;
  if (blocks) *blocks = sh.blocks;
  return RBP_OK;
}

int rbp_decode(rbp_decoder* d, int64_t B, const rbp_batch* in, const rbp_outputs* out, void* stream) {
  if (!d || !in || !out) return fail(RBP_ERR_ARGUMENT, "rbp_decode: null argument");
  int rc = check_batch("rbp_decode", B, in, out, d->p, d->n_alpha);
  if (rc != RBP_OK || B == 0) return rc;
  const rbp_graph* g = d->g;
  DeviceGuard dg(g->device);
  if (!dg.ok) return fail(RBP_ERR_CUDA, "rbp_decode: cannot select the CUDA device");
  // a launch that skips the relay legs runs at most pre_iter iterations per shot
  const rbp_decoder::Shape& sh = d->shape[in->skip_relay_legs ? 0 : 1];
  const Layout L = make_layout(g->C, g->V, d->rows, d->p.msg_type, sh.group_threads, sh.slots_kernel && sh.nshots == 1);
  const DevGraph dgph{g->C, g->V, g->E, g->slots, d->rows, g->vslots, g->chk_deg.p, g->chk_ptr.p, d->var_pos.p};
  const Launch lc{sh.kernel, sh.group_threads, sh.groups, sh.blocks, sh.nshots, sh.slots_kernel, sh.minb};
  return launch_decode(dgph, d->p, L, lc, d->llr.p, d->gamma_legs.p, d->alpha.p, d->queue.p, B, in,
                       out, reinterpret_cast<cudaStream_t>(stream), "rbp_decode");
}

// ------------------------------------------------------------------ mixed-code launch

}  // extern "C"

struct rbp_mixed {
  int n = 0;
  int device = 0;
  const rbp_decoder* dec[rbpk::kMaxMixedCodes] = {};
  int G[rbpk::kMaxMixedCodes] = {}, NG[rbpk::kMaxMixedCodes] = {};
  rbpk::MixedKernelFn kernel = nullptr;
  int vpt = 0;                 // owned variables per thread of the instantiation
  int block_threads = 0, blocks = 0;
  size_t smem = 0;
  DevBuf<int> queues;
  cudaStream_t capture_stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  ~rbp_mixed() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (capture_stream) cudaStreamDestroy(capture_stream);
  }
};

namespace {

// Kernel arguments of one mixed launch.
int mixed_args(rbp_mixed* m, const int64_t* B, const rbp_batch* ins, const rbp_outputs* outs, rbpk::MixedArgs* ma) {
  std::memset(ma, 0, sizeof(*ma));
  ma->ncodes = m->n;
  double work[rbpk::kMaxMixedCodes] = {}, total = 0;
  for (int i = 0; i < m->n; ++i) {
    const rbp_decoder* d = m->dec[i];
    const rbp_graph* g = d->g;
    int rc = check_batch("rbp_mixed_decode", B[i], &ins[i], &outs[i], d->p, d->n_alpha);
    if (rc != RBP_OK) return rc;
    const Layout L = make_layout(g->C, g->V, d->rows, d->p.msg_type, m->G[i]);
    ma->code[i].g = DevGraph{g->C, g->V, g->E, g->slots, d->rows, g->vslots, g->chk_deg.p, g->chk_ptr.p,
                             d->var_pos.p};
    DevArgs& a = ma->code[i].a;
    const rbp_params& p = d->p;
    const rbp_batch* in = &ins[i];
    const rbp_outputs* out = &outs[i];
    a.pre_iter = in->pre_iter;
    a.num_sets = p.num_sets;
    a.set_max_iter = p.set_max_iter;
    a.stop_nconv = p.stop_nconv;
    a.last_leg = p.last_leg;
    a.use_alpha = p.use_alpha;
    a.use_beta = p.use_beta;
    a.mix_mode = p.mix_mode;
    a.skip_legs = in->skip_relay_legs;
    a.beta = p.beta;
    a.gamma0 = in->gamma0;
    a.llr = d->llr.p;
    a.gamma_legs = d->gamma_legs.p;
    a.alpha = d->alpha.p;
    a.B = B[i];
    a.syn = in->syndromes;
    a.llr_shot = in->llr_per_shot;
    a.gamma_pre = in->gamma_pre;
    a.gamma_legs_shot = in->gamma_legs_shot;
    a.n_shot_legs = in->n_shot_legs;
    a.shot_leg_rows = in->shot_leg_rows > 0 ? in->shot_leg_rows : std::max(1, in->n_shot_legs);
    a.order = in->shot_order;
    a.queue_len = in->queue_len;
    a.solved_gamma = in->solved_gamma;
    a.solved_legs = in->solved_legs;
    a.suspend_unsolved = in->suspend_unsolved;
    a.parity_first = in->parity_first;
    a.init_post = in->init_posterior;
    a.errors = out->errors;
    a.errors_packed = out->errors_packed;
    a.weights = out->weights;
    a.wfixed = reinterpret_cast<long long*>(out->weight_fixed);
    a.found = out->found_count;
    a.iters = out->iterations;
    a.last_post = out->last_posterior;
    a.legs_begin = in->legs_begin;
    a.legs_end = in->legs_end;
    a.resume = static_cast<const unsigned char*>(in->resume_state);
    a.suspend = static_cast<unsigned char*>(in->suspend_state);
    a.state_stride = rbpk::state_stride(g->V, 4);
    a.queue = m->queues.p + i;
    a.group_threads = m->G[i];
    a.groups = m->NG[i];
    a.off_chk_deg = L.off_chk_deg;
    a.off_llr = L.off_llr;
    a.off_first = L.off_first;
    a.first_table = 1;
    a.off_group0 = L.off_group0;
    a.group_bytes = L.group_bytes;
    a.g_msg = L.g_msg;
    a.g_par = L.g_par;
    a.g_best = L.g_best;
    a.g_first = L.g_first;
    a.g_red = L.g_red;
    a.g_s1 = L.g_s1;
    work[i] = (double)B[i] * (double)g->E;
    total += work[i];
  }
  // initial blocks per code in proportion to shots x edges; the kernel rebalances
  double acc = 0;
  for (int i = 0; i < m->n; ++i) {
    ma->first_block[i] = (int)std::lround(total > 0 ? acc / total * m->blocks : 0);
    acc += work[i];
  }
  ma->first_block[m->n] = m->blocks;
  return RBP_OK;
}

int mixed_enqueue(rbp_mixed* m, const rbpk::MixedArgs& ma, cudaStream_t st) {
  RBP_CUDA(cudaMemsetAsync(m->queues.p, 0, sizeof(int) * m->n, st));
  m->kernel<<<m->blocks, m->block_threads, m->smem, st>>>(ma);
  RBP_CUDA(cudaGetLastError());
  return RBP_OK;
}

}  // namespace

extern "C" {

int rbp_mixed_create(const rbp_decoder* const* decoders, int32_t n, rbp_mixed** out) {
  if (!out) return fail(RBP_ERR_ARGUMENT, "rbp_mixed_create: out is null");
  *out = nullptr;
  if (!decoders || n < 1 || n > rbpk::kMaxMixedCodes)
    return fail(RBP_ERR_ARGUMENT, "rbp_mixed_create: between 1 and 8 decoders");
  int vpt_need = 1, dc = 0, dv = 0;
  for (int i = 0; i < n; ++i) {
    const rbp_decoder* d = decoders[i];
    if (!d) return fail(RBP_ERR_ARGUMENT, "rbp_mixed_create: null decoder");
    if (d->p.msg_type != RBP_MSG_F32)
      return fail(RBP_ERR_UNSUPPORTED, "rbp_mixed_create: mixed launches use float32 messages");
    if (d->g->device != decoders[0]->g->device)
      return fail(RBP_ERR_ARGUMENT, "rbp_mixed_create: all decoders must be on one device");
    dc = std::max(dc, d->g->slots);
    dv = std::max(dv, d->g->vslots);
    vpt_need = std::max(vpt_need, vpt_for(d->g->V, std::min(d->shape[1].group_threads, 512)));
  }
  // The vectorised check pass moves MAXDC slots per row (8 or 16), so every
  // code's padded layout must have exactly that many rows; codes whose rows
  // differ cannot share a launch.  Beyond 16 the generic path reads each
  // code's own degrees.
  const int mixed_rows = dc <= 8 ? 8 : (dc <= 16 ? 16 : 0);
  for (int i = 0; i < n && mixed_rows; ++i)
    if (decoders[i]->rows != mixed_rows)
      return fail(RBP_ERR_UNSUPPORTED,
                  "rbp_mixed_create: codes with check degree <= 8 and 9..16 cannot share a launch");
  // One instantiation serves every code: owned variables per thread VPT in
  // {4, 8, 16}; a block of T threads (the register budget of VPT) holds, per
  // code, as many groups as fit with at most VPT variables per thread.
  int vpt = vpt_need <= 4 ? 4 : (vpt_need <= 8 ? 8 : 16);
  rbp_mixed* m = new rbp_mixed();
  m->n = n;
  m->device = decoders[0]->g->device;
  for (int i = 0; i < n; ++i) m->dec[i] = decoders[i];
  DeviceGuard dg(m->device);
  for (;; vpt *= 2) {
    if (vpt > 16) {
      delete m;
      return fail(RBP_ERR_UNSUPPORTED, "rbp_mixed_create: a code needs more than 16 variables per thread");
    }
    const int T = rbpk::max_block_threads(vpt);
    size_t smem = 0;
    bool ok = true;
    for (int i = 0; i < n && ok; ++i) {
      const rbp_decoder* d = decoders[i];
      const rbp_graph* g = d->g;
      int best_G = 0, best_NG = 0;
      for (int k = T / 32; k >= 1; --k) {  // most groups first
        if ((T / k) % 32) continue;
        const int Gc = T / k;
        if (vpt_for(g->V, Gc) < 0 || vpt_for(g->V, Gc) > vpt || (g->C + Gc - 1) / Gc > 32) continue;
        const Layout L = make_layout(g->C, g->V, d->rows, d->p.msg_type, Gc);
        int ng = std::min(k, Gc == 32 ? k : 15);
        while (ng >= 1 && (size_t)L.off_group0 + (size_t)ng * L.group_bytes > d->max_smem) --ng;
        if (ng < 1) continue;
        best_G = Gc;
        best_NG = ng;
        smem = std::max(smem, (size_t)L.off_group0 + (size_t)ng * L.group_bytes);
        break;
      }
      if (!best_G) ok = false;
      m->G[i] = best_G;
      m->NG[i] = best_NG;
    }
    if (!ok) continue;
    m->kernel = rbpk::pick_mixed_f32(dc, dv, vpt);
    if (!m->kernel) {
      delete m;
      return fail(RBP_ERR_UNSUPPORTED, "rbp_mixed_create: no mixed kernel for these degrees");
    }
    m->block_threads = T;
    m->vpt = vpt;
    m->smem = smem;
    break;
  }
  size_t static_smem = 0;
  cudaError_t e = set_max_dynamic_smem(reinterpret_cast<const void*>(m->kernel), decoders[0]->max_smem,
                                       &static_smem);
  if (e == cudaSuccess && m->smem + static_smem > decoders[0]->max_smem) e = cudaErrorInvalidValue;
  int per_sm = 0;
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, m->kernel, m->block_threads, m->smem);
  if (e != cudaSuccess || per_sm < 1) {
    delete m;
    return fail(e != cudaSuccess ? RBP_ERR_CUDA : RBP_ERR_UNSUPPORTED,
                std::string("rbp_mixed_create: occupancy: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "zero"));
  }
  m->blocks = per_sm * decoders[0]->sm_count;
  int rc;
  if ((rc = m->queues.upload(nullptr, n))) {
    delete m;
    return rc;
  }
  *out = m;
  return RBP_OK;
}

int rbp_mixed_destroy(rbp_mixed* m) {
  if (!m) return RBP_OK;
  DeviceGuard dg(m->device);
  delete m;
  return RBP_OK;
}

int rbp_mixed_decode(rbp_mixed* m, const int64_t* B, const rbp_batch* ins, const rbp_outputs* outs, void* stream) {
  if (!m || !B || !ins || !outs) return fail(RBP_ERR_ARGUMENT, "rbp_mixed_decode: null argument");
  DeviceGuard dg(m->device);
  rbpk::MixedArgs ma;
  int rc = mixed_args(m, B, ins, outs, &ma);
  if (rc != RBP_OK) return rc;
  return mixed_enqueue(m, ma, reinterpret_cast<cudaStream_t>(stream));
}

int rbp_mixed_capture(rbp_mixed* m, const int64_t* B, const rbp_batch* ins, const rbp_outputs* outs) {
  if (!m || !B || !ins || !outs) return fail(RBP_ERR_ARGUMENT, "rbp_mixed_capture: null argument");
  DeviceGuard dg(m->device);
  rbpk::MixedArgs ma;
  int rc = mixed_args(m, B, ins, outs, &ma);
  if (rc != RBP_OK) return rc;
  if (!m->capture_stream) RBP_CUDA(cudaStreamCreateWithFlags(&m->capture_stream, cudaStreamNonBlocking));
  if (m->exec) {
    cudaGraphExecDestroy(m->exec);
    m->exec = nullptr;
  }
  if (m->graph) {
    cudaGraphDestroy(m->graph);
    m->graph = nullptr;
  }
  RBP_CUDA(cudaStreamBeginCapture(m->capture_stream, cudaStreamCaptureModeThreadLocal));
  rc = mixed_enqueue(m, ma, m->capture_stream);
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(m->capture_stream, &graph);
  if (rc != RBP_OK) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (e != cudaSuccess) return fail(RBP_ERR_CUDA, std::string("rbp_mixed_capture: ") + cudaGetErrorString(e));
  m->graph = graph;
  RBP_CUDA(cudaGraphInstantiate(&m->exec, m->graph, 0));
  return RBP_OK;
}

int rbp_mixed_replay(rbp_mixed* m, void* stream) {
  if (!m) return fail(RBP_ERR_ARGUMENT, "rbp_mixed_replay: null argument");
  if (!m->exec) return fail(RBP_ERR_ARGUMENT, "rbp_mixed_replay: nothing captured");
  DeviceGuard dg(m->device);
  RBP_CUDA(cudaGraphLaunch(m->exec, reinterpret_cast<cudaStream_t>(stream)));
  return RBP_OK;
}

int rbp_mixed_query(const rbp_mixed* m, int32_t i, int32_t* group_threads, int32_t* groups_per_block,
                    int32_t* block_threads, int32_t* blocks) {
  if (!m || i < 0 || i >= m->n) return fail(RBP_ERR_ARGUMENT, "rbp_mixed_query: bad arguments");
  if (group_threads) *group_threads = m->G[i];
  if (groups_per_block) *groups_per_block = m->NG[i];
  if (block_threads) *block_threads = m->block_threads;
  if (blocks) *blocks = m->blocks;
  return RBP_OK;
}

// Per-code group sizes of a mixed launch (autotuner hook; no reference counterpart).
int rbp_mixed_configure(rbp_mixed* m, const int32_t* group_threads) {
  if (!m || !group_threads) return fail(RBP_ERR_ARGUMENT, "rbp_mixed_configure: null argument");
  const int T = m->block_threads;
  int G[rbpk::kMaxMixedCodes], NG[rbpk::kMaxMixedCodes];
  size_t smem = 0;
  for (int i = 0; i < m->n; ++i) {
    const rbp_decoder* d = m->dec[i];
    const rbp_graph* g = d->g;
    const int Gi = group_threads[i] > 0 ? group_threads[i] : m->G[i];
    if (Gi % 32 || T % Gi)
      return fail(RBP_ERR_ARGUMENT, "rbp_mixed_configure: code " + std::to_string(i) + ": " + std::to_string(Gi) +
                                        " threads must be a multiple of 32 dividing the block's " +
                                        std::to_string(T));
    const int need = vpt_for(g->V, Gi);
    if (need < 0 || need > m->vpt || (g->C + Gi - 1) / Gi > 32)
      return fail(RBP_ERR_UNSUPPORTED, "rbp_mixed_configure: code " + std::to_string(i) + ": " +
                                           std::to_string(Gi) + " threads own more than " + std::to_string(m->vpt) +
                                           " variables or 32 checks each");
    const Layout L = make_layout(g->C, g->V, d->rows, d->p.msg_type, Gi);
    int ng = std::min(T / Gi, Gi == 32 ? T / Gi : 15);
    while (ng >= 1 && (size_t)L.off_group0 + (size_t)ng * L.group_bytes > d->max_smem) --ng;
    if (ng < 1)
      return fail(RBP_ERR_UNSUPPORTED, "rbp_mixed_configure: code " + std::to_string(i) + ": no group fits");
    G[i] = Gi;
    NG[i] = ng;
    smem = std::max(smem, (size_t)L.off_group0 + (size_t)ng * L.group_bytes);
  }
  DeviceGuard dg(m->device);
  int per_sm = 0;
  RBP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, m->kernel, T, smem));
  if (per_sm < 1) return fail(RBP_ERR_UNSUPPORTED, "rbp_mixed_configure: zero occupancy");
  for (int i = 0; i < m->n; ++i) {
    m->G[i] = G[i];
    m->NG[i] = NG[i];
  }
  m->smem = smem;
  m->blocks = per_sm * m->dec[0]->sm_count;
  if (m->exec) {  // a captured graph holds the old shapes
    cudaGraphExecDestroy(m->exec);
    m->exec = nullptr;
  }
  if (m->graph) {
    cudaGraphDestroy(m->graph);
    m->graph = nullptr;
  }
  return RBP_OK;
}

// ------------------------------------------------------------------ decode without allocation

int rbp_decode_static(int32_t C, int32_t V, int32_t E, const int32_t* chk_ptr, const int32_t* edge_var,
                      const int32_t* var_ptr, const int32_t* var_edges, const rbp_params* p, const float* llr,
                      const float* gamma_legs, const float* alpha, int32_t n_alpha, int32_t device, int64_t B,
                      const rbp_batch* in, const rbp_outputs* out, void* stream) {
  const char* who = "rbp_decode_static";
  if (!p || !in || !out || !llr) return fail(RBP_ERR_ARGUMENT, std::string(who) + ": null argument");
  if (C <= 0 || V <= 0 || E <= 0) return fail(RBP_ERR_ARGUMENT, std::string(who) + ": C, V and E must be positive");
  if (!chk_ptr || !edge_var || !var_ptr || !var_edges)
    return fail(RBP_ERR_ARGUMENT, std::string(who) + ": null graph array");
  if (chk_ptr[0] != 0 || chk_ptr[C] != E || var_ptr[0] != 0 || var_ptr[V] != E)
    return fail(RBP_ERR_ARGUMENT, std::string(who) + ": chk_ptr/var_ptr must start at 0 and end at E");
  if (p->msg_type < RBP_MSG_F32 || p->msg_type > RBP_MSG_F64 || p->mix_mode < RBP_MIX_SEPARATE ||
      p->mix_mode > RBP_MIX_FMA_LP || p->pre_iter < 0 || p->num_sets < 0 || p->set_max_iter < 0)
    return fail(RBP_ERR_ARGUMENT, std::string(who) + ": invalid parameters");
  if (p->num_sets > 0 && !gamma_legs) return fail(RBP_ERR_ARGUMENT, std::string(who) + ": gamma_legs is null");
  if (p->use_alpha && (!alpha || n_alpha < std::max(p->pre_iter, p->set_max_iter)))
    return fail(RBP_ERR_ARGUMENT, std::string(who) + ": alpha table shorter than max(pre_iter, set_max_iter)");
  // degrees (no host storage)
  int slots = 0, vslots = 0;
  for (int c = 0; c < C; ++c) {
    if (chk_ptr[c + 1] < chk_ptr[c]) return fail(RBP_ERR_ARGUMENT, std::string(who) + ": chk_ptr not monotone");
    slots = std::max(slots, chk_ptr[c + 1] - chk_ptr[c]);
  }
  for (int v = 0; v < V; ++v) {
    if (var_ptr[v + 1] < var_ptr[v]) return fail(RBP_ERR_ARGUMENT, std::string(who) + ": var_ptr not monotone");
    vslots = std::max(vslots, var_ptr[v + 1] - var_ptr[v]);
  }
  if (vslots > 8) return fail(RBP_ERR_UNSUPPORTED, std::string(who) + ": variable degree exceeds 8");
  const int rows = layout_rows(slots, p->msg_type);
  if ((long long)rows * C >= 65535)
    return fail(RBP_ERR_UNSUPPORTED, std::string(who) + ": message layout exceeds 65535 slots");
  // scratch layout: [counter | chk_deg u8 | chk_ptr i32 | var_pos u16]
  const size_t off_deg = 256;
  const size_t off_ptr = (off_deg + (size_t)C + 15) / 16 * 16;
  const size_t off_pos = (off_ptr + 4 * ((size_t)C + 1) + 15) / 16 * 16;
  const size_t need = off_pos + 2 * (size_t)vslots * V;
  if (need > (size_t)RBP_STATIC_SCRATCH_BYTES)
    return fail(RBP_ERR_UNSUPPORTED, std::string(who) + ": graph tables need " + std::to_string(need) +
                                         " bytes of scratch; the static scratch holds " +
                                         std::to_string((long long)RBP_STATIC_SCRATCH_BYTES));
  const int rc0 = check_batch(who, B, in, out, *p, p->use_alpha ? n_alpha : 1);
  if (rc0 != RBP_OK || B == 0) return rc0;
  // var_edges must list every edge once, under its own variable (rbp_graph_create's
  // test).  E <= rows * C < 65535, so a fixed 8 KiB bitmap holds the edges seen.
  {
    uint32_t seen[65536 / 32] = {};
    for (int v = 0; v < V; ++v)
      for (int q = var_ptr[v]; q < var_ptr[v + 1]; ++q) {
        const int e = var_edges[q];
        if (e < 0 || e >= E || edge_var[e] != v || (seen[e >> 5] >> (e & 31)) & 1u)
          return fail(RBP_ERR_ARGUMENT,
                      std::string(who) + ": var_edges is not the variable-major permutation of edge_var");
        seen[e >> 5] |= 1u << (e & 31);
      }
  }
  DeviceGuard dg(device);
  if (!dg.ok) return fail(RBP_ERR_CUDA, std::string(who) + ": cannot select the CUDA device");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  // The tables are copied from host memory that exists only during this call,
  // so a copy recorded into a graph would read freed memory when replayed.
  {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    RBP_CUDA(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone)
      return fail(RBP_ERR_UNSUPPORTED, std::string(who) +
                                           ": the stream is being captured; this call copies its tables from host "
                                           "memory that is gone when a graph replays, so it runs on eager streams only");
  }
  unsigned char* scratch = nullptr;
  int rc = static_scratch(device, &scratch);
  if (rc != RBP_OK) return rc;

  // Tables are staged through a fixed stack buffer; a pageable-memory copy has
  // consumed the buffer when cudaMemcpyAsync returns, so the buffer is reused.
  unsigned char stage[4096];
  size_t fill = 0, at = off_deg;
  auto flush = [&]() -> int {
    if (fill) RBP_CUDA(cudaMemcpyAsync(scratch + at, stage, fill, cudaMemcpyHostToDevice, st));
    at += fill;
    fill = 0;
    return RBP_OK;
  };
  for (int c = 0; c < C; ++c) {
    stage[fill++] = (unsigned char)std::min(255, chk_ptr[c + 1] - chk_ptr[c]);
    if (fill == sizeof(stage) && (rc = flush())) return rc;
  }
  if ((rc = flush())) return rc;
  RBP_CUDA(cudaMemcpyAsync(scratch + off_ptr, chk_ptr, 4 * ((size_t)C + 1), cudaMemcpyHostToDevice, st));
  at = off_pos;
  for (int k = 0; k < vslots; ++k) {
    for (int v = 0; v < V; ++v) {
      uint16_t pos = rbpk::kNoSlot;
      const int q = var_ptr[v] + k;
      if (q < var_ptr[v + 1]) {
        const int e = var_edges[q];  // validated above
        const int c = (int)(std::upper_bound(chk_ptr, chk_ptr + C + 1, e) - chk_ptr) - 1;  // check of edge e
        pos = (uint16_t)slot_index_host(e - chk_ptr[c], c, C, p->msg_type);
      }
      std::memcpy(stage + fill, &pos, 2);
      fill += 2;
      if (fill == sizeof(stage) && (rc = flush())) return rc;
    }
  }
  if ((rc = flush())) return rc;

  int G = default_group_threads(C, V), max_smem = 0, sms = 0;
  RBP_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
  RBP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  Launch lc{};
  if ((rc = choose_launch(C, V, slots, vslots, rows, p->msg_type, G, 0, (size_t)max_smem, sms, &lc, who))) return rc;
  const Layout L = make_layout(C, V, rows, p->msg_type, G);
  const DevGraph dgph{C, V, E, slots, rows, vslots, scratch + off_deg, reinterpret_cast<const int*>(scratch + off_ptr),
                      reinterpret_cast<const uint16_t*>(scratch + off_pos)};
  return launch_decode(dgph, *p, L, lc, llr, gamma_legs, alpha, reinterpret_cast<int*>(scratch), B, in, out,
                       st, who);
}

}  // extern "C"
