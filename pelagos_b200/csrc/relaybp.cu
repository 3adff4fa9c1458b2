// B200-native Relay-BP-S decoder: one persistent kernel + the C ABI of
// include/relaybp.h.
//
// Execution model
// ---------------
// A thread block holds `groups_per_block` independent *groups* of
// `group_threads` threads.  A group decodes one shot at a time, start to
// finish (first phase, relay legs, selection, output), and then takes the
// next shot index from a global atomic work queue, so shots that converge
// early free their group for new work instead of idling until the slowest
// shot of a batch finishes.  Nothing crosses groups except the read-only
// block-wide tables, and there is no host round trip per iteration.
//
// Per-shot state lives in shared memory:
//   msg[slots * C]   edge messages, check-slot-major: edge j of check c sits at
//                    j * C + c, so thread c of a check pass reads its row with
//                    unit stride across the warp (no bank conflicts);
//   hard[slots * C]  per-edge copy of the variable's hard decision, written by
//                    the variable pass, read by the next check pass;
//   post[V]          posterior LLRs (the memory carried between legs);
//   best[W], first[W] bit sets (W = ceil(V/32)) of the best solution and of the
//                    first leg's hard decision.
// A message slot holds mu (variable-to-check) after a variable pass and nu
// (check-to-variable) after a check pass.
//
// Iteration t of a phase (reference: decoder.py:2610-2875):
//   check pass  (c2v min-sum, kernels.py:1052-1215) + parity of iteration t-1
//   variable pass (v2c + memory mix + posterior + hard, kernels.py:1220-1350)
// The parity check / selection / freeze of iteration t-1 (kernels.py:510-847)
// is fused into the check pass of iteration t: the pass reads the per-edge hard
// bytes of its row and a barrier-reduction (bar.red.and) tells the whole group
// whether every check is satisfied.  The nu values such a pass writes after a
// converged iteration are never read (messages restart at every leg).
//
// Numerics follow the reference kernels operation by operation, with one
// rounding per operation (explicit _rn intrinsics; the file is also built with
// --fmad=false).  The memory mix rounding is selectable (mix_mode).  The sum
// of incoming messages follows the graph's var_edges order.  Solution weights
// are exact 64-bit fixed point (2^-32 units).

#include "relaybp.h"

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define RBP_CUDA(expr)                                                                   \
  do {                                                                                    \
    cudaError_t e_ = (expr);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return fail(RBP_ERR_CUDA, std::string(#expr) + " failed: " + cudaGetErrorString(e_)); \
  } while (0)

// Restores the caller's current device on scope exit.
struct DeviceGuard {
  int prev = -1;
  bool ok = false;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) == cudaSuccess && cudaSetDevice(dev) == cudaSuccess) ok = true;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// ------------------------------------------------------------------ message types

template <typename M>
struct MsgT;
template <>
struct MsgT<float> {
  using A = float;
  static __device__ __forceinline__ float ld(float v) { return v; }
  static __device__ __forceinline__ float st(float v) { return v; }
};
template <>
struct MsgT<double> {
  using A = double;
  static __device__ __forceinline__ double ld(double v) { return v; }
  static __device__ __forceinline__ double st(double v) { return v; }
};
template <>
struct MsgT<__half> {
  using A = float;
  static __device__ __forceinline__ float ld(__half v) { return __half2float(v); }
  static __device__ __forceinline__ __half st(float v) { return __float2half_rn(v); }
};
template <>
struct MsgT<__nv_bfloat16> {
  using A = float;
  static __device__ __forceinline__ float ld(__nv_bfloat16 v) { return __bfloat162float(v); }
  static __device__ __forceinline__ __nv_bfloat16 st(float v) { return __float2bfloat16_rn(v); }
};

__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }

// lambda_mixed = (1 - g) * llr + g * posterior   (kernels.py:1309)
template <typename A>
__device__ __forceinline__ A memory_mix(int mode, A g, A l0, A post) {
  A one_m = sub_rn(A(1), g);
  if (mode == RBP_MIX_FMA_GP) return fma_rn(g, post, mul_rn(one_m, l0));
  if (mode == RBP_MIX_FMA_LP) return fma_rn(one_m, l0, mul_rn(g, post));
  return add_rn(mul_rn(one_m, l0), mul_rn(g, post));
}

// Weight of one set bit in units of 2^-32; non-finite priors weigh 0
// (decoder.py:741-753).  w * 2^32 is exact in float; the conversion rounds
// to nearest-even.
__device__ __forceinline__ long long weight_units(float w) {
  if (!isfinite(w)) return 0;
  return __float2ll_rn(w * 4294967296.0f);
}

// ------------------------------------------------------------------ group sync

// Named barrier over the `n` threads of one group.
__device__ __forceinline__ void group_sync(int id, int n) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

// Barrier + AND-reduction of a predicate over the group.
__device__ __forceinline__ bool group_all(int id, int n, bool p) {
  unsigned r;
  asm volatile(
      "{\n\t.reg .pred pi, po;\n\t"
      "setp.ne.u32 pi, %1, 0;\n\t"
      "bar.red.and.pred po, %2, %3, pi;\n\t"
      "selp.u32 %0, 1, 0, po;\n\t}"
      : "=r"(r)
      : "r"((unsigned)p), "r"(id), "r"(n)
      : "memory");
  return r != 0;
}

// ------------------------------------------------------------------ kernel params

struct DevGraph {
  int C, V, E;
  int slots;                 // max check degree: rows of the check-slot layout
  int vslots;                // max variable degree
  const uint16_t* chk_deg;   // [C]
  const uint8_t* var_deg;    // [V]
  const uint16_t* var_pos;   // [vslots, V] slot position of variable v's k-th edge (summation order)
};

struct DevArgs {
  // parameters
  int pre_iter, num_sets, set_max_iter, stop_nconv;
  int last_leg, use_alpha, use_beta, mix_mode, skip_legs;
  float beta, gamma0;
  // tables
  const float* llr;              // [V]
  const long long* wunits;       // [V]
  const float* gamma_legs;       // [num_sets, V]
  const float* alpha;            // [n_alpha]
  // batch inputs
  long long B;
  const uint8_t* syn;            // [B, C]
  const float* llr_shot;         // [B, V] or null
  const float* gamma_pre;        // [B, V] or null
  const float* gamma_legs_shot;  // [B, n_shot_legs, V] or null
  int n_shot_legs;
  const float* init_post;        // [B, V] or null
  // outputs
  uint8_t* errors;
  uint32_t* errors_packed;
  float* weights;
  long long* wfixed;
  int* found;
  int* iters;
  void* last_post;
  // scheduling
  int* queue;
  int group_threads, groups;
  // shared-memory layout (byte offsets)
  int off_chk_deg, off_var_deg, off_var_pos, off_llr, off_group0, group_bytes;
  int g_msg, g_hard, g_post, g_best, g_first, g_red;
};

// Largest thread block the kernel is compiled for (lets it use up to 128 registers).
constexpr int kMaxBlockThreads = 512;

__host__ __device__ inline int align16(int x) { return (x + 15) & ~15; }

enum HardSrc { HARD_ZERO = 0, HARD_POST = 1, HARD_BEST = 2 };

// Shared-memory views and thread coordinates of one group.
template <typename M>
struct GroupCtx {
  using A = typename MsgT<M>::A;
  int C, V, W, G, t, lane, warp, nwarps, bar;
  const uint16_t* chk_deg;
  const uint8_t* var_deg;
  const uint16_t* var_pos;
  const float* llr_shared;
  M* msg;
  uint8_t* hard;
  A* post;
  uint32_t* best_bits;
  uint32_t* first_bits;
  long long* red;
};

// Mutable per-shot bookkeeping (group-uniform: every thread holds a copy).
struct ShotState {
  long long best_w;
  int found, iters, hard_src, sought;
  bool has_best;
};

template <typename M>
__device__ __forceinline__ typename MsgT<M>::A llr_of(const GroupCtx<M>& x, const float* llr_row, int v) {
  using A = typename MsgT<M>::A;
  return llr_row ? A(__ldg(llr_row + v)) : A(x.llr_shared[v]);
}

// Bit set of the current hard decision (as selected by hard_src) into dst.
template <typename M>
__device__ __forceinline__ void snapshot_hard(const GroupCtx<M>& x, const ShotState& st, uint32_t* dst) {
  using A = typename MsgT<M>::A;
  group_sync(x.bar, x.G);
  if (st.hard_src == HARD_POST) {
    for (int v0 = x.warp * 32; v0 < x.V; v0 += x.G) {
      const int v = v0 + x.lane;
      const unsigned m = __ballot_sync(0xffffffffu, v < x.V && x.post[v] <= A(0));
      if (x.lane == 0) dst[v0 >> 5] = m;
    }
  } else if (st.hard_src == HARD_BEST) {
    for (int w = x.t; w < x.W; w += x.G) dst[w] = x.best_bits[w];
  } else {
    for (int w = x.t; w < x.W; w += x.G) dst[w] = 0u;
  }
  group_sync(x.bar, x.G);
}

// One decoding phase (the pre-iterations or one relay leg): message init, then
// up to max_iter iterations, each followed by parity / selection / freeze.
// grow: per-variable memory strengths of this phase (null: the scalar gs).
template <typename M, int MAXDC, int MAXDV>
__device__ __forceinline__ void run_phase(const GroupCtx<M>& x, const DevArgs& a, ShotState& st,
                                          unsigned long long synm, const float* llr_row,
                                          int max_iter, const float* grow, float gs) {
  using IO = MsgT<M>;
  using A = typename IO::A;
  const int C = x.C, V = x.V, G = x.G, t = x.t;
  const int S = a.stop_nconv;
  if (max_iter <= 0) {
    // freeze_finished_lanes_kernel(count_iteration=False) after an empty phase
    if (st.found >= min(st.sought, S)) st.hard_src = HARD_BEST;
    return;
  }
  // message init: mu_e = llr[var(e)]  (kernels.py:904-1000)
  for (int v = t; v < V; v += G) {
    const M m0 = IO::st(llr_of(x, llr_row, v));
    const int dv = x.var_deg[v];
    for (int k = 0; k < dv; ++k) x.msg[x.var_pos[k * V + v]] = m0;
  }
  group_sync(x.bar, G);
  int valid = 0;
  for (int it = 0; it <= max_iter; ++it) {
    const bool check_parity = it > 0;
    const bool write_nu = it < max_iter;
    const A alpha = (a.use_alpha && write_nu) ? A(__ldg(a.alpha + it)) : A(1);
    const A beta = A(a.beta);

    // ---------------- check pass (kernels.py:1052-1215) + parity of it-1 (kernels.py:510-569)
    bool ok_all = true;
    int k = 0;
    for (int c = t; c < C; c += G, ++k) {
      const int deg = x.chk_deg[c];
      const int s = (int)((synm >> k) & 1ull);
      int hp = 0, neg = 0, cnt1 = 0;
      A min1 = A(1e30), min2 = A(1e30);
      if constexpr (MAXDC > 0) {
        A mv[MAXDC];
#pragma unroll
        for (int j = 0; j < MAXDC; ++j) {
          if (j < deg) {
            const A m = IO::ld(x.msg[j * C + c]);
            mv[j] = m;
            if (check_parity) hp ^= x.hard[j * C + c];
            neg ^= (m < A(0)) ? 1 : 0;
            const A am = fabs(m);
            if (am < min1) { min2 = min1; min1 = am; cnt1 = 1; }
            else if (am == min1) { cnt1 += 1; }
            else if (am < min2) { min2 = am; }
          }
        }
        if (check_parity) ok_all = ok_all && ((hp & 1) == s);
        if (write_nu) {
          const int par = (neg ^ s) & 1;
#pragma unroll
          for (int j = 0; j < MAXDC; ++j) {
            if (j < deg) {
              const A m = mv[j];
              const A am = fabs(m);
              A mag = (cnt1 == 1 && am == min1) ? min2 : min1;
              if (deg == 1) mag = A(0);
              if (a.use_alpha) mag = mul_rn(alpha, mag);
              if (a.use_beta) mag = fmax(sub_rn(mag, beta), A(0));
              const bool flip = (par != 0) != !(m >= A(0));
              x.msg[j * C + c] = IO::st(flip ? -mag : mag);
            }
          }
        }
      } else {
        for (int j = 0; j < deg; ++j) {
          const A m = IO::ld(x.msg[j * C + c]);
          if (check_parity) hp ^= x.hard[j * C + c];
          neg ^= (m < A(0)) ? 1 : 0;
          const A am = fabs(m);
          if (am < min1) { min2 = min1; min1 = am; cnt1 = 1; }
          else if (am == min1) { cnt1 += 1; }
          else if (am < min2) { min2 = am; }
        }
        if (check_parity) ok_all = ok_all && ((hp & 1) == s);
        if (write_nu) {
          const int par = (neg ^ s) & 1;
          for (int j = 0; j < deg; ++j) {
            const A m = IO::ld(x.msg[j * C + c]);
            const A am = fabs(m);
            A mag = (cnt1 == 1 && am == min1) ? min2 : min1;
            if (deg == 1) mag = A(0);
            if (a.use_alpha) mag = mul_rn(alpha, mag);
            if (a.use_beta) mag = fmax(sub_rn(mag, beta), A(0));
            const bool flip = (par != 0) != !(m >= A(0));
            x.msg[j * C + c] = IO::st(flip ? -mag : mag);
          }
        }
      }
    }
    const bool all_ok = group_all(x.bar, G, ok_all);

    if (check_parity) {
      // check_and_select_kernel (kernels.py:609-741) for iteration it-1
      if (all_ok) {
        long long w = 0;
        for (int v = t; v < V; v += G) {
          if (x.post[v] <= A(0))
            w += llr_row ? weight_units(__ldg(llr_row + v)) : __ldg(a.wunits + v);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
        if (x.lane == 0) x.red[x.warp] = w;
        group_sync(x.bar, G);
        long long tot = 0;
        for (int i = 0; i < x.nwarps; ++i) tot += x.red[i];
        if (!st.has_best || tot < st.best_w) {
          st.best_w = tot;
          st.has_best = true;
          for (int v0 = x.warp * 32; v0 < V; v0 += G) {
            const int v = v0 + x.lane;
            const unsigned m = __ballot_sync(0xffffffffu, v < V && x.post[v] <= A(0));
            if (x.lane == 0) x.best_bits[v0 >> 5] = m;
          }
        }
        if (valid == 0) st.found += 1;
        valid = 1;
      }
      // freeze_finished_lanes_kernel (kernels.py:746-847): the iteration is counted
      if (st.found >= min(st.sought, S)) {
        st.iters += it;
        st.hard_src = HARD_BEST;
        group_sync(x.bar, G);  // best_bits / red settled before reuse
        return;
      }
    }
    if (!write_nu) break;

    // ---------------- variable pass (kernels.py:1220-1350)
    for (int v = t; v < V; v += G) {
      const int dv = x.var_deg[v];
      const A gv = grow ? A(__ldg(grow + v)) : A(gs);
      const A lm = memory_mix<A>(a.mix_mode, gv, llr_of(x, llr_row, v), x.post[v]);
      if constexpr (MAXDV > 0) {
        A nv[MAXDV];
        int pos[MAXDV];
        A sum = A(0);
#pragma unroll
        for (int j = 0; j < MAXDV; ++j) {
          if (j < dv) {
            pos[j] = x.var_pos[j * V + v];
            nv[j] = IO::ld(x.msg[pos[j]]);
            sum = add_rn(sum, nv[j]);
          }
        }
        const A pv = add_rn(lm, sum);
        x.post[v] = pv;
        const uint8_t h = pv <= A(0) ? 1 : 0;
#pragma unroll
        for (int j = 0; j < MAXDV; ++j) {
          if (j < dv) {
            x.msg[pos[j]] = IO::st(add_rn(lm, sub_rn(sum, nv[j])));
            x.hard[pos[j]] = h;
          }
        }
      } else {
        A sum = A(0);
        for (int j = 0; j < dv; ++j) sum = add_rn(sum, IO::ld(x.msg[x.var_pos[j * V + v]]));
        const A pv = add_rn(lm, sum);
        x.post[v] = pv;
        const uint8_t h = pv <= A(0) ? 1 : 0;
        for (int j = 0; j < dv; ++j) {
          const int p = x.var_pos[j * V + v];
          x.msg[p] = IO::st(add_rn(lm, sub_rn(sum, IO::ld(x.msg[p]))));
          x.hard[p] = h;
        }
      }
    }
    st.hard_src = HARD_POST;
    group_sync(x.bar, G);
  }
  st.iters += max_iter;
}

// MAXDC: register-cached check degree bound (0: generic, row reloaded from smem)
// MAXDV: register-cached variable degree bound (0: generic)
template <typename M, int MAXDC, int MAXDV>
__global__ void __launch_bounds__(kMaxBlockThreads) relaybp_decode_kernel(DevGraph g, DevArgs a) {
  using IO = MsgT<M>;
  using A = typename IO::A;
  extern __shared__ __align__(16) unsigned char smem[];

  const int C = g.C, V = g.V;
  uint16_t* s_chk_deg = reinterpret_cast<uint16_t*>(smem + a.off_chk_deg);
  uint8_t* s_var_deg = smem + a.off_var_deg;
  uint16_t* s_var_pos = reinterpret_cast<uint16_t*>(smem + a.off_var_pos);
  float* s_llr = reinterpret_cast<float*>(smem + a.off_llr);

  for (int i = threadIdx.x; i < C; i += blockDim.x) s_chk_deg[i] = g.chk_deg[i];
  for (int i = threadIdx.x; i < V; i += blockDim.x) {
    s_var_deg[i] = g.var_deg[i];
    s_llr[i] = a.llr[i];
  }
  for (int i = threadIdx.x; i < g.vslots * V; i += blockDim.x) s_var_pos[i] = g.var_pos[i];
  __syncthreads();

  GroupCtx<M> x;
  x.C = C;
  x.V = V;
  x.W = (V + 31) >> 5;
  x.G = a.group_threads;
  const int gid = threadIdx.x / x.G;
  if (gid >= a.groups) return;
  x.t = threadIdx.x - gid * x.G;
  x.lane = threadIdx.x & 31;
  x.warp = x.t >> 5;
  x.nwarps = x.G >> 5;
  x.bar = 1 + gid;
  x.chk_deg = s_chk_deg;
  x.var_deg = s_var_deg;
  x.var_pos = s_var_pos;
  x.llr_shared = s_llr;
  unsigned char* gsm = smem + a.off_group0 + gid * a.group_bytes;
  x.msg = reinterpret_cast<M*>(gsm + a.g_msg);
  x.hard = gsm + a.g_hard;
  x.post = reinterpret_cast<A*>(gsm + a.g_post);
  x.best_bits = reinterpret_cast<uint32_t*>(gsm + a.g_best);
  x.first_bits = reinterpret_cast<uint32_t*>(gsm + a.g_first);
  x.red = reinterpret_cast<long long*>(gsm + a.g_red);
  volatile long long* shot_slot = x.red + x.nwarps;
  const int G = x.G, t = x.t, W = x.W;

  while (true) {
    if (t == 0) *shot_slot = (long long)atomicAdd(a.queue, 1);
    group_sync(x.bar, G);
    const long long b = *shot_slot;
    if (b >= a.B) break;

    // ---------------- per-shot setup (decoder.py:3429-3478)
    const uint8_t* syn_row = a.syn + b * (long long)C;
    unsigned long long synm = 0;  // bit k: syndrome of check t + k*G
    {
      int k = 0;
      for (int c = t; c < C; c += G, ++k) synm |= (unsigned long long)(syn_row[c] & 1) << k;
    }
    const float* llr_row = a.llr_shot ? a.llr_shot + b * (long long)V : nullptr;
    for (int v = t; v < V; v += G)
      x.post[v] = a.init_post ? A(__ldg(a.init_post + b * (long long)V + v)) : llr_of(x, llr_row, v);
    for (int w = t; w < W; w += G) {
      x.best_bits[w] = 0u;
      x.first_bits[w] = 0u;
    }
    ShotState st;
    st.best_w = LLONG_MAX;
    st.found = 0;
    st.iters = 0;
    st.hard_src = HARD_ZERO;
    st.sought = 1;
    st.has_best = false;

    // ---------------- first phase (pre-iterations), decoder.py:3480-3616
    const int pre = a.pre_iter;
    run_phase<M, MAXDC, MAXDV>(x, a, st, synm, llr_row, pre,
                               a.gamma_pre ? a.gamma_pre + b * (long long)V : nullptr, a.gamma0);
    if (!a.last_leg) snapshot_hard(x, st, x.first_bits);
    // ---------------- relay legs, decoder.py:3672-3837
    if (!(st.found >= a.stop_nconv || a.skip_legs)) {
      for (int leg = 0; leg < a.num_sets && st.found < a.stop_nconv; ++leg) {
        st.sought = st.found + 1;
        const float* grow = (a.gamma_legs_shot && leg < a.n_shot_legs)
                                ? a.gamma_legs_shot + (b * (long long)a.n_shot_legs + leg) * V
                                : a.gamma_legs + (long long)leg * V;
        run_phase<M, MAXDC, MAXDV>(x, a, st, synm, llr_row, a.set_max_iter, grow, 0.f);
        if (leg == 0 && pre == 0 && !a.last_leg) snapshot_hard(x, st, x.first_bits);
      }
    }

    // ---------------- outputs, decoder.py:3839-3873
    group_sync(x.bar, G);
    const uint32_t* src_bits = st.has_best ? x.best_bits : x.first_bits;
    const bool from_post = !st.has_best && a.last_leg && st.hard_src == HARD_POST;
    const bool zero_bits = !st.has_best && a.last_leg && st.hard_src != HARD_POST;
    if (a.errors) {
      uint8_t* erow = a.errors + b * (long long)V;
      for (int v = t; v < V; v += G) {
        uint8_t e;
        if (from_post) e = x.post[v] <= A(0) ? 1 : 0;
        else if (zero_bits) e = 0;
        else e = (src_bits[v >> 5] >> (v & 31)) & 1u;
        erow[v] = e;
      }
    }
    if (a.errors_packed) {
      uint32_t* prow = a.errors_packed + b * (long long)W;
      for (int v0 = x.warp * 32; v0 < V; v0 += G) {
        const int v = v0 + x.lane;
        unsigned m;
        if (from_post) m = __ballot_sync(0xffffffffu, v < V && x.post[v] <= A(0));
        else if (zero_bits) m = 0u;
        else m = src_bits[v0 >> 5];
        if (x.lane == 0) prow[v0 >> 5] = m;
      }
    }
    if (a.last_post) {
      if constexpr (sizeof(A) == 8) {
        double* lp = reinterpret_cast<double*>(a.last_post) + b * (long long)V;
        for (int v = t; v < V; v += G) lp[v] = (double)x.post[v];
      } else {
        float* lp = reinterpret_cast<float*>(a.last_post) + b * (long long)V;
        for (int v = t; v < V; v += G) lp[v] = (float)x.post[v];
      }
    }
    if (t == 0) {
      if (a.weights)
        a.weights[b] = st.has_best ? __ll2float_rn(st.best_w) * 2.3283064365386963e-10f  // 2^-32
                                   : __int_as_float(0x7f800000);
      if (a.wfixed) a.wfixed[b] = st.has_best ? st.best_w : LLONG_MAX;
      a.found[b] = st.found;
      a.iters[b] = st.iters;
    }
    group_sync(x.bar, G);
  }
}

// ------------------------------------------------------------------ host objects

template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  int upload(const T* host, size_t count) {
    if (p) { cudaFree(p); p = nullptr; }
    n = count;
    if (count == 0) return RBP_OK;
    RBP_CUDA(cudaMalloc(&p, count * sizeof(T)));
    if (host) RBP_CUDA(cudaMemcpy(p, host, count * sizeof(T), cudaMemcpyHostToDevice));
    return RBP_OK;
  }
};

}  // namespace

struct rbp_graph {
  int device = 0;
  int C = 0, V = 0, E = 0, slots = 0, vslots = 0;
  DevBuf<uint16_t> chk_deg;
  DevBuf<uint8_t> var_deg;
  DevBuf<uint16_t> var_pos;
};

struct rbp_decoder {
  const rbp_graph* g = nullptr;
  rbp_params p{};
  DevBuf<float> llr;
  DevBuf<long long> wunits;
  DevBuf<float> gamma_legs;
  DevBuf<float> alpha;
  DevBuf<int> queue;
  int n_alpha = 0;
  int group_threads = 0, groups = 0, blocks = 0;
  int group_bytes = 0, block_bytes = 0;
  int sm_count = 0;
  size_t max_smem = 0;
};

namespace {

size_t msg_size(int t) { return t == RBP_MSG_F64 ? 8 : (t == RBP_MSG_F32 ? 4 : 2); }
size_t acc_size(int t) { return t == RBP_MSG_F64 ? 8 : 4; }

struct Layout {
  int off_chk_deg, off_var_deg, off_var_pos, off_llr, off_group0;
  int g_msg, g_hard, g_post, g_best, g_first, g_red, group_bytes;
};

Layout make_layout(const rbp_graph* g, int msg_type, int group_threads) {
  Layout L{};
  int o = 0;
  L.off_chk_deg = o; o = align16(o + 2 * g->C);
  L.off_var_deg = o; o = align16(o + g->V);
  L.off_var_pos = o; o = align16(o + 2 * g->vslots * g->V);
  L.off_llr = o; o = align16(o + 4 * g->V);
  L.off_group0 = o;
  const int slots_total = g->slots * g->C;
  const int W = (g->V + 31) / 32;
  int q = 0;
  L.g_msg = q; q = align16(q + (int)msg_size(msg_type) * slots_total);
  L.g_hard = q; q = align16(q + slots_total);
  L.g_post = q; q = align16(q + (int)acc_size(msg_type) * g->V);
  L.g_best = q; q = align16(q + 4 * W);
  L.g_first = q; q = align16(q + 4 * W);
  L.g_red = q; q = align16(q + 8 * (group_threads / 32 + 1));
  L.group_bytes = q;
  return L;
}

using KernelFn = void (*)(DevGraph, DevArgs);

template <typename M>
KernelFn pick_kernel_m(int dc, int dv) {
  if (dc <= 8) return dv <= 4 ? relaybp_decode_kernel<M, 8, 4> : relaybp_decode_kernel<M, 8, 0>;
  if (dc <= 16) return dv <= 4 ? relaybp_decode_kernel<M, 16, 4> : relaybp_decode_kernel<M, 16, 0>;
  return dv <= 4 ? relaybp_decode_kernel<M, 0, 4> : relaybp_decode_kernel<M, 0, 0>;
}

KernelFn pick_kernel(int msg_type, int dc, int dv) {
  switch (msg_type) {
    case RBP_MSG_F32: return pick_kernel_m<float>(dc, dv);
    case RBP_MSG_F16: return pick_kernel_m<__half>(dc, dv);
    case RBP_MSG_BF16: return pick_kernel_m<__nv_bfloat16>(dc, dv);
    case RBP_MSG_F64: return pick_kernel_m<double>(dc, dv);
    default: return nullptr;
  }
}

int default_group_threads(const rbp_graph* g) {
  int n = std::max(g->C, g->V);
  if (n <= 128) return 32;
  if (n <= 512) return 64;
  if (n <= 1024) return 128;
  return 256;
}

}  // namespace

extern "C" {

const char* rbp_last_error(void) { return g_err.c_str(); }

const char* rbp_version(void) { return "relaybp-b200 0.1 (sm_100a)"; }

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
      int e = var_edges[k];
      if (e < 0 || e >= E || edge_var[e] != v || seen[e])
        return fail(RBP_ERR_ARGUMENT, "rbp_graph_create: var_edges is not the variable-major permutation of edge_var");
      seen[e] = 1;
    }
  }
  if (slots > 65535 || vslots > 255)
    return fail(RBP_ERR_UNSUPPORTED, "rbp_graph_create: check degree > 65535 or variable degree > 255");
  if ((long long)slots * C > 65535)
    return fail(RBP_ERR_UNSUPPORTED,
                "rbp_graph_create: max_check_degree * C exceeds 65535 message slots; this decoder keeps a shot's "
                "messages in shared memory");
  std::vector<uint16_t> h_chk_deg(C);
  for (int c = 0; c < C; ++c) h_chk_deg[c] = (uint16_t)(chk_ptr[c + 1] - chk_ptr[c]);
  std::vector<uint8_t> h_var_deg(V);
  std::vector<uint16_t> h_var_pos((size_t)vslots * V, 0);
  for (int v = 0; v < V; ++v) {
    h_var_deg[v] = (uint8_t)(var_ptr[v + 1] - var_ptr[v]);
    for (int k = var_ptr[v]; k < var_ptr[v + 1]; ++k) {
      int e = var_edges[k];
      h_var_pos[(size_t)(k - var_ptr[v]) * V + v] = (uint16_t)(edge_slot[e] * C + edge_chk[e]);
    }
  }
  DeviceGuard dg(device);
  if (!dg.ok) return fail(RBP_ERR_CUDA, "rbp_graph_create: cannot select the CUDA device");
  rbp_graph* g = new rbp_graph();
  g->device = device;
  g->C = C; g->V = V; g->E = E; g->slots = slots; g->vslots = vslots;
  int rc;
  if ((rc = g->chk_deg.upload(h_chk_deg.data(), C)) || (rc = g->var_deg.upload(h_var_deg.data(), V)) ||
      (rc = g->var_pos.upload(h_var_pos.data(), h_var_pos.size()))) {
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

int rbp_decoder_configure(rbp_decoder* d, int32_t group_threads, int32_t groups_per_block) {
  if (!d) return fail(RBP_ERR_ARGUMENT, "rbp_decoder_configure: null decoder");
  const rbp_graph* g = d->g;
  int G = group_threads > 0 ? group_threads : default_group_threads(g);
  if (G % 32 != 0 || G > kMaxBlockThreads)
    return fail(RBP_ERR_ARGUMENT, "rbp_decoder_configure: group_threads must be a multiple of 32, at most " +
                                      std::to_string(kMaxBlockThreads));
  if ((g->C + G - 1) / G > 64)
    return fail(RBP_ERR_UNSUPPORTED, "rbp_decoder_configure: more than 64 checks per thread; use more group threads");
  Layout L = make_layout(g, d->p.msg_type, G);
  size_t block_fixed = (size_t)L.off_group0;
  if (block_fixed + L.group_bytes > d->max_smem)
    return fail(RBP_ERR_UNSUPPORTED, "rbp_decoder_configure: one shot's state (" + std::to_string(L.group_bytes) +
                                         " B) does not fit in shared memory");
  int max_groups = (int)((d->max_smem - block_fixed) / L.group_bytes);
  max_groups = std::min(max_groups, kMaxBlockThreads / G);
  max_groups = std::min(max_groups, 15);  // named barriers 1..15
  int NG = groups_per_block > 0 ? groups_per_block : max_groups;
  if (NG < 1 || NG > max_groups)
    return fail(RBP_ERR_UNSUPPORTED, "rbp_decoder_configure: groups_per_block must be in [1, " +
                                         std::to_string(max_groups) + "] for this shape");
  KernelFn k = pick_kernel(d->p.msg_type, g->slots, g->vslots);
  if (!k) return fail(RBP_ERR_ARGUMENT, "rbp_decoder_configure: unknown msg_type");
  DeviceGuard dg(g->device);
  size_t smem = block_fixed + (size_t)NG * L.group_bytes;
  // The attribute is per kernel function and shared by every decoder using this
  // instantiation, so it is set to the device limit; occupancy uses `smem`.
  RBP_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)d->max_smem));
  int per_sm = 0;
  RBP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, G * NG, smem));
  if (per_sm < 1) return fail(RBP_ERR_UNSUPPORTED, "rbp_decoder_configure: launch shape has zero occupancy");
  d->group_threads = G;
  d->groups = NG;
  d->blocks = per_sm * d->sm_count;
  d->group_bytes = L.group_bytes;
  d->block_bytes = (int)block_fixed;
  return RBP_OK;
}

int rbp_decoder_create(const rbp_graph* g, const rbp_params* p, const float* llr,
                       const float* gamma_legs, const float* alpha, int32_t n_alpha,
                       rbp_decoder** out) {
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
  int rc;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, g->device) != cudaSuccess) {
    delete d;
    return fail(RBP_ERR_CUDA, "rbp_decoder_create: cudaGetDeviceProperties failed");
  }
  d->sm_count = prop.multiProcessorCount;
  d->max_smem = prop.sharedMemPerBlockOptin;
  std::vector<float> a_host;
  if (p->use_alpha) a_host.assign(alpha, alpha + n_alpha);
  else a_host.assign(1, 1.0f);
  d->n_alpha = (int)a_host.size();
  int zero = 0;
  if ((rc = d->gamma_legs.upload(gamma_legs, (size_t)p->num_sets * g->V)) ||
      (rc = d->alpha.upload(a_host.data(), a_host.size())) || (rc = d->queue.upload(&zero, 1)) ||
      (rc = rbp_decoder_set_llr(d, llr)) || (rc = rbp_decoder_configure(d, 0, 0))) {
    delete d;
    return rc;
  }
  *out = d;
  return RBP_OK;
}

int rbp_decoder_set_llr(rbp_decoder* d, const float* llr) {
  if (!d || !llr) return fail(RBP_ERR_ARGUMENT, "rbp_decoder_set_llr: null argument");
  const int V = d->g->V;
  std::vector<long long> w(V);
  for (int v = 0; v < V; ++v)
    w[v] = std::isfinite(llr[v]) ? (long long)std::llrint(std::ldexp((double)llr[v], 32)) : 0;
  DeviceGuard dg(d->g->device);
  int rc;
  if ((rc = d->llr.upload(llr, V)) || (rc = d->wunits.upload(w.data(), V))) return rc;
  return RBP_OK;
}

int rbp_decoder_destroy(rbp_decoder* d) {
  if (!d) return RBP_OK;
  DeviceGuard dg(d->g->device);
  delete d;
  return RBP_OK;
}

int rbp_decoder_query(const rbp_decoder* d, int64_t* group_smem, int64_t* block_smem,
                      int32_t* group_threads, int32_t* groups_per_block, int32_t* blocks) {
  if (!d) return fail(RBP_ERR_ARGUMENT, "rbp_decoder_query: null decoder");
  if (group_smem) *group_smem = d->group_bytes;
  if (block_smem) *block_smem = d->block_bytes;
  if (group_threads) *group_threads = d->group_threads;
  if (groups_per_block) *groups_per_block = d->groups;
  if (blocks) *blocks = d->blocks;
  return RBP_OK;
}

int rbp_decode(rbp_decoder* d, int64_t B, const rbp_batch* in, const rbp_outputs* out, void* stream) {
  if (!d || !in || !out) return fail(RBP_ERR_ARGUMENT, "rbp_decode: null argument");
  if (B < 0) return fail(RBP_ERR_ARGUMENT, "rbp_decode: negative batch");
  if (B == 0) return RBP_OK;
  if (B > INT_MAX) return fail(RBP_ERR_UNSUPPORTED, "rbp_decode: batch exceeds 2^31-1 shots");
  if (!in->syndromes || !out->found_count || !out->iterations)
    return fail(RBP_ERR_ARGUMENT, "rbp_decode: syndromes, found_count and iterations are required");
  if (in->pre_iter < 0) return fail(RBP_ERR_ARGUMENT, "rbp_decode: pre_iter must be >= 0");
  if (d->p.use_alpha && in->pre_iter > d->n_alpha)
    return fail(RBP_ERR_ARGUMENT, "rbp_decode: pre_iter exceeds the alpha table");
  if (in->n_shot_legs < 0 || (in->n_shot_legs > 0 && !in->gamma_legs_shot))
    return fail(RBP_ERR_ARGUMENT, "rbp_decode: gamma_legs_shot missing");
  const rbp_graph* g = d->g;
  DeviceGuard dg(g->device);
  if (!dg.ok) return fail(RBP_ERR_CUDA, "rbp_decode: cannot select the CUDA device");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  Layout L = make_layout(g, d->p.msg_type, d->group_threads);

  DevGraph dgph{g->C, g->V, g->E, g->slots, g->vslots, g->chk_deg.p, g->var_deg.p, g->var_pos.p};
  DevArgs a{};
  a.pre_iter = in->pre_iter;
  a.num_sets = d->p.num_sets;
  a.set_max_iter = d->p.set_max_iter;
  a.stop_nconv = d->p.stop_nconv;
  a.last_leg = d->p.last_leg;
  a.use_alpha = d->p.use_alpha;
  a.use_beta = d->p.use_beta;
  a.mix_mode = d->p.mix_mode;
  a.skip_legs = in->skip_relay_legs;
  a.beta = d->p.beta;
  a.gamma0 = in->gamma0;
  a.llr = d->llr.p;
  a.wunits = d->wunits.p;
  a.gamma_legs = d->gamma_legs.p;
  a.alpha = d->alpha.p;
  a.B = B;
  a.syn = in->syndromes;
  a.llr_shot = in->llr_per_shot;
  a.gamma_pre = in->gamma_pre;
  a.gamma_legs_shot = in->gamma_legs_shot;
  a.n_shot_legs = in->n_shot_legs;
  a.init_post = in->init_posterior;
  a.errors = out->errors;
  a.errors_packed = out->errors_packed;
  a.weights = out->weights;
  a.wfixed = reinterpret_cast<long long*>(out->weight_fixed);
  a.found = out->found_count;
  a.iters = out->iterations;
  a.last_post = out->last_posterior;
  a.queue = d->queue.p;
  a.group_threads = d->group_threads;
  a.groups = d->groups;
  a.off_chk_deg = L.off_chk_deg;
  a.off_var_deg = L.off_var_deg;
  a.off_var_pos = L.off_var_pos;
  a.off_llr = L.off_llr;
  a.off_group0 = L.off_group0;
  a.group_bytes = L.group_bytes;
  a.g_msg = L.g_msg;
  a.g_hard = L.g_hard;
  a.g_post = L.g_post;
  a.g_best = L.g_best;
  a.g_first = L.g_first;
  a.g_red = L.g_red;

  KernelFn k = pick_kernel(d->p.msg_type, g->slots, g->vslots);
  const long long need_blocks = (B + d->groups - 1) / d->groups;
  const int blocks = (int)std::min<long long>(d->blocks, need_blocks);
  const size_t smem = (size_t)L.off_group0 + (size_t)d->groups * L.group_bytes;
  RBP_CUDA(cudaMemsetAsync(d->queue.p, 0, sizeof(int), st));
  k<<<blocks, d->group_threads * d->groups, smem, st>>>(dgph, a);
  RBP_CUDA(cudaGetLastError());
  return RBP_OK;
}

}  // extern "C"
