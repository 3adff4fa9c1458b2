// Device code of the Relay-BP-S decode kernel (sm_100a).  Instantiated per
// message type by relaybp_inst_*.cu; launched by relaybp.cu (the C ABI).
//
// Execution model
// ---------------
// A thread block holds `groups` independent groups of `group_threads` (G)
// threads.  A group decodes one shot at a time, start to finish (first phase,
// relay legs, selection, outputs), then takes the next shot index from a
// global atomic work queue: shots that converge early free their group for new
// work instead of waiting for the slowest shot of a batch.  Groups share only
// read-only tables; there is no host round trip per iteration.
//
// Ownership
// ---------
// Thread t of a group owns variables v = t + k*G (k < VPT) and checks
// c = t + k*G (k < ceil(C/G)).  Everything per variable stays in that thread's
// registers for the whole kernel: the slot positions of its edges (loaded once
// per kernel), its posterior (carried across legs: the memory), and the leg's
// memory strength.  Shared memory per group holds only the edge messages, one
// parity bit per check, and two bit sets.
//
//   msg[rows * C + 1]  edge messages; the slots of check c sit in 16-byte
//                    chunks (see slot_index), so a check pass moves a row with
//                    128-bit loads/stores and a warp covers contiguous memory
//                    (no bank conflicts).  A slot holds mu after a variable pass
//                    and nu after a check pass.  The last slot is a dummy that
//                    absent variable edges point at.
//   par[ceil(C/32)]  parity of each check's current hard decisions.  Every
//                    hard decision starts at 0 with a shot; when the variable
//                    pass flips one it XORs (shared atomic) the bits of that
//                    variable's checks, so the bit equals the check's parity.
//   best[W], first[W] bit sets (W = ceil(V/32)): best solution, first-leg hard
//                    decision.
//
// Iteration t of a phase (reference: decoder.py:2610-2875):
//   check pass    (c2v min-sum, kernels.py:1052-1215) + parity of iteration t-1
//   variable pass (v2c + memory mix + posterior + hard, kernels.py:1220-1350)
// The parity / selection / freeze of iteration t-1 (kernels.py:510-847) comes
// before the check pass of iteration t: each check compares its parity bit with
// its syndrome bit and a barrier reduction (bar.red.and) tells the whole group
// whether all checks hold; the min-sum pass runs only if one fails.
//
// Numerics follow the reference kernels operation by operation with one
// rounding per operation (explicit _rn intrinsics; built with --fmad=false);
// the memory-mix rounding is selectable.  Incoming messages are summed in the
// graph's var_edges order.  Solution weights are exact 64-bit fixed point.

#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>

#include "relaybp.h"

namespace rbpk {

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
// float16 messages saturate at the largest finite value (+-65504) before
// rounding: posteriors with memory grow past float16's range on hard shots,
// and an infinite message would turn the variable pass's inf - inf into NaN.
__device__ __forceinline__ __half f16_saturate(float v) {
  return __float2half_rn(fminf(fmaxf(v, -65504.0f), 65504.0f));
}
template <>
struct MsgT<__half> {
  using A = float;
  static __device__ __forceinline__ float ld(__half v) { return __half2float(v); }
  static __device__ __forceinline__ __half st(float v) { return f16_saturate(v); }
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
  const A one_m = sub_rn(A(1), g);
  if (mode == RBP_MIX_FMA_GP) return fma_rn(g, post, mul_rn(one_m, l0));
  if (mode == RBP_MIX_FMA_LP) return fma_rn(one_m, l0, mul_rn(g, post));
  return add_rn(mul_rn(one_m, l0), mul_rn(g, post));
}

// Weight of one set bit in units of 2^-32; non-finite priors weigh 0
// (decoder.py:741-753).  w * 2^32 is exact in float; rounding to nearest-even.
__device__ __forceinline__ long long weight_units(float w) {
  if (!isfinite(w)) return 0;
  return __float2ll_rn(w * 4294967296.0f);
}

// ------------------------------------------------------------------ group sync

// Barrier over one group: a warp-level sync for 32-thread groups, otherwise a
// named barrier (id 1 + group index) over the group's threads.
__device__ __forceinline__ void group_sync(int id, int n) {
  if (n == 32) {
    __syncwarp();
  } else {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
  }
}

// Barrier + OR-reduction of a predicate over the group.
__device__ __forceinline__ bool group_any(int id, int n, bool p) {
  if (n == 32) return __any_sync(0xffffffffu, p);
  unsigned r;
  asm volatile(
      "{\n\t.reg .pred pi, po;\n\t"
      "setp.ne.u32 pi, %1, 0;\n\t"
      "bar.red.or.pred po, %2, %3, pi;\n\t"
      "selp.u32 %0, 1, 0, po;\n\t}"
      : "=r"(r)
      : "r"((unsigned)p), "r"(id), "r"(n)
      : "memory");
  return r != 0;
}

// Barrier + AND-reduction of a predicate over the group.
__device__ __forceinline__ bool group_all(int id, int n, bool p) {
  if (n == 32) return __all_sync(0xffffffffu, p);
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

// ------------------------------------------------------------------ parameters

struct DevGraph {
  int C, V, E;
  int slots;                 // max check degree
  int rows;                  // slot rows of the layout (padded to MAXDC and to whole 16-byte chunks)
  int vslots;                // max variable degree (<= MAXDV of the instantiation)
  const uint8_t* chk_deg;    // [C] (degrees > 255 use the generic check path, which reads chk_ptr)
  const int* chk_ptr;        // [C+1]
  const uint16_t* var_pos;   // [vslots, V] slot position of variable v's k-th edge (summation order),
                             // kNoSlot where v has fewer edges
};

struct DevArgs {
  // parameters
  int pre_iter, num_sets, set_max_iter, stop_nconv;
  int last_leg, use_alpha, use_beta, mix_mode, skip_legs;
  float beta, gamma0;
  // tables
  const float* llr;              // [V]
  const float* gamma_legs;       // [num_sets, V]
  const float* alpha;            // [n_alpha]
  // batch inputs
  long long B;
  const uint8_t* syn;            // [B, C]
  const float* llr_shot;         // [B, V] or null
  const float* gamma_pre;        // [B, V] or null
  const float* gamma_legs_shot;  // [B, shot_leg_rows, V] or null
  int n_shot_legs;
  int shot_leg_rows;             // >= 1; leg l uses row min(l, shot_leg_rows - 1)
  const float* init_post;        // [B, V] or null
  // outputs
  uint8_t* errors;
  uint32_t* errors_packed;
  float* weights;
  long long* wfixed;
  int* found;
  int* iters;
  void* last_post;
  // resumable decoding: shot state after/before a phase (see ShotStateLayout)
  int legs_begin;                // first relay leg when resuming
  int legs_end;                  // relay legs < legs_end run (<= 0: all)
  const unsigned char* resume;   // [B, state_stride] or null: start from the pre-iterations
  unsigned char* suspend;        // [B, state_stride] or null
  int state_stride;
  // scheduling
  int* queue;
  const int* order;              // [B] queue position -> shot index, or null (identity)
  const int* queue_len;          // device count of queue positions to take, or null: B
  // split decode: after the pre-iterations a solved shot runs relay legs < solved_legs at the
  // constant strength solved_gamma; with suspend_unsolved an unsolved shot saves its state and stops
  float solved_gamma;
  int solved_legs;
  int suspend_unsolved;
  int parity_first;              // 0 never, 1 at iteration 1 of relay legs, 2 every iteration
  int group_threads, groups;
  // shared-memory layout (byte offsets)
  int off_chk_deg, off_llr, off_first, off_group0, group_bytes;
  int first_table;               // 1: take each phase's first check pass from the block's table
  int g_msg, g_par, g_best, g_first, g_red;
  int g_s1;                      // one-shot block-per-group kernel: the shot's first-pass sums
};

enum HardSrc { HARD_ZERO = 0, HARD_POST = 1, HARD_BEST = 2 };

// Per-shot decode state between launches (bytes):
//   [0,4) found  [4,8) iterations  [8,12) hard source  [12,16) has-best
//   [16,24) best weight (2^-32 units)  [24,32) unused
//   [32, 32+4W) best-solution bits, [32+4W, 32+8W) first-leg bits,
//   then the posterior [V] (accumulation type) at post_offset.
__host__ __device__ constexpr int state_post_offset(int V) { return (32 + 8 * ((V + 31) / 32) + 15) / 16 * 16; }
__host__ __device__ constexpr int state_stride(int V, int acc_bytes) {
  return (state_post_offset(V) + acc_bytes * V + 15) / 16 * 16;
}
constexpr uint16_t kNoSlot = 0xFFFFu;

// Shared-memory index of slot j of check c.  The slots of a check sit in
// 16-byte chunks of VEC = 16 / sizeof(M) messages, so a check pass moves a row
// with 128-bit loads/stores and consecutive checks occupy consecutive chunks:
//   index = (j / VEC) * (VEC * C) + c * VEC + ((j % VEC) ^ chunk_swizzle(c))
// The XOR swizzle permutes the slots inside a chunk by bits 3-4 of c, so the
// variable pass, whose warps touch the same slot of ~32 consecutive checks,
// spreads those accesses over all 32 banks instead of 8.  The check pass's
// work is symmetric in the slots of a row; it only needs the swizzle to know
// which positions are padding.  A slot's check is (index mod VEC*C) / VEC.
template <typename M>
__host__ __device__ __forceinline__ int chunk_swizzle(int c) {
  constexpr int VEC = 16 / (int)sizeof(M);
  if constexpr (VEC == 8) return ((c >> 3) & 3) << 1;  // 16-bit messages: permute 4-byte words
  else if constexpr (VEC == 4) return (c >> 3) & 3;
  else return (c >> 3) & 1;
}

template <typename M>
__host__ __device__ __forceinline__ int slot_index(int j, int c, int C) {
  constexpr int VEC = 16 / (int)sizeof(M);
  return (j / VEC) * (VEC * C) + c * VEC + ((j % VEC) ^ chunk_swizzle<M>(c));
}

// Index of the first element of chunk q of check c: the 16-byte aligned
// address vector loads and stores use (physical element p of the chunk holds
// slot q * VEC + (p ^ chunk_swizzle(c))).
template <typename M>
__host__ __device__ __forceinline__ int chunk_base(int q, int c, int C) {
  constexpr int VEC = 16 / (int)sizeof(M);
  return q * (VEC * C) + c * VEC;
}

// 16-byte vector access to VEC consecutive slots, converted to/from the
// accumulation type.
template <typename M>
struct VecIO;
template <>
struct VecIO<float> {
  static constexpr int N = 4;
  static __device__ __forceinline__ void load(const float* p, float* o) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
  }
  static __device__ __forceinline__ void store(float* p, const float* o) {
    *reinterpret_cast<float4*>(p) = make_float4(o[0], o[1], o[2], o[3]);
  }
};
template <>
struct VecIO<double> {
  static constexpr int N = 2;
  static __device__ __forceinline__ void load(const double* p, double* o) {
    const double2 v = *reinterpret_cast<const double2*>(p);
    o[0] = v.x; o[1] = v.y;
  }
  static __device__ __forceinline__ void store(double* p, const double* o) {
    *reinterpret_cast<double2*>(p) = make_double2(o[0], o[1]);
  }
};
template <typename H, float (*ToF)(H), H (*FromF)(float), unsigned short (*Bits)(H), H (*FromBits)(unsigned short)>
struct VecIO16 {
  static constexpr int N = 8;
  static __device__ __forceinline__ void load(const H* p, float* o) {
    const uint4 v = *reinterpret_cast<const uint4*>(p);
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      o[2 * i] = ToF(FromBits((unsigned short)(w[i] & 0xFFFFu)));
      o[2 * i + 1] = ToF(FromBits((unsigned short)(w[i] >> 16)));
    }
  }
  static __device__ __forceinline__ void store(H* p, const float* o) {
    uint32_t w[4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
      w[i] = (uint32_t)Bits(FromF(o[2 * i])) | ((uint32_t)Bits(FromF(o[2 * i + 1])) << 16);
    *reinterpret_cast<uint4*>(p) = make_uint4(w[0], w[1], w[2], w[3]);
  }
};
__device__ __forceinline__ float h2f(__half h) { return __half2float(h); }
__device__ __forceinline__ __half f2h(float f) { return f16_saturate(f); }
__device__ __forceinline__ unsigned short hbits(__half h) { return __half_as_ushort(h); }
__device__ __forceinline__ __half hfrom(unsigned short b) { return __ushort_as_half(b); }
__device__ __forceinline__ float b2f(__nv_bfloat16 h) { return __bfloat162float(h); }
__device__ __forceinline__ __nv_bfloat16 f2b(float f) { return __float2bfloat16_rn(f); }
__device__ __forceinline__ unsigned short bbits(__nv_bfloat16 h) { return __bfloat16_as_ushort(h); }
__device__ __forceinline__ __nv_bfloat16 bfrom(unsigned short b) { return __ushort_as_bfloat16(b); }
template <>
struct VecIO<__half> : VecIO16<__half, h2f, f2h, hbits, hfrom> {};
template <>
struct VecIO<__nv_bfloat16> : VecIO16<__nv_bfloat16, b2f, f2b, bbits, bfrom> {};

// Largest thread block an instantiation with VPT owned variables per thread
// is compiled for; bounds the registers the owned-variable state may take.
__host__ __device__ constexpr int max_block_threads(int vpt) {
  return vpt <= 2 ? 1024 : (vpt == 3 ? 896 : (vpt == 4 ? 768 : (vpt <= 8 ? 512 : 256)));
}

// Bit set of the hard decisions post <= 0 of the group's variables into dst
// (one ballot per warp and owned-variable slot).
template <typename A, int VPT>
__device__ __forceinline__ void ballot_post(const A (&post)[VPT], uint32_t* dst, int warp, int lane, int G, int V) {
#pragma unroll
  for (int k = 0; k < VPT; ++k) {
    const int v0 = warp * 32 + k * G;
    const unsigned m = __ballot_sync(0xffffffffu, v0 + lane < V && post[k] <= A(0));
    if (lane == 0 && v0 < V) dst[v0 >> 5] = m;
  }
}

// ------------------------------------------------------------------ the kernel
//
// M     message storage type (float, __half, __nv_bfloat16, double)
// MAXDC check degree bound held in registers by the check pass (0: generic loop)
// VPT   variables owned per thread
// MAXDV variable degree bound (slot positions held in registers)
// Negate every message of a 16-byte chunk (IEEE sign flip, exact in every
// storage type: float16 / bfloat16 saturate and round symmetrically).
template <typename M>
__device__ __forceinline__ uint4 flip_signs(uint4 v) {
  if constexpr (sizeof(M) == 2) {
    v.x ^= 0x80008000u; v.y ^= 0x80008000u; v.z ^= 0x80008000u; v.w ^= 0x80008000u;
  } else if constexpr (sizeof(M) == 4) {
    v.x ^= 0x80000000u; v.y ^= 0x80000000u; v.z ^= 0x80000000u; v.w ^= 0x80000000u;
  } else {
    v.y ^= 0x80000000u; v.w ^= 0x80000000u;
  }
  return v;
}

// The first check pass of every phase reads mu_e = llr[var(e)]: it is the same
// for every shot except for the syndrome bit, which only negates the check's
// outputs (par flips, the magnitudes do not change).  This computes that pass
// once per block for s = 0, with the same operations the check pass uses
// (alpha of iteration 0, beta, the degree-1 rule, storage rounding), into the
// table at off_first; the kernel then copies a row, negated when s = 1.
template <typename M, int MAXDC>
__device__ void build_first_pass_table(const DevGraph& g, const DevArgs& a, unsigned char* smem) {
  if constexpr (MAXDC > 0) {
    using IO = MsgT<M>;
    using A = typename IO::A;
    constexpr int VEC = VecIO<M>::N;
    constexpr int NQ = MAXDC / VEC;
    M* tab = reinterpret_cast<M*>(smem + a.off_first);
    const float* s_llr = reinterpret_cast<const float*>(smem + a.off_llr);
    const uint8_t* s_chk_deg = smem + a.off_chk_deg;
    for (int v = threadIdx.x; v < g.V; v += blockDim.x)
      for (int j = 0; j < g.vslots; ++j) {
        const uint16_t p = g.var_pos[j * g.V + v];
        if (p != kNoSlot) tab[p] = IO::st(A(s_llr[v]));
      }
    __syncthreads();
    const A alpha = a.use_alpha ? A(__ldg(a.alpha)) : A(1);
    const A beta = A(a.beta);
    const A kInf = A(__int_as_float(0x7f800000));
    for (int c = threadIdx.x; c < g.C; c += blockDim.x) {
      const int deg = s_chk_deg[c];
      const int swz = chunk_swizzle<M>(c);
      A mv[MAXDC];
#pragma unroll
      for (int q = 0; q < NQ; ++q) VecIO<M>::load(tab + chunk_base<M>(q, c, g.C), mv + q * VEC);
      int neg = 0;
      A min1 = A(1e30), min2 = A(1e30);
#pragma unroll
      for (int j = 0; j < MAXDC; ++j) {
        const bool in = ((j % VEC) ^ swz) < deg - (j / VEC) * VEC;
        neg ^= (in && mv[j] < A(0)) ? 1 : 0;
        const A x = in ? fmin(fabs(mv[j]), kInf) : kInf;
        min2 = fmin(min2, fmax(min1, x));
        min1 = fmin(min1, x);
      }
      const bool par = (neg & 1) != 0;  // syndrome bit 0
      A lo = deg == 1 ? A(0) : min1;
      A hi = deg == 1 ? A(0) : min2;
      if (a.use_alpha) {
        lo = mul_rn(alpha, lo);
        hi = mul_rn(alpha, hi);
      }
      if (a.use_beta) {
        lo = fmax(sub_rn(lo, beta), A(0));
        hi = fmax(sub_rn(hi, beta), A(0));
      }
      A out[MAXDC];
#pragma unroll
      for (int j = 0; j < MAXDC; ++j) {
        const A m = mv[j];
        const A mag = (fabs(m) == min1) ? hi : lo;
        out[j] = (par != !(m >= A(0))) ? -mag : mag;
      }
#pragma unroll
      for (int q = 0; q < NQ; ++q) VecIO<M>::store(tab + chunk_base<M>(q, c, g.C), out + q * VEC);
    }
    __syncthreads();
  }
}

// Copy the code's block-wide tables (check degrees, prior LLRs) to shared memory.
__device__ __forceinline__ void load_block_tables(const DevGraph& g, const DevArgs& a, unsigned char* smem) {
  uint8_t* s_chk_deg = smem + a.off_chk_deg;
  float* s_llr = reinterpret_cast<float*>(smem + a.off_llr);
  for (int i = threadIdx.x; i < g.C; i += blockDim.x) s_chk_deg[i] = g.chk_deg[i];
  for (int i = threadIdx.x; i < g.V; i += blockDim.x) s_llr[i] = a.llr[i];
}

// The groups of this block decode shots of one code until its work queue is
// empty.  The block-wide tables must be in shared memory (load_block_tables +
// a block barrier); threads beyond a.groups * a.group_threads return at once.
template <typename M, int MAXDC, int VPT, int MAXDV>
__device__ __forceinline__ void run_groups(const DevGraph& g, const DevArgs& a, unsigned char* smem) {
  using IO = MsgT<M>;
  using A = typename IO::A;

  const int C = g.C, V = g.V;
  const uint8_t* s_chk_deg = smem + a.off_chk_deg;
  const float* s_llr = reinterpret_cast<const float*>(smem + a.off_llr);

  const int G = a.group_threads;
  const int gid = threadIdx.x / G;
  const int t = threadIdx.x - gid * G;
  const int lane = threadIdx.x & 31;
  const int warp = t >> 5;
  const int nwarps = G >> 5;
  const int bar = 1 + gid;
  const int W = (V + 31) >> 5;
  const int S = a.stop_nconv;

  // slot positions of the owned variables' edges in summation order; absent
  // edges (degree < MAXDV) point at the dummy slot after the last row
  const uint32_t dummy = (uint32_t)(g.rows * C);
  uint32_t vpos[VPT][MAXDV];
#pragma unroll
  for (int k = 0; k < VPT; ++k) {
    const int v = t + k * G;
#pragma unroll
    for (int j = 0; j < MAXDV; ++j) {
      uint32_t p = dummy;
      if (v < V && j < g.vslots) p = g.var_pos[j * V + v];
      vpos[k][j] = p == kNoSlot ? dummy : p;
    }
  }
  if (gid >= a.groups) return;

  unsigned char* gsm = smem + a.off_group0 + gid * a.group_bytes;
  M* msg = reinterpret_cast<M*>(gsm + a.g_msg);
  // parity of each check's current hard decisions, bit c%32 of word c/32
  uint32_t* par_bits = reinterpret_cast<uint32_t*>(gsm + a.g_par);
  const int Wc = (C + 31) >> 5;
  const int VC = VecIO<M>::N * C;  // elements per chunk column: slot p belongs to check (p % VC) / VEC
  uint32_t* best_bits = reinterpret_cast<uint32_t*>(gsm + a.g_best);
  uint32_t* first_bits = reinterpret_cast<uint32_t*>(gsm + a.g_first);
  long long* red = reinterpret_cast<long long*>(gsm + a.g_red);
  volatile long long* shot_slot = red + nwarps;
  const A beta = A(a.beta);
  const bool first_from_table = MAXDC > 0 && a.first_table && a.llr_shot == nullptr;
  const M* first_tab = reinterpret_cast<const M*>(smem + a.off_first);

  A post[VPT];
  A gam[VPT];

  int q_early = -1;  // thread 0: the queue position claimed while the last shot wrote its outputs
  while (true) {
    if (t == 0) {
      const long long q = (long long)(q_early >= 0 ? q_early : atomicAdd(a.queue, 1));
      q_early = -1;
      const long long qn = a.queue_len ? (long long)max(0, min(*a.queue_len, (int)a.B)) : a.B;
      long long sb = q < qn ? q : a.B;
      if (q < qn && a.order) {
        sb = (long long)a.order[q];
        if (sb < 0 || sb >= a.B) sb = -1;  // not a shot index: this queue entry is skipped
      }
      *shot_slot = sb;
    }
    group_sync(bar, G);
    const long long b = *shot_slot;
    if (b >= a.B) break;
    if (b < 0) {
      group_sync(bar, G);  // every thread has read the slot before thread 0 refills it
      continue;
    }

    // ---------------- per-shot setup (decoder.py:3429-3478)
    // Every load of the shot's inputs is issued before any of them is used, so the
    // latencies of the saved state and the syndrome overlap.
    const uint8_t* syn_row = a.syn + b * (long long)C;
    const float* llr_row = a.llr_shot ? a.llr_shot + b * (long long)V : nullptr;
    long long best_w = LLONG_MAX;
    int found = 0, iters = 0, hard_src = HARD_ZERO, sought = 1, has_best_raw = 0;
    const int pre = a.pre_iter;
    const unsigned char* st = a.resume ? a.resume + b * (long long)a.state_stride : nullptr;
    const uint32_t* st_bits = st ? reinterpret_cast<const uint32_t*>(st + 32) : nullptr;
    uint32_t bits0 = 0u, bits1 = 0u;  // this thread's first words of the two saved bit sets
    if (st) {
      // continue a shot suspended after an earlier phase
      const int* hdr = reinterpret_cast<const int*>(st);
      found = hdr[0];
      iters = hdr[1];
      hard_src = hdr[2];
      has_best_raw = hdr[3];
      best_w = *reinterpret_cast<const long long*>(st + 16);
      if (t < W) {
        bits0 = st_bits[t];
        bits1 = st_bits[W + t];
      }
      const A* sp = reinterpret_cast<const A*>(st + state_post_offset(V));
#pragma unroll
      for (int k = 0; k < VPT; ++k) {
        const int v = t + k * G;
        post[k] = v < V ? sp[v] : A(0);
      }
    } else {
#pragma unroll
      for (int k = 0; k < VPT; ++k) {
        const int v = t + k * G;
        A p0 = A(0);
        if (v < V) {
          if (a.init_post) p0 = A(__ldg(a.init_post + b * (long long)V + v));
          else p0 = llr_row ? A(__ldg(llr_row + v)) : A(s_llr[v]);
        }
        post[k] = p0;
      }
    }
    uint32_t synm = 0;  // bit k: syndrome of check t + k*G; four loads in flight per round
    for (int k = 0, c = t; c < C; k += 4, c += 4 * G) {
      const uint32_t s0 = syn_row[c];
      const uint32_t s1 = c + G < C ? (uint32_t)syn_row[c + G] : 0u;
      const uint32_t s2 = c + 2 * G < C ? (uint32_t)syn_row[c + 2 * G] : 0u;
      const uint32_t s3 = c + 3 * G < C ? (uint32_t)syn_row[c + 3 * G] : 0u;
      synm |= ((s0 & 1u) | ((s1 & 1u) << 1) | ((s2 & 1u) << 2) | ((s3 & 1u) << 3)) << k;
    }
    // every hard decision starts at 0 (parity 0 for every check); the first variable pass
    // flips the ones it sets
    for (int w = t; w < Wc; w += G) par_bits[w] = 0u;
    uint32_t hmask = 0;  // bit k: hard decision of variable t + k*G
    uint32_t hmask_sel = 0;   // this thread's decisions at the shot's last computed selection
    bool sel_seen = false;    // a selection has been computed for this shot (group-uniform)
    bool has_best = has_best_raw != 0;
    if (st) {
      if (t < W) {
        best_bits[t] = bits0;
        first_bits[t] = bits1;
      }
      for (int w = t + G; w < W; w += G) {
        best_bits[w] = st_bits[w];
        first_bits[w] = st_bits[W + w];
      }
    } else {
      for (int w = t; w < W; w += G) {
        best_bits[w] = 0u;
        first_bits[w] = 0u;
      }
    }
    const int legs_stop = (a.legs_end > 0 && a.legs_end < a.num_sets) ? a.legs_end : a.num_sets;
    bool solved_pre = false, stopped_unsolved = false;
    // a shot resumed at leg 0 was solved by the pre-iterations if it found a solution there
    if (a.resume && a.legs_begin == 0) solved_pre = found > 0;

    // Phase -1: the pre-iterations (decoder.py:3480-3616); phase l >= 0: relay
    // leg l (decoder.py:3672-3837).  A resumed shot starts at leg legs_begin.
    for (int phase = a.resume ? a.legs_begin : -1; phase < legs_stop; ++phase) {
      int max_iter;
      const float* grow;
      float gs = 0.f;
      if (phase < 0) {
        max_iter = pre;
        grow = a.gamma_pre ? a.gamma_pre + b * (long long)V : nullptr;
        gs = a.gamma0;
      } else {
        if (found >= S) break;
        sought = found + 1;
        max_iter = a.set_max_iter;
        grow = (a.gamma_legs_shot && phase < a.n_shot_legs)
                   ? a.gamma_legs_shot + (b * (long long)a.shot_leg_rows + min(phase, a.shot_leg_rows - 1)) * V
                   : a.gamma_legs + (long long)phase * V;
        if (solved_pre && phase < a.solved_legs) {
          grow = nullptr;
          gs = a.solved_gamma;
        }
      }

      if (max_iter <= 0) {
        // freeze_finished_lanes_kernel(count_iteration=False) after an empty phase
        if (found >= min(sought, S)) hard_src = HARD_BEST;
      } else {
        // memory strengths of this phase; message init mu_e = llr[var(e)] (kernels.py:904-1000)
#pragma unroll
        for (int k = 0; k < VPT; ++k) {
          const int v = t + k * G;
          if (v < V) {
            gam[k] = A(gs);
            if (grow) gam[k] = A(__ldg(grow + v));  // first read in the variable pass
            if (!first_from_table) {  // the first check pass reads mu = llr; the table stands in for it
              const M m0 = IO::st(llr_row ? A(__ldg(llr_row + v)) : A(s_llr[v]));
#pragma unroll
              for (int j = 0; j < MAXDV; ++j) msg[vpos[k][j]] = m0;
            }
          }
        }
        // The first check pass must see the initial messages.  The table path
        // writes none here, and the previous phase's (or shot's) last reads of
        // the messages and parity bits ended at a group barrier.
        if (!first_from_table) group_sync(bar, G);
        int valid = 0;
        bool frozen = false;
        for (int it = 0; it <= max_iter; ++it) {
          const bool check_parity = it > 0;
          const bool write_nu = it < max_iter;
          // Parity first: test iteration it-1's hard decisions alone, and run the
          // min-sum pass only if some check fails.  The nu a converged pass would
          // write is never read (messages restart every leg), so results are the same.
          const bool parity_first = check_parity && write_nu &&
                                    (a.parity_first == 2 || (a.parity_first == 1 && phase >= 0 && it == 1));
          const A alpha = (a.use_alpha && write_nu) ? A(__ldg(a.alpha + it)) : A(1);
          bool all_ok = false;
          if (parity_first) {
            bool okp = true;
            int kp = 0;
            for (int c = t; c < C; c += G, ++kp) {
              const int s = (int)((synm >> kp) & 1u);
              const int par = (int)((par_bits[c >> 5] >> (c & 31)) & 1u);
              okp = okp && (par == s);
            }
            all_ok = group_all(bar, G, okp);
          }
          if (!parity_first || !all_ok) {
          const bool chk_par = check_parity && !parity_first;

          // ---------------- check pass (kernels.py:1052-1215) + parity of it-1 (kernels.py:510-569)
          bool ok_all = true;
          int k = 0;
          for (int c = t; c < C; c += G, ++k) {
            const int s = (int)((synm >> k) & 1u);
            int neg = 0, cnt1 = 0;
            A min1 = A(1e30), min2 = A(1e30);
            if constexpr (MAXDC > 0) {
              // The row's slots are contiguous in 16-byte chunks (VEC messages each)
              // and padded to MAXDC: NQ vector loads/stores, padding masked by selects.
              constexpr int NQ = MAXDC / VecIO<M>::N;
              constexpr int VEC = VecIO<M>::N;
              if (it == 0 && first_from_table) {
                // first pass of the phase: the block's table row, negated when s = 1
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                  uint4 w = *reinterpret_cast<const uint4*>(first_tab + chunk_base<M>(q, c, C));
                  if (s) w = flip_signs<M>(w);
                  *reinterpret_cast<uint4*>(msg + chunk_base<M>(q, c, C)) = w;
                }
                continue;
              }
              const int deg = s_chk_deg[c];
              const int swz = chunk_swizzle<M>(c);
              A mv[MAXDC];
#pragma unroll
              for (int q = 0; q < NQ; ++q)
                VecIO<M>::load(msg + chunk_base<M>(q, c, C), mv + q * VecIO<M>::N);
              if (chk_par) ok_all = ok_all && ((int)((par_bits[c >> 5] >> (c & 31)) & 1u) == s);
              if (write_nu) {
                // min1 = min(1e30, |mu_j|), min2 = the second smallest (a tie gives
                // min2 == min1): the argmin edge receives min2 exactly when it is
                // unique, as in kernels.py:1128-1194.  NaN magnitudes are ignored,
                // like the reference's comparisons.
                const A kInf = A(__int_as_float(0x7f800000));
#pragma unroll
                for (int j = 0; j < MAXDC; ++j) {
                  // physical position j holds slot (j / VEC) * VEC + ((j % VEC) ^ swz)
                  const bool in = ((j % VEC) ^ swz) < deg - (j / VEC) * VEC;
                  neg ^= (in && mv[j] < A(0)) ? 1 : 0;  // parity of negative messages (kernels.py:1134)
                  const A x = in ? fmin(fabs(mv[j]), kInf) : kInf;
                  min2 = fmin(min2, fmax(min1, x));
                  min1 = fmin(min1, x);
                }
                const bool par = ((neg ^ s) & 1) != 0;
                A lo = deg == 1 ? A(0) : min1;
                A hi = deg == 1 ? A(0) : min2;
                if (a.use_alpha) {
                  lo = mul_rn(alpha, lo);
                  hi = mul_rn(alpha, hi);
                }
                if (a.use_beta) {
                  lo = fmax(sub_rn(lo, beta), A(0));
                  hi = fmax(sub_rn(hi, beta), A(0));
                }
                A out[MAXDC];
#pragma unroll
                for (int j = 0; j < MAXDC; ++j) {
                  const A m = mv[j];
                  const A mag = (fabs(m) == min1) ? hi : lo;
                  // sign (mu >= 0 ? 1 : -1) * parity sign (kernels.py:1189-1202)
                  out[j] = (par != !(m >= A(0))) ? -mag : mag;
                }
#pragma unroll
                for (int q = 0; q < NQ; ++q)
                  VecIO<M>::store(msg + chunk_base<M>(q, c, C), out + q * VecIO<M>::N);
              }
            } else {
              const int deg = g.chk_ptr[c + 1] - g.chk_ptr[c];
              for (int j = 0; j < deg; ++j) {
                const int ix = slot_index<M>(j, c, C);
                const A m = IO::ld(msg[ix]);
                neg ^= (m < A(0)) ? 1 : 0;
                const A x = fabs(m);
                if (x < min1) { min2 = min1; min1 = x; cnt1 = 1; }
                else if (x == min1) { cnt1 += 1; }
                else if (x < min2) { min2 = x; }
              }
              if (chk_par) ok_all = ok_all && ((int)((par_bits[c >> 5] >> (c & 31)) & 1u) == s);
              if (write_nu) {
                const bool par = ((neg ^ s) & 1) != 0;
                for (int j = 0; j < deg; ++j) {
                  const int ix = slot_index<M>(j, c, C);
                  const A m = IO::ld(msg[ix]);
                  A mag = (cnt1 == 1 && fabs(m) == min1) ? min2 : min1;
                  if (deg == 1) mag = A(0);
                  if (a.use_alpha) mag = mul_rn(alpha, mag);
                  if (a.use_beta) mag = fmax(sub_rn(mag, beta), A(0));
                  msg[ix] = IO::st((par != !(m >= A(0))) ? -mag : mag);
                }
              }
            }
          }
          const bool a2 = group_all(bar, G, ok_all);
          if (!parity_first) all_ok = a2;
          }

          if (check_parity) {
            // check_and_select_kernel (kernels.py:609-741) for iteration it-1
            // the decisions of the last computed selection again: same weight, best unchanged
            const bool repeat = all_ok && sel_seen && !group_any(bar, G, hmask != hmask_sel);
            if (repeat) {
              if (valid == 0) found += 1;
              valid = 1;
            } else if (all_ok) {
              hmask_sel = hmask;
              sel_seen = true;
              long long w = 0;
#pragma unroll
              for (int kk = 0; kk < VPT; ++kk) {
                const int v = t + kk * G;
                if (v < V && post[kk] <= A(0))
                  w += weight_units(llr_row ? __ldg(llr_row + v) : s_llr[v]);
              }
#pragma unroll
              for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
              // red[0] was cleared by this phase's variable pass (before its barrier)
              if (lane == 0) atomicAdd(reinterpret_cast<unsigned long long*>(red), (unsigned long long)w);
              group_sync(bar, G);
              const long long tot = red[0];
              if (!has_best || tot < best_w) {
                best_w = tot;
                has_best = true;
                ballot_post<A, VPT>(post, best_bits, warp, lane, G, V);
              }
              if (valid == 0) found += 1;
              valid = 1;
            }
            // freeze_finished_lanes_kernel (kernels.py:746-847): this iteration counts
            if (found >= min(sought, S)) {
              iters += it;
              hard_src = HARD_BEST;
              frozen = true;
              // No barrier here: each warp's best_bits words are written by that
              // warp alone and read only after a later barrier, and `red` is
              // rewritten no sooner than the next phase's check-pass barrier.
              break;
            }
          }
          if (!write_nu) break;

          // ---------------- variable pass (kernels.py:1220-1350)
#pragma unroll
          for (int kk = 0; kk < VPT; ++kk) {
            const int v = t + kk * G;
            if (v < V) {
              const A l0 = llr_row ? A(__ldg(llr_row + v)) : A(s_llr[v]);
              const A lm = memory_mix<A>(a.mix_mode, gam[kk], l0, post[kk]);
              A nv[MAXDV];
              A sum = A(0);
#pragma unroll
              for (int j = 0; j < MAXDV; ++j) {
                const uint32_t p = vpos[kk][j];
                nv[j] = IO::ld(msg[p]);
                // absent edges point at the group's dummy slot and are not summed
                sum = (p != dummy) ? add_rn(sum, nv[j]) : sum;
              }
              const A pv = add_rn(lm, sum);
              post[kk] = pv;
#pragma unroll
              for (int j = 0; j < MAXDV; ++j) {
                const uint32_t p = vpos[kk][j];
                msg[p] = IO::st(add_rn(lm, sub_rn(sum, nv[j])));
              }
              const uint32_t h = pv <= A(0) ? 1u : 0u;
              if (h != ((hmask >> kk) & 1u)) {
                // the decision flipped: so does the parity of each of its checks
                hmask ^= 1u << kk;
#pragma unroll
                for (int j = 0; j < MAXDV; ++j) {
                  uint32_t q = vpos[kk][j];
                  if (q != dummy) {
                    if constexpr (MAXDC > 0) {
#pragma unroll
                      for (int r = 1; r < MAXDC / VecIO<M>::N; ++r) q = q >= (uint32_t)VC ? q - (uint32_t)VC : q;
                    } else {
                      while (q >= (uint32_t)VC) q -= (uint32_t)VC;
                    }
                    const uint32_t c = q / (uint32_t)VecIO<M>::N;
                    atomicXor(par_bits + (c >> 5), 1u << (c & 31u));
                  }
                }
              }
            }
          }
          hard_src = HARD_POST;
          if (t == 0) red[0] = 0;  // the next selection's sum; its last reader passed a barrier since
          group_sync(bar, G);
        }
        if (!frozen) iters += max_iter;
      }

      // first-leg hard decision: after the pre-iterations, or after relay leg 1
      // when there were none (decoder.py:3595-3598, 3807-3810)
      if (!a.last_leg && (phase < 0 || (phase == 0 && pre == 0))) {
        group_sync(bar, G);
        if (hard_src == HARD_POST) {
          ballot_post<A, VPT>(post, first_bits, warp, lane, G, V);
        } else {
          for (int w = t; w < W; w += G) first_bits[w] = hard_src == HARD_BEST ? best_bits[w] : 0u;
        }
        group_sync(bar, G);
      }
      if (phase < 0 && (found >= S || a.skip_legs)) break;
      if (phase < 0) {
        solved_pre = found > 0;
        if (!solved_pre && a.suspend_unsolved) {
          stopped_unsolved = true;
          break;
        }
      }
    }

    // ---------------- outputs, decoder.py:3839-3873
    group_sync(bar, G);
    if (t == 0) q_early = atomicAdd(a.queue, 1);
    if (a.suspend && (!a.suspend_unsolved || stopped_unsolved)) {
      unsigned char* st = a.suspend + b * (long long)a.state_stride;
      if (t == 0) {
        int* hdr = reinterpret_cast<int*>(st);
        hdr[0] = found;
        hdr[1] = iters;
        hdr[2] = hard_src;
        hdr[3] = has_best ? 1 : 0;
        *reinterpret_cast<long long*>(st + 16) = best_w;
      }
      uint32_t* bits = reinterpret_cast<uint32_t*>(st + 32);
      for (int w = t; w < W; w += G) {
        bits[w] = best_bits[w];
        bits[W + w] = first_bits[w];
      }
      A* sp = reinterpret_cast<A*>(st + state_post_offset(V));
#pragma unroll
      for (int k = 0; k < VPT; ++k) {
        const int v = t + k * G;
        if (v < V) sp[v] = post[k];
      }
    }
    const uint32_t* src_bits = has_best ? best_bits : first_bits;
    const bool from_post = !has_best && a.last_leg && hard_src == HARD_POST;
    const bool zero_bits = !has_best && a.last_leg && hard_src != HARD_POST;
    if (a.errors) {
      uint8_t* erow = a.errors + b * (long long)V;
#pragma unroll
      for (int k = 0; k < VPT; ++k) {
        const int v = t + k * G;
        if (v < V) {
          uint8_t e;
          if (from_post) e = post[k] <= A(0) ? 1 : 0;
          else if (zero_bits) e = 0;
          else e = (src_bits[v >> 5] >> (v & 31)) & 1u;
          erow[v] = e;
        }
      }
    }
    if (a.errors_packed) {
      uint32_t* prow = a.errors_packed + b * (long long)W;
#pragma unroll
      for (int k = 0; k < VPT; ++k) {
        const int v0 = warp * 32 + k * G;
        unsigned m;
        if (from_post) m = __ballot_sync(0xffffffffu, v0 + lane < V && post[k] <= A(0));
        else if (zero_bits) m = 0u;
        else m = v0 < V ? src_bits[v0 >> 5] : 0u;
        if (lane == 0 && v0 < V) prow[v0 >> 5] = m;
      }
    }
    if (a.last_post) {
#pragma unroll
      for (int k = 0; k < VPT; ++k) {
        const int v = t + k * G;
        if (v < V) {
          if constexpr (sizeof(A) == 8) reinterpret_cast<double*>(a.last_post)[b * (long long)V + v] = post[k];
          else reinterpret_cast<float*>(a.last_post)[b * (long long)V + v] = post[k];
        }
      }
    }
    if (t == 0) {
      if (a.weights)
        a.weights[b] = has_best ? __ll2float_rn(best_w) * 2.3283064365386963e-10f  // 2^-32
                                : __int_as_float(0x7f800000);
      if (a.wfixed) a.wfixed[b] = has_best ? best_w : LLONG_MAX;
      a.found[b] = found;
      a.iters[b] = iters;
    }
    group_sync(bar, G);
  }
}

// One code, one launch (rbp_decode, rbp_decode_static).
template <typename M, int MAXDC, int VPT, int MAXDV>
__global__ void __launch_bounds__(max_block_threads(VPT))
relaybp_decode_kernel(DevGraph g, DevArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  load_block_tables(g, a, smem);
  __syncthreads();
  if (a.first_table) build_first_pass_table<M, MAXDC>(g, a, smem);
  run_groups<M, MAXDC, VPT, MAXDV>(g, a, smem);
}

// Several codes in one launch (rbp_mixed_*).  Block b starts on the code whose
// block range holds b (first_block[], from the host's work estimate).  When
// that code's queue is empty the whole block moves to the next code that still
// has shots, re-partitioning its threads into that code's group shape, until
// every queue is empty.  Queue counters only grow, so the loop ends.
constexpr int kMaxMixedCodes = 8;

struct MixedCode {
  DevGraph g;
  DevArgs a;
};

struct MixedArgs {
  MixedCode code[kMaxMixedCodes];
  int ncodes;
  int first_block[kMaxMixedCodes + 1];
};

template <typename M, int MAXDC, int VPT, int MAXDV>
__global__ void __launch_bounds__(max_block_threads(VPT))
relaybp_mixed_kernel(const __grid_constant__ MixedArgs m) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_next;
  int code = 0;
  while (code + 1 < m.ncodes && (int)blockIdx.x >= m.first_block[code + 1]) ++code;
  while (code >= 0) {
    const DevGraph g = m.code[code].g;
    const DevArgs a = m.code[code].a;
    load_block_tables(g, a, smem);
    __syncthreads();
    if (a.first_table) build_first_pass_table<M, MAXDC>(g, a, smem);
    run_groups<M, MAXDC, VPT, MAXDV>(g, a, smem);
    __syncthreads();
    if (threadIdx.x == 0) {
      int next = -1;
      for (int i = 1; i <= m.ncodes && next < 0; ++i) {
        const int c = (code + i) % m.ncodes;
        if (*reinterpret_cast<volatile const int*>(m.code[c].a.queue) < m.code[c].a.B) next = c;
      }
      s_next = next;
    }
    __syncthreads();
    code = s_next;
    __syncthreads();
  }
}

using KernelFn = void (*)(DevGraph, DevArgs);

// Kernel for (check degree bound, variable degree, owned variables per thread),
// or null when this build has no such instantiation.  One per message type.
KernelFn pick_f32(int dc, int dv, int vpt);
KernelFn pick_f16(int dc, int dv, int vpt);
KernelFn pick_bf16(int dc, int dv, int vpt);
KernelFn pick_f64(int dc, int dv, int vpt);

using MixedKernelFn = void (*)(MixedArgs);
MixedKernelFn pick_mixed_f32(int dc, int dv, int vpt);

// Supported owned-variable counts, ascending.
constexpr int kVptChoices[] = {1, 2, 3, 4, 6, 8, 12, 16};

}  // namespace rbpk

// Instantiation table of one message type (used by relaybp_inst_*.cu).
#define RBPK_DC_DV(M, DC, VPT)                                                 \
  if (dv <= 3) return &rbpk::relaybp_decode_kernel<M, DC, VPT, 3>;             \
  if (dv <= 8) return &rbpk::relaybp_decode_kernel<M, DC, VPT, 8>;             \
  return nullptr;
#define RBPK_DC(M, VPT)                                                        \
  if (dc <= 8) { RBPK_DC_DV(M, 8, VPT) }                                       \
  if (dc <= 16) { RBPK_DC_DV(M, 16, VPT) }                                     \
  { RBPK_DC_DV(M, 0, VPT) }
#define RBPK_MDC_DV(M, DC, VPT)                                                \
  if (dv <= 3) return &rbpk::relaybp_mixed_kernel<M, DC, VPT, 3>;              \
  if (dv <= 8) return &rbpk::relaybp_mixed_kernel<M, DC, VPT, 8>;              \
  return nullptr;
#define RBPK_MDC(M, VPT)                                                       \
  if (dc <= 8) { RBPK_MDC_DV(M, 8, VPT) }                                      \
  if (dc <= 16) { RBPK_MDC_DV(M, 16, VPT) }                                    \
  { RBPK_MDC_DV(M, 0, VPT) }
#define RBPK_DEFINE_PICK_MIXED(NAME, M)                                        \
  rbpk::MixedKernelFn rbpk::NAME(int dc, int dv, int vpt) {                    \
    switch (vpt) {                                                             \
      case 4: { RBPK_MDC(M, 4) }                                               \
      case 8: { RBPK_MDC(M, 8) }                                               \
      case 16: { RBPK_MDC(M, 16) }                                             \
      default: return nullptr;                                                 \
    }                                                                          \
  }
#define RBPK_DEFINE_PICK(NAME, M)                                              \
  rbpk::KernelFn rbpk::NAME(int dc, int dv, int vpt) {                         \
    switch (vpt) {                                                             \
      case 1: { RBPK_DC(M, 1) }                                                \
      case 2: { RBPK_DC(M, 2) }                                                \
      case 3: { RBPK_DC(M, 3) }                                                \
      case 4: { RBPK_DC(M, 4) }                                                \
      case 6: { RBPK_DC(M, 6) }                                                \
      case 8: { RBPK_DC(M, 8) }                                                \
      case 12: { RBPK_DC(M, 12) }                                              \
      case 16: { RBPK_DC(M, 16) }                                              \
      default: return nullptr;                                                 \
    }                                                                          \
  }
