// The block-per-group decode kernel (sm_100a): one thread block is one group of
// G threads that decodes NS shots (1 or 2) at once, each in its own "slot".
//
// Why: the one-shot kernel (relaybp_kernel.cuh) runs one 15-warp group per SM
// for the benchmark code; its registers leave no room for a second group, so
// the SM waits on dependent-instruction and barrier latency.  A thread here
// owns the same variables and checks in every slot, so the per-edge slot
// positions (the largest part of its registers) are held once, and each pass
// interleaves NS independent dependency chains.  All slots' passes share one
// pair of barriers.
//
// Execution.  Every "tick" runs one iteration for each slot whose shot is in a
// running phase: a check pass of all running slots, a barrier, a variable pass
// of all running slots, a barrier.  Then, slot by slot (group-uniform control),
// come the events of the iteration just finished: a convergence (selection,
// freeze), the end of a phase (first-leg decision, the next relay leg), the
// end of a shot (outputs, the next queue position, the next shot's set-up).
// A slot whose queue is empty retires; the kernel ends when every slot has.
// Each shot's arithmetic is exactly that of the one-shot kernel, so results
// do not depend on which kernel or slot decodes a shot.
//
// Two resident blocks per SM (MINB 2, one shot per group): the same code with
// half the register file per block, so two shots decode side by side on an SM
// and one block's barrier and dependency waits become the other's issue slots.
//
// Relay legs' first iteration (one shot per group): a leg restarts the
// messages, so its first check pass is the block's table with the shot's
// syndrome signs, the same at every leg.  The shot's first leg in a launch
// keeps each variable's sum of those messages (the s1 array of its slot);
// later legs add the kept sum to the memory mix instead of running the check
// pass and reloading the messages, which gives the same posterior bit for bit.
//
// Convergence test without a pass.  mis[c/32] bit c%32 holds (parity of check
// c's current hard decisions) XOR (its syndrome bit): it starts as the syndrome
// (all decisions start at 0) and the variable pass flips it with a shared
// atomicXor whenever a decision flips.  The atomic's old value tells whether
// the check became satisfied or unsatisfied, so each thread sums +-1 per flip
// and adds that to the slot's count of unsatisfied checks.  After the
// variable pass's barrier a count of zero is a converged iteration
// (kernels.py:510-741's parity + all-checks test), at no cost beyond the flips.
//
// Shared memory: the block tables (relaybp_kernel.cuh), then NS slot regions
// of `group_bytes` each laid out like the one-shot kernel's group region:
// messages, mis bits, best bits, first-leg bits, and `red`:
//   red[0] weight sum of a selection (one-shot groups alternate it with red[4]),
//   red[1..2] the claimed shot index (two entries used in turn, so a claim never
//   overwrites one a thread has not read yet), red[3] (int) the count of
//   unsatisfied checks.
//
// Bit-set words are "owned" by the warp whose threads own their bits: thread
// t = 32 w + l owns variables t + k G, whose bits sit in word w + k (G/32) at
// bit l.  Only the owning warp writes or reads a word of the best / first-leg
// sets (ballots by lane 0, copies by lanes), so those accesses need __syncwarp
// only.  The same holds for the mis words at a shot's set-up.

#pragma once

#include "relaybp_kernel.cuh"

#include <type_traits>

namespace rbpk {

// Largest block an instantiation with VPT owned variables per thread and NS
// shots per group is compiled for (its register budget; two slots hold two
// posteriors and strengths per variable).
__host__ __device__ constexpr int max_slots_block_threads(int vpt, int ns = 2, int maxdv = 3) {
  (void)maxdv;  // the same budget for 3- and 8-edge variables
  return ns == 1 ? max_block_threads(vpt)
                 : (vpt <= 4 ? 512 : (vpt == 6 ? 480 : (vpt == 8 ? 384 : (vpt == 12 ? 256 : 192))));
}

// Largest block of the one-shot instantiations compiled for two resident
// blocks per SM (MINB 2): each block gets half the register file, so a thread
// has at most 64 registers (VPT <= 4), 72 (VPT 6), 80 (VPT 8) or 128.  Two
// shots then decode side by side on one SM with their own barriers, so one
// block's barrier and dependency waits are filled by the other's work.
__host__ __device__ constexpr int max_slots_block_threads2(int vpt) {
  return vpt <= 4 ? 512 : (vpt == 6 ? 448 : (vpt == 8 ? 384 : 256));
}

template <typename A, int VPT>
struct SlotState {
  A post[VPT];          // posteriors of the owned variables (the memory)
  A gam[VPT];           // memory strengths of the running phase
  uint32_t hmask;       // bit k: hard decision of variable t + k G
  uint32_t hmask_sel;   // the decisions at the shot's last computed selection
  uint32_t synm;        // bit k: syndrome of check t + k G
  // group-uniform control (every thread holds the same values)
  long long b;          // shot index
  long long best_w;     // best solution weight (2^-32 units)
  const float* grow;    // strength row of the running phase, or null: constant gs
  const float* llr_row; // per-shot prior LLRs or null
  float gs;
  int phase, it, max_iter, found, iters, hard_src;
  int claim;            // which red[1 + claim] entry the next claim writes
  int wsel;             // one-shot kernel: the next selection sums into red[0] (0) or red[4] (1)
  bool run, has_best, sel_seen, solved_pre, stopped;
  bool s1_ok;           // one-shot kernel: the slot's first-pass sums belong to this shot
  bool synced;          // the last iteration's test of the unsatisfied count was followed by a barrier
};

// One check row of one slot: min-sum (kernels.py:1052-1215) from the slot's
// messages, or on a phase's first pass the block's table row negated when the
// syndrome bit is set.  MAXDC > 0 only (vectorised rows).
template <typename M, int MAXDC>
__device__ __forceinline__ void slot_check_row(M* msg, const M* first_tab, bool tab, int c, int C, int deg, int s,
                                               typename MsgT<M>::A alpha, bool use_alpha, bool use_beta,
                                               typename MsgT<M>::A beta) {
  using A = typename MsgT<M>::A;
  constexpr int VEC = VecIO<M>::N;
  constexpr int NQ = MAXDC / VEC;
  if (tab) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      uint4 w = *reinterpret_cast<const uint4*>(first_tab + chunk_base<M>(q, c, C));
      if (s) w = flip_signs<M>(w);
      *reinterpret_cast<uint4*>(msg + chunk_base<M>(q, c, C)) = w;
    }
    return;
  }
  const int swz = chunk_swizzle<M>(c);
  A mv[MAXDC];
#pragma unroll
  for (int q = 0; q < NQ; ++q) VecIO<M>::load(msg + chunk_base<M>(q, c, C), mv + q * VEC);
  const A kInf = A(__int_as_float(0x7f800000));
  int neg = 0;
  A min1 = A(1e30), min2 = A(1e30);
#pragma unroll
  for (int j = 0; j < MAXDC; ++j) {
    // physical position j holds slot (j / VEC) * VEC + ((j % VEC) ^ swz)
    const bool in = ((j % VEC) ^ swz) < deg - (j / VEC) * VEC;
    neg ^= (in && mv[j] < A(0)) ? 1 : 0;
    const A x = in ? fmin(fabs(mv[j]), kInf) : kInf;
    min2 = fmin(min2, fmax(min1, x));
    min1 = fmin(min1, x);
  }
  const bool par = ((neg ^ s) & 1) != 0;
  A lo = deg == 1 ? A(0) : min1;
  A hi = deg == 1 ? A(0) : min2;
  if (use_alpha) {
    lo = mul_rn(alpha, lo);
    hi = mul_rn(alpha, hi);
  }
  if (use_beta) {
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
  for (int q = 0; q < NQ; ++q) VecIO<M>::store(msg + chunk_base<M>(q, c, C), out + q * VEC);
}

// Variable pass of one owned variable in one slot (kernels.py:1220-1350): memory
// mix, posterior, new edge messages; returns the hard decision.  No branch: a
// slot beyond the variable count has every edge on the dummy slot, a positive
// prior and a positive posterior, so its decision stays 0.
template <typename M, int MAXDV, bool STORE = true>
__device__ __forceinline__ uint32_t slot_var(M* msg, const uint32_t (&vp)[MAXDV], uint32_t dummy,
                                             typename MsgT<M>::A l0, typename MsgT<M>::A gam, int mix_mode,
                                             typename MsgT<M>::A& post, typename MsgT<M>::A* lm_out = nullptr,
                                             typename MsgT<M>::A* sum_out = nullptr) {
  using IO = MsgT<M>;
  using A = typename IO::A;
  const A lm = memory_mix<A>(mix_mode, gam, l0, post);
  if (lm_out) *lm_out = lm;
  A nv[MAXDV];
  A sum = A(0);
#pragma unroll
  for (int j = 0; j < MAXDV; ++j) {
    nv[j] = IO::ld(msg[vp[j]]);
    sum = (vp[j] != dummy) ? add_rn(sum, nv[j]) : sum;  // absent edges read the dummy slot
  }
  if (sum_out) *sum_out = sum;
  const A pv = add_rn(lm, sum);
  post = pv;
  if constexpr (STORE) {
#pragma unroll
    for (int j = 0; j < MAXDV; ++j) msg[vp[j]] = IO::st(add_rn(lm, sub_rn(sum, nv[j])));
  }
  return pv <= A(0) ? 1u : 0u;
}

// The variable-to-check messages of a variable pass that skipped them (slot_var with
// STORE false): the incoming messages are reloaded (still in their slots) and summed in
// the same order, so the values are those the pass would have stored.
template <typename M, int MAXDV>
__device__ __forceinline__ void slot_var_store(M* msg, const uint32_t (&vp)[MAXDV], uint32_t dummy,
                                               typename MsgT<M>::A lm) {
  using IO = MsgT<M>;
  using A = typename IO::A;
  A nv[MAXDV];
  A sum = A(0);
#pragma unroll
  for (int j = 0; j < MAXDV; ++j) {
    nv[j] = IO::ld(msg[vp[j]]);
    sum = (vp[j] != dummy) ? add_rn(sum, nv[j]) : sum;
  }
#pragma unroll
  for (int j = 0; j < MAXDV; ++j) msg[vp[j]] = IO::st(add_rn(lm, sub_rn(sum, nv[j])));
}

// The variables in `flips` (bit k: variable t + k G) changed their hard decision:
// flip their checks' mis bits and add +-1 per check to dunsat (the atomic's old
// value says whether the check was unsatisfied).
template <typename M, int MAXDC, int VPT, int MAXDV>
__device__ __forceinline__ void slot_flips(uint32_t* mis, const uint32_t (&vpos)[VPT][MAXDV], uint32_t dummy,
                                           uint32_t flips, int& dunsat, int VC) {
#pragma unroll
  for (int kk = 0; kk < VPT; ++kk) {
    if ((flips >> kk) & 1u) {
#pragma unroll
      for (int j = 0; j < MAXDV; ++j) {
        uint32_t q = vpos[kk][j];
        if (q != dummy) {
#pragma unroll
          for (int r = 1; r < MAXDC / VecIO<M>::N; ++r) q = q >= (uint32_t)VC ? q - (uint32_t)VC : q;
          const uint32_t c = q / (uint32_t)VecIO<M>::N;
          const uint32_t bit = 1u << (c & 31u);
          const uint32_t old = atomicXor(mis + (c >> 5), bit);
          dunsat += (old & bit) ? -1 : 1;
        }
      }
    }
  }
}

// The multi-shot decode loop of one block (= one group of G = blockDim.x threads).
template <typename M, int MAXDC, int VPT, int MAXDV, int NS>
__device__ __forceinline__ void run_slots(const DevGraph& g, const DevArgs& a, unsigned char* smem) {
  static_assert(MAXDC > 0, "the two-shot kernel moves check rows as 16-byte chunks");
  using IO = MsgT<M>;
  using A = typename IO::A;

  const int C = g.C, V = g.V;
  const uint8_t* s_chk_deg = smem + a.off_chk_deg;
  const float* s_llr = reinterpret_cast<const float*>(smem + a.off_llr);
  const int G = blockDim.x;
  const int t = threadIdx.x;
  const int lane = t & 31;
  const int warp = t >> 5;
  const int nwarps = G >> 5;
  const int W = (V + 31) >> 5;
  const int Wc = (C + 31) >> 5;
  const int S = a.stop_nconv;
  const int pre = a.pre_iter;
  const int VC = VecIO<M>::N * C;
  const A beta = A(a.beta);
  const bool first_from_table = a.first_table && a.llr_shot == nullptr;
  const M* first_tab = reinterpret_cast<const M*>(smem + a.off_first);
  const int legs_stop = (a.legs_end > 0 && a.legs_end < a.num_sets) ? a.legs_end : a.num_sets;

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

  unsigned char* region0 = smem + a.off_group0;
  auto msg_of = [&](int s) { return reinterpret_cast<M*>(region0 + s * a.group_bytes + a.g_msg); };
  auto mis_of = [&](int s) { return reinterpret_cast<uint32_t*>(region0 + s * a.group_bytes + a.g_par); };
  auto best_of = [&](int s) { return reinterpret_cast<uint32_t*>(region0 + s * a.group_bytes + a.g_best); };
  auto first_of = [&](int s) { return reinterpret_cast<uint32_t*>(region0 + s * a.group_bytes + a.g_first); };
  auto red_of = [&](int s) { return reinterpret_cast<long long*>(region0 + s * a.group_bytes + a.g_red); };
  auto unsat_of = [&](int s) { return reinterpret_cast<int*>(red_of(s) + 3); };
  auto s1_of = [&](int s) { return reinterpret_cast<A*>(region0 + s * a.group_bytes + a.g_s1); };

  // every slot's mis bits and unsatisfied count start at 0 (set-ups adjust them by differences)
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    for (int w = t; w < Wc; w += G) mis_of(s)[w] = 0u;
    if (t == 0) {
      *unsat_of(s) = 0;
      red_of(s)[0] = 0;
      red_of(s)[4] = 0;
    }
  }
  __syncthreads();

  SlotState<A, VPT> st[NS];

  // ---------------------------------------------------------------- events
  // Everything below runs under group-uniform control: each thread holds the
  // same control values, so barriers inside are reached by every thread.

  // Weight of the owned variables decided 1, in 2^-32 units (decoder.py:741-753).
  auto owned_weight = [&](const SlotState<A, VPT>& x) {
    long long w = 0;
#pragma unroll
    for (int k = 0; k < VPT; ++k) {
      const int v = t + k * G;
      if (v < V && ((x.hmask >> k) & 1u)) w += weight_units(x.llr_row ? __ldg(x.llr_row + v) : s_llr[v]);
    }
    return w;
  };

  // Map queue position q (thread 0's) to a shot index and broadcast it: B when the
  // queue is exhausted, -1 for an order entry that is not a shot index (skipped).
  auto claim = [&](SlotState<A, VPT>& x, int s, int q_issued) -> long long {
    long long* red = red_of(s);
    if (t == 0) {
      const long long q = (long long)q_issued;
      const long long qn = a.queue_len ? (long long)max(0, min(*a.queue_len, (int)a.B)) : a.B;
      long long sb = q < qn ? q : a.B;
      if (q < qn && a.order) {
        sb = (long long)a.order[q];
        if (sb < 0 || sb >= a.B) sb = -1;
      }
      reinterpret_cast<volatile long long*>(red)[1 + x.claim] = sb;
    }
    __syncthreads();
    const long long b = reinterpret_cast<volatile long long*>(red)[1 + x.claim];
    x.claim ^= 1;
    return b;
  };

  // Set-up of shot x.b (decoder.py:3429-3478): inputs, bit sets, mis bits.
  auto setup_shot = [&](SlotState<A, VPT>& x, int s) {
    const long long b = x.b;
    const uint8_t* syn_row = a.syn + b * (long long)C;
    x.llr_row = a.llr_shot ? a.llr_shot + b * (long long)V : nullptr;
    x.best_w = LLONG_MAX;
    x.found = 0;
    x.iters = 0;
    x.hard_src = HARD_ZERO;
    int has_best_raw = 0;
    const unsigned char* sst = a.resume ? a.resume + b * (long long)a.state_stride : nullptr;
    uint32_t* best = best_of(s);
    uint32_t* first = first_of(s);
    if (sst) {
      // continue a shot suspended after an earlier phase
      const int* hdr = reinterpret_cast<const int*>(sst);
      x.found = hdr[0];
      x.iters = hdr[1];
      x.hard_src = hdr[2];
      has_best_raw = hdr[3];
      x.best_w = *reinterpret_cast<const long long*>(sst + 16);
      const uint32_t* bits = reinterpret_cast<const uint32_t*>(sst + 32);
      if (lane < VPT) {
        const int w = warp + lane * nwarps;
        if (w < W) {
          best[w] = bits[w];
          first[w] = bits[W + w];
        }
      }
      const A* sp = reinterpret_cast<const A*>(sst + state_post_offset(V));
#pragma unroll
      for (int k = 0; k < VPT; ++k) {
        const int v = t + k * G;
        x.post[k] = v < V ? sp[v] : A(1);  // variable slots beyond V keep a positive posterior
      }
    } else {
      if (lane < VPT) {
        const int w = warp + lane * nwarps;
        if (w < W) {
          best[w] = 0u;
          first[w] = 0u;
        }
      }
#pragma unroll
      for (int k = 0; k < VPT; ++k) {
        const int v = t + k * G;
        A p0 = A(1);  // variable slots beyond V keep a positive posterior
        if (v < V) {
          if (a.init_post) p0 = A(__ldg(a.init_post + b * (long long)V + v));
          else p0 = x.llr_row ? A(__ldg(x.llr_row + v)) : A(s_llr[v]);
        }
        x.post[k] = p0;
      }
    }
    // syndrome bits of the owned checks, four loads in flight per round
    uint32_t synm = 0;
    for (int k = 0, c = t; c < C; k += 4, c += 4 * G) {
      const uint32_t s0 = syn_row[c];
      const uint32_t s1 = c + G < C ? (uint32_t)syn_row[c + G] : 0u;
      const uint32_t s2 = c + 2 * G < C ? (uint32_t)syn_row[c + 2 * G] : 0u;
      const uint32_t s3 = c + 3 * G < C ? (uint32_t)syn_row[c + 3 * G] : 0u;
      synm |= ((s0 & 1u) | ((s1 & 1u) << 1) | ((s2 & 1u) << 2) | ((s3 & 1u) << 3)) << k;
    }
    x.synm = synm;
    // Decisions restart at 0, so each check's mis bit is its syndrome bit; the
    // unsatisfied count changes by the difference of the words' popcounts.
    // (Every thread read the count before the claim's barrier.)
    uint32_t* mis = mis_of(s);
    int d = 0;
    for (int k = 0; k * G < C; ++k) {
      const int c = t + k * G;
      const unsigned m = __ballot_sync(0xffffffffu, c < C && ((synm >> k) & 1u));
      const int w = warp + k * nwarps;
      if (lane == 0 && w < Wc) {
        d += __popc(m) - __popc(mis[w]);
        mis[w] = m;
      }
    }
    if (lane == 0 && d != 0) atomicAdd(unsat_of(s), d);
    x.hmask = 0u;
    x.hmask_sel = 0u;
    x.sel_seen = false;
    x.s1_ok = false;
    x.has_best = has_best_raw != 0;
    x.stopped = false;
    // a shot resumed at leg 0 was solved by the pre-iterations if it found a solution there
    x.solved_pre = (a.resume && a.legs_begin == 0) ? x.found > 0 : false;
    x.phase = a.resume ? a.legs_begin : -1;
  };

  // Outputs of shot x.b (decoder.py:3839-3873) and the optional saved state.
  auto write_outputs = [&](SlotState<A, VPT>& x, int s) {
    const long long b = x.b;
    uint32_t* best = best_of(s);
    uint32_t* first = first_of(s);
    __syncwarp();
    if (a.suspend && (!a.suspend_unsolved || x.stopped)) {
      unsigned char* sst = a.suspend + b * (long long)a.state_stride;
      if (t == 0) {
        int* hdr = reinterpret_cast<int*>(sst);
        hdr[0] = x.found;
        hdr[1] = x.iters;
        hdr[2] = x.hard_src;
        hdr[3] = x.has_best ? 1 : 0;
        *reinterpret_cast<long long*>(sst + 16) = x.best_w;
      }
      uint32_t* bits = reinterpret_cast<uint32_t*>(sst + 32);
      if (lane < VPT) {
        const int w = warp + lane * nwarps;
        if (w < W) {
          bits[w] = best[w];
          bits[W + w] = first[w];
        }
      }
      A* sp = reinterpret_cast<A*>(sst + state_post_offset(V));
#pragma unroll
      for (int k = 0; k < VPT; ++k) {
        const int v = t + k * G;
        if (v < V) sp[v] = x.post[k];
      }
    }
    const uint32_t* src_bits = x.has_best ? best : first;
    const bool from_post = !x.has_best && a.last_leg && x.hard_src == HARD_POST;
    const bool zero_bits = !x.has_best && a.last_leg && x.hard_src != HARD_POST;
    if (a.errors) {
      uint8_t* erow = a.errors + b * (long long)V;
#pragma unroll
      for (int k = 0; k < VPT; ++k) {
        const int v = t + k * G;
        if (v < V) {
          uint8_t e;
          if (from_post) e = x.post[k] <= A(0) ? 1 : 0;
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
        if (from_post) m = __ballot_sync(0xffffffffu, v0 + lane < V && x.post[k] <= A(0));
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
          if constexpr (sizeof(A) == 8) reinterpret_cast<double*>(a.last_post)[b * (long long)V + v] = x.post[k];
          else reinterpret_cast<float*>(a.last_post)[b * (long long)V + v] = x.post[k];
        }
      }
    }
    if (t == 0) {
      if (a.weights)
        a.weights[b] = x.has_best ? __ll2float_rn(x.best_w) * 2.3283064365386963e-10f  // 2^-32
                                  : __int_as_float(0x7f800000);
      if (a.wfixed) a.wfixed[b] = x.has_best ? x.best_w : LLONG_MAX;
      a.found[b] = x.found;
      a.iters[b] = x.iters;
    }
  };

  enum { EV_NONE, EV_PHASE_DONE, EV_START_PHASE, EV_SHOT_DONE, EV_NEW_SHOT };

  // Process one slot's events until it runs a phase again or retires.
  auto events = [&](SlotState<A, VPT>& x, int s, int ev) {
    while (ev != EV_NONE) {
      if (ev == EV_PHASE_DONE) {
        // first-leg hard decision: after the pre-iterations, or after relay leg 0 when there
        // were none (decoder.py:3595-3598, 3807-3810)
        if (!a.last_leg && (x.phase < 0 || (x.phase == 0 && pre == 0))) {
          uint32_t* first = first_of(s);
          if (x.hard_src == HARD_POST) {
            ballot_post<A, VPT>(x.post, first, warp, lane, G, V);
          } else {
            const uint32_t* best = best_of(s);
            __syncwarp();
            if (lane < VPT) {
              const int w = warp + lane * nwarps;
              if (w < W) first[w] = x.hard_src == HARD_BEST ? best[w] : 0u;
            }
          }
        }
        ev = EV_START_PHASE;
        if (x.phase < 0) {
          if (x.found >= S || a.skip_legs) {
            ev = EV_SHOT_DONE;
          } else {
            x.solved_pre = x.found > 0;
            if (!x.solved_pre && a.suspend_unsolved) {
              x.stopped = true;
              ev = EV_SHOT_DONE;
            }
          }
        }
        if (ev == EV_START_PHASE) x.phase += 1;
      } else if (ev == EV_START_PHASE) {
        // Phase -1: the pre-iterations (decoder.py:3480-3616); phase l >= 0: relay leg l
        // (decoder.py:3672-3837).
        if (x.phase >= legs_stop || (x.phase >= 0 && x.found >= S)) {
          ev = EV_SHOT_DONE;
          continue;
        }
        int sought;
        x.gs = 0.f;
        if (x.phase < 0) {
          x.max_iter = pre;
          x.grow = a.gamma_pre ? a.gamma_pre + x.b * (long long)V : nullptr;
          x.gs = a.gamma0;
          sought = 1;
        } else {
          sought = x.found + 1;
          x.max_iter = a.set_max_iter;
          x.grow = (a.gamma_legs_shot && x.phase < a.n_shot_legs)
                       ? a.gamma_legs_shot +
                             (x.b * (long long)a.shot_leg_rows + min(x.phase, a.shot_leg_rows - 1)) * V
                       : a.gamma_legs + (long long)x.phase * V;
          if (x.solved_pre && x.phase < a.solved_legs) {
            x.grow = nullptr;
            x.gs = a.solved_gamma;
          }
        }
        if (x.max_iter <= 0) {
          // freeze_finished_lanes_kernel(count_iteration=False) after an empty phase
          if (x.found >= min(sought, S)) x.hard_src = HARD_BEST;
          ev = EV_PHASE_DONE;
        } else {
          // memory strengths of this phase: loaded here, first used by the variable pass
#pragma unroll
          for (int k = 0; k < VPT; ++k) {
            const int v = t + k * G;
            x.gam[k] = A(x.gs);
            if (v < V && x.grow) x.gam[k] = A(__ldg(x.grow + v));
          }
          if (!first_from_table) {
            // message init mu_e = llr[var(e)] (kernels.py:904-1000), read by the next check pass
            M* msg = msg_of(s);
#pragma unroll
            for (int k = 0; k < VPT; ++k) {
              const int v = t + k * G;
              if (v < V) {
                const M m0 = IO::st(x.llr_row ? A(__ldg(x.llr_row + v)) : A(s_llr[v]));
#pragma unroll
                for (int j = 0; j < MAXDV; ++j) msg[vpos[k][j]] = m0;
              }
            }
            __syncthreads();
          }
          x.it = 0;
          x.run = true;
          ev = EV_NONE;
        }
      } else if (ev == EV_SHOT_DONE) {
        x.run = false;
        int q = 0;
        if (t == 0) q = atomicAdd(a.queue, 1);  // latency overlaps the output writes
        if (x.b >= 0) write_outputs(x, s);
        x.b = claim(x, s, q);
        if (x.b >= a.B) {
          ev = EV_NONE;  // the queue is empty: the slot retires
        } else {
          ev = x.b < 0 ? EV_SHOT_DONE : EV_NEW_SHOT;
        }
      } else {  // EV_NEW_SHOT
        setup_shot(x, s);
        ev = EV_START_PHASE;
      }
    }
  };

  // ---------------------------------------------------------------- passes
  // Check pass of slot x (c2v min-sum, or the first-pass table at a phase's first
  // iteration), two owned rows per step so two rows' dependency chains interleave.
  auto check_pass = [&](SlotState<A, VPT>& x, int s) {
    const A alpha = a.use_alpha ? A(__ldg(a.alpha + x.it)) : A(1);
    const bool tab = first_from_table && x.it == 0;
    M* msg = msg_of(s);
    int k = 0;
    for (; t + (k + 1) * G < C; k += 2) {
      const int c0 = t + k * G, c1 = c0 + G;
      const int d0 = s_chk_deg[c0], d1 = s_chk_deg[c1];
      slot_check_row<M, MAXDC>(msg, first_tab, tab, c0, C, d0, (int)((x.synm >> k) & 1u), alpha, a.use_alpha,
                               a.use_beta, beta);
      slot_check_row<M, MAXDC>(msg, first_tab, tab, c1, C, d1, (int)((x.synm >> (k + 1)) & 1u), alpha,
                               a.use_alpha, a.use_beta, beta);
    }
    if (t + k * G < C)  // the last owned row when their number is odd
      slot_check_row<M, MAXDC>(msg, first_tab, tab, t + k * G, C, s_chk_deg[t + k * G], (int)((x.synm >> k) & 1u),
                               alpha, a.use_alpha, a.use_beta, beta);
  };

  // Variable pass of slot x, straight-line over the owned variables: the decisions are
  // collected in a mask and the few flips applied after the loop, so no branch splits the
  // loop body.  Ends with this thread's share of the unsatisfied-check count.
  // With DEFER the outgoing messages are not stored (see the one-shot schedule below);
  // the memory mixes are kept in the slot's shared lmk array (each thread's own entries, out
  // of its registers) for slot_var_store.  A DEFER pass of a one-shot
  // group whose first check pass came from the table also keeps each variable's sum of
  // incoming messages in the slot's s1 array: those are the first-pass sums of every relay
  // leg of the shot (the table and the shot's syndrome signs do not change between legs).
  auto lmk_of = [&](int s) { return s1_of(s) + VPT * G; };  // memory mixes kept for deferred stores
  auto var_pass = [&](SlotState<A, VPT>& x, int s, auto defer) {
    constexpr bool DEFER = decltype(defer)::value;
    M* msg = msg_of(s);
    A* s1 = s1_of(s);
    const bool keep_sums = DEFER && NS == 1 && first_from_table;
    uint32_t hnew = 0u;
#pragma unroll
    for (int kk = 0; kk < VPT; ++kk) {
      const int v = t + kk * G;
      const A l0 = x.llr_row ? (v < V ? A(__ldg(x.llr_row + v)) : A(1)) : (v < V ? A(s_llr[v]) : A(1));
      A sum = A(0);
      hnew |= slot_var<M, MAXDV, !DEFER>(msg, vpos[kk], dummy, l0, x.gam[kk], a.mix_mode, x.post[kk],
                                         DEFER ? lmk_of(s) + v : nullptr, keep_sums ? &sum : nullptr)
              << kk;
      if (keep_sums) s1[v] = sum;  // read back only by this thread (its own variables)
    }
    if (keep_sums) x.s1_ok = true;
    const uint32_t flips = hnew ^ x.hmask;
    x.hmask = hnew;
    int dun = 0;
    if (flips) slot_flips<M, MAXDC, VPT, MAXDV>(mis_of(s), vpos, dummy, flips, dun, VC);
    if (dun != 0) atomicAdd(unsat_of(s), dun);
  };

  // A relay leg's first iteration once the shot's first-pass sums are kept (one-shot groups):
  // its check pass would copy the block's table with the shot's syndrome signs, the same
  // messages as at every earlier leg's first iteration, and its variable pass would sum them
  // in the same order again, so both are replaced by the kept sums.  The posterior, decision
  // and memory mix are those var_pass computes; lmk serves the deferred stores.
  auto var_pass_quick = [&](SlotState<A, VPT>& x, int s) {
    const A* s1 = s1_of(s);
    uint32_t hnew = 0u;
#pragma unroll
    for (int kk = 0; kk < VPT; ++kk) {
      const int v = t + kk * G;
      const A l0 = v < V ? A(s_llr[v]) : A(1);  // first pass from the table: no per-shot priors
      const A lm = memory_mix<A>(a.mix_mode, x.gam[kk], l0, x.post[kk]);
      lmk_of(s)[v] = lm;
      const A pv = add_rn(lm, s1[v]);
      x.post[kk] = pv;
      hnew |= (pv <= A(0) ? 1u : 0u) << kk;
    }
    const uint32_t flips = hnew ^ x.hmask;
    x.hmask = hnew;
    int dun = 0;
    if (flips) slot_flips<M, MAXDC, VPT, MAXDV>(mis_of(s), vpos, dummy, flips, dun, VC);
    if (dun != 0) atomicAdd(unsat_of(s), dun);
  };

  // The first check pass from the table (the messages a quick first iteration skipped).
  auto table_copy = [&](SlotState<A, VPT>& x, int s) {
    M* msg = msg_of(s);
    for (int k = 0; t + k * G < C; ++k) {
      const int c = t + k * G;
      slot_check_row<M, MAXDC>(msg, first_tab, true, c, C, s_chk_deg[c], (int)((x.synm >> k) & 1u), A(1), false,
                               false, beta);
    }
  };

  // After slot x's variable pass and the barrier: the iteration's convergence test,
  // selection and freeze.  Returns the slot's next event.
  auto after_var = [&](SlotState<A, VPT>& x, int s) -> int {
    x.it += 1;
    const bool conv = *reinterpret_cast<volatile int*>(unsat_of(s)) == 0;
    if (conv) {
      // check_and_select_kernel (kernels.py:609-741).  Decisions equal to the shot's last
      // selection's have its weight, so the best cannot change: after the shot's first selection
      // the "decisions differ" test comes first (one OR-barrier) and the weight sum, with a second
      // barrier, only when they do.  The sum goes to red[0] or red[4], alternating: once a
      // selection's sum barrier has passed, the other entry's last readers (the previous
      // selection's) are done and thread 0 clears it, so no pass between two selections has to.
      long long* wsum = red_of(s) + (x.wsel ? 4 : 0);
      auto add_weight = [&]() {
        long long w = owned_weight(x);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
        if (lane == 0 && w != 0) atomicAdd(reinterpret_cast<unsigned long long*>(wsum), (unsigned long long)w);
        __syncthreads();
      };
      bool select = true;
      if (x.sel_seen) {
        select = __syncthreads_or(x.hmask != x.hmask_sel) != 0;
        if (select) add_weight();
      } else {
        add_weight();
      }
      if (select) {
        if (t == 0) red_of(s)[x.wsel ? 0 : 4] = 0;
        x.hmask_sel = x.hmask;
        x.sel_seen = true;
        const long long tot = *reinterpret_cast<volatile long long*>(wsum);
        if (!x.has_best || tot < x.best_w) {
          x.best_w = tot;
          x.has_best = true;
          ballot_post<A, VPT>(x.post, best_of(s), warp, lane, G, V);
        }
        x.wsel ^= 1;
      }
      // freeze_finished_lanes_kernel (kernels.py:746-847): a convergence always freezes
      x.found += 1;
      x.iters += x.it;
      x.hard_src = HARD_BEST;
      x.run = false;
      x.synced = true;  // a selection barrier followed every thread's read of the count
      return EV_PHASE_DONE;
    }
    x.hard_src = HARD_POST;
    x.synced = false;
    if (x.it >= x.max_iter) {
      x.iters += x.max_iter;
      x.run = false;
      return EV_PHASE_DONE;
    }
    return EV_NONE;
  };

  // ---------------------------------------------------------------- schedule
  // ev[s]: the event slot s has pending; every slot starts by claiming a shot.
  int ev[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    st[s].claim = 0;
    st[s].wsel = 0;
    st[s].run = false;
    st[s].b = -1;  // no shot yet: the first EV_SHOT_DONE only claims
    st[s].has_best = false;
    st[s].stopped = false;
    st[s].s1_ok = false;
    st[s].synced = false;
    ev[s] = EV_SHOT_DONE;
  }
  if constexpr (NS == 1) {
    // one shot: check pass, barrier, variable pass, barrier, events
    while (true) {
      if (ev[0] != EV_NONE) events(st[0], 0, ev[0]);
      if (!st[0].run) break;
      // A relay leg's first iteration usually converges (most legs of solved shots repeat
      // their solution), and then its outgoing messages are never read: the next leg restarts
      // them.  Those passes store them only once the iteration is known not to have converged.
      const bool defer = st[0].phase >= 0 && st[0].it == 0;
      // From the shot's second leg in this launch on, that iteration needs no check pass.
      const bool quick = defer && st[0].s1_ok;
      if (quick) {
        // the variable pass updates the unsatisfied count: every thread's read of it in the
        // last iteration's test must come first (a convergence's selection ordered them)
        if (!st[0].synced) __syncthreads();
        var_pass_quick(st[0], 0);
      } else {
        check_pass(st[0], 0);
        __syncthreads();
        if (defer) var_pass(st[0], 0, std::true_type{});
        else var_pass(st[0], 0, std::false_type{});
      }
      __syncthreads();
      ev[0] = after_var(st[0], 0);
      if (defer && st[0].run) {
        M* msg = msg_of(0);
        if (quick) {
          table_copy(st[0], 0);  // the incoming messages the deferred stores re-sum
          __syncthreads();
        }
#pragma unroll
        for (int kk = 0; kk < VPT; ++kk) slot_var_store<M, MAXDV>(msg, vpos[kk], dummy, lmk_of(0)[t + kk * G]);
        __syncthreads();  // the next check pass reads them
      }
    }
  } else {
    // Two shots: one check pass of both slots (their rows interleaved), a barrier, one
    // variable pass of both, a barrier, then each slot's events.
    while (true) {
      bool any = false;
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        if (ev[s] != EV_NONE) events(st[s], s, ev[s]);
        any = any || st[s].run;
      }
      if (!any) break;

      // check pass of every running slot (c2v min-sum, or the first-pass table)
      A alpha[NS];
      bool tab[NS];
      bool fused = true;
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        alpha[s] = (a.use_alpha && st[s].run) ? A(__ldg(a.alpha + st[s].it)) : A(1);
        tab[s] = first_from_table && st[s].it == 0;
        fused = fused && st[s].run && !tab[s];
      }
      {
        // ROWS owned rows per step (two for one slot): straight-line code with
        // ROWS * NS independent chains when every slot computes
        constexpr int ROWS = NS == 1 ? 2 : 1;
        int k = 0;
        for (; t + (k + ROWS - 1) * G < C; k += ROWS) {
          if (fused) {
#pragma unroll
            for (int r = 0; r < ROWS; ++r) {
              const int c = t + (k + r) * G;
              const int deg = s_chk_deg[c];
#pragma unroll
              for (int s = 0; s < NS; ++s)
                slot_check_row<M, MAXDC>(msg_of(s), first_tab, false, c, C, deg, (int)((st[s].synm >> (k + r)) & 1u),
                                         alpha[s], a.use_alpha, a.use_beta, beta);
            }
          } else {
#pragma unroll
            for (int r = 0; r < ROWS; ++r) {
              const int c = t + (k + r) * G;
              const int deg = s_chk_deg[c];
#pragma unroll
              for (int s = 0; s < NS; ++s)
                if (st[s].run)
                  slot_check_row<M, MAXDC>(msg_of(s), first_tab, tab[s], c, C, deg,
                                           (int)((st[s].synm >> (k + r)) & 1u), alpha[s], a.use_alpha, a.use_beta,
                                           beta);
            }
          }
        }
        if constexpr (ROWS > 1) {
          if (t + k * G < C) {  // the last owned row when their number is odd
            const int c = t + k * G;
            const int deg = s_chk_deg[c];
#pragma unroll
            for (int s = 0; s < NS; ++s)
              if (st[s].run)
                slot_check_row<M, MAXDC>(msg_of(s), first_tab, tab[s], c, C, deg, (int)((st[s].synm >> k) & 1u),
                                         alpha[s], a.use_alpha, a.use_beta, beta);
          }
        }
      }
      __syncthreads();

      // variable pass of every running slot
      int dun[NS];
      bool all_run = true;
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        dun[s] = 0;
        all_run = all_run && st[s].run;
      }
      // Straight-line over the owned variables (and slots): the decisions are collected in a
      // mask and the few flips handled after the loop, so no branch splits the loop body.
      uint32_t hnew[NS];
#pragma unroll
      for (int s = 0; s < NS; ++s) hnew[s] = 0u;
      auto var_slot = [&](int s, int kk, A l0s) {
        const int v = t + kk * G;
        const A l0 = st[s].llr_row ? (v < V ? A(__ldg(st[s].llr_row + v)) : A(1)) : l0s;
        hnew[s] |= slot_var<M, MAXDV>(msg_of(s), vpos[kk], dummy, l0, st[s].gam[kk], a.mix_mode, st[s].post[kk])
                   << kk;
      };
      if (all_run) {
#pragma unroll
        for (int kk = 0; kk < VPT; ++kk) {
          const int v = t + kk * G;
          const A l0s = v < V ? A(s_llr[v]) : A(1);
#pragma unroll
          for (int s = 0; s < NS; ++s) var_slot(s, kk, l0s);
        }
      } else {
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          if (!st[s].run) continue;
#pragma unroll
          for (int kk = 0; kk < VPT; ++kk) {
            const int v = t + kk * G;
            var_slot(s, kk, v < V ? A(s_llr[v]) : A(1));
          }
        }
      }
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        if (st[s].run) {
          const uint32_t flips = hnew[s] ^ st[s].hmask;
          st[s].hmask = hnew[s];
          if (flips) slot_flips<M, MAXDC, VPT, MAXDV>(mis_of(s), vpos, dummy, flips, dun[s], VC);
          if (dun[s] != 0) atomicAdd(unsat_of(s), dun[s]);
        }
        if (t == 0) red_of(s)[0] = 0;  // the next selection's sum; its last reader passed a barrier since
      }
      __syncthreads();

      // the iteration's convergence test, selection and freeze, per slot
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        SlotState<A, VPT>& x = st[s];
        ev[s] = EV_NONE;
        if (!x.run) continue;
        x.it += 1;
        const bool conv = *reinterpret_cast<volatile int*>(unsat_of(s)) == 0;
        if (conv) {
          // check_and_select_kernel (kernels.py:609-741): the weight sum and the test for
          // decisions unchanged since the shot's last selection share one barrier
          long long w = owned_weight(x);
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
          if (lane == 0 && w != 0) atomicAdd(reinterpret_cast<unsigned long long*>(red_of(s)), (unsigned long long)w);
          const bool differ = __syncthreads_or(x.hmask != x.hmask_sel) != 0;
          if (!x.sel_seen || differ) {
            // decisions equal to the last selection's have its weight: the best cannot change
            x.hmask_sel = x.hmask;
            x.sel_seen = true;
            const long long tot = *reinterpret_cast<volatile long long*>(red_of(s));
            if (!x.has_best || tot < x.best_w) {
              x.best_w = tot;
              x.has_best = true;
              ballot_post<A, VPT>(x.post, best_of(s), warp, lane, G, V);
            }
          }
          // freeze_finished_lanes_kernel (kernels.py:746-847): a convergence always freezes
          x.found += 1;
          x.iters += x.it;
          x.hard_src = HARD_BEST;
          x.run = false;
          ev[s] = EV_PHASE_DONE;
        } else {
          x.hard_src = HARD_POST;
          if (x.it >= x.max_iter) {
            x.iters += x.max_iter;
            x.run = false;
            ev[s] = EV_PHASE_DONE;
          }
        }
      }
    }
  }
}

// One code, one group of NS shots per block (rbp_decode with groups_per_block 1),
// compiled for MINB resident blocks per SM (1, or 2 for one-shot groups).
template <typename M, int MAXDC, int VPT, int MAXDV, int NS, int MINB>
__global__ void __launch_bounds__(MINB == 2 ? max_slots_block_threads2(VPT) : max_slots_block_threads(VPT, NS, MAXDV),
                                  MINB)
relaybp_slots_kernel(DevGraph g, DevArgs a) {
  static_assert(MINB == 1 || (MINB == 2 && NS == 1), "two resident blocks per SM: one-shot groups only");
  extern __shared__ __align__(16) unsigned char smem[];
  load_block_tables(g, a, smem);
  __syncthreads();
  if (a.first_table) build_first_pass_table<M, MAXDC>(g, a, smem);
  run_slots<M, MAXDC, VPT, MAXDV, NS>(g, a, smem);
}

// Kernel for (check degree bound, variable degree, owned variables per thread,
// shots per group 1 or 2, resident blocks per SM 1 or 2), or null when this
// build has no such instantiation (two blocks per SM: one shot per group).
KernelFn pick_slots_f32(int dc, int dv, int vpt, int ns, int minb);
KernelFn pick_slots_f16(int dc, int dv, int vpt, int ns, int minb);
KernelFn pick_slots_bf16(int dc, int dv, int vpt, int ns, int minb);
KernelFn pick_slots_f64(int dc, int dv, int vpt, int ns, int minb);

}  // namespace rbpk

// Instantiation table of the block-per-group kernel for one message type
// (check rows of at most 8 or 16 slots; wider rows use relaybp_decode_kernel).
#define RBPK_SLOTS_DC_DV(M, DC, VPT, NS, MB)                                   \
  if (dv <= 3) return &rbpk::relaybp_slots_kernel<M, DC, VPT, 3, NS, MB>;      \
  if (dv <= 8) return &rbpk::relaybp_slots_kernel<M, DC, VPT, 8, NS, MB>;      \
  return nullptr;
#define RBPK_SLOTS_DC(M, VPT, NS, MB)                                          \
  if (dc <= 8) { RBPK_SLOTS_DC_DV(M, 8, VPT, NS, MB) }                         \
  if (dc <= 16) { RBPK_SLOTS_DC_DV(M, 16, VPT, NS, MB) }                       \
  return nullptr;
#define RBPK_SLOTS_VPT(M, NS)                                                  \
  switch (vpt) {                                                               \
    case 1: { RBPK_SLOTS_DC(M, 1, NS, 1) }                                     \
    case 2: { RBPK_SLOTS_DC(M, 2, NS, 1) }                                     \
    case 3: { RBPK_SLOTS_DC(M, 3, NS, 1) }                                     \
    case 4: { RBPK_SLOTS_DC(M, 4, NS, 1) }                                     \
    case 6: { RBPK_SLOTS_DC(M, 6, NS, 1) }                                     \
    case 8: { RBPK_SLOTS_DC(M, 8, NS, 1) }                                     \
    case 12: { RBPK_SLOTS_DC(M, 12, NS, 1) }                                   \
    case 16: { RBPK_SLOTS_DC(M, 16, NS, 1) }                                   \
    default: return nullptr;                                                   \
  }
#define RBPK_SLOTS_VPT_2PERSM(M)                                               \
  switch (vpt) {                                                               \
    case 1: { RBPK_SLOTS_DC(M, 1, 1, 2) }                                      \
    case 2: { RBPK_SLOTS_DC(M, 2, 1, 2) }                                      \
    case 3: { RBPK_SLOTS_DC(M, 3, 1, 2) }                                      \
    case 4: { RBPK_SLOTS_DC(M, 4, 1, 2) }                                      \
    case 6: { RBPK_SLOTS_DC(M, 6, 1, 2) }                                      \
    case 8: { RBPK_SLOTS_DC(M, 8, 1, 2) }                                      \
    case 12: { RBPK_SLOTS_DC(M, 12, 1, 2) }                                    \
    case 16: { RBPK_SLOTS_DC(M, 16, 1, 2) }                                    \
    default: return nullptr;                                                   \
  }

#define RBPK_DEFINE_PICK_SLOTS(NAME, M)                                        \
  rbpk::KernelFn rbpk::NAME(int dc, int dv, int vpt, int ns, int minb) {       \
    if (minb == 2) {                                                           \
      if (ns == 1) { RBPK_SLOTS_VPT_2PERSM(M) }                                \
      return nullptr;                                                          \
    }                                                                          \
    if (ns == 1) { RBPK_SLOTS_VPT(M, 1) }                                      \
    if (ns == 2) { RBPK_SLOTS_VPT(M, 2) }                                      \
    return nullptr;                                                            \
  }
