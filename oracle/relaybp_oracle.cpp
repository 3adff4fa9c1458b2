// CPU oracle for the Relay-BP-S decode path.  TEST INFRASTRUCTURE ONLY.
//
// This file restates, shot by shot and in plain sequential C++, what the
// reference decoder (quantum-supercomputing/pelagos, Python + Triton) computes
// for `RelayBPDecoder.decode()` with perf="throughput" and flood-fill
// scheduling.  It is the checker the CUDA path is compared against (tests,
// the smoke check and the CPU-baseline leg of the benchmark); it is never part
// of the product path.
//
// Followed reference code (file:line in the reference tree):
//   decode loop, legs, first/last-leg correction  src/pelagos/decoder.py:3394-3873
//   one BP iteration (alpha schedule)             src/pelagos/decoder.py:2610-2875
//   message init  mu = llr[edge_var], nu = 0      src/pelagos/kernels.py:904-1000
//   check-to-variable min-sum                     src/pelagos/kernels.py:1052-1215
//   variable-to-check + memory (gamma) mixing     src/pelagos/kernels.py:1220-1350
//   parity of hard decisions per check            src/pelagos/kernels.py:510-569
//   solution check and lowest-weight selection    src/pelagos/kernels.py:609-741
//   freeze / iteration counting                   src/pelagos/kernels.py:746-847
//   unfreeze, all-done                            src/pelagos/kernels.py:1005-1045
//   edge-centric graph (edge id = CSR position,
//   var_edges = argsort(edge_var) order)          src/pelagos/graph.py:101-211
//
// Deliberate, documented definitions where the reference's result depends on
// its launch configuration:
//   * solution weight: sum over set bits of wj, accumulated EXACTLY in 64-bit
//     fixed point (units of 2^-32, each wj rounded to the nearest unit), and
//     compared as integers; the reported float weight is the nearest float32.
//     (The reference sums float32 in a tile tree whose shape is autotuned,
//     kernels.py:687-704.)
//   * memory mixing rounding: `mix_mode` selects one rounding per operation
//     (0), or a fused multiply-add on the gamma*posterior term (1) or on the
//     (1-gamma)*llr term (2).
//   * the summation order of incoming check messages is the caller-supplied
//     `var_edges` order (the reference uses numpy's default argsort).
//
// Build: see oracle/Makefile (-O2 -ffp-contract=off -fopenmp).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <limits>
#include <omp.h>

namespace {

// ---------------------------------------------------------------- storage types
// IEEE binary16 and bfloat16 with round-to-nearest-even, from the format
// definitions.
struct half_t { uint16_t bits; };
struct bf16_t { uint16_t bits; };

inline float bits_to_float(uint32_t x) { float f; std::memcpy(&f, &x, 4); return f; }
inline uint32_t float_to_bits(float f) { uint32_t x; std::memcpy(&x, &f, 4); return x; }

inline uint16_t f32_to_f16(float f) {
  uint32_t x = float_to_bits(f);
  uint32_t sign = (x >> 16) & 0x8000u;
  uint32_t ax = x & 0x7fffffffu;
  if (ax >= 0x7f800000u) return (uint16_t)(sign | 0x7c00u | (ax > 0x7f800000u ? 0x200u : 0u));
  if (ax >= 0x477ff000u) return (uint16_t)(sign | 0x7c00u);  // >= 65520 rounds to inf
  if (ax < 0x38800000u) {                                    // below 2^-14: subnormal / zero
    double units = (double)bits_to_float(ax) * 16777216.0;   // multiples of 2^-24, exact
    double r = std::nearbyint(units);                        // ties to even
    return (uint16_t)(sign | (uint32_t)r);
  }
  uint32_t mant = ax & 0x7fffffu;
  uint32_t e = (ax >> 23) - 127u + 15u;
  uint32_t h = (e << 10) | (mant >> 13);
  uint32_t rem = mant & 0x1fffu;
  if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h++;
  return (uint16_t)(sign | h);
}

inline float f16_to_f32(uint16_t h) {
  uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
  uint32_t e = (h >> 10) & 0x1fu;
  uint32_t m = h & 0x3ffu;
  if (e == 0) {
    float v = (float)m * (1.0f / 16777216.0f);  // m * 2^-24, exact
    return sign ? -v : v;
  }
  if (e == 31) return bits_to_float(sign | 0x7f800000u | (m << 13));
  return bits_to_float(sign | ((e - 15u + 127u) << 23) | (m << 13));
}

inline uint16_t f32_to_bf16(float f) {
  uint32_t x = float_to_bits(f);
  if ((x & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((x >> 16) | 0x40u);
  uint32_t lsb = (x >> 16) & 1u;
  return (uint16_t)((x + 0x7fffu + lsb) >> 16);
}
inline float bf16_to_f32(uint16_t b) { return bits_to_float((uint32_t)b << 16); }

template <typename M> struct Msg;
template <> struct Msg<float> {
  static float load(float v) { return v; }
  static float store(float v) { return v; }
};
template <> struct Msg<double> {
  static double load(double v) { return v; }
  static double store(double v) { return v; }
};
template <> struct Msg<half_t> {
  static float load(half_t v) { return f16_to_f32(v.bits); }
  // saturate at +-65504 (the largest finite binary16) before rounding, as the kernel does
  static half_t store(float v) { return half_t{f32_to_f16(std::fmin(std::fmax(v, -65504.0f), 65504.0f))}; }
};
template <> struct Msg<bf16_t> {
  static float load(bf16_t v) { return bf16_to_f32(v.bits); }
  static bf16_t store(float v) { return bf16_t{f32_to_bf16(v)}; }
};

}  // namespace

extern "C" {

// Decode parameters (mirrors the reference constructor arguments that reach
// the decode loop).  All arrays are host memory.
struct rbo_params {
  int32_t pre_iter;        // iterations of the first (ordered-memory) phase
  int32_t num_sets;        // relay legs
  int32_t set_max_iter;    // iterations per relay leg
  int32_t stop_nconv;      // solutions to collect before a shot stops
  int32_t last_leg;        // 0: unconverged shots return the first leg's hard decision
  int32_t use_alpha;       // normalized min-sum: magnitude *= alpha_table[t]
  int32_t use_beta;        // offset min-sum: magnitude = max(magnitude - beta, 0)
  float beta;
  int32_t mix_mode;        // 0 separate roundings, 1 fma(g, post, (1-g) llr), 2 fma(1-g, llr, g post)
  int32_t msg_type;        // 0 f32, 1 f16, 2 bf16, 3 f64 (f64 also accumulates in f64)
  int32_t skip_relay_legs; // return right after the first phase
  int32_t num_threads;     // OpenMP threads (<= 0: library default)
};

// Graph in the reference's edge-centric form.  Edge e is the e-th nonzero of
// the CSR matrix; var_edges[var_ptr[v]..var_ptr[v+1]) lists v's edges in the
// order their messages are summed.
struct rbo_graph {
  int32_t C, V, E;
  const int32_t* chk_ptr;    // [C+1]
  const int32_t* edge_var;   // [E]
  const int32_t* var_ptr;    // [V+1]
  const int32_t* var_edges;  // [E]
};

// Per-decode inputs.  Optional arrays may be null.
struct rbo_inputs {
  int64_t B;
  const uint8_t* syndromes;      // [B, C]
  const float* llr;              // [V] prior LLRs (shared), or
  const float* llr_per_shot;     // [B, V] (prior_llr), overrides llr
  float gamma0;                  // first-phase memory strength (ignored when gamma_pre given)
  const float* gamma_pre;        // [B, V] first-phase memory strengths (init_gamma)
  const float* gamma_legs;       // [num_sets, V] leg memory strengths
  const float* gamma_legs_shot;  // [B, n_shot_legs, V] per-shot strengths for legs < n_shot_legs
  int32_t n_shot_legs;
  const float* init_posterior;   // [B, V]
  const float* alpha_table;      // [max(pre_iter, set_max_iter)] per-iteration alpha
};

struct rbo_outputs {
  uint8_t* errors;         // [B, V]
  float* weights;          // [B] (+inf when no solution)
  int64_t* weight_fixed;   // [B] exact weight in 2^-32 units (INT64_MAX when none), may be null
  int32_t* found_count;    // [B]
  int32_t* iterations;     // [B]
  double* last_posterior;  // [B, V], may be null
};

int rbo_decode(const rbo_graph* g, const rbo_params* p, const rbo_inputs* in, rbo_outputs* out);

}  // extern "C"

namespace {

template <typename A>
inline A mix(int mode, A g, A lp, A post) {
  A one_m = (A)1 - g;
  if (mode == 1) return std::fma(g, post, one_m * lp);
  if (mode == 2) return std::fma(one_m, lp, g * post);
  A a = one_m * lp;
  A b = g * post;
  return a + b;
}

inline int64_t weight_units(float w) {
  if (!std::isfinite(w)) return 0;  // reference: non-finite log-prior ratios weigh 0
  return (int64_t)std::llrint(std::ldexp((double)w, 32));
}

template <typename M, typename A>
struct ShotDecoder {
  const rbo_graph& g;
  const rbo_params& p;
  std::vector<M> mu, nu;
  std::vector<A> post, lam, llr, gamma;
  std::vector<int64_t> wfix;
  std::vector<uint8_t> hard, best, first_leg, check_ok, syn;

  ShotDecoder(const rbo_graph& g_, const rbo_params& p_) : g(g_), p(p_) {
    mu.resize(g.E); nu.resize(g.E);
    post.resize(g.V); lam.resize(g.V); llr.resize(g.V); gamma.resize(g.V);
    wfix.resize(g.V); hard.resize(g.V); best.resize(g.V); first_leg.resize(g.V);
    check_ok.resize(g.C); syn.resize(g.C);
  }

  // init_messages_with_priors_EB_kernel: nu = 0, mu = llr[edge_var[e]]
  void init_messages() {
    for (int e = 0; e < g.E; ++e) {
      nu[e] = Msg<M>::store((A)0);
      mu[e] = Msg<M>::store(llr[g.edge_var[e]]);
    }
  }

  // c2v_min_sum_btile_kernel for one lane
  void check_pass(A alpha) {
    const A BIG = (A)1e30;
    for (int i = 0; i < g.C; ++i) {
      int r0 = g.chk_ptr[i], r1 = g.chk_ptr[i + 1];
      if (r1 <= r0) continue;
      int neg = 0, cnt1 = 0;
      A min1 = BIG, min2 = BIG;
      for (int e = r0; e < r1; ++e) {
        A m = Msg<M>::load(mu[e]);
        neg ^= (m < (A)0) ? 1 : 0;
        A a = std::fabs(m);
        if (a < min1) { min2 = min1; min1 = a; cnt1 = 1; }
        else if (a == min1) { cnt1 += 1; }
        else if (a < min2) { min2 = a; }
      }
      A sign_prod = ((neg ^ syn[i]) & 1) ? (A)-1 : (A)1;
      bool deg1 = (r1 - r0) == 1;
      for (int e = r0; e < r1; ++e) {
        A m = Msg<M>::load(mu[e]);
        A sgn = (m >= (A)0) ? (A)1 : (A)-1;
        A a = std::fabs(m);
        A mag = (cnt1 == 1 && a == min1) ? min2 : min1;
        if (deg1) mag = (A)0;
        if (p.use_alpha) mag = alpha * mag;
        if (p.use_beta) mag = std::max(mag - (A)p.beta, (A)0);
        nu[e] = Msg<M>::store((sign_prod * sgn) * mag);
      }
    }
  }

  // v2c_and_gamma_btile_kernel for one lane (WRITE_HARD=True)
  void var_pass() {
    for (int j = 0; j < g.V; ++j) {
      A lm = mix<A>(p.mix_mode, gamma[j], llr[j], post[j]);
      A s = (A)0;
      for (int k = g.var_ptr[j]; k < g.var_ptr[j + 1]; ++k) s = s + Msg<M>::load(nu[g.var_edges[k]]);
      A pj = lm + s;
      post[j] = pj;
      hard[j] = pj <= (A)0 ? 1 : 0;
      lam[j] = lm;
      for (int k = g.var_ptr[j]; k < g.var_ptr[j + 1]; ++k) {
        int e = g.var_edges[k];
        mu[e] = Msg<M>::store(lm + (s - Msg<M>::load(nu[e])));
      }
    }
  }

  // parity_from_hard_* : all checks satisfied?
  bool parity_all_ok() {
    bool all = true;
    for (int i = 0; i < g.C; ++i) {
      int par = 0;
      for (int e = g.chk_ptr[i]; e < g.chk_ptr[i + 1]; ++e) par ^= hard[g.edge_var[e]];
      check_ok[i] = (uint8_t)(par == syn[i]);
      all = all && check_ok[i];
    }
    return all;
  }
};

template <typename M, typename A>
void decode_range(const rbo_graph& g, const rbo_params& p, const rbo_inputs& in,
                  rbo_outputs& out, int64_t b0, int64_t b1) {
  ShotDecoder<M, A> d(g, p);
  const int S = p.stop_nconv;
  for (int64_t b = b0; b < b1; ++b) {
    for (int i = 0; i < g.C; ++i) d.syn[i] = in.syndromes[b * g.C + i] & 1;
    for (int j = 0; j < g.V; ++j) {
      float l = in.llr_per_shot ? in.llr_per_shot[b * g.V + j] : in.llr[j];
      d.llr[j] = (A)l;
      d.wfix[j] = weight_units(l);
      d.post[j] = in.init_posterior ? (A)in.init_posterior[b * g.V + j] : (A)l;
      d.lam[j] = (A)l;
      d.hard[j] = 0; d.best[j] = 0; d.first_leg[j] = 0;
    }
    bool has_best = false;
    int64_t best_w = std::numeric_limits<int64_t>::max();
    int found = 0, valid = 0, sought = 1, iters = 0;
    bool active = true;

    // One phase (pre-iterations or a relay leg): up to `max_iter` iterations,
    // each followed by parity, selection and freeze (count_iteration=True).
    auto run_phase = [&](int max_iter) {
      for (int t = 0; t < max_iter && active; ++t) {
        A alpha = p.use_alpha ? (A)in.alpha_table[t] : (A)1;
        d.check_pass(alpha);
        d.var_pass();
        if (d.parity_all_ok()) {
          int64_t w = 0;
          for (int j = 0; j < g.V; ++j) if (d.post[j] <= (A)0) w += d.wfix[j];
          if (!has_best || w < best_w) {
            best_w = w; has_best = true;
            for (int j = 0; j < g.V; ++j) d.best[j] = d.post[j] <= (A)0 ? 1 : 0;
          }
          if (valid == 0) found += 1;
          valid = 1;
        }
        iters += 1;
        if (found >= std::min(sought, S)) {  // freeze_finished_lanes_kernel
          d.hard = d.best;
          active = false;
        }
      }
    };

    d.init_messages();
    for (int j = 0; j < g.V; ++j)
      d.gamma[j] = in.gamma_pre ? (A)in.gamma_pre[b * g.V + j] : (A)in.gamma0;
    valid = 0;
    run_phase(p.pre_iter);
    if (!p.last_leg) d.first_leg = d.hard;
    if (active && found >= std::min(sought, S)) { d.hard = d.best; active = false; }
    bool done = (found >= S) || p.skip_relay_legs;
    if (!done) {
      active = found < S;
      for (int leg = 0; leg < p.num_sets && found < S; ++leg) {
        sought = found + 1;
        const float* row = (leg < in.n_shot_legs && in.gamma_legs_shot)
                               ? in.gamma_legs_shot + ((size_t)b * in.n_shot_legs + leg) * g.V
                               : in.gamma_legs + (size_t)leg * g.V;
        for (int j = 0; j < g.V; ++j) d.gamma[j] = (A)row[j];
        if (active) d.init_messages();
        valid = 0;
        run_phase(p.set_max_iter);
        if (leg == 0 && p.pre_iter == 0 && !p.last_leg) d.first_leg = d.hard;
        active = found < S;
      }
    }
    const std::vector<uint8_t>& fallback = p.last_leg ? d.hard : d.first_leg;
    const std::vector<uint8_t>& e = has_best ? d.best : fallback;
    std::memcpy(out.errors + b * g.V, e.data(), g.V);
    if (has_best) {
      out.weights[b] = (float)std::ldexp((double)best_w, -32);
    } else {
      out.weights[b] = std::numeric_limits<float>::infinity();
    }
    if (out.weight_fixed) out.weight_fixed[b] = has_best ? best_w : std::numeric_limits<int64_t>::max();
    out.found_count[b] = found;
    out.iterations[b] = iters;
    if (out.last_posterior)
      for (int j = 0; j < g.V; ++j) out.last_posterior[b * g.V + j] = (double)d.post[j];
  }
}

template <typename M, typename A>
void decode_all(const rbo_graph& g, const rbo_params& p, const rbo_inputs& in, rbo_outputs& out) {
  const int64_t B = in.B;
  const int64_t chunk = 8;
  const int64_t nchunks = (B + chunk - 1) / chunk;
#pragma omp parallel for schedule(dynamic, 1) num_threads(p.num_threads > 0 ? p.num_threads : omp_get_max_threads())
  for (int64_t c = 0; c < nchunks; ++c) {
    int64_t b0 = c * chunk, b1 = std::min(B, b0 + chunk);
    decode_range<M, A>(g, p, in, out, b0, b1);
  }
}

}  // namespace

extern "C" int rbo_decode(const rbo_graph* g, const rbo_params* p, const rbo_inputs* in,
                          rbo_outputs* out) {
  if (!g || !p || !in || !out || in->B < 0) return 1;
  switch (p->msg_type) {
    case 0: decode_all<float, float>(*g, *p, *in, *out); return 0;
    case 1: decode_all<half_t, float>(*g, *p, *in, *out); return 0;
    case 2: decode_all<bf16_t, float>(*g, *p, *in, *out); return 0;
    case 3: decode_all<double, double>(*g, *p, *in, *out); return 0;
    default: return 2;
  }
}

// Element-wise conversions exposed for testing the storage rounding.
extern "C" void rbo_round_f16(const float* x, float* y, int64_t n) {
  for (int64_t i = 0; i < n; ++i) y[i] = f16_to_f32(f32_to_f16(x[i]));
}
extern "C" void rbo_round_bf16(const float* x, float* y, int64_t n) {
  for (int64_t i = 0; i < n; ++i) y[i] = bf16_to_f32(f32_to_bf16(x[i]));
}
