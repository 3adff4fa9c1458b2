// Learned relay-leg proposal: a 2-layer edge-conditioned message-passing
// network on the Tanner graph that maps a shot's syndrome and pre-iteration
// posterior to per-variable memory strengths for the first relay legs.
//
// The reference has no learned proposal.  Its interface is the one these
// strengths go through: per-shot leg gammas, used like explicit_gammas rows
// (src/pelagos/decoder.py:338-340, 481-491, 3685-3688) and bounded by
// gamma_dist_interval (src/pelagos/utils.py:128-160).
//
// Network (widths: node state H=64, message D=16; per shot):
//   z_v = (tanh(P_v/16), [P_v<=0], unsat_v, tanh(llr_v/16)), P clipped to +-1e4
//   t_v = 2[P_v<=0] + [|P_v|<8]                     edge type of v's edges
//   x_c = (s_c, mean_{v in c} z_v, 1)
//   g0  = relu(E x^)
//   layer l = 1, 2:
//     m_c = (W_l g^_c)^,  n_v = (sum_{c in M(v)} m_c)^
//     a_c = sum_{v in N(c)} G_l[t_v] * (n_v - m_c)
//     g_c = relu(g_c + U_l a^_c + b_l)
//   o_c = O . g2^_c,  r_v = sum_{c in M(v)} o_c / deg_v + Oz . z_v + ob
//   gamma_v = lo + (hi - lo) sigmoid(r_v)
// ^ = rounded to bf16.  Weights are bf16 (an fp32 master copy is what AdamW
// updates); every sum accumulates in fp32.
//
// Two implementations of the forward pass:
//   * training kernels: one thread per output element, fp32, activations kept
//     in device memory for the backward kernels (dense / gather / scatter
//     forward and backward, loss, AdamW);
//   * net_propose_kernel: the inference pass, one 512-thread block per SM
//     looping over shots, with the graph, a shot's features, messages and
//     per-variable sums in shared memory and the dense layers on the tensor
//     cores (mma.sync m16n8k16 bf16 -> fp32).  A warp owns 16 checks at a
//     time; the 64-wide node states g0/g1/g2 never leave its registers (they
//     are recomputed from the saved 16-wide inputs x, a1, a2 instead of stored).
// Both round at the same points, so they agree to fp32 summation order.

#include "relaybp.h"
#include "relaybp_host.h"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

namespace {

using rbph::DevBuf;
using rbph::DeviceGuard;
using rbph::fail;
using bf16 = __nv_bfloat16;

constexpr int NH = 64;   // node state width
constexpr int ND = 16;   // message width
constexpr int NF = 4;    // variable features
constexpr int NTY = 4;   // edge types
constexpr int NX = 6;    // check inputs

// flat parameter layout (offsets into theta)
constexpr int P_E = 0;
constexpr int P_W1 = P_E + NH * NX;
constexpr int P_G1 = P_W1 + ND * NH;
constexpr int P_U1 = P_G1 + NTY * ND;
constexpr int P_B1 = P_U1 + NH * ND;
constexpr int P_W2 = P_B1 + NH;
constexpr int P_G2 = P_W2 + ND * NH;
constexpr int P_U2 = P_G2 + NTY * ND;
constexpr int P_B2 = P_U2 + NH * ND;
constexpr int P_O = P_B2 + NH;
constexpr int P_OZ = P_O + NH;
constexpr int P_OB = P_OZ + NF;
constexpr int N_PARAMS = P_OB + 1;
static_assert(N_PARAMS == 4805, "parameter layout");
static_assert(P_W1 % 2 == 0 && P_U1 % 2 == 0 && P_W2 % 2 == 0 && P_U2 % 2 == 0 && P_O % 2 == 0 && P_B1 % 2 == 0 &&
                  P_B2 % 2 == 0,
              "paired bf16 weight loads need even offsets");
static_assert(P_G1 % 8 == 0 && P_G2 % 8 == 0, "gate rows are read as 16-byte vectors");

struct NetGraph {
  int C, V, E;
  const int* chk_ptr;     // [C+1]
  const int* chk_var;     // [E] variable of each edge, check-major
  const int* var_ptr;     // [V+1]
  const int* var_chk;     // [E] check of each edge, variable-major
  const float* llr_feat;  // [V] tanh(llr/16)
};

__device__ __forceinline__ float rbf(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float ldw(const bf16* p, int i) { return __bfloat162float(p[i]); }

// Sum over the block (valid in thread 0); every thread of the block must call it.
__device__ __forceinline__ float block_sum(float v, float* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  float s = 0.f;
  if (threadIdx.x == 0)
    for (int i = 0; i < nw; ++i) s += red[i];
  return s;
}

// ------------------------------------------------------------------ features (training path)

__global__ void feat_var_kernel(NetGraph g, long long B, const uint8_t* syn, const float* post, float* z,
                                uint8_t* ty) {
  const long long n = B * g.V;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long b = i / g.V;
    const int v = (int)(i - b * g.V);
    const float pc = fminf(fmaxf(post[i], -1e4f), 1e4f);
    const bool hard = pc <= 0.f;
    const int k0 = g.var_ptr[v], k1 = g.var_ptr[v + 1];
    int cnt = 0;
    for (int k = k0; k < k1; ++k) cnt += syn[b * g.C + g.var_chk[k]] & 1;
    const float deg = (float)max(k1 - k0, 1);
    float4 f;
    f.x = tanhf(pc * 0.0625f);
    f.y = hard ? 1.f : 0.f;
    f.z = (float)cnt / deg;
    f.w = g.llr_feat[v];
    reinterpret_cast<float4*>(z)[i] = f;
    ty[i] = (uint8_t)((hard ? 2 : 0) + (fabsf(pc) < 8.f ? 1 : 0));
  }
}

__global__ void feat_chk_kernel(NetGraph g, long long B, const uint8_t* syn, const float* z, const float* lmean,
                                float* xr) {
  const long long n = B * g.C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long b = i / g.C;
    const int c = (int)(i - b * g.C);
    const int e0 = g.chk_ptr[c], e1 = g.chk_ptr[c + 1];
    float s0 = 0.f, s1 = 0.f, s2 = 0.f;
    for (int e = e0; e < e1; ++e) {
      const float4 f = reinterpret_cast<const float4*>(z)[b * g.V + g.chk_var[e]];
      s0 += f.x;
      s1 += f.y;
      s2 += f.z;
    }
    const float deg = (float)max(e1 - e0, 1);
    float* o = xr + i * NX;
    o[0] = (float)(syn[i] & 1);
    o[1] = rbf(s0 / deg);
    o[2] = rbf(s1 / deg);
    o[3] = rbf(s2 / deg);
    o[4] = rbf(lmean[c]);
    o[5] = 1.f;
  }
}

// ------------------------------------------------------------------ dense layers (training path)

// Q[r, j] = sum_k round(act(X[r, k])) W[j, k] (+ bias[j]) (+ relu(R[r, j])), optionally rounded.
template <int K, int N, bool XRELU, bool BIAS, bool RES, bool ROUND_OUT>
__global__ void dense_fwd_kernel(long long n, const float* X, const bf16* W, const bf16* bias, const float* R,
                                 float* Q) {
  __shared__ float w[N * K];
  __shared__ float bs[N];
  for (int i = threadIdx.x; i < N * K; i += blockDim.x) w[i] = ldw(W, i);
  if (BIAS)
    for (int i = threadIdx.x; i < N; i += blockDim.x) bs[i] = ldw(bias, i);
  __syncthreads();
  const long long tot = n * N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
    const long long r = i / N;
    const int j = (int)(i - r * N);
    const float* x = X + r * K;
    float acc = 0.f;
#pragma unroll 8
    for (int k = 0; k < K; ++k) {
      float xv = x[k];
      if (XRELU) xv = fmaxf(xv, 0.f);
      acc = fmaf(rbf(xv), w[j * K + k], acc);
    }
    if (BIAS) acc += bs[j];
    if (RES) acc += fmaxf(R[i], 0.f);
    Q[i] = ROUND_OUT ? rbf(acc) : acc;
  }
}

// dX[r, k] (=|+=) sum_j dY[r, j] W[j, k]
template <int K, int N, bool ACCUM>
__global__ void dense_bwd_x_kernel(long long n, const float* dY, const bf16* W, float* dX) {
  __shared__ float w[N * K];
  for (int i = threadIdx.x; i < N * K; i += blockDim.x) w[i] = ldw(W, i);
  __syncthreads();
  const long long tot = n * K;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
    const long long r = i / K;
    const int k = (int)(i - r * K);
    const float* dy = dY + r * N;
    float acc = 0.f;
#pragma unroll 8
    for (int j = 0; j < N; ++j) acc = fmaf(dy[j], w[j * K + k], acc);
    dX[i] = ACCUM ? dX[i] + acc : acc;
  }
}

// dW[j, k] += sum_r dY[r, j] round(act(X[r, k])),  db[j] += sum_r dY[r, j].  256 threads per block.
template <int K, int N, bool XRELU, bool BIAS>
__global__ void __launch_bounds__(256) dense_bwd_w_kernel(long long n, const float* dY, const float* X, float* dW,
                                                           float* db) {
  constexpr int TR = 32;
  constexpr int NP = N * K + (BIAS ? N : 0);
  constexpr int PPT = (NP + 255) / 256;
  __shared__ float sy[TR][N];
  __shared__ float sx[TR][K];
  float acc[PPT];
#pragma unroll
  for (int q = 0; q < PPT; ++q) acc[q] = 0.f;
  const long long per = (n + gridDim.x - 1) / gridDim.x;
  const long long r0 = blockIdx.x * per;
  const long long r1 = min(n, r0 + per);
  for (long long rb = r0; rb < r1; rb += TR) {
    const int rows = (int)min((long long)TR, r1 - rb);
    __syncthreads();
    for (int i = threadIdx.x; i < TR * N; i += blockDim.x) {
      const int rr = i / N, j = i - rr * N;
      sy[rr][j] = rr < rows ? dY[(rb + rr) * N + j] : 0.f;
    }
    for (int i = threadIdx.x; i < TR * K; i += blockDim.x) {
      const int rr = i / K, k = i - rr * K;
      float xv = rr < rows ? X[(rb + rr) * K + k] : 0.f;
      if (XRELU) xv = fmaxf(xv, 0.f);
      sx[rr][k] = rbf(xv);
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < PPT; ++q) {
      const int p = threadIdx.x + q * 256;
      if (p < N * K) {
        const int j = p / K, k = p - j * K;
        float a = acc[q];
        for (int rr = 0; rr < TR; ++rr) a = fmaf(sy[rr][j], sx[rr][k], a);
        acc[q] = a;
      } else if (BIAS && p < NP) {
        const int j = p - N * K;
        float a = acc[q];
        for (int rr = 0; rr < TR; ++rr) a += sy[rr][j];
        acc[q] = a;
      }
    }
  }
#pragma unroll
  for (int q = 0; q < PPT; ++q) {
    const int p = threadIdx.x + q * 256;
    if (p < N * K) atomicAdd(dW + p, acc[q]);
    else if (BIAS && p < NP) atomicAdd(db + (p - N * K), acc[q]);
  }
}

__global__ void relu_mask_kernel(long long n, const float* Q, float* dY) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (!(Q[i] > 0.f)) dY[i] = 0.f;
}

// ------------------------------------------------------------------ message passing (training path)

// n[b, v, d] = round(sum_{c in M(v)} m[b, c, d])
__global__ void varsum_kernel(NetGraph g, long long B, const float* m, float* nv) {
  const long long tot = B * g.V * ND;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
    const int d = (int)(i % ND);
    const long long bv = i / ND;
    const long long b = bv / g.V;
    const int v = (int)(bv - b * g.V);
    float s = 0.f;
    for (int k = g.var_ptr[v]; k < g.var_ptr[v + 1]; ++k) s += m[(b * g.C + g.var_chk[k]) * ND + d];
    nv[i] = rbf(s);
  }
}

// a[b, c, d] = sum_{v in N(c)} G[t_v, d] (n[b, v, d] - m[b, c, d])
__global__ void agg_kernel(NetGraph g, long long B, const bf16* G, const uint8_t* ty, const float* m,
                           const float* nv, float* a) {
  __shared__ float gs[NTY * ND];
  for (int i = threadIdx.x; i < NTY * ND; i += blockDim.x) gs[i] = ldw(G, i);
  __syncthreads();
  const long long tot = B * g.C * ND;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
    const int d = (int)(i % ND);
    const long long bc = i / ND;
    const long long b = bc / g.C;
    const int c = (int)(bc - b * g.C);
    const float mc = m[i];
    float s = 0.f;
    for (int e = g.chk_ptr[c]; e < g.chk_ptr[c + 1]; ++e) {
      const long long bv = b * g.V + g.chk_var[e];
      s = fmaf(gs[ty[bv] * ND + d], nv[bv * ND + d] - mc, s);
    }
    a[i] = s;
  }
}

// Backward of agg: dG += da (n_v - m_c) per edge type; dm = -(sum_v G[t_v]) da.
__global__ void agg_bwd_kernel(NetGraph g, long long B, const bf16* G, const uint8_t* ty, const float* m,
                               const float* nv, const float* da, float* dm, float* dG) {
  __shared__ float gs[NTY * ND];
  __shared__ float acc[NTY * ND];
  for (int i = threadIdx.x; i < NTY * ND; i += blockDim.x) {
    gs[i] = ldw(G, i);
    acc[i] = 0.f;
  }
  __syncthreads();
  const long long tot = B * g.C * ND;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
    const int d = (int)(i % ND);
    const long long bc = i / ND;
    const long long b = bc / g.C;
    const int c = (int)(bc - b * g.C);
    const float mc = m[i], dac = da[i];
    float gsum = 0.f;
    float part[NTY] = {0.f, 0.f, 0.f, 0.f};
    for (int e = g.chk_ptr[c]; e < g.chk_ptr[c + 1]; ++e) {
      const long long bv = b * g.V + g.chk_var[e];
      const int tt = ty[bv];
      gsum += gs[tt * ND + d];
      part[tt] = fmaf(dac, nv[bv * ND + d] - mc, part[tt]);
    }
    dm[i] = -gsum * dac;
#pragma unroll
    for (int tt = 0; tt < NTY; ++tt)
      if (part[tt] != 0.f) atomicAdd(&acc[tt * ND + d], part[tt]);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < NTY * ND; i += blockDim.x)
    if (acc[i] != 0.f) atomicAdd(dG + i, acc[i]);
}

// dn[b, v, d] = G[t_v, d] sum_{c in M(v)} da[b, c, d]
__global__ void dn_kernel(NetGraph g, long long B, const bf16* G, const uint8_t* ty, const float* da, float* dn) {
  __shared__ float gs[NTY * ND];
  for (int i = threadIdx.x; i < NTY * ND; i += blockDim.x) gs[i] = ldw(G, i);
  __syncthreads();
  const long long tot = B * g.V * ND;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
    const int d = (int)(i % ND);
    const long long bv = i / ND;
    const long long b = bv / g.V;
    const int v = (int)(bv - b * g.V);
    float s = 0.f;
    for (int k = g.var_ptr[v]; k < g.var_ptr[v + 1]; ++k) s += da[(b * g.C + g.var_chk[k]) * ND + d];
    dn[i] = gs[ty[bv] * ND + d] * s;
  }
}

// dm[b, c, d] += sum_{v in N(c)} dn[b, v, d]
__global__ void varsum_bwd_kernel(NetGraph g, long long B, const float* dn, float* dm) {
  const long long tot = B * g.C * ND;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
    const int d = (int)(i % ND);
    const long long bc = i / ND;
    const long long b = bc / g.C;
    const int c = (int)(bc - b * g.C);
    float s = 0.f;
    for (int e = g.chk_ptr[c]; e < g.chk_ptr[c + 1]; ++e) s += dn[(b * g.V + g.chk_var[e]) * ND + d];
    dm[i] += s;
  }
}

// ------------------------------------------------------------------ readout and loss (training path)

// r = sum_{c in M(v)} o_c / deg_v + Oz.z_v + ob.  With targets: the weighted
// logistic loss (summed into *loss, divided by B V), dr, and the Oz / ob gradients.
__global__ void __launch_bounds__(256) readout_kernel(NetGraph g, long long B, const bf16* theta, const float* o,
                                                      const float* z, const uint8_t* y, float w_neg, float* r,
                                                      float* dr, float* loss, float* grad) {
  __shared__ float red[32];
  const float oz0 = ldw(theta, P_OZ), oz1 = ldw(theta, P_OZ + 1), oz2 = ldw(theta, P_OZ + 2),
              oz3 = ldw(theta, P_OZ + 3), ob = ldw(theta, P_OB);
  const long long tot = B * g.V;
  const float inv_n = 1.f / (float)tot;
  float l_acc = 0.f, g0 = 0.f, g1 = 0.f, g2 = 0.f, g3 = 0.f, gb = 0.f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
    const long long b = i / g.V;
    const int v = (int)(i - b * g.V);
    const int k0 = g.var_ptr[v], k1 = g.var_ptr[v + 1];
    float s = 0.f;
    for (int k = k0; k < k1; ++k) s += o[b * g.C + g.var_chk[k]];
    const float4 f = reinterpret_cast<const float4*>(z)[i];
    const float rv = s / (float)max(k1 - k0, 1) + (oz0 * f.x + oz1 * f.y + oz2 * f.z + oz3 * f.w) + ob;
    r[i] = rv;
    if (y) {
      const float yv = (float)(y[i] & 1);
      const float w = yv > 0.f ? 1.f : w_neg;
      const float sp = fmaxf(rv, 0.f) + log1pf(expf(-fabsf(rv)));
      l_acc += w * (sp - yv * rv);
      const float d = w * (1.f / (1.f + expf(-rv)) - yv) * inv_n;
      dr[i] = d;
      g0 += d * f.x;
      g1 += d * f.y;
      g2 += d * f.z;
      g3 += d * f.w;
      gb += d;
    }
  }
  if (!y) return;  // uniform over the block
  const float vals[6] = {l_acc * inv_n, g0, g1, g2, g3, gb};
  float* dst[6] = {loss, grad + P_OZ, grad + P_OZ + 1, grad + P_OZ + 2, grad + P_OZ + 3, grad + P_OB};
  for (int q = 0; q < 6; ++q) {
    const float t = block_sum(vals[q], red);
    if (threadIdx.x == 0) atomicAdd(dst[q], t);
  }
}

// do[b, c] = sum_{v in N(c)} dr[b, v] / deg_v
__global__ void readout_bwd_kernel(NetGraph g, long long B, const float* dr, float* dout) {
  const long long tot = B * g.C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
    const long long b = i / g.C;
    const int c = (int)(i - b * g.C);
    float s = 0.f;
    for (int e = g.chk_ptr[c]; e < g.chk_ptr[c + 1]; ++e) {
      const int v = g.chk_var[e];
      s += dr[b * g.V + v] / (float)max(g.var_ptr[v + 1] - g.var_ptr[v], 1);
    }
    dout[i] = s;
  }
}

// AdamW with decoupled weight decay and bias-corrected moments; refreshes the bf16 copy.
__global__ void adamw_kernel(int n, float* theta, float* m, float* v, const float* grad, bf16* theta_bf, float lr,
                             float beta1, float beta2, float eps, float wd, float bc1, float bc2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = grad[i];
    float p = theta[i] * (1.f - lr * wd);
    const float mi = beta1 * m[i] + (1.f - beta1) * gi;
    const float vi = beta2 * v[i] + (1.f - beta2) * gi * gi;
    p -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    m[i] = mi;
    v[i] = vi;
    theta[i] = p;
    theta_bf[i] = __float2bfloat16_rn(p);
  }
}

__global__ void to_bf16_kernel(int n, const float* x, bf16* y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = __float2bfloat16_rn(x[i]);
}

// ------------------------------------------------------------------ fused inference (tensor cores)
//
// One 512-thread block per SM takes shots from a grid-stride loop.  Shared
// memory (bf16 rows unless noted):
//   s_w  all weights, staged once per block     s_g  the graph's index arrays (u16), once per block
//   s_x  [C][8]  check inputs x^ (6 used)       s_th [V] f32 tanh feature
//   s_m  [C][16] messages of the current layer  s_tu [V] u8  type | unsat-count << 2
//   s_n  [V][8]  their per-variable sums, for   s_syn [C] u8
//                one half of the channels at a time
//   s_a1, s_a2 [C][16] aggregated layer inputs a^ (kept: the tile passes
//                recompute g0 and g1 from x^ and a1^ instead of storing them)
// Phases per shot, separated by block barriers: variable features; check
// inputs; per layer: tile pass (messages), then per half of the channels the
// variable sums and the check aggregation; tile pass 3 (layer-2 update and
// o); variable readout.  A warp's tile is 16 checks: x^ / a^ rows are loaded
// as mma A fragments, weights as B fragments from s_w, and each layer's fp32
// accumulators become the next layer's A fragments in registers.

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 p = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&p);
}

__device__ __forceinline__ float sw_f(const bf16* w, int i) { return __bfloat162float(w[i]); }

__device__ __forceinline__ void unpack8(const uint4& q, float (&f)[8]) {
  const __nv_bfloat162* p = reinterpret_cast<const __nv_bfloat162*>(&q);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float2 t = __bfloat1622float2(p[i]);
    f[2 * i] = t.x;
    f[2 * i + 1] = t.y;
  }
}

__device__ __forceinline__ uint4 pack8(const float (&f)[8]) {
  uint4 q;
  q.x = pack_bf16(f[0], f[1]);
  q.y = pack_bf16(f[2], f[3]);
  q.z = pack_bf16(f[4], f[5]);
  q.w = pack_bf16(f[6], f[7]);
  return q;
}

// B operands of the tensor-core layers, stored per fragment so that a warp
// reads each fragment as 32 consecutive words (lane l at word l): no bank
// conflicts, unlike reading the [n][k] weight rows directly (a 128-byte row
// stride puts the 8 rows of a fragment in one bank).
constexpr int FR_E = 0;                   // [nt 8] (k 0..7; k >= 6 is zero)
constexpr int FR_W1 = FR_E + 8 * 32;      // [nt 2][kk 4][half 2]
constexpr int FR_W2 = FR_W1 + 16 * 32;
constexpr int FR_U1 = FR_W2 + 16 * 32;    // [nt 8][half 2]
constexpr int FR_U2 = FR_U1 + 16 * 32;
constexpr int FR_O = FR_U2 + 16 * 32;     // [kk 4][half 2], column 0 only
constexpr int FR_WORDS = FR_O + 8 * 32;

__device__ __forceinline__ uint32_t theta_pair(const bf16* th, int i) {
  return (uint32_t)__bfloat16_as_ushort(th[i]) | ((uint32_t)__bfloat16_as_ushort(th[i + 1]) << 16);
}

// Word w of the fragment table (lane = w % 32: row n = nt*8 + lane/4, columns k, k+1 with k = ... + 2 (lane%4)).
__device__ uint32_t fragment_word(const bf16* th, int w) {
  const int lane = w & 31, f = w >> 5, gq = lane >> 2, k2 = 2 * (lane & 3);
  if (w < FR_W1) {
    const int n = f * 8 + gq;
    return k2 < NX ? theta_pair(th, P_E + n * NX + k2) : 0u;
  }
  if (w < FR_U1) {
    const int base = w < FR_W2 ? P_W1 : P_W2;
    const int ff = f - (w < FR_W2 ? FR_W1 : FR_W2) / 32;
    const int nt = ff >> 3, kk = (ff >> 1) & 3, half = ff & 1;
    return theta_pair(th, base + (nt * 8 + gq) * NH + kk * 16 + half * 8 + k2);
  }
  if (w < FR_O) {
    const int base = w < FR_U2 ? P_U1 : P_U2;
    const int ff = f - (w < FR_U2 ? FR_U1 : FR_U2) / 32;
    const int nt = ff >> 1, half = ff & 1;
    return theta_pair(th, base + (nt * 8 + gq) * ND + half * 8 + k2);
  }
  const int ff = f - FR_O / 32;
  const int kk = ff >> 1, half = ff & 1;
  return gq == 0 ? theta_pair(th, P_O + kk * 16 + half * 8 + k2) : 0u;
}

struct ProposeArgs {
  long long B;
  const uint8_t* syn;       // [B, C]
  const float* post;        // row b at post + b * post_stride
  long long post_stride;    // elements between rows (>= V)
  float lo, hi;
  float* gammas;            // [B, V] or null
  float* logits;            // [B, V] or null
  const int32_t* shot_list;   // [B] shots to evaluate, or null: all
  const int32_t* list_count;  // device count of shot_list entries, or null: B
  const bf16* theta;        // [N_PARAMS]
  const float* chk_lmean;   // [C] mean of the check's variables' tanh(llr/16)
  const uint16_t* graph16;  // chk_ptr [C+1], chk_var [E], var_ptr [V+1], var_chk [E]
  int graph16_len;          // entries, a multiple of 8
  int off_w, off_fr, off_g, off_x, off_m, off_n, off_a1, off_a2, off_th, off_tu, off_syn;  // shared-memory byte offsets
};

// Rows r0, r0+8 of a bf16 [rows][16] array as an A fragment (zero past C).
__device__ __forceinline__ void load_a16(const bf16* s, int r0, int tq, int C, uint32_t (&a)[4]) {
  const int r1 = r0 + 8;
  a[0] = r0 < C ? *reinterpret_cast<const uint32_t*>(s + r0 * ND + 2 * tq) : 0u;
  a[1] = r1 < C ? *reinterpret_cast<const uint32_t*>(s + r1 * ND + 2 * tq) : 0u;
  a[2] = r0 < C ? *reinterpret_cast<const uint32_t*>(s + r0 * ND + 8 + 2 * tq) : 0u;
  a[3] = r1 < C ? *reinterpret_cast<const uint32_t*>(s + r1 * ND + 8 + 2 * tq) : 0u;
}

// q0 = x^ E^T for the warp's 16 checks (8 n-tiles of 8 columns); x rows are 8 wide.
__device__ __forceinline__ void tile_embed(const uint32_t* fr, const bf16* s_x, int r0, int lane, int tq, int C,
                                           float (&acc)[8][4]) {
  uint32_t a[4];
  a[0] = (r0 < C && tq < 3) ? *reinterpret_cast<const uint32_t*>(s_x + r0 * 8 + 2 * tq) : 0u;
  a[1] = (r0 + 8 < C && tq < 3) ? *reinterpret_cast<const uint32_t*>(s_x + (r0 + 8) * 8 + 2 * tq) : 0u;
  a[2] = 0u;
  a[3] = 0u;
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
    mma_bf16(acc[nt], a, fr[FR_E + nt * 32 + lane], 0u);
  }
}

// A fragments (4 k-tiles of 16) of round(relu(acc)).
__device__ __forceinline__ void relu_to_a(const float (&acc)[8][4], uint32_t (&ga)[4][4]) {
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    ga[kk][0] = pack_bf16(fmaxf(acc[2 * kk][0], 0.f), fmaxf(acc[2 * kk][1], 0.f));
    ga[kk][1] = pack_bf16(fmaxf(acc[2 * kk][2], 0.f), fmaxf(acc[2 * kk][3], 0.f));
    ga[kk][2] = pack_bf16(fmaxf(acc[2 * kk + 1][0], 0.f), fmaxf(acc[2 * kk + 1][1], 0.f));
    ga[kk][3] = pack_bf16(fmaxf(acc[2 * kk + 1][2], 0.f), fmaxf(acc[2 * kk + 1][3], 0.f));
  }
}

// m = round(g^ W^T) for the tile, stored as bf16 rows of 16.
__device__ __forceinline__ void tile_message(const uint32_t* fr, int fw, const uint32_t (&ga)[4][4], int r0,
                                             int lane, int tq, int C, bf16* s_m) {
  float mc[2][4];
#pragma unroll
  for (int nt = 0; nt < 2; ++nt) {
    mc[nt][0] = mc[nt][1] = mc[nt][2] = mc[nt][3] = 0.f;
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      const uint32_t* f = fr + fw + (nt * 8 + kk * 2) * 32 + lane;
      mma_bf16(mc[nt], ga[kk], f[0], f[32]);
    }
  }
  const int r1 = r0 + 8;
#pragma unroll
  for (int nt = 0; nt < 2; ++nt) {
    if (r0 < C) *reinterpret_cast<uint32_t*>(s_m + r0 * ND + nt * 8 + 2 * tq) = pack_bf16(mc[nt][0], mc[nt][1]);
    if (r1 < C) *reinterpret_cast<uint32_t*>(s_m + r1 * ND + nt * 8 + 2 * tq) = pack_bf16(mc[nt][2], mc[nt][3]);
  }
}

// acc <- relu(acc) + b + a^ U^T  (the residual update of one layer)
__device__ __forceinline__ void tile_update(const bf16* sw, const uint32_t* fr, int fu, int pb, const bf16* s_a,
                                            int r0, int lane, int tq, int C, float (&acc)[8][4]) {
  uint32_t a[4];
  load_a16(s_a, r0, tq, C, a);
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const int col = nt * 8 + 2 * tq;
    const float2 bb = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(sw + pb + col));
    acc[nt][0] = fmaxf(acc[nt][0], 0.f) + bb.x;
    acc[nt][1] = fmaxf(acc[nt][1], 0.f) + bb.y;
    acc[nt][2] = fmaxf(acc[nt][2], 0.f) + bb.x;
    acc[nt][3] = fmaxf(acc[nt][3], 0.f) + bb.y;
    const uint32_t* f = fr + fu + nt * 64 + lane;
    mma_bf16(acc[nt], a, f[0], f[32]);
  }
}

constexpr int PROPOSE_THREADS = 512;

__global__ void __launch_bounds__(PROPOSE_THREADS, 1) net_propose_kernel(NetGraph g, ProposeArgs pa) {
  extern __shared__ __align__(16) unsigned char smem[];
  bf16* sw = reinterpret_cast<bf16*>(smem + pa.off_w);
  uint32_t* fr = reinterpret_cast<uint32_t*>(smem + pa.off_fr);
  bf16* s_x = reinterpret_cast<bf16*>(smem + pa.off_x);
  bf16* s_m = reinterpret_cast<bf16*>(smem + pa.off_m);
  float* s_o = reinterpret_cast<float*>(smem + pa.off_m);  // reuses the message rows after layer 2
  bf16* s_n = reinterpret_cast<bf16*>(smem + pa.off_n);
  bf16* s_a1 = reinterpret_cast<bf16*>(smem + pa.off_a1);
  bf16* s_a2 = reinterpret_cast<bf16*>(smem + pa.off_a2);
  float* s_th = reinterpret_cast<float*>(smem + pa.off_th);
  uint8_t* s_tu = smem + pa.off_tu;
  uint8_t* s_syn = smem + pa.off_syn;
  const int C = g.C, V = g.V, E = g.E;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  const int gq = lane >> 2, tq = lane & 3;
  const int ntiles = (C + 15) >> 4;
  uint16_t* sg = reinterpret_cast<uint16_t*>(smem + pa.off_g);
  const uint16_t* chk_ptr = sg;
  const uint16_t* chk_var = chk_ptr + C + 1;
  const uint16_t* var_ptr = chk_var + E;
  const uint16_t* var_chk = var_ptr + V + 1;

  for (int i = tid; i < N_PARAMS; i += blockDim.x) sw[i] = pa.theta[i];
  for (int i = tid; i < FR_WORDS; i += blockDim.x) fr[i] = fragment_word(pa.theta, i);
  for (int i = tid; i < pa.graph16_len / 8; i += blockDim.x)
    reinterpret_cast<uint4*>(sg)[i] = __ldg(reinterpret_cast<const uint4*>(pa.graph16) + i);
  __syncthreads();

  const long long n_items = pa.shot_list && pa.list_count ? (long long)min(max(*pa.list_count, 0), (int)pa.B) : pa.B;
  for (long long item = blockIdx.x; item < n_items; item += gridDim.x) {
    const long long b = pa.shot_list ? (long long)pa.shot_list[item] : item;
    if (b < 0 || b >= pa.B) continue;  // block-uniform: no barrier is skipped by part of the block
    // variable features
    for (int c = tid; c < C; c += blockDim.x) s_syn[c] = pa.syn[b * C + c] & 1;
    __syncthreads();
    for (int v = tid; v < V; v += blockDim.x) {
      const float pc = fminf(fmaxf(pa.post[b * pa.post_stride + v], -1e4f), 1e4f);
      int cnt = 0;
      for (int k = var_ptr[v]; k < var_ptr[v + 1]; ++k) cnt += s_syn[var_chk[k]];
      s_th[v] = tanhf(pc * 0.0625f);
      s_tu[v] = (uint8_t)((pc <= 0.f ? 2 : 0) + (fabsf(pc) < 8.f ? 1 : 0) + (cnt << 2));
    }
    __syncthreads();
    // check inputs x^ = (s, mean tanh, mean hard, mean unsat, mean tanh(llr/16), 1, 0, 0)
    for (int c = tid; c < C; c += blockDim.x) {
      const int e0 = chk_ptr[c], e1 = chk_ptr[c + 1];
      float s0 = 0.f, s1 = 0.f, s2 = 0.f;
      for (int e = e0; e < e1; ++e) {
        const int v = chk_var[e];
        const int tu = s_tu[v];
        s0 += s_th[v];
        s1 += (float)((tu >> 1) & 1);
        s2 += (float)(tu >> 2) / (float)max(var_ptr[v + 1] - var_ptr[v], 1);
      }
      const float deg = (float)max(e1 - e0, 1);
      uint4 q;
      q.x = pack_bf16((float)s_syn[c], s0 / deg);
      q.y = pack_bf16(s1 / deg, s2 / deg);
      q.z = pack_bf16(__ldg(pa.chk_lmean + c), 1.f);
      q.w = 0u;
      *reinterpret_cast<uint4*>(s_x + c * 8) = q;
    }
    __syncthreads();
#pragma unroll 1
    for (int layer = 1; layer <= 2; ++layer) {
      const int pg = layer == 1 ? P_G1 : P_G2;
      bf16* s_a = layer == 1 ? s_a1 : s_a2;
      // tile pass: this layer's messages
      for (int tile = warp; tile < ntiles; tile += nwarps) {
        float acc[8][4];
        uint32_t ga[4][4];
        const int r0 = tile * 16 + gq;
        tile_embed(fr, s_x, r0, lane, tq, C, acc);
        if (layer == 2) tile_update(sw, fr, FR_U1, P_B1, s_a1, r0, lane, tq, C, acc);
        relu_to_a(acc, ga);
        tile_message(fr, layer == 1 ? FR_W1 : FR_W2, ga, r0, lane, tq, C, s_m);
      }
      __syncthreads();
      // per half h of the 16 channels: n_v = round(sum_{c in M(v)} m_c), then
      // a_c = sum_{v in N(c)} G[t_v] (n_v - m_c)
#pragma unroll 1
      for (int h = 0; h < 2; ++h) {
        for (int v = tid; v < V; v += blockDim.x) {
          float n[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
          for (int k = var_ptr[v]; k < var_ptr[v + 1]; ++k) {
            float f[8];
            unpack8(*reinterpret_cast<const uint4*>(s_m + var_chk[k] * ND + h * 8), f);
#pragma unroll
            for (int j = 0; j < 8; ++j) n[j] += f[j];
          }
          *reinterpret_cast<uint4*>(s_n + v * 8) = pack8(n);
        }
        __syncthreads();
        for (int c = tid; c < C; c += blockDim.x) {
          float mc[8], a[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
          unpack8(*reinterpret_cast<const uint4*>(s_m + c * ND + h * 8), mc);
          for (int e = chk_ptr[c]; e < chk_ptr[c + 1]; ++e) {
            const int v = chk_var[e];
            float n[8], gt[8];
            unpack8(*reinterpret_cast<const uint4*>(s_n + v * 8), n);
            unpack8(*reinterpret_cast<const uint4*>(sw + pg + (s_tu[v] & 3) * ND + h * 8), gt);
#pragma unroll
            for (int j = 0; j < 8; ++j) a[j] = fmaf(gt[j], n[j] - mc[j], a[j]);
          }
          *reinterpret_cast<uint4*>(s_a + c * ND + h * 8) = pack8(a);
        }
        __syncthreads();
      }
    }
    // layer-2 update and the check readout o_c = O . g2^
    for (int tile = warp; tile < ntiles; tile += nwarps) {
      float acc[8][4];
      uint32_t ga[4][4];
      const int r0 = tile * 16 + gq;
      tile_embed(fr, s_x, r0, lane, tq, C, acc);
      tile_update(sw, fr, FR_U1, P_B1, s_a1, r0, lane, tq, C, acc);
      tile_update(sw, fr, FR_U2, P_B2, s_a2, r0, lane, tq, C, acc);
      relu_to_a(acc, ga);
      float oc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) mma_bf16(oc, ga[kk], fr[FR_O + kk * 64 + lane], fr[FR_O + kk * 64 + 32 + lane]);
      if (tq == 0) {
        if (r0 < C) s_o[r0] = oc[0];
        if (r0 + 8 < C) s_o[r0 + 8] = oc[2];
      }
    }
    __syncthreads();
    // variable readout
    const float oz0 = sw_f(sw, P_OZ), oz1 = sw_f(sw, P_OZ + 1), oz2 = sw_f(sw, P_OZ + 2), oz3 = sw_f(sw, P_OZ + 3),
                ob = sw_f(sw, P_OB);
    for (int v = tid; v < V; v += blockDim.x) {
      const int k0 = var_ptr[v], k1 = var_ptr[v + 1];
      float s = 0.f;
      for (int k = k0; k < k1; ++k) s += s_o[var_chk[k]];
      const float deg = (float)max(k1 - k0, 1);
      const int tu = s_tu[v];
      const float r = s / deg +
                      (oz0 * s_th[v] + oz1 * (float)((tu >> 1) & 1) + oz2 * ((float)(tu >> 2) / deg) +
                       oz3 * __ldg(g.llr_feat + v)) +
                      ob;
      if (pa.logits) pa.logits[b * V + v] = r;
      if (pa.gammas) pa.gammas[b * V + v] = pa.lo + (pa.hi - pa.lo) / (1.f + expf(-r));
    }
    __syncthreads();
  }
}

int grid_for(long long n, int threads = 256) {
  const long long b = (n + threads - 1) / threads;
  return (int)std::max(1LL, std::min(b, 148LL * 16));
}

}  // namespace

// ------------------------------------------------------------------ host object

struct rbp_net {
  int device = 0;
  int C = 0, V = 0, E = 0;
  DevBuf<int> chk_ptr, chk_var, var_ptr, var_chk;
  DevBuf<float> llr_feat, chk_lmean;
  DevBuf<uint16_t> graph16;
  DevBuf<float> theta, adam_m, adam_v, grad, loss;
  DevBuf<bf16> theta_bf;
  long long step = 0;
  long long ws_B = 0;
  DevBuf<float> z, xr, q0, q1, q2, m1, m2, n1, n2, a1, a2, o, r, dr, dg, da, dn, dm, dout;
  DevBuf<uint8_t> ty;
  int propose_smem = 0, propose_blocks = 0;
  ProposeArgs layout{};

  NetGraph graph() const { return NetGraph{C, V, E, chk_ptr.p, chk_var.p, var_ptr.p, var_chk.p, llr_feat.p}; }

  int workspace(long long B) {
    if (B <= ws_B) return RBP_OK;
    const size_t nc = (size_t)B * C, nv = (size_t)B * V;
    int rc;
    if ((rc = z.upload(nullptr, nv * NF)) || (rc = ty.upload(nullptr, nv)) || (rc = xr.upload(nullptr, nc * NX)) ||
        (rc = q0.upload(nullptr, nc * NH)) || (rc = q1.upload(nullptr, nc * NH)) ||
        (rc = q2.upload(nullptr, nc * NH)) || (rc = m1.upload(nullptr, nc * ND)) ||
        (rc = m2.upload(nullptr, nc * ND)) || (rc = n1.upload(nullptr, nv * ND)) ||
        (rc = n2.upload(nullptr, nv * ND)) || (rc = a1.upload(nullptr, nc * ND)) ||
        (rc = a2.upload(nullptr, nc * ND)) || (rc = o.upload(nullptr, nc)) || (rc = r.upload(nullptr, nv)) ||
        (rc = dr.upload(nullptr, nv)) || (rc = dg.upload(nullptr, nc * NH)) || (rc = da.upload(nullptr, nc * ND)) ||
        (rc = dn.upload(nullptr, nv * ND)) || (rc = dm.upload(nullptr, nc * ND)) || (rc = dout.upload(nullptr, nc))) {
      ws_B = 0;
      return rc;
    }
    ws_B = B;
    return RBP_OK;
  }

  // Training-path forward; leaves every activation in the workspace.
  void forward(long long B, const uint8_t* syn, const float* post, cudaStream_t st) {
    const NetGraph g = graph();
    const long long nc = B * C, nv = B * V;
    const bf16* t = theta_bf.p;
    feat_var_kernel<<<grid_for(nv), 256, 0, st>>>(g, B, syn, post, z.p, ty.p);
    feat_chk_kernel<<<grid_for(nc), 256, 0, st>>>(g, B, syn, z.p, chk_lmean.p, xr.p);
    dense_fwd_kernel<NX, NH, false, false, false, false><<<grid_for(nc * NH), 256, 0, st>>>(nc, xr.p, t + P_E, nullptr,
                                                                                             nullptr, q0.p);
    // layer 1
    dense_fwd_kernel<NH, ND, true, false, false, true><<<grid_for(nc * ND), 256, 0, st>>>(nc, q0.p, t + P_W1, nullptr,
                                                                                           nullptr, m1.p);
    varsum_kernel<<<grid_for(nv * ND), 256, 0, st>>>(g, B, m1.p, n1.p);
    agg_kernel<<<grid_for(nc * ND), 256, 0, st>>>(g, B, t + P_G1, ty.p, m1.p, n1.p, a1.p);
    dense_fwd_kernel<ND, NH, false, true, true, false><<<grid_for(nc * NH), 256, 0, st>>>(nc, a1.p, t + P_U1, t + P_B1,
                                                                                           q0.p, q1.p);
    // layer 2
    dense_fwd_kernel<NH, ND, true, false, false, true><<<grid_for(nc * ND), 256, 0, st>>>(nc, q1.p, t + P_W2, nullptr,
                                                                                           nullptr, m2.p);
    varsum_kernel<<<grid_for(nv * ND), 256, 0, st>>>(g, B, m2.p, n2.p);
    agg_kernel<<<grid_for(nc * ND), 256, 0, st>>>(g, B, t + P_G2, ty.p, m2.p, n2.p, a2.p);
    dense_fwd_kernel<ND, NH, false, true, true, false><<<grid_for(nc * NH), 256, 0, st>>>(nc, a2.p, t + P_U2, t + P_B2,
                                                                                           q1.p, q2.p);
    // check readout
    dense_fwd_kernel<NH, 1, true, false, false, false><<<grid_for(nc), 256, 0, st>>>(nc, q2.p, t + P_O, nullptr,
                                                                                      nullptr, o.p);
  }

  // Backward of one layer.  On entry dg = dL/d relu(q); on exit dg = dL/d relu(q_prev).
  void layer_backward(long long B, const float* q_prev, const float* q, const float* a, const float* m,
                      const float* n, int pw, int pg, int pu, int pb, cudaStream_t st) {
    const NetGraph g = graph();
    const long long nc = B * C, nv = B * V;
    const bf16* t = theta_bf.p;
    relu_mask_kernel<<<grid_for(nc * NH), 256, 0, st>>>(nc * NH, q, dg.p);  // dg = dL/dq
    dense_bwd_w_kernel<ND, NH, false, true><<<148 * 2, 256, 0, st>>>(nc, dg.p, a, grad.p + pu, grad.p + pb);
    dense_bwd_x_kernel<ND, NH, false><<<grid_for(nc * ND), 256, 0, st>>>(nc, dg.p, t + pu, da.p);
    agg_bwd_kernel<<<grid_for(nc * ND), 256, 0, st>>>(g, B, t + pg, ty.p, m, n, da.p, dm.p, grad.p + pg);
    dn_kernel<<<grid_for(nv * ND), 256, 0, st>>>(g, B, t + pg, ty.p, da.p, dn.p);
    varsum_bwd_kernel<<<grid_for(nc * ND), 256, 0, st>>>(g, B, dn.p, dm.p);
    dense_bwd_w_kernel<NH, ND, true, false><<<148 * 2, 256, 0, st>>>(nc, dm.p, q_prev, grad.p + pw, nullptr);
    dense_bwd_x_kernel<NH, ND, true><<<grid_for(nc * NH), 256, 0, st>>>(nc, dm.p, t + pw, dg.p);  // + residual
  }

  void backward(long long B, cudaStream_t st) {
    const NetGraph g = graph();
    const long long nc = B * C;
    const bf16* t = theta_bf.p;
    readout_bwd_kernel<<<grid_for(nc), 256, 0, st>>>(g, B, dr.p, dout.p);
    dense_bwd_w_kernel<NH, 1, true, false><<<148 * 2, 256, 0, st>>>(nc, dout.p, q2.p, grad.p + P_O, nullptr);
    dense_bwd_x_kernel<NH, 1, false><<<grid_for(nc * NH), 256, 0, st>>>(nc, dout.p, t + P_O, dg.p);
    layer_backward(B, q1.p, q2.p, a2.p, m2.p, n2.p, P_W2, P_G2, P_U2, P_B2, st);
    layer_backward(B, q0.p, q1.p, a1.p, m1.p, n1.p, P_W1, P_G1, P_U1, P_B1, st);
    relu_mask_kernel<<<grid_for(nc * NH), 256, 0, st>>>(nc * NH, q0.p, dg.p);
    dense_bwd_w_kernel<NX, NH, false, false><<<148 * 2, 256, 0, st>>>(nc, dg.p, xr.p, grad.p + P_E, nullptr);
  }
};

extern "C" {

int rbp_net_param_count(int64_t* n) {
  if (!n) return fail(RBP_ERR_ARGUMENT, "rbp_net_param_count: null argument");
  *n = N_PARAMS;
  return RBP_OK;
}

int rbp_net_create(const rbp_graph* g, const float* llr, rbp_net** out) {
  if (!out) return fail(RBP_ERR_ARGUMENT, "rbp_net_create: out is null");
  *out = nullptr;
  if (!g || !llr) return fail(RBP_ERR_ARGUMENT, "rbp_net_create: null graph or llr");
  const int C = g->C, V = g->V, E = g->E;
  std::vector<int> chk_ptr(C + 1, 0), edge_var(E), var_chk(E);
  for (int e = 0; e < E; ++e) chk_ptr[g->edge_chk[e] + 1]++;
  for (int c = 0; c < C; ++c) chk_ptr[c + 1] += chk_ptr[c];
  int max_dv = 0;
  for (int v = 0; v < V; ++v) {
    const int k0 = g->var_ptr[v], k1 = g->var_ptr[v + 1];
    max_dv = std::max(max_dv, k1 - k0);
    for (int k = k0; k < k1; ++k) {
      edge_var[g->var_edges[k]] = v;
      var_chk[k] = g->edge_chk[g->var_edges[k]];
    }
    std::sort(var_chk.begin() + k0, var_chk.begin() + k1);
  }
  if (max_dv > 63) return fail(RBP_ERR_UNSUPPORTED, "rbp_net_create: variable degree above 63");
  std::vector<float> lf(V), lmean(C);
  for (int v = 0; v < V; ++v) lf[v] = std::tanh(llr[v] / 16.0f);
  for (int c = 0; c < C; ++c) {
    float s = 0.f;  // edge order, float sums
    for (int e = chk_ptr[c]; e < chk_ptr[c + 1]; ++e) s += lf[edge_var[e]];
    lmean[c] = s / (float)std::max(chk_ptr[c + 1] - chk_ptr[c], 1);
  }
  DeviceGuard dg(g->device);
  if (!dg.ok) return fail(RBP_ERR_CUDA, "rbp_net_create: cannot select the CUDA device");
  rbp_net* n = new rbp_net();
  n->device = g->device;
  n->C = C;
  n->V = V;
  n->E = E;
  int rc;
  std::vector<float> zeros(N_PARAMS, 0.f);
  if ((rc = n->chk_ptr.upload(chk_ptr.data(), C + 1)) || (rc = n->chk_var.upload(edge_var.data(), E)) ||
      (rc = n->var_ptr.upload(g->var_ptr.data(), V + 1)) || (rc = n->var_chk.upload(var_chk.data(), E)) ||
      (rc = n->llr_feat.upload(lf.data(), V)) || (rc = n->chk_lmean.upload(lmean.data(), C)) ||
      (rc = n->theta.upload(zeros.data(), N_PARAMS)) || (rc = n->adam_m.upload(zeros.data(), N_PARAMS)) ||
      (rc = n->adam_v.upload(zeros.data(), N_PARAMS)) || (rc = n->grad.upload(zeros.data(), N_PARAMS)) ||
      (rc = n->loss.upload(zeros.data(), 1)) || (rc = n->theta_bf.upload(nullptr, N_PARAMS))) {
    delete n;
    return rc;
  }
  to_bf16_kernel<<<4, 256>>>(N_PARAMS, n->theta.p, n->theta_bf.p);
  // inference kernel shared memory (see net_propose_kernel)
  int off = 0;
  auto take = [&](int bytes) {
    const int o = off;
    off = rbph::align16(off + bytes);
    return o;
  };
  const int g16 = (2 * C + 2 * V + 2 + 2 * E + 7) / 8 * 8;
  n->layout.graph16_len = g16;
  n->layout.off_w = take(N_PARAMS * 2);
  n->layout.off_fr = take(FR_WORDS * 4);
  n->layout.off_g = take(g16 * 2);
  n->layout.off_x = take(C * 8 * 2);
  n->layout.off_m = take(std::max(C * ND * 2, C * 4));
  n->layout.off_n = take(V * 8 * 2);
  n->layout.off_a1 = take(C * ND * 2);
  n->layout.off_a2 = take(C * ND * 2);
  n->layout.off_th = take(V * 4);
  n->layout.off_tu = take(V);
  n->layout.off_syn = take(C);
  n->propose_smem = off;
  const bool small_graph = C < 65536 && V < 65536 && E < 65536;
  if (small_graph) {
    std::vector<uint16_t> h16(g16, 0);
    size_t o = 0;
    for (int c = 0; c <= C; ++c) h16[o++] = (uint16_t)chk_ptr[c];
    for (int e = 0; e < E; ++e) h16[o++] = (uint16_t)edge_var[e];
    for (int v = 0; v <= V; ++v) h16[o++] = (uint16_t)g->var_ptr[v];
    for (int k = 0; k < E; ++k) h16[o++] = (uint16_t)var_chk[k];
    if ((rc = n->graph16.upload(h16.data(), g16))) {
      delete n;
      return rc;
    }
  }
  int optin = 0, sms = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, n->device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, n->device);
  if (small_graph && off <= optin) {
    if (cudaFuncSetAttribute(net_propose_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, off) != cudaSuccess) {
      delete n;
      return fail(RBP_ERR_CUDA, "rbp_net_create: cannot reserve shared memory for the inference kernel");
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, net_propose_kernel, PROPOSE_THREADS, off);
    n->propose_blocks = std::max(1, per_sm) * sms;
  }
  if (cudaDeviceSynchronize() != cudaSuccess) {
    delete n;
    return fail(RBP_ERR_CUDA, "rbp_net_create: device error");
  }
  *out = n;
  return RBP_OK;
}

int rbp_net_destroy(rbp_net* n) {
  if (!n) return RBP_OK;
  DeviceGuard dg(n->device);
  delete n;
  return RBP_OK;
}

int rbp_net_set_params(rbp_net* n, const float* theta, void* stream) {
  if (!n || !theta) return fail(RBP_ERR_ARGUMENT, "rbp_net_set_params: null argument");
  DeviceGuard dg(n->device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  RBP_CUDA(cudaMemcpyAsync(n->theta.p, theta, N_PARAMS * sizeof(float), cudaMemcpyDeviceToDevice, st));
  RBP_CUDA(cudaMemsetAsync(n->adam_m.p, 0, N_PARAMS * sizeof(float), st));
  RBP_CUDA(cudaMemsetAsync(n->adam_v.p, 0, N_PARAMS * sizeof(float), st));
  to_bf16_kernel<<<4, 256, 0, st>>>(N_PARAMS, n->theta.p, n->theta_bf.p);
  RBP_CUDA(cudaGetLastError());
  n->step = 0;
  return RBP_OK;
}

int rbp_net_get_params(const rbp_net* n, float* theta, void* stream) {
  if (!n || !theta) return fail(RBP_ERR_ARGUMENT, "rbp_net_get_params: null argument");
  DeviceGuard dg(n->device);
  RBP_CUDA(cudaMemcpyAsync(theta, n->theta.p, N_PARAMS * sizeof(float), cudaMemcpyDeviceToDevice,
                           static_cast<cudaStream_t>(stream)));
  return RBP_OK;
}

int rbp_net_forward(rbp_net* n, int64_t B, const uint8_t* syn, const float* post, float* logits, void* stream) {
  if (!n) return fail(RBP_ERR_ARGUMENT, "rbp_net_forward: null network");
  if (B < 0) return fail(RBP_ERR_ARGUMENT, "rbp_net_forward: negative batch");
  if (B == 0) return RBP_OK;
  if (!syn || !post || !logits) return fail(RBP_ERR_ARGUMENT, "rbp_net_forward: null buffer");
  DeviceGuard dg(n->device);
  int rc;
  if ((rc = n->workspace(B))) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  n->forward(B, syn, post, st);
  readout_kernel<<<grid_for(B * n->V), 256, 0, st>>>(n->graph(), B, n->theta_bf.p, n->o.p, n->z.p, nullptr, 0.f,
                                                      logits, nullptr, nullptr, nullptr);
  RBP_CUDA(cudaGetLastError());
  return RBP_OK;
}

int rbp_net_train_step(rbp_net* n, int64_t B, const uint8_t* syn, const float* post, const uint8_t* target,
                       const rbp_net_hparams* hp, float* loss, float* grads, void* stream) {
  if (!n || !hp) return fail(RBP_ERR_ARGUMENT, "rbp_net_train_step: null argument");
  if (B <= 0) return fail(RBP_ERR_ARGUMENT, "rbp_net_train_step: batch must be positive");
  if (!syn || !post || !target) return fail(RBP_ERR_ARGUMENT, "rbp_net_train_step: null buffer");
  if (!(hp->w_neg > 0.f) || hp->lr < 0.f) return fail(RBP_ERR_ARGUMENT, "rbp_net_train_step: bad hyper-parameters");
  DeviceGuard dg(n->device);
  int rc;
  if ((rc = n->workspace(B))) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  RBP_CUDA(cudaMemsetAsync(n->grad.p, 0, N_PARAMS * sizeof(float), st));
  RBP_CUDA(cudaMemsetAsync(n->loss.p, 0, sizeof(float), st));
  n->forward(B, syn, post, st);
  readout_kernel<<<grid_for(B * n->V), 256, 0, st>>>(n->graph(), B, n->theta_bf.p, n->o.p, n->z.p, target,
                                                      hp->w_neg, n->r.p, n->dr.p, n->loss.p, n->grad.p);
  n->backward(B, st);
  if (loss) RBP_CUDA(cudaMemcpyAsync(loss, n->loss.p, sizeof(float), cudaMemcpyDeviceToDevice, st));
  if (grads) RBP_CUDA(cudaMemcpyAsync(grads, n->grad.p, N_PARAMS * sizeof(float), cudaMemcpyDeviceToDevice, st));
  if (hp->lr > 0.f) {
    n->step += 1;
    const float bc1 = 1.f - std::pow(hp->beta1, (float)n->step), bc2 = 1.f - std::pow(hp->beta2, (float)n->step);
    adamw_kernel<<<(N_PARAMS + 255) / 256, 256, 0, st>>>(N_PARAMS, n->theta.p, n->adam_m.p, n->adam_v.p, n->grad.p,
                                                         n->theta_bf.p, hp->lr, hp->beta1, hp->beta2, hp->eps,
                                                         hp->weight_decay, bc1, bc2);
  }
  RBP_CUDA(cudaGetLastError());
  return RBP_OK;
}

int rbp_net_propose(rbp_net* n, int64_t B, const uint8_t* syn, const float* post, int64_t post_stride, float lo,
                    float hi, const int32_t* shot_list, const int32_t* list_count, float* gammas, float* logits,
                    void* stream) {
  if (!n) return fail(RBP_ERR_ARGUMENT, "rbp_net_propose: null network");
  if (B < 0) return fail(RBP_ERR_ARGUMENT, "rbp_net_propose: negative batch");
  if (B == 0) return RBP_OK;
  if (!syn || !post || (!gammas && !logits)) return fail(RBP_ERR_ARGUMENT, "rbp_net_propose: null buffer");
  if (!(lo <= hi)) return fail(RBP_ERR_ARGUMENT, "rbp_net_propose: lo must not exceed hi");
  if (post_stride != 0 && post_stride < n->V) return fail(RBP_ERR_ARGUMENT, "rbp_net_propose: post_stride below V");
  if (n->propose_blocks == 0)
    return fail(RBP_ERR_UNSUPPORTED, "rbp_net_propose: the graph and a shot's state (" +
                                         std::to_string(n->propose_smem) +
                                         " B) exceed shared memory, or the graph exceeds 65535 edges");
  DeviceGuard dg(n->device);
  ProposeArgs pa = n->layout;
  pa.B = B;
  pa.syn = syn;
  pa.post = post;
  pa.post_stride = post_stride ? post_stride : n->V;
  pa.lo = lo;
  pa.hi = hi;
  pa.gammas = gammas;
  pa.logits = logits;
  pa.shot_list = shot_list;
  pa.list_count = list_count;
  pa.theta = n->theta_bf.p;
  pa.chk_lmean = n->chk_lmean.p;
  pa.graph16 = n->graph16.p;
  const int blocks = (int)std::min<long long>(B, n->propose_blocks);
  net_propose_kernel<<<blocks, PROPOSE_THREADS, n->propose_smem, static_cast<cudaStream_t>(stream)>>>(n->graph(), pa);
  RBP_CUDA(cudaGetLastError());
  return RBP_OK;
}

}  // extern "C"
