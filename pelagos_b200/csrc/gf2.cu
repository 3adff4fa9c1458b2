// GF(2) products on the device: out[b, r] = XOR over the columns j of row r of
// a sparse 0/1 matrix of x[b, j].  With the check matrix H it turns error rows
// into syndromes (s = H e); with the observables matrix it gives the logical
// observables of true and decoded errors (O e, O e_hat).  The reference does
// both on the host with scipy (src/pelagos/adapter.py:545-560, 601-613, 679).
//
// One thread block per shot at a time: the shot's x row (N bytes) is staged in
// shared memory once and every row of the matrix is evaluated against it, so a
// shot's bytes cross DRAM once however many rows the matrix has.

#include "relaybp.h"
#include "relaybp_host.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

namespace {

using rbph::fail;

constexpr int GF2_THREADS = 256;

// Block b handles shot b (grid-stride): stage x[b, :] in shared memory, then
// each thread evaluates rows r = threadIdx.x, threadIdx.x + blockDim.x, ...
__global__ void __launch_bounds__(GF2_THREADS) gf2_rows_kernel(const uint8_t* x, long long B, int N,
                                                             const int* row_ptr, const int* cols, int R,
                                                             uint8_t* out) {
  extern __shared__ __align__(16) uint8_t sx[];
  for (long long b = blockIdx.x; b < B; b += gridDim.x) {
    const uint8_t* xr = x + b * (long long)N;
    __syncthreads();  // the previous shot's rows are done with sx
    for (int j = threadIdx.x; j < N; j += blockDim.x) sx[j] = xr[j];
    __syncthreads();
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
      uint32_t p = 0;
      for (int k = row_ptr[r]; k < row_ptr[r + 1]; ++k) p ^= sx[cols[k]];
      out[b * (long long)R + r] = (uint8_t)(p & 1u);
    }
  }
}

}  // namespace

extern "C" int rbp_gf2_matvec(const uint8_t* x, int64_t B, int32_t N, const int32_t* row_ptr, const int32_t* cols,
                              int32_t R, uint8_t* out, void* stream) {
  if (B < 0 || N < 0 || R < 0) return fail(RBP_ERR_ARGUMENT, "rbp_gf2_matvec: negative size");
  if (B == 0 || R == 0) return RBP_OK;
  if (!x || !row_ptr || !out || (!cols && N > 0)) return fail(RBP_ERR_ARGUMENT, "rbp_gf2_matvec: null buffer");
  if (N > 48 * 1024) return fail(RBP_ERR_UNSUPPORTED, "rbp_gf2_matvec: rows longer than 49,152 columns");
  const int blocks = (int)std::min<long long>(B, 148LL * 8);
  gf2_rows_kernel<<<blocks, GF2_THREADS, (size_t)std::max(N, 1), static_cast<cudaStream_t>(stream)>>>(
      x, B, N, row_ptr, cols, R, out);
  RBP_CUDA(cudaGetLastError());
  return RBP_OK;
}
