// Host-side pieces shared by the decoder (relaybp.cu) and the proposal
// network (proposal.cu): error reporting, CUDA call checking, device
// selection, owned device buffers and the Tanner graph object.
#pragma once

#include "relaybp.h"

#include <cuda_runtime.h>

#include <string>
#include <vector>

namespace rbph {

// Per-host-thread message behind rbp_last_error().
std::string& err_slot();

inline int fail(int code, const std::string& msg) {
  err_slot() = msg;
  return code;
}

#define RBP_CUDA(expr)                                                                      \
  do {                                                                                       \
    cudaError_t e_ = (expr);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return ::rbph::fail(RBP_ERR_CUDA, std::string(#expr) + " failed: " + cudaGetErrorString(e_)); \
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

inline int align16(int x) { return (x + 15) & ~15; }

template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  int upload(const T* host, size_t count) {
    if (p) {
      cudaFree(p);
      p = nullptr;
    }
    n = count;
    if (count == 0) return RBP_OK;
    RBP_CUDA(cudaMalloc(&p, count * sizeof(T)));
    if (host) RBP_CUDA(cudaMemcpy(p, host, count * sizeof(T), cudaMemcpyHostToDevice));
    return RBP_OK;
  }
};

}  // namespace rbph

struct rbp_graph {
  int device = 0;
  int C = 0, V = 0, E = 0, slots = 0, vslots = 0;
  // host copy of the edge-centric graph (slot positions depend on the message type)
  std::vector<int> edge_chk, edge_slot, var_ptr, var_edges;
  rbph::DevBuf<uint8_t> chk_deg;
  rbph::DevBuf<int> chk_ptr;
};
