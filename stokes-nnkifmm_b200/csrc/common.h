// Shared host-side helpers: status propagation, device buffers, context.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/nnkifmm.h"

namespace nnk {

// Internal failures travel as this exception up to the C-ABI boundary,
// where they become a status code plus the message of nnk_last_error().
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define NNK_CUDA(call)                                                              \
  do {                                                                              \
    cudaError_t _e = (call);                                                        \
    if (_e != cudaSuccess)                                                          \
      throw ::nnk::Error(_e == cudaErrorMemoryAllocation ? NNK_E_OOM : NNK_E_CUDA,  \
                         std::string(#call) + ": " + cudaGetErrorString(_e));      \
  } while (0)

#define NNK_CHECK_LAUNCH() NNK_CUDA(cudaGetLastError())

// Owning device buffer (cudaMallocAsync on the context stream is avoided so
// buffers may outlive stream changes).
template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  explicit DBuf(size_t count) { alloc(count); }
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DBuf& operator=(DBuf&& o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DBuf() { release(); }
  void alloc(size_t count) {
    release();
    n = count;
    if (count) NNK_CUDA(cudaMalloc((void**)&p, count * sizeof(T)));
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void upload(const std::vector<T>& h, cudaStream_t s) {
    alloc(h.size());
    if (n) NNK_CUDA(cudaMemcpyAsync(p, h.data(), n * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void zero(cudaStream_t s) {
    if (n) NNK_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
  }
  size_t bytes() const { return n * sizeof(T); }
};

}  // namespace nnk

struct nnk_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string last_error;
  bool has_gpu = false;
  // the caller's handle plus one per tree, FMM and batch made from it: the
  // context (and its stream) goes when the last of them is destroyed
  std::atomic<int> refs{1};
  // cuSOLVER / cuBLAS handles of the set-up steps, created on first use and
  // kept with the context (creating them costs milliseconds, which every
  // right-hand side of a time step that rebuilds its FMM would pay)
  void* dn_solver = nullptr;  // cusolverDnHandle_t
  void* blas = nullptr;       // cublasHandle_t
  // the cuBLAS handle's workspace, owned here so that no cuBLAS call
  // allocates while a matvec is captured into a CUDA graph
  void* blas_ws = nullptr;
  size_t blas_ws_bytes = 0;
};
