// Device bandwidth measurement for roofline reporting: the L2 read rate of
// this GPU, as the Fourier-space M2L accumulation sees it (16-byte loads of
// data that stays in L2).
#include <cuda_runtime.h>

#include <algorithm>

#include "common.h"
#include "probe.h"

namespace nnk {

namespace {

// Every thread streams 16-byte elements of buf with a grid stride, `passes`
// times; each pass starts at another offset so blocks do not read in step.
// The sums only keep the loads live.
__global__ void l2_read_kernel(const double2* __restrict__ buf, size_t n, int passes, double* __restrict__ sink) {
  double sx = 0, sy = 0;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (int p = 0; p < passes; ++p) {
    const size_t off = ((size_t)p * 7919 * 128) % n;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      size_t j = i + off;
      if (j >= n) j -= n;
      const double2 v = buf[j];
      sx += v.x;
      sy += v.y;
    }
  }
  if (sx + sy == 1234.5) sink[0] = sx;  // never true for the zero-filled buffer
}

}  // namespace

double measure_l2_read_gbs(cudaStream_t st) {
  int dev = 0, sms = 0;
  NNK_CUDA(cudaGetDevice(&dev));
  NNK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const size_t max_bytes = (size_t)48 << 20;
  DBuf<double2> buf(max_bytes / sizeof(double2));
  DBuf<double> sink(1);
  NNK_CUDA(cudaMemsetAsync(buf.p, 0, max_bytes, st));
  struct Events {  // released on every exit
    cudaEvent_t a = nullptr, b = nullptr;
    ~Events() {
      if (a) cudaEventDestroy(a);
      if (b) cudaEventDestroy(b);
    }
  } ev;
  NNK_CUDA(cudaEventCreate(&ev.a));
  NNK_CUDA(cudaEventCreate(&ev.b));
  cudaEvent_t a = ev.a, b = ev.b;
  double best = 0;
  for (size_t mib : {24, 48}) {
    const size_t n = (mib << 20) / sizeof(double2);
    const int passes = (int)(2048 / mib);  // 2 GiB read per timed launch
    for (int per_sm : {8, 16}) {
      const int blocks = sms * per_sm;
      l2_read_kernel<<<blocks, 256, 0, st>>>(buf.p, n, 1, sink.p);  // warm: the buffer into L2
      NNK_CHECK_LAUNCH();
      NNK_CUDA(cudaEventRecord(a, st));
      l2_read_kernel<<<blocks, 256, 0, st>>>(buf.p, n, passes, sink.p);
      NNK_CHECK_LAUNCH();
      NNK_CUDA(cudaEventRecord(b, st));
      NNK_CUDA(cudaEventSynchronize(b));
      float ms = 0;
      NNK_CUDA(cudaEventElapsedTime(&ms, a, b));
      if (ms > 0) best = std::max(best, (double)n * sizeof(double2) * passes / (ms * 1e-3) / 1e9);
    }
  }
  return best;
}

}  // namespace nnk
