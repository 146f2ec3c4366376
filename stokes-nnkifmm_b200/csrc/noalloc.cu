// Direct NEAREST velocity evaluation that allocates nothing.
//
// Who needs it: callers that must not allocate device memory when they call
// -- a MATLAB MEX gateway whose device memory belongs to MATLAB's own pool
// (an allocation of ours there competes with MATLAB's and is invisible to
// it), or a real-time loop that fixed its memory budget up front and must not
// pay cudaMalloc/cudaFree (which can synchronize the whole device) per step.
// They pass their own device buffers for every input and output; the only
// scratch this evaluation needs, the fine-point forces g = kron(NN,I3)*f,
// lives in the file-scope array below, which every GPU that loads the library
// holds until the process exits.
//
// Limit: at most NNK_NOALLOC_MAX_FINE fine points per call (6 MiB of scratch).
// All calls share the one array, so two calls whose work overlaps on the GPU
// (different streams, or different host threads on the same device) race on
// it; serialise them.  The gather writes every one of the q scratch rows a
// call uses before the sum reads them, so nothing needs clearing between
// calls, and rows past q keep whatever an earlier call left.
//
// The first call on a device looks up the array's device address with
// cudaGetSymbolAddress (once per device, with that device current) and keeps
// it for the life of the process's context on that device (a cudaDeviceReset
// ends that context and with it the address; this library does not support
// calls after one).  Make that first call before any stream capture begins.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/nnkifmm.h"
#include "common.h"

namespace {

constexpr int kMaxDevices = 64;

// Fine-point forces, 3 doubles per fine point.
static __device__ __align__(256) double g_noalloc_scratch[3 * NNK_NOALLOC_MAX_FINE];

std::mutex g_mu;
double* g_addr[kMaxDevices] = {nullptr};

// u(t) = 1/(8 pi mu) sum_q [(r^2 + 2 eps^2) g_q + (r.g_q) r] / (r^2+eps^2)^{3/2},
// r = t - x_q, all of the q fine points for every target (FP64).
__global__ void __launch_bounds__(256) direct_kernel(long long m, const double* __restrict__ tgt, long long q,
                                                     const double* __restrict__ src,
                                                     const double* __restrict__ g, double e2, double scale,
                                                     double* __restrict__ out) {
  __shared__ double sx[256], sy[256], sz[256], gx[256], gy[256], gz[256];
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = t < m;
  double tx = 0, ty = 0, tz = 0;
  if (active) {
    tx = tgt[3 * t];
    ty = tgt[3 * t + 1];
    tz = tgt[3 * t + 2];
  }
  double ax = 0, ay = 0, az = 0;
  for (long long j0 = 0; j0 < q; j0 += 256) {
    const int nj = (int)min(256LL, q - j0);
    __syncthreads();
    if (threadIdx.x < nj) {
      const long long j = j0 + threadIdx.x;
      sx[threadIdx.x] = src[3 * j];
      sy[threadIdx.x] = src[3 * j + 1];
      sz[threadIdx.x] = src[3 * j + 2];
      gx[threadIdx.x] = g[3 * j];
      gy[threadIdx.x] = g[3 * j + 1];
      gz[threadIdx.x] = g[3 * j + 2];
    }
    __syncthreads();
    if (active) {
      for (int j = 0; j < nj; ++j) {
        const double dx = tx - sx[j], dy = ty - sy[j], dz = tz - sz[j];
        const double r2 = dx * dx + dy * dy + dz * dz;
        const double d = r2 + e2;
        const double inv = rsqrt(d);
        const double inv3 = inv * inv * inv;
        const double a = (d + e2) * inv3;
        const double b = (dx * gx[j] + dy * gy[j] + dz * gz[j]) * inv3;
        ax += a * gx[j] + b * dx;
        ay += a * gy[j] + b * dy;
        az += a * gz[j] + b * dz;
      }
    }
  }
  if (active) {
    out[3 * t] = scale * ax;
    out[3 * t + 1] = scale * ay;
    out[3 * t + 2] = scale * az;
  }
}

// The gather of kron(NN,I3)*f into the scratch rows, for column indices the
// caller supplied on the device and the host cannot see: an index outside
// [0, n) is not read, and its fine point's force becomes NaN, so every
// velocity it reaches comes out non-finite instead of from memory out of
// bounds.
__global__ void checked_gather_kernel(long long q, const long long* __restrict__ rowptr,
                                      const int* __restrict__ col, const double* __restrict__ val,
                                      const double* __restrict__ f, long long n, double* __restrict__ g) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= q) return;
  double x = 0, y = 0, z = 0;
  for (long long k = rowptr[e]; k < rowptr[e + 1]; ++k) {
    const int c = col[k];
    if (c < 0 || c >= n) {
      x = y = z = __longlong_as_double(0x7ff8000000000000LL);  // quiet NaN
      break;
    }
    const double w = val[k];
    x += w * f[3 * (long long)c];
    y += w * f[3 * (long long)c + 1];
    z += w * f[3 * (long long)c + 2];
  }
  g[3 * e] = x;
  g[3 * e + 1] = y;
  g[3 * e + 2] = z;
}

}  // namespace

extern "C" int nnk_direct_nearest_noalloc(int32_t device, void* stream, const double* forces, int64_t n,
                                          const int64_t* nn_rowptr, const int32_t* nn_col, const double* nn_val,
                                          const double* fine, int64_t q, const double* targets, int64_t m,
                                          double eps, double mu, double* vel) {
  if (device < 0 || device >= kMaxDevices || n < 0 || q < 0 || m < 0) return NNK_E_ARG;
  if (q > NNK_NOALLOC_MAX_FINE) return NNK_E_ARG;  // beyond the static scratch
  if (!(eps > 0) || !(mu > 0)) return NNK_E_ARG;
  if ((n && !forces) || (q && (!nn_rowptr || !nn_col || !nn_val || !fine)) || (m && (!targets || !vel)))
    return NNK_E_ARG;
  // an error already pending on this thread belongs to the caller: report
  // it without launching and leave it in place for the caller to read
  if (cudaPeekAtLastError() != cudaSuccess) return NNK_E_CUDA;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (st && st != cudaStreamLegacy && st != cudaStreamPerThread) {
    int sdev = -1;
    if (cudaStreamGetDevice(st, &sdev) != cudaSuccess) return NNK_E_ARG;
    if (sdev != device) return NNK_E_ARG;  // the stream belongs to another device
  }
  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess) return NNK_E_CUDA;
  if (prev != device && cudaSetDevice(device) != cudaSuccess) return NNK_E_CUDA;
  int rc = NNK_OK;
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[device]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) rc = NNK_E_CUDA;
      else g_addr[device] = static_cast<double*>(p);
    }
    scratch = g_addr[device];
  }
  if (rc == NNK_OK && m > 0) {
    if (q > 0)
      checked_gather_kernel<<<(unsigned)((q + 255) / 256), 256, 0, st>>>(
          (long long)q, (const long long*)nn_rowptr, nn_col, nn_val, forces, (long long)n, scratch);
    direct_kernel<<<(unsigned)((m + 255) / 256), 256, 0, st>>>((long long)m, targets, (long long)q, fine, scratch,
                                                              eps * eps, 1.0 / (8.0 * M_PI * mu), vel);
    if (cudaGetLastError() != cudaSuccess) rc = NNK_E_CUDA;
  }
  if (prev != device) cudaSetDevice(prev);
  return rc;
}
