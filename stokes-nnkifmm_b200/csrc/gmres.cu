// Device GMRES, see gmres.h.
#include <cmath>
#include <vector>

#include "gmres.h"

namespace nnk {

namespace {

constexpr int kRedBlocks = 148 * 2;  // two CTAs per SM for the reductions

// h[j] += sum_i V[j][i] * w[i] for j < k.  grid.y = basis vector, grid.x
// strides over the vector; partial sums are added with FP64 atomics.
__global__ void multidot_kernel(const double* __restrict__ V, int64_t n, const double* __restrict__ w,
                                double* __restrict__ h) {
  const int j = blockIdx.y;
  const double* v = V + (size_t)j * n;
  double s = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s += v[i] * w[i];
  __shared__ double red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(&h[j], red[0]);
}

// w[i] -= sum_j V[j][i] h[j]
__global__ void multiaxpy_kernel(const double* __restrict__ V, int64_t n, int k, const double* __restrict__ h,
                                 double* __restrict__ w) {
  extern __shared__ double hs[];
  for (int j = threadIdx.x; j < k; j += blockDim.x) hs[j] = h[j];
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double s = w[i];
    for (int j = 0; j < k; ++j) s -= V[(size_t)j * n + i] * hs[j];
    w[i] = s;
  }
}

__global__ void axpby_kernel(double a, const double* __restrict__ x, double b, const double* __restrict__ y,
                             double* __restrict__ out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = a * x[i] + (y ? b * y[i] : 0.0);
}

// x += sum_j V[j] y[j]
__global__ void combine_kernel(const double* __restrict__ V, int64_t n, int k, const double* __restrict__ y,
                               double* __restrict__ x) {
  extern __shared__ double ys[];
  for (int j = threadIdx.x; j < k; j += blockDim.x) ys[j] = y[j];
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double s = x[i];
    for (int j = 0; j < k; ++j) s += V[(size_t)j * n + i] * ys[j];
    x[i] = s;
  }
}

// v = w / sqrt(nrm2[0]) (zero when nrm2 <= 0): the new Arnoldi vector,
// normalized on the device so that a step needs one host synchronisation
__global__ void normalize_kernel(const double* __restrict__ w, const double* __restrict__ nrm2,
                                 double* __restrict__ v, int64_t n) {
  const double q = nrm2[0];
  const double a = q > 0.0 ? 1.0 / sqrt(q) : 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[i] = a * w[i];
}

unsigned grid_for(int64_t n) {
  int64_t g = (n + 255) / 256;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(g, kRedBlocks));
}

}  // namespace

double dev_dot(nnk_ctx* ctx, const double* a, const double* b, int64_t n, DBuf<double>& scratch) {
  if (scratch.n < 1) scratch.alloc(1);
  NNK_CUDA(cudaMemsetAsync(scratch.p, 0, sizeof(double), ctx->stream));
  multidot_kernel<<<dim3(grid_for(n), 1), 256, 0, ctx->stream>>>(a, n, b, scratch.p);
  NNK_CHECK_LAUNCH();
  double h = 0;
  NNK_CUDA(cudaMemcpyAsync(&h, scratch.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  NNK_CUDA(cudaStreamSynchronize(ctx->stream));
  return h;
}

void dev_axpby(nnk_ctx* ctx, double a, const double* x, double b, const double* y, double* out, int64_t n) {
  axpby_kernel<<<grid_for(n), 256, 0, ctx->stream>>>(a, x, b, y, out, n);
  NNK_CHECK_LAUNCH();
}

Gmres::Gmres(nnk_ctx* ctx, int64_t n) : ctx_(ctx), n_(n) {}

void Gmres::solve(const Op& op, const Op* post, const double* b, double* x, const nnk_solve_params& sp,
                  nnk_solve_info& info) {
  cudaStream_t st = ctx_->stream;
  const int64_t n = n_;
  const double tol = sp.tol > 0 ? sp.tol : 1e-6;
  const int maxit = sp.maxit > 0 ? sp.maxit : (int)std::min<int64_t>(n, 10);
  int m = sp.restart > 0 ? sp.restart : maxit;  // restart = [] -> unrestarted
  m = (int)std::min<int64_t>(m, std::max<int64_t>(n, 1));
  // The Krylov basis grows on demand (doubling up to m + 1 vectors): a solve
  // that converges in a few dozen steps does not allocate maxit + 1 vectors
  // (1.2 GB for 150k unknowns and maxit 1000) every time.
  int vcap = std::min(m + 1, 32);
  V_.alloc((size_t)vcap * n);
  auto reserve = [&](int need) {
    if (need <= vcap) return;
    int nc = vcap;
    while (nc < need) nc = std::min(m + 1, 2 * nc);
    DBuf<double> V2((size_t)nc * n);
    NNK_CUDA(cudaMemcpyAsync(V2.p, V_.p, (size_t)vcap * n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    NNK_CUDA(cudaStreamSynchronize(st));
    V_ = std::move(V2);
    vcap = nc;
  };
  w_.alloc(n);
  r_.alloc(n);
  tmp_.alloc(n);
  // per step: [pass-1 h (m+1) | pass-2 h (m+1) | ||w||^2]
  h_.alloc(2 * (size_t)(m + 1) + 1);
  std::vector<double> hh(2 * (size_t)(m + 1) + 1);
  NNK_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), st));
  const double nb = std::sqrt(dev_dot(ctx_, b, b, n, tmp_));
  info = nnk_solve_info{0, 0, 0.0};
  if (nb == 0.0) {
    if (post) {
      (*post)(x, w_.p);
      NNK_CUDA(cudaMemcpyAsync(x, w_.p, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    return;
  }
  // x0 = 0 -> r0 = b
  NNK_CUDA(cudaMemcpyAsync(r_.p, b, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  double beta = nb;
  int total = 0;
  std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), hcol(m + 2), y(m);
  double relres = 1.0;
  while (true) {
    dev_axpby(ctx_, 1.0 / beta, r_.p, 0.0, nullptr, V_.p, n);
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int k = 0;
    bool stop = false;
    for (int j = 0; j < m && total < maxit; ++j) {
      reserve(j + 2);  // reads V_0..V_j, writes V_{j+1}
      double* vj = V_.p + (size_t)j * n;
      double* vn = V_.p + (size_t)(j + 1) * n;
      op(vj, w_.p);
      // CGS2: two passes of h = V^T w, w -= V h, then ||w||^2 and the new
      // vector on the device; one copy of the coefficients to the host
      double* h2 = h_.p + (j + 1);
      double* nrm = h_.p + 2 * (j + 1);
      NNK_CUDA(cudaMemsetAsync(h_.p, 0, (2 * (size_t)(j + 1) + 1) * sizeof(double), st));
      for (int pass = 0; pass < 2; ++pass) {
        double* hp = pass ? h2 : h_.p;
        multidot_kernel<<<dim3(grid_for(n), j + 1), 256, 0, st>>>(V_.p, n, w_.p, hp);
        NNK_CHECK_LAUNCH();
        multiaxpy_kernel<<<grid_for(n), 256, (j + 1) * sizeof(double), st>>>(V_.p, n, j + 1, hp, w_.p);
        NNK_CHECK_LAUNCH();
      }
      multidot_kernel<<<dim3(grid_for(n), 1), 256, 0, st>>>(w_.p, n, w_.p, nrm);
      NNK_CHECK_LAUNCH();
      normalize_kernel<<<grid_for(n), 256, 0, st>>>(w_.p, nrm, vn, n);
      NNK_CHECK_LAUNCH();
      NNK_CUDA(cudaMemcpyAsync(hh.data(), h_.p, (2 * (size_t)(j + 1) + 1) * sizeof(double), cudaMemcpyDeviceToHost,
                               st));
      NNK_CUDA(cudaStreamSynchronize(st));
      std::fill(hcol.begin(), hcol.end(), 0.0);
      for (int i = 0; i <= j; ++i) hcol[i] = hh[i] + hh[j + 1 + i];
      const double hn = std::sqrt(std::max(0.0, hh[2 * (j + 1)]));
      hcol[j + 1] = hn;
      // apply previous rotations, then a new one that zeroes hcol[j+1]
      for (int i = 0; i < j; ++i) {
        const double t0 = cs[i] * hcol[i] + sn[i] * hcol[i + 1];
        hcol[i + 1] = -sn[i] * hcol[i] + cs[i] * hcol[i + 1];
        hcol[i] = t0;
      }
      const double den = std::hypot(hcol[j], hcol[j + 1]);
      cs[j] = den > 0 ? hcol[j] / den : 1.0;
      sn[j] = den > 0 ? hcol[j + 1] / den : 0.0;
      hcol[j] = den;
      hcol[j + 1] = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      for (int i = 0; i <= j; ++i) H[(size_t)j * (m + 1) + i] = hcol[i];
      ++total;
      k = j + 1;
      if (std::fabs(g[j + 1]) / nb <= tol || hn == 0.0) {
        stop = true;
        break;
      }
    }
    // y = R^-1 g, x += V y
    for (int i = k - 1; i >= 0; --i) {
      double s = g[i];
      for (int l = i + 1; l < k; ++l) s -= H[(size_t)l * (m + 1) + i] * y[l];
      const double d = H[(size_t)i * (m + 1) + i];
      y[i] = d != 0 ? s / d : 0.0;
    }
    if (k > 0) {
      NNK_CUDA(cudaMemcpyAsync(h_.p, y.data(), k * sizeof(double), cudaMemcpyHostToDevice, st));
      combine_kernel<<<grid_for(n), 256, k * sizeof(double), st>>>(V_.p, n, k, h_.p, x);
      NNK_CHECK_LAUNCH();
    }
    // explicit residual r = b - A x
    op(x, w_.p);
    dev_axpby(ctx_, 1.0, b, -1.0, w_.p, r_.p, n);
    beta = std::sqrt(dev_dot(ctx_, r_.p, r_.p, n, tmp_));
    relres = beta / nb;
    if (relres <= tol || total >= maxit || (!stop && k == 0) || beta == 0.0) break;
    (void)stop;
  }
  info.iters = total;
  info.relres = relres;
  info.flag = relres <= tol ? 0 : 1;
  if (post) {
    (*post)(x, w_.p);
    NNK_CUDA(cudaMemcpyAsync(x, w_.p, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  }
  NNK_CUDA(cudaStreamSynchronize(st));
}

}  // namespace nnk
