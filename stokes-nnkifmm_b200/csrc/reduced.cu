// Leaf-local self interaction (reducedPass.m:21-81) and the leaf block-diagonal
// direct solve (ReducedSolve.m:86-134): per non-empty target leaf the square
// block A_i = S(sources of i -> targets of i) * kron(NN_sub, I3), factored once
// by batched LU (padded to a common size with an identity tail).
#include <cublas_v2.h>

#include <algorithm>
#include <cmath>

#include "fmm.h"

namespace nnk {

namespace {

// One CTA per leaf; thread a owns rows 3a..3a+2 of the leaf block.
__global__ void reduced_build_kernel(int D, const int* __restrict__ leaves, const long long* __restrict__ tstart,
                                     const long long* __restrict__ sstart, const double* __restrict__ tpos,
                                     const double* __restrict__ spos, const long long* __restrict__ goff,
                                     const int* __restrict__ gidx, const double* __restrict__ gw,
                                     const int* __restrict__ local, double e2, double scale,
                                     double* __restrict__ mats) {
  const int li = blockIdx.x;
  const int leaf = leaves[li];
  double* A = mats + (size_t)li * D * D;
  const long long t0 = tstart[leaf];
  const int nt = (int)(tstart[leaf + 1] - t0);
  for (int a = threadIdx.x; a < D / 3; a += blockDim.x) {
    if (a >= nt) {
      for (int k = 0; k < 3; ++k) A[(size_t)(3 * a + k) * D + 3 * a + k] = 1.0;
      continue;
    }
    const double tx = tpos[3 * (t0 + a)], ty = tpos[3 * (t0 + a) + 1], tz = tpos[3 * (t0 + a) + 2];
    for (long long e = sstart[leaf]; e < sstart[leaf + 1]; ++e) {
      const double r[3] = {tx - spos[3 * e], ty - spos[3 * e + 1], tz - spos[3 * e + 2]};
      const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
      const double inv = scale / (sqrt(r2 + e2) * (r2 + e2));
      double S[9];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) S[3 * i + j] = (r[i] * r[j] + (i == j ? r2 + 2 * e2 : 0.0)) * inv;
      for (long long k = goff[e]; k < goff[e + 1]; ++k) {
        const int c = local[gidx[k]];
        const double w = gw[k];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) A[(size_t)(3 * c + j) * D + 3 * a + i] += w * S[3 * i + j];
      }
    }
  }
}

__global__ void reduced_gather_kernel(int D, const int* __restrict__ leaves, const long long* __restrict__ tstart,
                                      const int* __restrict__ trow, const double* __restrict__ in, int layout,
                                      long long ntgt, double* __restrict__ rhs) {
  const int li = blockIdx.x;
  const int leaf = leaves[li];
  const long long t0 = tstart[leaf];
  const int nt = (int)(tstart[leaf + 1] - t0);
  for (int k = threadIdx.x; k < D; k += blockDim.x) {
    const int a = k / 3, c = k % 3;
    double v = 0;
    if (a < nt) {
      const long long r = trow[t0 + a];
      v = layout == NNK_LAYOUT_BLOCKED ? in[c * ntgt + r] : in[3 * r + c];
    }
    rhs[(size_t)li * D + k] = v;
  }
}

__global__ void reduced_scatter_kernel(int D, const int* __restrict__ leaves, const long long* __restrict__ tstart,
                                       const int* __restrict__ trow, const double* __restrict__ sol, int layout,
                                       long long ntgt, double* __restrict__ out) {
  const int li = blockIdx.x;
  const int leaf = leaves[li];
  const long long t0 = tstart[leaf];
  const int nt = (int)(tstart[leaf + 1] - t0);
  for (int k = threadIdx.x; k < 3 * nt; k += blockDim.x) {
    const int a = k / 3, c = k % 3;
    const long long r = trow[t0 + a];
    const double v = sol[(size_t)li * D + k];
    if (layout == NNK_LAYOUT_BLOCKED) out[c * ntgt + r] = v;
    else out[3 * r + c] = v;
  }
}

// y_i = A_i x_i for every leaf block (column-major D x D)
__global__ void block_gemv_kernel(int D, const double* __restrict__ mats, const double* __restrict__ x,
                                  double* __restrict__ y) {
  const int li = blockIdx.x;
  const double* A = mats + (size_t)li * D * D;
  const double* xv = x + (size_t)li * D;
  for (int r = threadIdx.x; r < D; r += blockDim.x) {
    double s = 0;
    for (int c = 0; c < D; ++c) s += A[(size_t)c * D + r] * xv[c];
    y[(size_t)li * D + r] = s;
  }
}

}  // namespace

void Fmm::build_reduced() {
  if (reduced_ready_) return;
  rinv_ready_ = false;
  const HostTree& t = *t_;
  if (t.n_pot != t.n_tgt || t.n_pot != t.n)
    throw Error(NNK_E_ARG, "reducedSolve needs potentials == targets");
  cudaStream_t st = ctx_->stream;
  rleaf_.clear();
  int maxt = 0;
  for (int32_t i = 0; i < N_; ++i)
    if (t.tleaf[i]) {
      rleaf_.push_back(i);
      maxt = std::max<int>(maxt, (int)(t.tgt_start[i + 1] - t.tgt_start[i]));
    }
  const int nl = (int)rleaf_.size();
  rdim_ = 3 * std::max(maxt, 1);
  const int D = rdim_;
  // local column of each potential row inside its leaf
  std::vector<int32_t> local(t.n_pot, 0);
  for (int32_t i : rleaf_)
    for (int64_t k = t.tgt_start[i]; k < t.tgt_start[i + 1]; ++k) local[t.tgt_row[k]] = (int32_t)(k - t.tgt_start[i]);
  DBuf<int32_t> dlocal, dleaf;
  DBuf<int64_t> dts, dss;
  DBuf<double> dtp, dsp;
  dlocal.upload(local, st);
  rleaf_d_.upload(rleaf_, st);
  dts.upload(t.tgt_start, st);
  dss.upload(t.src_start, st);
  dtp.upload(t.tgt_pos, st);
  dsp.upload(t.src_pos, st);
  rmat_.alloc((size_t)nl * D * D);
  rmat_.zero(st);
  if (nl) {
    reduced_build_kernel<<<nl, 128, 0, st>>>(D, rleaf_d_.p, (const long long*)dts.p, (const long long*)dss.p, dtp.p,
                                             dsp.p, (const long long*)goff_.p, gidx_.p, gw_.p, dlocal.p,
                                             p_.eps * p_.eps, 1.0 / (8.0 * M_PI * p_.mu), rmat_.p);
    NNK_CHECK_LAUNCH();
  }
  rlu_.alloc((size_t)nl * D * D);
  if (nl) NNK_CUDA(cudaMemcpyAsync(rlu_.p, rmat_.p, rmat_.bytes(), cudaMemcpyDeviceToDevice, st));
  rpiv_.alloc((size_t)nl * D);
  rinfo_.alloc(std::max(nl, 1));
  std::vector<double*> ptr(nl), rptr(nl);
  rrhs_.alloc((size_t)std::max(nl, 1) * D);
  for (int k = 0; k < nl; ++k) {
    ptr[k] = rlu_.p + (size_t)k * D * D;
    rptr[k] = rrhs_.p + (size_t)k * D;
  }
  rptr_.upload(ptr, st);
  rrhsptr_.upload(rptr, st);
  rts_.upload(t.tgt_start, st);
  if (!blas_) {
    cublasHandle_t h;
    if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) throw Error(NNK_E_CUDA, "cublasCreate failed");
    blas_ = h;
    cudaGetLastError();
  }
  if (nl) {
    cublasHandle_t h = (cublasHandle_t)blas_;
    cublasSetStream(h, st);
    const cublasStatus_t s = cublasDgetrfBatched(h, D, rptr_.p, D, rpiv_.p, rinfo_.p, nl);
    if (s != CUBLAS_STATUS_SUCCESS) throw Error(NNK_E_CUDA, "batched LU of the leaf blocks failed");
    std::vector<int> info(nl);
    NNK_CUDA(cudaMemcpyAsync(info.data(), rinfo_.p, nl * sizeof(int), cudaMemcpyDeviceToHost, st));
    NNK_CUDA(cudaStreamSynchronize(st));
    for (int k = 0; k < nl; ++k)
      if (info[k] != 0) throw Error(NNK_E_ARG, "singular leaf block in reducedSolve");
  }
  NNK_CUDA(cudaStreamSynchronize(st));
  reduced_ready_ = true;
}

void Fmm::reduced_apply(const double* d_in, double* d_out, int layout) {
  build_reduced();
  const HostTree& t = *t_;
  cudaStream_t st = ctx_->stream;
  const int nl = (int)rleaf_.size(), D = rdim_;
  if (!nl) return;
  DBuf<double> y((size_t)nl * D);
  reduced_gather_kernel<<<nl, 128, 0, st>>>(D, rleaf_d_.p, (const long long*)rts_.p, trow_.p, d_in, layout, t.n_tgt,
                                            rrhs_.p);
  NNK_CHECK_LAUNCH();
  block_gemv_kernel<<<nl, 128, 0, st>>>(D, rmat_.p, rrhs_.p, y.p);
  NNK_CHECK_LAUNCH();
  reduced_scatter_kernel<<<nl, 128, 0, st>>>(D, rleaf_d_.p, (const long long*)rts_.p, trow_.p, y.p, layout, t.n_tgt,
                                             d_out);
  NNK_CHECK_LAUNCH();
  NNK_CUDA(cudaStreamSynchronize(st));
}

void Fmm::reduced_solve(const double* d_in, double* d_out, int layout) {
  build_reduced();
  const HostTree& t = *t_;
  cudaStream_t st = ctx_->stream;
  const int nl = (int)rleaf_.size(), D = rdim_;
  if (!nl) return;
  reduced_gather_kernel<<<nl, 128, 0, st>>>(D, rleaf_d_.p, (const long long*)rts_.p, trow_.p, d_in, layout, t.n_tgt,
                                            rrhs_.p);
  NNK_CHECK_LAUNCH();
  cublasHandle_t h = (cublasHandle_t)blas_;
  cublasSetStream(h, st);
  int info = 0;
  const cublasStatus_t s =
      cublasDgetrsBatched(h, CUBLAS_OP_N, D, 1, rptr_.p, D, rpiv_.p, rrhsptr_.p, D, &info, nl);
  if (s != CUBLAS_STATUS_SUCCESS || info != 0) throw Error(NNK_E_CUDA, "batched leaf-block solve failed");
  reduced_scatter_kernel<<<nl, 128, 0, st>>>(D, rleaf_d_.p, (const long long*)rts_.p, trow_.p, rrhs_.p, layout,
                                             t.n_tgt, d_out);
  NNK_CHECK_LAUNCH();
}

void Fmm::reduced_solve_inv(const double* d_in, double* d_out, int layout) {
  build_reduced();
  const HostTree& t = *t_;
  cudaStream_t st = ctx_->stream;
  const int nl = (int)rleaf_.size(), D = rdim_;
  if (!nl) return;
  if (!rinv_ready_) {
    rinv_.alloc((size_t)nl * D * D);
    rsol_.alloc((size_t)nl * D);
    std::vector<double*> ptr(nl);
    for (int k = 0; k < nl; ++k) ptr[k] = rinv_.p + (size_t)k * D * D;
    rinvptr_.upload(ptr, st);
    cublasHandle_t h = (cublasHandle_t)blas_;
    cublasSetStream(h, st);
    if (cublasDgetriBatched(h, D, rptr_.p, D, rpiv_.p, rinvptr_.p, D, rinfo_.p, nl) != CUBLAS_STATUS_SUCCESS)
      throw Error(NNK_E_CUDA, "batched inverse of the leaf blocks failed");
    std::vector<int> info(nl);
    NNK_CUDA(cudaMemcpyAsync(info.data(), rinfo_.p, nl * sizeof(int), cudaMemcpyDeviceToHost, st));
    NNK_CUDA(cudaStreamSynchronize(st));
    for (int k = 0; k < nl; ++k)
      if (info[k] != 0) throw Error(NNK_E_ARG, "singular leaf block in reducedSolve");
    rinv_ready_ = true;
  }
  reduced_gather_kernel<<<nl, 128, 0, st>>>(D, rleaf_d_.p, (const long long*)rts_.p, trow_.p, d_in, layout, t.n_tgt,
                                            rrhs_.p);
  NNK_CHECK_LAUNCH();
  block_gemv_kernel<<<nl, 128, 0, st>>>(D, rinv_.p, rrhs_.p, rsol_.p);
  NNK_CHECK_LAUNCH();
  reduced_scatter_kernel<<<nl, 128, 0, st>>>(D, rleaf_d_.p, (const long long*)rts_.p, trow_.p, rsol_.p, layout,
                                             t.n_tgt, d_out);
  NNK_CHECK_LAUNCH();
}

}  // namespace nnk
