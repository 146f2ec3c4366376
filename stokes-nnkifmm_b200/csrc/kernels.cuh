// Device kernels of the FMM passes.
#pragma once
#include <cuda_runtime.h>

#include "common.h"
#include "fmm.h"

namespace nnk {

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ void ldpos(const double* __restrict__ p, long long j, double& x, double& y,
                                      double& z) {
  x = p[3 * j];
  y = p[3 * j + 1];
  z = p[3 * j + 2];
}
__device__ __forceinline__ void ldpos(const float* __restrict__ p, long long j, float& x, float& y,
                                      float& z) {
  const float4 v = reinterpret_cast<const float4*>(p)[j];
  x = v.x;
  y = v.y;
  z = v.z;
}
__device__ __forceinline__ double rsq(double d) { return rsqrt(d); }
__device__ __forceinline__ float rsq(float d) { return rsqrtf(d); }

// ----------------------------------------------------------------- gather
// Force density of each leaf source entry: sum_k w_k f(row_k), i.e. the row of
// kron(NN_sub, I3) * f for NEAREST entries (nearestBlockComputation.m:28-29),
// or the potential itself in plain mode.  f is FP64 in the caller's layout.
template <typename Real>
__global__ void gather_kernel(long long E, const long long* __restrict__ goff, const int* __restrict__ gidx,
                              const double* __restrict__ gw, const double* __restrict__ f, int layout,
                              long long npot, Real* __restrict__ str) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  double x = 0, y = 0, z = 0;
  for (long long k = goff[e]; k < goff[e + 1]; ++k) {
    const double w = gw[k];
    const long long r = gidx[k];
    if (layout == NNK_LAYOUT_BLOCKED) {
      x += w * f[r];
      y += w * f[npot + r];
      z += w * f[2 * npot + r];
    } else {
      x += w * f[3 * r];
      y += w * f[3 * r + 1];
      z += w * f[3 * r + 2];
    }
  }
  str[3 * e] = (Real)x;
  str[3 * e + 1] = (Real)y;
  str[3 * e + 2] = (Real)z;
}

template <typename Real>
inline void launch_gather(int64_t E, const int64_t* goff, const int32_t* gidx, const double* gw,
                          const double* f, int layout, int64_t npot, Real* str, cudaStream_t st) {
  if (E == 0) return;
  gather_kernel<Real><<<(unsigned)((E + 255) / 256), 256, 0, st>>>(
      E, (const long long*)goff, gidx, gw, f, layout, npot, str);
  NNK_CHECK_LAUNCH();
}

// ------------------------------------------------------------ pair kernel
// One CTA per task.  Targets of the task are split over the CTA; when a task
// has fewer targets than threads, several threads share a target and split
// its sources, then reduce through shared memory.  Sources stream through
// shared memory one segment tile at a time.
//   u(t) = 1/(8 pi mu) sum_s [ (r^2 + 2 eps^2) f_s + (r.f_s) r ] / (r^2+eps^2)^{3/2},
//   r = t - s (Tools/kernel.m:23-47).
template <typename Real, int BS>
__global__ void __launch_bounds__(BS) p2p_kernel(const TaskD* __restrict__ tasks,
                                                 const SegD* __restrict__ segs,
                                                 const Real* __restrict__ spos,
                                                 const Real* __restrict__ sstr,
                                                 const Real* __restrict__ tpos, Real* __restrict__ out,
                                                 Real e2, Real scale, int accumulate) {
  __shared__ Real sx[BS], sy[BS], sz[BS], gx[BS], gy[BS], gz[BS];
  __shared__ Real red[3 * BS];
  const TaskD tk = tasks[blockIdx.x];
  const int tid = threadIdx.x;
  for (int t0 = 0; t0 < tk.ntgt; t0 += BS) {
    const int nt = min(BS, tk.ntgt - t0);
    const int splits = BS / nt;
    const int mt = tid % nt, ms = tid / nt;
    const bool active = ms < splits;
    Real tx = 0, ty = 0, tz = 0;
    if (active) ldpos(tpos, tk.tgt + t0 + mt, tx, ty, tz);
    Real ax = 0, ay = 0, az = 0;
    for (int s = 0; s < tk.nseg; ++s) {
      const SegD sg = segs[tk.seg0 + s];
      for (int j0 = 0; j0 < sg.count; j0 += BS) {
        const int nj = min(BS, sg.count - j0);
        __syncthreads();
        if (tid < nj) {
          const long long j = sg.start + j0 + tid;
          Real x, y, z;
          ldpos(spos, j, x, y, z);
          sx[tid] = x;
          sy[tid] = y;
          sz[tid] = z;
          gx[tid] = sstr[3 * j];
          gy[tid] = sstr[3 * j + 1];
          gz[tid] = sstr[3 * j + 2];
        }
        __syncthreads();
        if (active) {
#pragma unroll 4
          for (int j = ms; j < nj; j += splits) {
            const Real dx = tx - sx[j], dy = ty - sy[j], dz = tz - sz[j];
            const Real r2 = dx * dx + dy * dy + dz * dz;
            const Real d = r2 + e2;
            const Real inv = rsq(d);
            const Real inv3 = inv * inv * inv;
            const Real fx = gx[j], fy = gy[j], fz = gz[j];
            const Real a = (d + e2) * inv3;
            const Real b = (dx * fx + dy * fy + dz * fz) * inv3;
            ax += a * fx + b * dx;
            ay += a * fy + b * dy;
            az += a * fz + b * dz;
          }
        }
      }
    }
    red[tid] = ax;
    red[BS + tid] = ay;
    red[2 * BS + tid] = az;
    __syncthreads();
    if (tid < nt) {
      Real vx = 0, vy = 0, vz = 0;
      for (int k = 0; k < splits; ++k) {
        vx += red[tid + k * nt];
        vy += red[BS + tid + k * nt];
        vz += red[2 * BS + tid + k * nt];
      }
      const long long o = 3 * (tk.out + t0 + tid);
      if (accumulate) {
        out[o] += scale * vx;
        out[o + 1] += scale * vy;
        out[o + 2] += scale * vz;
      } else {
        out[o] = scale * vx;
        out[o + 1] = scale * vy;
        out[o + 2] = scale * vz;
      }
    }
    __syncthreads();
  }
}

template <typename Real>
inline void launch_p2p(const TaskD* tasks, int ntasks, const SegD* segs, const Real* spos, const Real* sstr,
                       const Real* tpos, Real* out, Real e2, Real scale, cudaStream_t st, int accumulate = 0) {
  if (ntasks == 0) return;
  p2p_kernel<Real, 128><<<ntasks, 128, 0, st>>>(tasks, segs, spos, sstr, tpos, out, e2, scale, accumulate);
  NNK_CHECK_LAUNCH();
}

// -------------------------------------------------------------------- C2E
// Check-to-equivalent step for all nodes of one level:
//   dst(node) = Aop * check(node), Aop = A (upward) or A^T (downward),
// A stored column-major (n x n), FP64 arithmetic.  dst(node) is the
// strength block of the node's surface points in the unified arrays.
template <typename Real>
__global__ void __launch_bounds__(256) c2e_kernel(const double* __restrict__ A, int n, int trans,
                                                  const int* __restrict__ nodes, int nnodes,
                                                  const Real* __restrict__ check, Real* __restrict__ dst,
                                                  long long base, int P, float* __restrict__ m2l_dst, int NP) {
  constexpr int BM = 64, BN = 32, BK = 16;
  __shared__ double As[BK][BM + 1];
  __shared__ double Bs[BK][BN + 1];
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int tid = threadIdx.x;
  const int tr = tid % 16, tc = tid / 16;
  double acc[4][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
  for (int k0 = 0; k0 < n; k0 += BK) {
    // A tile: rows m0..m0+63, k k0..k0+15
    for (int e = tid; e < BK * BM; e += 256) {
      int kk, mm;
      if (!trans) { mm = e % BM; kk = e / BM; }   // A[r][c] at c*n + r: contiguous in r
      else { kk = e % BK; mm = e / BK; }          // A^T[r][c] = A[c][r] at r*n + c: contiguous in c
      const int r = m0 + mm, c = k0 + kk;
      double v = 0;
      if (r < n && c < n) v = trans ? A[(size_t)r * n + c] : A[(size_t)c * n + r];
      As[kk][mm] = v;
    }
    for (int e = tid; e < BK * BN; e += 256) {
      const int kk = e % BK, nn = e / BK;
      const int c = k0 + kk, j = n0 + nn;
      double v = 0;
      if (c < n && j < nnodes) v = (double)check[(size_t)nodes[j] * n + c];
      Bs[kk][nn] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      double a[4], b[2];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][tr + 16 * i];
#pragma unroll
      for (int j = 0; j < 2; ++j) b[j] = Bs[kk][tc + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) acc[i][j] += a[i] * b[j];
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int r = m0 + tr + 16 * i, jj = n0 + tc + 16 * j;
      if (r < n && jj < nnodes) {
        dst[(base + (long long)P * nodes[jj]) * 3 + r] = (Real)acc[i][j];
        if (m2l_dst) {
          uint32_t t;
          asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t) : "f"((float)acc[i][j]));
          m2l_dst[(size_t)nodes[jj] * NP + r] = __uint_as_float(t);
        }
      }
    }
}

template <typename Real>
inline void launch_c2e(const double* A, int n, int trans, const int32_t* nodes, int nnodes, const Real* check,
                       Real* dst, int64_t base, int P, cudaStream_t st, float* m2l_dst = nullptr, int NP = 0) {
  if (nnodes == 0) return;
  dim3 grid((n + 63) / 64, (nnodes + 31) / 32);
  c2e_kernel<Real><<<grid, 256, 0, st>>>(A, n, trans, nodes, nnodes, check, dst, base, P, m2l_dst, NP);
  NNK_CHECK_LAUNCH();
}

// ---------------------------------------------------------------- scatter
// Sorted-by-leaf velocities back to the reference's target order
// (downwardPass.m:297-305), in the caller's layout.
template <typename Real>
__global__ void scatter_kernel(long long nt, const int* __restrict__ row, const Real* __restrict__ vel,
                               int layout, long long ntgt, double* __restrict__ out) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nt) return;
  const long long r = row[k];
  if (layout == NNK_LAYOUT_BLOCKED) {
    out[r] = (double)vel[3 * k];
    out[ntgt + r] = (double)vel[3 * k + 1];
    out[2 * ntgt + r] = (double)vel[3 * k + 2];
  } else {
    out[3 * r] = (double)vel[3 * k];
    out[3 * r + 1] = (double)vel[3 * k + 1];
    out[3 * r + 2] = (double)vel[3 * k + 2];
  }
}

template <typename Real>
inline void launch_scatter(int64_t nt, const int32_t* row, const Real* vel, int layout, int64_t ntgt,
                           double* out, cudaStream_t st) {
  if (nt == 0) return;
  scatter_kernel<Real><<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(nt, row, vel, layout, ntgt, out);
  NNK_CHECK_LAUNCH();
}

}  // namespace nnk
