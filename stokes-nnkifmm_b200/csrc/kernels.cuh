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
// One CTA per task.  The task's source segments are flattened: each tile of
// BS sources may span several segments (a thread finds its segment by binary
// search over the segment prefix sums in shared memory).  Sources are staged
// as (x,y,z,f_x) + (f_y,f_z).  A chunk of up to 2*BS targets is processed per
// pass: above BS targets every thread carries two targets (the second shares
// the source loads); below, several threads share a target and split its
// sources, then reduce through shared memory.
//   u(t) = 1/(8 pi mu) sum_s [ (r^2 + 2 eps^2) f_s + (r.f_s) r ] / (r^2+eps^2)^{3/2},
//   r = t - s (Tools/kernel.m:23-47).
template <typename Real> struct Vec4T;
template <> struct Vec4T<float> { using t4 = float4; using t2 = float2; };
template <> struct Vec4T<double> { using t4 = double4; using t2 = double2; };

template <typename Real>
__device__ __forceinline__ void pair_acc(Real tx, Real ty, Real tz, const typename Vec4T<Real>::t4& s4,
                                         const typename Vec4T<Real>::t2& s2, Real e2, Real& ax, Real& ay,
                                         Real& az) {
  const Real dx = tx - s4.x, dy = ty - s4.y, dz = tz - s4.z;
  const Real r2 = dx * dx + dy * dy + dz * dz;
  const Real d = r2 + e2;
  const Real inv = rsq(d);
  const Real inv3 = inv * inv * inv;
  const Real a = e2 * inv3 + inv;  // (r^2 + 2 eps^2) / d^{3/2} = d^{-1/2} + eps^2 d^{-3/2}
  const Real b = (dx * s4.w + dy * s2.x + dz * s2.y) * inv3;
  ax += a * s4.w + b * dx;
  ay += a * s2.x + b * dy;
  az += a * s2.y + b * dz;
}

template <typename Real, int BS>
__global__ void __launch_bounds__(BS) p2p_kernel(const TaskD* __restrict__ tasks,
                                                 const SegD* __restrict__ segs,
                                                 const Real* __restrict__ spos,
                                                 const Real* __restrict__ sstr,
                                                 const Real* __restrict__ tpos, Real* __restrict__ out_main,
                                                 Real* __restrict__ partial, Real e2, Real scale,
                                                 int accumulate_main) {
  using T4 = typename Vec4T<Real>::t4;
  using T2 = typename Vec4T<Real>::t2;
  __shared__ T4 s4[BS];
  __shared__ T2 s2[BS];
  __shared__ long long seg_start[BS];
  __shared__ int seg_end[BS];  // inclusive prefix sums of the counts
  __shared__ Real red[3 * BS];
  const TaskD tk = tasks[blockIdx.x];
  const int tid = threadIdx.x;
  Real* __restrict__ out = tk.partial ? partial : out_main;
  const int accumulate = tk.partial ? 0 : accumulate_main;
  for (int t0 = 0; t0 < tk.ntgt; t0 += 2 * BS) {
    // every thread carries two targets, t and t + npair, so that each source
    // read from shared memory serves two pair evaluations; when there are
    // fewer target pairs than threads, threads split the sources
    const int nt = min(2 * BS, tk.ntgt - t0);
    const int npair = (nt + 1) >> 1;
    const int splits = max(1, BS / npair);
    const int mt = tid % npair, ms = tid / npair;
    const bool act0 = ms < splits;
    const bool act1 = act0 && mt + npair < nt;
    Real tx = 0, ty = 0, tz = 0, ux = 0, uy = 0, uz = 0;
    if (act0) ldpos(tpos, tk.tgt + t0 + mt, tx, ty, tz);
    if (act1) ldpos(tpos, tk.tgt + t0 + npair + mt, ux, uy, uz);
    Real ax = 0, ay = 0, az = 0, bx = 0, by = 0, bz = 0;
    for (int sb = 0; sb < tk.nseg; sb += BS) {
      const int nsb = min(BS, tk.nseg - sb);
      __syncthreads();
      int cnt = 0;
      if (tid < nsb) {
        const SegD sg = segs[tk.seg0 + sb + tid];
        seg_start[tid] = sg.start;
        cnt = sg.count;
      }
      seg_end[tid] = cnt;
      __syncthreads();
      for (int o = 1; o < BS; o <<= 1) {  // inclusive scan
        const int v = tid >= o ? seg_end[tid - o] : 0;
        __syncthreads();
        seg_end[tid] += v;
        __syncthreads();
      }
      const int total = seg_end[nsb - 1];
      // software pipeline: the next tile's source is fetched into registers
      // while the current tile is computed from shared memory
      auto fetch = [&](int f, T4& a, T2& b) {
        int lo = 0, hi = nsb - 1;  // first k with seg_end[k] > f
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (seg_end[mid] > f) hi = mid;
          else lo = mid + 1;
        }
        const long long j = seg_start[lo] + (f - (lo ? seg_end[lo - 1] : 0));
        Real x, y, z;
        ldpos(spos, j, x, y, z);
        a.x = x;
        a.y = y;
        a.z = z;
        a.w = sstr[3 * j];
        b.x = sstr[3 * j + 1];
        b.y = sstr[3 * j + 2];
      };
      T4 pa;
      T2 pb;
      if (tid < total) fetch(tid, pa, pb);
      for (int f0 = 0; f0 < total; f0 += BS) {
        if (f0 + tid < total) {
          s4[tid] = pa;
          s2[tid] = pb;
        }
        __syncthreads();
        if (f0 + BS + tid < total) fetch(f0 + BS + tid, pa, pb);
        const int nj = min(BS, total - f0);
        if (act0) {
#pragma unroll 4
          for (int j = ms; j < nj; j += splits) {
            const T4 a = s4[j];
            const T2 b = s2[j];
            pair_acc<Real>(tx, ty, tz, a, b, e2, ax, ay, az);
            pair_acc<Real>(ux, uy, uz, a, b, e2, bx, by, bz);  // dummy target (0,0,0) when !act1
          }
        }
        __syncthreads();
      }
    }
    __shared__ Real red2[3 * BS];
    red[tid] = ax;
    red[BS + tid] = ay;
    red[2 * BS + tid] = az;
    red2[tid] = bx;
    red2[BS + tid] = by;
    red2[2 * BS + tid] = bz;
    __syncthreads();
    for (int q = tid; q < nt; q += BS) {
      const bool second = q >= npair;
      const int m = second ? q - npair : q;
      const Real* rr = second ? red2 : red;
      Real vx = 0, vy = 0, vz = 0;
      for (int k = 0; k < splits; ++k) {
        vx += rr[m + k * npair];
        vy += rr[BS + m + k * npair];
        vz += rr[2 * BS + m + k * npair];
      }
      const long long o = 3 * (tk.out + t0 + q);
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
                       const Real* tpos, Real* out, Real* partial, Real e2, Real scale, cudaStream_t st,
                       int accumulate = 0) {
  if (ntasks == 0) return;
  p2p_kernel<Real, 128><<<ntasks, 128, 0, st>>>(tasks, segs, spos, sstr, tpos, out, partial, e2, scale, accumulate);
  NNK_CHECK_LAUNCH();
}

// out(task) (+)= sum_i partial(piece i), pieces summed in index order so the
// result does not depend on scheduling.
template <typename Real>
__global__ void reduce_partials_kernel(const RedD* __restrict__ reds, const Real* __restrict__ partial,
                                       Real* __restrict__ out, int accumulate) {
  const RedD r = reds[blockIdx.x];
  const int n = 3 * r.ntgt;
  for (int v = threadIdx.x; v < n; v += blockDim.x) {
    Real s = 0;
    for (int i = 0; i < r.k; ++i) s += partial[3 * (r.pbase + (long long)i * r.ntgt) + v];
    if (accumulate) out[3 * r.out + v] += s;
    else out[3 * r.out + v] = s;
  }
}

template <typename Real>
inline void launch_reduce(const RedD* reds, int nreds, const Real* partial, Real* out, int accumulate,
                          cudaStream_t st) {
  if (nreds == 0) return;
  reduce_partials_kernel<Real><<<nreds, 128, 0, st>>>(reds, partial, out, accumulate);
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
