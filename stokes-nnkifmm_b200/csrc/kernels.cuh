// Device kernels of the FMM passes.
#pragma once
#include <cuda_runtime.h>

#include <type_traits>

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
// 1/sqrt(d) for d > 0 (here d = r^2 + eps^2 >= eps^2): the hardware's FP64
// approximation y (PTX rsqrt.approx.ftz.f64, relative error e ~ 1e-6) refined
// by one third-order step of the binomial series
//   d^(-1/2) = y (1 - t)^(-1/2) = y (1 + t/2 + 3 t^2/8 + 5 t^3/16 + ...),
//   t = 1 - d y^2 ~ -2e,
// truncated after t^2, so the step leaves 5 t^3 / 16 ~ 2.5 e^3 ~ 1e-18: below
// FP64 rounding, in 5 FP64 operations where two Newton-Raphson steps take 7
// (measured on a B200 over d in [1e-12, 1e4] against 1/sqrt in FP64: 1.3e-12
// after one Newton step, 3.1e-16 after two, 2.6e-16 after this step).
__device__ __forceinline__ double rsq(double d) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(d));
  const double t = fma(-d * y, y, 1.0);
  return fma(y * t, fma(0.375, t, 0.5), y);
}
__device__ __forceinline__ float rsq(float d) { return rsqrtf(d); }

// ------------------------------------------------------------ vector I/O
__device__ __forceinline__ void io_index(const IoMap& m, long long r, long long& off, long long& cs,
                                         long long& rs) {
  if (m.off) {
    off = m.off[r];
    cs = m.cstr[r];
    rs = m.rstr[r];
  } else if (m.layout == NNK_LAYOUT_BLOCKED) {
    off = r;
    cs = m.nrows;
    rs = 3 * m.nrows;
  } else {
    off = 3 * r;
    cs = 1;
    rs = 3 * m.nrows;
  }
}

// ----------------------------------------------------------------- gather
// Force density of each leaf source entry for right-hand sides k0..k0+R-1:
// sum_k w_k f(row_k), i.e. the row of kron(NN_sub, I3) * f for NEAREST
// entries (nearestBlockComputation.m:28-29), or the potential itself in plain
// mode.  Strengths are stored entry-major: str[(e * R + k) * 3 + c].
template <typename Real>
__global__ void gather_kernel(long long E, const long long* __restrict__ goff, const int* __restrict__ gidx,
                              const double* __restrict__ gw, const double* __restrict__ f, IoMap m, int k0, int R,
                              Real* __restrict__ str) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  for (int k = 0; k < R; ++k) {
    double x = 0, y = 0, z = 0;
    for (long long g = goff[e]; g < goff[e + 1]; ++g) {
      const double w = gw[g];
      long long off, cs, rs;
      io_index(m, gidx[g], off, cs, rs);
      const double* v = f + off + (k0 + k) * rs;
      x += w * v[0];
      y += w * v[cs];
      z += w * v[2 * cs];
    }
    Real* o = str + 3 * (e * R + k);
    o[0] = (Real)x;
    o[1] = (Real)y;
    o[2] = (Real)z;
  }
}

template <typename Real>
inline void launch_gather(int64_t E, const int64_t* goff, const int32_t* gidx, const double* gw,
                          const double* f, const IoMap& m, int k0, int R, Real* str, cudaStream_t st) {
  if (E == 0) return;
  gather_kernel<Real><<<(unsigned)((E + 255) / 256), 256, 0, st>>>(E, (const long long*)goff, gidx, gw, f, m, k0,
                                                                    R, str);
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
// Inclusive prefix sums of one int per thread over a block of BS threads (BS
// a multiple of 32): within each warp by shuffles, then the warps' totals
// through wsum (BS / 32 ints), with one barrier.  Every thread of the block
// calls it; wsum is read until the caller's next barrier.
template <int BS>
__device__ __forceinline__ int block_inclusive_scan(int v, int* wsum) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  if (lane == 31) wsum[warp] = v;
  __syncthreads();
  int add = 0;
#pragma unroll
  for (int w = 0; w < BS / 32; ++w)
    if (w < warp) add += wsum[w];
  return v + add;
}

template <typename Real> struct Vec4T;
template <> struct Vec4T<float> { using t4 = float4; using t2 = float2; };
template <> struct Vec4T<double> { using t4 = double4; using t2 = double2; };

// KD = true: the kernel's derivative with respect to eps (times 1/eps, the
// caller folds eps into `scale`):
//   dS/deps = eps [(r^2 - 2 eps^2) I - 3 r r^T] / (8 pi mu D^{5/2}),  D = r^2 + eps^2
// (Tools/kernel.m:29-47 differentiated).
template <typename Real, bool KD = false>
__device__ __forceinline__ void pair_acc(Real tx, Real ty, Real tz, const typename Vec4T<Real>::t4& s4,
                                         const typename Vec4T<Real>::t2& s2, Real e2, Real& ax, Real& ay,
                                         Real& az) {
  const Real dx = tx - s4.x, dy = ty - s4.y, dz = tz - s4.z;
  const Real d = fma(dz, dz, fma(dy, dy, fma(dx, dx, e2)));  // r^2 + eps^2
  const Real inv = rsq(d);
  const Real inv3 = inv * inv * inv;
  Real a, b;
  if (KD) {
    const Real inv5 = inv3 * inv * inv;
    a = (d - 3 * e2) * inv5;  // (r^2 - 2 eps^2) / D^{5/2}
    b = -3 * (dx * s4.w + dy * s2.x + dz * s2.y) * inv5;
  } else {
    a = e2 * inv3 + inv;  // (r^2 + 2 eps^2) / d^{3/2} = d^{-1/2} + eps^2 d^{-3/2}
    b = (dx * s4.w + dy * s2.x + dz * s2.y) * inv3;
  }
  ax += a * s4.w + b * dx;
  ay += a * s2.x + b * dy;
  az += a * s2.y + b * dz;
}

template <typename Real, int BS, bool KD = false>
__global__ void __launch_bounds__(BS) p2p_kernel(const TaskD* __restrict__ tasks,
                                                 const SegD* __restrict__ segs,
                                                 const Real* __restrict__ spos,
                                                 const Real* __restrict__ sstr,
                                                 const Real* __restrict__ tpos, Real* __restrict__ out_main,
                                                 Real* __restrict__ partial, Real e2, Real scale,
                                                 int accumulate_main, const int* __restrict__ nact = nullptr) {
  using T4 = typename Vec4T<Real>::t4;
  using T2 = typename Vec4T<Real>::t2;
  __shared__ T4 s4[2][BS];  // source tiles, double-buffered: one barrier a tile
  __shared__ T2 s2[2][BS];
  __shared__ long long seg_start[BS];
  __shared__ int seg_end[BS];  // inclusive prefix sums of the counts
  __shared__ int wsum[BS / 32];
  __shared__ Real red[3 * BS];
  const TaskD tk = tasks[blockIdx.x];
  if (nact && !nact[tk.node]) return;  // a tree of the forest whose systems all converged
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
      seg_end[tid] = block_inclusive_scan<BS>(cnt, wsum);
      __syncthreads();
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
      int buf = 0;
      // a tile is written to one buffer while the previous one is read from
      // the other; a thread writes a buffer again only after the next
      // barrier, which every thread reaches after reading it
      for (int f0 = 0; f0 < total; f0 += BS, buf ^= 1) {
        if (f0 + tid < total) {
          s4[buf][tid] = pa;
          s2[buf][tid] = pb;
        }
        __syncthreads();
        if (f0 + BS + tid < total) fetch(f0 + BS + tid, pa, pb);
        const T4* __restrict__ S4 = s4[buf];
        const T2* __restrict__ S2 = s2[buf];
        const int nj = min(BS, total - f0);
        if (act0) {
          if constexpr (std::is_same<Real, float>::value && !KD) {
            // the two targets in the two lanes of packed FP32 arithmetic
            const float2 X = make_float2(tx, ux), Y = make_float2(ty, uy), Z = make_float2(tz, uz);
            const float2 E = make_float2(e2, e2);
            float2 cx = make_float2(ax, bx), cy = make_float2(ay, by), cz = make_float2(az, bz);
#pragma unroll 4
            for (int j = ms; j < nj; j += splits) {
              const float4 a = S4[j];
              const float2 b = S2[j];
              const float2 dx = __fadd2_rn(X, make_float2(-a.x, -a.x));
              const float2 dy = __fadd2_rn(Y, make_float2(-a.y, -a.y));
              const float2 dz = __fadd2_rn(Z, make_float2(-a.z, -a.z));
              float2 d = __ffma2_rn(dx, dx, E);
              d = __ffma2_rn(dy, dy, d);
              d = __ffma2_rn(dz, dz, d);
              const float2 inv = make_float2(rsqrtf(d.x), rsqrtf(d.y));
              const float2 inv3 = __fmul2_rn(__fmul2_rn(inv, inv), inv);
              const float2 A = __ffma2_rn(E, inv3, inv);
              const float2 fx = make_float2(a.w, a.w), fy = make_float2(b.x, b.x), fz = make_float2(b.y, b.y);
              float2 dot = __fmul2_rn(dx, fx);
              dot = __ffma2_rn(dy, fy, dot);
              dot = __ffma2_rn(dz, fz, dot);
              const float2 B = __fmul2_rn(dot, inv3);
              cx = __ffma2_rn(A, fx, __ffma2_rn(B, dx, cx));
              cy = __ffma2_rn(A, fy, __ffma2_rn(B, dy, cy));
              cz = __ffma2_rn(A, fz, __ffma2_rn(B, dz, cz));
            }
            ax = cx.x;
            bx = cx.y;
            ay = cy.x;
            by = cy.y;
            az = cz.x;
            bz = cz.y;
          } else {
#pragma unroll 4
            for (int j = ms; j < nj; j += splits) {
              const T4 a = S4[j];
              const T2 b = S2[j];
              pair_acc<Real, KD>(tx, ty, tz, a, b, e2, ax, ay, az);
              pair_acc<Real, KD>(ux, uy, uz, a, b, e2, bx, by, bz);  // dummy target (0,0,0) when !act1
            }
          }
        }
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

// The same pair sum for R right-hand sides at once: the geometry (r, the
// inverse square root and the Stokeslet weight) is shared, and each source
// carries R force vectors, str[(j * R + k) * 3 + c]; outputs are stored the
// same way.  One target per thread; below BS targets, threads split the
// sources and reduce through shared memory.
//
// GRAD (R = 1): instead of the velocity, the gradient with respect to the
// target position of w_t . u(t), w_t a weight vector per target (tw, indexed
// like tpos):  d/dt [w . K(t - s) f] =
//   [2 (w.f) r + (r.f) w + (w.r) f] / D^{3/2} - 3 [(w.f)(r^2 + 2 eps^2) + (w.r)(r.f)] r / D^{5/2},
// r = t - s, D = r^2 + eps^2 (the derivative of Tools/kernel.m:23-47).
template <typename Real, int BS, int R, bool GRAD = false>
__global__ void __launch_bounds__(BS) p2p_multi_kernel(const TaskD* __restrict__ tasks,
                                                       const SegD* __restrict__ segs,
                                                       const Real* __restrict__ spos,
                                                       const Real* __restrict__ sstr,
                                                       const Real* __restrict__ tpos, Real* __restrict__ out_main,
                                                       Real* __restrict__ partial, Real e2, Real scale,
                                                       int accumulate_main, const Real* __restrict__ tw = nullptr,
                                                       const int* __restrict__ nact = nullptr) {
  using T4 = typename Vec4T<Real>::t4;
  constexpr int C = 3 * R;
  __shared__ T4 sp[BS];
  __shared__ __align__(16) Real sf[BS][C];  // rows of 3R values; float2 pairs need 8-byte alignment
  constexpr bool kPacked = std::is_same<Real, float>::value && R % 2 == 0 && !GRAD;
  __shared__ long long seg_start[BS];
  __shared__ int seg_end[BS];
  __shared__ int wsum[BS / 32];
  __shared__ Real red[C][BS];
  const TaskD tk = tasks[blockIdx.x];
  if (nact && !nact[tk.node]) return;
  const int tid = threadIdx.x;
  Real* __restrict__ out = tk.partial ? partial : out_main;
  const int accumulate = tk.partial ? 0 : accumulate_main;
  for (int t0 = 0; t0 < tk.ntgt; t0 += BS) {
    const int nt = min(BS, tk.ntgt - t0);
    const int splits = max(1, BS / nt);
    const int mt = tid % nt, ms = tid / nt;
    const bool act = ms < splits;
    Real tx = 0, ty = 0, tz = 0, wx = 0, wy = 0, wz = 0;
    if (act) ldpos(tpos, tk.tgt + t0 + mt, tx, ty, tz);
    if (GRAD && act) {
      const long long q = 3 * (tk.tgt + t0 + mt);
      wx = tw[q];
      wy = tw[q + 1];
      wz = tw[q + 2];
    }
    Real acc[C];
#pragma unroll
    for (int c = 0; c < C; ++c) acc[c] = 0;
    float2 acc2[kPacked ? C / 2 : 1];  // packed form: acc2[i] = (acc[2 i], acc[2 i + 1])
#pragma unroll
    for (int i = 0; i < (kPacked ? C / 2 : 1); ++i) acc2[i] = make_float2(0.f, 0.f);
    for (int sb = 0; sb < tk.nseg; sb += BS) {
      const int nsb = min(BS, tk.nseg - sb);
      __syncthreads();
      int cnt = 0;
      if (tid < nsb) {
        const SegD sg = segs[tk.seg0 + sb + tid];
        seg_start[tid] = sg.start;
        cnt = sg.count;
      }
      seg_end[tid] = block_inclusive_scan<BS>(cnt, wsum);
      __syncthreads();
      const int total = seg_end[nsb - 1];
      auto fetch = [&](int f, T4& a, Real* b) {
        int lo = 0, hi = nsb - 1;
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
        a.w = 0;
#pragma unroll
        for (int c = 0; c < C; ++c) b[c] = sstr[j * C + c];
      };
      T4 pa;
      Real pb[C];
      if (tid < total) fetch(tid, pa, pb);
      for (int f0 = 0; f0 < total; f0 += BS) {
        if (f0 + tid < total) {
          sp[tid] = pa;
          // component-major: sf[j][c * R + k] = f_c of right-hand side k
#pragma unroll
          for (int k = 0; k < R; ++k)
#pragma unroll
            for (int c = 0; c < 3; ++c) sf[tid][c * R + k] = pb[3 * k + c];
        }
        __syncthreads();
        if (f0 + BS + tid < total) fetch(f0 + BS + tid, pa, pb);
        const int nj = min(BS, total - f0);
        if (GRAD && act) {
#pragma unroll 2
          for (int j = ms; j < nj; j += splits) {
            const T4 q = sp[j];
            const Real dx = tx - q.x, dy = ty - q.y, dz = tz - q.z;
            const Real d = dx * dx + dy * dy + dz * dz + e2;
            const Real inv = rsq(d);
            const Real inv2 = inv * inv;
            const Real inv3 = inv2 * inv;
            const Real inv5 = inv3 * inv2;
            const Real fx = sf[j][0], fy = sf[j][R], fz = sf[j][2 * R];
            const Real wf = wx * fx + wy * fy + wz * fz;
            const Real rf = dx * fx + dy * fy + dz * fz;
            const Real wr = wx * dx + wy * dy + wz * dz;
            const Real a = 2 * wf * inv3 - 3 * (wf * (d + e2) + wr * rf) * inv5;
            const Real b = rf * inv3, c = wr * inv3;
            acc[0] += a * dx + b * wx + c * fx;
            acc[1] += a * dy + b * wy + c * fy;
            acc[2] += a * dz + b * wz + c * fz;
          }
        } else if (act) {
          if constexpr (kPacked) {
            // right-hand sides in pairs in the two lanes of packed FP32 arithmetic
#pragma unroll 2
            for (int j = ms; j < nj; j += splits) {
              const T4 q = sp[j];
              const float dx = tx - q.x, dy = ty - q.y, dz = tz - q.z;
              const float d = fmaf(dz, dz, fmaf(dy, dy, fmaf(dx, dx, e2)));
              const float inv = rsqrtf(d);
              const float inv3 = inv * inv * inv;
              const float a = fmaf(e2, inv3, inv);
              const float2 DX = make_float2(dx, dx), DY = make_float2(dy, dy), DZ = make_float2(dz, dz);
              const float2 A = make_float2(a, a), I3 = make_float2(inv3, inv3);
              const float2* fr = reinterpret_cast<const float2*>(&sf[j][0]);
#pragma unroll
              for (int m = 0; m < R / 2; ++m) {
                const float2 fx = fr[m], fy = fr[R / 2 + m], fz = fr[R + m];
                float2 dot = __fmul2_rn(DX, fx);
                dot = __ffma2_rn(DY, fy, dot);
                dot = __ffma2_rn(DZ, fz, dot);
                const float2 B = __fmul2_rn(dot, I3);
                acc2[m] = __ffma2_rn(A, fx, __ffma2_rn(B, DX, acc2[m]));
                acc2[R / 2 + m] = __ffma2_rn(A, fy, __ffma2_rn(B, DY, acc2[R / 2 + m]));
                acc2[R + m] = __ffma2_rn(A, fz, __ffma2_rn(B, DZ, acc2[R + m]));
              }
            }
          } else {
#pragma unroll 2
            for (int j = ms; j < nj; j += splits) {
              const T4 q = sp[j];
              const Real dx = tx - q.x, dy = ty - q.y, dz = tz - q.z;
              const Real d = dx * dx + dy * dy + dz * dz + e2;
              const Real inv = rsq(d);
              const Real inv3 = inv * inv * inv;
              const Real a = e2 * inv3 + inv;
#pragma unroll
              for (int k = 0; k < R; ++k) {
                const Real fx = sf[j][k], fy = sf[j][R + k], fz = sf[j][2 * R + k];
                const Real b = (dx * fx + dy * fy + dz * fz) * inv3;
                acc[k] += a * fx + b * dx;
                acc[R + k] += a * fy + b * dy;
                acc[2 * R + k] += a * fz + b * dz;
              }
            }
          }
        }
        __syncthreads();
      }
    }
    if constexpr (kPacked) {
#pragma unroll
      for (int i = 0; i < C / 2; ++i) {
        red[2 * i][tid] = acc2[i].x;
        red[2 * i + 1][tid] = acc2[i].y;
      }
    } else {
#pragma unroll
      for (int c = 0; c < C; ++c) red[c][tid] = acc[c];
    }
    __syncthreads();
    for (int v = tid; v < nt * C; v += BS) {
      const int q = v / C, cc = v - q * C;  // output component cc = 3 k + c
      const int rr = (cc % 3) * R + cc / 3;  // its accumulator c * R + k
      Real sum = 0;
      for (int k = 0; k < splits; ++k) sum += red[rr][q + k * nt];
      const long long o = (long long)C * (tk.out + t0 + q) + cc;
      if (accumulate) out[o] += scale * sum;
      else out[o] = scale * sum;
    }
    __syncthreads();
  }
}

// Static shared memory of p2p_multi_kernel<Real, BS, R> stays under 48 KB.
template <typename Real, int BS, int R>
constexpr bool p2p_fits() {
  return 4 * sizeof(Real) * BS + 2 * 3 * R * sizeof(Real) * BS + 12 * BS <= 48 * 1024;
}

template <typename Real, int BS, int R>
inline void launch_multi(const TaskD* tasks, int ntasks, const SegD* segs, const Real* spos, const Real* sstr,
                         const Real* tpos, Real* out, Real* partial, Real e2, Real scale, cudaStream_t st,
                         int accumulate, const int* nact) {
  if constexpr (p2p_fits<Real, BS, R>()) {
    p2p_multi_kernel<Real, BS, R><<<ntasks, BS, 0, st>>>(tasks, segs, spos, sstr, tpos, out, partial, e2, scale,
                                                          accumulate, nullptr, nact);
  } else {
    throw Error(NNK_E_ARG, "pair kernel tile too large for shared memory");
  }
}

template <typename Real, int BS>
inline void launch_p2p_bs(const TaskD* tasks, int ntasks, const SegD* segs, const Real* spos, const Real* sstr,
                          const Real* tpos, Real* out, Real* partial, Real e2, Real scale, cudaStream_t st,
                          int accumulate, int R, const int* nact) {
  switch (R) {
    case 1:
      p2p_kernel<Real, BS><<<ntasks, BS, 0, st>>>(tasks, segs, spos, sstr, tpos, out, partial, e2, scale, accumulate,
                                                  nact);
      break;
    case 2:
      launch_multi<Real, BS, 2>(tasks, ntasks, segs, spos, sstr, tpos, out, partial, e2, scale, st, accumulate, nact);
      break;
    case 3:
      launch_multi<Real, BS, 3>(tasks, ntasks, segs, spos, sstr, tpos, out, partial, e2, scale, st, accumulate, nact);
      break;
    case 4:
      launch_multi<Real, BS, 4>(tasks, ntasks, segs, spos, sstr, tpos, out, partial, e2, scale, st, accumulate, nact);
      break;
    case 6:
      launch_multi<Real, BS, 6>(tasks, ntasks, segs, spos, sstr, tpos, out, partial, e2, scale, st, accumulate, nact);
      break;
    default:
      throw Error(NNK_E_ARG, "pair kernel supports 1, 2, 3, 4 or 6 right-hand sides per launch");
  }
}

// Block sizes the pair kernels are built for (static shared memory stays
// under 48 KB: FP64 tiles of 256 sources with 4-6 right-hand sides do not).
template <typename Real>
inline bool p2p_bs_ok(int bs, int R) {
  auto fits = [&](auto bsc) {
    constexpr int B = decltype(bsc)::value;
    switch (R) {
      case 2: return p2p_fits<Real, B, 2>();
      case 3: return p2p_fits<Real, B, 3>();
      case 4: return p2p_fits<Real, B, 4>();
      case 6: return p2p_fits<Real, B, 6>();
      default: return true;
    }
  };
  if (bs == 64) return fits(std::integral_constant<int, 64>());
  if (bs == 128) return fits(std::integral_constant<int, 128>());
  if (bs == 256) return fits(std::integral_constant<int, 256>());
  return false;
}

template <typename Real>
inline void launch_p2p(const TaskD* tasks, int ntasks, const SegD* segs, const Real* spos, const Real* sstr,
                       const Real* tpos, Real* out, Real* partial, Real e2, Real scale, cudaStream_t st,
                       int accumulate = 0, int R = 1, int bs = 128, const int* nact = nullptr) {
  if (ntasks == 0) return;
  if (!p2p_bs_ok<Real>(bs, R)) bs = 128;
  if (bs == 64)
    launch_p2p_bs<Real, 64>(tasks, ntasks, segs, spos, sstr, tpos, out, partial, e2, scale, st, accumulate, R, nact);
  else if (bs == 256)
    launch_p2p_bs<Real, 256>(tasks, ntasks, segs, spos, sstr, tpos, out, partial, e2, scale, st, accumulate, R, nact);
  else
    launch_p2p_bs<Real, 128>(tasks, ntasks, segs, spos, sstr, tpos, out, partial, e2, scale, st, accumulate, R, nact);
  NNK_CHECK_LAUNCH();
}

// Pair sums with the kernel's eps-derivative (one right-hand side, FP64):
// out = sum (dS/deps) str over the tasks' sources, `scale` = eps / (8 pi mu).
inline void launch_p2p_deps(const TaskD* tasks, int ntasks, const SegD* segs, const double* spos,
                            const double* sstr, const double* tpos, double* out, double* partial, double e2,
                            double scale, cudaStream_t st, int accumulate) {
  if (ntasks == 0) return;
  p2p_kernel<double, 128, true><<<ntasks, 128, 0, st>>>(tasks, segs, spos, sstr, tpos, out, partial, e2, scale,
                                                        accumulate, nullptr);
  NNK_CHECK_LAUNCH();
}

// Gradient pair sums (GRAD form of p2p_multi_kernel, one right-hand side).
template <typename Real>
inline void launch_p2p_grad(const TaskD* tasks, int ntasks, const SegD* segs, const Real* spos, const Real* sstr,
                            const Real* tpos, const Real* tw, Real* out, Real* partial, Real e2, Real scale,
                            cudaStream_t st) {
  if (ntasks == 0) return;
  p2p_multi_kernel<Real, 128, 1, true><<<ntasks, 128, 0, st>>>(tasks, segs, spos, sstr, tpos, out, partial, e2,
                                                                scale, 0, tw);
  NNK_CHECK_LAUNCH();
}

// Right-hand-side counts with a pair kernel, largest first.
inline int rhs_chunk(int remaining, int max_rhs) {
  static const int sizes[] = {6, 4, 3, 2, 1};
  for (int r : sizes)
    if (r <= remaining && r <= max_rhs) return r;
  return 1;
}

// out(task) (+)= sum_i partial(piece i), pieces summed in index order so the
// result does not depend on scheduling.  C = 3 R values per target.
template <typename Real>
__global__ void reduce_partials_kernel(const RedD* __restrict__ reds, const Real* __restrict__ partial,
                                       Real* __restrict__ out, int accumulate, int C, const int* __restrict__ nact) {
  const RedD r = reds[blockIdx.x];
  if (nact && !nact[r.node]) return;
  const int n = C * r.ntgt;
  for (int v = threadIdx.x; v < n; v += blockDim.x) {
    Real s = 0;
    for (int i = 0; i < r.k; ++i) s += partial[C * (r.pbase + (long long)i * r.ntgt) + v];
    if (accumulate) out[C * r.out + v] += s;
    else out[C * r.out + v] = s;
  }
}

template <typename Real>
inline void launch_reduce(const RedD* reds, int nreds, const Real* partial, Real* out, int accumulate,
                          cudaStream_t st, int R = 1, const int* nact = nullptr) {
  if (nreds == 0) return;
  reduce_partials_kernel<Real><<<nreds, 128, 0, st>>>(reds, partial, out, accumulate, 3 * R, nact);
  NNK_CHECK_LAUNCH();
}

// -------------------------------------------------------------------- C2E
// Products of one fixed FP64 operator with the vectors of a list of nodes,
//   dst(node, k) (+)= Aop * src(in_node, k),   k < R,
// FP64 arithmetic.  Aop is M x Kd, column-major at ops + op * op_stride, or
// (trans, square) its transpose.  src and dst hold, per surface point p of a
// node, R consecutive 3-vectors: src[(in_node * P + p) * R + k], p < Kd / 3,
// and dst[(base + node * P + p) * R + k], p < M / 3; a vector longer than one
// node's 3P values runs on into the next node ids.  A tile is up to 64 nodes
// sharing one operator (a level of one tree of the forest).  Uses:
//   * the check-to-equivalent step of a level (M = Kd = 3P, in_node = node):
//     Aop = A (upward, A = K_up^-1) or A^T (downward);
//   * the upward step of a parent from its 8 children, folded into one
//     operator (M = 3P, Kd = 8 * 3P, in_node = first child, node = parent);
//   * the downward step of the 8 children from their parent, folded
//     (M = 8 * 3P, Kd = 3P, in_node = parent, node = first child), added to
//     the children's check-to-equivalent result.
// 64 x 64 output tile (operator rows x (node, right-hand side) columns) per
// CTA of 256 threads, each accumulating 4 x 4 in FP64; K in steps of 16 with
// the next step's operands fetched into registers while the current one is
// multiplied from shared memory.  (A 128 x 64 tile with 8 x 8 per thread and
// 16-byte shared loads ran 10-20% slower here: with 8 warps per SM the
// global-load latency of each K step stayed exposed.)
constexpr int kC2ETileNodes = 64;
constexpr int kC2EBM = 64;

struct NodeGemm {
  const double* ops;
  size_t op_stride;
  int M, Kd, trans;
  const C2ETile* tiles;
  const int* nodes;     // output node per tile column
  const int* in_nodes;  // input node per tile column (nullptr: nodes)
  long long base;
  int P, R, accumulate;
  float* m2l_dst;  // optional TF32 copy of the result (rows < NP)
  int NP;
};

template <typename Real>
__global__ void __launch_bounds__(256) c2e_kernel(NodeGemm g, const Real* __restrict__ check, Real* __restrict__ dst,
                                                  int ksplit, int kper, double* __restrict__ part,
                                                  const int* __restrict__ nact) {
  constexpr int BM = kC2EBM, BN = 64, BK = 16;
  __shared__ double As[BK][BM + 1];
  __shared__ double Bs[BK][BN + 1];
  __shared__ int col_node[BN];
  __shared__ int col_in[BN];
  __shared__ int col_k[BN];
  const C2ETile tl = g.tiles[blockIdx.y];
  if (nact && !nact[g.nodes[tl.first]]) return;  // the nodes of a tile belong to one tree
  const int M = g.M, Kd = g.Kd, P = g.P, R = g.R, trans = g.trans;
  const int zch = gridDim.z / ksplit;
  const int split = blockIdx.z / zch, zc = blockIdx.z - split * zch;
  const int kbeg = split * kper, kend = min(Kd, kbeg + kper);
  const int m0 = blockIdx.x * BM, j0 = zc * BN;
  const int ncol = tl.count * R;
  if (j0 >= ncol) return;
  const double* __restrict__ A = g.ops + (size_t)tl.op * g.op_stride;
  const int tid = threadIdx.x;
  if (tid < BN) {
    const int j = j0 + tid;
    col_node[tid] = j < ncol ? g.nodes[tl.first + j / R] : -1;
    col_in[tid] = j < ncol ? (g.in_nodes ? g.in_nodes : g.nodes)[tl.first + j / R] : -1;
    col_k[tid] = j < ncol ? j % R : 0;
  }
  __syncthreads();
  const int tr = tid % 16, tc = tid / 16;
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0;
  // register staging: 4 operator values and 4 source values per thread per K step
  double ra[4], rb[4];
  // operator element e of the step: Aop[r][c] at c M + r (contiguous in r)
  // or, transposed, A[c][r] at r Kd + c (contiguous in c = the K index)
  auto a_index = [&](int e, int& kk, int& mm) {
    if (!trans) { mm = e % BM; kk = e / BM; }
    else { kk = e % BK; mm = e / BK; }
  };
  auto load = [&](int k0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int kk, mm;
      a_index(tid + 256 * q, kk, mm);
      const int r = m0 + mm, c = k0 + kk;
      ra[q] = (r < M && c < kend) ? (trans ? A[(size_t)r * Kd + c] : A[(size_t)c * M + r]) : 0.0;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + 256 * q;  // BK * BN
      const int kk = e % BK, nn = e / BK;
      const int c = k0 + kk, node = col_in[nn];
      double v = 0;
      if (c < kend && node >= 0) {
        const int p = c / 3, comp = c - 3 * p;
        v = (double)check[(((size_t)node * P + p) * R + col_k[nn]) * 3 + comp];
      }
      rb[q] = v;
    }
  };
  auto store = [&]() {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int kk, mm;
      a_index(tid + 256 * q, kk, mm);
      As[kk][mm] = ra[q];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + 256 * q;
      Bs[e % BK][e / BK] = rb[q];
    }
  };
  load(kbeg);
  for (int k0 = kbeg; k0 < kend; k0 += BK) {
    store();
    __syncthreads();
    if (k0 + BK < kend) load(k0 + BK);
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][tr + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tc + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int r = m0 + tr + 16 * i, jj = tc + 16 * j;
      const int node = col_node[jj];
      if (ksplit > 1) {
        // partial sum of this K range: part[split][tile][column][row]
        if (r < M && node >= 0)
          part[(((size_t)split * gridDim.y + blockIdx.y) * (kC2ETileNodes * R) + j0 + jj) * M + r] = acc[i][j];
        continue;
      }
      if (r < M && node >= 0) {
        const int p = r / 3, comp = r - 3 * p;
        Real* o = dst + ((g.base + (long long)P * node + p) * R + col_k[jj]) * 3 + comp;
        *o = g.accumulate ? (Real)((double)*o + acc[i][j]) : (Real)acc[i][j];
        if (g.m2l_dst && r < g.NP) {
          uint32_t t;
          asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t) : "f"((float)acc[i][j]));
          g.m2l_dst[(size_t)node * g.NP + r] = __uint_as_float(t);
        }
      }
    }
}

// Sum of the K-range partials in split order (deterministic), written out
// like the single-pass epilogue.
template <typename Real>
__global__ void c2e_reduce_kernel(NodeGemm g, int ksplit, int ntiles, const double* __restrict__ part,
                                  Real* __restrict__ dst, const int* __restrict__ nact) {
  const int tile = blockIdx.y;
  const C2ETile tl = g.tiles[tile];
  if (nact && !nact[g.nodes[tl.first]]) return;
  const int M = g.M, R = g.R;
  const int cols = kC2ETileNodes * R;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < (long long)cols * M;
       e += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(e / M), r = (int)(e - (long long)j * M);
    if (j >= tl.count * R) continue;
    double s = 0;
    for (int q = 0; q < ksplit; ++q) s += part[(((size_t)q * ntiles + tile) * cols + j) * M + r];
    const int node = g.nodes[tl.first + j / R], k = j % R;
    const int p = r / 3, comp = r - 3 * p;
    Real* o = dst + ((g.base + (long long)g.P * node + p) * R + k) * 3 + comp;
    *o = g.accumulate ? (Real)((double)*o + s) : (Real)s;
    if (g.m2l_dst && r < g.NP) {
      uint32_t t;
      asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t) : "f"((float)s));
      g.m2l_dst[(size_t)node * g.NP + r] = __uint_as_float(t);
    }
  }
}

// K splits for a launch of `blocks` CTAs: enough CTAs for two per SM, each
// K range at least 32 long.
inline int c2e_splits(int Kd, int blocks) {
  int k = 1;
  while (k < 8 && blocks * k < 2 * 148 && Kd / (2 * k) >= 32) k *= 2;
  return k;
}
inline size_t c2e_part_size(int M, int Kd, int ntiles, int R) {
  const int blocks = ((M + kC2EBM - 1) / kC2EBM) * ntiles * R;
  const int k = c2e_splits(Kd, blocks);
  return k > 1 ? (size_t)k * ntiles * kC2ETileNodes * R * M : 0;
}

template <typename Real>
inline void launch_node_gemm(NodeGemm g, int ntiles, const Real* src, Real* dst, cudaStream_t st,
                             double* part = nullptr, size_t part_n = 0, const int* nact = nullptr) {
  if (ntiles == 0) return;
  const int zch = (kC2ETileNodes * g.R + 63) / 64;
  const int blocks = ((g.M + kC2EBM - 1) / kC2EBM) * ntiles * zch;
  int ksplit = c2e_splits(g.Kd, blocks);
  if (!part || part_n < c2e_part_size(g.M, g.Kd, ntiles, g.R)) ksplit = 1;
  const int kper = ((g.Kd + ksplit - 1) / ksplit + 15) / 16 * 16;
  dim3 grid((g.M + kC2EBM - 1) / kC2EBM, ntiles, zch * ksplit);
  c2e_kernel<Real><<<grid, 256, 0, st>>>(g, src, dst, ksplit, kper, part, nact);
  NNK_CHECK_LAUNCH();
  if (ksplit > 1) {
    dim3 g2(std::max(1, std::min(64, (kC2ETileNodes * g.R * g.M + 255) / 256)), ntiles);
    c2e_reduce_kernel<Real><<<g2, 256, 0, st>>>(g, ksplit, ntiles, part, dst, nact);
    NNK_CHECK_LAUNCH();
  }
}

// The library-GEMM form of a node product (NodeGemm): columns j of a run of
// `ncol` = nodes x R columns (node nodes[first + j / R], right-hand side
// j % R) gathered as FP64 into X (rows x ncol, column-major; row m is point
// m / 3 from the node on, so rows = 8 x 3P spans a first child's 8
// consecutive siblings) ...
template <typename Real>
__global__ void c2e_gather_kernel(const Real* __restrict__ check, const int32_t* __restrict__ nodes, int first,
                                  int ncol, int R, int P, int rows, double* __restrict__ X) {
  const long long total = (long long)ncol * rows;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(e / rows), m = (int)(e - (long long)j * rows);
    const int node = nodes[first + j / R], r = j - (j / R) * R;
    X[e] = (double)check[(((size_t)node * P + m / 3) * R + r) * 3 + m % 3];
  }
}
// ... and the products Y (rows x ncol) written like c2e_kernel's epilogue.
template <typename Real>
__global__ void c2e_scatter_kernel(const double* __restrict__ Y, const int32_t* __restrict__ nodes, int first,
                                   int ncol, int R, int P, int rows, long long base, int accumulate,
                                   Real* __restrict__ dst, float* __restrict__ m2l_dst, int NP) {
  const long long total = (long long)ncol * rows;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(e / rows), m = (int)(e - (long long)j * rows);
    const int node = nodes[first + j / R], r = j - (j / R) * R;
    Real* o = dst + ((base + (long long)P * node + m / 3) * R + r) * 3 + m % 3;
    const double y = Y[e];
    *o = accumulate ? (Real)((double)*o + y) : (Real)y;
    if (m2l_dst && m < NP) {
      uint32_t t;
      asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t) : "f"((float)y));
      m2l_dst[(size_t)node * NP + m] = __uint_as_float(t);
    }
  }
}

// The check-to-equivalent step of a level (n = 3P).
template <typename Real>
inline void launch_c2e(const double* ops, int n, int trans, const C2ETile* tiles, int ntiles, const int32_t* nodes,
                       const Real* check, Real* dst, int64_t base, int P, int R, cudaStream_t st,
                       float* m2l_dst = nullptr, int NP = 0, double* part = nullptr, size_t part_n = 0,
                       const int* nact = nullptr) {
  NodeGemm g{ops, (size_t)n * n, n, n, trans, tiles, nodes, nullptr, (long long)base, P, R, 0, m2l_dst, NP};
  launch_node_gemm<Real>(g, ntiles, check, dst, st, part, part_n, nact);
}

// ---------------------------------------------------------------- scatter
// Sorted-by-leaf velocities back to the reference's target order
// (downwardPass.m:297-305), in the caller's layout, right-hand sides
// k0..k0+R-1.  With a node mask (nact, tnode = leaf of each sorted target),
// the rows of masked trees are written as zeros.
template <typename Real>
__global__ void scatter_kernel(long long nt, const int* __restrict__ row, const Real* __restrict__ vel, IoMap m,
                               int k0, int R, double* __restrict__ out, const int* __restrict__ tnode,
                               const int* __restrict__ nact) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  long long off, cs, rs;
  io_index(m, row[t], off, cs, rs);
  const bool on = !nact || nact[tnode[t]];
  for (int k = 0; k < R; ++k) {
    const Real* v = vel + 3 * (t * R + k);
    double* o = out + off + (k0 + k) * rs;
    o[0] = on ? (double)v[0] : 0.0;
    o[cs] = on ? (double)v[1] : 0.0;
    o[2 * cs] = on ? (double)v[2] : 0.0;
  }
}

// Transpose of the gather: out(row) = sum over the (entry, weight) pairs of
// the potential row of w * vel(entry), right-hand sides k0..k0+R-1.
template <typename Real>
__global__ void scatter_sum_kernel(long long nrows, const long long* __restrict__ row_off,
                                   const long long* __restrict__ row_ent, const double* __restrict__ row_w,
                                   const Real* __restrict__ vel, IoMap m, int k0, int R, double* __restrict__ out) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrows) return;
  long long off, cs, rs;
  io_index(m, r, off, cs, rs);
  for (int k = 0; k < R; ++k) {
    double x = 0, y = 0, z = 0;
    for (long long q = row_off[r]; q < row_off[r + 1]; ++q) {
      const Real* v = vel + 3 * (row_ent[q] * R + k);
      const double w = row_w[q];
      x += w * (double)v[0];
      y += w * (double)v[1];
      z += w * (double)v[2];
    }
    double* o = out + off + (k0 + k) * rs;
    o[0] = x;
    o[cs] = y;
    o[2 * cs] = z;
  }
}

// out[3 o + c] = sum of vel over the entries of origin o (one right-hand side)
template <typename Real>
__global__ void origin_sum_kernel(long long norg, const long long* __restrict__ org_off,
                                  const long long* __restrict__ org_ent, const Real* __restrict__ vel,
                                  double* __restrict__ out) {
  const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= norg) return;
  double x = 0, y = 0, z = 0;
  for (long long q = org_off[o]; q < org_off[o + 1]; ++q) {
    const Real* v = vel + 3 * org_ent[q];
    x += (double)v[0];
    y += (double)v[1];
    z += (double)v[2];
  }
  out[3 * o] = x;
  out[3 * o + 1] = y;
  out[3 * o + 2] = z;
}

template <typename Real>
inline void launch_scatter(int64_t nt, const int32_t* row, const Real* vel, const IoMap& m, int k0, int R,
                           double* out, cudaStream_t st, const int32_t* tnode = nullptr, const int* nact = nullptr) {
  if (nt == 0) return;
  scatter_kernel<Real><<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(nt, row, vel, m, k0, R, out, tnode, nact);
  NNK_CHECK_LAUNCH();
}

}  // namespace nnk
