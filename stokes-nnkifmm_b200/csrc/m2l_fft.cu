// Fourier-space M2L (see m2l_fft.h).
//
// Transforms are separable DFTs of length G over the zero-padded lattice,
// written out as small sums in shared memory: each pass
// maps one axis, and only the res non-zero inputs (forward) or res needed
// outputs (inverse) of that axis are touched.  Frequency index
// k = (kx * G + ky) * H + kz, H = G / 2 + 1 (half spectrum along z).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <map>

#include "m2l_fft.h"

namespace nnk {

namespace {

template <typename Real> struct Cplx;
template <> struct Cplx<float> { using t = float2; };
template <> struct Cplx<double> { using t = double2; };

__device__ __forceinline__ float2 cmake(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 cmake(double a, double b) { return make_double2(a, b); }
__device__ __forceinline__ float rfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double rfma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ void cmac(float2& acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, fmaf(-a.y, b.y, acc.x));
  acc.y = fmaf(a.x, b.y, fmaf(a.y, b.x, acc.y));
}
__device__ __forceinline__ void cmac(double2& acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
  acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
}

// e^{sign * 2 pi i m / G}, m in [0, G)
template <typename Real>
__device__ __forceinline__ void twiddles(typename Cplx<Real>::t* tw, int G, double sign) {
  for (int m = threadIdx.x; m < G; m += blockDim.x) {
    double s, c;
    sincospi(2.0 * m / G, &s, &c);
    tw[m] = cmake((Real)c, (Real)(sign * s));
  }
}

// ------------------------------------------------------------------ setup
// Spectrum of the kernel on the difference grid for one (box width, offset),
// FP64, one component at a time:
//   Kgrid[d] = K((d - (res - 1) o) h) / (8 pi mu G^3) for |d|_inf <= res - 1
// (d the signed index of the grid point, 0 elsewhere), then three DFT passes.
// deriv = 1: the kernel's eps-derivative,
//   eps [(r^2 - 2 eps^2) I - 3 r r^T] / D^{5/2}, D = r^2 + eps^2
// (scale then carries the eps factor).
// Doubles of the spectra kernel's real grid, rounded up to an even count so
// that the complex arrays after it stay 16-byte aligned (G is odd).
__host__ __device__ constexpr int spectra_real_len(int G) { return (G * G * G + 1) & ~1; }

template <typename Real>
__global__ void fft_spectra_kernel(int G, int res, const double* __restrict__ slot_w,
                                   const int* __restrict__ slot_code, double e2, double scale,
                                   typename Cplx<Real>::t* __restrict__ spec, int NK, int deriv = 0) {
  extern __shared__ double sm[];
  const int H = G / 2 + 1;
  double* K = sm;                         // [x][y][z]
  double2* A = (double2*)(K + spectra_real_len(G));  // [x][y][kz]
  double2* B = A + G * G * H;              // [x][ky][kz]
  const int s = blockIdx.x;
  const double h = slot_w[s] / (res - 1);
  const int code = slot_code[s];
  const int o[3] = {code / 49 - 3, (code / 7) % 7 - 3, code % 7 - 3};
  const int tid = threadIdx.x, nt = blockDim.x;
  auto sd = [&](int a) { return 2 * a < G ? a : a - G; };  // signed grid index
  auto tw = [&](int m, double& c, double& sn) {  // e^{-2 pi i m / G}
    double si;
    sincospi(2.0 * (m % G) / G, &si, &c);
    sn = -si;
  };
  for (int comp = 0; comp < 6; ++comp) {
    // xx xy xz yy yz zz
    const int ci = comp < 3 ? 0 : (comp < 5 ? 1 : 2);
    const int cj = comp < 3 ? comp : (comp < 5 ? comp - 2 : 2);
    for (int e = tid; e < G * G * G; e += nt) {
      const int d[3] = {sd(e / (G * G)), sd((e / G) % G), sd(e % G)};
      double v = 0;
      if (abs(d[0]) <= res - 1 && abs(d[1]) <= res - 1 && abs(d[2]) <= res - 1) {
        double r[3];
        for (int a = 0; a < 3; ++a) r[a] = (double)(d[a] - (res - 1) * o[a]) * h;
        const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        const double dd = r2 + e2;
        if (deriv)
          v = ((ci == cj ? r2 - 2.0 * e2 : 0.0) - 3.0 * r[ci] * r[cj]) * scale / (dd * dd * sqrt(dd));
        else
          v = ((ci == cj ? r2 + 2.0 * e2 : 0.0) + r[ci] * r[cj]) * scale / (dd * sqrt(dd));
      }
      K[e] = v;
    }
    __syncthreads();
    for (int e = tid; e < G * G * H; e += nt) {  // z
      const int xy = e / H, kz = e % H;
      double re = 0, im = 0;
      for (int z = 0; z < G; ++z) {
        double c, sn;
        tw(kz * z, c, sn);
        re += K[xy * G + z] * c;
        im += K[xy * G + z] * sn;
      }
      A[e] = make_double2(re, im);
    }
    __syncthreads();
    for (int e = tid; e < G * G * H; e += nt) {  // y
      const int x = e / (G * H), ky = (e / H) % G, kz = e % H;
      double re = 0, im = 0;
      for (int y = 0; y < G; ++y) {
        double c, sn;
        tw(ky * y, c, sn);
        const double2 a = A[(x * G + y) * H + kz];
        re += a.x * c - a.y * sn;
        im += a.x * sn + a.y * c;
      }
      B[e] = make_double2(re, im);
    }
    __syncthreads();
    for (int e = tid; e < G * G * H; e += nt) {  // x
      const int kx = e / (G * H), kyz = e % (G * H);
      double re = 0, im = 0;
      for (int x = 0; x < G; ++x) {
        double c, sn;
        tw(kx * x, c, sn);
        const double2 b = B[x * G * H + kyz];
        re += b.x * c - b.y * sn;
        im += b.x * sn + b.y * c;
      }
      spec[((size_t)s * 6 + comp) * NK + e] = cmake((Real)re, (Real)im);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- forward
// Q_v[cr][k] for one source node: its shell densities on the res^3 lattice
// (interior zero), transformed along z (res -> H), y (res -> G), x (res -> G).
// RES > 0: the lattice size at compile time (loops unrolled, per-thread
// arrays in registers); RES = 0 takes it from `res_rt`.
template <int RES, typename Real>
__global__ void fft_forward_kernel(int G_rt, int res_rt, int P, const int* __restrict__ lat,
                                   const int* __restrict__ src_node, const Real* __restrict__ str, long long upbase,
                                   int R, typename Cplx<Real>::t* __restrict__ qhat, int NK,
                                   const int* __restrict__ nact) {
  using T2 = typename Cplx<Real>::t;
  extern __shared__ __align__(16) unsigned char fft_smem[];
  T2* smq = reinterpret_cast<T2*>(fft_smem);
  const int res = RES > 0 ? RES : res_rt;
  const int G = RES > 0 ? fft_grid(RES) : G_rt;
  const int H = G / 2 + 1, C = 3 * R, r3 = res * res * res;
  T2* tw = smq;                          // G
  T2* Z = tw + G;                        // [cr][x][y][kz]   C res res H
  T2* Y = Z + C * res * res * H;         // [cr][x][ky][kz]  C res G H
  Real* g = reinterpret_cast<Real*>(Y + C * res * G * H);  // [cr][x][y][z] C res^3
  const int node = src_node[blockIdx.x];
  if (nact && !nact[node]) return;  // a masked tree of the forest
  const int tid = threadIdx.x, nt = blockDim.x;
  twiddles<Real>(tw, G, -1.0);
  for (int e = tid; e < C * r3; e += nt) g[e] = 0;
  __syncthreads();
  const Real* src = str + (upbase + (long long)P * node) * C;
  for (int e = tid; e < P * C; e += nt) {
    const int p = e / C, cr = e - p * C;
    const int l = lat[p];
    g[cr * r3 + ((l & 255) * res + ((l >> 8) & 255)) * res + (l >> 16)] = src[e];
  }
  __syncthreads();
  for (int e = tid; e < C * res * res; e += nt) {  // z: one (cr, x, y) per thread
    const Real* gz = g + e * res;
#pragma unroll
    for (int kz = 0; kz < H; ++kz) {
      T2 a = cmake((Real)0, (Real)0);
#pragma unroll
      for (int z = 0; z < res; ++z) {
        const T2 w = tw[(kz * z) % G];
        a.x = rfma(gz[z], w.x, a.x);
        a.y = rfma(gz[z], w.y, a.y);
      }
      Z[e * H + kz] = a;
    }
  }
  __syncthreads();
  for (int e = tid; e < C * res * H; e += nt) {  // y: one (cr, x, kz) per thread
    const int crx = e / H, kz = e % H;
    T2 in[8];
#pragma unroll
    for (int y = 0; y < (RES > 0 ? RES : 8); ++y)
      if (y < res) in[y] = Z[(crx * res + y) * H + kz];
#pragma unroll
    for (int ky = 0; ky < G; ++ky) {
      T2 a = cmake((Real)0, (Real)0);
#pragma unroll
      for (int y = 0; y < (RES > 0 ? RES : 8); ++y)
        if (y < res) cmac(a, in[y], tw[(ky * y) % G]);
      Y[(crx * G + ky) * H + kz] = a;
    }
  }
  __syncthreads();
  T2* out = qhat + (size_t)blockIdx.x * C * NK;
  for (int e = tid; e < C * G * H; e += nt) {  // x: one (cr, ky, kz) per thread
    const int cr = e / (G * H), kyz = e % (G * H);
    T2 in[8];
#pragma unroll
    for (int x = 0; x < (RES > 0 ? RES : 8); ++x)
      if (x < res) in[x] = Y[(cr * res + x) * G * H + kyz];
#pragma unroll
    for (int kx = 0; kx < G; ++kx) {
      T2 a = cmake((Real)0, (Real)0);
#pragma unroll
      for (int x = 0; x < (RES > 0 ? RES : 8); ++x)
        if (x < res) cmac(a, in[x], tw[(kx * x) % G]);
      out[(size_t)cr * NK + kx * G * H + kyz] = a;
    }
  }
}

// ------------------------------------------------------------- accumulate
// C_i(k) = sum_{v in V(i)} Khat_{w,o}(k) Q_v(k): one target and frequency per
// thread; blocks run frequency-block-major so that the spectra in use at a
// time are a slice that stays in L2.
template <int R, typename Real>
__global__ void __launch_bounds__(128) fft_accumulate_kernel(int NK, const int* __restrict__ voff,
                                                             const int* __restrict__ vsrc,
                                                             const int* __restrict__ vspec,
                                                             const typename Cplx<Real>::t* __restrict__ spec,
                                                             const typename Cplx<Real>::t* __restrict__ qhat,
                                                             typename Cplx<Real>::t* __restrict__ chat,
                                                             const int* __restrict__ tgt_node,
                                                             const int* __restrict__ nact) {
  using T2 = typename Cplx<Real>::t;
  constexpr int C = 3 * R;
  const int t = blockIdx.x;
  const int k = blockIdx.y * blockDim.x + threadIdx.x;
  if (k >= NK) return;
  if (nact && !nact[tgt_node[t]]) return;
  T2 acc[C];
#pragma unroll
  for (int c = 0; c < C; ++c) acc[c] = cmake((Real)0, (Real)0);
  const int e1 = voff[t + 1];
  for (int e = voff[t]; e < e1; ++e) {
    const T2* Kp = spec + (size_t)vspec[e] * 6 * NK + k;
    const T2 kxx = Kp[0], kxy = Kp[NK], kxz = Kp[2 * NK], kyy = Kp[3 * NK], kyz = Kp[4 * NK], kzz = Kp[5 * NK];
    const T2* Q = qhat + (size_t)vsrc[e] * C * NK + k;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const T2 qx = Q[(3 * r) * NK], qy = Q[(3 * r + 1) * NK], qz = Q[(3 * r + 2) * NK];
      cmac(acc[3 * r], kxx, qx);
      cmac(acc[3 * r], kxy, qy);
      cmac(acc[3 * r], kxz, qz);
      cmac(acc[3 * r + 1], kxy, qx);
      cmac(acc[3 * r + 1], kyy, qy);
      cmac(acc[3 * r + 1], kyz, qz);
      cmac(acc[3 * r + 2], kxz, qx);
      cmac(acc[3 * r + 2], kyz, qy);
      cmac(acc[3 * r + 2], kzz, qz);
    }
  }
  T2* out = chat + (size_t)t * C * NK + k;
#pragma unroll
  for (int c = 0; c < C; ++c) out[(size_t)c * NK] = acc[c];
}

// Child pairs of a (P, N) record at difference dl = (ex+1) * 9 + (ey+1) * 3 +
// (ez+1): bit 8 a + b for every child a of P whose neighbour b = a + (ex, ey,
// ez) lies in N's box (a compile-time constant for a constant dl).
__host__ __device__ constexpr uint64_t group_mask(int dl) {
  uint64_t gm = 0;
  for (int a = 0; a < 8; ++a) {
    const int bx = (a >> 2) + dl / 9 - 1, by = ((a >> 1) & 1) + (dl / 3) % 3 - 1, bz = (a & 1) + dl % 3 - 1;
    if (bx >= 0 && bx <= 1 && by >= 0 && by <= 1 && bz >= 0 && bz <= 1)
      gm |= 1ull << (a * 8 + (bx * 4 + by * 2 + bz));
  }
  return gm;
}

// The pairs of one difference (ex, ey, ez) of a (P, N) record: child a of P
// takes child b = a + (ex, ey, ez) of N through the kernel spectrum K (xx, xy,
// xz, yy, yz, zz) when its bit 8 a + b is set; my[(b * 3 + c) * BLK] holds
// N's child spectra.
template <int BLK, typename T2>
__device__ __forceinline__ void family_group(T2 (&acc)[8][3], const T2 (&K)[6], const T2* my, int ex, int ey,
                                             int ez, uint64_t bits) {
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int bx = (a >> 2) + ex, by = ((a >> 1) & 1) + ey, bz = (a & 1) + ez;
    if (!(bx >= 0 && bx <= 1 && by >= 0 && by <= 1 && bz >= 0 && bz <= 1)) continue;
    const int b = bx * 4 + by * 2 + bz;
    if (!((bits >> (a * 8 + b)) & 1)) continue;
    const T2 qx = my[(b * 3) * BLK], qy = my[(b * 3 + 1) * BLK], qz = my[(b * 3 + 2) * BLK];
    cmac(acc[a][0], K[0], qx);
    cmac(acc[a][0], K[1], qy);
    cmac(acc[a][0], K[2], qz);
    cmac(acc[a][1], K[1], qx);
    cmac(acc[a][1], K[3], qy);
    cmac(acc[a][1], K[4], qz);
    cmac(acc[a][2], K[2], qx);
    cmac(acc[a][2], K[4], qy);
    cmac(acc[a][2], K[5], qz);
  }
}

constexpr int kFamBlk = 128;  // frequencies per block of the direct-load form
template <typename Real>
size_t family_smem() {
  return sizeof(typename Cplx<Real>::t) * 24 * kFamBlk + sizeof(int) * 343;
}

// Parent-grouped accumulation (see FftFamily): thread (family, frequency k)
// holds the 8 children's accumulators of one right-hand side at a time; per
// (P, N) record the 8 source spectra go to this thread's own shared-memory
// slots, then for each of the 27 values of pos_v - pos_i present in the
// record the kernel spectrum of offset 2 d + delta is loaded once and applied
// to every pair with that difference (the spectrum slots of the family's
// operator, one per offset code, are read into shared memory once, so a
// spectrum's address needs no global load).  Loop bounds and child positions
// are compile-time, so accumulators stay in registers.  The kernel is bound
// by moving kernel spectra from L2 (96 bytes a frequency per difference, for
// 2.5 pairs on average): hiding their latency did not pay -- loading the
// next difference's spectrum one step ahead into registers (42 more
// registers, 2 blocks per SM instead of 3) ran 45% slower, an L1 prefetch of
// it 32% slower, a producer warp staging spectra in a 5-stage shared-memory
// ring 27% slower with bulk copies and 36% slower with 16-byte cp.async
// (the ring and the source slots leave 8 arithmetic warps per SM, whose
// per-record source loads stay exposed).  Every right-hand side sums its pairs in
// the same order, so a pass of R right-hand sides gives each of them bitwise
// the result of a pass of one.
template <typename Real>
__global__ void __launch_bounds__(128) fft_accumulate_family_kernel(
    int NK, const FftFamily* __restrict__ fams, const FftFamilyPair* __restrict__ pairs,
    const int* __restrict__ spec_of, const typename Cplx<Real>::t* __restrict__ spec,
    const typename Cplx<Real>::t* __restrict__ qhat, typename Cplx<Real>::t* __restrict__ chat,
    const int* __restrict__ tgt_node, const int* __restrict__ nact, int R) {
  using T2 = typename Cplx<Real>::t;
  constexpr int BLK = kFamBlk;
  extern __shared__ __align__(16) unsigned char fam_direct_smem[];
  T2* sq = reinterpret_cast<T2*>(fam_direct_smem);  // this thread's source spectra: [pos * 3 + c][thread]
  int* so = reinterpret_cast<int*>(sq + 24 * BLK);   // spectrum slot of each offset code (the family's operator)
  const FftFamily fam = fams[blockIdx.x];
  const int k = blockIdx.y * BLK + threadIdx.x;
  if (nact) {
    int t0 = 0;
    while (t0 < 7 && fam.tgt[t0] < 0) ++t0;
    if (!nact[tgt_node[fam.tgt[t0]]]) return;
  }
  for (int c = threadIdx.x; c < 343; c += BLK) so[c] = spec_of[(size_t)fam.op * 343 + c];
  __syncthreads();
  if (k >= NK) return;
  const int C = 3 * R;
  T2* my = sq + threadIdx.x;
  for (int r = 0; r < R; ++r) {
  T2 acc[8][3];
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[a][c] = cmake((Real)0, (Real)0);
  for (int pr = fam.first; pr < fam.first + fam.count; ++pr) {
    const FftFamilyPair rec = pairs[pr];
    const uint64_t mask = (uint64_t)rec.mask_lo | ((uint64_t)rec.mask_hi << 32);
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const int sl = rec.src[b];
      if (sl >= 0) {
        const T2* Q = qhat + ((size_t)sl * C + 3 * r) * NK + k;
#pragma unroll
        for (int c = 0; c < 3; ++c) my[(b * 3 + c) * BLK] = Q[(size_t)c * NK];
      }
    }
    const int dx2 = 2 * (rec.dcode / 9 - 1), dy2 = 2 * ((rec.dcode / 3) % 3 - 1), dz2 = 2 * (rec.dcode % 3 - 1);
#pragma unroll
    for (int dl = 0; dl < 27; ++dl) {
      const int ex = dl / 9 - 1, ey = (dl / 3) % 3 - 1, ez = dl % 3 - 1;
      const uint64_t bits = mask & group_mask(dl);
      if (bits == 0) continue;
      const int code = (dx2 + ex + 3) * 49 + (dy2 + ey + 3) * 7 + (dz2 + ez + 3);
      const T2* Kp = spec + (size_t)so[code] * 6 * NK + k;
      const T2 K[6] = {Kp[0], Kp[NK], Kp[2 * NK], Kp[3 * NK], Kp[4 * NK], Kp[5 * NK]};
      family_group<BLK>(acc, K, my, ex, ey, ez, bits);
    }
  }
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int t = fam.tgt[a];
    if (t < 0) continue;
    T2* out = chat + ((size_t)t * C + 3 * r) * NK + k;
#pragma unroll
    for (int c = 0; c < 3; ++c) out[(size_t)c * NK] = acc[a][c];
  }
  }
}

// ---------------------------------------------------------------- inverse
// check of one target node at its shell lattice points from C_i: inverse
// passes along x (G -> res), y (G -> res) and z (half spectrum -> res, real).
template <int RES, typename Real>
__global__ void fft_inverse_kernel(int G_rt, int res_rt, int P, const int* __restrict__ lat,
                                   const int* __restrict__ tgt_node, const typename Cplx<Real>::t* __restrict__ chat,
                                   int R, Real* __restrict__ check, int NK, const int* __restrict__ nact) {
  using T2 = typename Cplx<Real>::t;
  extern __shared__ __align__(16) unsigned char fft_smem[];
  T2* smc = reinterpret_cast<T2*>(fft_smem);
  const int res = RES > 0 ? RES : res_rt;
  const int G = RES > 0 ? fft_grid(RES) : G_rt;
  const int H = G / 2 + 1, C = 3 * R, r3 = res * res * res;
  T2* tw = smc;                   // G
  T2* X = tw + G;                 // [cr][x][ky][kz]  C res G H
  T2* Yv = X + C * res * G * H;   // [cr][x][y][kz]   C res res H
  Real* out = reinterpret_cast<Real*>(X);  // [cr][x][y][z] (X is dead by then)
  const int node = tgt_node[blockIdx.x];
  if (nact && !nact[node]) return;
  const int tid = threadIdx.x, nt = blockDim.x;
  twiddles<Real>(tw, G, 1.0);
  __syncthreads();
  const T2* ci = chat + (size_t)blockIdx.x * C * NK;
  for (int e = tid; e < C * G * H; e += nt) {  // x: one (cr, ky, kz) per thread
    const int cr = e / (G * H), kyz = e % (G * H);
    T2 a[8];
#pragma unroll
    for (int x = 0; x < 8; ++x) a[x] = cmake((Real)0, (Real)0);
#pragma unroll
    for (int kx = 0; kx < G; ++kx) {
      const T2 v = ci[(size_t)cr * NK + kx * G * H + kyz];
#pragma unroll
      for (int x = 0; x < (RES > 0 ? RES : 8); ++x)
        if (x < res) cmac(a[x], v, tw[(kx * x) % G]);
    }
#pragma unroll
    for (int x = 0; x < (RES > 0 ? RES : 8); ++x)
      if (x < res) X[(cr * res + x) * G * H + kyz] = a[x];
  }
  __syncthreads();
  for (int e = tid; e < C * res * H; e += nt) {  // y: one (cr, x, kz) per thread
    const int crx = e / H, kz = e % H;
    T2 a[8];
#pragma unroll
    for (int y = 0; y < 8; ++y) a[y] = cmake((Real)0, (Real)0);
#pragma unroll
    for (int ky = 0; ky < G; ++ky) {
      const T2 v = X[(crx * G + ky) * H + kz];
#pragma unroll
      for (int y = 0; y < (RES > 0 ? RES : 8); ++y)
        if (y < res) cmac(a[y], v, tw[(ky * y) % G]);
    }
#pragma unroll
    for (int y = 0; y < (RES > 0 ? RES : 8); ++y)
      if (y < res) Yv[(crx * res + y) * H + kz] = a[y];
  }
  __syncthreads();
  for (int e = tid; e < C * res * res; e += nt) {  // z: one (cr, x, y) per thread, real output
    const T2* yz = Yv + e * H;
#pragma unroll
    for (int z = 0; z < (RES > 0 ? RES : 8); ++z) {
      if (z >= res) break;
      Real v = 0;
#pragma unroll
      for (int kz = 0; kz < (RES > 0 ? RES + 1 : 9); ++kz) {
        if (kz >= H) break;
        const Real w = (kz == 0 || 2 * kz == G) ? (Real)1 : (Real)2;
        const T2 t = tw[(kz * z) % G];
        v = rfma(w, yz[kz].x * t.x - yz[kz].y * t.y, v);
      }
      out[e * res + z] = v;
    }
  }
  __syncthreads();
  Real* dst = check + (long long)P * node * C;
  for (int e = tid; e < P * C; e += nt) {
    const int p = e / C, cr = e - p * C;
    const int l = lat[p];
    dst[e] = out[cr * r3 + ((l & 255) * res + ((l >> 8) & 255)) * res + (l >> 16)];
  }
}

// es: bytes of one real number (a complex one takes 2 es)
size_t forward_smem(int G, int res, int R, size_t es) {
  const int H = G / 2 + 1, C = 3 * R;
  return 2 * es * (G + (size_t)C * res * res * H + (size_t)C * res * G * H) + es * (size_t)C * res * res * res;
}
size_t inverse_smem(int G, int res, int R, size_t es) {
  const int H = G / 2 + 1, C = 3 * R;
  return 2 * es * (G + (size_t)C * res * G * H + (size_t)C * res * res * H);
}

// The parent-grouped plan (FftFamily): families in parent order, records in
// colleague order.  Leaves f.family false if some V pair does not join
// children of two touching parents of one level.
void build_families(const HostTree& t, const std::vector<int>& tgt, const std::vector<int>& src,
                    const std::vector<int>& voff, const std::vector<int>& vsrc, const std::vector<int>& node_op,
                    const std::map<int64_t, int>& spec_slot, size_t nops, FftM2L& f, cudaStream_t st) {
  f.family = false;
  f.nfam = 0;
  if (tgt.empty()) return;
  auto pos = [&](int32_t c, int32_t p, int d) {
    const std::vector<int32_t>& v = d == 0 ? t.ix : d == 1 ? t.iy : t.iz;
    return v[c] - 2 * v[p];
  };
  auto pcode = [&](int32_t c, int32_t p) {
    int code = 0;
    for (int d = 0; d < 3; ++d) {
      const int q = pos(c, p, d);
      if (q < 0 || q > 1) return -1;
      code = code * 2 + q;
    }
    return code;
  };
  std::map<int32_t, int> fam_of;                      // parent -> family
  std::vector<FftFamily> fams;
  std::vector<std::map<int32_t, FftFamilyPair>> recs;  // per family: colleague -> record
  for (size_t ts = 0; ts < tgt.size(); ++ts) {
    const int32_t i = tgt[ts], P = t.parent[i];
    if (P < 0) return;
    const int pa = pcode(i, P);
    if (pa < 0) return;
    auto it = fam_of.find(P);
    if (it == fam_of.end()) {
      it = fam_of.emplace(P, (int)fams.size()).first;
      FftFamily fm{};
      for (int a = 0; a < 8; ++a) fm.tgt[a] = -1;
      fams.push_back(fm);
      recs.emplace_back();
    }
    FftFamily& fm = fams[it->second];
    fm.tgt[pa] = (int)ts;
    for (int e = voff[ts]; e < voff[ts + 1]; ++e) {
      const int32_t v = src[vsrc[e]], N = t.parent[v];
      if (N < 0 || N == P || t.level[v] != t.level[i] || t.level[N] != t.level[P]) return;
      const int dx = t.ix[N] - t.ix[P], dy = t.iy[N] - t.iy[P], dz = t.iz[N] - t.iz[P];
      if (std::abs(dx) > 1 || std::abs(dy) > 1 || std::abs(dz) > 1) return;
      const int pb = pcode(v, N);
      if (pb < 0) return;
      auto& m = recs[it->second];
      auto rit = m.find(N);
      if (rit == m.end()) {
        FftFamilyPair r{};
        r.dcode = (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1);
        r.op = node_op[i];
        for (int b = 0; b < 8; ++b) r.src[b] = -1;
        rit = m.emplace(N, r).first;
      }
      FftFamilyPair& r = rit->second;
      if (r.op != node_op[i]) return;
      const int bit = pa * 8 + pb;
      if (bit < 32) r.mask_lo |= 1u << bit;
      else r.mask_hi |= 1u << (bit - 32);
      r.src[pb] = vsrc[e];
    }
  }
  std::vector<FftFamilyPair> pairs;
  for (size_t fi = 0; fi < fams.size(); ++fi) {
    fams[fi].first = (int)pairs.size();
    fams[fi].op = recs[fi].empty() ? 0 : recs[fi].begin()->second.op;
    for (auto& kv : recs[fi]) {
      // the accumulation reads one row of spec_of per family
      if (kv.second.op != fams[fi].op) return;
      pairs.push_back(kv.second);
    }
    fams[fi].count = (int)pairs.size() - fams[fi].first;
  }
  f.records = (int64_t)pairs.size();
  f.groups = 0;
  for (const FftFamilyPair& r : pairs) {
    const uint64_t mask = (uint64_t)r.mask_lo | ((uint64_t)r.mask_hi << 32);
    for (int dl = 0; dl < 27; ++dl) f.groups += (mask & group_mask(dl)) != 0;
  }
  std::vector<int> spec_of(std::max<size_t>(nops, 1) * 343, -1);
  for (const auto& kv : spec_slot) spec_of[(size_t)(kv.first / 343) * 343 + (size_t)(kv.first % 343)] = kv.second;
  f.fams.upload(fams, st);
  f.fpairs.upload(pairs, st);
  f.spec_of.upload(spec_of, st);
  f.nfam = (int)fams.size();
  f.family = true;
}

int optin_smem() {
  int dev = 0, optin = 0;
  NNK_CUDA(cudaGetDevice(&dev));
  NNK_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  return optin;
}

template <typename Real>
void set_smem_attributes(int optin) {
  // The limit is an attribute of the kernel, shared by every plan of the
  // process (a p = 4 plan built after a p = 6 one must not lower it): set
  // the device's opt-in maximum.
  NNK_CUDA(cudaFuncSetAttribute(fft_forward_kernel<0, Real>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
  NNK_CUDA(cudaFuncSetAttribute(fft_inverse_kernel<0, Real>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
  NNK_CUDA(cudaFuncSetAttribute(fft_forward_kernel<4, Real>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
  NNK_CUDA(cudaFuncSetAttribute(fft_inverse_kernel<4, Real>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
  NNK_CUDA(cudaFuncSetAttribute(fft_forward_kernel<6, Real>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
  NNK_CUDA(cudaFuncSetAttribute(fft_inverse_kernel<6, Real>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
  NNK_CUDA(cudaFuncSetAttribute(fft_accumulate_family_kernel<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)family_smem<Real>()));
}

template <typename Real>
void run_fft_m2l(FftM2L& f, const Real* str, long long upbase, int R, Real* check, cudaStream_t st,
                 const int* nact, typename Cplx<Real>::t* spec, typename Cplx<Real>::t* qhat,
                 typename Cplx<Real>::t* chat) {
  if (f.ntgt == 0) return;
  if (R > f.Rcap) throw Error(NNK_E_STATE, "Fourier M2L sized for fewer right-hand sides");
  const int G = f.G, res = f.res;
  const size_t es = sizeof(Real);
  auto fwd = res == 6 ? fft_forward_kernel<6, Real> : res == 4 ? fft_forward_kernel<4, Real>
                                                                : fft_forward_kernel<0, Real>;
  auto inv = res == 6 ? fft_inverse_kernel<6, Real> : res == 4 ? fft_inverse_kernel<4, Real>
                                                                : fft_inverse_kernel<0, Real>;
  fwd<<<f.nsrc, 256, forward_smem(G, res, R, es), st>>>(G, res, f.P, f.lat.p, f.src_node.p, str, upbase, R, qhat,
                                                        f.NK, nact);
  NNK_CHECK_LAUNCH();
  if (f.family) {
    fft_accumulate_family_kernel<Real><<<dim3(f.nfam, (f.NK + kFamBlk - 1) / kFamBlk), kFamBlk, family_smem<Real>(),
                                         st>>>(f.NK, f.fams.p, f.fpairs.p, f.spec_of.p, spec, qhat, chat,
                                               f.tgt_node.p, nact, R);
    NNK_CHECK_LAUNCH();
    inv<<<f.ntgt, 256, inverse_smem(G, res, R, es), st>>>(G, res, f.P, f.lat.p, f.tgt_node.p, chat, R, check, f.NK,
                                                          nact);
    NNK_CHECK_LAUNCH();
    return;
  }
  dim3 grid(f.ntgt, (f.NK + 127) / 128);
#define NNK_FFT_ACC(RR)                                                                                       \
  fft_accumulate_kernel<RR, Real><<<grid, 128, 0, st>>>(f.NK, f.voff.p, f.vsrc.p, f.vspec.p, spec, qhat, chat, \
                                                        f.tgt_node.p, nact)
  switch (R) {
    case 1: NNK_FFT_ACC(1); break;
    case 2: NNK_FFT_ACC(2); break;
    case 3: NNK_FFT_ACC(3); break;
    case 4: NNK_FFT_ACC(4); break;
    case 6: NNK_FFT_ACC(6); break;
    default:
      throw Error(NNK_E_ARG, "Fourier M2L supports 1, 2, 3, 4 or 6 right-hand sides per pass");
  }
#undef NNK_FFT_ACC
  NNK_CHECK_LAUNCH();
  inv<<<f.ntgt, 256, inverse_smem(G, res, R, es), st>>>(G, res, f.P, f.lat.p, f.tgt_node.p, chat, R, check, f.NK,
                                                        nact);
  NNK_CHECK_LAUNCH();
}

}  // namespace

int fft_m2l_max_rhs(int res, bool fp64) {
  const int optin = optin_smem();
  const size_t es = fp64 ? sizeof(double) : sizeof(float);
  for (int R : {6, 4, 3, 2, 1})
    if (forward_smem(fft_grid(res), res, R, es) <= (size_t)optin &&
        inverse_smem(fft_grid(res), res, R, es) <= (size_t)optin)
      return R;
  return 0;
}

void build_fft_m2l(const HostTree& t, int res, int shells, double eps, double mu, const std::vector<double>& op_w,
                   const std::vector<int>& node_op, int Rmax, bool fp64, FftM2L& f, cudaStream_t st) {
  if (res > 8) throw Error(NNK_E_ARG, "Fourier M2L supports coronaRes up to 8");
  f.fp64 = fp64;
  f.res = res;
  f.G = fft_grid(res);
  const int G = f.G, H = G / 2 + 1;
  f.NK = G * G * H;
  f.Rcap = Rmax;
  // shell lattice in the order of the surface points (genupsurf.m:24-33)
  std::vector<int> lat;
  auto inner = [&](int a) { return a >= shells && a <= res - 1 - shells; };
  for (int k = 0; k < res; ++k)
    for (int i = 0; i < res; ++i)
      for (int j = 0; j < res; ++j)
        if (!(inner(j) && inner(i) && inner(k))) lat.push_back(i | (j << 8) | (k << 16));
  f.P = (int)lat.size();
  std::vector<int> tgt, voff{0}, vsrc, vspec, src;
  std::vector<double> slot_w;
  std::vector<int> slot_code;
  std::map<int32_t, int> src_slot;
  std::map<int64_t, int> spec_slot;
  for (int32_t i = 0; i < t.nodes; ++i) {
    if (t.V.off[i + 1] == t.V.off[i]) continue;
    tgt.push_back(i);
    for (int64_t k = t.V.off[i]; k < t.V.off[i + 1]; ++k) {
      const int32_t v = t.V.idx[k];
      const int ox = t.ix[v] - t.ix[i], oy = t.iy[v] - t.iy[i], oz = t.iz[v] - t.iz[i];
      if (std::abs(ox) > 3 || std::abs(oy) > 3 || std::abs(oz) > 3)
        throw Error(NNK_E_STATE, "V-list offset outside [-3,3]^3");
      const int code = (ox + 3) * 49 + (oy + 3) * 7 + (oz + 3);
      const int op = node_op[i];
      auto sit = src_slot.find(v);
      if (sit == src_slot.end()) {
        sit = src_slot.emplace(v, (int)src.size()).first;
        src.push_back(v);
      }
      const int64_t key = (int64_t)op * 343 + code;
      auto kit = spec_slot.find(key);
      if (kit == spec_slot.end()) {
        kit = spec_slot.emplace(key, (int)slot_w.size()).first;
        slot_w.push_back(op_w[op]);
        slot_code.push_back(code);
      }
      vsrc.push_back(sit->second);
      vspec.push_back(kit->second);
    }
    voff.push_back((int)vsrc.size());
  }
  // sources in node order keep siblings' spectra adjacent
  {
    std::vector<int> order(src.size());
    for (size_t a = 0; a < order.size(); ++a) order[a] = (int)a;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return src[a] < src[b]; });
    std::vector<int> remap(src.size()), s2(src.size());
    for (size_t a = 0; a < order.size(); ++a) {
      remap[order[a]] = (int)a;
      s2[a] = src[order[a]];
    }
    src.swap(s2);
    for (int& s : vsrc) s = remap[s];
  }
  f.slot_w_host = slot_w;
  f.slot_code_host = slot_code;
  f.ntgt = (int)tgt.size();
  f.nsrc = (int)src.size();
  f.nspec = (int)slot_w.size();
  f.pairs = (int64_t)vsrc.size();
  build_families(t, tgt, src, voff, vsrc, node_op, spec_slot, op_w.size(), f, st);
  f.lat.upload(lat, st);
  f.tgt_node.upload(tgt, st);
  f.src_node.upload(src, st);
  f.voff.upload(voff, st);
  f.vsrc.upload(vsrc, st);
  f.vspec.upload(vspec, st);
  const size_t nspec = std::max<size_t>(1, (size_t)f.nspec * 6 * f.NK);
  const size_t nq = std::max<size_t>(1, (size_t)f.nsrc * 3 * Rmax * f.NK);
  const size_t nc = std::max<size_t>(1, (size_t)f.ntgt * 3 * Rmax * f.NK);
  if (fp64) {
    f.spec64.alloc(nspec);
    f.qhat64.alloc(nq);
    f.chat64.alloc(nc);
  } else {
    f.spec.alloc(nspec);
    f.qhat.alloc(nq);
    f.chat.alloc(nc);
  }
  if (f.nspec) {
    DBuf<double> dw;
    DBuf<int> dc;
    dw.upload(slot_w, st);
    dc.upload(slot_code, st);
    const size_t sm = sizeof(double) * (size_t)spectra_real_len(G) + 2 * sizeof(double2) * (size_t)G * G * H;
    const double scale = 1.0 / (8.0 * M_PI * mu * (double)G * G * G);
    if (fp64) {
      NNK_CUDA(cudaFuncSetAttribute(fft_spectra_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)sm));
      fft_spectra_kernel<double><<<f.nspec, 256, sm, st>>>(G, res, dw.p, dc.p, eps * eps, scale, f.spec64.p, f.NK);
    } else {
      NNK_CUDA(cudaFuncSetAttribute(fft_spectra_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)sm));
      fft_spectra_kernel<float><<<f.nspec, 256, sm, st>>>(G, res, dw.p, dc.p, eps * eps, scale, f.spec.p, f.NK);
    }
    NNK_CHECK_LAUNCH();
    NNK_CUDA(cudaStreamSynchronize(st));
  }
  const size_t es = fp64 ? sizeof(double) : sizeof(float);
  f.fwd_smem = forward_smem(G, res, Rmax, es);
  f.inv_smem = inverse_smem(G, res, Rmax, es);
  const int optin = optin_smem();
  if (f.fwd_smem > (size_t)optin || f.inv_smem > (size_t)optin)
    throw Error(NNK_E_ARG, "Fourier M2L: too many right-hand sides per pass for shared memory");
  if (fp64) set_smem_attributes<double>(optin);
  else set_smem_attributes<float>(optin);
  NNK_CUDA(cudaStreamSynchronize(st));
}

void launch_fft_m2l(FftM2L& f, const float* str, long long upbase, int R, float* check, cudaStream_t st,
                    const int* nact) {
  if (f.fp64) throw Error(NNK_E_STATE, "Fourier M2L built for FP64 densities");
  run_fft_m2l<float>(f, str, upbase, R, check, st, nact, f.spec.p, f.qhat.p, f.chat.p);
}

void launch_fft_m2l(FftM2L& f, const double* str, long long upbase, int R, double* check, cudaStream_t st,
                    const int* nact) {
  if (!f.fp64) throw Error(NNK_E_STATE, "Fourier M2L built for FP32 densities");
  run_fft_m2l<double>(f, str, upbase, R, check, st, nact, f.spec64.p, f.qhat64.p, f.chat64.p);
}

void build_fft_deriv(FftM2L& f, double eps, double mu, cudaStream_t st) {
  if (!f.fp64) throw Error(NNK_E_STATE, "the eps-derivative spectra need an FP64 Fourier M2L");
  f.dspec64.alloc(std::max<size_t>(1, (size_t)f.nspec * 6 * f.NK));
  if (!f.nspec) return;
  const int G = f.G, H = G / 2 + 1;
  DBuf<double> dw;
  DBuf<int> dc;
  dw.upload(f.slot_w_host, st);
  dc.upload(f.slot_code_host, st);
  const size_t sm = sizeof(double) * (size_t)spectra_real_len(G) + 2 * sizeof(double2) * (size_t)G * G * H;
  NNK_CUDA(cudaFuncSetAttribute(fft_spectra_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  fft_spectra_kernel<double><<<f.nspec, 256, sm, st>>>(G, f.res, dw.p, dc.p, eps * eps,
                                                        eps / (8.0 * M_PI * mu * (double)G * G * G), f.dspec64.p,
                                                        f.NK, 1);
  NNK_CHECK_LAUNCH();
  NNK_CUDA(cudaStreamSynchronize(st));
}

void launch_fft_m2l_deriv(FftM2L& f, const double* str, long long upbase, double* check, cudaStream_t st) {
  if (!f.fp64 || !f.dspec64.p) throw Error(NNK_E_STATE, "eps-derivative spectra not built");
  run_fft_m2l<double>(f, str, upbase, 1, check, st, nullptr, f.dspec64.p, f.qhat64.p, f.chat64.p);
}

}  // namespace nnk
