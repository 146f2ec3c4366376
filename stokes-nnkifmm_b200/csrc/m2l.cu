// TF32 tcgen05 M2L (see m2l.h).
//
// Shared memory per stage (2 stages):
//   A: 128 rows x 128 B (32 TF32 of K), K-major, 128-byte swizzle
//   B: NP rows x 128 B, same layout, one bulk copy of a pre-swizzled chunk
// One thread issues the MMAs (kind::tf32, M = 128, N = NP or NP/2, K = 8 per
// instruction, four per 32-wide K chunk); all 128 threads gather A rows; the
// accumulator (128 lanes x NP columns FP32) lives in TMEM.  Every mbarrier
// wait is bounded; a timeout sets the error flag and the CTA drains and exits.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <map>

#include "m2l.h"
#include "tc_util.cuh"

namespace nnk {

namespace {

constexpr int kTileRows = 128;
constexpr int kCodesPerUnit = 32;  // offset codes per work unit (7^3 = 343 codes)
constexpr size_t kImgSmemMax = 200 * 1024;  // dynamic shared memory of the image kernel, at most

using namespace tc;

__device__ __forceinline__ float to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__global__ void __launch_bounds__(128, 1)
    m2l_gen_kernel(const M2LUnit* __restrict__ units, const int* __restrict__ tile_nodes,
                    const int* __restrict__ tile_slot0, const int* __restrict__ slot_code,
                    const float* __restrict__ slot_h, const int* __restrict__ slot_src,
                    const int* __restrict__ lat_packed, int P, int res, float e2, float scale,
                    const float* __restrict__ src, float* __restrict__ check, int ldc, int NP, int* err) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  uint8_t* sbase = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  const uint32_t A_BYTES = kTileRows * 128, B_BYTES = (uint32_t)NP * 128;
  uint8_t* sA0 = sbase;
  uint8_t* sB0 = sbase + 2 * A_BYTES;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sbase + 2 * A_BYTES + 2 * B_BYTES);  // done[2] acc
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 3);
  volatile int* abort_s = reinterpret_cast<volatile int*>(tmem_slot + 1);
  int* lat = reinterpret_cast<int*>(tmem_slot + 2);  // P packed lattice indices

  const int tid = threadIdx.x, warp = tid >> 5;
  const M2LUnit u = units[blockIdx.x];
  const int nchunks = NP / 32;
  const int nhalves = NP > 256 ? 2 : 1;
  const int nh = NP / nhalves;
  const uint32_t ncols = NP > 256 ? 512u : 256u;
  const uint32_t idesc = tf32_idesc(nh);
  const int n3 = 3 * P;

  if (tid == 0) {
    for (int k = 0; k < 3; ++k) mbar_init(&bars[k], 1);
    *abort_s = 0;
    fence_barrier_init();
  }
  for (int p = tid; p < P; p += blockDim.x) lat[p] = lat_packed[p];
  // operator rows >= 3P stay zero in both stages
  for (int i = tid; i < (int)(2 * B_BYTES / 16); i += blockDim.x)
    reinterpret_cast<float4*>(sB0)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  if (warp == 0) tmem_alloc(tmem_slot, ncols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int node = tile_nodes[u.tile * kTileRows + tid];
  const int slot_base = tile_slot0[u.tile] + u.slot0;
  const int nsteps = u.nslot * nchunks;
  int issued = 0;
  // Step s uses stage s & 1: every thread gathers its A row (32 TF32 of its
  // source node's density) and computes a share of the operator chunk
  //   T[n = 3a+al][k = 3b+be] = S_al,be(r) / (8 pi mu),  r = (lat_a - lat_b - (res-1) o) h,
  // k in [32c, 32c+32), rounded to TF32 into the swizzled B tile.
  auto prepare = [&](int s) {
    const int st = s & 1;
    const int slot = slot_base + s / nchunks;
    const int c = s % nchunks;
    const int v = slot_src[(size_t)slot * kTileRows + tid];
    float4* dA = reinterpret_cast<float4*>(sA0 + st * A_BYTES + tid * 128);
    if (v >= 0) {
      const float4* g4 = reinterpret_cast<const float4*>(src + (size_t)v * NP + c * 32);
#pragma unroll
      for (int j = 0; j < 8; ++j) dA[j ^ (tid & 7)] = __ldg(g4 + j);
    } else {
#pragma unroll
      for (int j = 0; j < 8; ++j) dA[j] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    const int code = slot_code[slot];
    const float h = slot_h[slot];
    const int ox = (code / 49 - 3) * (res - 1), oy = ((code / 7) % 7 - 3) * (res - 1), oz = (code % 7 - 3) * (res - 1);
    const int k0 = 32 * c;
    const int b0 = k0 / 3, b1 = min(P - 1, (k0 + 31) / 3);
    const int nbp = b1 - b0 + 1;
    uint8_t* sB = sB0 + st * B_BYTES;
    for (int pr = tid; pr < P * nbp; pr += blockDim.x) {
      const int a = pr / nbp, b = b0 + pr % nbp;
      const int la = lat[a], lb = lat[b];
      const float rx = (float)((la & 15) - (lb & 15) - ox) * h;
      const float ry = (float)(((la >> 4) & 15) - ((lb >> 4) & 15) - oy) * h;
      const float rz = (float)(((la >> 8) & 15) - ((lb >> 8) & 15) - oz) * h;
      const float r2 = rx * rx + ry * ry + rz * rz;
      const float d = r2 + e2;
      const float inv = rsqrtf(d);
      const float w3 = inv * inv * inv * scale;
      const float r[3] = {rx, ry, rz};
#pragma unroll
      for (int be = 0; be < 3; ++be) {
        const int kl = 3 * b + be - k0;
        if (kl < 0 || kl >= 32) continue;
        const int j = kl >> 2, e = kl & 3;
#pragma unroll
        for (int al = 0; al < 3; ++al) {
          const int n = 3 * a + al;
          const float val = (r[al] * r[be] + (al == be ? d + e2 : 0.f)) * w3;
          *reinterpret_cast<float*>(sB + n * 128 + ((j ^ (n & 7)) << 4) + e * 4) = to_tf32(val);
        }
      }
    }
    if (k0 + 32 > n3) {  // padded K columns of the last chunk
      const int kpad = k0 + 32 - n3;
      for (int q = tid; q < n3 * kpad; q += blockDim.x) {
        const int n = q / kpad, kl = (n3 - k0) + q % kpad;
        const int j = kl >> 2, e = kl & 3;
        *reinterpret_cast<float*>(sB + n * 128 + ((j ^ (n & 7)) << 4) + e * 4) = 0.f;
      }
    }
    fence_proxy_async();
  };
  if (nsteps > 0) prepare(0);
  __syncthreads();
  for (int s = 0; s < nsteps; ++s) {
    const int st = s & 1;
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a0 = smem_u32(sA0 + st * A_BYTES), b0 = smem_u32(sB0 + st * B_BYTES);
#pragma unroll
      for (int k8 = 0; k8 < 4; ++k8)
        for (int h = 0; h < nhalves; ++h)
          umma_tf32(tmem + (uint32_t)(h * nh), sw128_desc(a0 + k8 * 32), sw128_desc(b0 + h * nh * 128 + k8 * 32),
                    idesc, (s > 0 || k8 > 0) ? 1u : 0u);
      umma_commit(&bars[st]);
      ++issued;
    }
    // while the MMAs of step s run, fill the other stage with step s+1 once
    // the MMAs of step s-1 (its previous user) are done
    if (s + 1 < nsteps) {
      if (s >= 1 && !mbar_wait(&bars[st ^ 1], ((s - 1) >> 1) & 1)) {
        *abort_s = 1;
        atomicOr(err, 1);
      }
      if (!*abort_s) prepare(s + 1);
    }
    __syncthreads();
    if (*abort_s) break;
  }
  __syncthreads();
  // drain: the commit tracks every MMA this thread issued
  if (tid == 0) umma_commit(&bars[2]);
  // the read-back is warp-collective: a warp reads only if all its lanes saw
  // the accumulator complete
  const bool acc_ok = __all_sync(0xffffffffu, mbar_wait(&bars[2], 0));
  if (!acc_ok && (tid & 31) == 0) atomicOr(err, 4);
  (void)issued;
  tc_fence_after();
  if (!*abort_s && acc_ok && nsteps > 0) {
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
    for (int col = 0; col < NP; col += 16) {
      float vals[16];
      tmem_ld16(lane_addr + col, vals);
      if (node >= 0) {
        float* dst = check + (size_t)node * ldc;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int c0 = col + 4 * q;
          if (c0 < ldc)
            atomicAdd(reinterpret_cast<float4*>(dst + c0), make_float4(vals[4 * q], vals[4 * q + 1],
                                                                       vals[4 * q + 2], vals[4 * q + 3]));
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, ncols);
}

// src_lo (optional): a second TF32 term of the densities (src + src_lo ~= the
// FP32 value); each step then issues the MMAs of both terms into the same
// accumulator, so the densities carry ~21 bits instead of TF32's 11.
__global__ void __launch_bounds__(128, 1)
    m2l_img_kernel(const M2LUnit* __restrict__ units, const int* __restrict__ tile_nodes,
                    const int* __restrict__ tile_slot0, const int* __restrict__ slot_op,
                    const int* __restrict__ slot_src, const float* __restrict__ images,
                    const float* __restrict__ src, float* __restrict__ check, int ldc, int NP, int* err,
                    const float* __restrict__ src_lo, int ns) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  uint8_t* sbase = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  const uint32_t A_BYTES = kTileRows * 128, B_BYTES = (uint32_t)NP * 128;
  const int na = src_lo ? 2 : 1;  // A terms per stage
  uint8_t* sA0 = sbase;           // stage st, term q at sA0 + (st * na + q) * A_BYTES
  uint8_t* sB0 = sbase + ns * na * A_BYTES;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sB0 + ns * B_BYTES);  // full[ns] done[ns] acc
  uint64_t* full = bars;
  uint64_t* done = bars + ns;
  uint64_t* accb = bars + 2 * ns;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * ns + 1);
  volatile int* abort_s = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5;
  const M2LUnit u = units[blockIdx.x];
  const int nchunks = NP / 32;
  const int nhalves = NP > 256 ? 2 : 1;
  const int nh = NP / nhalves;
  const uint32_t ncols = NP > 256 ? 512u : 256u;
  const uint32_t idesc = tf32_idesc(nh);

  if (tid == 0) {
    for (int k = 0; k < 2 * ns + 1; ++k) mbar_init(&bars[k], 1);
    *abort_s = 0;
    fence_barrier_init();
  }
  if (warp == 0) tmem_alloc(tmem_slot, ncols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int node = tile_nodes[u.tile * kTileRows + tid];
  const int slot_base = tile_slot0[u.tile] + u.slot0;
  const int nsteps = u.nslot * nchunks;
  int issued = 0;  // MMA steps committed
  int copies = 0;  // B copies issued
  // Step s uses stage s % ns (its k-th use completes phase k of full[] and
  // done[], parity (s / ns) & 1): thread 0 bulk-copies the operator chunk
  // into B, every thread gathers its own A row (32 TF32 of its source node's
  // density, per term).
  auto prepare = [&](int s) {
    const int st = s % ns;
    const int slot = slot_base + s / nchunks;
    const int c = s % nchunks;
    if (tid == 0) {
      mbar_expect_tx(&full[st], B_BYTES);
      const float* gB = images + (size_t)slot_op[slot] * ((size_t)nchunks * NP * 32) + (size_t)c * NP * 32;
      bulk_g2s(sB0 + st * B_BYTES, gB, B_BYTES, &full[st]);
      ++copies;
    }
    const int v = slot_src[(size_t)slot * kTileRows + tid];
    for (int q = 0; q < na; ++q) {
      float4* dA = reinterpret_cast<float4*>(sA0 + (st * na + q) * A_BYTES + tid * 128);
      if (v >= 0) {
        const float4* g4 = reinterpret_cast<const float4*>((q ? src_lo : src) + (size_t)v * NP + c * 32);
#pragma unroll
        for (int j = 0; j < 8; ++j) dA[j ^ (tid & 7)] = __ldg(g4 + j);
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) dA[j] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
    fence_proxy_async();
  };
  for (int i = 0; i < ns - 1 && i < nsteps; ++i) prepare(i);
  __syncthreads();
  for (int s = 0; s < nsteps; ++s) {
    const int st = s % ns;
    if (tid == 0 && !*abort_s) {
      if (!mbar_wait(&full[st], (s / ns) & 1)) {
        *abort_s = 1;
        atomicOr(err, 2);
      } else {
        tc_fence_after();
        const uint32_t b0 = smem_u32(sB0 + st * B_BYTES);
#pragma unroll
        for (int k8 = 0; k8 < 4; ++k8)
          for (int q = 0; q < na; ++q) {
            const uint32_t a0 = smem_u32(sA0 + (st * na + q) * A_BYTES);
            for (int h = 0; h < nhalves; ++h)
              umma_tf32(tmem + (uint32_t)(h * nh), sw128_desc(a0 + k8 * 32), sw128_desc(b0 + h * nh * 128 + k8 * 32),
                        idesc, (s > 0 || k8 > 0 || q > 0) ? 1u : 0u);
          }
        umma_commit(&done[st]);
        ++issued;
      }
    }
    // while the MMAs of steps s (and s-1..) run, fill stage (s-1) % ns with
    // step s+ns-1 once the MMAs of step s-1, its previous user, are done
    const int nxt = s + ns - 1;
    if (nxt < nsteps) {
      if (s >= 1 && !mbar_wait(&done[(s - 1) % ns], ((s - 1) / ns) & 1)) {
        *abort_s = 1;
        atomicOr(err, 1);
      }
      if (!*abort_s) prepare(nxt);
    }
    __syncthreads();
    if (*abort_s) break;
  }
  __syncthreads();
  // drain: every MMA this thread issued completes before acc (commit tracks all)
  if (tid == 0) umma_commit(accb);
  const bool acc_ok = __all_sync(0xffffffffu, mbar_wait(accb, 0));
  if (!acc_ok && (tid & 31) == 0) atomicOr(err, 4);
  // B copies issued for steps whose MMAs never ran must land before exit
  if (tid == 0)
    for (int s = issued; s < copies; ++s)
      if (!mbar_wait(&full[s % ns], (s / ns) & 1)) atomicOr(err, 8);
  tc_fence_after();
  if (!*abort_s && acc_ok && nsteps > 0) {
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
    for (int col = 0; col < NP; col += 16) {
      float vals[16];
      tmem_ld16(lane_addr + col, vals);
      if (node >= 0) {
        float* dst = check + (size_t)node * ldc;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int c0 = col + 4 * q;
          if (c0 < ldc)
            atomicAdd(reinterpret_cast<float4*>(dst + c0), make_float4(vals[4 * q], vals[4 * q + 1],
                                                                       vals[4 * q + 2], vals[4 * q + 3]));
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, ncols);
}

// Warp-specialised form of m2l_img_kernel for the compressed operators
// (NP = RC <= 256, two density terms), 288 threads:
//   warp 0, lane 0: bulk-copies operator chunks up to ns steps ahead and
//                   issues the MMAs of each step once its stage is full;
//   warps 1-8:      warp 1 + 4q + i gathers rows 32 i .. 32 i + 31 of term q
//                   of every step into its stage as soon as the MMAs of the
//                   stage's previous use are done, then arrives on the
//                   stage's barrier.
// full[st] completes when the 8 gather warps have arrived and the copy has
// landed (count 9: 8 arrivals + the producer's expect_tx arrival); done[st]
// when the stage's MMAs are done (tcgen05.commit).  Warps 1-4 read the
// accumulator back (warp w reads TMEM lanes 32 (w % 4) ..).  Every wait is
// bounded; a timeout sets err and the roles drain and exit.
constexpr int kWsGatherWarps = 8;
__global__ void __launch_bounds__(32 * (1 + kWsGatherWarps), 1)
    m2l_ws_kernel(const M2LUnit* __restrict__ units, const int* __restrict__ tile_nodes,
                   const int* __restrict__ tile_slot0, const int* __restrict__ slot_op,
                   const int* __restrict__ slot_src, const float* __restrict__ images,
                   const float* __restrict__ src, const float* __restrict__ src_lo, float* __restrict__ out,
                   int ldc, int NP, int* err, int ns, uint32_t wlim, int probe, float* __restrict__ part) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  uint8_t* sbase = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  const uint32_t A_BYTES = kTileRows * 128, B_BYTES = (uint32_t)NP * 128;
  uint8_t* sA0 = sbase;  // stage st, term q at sA0 + (2 st + q) A_BYTES
  uint8_t* sB0 = sbase + ns * 2 * A_BYTES;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sB0 + ns * B_BYTES);
  uint64_t* full = bars;
  uint64_t* done = bars + ns;
  uint64_t* accb = bars + 2 * ns;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * ns + 1);
  volatile int* abort_s = reinterpret_cast<volatile int*>(tmem_slot + 1);
  uint64_t* probe_bar = bars + 2 * ns + 2;  // failure-path test only: nothing arrives here

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const M2LUnit u = units[blockIdx.x];
  const int nchunks = NP / 32;
  const uint32_t idesc = tf32_idesc(NP);
  if (tid == 0) {
    for (int k = 0; k < ns; ++k) {
      mbar_init(&full[k], 1 + kWsGatherWarps);
      mbar_init(&done[k], 1);
    }
    mbar_init(accb, 1);
    mbar_init(probe_bar, 1);
    *abort_s = 0;
    fence_barrier_init();
  }
  if (warp == 0) tmem_alloc(tmem_slot, 256);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  if (probe) {
    // every thread waits on a barrier that no thread or copy completes; the
    // bounded wait gives up before any copy or MMA is issued
    if (!mbar_wait(probe_bar, 0, wlim)) {
      *abort_s = 1;
      if (tid == 0) atomicOr(err, 32);
    }
    __syncthreads();
  }
  const int slot_base = tile_slot0[u.tile] + u.slot0;
  const int nsteps = u.nslot * nchunks;
  int issued = 0, copies = 0;  // lane 0 of warp 0
  if (warp == 0) {
    if (lane == 0) {
      auto copy = [&](int s) {
        const int st = s % ns;
        const int slot = slot_base + s / nchunks, c = s % nchunks;
        mbar_expect_tx(&full[st], B_BYTES);
        const float* gB = images + (size_t)slot_op[slot] * ((size_t)nchunks * NP * 32) + (size_t)c * NP * 32;
        bulk_g2s(sB0 + st * B_BYTES, gB, B_BYTES, &full[st]);
        ++copies;
      };
      for (int s = 0; s < ns && s < nsteps && !*abort_s; ++s) copy(s);
      for (int s = 0; s < nsteps && !*abort_s; ++s) {
        const int st = s % ns;
        if (!mbar_wait(&full[st], (s / ns) & 1, wlim)) {
          *abort_s = 1;
          atomicOr(err, 2);
          break;
        }
        tc_fence_after();
        const uint32_t b0 = smem_u32(sB0 + st * B_BYTES);
#pragma unroll
        for (int k8 = 0; k8 < 4; ++k8)
#pragma unroll
          for (int q = 0; q < 2; ++q)
            umma_tf32(tmem, sw128_desc(smem_u32(sA0 + (2 * st + q) * A_BYTES) + k8 * 32), sw128_desc(b0 + k8 * 32),
                      idesc, (s > 0 || k8 > 0 || q > 0) ? 1u : 0u);
        umma_commit(&done[st]);
        ++issued;
        // refill the stage of step s-1 with step s-1+ns once its MMAs are done
        const int prev = s - 1, nxt = s - 1 + ns;
        if (prev >= 0 && nxt < nsteps) {
          if (!mbar_wait(&done[prev % ns], (prev / ns) & 1, wlim)) {
            *abort_s = 1;
            atomicOr(err, 1);
            break;
          }
          copy(nxt);
        }
      }
      umma_commit(accb);  // tracks every MMA issued above
    }
    __syncwarp();
  } else {
    const int g = warp - 1, q = g / 4;  // term
    const int r = 32 * (g % 4) + lane;  // A row
    const float* __restrict__ term = q ? src_lo : src;
    for (int s = 0; s < nsteps && !*abort_s; ++s) {
      const int st = s % ns, use = s / ns;
      if (use >= 1 && !mbar_wait(&done[st], (use - 1) & 1, wlim)) {
        *abort_s = 1;
        atomicOr(err, 16);
        break;
      }
      const int slot = slot_base + s / nchunks, c = s % nchunks;
      const int v = slot_src[(size_t)slot * kTileRows + r];
      float4* dA = reinterpret_cast<float4*>(sA0 + (2 * st + q) * A_BYTES + r * 128);
      if (v >= 0) {
        const float4* g4 = reinterpret_cast<const float4*>(term + (size_t)v * NP + c * 32);
        float4 t[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) t[j] = __ldg(g4 + j);
#pragma unroll
        for (int j = 0; j < 8; ++j) dA[j ^ (r & 7)] = t[j];
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) dA[j] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
      fence_proxy_async();
      __syncwarp();
      if (lane == 0) mbar_arrive(&full[st]);
    }
  }
  // every role waits for the accumulator (committed after the last MMA); the
  // read-back below is warp-collective, so a warp reads only if all its lanes
  // saw the accumulator complete
  const bool acc_ok = __all_sync(0xffffffffu, mbar_wait(accb, 0, wlim));
  if (!acc_ok && lane == 0) atomicOr(err, 4);
  // operator copies issued for steps whose MMAs never ran land before exit
  if (tid == 0)
    for (int s = issued; s < copies; ++s)
      if (!mbar_wait(&full[s % ns], (s / ns) & 1, wlim)) atomicOr(err, 8);
  tc_fence_after();
  if (warp >= 1 && warp <= 4 && !*abort_s && acc_ok && nsteps > 0) {
    const int q4 = warp & 3;  // TMEM lane quarter of this warp
    const int row = 32 * q4 + lane;
    const int node = tile_nodes[u.tile * kTileRows + row];
    const uint32_t lane_addr = tmem + ((uint32_t)(32 * q4) << 16);
    for (int col = 0; col < NP; col += 16) {
      float vals[16];
      tmem_ld16(lane_addr + col, vals);
      if (node >= 0) {
        if (part) {  // this unit's own block; the tile's blocks are added in order afterwards
          float4* dst = reinterpret_cast<float4*>(part + ((size_t)blockIdx.x * kTileRows + row) * NP + col);
#pragma unroll
          for (int q = 0; q < 4; ++q)
            dst[q] = make_float4(vals[4 * q], vals[4 * q + 1], vals[4 * q + 2], vals[4 * q + 3]);
          continue;
        }
        float* dst = out + (size_t)node * ldc;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int c0 = col + 4 * q;
          if (c0 < ldc)
            atomicAdd(reinterpret_cast<float4*>(dst + c0), make_float4(vals[4 * q], vals[4 * q + 1],
                                                                       vals[4 * q + 2], vals[4 * q + 3]));
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 256);
}

// out[node] = sum over the tile's units, in unit order, of their partial
// blocks (rows of empty tile slots are skipped).  One block per tile.
__global__ void __launch_bounds__(256) m2l_unit_reduce_kernel(const int* __restrict__ tile_uoff,
                                                              const int* __restrict__ tile_units,
                                                              const int* __restrict__ tile_nodes,
                                                              const float* __restrict__ part, int NP,
                                                              float* __restrict__ out, int ldc) {
  const int t = blockIdx.x;
  const int u0 = tile_uoff[t], u1 = tile_uoff[t + 1];
  const int n4 = NP / 4;
  const float4* p4 = reinterpret_cast<const float4*>(part);
  for (int idx = threadIdx.x; idx < kTileRows * n4; idx += blockDim.x) {
    const int r = idx / n4, c4 = idx - r * n4;
    const int node = tile_nodes[t * kTileRows + r];
    if (node < 0) continue;
    float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int k = u0; k < u1; ++k) {
      const float4 v = p4[((size_t)tile_units[k] * kTileRows + r) * n4 + c4];
      s.x += v.x;
      s.y += v.y;
      s.z += v.z;
      s.w += v.w;
    }
    reinterpret_cast<float4*>(out + (size_t)node * ldc)[c4] = s;
  }
}

// T_{L,o}[n = 3a+al][k = 3b+be] = S_al,be(x_a - y_b) / (8 pi mu),
// x_a = lattice_a * h, y_b = lattice_b * h + o * w, h = w/(res-1), rounded to
// TF32 and written at its SW128 K-major position of chunk k/32.
__global__ void m2l_operator_kernel(int nimg, const int* __restrict__ img_code, const double* __restrict__ img_w,
                                    const int* __restrict__ lat, int P, int res, double eps, double mu, int NP,
                                    float* __restrict__ images) {
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long per = (long long)P * P;
  if (gid >= per * nimg) return;
  const int img = (int)(gid / per);
  const int a = (int)((gid % per) / P), b = (int)(gid % P);
  const int code = img_code[img];
  const int ox = code / 49 - 3, oy = (code / 7) % 7 - 3, oz = code % 7 - 3;
  const double w = img_w[img], h = w / (res - 1);
  const double r[3] = {(lat[3 * a] - lat[3 * b]) * h - ox * w, (lat[3 * a + 1] - lat[3 * b + 1]) * h - oy * w,
                       (lat[3 * a + 2] - lat[3 * b + 2]) * h - oz * w};
  const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
  const double e2 = eps * eps;
  const double inv = 1.0 / (8.0 * M_PI * mu * (r2 + e2) * sqrt(r2 + e2));
  uint8_t* base = reinterpret_cast<uint8_t*>(images) + (size_t)img * ((size_t)NP / 32) * NP * 128;
  for (int al = 0; al < 3; ++al)
    for (int be = 0; be < 3; ++be) {
      const double val = (r[al] * r[be] + (al == be ? r2 + 2 * e2 : 0.0)) * inv;
      const int n = 3 * a + al, k = 3 * b + be;
      const int c = k >> 5, kl = k & 31, j = kl >> 2, e = kl & 3;
      float* dst = reinterpret_cast<float*>(base + (size_t)c * NP * 128 + (size_t)n * 128 + ((j ^ (n & 7)) << 4) +
                                            e * 4);
      *dst = to_tf32((float)val);
    }
}

// T_o in FP64 for the offsets codes[i] at box width w: column-major 3P x 3P,
// T[n = 3a+al][k = 3b+be] = S_al,be(x_a - y_b) at k * 3P + n (the matrix of
// m2l_operator_kernel before rounding).
__global__ void m2l_full_operator_kernel(int ncodes, const int* __restrict__ codes, double w,
                                         const int* __restrict__ lat, int P, int res, double eps, double mu,
                                         double* __restrict__ K) {
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long per = (long long)P * P;
  if (gid >= per * ncodes) return;
  const int img = (int)(gid / per);
  const int a = (int)((gid % per) / P), b = (int)(gid % P);
  const int code = codes[img];
  const int ox = code / 49 - 3, oy = (code / 7) % 7 - 3, oz = code % 7 - 3;
  const double h = w / (res - 1);
  const double r[3] = {(lat[3 * a] - lat[3 * b]) * h - ox * w, (lat[3 * a + 1] - lat[3 * b + 1]) * h - oy * w,
                       (lat[3 * a + 2] - lat[3 * b + 2]) * h - oz * w};
  const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
  const double e2 = eps * eps;
  const double inv = 1.0 / (8.0 * M_PI * mu * (r2 + e2) * sqrt(r2 + e2));
  const int n3 = 3 * P;
  double* base = K + (size_t)img * n3 * n3;
  for (int al = 0; al < 3; ++al)
    for (int be = 0; be < 3; ++be)
      base[(size_t)(3 * b + be) * n3 + 3 * a + al] = (r[al] * r[be] + (al == be ? r2 + 2 * e2 : 0.0)) * inv;
}

// Compressed operator images: C (RC x RC, column-major per image, FP64) to
// the TF32 SW128 K-major chunks the image kernel streams (NP = RC).
__global__ void compressed_image_kernel(int nimg, const int* __restrict__ src_of, const double* __restrict__ C,
                                        int RC, float* __restrict__ images) {
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long per = (long long)RC * RC;
  if (gid >= per * nimg) return;
  const int img = (int)(gid / per);
  const int k = (int)((gid % per) / RC), n = (int)(gid % RC);
  const double v = C[(size_t)src_of[img] * per + (size_t)k * RC + n];
  const int c = k >> 5, kl = k & 31, j = kl >> 2, e = kl & 3;
  uint8_t* base = reinterpret_cast<uint8_t*>(images) + (size_t)img * per * sizeof(float);
  *reinterpret_cast<float*>(base + (size_t)c * RC * 128 + (size_t)n * 128 + ((j ^ (n & 7)) << 4) + e * 4) =
      to_tf32((float)v);
}

// The basis in FP32, row-major 3P x RC, from its FP64 column-major form.
__global__ void basis_float_kernel(const double* __restrict__ Bd, int n3, int RC, float* __restrict__ B) {
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= n3 * RC) return;
  const int row = gid / RC, j = gid % RC;
  B[gid] = (float)Bd[(size_t)j * n3 + row];
}

// y[node * ldy + r] = sum_k A(r, k) x[node * ldx + k] for the nodes of each
// tile, A the tile's basis B (3P x RC, row-major):
//   trans = 1 (projection u^ = B^T u): A(r, k) = B[k][r], r < RC, k < 3P,
//              y written as two TF32 terms (the tensor-core operands):
//              y = tf32(v), y_lo = tf32(v - y);
//   trans = 0 (expansion check += B c^): A(r, k) = B[r][k], r < 3P, k < RC,
//              y accumulated.
// 64 x 64 output tile (rows x nodes) per CTA of 256 threads, 4 x 4 each
// (rows 4 tr .. 4 tr + 3, nodes 4 tc .. 4 tc + 3, both read from shared memory
// as one float4), K in steps of 16, FP32.
__global__ void __launch_bounds__(256) basis_apply_kernel(const float* __restrict__ basis, int n3, int RC,
                                                          int trans, const BasisTile* __restrict__ tiles,
                                                          const int* __restrict__ nodes,
                                                          const float* __restrict__ x, long long ldx,
                                                          float* __restrict__ y, long long ldy,
                                                          float* __restrict__ y_lo = nullptr) {
  constexpr int BM = 64, BN = 64, BK = 16;
  __shared__ __align__(16) float As[BK][BM + 4];
  __shared__ __align__(16) float Xs[BK][BN + 4];
  __shared__ int col_node[BN];
  const BasisTile tl = tiles[blockIdx.y];
  const int rows = trans ? RC : n3, K = trans ? n3 : RC;
  const int m0 = blockIdx.x * BM;
  const float* __restrict__ B = basis + (size_t)tl.basis * n3 * RC;
  const int tid = threadIdx.x;
  if (tid < BN) col_node[tid] = tid < tl.count ? nodes[tl.first + tid] : -1;
  const int tr = tid % 16, tc = tid / 16;
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
  for (int k0 = 0; k0 < K; k0 += BK) {
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + 256 * q;  // BK * BM
      int kk, mm;
      if (trans) { mm = e % BM; kk = e / BM; }  // B[k][r]: contiguous in r
      else { kk = e % BK; mm = e / BK; }        // B[r][k]: contiguous in k
      const int r = m0 + mm, k = k0 + kk;
      As[kk][mm] = (r < rows && k < K) ? (trans ? B[(size_t)k * RC + r] : B[(size_t)r * RC + k]) : 0.f;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + 256 * q;  // BK * BN
      const int kk = e % BK, nn = e / BK;
      const int k = k0 + kk, node = col_node[nn];
      Xs[kk][nn] = (k < K && node >= 0) ? x[(size_t)node * ldx + k] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      const float4 a4 = *reinterpret_cast<const float4*>(&As[kk][4 * tr]);
      const float4 b4 = *reinterpret_cast<const float4*>(&Xs[kk][4 * tc]);
      const float a[4] = {a4.x, a4.y, a4.z, a4.w}, b[4] = {b4.x, b4.y, b4.z, b4.w};
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int r = m0 + 4 * tr + i, node = col_node[4 * tc + j];
      if (r >= rows || node < 0) continue;
      float* o = y + (size_t)node * ldy + r;
      if (trans) {
        const float hi = to_tf32(acc[i][j]);
        *o = hi;
        y_lo[(size_t)node * ldy + r] = to_tf32(acc[i][j] - hi);
      } else {
        *o += acc[i][j];
      }
    }
}

// Compression of the operators of one level pass (see m2l.h).  Builds the
// FP64 operators of all 316 far offsets, the eigenvectors of sum_o T_o T_o^T,
// and C_o = B^T T_o B for every offset; returns B (FP32) and C in FP64.
struct Compressor {
  cublasHandle_t b = nullptr;
  cusolverDnHandle_t s = nullptr;
  int n3 = 0, RC = 0, P = 0, res = 0;
  std::vector<int> far_codes;
  DBuf<int> dcodes, dlat;
  DBuf<double> K, G, W, T, C, work, H, Br;
  DBuf<int> info;
  int lwork = 0;
  Compressor(const std::vector<int>& lat, int P_, int res_, int RC_, cudaStream_t st) : n3(3 * P_), RC(RC_), P(P_), res(res_) {
    if (cublasCreate(&b) != CUBLAS_STATUS_SUCCESS) throw Error(NNK_E_CUDA, "cublasCreate failed");
    cublasSetStream(b, st);
    if (cusolverDnCreate(&s) != CUSOLVER_STATUS_SUCCESS) throw Error(NNK_E_CUDA, "cusolverDnCreate failed");
    cusolverDnSetStream(s, st);
    cudaGetLastError();
    for (int c = 0; c < 343; ++c) {
      const int ox = c / 49 - 3, oy = (c / 7) % 7 - 3, oz = c % 7 - 3;
      if (std::max(std::abs(ox), std::max(std::abs(oy), std::abs(oz))) >= 2) far_codes.push_back(c);
    }
    dcodes.upload(far_codes, st);
    dlat.upload(lat, st);
    const size_t nc = far_codes.size();
    K.alloc(nc * n3 * n3);
    G.alloc((size_t)n3 * n3);
    W.alloc(n3);
    T.alloc(nc * n3 * RC);
    C.alloc(nc * RC * RC);
    info.alloc(1);
    // normalized Sylvester-Hadamard matrix (RC a power of two): rotating the
    // basis by it spreads every vector's energy over all RC coordinates, so
    // the TF32 rounding errors of the compressed products average out as
    // they do over the 3P physical coordinates
    if (RC & (RC - 1)) throw Error(NNK_E_ARG, "compressed M2L rank must be a power of two");
    std::vector<double> h((size_t)RC * RC);
    const double sc = 1.0 / std::sqrt((double)RC);
    for (int i = 0; i < RC; ++i)
      for (int j = 0; j < RC; ++j) h[(size_t)j * RC + i] = (__builtin_popcount(i & j) & 1) ? -sc : sc;
    H.upload(h, st);
    Br.alloc((size_t)n3 * RC);
    if (cusolverDnDsyevd_bufferSize(s, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n3, G.p, n3, W.p, &lwork) !=
        CUSOLVER_STATUS_SUCCESS)
      throw Error(NNK_E_CUDA, "syevd_bufferSize failed");
    work.alloc(std::max(lwork, 1));
  }
  ~Compressor() {
    if (s) cusolverDnDestroy(s);
    if (b) cublasDestroy(b);
  }
  int far_index(int code) const {
    return (int)(std::lower_bound(far_codes.begin(), far_codes.end(), code) - far_codes.begin());
  }
  // basis (3P x RC FP32 row-major) into B_out; C (per far offset) in this->C
  void run(double w, double eps, double mu, float* B_out, cudaStream_t st) {
    const int nc = (int)far_codes.size();
    const long long total = (long long)P * P * nc;
    m2l_full_operator_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(nc, dcodes.p, w, dlat.p, P, res, eps,
                                                                             mu, K.p);
    NNK_CHECK_LAUNCH();
    const double one = 1.0, zero = 0.0;
    // G = [T_1 ... T_nc] [T_1 ... T_nc]^T
    if (cublasDgemm(b, CUBLAS_OP_N, CUBLAS_OP_T, n3, n3, n3 * nc, &one, K.p, n3, K.p, n3, &zero, G.p, n3) !=
        CUBLAS_STATUS_SUCCESS)
      throw Error(NNK_E_CUDA, "M2L Gram product failed");
    if (cusolverDnDsyevd(s, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n3, G.p, n3, W.p, work.p, lwork,
                         info.p) != CUSOLVER_STATUS_SUCCESS)
      throw Error(NNK_E_CUDA, "M2L basis eigendecomposition failed");
    int h_info = 0;
    NNK_CUDA(cudaMemcpyAsync(&h_info, info.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    NNK_CUDA(cudaStreamSynchronize(st));
    if (h_info != 0) throw Error(NNK_E_CUDA, "M2L basis eigendecomposition info=" + std::to_string(h_info));
    // B = (leading RC eigenvectors) x H, n3 x RC column-major
    if (cublasDgemm(b, CUBLAS_OP_N, CUBLAS_OP_N, n3, RC, RC, &one, G.p + (size_t)(n3 - RC) * n3, n3, H.p, RC, &zero,
                    Br.p, n3) != CUBLAS_STATUS_SUCCESS)
      throw Error(NNK_E_CUDA, "M2L basis rotation failed");
    const double* Bd = Br.p;
    // T_o B, then C_o = B^T (T_o B)
    if (cublasDgemmStridedBatched(b, CUBLAS_OP_N, CUBLAS_OP_N, n3, RC, n3, &one, K.p, n3, (long long)n3 * n3, Bd, n3,
                                  0, &zero, T.p, n3, (long long)n3 * RC, nc) != CUBLAS_STATUS_SUCCESS ||
        cublasDgemmStridedBatched(b, CUBLAS_OP_T, CUBLAS_OP_N, RC, RC, n3, &one, Bd, n3, 0, T.p, n3,
                                  (long long)n3 * RC, &zero, C.p, RC, (long long)RC * RC, nc) != CUBLAS_STATUS_SUCCESS)
      throw Error(NNK_E_CUDA, "M2L compressed operator products failed");
    basis_float_kernel<<<(n3 * RC + 255) / 256, 256, 0, st>>>(Br.p, n3, RC, B_out);
    NNK_CHECK_LAUNCH();
  }
};

}  // namespace

M2LPlan::~M2LPlan() {
  if (h_err) cudaFreeHost(h_err);
  if (err_ev) cudaEventDestroy(err_ev);
}

void build_m2l_plan(const HostTree& t, int res, int shells, double eps, double mu, M2LPlan& plan,
                    cudaStream_t st) {
  // surface lattice (same order as the unified surface points)
  std::vector<int> lat;
  auto inner = [&](int a) { return a >= shells && a <= res - 1 - shells; };
  for (int k = 0; k < res; ++k)
    for (int i = 0; i < res; ++i)
      for (int j = 0; j < res; ++j)
        if (!(inner(j) && inner(i) && inner(k))) {
          lat.push_back(i);
          lat.push_back(j);
          lat.push_back(k);
        }
  const int P = (int)lat.size() / 3;
  int NP = ((3 * P + 31) / 32) * 32;
  if (NP > 512 || NP / (NP > 256 ? 2 : 1) % 16 != 0)
    throw Error(NNK_E_ARG, "tensor-core M2L supports 3P up to 512 with N halves a multiple of 16");
  plan.n3 = 3 * P;
  plan.compressed = plan.compress && 3 * P > plan.RC && plan.image_budget > 0;
  if (plan.compressed) NP = plan.RC;
  plan.NP = NP;
  struct Pass {
    double w;
    std::vector<int32_t> nodes;  // V targets and V sources, ascending
  };
  std::vector<Pass> passes;
  std::vector<int> img_pass;  // per image: its pass
  std::vector<int> tile_nodes, tile_slot0, slot_code, slot_src, slot_op;
  std::vector<float> slot_h;
  std::vector<M2LUnit> units;
  std::vector<int> img_code;      // per operator image: offset code
  std::vector<double> img_w;      // per operator image: box width of its level
  int64_t useful = 0, tslots = 0;
  // one pass per (level, tree of the forest): the operators depend on the
  // box width, which differs between trees
  for (int L = 1; L <= t.max_level; ++L)
  for (int g = 0; g < t.groups(); ++g) {
    const double* root = &t.corners[6 * (size_t)t.root_of(g)];
    const double W0 = root[3] - root[0];
    std::vector<int32_t> nodes;
    for (int32_t n : t.by_level[L])
      if (t.group_of(n) == g && t.V.off[n + 1] > t.V.off[n]) nodes.push_back(n);
    if (nodes.empty()) continue;
    auto oct = [&](int32_t n) { return ((t.ix[n] & 1) << 2) | ((t.iy[n] & 1) << 1) | (t.iz[n] & 1); };
    // signature: octant, then the bitset of V offsets (343 codes), so that
    // nodes using the same offsets share tiles and padding rows stay few
    std::map<int32_t, std::array<uint64_t, 7>> sig;
    for (int32_t n : nodes) {
      std::array<uint64_t, 7> b{};
      b[0] = (uint64_t)oct(n) << 60;
      for (int64_t k = t.V.off[n]; k < t.V.off[n + 1]; ++k) {
        const int32_t v = t.V.idx[k];
        const int code = (t.ix[v] - t.ix[n] + 3) * 49 + (t.iy[v] - t.iy[n] + 3) * 7 + (t.iz[v] - t.iz[n] + 3);
        if (code >= 0 && code < 343) b[1 + code / 64] |= 1ull << (code % 64);
      }
      sig[n] = b;
    }
    std::stable_sort(nodes.begin(), nodes.end(), [&](int32_t a, int32_t b) { return sig[a] > sig[b]; });
    {
      Pass ps{std::ldexp(W0, -L), {}};
      for (int32_t n : nodes) {
        ps.nodes.push_back(n);
        for (int64_t k = t.V.off[n]; k < t.V.off[n + 1]; ++k) ps.nodes.push_back(t.V.idx[k]);
      }
      std::sort(ps.nodes.begin(), ps.nodes.end());
      ps.nodes.erase(std::unique(ps.nodes.begin(), ps.nodes.end()), ps.nodes.end());
      passes.push_back(std::move(ps));
    }
    std::map<int, int> img_of;  // offset code -> image of this level
    const int first_tile = (int)tile_slot0.size();
    std::vector<std::vector<int>> tile_codes;  // per tile in this level: its offset codes, ascending
    for (size_t t0 = 0; t0 < nodes.size(); t0 += kTileRows) {
      const int tile = (int)tile_slot0.size();
      const int rows = (int)std::min<size_t>(kTileRows, nodes.size() - t0);
      std::map<int, std::vector<int>> by_code;  // code -> 128 sources
      for (int r = 0; r < rows; ++r) {
        const int32_t i = nodes[t0 + r];
        for (int64_t k = t.V.off[i]; k < t.V.off[i + 1]; ++k) {
          const int32_t v = t.V.idx[k];
          const int ox = t.ix[v] - t.ix[i], oy = t.iy[v] - t.iy[i], oz = t.iz[v] - t.iz[i];
          if (std::abs(ox) > 3 || std::abs(oy) > 3 || std::abs(oz) > 3)
            throw Error(NNK_E_STATE, "V-list offset outside [-3,3]^3");
          const int code = (ox + 3) * 49 + (oy + 3) * 7 + (oz + 3);
          auto& vec = by_code[code];
          if (vec.empty()) vec.assign(kTileRows, -1);
          vec[r] = v;
          ++useful;
        }
      }
      tile_slot0.push_back((int)slot_code.size());
      for (int r = 0; r < kTileRows; ++r) tile_nodes.push_back(r < rows ? nodes[t0 + r] : -1);
      std::vector<int> codes;
      for (auto& kv : by_code) {
        auto it = img_of.find(kv.first);
        if (it == img_of.end()) {
          it = img_of.emplace(kv.first, (int)img_code.size()).first;
          img_code.push_back(kv.first);
          img_w.push_back(std::ldexp(W0, -L));
          img_pass.push_back((int)passes.size() - 1);
        }
        slot_op.push_back(it->second);
        slot_code.push_back(kv.first);
        slot_h.push_back((float)(std::ldexp(W0, -L) / (res - 1)));
        slot_src.insert(slot_src.end(), kv.second.begin(), kv.second.end());
        codes.push_back(kv.first);
      }
      tslots += (int64_t)codes.size();
      (void)tile;
      tile_codes.push_back(codes);
    }
    // Work units cut the (code-sorted) slot list of every tile at fixed code
    // boundaries and run range by range over all tiles of the level, so the
    // CTAs resident at one time read the same operator images (L2 reuse).
    for (int c0 = 0; c0 < 343; c0 += kCodesPerUnit) {
      for (size_t ti = 0; ti < tile_codes.size(); ++ti) {
        const auto& codes = tile_codes[ti];
        const int lo = (int)(std::lower_bound(codes.begin(), codes.end(), c0) - codes.begin());
        const int hi = (int)(std::lower_bound(codes.begin(), codes.end(), c0 + kCodesPerUnit) - codes.begin());
        if (hi > lo) units.push_back(M2LUnit{first_tile + (int)ti, lo, hi - lo, 0});
      }
    }
  }
  plan.ntiles = (int)tile_slot0.size();
  plan.nunits = (int)units.size();
  {
    std::vector<int> uoff(plan.ntiles + 1, 0), tu(units.size());
    for (const M2LUnit& u : units) uoff[u.tile + 1]++;
    for (int t2 = 0; t2 < plan.ntiles; ++t2) uoff[t2 + 1] += uoff[t2];
    std::vector<int> at(uoff.begin(), uoff.end() - 1);
    for (size_t k = 0; k < units.size(); ++k) tu[at[units[k].tile]++] = (int)k;
    plan.tile_uoff.upload(uoff, st);
    plan.tile_units.upload(tu, st);
  }
  plan.useful_pairs = useful;
  plan.tile_slots = tslots;
  plan.tile_nodes.upload(tile_nodes, st);
  plan.tile_slot0.upload(tile_slot0, st);
  plan.slot_code.upload(slot_code, st);
  plan.slot_h.upload(slot_h, st);
  plan.slot_src.upload(slot_src, st);
  plan.units.upload(units, st);
  std::vector<int> packed(P);
  for (int p = 0; p < P; ++p) packed[p] = lat[3 * p] | (lat[3 * p + 1] << 4) | (lat[3 * p + 2] << 8);
  plan.lat.upload(packed, st);
  // Operator images (one NP x NP TF32 matrix per level and offset, streamed
  // by the image kernel) when they fit the budget; otherwise the generating
  // kernel computes each chunk in shared memory.
  const size_t img_bytes = img_code.size() * (size_t)NP * NP * sizeof(float);
  plan.use_images = plan.compressed || img_bytes <= plan.image_budget;
  plan.image_bytes = plan.use_images ? img_bytes : 0;
  if (plan.compressed && !img_code.empty()) {
    // per pass: basis B and the compressed images of the offsets it uses
    const int RC = plan.RC, n3 = 3 * P;
    plan.slot_op.upload(slot_op, st);
    plan.images.alloc(img_code.size() * (size_t)RC * RC);
    plan.basis.alloc(passes.size() * (size_t)n3 * RC);
    Compressor cmp(lat, P, res, RC, st);
    std::vector<BasisTile> bt;
    std::vector<int> bn;
    DBuf<int> dsrc;
    for (size_t ps = 0; ps < passes.size(); ++ps) {
      cmp.run(passes[ps].w, eps, mu, plan.basis.p + ps * (size_t)n3 * RC, st);
      std::vector<int> imgs, src_of;
      for (size_t i = 0; i < img_code.size(); ++i)
        if (img_pass[i] == (int)ps) {
          imgs.push_back((int)i);
          src_of.push_back(cmp.far_index(img_code[i]));
        }
      // images of a pass are consecutive (appended while its tiles were built)
      if (imgs.empty() || imgs.back() != imgs.front() + (int)imgs.size() - 1)
        throw Error(NNK_E_STATE, "M2L images of a level pass are not consecutive");
      dsrc.upload(src_of, st);
      const long long total = (long long)RC * RC * (long long)imgs.size();
      compressed_image_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(
          (int)imgs.size(), dsrc.p, cmp.C.p, RC, plan.images.p + (size_t)imgs[0] * RC * RC);
      NNK_CHECK_LAUNCH();
      NNK_CUDA(cudaStreamSynchronize(st));  // dsrc and cmp's buffers are reused by the next pass
      const auto& nd = passes[ps].nodes;
      for (size_t f = 0; f < nd.size(); f += 64) {
        bt.push_back(BasisTile{(int)ps, (int)bn.size(), (int)std::min<size_t>(64, nd.size() - f), 0});
        bn.insert(bn.end(), nd.begin() + f, nd.begin() + std::min(nd.size(), f + 64));
      }
    }
    plan.btiles.upload(bt, st);
    plan.bnodes.upload(bn, st);
    plan.nbtiles = (int)bt.size();
    plan.chat.alloc((size_t)t.nodes * RC);
    plan.part.alloc(std::max<size_t>((size_t)plan.nunits * kTileRows * RC, 1));
    plan.src_lo.alloc((size_t)t.nodes * RC);
    plan.src_lo.zero(st);
  } else if (plan.use_images && !img_code.empty()) {
    plan.slot_op.upload(slot_op, st);
    plan.images.alloc(img_code.size() * (size_t)NP * NP);
    plan.images.zero(st);
    DBuf<int> dcode, dlat;
    DBuf<double> dw;
    dcode.upload(img_code, st);
    dw.upload(img_w, st);
    dlat.upload(lat, st);
    const long long total = (long long)P * P * (long long)img_code.size();
    m2l_operator_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(
        (int)img_code.size(), dcode.p, dw.p, dlat.p, P, res, eps, mu, NP, plan.images.p);
    NNK_CHECK_LAUNCH();
    NNK_CUDA(cudaStreamSynchronize(st));
  }
  plan.P = P;
  plan.res = res;
  plan.e2 = (float)(eps * eps);
  plan.scale = (float)(1.0 / (8.0 * M_PI * mu));
  plan.src.alloc((size_t)t.nodes * NP);
  plan.src.zero(st);
  plan.err.alloc(1);
  plan.err.zero(st);
  if (!plan.h_err) NNK_CUDA(cudaMallocHost((void**)&plan.h_err, sizeof(int)));
  *plan.h_err = 0;
  if (!plan.err_ev) NNK_CUDA(cudaEventCreateWithFlags(&plan.err_ev, cudaEventDisableTiming));
  // image kernel: 3 stages where they fit (the compressed form's 64 KB stages), else 2
  const size_t na = plan.compressed ? 2 : 1;
  auto img_smem = [&](size_t ns) { return 1024 + ns * (na * kTileRows * 128 + (size_t)NP * 128) + 128; };
  plan.stages = img_smem(3) <= kImgSmemMax ? 3 : 2;
  plan.smem_bytes = plan.use_images ? img_smem(plan.stages)
                                    : 1024 + 2 * (size_t)kTileRows * 128 + 2 * (size_t)NP * 128 + 64 + 4 * (size_t)P;
  // the attributes are per kernel, shared by every plan: set them for the largest
  const int max_gen = 1024 + 2 * kTileRows * 128 + 2 * 512 * 128 + 64 + 4 * 512;
  NNK_CUDA(cudaFuncSetAttribute(m2l_gen_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, max_gen));
  NNK_CUDA(cudaFuncSetAttribute(m2l_img_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kImgSmemMax));
  NNK_CUDA(cudaFuncSetAttribute(m2l_ws_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kImgSmemMax));
  NNK_CUDA(cudaStreamSynchronize(st));
  plan.ready = true;
}

namespace {
// Copies the error flag to its pinned host mirror after a launch and marks
// the copy with the plan's event.
void mirror_err(M2LPlan& plan, cudaStream_t st) {
  NNK_CUDA(cudaMemcpyAsync(plan.h_err, plan.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  NNK_CUDA(cudaEventRecord(plan.err_ev, st));
}
}  // namespace

void launch_m2l(M2LPlan& plan, float* check, int ldc, cudaStream_t st, const float* up, long long ld_up) {
  if (!plan.nunits) return;
  if (plan.compressed) {
    if (!up) throw Error(NNK_E_STATE, "compressed M2L needs the up densities");
    const int RC = plan.RC;
    basis_apply_kernel<<<dim3((RC + 63) / 64, plan.nbtiles), 256, 0, st>>>(
        plan.basis.p, plan.n3, RC, 1, plan.btiles.p, plan.bnodes.p, up, ld_up, plan.src.p, RC, plan.src_lo.p);
    NNK_CHECK_LAUNCH();
    NNK_CUDA(cudaMemsetAsync(plan.chat.p, 0, plan.chat.bytes(), st));
    m2l_ws_kernel<<<plan.nunits, 32 * (1 + kWsGatherWarps), plan.smem_bytes, st>>>(
        plan.units.p, plan.tile_nodes.p, plan.tile_slot0.p, plan.slot_op.p, plan.slot_src.p, plan.images.p,
        plan.src.p, plan.src_lo.p, plan.chat.p, RC, RC, plan.err.p, plan.stages, plan.wait_limit, 0, plan.part.p);
    NNK_CHECK_LAUNCH();
    mirror_err(plan, st);
    m2l_unit_reduce_kernel<<<plan.ntiles, 256, 0, st>>>(plan.tile_uoff.p, plan.tile_units.p, plan.tile_nodes.p,
                                                        plan.part.p, RC, plan.chat.p, RC);
    NNK_CHECK_LAUNCH();
    basis_apply_kernel<<<dim3((plan.n3 + 63) / 64, plan.nbtiles), 256, 0, st>>>(
        plan.basis.p, plan.n3, RC, 0, plan.btiles.p, plan.bnodes.p, plan.chat.p, RC, check, ldc);
    NNK_CHECK_LAUNCH();
    return;
  }
  if (plan.use_images) {
    m2l_img_kernel<<<plan.nunits, 128, plan.smem_bytes, st>>>(plan.units.p, plan.tile_nodes.p, plan.tile_slot0.p,
                                                              plan.slot_op.p, plan.slot_src.p, plan.images.p,
                                                              plan.src.p, check, ldc, plan.NP, plan.err.p, nullptr,
                                                              plan.stages);
    NNK_CHECK_LAUNCH();
    mirror_err(plan, st);
    return;
  }
  m2l_gen_kernel<<<plan.nunits, 128, plan.smem_bytes, st>>>(
      plan.units.p, plan.tile_nodes.p, plan.tile_slot0.p, plan.slot_code.p, plan.slot_h.p, plan.slot_src.p,
      plan.lat.p, plan.P, plan.res, plan.e2, plan.scale, plan.src.p, check, ldc, plan.NP, plan.err.p);
  NNK_CHECK_LAUNCH();
  mirror_err(plan, st);
}

namespace {
// Reads the mirrored flag once its copy has completed; clears a set flag
// (device and host) and returns it.
int take_err(M2LPlan& plan, cudaStream_t st) {
  if (!plan.h_err || !plan.err_ev) return 0;
  const cudaError_t q = cudaEventQuery(plan.err_ev);
  if (q == cudaErrorNotReady) return 0;
  NNK_CUDA(q);
  const int f = *plan.h_err;
  if (f) {
    *plan.h_err = 0;
    NNK_CUDA(cudaMemsetAsync(plan.err.p, 0, sizeof(int), st));
  }
  return f;
}
}  // namespace

void check_m2l_error(M2LPlan& plan, cudaStream_t st) {
  if (!plan.h_err) return;
  NNK_CUDA(cudaStreamSynchronize(st));
  poll_m2l_error(plan, st);
}

void poll_m2l_error(M2LPlan& plan, cudaStream_t st) {
  const int f = take_err(plan, st);
  if (f) throw Error(NNK_E_TIMEOUT, "tensor-core M2L gave up a bounded wait (flag " + std::to_string(f) + ")");
}

int stall_m2l_probe(M2LPlan& plan, uint32_t polls, cudaStream_t st) {
  if (!plan.compressed || !plan.nunits)
    throw Error(NNK_E_STATE, "the failure-path probe needs the compressed tensor-core M2L with V pairs");
  if (polls == 0) throw Error(NNK_E_ARG, "the probe needs a positive wait limit");
  check_m2l_error(plan, st);  // an earlier flag is not the probe's
  m2l_ws_kernel<<<plan.nunits, 32 * (1 + kWsGatherWarps), plan.smem_bytes, st>>>(
      plan.units.p, plan.tile_nodes.p, plan.tile_slot0.p, plan.slot_op.p, plan.slot_src.p, plan.images.p,
      plan.src.p, plan.src_lo.p, plan.chat.p, plan.RC, plan.RC, plan.err.p, plan.stages, polls, 1, plan.part.p);
  NNK_CHECK_LAUNCH();
  mirror_err(plan, st);
  NNK_CUDA(cudaStreamSynchronize(st));
  const int f = take_err(plan, st);
  NNK_CUDA(cudaStreamSynchronize(st));
  return f;
}

}  // namespace nnk
