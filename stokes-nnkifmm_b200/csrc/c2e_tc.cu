// Check-to-equivalent products on the tensor cores (see c2e_tc.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "c2e_tc.h"
#include "kernels.cuh"
#include "tc_util.cuh"

namespace nnk {

namespace {

using namespace tc;

constexpr int kRows = 128;                    // operator rows per CTA (the MMA's M)
constexpr int kCols = 32;                     // check columns per CTA (the MMA's N)
constexpr int kKChunk = 128;                  // K per staged chunk (one 128-byte swizzled row)
constexpr int kKPad = 512;                    // K padded to four chunks (3P <= 512)
constexpr int kATile = kRows * kKChunk;       // bytes of one operator digit tile
constexpr int kBTile = kCols * kKChunk;       // bytes of one check digit tile

// Byte offset of element (row, k) in a K-major tile of 128-byte rows with the
// 128-byte swizzle: 16-byte chunk k / 16 of row `row` sits at chunk
// (k / 16) ^ (row % 8).
__device__ __forceinline__ int swz(int row, int k) { return row * 128 + ((((k >> 4) ^ (row & 7)) << 4) | (k & 15)); }

// Exponent e with |x| / 2^e < 1 for every x of the row or column (max > 0),
// and 0 for an all-zero one.
__device__ __forceinline__ int digit_exponent(double m) { return m > 0 ? ilogb(m) + 1 : 0; }

// Digits of one value: r = x 2^-e in (-1, 1); digit t is the integer part of
// r 128^(t+1) after the earlier digits are taken off (truncation toward zero,
// so each remainder stays in (-1, 1) and every digit in [-127, 127]).  Every
// step is exact in FP64: scaling by 128, the integer part, the subtraction.
__device__ __forceinline__ int8_t next_digit(double& r) {
  r *= 128.0;
  const double q = trunc(r);
  r -= q;
  return (int8_t)q;
}

// Operator digits: one warp per (op, dir, row); rows >= n and K >= n are 0.
__global__ void a_digits_kernel(const double* __restrict__ ops, int nops, int n, int sA, int8_t* __restrict__ adig,
                                int* __restrict__ aexp) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= nops * 2 * kKPad) return;
  const int row = warp % kKPad, od = warp / kKPad, dir = od & 1, op = od >> 1;
  const double* A = ops + (size_t)op * n * n;
  double v[kKPad / 32];
  double m = 0;
#pragma unroll
  for (int q = 0; q < kKPad / 32; ++q) {
    const int k = lane + 32 * q;
    double x = 0;
    if (row < n && k < n) x = dir ? A[(size_t)row * n + k] : A[(size_t)k * n + row];  // A^T[row][k] = A[k][row]
    v[q] = x;
    m = fmax(m, fabs(x));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  const int e = digit_exponent(m);
  if (lane == 0) aexp[(size_t)od * kKPad + row] = e;
  const int rb = row / kRows, r = row % kRows;
  int8_t* base = adig + ((size_t)od * 4 + rb) * 4 * sA * kATile;
#pragma unroll
  for (int q = 0; q < kKPad / 32; ++q) {
    const int k = lane + 32 * q, kc = k / kKChunk;
    double x = ldexp(v[q], -e);
    for (int t = 0; t < sA; ++t) base[((size_t)kc * sA + t) * kATile + swz(r, k % kKChunk)] = next_digit(x);
  }
}

// Check digits of the launch: block (tile, z) covers columns 32 z .. 32 z + 31
// of the tile (column j: node tiles[tile].first + j / R, right-hand side j % R);
// one warp per column, lane l owning K = 16 l .. 16 l + 15 (one 16-byte chunk
// of every digit row, written with one 16-byte store per digit); columns past
// the tile are 0.
template <typename Real>
__global__ void b_digits_kernel(const C2ETile* __restrict__ tiles, const int* __restrict__ nodes,
                                const Real* __restrict__ check, int n, int P, int R, int sB, int zch,
                                int8_t* __restrict__ bdig, int* __restrict__ bexp, const int* __restrict__ nact) {
  const int blk = blockIdx.x * zch + blockIdx.y;
  const C2ETile tl = tiles[blockIdx.x];
  if (nact && !nact[nodes[tl.first]]) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int8_t* base = bdig + (size_t)blk * 4 * sB * kBTile;
  const int k0 = 16 * lane, kc = k0 / kKChunk;
  for (int c = warp; c < kCols; c += blockDim.x >> 5) {
    const int j = blockIdx.y * kCols + c;
    const bool on = j < tl.count * R;
    const int node = on ? nodes[tl.first + j / R] : 0, kr = on ? j % R : 0;
    double v[16];
    double m = 0;
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int k = k0 + q;
      double x = 0;
      if (on && k < n) x = (double)check[(((size_t)node * P + k / 3) * R + kr) * 3 + k % 3];
      v[q] = x;
      m = fmax(m, fabs(x));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    const int e = digit_exponent(m);
    if (lane == 0) bexp[(size_t)blk * kCols + c] = e;
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = ldexp(v[q], -e);
    // this lane's chunk sits at chunk (k0 % 128) / 16 ^ (c % 8) of row c
    const int off = swz(c, k0 % kKChunk);
    for (int u = 0; u < sB; ++u) {
      uint32_t w[4];
#pragma unroll
      for (int q4 = 0; q4 < 4; ++q4) {
        uint32_t word = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) word |= (uint32_t)(uint8_t)next_digit(v[4 * q4 + b]) << (8 * b);
        w[q4] = word;
      }
      *reinterpret_cast<uint4*>(base + ((size_t)kc * sB + u) * kBTile + off) = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

// Instruction descriptor: D S32, A and B signed 8-bit, both K-major, M = 128,
// N = 32.
constexpr uint32_t kI8Idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kCols >> 3) << 17) |
                              ((uint32_t)(kRows >> 4) << 24);

__device__ __forceinline__ void umma_i8(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(kI8Idesc), "r"(accumulate)
      : "memory");
}

// CTA (row block, tile, z): 128 operator rows x 32 columns.  Thread 0 moves
// the digits of one K chunk into shared memory with two bulk copies (all
// operator digits, all check digits), waits, and issues the MMAs of every
// digit pair (t, u) with t + u < L into the level's int32 accumulator
// (TMEM columns 32 l .. 32 l + 31), four K = 32 steps per chunk; the chunk's
// shared memory is reused once those MMAs are done.  Then the 4 warps read
// their 32 rows of every level and combine them in FP64.  Every wait is
// bounded; a timeout sets err, the CTA drains its copies and exits.
template <typename Real>
__global__ void __launch_bounds__(128, 1)
    c2e_tc_kernel(const int8_t* __restrict__ adig, const int* __restrict__ aexp, int dir, int sA, int sB, int L,
                  const C2ETile* __restrict__ tiles, const int* __restrict__ nodes, int zch,
                  const int8_t* __restrict__ bdig, const int* __restrict__ bexp, int n, int P, int R,
                  Real* __restrict__ dst, long long base, float* __restrict__ m2l_dst, int NP, int* err,
                  uint32_t wlim, const int* __restrict__ nact) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  uint8_t* sbase = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  uint8_t* sA_ = sbase;                                  // sA digit tiles of 128 x 128 bytes
  uint8_t* sB_ = sbase + (size_t)sA * kATile;            // sB digit tiles of 32 x 128 bytes
  uint64_t* bars = reinterpret_cast<uint64_t*>(sB_ + (size_t)sB * kBTile);  // full, done
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2);
  volatile int* abort_s = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int rb = blockIdx.x, tile = blockIdx.y, z = blockIdx.z;
  const C2ETile tl = tiles[tile];
  if (nact && !nact[nodes[tl.first]]) return;  // uniform over the CTA, before any barrier
  if (z * kCols >= tl.count * R) return;
  const int blk = tile * zch + z;
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    *abort_s = 0;
    fence_barrier_init();
  }
  // accumulator columns: L levels x 32, rounded up to a power of two (256
  // for L <= 8: two CTAs of the mixed mode's size share an SM's 512)
  const uint32_t ncols = L * kCols <= 256 ? 256u : 512u;
  if (warp == 0) tmem_alloc(tmem_slot, ncols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int od = tl.op * 2 + dir;
  const uint32_t bytes = (uint32_t)(sA * kATile + sB * kBTile);
  int copies = 0, landed = 0;  // thread 0
  if (tid == 0) {
    uint32_t started = 0;  // levels whose accumulator holds a product
    for (int kc = 0; kc < 4; ++kc) {
      mbar_expect_tx(&bars[0], bytes);
      bulk_g2s(sA_, adig + (((size_t)od * 4 + rb) * 4 + kc) * sA * kATile, (uint32_t)(sA * kATile), &bars[0]);
      bulk_g2s(sB_, bdig + ((size_t)blk * 4 + kc) * sB * kBTile, (uint32_t)(sB * kBTile), &bars[0]);
      ++copies;
      if (!mbar_wait(&bars[0], kc & 1, wlim)) {
        *abort_s = 1;
        atomicOr(err, 1);
        break;
      }
      ++landed;
      tc_fence_after();
      for (int t = 0; t < sA; ++t)
        for (int u = 0; u < sB && t + u < L; ++u) {
          const int l = t + u;
          const uint32_t a0 = smem_u32(sA_ + (size_t)t * kATile), b0 = smem_u32(sB_ + (size_t)u * kBTile);
#pragma unroll
          for (int k32 = 0; k32 < 4; ++k32) {
            umma_i8(tmem + (uint32_t)(l * kCols), sw128_desc(a0 + k32 * 32), sw128_desc(b0 + k32 * 32),
                    ((started >> l) & 1) ? 1u : 0u);
            started |= 1u << l;
          }
        }
      umma_commit(&bars[1]);  // the chunk's MMAs (and all before them)
      if (!mbar_wait(&bars[1], kc & 1, wlim)) {
        *abort_s = 1;
        atomicOr(err, 2);
        break;
      }
    }
    // a copy that never landed must not outlive the CTA
    for (int c = landed; c < copies; ++c)
      if (!mbar_wait(&bars[0], c & 1, wlim)) atomicOr(err, 4);
  }
  __syncthreads();
  tc_fence_after();
  if (!*abort_s) {
    const int row = rb * kRows + warp * 32 + (tid & 31);
    const int ea = aexp[(size_t)od * kKPad + min(row, kKPad - 1)];
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c0 = 0; c0 < kCols; c0 += 16) {
      double acc[16];
#pragma unroll
      for (int c = 0; c < 16; ++c) acc[c] = 0;
      for (int l = L - 1; l >= 0; --l) {  // smallest terms first
        float raw16[16];
        tmem_ld16(lane_addr + (uint32_t)(l * kCols + c0), raw16);
        const double sc = ldexp(1.0, -7 * (l + 2));
#pragma unroll
        for (int c = 0; c < 16; ++c) acc[c] = fma((double)__float_as_int(raw16[c]), sc, acc[c]);
      }
      if (row < n) {
        const int p = row / 3, comp = row - 3 * p;
#pragma unroll
        for (int c = 0; c < 16; ++c) {
          const int j = z * kCols + c0 + c;
          if (j >= tl.count * R) continue;
          const int node = nodes[tl.first + j / R];
          const double v = ldexp(acc[c], ea + bexp[(size_t)blk * kCols + c0 + c]);
          dst[((base + (long long)P * node + p) * R + j % R) * 3 + comp] = (Real)v;
          if (m2l_dst) {
            uint32_t t32;
            asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t32) : "f"((float)v));
            m2l_dst[(size_t)node * NP + row] = __uint_as_float(t32);
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, ncols);
}

size_t tc_smem(int sA, int sB) { return 1024 + (size_t)sA * kATile + (size_t)sB * kBTile + 64; }

}  // namespace


size_t c2e_tc_blocks(int ntiles, int R) { return (size_t)ntiles * ((kC2ETileNodes * R + kCols - 1) / kCols); }

void build_c2e_tc(C2ETcPlan& plan, const double* ops, int nops, int n, int sA, int sB, int L, cudaStream_t st) {
  if (n > kKPad) throw Error(NNK_E_ARG, "tensor-core C2E supports 3P <= 512");
  if (sA < 1 || sA > 9 || sB < 1 || sB > 9 || L < 1 || L > 9 || L > sA + sB - 1)
    throw Error(NNK_E_ARG, "tensor-core C2E digit counts out of range");
  plan.sA = sA;
  plan.sB = sB;
  plan.L = L;
  plan.n = n;
  plan.nops = nops;
  plan.adig.alloc((size_t)nops * 2 * 4 * 4 * sA * kATile);
  plan.aexp.alloc((size_t)nops * 2 * kKPad);
  const int warps = nops * 2 * kKPad;
  a_digits_kernel<<<(warps + 7) / 8, 256, 0, st>>>(ops, nops, n, sA, plan.adig.p, plan.aexp.p);
  NNK_CHECK_LAUNCH();
  if (!plan.err.p) {
    plan.err.alloc(1);
    plan.err.zero(st);
  }
  plan.smem_bytes = tc_smem(sA, sB);
  NNK_CUDA(cudaFuncSetAttribute(c2e_tc_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)plan.smem_bytes));
  NNK_CUDA(cudaFuncSetAttribute(c2e_tc_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)plan.smem_bytes));
  NNK_CUDA(cudaStreamSynchronize(st));
  plan.ready = true;
}

void release_c2e_tc(C2ETcPlan& plan) {
  plan.adig.release();
  plan.aexp.release();
  plan.bdig.release();
  plan.bexp.release();
  plan.bblocks = 0;
  plan.ready = false;
}

void reserve_c2e_tc(C2ETcPlan& plan, size_t blocks) {
  if (blocks <= plan.bblocks) return;
  plan.bdig.alloc(blocks * 4 * plan.sB * kBTile);
  plan.bexp.alloc(blocks * kCols);
  plan.bblocks = blocks;
}

template <typename Real>
void launch_c2e_tc(C2ETcPlan& plan, int trans, const C2ETile* tiles, int ntiles, const int32_t* nodes,
                   const Real* check, Real* dst, int64_t base, int P, int R, cudaStream_t st, float* m2l_dst, int NP,
                   const int* nact) {
  if (ntiles == 0) return;
  if (!plan.ready) throw Error(NNK_E_STATE, "tensor-core C2E plan not built");
  const int zch = (kC2ETileNodes * R + kCols - 1) / kCols;
  if ((size_t)ntiles * zch > plan.bblocks) throw Error(NNK_E_STATE, "tensor-core C2E scratch too small");
  b_digits_kernel<Real><<<dim3(ntiles, zch), 256, 0, st>>>(tiles, nodes, check, plan.n, P, R, plan.sB, zch,
                                                           plan.bdig.p, plan.bexp.p, nact);
  NNK_CHECK_LAUNCH();
  c2e_tc_kernel<Real><<<dim3((plan.n + kRows - 1) / kRows, ntiles, zch), 128, plan.smem_bytes, st>>>(
      plan.adig.p, plan.aexp.p, trans ? 1 : 0, plan.sA, plan.sB, plan.L, tiles, nodes, zch, plan.bdig.p,
      plan.bexp.p, plan.n, P, R, dst, (long long)base, m2l_dst, NP, plan.err.p, plan.wait_limit, nact);
  NNK_CHECK_LAUNCH();
}

template void launch_c2e_tc<double>(C2ETcPlan&, int, const C2ETile*, int, const int32_t*, const double*, double*,
                                    int64_t, int, int, cudaStream_t, float*, int, const int*);
template void launch_c2e_tc<float>(C2ETcPlan&, int, const C2ETile*, int, const int32_t*, const float*, float*,
                                   int64_t, int, int, cudaStream_t, float*, int, const int*);

void check_c2e_tc_error(C2ETcPlan& plan, cudaStream_t st) {
  if (!plan.err.p) return;
  NNK_CUDA(cudaStreamSynchronize(st));
  int f = 0;
  NNK_CUDA(cudaMemcpy(&f, plan.err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (f) {
    NNK_CUDA(cudaMemsetAsync(plan.err.p, 0, sizeof(int), st));
    throw Error(NNK_E_TIMEOUT, "tensor-core C2E gave up a bounded wait (flag " + std::to_string(f) + ")");
  }
}

}  // namespace nnk
