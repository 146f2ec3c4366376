// Check-to-equivalent products on the tensor cores (tcgen05.mma kind::i8)
// with FP64 accuracy: int8 slices of the operator and of the check vectors
// multiplied with exact int32 sums and combined in FP64 (the Ozaki scheme).
//
// An operator row i (FP64) is written as 2^ea_i * sum_t A_t[i] 128^-(t+1)
// with int8 digits A_t in [-127, 127] (truncation, so every remainder stays
// below one digit), a check column j likewise as 2^eb_j * sum_u B_u[j]
// 128^-(u+1).  The product keeps the digit pairs with t + u < L:
//   out[i][j] = 2^(ea_i + eb_j) sum_l 128^-(l+2) C_l[i][j],
//   C_l = sum_{t+u=l} A_t B_u,
// each C_l an exact int32 sum (|C_l| <= 9 * 456 * 127^2 < 2^31) accumulated
// in tensor memory.  With 9 + 9 digits and L = 9 (45 digit products) the
// result carries the FP64 product's error (the rows of the exact inverses
// cancel by ~1e5, so the product's own rounding is ~1e-11 relative); the
// mixed mode's FP32 check vectors take 5 operator digits, 4 check digits and
// L = 5 (14 products).
//
// Layout: the operator digits are prepared once per operator and direction
// (A, or A^T for the downward step) in the tile order of the kernel:
// [op][dir][row block of 128][K chunk of 128][digit t][128 x 128 bytes],
// each 16 KiB tile K-major with the 128-byte swizzle, so one bulk copy moves
// all digits of a (row block, K chunk).  The check digits are written per
// launch by a pre-pass in the same form for 32 columns.
#pragma once
#include <cstdint>

#include "common.h"

namespace nnk {

struct C2ETile;  // fmm.h

struct C2ETcPlan {
  int sA = 0, sB = 0, L = 0;  // operator digits, check digits, levels (t + u < L)
  int n = 0;                  // 3P, at most 512
  int nops = 0;
  DBuf<int8_t> adig;          // [op][dir][4][4][sA][128 x 128]
  DBuf<int> aexp;             // [op][dir][512]
  DBuf<int8_t> bdig;          // launch scratch: [block][4][sB][32 x 128]
  DBuf<int> bexp;             // launch scratch: [block][32]
  size_t bblocks = 0;         // blocks the scratch holds
  DBuf<int> err;              // bounded-wait timeout flag (read at the caller's synchronizations)
  uint32_t wait_limit = 1u << 26;
  size_t smem_bytes = 0;
  bool ready = false;
};

// Digits of the n x n column-major operators ops[op] (A and A^T) for the
// given digit counts; device work on st.
void build_c2e_tc(C2ETcPlan& plan, const double* ops, int nops, int n, int sA, int sB, int L, cudaStream_t st);
// Frees the digits and the scratch (the plan is no longer ready).
void release_c2e_tc(C2ETcPlan& plan);
// Scratch for launches of up to `blocks` 32-column blocks.
void reserve_c2e_tc(C2ETcPlan& plan, size_t blocks);
// Blocks (32 columns each) a launch over ntiles tiles of R right-hand sides needs.
size_t c2e_tc_blocks(int ntiles, int R);
// dst(node, k) = Aop check(node, k) for the nodes of `tiles` (as launch_c2e).
template <typename Real>
void launch_c2e_tc(C2ETcPlan& plan, int trans, const C2ETile* tiles, int ntiles, const int32_t* nodes,
                   const Real* check, Real* dst, int64_t base, int P, int R, cudaStream_t st,
                   float* m2l_dst = nullptr, int NP = 0, const int* nact = nullptr);
// A flag set by an earlier launch: NNK_E_TIMEOUT.  Synchronizes the stream
// and reads the flag (no event is recorded with the launches, so they can be
// captured into CUDA graphs).
void check_c2e_tc_error(C2ETcPlan& plan, cudaStream_t st);

}  // namespace nnk
