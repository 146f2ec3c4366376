// M2L (V-list, DownNonleaf.m:34-38 / downwardPass.m:59-74) in Fourier space.
//
// The up-equivalent surface of a node is the outer shell of a res^3 lattice
// of spacing h = w / (res - 1) on its box.  For a target node i and a source
// v in V(i) at offset o = (v - i) in box widths, the reference adds
//   check_i(a) += sum_b K((a - b - (res - 1) o) h) q_v(b)
// over lattice points a, b (the kernel matrix of upsurf(v) -> upsurf(i)).
// This is a discrete convolution: a - b spans 2 res - 1 values per axis, so
// with the densities zero-padded to a G^3 grid, G = 2 res - 1, the cyclic
// convolution has no wrap-around and becomes a pointwise product of spectra:
//   C_i(k) = sum_{v in V(i)} Khat_{w,o}(k) Q_v(k),
// Khat the 3 x 3 (symmetric) spectrum of the kernel sampled on the difference
// grid, Q_v the spectrum of v's densities.  Per V pair this costs
// 9 complex multiply-adds per frequency and right-hand side on
// G^2 (G/2 + 1) frequencies (real-to-complex), against (3P)^2 for the dense
// matrix.  Spectra are FP32 (mixed mode) or FP64 (FP64 mode); the kernel
// spectra are computed in FP64 once per (box width, offset) with 1/(8 pi mu)
// and the 1/G^3 of the inverse transform folded in.
#pragma once
#include <vector>

#include "common.h"
#include "tree.h"

namespace nnk {

// Grid size of the transforms for a res^3 lattice (11 for res = 6: 11 x 11 x 6
// = 726 frequencies in the half spectrum).
__host__ __device__ constexpr int fft_grid(int res) { return 2 * res - 1; }

// Parent-grouped form of the accumulation for one right-hand side: every V
// pair (i, v) of the reference's lists joins a child i of a parent P with a
// child v of a colleague N of P (same level, touching P).  One record per
// (P, N) holds which of the 8 x 8 (child of P, child of N) pairs are V pairs,
// indexed by child position (x * 4 + y * 2 + z within the parent box), and
// the direction d = N - P; the pair's offset is 2 d + (pos_v - pos_i).  A
// thread accumulates all 8 children of P at one frequency: each kernel
// spectrum it loads serves every pair with the same pos_v - pos_i, and each
// source spectrum every child of P.
struct FftFamily {
  int first, count;  // its (P, N) records
  int op;            // operator (box width) of the children's level
  int tgt[8];        // target slot of the child at each position (-1 none)
};
struct FftFamilyPair {
  uint32_t mask_lo, mask_hi;  // bit 8 * pos_i + pos_v
  int dcode;                  // (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1)
  int op;                     // operator (box width) of the children's level
  int src[8];                 // source slot of N's child at each position (-1 none)
};

struct FftM2L {
  int res = 0, G = 0, NK = 0, P = 0;
  int nsrc = 0, ntgt = 0, nspec = 0, Rcap = 1;
  int64_t pairs = 0;
  DBuf<int> lat;        // per surface point: x | y << 8 | z << 16 lattice indices
  bool fp64 = false;    // FP64 spectra and transforms (the *64 buffers)
  DBuf<float2> spec;    // nspec x 6 x NK (xx, xy, xz, yy, yz, zz)
  DBuf<int> src_node;   // per source slot: node
  DBuf<int> tgt_node;   // per target slot: node
  DBuf<int> voff;       // per target slot: first pair (ntgt + 1)
  DBuf<int> vsrc;       // per pair: source slot
  DBuf<int> vspec;      // per pair: kernel spectrum
  DBuf<float2> qhat;    // nsrc x 3R x NK
  DBuf<float2> chat;    // ntgt x 3R x NK
  DBuf<double2> spec64, qhat64, chat64;
  DBuf<double2> dspec64;  // spectra of the kernel's eps-derivative (built on demand)
  std::vector<double> slot_w_host;  // per spectrum: box width
  std::vector<int> slot_code_host;  // per spectrum: offset code
  // parent-grouped accumulation, when every V pair fits it
  bool family = false;
  int nfam = 0;
  DBuf<FftFamily> fams;
  DBuf<FftFamilyPair> fpairs;
  DBuf<int> spec_of;  // per (operator, offset code): spectrum slot (-1 unused)
  int64_t records = 0, groups = 0;  // (P, N) records; (record, difference) groups
  size_t fwd_smem = 0, inv_smem = 0;
};

// Largest right-hand side count per pass (6, 4, 3, 2 or 1; 0 if none) whose
// transforms fit the device's shared memory.
int fft_m2l_max_rhs(int res, bool fp64);
// node_op[n]: check-to-equivalent operator index of node n's (tree, level);
// op_w[op]: its box width.  Rmax: right-hand sides per pass.
void build_fft_m2l(const HostTree& t, int res, int shells, double eps, double mu, const std::vector<double>& op_w,
                   const std::vector<int>& node_op, int Rmax, bool fp64, FftM2L& f, cudaStream_t st);
// check[((P * node + p) * R + r) * 3 + c] = M2L result for every node with a
// V-list (other entries untouched); str holds the up-equivalent densities of
// node n at str[((upbase + P * n + p) * R + r) * 3 + c].  nact (per node,
// or nullptr): nodes with nact = 0 are neither transformed nor written.
void launch_fft_m2l(FftM2L& f, const float* str, long long upbase, int R, float* check, cudaStream_t st,
                    const int* nact = nullptr);
void launch_fft_m2l(FftM2L& f, const double* str, long long upbase, int R, double* check, cudaStream_t st,
                    const int* nact = nullptr);
// The same M2L with the kernel's eps-derivative (FP64 plans, one right-hand
// side); build_fft_deriv computes its spectra.
void build_fft_deriv(FftM2L& f, double eps, double mu, cudaStream_t st);
void launch_fft_m2l_deriv(FftM2L& f, const double* str, long long upbase, double* check, cudaStream_t st);

}  // namespace nnk
