// M2L (V-list, DownNonleaf.m:34-38 / downwardPass.m:59-74) on the tensor cores.
//
// For a target node i at level L and a source node v in V(i), the reference
// adds kernel(upsurf(v), upsurf(i)) * uppot(v) to the check potential of i.
// Both surfaces are the same lattice shifted by o = (v - i) in box widths,
// |o|_inf in {2,3}, so the 3P x 3P matrix T_{L,o} depends only on the level
// and the offset.  Here, for each level, target nodes are tiled 128 at a time
// (grouped by octant inside the parent, which fixes the set of offsets their
// V-lists can use) and
//     D[node, row] += sum_o sum_k U_o[node, k] * T_{L,o}[row, k]
// runs as a TF32 tcgen05 GEMM with the accumulator in TMEM: M = 128 nodes,
// N = 3P padded to a multiple of 32 (480 for p = 6), K = 3P per offset,
// U_o gathered from the TF32 copy of the up densities.  T_{L,o} comes either
// from pre-swizzled operator images streamed with cp.async.bulk (default), or,
// when the images would exceed the memory budget (many trees of different
// sizes), it is computed chunk by chunk from the kernel formula into shared
// memory by the CTA itself (about 2.7x slower per chunk, no memory).  The result is added into
// the check buffer, which the P2L / L2L pair tasks then add to.
//
// Compressed form (default for 3P > 256): T_o^T = T_{-o} (the Stokeslet is
// even and its 3x3 blocks symmetric), so sum_o T_o T_o^T = sum_o T_o^T T_o
// and one orthonormal basis B_L (3P x RC, the leading RC eigenvectors of
// that sum over the 316 far offsets) captures both sides:
//     T_{L,o} ~= B_L C_{L,o} B_L^T,   C_{L,o} = B_L^T T_{L,o} B_L  (RC x RC).
// B is the eigenvector basis rotated by a normalized Hadamard matrix, which
// spreads each vector over all RC coordinates (in the eigenbasis a few
// leading terms carry the sums, and their TF32 rounding errors do not
// average out).  Per matvec: u^ = B^T u for every node that is a V source
// (FP32 GEMM, split into two TF32 terms), c^ = sum_o C_o u^_v on the tensor
// cores (the image kernel with NP = RC, both terms into one accumulator;
// each work unit writes its own partial block, and the blocks of a tile are
// added in unit order, so the result is the same bit for bit on every run),
// check += B c^ for every V target.  RC = 256 for p = 6: 2 x (RC/NP)^2 = 57%
// of the tensor work and 28% of the operator bytes; the truncation error of
// the summed M2L on physical densities is ~1e-6, the TF32 rounding of C_o
// ~4e-5 (the full TF32 operators: ~5e-5).
#pragma once
#include <vector>

#include "common.h"
#include "tree.h"

namespace nnk {

struct M2LUnit {
  int tile;   // tile of 128 target nodes
  int slot0;  // first offset slot of the tile handled by this unit
  int nslot;  // number of offset slots
  int pad;
};

// Nodes nodes[first .. first+count) (count <= 64) that share basis `basis`.
struct BasisTile {
  int basis;
  int first;
  int count;
  int pad;
};

struct M2LPlan {
  int NP = 0;                   // padded 3P (multiple of 32); RC when compressed
  int ntiles = 0, nunits = 0;
  int64_t useful_pairs = 0;     // V pairs (node, source)
  int64_t tile_slots = 0;       // sum over tiles of offset slots (x128 rows each)
  DBuf<int> tile_nodes;         // ntiles * 128, -1 for empty rows
  DBuf<int> tile_slot0;         // per tile: first global slot
  DBuf<int> slot_code;          // per global slot: offset code (ox+3)*49 + (oy+3)*7 + (oz+3)
  DBuf<float> slot_h;           // per global slot: lattice spacing w_L / (res-1) of its level
  DBuf<int> slot_src;           // per global slot: 128 source nodes (-1 none)
  DBuf<M2LUnit> units;
  DBuf<int> lat;                // surface lattice indices, i | j<<4 | k<<8
  bool use_images = false;      // stream operator images (fast) or generate chunks in the kernel
  size_t image_budget = (size_t)8 << 30;
  size_t image_bytes = 0;
  DBuf<int> slot_op;            // per global slot: operator image (image kernel)
  DBuf<float> images;           // per (level, offset): NP/32 chunks of NP x 32 TF32, SW128 K-major
  int P = 0, res = 0;
  float e2 = 0.f, scale = 0.f;
  DBuf<float> src;              // nodes * NP: TF32 copy of the up densities (compressed: B^T u)
  bool compress = true;         // use the compressed form where 3P > RC
  bool compressed = false;
  int n3 = 0;                   // 3P
  int RC = 256;                 // compressed rank
  DBuf<float> basis;            // per level pass: B (3P x RC, row-major)
  DBuf<BasisTile> btiles;       // V targets and sources, by pass
  DBuf<int> bnodes;
  int nbtiles = 0;
  DBuf<float> chat;             // nodes * RC: compressed check potentials
  DBuf<float> part;             // compressed form: nunits * 128 * RC partial sums, one block per unit
  DBuf<int> tile_uoff;          // per tile: its units (ntiles + 1 offsets into tile_units)
  DBuf<int> tile_units;         // unit ids of each tile, ascending (the order their partials are added)
  DBuf<float> src_lo;           // nodes * RC: second TF32 term of B^T u
  DBuf<int> err;                // bounded-wait timeout flag
  int* h_err = nullptr;         // pinned mirror of err
  cudaEvent_t err_ev = nullptr; // recorded after each copy of err into h_err
  uint32_t wait_limit = 1u << 26;  // polls per bounded mbarrier wait (~1-3 s)
  size_t smem_bytes = 0;
  int stages = 2;               // image kernel pipeline depth
  bool ready = false;
  ~M2LPlan();
};

// Builds tiles and slot tables for every level with V pairs.
void build_m2l_plan(const HostTree& t, int res, int shells, double eps, double mu, M2LPlan& plan,
                    cudaStream_t st);
// check[node * ldc + row] += M2L contribution, for every node with a V-list.
// The compressed form first projects the up densities up[node * ld_up + k]
// (k < 3P); the uncompressed one reads plan.src, filled by the up C2E.
void launch_m2l(M2LPlan& plan, float* check, int ldc, cudaStream_t st, const float* up = nullptr,
                long long ld_up = 0);
// Waits for the stream, then throws NNK_E_TIMEOUT if an M2L launch gave up a
// bounded wait.  The flag is cleared when it is reported, so the next call
// on the same plan runs normally.
void check_m2l_error(M2LPlan& plan, cudaStream_t st);
// The same without waiting: reads the flag only if the copy that mirrors it
// to the host has completed (a flag still in flight is seen by a later poll).
void poll_m2l_error(M2LPlan& plan, cudaStream_t st);
// Failure-path test of the compressed tensor-core kernel: one launch whose
// threads first wait, `polls` times at most, on an mbarrier that nothing
// arrives at.  The wait gives up, the kernel sets the error flag, issues no
// copy or MMA, frees its tensor memory and returns; the host reads the flag.
// Returns the flag (nonzero: the timeout was seen), cleared afterwards.
int stall_m2l_probe(M2LPlan& plan, uint32_t polls, cudaStream_t st);

}  // namespace nnk
