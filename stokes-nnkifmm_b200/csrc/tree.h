// Host-side octree, interaction lists and NEAREST source entries.
//
// The tree follows Classes/OcTree.m bit for bit: one scalar root cube from the
// global min/max (OcTree.m:97-98), FP64 midpoints (lo+hi)/2 (:197), strict
// p > centre (:211), children in nodeMap order (x bit most significant,
// :200-212), DFS block numbering (:174-175), maxDepth error (:168-170).
// Node ids are 0-based here (reference id - 1); exports add 1.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

struct nnk_ctx;

namespace nnk {

struct TreeParams {
  int node_capacity = 200;
  int max_depth = 21;
  int nearest = 0;
  int builder = 0;  // 0 auto, 1 host, 2 GPU (node structure and NN matrix)
};

struct Csr {
  std::vector<int64_t> off;  // size rows+1
  std::vector<int32_t> idx;
  int64_t rows() const { return off.empty() ? 0 : (int64_t)off.size() - 1; }
  int64_t begin(int64_t r) const { return off[r]; }
  int64_t end(int64_t r) const { return off[r + 1]; }
};

struct HostTree {
  // ---- points (OcTree.m:80-82)
  int64_t n = 0;                 // unique points
  std::vector<double> pts;       // n*3
  std::vector<uint8_t> is_pot, is_tgt;
  std::vector<int64_t> pot_rank; // point -> row in the potentials input (-1)
  std::vector<int64_t> tgt_rank; // point -> row in the velocity output (-1)
  int64_t n_pot = 0, n_tgt = 0;
  int capacity = 0;              // min(nodeCapacity, n-1)
  TreeParams params;

  // ---- nodes, indexed by 0-based id
  int32_t nodes = 0;
  int32_t max_level = 0;
  std::vector<int32_t> level, parent, child0;  // parent -1 at root, child0 -1 leaf
  std::vector<int32_t> ix, iy, iz;             // integer box coords at own level
  std::vector<double> corners;                 // 6 per node [lo hi]
  std::vector<int64_t> pstart, pcount;         // range of the node in `order`
  std::vector<int64_t> order;                  // points sorted by leaf (orig order inside)
  std::vector<int32_t> point_index;            // leaf id per point
  std::vector<uint8_t> tleaf, pleaf;           // non-empty target / potential leaf
  std::vector<uint8_t> full;                   // subtree has no empty-potential leaf
  std::vector<std::vector<int32_t>> colleagues;  // same-level touching nodes (incl. self)
  std::vector<std::vector<int32_t>> by_level;    // node ids per level, ascending

  // ---- lists in the reference's order (0-based ids)
  Csr U, V, W, X;

  // ---- NEAREST
  int64_t q = 0;
  std::vector<double> fine;         // q*3
  std::vector<int64_t> nn_rowptr;   // CSR by fine point
  std::vector<int32_t> nn_col;      // column = row in potPoints (= point, NEAREST)
  std::vector<double> nn_val;

  // ---- leaf source entries (sorted by leaf, then fine index / point index)
  //  entry e: position src_pos[e], force = sum_k w * f[pot row] over its gather
  std::vector<int64_t> src_start;   // per node, size nodes+1 (only leaves non-empty)
  std::vector<double> src_pos;      // E*3
  std::vector<int64_t> src_goff;    // E+1
  std::vector<int32_t> src_gidx;    // potential row
  std::vector<double> src_gw;       // weight
  std::vector<int64_t> src_origin;  // per entry: fine point (NEAREST) or potential row (plain)
  // ---- leaf targets (sorted by leaf)
  std::vector<int64_t> tgt_start;   // per node, size nodes+1
  std::vector<int32_t> tgt_row;     // output row per sorted target
  std::vector<double> tgt_pos;      // sorted target positions

  // ---- forest: several independent trees in one set of arrays (batched
  // bodies).  A single tree is the forest of one group.
  std::vector<int32_t> group;       // per node: tree of the forest (empty: all 0)
  std::vector<int32_t> roots;       // root node per group (empty: {0})
  int32_t groups() const { return roots.empty() ? 1 : (int32_t)roots.size(); }
  int32_t group_of(int32_t n) const { return group.empty() ? 0 : group[n]; }
  int32_t root_of(int32_t g) const { return roots.empty() ? 0 : roots[g]; }

  bool touch(int32_t a, int32_t b) const;  // nodeintersection.m closed-box test
};

// Returns 0 or an NNK_E_* code; msg gets the reason.  With a GPU context
// the node structure (build_nodes_gpu) and the NN matrix
// (nearest_matrix_gpu) are built on the device.
int build_tree(const double* pot, int64_t n_pot, const double* tgt, int64_t n_tgt,
               const double* fine, int64_t q, const int64_t* nn_rowptr,
               const int32_t* nn_col, const double* nn_val, const TreeParams& p,
               HostTree& t, std::string& msg, struct ::nnk_ctx* gpu = nullptr);
int build_nodes_gpu(struct ::nnk_ctx* ctx, HostTree& t, std::string& msg);
void nearest_matrix_gpu(struct ::nnk_ctx* ctx, const double* coarse, int64_t n, const double* fine, int64_t q,
                        std::vector<int64_t>& rowptr, std::vector<int32_t>& col, std::vector<double>& val);

// Concatenates trees into one forest: node ids, list entries, leaf source
// entries, gather rows and target rows of tree k are offset by the totals of
// trees 0..k-1, and `group` records the tree of every node.  No list links
// two trees, so the FMM of the forest is the block-diagonal operator of the
// separate trees.  A tree may appear several times.
void merge_forest(const std::vector<const HostTree*>& trees, HostTree& out);
// The U/V/W/X lists of a tree whose node arrays are built (lists_gpu.cu),
// identical to the host builder's.
void build_lists_gpu(struct ::nnk_ctx* ctx, HostTree& t);

// nearestMatrix (Tools/Nearest/nearestMatrix.m:17-41), exact FP64 ties.
// Rewrites the tie weights of a nearest-neighbour matrix (CSR by fine point,
// every tied pair present with weight 1/k) into the pairing that
// Tools/Nearest/nearestMatrix.m:23-39 produces as written: per block of
// floor(block_size 2^27 / (9 q)) fine points, the j-th tied pair in
// column-major order receives the j-th weight in row-major order.  Throws
// NNK_E_ARG when that block size is 0 (the reference then builds no matrix).
void nearest_reference_weights(int64_t q, const int64_t* rowptr, const int32_t* col, double* val,
                               double block_size);
void nearest_matrix(const double* coarse, int64_t n, const double* fine, int64_t q,
                    std::vector<int64_t>& rowptr, std::vector<int32_t>& col,
                    std::vector<double>& val);

}  // namespace nnk
