// KIFMM operator on one tree (device side).
//
// All pair interactions of the reference passes -- S2M and M2M
// (upwardPass.m), M2L, P2L and L2L (DownNonleaf.m), L2T, P2P and M2T
// (Downleaf.m), with their NEAREST variants -- run through one batched pair
// kernel over "tasks": a target point set plus a list of source segments in
// one unified point array
//   [ leaf source entries | up-equivalent surfaces | down-equivalent surfaces ].
// The per-node check-to-equivalent solves (kernel(...) \ check, Up.m:31-33,
// DownNonleaf.m:42-46) become one precomputed FP64 operator per level, applied
// to all nodes of the level as a batched product.  With the M2L outside the
// pair tasks, the M2M and L2L sums are folded into those products: one FP64
// operator maps a parent's 8 children to its up-equivalent density, another
// a parent to the L2L part of its children's down-equivalent densities.
#pragma once
#include <array>
#include <memory>
#include <vector>

#include "common.h"
#include "m2l.h"
#include "m2l_fft.h"
#include "c2e_tc.h"
#include "tree.h"

namespace nnk {

struct TaskD {
  long long tgt;  // first target (index into the target position array)
  long long out;  // first output slot (3 values each)
  int ntgt;
  int seg0;
  int nseg;
  int partial;    // 1: a piece of a split task, writes its partial-sum slot at `out`
  int node;       // the node whose expansion or leaf targets the task computes
  int pad;
};
// Sum of the k partial-sum slots of a split task, added in a fixed order.
struct RedD {
  long long out;    // output slot of the task
  long long pbase;  // first partial slot; piece i uses pbase + i * ntgt
  int ntgt;
  int k;
  int node;
  int pad;
};
struct SegD {
  long long start;  // first source in the unified arrays
  int count;
  int pad;
};

struct TaskGroup {
  int64_t first = 0, count = 0;  // range in the task array
  int64_t red_first = 0, red_count = 0;  // reductions of its split tasks
  int bs = 128;                  // threads per task (source tile), set by the autotuner
};

struct FmmParams {
  double eps = 0.0, mu = 1.0;
  int res = 6, shells = 1;
  int precision = NNK_PREC_FP64;
  int m2l_mode = 0;
  double reg = 0.0;
  int max_rhs = 1;  // right-hand sides evaluated together (work buffers scale with it)
};

// Where the x, y and z components of row r of right-hand side k live in a
// caller's FP64 vector: x at off(r) + k * rstr(r), y and z at +cstr(r) and
// +2 cstr(r) (device tables).  Without per-row tables (off == nullptr) the
// standard layouts apply: rows (interleaved, KIFMM format 1) or blocked
// (format 2), with the right-hand sides 3 * nrows apart.
struct IoMap {
  const long long* off = nullptr;
  const int* cstr = nullptr;
  const long long* rstr = nullptr;
  int layout = NNK_LAYOUT_ROWS;
  long long nrows = 0;
};

// Nodes nodes[first .. first+count) of one level (count <= 64) that share
// the check-to-equivalent operator `op`.
struct C2ETile {
  int op;
  int first;
  int count;
  int pad;
};

// The pair tasks of one direction of the operator (the matvec, or its
// transpose), grouped by pass and level.
struct TaskSet {
  DBuf<TaskD> tasks;
  DBuf<SegD> segs;
  DBuf<RedD> reds;
  std::vector<TaskGroup> up, down, down_nov;  // per level
  TaskGroup leaf;
  // NEAR32 split (the matvec's task set only): the X-list P2L of every level
  // and the U-list P2P, whose sources are the forces (FP32), apart from the
  // L2L of each level and the L2T + W-list of the leaves (FP64)
  bool near = false;
  std::vector<TaskGroup> l2l;  // per level
  TaskGroup x_only, leaf_u, leaf_far;
  std::vector<int32_t> up_nodes_host;  // nodes whose up-equivalent density is formed, by level
  DBuf<int32_t> up_nodes;
  std::vector<int64_t> up_off;
  DBuf<C2ETile> up_tiles;
  std::vector<C2ETile> up_tiles_host;  // host copies (the library-GEMM C2E form groups them)
  std::vector<int64_t> up_toff;
  // folded form (the matvec's task set only): the M2M and L2L steps run as
  // products with operators that include the check-to-equivalent step, so
  // the pair tasks are the leaves' S2M (up_leaf) and the X-list P2L (down_x),
  // and the C2E step of the upward pass covers the leaves only (upl_*)
  bool fold = false;
  std::vector<TaskGroup> up_leaf, down_x;  // per level
  std::vector<int32_t> upl_nodes_host;
  DBuf<int32_t> upl_nodes;
  std::vector<int64_t> upl_off;
  DBuf<C2ETile> upl_tiles;
  std::vector<C2ETile> upl_tiles_host;
  std::vector<int64_t> upl_toff;
  int64_t partial_slots = 0;
};

// Which points play the leaf sources and the leaf targets, and the lists.
// The matvec: sources = leaf source entries, targets = sorted targets, lists
// U, V, W, X.  Its transpose: sources = sorted targets, targets = entries,
// lists inverted (U^-1, V^-1, and X^-1 in the role of W, W^-1 in that of X).
struct TaskRoles {
  int64_t regionA = 0;                       // leaf source points in the unified array
  const std::vector<int64_t>* src_range = nullptr;  // per node: first leaf source (N + 1)
  const std::vector<int64_t>* tgt_range = nullptr;  // per node: first leaf target (N + 1)
  const std::vector<uint8_t>* src_leaf = nullptr;   // leaves whose up-equivalent density is formed
  const std::vector<uint8_t>* tgt_leaf = nullptr;   // leaves with a leaf stage
  const Csr *U = nullptr, *V = nullptr, *W = nullptr, *X = nullptr;
};

class Fmm {
 public:
  Fmm(nnk_ctx* ctx, const HostTree* tree, const FmmParams& p);
  ~Fmm();
  // in: potentials (n_pot x 3, FP64, device), out: velocities (n_tgt x 3, FP64, device)
  void apply(const double* d_in, double* d_out, int layout, int nrhs);
  // Same with explicit per-row placement of the input and output vectors.
  void apply_mapped(const double* d_in, const IoMap& in, double* d_out, const IoMap& out, int nrhs);
  // The exact transpose of apply: in at the targets, out at the potentials.
  void apply_adjoint(const double* d_in, double* d_out, int layout, int nrhs);
  void apply_adjoint_mapped(const double* d_in, const IoMap& in, double* d_out, const IoMap& out, int nrhs);
  // Gradient of <w, apply(f)> with respect to the positions: at the targets
  // (n_tgt x 3, target order) and at the sources (potential rows in plain
  // mode, fine points in NEAREST mode; n x 3).  Either output may be null.
  void grad_positions(const double* d_f, const double* d_w, int layout, double* d_gt, double* d_gs);
  // w^T (dF/deps) f for the FMM operator F of this object (FP64 with the
  // exact check-to-equivalent inverses): every stage's derivative -- the
  // kernel's eps-derivative in each pair sum and in the M2L, and
  // d(K^-1)/deps = -K^-1 (dK/deps) K^-1 of the check-to-equivalent solves --
  // contracted with the forward pass's inputs to the stage and the
  // transpose pass's sensitivities of its output (one forward, one
  // transpose and one derivative pass).  f at the potentials, w at the
  // targets, both in `layout`.
  double grad_eps(const double* d_f, const double* d_w, int layout);
  int64_t source_origins() const;
  // Rebuild every eps-dependent part (check-to-equivalent operators, M2L
  // images or spectra) for a new eps; the tree-dependent task lists stay.
  void set_eps(double eps);
  // Picks, per launch group of the pair kernel, the block size (source tile
  // of bs points, target chunk of bs or 2 bs) with the shortest measured
  // launch, from {64, 128, 256} (FP64: {64, 128}), for passes of nrhs
  // right-hand sides.  Returns the total pair-kernel time before and after.
  std::pair<double, double> autotune(int nrhs);
  // Changes whenever launches captured earlier would be stale (new operators
  // or tiles: set_eps, autotune).  Drawn from one process-wide counter, so an
  // Fmm created later at a recycled address never repeats a value either.
  uint64_t version() const { return version_; }
  // Trees of the forest the matvec evaluates (flags per tree, nullptr: all).
  // The kernels of a masked tree return at once and its output rows are
  // zero; the transpose and the gradients always evaluate every tree.
  void set_active_trees(const char* on);
  // Same, but over the p=4 surfaces (computeVelSparse).
  Fmm& sparse();
  void reduced_apply(const double* d_in, double* d_out, int layout);
  void reduced_solve(const double* d_in, double* d_out, int layout);
  // The same through the explicit inverses of the leaf blocks (built on
  // first use): not backward stable, but one batched product; for the
  // preconditioner.
  void reduced_solve_inv(const double* d_in, double* d_out, int layout);
  nnk_fmm_stats stats() const { return stats_; }
  // Device-side failures of earlier launches (a bounded wait of the
  // tensor-core M2L that gave up): check_errors waits for the stream and
  // throws NNK_E_TIMEOUT; poll_errors reads only flags whose copy to the host
  // has completed, without waiting.  A reported flag is cleared.
  void check_errors();
  void poll_errors();
  // Failure-path probe of the tensor-core M2L (see stall_m2l_probe); returns
  // the error flag the probe launch set (nonzero when the wait gave up).
  int m2l_stall_probe(uint32_t polls);
  // per-phase CUDA-event timing (NNK_PHASE_*)
  void set_profile(bool on);
  bool profiling() const { return prof_; }
  void read_profile(double* ms, int64_t* launches);
  const HostTree& tree() const { return *t_; }
  nnk_ctx* ctx() const { return ctx_; }
  const FmmParams& params() const { return p_; }
  // FP64 work arrays (FP64 and NEAR32 modes); NEAR32 adds FP32 copies of the
  // points and forces for its near-field pair sums
  bool f64() const { return p_.precision != NNK_PREC_MIXED; }
  // M2M and L2L (2, the default where the tree allows it), or M2M alone
  // (1), in the matvec as products with their kernel matrices, or both as
  // pair sums (0); the form in use.
  void set_m2m_form(int form);
  int m2m_form() const { return m2m_products() ? m2m_on_ : 0; }
  // target-source pairs of each of M2M and L2L (non-leaf nodes x 8 P^2)
  int64_t m2m_pairs() const { return fpar_off_.empty() ? 0 : fpar_off_.back() * 8 * (int64_t)P_ * P_; }
  // Folded M2M / L2L in the matvec (regularized operators only): 0 off (the
  // default), 1 where it pays, 2 wherever available; whether the matvec
  // uses it.
  void set_fold(int mode);
  bool folded() const { return fold_ok_ && fold_on_ > 0; }
  // Check-to-equivalent products: 2 (the default) one cuBLAS DGEMM per run
  // of nodes sharing an operator on gathered check vectors (single-tree
  // FMMs; a matvec being captured into a CUDA graph, and forests, use the
  // SIMT products), 0 FP64 SIMT, 1 tensor cores (where 3P <= 512), -1 the
  // fastest as timed by autotune; the form in use (0, 1 or 2).
  void set_c2e_mode(int mode);
  int c2e_mode() const { return blas_c2e() ? 2 : tc_c2e() ? 1 : 0; }
  // host wall time of the set-up steps (NNK_SETUP_*), milliseconds
  const double* setup_ms() const { return setup_ms_; }
  bool near32() const { return p_.precision == NNK_PREC_NEAR32; }
  // scratch for host-pointer calls
  DBuf<double> io_in, io_out;

 private:
  template <typename Real>
  void apply_impl(const double* d_in, const IoMap& in, double* d_out, const IoMap& out, int k0, int R);
  template <typename Real>
  void adjoint_impl(const double* d_in, const IoMap& in, double* d_out, const IoMap& out, int k0, int R);
  // upward and downward passes of one direction (everything before the leaf stage)
  // near: the NEAR32 split of the matvec (FP32 X-list sums from str32_)
  // fold: the folded M2M / L2L (the matvec only; ignored where not built)
  template <typename Real>
  void far_field(TaskSet& ts, const Real* spos, Real* str, int64_t regionA, int R, bool near = false,
                 bool fold = false);
  template <typename Real>
  void grad_impl(const double* d_f, const double* d_w, int layout, double* d_gt, double* d_gs);
  void build_adjoint();
  int rhs_cap(bool adjoint) const;
  void build_deps();
  double dot_dev(const double* a, const double* b, int64_t n);
  // eps-derivative (grad_eps): dA/deps per operator, saved pass quantities
  bool deps_ready_ = false;
  bool exact_ops_ = false;
  DBuf<double> dops_;
  DBuf<double> gsave_cup_, gsave_d_, gsave_avt_, gdchk_, gdvel_, gdscr_, gpart_;
  double* save_up_ = nullptr;  // far_field copies the up pass's check potentials here when set
  void build_taskset(TaskSet& ts, const TaskRoles& roles, bool stats);
  void build_points();
  void build_tasks();
  void assign_operators();
  void build_operators();
  void build_reduced();
  void split_tasks(TaskSet& ts, std::vector<TaskD>& tasks, std::vector<SegD>& segs);
  template <typename Real>
  void run_group(const TaskSet& ts, const TaskGroup& g, const Real* spos, const Real* sstr, const Real* tpos,
                 Real* out, Real e2, Real scale, int accumulate, int phase_id, int R);
  // dl: the tiles take the operator of level L + dl (the children's level
  // for the folded L2L over parents at level L)
  void build_c2e_tiles(const std::vector<int32_t>& nodes, const std::vector<int64_t>& off,
                       std::vector<C2ETile>& tiles, std::vector<int64_t>& toff, int dl = 0);

  nnk_ctx* ctx_;
  const HostTree* t_;
  FmmParams p_;
  int P_ = 0;            // surface points per node
  int N_ = 0;            // nodes
  int64_t E_ = 0;        // leaf source entries
  int64_t tot_ = 0;      // E + 2 P N
  int maxl_ = 0;
  int R_ = 1;            // right-hand sides the work buffers hold
  std::vector<double> shift_;  // per tree of the forest: FP32 positions are relative to its root centre

  // unified point/strength arrays
  DBuf<double> pos64_;   // tot*3
  DBuf<float> pos32_;    // tot*4
  DBuf<double> str64_;   // tot*3
  DBuf<float> str32_;    // tot*3
  // sorted targets
  DBuf<double> tpos64_;  // ntgt*3
  DBuf<float> tpos32_;   // ntgt*4
  DBuf<int32_t> trow_;
  // gather (NEAREST: kron(NN,I3)*f per entry)
  DBuf<int64_t> goff_;
  DBuf<int32_t> gidx_;
  DBuf<double> gw_;
  // tasks of the matvec; down_nov groups leave the V-list to the M2L kernels
  TaskSet fwd_;
  DBuf<double> partial64_;
  DBuf<float> partial32_;
  M2LPlan m2l_;
  bool tensor_m2l_ = false;
  FftM2L fft_;
  bool fft_m2l_ = false;
  DBuf<int32_t> lvl_nodes_;
  DBuf<int32_t> roots_;
  std::vector<int64_t> lvl_off_;
  // operators: per (tree, level), uppot = A * check (A = K_up^-1 or its
  // Tikhonov form), downpot = A^T * check.  A depends only on the box width,
  // so trees and levels of equal width share one operator.
  DBuf<double> ops_;
  int nops_ = 0;
  std::vector<double> op_w_;          // box width of each operator
  std::vector<int> op_of_;            // (group * (maxl + 1) + level) -> operator
  DBuf<C2ETile> dn_tiles_;  // per level, tiles of nodes sharing an operator
  std::vector<C2ETile> dn_tiles_host_;
  DBuf<double> blas_x_, blas_y_;  // gathered check vectors and products of the library-GEMM C2E form
  // check-to-equivalent products on the tensor cores (int8 digits, FP64
  // accuracy; c2e_tc.h), as library DGEMMs or on the FP64 SIMT units
  C2ETcPlan c2e_tc_;
  // 2 library DGEMM (the default), 1 tensor cores where available, 0 SIMT,
  // -1 the fastest as timed by autotune (SIMT until then)
  int c2e_mode_ = 2;
  int auto_form_ = 0;  // the form autotune chose for mode -1 (0, 1 or 2)
  bool tc_c2e() const { return (c2e_mode_ < 0 ? auto_form_ == 1 : c2e_mode_ == 1) && c2e_tc_.ready; }
  bool blas_c2e() const { return t_->groups() == 1 && (c2e_mode_ < 0 ? auto_form_ == 2 : c2e_mode_ == 2); }
  void tune_c2e(int R);
  std::pair<double, double> autotune_tiles(int nrhs);
  void build_tc_digits();
  void reserve_tc_scratch();
  template <typename Real>
  void c2e(int trans, const C2ETile* tiles, const C2ETile* tiles_host, int ntiles, const int32_t* nodes,
           const Real* check, Real* dst, int64_t base, int R, float* m2l_dst, int NP, const int* nact);
  // the library-GEMM form: per run of tiles with one operator, gather the
  // check vectors, one cuBLAS DGEMM, scatter the products
  template <typename Real>
  void c2e_blas(int trans, const C2ETile* tiles_host, int ntiles, const int32_t* nodes, const Real* check, Real* dst,
                int64_t base, int R, float* m2l_dst, int NP);
  void reserve_blas_scratch();
  // folded M2M / L2L: per operator (box width w), U = A(w) [M2M_0 .. M2M_7]
  // (3P x 8 * 3P; M2M_k: child k's up surface -> the down surface of its
  // parent of width w) and D = [A(w)^T L2L_0; ..; A(w)^T L2L_7] (8 * 3P x 3P;
  // L2L_k: the down surface of the parent of width 2w -> child k's up
  // surface), child k = child0 + k; over the non-leaf nodes of each level
  double setup_ms_[NNK_SETUP_COUNT] = {};
  bool fold_ok_ = false;  // the tree and the operators allow folding
  bool fold_lists_ok_ = false;
  std::array<int, 8> fold_pos_{};  // position code (x * 4 + y * 2 + z) of child k in its parent
  int fold_on_ = 0;       // the caller's choice (set_fold)
  DBuf<double> fold_up_, fold_dn_;
  DBuf<int32_t> fpar_, fch_;  // non-leaf nodes by level, and their first children
  std::vector<int64_t> fpar_off_;
  DBuf<C2ETile> fup_tiles_, fdn_tiles_;
  std::vector<C2ETile> fup_tiles_host_, fdn_tiles_host_;
  std::vector<int64_t> fup_toff_, fdn_toff_;
  void build_fold_lists();
  // M2M and L2L as products with their kernel matrices, not folded: per
  // operator (box width w) [M2M_0 .. M2M_7] (3P x 8 * 3P) from the 8
  // children's up-equivalent densities to the parent's up check, and
  // [L2L_0; ..; L2L_7] (8 * 3P x 3P) from the parent's down-equivalent
  // density to the 8 children's down checks, each one library DGEMM per
  // level on gathered densities.  The check potentials are the pair sums'
  // to FP64 rounding, so the exact inverses allow it (unlike folding).
  DBuf<double> m2m_ops_, l2l_ops_;
  bool m2m_ok_ = false;  // the operators are built
  int m2m_on_ = 2;       // the caller's choice (set_m2m_form): 2 M2M and L2L, 1 M2M
  void build_m2m_operators();
  // kernel matrices M2M_k (dM: k-th 3P x 3P block at k (3P)^2) and L2L_k (dL)
  // of operator o, on the device
  void kernel_blocks(int o, const double* surf, double* dM, double* dL);
  std::vector<double> fold_surfaces() const;
  bool m2m_products() const { return m2m_ok_ && m2m_on_ > 0 && t_->groups() == 1; }
  bool l2l_products() const { return m2m_products() && m2m_on_ == 2; }
  // dst(out node) [+]= op * src(in node) over runs of tiles sharing an
  // operator (op: M x Kd column-major, op_stride apart): gather, one cuBLAS
  // DGEMM per run, scatter
  template <typename Real>
  void node_gemm_blas(const double* ops, size_t op_stride, int M, int Kd, int trans, const C2ETile* tiles_host,
                      int ntiles, const int32_t* out_nodes, const int32_t* in_nodes, const Real* src, Real* dst,
                      int64_t base, int R, int accumulate, float* m2l_dst, int NP);
  void build_fold_operators(bool force);
  DBuf<double> c2e_part_;   // K-split partial sums of the small C2E launches
  std::vector<int64_t> dn_toff_;
  // transpose (built on first use): tasks with inverted lists, unified
  // points [sorted targets | surfaces], identity gather of the targets and
  // the entry -> potential-row sums of the scatter
  bool adj_ready_ = false;
  bool v_symmetric_ = false;
  TaskSet adj_;
  Csr inv_U_, inv_V_, inv_W_, inv_X_;
  DBuf<double> apos64_, astr64_, avel64_;
  DBuf<float> apos32_, astr32_, avel32_;
  DBuf<int64_t> agoff_;
  DBuf<int32_t> agidx_;
  DBuf<double> agw_;
  DBuf<int64_t> row_off_;   // per potential row: its (entry, weight) pairs
  DBuf<int64_t> row_ent_;
  DBuf<double> row_w_;
  DBuf<int64_t> org_off_;   // per source origin: its entries
  DBuf<int64_t> org_ent_;
  int64_t norigin_ = 0;
  // work buffers
  DBuf<double> check64_, vel64_;
  DBuf<float> check32_, vel32_;
  // reduced (leaf block) solve: LU of S_leaf*NN_leaf per target leaf, padded
  bool reduced_ready_ = false;
  int rdim_ = 0;                 // padded block size (3 * max leaf targets)
  DBuf<double> rlu_;             // nleaf * rdim * rdim (column-major per block)
  DBuf<int> rpiv_, rinfo_;
  DBuf<double*> rptr_;
  DBuf<double> rrhs_;
  DBuf<double*> rrhsptr_;
  DBuf<double> rmat_;            // unfactored blocks for reduced_apply
  bool rinv_ready_ = false;
  DBuf<double> rinv_;            // explicit inverses of the blocks (reduced_solve_inv)
  DBuf<double*> rinvptr_;
  DBuf<double> rsol_;            // nleaf * rdim: block solutions
  std::vector<int32_t> rleaf_;   // target leaves in order
  DBuf<int32_t> rleaf_d_;
  DBuf<int64_t> rts_;            // tgt_start on the device
  void* blas_ = nullptr;         // cublasHandle_t for the batched leaf solves
  nnk_fmm_stats stats_{};
  template <typename F> void phase(int ph, F&& launch);
  struct PhaseRec { int ph; cudaEvent_t a, b; };
  bool prof_ = false;
  std::vector<PhaseRec> recs_;
  std::vector<cudaEvent_t> pool_;
  int64_t launches_[NNK_NUM_PHASES] = {0};
  cudaEvent_t event();
  std::unique_ptr<Fmm> sparse_;
  uint64_t version_ = 0;
  void bump_version();
  // tree mask of the matvec (forests only): per tree, per node (expanded on
  // the device), and the leaf of each sorted target
  DBuf<int32_t> tree_on_, node_on_, node_tree_, tgt_leaf_;
  std::vector<int32_t> tree_on_host_;
  const int* nact() const { return node_on_.p; }
};

}  // namespace nnk
