// Batched rigid-body mobility solves: many independent bodies, several
// right-hand sides each, solved together on one GPU.
//
// The bodies' trees are merged into one forest (merge_forest), so a single
// FMM pass evaluates every body -- one launch per pass step for the whole
// batch instead of one per body -- and the pair kernels evaluate the R
// right-hand sides of a body together, sharing the geometry of each pair.
// Every (body, right-hand side) is its own linear system (a "system"):
//   [ S NN  BT ] [ f      ]   [ rhs_f  ]
//   [ B     0  ] [ U ; Om ] = [ F ; M  ]
// (mobilityMatrixMulti.m:17-36 for one free swimmer per body).  The batch
// vector is the concatenation of the systems, system s = b * R + r, each laid
// out as [f_x(1..N_b) f_y f_z | U_x U_y U_z | Om_x Om_y Om_z]
// (mobilityProblem.m:45-46).  GMRES runs per system (own Krylov space,
// Hessenberg matrix and stopping test, as separate gmres calls would), with
// the systems advancing in lockstep so that each step is one batched matvec.
#pragma once
#include <functional>
#include <memory>
#include <vector>

#include "common.h"
#include "fmm.h"

namespace nnk {

struct BatchBody {
  const HostTree* tree;      // tree of the body's force points (potentials == targets)
  const double* rel_points;  // N x 3 rotated, untranslated force points (Swimmers.m:177-189)
  const double* rel_fine;    // Q x 3 rotated, untranslated fine points (NEAREST), else null
};

// GMRES over independent segments [off[s], off[s+1]) of one vector: one
// Krylov space per segment, every step one call of `op` for all segments.
class SegGmres {
 public:
  SegGmres(nnk_ctx* ctx, const std::vector<int64_t>& off);
  using Op = std::function<void(const double* in, double* out)>;
  // x = 0 start; segments with solve[s] == 0 get x_s = 0 and no iterations.
  // confirm = false skips the closing explicit residual (the caller forms it,
  // as iterative refinement does) and reports the recurrence's estimate.
  void solve(const Op& op, const double* b, double* x, const std::vector<double>& tol, int maxit, int restart,
             const std::vector<char>& solve, std::vector<nnk_solve_info>& info, bool confirm = true);
  int64_t matvecs() const { return matvecs_; }
  std::vector<double> norms(const double* v);  // ||v_s|| per segment
  // Called with the segments whose op outputs the next calls use (1) and
  // those whose outputs are ignored (0), before the calls that change; with
  // all 1 when solve returns.  The op may skip the work of the 0 segments,
  // provided their outputs stay finite.
  std::function<void(const std::vector<char>& active)> on_active;

 private:
  struct Chunk {
    long long start;
    int len;
    int seg;
  };
  void seg_dots(const double* V, int nvec, const double* w, double* h, int ldh, const double* active = nullptr);
  nnk_ctx* ctx_;
  std::vector<int64_t> off_;
  int S_;
  int64_t n_;
  DBuf<Chunk> chunks_;
  DBuf<int32_t> cfirst_;  // per segment: first chunk (S + 1)
  DBuf<double> part_;     // per (vector, chunk) partial dot products
  int nchunks_ = 0;
  int64_t matvecs_ = 0;
};

class BatchMobility {
 public:
  BatchMobility(nnk_ctx* ctx, const std::vector<BatchBody>& bodies, const FmmParams& fp, int nrhs);
  ~BatchMobility();
  int systems() const { return S_; }
  int bodies() const { return B_; }
  int64_t size() const { return n_; }
  const std::vector<int64_t>& offsets() const { return off_; }
  void apply(const double* x, double* y);
  void solve(const double* rhs, double* x, const nnk_solve_params& sp, nnk_solve_info* info);
  // Mixed-precision refinement: outer residuals with an FP64 FMM on the same
  // forest (same Tikhonov weight), inner GMRES on this FMM.
  void set_refinement(bool fp64, int max_outer, double inner_tol);
  Fmm& fmm() { return *fmm_; }
  Fmm* ref64() { return ref64_.get(); }
  // Replay each FMM's matvec (all bodies, all right-hand sides, B and BT
  // blocks: about 50 launches) from a CUDA graph captured on first use.
  void set_deflation(bool on) { deflate_ = on; }
  void use_graphs(bool on);
  int64_t matvecs() const { return matvecs_; }

 private:
  void apply_with(Fmm& f, const double* x, double* y);
  void apply_raw(Fmm& f, const double* x, double* y);
  std::vector<char> body_flags(const std::vector<char>& systems) const;  // any system of the body set
  bool deflate_ = true;
  void solve_plain(const double* rhs, double* x, const nnk_solve_params& sp, const std::vector<double>& tol,
                   const std::vector<char>& act, std::vector<nnk_solve_info>& info);

  nnk_ctx* ctx_;
  int B_ = 0, R_ = 1, S_ = 0;
  int64_t n_ = 0, Nt_ = 0;           // batch vector length, force points of all bodies
  std::vector<int64_t> off_;         // per system: first entry (S + 1)
  std::vector<int64_t> bN_;          // per body: force points
  HostTree forest_;
  std::unique_ptr<Fmm> fmm_, ref64_;
  FmmParams fp_;
  int ref_outer_ = 0;
  double ref_inner_tol_ = 1e-4;
  IoMap io_;
  DBuf<long long> io_off_, io_rstr_;
  DBuf<int> io_cstr_;
  DBuf<int> row_body_;      // per force point of the forest: body
  DBuf<int> row_local_;     // per force point: index inside its body
  DBuf<long long> sys_off_; // per system: first entry
  DBuf<int> sys_n_;         // per system: force points of its body
  DBuf<double> xrel_, xm_, af_;  // per force point (forest order)
  DBuf<long long> body_row0_;  // per body: first force point in forest order (B + 1)
  bool graphs_on_ = true;
  cudaGraphExec_t graph_[2] = {nullptr, nullptr};  // matvec of fmm_ and of ref64_
  uint64_t graph_version_[2] = {0, 0};             // the FMM version each was captured at
  DBuf<double> gin_, gout_;                        // the captured matvec's input and output
  int64_t matvecs_ = 0;
};

}  // namespace nnk
