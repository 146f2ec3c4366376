// Rigid-body mobility system on one FMM (Mobility/*.m):
//   [ S*NN  BT ] [ f     ]   [ u_slip - u_bg ]
//   [ B     0  ] [ U; Om ] = [ F; M          ]
// Vector layout (mobilityProblem.m:45-46, MobilityMatrixMulti.m:19-36):
//   [ f_x(1..N) f_y(1..N) f_z(1..N) | U_x(1..nb) U_y U_z | Om_x(1..nb) Om_y Om_z ].
#pragma once
#include <memory>
#include <vector>

#include "common.h"
#include "fmm.h"

namespace nnk {

class Mobility {
 public:
  Mobility(Fmm* fmm, int nbodies, const int64_t* body_start, const int64_t* fine_start,
           const double* rel_points, const double* rel_fine);
  ~Mobility();
  Mobility(const Mobility&) = delete;
  Mobility& operator=(const Mobility&) = delete;
  // Replay each matvec (per FMM it runs on) from a CUDA graph captured on
  // first use and again after the FMM changed (default on; off launches
  // kernel by kernel).
  void use_graphs(bool on);
  int64_t size() const { return 3 * N_ + 6 * (int64_t)nb_; }
  void apply(const double* x, double* y);   // mobilityMatrixMulti.m:17-36
  void apply_with(Fmm* f, const double* x, double* y);
  void apply_raw(Fmm* f, const double* x, double* y);
  // A^T = [F^T B^T; BT^T 0], F the FMM block (exact transpose of the passes)
  void apply_adjoint(const double* x, double* y);
  void apply_adjoint_with(Fmm* f, const double* x, double* y);
  // GMRES on A^T (the adjoint solve of a gradient), refined like solve
  void solve_adjoint(const double* rhs, double* x, const nnk_solve_params& sp, nnk_solve_info& info);
  // -lam^T (dA/dpositions) z: gX (N x 3, force points), gY (Q x 3, fine
  // points in NEAREST mode, else null), device pointers; z the solution of
  // A z = b and lam that of A^T lam = dL/dz.
  void grad_positions(const double* z, const double* lam, double* gX, double* gY);
  void precon(const double* x, double* y);  // MobilityPrecon.m:17-40
  void solve(const double* rhs, double* x, const nnk_solve_params& sp, bool precondition, nnk_solve_info& info);
  // Mixed-precision iterative refinement: inner GMRES on this (mixed) FMM,
  // outer residual b - A x with `fp64` (an FP64 FMM on the same tree).
  void set_refinement(Fmm* fp64, int max_outer, double inner_tol);
  void solve_plain(const double* rhs, double* x, const nnk_solve_params& sp, bool precondition,
                   nnk_solve_info& info);
  void refine(bool adjoint, const double* rhs, double* x, const nnk_solve_params& sp, bool precondition,
              nnk_solve_info& info);
  DBuf<double> io_in, io_out;

 private:
  void body_sums(const double* f, double* out6);          // B * f
  void body_sums_t(const double* z6, double* f, double a); // f = a*f + B^T z
  void bt_apply(const double* uo, double* y);              // y += BT * [U;Om]
  void btt_apply(const double* v, double* out6);           // BT^T v
  void small_solve(const DBuf<double>& inv, const double* in6, double* out6);  // per body 6x6 blocks

  Fmm* fmm_;
  Fmm* ref64_ = nullptr;
  int ref_outer_ = 0;
  double ref_inner_tol_ = 1e-4;
  nnk_ctx* ctx_;
  int nb_;
  int64_t N_;
  std::vector<int64_t> bstart_;
  DBuf<int32_t> body_of_;   // per point: body or -1 (boundary)
  DBuf<int64_t> bstart_d_;
  DBuf<double> xrel_;       // per point rotated untranslated position (BT, Swimmers.m:177-189)
  DBuf<double> xm_;         // per point torque arm: sum_q NN(q,n) X_q (NEAREST) or xrel (genMatrixComponets.m:69-75)
  DBuf<double> af_;         // per point force weight: column sum of NN (NEAREST) or 1 (:208-209, :228)
  std::vector<double> a1inv_, a2inv_;  // per body 6x6 inverses of B B^T and BT^T BT
  DBuf<double> a1inv_d_, a2inv_d_;     // the same on the device
  std::vector<int32_t> hbody_;         // per point: body or -1 (host copy)
  std::vector<int64_t> fstart_;        // per body: first fine row (NEAREST)
  DBuf<double> t6a_, t6b_, tv_, tv2_, tv3_;
  struct Graph {
    Fmm* f;
    uint64_t version;
    cudaGraphExec_t exec;
  };
  std::vector<Graph> graphs_;
  bool graphs_on_ = true;
  DBuf<double> gin_, gout_;  // the captured matvec's input and output
};

}  // namespace nnk
