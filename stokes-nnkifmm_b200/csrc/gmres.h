// Device GMRES (FP64) with MATLAB gmres semantics:
//   x0 = 0, stop when ||b - A x|| / ||b|| <= tol, at most maxit inner steps,
//   restart = 0 means unrestarted (gmres(A,b,[],tol,maxit)).
// The Krylov basis lives on the device; Arnoldi uses classical Gram-Schmidt
// applied twice (CGS2) in FP64; the Givens least-squares update runs on the
// host on the (m+1) x m Hessenberg matrix.  As MATLAB does, convergence of
// the recurrence residual is confirmed with an explicit residual b - A x.
#pragma once
#include <functional>

#include "common.h"

namespace nnk {

class Gmres {
 public:
  Gmres(nnk_ctx* ctx, int64_t n);
  using Op = std::function<void(const double* in, double* out)>;
  // Solves op(x) = b.  `post` (may be null) is applied to the final x, e.g.
  // the right preconditioner of mobilityProblem.m:48-55.
  void solve(const Op& op, const Op* post, const double* b, double* x, const nnk_solve_params& sp,
             nnk_solve_info& info);

 private:
  nnk_ctx* ctx_;
  int64_t n_;
  DBuf<double> V_, w_, r_, tmp_, h_;
};

// Device vector helpers shared with the mobility code.
double dev_dot(nnk_ctx* ctx, const double* a, const double* b, int64_t n, DBuf<double>& scratch);
void dev_axpby(nnk_ctx* ctx, double a, const double* x, double b, const double* y, double* out, int64_t n);

}  // namespace nnk
