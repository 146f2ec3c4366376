// Mobility matvec, block preconditioner and GMRES driver (see mobility.h).
#include <cmath>

#include "gmres.h"
#include "mobility.h"

namespace nnk {

namespace {

__device__ __forceinline__ void cross3(const double* a, const double* b, double* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

// y_c(n) += -U_b,c + (x_n x Om_b)_c : BT*[U;Om] (genMatrixComponets.m:34-50)
// out6 = per body its 6x6 inverse times in6 (layout [U_x(1..nb) U_y U_z Om_x Om_y Om_z])
__global__ void small_solve_kernel(int nb, const double* __restrict__ inv, const double* __restrict__ in6,
                                   double* __restrict__ out6) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= 6 * nb) return;
  const int b = g / 6, i = g % 6;
  double s = 0;
  for (int k = 0; k < 6; ++k) s += inv[36 * b + i * 6 + k] * in6[k * nb + b];
  out6[i * nb + b] = s;
}

__global__ void bt_kernel(int64_t N, int nb, const int* __restrict__ body, const double* __restrict__ xrel,
                          const double* __restrict__ uo, double* __restrict__ y) {
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const int b = body[n];
  if (b < 0) return;
  const double U[3] = {uo[b], uo[nb + b], uo[2 * nb + b]};
  const double O[3] = {uo[3 * nb + b], uo[4 * nb + b], uo[5 * nb + b]};
  const double x[3] = {xrel[3 * n], xrel[3 * n + 1], xrel[3 * n + 2]};
  double c[3];
  cross3(x, O, c);
  for (int k = 0; k < 3; ++k) y[k * N + n] += -U[k] + c[k];
}

// out = B * f: F_b = sum af_n f_n, M_b = sum xm_n x f_n (genMatrixComponets.m:53-95)
// mode 1: out = BT^T v: [-sum v_n ; sum v_n x xrel_n]
__global__ void body_reduce_kernel(int64_t N, int nb, const int64_t* __restrict__ bstart,
                                   const double* __restrict__ w, const double* __restrict__ arm,
                                   const double* __restrict__ f, double* __restrict__ out, int mode) {
  const int b = blockIdx.x;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int64_t n = bstart[b] + threadIdx.x; n < bstart[b + 1]; n += blockDim.x) {
    const double v[3] = {f[n], f[N + n], f[2 * N + n]};
    const double x[3] = {arm[3 * n], arm[3 * n + 1], arm[3 * n + 2]};
    double c[3];
    if (mode == 0) {
      const double a = w[n];
      cross3(x, v, c);
      acc[0] += a * v[0];
      acc[1] += a * v[1];
      acc[2] += a * v[2];
    } else {
      cross3(v, x, c);
      acc[0] -= v[0];
      acc[1] -= v[1];
      acc[2] -= v[2];
    }
    acc[3] += c[0];
    acc[4] += c[1];
    acc[5] += c[2];
  }
  __shared__ double red[6][256];
  for (int k = 0; k < 6; ++k) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int k = 0; k < 6; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x < 6) out[threadIdx.x * nb + b] = red[threadIdx.x][0];
}

// f = a f + B^T z: af_n z_F,b + z_M,b x xm_n on body points
__global__ void bt_transpose_kernel(int64_t N, int nb, const int* __restrict__ body, const double* __restrict__ af,
                                    const double* __restrict__ xm, const double* __restrict__ z,
                                    double* __restrict__ f, double a) {
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const int b = body[n];
  double add[3] = {0, 0, 0};
  if (b >= 0) {
    const double F[3] = {z[b], z[nb + b], z[2 * nb + b]};
    const double M[3] = {z[3 * nb + b], z[4 * nb + b], z[5 * nb + b]};
    const double x[3] = {xm[3 * n], xm[3 * n + 1], xm[3 * n + 2]};
    double c[3];
    cross3(M, x, c);
    for (int k = 0; k < 3; ++k) add[k] = af[n] * F[k] + c[k];
  }
  for (int k = 0; k < 3; ++k) f[k * N + n] = (a == 0.0 ? 0.0 : a * f[k * N + n]) + add[k];
}

bool invert6(const double* A, double* Ai) {
  double M[6][12];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 12; ++j) M[i][j] = j < 6 ? A[i * 6 + j] : (j - 6 == i ? 1.0 : 0.0);
  for (int c = 0; c < 6; ++c) {
    int p = c;
    for (int r = c + 1; r < 6; ++r)
      if (std::fabs(M[r][c]) > std::fabs(M[p][c])) p = r;
    if (M[p][c] == 0.0) return false;
    if (p != c)
      for (int j = 0; j < 12; ++j) std::swap(M[p][j], M[c][j]);
    const double d = M[c][c];
    for (int j = 0; j < 12; ++j) M[c][j] /= d;
    for (int r = 0; r < 6; ++r)
      if (r != c) {
        const double fct = M[r][c];
        for (int j = 0; j < 12; ++j) M[r][j] -= fct * M[c][j];
      }
  }
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) Ai[i * 6 + j] = M[i][6 + j];
  return true;
}

inline void skew(const double* x, double* S) {  // S v = x cross v
  S[0] = 0; S[1] = -x[2]; S[2] = x[1];
  S[3] = x[2]; S[4] = 0; S[5] = -x[0];
  S[6] = -x[1]; S[7] = x[0]; S[8] = 0;
}

}  // namespace

Mobility::Mobility(Fmm* fmm, int nbodies, const int64_t* body_start, const int64_t* fine_start,
                   const double* rel_points, const double* rel_fine)
    : fmm_(fmm), ctx_(fmm->ctx()), nb_(nbodies) {
  const HostTree& t = fmm->tree();
  if (t.n_pot != t.n_tgt || t.n_pot != t.n) throw Error(NNK_E_ARG, "mobility needs potentials == targets");
  N_ = t.n_tgt;
  bstart_.assign(body_start, body_start + nb_ + 1);
  if (bstart_[0] != 0 || bstart_[nb_] > N_) throw Error(NNK_E_ARG, "bad body_start");
  for (int b = 0; b < nb_; ++b)
    if (bstart_[b + 1] < bstart_[b]) throw Error(NNK_E_ARG, "bad body_start");
  const int64_t Nsw = bstart_[nb_];
  if (Nsw > 0 && !rel_points) throw Error(NNK_E_ARG, "rel_points missing");
  if (t.params.nearest && fine_start) {
    if (fine_start[0] != 0 || fine_start[nb_] > t.q) throw Error(NNK_E_ARG, "bad fine_start");
    for (int b = 0; b < nb_; ++b)
      if (fine_start[b + 1] < fine_start[b]) throw Error(NNK_E_ARG, "bad fine_start");
  }
  std::vector<int32_t> body(N_, -1);
  for (int b = 0; b < nb_; ++b)
    for (int64_t n = bstart_[b]; n < bstart_[b + 1]; ++n) body[n] = b;
  std::vector<double> xrel(3 * N_, 0.0), xm(3 * N_, 0.0), af(N_, 0.0);
  for (int64_t n = 0; n < Nsw; ++n)
    for (int d = 0; d < 3; ++d) xrel[3 * n + d] = rel_points[3 * n + d];
  if (t.params.nearest) {
    if (!fine_start || !rel_fine) throw Error(NNK_E_ARG, "NEAREST mobility needs fine_start and rel_fine");
    const int64_t Qsw = fine_start[nb_];
    // af = sum(NN(1:Q,cols),1); pointMap = finePoints' * NN over swimmer fine rows
    for (int64_t r = 0; r < Qsw && r < t.q; ++r)
      for (int64_t k = t.nn_rowptr[r]; k < t.nn_rowptr[r + 1]; ++k) {
        const int64_t c = t.nn_col[k];
        if (c >= Nsw) continue;
        const double w = t.nn_val[k];
        af[c] += w;
        for (int d = 0; d < 3; ++d) xm[3 * c + d] += w * rel_fine[3 * r + d];
      }
  } else {
    for (int64_t n = 0; n < Nsw; ++n) {
      af[n] = 1.0;
      for (int d = 0; d < 3; ++d) xm[3 * n + d] = xrel[3 * n + d];
    }
  }
  // A1 = B B^T and A2 = BT^T BT per body (genMatrixComponets.m:99-100)
  a1inv_.assign(36 * (size_t)nb_, 0.0);
  a2inv_.assign(36 * (size_t)nb_, 0.0);
  for (int b = 0; b < nb_; ++b) {
    double A1[36] = {0}, A2[36] = {0};
    for (int64_t n = bstart_[b]; n < bstart_[b + 1]; ++n) {
      double X[9], R[9];
      skew(&xm[3 * n], X);
      skew(&xrel[3 * n], R);
      // B_n = [af I ; X]  (6x3)
      double Bn[18];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          Bn[i * 3 + j] = (i == j) ? af[n] : 0.0;
          Bn[(3 + i) * 3 + j] = X[i * 3 + j];
        }
      // BT_n = [-I , R]  (3x6)
      double Tn[18];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          Tn[i * 6 + j] = (i == j) ? -1.0 : 0.0;
          Tn[i * 6 + 3 + j] = R[i * 3 + j];
        }
      for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
          double s1 = 0, s2 = 0;
          for (int k = 0; k < 3; ++k) {
            s1 += Bn[i * 3 + k] * Bn[j * 3 + k];
            s2 += Tn[k * 6 + i] * Tn[k * 6 + j];
          }
          A1[i * 6 + j] += s1;
          A2[i * 6 + j] += s2;
        }
    }
    if (!invert6(A1, &a1inv_[36 * b]) || !invert6(A2, &a2inv_[36 * b]))
      throw Error(NNK_E_ARG, "singular body block in B*B' or BT'*BT (empty body?)");
  }
  cudaStream_t st = ctx_->stream;
  hbody_ = body;
  if (t.params.nearest && fine_start) fstart_.assign(fine_start, fine_start + nb_ + 1);
  body_of_.upload(body, st);
  bstart_d_.upload(bstart_, st);
  xrel_.upload(xrel, st);
  xm_.upload(xm, st);
  af_.upload(af, st);
  t6a_.alloc(6 * (size_t)std::max(nb_, 1));
  t6b_.alloc(6 * (size_t)std::max(nb_, 1));
  tv_.alloc(3 * N_);
  tv2_.alloc(3 * N_);
  tv3_.alloc(3 * N_);
  a1inv_d_.upload(a1inv_, st);
  a2inv_d_.upload(a2inv_, st);
  NNK_CUDA(cudaStreamSynchronize(st));
}

void Mobility::body_sums(const double* f, double* out6) {
  if (nb_ == 0) return;
  body_reduce_kernel<<<nb_, 256, 0, ctx_->stream>>>(N_, nb_, bstart_d_.p, af_.p, xm_.p, f, out6, 0);
  NNK_CHECK_LAUNCH();
}

void Mobility::btt_apply(const double* v, double* out6) {
  if (nb_ == 0) return;
  body_reduce_kernel<<<nb_, 256, 0, ctx_->stream>>>(N_, nb_, bstart_d_.p, af_.p, xrel_.p, v, out6, 1);
  NNK_CHECK_LAUNCH();
}

void Mobility::bt_apply(const double* uo, double* y) {
  if (nb_ == 0) return;
  bt_kernel<<<(unsigned)((N_ + 255) / 256), 256, 0, ctx_->stream>>>(N_, nb_, body_of_.p, xrel_.p, uo, y);
  NNK_CHECK_LAUNCH();
}

void Mobility::body_sums_t(const double* z6, double* f, double a) {
  bt_transpose_kernel<<<(unsigned)((N_ + 255) / 256), 256, 0, ctx_->stream>>>(N_, nb_, body_of_.p, af_.p, xm_.p,
                                                                           z6, f, a);
  NNK_CHECK_LAUNCH();
}

void Mobility::small_solve(const DBuf<double>& inv, const double* in6, double* out6) {
  if (nb_ == 0) return;
  small_solve_kernel<<<(6 * nb_ + 127) / 128, 128, 0, ctx_->stream>>>(nb_, inv.p, in6, out6);
  NNK_CHECK_LAUNCH();
}

void Mobility::apply(const double* x, double* y) { apply_with(fmm_, x, y); }

Mobility::~Mobility() {
  for (auto& g : graphs_)
    if (g.exec) cudaGraphExecDestroy(g.exec);
}

void Mobility::use_graphs(bool on) {
  graphs_on_ = on;
  for (auto& g : graphs_)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  graphs_.clear();
}

void Mobility::apply_raw(Fmm* f, const double* x, double* y) {
  // b(1:3N) = FMM(f) + BT*UOm ; b(3N+1:end) = B*f
  f->apply(x, y, NNK_LAYOUT_BLOCKED, 1);
  bt_apply(x + 3 * N_, y);
  body_sums(x, y + 3 * N_);
}

// A small system's matvec is some 50 short launches: replayed from a graph
// it costs one launch.  The graph reads and writes fixed buffers; a changed
// FMM (new eps, new tiles) is captured again.
void Mobility::apply_with(Fmm* f, const double* x, double* y) {
  cudaStream_t st = ctx_->stream;
  if (!graphs_on_ || f->profiling() || st == nullptr) {  // the legacy default stream cannot be captured
    apply_raw(f, x, y);
    return;
  }
  const int64_t n = size();
  if (!gin_.p) {
    gin_.alloc(n);
    gout_.alloc(n);
  }
  Graph* g = nullptr;
  for (auto& e : graphs_)
    if (e.f == f) g = &e;
  if (g && g->version != f->version()) {
    cudaGraphExecDestroy(g->exec);
    g->exec = nullptr;
  }
  if (!g) {
    graphs_.push_back(Graph{f, 0, nullptr});
    g = &graphs_.back();
  }
  if (!g->exec) {
    NNK_CUDA(cudaStreamSynchronize(st));
    NNK_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaGraph_t graph = nullptr;
    try {
      apply_raw(f, gin_.p, gout_.p);
    } catch (...) {
      cudaStreamEndCapture(st, &graph);
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
      throw;
    }
    NNK_CUDA(cudaStreamEndCapture(st, &graph));
    const cudaError_t e = cudaGraphInstantiate(&g->exec, graph, 0);
    cudaGraphDestroy(graph);
    NNK_CUDA(e);
    g->version = f->version();
  }
  NNK_CUDA(cudaMemcpyAsync(gin_.p, x, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  NNK_CUDA(cudaGraphLaunch(g->exec, st));
  NNK_CUDA(cudaMemcpyAsync(y, gout_.p, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
}

void Mobility::set_refinement(Fmm* fp64, int max_outer, double inner_tol) {
  if (fp64 && &fp64->tree() != &fmm_->tree()) throw Error(NNK_E_ARG, "refinement FMM must share the tree");
  ref64_ = fp64;
  ref_outer_ = max_outer > 0 ? max_outer : 10;
  ref_inner_tol_ = inner_tol > 0 ? inner_tol : 1e-4;
}

void Mobility::precon(const double* x, double* y) {
  cudaStream_t st = ctx_->stream;
  const double* f = x;
  const double* uo = x + 3 * N_;
  // b_f = reducedSolve(f), through the leaf blocks' explicit inverses (a
  // preconditioner needs no backward-stable solve; one batched product is
  // several times faster than the batched triangular solves)
  fmm_->reduced_solve_inv(f, y, NNK_LAYOUT_BLOCKED);
  if (nb_ > 0) {
    // out = -A2 \ (BT' * computeVelSparse(B' * (A1 \ UOm)))
    small_solve(a1inv_d_, uo, t6a_.p);
    body_sums_t(t6a_.p, tv_.p, 0.0);
    fmm_->sparse().apply(tv_.p, tv2_.p, NNK_LAYOUT_BLOCKED, 1);
    btt_apply(tv2_.p, t6b_.p);
    small_solve(a2inv_d_, t6b_.p, y + 3 * N_);
    dev_axpby(ctx_, -1.0, y + 3 * N_, 0.0, nullptr, y + 3 * N_, 6 * nb_);
    // b_f -= reducedSolve(BT * out)
    NNK_CUDA(cudaMemsetAsync(tv_.p, 0, 3 * N_ * sizeof(double), st));
    bt_apply(y + 3 * N_, tv_.p);
    fmm_->reduced_solve_inv(tv_.p, tv3_.p, NNK_LAYOUT_BLOCKED);
    dev_axpby(ctx_, 1.0, y, -1.0, tv3_.p, y, 3 * N_);
  }
}

void Mobility::solve(const double* rhs, double* x, const nnk_solve_params& sp, bool precondition,
                     nnk_solve_info& info) {
  if (ref64_) {
    refine(false, rhs, x, sp, precondition, info);
    return;
  }
  solve_plain(rhs, x, sp, precondition, info);
}

void Mobility::solve_adjoint(const double* rhs, double* x, const nnk_solve_params& sp, nnk_solve_info& info) {
  if (ref64_) {
    refine(true, rhs, x, sp, false, info);
    return;
  }
  Gmres g(ctx_, size());
  Gmres::Op op = [&](const double* in, double* out) { apply_adjoint(in, out); };
  g.solve(op, nullptr, rhs, x, sp, info);
}

// x = 0, r = b; repeat: A_mixed d ~= r (GMRES), x += d, r = b - A_fp64 x
// (A^T for the adjoint)
void Mobility::refine(bool adjoint, const double* rhs, double* x, const nnk_solve_params& sp, bool precondition,
                      nnk_solve_info& info) {
  const int64_t n = size();
  DBuf<double> r(n), d(n), ax(n), scratch(1);
  NNK_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), ctx_->stream));
  NNK_CUDA(cudaMemcpyAsync(r.p, rhs, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx_->stream));
  const double nb = std::sqrt(dev_dot(ctx_, rhs, rhs, n, scratch));
  const double tol = sp.tol > 0 ? sp.tol : 1e-6;
  info = nnk_solve_info{0, 0, 0.0};
  if (nb == 0.0) return;
  double relres = 1.0;
  for (int outer = 0; outer < ref_outer_; ++outer) {
    nnk_solve_params in = sp;
    const double target = tol / relres;  // inner tolerance relative to ||r||
    in.tol = std::max(ref_inner_tol_, std::min(0.5, target));
    nnk_solve_info ii{};
    if (adjoint) {
      Gmres g(ctx_, n);
      Gmres::Op op = [&](const double* a, double* b) { apply_adjoint(a, b); };
      g.solve(op, nullptr, r.p, d.p, in, ii);
    } else {
      solve_plain(r.p, d.p, in, precondition, ii);
    }
    info.iters += ii.iters;
    dev_axpby(ctx_, 1.0, x, 1.0, d.p, x, n);
    if (adjoint) apply_adjoint_with(ref64_, x, ax.p);
    else apply_with(ref64_, x, ax.p);
    dev_axpby(ctx_, 1.0, rhs, -1.0, ax.p, r.p, n);
    relres = std::sqrt(dev_dot(ctx_, r.p, r.p, n, scratch)) / nb;
    if (relres <= tol) break;
  }
  info.relres = relres;
  info.flag = relres <= tol ? 0 : 1;
}

void Mobility::apply_adjoint(const double* x, double* y) { apply_adjoint_with(fmm_, x, y); }

void Mobility::apply_adjoint_with(Fmm* f, const double* x, double* y) {
  // y_f = F^T x_f + B^T x_UOm ; y_UOm = BT^T x_f
  f->apply_adjoint(x, y, NNK_LAYOUT_BLOCKED, 1);
  if (nb_ > 0) {
    body_sums_t(x + 3 * N_, y, 1.0);
    btt_apply(x, y + 3 * N_);
  }
}

void Mobility::grad_positions(const double* z, const double* lam, double* gX, double* gY) {
  cudaStream_t st = ctx_->stream;
  const HostTree& t = fmm_->tree();
  const int64_t Q = fmm_->source_origins();
  DBuf<double> J(3 * N_), H(3 * std::max<int64_t>(Q, 1));
  // the FMM block: d/dX <lam_f, F f> and d/dY <lam_f, F f>
  fmm_->grad_positions(z, lam, NNK_LAYOUT_BLOCKED, J.p, t.params.nearest ? H.p : nullptr);
  const int64_t n = size();
  std::vector<double> hz(n), hl(n), hJ(3 * N_), hH(t.params.nearest ? 3 * Q : 0);
  NNK_CUDA(cudaMemcpyAsync(hz.data(), z, n * sizeof(double), cudaMemcpyDeviceToHost, st));
  NNK_CUDA(cudaMemcpyAsync(hl.data(), lam, n * sizeof(double), cudaMemcpyDeviceToHost, st));
  NNK_CUDA(cudaMemcpyAsync(hJ.data(), J.p, 3 * N_ * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (!hH.empty()) NNK_CUDA(cudaMemcpyAsync(hH.data(), H.p, hH.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  NNK_CUDA(cudaStreamSynchronize(st));
  auto fvec = [&](const std::vector<double>& v, int64_t i, double* o) {
    for (int k = 0; k < 3; ++k) o[k] = v[k * N_ + i];
  };
  auto cross = [](const double* a, const double* b, double* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
  };
  // dL/dX_n = -(J_n + Om_b x lam_n): BT carries xrel = X - x0
  std::vector<double> gx(3 * N_);
  for (int64_t i = 0; i < N_; ++i) {
    double add[3] = {0, 0, 0};
    const int b = hbody_[i];
    if (b >= 0) {
      const double Om[3] = {hz[3 * N_ + 3 * nb_ + b], hz[3 * N_ + 4 * nb_ + b], hz[3 * N_ + 5 * nb_ + b]};
      double l[3];
      fvec(hl, i, l);
      cross(Om, l, add);
    }
    for (int k = 0; k < 3; ++k) gx[3 * i + k] = -(hJ[3 * i + k] + add[k]);
  }
  NNK_CUDA(cudaMemcpyAsync(gX, gx.data(), gx.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  if (gY && t.params.nearest) {
    // dL/dY_q = -(H_q + sum_n NN(q,n) f_n x lam_M,b): B's torque arm is sum_q NN(q,n) (Y_q - x0)
    std::vector<double> gy(3 * Q);
    for (int64_t q = 0; q < Q; ++q) {
      double add[3] = {0, 0, 0};
      const bool body_row = !fstart_.empty() && q < fstart_[nb_];
      if (body_row)
        for (int64_t k = t.nn_rowptr[q]; k < t.nn_rowptr[q + 1]; ++k) {
          const int64_t c = t.nn_col[k];
          const int b = c < N_ ? hbody_[c] : -1;
          if (b < 0) continue;
          double f[3], c3[3];
          fvec(hz, c, f);
          const double lM[3] = {hl[3 * N_ + 3 * nb_ + b], hl[3 * N_ + 4 * nb_ + b], hl[3 * N_ + 5 * nb_ + b]};
          cross(f, lM, c3);
          for (int d = 0; d < 3; ++d) add[d] += t.nn_val[k] * c3[d];
        }
      for (int d = 0; d < 3; ++d) gy[3 * q + d] = -(hH[3 * q + d] + add[d]);
    }
    NNK_CUDA(cudaMemcpyAsync(gY, gy.data(), gy.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  }
  NNK_CUDA(cudaStreamSynchronize(st));
}

void Mobility::solve_plain(const double* rhs, double* x, const nnk_solve_params& sp, bool precondition,
                           nnk_solve_info& info) {
  const int64_t n = size();
  Gmres g(ctx_, n);
  DBuf<double> tmp(n);
  if (precondition) {
    Gmres::Op op = [&](const double* in, double* out) {
      precon(in, tmp.p);
      apply(tmp.p, out);
    };
    Gmres::Op post = [&](const double* in, double* out) { precon(in, out); };
    g.solve(op, &post, rhs, x, sp, info);
  } else {
    Gmres::Op op = [&](const double* in, double* out) { apply(in, out); };
    g.solve(op, nullptr, rhs, x, sp, info);
  }
}

}  // namespace nnk
