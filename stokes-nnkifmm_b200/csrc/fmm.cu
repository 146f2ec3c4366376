// KIFMM passes on the GPU (see fmm.h for the formulation).
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <chrono>
#include <atomic>
#include <array>
#include <type_traits>
#include <cmath>
#include <cstring>
#include <functional>
#include <map>

#include "fmm.h"
#include "kernels.cuh"

namespace nnk {

namespace {

// MATLAB linspace(a,b,n)(m) with exact end points (genupsurf.m:20-22).
inline double mlin(double a, double b, int n, int m) {
  if (m == 0) return a;
  if (m == n - 1) return b;
  return a + ((double)m * (b - a)) / (double)(n - 1);
}

// Lattice indices (x index i, y index j, z index k) of the outer `shells`
// layers of a res^3 meshgrid, in column-major meshgrid order: y fastest,
// then x, then z (genupsurf.m:24-33).
std::vector<std::array<int, 3>> shell_lattice(int res, int shells) {
  std::vector<std::array<int, 3>> out;
  auto inner = [&](int a) { return a >= shells && a <= res - 1 - shells; };
  for (int k = 0; k < res; ++k)
    for (int i = 0; i < res; ++i)
      for (int j = 0; j < res; ++j)
        if (!(inner(j) && inner(i) && inner(k))) out.push_back({i, j, k});
  return out;
}

void surface(const double* lo, const double* hi, int res,
             const std::vector<std::array<int, 3>>& lat, double* out) {
  for (size_t p = 0; p < lat.size(); ++p) {
    out[3 * p + 0] = mlin(lo[0], hi[0], res, lat[p][0]);
    out[3 * p + 1] = mlin(lo[1], hi[1], res, lat[p][1]);
    out[3 * p + 2] = mlin(lo[2], hi[2], res, lat[p][2]);
  }
}

// Stokeslet block S(x0 - x) without the 1/(8 pi mu) factor folded in
// (kernel.m:23-47), added into a column-major matrix.
void kernel_matrix(const std::vector<double>& src, const std::vector<double>& tgt, double eps,
                   double mu, std::vector<double>& Kcm, int ld) {
  const size_t ns = src.size() / 3, nt = tgt.size() / 3;
  const double c = 1.0 / (8.0 * M_PI * mu);
  for (size_t a = 0; a < nt; ++a)
    for (size_t b = 0; b < ns; ++b) {
      const double r[3] = {tgt[3 * a] - src[3 * b], tgt[3 * a + 1] - src[3 * b + 1],
                           tgt[3 * a + 2] - src[3 * b + 2]};
      const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
      const double inv = c / std::pow(r2 + eps * eps, 1.5);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          const double v = (r[i] * r[j] + (i == j ? r2 + 2 * eps * eps : 0.0)) * inv;
          Kcm[(3 * b + j) * (size_t)ld + 3 * a + i] = v;  // row 3a+i, col 3b+j
        }
    }
}

// dS/deps (Tools/kernel.m:23-47 differentiated), the layout of kernel_matrix:
//   eps [(r^2 - 2 eps^2) I - 3 r r^T] / (8 pi mu (r^2 + eps^2)^{5/2}).
void kernel_deriv_matrix(const std::vector<double>& src, const std::vector<double>& tgt, double eps, double mu,
                         std::vector<double>& Kcm, int ld) {
  const size_t ns = src.size() / 3, nt = tgt.size() / 3;
  const double c = eps / (8.0 * M_PI * mu), e2 = eps * eps;
  for (size_t a = 0; a < nt; ++a)
    for (size_t b = 0; b < ns; ++b) {
      const double r[3] = {tgt[3 * a] - src[3 * b], tgt[3 * a + 1] - src[3 * b + 1],
                           tgt[3 * a + 2] - src[3 * b + 2]};
      const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
      const double inv = c / std::pow(r2 + e2, 2.5);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          Kcm[(3 * b + j) * (size_t)ld + 3 * a + i] = ((i == j ? r2 - 2 * e2 : 0.0) - 3 * r[i] * r[j]) * inv;
    }
}

__global__ void dot_partial_kernel(long long n, const double* __restrict__ a, const double* __restrict__ b,
                                   double* __restrict__ part) {
  __shared__ double red[256];
  double s = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    s += a[i] * b[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// The context's cuSOLVER / cuBLAS handles (created on first use), bound to
// its stream.
struct Solver {
  cusolverDnHandle_t s = nullptr;
  cublasHandle_t b = nullptr;
  explicit Solver(nnk_ctx* ctx) {
    if (!ctx->dn_solver) {
      cusolverDnHandle_t h = nullptr;
      if (cusolverDnCreate(&h) != CUSOLVER_STATUS_SUCCESS) throw Error(NNK_E_CUDA, "cusolverDnCreate failed");
      ctx->dn_solver = h;
    }
    if (!ctx->blas) {
      cublasHandle_t h = nullptr;
      if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) throw Error(NNK_E_CUDA, "cublasCreate failed");
      ctx->blas = h;
    }
    s = static_cast<cusolverDnHandle_t>(ctx->dn_solver);
    b = static_cast<cublasHandle_t>(ctx->blas);
    cusolverDnSetStream(s, ctx->stream);
    cublasSetStream(b, ctx->stream);  // (this also drops a workspace set on the handle)
    cudaGetLastError();  // library set-up may leave a handled error behind
  }
  // The context's own cuBLAS workspace (allocated once), set on the handle,
  // so that GEMMs captured into CUDA graphs allocate nothing.
  void own_workspace(nnk_ctx* ctx) {
    constexpr size_t kBytes = (size_t)32 << 20;
    if (!ctx->blas_ws) {
      NNK_CUDA(cudaMalloc(&ctx->blas_ws, kBytes));
      ctx->blas_ws_bytes = kBytes;
    }
    if (cublasSetWorkspace(b, ctx->blas_ws, ctx->blas_ws_bytes) != CUBLAS_STATUS_SUCCESS)
      throw Error(NNK_E_CUDA, "cublasSetWorkspace failed");
  }
};

}  // namespace

void Fmm::bump_version() {
  static std::atomic<uint64_t> counter{0};
  version_ = ++counter;
}

Fmm::Fmm(nnk_ctx* ctx, const HostTree* tree, const FmmParams& p) : ctx_(ctx), t_(tree), p_(p) {
  bump_version();
  if (!(p.eps > 0) || !(p.mu > 0)) throw Error(NNK_E_ARG, "kernelPar needs eps > 0 and mu > 0");
  if (p.res < 2 || p.shells < 1 || 2 * p.shells > p.res)
    throw Error(NNK_E_ARG, "bad coronaRes/coronaShells");
  if (p.max_rhs < 1) throw Error(NNK_E_ARG, "max_rhs must be >= 1");
  R_ = p.max_rhs;
  P_ = (int)shell_lattice(p.res, p.shells).size();
  N_ = t_->nodes;
  E_ = t_->src_start[N_];
  tot_ = E_ + 2LL * P_ * N_;
  maxl_ = t_->max_level;
  using clk = std::chrono::steady_clock;
  const auto t0 = clk::now();
  auto lap = [&](int i, clk::time_point a) {
    setup_ms_[i] = std::chrono::duration<double, std::milli>(clk::now() - a).count();
    return clk::now();
  };
  assign_operators();
  build_points();
  auto t = lap(NNK_SETUP_POINTS, t0);
  build_tasks();
  t = lap(NNK_SETUP_TASKS, t);
  build_operators();
  if (blas_c2e() || m2m_products()) {
    // the library-GEMM products' scratch and workspace before any matvec,
    // which may be captured into a CUDA graph
    reserve_blas_scratch();
    Solver sv(ctx_);
    sv.own_workspace(ctx_);
  }
  lap(NNK_SETUP_TOTAL, t0);
  if (t_->groups() > 1) {
    // tree mask of a forest, all trees on; allocated here because applies
    // may be captured into CUDA graphs that read it by address
    cudaStream_t st = ctx_->stream;
    std::vector<int32_t> tl(t_->tgt_row.size(), 0);
    for (int32_t i = 0; i < N_; ++i)
      for (int64_t k = t_->tgt_start[i]; k < t_->tgt_start[i + 1]; ++k) tl[k] = i;
    tgt_leaf_.upload(tl, st);
    node_tree_.upload(t_->group, st);
    tree_on_host_.assign(t_->groups(), 1);
    tree_on_.upload(tree_on_host_, st);
    node_on_.upload(std::vector<int32_t>(N_, 1), st);
    NNK_CUDA(cudaStreamSynchronize(st));
  }
}

namespace {
__global__ void expand_tree_mask_kernel(int n, const int32_t* __restrict__ node_tree,
                                        const int32_t* __restrict__ tree_on, int32_t* __restrict__ node_on) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) node_on[i] = tree_on[node_tree[i]];
}
}  // namespace

void Fmm::set_active_trees(const char* on) {
  if (!node_on_.p) return;  // a single tree: always evaluated
  bool same = true;
  for (size_t g = 0; g < tree_on_host_.size(); ++g) {
    const int32_t v = on ? (on[g] ? 1 : 0) : 1;
    same = same && tree_on_host_[g] == v;
    tree_on_host_[g] = v;
  }
  if (same) return;
  cudaStream_t st = ctx_->stream;
  NNK_CUDA(cudaMemcpyAsync(tree_on_.p, tree_on_host_.data(), tree_on_host_.size() * sizeof(int32_t),
                           cudaMemcpyHostToDevice, st));
  expand_tree_mask_kernel<<<(N_ + 255) / 256, 256, 0, st>>>(N_, node_tree_.p, tree_on_.p, node_on_.p);
  NNK_CHECK_LAUNCH();
}

Fmm::~Fmm() {
  if (blas_) cublasDestroy((cublasHandle_t)blas_);
  for (auto& r : recs_) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (auto e : pool_) cudaEventDestroy(e);
}

cudaEvent_t Fmm::event() {
  if (!pool_.empty()) {
    cudaEvent_t e = pool_.back();
    pool_.pop_back();
    return e;
  }
  cudaEvent_t e;
  NNK_CUDA(cudaEventCreate(&e));
  return e;
}

template <typename F>
void Fmm::phase(int ph, F&& launch) {
  if (!prof_) {
    launch();
    launches_[ph]++;
    return;
  }
  PhaseRec r{ph, event(), event()};
  NNK_CUDA(cudaEventRecord(r.a, ctx_->stream));
  launch();
  NNK_CUDA(cudaEventRecord(r.b, ctx_->stream));
  recs_.push_back(r);
  launches_[ph]++;
}

void Fmm::set_profile(bool on) {
  prof_ = on;
  if (sparse_) sparse_->set_profile(on);
}

void Fmm::check_errors() {
  if (tensor_m2l_) check_m2l_error(m2l_, ctx_->stream);
  if (c2e_tc_.ready) check_c2e_tc_error(c2e_tc_, ctx_->stream);
  if (sparse_) sparse_->check_errors();
}

void Fmm::poll_errors() {
  if (tensor_m2l_) poll_m2l_error(m2l_, ctx_->stream);
  if (sparse_) sparse_->poll_errors();
}

int Fmm::m2l_stall_probe(uint32_t polls) {
  if (!tensor_m2l_) throw Error(NNK_E_STATE, "the failure-path probe needs the tensor-core M2L (mixed precision)");
  return stall_m2l_probe(m2l_, polls, ctx_->stream);
}

void Fmm::read_profile(double* ms, int64_t* launches) {
  NNK_CUDA(cudaStreamSynchronize(ctx_->stream));
  if (tensor_m2l_) check_m2l_error(m2l_, ctx_->stream);
  for (int k = 0; k < NNK_NUM_PHASES; ++k) {
    if (ms) ms[k] = 0;
    if (launches) launches[k] = launches_[k];
    launches_[k] = 0;
  }
  for (auto& r : recs_) {
    float t = 0;
    NNK_CUDA(cudaEventElapsedTime(&t, r.a, r.b));
    if (ms) ms[r.ph] += t;
    pool_.push_back(r.a);
    pool_.push_back(r.b);
  }
  recs_.clear();
}

Fmm& Fmm::sparse() {
  if (!sparse_) {
    FmmParams q = p_;
    q.res = 4;  // computeVelSparse (KIFMM.m:136-138)
    sparse_.reset(new Fmm(ctx_, t_, q));
  }
  return *sparse_;
}

void Fmm::build_points() {
  const HostTree& t = *t_;
  cudaStream_t st = ctx_->stream;
  const int G = t.groups();
  shift_.assign(3 * (size_t)G, 0.0);
  for (int g = 0; g < G; ++g) {
    const double* root = &t.corners[6 * (size_t)t.root_of(g)];
    for (int d = 0; d < 3; ++d) shift_[3 * g + d] = 0.5 * (root[d] + root[3 + d]);
  }
  auto lat = shell_lattice(p_.res, p_.shells);
  std::vector<double> pos(3 * (size_t)tot_);
  std::vector<int32_t> pgroup(tot_, 0);  // tree of every unified point
  std::copy(t.src_pos.begin(), t.src_pos.end(), pos.begin());
  for (int n = 0; n < N_; ++n) {
    const double* c = &t.corners[6 * n];
    const double lo[3] = {c[0], c[1], c[2]}, hi[3] = {c[3], c[4], c[5]};
    surface(lo, hi, p_.res, lat, &pos[3 * (E_ + (size_t)P_ * n)]);  // genupsurf
    double w[3], dlo[3], dhi[3];
    for (int d = 0; d < 3; ++d) {
      w[d] = hi[d] - lo[d];  // gendownsurf.m:23-24
      dlo[d] = lo[d] - w[d];
      dhi[d] = hi[d] + w[d];
    }
    surface(dlo, dhi, p_.res, lat, &pos[3 * (E_ + (size_t)P_ * N_ + (size_t)P_ * n)]);
    const int32_t g = t.group_of(n);
    for (int64_t e = t.src_start[n]; e < t.src_start[n + 1]; ++e) pgroup[e] = g;
    for (int k = 0; k < P_; ++k) {
      pgroup[E_ + (size_t)P_ * n + k] = g;
      pgroup[E_ + (size_t)P_ * N_ + (size_t)P_ * n + k] = g;
    }
  }
  const int64_t nt = (int64_t)t.tgt_row.size();
  if (f64()) {
    pos64_.upload(pos, st);
    tpos64_.upload(t.tgt_pos, st);
    str64_.alloc(3 * tot_ * R_);
    check64_.alloc((size_t)N_ * 3 * P_ * R_);
    vel64_.alloc(3 * nt * R_);
  }
  if (!f64() || near32()) {
    std::vector<float> p4(4 * (size_t)tot_);
    for (int64_t i = 0; i < tot_; ++i) {
      const double* sh = &shift_[3 * (size_t)pgroup[i]];
      for (int d = 0; d < 3; ++d) p4[4 * i + d] = (float)(pos[3 * i + d] - sh[d]);
      p4[4 * i + 3] = 0.f;
    }
    pos32_.upload(p4, st);
    std::vector<float> t4(4 * (size_t)nt);
    for (int32_t n = 0; n < N_; ++n) {
      const double* sh = &shift_[3 * (size_t)t.group_of(n)];
      for (int64_t i = t.tgt_start[n]; i < t.tgt_start[n + 1]; ++i) {
        for (int d = 0; d < 3; ++d) t4[4 * i + d] = (float)(t.tgt_pos[3 * i + d] - sh[d]);
        t4[4 * i + 3] = 0.f;
      }
    }
    tpos32_.upload(t4, st);
    str32_.alloc(3 * (near32() ? E_ : tot_) * R_);  // NEAR32: the forces of the leaf entries only
    check32_.alloc((size_t)N_ * 3 * P_ * R_);
    vel32_.alloc(3 * nt * R_);
  }
  trow_.upload(t.tgt_row, st);
  goff_.upload(t.src_goff, st);
  gidx_.upload(t.src_gidx, st);
  gw_.upload(t.src_gw, st);
  NNK_CUDA(cudaStreamSynchronize(st));
}

void Fmm::build_tasks() {
  const HostTree& t = *t_;
  TaskRoles r;
  r.regionA = E_;
  r.src_range = &t.src_start;
  r.tgt_range = &t.tgt_start;
  r.src_leaf = &t.pleaf;
  r.tgt_leaf = &t.tleaf;
  r.U = &t.U;
  r.V = &t.V;
  r.W = &t.W;
  r.X = &t.X;
  // node lists per level for the downward C2E step (every node of levels >= 1)
  lvl_off_.assign(maxl_ + 2, 0);
  std::vector<int32_t> ln;
  for (int L = 0; L <= maxl_; ++L) {
    lvl_off_[L] = (int64_t)ln.size();
    if (L >= 1) ln.insert(ln.end(), t.by_level[L].begin(), t.by_level[L].end());
  }
  lvl_off_[maxl_ + 1] = (int64_t)ln.size();
  cudaStream_t st = ctx_->stream;
  {
    std::vector<C2ETile> dt;
    build_c2e_tiles(ln, lvl_off_, dt, dn_toff_);
    dn_tiles_.upload(dt, st);
    dn_tiles_host_ = dt;
  }
  lvl_nodes_.upload(ln, st);
  {
    std::vector<int32_t> roots(t.groups());
    for (int g = 0; g < t.groups(); ++g) roots[g] = t.root_of(g);
    roots_.upload(roots, st);
  }
  fwd_.near = near32();
  build_taskset(fwd_, r, true);
  build_fold_lists();
  stats_.c2e_columns = (int64_t)ln.size() + (int64_t)fwd_.up_nodes_host.size();
  stats_.surface_points = P_;
  stats_.levels = maxl_ + 1;
  const int64_t slots = std::max<int64_t>(3 * fwd_.partial_slots * R_, 1);
  if (f64()) partial64_.alloc(slots);
  if (!f64() || near32()) partial32_.alloc(slots);
  NNK_CUDA(cudaStreamSynchronize(st));
}

void Fmm::build_taskset(TaskSet& ts, const TaskRoles& r, bool stats) {
  const HostTree& t = *t_;
  std::vector<TaskD> tasks;
  std::vector<SegD> segs;
  const long long upB = r.regionA, dnB = r.regionA + (long long)P_ * N_;
  const std::vector<int64_t>& sr = *r.src_range;
  const std::vector<int64_t>& tr = *r.tgt_range;
  auto src_seg = [&](int32_t leaf) {
    const long long s = sr[leaf], e = sr[leaf + 1];
    if (e > s) segs.push_back(SegD{s, (int)(e - s), 0});
    return e - s;
  };
  int64_t pairs_up = 0, pairs_down = 0, pairs_leaf = 0, pairs_p2p = 0, m2l = 0;
  ts.up.assign(maxl_ + 1, {});
  ts.down.assign(maxl_ + 1, {});
  ts.down_nov.assign(maxl_ + 1, {});
  // upward pass (upwardPass.m:32-99): leaves with sources and non-leaves,
  // level by level from the bottom.  The root's expansion is never used by
  // any list, so level 0 is skipped.
  for (int L = maxl_; L >= 1; --L) {
    ts.up[L].first = (int64_t)tasks.size();
    for (int32_t n : t.by_level[L]) {
      const bool leaf = t.child0[n] < 0;
      if (leaf && !(*r.src_leaf)[n]) continue;
      TaskD tk{dnB + (long long)P_ * n, (long long)P_ * n, P_, (int)segs.size(), 0, 0, n, 0};
      if (leaf) {
        pairs_up += (int64_t)P_ * src_seg(n);
      } else {
        for (int k = 0; k < 8; ++k) segs.push_back(SegD{upB + (long long)P_ * (t.child0[n] + k), P_, 0});
        pairs_up += 8LL * P_ * P_;
      }
      tk.nseg = (int)segs.size() - tk.seg0;
      tasks.push_back(tk);
    }
    ts.up[L].count = (int64_t)tasks.size() - ts.up[L].first;
  }
  ts.up_nodes_host.clear();
  ts.up_off.assign(maxl_ + 2, 0);
  for (int L = 0; L <= maxl_; ++L) {
    ts.up_off[L] = (int64_t)ts.up_nodes_host.size();
    if (L == 0) continue;
    for (int32_t n : t.by_level[L])
      if (t.child0[n] >= 0 || (*r.src_leaf)[n]) ts.up_nodes_host.push_back(n);
  }
  ts.up_off[maxl_ + 1] = (int64_t)ts.up_nodes_host.size();
  // downward pass (downwardPass.m:39-168): every node of levels 1..max.
  // The root's downward expansion is zero, so its L2L term is dropped.
  // Two task sets: with the V-list as pair segments, and without it (M2L by
  // the tensor-core or Fourier-space kernels before the pass).
  for (int L = 1; L <= maxl_; ++L) {
    ts.down_nov[L].first = (int64_t)tasks.size();
    for (int32_t n : t.by_level[L]) {
      TaskD tk{upB + (long long)P_ * n, (long long)P_ * n, P_, (int)segs.size(), 0, 0, n, 0};
      for (int64_t k = r.X->off[n]; k < r.X->off[n + 1]; ++k) src_seg(r.X->idx[k]);
      if (t.level[n] >= 2) segs.push_back(SegD{dnB + (long long)P_ * t.parent[n], P_, 0});
      tk.nseg = (int)segs.size() - tk.seg0;
      tasks.push_back(tk);
    }
    ts.down_nov[L].count = (int64_t)tasks.size() - ts.down_nov[L].first;
  }
  for (int L = 1; L <= maxl_; ++L) {
    ts.down[L].first = (int64_t)tasks.size();
    for (int32_t n : t.by_level[L]) {
      TaskD tk{upB + (long long)P_ * n, (long long)P_ * n, P_, (int)segs.size(), 0, 0, n, 0};
      for (int64_t k = r.V->off[n]; k < r.V->off[n + 1]; ++k) {
        segs.push_back(SegD{upB + (long long)P_ * r.V->idx[k], P_, 0});
        pairs_down += (int64_t)P_ * P_;
        ++m2l;
      }
      for (int64_t k = r.X->off[n]; k < r.X->off[n + 1]; ++k) pairs_down += (int64_t)P_ * src_seg(r.X->idx[k]);
      if (t.level[n] >= 2) {  // the root's downward expansion is zero
        segs.push_back(SegD{dnB + (long long)P_ * t.parent[n], P_, 0});
        pairs_down += (int64_t)P_ * P_;
      }
      tk.nseg = (int)segs.size() - tk.seg0;
      tasks.push_back(tk);
    }
    ts.down[L].count = (int64_t)tasks.size() - ts.down[L].first;
  }
  // leaf stage (downwardPass.m:170-294): L2T + U (P2P) + W (M2T)
  ts.leaf.first = (int64_t)tasks.size();
  for (int32_t i = 0; i < N_; ++i) {
    if (!(*r.tgt_leaf)[i]) continue;
    const int nt = (int)(tr[i + 1] - tr[i]);
    if (nt == 0) continue;
    TaskD tk{tr[i], tr[i], nt, (int)segs.size(), 0, 0, i, 0};
    for (int64_t k = r.U->off[i]; k < r.U->off[i + 1]; ++k) {
      const int64_t s = src_seg(r.U->idx[k]);
      pairs_leaf += (int64_t)nt * s;
      pairs_p2p += (int64_t)nt * s;
    }
    for (int64_t k = r.W->off[i]; k < r.W->off[i + 1]; ++k) {
      segs.push_back(SegD{upB + (long long)P_ * r.W->idx[k], P_, 0});
      pairs_leaf += (int64_t)nt * P_;
    }
    segs.push_back(SegD{dnB + (long long)P_ * i, P_, 0});
    pairs_leaf += (int64_t)nt * P_;
    tk.nseg = (int)segs.size() - tk.seg0;
    tasks.push_back(tk);
  }
  ts.leaf.count = (int64_t)tasks.size() - ts.leaf.first;
  if (ts.near) {
    // the same sums split by the precision of their sources: X-list P2L of
    // every level (forces, FP32) apart from each level's L2L (FP64); the leaf
    // stage's U-list P2P (forces, FP32) apart from its L2T and W-list (FP64)
    ts.l2l.assign(maxl_ + 1, {});
    ts.x_only.first = (int64_t)tasks.size();
    for (int L = 1; L <= maxl_; ++L)
      for (int32_t n : t.by_level[L]) {
        if (r.X->off[n + 1] == r.X->off[n]) continue;
        TaskD tk{upB + (long long)P_ * n, (long long)P_ * n, P_, (int)segs.size(), 0, 0, n, 0};
        for (int64_t k = r.X->off[n]; k < r.X->off[n + 1]; ++k) src_seg(r.X->idx[k]);
        tk.nseg = (int)segs.size() - tk.seg0;
        if (tk.nseg) tasks.push_back(tk);
      }
    ts.x_only.count = (int64_t)tasks.size() - ts.x_only.first;
    for (int L = 2; L <= maxl_; ++L) {
      ts.l2l[L].first = (int64_t)tasks.size();
      for (int32_t n : t.by_level[L]) {
        TaskD tk{upB + (long long)P_ * n, (long long)P_ * n, P_, (int)segs.size(), 1, 0, n, 0};
        segs.push_back(SegD{dnB + (long long)P_ * t.parent[n], P_, 0});
        tk.partial = 0;
        tasks.push_back(tk);
      }
      ts.l2l[L].count = (int64_t)tasks.size() - ts.l2l[L].first;
    }
    ts.leaf_u.first = (int64_t)tasks.size();
    for (int32_t i = 0; i < N_; ++i) {
      if (!(*r.tgt_leaf)[i]) continue;
      const int nt = (int)(tr[i + 1] - tr[i]);
      if (nt == 0) continue;
      TaskD tk{tr[i], tr[i], nt, (int)segs.size(), 0, 0, i, 0};
      for (int64_t k = r.U->off[i]; k < r.U->off[i + 1]; ++k) src_seg(r.U->idx[k]);
      tk.nseg = (int)segs.size() - tk.seg0;
      if (tk.nseg) tasks.push_back(tk);
    }
    ts.leaf_u.count = (int64_t)tasks.size() - ts.leaf_u.first;
    ts.leaf_far.first = (int64_t)tasks.size();
    for (int32_t i = 0; i < N_; ++i) {
      if (!(*r.tgt_leaf)[i]) continue;
      const int nt = (int)(tr[i + 1] - tr[i]);
      if (nt == 0) continue;
      TaskD tk{tr[i], tr[i], nt, (int)segs.size(), 0, 0, i, 0};
      for (int64_t k = r.W->off[i]; k < r.W->off[i + 1]; ++k)
        segs.push_back(SegD{upB + (long long)P_ * r.W->idx[k], P_, 0});
      segs.push_back(SegD{dnB + (long long)P_ * i, P_, 0});
      tk.nseg = (int)segs.size() - tk.seg0;
      tasks.push_back(tk);
    }
    ts.leaf_far.count = (int64_t)tasks.size() - ts.leaf_far.first;
  }
  if (&ts == &fwd_) {
    // folded form: the leaves' S2M of each level; the X-list P2L of each
    // level (NEAR32: none, its X-list runs in FP32 from x_only)
    ts.fold = true;
    ts.up_leaf.assign(maxl_ + 1, {});
    ts.down_x.assign(maxl_ + 1, {});
    ts.upl_nodes_host.clear();
    ts.upl_off.assign(maxl_ + 2, 0);
    for (int L = maxl_; L >= 1; --L) {
      ts.up_leaf[L].first = (int64_t)tasks.size();
      for (int32_t n : t.by_level[L]) {
        if (t.child0[n] >= 0 || !(*r.src_leaf)[n]) continue;
        TaskD tk{dnB + (long long)P_ * n, (long long)P_ * n, P_, (int)segs.size(), 0, 0, n, 0};
        src_seg(n);
        tk.nseg = (int)segs.size() - tk.seg0;
        tasks.push_back(tk);
      }
      ts.up_leaf[L].count = (int64_t)tasks.size() - ts.up_leaf[L].first;
    }
    for (int L = 0; L <= maxl_; ++L) {
      ts.upl_off[L] = (int64_t)ts.upl_nodes_host.size();
      if (L == 0) continue;
      for (int32_t n : t.by_level[L])
        if (t.child0[n] < 0 && (*r.src_leaf)[n]) ts.upl_nodes_host.push_back(n);
    }
    ts.upl_off[maxl_ + 1] = (int64_t)ts.upl_nodes_host.size();
    for (int L = 1; L <= maxl_; ++L) {
      ts.down_x[L].first = (int64_t)tasks.size();
      if (!ts.near)
        for (int32_t n : t.by_level[L]) {
          TaskD tk{upB + (long long)P_ * n, (long long)P_ * n, P_, (int)segs.size(), 0, 0, n, 0};
          for (int64_t k = r.X->off[n]; k < r.X->off[n + 1]; ++k) src_seg(r.X->idx[k]);
          tk.nseg = (int)segs.size() - tk.seg0;
          if (tk.nseg) tasks.push_back(tk);
        }
      ts.down_x[L].count = (int64_t)tasks.size() - ts.down_x[L].first;
    }
  }
  cudaStream_t st = ctx_->stream;
  if (ts.fold) {
    std::vector<C2ETile> ut;
    build_c2e_tiles(ts.upl_nodes_host, ts.upl_off, ut, ts.upl_toff);
    ts.upl_tiles_host = ut;
    ts.upl_tiles.upload(ut, st);
    ts.upl_nodes.upload(ts.upl_nodes_host, st);
  }
  {
    std::vector<C2ETile> ut;
    build_c2e_tiles(ts.up_nodes_host, ts.up_off, ut, ts.up_toff);
    ts.up_tiles.upload(ut, st);
    ts.up_tiles_host = ut;
    // scratch of the K-split C2E launches (allocated here: applies may be
    // captured into CUDA graphs, where allocation is not allowed)
    size_t need = 0;
    for (int R = 1; R <= R_; ++R)
      for (int L = 1; L <= maxl_; ++L) {
        need = std::max(need, c2e_part_size(3 * P_, 3 * P_, (int)(ts.up_toff[L + 1] - ts.up_toff[L]), R));
        need = std::max(need, c2e_part_size(3 * P_, 3 * P_, (int)(dn_toff_[L + 1] - dn_toff_[L]), R));
      }
    if (need > c2e_part_.n) c2e_part_.alloc(need);
  }
  split_tasks(ts, tasks, segs);
  ts.tasks.upload(tasks, st);
  ts.segs.upload(segs, st);
  ts.up_nodes.upload(ts.up_nodes_host, st);
  if (stats) {
    stats_.pairs_leaf = pairs_leaf;
    stats_.pairs_p2p = pairs_p2p;
    stats_.pairs_up = pairs_up;
    stats_.pairs_down = pairs_down;
    stats_.m2l_pairs = m2l;
  }
}

// Per level, runs of nodes of the same tree cut into tiles of at most
// kC2ETileNodes nodes, each tile with the operator of its (tree, level).
void Fmm::build_c2e_tiles(const std::vector<int32_t>& nodes, const std::vector<int64_t>& off,
                          std::vector<C2ETile>& tiles, std::vector<int64_t>& toff, int dl) {
  const HostTree& t = *t_;
  toff.assign(off.size(), 0);
  for (size_t L = 0; L + 1 < off.size(); ++L) {
    toff[L] = (int64_t)tiles.size();
    int64_t i = off[L];
    while (i < off[L + 1]) {
      const int32_t g = t.group_of(nodes[i]);
      int64_t j = i;
      while (j < off[L + 1] && j - i < kC2ETileNodes && t.group_of(nodes[j]) == g) ++j;
      const int op = L + dl <= maxl_ ? op_of_[(size_t)g * (maxl_ + 1) + L + dl] : -1;
      if (op < 0) throw Error(NNK_E_STATE, "node above its tree's depth");
      tiles.push_back(C2ETile{op, (int)i, (int)(j - i), 0});
      i = j;
    }
  }
  toff[off.size() - 1] = (int64_t)tiles.size();
}

// Load balance: within each launch group, tasks run heaviest first, and a
// task above the group's piece size is cut into pieces over its flattened
// sources; each piece writes its own partial-sum slot and one reduction per
// task adds the slots in a fixed order.  The piece size is 65,536
// target-source pairs, or a 1/1184 share (8 per SM) of the group's pairs if
// that is larger: a group of thousands of heavy tasks (a forest of NEAREST
// bodies) balances without cutting them, and its partial-sum slots (3R
// values per piece and target) stay small.
void Fmm::split_tasks(TaskSet& ts, std::vector<TaskD>& tasks, std::vector<SegD>& segs) {
  constexpr int64_t kMinPiecePairs = 1 << 16;
  constexpr int64_t kPiecesPerGroup = 148 * 8;
  constexpr int64_t kMinSources = 64;
  std::vector<TaskD> nt;
  std::vector<SegD> ns;
  std::vector<RedD> reds;
  int64_t pbase = 0;
  nt.reserve(tasks.size());
  ns.reserve(segs.size());
  auto process = [&](TaskGroup& g) {
    std::vector<int64_t> cost(g.count), nsrc(g.count), order(g.count);
    for (int64_t i = 0; i < g.count; ++i) {
      const TaskD& r = tasks[g.first + i];
      int64_t c = 0;
      for (int k = 0; k < r.nseg; ++k) c += segs[r.seg0 + k].count;
      nsrc[i] = c;
      cost[i] = c * r.ntgt;
      order[i] = i;
    }
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return cost[a] > cost[b]; });
    int64_t total = 0;
    for (int64_t i = 0; i < g.count; ++i) total += cost[i];
    const int64_t piece = std::max(kMinPiecePairs, total / kPiecesPerGroup);
    const int64_t first = (int64_t)nt.size(), rfirst = (int64_t)reds.size();
    for (int64_t i : order) {
      const TaskD r = tasks[g.first + i];
      int64_t k = (cost[i] + piece - 1) / piece;
      k = std::max<int64_t>(1, std::min<int64_t>(k, nsrc[i] / kMinSources));
      if (k <= 1) {
        TaskD c = r;
        c.seg0 = (int)ns.size();
        c.partial = 0;
        for (int q = 0; q < r.nseg; ++q) ns.push_back(segs[r.seg0 + q]);
        nt.push_back(c);
        continue;
      }
      const int64_t per = (nsrc[i] + k - 1) / k;
      int q = 0;
      int64_t used = 0;  // sources of segment q already assigned
      for (int64_t piece = 0; piece < k; ++piece) {
        TaskD c = r;
        c.seg0 = (int)ns.size();
        c.partial = 1;
        c.out = pbase + piece * r.ntgt;
        int64_t need = per;
        while (need > 0 && q < r.nseg) {
          const SegD sg = segs[r.seg0 + q];
          const int64_t take = std::min<int64_t>(need, sg.count - used);
          if (take > 0) ns.push_back(SegD{sg.start + used, (int)take, 0});
          used += take;
          need -= take;
          if (used == sg.count) {
            ++q;
            used = 0;
          }
        }
        c.nseg = (int)ns.size() - c.seg0;
        nt.push_back(c);
      }
      reds.push_back(RedD{r.out, pbase, r.ntgt, (int)k, r.node, 0});
      pbase += k * r.ntgt;
    }
    g.first = first;
    g.count = (int64_t)nt.size() - first;
    g.red_first = rfirst;
    g.red_count = (int64_t)reds.size() - rfirst;
  };
  for (auto& g : ts.up) process(g);
  for (auto& g : ts.down_nov) process(g);
  for (auto& g : ts.down) process(g);
  process(ts.leaf);
  for (auto& g : ts.up_leaf) process(g);
  for (auto& g : ts.down_x) process(g);
  if (ts.near) {
    process(ts.x_only);
    for (auto& g : ts.l2l) process(g);
    process(ts.leaf_u);
    process(ts.leaf_far);
  }
  tasks.swap(nt);
  segs.swap(ns);
  ts.reds.upload(reds, ctx_->stream);
  ts.partial_slots = pbase;
}

template <typename Real>
void Fmm::run_group(const TaskSet& ts, const TaskGroup& g, const Real* spos, const Real* sstr, const Real* tpos,
                    Real* out, Real e2, Real scale, int accumulate, int phase_id, int R) {
  if (g.count == 0) return;
  cudaStream_t st = ctx_->stream;
  Real* partial = std::is_same<Real, double>::value ? (Real*)partial64_.p : (Real*)partial32_.p;
  const int* na = &ts == &fwd_ ? nact() : nullptr;  // the tree mask applies to the matvec only
  phase(phase_id, [&] {
    launch_p2p<Real>(ts.tasks.p + g.first, (int)g.count, ts.segs.p, spos, sstr, tpos, out, partial, e2, scale, st,
                     accumulate, R, g.bs, na);
  });
  if (g.red_count)
    phase(phase_id, [&] {
      launch_reduce<Real>(ts.reds.p + g.red_first, (int)g.red_count, partial, out, accumulate, st, R, na);
    });
}

// Non-leaf nodes of levels 1 .. max-1 (the root's up expansion is never used
// and its down expansion is zero), their first children, and the tiles of
// the folded upward (operator of the parent's level) and downward (operator
// of the children's level) products.  Folding needs child k of every parent
// at the same position in its parent box.
void Fmm::build_fold_lists() {
  const HostTree& t = *t_;
  fold_pos_.fill(-1);
  bool consistent = true;
  std::vector<int32_t> par, ch;
  fpar_off_.assign(maxl_ + 2, 0);
  for (int L = 0; L <= maxl_; ++L) {
    fpar_off_[L] = (int64_t)par.size();
    for (int32_t n : t.by_level[L]) {
      if (t.child0[n] < 0) continue;
      for (int k = 0; k < 8; ++k) {
        const int32_t c = t.child0[n] + k;
        const int qx = t.ix[c] - 2 * t.ix[n], qy = t.iy[c] - 2 * t.iy[n], qz = t.iz[c] - 2 * t.iz[n];
        const bool in = qx >= 0 && qx <= 1 && qy >= 0 && qy <= 1 && qz >= 0 && qz <= 1;
        const int q = qx * 4 + qy * 2 + qz;
        if (!in || (fold_pos_[k] >= 0 && fold_pos_[k] != q)) consistent = false;
        fold_pos_[k] = q;
      }
      if (L >= 1) {
        par.push_back(n);
        ch.push_back(t.child0[n]);
      }
    }
  }
  fpar_off_[maxl_ + 1] = (int64_t)par.size();
  fold_lists_ok_ = consistent && !par.empty();
  if (!fold_lists_ok_) return;
  cudaStream_t st = ctx_->stream;
  fpar_.upload(par, st);
  fch_.upload(ch, st);
  std::vector<C2ETile> tu, td;
  build_c2e_tiles(par, fpar_off_, tu, fup_toff_);
  build_c2e_tiles(par, fpar_off_, td, fdn_toff_, 1);
  fup_tiles_.upload(tu, st);
  fdn_tiles_.upload(td, st);
  fup_tiles_host_ = tu;
  fdn_tiles_host_ = td;
  const int n = 3 * P_;
  size_t need = c2e_part_.n;
  for (int R = 1; R <= R_; ++R)
    for (int L = 1; L <= maxl_; ++L) {
      need = std::max(need, c2e_part_size(n, 8 * n, (int)(fup_toff_[L + 1] - fup_toff_[L]), R));
      need = std::max(need, c2e_part_size(8 * n, n, (int)(fdn_toff_[L + 1] - fdn_toff_[L]), R));
      need = std::max(need, c2e_part_size(n, n, (int)(fwd_.upl_toff[L + 1] - fwd_.upl_toff[L]), R));
    }
  if (need > c2e_part_.n) c2e_part_.alloc(need);
  NNK_CUDA(cudaStreamSynchronize(st));
}

namespace {
// Kernel matrix in the layout of kernel_matrix (row 3a+i: target a, column
// 3b+j: source b; column-major, leading dimension ld), on the device.
__global__ void kernel_matrix_kernel(const double* __restrict__ src, int ns, const double* __restrict__ tgt, int nt,
                                     double e2, double c, double* __restrict__ K, int ld) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)ns * nt) return;
  const int a = (int)(e % nt), b = (int)(e / nt);
  const double r[3] = {tgt[3 * a] - src[3 * b], tgt[3 * a + 1] - src[3 * b + 1], tgt[3 * a + 2] - src[3 * b + 2]};
  const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
  const double d = r2 + e2;
  const double inv = c / (d * sqrt(d));
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      K[(size_t)(3 * b + j) * ld + 3 * a + i] = (r[i] * r[j] + (i == j ? r2 + 2 * e2 : 0.0)) * inv;
}
}  // namespace

// Canonical surfaces per operator: [parent down surface (w), parent down
// surface (2w), 8 children's up surfaces of [0, w]^3, 8 of [0, 2w]^3].
std::vector<double> Fmm::fold_surfaces() const {
  const auto lat = shell_lattice(p_.res, p_.shells);
  const size_t ps = 3 * (size_t)P_;
  std::vector<double> surf((size_t)nops_ * 18 * ps);
  for (int o = 0; o < nops_; ++o) {
    const double w = op_w_[o];
    double* S = surf.data() + (size_t)o * 18 * ps;
    const double a[3] = {-w, -w, -w}, b[3] = {2 * w, 2 * w, 2 * w};
    surface(a, b, p_.res, lat, S);
    const double a2[3] = {-2 * w, -2 * w, -2 * w}, b2[3] = {4 * w, 4 * w, 4 * w};
    surface(a2, b2, p_.res, lat, S + ps);
    for (int k = 0; k < 8; ++k) {
      const int q = fold_pos_[k];
      const int qd[3] = {(q >> 2) & 1, (q >> 1) & 1, q & 1};
      double lo[3], hi[3], lo2[3], hi2[3];
      for (int d = 0; d < 3; ++d) {
        lo[d] = qd[d] * 0.5 * w;
        hi[d] = lo[d] + 0.5 * w;
        lo2[d] = qd[d] * w;
        hi2[d] = lo2[d] + w;
      }
      surface(lo, hi, p_.res, lat, S + (2 + k) * ps);
      surface(lo2, hi2, p_.res, lat, S + (10 + k) * ps);
    }
  }
  return surf;
}

// M2M_k (child k's up surface -> the down surface of its parent of width w)
// into dM + k (3P)^2 and L2L_k (the down surface of the parent of width 2w ->
// child k's up surface) into dL + k (3P)^2, for operator o (surf: the device
// copy of fold_surfaces()).
void Fmm::kernel_blocks(int o, const double* surf, double* dM, double* dL) {
  const int n = 3 * P_;
  const size_t blk = (size_t)n * n, ps = 3 * (size_t)P_;
  const double e2 = p_.eps * p_.eps, c = 1.0 / (8.0 * M_PI * p_.mu);
  const unsigned kb = (unsigned)(((size_t)P_ * P_ + 255) / 256);
  const double* S = surf + (size_t)o * 18 * ps;
  cudaStream_t st = ctx_->stream;
  for (int k = 0; k < 8; ++k) {
    kernel_matrix_kernel<<<kb, 256, 0, st>>>(S + (2 + k) * ps, P_, S, P_, e2, c, dM + k * blk, n);
    NNK_CHECK_LAUNCH();
    kernel_matrix_kernel<<<kb, 256, 0, st>>>(S + ps, P_, S + (10 + k) * ps, P_, e2, c, dL + k * blk, n);
    NNK_CHECK_LAUNCH();
  }
}

// The folded operators U and D of every box width (see fmm.h), from the
// check-to-equivalent operators A: on canonical boxes (a parent [0, w]^3 with
// its children, or [0, 2w]^3), kernel matrices and products on the device
// (FP64; the products by cuBLAS).  Built for regularized (Tikhonov)
// check-to-equivalent operators only: with the exact inverses (cond ~1e10)
// the folded operators A M2M_k carry FP64 rounding relative to |A| |M2M_k|
// into the very large equivalent densities of NEAREST trees, 4e-5 away from
// the pair sums on a 1200-point NEAREST cloud, where the regularized ones
// stay within 3e-7.  Also needs a matvec whose M2L runs apart from the pair
// tasks (Fourier-space or tensor-core M2L), at most 1 GiB of operators, and
// (unless forced) at least 64 non-leaf nodes per operator: below that the
// set-up costs more than the folded products save.
void Fmm::build_fold_operators(bool force) {
  fold_ok_ = false;
  if (exact_ops_ || !fold_lists_ok_ || !(fft_m2l_ || tensor_m2l_)) return;
  if (!force && fpar_off_.back() < 64 * (int64_t)nops_) return;
  const int n = 3 * P_;
  const size_t blk = (size_t)n * n, per = 8 * blk;
  if ((size_t)nops_ * 2 * per * sizeof(double) > ((size_t)1 << 30)) return;
  cudaStream_t st = ctx_->stream;
  fold_up_.alloc(nops_ * per);
  fold_dn_.alloc(nops_ * per);
  DBuf<double> dS;
  dS.upload(fold_surfaces(), st);
  DBuf<double> dM(per), dL(per);
  Solver sv(ctx_);
  const double one = 1.0, zero = 0.0;
  for (int o = 0; o < nops_; ++o) {
    kernel_blocks(o, dS.p, dM.p, dL.p);
    const double* A = ops_.p + (size_t)o * blk;
    // U = A [M2M_0 .. M2M_7]  (n x 8n)
    if (cublasDgemm(sv.b, CUBLAS_OP_N, CUBLAS_OP_N, n, 8 * n, n, &one, A, n, dM.p, n, &zero,
                    fold_up_.p + (size_t)o * per, n) != CUBLAS_STATUS_SUCCESS)
      throw Error(NNK_E_CUDA, "folded M2M operator product failed");
    // D rows k n .. k n + n - 1 = A^T L2L_k  (8n x n)
    for (int k = 0; k < 8; ++k)
      if (cublasDgemm(sv.b, CUBLAS_OP_T, CUBLAS_OP_N, n, n, n, &one, A, n, dL.p + k * blk, n, &zero,
                      fold_dn_.p + (size_t)o * per + (size_t)k * n, 8 * n) != CUBLAS_STATUS_SUCCESS)
        throw Error(NNK_E_CUDA, "folded L2L operator product failed");
  }
  NNK_CUDA(cudaStreamSynchronize(st));  // dS, dM, dL are freed on return
  fold_ok_ = true;
}

// The unfolded M2M / L2L operators (see fmm.h): for single-tree FMMs whose
// M2L runs apart from the pair tasks, at most 1 GiB of them.
void Fmm::build_m2m_operators() {
  m2m_ok_ = false;
  if (!fold_lists_ok_ || !(fft_m2l_ || tensor_m2l_) || t_->groups() != 1) return;
  const int n = 3 * P_;
  const size_t blk = (size_t)n * n, per = 8 * blk;
  if ((size_t)nops_ * 2 * per * sizeof(double) > ((size_t)1 << 30)) return;
  cudaStream_t st = ctx_->stream;
  m2m_ops_.alloc(nops_ * per);
  l2l_ops_.alloc(nops_ * per);
  DBuf<double> dS;
  dS.upload(fold_surfaces(), st);
  DBuf<double> dL(per);
  for (int o = 0; o < nops_; ++o) {
    // [M2M_0 .. M2M_7] is the blocks side by side (n x 8n, leading dimension n)
    kernel_blocks(o, dS.p, m2m_ops_.p + (size_t)o * per, dL.p);
    // [L2L_0; ..; L2L_7]: block k in rows k n .. k n + n - 1 (8n x n, leading dimension 8n)
    for (int k = 0; k < 8; ++k)
      NNK_CUDA(cudaMemcpy2DAsync(l2l_ops_.p + (size_t)o * per + (size_t)k * n, 8 * n * sizeof(double),
                                 dL.p + k * blk, n * sizeof(double), n * sizeof(double), n,
                                 cudaMemcpyDeviceToDevice, st));
  }
  NNK_CUDA(cudaStreamSynchronize(st));  // dS, dL are freed on return
  m2m_ok_ = true;
}

void Fmm::set_m2m_form(int form) {
  if (form < 0 || form > 2) throw Error(NNK_E_ARG, "M2M / L2L form must be 0, 1 or 2");
  NNK_CUDA(cudaStreamSynchronize(ctx_->stream));
  m2m_on_ = form;
  if (form && !m2m_ok_) build_m2m_operators();
  if (m2m_products()) reserve_blas_scratch();
  bump_version();
}

void Fmm::set_fold(int mode) {
  if (mode < 0 || mode > 2) throw Error(NNK_E_ARG, "fold mode must be 0, 1 or 2");
  NNK_CUDA(cudaStreamSynchronize(ctx_->stream));
  fold_on_ = mode;
  if (mode > 0 && !fold_ok_) build_fold_operators(mode == 2);
  bump_version();
}

// Operator index of every (tree, level): one per distinct box width.
void Fmm::assign_operators() {
  const HostTree& t = *t_;
  const int G = t.groups();
  std::vector<int> gmax(G, 0);
  for (int32_t n = 0; n < N_; ++n) gmax[t.group_of(n)] = std::max(gmax[t.group_of(n)], t.level[n]);
  op_of_.assign((size_t)G * (maxl_ + 1), -1);
  op_w_.clear();
  std::map<double, int> by_w;
  for (int g = 0; g < G; ++g) {
    const double* root = &t.corners[6 * (size_t)t.root_of(g)];
    const double W0 = root[3] - root[0];
    for (int L = 0; L <= gmax[g]; ++L) {
      const double w = std::ldexp(W0, -L);
      auto it = by_w.find(w);
      if (it == by_w.end()) {
        it = by_w.emplace(w, (int)op_w_.size()).first;
        op_w_.push_back(w);
      }
      op_of_[(size_t)g * (maxl_ + 1) + L] = it->second;
    }
  }
  nops_ = (int)op_w_.size();
}

namespace {
// G = I (n x n)
__global__ void identity_kernel(double* G, int n) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < (size_t)n * n) G[e] = (e % (n + 1) == 0) ? 1.0 : 0.0;
}
__global__ void add_diag_kernel(double* G, int n, double v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) G[(size_t)i * n + i] += v;
}
}  // namespace

void Fmm::build_operators() {
  const HostTree& t = *t_;
  if (p_.m2l_mode < 0 || p_.m2l_mode > 4) throw Error(NNK_E_ARG, "m2l_mode must be 0..4");
  // Fourier-space M2L: mode 4 in mixed precision (FP32 spectra); in FP64
  // every mode but 3 (the FP64 pair kernel) when the transforms of one
  // right-hand side fit shared memory (FP64 spectra)
  using clk = std::chrono::steady_clock;
  auto ms_since = [](clk::time_point a) { return std::chrono::duration<double, std::milli>(clk::now() - a).count(); };
  auto tm2l = clk::now();
  const bool fp64 = f64();
  const int fft_cap = fft_m2l_max_rhs(p_.res, fp64);
  if ((!fp64 && p_.m2l_mode == 4) || (fp64 && p_.m2l_mode != 3 && fft_cap >= 1)) {
    std::vector<int> node_op(N_);
    for (int32_t v = 0; v < N_; ++v) node_op[v] = op_of_[(size_t)t.group_of(v) * (maxl_ + 1) + t.level[v]];
    build_fft_m2l(t, p_.res, p_.shells, p_.eps, p_.mu, op_w_, node_op, std::min(R_, std::max(fft_cap, 1)), fp64,
                  fft_, ctx_->stream);
    fft_m2l_ = true;
    stats_.m2l_frequencies = fft_.NK;
    stats_.m2l_family = fft_.family ? 1 : 0;
    stats_.m2l_records = fft_.family ? fft_.records : 0;
    stats_.m2l_groups = fft_.family ? fft_.groups : 0;
  }
  if (p_.precision == NNK_PREC_MIXED && p_.m2l_mode != 3 && p_.m2l_mode != 4) {
    if (p_.m2l_mode == 1) m2l_.image_budget = ~(size_t)0;
    if (p_.m2l_mode == 2) m2l_.image_budget = 0;
    m2l_.compress = p_.m2l_mode == 0;
    build_m2l_plan(t, p_.res, p_.shells, p_.eps, p_.mu, m2l_, ctx_->stream);
    tensor_m2l_ = true;
    stats_.m2l_tile_rows = m2l_.tile_slots * 128;
    stats_.m2l_rank = m2l_.compressed ? m2l_.RC : 0;
  }
  setup_ms_[NNK_SETUP_M2L] = ms_since(tm2l);
  const auto tops = clk::now();
  const int n = 3 * P_;
  cudaStream_t st = ctx_->stream;
  ops_.alloc((size_t)nops_ * n * n);
  auto lat = shell_lattice(p_.res, p_.shells);
  // FP64 mode uses the exact inverse (the reference's LU solve) unless a
  // Tikhonov weight is given; mixed mode always regularizes.
  const bool exact = f64() && !(p_.reg > 0);
  exact_ops_ = exact;
  deps_ready_ = false;
  const double reg = p_.reg > 0 ? p_.reg : 1e-5;
  // host part, in parallel over operators: K_up = kernel(upsurf, downsurf)
  // (up-equivalent densities -> down check) and, for the Tikhonov form,
  // sigma_max(K) by power iteration
  // per operator: its up surface [0, w]^3 and down surface [-w, 2w]^3
  std::vector<double> surf(2 * (size_t)n * std::max(nops_, 1));
  std::vector<std::vector<double>> Ks(nops_);
  std::vector<double> lam2(nops_, 0.0);
#pragma omp parallel for schedule(dynamic, 1)
  for (int o = 0; o < nops_; ++o) {
    const double w = op_w_[o];
    const double lo[3] = {0, 0, 0}, hi[3] = {w, w, w};
    const double dlo[3] = {-w, -w, -w}, dhi[3] = {2 * w, 2 * w, 2 * w};
    surface(lo, hi, p_.res, lat, &surf[2 * (size_t)n * o]);
    surface(dlo, dhi, p_.res, lat, &surf[2 * (size_t)n * o + n]);
    if (!exact) {
      // Tikhonov form: K on the host, for sigma_max(K) by power iteration
      std::vector<double> us(surf.begin() + 2 * (size_t)n * o, surf.begin() + 2 * (size_t)n * o + n);
      std::vector<double> ds(surf.begin() + 2 * (size_t)n * o + n, surf.begin() + 2 * (size_t)n * (o + 1));
      std::vector<double>& K = Ks[o];
      K.assign((size_t)n * n, 0.0);
      kernel_matrix(us, ds, p_.eps, p_.mu, K, n);
      std::vector<double> v(n, 1.0), u(n);
      double smax = 0;
      for (int it = 0; it < 40; ++it) {
        for (int r = 0; r < n; ++r) {
          double sum = 0;
          for (int c = 0; c < n; ++c) sum += K[(size_t)c * n + r] * v[c];
          u[r] = sum;
        }
        double nu = 0;
        for (int c = 0; c < n; ++c) {
          double sum = 0;
          for (int r = 0; r < n; ++r) sum += K[(size_t)c * n + r] * u[r];
          v[c] = sum;
          nu += sum * sum;
        }
        nu = std::sqrt(nu);
        smax = std::sqrt(nu);
        for (double& x : v) x /= nu;
      }
      lam2[o] = (reg * smax) * (reg * smax);
    }
  }
  DBuf<double> dsurf;
  dsurf.upload(surf, st);
  Solver sv(ctx_);
  DBuf<double> dK((size_t)n * n), dG((size_t)n * n);
  DBuf<int> dpiv(n), dinfo(std::max(nops_, 1));
  dinfo.zero(st);
  int lwork = 0;
  if (exact) {
    if (cusolverDnDgetrf_bufferSize(sv.s, n, n, dK.p, n, &lwork) != CUSOLVER_STATUS_SUCCESS)
      throw Error(NNK_E_CUDA, "getrf_bufferSize failed");
  } else {
    if (cusolverDnDpotrf_bufferSize(sv.s, CUBLAS_FILL_MODE_LOWER, n, dG.p, n, &lwork) !=
        CUSOLVER_STATUS_SUCCESS)
      throw Error(NNK_E_CUDA, "potrf_bufferSize failed");
  }
  DBuf<double> dwork(std::max(lwork, 1));
  std::vector<double> KT;
  for (int o = 0; o < nops_; ++o) {
    double* dst = ops_.p + (size_t)o * n * n;
    if (exact) {
      // K = kernel(upsurf, downsurf) on the device; A = K^-1 by LU with
      // partial pivoting, as MATLAB's mldivide (the identity solved in place)
      const double* S = dsurf.p + 2 * (size_t)n * o;
      kernel_matrix_kernel<<<(unsigned)(((size_t)P_ * P_ + 255) / 256), 256, 0, st>>>(
          S, P_, S + n, P_, p_.eps * p_.eps, 1.0 / (8.0 * M_PI * p_.mu), dK.p, n);
      NNK_CHECK_LAUNCH();
      identity_kernel<<<(unsigned)(((size_t)n * n + 255) / 256), 256, 0, st>>>(dst, n);
      NNK_CHECK_LAUNCH();
      if (cusolverDnDgetrf(sv.s, n, n, dK.p, n, dwork.p, dpiv.p, dinfo.p + o) != CUSOLVER_STATUS_SUCCESS ||
          cusolverDnDgetrs(sv.s, CUBLAS_OP_N, n, n, dK.p, n, dpiv.p, dst, n, dinfo.p + o) !=
              CUSOLVER_STATUS_SUCCESS)
        throw Error(NNK_E_CUDA, "LU of the surface matrix failed");
    } else {
      // A = (K^T K + lam^2 I)^-1 K^T, lam = reg * sigma_max(K)
      const std::vector<double>& K = Ks[o];
      NNK_CUDA(cudaMemcpyAsync(dK.p, K.data(), K.size() * 8, cudaMemcpyHostToDevice, st));
      KT.resize((size_t)n * n);
      for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) KT[(size_t)c * n + r] = K[(size_t)r * n + c];
      NNK_CUDA(cudaMemcpyAsync(dst, KT.data(), KT.size() * 8, cudaMemcpyHostToDevice, st));
      const double one = 1.0, zero = 0.0;
      if (cublasDgemm(sv.b, CUBLAS_OP_T, CUBLAS_OP_N, n, n, n, &one, dK.p, n, dK.p, n, &zero, dG.p, n) !=
          CUBLAS_STATUS_SUCCESS)
        throw Error(NNK_E_CUDA, "K^T K product failed");
      add_diag_kernel<<<(n + 127) / 128, 128, 0, st>>>(dG.p, n, lam2[o]);
      NNK_CHECK_LAUNCH();
      if (cusolverDnDpotrf(sv.s, CUBLAS_FILL_MODE_LOWER, n, dG.p, n, dwork.p, lwork, dinfo.p + o) !=
              CUSOLVER_STATUS_SUCCESS ||
          cusolverDnDpotrs(sv.s, CUBLAS_FILL_MODE_LOWER, n, n, dG.p, n, dst, n, dinfo.p + o) !=
              CUSOLVER_STATUS_SUCCESS)
        throw Error(NNK_E_CUDA, "Cholesky of the regularized surface matrix failed");
      // the host copies above read pageable memory; keep K and KT alive until done
      NNK_CUDA(cudaStreamSynchronize(st));
    }
  }
  std::vector<int> info(std::max(nops_, 1), 0);
  NNK_CUDA(cudaMemcpyAsync(info.data(), dinfo.p, info.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
  NNK_CUDA(cudaStreamSynchronize(st));
  for (int o = 0; o < nops_; ++o)
    if (info[o] != 0)
      throw Error(NNK_E_CUDA, "surface matrix factorization reported info=" + std::to_string(info[o]));
  // their int8 digits, when the tensor-core products are asked for or chosen
  if (c2e_mode_ == 1 || (c2e_mode_ < 0 && auto_form_ == 1)) build_tc_digits();
  setup_ms_[NNK_SETUP_OPERATORS] = ms_since(tops);
  const auto tfold = clk::now();
  build_fold_operators(fold_on_ == 2);
  if (m2m_on_) build_m2m_operators();
  setup_ms_[NNK_SETUP_FOLD] = ms_since(tfold);
}

namespace {
// Zeroes the down-equivalent densities of the roots (never computed: the
// root's downward expansion is zero, downwardPass.m:39-40).
template <typename Real>
__global__ void zero_roots_kernel(const int32_t* __restrict__ roots, long long base, int P, int C,
                                  Real* __restrict__ str) {
  Real* p = str + (long long)C * (base + (long long)P * roots[blockIdx.x]);
  for (int i = threadIdx.x; i < P * C; i += blockDim.x) p[i] = 0;
}
}  // namespace

namespace {
// a[i] += b[i] (the FP32 near-field sums into the FP64 ones)
__global__ void add_f32_kernel(long long n, const float* __restrict__ b, double* __restrict__ a) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] += (double)b[i];
}
void add_f32(long long n, const float* b, double* a, cudaStream_t st) {
  if (n <= 0) return;
  add_f32_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, b, a);
  NNK_CHECK_LAUNCH();
}
}  // namespace

template <typename Real>
void Fmm::c2e(int trans, const C2ETile* tiles, const C2ETile* tiles_host, int ntiles, const int32_t* nodes,
              const Real* check, Real* dst, int64_t base, int R, float* m2l_dst, int NP, const int* nact) {
  if (blas_c2e() && tiles_host && !nact && (!m2l_dst || R == 1)) {
    c2e_blas<Real>(trans, tiles_host, ntiles, nodes, check, dst, base, R, m2l_dst, NP);
    return;
  }
  if (tc_c2e())
    launch_c2e_tc<Real>(c2e_tc_, trans, tiles, ntiles, nodes, check, dst, base, P_, R, ctx_->stream, m2l_dst, NP,
                        nact);
  else
    launch_c2e<Real>(ops_.p, 3 * P_, trans, tiles, ntiles, nodes, check, dst, base, P_, R, ctx_->stream, m2l_dst, NP,
                     c2e_part_.p, c2e_part_.n, nact);
}

template <typename Real>
void Fmm::node_gemm_blas(const double* ops, size_t op_stride, int M, int Kd, int trans, const C2ETile* tiles_host,
                         int ntiles, const int32_t* out_nodes, const int32_t* in_nodes, const Real* src, Real* dst,
                         int64_t base, int R, int accumulate, float* m2l_dst, int NP) {
  cudaStream_t st = ctx_->stream;
  if (!blas_x_.p) reserve_blas_scratch();  // normally done at construction
  Solver sv(ctx_);
  sv.own_workspace(ctx_);
  const double one = 1.0, zero = 0.0;
  for (int i = 0; i < ntiles;) {
    // a run of tiles with one operator over consecutive entries of the node lists
    int j = i + 1;
    while (j < ntiles && tiles_host[j].op == tiles_host[i].op &&
           tiles_host[j].first == tiles_host[j - 1].first + tiles_host[j - 1].count)
      ++j;
    const int first = tiles_host[i].first;
    const int ncol = (tiles_host[j - 1].first + tiles_host[j - 1].count - first) * R;
    if ((size_t)ncol * std::max(M, Kd) > blas_x_.n)  // sized for every level's nodes x max_rhs at construction
      throw Error(NNK_E_STATE, "node-product GEMM scratch smaller than a level");
    const int bx = (int)std::min<long long>(148 * 8, ((long long)ncol * Kd + 255) / 256);
    c2e_gather_kernel<Real><<<bx, 256, 0, st>>>(src, in_nodes, first, ncol, R, P_, Kd, blas_x_.p);
    NNK_CHECK_LAUNCH();
    const double* A = ops + (size_t)tiles_host[i].op * op_stride;
    if (cublasDgemm(sv.b, trans ? CUBLAS_OP_T : CUBLAS_OP_N, CUBLAS_OP_N, M, ncol, Kd, &one, A, trans ? Kd : M,
                    blas_x_.p, Kd, &zero, blas_y_.p, M) != CUBLAS_STATUS_SUCCESS)
      throw Error(NNK_E_CUDA, "cublasDgemm (node products) failed");
    const int by = (int)std::min<long long>(148 * 8, ((long long)ncol * M + 255) / 256);
    c2e_scatter_kernel<Real><<<by, 256, 0, st>>>(blas_y_.p, out_nodes, first, ncol, R, P_, M, base, accumulate, dst,
                                                m2l_dst, NP);
    NNK_CHECK_LAUNCH();
    i = j;
  }
}

template <typename Real>
void Fmm::c2e_blas(int trans, const C2ETile* tiles_host, int ntiles, const int32_t* nodes, const Real* check,
                   Real* dst, int64_t base, int R, float* m2l_dst, int NP) {
  const int n3 = 3 * P_;
  node_gemm_blas<Real>(ops_.p, (size_t)n3 * n3, n3, n3, trans, tiles_host, ntiles, nodes, nodes, check, dst, base, R,
                       0, m2l_dst, NP);
}

// Scratch of the library-GEMM C2E for the longest run of one operator in any
// level of either task set.
void Fmm::reserve_blas_scratch() {
  size_t need = 0;
  auto scan = [&](const std::vector<C2ETile>& t) {
    for (size_t i = 0; i < t.size();) {
      size_t j = i + 1;
      while (j < t.size() && t[j].op == t[i].op && t[j].first == t[j - 1].first + t[j - 1].count) ++j;
      need = std::max(need, (size_t)(t[j - 1].first + t[j - 1].count - t[i].first));
      i = j;
    }
  };
  scan(dn_tiles_host_);
  scan(fwd_.up_tiles_host);
  scan(fwd_.upl_tiles_host);
  scan(adj_.up_tiles_host);
  {  // the M2M / L2L products: 8 x 3P rows per parent
    const size_t keep = need;
    need = 0;
    scan(fup_tiles_host_);
    scan(fdn_tiles_host_);
    need = std::max(keep, 8 * need);
  }
  need *= (size_t)3 * P_ * R_;
  if (need > blas_x_.n) {
    blas_x_.alloc(need);
    blas_y_.alloc(need);
  }
}

// Scratch of the tensor-core C2E for the largest launch of either task set.
void Fmm::reserve_tc_scratch() {
  if (!c2e_tc_.ready) return;
  size_t need = 0;
  auto scan = [&](const std::vector<int64_t>& toff) {
    for (size_t L = 0; L + 1 < toff.size(); ++L) need = std::max(need, c2e_tc_blocks((int)(toff[L + 1] - toff[L]), R_));
  };
  scan(dn_toff_);
  scan(fwd_.up_toff);
  if (fwd_.fold) scan(fwd_.upl_toff);
  if (!adj_.up_toff.empty()) scan(adj_.up_toff);  // the transpose's, once built
  reserve_c2e_tc(c2e_tc_, need);
}

// Digits of the operators for the tensor-core products: 9 x 9 digits, levels
// t + u < 9 with FP64 check vectors; 5 x 4, t + u < 5 with FP32 ones.
void Fmm::build_tc_digits() {
  const int n = 3 * P_;
  if (n > 512) return;  // the products stay on the SIMT units
  if (f64()) build_c2e_tc(c2e_tc_, ops_.p, nops_, n, 9, 9, 9, ctx_->stream);
  else build_c2e_tc(c2e_tc_, ops_.p, nops_, n, 5, 4, 5, ctx_->stream);
  reserve_tc_scratch();
}

void Fmm::set_c2e_mode(int mode) {
  if (mode < -1 || mode > 2) throw Error(NNK_E_ARG, "C2E mode must be -1, 0, 1 or 2");
  NNK_CUDA(cudaStreamSynchronize(ctx_->stream));
  c2e_mode_ = mode;
  if (mode == 1 && !c2e_tc_.ready) build_tc_digits();
  if (mode == 2) reserve_blas_scratch();
  bump_version();
}

template <typename Real>
void Fmm::far_field(TaskSet& ts, const Real* spos, Real* str, int64_t regionA, int R, bool near, bool fold) {
  cudaStream_t st = ctx_->stream;
  Real* check = f64() ? (Real*)check64_.p : (Real*)check32_.p;
  const Real e2 = (Real)(p_.eps * p_.eps);
  const Real scale = (Real)(1.0 / (8.0 * M_PI * p_.mu));
  const int n = 3 * P_;
  const int C = 3 * R;
  // up-equivalent densities of nodes that are not computed stay zero
  NNK_CUDA(cudaMemsetAsync(str + C * regionA, 0, sizeof(Real) * C * (size_t)P_ * N_, st));
  zero_roots_kernel<Real><<<(unsigned)roots_.n, 256, 0, st>>>(roots_.p, regionA + (long long)P_ * N_, P_, C, str);
  NNK_CHECK_LAUNCH();
  // the M2L kernels read V(i); the transpose needs V^-1(i), the same set
  // when the relation is symmetric (it is for every tree of the reference)
  const bool fast = &ts == &fwd_ || v_symmetric_;
  const bool tm = fast && tensor_m2l_ && std::is_same<Real, float>::value;
  const bool fm = fast && fft_m2l_;
  if (tm && R != 1) throw Error(NNK_E_STATE, "tensor-core M2L takes one right-hand side per pass");
  if (tm) poll_m2l_error(m2l_, st);  // a wait that gave up in an earlier call
  const int* na = &ts == &fwd_ ? nact() : nullptr;
  // folded M2M / L2L: the M2L must run apart from the pair tasks (it writes
  // every check first), and nothing may need a non-leaf's check afterwards
  const bool fo = fold && ts.fold && folded() && (tm || fm) && !save_up_;
  // M2M / L2L as products with their kernel matrices (the same split of the
  // pair tasks as folding, but into the checks)
  const bool mo = !fo && fold && ts.fold && m2m_products() && (tm || fm) && !save_up_ && !na;
  const bool lo = mo && l2l_products();
  float* m2l_src = tm && !m2l_.compressed ? m2l_.src.p : nullptr;
  // upward pass
  for (int L = maxl_; L >= 1; --L) {
    if (mo) {
      // leaves: S2M pairs; non-leaves: [M2M_0 .. M2M_7] on their 8 children; then C2E
      run_group<Real>(ts, ts.up_leaf[L], spos, str, spos, check, e2, scale, 0, NNK_PHASE_UP_PAIRS, R);
      const int64_t nf = fup_toff_[L + 1] - fup_toff_[L];
      const int64_t nt = ts.up_toff[L + 1] - ts.up_toff[L];
      if (nf + nt > 0)
        phase(NNK_PHASE_UP_C2E, [&] {  // the operator products: M2M, then check-to-equivalent
          if (nf > 0)
            node_gemm_blas<Real>(m2m_ops_.p, (size_t)8 * n * n, n, 8 * n, 0, fup_tiles_host_.data() + fup_toff_[L],
                                 (int)nf, fpar_.p, fch_.p, str + (size_t)C * regionA, check, 0, R, 0, nullptr, 0);
          if (nt > 0)
            c2e<Real>(0, ts.up_tiles.p + ts.up_toff[L], ts.up_tiles_host.data() + ts.up_toff[L], (int)nt,
                      ts.up_nodes.p, check, str, regionA, R, m2l_src, m2l_.NP, na);
        });
      continue;
    }
    if (fo) {
      // leaves: S2M + C2E; non-leaves: U applied to their 8 children
      run_group<Real>(ts, ts.up_leaf[L], spos, str, spos, check, e2, scale, 0, NNK_PHASE_UP_PAIRS, R);
      const int64_t nt = ts.upl_toff[L + 1] - ts.upl_toff[L];
      const int64_t nf = fup_toff_[L + 1] - fup_toff_[L];
      phase(NNK_PHASE_UP_C2E, [&] {
        c2e<Real>(0, ts.upl_tiles.p + ts.upl_toff[L], ts.upl_tiles_host.data() + ts.upl_toff[L], (int)nt,
                  ts.upl_nodes.p, check, str, regionA, R, m2l_src,
                  m2l_.NP, na);
        NodeGemm g{fold_up_.p, (size_t)8 * n * n, n, 8 * n, 0, fup_tiles_.p + fup_toff_[L], fpar_.p, fch_.p,
                   (long long)regionA, P_, R, 0, m2l_src, m2l_.NP};
        launch_node_gemm<Real>(g, (int)nf, str + (size_t)C * regionA, str, st, c2e_part_.p, c2e_part_.n, na);
      });
      continue;
    }
    if (ts.up[L].count == 0) continue;
    run_group<Real>(ts, ts.up[L], spos, str, spos, check, e2, scale, 0, NNK_PHASE_UP_PAIRS, R);
    const int64_t nt = ts.up_toff[L + 1] - ts.up_toff[L];
    phase(NNK_PHASE_UP_C2E, [&] {
      c2e<Real>(0, ts.up_tiles.p + ts.up_toff[L], ts.up_tiles_host.data() + ts.up_toff[L], (int)nt, ts.up_nodes.p,
                check, str, regionA, R, m2l_src, m2l_.NP,
                na);
    });
  }
  if (save_up_) NNK_CUDA(cudaMemcpyAsync(save_up_, check, sizeof(Real) * (size_t)N_ * n * R, cudaMemcpyDeviceToDevice,
                                         st));
  // downward pass
  if (tm) {
    // M2L of every level at once: the V-list only reads up densities
    NNK_CUDA(cudaMemsetAsync(check, 0, sizeof(Real) * (size_t)N_ * n, st));
    // the compressed form projects the up densities (R = 1: 3P floats per node at
    // str + 3 (regionA + P node)) itself
    phase(NNK_PHASE_M2L, [&] { launch_m2l(m2l_, (float*)check, n, st, (const float*)str + 3 * regionA, n); });
  }
  if (fm) {
    // M2L of every level at once in Fourier space
    NNK_CUDA(cudaMemsetAsync(check, 0, sizeof(Real) * (size_t)N_ * n * R, st));
    phase(NNK_PHASE_M2L, [&] { launch_fft_m2l(fft_, (const Real*)str, regionA, R, check, st, na); });
  }
  if (near) {
    // NEAR32: the X-list P2L of every level in FP32 (its sources are the
    // leaf entries' forces), added to the FP64 M2L result
    if (!fm || !std::is_same<Real, double>::value || !ts.near)
      throw Error(NNK_E_STATE, "NEAR32 needs the FP64 Fourier-space M2L");
    const size_t nc = (size_t)N_ * n * R;
    NNK_CUDA(cudaMemsetAsync(check32_.p, 0, sizeof(float) * nc, st));
    run_group<float>(ts, ts.x_only, pos32_.p, str32_.p, pos32_.p, check32_.p, (float)(p_.eps * p_.eps),
                     (float)(1.0 / (8.0 * M_PI * p_.mu)), 1, NNK_PHASE_DOWN_PAIRS, R);
    phase(NNK_PHASE_DOWN_PAIRS, [&] { add_f32((long long)nc, check32_.p, (double*)check, st); });
  }
  const std::vector<TaskGroup>& dgroups =
      (fo || lo) ? ts.down_x : near ? ts.l2l : (tm || fm) ? ts.down_nov : ts.down;
  const int64_t dnB = regionA + (int64_t)P_ * N_;
  for (int L = 1; L <= maxl_; ++L) {
    if (dgroups[L].count > 0)
      run_group<Real>(ts, dgroups[L], spos, str, spos, check, e2, scale, (tm || fm) ? 1 : 0, NNK_PHASE_DOWN_PAIRS,
                      R);
    const int64_t nt = dn_toff_[L + 1] - dn_toff_[L];
    if (nt == 0) continue;
    phase(NNK_PHASE_DOWN_C2E, [&] {  // the operator products: L2L (product form), then check-to-equivalent
      if (lo && L >= 2) {
        // + [L2L_0; ..; L2L_7] from the parents (level L - 1) into their 8 children's checks
        const int64_t nf = fdn_toff_[L] - fdn_toff_[L - 1];
        if (nf > 0)
          node_gemm_blas<Real>(l2l_ops_.p, (size_t)8 * n * n, 8 * n, n, 0, fdn_tiles_host_.data() + fdn_toff_[L - 1],
                               (int)nf, fch_.p, fpar_.p, str + (size_t)C * dnB, check, 0, R, 1, nullptr, 0);
      }
      c2e<Real>(1, dn_tiles_.p + dn_toff_[L], dn_tiles_host_.data() + dn_toff_[L], (int)nt, lvl_nodes_.p, check, str,
                dnB, R, nullptr, 0, na);
      if (fo && L >= 2) {
        // + D applied to the parents (level L - 1) for their 8 children
        const int64_t nf = fdn_toff_[L] - fdn_toff_[L - 1];
        NodeGemm g{fold_dn_.p, (size_t)8 * n * n, 8 * n, n, 0, fdn_tiles_.p + fdn_toff_[L - 1], fch_.p, fpar_.p,
                   (long long)dnB, P_, R, 1, nullptr, 0};
        launch_node_gemm<Real>(g, (int)nf, str + (size_t)C * dnB, str, st, c2e_part_.p, c2e_part_.n, na);
      }
    });
  }
}

template <typename Real>
void Fmm::apply_impl(const double* d_in, const IoMap& in, double* d_out, const IoMap& out, int k0, int R) {
  cudaStream_t st = ctx_->stream;
  const HostTree& t = *t_;
  Real* str = f64() ? (Real*)str64_.p : (Real*)str32_.p;
  const Real* pos = f64() ? (const Real*)pos64_.p : (const Real*)pos32_.p;
  const Real* tpos = f64() ? (const Real*)tpos64_.p : (const Real*)tpos32_.p;
  Real* vel = f64() ? (Real*)vel64_.p : (Real*)vel32_.p;
  const Real e2 = (Real)(p_.eps * p_.eps);
  const Real scale = (Real)(1.0 / (8.0 * M_PI * p_.mu));
  // forces on the leaf source entries (kron(NN,I3)*f per leaf)
  phase(NNK_PHASE_GATHER, [&] { launch_gather<Real>(E_, goff_.p, gidx_.p, gw_.p, d_in, in, k0, R, str, st); });
  const bool near = near32() && std::is_same<Real, double>::value;
  if (near)  // the same forces in FP32 for the near-field sums
    phase(NNK_PHASE_GATHER, [&] { launch_gather<float>(E_, goff_.p, gidx_.p, gw_.p, d_in, in, k0, R, str32_.p, st); });
  far_field<Real>(fwd_, pos, str, E_, R, near, true);
  // leaf stage
  if (near) {
    run_group<Real>(fwd_, fwd_.leaf_far, pos, str, tpos, vel, e2, scale, 0, NNK_PHASE_LEAF_PAIRS, R);
    const size_t nv = 3 * t.tgt_row.size() * (size_t)R;
    NNK_CUDA(cudaMemsetAsync(vel32_.p, 0, sizeof(float) * nv, st));
    run_group<float>(fwd_, fwd_.leaf_u, pos32_.p, str32_.p, tpos32_.p, vel32_.p, (float)(p_.eps * p_.eps),
                     (float)(1.0 / (8.0 * M_PI * p_.mu)), 1, NNK_PHASE_LEAF_PAIRS, R);
    phase(NNK_PHASE_LEAF_PAIRS, [&] { add_f32((long long)nv, vel32_.p, (double*)vel, st); });
  } else {
    run_group<Real>(fwd_, fwd_.leaf, pos, str, tpos, vel, e2, scale, 0, NNK_PHASE_LEAF_PAIRS, R);
  }
  phase(NNK_PHASE_SCATTER, [&] {
    launch_scatter<Real>((int64_t)t.tgt_row.size(), trow_.p, vel, out, k0, R, d_out, st, tgt_leaf_.p, nact());
  });
}

// Transpose: the same passes on the same tree with the roles of the point
// sets exchanged (leaf sources = sorted targets, leaf targets = entries) and
// the lists inverted; the up and down operators are A and A^T as in the
// matvec, since (A^T)^T = A takes the place of each.
template <typename Real>
void Fmm::adjoint_impl(const double* d_in, const IoMap& in, double* d_out, const IoMap& out, int k0, int R) {
  cudaStream_t st = ctx_->stream;
  const HostTree& t = *t_;
  const int64_t nt = (int64_t)t.tgt_row.size();
  Real* astr = f64() ? (Real*)astr64_.p : (Real*)astr32_.p;
  const Real* apos = f64() ? (const Real*)apos64_.p : (const Real*)apos32_.p;
  const Real* pos = f64() ? (const Real*)pos64_.p : (const Real*)pos32_.p;
  Real* avel = f64() ? (Real*)avel64_.p : (Real*)avel32_.p;
  const Real e2 = (Real)(p_.eps * p_.eps);
  const Real scale = (Real)(1.0 / (8.0 * M_PI * p_.mu));
  phase(NNK_PHASE_GATHER, [&] { launch_gather<Real>(nt, agoff_.p, agidx_.p, agw_.p, d_in, in, k0, R, astr, st); });
  far_field<Real>(adj_, apos, astr, nt, R);
  run_group<Real>(adj_, adj_.leaf, apos, astr, pos, avel, e2, scale, 0, NNK_PHASE_LEAF_PAIRS, R);
  phase(NNK_PHASE_SCATTER, [&] {
    scatter_sum_kernel<Real><<<(unsigned)((t.n_pot + 255) / 256), 256, 0, st>>>(
        t.n_pot, (const long long*)row_off_.p, (const long long*)row_ent_.p, row_w_.p, avel, out, k0, R, d_out);
    NNK_CHECK_LAUNCH();
  });
}

// Gradient of <w, apply(f)> with respect to the positions:
//   targets: sum_i w_t,i d/dt u_i(t), u the velocity field of f, from the
//   leaf-stage sources of the matvec (entries, W up-densities, own down-density);
//   sources: sum_j g_e,j d/de w~_j(e), w~ the field of the transpose applied
//   to w and g_e the force of entry e, summed over the entries of each origin.
template <typename Real>
void Fmm::grad_impl(const double* d_f, const double* d_w, int layout, double* d_gt, double* d_gs) {
  cudaStream_t st = ctx_->stream;
  const HostTree& t = *t_;
  const int64_t nt = (int64_t)t.tgt_row.size();
  Real* str = f64() ? (Real*)str64_.p : (Real*)str32_.p;
  const Real* pos = f64() ? (const Real*)pos64_.p : (const Real*)pos32_.p;
  const Real* tpos = f64() ? (const Real*)tpos64_.p : (const Real*)tpos32_.p;
  Real* vel = f64() ? (Real*)vel64_.p : (Real*)vel32_.p;
  Real* astr = f64() ? (Real*)astr64_.p : (Real*)astr32_.p;
  const Real* apos = f64() ? (const Real*)apos64_.p : (const Real*)apos32_.p;
  Real* avel = f64() ? (Real*)avel64_.p : (Real*)avel32_.p;
  Real* partial = f64() ? (Real*)partial64_.p : (Real*)partial32_.p;
  const Real e2 = (Real)(p_.eps * p_.eps);
  const Real scale = (Real)(1.0 / (8.0 * M_PI * p_.mu));
  IoMap fin, win;
  fin.layout = win.layout = layout;
  fin.nrows = t.n_pot;
  win.nrows = t.n_tgt;
  // matvec far field of f; the weights w at the sorted targets
  launch_gather<Real>(E_, goff_.p, gidx_.p, gw_.p, d_f, fin, 0, 1, str, st);
  far_field<Real>(fwd_, pos, str, E_, 1);
  launch_gather<Real>(nt, agoff_.p, agidx_.p, agw_.p, d_w, win, 0, 1, astr, st);
  if (d_gt) {
    const TaskGroup& g = fwd_.leaf;
    launch_p2p_grad<Real>(fwd_.tasks.p + g.first, (int)g.count, fwd_.segs.p, pos, str, tpos, astr, vel, partial, e2,
                          scale, st);
    launch_reduce<Real>(fwd_.reds.p + g.red_first, (int)g.red_count, partial, vel, 0, st, 1);
    IoMap rows;
    rows.layout = NNK_LAYOUT_ROWS;
    rows.nrows = t.n_tgt;
    launch_scatter<Real>(nt, trow_.p, vel, rows, 0, 1, d_gt, st);
  }
  if (d_gs) {
    // transpose far field of w (the gather of w into astr region A is done)
    far_field<Real>(adj_, apos, astr, nt, 1);
    const TaskGroup& g = adj_.leaf;
    launch_p2p_grad<Real>(adj_.tasks.p + g.first, (int)g.count, adj_.segs.p, apos, astr, pos, str, avel, partial, e2,
                          scale, st);
    launch_reduce<Real>(adj_.reds.p + g.red_first, (int)g.red_count, partial, avel, 0, st, 1);
    origin_sum_kernel<Real><<<(unsigned)((norigin_ + 255) / 256), 256, 0, st>>>(
        norigin_, (const long long*)org_off_.p, (const long long*)org_ent_.p, avel, d_gs);
    NNK_CHECK_LAUNCH();
  }
}

void Fmm::apply(const double* d_in, double* d_out, int layout, int nrhs) {
  const HostTree& t = *t_;
  IoMap in, out;
  in.layout = out.layout = layout;
  in.nrows = t.n_pot;
  out.nrows = t.n_tgt;
  apply_mapped(d_in, in, d_out, out, nrhs);
}

void Fmm::apply_mapped(const double* d_in, const IoMap& in, double* d_out, const IoMap& out, int nrhs) {
  if (t_->n_tgt == 0) return;
  const int cap = rhs_cap(false);
  for (int k0 = 0; k0 < nrhs;) {
    const int R = rhs_chunk(nrhs - k0, cap);
    if (f64())
      apply_impl<double>(d_in, in, d_out, out, k0, R);
    else
      apply_impl<float>(d_in, in, d_out, out, k0, R);
    k0 += R;
  }
}

void Fmm::apply_adjoint(const double* d_in, double* d_out, int layout, int nrhs) {
  const HostTree& t = *t_;
  IoMap in, out;
  in.layout = out.layout = layout;
  in.nrows = t.n_tgt;
  out.nrows = t.n_pot;
  apply_adjoint_mapped(d_in, in, d_out, out, nrhs);
}

void Fmm::apply_adjoint_mapped(const double* d_in, const IoMap& in, double* d_out, const IoMap& out, int nrhs) {
  if (t_->n_pot == 0) return;
  build_adjoint();
  const int cap = rhs_cap(true);
  for (int k0 = 0; k0 < nrhs;) {
    const int R = rhs_chunk(nrhs - k0, cap);
    if (f64())
      adjoint_impl<double>(d_in, in, d_out, out, k0, R);
    else
      adjoint_impl<float>(d_in, in, d_out, out, k0, R);
    k0 += R;
  }
}

void Fmm::set_eps(double eps) {
  if (!(eps > 0)) throw Error(NNK_E_ARG, "eps must be > 0");
  NNK_CUDA(cudaStreamSynchronize(ctx_->stream));
  p_.eps = eps;
  bump_version();
  tensor_m2l_ = false;
  fft_m2l_ = false;
  build_operators();
  reduced_ready_ = false;
  sparse_.reset();
}

namespace {
template <typename Real>
double tune_groups(Fmm* self, std::vector<TaskGroup*>& groups, const std::vector<int>& kinds, int R,
                   const std::function<void(const TaskGroup&, int)>& run, cudaStream_t st, bool pick) {
  (void)self;
  (void)kinds;
  cudaEvent_t a, b;
  NNK_CUDA(cudaEventCreate(&a));
  NNK_CUDA(cudaEventCreate(&b));
  double total = 0;
  for (TaskGroup* g : groups) {
    if (g->count == 0) continue;
    float best = 1e30f;
    int best_bs = g->bs;
    const int cand[3] = {64, 128, 256};
    for (int bs : cand) {
      if (!pick && bs != g->bs) continue;
      if (!p2p_bs_ok<Real>(bs, R)) continue;
      TaskGroup t = *g;
      t.bs = bs;
      float ms = 1e30f;
      for (int rep = 0; rep < 2; ++rep) {
        NNK_CUDA(cudaEventRecord(a, st));
        run(t, R);
        NNK_CUDA(cudaEventRecord(b, st));
        NNK_CUDA(cudaEventSynchronize(b));
        float x = 0;
        NNK_CUDA(cudaEventElapsedTime(&x, a, b));
        ms = std::min(ms, x);
      }
      if (ms < best) {
        best = ms;
        best_bs = bs;
      }
    }
    g->bs = best_bs;
    total += best;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return total;
}
}  // namespace

std::pair<double, double> Fmm::autotune(int nrhs) {
  const std::pair<double, double> r = autotune_tiles(nrhs);
  if (c2e_mode_ < 0) tune_c2e(rhs_chunk(nrhs, rhs_cap(false)));
  return r;
}

// The check-to-equivalent products' form in auto mode: one matvec of R
// right-hand sides timed (best of three) with each, the faster kept; the
// operator digits are dropped when the SIMT products win.
void Fmm::tune_c2e(int R) {
  // the candidates: SIMT, tensor cores (where 3P <= 512), library DGEMM (one tree)
  if (3 * P_ <= 512 && !c2e_tc_.ready) build_tc_digits();
  const HostTree& t = *t_;
  cudaStream_t st = ctx_->stream;
  DBuf<double> in(3 * (size_t)t.n_pot * R), out(3 * (size_t)t.n_tgt * R);
  in.zero(st);
  cudaEvent_t a, b;
  NNK_CUDA(cudaEventCreate(&a));
  NNK_CUDA(cudaEventCreate(&b));
  float best[3] = {1e30f, 1e30f, 1e30f};
  for (int m = 0; m < 3; ++m) {
    if ((m == 1 && !c2e_tc_.ready) || (m == 2 && t.groups() != 1)) continue;
    auto_form_ = m;
    bump_version();
    apply(in.p, out.p, NNK_LAYOUT_ROWS, R);  // warm
    for (int rep = 0; rep < 3; ++rep) {
      NNK_CUDA(cudaEventRecord(a, st));
      apply(in.p, out.p, NNK_LAYOUT_ROWS, R);
      NNK_CUDA(cudaEventRecord(b, st));
      NNK_CUDA(cudaEventSynchronize(b));
      float x = 0;
      NNK_CUDA(cudaEventElapsedTime(&x, a, b));
      best[m] = std::min(best[m], x);
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  auto_form_ = (int)(std::min_element(best, best + 3) - best);
  if (auto_form_ != 1 && c2e_tc_.ready) release_c2e_tc(c2e_tc_);
  bump_version();
}

std::pair<double, double> Fmm::autotune_tiles(int nrhs) {
  bump_version();
  const HostTree& t = *t_;
  const int R = rhs_chunk(nrhs, rhs_cap(false));
  cudaStream_t st = ctx_->stream;
  // one pass with real data, so the tuned launches see the real sources
  DBuf<double> in(3 * (size_t)t.n_pot * R), out(3 * (size_t)t.n_tgt * R);
  in.zero(st);
  apply(in.p, out.p, NNK_LAYOUT_ROWS, R);
  if (near32()) {
    // FP64 groups (S2M/M2M, L2L, L2T + W-list) and FP32 groups (X-list P2L,
    // U-list P2P) of the NEAR32 split, each tuned in its own arithmetic
    std::vector<TaskGroup*> g64, g32;
    // (the groups the matvec runs: S2M alone where M2M runs folded or as
    // products, no L2L pairs where L2L does)
    const bool nov = tensor_m2l_ || fft_m2l_;
    for (auto& g : (folded() || (m2m_products() && nov)) ? fwd_.up_leaf : fwd_.up) g64.push_back(&g);
    if (!folded() && !(l2l_products() && nov))
      for (auto& g : fwd_.l2l) g64.push_back(&g);
    g64.push_back(&fwd_.leaf_far);
    g32.push_back(&fwd_.x_only);
    g32.push_back(&fwd_.leaf_u);
    const double e2 = p_.eps * p_.eps, sc = 1.0 / (8.0 * M_PI * p_.mu);
    auto run64 = [&](const TaskGroup& g, int r) {
      const bool leaf = g.first == fwd_.leaf_far.first;
      run_group<double>(fwd_, g, pos64_.p, str64_.p, leaf ? tpos64_.p : pos64_.p, leaf ? vel64_.p : check64_.p, e2,
                        sc, 0, NNK_PHASE_LEAF_PAIRS, r);
    };
    auto run32 = [&](const TaskGroup& g, int r) {
      const bool leaf = g.first == fwd_.leaf_u.first;
      run_group<float>(fwd_, g, pos32_.p, str32_.p, leaf ? tpos32_.p : pos32_.p, leaf ? vel32_.p : check32_.p,
                       (float)e2, (float)sc, 0, NNK_PHASE_LEAF_PAIRS, r);
    };
    std::vector<int> kinds;
    std::pair<double, double> res;
    res.first = tune_groups<double>(this, g64, kinds, R, run64, st, false) +
                tune_groups<float>(this, g32, kinds, R, run32, st, false);
    res.second = tune_groups<double>(this, g64, kinds, R, run64, st, true) +
                 tune_groups<float>(this, g32, kinds, R, run32, st, true);
    NNK_CUDA(cudaStreamSynchronize(st));
    return res;
  }
  std::vector<TaskGroup*> groups;
  const bool nov = tensor_m2l_ || fft_m2l_;
  const bool fo = folded() && nov;
  const bool mo = m2m_products() && nov, lo = l2l_products() && nov;  // the groups the matvec runs
  for (auto& g : (fo || mo) ? fwd_.up_leaf : fwd_.up) groups.push_back(&g);
  for (auto& g : ((fo || lo) ? fwd_.down_x : nov ? fwd_.down_nov : fwd_.down)) groups.push_back(&g);
  groups.push_back(&fwd_.leaf);
  std::pair<double, double> res;
  auto go = [&](auto tag) {
    using Real = decltype(tag);
    Real* str = f64() ? (Real*)str64_.p : (Real*)str32_.p;
    const Real* pos = f64() ? (const Real*)pos64_.p : (const Real*)pos32_.p;
    const Real* tpos = f64() ? (const Real*)tpos64_.p : (const Real*)tpos32_.p;
    Real* check = f64() ? (Real*)check64_.p : (Real*)check32_.p;
    Real* vel = f64() ? (Real*)vel64_.p : (Real*)vel32_.p;
    const Real e2 = (Real)(p_.eps * p_.eps);
    const Real scale = (Real)(1.0 / (8.0 * M_PI * p_.mu));
    auto run = [&](const TaskGroup& g, int r) {
      const bool leaf = &g == &fwd_.leaf || g.first == fwd_.leaf.first;
      run_group<Real>(fwd_, g, pos, str, leaf ? tpos : pos, leaf ? vel : check, e2, scale, 0,
                      NNK_PHASE_LEAF_PAIRS, r);
    };
    std::vector<int> kinds;
    res.first = tune_groups<Real>(this, groups, kinds, R, run, st, false);
    res.second = tune_groups<Real>(this, groups, kinds, R, run, st, true);
  };
  if (f64()) go(double());
  else go(float());
  // the tuned launches overwrote work buffers: nothing to keep
  NNK_CUDA(cudaStreamSynchronize(st));
  return res;
}

// Right-hand sides per pass: the work buffers hold R_; the tensor-core M2L
// takes one and the Fourier M2L its plan's count (the adjoint uses them
// only when V is symmetric).
int Fmm::rhs_cap(bool adjoint) const {
  const bool fast = !adjoint || v_symmetric_;
  if (fast && tensor_m2l_) return 1;
  if (fast && fft_m2l_) return std::min(R_, fft_.Rcap);
  return R_;
}

// A deterministic FP64 dot product on the device (fixed blocks, partial
// sums added on the host in block order).
double Fmm::dot_dev(const double* a, const double* b, int64_t n) {
  constexpr int kBlocks = 592;  // 4 per SM
  if (gpart_.n < (size_t)kBlocks) gpart_.alloc(kBlocks);
  cudaStream_t st = ctx_->stream;
  dot_partial_kernel<<<kBlocks, 256, 0, st>>>((long long)n, a, b, gpart_.p);
  NNK_CHECK_LAUNCH();
  std::vector<double> h(kBlocks);
  NNK_CUDA(cudaMemcpyAsync(h.data(), gpart_.p, sizeof(double) * kBlocks, cudaMemcpyDeviceToHost, st));
  NNK_CUDA(cudaStreamSynchronize(st));
  double s = 0;
  for (double v : h) s += v;
  return s;
}

// dA/deps = -A (dK/deps) A per operator (A = K^-1, K = kernel(upsurf,
// downsurf) of the box width), and the M2L's derivative spectra.
void Fmm::build_deps() {
  if (deps_ready_) return;
  const int n = 3 * P_;
  cudaStream_t st = ctx_->stream;
  auto lat = shell_lattice(p_.res, p_.shells);
  std::vector<std::vector<double>> dKs(nops_);
#pragma omp parallel for schedule(dynamic, 1)
  for (int o = 0; o < nops_; ++o) {
    const double w = op_w_[o];
    const double lo[3] = {0, 0, 0}, hi[3] = {w, w, w};
    const double dlo[3] = {-w, -w, -w}, dhi[3] = {2 * w, 2 * w, 2 * w};
    std::vector<double> us(3 * P_), ds(3 * P_);
    surface(lo, hi, p_.res, lat, us.data());
    surface(dlo, dhi, p_.res, lat, ds.data());
    dKs[o].assign((size_t)n * n, 0.0);
    kernel_deriv_matrix(us, ds, p_.eps, p_.mu, dKs[o], n);
  }
  Solver sv(ctx_);
  dops_.alloc((size_t)nops_ * n * n);
  DBuf<double> dK((size_t)n * n), T((size_t)n * n);
  for (int o = 0; o < nops_; ++o) {
    NNK_CUDA(cudaMemcpyAsync(dK.p, dKs[o].data(), dKs[o].size() * 8, cudaMemcpyHostToDevice, st));
    const double* A = ops_.p + (size_t)o * n * n;
    const double one = 1.0, zero = 0.0, mone = -1.0;
    if (cublasDgemm(sv.b, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, dK.p, n, A, n, &zero, T.p, n) !=
            CUBLAS_STATUS_SUCCESS ||
        cublasDgemm(sv.b, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &mone, A, n, T.p, n, &zero, dops_.p + (size_t)o * n * n,
                    n) != CUBLAS_STATUS_SUCCESS)
      throw Error(NNK_E_CUDA, "dA/deps products failed");
    NNK_CUDA(cudaStreamSynchronize(st));  // dKs[o] is pageable host memory
  }
  if (fft_m2l_) build_fft_deriv(fft_, p_.eps, p_.mu, st);
  const int64_t nt = (int64_t)t_->tgt_row.size();
  const size_t nc = (size_t)N_ * n;
  gsave_cup_.alloc(nc);
  gsave_d_.alloc(nc);
  gsave_avt_.alloc(nc);
  gdchk_.alloc(nc);
  gdscr_.alloc(nc);
  gdvel_.alloc(std::max<size_t>(3 * (size_t)nt, 1));
  NNK_CUDA(cudaStreamSynchronize(st));
  deps_ready_ = true;
}

double Fmm::grad_eps(const double* d_f, const double* d_w, int layout) {
  const HostTree& t = *t_;
  if (!f64() || near32() || !exact_ops_)
    throw Error(NNK_E_STATE, "the eps-derivative needs an FP64 FMM with the exact check-to-equivalent inverses");
  if (t.groups() > 1) throw Error(NNK_E_STATE, "the eps-derivative is for a single tree");
  if (t.n_tgt == 0 || t.n_pot == 0) return 0.0;
  build_adjoint();
  build_deps();
  cudaStream_t st = ctx_->stream;
  const int n = 3 * P_;
  const size_t nc = (size_t)N_ * n;
  const int64_t nt = (int64_t)t.tgt_row.size();
  IoMap fin, win;
  fin.layout = win.layout = layout;
  fin.nrows = t.n_pot;
  win.nrows = t.n_tgt;
  const double e2 = p_.eps * p_.eps, sc = p_.eps / (8.0 * M_PI * p_.mu);
  // forward pass: f, u, v stay in str64_; the up and down check potentials are saved
  launch_gather<double>(E_, goff_.p, gidx_.p, gw_.p, d_f, fin, 0, 1, str64_.p, st);
  NNK_CUDA(cudaMemsetAsync(check64_.p, 0, sizeof(double) * nc, st));
  save_up_ = gsave_cup_.p;
  far_field<double>(fwd_, pos64_.p, str64_.p, E_, 1);
  save_up_ = nullptr;
  NNK_CUDA(cudaMemcpyAsync(gsave_d_.p, check64_.p, sizeof(double) * nc, cudaMemcpyDeviceToDevice, st));
  // transpose pass: its up checks are the sensitivities of the down
  // densities, its up densities those of the down checks, its down checks
  // those of the up densities and its down densities those of the up checks
  launch_gather<double>(nt, agoff_.p, agidx_.p, agw_.p, d_w, win, 0, 1, astr64_.p, st);
  NNK_CUDA(cudaMemsetAsync(check64_.p, 0, sizeof(double) * nc, st));
  save_up_ = gsave_avt_.p;
  far_field<double>(adj_, apos64_.p, astr64_.p, nt, 1);
  save_up_ = nullptr;
  const double* adj_up = astr64_.p + 3 * nt;                          // sensitivities of the down checks
  const double* adj_dn = astr64_.p + 3 * (nt + (int64_t)P_ * N_);     // sensitivities of the up checks
  auto deps_group = [&](const TaskGroup& g, const double* tpos, double* out) {
    if (g.count == 0) return;
    launch_p2p_deps(fwd_.tasks.p + g.first, (int)g.count, fwd_.segs.p, pos64_.p, str64_.p, tpos, out, partial64_.p,
                    e2, sc, st, 1);
    if (g.red_count) launch_reduce<double>(fwd_.reds.p + g.red_first, (int)g.red_count, partial64_.p, out, 1, st, 1);
  };
  double g = 0;
  // S2M and M2M with dS/deps, against the up checks' sensitivities
  NNK_CUDA(cudaMemsetAsync(gdchk_.p, 0, sizeof(double) * nc, st));
  for (int L = maxl_; L >= 1; --L) deps_group(fwd_.up[L], pos64_.p, gdchk_.p);
  g += dot_dev(gdchk_.p, adj_dn, (int64_t)nc);
  // M2L (Fourier, derivative spectra, or V pairs), P2L and L2L, against the down checks' sensitivities
  NNK_CUDA(cudaMemsetAsync(gdchk_.p, 0, sizeof(double) * nc, st));
  if (fft_m2l_) launch_fft_m2l_deriv(fft_, str64_.p, E_, gdchk_.p, st);
  for (int L = 1; L <= maxl_; ++L) deps_group(fft_m2l_ ? fwd_.down_nov[L] : fwd_.down[L], pos64_.p, gdchk_.p);
  g += dot_dev(gdchk_.p, adj_up, (int64_t)nc);
  // L2T, P2P and M2T with dS/deps, against the weights
  NNK_CUDA(cudaMemsetAsync(gdvel_.p, 0, sizeof(double) * 3 * nt, st));
  deps_group(fwd_.leaf, tpos64_.p, gdvel_.p);
  g += dot_dev(gdvel_.p, astr64_.p, 3 * nt);
  // check-to-equivalent solves: <sens(u), dA c> over the up nodes and
  // <sens(v), dA^T d> over the nodes below the root
  NNK_CUDA(cudaMemsetAsync(gdscr_.p, 0, sizeof(double) * nc, st));
  for (int L = maxl_; L >= 1; --L) {
    const int64_t ntl = fwd_.up_toff[L + 1] - fwd_.up_toff[L];
    launch_c2e<double>(dops_.p, n, 0, fwd_.up_tiles.p + fwd_.up_toff[L], (int)ntl, fwd_.up_nodes.p, gsave_cup_.p,
                       gdscr_.p, 0, P_, 1, st, nullptr, 0, c2e_part_.p, c2e_part_.n);
  }
  g += dot_dev(gdscr_.p, check64_.p, (int64_t)nc);
  NNK_CUDA(cudaMemsetAsync(gdscr_.p, 0, sizeof(double) * nc, st));
  for (int L = 1; L <= maxl_; ++L) {
    const int64_t ntl = dn_toff_[L + 1] - dn_toff_[L];
    launch_c2e<double>(dops_.p, n, 1, dn_tiles_.p + dn_toff_[L], (int)ntl, lvl_nodes_.p, gsave_d_.p, gdscr_.p, 0, P_,
                       1, st, nullptr, 0, c2e_part_.p, c2e_part_.n);
  }
  g += dot_dev(gdscr_.p, gsave_avt_.p, (int64_t)nc);
  return g;
}

int64_t Fmm::source_origins() const { return t_->params.nearest ? t_->q : t_->n_pot; }

void Fmm::grad_positions(const double* d_f, const double* d_w, int layout, double* d_gt, double* d_gs) {
  if (t_->n_tgt == 0 || t_->n_pot == 0) return;
  build_adjoint();
  if (f64())
    grad_impl<double>(d_f, d_w, layout, d_gt, d_gs);
  else
    grad_impl<float>(d_f, d_w, layout, d_gt, d_gs);
}

namespace {
// inverse of a list relation: out(j) = { i : j in L(i) }, ascending i
Csr invert(const Csr& L, int32_t nodes) {
  Csr out;
  out.off.assign(nodes + 1, 0);
  for (int32_t j : L.idx) out.off[j + 1]++;
  for (int32_t j = 0; j < nodes; ++j) out.off[j + 1] += out.off[j];
  out.idx.assign(L.idx.size(), 0);
  std::vector<int64_t> pos(out.off.begin(), out.off.end() - 1);
  for (int32_t i = 0; i < nodes; ++i)
    for (int64_t k = L.off[i]; k < L.off[i + 1]; ++k) out.idx[pos[L.idx[k]]++] = i;
  return out;
}
}  // namespace

void Fmm::build_adjoint() {
  if (adj_ready_) return;
  const HostTree& t = *t_;
  cudaStream_t st = ctx_->stream;
  const int64_t nt = (int64_t)t.tgt_row.size();
  inv_U_ = invert(t.U, N_);
  inv_V_ = invert(t.V, N_);
  inv_W_ = invert(t.W, N_);
  inv_X_ = invert(t.X, N_);
  v_symmetric_ = true;
  for (int32_t i = 0; i < N_ && v_symmetric_; ++i) {
    std::vector<int32_t> a(t.V.idx.begin() + t.V.off[i], t.V.idx.begin() + t.V.off[i + 1]);
    std::vector<int32_t> b(inv_V_.idx.begin() + inv_V_.off[i], inv_V_.idx.begin() + inv_V_.off[i + 1]);
    std::sort(a.begin(), a.end());
    v_symmetric_ = a == b;
  }
  TaskRoles r;
  r.regionA = nt;
  r.src_range = &t.tgt_start;
  r.tgt_range = &t.src_start;
  r.src_leaf = &t.tleaf;
  r.tgt_leaf = &t.pleaf;
  r.U = &inv_U_;
  r.V = &inv_V_;
  r.W = &inv_X_;  // leaves s receive from upsurf(t) for t with s in X(t)
  r.X = &inv_W_;  // node t receives from the targets of leaves s with t in W(s)
  build_taskset(adj_, r, false);
  reserve_tc_scratch();
  const int64_t slots = 3 * std::max(fwd_.partial_slots, adj_.partial_slots) * R_;
  if (f64()) {
    if ((int64_t)partial64_.n < slots) partial64_.alloc(slots);
  } else if ((int64_t)partial32_.n < slots) {
    partial32_.alloc(slots);
  }
  // unified points of the transpose: [sorted targets | up surfaces | down surfaces]
  const int64_t atot = nt + 2LL * P_ * N_;
  auto lat = shell_lattice(p_.res, p_.shells);
  std::vector<double> pos(3 * (size_t)atot);
  std::vector<int32_t> pg(atot, 0);
  std::copy(t.tgt_pos.begin(), t.tgt_pos.end(), pos.begin());
  for (int32_t n = 0; n < N_; ++n) {
    const int32_t g = t.group_of(n);
    for (int64_t i = t.tgt_start[n]; i < t.tgt_start[n + 1]; ++i) pg[i] = g;
    const double* c = &t.corners[6 * n];
    const double lo[3] = {c[0], c[1], c[2]}, hi[3] = {c[3], c[4], c[5]};
    surface(lo, hi, p_.res, lat, &pos[3 * (nt + (size_t)P_ * n)]);
    double dlo[3], dhi[3];
    for (int d = 0; d < 3; ++d) {
      const double w = hi[d] - lo[d];
      dlo[d] = lo[d] - w;
      dhi[d] = hi[d] + w;
    }
    surface(dlo, dhi, p_.res, lat, &pos[3 * (nt + (size_t)P_ * N_ + (size_t)P_ * n)]);
    for (int k = 0; k < P_; ++k) {
      pg[nt + (size_t)P_ * n + k] = g;
      pg[nt + (size_t)P_ * N_ + (size_t)P_ * n + k] = g;
    }
  }
  if (f64()) {
    apos64_.upload(pos, st);
    astr64_.alloc(3 * atot * R_);
    avel64_.alloc(std::max<int64_t>(3 * E_ * R_, 1));
  } else {
    std::vector<float> p4(4 * (size_t)atot);
    for (int64_t i = 0; i < atot; ++i) {
      const double* sh = &shift_[3 * (size_t)pg[i]];
      for (int d = 0; d < 3; ++d) p4[4 * i + d] = (float)(pos[3 * i + d] - sh[d]);
      p4[4 * i + 3] = 0.f;
    }
    apos32_.upload(p4, st);
    astr32_.alloc(3 * atot * R_);
    avel32_.alloc(std::max<int64_t>(3 * E_ * R_, 1));
  }
  // identity gather of the target values in sorted order
  std::vector<int64_t> goff(nt + 1);
  for (int64_t i = 0; i <= nt; ++i) goff[i] = i;
  agoff_.upload(goff, st);
  agidx_.upload(t.tgt_row, st);
  agw_.upload(std::vector<double>(std::max<int64_t>(nt, 1), 1.0), st);
  // transpose of the gather: per potential row its (entry, weight) pairs
  {
    std::vector<int64_t> off(t.n_pot + 1, 0);
    for (int32_t r : t.src_gidx) off[r + 1]++;
    for (int64_t r = 0; r < t.n_pot; ++r) off[r + 1] += off[r];
    std::vector<int64_t> ent(t.src_gidx.size()), at(off.begin(), off.end() - 1);
    std::vector<double> w(t.src_gidx.size());
    for (int64_t e = 0; e < E_; ++e)
      for (int64_t k = t.src_goff[e]; k < t.src_goff[e + 1]; ++k) {
        const int64_t q = at[t.src_gidx[k]]++;
        ent[q] = e;
        w[q] = t.src_gw[k];
      }
    row_off_.upload(off, st);
    row_ent_.upload(ent, st);
    row_w_.upload(w, st);
  }
  // entries of each source origin (fine point or potential row)
  {
    norigin_ = source_origins();
    std::vector<int64_t> off(norigin_ + 1, 0);
    for (int64_t o : t.src_origin) off[o + 1]++;
    for (int64_t o = 0; o < norigin_; ++o) off[o + 1] += off[o];
    std::vector<int64_t> ent(t.src_origin.size()), at(off.begin(), off.end() - 1);
    for (int64_t e = 0; e < (int64_t)t.src_origin.size(); ++e) ent[at[t.src_origin[e]]++] = e;
    org_off_.upload(off, st);
    org_ent_.upload(ent, st);
  }
  NNK_CUDA(cudaStreamSynchronize(st));
  adj_ready_ = true;
}

template void Fmm::apply_impl<double>(const double*, const IoMap&, double*, const IoMap&, int, int);
template void Fmm::apply_impl<float>(const double*, const IoMap&, double*, const IoMap&, int, int);

}  // namespace nnk
