// Batched mobility solves (see batch.h).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "batch.h"
#include "gmres.h"

namespace nnk {

namespace {

constexpr int kChunk = 4096;  // entries per reduction block of a segment

struct ChunkD {
  long long start;
  int len;
  int seg;
};

// part[i * nchunks + chunk] = sum over the chunk of V_i * w (i = blockIdx.y),
// in a fixed order; seg_dot_sum_kernel adds a segment's chunks in order, so
// the dot products (and the whole solve) do not depend on scheduling.
// Segments with active[seg] == 0 (when given) contribute 0 without reading.
__global__ void seg_dot_part_kernel(const double* __restrict__ V, long long n, const double* __restrict__ w,
                                    const ChunkD* __restrict__ chunks, double* __restrict__ part, int nchunks,
                                    const double* __restrict__ active) {
  const ChunkD c = chunks[blockIdx.x];
  const int i = blockIdx.y;
  if (active && active[c.seg] == 0.0) {
    if (threadIdx.x == 0) part[(size_t)i * nchunks + blockIdx.x] = 0.0;
    return;
  }
  const double* v = V + (size_t)i * n;
  double s = 0;
  for (int k = threadIdx.x; k < c.len; k += blockDim.x) s += v[c.start + k] * w[c.start + k];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ double red[8];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
    part[(size_t)i * nchunks + blockIdx.x] = t;
  }
}

// h[seg * ldh + i] += sum of the segment's chunk partials, in chunk order
__global__ void seg_dot_sum_kernel(const double* __restrict__ part, int nchunks, const int* __restrict__ cfirst,
                                   int S, int nvec, double* __restrict__ h, int ldh) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)S * nvec) return;
  const int s = (int)(e % S), i = (int)(e / S);
  double t = 0;
  for (int c = cfirst[s]; c < cfirst[s + 1]; ++c) t += part[(size_t)i * nchunks + c];
  h[(size_t)s * ldh + i] += t;
}

// w -= sum_{i<k} V_i h[seg][i] (sign = -1), or x += sum V_i y[seg][i] (sign = +1);
// segments with active[seg] == 0 (when given) are left as they are
__global__ void seg_axpy_kernel(const double* __restrict__ V, long long n, int k, const double* __restrict__ h,
                                int ldh, const ChunkD* __restrict__ chunks, double* __restrict__ w, double sign,
                                const double* __restrict__ active) {
  extern __shared__ double hs[];
  const ChunkD c = chunks[blockIdx.x];
  if (active && active[c.seg] == 0.0) return;
  for (int i = threadIdx.x; i < k; i += blockDim.x) hs[i] = h[(size_t)c.seg * ldh + i];
  __syncthreads();
  for (int e = threadIdx.x; e < c.len; e += blockDim.x) {
    const long long x = c.start + e;
    double s = 0;
    for (int i = 0; i < k; ++i) s += V[(size_t)i * n + x] * hs[i];
    w[x] += sign * s;
  }
}

// v = w / sqrt(nrm2[seg]) for active segments with nrm2 > 0, else 0
__global__ void seg_normalize_kernel(const double* __restrict__ w, const double* __restrict__ nrm2,
                                     const double* __restrict__ active, const ChunkD* __restrict__ chunks,
                                     double* __restrict__ v) {
  const ChunkD c = chunks[blockIdx.x];
  const double q = nrm2[c.seg];
  const double a = (active[c.seg] != 0.0 && q > 0.0) ? 1.0 / sqrt(q) : 0.0;
  for (int e = threadIdx.x; e < c.len; e += blockDim.x) v[c.start + e] = a != 0.0 ? a * w[c.start + e] : 0.0;
}

__device__ __forceinline__ void cross3(const double* a, const double* b, double* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

// y_f += BT [U; Om] = -U + xrel x Om on every force point, for each
// right-hand side of its body (genMatrixComponets.m:34-50)
__global__ void batch_bt_kernel(long long Nt, int R, const int* __restrict__ row_body,
                                const int* __restrict__ row_local, const long long* __restrict__ sys_off,
                                const int* __restrict__ sys_n, const double* __restrict__ xrel,
                                const double* __restrict__ x, double* __restrict__ y) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= Nt) return;
  const int b = row_body[g], i = row_local[g];
  const double xr[3] = {xrel[3 * g], xrel[3 * g + 1], xrel[3 * g + 2]};
  for (int r = 0; r < R; ++r) {
    const int s = b * R + r;
    const long long base = sys_off[s];
    const int N = sys_n[s];
    const double* uo = x + base + 3LL * N;
    const double O[3] = {uo[3], uo[4], uo[5]};
    double c[3];
    cross3(xr, O, c);
    for (int k = 0; k < 3; ++k) y[base + (long long)k * N + i] += -uo[k] + c[k];
  }
}

// y_UOm = B f = [sum af f ; sum xm x f] per system (genMatrixComponets.m:53-95)
__global__ void batch_bsum_kernel(const long long* __restrict__ body_row0, int R, const long long* __restrict__ sys_off,
                                  const int* __restrict__ sys_n, const double* __restrict__ af,
                                  const double* __restrict__ xm, const double* __restrict__ x,
                                  double* __restrict__ y) {
  const int s = blockIdx.x;
  const int b = s / R;
  const long long base = sys_off[s], g0 = body_row0[b];
  const int N = sys_n[s];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const double v[3] = {x[base + i], x[base + N + i], x[base + 2LL * N + i]};
    const long long g = g0 + i;
    const double arm[3] = {xm[3 * g], xm[3 * g + 1], xm[3 * g + 2]};
    const double a = af[g];
    double c[3];
    cross3(arm, v, c);
    acc[0] += a * v[0];
    acc[1] += a * v[1];
    acc[2] += a * v[2];
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
  if (threadIdx.x < 6) y[base + 3LL * N + threadIdx.x] = red[threadIdx.x][0];
}

unsigned blocks_for(int64_t n) { return (unsigned)std::max<int64_t>(1, (n + 255) / 256); }

}  // namespace

// ------------------------------------------------------------------ SegGmres

SegGmres::SegGmres(nnk_ctx* ctx, const std::vector<int64_t>& off) : ctx_(ctx), off_(off) {
  S_ = (int)off.size() - 1;
  n_ = off.back();
  std::vector<ChunkD> ch;
  std::vector<int32_t> cf(S_ + 1, 0);
  for (int s = 0; s < S_; ++s) {
    cf[s] = (int32_t)ch.size();
    for (int64_t a = off[s]; a < off[s + 1]; a += kChunk)
      ch.push_back(ChunkD{a, (int)std::min<int64_t>(kChunk, off[s + 1] - a), s});
  }
  cf[S_] = (int32_t)ch.size();
  cfirst_.upload(cf, ctx_->stream);
  nchunks_ = (int)ch.size();
  std::vector<Chunk> c2(ch.size());
  std::memcpy(c2.data(), ch.data(), ch.size() * sizeof(ChunkD));
  static_assert(sizeof(Chunk) == sizeof(ChunkD), "chunk layout");
  chunks_.upload(c2, ctx_->stream);
}

void SegGmres::seg_dots(const double* V, int nvec, const double* w, double* h, int ldh, const double* active) {
  if (nchunks_ == 0 || nvec == 0) return;
  cudaStream_t st = ctx_->stream;
  const size_t need = (size_t)nvec * nchunks_;
  if (need > part_.n) {
    NNK_CUDA(cudaStreamSynchronize(st));  // the old buffer may still be read
    part_.alloc(std::max(need, 2 * part_.n));
  }
  seg_dot_part_kernel<<<dim3(nchunks_, nvec), 256, 0, st>>>(V, n_, w, (const ChunkD*)chunks_.p, part_.p, nchunks_,
                                                             active);
  NNK_CHECK_LAUNCH();
  seg_dot_sum_kernel<<<blocks_for((int64_t)S_ * nvec), 256, 0, st>>>(part_.p, nchunks_, cfirst_.p, S_, nvec, h, ldh);
  NNK_CHECK_LAUNCH();
}

std::vector<double> SegGmres::norms(const double* v) {
  cudaStream_t st = ctx_->stream;
  DBuf<double> d(std::max(S_, 1));
  d.zero(st);
  seg_dots(v, 1, v, d.p, 1);
  std::vector<double> h(S_);
  NNK_CUDA(cudaMemcpyAsync(h.data(), d.p, S_ * sizeof(double), cudaMemcpyDeviceToHost, st));
  NNK_CUDA(cudaStreamSynchronize(st));
  for (double& x : h) x = std::sqrt(x);
  return h;
}

void SegGmres::solve(const Op& op, const double* b, double* x, const std::vector<double>& tol, int maxit,
                     int restart, const std::vector<char>& want, std::vector<nnk_solve_info>& info, bool confirm) {
  cudaStream_t st = ctx_->stream;
  const int S = S_;
  const int64_t n = n_;
  const ChunkD* chunks = (const ChunkD*)chunks_.p;
  int64_t maxlen = 0;
  for (int s = 0; s < S; ++s) maxlen = std::max(maxlen, off_[s + 1] - off_[s]);
  maxit = maxit > 0 ? maxit : (int)std::min<int64_t>(maxlen, 10);
  int m = restart > 0 ? std::min(restart, maxit) : maxit;
  m = (int)std::max<int64_t>(1, std::min<int64_t>(m, maxlen));
  const int ldh = m + 1;
  // The Krylov basis grows on demand (doubling, up to m + 1 vectors): a batch
  // of tens of millions of unknowns that converges in a few dozen steps must
  // not hold maxit + 1 vectors.
  int vcap = std::min(m + 1, 16);
  DBuf<double> V((size_t)vcap * n), w(n), r(n), scal(S), act(S);
  auto reserve = [&](int need) {
    if (need <= vcap) return;
    int nc = vcap;
    while (nc < need) nc = std::min(m + 1, 2 * nc);
    DBuf<double> V2((size_t)nc * n);
    // stream order: the copy follows every step already enqueued on V
    NNK_CUDA(cudaMemcpyAsync(V2.p, V.p, (size_t)vcap * n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    NNK_CUDA(cudaStreamSynchronize(st));
    V = std::move(V2);
    vcap = nc;
  };
  // per step: [pass-1 h (S x ldh) | pass-2 h (S x ldh) | ||w||^2 (S)], two slots
  const size_t slot = 2 * (size_t)S * ldh + S;
  DBuf<double> hdev(2 * slot);
  double* hhost = nullptr;
  NNK_CUDA(cudaMallocHost((void**)&hhost, 2 * slot * sizeof(double)));
  struct HostFree {
    double* p;
    ~HostFree() { cudaFreeHost(p); }
  } hf{hhost};
  cudaEvent_t ev[2];
  NNK_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
  NNK_CUDA(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
  struct EvFree {
    cudaEvent_t* e;
    ~EvFree() {
      cudaEventDestroy(e[0]);
      cudaEventDestroy(e[1]);
    }
  } ef{ev};

  info.assign(S, nnk_solve_info{0, 0, 0.0});
  struct ActiveReset {
    const std::function<void(const std::vector<char>&)>& f;
    int S;
    ~ActiveReset() {
      if (f) {
        try {
          f(std::vector<char>(S, 1));
        } catch (...) {
        }
      }
    }
  } active_reset{on_active, S};
  NNK_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), st));
  // ||b_s||
  std::vector<double> nb(S, 0.0), beta(S, 0.0), relres(S, 1.0);
  {
    NNK_CUDA(cudaMemsetAsync(scal.p, 0, S * sizeof(double), st));
    seg_dots(b, 1, b, scal.p, 1);
    NNK_CUDA(cudaMemcpyAsync(nb.data(), scal.p, S * sizeof(double), cudaMemcpyDeviceToHost, st));
    NNK_CUDA(cudaStreamSynchronize(st));
    for (int s = 0; s < S; ++s) nb[s] = std::sqrt(nb[s]);
  }
  std::vector<char> live(S, 0);  // still to be solved
  for (int s = 0; s < S; ++s) {
    live[s] = want[s] && nb[s] > 0.0;
    beta[s] = nb[s];
    if (!live[s]) relres[s] = 0.0;
  }
  NNK_CUDA(cudaMemcpyAsync(r.p, b, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  std::vector<double> H((size_t)S * ldh * m), cs((size_t)S * m), sn((size_t)S * m), g((size_t)S * ldh),
      Y((size_t)S * ldh), hact(S), hb2(S);
  std::vector<int> k_of(S, 0);
  auto enqueue_step = [&](int j) {
    reserve(j + 2);  // reads V_0..V_j, writes V_{j+1}
    double* hs = hdev.p + (j & 1) * slot;
    double* vj = V.p + (size_t)j * n;
    op(vj, w.p);
    ++matvecs_;
    NNK_CUDA(cudaMemsetAsync(hs, 0, slot * sizeof(double), st));
    for (int pass = 0; pass < 2; ++pass) {
      double* hp = hs + (size_t)pass * S * ldh;
      // segments that stopped are skipped: their h and w are never read again
      seg_dots(V.p, j + 1, w.p, hp, ldh, act.p);
      seg_axpy_kernel<<<nchunks_, 256, (j + 1) * sizeof(double), st>>>(V.p, n, j + 1, hp, ldh, chunks, w.p, -1.0,
                                                                       act.p);
      NNK_CHECK_LAUNCH();
    }
    double* nrm = hs + 2 * (size_t)S * ldh;
    seg_dots(w.p, 1, w.p, nrm, 1, act.p);
    seg_normalize_kernel<<<nchunks_, 256, 0, st>>>(w.p, nrm, act.p, chunks, V.p + (size_t)(j + 1) * n);
    NNK_CHECK_LAUNCH();
    NNK_CUDA(cudaMemcpyAsync(hhost + (j & 1) * slot, hs, slot * sizeof(double), cudaMemcpyDeviceToHost, st));
    NNK_CUDA(cudaEventRecord(ev[j & 1], st));
  };
  while (true) {
    // start a cycle: V_0 = r / beta on the live segments
    std::vector<char> active = live;
    int nact = 0;
    for (int s = 0; s < S; ++s) {
      hact[s] = active[s] ? 1.0 : 0.0;
      hb2[s] = active[s] ? beta[s] * beta[s] : 0.0;
      nact += active[s];
      k_of[s] = 0;
      std::fill(g.begin() + (size_t)s * ldh, g.begin() + (size_t)(s + 1) * ldh, 0.0);
      g[(size_t)s * ldh] = beta[s];
    }
    if (nact == 0) break;
    if (on_active) on_active(active);
    NNK_CUDA(cudaMemcpyAsync(act.p, hact.data(), S * sizeof(double), cudaMemcpyHostToDevice, st));
    NNK_CUDA(cudaMemcpyAsync(scal.p, hb2.data(), S * sizeof(double), cudaMemcpyHostToDevice, st));
    seg_normalize_kernel<<<nchunks_, 256, 0, st>>>(r.p, scal.p, act.p, chunks, V.p);
    NNK_CHECK_LAUNCH();
    int j = 0;
    enqueue_step(0);
    for (;; ++j) {
      // run one step ahead: step j+1 only needs V_{j+1}, which step j made
      bool ahead = false;
      if (j + 1 < m) {
        enqueue_step(j + 1);
        ahead = true;
      }
      NNK_CUDA(cudaEventSynchronize(ev[j & 1]));
      const double* hs = hhost + (j & 1) * slot;
      bool changed = false;
      for (int s = 0; s < S; ++s) {
        if (!active[s]) continue;
        double* hc = &H[((size_t)s * m + j) * ldh];
        for (int i = 0; i <= j; ++i)
          hc[i] = hs[(size_t)s * ldh + i] + hs[(size_t)S * ldh + (size_t)s * ldh + i];
        const double hn = std::sqrt(std::max(0.0, hs[2 * (size_t)S * ldh + s]));
        hc[j + 1] = hn;
        double* c = &cs[(size_t)s * m];
        double* sv = &sn[(size_t)s * m];
        for (int i = 0; i < j; ++i) {
          const double t0 = c[i] * hc[i] + sv[i] * hc[i + 1];
          hc[i + 1] = -sv[i] * hc[i] + c[i] * hc[i + 1];
          hc[i] = t0;
        }
        const double den = std::hypot(hc[j], hc[j + 1]);
        c[j] = den > 0 ? hc[j] / den : 1.0;
        sv[j] = den > 0 ? hc[j + 1] / den : 0.0;
        hc[j] = den;
        hc[j + 1] = 0.0;
        double* gs = &g[(size_t)s * ldh];
        gs[j + 1] = -sv[j] * gs[j];
        gs[j] = c[j] * gs[j];
        k_of[s] = j + 1;
        info[s].iters += 1;
        if (std::fabs(gs[j + 1]) / nb[s] <= tol[s] || hn == 0.0 || info[s].iters >= maxit) {
          active[s] = 0;
          hact[s] = 0.0;
          changed = true;
          --nact;
        }
      }
      if (nact == 0 || j + 1 >= m) {
        if (ahead) NNK_CUDA(cudaEventSynchronize(ev[(j + 1) & 1]));
        break;
      }
      // segments that stopped produce zero vectors from the next step on
      if (changed) {
        NNK_CUDA(cudaMemcpyAsync(act.p, hact.data(), S * sizeof(double), cudaMemcpyHostToDevice, st));
        if (on_active) on_active(active);
      }
    }
    // y_s = R_s^-1 g_s, x += V y
    std::fill(Y.begin(), Y.end(), 0.0);
    int kmax = 0;
    for (int s = 0; s < S; ++s) {
      const int k = k_of[s];
      kmax = std::max(kmax, k);
      for (int i = k - 1; i >= 0; --i) {
        double v = g[(size_t)s * ldh + i];
        for (int l = i + 1; l < k; ++l) v -= H[((size_t)s * m + l) * ldh + i] * Y[(size_t)s * ldh + l];
        const double d = H[((size_t)s * m + i) * ldh + i];
        Y[(size_t)s * ldh + i] = d != 0 ? v / d : 0.0;
      }
    }
    if (kmax > 0) {
      DBuf<double> dY(Y.size());
      NNK_CUDA(cudaMemcpyAsync(dY.p, Y.data(), Y.size() * sizeof(double), cudaMemcpyHostToDevice, st));
      seg_axpy_kernel<<<nchunks_, 256, kmax * sizeof(double), st>>>(V.p, n, kmax, dY.p, ldh, chunks, x, 1.0,
                                                                    nullptr);
      NNK_CHECK_LAUNCH();
      NNK_CUDA(cudaStreamSynchronize(st));
    }
    if (!confirm) {
      // the caller checks the residual itself (iterative refinement): stop
      // when every segment met tol by the recurrence or ran out of steps
      bool done = true;
      for (int s = 0; s < S; ++s) {
        if (!live[s]) continue;
        relres[s] = std::fabs(g[(size_t)s * ldh + k_of[s]]) / nb[s];
        if (relres[s] > tol[s] && info[s].iters < maxit && k_of[s] > 0) done = false;
      }
      if (done) break;
    }
    // explicit residuals r = b - A x (MATLAB gmres confirms convergence this way)
    if (on_active) on_active(live);
    op(x, w.p);
    ++matvecs_;
    dev_axpby(ctx_, 1.0, b, -1.0, w.p, r.p, n);
    NNK_CUDA(cudaMemsetAsync(scal.p, 0, S * sizeof(double), st));
    seg_dots(r.p, 1, r.p, scal.p, 1);
    std::vector<double> rn(S);
    NNK_CUDA(cudaMemcpyAsync(rn.data(), scal.p, S * sizeof(double), cudaMemcpyDeviceToHost, st));
    NNK_CUDA(cudaStreamSynchronize(st));
    int again = 0;
    for (int s = 0; s < S; ++s) {
      if (!live[s]) continue;
      beta[s] = std::sqrt(rn[s]);
      relres[s] = beta[s] / nb[s];
      const bool more = relres[s] > tol[s] && info[s].iters < maxit && k_of[s] > 0 && beta[s] > 0.0;
      live[s] = more;
      again += more;
    }
    if (!again) break;
  }
  for (int s = 0; s < S; ++s) {
    info[s].relres = relres[s];
    info[s].flag = relres[s] <= tol[s] ? 0 : 1;
  }
}

// -------------------------------------------------------------- BatchMobility

BatchMobility::BatchMobility(nnk_ctx* ctx, const std::vector<BatchBody>& bodies, const FmmParams& fp, int nrhs)
    : ctx_(ctx), fp_(fp) {
  if (bodies.empty()) throw Error(NNK_E_ARG, "batch needs at least one body");
  if (nrhs < 1) throw Error(NNK_E_ARG, "batch needs nrhs >= 1");
  B_ = (int)bodies.size();
  R_ = nrhs;
  S_ = B_ * R_;
  std::vector<const HostTree*> trees;
  for (const auto& bd : bodies) {
    const HostTree& t = *bd.tree;
    if (t.n_pot != t.n_tgt || t.n_pot != t.n) throw Error(NNK_E_ARG, "mobility needs potentials == targets");
    if (t.n_tgt < 1) throw Error(NNK_E_ARG, "empty body");
    if (!bd.rel_points) throw Error(NNK_E_ARG, "body without rel_points");
    if (t.params.nearest && !bd.rel_fine) throw Error(NNK_E_ARG, "NEAREST body needs rel_fine");
    trees.push_back(&t);
    bN_.push_back(t.n_tgt);
  }
  merge_forest(trees, forest_);
  Nt_ = forest_.n_tgt;
  off_.assign(S_ + 1, 0);
  for (int b = 0; b < B_; ++b)
    for (int r = 0; r < R_; ++r) {
      const int s = b * R_ + r;
      off_[s + 1] = off_[s] + 3 * bN_[b] + 6;
    }
  n_ = off_[S_];
  // per force point: placement in the batch vector, body, rigid-body weights
  std::vector<long long> ioff(Nt_), irstr(Nt_);
  std::vector<int> icstr(Nt_), rbody(Nt_), rlocal(Nt_);
  std::vector<double> xrel(3 * Nt_, 0.0), xm(3 * Nt_, 0.0), af(Nt_, 0.0);
  std::vector<long long> body_row0(B_ + 1, 0), soff(S_);
  std::vector<int> sn(S_);
  int64_t g0 = 0;
  for (int b = 0; b < B_; ++b) {
    const HostTree& t = *bodies[b].tree;
    const int64_t N = bN_[b];
    body_row0[b] = g0;
    for (int64_t i = 0; i < N; ++i) {
      const int64_t g = g0 + i;
      ioff[g] = off_[b * R_] + i;
      icstr[g] = (int)N;
      irstr[g] = 3 * N + 6;
      rbody[g] = b;
      rlocal[g] = (int)i;
      for (int d = 0; d < 3; ++d) xrel[3 * g + d] = bodies[b].rel_points[3 * i + d];
    }
    if (t.params.nearest) {
      // af = column sums of NN, xm = sum_q NN(q, n) X_q (genMatrixComponets.m:53-76)
      for (int64_t q = 0; q < t.q; ++q)
        for (int64_t k = t.nn_rowptr[q]; k < t.nn_rowptr[q + 1]; ++k) {
          const int64_t c = g0 + t.nn_col[k];
          const double wgt = t.nn_val[k];
          af[c] += wgt;
          for (int d = 0; d < 3; ++d) xm[3 * c + d] += wgt * bodies[b].rel_fine[3 * q + d];
        }
    } else {
      for (int64_t i = 0; i < N; ++i) {
        af[g0 + i] = 1.0;
        for (int d = 0; d < 3; ++d) xm[3 * (g0 + i) + d] = xrel[3 * (g0 + i) + d];
      }
    }
    for (int r = 0; r < R_; ++r) {
      soff[b * R_ + r] = off_[b * R_ + r];
      sn[b * R_ + r] = (int)N;
    }
    g0 += N;
  }
  body_row0[B_] = g0;
  cudaStream_t st = ctx_->stream;
  io_off_.upload(ioff, st);
  io_cstr_.upload(icstr, st);
  io_rstr_.upload(irstr, st);
  io_.off = io_off_.p;
  io_.cstr = io_cstr_.p;
  io_.rstr = io_rstr_.p;
  io_.nrows = Nt_;
  row_body_.upload(rbody, st);
  row_local_.upload(rlocal, st);
  sys_off_.upload(soff, st);
  sys_n_.upload(sn, st);
  xrel_.upload(xrel, st);
  xm_.upload(xm, st);
  af_.upload(af, st);
  body_row0_.upload(body_row0, st);
  FmmParams q = fp;
  q.max_rhs = std::min(R_, 6);
  // several right-hand sides per pass: the FP32 pair or Fourier-space M2L
  if (q.precision == NNK_PREC_MIXED && q.m2l_mode != 3) q.m2l_mode = 4;
  fp_ = q;
  fmm_.reset(new Fmm(ctx_, &forest_, q));
  fmm_->autotune(R_);
  NNK_CUDA(cudaStreamSynchronize(st));
}

BatchMobility::~BatchMobility() {
  for (auto& g : graph_)
    if (g) cudaGraphExecDestroy(g);
}

void BatchMobility::use_graphs(bool on) {
  graphs_on_ = on;
  for (auto& g : graph_) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
}

void BatchMobility::apply_with(Fmm& f, const double* x, double* y) {
  ++matvecs_;
  // the legacy default stream cannot be captured
  if (!graphs_on_ || f.profiling() || ctx_->stream == nullptr) {
    apply_raw(f, x, y);
    return;
  }
  cudaStream_t st = ctx_->stream;
  const int slot = &f == fmm_.get() ? 0 : 1;
  if (!gin_.p) {
    gin_.alloc(n_);
    gout_.alloc(n_);
  }
  if (graph_[slot] && graph_version_[slot] != f.version()) {  // a new or changed FMM in this slot
    cudaGraphExecDestroy(graph_[slot]);
    graph_[slot] = nullptr;
  }
  if (!graph_[slot]) {
    NNK_CUDA(cudaStreamSynchronize(st));
    NNK_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaGraph_t g = nullptr;
    try {
      apply_raw(f, gin_.p, gout_.p);
    } catch (...) {
      cudaStreamEndCapture(st, &g);
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      throw;
    }
    NNK_CUDA(cudaStreamEndCapture(st, &g));
    const cudaError_t e = cudaGraphInstantiate(&graph_[slot], g, 0);
    cudaGraphDestroy(g);
    NNK_CUDA(e);
    graph_version_[slot] = f.version();
  }
  NNK_CUDA(cudaMemcpyAsync(gin_.p, x, n_ * sizeof(double), cudaMemcpyDeviceToDevice, st));
  NNK_CUDA(cudaGraphLaunch(graph_[slot], st));
  NNK_CUDA(cudaMemcpyAsync(y, gout_.p, n_ * sizeof(double), cudaMemcpyDeviceToDevice, st));
}

void BatchMobility::apply_raw(Fmm& f, const double* x, double* y) {
  cudaStream_t st = ctx_->stream;
  f.apply_mapped(x, io_, y, io_, R_);
  batch_bt_kernel<<<blocks_for(Nt_), 256, 0, st>>>(Nt_, R_, row_body_.p, row_local_.p, sys_off_.p, sys_n_.p,
                                                    xrel_.p, x, y);
  NNK_CHECK_LAUNCH();
  batch_bsum_kernel<<<S_, 256, 0, st>>>(body_row0_.p, R_, sys_off_.p, sys_n_.p, af_.p, xm_.p, x, y);
  NNK_CHECK_LAUNCH();
}

void BatchMobility::apply(const double* x, double* y) { apply_with(*fmm_, x, y); }

void BatchMobility::set_refinement(bool fp64, int max_outer, double inner_tol) {
  if (!fp64) {
    ref64_.reset();
    return;
  }
  if (fp_.precision != NNK_PREC_MIXED) throw Error(NNK_E_ARG, "refinement needs a mixed-precision batch");
  ref_outer_ = max_outer > 0 ? max_outer : 12;
  ref_inner_tol_ = inner_tol > 0 ? inner_tol : 1e-4;
  if (!ref64_) {
    FmmParams q = fp_;
    q.precision = NNK_PREC_FP64;
    q.reg = fp_.reg > 0 ? fp_.reg : 1e-5;  // the same regularized operators as the mixed FMM
    ref64_.reset(new Fmm(ctx_, &forest_, q));
    ref64_->autotune(R_);
  }
}

void BatchMobility::solve_plain(const double* rhs, double* x, const nnk_solve_params& sp,
                                const std::vector<double>& tol, const std::vector<char>& act,
                                std::vector<nnk_solve_info>& info) {
  SegGmres g(ctx_, off_);
  SegGmres::Op op = [&](const double* in, double* out) { apply(in, out); };
  // bodies whose systems all converged drop out of the forest FMM
  if (deflate_) g.on_active = [&](const std::vector<char>& a) { fmm_->set_active_trees(body_flags(a).data()); };
  g.solve(op, rhs, x, tol, sp.maxit, sp.restart, act, info, /*confirm=*/!ref64_);
}

std::vector<char> BatchMobility::body_flags(const std::vector<char>& systems) const {
  std::vector<char> on(B_, 0);
  for (int s = 0; s < S_; ++s)
    if (systems[s]) on[s / R_] = 1;
  return on;
}

void BatchMobility::solve(const double* rhs, double* x, const nnk_solve_params& sp, nnk_solve_info* info) {
  cudaStream_t st = ctx_->stream;
  const double tol = sp.tol > 0 ? sp.tol : 1e-6;
  std::vector<nnk_solve_info> inf;
  if (!ref64_) {
    solve_plain(rhs, x, sp, std::vector<double>(S_, tol), std::vector<char>(S_, 1), inf);
    std::copy(inf.begin(), inf.end(), info);
    return;
  }
  // x = 0, r = b; repeat: A_mixed d ~= r (batched GMRES), x += d, r = b - A_fp64 x
  DBuf<double> r(n_), d(n_), ax(n_);
  SegGmres dots(ctx_, off_);
  NNK_CUDA(cudaMemsetAsync(x, 0, n_ * sizeof(double), st));
  NNK_CUDA(cudaMemcpyAsync(r.p, rhs, n_ * sizeof(double), cudaMemcpyDeviceToDevice, st));
  auto seg_norms = [&](const double* v) { return dots.norms(v); };
  const std::vector<double> nb = seg_norms(rhs);
  std::vector<double> relres(S_, 1.0);
  std::vector<nnk_solve_info> out(S_, nnk_solve_info{0, 0, 0.0});
  for (int s = 0; s < S_; ++s)
    if (nb[s] == 0.0) relres[s] = 0.0;
  for (int outer = 0; outer < ref_outer_; ++outer) {
    std::vector<double> itol(S_);
    std::vector<char> act(S_);
    int nact = 0;
    for (int s = 0; s < S_; ++s) {
      act[s] = relres[s] > tol;
      nact += act[s];
      itol[s] = std::max(ref_inner_tol_, std::min(0.5, tol / std::max(relres[s], 1e-300)));
    }
    if (!nact) break;
    solve_plain(r.p, d.p, sp, itol, act, inf);
    for (int s = 0; s < S_; ++s) out[s].iters += inf[s].iters;
    dev_axpby(ctx_, 1.0, x, 1.0, d.p, x, n_);
    // the FP64 residual of bodies with no system solved in this refinement pass is the
    // previous one (their x did not change): those trees are skipped and
    // their relres kept
    const std::vector<char> bon = deflate_ ? body_flags(act) : std::vector<char>(B_, 1);
    ref64_->set_active_trees(bon.data());
    apply_with(*ref64_, x, ax.p);
    ref64_->set_active_trees(nullptr);
    dev_axpby(ctx_, 1.0, rhs, -1.0, ax.p, r.p, n_);
    const std::vector<double> rn = seg_norms(r.p);
    for (int s = 0; s < S_; ++s)
      if (bon[s / R_]) relres[s] = nb[s] > 0 ? rn[s] / nb[s] : 0.0;
  }
  for (int s = 0; s < S_; ++s) {
    out[s].relres = relres[s];
    out[s].flag = relres[s] <= tol ? 0 : 1;
    info[s] = out[s];
  }
}

}  // namespace nnk
