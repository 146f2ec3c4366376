// extern "C" entry points of libnnkifmm.so (declared in include/nnkifmm.h).
#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <new>

#include <cublas_v2.h>
#include <cusolverDn.h>

#include "../../include/nnkifmm.h"
#include "common.h"
#include "fmm.h"
#include "probe.h"
#include "gmres.h"
#include "batch.h"
#include "mobility.h"
#include "tree.h"

struct nnk_tree {
  nnk_ctx* ctx;
  nnk::HostTree t;
};
struct nnk_fmm {
  nnk_ctx* ctx;
  const nnk_tree* tree;
  std::unique_ptr<nnk::Fmm> f;
};
struct nnk_mob {
  nnk_fmm* fmm;
  std::unique_ptr<nnk::Mobility> m;
};
struct nnk_batch {
  nnk_ctx* ctx;
  std::unique_ptr<nnk::BatchMobility> m;
  nnk::DBuf<double> io_in, io_out;
};

namespace {

int fail(nnk_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  return code;
}

#define API_TRY try {
#define API_CATCH(ctx)                                                       \
  }                                                                          \
  catch (const nnk::Error& e) { return fail(ctx, e.code, e.what()); }        \
  catch (const std::bad_alloc&) { return fail(ctx, NNK_E_OOM, "out of host memory"); } \
  catch (const std::exception& e) { return fail(ctx, NNK_E_ARG, e.what()); } \
  return NNK_OK;

void ctx_retain(nnk_ctx* c) { c->refs.fetch_add(1, std::memory_order_relaxed); }

void ctx_release(nnk_ctx* c) {
  if (c->refs.fetch_sub(1, std::memory_order_acq_rel) != 1) return;
  if (c->has_gpu) {
    cudaSetDevice(c->device);
    if (c->dn_solver) cusolverDnDestroy(static_cast<cusolverDnHandle_t>(c->dn_solver));
    if (c->blas) cublasDestroy(static_cast<cublasHandle_t>(c->blas));
    if (c->blas_ws) cudaFree(c->blas_ws);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    cudaGetLastError();  // an error here must not surface at a later call's launch check
  }
  delete c;
}

void need_gpu(nnk_ctx* ctx) {
  if (!ctx->has_gpu) throw nnk::Error(NNK_E_CUDA, "no CUDA device available: the FMM runs only on the GPU");
  NNK_CUDA(cudaSetDevice(ctx->device));
  // a launch check reports the last runtime error of this thread; drop any
  // error left by an earlier call that its caller already handled
  cudaGetLastError();
}

// Copies a host or device input to device memory owned by `buf` if needed.
const double* stage_in(nnk_ctx* ctx, nnk::DBuf<double>& buf, const double* p, size_t count, int on_device) {
  if (on_device) return p;
  if (buf.n < count) buf.alloc(count);
  if (count)
    NNK_CUDA(cudaMemcpyAsync(buf.p, p, count * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  return buf.p;
}
double* stage_out(nnk::DBuf<double>& buf, double* p, size_t count, int on_device) {
  if (on_device) return p;
  if (buf.n < count) buf.alloc(count);
  return buf.p;
}
void finish_out(nnk_ctx* ctx, nnk::DBuf<double>& buf, double* p, size_t count, int on_device) {
  if (!on_device && count)
    NNK_CUDA(cudaMemcpyAsync(p, buf.p, count * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  if (!on_device) NNK_CUDA(cudaStreamSynchronize(ctx->stream));
}
// Device-side failures of the call's launches (a bounded wait that gave up)
// become the call's status: after a host-output call, which has waited for
// the stream anyway, or after a solve (synchronized at every step), every
// flag is read; a device-output call reads the flags whose copies have
// completed, and a later call on the same FMM reports the rest.
void device_errors(nnk::Fmm& F, int waited) {
  if (waited) F.check_errors();
  else F.poll_errors();
}
// The same for the FMMs of a forest batch (its matvec and, with FP64
// refinement, the FP64 residual FMM).
void batch_errors(nnk::BatchMobility& M, int waited) {
  device_errors(M.fmm(), waited);
  if (M.ref64()) device_errors(*M.ref64(), waited);
}

}  // namespace

extern "C" {

const char* nnk_version(void) { return "nnkifmm 0.1 sm_100a"; }

int nnk_ctx_create(int32_t device, nnk_ctx** out) {
  if (!out) return NNK_E_ARG;
  nnk_ctx* c = new (std::nothrow) nnk_ctx();
  if (!c) return NNK_E_OOM;
  c->device = device;
  int count = 0;
  if (cudaGetDeviceCount(&count) == cudaSuccess && device >= 0 && device < count &&
      cudaSetDevice(device) == cudaSuccess) {
    c->has_gpu = true;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete c;
      return NNK_E_CUDA;
    }
    c->own_stream = true;
  } else {
    cudaGetLastError();  // clear the sticky "no device" error
    c->has_gpu = false;
  }
  *out = c;
  return NNK_OK;
}

int nnk_ctx_destroy(nnk_ctx* ctx) {
  if (!ctx) return NNK_E_ARG;
  ctx_release(ctx);
  return NNK_OK;
}

int nnk_ctx_set_stream(nnk_ctx* ctx, void* stream) {
  if (!ctx) return NNK_E_ARG;
  API_TRY
  need_gpu(ctx);
  if (ctx->own_stream && ctx->stream) NNK_CUDA(cudaStreamDestroy(ctx->stream));
  ctx->stream = (cudaStream_t)stream;
  ctx->own_stream = false;
  API_CATCH(ctx)
}

int nnk_ctx_synchronize(nnk_ctx* ctx) {
  if (!ctx) return NNK_E_ARG;
  API_TRY
  need_gpu(ctx);
  NNK_CUDA(cudaStreamSynchronize(ctx->stream));
  API_CATCH(ctx)
}

const char* nnk_last_error(const nnk_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

static int nearest_common(nnk_ctx* ctx, const double* coarse, int64_t n, const double* fine, int64_t q,
                          int64_t* nnz, int64_t* rowptr, int32_t* col, double* val, bool host) {
  if (!ctx || !nnz || n < 0 || q < 0 || (n && !coarse) || (q && !fine)) return fail(ctx, NNK_E_ARG, "bad arguments");
  API_TRY
  std::vector<int64_t> rp;
  std::vector<int32_t> cl;
  std::vector<double> vl;
  if (!host && ctx->has_gpu) {
    need_gpu(ctx);
    nnk::nearest_matrix_gpu(ctx, coarse, n, fine, q, rp, cl, vl);
  } else {
    nnk::nearest_matrix(coarse, n, fine, q, rp, cl, vl);
  }
  *nnz = rp.empty() ? 0 : rp.back();
  if (rowptr) {
    std::memcpy(rowptr, rp.data(), rp.size() * sizeof(int64_t));
    if (col) std::memcpy(col, cl.data(), cl.size() * sizeof(int32_t));
    if (val) std::memcpy(val, vl.data(), vl.size() * sizeof(double));
  }
  API_CATCH(ctx)
}

int nnk_nearest_matrix(nnk_ctx* ctx, const double* coarse, int64_t n, const double* fine, int64_t q,
                       int64_t* nnz, int64_t* rowptr, int32_t* col, double* val) {
  return nearest_common(ctx, coarse, n, fine, q, nnz, rowptr, col, val, false);
}

int nnk_nearest_matrix_host(nnk_ctx* ctx, const double* coarse, int64_t n, const double* fine, int64_t q,
                            int64_t* nnz, int64_t* rowptr, int32_t* col, double* val) {
  return nearest_common(ctx, coarse, n, fine, q, nnz, rowptr, col, val, true);
}

int nnk_nearest_reference_weights(nnk_ctx* ctx, int64_t q, const int64_t* rowptr, const int32_t* col, double* val,
                                  double block_size) {
  if (q < 0 || (q > 0 && (!rowptr || !col || !val)) || !(block_size > 0))
    return fail(ctx, NNK_E_ARG, "bad arguments");
  API_TRY
  nnk::nearest_reference_weights(q, rowptr, col, val, block_size);
  API_CATCH(ctx)
}

int nnk_tree_build(nnk_ctx* ctx, const double* pot, int64_t n_pot, const double* tgt, int64_t n_tgt,
                   const double* fine, int64_t q, const int64_t* nn_rowptr, const int32_t* nn_col,
                   const double* nn_val, const nnk_tree_params* params, nnk_tree** out) {
  if (!ctx || !out) return NNK_E_ARG;
  API_TRY
  nnk::TreeParams p;
  if (params) {
    p.node_capacity = params->node_capacity;
    p.max_depth = params->max_depth;
    p.nearest = params->nearest;
    p.builder = params->builder;
  }
  if (p.builder < 0 || p.builder > 2) return fail(ctx, NNK_E_ARG, "builder must be 0, 1 or 2");
  if (p.builder == 2 && !ctx->has_gpu) return fail(ctx, NNK_E_CUDA, "no CUDA device available for the GPU builder");
  nnk_ctx* gpu = (p.builder == 2 || (p.builder == 0 && ctx->has_gpu)) ? ctx : nullptr;
  if (gpu) need_gpu(ctx);
  std::unique_ptr<nnk_tree> t(new nnk_tree());
  t->ctx = ctx;
  std::string msg;
  const int rc = nnk::build_tree(pot, n_pot, tgt, n_tgt, fine, q, nn_rowptr, nn_col, nn_val, p, t->t, msg, gpu);
  if (rc != NNK_OK) return fail(ctx, rc, msg);
  *out = t.release();
  ctx_retain(ctx);
  API_CATCH(ctx)
}

int nnk_tree_info_get(const nnk_tree* tree, nnk_tree_info* info) {
  if (!tree || !info) return NNK_E_ARG;
  const nnk::HostTree& t = tree->t;
  std::memset(info, 0, sizeof(*info));
  info->num_points = t.n;
  info->num_potentials = t.n_pot;
  info->num_targets = t.n_tgt;
  info->num_fine = t.q;
  info->nn_nnz = t.nn_rowptr.empty() ? 0 : t.nn_rowptr.back();
  info->source_entries = t.src_start.empty() ? 0 : t.src_start.back();
  info->u_total = (int64_t)t.U.idx.size();
  info->v_total = (int64_t)t.V.idx.size();
  info->w_total = (int64_t)t.W.idx.size();
  info->x_total = (int64_t)t.X.idx.size();
  info->node_count = t.nodes;
  info->max_level = t.max_level;
  info->node_capacity = t.capacity;
  info->nearest = t.params.nearest;
  return NNK_OK;
}

int nnk_tree_export_nodes(const nnk_tree* tree, int32_t* level, int32_t* parent, int32_t* children,
                          double* corners, int32_t* point_index) {
  if (!tree) return NNK_E_ARG;
  const nnk::HostTree& t = tree->t;
  for (int32_t i = 0; i < t.nodes; ++i) {
    if (level) level[i] = t.level[i];
    if (parent) parent[i] = t.parent[i] + 1;  // root parent 0 (OcTree.m:102)
    if (children)
      for (int k = 0; k < 8; ++k) children[8 * i + k] = t.child0[i] < 0 ? 0 : t.child0[i] + k + 1;
    if (corners) std::memcpy(corners + 6 * i, &t.corners[6 * i], 6 * sizeof(double));
  }
  if (point_index)
    for (int64_t k = 0; k < t.n; ++k) point_index[k] = t.point_index[k] + 1;
  return NNK_OK;
}

int nnk_tree_export_points(const nnk_tree* tree, double* points, uint8_t* potentials, uint8_t* targets) {
  if (!tree) return NNK_E_ARG;
  const nnk::HostTree& t = tree->t;
  if (points) std::memcpy(points, t.pts.data(), t.pts.size() * sizeof(double));
  if (potentials) std::memcpy(potentials, t.is_pot.data(), t.is_pot.size());
  if (targets) std::memcpy(targets, t.is_tgt.data(), t.is_tgt.size());
  return NNK_OK;
}

int nnk_tree_export_list(const nnk_tree* tree, int32_t which, int64_t* offsets, int32_t* ids) {
  if (!tree || which < 0 || which > 3) return NNK_E_ARG;
  const nnk::HostTree& t = tree->t;
  const nnk::Csr& L = which == 0 ? t.U : which == 1 ? t.V : which == 2 ? t.W : t.X;
  if (offsets) std::memcpy(offsets, L.off.data(), L.off.size() * sizeof(int64_t));
  if (ids)
    for (size_t k = 0; k < L.idx.size(); ++k) ids[k] = L.idx[k] + 1;
  return NNK_OK;
}

int nnk_tree_destroy(nnk_tree* tree) {
  if (!tree) return NNK_OK;
  nnk_ctx* c = tree->ctx;
  delete tree;
  ctx_release(c);
  return NNK_OK;
}

int nnk_fmm_create(nnk_ctx* ctx, const nnk_tree* tree, const nnk_fmm_params* params, nnk_fmm** out) {
  if (!ctx || !tree || !params || !out) return NNK_E_ARG;
  API_TRY
  need_gpu(ctx);
  nnk::FmmParams p;
  p.eps = params->eps;
  p.mu = params->mu;
  p.res = params->corona_res ? params->corona_res : 6;
  p.shells = params->corona_shells ? params->corona_shells : 1;
  p.precision = params->precision;
  p.m2l_mode = params->m2l_mode;
  p.reg = params->reg;
  if (p.precision != NNK_PREC_FP64 && p.precision != NNK_PREC_MIXED && p.precision != NNK_PREC_NEAR32)
    return fail(ctx, NNK_E_ARG, "unknown precision mode");
  std::unique_ptr<nnk_fmm> f(new nnk_fmm());
  f->ctx = ctx;
  f->tree = tree;
  f->f.reset(new nnk::Fmm(ctx, &tree->t, p));
  *out = f.release();
  ctx_retain(ctx);
  API_CATCH(ctx)
}

static int fmm_apply_common(nnk_fmm* fmm, const double* in, double* out, int32_t layout, int32_t nrhs,
                            int32_t on_device, int which) {
  if (!fmm || !in || !out || nrhs < 1 || (layout != NNK_LAYOUT_ROWS && layout != NNK_LAYOUT_BLOCKED))
    return fail(fmm ? fmm->ctx : nullptr, NNK_E_ARG, "bad arguments");
  nnk_ctx* ctx = fmm->ctx;
  API_TRY
  need_gpu(ctx);
  nnk::Fmm& F = *fmm->f;
  const nnk::HostTree& t = F.tree();
  const size_t nin = (size_t)nrhs * 3 * (which >= 2 ? t.n_tgt : t.n_pot);
  const size_t nout = (size_t)nrhs * 3 * t.n_tgt;
  const double* din = stage_in(ctx, F.io_in, in, nin, on_device);
  double* dout = stage_out(F.io_out, out, nout, on_device);
  if (which == 0) F.apply(din, dout, layout, nrhs);
  else if (which == 1) F.sparse().apply(din, dout, layout, nrhs);
  else if (which == 2) F.reduced_apply(din, dout, layout);
  else F.reduced_solve(din, dout, layout);
  finish_out(ctx, F.io_out, out, nout, on_device);
  device_errors(F, !on_device);
  API_CATCH(ctx)
}

int nnk_fmm_apply(nnk_fmm* fmm, const double* in, double* out, int32_t layout, int32_t nrhs,
                  int32_t on_device) {
  return fmm_apply_common(fmm, in, out, layout, nrhs, on_device, 0);
}
int nnk_fmm_apply_sparse(nnk_fmm* fmm, const double* in, double* out, int32_t layout, int32_t nrhs,
                         int32_t on_device) {
  return fmm_apply_common(fmm, in, out, layout, nrhs, on_device, 1);
}
int nnk_fmm_reduced_apply(nnk_fmm* fmm, const double* in, double* out, int32_t layout, int32_t on_device) {
  return fmm_apply_common(fmm, in, out, layout, 1, on_device, 2);
}
int nnk_fmm_reduced_solve(nnk_fmm* fmm, const double* in, double* out, int32_t layout, int32_t on_device) {
  return fmm_apply_common(fmm, in, out, layout, 1, on_device, 3);
}

int nnk_fmm_apply_adjoint(nnk_fmm* fmm, const double* in, double* out, int32_t layout, int32_t nrhs,
                          int32_t on_device) {
  if (!fmm || !in || !out || nrhs < 1 || (layout != NNK_LAYOUT_ROWS && layout != NNK_LAYOUT_BLOCKED))
    return fail(fmm ? fmm->ctx : nullptr, NNK_E_ARG, "bad arguments");
  nnk_ctx* ctx = fmm->ctx;
  API_TRY
  need_gpu(ctx);
  nnk::Fmm& F = *fmm->f;
  const nnk::HostTree& t = F.tree();
  const size_t nin = (size_t)nrhs * 3 * t.n_tgt, nout = (size_t)nrhs * 3 * t.n_pot;
  const double* din = stage_in(ctx, F.io_in, in, nin, on_device);
  double* dout = stage_out(F.io_out, out, nout, on_device);
  F.apply_adjoint(din, dout, layout, nrhs);
  finish_out(ctx, F.io_out, out, nout, on_device);
  device_errors(F, !on_device);
  API_CATCH(ctx)
}

int nnk_fmm_autotune(nnk_fmm* fmm, int32_t nrhs, double* ms_before, double* ms_after) {
  if (!fmm || nrhs < 1) return NNK_E_ARG;
  nnk_ctx* ctx = fmm->ctx;
  API_TRY
  need_gpu(ctx);
  const auto r = fmm->f->autotune(nrhs);
  if (ms_before) *ms_before = r.first;
  if (ms_after) *ms_after = r.second;
  API_CATCH(ctx)
}

int nnk_fmm_set_eps(nnk_fmm* fmm, double eps) {
  if (!fmm) return NNK_E_ARG;
  nnk_ctx* ctx = fmm->ctx;
  API_TRY
  need_gpu(ctx);
  fmm->f->set_eps(eps);
  API_CATCH(ctx)
}

int nnk_fmm_source_count(const nnk_fmm* fmm, int64_t* count) {
  if (!fmm || !count) return NNK_E_ARG;
  *count = fmm->f->source_origins();
  return NNK_OK;
}

int nnk_fmm_grad_positions(nnk_fmm* fmm, const double* forces, const double* weights, int32_t layout,
                           double* grad_targets, double* grad_sources, int32_t on_device) {
  if (!fmm || !forces || !weights || (!grad_targets && !grad_sources) ||
      (layout != NNK_LAYOUT_ROWS && layout != NNK_LAYOUT_BLOCKED))
    return fail(fmm ? fmm->ctx : nullptr, NNK_E_ARG, "bad arguments");
  nnk_ctx* ctx = fmm->ctx;
  API_TRY
  need_gpu(ctx);
  nnk::Fmm& F = *fmm->f;
  const nnk::HostTree& t = F.tree();
  const size_t nf = 3 * (size_t)t.n_pot, nw = 3 * (size_t)t.n_tgt, ns = 3 * (size_t)F.source_origins();
  nnk::DBuf<double> buf;
  double *df = nullptr, *dw = nullptr, *dgt = grad_targets, *dgs = grad_sources;
  if (!on_device) {
    buf.alloc(nf + 2 * nw + ns);
    df = buf.p;
    dw = buf.p + nf;
    NNK_CUDA(cudaMemcpyAsync(df, forces, nf * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    NNK_CUDA(cudaMemcpyAsync(dw, weights, nw * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    dgt = grad_targets ? buf.p + nf + nw : nullptr;
    dgs = grad_sources ? buf.p + nf + 2 * nw : nullptr;
  }
  F.grad_positions(on_device ? forces : df, on_device ? weights : dw, layout, dgt, dgs);
  if (!on_device) {
    if (grad_targets)
      NNK_CUDA(cudaMemcpyAsync(grad_targets, dgt, nw * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (grad_sources)
      NNK_CUDA(cudaMemcpyAsync(grad_sources, dgs, ns * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  }
  NNK_CUDA(cudaStreamSynchronize(ctx->stream));
  API_CATCH(ctx)
}

int nnk_fmm_stats_get(const nnk_fmm* fmm, nnk_fmm_stats* stats) {
  if (!fmm || !stats) return NNK_E_ARG;
  *stats = fmm->f->stats();
  stats->folded = fmm->f->folded() ? 1 : 0;
  stats->m2m_product_pairs = fmm->f->m2m_form() ? fmm->f->m2m_pairs() : 0;
  stats->l2l_product_pairs = fmm->f->m2m_form() == 2 ? fmm->f->m2m_pairs() : 0;
  return NNK_OK;
}

int nnk_measure_l2_read(nnk_ctx* ctx, double* gbs) {
  if (!ctx || !gbs) return NNK_E_ARG;
  API_TRY
  need_gpu(ctx);
  *gbs = nnk::measure_l2_read_gbs(ctx->stream);
  API_CATCH(ctx)
}

int nnk_fmm_setup_times(const nnk_fmm* fmm, double* ms, int32_t n) {
  if (!fmm || (!ms && n > 0) || n < 0) return NNK_E_ARG;
  for (int i = 0; i < n && i < NNK_SETUP_COUNT; ++i) ms[i] = fmm->f->setup_ms()[i];
  return NNK_OK;
}

int nnk_fmm_set_c2e(nnk_fmm* fmm, int32_t mode) {
  if (!fmm) return NNK_E_ARG;
  nnk_ctx* ctx = fmm->ctx;
  API_TRY
  need_gpu(ctx);
  fmm->f->set_c2e_mode(mode);
  API_CATCH(ctx)
}

int nnk_fmm_c2e_mode(const nnk_fmm* fmm, int32_t* mode) {
  if (!fmm || !mode) return NNK_E_ARG;
  *mode = fmm->f->c2e_mode();
  return NNK_OK;
}

int nnk_fmm_set_m2m_form(nnk_fmm* fmm, int32_t form) {
  if (!fmm) return NNK_E_ARG;
  nnk_ctx* ctx = fmm->ctx;
  API_TRY
  need_gpu(ctx);
  fmm->f->set_m2m_form(form);
  API_CATCH(ctx)
}

int nnk_fmm_set_fold(nnk_fmm* fmm, int32_t on) {
  if (!fmm) return NNK_E_ARG;
  nnk_ctx* ctx = fmm->ctx;
  API_TRY
  need_gpu(ctx);
  fmm->f->set_fold(on);
  API_CATCH(ctx)
}

int nnk_fmm_profile(nnk_fmm* fmm, int32_t enable) {
  if (!fmm) return NNK_E_ARG;
  fmm->f->set_profile(enable != 0);
  return NNK_OK;
}

int nnk_fmm_profile_read(nnk_fmm* fmm, double* ms, int64_t* launches) {
  if (!fmm) return NNK_E_ARG;
  nnk_ctx* ctx = fmm->ctx;
  API_TRY
  need_gpu(ctx);
  fmm->f->read_profile(ms, launches);
  API_CATCH(ctx)
}

int nnk_fmm_grad_eps(nnk_fmm* fmm, const double* forces, const double* weights, int32_t layout, double* out,
                     int32_t on_device) {
  if (!fmm || !forces || !weights || !out || (layout != NNK_LAYOUT_ROWS && layout != NNK_LAYOUT_BLOCKED))
    return fail(fmm ? fmm->ctx : nullptr, NNK_E_ARG, "bad arguments");
  nnk_ctx* ctx = fmm->ctx;
  API_TRY
  need_gpu(ctx);
  nnk::Fmm& F = *fmm->f;
  const nnk::HostTree& t = F.tree();
  nnk::DBuf<double> wbuf;
  const double* df = stage_in(ctx, F.io_in, forces, 3 * (size_t)t.n_pot, on_device);
  const double* dw = stage_in(ctx, wbuf, weights, 3 * (size_t)t.n_tgt, on_device);
  *out = F.grad_eps(df, dw, layout);
  API_CATCH(ctx)
}

int nnk_fmm_test_wait_timeout(nnk_fmm* fmm, uint32_t polls) {
  if (!fmm || polls == 0) return fail(fmm ? fmm->ctx : nullptr, NNK_E_ARG, "bad arguments");
  nnk_ctx* ctx = fmm->ctx;
  API_TRY
  need_gpu(ctx);
  const int flag = fmm->f->m2l_stall_probe(polls);
  if (flag)
    return fail(ctx, NNK_E_TIMEOUT, "tensor-core M2L gave up a bounded wait (flag " + std::to_string(flag) + ")");
  return fail(ctx, NNK_E_STATE, "the probe's bounded wait did not give up");
  API_CATCH(ctx)
}

int nnk_fmm_destroy(nnk_fmm* fmm) {
  if (!fmm) return NNK_E_ARG;
  nnk_ctx* c = fmm->ctx;
  if (c->has_gpu) cudaSetDevice(c->device);
  delete fmm;
  if (c->has_gpu) cudaGetLastError();  // destroy errors are not reported
  ctx_release(c);
  return NNK_OK;
}

int nnk_fmm_solve(nnk_fmm* fmm, const double* b, double* x, int32_t layout, const nnk_solve_params* sp,
                  nnk_solve_info* info, int32_t on_device) {
  if (!fmm || !b || !x || !sp) return fail(fmm ? fmm->ctx : nullptr, NNK_E_ARG, "bad arguments");
  nnk_ctx* ctx = fmm->ctx;
  API_TRY
  need_gpu(ctx);
  nnk::Fmm& F = *fmm->f;
  const nnk::HostTree& t = F.tree();
  if (t.n_pot != t.n_tgt) return fail(ctx, NNK_E_ARG, "solve needs potentials == targets");
  const size_t n = 3 * (size_t)t.n_tgt;
  const double* db = stage_in(ctx, F.io_in, b, n, on_device);
  double* dx = stage_out(F.io_out, x, n, on_device);
  nnk_solve_info inf{};
  nnk::Gmres g(ctx, (int64_t)n);
  auto op = [&](const double* in, double* outp) { F.apply(in, outp, layout, 1); };
  g.solve(op, nullptr, db, dx, *sp, inf);
  finish_out(ctx, F.io_out, x, n, on_device);
  device_errors(F, 1);
  if (info) *info = inf;
  if (inf.flag != 0) return fail(ctx, NNK_E_NOCONV, "gmres stopped at maxit above tol");
  API_CATCH(ctx)
}

int nnk_mob_create(nnk_fmm* fmm, int32_t nbodies, const int64_t* body_start, const int64_t* fine_start,
                   const double* rel_points, const double* rel_fine, nnk_mob** out) {
  if (!fmm || !out || nbodies < 0 || !body_start) return fail(fmm ? fmm->ctx : nullptr, NNK_E_ARG, "bad arguments");
  nnk_ctx* ctx = fmm->ctx;
  API_TRY
  need_gpu(ctx);
  std::unique_ptr<nnk_mob> m(new nnk_mob());
  m->fmm = fmm;
  m->m.reset(new nnk::Mobility(fmm->f.get(), nbodies, body_start, fine_start, rel_points, rel_fine));
  *out = m.release();
  API_CATCH(ctx)
}

int nnk_mob_apply(nnk_mob* mob, const double* x, double* y, int32_t on_device) {
  if (!mob || !x || !y) return NNK_E_ARG;
  nnk_ctx* ctx = mob->fmm->ctx;
  API_TRY
  need_gpu(ctx);
  nnk::Mobility& M = *mob->m;
  const size_t n = (size_t)M.size();
  const double* dx = stage_in(ctx, M.io_in, x, n, on_device);
  double* dy = stage_out(M.io_out, y, n, on_device);
  M.apply(dx, dy);
  finish_out(ctx, M.io_out, y, n, on_device);
  device_errors(*mob->fmm->f, !on_device);
  API_CATCH(ctx)
}

int nnk_mob_use_graphs(nnk_mob* mob, int32_t enable) {
  if (!mob) return NNK_E_ARG;
  nnk_ctx* ctx = mob->fmm->ctx;
  API_TRY
  need_gpu(ctx);
  mob->m->use_graphs(enable != 0);
  API_CATCH(ctx)
}

int nnk_mob_precon(nnk_mob* mob, const double* x, double* y, int32_t on_device) {
  if (!mob || !x || !y) return NNK_E_ARG;
  nnk_ctx* ctx = mob->fmm->ctx;
  API_TRY
  need_gpu(ctx);
  nnk::Mobility& M = *mob->m;
  const size_t n = (size_t)M.size();
  const double* dx = stage_in(ctx, M.io_in, x, n, on_device);
  double* dy = stage_out(M.io_out, y, n, on_device);
  M.precon(dx, dy);
  finish_out(ctx, M.io_out, y, n, on_device);
  device_errors(*mob->fmm->f, !on_device);
  API_CATCH(ctx)
}

int nnk_mob_solve(nnk_mob* mob, const double* rhs, double* x, const nnk_solve_params* sp, int32_t precondition,
                  nnk_solve_info* info, int32_t on_device) {
  if (!mob || !rhs || !x || !sp) return NNK_E_ARG;
  nnk_ctx* ctx = mob->fmm->ctx;
  API_TRY
  need_gpu(ctx);
  nnk::Mobility& M = *mob->m;
  const size_t n = (size_t)M.size();
  const double* db = stage_in(ctx, M.io_in, rhs, n, on_device);
  double* dx = stage_out(M.io_out, x, n, on_device);
  nnk_solve_info inf{};
  M.solve(db, dx, *sp, precondition != 0, inf);
  finish_out(ctx, M.io_out, x, n, on_device);
  device_errors(*mob->fmm->f, 1);
  if (info) *info = inf;
  if (inf.flag != 0) return fail(ctx, NNK_E_NOCONV, "gmres stopped at maxit above tol");
  API_CATCH(ctx)
}

int nnk_mob_set_refinement(nnk_mob* mob, nnk_fmm* fp64, int32_t max_outer, double inner_tol) {
  if (!mob) return NNK_E_ARG;
  nnk_ctx* ctx = mob->fmm->ctx;
  API_TRY
  if (fp64 && fp64->f->params().precision != NNK_PREC_FP64)
    return fail(ctx, NNK_E_ARG, "refinement needs an FP64 FMM");
  mob->m->set_refinement(fp64 ? fp64->f.get() : nullptr, max_outer, inner_tol);
  API_CATCH(ctx)
}

int nnk_mob_apply_adjoint(nnk_mob* mob, const double* x, double* y, int32_t on_device) {
  if (!mob || !x || !y) return NNK_E_ARG;
  nnk_ctx* ctx = mob->fmm->ctx;
  API_TRY
  need_gpu(ctx);
  nnk::Mobility& M = *mob->m;
  const size_t n = (size_t)M.size();
  const double* dx = stage_in(ctx, M.io_in, x, n, on_device);
  double* dy = stage_out(M.io_out, y, n, on_device);
  M.apply_adjoint(dx, dy);
  finish_out(ctx, M.io_out, y, n, on_device);
  device_errors(*mob->fmm->f, !on_device);
  API_CATCH(ctx)
}

int nnk_mob_apply_fmm(nnk_mob* mob, nnk_fmm* fmm, const double* x, double* y, int32_t on_device) {
  if (!mob || !fmm || !x || !y) return NNK_E_ARG;
  nnk_ctx* ctx = mob->fmm->ctx;
  API_TRY
  need_gpu(ctx);
  if (&fmm->f->tree() != &mob->fmm->f->tree()) return fail(ctx, NNK_E_ARG, "the FMM must share the mobility tree");
  nnk::Mobility& M = *mob->m;
  const size_t n = (size_t)M.size();
  const double* dx = stage_in(ctx, M.io_in, x, n, on_device);
  double* dy = stage_out(M.io_out, y, n, on_device);
  M.apply_with(fmm->f.get(), dx, dy);
  finish_out(ctx, M.io_out, y, n, on_device);
  device_errors(*fmm->f, !on_device);
  API_CATCH(ctx)
}

int nnk_mob_solve_adjoint(nnk_mob* mob, const double* rhs, double* x, const nnk_solve_params* sp,
                          nnk_solve_info* info, int32_t on_device) {
  if (!mob || !rhs || !x || !sp) return NNK_E_ARG;
  nnk_ctx* ctx = mob->fmm->ctx;
  API_TRY
  need_gpu(ctx);
  nnk::Mobility& M = *mob->m;
  const size_t n = (size_t)M.size();
  const double* db = stage_in(ctx, M.io_in, rhs, n, on_device);
  double* dx = stage_out(M.io_out, x, n, on_device);
  nnk_solve_info inf{};
  M.solve_adjoint(db, dx, *sp, inf);
  finish_out(ctx, M.io_out, x, n, on_device);
  device_errors(*mob->fmm->f, 1);
  if (info) *info = inf;
  if (inf.flag != 0) return fail(ctx, NNK_E_NOCONV, "gmres stopped at maxit above tol");
  API_CATCH(ctx)
}

int nnk_mob_grad_positions(nnk_mob* mob, const double* z, const double* lam, double* grad_points,
                           double* grad_fine, int32_t on_device) {
  if (!mob || !z || !lam || !grad_points) return NNK_E_ARG;
  nnk_ctx* ctx = mob->fmm->ctx;
  API_TRY
  need_gpu(ctx);
  nnk::Mobility& M = *mob->m;
  const nnk::HostTree& t = mob->fmm->f->tree();
  const size_t n = (size_t)M.size(), nx = 3 * (size_t)t.n_tgt;
  const size_t ny = t.params.nearest ? 3 * (size_t)t.q : 0;
  if (on_device) {
    M.grad_positions(z, lam, grad_points, grad_fine);
  } else {
    nnk::DBuf<double> buf(2 * n + nx + std::max<size_t>(ny, 1));
    NNK_CUDA(cudaMemcpyAsync(buf.p, z, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    NNK_CUDA(cudaMemcpyAsync(buf.p + n, lam, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    double* gx = buf.p + 2 * n;
    double* gy = grad_fine && ny ? gx + nx : nullptr;
    M.grad_positions(buf.p, buf.p + n, gx, gy);
    NNK_CUDA(cudaMemcpyAsync(grad_points, gx, nx * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (gy) NNK_CUDA(cudaMemcpyAsync(grad_fine, gy, ny * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    NNK_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  API_CATCH(ctx)
}

int nnk_mob_grad_eps(nnk_mob* mob, nnk_fmm* fp64, const double* z, const double* lam, double* out,
                     int32_t on_device) {
  if (!mob || !z || !lam || !out) return NNK_E_ARG;
  nnk_ctx* ctx = mob->fmm->ctx;
  API_TRY
  need_gpu(ctx);
  if (fp64 && &fp64->f->tree() != &mob->fmm->f->tree())
    return fail(ctx, NNK_E_ARG, "the FMM must share the mobility tree");
  nnk::Mobility& M = *mob->m;
  nnk::Fmm& F = fp64 ? *fp64->f : *mob->fmm->f;
  const size_t n = (size_t)M.size();
  nnk::DBuf<double> lbuf;
  const double* dz = stage_in(ctx, M.io_in, z, n, on_device);
  const double* dl = stage_in(ctx, lbuf, lam, n, on_device);
  // [f (3N, blocked) | U | Omega]: the FMM block reads the first 3N values
  *out = -F.grad_eps(dz, dl, NNK_LAYOUT_BLOCKED);
  API_CATCH(ctx)
}

int nnk_mob_destroy(nnk_mob* mob) {
  delete mob;
  return NNK_OK;
}

int nnk_batch_create(nnk_ctx* ctx, int32_t nbodies, nnk_tree* const* trees, const double* const* rel_points,
                     const double* const* rel_fine, const nnk_fmm_params* params, int32_t nrhs, nnk_batch** out) {
  if (!ctx || !trees || !rel_points || !params || !out || nbodies < 1 || nrhs < 1)
    return fail(ctx, NNK_E_ARG, "bad arguments");
  API_TRY
  need_gpu(ctx);
  std::vector<nnk::BatchBody> bodies(nbodies);
  for (int b = 0; b < nbodies; ++b) {
    if (!trees[b] || !rel_points[b]) return fail(ctx, NNK_E_ARG, "null tree or rel_points");
    bodies[b] = nnk::BatchBody{&trees[b]->t, rel_points[b], rel_fine ? rel_fine[b] : nullptr};
  }
  nnk::FmmParams p;
  p.eps = params->eps;
  p.mu = params->mu;
  p.res = params->corona_res > 0 ? params->corona_res : 6;
  p.shells = params->corona_shells > 0 ? params->corona_shells : 1;
  p.precision = params->precision;
  p.m2l_mode = params->m2l_mode;
  p.reg = params->reg;
  if (p.precision != NNK_PREC_FP64 && p.precision != NNK_PREC_MIXED) return fail(ctx, NNK_E_ARG, "bad precision");
  std::unique_ptr<nnk_batch> bt(new nnk_batch());
  bt->ctx = ctx;
  bt->m.reset(new nnk::BatchMobility(ctx, bodies, p, nrhs));
  *out = bt.release();
  ctx_retain(ctx);
  API_CATCH(ctx)
}

int nnk_batch_layout(const nnk_batch* batch, int64_t* length, int64_t* offsets) {
  if (!batch) return NNK_E_ARG;
  if (length) *length = batch->m->size();
  if (offsets) {
    const auto& o = batch->m->offsets();
    std::copy(o.begin(), o.end(), offsets);
  }
  return NNK_OK;
}

int nnk_batch_apply(nnk_batch* batch, const double* x, double* y, int32_t on_device) {
  if (!batch || !x || !y) return NNK_E_ARG;
  nnk_ctx* ctx = batch->ctx;
  API_TRY
  need_gpu(ctx);
  const size_t n = (size_t)batch->m->size();
  const double* dx = stage_in(ctx, batch->io_in, x, n, on_device);
  double* dy = stage_out(batch->io_out, y, n, on_device);
  batch->m->apply(dx, dy);
  finish_out(ctx, batch->io_out, y, n, on_device);
  batch_errors(*batch->m, !on_device);
  API_CATCH(ctx)
}

int nnk_batch_solve(nnk_batch* batch, const double* rhs, double* x, const nnk_solve_params* sp, nnk_solve_info* info,
                    int32_t on_device) {
  if (!batch || !rhs || !x || !sp) return NNK_E_ARG;
  nnk_ctx* ctx = batch->ctx;
  API_TRY
  need_gpu(ctx);
  nnk::BatchMobility& M = *batch->m;
  const size_t n = (size_t)M.size();
  const double* db = stage_in(ctx, batch->io_in, rhs, n, on_device);
  double* dx = stage_out(batch->io_out, x, n, on_device);
  std::vector<nnk_solve_info> inf(M.systems());
  M.solve(db, dx, *sp, inf.data());
  finish_out(ctx, batch->io_out, x, n, on_device);
  batch_errors(M, 1);
  if (info) std::copy(inf.begin(), inf.end(), info);
  for (const auto& i : inf)
    if (i.flag != 0) return fail(ctx, NNK_E_NOCONV, "gmres stopped at maxit above tol for some system");
  API_CATCH(ctx)
}

int nnk_batch_set_refinement(nnk_batch* batch, int32_t fp64, int32_t max_outer, double inner_tol) {
  if (!batch) return NNK_E_ARG;
  nnk_ctx* ctx = batch->ctx;
  API_TRY
  need_gpu(ctx);
  batch->m->set_refinement(fp64 != 0, max_outer, inner_tol);
  API_CATCH(ctx)
}

int nnk_batch_use_graphs(nnk_batch* batch, int32_t enable) {
  if (!batch) return NNK_E_ARG;
  nnk_ctx* ctx = batch->ctx;
  API_TRY
  need_gpu(ctx);
  batch->m->use_graphs(enable != 0);
  API_CATCH(ctx)
}

int nnk_batch_set_deflation(nnk_batch* batch, int32_t enable) {
  if (!batch) return NNK_E_ARG;
  batch->m->set_deflation(enable != 0);
  return NNK_OK;
}

int nnk_batch_matvecs(const nnk_batch* batch, int64_t* count) {
  if (!batch || !count) return NNK_E_ARG;
  *count = batch->m->matvecs();
  return NNK_OK;
}

int nnk_batch_profile(nnk_batch* batch, int32_t enable) {
  if (!batch) return NNK_E_ARG;
  nnk_ctx* ctx = batch->ctx;
  API_TRY
  batch->m->fmm().set_profile(enable != 0);
  if (batch->m->ref64()) batch->m->ref64()->set_profile(enable != 0);
  API_CATCH(ctx)
}

int nnk_batch_profile_read(nnk_batch* batch, int32_t which, double* ms, int64_t* launches) {
  if (!batch || which < 0 || which > 1) return NNK_E_ARG;
  nnk_ctx* ctx = batch->ctx;
  API_TRY
  need_gpu(ctx);
  nnk::Fmm* f = which == 0 ? &batch->m->fmm() : batch->m->ref64();
  if (!f) return fail(ctx, NNK_E_STATE, "no refinement FMM");
  f->read_profile(ms, launches);
  API_CATCH(ctx)
}

int nnk_batch_destroy(nnk_batch* batch) {
  if (!batch) return NNK_OK;
  nnk_ctx* c = batch->ctx;
  if (c->has_gpu) cudaSetDevice(c->device);
  delete batch;
  if (c->has_gpu) cudaGetLastError();
  ctx_release(c);
  return NNK_OK;
}

}  // extern "C"
