/*
 * nnk_mex.c -- MATLAB MEX gateway over the C ABI of libnnkifmm.so
 * (include/nnkifmm.h), for the Stokes-NNKIFMM MATLAB code:
 *
 *   NN   = nnk_mex('nearestMatrix', coarse, fine)           nearestMatrix.m:17-41
 *   T    = nnk_mex('tree', pot, tgt, cap, maxDepth [, fine, NN])  OcTree.m:77-129
 *   info = nnk_mex('treeInfo', T)                           [nodeCount maxLevel ...]
 *   L    = nnk_mex('treeList', T, k)                        tree.interactions{:,k+1}
 *   F    = nnk_mex('fmm', T, eps, mu [, coronaRes, coronaShells, precision])  KIFMM.m:46-61
 *   v    = nnk_mex('computeVel', F, x, format)              KIFMM.m:63-105
 *   v    = nnk_mex('computeVelSparse', F, x, format)        KIFMM.m:107-155
 *   v    = nnk_mex('reducedComputeVel', F, x, format)       KIFMM.m:157-198
 *   v    = nnk_mex('reducedSolve', F, x, format)            KIFMM.m:200-242
 *   [x, flag, relres, iters] = nnk_mex('gmres', F, b, tol, maxit)
 *                                    gmres(@(x) fmm.computeVel(x), b, [], tol, maxit)
 *   M    = nnk_mex('mobility', F, bodyStart, fineStart, relPoints, relFine)
 *   y    = nnk_mex('mobilityMatrixMulti', M, x)             MobilityMatrixMulti.m:17-36
 *   y    = nnk_mex('mobilityPrecon', M, x)                  MobilityPrecon.m:17-40
 *   [x, flag, relres, iters] = nnk_mex('mobilitySolve', M, rhs, tol, maxit, precondition)
 *                                    mobilityProblem.m:48-58
 *   nnk_mex('destroy', H)                                   any handle above
 *
 * Build (where MATLAB is installed; not in this repository's image):
 *   mex -R2018a -I<repo>/include nnk_mex.c -L<lib dir> -lnnkifmm
 *
 * Handles are returned as uint64 scalars holding the library pointer with a
 * kind tag in the low bits (the library's objects are 16-byte aligned); a
 * MATLAB handle class keeps one and calls nnk_mex('destroy', h) from its
 * delete method.  Points are MATLAB (n,3) column-major arrays, transposed here
 * to the library's row-major layout; NN is MATLAB's sparse Q x N matrix
 * (compressed columns), converted here to the library's rows by fine point.
 * Vectors use the KIFMM 'format' option: 1 interleaved [x1 y1 z1 ...]', 2
 * blocked [x1..xN y1..yN z1..zN]'.  Every status other than NNK_OK becomes a
 * MATLAB error with the library's message; NNK_E_MAXDEPTH carries the
 * reference's identifier and text (OcTree.m:168-170).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"
#include "nnkifmm.h"

enum { KIND_TREE = 1, KIND_FMM = 2, KIND_MOB = 3 };

static nnk_ctx* g_ctx = NULL;

static void cleanup(void) {
  if (g_ctx) nnk_ctx_destroy(g_ctx);
  g_ctx = NULL;
}

static void check(int rc, const char* what) {
  if (rc == NNK_OK) return;
  if (rc == NNK_E_MAXDEPTH) mexErrMsgIdAndTxt("OcTree:maxDepth", "Max level reached: Increase Max Depth");
  mexErrMsgIdAndTxt("nnkifmm:error", "%s: %s (status %d)", what, g_ctx ? nnk_last_error(g_ctx) : "", rc);
}

static void need_args(int nrhs, int n, const char* cmd) {
  if (nrhs < n) mexErrMsgIdAndTxt("nnkifmm:args", "%s: expected at least %d arguments", cmd, n - 1);
}

static mxArray* make_handle(void* p, int kind) {
  mxArray* h = mxCreateNumericMatrix(1, 1, mxUINT64_CLASS, mxREAL);
  *(uint64_t*)mxGetData(h) = (uint64_t)(uintptr_t)p | (uint64_t)kind;
  return h;
}

static void* get_handle(const mxArray* a, int kind) {
  if (!mxIsUint64(a) || mxGetNumberOfElements(a) != 1)
    mexErrMsgIdAndTxt("nnkifmm:handle", "expected a uint64 handle");
  const uint64_t v = *(const uint64_t*)mxGetData(a);
  if ((int)(v & 15u) != kind) mexErrMsgIdAndTxt("nnkifmm:handle", "handle of another kind");
  return (void*)(uintptr_t)(v & ~(uint64_t)15u);
}

static double scalar(const mxArray* a) { return mxGetScalar(a); }

/* (n,3) column-major -> row-major copy (mxFree by the caller) */
static double* points_rm(const mxArray* a, int64_t* n) {
  if (!mxIsDouble(a) || mxIsComplex(a) || mxIsSparse(a) || (mxGetN(a) != 3 && mxGetNumberOfElements(a) != 0))
    mexErrMsgIdAndTxt("nnkifmm:points", "points must be a real (n,3) double array");
  const size_t m = mxGetM(a);
  const double* src = mxGetPr(a);
  double* out = (double*)mxMalloc(sizeof(double) * 3 * (m ? m : 1));
  for (size_t i = 0; i < m; ++i)
    for (int d = 0; d < 3; ++d) out[3 * i + d] = src[(size_t)d * m + i];
  *n = (int64_t)m;
  return out;
}

/* sparse Q x N (compressed columns) -> rows by fine point, ascending columns */
static void nn_rows(const mxArray* a, int64_t q, int64_t** rowptr, int32_t** col, double** val) {
  if (!mxIsSparse(a) || mxGetM(a) != (size_t)q) mexErrMsgIdAndTxt("nnkifmm:NN", "NN must be a sparse Q x N matrix");
  const size_t ncols = mxGetN(a);
  const mwIndex* ir = mxGetIr(a);
  const mwIndex* jc = mxGetJc(a);
  const double* pr = mxGetPr(a);
  const size_t nnz = jc[ncols];
  int64_t* rp = (int64_t*)mxCalloc((size_t)q + 1, sizeof(int64_t));
  int32_t* c = (int32_t*)mxMalloc(sizeof(int32_t) * (nnz ? nnz : 1));
  double* v = (double*)mxMalloc(sizeof(double) * (nnz ? nnz : 1));
  for (size_t k = 0; k < nnz; ++k) rp[ir[k] + 1]++;
  for (int64_t r = 0; r < q; ++r) rp[r + 1] += rp[r];
  int64_t* at = (int64_t*)mxMalloc(sizeof(int64_t) * ((size_t)q + 1));
  memcpy(at, rp, sizeof(int64_t) * ((size_t)q + 1));
  for (size_t j = 0; j < ncols; ++j) /* columns in order: rows come out with ascending columns */
    for (mwIndex k = jc[j]; k < jc[j + 1]; ++k) {
      const int64_t p = at[ir[k]]++;
      c[p] = (int32_t)j;
      v[p] = pr[k];
    }
  mxFree(at);
  *rowptr = rp;
  *col = c;
  *val = v;
}

static int layout_of(const mxArray* a) {
  const int f = (int)scalar(a);
  if (f != 1 && f != 2) mexErrMsgIdAndTxt("nnkifmm:format", "format must be 1 or 2");
  return f == 1 ? NNK_LAYOUT_ROWS : NNK_LAYOUT_BLOCKED;
}

static void cmd_nearest(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  need_args(nrhs, 3, "nearestMatrix");
  int64_t n, q, nnz = 0;
  double* c = points_rm(prhs[1], &n);
  double* f = points_rm(prhs[2], &q);
  check(nnk_nearest_matrix(g_ctx, c, n, f, q, &nnz, NULL, NULL, NULL), "nearestMatrix");
  int64_t* rp = (int64_t*)mxMalloc(sizeof(int64_t) * ((size_t)q + 1));
  int32_t* col = (int32_t*)mxMalloc(sizeof(int32_t) * (nnz ? (size_t)nnz : 1));
  double* val = (double*)mxMalloc(sizeof(double) * (nnz ? (size_t)nnz : 1));
  check(nnk_nearest_matrix(g_ctx, c, n, f, q, &nnz, rp, col, val), "nearestMatrix");
  /* rows by fine point -> MATLAB's compressed columns */
  mxArray* S = mxCreateSparse((mwSize)q, (mwSize)n, (mwSize)(nnz ? nnz : 1), mxREAL);
  mwIndex* ir = mxGetIr(S);
  mwIndex* jc = mxGetJc(S);
  double* pr = mxGetPr(S);
  for (int64_t j = 0; j <= n; ++j) jc[j] = 0;
  for (int64_t k = 0; k < nnz; ++k) jc[col[k] + 1]++;
  for (int64_t j = 0; j < n; ++j) jc[j + 1] += jc[j];
  mwIndex* at = (mwIndex*)mxMalloc(sizeof(mwIndex) * ((size_t)n + 1));
  memcpy(at, jc, sizeof(mwIndex) * ((size_t)n + 1));
  for (int64_t r = 0; r < q; ++r) /* rows in order: row indices ascend within each column */
    for (int64_t k = rp[r]; k < rp[r + 1]; ++k) {
      const mwIndex p = at[col[k]]++;
      ir[p] = (mwIndex)r;
      pr[p] = val[k];
    }
  mxFree(at);
  mxFree(rp);
  mxFree(col);
  mxFree(val);
  mxFree(c);
  mxFree(f);
  (void)nlhs;
  plhs[0] = S;
}

static void cmd_tree(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  need_args(nrhs, 5, "tree");
  int64_t np, nt, q = 0;
  double* pot = points_rm(prhs[1], &np);
  double* tgt = points_rm(prhs[2], &nt);
  /* OcTree(points, points, ...): the library recognises the common case of
     potentials == targets (required in NEAREST mode) by one shared buffer */
  if (np == nt && memcmp(pot, tgt, sizeof(double) * 3 * (size_t)np) == 0) {
    mxFree(tgt);
    tgt = pot;
  }
  nnk_tree_params p;
  p.node_capacity = (int32_t)scalar(prhs[3]);
  p.max_depth = (int32_t)scalar(prhs[4]);
  p.nearest = nrhs >= 6 ? 1 : 0;
  p.builder = 0;
  double* fine = NULL;
  int64_t* rp = NULL;
  int32_t* col = NULL;
  double* val = NULL;
  if (p.nearest) {
    fine = points_rm(prhs[5], &q);
    if (nrhs >= 7) nn_rows(prhs[6], q, &rp, &col, &val);
  }
  nnk_tree* t = NULL;
  check(nnk_tree_build(g_ctx, pot, np, tgt, nt, fine, q, rp, col, val, &p, &t), "OcTree");
  if (tgt != pot) mxFree(tgt);
  mxFree(pot);
  if (fine) mxFree(fine);
  if (rp) {
    mxFree(rp);
    mxFree(col);
    mxFree(val);
  }
  (void)nlhs;
  plhs[0] = make_handle(t, KIND_TREE);
}

static void cmd_tree_info(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  need_args(nrhs, 2, "treeInfo");
  nnk_tree_info inf;
  check(nnk_tree_info_get((const nnk_tree*)get_handle(prhs[1], KIND_TREE), &inf), "treeInfo");
  plhs[0] = mxCreateDoubleMatrix(1, 6, mxREAL);
  double* o = mxGetPr(plhs[0]);
  o[0] = inf.node_count;
  o[1] = inf.max_level;
  o[2] = (double)inf.num_points;
  o[3] = (double)inf.num_potentials;
  o[4] = (double)inf.num_targets;
  o[5] = inf.node_capacity;
  (void)nlhs;
}

/* tree.interactions{:,k+1} as a nodeCount x 1 cell of 1-based id rows */
static void cmd_tree_list(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  need_args(nrhs, 3, "treeList");
  const nnk_tree* t = (const nnk_tree*)get_handle(prhs[1], KIND_TREE);
  nnk_tree_info inf;
  check(nnk_tree_info_get(t, &inf), "treeList");
  const int32_t which = (int32_t)scalar(prhs[2]);
  int64_t* off = (int64_t*)mxMalloc(sizeof(int64_t) * ((size_t)inf.node_count + 1));
  check(nnk_tree_export_list(t, which, off, NULL), "treeList");
  const int64_t tot = off[inf.node_count];
  int32_t* ids = (int32_t*)mxMalloc(sizeof(int32_t) * (tot ? (size_t)tot : 1));
  check(nnk_tree_export_list(t, which, off, ids), "treeList");
  mxArray* cell = mxCreateCellMatrix((mwSize)inf.node_count, 1);
  for (int32_t i = 0; i < inf.node_count; ++i) {
    const int64_t a = off[i], b = off[i + 1];
    mxArray* row = mxCreateDoubleMatrix(1, (mwSize)(b - a), mxREAL);
    double* r = mxGetPr(row);
    for (int64_t k = a; k < b; ++k) r[k - a] = ids[k];
    mxSetCell(cell, (mwIndex)i, row);
  }
  mxFree(off);
  mxFree(ids);
  (void)nlhs;
  plhs[0] = cell;
}

static void cmd_fmm(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  need_args(nrhs, 4, "fmm");
  nnk_fmm_params p;
  memset(&p, 0, sizeof p);
  p.eps = scalar(prhs[2]);
  p.mu = scalar(prhs[3]);
  p.corona_res = nrhs >= 5 ? (int32_t)scalar(prhs[4]) : 6;
  p.corona_shells = nrhs >= 6 ? (int32_t)scalar(prhs[5]) : 1;
  p.precision = nrhs >= 7 ? (int32_t)scalar(prhs[6]) : NNK_PREC_FP64;
  nnk_fmm* f = NULL;
  check(nnk_fmm_create(g_ctx, (const nnk_tree*)get_handle(prhs[1], KIND_TREE), &p, &f), "KIFMM");
  (void)nlhs;
  plhs[0] = make_handle(f, KIND_FMM);
}

/* the apply-like FMM calls: which 0 computeVel, 1 computeVelSparse,
   2 reducedComputeVel, 3 reducedSolve */
static void cmd_apply(int which, int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  need_args(nrhs, 4, "computeVel");
  nnk_fmm* f = (nnk_fmm*)get_handle(prhs[1], KIND_FMM);
  const size_t n = mxGetNumberOfElements(prhs[2]);
  if (!mxIsDouble(prhs[2]) || mxIsComplex(prhs[2]) || mxIsSparse(prhs[2]) || n % 3)
    mexErrMsgIdAndTxt("nnkifmm:vector", "x must be a real double vector of 3N values");
  const int layout = layout_of(prhs[3]);
  plhs[0] = mxCreateDoubleMatrix(n, 1, mxREAL);
  const double* x = mxGetPr(prhs[2]);
  double* y = mxGetPr(plhs[0]);
  int rc;
  if (which == 0) rc = nnk_fmm_apply(f, x, y, layout, 1, 0);
  else if (which == 1) rc = nnk_fmm_apply_sparse(f, x, y, layout, 1, 0);
  else if (which == 2) rc = nnk_fmm_reduced_apply(f, x, y, layout, 0);
  else rc = nnk_fmm_reduced_solve(f, x, y, layout, 0);
  check(rc, "computeVel");
  (void)nlhs;
}

static void solve_outputs(int nlhs, mxArray* plhs[], const nnk_solve_info* inf) {
  if (nlhs > 1) plhs[1] = mxCreateDoubleScalar(inf->flag);
  if (nlhs > 2) plhs[2] = mxCreateDoubleScalar(inf->relres);
  if (nlhs > 3) plhs[3] = mxCreateDoubleScalar(inf->iters);
}

static void cmd_gmres(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  need_args(nrhs, 5, "gmres");
  nnk_fmm* f = (nnk_fmm*)get_handle(prhs[1], KIND_FMM);
  const size_t n = mxGetNumberOfElements(prhs[2]);
  nnk_solve_params sp;
  sp.tol = scalar(prhs[3]);
  sp.maxit = (int32_t)scalar(prhs[4]);
  sp.restart = 0;
  nnk_solve_info inf;
  plhs[0] = mxCreateDoubleMatrix(n, 1, mxREAL);
  const int rc = nnk_fmm_solve(f, mxGetPr(prhs[2]), mxGetPr(plhs[0]), NNK_LAYOUT_ROWS, &sp, &inf, 0);
  if (rc != NNK_E_NOCONV) check(rc, "gmres"); /* flag 1 is an output, as in MATLAB */
  solve_outputs(nlhs, plhs, &inf);
}

static void cmd_mobility(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  need_args(nrhs, 6, "mobility");
  nnk_fmm* f = (nnk_fmm*)get_handle(prhs[1], KIND_FMM);
  const size_t nb1 = mxGetNumberOfElements(prhs[2]);
  if (nb1 < 1 || mxGetNumberOfElements(prhs[3]) != nb1)
    mexErrMsgIdAndTxt("nnkifmm:mobility", "bodyStart and fineStart need nbodies + 1 entries");
  int64_t* bs = (int64_t*)mxMalloc(sizeof(int64_t) * nb1);
  int64_t* fs = (int64_t*)mxMalloc(sizeof(int64_t) * nb1);
  const double* b = mxGetPr(prhs[2]);
  const double* c = mxGetPr(prhs[3]);
  for (size_t k = 0; k < nb1; ++k) {
    bs[k] = (int64_t)b[k];
    fs[k] = (int64_t)c[k];
  }
  int64_t nr, nf;
  double* rel = points_rm(prhs[4], &nr);
  double* frel = points_rm(prhs[5], &nf);
  nnk_mob* m = NULL;
  check(nnk_mob_create(f, (int32_t)(nb1 - 1), bs, fs, rel, frel, &m), "mobility");
  mxFree(bs);
  mxFree(fs);
  mxFree(rel);
  mxFree(frel);
  (void)nlhs;
  plhs[0] = make_handle(m, KIND_MOB);
}

static void cmd_mob_apply(int precon, int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  need_args(nrhs, 3, "mobilityMatrixMulti");
  nnk_mob* m = (nnk_mob*)get_handle(prhs[1], KIND_MOB);
  const size_t n = mxGetNumberOfElements(prhs[2]);
  plhs[0] = mxCreateDoubleMatrix(n, 1, mxREAL);
  const int rc = precon ? nnk_mob_precon(m, mxGetPr(prhs[2]), mxGetPr(plhs[0]), 0)
                        : nnk_mob_apply(m, mxGetPr(prhs[2]), mxGetPr(plhs[0]), 0);
  check(rc, precon ? "mobilityPrecon" : "mobilityMatrixMulti");
  (void)nlhs;
}

static void cmd_mob_solve(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  need_args(nrhs, 6, "mobilitySolve");
  nnk_mob* m = (nnk_mob*)get_handle(prhs[1], KIND_MOB);
  const size_t n = mxGetNumberOfElements(prhs[2]);
  nnk_solve_params sp;
  sp.tol = scalar(prhs[3]);
  sp.maxit = (int32_t)scalar(prhs[4]);
  sp.restart = 0;
  nnk_solve_info inf;
  plhs[0] = mxCreateDoubleMatrix(n, 1, mxREAL);
  const int rc = nnk_mob_solve(m, mxGetPr(prhs[2]), mxGetPr(plhs[0]), &sp, scalar(prhs[5]) != 0, &inf, 0);
  if (rc != NNK_E_NOCONV) check(rc, "mobilitySolve");
  solve_outputs(nlhs, plhs, &inf);
}

static void cmd_destroy(int nrhs, const mxArray* prhs[]) {
  need_args(nrhs, 2, "destroy");
  if (!mxIsUint64(prhs[1])) mexErrMsgIdAndTxt("nnkifmm:handle", "expected a uint64 handle");
  const uint64_t v = *(const uint64_t*)mxGetData(prhs[1]);
  void* p = (void*)(uintptr_t)(v & ~(uint64_t)15u);
  switch ((int)(v & 15u)) {
    case KIND_TREE: check(nnk_tree_destroy((nnk_tree*)p), "destroy"); break;
    case KIND_FMM: check(nnk_fmm_destroy((nnk_fmm*)p), "destroy"); break;
    case KIND_MOB: check(nnk_mob_destroy((nnk_mob*)p), "destroy"); break;
    default: mexErrMsgIdAndTxt("nnkifmm:handle", "unknown handle kind");
  }
}

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  char cmd[64];
  if (nrhs < 1 || !mxIsChar(prhs[0]) || mxGetString(prhs[0], cmd, sizeof cmd) != 0)
    mexErrMsgIdAndTxt("nnkifmm:args", "nnk_mex(command, ...)");
  if (!g_ctx) {
    check(nnk_ctx_create(0, &g_ctx), "context");
    mexAtExit(cleanup);
  }
  if (!strcmp(cmd, "nearestMatrix")) cmd_nearest(nlhs, plhs, nrhs, prhs);
  else if (!strcmp(cmd, "tree")) cmd_tree(nlhs, plhs, nrhs, prhs);
  else if (!strcmp(cmd, "treeInfo")) cmd_tree_info(nlhs, plhs, nrhs, prhs);
  else if (!strcmp(cmd, "treeList")) cmd_tree_list(nlhs, plhs, nrhs, prhs);
  else if (!strcmp(cmd, "fmm")) cmd_fmm(nlhs, plhs, nrhs, prhs);
  else if (!strcmp(cmd, "computeVel")) cmd_apply(0, nlhs, plhs, nrhs, prhs);
  else if (!strcmp(cmd, "computeVelSparse")) cmd_apply(1, nlhs, plhs, nrhs, prhs);
  else if (!strcmp(cmd, "reducedComputeVel")) cmd_apply(2, nlhs, plhs, nrhs, prhs);
  else if (!strcmp(cmd, "reducedSolve")) cmd_apply(3, nlhs, plhs, nrhs, prhs);
  else if (!strcmp(cmd, "gmres")) cmd_gmres(nlhs, plhs, nrhs, prhs);
  else if (!strcmp(cmd, "mobility")) cmd_mobility(nlhs, plhs, nrhs, prhs);
  else if (!strcmp(cmd, "mobilityMatrixMulti")) cmd_mob_apply(0, nlhs, plhs, nrhs, prhs);
  else if (!strcmp(cmd, "mobilityPrecon")) cmd_mob_apply(1, nlhs, plhs, nrhs, prhs);
  else if (!strcmp(cmd, "mobilitySolve")) cmd_mob_solve(nlhs, plhs, nrhs, prhs);
  else if (!strcmp(cmd, "destroy")) cmd_destroy(nrhs, prhs);
  else mexErrMsgIdAndTxt("nnkifmm:args", "unknown command '%s'", cmd);
}
