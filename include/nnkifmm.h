/*
 * nnkifmm.h -- C ABI of the B200 KIFMM / mobility library (libnnkifmm.so).
 *
 * Drop-in for the Stokes-NNKIFMM MATLAB path
 *   OcTree(...)                      Classes/OcTree.m:77-129
 *   nearestMatrix(...)               Tools/Nearest/nearestMatrix.m:17-41
 *   KIFMM(tree,[eps mu],...)         Classes/KIFMM.m:46-61
 *   KIFMM.computeVel                 Classes/KIFMM.m:63-105
 *   KIFMM.computeVelSparse           Classes/KIFMM.m:107-155
 *   KIFMM.reducedComputeVel          Classes/KIFMM.m:157-198
 *   KIFMM.reducedSolve               Classes/KIFMM.m:200-242
 *   gmres(@(x) fmm.computeVel(x),..) Data Generation/DirectMethodComparison.m:28
 *   mobilityProblem(...)             Mobility/mobilityProblem.m:1-72
 *
 * Conventions
 *   - Every function returns an int status (NNK_OK = 0).  No C++ exception
 *     crosses the ABI.  nnk_last_error() gives a message for the last failure
 *     on a context.
 *   - Points are row-major (n,3) FP64 arrays [x0 y0 z0 x1 y1 z1 ...].
 *   - Node ids, list entries and pointIndex are exported as the reference's
 *     1-based node ids (DFS block numbering, OcTree.m:174-175).
 *   - Vector layouts (KIFMM.m:83-103): NNK_LAYOUT_ROWS = (N,3) row-major,
 *     which is also the 'GMRES',1,'format',1 interleaved vector;
 *     NNK_LAYOUT_BLOCKED = 'format',2 [x1..xN y1..yN z1..zN].
 *   - Buffers are owned by the caller.  on_device = 0: host pointers;
 *     on_device = 1: device pointers on the context's device.
 *   - A handle is used by one thread at a time.  Work is issued on the
 *     context's CUDA stream (nnk_ctx_set_stream).
 */
#ifndef NNKIFMM_H
#define NNKIFMM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NNK_OK 0
#define NNK_E_ARG 1        /* bad argument or unsupported combination          */
#define NNK_E_MAXDEPTH 2   /* OcTree.m:168-170 'Max level reached'              */
#define NNK_E_NONFINITE 3  /* NaN/Inf in input or result                        */
#define NNK_E_NOCONV 4     /* GMRES stopped at maxit above tol                  */
#define NNK_E_OOM 5        /* device or host allocation failed                  */
#define NNK_E_CUDA 6       /* CUDA runtime error (message in nnk_last_error)    */
#define NNK_E_TIMEOUT 7    /* a bounded device wait gave up                     */
#define NNK_E_STATE 8      /* call out of order / object not ready              */

#define NNK_LAYOUT_ROWS 1
#define NNK_LAYOUT_BLOCKED 2

#define NNK_PREC_FP64 0    /* every FMM step in FP64                            */
#define NNK_PREC_MIXED 1   /* FP32 pair kernels, tensor-core M2L, FP64 C2E ops   */
#define NNK_PREC_NEAR32 2  /* the FP64 operator (exact check-to-equivalent
                              inverses) with the pair sums whose sources are
                              the forces themselves -- U-list P2P and X-list
                              P2L -- in FP32; every sum over equivalent
                              densities stays FP64.  Adjoint and gradients of
                              such an FMM run in FP64.                       */

typedef struct nnk_ctx nnk_ctx;
typedef struct nnk_tree nnk_tree;
typedef struct nnk_fmm nnk_fmm;
typedef struct nnk_mob nnk_mob;
typedef struct nnk_batch nnk_batch;

/* OcTree name-value options (OcTree.m:86-95). */
typedef struct nnk_tree_params {
  int32_t node_capacity; /* 'nodeCapacity' (default 200)                      */
  int32_t max_depth;     /* 'maxDepth' (default 21; at most 23 here)           */
  int32_t nearest;       /* 'nearest' 0/1                                      */
  int32_t builder;       /* where the octree's node structure and the NN
                            matrix are built: 0 auto (the GPU when the
                            context has one), 1 host, 2 GPU.  The results are
                            identical bit for bit; the lists are built on the
                            host from the node arrays either way.          */
} nnk_tree_params;

typedef struct nnk_tree_info {
  int64_t num_points;     /* unique points (OcTree.m:80)                        */
  int64_t num_potentials; /* sum(tree.potentials)                               */
  int64_t num_targets;    /* sum(tree.targets)                                  */
  int64_t num_fine;       /* Q (NEAREST)                                        */
  int64_t nn_nnz;         /* nonzeros of NN (NEAREST)                           */
  int64_t source_entries; /* leaf source entries (fine points per leaf, NEAREST;
                             potential points otherwise)                        */
  int64_t u_total, v_total, w_total, x_total; /* list lengths summed over nodes */
  int32_t node_count;     /* tree.nodeCount                                     */
  int32_t max_level;      /* max(tree.nodeLevel)                                */
  int32_t node_capacity;  /* min(nodeCapacity, numPts-1) (OcTree.m:105)         */
  int32_t nearest;
} nnk_tree_info;

/* KIFMM name-value options (KIFMM.m:50-60) plus the precision mode. */
typedef struct nnk_fmm_params {
  double eps;            /* kernelPar(1)                                       */
  double mu;             /* kernelPar(2)                                       */
  int32_t corona_res;    /* 'coronaRes' (default 6)                            */
  int32_t corona_shells; /* 'coronaShells' (default 1)                         */
  int32_t precision;     /* NNK_PREC_FP64, NNK_PREC_MIXED or NNK_PREC_NEAR32   */
  int32_t m2l_mode;      /* mixed mode M2L: 0 auto (tensor cores on rank-256
                            compressed operators B C_o B^T when 3P > 256, else
                            images when they fit 8 GiB), 1 tensor cores +
                            streamed full images,
                            2 tensor cores + in-kernel operators, 3 FP32 pair
                            kernel (no tensor cores; FP32-rounding accuracy),
                            4 FP32 Fourier-space product (FFT of the surface
                            lattice; FP32-rounding accuracy).
                            FP64 and NEAR32 modes: 3 the FP64 pair kernel, any
                            other value the FP64 Fourier-space product (at
                            most 6 right-hand sides per pass)                 */
  double reg;            /* relative Tikhonov weight of the check-to-equivalent
                            pseudo-inverse: NNK_PREC_MIXED 0 = default 1e-5;
                            NNK_PREC_FP64 0 = exact LU inverse (reference)   */
} nnk_fmm_params;

/* Algorithmic work of one matvec, from the tree statistics (for rooflines). */
typedef struct nnk_fmm_stats {
  int64_t pairs_leaf;   /* U-list P2P + W-list M2T + L2T target-source pairs   */
  int64_t pairs_p2p;    /* U-list P2P pairs only                               */
  int64_t pairs_up;     /* S2M + M2M pairs                                     */
  int64_t pairs_down;   /* M2L + P2L + L2L pairs (pair-kernel form)            */
  int64_t m2l_pairs;    /* V-list (target node, source node) pairs             */
  int64_t c2e_columns;  /* check-to-equivalent applications (up + down)        */
  int64_t m2l_tile_rows; /* tensor-core M2L rows processed, padding included     */
  int32_t surface_points;
  int32_t levels;
  int32_t m2l_rank;     /* compressed tensor-core M2L: rank of the per-level
                           bases (its GEMMs are m2l_rank square); 0 otherwise */
  int32_t folded;       /* 1: the matvec runs M2M and L2L folded into the
                           check-to-equivalent products (nnk_fmm_set_fold)  */
  int32_t m2l_frequencies; /* Fourier-space M2L: frequencies of the half
                              spectrum (0 without it)                       */
  int32_t m2l_family;   /* 1: its parent-grouped accumulation is used         */
  int64_t m2l_records;  /* parent-grouped: (parent, colleague) records; each
                           reads its colleague's 8 children's source spectra
                           (3 complex values a frequency each)              */
  int64_t m2l_groups;   /* parent-grouped: (record, child difference) groups;
                           each reads one kernel spectrum (6 complex values a
                           frequency) for all its V pairs                   */
  int64_t m2m_product_pairs; /* M2M as products with its kernel matrices
                           (nnk_fmm_set_m2m_form): the target-source pairs
                           that pairs_up counts but the pair kernels no
                           longer evaluate (0 with the pair form)           */
  int64_t l2l_product_pairs; /* the same for L2L and pairs_down (form 2)    */
} nnk_fmm_stats;

/* GMRES options/result (MATLAB gmres(A,b,restart,tol,maxit), x0 = 0). */
typedef struct nnk_solve_params {
  double tol;       /* relative residual ||b-Ax||/||b|| (default 1e-6)        */
  int32_t maxit;    /* total inner iterations                                 */
  int32_t restart;  /* 0 = unrestarted (restart = [])                         */
} nnk_solve_params;

typedef struct nnk_solve_info {
  int32_t flag;     /* 0 converged, 1 maxit reached                           */
  int32_t iters;    /* inner iterations used                                  */
  double relres;    /* true relative residual at exit                         */
} nnk_solve_info;

/* ------------------------------------------------------------ context -- */
int nnk_ctx_create(int32_t device, nnk_ctx** out);
/* Releases the caller's handle.  Trees, FMMs and batches made from the
 * context hold it too, so handles may be destroyed in any order: the context
 * and its stream go with the last of them. */
int nnk_ctx_destroy(nnk_ctx* ctx);
/* Use this stream (a cudaStream_t) for all later work on the context. */
int nnk_ctx_set_stream(nnk_ctx* ctx, void* stream);
int nnk_ctx_synchronize(nnk_ctx* ctx);
const char* nnk_last_error(const nnk_ctx* ctx);
/* Library version string, e.g. "nnkifmm 0.1 sm_100a". */
const char* nnk_version(void);

/* ------------------------------------------------- nearest neighbours -- */
/* nearestMatrix(coarse,fine) (nearestMatrix.m:17-41): FP64 d2 = (dx^2+dy^2)+dz^2,
 * ties share 1/k.  Returns CSR by fine point: *nnz is set; if rowptr is NULL
 * only the count is returned, else rowptr (q+1), col (0-based coarse index)
 * and val (weights) are filled. */
/* nearestMatrix on the context's GPU when it has one (same result as the
 * host search, bit for bit); nnk_nearest_matrix_host forces the host. */
int nnk_nearest_matrix_host(nnk_ctx* ctx, const double* coarse, int64_t n, const double* fine, int64_t q,
                            int64_t* nnz, int64_t* rowptr, int32_t* col, double* val);
int nnk_nearest_matrix(nnk_ctx* ctx, const double* coarse, int64_t n,
                       const double* fine, int64_t q, int64_t* nnz,
                       int64_t* rowptr, int32_t* col, double* val);
/* The tie weights of nearestMatrix.m as written (nearestMatrix.m:23-39), for
 * callers that need the reference's matrix entry for entry.  The reference
 * cuts the fine points into blocks of floor(blockSize 2^27 / (9 q)) and, per
 * block, pairs the tied (fine, coarse) entries taken in column-major order
 * (find) with the weights 1/k taken in row-major order (logical indexing of
 * the transpose): where rows with different tie counts share a block,
 * weights move to other rows and rows stop summing to one.  Rewrites val of
 * a matrix from nnk_nearest_matrix (rowptr q+1, ascending col per row) in
 * place into that pairing; tie-free rows keep weight 1.  NNK_E_ARG when the
 * block is empty (the reference builds no matrix then).  Host only. */
int nnk_nearest_reference_weights(nnk_ctx* ctx, int64_t q, const int64_t* rowptr,
                                  const int32_t* col, double* val,
                                  double block_size);

/* --------------------------------------------------------------- tree -- */
/* OcTree(potPoints, targetPoints, ...) (OcTree.m:77-129).
 * NEAREST: fine (q,3) and the NN CSR (rowptr q+1, 0-based col into potPoints,
 * val).  If nn_rowptr is NULL and params->nearest, NN is built as
 * nnk_nearest_matrix(potPoints, fine).  NEAREST requires targetPoints ==
 * potPoints (the reference gathers NEAREST sources by pointIndex over all
 * points, downwardPass.m:92,221).  Returns NNK_E_MAXDEPTH with the
 * reference message when any node reaches level maxDepth-1. */
int nnk_tree_build(nnk_ctx* ctx, const double* pot, int64_t n_pot,
                   const double* tgt, int64_t n_tgt, const double* fine,
                   int64_t q, const int64_t* nn_rowptr, const int32_t* nn_col,
                   const double* nn_val, const nnk_tree_params* params,
                   nnk_tree** out);
int nnk_tree_info_get(const nnk_tree* tree, nnk_tree_info* info);
/* nodeLevel, nodeParents (0 for the root), nodeChildren (8 per node, 0 for
 * leaves), nodeCorners (6 per node) and pointIndex (per unique point).
 * Any pointer may be NULL. */
int nnk_tree_export_nodes(const nnk_tree* tree, int32_t* level,
                          int32_t* parent, int32_t* children, double* corners,
                          int32_t* point_index);
/* potentials / targets masks (OcTree.m:81-82) and the unique points (n,3). */
int nnk_tree_export_points(const nnk_tree* tree, double* points,
                           uint8_t* potentials, uint8_t* targets);
/* tree.interactions{:,k}, k = 0 U, 1 V, 2 W, 3 X: offsets (nodeCount+1, by
 * reference node id - 1) and 1-based ids in the reference's order. */
int nnk_tree_export_list(const nnk_tree* tree, int32_t which, int64_t* offsets,
                         int32_t* ids);
int nnk_tree_destroy(nnk_tree* tree);

/* ---------------------------------------------------------------- FMM -- */
/* KIFMM(tree,[eps mu],...).  The tree must outlive the FMM. */
int nnk_fmm_create(nnk_ctx* ctx, const nnk_tree* tree,
                   const nnk_fmm_params* params, nnk_fmm** out);
/* computeVel: in = potentials (num_potentials x 3), out = velocities
 * (num_targets x 3), in the given layout, nrhs right-hand sides stored one
 * after another. */
int nnk_fmm_apply(nnk_fmm* fmm, const double* in, double* out, int32_t layout,
                  int32_t nrhs, int32_t on_device);
/* computeVelSparse: the same with coronaRes 4 (KIFMM.m:136-145). */
int nnk_fmm_apply_sparse(nnk_fmm* fmm, const double* in, double* out,
                         int32_t layout, int32_t nrhs, int32_t on_device);
/* reducedComputeVel (reducedPass.m) and reducedSolve (ReducedSolve.m). */
int nnk_fmm_reduced_apply(nnk_fmm* fmm, const double* in, double* out,
                          int32_t layout, int32_t on_device);
int nnk_fmm_reduced_solve(nnk_fmm* fmm, const double* in, double* out,
                          int32_t layout, int32_t on_device);
int nnk_fmm_stats_get(const nnk_fmm* fmm, nnk_fmm_stats* stats);

/* Per-phase device timing of later applies (no counterpart in the reference;
 * it replaces the tic/toc around whole solves, DirectMethodComparison.m:25-29).
 * enable != 0 records CUDA events around every kernel phase on the context
 * stream; nnk_fmm_profile_read returns accumulated milliseconds and launch
 * counts per phase (NNK_PHASE_*) since the last reset, then resets. */
#define NNK_PHASE_GATHER 0
#define NNK_PHASE_UP_PAIRS 1
#define NNK_PHASE_UP_C2E 2
#define NNK_PHASE_DOWN_PAIRS 3
#define NNK_PHASE_DOWN_C2E 4
#define NNK_PHASE_LEAF_PAIRS 5
#define NNK_PHASE_SCATTER 6
#define NNK_PHASE_M2L 7
#define NNK_NUM_PHASES 8
/* ------------------------------------------------------------- adjoint -- */
/* No counterpart in the reference (gradients are new here).  The exact
 * transpose of nnk_fmm_apply: in (targets, n_tgt x 3 per right-hand side),
 * out (potentials, n_pot x 3); <y, apply(x)> = <apply_adjoint(y), x>.  The
 * same passes run on the same tree with the point sets' roles exchanged and
 * the interaction lists inverted. */
int nnk_fmm_apply_adjoint(nnk_fmm* fmm, const double* in, double* out, int32_t layout,
                          int32_t nrhs, int32_t on_device);
/* Autotuner: times every launch group of the pair kernel (upward and
 * downward levels, leaf stage) with source tiles of 64, 128 and 256 points
 * for passes of nrhs right-hand sides and keeps the fastest per group.
 * ms_before / ms_after (may be NULL): summed pair-kernel time with the
 * default tiles and with the picked ones. */
int nnk_fmm_autotune(nnk_fmm* fmm, int32_t nrhs, double* ms_before, double* ms_after);
/* Rebuild the eps-dependent parts of the FMM (operators, M2L images or
 * spectra) for kernelPar(1) = eps, keeping the tree-dependent task lists:
 * the cheap way to evaluate the operator at eps +- d for its eps-derivative. */
int nnk_fmm_set_eps(nnk_fmm* fmm, double eps);
/* Check-to-equivalent products (the batched form of the LU solves of
 * Up.m:31-33 and DownNonleaf.m:42-46).  Mode 2, the default: per run of
 * nodes of one level sharing an operator, their check vectors gathered into
 * one matrix, one cuBLAS DGEMM with the FP64 operator, the products
 * scattered back (single-tree FMMs; forests, and a matvec being captured
 * into a CUDA graph, use mode 0).  Mode 0: our FP64 SIMT product kernel.
 * Mode 1: on the tensor cores as int8 digit products with exact int32 sums
 * combined in FP64 -- 9 x 9 digits for FP64 check vectors, 5 x 4 for the
 * mixed mode's FP32 ones, the FP64 product's accuracy either way (needs 3P
 * <= 512).  Mode -1 keeps whichever nnk_fmm_autotune times fastest on one
 * matvec (SIMT until it runs).  Measured on the 250k matvec (C2E time per
 * matvec): FP64 check vectors 0.78 ms (mode 2), 1.12 (0), 1.97 (1); the
 * mixed mode's FP32 ones 0.78, 1.32, 0.91; the modes agree to 1.4e-8 (FP64)
 * and 3e-7 / 4e-6 (mixed, modes 2 / 1 against 0).  nnk_fmm_c2e_mode
 * reports the form in use (0, 1 or 2). */
int nnk_fmm_set_c2e(nnk_fmm* fmm, int32_t mode);
int nnk_fmm_c2e_mode(const nnk_fmm* fmm, int32_t* mode);
/* M2M and L2L in the matvec (the parent sums of upwardPass.m:81-93 and the
 * parentsurf term of DownNonleaf.m:42-46) as products with their kernel
 * matrices -- per box width [M2M_0 .. M2M_7] from a parent's 8 children and
 * [L2L_0; ..; L2L_7] from a parent to its 8 children, one cuBLAS DGEMM per
 * level on gathered densities, into the check potentials, before the
 * check-to-equivalent step -- or as pair sums: form 2, the default where
 * the tree allows it (one tree; the Fourier-space or tensor-core M2L), both
 * as products; form 1 M2M as products and L2L as pair sums; form 0 both as
 * pair sums.  Measured on the 250k FP64 matvec: 13.47 ms (form 2), 13.80
 * (1), 14.20 (0), 1.9e-8 apart.  Both give the reference's check potentials to FP64 rounding
 * (unlike folding, which pre-multiplies by the inverse), so the exact
 * inverses allow it.  The per-phase profile counts the products with the
 * check-to-equivalent phases. */
int nnk_fmm_set_m2m_form(nnk_fmm* fmm, int32_t form);
/* Folded M2M / L2L in the matvec: mode 0 off (the default), 1 where it
 * pays (at least 64 non-leaf nodes per box width), 2 wherever available.  A
 * parent's up-equivalent density becomes one FP64 product
 * A(w) [M2M_0 .. M2M_7] with its 8 children's (Up.m:31-33 applied to the
 * M2M sums of upwardPass.m:81-93), and the L2L part of a child's
 * down-equivalent density the product A(w)^T L2L_k with its parent's
 * (the parentsurf term of DownNonleaf.m:42-46), in place of the pair sums
 * followed by the check-to-equivalent step.  Only for regularized
 * operators (NNK_PREC_MIXED, or reg > 0), where it is the same operator to
 * ~3e-7; with the exact inverses the folded products lift FP64 rounding by
 * the surface matrices' condition number (4e-5 on a NEAREST cloud), so
 * there the call leaves the pair sums in place.  Needs the Fourier-space or
 * tensor-core M2L and at most 1 GiB of folded operators; the transpose, the
 * gradients and the eps-derivative always run unfolded. */
int nnk_fmm_set_fold(nnk_fmm* fmm, int32_t mode);
/* No counterpart in the reference: the device's L2 read bandwidth in GB/s,
 * measured on the context's stream with a streaming read of an L2-resident
 * buffer (16-byte loads from 8 and 16 blocks of 256 threads per SM over 24
 * and 48 MiB; the best of the four), the denominator of the L2 roofline of
 * the Fourier-space M2L accumulation.  Allocates and frees 48 MiB. */
int nnk_measure_l2_read(nnk_ctx* ctx, double* gbs);
/* Host wall time (milliseconds) of the set-up steps of nnk_fmm_create, in
 * the order of the NNK_SETUP_* indices: the unified point array and its
 * surfaces, the pair task lists, the M2L plan (Fourier-space spectra and
 * families, or the tensor-core plan), the check-to-equivalent operators
 * (kernel matrices and their LU or Tikhonov solves), the folded operators,
 * and the whole of it.  Writes min(n, NNK_SETUP_COUNT) values; the last
 * nnk_fmm_set_eps updates the M2L, operator and fold entries. */
enum {
  NNK_SETUP_POINTS = 0,
  NNK_SETUP_TASKS = 1,
  NNK_SETUP_M2L = 2,
  NNK_SETUP_OPERATORS = 3,
  NNK_SETUP_FOLD = 4,
  NNK_SETUP_TOTAL = 5,
  NNK_SETUP_COUNT = 6
};
int nnk_fmm_setup_times(const nnk_fmm* fmm, double* ms, int32_t n);
/* Number of source origins: fine points (NEAREST) or potential rows. */
int nnk_fmm_source_count(const nnk_fmm* fmm, int64_t* count);
/* Gradient of <weights, apply(forces)> with respect to the positions, with
 * the kernel's derivative (Tools/kernel.m:23-47 differentiated):
 * grad_targets (n_tgt x 3, row-major) at the targets, grad_sources
 * (nnk_fmm_source_count x 3) at the fine points (NEAREST) or potentials.
 * forces and weights in `layout`; either output may be NULL. */
int nnk_fmm_grad_positions(nnk_fmm* fmm, const double* forces, const double* weights, int32_t layout,
                           double* grad_targets, double* grad_sources, int32_t on_device);
/* *out = weights^T (dF/deps) forces for the FMM operator F (FP64 with the
 * exact check-to-equivalent inverses, reg = 0; NNK_E_STATE otherwise): every
 * stage differentiated -- the kernel's eps-derivative (Tools/kernel.m:29-47
 * differentiated) in every pair sum and in the M2L, and
 * d(K^-1)/deps = -K^-1 (dK/deps) K^-1 in the check-to-equivalent solves --
 * and contracted with the matvec's inputs to the stage and the transpose
 * pass's sensitivities of its output.  Costs one matvec, one transpose and
 * one derivative pass.  forces and weights in `layout`. */
int nnk_fmm_grad_eps(nnk_fmm* fmm, const double* forces, const double* weights, int32_t layout, double* out,
                     int32_t on_device);

int nnk_fmm_profile(nnk_fmm* fmm, int32_t enable);
int nnk_fmm_profile_read(nnk_fmm* fmm, double* ms, int64_t* launches);
/* No counterpart in the reference (its waits are MATLAB's): failure-path test
 * of the bounded device waits.  Every wait of the tensor-core M2L kernel on an
 * mbarrier gives up after a limit, sets the FMM's error flag and lets the
 * kernel drain and return; the call that launched it (or, with on_device = 1,
 * a later call on the same FMM) returns NNK_E_TIMEOUT and the flag is cleared.
 * This runs that kernel of a mixed FMM once with every thread first waiting,
 * at most `polls` polls, on a barrier that nothing completes: the wait gives
 * up before any copy or MMA is issued, the kernel frees its tensor memory and
 * returns, and the call returns NNK_E_TIMEOUT.  Later applies run normally.
 * NNK_E_STATE for an FMM without the tensor-core M2L. */
int nnk_fmm_test_wait_timeout(nnk_fmm* fmm, uint32_t polls);
int nnk_fmm_destroy(nnk_fmm* fmm);

/* Device GMRES on the FMM operator: solves computeVel(x) = b, the resistance
 * solve of DirectMethodComparison.m:28 / Rigid_Resistance.m:23. */
int nnk_fmm_solve(nnk_fmm* fmm, const double* b, double* x, int32_t layout,
                  const nnk_solve_params* sp, nnk_solve_info* info,
                  int32_t on_device);

/* ----------------------------------------------------------- mobility -- */
/* Rigid bodies (Swimmers.m) on one NEAREST tree: body b owns force points
 * [body_start[b], body_start[b+1]) of the tree's points and fine points
 * [fine_start[b], fine_start[b+1]); points after body_start[nb] are boundary
 * points (no rigid unknowns).  rel_points / rel_fine are the rotated,
 * untranslated positions (Swimmers.m:177-189) used for torques. */
int nnk_mob_create(nnk_fmm* fmm, int32_t nbodies, const int64_t* body_start,
                   const int64_t* fine_start, const double* rel_points,
                   const double* rel_fine, nnk_mob** out);
/* Mobility matvec (mobilityMatrixMulti.m:17-36) on [f (3N blocked); U; Omega]. */
int nnk_mob_apply(nnk_mob* mob, const double* x, double* y, int32_t on_device);
/* Block preconditioner (MobilityPrecon.m:17-40). */
int nnk_mob_precon(nnk_mob* mob, const double* x, double* y, int32_t on_device);
/* No counterpart in the reference: replay the matvec (per FMM it runs on)
 * from a CUDA graph captured on first use, and again after nnk_fmm_set_eps
 * or nnk_fmm_autotune (default on; the result is bitwise that of the
 * launches).  enable = 0 launches kernel by kernel. */
int nnk_mob_use_graphs(nnk_mob* mob, int32_t enable);
/* gmres(afunc, rhs, [], tol, maxit) with optional right preconditioning
 * (mobilityProblem.m:48-58); x receives the (preconditioned-back) solution. */
int nnk_mob_solve(nnk_mob* mob, const double* rhs, double* x,
                  const nnk_solve_params* sp, int32_t precondition,
                  nnk_solve_info* info, int32_t on_device);
/* Mixed-precision iterative refinement for nnk_mob_solve (no counterpart in
 * the reference, which solves in FP64 only): when `fp64` is an FP64 FMM on
 * the same tree as the mobility object's (mixed) FMM, each solve repeats
 * "GMRES on the mixed operator for r, x += d, r = b - A_fp64 x" until the
 * FP64 residual meets tol (at most max_outer times; inner tolerance at least
 * inner_tol).  fp64 = NULL switches refinement off. */
int nnk_mob_set_refinement(nnk_mob* mob, nnk_fmm* fp64, int32_t max_outer, double inner_tol);
/* Adjoint of the mobility matvec, A^T = [F^T B^T; BT^T 0] (F = the FMM block). */
int nnk_mob_apply_adjoint(nnk_mob* mob, const double* x, double* y, int32_t on_device);
/* The mobility matvec with another FMM on the same tree (e.g. at eps +- d
 * for the eps-derivative of the operator). */
int nnk_mob_apply_fmm(nnk_mob* mob, nnk_fmm* fmm, const double* x, double* y, int32_t on_device);
/* gmres on A^T (refined like nnk_mob_solve when refinement is set). */
int nnk_mob_solve_adjoint(nnk_mob* mob, const double* rhs, double* x, const nnk_solve_params* sp,
                          nnk_solve_info* info, int32_t on_device);
/* -lam^T (dA/dpositions) z for z = A^-1 b and lam = A^-T dL/dz: the
 * position gradient of a loss L(z) (b independent of positions, as for
 * forces, torques and a zero slip): grad_points (N x 3, force points,
 * row-major) and grad_fine (Q x 3, fine points, NEAREST; may be NULL).
 * NN is held fixed (it is piecewise constant in the positions). */
int nnk_mob_grad_positions(nnk_mob* mob, const double* z, const double* lam, double* grad_points,
                           double* grad_fine, int32_t on_device);
/* *out = -lam^T (dA/deps) z, the eps part of a loss gradient (only the FMM
 * block of the mobility matrix depends on eps), through nnk_fmm_grad_eps of
 * `fp64` -- an exact FP64 FMM on the mobility object's tree -- or of the
 * mobility object's own FMM when fp64 is NULL. */
int nnk_mob_grad_eps(nnk_mob* mob, nnk_fmm* fp64, const double* z, const double* lam, double* out,
                     int32_t on_device);
int nnk_mob_destroy(nnk_mob* mob);

/* ---------------------------------------------------- batched mobility -- */
/* No counterpart in the reference, which solves one swimmer system and one
 * right-hand side per gmres call (mobilityProblem.m:53): nbodies independent
 * free bodies, each with nrhs right-hand sides (e.g. the 6 rigid modes of
 * Gen_Resistance.m), solved together.  Body b is trees[b] (potentials ==
 * targets = its force points; NEAREST trees carry their NN matrix) with
 * rel_points[b] (N_b x 3) and, for NEAREST, rel_fine[b] (Q_b x 3), the
 * rotated, untranslated positions of Swimmers.m:177-189.  The trees may be
 * destroyed after the call.  One FMM pass evaluates all bodies and all their
 * right-hand sides.  The batch vector is the concatenation of the systems
 * s = b * nrhs + r, each [f_x(1..N_b) f_y f_z | U (3) | Omega (3)]
 * (mobilityProblem.m:45-46); system s starts at offsets[s].
 * params->precision MIXED evaluates pairs (M2L included) in FP32. */
int nnk_batch_create(nnk_ctx* ctx, int32_t nbodies, nnk_tree* const* trees,
                     const double* const* rel_points, const double* const* rel_fine,
                     const nnk_fmm_params* params, int32_t nrhs, nnk_batch** out);
/* Length of the batch vector and, if offsets != NULL, the nbodies*nrhs + 1
 * system offsets. */
int nnk_batch_layout(const nnk_batch* batch, int64_t* length, int64_t* offsets);
/* Every system's mobility matvec (mobilityMatrixMulti.m:17-36). */
int nnk_batch_apply(nnk_batch* batch, const double* x, double* y, int32_t on_device);
/* Unpreconditioned gmres per system (own Krylov space and stopping test,
 * MATLAB semantics as nnk_mob_solve), all systems advancing together;
 * info receives one record per system (may be NULL).  Returns NNK_E_NOCONV
 * if any system stopped above tol.  Like the single-FMM calls, a batch apply
 * or solve returns NNK_E_TIMEOUT when a bounded device wait of one of its
 * FMMs (the forest's, or the FP64 refinement FMM's) gave up (an apply with
 * on_device = 1 reads the flags whose copies have completed; a later call
 * reports the rest). */
int nnk_batch_solve(nnk_batch* batch, const double* rhs, double* x,
                    const nnk_solve_params* sp, nnk_solve_info* info, int32_t on_device);
/* Mixed-precision iterative refinement for a MIXED batch: fp64 != 0 builds an
 * FP64 FMM on the same bodies (same Tikhonov weight) for the outer residuals
 * of nnk_batch_solve, as nnk_mob_set_refinement does. */
int nnk_batch_set_refinement(nnk_batch* batch, int32_t fp64, int32_t max_outer, double inner_tol);
/* Replay each matvec from a CUDA graph captured on first use (default on;
 * off while profiling).  enable = 0 launches the kernels one by one. */
int nnk_batch_use_graphs(nnk_batch* batch, int32_t enable);
/* Deflation by body (default on): once every right-hand side of a body has
 * converged, its tree drops out of the forest FMM for the rest of the solve
 * (its kernels return at once), so a batch costs the sum of its bodies'
 * iterations rather than the slowest body's count times the batch.  The
 * solution is bitwise the same either way; enable = 0 evaluates every tree
 * in every matvec. */
int nnk_batch_set_deflation(nnk_batch* batch, int32_t enable);
/* Total FMM matvecs issued so far (inner and outer). */
int nnk_batch_matvecs(const nnk_batch* batch, int64_t* count);
/* Per-phase CUDA-event timing of the batch's FMM passes, as
 * nnk_fmm_profile / nnk_fmm_profile_read (NNK_PHASE_* order); which = 0
 * reads the batch's own FMM, 1 the FP64 refinement FMM. */
int nnk_batch_profile(nnk_batch* batch, int32_t enable);
int nnk_batch_profile_read(nnk_batch* batch, int32_t which, double* ms, int64_t* launches);
int nnk_batch_destroy(nnk_batch* batch);

/* ------------------------------------------------- allocation-free call -- */
/* No counterpart in the reference: an extra entry point for callers that
 * cannot allocate device memory when they call -- a MEX gateway whose device
 * memory belongs to MATLAB's own pool, or a loop that fixed its memory budget
 * up front and must not pay cudaMalloc/cudaFree (which can synchronize the
 * device) per step.  It evaluates the NEAREST velocity by direct summation,
 * vel(t) = S(fine -> t) * kron(NN,I3) * forces, the dense product of
 * nearestBlockComputation.m, with every input and output a device pointer
 * supplied by the caller (forces n x 3, NN CSR by fine point with 0-based
 * columns into forces, fine q x 3, targets m x 3, vel m x 3, row-major FP64),
 * issued on `stream` (which must belong to `device`; NULL is the legacy
 * default stream).  Its one scratch buffer, the fine-point forces, is a static
 * device array of NNK_NOALLOC_MAX_FINE rows that every GPU loading the library
 * holds until exit; larger q is rejected with NNK_E_ARG.  The first call on a
 * device looks up that array's address and should come before any stream
 * capture.  Calls share the array: calls that overlap on the GPU race.  A
 * column index outside [0, n) is not read: the velocities it reaches come out
 * NaN.  A CUDA error already pending on the calling thread is returned as
 * NNK_E_CUDA without launching and left in place.  Returns without
 * synchronizing. */
#define NNK_NOALLOC_MAX_FINE 262144
int nnk_direct_nearest_noalloc(int32_t device, void* stream, const double* forces,
                               int64_t n, const int64_t* nn_rowptr,
                               const int32_t* nn_col, const double* nn_val,
                               const double* fine, int64_t q,
                               const double* targets, int64_t m, double eps,
                               double mu, double* vel);

#ifdef __cplusplus
}
#endif

#endif /* NNKIFMM_H */
