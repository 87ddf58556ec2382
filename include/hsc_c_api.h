/*
 * hsc_c_api.h -- C ABI of the B200 HSC linear solver.
 *
 * One call solves one Newton-step linear system
 *
 *     [ A   E ] [dq]   [bq]      A: affine bodies (12 dof each)
 *     [ E^T D ] [dx] = [bx]      D: FEM Tet4 nodes (3 dof each)
 *
 * by heterogeneous subspace correction: full-pivot ACA of the coupling
 * E ~ U V^T, an approximate ABD inverse P, Schur-complement PCG on
 * S = D - V (U^T P U) V^T with a Neumann-series preconditioner, then
 * back-substitution dq = P (bq - U V^T dx) and a full-system residual check.
 *
 * It replaces the libuipc linear-system plugin body of the reference
 * (reproduction/hsc_backend/linear_hsc.cu):
 *   class LinearHSC : IterativeSolver  (linear_hsc.cu:153-437)
 *     do_build(BuildInfo&)             (linear_hsc.cu:172-193)  -> hsc_create / hsc_options
 *     do_solve(SolvingInfo&)           (linear_hsc.cu:344-436)  -> hsc_solve
 *   IterativeSolver::spmv(x, y)        (iterative_solver.h:28-32) -> hsc_spmv
 * The inputs are the ones SolvingInfo exposes (global_linear_system.h:347-365):
 * x() a device FP64 vector (written), b() a device FP64 vector (read) and
 * A() a device CBCOOMatrixView<double,3>.
 *
 * All pointers named d_* are device pointers.  No function throws; every
 * function returns an HSC_* status.  A context serves one host thread.
 */
#ifndef HSC_C_API_H
#define HSC_C_API_H

#include <stdint.h>

#if defined(__GNUC__)
#define HSC_EXPORT __attribute__((visibility("default")))
#else
#define HSC_EXPORT
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define HSC_API_VERSION 1

/* status codes (linear_hsc.cu raises UIPC_ASSERT / runtime_error for these) */
#define HSC_OK 0
#define HSC_ERR_INVALID 1     /* bad arguments or input layout (linear_hsc.cu:199-200) */
#define HSC_ERR_NONSPD 2      /* FEM 3x3 diagonal det<=0 (:208), ABD block not SPD (:269) */
#define HSC_ERR_BREAKDOWN 3   /* PCG pSp<=0 or rz<=0 or non-finite (:370-371) */
#define HSC_ERR_NOCONV 4      /* PCG hit max_iter above tol (:394) */
#define HSC_ERR_NONDESCENT 5  /* b^T x <= 0 (:400-402) */
#define HSC_ERR_RESIDUAL 6    /* full residual above full_residual_limit (:433-435) */
#define HSC_ERR_CUDA 7        /* CUDA runtime error (hsc::check, :34-37) */
#define HSC_ERR_TIMEOUT 8     /* a bounded device-side wait gave up */
#define HSC_ERR_ALLOC 9       /* device allocation failed */
#define HSC_ERR_NOTREADY 10   /* query before any solve */

/* arithmetic of the Schur PCG bulk (SpMV, Neumann terms, low-rank apply) */
#define HSC_FP64 0            /* everything FP64 (the reference form) */
#define HSC_FP32 1            /* FP32 bulk values and search vectors; FP64 x, r, coupled-node blocks, low-rank
                                  term and residual replacement */
#define HSC_BF16 2            /* FP32 operator, BF16 preconditioner planes, FP32 accumulation, FP64 replacement */

/* approximate ABD inverse P (linear_hsc.cu:263-297, core.py:148-150) */
#define HSC_ABD_NEUMANN 0     /* fixed-order block-Jacobi Neumann */
#define HSC_ABD_ADAPTIVE 1    /* Neumann extended by doubling until |I-AP|_F/sqrt(qm) <= tol */
#define HSC_ABD_EXACT 2       /* dense FP64 Cholesky inverse */

/* FEM preconditioner polynomial z = sum_k w_k (I - w Dd^-1 D)^k w Dd^-1 r */
#define HSC_PRECOND_NEUMANN 0 /* w_k = 1, k < neumann_order (linear_hsc.cu:330-343) */
#define HSC_PRECOND_POLY 1    /* caller-supplied w_k on the same D-basis terms */
/* Schur basis: z = sum_k w_k (I - w Dd^-1 S)^k w Dd^-1 r, S = D - V C V^T.  For an eigenvalue mu of
   w Dd^-1 S the preconditioned operator has the eigenvalue mu * sum_k w_k (1 - mu)^k, so the weights
   shape the spectrum of the operator PCG actually iterates on.  No reference counterpart. */
#define HSC_PRECOND_SCHUR_POLY 2 /* caller-supplied w_k (poly_degree of them) */
#define HSC_PRECOND_LEARNED 3    /* 8 weights per system from the context's learned model
                                    (hsc_set_learned_model), computed on the device from the
                                    system's features; falls back to plain Neumann on a stall */
/* Block-local Woodbury preconditioner (no reference counterpart): z = L r + Y K Y^T r with
   L = sum_k w_k (I - w Dd^-1 D_loc)^k w Dd^-1, D_loc the blocks of D whose two nodes lie in the same
   part (one part per PCG CTA, from the analysis' renumbering), Y = L V and K = (C^-1 - V^T Y)^-1, so
   that M = L^-1 - V C V^T (Woodbury): the coupling's soft modes are handled exactly and the PCG
   iterates only against the local polynomial's error.  A term needs no grid barrier.  Runs in a
   pipelined PCG (two grid barriers per iteration); one system per call. */
#define HSC_PRECOND_BLOCK 4          /* poly_degree caller weights (0: neumann_order unit weights) */
#define HSC_PRECOND_BLOCK_LEARNED 5  /* 8 weights per system from the learned model (as _LEARNED) */

/* learned model: 16 features -> 64 -> 64 -> 8 positive weights (ReLU, softplus), BF16 parameters,
   flat row-major (out x in): W1[64][16], b1[64], W2[64][64], b2[64], W3[8][64], b3[8] */
#define HSC_FEATURES 16
#define HSC_MLP_HIDDEN 64
#define HSC_MLP_OUT 8
#define HSC_MLP_PARAMS 5768

#define HSC_MAX_POLY 16

typedef struct hsc_options {
    int32_t max_rank;            /* linear_system/hsc/max_rank (reference default 128) */
    double aca_rtol;             /* 0: fixed rank with a roundoff zero-pivot guard (reference) */
    int32_t neumann_order;       /* linear_system/hsc/neumann_order (reference default 5) */
    double omega;                /* linear_system/hsc/omega (0.7) */
    int32_t max_iter;            /* linear_system/hsc/max_iter (2000) */
    double tol;                  /* linear_system/tol_rate: relative Schur residual */
    int32_t abd_inverse;         /* HSC_ABD_*; adaptive_abd_inverse=1 maps to HSC_ABD_ADAPTIVE */
    double abd_inverse_tol;      /* linear_system/hsc/abd_inverse_tol (1e-5) */
    double full_residual_limit;  /* linear_system/hsc/full_residual_limit (0.1) */
    int32_t precision;           /* HSC_FP64 / HSC_FP32 / HSC_BF16 */
    int32_t preconditioner;      /* HSC_PRECOND_* */
    int32_t poly_degree;         /* number of weights used with HSC_PRECOND_POLY / _SCHUR_POLY */
    double poly_weights[HSC_MAX_POLY];
    int32_t residual_replacement;/* iterations between FP64 true-residual replacements; 0 = only at convergence */
    double refine_target;        /* > 0: repeat HSC directions with exact line search until
                                    |b - H x|/|b| <= target (core.py:171-198) */
    int32_t max_refinements;
    int32_t fallback_on_stall;   /* polynomial / learned preconditioners: redo a single-system solve with plain
                                    Neumann (neumann_order) when PCG breaks down or hits max_iter */
    int32_t threads_per_row;     /* SpMV tile width: 2, 4 or 8 -> 1, 2 or 4 slices of 32 blocks loaded per
                                    warp round trip (autotuned); 0 (default): 4 on the shared-memory-resident
                                    path, 2 when the slices stream from memory */
    int64_t spin_limit;          /* bound on every device-side barrier wait */
    int32_t check_residual;      /* 1: compute the full residual and enforce full_residual_limit */
    int32_t trace_iterations;    /* > 0: record per-CTA SM clocks at the PCG phase boundaries of the
                                    first iterations (hsc_get_trace) */
    int32_t resident;            /* 1 (default): each PCG CTA keeps its BSR slice, vector window and own-row
                                    vectors in shared memory when they fit (vehicle system: 10-15 % less time
                                    per iteration in FP32, FP64 within 1 %); 0: stream them from L2 */
    int32_t fuse_update;         /* resident mode, FEM-basis polynomial of 2+ terms: 1 folds the x/r update
                                    into the first preconditioner phase (each CTA forms
                                    t0 = w Dd^-1 (r - alpha S p) over its own window), one grid barrier
                                    fewer per iteration; 0 (default): separate update phase, which measured
                                    as fast on the vehicle system (the window-wide t0 costs what the barrier did) */
    int32_t aca_cluster;         /* 1 (default): 16-CTA cluster ACA (distributed shared memory) when the
                                    coupling fits it; 0: always the grid kernel (column strips, one grid
                                    barrier per rank step), which also serves couplings too large for it */
    int32_t reorder;             /* 1 (default): renumber the FEM nodes internally into compact parts of
                                    balanced weight, one per PCG CTA (smaller vector windows; the parts are the
                                    blocks of HSC_PRECOND_BLOCK*); 0: keep the caller's order.  Inputs and
                                    outputs are always in the caller's order */
    int32_t aca_components;      /* 1 (default): run the ACA per coupling component (bodies joined through
                                    shared FEM nodes, on which E is block diagonal), one CTA each, and merge
                                    the pivot sequences by magnitude: the same pivots, columns and column
                                    order as the global full-pivot ACA; 0: the global cluster / grid ACA */
    int32_t lanczos_stats;       /* 1: after each solve, the extreme Ritz values of the preconditioned Schur
                                    operator from the CG coefficients (host bisection) into the stats and the
                                    next solve's feature record; 0 (default): only for the learned
                                    preconditioners, which read that record */
    double coupled_part_weight;  /* block preconditioners: the node partition runs twice, the second time
                                    with the nodes of the first pass's parts that hold a coupled node
                                    weighted by this factor (those parts also do their components' low-rank
                                    work on every row), so they come out smaller; 1: one pass.  The
                                    partition is cached per FEM pattern: a contact change reuses it.
                                    Default 1.2 */
    int32_t graph_replay;        /* 1: hsc_solve on a non-default stream captures its numeric phase into a CUDA
                                    graph once per pattern (and pointers, options) and replays it (one launch
                                    instead of ~44; the per-stage times in hsc_stats are then 0, total_ms
                                    stays); 0 (default): direct launches.  Not with refinement or the
                                    adaptive ABD inverse (their host decisions run between launches) */
} hsc_options;

typedef struct hsc_stats {        /* superset of the hsc_stats.jsonl record (linear_hsc.cu:420-431) */
    int32_t status;
    int32_t fem_dofs, abd_dofs, active_fem_dofs, rank;
    int32_t pcg_iterations, neumann_doublings, refinement_steps;
    int32_t precision, preconditioner, fallback, accepted;
    int32_t residual_replacements;
    double aca_relative_error;
    double schur_relative_residual;   /* recursive residual at exit (true residual after a check) */
    double full_relative_residual;    /* |b - H x| / |b| in FP64 on the assembled H */
    double abd_inverse_residual;      /* |I - A P|_F / sqrt(qm) */
    double full_residual_limit;
    double descent;                   /* b^T x */
    double setup_ms, pcg_ms, total_ms;/* device time between stream events */
    double lanczos_min, lanczos_max;  /* extreme Ritz values of the preconditioned Schur operator */
    double stage_ms[8];               /* fill+extract, ACA, the ABD inverse's time beyond the ACA (the two run
                                         concurrently), reduced core, rhs, PCG, back-sub+residual, block
                                         preconditioner setup (Y = L V, K; the PCG stage excludes it) */
    int64_t nnzb;
    double analysis_ms;               /* host time of this call's pattern analysis (CSR plans, node partition,
                                         CTA windows, block plan), 0 when the pattern was already analysed */
} hsc_stats;

typedef struct hsc_bcoo3 {        /* CBCOOMatrixView<double,3> */
    const int32_t* d_rows;        /* block row index per triplet */
    const int32_t* d_cols;        /* block column index per triplet */
    const double* d_values;       /* 9 doubles per triplet, column-major 3x3 (Eigen Matrix3x3) */
    int64_t nnzb;                 /* triplet count; ONE triangle stored, (row, col) unique */
    int32_t nblock;               /* block rows = dofs / 3 */
} hsc_bcoo3;

typedef struct hsc_dof_layout {   /* ABDLinearSubsystem / FEMLinearSubsystem dof_offset, dof_count */
    int32_t qo, qm, fo, fn;
} hsc_dof_layout;

typedef struct hsc_ctx hsc_ctx;

/* Fill *opt with the framework defaults (FP64, exact ABD inverse, order 2). */
HSC_EXPORT int hsc_options_default(hsc_options* opt);
/* The reference plugin's defaults (linear_hsc.cu:162-164): order 5, adaptive ABD, tol 1e-4. */
HSC_EXPORT int hsc_options_reference(hsc_options* opt);

/* do_build: create a context on the current CUDA device. */
HSC_EXPORT int hsc_create(const hsc_options* opt, hsc_ctx** out);
HSC_EXPORT void hsc_destroy(hsc_ctx* ctx);
HSC_EXPORT int hsc_set_options(hsc_ctx* ctx, const hsc_options* opt);
/* Message of the last failing call on this context ("" when none). */
HSC_EXPORT const char* hsc_last_error(const hsc_ctx* ctx);

/* do_solve: x = HSC(A, b).  The sparsity analysis is cached while the A
 * pointers, nnzb, nblock and layout stay the same; a changed pattern behind
 * the same pointers is detected on the device and triggers a fresh analysis.
 * `stream` is a cudaStream_t (NULL = legacy default stream).  With the
 * graph_replay option and a non-default stream the solve replays its
 * captured CUDA graph. */
HSC_EXPORT int hsc_solve(hsc_ctx* ctx, const hsc_bcoo3* A, const hsc_dof_layout* layout,
              const double* d_b, double* d_x, void* stream, hsc_stats* out);

/* Many independent systems in one persistent PCG launch.  With
 * use_graph != 0 the numeric phase is captured once into a CUDA graph and
 * replayed while the pointers and patterns are unchanged. */
HSC_EXPORT int hsc_solve_batch(hsc_ctx* ctx, int32_t count, const hsc_bcoo3* A, const hsc_dof_layout* layouts,
                    const double* const* d_b, double* const* d_x, int32_t use_graph,
                    void* stream, hsc_stats* out);

/* IterativeSolver::spmv: y = H x with the full symmetric H (both triangles). */
HSC_EXPORT int hsc_spmv(hsc_ctx* ctx, const hsc_bcoo3* A, const hsc_dof_layout* layout,
             const double* d_x, double* d_y, void* stream);

/* y = H x like hsc_spmv, but with no context and no device allocation, for
 * callers that cannot allocate when they need the product (a fixed up-front
 * memory pool, or a loop that must not take cudaFree's device-wide sync).  It
 * accumulates in a static 8 MiB device array of this library, so at most
 * 1,048,576 dofs (3 * nblock); larger systems get HSC_ERR_INVALID.  Calls that
 * overlap on the GPU share that array and race; the first call on a device
 * looks up the array's address and should come before any stream capture.
 * Under lazy module loading (the CUDA 12 default) that first call also loads
 * the module that holds the array, so nothing is allocated from the second
 * call on.  Triplets with a block index outside [0, nblock) are skipped by the
 * kernel and make the call return HSC_ERR_INVALID (y then holds the product of
 * the valid triplets).  The call waits for its stream before it returns.
 * y may alias x.  This entry point has no counterpart in the reference. */
HSC_EXPORT int hsc_spmv_noalloc(const hsc_bcoo3* A, const double* d_x, double* d_y, void* stream);

/* Host copies of the last solve's coupling factors (tests / diagnostics).
 * U: qm x rank, V: active x rank, both column-major; active: FEM dof indices. */
HSC_EXPORT int hsc_get_factors(hsc_ctx* ctx, int32_t sys, int32_t* rank, int32_t* n_active,
                    double* U, int32_t ldu, double* V, int32_t ldv, int32_t* active);

/* Phase-boundary SM clocks of the last PCG launch when trace_iterations > 0:
 * out[(cta * iterations + it) * 16 + event], events 0 loop top, 1 phase A done,
 * 2 after its barrier, 3 phase B done, 4 after its barrier, 5 last
 * preconditioner phase done, 6 after its barrier; resident mode also records
 * 7 / 8 the last preconditioner phase's window staged / SpMV done, 9 / 10 the
 * same for phase A, 11 phase B's alpha known, 12 its low-rank correction done,
 * 13 its row update done.  Events 5-8 of an iteration record the preconditioner
 * phases that run just before its loop top (event 0).  *ctas receives the grid size. */
HSC_EXPORT int hsc_get_trace(hsc_ctx* ctx, unsigned long long* out, int64_t max_entries, int32_t* ctas,
                             int32_t* iterations);

/* The internal FEM node numbering of system `sys` (after a solve or hsc_spmv): perm[i] = the caller's
 * node of internal node i (n entries), part_ptr[p] = first internal node of part p (nparts + 1
 * entries); any pointer may be NULL.  *n and *nparts receive the sizes. */
HSC_EXPORT int hsc_get_partition(hsc_ctx* ctx, int32_t sys, int32_t* n, int32_t* nparts, int32_t* perm,
                                 int32_t* part_ptr);
/* The node partition the analysis uses, on host arrays (no device needed): adjacency CSR over n nodes
 * (symmetric, no self loops), a positive weight per node; part[i] in [0, nparts). */
HSC_EXPORT int hsc_partition_nodes(int32_t n, const int32_t* adj_ptr, const int32_t* adj, const double* weight,
                                   int32_t nparts, int32_t* part);

/* Host copy of the last solve's ABD inverse P (qm x qm, row-major). */
HSC_EXPORT int hsc_get_abd_inverse(hsc_ctx* ctx, int32_t sys, double* P);

/* ---------------------------------------------------------------------------
 * GPU assembly of the log-Neo-Hookean Tet4 Hessian (the FEM block of a Newton
 * system) into the solver's input form: one-triangle BCOO over nodes, sorted,
 * unique, column-major 3x3 values; dt^2 V-scaled, SPD-projected per tet, plus
 * the lumped mass.  Replaces log_neo_hookean_3d.cu:62-135 (per-tet Hessian,
 * ddEddF_spd of log_neo_hookean_function.h:108-150) and the triplet-to-BCOO
 * conversion of global_linear_system.cu:215-248 (ge2sym) for this block.
 * ------------------------------------------------------------------------- */
typedef struct hsc_fem_assembler hsc_fem_assembler;
/* Mesh analysis (host arrays: tets ntet x 4 node ids, rest positions nnode x 3): rest shape
 * matrices, volumes, lumped masses (rho V / 4 per tet corner) and the block pattern. */
HSC_EXPORT int hsc_fem_assembler_create(const int32_t* tets, int32_t ntet, int32_t nnode, const double* rest_x,
                                        double rho, double nu, double dt, int32_t project,
                                        hsc_fem_assembler** out);
HSC_EXPORT void hsc_fem_assembler_destroy(hsc_fem_assembler* a);
/* The pattern: *nnzb blocks; d_rows / d_cols (device, may be NULL) receive the node indices. */
HSC_EXPORT int hsc_fem_pattern(const hsc_fem_assembler* a, int32_t* d_rows, int32_t* d_cols, int64_t* nnzb);
/* Numeric assembly at positions d_x (nnode x 3) with Young's moduli d_E (per tet) into d_values
 * (nnzb x 9).  With `inverted` (host) set, waits and reports tets with det F <= 0 (HSC_ERR_NONSPD). */
HSC_EXPORT int hsc_fem_assemble(hsc_fem_assembler* a, const double* d_x, const double* d_E, double* d_values,
                                int32_t* inverted, void* stream);
/* Line-search feasibility of a Newton direction (feasible_segment, log_neo_hookean_function.h:37-75, as the
 * energy kernel applies it, log_neo_hookean_3d.cu:45-52): the largest alpha = alpha0 * 2^-m, m <= max_halvings,
 * such that det F(x0 + s dx) > 1e-8 on every tet for all s in [0, alpha].  *halvings = m, *limited = the tets
 * that needed m > 0.  HSC_ERR_NONSPD (alpha = 0) when no such step exists or x0 itself is inverted. */
/* ABD-FEM contact coupling, assembled on the device (reference: ABDFEMLinearSubsystem_assemble_kernel,
 * abd_fem_linear_subsystem.cu:18-61) and fused with the solver's active-column and E extraction
 * (linear_hsc.cu:205-247).  Per contact: H12x3 = J(xbar)^T H (zero when the body or the FEM node is fixed),
 * summed per (body, node) pair in input order; output, sorted by (row, col): the upper-triangle blocks
 * (abd_block_offset + 4 body + k, fem_block_offset + node), k = 0..3, of every pair with a nonzero block
 * (column-major 3x3 values); the sorted global dofs 3 (fem_block_offset + node) + j of the nodes with a
 * coupling block of nonzero squared norm; and E (12 nbody x nactive, row-major) over them.
 * p_first = 1: body dofs (p, a1, a2, a3) with x = p + (a1.xbar, a2.xbar, a3.xbar) (libuipc's order);
 * p_first = 0: (a1, a2, a3, p).  body_fixed / fem_fixed may be NULL. */
typedef struct hsc_coupling_assembler hsc_coupling_assembler;
HSC_EXPORT int hsc_coupling_assembler_create(int32_t n_abd_vertices, const int32_t* v2b, const double* x_bar,
                                             int32_t nbody, const int32_t* body_fixed, int32_t nfem,
                                             const int32_t* fem_fixed, int32_t abd_block_offset,
                                             int32_t fem_block_offset, int32_t p_first, hsc_coupling_assembler** out);
HSC_EXPORT int hsc_coupling_assembler_destroy(hsc_coupling_assembler* a);
/* d_abd_vertex: ABD-local vertex per contact; d_fem_vertex: FEM-local node; d_H: 9 doubles per contact, the
 * column-major 3x3 block (rows: the ABD vertex's dofs, columns: the FEM node's).  Synchronises the stream once
 * to size E; *nblocks and *nactive are the output sizes.  HSC_ERR_INVALID on an index out of range. */
HSC_EXPORT int hsc_coupling_assemble(hsc_coupling_assembler* a, const int32_t* d_abd_vertex,
                                     const int32_t* d_fem_vertex, const double* d_H, int32_t ncontact,
                                     int32_t* nblocks, int32_t* nactive, void* stream);
/* Copies the last assembly's outputs (any pointer may be NULL): rows/cols [nblocks], values [9 nblocks],
 * active [nactive], E [12 nbody x nactive]. */
HSC_EXPORT int hsc_coupling_read(hsc_coupling_assembler* a, int32_t* d_rows, int32_t* d_cols, double* d_values,
                                 int32_t* d_active, double* d_E, void* stream);
HSC_EXPORT int hsc_fem_feasible_step(hsc_fem_assembler* a, const double* d_x0, const double* d_dx, double alpha0,
                                     int32_t max_halvings, double* alpha, int32_t* halvings, int32_t* limited,
                                     void* stream);

/* ---------------------------------------------------------------------------
 * Learned polynomial preconditioner (no reference counterpart; the reference
 * fixes the Neumann weights to 1, linear_hsc.cu:330-343).
 * ------------------------------------------------------------------------- */
/* Load the model used by HSC_PRECOND_LEARNED: HSC_MLP_PARAMS BF16 values (host memory). */
HSC_EXPORT int hsc_set_learned_model(hsc_ctx* ctx, const uint16_t* params_bf16);
/* The HSC_FEATURES features of system `sys` as the learned model sees them: statistics of the
 * current numeric system plus the record of the solve before the last one.  Call after a solve. */
HSC_EXPORT int hsc_get_features(hsc_ctx* ctx, int32_t sys, float* out);
/* Polynomial weights the last solve of `sys` used (learned: the model's output). */
HSC_EXPORT int hsc_get_poly_weights(hsc_ctx* ctx, int32_t sys, double* out, int32_t max, int32_t* degree);
/* CG coefficients (alpha_k, beta_k) of the last solve of `sys`, up to max_pairs pairs; they define
 * the Lanczos tridiagonal of the preconditioned Schur operator seen from the right-hand side. */
HSC_EXPORT int hsc_get_lanczos(hsc_ctx* ctx, int32_t sys, double* coef, int32_t max_pairs, int32_t* pairs);

/* Training kernels of the model (device pointers, the caller's stream).  batch samples, row-major.
 * forward: x (batch x 16) -> h1, h2 (batch x 64, after ReLU), o (batch x 8, before softplus),
 * w = softplus(o); any of h1, h2, o, w may be NULL. */
HSC_EXPORT int hsc_mlp_forward(const uint16_t* d_params, const float* d_x, int32_t batch, float* d_h1,
                               float* d_h2, float* d_o, float* d_w, void* stream);
/* backward: gradient of the parameters (HSC_MLP_PARAMS floats, summed over the batch in sample order)
 * from gw = dL/dw (batch x 8); d_scratch holds batch * (8 + 64 + 64) floats. */
HSC_EXPORT int hsc_mlp_backward(const uint16_t* d_params, const float* d_x, const float* d_h1, const float* d_h2,
                                const float* d_o, const float* d_gw, int32_t batch, float* d_scratch,
                                float* d_grad, void* stream);
/* least-squares residual-polynomial loss of each sample and its gradient in w:
 * L = scale * sum_i tau_i (1 - theta_i sum_k w_k (1 - theta_i)^k)^2, theta and tau batch x m. */
HSC_EXPORT int hsc_poly_ls_loss(const float* d_w, const float* d_theta, const float* d_tau, int32_t batch,
                                int32_t m, float scale, float* d_loss, float* d_gw, void* stream);
/* one Adam step on FP32 master parameters, writing their BF16 copy. */
HSC_EXPORT int hsc_adam_step(float* d_master, uint16_t* d_params, const float* d_grad, float* d_m, float* d_v,
                             int32_t n, float lr, float beta1, float beta2, float eps, float weight_decay,
                             int32_t step, void* stream);

HSC_EXPORT int hsc_version(void);
/* Kernels this library has launched in the process so far (all contexts). */
HSC_EXPORT long long hsc_kernel_launches(void);
/* First failed index guard of a self-checking build (-DHSC_CHECKED) as
 * (code, value) pairs for the ACA, PCG and setup kernels; zeros otherwise. */
HSC_EXPORT int hsc_debug_checks(long long* out6);
/* Self-test of the PCG grid barrier's failure path, with no GPU fault: one cooperative launch of `ctas`
 * CTAs (2..SM count) where CTA `absent` never arrives (-1: every CTA arrives); CTA 1 polls at most
 * `first_limit` times and the others at most `limit` times.  statuses[c] = 1 barrier passed, 0 left with
 * failure, 2 absent; *abort_flag / *where are the barrier's abort flag and the epoch that gave up.
 * (No reference counterpart: it checks this library's bounded waits.) */
HSC_EXPORT int hsc_debug_barrier_selftest(int32_t ctas, int32_t absent, int64_t first_limit, int64_t limit,
                                          int32_t* statuses, int32_t* abort_flag, int32_t* where);

/* z += omega * blockdiag(B) x over nblocks bs x bs blocks (bs 3 or 12), B given as bs*bs planes
 * d_planes[(i * bs + j) * nblocks + b] = B_b(i, j).  The shape of the authors' dmv_accumulate_kernel
 * (Guo-2026-HSC conjugate_gradient_cuda.cuh, run by reproduction/cuda_original.py); bs = 3 runs the PCG
 * kernel's own block-Jacobi product.  Test hook. */
HSC_EXPORT int hsc_debug_dmv_accumulate(int32_t bs, int32_t nblocks, const double* d_planes, const double* d_x,
                                        double* d_z, double omega, void* stream);

/* The block preconditioner's plan after a solve with it (first n of: CTAs, and the per-CTA maxima
 * R (rows), NS (16-row slices), NCH (chunks), W (window nodes), NA (coupled dofs), NCOL (Y columns);
 * value chunks staged (0/1), Y columns staged per CTA, the two kernels' shared-memory bytes,
 * coupling components, contributor slots, rank cap).  Test and profiling hook. */
HSC_EXPORT int hsc_debug_block_plan(hsc_ctx* ctx, int64_t* out, int32_t n);

#ifdef __cplusplus
}
#endif
#endif /* HSC_C_API_H */
