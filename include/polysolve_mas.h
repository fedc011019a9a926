/*
 * polysolve_mas.h — C ABI of the B200 MAS-PCG solver.
 *
 * A drop-in for polysolve's "MAS" linear solver (src/polysolve/linear/MASSolver.hpp:35-72 behind
 * the polysolve::linear::Solver interface, src/polysolve/linear/Solver.hpp:31-132). Plain C types
 * only: no exceptions cross this boundary. Every call returns an int status (MAS_OK = 0); on a
 * non-zero status mas_last_error() returns a message that starts with "[MAS]", as the reference's
 * exceptions do. The C++ header include/polysolve/linear/MASSolver.hpp turns statuses back into
 * the reference's exception types.
 *
 * Matrices are square CSC (column-major) with int32 indices, the layout of polysolve's
 * StiffnessMatrix = Eigen::SparseMatrix<double, ColMajor, int> (src/polysolve/Types.hpp:11).
 * A must be symmetric (CG requires it; the preconditioner reads only its upper triangle).
 *
 * Threading: a handle is used by one host thread at a time. All device work of a handle runs on
 * the handle's own CUDA stream on the device that was current when the handle was created.
 */
#ifndef POLYSOLVE_MAS_H
#define POLYSOLVE_MAS_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define MAS_OK 0
#define MAS_ERR_INVALID 1         /* bad argument or parameter (reference: std::runtime_error) */
#define MAS_ERR_OOM 2             /* device allocation failed (reference: CudaOutOfMemoryError) */
#define MAS_ERR_NOT_FACTORIZED 3  /* solve before factorize / size mismatch (MASSolver.cu:380-383) */
#define MAS_ERR_CUDA 4            /* a CUDA runtime call failed */
#define MAS_ERR_NONFINITE 5       /* NaN/inf initial residual (MASSolver.cu:483-486) */
#define MAS_ERR_INVERSE 6         /* a subdomain inverse hit a zero/non-finite pivot (MASPreconditioner.cu:931-935) */
#define MAS_ERR_TIMEOUT 7         /* a device-side wait hit its iteration limit */
#define MAS_ERR_NO_DEVICE 8       /* no CUDA device (MASSolver.cu:188-191, "No Nvidia GPU!!") */

/* Solver status after a solve, MASSolverStatus (MASSolver.hpp:10-16). */
#define MAS_STATUS_RUNNING 0
#define MAS_STATUS_REACH_RELATIVE_TOLERANCE 1
#define MAS_STATUS_REACH_ABSOLUTE_TOLERANCE 2
#define MAS_STATUS_REACH_MAX_ITERATIONS 3

typedef struct mas_solver mas_solver;

/* Solver::create(solver, precond) (Solver.cpp:310-499; "MAS" at :403-407). Only "MAS" is
 * accepted; precond is ignored as in the reference. Parameters get the implementation defaults
 * (MASSolver.cu:137-143): block_dim 1, max_iter 5000, relative_tolerance 1e-5,
 * absolute_tolerance 1e-8, lazy_partitioning false, use_preconditioned_residual_norm false. */
int mas_create(const char *solver, const char *precond, mas_solver **out);

/* Solver::create(json params, logger, strict) (Solver.cpp:145-167): validates params against
 * the /MAS spec (linear-solver-spec.json:456-509), injects the spec defaults (max_iter 10000,
 * relative_tolerance 1e-4, lazy_partitioning true, ...) and calls set_parameters. */
int mas_create_json(const char *params_json, int strict_validation, mas_solver **out);

/* ~MASSolver. Safe on NULL. */
void mas_destroy(mas_solver *h);

/* MASSolver::set_parameters (MASSolver.cu:605-614, 198-212): reads the "MAS" object of the given
 * JSON object and silently ignores the call when it is absent. Keys of the reference: block_dim,
 * max_iter, relative_tolerance, absolute_tolerance, lazy_partitioning,
 * use_preconditioned_residual_norm. Keys this implementation adds (ignored by the reference):
 * precision ("fp64" | "fp32" | "fp16": storage of the MAS inverses; fp16 keeps one power-of-two
 * scale per matrix and multiplies in FP32), true_residual_period (int, reference 4), check_period (int,
 * reference 10), initial_guess ("zero" | "input" | "learned"; reference: zero), beta
 * ("fletcher_reeves" | "polak_ribiere"), ordering ("auto" | "morton" | "graph" | "natural"),
 * poll_period (int: iterations launched between looks at the device state), cuda_graphs (bool),
 * preconditioner_refresh (int k: values-only refactorizations rebuild the MAS inverses every k-th
 * time; 1, every time, as the reference), profile_kernels (bool: CUDA-event time per kernel kind,
 * reported by get_info), device_wait_limit (int >= 0: iterations of each bounded device-side wait
 * before the solve stops with MAS_ERR_TIMEOUT; default 1048576, 0 makes every wait give up at
 * once, which tests the timeout path), rhs_group (0 | 4 | 16: right-hand sides per group of
 * mas_solve_multi; 0 picks 16 for more than four with block_dim 3, else 4), chained_launch (bool,
 * default true: the single-right-hand-side PCG kernels use programmatic dependent launch, each
 * becoming resident while its predecessor drains; results are the same either way), spmv_unroll (1 |
 * 2 | 4, default 2: block slots per loop trip of the SpMV, a launch shape the autotuner picks; the
 * same bits either way), wide_apply ("mma_sync" | "tcgen05": tensor-core path of the sixteen-wide
 * apply of mas_solve_multi), batch_launch ("fused" | "streams", default streams: how
 * mas_solve_batch runs the handle, see there), batch_groups (0..64, default 0 = 1: fused groups of
 * a batch), apply_items_per_warp (1..64, default 1: the fewest inverses per warp of the MAS apply,
 * which sets its grid; more suit batches of small systems, and the dot products' summation
 * grouping follows the grid, so results can differ in the last bits between settings). */
int mas_set_parameters(mas_solver *h, const char *params_json);

/* MASSolver::get_info (MASSolver.cu:214-219): writes a JSON object with solver_iter,
 * solver_error (absolute residual norm), solver_status (reference strings), plus extras.
 * *needed receives strlen+1; the text is truncated to cap bytes (always NUL terminated). */
int mas_get_info(const mas_solver *h, char *buf, size_t cap, size_t *needed);

/* MASSolver::name() == "MAS" (MASSolver.cu:636-639). */
const char *mas_name(void);

/* MASSolver::analyze_pattern (MASSolver.cu:621-624): a no-op in the reference; here it only
 * checks the arguments. */
int mas_analyze_pattern(mas_solver *h, int n, const int *outer, const int *inner, int nnz, int precond_num);

/* New, optional: vertex positions (xyz per block row, nverts = ceil(n / block_dim)) for the
 * Morton subdomain ordering. Without positions factorize orders the blocks by graph bisection.
 * The reference partitions with KaMinPar instead (MASSolver.cu:223-242). */
int mas_set_positions(mas_solver *h, const double *xyz, int nverts);

/* MASSolver::factorize(A) (MASSolver.cu:292-374): A as CSC host arrays outer[n+1], inner[nnz],
 * vals[nnz]. Builds the subdomain ordering, the permuted block matrix and the MAS
 * preconditioner on the device. The ordering is reused while the pattern, the positions and the
 * ordering parameter are unchanged (with lazy_partitioning: while n is unchanged); with the
 * same pattern only the values are re-scattered and the inverses rebuilt (the coarse space,
 * buffers and CUDA graphs are kept). Row order inside a column is free; row indices outside
 * [0, n), decreasing column pointers or outer[n] != nnz give MAS_ERR_INVALID before the pattern
 * is used (checked in the same host pass that hashes the pattern). */
int mas_factorize_csc(mas_solver *h, int n, const int *outer, const int *inner, const double *vals, int nnz);

/* New, no reference counterpart: a values-only refactorization the caller declares. vals are the
 * new values in the CSC order of the last factorized matrix (same pattern, nnz of them); the row
 * indices are neither passed nor read, so the pattern check (a hash of 4 bytes per entry) is
 * skipped. Requires an earlier factorization with unchanged positions, ordering, block_dim and
 * precision (otherwise MAS_ERR_INVALID; MAS_ERR_NOT_FACTORIZED before any factorization). */
int mas_factorize_values(mas_solver *h, const double *vals, int nnz);

/* MASSolver::solve(b, x) (MASSolver.cu:376-409): host vectors of length n. With initial_guess
 * "zero" (the reference's behaviour, MASSolver.cu:395-398) x is output only; with "input" x is
 * also the starting guess. Synchronous. Non-convergence is not an error: see get_info. */
int mas_solve(mas_solver *h, const double *b, double *x, int n);

/* New: learned warm start for sequences of systems with one pattern (initial_guess
 * "learned"). The solver keeps its last four solutions on the device; the next solve starts
 * from the energy-minimising combination of x_{k-1}, the differences x_{k-i} - x_{k-i-1} and a
 * message-passing network's correction (falling back to x_{k-1}), computed on the GPU from b,
 * the diagonal blocks and the kept solutions. block_dim 3 only. The reference always starts from x0 = 0
 * (MASSolver.cu:395-398); its caller refactorizes and solves every Newton step
 * (Newton.cpp:173-214).
 * params: MAS_WS_PARAMS float32 in the .psws order (polysolve_b200/warmstart.py). */
#define MAS_WS_FEATURES 16
#define MAS_WS_HIDDEN 64
#define MAS_WS_LAYERS 3
#define MAS_WS_PARAMS 26051
int mas_set_warm_start_model(mas_solver *h, const float *params, long long count);
/* Forget the kept solutions (the next solve starts from zero). A factorization with a new
 * pattern or ordering also forgets them. */
int mas_reset_warm_start(mas_solver *h);

/* New, no reference counterpart: training of the learned warm start's network on the GPU with this
 * library's own forward and reverse-pass kernels (BF16 tensor-core products, FP32 accumulation and
 * FP32 Adam state). A sample is one step of a sequence of systems with one pattern: add it from a
 * solver factorized with that step's matrix, with b, 2 to 4 kept solutions history[j * n ..]
 * (x_{k-1} first) and the exact solution x_exact (all caller order, length n); the trainer runs the
 * solver's own prediction pipeline up to the features and keeps the sample in device memory. The
 * loss of a sample is 1 - rho, rho = (c . r_g)^2 / ((c . A c) (e . r_g)) with r_g the residual of the
 * kept solutions' Galerkin combination x_g and e = x_exact - x_g.
 *   create:   initial parameters (MAS_WS_PARAMS float32, the .psws order); Adam moments start at 0.
 *   train:    one Adam step (beta1 0.9, beta2 0.999, eps 1e-8) per listed sample, in order, with the
 *             given learning rates; losses (optional) receives each step's loss before its update.
 *   evaluate: rho of each listed sample under the current parameters.
 *   gradient: the loss and its gradient (MAS_WS_PARAMS floats) for one sample; no update. */
typedef struct mas_ws_trainer mas_ws_trainer;
int mas_ws_trainer_create(const float *params, long long count, mas_ws_trainer **out);
void mas_ws_trainer_destroy(mas_ws_trainer *t);
int mas_ws_trainer_add_sample(mas_ws_trainer *t, mas_solver *h, const double *b, const double *history, int nhist,
                              const double *x_exact, int n);
int mas_ws_trainer_sample_count(const mas_ws_trainer *t);
int mas_ws_trainer_train(mas_ws_trainer *t, const int *samples, const float *lr, int count, double *losses);
int mas_ws_trainer_evaluate(mas_ws_trainer *t, const int *samples, int count, double *rho);
int mas_ws_trainer_gradient(mas_ws_trainer *t, int sample, float *grad, long long count, double *loss);
int mas_ws_trainer_get_params(const mas_ws_trainer *t, float *params, long long count);
/* Last error of the trainer ("" if none); with t == NULL the last mas_ws_trainer_create error. */
const char *mas_ws_trainer_last_error(const mas_ws_trainer *t);

/* New: nrhs independent right-hand sides, column-major B[n * nrhs] / X[n * nrhs]. */
int mas_solve_multi(mas_solver *h, const double *B, double *X, int n, int nrhs);

/* Batched solves of independent systems (the 64-system workload; no reference counterpart in
 * MASSolver, which solves one system per call): every handle must be factorized and distinct;
 * b[i], x[i] have length n[i] (host arrays, or device arrays when device_pointers != 0).
 * Fused (every handle with batch_launch "fused", graphs on, no profiling, no learned warm start,
 * the same device, block_dim, precision, true_residual_period, poll_period, spmv_unroll and
 * batch_groups): the systems are cut by size into batch_groups groups, and each PCG phase is one
 * launch for all unfinished systems of a group, on the group's own stream; each system's results
 * are bit-identical to mas_solve's. Otherwise each handle runs on its own CUDA stream. In both
 * forms a pool of `threads` host threads (<= 0: one per hardware thread, at most 64) runs the
 * per-handle steps. statuses (optional, count entries) receives each handle's status; the return
 * value is the first non-zero status. */
int mas_solve_batch(mas_solver *const *handles, int count, const double *const *b, double *const *x,
                    const int *n, int device_pointers, int threads, int *statuses);

/* New: solve with device pointers (length n, caller's order) on the handle's stream; the call
 * returns when the solve has finished. */
int mas_solve_device(mas_solver *h, const double *d_b, double *d_x, int n);

/* New: run the handle's device work on the caller's CUDA stream (a cudaStream_t; NULL restores
 * the handle's own stream). Calls still return only when their work has finished. */
int mas_set_stream(mas_solver *h, void *stream);

/* New, no counterpart in the reference: y = A x and *d_dot = x . (A x) on the factorized matrix,
 * with no device allocation at all, for callers that cannot allocate at call time (inside a CUDA
 * stream capture, or in applications that reserve all device memory up front and forbid later
 * allocations). d_x, d_y: device vectors of length len = nodes * block_dim in the solver's padded
 * block order (see mas_get_sizes); d_dot: one device double. The three buffers must not overlap
 * (MAS_ERR_INVALID otherwise). Runs on `stream` (a cudaStream_t, NULL = the handle's stream)
 * without synchronizing. The reduction scratch is a static device array of 256 KB + 8 B (held by
 * every GPU where the library's module is loaded, until exit), which limits the matrix to 262,144
 * banks (8,388,608 block rows); larger matrices get MAS_ERR_INVALID. All calls share that scratch:
 * calls that overlap on the GPU race. The first call on a device (and the first after a
 * cudaDeviceReset) looks the scratch address up (cudaGetSymbolAddress), which under CUDA's lazy
 * module loading also loads the module and its array onto the device: make it before any stream
 * capture and before reserving the rest of the device's memory. */
int mas_spmv_dot_noalloc(mas_solver *h, const double *d_x, double *d_y, double *d_dot, int len, void *stream);

/* Test hook, process-wide (no reference counterpart; the reference's allocation failure is
 * mas::CudaOutOfMemoryError, mas_utils/CudaUtils.cuh:41-124): after `after` more successful device
 * allocations the next one fails as if the device were out of memory, once, and the call that made
 * it returns MAS_ERR_OOM with the requested and free MB in its message. Negative: off. */
int mas_debug_fail_allocation(long long after);

/* Last error message of the handle ("" if none). With h == NULL: the last mas_create error. */
const char *mas_last_error(const mas_solver *h);

/* ------------------------------------------------------------------------------------------
 * Inspection entry points (new; used by parity tests and tools). Vectors here are in the
 * solver's padded block order: node = bank * 32 + lane, length nodes * block_dim.
 * ---------------------------------------------------------------------------------------- */

/* sizes[0..11] = n, block_dim, V (block rows), banks, nodes (= banks*32), nnzb, level_num,
 * total_mats, cco_nums[0..3]. */
int mas_get_sizes(const mas_solver *h, int *sizes);

/* padded[V]: padded node id of each original block row. */
int mas_get_ordering(const mas_solver *h, int *padded, int V);

/* Host-only (no device needed): the subdomain ordering factorize would compute. mode is "morton"
 * (xyz required, one point per block row), "graph" or "natural". Writes padded[ceil(n/bd)] and
 * *banks. Replaces the reference's KaMinPar partition (mas_utils/GraphPartition.cpp:176-289). */
int mas_order_blocks(int n, const int *outer, const int *inner, int block_dim, const double *xyz, const char *mode,
                     int *padded, int *banks);

/* map[nodes * 4]: coarse-space id per padded node and level (-1 for virtual nodes and unused
 * levels), the CoarseSpace map of MASPreconditioner.hpp:30-39 in padded order. */
int mas_get_coarse_map(const mas_solver *h, int *map, int nodes);

/* Inverse matrices in packed-upper row-major FP64 (MASPreconditioner.hpp:41-53 layout), matrix
 * m at out + m * (N*(N+1)/2), N = 32 * block_dim, for all total_mats matrices. */
int mas_get_inverses(const mas_solver *h, double *out, size_t count);

/* y = A x on host vectors in padded order. */
int mas_debug_spmv(mas_solver *h, const double *x, double *y, int len);

/* z = M^-1 r (MAS apply) on host vectors in padded order. */
int mas_debug_apply(mas_solver *h, const double *r, double *z, int len);
/* Test hooks of the several-right-hand-side kernels: padded block order with RHS_GROUP (4)
 * interleaved columns (value index (node * bd + component) * 4 + column); len = padded length * 4.
 * No reference counterpart. */
int mas_debug_apply_multi(mas_solver *h, const double *rin, double *zout, int len);
int mas_debug_spmv_multi(mas_solver *h, const double *xin, double *yout, int len);
/* Test hook of the learned warm start: the prediction for caller-order b and nhist (2 to 4) kept
 * solutions history[j * n ..] (x_{k-1} first) without a solve. Outputs (each may be NULL):
 * c_out[n] the network's correction, x0_out[n] the starting guess, features_out[nverts * 16] the
 * raw per-vertex features, state_out[39] = feature sums (5), Galerkin matrix (upper triangle by
 * rows, 15) and right-hand side (5) of the basis {x1, x1 - x2, x2 - x3, x3 - x4, c},
 * coefficients (5), energy of x0, energy of x1, fallback flag, kept basis vectors, and the
 * coefficients of x_g, the first pass over the basis without c (5). */
int mas_debug_warm_start(mas_solver *h, const double *b, const double *history, int nhist, double *c_out,
                         double *x0_out, float *features_out, double *state_out);

/* New: Matrix Market files for A and b, the format the reference's tests load with Eigen's
 * loadMarket / loadMarketVector (tests/test_linear_solver.cpp:25-50, :211-213). Host only.
 * mas_market_load reads "coordinate" (real / integer / pattern, general / symmetric: duplicates
 * summed, symmetric files expanded to the full matrix) into CSC with sorted rows, or "array"
 * files into a dense column-major array (a vector is n x 1). dims gives rows, cols, the CSC
 * entry count (or rows * cols for arrays) and whether it is dense; copy_csc fills outer[cols+1],
 * inner[nnz], vals[nnz]; copy_dense fills count = rows * cols values. Errors: MAS_ERR_INVALID
 * with the message in mas_market_last_error() (per thread). */
typedef struct mas_market mas_market;
int mas_market_load(const char *path, mas_market **out);
int mas_market_dims(const mas_market *m, int *rows, int *cols, long long *nnz, int *dense);
int mas_market_copy_csc(const mas_market *m, int *outer, int *inner, double *vals);
int mas_market_copy_dense(const mas_market *m, double *out, long long count);
void mas_market_free(mas_market *m);
const char *mas_market_last_error(void);
/* Writes a square CSC matrix as "coordinate real general", or only its lower triangle as
 * "coordinate real symmetric"; a vector as "array real general". 17 significant digits. */
int mas_market_write_csc(const char *path, int n, const int *outer, const int *inner, const double *vals,
                         int symmetric);
int mas_market_write_vector(const char *path, const double *x, long long n);

#ifdef __cplusplus
}
#endif

#endif /* POLYSOLVE_MAS_H */
