/*
 * jxcpr_b200.h -- C ABI of the B200 CPR-GMRES library (libjxcpr_b200.so).
 *
 * Plain pointers and sizes only.  Two layers:
 *
 *  1. Device-kernel entry points (jxcpr_*_dev): device pointers, the caller's
 *     CUDA stream passed as void*.  They replace the inner loops the
 *     reference runs on the CPU and are what a solver built on this library
 *     chains together.
 *  2. Host entry points with host arrays (jxcpr_* without _dev), used by the
 *     drop-in layer in jxcpr_dropin.h and by FFI callers.
 *
 * Every function returns a status code: 0 success, 1 generic, 2 memory,
 * 4 argument, 256 not converged (the reference's codes, jxfpamg-0220/include/
 * jxf_util.h:152-159), 512 CUDA failure, 1024 NaN/Inf found on the device.
 * jxcpr_last_error() returns a message for the calling thread's last failure.
 */
#ifndef JXCPR_B200_H
#define JXCPR_B200_H

#if defined(__GNUC__)
#define JXCPR_API __attribute__((visibility("default")))
#else
#define JXCPR_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define JXCPR_SUCCESS 0
#define JXCPR_ERROR_GENERIC 1
#define JXCPR_ERROR_MEMORY 2
#define JXCPR_ERROR_ARG 4
#define JXCPR_ERROR_CONV 256
#define JXCPR_ERROR_DEVICE 512
#define JXCPR_ERROR_NUMERIC 1024

/* Library version (major*10000 + minor*100 + patch). */
JXCPR_API int jxcpr_version(void);
/* Number of kernels this library has launched in the process so far. */
JXCPR_API unsigned long long jxcpr_launch_count(void);
/* Message describing the calling thread's last failure ("" if none). */
JXCPR_API const char *jxcpr_last_error(void);
/* The library keeps freed device blocks for reuse: a block made for a solver is reused on that
 * solver's stream at once (stream order), any other block only after a device synchronisation;
 * small blocks are carved from 32 MiB slabs.  This returns every idle block (and the slabs, once
 * none of their blocks is in use) to the driver. */
JXCPR_API int jxcpr_release_cached_memory(void);
/* out[4] = {cudaMalloc calls, their total ms, device synchronisations of the cache, their total ms}
 * since the library was loaded. */
JXCPR_API int jxcpr_pool_stats(double *out);

/* ---- BSR SpMV ------------------------------------------------------------
 * y = alpha*A*x + beta*y for a block-CSR matrix with bs x bs row-major blocks
 * (bs = 2 or 3), 0-based ia[nb+1], ja[nnzb], a[nnzb*bs*bs]; x, y have nb*bs
 * entries and must not alias.  Replaces jxf_BSRMatrixMatvec
 * (jxfpamg-0220/csrc/operation/mvops/seq_bsr_matvec.c:22-140) and the local
 * part of jxf_ParBSRMatrixMatvec (par_bsr_matvec.c:21-221), with the same
 * rounding sequence (bit-identical results).  staged != 0 selects the
 * TMA-staged kernel; 0 the direct-load kernel.  x and y must be 16-byte
 * aligned.
 */
JXCPR_API int jxcpr_bsr_matvec_dev(int nb, int bs, long long nnzb, const int *ia, const int *ja, const double *a,
                                   double alpha, const double *x, double beta, double *y, int staged,
                                   void *stream);
/* Same with FP32 block values and FP64 vectors (products formed in FP64). */
JXCPR_API int jxcpr_bsr_matvec_dev_f32(int nb, int bs, long long nnzb, const int *ia, const int *ja,
                                       const float *a, double alpha, const double *x, double beta, double *y,
                                       int staged, void *stream);
/* Reads and clears the per-device flag that the staged kernels raise when a
 * bounded wait on the copy engine gives up (0 = none). */
JXCPR_API int jxcpr_kernel_error_flag(void);

/* ---- BLAS-1 --------------------------------------------------------------
 * <x, y> over n doubles (16-byte aligned), deterministic order; the result is
 * written to *out_host after a stream synchronisation.  Replaces
 * jxf_SeqVectorInnerProd (jxfpamg-0220/csrc/operation/vecops/seq_vecop.c:239).
 */
JXCPR_API int jxcpr_dot_dev(long long n, const double *x, const double *y, double *out_host, void *stream);

/* <x, y> like jxcpr_dot_dev, but allocating nothing.  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory when
 * they need the product -- an application whose own memory pool has reserved
 * the whole device, or a time-critical loop that allows no allocator call
 * (cudaMalloc can synchronise the device and stall every stream).  The partial
 * sums live in a static device array (JXCPR_NOALLOC_DOT_MAX_PARTIALS partials of
 * JXCPR_NOALLOC_DOT_CHUNK elements each, 512 KB per GPU, kept until exit), so
 * n is limited to JXCPR_NOALLOC_DOT_MAX_PARTIALS * JXCPR_NOALLOC_DOT_CHUNK
 * (268,435,456) elements; larger n returns JXCPR_ERROR_ARG with a message.
 * The array is loaded with its code module on each device at the FIRST call
 * there (CUDA loads modules lazily), which takes device memory once: make a
 * warm-up call (n = 0 will do) on each device before your pool reserves it;
 * later calls allocate nothing.  The first call also resolves the array's
 * device address.  Every call copies the result to *out_host and synchronises
 * `stream`, so it must not be called while that stream is being captured.
 * The result equals jxcpr_dot_dev's up to rounding (a different, fixed
 * summation order; both are deterministic).  All calls share the array: calls
 * that overlap on the GPU (concurrent streams) race and must be serialised. */
#define JXCPR_NOALLOC_DOT_CHUNK 4096
#define JXCPR_NOALLOC_DOT_MAX_PARTIALS 65536
JXCPR_API int jxcpr_dot_dev_noalloc(long long n, const double *x, const double *y, double *out_host,
                                    void *stream);

/* ---- BSR files into device memory -------------------------------------------
 * Reads a BSR matrix file in the text (binary = 0) or binary (1) format of jxf_BSRMatrixRead /
 * jxf_BSRMatrixRead_Binary (jxfpamg-0220/csrc/mat_vec_data/seq_bsr_matrix.c:1735-2120) straight into
 * device arrays: the file is read in 64 MB chunks into pinned host memory and each chunk is copied
 * to the device while the next is read; a text file is tokenised and its numbers converted on the
 * device (values to the nearest FP64, as the host reader's fscanf gives: bit-identical arrays).
 * As the host readers: 1-based indices become 0-based, the largest column must be cols - 1, and
 * column-major blocks (storage 1) become row-major.  *ia (rows + 1), *ja (nnzb) and *a (nnzb*bs*bs)
 * are device allocations the caller releases with jxcpr_bsr_free_device.  Returns 4 (message in
 * jxcpr_last_error) for a file that cannot be opened or is malformed, 512 for a CUDA failure. */
JXCPR_API int jxcpr_bsr_read_device(const char *file, int binary, int *rows, int *cols, int *bs, long long *nnzb,
                                    int **ia, int **ja, double **a, void *stream);
JXCPR_API int jxcpr_bsr_free_device(int *ia, int *ja, double *a);
/* The device reader's conversion of one number token (no white space) on the host: 0 converted
 * (*out = the nearest FP64), 1 a form it leaves to strtod (more than 19 significant digits, inf,
 * nan), 2 not a number. */
JXCPR_API int jxcpr_parse_double_host(const char *token, int len, double *out);

/* ---- dense inverse (coarsest AMG level) ------------------------------------
 * ainv = a^-1 for a dense n x n row-major FP64 matrix (n <= 8192; device pointers, may not alias) by
 * blocked Gauss-Jordan elimination without pivoting, as the reference eliminates its coarsest level
 * (jxf_gselim, jxfpamg-0220/csrc/operation/matops/par_gs.c:20-74, no pivoting): one cooperative kernel,
 * trailing updates on the FP64 tensor cores.  The fast path's coarse solve is a GEMV with this inverse.
 * A zero pivot returns JXCPR_ERROR_ARG ("singular without pivoting").  Synchronises `stream`. */
JXCPR_API int jxcpr_dense_inverse_dev(int n, const double *a, double *ainv, void *stream);

/* ---- solver object ---------------------------------------------------------
 * CPR-GMRES on one GPU: jxcpr_solver_setup copies a BSR matrix (host or
 * device arrays), applies the configured decoupling (jxf_BSRMatrixDecouple,
 * jxfpamg-0220/csrc/cpr/jxf_bsr_decoup.c:1273) and builds the CPR
 * preconditioner (JXF_CPRSetup, jxfpamg-0220/csrc/cpr/jxf_cpr.c:268-422);
 * jxcpr_solver_solve decouples b and runs restarted GMRES
 * (jxf_GMRESSolve, jxfpamg-0220/csrc/krylov/pgmres.c:950-1713) with CPR
 * (JXF_CPRPrecond, jxf_cpr.c:424-610) as right preconditioner.  It returns 0
 * when the relative residual reached tol, JXCPR_ERROR_CONV (256) otherwise.
 *
 * Options (jxcpr_solver_set_int / _set_real; unknown keys return 4, as
 * JXF_CPRSetParameter does, jxf_cpr.c:226-262):
 *   int : k_dim (30), max_iter (100), min_iter (0), is_check_restarted (1),
 *         pressure_index (0), stage1_maxit (1), stage2_maxit (3),
 *         stage1_solver_type (1 AMG; 0 none), stage2_solver_type (2 HGS; 5 block ILU(0)
 *         correction z += BILU^-1 (r - A z) after CPR without sweeps; bilu_sweeps (3),
 *         bilu_ir_iters (5), bilu_lower_iters (5), bilu_upper_iters (5), bilu_exact (0; 1 exact
 *         factors and level-scheduled substitutions, FP32 factors in the mixed path)),
 *         decouple (0 none, 1 ABF, 5 True-IMPES), consistent_rhs (0: the
 *         reference's right-hand-side arithmetic, 1: solution-preserving),
 *         smoother_order (0 exact sequential order, 1 multicolour),
 *         rs_range_rows (131072; order 1: the coarsening's first pass on row
 *         ranges of this size, as each process of a distributed run does it,
 *         par_coarsen_ruge.c:37-44; 0 one pass over the level),
 *         rs_range_rows_coarse (0: as rs_range_rows; the range size on the
 *         levels below the finest),
 *         coarse_exact (1 substitution in the reference's order, 0 inverse),
 *         dep_launch (1; order 1: the preconditioner's kernels launched as
 *         programmatic dependents inside its CUDA graphs),
 *         use_tma_spmv (1), print_level, logging, block_size (ignored),
 *         order-1 (fast path) choices: precision (0 FP64, 1 FP32, 2 FP32 + BF16
 *         from level bf16_level (1), 3 FP32 stage 1 + FP64 stage 2),
 *         fast_smoother (0 colour GS / l1-Jacobi, 1 Chebyshev-3 on the dense
 *         levels, 2 learned settings, 3 Chebyshev-3 everywhere), max_colors (8:
 *         levels needing more colours use l1-Jacobi), flexible (0), graphs (1),
 *         graph_gmres (0), krylov_fp32 (0; 1 with graph_gmres: the Krylov
 *         basis and the flexible directions stored in FP32, every product,
 *         norm, rotation, residual and x in FP64), selective_reorth (0; 1
 *         with graph_gmres: the second classical Gram-Schmidt pass only when
 *         the first removed more than half of ||w||^2), orthog (0 modified, 1 one-pass classical
 *         Gram-Schmidt), autotune (1; 2 shared per shape class), stage2_lanes
 *         (4: CSR stage 2 without autotuning), stage2_chunk (4: stage 2 visits
 *         chunks of this many consecutive block rows in natural order, the
 *         chunks coloured for parallelism; 8 or 16 also accepted; 0: the
 *         level-0 colour order), tail_rows (0: fast path, the V-cycle's
 *         levels from the first with at most this many rows, the coarsest
 *         included, run as one cooperative kernel; 0 one launch per pass),
 *         tail_ctas (0: that kernel's grid, sized by its largest pass),
 *         sell_lanes (1: with autotune 0, lanes per row of the sliced-ELL
 *         level operators; 2 splits each row into its even- and
 *         odd-position entries),
 *         learned_fallback (1: the probe
 *         and the stall guard may replace the learned settings),
 *         record_features (0), thermal (0)
 *   real: tol (1e-6), a_tol (0), threshold (ignored, as in the reference),
 *         convfac_threshold (1e4), stage2_relax_weight (0.7), stage2_omega (0.9),
 *         strong_threshold (0.25, jxf_cpr.c:331), strong_threshold_coarse (-1:
 *         levels >= 1 use strong_threshold; fast path), cheb_lower (0.3),
 *         cheb_upper (1.1): the Chebyshev interval times lambda_max(D^-1 A),
 *         jacobi_mean_row (12: fast path, levels with longer mean rows use
 *         l1-Jacobi instead of multicolour GS)
 */
typedef struct jxcpr_solver jxcpr_solver;

JXCPR_API int jxcpr_solver_create(jxcpr_solver **solver);
JXCPR_API int jxcpr_solver_destroy(jxcpr_solver *solver);
/* Run on the caller's CUDA stream (as void*) instead of a private one; call before setup. */
JXCPR_API int jxcpr_solver_set_stream(jxcpr_solver *solver, void *stream);
JXCPR_API int jxcpr_solver_set_int(jxcpr_solver *solver, const char *key, int value);
JXCPR_API int jxcpr_solver_set_real(jxcpr_solver *solver, const char *key, double value);
/* device != 0: ia/ja/a are device pointers. */
JXCPR_API int jxcpr_solver_setup(jxcpr_solver *solver, int nb, int bs, long long nnzb, const int *ia,
                                 const int *ja, const double *a, int device);
/* b, x: nb*bs entries (host or device); x holds the initial guess on entry. */
JXCPR_API int jxcpr_solver_solve(jxcpr_solver *solver, const double *b, double *x, int device, int *iterations,
                                 double *rel_residual);
/* Residual history of the last solve; returns its length (iterations + 1). */
JXCPR_API int jxcpr_solver_get_norms(jxcpr_solver *solver, double *norms, int capacity);
/* stats[0..3]: setup ms, solve ms, CPR stage-1 setup s, number of AMG levels. */
JXCPR_API int jxcpr_solver_stats(jxcpr_solver *solver, double *stats);
/* Text report of the last setup's phases ("name ms" per line); returns its length. */
JXCPR_API int jxcpr_solver_setup_report(jxcpr_solver *solver, char *buf, int capacity);
/* AMG hierarchy inspection: what = 0 A_l, 1 P_l, 2 R_l = P_l^T; sizes = {rows, cols, nnz}. */
JXCPR_API int jxcpr_solver_num_levels(jxcpr_solver *solver);
JXCPR_API int jxcpr_solver_level_sizes(jxcpr_solver *solver, int level, int what, int *sizes);
JXCPR_API int jxcpr_solver_level_matrix(jxcpr_solver *solver, int level, int what, int *ia, int *ja, double *a);
JXCPR_API int jxcpr_solver_level_cf(jxcpr_solver *solver, int level, int *cf);
/* Decoupled block values after setup (host copy). */
JXCPR_API int jxcpr_solver_decoupled_values(jxcpr_solver *solver, double *a);
/* One CPR application z = M^{-1} r / one AMG V-cycle on the pressure system (xp in/out). */
JXCPR_API int jxcpr_solver_cpr_apply(jxcpr_solver *solver, const double *r, double *z, int device);
JXCPR_API int jxcpr_solver_vcycle(jxcpr_solver *solver, const double *rp, double *xp, int device);
/* One CPR stage-2 sweep on the decoupled system A x = b, x in/out
 * (jxf_ParBSRHGSRelax, jxfpamg-0220/csrc/amg/par_relax_bsr.c:193-573,
 * relax_weight / omega from the stage2_* options). */
JXCPR_API int jxcpr_solver_stage2_sweep(jxcpr_solver *solver, const double *b, double *x, int device);

/* Block ILU(0) stage 2 (stage2_solver_type 5): the factors jxf_BILUSetup builds with type 3
 * (jxf_ILUSetupFGPBILU_v3, jxfpamg-0220/csrc/ilu/par_bilu_setup.c:4996) and one jxf_BILUSolve with
 * tri-solve 14 (par_bilu_solve.c:360, 2893) on the decoupled matrix.  sizes = {L blocks, U blocks};
 * factors: L (strictly lower, A's entry order), U (strictly upper), D^-1 (nb blocks), host arrays;
 * apply: u = BILU^-1 f (u starts at 0). */
JXCPR_API int jxcpr_solver_bilu_sizes(jxcpr_solver *solver, long long *sizes);
JXCPR_API int jxcpr_solver_bilu_factors(jxcpr_solver *solver, double *la, double *ua, double *dinv);
JXCPR_API int jxcpr_solver_bilu_apply(jxcpr_solver *solver, const double *f, double *u, int device);
/* With bilu_exact 1 (exact BILU(0) factors, the fixed point of the sweeps above, and level-scheduled block
 * substitutions in place of the Jacobi iterations; no reference routine computes them in one pass): the
 * level of each block row in the lower DAG (row r after the rows of its L entries) and in the upper DAG
 * (after the rows of its U entries), host arrays of nb ints, and counts = {lower levels, upper levels}. */
JXCPR_API int jxcpr_solver_bilu_levels(jxcpr_solver *solver, int *lev_l, int *lev_u, int *counts);

/* Queues `sweeps` stage-2 sweeps in the fast path's own storage precision (FP64, or FP32 in the mixed
 * path) on internal vectors, asynchronously on the solver's stream (no reference counterpart): the
 * kernel a roofline measurement times with events on that stream. */
JXCPR_API int jxcpr_solver_stage2_native(jxcpr_solver *solver, int sweeps);

/* Host only (no device work): the stage-2 sweep order of the fast path for a block pattern (no
 * reference counterpart; it reorders jxf_ParBSRHGSRelax's natural sweep, jxfpamg-0220/csrc/amg/
 * par_relax_bsr.c:193-573).  Chunks of `chunk` (4, 8 or 16) consecutive block rows, greedily coloured
 * in natural order so that no two coupled chunks share a colour; order = the stored rows colour by
 * colour, chunk by chunk, rows ascending, each chunk padded to `chunk` and each colour to a multiple of
 * 32 entries with -1; segments = the colours' offsets into order (colours + 1 values).  Returns the
 * length of order (filled when capacity suffices; segments when seg_capacity suffices), or minus a
 * status code. */
JXCPR_API int jxcpr_stage2_chunk_order(int nb, const int *ia, const int *ja, int chunk, int *order, int capacity,
                                       int *segments, int seg_capacity);

/* Queues `reps` passes over AMG level `level`'s operator (not the coarsest) in the fast path's storage
 * precision and layout, on the level's own work vectors, asynchronously on the solver's stream (no
 * reference counterpart; the kernel a roofline measurement times with events on that stream):
 * op 0 y = A x, 1 one Chebyshev step y = c z + D^-1 A x, 2 the residual r = f - A u. */
JXCPR_API int jxcpr_solver_level_native(jxcpr_solver *solver, int level, int op, int reps);
/* Queues `reps` times the orthogonalisation kernels of one device-GMRES Arnoldi step with m basis
 * vectors (1 <= m <= k_dim): the first Gram products, the fused first update + second products and
 * the final update into v_m, outside the solve's graph, on the basis the last solve left and the
 * solver's work vector, asynchronously on the solver's stream (no reference counterpart; the CGS2
 * kernels a roofline measurement or a profiler captures).  Needs a solve with graph_gmres 1 first;
 * the next solve starts from scratch. */
JXCPR_API int jxcpr_solver_krylov_native(jxcpr_solver *solver, int m, int reps);
/* Level `level`'s operator values as the fast path stores them (FP64, FP32, or BF16 times its block scale),
 * widened to FP64, in the entry order of jxcpr_solver_level_matrix (host array of its nnz values); no
 * reference counterpart.  Levels without a smoothed operator (the coarsest) return JXCPR_ERROR_ARG. */
JXCPR_API int jxcpr_solver_level_stored_values(jxcpr_solver *solver, int level, double *values);
/* Modelled bytes one preconditioner application of the fast path moves (every smoother pass, residual,
 * transfer, coarse solve and stage-2 sweep at its storage precision); no reference counterpart. */
JXCPR_API int jxcpr_solver_apply_bytes(jxcpr_solver *solver, double *bytes);

/* ---- fast path (smoother_order 1) inspection: no reference counterpart ---------------------
 * level_info: smoother (1 multicolour GS, 2 l1-Jacobi, 3 Chebyshev-3; 0 exact path), storage
 * (0 FP64, 1 FP32, 2 BF16 + a power-of-two FP32 scale per 32 stored values), the strength threshold the
 * level was coarsened with and
 * cheb[6] = {c0, c1, c2, interval low, interval high, lambda_max(D^-1 A)}.  Returns 0 or -1. */
JXCPR_API int jxcpr_solver_level_info(jxcpr_solver *solver, int level, int *smoother, int *storage, double *theta,
                                      double *cheb);
/* Features (16 floats) recorded for `level` by a setup with fast_smoother 2 or record_features 1;
 * returns the count or -1. */
JXCPR_API int jxcpr_solver_level_features(jxcpr_solver *solver, int level, float *features);
/* out[5] = {learned settings in use (1/0), GMRES residual reduction per iteration over an 8-iteration
 * probe (tol 0, b = A 1) with the learned settings, the same with the plain smoothers on the same
 * hierarchy, modelled bytes per GMRES iteration with each}.  The setup keeps the learned settings
 * unless their residual reduction per byte is worse. */
JXCPR_API int jxcpr_solver_learned_status(jxcpr_solver *solver, double *out);
/* Solves since the last setup in which the learned settings stalled (a full restart cycle reduced the
 * residual by less than a factor 10) and the plain preconditioner (default strength thresholds, plain
 * smoothers) was built in their place for the rest of the solve and for later solves.  When the setup probe rejects the learned settings, the
 * same plain preconditioner is built at once (learned_status reports them unused). */
JXCPR_API int jxcpr_solver_learned_fallbacks(jxcpr_solver *solver);

/* ---- batched solves: many set-up solvers, one graph launch; no reference counterpart -------------
 * create: records every solver's whole GMRES solve (option graph_gmres is switched on: flexible GMRES
 * with two-pass classical Gram-Schmidt and true-residual restarts, run on the device with conditional
 * graph nodes) as an independent branch of one CUDA graph.  The solvers must be set up with the fast
 * CPR path (smoother_order 1, stage1_solver_type 1) and stay alive and unchanged while the batch exists.
 * solve: b[k], x[k] (x = initial guess, overwritten) host arrays, or device arrays with device = 1; one
 * graph launch for all systems.  Per system: iterations, FP64 relative residual, latency_ms = its own
 * solve time on the device, finish_ms = completion time since the first system started, status
 * (0, 256 not converged, 512 device error).  Returns 0, or the first error other than 256.
 * last_ms: device time of the last solve (CUDA events around the input copies, the launch and the output
 * copies).  launch: the graph alone on `stream` (NULL:
 * the batch's own), with the inputs already in the solvers' buffers. */
/* batch_setup: jxcpr_solver_setup of system k (nb[k], bs[k], nnzb[k], ia[k], ja[k], a[k]; host arrays, or
 * device arrays with device = 1) for every k on `threads` host threads (<= 0: one per core), each
 * solver on its own stream.  Batches with an exact-order (smoother_order 0) or BILU (stage2_solver_type
 * 5) solver are set up one system after another.  status[k] (may be NULL) gets each setup's code;
 * returns the first failure (its message names the system) or 0. */
JXCPR_API int jxcpr_batch_setup(int nsys, jxcpr_solver *const *solvers, const int *nb, const int *bs,
                                const long long *nnzb, const int *const *ia, const int *const *ja,
                                const double *const *a, int device, int threads, int *status);
typedef struct jxcpr_batch jxcpr_batch;
JXCPR_API int jxcpr_batch_create(jxcpr_batch **batch, int nsys, jxcpr_solver *const *solvers);
JXCPR_API int jxcpr_batch_destroy(jxcpr_batch *batch);
JXCPR_API int jxcpr_batch_solve(jxcpr_batch *batch, const double *const *b, double *const *x, int device,
                                int *iterations, double *rel_residual, double *latency_ms, double *finish_ms,
                                int *status);
JXCPR_API int jxcpr_batch_last_ms(jxcpr_batch *batch, double *ms);
JXCPR_API int jxcpr_batch_launch(jxcpr_batch *batch, void *stream);

/* ---- learned settings: 16 -> 64 (tanh) -> 3 MLP, FP32; no reference counterpart -----------------
 * Weight blob (jxcpr_mlp_num_weights() floats): mu[16], sigma[16], W1[64][16], b1[64], W2[3][64], b2[3];
 * outputs y -> strength threshold 0.1 + 0.8 sigmoid(y0), Chebyshev interval
 * [0.02 + 0.68 sigmoid(y1), 0.8 + 0.7 sigmoid(y2)] x lambda_max(D^-1 A).
 * set/get: the weights the solver's learned mode (fast_smoother 2) uses (host arrays).
 * forward / loss_grad / adam: batch kernels on DEVICE arrays X[B][16], T[B][3], Y[B][3], H[B][64]
 * (H may be NULL); loss_grad needs work[B * 134] floats and writes the mean squared error to *loss
 * (device) and its gradient to grad[num_weights] (mu and sigma get zero gradient). */
JXCPR_API int jxcpr_mlp_num_weights(void);
JXCPR_API int jxcpr_mlp_set_weights(const float *w);
JXCPR_API int jxcpr_mlp_get_weights(float *w);
JXCPR_API int jxcpr_mlp_forward_host(const float *w, const float *x, float *y);
JXCPR_API int jxcpr_mlp_forward(const float *w, const float *X, int B, float *H, float *Y, void *stream);
JXCPR_API int jxcpr_mlp_loss_grad(const float *w, const float *X, const float *T, int B, float *grad, float *loss,
                                  float *work, void *stream);
JXCPR_API int jxcpr_mlp_adam(float *w, const float *grad, float *m, float *v, float lr, float beta1, float beta2,
                             float eps, int step, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* JXCPR_B200_H */
