/* spaqr_b200.h -- C ABI of the B200 pspaQR factorize-and-solve path.
 *
 * One opaque handle per factorization.  Every call returns an int status
 * (0 = success, negative = error; spq_last_error() gives the message) and no
 * call exits the process.  Host pointers are never retained: matrices and
 * coordinates are copied.  Device memory belongs to the handle.
 *
 * Each entry point names the reference interface it replaces
 * (Abeynaya/pspaQR_public, paths relative to that project).
 *
 * Status codes: -1 bad argument, -2 unsupported input (non-square, levels),
 * -3 coordinates missing or mismatched, -4 call out of order, -5 / -6 symbolic
 * structure inconsistent, -10 CUDA error, -11 device memory exhausted,
 * -12 device-side wait timed out / preconditioner failure, -13 zero or
 * non-finite pivot in the factorization, -14 fixed workspace too small.
 */
#ifndef SPAQR_B200_H
#define SPAQR_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct spq_tree spq_tree;

/* ParTree(int nlevels, int skip)  -- include/ptree.h:135-141 */
int spq_create(int nlevels, int skip, spq_tree** out);
/* ~ParTree()  -- include/ptree.h:160 */
int spq_destroy(spq_tree* t);

/* Tree::set_tol / set_skip / set_scale / set_order / set_hsl / set_square
 * (src/tree.cpp:14-20) and ParTree::set_nthreads / set_verbose / set_ttor_log
 * (src/ptree.cpp:21-23).  order, hsl, nthreads and ttor_log are accepted and
 * recorded like the reference (ParTree never reads order; the rest steer its
 * CPU runtime, which this path replaces).  set_skip follows the driver rule
 * skip = nlevels-1 when tol == 0 (pspaQR.cpp:150) at partition time.
 * The tolerance of the sparsification is read at each factorize; whether it
 * is zero (no sparsification at all) is fixed by partition. */
int spq_set_tol(spq_tree* t, double tol);
int spq_set_skip(spq_tree* t, int skip);
int spq_set_scale(spq_tree* t, int scale);
int spq_set_order(spq_tree* t, float order);
int spq_set_hsl(spq_tree* t, int hsl);
int spq_set_nthreads(spq_tree* t, int n);
int spq_set_verbose(spq_tree* t, int v);
int spq_set_ttor_log(spq_tree* t, int l);
int spq_set_square(spq_tree* t, int s);
/* RRQR pivot tie rule (no reference counterpart; LAPACK's dgeqp3 breaks
 * equal-norm ties by rounding noise): the pivot is the first column whose
 * partial norm is within rtol of the largest.  0 = first maximum. Default 1e-6. */
int spq_set_pivot_rtol(spq_tree* t, double rtol);
/* Tuning of the pivoted QR (no reference counterpart).  Each interface gets
 * the smallest thread-block cluster (1..16 CTAs) whose CTAs handle at most
 * max(elems, level total / (fill * SMs)) elements of the compression matrix
 * per pivot step.  elems >= 1024 (default 65536), 0 < fill <= 64 (default 2). */
int spq_set_rrqr_work(spq_tree* t, double elems, double fill);
/* Mixed precision (no reference counterpart; the reference is FP64 only):
 * bits = 32 stores the factor blocks and applies the preconditioner in float
 * while the SpMV on the original matrix, the GMRES orthogonalisation and the
 * pivoted QR of the compression matrices stay in double; bits = 64 (default)
 * is the plain FP64 method.  Takes effect at the next assemble. */
int spq_set_precision(spq_tree* t, int bits);
/* Tensor cores of the mixed-precision factorization (no reference counterpart).
 * The block-reflector applies of float factors -- the trailing updates (the
 * reference's larfb / tpmqrt, ptree.cpp:216-266), the row scaling and left
 * compression applies and the right compression applies (ptree.cpp:1613-1659,
 * 1860-1903) -- run either as 3xTF32 tcgen05 MMAs with FP32 accumulation or in
 * FP32 on the CUDA cores.  mode 0 = CUDA cores, 1 = tensor cores, 2 (default) =
 * tuned: the first float factorization of a partition runs every apply on the
 * tensor cores, the second on the CUDA cores, and later ones run, per level and
 * kind of apply, the tensor cores where they measured at least 5 % faster, else
 * the CUDA cores (so the first two factorizations of a partition differ from
 * later ones in rounding; the margin keeps near-ties from flipping between
 * runs).  No effect on FP64 factors.  Takes effect at the next factorize.
 * spq_tune_table: per level 9 floats -- for updates, left applies, right
 * applies: tensor-core ms, CUDA-core ms, choice (1 tensor, 0 CUDA, -1 not
 * tuned yet). */
int spq_set_tensor_cores(spq_tree* t, int mode);
int spq_tune_table(spq_tree* t, float* out);
/* Diagnostic of the tensor-core operand layouts (no reference counterpart):
 * runs the two GEMMs of one panel apply once, on host inputs C (m x 64,
 * column-major, ld m, m <= 64), V (m x 32, ld m) and W2 (32 x 64, ld 32), and
 * returns every TMEM lane: out1 (128 x 32, row = lane) holds C^T V (M = 64
 * layout), out2 (128 x 64) holds V W2.  flags (0..15) swap the leading and
 * stride byte offsets of the descriptors (bit 0 / 1: first GEMM A / B, bit 2 /
 * 3: second GEMM A / B). */
int spq_debug_tc_probe(const float* C, const float* V, const float* W2, int m, int flags, float* out1, float* out2);
/* Reuse of descriptor lists across factorizations of one partition (no
 * reference counterpart; the reference rebuilds its task graph every time,
 * ptree.cpp:885-2123).  A level's lists depend only on its cluster sizes and on
 * the allocators' states, so when a later factorize meets the same sizes (the
 * same kept ranks below that level) it reuses them; the merge list is reused
 * when the level's kept ranks are equal too.  on = 1 (default) enables it;
 * spq_plan_hits counts the levels that reused their lists. */
int spq_set_plan_cache(spq_tree* t, int on);
long long spq_plan_hits(spq_tree* t);
/* Failure detection (no reference counterpart; the reference asserts, which
 * its Release build compiles out, or exits).
 * spq_set_spin_limit: clock-cycle budget of each bounded wait of the
 * preconditioner apply's forward sweep (default 2e9); a wait that runs out
 * makes the solve / GMRES call fail with -12.  Takes effect at the next
 * factorize.
 * spq_set_checks: on = 1 checks on the host, before every upload, that the
 * trailing-update, compression and merge descriptors address memory inside
 * the block pool; a bad descriptor fails factorize with -5 before anything is
 * launched for its stage.
 * spq_debug_corrupt_descriptor: fault injection for tests of those checks --
 * the next factorize moves one trailing-update descriptor's block address far
 * outside the pool on the host, and turns the checks on so that it is never
 * launched.
 * factorize also fails with -13 when a QR factorization of the elimination or
 * of the scaling meets a zero or non-finite pivot (a device status word set by
 * the kernels, read after each level), and partition fails with -2 on a
 * non-finite matrix value. */
int spq_set_spin_limit(spq_tree* t, long long cycles);
int spq_set_checks(spq_tree* t, int on);
int spq_debug_corrupt_descriptor(spq_tree* t);
/* Krylov method of spq_gmres / spq_gmres_device (no reference counterpart):
 * 0 = left-preconditioned GMRES of is.cpp:447-527; 1 = flexible
 * right-preconditioned GMRES, whose residual is the true ||b - A x|| however
 * inexact the preconditioner; -1 (default) = flexible exactly when the
 * factors are float (spq_set_precision(t, 32)). */
int spq_set_krylov(spq_tree* t, int method);

/* Tree::set_Xcoo(MatrixXd*) (src/tree.cpp:21): coordinates, dim x n
 * column-major (the reference borrows the pointer; this copies it). */
int spq_set_coords(spq_tree* t, int dim, int n, const double* X);
/* linspace_nd(n, d) + set_Xcoo (util.cpp:901-930, pspaQR.cpp:153-160). */
int spq_set_coords_tensor(spq_tree* t, int n, int d);

/* ParTree::partition(SpMat& A)  -- src/ptree.cpp:495-701.  A in CSC, 0-based,
 * sorted row indices; copied. */
int spq_partition(spq_tree* t, int nrows, int ncols, const int* colptr, const int* rowidx, const double* vals);
/* ParTree::assemble(SpMat& A)  -- src/ptree.cpp:703-864 (uses the matrix given
 * to spq_partition). */
int spq_assemble(spq_tree* t);
/* int ParTree::factorize()  -- src/ptree.cpp:873-2154 */
int spq_factorize(spq_tree* t);

/* void ParTree::solve(VectorXd& x) const  -- src/ptree.cpp:2788-3210.
 * x (host pointer, length n, permuted order) is overwritten by M^{-1} x. */
int spq_solve_inplace(spq_tree* t, double* x);
/* Same, x is a device pointer (stream-ordered on the handle's stream). */
int spq_solve_inplace_device(spq_tree* t, double* x);
/* void ParTree::solve(VectorXd b, VectorXd& x) const  -- src/ptree.cpp:2268-2785
 * (square branch): b and x in the original ordering. */
int spq_solve_global(spq_tree* t, const double* b, double* x);
/* VectorXd ParTree::spmv(VectorXd x) const  -- src/ptree.cpp:3212-3262 (permuted order). */
int spq_spmv(spq_tree* t, const double* x, double* y);
/* Factor backward error (no single reference counterpart; the reference prints
 * the one-shot residual ||A x - b|| / ||b|| of x = M^{-1} b for one b at
 * pspaQR.cpp:207-225): eta[p] = ||A z_p - u_p|| / ||u_p|| with z_p = M^{-1} u_p
 * for nprobe probe vectors, i.e. ||(A P - Q R) z_p|| / ||Q R z_p||, the relative
 * backward error of the factorization QR ~ A P in the direction z_p.  U (host,
 * n x nprobe column-major, permuted order) holds the probes; U = NULL draws
 * u_p ~ N(0,1) from std::mt19937_64(seed + p). */
int spq_factor_backward_error(spq_tree* t, int nprobe, const double* U, unsigned long long seed, double* eta);
/* unsigned long dist_gmres(A, b, M, iter, tol, verb)  -- src/is.cpp:447-527.
 * b (host, permuted order) is overwritten by the solution; iters = the
 * reference's k; relres = true ||b - A x|| / ||b|| (pspaQR.cpp:264-268);
 * hist (may be null) receives the preconditioned residual per step. */
int spq_gmres(spq_tree* t, double* b, int maxit, double tol, int* iters, double* relres, double* hist, int hist_cap);
/* Same with a device-resident right-hand side / solution. */
int spq_gmres_device(spq_tree* t, double* b, int maxit, double tol, int* iters, double* relres, double* hist,
                     int hist_cap);
/* spq_gmres_device without any device allocation.  No counterpart in the
 * reference, which always allocates its Krylov vectors per solve.
 *
 * For callers that cannot allocate device memory at solve time: a service
 * that reserves all device memory when it starts, or a process whose device
 * memory belongs to another framework's pool.  spq_gmres_device grows a cached
 * workspace with cudaMalloc; this entry point uses instead one fixed device
 * array of 6,291,456 doubles (48 MiB) built into the library, which bounds
 * the problem: n * (maxit + 3) + maxit + 1028 <= 6,291,456 (the 64^3 grid,
 * n = 262,144, allows maxit <= 20), and maxit <= 100.  Larger requests fail
 * with an error naming the size; nothing is truncated.  The array lives in a
 * code module of its own, which CUDA 12.2 and later load lazily: the first
 * call on each device loads it, which commits the 48 MiB on that device, and
 * looks up the array's device address.  So make that first call (a small solve
 * will do) before the caller reserves the rest of the device's memory and
 * before any stream capture on the device, or run with
 * CUDA_MODULE_LOADING=EAGER; later calls commit nothing.  The array is shared by every tree
 * on a device: calls that overlap in time (several host threads or streams)
 * race on it and must be serialised.  b, iters and relres as spq_gmres_device;
 * no residual history.  It always runs the reference's left-preconditioned
 * GMRES, which is what spq_gmres_device runs with double factors; with float
 * factors spq_gmres_device defaults to flexible GMRES instead, and the left
 * method's stopping test is then only reliable to about 1e-7. */
int spq_gmres_device_noalloc(spq_tree* t, double* b, int maxit, double tol, int* iters, double* relres);

/* Several right-hand sides at once (no reference counterpart; the reference
 * solves one right-hand side per dist_gmres call, is.cpp:447-527).
 * spq_solve_block_device: X (device, column r at X + r * ldx, permuted order)
 * is overwritten by M^{-1} X; the nrhs sweeps run as parallel branches of one
 * CUDA graph, built on the first call per factorization and nrhs (allocates).
 * spq_gmres_block / spq_gmres_block_device: flexible right-preconditioned GMRES
 * of the nrhs systems in lockstep, one block apply per iteration and one host
 * synchronisation per iteration for all of them; B (host / device, column r at
 * B + r * ldb) is overwritten by the solutions; iters[r] and relres[r] (true
 * ||b_r - A x_r|| / ||b_r||) per right-hand side.  Krylov storage grows to
 * nrhs * n * (2 maxit + 3) doubles: size maxit to the iterations expected. */
int spq_solve_block_device(spq_tree* t, double* X, int nrhs, long long ldx);
int spq_gmres_block(spq_tree* t, double* B, int nrhs, long long ldb, int maxit, double tol, int* iters,
                    double* relres);
int spq_gmres_block_device(spq_tree* t, double* B, int nrhs, long long ldb, int maxit, double tol, int* iters,
                           double* relres);

/* ParTree::distribute_x / extract_x (src/ptree.cpp:3264-3303), single rank:
 * x_local = x[rperm]  and  x[cperm] = x_local. */
int spq_distribute_x(spq_tree* t, const double* x, double* x_local);
int spq_extract_x(spq_tree* t, const double* x_local, double* x);
/* ParTree::nrows_local / ncols_local (src/ptree.cpp:25-26). */
int spq_n(spq_tree* t);

/* Stream the handle launches on (a cudaStream_t passed as void*); null = own stream. */
int spq_set_stream(spq_tree* t, void* stream);

/* Driver preprocessing (pspaQR.cpp:133-146): vals <- A diag(1/||A(:,j)||) * 10. */
int spq_scale_columns(int ncols, const int* colptr, double* vals);
/* util.cpp:992-1001 random(size, seed): mt19937 + uniform_real_distribution(-1,1). */
int spq_random_reference(int n, int seed, double* out);

/* Introspection for parity checks. */
int spq_get_perm(spq_tree* t, int* cperm);
int spq_num_clusters(spq_tree* t);
int spq_num_levels(spq_tree* t);
/* info[16]: lvl, merge_lvl, size (current), rank, parent, cstart, sep, l_lvl,
 * l_sep, r_lvl, r_sep, section, size at creation, sparsified, nchildren, interior */
int spq_cluster_info(spq_tree* t, int order, int* info);
int spq_level_range(spq_tree* t, int lvl, int* first, int* count);
int spq_num_edges(spq_tree* t);
/* Index of the block A(n2 rows, n1 cols) in the symbolic structure, or -1. */
int spq_find_edge(spq_tree* t, int n1, int n2);
/* Final block A(n2 rows, n1 cols): shape[0..2] = rows, cols, ld; out may be null. */
int spq_get_block(spq_tree* t, int n1, int n2, double* out, int* shape);
/* Factors of cluster `order` (which: 0 = block factors T of an interior's
 * diagonal QR (32 x n, one upper triangle per 32 columns), 1 = scaling block
 * factors, 2 = sparsification reflectors V (n x rank), 3 = their block factors);
 * shape[0..2] = rows, cols, ld of the stored factor; out receives rows x cols. */
int spq_get_factor(spq_tree* t, int order, int which, double* out, int* shape);
/* times[0..4] = partition, assemble, factorize, last solve, last gmres (seconds). */
int spq_times(spq_tree* t, double* times);
/* Per level, 8 values (milliseconds): geqrt+tsqrt chains, trailing updates,
 * scaling QR, scaling applies, RRQR, compression applies, merge, level total. */
int spq_level_times(spq_tree* t, float* ms);
/* Per level, 6 values: nominal flops of the first six phases of spq_level_times
 * (chains, updates, scaling QR, scaling applies, pivoted QR or learned ranks,
 * compression applies). */
int spq_level_flops(spq_tree* t, double* flops);
/* Nominal FP64 flops of the last factorization (LAPACK Working Note 41 counts). */
double spq_factor_flops(spq_tree* t);
/* Bytes of compression-matrix data the pivoted QR of the last factorization
 * moves: the transposed gather (read + write), one pass for the column norms
 * and one per pivot step over the columns still active (the algorithmic
 * traffic of its roofline).  No reference counterpart. */
double spq_rrqr_bytes(spq_tree* t);
/* Bytes of device memory held by factor blocks. */
double spq_pool_bytes(spq_tree* t);
/* Kernels this library has launched in the process so far (graph nodes counted
 * per graph launch); no reference counterpart, used to attribute device work. */
long long spq_kernel_launches(void);
/* ---- learned ranks (no reference counterpart) ------------------------------
 * Instead of the column-pivoted QR of every interface's compression matrix C
 * (m x w), a 3-layer MLP (width 64) predicts the kept fraction rank/min(m,w)
 * from 11 features of C.  C is sketched with ell = predicted rank + oversample
 * Rademacher columns, the sketch gets the pivoted QR (stopped at tol / 10),
 * and the kept rank is the smallest k whose largest residual column norm
 * max_j ||c_j - Q_k Q_k^T c_j|| is below tol * max_j ||c_j|| (the pivoted
 * QR's own stop rule, util.cpp:830-851).  Interfaces where no such k exists
 * fall back to the plain pivoted QR.  Features: log2(m+1), log2(w+1),
 * log10(tol), the fractions (of min(m,w)) of columns with norm >= tol, 0.1,
 * 0.5 x the largest, Frobenius norm^2 / (largest^2 min(m,w)), log10 of the
 * 2nd-4th over the 1st diagonal entry of R in a QR of a 4-column sketch, and
 * the level. */
/* nparams = parameters of the MLP, nfeatures = 11 */
int spq_rank_model_size(int* nparams, int* nfeatures);
/* Use the learned ranks with this model (params as spq_mlp_train; mean / std
 * standardise the features); params = NULL restores the plain pivoted QR.
 * Resets the counters of spq_learned_counts. */
int spq_set_rank_model(spq_tree* t, const float* params, const float* mean, const float* stdev, int oversample);
/* Margin (0..1, default 0) added to the predicted kept fraction before the
 * sketch is sized: ell = ceil(min(pred + margin, 1) min(m, w)) + oversample.
 * An upper quantile of the predictor's error on its training pairs keeps the
 * fallback rate near the quantile's complement. */
int spq_set_rank_margin(spq_tree* t, float margin);
/* Tuning of the learned path: the sketch's pivoted QR stops at
 * sketch_tol * tol (default 0.1); smem = 1 holds each CTA's block of the
 * sketch in shared memory when it fits (default 0: reads it from global memory,
 * measured faster on the 64^3 diffusion problem). */
int spq_set_sketch_tuning(spq_tree* t, double sketch_tol, int smem);
/* out[0..2] = interfaces whose learned rank was accepted, interfaces that fell
 * back to the pivoted QR, and the sum of the sketch widths, since the model was set. */
int spq_learned_counts(spq_tree* t, long long* out);
/* Log (features, kept rank, min(m,w), level) of every sparsified interface of
 * later factorizations (the training pairs of the rank model). */
int spq_set_rank_log(spq_tree* t, int on);
int spq_rank_log_count(spq_tree* t);
/* features: count x nfeatures row-major; ranks, kmin, levels: count each */
int spq_rank_log(spq_tree* t, float* features, int* ranks, int* kmin, int* levels);
int spq_rank_log_clear(spq_tree* t);
/* The rank MLP on the GPU, host arrays in and out.  X: n x nfeatures
 * standardised features (row-major), y in [0,1]; loss = mean (sigmoid(z)-y)^2.
 * Layout of params: W1 (64 x 11, row-major), b1 (64), W2 (64 x 64), b2 (64),
 * w3 (64), b3.  Status -10 = CUDA failure (message: spq_mlp_last_error). */
int spq_mlp_loss_grad(const float* params, const float* X, const float* y, int n, float* loss, float* grad);
int spq_mlp_predict(const float* params, const float* X, int n, float* out);
/* Adam (beta 0.9 / 0.999) over `epochs` seeded shuffles in mini-batches;
 * params updated in place; loss_hist (epochs values, may be NULL). */
int spq_mlp_train(float* params, const float* X, const float* y, int n, int epochs, int batch, float lr,
                  unsigned long long seed, float* loss_hist);
const char* spq_mlp_last_error(void);

/* ---- nested-dissection subtree sharding over ranks (one GPU per rank) ----
 * ParTree::get_rank / cluster2rank / edge2rank (ptree.cpp:65-91): the owner of
 * every cluster (cluster_owner, one per cluster order), of every permuted
 * unknown (row_owner, n), and per level the number of transfers between ranks
 * (nexchange, nlevels): the reference's active messages of factors
 * (ptree.cpp:1081-1098, 1419-1441, 1500-1531, 1662-1693), of compression
 * blocks, and of blocks merged into a parent owned elsewhere (send_edge_am,
 * ptree.cpp:2005-2038).  nranks: a power of two <= 2^(nlevels-1).  Any output
 * may be NULL.  Available after spq_partition. */
int spq_shard_plan(spq_tree* t, int nranks, int* cluster_owner, int* row_owner, int* nexchange);
/* The transfers of level lvl, 5 ints each: kind (0 merge of block `id` into
 * parent block `dst`, 1 elimination factors of interior cluster `id`, 2
 * scaling/sparsification factors of interface `id`, 3 compression block `id`
 * to its interface's owner), id, dst (-1 unless kind 0), from rank, to rank. */
int spq_shard_exchange(spq_tree* t, int nranks, int lvl, int* out);
/* Every block of the symbolic structure, 3 ints each: column cluster n1, row
 * cluster n2, level (edge index = position). */
int spq_get_edges(spq_tree* t, int* out);

const char* spq_last_error(spq_tree* t);

#ifdef __cplusplus
}
#endif
#endif
