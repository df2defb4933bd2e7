/*
 * libttb200: B200 (sm_100a) kernels for the tensor-train solve path.
 *
 * C ABI.  Every pointer argument named in a problem struct is a device
 * pointer (float64 unless stated), every size is in elements, every stride
 * is an element stride, and dense arrays are row major unless the field
 * says otherwise.  Problem structs are passed as host arrays; one call
 * processes ``count`` independent problems in grouped launches.  Calls are
 * asynchronous on ``stream`` (a cudaStream_t; NULL is the legacy default
 * stream) unless stated, and return 0 or a cudaError_t code.  No entry point
 * allocates device memory: work areas are passed in, sized by the
 * ttb_*_work_doubles functions.
 *
 * Index conventions follow the reference (ttnumpy 0.3.0,
 * ttnumpy/tensor_train.py:150-244): cores are (r, row_mode, col_mode, r'),
 * environments with an operator are indexed (target, operator, frame),
 * without one (target, frame) (ttnumpy/solvers/common.py:149-217).
 */
#ifndef TTB200_H
#define TTB200_H

#ifdef __cplusplus
extern "C" {
#endif

/* Version of the library ABI (incremented on incompatible changes). */
int ttb_version(void);

/* Number of the library's own kernels launched since load (all devices). */
long long ttb_launch_count(void);

/* Optional timing of the library's launches with CUDA events, for
 * measurement only (no counterpart in the reference).  Bit c of ``mask``
 * enables kernel class c: 0 GEMM, 1 copy, 2 TTM core product, 3 norm,
 * 4 explicit local matrix, 5 QR, 6 SVD, 7 LU solve, 8 truncation rank,
 * 9 MINRES vector kernels, 10 GMRES, 11 batched rounding.  ttb_profile_read
 * synchronises on the recorded events and returns, for one class, the
 * summed device milliseconds, the launch count and the algorithmic FLOPs
 * and bytes the launches were sized for (GEMM: 2mnk per product and the
 * operand/result bytes; MINRES: the vector traffic). */
void ttb_profile_enable(int mask);
int ttb_profile_read(int cls, double* ms, long long* launches, double* flops, double* bytes);
void ttb_profile_reset(void);

/* FP64 fused multiply-add throughput probe for the roofline denominator of
 * the float64 kernels (no counterpart in the reference): ``blocks`` blocks
 * of 256 threads each run 8 independent FMA chains of ``iters`` steps,
 * 2 * 8 * iters * 256 * blocks FLOPs in all.  ``out`` (1 double) is written
 * only to keep the chains live. */
int ttb_fma_peak(double* out, int blocks, int iters, void* stream);

/* ------------------------------------------------------------------------
 * Dense float64 GEMM on strided batched views:
 *   C[b] = alpha * A[b] * B[b] + beta * C[b],  b = 0..batch-1
 * with A[b](i, k) = a[b*a_bs + i*a_rs + k*a_cs] and likewise for B and C
 * (a stride of 0 shares an operand across the batch; beta == 0 never reads
 * C).  This is the contraction engine under every tensordot/einsum of the
 * reference path (e.g. ttnumpy/utils.py:72-83 _multiply_left/_right).
 * --------------------------------------------------------------------- */
typedef struct {
  const double* a;
  const double* b;
  double* c;
  int m, n, k, batch;
  long long a_rs, a_cs, a_bs;
  long long b_rs, b_cs, b_bs;
  long long c_rs, c_cs, c_bs;
  double alpha, beta;
} ttb_gemm_t;
int ttb_gemm(const ttb_gemm_t* problems, int count, void* stream);

/* The same products on the tcgen05 tensor cores in mixed precision (no
 * counterpart in the reference, which multiplies in float64 throughout):
 * every float64 operand element is split into two TF32 parts (hi, lo) and
 * the three leading products hi*hi + hi*lo + lo*hi are accumulated in FP32
 * in tensor memory, then scaled into C in float64.  Relative accuracy about
 * 1e-6 of |A| |B| (22-bit operand parts, FP32 accumulation).  ``status``
 * (device int, may be NULL) is set to 1 if a block gave up waiting on the
 * tensor core (its tile of C is then left unwritten). */
int ttb_gemm_3xtf32(const ttb_gemm_t* problems, int count, int* status, void* stream);

/* ------------------------------------------------------------------------
 * Environment update: one step of the left or right projection recursion,
 * replacing prepare_left_environment / prepare_right_environment
 * (ttnumpy/solvers/common.py:149-188, 191-217).
 *   left  (side 0): env (t, R, f) or (t, f); frame core (f, n, f2);
 *                   op (R, n, m, R2) or NULL; target (t, m, t2);
 *                   out (t2, R2, f2) or (t2, f2)
 *   right (side 1): env (t, R, f) or (t, f); frame core (f2, n, f);
 *                   op (R2, n, m, R) or NULL; target (t2, m, t);
 *                   out (t2, R2, f2) or (t2, f2)
 * Without an operator set R = R2 = 1 and n = m.  ``work`` holds
 * ttb_env_work_doubles() doubles.
 * --------------------------------------------------------------------- */
typedef struct {
  const double* env;
  const double* frame;
  const double* op;
  const double* target;
  double* out;
  double* work;
  int side;
  int f, f2, t, t2, R, R2, n, m;
} ttb_env_t;
long long ttb_env_work_doubles(const ttb_env_t* problem);
int ttb_env_update(const ttb_env_t* problems, int count, void* stream);

/* ------------------------------------------------------------------------
 * One-site local operator applied to ``cols`` vectors (matrix-free matvec /
 * matmat), replacing local_operator_one_site (ttnumpy/solvers/one_site.py:
 * 78-115), and, with a rectangular frame, the A x part of residual_core
 * (ttnumpy/solvers/amen.py:142-158):
 *   y[c, j, k, q] = alpha * sum L[i, a, j] A[a, k, l, b] Rt[p, b, q] x[c, i, l, p]
 *                   + beta * y[c, j, k, q]
 * left (lt, R, lf), op (R, n, m, R2), right (rt, R2, rf), x cols x (lt, m, rt),
 * y cols x (lf, n, rf).  ``work`` holds ttb_local_work_doubles() doubles.
 * --------------------------------------------------------------------- */
typedef struct {
  const double* left;
  const double* op;
  const double* right;
  const double* x;
  double* y;
  double* work;
  int lt, lf, R, R2, n, m, rt, rf, cols;
  double alpha, beta;
} ttb_local_t;
long long ttb_local_work_doubles(const ttb_local_t* problem);
int ttb_local_apply(const ttb_local_t* problems, int count, void* stream);

/* Explicit one-site local matrix, replacing local_explicit_matrix_one_site
 * (ttnumpy/solvers/one_site.py:49-75).  Output is column major with
 * leading dimension rows = lf*n*rf: out[row + col*rows], rows indexed
 * (lf, n, rf), columns (lt, m, rt). */
typedef struct {
  const double* left;
  const double* op;
  const double* right;
  double* out;
  int lt, lf, R, R2, n, m, rt, rf;
} ttb_local_matrix_t;
int ttb_local_matrix(const ttb_local_matrix_t* problems, int count, void* stream);

/* One-site right-hand side / projection of a TT core, replacing
 * local_rhs_one_site (ttnumpy/solvers/one_site.py:27-46):
 *   out[i, j, l] = alpha * sum_{a,c} Lb[a, i] core[a, j, c] Rb[c, l] + beta * out
 * left (a, i), core (a, n, c), right (c, l), out (i, n, l).
 * ``work`` holds a*n*l doubles. */
typedef struct {
  const double* left;
  const double* core;
  const double* right;
  double* out;
  double* work;
  int a, i, n, c, l;
  double alpha, beta;
} ttb_project_t;
int ttb_project(const ttb_project_t* problems, int count, void* stream);

/* ------------------------------------------------------------------------
 * Economic Householder QR of an m x k strided matrix: Q (m x p), R (p x k),
 * p = min(m, k), as scipy.linalg.qr(mode="economic") is used by
 * left_orthonormalize / right_orthonormalize (ttnumpy/utils.py:86-136) and
 * _shift_center_right / _shift_center_left
 * (ttnumpy/solvers/one_site.py:181-209).  q or r may be NULL.  ``work``
 * holds ttb_qr_work_doubles(m, k) doubles (used when the factorisation does
 * not fit in shared memory).
 * --------------------------------------------------------------------- */
typedef struct {
  const double* a;
  long long a_rs, a_cs;
  double* q;
  long long q_rs, q_cs;
  double* r;
  long long r_rs, r_cs;
  double* work;
  int m, k;
} ttb_qr_t;
long long ttb_qr_work_doubles(int m, int k);
int ttb_qr(const ttb_qr_t* problems, int count, void* stream);

/* ttb_qr for callers that cannot allocate device memory (no counterpart in
 * the reference).  Same factorisation and results as ttb_qr; the ``work``
 * field is ignored and the work areas come from one fixed array of
 * TTB_QR_STATIC_DOUBLES doubles (16 MiB) inside the library.  It is meant
 * for a caller whose device memory is all owned by another allocator it may
 * not call into (a serving process that reserved its HBM up front, a
 * host-language binding that holds only its input and output buffers), or
 * that must not take the implicit device synchronisation of
 * cudaMalloc/cudaFree.
 *
 * Limit: the problems of one call that do not fit in shared memory
 * (8 * (m*k + min(m, k)) bytes above 200 KiB) need
 * m*k + min(m, k) doubles each, rounded up to 32, and together at most
 * TTB_QR_STATIC_DOUBLES; a call over the limit launches nothing and
 * returns TTB_ERR_STATIC_SCRATCH.  Nothing in the array must start at zero.
 * The array is shared by every call on a device: calls that overlap in time
 * (on different streams or host threads) race and must be serialised by the
 * caller.  The first call on each device, made with that device current,
 * looks up the array's address (count = 0 is enough); make it before any
 * stream capture begins on that device.  The address is kept for the life
 * of the process: after the caller resets a device (cudaDeviceReset) the
 * kept address is stale, so do not call ttb_qr_static on that device
 * again. */
#define TTB_QR_STATIC_DOUBLES 2097152
#define TTB_ERR_STATIC_SCRATCH (-2)
int ttb_qr_static(const ttb_qr_t* problems, int count, void* stream);

/* ------------------------------------------------------------------------
 * Thin SVD of an m x k strided matrix, a = u diag(s) vh with s descending,
 * p = min(m, k): u (m x p), s (p), vh (p x k).  Householder QR followed by
 * one-sided Jacobi on the triangular factor.  Replaces the LAPACK gesdd /
 * gesvd calls of left_svd / right_svd (ttnumpy/utils.py:336-460) and of
 * _truncate_core_right / _left (ttnumpy/solvers/amen.py:254-260, 301-307).
 * ``status`` (device int, may be NULL) receives the Jacobi sweeps used or
 * -1 when the sweep cap was reached.  ``work`` holds
 * ttb_svd_work_doubles(m, k) doubles.
 * --------------------------------------------------------------------- */
typedef struct {
  const double* a;
  long long a_rs, a_cs;
  double* u;
  long long u_rs, u_cs;
  double* s;
  double* vh;
  long long vh_rs, vh_cs;
  double* work;
  int* status;
  int m, k;
} ttb_svd_t;
long long ttb_svd_work_doubles(int m, int k);
int ttb_svd(const ttb_svd_t* problems, int count, void* stream);

/* ------------------------------------------------------------------------
 * Dense solve a x = b by Gaussian elimination with partial pivoting,
 * replacing scipy.linalg.solve in _solve_local_system
 * (ttnumpy/solvers/common.py:766-774).  a is n x n column major with
 * leading dimension lda and is overwritten; b (n) is overwritten with x.
 * ``info`` (device int, may be NULL) receives 0 or the 1-based index of a
 * zero pivot.  Systems up to n = 161 are factored in shared memory; larger
 * ones by panels of 16 columns with GEMM trailing updates.
 * --------------------------------------------------------------------- */
typedef struct {
  double* a;
  long long lda;
  double* b;
  int* info;
  double* work;  /* ttb_lu_work_doubles(n) doubles, needed only for n > 1600 */
  int n;
} ttb_lu_t;
long long ttb_lu_work_doubles(int n);
int ttb_lu_solve(const ttb_lu_t* problems, int count, void* stream);

/* ------------------------------------------------------------------------
 * Strided 4-D copy dst = alpha * scale[i_axis] * src (src NULL: the value
 * without the src factor; scale NULL: no per-index factor), the core
 * concatenations, zero padding and diagonal scalings of the reference
 * (ttnumpy/tensor_train.py:254-322 add, ttnumpy/solvers/amen.py:275, 322,
 * 325-392 truncation carries and enrichment).
 * --------------------------------------------------------------------- */
typedef struct {
  const double* src;
  double* dst;
  const double* scale;
  int d0, d1, d2, d3;
  long long s0, s1, s2, s3;
  long long t0, t1, t2, t3;
  double alpha;
  int scale_axis;
} ttb_copy_t;
int ttb_copy(const ttb_copy_t* problems, int count, void* stream);

/* ------------------------------------------------------------------------
 * TTM-by-TT core product, replacing the einsum of TensorTrain.dot
 * (ttnumpy/tensor_train.py:483-495):
 *   out[(a, x), i, k, (b, y)] = sum_j op[a, i, j, b] * core[x, j, k, y]
 * op (ra, n, m, ra2), core (rx, m, kk, rx2), out (ra*rx, n, kk, ra2*rx2).
 * --------------------------------------------------------------------- */
typedef struct {
  const double* op;
  const double* core;
  double* out;
  int ra, ra2, n, m, rx, rx2, kk;
} ttb_kron_t;
int ttb_kron(const ttb_kron_t* problems, int count, void* stream);

/* ------------------------------------------------------------------------
 * Element-wise (Hadamard) product core, replacing the einsum of
 * TensorTrain.multiply for two trains (ttnumpy/tensor_train.py:380-395):
 *   out[(a, x), p, (b, y)] = lhs[a, p, b] * rhs[x, p, y]
 * lhs (ra, modes, ra2), rhs (rx, modes, rx2), out (ra*rx, modes, ra2*rx2),
 * with modes = row mode * column mode of the core.
 * --------------------------------------------------------------------- */
typedef struct {
  const double* lhs;
  const double* rhs;
  double* out;
  int ra, ra2, rx, rx2, modes;
} ttb_hadamard_t;
int ttb_hadamard(const ttb_hadamard_t* problems, int count, void* stream);

/* ------------------------------------------------------------------------
 * Sums of squares and norms.  out[p] = sqrt(sum of squares of x[0..n-1])
 * (the np.linalg.norm calls of the reference, e.g.
 * ttnumpy/tensor_train.py:529-538, ttnumpy/solvers/common.py:776,787),
 * with an optional y: out = ||x - y||.  Deterministic order.
 * --------------------------------------------------------------------- */
typedef struct {
  const double* x;
  const double* y;
  double* out;
  long long n;
} ttb_norm_t;
int ttb_norm(const ttb_norm_t* problems, int count, void* stream);

/* ------------------------------------------------------------------------
 * Residual-budget truncation rank, replacing _truncation_rank_by_residual
 * (ttnumpy/solvers/common.py:812-866).  contrib holds ``limit`` rows of
 * length n (row r = A_loc applied to the r-th rank-one term of the SVD);
 * b is b_loc.  rank[0] receives the smallest r + 1 with
 * ||-b + sum_{i<=r} contrib_i|| <= max(damp * exact[0], 0.5 * tol * ||b||),
 * or ``limit`` when no prefix meets it (capped[0] = 1 then if limit < p).
 * s0 is the largest singular value; s0 == 0 gives rank 1.  work holds
 * ttb_rank_work_doubles(n, limit) doubles.
 * --------------------------------------------------------------------- */
typedef struct {
  const double* contrib;
  const double* b;
  const double* exact;
  const double* s;
  int* rank;
  double* work;
  long long n;
  int limit, p;
  double damp, tol;
} ttb_rank_t;
long long ttb_rank_work_doubles(long long n, int limit);
int ttb_rank_residual(const ttb_rank_t* problems, int count, void* stream);

/* Threshold rank rules on descending singular values s (p of them):
 * mode 0: _svd_truncation_rank (ttnumpy/solvers/common.py:872-885),
 *         count of s / s[0] > value, floored at 1, capped at max_rank;
 * mode 1: truncated_bond (ttnumpy/utils.py:22-69), smallest r whose tail
 *         norm is <= value after the eps * p * s[0] noise floor, floored
 *         at 1, capped at max_rank.
 * max_rank <= 0 means no cap. */
typedef struct {
  const double* s;
  int* rank;
  int p, mode, max_rank;
  double value;
} ttb_rank_rule_t;
int ttb_rank_threshold(const ttb_rank_rule_t* problems, int count, void* stream);

/* ------------------------------------------------------------------------
 * MINRES on the one-site local operator, replacing scipy.sparse.linalg
 * .minres as _solve_local_system calls it (ttnumpy/solvers/common.py:
 * 783-784; SciPy 1.18.1, the Paige-Saunders algorithm with SciPy's
 * stopping rules).  Solves op x = b from the initial guess in x (zero
 * when ``warm`` is 0), relative tolerance rtol, at most maxiter
 * iterations (<= 0 means 5 n).  The call blocks the host until every
 * problem stopped: it launches the iterations and reads the stop flags
 * back every few iterations.  istop[0] receives SciPy's istop code and
 * iters[0] the iterations run (both device ints).  work holds
 * ttb_minres_work_doubles() doubles; ``flags`` is a device array of
 * ``count`` ints the solver uses to report which problems stopped.
 * --------------------------------------------------------------------- */
typedef struct {
  ttb_local_t op;  /* x, y, alpha, beta, cols are set by the solver */
  const double* b;
  double* x;
  double* work;
  int* istop;
  int* iters;
  long long n;
  double rtol;
  int maxiter;
  int warm;
} ttb_krylov_t;
long long ttb_minres_work_doubles(const ttb_krylov_t* problem);
int ttb_minres(const ttb_krylov_t* problems, int count, int* flags, void* stream);

/* GMRES(restart) with SciPy 1.18.1's gmres semantics (modified
 * Gram-Schmidt Arnoldi, Givens rotations, atol = rtol * ||b||, restart 20,
 * maxiter outer cycles, <= 0 meaning 10 n), replacing
 * scipy.sparse.linalg.gmres in _solve_local_system
 * (ttnumpy/solvers/common.py:785-786).  Same calling convention as
 * ttb_minres; istop receives 0 on convergence, 1 otherwise. */
long long ttb_gmres_work_doubles(const ttb_krylov_t* problem, int restart);
int ttb_gmres(const ttb_krylov_t* problems, int count, int restart, int* flags, void* stream);

/* ------------------------------------------------------------------------
 * Batched TT rounding of sums of two trains, one thread block per pair,
 * replacing (p + q).truncate(error, max_rank) with method="direct"
 * (ttnumpy/tensor_train.py:254-322, 852-940; ttnumpy/utils.py:86-136,
 * 364-460): left QR sweep of the block-diagonal sum, then right SVD sweep
 * with the tail-norm rule.  All trains of a batch share d and the mode
 * sizes; p, q are packed core by core (core k of pair i at
 * p + i*p_stride + p_off[k]), likewise q.  The rounded cores are written to
 * out (pair i at out + i*out_stride, core k at offset out_off[i*d + k] of
 * that block, computed on the device) and the bonds to bonds[i*(d+1)..].
 * Requires every bond of p + q to be <= 64 and mode * bond <= 256 on both
 * sides of every core (status[i] = -2 otherwise; -1 when a Jacobi sweep
 * cap was reached).  Core k of the result is stored at slot k of
 * TTB_ROUND_SLOT doubles (out_stride >= d * TTB_ROUND_SLOT).  work holds
 * ttb_round_work_doubles() doubles per pair (work_stride).
 * --------------------------------------------------------------------- */
typedef struct {
  const double* p;
  const double* q;
  const long long* p_off;   /* device, d entries */
  const long long* q_off;   /* device, d entries */
  const int* p_bonds;       /* device, d + 1 entries */
  const int* q_bonds;       /* device, d + 1 entries */
  const int* modes;         /* device, d entries */
  long long p_stride, q_stride;
  double* out;
  long long out_stride;
  long long* out_off;       /* device, pairs * d entries (written) */
  int* bonds;               /* device, pairs * (d + 1) entries (written) */
  double* work;
  long long work_stride;
  int* status;              /* device, pairs entries (written) */
  int pairs, d;
  double error;
  int max_rank;
} ttb_round_t;
#define TTB_ROUND_SLOT 16384
long long ttb_round_work_doubles(int d, int max_mode, int max_bond);
int ttb_round_batch(const ttb_round_t* problem, void* stream);


/* ------------------------------------------------------------------------
 * Whole AMEn solves on the device, one thread block per solve, all solves
 * of the launch running concurrently: the amen() sweep
 * (ttnumpy/solvers/amen.py:395-725) with the residual train fit
 * (amen.py:162-224), environments, local solves (direct GEPP for at most
 * direct_solve_size unknowns, else MINRES with the reference's true-residual
 * restarts, common.py:729-809), residual-budget or threshold truncation
 * (common.py:812-929), enrichment and the per-sweep relative residual
 * (common.py:118-146), with every rank decision taken on the device.
 *
 * ``tasks`` is a DEVICE array of ``count`` task structs.  Per task, ``dims``
 * (device ints) holds n[0..d-1], R[0..d], rb[0..d], x0 bonds[0..d] and
 * z0 bonds[0..d]; A, b, x0 and z0 are packed core by core at the given
 * offsets (z0: the random rank-kickrank start, drawn on the host as the
 * reference does).  The solve keeps every core and environment in its
 * ``slab`` (ttb_amen_slab_doubles() doubles); x bonds are capped at
 * ``rmax`` (status -4 when a bond would exceed it).  Results: result[0]
 * status (0 ok, -1 singular local system, -3 slab too small, -4 rank cap,
 * -5 unsupported settings, -6 time limit, -7 tensor-core pipeline),
 * result[1] sweeps run,
 * result[2] stop reason (0 converged, 1 stagnated, 2 max sweeps),
 * result[3] local solves,
 * result[4] inexact local solves, result[5..5+d] x bonds;
 * residuals[0..sweeps-1] and, from residuals[max_sweeps], the largest
 * bond after each sweep; residuals[2 * max_sweeps] receives the FP64 FLOPs
 * of the block's dense products (2 m n k each; factorisations not
 * counted), residuals[2 * max_sweeps + 1] the operator applications and
 * residuals[2 * max_sweeps + 2 .. + 8] SM cycles spent in environment
 * updates, local solves, residual cores, truncation with enrichment, dense
 * products (a part of the other phases), residual checks and set-up,
 * residuals[2 * max_sweeps + 10] and [+ 11] the device's global timer (ns)
 * when the block started and finished the solve (``residuals`` holds
 * 2 * max_sweeps + 16 doubles); x core k at
 * slab + x_offsets[k].  Blocks start in task order, so listing the longest
 * solves first shortens the launch.  local_rtol > 0
 * selects MINRES for local systems above direct_solve_size unknowns (at
 * most min(5 N, 2000) iterations per call, SciPy's cap being 5 N), or
 * GMRES with local_gmres; local_rtol <= 0 refuses them (status -5).
 * --------------------------------------------------------------------- */
typedef struct {
  const double* A;
  const long long* A_off;
  const double* b;
  const long long* b_off;
  const double* x0;
  const long long* x0_off;
  const double* z0;
  const long long* z0_off;
  const int* dims;
  double* slab;
  long long slab_doubles;
  double* residuals;
  int* result;
  long long* x_offsets;
  int d, kickrank, max_rank, max_sweeps, direct_solve_size, track_residual, residual_mode,
      stagnation_on, x0_orth_center, b_orth_center;
  double residual_tol, error_threshold, residual_damp, stagnation_factor, local_rtol,
      truncation_tol;
  int debug; /* 1: also apply the operator to every rank-one term in full and
                record the worst relative gap in residuals[2*max_sweeps + 9];
                repeat every two-level R-only QR with the one-level one and
                record the worst relative gap of R in [2*max_sweeps + 12],
                the number of such QRs in [+ 13] */
  long long time_limit_ns; /* > 0: the solve stops with status -6 after the
                              first local step that ends this many ns of the
                              device timer after the block started (the
                              per-solve time limit of the reference's
                              benchmark runner, benchmarks/poisson.py:95-143);
                              sweeps, residuals and bonds so far are kept */
  int precision;           /* 0: float64 throughout; 1: mixed: iterative local
                              solves by float64 iterative refinement around
                              inner MINRES solves whose operator products run
                              on the tensor cores in 3xTF32 (residuals
                              [2*max_sweeps + 14] receives their FLOPs, [+ 15]
                              the refinement steps; status -7 if a tensor-core
                              wait gave up) */
  int local_gmres;         /* 1: iterative local solves by restarted GMRES
                              (symmetric=False; SciPy's gmres, restart 20, at
                              most 100 restart cycles per call), 0: MINRES */
} ttb_amen_task_t;
long long ttb_amen_slab_doubles(int d, const int* host_dims, int kickrank, int rmax,
                                int direct_solve_size);
int ttb_amen_persistent(const ttb_amen_task_t* tasks, int count, int rmax, void* stream);

/* The same solves with a cluster of ``cluster`` (2..8) thread blocks per
 * task (no counterpart in the reference, which solves on one host thread):
 * block 0 runs the solve and the other blocks of its cluster compute shares
 * of its larger dense products and sparse operator-core products, each
 * output tile or row exactly as a lone block computes it, so the results are
 * bitwise those of ttb_amen_persistent; the wall time of a large solve
 * drops, at the price of blocks that idle through its other steps.
 * cluster <= 1 is ttb_amen_persistent. */
int ttb_amen_persistent_cluster(const ttb_amen_task_t* tasks, int count, int rmax, int cluster,
                                void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TTB200_H */
