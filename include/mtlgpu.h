/*
 * mtlgpu -- B200-native (sm_100a) sparse iterative-solve path for MTL4/ITL.
 *
 * C ABI.  Plain pointers and sizes only; no C++ or CUDA types cross this
 * boundary (streams are passed as void*).  Every entry point returns an
 * mtlgpu_status and never throws.  The header-only C++ layer
 * <mtlgpu/mtl.hpp> maps these calls onto the MTL4/ITL names
 * (mtl::compressed2D, itl::pc::ic_0, itl::cg, ...) and re-raises the
 * reference's exception types.
 *
 * Each declaration cites the MTL4 interface it replaces (file:line inside the
 * MTL4 tree).
 *
 * Conventions
 *  - Matrices are CSR with int32 row pointers and column indices, rows sorted
 *    by column, no duplicates (the invariant mtl::compressed2D keeps,
 *    mtl/matrix/compressed2D.hpp:258-653).
 *  - Vector arguments named d_* are DEVICE pointers of the context's device;
 *    arguments named h_* are host pointers.  Device vectors are float64.
 *  - All work of a context is ordered on the context's stream.  Calls on one
 *    handle must be serialised by the caller; different contexts may be used
 *    from different threads.  There is no hidden global state.
 *  - A preconditioner handle keeps a non-owning reference to its matrix
 *    handle: destroy the preconditioner first.
 */
#ifndef MTLGPU_H
#define MTLGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The library is built with hidden visibility; only these entry points are
 * exported. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define MTLGPU_ABI_VERSION 1

/* Status codes.  MTLGPU_MAX_ITER has the value of basic_iteration's
 * "Too many iterations" error code (itl/iteration/basic_iteration.hpp:43-48);
 * the others map onto the reference's exceptions (mtl/utility/exception.hpp:
 * 95-232, itl/utility/exception.hpp:22-31). */
typedef enum {
  MTLGPU_OK = 0,
  MTLGPU_MAX_ITER = 1,          /* iteration limit reached */
  MTLGPU_INVALID_ARG = 2,       /* null handle/pointer, negative size ...   */
  MTLGPU_NOT_SQUARE = 3,        /* mtl::matrix_not_square                    */
  MTLGPU_MISSING_DIAGONAL = 4,  /* mtl::missing_diagonal                     */
  MTLGPU_ZERO_PIVOT = 5,        /* zero/non-positive/non-finite pivot; the
                                   factors are still produced exactly as the
                                   reference computes them (inf/NaN entries) */
  MTLGPU_BREAKDOWN = 6,         /* itl::unexpected_orthogonality             */
  MTLGPU_TIMEOUT = 7,           /* a bounded device wait ran out             */
  MTLGPU_INTERRUPTED = 8,       /* the interrupt flag was raised             */
  MTLGPU_CUDA_ERROR = 9,        /* CUDA runtime error (see mtlgpu_last_error) */
  MTLGPU_NOT_SORTED = 10,       /* CSR rows not sorted / duplicate columns   */
  MTLGPU_INDEX_RANGE = 11,      /* column index out of range                 */
  MTLGPU_OUT_OF_MEMORY = 12,
  MTLGPU_INCOMPATIBLE_SIZE = 13,/* mtl::incompatible_size                    */
  MTLGPU_NOT_SUPPORTED = 14
} mtlgpu_status;

typedef enum { MTLGPU_FP64 = 0, MTLGPU_FP32 = 1 } mtlgpu_precision;

/* itl/pc/identity.hpp:24-71, itl/pc/diagonal.hpp:28-103, itl/pc/ilu_0.hpp:86-92,
 * itl/pc/ic_0.hpp:39-194 */
typedef enum {
  MTLGPU_PC_IDENTITY = 0,
  MTLGPU_PC_DIAGONAL = 1,
  MTLGPU_PC_ILU0 = 2,
  MTLGPU_PC_IC0 = 3
} mtlgpu_pc_kind;

/* itl/krylov/cg.hpp:75-112, bicgstab.hpp:27-78, bicg.hpp:22-63, cgs.hpp:23-65,
 * bicgstab_2.hpp:33-131, bicgstab_ell.hpp:37-132, tfqmr.hpp:26-100,
 * qmr.hpp:24-109, idr_s.hpp:30-105, gmres.hpp:34-135 */
typedef enum {
  MTLGPU_CG = 0,
  MTLGPU_BICGSTAB = 1,
  MTLGPU_BICG = 2,
  MTLGPU_CGS = 3,
  MTLGPU_BICGSTAB_2 = 4,
  MTLGPU_BICGSTAB_ELL = 5,
  MTLGPU_TFQMR = 6,
  MTLGPU_QMR = 7,
  MTLGPU_IDR_S = 8,
  MTLGPU_GMRES = 9
} mtlgpu_method;

/* Solve modes.
 *  FP64         : the reference's arithmetic throughout (iteration counts
 *                 track the reference's).
 *  MIXED_REFINED: inner Krylov solve, factors and SpMV in FP32 (FP32 dots with
 *                 compensated two-sum accumulation); FP64 outer iterative
 *                 refinement r = b - A x, x += d and FP64 stopping norm.
 *                 Requires a preconditioner created with factor precision
 *                 MTLGPU_FP32. */
typedef enum { MTLGPU_SOLVE_FP64 = 0, MTLGPU_SOLVE_MIXED_REFINED = 1 } mtlgpu_solve_mode;

/* Which triangular factor (for sweeps and factor export). */
typedef enum { MTLGPU_LOWER = 0, MTLGPU_UPPER = 1 } mtlgpu_factor;

typedef struct mtlgpu_ctx mtlgpu_ctx;
typedef struct mtlgpu_csr mtlgpu_csr;
typedef struct mtlgpu_pc mtlgpu_pc;

/* Iteration control: the fields of itl::basic_iteration(r0, max_iter, rtol,
 * atol) (itl/iteration/basic_iteration.hpp:31-39): the solve stops when
 * resid <= rtol * norm_r0 or resid <= atol (resid <= atol only when
 * norm_r0 == 0); after max_iter iterations it stops with MTLGPU_MAX_ITER. */
typedef struct {
  int max_iter;
  double rtol;
  double atol;
  double norm_r0;        /* < 0: use two_norm(b), as basic_iteration(b, ...) */
  int mode;              /* mtlgpu_solve_mode */
  /* MIXED_REFINED only: */
  double inner_rtol;     /* largest relative reduction asked of one FP32 inner
                            solve (0: 1e-6); an inner solve never asks for more
                            than half the reduction still needed */
  int inner_max_iter;    /* per inner solve (0: max_iter)  */
  int max_outer;         /* refinement steps (0: 30) */
  /* optional: */
  double* h_resid_history;   /* host array receiving every residual passed to
                                the termination test, or NULL */
  int history_cap;
  const volatile int* h_interrupt; /* host flag (pinned or mapped memory is
                                      best); nonzero stops the solve with
                                      MTLGPU_INTERRUPTED between iterations,
                                      as itl::interruptible_iteration.  The
                                      flag is read between launches of 16
                                      recorded iterations; a solve without
                                      one repeats them in a device-side loop
                                      (one launch, no host round trips) */
} mtlgpu_iter_params;

typedef struct {
  int error;             /* basic_iteration::error_code(): 0 or 1 (MAX_ITER) */
  int status;            /* mtlgpu_status of the whole call */
  int iterations;        /* basic_iteration::iterations() (total inner ones
                            for MIXED_REFINED) */
  int outer_iterations;  /* refinement steps (MIXED_REFINED), else 0 */
  double resid;          /* last residual passed to the termination test */
  double norm_r0;
  double true_resid;     /* ||b - A x||_2 in FP64 at exit */
  int history_len;       /* entries written to h_resid_history */
  long long kernel_launches; /* device kernels this call launched (graph
                                nodes counted per graph launch) */
} mtlgpu_iter_result;

/* ---- context ----------------------------------------------------------- */
mtlgpu_status mtlgpu_ctx_create(int device, mtlgpu_ctx** out);
/* Use an existing stream (a cudaStream_t passed as void*). */
mtlgpu_status mtlgpu_ctx_create_on_stream(int device, void* stream, mtlgpu_ctx** out);
mtlgpu_status mtlgpu_ctx_destroy(mtlgpu_ctx* ctx);
/* Waits for the context's work; reports (and clears) a device-side error of
 * it, e.g. a bounded wait of an asynchronous call that ran out. */
mtlgpu_status mtlgpu_ctx_synchronize(mtlgpu_ctx* ctx);
void* mtlgpu_ctx_stream(mtlgpu_ctx* ctx);
/* Upper bound on polls of one bounded device wait before it gives up with
 * MTLGPU_TIMEOUT (default 1<<26). */
mtlgpu_status mtlgpu_ctx_set_spin_limit(mtlgpu_ctx* ctx, long long polls);
const char* mtlgpu_last_error(mtlgpu_ctx* ctx);
const char* mtlgpu_status_string(int status);
int mtlgpu_abi_version(void);

/* Stream-ordered helpers for callers without a CUDA runtime of their own. */
mtlgpu_status mtlgpu_malloc(mtlgpu_ctx* ctx, size_t bytes, void** d_out);
mtlgpu_status mtlgpu_free(mtlgpu_ctx* ctx, void* d_ptr);
mtlgpu_status mtlgpu_memcpy_h2d(mtlgpu_ctx* ctx, void* d_dst, const void* h_src, size_t bytes);
mtlgpu_status mtlgpu_memcpy_d2h(mtlgpu_ctx* ctx, void* h_dst, const void* d_src, size_t bytes);

/* ---- CSR matrix ---------------------------------------------------------
 * Replaces compressed2D's raw-array constructor
 * (mtl/matrix/compressed2D.hpp:355-364) and address_major/minor/data
 * (610-620).  Arrays are copied in; the caller keeps ownership.  The pattern
 * is validated on the device (sorted rows, indices in range). */
mtlgpu_status mtlgpu_csr_create(mtlgpu_ctx* ctx, int n_rows, int n_cols, int nnz,
                                const int32_t* h_row_ptr, const int32_t* h_col_idx,
                                const double* h_vals, mtlgpu_csr** out);
mtlgpu_status mtlgpu_csr_create_device(mtlgpu_ctx* ctx, int n_rows, int n_cols, int nnz,
                                       const int32_t* d_row_ptr, const int32_t* d_col_idx,
                                       const double* d_vals, mtlgpu_csr** out);
/* New values on the same pattern (h_vals or d_vals, the other NULL). */
mtlgpu_status mtlgpu_csr_set_values(mtlgpu_csr* A, const double* h_vals, const double* d_vals);
mtlgpu_status mtlgpu_csr_destroy(mtlgpu_csr* A);
/* num_rows, num_cols, nnz (compressed2D.hpp:636-640). */
mtlgpu_status mtlgpu_csr_info(const mtlgpu_csr* A, int* n_rows, int* n_cols, int* nnz);
/* Device views of the arrays (read-only for the caller). */
mtlgpu_status mtlgpu_csr_device_arrays(const mtlgpu_csr* A, const int32_t** d_row_ptr,
                                       const int32_t** d_col_idx, const double** d_vals);
/* A^T as a new handle (rows sorted by column), for adjoint solves of an
 * unsymmetric A (trans(A), transposed_sparse_matrix_vector_product_test.cpp:32). */
mtlgpu_status mtlgpu_csr_create_transpose(mtlgpu_csr* A, mtlgpu_csr** out);

/* ---- assembly --------------------------------------------------------------
 * The updaters of mtl::mat::inserter (mtl/operation/update.hpp:26-111): how a
 * value inserted at (r, c) combines with the entry already there, and what a
 * new entry starts as (MINUS starts at -v, the others at v). */
typedef enum {
  MTLGPU_UPDATE_STORE = 0,  /* x = v   (ins[r][c] << v with the default updater, ins[r][c] = v) */
  MTLGPU_UPDATE_PLUS = 1,   /* x += v  (ins[r][c] += v; inserter<M, update_plus<T>>)           */
  MTLGPU_UPDATE_MINUS = 2,  /* x -= v  (inserter<M, update_minus<T>>)                           */
  MTLGPU_UPDATE_TIMES = 3   /* x *= v  (inserter<M, update_times<T>>)                           */
} mtlgpu_updater;

/* Assembly from coordinate triplets on the device: the matrix that
 *   { mtl::mat::inserter<compressed2D<double>, Updater> ins(A);
 *     for k in 0..count-1: ins[d_rows[k]][d_cols[k]] << d_vals[k]; }
 * leaves (mtl/matrix/compressed2D.hpp:662-1151; modify() 947-989).  Triplets
 * apply in order, duplicates fold in that order, and the rows come out sorted
 * without duplicates, bit-identical to the reference's inserter.
 *   base     NULL: A starts empty; else A starts as a copy of base (the
 *            inserter on a matrix that holds entries, stretch() 864-914);
 *            n_rows / n_cols must then equal base's.
 *   d_ops    NULL: `updater` for every triplet; else a device array of count
 *            mtlgpu_updater bytes, one per triplet (ins[r][c] = v is STORE,
 *            ins[r][c] += v is PLUS whatever the inserter's updater).
 * Indices outside the matrix give MTLGPU_INDEX_RANGE (the reference's "Index
 * is out of range!").  All arrays are device arrays; *out is a new handle. */
mtlgpu_status mtlgpu_csr_assemble(mtlgpu_ctx* ctx, const mtlgpu_csr* base, int n_rows, int n_cols,
                                  long long count, const int32_t* d_rows, const int32_t* d_cols,
                                  const double* d_vals, const uint8_t* d_ops, int updater,
                                  mtlgpu_csr** out);
/* laplacian_setup(A, m, n) (mtl/matrix/laplacian_setup.hpp:25-44) built on
 * the device: the m*n x m*n 5-point Laplacian (4 on the diagonal, -1 to each
 * grid neighbour), identical to the reference's. */
mtlgpu_status mtlgpu_csr_laplacian2d(mtlgpu_ctx* ctx, int m, int n, mtlgpu_csr** out);
/* The 3-D 7-point Laplacian on an N^3 grid (row (i*N+j)*N+k, 6 on the
 * diagonal, -1 to each neighbour inside the grid), built on the device; the
 * reference has no 3-D setup, this is the 3-D counterpart of laplacian_setup. */
mtlgpu_status mtlgpu_csr_laplacian3d(mtlgpu_ctx* ctx, int N, mtlgpu_csr** out);
/* Gradient of a loss with respect to A's stored values in the solve
 * x = A^{-1} b, given the adjoint d_lambda (A^T lambda = dL/dx):
 * d_grad[k] = -lambda[i] * x[j] for the k-th stored entry (i, j).  The
 * gradient with respect to b is lambda itself.  No counterpart in the
 * reference (differentiation is not part of MTL4). */
mtlgpu_status mtlgpu_csr_values_grad(mtlgpu_csr* A, const double* d_lambda, const double* d_x,
                                     double* d_grad);

/* Choose the SpMV layout of this matrix by timing the bit-exact candidates
 * on it (CUDA events, 20 products each): SELL-32 where its padding is at most
 * 2 nnz, and the CSR-stream row blocks.  The fastest is kept on the handle;
 * *h_choice (when non-NULL) receives 2 (SELL-32) or 0 (CSR-stream).  No
 * counterpart in the reference (the layout behind mat_vec_mult.hpp:620-689). */
mtlgpu_status mtlgpu_csr_autotune(mtlgpu_csr* A, int* h_choice);

/* y = alpha * A * x + beta * y.  With (alpha, beta) = (1, 0), (1, 1), (-1, 1)
 * this is y = A*x, y += A*x, y -= A*x (mtl/operation/mult.hpp:43-70,
 * mtl/vector/crtp_base_vector.hpp:92-103,192-200,269-277, kernel
 * mtl/operation/mat_vec_mult.hpp:620-689).  beta == 0 never reads y. */
mtlgpu_status mtlgpu_spmv(mtlgpu_csr* A, const double* d_x, double* d_y, double alpha,
                          double beta);
/* y = A * x with float32 vectors and A's values rounded to float: the SpMV
 * the inner solves of MIXED_REFINED run (mat_vec_mult.hpp:620-689 on
 * compressed2D<float>).  Asynchronous on the context's stream. */
mtlgpu_status mtlgpu_spmv_f32(mtlgpu_csr* A, const float* d_x, float* d_y);
/* y = A^T x (trans(A) * x; transposed_sparse_matrix_vector_product_test.cpp:32). */
mtlgpu_status mtlgpu_spmv_transposed(mtlgpu_csr* A, const double* d_x, double* d_y);

/* CG's search-direction step in one kernel: p_out = z + beta * p (p_out = z
 * when d_p is NULL), q = A * p_out, *d_pq = dot(p_out, q) (device double).
 * itl::cg runs it as `p = z + beta * p; q = A * p; alpha = rho / dot(p, q)`
 * (itl/krylov/cg.hpp:99-104, the product and the dot fused as in
 * fused_expr.hpp:57-77); it is the product kernel of the device CG with
 * Jacobi-applied factors.  prec MTLGPU_FP32 (float vectors, A's values
 * rounded to float) or MTLGPU_FP64.  p_out must differ from z and p.  Needs
 * the SELL-32 layout (MTLGPU_NOT_SUPPORTED otherwise).  Asynchronous on the
 * context's stream. */
mtlgpu_status mtlgpu_cg_direction_product(mtlgpu_csr* A, int prec, const void* d_z, double beta,
                                          const void* d_p, void* d_p_out, void* d_q,
                                          double* d_pq);

/* ---- BLAS-1 (mtl/operation/dot.hpp:226-232, two_norm.hpp:33-57,
 *      unary_dot.hpp:29-65, vector/vec_vec_aop_expr.hpp:60-152).
 *      Results are written to host scalars. */
mtlgpu_status mtlgpu_dot(mtlgpu_ctx* ctx, int n, const double* d_x, const double* d_y,
                         double* h_result);
mtlgpu_status mtlgpu_two_norm(mtlgpu_ctx* ctx, int n, const double* d_x, double* h_result);
mtlgpu_status mtlgpu_unary_dot(mtlgpu_ctx* ctx, int n, const double* d_x, double* h_result);
/* Dot product that allocates nothing.  No counterpart in the reference.
 *
 * For callers that cannot allocate device memory -- code whose device heap
 * belongs to a host application or another runtime, or a loop that must not
 * touch the allocator -- and so cannot create the context mtlgpu_dot needs.
 * *d_result (a DEVICE pointer) receives x . y for the n-element device
 * vectors d_x, d_y, computed on `stream` (a cudaStream_t; NULL = the default
 * stream) of the current device with the same kernel and the same bits as
 * mtlgpu_dot.  Nothing is allocated: the reduction scratch is a fixed
 * 32 KiB + 256 B array inside the library that every GPU loading it keeps
 * until the process exits, holding at most 4096 partial sums; a call needing
 * more (never on a B200) returns MTLGPU_INCOMPATIBLE_SIZE.
 * The first call on a device looks up that device's copy of the array (set-up
 * done once per device); make that first call before any stream capture.
 * Later calls check the address again, so the entry point stays valid after
 * a cudaDeviceReset.
 * All calls on a device share the array, so calls whose kernels overlap on
 * the GPU race and give wrong results: order them (one stream, or events). */
mtlgpu_status mtlgpu_dot_noalloc(int n, const double* d_x, const double* d_y, double* d_result,
                                 void* stream);
/* y += alpha * x */
mtlgpu_status mtlgpu_axpy(mtlgpu_ctx* ctx, int n, double alpha, const double* d_x, double* d_y);
/* y = x + beta * y */
mtlgpu_status mtlgpu_xpay(mtlgpu_ctx* ctx, int n, const double* d_x, double beta, double* d_y);

/* ---- preconditioners ----------------------------------------------------
 * Constructors itl::pc::identity<M>(A), diagonal<M>(A) (diagonal.hpp:37),
 * ilu_0<M, V>(A) (ilu_0.hpp:92; factorisation ilu_0.hpp:45-82) and
 * ic_0<M, V>(A) (ic_0.hpp:57; factorisation ic_0.hpp:136-186).  The
 * factorisation always runs in FP64 on the device; factor_prec = MTLGPU_FP32
 * stores the factors in FP32 as ilu_0<M, float> / ic_0<M, float> do
 * (ic_0.hpp:122-130) and enables MIXED_REFINED solves.  The returned status
 * reports MTLGPU_ZERO_PIVOT when a pivot is zero, negative (IC) or not finite;
 * the handle is still created (the reference continues with inf/NaN). */
mtlgpu_status mtlgpu_pc_create(mtlgpu_csr* A, int kind, int factor_prec, mtlgpu_pc** out);
mtlgpu_status mtlgpu_pc_destroy(mtlgpu_pc* P);
/* z = solve(P, r)  (ilu.hpp:84-91, ic_0.hpp:80-87, diagonal.hpp:57-64, pc/solver.hpp:23-52) */
mtlgpu_status mtlgpu_pc_apply(mtlgpu_pc* P, const double* d_r, double* d_z);
/* z = adjoint_solve(P, r) (ilu.hpp:106-115, ic_0.hpp:99-103, diagonal.hpp:75-82) */
mtlgpu_status mtlgpu_pc_adjoint_apply(mtlgpu_pc* P, const double* d_r, double* d_z);
/* z = solve(P, r) with float32 vectors and the FP32 factors (preconditioner
 * created with factor precision MTLGPU_FP32): the apply the inner solves of
 * MIXED_REFINED run, honouring mtlgpu_pc_set_jacobi_sweeps.  Asynchronous on
 * the context's stream; a bounded wait that ran out is reported by the next
 * mtlgpu_ctx_synchronize. */
mtlgpu_status mtlgpu_pc_apply_f32(mtlgpu_pc* P, const float* d_r, float* d_z);
/* One triangular sweep: MTLGPU_LOWER is lower_trisolve v5 (ILU, unit
 * diagonal; lower_trisolve.hpp:173-189) or v6 (IC, inverted diagonal last;
 * 192-209); MTLGPU_UPPER is upper_trisolve v3 (inverted diagonal first;
 * upper_trisolve.hpp:160-176). */
mtlgpu_status mtlgpu_pc_sweep(mtlgpu_pc* P, int which, const double* d_in, double* d_out);
/* The same sweep on float32 vectors with the FP32 factors (preconditioner
 * created with factor precision MTLGPU_FP32): the sweep the inner solves of
 * MIXED_REFINED run. */
mtlgpu_status mtlgpu_pc_sweep_f32(mtlgpu_pc* P, int which, const float* d_in, float* d_out);
/* Apply the factors of an ic_0 / ilu_0 preconditioner with `iters` Jacobi
 * iterations per triangle instead of the exact triangular solves of
 * solve(P, r) (ic_0.hpp:80-87, ilu.hpp:84-91 with lower_trisolve.hpp:173-209
 * and upper_trisolve.hpp:160-176); iters = 0 (the default) restores the exact
 * solves.  For a triangle T = N + D^-1 (D the stored inverted diagonal, I for
 * ILU's unit lower factor) the apply computes w_0 = D v,
 * w_{m+1} = D (v - N w_m), m < iters.  Each iteration is one fully parallel
 * pass over the factor; the exact solve is a chain of one step per level.  For
 * IC(0) the applied operator is P(L)^T P(L), symmetric positive definite, so
 * CG stays valid.  This is an approximation with no counterpart in the
 * reference: iteration counts differ from the reference's; MIXED_REFINED
 * solves still stop on the FP64 true residual.  Affects mtlgpu_pc_apply,
 * mtlgpu_pc_adjoint_apply (IC(0) only; ILU(0) adjoints return
 * MTLGPU_NOT_SUPPORTED) and every solve with P; not mtlgpu_pc_sweep.
 * iters is at most 64. */
mtlgpu_status mtlgpu_pc_set_jacobi_sweeps(mtlgpu_pc* P, int iters);
/* Diagnostics (no counterpart in the reference): how the solves of P apply
 * factor `which` in precision `prec`: *kind = 0 level-ordered sync-free sweep,
 * 1 partitioned sweep (contexts created with MTLGPU_SWEEP=part, where the
 * partition fits shared memory), 2 Jacobi iterations
 * (mtlgpu_pc_set_jacobi_sweeps). */
mtlgpu_status mtlgpu_pc_sweep_kind(const mtlgpu_pc* P, int which, int prec, int* kind);
/* Factor sizes and level counts: nnz of the factor as the reference stores it
 * (L of IC(0) includes the diagonal, L of ILU(0) does not). */
mtlgpu_status mtlgpu_pc_factor_info(const mtlgpu_pc* P, int which, int* nnz, int* n_levels);
/* Export a factor in the reference's CSR layout (get_L()/get_U(),
 * ilu.hpp:118-119, ic_0.hpp:106-107) to host arrays of sizes n+1 / nnz / nnz.
 * Values are exported as double (FP32 factors widened). */
mtlgpu_status mtlgpu_pc_get_factor(const mtlgpu_pc* P, int which, int32_t* h_row_ptr,
                                   int32_t* h_col_idx, double* h_vals);
/* Level of every row in the factor's dependency graph (host array of n):
 * level[r] = 0 for rows without off-diagonal entries, else 1 + max level of
 * the off-diagonal columns (below the diagonal for LOWER, above it for
 * UPPER). */
mtlgpu_status mtlgpu_pc_get_levels(const mtlgpu_pc* P, int which, int32_t* h_levels);

/* ---- solvers ------------------------------------------------------------
 * itl::cg(A, x, b, P, iter) (cg.hpp:41-42,77-78) and
 * itl::bicgstab(A, x, b, P, iter) (bicgstab.hpp:29-30).  x holds the initial
 * guess on entry (warm start) and the solution on exit.  P may be NULL
 * (identity).  The iteration state is returned in *res. */
mtlgpu_status mtlgpu_solve(int method, mtlgpu_csr* A, mtlgpu_pc* P, double* d_x,
                           const double* d_b, const mtlgpu_iter_params* params,
                           mtlgpu_iter_result* res);
/* Same with HOST x and b: copies b and x in, solves, copies x back. */
mtlgpu_status mtlgpu_solve_host(int method, mtlgpu_csr* A, mtlgpu_pc* P, double* h_x,
                                const double* h_b, const mtlgpu_iter_params* params,
                                mtlgpu_iter_result* res);
void mtlgpu_iter_params_default(mtlgpu_iter_params* p);

/* The other ITL Krylov methods with a left preconditioner L and a right
 * preconditioner R (either may be NULL: identity), as the reference calls
 * them:
 *   MTLGPU_BICG          itl::bicg(A, x, b, L, iter)               (R unused)
 *   MTLGPU_CGS           itl::cgs(A, x, b, L, iter)                (R unused)
 *   MTLGPU_BICGSTAB_2    itl::bicgstab_2(A, x, b, L, iter)         (R unused)
 *   MTLGPU_BICGSTAB_ELL  itl::bicgstab_ell(A, x, b, L, R, iter, l) param = l (0: 8; <= 32)
 *   MTLGPU_TFQMR         itl::tfqmr(A, x, b, L, R, iter)
 *   MTLGPU_QMR           itl::qmr(A, x, b, L, R, iter)
 *   MTLGPU_IDR_S         itl::idr_s(A, x, b, L, R, iter, s)        param = s (0: 8; <= 15);
 *                        L and R are ignored, as by the reference; the random
 *                        shadow space is drawn as the reference draws it in a
 *                        fresh process (srand(17 (k + 2)) and rand() for
 *                        vector k), which reseeds the C library's generator
 *   MTLGPU_GMRES         itl::gmres(A, x, b, L, R, iter, restart)  param = restart (0: 8; <= 64)
 * (MTLGPU_CG / MTLGPU_BICGSTAB are mtlgpu_solve.)  FP64 only (params->mode
 * must be MTLGPU_SOLVE_FP64), preconditioners with FP64 factors.  The
 * iteration control and residual history follow basic_iteration as in
 * mtlgpu_solve.  A breakdown branch of the reference (`return
 * iter.fail(code, ...)`, and cgs's zero rho that only records code 2;
 * idr_s's matrix_singular) returns MTLGPU_BREAKDOWN with res->error = the
 * reference's code.  An empty system is MTLGPU_INVALID_ARG for the methods
 * whose reference throws "empty rhs vector". */
mtlgpu_status mtlgpu_solve_krylov(int method, mtlgpu_csr* A, mtlgpu_pc* L, mtlgpu_pc* R,
                                  int param, double* d_x, const double* d_b,
                                  const mtlgpu_iter_params* params, mtlgpu_iter_result* res);

/* Batched PCG: `count` independent systems in one solve.  Each system s is
 * the diagonal block of rows/columns [h_offsets[s], h_offsets[s+1]) of the
 * block-diagonal matrix A (h_offsets: host array of count+1, from 0 to the
 * row count; a row referencing a column outside its block is rejected with
 * MTLGPU_INVALID_ARG) and follows itl::cg(A_s, x_s, b_s, P_s, iter_s)
 * (cg.hpp:75-112) with iter_s = basic_iteration(b_s, max_iter, rtol, atol)
 * (basic_iteration.hpp:31-39): its own scalars, iteration count and stopping
 * test.  P may be NULL (identity) or a diagonal / ic_0 / ilu_0 preconditioner
 * of A (factorising a block-diagonal matrix factorises each block).  Only
 * MTLGPU_CG.  Mode MTLGPU_SOLVE_MIXED_REFINED runs FP32 inner batched PCG
 * (preconditioner created with MTLGPU_FP32) inside FP64 iterative refinement
 * per system, as mtlgpu_solve does for one system; iterations then counts
 * inner iterations and outer_iterations the refinement steps.  h_results
 * (host, count entries) receives each system's iteration state; the call
 * returns MTLGPU_MAX_ITER when any system stopped on max_iter.
 * Execution: with P NULL, diagonal, or ic_0 / ilu_0 applied by Jacobi
 * iterations (mtlgpu_pc_set_jacobi_sweeps), the whole solve -- refinement
 * included -- is ONE persistent kernel launch: thread-block clusters take
 * systems from a work queue (largest first) and each runs its system's
 * iterations, so a converged system releases its cluster at once.  With the
 * exact triangular solves of ic_0 / ilu_0 the iterations of all systems run
 * together, one level-scheduled sweep over the block-diagonal factors. */
mtlgpu_status mtlgpu_solve_batched(int method, mtlgpu_csr* A, mtlgpu_pc* P, int count,
                                   const int32_t* h_offsets, double* d_x, const double* d_b,
                                   const mtlgpu_iter_params* params,
                                   mtlgpu_iter_result* h_results);
/* Tunes mtlgpu_solve_batched for these systems: times short solves (at most
 * 8 iterations, one refinement step; x is not modified) for every candidate
 * of CTAs per large system (4, 8: the thread-block cluster that runs it),
 * lanes per matrix row (4, 8, 16), and the row count below which a system is
 * solved by a single CTA (0, 8192, 32768), and keeps the fastest on A.
 * *h_choice = 1000 * rows + 100 * CTAs + lanes.  Applies to the persistent-launch path
 * (P NULL, diagonal, or factors applied by Jacobi iterations); other
 * preconditioners return MTLGPU_NOT_SUPPORTED.  No counterpart in the
 * reference. */
mtlgpu_status mtlgpu_batched_autotune(mtlgpu_csr* A, mtlgpu_pc* P, int count,
                                      const int32_t* h_offsets, const double* d_x,
                                      const double* d_b, const mtlgpu_iter_params* params,
                                      int* h_choice);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif /* MTLGPU_H */
