// The other ITL Krylov methods on the device: bicg, cgs, bicgstab_2,
// bicgstab_ell, tfqmr, qmr, idr_s and gmres (itl/krylov/*.hpp), with a left
// and a right preconditioner and basic_iteration control
// (itl/iteration/basic_iteration.hpp:51-93, fail() 145-150).
//
// One engine serves all eight.  Every scalar of a method (rho, alpha, the
// Hessenberg matrix of gmres, the small LU systems of idr_s, the
// orthogonalisation factors of bicgstab_ell) lives in device memory; the
// vector work is done by three generic kernels whose coefficients are read
// from device memory at run time:
//   xdots_kernel   up to kMaxDots inner products in one pass over the
//                  vectors, a deterministic two-level reduction (fixed
//                  block partials, summed in a fixed order by the last
//                  block), results written to device addresses;
//   xlin_kernel    out = sum_k c_k v_k for up to kMaxTerms vectors, c_k =
//                  mul_k * (*coef_k); out may be one of the v_k (elementwise,
//                  so every v_k is read before out is written);
//   xscalar_kernel one thread running one step of a method's scalar
//                  recurrence, its termination test and breakdown checks.
// SpMV, A^T x (a transposed handle) and the preconditioner applies
// (solve / adjoint_solve) are the library's own kernels.  Each kernel returns
// at once when the state's halt word is set (the solve has finished, or a
// gmres step lies beyond this cycle's last), so an iteration can be captured
// in a CUDA graph and replayed without host round trips; the host looks at
// the state between graph launches only.  Per method the host records the
// kernels of one iteration (one restart cycle for gmres) in the order the
// reference's loop computes them; the recipes below cite the loop lines.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <vector>

#include "device.cuh"
#include "internal.h"

namespace mtlgpu {

using namespace dev;

// The device error word (a bounded wait that ran out), read without clearing it.
static mtlgpu_status read_error_word(Ctx* ctx, int* err) {
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(err, ctx->d_error, sizeof(int), cudaMemcpyDeviceToHost,
                                       ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return MTLGPU_OK;
}

namespace {

constexpr int kBlock = 256;
constexpr int kMaxDots = 8;
constexpr int kMaxTerms = 16;
constexpr int kSlots = 64;

struct XState {
  int done;       // the solve has finished (converged, max_iter or breakdown)
  int halt;       // nonzero: every vector kernel returns at once
  int error;      // basic_iteration::error (0, 1 too many iterations, or fail(code))
  int breakdown;  // a breakdown branch (iter.fail / matrix_singular) was taken
  int iter, max_iter, hist_len, hist_cap;
  int kmax, singular, pad0, pad1;
  double tol, atol, norm_r0, resid;
  double* history;
  double s[kSlots];
};

struct Term {
  const double* v;
  const double* coef;  // nullptr: coefficient = mul
  double mul;
};
struct LinArgs {
  double* out;
  int nt;
  Term t[kMaxTerms];
};
struct DotArgs {
  int nd;
  const double* x[kMaxDots];
  const double* y[kMaxDots];
  double* out[kMaxDots];
};

// basic_iteration::finished(r): converged() (basic_iteration.hpp:85-93), then
// check_max() (43-48).  One thread.
__device__ bool x_finished(XState* st, double r) {
  if (st->history && st->hist_len < st->hist_cap) st->history[st->hist_len] = r;
  st->hist_len++;
  st->resid = r;
  const bool conv = st->norm_r0 == 0.0 ? (r <= st->atol) : (r <= st->tol || r <= st->atol);
  if (conv) return true;
  if (st->iter >= st->max_iter) {
    st->error = 1;
    return true;
  }
  return false;
}
__device__ void x_stop(XState* st) { st->done = 1, st->halt = 1; }
// return iter.fail(code, ...): the solver returns with error code `code`
__device__ void x_fail(XState* st, int code) {
  st->error = code;
  st->breakdown = 1;
  x_stop(st);
}

__global__ void __launch_bounds__(kBlock) xlin_kernel(long long n, LinArgs a, const XState* st) {
  if (st->halt) return;
  double c[kMaxTerms];
#pragma unroll
  for (int k = 0; k < kMaxTerms; k++)
    c[k] = k < a.nt ? (a.t[k].coef ? a.t[k].mul * *a.t[k].coef : a.t[k].mul) : 0.0;
  for (long long i = gtid(); i < n; i += gstride()) {
    double acc = c[0] * a.t[0].v[i];
#pragma unroll
    for (int k = 1; k < kMaxTerms; k++)
      if (k < a.nt) acc += c[k] * a.t[k].v[i];
    a.out[i] = acc;
  }
}

__global__ void __launch_bounds__(kBlock)
    xdots_kernel(long long n, DotArgs a, const XState* st, Sum<kMaxDots>* partials,
                 unsigned* counter) {
  if (st->halt) return;  // every block sees the same word: none arrives at the counter
  Sum<kMaxDots> acc = Sum<kMaxDots>::zero();
  for (long long i = gtid(); i < n; i += gstride()) {
#pragma unroll
    for (int k = 0; k < kMaxDots; k++)
      if (k < a.nd) acc.add_prod(k, a.x[k][i], a.y[k][i]);
  }
  acc = block_reduce(acc);
  if (publish_partial(acc, partials, blockIdx.x, counter, gridDim.x)) {
    const Sum<kMaxDots> tot = reduce_partials(partials, gridDim.x);
    if (threadIdx.x == 0)
      for (int k = 0; k < a.nd; k++) *a.out[k] = tot.value(k);
  }
}

// ---- small dense algebra (one thread) --------------------------------------
// lu_solve (mtl/operation/lu.hpp:58-84 with partial pivoting, first largest
// magnitude; lu_apply 113-119): x = A^{-1} b for the m x m matrix at A (row
// stride lda), work = m*m + m doubles.  Returns false for a zero pivot
// before the last row (matrix_singular).
__device__ bool dense_lu_solve(const double* A, int lda, const double* b, int m, double* x,
                               double* work) {
  double* LU = work;
  double* y = work + m * m;
  int perm[64];
  for (int r = 0; r < m; r++) {
    perm[r] = r;
    for (int c = 0; c < m; c++) LU[r * m + c] = A[r * lda + c];
  }
  for (int i = 0; i + 1 < m; i++) {
    int rmax = i;
    double best = fabs(LU[i * m + i]);
    for (int r = i + 1; r < m; r++)
      if (fabs(LU[r * m + i]) > best) best = fabs(LU[r * m + i]), rmax = r;
    if (rmax != i) {
      for (int c = 0; c < m; c++) {
        const double t = LU[i * m + c];
        LU[i * m + c] = LU[rmax * m + c];
        LU[rmax * m + c] = t;
      }
      const int t = perm[i];
      perm[i] = perm[rmax];
      perm[rmax] = t;
    }
    if (fabs(LU[i * m + i]) <= 0.0) return false;
    for (int r = i + 1; r < m; r++) LU[r * m + i] /= LU[i * m + i];
    for (int r = i + 1; r < m; r++)
      for (int c = i + 1; c < m; c++) LU[r * m + c] -= LU[r * m + i] * LU[i * m + c];
  }
  for (int r = 0; r < m; r++) {  // unit lower
    double t = b[perm[r]];
    for (int c = 0; c < r; c++) t -= LU[r * m + c] * y[c];
    y[r] = t;
  }
  for (int r = m - 1; r >= 0; r--) {  // upper
    double t = y[r];
    for (int c = r + 1; c < m; c++) t -= LU[r * m + c] * x[c];
    x[r] = t / LU[r * m + r];
  }
  return true;
}

// ---------------------------------------------------------------------------
// Dense layouts (offsets in doubles) shared by the host recipes and the
// scalar steps.
//  bicgstab_ell (l1 = l + 1): tau[l1*l1], gamma[l1], gamma_a[l1],
//    gamma_aa[l1], -gamma_a[l1] and -gamma[l1], dot(r_hat[j], r_hat[0])[l1]
//  idr_s (s): M[s*s], m[s], c[s], -c[s], dm[s], LU work[s*s + s]
//  gmres (m = restart): H[(m+1)*m], g, c, s[m+1 each], y[m], hr[m+1],
//    spare[m+1], LU work[m*m + m]
__host__ __device__ inline int ell_gamma(int l1) { return l1 * l1; }
__host__ __device__ inline int ell_gamma_a(int l1) { return l1 * l1 + l1; }
__host__ __device__ inline int ell_gamma_aa(int l1) { return l1 * l1 + 2 * l1; }
__host__ __device__ inline int ell_neg(int l1) { return l1 * l1 + 3 * l1; }
__host__ __device__ inline int ell_dga(int l1) { return l1 * l1 + 5 * l1; }
__host__ __device__ inline int idr_m(int P) { return P * P; }
__host__ __device__ inline int idr_c(int P) { return P * P + P; }
__host__ __device__ inline int idr_nc(int P) { return P * P + 2 * P; }
__host__ __device__ inline int idr_dm(int P) { return P * P + 3 * P; }
__host__ __device__ inline int gm_g(int m) { return (m + 1) * m; }
__host__ __device__ inline int gm_y(int m) { return (m + 1) * m + 3 * (m + 1); }
__host__ __device__ inline int gm_hr(int m) { return (m + 1) * m + 3 * (m + 1) + m; }
inline int dense_len(int method, int P) {
  switch (method) {
    case MTLGPU_BICGSTAB_2:
    case MTLGPU_BICGSTAB_ELL: return (P + 1) * (P + 1) + 6 * (P + 1) + 8;
    case MTLGPU_IDR_S: return 2 * P * P + 5 * P + 8;
    case MTLGPU_GMRES: return 2 * (P + 1) * (P + 1) + 8 * (P + 1) + 8;
    default: return 8;
  }
}

// ---------------------------------------------------------------------------
// Scalar slots (st->s) and dense layouts of the methods.
enum Slot {
  S_RR = 0,      // a squared norm or a dot product just computed
  S_RR2,
  S_RHO1, S_RHO2, S_RHO0, S_ALPHA, S_NALPHA, S_BETA, S_NBETA, S_BETA2, S_OMEGA, S_NOMEGA,
  S_GAMMA, S_SIGMA, S_THETA, S_ETA, S_TAU, S_RHO, S_C, S_DCOEF, S_XI, S_DELTA, S_EP,
  S_GAMMA1, S_THETA1, S_ETA_P, S_INV_RHO, S_INV_XI, S_QCOEF, S_PCOEF, S_DMUL, S_ONE, S_TV,
  S_TT, S_INV, S_NINV,
  S_COUNT
};
static_assert(S_COUNT <= kSlots, "scalar slots");

// Steps of the scalar programs.
enum Step {
  // shared
  X_CHECK_RR = 1,   // finished(sqrt(s[RR]))
  X_INC,            // ++iter
  // bicg (itl/krylov/bicg.hpp:22-63)
  BICG_RHO, BICG_ALPHA, BICG_END,
  // cgs (itl/krylov/cgs.hpp:23-65)
  CGS_RHO, CGS_ALPHA, CGS_END,
  // bicgstab_ell / bicgstab_2 (bicgstab_ell.hpp:37-132, bicgstab_2.hpp:33-131)
  ELL_INIT_NORM, ELL_BEGIN, ELL_BETA, ELL_ALPHA, ELL_CHECK, ELL_TAU_T, ELL_TAU_D, ELL_GAMMA,
  // tfqmr (itl/krylov/tfqmr.hpp:26-100)
  TFQMR_INIT, TFQMR_SIGMA, TFQMR_THETA, TFQMR_RHO,
  // qmr (itl/krylov/qmr.hpp:24-109)
  QMR_INIT, QMR_BEGIN, QMR_DELTA, QMR_EP, QMR_NORMS, QMR_END,
  // idr_s (itl/krylov/idr_s.hpp:30-105)
  IDR_ORTH_DOT, IDR_ORTH_NORM, IDR_OMEGA0, IDR_STEP, IDR_M_INIT, IDR_LU, IDR_M,
  // gmres (itl/krylov/gmres.hpp:34-135)
  GM_START, GM_STEP_BEGIN, GM_NORM1, GM_STEP_END, GM_SOLVE, GM_END
};

struct ScalarArgs {
  int step;
  int a, b;     // step operands (loop indices)
  int param;    // l, s or restart
  long long n;
  double* dense;
};

__device__ void run_step(XState* st, const ScalarArgs& x) {
  double* s = st->s;
  double* D = x.dense;
  const int P = x.param;
  switch (x.step) {
    case X_CHECK_RR:
      if (st->done) return;
      if (x_finished(st, sqrt(fabs(s[S_RR])))) x_stop(st);
      return;
    case X_INC:
      if (!st->done) st->iter++;
      return;

    // ---- bicg -----------------------------------------------------------
    case BICG_RHO:  // rho_1 = dot(z~, z); breakdown; beta (bicg.hpp:39-50)
      if (st->done) return;
      if (s[S_RHO1] == 0.0) return x_fail(st, 2);
      s[S_BETA] = st->iter <= 1 ? 0.0 : s[S_RHO1] / s[S_RHO2];
      return;
    case BICG_ALPHA:  // alpha = rho_1 / dot(p~, q) (bicg.hpp:54)
      if (st->done) return;
      s[S_ALPHA] = s[S_RHO1] / s[S_RR2];
      s[S_NALPHA] = -s[S_ALPHA];
      return;
    case BICG_END:  // rho_2 = rho_1; while (!finished(r)) (bicg.hpp:31,60)
      if (st->done) return;
      s[S_RHO2] = s[S_RHO1];
      if (x_finished(st, sqrt(fabs(s[S_RR])))) x_stop(st);
      return;

    // ---- cgs --------------------------------------------------------------
    case CGS_RHO:  // cgs.hpp:35-46; a zero rho_1 records error 2 and carries on
      if (st->done) return;
      if (s[S_RHO1] == 0.0) st->error = 2, st->breakdown = 1;
      s[S_BETA] = st->iter <= 1 ? 0.0 : s[S_RHO1] / s[S_RHO2];
      s[S_BETA2] = s[S_BETA] * s[S_BETA];
      return;
    case CGS_ALPHA:  // alpha = rho_1 / dot(r~, vhat) (cgs.hpp:49)
      if (st->done) return;
      s[S_ALPHA] = s[S_RHO1] / s[S_RR2];
      s[S_NALPHA] = -s[S_ALPHA];
      return;
    case CGS_END:
      if (st->done) return;
      s[S_RHO2] = s[S_RHO1];
      if (x_finished(st, sqrt(fabs(s[S_RR])))) x_stop(st);
      return;

    // ---- bicgstab_ell -------------------------------------------------------
    // dense: tau[(l+1)^2], gamma[l+1], gamma_a[l+1], gamma_aa[l+1], then
    // per-coefficient negations used by the vector updates
    case ELL_INIT_NORM:  // r0_tilde = r_hat[0] / two_norm(r_hat[0]) (bicgstab_ell.hpp:57)
      s[S_INV] = 1.0 / sqrt(fabs(s[S_RR]));
      s[S_RHO0] = 1.0, s[S_ALPHA] = 0.0, s[S_OMEGA] = 1.0;
      return;
    case ELL_BEGIN:  // ++iter; rho_0 = -omega * rho_0 (66-67)
      if (st->done) return;
      st->iter++;
      s[S_RHO0] = -s[S_OMEGA] * s[S_RHO0];
      return;
    case ELL_BETA:  // rho_1 = dot(r0~, r_hat[j]); beta = alpha rho_1 / rho_0 (70-71)
      if (st->done) return;
      s[S_BETA] = s[S_ALPHA] * s[S_RHO1] / s[S_RHO0];
      s[S_NBETA] = -s[S_BETA];
      s[S_RHO0] = s[S_RHO1];
      return;
    case ELL_ALPHA:  // Gamma = dot(r0~, u_hat[j+1]); alpha = rho_0 / Gamma (78-79)
      if (st->done) return;
      s[S_ALPHA] = s[S_RHO0] / s[S_GAMMA];
      s[S_NALPHA] = -s[S_ALPHA];
      return;
    case ELL_CHECK:  // if (iter.finished(r_hat[j])) ... return (84-88)
      if (st->done) return;
      if (x_finished(st, sqrt(fabs(s[S_RR])))) x_stop(st);
      return;
    case ELL_TAU_T: {  // t = dot(tail_i, tail_j) / tau[i][i] (orth.hpp:80-84)
      if (st->done) return;
      const int l1 = P + 1, i = x.a, j = x.b;  // tail indices; tau index + 1
      double* tau = D;
      const double t = s[S_RR] / tau[(i + 1) * l1 + (i + 1)];
      tau[(i + 1) * l1 + (j + 1)] = t;
      s[S_NINV] = -t;
      return;
    }
    case ELL_TAU_D: {  // tau[j][j] = dot(tail_j, tail_j) (orth.hpp:71,86)
      if (st->done) return;
      const int l1 = P + 1, j = x.a;
      D[(j + 1) * l1 + (j + 1)] = s[S_RR];
      return;
    }
    case ELL_GAMMA: {  // bicgstab_ell.hpp:97-123: gammas; omega; breakdown #2
      if (st->done) return;
      const int l = P, l1 = P + 1;
      double* tau = D;
      double* gamma = D + ell_gamma(l1);
      double* gamma_a = D + ell_gamma_a(l1);
      double* gamma_aa = D + ell_gamma_aa(l1);
      double* neg = D + ell_neg(l1);  // -gamma_a[j], -gamma[j]
      const double* dga = D + ell_dga(l1);
      for (int j = 1; j <= l; j++) gamma_a[j] = dga[j] / tau[j * l1 + j];
      gamma[l] = gamma_a[l];
      s[S_OMEGA] = gamma[l];
      if (s[S_OMEGA] == 0.0) return x_fail(st, 3);
      for (int j = l - 1; j > 0; --j) {
        double sum = 0.0;
        for (int i = j + 1; i <= l; ++i) sum += tau[j * l1 + i] * gamma[i];
        gamma[j] = gamma_a[j] - sum;
      }
      // gamma_aa[1..l-1] = strict_upper(tau[1..l-1][1..l-1]) * gamma[2..l] + gamma[2..l]
      for (int a = 0; a < l - 1; a++) {
        double sum = 0.0;
        for (int b = a + 1; b < l - 1; b++) sum += tau[(1 + a) * l1 + (1 + b)] * gamma[2 + b];
        gamma_aa[1 + a] = sum + gamma[2 + a];
      }
      for (int j = 0; j <= l; j++) neg[j] = -gamma_a[j], neg[l1 + j] = -gamma[j];
      return;
    }

    // ---- tfqmr -----------------------------------------------------------
    case TFQMR_INIT:  // tau = two_norm(r); rho = tau * tau (tfqmr.hpp:43-44)
      s[S_TAU] = sqrt(fabs(s[S_RR]));
      s[S_RHO] = s[S_TAU] * s[S_TAU];
      s[S_THETA] = 0.0, s[S_ETA] = 0.0;
      return;
    case TFQMR_SIGMA:  // while (!finished(tau)) { ++iter; sigma; alpha (47-52)
      if (st->done) return;
      if (x_finished(st, s[S_TAU])) return x_stop(st);
      st->iter++;
      if (s[S_SIGMA] == 0.0) return x_fail(st, 1);
      s[S_ALPHA] = s[S_RHO] / s[S_SIGMA];
      s[S_NALPHA] = -s[S_ALPHA];
      s[S_DCOEF] = s[S_THETA] * s[S_THETA] * s[S_ETA] / s[S_ALPHA];
      return;
    case TFQMR_THETA:  // theta, c, tau, eta (68-71); coefficient for the next d
      if (st->done) return;
      s[S_THETA] = sqrt(fabs(s[S_RR])) / s[S_TAU];
      s[S_C] = 1.0 / sqrt(1.0 + s[S_THETA] * s[S_THETA]);
      s[S_TAU] *= s[S_THETA] * s[S_C];
      s[S_ETA] = s[S_C] * s[S_C] * s[S_ALPHA];
      s[S_DCOEF] = s[S_THETA] * s[S_THETA] * s[S_ETA] / s[S_ALPHA];
      return;
    case TFQMR_RHO:  // rho == 0 breakdown; rhon; beta (74-79)
      if (st->done) return;
      if (s[S_RHO] == 0.0) return x_fail(st, 1);
      s[S_BETA] = s[S_RR2] / s[S_RHO];
      s[S_RHO] = s[S_RR2];
      s[S_BETA2] = s[S_BETA] * s[S_BETA];
      return;

    // ---- qmr ---------------------------------------------------------------
    case QMR_INIT:  // rho = two_norm(y), xi = two_norm(z); gamma, eta, ep, theta (34,42)
      s[S_RHO] = sqrt(fabs(s[S_RR]));
      s[S_XI] = sqrt(fabs(s[S_RR2]));
      s[S_GAMMA] = 1.0, s[S_ETA] = -1.0, s[S_EP] = 1.0, s[S_THETA] = 0.0;
      return;
    case QMR_BEGIN:  // while (!finished(rho)) { ++iter; checks; 1/rho, 1/xi (43-53)
      if (st->done) return;
      if (x_finished(st, s[S_RHO])) return x_stop(st);
      st->iter++;
      if (s[S_RHO] == 0.0) return x_fail(st, 1);
      if (s[S_XI] == 0.0) return x_fail(st, 2);
      s[S_INV_RHO] = 1.0 / s[S_RHO];
      s[S_INV_XI] = 1.0 / s[S_XI];
      return;
    case QMR_DELTA:  // delta = dot(z, y) (55-57); p, q coefficients (65-66)
      if (st->done) return;
      s[S_DELTA] = s[S_RR];
      if (s[S_DELTA] == 0.0) return x_fail(st, 3);
      if (st->iter <= 1) {
        s[S_PCOEF] = 0.0, s[S_QCOEF] = 0.0;
      } else {
        s[S_PCOEF] = -((s[S_XI] * s[S_DELTA]) / s[S_EP]);
        s[S_QCOEF] = -((s[S_RHO] * s[S_DELTA]) / s[S_EP]);
      }
      return;
    case QMR_EP:  // ep = dot(q, p~); beta (70-75)
      if (st->done) return;
      s[S_EP] = s[S_RR];
      if (s[S_EP] == 0.0) return x_fail(st, 4);
      s[S_BETA] = s[S_EP] / s[S_DELTA];
      if (s[S_BETA] == 0.0) return x_fail(st, 5);
      s[S_NBETA] = -s[S_BETA];
      return;
    case QMR_NORMS:  // rho_1 = rho; rho = two_norm(y) (77-78)
      if (st->done) return;
      s[S_RHO1] = s[S_RHO];
      s[S_RHO] = sqrt(fabs(s[S_RR]));
      return;
    case QMR_END: {  // xi; gamma, theta, eta; d and s coefficients (82-101)
      if (st->done) return;
      s[S_XI] = sqrt(fabs(s[S_RR2]));
      s[S_GAMMA1] = s[S_GAMMA];
      s[S_THETA1] = s[S_THETA];
      s[S_THETA] = s[S_RHO] / (s[S_GAMMA1] * s[S_BETA]);
      s[S_GAMMA] = 1.0 / sqrt(1.0 + s[S_THETA] * s[S_THETA]);
      if (s[S_GAMMA] == 0.0) return x_fail(st, 6);
      s[S_ETA] = -s[S_ETA] * s[S_RHO1] * s[S_GAMMA] * s[S_GAMMA] /
                 (s[S_BETA] * s[S_GAMMA1] * s[S_GAMMA1]);
      s[S_DMUL] = st->iter <= 1 ? 0.0
                                : s[S_THETA1] * s[S_THETA1] * s[S_GAMMA] * s[S_GAMMA];
      return;
    }

    // ---- idr_s ---------------------------------------------------------------
    // dense: M[s*s] (row-major, M[r][c]), m[s], c[s], -c[s], dm[s], LU work
    case IDR_ORTH_DOT:  // P_j -= dot(P_i, P_j) P_i (orth.hpp:30-31)
      s[S_NINV] = -s[S_RR];
      return;
    case IDR_ORTH_NORM:  // P_j /= two_norm(P_j) (orth.hpp:32)
      s[S_INV] = 1.0 / sqrt(fabs(s[S_RR]));
      return;
    case IDR_OMEGA0:  // omega = dot(v, r) / dot(v, v) (idr_s.hpp:57 and 79)
      if (st->done) return;
      s[S_OMEGA] = s[S_TV] / s[S_TT];
      s[S_NOMEGA] = -s[S_OMEGA];
      return;
    case IDR_STEP:  // (++iter).finished(r) (idr_s.hpp:62, 90)
      if (st->done) return;
      st->iter++;
      if (x_finished(st, sqrt(fabs(s[S_RR])))) x_stop(st);
      return;
    case IDR_M_INIT: {  // M[iall][k] = trans(P) * dR.vector(k) (idr_s.hpp:63)
      if (st->done) return;
      const int k = x.a;
      const double* dm = D + idr_dm(P);
      for (int r = 0; r < P; r++) D[r * P + k] = dm[r];
      return;
    }
    case IDR_LU: {  // c = lu_solve(M, m) (idr_s.hpp:72)
      if (st->done) return;
      double* m = D + idr_m(P);
      double* c = D + idr_c(P);
      double* nc = D + idr_nc(P);
      double* work = D + P * P + 4 * P;
      if (!dense_lu_solve(D, P, m, P, c, work)) {  // matrix_singular propagates out
        st->singular = 1, st->breakdown = 1;
        return x_stop(st);
      }
      for (int j = 0; j < P; j++) nc[j] = -c[j];
      return;
    }
    case IDR_M: {  // dm = trans(P) dR_oldest; M[iall][oldest] = dm; m += dm (93-95)
      if (st->done) return;
      const int k = x.a;
      double* m = D + idr_m(P);
      const double* dm = D + idr_dm(P);
      for (int r = 0; r < P; r++) D[r * P + k] = dm[r], m[r] += dm[r];
      return;
    }

    // ---- gmres ---------------------------------------------------------------
    // dense (restart m): H[(m+1)*m] row-major H[r][c] = H[r*m + c], g[m+1],
    // c[m+1], s[m+1], y[m], hr[m+1], ny / -H column [m+1], work
    case GM_START: {  // gmres_full: rho = g[0] = two_norm(r); finished(rho) (57-62)
      if (st->done) return;
      const int m = P;
      double* H = D;
      double* g = H + (m + 1) * m;
      double* cc = g + (m + 1);
      double* ss = cc + (m + 1);
      for (int i = 0; i < (m + 1) * m; i++) H[i] = 0.0;
      for (int i = 0; i <= m; i++) g[i] = 0.0, cc[i] = 0.0, ss[i] = 0.0;
      const double rho = sqrt(fabs(s[S_RR]));
      g[0] = rho;
      if (x_finished(st, rho)) return x_stop(st);
      const long long room = (long long)st->max_iter - st->iter;
      st->kmax = (int)std::min<long long>(std::min<long long>(x.n, room), m);
      s[S_INV] = 1.0 / rho;
      return;
    }
    case GM_STEP_BEGIN:  // the kernels of step k run only for k < kmax
      st->halt = st->done || x.a >= st->kmax;
      return;
    case GM_NORM1: {  // H[k+1][k] = two_norm(V[k+1]) after the first sweep (gmres.hpp:74)
      if (st->halt) return;
      const int m = P, k = x.a;
      D[(k + 1) * m + k] = sqrt(fabs(s[S_RR]));
      return;
    }
    case GM_STEP_END: {  // reorthogonalisation sums, H[k+1][k], Givens (75-102)
      if (st->halt) return;
      const int m = P, k = x.a;
      double* H = D;
      double* g = H + (m + 1) * m;
      double* cc = g + (m + 1);
      double* ss = cc + (m + 1);
      const double* hr = D + gm_hr(m);
      for (int j = 0; j <= k; j++) H[j * m + k] += hr[j];
      H[(k + 1) * m + k] = sqrt(fabs(s[S_RR]));
      s[S_INV] = H[(k + 1) * m + k] != 0.0 ? 1.0 / H[(k + 1) * m + k] : 1.0;
      // k Givens rotations from column k-1 (mtl::mat::givens, givens.hpp:33-82):
      // rows i, i+1 by G^T, then columns i, i+1 by G
      for (int i = 0; i < k; i++) {
        const double a = H[i * m + (k - 1)], b = H[(i + 1) * m + (k - 1)];
        double c, sn;
        if (b == 0.0) {
          c = 1.0, sn = 0.0;
        } else if (fabs(b) > fabs(a)) {
          const double t = -a / b;
          sn = 1.0 / sqrt(1.0 + t * t);
          c = sn * t;
        } else {
          const double t = -b / a;
          c = 1.0 / sqrt(1.0 + t * t);
          sn = c * t;
        }
        for (int col = 0; col < m; col++) {  // G^T * rows
          const double u = H[i * m + col], w = H[(i + 1) * m + col];
          H[i * m + col] = c * u + (-sn) * w;
          H[(i + 1) * m + col] = sn * u + c * w;
        }
        for (int row = 0; row <= m; row++) {  // columns * G
          const double u = H[row * m + i], w = (i + 1 < m) ? H[row * m + i + 1] : 0.0;
          H[row * m + i] = u * c + w * (-sn);
          if (i + 1 < m) H[row * m + i + 1] = u * sn + w * c;
        }
      }
      const double hkk = H[k * m + k], hk1 = H[(k + 1) * m + k];
      const double nu = sqrt(hkk * hkk + hk1 * hk1);
      if (nu != 0.0) {
        cc[k] = hkk / nu;
        ss[k] = -hk1 / nu;
        H[k * m + k] = cc[k] * hkk - ss[k] * hk1;
        H[(k + 1) * m + k] = 0.0;
        const double w1 = cc[k] * g[k] - ss[k] * g[k + 1];
        const double w2 = ss[k] * g[k] + cc[k] * g[k + 1];
        g[k] = w1, g[k + 1] = w2;
      }
      st->iter++;
      return;
    }
    case GM_SOLVE: {  // reduce k; y = lu_solve(H[range][range], g[range]) (106-124)
      st->halt = st->done;
      if (st->done) return;
      const int m = P;
      double* H = D;
      double* g = D + gm_g(m);
      double* y = D + gm_y(m);
      double* work = D + gm_hr(m) + 2 * (m + 1);
      int k = st->kmax;
      while (k > 0 && fabs(g[k - 1]) <= st->atol) k--;
      int range = k;
      for (; range > 0; --range)
        if (dense_lu_solve(H, m, g, range, y, work)) break;
      for (int j = range; j < m; j++) y[j] = 0.0;
      if (range == 0) return x_fail(st, 2);
      return;
    }
    case GM_END:  // r = b - A x; return iter.terminate(r) (127-128) + update_progress
      if (st->done) return;
      if (x_finished(st, sqrt(fabs(s[S_RR])))) x_stop(st);
      return;
  }
}

__global__ void xscalar_kernel(XState* st, ScalarArgs a) {
  if (threadIdx.x == 0 && blockIdx.x == 0) run_step(st, a);
}

__global__ void xset_halt_kernel(XState* st) {
  if (threadIdx.x == 0) st->halt = st->done;
}

// ---------------------------------------------------------------------------
// Host side: workspace, recording helpers and the eight recipes.

// Vector slots of each method (0: x, 1: b).
enum { VX = 0, VB = 1 };
namespace bicg_v { enum { R = 2, Z, P, Q, RT, ZT, PT, QT, COUNT }; }
namespace cgs_v { enum { R = 2, RTIL, P, PHAT, Q, QHAT, VHAT, U, UHAT, COUNT }; }
namespace ell_v { enum { X0 = 2, Y, R0T, TMP, RH0 }; }  // then r_hat[0..l], u_hat[0..l]
namespace tfqmr_v { enum { RT = 2, R, U1, U2, Y1, Y2, WV, D, V, TMP, COUNT }; }
namespace qmr_v { enum { R = 2, VT, Y, WT, Z, V, WV, YT, ZT, P, Q, PT, D, S, TMP, COUNT }; }
namespace idr_v { enum { R = 2, V, TV, Q, TMP, P0 }; }   // then P[s], dR[s], dX[s]
namespace gm_v { enum { R0 = 2, RV, VA0, WV, Z, V0 }; }  // then V[0..m]

int vec_count(int method, int P) {
  switch (method) {
    case MTLGPU_BICG: return bicg_v::COUNT;
    case MTLGPU_CGS: return cgs_v::COUNT;
    case MTLGPU_BICGSTAB_2:
    case MTLGPU_BICGSTAB_ELL: return ell_v::RH0 + 2 * (P + 1);
    case MTLGPU_TFQMR: return tfqmr_v::COUNT;
    case MTLGPU_QMR: return qmr_v::COUNT;
    case MTLGPU_IDR_S: return idr_v::P0 + 3 * P;
    case MTLGPU_GMRES: return gm_v::V0 + P + 1;
  }
  return 0;
}

// Iterations recorded per graph launch (a gmres restart cycle counts as one).
int graph_iters(int method) {
  switch (method) {
    case MTLGPU_BICGSTAB_ELL:
    case MTLGPU_IDR_S: return 2;
    case MTLGPU_GMRES: return 1;
    default: return 8;
  }
}

}  // namespace

struct XWork {
  Csr* A = nullptr;
  Csr* AT = nullptr;  // transposed matrix (bicg, qmr)
  Pc* L = nullptr;
  Pc* R = nullptr;
  int method = 0, param = 0, n = 0, grid = 1;
  std::vector<double*> vec;
  XState* st = nullptr;
  XState* h_st = nullptr;
  double* dense = nullptr;
  int dense_n = 0;
  Sum<kMaxDots>* partials = nullptr;
  unsigned* counter = nullptr;
  double* history = nullptr;
  int hist_cap = 0;
  cudaGraphExec_t exec = nullptr;
  size_t graph_nodes = 0;
};

namespace {

Term T(const double* v, double mul = 1.0) { return Term{v, nullptr, mul}; }
Term T(const double* v, const double* coef, double mul = 1.0) { return Term{v, coef, mul}; }
struct DotSpec {
  const double* x;
  const double* y;
  double* out;
};

struct Rec {
  XWork* W;
  Ctx* ctx;
  double* v(int i) const { return W->vec[i]; }
  double* sl(int k) const { return &W->st->s[k]; }
  double* dn(int off) const { return W->dense + off; }
  const int* halt() const { return &W->st->halt; }

  mtlgpu_status lin(double* out, std::initializer_list<Term> terms) {
    return lin_n(out, std::vector<Term>(terms));
  }
  // out = sum of the terms; more than kMaxTerms are taken in chunks, each
  // later chunk adding to out (out must not be a source of a later chunk).
  mtlgpu_status lin_n(double* out, const std::vector<Term>& terms) {
    size_t done = 0;
    bool first = true;
    while (done < terms.size() || first) {
      LinArgs a{};
      a.out = out;
      a.nt = 0;
      if (!first) a.t[a.nt++] = T(out);
      while (done < terms.size() && a.nt < kMaxTerms) a.t[a.nt++] = terms[done++];
      if (a.nt == 0) a.t[a.nt++] = T(out, 0.0);
      xlin_kernel<<<W->grid, kBlock, 0, ctx->stream>>>(W->n, a, W->st);
      ctx->launches++;
      first = false;
    }
    MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
    return MTLGPU_OK;
  }
  mtlgpu_status dots(const std::vector<DotSpec>& d) {
    for (size_t i = 0; i < d.size(); i += kMaxDots) {
      DotArgs a{};
      a.nd = (int)std::min<size_t>(kMaxDots, d.size() - i);
      for (int k = 0; k < a.nd; k++) a.x[k] = d[i + k].x, a.y[k] = d[i + k].y, a.out[k] = d[i + k].out;
      xdots_kernel<<<W->grid, kBlock, 0, ctx->stream>>>(W->n, a, W->st, W->partials, W->counter);
      ctx->launches++;
    }
    MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
    return MTLGPU_OK;
  }
  mtlgpu_status dot(const double* x, const double* y, double* out) { return dots({{x, y, out}}); }
  mtlgpu_status spmv(Csr* M, const double* x, double* y) {
    SpmvArgs a;
    a.skip = halt();
    return spmv_launch<double>(M, x, y, a);
  }
  // z = solve(P, r) / adjoint_solve(P, r); no preconditioner: a copy
  mtlgpu_status pc(Pc* P, const double* r, double* z, bool adjoint = false) {
    if (!P) return lin(z, {T(r)});
    return pc_apply_t<double>(P, r, z, adjoint, halt(), false, false);
  }
  mtlgpu_status scal(int step, int a = 0, int b = 0) {
    ScalarArgs x{step, a, b, W->param, W->n, W->dense};
    xscalar_kernel<<<1, 32, 0, ctx->stream>>>(W->st, x);
    ctx->launches++;
    MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
    return MTLGPU_OK;
  }
  mtlgpu_status zero(double* p, long long count) {
    MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(p, 0, sizeof(double) * count, ctx->stream));
    return MTLGPU_OK;
  }
  mtlgpu_status sync_state() {
    MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(W->h_st, W->st, sizeof(XState), cudaMemcpyDeviceToHost,
                                         ctx->stream));
    MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return MTLGPU_OK;
  }
};

// r = b - A x (into out)
mtlgpu_status residual(Rec& r, const double* x, double* out) {
  MTLGPU_TRY(r.spmv(r.W->A, x, out));
  return r.lin(out, {T(r.v(VB)), T(out, -1.0)});
}

// ---- bicg: itl/krylov/bicg.hpp:22-63 ------------------------------------------
mtlgpu_status bicg_prologue(Rec& r) {
  using namespace bicg_v;
  MTLGPU_TRY(residual(r, r.v(VX), r.v(R)));                        // r(b - A * x)
  MTLGPU_TRY(r.lin(r.v(RT), {T(r.v(R))}));                          // r_tilde(r)
  MTLGPU_TRY(r.zero(r.v(P), r.W->n));
  MTLGPU_TRY(r.zero(r.v(PT), r.W->n));
  MTLGPU_TRY(r.dot(r.v(R), r.v(R), r.sl(S_RR)));
  return r.scal(X_CHECK_RR);                                        // while (!finished(r))
}
mtlgpu_status bicg_record(Rec& r) {
  using namespace bicg_v;
  XWork* W = r.W;
  MTLGPU_TRY(r.scal(X_INC));                                         // ++iter
  MTLGPU_TRY(r.pc(W->L, r.v(R), r.v(Z)));                            // z = solve(M, r)
  MTLGPU_TRY(r.pc(W->L, r.v(RT), r.v(ZT), true));                    // z~ = adjoint_solve(M, r~)
  MTLGPU_TRY(r.dot(r.v(ZT), r.v(Z), r.sl(S_RHO1)));                  // rho_1 = dot(z~, z)
  MTLGPU_TRY(r.scal(BICG_RHO));
  MTLGPU_TRY(r.lin(r.v(P), {T(r.v(Z)), T(r.v(P), r.sl(S_BETA))}));   // p = z + beta p
  MTLGPU_TRY(r.lin(r.v(PT), {T(r.v(ZT)), T(r.v(PT), r.sl(S_BETA))}));
  MTLGPU_TRY(r.spmv(W->A, r.v(P), r.v(Q)));                          // q = A p
  MTLGPU_TRY(r.spmv(W->AT, r.v(PT), r.v(QT)));                       // q~ = adjoint(A) p~
  MTLGPU_TRY(r.dot(r.v(PT), r.v(Q), r.sl(S_RR2)));
  MTLGPU_TRY(r.scal(BICG_ALPHA));                                    // alpha = rho_1 / dot(p~, q)
  MTLGPU_TRY(r.lin(r.v(VX), {T(r.v(VX)), T(r.v(P), r.sl(S_ALPHA))}));
  MTLGPU_TRY(r.lin(r.v(R), {T(r.v(R)), T(r.v(Q), r.sl(S_NALPHA))}));
  MTLGPU_TRY(r.lin(r.v(RT), {T(r.v(RT)), T(r.v(QT), r.sl(S_NALPHA))}));
  MTLGPU_TRY(r.dot(r.v(R), r.v(R), r.sl(S_RR)));
  return r.scal(BICG_END);
}

// ---- cgs: itl/krylov/cgs.hpp:23-65 --------------------------------------------
mtlgpu_status cgs_prologue(Rec& r) {
  using namespace cgs_v;
  MTLGPU_TRY(residual(r, r.v(VX), r.v(R)));
  MTLGPU_TRY(r.lin(r.v(RTIL), {T(r.v(R))}));
  MTLGPU_TRY(r.zero(r.v(P), r.W->n));
  MTLGPU_TRY(r.zero(r.v(Q), r.W->n));
  MTLGPU_TRY(r.dot(r.v(R), r.v(R), r.sl(S_RR)));
  return r.scal(X_CHECK_RR);
}
mtlgpu_status cgs_record(Rec& r) {
  using namespace cgs_v;
  XWork* W = r.W;
  MTLGPU_TRY(r.scal(X_INC));
  MTLGPU_TRY(r.dot(r.v(RTIL), r.v(R), r.sl(S_RHO1)));               // rho_1 = dot(r~, r)
  MTLGPU_TRY(r.scal(CGS_RHO));
  MTLGPU_TRY(r.lin(r.v(U), {T(r.v(R)), T(r.v(Q), r.sl(S_BETA))}));  // u = r + beta q
  MTLGPU_TRY(r.lin(r.v(P), {T(r.v(U)), T(r.v(Q), r.sl(S_BETA)),     // p = u + beta (q + beta p)
                            T(r.v(P), r.sl(S_BETA2))}));
  MTLGPU_TRY(r.pc(W->L, r.v(P), r.v(PHAT)));
  MTLGPU_TRY(r.spmv(W->A, r.v(PHAT), r.v(VHAT)));                    // vhat = A solve(M, p)
  MTLGPU_TRY(r.dot(r.v(RTIL), r.v(VHAT), r.sl(S_RR2)));
  MTLGPU_TRY(r.scal(CGS_ALPHA));
  MTLGPU_TRY(r.lin(r.v(Q), {T(r.v(U)), T(r.v(VHAT), r.sl(S_NALPHA))}));  // q = u - alpha vhat
  MTLGPU_TRY(r.lin(r.v(U), {T(r.v(U)), T(r.v(Q))}));                 // u += q
  MTLGPU_TRY(r.pc(W->L, r.v(U), r.v(UHAT)));                         // uhat = solve(M, u)
  MTLGPU_TRY(r.lin(r.v(VX), {T(r.v(VX)), T(r.v(UHAT), r.sl(S_ALPHA))}));
  MTLGPU_TRY(r.spmv(W->A, r.v(UHAT), r.v(QHAT)));
  MTLGPU_TRY(r.lin(r.v(R), {T(r.v(R)), T(r.v(QHAT), r.sl(S_NALPHA))}));
  MTLGPU_TRY(r.dot(r.v(R), r.v(R), r.sl(S_RR)));
  return r.scal(CGS_END);
}

// ---- bicgstab_ell / bicgstab_2: bicgstab_ell.hpp:37-132, bicgstab_2.hpp:33-131
// bicgstab_2 is the same loop with l = 2 and no right preconditioner.
int ell_l(const XWork* W) { return W->param; }
double* rh(Rec& r, int i) { return r.v(ell_v::RH0 + i); }
double* uh(Rec& r, int i) { return r.v(ell_v::RH0 + ell_l(r.W) + 1 + i); }

mtlgpu_status ell_prologue(Rec& r) {
  using namespace ell_v;
  XWork* W = r.W;
  const int l = ell_l(W);
  for (int i = 0; i <= l; i++) {
    MTLGPU_TRY(r.zero(rh(r, i), W->n));
    MTLGPU_TRY(r.zero(uh(r, i), W->n));
  }
  MTLGPU_TRY(r.zero(r.v(X0), W->n));                                 // x0 = zero
  MTLGPU_TRY(r.zero(W->dense, W->dense_n));
  MTLGPU_TRY(r.lin(rh(r, 0), {T(r.v(VB))}));                         // r_hat[0] = b
  MTLGPU_TRY(r.dot(r.v(VX), r.v(VX), r.sl(S_RR)));
  MTLGPU_TRY(r.sync_state());
  if (W->h_st->s[S_RR] != 0.0) {                                     // shift problem (47-52)
    MTLGPU_TRY(r.spmv(W->A, r.v(VX), r.v(Y)));
    MTLGPU_TRY(r.lin(rh(r, 0), {T(rh(r, 0)), T(r.v(Y), -1.0)}));
    MTLGPU_TRY(r.lin(r.v(X0), {T(r.v(VX))}));
    MTLGPU_TRY(r.zero(r.v(VX), W->n));
  }
  MTLGPU_TRY(r.dot(rh(r, 0), rh(r, 0), r.sl(S_RR)));
  MTLGPU_TRY(r.scal(ELL_INIT_NORM));
  MTLGPU_TRY(r.lin(r.v(R0T), {T(rh(r, 0), r.sl(S_INV))}));           // r0~ = r_hat[0] / two_norm
  MTLGPU_TRY(r.pc(W->L, rh(r, 0), r.v(Y)));                          // y = solve(L, r_hat[0])
  MTLGPU_TRY(r.lin(rh(r, 0), {T(r.v(Y))}));                          // r_hat[0] = y
  MTLGPU_TRY(r.dot(rh(r, 0), rh(r, 0), r.sl(S_RR)));
  return r.scal(X_CHECK_RR);                                         // while (!finished(r_hat[0]))
}
mtlgpu_status ell_record(Rec& r) {
  using namespace ell_v;
  XWork* W = r.W;
  const int l = ell_l(W), l1 = l + 1;
  const bool right = W->method == MTLGPU_BICGSTAB_ELL;
  MTLGPU_TRY(r.scal(ELL_BEGIN));
  for (int j = 0; j < l; j++) {
    MTLGPU_TRY(r.dot(r.v(R0T), rh(r, j), r.sl(S_RHO1)));
    MTLGPU_TRY(r.scal(ELL_BETA));
    for (int i = 0; i <= j; i++)                                     // u_hat[i] = r_hat[i] - beta u_hat[i]
      MTLGPU_TRY(r.lin(uh(r, i), {T(rh(r, i)), T(uh(r, i), r.sl(S_NBETA))}));
    if (right) {                                                     // y = A * solve(R, u_hat[j])
      MTLGPU_TRY(r.pc(W->R, uh(r, j), r.v(TMP)));
      MTLGPU_TRY(r.spmv(W->A, r.v(TMP), r.v(Y)));
    } else {
      MTLGPU_TRY(r.spmv(W->A, uh(r, j), r.v(Y)));
    }
    MTLGPU_TRY(r.pc(W->L, r.v(Y), uh(r, j + 1)));                    // u_hat[j+1] = solve(L, y)
    MTLGPU_TRY(r.dot(r.v(R0T), uh(r, j + 1), r.sl(S_GAMMA)));
    MTLGPU_TRY(r.scal(ELL_ALPHA));
    for (int i = 0; i <= j; i++)                                     // r_hat[i] -= alpha u_hat[i+1]
      MTLGPU_TRY(r.lin(rh(r, i), {T(rh(r, i)), T(uh(r, i + 1), r.sl(S_NALPHA))}));
    MTLGPU_TRY(r.dot(rh(r, j), rh(r, j), r.sl(S_RR)));
    MTLGPU_TRY(r.scal(ELL_CHECK));                                   // if (finished(r_hat[j])) return
    if (right) {                                                     // r_hat[j+1] = solve(R, r_hat[j])
      MTLGPU_TRY(r.pc(W->R, rh(r, j), rh(r, j + 1)));
      MTLGPU_TRY(r.spmv(W->A, rh(r, j + 1), r.v(Y)));
    } else {
      MTLGPU_TRY(r.spmv(W->A, rh(r, j), r.v(Y)));
    }
    MTLGPU_TRY(r.pc(W->L, r.v(Y), rh(r, j + 1)));                    // r_hat[j+1] = solve(L, y)
    MTLGPU_TRY(r.lin(r.v(VX), {T(r.v(VX)), T(uh(r, 0), r.sl(S_ALPHA))}));
  }
  // mod GS (MR part): tau = orthogonalize_factors(r_hat[1..l]) (orth.hpp:53-88)
  MTLGPU_TRY(r.dot(rh(r, 1), rh(r, 1), r.sl(S_RR)));
  MTLGPU_TRY(r.scal(ELL_TAU_D, 0));
  for (int jj = 1; jj < l; jj++) {
    for (int ii = 0; ii < jj; ii++) {
      MTLGPU_TRY(r.dot(rh(r, ii + 1), rh(r, jj + 1), r.sl(S_RR)));
      MTLGPU_TRY(r.scal(ELL_TAU_T, ii, jj));
      MTLGPU_TRY(r.lin(rh(r, jj + 1), {T(rh(r, jj + 1)), T(rh(r, ii + 1), r.sl(S_NINV))}));
    }
    MTLGPU_TRY(r.dot(rh(r, jj + 1), rh(r, jj + 1), r.sl(S_RR)));
    MTLGPU_TRY(r.scal(ELL_TAU_D, jj));
  }
  std::vector<DotSpec> dg;
  for (int j = 1; j <= l; j++) dg.push_back({rh(r, j), rh(r, 0), r.dn(ell_dga(l1) + j)});
  MTLGPU_TRY(r.dots(dg));                                            // dot(r_hat[j], r_hat[0])
  MTLGPU_TRY(r.scal(ELL_GAMMA));
  const double* gamma = r.dn(ell_gamma(l1));
  const double* gamma_aa = r.dn(ell_gamma_aa(l1));
  const double* ngamma_a = r.dn(ell_neg(l1));
  const double* ngamma = r.dn(ell_neg(l1) + l1);
  MTLGPU_TRY(r.lin(r.v(VX), {T(r.v(VX)), T(rh(r, 0), gamma + 1)}));          // x += gamma[1] r_hat[0]
  MTLGPU_TRY(r.lin(rh(r, 0), {T(rh(r, 0)), T(rh(r, l), ngamma_a + l)}));     // r_hat[0] -= gamma_a[l] r_hat[l]
  MTLGPU_TRY(r.lin(uh(r, 0), {T(uh(r, 0)), T(uh(r, l), ngamma + l)}));       // u_hat[0] -= gamma[l] u_hat[l]
  for (int j = 1; j < l; j++) {
    MTLGPU_TRY(r.lin(uh(r, 0), {T(uh(r, 0)), T(uh(r, j), ngamma + j)}));
    MTLGPU_TRY(r.lin(r.v(VX), {T(r.v(VX)), T(rh(r, j), gamma_aa + j)}));
    MTLGPU_TRY(r.lin(rh(r, 0), {T(rh(r, 0)), T(rh(r, j), ngamma_a + j)}));
  }
  MTLGPU_TRY(r.dot(rh(r, 0), rh(r, 0), r.sl(S_RR)));
  return r.scal(X_CHECK_RR);
}
// x = solve(R, x); x += x0 -- on every way out of the loop
mtlgpu_status ell_epilogue(Rec& r) {
  using namespace ell_v;
  if (r.W->method == MTLGPU_BICGSTAB_ELL && r.W->R) {
    MTLGPU_TRY(r.pc(r.W->R, r.v(VX), r.v(TMP)));
    return r.lin(r.v(VX), {T(r.v(TMP)), T(r.v(X0))});
  }
  return r.lin(r.v(VX), {T(r.v(VX)), T(r.v(X0))});
}

// ---- tfqmr: itl/krylov/tfqmr.hpp:26-100 ------------------------------------------
mtlgpu_status tfqmr_prologue(Rec& r) {
  using namespace tfqmr_v;
  XWork* W = r.W;
  MTLGPU_TRY(r.pc(W->R, r.v(VX), r.v(TMP)));
  MTLGPU_TRY(residual(r, r.v(TMP), r.v(RT)));                       // rt(b - A * solve(R, x))
  MTLGPU_TRY(r.pc(W->L, r.v(RT), r.v(R)));                           // r(solve(L, rt))
  MTLGPU_TRY(r.zero(r.v(D), W->n));                                  // d(resource(x), zero)
  MTLGPU_TRY(r.dot(r.v(RT), r.v(RT), r.sl(S_RR)));
  MTLGPU_TRY(r.scal(X_CHECK_RR));                                    // if (finished(rt)) return
  MTLGPU_TRY(r.lin(r.v(Y1), {T(r.v(R))}));
  MTLGPU_TRY(r.lin(r.v(WV), {T(r.v(R))}));
  MTLGPU_TRY(r.pc(W->R, r.v(Y1), r.v(TMP)));
  MTLGPU_TRY(r.spmv(W->A, r.v(TMP), r.v(RT)));                       // rt = A solve(R, y1)
  MTLGPU_TRY(r.pc(W->L, r.v(RT), r.v(U1)));                          // u1 = v = solve(L, rt)
  MTLGPU_TRY(r.lin(r.v(V), {T(r.v(U1))}));
  MTLGPU_TRY(r.dot(r.v(R), r.v(R), r.sl(S_RR)));
  return r.scal(TFQMR_INIT);
}
mtlgpu_status tfqmr_record(Rec& r) {
  using namespace tfqmr_v;
  XWork* W = r.W;
  MTLGPU_TRY(r.dot(r.v(R), r.v(V), r.sl(S_SIGMA)));                  // sigma = dot(r, v)
  MTLGPU_TRY(r.scal(TFQMR_SIGMA));
  // j = 1
  MTLGPU_TRY(r.lin(r.v(WV), {T(r.v(WV)), T(r.v(U1), r.sl(S_NALPHA))}));
  MTLGPU_TRY(r.lin(r.v(D), {T(r.v(Y1)), T(r.v(D), r.sl(S_DCOEF))}));
  MTLGPU_TRY(r.dot(r.v(WV), r.v(WV), r.sl(S_RR)));
  MTLGPU_TRY(r.scal(TFQMR_THETA));
  MTLGPU_TRY(r.lin(r.v(VX), {T(r.v(VX)), T(r.v(D), r.sl(S_ETA))}));
  // j = 2
  MTLGPU_TRY(r.lin(r.v(Y2), {T(r.v(Y1)), T(r.v(V), r.sl(S_NALPHA))}));
  MTLGPU_TRY(r.pc(W->R, r.v(Y2), r.v(TMP)));
  MTLGPU_TRY(r.spmv(W->A, r.v(TMP), r.v(RT)));
  MTLGPU_TRY(r.pc(W->L, r.v(RT), r.v(U2)));
  MTLGPU_TRY(r.lin(r.v(WV), {T(r.v(WV)), T(r.v(U2), r.sl(S_NALPHA))}));
  MTLGPU_TRY(r.lin(r.v(D), {T(r.v(Y2)), T(r.v(D), r.sl(S_DCOEF))}));
  MTLGPU_TRY(r.dot(r.v(WV), r.v(WV), r.sl(S_RR)));
  MTLGPU_TRY(r.scal(TFQMR_THETA));
  MTLGPU_TRY(r.lin(r.v(VX), {T(r.v(VX)), T(r.v(D), r.sl(S_ETA))}));
  // rhon = dot(r, w); beta; y1 = w + beta y2; u1; v = u1 + beta (u2 + beta v)
  MTLGPU_TRY(r.dot(r.v(R), r.v(WV), r.sl(S_RR2)));
  MTLGPU_TRY(r.scal(TFQMR_RHO));
  MTLGPU_TRY(r.lin(r.v(Y1), {T(r.v(WV)), T(r.v(Y2), r.sl(S_BETA))}));
  MTLGPU_TRY(r.pc(W->R, r.v(Y1), r.v(TMP)));
  MTLGPU_TRY(r.spmv(W->A, r.v(TMP), r.v(RT)));
  MTLGPU_TRY(r.pc(W->L, r.v(RT), r.v(U1)));
  // (the reference's final rt = A * x - b is never read and is not computed)
  return r.lin(r.v(V), {T(r.v(U1)), T(r.v(U2), r.sl(S_BETA)), T(r.v(V), r.sl(S_BETA2))});
}
mtlgpu_status tfqmr_epilogue(Rec& r) {  // x = solve(R, x): shift back
  using namespace tfqmr_v;
  if (!r.W->R) return MTLGPU_OK;
  MTLGPU_TRY(r.pc(r.W->R, r.v(VX), r.v(TMP)));
  return r.lin(r.v(VX), {T(r.v(TMP))});
}

// ---- qmr: itl/krylov/qmr.hpp:24-109 ------------------------------------------------
mtlgpu_status qmr_prologue(Rec& r) {
  using namespace qmr_v;
  XWork* W = r.W;
  MTLGPU_TRY(residual(r, r.v(VX), r.v(R)));                         // r(b - A * x)
  MTLGPU_TRY(r.lin(r.v(VT), {T(r.v(R))}));                           // v_tld(r)
  MTLGPU_TRY(r.pc(W->L, r.v(VT), r.v(Y)));                           // y(solve(L, v_tld))
  MTLGPU_TRY(r.lin(r.v(WT), {T(r.v(R))}));                           // w_tld(r)
  MTLGPU_TRY(r.pc(W->R, r.v(WT), r.v(Z), true));                     // z(adjoint_solve(R, w_tld))
  for (int k : {P, Q, D, S}) MTLGPU_TRY(r.zero(r.v(k), W->n));
  MTLGPU_TRY(r.dot(r.v(R), r.v(R), r.sl(S_RR)));
  MTLGPU_TRY(r.scal(X_CHECK_RR));                                    // if (finished(r)) return
  MTLGPU_TRY(r.dots({{r.v(Y), r.v(Y), r.sl(S_RR)}, {r.v(Z), r.v(Z), r.sl(S_RR2)}}));
  return r.scal(QMR_INIT);
}
mtlgpu_status qmr_record(Rec& r) {
  using namespace qmr_v;
  XWork* W = r.W;
  MTLGPU_TRY(r.scal(QMR_BEGIN));
  MTLGPU_TRY(r.lin(r.v(V), {T(r.v(VT), r.sl(S_INV_RHO))}));          // v = v_tld / rho
  MTLGPU_TRY(r.lin(r.v(Y), {T(r.v(Y), r.sl(S_INV_RHO))}));           // y /= rho
  MTLGPU_TRY(r.lin(r.v(WV), {T(r.v(WT), r.sl(S_INV_XI))}));           // w = w_tld / xi
  MTLGPU_TRY(r.lin(r.v(Z), {T(r.v(Z), r.sl(S_INV_XI))}));            // z /= xi
  MTLGPU_TRY(r.dot(r.v(Z), r.v(Y), r.sl(S_RR)));                     // delta = dot(z, y)
  MTLGPU_TRY(r.scal(QMR_DELTA));
  MTLGPU_TRY(r.pc(W->R, r.v(Y), r.v(YT)));                           // y_tld = solve(R, y)
  MTLGPU_TRY(r.pc(W->L, r.v(Z), r.v(ZT), true));                     // z_tld = adjoint_solve(L, z)
  MTLGPU_TRY(r.lin(r.v(P), {T(r.v(YT)), T(r.v(P), r.sl(S_PCOEF))}));
  MTLGPU_TRY(r.lin(r.v(Q), {T(r.v(ZT)), T(r.v(Q), r.sl(S_QCOEF))}));
  MTLGPU_TRY(r.spmv(W->A, r.v(P), r.v(PT)));                         // p_tld = A p
  MTLGPU_TRY(r.dot(r.v(Q), r.v(PT), r.sl(S_RR)));                    // ep = dot(q, p_tld)
  MTLGPU_TRY(r.scal(QMR_EP));
  MTLGPU_TRY(r.lin(r.v(VT), {T(r.v(PT)), T(r.v(V), r.sl(S_NBETA))}));  // v_tld = p_tld - beta v
  MTLGPU_TRY(r.pc(W->L, r.v(VT), r.v(Y)));                           // y = solve(L, v_tld)
  MTLGPU_TRY(r.dot(r.v(Y), r.v(Y), r.sl(S_RR)));
  MTLGPU_TRY(r.scal(QMR_NORMS));
  MTLGPU_TRY(r.spmv(W->AT, r.v(Q), r.v(TMP)));                       // w_tld = trans(A) q - beta w
  MTLGPU_TRY(r.lin(r.v(WT), {T(r.v(TMP)), T(r.v(WV), r.sl(S_NBETA))}));
  MTLGPU_TRY(r.pc(W->R, r.v(WT), r.v(Z), true));                     // z = adjoint_solve(R, w_tld)
  MTLGPU_TRY(r.dot(r.v(Z), r.v(Z), r.sl(S_RR2)));
  MTLGPU_TRY(r.scal(QMR_END));
  MTLGPU_TRY(r.lin(r.v(D), {T(r.v(P), r.sl(S_ETA)), T(r.v(D), r.sl(S_DMUL))}));
  MTLGPU_TRY(r.lin(r.v(S), {T(r.v(PT), r.sl(S_ETA)), T(r.v(S), r.sl(S_DMUL))}));
  MTLGPU_TRY(r.lin(r.v(VX), {T(r.v(VX)), T(r.v(D))}));               // x += d
  return r.lin(r.v(R), {T(r.v(R)), T(r.v(S), -1.0)});               // r -= s
}

// ---- idr_s: itl/krylov/idr_s.hpp:30-105 (preconditioners ignored) ---------------------
double* idr_p(Rec& r, int k) { return r.v(idr_v::P0 + k); }
double* idr_dr(Rec& r, int k) { return r.v(idr_v::P0 + r.W->param + k); }
double* idr_dx(Rec& r, int k) { return r.v(idr_v::P0 + 2 * r.W->param + k); }

// The random shadow space: mtl::mat::random on the multi_vector P
// (mtl/operation/random.hpp:27-37, 45-50, 70-75, 105-110) -- the matrix-level
// seed object takes srand(17), vector k is then filled from srand(17 (k + 2))
// and rand(), as in a process whose seed counter starts at 0.  Like the
// reference, this reseeds the C library's generator.
mtlgpu_status idr_random_shadow(Rec& r) {
  XWork* W = r.W;
  std::vector<double> h(W->n);
  for (int k = 0; k < W->param; k++) {
    srand(17u * unsigned(k + 2));
    for (int i = 0; i < W->n; i++) h[i] = double(rand());
    MTLGPU_TRY_CUDA(r.ctx, cudaMemcpyAsync(idr_p(r, k), h.data(), sizeof(double) * W->n,
                                           cudaMemcpyHostToDevice, r.ctx->stream));
    MTLGPU_TRY_CUDA(r.ctx, cudaStreamSynchronize(r.ctx->stream));
  }
  return MTLGPU_OK;
}
mtlgpu_status idr_m_update(Rec& r, int k, int step) {  // dm = trans(P) * dR.vector(k)
  const int s = r.W->param;
  std::vector<DotSpec> d;
  for (int i = 0; i < s; i++) d.push_back({idr_p(r, i), idr_dr(r, k), r.dn(idr_dm(s) + i)});
  MTLGPU_TRY(r.dots(d));
  return r.scal(step, k);
}
mtlgpu_status idr_prologue(Rec& r) {
  using namespace idr_v;
  XWork* W = r.W;
  const int s = W->param;
  MTLGPU_TRY(residual(r, r.v(VX), r.v(R)));                         // r(b - A * x)
  MTLGPU_TRY(r.zero(W->dense, W->dense_n));
  for (int k = 0; k < s; k++) {
    MTLGPU_TRY(r.zero(idr_dr(r, k), W->n));
    MTLGPU_TRY(r.zero(idr_dx(r, k), W->n));
  }
  MTLGPU_TRY(idr_random_shadow(r));                                  // random(P)
  MTLGPU_TRY(r.lin(idr_p(r, 0), {T(r.v(R))}));                       // P.vector(0) = r
  for (int j = 0; j < s; j++) {                                      // orth(P) (orth.hpp:22-42)
    for (int i = 0; i < j; i++) {
      MTLGPU_TRY(r.dot(idr_p(r, i), idr_p(r, j), r.sl(S_RR)));
      MTLGPU_TRY(r.scal(IDR_ORTH_DOT));
      MTLGPU_TRY(r.lin(idr_p(r, j), {T(idr_p(r, j)), T(idr_p(r, i), r.sl(S_NINV))}));
    }
    MTLGPU_TRY(r.dot(idr_p(r, j), idr_p(r, j), r.sl(S_RR)));
    MTLGPU_TRY(r.scal(IDR_ORTH_NORM));
    MTLGPU_TRY(r.lin(idr_p(r, j), {T(idr_p(r, j), r.sl(S_INV))}));
  }
  for (int k = 0; k < s; k++) {                                      // idr_s.hpp:55-64
    MTLGPU_TRY(r.spmv(W->A, r.v(R), r.v(V)));                        // v = A r
    MTLGPU_TRY(r.dots({{r.v(V), r.v(R), r.sl(S_TV)}, {r.v(V), r.v(V), r.sl(S_TT)}}));
    MTLGPU_TRY(r.scal(IDR_OMEGA0));                                  // omega = dot(v,r)/dot(v,v)
    MTLGPU_TRY(r.lin(idr_dx(r, k), {T(r.v(R), r.sl(S_OMEGA))}));
    MTLGPU_TRY(r.lin(idr_dr(r, k), {T(r.v(V), r.sl(S_NOMEGA))}));
    MTLGPU_TRY(r.lin(r.v(VX), {T(r.v(VX)), T(idr_dx(r, k))}));
    MTLGPU_TRY(r.lin(r.v(R), {T(r.v(R)), T(idr_dr(r, k))}));
    MTLGPU_TRY(r.dot(r.v(R), r.v(R), r.sl(S_RR)));
    MTLGPU_TRY(r.scal(IDR_STEP));                                    // (++iter).finished(r)
    MTLGPU_TRY(idr_m_update(r, k, IDR_M_INIT));                      // M[iall][k] = trans(P) dR_k
  }
  std::vector<DotSpec> d;                                            // m = trans(P) * r
  for (int i = 0; i < s; i++) d.push_back({idr_p(r, i), r.v(R), r.dn(idr_m(s) + i)});
  return r.dots(d);
}
mtlgpu_status idr_record(Rec& r) {
  using namespace idr_v;
  XWork* W = r.W;
  const int s = W->param;
  MTLGPU_TRY(r.dot(r.v(R), r.v(R), r.sl(S_RR)));
  MTLGPU_TRY(r.scal(X_CHECK_RR));                                    // while (!finished(r))
  // `oldest` runs through 0 .. s-1 in every pass of the outer loop
  for (int k = 0; k < s; k++) {
    MTLGPU_TRY(r.scal(IDR_LU));                                      // c = lu_solve(M, m)
    std::vector<Term> q;
    for (int j = 0; j < s; j++) q.push_back(T(idr_dr(r, j), r.dn(idr_nc(s) + j)));
    MTLGPU_TRY(r.lin_n(r.v(Q), q));                                  // q = dR * -c
    MTLGPU_TRY(r.lin(r.v(V), {T(r.v(R)), T(r.v(Q))}));               // v = r + q
    if (k == 0) {
      MTLGPU_TRY(r.spmv(W->A, r.v(V), r.v(TV)));                      // t = A v
      MTLGPU_TRY(r.dots({{r.v(TV), r.v(V), r.sl(S_TV)}, {r.v(TV), r.v(TV), r.sl(S_TT)}}));
      MTLGPU_TRY(r.scal(IDR_OMEGA0));
      MTLGPU_TRY(r.lin(idr_dr(r, k), {T(r.v(Q)), T(r.v(TV), r.sl(S_NOMEGA))}));
    }
    std::vector<Term> dx{T(r.v(V), r.sl(S_OMEGA))};                  // dX_k = omega v - dX * c
    for (int j = 0; j < s; j++) dx.push_back(T(idr_dx(r, j), r.dn(idr_c(s) + j), -1.0));
    LinArgs a{};  // one launch: every dX_j is read before dX_k is written
    a.out = idr_dx(r, k);
    a.nt = (int)dx.size();
    for (int t = 0; t < a.nt; t++) a.t[t] = dx[t];
    xlin_kernel<<<W->grid, kBlock, 0, r.ctx->stream>>>(W->n, a, W->st);
    r.ctx->launches++;
    if (k != 0) {                                                    // dR_k = A * -dX_k
      MTLGPU_TRY(r.lin(r.v(TMP), {T(idr_dx(r, k), -1.0)}));
      MTLGPU_TRY(r.spmv(W->A, r.v(TMP), idr_dr(r, k)));
    }
    MTLGPU_TRY(r.lin(r.v(R), {T(r.v(R)), T(idr_dr(r, k))}));
    MTLGPU_TRY(r.lin(r.v(VX), {T(r.v(VX)), T(idr_dx(r, k))}));
    MTLGPU_TRY(r.dot(r.v(R), r.v(R), r.sl(S_RR)));
    MTLGPU_TRY(r.scal(IDR_STEP));                                    // (++iter).finished(r)
    MTLGPU_TRY(idr_m_update(r, k, IDR_M));                           // M[iall][k] = dm; m += dm
  }
  return MTLGPU_OK;
}

// ---- gmres: itl/krylov/gmres.hpp:34-135 ------------------------------------------------
// One recorded iteration is one restart cycle (gmres_full on an inner
// iteration limited to `restart` steps, then update_progress).
double* gm_vk(Rec& r, int k) { return r.v(gm_v::V0 + k); }
mtlgpu_status gmres_prologue(Rec& r) { return r.zero(r.W->dense, r.W->dense_n); }
mtlgpu_status gmres_record(Rec& r) {
  using namespace gm_v;
  XWork* W = r.W;
  const int m = W->param;
  xset_halt_kernel<<<1, 32, 0, r.ctx->stream>>>(W->st);
  r.ctx->launches++;
  MTLGPU_TRY(residual(r, r.v(VX), r.v(R0)));                        // r0(b - A x)
  MTLGPU_TRY(r.pc(W->L, r.v(R0), r.v(RV)));                          // r(solve(L, r0))
  MTLGPU_TRY(r.dot(r.v(RV), r.v(RV), r.sl(S_RR)));
  MTLGPU_TRY(r.scal(GM_START));                                      // rho = g[0] = two_norm(r)
  MTLGPU_TRY(r.lin(gm_vk(r, 0), {T(r.v(RV), r.sl(S_INV))}));         // V[0] = r / rho
  for (int k = 0; k < m; k++) {
    MTLGPU_TRY(r.scal(GM_STEP_BEGIN, k));
    MTLGPU_TRY(r.pc(W->R, gm_vk(r, k), r.v(Z)));                     // va0 = A solve(R, V[k])
    MTLGPU_TRY(r.spmv(W->A, r.v(Z), r.v(VA0)));
    MTLGPU_TRY(r.pc(W->L, r.v(VA0), gm_vk(r, k + 1)));               // V[k+1] = solve(L, va0)
    for (int j = 0; j <= k; j++) {                                   // modified Gram-Schmidt
      double* h = r.dn(j * m + k);
      MTLGPU_TRY(r.dot(gm_vk(r, j), gm_vk(r, k + 1), h));
      MTLGPU_TRY(r.lin(gm_vk(r, k + 1), {T(gm_vk(r, k + 1)), T(gm_vk(r, j), h, -1.0)}));
    }
    for (int j = 0; j <= k; j++) {                                   // reorthogonalise
      double* hr = r.dn(gm_hr(m) + j);
      MTLGPU_TRY(r.dot(gm_vk(r, k + 1), gm_vk(r, j), hr));
      MTLGPU_TRY(r.lin(gm_vk(r, k + 1), {T(gm_vk(r, k + 1)), T(gm_vk(r, j), hr, -1.0)}));
    }
    MTLGPU_TRY(r.dot(gm_vk(r, k + 1), gm_vk(r, k + 1), r.sl(S_RR)));
    MTLGPU_TRY(r.scal(GM_STEP_END, k));                              // H, Givens, ++iter
    MTLGPU_TRY(r.lin(gm_vk(r, k + 1), {T(gm_vk(r, k + 1), r.sl(S_INV))}));
  }
  MTLGPU_TRY(r.scal(GM_SOLVE));                                      // y = lu_solve(H, g)
  std::vector<Term> w;
  for (int j = 0; j < m; j++) w.push_back(T(gm_vk(r, j), r.dn(gm_y(m) + j)));
  MTLGPU_TRY(r.lin_n(r.v(WV), w));                                    // V[range] * y[range]
  MTLGPU_TRY(r.pc(W->R, r.v(WV), r.v(Z)));
  MTLGPU_TRY(r.lin(r.v(VX), {T(r.v(VX)), T(r.v(Z))}));               // x += solve(R, ...)
  MTLGPU_TRY(residual(r, r.v(VX), r.v(R0)));                        // r = b - A x
  MTLGPU_TRY(r.dot(r.v(R0), r.v(R0), r.sl(S_RR)));
  return r.scal(GM_END);                                             // terminate(r)
}

mtlgpu_status prologue(Rec& r) {
  switch (r.W->method) {
    case MTLGPU_BICG: return bicg_prologue(r);
    case MTLGPU_CGS: return cgs_prologue(r);
    case MTLGPU_BICGSTAB_2:
    case MTLGPU_BICGSTAB_ELL: return ell_prologue(r);
    case MTLGPU_TFQMR: return tfqmr_prologue(r);
    case MTLGPU_QMR: return qmr_prologue(r);
    case MTLGPU_IDR_S: return idr_prologue(r);
    case MTLGPU_GMRES: return gmres_prologue(r);
  }
  return MTLGPU_INVALID_ARG;
}
mtlgpu_status record(Rec& r) {
  switch (r.W->method) {
    case MTLGPU_BICG: return bicg_record(r);
    case MTLGPU_CGS: return cgs_record(r);
    case MTLGPU_BICGSTAB_2:
    case MTLGPU_BICGSTAB_ELL: return ell_record(r);
    case MTLGPU_TFQMR: return tfqmr_record(r);
    case MTLGPU_QMR: return qmr_record(r);
    case MTLGPU_IDR_S: return idr_record(r);
    case MTLGPU_GMRES: return gmres_record(r);
  }
  return MTLGPU_INVALID_ARG;
}

mtlgpu_status build_graph(Rec& r) {
  XWork* W = r.W;
  Ctx* ctx = r.ctx;
  if (W->exec) return MTLGPU_OK;
  cudaGraph_t g = nullptr;
  const long long before = ctx->launches;
  MTLGPU_TRY_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  mtlgpu_status s = MTLGPU_OK;
  for (int k = 0; k < graph_iters(W->method) && s == MTLGPU_OK; k++) s = record(r);
  cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
  ctx->launches = before;
  if (s != MTLGPU_OK) {
    if (g) cudaGraphDestroy(g);
    return s;
  }
  MTLGPU_TRY_CUDA(ctx, e);
  size_t nodes = 0;
  MTLGPU_TRY_CUDA(ctx, cudaGraphGetNodes(g, nullptr, &nodes));
  std::vector<cudaGraphNode_t> nv(nodes);
  if (nodes) MTLGPU_TRY_CUDA(ctx, cudaGraphGetNodes(g, nv.data(), &nodes));
  W->graph_nodes = 0;
  for (auto nd : nv) {
    cudaGraphNodeType ty;
    MTLGPU_TRY_CUDA(ctx, cudaGraphNodeGetType(nd, &ty));
    W->graph_nodes += ty == cudaGraphNodeTypeKernel;
  }
  e = cudaGraphInstantiate(&W->exec, g, 0);
  cudaGraphDestroy(g);
  MTLGPU_TRY_CUDA(ctx, e);
  return MTLGPU_OK;
}

void release_xwork_one(XWork* W) {
  Ctx* ctx = W->A->ctx;
  if (W->exec) cudaGraphExecDestroy(W->exec);
  for (double*& p : W->vec) dfree(ctx, p);
  dfree(ctx, W->st);
  dfree(ctx, W->dense);
  dfree(ctx, W->partials);
  dfree(ctx, W->counter);
  dfree(ctx, W->history);
  if (W->h_st) cudaFreeHost(W->h_st);
  if (W->AT) mtlgpu_csr_destroy(static_cast<mtlgpu_csr*>(W->AT));
  delete W;
}

mtlgpu_status create_xwork(Csr* A, Pc* L, Pc* R, int method, int param, XWork** out) {
  for (XWork* W : A->xwork)
    if (W->L == L && W->R == R && W->method == method && W->param == param) {
      *out = W;
      return MTLGPU_OK;
    }
  Ctx* ctx = A->ctx;
  XWork* W = new XWork();
  W->A = A, W->L = L, W->R = R, W->method = method, W->param = param, W->n = A->n_rows;
  W->grid = (int)std::max(1ll, std::min<long long>((W->n + kBlock - 1) / kBlock,
                                                   (long long)ctx->num_sms * 8));
  auto fail = [&](mtlgpu_status s) {
    release_xwork_one(W);
    return s;
  };
  W->vec.assign(vec_count(method, param), nullptr);
  for (double*& p : W->vec) {
    mtlgpu_status s = dalloc(ctx, &p, W->n);
    if (s != MTLGPU_OK) return fail(s);
  }
  W->dense_n = dense_len(method, param);
  mtlgpu_status s = MTLGPU_OK;
  if ((s = dalloc(ctx, &W->st, 1)) != MTLGPU_OK || (s = dalloc(ctx, &W->dense, W->dense_n)) ||
      (s = dalloc(ctx, &W->partials, W->grid)) || (s = dalloc(ctx, &W->counter, 1)))
    return fail(s);
  if (cudaMemsetAsync(W->counter, 0, sizeof(unsigned), ctx->stream) != cudaSuccess ||
      cudaMallocHost(reinterpret_cast<void**>(&W->h_st), sizeof(XState)) != cudaSuccess)
    return fail(set_cuda_error(ctx, cudaGetLastError(), "krylov workspace"));
  if (method == MTLGPU_BICG || method == MTLGPU_QMR) {
    mtlgpu_csr* T = nullptr;
    s = mtlgpu_csr_create_transpose(static_cast<mtlgpu_csr*>(A), &T);
    if (s != MTLGPU_OK) return fail(s);
    W->AT = T;
  }
  // adjoint sweeps are built outside stream capture
  if (method == MTLGPU_BICG && L && (s = pc_ensure_adjoint(L)) != MTLGPU_OK) return fail(s);
  if (method == MTLGPU_QMR) {
    if (L && (s = pc_ensure_adjoint(L)) != MTLGPU_OK) return fail(s);
    if (R && (s = pc_ensure_adjoint(R)) != MTLGPU_OK) return fail(s);
  }
  A->xwork.push_back(W);
  *out = W;
  return MTLGPU_OK;
}

}  // namespace

void release_xwork(Csr* A, const Pc* only_P) {
  std::vector<XWork*> keep;
  for (XWork* W : A->xwork) {
    if (only_P && W->L != only_P && W->R != only_P) {
      keep.push_back(W);
      continue;
    }
    release_xwork_one(W);
  }
  A->xwork = keep;
}

mtlgpu_status solve_krylov_impl(int method, Csr* A, Pc* L, Pc* R, int param, double* d_x,
                                const double* d_b, const mtlgpu_iter_params* prm,
                                mtlgpu_iter_result* res) {
  Ctx* ctx = A->ctx;
  std::memset(res, 0, sizeof(*res));
  if (A->n_rows != A->n_cols) return MTLGPU_NOT_SQUARE;
  if ((L && L->A != A) || (R && R->A != A)) return MTLGPU_INVALID_ARG;
  if (prm->mode != MTLGPU_SOLVE_FP64) return MTLGPU_NOT_SUPPORTED;
  for (Pc* P : {L, R})
    if (P && P->kind == MTLGPU_PC_IDENTITY) {  // identity: a copy, as no preconditioner
      if (P == L) L = nullptr;
      else R = nullptr;
    }
  for (Pc* P : {L, R})
    if (P && P->prec != MTLGPU_FP64) return MTLGPU_INVALID_ARG;
  switch (method) {  // the reference's defaults: l = 8, s = 8, restart = 8
    case MTLGPU_BICG:
    case MTLGPU_CGS:
    case MTLGPU_TFQMR:
    case MTLGPU_QMR:
      param = 0;
      break;
    case MTLGPU_BICGSTAB_2: param = 2; break;  // bicgstab_ell's loop with l = 2
    case MTLGPU_BICGSTAB_ELL: param = param > 0 ? param : 8; if (param > 32) return MTLGPU_INVALID_ARG; break;
    case MTLGPU_IDR_S: param = param > 0 ? param : 8; if (param > kMaxTerms - 1) return MTLGPU_INVALID_ARG; break;
    case MTLGPU_GMRES: param = param > 0 ? param : 8; if (param > 64) return MTLGPU_INVALID_ARG; break;
    default: return MTLGPU_INVALID_ARG;
  }
  if (method == MTLGPU_BICG || method == MTLGPU_CGS || method == MTLGPU_BICGSTAB_2) R = nullptr;
  if (method == MTLGPU_IDR_S) L = nullptr, R = nullptr;  // idr_s ignores both
  const int n = A->n_rows;
  if (n == 0 && method != MTLGPU_BICG && method != MTLGPU_CGS)
    return MTLGPU_INVALID_ARG;  // "empty rhs vector" (mtl::logic_error)
  if (n == 0) {
    res->norm_r0 = prm->norm_r0 < 0 ? 0.0 : prm->norm_r0;
    return MTLGPU_OK;
  }
  XWork* W = nullptr;
  MTLGPU_TRY(create_xwork(A, L, R, method, param, &W));
  Rec r{W, ctx};
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(W->vec[VX], d_x, sizeof(double) * n,
                                       cudaMemcpyDeviceToDevice, ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(W->vec[VB], d_b, sizeof(double) * n,
                                       cudaMemcpyDeviceToDevice, ctx->stream));
  // iteration state: basic_iteration(b or norm_r0, max_iter, rtol, atol)
  double norm_r0 = prm->norm_r0;
  if (norm_r0 < 0) {
    MTLGPU_TRY(dot_launch(ctx, n, d_b, d_b, ctx->d_scalars, 1));
    double nb2 = 0;
    MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(&nb2, ctx->d_scalars, sizeof(double),
                                         cudaMemcpyDeviceToHost, ctx->stream));
    MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    norm_r0 = std::sqrt(nb2);
  }
  const int per_iter = method == MTLGPU_BICGSTAB_ELL || method == MTLGPU_BICGSTAB_2
                           ? param + 3 : 3;
  const long long want = (long long)per_iter * ((long long)prm->max_iter + 2) + 16;
  const int cap = (int)std::min<long long>(want, 1 << 22);
  if (cap > W->hist_cap) {
    dfree(ctx, W->history);
    MTLGPU_TRY(dalloc(ctx, &W->history, cap));
    W->hist_cap = cap;
  }
  XState* h = W->h_st;
  std::memset(h, 0, sizeof(XState));
  h->max_iter = prm->max_iter;
  h->tol = prm->rtol * norm_r0;
  h->atol = prm->atol;
  h->norm_r0 = norm_r0;
  h->history = W->history;
  h->hist_cap = W->hist_cap;
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(W->st, h, sizeof(XState), cudaMemcpyHostToDevice,
                                       ctx->stream));
  MTLGPU_TRY(prologue(r));
  MTLGPU_TRY(r.sync_state());
  // tfqmr and qmr return straight from their first test (no shift back)
  const bool early = h->done && (method == MTLGPU_TFQMR || method == MTLGPU_QMR);
  bool interrupted = false;
  while (!h->done) {
    if (prm->h_interrupt && *prm->h_interrupt) {
      interrupted = true;
      break;
    }
    MTLGPU_TRY(build_graph(r));
    MTLGPU_TRY_CUDA(ctx, cudaGraphLaunch(W->exec, ctx->stream));
    ctx->launches += (long long)W->graph_nodes;
    int err = 0;
    MTLGPU_TRY(read_error_word(ctx, &err));
    MTLGPU_TRY(r.sync_state());
    if (err) break;
  }
  MTLGPU_TRY(take_device_error(ctx));
  if (!early && !interrupted) {
    // the epilogue's kernels run after the state has halted
    MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(&W->st->halt, 0, sizeof(int), ctx->stream));
    if (method == MTLGPU_BICGSTAB_ELL || method == MTLGPU_BICGSTAB_2) MTLGPU_TRY(ell_epilogue(r));
    if (method == MTLGPU_TFQMR) MTLGPU_TRY(tfqmr_epilogue(r));
  }
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(d_x, W->vec[VX], sizeof(double) * n,
                                       cudaMemcpyDeviceToDevice, ctx->stream));
  // true residual ||b - A x|| in FP64
  MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(&W->st->halt, 0, sizeof(int), ctx->stream));
  double* scratch = W->vec.back();
  MTLGPU_TRY(residual(r, W->vec[VX], scratch));
  MTLGPU_TRY(r.dot(scratch, scratch, r.sl(S_RR)));
  MTLGPU_TRY(r.sync_state());
  res->iterations = h->iter;
  res->error = h->error;
  res->resid = h->resid;
  res->norm_r0 = norm_r0;
  res->true_resid = std::sqrt(std::fabs(h->s[S_RR]));
  res->history_len = h->hist_len;
  if (prm->h_resid_history && prm->history_cap > 0) {
    const int m = std::min(std::min(h->hist_len, W->hist_cap), prm->history_cap);
    if (m > 0) {
      MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(prm->h_resid_history, W->history, sizeof(double) * m,
                                           cudaMemcpyDeviceToHost, ctx->stream));
      MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
  }
  res->status = interrupted ? MTLGPU_INTERRUPTED
                : (h->breakdown ? MTLGPU_BREAKDOWN : (h->error ? MTLGPU_MAX_ITER : MTLGPU_OK));
  return (mtlgpu_status)res->status;
}

}  // namespace mtlgpu
