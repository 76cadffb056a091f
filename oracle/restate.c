/* CPU restatement of the MTL4/ITL sparse iterative-solve path (see restate.h).
 * TEST INFRASTRUCTURE ONLY.  Compiled with -ffp-contract=off so that every
 * multiply and add rounds separately, as in the reference built for the
 * x86-64 baseline ISA. */
#include "restate.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* laplacian_setup(A, m, n): mtl/matrix/laplacian_setup.hpp:25-44.  Row
 * row = i*n + j holds 4 on the diagonal and -1 for each grid neighbour; the
 * inserter keeps each row sorted by column, so the CSR order is
 * row-n, row-1, row, row+1, row+n (those that exist). */
int or_laplacian_setup(unsigned m, unsigned n, int* rp, int* ci, double* v) {
  int nnz = 0;
  if (rp) rp[0] = 0;
  for (unsigned i = 0; i < m; i++)
    for (unsigned j = 0; j < n; j++) {
      unsigned row = i * n + j;
      int c[5];
      double w[5];
      int k = 0;
      if (i > 0) c[k] = (int)(row - n), w[k++] = -1.0;
      if (j > 0) c[k] = (int)(row - 1), w[k++] = -1.0;
      c[k] = (int)row, w[k++] = 4.0;
      if (j < n - 1) c[k] = (int)(row + 1), w[k++] = -1.0;
      if (i < m - 1) c[k] = (int)(row + n), w[k++] = -1.0;
      for (int t = 0; t < k; t++) {
        if (ci) ci[nnz] = c[t], v[nnz] = w[t];
        nnz++;
      }
      if (rp) rp[row + 1] = nnz;
    }
  return nnz;
}

/* smat_cvec_mult, mtl/operation/mat_vec_mult.hpp:620-689: per row a single
 * accumulator summed in column order, then Assign::first_update
 * (mode 0: y = t, 1: y += t, 2: y -= t; assign_mode.hpp). */
void or_spmv(int n, const int* rp, const int* ci, const double* v, const double* x, double* y,
             int mode) {
  for (int i = 0; i < n; i++) {
    double t = 0.0;
    for (int j = rp[i]; j < rp[i + 1]; j++) t += v[j] * x[ci[j]];
    if (mode == 0)
      y[i] = t;
    else if (mode == 1)
      y[i] += t;
    else
      y[i] -= t;
  }
}

/* sfunctor::dot<4>, mtl/operation/dot.hpp:98-152 (serial branch 136-147):
 * element i+o of each block of four goes to accumulator o, the tail to
 * accumulator 0, result ((t0+t1)+(t2+t3)) + ((t4+t5)+(t6+t7)) with t4..t7 = 0. */
double or_dot(int n, const double* x, const double* y) {
  double t[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int nb = n / 4 * 4;
  for (int i = 0; i < nb; i += 4) {
    t[0] += x[i] * y[i];
    t[1] += x[i + 1] * y[i + 1];
    t[2] += x[i + 2] * y[i + 2];
    t[3] += x[i + 3] * y[i + 3];
  }
  for (int i = nb; i < n; i++) t[0] += x[i] * y[i];
  return ((t[0] + t[1]) + (t[2] + t[3])) + ((t[4] + t[5]) + (t[6] + t[7]));
}

/* reduction<U, Functor>, mtl/vector/reduction.hpp:28-81,154-173: U
 * accumulators, tail into accumulator 0, finish folds from the right:
 * t0 + (t1 + (t2 + ... )). */
static double reduce_squares(int n, const double* x, int unroll) {
  double t[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int nb = n / unroll * unroll;
  for (int i = 0; i < nb; i += unroll)
    for (int o = 0; o < unroll; o++) t[o] += x[i + o] * x[i + o];
  for (int i = nb; i < n; i++) t[0] += x[i] * x[i];
  for (int o = unroll - 2; o >= 0; o--) t[o] += t[o + 1];
  return t[0];
}

/* two_norm<4>: mtl/operation/two_norm.hpp:33-57 with two_norm_functor
 * (mtl/vector/reduction_functors.hpp:53-80): sqrt of the 4-way reduction. */
double or_two_norm(int n, const double* x) { return sqrt(reduce_squares(n, x, 4)); }

/* unary_dot<8>: mtl/operation/unary_dot.hpp:29-65. */
double or_unary_dot(int n, const double* x) { return reduce_squares(n, x, 8); }

int or_upper_nnz(int n, const int* rp, const int* ci) {
  int c = 0;
  for (int i = 0; i < n; i++)
    for (int j = rp[i]; j < rp[i + 1]; j++) c += ci[j] >= i;
  return c;
}

int or_strict_lower_nnz(int n, const int* rp, const int* ci) {
  int c = 0;
  for (int i = 0; i < n; i++)
    for (int j = rp[i]; j < rp[i + 1]; j++) c += ci[j] < i;
  return c;
}

void or_transpose(int n, const int* rp, const int* ci, const double* v, int* trp, int* tci,
                  double* tv) {
  int nnz = rp[n];
  int* fill = (int*)calloc((size_t)n + 1, sizeof(int));
  memset(trp, 0, sizeof(int) * ((size_t)n + 1));
  for (int j = 0; j < nnz; j++) trp[ci[j] + 1]++;
  for (int i = 0; i < n; i++) trp[i + 1] += trp[i];
  for (int i = 0; i < n; i++)
    for (int j = rp[i]; j < rp[i + 1]; j++) {
      int c = ci[j];
      int pos = trp[c] + fill[c]++;
      tci[pos] = i;
      if (tv) tv[pos] = v[j];
    }
  free(fill);
}

static int find_in_row(const int* rp, const int* ci, int row, int col) {
  for (int j = rp[row]; j < rp[row + 1]; j++) {
    if (ci[j] == col) return j;
    if (ci[j] > col) break;
  }
  return -1;
}

static double round_float(double x, int as_float) { return as_float ? (double)(float)x : x; }

/* ic_0::factorizer::factorize, itl/pc/ic_0.hpp:136-186.
 * U = upper(A) (148).  For each row k: U(k,k) <- 1/sqrt(U(k,k)) (160-161);
 * each later entry U(k,i) <- d = U(k,i)*U(k,k) (164-168); the update loop
 * (170-182) visits the entries of row i of U with column in (k, i], which in
 * an upper factor is the diagonal alone, so it applies U(i,i) -= d*d.  L is
 * the CSR copy of trans(U) (57).  With as_float the factorisation still runs
 * in double and the result is rounded to float (122-130). */
int or_ic0(int n, const int* rp, const int* ci, const double* v, int as_float, int* Lrp, int* Lci,
           double* Lv, int* Urp, int* Uci, double* Uv) {
  int nu = 0;
  Urp[0] = 0;
  for (int i = 0; i < n; i++) {
    for (int j = rp[i]; j < rp[i + 1]; j++)
      if (ci[j] >= i) Uci[nu] = ci[j], Uv[nu] = v[j], nu++;
    Urp[i + 1] = nu;
  }
  for (int k = 0; k < n; k++) {
    int jk = Urp[k];
    if (jk == Urp[k + 1] || Uci[jk] != k) return -(k + 1);
    double inv = 1.0 / sqrt(Uv[jk]);
    Uv[jk] = inv;
    for (int j = jk + 1; j < Urp[k + 1]; j++) {
      double d = Uv[j] * inv;
      Uv[j] = d;
      int i = Uci[j];
      int di = Urp[i];
      if (di == Urp[i + 1] || Uci[di] != i) return -(i + 1);
      Uv[di] -= d * Uv[j];
    }
  }
  for (int j = 0; j < nu; j++) Uv[j] = round_float(Uv[j], as_float);
  or_transpose(n, Urp, Uci, Uv, Lrp, Lci, Lv);
  return 0;
}

/* ilu_0_factorizer::factorize, itl/pc/ilu_0.hpp:45-82 (IKJ, no fill):
 * for row i and each k < i in it (column order): a_ik <- a_ik * inv_dia[k]
 * (70-71), then every later entry a_ij of row i gets a_ij - a_ik * LU[k][j]
 * with LU[k][j] = 0 where (k, j) is not stored (73-74); inv_dia[i] = 1/a_ii
 * (77).  invert_diagonal (79; mtl/operation/invert_diagonal.hpp:47-54) then
 * stores the reciprocal on the diagonal; L = strict_lower, U = upper (80-81). */
int or_ilu0(int n, const int* rp, const int* ci, const double* v, int as_float, int* Lrp, int* Lci,
            double* Lv, int* Urp, int* Uci, double* Uv) {
  int nnz = rp[n];
  double* lu = (double*)malloc(sizeof(double) * (size_t)(nnz ? nnz : 1));
  double* inv_dia = (double*)calloc((size_t)n + 1, sizeof(double));
  memcpy(lu, v, sizeof(double) * (size_t)nnz);
  int status = 0;
  for (int i = 0; i < n; i++) {
    for (int kc = rp[i]; kc < rp[i + 1]; kc++) {
      int k = ci[kc];
      if (k == i) break;
      double aik = lu[kc] * inv_dia[k];
      lu[kc] = aik;
      for (int jc = kc + 1; jc < rp[i + 1]; jc++) {
        int p = find_in_row(rp, ci, k, ci[jc]);
        double ukj = p >= 0 ? lu[p] : 0.0;
        lu[jc] = lu[jc] - aik * ukj;
      }
    }
    int d = find_in_row(rp, ci, i, i);
    if (d < 0) {
      status = -(i + 1);
      break;
    }
    inv_dia[i] = 1.0 / lu[d];
  }
  if (status == 0) {
    for (int i = 0; i < n; i++) {
      int d = find_in_row(rp, ci, i, i);
      lu[d] = 1.0 / lu[d];
    }
    int nl = 0, nu = 0;
    Lrp[0] = Urp[0] = 0;
    for (int i = 0; i < n; i++) {
      for (int j = rp[i]; j < rp[i + 1]; j++) {
        if (ci[j] < i)
          Lci[nl] = ci[j], Lv[nl] = round_float(lu[j], as_float), nl++;
        else
          Uci[nu] = ci[j], Uv[nu] = round_float(lu[j], as_float), nu++;
      }
      Lrp[i + 1] = nl;
      Urp[i + 1] = nu;
    }
  }
  free(lu);
  free(inv_dia);
  return status;
}

/* lower_trisolve_t::apply(int_<5>), mtl/operation/lower_trisolve.hpp:173-189:
 * unit diagonal, strictly lower CSR. */
void or_lower_unit(int n, const int* rp, const int* ci, const double* v, const double* in,
                   double* out) {
  for (int r = 0; r < n; r++) {
    double rr = in[r];
    for (int j = rp[r]; j < rp[r + 1]; j++) rr -= v[j] * out[ci[j]];
    out[r] = rr;
  }
}

/* lower_trisolve_t::apply(int_<6>), lower_trisolve.hpp:192-209: inverted
 * diagonal stored last in each row. */
void or_lower_invdiag_last(int n, const int* rp, const int* ci, const double* v, const double* in,
                           double* out) {
  for (int r = 0; r < n; r++) {
    int j0 = rp[r], j1 = rp[r + 1] - 1;
    double dia = v[j1];
    double rr = in[r];
    for (; j0 != j1; j0++) rr -= v[j0] * out[ci[j0]];
    out[r] = rr * dia;
  }
}

/* upper_trisolve_t::apply(int_<3>), mtl/operation/upper_trisolve.hpp:160-176
 * with row_update for inverse_diagonal (101-103): inverted diagonal first. */
void or_upper_invdiag_first(int n, const int* rp, const int* ci, const double* v,
                            const double* in, double* out) {
  for (int r = n; r-- > 0;) {
    int j0 = rp[r], j1 = rp[r + 1];
    double rr = in[r];
    double dia = v[j0++];
    for (; j0 != j1; j0++) rr -= v[j0] * out[ci[j0]];
    out[r] = rr * dia;
  }
}

/* Column-oriented forward substitution used by adjoint solves
 * (lower_trisolve.hpp:155-170, version 4, on a transposed upper factor):
 * w = v; for column r: w[r] *= dia (first entry, inverted); then
 * w[row] -= value * w[r] for the rest of the column. */
static void lower_colwise_invdiag_first(int n, const int* crp, const int* cri, const double* cv,
                                        const double* in, double* out) {
  memcpy(out, in, sizeof(double) * (size_t)n);
  for (int r = 0; r < n; r++) {
    int j = crp[r];
    double rr = out[r] *= cv[j++];
    for (; j < crp[r + 1]; j++) out[cri[j]] -= cv[j] * rr;
  }
}

/* Column-oriented backward substitution with unit diagonal
 * (upper_trisolve.hpp:130-149, version 2, on a transposed strict-lower factor). */
static void upper_colwise_unit(int n, const int* crp, const int* cri, const double* cv,
                               const double* in, double* out) {
  memcpy(out, in, sizeof(double) * (size_t)n);
  for (int r = n; r-- > 0;) {
    double rr = out[r];
    for (int j = crp[r]; j < crp[r + 1]; j++) out[cri[j]] -= cv[j] * rr;
  }
}

int or_levels_lower(int n, const int* rp, const int* ci, int* level) {
  int nlev = 0;
  for (int r = 0; r < n; r++) {
    int l = 0;
    for (int j = rp[r]; j < rp[r + 1]; j++)
      if (ci[j] < r && level[ci[j]] + 1 > l) l = level[ci[j]] + 1;
    level[r] = l;
    if (l + 1 > nlev) nlev = l + 1;
  }
  return nlev;
}

int or_levels_upper(int n, const int* rp, const int* ci, int* level) {
  int nlev = 0;
  for (int r = n; r-- > 0;) {
    int l = 0;
    for (int j = rp[r]; j < rp[r + 1]; j++)
      if (ci[j] > r && level[ci[j]] + 1 > l) l = level[ci[j]] + 1;
    level[r] = l;
    if (l + 1 > nlev) nlev = l + 1;
  }
  return nlev;
}

/* ---------------------------------------------------------------------- */
/* Preconditioners (itl/pc/*.hpp) as objects for the solver restatements.  */

typedef struct {
  int kind, n;
  double* inv_diag;                     /* diagonal (diagonal.hpp:37-45) */
  int *Lrp, *Lci, *Urp, *Uci;           /* factors */
  double *Lv, *Uv;
  int *LTrp, *LTci, *UTrp, *UTci;       /* transposes for adjoint solves */
  double *LTv, *UTv;
  double* tmp;                          /* y0 of solve_lower */
} or_pc;

static void pc_free(or_pc* P) {
  free(P->inv_diag);
  free(P->Lrp), free(P->Lci), free(P->Lv), free(P->Urp), free(P->Uci), free(P->Uv);
  free(P->LTrp), free(P->LTci), free(P->LTv), free(P->UTrp), free(P->UTci), free(P->UTv);
  free(P->tmp);
  memset(P, 0, sizeof(*P));
}

static int pc_init(or_pc* P, int kind, int n, const int* rp, const int* ci, const double* v) {
  memset(P, 0, sizeof(*P));
  P->kind = kind;
  P->n = n;
  P->tmp = (double*)malloc(sizeof(double) * (size_t)(n ? n : 1));
  if (kind == OR_PC_DIAGONAL) {
    P->inv_diag = (double*)malloc(sizeof(double) * (size_t)(n ? n : 1));
    for (int i = 0; i < n; i++) {
      int d = find_in_row(rp, ci, i, i);
      P->inv_diag[i] = 1.0 / (d >= 0 ? v[d] : 0.0);
    }
    return 0;
  }
  if (kind == OR_PC_IDENTITY) return 0;
  int as_float = kind == OR_PC_ILU0_FLOAT || kind == OR_PC_IC0_FLOAT;
  int nl, nu;
  if (kind == OR_PC_IC0 || kind == OR_PC_IC0_FLOAT)
    nl = nu = or_upper_nnz(n, rp, ci);
  else
    nl = or_strict_lower_nnz(n, rp, ci), nu = or_upper_nnz(n, rp, ci);
  size_t sn = (size_t)n + 1;
  P->Lrp = (int*)malloc(sizeof(int) * sn), P->Urp = (int*)malloc(sizeof(int) * sn);
  P->Lci = (int*)malloc(sizeof(int) * (size_t)(nl + 1));
  P->Uci = (int*)malloc(sizeof(int) * (size_t)(nu + 1));
  P->Lv = (double*)malloc(sizeof(double) * (size_t)(nl + 1));
  P->Uv = (double*)malloc(sizeof(double) * (size_t)(nu + 1));
  int st;
  if (kind == OR_PC_IC0 || kind == OR_PC_IC0_FLOAT)
    st = or_ic0(n, rp, ci, v, as_float, P->Lrp, P->Lci, P->Lv, P->Urp, P->Uci, P->Uv);
  else
    st = or_ilu0(n, rp, ci, v, as_float, P->Lrp, P->Lci, P->Lv, P->Urp, P->Uci, P->Uv);
  if (st) return st;
  P->LTrp = (int*)malloc(sizeof(int) * sn), P->UTrp = (int*)malloc(sizeof(int) * sn);
  P->LTci = (int*)malloc(sizeof(int) * (size_t)(nl + 1));
  P->UTci = (int*)malloc(sizeof(int) * (size_t)(nu + 1));
  P->LTv = (double*)malloc(sizeof(double) * (size_t)(nl + 1));
  P->UTv = (double*)malloc(sizeof(double) * (size_t)(nu + 1));
  or_transpose(n, P->Lrp, P->Lci, P->Lv, P->LTrp, P->LTci, P->LTv);
  or_transpose(n, P->Urp, P->Uci, P->Uv, P->UTrp, P->UTci, P->UTv);
  return 0;
}

/* solve(P, r): ilu.hpp:74-91 (lower v5 then upper v3), ic_0.hpp:68-87
 * (lower v6 on L then upper v3 on U), diagonal.hpp:57-64, identity.
 * adjoint_solve: ilu.hpp:106-115 (U^T column-wise, then L^T column-wise),
 * ic_0.hpp:89-103 (same as solve). */
static void pc_apply(const or_pc* P, const double* r, double* z, int adjoint) {
  int n = P->n;
  switch (P->kind) {
    case OR_PC_IDENTITY:
      memcpy(z, r, sizeof(double) * (size_t)n);
      break;
    case OR_PC_DIAGONAL:
      for (int i = 0; i < n; i++) z[i] = P->inv_diag[i] * r[i];
      break;
    case OR_PC_IC0:
    case OR_PC_IC0_FLOAT:
      or_lower_invdiag_last(n, P->Lrp, P->Lci, P->Lv, r, P->tmp);
      or_upper_invdiag_first(n, P->Urp, P->Uci, P->Uv, P->tmp, z);
      break;
    default:
      if (!adjoint) {
        or_lower_unit(n, P->Lrp, P->Lci, P->Lv, r, P->tmp);
        or_upper_invdiag_first(n, P->Urp, P->Uci, P->Uv, P->tmp, z);
      } else {
        /* adjoint(U) is U^T viewed column-major: its columns are U's rows. */
        lower_colwise_invdiag_first(n, P->Urp, P->Uci, P->Uv, r, P->tmp);
        upper_colwise_unit(n, P->Lrp, P->Lci, P->Lv, P->tmp, z);
      }
  }
}

int or_pc_apply(int pc, int n, const int* rp, const int* ci, const double* v, const double* r,
                double* z, int adjoint) {
  or_pc P;
  int st = pc_init(&P, pc, n, rp, ci, v);
  if (st == 0) pc_apply(&P, r, z, adjoint);
  pc_free(&P);
  return st;
}

/* ---------------------------------------------------------------------- */
/* basic_iteration, itl/iteration/basic_iteration.hpp:24-164.              */
typedef struct {
  int error, i, max_iter;
  double norm_r0, rtol, atol, resid;
  double* hist;
  int cap, count;
} or_iter;

static int iter_finished(or_iter* it, double r) {
  if (it->hist && it->count < it->cap) it->hist[it->count] = r;
  it->count++;
  it->resid = r;
  int conv = it->norm_r0 == 0 ? r <= it->atol : (r <= it->rtol * it->norm_r0 || r <= it->atol);
  if (conv) return 1;
  if (it->i >= it->max_iter) {
    it->error = 1;
    return 1;
  }
  return 0;
}

/* Fused CG loop bodies (mtl/operation/fused_expr.hpp:57-77 with
 * row_mat_cvec_index_evaluator and dot_index_evaluator /
 * reduction_index_evaluator): four partial sums by i mod 4, tail into
 * partial 0. */
static double fused_spmv_dot(int n, const int* rp, const int* ci, const double* v, const double* p,
                             double* q) {
  double t[4] = {0, 0, 0, 0};
  int nb = n >> 2 << 2;
  for (int i = 0; i < n; i++) {
    double s = 0.0;
    for (int j = rp[i]; j < rp[i + 1]; j++) s += v[j] * p[ci[j]];
    q[i] = s;
    t[i < nb ? (i & 3) : 0] += p[i] * q[i];
  }
  return t[0] + t[1] + t[2] + t[3];
}

static double fused_axpy_unary_dot(int n, double alpha, const double* q, double* r) {
  double t[4] = {0, 0, 0, 0};
  int nb = n >> 2 << 2;
  for (int i = 0; i < n; i++) {
    r[i] -= alpha * q[i];
    t[i < nb ? (i & 3) : 0] += r[i] * r[i];
  }
  t[0] += t[1];
  t[2] += t[3];
  t[0] += t[2];
  return t[0];
}

/* itl::cg, itl/krylov/cg.hpp:39-72 (identity) and 75-112 (preconditioned). */
static int cg_restated(const or_pc* P, int n, const int* rp, const int* ci, const double* v,
                       const double* b, double* x, or_iter* it) {
  size_t sz = sizeof(double) * (size_t)(n ? n : 1);
  double *p = (double*)malloc(sz), *q = (double*)malloc(sz), *r = (double*)malloc(sz),
         *z = (double*)malloc(sz);
  double rho = 0, rho_1 = 0, rr, alpha, alpha_1;
  or_spmv(n, rp, ci, v, x, q, 0);
  for (int i = 0; i < n; i++) r[i] = b[i] - q[i];
  if (P->kind == OR_PC_IDENTITY) {
    rho = or_dot(n, r, r);
    while (!iter_finished(it, sqrt(fabs(rho)))) {
      ++it->i;
      if (it->i <= 1)
        memcpy(p, r, sz);
      else {
        double beta = rho / rho_1;
        for (int i = 0; i < n; i++) p[i] = r[i] + beta * p[i];
      }
      alpha_1 = fused_spmv_dot(n, rp, ci, v, p, q);
      alpha = rho / alpha_1;
      for (int i = 0; i < n; i++) x[i] += alpha * p[i];
      rho_1 = rho;
      rho = fused_axpy_unary_dot(n, alpha, q, r);
    }
  } else {
    rr = or_dot(n, r, r);
    while (!iter_finished(it, sqrt(fabs(rr)))) {
      ++it->i;
      pc_apply(P, r, z, 0);
      rho = or_dot(n, r, z);
      if (it->i <= 1)
        memcpy(p, z, sz);
      else {
        double beta = rho / rho_1;
        for (int i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
      }
      alpha_1 = fused_spmv_dot(n, rp, ci, v, p, q);
      alpha = rho / alpha_1;
      for (int i = 0; i < n; i++) x[i] += alpha * p[i];
      rho_1 = rho;
      rr = fused_axpy_unary_dot(n, alpha, q, r);
    }
  }
  free(p), free(q), free(r), free(z);
  return it->error;
}

/* itl::bicgstab, itl/krylov/bicgstab.hpp:27-78 (unfused).  Returns -2 where
 * the reference throws unexpected_orthogonality (46, 51, 59). */
static int bicgstab_restated(const or_pc* P, int n, const int* rp, const int* ci, const double* v,
                             const double* b, double* x, or_iter* it) {
  size_t sz = sizeof(double) * (size_t)(n ? n : 1);
  double *p = (double*)malloc(sz), *phat = (double*)malloc(sz), *s = (double*)malloc(sz),
         *shat = (double*)malloc(sz), *t = (double*)malloc(sz), *vv = (double*)malloc(sz),
         *r = (double*)malloc(sz), *rt = (double*)malloc(sz);
  double rho_1 = 0, rho_2 = 0, alpha = 0, beta = 0, gamma, omega = 0;
  int ret = 0;
  or_spmv(n, rp, ci, v, x, t, 0);
  for (int i = 0; i < n; i++) r[i] = b[i] - t[i];
  memcpy(rt, r, sz);
  while (!iter_finished(it, or_two_norm(n, r))) {
    ++it->i;
    rho_1 = or_dot(n, rt, r);
    if (rho_1 == 0.0) { ret = -2; goto done; }
    if (it->i <= 1)
      memcpy(p, r, sz);
    else {
      if (omega == 0.0) { ret = -2; goto done; }
      beta = (rho_1 / rho_2) * (alpha / omega);
      for (int i = 0; i < n; i++) p[i] = r[i] + beta * (p[i] - omega * vv[i]);
    }
    pc_apply(P, p, phat, 0);
    or_spmv(n, rp, ci, v, phat, vv, 0);
    gamma = or_dot(n, rt, vv);
    if (gamma == 0.0) { ret = -2; goto done; }
    alpha = rho_1 / gamma;
    for (int i = 0; i < n; i++) s[i] = r[i] - alpha * vv[i];
    if (iter_finished(it, or_two_norm(n, s))) {
      for (int i = 0; i < n; i++) x[i] += alpha * phat[i];
      break;
    }
    pc_apply(P, s, shat, 0);
    or_spmv(n, rp, ci, v, shat, t, 0);
    omega = or_dot(n, t, s) / or_dot(n, t, t);
    for (int i = 0; i < n; i++) x[i] += omega * shat[i] + alpha * phat[i];
    for (int i = 0; i < n; i++) r[i] = s[i] - omega * t[i];
    rho_2 = rho_1;
  }
  ret = it->error;
done:
  free(p), free(phat), free(s), free(shat), free(t), free(vv), free(r), free(rt);
  return ret;
}

int or_solve(int method, int pc, int n, const int* rp, const int* ci, const double* v,
             const double* b, double* x, int max_iter, double rtol, double atol, double norm_r0,
             double* hist, int hist_cap, double* out) {
  or_pc P;
  int st = pc_init(&P, pc, n, rp, ci, v);
  if (st) {
    pc_free(&P);
    return -3;
  }
  or_iter it;
  memset(&it, 0, sizeof(it));
  it.max_iter = max_iter;
  it.rtol = rtol;
  it.atol = atol;
  it.norm_r0 = norm_r0 < 0 ? or_two_norm(n, b) : norm_r0;
  it.hist = hist;
  it.cap = hist_cap;
  int err = method == 0 ? cg_restated(&P, n, rp, ci, v, b, x, &it)
                        : bicgstab_restated(&P, n, rp, ci, v, b, x, &it);
  if (out) {
    out[0] = it.i;
    out[1] = it.resid;
    out[2] = it.norm_r0;
    out[3] = 0;
    out[4] = 0;
    out[5] = it.count;
  }
  pc_free(&P);
  return err;
}

/* Assembly through mtl::mat::inserter<compressed2D, Updater>
 * (mtl/matrix/compressed2D.hpp:662-1151).  Each row is kept as a sorted
 * (column, value) list, the union of the inserter's slot and spare map.
 * modify() (947-989) looks the entry up: present -> the updater of
 * update.hpp:26-111 (0 store x = y, 1 plus x += y, 2 minus x -= y, 3 times
 * x *= y); absent -> inserted with init(y) (minus: -y, else y).  The matrix
 * starts as the base CSR (stretch(), 864-914, keeps its entries); triplet k
 * uses ops[k] when ops != NULL, else `updater`.  Output: rp (n_rows+1), ci, v
 * with room for base_nnz + count entries; returns nnz, or -1 for an index
 * out of range (the reference's "Index is out of range!"). */
typedef struct {
  int n, cap;
  int* c;
  double* v;
} or_row;

int or_assemble(int n_rows, int n_cols, int base_nnz, const int* brp, const int* bci,
                const double* bv, long long count, const int* rows, const int* cols,
                const double* vals, const unsigned char* ops, int updater, int* rp, int* ci,
                double* v) {
  or_row* R = (or_row*)calloc(n_rows > 0 ? (size_t)n_rows : 1, sizeof(or_row));
  int ret = 0;
  if (!R) return -2;
  for (int r = 0; r < n_rows && base_nnz > 0; r++) {
    const int len = brp[r + 1] - brp[r];
    R[r].cap = len > 4 ? len : 4;
    R[r].c = (int*)malloc(sizeof(int) * (size_t)R[r].cap);
    R[r].v = (double*)malloc(sizeof(double) * (size_t)R[r].cap);
    for (int j = 0; j < len; j++) R[r].c[j] = bci[brp[r] + j], R[r].v[j] = bv[brp[r] + j];
    R[r].n = len;
  }
  for (long long k = 0; k < count; k++) {
    const int r = rows[k], c = cols[k];
    const int op = ops ? (int)ops[k] : updater;
    if (r < 0 || r >= n_rows || c < 0 || c >= n_cols) {
      ret = -1;
      break;
    }
    or_row* w = &R[r];
    int lo = 0, hi = w->n;            /* first position with column >= c */
    while (lo < hi) {
      const int mid = (lo + hi) / 2;
      if (w->c[mid] < c) lo = mid + 1;
      else hi = mid;
    }
    if (lo < w->n && w->c[lo] == c) {
      double* x = &w->v[lo];
      if (op == 1) *x = *x + vals[k];
      else if (op == 2) *x = *x - vals[k];
      else if (op == 3) *x = *x * vals[k];
      else *x = vals[k];
      continue;
    }
    if (w->n == w->cap) {
      w->cap = w->cap ? 2 * w->cap : 4;
      w->c = (int*)realloc(w->c, sizeof(int) * (size_t)w->cap);
      w->v = (double*)realloc(w->v, sizeof(double) * (size_t)w->cap);
    }
    memmove(w->c + lo + 1, w->c + lo, sizeof(int) * (size_t)(w->n - lo));
    memmove(w->v + lo + 1, w->v + lo, sizeof(double) * (size_t)(w->n - lo));
    w->c[lo] = c;
    w->v[lo] = op == 2 ? -vals[k] : vals[k];
    w->n++;
  }
  if (ret == 0) {
    int nnz = 0;
    rp[0] = 0;
    for (int r = 0; r < n_rows; r++) {
      for (int j = 0; j < R[r].n; j++) ci[nnz] = R[r].c[j], v[nnz] = R[r].v[j], nnz++;
      rp[r + 1] = nnz;
    }
    ret = nnz;
  }
  for (int r = 0; r < n_rows; r++) free(R[r].c), free(R[r].v);
  free(R);
  return ret;
}
