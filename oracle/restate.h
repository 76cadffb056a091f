/* CPU restatement of the MTL4/ITL sparse iterative-solve path in plain C.
 *
 * TEST INFRASTRUCTURE ONLY: the checker the GPU library is compared against.
 * Nothing in the shipped library links or calls this code.  Each function
 * follows the reference loop it names (file:line inside the MTL4 tree), in the
 * same loop order and floating-point accumulation order, so that its results
 * can be pinned bit-for-bit against the reference compiled from its own
 * headers (oracle/_ref/libmtlref.so).
 *
 * CSR arrays: rp[n+1], ci[nnz], v[nnz]; rows sorted by column, no duplicates.
 */
#ifndef MTLGPU_ORACLE_RESTATE_H
#define MTLGPU_ORACLE_RESTATE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Preconditioner kinds (same numbering as the reference driver). */
enum { OR_PC_IDENTITY = 0, OR_PC_DIAGONAL = 1, OR_PC_ILU0 = 2, OR_PC_IC0 = 3,
       OR_PC_ILU0_FLOAT = 4, OR_PC_IC0_FLOAT = 5 };

int or_laplacian_setup(unsigned m, unsigned n, int* rp, int* ci, double* v);
void or_spmv(int n, const int* rp, const int* ci, const double* v, const double* x, double* y,
             int mode);
double or_dot(int n, const double* x, const double* y);
double or_two_norm(int n, const double* x);
double or_unary_dot(int n, const double* x);

/* Factor extraction: sizes first (pass NULL arrays), then fill. */
int or_upper_nnz(int n, const int* rp, const int* ci);
int or_strict_lower_nnz(int n, const int* rp, const int* ci);

/* IC(0): U (n, nnz_u) with inverted diagonal first, L = U^T with inverted
 * diagonal last.  Returns 0, or a negative row-(1+index) on a missing diagonal. */
int or_ic0(int n, const int* rp, const int* ci, const double* v, int as_float, int* Lrp, int* Lci,
           double* Lv, int* Urp, int* Uci, double* Uv);
/* ILU(0): L strict lower (unit diagonal implicit), U upper, inverted diagonal first. */
int or_ilu0(int n, const int* rp, const int* ci, const double* v, int as_float, int* Lrp, int* Lci,
            double* Lv, int* Urp, int* Uci, double* Uv);

/* Triangular sweeps (lower_trisolve.hpp:173-209, upper_trisolve.hpp:160-176). */
void or_lower_unit(int n, const int* rp, const int* ci, const double* v, const double* in,
                   double* out);
void or_lower_invdiag_last(int n, const int* rp, const int* ci, const double* v, const double* in,
                           double* out);
void or_upper_invdiag_first(int n, const int* rp, const int* ci, const double* v,
                            const double* in, double* out);

/* Level sets of a factor pattern: level[r] = 0 without off-diagonal entries,
 * else 1 + max level over the off-diagonal columns (below the diagonal for a
 * lower factor, above it for an upper one).  Returns the number of levels. */
int or_levels_lower(int n, const int* rp, const int* ci, int* level);
int or_levels_upper(int n, const int* rp, const int* ci, int* level);

/* CSR transpose (stable: rows of the result sorted by column). */
void or_transpose(int n, const int* rp, const int* ci, const double* v, int* trp, int* tci,
                  double* tv);

/* Preconditioner apply z = solve(P, r) / adjoint_solve(P, r). */
int or_pc_apply(int pc, int n, const int* rp, const int* ci, const double* v, const double* r,
                double* z, int adjoint);

/* itl::cg (method 0) / itl::bicgstab (method 1) with basic_iteration control.
 * Same argument meaning as ref_solve in the reference driver. */
int or_solve(int method, int pc, int n, const int* rp, const int* ci, const double* v,
             const double* b, double* x, int max_iter, double rtol, double atol, double norm_r0,
             double* hist, int hist_cap, double* out);

/* Assembly through mtl::mat::inserter (compressed2D.hpp:662-1151) from a base
 * CSR plus coordinate triplets; ops[k] (or `updater` for all) is 0 store,
 * 1 plus, 2 minus, 3 times.  Returns nnz, -1 on an index out of range. */
int or_assemble(int n_rows, int n_cols, int base_nnz, const int* brp, const int* bci,
                const double* bv, long long count, const int* rows, const int* cols,
                const double* vals, const unsigned char* ops, int updater, int* rp, int* ci,
                double* v);

#ifdef __cplusplus
}
#endif
#endif
