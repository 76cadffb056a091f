// Preconditioned CG with the IC(0) / ILU(0) factors applied by Jacobi
// iterations (jacobi_sweep.cu), in three kernels per iteration instead of
// five.
//
// itl::cg (itl/krylov/cg.hpp:75-112) runs, per iteration,
//     z = solve(P, r); rho = dot(r, z); p = z + (rho / rho_1) p;
//     q = A p; alpha = rho / dot(p, q); x += alpha p; r -= alpha q;
//     ++iter; test ||r||.
// The unfused recording (krylov.cu) makes that L pass, U pass + rho, p
// update, SpMV + p.q, update + r.r.  Here the two vector kernels go into
// their neighbours:
//   K_A  x += alpha p, r' = r - alpha q, r'.r', ++iter and the termination
//        test (last block), and the first Jacobi pass of the L triangle on
//        r', whose gathers form r'[c] = r[c] - alpha q[c] on the fly;
//   K_B  the remaining passes, the U triangle and rho = r'.z (unchanged);
//   K_C  p' = z + beta p formed on the fly at every gathered column, written
//        for the own row, q = A p' and p'.q (last block: alpha_1).
// r and p are double-buffered (the kernels that write r' and p' gather the
// old vectors), x is updated in place (row-local).  Every value of r' and
// p' is produced by one helper, so a gathered value and the stored one are
// the same bits: the iteration computes what the unfused one computes, in
// fewer passes over HBM (per iteration on the 128^3 Laplacian, FP32: r, q,
// p, z each read once less, two launches and one grid reduction fewer).
// The first iteration's front half (z, rho, p = z, q, alpha_1) is a
// prologue run once before the graph.
//
// itl::bicgstab (itl/krylov/bicgstab.hpp:27-78) with Jacobi-applied factors
// takes two pieces from here: K_A in its BiCGSTAB form (s = r - alpha v,
// ||s|| and the half-step test, fused into the first L pass of
// shat = solve(M, s)) and bicg_tprod_kernel (t = A shat with omega's dots
// t.s and t.t).  The product kernel K_C is also the C-ABI operation
// mtlgpu_cg_direction_product.
#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "device.cuh"
#include "internal.h"
#include "solver_state.cuh"

namespace mtlgpu {

using namespace dev;

namespace {

constexpr int kBlock = 256;
// Resident blocks per SM.  K_A makes two gathers per entry: 6 (40
// registers) in FP32, 4 in FP64 (no spills).  K_C holds 8 entries' gathers
// in flight: in FP32 6 blocks (40 registers) measured best on the 128^3
// mixed solve (18.57 ms; 5 blocks 18.91, 4 entries per batch: 19.5-20.6);
// in FP64 5 blocks (48 registers, no spills).
template <typename T>
constexpr int min_blocks_a() { return sizeof(T) == 4 ? 6 : 4; }
template <typename T>
constexpr int min_blocks_c() { return sizeof(T) == 4 ? 6 : 5; }

int rows_grid(Ctx* ctx, long long n, int per_sm) {
  const long long need = (n + kBlock - 1) / kBlock;
  const long long cap = (long long)ctx->num_sms * per_sm;
  return (int)std::max(1ll, std::min(need, cap));
}

__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fma_t(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return __fma_rn(a, b, c); }

// r' = r - alpha q (the one formula for stored and gathered values)
template <typename T>
__device__ __forceinline__ T next_r(T r, T q, T alpha) {
  return fma_t(-alpha, q, r);
}
// p' = z + beta p
template <typename T>
__device__ __forceinline__ T next_p(T z, T p, T beta) {
  return fma_t(beta, p, z);
}

// Column index of entry k of this lane's row in a SELL-32 slice.
template <bool D16>
__device__ __forceinline__ int sell_col(const int32_t* __restrict__ col,
                                        const int16_t* __restrict__ dcol, int o, int row,
                                        bool in) {
  if (D16) {
    const int d = in ? (int)__ldlu(dcol + o) : -32768;
    return d == -32768 ? -1 : row + d;
  }
  return in ? __ldlu(col + o) : -1;
}

// K_A.  The Jacobi pass is jacobi_pass_kernel's (same chunking, same
// accumulation), with v = r' and its gathers formed from r and q.
// BICG: the same kernel makes BiCGSTAB's s = r - alpha v (q = v, r_next = s,
// no x update; alpha = rho / gamma) with ||s||^2 and the half-step test of
// bicgstab.hpp:58-67 (bicg_s_kernel's), fused into the first L pass of
// shat = solve(M, s).
template <typename T, bool SCALE, int C, bool D16, bool BICG>
__global__ void __launch_bounds__(kBlock, min_blocks_a<T>())
    cg_lupd_kernel(int n, const int32_t* __restrict__ slice_ptr, const int32_t* __restrict__ col,
                   const int16_t* __restrict__ dcol, const T* __restrict__ val,
                   const T* __restrict__ dinv, T* __restrict__ x, const T* __restrict__ p,
                   const T* __restrict__ r, const T* __restrict__ q, T* __restrict__ r_next,
                   T* __restrict__ out, SolverState* st, void* partials, unsigned* counter) {
  if (st->done) return;
  typedef typename AccOf<T, 1>::type R;
  const double gamma = st->gamma;
  const T alpha = (T)(BICG ? st->rho / gamma : st->rho / st->alpha_1);
  R acc_rr = R::zero();
  for (long long rl = gtid(); rl < n; rl += gstride()) {
    const int row = (int)rl;
    const int lane = row & 31;
    const int s = row >> 5;
    const int base = __ldg(slice_ptr + s);
    const int width = (__ldg(slice_ptr + s + 1) - base) >> 5;
    const T rv = next_r(__ldg(r + row), __ldg(q + row), alpha);
    const T dr = SCALE ? __ldg(dinv + row) : T(1);
    r_next[row] = rv;
    if (!BICG) x[row] = fma_t(alpha, __ldg(p + row), x[row]);
    acc_rr.add_prod(0, rv, rv);
    T acc = T(0);
    for (int k0 = 0; k0 < width; k0 += C) {
      int c[C];
      T a[C], g[C];
#pragma unroll
      for (int u = 0; u < C; u++) {
        const bool in = k0 + u < width;
        const int o = base + 32 * (k0 + u) + lane;
        c[u] = sell_col<D16>(col, dcol, o, row, in);
        a[u] = in ? __ldlu(val + o) : T(0);
      }
#pragma unroll
      for (int u = 0; u < C; u++)
        g[u] = c[u] >= 0 ? next_r(__ldg(r + c[u]), __ldg(q + c[u]), alpha) : T(0);
#pragma unroll
      for (int u = 0; u < C; u++) acc += a[u] * g[u];
    }
    T res = rv - acc;
    if (SCALE) res *= dr;
    out[row] = res;
  }
  R bs = block_reduce(acc_rr);
  R* parts = reinterpret_cast<R*>(partials);
  if (publish_partial(bs, parts, blockIdx.x, counter, gridDim.x)) {
    R tot = reduce_partials(parts, gridDim.x);
    if (threadIdx.x == 0) {
      if (BICG) {
        if (gamma == 0.0) {
          st->status = MTLGPU_BREAKDOWN;
          st->done = 1;
          st->skip2 = 1;
        } else {
          st->alpha_1 = st->rho / gamma;  // alpha
          st->ss = tot.value(0);
          if (iter_finished(st, sqrt(st->ss))) {
            st->half_exit = 1;
            st->skip2 = 1;
          }
        }
      } else {
        const double rr = tot.value(0);
        st->iter++;
        st->rho_1 = st->rho;
        st->rr = rr;
        if (iter_finished(st, sqrt(fabs(rr)))) st->done = 1;
      }
    }
  }
}

// K_C.  The product is spmv_sell's (stored order, products and sums rounded
// separately) on x = p'; FIRST: p' = z (the first iteration).  beta is
// num / den read from device memory (the solve's rho / rho_1), or
// beta_value when num is null; p'.q goes to *pq.
template <typename T, int C, bool D16, bool FIRST>
__global__ void __launch_bounds__(kBlock, min_blocks_c<T>())
    cg_pspmv_kernel(int n, const int32_t* __restrict__ slice_ptr, const int32_t* __restrict__ col,
                    const int16_t* __restrict__ dcol, const T* __restrict__ val,
                    const T* __restrict__ z, const T* __restrict__ p, T* __restrict__ p_next,
                    T* __restrict__ q, const int* skip, const double* num, const double* den,
                    double beta_value, double* pq, void* partials, unsigned* counter) {
  if (skip && *skip) return;
  typedef typename AccOf<T, 1>::type R;
  const T beta = FIRST ? T(0) : (T)(num ? *num / *den : beta_value);
  R acc_pq = R::zero();
  for (long long rl = gtid(); rl < n; rl += gstride()) {
    const int row = (int)rl;
    const int lane = row & 31;
    const int s = row >> 5;
    const int base = __ldg(slice_ptr + s);
    const int width = (__ldg(slice_ptr + s + 1) - base) >> 5;
    const T pr = FIRST ? __ldg(z + row) : next_p(__ldg(z + row), __ldg(p + row), beta);
    p_next[row] = pr;
    T sum = T(0);
    for (int k0 = 0; k0 < width; k0 += C) {
      int c[C];
      T a[C], g[C];
#pragma unroll
      for (int u = 0; u < C; u++) {
        const bool in = k0 + u < width;
        const int o = base + 32 * (k0 + u) + lane;
        c[u] = sell_col<D16>(col, dcol, o, row, in);
        a[u] = in ? __ldlu(val + o) : T(0);
      }
#pragma unroll
      for (int u = 0; u < C; u++) {
        if (c[u] < 0)
          g[u] = T(0);
        else
          g[u] = FIRST ? __ldg(z + c[u]) : next_p(__ldg(z + c[u]), __ldg(p + c[u]), beta);
      }
#pragma unroll
      for (int u = 0; u < C; u++)
        if (c[u] >= 0) sum = add_rn(sum, mul_rn(a[u], g[u]));
    }
    q[row] = sum;
    acc_pq.add_prod(0, pr, sum);
  }
  R bs = block_reduce(acc_pq);
  R* parts = reinterpret_cast<R*>(partials);
  if (publish_partial(bs, parts, blockIdx.x, counter, gridDim.x)) {
    R tot = reduce_partials(parts, gridDim.x);
    if (threadIdx.x == 0) *pq = tot.value(0);
  }
}

template <typename T>
struct Vals;
template <>
struct Vals<double> {
  static const double* val(const Sell& S) { return S.d_val; }
  static const double* dinv(const Sell& S) { return S.d_dinv; }
  static double* tmp(Pc* P) { return P->d_tmp; }
  static double* jtmp(Pc* P) { return P->d_jtmp; }
};
template <>
struct Vals<float> {
  static const float* val(const Sell& S) { return S.d_val32; }
  static const float* dinv(const Sell& S) { return S.d_dinv32; }
  static float* tmp(Pc* P) { return P->d_tmp32; }
  static float* jtmp(Pc* P) { return P->d_jtmp32; }
};

// 16-bit column offsets wherever the SELL-32 copy has them.  Measured on the
// 128^3 mixed solve (FP32): 18.88 ms with offsets in both kernels, 18.94
// with them in the factor pass only, 19.3-19.5 with neither; unlike the
// plain FP32 SpMV (spmv.cu), the product with its second gather per entry
// gains from the smaller index.
bool product_d16(const Sell& S) { return S.d_dcol != nullptr; }

// BiCGSTAB's t = A shat with omega's two dots, t.s and t.t (bicgstab.hpp:
// 69-70), in one pass: the product is spmv_sell's; the dots replace the
// separate omega kernel of the unfused recording (their blocking differs
// from that kernel's, so omega may differ in its last bits: used only with
// Jacobi-applied factors, whose solves are not held to the reference's
// iteration counts).
template <typename T, int C, bool D16>
__global__ void __launch_bounds__(kBlock, min_blocks_c<T>())
    bicg_tprod_kernel(int n, const int32_t* __restrict__ slice_ptr,
                      const int32_t* __restrict__ col, const int16_t* __restrict__ dcol,
                      const T* __restrict__ val, const T* __restrict__ shat,
                      const T* __restrict__ s, T* __restrict__ t, SolverState* st, void* partials,
                      unsigned* counter) {
  if (st->done || st->skip2) return;
  typedef typename AccOf<T, 2>::type R;
  R acc = R::zero();
  for (long long rl = gtid(); rl < n; rl += gstride()) {
    const int row = (int)rl;
    const int lane = row & 31;
    const int sl = row >> 5;
    const int base = __ldg(slice_ptr + sl);
    const int width = (__ldg(slice_ptr + sl + 1) - base) >> 5;
    T sum = T(0);
    for (int k0 = 0; k0 < width; k0 += C) {
      int c[C];
      T a[C], g[C];
#pragma unroll
      for (int u = 0; u < C; u++) {
        const bool in = k0 + u < width;
        const int o = base + 32 * (k0 + u) + lane;
        c[u] = sell_col<D16>(col, dcol, o, row, in);
        a[u] = in ? __ldlu(val + o) : T(0);
      }
#pragma unroll
      for (int u = 0; u < C; u++) g[u] = c[u] >= 0 ? __ldg(shat + c[u]) : T(0);
#pragma unroll
      for (int u = 0; u < C; u++)
        if (c[u] >= 0) sum = add_rn(sum, mul_rn(a[u], g[u]));
    }
    t[row] = sum;
    acc.add_prod(0, sum, __ldg(s + row));
    acc.add_prod(1, sum, sum);
  }
  R bs = block_reduce(acc);
  R* parts = reinterpret_cast<R*>(partials);
  if (publish_partial(bs, parts, blockIdx.x, counter, gridDim.x)) {
    R tot = reduce_partials(parts, gridDim.x);
    if (threadIdx.x == 0) {
      st->ts = tot.value(0);
      st->tt = tot.value(1);
    }
  }
}

struct BetaSrc {
  const int* skip;
  const double *num, *den;  // beta = *num / *den, or value when num is null
  double value;
  double* pq;
};

template <typename T, bool FIRST>
void launch_pspmv(Ctx* ctx, const Sell& S, const T* val, const T* z, const T* p, T* p_next, T* q,
                  const BetaSrc& b) {
  const int grid = rows_grid(ctx, S.n, min_blocks_c<T>());
  unsigned* ctr = counter_slot(ctx, 11);
  if (product_d16(S))
    cg_pspmv_kernel<T, 8, true, FIRST><<<grid, kBlock, 0, ctx->stream>>>(
        S.n, S.d_slice_ptr, S.d_col, S.d_dcol, val, z, p, p_next, q, b.skip, b.num, b.den,
        b.value, b.pq, ctx->d_partials, ctr);
  else
    cg_pspmv_kernel<T, 8, false, FIRST><<<grid, kBlock, 0, ctx->stream>>>(
        S.n, S.d_slice_ptr, S.d_col, S.d_dcol, val, z, p, p_next, q, b.skip, b.num, b.den,
        b.value, b.pq, ctx->d_partials, ctr);
  ctx->launches++;
}

BetaSrc state_beta(SolverState* st) {
  return BetaSrc{&st->done, &st->rho, &st->rho_1, 0.0, &st->alpha_1};
}

template <typename T, bool SCALE, int C, bool BICG>
void launch_lupd_c(Ctx* ctx, const Sell& L, const T* val, const T* dinv, T* x, const T* p,
                   const T* r, const T* q, T* r_next, T* out, SolverState* st) {
  const int grid = rows_grid(ctx, L.n, min_blocks_a<T>());
  unsigned* ctr = counter_slot(ctx, 10);
  if (L.d_dcol)
    cg_lupd_kernel<T, SCALE, C, true, BICG><<<grid, kBlock, 0, ctx->stream>>>(
        L.n, L.d_slice_ptr, L.d_col, L.d_dcol, val, dinv, x, p, r, q, r_next, out, st,
        ctx->d_partials, ctr);
  else
    cg_lupd_kernel<T, SCALE, C, false, BICG><<<grid, kBlock, 0, ctx->stream>>>(
        L.n, L.d_slice_ptr, L.d_col, L.d_dcol, val, dinv, x, p, r, q, r_next, out, st,
        ctx->d_partials, ctr);
  ctx->launches++;
}

template <typename T, bool SCALE, bool BICG>
void launch_lupd(Ctx* ctx, const Sell& L, const T* val, const T* dinv, T* x, const T* p,
                 const T* r, const T* q, T* r_next, T* out, SolverState* st) {
  if (L.max_width <= 4)
    launch_lupd_c<T, SCALE, 4, BICG>(ctx, L, val, dinv, x, p, r, q, r_next, out, st);
  else
    launch_lupd_c<T, SCALE, 8, BICG>(ctx, L, val, dinv, x, p, r, q, r_next, out, st);
}

// The first L pass of solve(M, v') where v' = v0 - alpha w is formed in the
// pass (CG: r' and the x update; BiCGSTAB: s), then the remaining passes
// and the U triangle; the U triangle's last pass reduces dot_with . z into
// *dot_out when dot_with is given.  skip2: the passes after the first skip
// on it (BiCGSTAB's half-step exit), else on done.
template <typename T, bool BICG>
mtlgpu_status fused_apply(Ctx* ctx, Pc* P, SolverState* st, T* x, const T* p, const T* v0,
                          const T* w, T* v_next, T* z, const int* skip_rest, const T* dot_with,
                          double* dot_out) {
  const int k = P->jacobi_iters;
  const Sell& L = P->jac_lower;
  T* tmp = Vals<T>::tmp(P);
  T* scratch = Vals<T>::jtmp(P);
  // pass 0 of the L triangle writes where jacobi_solve would: tmp when it is
  // the only pass (k odd), else scratch
  T* out0 = (k % 2 == 1) ? tmp : scratch;
  const T* val = Vals<T>::val(L);
  const T* dinv = Vals<T>::dinv(L);
  if (k == 1 && !L.unit_diag)
    launch_lupd<T, true, BICG>(ctx, L, val, dinv, x, p, v0, w, v_next, out0, st);
  else
    launch_lupd<T, false, BICG>(ctx, L, val, dinv, x, p, v0, w, v_next, out0, st);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  if (k > 1) MTLGPU_TRY(jacobi_solve_from<T>(ctx, L, k, 1, v_next, tmp, scratch, skip_rest));
  MTLGPU_TRY(jacobi_solve<T>(ctx, P->jac_upper, k, tmp, z, scratch, skip_rest, dot_with,
                             dot_out));
  return MTLGPU_OK;
}

}  // namespace

// The fused recording needs A's SELL-32 copy (the product walks its slices)
// and Jacobi-applied IC(0) / ILU(0) factors.  MTLGPU_CG_FUSED=0 keeps the
// five-kernel recording.
bool cg_fused_eligible(Csr* A, Pc* P, int prec) {
  if (const char* e = std::getenv("MTLGPU_CG_FUSED"))
    if (!std::strcmp(e, "0")) return false;
  if (!P || (P->kind != MTLGPU_PC_IC0 && P->kind != MTLGPU_PC_ILU0) || P->jacobi_iters <= 0)
    return false;
  if (A->n_rows == 0 || A->spmv_kernel != 2 || !A->sell.d_slice_ptr) return false;
  const Sell& L = P->jac_lower;
  if (!L.d_slice_ptr || (!L.unit_diag && !L.col_scaled)) return false;
  if (prec == MTLGPU_FP32)
    return A->sell.d_val32 && L.d_val32 && P->jac_upper.d_val32 && P->d_tmp32 && P->d_jtmp32 &&
           (L.unit_diag || L.d_dinv32);
  return A->sell.d_val && L.d_val && P->jac_upper.d_val && P->d_tmp && P->d_jtmp &&
         (L.unit_diag || L.d_dinv);
}

template <typename T>
mtlgpu_status cg_fused_prologue(Csr* A, Pc* P, SolverState* st, const T* r, T* z, T* p, T* q) {
  Ctx* ctx = A->ctx;
  MTLGPU_TRY(pc_apply_t<T>(P, r, z, false, &st->done, false, false, &st->rho));
  launch_pspmv<T, true>(ctx, A->sell, Vals<T>::val(A->sell), z, nullptr, p, q, state_beta(st));
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  return MTLGPU_OK;
}

template <typename T>
mtlgpu_status cg_fused_iteration(Csr* A, Pc* P, SolverState* st, T* x, const T* r, T* r_next,
                                 const T* p, T* p_next, T* z, T* q) {
  Ctx* ctx = A->ctx;
  MTLGPU_TRY((fused_apply<T, false>(ctx, P, st, x, p, r, q, r_next, z, &st->done, r_next,
                                    &st->rho)));
  launch_pspmv<T, false>(ctx, A->sell, Vals<T>::val(A->sell), z, p, p_next, q, state_beta(st));
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  return MTLGPU_OK;
}

// BiCGSTAB: s = r - alpha v with ||s|| and the half-step test in the first
// L pass of shat = solve(M, s); the later passes skip on skip2.
template <typename T>
mtlgpu_status bicg_fused_s_apply(Csr* A, Pc* P, SolverState* st, const T* r, const T* v, T* s,
                                 T* shat) {
  return fused_apply<T, true>(A->ctx, P, st, nullptr, nullptr, r, v, s, shat, &st->skip2,
                              nullptr, nullptr);
}

template mtlgpu_status bicg_fused_s_apply<double>(Csr*, Pc*, SolverState*, const double*,
                                                  const double*, double*, double*);
template mtlgpu_status bicg_fused_s_apply<float>(Csr*, Pc*, SolverState*, const float*,
                                                 const float*, float*, float*);

template <typename T>
mtlgpu_status bicg_t_product(Csr* A, SolverState* st, const T* shat, const T* s, T* t) {
  Ctx* ctx = A->ctx;
  const Sell& S = A->sell;
  const T* val = Vals<T>::val(S);
  const int grid = rows_grid(ctx, S.n, min_blocks_c<T>());
  unsigned* ctr = counter_slot(ctx, 12);
  if (product_d16(S))
    bicg_tprod_kernel<T, 8, true><<<grid, kBlock, 0, ctx->stream>>>(
        S.n, S.d_slice_ptr, S.d_col, S.d_dcol, val, shat, s, t, st, ctx->d_partials, ctr);
  else
    bicg_tprod_kernel<T, 8, false><<<grid, kBlock, 0, ctx->stream>>>(
        S.n, S.d_slice_ptr, S.d_col, S.d_dcol, val, shat, s, t, st, ctx->d_partials, ctr);
  ctx->launches++;
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  return MTLGPU_OK;
}

template mtlgpu_status bicg_t_product<double>(Csr*, SolverState*, const double*, const double*,
                                              double*);
template mtlgpu_status bicg_t_product<float>(Csr*, SolverState*, const float*, const float*,
                                             float*);

// p' = z + beta p (p' = z when p is null), q = A p', *d_pq = p'.q: the
// product kernel of the fused CG on its own (mtlgpu_cg_direction_product).
template <typename T>
mtlgpu_status cg_direction_product(Csr* A, const T* z, double beta, const T* p, T* p_next, T* q,
                                   double* d_pq) {
  Ctx* ctx = A->ctx;
  if (A->n_rows == 0) return MTLGPU_OK;
  if (A->spmv_kernel != 2 || !A->sell.d_slice_ptr) return MTLGPU_NOT_SUPPORTED;
  const T* val = Vals<T>::val(A->sell);
  if (!val) return MTLGPU_INVALID_ARG;
  const BetaSrc b{nullptr, nullptr, nullptr, beta, d_pq};
  if (p)
    launch_pspmv<T, false>(ctx, A->sell, val, z, p, p_next, q, b);
  else
    launch_pspmv<T, true>(ctx, A->sell, val, z, nullptr, p_next, q, b);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  return MTLGPU_OK;
}

template mtlgpu_status cg_direction_product<double>(Csr*, const double*, double, const double*,
                                                    double*, double*, double*);
template mtlgpu_status cg_direction_product<float>(Csr*, const float*, double, const float*,
                                                   float*, float*, double*);
template mtlgpu_status cg_fused_prologue<double>(Csr*, Pc*, SolverState*, const double*, double*,
                                                 double*, double*);
template mtlgpu_status cg_fused_prologue<float>(Csr*, Pc*, SolverState*, const float*, float*,
                                                float*, float*);
template mtlgpu_status cg_fused_iteration<double>(Csr*, Pc*, SolverState*, double*, const double*,
                                                  double*, const double*, double*, double*,
                                                  double*);
template mtlgpu_status cg_fused_iteration<float>(Csr*, Pc*, SolverState*, float*, const float*,
                                                 float*, const float*, float*, float*, float*);

}  // namespace mtlgpu
