// Preconditioner set-up on the device: Jacobi, IC(0), ILU(0), and apply.
//
// Arithmetic follows the reference operation by operation, with every
// multiply and subtract rounded separately (__dmul_rn/__dsub_rn: no FMA
// contraction) and IEEE division and square root, so the factors are
// bit-identical to MTL4's for the same input:
//  * IC(0) (itl/pc/ic_0.hpp:136-186).  As written, the update loop of row k
//    touches only the diagonal of each later row i (the entries of row i of
//    the upper factor with column in (k, i] are the diagonal alone):
//      inv_k  = 1 / sqrt(a_kk - sum_{m<k, (m,k) in U} d_mk^2)  (m ascending)
//      d_mk   = a_mk * inv_m,  U(k,k) = inv_k,  U(k,i) = d_ki,
//    and L is the CSR copy of trans(U) (ic_0.hpp:57).  The dependency graph of
//    inv is the pattern of L, so inv is computed in L's level order, sync-free.
//  * ILU(0) (itl/pc/ilu_0.hpp:45-82): IKJ per row in column order with
//    lookups LU[k][j] that read 0 where (k, j) is not stored; inv_dia[i] =
//    1/LU(i,i); invert_diagonal (mtl/operation/invert_diagonal.hpp:47-54); L =
//    strict_lower, U = upper (ilu_0.hpp:80-81).  A row depends on the rows of
//    its strict-lower pattern; rows are factorised one warp each in that
//    pattern's level order, waiting on per-row completion flags.
//  * diagonal (itl/pc/diagonal.hpp:37-45): inv_diag[i] = 1 / A[i][i].
#include <algorithm>
#include <cmath>

#include "device.cuh"
#include "internal.h"

namespace mtlgpu {

using namespace dev;

// Exclusive prefix sum of int32 on the context's stream (analysis.cu).
mtlgpu_status scan_i32(Ctx* ctx, const int32_t* in, int32_t* out, int n);

namespace {

constexpr int kBlock = 256;

int grid_cap(Ctx* ctx, long long count, int per_block = kBlock) {
  long long need = (count + per_block - 1) / per_block;
  long long cap = (long long)ctx->num_sms * 8;
  return (int)std::max(1ll, std::min(need, cap));
}

__device__ __forceinline__ bool bad_pivot(double x) { return !(x != 0.0) || !isfinite(x); }

__global__ void jacobi_kernel(int n, const int32_t* __restrict__ diag,
                              const double* __restrict__ v, double* inv, float* inv32) {
  for (long long i = gtid(); i < n; i += gstride()) {
    const int d = diag[i];
    const double a = d >= 0 ? v[d] : 0.0;  // A[i][i] reads 0 where not stored
    const double r = __ddiv_rn(1.0, a);
    // float storage (diagonal<M, float>): both copies hold the float value
    inv[i] = inv32 ? (double)(float)r : r;
    if (inv32) inv32[i] = (float)r;
  }
}

// Reverses the entries of every row in place.
__global__ void reverse_rows_kernel(int n, const int32_t* __restrict__ rp, int32_t* ci,
                                    double* v) {
  for (long long r = gtid(); r < n; r += gstride()) {
    for (int a = rp[r], b = rp[r + 1] - 1; a < b; a++, b--) {
      const int32_t tc = ci[a];
      ci[a] = ci[b];
      ci[b] = tc;
      const double tv = v[a];
      v[a] = v[b];
      v[b] = tv;
    }
  }
}

__global__ void check_diag_kernel(int n, const int32_t* __restrict__ diag, int* err) {
  for (long long i = gtid(); i < n; i += gstride())
    if (diag[i] < 0) atomicCAS(err, 0, (int)MTLGPU_MISSING_DIAGONAL);
}

// upper(A): count / copy entries with column >= row.
__global__ void upper_count_kernel(int n, const int32_t* __restrict__ rp,
                                   const int32_t* __restrict__ ci, int32_t* cnt) {
  for (long long r = gtid(); r < n; r += gstride()) {
    int c = 0;
    for (int j = rp[r]; j < rp[r + 1]; j++) c += ci[j] >= r;
    cnt[r] = c;
  }
}
__global__ void upper_copy_kernel(int n, const int32_t* __restrict__ rp,
                                  const int32_t* __restrict__ ci, const double* __restrict__ v,
                                  const int32_t* __restrict__ urp, int32_t* uci, double* uv) {
  for (long long r = gtid(); r < n; r += gstride()) {
    int o = urp[r];
    for (int j = rp[r]; j < rp[r + 1]; j++)
      if (ci[j] >= r) uci[o] = ci[j], uv[o] = v[j], o++;
  }
}

// IC(0) inverse diagonal in L's level order.  Plan rows are L rows: the
// off-diagonal entries (columns m < k, ascending) carry a_mk, dinv carries
// a_kk.  Lane l of a G-group holds entries l, l+G, ...; the squares d_mk^2
// are folded into s sequentially in ascending m, as the reference applies
// its updates.
template <int G>
__global__ void __launch_bounds__(kBlock)
    ic0_inv_kernel(int n_tasks, const int32_t* __restrict__ task_ptr,
                   const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                   const double* __restrict__ a_off, const double* __restrict__ a_diag,
                   const int32_t* __restrict__ row_of, double* inv, unsigned* ticket, int* err,
                   int* pivot, long long limit) {
  const int lane = threadIdx.x & 31;
  const int sub = lane / G, gl = lane % G;
  const int base = sub * G;
  while (true) {
    unsigned t = 0;
    if (lane == 0) t = atomicAdd(ticket, 1u);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= (unsigned)n_tasks) break;
    const int p = task_ptr[t] + sub;
    const bool valid = p < task_ptr[t + 1];
    int b = 0, e = 0, row = 0;
    double s = 0.0;
    if (valid) {
      row = row_of[p];
      b = rp[p];
      e = rp[p + 1];
      s = a_diag[p];
    }
    // uniform pass count across the warp (shuffles need every lane)
    int passes = valid ? (e - b + G - 1) / G : 0;
    for (int off = 16; off > 0; off >>= 1) passes = max(passes, __shfl_xor_sync(0xffffffffu, passes, off));
    for (int ps = 0; ps < passes; ps++) {
      const int j = b + ps * G + gl;
      double sq = 0.0;
      if (valid && j < e) {
        const int m = ci[j];
        const double d = __dmul_rn(a_off[j], wait_value(inv + m, limit, err));
        sq = __dmul_rn(d, d);
      }
      for (int q = 0; q < G; q++) {
        const double v = __shfl_sync(0xffffffffu, sq, base + q);
        if (valid && b + ps * G + q < e) s = __dsub_rn(s, v);
      }
    }
    if (valid && gl == 0) {
      const double r = __ddiv_rn(1.0, __dsqrt_rn(s));
      if (!(s > 0.0) || !isfinite(r)) atomicCAS(pivot, 0, (int)MTLGPU_ZERO_PIVOT);
      st_relaxed(inv + row, canonical(r));
    }
  }
}

// Final IC(0) values: U(k,k) = inv_k, U(k,i) = a_ki * inv_k; L = trans(U):
// L(k,m) = a_mk * inv_m (same product), L(k,k) = inv_k (last in the row).
__global__ void ic0_values_kernel(int n, const int32_t* __restrict__ urp,
                                  const int32_t* __restrict__ uci, double* uv,
                                  const int32_t* __restrict__ lrp, const int32_t* __restrict__ lci,
                                  double* lv, const double* __restrict__ inv) {
  for (long long k = gtid(); k < n; k += gstride()) {
    const double ik = inv[k];
    const int ub = urp[k], ue = urp[k + 1];
    uv[ub] = ik;
    for (int j = ub + 1; j < ue; j++) uv[j] = __dmul_rn(uv[j], ik);
    const int lb = lrp[k], le = lrp[k + 1];
    for (int j = lb; j < le - 1; j++) lv[j] = __dmul_rn(lv[j], inv[lci[j]]);
    lv[le - 1] = ik;
  }
}

// Strict-lower counts of A (the ILU dependency pattern).
__global__ void lower_count_kernel(int n, const int32_t* __restrict__ rp,
                                   const int32_t* __restrict__ ci, int32_t* cnt, bool strict) {
  for (long long r = gtid(); r < n; r += gstride()) {
    int c = 0;
    for (int j = rp[r]; j < rp[r + 1]; j++) c += strict ? (ci[j] < r) : (ci[j] >= r);
    cnt[r] = c;
  }
}
__global__ void split_kernel(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                             const double* __restrict__ v, const int32_t* __restrict__ lrp,
                             int32_t* lci, double* lv, const int32_t* __restrict__ urp,
                             int32_t* uci, double* uv) {
  for (long long r = gtid(); r < n; r += gstride()) {
    int ol = lrp[r], ou = urp[r];
    for (int j = rp[r]; j < rp[r + 1]; j++) {
      if (ci[j] < r) {
        lci[ol] = ci[j];
        if (lv) lv[ol] = v[j];
        ol++;
      } else {
        uci[ou] = ci[j];
        if (uv) uv[ou] = v[j];
        ou++;
      }
    }
  }
}

// Binary search of column c in row k of A's pattern; -1 if absent.
__device__ __forceinline__ int find_col(const int32_t* __restrict__ ci, int b, int e, int c) {
  while (b < e) {
    const int m = (b + e) >> 1;
    const int v = ci[m];
    if (v == c) return m;
    if (v < c) b = m + 1; else e = m;
  }
  return -1;
}

// Pivot rows of at most this many entries are searched in shared memory.
constexpr int kIluRowCache = 64;

// ILU(0), one warp per row, rows in level order of the strict-lower pattern.
// lu holds A's values in A's CSR layout and is updated in place.  For each
// pivot row k of row i the warp loads row k's columns and (final) values
// into its shared buffer with one coalesced pass, and every lane finds its
// column there by binary search: one global round trip per pivot instead of
// a chain of dependent global loads per lane.  The arithmetic and its order
// are unchanged (longer pivot rows are searched in global memory).
__global__ void __launch_bounds__(kBlock)
    ilu0_kernel(int n_tasks, const int32_t* __restrict__ task_ptr,
                const int32_t* __restrict__ row_of, const int32_t* __restrict__ rp,
                const int32_t* __restrict__ ci, const int32_t* __restrict__ diag, double* lu,
                double* inv_dia, int* done, unsigned* ticket, int* err, int* pivot,
                long long limit) {
  __shared__ int32_t row_col[kBlock / 32][kIluRowCache];
  __shared__ double row_val[kBlock / 32][kIluRowCache];
  const int lane = threadIdx.x & 31;
  const int wid = threadIdx.x >> 5;
  while (true) {
    unsigned t = 0;
    if (lane == 0) t = atomicAdd(ticket, 1u);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= (unsigned)n_tasks) break;
    for (int p = task_ptr[t]; p < task_ptr[t + 1]; p++) {
      const int i = row_of[p];
      const int b = rp[i], e = rp[i + 1];
      if (e - b <= 32) {
        // the row in registers (lane q holds entry b + q) for the whole
        // elimination; the same operations in the same order as below
        const int len = e - b;
        const int mycol = lane < len ? __ldg(ci + b + lane) : 0x7fffffff;
        double my = lane < len ? lu[b + lane] : 0.0;
        for (int kq = 0; kq < len; kq++) {
          const int k = __shfl_sync(0xffffffffu, mycol, kq);
          if (k == i) break;
          if (lane == 0) {
            long long spins = 0;
            while (ld_acquire(done + k) == 0) {
              if (++spins >= limit) {
                atomicCAS(err, 0, (int)MTLGPU_TIMEOUT);
                break;
              }
              if ((spins & 1023) == 0 && ld_relaxed(err) != 0) break;
            }
          }
          __syncwarp();
          const double aik = __dmul_rn(__shfl_sync(0xffffffffu, my, kq), __ldcg(inv_dia + k));
          if (lane == kq) my = aik;
          const int kb = rp[k], ke = rp[k + 1];
          const bool upd = lane > kq && lane < len;
          if (ke - kb <= kIluRowCache) {
            for (int q = lane; q < ke - kb; q += 32) {
              row_col[wid][q] = __ldg(ci + kb + q);
              row_val[wid][q] = __ldcg(lu + kb + q);
            }
            __syncwarp();
            if (upd) {
              const int pos = find_col(row_col[wid], 0, ke - kb, mycol);
              my = __dsub_rn(my, __dmul_rn(aik, pos >= 0 ? row_val[wid][pos] : 0.0));
            }
          } else if (upd) {
            const int pos = find_col(ci, kb, ke, mycol);
            my = __dsub_rn(my, __dmul_rn(aik, pos >= 0 ? __ldcg(lu + pos) : 0.0));
          }
          __syncwarp();
        }
        if (lane < len) lu[b + lane] = my;
        const int d = diag[i];
        const double dv = __shfl_sync(0xffffffffu, my, d >= b && d < e ? d - b : 0);
        __syncwarp();
        if (lane == 0) {
          const double piv = d >= 0 ? dv : 0.0;
          if (bad_pivot(piv)) atomicCAS(pivot, 0, (int)MTLGPU_ZERO_PIVOT);
          inv_dia[i] = __ddiv_rn(1.0, piv);
          __threadfence();
          st_release(done + i, 1);
        }
        __syncwarp();
        continue;
      }
      for (int kc = b; kc < e; kc++) {
        const int k = ci[kc];
        if (k == i) break;
        // wait until row k is final (flag published after its values)
        if (lane == 0) {
          long long spins = 0;
          while (ld_acquire(done + k) == 0) {
            if (++spins >= limit) {
              atomicCAS(err, 0, (int)MTLGPU_TIMEOUT);
              break;
            }
            if ((spins & 1023) == 0 && ld_relaxed(err) != 0) break;
          }
        }
        __syncwarp();
        const double aik = __dmul_rn(lu[kc], __ldcg(inv_dia + k));
        __syncwarp();
        if (lane == 0) lu[kc] = aik;
        const int kb = rp[k], ke = rp[k + 1];
        if (ke - kb <= kIluRowCache) {
          for (int q = lane; q < ke - kb; q += 32) {
            row_col[wid][q] = __ldg(ci + kb + q);
            row_val[wid][q] = __ldcg(lu + kb + q);
          }
          __syncwarp();
          for (int jc = kc + 1 + lane; jc < e; jc += 32) {
            const int pos = find_col(row_col[wid], 0, ke - kb, ci[jc]);
            const double ukj = pos >= 0 ? row_val[wid][pos] : 0.0;
            lu[jc] = __dsub_rn(lu[jc], __dmul_rn(aik, ukj));
          }
        } else {
          for (int jc = kc + 1 + lane; jc < e; jc += 32) {
            const int pos = find_col(ci, kb, ke, ci[jc]);
            const double ukj = pos >= 0 ? __ldcg(lu + pos) : 0.0;
            lu[jc] = __dsub_rn(lu[jc], __dmul_rn(aik, ukj));
          }
        }
        __syncwarp();
      }
      if (lane == 0) {
        const int d = diag[i];
        const double piv = d >= 0 ? lu[d] : 0.0;
        if (bad_pivot(piv)) atomicCAS(pivot, 0, (int)MTLGPU_ZERO_PIVOT);
        inv_dia[i] = __ddiv_rn(1.0, piv);
        __threadfence();
        st_release(done + i, 1);
      }
      __syncwarp();
    }
  }
}

// invert_diagonal + split into L (strict lower) and U (upper) values.
__global__ void ilu0_split_kernel(int n, const int32_t* __restrict__ rp,
                                  const int32_t* __restrict__ ci, const double* __restrict__ lu,
                                  const int32_t* __restrict__ diag, const int32_t* __restrict__ lrp,
                                  double* lv, const int32_t* __restrict__ urp, double* uv) {
  for (long long r = gtid(); r < n; r += gstride()) {
    int ol = lrp[r], ou = urp[r];
    const int d = diag[r];
    for (int j = rp[r]; j < rp[r + 1]; j++) {
      if (ci[j] < r)
        lv[ol++] = lu[j];
      else
        uv[ou++] = (j == d) ? __ddiv_rn(1.0, lu[j]) : lu[j];
    }
  }
}

template <typename T>
__global__ void jacobi_apply_kernel(int n, const T* __restrict__ inv, const T* __restrict__ r,
                                    T* __restrict__ z, const int* skip) {
  if (skip && ld_relaxed(skip)) return;
  for (long long i = gtid(); i < n; i += gstride()) z[i] = inv[i] * r[i];
}

template <typename T>
__global__ void copy_kernel(int n, const T* __restrict__ r, T* __restrict__ z, const int* skip) {
  if (skip && ld_relaxed(skip)) return;
  for (long long i = gtid(); i < n; i += gstride()) z[i] = r[i];
}

__global__ void refill_plan_kernel(int n, const int32_t* __restrict__ row_of,
                                   const int32_t* __restrict__ frp, const double* __restrict__ fv,
                                   bool unit_diag, bool diag_last, const int32_t* __restrict__ prp,
                                   double* pv, double* dinv) {
  for (long long t = gtid(); t < n; t += gstride()) {
    const int r = row_of[t];
    int b = frp[r], e = frp[r + 1];
    if (!unit_diag) {
      const int d = diag_last ? e - 1 : b;
      dinv[t] = fv[d];
      if (diag_last) e--; else b++;
    }
    int o = prp[t];
    for (int j = b; j < e; j++, o++) pv[o] = fv[j];
  }
}


mtlgpu_status read_pivot(Ctx* ctx, int* d_pivot, int* status) {
  int h = 0;
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(&h, d_pivot, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  MTLGPU_TRY(take_device_error(ctx));
  *status = h;
  return MTLGPU_OK;
}

// Rebuilds a plan's values from a factor with the same pattern.
mtlgpu_status refill_plan(Ctx* ctx, SweepPlan* P, const int32_t* frp, const double* fv,
                          bool diag_last) {
  if (P->n == 0) return MTLGPU_OK;
  refill_plan_kernel<<<grid_cap(ctx, P->n), kBlock, 0, ctx->stream>>>(
      P->n, P->d_row_of, frp, fv, P->unit_diag, diag_last, P->d_rp, P->d_val, P->d_dinv);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  return MTLGPU_OK;
}

mtlgpu_status build_ic0(Pc* P) {
  Csr* A = P->A;
  Ctx* ctx = A->ctx;
  const int n = A->n_rows;
  // U pattern and values = upper(A)
  int32_t* d_cnt = nullptr;
  MTLGPU_TRY(dalloc(ctx, &d_cnt, n + 1));
  MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(d_cnt, 0, sizeof(int32_t) * (n + 1), ctx->stream));
  upper_count_kernel<<<grid_cap(ctx, n), kBlock, 0, ctx->stream>>>(n, A->d_rp, A->d_ci, d_cnt);
  MTLGPU_TRY(dalloc(ctx, &P->d_Urp, n + 1));
  MTLGPU_TRY(scan_i32(ctx, d_cnt, P->d_Urp, n + 1));
  dfree(ctx, d_cnt);
  int nu = 0;
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(&nu, P->d_Urp + n, sizeof(int), cudaMemcpyDeviceToHost,
                                       ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  P->nnz_U = P->nnz_L = nu;
  MTLGPU_TRY(dalloc(ctx, &P->d_Uci, nu));
  MTLGPU_TRY(dalloc(ctx, &P->d_Uv, nu));
  upper_copy_kernel<<<grid_cap(ctx, n), kBlock, 0, ctx->stream>>>(n, A->d_rp, A->d_ci, A->d_v,
                                                                  P->d_Urp, P->d_Uci, P->d_Uv);
  // L = trans(U) pattern, carrying a_mk (diagonal a_kk last)
  MTLGPU_TRY(dalloc(ctx, &P->d_Lrp, n + 1));
  MTLGPU_TRY(dalloc(ctx, &P->d_Lci, nu));
  MTLGPU_TRY(dalloc(ctx, &P->d_Lv, nu));
  MTLGPU_TRY(csr_transpose(ctx, n, n, nu, P->d_Urp, P->d_Uci, P->d_Uv, P->d_Lrp, P->d_Lci,
                           P->d_Lv));
  // lower plan of L (levels of trans(U)) with a-values, then the inverses
  MTLGPU_TRY(build_sweep_plan(ctx, n, P->d_Lrp, P->d_Lci, P->d_Lv, true, false, true, &P->lower));
  double* d_inv = nullptr;
  int* d_pivot = nullptr;
  MTLGPU_TRY(dalloc(ctx, &d_inv, n));
  MTLGPU_TRY(dalloc(ctx, &d_pivot, 1));
  MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(d_pivot, 0, sizeof(int), ctx->stream));
  MTLGPU_TRY(fill_sentinel<double>(ctx, d_inv, n));
  unsigned* d_ticket = nullptr;
  MTLGPU_TRY(dalloc(ctx, &d_ticket, 1));
  MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(d_ticket, 0, sizeof(unsigned), ctx->stream));
  const SweepPlan& L = P->lower;
  int G = L.group;
  long long warps = std::max(1ll, std::min<long long>(L.n_tasks, (long long)ctx->num_sms * 64));
  int grid = (int)((warps * 32 + kBlock - 1) / kBlock);
#define IC0_CASE(GG)                                                                          \
  case GG:                                                                                    \
    ic0_inv_kernel<GG><<<grid, kBlock, 0, ctx->stream>>>(L.n_tasks, L.d_task_ptr, L.d_rp,     \
                                                          L.d_ci, L.d_val, L.d_dinv,          \
                                                          L.d_row_of, d_inv, d_ticket,        \
                                                          ctx->d_error, d_pivot,              \
                                                          ctx->spin_limit);                   \
    break;
  switch (G) {
    IC0_CASE(1) IC0_CASE(2) IC0_CASE(4) IC0_CASE(8) IC0_CASE(16) IC0_CASE(32)
    default: return MTLGPU_INVALID_ARG;
  }
#undef IC0_CASE
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  ic0_values_kernel<<<grid_cap(ctx, n), kBlock, 0, ctx->stream>>>(n, P->d_Urp, P->d_Uci, P->d_Uv,
                                                                  P->d_Lrp, P->d_Lci, P->d_Lv,
                                                                  d_inv);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  MTLGPU_TRY(read_pivot(ctx, d_pivot, &P->factor_status));
  dfree(ctx, d_inv);
  dfree(ctx, d_pivot);
  dfree(ctx, d_ticket);
  // sweep plans with the final values
  MTLGPU_TRY(refill_plan(ctx, &P->lower, P->d_Lrp, P->d_Lv, true));
  MTLGPU_TRY(build_sweep_plan(ctx, n, P->d_Urp, P->d_Uci, P->d_Uv, false, false, false, &P->upper));
  return MTLGPU_OK;
}

mtlgpu_status build_ilu0(Pc* P) {
  Csr* A = P->A;
  Ctx* ctx = A->ctx;
  const int n = A->n_rows;
  int32_t *d_lcnt = nullptr, *d_ucnt = nullptr;
  MTLGPU_TRY(dalloc(ctx, &d_lcnt, n + 1));
  MTLGPU_TRY(dalloc(ctx, &d_ucnt, n + 1));
  MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(d_lcnt, 0, sizeof(int32_t) * (n + 1), ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(d_ucnt, 0, sizeof(int32_t) * (n + 1), ctx->stream));
  lower_count_kernel<<<grid_cap(ctx, n), kBlock, 0, ctx->stream>>>(n, A->d_rp, A->d_ci, d_lcnt,
                                                                   true);
  lower_count_kernel<<<grid_cap(ctx, n), kBlock, 0, ctx->stream>>>(n, A->d_rp, A->d_ci, d_ucnt,
                                                                   false);
  MTLGPU_TRY(dalloc(ctx, &P->d_Lrp, n + 1));
  MTLGPU_TRY(dalloc(ctx, &P->d_Urp, n + 1));
  MTLGPU_TRY(scan_i32(ctx, d_lcnt, P->d_Lrp, n + 1));
  MTLGPU_TRY(scan_i32(ctx, d_ucnt, P->d_Urp, n + 1));
  dfree(ctx, d_lcnt);
  dfree(ctx, d_ucnt);
  int nl = 0, nu = 0;
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(&nl, P->d_Lrp + n, sizeof(int), cudaMemcpyDeviceToHost,
                                       ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(&nu, P->d_Urp + n, sizeof(int), cudaMemcpyDeviceToHost,
                                       ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  P->nnz_L = nl;
  P->nnz_U = nu;
  MTLGPU_TRY(dalloc(ctx, &P->d_Lci, nl));
  MTLGPU_TRY(dalloc(ctx, &P->d_Lv, nl));
  MTLGPU_TRY(dalloc(ctx, &P->d_Uci, nu));
  MTLGPU_TRY(dalloc(ctx, &P->d_Uv, nu));
  // pattern split (values filled after the factorisation)
  split_kernel<<<grid_cap(ctx, n), kBlock, 0, ctx->stream>>>(n, A->d_rp, A->d_ci, A->d_v, P->d_Lrp,
                                                             P->d_Lci, P->d_Lv, P->d_Urp, P->d_Uci,
                                                             P->d_Uv);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  // level order of the strict-lower pattern (unit diagonal plan)
  MTLGPU_TRY(build_sweep_plan(ctx, n, P->d_Lrp, P->d_Lci, P->d_Lv, true, true, false, &P->lower));
  // factorise in place on a copy of A's values
  double *d_lu = nullptr, *d_inv = nullptr;
  int *d_done = nullptr, *d_pivot = nullptr;
  unsigned* d_ticket = nullptr;
  MTLGPU_TRY(dalloc(ctx, &d_lu, A->nnz));
  MTLGPU_TRY(dalloc(ctx, &d_inv, n));
  MTLGPU_TRY(dalloc(ctx, &d_done, n));
  MTLGPU_TRY(dalloc(ctx, &d_pivot, 1));
  MTLGPU_TRY(dalloc(ctx, &d_ticket, 1));
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(d_lu, A->d_v, sizeof(double) * A->nnz,
                                       cudaMemcpyDeviceToDevice, ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(d_done, 0, sizeof(int) * n, ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(d_pivot, 0, sizeof(int), ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(d_ticket, 0, sizeof(unsigned), ctx->stream));
  const SweepPlan& L = P->lower;
  long long warps = std::max(1ll, std::min<long long>(L.n_tasks, (long long)ctx->num_sms * 64));
  int grid = (int)((warps * 32 + kBlock - 1) / kBlock);
  ilu0_kernel<<<grid, kBlock, 0, ctx->stream>>>(L.n_tasks, L.d_task_ptr, L.d_row_of, A->d_rp,
                                                A->d_ci, A->d_diag, d_lu, d_inv, d_done, d_ticket,
                                                ctx->d_error, d_pivot, ctx->spin_limit);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  ilu0_split_kernel<<<grid_cap(ctx, n), kBlock, 0, ctx->stream>>>(
      n, A->d_rp, A->d_ci, d_lu, A->d_diag, P->d_Lrp, P->d_Lv, P->d_Urp, P->d_Uv);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  MTLGPU_TRY(read_pivot(ctx, d_pivot, &P->factor_status));
  dfree(ctx, d_lu);
  dfree(ctx, d_inv);
  dfree(ctx, d_done);
  dfree(ctx, d_pivot);
  dfree(ctx, d_ticket);
  MTLGPU_TRY(refill_plan(ctx, &P->lower, P->d_Lrp, P->d_Lv, false));
  MTLGPU_TRY(build_sweep_plan(ctx, n, P->d_Urp, P->d_Uci, P->d_Uv, false, false, false, &P->upper));
  return MTLGPU_OK;
}

}  // namespace

mtlgpu_status pc_build(Pc* P) {
  Csr* A = P->A;
  Ctx* ctx = A->ctx;
  const int n = A->n_rows;
  P->n = n;
  if (A->n_rows != A->n_cols) return MTLGPU_NOT_SQUARE;
  if (P->kind == MTLGPU_PC_IDENTITY) return MTLGPU_OK;
  if (P->kind == MTLGPU_PC_DIAGONAL) {
    MTLGPU_TRY(dalloc(ctx, &P->d_inv_diag, n));
    if (P->prec == MTLGPU_FP32) MTLGPU_TRY(dalloc(ctx, &P->d_inv_diag32, n));
    if (n)
      jacobi_kernel<<<grid_cap(ctx, n), kBlock, 0, ctx->stream>>>(n, A->d_diag, A->d_v,
                                                                  P->d_inv_diag, P->d_inv_diag32);
    MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
    return take_device_error(ctx);
  }
  if (P->kind != MTLGPU_PC_IC0 && P->kind != MTLGPU_PC_ILU0) return MTLGPU_INVALID_ARG;
  if (n) check_diag_kernel<<<grid_cap(ctx, n), kBlock, 0, ctx->stream>>>(n, A->d_diag, ctx->d_error);
  MTLGPU_TRY(take_device_error(ctx));
  MTLGPU_TRY(dalloc(ctx, &P->d_tmp, n));
  if (P->kind == MTLGPU_PC_IC0)
    MTLGPU_TRY(build_ic0(P));
  else
    MTLGPU_TRY(build_ilu0(P));
  if (P->prec == MTLGPU_FP32) {
    // factors rounded to float after the FP64 factorisation (ic_0.hpp:122-130)
    MTLGPU_TRY(sweep_plan_make_fp32(ctx, &P->lower));
    MTLGPU_TRY(sweep_plan_make_fp32(ctx, &P->upper));
    MTLGPU_TRY(dalloc(ctx, &P->d_tmp32, n));
  }
  MTLGPU_TRY(take_device_error(ctx));
  MTLGPU_TRY(part_plan_build(ctx, &P->lower, P->prec == MTLGPU_FP32));
  MTLGPU_TRY(part_plan_build(ctx, &P->upper, P->prec == MTLGPU_FP32));
  return take_device_error(ctx);
}

mtlgpu_status pc_ensure_adjoint(Pc* P) {
  if (P->adj_built || P->kind != MTLGPU_PC_ILU0) return MTLGPU_OK;
  Ctx* ctx = P->A->ctx;
  const int n = P->n;
  // U^T: lower with the inverted diagonal last; L^T: upper with unit diagonal
  int32_t *trp = nullptr, *tci = nullptr;
  double* tv = nullptr;
  MTLGPU_TRY(dalloc(ctx, &trp, n + 1));
  MTLGPU_TRY(dalloc(ctx, &tci, P->nnz_U));
  MTLGPU_TRY(dalloc(ctx, &tv, P->nnz_U));
  MTLGPU_TRY(csr_transpose(ctx, n, n, P->nnz_U, P->d_Urp, P->d_Uci, P->d_Uv, trp, tci, tv));
  MTLGPU_TRY(build_sweep_plan(ctx, n, trp, tci, tv, true, false, true, &P->adj_lower));
  MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  dfree(ctx, trp);
  dfree(ctx, tci);
  dfree(ctx, tv);
  MTLGPU_TRY(dalloc(ctx, &trp, n + 1));
  MTLGPU_TRY(dalloc(ctx, &tci, P->nnz_L));
  MTLGPU_TRY(dalloc(ctx, &tv, P->nnz_L));
  MTLGPU_TRY(csr_transpose(ctx, n, n, P->nnz_L, P->d_Lrp, P->d_Lci, P->d_Lv, trp, tci, tv));
  // The reference applies L^T column by column from the last column down
  // (upper_trisolve on the adjoint view, column-major: w[j] -= L[r][j] w[r]
  // for r descending), so each row of L^T takes its entries in descending
  // column order.
  if (n)
    reverse_rows_kernel<<<grid_cap(ctx, n), kBlock, 0, ctx->stream>>>(n, trp, tci, tv);
  MTLGPU_TRY(build_sweep_plan(ctx, n, trp, tci, tv, false, true, false, &P->adj_upper));
  MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  dfree(ctx, trp);
  dfree(ctx, tci);
  dfree(ctx, tv);
  if (P->prec == MTLGPU_FP32) {
    MTLGPU_TRY(sweep_plan_make_fp32(ctx, &P->adj_lower));
    MTLGPU_TRY(sweep_plan_make_fp32(ctx, &P->adj_upper));
  }
  MTLGPU_TRY(take_device_error(ctx));
  MTLGPU_TRY(part_plan_build(ctx, &P->adj_lower, P->prec == MTLGPU_FP32));
  MTLGPU_TRY(part_plan_build(ctx, &P->adj_upper, P->prec == MTLGPU_FP32));
  P->adj_built = true;
  return take_device_error(ctx);
}

void pc_release(Pc* P) {
  Ctx* ctx = P->A->ctx;
  dfree(ctx, P->d_inv_diag);
  dfree(ctx, P->d_inv_diag32);
  dfree(ctx, P->d_Lrp);
  dfree(ctx, P->d_Lci);
  dfree(ctx, P->d_Lv);
  dfree(ctx, P->d_Urp);
  dfree(ctx, P->d_Uci);
  dfree(ctx, P->d_Uv);
  dfree(ctx, P->d_tmp);
  dfree(ctx, P->d_tmp32);
  free_sweep_plan(ctx, &P->lower);
  free_sweep_plan(ctx, &P->upper);
  free_sweep_plan(ctx, &P->adj_lower);
  free_sweep_plan(ctx, &P->adj_upper);
  sell_free(ctx, &P->jac_lower);
  sell_free(ctx, &P->jac_upper);
  dfree(ctx, P->d_jtmp);
  dfree(ctx, P->d_jtmp32);
}

// Switches the triangular solves of P between the exact sweeps (iters = 0)
// and `iters` Jacobi iterations per triangle, building the SELL-32 copies of
// the factors on first use.  The factors are the reference-layout ones: IC(0)
// L has its inverted diagonal last, U first; ILU(0) L has a unit diagonal.
mtlgpu_status pc_set_jacobi(Pc* P, int iters) {
  if (iters < 0) return MTLGPU_INVALID_ARG;
  if (P->kind != MTLGPU_PC_IC0 && P->kind != MTLGPU_PC_ILU0) return iters ? MTLGPU_INVALID_ARG : MTLGPU_OK;
  Ctx* ctx = P->A->ctx;
  if (iters > 0 && !P->jac_lower.d_slice_ptr && P->n > 0) {
    const bool f32 = P->prec == MTLGPU_FP32;
    const int lower_diag = P->kind == MTLGPU_PC_IC0 ? 2 : 0;
    MTLGPU_TRY(sell_build(ctx, P->n, P->d_Lrp, P->d_Lci, P->d_Lv, lower_diag, true, f32, f32,
                          true, &P->jac_lower));
    MTLGPU_TRY(sell_build(ctx, P->n, P->d_Urp, P->d_Uci, P->d_Uv, 1, true, f32, f32, true,
                          &P->jac_upper));
    MTLGPU_TRY(dalloc(ctx, &P->d_jtmp, P->n));
    if (f32) MTLGPU_TRY(dalloc(ctx, &P->d_jtmp32, P->n));
    MTLGPU_TRY(take_device_error(ctx));
  }
  P->jacobi_iters = iters;
  return MTLGPU_OK;
}

template <typename T>
struct PcVec;
template <>
struct PcVec<double> {
  static double* tmp(Pc* P) { return P->d_tmp; }
  static double* jtmp(Pc* P) { return P->d_jtmp; }
  static const double* inv(Pc* P) { return P->d_inv_diag; }
};
template <>
struct PcVec<float> {
  static float* tmp(Pc* P) { return P->d_tmp32; }
  static float* jtmp(Pc* P) { return P->d_jtmp32; }
  static const float* inv(Pc* P) { return P->d_inv_diag32; }
};

template <typename T>
mtlgpu_status pc_apply_t(Pc* P, const T* r, T* z, bool adjoint, const int* skip,
                         bool prefilled_tmp, bool prefilled_out, double* rho_out) {
  Ctx* ctx = P->A->ctx;
  const int n = P->n;
  if (n == 0) return MTLGPU_OK;
  switch (P->kind) {
    case MTLGPU_PC_IDENTITY:
      copy_kernel<T><<<grid_cap(ctx, n), kBlock, 0, ctx->stream>>>(n, r, z, skip);
      break;
    case MTLGPU_PC_DIAGONAL: {
      const T* inv = PcVec<T>::inv(P);
      if (!inv) return MTLGPU_INVALID_ARG;
      jacobi_apply_kernel<T><<<grid_cap(ctx, n), kBlock, 0, ctx->stream>>>(n, inv, r, z, skip);
      break;
    }
    default: {
      T* tmp = PcVec<T>::tmp(P);
      if (!tmp) return MTLGPU_INVALID_ARG;
      if (P->jacobi_iters > 0) {
        // IC(0): the adjoint solve is the solve itself (U = trans(L)).
        if (adjoint && P->kind == MTLGPU_PC_ILU0) return MTLGPU_NOT_SUPPORTED;
        T* scratch = PcVec<T>::jtmp(P);
        if (!scratch) return MTLGPU_INVALID_ARG;
        MTLGPU_TRY(jacobi_solve<T>(ctx, P->jac_lower, P->jacobi_iters, r, tmp, scratch, skip));
        MTLGPU_TRY(jacobi_solve<T>(ctx, P->jac_upper, P->jacobi_iters, tmp, z, scratch, skip,
                                   rho_out ? r : nullptr, rho_out));
        break;
      }
      if (adjoint && P->kind == MTLGPU_PC_ILU0) {
        MTLGPU_TRY(pc_ensure_adjoint(P));
        MTLGPU_TRY(sweep_launch<T>(ctx, P->adj_lower, r, tmp, prefilled_tmp, skip));
        MTLGPU_TRY(sweep_launch<T>(ctx, P->adj_upper, tmp, z, prefilled_out, skip));
      } else {
        MTLGPU_TRY(sweep_launch<T>(ctx, P->lower, r, tmp, prefilled_tmp, skip));
        MTLGPU_TRY(sweep_launch<T>(ctx, P->upper, tmp, z, prefilled_out, skip));
      }
    }
  }
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  return MTLGPU_OK;
}

template mtlgpu_status pc_apply_t<double>(Pc*, const double*, double*, bool, const int*, bool,
                                          bool, double*);
template mtlgpu_status pc_apply_t<float>(Pc*, const float*, float*, bool, const int*, bool, bool,
                                         double*);

}  // namespace mtlgpu
