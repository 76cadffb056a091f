// Level-set analysis of triangular factors and sweep plans.
//
// The reference solves its factors with sequential row loops
// (mtl/operation/lower_trisolve.hpp:173-209, upper_trisolve.hpp:160-176) and
// computes no level sets.  Here the level of a row is the deterministic
// function of the factor pattern
//   level[r] = 0 if row r has no off-diagonal entry, else
//              1 + max(level[c]) over its off-diagonal columns c,
// which is the longest dependency chain ending at r.  Rows of one level are
// independent, so a sweep that visits levels in order can process every row
// of a level in parallel.  The GPU computes the levels itself (sync-free:
// every row waits on its dependencies' NaN-boxed level words) and the result
// is bit-identical to the sequential definition.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "device.cuh"
#include "internal.h"

namespace mtlgpu {

using namespace dev;

namespace {

constexpr int kBlock = 256;

int grid_cap(Ctx* ctx, long long count, int per_block = kBlock) {
  long long need = (count + per_block - 1) / per_block;
  long long cap = (long long)ctx->num_sms * 8;
  return (int)std::max(1ll, std::min(need, cap));
}

__global__ void fill_int_kernel(long long n, int32_t* p, int32_t v) {
  for (long long i = gtid(); i < n; i += gstride()) p[i] = v;
}

template <typename T>
__global__ void fill_box_kernel(long long n, T* p) {
  const T s = Box<T>::sentinel();
  for (long long i = gtid(); i < n; i += gstride()) p[i] = s;
}

// Level computation, a warp per chunk of kLevelChunk consecutive rows in
// dependency order (ascending for a lower factor, descending for an upper
// one), chunks claimed through an atomic ticket.  A warp takes its chunk's
// rows in order, lanes splitting a row's entries (maximum by shuffles); a
// dependency inside the chunk is read from the warp's shared copy, one
// outside it waits (bounded) on the global level array.  Every row waited on
// lies in a chunk claimed earlier by a running warp that takes its rows in
// order, so the waits always end.  One ticket per chunk rather than per row:
// a ticket per row serialised 2.1M atomics on one word (32 ms at 128^3).
constexpr int kLevelChunk = 32;

__global__ void levels_kernel(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                              bool lower, int* level, unsigned* ticket, int* err,
                              long long limit) {
  __shared__ int chunk_level[kBlock / 32][kLevelChunk];
  const int lane = threadIdx.x & 31;
  const int wid = threadIdx.x >> 5;
  while (true) {
    unsigned t0 = 0;
    if (lane == 0) t0 = atomicAdd(ticket, (unsigned)kLevelChunk);
    t0 = __shfl_sync(0xffffffffu, t0, 0);
    if (t0 >= (unsigned)n) break;
    const int cnt = min(kLevelChunk, n - (int)t0);
    for (int i = 0; i < cnt; i++) {
      const int t = (int)t0 + i;
      const int r = lower ? t : n - 1 - t;
      int l = 0;
      for (int j = rp[r] + lane; j < rp[r + 1]; j += 32) {
        const int c = ci[j];
        if (lower ? (c < r) : (c > r)) {
          const int tc = lower ? c : n - 1 - c;  // tc < t
          const int lc = tc >= (int)t0 ? chunk_level[wid][tc - (int)t0]
                                       : wait_value(level + c, limit, err);
          l = max(l, lc + 1);
        }
      }
      for (int off = 16; off > 0; off >>= 1) l = max(l, __shfl_xor_sync(0xffffffffu, l, off));
      if (lane == 0) {
        chunk_level[wid][i] = l;
        st_relaxed(level + r, l);
      }
      __syncwarp();
    }
  }
}

__global__ void level_hist_kernel(int n, const int32_t* __restrict__ level, int32_t* counts) {
  for (long long i = gtid(); i < n; i += gstride()) atomicAdd(&counts[level[i]], 1);
}

__global__ void iota_kernel(int n, int32_t* p) {
  for (long long i = gtid(); i < n; i += gstride()) p[i] = (int32_t)i;
}

// Off-diagonal entries of plan row t (original row row_of[t]).
__global__ void plan_counts_kernel(int n, const int32_t* __restrict__ row_of,
                                   const int32_t* __restrict__ frp, bool unit_diag,
                                   int32_t* cnt) {
  for (long long t = gtid(); t < n; t += gstride()) {
    const int r = row_of[t];
    const int len = frp[r + 1] - frp[r];
    cnt[t] = unit_diag ? len : len - 1;
  }
}

__global__ void plan_fill_kernel(int n, const int32_t* __restrict__ row_of,
                                 const int32_t* __restrict__ frp, const int32_t* __restrict__ fci,
                                 const double* __restrict__ fv, bool unit_diag, bool diag_last,
                                 const int32_t* __restrict__ prp, int32_t* pci, double* pv,
                                 double* dinv, int* err) {
  for (long long t = gtid(); t < n; t += gstride()) {
    const int r = row_of[t];
    int b = frp[r], e = frp[r + 1];
    if (!unit_diag) {
      // the stored diagonal: last entry (IC lower, v6) or first (upper, v3)
      const int d = diag_last ? e - 1 : b;
      if (e == b || fci[d] != r) {
        atomicCAS(err, 0, (int)MTLGPU_MISSING_DIAGONAL);
        dinv[t] = 0.0;
      } else {
        dinv[t] = fv[d];
      }
      if (diag_last) e--; else b++;
    }
    int o = prp[t];
    for (int j = b; j < e; j++, o++) {
      pci[o] = fci[j];
      pv[o] = fv[j];
    }
  }
}

__global__ void row_of_entry_kernel(int n, const int32_t* __restrict__ rp, int32_t* row) {
  for (long long r = gtid(); r < n; r += gstride())
    for (int j = rp[r]; j < rp[r + 1]; j++) row[j] = (int32_t)r;
}

__global__ void col_hist_kernel(long long nnz, const int32_t* __restrict__ ci, int32_t* counts) {
  for (long long j = gtid(); j < nnz; j += gstride()) atomicAdd(&counts[ci[j]], 1);
}

__global__ void transpose_gather_kernel(long long nnz, const int32_t* __restrict__ perm,
                                        const int32_t* __restrict__ row_of_entry,
                                        const double* __restrict__ v, int32_t* tci, double* tv) {
  for (long long k = gtid(); k < nnz; k += gstride()) {
    const int j = perm[k];
    tci[k] = row_of_entry[j];
    if (tv) tv[k] = v[j];
  }
}

// b = (float)a, and a rounded in place to the same value: factors stored as
// float are used with float64 vectors at their float values, as
// ic_0<M, float> / ilu_0<M, float> do (float entries promoted to double inside
// the trisolves, mtl/operation/lower_trisolve.hpp:173-209).
__global__ void d2f_kernel(long long n, double* __restrict__ a, float* __restrict__ b) {
  for (long long i = gtid(); i < n; i += gstride()) {
    const float f = (float)a[i];
    b[i] = f;
    a[i] = (double)f;
  }
}

}  // namespace

mtlgpu_status scan_i32(Ctx* ctx, const int32_t* in, int32_t* out, int n) {
  size_t bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, ctx->stream);
  char* tmp = nullptr;
  MTLGPU_TRY(dalloc(ctx, &tmp, bytes));
  cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, n, ctx->stream);
  dfree(ctx, tmp);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  return MTLGPU_OK;
}

template <typename T>
mtlgpu_status fill_sentinel(Ctx* ctx, T* p, int n) {
  if (n <= 0) return MTLGPU_OK;
  fill_box_kernel<T><<<grid_cap(ctx, n), kBlock, 0, ctx->stream>>>(n, p);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  return MTLGPU_OK;
}
template mtlgpu_status fill_sentinel<double>(Ctx*, double*, int);
template mtlgpu_status fill_sentinel<float>(Ctx*, float*, int);
template mtlgpu_status fill_sentinel<int>(Ctx*, int*, int);

mtlgpu_status compute_levels(Ctx* ctx, int n, const int32_t* d_rp, const int32_t* d_ci, bool lower,
                             int32_t* d_level, int* n_levels) {
  *n_levels = 0;
  if (n == 0) return MTLGPU_OK;
  MTLGPU_TRY(fill_sentinel<int>(ctx, d_level, n));
  unsigned* d_ticket = nullptr;
  MTLGPU_TRY(dalloc(ctx, &d_ticket, 1));
  MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(d_ticket, 0, sizeof(unsigned), ctx->stream));
  int grid = std::min(grid_cap(ctx, n), ctx->num_sms * 4);
  levels_kernel<<<grid, kBlock, 0, ctx->stream>>>(n, d_rp, d_ci, lower, d_level, d_ticket,
                                                  ctx->d_error, ctx->spin_limit);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  dfree(ctx, d_ticket);
  // number of levels = 1 + max level
  int32_t* d_max = nullptr;
  MTLGPU_TRY(dalloc(ctx, &d_max, 1));
  size_t bytes = 0;
  cub::DeviceReduce::Max(nullptr, bytes, d_level, d_max, n, ctx->stream);
  char* tmp = nullptr;
  MTLGPU_TRY(dalloc(ctx, &tmp, bytes));
  cub::DeviceReduce::Max(tmp, bytes, d_level, d_max, n, ctx->stream);
  int h_max = 0;
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(&h_max, d_max, sizeof(int), cudaMemcpyDeviceToHost,
                                       ctx->stream));
  dfree(ctx, tmp);
  dfree(ctx, d_max);
  MTLGPU_TRY(take_device_error(ctx));
  *n_levels = h_max + 1;
  return MTLGPU_OK;
}

void free_sweep_plan(Ctx* ctx, SweepPlan* p) {
  part_plan_free(ctx, p);
  dfree(ctx, p->d_rp);
  dfree(ctx, p->d_ci);
  dfree(ctx, p->d_val);
  dfree(ctx, p->d_val32);
  dfree(ctx, p->d_dinv);
  dfree(ctx, p->d_dinv32);
  dfree(ctx, p->d_row_of);
  dfree(ctx, p->d_task_ptr);
  dfree(ctx, p->d_level_ptr);
  dfree(ctx, p->d_level);
  dfree(ctx, p->d_ticket);
  *p = SweepPlan();
}

// Builds the level-ordered copy of a factor given in the reference's CSR
// layout: lower (IC: inverted diagonal last; ILU: unit diagonal, not stored)
// or upper (inverted diagonal first).
mtlgpu_status build_sweep_plan(Ctx* ctx, int n, const int32_t* frp, const int32_t* fci,
                               const double* fv, bool lower, bool unit_diag, bool diag_last,
                               SweepPlan* P) {
  free_sweep_plan(ctx, P);
  P->n = n;
  P->unit_diag = unit_diag;
  P->reverse = !lower;
  if (n == 0) return MTLGPU_OK;
  MTLGPU_TRY(dalloc(ctx, &P->d_level, n));
  MTLGPU_TRY(compute_levels(ctx, n, frp, fci, lower, P->d_level, &P->n_levels));
  const int L = P->n_levels;

  // rows sorted by (level, row)
  int32_t *d_rows = nullptr, *d_keys_sorted = nullptr;
  MTLGPU_TRY(dalloc(ctx, &d_rows, n));
  MTLGPU_TRY(dalloc(ctx, &d_keys_sorted, n));
  MTLGPU_TRY(dalloc(ctx, &P->d_row_of, n));
  iota_kernel<<<grid_cap(ctx, n), kBlock, 0, ctx->stream>>>(n, d_rows);
  int bits = 1;
  while ((1ll << bits) < L) bits++;
  size_t bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, P->d_level, d_keys_sorted, d_rows, P->d_row_of, n,
                                  0, bits, ctx->stream);
  char* tmp = nullptr;
  MTLGPU_TRY(dalloc(ctx, &tmp, bytes));
  cub::DeviceRadixSort::SortPairs(tmp, bytes, P->d_level, d_keys_sorted, d_rows, P->d_row_of, n, 0,
                                  bits, ctx->stream);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  dfree(ctx, tmp);
  dfree(ctx, d_keys_sorted);
  dfree(ctx, d_rows);

  // level pointers
  int32_t* d_counts = nullptr;
  MTLGPU_TRY(dalloc(ctx, &d_counts, L + 1));
  MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(d_counts, 0, sizeof(int32_t) * (L + 1), ctx->stream));
  level_hist_kernel<<<grid_cap(ctx, n), kBlock, 0, ctx->stream>>>(n, P->d_level, d_counts);
  MTLGPU_TRY(dalloc(ctx, &P->d_level_ptr, L + 1));
  MTLGPU_TRY(scan_i32(ctx, d_counts, P->d_level_ptr, L + 1));
  dfree(ctx, d_counts);
  std::vector<int32_t> h_lp(L + 1);
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(h_lp.data(), P->d_level_ptr, sizeof(int32_t) * (L + 1),
                                       cudaMemcpyDeviceToHost, ctx->stream));

  // off-diagonal counts -> plan row pointers
  int32_t* d_cnt = nullptr;
  MTLGPU_TRY(dalloc(ctx, &d_cnt, n + 1));
  MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(d_cnt, 0, sizeof(int32_t) * (n + 1), ctx->stream));
  plan_counts_kernel<<<grid_cap(ctx, n), kBlock, 0, ctx->stream>>>(n, P->d_row_of, frp, unit_diag,
                                                                   d_cnt);
  MTLGPU_TRY(dalloc(ctx, &P->d_rp, n + 1));
  MTLGPU_TRY(scan_i32(ctx, d_cnt, P->d_rp, n + 1));
  // largest off-diagonal count decides the lanes per row
  int32_t* d_max = nullptr;
  MTLGPU_TRY(dalloc(ctx, &d_max, 1));
  cub::DeviceReduce::Max(nullptr, bytes, d_cnt, d_max, n, ctx->stream);
  MTLGPU_TRY(dalloc(ctx, &tmp, bytes));
  cub::DeviceReduce::Max(tmp, bytes, d_cnt, d_max, n, ctx->stream);
  int h_max_off = 0, h_nnz_off = 0;
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(&h_max_off, d_max, sizeof(int), cudaMemcpyDeviceToHost,
                                       ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(&h_nnz_off, P->d_rp + n, sizeof(int),
                                       cudaMemcpyDeviceToHost, ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  dfree(ctx, tmp);
  dfree(ctx, d_max);
  dfree(ctx, d_cnt);
  P->nnz_off = h_nnz_off;
  int G = 1;
  while (G < h_max_off && G < 32) G <<= 1;
  P->group = G;

  MTLGPU_TRY(dalloc(ctx, &P->d_ci, h_nnz_off));
  MTLGPU_TRY(dalloc(ctx, &P->d_val, h_nnz_off));
  if (!unit_diag) MTLGPU_TRY(dalloc(ctx, &P->d_dinv, n));
  plan_fill_kernel<<<grid_cap(ctx, n), kBlock, 0, ctx->stream>>>(
      n, P->d_row_of, frp, fci, fv, unit_diag, diag_last, P->d_rp, P->d_ci, P->d_val, P->d_dinv,
      ctx->d_error);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());

  // tasks: at most 32/G plan rows each, never crossing a level boundary
  const int R = 32 / G;
  std::vector<int32_t> h_tp;
  h_tp.reserve((size_t)n / R + L + 1);
  for (int l = 0; l < L; l++)
    for (int t = h_lp[l]; t < h_lp[l + 1]; t += R) h_tp.push_back(t);
  P->n_tasks = (int)h_tp.size();
  h_tp.push_back(n);
  MTLGPU_TRY(dalloc(ctx, &P->d_task_ptr, h_tp.size()));
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(P->d_task_ptr, h_tp.data(), sizeof(int32_t) * h_tp.size(),
                                       cudaMemcpyHostToDevice, ctx->stream));
  MTLGPU_TRY(dalloc(ctx, &P->d_ticket, 2));
  MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(P->d_ticket, 0, 2 * sizeof(unsigned), ctx->stream));
  MTLGPU_TRY(take_device_error(ctx));  // also keeps h_tp alive until the copy is done
  return MTLGPU_OK;
}

mtlgpu_status sweep_plan_make_fp32(Ctx* ctx, SweepPlan* P) {
  if (P->n == 0) return MTLGPU_OK;
  if (!P->d_val32) {
    MTLGPU_TRY(dalloc(ctx, &P->d_val32, P->nnz_off));
    if (P->nnz_off)
      d2f_kernel<<<grid_cap(ctx, P->nnz_off), kBlock, 0, ctx->stream>>>(P->nnz_off, P->d_val,
                                                                        P->d_val32);
  }
  if (P->d_dinv && !P->d_dinv32) {
    MTLGPU_TRY(dalloc(ctx, &P->d_dinv32, P->n));
    d2f_kernel<<<grid_cap(ctx, P->n), kBlock, 0, ctx->stream>>>(P->n, P->d_dinv, P->d_dinv32);
  }
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  return MTLGPU_OK;
}

// CSR transpose with rows of the result sorted by column: a stable radix sort
// of the entries by column keeps them in ascending original-row order.
mtlgpu_status csr_transpose(Ctx* ctx, int n_rows, int n_cols, int nnz, const int32_t* d_rp,
                            const int32_t* d_ci, const double* d_v, int32_t* d_trp,
                            int32_t* d_tci, double* d_tv) {
  MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(d_trp, 0, sizeof(int32_t) * (n_cols + 1), ctx->stream));
  if (nnz == 0) return MTLGPU_OK;
  int32_t *d_rowe = nullptr, *d_idx = nullptr, *d_perm = nullptr, *d_keys = nullptr,
          *d_cnt = nullptr;
  MTLGPU_TRY(dalloc(ctx, &d_rowe, nnz));
  MTLGPU_TRY(dalloc(ctx, &d_idx, nnz));
  MTLGPU_TRY(dalloc(ctx, &d_perm, nnz));
  MTLGPU_TRY(dalloc(ctx, &d_keys, nnz));
  MTLGPU_TRY(dalloc(ctx, &d_cnt, n_cols + 1));
  row_of_entry_kernel<<<grid_cap(ctx, n_rows), kBlock, 0, ctx->stream>>>(n_rows, d_rp, d_rowe);
  iota_kernel<<<grid_cap(ctx, nnz), kBlock, 0, ctx->stream>>>(nnz, d_idx);
  int bits = 1;
  while ((1ll << bits) < n_cols) bits++;
  size_t bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, d_ci, d_keys, d_idx, d_perm, nnz, 0, bits,
                                  ctx->stream);
  char* tmp = nullptr;
  MTLGPU_TRY(dalloc(ctx, &tmp, bytes));
  cub::DeviceRadixSort::SortPairs(tmp, bytes, d_ci, d_keys, d_idx, d_perm, nnz, 0, bits,
                                  ctx->stream);
  dfree(ctx, tmp);
  MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(d_cnt, 0, sizeof(int32_t) * (n_cols + 1), ctx->stream));
  col_hist_kernel<<<grid_cap(ctx, nnz), kBlock, 0, ctx->stream>>>(nnz, d_ci, d_cnt);
  MTLGPU_TRY(scan_i32(ctx, d_cnt, d_trp, n_cols + 1));
  transpose_gather_kernel<<<grid_cap(ctx, nnz), kBlock, 0, ctx->stream>>>(nnz, d_perm, d_rowe, d_v,
                                                                          d_tci, d_tv);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  dfree(ctx, d_rowe);
  dfree(ctx, d_idx);
  dfree(ctx, d_perm);
  dfree(ctx, d_keys);
  dfree(ctx, d_cnt);
  return MTLGPU_OK;
}

mtlgpu_status csr_ensure_transpose(Csr* A) {
  if (A->d_trp) return MTLGPU_OK;
  Ctx* ctx = A->ctx;
  MTLGPU_TRY(dalloc(ctx, &A->d_trp, A->n_cols + 1));
  MTLGPU_TRY(dalloc(ctx, &A->d_tci, A->nnz));
  MTLGPU_TRY(dalloc(ctx, &A->d_tv, A->nnz));
  return csr_transpose(ctx, A->n_rows, A->n_cols, A->nnz, A->d_rp, A->d_ci, A->d_v, A->d_trp,
                       A->d_tci, A->d_tv);
}

}  // namespace mtlgpu
