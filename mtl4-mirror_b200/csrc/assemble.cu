// Assembly on the device: coordinate triplets -> sorted, duplicate-free CSR.
//
// The result is what mtl::mat::inserter<compressed2D<double>, Updater> leaves
// in the matrix after `ins[r][c] << v` (or `= v`, `+= v`) for every triplet in
// order (mtl/matrix/compressed2D.hpp:662-1151):
//   * modify() (compressed2D.hpp:947-989) applies the updater to an entry that
//     is already there -- in the matrix before insertion began, in a slot or in
//     the spare map -- and init() to a new one; the updaters are
//     mtl/operation/update.hpp:26-111 (store: x = y; plus: x += y; minus:
//     x -= y, a new entry -y; times: x *= y);
//   * entries the matrix held before insertion (stretch(), 864-914) come first
//     and are updated like any other;
//   * final_place() / insert_spare() (1073-1151) merge slots and spare map into
//     rows sorted by column.  Slot size and the slot/spare split change where
//     an entry waits, never its value, so the result is determined by the
//     triplet order alone.
//
// Device algorithm:
//   1. keys r * n_cols + c for the base matrix's entries (tagged LOAD) followed
//      by the triplets; index range checked;
//   2. stable LSD radix sort of (key, item) pairs, 8-bit digits, as many
//      passes as the key has bits: per 2048-item tile a digit histogram, an
//      exclusive scan over (digit, tile), and a stable scatter that ranks
//      equal digits inside a warp with __match_any_sync and across warps and
//      rounds through shared-memory counters;
//   3. one thread per run of equal keys folds its items in insertion order
//      (init on the first, the updater on the rest), so sums of duplicates are
//      added in the same order as the reference adds them -- bit for bit;
//   4. row counts -> row starts by scan; the CSR arrays are adopted by a new
//      matrix handle.
//
// Device generation of laplacian_setup(A, m, n) (mtl/matrix/laplacian_setup.hpp:
// 25-44) and of the 3-D 7-point Laplacian writes the sorted rows directly.
#include <algorithm>
#include <cstdint>

#include "device.cuh"
#include "internal.h"

namespace mtlgpu {

mtlgpu_status csr_adopt(Ctx* ctx, int n_rows, int n_cols, int nnz, int32_t* d_rp, int32_t* d_ci,
                        double* d_v, Csr** out);  // capi.cpp

namespace {

using namespace dev;
typedef unsigned long long u64;

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kRounds = 8;                    // items per thread per tile (striped)
constexpr long long kTile = (long long)kThreads * kRounds;
constexpr int kRadix = 256;
static_assert(kThreads == kRadix, "one thread per digit in the radix kernels");

int grid_for(Ctx* ctx, long long count) {
  long long need = (count + kThreads - 1) / kThreads;
  return (int)std::max(1ll, std::min(need, (long long)ctx->num_sms * 16));
}

// base matrix entries: key and LOAD tag (a warp per row)
__global__ void base_keys_kernel(int n_rows, int n_cols, const int32_t* __restrict__ rp,
                                 const int32_t* __restrict__ ci, u64* __restrict__ key,
                                 int32_t* __restrict__ item) {
  const int lane = threadIdx.x & 31;
  for (long long r = gtid() >> 5; r < n_rows; r += gstride() >> 5)
    for (int j = rp[r] + lane; j < rp[r + 1]; j += 32) {
      key[j] = (u64)r * (u64)n_cols + (u64)ci[j];
      item[j] = j;
    }
}

// triplet keys; an index outside the matrix records MTLGPU_INDEX_RANGE
__global__ void triplet_keys_kernel(long long count, long long n_base, int n_rows, int n_cols,
                                    const int32_t* __restrict__ rows,
                                    const int32_t* __restrict__ cols, u64* __restrict__ key,
                                    int32_t* __restrict__ item, int* err) {
  for (long long k = gtid(); k < count; k += gstride()) {
    const int r = rows[k], c = cols[k];
    if (r < 0 || r >= n_rows || c < 0 || c >= n_cols) {
      atomicCAS(err, 0, (int)MTLGPU_INDEX_RANGE);
      key[n_base + k] = 0;
    } else {
      key[n_base + k] = (u64)r * (u64)n_cols + (u64)c;
    }
    item[n_base + k] = (int32_t)(n_base + k);
  }
}

// Digit histogram of one tile: counts[d * n_tiles + tile].
__global__ void __launch_bounds__(kThreads)
    radix_hist_kernel(long long count, const u64* __restrict__ key, int shift, int n_tiles,
                      int32_t* __restrict__ counts) {
  __shared__ int h[kRadix];
  h[threadIdx.x] = 0;
  __syncthreads();
  const long long t0 = (long long)blockIdx.x * kTile;
  for (int r = 0; r < kRounds; r++) {
    const long long i = t0 + (long long)r * kThreads + threadIdx.x;
    if (i < count) atomicAdd(&h[(int)((key[i] >> shift) & (kRadix - 1))], 1);
  }
  __syncthreads();
  counts[(long long)threadIdx.x * n_tiles + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter of one tile.  Items are taken in rounds of kThreads
// consecutive items (round-major, then thread order == input order); an
// item's place is its digit's offset for this tile, plus the items of that
// digit in earlier rounds and earlier warps of this round, plus its rank
// among equal digits of its own warp.
__global__ void __launch_bounds__(kThreads)
    radix_scatter_kernel(long long count, const u64* __restrict__ key_in,
                         const int32_t* __restrict__ item_in, u64* __restrict__ key_out,
                         int32_t* __restrict__ item_out, int shift, int n_tiles,
                         const int32_t* __restrict__ offsets) {
  __shared__ int base[kRadix];
  __shared__ int wcnt[kWarps][kRadix];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  base[threadIdx.x] = offsets[(long long)threadIdx.x * n_tiles + blockIdx.x];
  const long long t0 = (long long)blockIdx.x * kTile;
  for (int r = 0; r < kRounds; r++) {
    const long long i = t0 + (long long)r * kThreads + threadIdx.x;
    const bool valid = i < count;
    const u64 k = valid ? key_in[i] : 0ull;
    const int it = valid ? item_in[i] : 0;
    const int d = valid ? (int)((k >> shift) & (kRadix - 1)) : kRadix;  // invalid: own group
#pragma unroll
    for (int w = 0; w < kWarps; w++) wcnt[w][threadIdx.x] = 0;
    __syncthreads();
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    if (valid && lane == __ffs(peers) - 1) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    {  // thread t owns digit t: exclusive prefix over warps, carried across rounds
      int run = base[threadIdx.x];
#pragma unroll
      for (int w = 0; w < kWarps; w++) {
        const int c = wcnt[w][threadIdx.x];
        wcnt[w][threadIdx.x] = run;
        run += c;
      }
      base[threadIdx.x] = run;
    }
    __syncthreads();
    if (valid) {
      const int pos = wcnt[warp][d] + rank;
      key_out[pos] = k;
      item_out[pos] = it;
    }
    __syncthreads();
  }
}

__global__ void run_head_kernel(long long count, const u64* __restrict__ key,
                                int32_t* __restrict__ head) {
  for (long long i = gtid(); i <= count; i += gstride())
    head[i] = (i < count && (i == 0 || key[i] != key[i - 1])) ? 1 : 0;
}

__device__ __forceinline__ double op_init(int op, double y) {
  return op == MTLGPU_UPDATE_MINUS ? -y : y;  // update.hpp:37-40,55-58,73-76,91-94
}
__device__ __forceinline__ double op_apply(int op, double x, double y) {
  switch (op) {  // update.hpp:29-32,47-50,65-68,83-86
    case MTLGPU_UPDATE_PLUS: return __dadd_rn(x, y);
    case MTLGPU_UPDATE_MINUS: return __dsub_rn(x, y);
    case MTLGPU_UPDATE_TIMES: return __dmul_rn(x, y);
    default: return y;  // store
  }
}

// One thread per run of equal keys: the run's items in insertion order.
__global__ void fold_runs_kernel(long long count, int n_cols, long long n_base,
                                 const u64* __restrict__ key, const int32_t* __restrict__ item,
                                 const int32_t* __restrict__ head, const int32_t* __restrict__ pos,
                                 const double* __restrict__ vals, const uint8_t* __restrict__ ops,
                                 int default_op, int32_t* __restrict__ out_ci,
                                 double* __restrict__ out_v, int32_t* __restrict__ row_cnt) {
  for (long long i = gtid(); i < count; i += gstride()) {
    if (!head[i]) continue;
    const u64 k = key[i];
    int s = item[i];
    double v;
    if (s < n_base) {
      v = vals[s];
    } else {
      const int op = ops ? (int)ops[s - n_base] : default_op;
      v = op_init(op, vals[s]);
    }
    for (long long j = i + 1; j < count && key[j] == k; j++) {
      s = item[j];
      const int op = ops ? (int)ops[s - n_base] : default_op;  // base entries always lead
      v = op_apply(op, v, vals[s]);
    }
    const int u = pos[i];
    out_ci[u] = (int32_t)(k % (u64)n_cols);
    out_v[u] = v;
    atomicAdd(&row_cnt[k / (u64)n_cols], 1);
  }
}

// laplacian_setup(A, m, n): row i*n+j holds, by column, -1 (row-n), -1 (row-1),
// 4, -1 (row+1), -1 (row+n) where the neighbour exists.
__global__ void lap2d_count_kernel(int m, int n, int32_t* cnt) {
  const long long N = (long long)m * n;
  for (long long r = gtid(); r <= N; r += gstride()) {
    if (r == N) {
      cnt[r] = 0;
      continue;
    }
    const long long i = r / n, j = r % n;
    cnt[r] = 1 + (i > 0) + (j > 0) + (j < n - 1) + (i < m - 1);
  }
}
__global__ void lap2d_fill_kernel(int m, int n, const int32_t* __restrict__ rp,
                                  int32_t* __restrict__ ci, double* __restrict__ v) {
  const long long N = (long long)m * n;
  for (long long r = gtid(); r < N; r += gstride()) {
    const long long i = r / n, j = r % n;
    int p = rp[r];
    if (i > 0) ci[p] = (int32_t)(r - n), v[p++] = -1.0;
    if (j > 0) ci[p] = (int32_t)(r - 1), v[p++] = -1.0;
    ci[p] = (int32_t)r, v[p++] = 4.0;
    if (j < n - 1) ci[p] = (int32_t)(r + 1), v[p++] = -1.0;
    if (i < m - 1) ci[p] = (int32_t)(r + n), v[p++] = -1.0;
  }
}

// 3-D 7-point Laplacian on an N^3 grid, row (i*N+j)*N+k: 6 on the diagonal,
// -1 towards each existing neighbour (Dirichlet), columns ascending.
__global__ void lap3d_count_kernel(int N, int32_t* cnt) {
  const long long NN = (long long)N * N, n = NN * N;
  for (long long r = gtid(); r <= n; r += gstride()) {
    if (r == n) {
      cnt[r] = 0;
      continue;
    }
    const long long i = r / NN, j = (r / N) % N, k = r % N;
    cnt[r] = 1 + (i > 0) + (j > 0) + (k > 0) + (k < N - 1) + (j < N - 1) + (i < N - 1);
  }
}
__global__ void lap3d_fill_kernel(int N, const int32_t* __restrict__ rp, int32_t* __restrict__ ci,
                                  double* __restrict__ v) {
  const long long NN = (long long)N * N, n = NN * N;
  for (long long r = gtid(); r < n; r += gstride()) {
    const long long i = r / NN, j = (r / N) % N, k = r % N;
    int p = rp[r];
    if (i > 0) ci[p] = (int32_t)(r - NN), v[p++] = -1.0;
    if (j > 0) ci[p] = (int32_t)(r - N), v[p++] = -1.0;
    if (k > 0) ci[p] = (int32_t)(r - 1), v[p++] = -1.0;
    ci[p] = (int32_t)r, v[p++] = 6.0;
    if (k < N - 1) ci[p] = (int32_t)(r + 1), v[p++] = -1.0;
    if (j < N - 1) ci[p] = (int32_t)(r + N), v[p++] = -1.0;
    if (i < N - 1) ci[p] = (int32_t)(r + NN), v[p++] = -1.0;
  }
}

int key_bits(u64 max_key) {
  int b = 0;
  while (b < 64 && (max_key >> b) != 0) b++;
  return b;
}

struct DevBufs {
  Ctx* ctx;
  std::vector<void*> ptrs;
  template <typename T>
  mtlgpu_status get(T** p, size_t count) {
    MTLGPU_TRY(dalloc(ctx, p, count));
    ptrs.push_back(*p);
    return MTLGPU_OK;
  }
  ~DevBufs() {
    for (void* p : ptrs) cudaFreeAsync(p, ctx->stream);
  }
};

mtlgpu_status read_i32(Ctx* ctx, const int32_t* d, int32_t* h) {
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(h, d, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return MTLGPU_OK;
}

}  // namespace

// Stable sort of (key, item) pairs in place (keys < 2^bits); scratch from `bufs`.
static mtlgpu_status radix_sort_pairs(Ctx* ctx, DevBufs& bufs, long long count, int bits, u64*& key,
                                      int32_t*& item) {
  if (count <= 1 || bits == 0) return MTLGPU_OK;
  const int n_tiles = (int)((count + kTile - 1) / kTile);
  u64* key2 = nullptr;
  int32_t *item2 = nullptr, *counts = nullptr, *offs = nullptr;
  MTLGPU_TRY(bufs.get(&key2, count));
  MTLGPU_TRY(bufs.get(&item2, count));
  MTLGPU_TRY(bufs.get(&counts, (size_t)kRadix * n_tiles));
  MTLGPU_TRY(bufs.get(&offs, (size_t)kRadix * n_tiles));
  for (int shift = 0; shift < bits; shift += 8) {
    radix_hist_kernel<<<n_tiles, kThreads, 0, ctx->stream>>>(count, key, shift, n_tiles, counts);
    MTLGPU_TRY(scan_i32(ctx, counts, offs, kRadix * n_tiles));
    radix_scatter_kernel<<<n_tiles, kThreads, 0, ctx->stream>>>(count, key, item, key2, item2,
                                                                shift, n_tiles, offs);
    ctx->launches += 2;
    MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
    std::swap(key, key2);
    std::swap(item, item2);
  }
  return MTLGPU_OK;
}

mtlgpu_status csr_assemble(Ctx* ctx, const Csr* base, int n_rows, int n_cols, long long count,
                           const int32_t* d_rows, const int32_t* d_cols, const double* d_vals,
                           const uint8_t* d_ops, int updater, Csr** out) {
  const long long n_base = base ? base->nnz : 0;
  const long long total = n_base + count;
  if (total >= (1ll << 31) - 1) return MTLGPU_INVALID_ARG;  // int32 indices
  DevBufs bufs{ctx, {}};
  u64* key = nullptr;
  int32_t *item = nullptr, *head = nullptr, *pos = nullptr, *row_cnt = nullptr;
  double* vals = nullptr;
  MTLGPU_TRY(bufs.get(&key, total));
  MTLGPU_TRY(bufs.get(&item, total));
  MTLGPU_TRY(bufs.get(&vals, total));
  if (n_base) {
    base_keys_kernel<<<grid_for(ctx, 32ll * n_rows), kThreads, 0, ctx->stream>>>(
        n_rows, n_cols, base->d_rp, base->d_ci, key, item);
    ctx->launches++;
    MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(vals, base->d_v, sizeof(double) * n_base,
                                         cudaMemcpyDeviceToDevice, ctx->stream));
  }
  if (count) {
    triplet_keys_kernel<<<grid_for(ctx, count), kThreads, 0, ctx->stream>>>(
        count, n_base, n_rows, n_cols, d_rows, d_cols, key, item, ctx->d_error);
    ctx->launches++;
    MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(vals + n_base, d_vals, sizeof(double) * count,
                                         cudaMemcpyDeviceToDevice, ctx->stream));
  }
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  MTLGPU_TRY(take_device_error(ctx));  // index range, before anything is sorted
  const u64 max_key = (n_rows && n_cols) ? (u64)n_rows * (u64)n_cols - 1 : 0;
  MTLGPU_TRY(radix_sort_pairs(ctx, bufs, total, key_bits(max_key), key, item));
  // runs of equal keys -> unique entries
  MTLGPU_TRY(bufs.get(&head, total + 1));
  MTLGPU_TRY(bufs.get(&pos, total + 1));
  MTLGPU_TRY(bufs.get(&row_cnt, (size_t)n_rows + 1));
  run_head_kernel<<<grid_for(ctx, total + 1), kThreads, 0, ctx->stream>>>(total, key, head);
  ctx->launches++;
  MTLGPU_TRY(scan_i32(ctx, head, pos, (int)(total + 1)));
  int32_t nnz = 0;
  MTLGPU_TRY(read_i32(ctx, pos + total, &nnz));
  int32_t *rp = nullptr, *ci = nullptr;
  double* v = nullptr;
  MTLGPU_TRY(dalloc(ctx, &rp, (size_t)n_rows + 1));
  mtlgpu_status s = dalloc(ctx, &ci, nnz);
  if (s == MTLGPU_OK) s = dalloc(ctx, &v, nnz);
  if (s != MTLGPU_OK) {
    dfree(ctx, rp);
    dfree(ctx, ci);
    return s;
  }
  cudaError_t e = cudaMemsetAsync(row_cnt, 0, sizeof(int32_t) * ((size_t)n_rows + 1), ctx->stream);
  if (e == cudaSuccess && total) {
    fold_runs_kernel<<<grid_for(ctx, total), kThreads, 0, ctx->stream>>>(
        total, n_cols, n_base, key, item, head, pos, vals, d_ops, updater, ci, v, row_cnt);
    ctx->launches++;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) s = scan_i32(ctx, row_cnt, rp, n_rows + 1);
  else s = set_cuda_error(ctx, e, "assembly");
  if (s != MTLGPU_OK) {
    dfree(ctx, rp);
    dfree(ctx, ci);
    dfree(ctx, v);
    return s;
  }
  return csr_adopt(ctx, n_rows, n_cols, nnz, rp, ci, v, out);
}

mtlgpu_status csr_laplacian(Ctx* ctx, int dim, int a, int b, Csr** out) {
  const long long n = dim == 2 ? (long long)a * b : (long long)a * a * a;
  if (a < 0 || b < 0 || n >= (1ll << 31) - 1) return MTLGPU_INVALID_ARG;
  const long long nnz_max = dim == 2 ? 5 * n : 7 * n;
  if (nnz_max >= (1ll << 31) - 1) return MTLGPU_INVALID_ARG;
  int32_t *rp = nullptr, *cnt = nullptr, *ci = nullptr;
  double* v = nullptr;
  {
    DevBufs bufs{ctx, {}};
    MTLGPU_TRY(bufs.get(&cnt, n + 1));
    MTLGPU_TRY(dalloc(ctx, &rp, n + 1));
    const int g = grid_for(ctx, n + 1);
    if (dim == 2) lap2d_count_kernel<<<g, kThreads, 0, ctx->stream>>>(a, b, cnt);
    else lap3d_count_kernel<<<g, kThreads, 0, ctx->stream>>>(a, cnt);
    ctx->launches++;
    mtlgpu_status s = scan_i32(ctx, cnt, rp, (int)(n + 1));
    int32_t nnz = 0;
    if (s == MTLGPU_OK) s = read_i32(ctx, rp + n, &nnz);
    if (s == MTLGPU_OK) s = dalloc(ctx, &ci, nnz);
    if (s == MTLGPU_OK) s = dalloc(ctx, &v, nnz);
    if (s != MTLGPU_OK) {
      dfree(ctx, rp);
      dfree(ctx, ci);
      dfree(ctx, v);
      return s;
    }
    if (dim == 2) lap2d_fill_kernel<<<g, kThreads, 0, ctx->stream>>>(a, b, rp, ci, v);
    else lap3d_fill_kernel<<<g, kThreads, 0, ctx->stream>>>(a, rp, ci, v);
    ctx->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      dfree(ctx, rp);
      dfree(ctx, ci);
      dfree(ctx, v);
      return set_cuda_error(ctx, e, "laplacian generation");
    }
    return csr_adopt(ctx, (int)n, (int)n, nnz, rp, ci, v, out);
  }
}

}  // namespace mtlgpu
