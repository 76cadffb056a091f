// CSR sparse matrix-vector products for sm_100a.
//
// Replaces smat_cvec_mult<compressed2D> (mtl/operation/mat_vec_mult.hpp:
// 620-689) and the fused row evaluator of CG (mtl/vector/
// row_mat_cvec_index_evaluator.hpp:26-67 with dot_index_evaluator.hpp:19-45).
//
// Design: rows are binned by length; a bin with G lanes per row runs
// spmv_group<G>: each G-lane group walks its row with stride G (coalesced
// loads of values and column indices across the warp), gathers x through the
// read-only path (x stays resident in the 126 MB L2 for every configuration
// here), reduces with shuffles and lane 0 writes the row result and feeds
// the optional epilogue reduction.  Rows longer than 1024 entries get a CTA
// each.  Grids are persistent-style (a multiple of the SM count) so that
// epilogue reductions have a fixed number of partials and are deterministic.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "device.cuh"
#include "internal.h"
#include "tma.cuh"

namespace mtlgpu {

using namespace dev;

namespace {

constexpr int kBlock = 256;
constexpr int kStreamK = 8;            // entries per lane per row block (CSR-stream)
constexpr double kSellMaxPadding = 1.2;  // SELL-32 when padded entries <= 1.2 nnz

__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }

__device__ __forceinline__ int pow2_group(int len) {
  int g = 2;
  while (g < len && g < 32) g <<= 1;
  return g;
}

// Row statistics, validation and diagonal positions.
__global__ void csr_analyse_kernel(int n_rows, int n_cols, int nnz, const int32_t* __restrict__ rp,
                                   const int32_t* __restrict__ ci, int32_t* __restrict__ diag,
                                   unsigned long long* stats, int* err) {
  // stats[0] = max row length, stats[1] = sum of row lengths
  unsigned long long my_max = 0, my_sum = 0;
  for (long long r = gtid(); r < n_rows; r += gstride()) {
    int b = rp[r], e = rp[r + 1];
    if (r == 0 && b != 0) atomicCAS(err, 0, (int)MTLGPU_INVALID_ARG);
    if (r == n_rows - 1 && e != nnz) atomicCAS(err, 0, (int)MTLGPU_INVALID_ARG);
    if (e < b || b < 0 || e > nnz) {
      atomicCAS(err, 0, (int)MTLGPU_INVALID_ARG);
      diag[r] = -1;
      continue;
    }
    int d = -1, prev = -1;
    for (int j = b; j < e; j++) {
      int c = ci[j];
      if (c < 0 || c >= n_cols) atomicCAS(err, 0, (int)MTLGPU_INDEX_RANGE);
      if (c <= prev) atomicCAS(err, 0, (int)MTLGPU_NOT_SORTED);
      if (c == r) d = j;
      prev = c;
    }
    diag[r] = d;
    unsigned long long len = (unsigned long long)(e - b);
    my_max = len > my_max ? len : my_max;
    my_sum += len;
  }
  // warp-level combine then one atomic per warp (integer: order-independent)
  for (int off = 16; off > 0; off >>= 1) {
    unsigned long long om = __shfl_down_sync(0xffffffffu, my_max, off);
    unsigned long long os = __shfl_down_sync(0xffffffffu, my_sum, off);
    my_max = om > my_max ? om : my_max;
    my_sum += os;
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&stats[0], my_max);
    atomicAdd(&stats[1], my_sum);
  }
}

__global__ void row_bin_kernel(int n_rows, const int32_t* __restrict__ rp, int32_t* bin,
                               int32_t* rows) {
  for (long long r = gtid(); r < n_rows; r += gstride()) {
    int len = rp[r + 1] - rp[r];
    int g = len > 1024 ? 64 : pow2_group(len);  // 64 marks the CTA-per-row bin
    bin[r] = __ffs(g) - 1;                        // 1..5 for 2..32, 6 for CTA
    rows[r] = (int32_t)r;
  }
}

__global__ void to_fp32_kernel(long long n, const double* __restrict__ a, float* __restrict__ b) {
  for (long long i = gtid(); i < n; i += gstride()) b[i] = (float)a[i];
}

template <typename T>
struct EpiParams {
  int epi;
  T alpha, beta;
  const T* x2;
  const T* b;
  double* out;
  const int* skip;
  void* partials;
  int part_off, part_total;
  bool final_launch;
  unsigned* counter;
};

template <typename T>
__device__ __forceinline__ void row_epilogue(const EpiParams<T>& ep, int row, T s, T* y,
                                             typename AccOf<T, 1>::type& acc) {
  if (ep.epi == EPI_AXPBY) {
    T r = ep.alpha * s;
    if (ep.beta != T(0)) r = ep.beta * y[row] + r;
    y[row] = r;
  } else if (ep.epi == EPI_DOT_X2) {
    y[row] = s;
    acc.add_prod(0, ep.x2[row], s);
  } else {
    T r = ep.b[row] - s;
    y[row] = r;
    acc.add_prod(0, r, r);
  }
}

template <typename T>
__device__ __forceinline__ void finish_epilogue(const EpiParams<T>& ep,
                                                typename AccOf<T, 1>::type acc) {
  typedef typename AccOf<T, 1>::type R;
  if (ep.epi == EPI_AXPBY) return;
  R bs = block_reduce(acc);
  R* parts = reinterpret_cast<R*>(ep.partials);
  if (!ep.final_launch) {
    if (threadIdx.x == 0) parts[ep.part_off + blockIdx.x] = bs;
    return;
  }
  if (publish_partial(bs, parts, ep.part_off + blockIdx.x, ep.counter, gridDim.x)) {
    R tot = reduce_partials(parts, ep.part_total);
    if (threadIdx.x == 0) *ep.out = tot.value(0);
  }
}

// G lanes per row; rows either 0..nrows-1 or rows[0..nrows).
template <typename T, int G>
__global__ void __launch_bounds__(kBlock) spmv_group(int nrows, const int32_t* __restrict__ rows,
                                                     const int32_t* __restrict__ rp,
                                                     const int32_t* __restrict__ ci,
                                                     const T* __restrict__ val,
                                                     const T* __restrict__ x, T* __restrict__ y,
                                                     EpiParams<T> ep) {
  if (ep.skip && *ep.skip) return;
  typedef typename AccOf<T, 1>::type R;
  R acc = R::zero();
  constexpr int GPB = kBlock / G;
  const int gl = threadIdx.x % G;
  for (long long base = (long long)blockIdx.x * GPB; base < nrows; base += (long long)gridDim.x * GPB) {
    const long long gid = base + threadIdx.x / G;
    T s = T(0);
    int row = -1;
    if (gid < nrows) {
      row = rows ? rows[gid] : (int)gid;
      const int b = rp[row], e = rp[row + 1];
      for (int j = b + gl; j < e; j += G) s += val[j] * __ldg(x + ci[j]);
    }
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (gl == 0 && row >= 0) row_epilogue(ep, row, s, y, acc);
  }
  finish_epilogue(ep, acc);
}

// One CTA per row (rows longer than 1024 entries).
template <typename T>
__global__ void __launch_bounds__(kBlock) spmv_cta(int nrows, const int32_t* __restrict__ rows,
                                                   const int32_t* __restrict__ rp,
                                                   const int32_t* __restrict__ ci,
                                                   const T* __restrict__ val,
                                                   const T* __restrict__ x, T* __restrict__ y,
                                                   EpiParams<T> ep) {
  if (ep.skip && *ep.skip) return;
  typedef typename AccOf<T, 1>::type R;
  typedef typename AccOf<T, 1>::type RS;
  R acc = R::zero();
  for (long long g = blockIdx.x; g < nrows; g += gridDim.x) {
    const int row = rows ? rows[g] : (int)g;
    const int b = rp[row], e = rp[row + 1];
    Sum<1> part = Sum<1>::zero();
    T s = T(0);
    for (int j = b + threadIdx.x; j < e; j += kBlock) s += val[j] * __ldg(x + ci[j]);
    part.v[0] = (double)s;
    Sum<1> tot = block_reduce(part);
    __shared__ T row_sum;
    if (threadIdx.x == 0) row_sum = (T)tot.v[0];
    __syncthreads();
    if (threadIdx.x == 0) row_epilogue(ep, row, row_sum, y, acc);
    __syncthreads();
  }
  (void)sizeof(RS);
  finish_epilogue(ep, acc);
}

// CSR-stream: one warp per row block (<= 32 rows, <= 32*K entries), for
// matrices whose rows are too uneven for SELL-32.  meta[b] = (first row,
// first entry) of block b, meta[n_blocks] = (n, nnz).  Lane l loads entries
// e0 + l + 32k (k < K): K coalesced loads of values and column indices
// (last-use hint: they are streamed once, and x keeps its place in L2), then
// K gathers of x, all in flight at once, while the row bounds of its row and
// the next block's metadata are on their way.  The products are staged in
// shared memory and lane l sums row r0 + l in column order, product and sum
// rounded separately: every row sum equals the reference's
// `tmp += A.data[j] * v[A.ref_minor()[j]]` (mat_vec_mult.hpp:666-688) bit for
// bit.  A block holding a single row longer than 32*K entries is summed by
// the whole warp instead (tree order).  Registers stay at 32 so that 8 CTAs
// (64 warps) fit an SM: on B200 every variant with more state per lane and
// fewer warps measured slower.
template <typename T, int K>
__global__ void __launch_bounds__(kBlock, 8)
    spmv_stream(int n_blocks, const int2* __restrict__ meta, const int32_t* __restrict__ rp,
                const int32_t* __restrict__ ci, const T* __restrict__ val,
                const T* __restrict__ x, T* __restrict__ y, EpiParams<T> ep) {
  if (ep.skip && ld_relaxed(ep.skip)) return;
  typedef typename AccOf<T, 1>::type R;
  __shared__ T prod[kBlock / 32][32 * K];
  R acc = R::zero();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  T* pw = prod[wib];
  const int warp = (blockIdx.x * kBlock + threadIdx.x) >> 5;
  const int W = (gridDim.x * kBlock) >> 5;
  int2 ma = make_int2(0, 0), mb = ma;
  if (warp < n_blocks) {
    ma = __ldg(meta + warp);
    mb = __ldg(meta + warp + 1);
  }
  for (int b = warp; b < n_blocks; b += W) {
    const int r0 = ma.x, e0 = ma.y, r1 = mb.x, e1 = mb.y;
    if (b + W < n_blocks) {
      ma = __ldg(meta + b + W);
      mb = __ldg(meta + b + W + 1);
    }
    if (e1 - e0 > 32 * K) {  // a single long row
      T s = T(0);
      for (int j = e0 + lane; j < e1; j += 32) s = s + val[j] * __ldg(x + ci[j]);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
      if (lane == 0) row_epilogue(ep, r0, s, y, acc);
      continue;
    }
    T v[K];
    int c[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      const int j = e0 + k * 32 + lane;
      c[k] = j < e1 ? __ldlu(ci + j) : 0;
      v[k] = j < e1 ? __ldlu(val + j) : T(0);
    }
    const int row = r0 + lane;
    int rb = 0, re = 0;
    if (row < r1) {
      rb = __ldg(rp + row) - e0;
      re = __ldg(rp + row + 1) - e0;
    }
#pragma unroll
    for (int k = 0; k < K; k++) {
      const int j = e0 + k * 32 + lane;
      if (j < e1) pw[k * 32 + lane] = mul_rn(v[k], __ldg(x + c[k]));
    }
    __syncwarp();
    if (row < r1) {
      T s = T(0);
      for (int j = rb; j < re; j++) s = add_rn(s, pw[j]);
      row_epilogue(ep, row, s, y, acc);
    }
    __syncwarp();
  }
  finish_epilogue(ep, acc);
}

// SELL-32 SpMV (sell.cu layout): thread per row, a warp per slice.  Entries
// are taken in chunks of C: C coalesced loads of column indices and values
// (last-use hint), then C gathers of x -- for a stencil matrix the k-th
// gathers of a warp hit 32 consecutive rows' k-th neighbours, so they
// coalesce as well -- then the row sum continues in stored (column) order,
// product and sum rounded separately: bit for bit the reference's row loop
// (mat_vec_mult.hpp:666-688).  Padding (column -1) is skipped.  With D16 the
// column indices are read as 16-bit offsets from the row (Sell::d_dcol): 2
// bytes of index per entry instead of 4.
template <typename T, int C, bool D16>
__global__ void __launch_bounds__(kBlock, 8)
    spmv_sell(int n, const int32_t* __restrict__ slice_ptr, const int32_t* __restrict__ col,
              const int16_t* __restrict__ dcol, const T* __restrict__ val,
              const T* __restrict__ x, T* __restrict__ y, EpiParams<T> ep) {
  if (ep.skip && ld_relaxed(ep.skip)) return;
  typedef typename AccOf<T, 1>::type R;
  R acc = R::zero();
  for (long long r = gtid(); r < n; r += gstride()) {
    const long long s = r >> 5;
    const int lane = (int)(r & 31);
    const int base = __ldg(slice_ptr + s);
    const int width = (__ldg(slice_ptr + s + 1) - base) >> 5;
    const int32_t* cp = col + base + lane;
    const int16_t* dp = dcol + base + lane;
    const T* vp = val + base + lane;
    T sum = T(0);
    for (int k0 = 0; k0 < width; k0 += C) {
      int c[C];
      T a[C], xv[C];
#pragma unroll
      for (int u = 0; u < C; u++) {
        const bool in = k0 + u < width;
        if (D16) {
          const int d = in ? (int)__ldlu(dp + 32 * (k0 + u)) : -32768;
          c[u] = d == -32768 ? -1 : (int)r + d;
        } else {
          c[u] = in ? __ldlu(cp + 32 * (k0 + u)) : -1;
        }
        a[u] = in ? __ldlu(vp + 32 * (k0 + u)) : T(0);
      }
#pragma unroll
      for (int u = 0; u < C; u++) xv[u] = c[u] >= 0 ? __ldg(x + c[u]) : T(0);
#pragma unroll
      for (int u = 0; u < C; u++)
        if (c[u] >= 0) sum = add_rn(sum, mul_rn(a[u], xv[u]));
    }
    row_epilogue(ep, (int)r, sum, y, acc);
  }
  finish_epilogue(ep, acc);
}

template <typename T>
void launch_group(int G, int grid, cudaStream_t st, int nrows, const int32_t* rows,
                  const int32_t* rp, const int32_t* ci, const T* v, const T* x, T* y,
                  const EpiParams<T>& ep) {
  switch (G) {
    case 2: spmv_group<T, 2><<<grid, kBlock, 0, st>>>(nrows, rows, rp, ci, v, x, y, ep); break;
    case 4: spmv_group<T, 4><<<grid, kBlock, 0, st>>>(nrows, rows, rp, ci, v, x, y, ep); break;
    case 8: spmv_group<T, 8><<<grid, kBlock, 0, st>>>(nrows, rows, rp, ci, v, x, y, ep); break;
    case 16: spmv_group<T, 16><<<grid, kBlock, 0, st>>>(nrows, rows, rp, ci, v, x, y, ep); break;
    case 32: spmv_group<T, 32><<<grid, kBlock, 0, st>>>(nrows, rows, rp, ci, v, x, y, ep); break;
    default: spmv_cta<T><<<grid, kBlock, 0, st>>>(nrows, rows, rp, ci, v, x, y, ep); break;
  }
}

int grid_for(Ctx* ctx, long long items_per_block_unit, long long count) {
  long long need = (count + items_per_block_unit - 1) / items_per_block_unit;
  long long cap = (long long)ctx->num_sms * 8;  // 8 resident 256-thread CTAs per SM
  if (need > cap) need = cap;
  if (need < 1) need = 1;
  return (int)need;
}

}  // namespace

int sm_count(Ctx* ctx) { return ctx->num_sms; }
unsigned* counter_slot(Ctx* ctx, int i) { return ctx->d_counters + i; }

mtlgpu_status csr_analyse(Csr* A) {
  Ctx* ctx = A->ctx;
  MTLGPU_TRY(dalloc(ctx, &A->d_diag, A->n_rows));
  unsigned long long* d_stats = nullptr;
  MTLGPU_TRY(dalloc(ctx, &d_stats, 2));
  MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(d_stats, 0, 2 * sizeof(unsigned long long), ctx->stream));
  if (A->n_rows > 0) {
    int grid = grid_for(ctx, kBlock, A->n_rows);
    csr_analyse_kernel<<<grid, kBlock, 0, ctx->stream>>>(A->n_rows, A->n_cols, A->nnz, A->d_rp,
                                                        A->d_ci, A->d_diag, d_stats, ctx->d_error);
    MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  }
  unsigned long long h_stats[2] = {0, 0};
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(h_stats, d_stats, sizeof(h_stats), cudaMemcpyDeviceToHost,
                                       ctx->stream));
  dfree(ctx, d_stats);
  MTLGPU_TRY(take_device_error(ctx));
  A->max_row = (int)h_stats[0];
  A->mean_row = A->n_rows ? double(h_stats[1]) / A->n_rows : 0.0;

  // SpMV layout.  SELL-32 where its padding is small (stencils: < 1 %);
  // otherwise CSR-stream row blocks (greedy: up to 32 rows and 32*kStreamK
  // entries; a longer row forms a block of its own).
  {
    std::vector<int32_t> h_rp(A->n_rows + 1);
    MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(h_rp.data(), A->d_rp, sizeof(int32_t) * (A->n_rows + 1),
                                         cudaMemcpyDeviceToHost, ctx->stream));
    MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    const long long padded = sell_padded_entries(A->n_rows, h_rp.data(), 0);
    A->spmv_kernel = (A->nnz > 0 && padded <= (long long)(kSellMaxPadding * A->nnz) &&
                      padded < (1ll << 31))
                         ? 2
                         : 0;
    if (const char* m = std::getenv("MTLGPU_SPMV")) {
      if (!std::strcmp(m, "stream")) A->spmv_kernel = 0;
      if (!std::strcmp(m, "group")) A->spmv_kernel = 1;
    }
    if (A->spmv_kernel == 2)
      MTLGPU_TRY(sell_build(ctx, A->n_rows, A->d_rp, A->d_ci, A->d_v, 0, true, false, false,
                            false, &A->sell));
    const int cap = 32 * kStreamK;
    std::vector<int2> blk;
    blk.reserve(A->n_rows / 16 + 2);
    int r = 0;
    while (r < A->n_rows) {
      blk.push_back(make_int2(r, h_rp[r]));
      int rows = 0, cnt = 0;
      while (r < A->n_rows && rows < 32) {
        const int len = h_rp[r + 1] - h_rp[r];
        if (rows > 0 && cnt + len > cap) break;
        cnt += len;
        rows++;
        r++;
        if (cnt > cap) break;
      }
    }
    blk.push_back(make_int2(A->n_rows, A->nnz));
    A->n_blk = (int)blk.size() - 1;
    MTLGPU_TRY(dalloc(ctx, &A->d_meta, blk.size()));
    MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(A->d_meta, blk.data(), sizeof(int2) * blk.size(),
                                         cudaMemcpyHostToDevice, ctx->stream));
    MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }

  int g = 2;
  while (g < A->mean_row && g < 32) g <<= 1;
  A->uniform_group = g;
  A->uniform = A->max_row <= 2 * g || A->max_row <= 32;
  if (A->uniform) {
    if (A->max_row <= 32 && A->max_row > 2 * g) {
      while (g < A->max_row) g <<= 1;
      A->uniform_group = g;
    }
    A->bins.clear();
    return MTLGPU_OK;
  }
  // Binned: stable sort of rows by bin id (cub radix sort keeps equal keys in
  // input order, so rows inside a bin stay ascending).
  int n = A->n_rows;
  int32_t *d_bin = nullptr, *d_rows = nullptr, *d_bin_sorted = nullptr;
  MTLGPU_TRY(dalloc(ctx, &d_bin, n));
  MTLGPU_TRY(dalloc(ctx, &d_rows, n));
  MTLGPU_TRY(dalloc(ctx, &d_bin_sorted, n));
  MTLGPU_TRY(dalloc(ctx, &A->d_bin_rows, n));
  row_bin_kernel<<<grid_for(ctx, kBlock, n), kBlock, 0, ctx->stream>>>(n, A->d_rp, d_bin, d_rows);
  size_t tmp_bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, d_bin, d_bin_sorted, d_rows, A->d_bin_rows, n,
                                  0, 3, ctx->stream);
  void* d_tmp = nullptr;
  MTLGPU_TRY(dalloc(ctx, reinterpret_cast<char**>(&d_tmp), tmp_bytes));
  cub::DeviceRadixSort::SortPairs(d_tmp, tmp_bytes, d_bin, d_bin_sorted, d_rows, A->d_bin_rows, n,
                                  0, 3, ctx->stream);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  std::vector<int32_t> h_bins(n);
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(h_bins.data(), d_bin_sorted, sizeof(int32_t) * n,
                                       cudaMemcpyDeviceToHost, ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  dfree(ctx, d_tmp);
  dfree(ctx, d_bin);
  dfree(ctx, d_rows);
  dfree(ctx, d_bin_sorted);
  A->bins.clear();
  int i = 0;
  while (i < n) {
    int b = h_bins[i], j = i;
    while (j < n && h_bins[j] == b) j++;
    SpmvBin bin;
    bin.group = b >= 6 ? 0 : (1 << b);
    bin.begin = i;
    bin.count = j - i;
    A->bins.push_back(bin);
    i = j;
  }
  return MTLGPU_OK;
}

mtlgpu_status csr_ensure_fp32(Csr* A) {
  if (A->d_v32 || A->nnz == 0) return MTLGPU_OK;
  Ctx* ctx = A->ctx;
  MTLGPU_TRY(dalloc(ctx, &A->d_v32, A->nnz));
  to_fp32_kernel<<<grid_for(ctx, kBlock, A->nnz), kBlock, 0, ctx->stream>>>(A->nnz, A->d_v,
                                                                            A->d_v32);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  if (A->spmv_kernel == 2)
    MTLGPU_TRY(sell_ensure_fp32(ctx, A->d_rp, A->d_ci, A->d_v, 0, &A->sell));
  return MTLGPU_OK;
}

template <typename T>
const T* csr_sell_values(Csr* A);
template <>
const double* csr_sell_values<double>(Csr* A) { return A->sell.d_val; }
template <>
const float* csr_sell_values<float>(Csr* A) { return A->sell.d_val32; }

template <typename T>
const T* csr_values(Csr* A);
template <>
const double* csr_values<double>(Csr* A) { return A->d_v; }
template <>
const float* csr_values<float>(Csr* A) { return A->d_v32; }

template <typename T>
mtlgpu_status spmv_launch(Csr* A, const T* x, T* y, const SpmvArgs& args) {
  Ctx* ctx = A->ctx;
  if (A->n_rows == 0) return MTLGPU_OK;
  const T* v = csr_values<T>(A);
  if (!v && A->nnz > 0) return MTLGPU_INVALID_ARG;
  EpiParams<T> ep;
  ep.epi = args.epi;
  ep.alpha = (T)args.alpha;
  ep.beta = (T)args.beta;
  ep.x2 = static_cast<const T*>(args.x2);
  ep.b = static_cast<const T*>(args.b);
  ep.out = args.out;
  ep.skip = args.skip;
  ep.partials = ctx->d_partials;
  ep.counter = counter_slot(ctx, 0);
  if (A->spmv_kernel == 2) {
    const T* sv = csr_sell_values<T>(A);
    if (!sv) return MTLGPU_INVALID_ARG;
    const int grid = grid_for(ctx, kBlock, A->n_rows);
    ep.part_off = 0;
    ep.part_total = grid;
    ep.final_launch = true;
    // 16-bit indices for FP64 values, and for FP32 values with rows wider
    // than 8 entries.  Measured: the 128^3 7-point FP64 product from 31.8 to
    // 28.7 us (cold L2: 43.5 to 38.3), while its FP32 product, back to back,
    // slows from 22.9 to 24.6; the 96^3 27-point FP32 product goes from 33.2
    // to 32.8 us (config-3 mixed solve 14.28 to 14.01 ms).
    if (A->sell.d_dcol && (sizeof(T) == 8 || A->sell.max_width > 8))
      spmv_sell<T, 8, true><<<grid, kBlock, 0, ctx->stream>>>(
          A->n_rows, A->sell.d_slice_ptr, A->sell.d_col, A->sell.d_dcol, sv, x, y, ep);
    else
      spmv_sell<T, 8, false><<<grid, kBlock, 0, ctx->stream>>>(
          A->n_rows, A->sell.d_slice_ptr, A->sell.d_col, A->sell.d_dcol, sv, x, y, ep);
    ctx->launches++;
    MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
    return MTLGPU_OK;
  }
  if (A->spmv_kernel == 0) {
    int grid = grid_for(ctx, kBlock / 32, A->n_blk);
    ep.part_off = 0;
    ep.part_total = grid;
    ep.final_launch = true;
    spmv_stream<T, kStreamK><<<grid, kBlock, 0, ctx->stream>>>(A->n_blk, A->d_meta, A->d_rp,
                                                              A->d_ci, v, x, y, ep);
    ctx->launches++;
    MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
    return MTLGPU_OK;
  }
  if (A->uniform) {
    const int G = A->uniform_group;
    int grid = grid_for(ctx, kBlock / G, A->n_rows);
    ep.part_off = 0;
    ep.part_total = grid;
    ep.final_launch = true;
    ctx->launches++;
    launch_group<T>(G, grid, ctx->stream, A->n_rows, nullptr, A->d_rp, A->d_ci, v, x, y, ep);
    MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
    return MTLGPU_OK;
  }
  // binned: partial slots are laid out bin after bin; the last launch reduces all
  std::vector<int> grids(A->bins.size());
  int total = 0;
  for (size_t k = 0; k < A->bins.size(); k++) {
    const SpmvBin& bn = A->bins[k];
    int per = bn.group ? kBlock / bn.group : 1;
    grids[k] = grid_for(ctx, per, bn.count);
    total += grids[k];
  }
  if (total > kMaxPartials) return MTLGPU_NOT_SUPPORTED;
  int off = 0;
  for (size_t k = 0; k < A->bins.size(); k++) {
    const SpmvBin& bn = A->bins[k];
    ep.part_off = off;
    ep.part_total = total;
    ep.final_launch = (k + 1 == A->bins.size());
    ctx->launches++;
    launch_group<T>(bn.group, grids[k], ctx->stream, bn.count, A->d_bin_rows + bn.begin, A->d_rp,
                    A->d_ci, v, x, y, ep);
    MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
    off += grids[k];
  }
  return MTLGPU_OK;
}

template mtlgpu_status spmv_launch<double>(Csr*, const double*, double*, const SpmvArgs&);

// Times the bit-exact SpMV layouts on this matrix (SELL-32 where its padding
// is at most 2 nnz, CSR-stream) with CUDA events, 20 products each after a
// warm-up, and keeps the fastest on the handle.  *choice: the kernel kept
// (0 CSR-stream, 2 SELL-32); ms[k]: its mean time per product (-1: not a
// candidate).
mtlgpu_status csr_autotune_spmv(Csr* A, int* choice, float* ms) {
  Ctx* ctx = A->ctx;
  ms[0] = ms[1] = ms[2] = -1.f;
  if (A->n_rows == 0 || A->nnz == 0) {
    *choice = A->spmv_kernel;
    return MTLGPU_OK;
  }
  if (A->spmv_kernel != 2 && !A->sell.d_slice_ptr) {
    std::vector<int32_t> h_rp(A->n_rows + 1);
    MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(h_rp.data(), A->d_rp, sizeof(int32_t) * (A->n_rows + 1),
                                         cudaMemcpyDeviceToHost, ctx->stream));
    MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    const long long padded = sell_padded_entries(A->n_rows, h_rp.data(), 0);
    if (padded <= 2ll * A->nnz && padded < (1ll << 31))
      MTLGPU_TRY(sell_build(ctx, A->n_rows, A->d_rp, A->d_ci, A->d_v, 0, true, false, false,
                            false, &A->sell));
  }
  double *x = nullptr, *y = nullptr;
  MTLGPU_TRY(dalloc(ctx, &x, A->n_cols));
  MTLGPU_TRY(dalloc(ctx, &y, A->n_rows));
  MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(x, 0, sizeof(double) * A->n_cols, ctx->stream));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int keep = A->spmv_kernel;
  int best = keep;
  float best_ms = 1e30f;
  SpmvArgs plain;
  for (int k : {2, 0}) {
    if (k == 2 && !A->sell.d_slice_ptr) continue;
    A->spmv_kernel = k;
    mtlgpu_status st = spmv_launch<double>(A, x, y, plain);
    cudaEventRecord(e0, ctx->stream);
    for (int r = 0; r < 20 && st == MTLGPU_OK; r++) st = spmv_launch<double>(A, x, y, plain);
    cudaEventRecord(e1, ctx->stream);
    cudaEventSynchronize(e1);
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    if (st != MTLGPU_OK) {
      A->spmv_kernel = keep;
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      dfree(ctx, x);
      dfree(ctx, y);
      return st;
    }
    ms[k] = t / 20;
    if (ms[k] < best_ms) best_ms = ms[k], best = k;
  }
  A->spmv_kernel = best;
  release_workspaces(A, nullptr);  // solver graphs captured the previous kernel
  if (best != 2 && A->sell.d_slice_ptr) sell_free(ctx, &A->sell);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  dfree(ctx, x);
  dfree(ctx, y);
  *choice = best;
  return take_device_error(ctx);
}
template mtlgpu_status spmv_launch<float>(Csr*, const float*, float*, const SpmvArgs&);

mtlgpu_status spmv_transposed_launch(Csr* A, const double* x, double* y) {
  MTLGPU_TRY(csr_ensure_transpose(A));
  Ctx* ctx = A->ctx;
  if (A->n_cols == 0) return MTLGPU_OK;
  EpiParams<double> ep{};
  ep.epi = EPI_AXPBY;
  ep.alpha = 1.0;
  ep.beta = 0.0;
  ep.partials = ctx->d_partials;
  ep.counter = counter_slot(ctx, 0);
  ep.final_launch = true;
  int G = A->uniform_group;
  int grid = grid_for(ctx, kBlock / G, A->n_cols);
  launch_group<double>(G, grid, ctx->stream, A->n_cols, nullptr, A->d_trp, A->d_tci, A->d_tv, x, y,
                       ep);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  return MTLGPU_OK;
}

}  // namespace mtlgpu
