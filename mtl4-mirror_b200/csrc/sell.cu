// SELL-32: a sliced-ELL copy of a CSR matrix (or of a factor's off-diagonal
// part) for the streaming kernels of sm_100a.
//
// Rows are cut into slices of 32 consecutive rows; slice s stores
// width_s = (longest row of the slice) columns of entries column-major:
// entry k of row r sits at slice_ptr[s] + 32 k + (r mod 32).  Shorter rows
// are padded with column -1 (skipped by every kernel, so a padded slot never
// enters an arithmetic operation).  A warp owns a slice: its k-th load of
// column indices / values is one coalesced 128 / 256-byte line, and for
// stencil matrices the k-th gathers of x of 32 consecutive rows share the same
// offset, so they coalesce too.  Entries keep their CSR order inside each row,
// so a row processed in k order is processed in the reference's order.
//
// Used by the SpMV (spmv.cu, for matrices whose padding is small) and by the
// Jacobi-iteration triangular solves (jacobi_sweep.cu, off-diagonal part with
// the diagonal kept apart).
#include <algorithm>
#include <cstdlib>
#include <vector>

#include "device.cuh"
#include "internal.h"

namespace mtlgpu {

using namespace dev;

namespace {

constexpr int kBlock = 256;

int grid_rows(Ctx* ctx, long long n) {
  long long need = (n + kBlock - 1) / kBlock;
  long long cap = (long long)ctx->num_sms * 8;
  return (int)std::max(1ll, std::min(need, cap));
}

// diag_pos: 0 = no stored diagonal (unit lower), 1 = first entry of the row,
// 2 = last entry of the row.
__device__ __forceinline__ void off_range(const int32_t* rp, int r, int diag_pos, int& b, int& e) {
  b = rp[r];
  e = rp[r + 1];
  if (diag_pos == 1 && e > b) b++;
  if (diag_pos == 2 && e > b) e--;
}

// Slice widths (in entries per row) -> width32[s] = 32 * width.
__global__ void slice_width_kernel(int n, int n_slices, const int32_t* __restrict__ rp,
                                   int diag_pos, int32_t* __restrict__ width32) {
  const int lane = threadIdx.x & 31;
  const long long warp0 = gtid() >> 5, nwarps = gstride() >> 5;
  for (long long s = warp0; s < n_slices; s += nwarps) {
    const long long r = s * 32 + lane;
    int cnt = 0;
    if (r < n) {
      int b, e;
      off_range(rp, (int)r, diag_pos, b, e);
      cnt = e - b;
    }
    for (int off = 16; off > 0; off >>= 1) cnt = max(cnt, __shfl_xor_sync(0xffffffffu, cnt, off));
    if (lane == 0) width32[s] = 32 * cnt;
  }
}

// The stored diagonal of row r (diag_pos 1: first entry, 2: last entry).
__device__ __forceinline__ double diag_of(const int32_t* rp, const double* v, int r,
                                          int diag_pos) {
  return v[diag_pos == 1 ? rp[r] : rp[r + 1] - 1];
}

// Scatter the off-diagonal entries into the slices; pad; copy the diagonal.
// scale_cols: each entry (r, c) is stored multiplied by the stored diagonal
// of row c (the factor N D of the Jacobi solves); with round64 both factors
// are the float values, whose product a double holds exactly.
__global__ void slice_fill_kernel(int n, const int32_t* __restrict__ rp,
                                  const int32_t* __restrict__ ci, const double* __restrict__ v,
                                  int diag_pos, const int32_t* __restrict__ slice_ptr,
                                  int32_t* __restrict__ col, double* __restrict__ val,
                                  float* __restrict__ val32, double* __restrict__ dinv,
                                  float* __restrict__ dinv32, bool round64, bool scale_cols) {
  for (long long r = gtid(); r < n; r += gstride()) {
    const long long s = r >> 5;
    const int lane = (int)(r & 31);
    const int base = slice_ptr[s], width = (slice_ptr[s + 1] - base) >> 5;
    int b, e;
    off_range(rp, (int)r, diag_pos, b, e);
    for (int k = 0; k < width; k++) {
      const int j = b + k;
      const long long o = base + 32ll * k + lane;
      const bool real = j < e;
      col[o] = real ? ci[j] : -1;
      double a = real ? v[j] : 0.0;
      // round64: the double copy holds the float values (FP32 factors are
      // applied at their float values, as the exact sweeps do)
      if (round64) a = (double)(float)a;
      if (scale_cols && real) {
        double dc = diag_of(rp, v, ci[j], diag_pos);
        if (round64) dc = (double)(float)dc;
        a *= dc;
      }
      if (val) val[o] = a;
      if (val32) val32[o] = (float)a;
    }
    if (diag_pos) {
      const double d = diag_of(rp, v, (int)r, diag_pos);
      if (dinv) dinv[r] = round64 ? (double)(float)d : d;
      if (dinv32) dinv32[r] = (float)d;
    }
  }
}

// Largest |column - row| over the stored entries (padding skipped).
__global__ void delta_max_kernel(int n, const int32_t* __restrict__ slice_ptr,
                                 const int32_t* __restrict__ col, int* __restrict__ out) {
  int m = 0;
  for (long long r = gtid(); r < n; r += gstride()) {
    const long long s = r >> 5;
    const int lane = (int)(r & 31);
    const int base = slice_ptr[s], width = (slice_ptr[s + 1] - base) >> 5;
    for (int k = 0; k < width; k++) {
      const int c = col[base + 32 * k + lane];
      if (c >= 0) m = max(m, abs(c - (int)r));
    }
  }
  for (int off = 16; off > 0; off >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// 16-bit column deltas: column - row, padding -32768.
__global__ void dcol_fill_kernel(int n, const int32_t* __restrict__ slice_ptr,
                                 const int32_t* __restrict__ col, int16_t* __restrict__ dcol) {
  for (long long r = gtid(); r < n; r += gstride()) {
    const long long s = r >> 5;
    const int lane = (int)(r & 31);
    const int base = slice_ptr[s], width = (slice_ptr[s + 1] - base) >> 5;
    for (int k = 0; k < width; k++) {
      const int o = base + 32 * k + lane;
      const int c = col[o];
      dcol[o] = (int16_t)(c >= 0 ? c - (int)r : -32768);
    }
  }
}

}  // namespace

// Builds J->d_dcol when every stored entry lies within 32,767 of its row
// (MTLGPU_SELL_INDEX=32 keeps 32-bit indices only).
static mtlgpu_status sell_build_deltas(Ctx* ctx, Sell* J) {
  if (const char* m = std::getenv("MTLGPU_SELL_INDEX"))
    if (std::atoi(m) == 32) return MTLGPU_OK;
  int* d_max = nullptr;
  MTLGPU_TRY(dalloc(ctx, &d_max, 1));
  MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(d_max, 0, sizeof(int), ctx->stream));
  delta_max_kernel<<<grid_rows(ctx, J->n), kBlock, 0, ctx->stream>>>(J->n, J->d_slice_ptr,
                                                                      J->d_col, d_max);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  int h_max = 0;
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(&h_max, d_max, sizeof(int), cudaMemcpyDeviceToHost,
                                       ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  dfree(ctx, d_max);
  if (h_max > 32767) return MTLGPU_OK;
  MTLGPU_TRY(dalloc(ctx, &J->d_dcol, J->n_ent));
  dcol_fill_kernel<<<grid_rows(ctx, J->n), kBlock, 0, ctx->stream>>>(J->n, J->d_slice_ptr,
                                                                      J->d_col, J->d_dcol);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  return MTLGPU_OK;
}

// Padded entry count of the SELL-32 form of a CSR pattern (diag_pos as
// sell_build), from host row pointers.
long long sell_padded_entries(int n, const int32_t* h_rp, int diag_pos) {
  long long total = 0;
  for (int s = 0; s * 32 < n; s++) {
    int w = 0;
    for (int r = s * 32; r < std::min(n, s * 32 + 32); r++) {
      int len = h_rp[r + 1] - h_rp[r];
      if (diag_pos && len > 0) len--;
      w = std::max(w, len);
    }
    total += 32ll * w;
  }
  return total;
}

// fp64 / fp32: which value copies to hold; round64: the double copy holds
// the float-rounded values (FP32 factors); scale_cols: entries stored times
// the stored diagonal of their column's row (needs diag_pos != 0).
mtlgpu_status sell_build(Ctx* ctx, int n, const int32_t* d_rp, const int32_t* d_ci,
                         const double* d_v, int diag_pos, bool fp64, bool fp32, bool round64,
                         bool scale_cols, Sell* J) {
  J->n = n;
  J->round64 = round64;
  J->col_scaled = scale_cols && diag_pos != 0;
  J->unit_diag = diag_pos == 0;
  J->n_slices = (n + 31) / 32;
  if (n == 0) return MTLGPU_OK;
  int32_t* d_w = nullptr;
  MTLGPU_TRY(dalloc(ctx, &d_w, J->n_slices + 1));
  MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(d_w, 0, sizeof(int32_t) * (J->n_slices + 1), ctx->stream));
  slice_width_kernel<<<grid_rows(ctx, 32ll * J->n_slices), kBlock, 0, ctx->stream>>>(
      n, J->n_slices, d_rp, diag_pos, d_w);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  MTLGPU_TRY(dalloc(ctx, &J->d_slice_ptr, J->n_slices + 1));
  MTLGPU_TRY(scan_i32(ctx, d_w, J->d_slice_ptr, J->n_slices + 1));
  {
    std::vector<int32_t> hw(J->n_slices);
    MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(hw.data(), d_w, sizeof(int32_t) * J->n_slices,
                                         cudaMemcpyDeviceToHost, ctx->stream));
    MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    int mx = 0;
    for (int32_t w : hw) mx = std::max(mx, (int)(w / 32));
    J->max_width = mx;
  }
  dfree(ctx, d_w);
  int total = 0;
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(&total, J->d_slice_ptr + J->n_slices, sizeof(int),
                                       cudaMemcpyDeviceToHost, ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (total < 0) return MTLGPU_NOT_SUPPORTED;  // more than 2^31 padded entries
  J->n_ent = total;
  MTLGPU_TRY(dalloc(ctx, &J->d_col, total));
  if (fp64) MTLGPU_TRY(dalloc(ctx, &J->d_val, total));
  if (fp32) MTLGPU_TRY(dalloc(ctx, &J->d_val32, total));
  if (diag_pos) {
    if (fp64) MTLGPU_TRY(dalloc(ctx, &J->d_dinv, n));
    if (fp32) MTLGPU_TRY(dalloc(ctx, &J->d_dinv32, n));
  }
  slice_fill_kernel<<<grid_rows(ctx, n), kBlock, 0, ctx->stream>>>(
      n, d_rp, d_ci, d_v, diag_pos, J->d_slice_ptr, J->d_col, J->d_val, J->d_val32, J->d_dinv,
      J->d_dinv32, J->round64, J->col_scaled);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  return sell_build_deltas(ctx, J);
}

void sell_free(Ctx* ctx, Sell* J) {
  dfree(ctx, J->d_slice_ptr);
  dfree(ctx, J->d_col);
  dfree(ctx, J->d_dcol);
  dfree(ctx, J->d_val);
  dfree(ctx, J->d_val32);
  dfree(ctx, J->d_dinv);
  dfree(ctx, J->d_dinv32);
  *J = Sell();
}

// New values on the same pattern (mtlgpu_csr_set_values).
mtlgpu_status sell_refill(Ctx* ctx, const int32_t* d_rp, const int32_t* d_ci, const double* d_v,
                          int diag_pos, Sell* J) {
  if (J->n == 0) return MTLGPU_OK;
  slice_fill_kernel<<<grid_rows(ctx, J->n), kBlock, 0, ctx->stream>>>(
      J->n, d_rp, d_ci, d_v, diag_pos, J->d_slice_ptr, J->d_col, J->d_val, J->d_val32, J->d_dinv,
      J->d_dinv32, J->round64, J->col_scaled);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  return MTLGPU_OK;
}

// Adds the float copy of the values (mixed-precision solves) when missing.
mtlgpu_status sell_ensure_fp32(Ctx* ctx, const int32_t* d_rp, const int32_t* d_ci,
                               const double* d_v, int diag_pos, Sell* J) {
  if (J->n == 0 || J->d_val32) return MTLGPU_OK;
  MTLGPU_TRY(dalloc(ctx, &J->d_val32, J->n_ent));
  if (diag_pos) MTLGPU_TRY(dalloc(ctx, &J->d_dinv32, J->n));
  return sell_refill(ctx, d_rp, d_ci, d_v, diag_pos, J);
}

}  // namespace mtlgpu
