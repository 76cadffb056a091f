// BLAS-1 kernels: dot (mtl/operation/dot.hpp:226-232), two_norm
// (two_norm.hpp:33-57), unary_dot (unary_dot.hpp:29-65), and the vector
// updates of vec_vec_aop_expr (mtl/vector/vec_vec_aop_expr.hpp:60-152).
//
// Streaming kernels: a grid of 8 CTAs per SM, 128-bit loads where the
// pointers allow, and a deterministic two-level reduction (fixed number of
// block partials summed by the last block to finish in a fixed order), so
// repeated calls on the same data give the same bits.
#include <algorithm>

#include "device.cuh"
#include "internal.h"

namespace mtlgpu {

using namespace dev;

namespace {

constexpr int kBlock = 256;

int vec_grid(Ctx* ctx, long long n) {
  long long need = (n + 2 * kBlock - 1) / (2 * kBlock);
  long long cap = (long long)ctx->num_sms * 8;
  return (int)std::max(1ll, std::min(need, cap));
}

// order 0: sum x*y; order 1: sum x*x (x == y)
__global__ void __launch_bounds__(kBlock)
    dot_kernel(long long n, const double* __restrict__ x, const double* __restrict__ y,
               double* out, void* partials, unsigned* counter) {
  typedef Sum<1> R;
  R acc = R::zero();
  const bool aligned = ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15) == 0;
  if (aligned) {
    const long long n2 = n / 2;
    const double2* x2 = reinterpret_cast<const double2*>(x);
    const double2* y2 = reinterpret_cast<const double2*>(y);
    for (long long i = gtid(); i < n2; i += gstride()) {
      const double2 a = x2[i], b = y2[i];
      acc.add_prod(0, a.x, b.x);
      acc.add_prod(0, a.y, b.y);
    }
    if (gtid() == 0 && (n & 1)) acc.add_prod(0, x[n - 1], y[n - 1]);
  } else {
    for (long long i = gtid(); i < n; i += gstride()) acc.add_prod(0, x[i], y[i]);
  }
  R bs = block_reduce(acc);
  R* parts = reinterpret_cast<R*>(partials);
  if (publish_partial(bs, parts, blockIdx.x, counter, gridDim.x)) {
    R tot = reduce_partials(parts, gridDim.x);
    if (threadIdx.x == 0) *out = tot.value(0);
  }
}

// y = alpha x + beta y   (beta == 0 never reads y)
__global__ void __launch_bounds__(kBlock)
    axpby_kernel(long long n, double alpha, const double* __restrict__ x, double beta,
                 double* __restrict__ y) {
  if (beta == 0.0) {
    for (long long i = gtid(); i < n; i += gstride()) y[i] = alpha * x[i];
  } else if (alpha == 1.0) {
    for (long long i = gtid(); i < n; i += gstride()) y[i] = x[i] + beta * y[i];
  } else if (beta == 1.0) {
    for (long long i = gtid(); i < n; i += gstride()) y[i] += alpha * x[i];
  } else {
    for (long long i = gtid(); i < n; i += gstride()) y[i] = alpha * x[i] + beta * y[i];
  }
}

}  // namespace

mtlgpu_status dot_launch(Ctx* ctx, int n, const double* x, const double* y, double* d_out,
                         int /*order*/) {
  if (n <= 0) {
    MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(d_out, 0, sizeof(double), ctx->stream));
    return MTLGPU_OK;
  }
  ctx->launches++;
  dot_kernel<<<vec_grid(ctx, n), kBlock, 0, ctx->stream>>>(n, x, y, d_out, ctx->d_partials,
                                                           counter_slot(ctx, 8));
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  return MTLGPU_OK;
}

mtlgpu_status axpby_launch(Ctx* ctx, int n, double alpha, const double* x, double beta,
                           double* y) {
  if (n <= 0) return MTLGPU_OK;
  axpby_kernel<<<vec_grid(ctx, n), kBlock, 0, ctx->stream>>>(n, alpha, x, beta, y);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  return MTLGPU_OK;
}

}  // namespace mtlgpu
