// BLAS-1 kernels: dot (mtl/operation/dot.hpp:226-232), two_norm
// (two_norm.hpp:33-57), unary_dot (unary_dot.hpp:29-65), and the vector
// updates of vec_vec_aop_expr (mtl/vector/vec_vec_aop_expr.hpp:60-152).
//
// Streaming kernels: a grid of 8 CTAs per SM, 128-bit loads where the
// pointers allow, and a deterministic two-level reduction (fixed number of
// block partials summed by the last block to finish in a fixed order), so
// repeated calls on the same data give the same bits.
#include <algorithm>
#include <mutex>

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

// ---------------------------------------------------------------------------
// Dot product for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc at all: code running where the device
// heap belongs to someone else (a host application's own pool, a plugin
// inside another runtime), or a loop that must not touch the allocator.
// mtlgpu_dot needs a context, and creating one allocates the reduction
// scratch.  mtlgpu_dot_noalloc runs the same kernel (dot_kernel, same grid,
// same reduction order, hence the same bits) with its scratch -- the block
// partial sums and the arrival counter -- in the file-scope array below, so
// the call allocates nothing.
//
// The array is a fixed 32 KiB + 256 B that every GPU loading this library
// keeps until the process exits.  It holds at most kNoAllocPartials partial
// sums; a call whose grid (min(ceil(n / 512), 8 * SM count)) would need more
// is rejected with MTLGPU_INCOMPATIBLE_SIZE (never the case on a B200, whose
// grid is at most 1184).  All calls on a device share the array: calls whose
// kernels overlap on the GPU (different streams, or different host threads
// without ordering) race on it and give wrong results.  The first call on each
// device does that device's set-up (cudaGetSymbolAddress of the array, with the
// device current); that first call should come before any stream capture.
// Later calls look the address up again, so a call after cudaDeviceReset
// (which reloads the module) uses the array's current address.
namespace {
constexpr int kNoAllocPartials = 4096;
constexpr size_t kNoAllocCounterOffset = kNoAllocPartials * sizeof(double);
}  // namespace

// partials[0 .. kNoAllocPartials) | arrival counter (unsigned)
static __device__ __align__(256) unsigned char g_dot_noalloc_scratch[kNoAllocCounterOffset + 256];

namespace {
// Per-device set-up: the device address of the array (in host code its name
// is only a stand-in, never a device address) and the SM count.
struct NoAllocDevice {
  bool ready = false;
  unsigned char* scratch = nullptr;
  int num_sms = 0;
};
constexpr int kNoAllocMaxDevices = 64;
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];
std::mutex g_noalloc_mutex;

mtlgpu_status noalloc_setup(int device, NoAllocDevice** out) {
  if (device < 0 || device >= kNoAllocMaxDevices) return MTLGPU_INVALID_ARG;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  NoAllocDevice& d = g_noalloc_dev[device];
  if (d.ready) {
    // A cudaDeviceReset reloads the module, which may place the array
    // elsewhere: look the address up again (cheap after the first time) and
    // keep the current one.
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_dot_noalloc_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return MTLGPU_CUDA_ERROR;
    }
    d.scratch = static_cast<unsigned char*>(p);
  } else {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_dot_noalloc_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return MTLGPU_CUDA_ERROR;
    }
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        sms <= 0) {
      cudaGetLastError();
      return MTLGPU_CUDA_ERROR;
    }
    d.scratch = static_cast<unsigned char*>(p);
    d.num_sms = sms;
    d.ready = true;
  }
  *out = &d;
  return MTLGPU_OK;
}
}  // namespace

extern "C" mtlgpu_status mtlgpu_dot_noalloc(int n, const double* d_x, const double* d_y,
                                            double* d_result, void* stream) {
  using namespace mtlgpu;
  if (n < 0 || !d_result || (n > 0 && (!d_x || !d_y))) return MTLGPU_INVALID_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) {
    cudaGetLastError();
    return MTLGPU_CUDA_ERROR;
  }
  NoAllocDevice* d = nullptr;
  mtlgpu_status s = noalloc_setup(device, &d);
  if (s != MTLGPU_OK) return s;
  if (n == 0) {
    if (cudaMemsetAsync(d_result, 0, sizeof(double), st) != cudaSuccess) {
      cudaGetLastError();
      return MTLGPU_CUDA_ERROR;
    }
    return MTLGPU_OK;
  }
  // the grid mtlgpu_dot uses on this device
  const long long need = ((long long)n + 2 * kBlock - 1) / (2 * kBlock);
  const long long grid = std::max(1ll, std::min(need, (long long)d->num_sms * 8));
  if (grid > kNoAllocPartials) return MTLGPU_INCOMPATIBLE_SIZE;
  unsigned* counter = reinterpret_cast<unsigned*>(d->scratch + kNoAllocCounterOffset);
  // the counter must start at zero (the array keeps the last call's contents)
  if (cudaMemsetAsync(counter, 0, sizeof(unsigned), st) != cudaSuccess) {
    cudaGetLastError();
    return MTLGPU_CUDA_ERROR;
  }
  dot_kernel<<<(int)grid, kBlock, 0, st>>>(n, d_x, d_y, d_result, d->scratch, counter);
  if (cudaGetLastError() != cudaSuccess) return MTLGPU_CUDA_ERROR;
  return MTLGPU_OK;
}
