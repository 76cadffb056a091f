// Pieces of a differentiable solve x = A^{-1} b.
//
// With a loss L(x), the adjoint lambda solves A^T lambda = dL/dx; then
//   dL/db       = lambda
//   dL/dA[i][j] = -lambda_i x_j        for every stored entry (i, j) of A,
// i.e. the gradient with respect to A's nonzero values lives on A's own
// pattern.  The adjoint solve reuses the preconditioned Krylov path
// (mtlgpu_solve); for an unsymmetric A it runs on the transposed handle that
// mtlgpu_csr_create_transpose builds.
#include "device.cuh"
#include "internal.h"

namespace mtlgpu {

using namespace dev;

namespace {

constexpr int kBlock = 256;

// grad[k] = -lambda[row(k)] * x[col(k)]; a warp per row keeps the pattern's
// entries of a row coalesced.
__global__ void __launch_bounds__(kBlock)
    values_grad_kernel(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                       const double* __restrict__ lambda, const double* __restrict__ x,
                       double* __restrict__ grad) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x / 32);
  for (long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32; r < n; r += warps) {
    const double l = lambda[r];
    for (int j = rp[r] + lane; j < rp[r + 1]; j += 32) grad[j] = -(l * x[ci[j]]);
  }
}

}  // namespace
}  // namespace mtlgpu

using namespace mtlgpu;

extern "C" mtlgpu_status mtlgpu_csr_values_grad(mtlgpu_csr* A, const double* d_lambda,
                                                const double* d_x, double* d_grad) {
  if (!A || (A->n_rows && (!d_lambda || !d_x)) || (A->nnz && !d_grad)) return MTLGPU_INVALID_ARG;
  Ctx* ctx = A->ctx;
  if (A->n_rows == 0 || A->nnz == 0) return MTLGPU_OK;
  const long long warps_needed = A->n_rows;
  const int grid = (int)std::min<long long>((warps_needed * 32 + kBlock - 1) / kBlock,
                                            (long long)ctx->num_sms * 16);
  values_grad_kernel<<<grid, kBlock, 0, ctx->stream>>>(A->n_rows, A->d_rp, A->d_ci, d_lambda, d_x,
                                                       d_grad);
  ctx->launches++;
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  return take_device_error(ctx);
}

extern "C" mtlgpu_status mtlgpu_csr_create_transpose(mtlgpu_csr* A, mtlgpu_csr** out) {
  if (!A || !out) return MTLGPU_INVALID_ARG;
  Ctx* ctx = A->ctx;
  int32_t *trp = nullptr, *tci = nullptr;
  double* tv = nullptr;
  MTLGPU_TRY(dalloc(ctx, &trp, A->n_cols + 1));
  MTLGPU_TRY(dalloc(ctx, &tci, A->nnz > 0 ? A->nnz : 1));
  MTLGPU_TRY(dalloc(ctx, &tv, A->nnz > 0 ? A->nnz : 1));
  mtlgpu_status st = csr_transpose(ctx, A->n_rows, A->n_cols, A->nnz, A->d_rp, A->d_ci, A->d_v,
                                   trp, tci, tv);
  if (st == MTLGPU_OK)
    st = mtlgpu_csr_create_device(static_cast<mtlgpu_ctx*>(ctx), A->n_cols, A->n_rows, A->nnz, trp,
                                  tci, tv, out);
  cudaStreamSynchronize(ctx->stream);
  dfree(ctx, trp);
  dfree(ctx, tci);
  dfree(ctx, tv);
  return st;
}
