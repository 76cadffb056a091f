// Batched PCG: many independent SPD systems in one solve.
//
// Each system s follows itl::cg(A_s, x_s, b_s, P_s, iter_s) (itl/krylov/
// cg.hpp:75-112) with iter_s = basic_iteration(b_s, max_iter, rtol, atol)
// (itl/iteration/basic_iteration.hpp:31-39): the systems are the diagonal
// blocks of one block-diagonal CSR matrix, so the preconditioner (Jacobi,
// IC(0), ILU(0): no fill crosses a block) and the SpMV run once over all of
// them, while every system keeps its own scalars (rho, alpha, beta, the
// residual, its iteration count and its stopping decision) in device memory.
//
// Kernels: one CTA per system for everything that reduces over a system --
// rho = r.z with p = z + beta p, and p.q with x += alpha p, r -= alpha q and
// r.r -- so a system's reductions need no cross-CTA step and are
// deterministic.  A system that has stopped keeps its x; its CTAs return at
// once.  The host checks a stopped-systems counter every few iterations.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "device.cuh"
#include "internal.h"

namespace mtlgpu {

using namespace dev;

namespace {

constexpr int kBlock = 256;

struct BatchSys {
  double rho, rr, norm_b, resid;
  double tol_abs;  // > 0: stop when resid <= tol_abs (inner solves of the refinement)
  int it, done, error, pad;
};

// Outer FP64 state of one system in the refined (FP32 inner) batched solve.
struct BatchOuter {
  double resid, norm_b;
  int done, error, outer, inner_total;
};

__device__ __forceinline__ double block_sum(double v) {
  Sum<1> a = Sum<1>::zero();
  a.add(0, v);
  return block_reduce(a).value(0);
}

__device__ __forceinline__ bool converged(const BatchSys& S, double resid, double rtol,
                                          double atol) {
  if (S.tol_abs > 0) return resid <= S.tol_abs;
  return S.norm_b == 0 ? resid <= atol : (resid <= rtol * S.norm_b || resid <= atol);
}

// Rows of system s must only reference columns of system s.
__global__ void __launch_bounds__(kBlock)
    batch_check_kernel(const int32_t* __restrict__ off, const int32_t* __restrict__ rp,
                       const int32_t* __restrict__ ci, int* err) {
  const int s = blockIdx.x, lo = off[s], hi = off[s + 1];
  for (int r = lo + threadIdx.x; r < hi; r += blockDim.x)
    for (int j = rp[r]; j < rp[r + 1]; ++j)
      if (ci[j] < lo || ci[j] >= hi) atomicCAS(err, 0, (int)MTLGPU_INVALID_ARG);
}

// r = b - A x (Ax given), rr, ||b||; the loop-top termination test.
__global__ void __launch_bounds__(kBlock)
    batch_init_kernel(const int32_t* __restrict__ off, const double* __restrict__ b,
                      const double* __restrict__ ax, double* __restrict__ r, BatchSys* sys,
                      double rtol, double atol, int max_iter, unsigned* n_done) {
  const int s = blockIdx.x, lo = off[s], hi = off[s + 1];
  double rr = 0, bb = 0;
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    const double v = b[i] - ax[i];
    r[i] = v;
    rr += v * v;
    bb += b[i] * b[i];
  }
  rr = block_sum(rr);
  __syncthreads();
  bb = block_sum(bb);
  if (threadIdx.x == 0) {
    BatchSys S{};
    S.rr = rr;
    S.norm_b = sqrt(bb);
    S.resid = sqrt(fabs(rr));
    if (converged(S, S.resid, rtol, atol)) {
      S.done = 1;
    } else if (max_iter <= 0) {
      S.done = 1;
      S.error = 1;
    }
    if (S.done) atomicAdd(n_done, 1u);
    sys[s] = S;
  }
}

// ++iter; rho = r.z; p = z (first iteration) or z + (rho / rho_1) p
template <typename T>
__global__ void __launch_bounds__(kBlock)
    batch_rho_p_kernel(const int32_t* __restrict__ off, const T* __restrict__ r,
                       const T* __restrict__ z, T* __restrict__ p, BatchSys* sys) {
  const int s = blockIdx.x;
  if (sys[s].done) return;
  const int lo = off[s], hi = off[s + 1];
  double rho = 0;
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) rho += (double)r[i] * (double)z[i];
  rho = block_sum(rho);
  __shared__ double beta_s;
  __shared__ int first_s;
  if (threadIdx.x == 0) {
    BatchSys& S = sys[s];
    S.it += 1;
    first_s = S.it <= 1;
    beta_s = first_s ? 0.0 : rho / S.rho;
    S.rho = rho;
  }
  __syncthreads();
  const T beta = (T)beta_s;
  if (first_s) {
    for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) p[i] = z[i];
  } else {
    for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) p[i] = z[i] + beta * p[i];
  }
}

// alpha = rho / p.q; x += alpha p; r -= alpha q; rr = r.r; termination test
template <typename T>
__global__ void __launch_bounds__(kBlock)
    batch_update_kernel(const int32_t* __restrict__ off, const T* __restrict__ p,
                        const T* __restrict__ q, T* __restrict__ x, T* __restrict__ r,
                        BatchSys* sys, double rtol, double atol, int max_iter,
                        unsigned* n_done) {
  const int s = blockIdx.x;
  if (sys[s].done) return;
  const int lo = off[s], hi = off[s + 1];
  double pq = 0;
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) pq += (double)p[i] * (double)q[i];
  pq = block_sum(pq);
  __shared__ double alpha_s;
  if (threadIdx.x == 0) alpha_s = sys[s].rho / pq;
  __syncthreads();
  const T alpha = (T)alpha_s;
  double rr = 0;
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    x[i] += alpha * p[i];
    const T v = r[i] - alpha * q[i];
    r[i] = v;
    rr += (double)v * (double)v;
  }
  rr = block_sum(rr);
  if (threadIdx.x == 0) {
    BatchSys& S = sys[s];
    S.rr = rr;
    S.resid = sqrt(fabs(rr));
    if (converged(S, S.resid, rtol, atol)) {
      S.done = 1;
    } else if (S.it >= max_iter) {
      S.done = 1;
      S.error = 1;
    }
    if (S.done) atomicAdd(n_done, 1u);
  }
}

// Refinement step of system s: r = b - A x in FP64 (Ax given), its norm and
// the FP64 stopping test; for a running system the FP32 inner problem
// A d = r / ||r|| from d = 0, asking at most inner_rtol and at least half the
// reduction still needed.
__global__ void __launch_bounds__(kBlock)
    batch_outer_kernel(const int32_t* __restrict__ off, const double* __restrict__ b,
                       const double* __restrict__ ax, float* __restrict__ r32,
                       float* __restrict__ d32, BatchOuter* outer, BatchSys* sys, double rtol,
                       double atol, double inner_rtol, int max_outer, int max_iter,
                       unsigned* n_done) {
  const int s = blockIdx.x, lo = off[s], hi = off[s + 1];
  __shared__ double resid_s;
  __shared__ int run_s;
  if (outer[s].done) {
    if (threadIdx.x == 0) {
      sys[s].done = 1;
      atomicAdd(n_done, 1u);
    }
    return;
  }
  double rr = 0, bb = 0;
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    const double v = b[i] - ax[i];
    rr += v * v;
    bb += b[i] * b[i];
  }
  rr = block_sum(rr);
  __syncthreads();
  bb = block_sum(bb);
  if (threadIdx.x == 0) {
    BatchOuter& O = outer[s];
    if (O.outer == 0) O.norm_b = sqrt(bb);
    O.resid = sqrt(rr);
    BatchSys probe{};
    probe.norm_b = O.norm_b;
    const bool conv = converged(probe, O.resid, rtol, atol);
    if (conv || O.outer >= max_outer || O.inner_total >= max_iter) {
      O.done = 1;
      O.error = conv ? 0 : 1;
    }
    BatchSys S{};
    S.done = O.done;
    S.norm_b = 1.0;
    const double target = O.norm_b == 0 ? atol : fmax(rtol * O.norm_b, atol);
    S.tol_abs = fmax(inner_rtol, fmin(0.5, 0.5 * target / O.resid));
    sys[s] = S;
    if (O.done) atomicAdd(n_done, 1u);
    resid_s = O.resid;
    run_s = !O.done;
  }
  __syncthreads();
  if (!run_s) return;
  const double scale = 1.0 / resid_s;
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    r32[i] = (float)((b[i] - ax[i]) * scale);
    d32[i] = 0.f;
  }
}

// x += ||r|| d for every system that ran an inner solve
__global__ void __launch_bounds__(kBlock)
    batch_refine_kernel(const int32_t* __restrict__ off, double* __restrict__ x,
                        const float* __restrict__ d32, BatchOuter* outer,
                        const BatchSys* sys) {
  const int s = blockIdx.x;
  if (outer[s].done) return;
  const int lo = off[s], hi = off[s + 1];
  const double scale = outer[s].resid;
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) x[i] += scale * (double)d32[i];
  __syncthreads();
  if (threadIdx.x == 0) {
    outer[s].outer += 1;
    outer[s].inner_total += sys[s].it;
  }
}

// ||b - A x|| per system (Ax given)
__global__ void __launch_bounds__(kBlock)
    batch_true_resid_kernel(const int32_t* __restrict__ off, const double* __restrict__ b,
                            const double* __restrict__ ax, double* out) {
  const int s = blockIdx.x, lo = off[s], hi = off[s + 1];
  double rr = 0;
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    const double v = b[i] - ax[i];
    rr += v * v;
  }
  rr = block_sum(rr);
  if (threadIdx.x == 0) out[s] = sqrt(rr);
}

}  // namespace

// Rejects a row of system s referencing a column outside system s.
mtlgpu_status batch_check(Csr* A, int count, const int32_t* h_off) {
  Ctx* ctx = A->ctx;
  int32_t* d_off = nullptr;
  MTLGPU_TRY(dalloc(ctx, &d_off, count + 1));
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(d_off, h_off, sizeof(int32_t) * (count + 1),
                                       cudaMemcpyHostToDevice, ctx->stream));
  batch_check_kernel<<<count, kBlock, 0, ctx->stream>>>(d_off, A->d_rp, A->d_ci, ctx->d_error);
  ctx->launches++;
  dfree(ctx, d_off);
  return take_device_error(ctx);
}

// FP32 inner batched PCG with FP64 iterative refinement, per system: the
// outer loop (FP64 residual, stopping test, x += ||r|| d) runs for all
// systems at once, and systems that have converged sit out.
mtlgpu_status solve_batched_mixed(Csr* A, Pc* P, int count, const int32_t* h_off, double* d_x,
                                  const double* d_b, const mtlgpu_iter_params* prm,
                                  mtlgpu_iter_result* res) {
  Ctx* ctx = A->ctx;
  if (P && P->kind != MTLGPU_PC_IDENTITY && P->prec != MTLGPU_FP32) return MTLGPU_INVALID_ARG;
  MTLGPU_TRY(csr_ensure_fp32(A));
  const int n = A->n_rows;
  const double rtol = prm->rtol, atol = prm->atol;
  const double inner_rtol = prm->inner_rtol > 0 ? prm->inner_rtol : 1e-6;
  const int max_outer = prm->max_outer > 0 ? prm->max_outer : 30;
  const int inner_max = prm->inner_max_iter > 0 ? prm->inner_max_iter : prm->max_iter;

  int32_t* d_off = nullptr;
  double *q64 = nullptr, *d_tr = nullptr;
  float *r32 = nullptr, *z32 = nullptr, *p32 = nullptr, *q32 = nullptr, *d32 = nullptr;
  BatchSys* sys = nullptr;
  BatchOuter* outer = nullptr;
  unsigned* n_done = nullptr;
  unsigned* h_done = nullptr;
  mtlgpu_status st = MTLGPU_OK;
  auto cleanup = [&]() {
    dfree(ctx, d_off);
    dfree(ctx, q64);
    dfree(ctx, d_tr);
    dfree(ctx, r32);
    dfree(ctx, z32);
    dfree(ctx, p32);
    dfree(ctx, q32);
    dfree(ctx, d32);
    dfree(ctx, sys);
    dfree(ctx, outer);
    dfree(ctx, n_done);
    if (h_done) cudaFreeHost(h_done);
  };
#define MTLGPU_BTRY(call)  \
  do {                     \
    st = (call);           \
    if (st != MTLGPU_OK) { \
      cleanup();           \
      return st;           \
    }                      \
  } while (0)
#define MTLGPU_BTRY_CUDA(call) \
  MTLGPU_BTRY(((call) == cudaSuccess) ? MTLGPU_OK : set_cuda_error(ctx, cudaGetLastError(), #call))
  MTLGPU_BTRY(dalloc(ctx, &d_off, count + 1));
  MTLGPU_BTRY(dalloc(ctx, &q64, n));
  MTLGPU_BTRY(dalloc(ctx, &d_tr, count));
  MTLGPU_BTRY(dalloc(ctx, &r32, n));
  MTLGPU_BTRY(dalloc(ctx, &z32, n));
  MTLGPU_BTRY(dalloc(ctx, &p32, n));
  MTLGPU_BTRY(dalloc(ctx, &q32, n));
  MTLGPU_BTRY(dalloc(ctx, &d32, n));
  MTLGPU_BTRY(dalloc(ctx, &sys, count));
  MTLGPU_BTRY(dalloc(ctx, &outer, count));
  MTLGPU_BTRY(dalloc(ctx, &n_done, 1));
  MTLGPU_BTRY_CUDA(cudaMallocHost(&h_done, sizeof(unsigned)));
  MTLGPU_BTRY_CUDA(cudaMemcpyAsync(d_off, h_off, sizeof(int32_t) * (count + 1),
                                   cudaMemcpyHostToDevice, ctx->stream));
  MTLGPU_BTRY_CUDA(cudaMemsetAsync(outer, 0, sizeof(BatchOuter) * count, ctx->stream));
  batch_check_kernel<<<count, kBlock, 0, ctx->stream>>>(d_off, A->d_rp, A->d_ci, ctx->d_error);
  ctx->launches++;
  MTLGPU_BTRY(take_device_error(ctx));
  SpmvArgs plain;
  auto all_done = [&](bool& done) -> mtlgpu_status {
    if (cudaMemcpyAsync(h_done, n_done, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess)
      return set_cuda_error(ctx, cudaGetLastError(), "batched refinement");
    done = (int)*h_done >= count;
    return MTLGPU_OK;
  };
  bool interrupted = false;
  for (int step = 0; step <= max_outer; ++step) {
    MTLGPU_BTRY(spmv_launch<double>(A, d_x, q64, plain));
    MTLGPU_BTRY_CUDA(cudaMemsetAsync(n_done, 0, sizeof(unsigned), ctx->stream));
    batch_outer_kernel<<<count, kBlock, 0, ctx->stream>>>(d_off, d_b, q64, r32, d32, outer, sys,
                                                          rtol, atol, inner_rtol, max_outer,
                                                          prm->max_iter, n_done);
    ctx->launches++;
    bool done = false;
    MTLGPU_BTRY(all_done(done));
    if (done) break;
    if (prm->h_interrupt && *prm->h_interrupt) {
      interrupted = true;
      break;
    }
    MTLGPU_BTRY_CUDA(cudaMemsetAsync(p32, 0, sizeof(float) * n, ctx->stream));
    for (int k = 0; k < inner_max; ++k) {
      if ((k & 7) == 7) {
        MTLGPU_BTRY(all_done(done));
        if (done) break;
      }
      if (P && P->kind != MTLGPU_PC_IDENTITY) {
        MTLGPU_BTRY(pc_apply_t<float>(P, r32, z32, false, nullptr, false, false));
      } else {
        MTLGPU_BTRY_CUDA(cudaMemcpyAsync(z32, r32, sizeof(float) * n, cudaMemcpyDeviceToDevice,
                                         ctx->stream));
      }
      batch_rho_p_kernel<float><<<count, kBlock, 0, ctx->stream>>>(d_off, r32, z32, p32, sys);
      MTLGPU_BTRY(spmv_launch<float>(A, p32, q32, plain));
      batch_update_kernel<float><<<count, kBlock, 0, ctx->stream>>>(d_off, p32, q32, d32, r32, sys,
                                                                    0.0, 0.0, inner_max, n_done);
      ctx->launches += 2;
      MTLGPU_BTRY_CUDA(cudaGetLastError());
    }
    batch_refine_kernel<<<count, kBlock, 0, ctx->stream>>>(d_off, d_x, d32, outer, sys);
    ctx->launches++;
  }
  MTLGPU_BTRY(spmv_launch<double>(A, d_x, q64, plain));
  batch_true_resid_kernel<<<count, kBlock, 0, ctx->stream>>>(d_off, d_b, q64, d_tr);
  ctx->launches++;
  std::vector<BatchOuter> ho(count);
  std::vector<double> htr(count);
  MTLGPU_BTRY_CUDA(cudaMemcpyAsync(ho.data(), outer, sizeof(BatchOuter) * count,
                                   cudaMemcpyDeviceToHost, ctx->stream));
  MTLGPU_BTRY_CUDA(cudaMemcpyAsync(htr.data(), d_tr, sizeof(double) * count,
                                   cudaMemcpyDeviceToHost, ctx->stream));
  MTLGPU_BTRY_CUDA(cudaStreamSynchronize(ctx->stream));
  MTLGPU_BTRY(take_device_error(ctx));
  bool any_max = false;
  for (int s = 0; s < count; ++s) {
    mtlgpu_iter_result& R = res[s];
    std::memset(&R, 0, sizeof(R));
    R.iterations = ho[s].inner_total;
    R.outer_iterations = ho[s].outer;
    R.error = ho[s].done ? ho[s].error : 1;
    R.status = R.error ? MTLGPU_MAX_ITER : (interrupted ? MTLGPU_INTERRUPTED : MTLGPU_OK);
    R.resid = ho[s].resid;
    R.norm_r0 = ho[s].norm_b;
    R.true_resid = htr[s];
    any_max |= R.error != 0;
  }
  cleanup();
#undef MTLGPU_BTRY
#undef MTLGPU_BTRY_CUDA
  if (interrupted) return MTLGPU_INTERRUPTED;
  return any_max ? MTLGPU_MAX_ITER : MTLGPU_OK;
}

mtlgpu_status solve_batched_impl(int method, Csr* A, Pc* P, int count, const int32_t* h_off,
                                 double* d_x, const double* d_b, const mtlgpu_iter_params* prm,
                                 mtlgpu_iter_result* res) {
  Ctx* ctx = A->ctx;
  if (method != MTLGPU_CG) return MTLGPU_NOT_SUPPORTED;
  if (count <= 0 || !h_off || !d_x || !d_b || !prm || !res) return MTLGPU_INVALID_ARG;
  if (A->n_rows != A->n_cols) return MTLGPU_NOT_SQUARE;
  if (P && P->A != A) return MTLGPU_INVALID_ARG;
  if (h_off[0] != 0 || h_off[count] != A->n_rows) return MTLGPU_INCOMPATIBLE_SIZE;
  for (int s = 0; s < count; ++s)
    if (h_off[s + 1] < h_off[s]) return MTLGPU_INVALID_ARG;
  if (batched_cluster_supported(P)) {
    MTLGPU_TRY(batch_check(A, count, h_off));
    int cs = A->batch_cs, g = A->batch_g;
    int small = A->batch_small;
    // MTLGPU_BATCH_SHAPE="CTAs,lanes[,small rows]" overrides the tuned shape
    // (testing); lanes 1 selects the CSR-stream SpMV
    if (const char* m = std::getenv("MTLGPU_BATCH_SHAPE")) {
      int c2 = 0, g2 = 0, s2 = -1;
      const int k = std::sscanf(m, "%d,%d,%d", &c2, &g2, &s2);
      if (k >= 2 && (c2 == 1 || c2 == 2 || c2 == 4 || c2 == 8) &&
          (g2 == 1 || g2 == 4 || g2 == 8 || g2 == 16 || g2 == 32)) {
        cs = c2, g = g2;
        if (k == 3 && s2 >= 0) small = s2;
      }
    }
    return solve_batched_cluster(A, P, count, h_off, d_x, d_b, prm, res, cs, g, small, nullptr);
  }
  if (prm->mode == MTLGPU_SOLVE_MIXED_REFINED)
    return solve_batched_mixed(A, P, count, h_off, d_x, d_b, prm, res);
  const int n = A->n_rows;
  const double rtol = prm->rtol, atol = prm->atol;
  const int max_iter = prm->max_iter;

  int32_t* d_off = nullptr;
  double *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr, *d_tr = nullptr;
  BatchSys* sys = nullptr;
  unsigned* n_done = nullptr;
  unsigned* h_done = nullptr;
  mtlgpu_status st = MTLGPU_OK;
  auto cleanup = [&]() {
    dfree(ctx, d_off);
    dfree(ctx, r);
    dfree(ctx, z);
    dfree(ctx, p);
    dfree(ctx, q);
    dfree(ctx, d_tr);
    dfree(ctx, sys);
    dfree(ctx, n_done);
    if (h_done) cudaFreeHost(h_done);
  };
#define MTLGPU_BTRY(call)            \
  do {                               \
    st = (call);                     \
    if (st != MTLGPU_OK) {           \
      cleanup();                     \
      return st;                     \
    }                                \
  } while (0)
#define MTLGPU_BTRY_CUDA(call) MTLGPU_BTRY(((call) == cudaSuccess) ? MTLGPU_OK : set_cuda_error(ctx, cudaGetLastError(), #call))

  MTLGPU_BTRY(dalloc(ctx, &d_off, count + 1));
  MTLGPU_BTRY(dalloc(ctx, &r, n));
  MTLGPU_BTRY(dalloc(ctx, &z, n));
  MTLGPU_BTRY(dalloc(ctx, &p, n));
  MTLGPU_BTRY(dalloc(ctx, &q, n));
  MTLGPU_BTRY(dalloc(ctx, &d_tr, count));
  MTLGPU_BTRY(dalloc(ctx, &sys, count));
  MTLGPU_BTRY(dalloc(ctx, &n_done, 1));
  MTLGPU_BTRY_CUDA(cudaMallocHost(&h_done, sizeof(unsigned)));
  MTLGPU_BTRY_CUDA(cudaMemcpyAsync(d_off, h_off, sizeof(int32_t) * (count + 1),
                                   cudaMemcpyHostToDevice, ctx->stream));
  MTLGPU_BTRY_CUDA(cudaMemsetAsync(n_done, 0, sizeof(unsigned), ctx->stream));
  MTLGPU_BTRY_CUDA(cudaMemsetAsync(p, 0, sizeof(double) * n, ctx->stream));
  batch_check_kernel<<<count, kBlock, 0, ctx->stream>>>(d_off, A->d_rp, A->d_ci, ctx->d_error);
  ctx->launches++;
  MTLGPU_BTRY(take_device_error(ctx));

  SpmvArgs plain;
  MTLGPU_BTRY(spmv_launch<double>(A, d_x, q, plain));
  batch_init_kernel<<<count, kBlock, 0, ctx->stream>>>(d_off, d_b, q, r, sys, rtol, atol, max_iter,
                                                       n_done);
  ctx->launches++;
  // Each loop step is one CG iteration of every running system.
  for (int k = 0; k < max_iter; ++k) {
    if ((k & 7) == 0) {
      MTLGPU_BTRY_CUDA(cudaMemcpyAsync(h_done, n_done, sizeof(unsigned), cudaMemcpyDeviceToHost,
                                       ctx->stream));
      MTLGPU_BTRY_CUDA(cudaStreamSynchronize(ctx->stream));
      if ((int)*h_done >= count) break;
      if (prm->h_interrupt && *prm->h_interrupt) {
        st = MTLGPU_INTERRUPTED;
        break;
      }
    }
    if (P && P->kind != MTLGPU_PC_IDENTITY) {
      MTLGPU_BTRY(pc_apply_t<double>(P, r, z, false, nullptr, false, false));
    } else {
      MTLGPU_BTRY_CUDA(cudaMemcpyAsync(z, r, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                       ctx->stream));
    }
    batch_rho_p_kernel<double><<<count, kBlock, 0, ctx->stream>>>(d_off, r, z, p, sys);
    MTLGPU_BTRY(spmv_launch<double>(A, p, q, plain));
    batch_update_kernel<double><<<count, kBlock, 0, ctx->stream>>>(d_off, p, q, d_x, r, sys, rtol,
                                                                   atol, max_iter, n_done);
    ctx->launches += 2;
    MTLGPU_BTRY_CUDA(cudaGetLastError());
  }
  // true residuals and the per-system results
  MTLGPU_BTRY(spmv_launch<double>(A, d_x, q, plain));
  batch_true_resid_kernel<<<count, kBlock, 0, ctx->stream>>>(d_off, d_b, q, d_tr);
  ctx->launches++;
  std::vector<BatchSys> hs(count);
  std::vector<double> htr(count);
  MTLGPU_BTRY_CUDA(cudaMemcpyAsync(hs.data(), sys, sizeof(BatchSys) * count,
                                   cudaMemcpyDeviceToHost, ctx->stream));
  MTLGPU_BTRY_CUDA(cudaMemcpyAsync(htr.data(), d_tr, sizeof(double) * count,
                                   cudaMemcpyDeviceToHost, ctx->stream));
  MTLGPU_BTRY_CUDA(cudaStreamSynchronize(ctx->stream));
  MTLGPU_BTRY(take_device_error(ctx));
  bool any_max = false;
  for (int s = 0; s < count; ++s) {
    mtlgpu_iter_result& R = res[s];
    std::memset(&R, 0, sizeof(R));
    R.iterations = hs[s].it;
    R.error = hs[s].done ? hs[s].error : 1;
    R.status = R.error ? MTLGPU_MAX_ITER : (st == MTLGPU_INTERRUPTED ? MTLGPU_INTERRUPTED : MTLGPU_OK);
    R.resid = hs[s].resid;
    R.norm_r0 = hs[s].norm_b;
    R.true_resid = htr[s];
    any_max |= R.error != 0;
  }
  cleanup();
#undef MTLGPU_BTRY
#undef MTLGPU_BTRY_CUDA
  if (st == MTLGPU_INTERRUPTED) return st;
  return any_max ? MTLGPU_MAX_ITER : MTLGPU_OK;
}

// Times the persistent kernel's candidates -- CTAs per system (the cluster
// size), lanes per row, and the row count below which a system is solved by
// one CTA -- on the caller's systems: a short solve each (at most 8
// iterations, one refinement step), from a copy of x.  Keeps the fastest on A.
mtlgpu_status batched_autotune_impl(Csr* A, Pc* P, int count, const int32_t* h_off,
                                           const double* d_x, const double* d_b,
                                           const mtlgpu_iter_params* prm, int* choice) {
  Ctx* ctx = A->ctx;
  if (count <= 0 || !h_off || !d_x || !d_b || !prm) return MTLGPU_INVALID_ARG;
  if (h_off[0] != 0 || h_off[count] != A->n_rows) return MTLGPU_INCOMPATIBLE_SIZE;
  if (!batched_cluster_supported(P)) return MTLGPU_NOT_SUPPORTED;
  double* x = nullptr;
  MTLGPU_TRY(dalloc(ctx, &x, A->n_rows));
  std::vector<mtlgpu_iter_result> res(count);
  mtlgpu_iter_params p = *prm;
  p.max_iter = std::min(p.max_iter, 8);
  p.max_outer = 1;
  p.h_interrupt = nullptr;
  float best_ms = 1e30f;
  int best_cs = A->batch_cs, best_g = A->batch_g, best_small = A->batch_small;
  for (int cs : {4, 8})
    for (int g : {1, 4, 8, 16})
      for (int small : {0, 8192, 32768}) {
        cudaMemcpyAsync(x, d_x, sizeof(double) * A->n_rows, cudaMemcpyDeviceToDevice,
                        ctx->stream);
        float ms = 0;
        mtlgpu_status st = solve_batched_cluster(A, P, count, h_off, x, d_b, &p, res.data(), cs,
                                                 g, small, &ms);
        if (st != MTLGPU_OK && st != MTLGPU_MAX_ITER) {
          dfree(ctx, x);
          return st;
        }
        if (ms < best_ms) best_ms = ms, best_cs = cs, best_g = g, best_small = small;
      }
  A->batch_cs = best_cs;
  A->batch_g = best_g;
  A->batch_small = best_small;
  dfree(ctx, x);
  if (choice) *choice = best_small * 1000 + best_cs * 100 + best_g;
  return take_device_error(ctx);
}

}  // namespace mtlgpu

extern "C" mtlgpu_status mtlgpu_batched_autotune(mtlgpu_csr* A, mtlgpu_pc* P, int count,
                                                 const int32_t* h_offsets, const double* d_x,
                                                 const double* d_b,
                                                 const mtlgpu_iter_params* params, int* h_choice) {
  if (!A || (P && P->A != A)) return MTLGPU_INVALID_ARG;
  return mtlgpu::batched_autotune_impl(A, P, count, h_offsets, d_x, d_b, params, h_choice);
}

extern "C" mtlgpu_status mtlgpu_solve_batched(int method, mtlgpu_csr* A, mtlgpu_pc* P, int count,
                                              const int32_t* h_offsets, double* d_x,
                                              const double* d_b, const mtlgpu_iter_params* params,
                                              mtlgpu_iter_result* h_results) {
  if (!A) return MTLGPU_INVALID_ARG;
  return mtlgpu::solve_batched_impl(method, A, P, count, h_offsets, d_x, d_b, params, h_results);
}
