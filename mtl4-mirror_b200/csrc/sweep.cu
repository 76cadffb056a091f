// Sync-free triangular sweeps for sm_100a.
//
// Replaces the sequential row loops lower_trisolve_t::apply(int_<5>) (unit
// diagonal, mtl/operation/lower_trisolve.hpp:173-189), apply(int_<6>)
// (inverted diagonal stored last, 192-209) and upper_trisolve_t::apply(
// int_<3>) (inverted diagonal stored first, mtl/operation/upper_trisolve.hpp:
// 160-176, row_update 101-103):
//     w[r] = (v[r] - sum_j F[r][j] * w[j]) * dia[r]      (dia = 1 for v5)
//
// One launch per sweep.  The factor is stored in level order (SweepPlan);
// warps claim tasks (<= 32/G rows of one level) through an atomic ticket in
// level order, G lanes per row load the row's off-diagonal entries and wait
// for each dependency w[j] to become final; the row's products are folded in
// the reference's order (see sweep_kernel).  w is NaN-boxed (see device.cuh):
// the output buffer is prefilled with the sentinel and a row's result is
// published by a single relaxed store, so a dependency costs one L2 round
// trip and no fence.  Every wait is bounded; on exhaustion the kernel records
// MTLGPU_TIMEOUT in the context's error word and all waiters drain quickly.
// Because tasks are claimed in level order, a row only ever waits on rows
// claimed earlier by running warps, so the sweep needs no co-residency
// assumption.  The last warp to finish resets the ticket for the next launch.
#include <algorithm>

#include "device.cuh"
#include "internal.h"

namespace mtlgpu {

using namespace dev;

namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }

// G lanes per row.  Lane gl of a row's group waits for w[c] of entries
// gl, gl + G, ... and forms the separately rounded product a * w[c]; the
// group's G products of one pass go to shared memory, and lane 0 folds them
// into rr = v[r] in stored column order with separately rounded
// subtractions, then w[r] = rr * dia: the reference's `rr -= value *
// w[col]` loop, bit for bit.  (Folding through shared memory measured
// 3x faster on B200 than a chain of width-G shuffles for FP64, and as fast as
// the unordered shuffle tree it replaces.)
template <typename T, int G>
__global__ void __launch_bounds__(kBlock)
    sweep_kernel(int n_tasks, const int32_t* __restrict__ task_ptr, const int32_t* __restrict__ rp,
                 const int32_t* __restrict__ ci, const T* __restrict__ val,
                 const T* __restrict__ dinv, const int32_t* __restrict__ row_of,
                 const T* __restrict__ in, T* out, unsigned* ticket, int* err, long long limit,
                 const int* skip, unsigned total_warps) {
  if (skip && ld_relaxed(skip)) return;
  __shared__ T stage[kBlock];
  const int lane = threadIdx.x & 31;
  const int sub = lane / G, gl = lane % G;
  T* st = stage + (threadIdx.x & ~31) + sub * G;
  while (true) {
    unsigned t = 0;
    if (lane == 0) t = atomicAdd(ticket, 1u);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= (unsigned)n_tasks) break;
    const int p = task_ptr[t] + sub;
    const bool valid = p < task_ptr[t + 1];
    T rr = T(0), d = T(1);
    int row = 0, b = 0, len = 0;
    if (valid) {
      row = row_of[p];
      rr = in[row];
      if (dinv) d = dinv[p];
      b = rp[p];
      len = rp[p + 1] - b;
    }
    if (G == 1) {
      for (int j = 0; j < len; j++)
        rr = sub_rn(rr, mul_rn(val[b + j], wait_value(out + ci[b + j], limit, err)));
    } else {
      // the same number of passes in every lane (the warp syncs per pass)
      int passes = (len + G - 1) / G;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1)
        passes = max(passes, __shfl_xor_sync(0xffffffffu, passes, off));
      for (int ps = 0; ps < passes; ps++) {
        const int k = ps * G + gl;
        T prod = T(0);
        if (k < len) prod = mul_rn(val[b + k], wait_value(out + ci[b + k], limit, err));
        st[gl] = prod;
        __syncwarp();
        if (gl == 0) {
          const int cnt = min(len - ps * G, G);
          for (int q = 0; q < cnt; q++) rr = sub_rn(rr, st[q]);
        }
        __syncwarp();
      }
    }
    if (valid && gl == 0) {
      T res = rr;
      if (dinv) res = mul_rn(res, d);
      st_relaxed(out + row, canonical(res));
    }
  }
  if (lane == 0) {
    __threadfence();
    unsigned prev = atomicAdd(ticket + 1, 1u);
    if (prev == total_warps - 1) {
      ticket[0] = 0;
      ticket[1] = 0;
      __threadfence();
    }
  }
}

template <typename T>
struct PlanVals;
template <>
struct PlanVals<double> {
  static const double* val(const SweepPlan& P) { return P.d_val; }
  static const double* dinv(const SweepPlan& P) { return P.d_dinv; }
};
template <>
struct PlanVals<float> {
  static const float* val(const SweepPlan& P) { return P.d_val32; }
  static const float* dinv(const SweepPlan& P) { return P.d_dinv32; }
};

}  // namespace

template <typename T>
mtlgpu_status sweep_launch(Ctx* ctx, const SweepPlan& P, const T* in, T* out, bool prefilled,
                           const int* skip) {
  if (P.n == 0) return MTLGPU_OK;
  const T* val = PlanVals<T>::val(P);
  const T* dinv = PlanVals<T>::dinv(P);
  if ((P.nnz_off > 0 && !val) || (!P.unit_diag && !dinv)) return MTLGPU_INVALID_ARG;
  if (!prefilled) {
    MTLGPU_TRY(fill_sentinel<T>(ctx, out, P.n));
    ctx->launches++;
  }
  if (part_sweep_ready<T>(P, out)) return part_sweep_launch<T>(ctx, P, in, out, skip);
  ctx->launches++;
  const int R = 32 / P.group;
  long long warps_needed = (P.n_tasks + 0ll);
  // Fewer resident warps mean fewer concurrent pollers: with 2 CTAs per SM a
  // sweep of the 128^3 Laplacian ran 0.53 ms (FP64) against 0.70 ms with 8.
  long long max_warps = (long long)ctx->num_sms * (2048 / 32);
  if (ctx->sweep_blocks_per_sm > 0)
    max_warps = std::min(max_warps,
                         (long long)ctx->num_sms * ctx->sweep_blocks_per_sm * (kBlock / 32));
  long long warps = std::max(1ll, std::min(warps_needed, max_warps));
  int grid = (int)((warps * 32 + kBlock - 1) / kBlock);
  unsigned total_warps = (unsigned)(grid * (kBlock / 32));
  (void)R;
#define MTLGPU_SWEEP_CASE(GG)                                                                   \
  case GG:                                                                                      \
    sweep_kernel<T, GG><<<grid, kBlock, 0, ctx->stream>>>(                                      \
        P.n_tasks, P.d_task_ptr, P.d_rp, P.d_ci, val, dinv, P.d_row_of, in, out, P.d_ticket,    \
        ctx->d_error, ctx->spin_limit, skip, total_warps);                                      \
    break;
  switch (P.group) {
    MTLGPU_SWEEP_CASE(1)
    MTLGPU_SWEEP_CASE(2)
    MTLGPU_SWEEP_CASE(4)
    MTLGPU_SWEEP_CASE(8)
    MTLGPU_SWEEP_CASE(16)
    MTLGPU_SWEEP_CASE(32)
    default:
      return MTLGPU_INVALID_ARG;
  }
#undef MTLGPU_SWEEP_CASE
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  return MTLGPU_OK;
}

template mtlgpu_status sweep_launch<double>(Ctx*, const SweepPlan&, const double*, double*, bool,
                                            const int*);
template mtlgpu_status sweep_launch<float>(Ctx*, const SweepPlan&, const float*, float*, bool,
                                           const int*);

}  // namespace mtlgpu
