// Triangular solves applied as a fixed number of Jacobi iterations.
//
// The exact solves of solve(P, r) (itl/pc/ic_0.hpp:80-87, itl/pc/ilu.hpp:
// 84-91: lower_trisolve then upper_trisolve) carry a dependency chain as
// long as the factor's level count (382 levels for the 128^3 7-point IC(0)
// factor), and each level costs one cross-SM hop through L2.  This file
// applies the same factors with k Jacobi iterations per triangle instead:
//     T = N + D^-1   (N the off-diagonal part, D the stored inverted diagonal;
//                     D = I for the unit lower factor of ILU(0))
//     w_0     = D v
//     w_{m+1} = D (v - N w_m)            m = 0 .. k-1
// so w_k = sum_{i<=k} (-D N)^i D v, a fixed polynomial in T.  For IC(0) the
// upper factor is trans(L) with the same diagonal, so the applied operator
// is P_k(L)^T P_k(L): symmetric positive definite, as CG needs.  Each
// iteration is one fully parallel, HBM-bound pass.  No counterpart in the
// reference: it is an approximation of the exact solves, used where the
// caller asks for it (mtlgpu_pc_set_jacobi_sweeps); the mixed-precision
// solves check their answer with the FP64 true residual, so the
// preconditioner only changes how many iterations they take.
//
// Layout: the factors' off-diagonal entries in SELL-32 slices (sell.cu), one
// warp per slice, so every load of values and column indices is coalesced
// and the row pointers are not read; the (inverted) diagonal is a separate,
// coalesced array in row order.
#include <algorithm>

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

// Optional fused reduction of the last pass: dot_out = sum_r dot_with[r] *
// w_out[r] (CG's rho = r . z right after z = solve(P, r)), as a
// deterministic grid reduction (fixed partial per block, summed in a fixed
// order by the last block).
struct PassDot {
  const void* with = nullptr;
  double* out = nullptr;
  void* partials = nullptr;
  unsigned* counter = nullptr;
};

// One Jacobi iteration of one triangle in the scaled form.  With the
// off-diagonal part stored column-scaled, Nt = N D (sell.cu), the iteration
// w_{m+1} = D (v - N w_m), w_0 = D v, is w_m = D u_m with
//     u_0 = v,   u_{m+1} = v - Nt u_m,
// so every pass gathers one vector and only the last one (SCALE) multiplies
// by D.  For ILU(0)'s unit lower factor D = I and Nt = N.  The entries of a
// row are taken in chunks of C: all C column indices and values are loaded
// (last-use hint), then all C gathers issued, so a row costs one DRAM and
// one L2 round trip per chunk.
// With D16 the column indices are 16-bit offsets from the row (Sell::d_dcol).
template <typename T, bool SCALE, bool DOT, int C, bool D16>
__global__ void __launch_bounds__(kBlock, (C == 4 && sizeof(T) == 4) ? 8 : 6)
    jacobi_pass_kernel(int n, const int32_t* __restrict__ slice_ptr,
                       const int32_t* __restrict__ col, const int16_t* __restrict__ dcol,
                       const T* __restrict__ val,
                       const T* __restrict__ dinv, const T* __restrict__ v,
                       const T* __restrict__ in, T* __restrict__ out, const int* skip,
                       PassDot dot) {
  if (skip && ld_relaxed(skip)) return;
  typedef typename AccOf<T, 1>::type R;
  R acc_dot = R::zero();
  for (long long r = gtid(); r < n; r += gstride()) {
    const long long s = r >> 5;
    const int lane = (int)(r & 31);
    const int base = __ldg(slice_ptr + s);
    const int width = (__ldg(slice_ptr + s + 1) - base) >> 5;
    const T vr = __ldg(v + r);
    const T dr = SCALE ? __ldg(dinv + r) : T(1);
    const int32_t* cp = col + base + lane;
    const int16_t* dp = dcol + base + lane;
    const T* vp = val + base + lane;
    T acc = T(0);
    for (int k0 = 0; k0 < width; k0 += C) {
      int c[C];
      T a[C], x[C];
#pragma unroll
      for (int u = 0; u < C; u++) {
        const bool inr = k0 + u < width;
        if (D16) {
          const int d = inr ? (int)__ldlu(dp + 32 * (k0 + u)) : -32768;
          c[u] = d == -32768 ? -1 : (int)r + d;
        } else {
          c[u] = inr ? __ldlu(cp + 32 * (k0 + u)) : -1;
        }
        a[u] = inr ? __ldlu(vp + 32 * (k0 + u)) : T(0);
      }
#pragma unroll
      for (int u = 0; u < C; u++) x[u] = c[u] >= 0 ? __ldg(in + c[u]) : T(0);  // -1: padding
#pragma unroll
      for (int u = 0; u < C; u++) acc += a[u] * x[u];
    }
    T res = vr - acc;
    if (SCALE) res *= dr;
    out[r] = res;
    if (DOT) acc_dot.add_prod(0, __ldg(static_cast<const T*>(dot.with) + r), res);
  }
  if (DOT) {
    R bs = block_reduce(acc_dot);
    R* parts = reinterpret_cast<R*>(dot.partials);
    if (publish_partial(bs, parts, blockIdx.x, dot.counter, gridDim.x)) {
      R tot = reduce_partials(parts, gridDim.x);
      if (threadIdx.x == 0) *dot.out = tot.value(0);
    }
  }
}

template <typename T>
struct JVals;
template <>
struct JVals<double> {
  static const double* val(const Sell& J) { return J.d_val; }
  static const double* dinv(const Sell& J) { return J.d_dinv; }
};
template <>
struct JVals<float> {
  static const float* val(const Sell& J) { return J.d_val32; }
  static const float* dinv(const Sell& J) { return J.d_dinv32; }
};

// Chunk width C: 4 when no row has more than 4 off-diagonal entries (the
// 7-point factors), else 8.
template <typename T, bool SCALE>
void launch2(int grid, cudaStream_t st, const Sell& J, const T* val, const T* dinv, const T* v,
             const T* in, T* out, const int* skip, const PassDot& dot) {
#define MTLGPU_JP(DOT, C, D16)                                                          \
  jacobi_pass_kernel<T, SCALE, DOT, C, D16><<<grid, kBlock, 0, st>>>(                   \
      J.n, J.d_slice_ptr, J.d_col, J.d_dcol, val, dinv, v, in, out, skip, dot)
  const bool d16 = J.d_dcol != nullptr;
  if (J.max_width <= 4) {
    if (dot.out) {
      if (d16) MTLGPU_JP(true, 4, true); else MTLGPU_JP(true, 4, false);
    } else {
      if (d16) MTLGPU_JP(false, 4, true); else MTLGPU_JP(false, 4, false);
    }
  } else {
    if (dot.out) {
      if (d16) MTLGPU_JP(true, 8, true); else MTLGPU_JP(true, 8, false);
    } else {
      if (d16) MTLGPU_JP(false, 8, true); else MTLGPU_JP(false, 8, false);
    }
  }
#undef MTLGPU_JP
}

template <typename T>
mtlgpu_status pass_launch(Ctx* ctx, const Sell& J, bool scale, const T* v, const T* in, T* out,
                          const int* skip, const PassDot& dot) {
  const T* val = JVals<T>::val(J);
  const T* dinv = JVals<T>::dinv(J);
  if (!val || (scale && !dinv) || (!J.unit_diag && !J.col_scaled)) return MTLGPU_INVALID_ARG;
  const int grid = grid_rows(ctx, J.n);
  if (scale)
    launch2<T, true>(grid, ctx->stream, J, val, dinv, v, in, out, skip, dot);
  else
    launch2<T, false>(grid, ctx->stream, J, val, dinv, v, in, out, skip, dot);
  ctx->launches++;
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  return MTLGPU_OK;
}

}  // namespace

// k Jacobi iterations of one triangle: v -> out, intermediate iterates in
// `scratch` (never v or out).  The passes alternate between scratch and out
// so that the last one writes out.
// With dot_with non-null the last pass also writes dot_with . out to
// *dot_out (reduction slot `counter_index` of the context).
//
// jacobi_solve_from runs passes first..k-1 only, after pass 0 (first = 1)
// was made elsewhere (the fused CG kernel, cg_fused.cu) into the buffer that
// jacobi_solve would have used: out when k is odd, else scratch.
template <typename T>
mtlgpu_status jacobi_solve_from(Ctx* ctx, const Sell& J, int k, int first, const T* v, T* out,
                                T* scratch, const int* skip, const T* dot_with, double* dot_out) {
  if (J.n == 0) return MTLGPU_OK;
  const T* prev = first == 0 ? v : (((k - first) % 2 == 0) ? out : scratch);  // u_0 = v
  for (int i = first; i < k; i++) {
    T* dst = ((k - 1 - i) % 2 == 0) ? out : scratch;
    PassDot dot;
    if (i == k - 1 && dot_with) {
      dot.with = dot_with;
      dot.out = dot_out;
      dot.partials = ctx->d_partials;
      dot.counter = counter_slot(ctx, 9);
    }
    MTLGPU_TRY(pass_launch<T>(ctx, J, i == k - 1 && !J.unit_diag, v, prev, dst, skip, dot));
    prev = dst;
  }
  return MTLGPU_OK;
}

template <typename T>
mtlgpu_status jacobi_solve(Ctx* ctx, const Sell& J, int k, const T* v, T* out, T* scratch,
                           const int* skip, const T* dot_with, double* dot_out) {
  return jacobi_solve_from<T>(ctx, J, k, 0, v, out, scratch, skip, dot_with, dot_out);
}

template mtlgpu_status jacobi_solve_from<double>(Ctx*, const Sell&, int, int, const double*,
                                                 double*, double*, const int*, const double*,
                                                 double*);
template mtlgpu_status jacobi_solve_from<float>(Ctx*, const Sell&, int, int, const float*, float*,
                                                float*, const int*, const float*, double*);
template mtlgpu_status jacobi_solve<double>(Ctx*, const Sell&, int, const double*, double*,
                                            double*, const int*, const double*, double*);
template mtlgpu_status jacobi_solve<float>(Ctx*, const Sell&, int, const float*, float*,
                                           float*, const int*, const float*, double*);

}  // namespace mtlgpu
