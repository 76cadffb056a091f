// Device-resident CG and BiCGSTAB, captured into CUDA graphs.
//
// itl::cg (itl/krylov/cg.hpp:39-72 identity, 75-112 preconditioned) and
// itl::bicgstab (itl/krylov/bicgstab.hpp:27-78), with basic_iteration control
// (itl/iteration/basic_iteration.hpp:51-93).  All scalars (rho, alpha, ...)
// live in a device SolverState; every kernel of an iteration reads what it
// needs from there, reductions are deterministic grid reductions whose last
// block also applies the reference's termination test, and every kernel
// returns at once when the state says the solve has finished.  The host
// launches a graph of kGraphIters iterations at a time and only looks at the
// state between graph launches (that is also where the interrupt flag is
// polled, as itl::interruptible_iteration does between iterations).  Without
// an interrupt flag the iterations run in a device-side loop instead: one
// launch of a graph whose conditional WHILE node repeats the kGraphIters
// iterations until the state says done (or an error is raised, or a trip
// bound derived from max_iter is reached), with no host round trip between.
//
// Per CG iteration (preconditioned):
//   sweeps   y0 = L^-1 r, z = U^-1 y0          (sweep.cu)
//   K_rho    rho = r . z
//   K_p      p = z (first) | z + (rho/rho_1) p
//   K_spmv   q = A p, alpha_1 = p . q           (spmv.cu, fused epilogue)
//   K_upd    alpha = rho/alpha_1, x += alpha p, r -= alpha q, rr = r . r,
//            termination test on sqrt(|rr|); refills the sweep outputs with
//            the sentinel for the next iteration.
// The reference fuses q = A p with alpha_1 and r -= alpha q with rr in the
// same way (fused_expr.hpp:57-77, cg.hpp:104,109).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>

#include "device.cuh"
#include "internal.h"
#include "solver_state.cuh"

namespace mtlgpu {

using namespace dev;

// Iterations per graph (per body of the device-side loop): 16 measured
// 0.22 ms faster than 8 on the 128^3 mixed solve, 32 no faster than 16.
constexpr int kGraphIters = 16;
// The fused CG recording alternates two r and two p buffers by iteration
// parity; an even count per graph keeps the parity across graph launches.
static_assert(kGraphIters % 2 == 0, "graphs hold an even number of iterations");

namespace {

constexpr int kBlock = 256;

int vec_grid(Ctx* ctx, long long n) {
  long long need = (n + kBlock - 1) / kBlock;
  long long cap = (long long)ctx->num_sms * 8;
  return (int)std::max(1ll, std::min(need, cap));
}

template <typename T>
__device__ __forceinline__ typename AccOf<T, 1>::type acc1() {
  return AccOf<T, 1>::type::zero();
}

// ---- generic pieces -----------------------------------------------------
template <typename T>
__global__ void fill2_kernel(int n, T* a, T* b) {
  const T s = Box<T>::sentinel();
  for (long long i = gtid(); i < n; i += gstride()) {
    if (a) a[i] = s;
    if (b) b[i] = s;
  }
}

// first termination test after r = b - A x, rr = ||r||^2 (cg.hpp:93-95,
// bicgstab.hpp:40-43)
__global__ void init_check_kernel(SolverState* st, bool identity_pc) {
  if (threadIdx.x != 0) return;
  const double rr = st->rr;
  if (identity_pc) st->rho = rr;  // unpreconditioned cg: rho = dot(r, r)
  if (iter_finished(st, sqrt(fabs(rr)))) st->done = 1;
}

// Vectorised element loops: thread i handles the 16-byte vector i (V
// elements) of every array, grid-stride; the n mod V tail element-wise.
#define MTLGPU_VLOOP(n, V)                                                         \
  for (long long i0 = gtid() * (V); i0 + (V) <= (n); i0 += gstride() * (V))
#define MTLGPU_TAIL(n, V) for (long long i = ((n) / (V)) * (V) + gtid(); i < (n); i += gstride())

// rho = r . z
template <typename T>
__global__ void __launch_bounds__(kBlock, 4)
    cg_rho_kernel(int n, const T* __restrict__ r, const T* __restrict__ z, SolverState* st,
                  void* partials, unsigned* counter) {
  if (st->done) return;
  typedef typename AccOf<T, 1>::type R;
  constexpr int V = VN<T>::value;
  R acc = R::zero();
  MTLGPU_VLOOP(n, V) {
    T rv[V], zv[V];
    ld16(r + i0, rv);
    ld16(z + i0, zv);
#pragma unroll
    for (int u = 0; u < V; u++) acc.add_prod(0, rv[u], zv[u]);
  }
  MTLGPU_TAIL(n, V) acc.add_prod(0, r[i], z[i]);
  R bs = block_reduce(acc);
  R* parts = reinterpret_cast<R*>(partials);
  if (publish_partial(bs, parts, blockIdx.x, counter, gridDim.x)) {
    R tot = reduce_partials(parts, gridDim.x);
    if (threadIdx.x == 0) st->rho = tot.value(0);
  }
}

// p = z (first iteration) | z + (rho / rho_1) p   (cg.hpp:99-102, 57-60)
template <typename T>
__global__ void __launch_bounds__(kBlock, 4)
    cg_p_kernel(int n, const T* __restrict__ z, T* __restrict__ p, const SolverState* st) {
  if (st->done) return;
  constexpr int V = VN<T>::value;
  if (st->iter == 0) {
    MTLGPU_VLOOP(n, V) {
      T zv[V];
      ld16(z + i0, zv);
      st16(p + i0, zv);
    }
    MTLGPU_TAIL(n, V) p[i] = z[i];
    return;
  }
  const T beta = (T)(st->rho / st->rho_1);
  MTLGPU_VLOOP(n, V) {
    T zv[V], pv[V];
    ld16(z + i0, zv);
    ld16(p + i0, pv);
#pragma unroll
    for (int u = 0; u < V; u++) pv[u] = zv[u] + beta * pv[u];
    st16(p + i0, pv);
  }
  MTLGPU_TAIL(n, V) p[i] = z[i] + beta * p[i];
}

// alpha = rho / alpha_1; x += alpha p; r -= alpha q; rr = r . r; next test.
template <typename T>
__global__ void __launch_bounds__(kBlock, 4)
    cg_update_kernel(int n, T* __restrict__ x, const T* __restrict__ p, T* __restrict__ r,
                     const T* __restrict__ q, T* fill_a, T* fill_b, SolverState* st,
                     bool identity_pc, void* partials, unsigned* counter) {
  if (st->done) return;
  typedef typename AccOf<T, 1>::type R;
  constexpr int V = VN<T>::value;
  const double alpha_d = st->rho / st->alpha_1;
  const T alpha = (T)alpha_d;
  const T s = Box<T>::sentinel();
  R acc = R::zero();
  MTLGPU_VLOOP(n, V) {
    T xv[V], pv[V], rv[V], qv[V], sv[V];
    ld16(x + i0, xv);
    ld16(p + i0, pv);
    ld16(r + i0, rv);
    ld16(q + i0, qv);
#pragma unroll
    for (int u = 0; u < V; u++) {
      xv[u] += alpha * pv[u];
      rv[u] = rv[u] - alpha * qv[u];
      acc.add_prod(0, rv[u], rv[u]);
      sv[u] = s;
    }
    st16(x + i0, xv);
    st16(r + i0, rv);
    if (fill_a) st16(fill_a + i0, sv);
    if (fill_b) st16(fill_b + i0, sv);
  }
  MTLGPU_TAIL(n, V) {
    x[i] += alpha * p[i];
    const T ri = r[i] - alpha * q[i];
    r[i] = ri;
    acc.add_prod(0, ri, ri);
    if (fill_a) fill_a[i] = s;
    if (fill_b) fill_b[i] = s;
  }
  R bs = block_reduce(acc);
  R* parts = reinterpret_cast<R*>(partials);
  if (publish_partial(bs, parts, blockIdx.x, counter, gridDim.x)) {
    R tot = reduce_partials(parts, gridDim.x);
    if (threadIdx.x == 0) {
      const double rr = tot.value(0);
      st->iter++;
      st->rho_1 = st->rho;
      st->rr = rr;
      if (identity_pc) st->rho = rr;
      if (iter_finished(st, sqrt(fabs(rr)))) st->done = 1;
    }
  }
}

// ---- BiCGSTAB -------------------------------------------------------------
// rho_1 = rtilde . r, breakdown tests (bicgstab.hpp:45-52), ++iter.
template <typename T>
__global__ void __launch_bounds__(kBlock, 4)
    bicg_rho_kernel(int n, const T* __restrict__ rt, const T* __restrict__ r, SolverState* st,
                    void* partials, unsigned* counter) {
  if (st->done) return;
  typedef typename AccOf<T, 1>::type R;
  constexpr int V = VN<T>::value;
  R acc = R::zero();
  MTLGPU_VLOOP(n, V) {
    T a[V], c[V];
    ld16(rt + i0, a);
    ld16(r + i0, c);
#pragma unroll
    for (int u = 0; u < V; u++) acc.add_prod(0, a[u], c[u]);
  }
  MTLGPU_TAIL(n, V) acc.add_prod(0, rt[i], r[i]);
  R bs = block_reduce(acc);
  R* parts = reinterpret_cast<R*>(partials);
  if (publish_partial(bs, parts, blockIdx.x, counter, gridDim.x)) {
    R tot = reduce_partials(parts, gridDim.x);
    if (threadIdx.x == 0) {
      st->iter++;
      const double rho1 = tot.value(0);
      st->rho = rho1;
      if (rho1 == 0.0 || (st->iter > 1 && st->omega == 0.0)) {
        st->status = MTLGPU_BREAKDOWN;
        st->done = 1;
        st->skip2 = 1;
      }
    }
  }
}

// p = r (first) | r + beta (p - omega v), beta = (rho_1/rho_2)(alpha/omega)
template <typename T>
__global__ void __launch_bounds__(kBlock, 4)
    bicg_p_kernel(int n, const T* __restrict__ r, T* __restrict__ p, const T* __restrict__ v,
                  const SolverState* st) {
  if (st->done) return;
  constexpr int V = VN<T>::value;
  if (st->iter <= 1) {
    MTLGPU_VLOOP(n, V) {
      T a[V];
      ld16(r + i0, a);
      st16(p + i0, a);
    }
    MTLGPU_TAIL(n, V) p[i] = r[i];
    return;
  }
  // st->rho_1 holds rho_2 (previous rho), st->alpha_1 the previous alpha
  const double beta_d = (st->rho / st->rho_1) * (st->alpha_1 / st->omega);
  const T beta = (T)beta_d, omega = (T)st->omega;
  MTLGPU_VLOOP(n, V) {
    T rv[V], pv[V], vv[V];
    ld16(r + i0, rv);
    ld16(p + i0, pv);
    ld16(v + i0, vv);
#pragma unroll
    for (int u = 0; u < V; u++) pv[u] = rv[u] + beta * (pv[u] - omega * vv[u]);
    st16(p + i0, pv);
  }
  MTLGPU_TAIL(n, V) p[i] = r[i] + beta * (p[i] - omega * v[i]);
}

// alpha = rho_1 / gamma; s = r - alpha v; ||s||; half-step termination test
// (bicgstab.hpp:58-67).
template <typename T>
__global__ void __launch_bounds__(kBlock, 4)
    bicg_s_kernel(int n, const T* __restrict__ r, const T* __restrict__ v, T* __restrict__ s,
                  T* fill_a, T* fill_b, SolverState* st, void* partials, unsigned* counter) {
  if (st->done) return;
  typedef typename AccOf<T, 1>::type R;
  const double gamma = st->gamma;
  const T alpha = (T)(st->rho / gamma);
  const T sent = Box<T>::sentinel();
  constexpr int V = VN<T>::value;
  R acc = R::zero();
  MTLGPU_VLOOP(n, V) {
    T rv[V], vv[V], sv[V], fv[V];
    ld16(r + i0, rv);
    ld16(v + i0, vv);
#pragma unroll
    for (int u = 0; u < V; u++) {
      sv[u] = rv[u] - alpha * vv[u];
      acc.add_prod(0, sv[u], sv[u]);
      fv[u] = sent;
    }
    st16(s + i0, sv);
    if (fill_a) st16(fill_a + i0, fv);
    if (fill_b) st16(fill_b + i0, fv);
  }
  MTLGPU_TAIL(n, V) {
    const T si = r[i] - alpha * v[i];
    s[i] = si;
    acc.add_prod(0, si, si);
    if (fill_a) fill_a[i] = sent;
    if (fill_b) fill_b[i] = sent;
  }
  R bs = block_reduce(acc);
  R* parts = reinterpret_cast<R*>(partials);
  if (publish_partial(bs, parts, blockIdx.x, counter, gridDim.x)) {
    R tot = reduce_partials(parts, gridDim.x);
    if (threadIdx.x == 0) {
      if (gamma == 0.0) {
        st->status = MTLGPU_BREAKDOWN;
        st->done = 1;
        st->skip2 = 1;
      } else {
        st->alpha_1 = st->rho / gamma;  // alpha
        st->ss = tot.value(0);
        if (iter_finished(st, sqrt(st->ss))) {
          st->half_exit = 1;
          st->skip2 = 1;
        }
      }
    }
  }
}

// x += omega shat + alpha phat, r = s - omega t, ||r|| and the loop test
// (bicgstab.hpp:70-75, 43); on a half-step exit only x += alpha phat.
// The next iteration's start is folded in: rho_1 = rtilde . r over the new
// r (component 1 of the same reduction; component 0 is ||r||^2, summed as
// alone), the breakdown tests and ++iter of bicg_rho_kernel, and the reset
// of skip2.  The grid and the element order are bicg_rho_kernel's, so rho_1
// has the same bits as that kernel's.
template <typename T>
__global__ void __launch_bounds__(kBlock, 4)
    bicg_x_kernel(int n, T* __restrict__ x, const T* __restrict__ phat, const T* __restrict__ shat,
                  const T* __restrict__ s, const T* __restrict__ t, T* __restrict__ r,
                  const T* __restrict__ rt, T* fill_a, T* fill_b, SolverState* st, void* partials,
                  unsigned* counter) {
  if (st->done) return;
  typedef typename AccOf<T, 2>::type R;
  const T alpha = (T)st->alpha_1;
  constexpr int V = VN<T>::value;
  if (st->half_exit) {
    MTLGPU_VLOOP(n, V) {
      T xv[V], ph[V];
      ld16(x + i0, xv);
      ld16(phat + i0, ph);
#pragma unroll
      for (int u = 0; u < V; u++) xv[u] += alpha * ph[u];
      st16(x + i0, xv);
    }
    MTLGPU_TAIL(n, V) x[i] += alpha * phat[i];
    __syncthreads();
    if (publish_partial(R::zero(), reinterpret_cast<R*>(partials), blockIdx.x, counter,
                        gridDim.x)) {
      if (threadIdx.x == 0) st->done = 1;
    }
    return;
  }
  const double omega_d = st->ts / st->tt;
  const T omega = (T)omega_d;
  const T sent = Box<T>::sentinel();
  R acc = R::zero();
  MTLGPU_VLOOP(n, V) {
    T xv[V], sh[V], ph[V], sv[V], tv[V], fv[V];
    ld16(x + i0, xv);
    ld16(shat + i0, sh);
    ld16(phat + i0, ph);
    ld16(s + i0, sv);
    ld16(t + i0, tv);
#pragma unroll
    T rtv[V];
    ld16(rt + i0, rtv);
#pragma unroll
    for (int u = 0; u < V; u++) {
      xv[u] += omega * sh[u] + alpha * ph[u];
      sv[u] = sv[u] - omega * tv[u];  // r
      acc.add_prod(0, sv[u], sv[u]);
      acc.add_prod(1, rtv[u], sv[u]);
      fv[u] = sent;
    }
    st16(x + i0, xv);
    st16(r + i0, sv);
    if (fill_a) st16(fill_a + i0, fv);
    if (fill_b) st16(fill_b + i0, fv);
  }
  MTLGPU_TAIL(n, V) {
    x[i] += omega * shat[i] + alpha * phat[i];
    const T ri = s[i] - omega * t[i];
    r[i] = ri;
    acc.add_prod(0, ri, ri);
    acc.add_prod(1, rt[i], ri);
    if (fill_a) fill_a[i] = sent;
    if (fill_b) fill_b[i] = sent;
  }
  R bs = block_reduce(acc);
  R* parts = reinterpret_cast<R*>(partials);
  if (publish_partial(bs, parts, blockIdx.x, counter, gridDim.x)) {
    R tot = reduce_partials(parts, gridDim.x);
    if (threadIdx.x == 0) {
      st->omega = omega_d;
      st->rho_1 = st->rho;  // rho_2 = rho_1
      const double rr = tot.value(0);
      st->rr = rr;
      if (iter_finished(st, sqrt(rr))) st->done = 1;
      // the next iteration's start (bicg_rho_kernel, bicg_reset_skip_kernel)
      st->skip2 = st->done ? 1 : 0;
      if (!st->done) {
        st->iter++;
        const double rho1 = tot.value(1);
        st->rho = rho1;
        if (rho1 == 0.0 || (st->iter > 1 && st->omega == 0.0)) {
          st->status = MTLGPU_BREAKDOWN;
          st->done = 1;
          st->skip2 = 1;
        }
      }
    }
  }
}

// t . s and t . t after t = A shat (omega = dot(t,s) / dot(t,t)).
template <typename T>
__global__ void __launch_bounds__(kBlock, 4)
    bicg_omega_kernel(int n, const T* __restrict__ t, const T* __restrict__ s, SolverState* st,
                      void* partials, unsigned* counter) {
  if (st->done || st->skip2) return;
  typedef typename AccOf<T, 2>::type R;
  constexpr int V = VN<T>::value;
  R acc = R::zero();
  MTLGPU_VLOOP(n, V) {
    T tv[V], sv[V];
    ld16(t + i0, tv);
    ld16(s + i0, sv);
#pragma unroll
    for (int u = 0; u < V; u++) {
      acc.add_prod(0, tv[u], sv[u]);
      acc.add_prod(1, tv[u], tv[u]);
    }
  }
  MTLGPU_TAIL(n, V) {
    acc.add_prod(0, t[i], s[i]);
    acc.add_prod(1, t[i], t[i]);
  }
  R bs = block_reduce(acc);
  R* parts = reinterpret_cast<R*>(partials);
  if (publish_partial(bs, parts, blockIdx.x, counter, gridDim.x)) {
    R tot = reduce_partials(parts, gridDim.x);
    if (threadIdx.x == 0) {
      st->ts = tot.value(0);
      st->tt = tot.value(1);
    }
  }
}

// The second half of an iteration runs unless the solve is over.
__global__ void bicg_reset_skip_kernel(SolverState* st) {
  if (threadIdx.x == 0) st->skip2 = st->done ? 1 : 0;
}

// ---- mixed precision helpers ----------------------------------------------
__global__ void scale_to_f32_kernel(int n, const double* __restrict__ r, double inv_scale,
                                    float* __restrict__ r32, float* __restrict__ x32) {
  for (long long i = gtid(); i < n; i += gstride()) {
    r32[i] = (float)(r[i] * inv_scale);
    x32[i] = 0.f;
  }
}
__global__ void refine_update_kernel(int n, double* __restrict__ x, const float* __restrict__ d,
                                     double scale) {
  for (long long i = gtid(); i < n; i += gstride()) x[i] += scale * (double)d[i];
}

// Inner FP32 solve starting from x = 0: r = rhs, rr = ||r||^2.
__global__ void __launch_bounds__(kBlock)
    f32_norm_kernel(int n, const float* __restrict__ r, SolverState* st, void* partials,
                    unsigned* counter) {
  typedef CSum<1> R;
  R acc = R::zero();
  for (long long i = gtid(); i < n; i += gstride()) acc.add_prod(0, r[i], r[i]);
  R bs = block_reduce(acc);
  R* parts = reinterpret_cast<R*>(partials);
  if (publish_partial(bs, parts, blockIdx.x, counter, gridDim.x)) {
    R tot = reduce_partials(parts, gridDim.x);
    if (threadIdx.x == 0) st->rr = tot.value(0);
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Workspace: buffers, device state and the instantiated graph of one
// (matrix, preconditioner, method, precision) combination.
template <typename T>
struct Workspace {
  Csr* A = nullptr;
  Pc* P = nullptr;
  int method = MTLGPU_CG;
  int n = 0;
  T *x = nullptr, *b = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr,
    *rt = nullptr, *phat = nullptr, *s = nullptr, *shat = nullptr, *t = nullptr, *v = nullptr;
  // fused CG (cg_fused.cu): second r and p buffers, odd iterations write them
  bool fused = false;
  T *r2 = nullptr, *p2 = nullptr;
  SolverState* st = nullptr;   // device
  SolverState* h_st = nullptr; // pinned host mirror
  double* history = nullptr;
  int hist_cap = 0;
  cudaGraphExec_t exec = nullptr;
  size_t graph_nodes = 0;      // kernel nodes per graph launch
  cudaGraphExec_t exec_loop = nullptr;  // the same iterations in a device-side loop
  bool loop_failed = false;             // the loop graph could not be made: host loop
  bool state_on_host = false;           // h_st already holds the finished solve's state
  ~Workspace() {}
};

namespace {

bool is_identity(Pc* P) { return !P || P->kind == MTLGPU_PC_IDENTITY; }

template <typename T>
T* pc_tmp(Pc* P);
template <>
double* pc_tmp<double>(Pc* P) { return P ? P->d_tmp : nullptr; }
template <>
float* pc_tmp<float>(Pc* P) { return P ? P->d_tmp32 : nullptr; }

// Exact sweeps read NaN-boxed outputs that the previous kernel prefilled;
// Jacobi-iteration solves need no prefill.
bool uses_sweeps(Pc* P) {
  return P && (P->kind == MTLGPU_PC_IC0 || P->kind == MTLGPU_PC_ILU0) && P->jacobi_iters == 0;
}

template <typename T>
__global__ void copy_if_kernel(int n, const T* __restrict__ a, T* __restrict__ b, const int* skip) {
  if (*skip) return;
  for (long long i = gtid(); i < n; i += gstride()) b[i] = a[i];
}

// z = solve(P, r); a missing preconditioner is the identity.
template <typename T>
mtlgpu_status apply_pc(Workspace<T>* W, const T* r, T* z, const int* skip, bool prefilled) {
  if (W->P) return pc_apply_t<T>(W->P, r, z, false, skip, prefilled, prefilled);
  Ctx* ctx = W->A->ctx;
  copy_if_kernel<T><<<vec_grid(ctx, W->n), kBlock, 0, ctx->stream>>>(W->n, r, z, skip);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  return MTLGPU_OK;
}

// Kernels of one CG iteration (k: its index inside the graph).
template <typename T>
mtlgpu_status record_cg_iteration(Workspace<T>* W, int k) {
  Csr* A = W->A;
  Ctx* ctx = A->ctx;
  if (W->fused) {
    const bool even = k % 2 == 0;
    return cg_fused_iteration<T>(A, W->P, W->st, W->x, even ? W->r : W->r2,
                                 even ? W->r2 : W->r, even ? W->p : W->p2, even ? W->p2 : W->p,
                                 W->z, W->q);
  }
  const int n = W->n;
  const int grid = vec_grid(ctx, n);
  const bool ident = is_identity(W->P);
  const int* skip = &W->st->done;
  T* zvec = W->r;
  if (!ident) {
    zvec = W->z;
    const bool sw = uses_sweeps(W->P);
    if (W->P->jacobi_iters > 0 && (W->P->kind == MTLGPU_PC_IC0 || W->P->kind == MTLGPU_PC_ILU0)) {
      // rho = r . z fused into the last Jacobi pass
      MTLGPU_TRY(pc_apply_t<T>(W->P, W->r, W->z, false, skip, false, false, &W->st->rho));
    } else {
      MTLGPU_TRY(pc_apply_t<T>(W->P, W->r, W->z, false, skip, sw, sw));
      cg_rho_kernel<T><<<grid, kBlock, 0, ctx->stream>>>(n, W->r, W->z, W->st, ctx->d_partials,
                                                         counter_slot(ctx, 1));
    }
  }
  cg_p_kernel<T><<<grid, kBlock, 0, ctx->stream>>>(n, zvec, W->p, W->st);
  SpmvArgs a;
  a.epi = EPI_DOT_X2;
  a.x2 = W->p;
  a.out = &W->st->alpha_1;
  a.skip = skip;
  MTLGPU_TRY(spmv_launch<T>(A, W->p, W->q, a));
  T* fa = uses_sweeps(W->P) ? pc_tmp<T>(W->P) : nullptr;
  T* fb = uses_sweeps(W->P) ? W->z : nullptr;
  cg_update_kernel<T><<<grid, kBlock, 0, ctx->stream>>>(n, W->x, W->p, W->r, W->q, fa, fb, W->st,
                                                        ident, ctx->d_partials,
                                                        counter_slot(ctx, 2));
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  return MTLGPU_OK;
}

// Kernels of one BiCGSTAB iteration.
template <typename T>
mtlgpu_status record_bicgstab_iteration(Workspace<T>* W) {
  Csr* A = W->A;
  Ctx* ctx = A->ctx;
  const int n = W->n;
  const int grid = vec_grid(ctx, n);
  const bool sw = uses_sweeps(W->P);
  T* tmp = pc_tmp<T>(W->P);
  // rho_1 and the skip reset of this iteration were made by the previous
  // iteration's x update (the first iteration's by bicgstab_prologue)
  bicg_p_kernel<T><<<grid, kBlock, 0, ctx->stream>>>(n, W->r, W->p, W->v, W->st);
  // phat = solve(M, p)  (sweep outputs prefilled by the previous x-update)
  MTLGPU_TRY(apply_pc<T>(W, W->p, W->phat, &W->st->done, sw));
  SpmvArgs a;
  a.epi = EPI_DOT_X2;
  a.x2 = W->rt;
  a.out = &W->st->gamma;
  a.skip = &W->st->done;
  MTLGPU_TRY(spmv_launch<T>(A, W->phat, W->v, a));
  if (W->fused) {
    // s = r - alpha v, ||s|| and the half-step test in the first L pass of
    // shat = solve(M, s)
    MTLGPU_TRY(bicg_fused_s_apply<T>(A, W->P, W->st, W->r, W->v, W->s, W->shat));
  } else {
    bicg_s_kernel<T><<<grid, kBlock, 0, ctx->stream>>>(n, W->r, W->v, W->s, sw ? tmp : nullptr,
                                                       sw ? W->shat : nullptr, W->st,
                                                       ctx->d_partials, counter_slot(ctx, 4));
    // shat = solve(M, s)
    MTLGPU_TRY(apply_pc<T>(W, W->s, W->shat, &W->st->skip2, sw));
  }
  // t = A shat; omega
  if (W->fused) {
    MTLGPU_TRY(bicg_t_product<T>(A, W->st, W->shat, W->s, W->t));  // t and omega's dots
  } else {
    SpmvArgs a2;
    a2.epi = EPI_AXPBY;
    a2.skip = &W->st->skip2;
    MTLGPU_TRY(spmv_launch<T>(A, W->shat, W->t, a2));
    bicg_omega_kernel<T><<<grid, kBlock, 0, ctx->stream>>>(n, W->t, W->s, W->st,
                                                           ctx->d_partials, counter_slot(ctx, 5));
  }
  bicg_x_kernel<T><<<grid, kBlock, 0, ctx->stream>>>(n, W->x, W->phat, W->shat, W->s, W->t, W->r,
                                                     W->rt, sw ? tmp : nullptr,
                                                     sw ? W->phat : nullptr, W->st,
                                                     ctx->d_partials, counter_slot(ctx, 6));
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  return MTLGPU_OK;
}

template <typename T>
mtlgpu_status build_graph(Workspace<T>* W) {
  Ctx* ctx = W->A->ctx;
  if (W->exec) return MTLGPU_OK;
  cudaGraph_t g = nullptr;
  const long long launches_before = ctx->launches;  // captured launches do not run now
  MTLGPU_TRY_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  mtlgpu_status s = MTLGPU_OK;
  for (int k = 0; k < kGraphIters && s == MTLGPU_OK; k++)
    s = W->method == MTLGPU_CG ? record_cg_iteration<T>(W, k) : record_bicgstab_iteration<T>(W);
  cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
  ctx->launches = launches_before;
  if (s != MTLGPU_OK) {
    if (g) cudaGraphDestroy(g);
    return s;
  }
  MTLGPU_TRY_CUDA(ctx, e);
  size_t nodes = 0;
  MTLGPU_TRY_CUDA(ctx, cudaGraphGetNodes(g, nullptr, &nodes));
  std::vector<cudaGraphNode_t> nv(nodes);
  if (nodes) MTLGPU_TRY_CUDA(ctx, cudaGraphGetNodes(g, nv.data(), &nodes));
  W->graph_nodes = 0;
  for (auto nd : nv) {
    cudaGraphNodeType ty;
    MTLGPU_TRY_CUDA(ctx, cudaGraphNodeGetType(nd, &ty));
    W->graph_nodes += ty == cudaGraphNodeTypeKernel;
  }
  e = cudaGraphInstantiate(&W->exec, g, 0);
  cudaGraphDestroy(g);
  MTLGPU_TRY_CUDA(ctx, e);
  return MTLGPU_OK;
}

// Condition of the device-side loop: run the body again unless the solve
// is over, an error was raised or the trip bound is reached.
__global__ void loop_cond_kernel(cudaGraphConditionalHandle h, SolverState* st, const int* err) {
  const int trips = ++st->trips;
  const bool more = !st->done && !*err && trips < st->max_trips;
  cudaGraphSetConditional(h, more ? 1u : 0u);
}

// One graph: a WHILE node whose body is kGraphIters iterations and the
// condition kernel.
template <typename T>
mtlgpu_status build_loop_graph(Workspace<T>* W) {
  Ctx* ctx = W->A->ctx;
  cudaGraph_t g = nullptr;
  MTLGPU_TRY_CUDA(ctx, cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle h;
  cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, nullptr, 0, &cp);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    MTLGPU_TRY_CUDA(ctx, e);
  }
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  const long long launches_before = ctx->launches;
  e = cudaStreamBeginCaptureToGraph(ctx->stream, body, nullptr, nullptr, 0,
                                    cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    MTLGPU_TRY_CUDA(ctx, e);
  }
  mtlgpu_status s = MTLGPU_OK;
  for (int k = 0; k < kGraphIters && s == MTLGPU_OK; k++)
    s = W->method == MTLGPU_CG ? record_cg_iteration<T>(W, k) : record_bicgstab_iteration<T>(W);
  if (s == MTLGPU_OK) loop_cond_kernel<<<1, 1, 0, ctx->stream>>>(h, W->st, ctx->d_error);
  cudaGraph_t captured = nullptr;
  e = cudaStreamEndCapture(ctx->stream, &captured);
  ctx->launches = launches_before;
  if (s != MTLGPU_OK || e != cudaSuccess) {
    cudaGraphDestroy(g);
    if (s != MTLGPU_OK) return s;
    MTLGPU_TRY_CUDA(ctx, e);
  }
  e = cudaGraphInstantiate(&W->exec_loop, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) W->exec_loop = nullptr;
  MTLGPU_TRY_CUDA(ctx, e);
  return MTLGPU_OK;
}

template <typename T>
mtlgpu_status alloc_workspace(Workspace<T>* W) {
  Ctx* ctx = W->A->ctx;
  const int n = W->n;
  MTLGPU_TRY(dalloc(ctx, &W->x, n));
  MTLGPU_TRY(dalloc(ctx, &W->b, n));
  MTLGPU_TRY(dalloc(ctx, &W->r, n));
  MTLGPU_TRY(dalloc(ctx, &W->p, n));
  MTLGPU_TRY(dalloc(ctx, &W->q, n));
  if (!is_identity(W->P) || W->method == MTLGPU_BICGSTAB) MTLGPU_TRY(dalloc(ctx, &W->z, n));
  if (W->fused && W->method == MTLGPU_CG) {
    MTLGPU_TRY(dalloc(ctx, &W->r2, n));
    MTLGPU_TRY(dalloc(ctx, &W->p2, n));
  }
  if (W->method == MTLGPU_BICGSTAB) {
    MTLGPU_TRY(dalloc(ctx, &W->rt, n));
    MTLGPU_TRY(dalloc(ctx, &W->phat, n));
    MTLGPU_TRY(dalloc(ctx, &W->s, n));
    MTLGPU_TRY(dalloc(ctx, &W->shat, n));
    MTLGPU_TRY(dalloc(ctx, &W->t, n));
    MTLGPU_TRY(dalloc(ctx, &W->v, n));
    MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(W->v, 0, sizeof(T) * n, ctx->stream));
    MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(W->p, 0, sizeof(T) * n, ctx->stream));
  }
  MTLGPU_TRY(dalloc(ctx, &W->st, 1));
  MTLGPU_TRY_CUDA(ctx, cudaMallocHost(reinterpret_cast<void**>(&W->h_st), sizeof(SolverState)));
  return MTLGPU_OK;
}

template <typename T>
void release_workspace(Workspace<T>* W) {
  if (!W) return;
  Ctx* ctx = W->A->ctx;
  if (W->exec) cudaGraphExecDestroy(W->exec);
  if (W->exec_loop) cudaGraphExecDestroy(W->exec_loop);
  T** bufs[] = {&W->x, &W->b, &W->r, &W->z, &W->p, &W->q, &W->rt, &W->phat, &W->s, &W->shat,
                &W->t, &W->v, &W->r2, &W->p2};
  for (T** b : bufs) dfree(ctx, *b);
  dfree(ctx, W->st);
  dfree(ctx, W->history);
  if (W->h_st) cudaFreeHost(W->h_st);
  W->h_st = nullptr;
}

}  // namespace

// Releases every workspace of A (called when A or a preconditioner of A is destroyed).
void release_workspaces(Csr* A, Pc* only_P);

namespace {

constexpr int prec_of(double*) { return MTLGPU_FP64; }
constexpr int prec_of(float*) { return MTLGPU_FP32; }

// Workspaces are cached on the matrix handle, keyed by (preconditioner,
// method, precision); nothing is shared between handles.
template <typename T>
mtlgpu_status get_workspace(Csr* A, Pc* P, int method, Workspace<T>** out) {
  const int prec = prec_of((T*)nullptr);
  for (auto& e : A->workspaces)
    if (e.P == P && e.method == method && e.prec == prec) {
      *out = static_cast<Workspace<T>*>(e.ws);
      return MTLGPU_OK;
    }
  Workspace<T>* W = new Workspace<T>();
  W->A = A;
  W->P = P;
  W->method = method;
  W->n = A->n_rows;
  W->fused = (method == MTLGPU_CG || method == MTLGPU_BICGSTAB) && cg_fused_eligible(A, P, prec);
  mtlgpu_status s = alloc_workspace<T>(W);
  if (s != MTLGPU_OK) {
    release_workspace<T>(W);
    delete W;
    return s;
  }
  A->workspaces.push_back({P, method, prec, W});
  *out = W;
  return MTLGPU_OK;
}

template <typename T>
mtlgpu_status ensure_history(Workspace<T>* W, int cap) {
  if (cap <= W->hist_cap) return MTLGPU_OK;
  Ctx* ctx = W->A->ctx;
  dfree(ctx, W->history);
  MTLGPU_TRY(dalloc(ctx, &W->history, cap));
  W->hist_cap = cap;
  if (W->exec) {  // state pointer unchanged; the history pointer lives in the state
  }
  return MTLGPU_OK;
}

// Runs graph launches until the state reports completion.
template <typename T>
mtlgpu_status run_iterations(Workspace<T>* W, const volatile int* h_interrupt, int* interrupted) {
  Ctx* ctx = W->A->ctx;
  MTLGPU_TRY(build_graph<T>(W));
  *interrupted = 0;
  if (!h_interrupt && !W->loop_failed && !W->exec_loop &&
      build_loop_graph<T>(W) != MTLGPU_OK) {
    // keep the host loop for this workspace
    W->loop_failed = true;
    cudaGetLastError();
    ctx->last_error.clear();
  }
  if (!h_interrupt && W->exec_loop) {
    MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(W->h_st, W->st, sizeof(SolverState),
                                         cudaMemcpyDeviceToHost, ctx->stream));
    MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (W->h_st->done) return take_device_error(ctx);
    MTLGPU_TRY_CUDA(ctx, cudaGraphLaunch(W->exec_loop, ctx->stream));
    int err = 0;
    MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(W->h_st, W->st, sizeof(SolverState),
                                         cudaMemcpyDeviceToHost, ctx->stream));
    MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(&err, ctx->d_error, sizeof(int), cudaMemcpyDeviceToHost,
                                         ctx->stream));
    MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->launches += (long long)W->h_st->trips * (long long)(W->graph_nodes + 1);
    if (err) return take_device_error(ctx);
    if (W->h_st->done) {
      W->state_on_host = true;  // h_st is the final state; the error word is clear
      return MTLGPU_OK;
    }
    // the trip bound ended the loop first: the host loop below carries on
  }
  while (true) {
    MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(W->h_st, W->st, sizeof(SolverState),
                                         cudaMemcpyDeviceToHost, ctx->stream));
    MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (W->h_st->done) break;
    if (h_interrupt && *h_interrupt) {
      *interrupted = 1;
      break;
    }
    // the error word is read after the graph: a bounded wait that ran out
    // inside it ends the solve at once
    int err = 0;
    MTLGPU_TRY_CUDA(ctx, cudaGraphLaunch(W->exec, ctx->stream));
    ctx->launches += (long long)W->graph_nodes;
    MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(&err, ctx->d_error, sizeof(int), cudaMemcpyDeviceToHost,
                                         ctx->stream));
    MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (err) break;
  }
  return take_device_error(ctx);
}

template <typename T>
void init_state(SolverState* h, const mtlgpu_iter_params* prm, double norm_r0, int max_iter,
                double* history, int hist_cap) {
  std::memset(h, 0, sizeof(SolverState));
  h->max_iter = max_iter;
  // every body run of the device-side loop makes kGraphIters iterations
  // unless the solve has ended, so max_iter bounds the runs
  h->max_trips = max_iter / kGraphIters + 4;
  h->tol = prm->rtol * norm_r0;
  h->atol = prm->atol;
  h->norm_r0 = norm_r0;
  h->history = history;
  h->hist_cap = hist_cap;
}

// One complete device solve in precision T on workspace W (x, b already in
// W->x, W->b; or, with rhs_is_residual, W->r holds the rhs and x = 0).
template <typename T>
mtlgpu_status device_solve(Workspace<T>* W, const mtlgpu_iter_params* prm, double norm_r0,
                           bool norm_from_b, int max_iter, bool rhs_is_residual, int* iters,
                           int* err_code, int* status, double* resid, int* hist_len,
                           double* h_hist, int h_hist_cap) {
  Csr* A = W->A;
  Ctx* ctx = A->ctx;
  const int n = W->n;
  const int cap = std::max(2 * max_iter + 4, 16);
  MTLGPU_TRY(ensure_history<T>(W, cap));
  const bool ident = is_identity(W->P);
  const bool sw = uses_sweeps(W->P);
  // norm_r0 = two_norm(b) when asked (basic_iteration(b, ...))
  if (norm_from_b) {
    SpmvArgs dummy;
    (void)dummy;
    MTLGPU_TRY(dot_launch(ctx, n, reinterpret_cast<const double*>(W->b),
                          reinterpret_cast<const double*>(W->b), ctx->d_scalars, 1));
    double nb2 = 0;
    MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(&nb2, ctx->d_scalars, sizeof(double),
                                         cudaMemcpyDeviceToHost, ctx->stream));
    MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    norm_r0 = std::sqrt(nb2);
  }
  init_state<T>(W->h_st, prm, norm_r0, max_iter, W->history, W->hist_cap);
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(W->st, W->h_st, sizeof(SolverState), cudaMemcpyHostToDevice,
                                       ctx->stream));
  const int grid = vec_grid(ctx, n);
  if (rhs_is_residual) {
    ctx->launches++;
    f32_norm_kernel<<<grid, kBlock, 0, ctx->stream>>>(n, reinterpret_cast<const float*>(W->r),
                                                      W->st, ctx->d_partials,
                                                      counter_slot(ctx, 7));
  } else {
    SpmvArgs a;
    a.epi = EPI_RESID;
    a.b = W->b;
    a.out = &W->st->rr;
    MTLGPU_TRY(spmv_launch<T>(A, W->x, W->r, a));  // r = b - A x, rr
  }
  if (W->method == MTLGPU_BICGSTAB)
    MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(W->rt, W->r, sizeof(T) * n, cudaMemcpyDeviceToDevice,
                                         ctx->stream));
  init_check_kernel<<<1, 32, 0, ctx->stream>>>(W->st, ident && W->method == MTLGPU_CG);
  ctx->launches++;
  if (sw) {
    T* second = W->method == MTLGPU_CG ? W->z : W->phat;
    fill2_kernel<T><<<grid, kBlock, 0, ctx->stream>>>(n, pc_tmp<T>(W->P), second);
    ctx->launches++;
  }
  // the fused recording starts inside the first iteration (z, rho, p, q)
  if (W->fused && W->method == MTLGPU_CG)
    MTLGPU_TRY(cg_fused_prologue<T>(A, W->P, W->st, W->r, W->z, W->p, W->q));
  // BiCGSTAB's first rho_1 (later ones come with the x update)
  if (W->method == MTLGPU_BICGSTAB) {
    bicg_reset_skip_kernel<<<1, 32, 0, ctx->stream>>>(W->st);
    bicg_rho_kernel<T><<<grid, kBlock, 0, ctx->stream>>>(n, W->rt, W->r, W->st, ctx->d_partials,
                                                         counter_slot(ctx, 3));
    ctx->launches += 2;
  }
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  int interrupted = 0;
  W->state_on_host = false;
  MTLGPU_TRY(run_iterations<T>(W, prm->h_interrupt, &interrupted));
  SolverState* h = W->h_st;
  if (!W->state_on_host) {
    MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(h, W->st, sizeof(SolverState), cudaMemcpyDeviceToHost,
                                         ctx->stream));
    MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  *iters = h->iter;
  *err_code = h->error;
  *status = interrupted ? MTLGPU_INTERRUPTED : (h->status ? h->status : (h->error ? MTLGPU_MAX_ITER : MTLGPU_OK));
  *resid = h->resid;
  *hist_len = h->hist_len;
  if (h_hist && h_hist_cap > 0) {
    int m = std::min(std::min(h->hist_len, W->hist_cap), h_hist_cap);
    if (m > 0) {
      MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(h_hist, W->history, sizeof(double) * m,
                                           cudaMemcpyDeviceToHost, ctx->stream));
      MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
  }
  return MTLGPU_OK;
}

mtlgpu_status true_residual(Csr* A, const double* x, const double* b, double* scratch,
                            double* out) {
  Ctx* ctx = A->ctx;
  SpmvArgs a;
  a.epi = EPI_RESID;
  a.b = b;
  a.out = ctx->d_scalars + 2;
  MTLGPU_TRY(spmv_launch<double>(A, x, scratch, a));
  double rr = 0;
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(&rr, ctx->d_scalars + 2, sizeof(double),
                                       cudaMemcpyDeviceToHost, ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *out = std::sqrt(rr);
  return MTLGPU_OK;
}

}  // namespace

void release_workspaces(Csr* A, Pc* only_P) {
  release_batch_work(A, only_P);
  release_xwork(A, only_P);
  std::vector<WorkspaceEntry> keep;
  for (auto& e : A->workspaces) {
    if (only_P && e.P != only_P) {
      keep.push_back(e);
      continue;
    }
    if (e.prec == MTLGPU_FP64) {
      auto* W = static_cast<Workspace<double>*>(e.ws);
      release_workspace<double>(W);
      delete W;
    } else {
      auto* W = static_cast<Workspace<float>*>(e.ws);
      release_workspace<float>(W);
      delete W;
    }
  }
  A->workspaces = keep;
}

// Iterative refinement: FP32 inner solves, FP64 residual / update / norm.
static mtlgpu_status solve_mixed(int method, Csr* A, Pc* P, double* d_x, const double* d_b,
                                 const mtlgpu_iter_params* prm, mtlgpu_iter_result* res) {
  Ctx* ctx = A->ctx;
  const int n = A->n_rows;
  if (P && P->prec != MTLGPU_FP32 && P->kind != MTLGPU_PC_IDENTITY) return MTLGPU_INVALID_ARG;
  MTLGPU_TRY(csr_ensure_fp32(A));
  Workspace<double>* W64 = nullptr;
  Workspace<float>* W32 = nullptr;
  MTLGPU_TRY(get_workspace<double>(A, P, -1 - method, &W64));  // buffers only
  MTLGPU_TRY(get_workspace<float>(A, P, method, &W32));
  const int grid = vec_grid(ctx, n);
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(W64->x, d_x, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                       ctx->stream));
  double norm_r0 = prm->norm_r0;
  if (norm_r0 < 0) {
    MTLGPU_TRY(dot_launch(ctx, n, d_b, d_b, ctx->d_scalars, 1));
    double nb2 = 0;
    MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(&nb2, ctx->d_scalars, sizeof(double),
                                         cudaMemcpyDeviceToHost, ctx->stream));
    MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    norm_r0 = std::sqrt(nb2);
  }
  const double tol = prm->rtol * norm_r0;
  const double inner_rtol = prm->inner_rtol > 0 ? prm->inner_rtol : 1e-6;
  const int max_outer = prm->max_outer > 0 ? prm->max_outer : 30;
  const int inner_max = prm->inner_max_iter > 0 ? prm->inner_max_iter : prm->max_iter;
  int total = 0, outer = 0, hist = 0;
  res->status = MTLGPU_OK;
  res->error = 0;
  double resid = 0;
  while (true) {
    MTLGPU_TRY(true_residual(A, W64->x, d_b, W64->r, &resid));
    if (prm->h_resid_history && hist < prm->history_cap) prm->h_resid_history[hist] = resid;
    hist++;
    const bool conv = norm_r0 == 0 ? resid <= prm->atol : (resid <= tol || resid <= prm->atol);
    if (conv) break;
    if (outer >= max_outer || total >= prm->max_iter) {
      res->error = 1;
      res->status = MTLGPU_MAX_ITER;
      break;
    }
    if (prm->h_interrupt && *prm->h_interrupt) {
      res->status = MTLGPU_INTERRUPTED;
      break;
    }
    // inner: A d = r / ||r|| in FP32 from d = 0
    scale_to_f32_kernel<<<grid, kBlock, 0, ctx->stream>>>(n, W64->r, 1.0 / resid, W32->r, W32->x);
    ctx->launches++;
    MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
    // Each inner solve asks for at most inner_rtol, and never for more than
    // the reduction still needed (with a margin of 2): the last refinement
    // step then costs only the iterations it needs.
    mtlgpu_iter_params ip = *prm;
    const double target = std::max(tol, prm->atol);
    ip.rtol = std::max(inner_rtol, std::min(0.5, 0.5 * target / resid));
    ip.atol = 0;
    int it = 0, ec = 0, st = 0, hl = 0;
    double rr = 0;
    MTLGPU_TRY(device_solve<float>(W32, &ip, 1.0, false, std::min(inner_max, prm->max_iter - total),
                                   true, &it, &ec, &st, &rr, &hl, nullptr, 0));
    total += it;
    outer++;
    if (st == MTLGPU_BREAKDOWN || st == MTLGPU_TIMEOUT || st == MTLGPU_INTERRUPTED) {
      res->status = st;
      if (st != MTLGPU_BREAKDOWN) break;
    }
    refine_update_kernel<<<grid, kBlock, 0, ctx->stream>>>(n, W64->x, W32->x, resid);
    ctx->launches++;
    MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
    if (st == MTLGPU_BREAKDOWN) break;
  }
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(d_x, W64->x, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                       ctx->stream));
  res->iterations = total;
  res->outer_iterations = outer;
  res->resid = resid;
  res->norm_r0 = norm_r0;
  res->true_resid = resid;
  res->history_len = hist;
  MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return (mtlgpu_status)res->status;
}

mtlgpu_status solve_impl(int method, Csr* A, Pc* P, double* d_x, const double* d_b,
                         const mtlgpu_iter_params* prm, mtlgpu_iter_result* res) {
  Ctx* ctx = A->ctx;
  std::memset(res, 0, sizeof(*res));
  if (A->n_rows != A->n_cols) return MTLGPU_NOT_SQUARE;
  if (P && P->A != A) return MTLGPU_INVALID_ARG;
  if (method != MTLGPU_CG && method != MTLGPU_BICGSTAB) return MTLGPU_INVALID_ARG;
  if (prm->mode == MTLGPU_SOLVE_MIXED_REFINED) return solve_mixed(method, A, P, d_x, d_b, prm, res);
  const int n = A->n_rows;
  Workspace<double>* W = nullptr;
  MTLGPU_TRY(get_workspace<double>(A, P, method, &W));
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(W->x, d_x, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                       ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(W->b, d_b, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                       ctx->stream));
  int it = 0, ec = 0, st = 0, hl = 0;
  double resid = 0;
  MTLGPU_TRY(device_solve<double>(W, prm, prm->norm_r0, prm->norm_r0 < 0, prm->max_iter, false, &it,
                                  &ec, &st, &resid, &hl, prm->h_resid_history, prm->history_cap));
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(d_x, W->x, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                       ctx->stream));
  res->iterations = it;
  res->error = ec;
  res->status = st;
  res->resid = resid;
  res->norm_r0 = W->h_st->norm_r0;
  res->history_len = hl;
  double tr = 0;
  MTLGPU_TRY(true_residual(A, W->x, W->b, W->q, &tr));
  res->true_resid = tr;
  return (mtlgpu_status)st;
}

}  // namespace mtlgpu
