// Batched PCG in one persistent launch: thread-block clusters pull systems
// from a work queue.
//
// Each system s of the block-diagonal matrix follows itl::cg(A_s, x_s, b_s,
// P_s, iter_s) (itl/krylov/cg.hpp:75-112) with iter_s = basic_iteration(b_s,
// max_iter, rtol, atol) (itl/iteration/basic_iteration.hpp:31-39).
//
// Design.  The kernel is launched once, with as many clusters of CS CTAs as
// fit the GPU at once.  A cluster takes the next system from a queue (systems
// ordered by decreasing work, so the longest ones start first) and runs that
// system's whole solve: its rows are split evenly over the CS CTAs of the
// cluster, every phase that needs values of other rows is separated by a
// cluster barrier (barrier.cluster, release/acquire at cluster scope), and
// every reduction goes through distributed shared memory: each CTA reduces
// its rows in a fixed order, publishes the partial in its shared memory, and
// after the barrier every CTA sums the CS partials in rank order -- the same
// bits in every CTA and on every run.  When the system has stopped, the
// cluster takes the next one; a converged system therefore costs nothing
// more, and there is no host round trip until the last system is done.
//
// Per CG iteration: z = M^-1 r with rho = r.z; p = z + beta p; [barrier]
// q = A p with p.q (G lanes per row, gathers of p through L2); x += alpha p,
// r -= alpha q with r.r and the stopping test.  Preconditioners: identity,
// diagonal (itl/pc/diagonal.hpp:28-103), and IC(0) / ILU(0) factors applied
// by Jacobi iterations (jacobi_sweep.cu's scaled form, one barrier per pass).
// Exact level-scheduled triangular solves stay in batched.cu.
//
// MIXED_REFINED runs, per system and still inside the same launch, FP64
// iterative refinement around an FP32 inner PCG: r = b - A x in FP64, the
// stopping test on ||r||, the inner solve of A d = r / ||r|| in FP32 (values,
// factors, vectors; FP64 accumulation of the dots), x += ||r|| d.
//
// Tunables (CS, G) are picked per matrix by mtlgpu_batched_autotune, which
// times the candidates on the caller's systems.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include "device.cuh"
#include "internal.h"

namespace cgx = cooperative_groups;

namespace mtlgpu {

using namespace dev;

namespace {

constexpr int kThreads = 256;

struct BatchState {
  double resid, norm_b;
  int it, error, outer, done;
};

template <typename T>
struct BatchVecs {
  T *r, *z, *p, *q, *d, *u, *w;  // d: inner solution (refinement); u, w: Jacobi passes
};

struct BatchArgs {
  int count;
  int n_large;           // order[0 .. n_large): systems solved by a whole cluster
  const int32_t* order;  // systems by decreasing work
  const int32_t* off;    // row offsets, count + 1
  const int32_t* rp;
  const int32_t* ci;
  const double* val64;
  const float* val32;
  const double* dinv64;  // diagonal preconditioner
  const float* dinv32;
  Sell L, U;             // factors for Jacobi-iteration solves
  int jac_k;
  int pc;                // 0 identity, 1 diagonal, 2 factors
  const double* b;
  double* x;
  double* r64;           // FP64 residual (refinement)
  BatchState* state;
  unsigned* queue;
  double rtol, atol, inner_rtol;
  int max_iter, inner_max, max_outer;
  int g;                 // lanes per row in the SpMV
};

template <typename T>
__device__ __forceinline__ const T* vals(const BatchArgs& a);
template <>
__device__ __forceinline__ const double* vals<double>(const BatchArgs& a) { return a.val64; }
template <>
__device__ __forceinline__ const float* vals<float>(const BatchArgs& a) { return a.val32; }
template <typename T>
__device__ __forceinline__ const T* dinv(const BatchArgs& a);
template <>
__device__ __forceinline__ const double* dinv<double>(const BatchArgs& a) { return a.dinv64; }
template <>
__device__ __forceinline__ const float* dinv<float>(const BatchArgs& a) { return a.dinv32; }
template <typename T>
__device__ __forceinline__ const T* sell_val(const Sell& S);
template <>
__device__ __forceinline__ const double* sell_val<double>(const Sell& S) { return S.d_val; }
template <>
__device__ __forceinline__ const float* sell_val<float>(const Sell& S) { return S.d_val32; }
template <typename T>
__device__ __forceinline__ const T* sell_dinv(const Sell& S);
template <>
__device__ __forceinline__ const double* sell_dinv<double>(const Sell& S) { return S.d_dinv; }
template <>
__device__ __forceinline__ const float* sell_dinv<float>(const Sell& S) { return S.d_dinv32; }

// Cluster-wide deterministic sum of K values: block reduction in a fixed
// order, partials published in this CTA's shared memory (two alternating
// buffers, so a buffer is rewritten only after a later barrier), one cluster
// barrier, then warp 0 adds the CS partials in rank order and broadcasts.
// The buffer index is per thread (every thread of every CTA of the cluster
// toggles its own copy on every call, so all agree); it must not live in
// shared memory, where concurrent toggles by many threads would race.
template <int K>
struct ClusterSum {
  double part[2][K];
  double bcast[K];
};

template <int K>
__device__ __forceinline__ void cluster_sum(cgx::cluster_group& cl, ClusterSum<K>& cs, int& buf,
                                            double (&v)[K]) {
  Sum<K> a = Sum<K>::zero();
#pragma unroll
  for (int k = 0; k < K; k++) a.v[k] = v[k];
  Sum<K> t = block_reduce(a);
  double* pb = cs.part[buf];
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < K; k++) pb[k] = t.v[k];
  cl.sync();
  if (threadIdx.x < K) {
    double s = 0;
    const int n = (int)cl.num_blocks();
    for (int r = 0; r < n; r++) s += cl.map_shared_rank(pb, r)[threadIdx.x];
    cs.bcast[threadIdx.x] = s;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; k++) v[k] = cs.bcast[k];
  buf ^= 1;
}

// The team that solves one system: the whole cluster (rows split over its
// CTAs, cluster barriers, distributed-shared-memory reductions) or a single
// CTA (block barriers, block reductions).  Both keep their per-thread state
// in registers.
struct ClusterTeam {
  cgx::cluster_group cl;
  ClusterSum<3>* cs;
  int buf;
  __device__ __forceinline__ void sync() { cl.sync(); }
  __device__ __forceinline__ void sum(double (&v)[3]) { cluster_sum<3>(cl, *cs, buf, v); }
};
struct CtaTeam {
  ClusterSum<3>* cs;
  __device__ __forceinline__ void sync() { __syncthreads(); }
  __device__ __forceinline__ void sum(double (&v)[3]) {
    Sum<3> a = Sum<3>::zero();
#pragma unroll
    for (int k = 0; k < 3; k++) a.v[k] = v[k];
    Sum<3> t = block_reduce(a);
    if (threadIdx.x == 0)
#pragma unroll
      for (int k = 0; k < 3; k++) cs->bcast[k] = t.v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 3; k++) v[k] = cs->bcast[k];
  }
};

// y = A p over rows [lo, hi) with G lanes per row (lanes read a row's
// entries with stride G, tree-sum), out[0] += p_row * y_row.  p is read
// through L2 (ld.global.cg): other CTAs of the cluster wrote it.  A row's
// result is written by lane 0 of its group: a __syncthreads must separate
// this from element loops that read y one row per thread.
// A lane takes its entries of a row in chunks of 4 (indices and values
// loaded together, then 4 gathers), so a row costs one DRAM and one L2 round
// trip per chunk rather than per entry.  Plain loads: a system's matrix is
// read again every iteration, and the systems in flight stay in L2.
template <typename T, int G>
__device__ __forceinline__ void spmv_rows(const int32_t* __restrict__ rp,
                                          const int32_t* __restrict__ ci,
                                          const T* __restrict__ val, const T* p, T* y, int lo,
                                          int hi, double& pq, bool dot) {
  constexpr int KK = 4;
  constexpr int R = 2;  // rows per lane group per pass, loaded together
  const int sub = threadIdx.x / G, gl = threadIdx.x % G;
  constexpr int rows_per_pass = kThreads / G;
  for (int base = lo; base < hi; base += R * rows_per_pass) {
    int rb[R], re[R];
#pragma unroll
    for (int q = 0; q < R; q++) {
      const int row = base + sub + q * rows_per_pass;
      rb[q] = row < hi ? rp[row] : 0;
      re[q] = row < hi ? rp[row + 1] : 0;
    }
    T s[R];
#pragma unroll
    for (int q = 0; q < R; q++) s[q] = T(0);
    int len = 0;
#pragma unroll
    for (int q = 0; q < R; q++) len = max(len, re[q] - rb[q]);
    for (int k0 = gl; k0 < len; k0 += G * KK) {
      int c[R][KK];
      T v[R][KK];
#pragma unroll
      for (int q = 0; q < R; q++)
#pragma unroll
        for (int u = 0; u < KK; u++) {
          const int j = rb[q] + k0 + G * u;
          c[q][u] = j < re[q] ? ci[j] : -1;
          v[q][u] = j < re[q] ? val[j] : T(0);
        }
#pragma unroll
      for (int q = 0; q < R; q++)
#pragma unroll
        for (int u = 0; u < KK; u++)
          if (c[q][u] >= 0) s[q] += v[q][u] * __ldcg(p + c[q][u]);
    }
#pragma unroll
    for (int q = 0; q < R; q++) {
#pragma unroll
      for (int off = G / 2; off > 0; off >>= 1)
        s[q] += __shfl_xor_sync(0xffffffffu, s[q], off, G);
      const int row = base + sub + q * rows_per_pass;
      if (row < hi && gl == 0) {
        y[row] = s[q];
        if (dot) pq += (double)__ldcg(p + row) * (double)s[q];
      }
    }
  }
}

// y = A p over rows [lo, hi) in CSR-stream order (G == 1 in the kernel's
// template): a warp takes 32 consecutive rows and streams their entries in
// chunks of 32 * KS -- KS coalesced loads of column indices and of values per
// lane, then KS gathers of p, all in flight at once -- stages the products in
// its shared-memory slice, and lane l adds the products of row r0 + l that
// fall in the chunk, in column order.  A warp keeps 2 KS coalesced loads in
// flight instead of a lane group's few strided ones: the large systems of a
// batch, solved by one cluster each, are bound by the bytes a CTA has in
// flight.
template <typename T>
__device__ __forceinline__ void spmv_rows_stream(const int32_t* __restrict__ rp,
                                                 const int32_t* __restrict__ ci,
                                                 const T* __restrict__ val, const T* p, T* y,
                                                 int lo, int hi, double& pq, bool dot) {
  constexpr int KS = 8;
  constexpr int W = kThreads / 32;
  __shared__ T sh[W][32 * KS];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T* pw = sh[warp];
  for (int r0 = lo + warp * 32; r0 < hi; r0 += W * 32) {
    const int nr = min(32, hi - r0);
    const int row = r0 + lane;
    int rb = 0, re = 0;
    if (lane < nr) {
      rb = rp[row];
      re = rp[row + 1];
    }
    const int e0 = __shfl_sync(0xffffffffu, rb, 0);
    const int e1 = __shfl_sync(0xffffffffu, re, nr - 1);
    T s = T(0);
    for (int c0 = e0; c0 < e1; c0 += 32 * KS) {
      int c[KS];
      T v[KS];
#pragma unroll
      for (int k = 0; k < KS; k++) {
        const int j = c0 + k * 32 + lane;
        c[k] = j < e1 ? ci[j] : 0;
        v[k] = j < e1 ? val[j] : T(0);
      }
#pragma unroll
      for (int k = 0; k < KS; k++) {
        const int j = c0 + k * 32 + lane;
        if (j < e1) pw[k * 32 + lane] = v[k] * __ldcg(p + c[k]);
      }
      __syncwarp();
      const int a = max(rb, c0), b = min(re, c0 + 32 * KS);
      for (int j = a; j < b; j++) s += pw[j - c0];
      __syncwarp();
    }
    if (lane < nr) {
      y[row] = s;
      if (dot) pq += (double)__ldcg(p + row) * (double)s;
    }
  }
}

// The SpMV of the kernel's shape: CSR-stream (G == 1) or G lanes per row.
template <typename T, int G>
__device__ __forceinline__ void spmv_team_rows(const int32_t* __restrict__ rp,
                                               const int32_t* __restrict__ ci,
                                               const T* __restrict__ val, const T* p, T* y,
                                               int lo, int hi, double& pq, bool dot) {
  if constexpr (G == 1)
    spmv_rows_stream<T>(rp, ci, val, p, y, lo, hi, pq, dot);
  else
    spmv_rows<T, G>(rp, ci, val, p, y, lo, hi, pq, dot);
}

// One Jacobi pass of a factor over rows [lo, hi): out = v - Nt in, times the
// stored diagonal when scale (jacobi_sweep.cu).
template <typename T>
__device__ __forceinline__ void jacobi_rows(const Sell& F, const T* v, const T* in, T* out,
                                            bool scale, int lo, int hi) {
  const T* fv = sell_val<T>(F);
  const T* fd = sell_dinv<T>(F);
  constexpr int KK = 4;
  for (int r = lo + threadIdx.x; r < hi; r += kThreads) {
    const int s = r >> 5, lane = r & 31;
    const int base = F.d_slice_ptr[s], width = (F.d_slice_ptr[s + 1] - base) >> 5;
    T acc = T(0);
    for (int k0 = 0; k0 < width; k0 += KK) {
      int c[KK];
      T v[KK];
#pragma unroll
      for (int u = 0; u < KK; u++) {
        const bool inr = k0 + u < width;
        c[u] = inr ? F.d_col[base + 32 * (k0 + u) + lane] : -1;
        v[u] = inr ? fv[base + 32 * (k0 + u) + lane] : T(0);
      }
#pragma unroll
      for (int u = 0; u < KK; u++)
        if (c[u] >= 0) acc += v[u] * __ldcg(in + c[u]);
    }
    T res = __ldcg(v + r) - acc;
    if (scale) res *= fd[r];
    out[r] = res;
  }
}

// Element loops over the CTA's rows take 4 rows per thread per pass (rows
// i, i + 256, i + 512, i + 768): all loads of a pass are issued before its
// arithmetic and stores, so a thread keeps 4 DRAM requests per array in
// flight instead of walking its rows one round trip at a time.
constexpr int kU = 4;
#define MTLGPU_ROWS_PASS(i0) for (int i0 = lo + (int)threadIdx.x; i0 < hi; i0 += kU * kThreads)
#define MTLGPU_ROW(i0, u) ((i0) + (u) * kThreads)

// z = M^-1 r over the CTA's rows; factors take 2 jac_k passes, each after a
// team barrier (a pass reads other rows of the previous one).
template <typename T, typename Team>
__device__ __forceinline__ void apply_pc(Team& tm, const BatchArgs& a, const BatchVecs<T>& V,
                                         int lo, int hi) {
  if (a.pc == 2) {
    const int k = a.jac_k;
    // lower: r -> ... -> u (intermediates alternate between w and u)
    const T* in = V.r;
    for (int m = 0; m < k; m++) {
      T* out = ((k - 1 - m) % 2 == 0) ? V.u : V.w;
      jacobi_rows<T>(a.L, V.r, in, out, m == k - 1 && !a.L.unit_diag, lo, hi);
      tm.sync();
      in = out;
    }
    // upper: u -> ... -> z
    in = V.u;
    for (int m = 0; m < k; m++) {
      T* out = ((k - 1 - m) % 2 == 0) ? V.z : V.w;
      jacobi_rows<T>(a.U, V.u, in, out, m == k - 1, lo, hi);
      if (m + 1 < k) tm.sync();
      in = out;
    }
    return;
  }
  const T* di = dinv<T>(a);
  MTLGPU_ROWS_PASS(i0) {
    T rv[kU], dv[kU];
#pragma unroll
    for (int u = 0; u < kU; u++) {
      const int i = MTLGPU_ROW(i0, u);
      rv[u] = i < hi ? V.r[i] : T(0);
      dv[u] = (i < hi && a.pc == 1) ? di[i] : T(1);
    }
#pragma unroll
    for (int u = 0; u < kU; u++) {
      const int i = MTLGPU_ROW(i0, u);
      if (i < hi) V.z[i] = a.pc == 1 ? dv[u] * rv[u] : rv[u];
    }
  }
}

// One PCG solve of the cluster's system on the CTA's rows [lo, hi), from
// x = 0 with r holding the right-hand side (refinement) or from the caller's
// x with r = b - A x computed here (direct FP64).  Stops when ||r|| <= tol or
// after max_it iterations; returns the iteration count, *resid the last
// residual, *norm_rhs ||rhs||.
template <typename T, int G, typename Team>
__device__ int pcg_system(Team& tm, const BatchArgs& a,
                          const BatchVecs<T>& V, T* x, int lo, int hi, bool direct, double rtol,
                          double atol, int max_it, double* resid, double* norm_rhs,
                          int* error) {
  const T* A = vals<T>(a);
  double pq_dummy = 0;
  if (direct) {  // r = b - A x (x is the caller's initial guess)
    spmv_team_rows<T, G>(a.rp, a.ci, A, x, V.q, lo, hi, pq_dummy, false);
    __syncthreads();  // rows were written by their lane groups, read by thread
    for (int i = lo + threadIdx.x; i < hi; i += kThreads) V.r[i] = (T)a.b[i] - V.q[i];
  }
  double s0[3] = {0, 0, 0};
  for (int i = lo + threadIdx.x; i < hi; i += kThreads) {
    const double ri = (double)V.r[i];
    s0[0] += ri * ri;
    if (direct) s0[1] += a.b[i] * a.b[i];
  }
  tm.sum(s0);
  double rr = s0[0];
  const double nrm = direct ? sqrt(s0[1]) : sqrt(rr);
  *norm_rhs = nrm;
  const double tol = direct ? (nrm == 0 ? -1.0 : rtol * nrm) : rtol;
  auto finished = [&](double r_, int it_) {
    const bool conv = direct ? (nrm == 0 ? r_ <= atol : (r_ <= tol || r_ <= atol)) : r_ <= tol;
    if (conv) return 1;
    if (it_ >= max_it) return 2;
    return 0;
  };
  double res = sqrt(fabs(rr));
  int it = 0, fin = finished(res, it);
  double rho_1 = 0;
  while (!fin) {
    apply_pc<T>(tm, a, V, lo, hi);
    double s1[3] = {0, 0, 0};
    MTLGPU_ROWS_PASS(i0) {
      T rv[kU], zv[kU];
#pragma unroll
      for (int u = 0; u < kU; u++) {
        const int i = MTLGPU_ROW(i0, u);
        rv[u] = i < hi ? V.r[i] : T(0);
        zv[u] = i < hi ? V.z[i] : T(0);
      }
#pragma unroll
      for (int u = 0; u < kU; u++) s1[0] += (double)rv[u] * (double)zv[u];
    }
    tm.sum(s1);
    const double rho = s1[0];
    const T beta = it == 0 ? T(0) : (T)(rho / rho_1);
    MTLGPU_ROWS_PASS(i0) {
      T zv[kU], pv[kU];
#pragma unroll
      for (int u = 0; u < kU; u++) {
        const int i = MTLGPU_ROW(i0, u);
        zv[u] = i < hi ? V.z[i] : T(0);
        pv[u] = (i < hi && it > 0) ? V.p[i] : T(0);
      }
#pragma unroll
      for (int u = 0; u < kU; u++) {
        const int i = MTLGPU_ROW(i0, u);
        if (i < hi) V.p[i] = it == 0 ? zv[u] : zv[u] + beta * pv[u];
      }
    }
    tm.sync();  // p complete before the SpMV gathers it
    double s2[3] = {0, 0, 0};
    spmv_team_rows<T, G>(a.rp, a.ci, A, V.p, V.q, lo, hi, s2[0], true);
    tm.sum(s2);
    const T alpha = (T)(rho / s2[0]);
    double s3[3] = {0, 0, 0};
    MTLGPU_ROWS_PASS(i0) {
      T xv[kU], pv[kU], rv[kU], qv[kU];
#pragma unroll
      for (int u = 0; u < kU; u++) {
        const int i = MTLGPU_ROW(i0, u);
        const bool in = i < hi;
        xv[u] = in ? x[i] : T(0);
        pv[u] = in ? V.p[i] : T(0);
        rv[u] = in ? V.r[i] : T(0);
        qv[u] = in ? V.q[i] : T(0);
      }
#pragma unroll
      for (int u = 0; u < kU; u++) {
        const int i = MTLGPU_ROW(i0, u);
        const T ri = rv[u] - alpha * qv[u];
        s3[0] += (double)ri * (double)ri;
        if (i < hi) {
          x[i] = xv[u] + alpha * pv[u];
          V.r[i] = ri;
        }
      }
    }
    tm.sum(s3);
    rho_1 = rho;
    it++;
    res = sqrt(fabs(s3[0]));
    fin = finished(res, it);
  }
  *resid = res;
  *error = fin == 2;
  return it;
}

// One system on rows [lo, hi) of the team: direct FP64 PCG, or FP64
// refinement around FP32 inner PCG.
template <typename T, int G, typename Team>
__device__ BatchState solve_system(Team& tm, const BatchArgs& a, const BatchVecs<T>& V, int lo,
                                   int hi, int refine) {
  BatchState st{};
  if (!refine) {
    double resid = 0, nb = 0;
    int err = 0;
    for (int i = lo + threadIdx.x; i < hi; i += kThreads) V.p[i] = T(0);
    st.it = pcg_system<T, G>(tm, a, V, reinterpret_cast<T*>(a.x), lo, hi, true, a.rtol, a.atol,
                             a.max_iter, &resid, &nb, &err);
    st.resid = resid;
    st.norm_b = nb;
    st.error = err;
  } else {
    // FP64 refinement around FP32 inner solves
    const double* A64 = a.val64;
    double nb = 0;
    int total = 0, outer = 0;
    while (true) {
      double pq_dummy = 0;
      spmv_team_rows<double, G>(a.rp, a.ci, A64, a.x, a.r64, lo, hi, pq_dummy, false);
      __syncthreads();  // rows were written by their lane groups, read by thread
      double s0[3] = {0, 0, 0};
      for (int i = lo + threadIdx.x; i < hi; i += kThreads) {
        const double ri = a.b[i] - a.r64[i];
        a.r64[i] = ri;
        s0[0] += ri * ri;
        if (outer == 0) s0[1] += a.b[i] * a.b[i];
      }
      tm.sum(s0);
      const double resid = sqrt(s0[0]);
      if (outer == 0) nb = sqrt(s0[1]);
      st.resid = resid;
      const bool conv = nb == 0 ? resid <= a.atol : (resid <= a.rtol * nb || resid <= a.atol);
      if (conv) break;
      if (outer >= a.max_outer || total >= a.max_iter) {
        st.error = 1;
        break;
      }
      const double target = nb == 0 ? a.atol : fmax(a.rtol * nb, a.atol);
      const double itol = fmax(a.inner_rtol, fmin(0.5, 0.5 * target / resid));
      const double inv = 1.0 / resid;
      for (int i = lo + threadIdx.x; i < hi; i += kThreads) {
        V.r[i] = (T)(a.r64[i] * inv);
        V.d[i] = T(0);
        V.p[i] = T(0);
      }
      tm.sync();
      double ir = 0, in_norm = 0;
      int ierr = 0;
      total += pcg_system<T, G>(tm, a, V, V.d, lo, hi, false, itol, 0.0,
                                min(a.inner_max, a.max_iter - total), &ir, &in_norm, &ierr);
      for (int i = lo + threadIdx.x; i < hi; i += kThreads) a.x[i] += resid * (double)V.d[i];
      outer++;
      tm.sync();  // x complete before the next residual
    }
    st.it = total;
    st.outer = outer;
    st.norm_b = nb;
  }
  st.done = 1;
  return st;
}

// Phase 1: each cluster takes the large systems (order[0 .. n_large)) one at
// a time from queue[0] and solves each with all its CTAs.  Phase 2, once the
// large queue is empty: every CTA takes small systems (order[n_large ..
// count)) from queue[1] and solves each alone.  No distributed-shared-memory
// access follows the last cluster barrier of phase 1, so CTAs may leave
// independently.
// 4 CTAs per SM: 64 registers a thread, no spills (measured 5 % faster for
// the FP32-refined and Jacobi-applied IC(0) solves than 3 CTAs at 80).
template <typename T, int G>
__global__ void __launch_bounds__(kThreads, 4)
    batch_cluster_kernel(BatchArgs a, BatchVecs<T> V, int refine) {
  __shared__ ClusterSum<3> cs;
  __shared__ int item;
  ClusterTeam tm{cgx::this_cluster(), &cs, 0};
  const unsigned crank = tm.cl.block_rank(), csz = tm.cl.num_blocks();
  while (true) {
    if (crank == 0 && threadIdx.x == 0) item = (int)atomicAdd(a.queue, 1u);
    tm.cl.sync();
    const int q = *tm.cl.map_shared_rank(&item, 0);
    tm.cl.sync();  // every CTA has read the item before rank 0 takes the next
    if (q >= a.n_large) break;
    const int s = a.order[q];
    const int slo = a.off[s], shi = a.off[s + 1], ns = shi - slo;
    const int lo = slo + (int)((long long)ns * crank / csz);
    const int hi = slo + (int)((long long)ns * (crank + 1) / csz);
    const BatchState st = solve_system<T, G>(tm, a, V, lo, hi, refine);
    if (crank == 0 && threadIdx.x == 0) a.state[s] = st;
    tm.cl.sync();  // the system's vectors are final before the cluster moves on
  }
  CtaTeam tb{&cs};
  const int n_small = a.count - a.n_large;
  while (true) {
    __syncthreads();
    if (threadIdx.x == 0) item = (int)atomicAdd(a.queue + 1, 1u);
    __syncthreads();
    const int q = item;
    if (q >= n_small) break;
    const int s = a.order[a.n_large + q];
    const BatchState st = solve_system<T, G>(tb, a, V, a.off[s], a.off[s + 1], refine);
    if (threadIdx.x == 0) a.state[s] = st;
  }
}

// ||b - A x|| per system (Ax given)
__global__ void __launch_bounds__(kThreads)
    batch_cluster_true_resid(const int32_t* __restrict__ off, const double* __restrict__ b,
                             const double* __restrict__ ax, double* out) {
  const int s = blockIdx.x, lo = off[s], hi = off[s + 1];
  Sum<1> acc = Sum<1>::zero();
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    const double v = b[i] - ax[i];
    acc.add(0, v * v);
  }
  acc = block_reduce(acc);
  if (threadIdx.x == 0) out[s] = sqrt(acc.value(0));
}

template <typename T, int G>
cudaError_t launch_cluster(cudaStream_t st, int cs, int clusters, const BatchArgs& a,
                           const BatchVecs<T>& V, int refine) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(clusters * cs));
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, batch_cluster_kernel<T, G>, a, V, refine);
}

template <typename T, int G>
int max_clusters(int cs) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(cs * 256));
  cfg.blockDim = dim3(kThreads);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, batch_cluster_kernel<T, G>, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

template <typename T>
cudaError_t launch_g(cudaStream_t st, int g, int cs, int clusters, const BatchArgs& a,
                     const BatchVecs<T>& V, int refine) {
  switch (g) {
    case 1: return launch_cluster<T, 1>(st, cs, clusters, a, V, refine);
    case 4: return launch_cluster<T, 4>(st, cs, clusters, a, V, refine);
    case 16: return launch_cluster<T, 16>(st, cs, clusters, a, V, refine);
    case 32: return launch_cluster<T, 32>(st, cs, clusters, a, V, refine);
    default: return launch_cluster<T, 8>(st, cs, clusters, a, V, refine);
  }
}

template <typename T>
int clusters_for(int g, int cs) {
  switch (g) {
    case 1: return max_clusters<T, 1>(cs);
    case 4: return max_clusters<T, 4>(cs);
    case 16: return max_clusters<T, 16>(cs);
    case 32: return max_clusters<T, 32>(cs);
    default: return max_clusters<T, 8>(cs);
  }
}

}  // namespace

// Whether the batched solve with P runs as one persistent cluster launch:
// identity, diagonal, and factors applied by Jacobi iterations.
bool batched_cluster_supported(const Pc* P) {
  return !P || P->kind == MTLGPU_PC_IDENTITY || P->kind == MTLGPU_PC_DIAGONAL ||
         ((P->kind == MTLGPU_PC_IC0 || P->kind == MTLGPU_PC_ILU0) && P->jacobi_iters > 0);
}

// Everything one configuration of the batched solve needs, cached on the
// matrix handle: the system order, the buffers, and a CUDA graph of the whole
// call -- reset of the queues, the persistent kernel, the true residuals and
// the copies of the per-system results to pinned host memory.  A call with
// the same systems, vectors, preconditioner and shape replays the graph.
struct BatchWork {
  // key
  const Pc* P = nullptr;
  int pc_kind = -1, jac_k = 0;
  int count = 0, small_rows = 0, refine = 0, cs = 0, g = 0;
  unsigned long long off_hash = 0;
  const double* x = nullptr;
  const double* b = nullptr;
  const float* val32 = nullptr;
  double rtol = 0, atol = 0, inner_rtol = 0;
  int max_iter = 0, inner_max = 0, max_outer = 0;
  // data
  int n_large = 0;
  int32_t *d_off = nullptr, *d_order = nullptr;
  BatchState* d_state = nullptr;
  unsigned* d_queue = nullptr;
  double *d_r64 = nullptr, *d_ax = nullptr, *d_tr = nullptr;
  char* vecs = nullptr;
  BatchState* h_state = nullptr;
  double* h_tr = nullptr;
  cudaGraphExec_t exec = nullptr;
};

void batch_work_free(Ctx* ctx, BatchWork* w) {
  if (!w) return;
  if (w->exec) cudaGraphExecDestroy(w->exec);
  dfree(ctx, w->d_off);
  dfree(ctx, w->d_order);
  dfree(ctx, w->d_state);
  dfree(ctx, w->d_queue);
  dfree(ctx, w->d_r64);
  dfree(ctx, w->d_ax);
  dfree(ctx, w->d_tr);
  dfree(ctx, w->vecs);
  if (w->h_state) cudaFreeHost(w->h_state);
  if (w->h_tr) cudaFreeHost(w->h_tr);
  delete w;
}

// Drops the cached batched configuration of A (all of it, or only if it
// uses preconditioner only_P).
void release_batch_work(Csr* A, const Pc* only_P) {
  BatchWork* w = static_cast<BatchWork*>(A->batch_work);
  if (!w || (only_P && w->P != only_P)) return;
  batch_work_free(A->ctx, w);
  A->batch_work = nullptr;
}

namespace {

unsigned long long hash_offsets(const int32_t* h_off, int count) {
  unsigned long long h = 1469598103934665603ull;
  for (int i = 0; i <= count; i++) h = (h ^ (unsigned)h_off[i]) * 1099511628211ull;
  return h;
}

template <typename T>
BatchVecs<T> carve(char* vecs, size_t vec_bytes) {
  BatchVecs<T> V;
  T* base = reinterpret_cast<T*>(vecs);
  const size_t stride = vec_bytes / sizeof(T);
  V.r = base, V.z = base + stride, V.p = base + 2 * stride, V.q = base + 3 * stride;
  V.d = base + 4 * stride, V.u = base + 5 * stride, V.w = base + 6 * stride;
  return V;
}

mtlgpu_status batch_work_build(Csr* A, Pc* P, int count, const int32_t* h_off, double* d_x,
                               const double* d_b, const mtlgpu_iter_params* prm, int cs, int g,
                               int small_rows, BatchWork* w) {
  Ctx* ctx = A->ctx;
  const bool refine = w->refine;
  const int n = A->n_rows;
  // order: the systems of at least small_rows rows (solved by a whole
  // cluster), then the others (solved by one CTA each), each group by
  // decreasing stored entries (longest solves first)
  std::vector<int32_t> h_rp(n + 1);
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(h_rp.data(), A->d_rp, sizeof(int32_t) * (n + 1),
                                       cudaMemcpyDeviceToHost, ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  std::vector<int32_t> order(count);
  std::iota(order.begin(), order.end(), 0);
  auto large = [&](int s_) { return h_off[s_ + 1] - h_off[s_] >= small_rows; };
  std::stable_sort(order.begin(), order.end(), [&](int a_, int b_) {
    if (large(a_) != large(b_)) return large(a_);
    return h_rp[h_off[a_ + 1]] - h_rp[h_off[a_]] > h_rp[h_off[b_ + 1]] - h_rp[h_off[b_]];
  });
  for (int s_ = 0; s_ < count; ++s_) w->n_large += large(s_);
  const size_t ts = refine ? sizeof(float) : sizeof(double);
  const size_t vec_bytes = ((ts * (size_t)n + 255) / 256) * 256;
  MTLGPU_TRY(dalloc(ctx, &w->d_off, count + 1));
  MTLGPU_TRY(dalloc(ctx, &w->d_order, count));
  MTLGPU_TRY(dalloc(ctx, &w->d_state, count));
  MTLGPU_TRY(dalloc(ctx, &w->d_queue, 2));
  MTLGPU_TRY(dalloc(ctx, &w->d_ax, n));
  MTLGPU_TRY(dalloc(ctx, &w->d_tr, count));
  if (refine) MTLGPU_TRY(dalloc(ctx, &w->d_r64, n));
  MTLGPU_TRY(dalloc(ctx, &w->vecs, 7 * vec_bytes));
  MTLGPU_TRY_CUDA(ctx, cudaMallocHost(reinterpret_cast<void**>(&w->h_state),
                                      sizeof(BatchState) * count));
  MTLGPU_TRY_CUDA(ctx, cudaMallocHost(reinterpret_cast<void**>(&w->h_tr), sizeof(double) * count));
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(w->d_off, h_off, sizeof(int32_t) * (count + 1),
                                       cudaMemcpyHostToDevice, ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(w->d_order, order.data(), sizeof(int32_t) * count,
                                       cudaMemcpyHostToDevice, ctx->stream));

  BatchArgs a;
  std::memset(&a, 0, sizeof(a));
  a.count = count;
  a.n_large = w->n_large;
  a.order = w->d_order;
  a.off = w->d_off;
  a.rp = A->d_rp;
  a.ci = A->d_ci;
  a.val64 = A->d_v;
  a.val32 = A->d_v32;
  if (P && P->kind == MTLGPU_PC_DIAGONAL) {
    a.pc = 1;
    a.dinv64 = P->d_inv_diag;
    a.dinv32 = P->d_inv_diag32;
  } else if (P && (P->kind == MTLGPU_PC_IC0 || P->kind == MTLGPU_PC_ILU0)) {
    a.pc = 2;
    a.L = P->jac_lower;
    a.U = P->jac_upper;
    a.jac_k = P->jacobi_iters;
  }
  a.b = d_b;
  a.x = d_x;
  a.r64 = w->d_r64;
  a.state = w->d_state;
  a.queue = w->d_queue;
  a.rtol = prm->rtol;
  a.atol = prm->atol;
  a.inner_rtol = prm->inner_rtol > 0 ? prm->inner_rtol : 1e-6;
  a.max_iter = prm->max_iter;
  a.inner_max = prm->inner_max_iter > 0 ? prm->inner_max_iter : prm->max_iter;
  a.max_outer = prm->max_outer > 0 ? prm->max_outer : 30;
  a.g = g;
  int mc = refine ? clusters_for<float>(g, cs) : clusters_for<double>(g, cs);
  if (mc <= 0) return MTLGPU_NOT_SUPPORTED;
  // persistent: as many clusters as fit the GPU at once (phase 2 keeps every
  // CTA busy on small systems once the large ones are taken)
  const int clusters = mc;

  // the graph of one call
  cudaGraph_t graph = nullptr;
  const long long launches_before = ctx->launches;
  MTLGPU_TRY_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaMemsetAsync(w->d_queue, 0, 2 * sizeof(unsigned), ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(w->d_state, 0, sizeof(BatchState) * count, ctx->stream);
  if (e == cudaSuccess)
    e = refine ? launch_g<float>(ctx->stream, g, cs, clusters, a,
                                 carve<float>(w->vecs, vec_bytes), 1)
               : launch_g<double>(ctx->stream, g, cs, clusters, a,
                                  carve<double>(w->vecs, vec_bytes), 0);
  mtlgpu_status st = MTLGPU_OK;
  if (e == cudaSuccess) {
    SpmvArgs plain;
    st = spmv_launch<double>(A, d_x, w->d_ax, plain);
  }
  if (e == cudaSuccess && st == MTLGPU_OK) {
    batch_cluster_true_resid<<<count, kThreads, 0, ctx->stream>>>(w->d_off, d_b, w->d_ax,
                                                                   w->d_tr);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && st == MTLGPU_OK)
    e = cudaMemcpyAsync(w->h_state, w->d_state, sizeof(BatchState) * count,
                        cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess && st == MTLGPU_OK)
    e = cudaMemcpyAsync(w->h_tr, w->d_tr, sizeof(double) * count, cudaMemcpyDeviceToHost,
                        ctx->stream);
  cudaError_t ee = cudaStreamEndCapture(ctx->stream, &graph);
  ctx->launches = launches_before;
  if (e == cudaSuccess) e = ee;
  if (e != cudaSuccess || st != MTLGPU_OK) {
    if (graph) cudaGraphDestroy(graph);
    return st != MTLGPU_OK ? st : set_cuda_error(ctx, e, "batched graph capture");
  }
  e = cudaGraphInstantiate(&w->exec, graph, 0);
  cudaGraphDestroy(graph);
  MTLGPU_TRY_CUDA(ctx, e);
  return MTLGPU_OK;
}

}  // namespace

mtlgpu_status solve_batched_cluster(Csr* A, Pc* P, int count, const int32_t* h_off, double* d_x,
                                    const double* d_b, const mtlgpu_iter_params* prm,
                                    mtlgpu_iter_result* res, int cs, int g, int small_rows,
                                    float* ms_out) {
  Ctx* ctx = A->ctx;
  const bool refine = prm->mode == MTLGPU_SOLVE_MIXED_REFINED;
  if (refine && P && P->kind != MTLGPU_PC_IDENTITY && P->prec != MTLGPU_FP32)
    return MTLGPU_INVALID_ARG;
  if (refine) MTLGPU_TRY(csr_ensure_fp32(A));
  const unsigned long long hsh = hash_offsets(h_off, count);
  BatchWork* w = static_cast<BatchWork*>(A->batch_work);
  const int pk = P ? P->kind : -1, jk = P ? P->jacobi_iters : 0;
  // the iteration parameters are baked into the graph: compare them too
  auto same_params = [&](const BatchWork* v) {
    return v->rtol == prm->rtol && v->atol == prm->atol && v->inner_rtol == prm->inner_rtol &&
           v->max_iter == prm->max_iter && v->inner_max == prm->inner_max_iter &&
           v->max_outer == prm->max_outer;
  };
  if (!w || w->P != P || w->pc_kind != pk || w->jac_k != jk || w->count != count ||
      w->small_rows != small_rows || w->refine != (int)refine || w->cs != cs || w->g != g ||
      w->off_hash != hsh || w->x != d_x || w->b != d_b || w->val32 != A->d_v32 || !same_params(w)) {
    release_batch_work(A, nullptr);
    w = new BatchWork();
    w->P = P, w->pc_kind = pk, w->jac_k = jk, w->count = count, w->small_rows = small_rows;
    w->refine = refine, w->cs = cs, w->g = g, w->off_hash = hsh, w->x = d_x, w->b = d_b;
    w->val32 = A->d_v32;
    w->rtol = prm->rtol, w->atol = prm->atol, w->inner_rtol = prm->inner_rtol;
    w->max_iter = prm->max_iter, w->inner_max = prm->inner_max_iter;
    w->max_outer = prm->max_outer;
    A->batch_work = w;
    mtlgpu_status st = batch_work_build(A, P, count, h_off, d_x, d_b, prm, cs, g, small_rows, w);
    if (st != MTLGPU_OK) {
      release_batch_work(A, nullptr);
      return st;
    }
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (ms_out) {
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, ctx->stream);
  }
  MTLGPU_TRY_CUDA(ctx, cudaGraphLaunch(w->exec, ctx->stream));
  ctx->launches += 3;  // persistent kernel, SpMV, true residuals
  if (ms_out) {
    cudaEventRecord(e1, ctx->stream);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms_out, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  MTLGPU_TRY(take_device_error(ctx));
  bool any_max = false;
  for (int s = 0; s < count; ++s) {
    mtlgpu_iter_result& R = res[s];
    std::memset(&R, 0, sizeof(R));
    const BatchState& hs = w->h_state[s];
    R.iterations = hs.it;
    R.outer_iterations = hs.outer;
    R.error = hs.done ? hs.error : 1;
    R.status = R.error ? MTLGPU_MAX_ITER : MTLGPU_OK;
    R.resid = hs.resid;
    R.norm_r0 = hs.norm_b;
    R.true_resid = w->h_tr[s];
    R.kernel_launches = 1;
    any_max |= R.error != 0;
  }
  return any_max ? MTLGPU_MAX_ITER : MTLGPU_OK;
}

}  // namespace mtlgpu
