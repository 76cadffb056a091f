// Device helpers: coherent loads/stores, bounded waits on NaN-boxed values,
// compensated FP32 accumulation and deterministic grid reductions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "mtlgpu.h"

namespace mtlgpu {
namespace dev {

// ---------------------------------------------------------------------------
// Coherent (L1-bypassing) accesses at GPU scope.
__device__ __forceinline__ double ld_relaxed(const double* p) {
  double v;
  asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ float ld_relaxed(const float* p) {
  float v;
  asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_relaxed(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed(double* p, double v) {
  asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(float* p, float v) {
  asm volatile("st.relaxed.gpu.global.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(int* p, int v) {
  asm volatile("st.relaxed.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// ---------------------------------------------------------------------------
// NaN boxing: a not-yet-computed entry of a sweep output holds a signalling
// NaN with a fixed payload.  Arithmetic never produces a signalling NaN (every
// NaN result is quiet), and results are canonicalised before being stored, so
// "value != sentinel" means "value is final".  One 64/32-bit word is both the
// datum and its ready flag: no separate flag array and no fence are needed.
template <typename T> struct Box;
template <> struct Box<double> {
  static constexpr unsigned long long bits = 0x7FF4DEADBEEF1234ull;
  __device__ __forceinline__ static double sentinel() { return __longlong_as_double((long long)bits); }
  __device__ __forceinline__ static bool is(double v) {
    return (unsigned long long)__double_as_longlong(v) == bits;
  }
};
template <> struct Box<float> {
  static constexpr unsigned bits = 0x7FA0BEEFu;
  __device__ __forceinline__ static float sentinel() { return __uint_as_float(bits); }
  __device__ __forceinline__ static bool is(float v) { return __float_as_uint(v) == bits; }
};
template <> struct Box<int> {
  static constexpr int bits = -0x7ABCDEF1;
  __device__ __forceinline__ static int sentinel() { return bits; }
  __device__ __forceinline__ static bool is(int v) { return v == bits; }
};

template <typename T>
__device__ __forceinline__ T canonical(T v) {
  return Box<T>::is(v) ? T(__int_as_float(0x7fc00000)) : v;
}
__device__ __forceinline__ int canonical(int v) { return v; }

// Bounded wait until *p holds a final value.  Gives up after `limit` polls
// (or as soon as another thread has already recorded an error), records
// MTLGPU_TIMEOUT in *err and returns 0.
template <typename T>
__device__ __forceinline__ T wait_value(const T* p, long long limit, int* err) {
  T v = ld_relaxed(p);
  if (!Box<T>::is(v)) return v;
  long long k = 0;
  while (true) {
    v = ld_relaxed(p);
    if (!Box<T>::is(v)) return v;
    if (++k >= limit) break;
    if ((k & 1023) == 0 && ld_relaxed(err) != 0) return T(0);
  }
  atomicCAS(err, 0, (int)MTLGPU_TIMEOUT);
  return T(0);
}

// ---------------------------------------------------------------------------
// Accumulators.  Sum<K>: K doubles.  CSum<K>: K compensated float sums
// (Ogita-Rump-Oishi Dot2: TwoSum on the running sum, the rounding error of
// each product recovered with an FMA).
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
  s = a + b;
  float bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}

template <int K>
struct Sum {
  double v[K];
  __device__ __forceinline__ static Sum zero() {
    Sum s;
#pragma unroll
    for (int i = 0; i < K; i++) s.v[i] = 0.0;
    return s;
  }
  __device__ __forceinline__ void add(int i, double x) { v[i] += x; }
  __device__ __forceinline__ void add_prod(int i, double a, double b) { v[i] += a * b; }
  __device__ __forceinline__ void merge(const Sum& o) {
#pragma unroll
    for (int i = 0; i < K; i++) v[i] += o.v[i];
  }
  __device__ __forceinline__ void shfl_down(int off) {
#pragma unroll
    for (int i = 0; i < K; i++) v[i] += __shfl_down_sync(0xffffffffu, v[i], off);
  }
  __device__ __forceinline__ double value(int i) const { return v[i]; }
};

template <int K>
struct CSum {
  float hi[K], lo[K];
  __device__ __forceinline__ static CSum zero() {
    CSum s;
#pragma unroll
    for (int i = 0; i < K; i++) s.hi[i] = 0.f, s.lo[i] = 0.f;
    return s;
  }
  __device__ __forceinline__ void add(int i, float x) {
    float s, e;
    two_sum(hi[i], x, s, e);
    hi[i] = s;
    lo[i] += e;
  }
  __device__ __forceinline__ void add_prod(int i, float a, float b) {
    float p = a * b;
    float ep = fmaf(a, b, -p);
    float s, e;
    two_sum(hi[i], p, s, e);
    hi[i] = s;
    lo[i] += e + ep;
  }
  __device__ __forceinline__ void merge(const CSum& o) {
#pragma unroll
    for (int i = 0; i < K; i++) {
      float s, e;
      two_sum(hi[i], o.hi[i], s, e);
      hi[i] = s;
      lo[i] += o.lo[i] + e;
    }
  }
  __device__ __forceinline__ void shfl_down(int off) {
    CSum o;
#pragma unroll
    for (int i = 0; i < K; i++) {
      o.hi[i] = __shfl_down_sync(0xffffffffu, hi[i], off);
      o.lo[i] = __shfl_down_sync(0xffffffffu, lo[i], off);
    }
    merge(o);
  }
  __device__ __forceinline__ double value(int i) const { return (double)hi[i] + (double)lo[i]; }
};

// Accumulator type for vector element type T with K values.
template <typename T, int K> struct AccOf { typedef Sum<K> type; };
template <int K> struct AccOf<float, K> { typedef CSum<K> type; };

template <typename R>
__device__ __forceinline__ R warp_reduce(R r) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) r.shfl_down(off);
  return r;  // lane 0 holds the total
}

// Block-wide reduction; the result is valid in thread 0.  Requires
// blockDim.x a multiple of 32 and <= 1024.
template <typename R>
__device__ __forceinline__ R block_reduce(R r) {
  __shared__ __align__(16) unsigned char smem_raw[32 * sizeof(R)];
  R* sm = reinterpret_cast<R*>(smem_raw);
  r = warp_reduce(r);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sm[wid] = r;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  R t = R::zero();
  if (wid == 0) {
    if (lane < nw) t = sm[lane];
    t = warp_reduce(t);
  }
  return t;
}

// Writes this block's partial to partials[slot]; returns true (in every
// thread of the block) in the last of `expected` blocks to arrive, after
// which the caller sums partials[0..count) with reduce_partials().  The
// counter is reset for the next use.
template <typename R>
__device__ __forceinline__ bool publish_partial(const R& blocksum, R* partials, int slot,
                                                unsigned* counter, unsigned expected) {
  __shared__ bool last;
  if (threadIdx.x == 0) {
    partials[slot] = blocksum;
    __threadfence();
    unsigned prev = atomicAdd(counter, 1u);
    last = (prev == expected - 1);
    if (last) {
      *counter = 0;
      __threadfence();
    }
  }
  __syncthreads();
  return last;
}

// Deterministic sum of partials[0..count) (fixed assignment of partials to
// threads and a fixed reduction tree).  Result valid in thread 0.
template <typename R>
__device__ __forceinline__ R reduce_partials(const R* partials, int count) {
  R acc = R::zero();
  for (int i = threadIdx.x; i < count; i += blockDim.x) {
    static_assert(sizeof(R) % 8 == 0, "partials are moved as 8-byte words");
    R p;
    // L2 loads: the partials were written by other blocks (ordered by the
    // fence + counter in publish_partial), so L1 must not serve them.
    const double* src = reinterpret_cast<const double*>(partials + i);
    double* dst = reinterpret_cast<double*>(&p);
#pragma unroll
    for (int w = 0; w < (int)(sizeof(R) / 8); w++) dst[w] = __ldcg(src + w);
    acc.merge(p);
  }
  return block_reduce(acc);
}

// 16-byte vector access: VN<T> elements per load / store (4 floats, 2
// doubles).  The pointer must be 16-byte aligned (every library buffer is).
template <typename T>
struct VN {
  static constexpr int value = 16 / (int)sizeof(T);
};
__device__ __forceinline__ void ld16(const float* p, float (&o)[4]) {
  const float4 v = *reinterpret_cast<const float4*>(p);
  o[0] = v.x, o[1] = v.y, o[2] = v.z, o[3] = v.w;
}
__device__ __forceinline__ void ld16(const double* p, double (&o)[2]) {
  const double2 v = *reinterpret_cast<const double2*>(p);
  o[0] = v.x, o[1] = v.y;
}
__device__ __forceinline__ void st16(float* p, const float (&o)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(o[0], o[1], o[2], o[3]);
}
__device__ __forceinline__ void st16(double* p, const double (&o)[2]) {
  *reinterpret_cast<double2*>(p) = make_double2(o[0], o[1]);
}

// Grid-stride loop bounds helper.
__device__ __forceinline__ long long gtid() {
  return (long long)blockIdx.x * blockDim.x + threadIdx.x;
}
__device__ __forceinline__ long long gstride() { return (long long)gridDim.x * blockDim.x; }

}  // namespace dev
}  // namespace mtlgpu
