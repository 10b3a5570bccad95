// Shared helpers of the B200 R-matrix solver: complex arithmetic on interleaved pairs,
// error plumbing, the bounded grid barrier used by cooperative kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

namespace hprmat {

// ---------------------------------------------------------------- complex arithmetic
template <typename R> struct Cplx;
template <> struct Cplx<double> { using T = double2; };
template <> struct Cplx<float> { using T = float2; };

template <typename T> struct RealOf;
template <> struct RealOf<double2> { using R = double; };
template <> struct RealOf<float2> { using R = float; };

__host__ __device__ inline double2 mk(double a, double b) { return make_double2(a, b); }
__host__ __device__ inline float2 mk(float a, float b) { return make_float2(a, b); }
template <typename T> __host__ __device__ inline T czero() { T z; z.x = 0; z.y = 0; return z; }

template <typename T> __host__ __device__ inline T cadd(T a, T b) { T r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename T> __host__ __device__ inline T csub(T a, T b) { T r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename T> __host__ __device__ inline T cmul(T a, T b) {
  T r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
// acc -= a*b with fused multiply-adds
template <typename T> __host__ __device__ inline void cfms(T& acc, T a, T b) {
  acc.x = fma(-a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(-a.x, b.y, acc.y);
  acc.y = fma(-a.y, b.x, acc.y);
}
// acc += a*b
template <typename T> __host__ __device__ inline void cfma(T& acc, T a, T b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
// |re| + |im|: the modulus izamax/icamax use to choose pivots (LAPACK dcabs1)
template <typename T> __host__ __device__ inline typename RealOf<T>::R cabs1(T a) {
  return fabs(a.x) + fabs(a.y);
}
// 1/a with scaling (Smith's method) so that neither tiny nor huge pivots overflow
template <typename T> __host__ __device__ inline T crecip(T a) {
  using R = typename RealOf<T>::R;
  T r;
  if (fabs(a.x) >= fabs(a.y)) {
    R t = a.y / a.x;
    R d = a.x + a.y * t;
    r.x = R(1) / d;
    r.y = -t / d;
  } else {
    R t = a.x / a.y;
    R d = a.x * t + a.y;
    r.x = t / d;
    r.y = R(-1) / d;
  }
  return r;
}
// a/b (Smith)
template <typename T> __host__ __device__ inline T cdiv(T a, T b) { return cmul(a, crecip(b)); }

// ---------------------------------------------------------------- magnitude keys
// Integer keys that order like non-negative magnitudes, for atomicMax reductions.
//
// Pivot keys (64 bits): the candidate's |re|+|im| in the high bits, the complement of its row
// in the low bits, so that one 64-bit atomicMax picks the largest modulus and, among equal
// ones, the lowest row (LAPACK izamax).  The magnitude part is never 0 for a real candidate
// (0 means "none").  FP32 panels keep all float bits; FP64 panels keep the top 44 bits of the
// double (sign, 11 exponent bits, 32 mantissa bits), which orders the whole double range --
// magnitudes below 1e-38 or above 3e38 included -- with rows below 2^20.
template <typename T> struct PivotKey;
template <> struct PivotKey<float2> {
  using M = unsigned;
  static constexpr int kMaxRows = 0x7fffffff;
  __device__ static __forceinline__ M mag(float2 v) { return __float_as_uint(fabsf(v.x) + fabsf(v.y)) + 1u; }
  __device__ static __forceinline__ unsigned long long key(M m, int row) {
    return ((unsigned long long)m << 32) | (unsigned long long)(0xFFFFFFFFu - (unsigned)row);
  }
  __device__ static __forceinline__ int row(unsigned long long k) {
    return (int)(0xFFFFFFFFu - (unsigned)(k & 0xFFFFFFFFull));
  }
};
template <> struct PivotKey<double2> {
  using M = unsigned long long;
  static constexpr int kMaxRows = 1 << 20;
  __device__ static __forceinline__ M mag(double2 v) {
    return ((unsigned long long)__double_as_longlong(fabs(v.x) + fabs(v.y)) >> 20) + 1ull;
  }
  __device__ static __forceinline__ unsigned long long key(M m, int row) {
    return (m << 20) | (unsigned long long)(0xFFFFFu - (unsigned)row);
  }
  __device__ static __forceinline__ int row(unsigned long long k) { return (int)(0xFFFFFu - (unsigned)(k & 0xFFFFFull)); }
};

// 32-bit key of a non-negative magnitude over the whole double range: the high word of its
// IEEE-754 double (11 exponent bits, 20 mantissa bits).  The pivot-growth and max |c_ij|
// words of the status block hold such keys (atomicMax), on both precisions.
__device__ __forceinline__ unsigned mag_hi(double v) { return (unsigned)__double2hiint(v); }
// The magnitude a key stands for (within a relative 2^-20 below the value it was made from).
__host__ inline double mag_hi_value(unsigned k) {
  const unsigned long long b = (unsigned long long)k << 32;
  double v;
  memcpy(&v, &b, sizeof(v));
  return v;
}

__host__ __device__ inline float2 to_f(double2 a) { return make_float2((float)a.x, (float)a.y); }
__host__ __device__ inline double2 to_d(float2 a) { return make_double2((double)a.x, (double)a.y); }

// ---------------------------------------------------------------- TF32 split
// Split x into an exactly-representable TF32 head and the FP32 remainder.  hi = x rounded
// to 10 explicit mantissa bits (round-to-nearest-even on the raw bits), lo = x - hi is
// exact in FP32 and |lo| <= 2^-11 |x|.
__device__ __forceinline__ void tf32_split(float x, float& hi, float& lo) {
  unsigned u = __float_as_uint(x);
  unsigned r = u + 0x0FFFu + ((u >> 13) & 1u);
  r &= 0xFFFFE000u;
  // keep inf/nan as they are
  if ((u & 0x7F800000u) == 0x7F800000u) r = u;
  hi = __uint_as_float(r);
  lo = x - hi;
}

// Device clock in ns (for optional timing traces).
__device__ __forceinline__ long long device_ns() {
  long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// ---------------------------------------------------------------- device status words
// Layout of the per-context device status block (int32 each).
enum StatusWord {
  SW_INFO = 0,       // first zero pivot, 1-based (LAPACK info), 0 if none
  SW_TIMEOUT = 1,    // nonzero if a bounded wait gave up (value = site id)
  SW_BARRIER = 2,    // grid barrier arrival counter (reset per cooperative launch)
  SW_COUNT = 8
};

// Bounded grid-wide barrier for cooperative launches.  `target` = number of CTAs times
// the barrier's ordinal (1-based) since the counter was zeroed.  Thread 0 arrives with a
// release-ordered add (publishing the CTA's earlier writes, ordered by __syncthreads) and
// polls with acquire loads; the error flag is looked at only every 4096 polls.  Returns
// false when the wait exceeded its limit; the caller must then stop touching shared data
// and return.
__device__ inline bool grid_barrier(int* counter, int* timeout_flag, unsigned target, int site) {
  __syncthreads();
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(counter) : "memory");
    int ok = 1;
    for (unsigned spins = 1;; ++spins) {
      unsigned v;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(counter) : "memory");
      if (v >= target) break;
      if ((spins & 4095u) == 0) {
        int tf;
        asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(tf) : "l"(timeout_flag) : "memory");
        if (tf != 0) { ok = 0; break; }
        if (spins >= (1u << 26)) {  // seconds: something is wrong
          atomicExch(timeout_flag, site);
          ok = 0;
          break;
        }
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// The two halves of grid_barrier, so that a CTA can work between arriving and waiting.
// grid_arrive is called by thread 0 after a __syncthreads that orders the CTA's writes.
__device__ inline void grid_arrive(int* counter) {
  asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(counter) : "memory");
}
// All threads; false when the bounded wait gave up (the caller must return): after `limit`
// polls (checked every 4096) it records `site` in *timeout_flag.
__device__ inline bool grid_wait(int* counter, int* timeout_flag, unsigned target, int site,
                                 unsigned limit = (1u << 26)) {
  __shared__ int s_ok_w;
  if (threadIdx.x == 0) {
    int ok = 1;
    for (unsigned spins = 1;; ++spins) {
      unsigned v;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(counter) : "memory");
      if (v >= target) break;
      if ((spins & 4095u) == 0) {
        int tf;
        asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(tf) : "l"(timeout_flag) : "memory");
        if (tf != 0) { ok = 0; break; }
        if (spins >= limit) {
          atomicExch(timeout_flag, site);
          ok = 0;
          break;
        }
      }
    }
    s_ok_w = ok;
  }
  __syncthreads();
  return s_ok_w != 0;
}

}  // namespace hprmat

// ---------------------------------------------------------------- host error plumbing
#define HPR_CUDA_TRY(expr)                                                           \
  do {                                                                               \
    cudaError_t _e = (expr);                                                         \
    if (_e != cudaSuccess) {                                                         \
      hprmat::set_last_error(_e, #expr, __FILE__, __LINE__);                         \
      return (_e == cudaErrorMemoryAllocation) ? -3 : -2;                            \
    }                                                                                \
  } while (0)

namespace hprmat {
void set_last_error(cudaError_t e, const char* what, const char* file, int line);
void set_last_error_msg(const char* msg);
}  // namespace hprmat
