// Common device/host helpers for the Tarang B200 hot path: a POD complex type whose layout
// matches the reference's complex<double> (two reals, real part first), error plumbing and
// the axis maps that describe which wavenumbers of an axis are stored.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

namespace tg {

template <typename R>
struct __align__(2 * sizeof(R)) cx {
  R x, y;
};

template <typename R>
__host__ __device__ __forceinline__ cx<R> mkc(R a, R b) {
  cx<R> c;
  c.x = a;
  c.y = b;
  return c;
}
template <typename R>
__host__ __device__ __forceinline__ cx<R> operator+(cx<R> a, cx<R> b) { return mkc<R>(a.x + b.x, a.y + b.y); }
template <typename R>
__host__ __device__ __forceinline__ cx<R> operator-(cx<R> a, cx<R> b) { return mkc<R>(a.x - b.x, a.y - b.y); }
template <typename R>
__host__ __device__ __forceinline__ cx<R> operator*(cx<R> a, cx<R> b) {
  return mkc<R>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename R>
__host__ __device__ __forceinline__ cx<R> operator*(R s, cx<R> a) { return mkc<R>(s * a.x, s * a.y); }
template <typename R>
__host__ __device__ __forceinline__ cx<R> conjc(cx<R> a) { return mkc<R>(a.x, -a.y); }
// multiply by (dir * i): dir = +1 -> i*a, dir = -1 -> -i*a
template <int DIR, typename R>
__host__ __device__ __forceinline__ cx<R> mul_i(cx<R> a) {
  return DIR > 0 ? mkc<R>(-a.y, a.x) : mkc<R>(a.y, -a.x);
}
// i * a
template <typename R>
__host__ __device__ __forceinline__ cx<R> ione(cx<R> a) { return mkc<R>(-a.y, a.x); }
// pointwise product of two packed-real values (Array_real_mult: re*re, im*im)
template <typename R>
__host__ __device__ __forceinline__ cx<R> rmul(cx<R> a, cx<R> b) { return mkc<R>(a.x * b.x, a.y * b.y); }

template <typename Rd, typename Rs>
__host__ __device__ __forceinline__ cx<Rd> cvt(cx<Rs> a) { return mkc<Rd>((Rd)a.x, (Rd)a.y); }

// FP32 complex arithmetic on the packed two-wide FP32 instructions of sm_100 (__fadd2_rn,
// __fmul2_rn: per component the same rounding as the scalar operation), one instruction per
// complex add, subtract, scaling or pointwise product instead of two.
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 1000) && !defined(TG_NO_F32X2)
__device__ __forceinline__ float2 f2(cx<float> a) { return make_float2(a.x, a.y); }
__device__ __forceinline__ cx<float> c2(float2 a) { return mkc<float>(a.x, a.y); }
__device__ __forceinline__ cx<float> operator+(cx<float> a, cx<float> b) { return c2(__fadd2_rn(f2(a), f2(b))); }
__device__ __forceinline__ cx<float> operator-(cx<float> a, cx<float> b) {
  return c2(__fadd2_rn(f2(a), make_float2(-b.x, -b.y)));
}
__device__ __forceinline__ cx<float> operator*(float s, cx<float> a) { return c2(__fmul2_rn(make_float2(s, s), f2(a))); }
__device__ __forceinline__ cx<float> rmul(cx<float> a, cx<float> b) { return c2(__fmul2_rn(f2(a), f2(b))); }
#endif

// Which FFT indices of an axis of length L are stored: [0, lo) and [L - hi, L), in that order,
// as rows 0 .. lo+hi-1.  A full axis has lo = L, hi = 0.
struct AxisMap {
  int L, lo, hi;
};

__host__ __device__ __forceinline__ int amap_row(const AxisMap& m, int n) {
  if (n < m.lo) return n;
  int off = m.L - m.hi;
  if (n >= off) return n - off + m.lo;
  return -1;
}
__host__ __device__ __forceinline__ int amap_index(const AxisMap& m, int r) {
  return r < m.lo ? r : r - m.lo + (m.L - m.hi);
}
__host__ __device__ __forceinline__ int amap_count(const AxisMap& m) { return m.lo + m.hi; }

// v of every active lane into row[bin], the same sum whatever the warp's timing: the lanes of a
// bin (__match_any_sync) add their values in lane order and the lowest of them adds the total to
// the warp's own row
__device__ __forceinline__ void warp_bin_add(double* row, int bin, double v, bool active) {
  const int lane = threadIdx.x & 31;
  const unsigned peers = __match_any_sync(0xffffffffu, active ? bin : -1 - lane);
  double sum = 0;
  for (unsigned m = peers; m; m &= m - 1) sum += __shfl_sync(peers, v, __ffs(m) - 1);
  if (active && lane == __ffs(peers) - 1) row[bin] += sum;
}

}  // namespace tg
