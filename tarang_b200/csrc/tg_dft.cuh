// Register-resident small DFTs (radix 2, 4, 8, 16, 32) used as the butterflies of every
// FFT stage.  X[k] = sum_n x[n] exp(DIR * 2 pi i n k / R); DIR = -1 is FFTW_FORWARD,
// DIR = +1 is FFTW_BACKWARD (unnormalised).  Inputs and outputs are in natural order.
// All indices are compile-time constants after unrolling, so the arrays stay in registers.
#pragma once

#include "tg_common.cuh"

namespace tg {

// cos(pi m / 16) and sin(pi m / 16), m = 0..31: the 32nd roots of unity.
__host__ __device__ __forceinline__ double c32tab(int m) {
  switch (m & 31) {
    case 0: return 1.0;
    case 1: return 0.98078528040323044913;
    case 2: return 0.92387953251128675613;
    case 3: return 0.83146961230254523708;
    case 4: return 0.70710678118654752440;
    case 5: return 0.55557023301960222474;
    case 6: return 0.38268343236508977173;
    case 7: return 0.19509032201612826785;
    case 8: return 0.0;
    case 9: return -0.19509032201612826785;
    case 10: return -0.38268343236508977173;
    case 11: return -0.55557023301960222474;
    case 12: return -0.70710678118654752440;
    case 13: return -0.83146961230254523708;
    case 14: return -0.92387953251128675613;
    case 15: return -0.98078528040323044913;
    case 16: return -1.0;
    case 17: return -0.98078528040323044913;
    case 18: return -0.92387953251128675613;
    case 19: return -0.83146961230254523708;
    case 20: return -0.70710678118654752440;
    case 21: return -0.55557023301960222474;
    case 22: return -0.38268343236508977173;
    case 23: return -0.19509032201612826785;
    case 24: return 0.0;
    case 25: return 0.19509032201612826785;
    case 26: return 0.38268343236508977173;
    case 27: return 0.55557023301960222474;
    case 28: return 0.70710678118654752440;
    case 29: return 0.83146961230254523708;
    case 30: return 0.92387953251128675613;
    default: return 0.98078528040323044913;
  }
}
__host__ __device__ __forceinline__ double s32tab(int m) { return c32tab(m - 8); }

// a * exp(DIR * 2 pi i J / N) for N dividing 32; exact handling of the +-1, +-i cases.
template <int DIR, int J, int N, typename R>
__device__ __forceinline__ cx<R> twc(cx<R> a) {
  constexpr int m = ((J % N) * (32 / N)) & 31;
  if constexpr (m == 0) return a;
  else if constexpr (m == 8) return mul_i<DIR>(a);
  else if constexpr (m == 16) return mkc<R>(-a.x, -a.y);
  else if constexpr (m == 24) return mul_i<-DIR>(a);
  else {
    const R c = (R)c32tab(m);
    const R s = (R)(DIR * s32tab(m));
    return mkc<R>(a.x * c - a.y * s, a.x * s + a.y * c);
  }
}

template <int N, int DIR, typename R>
struct DFT;

template <int DIR, typename R>
struct DFT<1, DIR, R> {
  __device__ __forceinline__ static void run(cx<R>*) {}
};

template <int DIR, typename R>
struct DFT<2, DIR, R> {
  __device__ __forceinline__ static void run(cx<R>* x) {
    cx<R> a = x[0], b = x[1];
    x[0] = a + b;
    x[1] = a - b;
  }
};

template <int DIR, typename R>
struct DFT<4, DIR, R> {
  __device__ __forceinline__ static void run(cx<R>* x) {
    cx<R> t0 = x[0] + x[2];
    cx<R> t1 = x[0] - x[2];
    cx<R> t2 = x[1] + x[3];
    cx<R> t3 = mul_i<DIR>(x[1] - x[3]);
    x[0] = t0 + t2;
    x[2] = t0 - t2;
    x[1] = t1 + t3;
    x[3] = t1 - t3;
  }
};

// Two-factor composition N = A * B: n = B n1 + n2, k = k1 + A k2.
template <int A, int B, int DIR, typename R>
__device__ __forceinline__ void dft_ab(cx<R>* x) {
  cx<R> y[A * B];
#pragma unroll
  for (int n2 = 0; n2 < B; ++n2) {
    cx<R> t[A];
#pragma unroll
    for (int n1 = 0; n1 < A; ++n1) t[n1] = x[B * n1 + n2];
    DFT<A, DIR, R>::run(t);
    y[n2 + B * 0] = t[0];
#pragma unroll
    for (int k1 = 1; k1 < A; ++k1) {
      // twiddle exp(DIR 2 pi i n2 k1 / N)
      cx<R> v = t[k1];
      switch ((n2 * k1 * (32 / (A * B))) & 31) {
#define TG_TW_CASE(MM) \
  case MM: v = twc<DIR, MM, 32, R>(v); break;
        TG_TW_CASE(0) TG_TW_CASE(1) TG_TW_CASE(2) TG_TW_CASE(3) TG_TW_CASE(4) TG_TW_CASE(5)
        TG_TW_CASE(6) TG_TW_CASE(7) TG_TW_CASE(8) TG_TW_CASE(9) TG_TW_CASE(10) TG_TW_CASE(11)
        TG_TW_CASE(12) TG_TW_CASE(13) TG_TW_CASE(14) TG_TW_CASE(15) TG_TW_CASE(16) TG_TW_CASE(17)
        TG_TW_CASE(18) TG_TW_CASE(19) TG_TW_CASE(20) TG_TW_CASE(21) TG_TW_CASE(22) TG_TW_CASE(23)
        TG_TW_CASE(24) TG_TW_CASE(25) TG_TW_CASE(26) TG_TW_CASE(27) TG_TW_CASE(28) TG_TW_CASE(29)
        TG_TW_CASE(30) TG_TW_CASE(31)
#undef TG_TW_CASE
      }
      y[n2 + B * k1] = v;
    }
  }
#pragma unroll
  for (int k1 = 0; k1 < A; ++k1) {
    cx<R> t[B];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) t[n2] = y[n2 + B * k1];
    DFT<B, DIR, R>::run(t);
#pragma unroll
    for (int k2 = 0; k2 < B; ++k2) x[k1 + A * k2] = t[k2];
  }
}

template <int DIR, typename R>
struct DFT<8, DIR, R> {
  __device__ __forceinline__ static void run(cx<R>* x) { dft_ab<2, 4, DIR, R>(x); }
};
template <int DIR, typename R>
struct DFT<16, DIR, R> {
  __device__ __forceinline__ static void run(cx<R>* x) { dft_ab<4, 4, DIR, R>(x); }
};
template <int DIR, typename R>
struct DFT<32, DIR, R> {
  __device__ __forceinline__ static void run(cx<R>* x) { dft_ab<4, 8, DIR, R>(x); }
};

}  // namespace tg
