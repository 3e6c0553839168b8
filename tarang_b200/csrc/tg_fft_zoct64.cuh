// Fused z-pass for N3 = 128 (M = N3/2 = 64) with eight lanes per row: the scheme of
// k_z_prod_oct (tg_fft_zoct.cuh) with one subsequence per lane instead of two.
//
//   inverse (c2r, sign +), n = 8 q + p, m = m1 + 8 m2:
//     load X[n], X[M - n] and pre-twiddle  Z'[q] = alpha X[n] + beta conj(X[M - n])
//     DFT8 over q (registers)                           -> A[m1; p]
//     twiddle W64^(p m1)
//     exchange: lane p' takes m1 = p' from every lane   (seven shuffle rounds of one value)
//     DFT8 over p as DFT4 x DFT2 with a middle twiddle   -> z[p' + 8 m2]
//   forward (r2c, sign -): the adjoint network in reverse order, then the r2c post-twiddle
//     X[k] = alpha' Zf[k] + beta' conj(Zf[M - k]) with the partner fetched by one shuffle.
//
// The sender keeps its DFT8 outputs rotated by its lane (slot t holds m1 = p + t), a phase
// W8^(p q) on the DFT8 inputs that the DFT8's own stages absorb (OctLane::dft8_rot_inv).  The
// receiver's slot t holds p = p' - t, so its DFT8 over p is a DFT8 of sign - over t followed by
// the phase W8^(p' m2) on output m2 = k0 + 4 k1: with the input split t = 2 tA + tB, the
// W8^(p' k0) part rides on the middle twiddle W8^(-tB k0) and the rest is the sign (-1)^(p' k1),
// left on the real-space values (every product multiplies two values of the same lane and slot,
// so it cancels; the forward network takes it back with its first stage).  The pre- and
// post-twiddles use h = exp(+i pi n / M) = W16^q g, g = W128^p.  Index maps and factors follow a
// CPU emulation checked against an FFT.
//
// PRUNE: at most 48 stored entries on input and output (the 2/3-dealiased rows, 42 of 64 for
// N3 = 128): inputs 48 .. 63 are zero, so slots q >= 6 have no X[n] term and q <= 1 no X[M - n]
// term, and outputs 48 .. 64 are not computed.
#pragma once

#include "tg_fft_zoct.cuh"

namespace tg {

// per-lane coefficient table, each [entry][8 lanes]: the DFT twiddles W64^(p m1) of slot t
// (m1 = p + t), the middle twiddles W8^(-tB k0) W8^(p k0) (entry 4 tB + k0), g = W128^p, W8^p;
// then, for the table form of the pre- and post-twiddles (slot q): alpha = (1 + i h) phi,
// beta = (1 - i h) phi, alpha' = (1 - i conj h) conj(phi) / 2, beta' = (1 + i conj h) phi(M - n) / 2
// with phi = W8^(p q) and phi(M - n) the phase of the slot holding (M - n) mod M
constexpr int kO64Tw = 0, kO64Mid = 8, kO64G = 16, kO64W8 = 17;
constexpr int kO64Alpha = 18, kO64Beta = 26, kO64AlphaF = 34, kO64BetaF = 42;
constexpr int kO64Entries = 50;

template <typename Rw, bool TABLE>
struct OctLane64 : OctLane<Rw, TABLE> {
  using Base = OctLane<Rw, TABLE>;
  using Base::p;
  using Base::base;
  using Base::sg;
  using Base::hs;
  using Base::sc;
  using Base::tab;
  cx<Rw> g1;         // W128^p
  cx<Rw> mid64[6];   // middle twiddles (tB, k0), k0 >= 1
  __device__ __forceinline__ cx<Rw> mid(int tB, int k0) const { return mid64[tB * 3 + k0 - 1]; }
  __device__ __forceinline__ cx<Rw> t(int e) const { return tab[e * 8 + p]; }

  // receiver: DFT8 of sign - over the rotated slots as DFT4 (over tA) x DFT2 (over tB), the
  // output phase folded into the middle twiddles; o[k0 + 4 k1] = value at m2 = k0 + 4 k1 times
  // (-1)^(p k1)
  __device__ __forceinline__ void dft8x_inv(const cx<Rw> (&u)[8], cx<Rw> (&o)[8]) const {
    cx<Rw> C[2][4];
#pragma unroll
    for (int tB = 0; tB < 2; ++tB) {
      cx<Rw> w[4] = {u[tB], u[tB + 2], u[tB + 4], u[tB + 6]};
      DFT<4, -1, Rw>::run(w);
      C[tB][0] = w[0];
#pragma unroll
      for (int k0 = 1; k0 < 4; ++k0) C[tB][k0] = w[k0] * mid(tB, k0);
    }
#pragma unroll
    for (int k0 = 0; k0 < 4; ++k0) {
      o[k0] = C[0][k0] + C[1][k0];
      o[k0 + 4] = C[0][k0] - C[1][k0];
    }
  }
  // adjoint of dft8x_inv with the sign (-1)^(p k1) of the inputs taken back
  __device__ __forceinline__ void dft8x_fwd(const cx<Rw> (&o)[8], cx<Rw> (&u)[8]) const {
    cx<Rw> C[2][4];
#pragma unroll
    for (int k0 = 0; k0 < 4; ++k0) {
      const cx<Rw> a = o[k0], b = o[k0 + 4];
      C[0][k0] = mkc<Rw>(fma(sg, b.x, a.x), fma(sg, b.y, a.y));
      C[1][k0] = mkc<Rw>(fma(-sg, b.x, a.x), fma(-sg, b.y, a.y));
    }
#pragma unroll
    for (int tB = 0; tB < 2; ++tB) {
      cx<Rw> w[4];
      w[0] = C[tB][0];
#pragma unroll
      for (int k0 = 1; k0 < 4; ++k0) w[k0] = cmul_conjb(C[tB][k0], mid(tB, k0));
      DFT<4, +1, Rw>::run(w);
#pragma unroll
      for (int tA = 0; tA < 4; ++tA) u[2 * tA + tB] = w[tA];
    }
  }

  // exchange of the inverse: round t, lane p' takes slot t of lane p' - t; and its adjoint
  __device__ __forceinline__ void exchange_inv(cx<Rw> (&u)[8]) const {
#pragma unroll
    for (int tt = 1; tt < 8; ++tt) u[tt] = shfl_c(u[tt], base | ((p - tt) & 7));
  }
  __device__ __forceinline__ void exchange_fwd(cx<Rw> (&u)[8]) const {
#pragma unroll
    for (int tt = 1; tt < 8; ++tt) u[tt] = shfl_c(u[tt], base | ((p + tt) & 7));
  }

  // c2r pre-twiddle of slot q: (xa + conj xb) + i h (xa - conj xb), h = W16^q g1
  template <int Q, bool HAVE_A, bool HAVE_B>
  __device__ __forceinline__ cx<Rw> pre(cx<Rw> xa, cx<Rw> xb) const {
    cx<Rw> s, d;
    if (HAVE_A && HAVE_B) {
      s = mkc<Rw>(xa.x + xb.x, xa.y - xb.y);
      d = mkc<Rw>(xa.x - xb.x, xa.y + xb.y);
    } else if (HAVE_A) {
      s = d = xa;
    } else {
      s = conjc(xb);
      d = mkc<Rw>(-xb.x, xb.y);
    }
    const cx<Rw> u = twc<+1, Q, 16, Rw>(g1 * d);
    return mkc<Rw>(s.x - u.y, s.y + u.x);
  }
  // r2c post-twiddle: hs [(y + conj yp) - i e (y - conj yp)], e = conj(h)
  template <int Q>
  __device__ __forceinline__ cx<Rw> post(cx<Rw> y, cx<Rw> yp) const {
    const cx<Rw> s = mkc<Rw>(y.x + yp.x, y.y - yp.y);
    const cx<Rw> d = mkc<Rw>(y.x - yp.x, y.y + yp.y);
    const cx<Rw> u = twc<-1, Q, 16, Rw>(cmul_conjb(d, g1));
    return mkc<Rw>(hs * (s.x + u.y), hs * (s.y - u.x));
  }

  // c2r of one row: X (row base, nin stored entries; null: an idle row) -> o (real-space values
  // of positions m = p + 8 (k0 + 4 k1) in slot k0 + 4 k1, times (-1)^(p k1))
  template <typename Ri, bool PRUNE>
  __device__ __forceinline__ void inverse(const cx<Ri>* X, int nin, cx<Rw> (&o)[8]) const {
    constexpr int M = 64;
    cx<Rw> u[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int n = 8 * q + p;
      cx<Rw> xa = mkc<Rw>(0, 0), xb = mkc<Rw>(0, 0);
      if (!PRUNE || q <= 5) {
        if (X && n < nin) xa = cvt<Rw>(X[n]);
        if (q == 0 && p == 0) xa.y = 0;  // imaginary part of X[0] ignored (c2r)
      }
      if (!PRUNE || q >= 2) {
        if (X && M - n < nin) xb = cvt<Rw>(X[M - n]);
        if (q == 0 && p == 0) xb.y = 0;  // X[M]: imaginary part ignored
      }
      cx<Rw> v;
      if constexpr (Base::kTablePre) {
        v = mkc<Rw>(0, 0);
        if (!PRUNE || q <= 5) v = t(kO64Alpha + q) * xa;
        if (!PRUNE || q >= 2) v = cmac(v, t(kO64Beta + q), conjc(xb));
        u[q] = v;
        continue;
      }
#define TG_O64_PRE(QQ)                                                   \
  if (q == QQ) {                                                         \
    if (PRUNE && QQ <= 1) v = pre<QQ, true, false>(xa, xb);              \
    else if (PRUNE && QQ >= 6) v = pre<QQ, false, true>(xa, xb);         \
    else v = pre<QQ, true, true>(xa, xb);                                \
  }
      TG_O64_PRE(0) TG_O64_PRE(1) TG_O64_PRE(2) TG_O64_PRE(3)
      TG_O64_PRE(4) TG_O64_PRE(5) TG_O64_PRE(6) TG_O64_PRE(7)
#undef TG_O64_PRE
      u[q] = v;
    }
    if constexpr (Base::kTablePre) DFT<8, +1, Rw>::run(u);
    else this->dft8_rot_inv(u);
#pragma unroll
    for (int tt = 0; tt < 8; ++tt) u[tt] = u[tt] * t(kO64Tw + tt);
    exchange_inv(u);
    dft8x_inv(u, o);
  }

  // r2c of one row of real-space values o (same layout, true values), scaled; writes entries
  // [0, nout) of Y and zeros [nout, nfill); Y null: an idle row (the shuffles still run)
  template <typename Ro, bool PRUNE>
  __device__ __forceinline__ void forward(const cx<Rw> (&o)[8], cx<Ro>* Y, int nout, int nfill) const {
    constexpr int M = 64;
    cx<Rw> u[8];
    dft8x_fwd(o, u);
    exchange_fwd(u);
#pragma unroll
    for (int tt = 0; tt < 8; ++tt) u[tt] = cmul_conjb(u[tt], t(kO64Tw + tt));
    if constexpr (Base::kTablePre) DFT<8, -1, Rw>::run(u);
    else this->dft8_rot_fwd(u);
    const int src0 = base | ((8 - p) & 7);
    constexpr int QMAX = PRUNE ? 6 : 8;
#pragma unroll
    for (int q = 0; q < QMAX; ++q) {
      // partner of n = 8 q + p: M - n at (q2 = 7 - q, lane 8 - p) or, on lane 0, its own slot
      // (8 - q) mod 8
      cx<Rw> z = shfl_c(u[7 - q], src0);
      if (p == 0) z = u[(8 - q) & 7];
      cx<Rw> X;
      if constexpr (Base::kTablePre) X = cmac(t(kO64AlphaF + q) * u[q], t(kO64BetaF + q), conjc(z));
#define TG_O64_POST(QQ) \
  if (!Base::kTablePre && q == QQ) X = post<QQ>(u[QQ], z);
      TG_O64_POST(0) TG_O64_POST(1) TG_O64_POST(2) TG_O64_POST(3)
      TG_O64_POST(4) TG_O64_POST(5) TG_O64_POST(6) TG_O64_POST(7)
#undef TG_O64_POST
      const int n = 8 * q + p;
      if (Y && n < nout) Y[n] = cvt<Ro>(X);
    }
    if (Y) {
      if (!PRUNE && p == 0 && nout > M) {
        // X[M] = Re Zf[0] - Im Zf[0] (slot 0 of lane 0)
        Y[M] = cvt<Ro>(mkc<Rw>(sc * (u[0].x - u[0].y), (Rw)0));
      }
      for (int k = nout + p; k < nfill; k += 8) Y[k] = mkc<Ro>(0, 0);
    }
  }
};

// resident blocks per SM the kernel is built for
template <typename Rw, int PHYS>
struct Oct64Occ {
  static constexpr int v = sizeof(Rw) == 8 ? 3 : 4;
};

template <typename Ri, typename Ro, typename Rw, int PHYS, bool PRUNE>
__global__ void __launch_bounds__(128, Oct64Occ<Rw, PHYS>::v) k_z_prod_oct64(ZArgs a, PtrSet ps) {
  using Lay = OctLayout<PHYS>;
  constexpr int NP = Lay::npark;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<Rw>* tab = reinterpret_cast<cx<Rw>*>(smem_raw);
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  cx<Rw>* rs = tab + kO64Entries * 8 + (size_t)wib * NP * 8 * 32;
  const Rw sc = (Rw)a.scale;
  for (int i = threadIdx.x; i < kO64Entries * 8; i += blockDim.x) {
    cx<Rw> v = cvt<Rw>(a.oct[i]);
    const int e = i >> 3;
    if (e >= kO64AlphaF) v = sc * v;  // the output scale rides on the post factors
    tab[i] = v;
  }
  __syncthreads();
  OctLane64<Rw, sizeof(Rw) == 4 && PHYS == 0> L;
  L.tab = tab;
  L.p = lane & 7;
  L.base = lane & ~7;
  L.sg = (L.p & 1) ? (Rw)-1 : (Rw)1;
  L.sc = sc;
  L.hs = (Rw)0.5 * sc;
  L.ipi.set(L.p);
  L.ipf.set(-L.p);
  L.w8 = tab[kO64W8 * 8 + L.p];
  L.g1 = tab[kO64G * 8 + L.p];
#pragma unroll
  for (int tB = 0; tB < 2; ++tB)
#pragma unroll
    for (int k0 = 1; k0 < 4; ++k0) L.mid64[tB * 3 + k0 - 1] = tab[(kO64Mid + tB * 4 + k0) * 8 + L.p];
  const long long nquad = (a.nrows + 3) >> 2;
  for (long long quad = (long long)blockIdx.x * 4 + wib; quad < nquad; quad += (long long)gridDim.x * 4) {
    const long long row = quad * 4 + (lane >> 3);
    const bool live = row < a.nrows;
    // inverse of the parked inputs
#pragma unroll 1
    for (int c = 0; c < NP; ++c) {
      const cx<Ri>* X = live ? reinterpret_cast<const cx<Ri>*>(ps.src[c]) + row * a.ss : nullptr;
      cx<Rw> o[8];
      L.template inverse<Ri, PRUNE>(X, a.nin, o);
#pragma unroll
      for (int s = 0; s < 8; ++s) rs[(c * 8 + s) * 32 + lane] = o[s];
    }
    if constexpr (PHYS == 0 || PHYS == 2) {
      // products of two parked inputs
#pragma unroll 1
      for (int q = 0; q < 6; ++q) {
        const int pa = q < 3 ? q : q - 3, pb = q < 3 ? q : (q == 5 ? 0 : q - 2);
        cx<Rw> v[8];
#pragma unroll
        for (int s = 0; s < 8; ++s) {
          const cx<Rw> x = rs[(pa * 8 + s) * 32 + lane];
          v[s] = (pa == pb) ? rmul(x, x) : rmul(x, rs[(pb * 8 + s) * 32 + lane]);
        }
        cx<Ro>* Y = live ? reinterpret_cast<cx<Ro>*>(ps.dst[q]) + row * a.ds : nullptr;
        L.template forward<Ro, PRUNE>(v, Y, a.nout, a.nfill);
      }
    }
    if constexpr (PHYS == 1 || PHYS == 2) {
      // register inputs, each multiplied with the three parked inputs
#pragma unroll 1
      for (int c = 3; c < Lay::nin; ++c) {
        const cx<Ri>* X = live ? reinterpret_cast<const cx<Ri>*>(ps.src[c]) + row * a.ss : nullptr;
        cx<Rw> w[8];
        L.template inverse<Ri, PRUNE>(X, a.nin, w);
#pragma unroll 1
        for (int j = 0; j < 3; ++j) {
          // PHYS 2: product 6 + j = u_j theta; PHYS 1: the three products of z-(c) in order
          int q = 6 + j, pa = j;
          if constexpr (PHYS == 1) {
            const int sh = 4 * (3 * (c - 3) + j);
            q = (int)((kOctMhdQ >> sh) & 15);
            pa = (int)((kOctMhdA >> sh) & 15);
          }
          cx<Rw> v[8];
#pragma unroll
          for (int s = 0; s < 8; ++s) v[s] = rmul(rs[(pa * 8 + s) * 32 + lane], w[s]);
          cx<Ro>* Y = live ? reinterpret_cast<cx<Ro>*>(ps.dst[q]) + row * a.ds : nullptr;
          L.template forward<Ro, PRUNE>(v, Y, a.nout, a.nfill);
        }
      }
    }
  }
}

}  // namespace tg
