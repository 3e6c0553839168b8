// Fused z-pass for N3 = 256 (M = N3/2 = 128) with eight lanes per row.
//
// A warp transforms four rows at once; the eight lanes p = 0..7 of a row each hold 16 values,
// so a length-128 FFT is two register DFTs joined by one exchange between the eight lanes:
//
//   inverse (c2r, sign +), n = 16 q + r, r = 2 p + b, m = m1 + 8 m2:
//     load X[n], X[M - n] and pre-twiddle  Z'[q, b] = alpha X[n] + beta conj(X[M - n])
//     DFT8 over q (registers, one per b)              -> A[m1; r]
//     twiddle W128^(r m1)
//     exchange: lane p' takes m1 = p' from every lane  (seven shuffle rounds of two values)
//     DFT16 over r as DFT4 x DFT4 with a middle twiddle -> z[p' + 8 m2]
//   forward (r2c, sign -): the adjoint network in reverse order, then the r2c post-twiddle
//     X[k] = alpha' Zf[k] + beta' conj(Zf[M - k]) with the partner fetched by one shuffle.
//
// The exchange moves values with a uniform register index and a lane-dependent source: the
// sender's DFT8 outputs are kept rotated by its lane (slot t holds m1 = p + t), which is a phase
// W8^(p q) on the DFT8 inputs.  That phase is built into the DFT8's own stages (decimation in
// frequency: W8^(4 p q) = (-1)^p at the first stage, a sign folded into a fused multiply-add;
// W8^(2 p q) = i^p at the second, a swap and signs; W8^p at the last, one multiply by a per-lane
// constant).  The receiver's slots are rotated too, which is a phase W8^(p' m2) on the DFT16
// outputs: with m2 = k0 + 4 k1 its W8^(p' k0) part is folded into the middle twiddle and the
// rest is a sign (-1)^(p' k1).  That sign is left on the real-space values: every product
// multiplies two values of the same lane and register, so the signs cancel; the forward network
// takes it back with its first DFT4 (a fused multiply-add by +-1 where a plain add stood).
// The c2r pre-twiddle and the r2c post-twiddle use h = exp(+i pi n / M) = W16^q g_b with
// g_b = W256^(2 p + b) a per-lane constant and W16^q a compile-time factor, so only the DFT
// twiddles W128^(r m1) are read from the shared-memory table (a 16-byte read per lane costs the
// same shared-memory bandwidth whether or not lanes share its address).  Relative to the 32-lane
// network (k_z_prod_net128) each value crosses lanes once per transform instead of 2.5 times.
// Index maps and factors follow a CPU emulation checked against an FFT.
//
// Real-space values of the first three inputs are parked in warp-private shared memory (each
// lane reads back only its own slots); a fourth to sixth input (the scalar, or z- of MHD) is
// transformed into registers and multiplied with the parked fields at once.
//
// PRUNE: at most 96 stored entries on input and output (the 2/3-dealiased rows): inputs
// 96 .. 127 are zero, so slots q >= 6 have no X[n] term and q <= 1 no X[M - n] term, and
// outputs 96 .. 128 are not computed.
#pragma once

#include "tg_fft.cuh"

namespace tg {

// entries of the per-lane coefficient table, each [entry][8 lanes]: the DFT twiddles
// W128^(r m1) of slot (t, b) (entry 2 t + b), the middle twiddles of the DFT16 (entry 4 sl + k0),
// g_0, g_1 and W8^p; then, for the table form of the pre- and post-twiddles (slot 2 q + b):
// alpha = (1 + i h) phi, beta = (1 - i h) phi, alpha' = (1 - i conj h) conj(phi) / 2 and
// beta' = (1 + i conj h) phi(M - n) / 2 with phi = W8^(p q) the lane phase of the slot and
// phi(M - n) that of the slot holding (M - n) mod M
constexpr int kOctTw2 = 0, kOctMid = 16, kOctG = 32, kOctW8 = 34;
constexpr int kOctAlpha = 36, kOctBeta = 52, kOctAlphaF = 68, kOctBetaF = 84;
constexpr int kOctEntries = 100;

template <typename R>
__device__ __forceinline__ cx<R> cmac(cx<R> acc, cx<R> a, cx<R> b) {  // acc + a b
  return mkc<R>(fma(a.x, b.x, fma(-a.y, b.y, acc.x)), fma(a.x, b.y, fma(a.y, b.x, acc.y)));
}
template <typename R>
__device__ __forceinline__ cx<R> cmul_conjb(cx<R> a, cx<R> b) {  // a conj(b)
  return mkc<R>(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -(a.x * b.y)));
}

// physics layouts of the fused products (the solver's ProdPairs, tg_ctx.cu):
//   0 fluid   inputs u1 u2 u3 (parked); products u1u1 u2u2 u3u3 u1u2 u2u3 u3u1
//   1 MHD     inputs z+1..3 (parked), z-1..3 (registers); PA = {0,1,2,0,3,1,4,2,5},
//             PB = {3,4,5,4,1,5,2,3,0}: each product pairs one z+ with one z-
//   2 scalar  inputs u1 u2 u3 (parked), theta (registers); products as fluid, then u_i theta
template <int PHYS>
struct OctLayout {
  static constexpr int nin = PHYS == 1 ? 6 : (PHYS == 2 ? 4 : 3);
  static constexpr int npark = 3;
};
// MHD: the three products of register input z-(3 + i), j-th of them: product index and the
// parked z+ it takes (nibble 3 i + j of each constant)
constexpr unsigned long long kOctMhdQ = 0x852631740ull;    // {0,4,7}, {1,3,6}, {2,5,8}
constexpr unsigned long long kOctMhdA = 0x012201210ull;    // {0,1,2}, {1,0,2}, {2,1,0}

// i^k a with k in 0..3 given as a swap flag and two signs: k = 0 (x, y), 1 (-y, x), 2 (-x, -y),
// 3 (y, -x); the signs are applied by the caller's fused multiply-adds
template <typename Rw>
struct IPow {
  bool swap;
  Rw c0, c1;
  __device__ __forceinline__ void set(int k) {
    k &= 3;
    swap = (k & 1) != 0;
    c0 = (k == 1 || k == 2) ? (Rw)-1 : (Rw)1;
    c1 = (k == 2 || k == 3) ? (Rw)-1 : (Rw)1;
  }
};

template <typename Rw, bool TABLE>
struct OctLane {
  const cx<Rw>* tab;  // shared-memory table [kOctEntries][8]
  int p, base;        // lane within the row, first lane of the row's octet
  Rw sg;              // (-1)^p
  Rw hs;              // half the output scale of the forward transforms
  Rw sc;              // output scale of the forward transforms
  IPow<Rw> ipi, ipf;  // i^p (inverse) and i^-p (forward)
  cx<Rw> w8;          // W8^p
  cx<Rw> g[2];        // W256^(2 p + b)
  cx<Rw> mid_r[12];   // middle twiddles of the DFT16, (sl, k0) with k0 >= 1
  __device__ __forceinline__ cx<Rw> mid(int sl, int k0) const { return mid_r[sl * 3 + k0 - 1]; }
  // TABLE: the pre- and post-twiddles (with the lane phases folded in) come from the table, for
  // the FP32 fluid form, whose limit is instruction issue (the table form takes fewer
  // instructions); otherwise they are computed (FP64 is limited by shared-memory bandwidth and
  // latency at two warps per scheduler; the FP32 forms with a register input would spill)
  static constexpr bool kTablePre = TABLE;

  __device__ __forceinline__ cx<Rw> t(int e) const { return tab[e * 8 + p]; }

  // a + i^k b and a - i^k b (k of ip)
  __device__ __forceinline__ void bfly_ip(cx<Rw>& a, cx<Rw>& b, const IPow<Rw>& ip) const {
    const Rw bx = ip.swap ? b.y : b.x, by = ip.swap ? b.x : b.y;
    const Rw c0 = ip.c0, c1 = ip.c1;
    const cx<Rw> s = mkc<Rw>(fma(c0, bx, a.x), fma(c1, by, a.y));
    b = mkc<Rw>(fma(-c0, bx, a.x), fma(-c1, by, a.y));
    a = s;
  }

  // out[t] = sum_q v[q] W8^(p q) W8^(q t) (sign +): decimation in frequency with the lane phase
  // split over the stages; v is overwritten by out in natural order
  __device__ __forceinline__ void dft8_rot_inv(cx<Rw> (&v)[8]) const {
    cx<Rw> y[8];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const cx<Rw> a = v[q], b = v[q + 4];
      y[q] = mkc<Rw>(fma(sg, b.x, a.x), fma(sg, b.y, a.y));
      y[q + 4] = twc<+1, 0, 8, Rw>(mkc<Rw>(fma(-sg, b.x, a.x), fma(-sg, b.y, a.y)));
      if (q == 1) y[q + 4] = twc<+1, 1, 8, Rw>(y[q + 4]);
      if (q == 2) y[q + 4] = twc<+1, 2, 8, Rw>(y[q + 4]);
      if (q == 3) y[q + 4] = twc<+1, 3, 8, Rw>(y[q + 4]);
    }
#pragma unroll
    for (int h = 0; h < 8; h += 4) {
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        cx<Rw> a = y[h + q], b = y[h + q + 2];
        bfly_ip(a, b, ipi);
        y[h + q] = a;
        y[h + q + 2] = (q == 1) ? mul_i<+1>(b) : b;
      }
    }
    cx<Rw> o[8];
#pragma unroll
    for (int h = 0; h < 8; h += 2) {
      const cx<Rw> a = y[h], b = y[h + 1] * w8;
      o[h] = a + b;
      o[h + 1] = a - b;
    }
    // bit-reversed output order of the three radix-2 stages
    v[0] = o[0]; v[4] = o[1]; v[2] = o[2]; v[6] = o[3];
    v[1] = o[4]; v[5] = o[5]; v[3] = o[6]; v[7] = o[7];
  }

  // adjoint: out[q] = sum_t u[t] W8^(-q (t + p)) (decimation in time, stages reversed)
  __device__ __forceinline__ void dft8_rot_fwd(cx<Rw> (&u)[8]) const {
    cx<Rw> x[8] = {u[0], u[4], u[2], u[6], u[1], u[5], u[3], u[7]};
    cx<Rw> z[8];
#pragma unroll
    for (int h = 0; h < 8; h += 2) {
      const cx<Rw> a = x[h], b = x[h + 1];
      z[h] = a + b;
      z[h + 1] = cmul_conjb(a - b, w8);
    }
#pragma unroll
    for (int h = 0; h < 8; h += 4) {
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const cx<Rw> a = z[h + q], b = (q == 1) ? mul_i<-1>(z[h + q + 2]) : z[h + q + 2];
        // (a + b, i^-p (a - b)): the second as a swap of (a - b) with signs
        const cx<Rw> d = a - b;
        z[h + q] = a + b;
        const Rw dx = ipf.swap ? d.y : d.x, dy = ipf.swap ? d.x : d.y;
        z[h + q + 2] = mkc<Rw>(ipf.c0 * dx, ipf.c1 * dy);
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      cx<Rw> b = z[q + 4];
      if (q == 1) b = twc<-1, 1, 8, Rw>(b);
      if (q == 2) b = twc<-1, 2, 8, Rw>(b);
      if (q == 3) b = twc<-1, 3, 8, Rw>(b);
      const cx<Rw> a = z[q];
      u[q] = a + b;
      u[q + 4] = mkc<Rw>(fma(-sg, b.x, sg * a.x), fma(-sg, b.y, sg * a.y));
    }
  }

  // slot sigma' = 2t - b (mod 16) of the DFT16 input, from the exchanged DFT8 outputs
  __device__ __forceinline__ void dft16_inv(cx<Rw> (&u)[2][8], cx<Rw> (&o)[16]) const {
    cx<Rw> x[16];
#pragma unroll
    for (int s = 0; s < 16; ++s) x[s] = (s & 1) ? u[1][((s + 1) >> 1) & 7] : u[0][s >> 1];
    cx<Rw> C[4][4];
#pragma unroll
    for (int sl = 0; sl < 4; ++sl) {
      cx<Rw> w[4] = {x[sl], x[sl + 4], x[sl + 8], x[sl + 12]};
      DFT<4, -1, Rw>::run(w);
      C[sl][0] = w[0];
#pragma unroll
      for (int k0 = 1; k0 < 4; ++k0) C[sl][k0] = w[k0] * mid(sl, k0);
    }
#pragma unroll
    for (int k0 = 0; k0 < 4; ++k0) {
      cx<Rw> w[4] = {C[0][k0], C[1][k0], C[2][k0], C[3][k0]};
      DFT<4, -1, Rw>::run(w);
#pragma unroll
      for (int k1 = 0; k1 < 4; ++k1) o[k0 + 4 * k1] = w[k1];
    }
  }

  // adjoint of dft16_inv with the sign (-1)^(p k1) of the inputs taken back
  __device__ __forceinline__ void dft16_fwd(const cx<Rw> (&o)[16], cx<Rw> (&u)[2][8]) const {
    cx<Rw> C[4][4];
#pragma unroll
    for (int k0 = 0; k0 < 4; ++k0) {
      // DFT4 (+) over k1 of (y0, s y1, y2, s y3)
      const cx<Rw> y0 = o[k0], y1 = o[k0 + 4], y2 = o[k0 + 8], y3 = o[k0 + 12];
      const cx<Rw> t0 = y0 + y2, t1 = y0 - y2, t2 = y1 + y3, t3 = y1 - y3;
      // t3 rotated by +i: (-t3.y, t3.x)
      C[0][k0] = mkc<Rw>(fma(sg, t2.x, t0.x), fma(sg, t2.y, t0.y));
      C[2][k0] = mkc<Rw>(fma(-sg, t2.x, t0.x), fma(-sg, t2.y, t0.y));
      C[1][k0] = mkc<Rw>(fma(-sg, t3.y, t1.x), fma(sg, t3.x, t1.y));
      C[3][k0] = mkc<Rw>(fma(sg, t3.y, t1.x), fma(-sg, t3.x, t1.y));
    }
    cx<Rw> x[16];
#pragma unroll
    for (int sl = 0; sl < 4; ++sl) {
      cx<Rw> w[4];
      w[0] = C[sl][0];
#pragma unroll
      for (int k0 = 1; k0 < 4; ++k0) w[k0] = cmul_conjb(C[sl][k0], mid(sl, k0));
      DFT<4, +1, Rw>::run(w);
#pragma unroll
      for (int sh = 0; sh < 4; ++sh) x[sl + 4 * sh] = w[sh];
    }
#pragma unroll
    for (int s = 0; s < 16; ++s) {
      if (s & 1) u[1][((s + 1) >> 1) & 7] = x[s];
      else u[0][s >> 1] = x[s];
    }
  }

  // exchange of the inverse: round t, lane p' takes slot t of lane p' - t
  __device__ __forceinline__ void exchange_inv(cx<Rw> (&u)[2][8]) const {
#pragma unroll
    for (int t = 1; t < 8; ++t) {
      const int src = base | ((p - t) & 7);
      u[0][t] = shfl_c(u[0][t], src);
      u[1][t] = shfl_c(u[1][t], src);
    }
  }
  // its adjoint: lane p takes slot t of lane p + t
  __device__ __forceinline__ void exchange_fwd(cx<Rw> (&u)[2][8]) const {
#pragma unroll
    for (int t = 1; t < 8; ++t) {
      const int src = base | ((p + t) & 7);
      u[0][t] = shfl_c(u[0][t], src);
      u[1][t] = shfl_c(u[1][t], src);
    }
  }

  // c2r pre-twiddle of slot (q, b): (xa + conj xb) + i h (xa - conj xb), h = W16^q g_b;
  // HAVE_A / HAVE_B: whether the X[n] / X[M - n] term exists
  template <int Q, int B, bool HAVE_A, bool HAVE_B>
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
    const cx<Rw> u = twc<+1, Q, 16, Rw>(g[B] * d);
    return mkc<Rw>(s.x - u.y, s.y + u.x);
  }
  // r2c post-twiddle: hs [(y + conj yp) - i e (y - conj yp)], e = conj(h)
  template <int Q, int B>
  __device__ __forceinline__ cx<Rw> post(cx<Rw> y, cx<Rw> yp) const {
    const cx<Rw> s = mkc<Rw>(y.x + yp.x, y.y - yp.y);
    const cx<Rw> d = mkc<Rw>(y.x - yp.x, y.y + yp.y);
    const cx<Rw> u = twc<-1, Q, 16, Rw>(cmul_conjb(d, g[B]));
    return mkc<Rw>(hs * (s.x + u.y), hs * (s.y - u.x));
  }

  // c2r of one row: X (row base, nin stored entries; null: an idle row) -> o (real-space values
  // of positions m = p + 8 (k0 + 4 k1) in slot k0 + 4 k1, times (-1)^(p k1))
  template <typename Ri, bool PRUNE>
  __device__ __forceinline__ void inverse(const cx<Ri>* X, int nin, cx<Rw> (&o)[16]) const {
    constexpr int M = 128;
    cx<Rw> u[2][8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const int n = 16 * q + 2 * p + b;
        cx<Rw> xa = mkc<Rw>(0, 0), xb = mkc<Rw>(0, 0);
        if (!PRUNE || q <= 5) {
          if (X && n < nin) xa = cvt<Rw>(X[n]);
          if (q == 0 && b == 0 && p == 0) xa.y = 0;  // imaginary part of X[0] ignored (c2r)
        }
        if (!PRUNE || q >= 2) {
          if (X && M - n < nin) xb = cvt<Rw>(X[M - n]);
          if (q == 0 && b == 0 && p == 0) xb.y = 0;  // X[M]: imaginary part ignored
        }
        cx<Rw> v;
        if constexpr (kTablePre) {
          v = mkc<Rw>(0, 0);
          if (!PRUNE || q <= 5) v = t(kOctAlpha + 2 * q + b) * xa;
          if (!PRUNE || q >= 2) v = cmac(v, t(kOctBeta + 2 * q + b), conjc(xb));
          u[b][q] = v;
          continue;
        }
#define TG_OCT_PRE(QQ, BB)                                                           \
  if (q == QQ && b == BB) {                                                          \
    if (PRUNE && QQ <= 1) v = pre<QQ, BB, true, false>(xa, xb);                      \
    else if (PRUNE && QQ >= 6) v = pre<QQ, BB, false, true>(xa, xb);                 \
    else v = pre<QQ, BB, true, true>(xa, xb);                                        \
  }
        TG_OCT_PRE(0, 0) TG_OCT_PRE(0, 1) TG_OCT_PRE(1, 0) TG_OCT_PRE(1, 1)
        TG_OCT_PRE(2, 0) TG_OCT_PRE(2, 1) TG_OCT_PRE(3, 0) TG_OCT_PRE(3, 1)
        TG_OCT_PRE(4, 0) TG_OCT_PRE(4, 1) TG_OCT_PRE(5, 0) TG_OCT_PRE(5, 1)
        TG_OCT_PRE(6, 0) TG_OCT_PRE(6, 1) TG_OCT_PRE(7, 0) TG_OCT_PRE(7, 1)
#undef TG_OCT_PRE
        u[b][q] = v;
      }
    }
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      if constexpr (kTablePre) DFT<8, +1, Rw>::run(u[b]);
      else dft8_rot_inv(u[b]);
#pragma unroll
      for (int tt = 0; tt < 8; ++tt) u[b][tt] = u[b][tt] * t(kOctTw2 + 2 * tt + b);
    }
    exchange_inv(u);
    dft16_inv(u, o);
  }

  // r2c of one row of real-space values o (same layout, true values), scaled; writes entries
  // [0, nout) of Y and zeros [nout, nfill); Y null: an idle row (the shuffles still run)
  template <typename Ro, bool PRUNE>
  __device__ __forceinline__ void forward(const cx<Rw> (&o)[16], cx<Ro>* Y, int nout, int nfill) const {
    constexpr int M = 128;
    cx<Rw> u[2][8];
    dft16_fwd(o, u);
    exchange_fwd(u);
#pragma unroll
    for (int b = 0; b < 2; ++b) {
#pragma unroll
      for (int tt = 0; tt < 8; ++tt) u[b][tt] = cmul_conjb(u[b][tt], t(kOctTw2 + 2 * tt + b));
      if constexpr (kTablePre) DFT<8, -1, Rw>::run(u[b]);
      else dft8_rot_fwd(u[b]);
    }
    const int src0 = base | ((8 - p) & 7), src1 = base | (7 - p);
    constexpr int QMAX = PRUNE ? 6 : 8;
#pragma unroll
    for (int q = 0; q < QMAX; ++q) {
      // partners of n = 16 q + 2 p + b: M - n at (q2 = 7 - q, lane 8 - p, b = 0) or, on lane 0,
      // its own slot (8 - q) mod 8; (q2 = 7 - q, lane 7 - p, b = 1)
      cx<Rw> z0 = shfl_c(u[0][7 - q], src0);
      if (p == 0) z0 = u[0][(8 - q) & 7];
      const cx<Rw> z1 = shfl_c(u[1][7 - q], src1);
      cx<Rw> X0, X1;
      if constexpr (kTablePre) {
        X0 = cmac(t(kOctAlphaF + 2 * q) * u[0][q], t(kOctBetaF + 2 * q), conjc(z0));
        X1 = cmac(t(kOctAlphaF + 2 * q + 1) * u[1][q], t(kOctBetaF + 2 * q + 1), conjc(z1));
      }
#define TG_OCT_POST(QQ)                    \
  if (!kTablePre && q == QQ) {             \
    X0 = post<QQ, 0>(u[0][QQ], z0);        \
    X1 = post<QQ, 1>(u[1][QQ], z1);        \
  }
      TG_OCT_POST(0) TG_OCT_POST(1) TG_OCT_POST(2) TG_OCT_POST(3)
      TG_OCT_POST(4) TG_OCT_POST(5) TG_OCT_POST(6) TG_OCT_POST(7)
#undef TG_OCT_POST
      const int n = 16 * q + 2 * p;
      if (Y) {
        if (n + 1 < nout) {
          store_pair(Y + n, X0, X1);
        } else if (n < nout) {
          Y[n] = cvt<Ro>(X0);
        }
      }
    }
    if (Y) {
      if (!PRUNE && p == 0 && nout > M) {
        // X[M] = Re Zf[0] - Im Zf[0] (slot (0, 0) of lane 0)
        Y[M] = cvt<Ro>(mkc<Rw>(sc * (u[0][0].x - u[0][0].y), (Rw)0));
      }
      for (int k = nout + p; k < nfill; k += 8) Y[k] = mkc<Ro>(0, 0);
    }
  }

  // two consecutive output entries; one 32-byte store for complex double (row bases and even
  // entries lie on 32-byte boundaries, checked by the launcher)
  template <typename Ro>
  __device__ __forceinline__ static void store_pair(cx<Ro>* y, cx<Rw> a, cx<Rw> b) {
    if constexpr (sizeof(Ro) == 8) {
      asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(y), "d"((double)a.x), "d"((double)a.y),
                   "d"((double)b.x), "d"((double)b.y)
                   : "memory");
    } else {
      *reinterpret_cast<float4*>(y) = make_float4((float)a.x, (float)a.y, (float)b.x, (float)b.y);
    }
  }
};

// resident blocks per SM the kernel is built for (registers: FP64 255, FP32 128 for the fluid
// layout and 170 with a register input)
template <typename Rw, int PHYS>
struct OctOcc {
  static constexpr int v = sizeof(Rw) == 8 ? 2 : (PHYS == 0 ? 4 : 3);
};

template <typename Ri, typename Ro, typename Rw, int PHYS, bool PRUNE>
__global__ void __launch_bounds__(128, OctOcc<Rw, PHYS>::v) k_z_prod_oct(ZArgs a, PtrSet ps) {
  using Lay = OctLayout<PHYS>;
  constexpr int NP = Lay::npark;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<Rw>* tab = reinterpret_cast<cx<Rw>*>(smem_raw);
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  cx<Rw>* rs = tab + kOctEntries * 8 + (size_t)wib * NP * 16 * 32;
  const Rw sc = (Rw)a.scale;
  for (int i = threadIdx.x; i < kOctEntries * 8; i += blockDim.x) {
    cx<Rw> v = cvt<Rw>(a.oct[i]);
    const int e = i >> 3;
    if (e >= kOctAlphaF) v = sc * v;  // the output scale rides on the post factors
    tab[i] = v;
  }
  __syncthreads();
  OctLane<Rw, sizeof(Rw) == 4 && PHYS == 0> L;
  L.tab = tab;
  L.p = lane & 7;
  L.base = lane & ~7;
  L.sg = (L.p & 1) ? (Rw)-1 : (Rw)1;
  L.sc = sc;
  L.hs = (Rw)0.5 * sc;
  L.ipi.set(L.p);
  L.ipf.set(-L.p);
  L.w8 = tab[kOctW8 * 8 + L.p];
  L.g[0] = tab[kOctG * 8 + L.p];
  L.g[1] = tab[(kOctG + 1) * 8 + L.p];
#pragma unroll
  for (int sl = 0; sl < 4; ++sl)
#pragma unroll
    for (int k0 = 1; k0 < 4; ++k0) L.mid_r[sl * 3 + k0 - 1] = tab[(kOctMid + sl * 4 + k0) * 8 + L.p];
  const long long nquad = (a.nrows + 3) >> 2;
  for (long long quad = (long long)blockIdx.x * 4 + wib; quad < nquad; quad += (long long)gridDim.x * 4) {
    const long long row = quad * 4 + (lane >> 3);
    const bool live = row < a.nrows;
    // inverse of the parked inputs
#pragma unroll 1
    for (int c = 0; c < NP; ++c) {
      const cx<Ri>* X = live ? reinterpret_cast<const cx<Ri>*>(ps.src[c]) + row * a.ss : nullptr;
      cx<Rw> o[16];
      L.template inverse<Ri, PRUNE>(X, a.nin, o);
#pragma unroll
      for (int s = 0; s < 16; ++s) rs[(c * 16 + s) * 32 + lane] = o[s];
    }
    if constexpr (PHYS == 0 || PHYS == 2) {
      // products of two parked inputs
#pragma unroll 1
      for (int q = 0; q < 6; ++q) {
        const int pa = q < 3 ? q : q - 3, pb = q < 3 ? q : (q == 5 ? 0 : q - 2);
        cx<Rw> v[16];
#pragma unroll
        for (int s = 0; s < 16; ++s) {
          const cx<Rw> x = rs[(pa * 16 + s) * 32 + lane];
          v[s] = (pa == pb) ? rmul(x, x) : rmul(x, rs[(pb * 16 + s) * 32 + lane]);
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
        cx<Rw> w[16];
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
          cx<Rw> v[16];
#pragma unroll
          for (int s = 0; s < 16; ++s) v[s] = rmul(rs[(pa * 16 + s) * 32 + lane], w[s]);
          cx<Ro>* Y = live ? reinterpret_cast<cx<Ro>*>(ps.dst[q]) + row * a.ds : nullptr;
          L.template forward<Ro, PRUNE>(v, Y, a.nout, a.nfill);
        }
      }
    }
  }
}

}  // namespace tg
