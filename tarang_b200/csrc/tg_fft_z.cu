// Dispatch of the z-pass (contiguous axis) c2r / r2c kernels and of the fused product z-pass.
#include <cstdint>
#include <cstdlib>

#include <cmath>

#include "tg_fft_launch.h"
#include "tg_fft_zoct.cuh"
#include "tg_fft_zoct64.cuh"

namespace tg {

namespace {

template <typename Ri, typename Ro, typename Rw, int R1, int R2>
cudaError_t run_z_fast(const ZLaunch& l, cudaStream_t s) {
  constexpr int M = R1 * R2;
  constexpr int ROWS = 256 / R1;
  if (l.kind == 0) {
    const size_t smem = (size_t)(3 * M + 256 * (R2 + 1)) * sizeof(cx<Rw>);
    auto kern = k_z_c2r<Ri, Ro, Rw, R1, R2>;
    static bool attr = false;
    if (!attr) {
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      attr = true;
    }
    dim3 grid((unsigned)((l.a.nrows + ROWS - 1) / ROWS), 1, l.nfields);
    kern<<<grid, 256, smem, s>>>(l.a, l.ps);
  } else {
    const size_t smem = (size_t)(3 * M + 256 * (R2 + 1) + ROWS * M) * sizeof(cx<Rw>);
    auto kern = k_z_r2c<Ri, Ro, Rw, R1, R2>;
    static bool attr = false;
    if (!attr) {
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      attr = true;
    }
    dim3 grid((unsigned)((l.a.nrows + ROWS - 1) / ROWS), 1, l.nfields);
    kern<<<grid, 256, smem, s>>>(l.a, l.ps);
  }
  return cudaGetLastError();
}

template <typename Ri, typename Ro, typename Rw>
cudaError_t run_z_dft(const ZLaunch& l, cudaStream_t s) {
  const int M = l.M;
  if (l.a.nrows > 2147483647LL) return cudaErrorInvalidValue;
  dim3 grid((unsigned)l.a.nrows, 1, l.nfields);
  if (l.kind == 0) {
    const size_t smem = (size_t)(2 * M + M + 1) * sizeof(cx<Rw>);
    auto kern = k_z_c2r_dft<Ri, Ro, Rw>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, 128, smem, s>>>(l.a, l.ps, M);
  } else {
    const size_t smem = (size_t)(2 * M) * sizeof(cx<Rw>) + (size_t)(2 * M) * sizeof(Rw);
    auto kern = k_z_r2c_dft<Ri, Ro, Rw>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, 128, smem, s>>>(l.a, l.ps, M);
  }
  return cudaGetLastError();
}

template <typename Ri, typename Ro, typename Rw>
cudaError_t run_z_prec(const ZLaunch& l, cudaStream_t s) {
  switch (l.M) {
    case 2: return run_z_fast<Ri, Ro, Rw, 2, 1>(l, s);
    case 4: return run_z_fast<Ri, Ro, Rw, 2, 2>(l, s);
    case 8: return run_z_fast<Ri, Ro, Rw, 4, 2>(l, s);
    case 16: return run_z_fast<Ri, Ro, Rw, 4, 4>(l, s);
    case 32: return run_z_fast<Ri, Ro, Rw, 8, 4>(l, s);
    case 64: return run_z_fast<Ri, Ro, Rw, 8, 8>(l, s);
    case 128: return run_z_fast<Ri, Ro, Rw, 16, 8>(l, s);
    case 256: return run_z_fast<Ri, Ro, Rw, 16, 16>(l, s);
    default:
      if (l.M < 1 || l.M > 4096) return cudaErrorInvalidValue;
      return run_z_dft<Ri, Ro, Rw>(l, s);
  }
}

// ---------------------------------------------------------------- fused product z-pass
template <typename Ri, typename Ro, typename Rw, int R1, int R2, int NIN, int NPROD>
cudaError_t run_zprod_fast(const ZProdLaunch& l, cudaStream_t s) {
  constexpr int M = R1 * R2;
  constexpr int TPB = (M >= 128) ? 128 : 256;
  constexpr int ROWS = TPB / R1;
  constexpr int EXA = R2 + 1, EXB = R1 + 1;
  constexpr int EXS = (R1 * EXA > R2 * EXB) ? R1 * EXA : R2 * EXB;
  const size_t smem = (size_t)(3 * M + ROWS * EXS + (size_t)ROWS * M * (1 + NIN)) * sizeof(cx<Rw>);
  auto kern = k_z_prod<Ri, Ro, Rw, R1, R2, NIN, NPROD>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  dim3 grid((unsigned)((l.a.nrows + ROWS - 1) / ROWS), 1, 1);
  kern<<<grid, TPB, smem, s>>>(l.a, l.ps, l.pp);
  return cudaGetLastError();
}

template <typename Ri, typename Ro, typename Rw, int E, int NIN, int NPROD>
cudaError_t run_zprod_warp(const ZProdLaunch& l, cudaStream_t s) {
  constexpr int WPB = 4;
  const size_t smem = (size_t)WPB * NIN * E * 32 * sizeof(cx<Rw>);
  auto kern = k_z_prod_warp<Ri, Ro, Rw, E, NIN, NPROD, WPB>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  long long blocks = (l.a.nrows + WPB - 1) / WPB;
  if (blocks > 148LL * 32) blocks = 148LL * 32;
  kern<<<(unsigned)blocks, 32 * WPB, smem, s>>>(l.a, l.ps, l.pp);
  return cudaGetLastError();
}

// M = 128: the transposed lane network (k_z_prod_net128) unless TG_ZPASS_NET=0 selects the
// five-stage shuffle network of k_z_prod_warp (both compute the same transform)
bool zpass_net_enabled() {
  static int v = -1;
  if (v < 0) {
    const char* e = std::getenv("TG_ZPASS_NET");
    v = (e && e[0] == '0') ? 0 : 1;
  }
  return v == 1;
}

template <typename Ri, typename Ro, typename Rw, int NIN, int NPROD, int PF>
cudaError_t run_zprod_net128_pf(const ZProdLaunch& l, int np, cudaStream_t s) {
  constexpr int WPB = 4;
  const size_t smem =
      (size_t)WPB * ((size_t)NIN * 4 * 32 * sizeof(cx<Rw>) + (PF ? (size_t)NIN * np * sizeof(cx<Ri>) : 0));
  auto kern = k_z_prod_net128<Ri, Ro, Rw, NIN, NPROD, WPB, PF>;
  static size_t attr = 0;
  if (smem > attr) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr = smem;
  }
  long long blocks = (l.a.nrows + WPB - 1) / WPB;
  if (blocks > 148LL * 32) blocks = 148LL * 32;
  kern<<<(unsigned)blocks, 32 * WPB, smem, s>>>(l.a, l.ps, l.pp, np);
  return cudaGetLastError();
}

// The prefetching form when its buffers fit beside the register-bound occupancy (at most four
// inputs) and every input row starts on a 16-byte boundary.
template <typename Ri, typename Ro, typename Rw, int NIN, int NPROD>
cudaError_t run_zprod_net128(const ZProdLaunch& l, cudaStream_t s) {
  bool pf = NIN <= 4 && sizeof(Ri) == sizeof(Rw) && l.a.nin <= 128 &&
            ((size_t)l.a.ss * sizeof(cx<Ri>)) % 16 == 0 &&
            ((size_t)l.a.ss * sizeof(cx<Ri>)) >= (((size_t)l.a.nin * sizeof(cx<Ri>) + 15) / 16) * 16;
  for (int c = 0; c < NIN && pf; ++c) pf = (reinterpret_cast<uintptr_t>(l.ps.src[c]) % 16) == 0;
  // entries per input buffer: nin rounded up to whole 16-byte chunks
  const int per16 = (int)(16 / sizeof(cx<Ri>));
  const int np = ((l.a.nin + per16 - 1) / per16) * per16;
  if (pf) return run_zprod_net128_pf<Ri, Ro, Rw, NIN, NPROD, 1>(l, np, s);
  return run_zprod_net128_pf<Ri, Ro, Rw, NIN, NPROD, 0>(l, 0, s);
}

// M = 128 and M = 64: the eight-lane networks (k_z_prod_oct, k_z_prod_oct64) unless TG_ZPASS_OCT=0
bool zpass_oct_enabled() {
  static int v = -1;
  if (v < 0) {
    const char* e = std::getenv("TG_ZPASS_OCT");
    v = (e && e[0] == '0') ? 0 : 1;
  }
  return v == 1;
}

// the physics layout k_z_prod_oct hard-codes (OctLayout), if the launch's product pairs are it
template <int NIN, int NPROD>
int oct_phys(const ProdPairs& pp) {
  static const signed char F_A[6] = {0, 1, 2, 0, 1, 2}, F_B[6] = {0, 1, 2, 1, 2, 0};
  static const signed char M_A[9] = {0, 1, 2, 0, 3, 1, 4, 2, 5}, M_B[9] = {3, 4, 5, 4, 1, 5, 2, 3, 0};
  static const signed char S_A[9] = {0, 1, 2, 0, 1, 2, 0, 1, 2}, S_B[9] = {0, 1, 2, 1, 2, 0, 3, 3, 3};
  const signed char *A, *B;
  int ph;
  if (NIN == 3 && NPROD == 6) {
    A = F_A, B = F_B, ph = 0;
  } else if (NIN == 6 && NPROD == 9) {
    A = M_A, B = M_B, ph = 1;
  } else if (NIN == 4 && NPROD == 9) {
    A = S_A, B = S_B, ph = 2;
  } else {
    return -1;
  }
  for (int q = 0; q < NPROD; ++q)
    if (pp.a[q] != A[q] || pp.b[q] != B[q]) return -1;
  return ph;
}

template <typename Ri, typename Ro, typename Rw, int PHYS, bool PRUNE>
cudaError_t run_zprod_oct(const ZProdLaunch& l, cudaStream_t s) {
  constexpr int WPB = 4;
  const size_t smem = sizeof(cx<Rw>) * ((size_t)kOctEntries * 8 + (size_t)WPB * OctLayout<PHYS>::npark * 16 * 32);
  auto kern = k_z_prod_oct<Ri, Ro, Rw, PHYS, PRUNE>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const long long nquad = (l.a.nrows + 3) / 4;
  long long blocks = (nquad + WPB - 1) / WPB;
  const long long resident = 148LL * OctOcc<Rw, PHYS>::v;
  if (blocks > resident) blocks = resident;
  kern<<<(unsigned)blocks, 32 * WPB, smem, s>>>(l.a, l.ps);
  return cudaGetLastError();
}

template <typename Ri, typename Ro, typename Rw, int NIN, int NPROD>
cudaError_t run_zprod_oct_any(const ZProdLaunch& l, int ph, cudaStream_t s) {
  const bool prune = l.a.nin <= 96 && l.a.nout <= 96;
  if (ph == 0) return prune ? run_zprod_oct<Ri, Ro, Rw, 0, true>(l, s) : run_zprod_oct<Ri, Ro, Rw, 0, false>(l, s);
  if (ph == 1) return prune ? run_zprod_oct<Ri, Ro, Rw, 1, true>(l, s) : run_zprod_oct<Ri, Ro, Rw, 1, false>(l, s);
  return prune ? run_zprod_oct<Ri, Ro, Rw, 2, true>(l, s) : run_zprod_oct<Ri, Ro, Rw, 2, false>(l, s);
}

template <typename Ri, typename Ro, typename Rw, int PHYS, bool PRUNE>
cudaError_t run_zprod_oct64(const ZProdLaunch& l, cudaStream_t s) {
  constexpr int WPB = 4;
  const size_t smem = sizeof(cx<Rw>) * ((size_t)kO64Entries * 8 + (size_t)WPB * OctLayout<PHYS>::npark * 8 * 32);
  auto kern = k_z_prod_oct64<Ri, Ro, Rw, PHYS, PRUNE>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const long long nquad = (l.a.nrows + 3) / 4;
  long long blocks = (nquad + WPB - 1) / WPB;
  const long long resident = 148LL * Oct64Occ<Rw, PHYS>::v;
  if (blocks > resident) blocks = resident;
  kern<<<(unsigned)blocks, 32 * WPB, smem, s>>>(l.a, l.ps);
  return cudaGetLastError();
}

template <typename Ri, typename Ro, typename Rw, int NIN, int NPROD>
cudaError_t run_zprod_oct64_any(const ZProdLaunch& l, int ph, cudaStream_t s) {
  const bool prune = l.a.nin <= 48 && l.a.nout <= 48;
  if (ph == 0) return prune ? run_zprod_oct64<Ri, Ro, Rw, 0, true>(l, s) : run_zprod_oct64<Ri, Ro, Rw, 0, false>(l, s);
  if (ph == 1) return prune ? run_zprod_oct64<Ri, Ro, Rw, 1, true>(l, s) : run_zprod_oct64<Ri, Ro, Rw, 1, false>(l, s);
  return prune ? run_zprod_oct64<Ri, Ro, Rw, 2, true>(l, s) : run_zprod_oct64<Ri, Ro, Rw, 2, false>(l, s);
}

template <typename Ri, typename Ro, typename Rw, int NIN, int NPROD>
cudaError_t run_zprod_m(const ZProdLaunch& l, cudaStream_t s) {
  if (l.M == 64 && l.a.oct && zpass_oct_enabled() && l.a.nin <= 65 && l.a.nout <= 65) {
    const int ph = oct_phys<NIN, NPROD>(l.pp);
    if (ph >= 0) return run_zprod_oct64_any<Ri, Ro, Rw, NIN, NPROD>(l, ph, s);
  }
  if (l.M == 128 && l.a.oct && zpass_oct_enabled() && l.a.nin <= 129 && l.a.nout <= 129) {
    // the paired output stores need even row strides and 2-entry-aligned product buffers
    bool aligned = (l.a.ds % 2) == 0;
    for (int q = 0; q < NPROD && aligned; ++q)
      aligned = (reinterpret_cast<uintptr_t>(l.ps.dst[q]) % (2 * sizeof(cx<Ro>))) == 0;
    const int ph = aligned ? oct_phys<NIN, NPROD>(l.pp) : -1;
    if (ph >= 0) return run_zprod_oct_any<Ri, Ro, Rw, NIN, NPROD>(l, ph, s);
  }
  if (l.M == 128 && zpass_net_enabled()) return run_zprod_net128<Ri, Ro, Rw, NIN, NPROD>(l, s);
  switch (l.M) {
    case 4: return run_zprod_fast<Ri, Ro, Rw, 2, 2, NIN, NPROD>(l, s);
    case 8: return run_zprod_fast<Ri, Ro, Rw, 4, 2, NIN, NPROD>(l, s);
    case 16: return run_zprod_fast<Ri, Ro, Rw, 4, 4, NIN, NPROD>(l, s);
    case 32: return run_zprod_warp<Ri, Ro, Rw, 1, NIN, NPROD>(l, s);
    case 64: return run_zprod_warp<Ri, Ro, Rw, 2, NIN, NPROD>(l, s);
    case 128: return run_zprod_warp<Ri, Ro, Rw, 4, NIN, NPROD>(l, s);
    case 256: return run_zprod_warp<Ri, Ro, Rw, 8, NIN, NPROD>(l, s);
    default: return cudaErrorInvalidValue;
  }
}

template <typename Ri, typename Ro, typename Rw>
cudaError_t run_zprod_prec(const ZProdLaunch& l, cudaStream_t s) {
  if (l.nin == 3 && l.nprod == 6) return run_zprod_m<Ri, Ro, Rw, 3, 6>(l, s);
  if (l.nin == 6 && l.nprod == 9) return run_zprod_m<Ri, Ro, Rw, 6, 9>(l, s);
  if (l.nin == 4 && l.nprod == 9) return run_zprod_m<Ri, Ro, Rw, 4, 9>(l, s);
  return cudaErrorInvalidValue;
}

}  // namespace

// entries [e][p] of k_z_prod_oct64 (tg_fft_zoct64.cuh), M = 64; W_N^e = exp(+2 pi i e / N)
void zoct64_table(cx<double>* out) {
  const long double two_pi = 6.283185307179586476925286766559005768L;
  auto put = [&](int e, int p, long double N, long double k) {
    out[e * 8 + p].x = (double)cosl(two_pi * k / N);
    out[e * 8 + p].y = (double)sinl(two_pi * k / N);
  };
  auto set = [&](int e, int p, long double re, long double im) {
    out[e * 8 + p].x = (double)re;
    out[e * 8 + p].y = (double)im;
  };
  const int M = 64;
  for (int p = 0; p < 8; ++p) {
    for (int t = 0; t < 8; ++t) put(kO64Tw + t, p, (long double)M, p * ((p + t) & 7));
    // W8^(-tB k0) W8^(p k0)
    for (int tB = 0; tB < 2; ++tB)
      for (int k0 = 0; k0 < 4; ++k0) put(kO64Mid + 4 * tB + k0, p, 8.0L, (p - tB) * k0);
    put(kO64G, p, 2.0L * M, p);
    put(kO64W8, p, 8.0L, p);
    for (int q = 0; q < 8; ++q) {
      const int n = 8 * q + p;
      const long double hr = cosl(two_pi * n / (2.0L * M)), hi = sinl(two_pi * n / (2.0L * M));
      const long double fr = cosl(two_pi * (p * q) / 8.0L), fi = sinl(two_pi * (p * q) / 8.0L);
      // alpha = (1 + i h) phi, beta = (1 - i h) phi
      const long double ar = 1 - hi, ai = hr, br = 1 + hi, bi = -hr;
      set(kO64Alpha + q, p, ar * fr - ai * fi, ar * fi + ai * fr);
      set(kO64Beta + q, p, br * fr - bi * fi, br * fi + bi * fr);
      // e = conj(h); A = (1 - i e) / 2, B = (1 + i e) / 2; alpha' = A conj(phi), beta' = B phi(M - n)
      const long double er = hr, ei = -hi;
      const long double Ar = 0.5L * (1 + ei), Ai = -0.5L * er, Br = 0.5L * (1 - ei), Bi = 0.5L * er;
      set(kO64AlphaF + q, p, Ar * fr + Ai * fi, Ai * fr - Ar * fi);
      const int k2 = (M - n) % M, q2 = k2 / 8, p2 = k2 % 8;
      const long double gr = cosl(two_pi * (p2 * q2) / 8.0L), gi = sinl(two_pi * (p2 * q2) / 8.0L);
      set(kO64BetaF + q, p, Br * gr - Bi * gi, Br * gi + Bi * gr);
    }
  }
}

void zoct_table(int M, cx<double>* out) {
  for (int e = 0; e < kZoctTableLen; ++e) out[e].x = out[e].y = 0.0;
  if (M == 64) {
    zoct64_table(out);
    return;
  }
  // entries [e][p] of k_z_prod_oct (tg_fft_zoct.cuh), M = 128; W_N^e = exp(+2 pi i e / N)
  const long double two_pi = 6.283185307179586476925286766559005768L;
  auto put = [&](int e, int p, long double N, long double k) {
    out[e * 8 + p].x = (double)cosl(two_pi * k / N);
    out[e * 8 + p].y = (double)sinl(two_pi * k / N);
  };
  M = 128;
  for (int p = 0; p < 8; ++p) {
    for (int t = 0; t < 8; ++t)
      for (int b = 0; b < 2; ++b) put(kOctTw2 + 2 * t + b, p, (long double)M, (2 * p + b) * ((p + t) & 7));
    // W16^(-sl k0) W8^(p k0) = W16^(2 p k0 - sl k0)
    for (int sl = 0; sl < 4; ++sl)
      for (int k0 = 0; k0 < 4; ++k0) put(kOctMid + 4 * sl + k0, p, 16.0L, 2 * p * k0 - sl * k0);
    put(kOctG, p, 2.0L * M, 2 * p);
    put(kOctG + 1, p, 2.0L * M, 2 * p + 1);
    put(kOctW8, p, 8.0L, p);
    for (int q = 0; q < 8; ++q)
      for (int b = 0; b < 2; ++b) {
        const int n = 16 * q + 2 * p + b, slot = 2 * q + b;
        const long double hr = cosl(two_pi * n / (2.0L * M)), hi = sinl(two_pi * n / (2.0L * M));
        const long double fr = cosl(two_pi * (p * q) / 8.0L), fi = sinl(two_pi * (p * q) / 8.0L);
        auto set = [&](int e, long double re, long double im) {
          out[e * 8 + p].x = (double)re;
          out[e * 8 + p].y = (double)im;
        };
        // alpha = (1 + i h) phi, beta = (1 - i h) phi
        const long double ar = 1 - hi, ai = hr, br = 1 + hi, bi = -hr;
        set(kOctAlpha + slot, ar * fr - ai * fi, ar * fi + ai * fr);
        set(kOctBeta + slot, br * fr - bi * fi, br * fi + bi * fr);
        // e = conj(h); A = (1 - i e) / 2, B = (1 + i e) / 2; alpha' = A conj(phi), beta' = B phi(M - n)
        const long double er = hr, ei = -hi;
        const long double Ar = 0.5L * (1 + ei), Ai = -0.5L * er, Br = 0.5L * (1 - ei), Bi = 0.5L * er;
        set(kOctAlphaF + slot, Ar * fr + Ai * fi, Ai * fr - Ar * fi);
        const int k2 = (M - n) % M, q2 = k2 / 16, p2 = (k2 % 16) / 2;
        const long double gr = cosl(two_pi * (p2 * q2) / 8.0L), gi = sinl(two_pi * (p2 * q2) / 8.0L);
        set(kOctBetaF + slot, Br * gr - Bi * gi, Br * gi + Bi * gr);
      }
  }
}

cudaError_t launch_z(const ZLaunch& l, cudaStream_t s) {
  if (l.a.nrows <= 0 || l.nfields <= 0) return cudaSuccess;
  if (l.nfields > kMaxPtr) return cudaErrorInvalidValue;
  if (l.pwork == F64) {
    if (l.pin == F64 && l.pout == F64) return run_z_prec<double, double, double>(l, s);
    return cudaErrorInvalidValue;
  }
  if (l.pin == F64 && l.pout == F64) return run_z_prec<double, double, float>(l, s);
  if (l.pin == F64 && l.pout == F32) return run_z_prec<double, float, float>(l, s);
  if (l.pin == F32 && l.pout == F32) return run_z_prec<float, float, float>(l, s);
  if (l.pin == F32 && l.pout == F64) return run_z_prec<float, double, float>(l, s);
  return cudaErrorInvalidValue;
}

cudaError_t launch_zprod(const ZProdLaunch& l, cudaStream_t s) {
  if (l.a.nrows <= 0) return cudaSuccess;
  if (l.pwork == F64 && l.pin == F64 && l.pout == F64) return run_zprod_prec<double, double, double>(l, s);
  if (l.pwork == F32 && l.pin == F32 && l.pout == F32) return run_zprod_prec<float, float, float>(l, s);
  return cudaErrorInvalidValue;
}

}  // namespace tg
