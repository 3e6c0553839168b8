// Dispatch of the z-pass (contiguous axis) c2r / r2c kernels and of the fused product z-pass.
#include <cstdint>
#include <cstdlib>

#include "tg_fft_launch.h"

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

template <typename Ri, typename Ro, typename Rw, int NIN, int NPROD>
cudaError_t run_zprod_m(const ZProdLaunch& l, cudaStream_t s) {
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
