// Dispatch of the strided-axis c2c kernels (x- and y-passes).
#include "tg_fft_launch.h"

namespace tg {

namespace {

template <typename Ri, typename Ro, typename Rw, int R1, int R2, int DIR>
cudaError_t run_axis_fast(const AxisLaunch& l, cudaStream_t s) {
  constexpr int L = R1 * R2;
  constexpr int W = 256 / R1;
  const size_t smem = (size_t)(L + (size_t)L * W) * sizeof(cx<Rw>);
  auto kern = k_axis_c2c<Ri, Ro, Rw, R1, R2, DIR>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  dim3 grid((l.a.ncols + W - 1) / W, l.nbatch, l.nfields);
  kern<<<grid, 256, smem, s>>>(l.a, l.ps);
  return cudaGetLastError();
}

template <typename Ri, typename Ro, typename Rw, int DIR>
cudaError_t run_axis_dft(const AxisLaunch& l, cudaStream_t s) {
  const size_t smem = (size_t)(l.L + (size_t)l.L * 8) * sizeof(cx<Rw>);
  auto kern = k_axis_dft<Ri, Ro, Rw, DIR>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((l.a.ncols + 7) / 8, l.nbatch, l.nfields);
  kern<<<grid, 256, smem, s>>>(l.a, l.ps, l.L);
  return cudaGetLastError();
}

template <typename Ri, typename Ro, typename Rw, int DIR>
cudaError_t run_axis_dir(const AxisLaunch& l, cudaStream_t s) {
  switch (l.L) {
    case 2: return run_axis_fast<Ri, Ro, Rw, 2, 1, DIR>(l, s);
    case 4: return run_axis_fast<Ri, Ro, Rw, 2, 2, DIR>(l, s);
    case 8: return run_axis_fast<Ri, Ro, Rw, 4, 2, DIR>(l, s);
    case 16: return run_axis_fast<Ri, Ro, Rw, 4, 4, DIR>(l, s);
    case 32: return run_axis_fast<Ri, Ro, Rw, 8, 4, DIR>(l, s);
    case 64: return run_axis_fast<Ri, Ro, Rw, 8, 8, DIR>(l, s);
    case 128: return run_axis_fast<Ri, Ro, Rw, 16, 8, DIR>(l, s);
    case 256: return run_axis_fast<Ri, Ro, Rw, 16, 16, DIR>(l, s);
    case 512: return run_axis_fast<Ri, Ro, Rw, 32, 16, DIR>(l, s);
    default:
      if (l.L < 1 || l.L > 2048) return cudaErrorInvalidValue;
      return run_axis_dft<Ri, Ro, Rw, DIR>(l, s);
  }
}

template <typename Ri, typename Ro, typename Rw>
cudaError_t run_axis_prec(const AxisLaunch& l, cudaStream_t s) {
  return l.dir < 0 ? run_axis_dir<Ri, Ro, Rw, -1>(l, s) : run_axis_dir<Ri, Ro, Rw, +1>(l, s);
}

template <typename Ri, typename Ro, typename Rw>
cudaError_t run_r2r(const AxisLaunch& l, const R2RArgs& r, int N, cudaStream_t s) {
  const int nin = amap_count(l.a.in);
  const size_t smem = (size_t)(4 * N + (size_t)nin * 32) * sizeof(cx<Rw>);
  auto kern = k_axis_r2r<Ri, Ro, Rw>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((l.a.ncols + 31) / 32, l.nbatch, l.nfields);
  kern<<<grid, 256, smem, s>>>(l.a, l.ps, r, N);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_r2r(const AxisLaunch& l, const R2RArgs& r, cudaStream_t s) {
  if (l.a.ncols <= 0 || l.nbatch <= 0 || l.nfields <= 0) return cudaSuccess;
  if (l.nbatch > 65535 || l.nfields > kMaxPtr || l.L < 2 || l.L > 1024) return cudaErrorInvalidValue;
  const int N = l.L;
  if (l.pwork == F64) {
    if (l.pin == F64 && l.pout == F64) return run_r2r<double, double, double>(l, r, N, s);
    return cudaErrorInvalidValue;
  }
  if (l.pin == F64 && l.pout == F64) return run_r2r<double, double, float>(l, r, N, s);
  if (l.pin == F64 && l.pout == F32) return run_r2r<double, float, float>(l, r, N, s);
  if (l.pin == F32 && l.pout == F32) return run_r2r<float, float, float>(l, r, N, s);
  if (l.pin == F32 && l.pout == F64) return run_r2r<float, double, float>(l, r, N, s);
  return cudaErrorInvalidValue;
}

cudaError_t launch_axis(const AxisLaunch& l, cudaStream_t s) {
  if (l.a.ncols <= 0 || l.nbatch <= 0 || l.nfields <= 0) return cudaSuccess;
  if (l.nbatch > 65535 || l.nfields > kMaxPtr) return cudaErrorInvalidValue;
  if (l.pwork == F64) {
    if (l.pin == F64 && l.pout == F64) return run_axis_prec<double, double, double>(l, s);
    return cudaErrorInvalidValue;
  }
  if (l.pin == F64 && l.pout == F64) return run_axis_prec<double, double, float>(l, s);
  if (l.pin == F64 && l.pout == F32) return run_axis_prec<double, float, float>(l, s);
  if (l.pin == F32 && l.pout == F32) return run_axis_prec<float, float, float>(l, s);
  if (l.pin == F32 && l.pout == F64) return run_axis_prec<float, double, float>(l, s);
  return cudaErrorInvalidValue;
}

}  // namespace tg
