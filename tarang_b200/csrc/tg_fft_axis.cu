// Dispatch of the strided-axis c2c kernels (x- and y-passes).
//
// Power-of-two lengths 16..256 whose stored input and kept output rows fit one TMA box (<= 256
// rows) run k_axis_tma: the block's column tile moves HBM -> shared memory and back as single
// tiled bulk tensor copies, so the threads spend no instructions on addresses or row maps of
// global memory.  Other lengths run the register-staged k_axis_c2c / k_axis_dft.  Both compute
// the same butterflies in the same order (equal results up to how the compiler contracts
// multiply-adds in each kernel).
#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "tg_fft_launch.h"
#include "tg_fft_tc.cuh"
#include "tg_tma.cuh"

namespace tg {

namespace {

// set by a TMA-staged block whose tile never arrived within the bounded wait
__device__ int g_axis_tma_timeout = 0;

constexpr int kTmaPolls = 1 << 20;

struct TmaSet {
  CUtensorMap src[kMaxPtr];
  CUtensorMap src2[kMaxPtr];
  CUtensorMap dst[kMaxPtr];
};

// One block: W columns (TmaW) of one batch of one field.  Tile rows in shared memory are
// row-major [row][W]; the same buffer holds the loaded input tile, then the transposed
// intermediate, then the output tile.
// Tile width of the TMA axis kernel: 8 columns (64 or 128 contiguous bytes per row), so the
// solver's column counts (kzp, a multiple of 8, and nky * kzp) split into whole tiles; the block
// has W * R1 threads (128 at L = 256).  (16-column FP32 tiles, 128-byte row segments at 256
// threads a block, measured no faster: 256^3 FP32-mixed step 1.85 ms against 1.81 ms.)
template <typename Rw>
struct TmaW {
  static constexpr int v = 8;
};
// resident blocks per SM the kernel is built for: 64 registers (FP32 arithmetic) or 80 (FP64)
template <typename Rw, int NT>
struct AxisOcc {
  static constexpr int v = (65536 / NT) / (sizeof(Rw) == 4 ? 64 : 80);
};

template <typename Ri, typename Ro, typename Rw, int R1, int R2, int DIR, bool COMB>
__global__ void __launch_bounds__(TmaW<Rw>::v * R1, AxisOcc<Rw, TmaW<Rw>::v * R1>::v)
    k_axis_tma(AxisArgs a, const __grid_constant__ TmaSet tm, int nin_rows, int nout_rows, unsigned tile_bytes) {
  constexpr int L = R1 * R2;
  constexpr int W = TmaW<Rw>::v;
  constexpr int NT = W * R1;
  constexpr int CEi = (int)(sizeof(cx<Ri>) / 8), CEo = (int)(sizeof(cx<Ro>) / 8);
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  uint64_t* bar = reinterpret_cast<uint64_t*>(base);
  int* ok_flag = reinterpret_cast<int*>(base + 8);
  cx<Rw>* tw = reinterpret_cast<cx<Rw>*>(base + 128);
  unsigned char* buf = base + 128 + ((L * sizeof(cx<Rw>) + 127) & ~(size_t)127);
  unsigned char* buf2 = buf + tile_bytes;
  const int tid = threadIdx.x;
  const int f = blockIdx.z, b = blockIdx.y, col0 = blockIdx.x * W;
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (tid == 0) {
    const unsigned in_bytes = (unsigned)(W * CEi * 8) * (unsigned)nin_rows;
    mbar_arrive_expect_tx(bar, COMB ? 2 * in_bytes : in_bytes);
    tma_load_3d(buf, &tm.src[f], col0 * CEi, 0, b, bar);
    if constexpr (COMB) tma_load_3d(buf2, &tm.src2[f], col0 * CEi, 0, b, bar);
  }
  for (int i = tid; i < L; i += NT) {
    cx<Rw> t = cvt<Rw>(a.tw[i]);
    if (DIR > 0) t.y = -t.y;
    tw[i] = t;
  }
  if (tid == 0) {
    const bool ok = mbar_wait_bounded(bar, 0, a.wait_short ? 0 : kTmaPolls);
    *ok_flag = ok ? 1 : 0;
    if (!ok) {
      atomicExch(a.wait_flag ? a.wait_flag : &g_axis_tma_timeout, 1);
      mbar_wait_bounded(bar, 0, kTmaPolls);  // let a late copy land before the block leaves
    }
  }
  __syncthreads();
  if (*ok_flag == 0) return;
  mbar_wait_bounded(bar, 0, 64);  // the phase has completed: acquire the copied tile
  const int w = tid % W;
  const int n2 = tid / W;
  cx<Rw> v[R1];
  if (n2 < R2) {
    const cx<Ri>* tin = reinterpret_cast<const cx<Ri>*>(buf);
    const cx<Ri>* tin2 = reinterpret_cast<const cx<Ri>*>(buf2);
    const int comb = COMB ? a.comb[f] : 0;
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) {
      const int r = amap_row(a.in, R2 * n1 + n2);
      v[n1] = mkc<Rw>(0, 0);
      if (r >= 0) {
        v[n1] = cvt<Rw>(tin[r * W + w]);
        if constexpr (COMB) {
          if (comb > 0) v[n1] = v[n1] + cvt<Rw>(tin2[r * W + w]);
          else if (comb < 0) v[n1] = v[n1] - cvt<Rw>(tin2[r * W + w]);
        }
      }
    }
    DFT<R1, DIR, Rw>::run(v);
  }
  __syncthreads();  // the input tile is consumed; its buffer takes the intermediate
  cx<Rw>* ex = reinterpret_cast<cx<Rw>*>(buf);
  if (n2 < R2) {
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) ex[(k1 * R2 + n2) * W + w] = v[k1] * tw[(n2 * k1) & (L - 1)];
  }
  __syncthreads();
  const int k1 = tid / W;
  cx<Rw> u[R2];
#pragma unroll
  for (int m = 0; m < R2; ++m) u[m] = ex[(k1 * R2 + m) * W + w];
  DFT<R2, DIR, Rw>::run(u);
  __syncthreads();  // the intermediate is consumed; the buffer takes the output tile
  cx<Ro>* tout = reinterpret_cast<cx<Ro>*>(buf);
  const Rw sc = (Rw)a.scale;
#pragma unroll
  for (int k2 = 0; k2 < R2; ++k2) {
    const int r = amap_row(a.out, k1 + R1 * k2);
    if (r >= 0) tout[r * W + w] = cvt<Ro>(sc * u[k2]);
  }
  fence_proxy_async_smem();
  __syncthreads();
  if (tid == 0) {
    tma_store_3d(&tm.dst[f], col0 * CEo, 0, b, buf);
    bulk_commit_group();
    bulk_wait_group_read0();
  }
}

bool axis_tma_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("TG_AXIS_TMA");
    return !(e && e[0] == '0');
  }();
  return on;
}

template <typename Ri, typename Ro, typename Rw, int R1, int R2, int DIR>
cudaError_t run_axis_tma(const AxisLaunch& l, cudaStream_t s, bool* used) {
  *used = false;
  constexpr int L = R1 * R2;
  constexpr int W = TmaW<Rw>::v;
  constexpr int NT = W * R1;
  constexpr int CEi = (int)(sizeof(cx<Ri>) / 8), CEo = (int)(sizeof(cx<Ro>) / 8);
  const int nin_rows = amap_count(l.a.in), nout_rows = amap_count(l.a.out);
  if (nin_rows < 1 || nin_rows > 256 || nout_rows < 1 || nout_rows > 256) return cudaSuccess;
  if (l.nbatch > 65535) return cudaSuccess;
  bool comb = false;
  for (int f = 0; f < l.nfields; ++f) comb = comb || (l.a.comb[f] != 0);
  TmaSet tm;  // host staging of the maps (copied into the launch parameters)
  std::memset(&tm, 0, sizeof(tm));
  for (int f = 0; f < l.nfields; ++f) {
    if (!tma_map_3d(&tm.src[f], l.ps.src[f], (unsigned long long)l.a.ncols * CEi, (unsigned long long)nin_rows,
                    (unsigned long long)l.nbatch, (unsigned long long)l.a.sr * sizeof(cx<Ri>),
                    (unsigned long long)l.a.sb * sizeof(cx<Ri>), W * CEi, nin_rows))
      return cudaSuccess;
    if (comb && l.a.comb[f] != 0 &&
        !tma_map_3d(&tm.src2[f], l.ps.src2[f], (unsigned long long)l.a.ncols * CEi, (unsigned long long)nin_rows,
                    (unsigned long long)l.nbatch, (unsigned long long)l.a.sr * sizeof(cx<Ri>),
                    (unsigned long long)l.a.sb * sizeof(cx<Ri>), W * CEi, nin_rows))
      return cudaSuccess;
    if (comb && l.a.comb[f] == 0) tm.src2[f] = tm.src[f];
    if (!tma_map_3d(&tm.dst[f], l.ps.dst[f], (unsigned long long)l.a.ncols * CEo, (unsigned long long)nout_rows,
                    (unsigned long long)l.nbatch, (unsigned long long)l.a.dr * sizeof(cx<Ro>),
                    (unsigned long long)l.a.db * sizeof(cx<Ro>), W * CEo, nout_rows))
      return cudaSuccess;
  }
  size_t tile = (size_t)W * nin_rows * sizeof(cx<Ri>);
  tile = tile > (size_t)W * L * sizeof(cx<Rw>) ? tile : (size_t)W * L * sizeof(cx<Rw>);
  tile = tile > (size_t)W * nout_rows * sizeof(cx<Ro>) ? tile : (size_t)W * nout_rows * sizeof(cx<Ro>);
  tile = (tile + 127) & ~(size_t)127;
  const size_t smem = 128 + 128 + ((L * sizeof(cx<Rw>) + 127) & ~(size_t)127) + tile +
                      (comb ? (size_t)W * nin_rows * sizeof(cx<Ri>) : 0);
  if (smem > 200 * 1024) return cudaSuccess;
  dim3 grid((l.a.ncols + W - 1) / W, l.nbatch, l.nfields);
  cudaError_t e;
  if (comb) {
    auto kern = k_axis_tma<Ri, Ro, Rw, R1, R2, DIR, true>;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e != cudaSuccess) return e;
    kern<<<grid, NT, smem, s>>>(l.a, tm, nin_rows, nout_rows, (unsigned)tile);
  } else {
    auto kern = k_axis_tma<Ri, Ro, Rw, R1, R2, DIR, false>;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e != cudaSuccess) return e;
    kern<<<grid, NT, smem, s>>>(l.a, tm, nin_rows, nout_rows, (unsigned)tile);
  }
  *used = true;
  return cudaGetLastError();
}

template <typename Ri, typename Ro, typename Rw, int R1, int R2, int DIR>
cudaError_t run_axis_fast(const AxisLaunch& l, cudaStream_t s) {
  constexpr int L = R1 * R2;
  constexpr int W = 256 / R1;
  if constexpr (L >= 16 && L <= 256) {
    if (axis_tma_enabled()) {
      bool used = false;
      cudaError_t e = run_axis_tma<Ri, Ro, Rw, R1, R2, DIR>(l, s, &used);
      if (e != cudaSuccess || used) return e;
    }
  }
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

// the matrix-product x-pass when every field's kind has its matrix and the tiles fit
template <typename Ri, typename Ro, typename Rw>
cudaError_t run_r2r_mm(const AxisLaunch& l, const R2RArgs& r, cudaStream_t s, bool* used) {
  *used = false;
  const int nin = amap_count(l.a.in);
  int rpad = 0;
  for (int f = 0; f < l.nfields; ++f) {
    const int k = r.kind[f];
    if (k < 0 || k > 3 || !r.mat[k] || r.mat_rows[k] != amap_count(l.a.out) || r.mat_cols[k] != nin)
      return cudaSuccess;
    rpad = std::max(rpad, (r.mat_rows[k] + 31) / 32 * 32);
  }
  // 64-column tiles when they fit in shared memory, else 32
  int cw = 64;
  size_t smem = (size_t)nin * cw * sizeof(cx<Rw>) + (size_t)nin * rpad * sizeof(Rw);
  if (smem > 200 * 1024) {
    cw = 32;
    smem = (size_t)nin * cw * sizeof(cx<Rw>) + (size_t)nin * rpad * sizeof(Rw);
  }
  if (smem > 200 * 1024) return cudaSuccess;
  auto kern = cw == 64 ? k_axis_r2r_mm<Ri, Ro, Rw, 64> : k_axis_r2r_mm<Ri, Ro, Rw, 32>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((l.a.ncols + cw - 1) / cw, l.nbatch, l.nfields);
  kern<<<grid, 256, smem, s>>>(l.a, l.ps, r);
  *used = true;
  return cudaGetLastError();
}

// the register-tiled matrix product (k_axis_r2r_gemm) unless TG_R2R_GEMM=0
bool r2r_gemm_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("TG_R2R_GEMM");
    return !(e && e[0] == '0');
  }();
  return on;
}

template <typename Ri, typename Ro, typename Rw, int RT>
cudaError_t run_r2r_gemm_rt(const AxisLaunch& l, const R2RArgs& r, int nrows, int nin, cudaStream_t s) {
  const int ntile = (nrows + RT - 1) / RT;
  const size_t smem = (size_t)nin * RT * sizeof(Rw);
  auto kern = k_axis_r2r_gemm<Ri, Ro, Rw, RT>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((l.a.ncols + 127) / 128, l.nbatch, l.nfields * ntile);
  kern<<<grid, 128, smem, s>>>(l.a, l.ps, r, ntile);
  return cudaGetLastError();
}

// when every field's kind has its matrix (all of the same size); the row tile leaving the fewest
// idle rows
template <typename Ri, typename Ro, typename Rw>
cudaError_t run_r2r_gemm(const AxisLaunch& l, const R2RArgs& r, cudaStream_t s, bool* used) {
  *used = false;
  if (!r2r_gemm_enabled()) return cudaSuccess;
  const int nin = amap_count(l.a.in), nout = amap_count(l.a.out);
  for (int f = 0; f < l.nfields; ++f) {
    const int k = r.kind[f];
    if (k < 0 || k > 3 || !r.mat[k] || r.mat_rows[k] != nout || r.mat_cols[k] != nin) return cudaSuccess;
  }
  if (nin < 1 || nout < 1 || (size_t)l.nfields * ((nout + 21) / 22) > 65535) return cudaSuccess;
  const int w43 = (nout + 42) / 43 * 43 - nout, w22 = (nout + 21) / 22 * 22 - nout;
  *used = true;
  if (w43 <= w22) return run_r2r_gemm_rt<Ri, Ro, Rw, 43>(l, r, nout, nin, s);
  return run_r2r_gemm_rt<Ri, Ro, Rw, 22>(l, r, nout, nin, s);
}

// FP32 forms: the x-pass contraction on the tensor cores (k_axis_r2r_tc, 3xTF32) when a field of
// one request spans at least kTcMinTiles column tiles (the per-block set-up, coefficient pairs and
// tensor memory, amortises; measured FP32-mixed steps against the register-tiled form: 129 x 256
// x 256 1.89 against 2.92 ms, 65 x 128 x 128 0.342 against 0.397 ms).  The rule looks at one
// request's geometry only, so a request batched in the serving loop takes the same path as on a
// lone context.  TG_R2R_TC=0 never, =1 always.
constexpr int kTcMinTiles = 16;
int r2r_tc_mode() {
  static const int m = [] {
    const char* e = std::getenv("TG_R2R_TC");
    if (e && e[0] == '0') return 0;
    if (e && e[0] == '1') return 1;
    return 2;
  }();
  return m;
}

template <typename Ri>
cudaError_t run_r2r_tc(const AxisLaunch& l, const R2RArgs& r, cudaStream_t s, bool* used) {
  *used = false;
  const int mode = r2r_tc_mode();
  if (mode == 0) return cudaSuccess;
  if (mode == 2 && (2LL * l.a.ncols + 127) / 128 < kTcMinTiles) return cudaSuccess;
  const int nin = amap_count(l.a.in), nout = amap_count(l.a.out);
  for (int f = 0; f < l.nfields; ++f) {
    const int k = r.kind[f];
    if (k < 0 || k > 3 || !r.mat[k] || r.mat_rows[k] != nout || r.mat_cols[k] != nin) return cudaSuccess;
    if (l.a.comb[f]) return cudaSuccess;
  }
  if (nin < 1 || nout < 1) return cudaSuccess;
  TcArgs t{};
  t.npad = (nout + 15) / 16 * 16;
  t.kpad = (nin + 7) / 8 * 8;
  if (t.npad > 256) return cudaSuccess;
  t.tmem_cols = 32;  // per accumulator; two of them
  while (t.tmem_cols < t.npad) t.tmem_cols *= 2;
  t.ntiles = (int)((2LL * l.a.ncols + 127) / 128);
  // coefficient pairs, nab operand slots of [hi, lo] chunks, eleven mbarriers, slot and flag;
  // three slots where they fit
  auto bytes = [&](int nab) {
    return sizeof(float) * (2 * (size_t)t.npad * t.kpad + 2 * (size_t)nab * 128 * kTcKC) +
           sizeof(uint64_t) * (2 * kTcMaxNab + 5) + 16;
  };
  int nab = kTcMaxNab;
  while (nab > 1 && bytes(nab) > 227 * 1024) --nab;
  const size_t smem = bytes(nab);
  if (smem > 227 * 1024) return cudaSuccess;
  t.nab = nab;
  auto kern = k_axis_r2r_tc<Ri>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  // one block per SM (shared memory, tensor memory): one persistent wave of at most 148 blocks,
  // or one block per (batch, field) when those alone exceed it
  const int per = l.nbatch * l.nfields;
  const int P = std::max(1, std::min(t.ntiles, 148 / per));
  *used = true;
  dim3 grid(P, l.nbatch, l.nfields);
  kern<<<grid, kTcThreads, smem, s>>>(l.a, l.ps, r, t);
  return cudaGetLastError();
}

template <typename Ri, typename Ro, typename Rw>
cudaError_t run_r2r(const AxisLaunch& l, const R2RArgs& r, int N, cudaStream_t s) {
  if constexpr (sizeof(Ro) == 4 && sizeof(Rw) == 4) {
    bool used = false;
    cudaError_t e = run_r2r_tc<Ri>(l, r, s, &used);
    if (e != cudaSuccess || used) return e;
  }
  {
    bool used = false;
    cudaError_t e = run_r2r_gemm<Ri, Ro, Rw>(l, r, s, &used);
    if (e != cudaSuccess || used) return e;
  }
  {
    bool used = false;
    cudaError_t e = run_r2r_mm<Ri, Ro, Rw>(l, r, s, &used);
    if (e != cudaSuccess || used) return e;
  }
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

int axis_tma_timeout(bool clear) {
  int h = 0;
  if (cudaMemcpyFromSymbol(&h, g_axis_tma_timeout, sizeof(int)) != cudaSuccess) return -1;
  if (clear && h) {
    const int z = 0;
    cudaMemcpyToSymbol(g_axis_tma_timeout, &z, sizeof(int));
  }
  return h;
}

}  // namespace tg
