// FFT pass kernels of the 3-D pseudo-spectral transforms.
//
// A 3-D FOUR transform of a (N1, N2, N3/2+1) complex field is three passes:
//   x-pass : batched c2c along axis 1 (row stride N2*(N3/2+1)),   kernel k_axis_c2c
//   y-pass : batched c2c along axis 2 (row stride N3/2+1),         kernel k_axis_c2c
//   z-pass : c2r / r2c along the contiguous axis 3 via a length-N3/2 complex FFT,
//            kernels k_z_c2r / k_z_r2c, or k_z_prod which fuses the inverse of several
//            fields, their pointwise real-space products and the forward of every product.
// Each pass reads and writes HBM once.  Inside a block the FFT of length L = R1*R2 is a
// two-step (four-step) FFT: a radix-R1 register DFT per thread, a twiddle, one transpose
// through shared memory, and a radix-R2 register DFT.  Axis maps (AxisMap) let a pass read
// only the stored (2/3-dealiased) wavenumbers and write only the ones that are kept, so the
// solver's fields live in a compact layout and the zero 1/3 band is neither read nor written.
#pragma once

#include "tg_common.cuh"
#include "tg_dft.cuh"

namespace tg {

constexpr int kMaxPtr = 12;

struct PtrSet {
  const void* src[kMaxPtr];
  void* dst[kMaxPtr];
  const void* src2[kMaxPtr];  // optional second source: input = src + comb * src2
};

struct AxisArgs {
  long long sb, sr;   // source: element stride between batches, between rows (FFT index)
  long long db, dr;   // destination strides
  int ncols;          // contiguous columns per batch processed
  AxisMap in, out;    // stored rows on input and output
  double scale;       // output scale
  const cx<double>* tw;  // exp(-2 pi i m / L), m in [0, L)
  int comb[kMaxPtr];  // per field: 0, or +1 / -1 to read src + comb * src2 (Elsasser z+-)
  // TMA-staged passes: set to 1 by a block whose tile did not arrive within the bounded wait
  // (the owning context's status word; null: a library-wide word)
  int* wait_flag;
  // test hook: 1 gives the first wait for a tile no polls at all, so every block reports a
  // timeout (the second, draining wait keeps its full limit and the copy lands before the
  // block leaves)
  int wait_short;
};

// ------------------------------------------------------------------------------------------
// strided-axis c2c, power-of-two L = R1 * R2 (R1 >= R2), 256 threads, W = 256/R1 columns
// ------------------------------------------------------------------------------------------
template <typename Ri, typename Ro, typename Rw, int R1, int R2, int DIR>
__global__ void __launch_bounds__(256) k_axis_c2c(AxisArgs a, PtrSet ps) {
  constexpr int L = R1 * R2;
  constexpr int W = 256 / R1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<Rw>* tw = reinterpret_cast<cx<Rw>*>(smem_raw);
  cx<Rw>* ex = tw + L;
  const int tid = threadIdx.x;
  const int f = blockIdx.z;
  const cx<Ri>* src = reinterpret_cast<const cx<Ri>*>(ps.src[f]) + (long long)blockIdx.y * a.sb;
  cx<Ro>* dst = reinterpret_cast<cx<Ro>*>(ps.dst[f]) + (long long)blockIdx.y * a.db;
  const int comb = a.comb[f];
  const cx<Ri>* src2 = comb ? reinterpret_cast<const cx<Ri>*>(ps.src2[f]) + (long long)blockIdx.y * a.sb : src;
  for (int i = tid; i < L; i += 256) tw[i] = cvt<Rw>(a.tw[i]);
  const int w = tid % W;
  const int col = blockIdx.x * W + w;
  const bool ok = col < a.ncols;
  __syncthreads();
  {
    const int n2 = tid / W;
    if (n2 < R2) {
      cx<Rw> v[R1];
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) {
        const int r = amap_row(a.in, R2 * n1 + n2);
        v[n1] = mkc<Rw>(0, 0);
        if (ok && r >= 0) {
          const long long o = (long long)r * a.sr + col;
          v[n1] = cvt<Rw>(src[o]);
          if (comb > 0) v[n1] = v[n1] + cvt<Rw>(src2[o]);
          else if (comb < 0) v[n1] = v[n1] - cvt<Rw>(src2[o]);
        }
      }
      DFT<R1, DIR, Rw>::run(v);
#pragma unroll
      for (int k1 = 0; k1 < R1; ++k1) {
        cx<Rw> t = tw[(n2 * k1) & (L - 1)];
        if (DIR > 0) t.y = -t.y;
        ex[(k1 * R2 + n2) * W + w] = v[k1] * t;
      }
    }
  }
  __syncthreads();
  {
    const int k1 = tid / W;
    cx<Rw> v[R2];
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) v[n2] = ex[(k1 * R2 + n2) * W + w];
    DFT<R2, DIR, Rw>::run(v);
    const Rw sc = (Rw)a.scale;
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) {
      const int r = amap_row(a.out, k1 + R1 * k2);
      if (ok && r >= 0) dst[(long long)r * a.dr + col] = cvt<Ro>(sc * v[k2]);
    }
  }
}

// ------------------------------------------------------------------------------------------
// strided-axis direct DFT for any L (used for lengths that are not a power of two)
// block = 256 threads, 8 columns, tile [L][8] in shared memory
// ------------------------------------------------------------------------------------------
template <typename Ri, typename Ro, typename Rw, int DIR>
__global__ void __launch_bounds__(256) k_axis_dft(AxisArgs a, PtrSet ps, int L) {
  constexpr int W = 8;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<Rw>* tw = reinterpret_cast<cx<Rw>*>(smem_raw);
  cx<Rw>* tile = tw + L;
  const int tid = threadIdx.x;
  const int f = blockIdx.z;
  const cx<Ri>* src = reinterpret_cast<const cx<Ri>*>(ps.src[f]) + (long long)blockIdx.y * a.sb;
  cx<Ro>* dst = reinterpret_cast<cx<Ro>*>(ps.dst[f]) + (long long)blockIdx.y * a.db;
  const int comb = a.comb[f];
  const cx<Ri>* src2 = comb ? reinterpret_cast<const cx<Ri>*>(ps.src2[f]) + (long long)blockIdx.y * a.sb : src;
  const int c0 = blockIdx.x * W;
  for (int i = tid; i < L; i += 256) {
    cx<Rw> t = cvt<Rw>(a.tw[i]);
    if (DIR > 0) t.y = -t.y;
    tw[i] = t;
  }
  for (int i = tid; i < L * W; i += 256) {
    const int n = i / W, w = i % W;
    const int r = amap_row(a.in, n);
    const int col = c0 + w;
    cx<Rw> v = mkc<Rw>(0, 0);
    if (col < a.ncols && r >= 0) {
      const long long o = (long long)r * a.sr + col;
      v = cvt<Rw>(src[o]);
      if (comb > 0) v = v + cvt<Rw>(src2[o]);
      else if (comb < 0) v = v - cvt<Rw>(src2[o]);
    }
    tile[i] = v;
  }
  __syncthreads();
  const Rw sc = (Rw)a.scale;
  for (int i = tid; i < L * W; i += 256) {
    const int k = i / W, w = i % W;
    const int r = amap_row(a.out, k);
    const int col = c0 + w;
    if (col >= a.ncols || r < 0) continue;
    cx<Rw> acc = mkc<Rw>(0, 0);
    int m = 0;
    for (int n = 0; n < L; ++n) {
      acc = acc + tile[n * W + w] * tw[m];
      m += k;
      if (m >= L) m -= L;
    }
    dst[(long long)r * a.dr + col] = cvt<Ro>(sc * acc);
  }
}

// ------------------------------------------------------------------------------------------
// SCFT x-pass: real-to-real transforms along axis 1 on complex columns (the real and imaginary
// parts transform alike, as the reference's separate calls on real() and imag() do,
// scft_tr.cc:249-259).  With t[j] = (cos, sin)(pi j / 2N), j in [0, 4N):
//   kind 0  forward CFT  (REDFT10)             Y[k] = 2 sum_n x_n cos(pi (2n+1) k / 2N)
//   kind 1  forward SFT  (RODFT10, shift right) Y[m] = 2 sum_n x_n sin(pi (2n+1) m / 2N)
//           (slot m <-> DST-II index m-1; m = 0 gives 0 and index N-1 is never produced,
//            exactly ArrayShiftRight_SCFT scft_tr.cc:153-184)
//   kind 2  inverse ICFT (REDFT01)             y_k = X_0 + 2 sum_{m>=1} X_m cos(pi m (2k+1) / 2N)
//   kind 3  inverse ISFT (shift left, RODFT01) y_k = 2 sum_{m>=1} X_m sin(pi m (2k+1) / 2N)
// Block: 32 columns (one per lane) x 8 warps; the stored input rows of the tile are staged
// in shared memory and each warp produces every eighth output row.
// ------------------------------------------------------------------------------------------
struct R2RArgs {
  int kind[kMaxPtr];
  const cx<double>* trig;  // (cos, sin)(pi j / 2N), j in [0, 4N)
  // optional: per kind the transform as a matrix for this launch's row maps, column-major
  // [stored input row][output row] (output row = destination row), or null
  const double* mat[4];
  int mat_rows[4];         // output rows of mat[kind] (= amap_count(out))
  int mat_cols[4];         // stored input rows of mat[kind] (= amap_count(in))
};

template <typename Ri, typename Ro, typename Rw>
__global__ void __launch_bounds__(256) k_axis_r2r(AxisArgs a, PtrSet ps, R2RArgs r, int N) {
  constexpr int W = 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<Rw>* tr = reinterpret_cast<cx<Rw>*>(smem_raw);  // 4N
  const int nin = amap_count(a.in);
  cx<Rw>* tile = tr + 4 * N;                         // [nin][W]
  const int tid = threadIdx.x, lane = tid & 31, wy = tid >> 5;
  const int f = blockIdx.z;
  const int kind = r.kind[f];
  const cx<Ri>* src = reinterpret_cast<const cx<Ri>*>(ps.src[f]) + (long long)blockIdx.y * a.sb;
  cx<Ro>* dst = reinterpret_cast<cx<Ro>*>(ps.dst[f]) + (long long)blockIdx.y * a.db;
  const int col = blockIdx.x * W + lane;
  const bool ok = col < a.ncols;
  for (int i = tid; i < 4 * N; i += 256) tr[i] = cvt<Rw>(r.trig[i]);
  for (int i = tid; i < nin * W; i += 256) {
    const int row = i / W, w = i % W;
    const int c2 = blockIdx.x * W + w;
    tile[i] = (c2 < a.ncols) ? cvt<Rw>(src[(long long)row * a.sr + c2]) : mkc<Rw>(0, 0);
  }
  __syncthreads();
  const int fourN = 4 * N;
  const bool sine = (kind == 1 || kind == 3);
  const Rw sc = (Rw)a.scale;
  for (int ko = wy; ko < a.out.L; ko += 8) {
    const int orow = amap_row(a.out, ko);
    if (orow < 0) continue;
    cx<Rw> acc = mkc<Rw>(0, 0);
    if (kind <= 1) {
      // forward: inputs are the N real-space points n (all stored), j = (2n+1) ko
      const int step = 2 * ko % fourN;
      int j = ko % fourN;
      for (int n = 0; n < nin; ++n) {
        const Rw t = sine ? tr[j].y : tr[j].x;
        const cx<Rw> x = tile[n * W + lane];
        acc.x += t * x.x;
        acc.y += t * x.y;
        j += step;
        if (j >= fourN) j -= fourN;
      }
      acc.x *= (Rw)2;
      acc.y *= (Rw)2;
    } else {
      // inverse: inputs are the stored spectral slots m, j = m (2 ko + 1)
      const int odd = (2 * ko + 1) % fourN;
      int j = 0;
      for (int rr = 0; rr < nin; ++rr) {
        const int m = amap_index(a.in, rr);
        if (rr == 0 || rr == a.in.lo) {
          j = (int)(((long long)m * odd) % fourN);
        } else {
          j += odd;
          if (j >= fourN) j -= fourN;
        }
        const Rw t = (sine ? tr[j].y : tr[j].x) * ((m == 0 && !sine) ? (Rw)1 : (Rw)2);
        const cx<Rw> x = tile[rr * W + lane];
        acc.x += t * x.x;
        acc.y += t * x.y;
      }
    }
    if (ok) dst[(long long)orow * a.dr + col] = cvt<Ro>(sc * acc);
  }
}

// The same transforms as a matrix product Y[orow][col] = scale * sum_rr T[rr][orow] X[rr][col]
// (T real, X complex).  Block: CW (64 or 32) columns of one batch and field; thread (lane, warp)
// owns CW/32 adjacent columns of the tile and output rows r0 .. r0+3 of each row pass, so every
// k step is a broadcast load of 4 coefficients, a load of its columns and 8 or 16 FMAs.
template <typename Ri, typename Ro, typename Rw, int CW>
__global__ void __launch_bounds__(256) k_axis_r2r_mm(AxisArgs a, PtrSet ps, R2RArgs r) {
  constexpr int TR = 4;
  constexpr int CL = CW / 32;  // columns per lane: 2 (64-column tiles) or 1 (32)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nin = amap_count(a.in);
  const int f = blockIdx.z;
  const int kind = r.kind[f];
  const int nrows = r.mat_rows[kind];
  const int rpad = (nrows + 8 * TR - 1) / (8 * TR) * (8 * TR);
  cx<Rw>* X = reinterpret_cast<cx<Rw>*>(smem_raw);               // [nin][CW]
  Rw* T = reinterpret_cast<Rw*>(X + (size_t)nin * CW);            // [nin][rpad]
  const int tid = threadIdx.x, lane = tid & 31, wy = tid >> 5;
  const cx<Ri>* src = reinterpret_cast<const cx<Ri>*>(ps.src[f]) + (long long)blockIdx.y * a.sb;
  cx<Ro>* dst = reinterpret_cast<cx<Ro>*>(ps.dst[f]) + (long long)blockIdx.y * a.db;
  const int c0 = blockIdx.x * CW;
  for (int i = tid; i < nin * CW; i += 256) {
    const int row = i / CW, w = i % CW;
    X[i] = (c0 + w < a.ncols) ? cvt<Rw>(src[(long long)row * a.sr + c0 + w]) : mkc<Rw>(0, 0);
  }
  const double* M = r.mat[kind];
  for (int i = tid; i < nin * rpad; i += 256) {
    const int k = i / rpad, rr = i % rpad;
    T[i] = rr < nrows ? (Rw)M[(size_t)k * nrows + rr] : (Rw)0;
  }
  __syncthreads();
  const Rw sc = (Rw)a.scale;
  const int col = c0 + CL * lane;
  for (int rb = 0; rb < rpad; rb += 8 * TR) {
    const int r0 = rb + wy * TR;
    cx<Rw> acc[TR][CL];
#pragma unroll
    for (int i = 0; i < TR; ++i)
#pragma unroll
      for (int q = 0; q < CL; ++q) acc[i][q] = mkc<Rw>(0, 0);
    for (int k = 0; k < nin; ++k) {
      cx<Rw> x[CL];
#pragma unroll
      for (int q = 0; q < CL; ++q) x[q] = X[k * CW + CL * lane + q];
#pragma unroll
      for (int i = 0; i < TR; ++i) {
        const Rw t = T[k * rpad + r0 + i];
#pragma unroll
        for (int q = 0; q < CL; ++q) {
          acc[i][q].x += t * x[q].x;
          acc[i][q].y += t * x[q].y;
        }
      }
    }
#pragma unroll
    for (int i = 0; i < TR; ++i) {
      const int orow = r0 + i;
      if (orow >= nrows) continue;
      cx<Ro>* d = dst + (long long)orow * a.dr;
#pragma unroll
      for (int q = 0; q < CL; ++q)
        if (col + q < a.ncols) d[col + q] = cvt<Ro>(sc * acc[i][q]);
    }
  }
}

// The same transforms as a register-tiled matrix product: a thread owns one complex column and
// RT consecutive output rows (the row tile blockIdx.z % ntile of field blockIdx.z / ntile), with
// the accumulators in registers; the tile's coefficients T[k][m0 .. m0 + RT) are broadcast from
// shared memory and the input column streams from global memory, coalesced across the block's
// columns.  Each input value feeds 2 RT fused multiply-adds (the matrix-product form above does
// five shared-memory loads per eight), so the FP64 form runs at the FP64 pipe's rate.  RT = 43
// tiles the row counts of N1 = 129 and 128 (129, 128, 86, 85 rows) with at most one idle row;
// RT = 22 those of N1 = 65 (65, 43).  Sums run over k in order, as in the forms above.
template <typename Ri, typename Ro, typename Rw, int RT>
__global__ void __launch_bounds__(128) k_axis_r2r_gemm(AxisArgs a, PtrSet ps, R2RArgs r, int ntile) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Rw* Ts = reinterpret_cast<Rw*>(smem_raw);  // [nin][RT]
  const int f = blockIdx.z / ntile, tile = blockIdx.z - f * ntile;
  const int kind = r.kind[f];
  const int nrows = r.mat_rows[kind], nin = r.mat_cols[kind];
  const int m0 = tile * RT;
  const double* M = r.mat[kind];
  for (int i = threadIdx.x; i < nin * RT; i += blockDim.x) {
    const int k = i / RT, m = i - k * RT;
    Ts[i] = (m0 + m < nrows) ? (Rw)M[(size_t)k * nrows + m0 + m] : (Rw)0;
  }
  __syncthreads();
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= a.ncols) return;
  const cx<Ri>* src = reinterpret_cast<const cx<Ri>*>(ps.src[f]) + (long long)blockIdx.y * a.sb + col;
  cx<Ro>* dst = reinterpret_cast<cx<Ro>*>(ps.dst[f]) + (long long)blockIdx.y * a.db + col;
  Rw ax[RT], ay[RT];
#pragma unroll
  for (int m = 0; m < RT; ++m) ax[m] = ay[m] = (Rw)0;
#pragma unroll 2
  for (int k = 0; k < nin; ++k) {
    const cx<Rw> x = cvt<Rw>(src[(long long)k * a.sr]);
    const Rw* t = Ts + k * RT;
#pragma unroll
    for (int m = 0; m < RT; ++m) {
      ax[m] = fma(t[m], x.x, ax[m]);
      ay[m] = fma(t[m], x.y, ay[m]);
    }
  }
  const Rw sc = (Rw)a.scale;
#pragma unroll
  for (int m = 0; m < RT; ++m)
    if (m0 + m < nrows) dst[(long long)(m0 + m) * a.dr] = cvt<Ro>(mkc<Rw>(sc * ax[m], sc * ay[m]));
}

// ------------------------------------------------------------------------------------------
// z-pass (contiguous axis) c2r / r2c.  Rows hold N3/2+1 spectral values of which the first
// `nin` are stored (the rest are zero); the real row of N3 = 2M values is packed as M complex
// (x[2m] + i x[2m+1]), the reference's in-place layout, followed by a zero padding slot.
// ------------------------------------------------------------------------------------------
struct ZArgs {
  long long nrows;
  long long ss, ds;     // row strides (complex elements)
  int nin, nout;        // stored spectral entries on input (c2r) / output (r2c)
  int nfill;            // r2c: entries [nout, nfill) of each output row are written as zero
  int pad;              // c2r: write a zero to slot M of each output row
  double scale;
  const cx<double>* twM;  // exp(-2 pi i m / M), m in [0, M)
  const cx<double>* twN;  // exp(-2 pi i k / N), k in [0, N), N = 2M
  const cx<double>* oct;  // N = 256: coefficient table of k_z_prod_oct (zoct_table), or null
};

// c2r pre-twiddle: Z[k] = (X[k] + conj(X[M-k])) + i e^{+i pi k/M} (X[k] - conj(X[M-k])); the
// imaginary parts of X[0] and X[M] are ignored (the c2r rule of FFTW and pocketfft).
template <typename Rw, typename Ri>
__device__ __forceinline__ cx<Rw> c2r_pre(const cx<Ri>* row, int k, int M, int nin, const cx<Rw>* twN) {
  cx<Rw> a = (k < nin) ? cvt<Rw>(row[k]) : mkc<Rw>(0, 0);
  const int km = M - k;
  cx<Rw> b = (km < nin) ? cvt<Rw>(row[km]) : mkc<Rw>(0, 0);
  if (k == 0) {
    a.y = 0;
    b.y = 0;
  }
  b.y = -b.y;
  cx<Rw> h = twN[k];
  h.y = -h.y;  // e^{+i pi k / M}
  return (a + b) + ione(h * (a - b));
}

// r2c post-twiddle: X[k] = (Z[k] + conj(Z[M-k]))/2 - (i/2) e^{-i pi k/M} (Z[k] - conj(Z[M-k]))
template <typename Rw>
__device__ __forceinline__ cx<Rw> r2c_post(const cx<Rw>* zrow, int k, int M, const cx<Rw>* twN) {
  const cx<Rw> zk = zrow[k & (M - 1)];
  cx<Rw> zm = zrow[(M - k) & (M - 1)];
  zm.y = -zm.y;
  const cx<Rw> s = zk + zm;
  const cx<Rw> d = twN[k] * (zk - zm);
  return mkc<Rw>((Rw)0.5 * (s.x + d.y), (Rw)0.5 * (s.y - d.x));
}

template <typename Ri, typename Ro, typename Rw, int R1, int R2>
__global__ void __launch_bounds__(256) k_z_c2r(ZArgs a, PtrSet ps) {
  constexpr int M = R1 * R2;
  constexpr int T = R1;
  constexpr int ROWS = 256 / T;
  constexpr int EXP = R2 + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<Rw>* twM = reinterpret_cast<cx<Rw>*>(smem_raw);
  cx<Rw>* twN = twM + M;
  cx<Rw>* ex = twN + 2 * M;
  const int tid = threadIdx.x;
  for (int i = tid; i < M; i += 256) twM[i] = cvt<Rw>(a.twM[i]);
  for (int i = tid; i < 2 * M; i += 256) twN[i] = cvt<Rw>(a.twN[i]);
  const int f = blockIdx.z;
  const int rl = tid / T, t = tid % T;
  const long long row = (long long)blockIdx.x * ROWS + rl;
  const bool ok = row < a.nrows;
  const cx<Ri>* src = reinterpret_cast<const cx<Ri>*>(ps.src[f]) + row * a.ss;
  cx<Ro>* dst = reinterpret_cast<cx<Ro>*>(ps.dst[f]) + row * a.ds;
  cx<Rw>* exr = ex + rl * R1 * EXP;
  __syncthreads();
  if (t < R2) {
    cx<Rw> v[R1];
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1)
      v[n1] = ok ? c2r_pre<Rw>(src, R2 * n1 + t, M, a.nin, twN) : mkc<Rw>(0, 0);
    DFT<R1, +1, Rw>::run(v);
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
      cx<Rw> w = twM[(t * k1) & (M - 1)];
      w.y = -w.y;
      exr[k1 * EXP + t] = v[k1] * w;
    }
  }
  __syncthreads();
  {
    const int k1 = t;
    cx<Rw> v[R2];
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) v[n2] = exr[k1 * EXP + n2];
    DFT<R2, +1, Rw>::run(v);
    const Rw sc = (Rw)a.scale;
    if (ok) {
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) dst[k1 + R1 * k2] = cvt<Ro>(sc * v[k2]);
      if (a.pad && k1 == 0) dst[M] = mkc<Ro>(0, 0);
    }
  }
}

template <typename Ri, typename Ro, typename Rw, int R1, int R2>
__global__ void __launch_bounds__(256) k_z_r2c(ZArgs a, PtrSet ps) {
  constexpr int M = R1 * R2;
  constexpr int T = R1;
  constexpr int ROWS = 256 / T;
  constexpr int EXP = R2 + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<Rw>* twM = reinterpret_cast<cx<Rw>*>(smem_raw);
  cx<Rw>* twN = twM + M;
  cx<Rw>* ex = twN + 2 * M;
  cx<Rw>* zb = ex + ROWS * R1 * EXP;
  const int tid = threadIdx.x;
  for (int i = tid; i < M; i += 256) twM[i] = cvt<Rw>(a.twM[i]);
  for (int i = tid; i < 2 * M; i += 256) twN[i] = cvt<Rw>(a.twN[i]);
  const int f = blockIdx.z;
  const int rl = tid / T, t = tid % T;
  const long long row = (long long)blockIdx.x * ROWS + rl;
  const bool ok = row < a.nrows;
  const cx<Ri>* src = reinterpret_cast<const cx<Ri>*>(ps.src[f]) + row * a.ss;
  cx<Ro>* dst = reinterpret_cast<cx<Ro>*>(ps.dst[f]) + row * a.ds;
  cx<Rw>* exr = ex + rl * R1 * EXP;
  cx<Rw>* zr = zb + rl * M;
  __syncthreads();
  if (t < R2) {
    cx<Rw> v[R1];
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) v[n1] = ok ? cvt<Rw>(src[R2 * n1 + t]) : mkc<Rw>(0, 0);
    DFT<R1, -1, Rw>::run(v);
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) exr[k1 * EXP + t] = v[k1] * twM[(t * k1) & (M - 1)];
  }
  __syncthreads();
  {
    const int k1 = t;
    cx<Rw> v[R2];
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) v[n2] = exr[k1 * EXP + n2];
    DFT<R2, -1, Rw>::run(v);
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) zr[k1 + R1 * k2] = v[k2];
  }
  __syncthreads();
  if (ok) {
    const Rw sc = (Rw)a.scale;
    for (int k = t; k < a.nout; k += T) dst[k] = cvt<Ro>(sc * r2c_post<Rw>(zr, k, M, twN));
    for (int k = a.nout + t; k < a.nfill; k += T) dst[k] = mkc<Ro>(0, 0);
  }
}

// direct z-pass DFTs for any even N3 (N3/2 not a power of two); one row per block
template <typename Ri, typename Ro, typename Rw>
__global__ void __launch_bounds__(128) k_z_c2r_dft(ZArgs a, PtrSet ps, int M) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = 2 * M;
  cx<Rw>* twN = reinterpret_cast<cx<Rw>*>(smem_raw);
  cx<Rw>* X = twN + N;
  const int f = blockIdx.z;
  const long long row = blockIdx.x;
  const cx<Ri>* src = reinterpret_cast<const cx<Ri>*>(ps.src[f]) + row * a.ss;
  cx<Ro>* dst = reinterpret_cast<cx<Ro>*>(ps.dst[f]) + row * a.ds;
  for (int i = threadIdx.x; i < N; i += blockDim.x) twN[i] = cvt<Rw>(a.twN[i]);
  for (int k = threadIdx.x; k <= M; k += blockDim.x) X[k] = (k < a.nin) ? cvt<Rw>(src[k]) : mkc<Rw>(0, 0);
  __syncthreads();
  const Rw sc = (Rw)a.scale;
  for (int n = threadIdx.x; n < N; n += blockDim.x) {
    // x[n] = Re X0 + Re XM (-1)^n + 2 sum_{k=1}^{M-1} Re(X_k e^{+2 pi i k n / N})
    Rw acc = X[0].x + ((n & 1) ? -X[M].x : X[M].x);
    int m = 0;
    for (int k = 1; k < M; ++k) {
      m += n;
      if (m >= N) m -= N;
      const cx<Rw> w = twN[m];  // e^{-i theta}; Re(X e^{+i theta}) = X.x w.x + X.y w.y
      acc += (Rw)2 * (X[k].x * w.x + X[k].y * w.y);
    }
    reinterpret_cast<Ro*>(dst)[n] = (Ro)(sc * acc);
  }
  if (a.pad && threadIdx.x == 0) dst[M] = mkc<Ro>(0, 0);
}

template <typename Ri, typename Ro, typename Rw>
__global__ void __launch_bounds__(128) k_z_r2c_dft(ZArgs a, PtrSet ps, int M) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = 2 * M;
  cx<Rw>* twN = reinterpret_cast<cx<Rw>*>(smem_raw);
  Rw* x = reinterpret_cast<Rw*>(twN + N);
  const int f = blockIdx.z;
  const long long row = blockIdx.x;
  const Ri* src = reinterpret_cast<const Ri*>(reinterpret_cast<const cx<Ri>*>(ps.src[f]) + row * a.ss);
  cx<Ro>* dst = reinterpret_cast<cx<Ro>*>(ps.dst[f]) + row * a.ds;
  for (int i = threadIdx.x; i < N; i += blockDim.x) twN[i] = cvt<Rw>(a.twN[i]);
  for (int i = threadIdx.x; i < N; i += blockDim.x) x[i] = (Rw)src[i];
  __syncthreads();
  const Rw sc = (Rw)a.scale;
  for (int k = threadIdx.x; k < a.nout; k += blockDim.x) {
    cx<Rw> acc = mkc<Rw>(0, 0);
    int m = 0;
    for (int n = 0; n < N; ++n) {
      acc = acc + x[n] * twN[m];
      m += k;
      if (m >= N) m -= N;
    }
    dst[k] = cvt<Ro>(sc * acc);
  }
  for (int k = a.nout + threadIdx.x; k < a.nfill; k += blockDim.x) dst[k] = mkc<Ro>(0, 0);
}

// ------------------------------------------------------------------------------------------
// Fused z-pass of the nonlinear term: inverse (c2r) of NIN fields, NPROD pointwise real-space
// products (pairs of inputs), forward (r2c) of every product with scale 1/(N1 N2 N3).
// Between the inverse and the forward FFT each thread keeps the same positions
// m = k1 + R1 k2, which are exactly the inputs of the forward FFT's first step with the radix
// roles swapped, so the products are formed without another exchange.
// ------------------------------------------------------------------------------------------
struct ProdPairs {
  signed char a[12], b[12];
};

template <typename Ri, typename Ro, typename Rw, int R1, int R2, int NIN, int NPROD>
__global__ void __launch_bounds__(256 / ((R1 * R2 >= 128) ? 2 : 1))
    k_z_prod(ZArgs a, PtrSet ps, ProdPairs pp) {
  constexpr int M = R1 * R2;
  constexpr int T = R1;
  constexpr int ROWS = (256 / ((M >= 128) ? 2 : 1)) / T;
  constexpr int EXA = R2 + 1;   // inverse exchange pitch
  constexpr int EXB = R1 + 1;   // forward exchange pitch
  constexpr int EXS = (R1 * EXA > R2 * EXB) ? R1 * EXA : R2 * EXB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<Rw>* twM = reinterpret_cast<cx<Rw>*>(smem_raw);
  cx<Rw>* twN = twM + M;
  cx<Rw>* ex = twN + 2 * M;
  cx<Rw>* zb = ex + ROWS * EXS;
  cx<Rw>* rs = zb + ROWS * M;  // [NIN][ROWS][M]
  const int tid = threadIdx.x;
  for (int i = tid; i < M; i += blockDim.x) twM[i] = cvt<Rw>(a.twM[i]);
  for (int i = tid; i < 2 * M; i += blockDim.x) twN[i] = cvt<Rw>(a.twN[i]);
  const int rl = tid / T, t = tid % T;
  const long long row = (long long)blockIdx.x * ROWS + rl;
  const bool ok = row < a.nrows;
  cx<Rw>* exr = ex + rl * EXS;
  cx<Rw>* zr = zb + rl * M;
  __syncthreads();
#pragma unroll 1
  for (int c = 0; c < NIN; ++c) {
    const cx<Ri>* src = reinterpret_cast<const cx<Ri>*>(ps.src[c]) + row * a.ss;
    if (t < R2) {
      cx<Rw> v[R1];
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1)
        v[n1] = ok ? c2r_pre<Rw>(src, R2 * n1 + t, M, a.nin, twN) : mkc<Rw>(0, 0);
      DFT<R1, +1, Rw>::run(v);
#pragma unroll
      for (int k1 = 0; k1 < R1; ++k1) {
        cx<Rw> w = twM[(t * k1) & (M - 1)];
        w.y = -w.y;
        exr[k1 * EXA + t] = v[k1] * w;
      }
    }
    __syncthreads();
    {
      cx<Rw> v[R2];
#pragma unroll
      for (int n2 = 0; n2 < R2; ++n2) v[n2] = exr[t * EXA + n2];
      DFT<R2, +1, Rw>::run(v);
      cx<Rw>* rsr = rs + ((long long)c * ROWS + rl) * M;
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) rsr[t + R1 * k2] = v[k2];
    }
    __syncthreads();
  }
  const Rw sc = (Rw)a.scale;
#pragma unroll 1
  for (int q = 0; q < NPROD; ++q) {
    const cx<Rw>* ra = rs + ((long long)pp.a[q] * ROWS + rl) * M;
    const cx<Rw>* rb = rs + ((long long)pp.b[q] * ROWS + rl) * M;
    {
      // forward step 1: radix R2 over k2 for this thread's n2' = t
      cx<Rw> v[R2];
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) v[k2] = rmul(ra[t + R1 * k2], rb[t + R1 * k2]);
      DFT<R2, -1, Rw>::run(v);
#pragma unroll
      for (int k1p = 0; k1p < R2; ++k1p) exr[k1p * EXB + t] = v[k1p] * twM[(t * k1p) & (M - 1)];
    }
    __syncthreads();
    if (t < R2) {
      cx<Rw> v[R1];
#pragma unroll
      for (int n2p = 0; n2p < R1; ++n2p) v[n2p] = exr[t * EXB + n2p];
      DFT<R1, -1, Rw>::run(v);
#pragma unroll
      for (int k2p = 0; k2p < R1; ++k2p) zr[t + R2 * k2p] = v[k2p];
    }
    __syncthreads();
    if (ok) {
      cx<Ro>* dst = reinterpret_cast<cx<Ro>*>(ps.dst[q]) + row * a.ds;
      for (int k = t; k < a.nout; k += T) dst[k] = cvt<Ro>(sc * r2c_post<Rw>(zr, k, M, twN));
      for (int k = a.nout + t; k < a.nfill; k += T) dst[k] = mkc<Ro>(0, 0);
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------------------------------
// Warp-per-row fused z-pass for M = N3/2 = 32 E (E in {1, 2, 4, 8}).
//
// Lane l holds the entries n = l + 32 j (j < E) of a row.  Inverse length-M DFT:
//   radix-E DFT over j in registers, twiddle e^{+2 pi i l k1 / M}, then a 32-point DFT across
//   lanes as five radix-2 decimation-in-frequency shuffle stages -> lane l, register k1 holds
//   z[k1 + E bitrev5(l)].
// The products are pointwise, so the permuted order is harmless, and the forward DFT is the
// exact adjoint network (decimation-in-time stages in reverse order, conjugate twiddles, then
// the forward radix-E DFT), which takes the permuted order and returns X[l + 32 j] in natural
// order.  No shared-memory transposes and no block barriers; the real-space values of the NIN
// inputs are parked in warp-private shared memory, each lane reading back only its own slots.
// ------------------------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ cx<R> shfl_xor_c(cx<R> v, int m) {
  return mkc<R>(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}
template <typename R>
__device__ __forceinline__ cx<R> shfl_c(cx<R> v, int src) {
  return mkc<R>(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

// Inverse 32-point DFT across lanes, DIF, branch-free.  Stage s pairs lanes l and l ^ h
// (h = 16 >> s); with p the partner's value the lower lane keeps v + p and the upper lane
// (p - v) w, w = e^{+2 pi i (l mod h) / (2h)}.  Both are (p + sg v) wl with sg = -1 / +1 and
// wl = w / 1 on the upper / lower lane (wl[s] precomputed per lane).
// The last two stages have trivial twiddles: h = 2 multiplies by i on lanes l = 3 mod 4 (w =
// e^{i pi / 2}) and by 1 elsewhere; h = 1 multiplies by 1.
template <typename R, int E>
__device__ __forceinline__ void lane_dif32(cx<R> (&v)[E], const cx<R> (&wl)[5], int lane) {
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    const int h = 16 >> s;
    const R sg = (lane & h) ? (R)-1 : (R)1;
    const bool rot = (lane & 3) == 3;
#pragma unroll
    for (int k = 0; k < E; ++k) {
      const cx<R> p = shfl_xor_c(v[k], h);
      const cx<R> a = mkc<R>(fma(sg, v[k].x, p.x), fma(sg, v[k].y, p.y));
      if (s == 4) v[k] = a;
      else if (s == 3) v[k] = rot ? mkc<R>(-a.y, a.x) : a;
      else v[k] = a * wl[s];
    }
  }
}

// Forward 32-point DFT across lanes: the adjoint of lane_dif32 (DIT, stages h = 1 .. 16).
// The upper lane pre-multiplies by conj(w) and both lanes finish with r + sg s, where s is the
// lane's (weighted) value and r the partner's.
template <typename R, int E>
__device__ __forceinline__ void lane_dit32_fwd(cx<R> (&v)[E], const cx<R> (&wl)[5], int lane) {
#pragma unroll
  for (int s = 4; s >= 0; --s) {
    const int h = 16 >> s;
    const R sg = (lane & h) ? (R)-1 : (R)1;
    const cx<R> wc = conjc(wl[s]);
    const bool rot = (lane & 3) == 3;
#pragma unroll
    for (int k = 0; k < E; ++k) {
      cx<R> sv;
      if (s == 4) sv = v[k];
      else if (s == 3) sv = rot ? mkc<R>(v[k].y, -v[k].x) : v[k];
      else sv = wc * v[k];
      const cx<R> r = shfl_xor_c(sv, h);
      v[k] = mkc<R>(fma(sg, sv.x, r.x), fma(sg, sv.y, r.y));
    }
  }
}

template <typename Ri, typename Ro, typename Rw, int E, int NIN, int NPROD, int WPB>
__global__ void __launch_bounds__(32 * WPB, (E <= 4 ? (sizeof(Rw) == 8 ? 4 : 6) : (sizeof(Rw) == 8 ? 3 : 4)))
    k_z_prod_warp(ZArgs a, PtrSet ps, ProdPairs pp) {
  constexpr int M = 32 * E;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  cx<Rw>* rs = reinterpret_cast<cx<Rw>*>(smem_raw) + (size_t)wib * NIN * E * 32;
  // per-lane twiddles from twN[k] = e^{-i pi k / M}, k < 2M
  cx<Rw> hw[E], tw1[E], tws[5];
#pragma unroll
  for (int j = 0; j < E; ++j) hw[j] = cvt<Rw>(a.twN[lane + 32 * j]);
#pragma unroll
  for (int k1 = 0; k1 < E; ++k1) tw1[k1] = conjc(cvt<Rw>(a.twN[(2 * lane * k1) % (2 * M)]));
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    const int h = 16 >> s;
    // e^{+2 pi i (l mod h) / (2h)} on the upper lane of each pair, 1 on the lower lane
    tws[s] = (lane & h) ? conjc(cvt<Rw>(a.twN[(lane & (h - 1)) * (M / h)])) : mkc<Rw>(1, 0);
  }
  const Rw sc = (Rw)a.scale;
  const long long nwarps = (long long)gridDim.x * WPB;
  for (long long row = (long long)blockIdx.x * WPB + wib; row < a.nrows; row += nwarps) {
    // ---- inverse (c2r) of every input
#pragma unroll 1
    for (int c = 0; c < NIN; ++c) {
      const cx<Ri>* src = reinterpret_cast<const cx<Ri>*>(ps.src[c]) + row * a.ss;
      cx<Rw> v[E];
#pragma unroll
      for (int j = 0; j < E; ++j) {
        const int k = lane + 32 * j;
        cx<Rw> xa = (k < a.nin) ? cvt<Rw>(src[k]) : mkc<Rw>(0, 0);
        const int km = M - k;
        cx<Rw> xb = (km < a.nin) ? cvt<Rw>(src[km]) : mkc<Rw>(0, 0);
        if (k == 0) {
          xa.y = 0;
          xb.y = 0;
        }
        xb.y = -xb.y;
        v[j] = (xa + xb) + ione(conjc(hw[j]) * (xa - xb));
      }
      DFT<E, +1, Rw>::run(v);
#pragma unroll
      for (int k1 = 1; k1 < E; ++k1) v[k1] = v[k1] * tw1[k1];
      lane_dif32<Rw, E>(v, tws, lane);
#pragma unroll
      for (int k1 = 0; k1 < E; ++k1) rs[(c * E + k1) * 32 + lane] = v[k1];
    }
    // ---- products and forward (r2c)
#pragma unroll 1
    for (int q = 0; q < NPROD; ++q) {
      const int pa = pp.a[q], pb = pp.b[q];
      cx<Rw> v[E];
#pragma unroll
      for (int k1 = 0; k1 < E; ++k1) v[k1] = rmul(rs[(pa * E + k1) * 32 + lane], rs[(pb * E + k1) * 32 + lane]);
      lane_dit32_fwd<Rw, E>(v, tws, lane);
#pragma unroll
      for (int k1 = 1; k1 < E; ++k1) v[k1] = v[k1] * conjc(tw1[k1]);
      DFT<E, -1, Rw>::run(v);
      cx<Ro>* dst = reinterpret_cast<cx<Ro>*>(ps.dst[q]) + row * a.ds;
      const int pl = (32 - lane) & 31;
#pragma unroll
      for (int j = 0; j < E; ++j) {
        // Z[M - k] for k = lane + 32 j: lane (32 - l) & 31, register E-1-j (own register
        // (E - j) mod E on lane 0)
        cx<Rw> zm = shfl_c(v[E - 1 - j], pl);
        if (lane == 0) zm = v[(E - j) % E];
        zm.y = -zm.y;
        const cx<Rw> s = v[j] + zm;
        const cx<Rw> d = hw[j] * (v[j] - zm);
        const int k = lane + 32 * j;
        if (k < a.nout) dst[k] = cvt<Ro>(mkc<Rw>(sc * (Rw)0.5 * (s.x + d.y), sc * (Rw)0.5 * (s.y - d.x)));
      }
      if (lane == 0 && a.nout > M) dst[M] = cvt<Ro>(mkc<Rw>(sc * (v[0].x - v[0].y), (Rw)0));
      for (int k = a.nout + lane; k < a.nfill; k += 32) dst[k] = mkc<Ro>(0, 0);
    }
  }
}

// ------------------------------------------------------------------------------------------
// Warp-per-row fused z-pass for M = N3/2 = 128 with two register<->lane transposes.
//
// The 32-point lane DFT of k_z_prod_warp costs five shuffle stages, each moving every value of
// the row.  Here the length-128 inverse DFT is split into digits n = n0 + 4 n1 + 8 n2 + 32 j
// (n0 = lane bits 0-1, n1 = lane bit 2, n2 = lane bits 3-4, j = register) and run as
//   DFT4 over j (registers), twiddle, transpose j <-> n2, DFT4 over n2, twiddle,
//   radix-2 over n1 (one shuffle stage), twiddle, transpose <-> n0, DFT4 over n0,
// so the lanes exchange 3 + 4 + 3 values instead of 5 x 4.  Each transpose is three shuffles of
// a fixed register from a lane-dependent source: the sending lane's registers are kept rotated
// by its lane digit, which costs nothing because a rotation of a DFT's outputs equals a phase
// i^(j g) on its inputs and the rotation the receiver sees becomes a phase on the next DFT's
// outputs; both phases are folded into the per-lane twiddles t1, t2, except the first input
// phase i^(j n2) and the last output phase i^(kB m), which are exact multiplies by i^p.
// Output layout: lane l, register m holds Z[(l >> 3) + 4 (l & 3) + 16 ((l >> 2) & 1) + 32 m].
// The forward transform is the adjoint network (reverse order, conjugate factors) and returns
// natural order.  Index map and factors are those of a CPU emulation checked against an FFT.
// ------------------------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ cx<R> cmul_unit(cx<R> a, cx<R> c) {
  return mkc<R>(c.x * a.x - c.y * a.y, c.x * a.y + c.y * a.x);
}
// i^p exactly (p taken mod 4)
template <typename R>
__device__ __forceinline__ cx<R> ipow_c(int p) {
  p &= 3;
  return mkc<R>(p == 0 ? (R)1 : (p == 2 ? (R)-1 : (R)0), p == 1 ? (R)1 : (p == 3 ? (R)-1 : (R)0));
}

template <typename R>
struct Net128 {
  cx<R> t1[4], t2[4], w8, ca, cb;
  R sa, sb;  // ca^2, cb^2 (+-1)
  int lane;
  // twN[k] = e^{-i pi k / 128}, k < 256; W_N^e (sign +) = conj(twN[(256 / N) e mod 256])
  __device__ __forceinline__ void init(const cx<double>* twN, int l) {
    lane = l;
    const int g0 = l & 3, c2 = (l >> 2) & 1, g3 = l >> 3;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int kA = (r + g3) & 3;
      t1[r] = cmul_unit(conjc(cvt<R>(twN[(2 * l * kA) & 255])), ipow_c<R>(-r * g0));
      const int kB = (r + g0) & 3;
      t2[r] = cmul_unit(conjc(cvt<R>(twN[(8 * (l & 7) * kB) & 255])), ipow_c<R>(g3 * (r + g0)));
    }
    w8 = conjc(cvt<R>(twN[(32 * g0 * c2) & 255]));
    ca = ipow_c<R>(g3);
    cb = ipow_c<R>(g0);
    sa = (g3 & 1) ? (R)-1 : (R)1;
    sb = (g0 & 1) ? (R)-1 : (R)1;
  }
  // v[j] *= i^(j n2) (before inv), v[j] *= i^(-j n2) (after fwd)
  __device__ __forceinline__ void phase_in(cx<R> (&v)[4], bool conj) const {
    const cx<R> c = conj ? conjc(ca) : ca;
    v[1] = cmul_unit(v[1], c);
    v[2] = sa * v[2];
    v[3] = cmul_unit(v[3], conjc(c));
  }
  // inverse (sign +) DFT of the row in natural order -> permuted order
  __device__ __forceinline__ void inv(cx<R> (&v)[4]) const {
    DFT<4, +1, R>::run(v);
#pragma unroll
    for (int r = 0; r < 4; ++r) v[r] = v[r] * t1[r];
    const int g3 = lane >> 3, g0 = lane & 3;
    {
      const cx<R> z1 = shfl_c(v[1], (lane & 7) | (((g3 - 1) & 3) << 3));
      const cx<R> z2 = shfl_c(v[2], (lane & 7) | (((g3 - 2) & 3) << 3));
      const cx<R> z3 = shfl_c(v[3], (lane & 7) | (((g3 - 3) & 3) << 3));
      v[1] = z1;
      v[2] = z2;
      v[3] = z3;
    }
    DFT<4, -1, R>::run(v);
#pragma unroll
    for (int r = 0; r < 4; ++r) v[r] = v[r] * t2[r];
    const R sg = (lane & 4) ? (R)-1 : (R)1;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const cx<R> p = shfl_xor_c(v[k], 4);
      v[k] = mkc<R>(fma(sg, v[k].x, p.x), fma(sg, v[k].y, p.y)) * w8;
    }
    {
      const cx<R> z1 = shfl_c(v[1], (lane & ~3) | ((g0 - 1) & 3));
      const cx<R> z2 = shfl_c(v[2], (lane & ~3) | ((g0 - 2) & 3));
      const cx<R> z3 = shfl_c(v[3], (lane & ~3) | ((g0 - 3) & 3));
      v[1] = z1;
      v[2] = z2;
      v[3] = z3;
    }
    DFT<4, -1, R>::run(v);
    v[1] = cmul_unit(v[1], cb);
    v[2] = sb * v[2];
    v[3] = cmul_unit(v[3], conjc(cb));
  }
  // forward (sign -) DFT: the adjoint of inv, permuted order -> natural order
  __device__ __forceinline__ void fwd(cx<R> (&v)[4]) const {
    v[1] = cmul_unit(v[1], conjc(cb));
    v[2] = sb * v[2];
    v[3] = cmul_unit(v[3], cb);
    DFT<4, +1, R>::run(v);
    const int g3 = lane >> 3, g0 = lane & 3;
    {
      const cx<R> z1 = shfl_c(v[1], (lane & ~3) | ((g0 + 1) & 3));
      const cx<R> z2 = shfl_c(v[2], (lane & ~3) | ((g0 + 2) & 3));
      const cx<R> z3 = shfl_c(v[3], (lane & ~3) | ((g0 + 3) & 3));
      v[1] = z1;
      v[2] = z2;
      v[3] = z3;
    }
    const R sg = (lane & 4) ? (R)-1 : (R)1;
    const cx<R> w8c = conjc(w8);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const cx<R> sv = v[k] * w8c;
      const cx<R> p = shfl_xor_c(sv, 4);
      v[k] = mkc<R>(fma(sg, sv.x, p.x), fma(sg, sv.y, p.y));
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) v[r] = v[r] * conjc(t2[r]);
    DFT<4, +1, R>::run(v);
    {
      const cx<R> z1 = shfl_c(v[1], (lane & 7) | (((g3 + 1) & 3) << 3));
      const cx<R> z2 = shfl_c(v[2], (lane & 7) | (((g3 + 2) & 3) << 3));
      const cx<R> z3 = shfl_c(v[3], (lane & 7) | (((g3 + 3) & 3) << 3));
      v[1] = z1;
      v[2] = z2;
      v[3] = z3;
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) v[r] = v[r] * conjc(t1[r]);
    DFT<4, -1, R>::run(v);
  }
};

// 16-byte asynchronous global -> shared copies (completion waited with cp.async.wait_group)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(smem)), "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// PF = 1: the warp's next row is copied into shared memory (cp.async, np entries per input)
// while the products of the current row are transformed, so the inverse transforms read their
// inputs from shared memory instead of waiting on global loads.  Requires row strides and
// input pointers on 16-byte boundaries (the launcher checks) and sizeof(Ri) == sizeof(Rw).
template <typename Ri, typename Ro, typename Rw, int NIN, int NPROD, int WPB, int PF>
__global__ void __launch_bounds__(32 * WPB, sizeof(Rw) == 8 ? 4 : 6)
    k_z_prod_net128(ZArgs a, PtrSet ps, ProdPairs pp, int np) {
  constexpr int M = 128, E = 4;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const size_t warp_bytes = (size_t)NIN * E * 32 * sizeof(cx<Rw>) + (PF ? (size_t)NIN * np * sizeof(cx<Ri>) : 0);
  unsigned char* wbase = smem_raw + (size_t)wib * warp_bytes;
  cx<Rw>* rs = reinterpret_cast<cx<Rw>*>(wbase);
  cx<Ri>* ib = reinterpret_cast<cx<Ri>*>(wbase + (size_t)NIN * E * 32 * sizeof(cx<Rw>));
  Net128<Rw> net;
  net.init(a.twN, lane);
  cx<Rw> hw[E];
#pragma unroll
  for (int j = 0; j < E; ++j) hw[j] = cvt<Rw>(a.twN[lane + 32 * j]);
  const Rw sc = (Rw)a.scale;
  const long long nwarps = (long long)gridDim.x * WPB;
  // copy row `row` of every input into ib (16-byte chunks of the first nin entries)
  const int chunks = (int)(((size_t)a.nin * sizeof(cx<Ri>) + 15) / 16);
  auto prefetch = [&](long long row) {
#pragma unroll 1
    for (int c = 0; c < NIN; ++c) {
      const unsigned char* g = reinterpret_cast<const unsigned char*>(ps.src[c]) + (size_t)row * a.ss * sizeof(cx<Ri>);
      unsigned char* d = reinterpret_cast<unsigned char*>(ib + (size_t)c * np);
      for (int t = lane; t < chunks; t += 32) cp_async16(d + 16 * t, g + 16 * t);
    }
    cp_async_commit();
  };
  long long row = (long long)blockIdx.x * WPB + wib;
  if (PF && row < a.nrows) prefetch(row);
  for (; row < a.nrows; row += nwarps) {
    if (PF) {
      cp_async_wait_all();
      __syncwarp();
    }
    // ---- inverse (c2r) of every input
#pragma unroll 1
    for (int c = 0; c < NIN; ++c) {
      const cx<Ri>* src = PF ? ib + (size_t)c * np : reinterpret_cast<const cx<Ri>*>(ps.src[c]) + row * a.ss;
      cx<Rw> v[E];
#pragma unroll
      for (int j = 0; j < E; ++j) {
        const int k = lane + 32 * j;
        cx<Rw> xa = (k < a.nin) ? cvt<Rw>(src[k]) : mkc<Rw>(0, 0);
        const int km = M - k;
        cx<Rw> xb = (km < a.nin) ? cvt<Rw>(src[km]) : mkc<Rw>(0, 0);
        if (k == 0) {
          xa.y = 0;
          xb.y = 0;
        }
        xb.y = -xb.y;
        v[j] = (xa + xb) + ione(conjc(hw[j]) * (xa - xb));
      }
      net.phase_in(v, false);
      net.inv(v);
#pragma unroll
      for (int k1 = 0; k1 < E; ++k1) rs[(c * E + k1) * 32 + lane] = v[k1];
    }
    if (PF) {
      __syncwarp();  // every lane has read this row's inputs
      if (row + nwarps < a.nrows) prefetch(row + nwarps);
    }
    // ---- products and forward (r2c); unrolled in FP32 (fewer issued instructions, no spills
    // at the 80-register bound: z-pass 209 -> 200 us at 256^3), rolled in FP64 (no gain there)
#pragma unroll (sizeof(Rw) == 4 ? NPROD : 1)
    for (int q = 0; q < NPROD; ++q) {
      const int pa = pp.a[q], pb = pp.b[q];
      cx<Rw> v[E];
#pragma unroll
      for (int k1 = 0; k1 < E; ++k1) v[k1] = rmul(rs[(pa * E + k1) * 32 + lane], rs[(pb * E + k1) * 32 + lane]);
      net.fwd(v);
      net.phase_in(v, true);
      cx<Ro>* dst = reinterpret_cast<cx<Ro>*>(ps.dst[q]) + row * a.ds;
      const int pl = (32 - lane) & 31;
#pragma unroll
      for (int j = 0; j < E; ++j) {
        cx<Rw> zm = shfl_c(v[E - 1 - j], pl);
        if (lane == 0) zm = v[(E - j) % E];
        zm.y = -zm.y;
        const cx<Rw> s = v[j] + zm;
        const cx<Rw> d = hw[j] * (v[j] - zm);
        const int k = lane + 32 * j;
        if (k < a.nout) dst[k] = cvt<Ro>(mkc<Rw>(sc * (Rw)0.5 * (s.x + d.y), sc * (Rw)0.5 * (s.y - d.x)));
      }
      if (lane == 0 && a.nout > M) dst[M] = cvt<Ro>(mkc<Rw>(sc * (v[0].x - v[0].y), (Rw)0));
      for (int k = a.nout + lane; k < a.nfill; k += 32) dst[k] = mkc<Ro>(0, 0);
    }
  }
  if (PF) cp_async_wait_all();
}

}  // namespace tg
