// The SCFT x-pass contraction Y[m][c] = scale * sum_k T[k][m] X[k][c] (T real, X complex) on the
// 5th-generation tensor cores, for the FP32 forms: 3xTF32 (T = Th + Tl, X = Xh + Xl split into
// TF32 pairs, Y ~ Th Xh + Th Xl + Tl Xh, FP32 accumulation), the sine/cosine transforms of
// scft_tr.cc:440-639 as in k_axis_r2r_gemm.
//
// The complex columns are read as real ones (re, im interleaved): a tile is 128 real columns, the
// MMA's M dimension (A = the tile transposed, 128 x K, its columns contiguous in memory: MN-major);
// the output rows are the MMA's N dimension (B = T, N x K, padded to a multiple of 16, MN-major);
// the accumulator D [128 lanes][N columns] lives in tensor memory.  Operands are split into TF32
// pairs by the threads and written to shared memory in the canonical no-swizzle MN-major layout:
// element (row r, k) of an R-row operand at float offset ((k / 8) (R / 4) + r / 4) 32 + (k % 8) 4
// + r % 4 (core matrices of 4 rows x 8 k, 128 bytes; the stride between row groups, SBO, is 128
// bytes, between k groups, LBO, R * 32 bytes).  One thread issues the MMAs (tcgen05.mma
// cta_group::1 kind::tf32, M = 128, K = 8 per instruction) and commits them to an mbarrier; the
// K dimension runs in chunks of 32 through two shared-memory buffers, so the threads fill one while
// the tensor cores read the other.  The epilogue reads tensor memory with tcgen05.ld (warp w owns
// lanes 32 w .. 32 w + 31, the columns of its quarter of the tile) and stores each output row's
// 128 columns coalesced.  Every wait on an mbarrier is bounded: past the limit the block records
// the failure in the context's status word (TG_ERR_TIMEOUT on the host), waits again (bounded) for
// its committed MMAs, frees its tensor memory and returns.
#pragma once

#include "tg_fft.cuh"
#include "tg_tma.cuh"

namespace tg {

constexpr int kTcKC = 32;          // K rows per shared-memory chunk
constexpr int kTcPolls = 1 << 22;  // bounded mbarrier waits

// the TF32 part of x: rounded to the nearest 10-bit mantissa and the 13 lower bits cleared, so
// that x - hi is exact (the tensor cores read only the upper 19 bits of each operand)
__device__ __forceinline__ float tf32_hi(float x) {
  uint32_t u = __float_as_uint(x);
  if ((u & 0x7f800000u) != 0x7f800000u) u += 0x1000u;
  return __uint_as_float(u & 0xffffe000u);
}

// shared-memory matrix descriptor, no swizzle (tcgen05 version 1): start, LBO, SBO in bytes
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // version
  return d;                // base offset 0, LBO mode 0, layout type 0 (no swizzle)
}

// instruction descriptor: D F32, A and B TF32, both MN-major, M = 128, N = n
__device__ __forceinline__ uint32_t tc_idesc(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | (1u << 15) | (1u << 16) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, int acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void tc_mbar_init(uint32_t mbar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

// wait until the phase of the given parity has completed; false past the poll limit
__device__ __forceinline__ bool tc_mbar_wait(uint32_t mbar, uint32_t parity, int polls) {
  for (int i = 0; i <= polls; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive accumulator columns of this thread's lane
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// float offset of element (row r, k) of an R-row MN-major no-swizzle operand
__device__ __forceinline__ int tc_off(int r, int k, int R) { return ((k >> 3) * (R >> 2) + (r >> 2)) * 32 + (k & 7) * 4 + (r & 3); }

struct TcArgs {
  int npad;        // output rows padded to a multiple of 16 (MMA N)
  int kpad;        // input rows padded to a multiple of 8
  int tmem_cols;   // tensor-memory columns allocated (a power of two >= 32, >= npad)
  int ntiles;      // 128-real-column tiles per batch row (ceil(2 ncols / 128))
};

// grid (P, nbatch, nfields): block (x, b, f) takes the tiles x, x + P, ... of batch b, field f
template <typename Ri>
__global__ void __launch_bounds__(128, 1) k_axis_r2r_tc(AxisArgs a, PtrSet ps, R2RArgs r, TcArgs t) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int f = blockIdx.z, b = blockIdx.y;
  const int kind = r.kind[f];
  const int nrows = r.mat_rows[kind], nin = r.mat_cols[kind];
  const double* M = r.mat[kind];
  const int NP = t.npad, KP = t.kpad;
  float* Bh = reinterpret_cast<float*>(smem_raw);
  float* Bl = Bh + NP * KP;
  float* Abuf = Bl + NP * KP;  // [2 buffers][hi, lo][128 x kKC]
  constexpr int ACH = 128 * kTcKC;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(Abuf + 4 * ACH);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 2);
  int* flag = reinterpret_cast<int*>(tmem_slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // B = T split into TF32 pairs, zero beyond nrows and nin
  for (int i = tid; i < NP * KP; i += 128) {
    const int k = i / NP, m = i - k * NP;
    const float v = (k < nin && m < nrows) ? (float)M[(size_t)k * nrows + m] : 0.0f;
    const float h = tf32_hi(v);
    const int o = tc_off(m, k, NP);
    Bh[o] = h;
    Bl[o] = v - h;
  }
  if (tid == 0) {
    tc_mbar_init(smem_u32(&mbar[0]), 1);
    tc_mbar_init(smem_u32(&mbar[1]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *flag = 1;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(t.tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  proxy_fence();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = tc_idesc(NP);
  const uint32_t bh = smem_u32(Bh), bl = smem_u32(Bl);
  const uint32_t lbo_b = (uint32_t)NP * 32, lbo_a = 128 * 32;
  const long long ncr = 2LL * a.ncols;  // real columns
  const Ri* src = reinterpret_cast<const Ri*>(ps.src[f]) + (long long)b * a.sb * 2;
  float* dst = reinterpret_cast<float*>(ps.dst[f]) + (long long)b * a.db * 2;
  const long long srr = 2 * a.sr, drr = 2 * a.dr;  // real strides of the rows
  const float sc = (float)a.scale;
  uint32_t uses[2] = {0, 0};  // commits issued to each buffer's mbarrier
  bool ok = true;
  int chunk = 0;
  const int nkc = (KP + kTcKC - 1) / kTcKC;
  for (int tile = blockIdx.x; tile < t.ntiles && ok; tile += gridDim.x) {
    const long long c0 = (long long)tile * 128;
    for (int kc = 0; kc < nkc && ok; ++kc, ++chunk) {
      const int buf = chunk & 1;
      const int k0 = kc * kTcKC, kn = min(kTcKC, KP - k0);
      // the buffer's previous MMAs must have read it
      if (uses[buf] > 0) {
        if (tid == 0 && !tc_mbar_wait(smem_u32(&mbar[buf]), (uses[buf] - 1) & 1, kTcPolls)) *flag = 0;
        __syncthreads();
        ok = *flag != 0;
        if (!ok) break;
      }
      float* Ah = Abuf + (size_t)buf * 2 * ACH;
      float* Al = Ah + ACH;
      // unit u = (k group g, 4-column group quad q of 4): lane = 8 x (quad in unit) + k within group
      const int units = (kn >> 3) * 8;  // k groups x 8 units of 4 x 4 columns
      for (int u = warp; u < units; u += 4) {
        const int g = u >> 3, q = (u & 7) * 4 + (lane >> 3), kk = g * 8 + (lane & 7);
        const int k = k0 + kk;
        const long long c = c0 + q * 4;
        float v[4] = {0.f, 0.f, 0.f, 0.f};
        if (k < nin) {
          const Ri* p = src + (long long)k * srr + c;
          if (c + 4 <= ncr) {
            // rows start on 16-element boundaries (row strides are multiples of 8 complex)
            if constexpr (sizeof(Ri) == 4) {
              const float4 w = *reinterpret_cast<const float4*>(p);
              v[0] = w.x, v[1] = w.y, v[2] = w.z, v[3] = w.w;
            } else {
              const double2 w0 = reinterpret_cast<const double2*>(p)[0], w1 = reinterpret_cast<const double2*>(p)[1];
              v[0] = (float)w0.x, v[1] = (float)w0.y, v[2] = (float)w1.x, v[3] = (float)w1.y;
            }
          } else {
#pragma unroll
            for (int e = 0; e < 4; ++e)
              if (c + e < ncr) v[e] = (float)p[e];
          }
        }
        const int o = tc_off(q * 4, kk, 128);
        float4 h, l;
        h.x = tf32_hi(v[0]);
        h.y = tf32_hi(v[1]);
        h.z = tf32_hi(v[2]);
        h.w = tf32_hi(v[3]);
        l.x = v[0] - h.x;
        l.y = v[1] - h.y;
        l.z = v[2] - h.z;
        l.w = v[3] - h.w;
        *reinterpret_cast<float4*>(Ah + o) = h;
        *reinterpret_cast<float4*>(Al + o) = l;
      }
      proxy_fence();
      __syncthreads();
      if (tid == 0) {
        tc_fence_after();
        const uint32_t ah = smem_u32(Ah), al = smem_u32(Al);
        for (int s = 0; s < (kn >> 3); ++s) {
          const int kg = (k0 >> 3) + s;  // k group of B
          const uint64_t dah = tc_desc(ah + (uint32_t)s * lbo_a, lbo_a, 128);
          const uint64_t dal = tc_desc(al + (uint32_t)s * lbo_a, lbo_a, 128);
          const uint64_t dbh = tc_desc(bh + (uint32_t)kg * lbo_b, lbo_b, 128);
          const uint64_t dbl = tc_desc(bl + (uint32_t)kg * lbo_b, lbo_b, 128);
          const int first = (kc == 0 && s == 0) ? 0 : 1;
          tc_mma(tmem, dal, dbh, idesc, first);
          tc_mma(tmem, dah, dbl, idesc, 1);
          tc_mma(tmem, dah, dbh, idesc, 1);
        }
        tc_commit(smem_u32(&mbar[buf]));
      }
      uses[buf] += 1;
    }
    if (!ok) break;
    // the tile's last commit covers every MMA of the tile
    {
      const int lb = (chunk - 1) & 1;
      if (tid == 0 && !tc_mbar_wait(smem_u32(&mbar[lb]), (uses[lb] - 1) & 1, kTcPolls)) *flag = 0;
      __syncthreads();
      ok = *flag != 0;
      if (!ok) break;
      tc_fence_after();
    }
    // epilogue: lane 32 warp + lane is real column c0 + 32 warp + lane
    const long long col = c0 + warp * 32 + lane;
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
    for (int j0 = 0; j0 < NP; j0 += 16) {
      float v[16];
      tc_ld16(trow + (uint32_t)j0, v);
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int m = j0 + j;
        if (m < nrows && col < ncr) dst[(long long)m * drr + col] = sc * v[j];
      }
    }
    tc_fence_before();
    __syncthreads();
  }
  if (!ok) {
    if (tid == 0) {
      if (a.wait_flag) atomicExch(a.wait_flag, 1);
      // let the committed MMAs finish before the tensor memory is freed
      for (int bb = 0; bb < 2; ++bb)
        if (uses[bb] > 0) tc_mbar_wait(smem_u32(&mbar[bb]), (uses[bb] - 1) & 1, kTcPolls);
    }
    __syncthreads();
  }
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(t.tmem_cols) : "memory");
}

}  // namespace tg
