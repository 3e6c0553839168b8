// The SCFT x-pass contraction Y[m][c] = scale * sum_k T[k][m] X[k][c] (T real, X complex) on the
// 5th-generation tensor cores, for the FP32 forms: 3xTF32 (T = Th + Tl, X = Xh + Xl split into
// TF32 pairs, Y ~ Th Xh + Th Xl + Tl Xh, FP32 accumulation), the sine/cosine transforms of
// scft_tr.cc:440-639 as in k_axis_r2r_gemm.
//
// The complex columns are read as real ones (re, im interleaved): a tile is 128 real columns, the
// MMA's M dimension (A = the tile transposed, 128 x K); the output rows are the MMA's N dimension
// (B = T, N x K, padded to a multiple of 16); the accumulator D [128 lanes][N columns] lives in
// tensor memory.  Operands are split into TF32 pairs by the threads and written to shared memory
// in the canonical no-swizzle K-major layout: element (row r, k) of an operand with KW k per row
// at float offset (r % 8) 4 + k % 4 + (k / 4) 32 + (r / 8) (KW / 4) 32 (core matrices of 8 rows x 4
// k, 128 bytes; the stride between k chunks of 4, LBO, is 128 bytes, between groups of 8 rows,
// SBO, KW * 32 bytes).  (With tcgen05 kind::tf32 the MN-major no-swizzle form returned zeros on
// B200; the K-major form is exact.)
//
// The block is warp-specialised and every hand-off is an mbarrier:
//   converter warps (8)  read each K chunk (32 rows x 128 columns) straight from global memory
//                        into registers several chunks ahead (coalesced: a warp reads 32
//                        consecutive columns of a row), split them into TF32 pairs and write the
//                        operand ring (NA slots), one arrival per thread -> op_full[slot]
//   MMA warp (1 thread)  waits op_full, issues the chunk's MMAs (tcgen05.mma cta_group::1
//                        kind::tf32, M = 128, K = 8 each) into one of two accumulators and commits
//                        them to op_empty[slot]; after a tile's last chunk it commits acc_full
//   epilogue warps (4)   wait acc_full, read the accumulator with tcgen05.ld (warp w: lanes
//                        32 w .. 32 w + 31, one column each) and store each output row's 128
//                        columns coalesced, then release the accumulator (acc_empty)
// so the loads of later chunks, the MMAs of the current one and the stores of the previous tile
// overlap; the bytes in flight per SM are the converters' register ring, not shared memory,
// which the coefficient pairs and the operand ring fill.  Every wait is bounded: past the limit
// the thread records the failure in the context's status word (TG_ERR_TIMEOUT on the host) and a
// block-wide abort flag that ends the other roles' waits; the MMA thread then waits (bounded) for
// its issued MMAs before the tensor memory is freed.
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

// instruction descriptor: D F32, A and B TF32, both K-major, M = 128, N = n
__device__ __forceinline__ uint32_t tc_idesc(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
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

// float offset of element (row r, k) of a K-major no-swizzle operand with KW k per row (KW % 4 == 0)
__device__ __forceinline__ int tc_off(int r, int k, int KW) {
  return (r & 7) * 4 + (k & 3) + (k >> 2) * 32 + (r >> 3) * (KW >> 2) * 32;
}


struct TcArgs {
  int npad;        // output rows padded to a multiple of 16 (MMA N)
  int kpad;        // input rows padded to a multiple of 8
  int tmem_cols;   // tensor-memory columns of one accumulator (a power of two >= 32, >= npad)
  int ntiles;      // 128-real-column tiles per batch row (ceil(2 ncols / 128))
  int nab;         // operand ring slots
};

constexpr int kTcEpiWarps = 4;   // warps 0-3: epilogue
constexpr int kTcMmaWarp = 4;    // warp 4: tensor-memory allocation and the MMA thread
constexpr int kTcCvtWarps = 8;   // warps 5-12: converters
constexpr int kTcThreads = 32 * (kTcEpiWarps + 1 + kTcCvtWarps);
constexpr int kTcMaxNab = 3;
// the first converter warp asks L2 for the rows of the chunk this many chunks ahead of the one it
// loads into registers (0: no prefetch)
#ifndef TG_TC_PREFETCH
#define TG_TC_PREFETCH 8
#endif
constexpr int kTcPrefetch = TG_TC_PREFETCH;
// chunks each converter thread holds in registers ahead of the one it splits (16 values per chunk)
template <typename Ri>
struct TcRing {
#ifndef TG_TC_RING32
#define TG_TC_RING32 5
#define TG_TC_RING64 3
#endif
  static constexpr int D = sizeof(Ri) == 4 ? TG_TC_RING32 : TG_TC_RING64;
};

// bounded wait that also ends when another role has aborted the block; false on either
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag, int* wait_flag) {
  for (int i = 0; i <= kTcPolls; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if ((i & 31) == 31 && *abort_flag) return false;
  }
  *abort_flag = 1;
  if (wait_flag) atomicExch(wait_flag, 1);
  return false;
}

__device__ __forceinline__ void tc_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// grid (P, nbatch, nfields): block (x, b, f) takes the tiles x, x + P, ... of batch b, field f.
template <typename Ri>
__global__ void __launch_bounds__(kTcThreads, 1) k_axis_r2r_tc(AxisArgs a, PtrSet ps, R2RArgs r, TcArgs t) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int D = TcRing<Ri>::D;
  constexpr int ACH = 128 * kTcKC;  // floats of one operand (hi or lo) chunk
  const int f = blockIdx.z, b = blockIdx.y;
  const int kind = r.kind[f];
  const int nrows = r.mat_rows[kind], nin = r.mat_cols[kind];
  const double* M = r.mat[kind];
  const int NP = t.npad, KP = t.kpad, NA = t.nab, TC = t.tmem_cols;
  float* Bh = reinterpret_cast<float*>(smem_raw);
  float* Bl = Bh + NP * KP;
  float* Abase = Bl + NP * KP;  // NA slots of [hi, lo] chunks
  uint64_t* op_full = reinterpret_cast<uint64_t*>(Abase + 2 * (size_t)NA * ACH);
  uint64_t* op_empty = op_full + kTcMaxNab;
  uint64_t* acc_full = op_empty + kTcMaxNab;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* done_bar = acc_empty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done_bar + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  for (int i = tid; i < NP * KP; i += kTcThreads) {
    const int k = i / NP, m = i - k * NP;
    const float v = (k < nin && m < nrows) ? (float)M[(size_t)k * nrows + m] : 0.0f;
    const float h = tf32_hi(v);
    const int o = tc_off(m, k, KP);
    Bh[o] = h;
    Bl[o] = v - h;
  }
  if (tid == 0) {
    for (int s = 0; s < kTcMaxNab; ++s) {
      tc_mbar_init(smem_u32(&op_full[s]), 32 * kTcCvtWarps);
      tc_mbar_init(smem_u32(&op_empty[s]), 1);
    }
    for (int s = 0; s < 2; ++s) {
      tc_mbar_init(smem_u32(&acc_full[s]), 1);
      tc_mbar_init(smem_u32(&acc_empty[s]), 32 * kTcEpiWarps);
    }
    tc_mbar_init(smem_u32(done_bar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *abort_flag = 0;
  }
  if (warp == kTcMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(2 * TC)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  proxy_fence();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const long long ncr = 2LL * a.ncols;  // real columns
  const int nkc = (KP + kTcKC - 1) / kTcKC;
  const int P = (int)gridDim.x;
  const int my_tiles = (t.ntiles - (int)blockIdx.x + P - 1) / P;
  const int nchunks = my_tiles * nkc;
  int* wflag = a.wait_flag;

  if (warp >= kTcMmaWarp + 1) {
    // ---- converters: thread (column cl, k half kh) of each chunk, D chunks in registers
    const int ct = tid - 32 * (kTcMmaWarp + 1);
    const int cl = ct & 127, kh = ct >> 7;
    const Ri* src = reinterpret_cast<const Ri*>(ps.src[f]) + (long long)b * a.sb * 2;
    const long long srr = 2 * a.sr;
    Ri v[D][16];
    // chunk i's 16 values of this thread into v[slot]
#define TC_LOAD(i, slot)                                                                    \
  do {                                                                                      \
    const int tile_ = (int)blockIdx.x + ((i) / nkc) * P;                                    \
    const long long col_ = (long long)tile_ * 128 + cl;                                     \
    const int k0_ = ((i) % nkc) * kTcKC + kh * 16;                                          \
    const bool cin_ = col_ < ncr;                                                           \
    const Ri* p_ = src + (long long)k0_ * srr + col_;                                       \
    _Pragma("unroll") for (int j = 0; j < 16; ++j) v[slot][j] =                             \
        (cin_ && k0_ + j < nin) ? p_[(long long)j * srr] : (Ri)0;                           \
  } while (0)
#pragma unroll
    for (int d = 0; d < D - 1; ++d)
      if (d < nchunks) TC_LOAD(d, d);
    bool ok = true;
    for (int i0 = 0; i0 < nchunks && ok; i0 += D) {
#pragma unroll
      for (int d = 0; d < D; ++d) {
        const int i = i0 + d;
        if (i < nchunks && ok) {
          if (i + D - 1 < nchunks) TC_LOAD(i + D - 1, (d + D - 1) % D);
          if (kTcPrefetch > 0 && ct < 32 && i + D - 1 + kTcPrefetch < nchunks) {
            // lane j: row j of that chunk, its 128 columns (four 128-byte lines at most)
            const int ip = i + D - 1 + kTcPrefetch;
            const int tile_p = (int)blockIdx.x + (ip / nkc) * P;
            const int kp = (ip % nkc) * kTcKC + ct;
            const long long c0p = (long long)tile_p * 128;
            if (kp < nin && c0p < ncr) {
              const char* rp = reinterpret_cast<const char*>(src + (long long)kp * srr + c0p);
              const long long nb = min(128LL, ncr - c0p) * (long long)sizeof(Ri);
              for (long long o = 0; o < nb; o += 128) asm volatile("prefetch.global.L2 [%0];" ::"l"(rp + o));
              asm volatile("prefetch.global.L2 [%0];" ::"l"(rp + nb - 1));
            }
          }
          const int s = i % NA;
          // the whole warp takes one decision (the split ends in warp-wide steps)
          const bool free_slot =
              __all_sync(0xffffffffu, i < NA || tc_wait(smem_u32(&op_empty[s]), (uint32_t)(((i / NA) - 1) & 1),
                                                         abort_flag, wflag));
          if (!free_slot) {
            ok = false;
          } else {
            float* Ah = Abase + (size_t)s * 2 * ACH;
            float* Al = Ah + ACH;
            const int kq0 = (i % nkc) * kTcKC + kh * 16;  // first k of this thread's 16
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              if (kq0 + 4 * q < KP) {
                const int o = tc_off(cl, kh * 16 + 4 * q, kTcKC);
                float4 h, l;
                const float x0 = (float)v[d][4 * q], x1 = (float)v[d][4 * q + 1];
                const float x2 = (float)v[d][4 * q + 2], x3 = (float)v[d][4 * q + 3];
                h.x = tf32_hi(x0);
                h.y = tf32_hi(x1);
                h.z = tf32_hi(x2);
                h.w = tf32_hi(x3);
                l.x = x0 - h.x;
                l.y = x1 - h.y;
                l.z = x2 - h.z;
                l.w = x3 - h.w;
                *reinterpret_cast<float4*>(Ah + o) = h;
                *reinterpret_cast<float4*>(Al + o) = l;
              }
            }
            // each thread's writes reach the tensor cores' (async) proxy before its arrival
            proxy_fence();
            tc_arrive(smem_u32(&op_full[s]));
          }
        }
      }
    }
#undef TC_LOAD
  } else if (warp == kTcMmaWarp) {
    // ---- the MMA thread
    if (lane == 0) {
      const uint32_t idesc = tc_idesc(NP);
      const uint32_t sbo_b = (uint32_t)KP * 32, sbo_a = kTcKC * 32;  // bytes between 8-row groups
      // descriptors of k group 0; a step of 256 bytes (8 k) adds 16 to the start-address field
      // (address / 16, 14 bits: shared-memory addresses stay below 256 KB, so no carry)
      const uint64_t dbh0 = tc_desc(smem_u32(Bh), 128, sbo_b), dbl0 = tc_desc(smem_u32(Bl), 128, sbo_b);
      const uint64_t da0 = tc_desc(smem_u32(Abase), 128, sbo_a);
      constexpr uint64_t kSlotStep = (uint64_t)(2 * ACH * sizeof(float)) >> 4, kLoStep = (uint64_t)(ACH * sizeof(float)) >> 4;
      int i = 0;
      bool ok = true;
      for (int lt = 0; lt < my_tiles && ok; ++lt) {
        const int acc = lt & 1;
        if (lt >= 2 && !tc_wait(smem_u32(&acc_empty[acc]), (uint32_t)(((lt >> 1) - 1) & 1), abort_flag, wflag)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t dt = tmem + (uint32_t)(acc * TC);
        for (int kc = 0; kc < nkc; ++kc, ++i) {
          const int s = i % NA;
          if (!tc_wait(smem_u32(&op_full[s]), (uint32_t)((i / NA) & 1), abort_flag, wflag)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const int k0 = kc * kTcKC, kn = min(kTcKC, KP - k0);
          const uint64_t dah0 = da0 + (uint64_t)s * kSlotStep;
          for (int sg = 0; sg < (kn >> 3); ++sg) {
            const int kg = (k0 >> 3) + sg;  // k group of 8 of B
            // two k chunks of 4 per MMA: start at chunk 2 sg (A) / 2 kg (B), 128 bytes each
            const uint64_t dah = dah0 + (uint64_t)sg * 16, dal = dah + kLoStep;
            const uint64_t dbh = dbh0 + (uint64_t)kg * 16, dbl = dbl0 + (uint64_t)kg * 16;
            tc_mma(dt, dal, dbh, idesc, (kc == 0 && sg == 0) ? 0 : 1);
            tc_mma(dt, dah, dbl, idesc, 1);
            tc_mma(dt, dah, dbh, idesc, 1);
          }
          tc_commit(smem_u32(&op_empty[s]));
        }
        if (ok) tc_commit(smem_u32(&acc_full[acc]));
      }
      // every MMA issued has completed before the block goes on to free the tensor memory
      tc_commit(smem_u32(done_bar));
      tc_mbar_wait(smem_u32(done_bar), 0, kTcPolls);
    }
    __syncwarp();
  } else {
    // ---- epilogue: warp w reads lanes 32 w .. 32 w + 31 (columns c0 + 32 w + lane)
    float* dst = reinterpret_cast<float*>(ps.dst[f]) + (long long)b * a.db * 2;
    const long long drr = 2 * a.dr;
    const float sc = (float)a.scale;
    for (int lt = 0; lt < my_tiles; ++lt) {
      const int acc = lt & 1;
      // one decision per warp: tcgen05.ld is warp-wide
      if (!__all_sync(0xffffffffu, tc_wait(smem_u32(&acc_full[acc]), (uint32_t)((lt >> 1) & 1), abort_flag, wflag)))
        break;
      tc_fence_after();
      const int tile = (int)blockIdx.x + lt * P;
      const long long col = (long long)tile * 128 + warp * 32 + lane;
      const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(acc * TC);
      for (int j0 = 0; j0 < NP; j0 += 16) {
        float w[16];
        tc_ld16(trow + (uint32_t)j0, w);
        if (col < ncr) {
#pragma unroll
          for (int j = 0; j < 16; ++j)
            if (j0 + j < nrows) dst[(long long)(j0 + j) * drr + col] = sc * w[j];
        }
      }
      tc_fence_before();
      tc_arrive(smem_u32(&acc_empty[acc]));
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == kTcMmaWarp)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * TC) : "memory");
}

}  // namespace tg
