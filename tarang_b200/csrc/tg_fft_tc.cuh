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
// B200; the K-major form is exact.)  The K dimension runs in chunks of 32: a chunk's rows arrive
// by untiled bulk copies (cp.async.bulk, no multicast) two chunks ahead in two staging buffers,
// the threads split them into one of two operand buffers, and one thread issues the chunk's MMAs
// (tcgen05.mma cta_group::1 kind::tf32, M = 128, K = 8 per instruction) and commits them to that
// buffer's mbarrier.  The epilogue reads tensor memory with tcgen05.ld (warps w and w + 4 own lanes
// 32 (w % 4) .. + 31, alternate 16-column groups) and stores each output row's 128 columns
// coalesced.  Every wait on an mbarrier is bounded: past the limit the block records the failure
// in the context's status word (TG_ERR_TIMEOUT on the host), waits again (bounded) for its
// committed MMAs and issued copies, frees its tensor memory and returns.
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
  int tmem_cols;   // tensor-memory columns allocated (a power of two >= 32, >= npad)
  int ntiles;      // 128-real-column tiles per batch row (ceil(2 ncols / 128))
};

// one contiguous row segment global -> shared, completion counted in bytes on an mbarrier
__device__ __forceinline__ void bulk_row(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// grid (P, nbatch, nfields): block (x, b, f) takes the tiles x, x + P, ... of batch b, field f.
// Chunk i of the block (tile i / nkc, k rows (i % nkc) kTcKC ..) moves in three steps: its rows
// arrive in staging buffer i % 2 by bulk copies issued two chunks ahead; the threads split them
// into the K-major TF32 pairs of the operand buffer; one thread issues the chunk's MMAs.
// NAB operand buffers (2: the split of chunk i + 1 overlaps the MMAs of chunk i; 1 where shared
// memory is short); 256 threads: thread t splits column t % 128, k half t / 128 of each chunk, and
// warps w and w + 4 read the same tensor-memory lanes, alternate 16-column groups of the accumulator
constexpr int kTcThreads = 256;
template <typename Ri, int NAB>
__global__ void __launch_bounds__(kTcThreads, 1) k_axis_r2r_tc(AxisArgs a, PtrSet ps, R2RArgs r, TcArgs t) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int f = blockIdx.z, b = blockIdx.y;
  const int kind = r.kind[f];
  const int nrows = r.mat_rows[kind], nin = r.mat_cols[kind];
  const double* M = r.mat[kind];
  const int NP = t.npad, KP = t.kpad;
  constexpr int ACH = 128 * kTcKC;
  float* Bh = reinterpret_cast<float*>(smem_raw);
  float* Bl = Bh + NP * KP;
  float* Abase = Bl + NP * KP;  // NAB operand chunks [hi, lo], K-major TF32 pairs
  Ri* stg = reinterpret_cast<Ri*>(Abase + 2 * NAB * ACH);  // [2][kTcKC][128] raw rows
  uint64_t* sbar = reinterpret_cast<uint64_t*>(stg + 2 * ACH);  // staging buffers
  uint64_t* mbar = sbar + 2;  // MMA completion, one per operand buffer (commits of chunks i % NAB)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 2);
  int* flag = reinterpret_cast<int*>(tmem_slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5;

  for (int i = tid; i < NP * KP; i += kTcThreads) {
    const int k = i / NP, m = i - k * NP;
    const float v = (k < nin && m < nrows) ? (float)M[(size_t)k * nrows + m] : 0.0f;
    const float h = tf32_hi(v);
    const int o = tc_off(m, k, KP);
    Bh[o] = h;
    Bl[o] = v - h;
  }
  if (tid == 0) {
    tc_mbar_init(smem_u32(&sbar[0]), 1);
    tc_mbar_init(smem_u32(&sbar[1]), 1);
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
  const uint32_t sbo_b = (uint32_t)KP * 32, sbo_a = kTcKC * 32;  // bytes between 8-row groups
  const long long ncr = 2LL * a.ncols;                             // real columns
  const Ri* src = reinterpret_cast<const Ri*>(ps.src[f]) + (long long)b * a.sb * 2;
  float* dst = reinterpret_cast<float*>(ps.dst[f]) + (long long)b * a.db * 2;
  const long long srr = 2 * a.sr, drr = 2 * a.dr;  // real strides of the rows
  const float sc = (float)a.scale;
  const int nkc = (KP + kTcKC - 1) / kTcKC;
  const int my_tiles = (t.ntiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
  const int nchunks = my_tiles * nkc;

  // thread 0: the bulk copies of chunk i into staging buffer i % 2 (rows k < nin only)
  auto issue = [&](int i) {
    const int tile = (int)blockIdx.x + (i / nkc) * (int)gridDim.x, k0 = (i % nkc) * kTcKC;
    const long long c0 = (long long)tile * 128;
    const int ncol = (int)min(128LL, ncr - c0);
    const int k1 = min(min(k0 + kTcKC, KP), nin);
    const unsigned row_bytes = (unsigned)ncol * sizeof(Ri);
    const unsigned total = k1 > k0 ? (unsigned)(k1 - k0) * row_bytes : 0u;
    uint64_t* bar = &sbar[i & 1];
    if (total == 0) {
      // no stored rows in this chunk: complete the phase by a plain arrival
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
      return;
    }
    mbar_arrive_expect_tx(bar, total);
    Ri* sb = stg + (size_t)(i & 1) * ACH;
    for (int k = k0; k < k1; ++k) bulk_row(sb + (size_t)(k - k0) * 128, src + (long long)k * srr + c0, row_bytes, bar);
  };
  int issued = 0, landed = 0, committed = 0;  // chunks (thread 0's counts)
  // chunk j's MMAs: the (j / NAB)-th completion of mbar[j % NAB], waited before that barrier is
  // committed again, so no barrier runs two phases ahead of its waiter
  if (tid == 0) {
    if (nchunks > 0) issue(0);
    if (nchunks > 1) issue(1);
    issued = min(nchunks, 2);
  }
  bool ok = true;
  for (int i = 0; i < nchunks && ok; ++i) {
    const int tile = (int)blockIdx.x + (i / nkc) * (int)gridDim.x, kc = i % nkc;
    const int k0 = kc * kTcKC, kn = min(kTcKC, KP - k0);
    const long long c0 = (long long)tile * 128;
    // staging i has landed, and the MMAs of chunk i - NAB have read operand buffer i % NAB
    if (tid == 0) {
      if (!tc_mbar_wait(smem_u32(&sbar[i & 1]), (uint32_t)((i >> 1) & 1), kTcPolls)) *flag = 0;
      else landed = i + 1;
      if (*flag && i >= NAB &&
          !tc_mbar_wait(smem_u32(&mbar[i % NAB]), (uint32_t)(((i - NAB) / NAB) & 1), kTcPolls))
        *flag = 0;
    }
    __syncthreads();
    ok = *flag != 0;
    if (!ok) break;
    float* Ah = Abase + (size_t)(i % NAB) * 2 * ACH;
    float* Al = Ah + ACH;
    // split: column c0 + (tid % 128), k quads of half tid / 128, 4 k per float4 of the K-major operand
    {
      const Ri* sb = stg + (size_t)(i & 1) * ACH;
      const int cl = tid & 127, half = tid >> 7;
      const bool cin = c0 + cl < ncr;
      const int nq = kn >> 2, q0 = half * ((nq + 1) >> 1), q1 = min(nq, q0 + ((nq + 1) >> 1));
      for (int kq = q0; kq < q1; ++kq) {
        float v[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int kk = kq * 4 + e;
          v[e] = (cin && k0 + kk < nin) ? (float)sb[(size_t)kk * 128 + cl] : 0.0f;
        }
        const int o = tc_off(cl, kq * 4, kTcKC);
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
    }
    proxy_fence();
    __syncthreads();
    if (tid == 0) {
      // staging buffer i % 2 is free again: chunk i + 2 goes there
      if (i + 2 < nchunks) {
        issue(i + 2);
        issued = i + 3;
      }
      tc_fence_after();
      const uint32_t ah = smem_u32(Ah), al = smem_u32(Al);
      for (int s = 0; s < (kn >> 3); ++s) {
        const int kg = (k0 >> 3) + s;  // k group of 8 of B
        // two k chunks of 4 per MMA: start at chunk 2 s (A) / 2 kg (B), 128 bytes each
        const uint64_t dah = tc_desc(ah + (uint32_t)s * 256, 128, sbo_a);
        const uint64_t dal = tc_desc(al + (uint32_t)s * 256, 128, sbo_a);
        const uint64_t dbh = tc_desc(bh + (uint32_t)kg * 256, 128, sbo_b);
        const uint64_t dbl = tc_desc(bl + (uint32_t)kg * 256, 128, sbo_b);
        const int first = (kc == 0 && s == 0) ? 0 : 1;
        tc_mma(tmem, dal, dbh, idesc, first);
        tc_mma(tmem, dah, dbl, idesc, 1);
        tc_mma(tmem, dah, dbh, idesc, 1);
      }
      tc_commit(smem_u32(&mbar[i % NAB]));
      committed = i + 1;
    }
    if (kc == nkc - 1) {
      // the tile's last chunk: its MMAs done, the accumulator out
      if (tid == 0 && !tc_mbar_wait(smem_u32(&mbar[i % NAB]), (uint32_t)((i / NAB) & 1), kTcPolls)) *flag = 0;
      __syncthreads();
      ok = *flag != 0;
      if (!ok) break;
      tc_fence_after();
      const long long col = c0 + (warp & 3) * 32 + (tid & 31);
      const uint32_t trow = tmem + ((uint32_t)((warp & 3) * 32) << 16);
      for (int j0 = (warp >> 2) * 16; j0 < NP; j0 += 32) {
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
      // the wait at the top of chunk i + 1 for this chunk's MMAs passes at once: phase i done
    }
  }
  if (!ok) {
    if (tid == 0) {
      if (a.wait_flag) atomicExch(a.wait_flag, 1);
      // let the committed MMAs and the issued copies finish before the block's memory goes away
      for (int j = max(0, committed - NAB); j < committed; ++j)
        tc_mbar_wait(smem_u32(&mbar[j % NAB]), (uint32_t)((j / NAB) & 1), kTcPolls);
      for (int j = landed; j < issued; ++j) tc_mbar_wait(smem_u32(&sbar[j & 1]), (uint32_t)((j >> 1) & 1), kTcPolls);
    }
    __syncthreads();
  }
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(t.tmem_cols) : "memory");
}

}  // namespace tg
