// Host-side launchers of the FFT pass kernels (tg_fft.cuh).  Precision of the input, output
// and arithmetic are runtime choices dispatched onto template instantiations.
#pragma once

#include "tg_fft.cuh"

namespace tg {

enum Prec { F64 = 0, F32 = 1 };

struct AxisLaunch {
  int L = 0;
  int dir = -1;  // -1 forward (e^{-i}), +1 inverse
  int pin = F64, pout = F64, pwork = F64;
  int nbatch = 1, nfields = 1;
  AxisArgs a{};
  PtrSet ps{};
};

struct ZLaunch {
  int M = 0;     // N3/2
  int kind = 0;  // 0: c2r, 1: r2c
  int pin = F64, pout = F64, pwork = F64;
  int nfields = 1;
  ZArgs a{};
  PtrSet ps{};
};

struct ZProdLaunch {
  int M = 0;
  int nin = 0, nprod = 0;
  int pin = F64, pout = F64, pwork = F64;
  ZArgs a{};
  PtrSet ps{};
  ProdPairs pp{};
};

cudaError_t launch_axis(const AxisLaunch& l, cudaStream_t s);
// 1 if a TMA-staged axis block gave up waiting for its tile (its output is not written), 0
// otherwise, -1 if the flag cannot be read; clear resets it
int axis_tma_timeout(bool clear);
// SCFT x-pass (real-to-real, per-field kind); l.L = N1, l.dir unused
cudaError_t launch_r2r(const AxisLaunch& l, const R2RArgs& r, cudaStream_t s);
cudaError_t launch_z(const ZLaunch& l, cudaStream_t s);
// coefficient table of the eight-lane z-pass for N3 = 256 (M = 128, k_z_prod_oct) or N3 = 128
// (M = 64, k_z_prod_oct64): at most kZoctTableLen complex values, evaluated in long double and
// rounded; M is 128 or 64
constexpr int kZoctTableLen = 100 * 8;
void zoct_table(int M, cx<double>* out);
cudaError_t launch_zprod(const ZProdLaunch& l, cudaStream_t s);

inline bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }
// L = R1 * R2 with R1 >= R2, both in {1,2,4,8,16,32}; returns false if unsupported
inline bool radix_split(int L, int& R1, int& R2) {
  switch (L) {
    case 2: R1 = 2; R2 = 1; return true;
    case 4: R1 = 2; R2 = 2; return true;
    case 8: R1 = 4; R2 = 2; return true;
    case 16: R1 = 4; R2 = 4; return true;
    case 32: R1 = 8; R2 = 4; return true;
    case 64: R1 = 8; R2 = 8; return true;
    case 128: R1 = 16; R2 = 8; return true;
    case 256: R1 = 16; R2 = 16; return true;
    case 512: R1 = 32; R2 = 16; return true;
    default: return false;
  }
}

}  // namespace tg
