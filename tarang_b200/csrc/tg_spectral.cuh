// Mode-space kernels of the time step: layout conversion, forcing, nonlinear-term assembly,
// pressure projection, the integrating-factor RK4 stage update and the energy reductions.
//
// Solver fields live in a compact layout [nkx][nky][kzp]: only the wavenumbers that the 2/3
// rule keeps (universal_misc.cc:118-159) are stored, kz padded to a multiple of 8 (zeros).
#pragma once

#include "tg_common.cuh"

namespace tg {

enum Phys { PH_FLUID = 0, PH_MHD = 1, PH_SCALAR = 2, PH_RB = 3 };

struct Geo {
  int N1, N2, N3;
  AxisMap ax, ay;       // stored kx, ky (FFT index space)
  int nkx, nky, nkz, kzp;
  long long S;          // compact elements per field (of the context's kx rows)
  double kf0, kf1, kf2; // kfactor
  int basis;            // 0 FOUR, 1 SCFT
  // a slab context holds compact kx rows x0 .. x0 + S / (nky kzp) - 1 of the nkx stored rows;
  // a whole-grid context has x0 = 0
  int x0;
};

__host__ __device__ __forceinline__ void compact_mode(const Geo& g, long long idx, int& r1, int& r2, int& l3) {
  l3 = (int)(idx % g.kzp);
  const long long rr = idx / g.kzp;
  r2 = (int)(rr % g.nky);
  r1 = (int)(rr / g.nky);
}
// FFT index l1 of the context's compact kx row r1
__host__ __device__ __forceinline__ int geo_l1(const Geo& g, int r1) { return amap_index(g.ax, r1 + g.x0); }
__host__ __device__ __forceinline__ int geo_kx(const Geo& g, int r1) {
  const int l1 = geo_l1(g, r1);
  if (g.basis == 1) return l1;
  return l1 <= g.N1 / 2 ? l1 : l1 - g.N1;
}
__host__ __device__ __forceinline__ int geo_ky(const Geo& g, int r2) {
  const int l2 = amap_index(g.ay, r2);
  return l2 <= g.N2 / 2 ? l2 : l2 - g.N2;
}

// Energy weight of Get_local_energy_FOUR (four_energy.cc:48-86): unstored -N/2 planes added,
// kz = 0 halved, origin excluded.
__host__ __device__ __forceinline__ double energy_weight_four(int l1, int l2, int l3, int N1, int N2) {
  double w = 1.0 + ((N2 > 1 && l2 == N2 / 2) ? 1.0 : 0.0) + (l1 == N1 / 2 ? 1.0 : 0.0);
  if (l3 == 0) w *= 0.5;
  if (l1 == 0 && l2 == 0 && l3 == 0) w -= 0.5;
  return w;
}
// Multiplicity_factor_FOUR (four_inline.h:347-365)
__host__ __device__ __forceinline__ double mult_four(int l1, int l2, int l3, int N1, int N2) {
  const double f = l3 > 0 ? 1.0 : 0.5;
  const int kx = l1 <= N1 / 2 ? l1 : l1 - N1;
  const int ky = l2 <= N2 / 2 ? l2 : l2 - N2;
  return (kx == N1 / 2 || (ky == N2 / 2 && N2 > 1)) ? 2 * f : f;
}
// Multiplicity_factor_SCFT (scft_inline.h:313-335)
__host__ __device__ __forceinline__ double mult_scft(int m, int l2, int l3, int N2) {
  double f = (l3 > 0) ? (m > 0 ? 2.0 : 1.0) : (m > 0 ? 1.0 : 0.5);
  const int ky = l2 <= N2 / 2 ? l2 : l2 - N2;
  return (ky == N2 / 2 && N2 > 1) ? 2 * f : f;
}

struct RKArgs {
  Geo g;
  int stage;               // RK4 1..4, EULER 5, RK2 7 then 6
  int nstate;              // state fields
  double nu[6];            // per state field
  double nuh[6];           // hyper coefficients per state field (0: off)
  const double* dt;        // device scalar
  cx<double>* U0[6];       // FP64 master state
  cx<double>* TOT[6];      // FP64 RK accumulator
  void* US[6];             // stage fields (transform precision)
  const void* PX[9];       // product spectra (compact)
  const cx<double>* RHS[6];// precomputed right-hand sides (SRC = 1)
  const cx<double>* FB;    // force box [nstate][box] or null
  int fx, fy, fz;          // force box half widths (kx, ky in [-f, f], kz in [0, fz])
  double* part;            // final stage (4, 5, 6): per-block partial sums [blocks][8]
  double rb_buoy_u, rb_buoy_t;  // RB forces: Force1 = rb_buoy_u * theta, T.Force = rb_buoy_t * u1
  const void* IN[6];       // the stage's input fields (the forces are computed from them)
  int inprec;              // 0 FP64, 1 FP32
  // batch: requests 0..nact-1 of the same shape, request r's fields at offset r * S, its
  // viscosities at nu_tab[6 r], its scalars (dt, ...) at dt[8 r], its partials in part[r]
  int nact;
  const double* nu_tab;
  // Coriolis force of the stage's velocity (Compute_force_Coriolis), when coriolis != 0
  int coriolis;
  double om[3];
  // liquid-metal force -(B0 . K)^2 / K^2 V of the stage's velocity (Compute_force_Liquid_metal),
  // when lm != 0
  int lm;
  double b0[3];
};

struct ForceArgs {
  Geo g;
  const void* U[6];        // the state fields the force reads (ns of them)
  int ns;                  // 3 fluid, 6 MHD (U, B), 4 passive scalar (U, T)
  int uprec;               // 0 FP64, 1 FP32
  int mode;                // 1: energy-helicity supply (proc 1), 2: constant energy-helicity (proc 2)
  int gate;                // skip U unless e_per_mode > MYEPS (all variants but proc 1 fluid)
  int fx, fy, fz;
  double inner, outer;
  double e_per_mode, eps_h;      // U
  double e_per_mode_b, eps_h_b;  // B (MHD) or e_per_mode_b = the scalar's energy per mode
  cx<double>* FB;          // [ns][box]
};

// launchers (tg_spectral.cu)
int reduction_blocks(long long S);  // grid of the reducing kernels (RK stage 4, energy partials)
cudaError_t launch_dense_to_compact(const Geo& g, const cx<double>* dense, void* compact, int cprec, cudaStream_t s);
cudaError_t launch_compact_to_dense(const Geo& g, const void* compact, int cprec, cx<double>* dense, cudaStream_t s);
cudaError_t launch_rk(const RKArgs& a, int phys, int pprec, int sprec, int src, cudaStream_t s, int* nblocks);
cudaError_t launch_force_supply(const ForceArgs& a, cudaStream_t s);
cudaError_t launch_assemble_nlin(const Geo& g, int phys, int pprec, const void* const* PX, cx<double>* const* NL, cudaStream_t s);
cudaError_t launch_sub_force_box(const Geo& g, int ncomp, const cx<double>* FB, int fx, int fy, int fz, cx<double>* const* NL, cudaStream_t s);
cudaError_t launch_pressure(const Geo& g, const cx<double>* const* NL, cx<double>* PR, cudaStream_t s);
cudaError_t launch_rhs_from_nlin(const Geo& g, int phys, cx<double>* const* NL, const cx<double>* PR, cudaStream_t s);
// NL[c] -= (U x om)[c], c < 3 (Add_force with the Coriolis force)
// NL[c] -= -(B0 . K)^2/K^2 U[c], c < 3 (Add_force with the liquid-metal force)
cudaError_t launch_sub_liquid_metal(const Geo& g, cx<double>* const* NL, const cx<double>* const* U, const double* b0,
                                    cudaStream_t s);
cudaError_t launch_sub_coriolis(const Geo& g, cx<double>* const* NL, const cx<double>* const* U, const double* om,
                                cudaStream_t s);
cudaError_t launch_rb_sub_force(const Geo& g, cx<double>* const* NL, const cx<double>* u1, const cx<double>* th,
                                double fu, double ft, cudaStream_t s);
cudaError_t launch_cross_partials(const Geo& g, const cx<double>* A, const cx<double>* B, double* part, int slot,
                                  int nslots, cudaStream_t s, int* nblocks);
// energy partials of a group of fields (FP64 compact), per block: [E, D]
cudaError_t launch_energy_partials(const Geo& g, const cx<double>* const* F, int nf, double* part, int slot, int nslots, cudaStream_t s, int* nblocks, int nact = 1);
// reduce partials [nblocks][nslots] -> out[nslots] in fixed order; then the dt rule
struct FinalizeArgs {
  const double* part;
  int nblocks, nslots;
  double* out;             // [nslots]
  double* scal;            // scalars: [0] dt, [1] t_now, [2] steps, [3] nonfinite flag
  double* ering;           // energy ring (may be null)
  int* ering_pos;
  int dt_mode;             // 0: none; 1: set dt from E (slots 0 [+2]) and advance t
  double dx, Tdt;
  int mhd;                 // add slot 2 (B energy) to the CFL energy
  const cx<double>* B0[3]; // mean magnetic field (mode 0) for MHD, or null
  int nact;                // requests of the batch (one block each)
  long long S;             // compact elements per request field
};
cudaError_t launch_finalize(const FinalizeArgs& a, cudaStream_t s);
// shell spectrum: ek[c][bin] += mult K^n |A|^2, counts
// part: scratch of shell_spectrum_blocks(g) x (nf + 1) x nbins doubles; ek and cnt are added to
int shell_spectrum_blocks(const Geo& g);
cudaError_t launch_shell_spectrum(const Geo& g, const cx<double>* const* F, int nf, double n_pow, double* ek, double* cnt,
                                  int nbins, double* part, cudaStream_t s);

}  // namespace tg
