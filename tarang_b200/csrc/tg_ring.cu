// Anisotropic energy spectra of a context's vector state (FOUR and SCFT bases): the ring
// spectrum E(k, theta) over spherical shells x polar sectors about an anisotropy axis, and the
// cylindrical ring spectrum E(k_perp, k_par) over cylindrical shells x slabs along the axis.
//
// SCFT: Compute_local_ring_spectrum_SCFT (lib/scft/scft_energy.cc:814-940), the helicity ring
// spectrum (:1334-1370), the cylinder ring spectra (:1423-1480, :1794-1830) with
// Multiplicity_factor_SCFT, kx = l1 kfactor[1] >= 0, the Fourier-basis vector (-i V1, V2, V3) and
// the SCFT radii AnisKpll/AnisKperp/Anis_max_Kpll/Anis_max_Krho_radius_inside_SCFT
// (lib/scft/scft_inline.h:361-535).  As written there, the off-axis branch of the spherical ring
// spectrum adds |V x K|_axis^2/k_perp^2 and its complement WITHOUT the multiplicity factor (the
// on-axis branch and every other SCFT spectrum apply it); this file does the same.
//
// Reference: CVF::CV_Compute_ring_spectrum / CV_Compute_cylinder_ring_spectrum
// (lib/fields/Cvf.cc:484-560, sector and slab arrays Cvf.cc:84-190) with
// Compute_local_ring_spectrum_FOUR (lib/four/four_energy.cc:828-955) and
// Compute_local_cylinder_ring_spectrum_FOUR (four_energy.cc:1450-1516); the angle, index and
// radius helpers are AnisKpll/AnisKperp/AnisKvect_polar_angle/Anis_max_Kpll/
// Anis_max_Krho_radius_inside_FOUR (lib/four/four_inline.h:382-580), Get_polar_angle
// (lib/basis_basicfn/basis_basicfn_inline.h:89-113), Get_sector_index and Get_slab_index
// (lib/basis_basicfn/basis_basicfn.cc:304-400).
//
// One thread per stored mode; each block bins its modes in shared memory (atomics) and adds
// its bins to the output once.  Modes the 2/3 rule does not store are zero in the reference's
// arrays and add nothing there either.
#include <algorithm>
#include <cmath>
#include <vector>

#include "tg_ctx.h"

using namespace tg;

namespace {

constexpr int TPB = 256;
constexpr double kEps = 1e-15;  // MYEPS (extern_def_vars.h:81)
constexpr int kMaxBounds = TG_RING_MAX_SECTORS + 1;

struct RingArgs {
  Geo g;
  const cx<double>* V[3];
  int cyl;              // 0: spherical shells x sectors, 1: cylindrical shells x slabs
  int axis;             // anisotropy axis 1 (x), 2 (y), 3 (z)
  int rows, cols;       // shells (0..kmax), sectors or slabs (0..n)
  int nb;               // entries of bound[] used: n + 1
  double bound[kMaxBounds];  // sector angles or slab k_par values
  double* out;          // [4][rows][cols]: S1, S2 (|K|^0), S1, S2 (|K|^2)
  int hel;              // 1: S1 = modal helicity 2 K . (Vr x Vi) (the helicity ring spectra)
};

// Get_polar_angle: atan(k_perp / k_par) in [0, pi)
__device__ __forceinline__ double polar_angle(double kperp, double kpll) {
  double t;
  if (fabs(kperp) > kEps) t = (fabs(kpll) > kEps) ? atan(kperp / kpll) : M_PI / 2;
  else t = (kpll >= 0) ? 0.0 : M_PI;
  return (t >= 0) ? t : t + M_PI;
}

// Get_sector_index: folded to [0, pi/2]; theta = 0 belongs to sector 1
__device__ __forceinline__ int sector_index(double theta, const RingArgs& a) {
  if (theta > M_PI / 2) theta = M_PI - theta;
  if (fabs(theta) < kEps) return 1;
  int i = 0;
  for (; i < a.nb; ++i)
    if (theta <= a.bound[i]) break;
  return i;
}

// Get_slab_index: |k_par|; k_par = 0 belongs to slab 1
__device__ __forceinline__ int slab_index(double kpll, const RingArgs& a) {
  kpll = fabs(kpll);
  if (kpll < kEps) return 1;
  int i = 1;
  for (; i < a.nb; ++i)
    if (kpll <= a.bound[i]) break;
  return i;
}

__global__ void __launch_bounds__(TPB) k_ring(RingArgs a, int use_smem) {
  extern __shared__ double sh[];
  const int nbins = a.rows * a.cols;
  double* acc = use_smem ? sh : a.out;
  if (use_smem) {
    for (int i = threadIdx.x; i < 4 * nbins; i += TPB) sh[i] = 0;
    __syncthreads();
  }
  const Geo& g = a.g;
  const long long stride = (long long)gridDim.x * TPB;
  for (long long idx = (long long)blockIdx.x * TPB + threadIdx.x; idx < g.S; idx += stride) {
    int r1, r2, l3;
    compact_mode(g, idx, r1, r2, l3);
    if (l3 >= g.nkz) continue;
    const int l1 = geo_l1(g, r1), l2 = amap_index(g.ay, r2);
    const double k[3] = {geo_kx(g, r1) * g.kf0, geo_ky(g, r2) * g.kf1, l3 * g.kf2};
    const int ax = a.axis - 1, p1 = (ax + 1) % 3, p2 = (ax + 2) % 3;
    const double kpll = k[ax];
    const double kperp = sqrt(k[p1] * k[p1] + k[p2] * k[p2]);
    const double K2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
    const double K = sqrt(K2);
    const bool scft = g.basis == 1;
    cx<double> v[3] = {a.V[0][idx], a.V[1][idx], a.V[2][idx]};
    if (scft) v[0] = mkc<double>(v[0].y, -v[0].x);  // -i V1: the SCFT x component in the Fourier basis
    const double vv = v[0].x * v[0].x + v[0].y * v[0].y + v[1].x * v[1].x + v[1].y * v[1].y +
                      v[2].x * v[2].x + v[2].y * v[2].y;
    const double f = scft ? mult_scft(l1, l2, l3, g.N2) : mult_four(l1, l2, l3, g.N1, g.N2);
    double fe = f;  // the factor on e1, e2 (see the SCFT off-axis note at the top of the file)
    int row, col;
    double e1, e2;
    if (!a.cyl) {
      row = (int)ceil(K);
      if (!(K > kEps) || row >= a.rows) continue;
      col = sector_index(polar_angle(kperp, kpll), a);
      if (kperp < kEps) {
        // on the axis: two components (axis x: y, z; y: z, then y in FOUR and x in SCFT; z: x, y)
        const int c1 = (ax == 0) ? 1 : (ax == 1 ? 2 : 0);
        const int c2 = (ax == 0) ? 2 : (ax == 1 ? (scft ? 0 : 1) : 1);
        e1 = v[c1].x * v[c1].x + v[c1].y * v[c1].y;
        e2 = v[c2].x * v[c2].x + v[c2].y * v[c2].y;
      } else {
        // (V x K)_axis / k_perp: the component along the axis-normal direction in the
        // plane of K and the axis; the rest of |V|^2 goes to S2
        const cx<double> c = k[p2] * v[p1] - k[p1] * v[p2];
        e1 = (c.x * c.x + c.y * c.y) / (kperp * kperp);
        e2 = vv - e1;
        if (scft) fe = 1.0;
      }
    } else {
      row = (int)ceil(kperp);
      if (row >= a.rows) continue;
      col = slab_index(kpll, a);
      e1 = v[ax].x * v[ax].x + v[ax].y * v[ax].y;
      e2 = vv - e1;
    }
    if (a.hel) {
      // Compute_local_(cylinder_)ring_spectrum_helicity_FOUR (four_energy.cc:1357-1413,
      // 1825-1880): 2 mult K . (Vr x Vi)
      const double c0 = v[1].x * v[2].y - v[2].x * v[1].y, c1 = v[2].x * v[0].y - v[0].x * v[2].y,
                   c2 = v[0].x * v[1].y - v[1].x * v[0].y;
      e1 = 2.0 * (k[0] * c0 + k[1] * c1 + k[2] * c2);
      e2 = 0.0;
      fe = f;
    }
    if (col < 0 || col >= a.cols) continue;
    const int b = row * a.cols + col;
    atomicAdd(&acc[b], fe * e1);
    atomicAdd(&acc[nbins + b], fe * e2);
    atomicAdd(&acc[2 * nbins + b], fe * K2 * e1);
    atomicAdd(&acc[3 * nbins + b], fe * K2 * e2);
  }
  if (use_smem) {
    __syncthreads();
    for (int i = threadIdx.x; i < 4 * nbins; i += TPB)
      if (sh[i] != 0) atomicAdd(&a.out[i], sh[i]);
  }
}

// Compute_local_shell_spectrum_helicity_FOUR (four_energy.cc:551-603): shell ceil|K| <=
// Min_radius_outside gets 2 mult K_i (Vr x Vi)_i per component i
__global__ void __launch_bounds__(TPB) k_shell_helicity(Geo g, const cx<double>* V0, const cx<double>* V1,
                                                        const cx<double>* V2, int nbins, double* out) {
  extern __shared__ double sh[];
  for (int i = threadIdx.x; i < 3 * nbins; i += TPB) sh[i] = 0;
  __syncthreads();
  const long long stride = (long long)gridDim.x * TPB;
  for (long long idx = (long long)blockIdx.x * TPB + threadIdx.x; idx < g.S; idx += stride) {
    int r1, r2, l3;
    compact_mode(g, idx, r1, r2, l3);
    if (l3 >= g.nkz) continue;
    const int l1 = geo_l1(g, r1), l2 = amap_index(g.ay, r2);
    const double kx = geo_kx(g, r1) * g.kf0, ky = geo_ky(g, r2) * g.kf1, kz = l3 * g.kf2;
    const int b = (int)ceil(sqrt(kx * kx + ky * ky + kz * kz));
    if (b >= nbins) continue;
    const cx<double> a = V0[idx], bb = V1[idx], d = V2[idx];
    const double f = 2.0 * mult_four(l1, l2, l3, g.N1, g.N2);
    atomicAdd(&sh[b], f * kx * (bb.x * d.y - d.x * bb.y));
    atomicAdd(&sh[nbins + b], f * ky * (d.x * a.y - a.x * d.y));
    atomicAdd(&sh[2 * nbins + b], f * kz * (a.x * bb.y - bb.x * a.y));
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 3 * nbins; i += TPB)
    if (sh[i] != 0) atomicAdd(&out[i], sh[i]);
}

// largest |k_i| inside the (de)aliased box along axis i = 0, 1, 2: FOUR (N_i/d) kf_i
// (Anis_max_Krho_radius_inside_FOUR four_inline.h); SCFT x: 2 N1/3 dealiased, N1 - 1 aliased
// (Anis_max_Krho_radius_inside_SCFT scft_inline.h:489-520)
double axis_extent(const tg_ctx* c, int i) {
  const int d = c->cfg.dealias ? 3 : 2;
  const int Nax[3] = {c->N1, c->N2, c->N3};
  if (c->basis != TG_FOUR && i == 0) return (c->cfg.dealias ? 2 * c->N1 / 3 : c->N1 - 1) * c->cfg.kfactor[0];
  return (Nax[i] / d) * c->cfg.kfactor[i];
}

// Anis_max_Krho_radius_inside: the cylinder radius inside the box across `axis` (1..3)
int krho_inside(const tg_ctx* c, int axis) {
  const int p1 = axis % 3, p2 = (axis + 1) % 3;
  return (int)std::min(axis_extent(c, p1), axis_extent(c, p2));
}

// Anis_max_Kpll: the largest K_par.  SCFT dealiased, axis y: (N2/2) kf (scft_inline.h:475-481,
// as written there; the box edge would be N2/3)
double kpll_max(const tg_ctx* c, int axis) {
  if (c->basis != TG_FOUR && c->cfg.dealias && axis == 2) return (c->N2 / 2) * c->cfg.kfactor[1];
  return axis_extent(c, axis - 1);
}

int run_ring(tg_ctx* c, int group, int axis, int n, int cyl, double* ek1, double* ek2, double* dissk, int cap,
             int hel = 0) {
  if (!c || !ek1) return TG_ERR_ARG;
  if (axis < 1 || axis > 3 || n < 1 || n > TG_RING_MAX_SECTORS) return TG_ERR_ARG;
  if (group != 0 && !(group == 1 && c->phys == TG_MHD)) return TG_ERR_ARG;
  RingArgs a{};
  a.g = c->g;
  for (int i = 0; i < 3; ++i) a.V[i] = c->U0[3 * group + i];
  a.cyl = cyl;
  a.hel = hel;
  a.axis = axis;
  a.cols = n + 1;
  a.nb = n + 1;
  if (!cyl) {
    // shells 0 .. Max_radius_inside; sectors of equal angle up to Get_max_polar_angle = pi/2
    a.rows = radius_inside(c) + 1;
    const double dtheta = (M_PI / 2) / n;
    for (int i = 0; i < n; ++i) a.bound[i] = i * dtheta;
    a.bound[n] = M_PI / 2;
  } else {
    // shells 0 .. Anis_max_Krho_radius_inside; slabs of equal k_par up to Anis_max_Kpll
    a.rows = krho_inside(c, axis) + 1;
    const double kmax = kpll_max(c, axis);
    const double dk = kmax / n;
    a.bound[0] = 0.0;
    for (int i = 1; i < n; ++i) a.bound[i] = i * dk;
    a.bound[n] = kmax;
  }
  const int nbins = a.rows * a.cols;
  if (cap < nbins) return set_err(c, TG_ERR_ARG, "ring spectrum: output arrays shorter than shells x (n + 1)");
  cudaSetDevice(c->dev);
  int rc = ensure_diag(c, (size_t)4 * nbins);
  if (rc) return rc;
  a.out = c->diag;
  cudaError_t e = cudaMemsetAsync(a.out, 0, sizeof(double) * 4 * nbins, c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "ring spectrum");
  const size_t smem = sizeof(double) * 4 * (size_t)nbins;
  const int use_smem = smem <= 96 * 1024 ? 1 : 0;
  if (use_smem && smem > 48 * 1024) {
    e = cudaFuncSetAttribute(k_ring, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_err(c, e, "ring spectrum");
  }
  long long nb = (c->g.S + TPB - 1) / TPB;
  if (nb > 148 * 4) nb = 148 * 4;
  k_ring<<<(unsigned)nb, TPB, use_smem ? smem : 0, c->st>>>(a, use_smem);
  e = cudaGetLastError();
  std::vector<double> h((size_t)4 * nbins);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), a.out, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "ring spectrum");
  TG_SYNC(c, "ring spectrum");
  for (int i = 0; i < nbins; ++i) {
    ek1[i] = h[i];
    if (ek2) ek2[i] = h[nbins + i];
    // CV_ring_dissk = 2 (S1 + S2 at |K|^2)
    if (dissk) dissk[i] = 2.0 * (h[2 * nbins + i] + h[3 * nbins + i]);
  }
  return TG_OK;
}

// ---------------------------------------------------------------------------------- ring-to-ring
// IncVF::Compute_ring_tr (EnergyTrdir/compute_ring_tr.cc:60-90, scalar :104-131, MHD and Elsasser
// kinds :174-285; cylinders compute_cylin_ring_tr.cc:54-330): for every
// giver ring (ring shell i = 1 .. n-1, sector j = 1 .. n_sectors) G = F on that ring (Fill_ring
// fill_ring.cc:70-90, Fill_array_ring universal_ET.cc:70-100), N = D_j F(H_j G_i)
// (EnergyTr_Compute_nlin) and T[i][j][shell][sector] = sign * sum 2 mult Re(N . R*) over the
// receiver rings (Local_ring_mult_all_FOUR four_ET.cc:330-386, Compute_ring_index
// basis_basicfn.cc:324-352).  Ring radii: scheme 0 of EnergyTr.cc:190-210.

constexpr int kMaxRingShells = 32;

struct RingBins {
  double r[kMaxRingShells + 1];  // ring shell radii 0 .. n (r[n] = INF_RADIUS)
  int n;
  double bound[kMaxBounds];      // sector angles 0 .. ns
  int ns;
  int axis;
  double kin;                    // rings: Max_radius_inside; cylinders: Anis_max_Krho_radius_inside
  int cyl;                       // 0: shells x sectors, 1: cylindrical shells x k_par slabs
};

// rings: K = |K| and theta the unfolded polar angle; cylinders: K = K_perp and theta = K_par
__device__ __forceinline__ void mode_angle(const Geo& g, long long idx, int axis, int cyl, int& r1, int& r2, int& l3,
                                           double& K, double& theta, double k[3]) {
  compact_mode(g, idx, r1, r2, l3);
  k[0] = geo_kx(g, r1) * g.kf0;
  k[1] = geo_ky(g, r2) * g.kf1;
  k[2] = l3 * g.kf2;
  const int ax = axis - 1, p1 = (ax + 1) % 3, p2 = (ax + 2) % 3;
  const double kperp = sqrt(k[p1] * k[p1] + k[p2] * k[p2]);
  if (cyl) {
    K = kperp;
    theta = k[ax];
  } else {
    K = sqrt(k[0] * k[0] + k[1] * k[1] + k[2] * k[2]);
    theta = polar_angle(kperp, k[ax]);
  }
}

// G = F where inner < K <= outer and left < theta <= right, or theta = 0 in the first sector or
// slab (Fill_array_ring / Fill_array_cylinder_ring: theta unfolded, K_par signed)
__global__ void k_fill_ring(Geo g, const cx<double>* F0, const cx<double>* F1, const cx<double>* F2, cx<double>* G0,
                            cx<double>* G1, cx<double>* G2, double lo, double hi, double left, double right, int axis,
                            int cyl) {
  const long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
  if (idx >= g.S) return;
  int r1, r2, l3;
  double K, th, k[3];
  mode_angle(g, idx, axis, cyl, r1, r2, l3, K, th, k);
  const bool in = (l3 < g.nkz) && (K > lo) && (K <= hi) &&
                  ((th > left && th <= right) || (fabs(th) < kEps && left < kEps));
  const cx<double> z = mkc<double>(0, 0);
  G0[idx] = in ? F0[idx] : z;
  G1[idx] = in ? F1[idx] : z;
  G2[idx] = in ? F2[idx] : z;
}

struct RingContractArgs {
  Geo g;
  const void* PX[9];  // P(i, j) = F(H_j G_i), q = 3 i + j
  const cx<double>* R[3];
  RingBins b;
  double* out;        // [n + 1][ns + 1]
};

// receiver ring of a mode, shell * (ns + 1) + sector, or -1 outside the rings
// (Local_ring_mult_all: 0 < |K| <= R_in, Compute_ring_index with the angle folded to [0, pi/2];
// Local_cyl_ring_mult_all: K_perp <= K_perp,max, Compute_cylinder_ring_index with |K_par|, K_par = 0
// in slab 1; first radius >= K, the radii need not be sorted)
__device__ __forceinline__ int ring_bin(const RingBins& b, double K, double th) {
  if (b.cyl ? !(K <= b.kin) : !(K <= b.kin && K > kEps)) return -1;
  int shell = 0;
  while (shell <= b.n && !(K <= b.r[shell])) ++shell;
  if (shell > b.n) return -1;
  int sector;
  if (!b.cyl) {
    if (th > M_PI / 2) th = M_PI - th;
    sector = 1;
    if (!(fabs(th) < kEps)) {
      sector = 0;
      while (sector <= b.ns && !(th <= b.bound[sector])) ++sector;
    }
  } else {
    th = fabs(th);
    sector = 1;
    if (!(th < kEps)) {
      while (sector <= b.ns && !(th <= b.bound[sector])) ++sector;
    }
  }
  if (sector > b.ns) return -1;
  return shell * (b.ns + 1) + sector;
}

// Compute_force_feed_ring / _cylinder_ring (compute_force_feed.cc:162-300): 2 mult Re(F . X*)
// binned by receiver ring, F from the force box (components c0 .. c0+nc-1) or, with lm, the
// liquid-metal force -(B0 . K)^2/K^2 V
struct RingFeedArgs {
  Geo g;
  RingBins b;
  const cx<double>* FB;
  int fx, fy, fz, c0, nc;
  const cx<double>* X[3];
  int lm;
  double b0[3];
  double* out;
};

__global__ void __launch_bounds__(TPB) k_ring_feed(RingFeedArgs a) {
  extern __shared__ double sh[];
  const int nbins = (a.b.n + 1) * (a.b.ns + 1);
  for (int i = threadIdx.x; i < nbins; i += TPB) sh[i] = 0;
  __syncthreads();
  const Geo& g = a.g;
  const int ny = 2 * a.fy + 1, nz = a.fz + 1;
  const long long stride = (long long)gridDim.x * TPB;
  for (long long idx = (long long)blockIdx.x * TPB + threadIdx.x; idx < g.S; idx += stride) {
    int r1, r2, l3;
    double K, th, k[3];
    mode_angle(g, idx, a.b.axis, a.b.cyl, r1, r2, l3, K, th, k);
    if (l3 >= g.nkz) continue;
    const int bin = ring_bin(a.b, K, th);
    if (bin < 0) continue;
    const int l1 = geo_l1(g, r1), l2 = amap_index(g.ay, r2);
    double re = 0;
    if (a.lm) {
      const double K2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
      const double bk = a.b0[0] * k[0] + a.b0[1] * k[1] + a.b0[2] * k[2];
      const double f = K2 > 0 ? -bk * bk / K2 : 0.0;
      for (int c = 0; c < 3; ++c) {
        const cx<double> v = a.X[c][idx];
        re += f * (v.x * v.x + v.y * v.y);
      }
    } else {
      const int kx = geo_kx(g, r1), ky = geo_ky(g, r2);
      if (kx < -a.fx || kx > a.fx || ky < -a.fy || ky > a.fy || l3 > a.fz) continue;
      const int box = (2 * a.fx + 1) * ny * nz;
      const int p = ((kx + a.fx) * ny + (ky + a.fy)) * nz + l3;
      for (int c = 0; c < a.nc; ++c) {
        const cx<double> f = a.FB[(long long)(a.c0 + c) * box + p], v = a.X[c][idx];
        re += f.x * v.x + f.y * v.y;
      }
    }
    if (re != 0)
      atomicAdd(&sh[bin], 2 * (g.basis == 1 ? mult_scft(l1, l2, l3, g.N2) : mult_four(l1, l2, l3, g.N1, g.N2)) * re);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nbins; i += TPB)
    if (sh[i] != 0) atomicAdd(&a.out[i], sh[i]);
}

template <typename Rp>
__global__ void __launch_bounds__(TPB) k_ring_contract(RingContractArgs a) {
  extern __shared__ double sh[];
  const int cols = a.b.ns + 1, nbins = (a.b.n + 1) * cols;
  for (int i = threadIdx.x; i < nbins; i += TPB) sh[i] = 0;
  __syncthreads();
  const Geo& g = a.g;
  const long long stride = (long long)gridDim.x * TPB;
  for (long long idx = (long long)blockIdx.x * TPB + threadIdx.x; idx < g.S; idx += stride) {
    int r1, r2, l3;
    double K, th, k[3];
    mode_angle(g, idx, a.b.axis, a.b.cyl, r1, r2, l3, K, th, k);
    if (l3 >= g.nkz) continue;
    const int bin = ring_bin(a.b, K, th);
    if (bin < 0) continue;
    const int shell = bin / cols, sector = bin - shell * cols;
    const int l1 = geo_l1(g, r1), l2 = amap_index(g.ay, r2);
    double v = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const cx<double> p0 = cvt<double>(reinterpret_cast<const cx<Rp>*>(a.PX[3 * i + 0])[idx]);
      const cx<double> p1 = cvt<double>(reinterpret_cast<const cx<Rp>*>(a.PX[3 * i + 1])[idx]);
      const cx<double> p2 = cvt<double>(reinterpret_cast<const cx<Rp>*>(a.PX[3 * i + 2])[idx]);
      // N_i = D_j P(i, j): FOUR i (k . P(i, .)); SCFT the x derivative of the cosine series P(0, 0)
      // is -kx P and of the sine series P(1, 0), P(2, 0) +kx P (Xderiv_SCFT scft_tr.cc:649-707)
      cx<double> Ni;
      if (g.basis == 0) {
        Ni = ione(mkc<double>(k[0] * p0.x + k[1] * p1.x + k[2] * p2.x, k[0] * p0.y + k[1] * p1.y + k[2] * p2.y));
      } else {
        const double dx = (i == 0) ? -k[0] : k[0];
        Ni = mkc<double>(dx * p0.x - (k[1] * p1.y + k[2] * p2.y), dx * p0.y + (k[1] * p1.x + k[2] * p2.x));
      }
      const cx<double> r = a.R[i][idx];
      v += Ni.x * r.x + Ni.y * r.y;
    }
    const double m = g.basis == 1 ? mult_scft(l1, l2, l3, g.N2) : mult_four(l1, l2, l3, g.N1, g.N2);
    atomicAdd(&sh[shell * cols + sector], 2.0 * m * v);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nbins; i += TPB)
    if (sh[i] != 0) atomicAdd(&a.out[i], sh[i]);
}

// EnergyTr.cc:190-210 (rings, Rin = Max_radius_inside) and :300-320 (cylinders, Rin =
// Anis_max_Krho_radius_inside), scheme 0
void ring_radii_from(double Rin, int n, double* r) {
  for (int i = 0; i <= n; ++i) r[i] = 0.0;
  r[1] = 4.0;
  r[2] = 8.0;
  r[n - 2] = Rin / 2;
  r[n - 1] = Rin;
  r[n] = 10000.0;  // INF_RADIUS
  if (n > 5) {
    const double s = std::log2(Rin / 16.0) / (n - 4);
    for (int i = 3; i <= n - 3; ++i) r[i] = 8 * std::pow(2.0, s * (i - 2));
  }
}

void ring_radii(const tg_ctx* c, int n, double* r) { ring_radii_from((double)radius_inside(c), n, r); }

}  // namespace

extern "C" {

int tg_ring_radii(tg_ctx* c, int n_ring_shells, double* radii, int n) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c || !radii || n_ring_shells < 5 || n_ring_shells > kMaxRingShells || n < n_ring_shells + 1) return TG_ERR_ARG;
  ring_radii(c, n_ring_shells, radii);
  return TG_OK;
}

}  // extern "C"

namespace {

// the receiver rings of a ring (scheme-0 radii, equal sectors up to pi/2) or cylinder-ring (radii
// up to Anis_max_Krho_radius_inside, slabs of K_par up to Anis_max_Kpll) table
void ring_bins_for(tg_ctx* c, int axis, int n_ring_shells, int n_sectors, int cyl, RingBins& b) {
  b = RingBins{};
  b.n = n_ring_shells;
  b.ns = n_sectors;
  b.axis = axis;
  b.cyl = cyl;
  if (!cyl) {
    ring_radii(c, n_ring_shells, b.r);
    const double dtheta = (M_PI / 2) / n_sectors;
    for (int i = 0; i < n_sectors; ++i) b.bound[i] = i * dtheta;
    b.bound[n_sectors] = M_PI / 2;
    b.kin = (double)radius_inside(c);
  } else {
    const int kr = krho_inside(c, axis);
    ring_radii_from((double)kr, n_ring_shells, b.r);
    const double kmax = kpll_max(c, axis);
    const double dk = kmax / n_sectors;
    b.bound[0] = 0.0;
    for (int i = 1; i < n_sectors; ++i) b.bound[i] = i * dk;
    b.bound[n_sectors] = kmax;
    b.kin = (double)kr;
  }
}

int run_ring_tr(tg_ctx* c, int kind, int axis, int n_ring_shells, int n_sectors, int cyl, double* tr, int n) {
  if (!c || !tr) return TG_ERR_ARG;
  if (axis < 1 || axis > 3 || n_sectors < 1 || n_sectors > TG_RING_MAX_SECTORS) return TG_ERR_ARG;
  if (n_ring_shells < 5 || n_ring_shells > kMaxRingShells) return TG_ERR_ARG;
  // U->U ring_to_ring_self, B->B W.ring_to_ring_self, U->B ring_to_ring_VF, Z+->Z+ and Z-->Z-
  // ring_to_ring_Elsasser, T->T ring_to_ring_SF; the reference has no B->U ring table
  if (kind == TG_ET_BU) return set_err(c, TG_ERR_ARG, "ring transfers have no B->U kind");
  const int rows = n_ring_shells + 1, cols = n_sectors + 1, per = rows * cols;
  if ((size_t)n < (size_t)per * per) return set_err(c, TG_ERR_ARG, "ring transfer: output shorter than (n+1)^2 (ns+1)^2");
  cudaSetDevice(c->dev);
  int rc = ensure_et_buffers(c);
  if (rc) return rc;
  const cx<double>* Hp[3];
  const cx<double>* Fp[3];
  const cx<double>* Rp[3];
  double sign = 1.0;
  rc = et_kind_fields(c, kind, Hp, Fp, Rp, sign);
  if (rc) return rc;
  RingBins b{};
  ring_bins_for(c, axis, n_ring_shells, n_sectors, cyl, b);
  const size_t need = (size_t)per * per;  // [giver shell][giver sector][shell][sector]
  rc = ensure_diag(c, need);
  if (rc) return rc;
  cudaError_t e = cudaMemsetAsync(c->diag, 0, sizeof(double) * need, c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "ring transfer");
  const Geo& g = c->g;
  const void* Hf[3] = {Hp[0], Hp[1], Hp[2]};
  rc = pipe_inverse_xy(c, 3, Hf, nullptr, nullptr, F64, 3, c->WX, c->etWY);
  if (rc) return rc;
  ProdPairs pp{};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      pp.a[3 * i + j] = (signed char)(3 + i);  // G_i
      pp.b[3 * i + j] = (signed char)j;        // H_j
    }
  const size_t smem = sizeof(double) * per;
  if (smem > 48 * 1024) {
    e = cudaFuncSetAttribute(k_ring_contract<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_ring_contract<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_err(c, e, "ring transfer");
  }
  const int nblk = (int)std::min<long long>((g.S + TPB - 1) / TPB, 148LL * 8);
  for (int i = 1; i < n_ring_shells; ++i)
    for (int j = 1; j <= n_sectors; ++j) {
      k_fill_ring<<<(int)((g.S + TPB - 1) / TPB), TPB, 0, c->st>>>(g, Fp[0], Fp[1], Fp[2], c->etG[0], c->etG[1],
                                                                   c->etG[2],
                                                                   b.r[i - 1], b.r[i], b.bound[j - 1], b.bound[j], axis,
                                                                   cyl);
      e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_err(c, e, "fill ring");
      const void* G[3] = {c->etG[0], c->etG[1], c->etG[2]};
      rc = pipe_inverse_xy(c, 3, G, nullptr, nullptr, F64, 3, c->WX, c->etWY + 3);
      if (rc) return rc;
      rc = pipe_products_forward(c, 6, c->etWY, 9, pp, c->etPP, c->etPY, c->etPX, kEtXKinds);
      if (rc) return rc;
      RingContractArgs a{};
      a.g = g;
      for (int q = 0; q < 9; ++q) a.PX[q] = c->etPX[q];
      for (int q = 0; q < 3; ++q) a.R[q] = Rp[q];
      a.b = b;
      a.out = c->diag + ((size_t)i * cols + j) * per;
      if (c->tprec == F64) k_ring_contract<double><<<nblk, TPB, smem, c->st>>>(a);
      else k_ring_contract<float><<<nblk, TPB, smem, c->st>>>(a);
      e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_err(c, e, "ring contract");
    }
  std::vector<double> h(need);
  e = cudaMemcpyAsync(h.data(), c->diag, sizeof(double) * need, cudaMemcpyDeviceToHost, c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "ring transfer");
  TG_SYNC(c, "ring transfer");
  for (size_t q = 0; q < need; ++q) tr[q] = sign * h[q];
  return TG_OK;
}


}  // namespace

extern "C" {

int tg_ring_sizes(tg_ctx* c, int axis, int* ring_shells, int* cylinder_shells) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c || axis < 1 || axis > 3) return TG_ERR_ARG;
  if (ring_shells) *ring_shells = radius_inside(c) + 1;
  if (cylinder_shells) *cylinder_shells = krho_inside(c, axis) + 1;
  return TG_OK;
}

int tg_ring_spectrum(tg_ctx* c, int group, int axis, int n_sectors, double* ek1, double* ek2, double* dissk, int n) {
  if (c && c->slab_W) return slab_refuse(c);
  return run_ring(c, group, axis, n_sectors, 0, ek1, ek2, dissk, n);
}

int tg_cylinder_ring_spectrum(tg_ctx* c, int group, int axis, int n_slabs, double* ek1, double* ek2, double* dissk,
                              int n) {
  if (c && c->slab_W) return slab_refuse(c);
  return run_ring(c, group, axis, n_slabs, 1, ek1, ek2, dissk, n);
}

int tg_ring_to_ring(tg_ctx* c, int kind, int axis, int n_ring_shells, int n_sectors, double* tr, int n) {
  if (c && c->slab_W) return slab_refuse(c);
  return run_ring_tr(c, kind, axis, n_ring_shells, n_sectors, 0, tr, n);
}

int tg_ring_spectrum_helicity(tg_ctx* c, int group, int axis, int n_sectors, double* h, int n) {
  if (c && c->slab_W) return slab_refuse(c);
  return run_ring(c, group, axis, n_sectors, 0, h, nullptr, nullptr, n, 1);
}

int tg_cylinder_ring_spectrum_helicity(tg_ctx* c, int group, int axis, int n_slabs, double* h, int n) {
  if (c && c->slab_W) return slab_refuse(c);
  return run_ring(c, group, axis, n_slabs, 1, h, nullptr, nullptr, n, 1);
}

int tg_shell_spectrum_helicity(tg_ctx* c, int group, double* h1, double* h2, double* h3, int n) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c || !h1) return TG_ERR_ARG;
  if (c->basis != TG_FOUR) return set_err(c, TG_ERR_UNSUPPORTED, "helicity spectrum: FOUR basis only");
  if (group != 0 && !(group == 1 && c->phys == TG_MHD)) return TG_ERR_ARG;
  // Min_radius_outside_FOUR (four_inline.h:172-228) and Max_radius_inside
  const int d = c->cfg.dealias ? 3 : 2;
  const double* kf = c->cfg.kfactor;
  const double a0 = (c->N1 / d) * kf[0], a1 = (c->N2 / d) * kf[1], a2 = (c->N3 / d) * kf[2];
  const int kkmax = (int)std::ceil(std::sqrt(a0 * a0 + a1 * a1 + a2 * a2));
  const int kin = radius_inside(c);
  const int nbins = kkmax + 1;
  if (n < nbins) return set_err(c, TG_ERR_ARG, "helicity spectrum: n < kmax_outside + 1");
  cudaSetDevice(c->dev);
  int rc = ensure_diag(c, (size_t)3 * nbins);
  if (rc) return rc;
  cudaError_t e = cudaMemsetAsync(c->diag, 0, sizeof(double) * 3 * nbins, c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "helicity spectrum");
  const size_t smem = sizeof(double) * 3 * (size_t)nbins;
  if (smem > 48 * 1024) {
    e = cudaFuncSetAttribute(k_shell_helicity, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_err(c, e, "helicity spectrum");
  }
  long long nb = (c->g.S + TPB - 1) / TPB;
  if (nb > 148 * 4) nb = 148 * 4;
  k_shell_helicity<<<(unsigned)nb, TPB, smem, c->st>>>(c->g, c->U0[3 * group], c->U0[3 * group + 1],
                                                       c->U0[3 * group + 2], nbins, c->diag);
  e = cudaGetLastError();
  std::vector<double> hh((size_t)3 * nbins);
  if (e == cudaSuccess) e = cudaMemcpyAsync(hh.data(), c->diag, sizeof(double) * hh.size(), cudaMemcpyDeviceToHost, c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "helicity spectrum");
  TG_SYNC(c, "helicity spectrum");
  // H1k_count: 2 mult over every mode of the dense grid (geometry only); partial shells
  // (kmax_inside, kmax] rescaled by Approx_number_modes_in_shell / count (four_energy.cc:637-651)
  std::vector<double> cnt(nbins, 0.0);
  for (int l1 = 0; l1 < c->N1; ++l1) {
    const int kxi = l1 > c->N1 / 2 ? l1 - c->N1 : l1;
    for (int l2 = 0; l2 < c->N2; ++l2) {
      const int kyi = l2 <= c->N2 / 2 ? l2 : l2 - c->N2;
      for (int l3 = 0; l3 < c->M3; ++l3) {
        const double kx = kxi * kf[0], ky = kyi * kf[1], kz = l3 * kf[2];
        const int b = (int)std::ceil(std::sqrt(kx * kx + ky * ky + kz * kz));
        if (b < nbins) cnt[b] += 2.0 * mult_four(l1, l2, l3, c->N1, c->N2);
      }
    }
  }
  const double approx_fac = 2 * M_PI / (kf[0] * kf[1] * kf[2]);
  double* out[3] = {h1, h2, h3};
  for (int i = 0; i < 3; ++i) {
    if (!out[i]) continue;
    for (int b = 0; b < n; ++b) out[i][b] = 0.0;
    for (int b = 0; b < nbins; ++b) {
      const bool resc = (b > kin) && (cnt[b] >= 1);
      out[i][b] = hh[(size_t)i * nbins + b] * (resc ? approx_fac * b * b / cnt[b] : 1.0);
    }
  }
  return TG_OK;
}

// Compute_force_feed_ring / Compute_force_feed_cylinder_ring (compute_force_feed.cc:162-300)
int tg_force_feed_ring(tg_ctx* c, int group, int cylinder, int axis, int n_ring_shells, int n_sectors, double* out,
                       int n) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c || !out) return TG_ERR_ARG;
  if (c->phys == TG_RB || (c->basis != TG_FOUR && !(c->force_on == 1 && c->phys != TG_MHD)))
    return set_err(c, TG_ERR_UNSUPPORTED, "ring force feed: FOUR or an SCFT band forcing, no convection");
  if (axis < 1 || axis > 3 || n_sectors < 1 || n_sectors > TG_RING_MAX_SECTORS) return TG_ERR_ARG;
  if (n_ring_shells < 5 || n_ring_shells > kMaxRingShells || group < 0 || group > 2) return TG_ERR_ARG;
  if ((group == 1 && c->phys != TG_MHD) || (group == 2 && c->phys != TG_SCALAR))
    return set_err(c, TG_ERR_ARG, "ring force feed: the group is not a field of this physics");
  const int per = (n_ring_shells + 1) * (n_sectors + 1);
  if (n < per) return set_err(c, TG_ERR_ARG, "ring force feed: output shorter than (n+1)(ns+1)");
  for (int i = 0; i < n; ++i) out[i] = 0;
  const bool lm = c->lm && group == 0;
  if (!lm && (!c->force_on || (c->force_on == 2 && !c->FB))) return TG_OK;  // no force, or Coriolis
  cudaSetDevice(c->dev);
  int rc = TG_OK;
  if (!lm) rc = ensure_force_box(c);
  if (!rc) rc = ensure_diag(c, (size_t)per);
  if (rc) return rc;
  RingFeedArgs a{};
  a.g = c->g;
  ring_bins_for(c, axis, n_ring_shells, n_sectors, cylinder ? 1 : 0, a.b);
  a.FB = c->FB;
  a.fx = c->fx;
  a.fy = c->fy;
  a.fz = c->fz;
  a.c0 = group == 0 ? 0 : 3;
  a.nc = group == 2 ? 1 : 3;
  for (int i = 0; i < 3; ++i) a.X[i] = c->U0[a.c0 + (a.nc > 1 ? i : 0)];
  a.lm = lm ? 1 : 0;
  for (int i = 0; i < 3; ++i) a.b0[i] = c->b0[i];
  a.out = c->diag;
  cudaError_t e = cudaMemsetAsync(c->diag, 0, sizeof(double) * per, c->st);
  const size_t smem = sizeof(double) * per;
  if (e == cudaSuccess && smem > 48 * 1024)
    e = cudaFuncSetAttribute(k_ring_feed, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) {
    const int nblk = (int)std::min<long long>((c->g.S + TPB - 1) / TPB, 148LL * 8);
    k_ring_feed<<<nblk, TPB, smem, c->st>>>(a);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, c->diag, sizeof(double) * per, cudaMemcpyDeviceToHost, c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "ring force feed");
  TG_SYNC(c, "ring force feed");
  return TG_OK;
}

int tg_cylinder_ring_to_ring(tg_ctx* c, int kind, int axis, int n_cylinder_shells, int n_slabs, double* tr, int n) {
  if (c && c->slab_W) return slab_refuse(c);
  return run_ring_tr(c, kind, axis, n_cylinder_shells, n_slabs, 1, tr, n);
}

int tg_cylinder_radii(tg_ctx* c, int axis, int n_cylinder_shells, double* radii, int n) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c || !radii || axis < 1 || axis > 3 || n_cylinder_shells < 5 || n_cylinder_shells > kMaxRingShells ||
      n < n_cylinder_shells + 1)
    return TG_ERR_ARG;
  ring_radii_from((double)krho_inside(c, axis), n_cylinder_shells, radii);
  return TG_OK;
}

}  // extern "C"
