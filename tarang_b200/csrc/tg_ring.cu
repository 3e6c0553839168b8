// Anisotropic energy spectra of a context's vector state (FOUR basis): the ring spectrum
// E(k, theta) over spherical shells x polar sectors about an anisotropy axis, and the
// cylindrical ring spectrum E(k_perp, k_par) over cylindrical shells x slabs along the axis.
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
    const int l1 = amap_index(g.ax, r1), l2 = amap_index(g.ay, r2);
    const double k[3] = {geo_kx(g, r1) * g.kf0, geo_ky(g, r2) * g.kf1, l3 * g.kf2};
    const int ax = a.axis - 1, p1 = (ax + 1) % 3, p2 = (ax + 2) % 3;
    const double kpll = k[ax];
    const double kperp = sqrt(k[p1] * k[p1] + k[p2] * k[p2]);
    const double K2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
    const double K = sqrt(K2);
    const cx<double> v[3] = {a.V[0][idx], a.V[1][idx], a.V[2][idx]};
    const double vv = v[0].x * v[0].x + v[0].y * v[0].y + v[1].x * v[1].x + v[1].y * v[1].y +
                      v[2].x * v[2].x + v[2].y * v[2].y;
    const double f = mult_four(l1, l2, l3, g.N1, g.N2);
    int row, col;
    double e1, e2;
    if (!a.cyl) {
      row = (int)ceil(K);
      if (!(K > kEps) || row >= a.rows) continue;
      col = sector_index(polar_angle(kperp, kpll), a);
      if (kperp < kEps) {
        // on the axis: the two components across it (axis x: y, z; y: z, y; z: x, y)
        const int c1 = (ax == 0) ? 1 : (ax == 1 ? 2 : 0), c2 = (ax == 0) ? 2 : 1;
        e1 = v[c1].x * v[c1].x + v[c1].y * v[c1].y;
        e2 = v[c2].x * v[c2].x + v[c2].y * v[c2].y;
      } else {
        // (V x K)_axis / k_perp: the component along the axis-normal direction in the
        // plane of K and the axis; the rest of |V|^2 goes to S2
        const cx<double> c = k[p2] * v[p1] - k[p1] * v[p2];
        e1 = (c.x * c.x + c.y * c.y) / (kperp * kperp);
        e2 = vv - e1;
      }
    } else {
      row = (int)ceil(kperp);
      if (row >= a.rows) continue;
      col = slab_index(kpll, a);
      e1 = v[ax].x * v[ax].x + v[ax].y * v[ax].y;
      e2 = vv - e1;
    }
    if (col < 0 || col >= a.cols) continue;
    const int b = row * a.cols + col;
    atomicAdd(&acc[b], f * e1);
    atomicAdd(&acc[nbins + b], f * e2);
    atomicAdd(&acc[2 * nbins + b], f * K2 * e1);
    atomicAdd(&acc[3 * nbins + b], f * K2 * e2);
  }
  if (use_smem) {
    __syncthreads();
    for (int i = threadIdx.x; i < 4 * nbins; i += TPB)
      if (sh[i] != 0) atomicAdd(&a.out[i], sh[i]);
  }
}

int run_ring(tg_ctx* c, int group, int axis, int n, int cyl, double* ek1, double* ek2, double* dissk, int cap) {
  if (!c || !ek1) return TG_ERR_ARG;
  if (c->basis != TG_FOUR) return set_err(c, TG_ERR_UNSUPPORTED, "ring spectra: FOUR basis only");
  if (axis < 1 || axis > 3 || n < 1 || n > TG_RING_MAX_SECTORS) return TG_ERR_ARG;
  if (group != 0 && !(group == 1 && c->phys == TG_MHD)) return TG_ERR_ARG;
  const int d = c->cfg.dealias ? 3 : 2;
  const double* kf = c->cfg.kfactor;
  const int Nax[3] = {c->N1, c->N2, c->N3};
  RingArgs a{};
  a.g = c->g;
  for (int i = 0; i < 3; ++i) a.V[i] = c->U0[3 * group + i];
  a.cyl = cyl;
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
    const int p1 = axis % 3, p2 = (axis + 1) % 3;
    a.rows = (int)std::min((Nax[p1] / d) * kf[p1], (Nax[p2] / d) * kf[p2]) + 1;
    const double kmax = (Nax[axis - 1] / d) * kf[axis - 1];
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
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "ring spectrum");
  for (int i = 0; i < nbins; ++i) {
    ek1[i] = h[i];
    if (ek2) ek2[i] = h[nbins + i];
    // CV_ring_dissk = 2 (S1 + S2 at |K|^2)
    if (dissk) dissk[i] = 2.0 * (h[2 * nbins + i] + h[3 * nbins + i]);
  }
  return TG_OK;
}

}  // namespace

extern "C" {

int tg_ring_sizes(tg_ctx* c, int axis, int* ring_shells, int* cylinder_shells) {
  if (!c || axis < 1 || axis > 3) return TG_ERR_ARG;
  const int d = c->cfg.dealias ? 3 : 2;
  const double* kf = c->cfg.kfactor;
  const int Nax[3] = {c->N1, c->N2, c->N3};
  const int p1 = axis % 3, p2 = (axis + 1) % 3;
  if (ring_shells) *ring_shells = radius_inside(c) + 1;
  if (cylinder_shells) *cylinder_shells = (int)std::min((Nax[p1] / d) * kf[p1], (Nax[p2] / d) * kf[p2]) + 1;
  return TG_OK;
}

int tg_ring_spectrum(tg_ctx* c, int group, int axis, int n_sectors, double* ek1, double* ek2, double* dissk, int n) {
  return run_ring(c, group, axis, n_sectors, 0, ek1, ek2, dissk, n);
}

int tg_cylinder_ring_spectrum(tg_ctx* c, int group, int axis, int n_slabs, double* ek1, double* ek2, double* dissk,
                              int n) {
  return run_ring(c, group, axis, n_slabs, 1, ek1, ek2, dissk, n);
}

}  // extern "C"
