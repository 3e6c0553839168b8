// Mode-space kernels of the time step (see tg_spectral.cuh).
#include "tg_spectral.cuh"

namespace tg {

namespace {

constexpr int TPB = 256;

template <typename R>
__device__ __forceinline__ cx<double> ldc(const void* p, long long i) {
  return cvt<double>(reinterpret_cast<const cx<R>*>(p)[i]);
}
template <typename R>
__device__ __forceinline__ void stc(void* p, long long i, cx<double> v) {
  reinterpret_cast<cx<R>*>(p)[i] = cvt<R>(v);
}

__device__ __forceinline__ cx<double> kdot(double kx, double ky, double kz, cx<double> a, cx<double> b, cx<double> c) {
  return mkc<double>(kx * a.x + ky * b.x + kz * c.x, kx * a.y + ky * b.y + kz * c.y);
}
// i (kx a + ky b + kz c)
__device__ __forceinline__ cx<double> ikdot(double kx, double ky, double kz, cx<double> a, cx<double> b, cx<double> c) {
  return ione(kdot(kx, ky, kz, a, b, c));
}

// block sum of NV doubles; thread 0 of the block gets the totals in v
template <int NV>
__device__ __forceinline__ void block_sum(double* v) {
  __shared__ double red[TPB / 32][NV];
#pragma unroll
  for (int j = 0; j < NV; ++j) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[j] += __shfl_down_sync(0xffffffffu, v[j], o);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) red[wid][j] = v[j];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      double s = 0;
      for (int w = 0; w < TPB / 32; ++w) s += red[w][j];
      v[j] = s;
    }
  }
}

// ------------------------------------------------------------------ layout conversion
template <typename R>
__global__ void k_dense_to_compact(Geo g, const cx<double>* __restrict__ dense, cx<R>* __restrict__ comp) {
  const long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
  if (idx >= g.S) return;
  int r1, r2, l3;
  compact_mode(g, idx, r1, r2, l3);
  cx<double> v = mkc<double>(0, 0);
  if (l3 < g.nkz) {
    const int l1 = geo_l1(g, r1), l2 = amap_index(g.ay, r2);
    const int M3 = g.N3 / 2 + 1;
    v = dense[((long long)l1 * g.N2 + l2) * M3 + l3];
  }
  comp[idx] = cvt<R>(v);
}

template <typename R>
__global__ void k_compact_to_dense(Geo g, const cx<R>* __restrict__ comp, cx<double>* __restrict__ dense) {
  const int M3 = g.N3 / 2 + 1;
  const long long D = (long long)g.N1 * g.N2 * M3;
  const long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
  if (idx >= D) return;
  const int l3 = (int)(idx % M3);
  const long long rr = idx / M3;
  const int l2 = (int)(rr % g.N2), l1 = (int)(rr / g.N2);
  const int r1 = amap_row(g.ax, l1), r2 = amap_row(g.ay, l2);
  cx<double> v = mkc<double>(0, 0);
  if (r1 >= 0 && r2 >= 0 && l3 < g.nkz) v = cvt<double>(comp[((long long)r1 * g.nky + r2) * g.kzp + l3]);
  dense[idx] = v;
}

// ------------------------------------------------------------------ nonlinear-term assembly
// Product order of the z-pass (see tg_ctx.cu):
//  fluid : 0 u1u1, 1 u2u2, 2 u3u3, 3 u1u2, 4 u2u3, 5 u3u1        (RSprod.cc:52-105)
//  MHD   : 0 zp1zm1, 1 zp2zm2, 2 zp3zm3, 3 zp1zm2 (v1), 4 zm1zp2 (w1), 5 zp2zm3 (v2),
//          6 zm2zp3 (w2), 7 zp3zm1 (v3), 8 zm3zp1 (w3)              (RSprod.cc:117-194)
//  scalar: fluid 0..5, then 6 u1 th, 7 u2 th, 8 u3 th               (compute_nlin_SF.cc)
// x-derivative of a coefficient (Xderiv universal_tr.cc:186-210): FOUR i kx; SCFT a real factor
// by the parity of the series, cos -> sin: -kx (Xderiv_Cos_SCFT), sin -> cos: +kx
// (Xderiv_Sin_SCFT, scft_tr.cc:649-672)
struct XDer {
  double kx;
  int scft;
  __device__ __forceinline__ cx<double> cos_in(cx<double> p) const {
    return scft ? mkc<double>(-kx * p.x, -kx * p.y) : ione(kx * p);
  }
  __device__ __forceinline__ cx<double> sin_in(cx<double> p) const {
    return scft ? mkc<double>(kx * p.x, kx * p.y) : ione(kx * p);
  }
};
__device__ __forceinline__ cx<double> iky_ikz(double ky, double kz, cx<double> b, cx<double> c) {
  return ione(mkc<double>(ky * b.x + kz * c.x, ky * b.y + kz * c.y));
}

template <typename Rp, int PHYS>
__device__ __forceinline__ void assemble(const void* const* PX, long long idx, const XDer& dx, double ky, double kz,
                                         cx<double>* n) {
  if constexpr (PHYS == PH_FLUID || PHYS == PH_SCALAR || PHYS == PH_RB) {
    // parities of the products (RV_Forward_transform_RSprod Rvf.cc:179-186): u1u1, u2u2, u3u3,
    // u2u3 cos; u1u2, u3u1 sin; and u1 th cos, u2 th, u3 th sin (compute_nlin_SF.cc:80-115)
    const cx<double> p0 = ldc<Rp>(PX[0], idx), p1 = ldc<Rp>(PX[1], idx), p2 = ldc<Rp>(PX[2], idx);
    const cx<double> p3 = ldc<Rp>(PX[3], idx), p4 = ldc<Rp>(PX[4], idx), p5 = ldc<Rp>(PX[5], idx);
    n[0] = dx.cos_in(p0) + iky_ikz(ky, kz, p3, p5);
    n[1] = dx.sin_in(p3) + iky_ikz(ky, kz, p1, p4);
    n[2] = dx.sin_in(p5) + iky_ikz(ky, kz, p4, p2);
    if constexpr (PHYS != PH_FLUID) {
      const cx<double> p6 = ldc<Rp>(PX[6], idx), p7 = ldc<Rp>(PX[7], idx), p8 = ldc<Rp>(PX[8], idx);
      n[3] = dx.cos_in(p6) + iky_ikz(ky, kz, p7, p8);
    }
  } else {
    const double kx = dx.kx;
    cx<double> p[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) p[q] = ldc<Rp>(PX[q], idx);
    // Zp.nlin (n) and Zm.nlin (nw)
    const cx<double> n0 = ikdot(kx, ky, kz, p[0], p[3], p[8]);
    const cx<double> n1 = ikdot(kx, ky, kz, p[4], p[1], p[5]);
    const cx<double> n2 = ikdot(kx, ky, kz, p[7], p[6], p[2]);
    const cx<double> w0 = ikdot(kx, ky, kz, p[0], p[4], p[7]);
    const cx<double> w1 = ikdot(kx, ky, kz, p[3], p[1], p[6]);
    const cx<double> w2 = ikdot(kx, ky, kz, p[8], p[5], p[2]);
    // Elsasser_to_UB_nlin (elsasser.cc:118-130)
    n[0] = 0.5 * (n0 + w0);
    n[1] = 0.5 * (n1 + w1);
    n[2] = 0.5 * (n2 + w2);
    n[3] = 0.5 * (n0 - w0);
    n[4] = 0.5 * (n1 - w1);
    n[5] = 0.5 * (n2 - w2);
  }
}

template <int PHYS>
struct NState {
  static constexpr int v = (PHYS == PH_FLUID) ? 3 : (PHYS == PH_MHD ? 6 : 4);
};

// rhs = -[nlin - f + grad p] with p = div(nlin - f)/K^2 on the velocity (Compute_pressure with
// Compute_divergence_nlin: Xderiv of nlin1 with parity 1; Add_pressure_gradient: Xderiv of p
// with parity 0; Compute_rhs); other fields rhs = -(nlin - f).
__device__ __forceinline__ void project_rhs(cx<double>* r, int ns, const XDer& dx, double ky, double kz, double K2) {
  cx<double> p = mkc<double>(0, 0);
  if (K2 > 0) {
    const cx<double> div = dx.sin_in(r[0]) + iky_ikz(ky, kz, r[1], r[2]);
    p = (1.0 / K2) * div;
  }
  const cx<double> g0 = dx.cos_in(p), g1 = ione(ky * p), g2 = ione(kz * p);
  r[0] = mkc<double>(-(r[0].x + g0.x), -(r[0].y + g0.y));
  r[1] = mkc<double>(-(r[1].x + g1.x), -(r[1].y + g1.y));
  r[2] = mkc<double>(-(r[2].x + g2.x), -(r[2].y + g2.y));
  for (int c = 3; c < ns; ++c) r[c] = mkc<double>(-r[c].x, -r[c].y);
}

// ------------------------------------------------------------------ RK stage kernel
// IncFluid::Time_advance (time_advance.cc:60-163) with E(a) = exp(-(nu + nu_h K^2) a dt K^2)
// (the hyper term when on, mult_exp_visc.cc:56-165) and Single_time_step(dt, a, b, c) =
// E(b)(E(a - b) u + c dt N) (single_time_step.cc:54-86):
//  RK4 stage 1: u1 = E(1/2)(u0 + dt/2 N0),        tot  = dt/6 E(1) N0
//      stage 2: u2 = E(1/2) u0 + dt/2 N1,         tot += dt/3 E(1/2) N1
//      stage 3: u3 = E(1/2)(E(1/2) u0 + dt N2),   tot += dt/3 E(1/2) N2
//      stage 4: u  = E(1) u0 + tot + dt/6 N3
//  EULER (5):   u  = E(1)(u0 + dt N0)                       Single_time_step(dt, 1, 1, 1)
//  RK2   (7):   u1 = E(1/2)(u0 + dt/2 N0)                   Single_time_step(dt, 1/2, 1/2, 1/2)
//        (6):   u  = E(1/2)(E(1/2) u0 + dt N1)              Single_time_step(dt, 1, 1/2, 1)
// after a final stage (4, 5, 6) the energy of u for the NaN check / Get_dt
// Resident blocks per SM the RK kernel is built for (fluid/scalar: 3 at 80 registers, MHD: 2).
template <int PHYS>
struct RKOcc {
  static constexpr int v = (PHYS == PH_MHD) ? 2 : 3;
};

// One thread per stored mode of one request (slot blockIdx.y).  Every value the mode needs
// (U0, TOT, the products) is loaded before anything is stored, so the loads of an element are
// in flight together; exp(-nu a dt K^2) is evaluated once per distinct viscosity.
template <typename Rp, typename Rs, int PHYS, int SRC, int STAGE>
__global__ void __launch_bounds__(TPB, RKOcc<PHYS>::v) k_rk(RKArgs a) {
  constexpr int NS = NState<PHYS>::v;
  const Geo& g = a.g;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const int slot = blockIdx.y;
  const long long base = (long long)slot * g.S;
  const double dt = a.dt[(long long)slot * 8];
  constexpr bool FINAL = STAGE == 4 || STAGE == 5 || STAGE == 6;
  double nus[NS], nuh[NS];
#pragma unroll
  for (int c = 0; c < NS; ++c) {
    nus[c] = a.nu_tab ? a.nu_tab[slot * 6 + c] : a.nu[c];
    nuh[c] = a.nuh[c];
  }
  const unsigned S = (unsigned)g.S, kzp = (unsigned)g.kzp, nky = (unsigned)g.nky;
  const unsigned stride = gridDim.x * TPB;
  for (unsigned i = blockIdx.x * TPB + threadIdx.x; i < S; i += stride) {
    const unsigned rr = i / kzp;
    const int l3 = (int)(i - rr * kzp);
    if (l3 >= g.nkz) continue;
    const int r1 = (int)(rr / nky), r2 = (int)(rr - (unsigned)r1 * nky);
    const long long gi = base + i;
    cx<double> u0[NS], tot[NS];
#pragma unroll
    for (int c = 0; c < NS; ++c) u0[c] = a.U0[c][gi];
    if constexpr (STAGE >= 2 && STAGE <= 4) {
#pragma unroll
      for (int c = 0; c < NS; ++c) tot[c] = a.TOT[c][gi];
    }
    const int kxi = geo_kx(g, r1), kyi = geo_ky(g, r2);
    const double kx = kxi * g.kf0, ky = kyi * g.kf1, kz = l3 * g.kf2;
    const double K2 = kx * kx + ky * ky + kz * kz;
    cx<double> r[NS];
    if constexpr (SRC == 0) {
      const XDer dx{kx, g.basis};
      assemble<Rp, PHYS>(a.PX, gi, dx, ky, kz, r);
      if (a.FB != nullptr && kxi >= -a.fx && kxi <= a.fx && kyi >= -a.fy && kyi <= a.fy && l3 <= a.fz) {
        const int box = (2 * a.fx + 1) * (2 * a.fy + 1) * (a.fz + 1);
        const int p = ((kxi + a.fx) * (2 * a.fy + 1) + (kyi + a.fy)) * (a.fz + 1) + l3;
#pragma unroll
        for (int c = 0; c < NS; ++c) r[c] = r[c] - a.FB[(long long)c * box + p];
      }
      if (a.coriolis) {
        // Compute_force_Coriolis (compute_force_Coriolis.cc:47-80) from the stage's velocity:
        // Force = V x Omega, then Add_force: nlin -= Force
        cx<double> v[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) v[c] = a.inprec ? ldc<float>(a.IN[c], gi) : ldc<double>(a.IN[c], gi);
        r[0] = r[0] - (a.om[1] * v[2] - a.om[2] * v[1]);
        r[1] = r[1] - (a.om[2] * v[0] - a.om[0] * v[2]);
        r[2] = r[2] - (a.om[0] * v[1] - a.om[1] * v[0]);
      }
      if (a.lm) {
        // Compute_force_Liquid_metal (compute_force_LM.cc:46-70): Force = -(B0 . K)^2/K^2 V
        // (Array_mult_V0_khat_sqr_FOUR four_basic.cc:413-439), then Add_force: nlin -= Force
        const double bk = a.b0[0] * kx + a.b0[1] * ky + a.b0[2] * kz;
        const double f = K2 > 0 ? bk * bk / K2 : 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const cx<double> v = a.inprec ? ldc<float>(a.IN[c], gi) : ldc<double>(a.IN[c], gi);
          r[c] = r[c] + f * v;
        }
      }
      if constexpr (PHYS == PH_RB) {
        // Compute_force_RB (compute_force_RB.cc:51-105) from the stage's fields, then Add_force:
        // nlin1 -= fu * theta, T.nlin -= ft * u1
        const cx<double> th = a.inprec ? ldc<float>(a.IN[3], gi) : ldc<double>(a.IN[3], gi);
        const cx<double> u1 = a.inprec ? ldc<float>(a.IN[0], gi) : ldc<double>(a.IN[0], gi);
        r[0] = r[0] - a.rb_buoy_u * th;
        r[3] = r[3] - a.rb_buoy_t * u1;
      }
      project_rhs(r, NS, dx, ky, kz, K2);
    } else {
#pragma unroll
      for (int c = 0; c < NS; ++c) r[c] = a.RHS[c][gi];
    }
    const int l1 = geo_l1(g, r1), l2 = amap_index(g.ay, r2);
    double eh = 0, e1 = 0;
#pragma unroll
    for (int c = 0; c < NS; ++c) {
      if (c == 0 || nus[c] != nus[c - 1] || nuh[c] != nuh[c - 1]) {
        // nu + nu_h K^2 (nu exactly when the hyper term is off)
        const double nuk = nuh[c] != 0.0 ? nus[c] + nuh[c] * K2 : nus[c];
        eh = exp(-nuk * 0.5 * dt * K2);
        if constexpr (STAGE == 1 || STAGE == 4 || STAGE == 5) e1 = exp(-nuk * dt * K2);
      }
      const cx<double> rc = r[c];
      if constexpr (STAGE == 1) {
        stc<Rs>(a.US[c], gi, eh * (u0[c] + (0.5 * dt) * rc));
        a.TOT[c][gi] = (dt / 6.0) * (e1 * rc);
      } else if constexpr (STAGE == 2) {
        stc<Rs>(a.US[c], gi, eh * u0[c] + (0.5 * dt) * rc);
        a.TOT[c][gi] = tot[c] + (dt / 3.0) * (eh * rc);
      } else if constexpr (STAGE == 3) {
        stc<Rs>(a.US[c], gi, eh * (eh * u0[c] + dt * rc));
        a.TOT[c][gi] = tot[c] + (dt / 3.0) * (eh * rc);
      } else if constexpr (STAGE == 7) {
        stc<Rs>(a.US[c], gi, eh * (u0[c] + (0.5 * dt) * rc));
      } else {
        cx<double> u;
        if constexpr (STAGE == 4) u = e1 * u0[c] + (tot[c] + (dt / 6.0) * rc);
        else if constexpr (STAGE == 5) u = e1 * (u0[c] + dt * rc);
        else u = eh * (eh * u0[c] + dt * rc);
        a.U0[c][gi] = u;
        const double m2 = u.x * u.x + u.y * u.y;
        const int grp = (PHYS == PH_MHD) ? (c / 3) * 2 : (c < 3 ? 0 : 4);
        double w, m;
        if (g.basis == 0) {
          w = energy_weight_four(l1, l2, l3, g.N1, g.N2);
          m = mult_four(l1, l2, l3, g.N1, g.N2);
        } else {
          // Get_total_energy_SCFT (scft_energy.cc:51-104): multiplicity, origin excluded
          m = mult_scft(l1, l2, l3, g.N2);
          w = (l1 == 0 && l2 == 0 && l3 == 0) ? m - 0.5 : m;
        }
        acc[grp] += w * m2;
        acc[grp + 1] += m * K2 * m2;
      }
    }
  }
  if constexpr (FINAL) {
    if (a.part != nullptr) {
      block_sum<6>(acc);
      if (threadIdx.x == 0) {
#pragma unroll
        for (int j = 0; j < 6; ++j) a.part[((long long)blockIdx.y * gridDim.x + blockIdx.x) * 8 + j] = acc[j];
      }
    }
  }
}

template <typename Rp, typename Rs, int PHYS>
cudaError_t run_rk_src(const RKArgs& a, int src, cudaStream_t s, int nblk) {
  const dim3 grid(nblk, a.nact > 0 ? a.nact : 1);
  if (src == 1) {
    // precomputed right-hand sides enter at a scheme's first stage only (Time_advance after
    // Compute_rhs): RK4 1, EULER 5, RK2 7
    switch (a.stage) {
      case 1: k_rk<Rp, Rs, PHYS, 1, 1><<<grid, TPB, 0, s>>>(a); break;
      case 5: k_rk<Rp, Rs, PHYS, 1, 5><<<grid, TPB, 0, s>>>(a); break;
      case 7: k_rk<Rp, Rs, PHYS, 1, 7><<<grid, TPB, 0, s>>>(a); break;
      default: return cudaErrorInvalidValue;
    }
  } else {
    switch (a.stage) {
      case 1: k_rk<Rp, Rs, PHYS, 0, 1><<<grid, TPB, 0, s>>>(a); break;
      case 2: k_rk<Rp, Rs, PHYS, 0, 2><<<grid, TPB, 0, s>>>(a); break;
      case 3: k_rk<Rp, Rs, PHYS, 0, 3><<<grid, TPB, 0, s>>>(a); break;
      case 4: k_rk<Rp, Rs, PHYS, 0, 4><<<grid, TPB, 0, s>>>(a); break;
      case 5: k_rk<Rp, Rs, PHYS, 0, 5><<<grid, TPB, 0, s>>>(a); break;
      case 6: k_rk<Rp, Rs, PHYS, 0, 6><<<grid, TPB, 0, s>>>(a); break;
      case 7: k_rk<Rp, Rs, PHYS, 0, 7><<<grid, TPB, 0, s>>>(a); break;
      default: return cudaErrorInvalidValue;
    }
  }
  return cudaGetLastError();
}
template <typename Rp, typename Rs>
cudaError_t run_rk_phys(const RKArgs& a, int phys, int src, cudaStream_t s, int nblk) {
  switch (phys) {
    case PH_FLUID: return run_rk_src<Rp, Rs, PH_FLUID>(a, src, s, nblk);
    case PH_MHD: return run_rk_src<Rp, Rs, PH_MHD>(a, src, s, nblk);
    case PH_SCALAR: return run_rk_src<Rp, Rs, PH_SCALAR>(a, src, s, nblk);
    case PH_RB: return run_rk_src<Rp, Rs, PH_RB>(a, src, s, nblk);
    default: return cudaErrorInvalidValue;
  }
}

// ------------------------------------------------------------------ forcing
// Band forcings on inner < |K| <= outer (FOUR), mode by mode from the current field:
//   proc 1, Compute_force_const_energy_helicity_supply (compute_force_ek_hk_supply.cc:51-437):
//     temp = e/(2 E_k), alpha = temp (1 - s h)/(1 - s^2), beta = temp (h - s)/(1 - s^2),
//     |s^2 - 1| <= MYEPS2: alpha = temp/2, beta = alpha/(s k);
//   proc 2, Compute_force_const_energy_helicity (compute_force_const_ek_hk.cc:53-446):
//     t1 = sqrt(e/E_k), t2 = sqrt((1 + h)/(1 + s)), t3 = sqrt((1 - h)/(1 - s)),
//     alpha = t1 (t2 + t3)/2, beta = t1 (t2 - t3)/(2 k); |s^2 - 1| <= MYEPS2: alpha = t1, beta = 0;
// with s = H_k/(k E_k), F = alpha V + beta omega (Force_alpha_beta force_alpha_beta.cc:60-88; the
// vorticity only when beta > MYEPS), the same for B with its own (e, h) in MHD, and for a passive
// scalar F_T = alpha_T T, alpha_T = e_T/E_T (proc 1) or sqrt(e_T/E_T) (proc 2)
// (Force_scalar_alpha force_alpha_beta.cc:183-198); then the reality condition of every force
// component (Satisfy_reality_array universal_misc.cc:51-109).  One block.
// v: the mode in the Fourier basis (SCFT: (-i V1, V2, V3)); wE: the modal-energy weight, 1/2
// (Modal_energy_FOUR, and SCFT at kx = 0) or 1 (Modal_energy_SCFT at kx > 0, scft_inline.h:347)
__device__ __forceinline__ void band_alpha_beta(int mode, const cx<double> (&v)[3], double kkx, double kky, double kkz,
                                                double km, double e, double h, double wE, double& alpha,
                                                double& beta, bool& on) {
  const double Ek = wE * (v[0].x * v[0].x + v[0].y * v[0].y + v[1].x * v[1].x + v[1].y * v[1].y +
                          v[2].x * v[2].x + v[2].y * v[2].y);
  on = Ek > 1e-15;
  alpha = beta = 0;
  if (!on) return;
  // modal helicity k . (Vr x Vi)  (Get_Modal_helicity_FOUR four_basic.cc:136-155)
  const double cx_ = v[1].x * v[2].y - v[2].x * v[1].y;
  const double cy_ = v[2].x * v[0].y - v[0].x * v[2].y;
  const double cz_ = v[0].x * v[1].y - v[1].x * v[0].y;
  const double Hk = kkx * cx_ + kky * cy_ + kkz * cz_;
  const double sk = Hk / (km * Ek);
  if (mode == 1) {
    const double temp = e / (2 * Ek);
    if (fabs(sk * sk - 1) > 1e-5) {
      alpha = temp * (1 - sk * h) / (1 - sk * sk);
      beta = temp * (h - sk) / (1 - sk * sk);
    } else {
      alpha = temp / 2;
      beta = alpha / (sk * km);
    }
  } else {
    const double t1 = sqrt(e / Ek);
    if (fabs(sk * sk - 1) > 1e-5) {
      const double t2 = sqrt((1 + h) / (1 + sk)), t3 = sqrt((1 - h) / (1 - sk));
      alpha = (t1 / 2) * (t2 + t3);
      beta = (t1 / (2 * km)) * (t2 - t3);
    } else {
      alpha = t1;
      beta = 0;
    }
  }
}

// scft: the mode is a sin/cos-Fourier one (kx >= 0): the helicity and vorticity take
// (-i V1, V2, V3) (Get_Modal_helicity_SCFT, Compute_Modal_vorticity_SCFT scft_basic.cc:137-186),
// the modal energy Modal_energy_SCFT, and Force_alpha_beta's SCFT form gives
// F1 = I (alpha (-I) V1 + beta omega_1) = alpha V1 + i beta omega_1 (force_alpha_beta.cc:90-110)
__device__ __forceinline__ void band_vector_force(int mode, const cx<double> (&v)[3], double kkx, double kky,
                                                  double kkz, double km, double e, double h, bool scft, int kx,
                                                  cx<double> (&F)[3]) {
  const cx<double> vf[3] = {scft ? mkc<double>(v[0].y, -v[0].x) : v[0], v[1], v[2]};
  const double wE = (scft && kx > 0) ? 1.0 : 0.5;
  double alpha, beta;
  bool on;
  band_alpha_beta(mode, vf, kkx, kky, kkz, km, e, h, wE, alpha, beta, on);
  if (!on) return;
  cx<double> w[3] = {mkc<double>(0, 0), mkc<double>(0, 0), mkc<double>(0, 0)};
  if (beta > 1e-15) {
    // vorticity i K x V (Compute_Modal_vorticity_FOUR four_basic.cc:166-186)
    w[0] = ione(kky * vf[2] - kkz * vf[1]);
    w[1] = ione(kkz * vf[0] - kkx * vf[2]);
    w[2] = ione(kkx * vf[1] - kky * vf[0]);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) F[c] = alpha * v[c] + beta * w[c];
  if (scft) F[0] = alpha * v[0] + ione(beta * w[0]);
}

template <typename Ru>
__global__ void __launch_bounds__(TPB) k_force_supply(ForceArgs a) {
  const Geo& g = a.g;
  const int ny = 2 * a.fy + 1, nz = a.fz + 1;
  const int box = (2 * a.fx + 1) * ny * nz;
  const bool scft = g.basis == 1;  // SCFT: kx >= 0 only (kx_min = 0, compute_force_ek_hk_supply.cc:91-95)
  for (int p = threadIdx.x; p < box; p += TPB) {
    const int kz = p % nz;
    const int ky = (p / nz) % ny - a.fy;
    const int kx = p / (nz * ny) - a.fx;
    cx<double> F[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) F[c] = mkc<double>(0, 0);
    const double kkx = kx * g.kf0, kky = ky * g.kf1, kkz = kz * g.kf2;
    const double km = sqrt(kkx * kkx + kky * kky + kkz * kkz);
    if (km > a.inner && km <= a.outer && !(scft && kx < 0)) {
      const int lx = (kx >= 0 || scft) ? kx : kx + g.N1;
      const int ly = ky >= 0 ? ky : ky + g.N2;
      const int r1 = (lx >= 0 && lx < g.N1) ? amap_row(g.ax, lx) : -1;
      const int r2 = (ly >= 0 && ly < g.N2) ? amap_row(g.ay, ly) : -1;
      cx<double> v[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) v[c] = mkc<double>(0, 0);
      if (r1 >= 0 && r2 >= 0 && kz < g.nkz) {
        const long long i = ((long long)r1 * g.nky + r2) * g.kzp + kz;
        for (int c = 0; c < a.ns; ++c) v[c] = ldc<Ru>(a.U[c], i);
      }
      if (!a.gate || a.e_per_mode > 1e-15) {
        const cx<double> u[3] = {v[0], v[1], v[2]};
        cx<double> f[3] = {F[0], F[1], F[2]};
        band_vector_force(a.mode, u, kkx, kky, kkz, km, a.e_per_mode, a.eps_h, scft, kx, f);
        F[0] = f[0];
        F[1] = f[1];
        F[2] = f[2];
      }
      if (a.ns == 6 && a.e_per_mode_b > 1e-15) {
        const cx<double> b[3] = {v[3], v[4], v[5]};
        cx<double> f[3] = {F[3], F[4], F[5]};
        band_vector_force(a.mode, b, kkx, kky, kkz, km, a.e_per_mode_b, a.eps_h_b, scft, kx, f);
        F[3] = f[0];
        F[4] = f[1];
        F[5] = f[2];
      } else if (a.ns == 4 && a.e_per_mode_b > 1e-15) {
        // CS_Modal_energy: |T|^2/2 (FOUR; SCFT at kx = 0), |T|^2 (SCFT, kx > 0)
        const double Et = ((scft && kx > 0) ? 1.0 : 0.5) * (v[3].x * v[3].x + v[3].y * v[3].y);
        if (Et > 1e-15) {
          const double al = a.mode == 1 ? a.e_per_mode_b / Et : sqrt(a.e_per_mode_b / Et);
          F[3] = al * v[3];
        }
      }
    }
    for (int c = 0; c < a.ns; ++c) a.FB[(long long)c * box + p] = F[c];
  }
  __syncthreads();
  // reality condition on the kz = 0 plane: F(kx, ky<0) = conj F(-kx, -ky); F(kx<0, 0) = conj F(-kx, 0)
  // (FOUR); F(kx, ky<0) = conj F(kx, -ky) (SCFT, Satisfy_reality_array universal_misc.cc:93-104)
  for (int p = threadIdx.x; p < box; p += TPB) {
    const int kz = p % nz;
    const int ky = (p / nz) % ny - a.fy;
    const int kx = p / (nz * ny) - a.fx;
    if (kz != 0) continue;
    if (scft ? !(ky < 0 && kx >= 0) : !(ky < 0 || (ky == 0 && kx < 0))) continue;
    const int mx = scft ? kx : -kx, my = -ky;
    if (mx < -a.fx || mx > a.fx || my < -a.fy || my > a.fy) continue;
    const int pm = ((mx + a.fx) * ny + (my + a.fy)) * nz;
    for (int c = 0; c < a.ns; ++c) a.FB[(long long)c * box + p] = conjc(a.FB[(long long)c * box + pm]);
  }
}

// ------------------------------------------------------------------ fine-grained API kernels
template <typename Rp, int PHYS>
__global__ void k_assemble(Geo g, const void* const* PXd, cx<double>* const* NLd) {
  constexpr int NS = NState<PHYS>::v;
  const long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
  if (idx >= g.S) return;
  int r1, r2, l3;
  compact_mode(g, idx, r1, r2, l3);
  cx<double> n[NS];
  if (l3 < g.nkz) {
    const double kx = geo_kx(g, r1) * g.kf0, ky = geo_ky(g, r2) * g.kf1, kz = l3 * g.kf2;
    assemble<Rp, PHYS>(PXd, idx, kx, ky, kz, n);
  } else {
#pragma unroll
    for (int c = 0; c < NS; ++c) n[c] = mkc<double>(0, 0);
  }
#pragma unroll
  for (int c = 0; c < NS; ++c) NLd[c][idx] = n[c];
}

struct PtrArr6 {
  cx<double>* p[6];
  const void* q[9];
};

template <typename Rp, int PHYS>
__global__ void k_assemble_v(Geo g, PtrArr6 pa) {
  constexpr int NS = NState<PHYS>::v;
  const long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
  if (idx >= g.S) return;
  int r1, r2, l3;
  compact_mode(g, idx, r1, r2, l3);
  cx<double> n[NS];
  if (l3 < g.nkz) {
    const double kx = geo_kx(g, r1) * g.kf0, ky = geo_ky(g, r2) * g.kf1, kz = l3 * g.kf2;
    assemble<Rp, PHYS>(pa.q, idx, XDer{kx, g.basis}, ky, kz, n);
  } else {
#pragma unroll
    for (int c = 0; c < NS; ++c) n[c] = mkc<double>(0, 0);
  }
#pragma unroll
  for (int c = 0; c < NS; ++c) pa.p[c][idx] = n[c];
}

__global__ void k_sub_force_box(Geo g, int ncomp, const cx<double>* FB, int fx, int fy, int fz, PtrArr6 pa) {
  const int ny = 2 * fy + 1, nz = fz + 1;
  const int box = (2 * fx + 1) * ny * nz;
  const int p = blockIdx.x * TPB + threadIdx.x;
  if (p >= box) return;
  const int kz = p % nz;
  const int ky = (p / nz) % ny - fy;
  const int kx = p / (nz * ny) - fx;
  if (g.basis == 1 && kx < 0) return;  // SCFT: kx >= 0
  const int lx = kx >= 0 ? kx : kx + g.N1;
  const int ly = ky >= 0 ? ky : ky + g.N2;
  if (lx < 0 || lx >= g.N1 || ly < 0 || ly >= g.N2 || kz >= g.nkz) return;
  const int r1 = amap_row(g.ax, lx), r2 = amap_row(g.ay, ly);
  if (r1 < 0 || r2 < 0) return;
  const long long i = ((long long)r1 * g.nky + r2) * g.kzp + kz;
  for (int c = 0; c < ncomp; ++c) pa.p[c][i] = pa.p[c][i] - FB[(long long)c * box + p];
}

__global__ void k_pressure(Geo g, PtrArr6 pa, cx<double>* PR) {
  const long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
  if (idx >= g.S) return;
  int r1, r2, l3;
  compact_mode(g, idx, r1, r2, l3);
  cx<double> p = mkc<double>(0, 0);
  if (l3 < g.nkz) {
    const double kx = geo_kx(g, r1) * g.kf0, ky = geo_ky(g, r2) * g.kf1, kz = l3 * g.kf2;
    const double K2 = kx * kx + ky * ky + kz * kz;
    // Compute_divergence_nlin (Xderiv of nlin1 with parity 1) then CS_divide_ksqr (A(0,0,0) = 0)
    const XDer dx{kx, g.basis};
    if (K2 > 0) p = (1.0 / K2) * (dx.sin_in(pa.p[0][idx]) + iky_ikz(ky, kz, pa.p[1][idx], pa.p[2][idx]));
  }
  PR[idx] = p;
}

__global__ void k_rhs_from_nlin(Geo g, int ns, PtrArr6 pa, const cx<double>* PR) {
  const long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
  if (idx >= g.S) return;
  int r1, r2, l3;
  compact_mode(g, idx, r1, r2, l3);
  if (l3 >= g.nkz) return;
  const double kx = geo_kx(g, r1) * g.kf0, ky = geo_ky(g, r2) * g.kf1, kz = l3 * g.kf2;
  const cx<double> p = PR[idx];
  // Add_pressure_gradient (Xderiv of p with parity 0, Yderiv, Zderiv); Compute_rhs: nlin = -nlin
  const cx<double> g0 = XDer{kx, g.basis}.cos_in(p), g1 = ione(ky * p), g2 = ione(kz * p);
  pa.p[0][idx] = mkc<double>(0, 0) - (pa.p[0][idx] + g0);
  pa.p[1][idx] = mkc<double>(0, 0) - (pa.p[1][idx] + g1);
  pa.p[2][idx] = mkc<double>(0, 0) - (pa.p[2][idx] + g2);
  for (int c = 3; c < ns; ++c) pa.p[c][idx] = mkc<double>(0, 0) - pa.p[c][idx];
}

// Add_force(T) for RB (add_force.cc:62-68) with Compute_force_RB: nlin1 -= fu theta,
// T.nlin -= ft u1 (theta, u1 from the master state)
__global__ void k_rb_sub_force(Geo g, PtrArr6 pa, const cx<double>* u1, const cx<double>* th, double fu, double ft) {
  const long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
  if (idx >= g.S) return;
  pa.p[0][idx] = pa.p[0][idx] - fu * th[idx];
  pa.p[3][idx] = pa.p[3][idx] - ft * u1[idx];
}

__global__ void k_sub_liquid_metal(Geo g, PtrArr6 nl, PtrArr6 u, double b0, double b1, double b2) {
  const long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
  if (idx >= g.S) return;
  int r1, r2, l3;
  compact_mode(g, idx, r1, r2, l3);
  const double kx = geo_kx(g, r1) * g.kf0, ky = geo_ky(g, r2) * g.kf1, kz = l3 * g.kf2;
  const double K2 = kx * kx + ky * ky + kz * kz, bk = b0 * kx + b1 * ky + b2 * kz;
  const double f = K2 > 0 ? bk * bk / K2 : 0.0;
#pragma unroll
  for (int c = 0; c < 3; ++c) nl.p[c][idx] = nl.p[c][idx] + f * u.p[c][idx];
}

__global__ void k_sub_coriolis(Geo g, PtrArr6 nl, PtrArr6 u, double o0, double o1, double o2) {
  const long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
  if (idx >= g.S) return;
  const cx<double> v0 = u.p[0][idx], v1 = u.p[1][idx], v2 = u.p[2][idx];
  nl.p[0][idx] = nl.p[0][idx] - (o1 * v2 - o2 * v1);
  nl.p[1][idx] = nl.p[1][idx] - (o2 * v0 - o0 * v2);
  nl.p[2][idx] = nl.p[2][idx] - (o0 * v1 - o1 * v0);
}

// ------------------------------------------------------------------ reductions
// cross energy Re(A B*) with the energy weights (Get_total_energy(A, B), four_energy.cc:108-168,
// scft_energy.cc:108-158), per block into part[b * nslots + slot]
__global__ void __launch_bounds__(TPB) k_cross_partials(Geo g, const cx<double>* A, const cx<double>* B, double* part, int slot, int nslots) {
  double acc[1] = {0};
  const long long stride = (long long)gridDim.x * TPB;
  for (long long idx = (long long)blockIdx.x * TPB + threadIdx.x; idx < g.S; idx += stride) {
    int r1, r2, l3;
    compact_mode(g, idx, r1, r2, l3);
    if (l3 >= g.nkz) continue;
    const int l1 = geo_l1(g, r1), l2 = amap_index(g.ay, r2);
    double w;
    if (g.basis == 0) {
      w = energy_weight_four(l1, l2, l3, g.N1, g.N2);
    } else {
      const double m = mult_scft(l1, l2, l3, g.N2);
      w = (l1 == 0 && l2 == 0 && l3 == 0) ? m - 0.5 : m;
    }
    const cx<double> a = A[idx], b = B[idx];
    acc[0] += w * (a.x * b.x + a.y * b.y);
  }
  block_sum<1>(acc);
  if (threadIdx.x == 0) part[(long long)blockIdx.x * nslots + slot] = acc[0];
}

__global__ void __launch_bounds__(TPB) k_energy_partials(Geo g, PtrArr6 pa, int nf, double* part, int slot, int nslots) {
  double acc[2] = {0, 0};
  const long long stride = (long long)gridDim.x * TPB;
  for (long long idx = (long long)blockIdx.x * TPB + threadIdx.x; idx < g.S; idx += stride) {
    int r1, r2, l3;
    compact_mode(g, idx, r1, r2, l3);
    if (l3 < g.nkz) {
      const int l1 = geo_l1(g, r1), l2 = amap_index(g.ay, r2);
      const double kx = geo_kx(g, r1) * g.kf0, ky = geo_ky(g, r2) * g.kf1, kz = l3 * g.kf2;
      const double K2 = kx * kx + ky * ky + kz * kz;
      double w, m;
      if (g.basis == 0) {
        w = energy_weight_four(l1, l2, l3, g.N1, g.N2);
        m = mult_four(l1, l2, l3, g.N1, g.N2);
      } else {
        m = mult_scft(l1, l2, l3, g.N2);
        w = (l1 == 0 && l2 == 0 && l3 == 0) ? m - 0.5 : m;
      }
      for (int c = 0; c < nf; ++c) {
        const cx<double> u = pa.p[c][(long long)blockIdx.y * g.S + idx];
        const double m2 = u.x * u.x + u.y * u.y;
        acc[0] += w * m2;
        acc[1] += m * K2 * m2;
      }
    }
  }
  block_sum<2>(acc);
  if (threadIdx.x == 0) {
    const long long b = (long long)blockIdx.y * gridDim.x + blockIdx.x;
    part[b * nslots + slot] = acc[0];
    part[b * nslots + slot + 1] = acc[1];
  }
}

// one block per request r: sums its partials in a fixed order, then the dt rule of Get_dt
// (compute_dt.cc:47-108); scal[8 r + 0..4] = dt, t, steps, non-finite flag, Tdt
__global__ void __launch_bounds__(TPB) k_finalize(FinalizeArgs a) {
  __shared__ double red[TPB];
  const int r = blockIdx.x;
  const double* part = a.part + (long long)r * a.nblocks * a.nslots;
  double* out = a.out + (long long)r * a.nslots;
  double* scal = a.scal + (long long)r * 8;
  for (int j = 0; j < a.nslots; ++j) {
    double s = 0;
    for (int b = threadIdx.x; b < a.nblocks; b += TPB) s += part[(long long)b * a.nslots + j];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = TPB / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[j] = red[0];
    __syncthreads();
  }
  if (threadIdx.x != 0 || a.dt_mode == 0) return;
  const double Tdt = scal[4] > 0 ? scal[4] : a.Tdt;
  const double E = out[0] + (a.mhd ? out[2] : 0.0);
  if (a.dt_mode == 1) {
    // the step that just ended advanced the time by dt
    scal[1] += scal[0];
    scal[2] += 1.0;
    if (!(E == E) || E > 1e300 || E < -1e300) scal[3] = 1.0;
    if (a.ering != nullptr && r == 0) {
      const int pos = *a.ering_pos;
      a.ering[pos] = E;
      *a.ering_pos = pos + 1;
    }
  }
  double dt = (E > 0) ? a.dx / (sqrt(E) * 20.0) : Tdt;
  if (a.mhd && a.B0[0] != nullptr) {
    const long long o = (long long)r * a.S;
    const double b0 = a.B0[0][o].x, b1 = a.B0[1][o].x, b2 = a.B0[2][o].x;
    const double B0sqr = b0 * b0 + b1 * b1 + b2 * b2;
    if (B0sqr > 1e-15) dt = fmin(dt, a.dx / (sqrt(B0sqr) * 20.0));
  }
  scal[0] = fmin(dt, Tdt);
}

// Shell sums of the fields' energies (and the mode counts) in a fixed order: per warp a row of
// bins (warp_bin_add: the lanes of a shell in lane order), the block's rows in warp order into
// part[block], then k_bins_accumulate adds the blocks in block order to ek / cnt -- the same bits
// on every run
__global__ void __launch_bounds__(TPB) k_shell_spectrum(Geo g, PtrArr6 pa, int nf, double n_pow, double* part,
                                                        int nbins) {
  constexpr int W = TPB / 32;
  extern __shared__ double sh[];  // [W][(nf + 1) * nbins]
  const int row = (nf + 1) * nbins;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < W * row; i += TPB) sh[i] = 0;
  __syncthreads();
  double* mine = sh + (size_t)warp * row;
  const long long stride = (long long)gridDim.x * TPB;
  for (long long w0 = (long long)blockIdx.x * TPB + warp * 32; w0 < g.S; w0 += stride) {
    const long long idx = w0 + lane;
    bool active = idx < g.S;
    int r1 = 0, r2 = 0, l3 = 0, bin = 0;
    double m = 0, kp = 0;
    if (active) {
      compact_mode(g, idx, r1, r2, l3);
      active = l3 < g.nkz;
    }
    if (active) {
      const int l1 = geo_l1(g, r1), l2 = amap_index(g.ay, r2);
      const double kx = geo_kx(g, r1) * g.kf0, ky = geo_ky(g, r2) * g.kf1, kz = l3 * g.kf2;
      const double K = sqrt(kx * kx + ky * ky + kz * kz);
      bin = (int)ceil(K);
      active = bin < nbins;
      m = (g.basis == 0) ? mult_four(l1, l2, l3, g.N1, g.N2) : mult_scft(l1, l2, l3, g.N2);
      kp = (n_pow == 0.0) ? 1.0 : pow(K, n_pow);
    }
    for (int c = 0; c < nf; ++c) {
      double v = 0;
      if (active) {
        const cx<double> u = pa.p[c][idx];
        v = m * kp * (u.x * u.x + u.y * u.y);
      }
      warp_bin_add(mine + c * nbins, bin, v, active);
    }
    warp_bin_add(mine + nf * nbins, bin, g.basis == 0 ? m : 0.5 * m, active);  // SCFT counts factor/2 (scft_energy.cc:279)
  }
  __syncthreads();
  for (int i = threadIdx.x; i < row; i += TPB) {
    double t = 0;
    for (int w = 0; w < W; ++w) t += sh[(size_t)w * row + i];
    part[(size_t)blockIdx.x * row + i] = t;
  }
}

// out[i] += the blocks' part[b][i] in block order (i < n), one thread per bin
__global__ void k_bins_accumulate(const double* __restrict__ part, int nblocks, int n, double* out0, int n0,
                                  double* out1) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double t = 0;
  for (int b = 0; b < nblocks; ++b) t += part[(size_t)b * n + i];
  if (i < n0) out0[i] += t;
  else out1[i - n0] += t;
}

inline int nblk(long long n) { return (int)((n + TPB - 1) / TPB); }
// reducing kernels: whole waves on 148 SMs (2 waves of the RK kernel at 3 blocks per SM, 3 at 2)
inline int nred(long long n) { return nblk(n) < 148 * 6 ? nblk(n) : 148 * 6; }

}  // namespace

int reduction_blocks(long long S) { return nred(S); }

cudaError_t launch_dense_to_compact(const Geo& g, const cx<double>* dense, void* compact, int cprec, cudaStream_t s) {
  if (cprec == 0) k_dense_to_compact<double><<<nblk(g.S), TPB, 0, s>>>(g, dense, (cx<double>*)compact);
  else k_dense_to_compact<float><<<nblk(g.S), TPB, 0, s>>>(g, dense, (cx<float>*)compact);
  return cudaGetLastError();
}

cudaError_t launch_compact_to_dense(const Geo& g, const void* compact, int cprec, cx<double>* dense, cudaStream_t s) {
  const long long D = (long long)g.N1 * g.N2 * (g.N3 / 2 + 1);
  if (cprec == 0) k_compact_to_dense<double><<<nblk(D), TPB, 0, s>>>(g, (const cx<double>*)compact, dense);
  else k_compact_to_dense<float><<<nblk(D), TPB, 0, s>>>(g, (const cx<float>*)compact, dense);
  return cudaGetLastError();
}

cudaError_t launch_rk(const RKArgs& a, int phys, int pprec, int sprec, int src, cudaStream_t s, int* nblocks) {
  const int nb = nred(a.g.S);
  if (nblocks) *nblocks = nb;
  if (pprec == 0 && sprec == 0) return run_rk_phys<double, double>(a, phys, src, s, nb);
  if (pprec == 1 && sprec == 1) return run_rk_phys<float, float>(a, phys, src, s, nb);
  return cudaErrorInvalidValue;
}

cudaError_t launch_force_supply(const ForceArgs& a, cudaStream_t s) {
  if (a.uprec == 0) k_force_supply<double><<<1, TPB, 0, s>>>(a);
  else k_force_supply<float><<<1, TPB, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_assemble_nlin(const Geo& g, int phys, int pprec, const void* const* PX, cx<double>* const* NL, cudaStream_t s) {
  PtrArr6 pa{};
  const int ns = phys == PH_FLUID ? 3 : (phys == PH_MHD ? 6 : 4);
  const int np = phys == PH_FLUID ? 6 : 9;
  for (int c = 0; c < ns; ++c) pa.p[c] = NL[c];
  for (int q = 0; q < np; ++q) pa.q[q] = PX[q];
  const int nb = nblk(g.S);
#define TG_ASM(RP)                                                         \
  switch (phys) {                                                          \
    case PH_FLUID: k_assemble_v<RP, PH_FLUID><<<nb, TPB, 0, s>>>(g, pa); break; \
    case PH_MHD: k_assemble_v<RP, PH_MHD><<<nb, TPB, 0, s>>>(g, pa); break;     \
    default: k_assemble_v<RP, PH_SCALAR><<<nb, TPB, 0, s>>>(g, pa); break;      \
  }
  if (pprec == 0) {
    TG_ASM(double)
  } else {
    TG_ASM(float)
  }
#undef TG_ASM
  return cudaGetLastError();
}

cudaError_t launch_sub_force_box(const Geo& g, int ncomp, const cx<double>* FB, int fx, int fy, int fz, cx<double>* const* NL, cudaStream_t s) {
  PtrArr6 pa{};
  for (int c = 0; c < ncomp; ++c) pa.p[c] = NL[c];
  const int box = (2 * fx + 1) * (2 * fy + 1) * (fz + 1);
  k_sub_force_box<<<(box + TPB - 1) / TPB, TPB, 0, s>>>(g, ncomp, FB, fx, fy, fz, pa);
  return cudaGetLastError();
}

cudaError_t launch_pressure(const Geo& g, const cx<double>* const* NL, cx<double>* PR, cudaStream_t s) {
  PtrArr6 pa{};
  for (int c = 0; c < 3; ++c) pa.p[c] = const_cast<cx<double>*>(NL[c]);
  k_pressure<<<nblk(g.S), TPB, 0, s>>>(g, pa, PR);
  return cudaGetLastError();
}

cudaError_t launch_rhs_from_nlin(const Geo& g, int phys, cx<double>* const* NL, const cx<double>* PR, cudaStream_t s) {
  PtrArr6 pa{};
  const int ns = phys == PH_FLUID ? 3 : (phys == PH_MHD ? 6 : 4);
  for (int c = 0; c < ns; ++c) pa.p[c] = NL[c];
  k_rhs_from_nlin<<<nblk(g.S), TPB, 0, s>>>(g, ns, pa, PR);
  return cudaGetLastError();
}

cudaError_t launch_rb_sub_force(const Geo& g, cx<double>* const* NL, const cx<double>* u1, const cx<double>* th,
                                double fu, double ft, cudaStream_t s) {
  PtrArr6 pa{};
  for (int c = 0; c < 4; ++c) pa.p[c] = NL[c];
  k_rb_sub_force<<<nblk(g.S), TPB, 0, s>>>(g, pa, u1, th, fu, ft);
  return cudaGetLastError();
}

cudaError_t launch_sub_liquid_metal(const Geo& g, cx<double>* const* NL, const cx<double>* const* U, const double* b0,
                                    cudaStream_t s) {
  PtrArr6 nl{}, u{};
  for (int c = 0; c < 3; ++c) {
    nl.p[c] = NL[c];
    u.p[c] = const_cast<cx<double>*>(U[c]);
  }
  k_sub_liquid_metal<<<nblk(g.S), TPB, 0, s>>>(g, nl, u, b0[0], b0[1], b0[2]);
  return cudaGetLastError();
}

cudaError_t launch_sub_coriolis(const Geo& g, cx<double>* const* NL, const cx<double>* const* U, const double* om,
                                cudaStream_t s) {
  PtrArr6 nl{}, u{};
  for (int c = 0; c < 3; ++c) {
    nl.p[c] = NL[c];
    u.p[c] = const_cast<cx<double>*>(U[c]);
  }
  k_sub_coriolis<<<nblk(g.S), TPB, 0, s>>>(g, nl, u, om[0], om[1], om[2]);
  return cudaGetLastError();
}

cudaError_t launch_cross_partials(const Geo& g, const cx<double>* A, const cx<double>* B, double* part, int slot,
                                  int nslots, cudaStream_t s, int* nblocks) {
  const int nb = nred(g.S);
  if (nblocks) *nblocks = nb;
  k_cross_partials<<<nb, TPB, 0, s>>>(g, A, B, part, slot, nslots);
  return cudaGetLastError();
}

cudaError_t launch_energy_partials(const Geo& g, const cx<double>* const* F, int nf, double* part, int slot, int nslots, cudaStream_t s, int* nblocks, int nact) {
  PtrArr6 pa{};
  for (int c = 0; c < nf; ++c) pa.p[c] = const_cast<cx<double>*>(F[c]);
  const int nb = nred(g.S);
  if (nblocks) *nblocks = nb;
  k_energy_partials<<<dim3(nb, nact > 0 ? nact : 1), TPB, 0, s>>>(g, pa, nf, part, slot, nslots);
  return cudaGetLastError();
}

cudaError_t launch_finalize(const FinalizeArgs& a, cudaStream_t s) {
  k_finalize<<<a.nact > 0 ? a.nact : 1, TPB, 0, s>>>(a);
  return cudaGetLastError();
}

int shell_spectrum_blocks(const Geo& g) {
  int nb = nblk(g.S);
  return nb > 148 * 8 ? 148 * 8 : nb;
}

cudaError_t launch_shell_spectrum(const Geo& g, const cx<double>* const* F, int nf, double n_pow, double* ek, double* cnt,
                                  int nbins, double* part, cudaStream_t s) {
  PtrArr6 pa{};
  for (int c = 0; c < nf; ++c) pa.p[c] = const_cast<cx<double>*>(F[c]);
  const int row = (nf + 1) * nbins;
  const size_t smem = (size_t)(TPB / 32) * row * sizeof(double);
  if (smem > 200 * 1024) return cudaErrorInvalidValue;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_shell_spectrum, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  const int nb = shell_spectrum_blocks(g);
  k_shell_spectrum<<<nb, TPB, smem, s>>>(g, pa, nf, n_pow, part, nbins);
  k_bins_accumulate<<<(row + 127) / 128, 128, 0, s>>>(part, nb, row, ek, nf * nbins, cnt);
  return cudaGetLastError();
}

}  // namespace tg
