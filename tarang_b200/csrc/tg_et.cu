// Energy transfer diagnostics: shell radii, flux Pi(R) and shell-to-shell transfer.
//
// The reference evaluates the energy-transfer nonlinearity N_i = D_j F(H_j G_i)
// (IncVF::EnergyTr_Compute_nlin, ET_compute_nlin.cc:85-251) once per sphere for the flux
// (compute_flux.cc:52-304, G = field inside sphere s) and once per shell for the
// shell-to-shell transfer (compute_shell_tr.cc:59-281, G = field in shell n): 2S-1
// evaluations of 15 transforms each.  N is linear in G, and every sphere and every shell is a
// union of the annuli (rho[a-1], rho[a]] between consecutive sorted distinct radii, so here N
// is evaluated once per giver annulus g (3 inverse + 9 forward transforms, the helper H
// inverse-transformed once) and contracted in FP64 against the receiver field into a
// histogram T[g][a] over receiver annuli.  Then
//   flux(s)       = sign * sum_{rho[g] <= R_s} sum_{rho[a-1] >= R_s} T[g][a]   (Prod_out_sphere_nlinV)
//   shell_tr(n,m) = sign * sum_{g in shell n} sum_{a: Get_shell_index = m, rho[a] <= R_in} T[g][a]
//                                                     (Shell_mult_all_FOUR four_ET.cc:181-256)
// Get_shell_index (basis_basicfn.cc:288-299) is constant on an annulus.  With monotonic radii
// (R_in > 16) the annuli are the S shells themselves.
#include <algorithm>
#include <cmath>
#include <vector>

#include "tg_ctx.h"

using namespace tg;

namespace tg {

// EnergyTr::EnergyTr shell radii, scheme 0 (EnergyTr.cc:136-160)
std::vector<double> et_radii(const tg_ctx* c) {
  const int S = c->cfg.n_shells;
  std::vector<double> R((size_t)S + 1, 0.0);
  const int d = c->cfg.dealias ? 3 : 2;
  const double* kf = c->cfg.kfactor;
  double km = std::min((c->N1 / d) * kf[0], (c->N2 / d) * kf[1]);
  if (c->N3 > 2) km = std::min(km, (c->N3 / d) * kf[2]);
  const double Rin = 1.0 * (int)km;
  if (S < 4) return R;
  R[0] = 0.0;
  R[1] = 2.0;
  R[2] = 4.0;
  R[3] = 8.0;
  R[S - 2] = Rin / 2;
  R[S - 1] = Rin;
  R[S] = 10000.0;  // INF_RADIUS (extern_def_vars.h:88)
  if (S > 6) {
    const double s = std::log2(Rin / 16.0) / (S - 5);
    for (int i = 4; i <= S - 3; ++i) R[i] = 8 * std::pow(2.0, s * (i - 3));
  }
  return R;
}

// the context's diagnostics scratch (c->diag) grown to at least `need` doubles
int ensure_diag(tg_ctx* c, size_t need) {
  if (c->diag_cap >= need) return TG_OK;
  if (c->diag) {
    cudaFree(c->diag);
    c->bytes -= sizeof(double) * c->diag_cap;
  }
  c->diag = nullptr;
  c->diag_cap = 0;
  int rc = dalloc_ctx(c, (void**)&c->diag, sizeof(double) * need);
  if (rc) return rc;
  c->diag_cap = need;
  return TG_OK;
}

// transfer scratch: etG (giver fields) and the helper / product pipeline buffers
int ensure_et_buffers(tg_ctx* c) {
  if (c->et_ready) return TG_OK;
  const Geo& g = c->g;
  const size_t Sd = sizeof(cx<double>) * (size_t)g.S;
  const size_t St = c->tsz * (size_t)g.S;
  const size_t WXb = c->tsz * (size_t)c->N1 * g.nky * g.kzp;
  const size_t WYb = c->tsz * (size_t)c->N1 * c->N2 * g.kzp;
  for (int i = 0; i < 3; ++i) {
    int rc = dalloc_ctx(c, (void**)&c->etG[i], Sd);
    if (rc) return rc;
  }
  for (int i = 0; i < 6; ++i) {
    if (i < c->nin) {
      c->etWY[i] = c->WY[i];
    } else {
      int rc = dalloc_ctx(c, &c->etWY[i], WYb);
      if (rc) return rc;
      c->et_own[c->n_et_own++] = c->etWY[i];
    }
  }
  for (int q = 0; q < 9; ++q) {
    if (q < c->nprod) {
      c->etPP[q] = c->PP[q];
      c->etPY[q] = c->PY[q];
      c->etPX[q] = c->PX[q];
    } else {
      int rc = dalloc_ctx(c, &c->etPP[q], WYb);
      if (!rc) rc = dalloc_ctx(c, &c->etPY[q], WXb);
      if (!rc) rc = dalloc_ctx(c, &c->etPX[q], St);
      if (rc) return rc;
      c->et_own[c->n_et_own++] = c->etPP[q];
      c->et_own[c->n_et_own++] = c->etPY[q];
      c->et_own[c->n_et_own++] = c->etPX[q];
    }
  }
  c->et_ready = true;
  return TG_OK;
}

}  // namespace tg

namespace {

constexpr int TPB = 256;
constexpr int kMaxShells = 63;

// sorted distinct radii rho[0] = 0 < rho[1] < ... < rho[A]; annulus a = (rho[a-1], rho[a]]
struct Radii {
  double r[kMaxShells + 1];
  int S;  // number of annuli A
};

// G = F on lo < |K| <= hi, else 0  (Fill_array_shell universal_ET.cc:45-65)
__global__ void k_fill_shell(Geo g, const cx<double>* F0, const cx<double>* F1, const cx<double>* F2,
                             cx<double>* G0, cx<double>* G1, cx<double>* G2, double lo, double hi) {
  const long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
  if (idx >= g.S) return;
  int r1, r2, l3;
  compact_mode(g, idx, r1, r2, l3);
  const double kx = geo_kx(g, r1) * g.kf0, ky = geo_ky(g, r2) * g.kf1, kz = l3 * g.kf2;
  const double K = sqrt(kx * kx + ky * ky + kz * kz);
  const bool in = (l3 < g.nkz) && (K > lo) && (K <= hi);
  const cx<double> z = mkc<double>(0, 0);
  G0[idx] = in ? F0[idx] : z;
  G1[idx] = in ? F1[idx] : z;
  G2[idx] = in ? F2[idx] : z;
}

struct ContractArgs {
  Geo g;
  const void* PX[9];      // P(i, j) = F(H_j G_i), q = 3 i + j
  const cx<double>* R[2][3];  // receiver fields
  int nrec;
  Radii rad;
  double* hist;           // [nrec][S+1]
  double* part;           // [blocks][nrec][S+1]: each block's sums, reduced in block order
  int cross;              // 1: N = F(H x G) (EnergyTr_Compute_nlin_UcrossB) instead of D_j F(H_j G_i)
};

// N_i = D_j P(i, j): FOUR i k_j P(i, j); SCFT (Xderiv_SCFT scft_tr.cc:649-707) the x derivative
// of the cosine series P(0, 0) is -kx P and of the sine series P(1, 0), P(2, 0) is +kx P, y and z
// as FOUR.  hist[r][shell(|K|)] += 2 mult Re(sum_i N_i conj(R_i)) (Multiplicity_factor_FOUR or
// _SCFT).
template <typename Rp>
__global__ void __launch_bounds__(TPB) k_et_contract(ContractArgs a) {
  constexpr int W = TPB / 32;
  constexpr int ROW = 2 * (kMaxShells + 1);
  __shared__ double sh[W][ROW];  // one row of bins per warp: no two warps add to one word
  const int nb = a.rad.S + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < W * ROW; i += TPB) sh[i / ROW][i % ROW] = 0;
  __syncthreads();
  const Geo& g = a.g;
  const long long stride = (long long)gridDim.x * TPB;
  // warp-uniform trip count: every lane of a warp takes part in the warp's bin sums
  for (long long w0 = (long long)blockIdx.x * TPB + warp * 32; w0 < g.S; w0 += stride) {
    const long long idx = w0 + lane;
    bool active = idx < g.S;
    int r1 = 0, r2 = 0, l3 = 0;
    if (active) {
      compact_mode(g, idx, r1, r2, l3);
      active = l3 < g.nkz;
    }
    int bin = 0;  // receiver annulus: first rho >= |K|
    double m = 0;
    cx<double> N[3] = {mkc<double>(0, 0), mkc<double>(0, 0), mkc<double>(0, 0)};
    if (active) {
      const int l1 = geo_l1(g, r1), l2 = amap_index(g.ay, r2);
      const double kx = geo_kx(g, r1) * g.kf0, ky = geo_ky(g, r2) * g.kf1, kz = l3 * g.kf2;
      const double K = sqrt(kx * kx + ky * ky + kz * kz);
      while (bin < a.rad.S && K > a.rad.r[bin]) ++bin;
      if (a.cross) {
        // (H x G)_i from P(i, j) = F(H_j G_i): x = P(2,1) - P(1,2), y = P(0,2) - P(2,0), z = P(1,0) - P(0,1)
        auto P = [&](int i, int j) { return cvt<double>(reinterpret_cast<const cx<Rp>*>(a.PX[3 * i + j])[idx]); };
        N[0] = P(2, 1) - P(1, 2);
        N[1] = P(0, 2) - P(2, 0);
        N[2] = P(1, 0) - P(0, 1);
      } else if (g.basis == 0) {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const cx<double> p0 = cvt<double>(reinterpret_cast<const cx<Rp>*>(a.PX[3 * i + 0])[idx]);
          const cx<double> p1 = cvt<double>(reinterpret_cast<const cx<Rp>*>(a.PX[3 * i + 1])[idx]);
          const cx<double> p2 = cvt<double>(reinterpret_cast<const cx<Rp>*>(a.PX[3 * i + 2])[idx]);
          const cx<double> s = mkc<double>(kx * p0.x + ky * p1.x + kz * p2.x, kx * p0.y + ky * p1.y + kz * p2.y);
          N[i] = ione(s);
        }
      } else {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const cx<double> p0 = cvt<double>(reinterpret_cast<const cx<Rp>*>(a.PX[3 * i + 0])[idx]);
          const cx<double> p1 = cvt<double>(reinterpret_cast<const cx<Rp>*>(a.PX[3 * i + 1])[idx]);
          const cx<double> p2 = cvt<double>(reinterpret_cast<const cx<Rp>*>(a.PX[3 * i + 2])[idx]);
          const double dx = (i == 0) ? -kx : kx;
          N[i] = mkc<double>(dx * p0.x - (ky * p1.y + kz * p2.y), dx * p0.y + (ky * p1.x + kz * p2.x));
        }
      }
      m = g.basis == 0 ? mult_four(l1, l2, l3, g.N1, g.N2) : mult_scft(l1, l2, l3, g.N2);
    }
    for (int r = 0; r < a.nrec; ++r) {
      double v = 0;
      if (active) {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const cx<double> b = a.R[r][i][idx];
          v += N[i].x * b.x + N[i].y * b.y;
        }
      }
      warp_bin_add(sh[warp] + r * nb, bin, 2.0 * m * v, active);
    }
  }
  __syncthreads();
  // the block's sums, warps in order
  for (int i = threadIdx.x; i < a.nrec * nb; i += TPB) {
    double t = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) t += sh[w][i];
    a.part[(size_t)blockIdx.x * a.nrec * nb + i] = t;
  }
}

// hist[i] = the blocks' sums of bin i in block order (one thread per bin)
__global__ void k_et_reduce(const double* __restrict__ part, int nblocks, int nbins, double* hist) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nbins) return;
  double t = 0;
  for (int b = 0; b < nblocks; ++b) t += part[(size_t)b * nbins + i];
  hist[i] = t;
}

struct KindSpec {
  int H, F;      // field groups: 0 = U (state 0..2), 1 = B (state 3..5)
  int R;         // receiver group
  double sign;
};

bool kind_spec(const tg_ctx* c, int kind, KindSpec& k) {
  switch (kind) {
    case TG_ET_UU: k = {0, 0, 0, -1.0}; return true;
    case TG_ET_BB: k = {0, 1, 1, -1.0}; break;   // W.flux_self: U.grad W< against W>
    case TG_ET_UB: k = {1, 0, 1, +1.0}; break;   // flux_VF_in_out: W.grad U< against W>
    case TG_ET_BU: k = {0, 1, 0, +1.0}; break;   // W.flux_VF_in_out: U.grad W< against U>
    default: return false;
  }
  return c->phys == TG_MHD;
}


// Sorted distinct radii of the transfer shells (the reference's radii need not be monotonic
// when R_in <= 16: EnergyTr.cc:118-126 only warns).
std::vector<double> et_annuli(const tg_ctx* c) {
  std::vector<double> R = et_radii(c);
  std::vector<double> rho(R.begin(), R.end());
  std::sort(rho.begin(), rho.end());
  rho.erase(std::unique(rho.begin(), rho.end()), rho.end());
  if (rho.empty() || rho[0] != 0.0) rho.insert(rho.begin(), 0.0);
  return rho;
}

// T[r][g][a]: giver annulus g = 1..A (field F inside (rho[g-1], rho[g]]), receiver annulus
// a = 0..A, receivers r of the given (H, F) pair
int et_tables_ptr(tg_ctx* c, const cx<double>* const* Hp, const cx<double>* const* Fp,
                  const cx<double>* const (*Rp)[3], int nrec, const std::vector<double>& rho,
                  std::vector<double>& T, int cross = 0);

// T[r][g][a] for helper fields Hp, giver fields Fp and receivers Rp (any compact FP64 fields)
int et_tables_ptr(tg_ctx* c, const cx<double>* const* Hp, const cx<double>* const* Fp,
                  const cx<double>* const (*Rp)[3], int nrec, const std::vector<double>& rho,
                  std::vector<double>& T, int cross) {
  const int A = (int)rho.size() - 1;
  if (A < 1 || A > kMaxShells) return set_err(c, TG_ERR_ARG, "energy transfer needs 6 <= n_shells <= 63");
  int rc = ensure_et_buffers(c);
  if (rc) return rc;
  const Geo& g = c->g;
  Radii rad{};
  rad.S = A;
  for (int i = 0; i <= A; ++i) rad.r[i] = rho[i];
  const int nb = A + 1;
  const size_t need = (size_t)nrec * (A + 1) * nb;
  const int nblk = (int)std::min<long long>((g.S + TPB - 1) / TPB, 148LL * 8);
  // the tables, then the per-block sums of one contraction (reduced in block order)
  rc = ensure_diag(c, need + (size_t)nblk * nrec * nb);
  if (rc) return rc;
  cudaError_t e = cudaMemsetAsync(c->diag, 0, sizeof(double) * need, c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "memset");
  // helper H: inverse x, y once (into etWY[0..2])
  const void* H[3] = {Hp[0], Hp[1], Hp[2]};
  rc = pipe_inverse_xy(c, 3, H, nullptr, nullptr, F64, 3, c->WX, c->etWY);
  if (rc) return rc;
  ProdPairs pp{};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      pp.a[3 * i + j] = (signed char)(3 + i);  // G_i
      pp.b[3 * i + j] = (signed char)j;        // H_j
    }
  for (int n = 1; n <= A; ++n) {
    k_fill_shell<<<(int)((g.S + TPB - 1) / TPB), TPB, 0, c->st>>>(
        g, Fp[0], Fp[1], Fp[2], c->etG[0], c->etG[1], c->etG[2], rho[n - 1], rho[n]);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_err(c, e, "fill shell");
    const void* G[3] = {c->etG[0], c->etG[1], c->etG[2]};
    rc = pipe_inverse_xy(c, 3, G, nullptr, nullptr, F64, 3, c->WX, c->etWY + 3);
    if (rc) return rc;
    rc = pipe_products_forward(c, 6, c->etWY, 9, pp, c->etPP, c->etPY, c->etPX, kEtXKinds);
    if (rc) return rc;
    ContractArgs a{};
    a.g = g;
    for (int q = 0; q < 9; ++q) a.PX[q] = c->etPX[q];
    for (int r = 0; r < nrec; ++r)
      for (int i = 0; i < 3; ++i) a.R[r][i] = Rp[r][i];
    a.nrec = nrec;
    a.rad = rad;
    a.cross = cross;
    a.hist = c->diag + (size_t)n * nrec * nb;  // layout [g][r][a]
    a.part = c->diag + need;
    {
      ProfScope pr(c, "et_contract", 0.0);
      if (c->tprec == F64) k_et_contract<double><<<nblk, TPB, 0, c->st>>>(a);
      else k_et_contract<float><<<nblk, TPB, 0, c->st>>>(a);
      k_et_reduce<<<(nrec * nb + 127) / 128, 128, 0, c->st>>>(a.part, nblk, nrec * nb, a.hist);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_err(c, e, "et contract");
  }
  std::vector<double> h(need);
  e = cudaMemcpyAsync(h.data(), c->diag, sizeof(double) * need, cudaMemcpyDeviceToHost, c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "et tables");
  TG_SYNC(c, "et tables");
  T.assign((size_t)nrec * (A + 1) * nb, 0.0);
  for (int n = 1; n <= A; ++n)
    for (int r = 0; r < nrec; ++r)
      for (int m = 0; m < nb; ++m) T[((size_t)r * (A + 1) + n) * nb + m] = h[((size_t)n * nrec + r) * nb + m];
  return TG_OK;
}

struct PtrPair6 {
  const cx<double>* in[6];
  cx<double>* out[6];
};

// Z+ = U + B, Z- = U - B (UB_to_Elsasser_field elsasser.cc:53-90)
__global__ void k_elsasser(Geo g, PtrPair6 p) {
  const long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
  if (idx >= g.S) return;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const cx<double> u = p.in[i][idx], b = p.in[3 + i][idx];
    p.out[i][idx] = u + b;
    p.out[3 + i][idx] = u - b;
  }
}

int own_field(tg_ctx* c, cx<double>** f) {
  if (*f) return TG_OK;
  if (c->n_et_own >= 32) return set_err(c, TG_ERR_STATE, "energy transfer: too many scratch fields");
  int rc = dalloc_ctx(c, (void**)f, sizeof(cx<double>) * (size_t)c->g.S);
  if (rc) return rc;
  c->et_own[c->n_et_own++] = *f;
  return TG_OK;
}

}  // namespace

namespace tg {

// The helper H, giver F and receiver R of an energy-transfer kind, and its sign.
//   U->U, B->B, U->B, B->U: the state fields (kind_spec).
//   T->T (Compute_flux_scalar / Compute_shell_tr_scalar compute_flux.cc:82-95,
//   compute_shell_tr.cc:93-109; Compute_ring_tr_scalar compute_ring_tr.cc:104-131): G = T<,
//   N = D_j F(U_j T<) against T, sign -1, run as the vector form with giver and receiver (T, 0, 0).
//   Z+->Z+, Z-->Z- (flux_Elsasser / shelltoshell_Elsasser compute_flux.cc:228-255,
//   compute_shell_tr.cc:201-246, ring_to_ring_Elsasser compute_ring_tr.cc:240-285): Z+ = U + B,
//   Z- = U - B written to scratch fields, G = Z+<, N = D_j F(Z-_j G_i) against Z+ (and with + and -
//   exchanged), sign -1.
int et_kind_fields(tg_ctx* c, int kind, const cx<double>* H[3], const cx<double>* F[3], const cx<double>* R[3],
                   double& sign) {
  if (kind == TG_ET_TT) {
    if (c->phys != TG_SCALAR && c->phys != TG_RB) return set_err(c, TG_ERR_ARG, "scalar transfer needs a scalar");
    const int rc = own_field(c, &c->etZero);
    if (rc) return rc;
    sign = -1.0;
    for (int i = 0; i < 3; ++i) H[i] = c->U0[i];
    F[0] = R[0] = c->U0[3];
    F[1] = F[2] = R[1] = R[2] = c->etZero;
    return TG_OK;
  }
  if (kind == TG_ET_ZP || kind == TG_ET_ZM) {
    if (c->phys != TG_MHD) return set_err(c, TG_ERR_ARG, "Elsasser transfers need MHD");
    int rc = TG_OK;
    for (int i = 0; i < 6 && !rc; ++i) rc = own_field(c, &c->etZ[i]);
    if (rc) return rc;
    PtrPair6 p{};
    for (int i = 0; i < 6; ++i) {
      p.in[i] = c->U0[i];
      p.out[i] = c->etZ[i];
    }
    k_elsasser<<<(int)((c->g.S + TPB - 1) / TPB), TPB, 0, c->st>>>(c->g, p);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_err(c, e, "elsasser");
    sign = -1.0;
    const int a = (kind == TG_ET_ZP) ? 0 : 3, b = 3 - a;
    for (int i = 0; i < 3; ++i) {
      H[i] = c->etZ[b + i];
      F[i] = R[i] = c->etZ[a + i];
    }
    return TG_OK;
  }
  KindSpec k{};
  if (!kind_spec(c, kind, k)) return set_err(c, TG_ERR_ARG, "energy-transfer kind not available for this physics");
  sign = k.sign;
  for (int i = 0; i < 3; ++i) {
    H[i] = c->U0[3 * k.H + i];
    F[i] = c->U0[3 * k.F + i];
    R[i] = c->U0[3 * k.R + i];
  }
  return TG_OK;
}

}  // namespace tg

namespace {

int et_table_kind(tg_ctx* c, int kind, std::vector<double>& T, std::vector<double>& rho, double& sign) {
  int rc = ensure_et_buffers(c);
  if (rc) return rc;
  const cx<double>* H[3];
  const cx<double>* F[3];
  const cx<double>* R[1][3];
  rc = et_kind_fields(c, kind, H, F, R[0], sign);
  if (rc) return rc;
  rho = et_annuli(c);
  return et_tables_ptr(c, H, F, R, 1, rho, T);
}


// omega = i K x V (Compute_Modal_vorticity_FOUR four_basic.cc:166-186), compact layout
__global__ void k_vorticity(Geo g, const cx<double>* V0, const cx<double>* V1, const cx<double>* V2, cx<double>* W0,
                            cx<double>* W1, cx<double>* W2) {
  const long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
  if (idx >= g.S) return;
  int r1, r2, l3;
  compact_mode(g, idx, r1, r2, l3);
  const double kx = geo_kx(g, r1) * g.kf0, ky = geo_ky(g, r2) * g.kf1, kz = l3 * g.kf2;
  const cx<double> a = V0[idx], b = V1[idx], d = V2[idx];
  W0[idx] = ione(ky * d - kz * b);
  W1[idx] = ione(kz * a - kx * d);
  W2[idx] = ione(kx * b - ky * a);
}

// a = i K x B / K^2 (zero at K = 0): the potential Shell_mult_vector_potential pairs with
// (four_ET.cc:905-965)
__global__ void k_vector_potential(Geo g, const cx<double>* B0, const cx<double>* B1, const cx<double>* B2,
                                   cx<double>* A0, cx<double>* A1, cx<double>* A2) {
  const long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
  if (idx >= g.S) return;
  int r1, r2, l3;
  compact_mode(g, idx, r1, r2, l3);
  const double kx = geo_kx(g, r1) * g.kf0, ky = geo_ky(g, r2) * g.kf1, kz = l3 * g.kf2;
  const double K2 = kx * kx + ky * ky + kz * kz;
  const double w = K2 > 0 ? 1.0 / K2 : 0.0;
  const cx<double> a = B0[idx], b = B1[idx], d = B2[idx];
  A0[idx] = w * ione(ky * d - kz * b);
  A1[idx] = w * ione(kz * a - kx * d);
  A2[idx] = w * ione(kx * b - ky * a);
}

// Force feed per shell (Compute_force_feed_shell compute_force_feed.cc:70-76 with
// Shell_mult_all_FOUR four_ET.cc:181-226): for |K| <= R_in, result[i] += 2 mult Re(F . V*),
// i = Get_shell_index(|K|).  The force is nonzero on its box only; thread i sums shell i over
// the box in a fixed order.
struct ShellRadii {
  double r[kMaxShells + 1];
};
// components c0 .. c0+nc-1 of the force box against the fields u0 .. (nc of them)
__global__ void k_force_feed(Geo g, const cx<double>* __restrict__ FB, int fx, int fy, int fz, int c0, int nc,
                             const cx<double>* __restrict__ u0, const cx<double>* __restrict__ u1,
                             const cx<double>* __restrict__ u2, ShellRadii R, int S, double kin, double* out) {
  const int i = threadIdx.x;
  if (i > S) return;
  const int ny = 2 * fy + 1, nz = fz + 1, box = (2 * fx + 1) * ny * nz;
  const cx<double>* U[3] = {u0, u1, u2};
  double acc = 0;
  for (int p = 0; p < box; ++p) {
    const int kz = p % nz, ky = (p / nz) % ny - fy, kx = p / (nz * ny) - fx;
    if (g.basis == 1 && kx < 0) continue;  // SCFT: kx >= 0
    const int l1 = kx >= 0 ? kx : kx + g.N1, l2 = ky >= 0 ? ky : ky + g.N2;
    if (l1 < 0 || l1 >= g.N1 || l2 < 0 || l2 >= g.N2 || kz >= g.nkz) continue;
    const int r1 = amap_row(g.ax, l1), r2 = amap_row(g.ay, l2);
    if (r1 < 0 || r2 < 0) continue;
    const double a = kx * g.kf0, b = ky * g.kf1, c = kz * g.kf2;
    const double K = sqrt(a * a + b * b + c * c);
    if (K > kin) continue;
    int sh = 0;
    while (sh <= S && !(K <= R.r[sh])) ++sh;
    if (sh != i) continue;
    const long long idx = ((long long)r1 * g.nky + r2) * g.kzp + kz;
    double re = 0;
    for (int cc = 0; cc < nc; ++cc) {
      const cx<double> f = FB[(long long)(c0 + cc) * box + p], v = U[cc][idx];
      re += f.x * v.x + f.y * v.y;
    }
    acc += 2 * (g.basis == 1 ? mult_scft(l1, l2, kz, g.N2) : mult_four(l1, l2, kz, g.N1, g.N2)) * re;
  }
  out[i] = acc;
}

// the liquid-metal force -(B0 . K)^2/K^2 V against V: -2 mult (B0 . K)^2/K^2 |V|^2, binned by
// Get_shell_index over |K| <= R_in (out zeroed by the caller, S + 1 bins)
__global__ void __launch_bounds__(256) k_force_feed_lm(Geo g, const cx<double>* u0, const cx<double>* u1,
                                                       const cx<double>* u2, double b0, double b1, double b2,
                                                       ShellRadii R, int S, double kin, double* out) {
  __shared__ double sh[kMaxShells + 1];
  for (int i = threadIdx.x; i <= S; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < g.S; idx += stride) {
    int r1, r2, l3;
    compact_mode(g, idx, r1, r2, l3);
    if (l3 >= g.nkz) continue;
    const double kx = geo_kx(g, r1) * g.kf0, ky = geo_ky(g, r2) * g.kf1, kz = l3 * g.kf2;
    const double K2 = kx * kx + ky * ky + kz * kz, K = sqrt(K2);
    if (K > kin || K2 <= 0) continue;
    int sh_i = 0;
    while (sh_i <= S && !(K <= R.r[sh_i])) ++sh_i;
    if (sh_i > S) continue;
    const double bk = b0 * kx + b1 * ky + b2 * kz;
    const cx<double> a = u0[idx], b = u1[idx], d = u2[idx];
    const double v2 = a.x * a.x + a.y * a.y + b.x * b.x + b.y * b.y + d.x * d.x + d.y * d.y;
    const int l1 = geo_l1(g, r1), l2 = amap_index(g.ay, r2);
    atomicAdd(&sh[sh_i], -2 * mult_four(l1, l2, l3, g.N1, g.N2) * (bk * bk / K2) * v2);
  }
  __syncthreads();
  for (int i = threadIdx.x; i <= S; i += blockDim.x)
    if (sh[i] != 0) atomicAdd(&out[i], sh[i]);
}
// Rows n = 1 .. S-1 of a shell-to-shell table (compute_shell_tr.cc: shell_from_index <
// no_shells) from a giver-annulus x receiver-annulus table T; receivers |K| <= R_in go to column
// Get_shell_index (first i with R[i] >= |K|), which is constant on an annulus.  tr is n x n.
void shell_rows(const std::vector<double>& R, const std::vector<double>& rho, const std::vector<double>& T,
                double sign, int S, double* tr, int n) {
  const int A = (int)rho.size() - 1, nb = A + 1;
  const double Rin = R[S - 1];
  std::vector<int> bin(nb, S);
  for (int a = 0; a <= A; ++a) {
    int i = 0;
    while (i <= S && !(rho[a] <= R[i])) ++i;
    bin[a] = i;
  }
  for (int i = 0; i < n * n; ++i) tr[i] = 0;
  for (int sh = 1; sh < S; ++sh) {
    const double lo = R[sh - 1], hi = R[sh];
    for (int g = 1; g <= A; ++g) {
      if (!(rho[g - 1] >= lo && rho[g] <= hi)) continue;
      for (int a = 0; a <= A; ++a) {
        if (rho[a] > Rin || bin[a] >= n) continue;
        tr[(size_t)sh * n + bin[a]] += sign * T[(size_t)g * nb + a];
      }
    }
  }
}

// Giver-annulus x receiver-annulus table of a helicity transfer, the three terms combined.
// Kinetic (IncVF::Compute_kinetic_helicity_flux compute_helicity_flux.cc:52-86 and
// Compute_kinetic_helicity_shell_tr compute_helicity_shell_tr.cc:56-109):
//   -(U.grad U<).omega/2 - (U.grad omega<).U/2 + (omega.grad U<).U/2, omega = i K x U.
// Magnetic (Compute_magnetic_helicity_flux compute_helicity_flux.cc:94-135 and
// Compute_magnetic_helicity_shell_tr compute_helicity_shell_tr.cc:114-172):
//   (B.grad U<).a/2 - (U.grad B<).a/2 + (U x B<).B/2, a = i K x B / K^2
// (Shell_mult_vector_potential_FOUR four_ET.cc:905-965; U x B< of EnergyTr_Compute_nlin_UcrossB
// ET_compute_nlin.cc:317-337).  At K = 0 the reference divides 0 by |K|^2 = 0 in the shell
// table; a is taken as 0 there.
int helicity_table(tg_ctx* c, int magnetic, const std::vector<double>& rho, std::vector<double>& Tc) {
  if (c->basis != TG_FOUR) return set_err(c, TG_ERR_UNSUPPORTED, "helicity transfer is built for the FOUR basis");
  if (magnetic && c->phys != TG_MHD) return set_err(c, TG_ERR_ARG, "magnetic helicity transfer needs MHD");
  int rc = ensure_et_buffers(c);
  for (int i = 0; i < 3 && !rc; ++i) rc = own_field(c, &c->etVort[i]);
  if (rc) return rc;
  const Geo& g = c->g;
  const int grid = (int)((g.S + TPB - 1) / TPB);
  const cx<double>* U[3] = {c->U0[0], c->U0[1], c->U0[2]};
  const cx<double>* W[3] = {c->etVort[0], c->etVort[1], c->etVort[2]};
  std::vector<double> T1, T2, T3;
  if (!magnetic) {
    k_vorticity<<<grid, TPB, 0, c->st>>>(g, U[0], U[1], U[2], c->etVort[0], c->etVort[1], c->etVort[2]);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_err(c, e, "vorticity");
    const cx<double>* RW[1][3] = {{W[0], W[1], W[2]}};
    const cx<double>* RU[1][3] = {{U[0], U[1], U[2]}};
    rc = et_tables_ptr(c, U, U, RW, 1, rho, T1);              // U.grad U<  against omega
    if (!rc) rc = et_tables_ptr(c, U, W, RU, 1, rho, T2);     // U.grad omega< against U
    if (!rc) rc = et_tables_ptr(c, W, U, RU, 1, rho, T3);     // omega.grad U< against U
  } else {
    const cx<double>* B[3] = {c->U0[3], c->U0[4], c->U0[5]};
    k_vector_potential<<<grid, TPB, 0, c->st>>>(g, B[0], B[1], B[2], c->etVort[0], c->etVort[1], c->etVort[2]);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_err(c, e, "vector potential");
    const cx<double>* RA[1][3] = {{W[0], W[1], W[2]}};
    const cx<double>* RB[1][3] = {{B[0], B[1], B[2]}};
    rc = et_tables_ptr(c, B, U, RA, 1, rho, T1);              // B.grad U< against a
    if (!rc) rc = et_tables_ptr(c, U, B, RA, 1, rho, T2);     // U.grad B< against a
    if (!rc) rc = et_tables_ptr(c, U, B, RB, 1, rho, T3, 1);  // U x B< against B
  }
  if (rc) return rc;
  const double s1 = magnetic ? 0.5 : -0.5;
  Tc.assign(T1.size(), 0.0);
  for (size_t q = 0; q < Tc.size(); ++q) Tc[q] = s1 * T1[q] - 0.5 * T2[q] + 0.5 * T3[q];
  return TG_OK;
}

// Sphere fluxes (giver annuli inside R_s, receivers outside; Prod_out_sphere_* prod_nlinV.cc:62-162;
// out has n >= S+1 entries) or the n x n shell-to-shell table (giver rows 1 .. S-1, receivers binned by Get_shell_index over
// |K| <= R_in; Shell_mult_*_all four_ET.cc:181-256, 999-1090, 1094-1190) of a helicity table.
int helicity_out(tg_ctx* c, int magnetic, int shells, double* out, int n) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c || !out) return TG_ERR_ARG;
  const int S = c->cfg.n_shells;
  if (S < 6 || n < S + 1) return TG_ERR_ARG;
  cudaSetDevice(c->dev);
  const std::vector<double> rho = et_annuli(c);
  std::vector<double> T;
  const int rc = helicity_table(c, magnetic, rho, T);
  if (rc) return rc;
  const std::vector<double> R = et_radii(c);
  if (shells) {
    shell_rows(R, rho, T, 1.0, S, out, n);
    return TG_OK;
  }
  const int A = (int)rho.size() - 1, nb = A + 1;
  for (int s = 0; s < n; ++s) out[s] = 0;
  for (int s = 1; s <= S; ++s) {
    double acc = 0;
    for (int gg = 1; gg <= A; ++gg) {
      if (rho[gg] > R[s]) continue;
      for (int a = 1; a <= A; ++a)
        if (rho[a - 1] >= R[s]) acc += T[(size_t)gg * nb + a];
    }
    out[s] = acc;
  }
  return TG_OK;
}

}  // namespace

extern "C" {

int tg_et_radii(tg_ctx* c, double* radii, int n) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c || !radii) return TG_ERR_ARG;
  const int S = c->cfg.n_shells;
  if (S < 6) return set_err(c, TG_ERR_ARG, "energy transfer needs at least 6 shells");
  if (n < S + 1) return TG_ERR_ARG;
  std::vector<double> R = et_radii(c);
  for (int i = 0; i <= S; ++i) radii[i] = R[i];
  return TG_OK;
}

int tg_flux(tg_ctx* c, int kind, double* flux, int n) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c || !flux) return TG_ERR_ARG;
  const int S = c->cfg.n_shells;
  if (S < 6 || n < S + 1) return TG_ERR_ARG;
  cudaSetDevice(c->dev);
  std::vector<double> T, rho;
  double sign = 1;
  int rc = et_table_kind(c, kind, T, rho, sign);
  if (rc) return rc;
  const std::vector<double> R = et_radii(c);
  const int A = (int)rho.size() - 1, nb = A + 1;
  for (int s = 0; s < n; ++s) flux[s] = 0;
  // flux(s): givers inside 0 < |K| <= R_s, receivers |K| > R_s (Prod_out_sphere_nlinV)
  for (int s = 1; s <= S; ++s) {
    double acc = 0;
    for (int g = 1; g <= A; ++g) {
      if (rho[g] > R[s]) continue;
      for (int a = 1; a <= A; ++a)
        if (rho[a - 1] >= R[s]) acc += T[(size_t)g * nb + a];
    }
    flux[s] = sign * acc;
  }
  return TG_OK;
}

// Kinetic helicity flux (IncVF::Compute_kinetic_helicity_flux compute_helicity_flux.cc:47-75):
// flux(s) = -P(U.grad U<, omega>)/2 - P(U.grad omega<, U>)/2 + P(omega.grad U<, U>)/2, with
// P(N, R>) = sum over |K| > R_s of 2 mult Re(N . R*) (Prod_out_sphere_nlinV,
// Prod_out_sphere_nlin_vorticity prod_nlinV.cc:62-150) and X< = X on 0 < |K| <= R_s
// (Fill_in_sphere, Fill_in_sphere_vorticity fill_sphere_shell.cc:57-210).
int tg_helicity_flux(tg_ctx* c, double* flux, int n) { return helicity_out(c, 0, 0, flux, n); }

int tg_magnetic_helicity_flux(tg_ctx* c, double* flux, int n) { return helicity_out(c, 1, 0, flux, n); }

int tg_helicity_shell_to_shell(tg_ctx* c, double* tr, int n) { return helicity_out(c, 0, 1, tr, n); }

int tg_magnetic_helicity_shell_to_shell(tg_ctx* c, double* tr, int n) { return helicity_out(c, 1, 1, tr, n); }

int tg_shell_to_shell(tg_ctx* c, int kind, double* tr, int n) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c || !tr) return TG_ERR_ARG;
  const int S = c->cfg.n_shells;
  if (S < 6 || n < S + 1) return TG_ERR_ARG;
  cudaSetDevice(c->dev);
  std::vector<double> T, rho;
  double sign = 1;
  int rc = et_table_kind(c, kind, T, rho, sign);
  if (rc) return rc;
  shell_rows(et_radii(c), rho, T, sign, S, tr, n);
  return TG_OK;
}


// convection (Compute_force_feed_shell_RB -> Compute_force_feed_shell_scalar, PRLARGE and
// PRSMALL): with Force1 = fu theta and T.Force = ft u1 (Compute_force_RB), group 0 bins
// 2 mult fu Re(theta u1*) and group 2 bins 2 mult ft Re(u1 theta*) by Get_shell_index over
// |K| <= R_in, SCFT or FOUR multiplicity (out zeroed by the caller)
__global__ void __launch_bounds__(256) k_force_feed_rb(Geo g, const cx<double>* u1, const cx<double>* th, double coef,
                                                       ShellRadii R, int S, double kin, double* out) {
  __shared__ double sh[kMaxShells + 1];
  for (int i = threadIdx.x; i <= S; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < g.S; idx += stride) {
    int r1, r2, l3;
    compact_mode(g, idx, r1, r2, l3);
    if (l3 >= g.nkz) continue;
    const double kx = geo_kx(g, r1) * g.kf0, ky = geo_ky(g, r2) * g.kf1, kz = l3 * g.kf2;
    const double K = sqrt(kx * kx + ky * ky + kz * kz);
    if (K > kin) continue;
    int sh_i = 0;
    while (sh_i <= S && !(K <= R.r[sh_i])) ++sh_i;
    if (sh_i > S) continue;
    const int l1 = geo_l1(g, r1), l2 = amap_index(g.ay, r2);
    const double m = g.basis == 0 ? mult_four(l1, l2, l3, g.N1, g.N2) : mult_scft(l1, l2, l3, g.N2);
    const cx<double> a = u1[idx], b = th[idx];
    atomicAdd(&sh[sh_i], 2 * m * coef * (a.x * b.x + a.y * b.y));
  }
  __syncthreads();
  for (int i = threadIdx.x; i <= S; i += blockDim.x)
    if (sh[i] != 0) atomicAdd(&out[i], sh[i]);
}

// group 0: Compute_force_feed_shell (forceV_shell, Re(F . V*)); 1: W.forceV_shell of
// Compute_force_feed_shell(W) (Re(F_B . B*), MHD); 2: forceSF_shell of
// Compute_force_feed_shell_scalar (Re(F_T . T*), passive scalar) (compute_force_feed.cc:70-155)
int tg_force_feed_group(tg_ctx* c, int group, double* feed, int n) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c || !feed) return TG_ERR_ARG;
  const int S = c->cfg.n_shells;
  if (S < 6 || S > kMaxShells || n < S + 1 || group < 0 || group > 2) return TG_ERR_ARG;
  if (c->basis != TG_FOUR && c->phys != TG_RB && !(c->force_on == 1 && c->phys != TG_MHD))
    return set_err(c, TG_ERR_UNSUPPORTED, "force feed: FOUR, convection, or an SCFT band forcing");
  if ((group == 1 && c->phys != TG_MHD) || (group == 2 && c->phys != TG_SCALAR && c->phys != TG_RB))
    return set_err(c, TG_ERR_ARG, "force feed: the group is not a field of this physics");
  for (int i = 0; i < n; ++i) feed[i] = 0;
  cudaSetDevice(c->dev);
  const std::vector<double> R = et_radii(c);
  ShellRadii rr{};
  for (int i = 0; i <= S; ++i) rr.r[i] = R[i];
  int rc = ensure_diag(c, (size_t)S + 1);
  if (rc) return rc;
  double* d = c->diag;
  cudaError_t e = cudaSuccess;
  if (c->phys == TG_RB) {
    e = cudaMemsetAsync(d, 0, sizeof(double) * (S + 1), c->st);
    if (e == cudaSuccess) {
      const int nb = (int)std::min<long long>((c->g.S + 255) / 256, 148LL * 4);
      k_force_feed_rb<<<nb, 256, 0, c->st>>>(c->g, c->U0[0], c->U0[3], group == 0 ? c->rb_fu : c->rb_ft, rr, S,
                                             R[S - 1], d);
      e = cudaGetLastError();
    }
  } else if (c->lm && group == 0) {
    e = cudaMemsetAsync(d, 0, sizeof(double) * (S + 1), c->st);
    if (e == cudaSuccess) {
      const int nb = (int)std::min<long long>((c->g.S + 255) / 256, 148LL * 4);
      k_force_feed_lm<<<nb, 256, 0, c->st>>>(c->g, c->U0[0], c->U0[1], c->U0[2], c->b0[0], c->b0[1], c->b0[2], rr, S,
                                             R[S - 1], d);
      e = cudaGetLastError();
    }
  } else {
    // decaying run, fixed modes never set: the force is zero; Coriolis: Re(F . V*) = Re(Omega .
    // (V* x V)) = 0 mode by mode (V* x V is imaginary)
    if (!c->force_on || (c->force_on == 2 && !c->FB)) return TG_OK;
    rc = ensure_force_box(c);
    if (rc) return rc;
    const int c0 = 3 * (group == 0 ? 0 : 1), nc = group == 2 ? 1 : 3;
    k_force_feed<<<1, 64, 0, c->st>>>(c->g, c->FB, c->fx, c->fy, c->fz, c0, nc, c->U0[c0], c->U0[c0 + (nc > 1)],
                                      c->U0[c0 + 2 * (nc > 1)], rr, S, R[S - 1], d);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(feed, d, sizeof(double) * (S + 1), cudaMemcpyDeviceToHost, c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "force feed");
  TG_SYNC(c, "force feed");
  return TG_OK;
}

int tg_force_feed(tg_ctx* c, double* feed, int n) { return tg_force_feed_group(c, 0, feed, n); }

}  // extern "C"
