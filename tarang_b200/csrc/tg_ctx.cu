// Solver context: geometry, device buffers, the nonlinear-term pipeline, the fused RK4 step
// and the C ABI entry points of include/tarang_gpu.h (except energy transfer and serving).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "tg_ctx.h"

using namespace tg;

namespace tg {

int set_err(tg_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

int cuda_err(tg_ctx* c, cudaError_t e, const char* where) {
  if (e == cudaSuccess) return TG_OK;
  std::string m = std::string(where) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return set_err(c, TG_ERR_OOM, m);
  return set_err(c, TG_ERR_CUDA, m);
}

int dalloc_ctx(tg_ctx* c, void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return set_err(c, TG_ERR_OOM, "device allocation of " + std::to_string(bytes) + " bytes failed");
  }
  c->bytes += bytes;
  e = cudaMemsetAsync(*p, 0, bytes, c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "cudaMemsetAsync");
  return TG_OK;
}

void wait_args(const tg_ctx* c, AxisArgs& a) {
  a.wait_flag = c->wait_status;
  a.wait_short = c->wait_short;
}

int ctx_sync(tg_ctx* c, const char* where) {
  cudaError_t e = cudaSuccess;
  if (c->wait_status && c->h_wait) {
    *c->h_wait = 0;
    e = cudaMemcpyAsync(c->h_wait, c->wait_status, sizeof(int), cudaMemcpyDeviceToHost, c->st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
  if (e != cudaSuccess) return cuda_err(c, e, where);
  if (c->h_wait && *c->h_wait) {
    *c->h_wait = 0;
    e = cudaMemsetAsync(c->wait_status, 0, sizeof(int), c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    if (e != cudaSuccess) return cuda_err(c, e, where);
    return set_err(c, TG_ERR_TIMEOUT,
                   std::string(where) + ": a transform pass gave up waiting for its tile; the fields it wrote are not valid");
  }
  return TG_OK;
}

}  // namespace tg

namespace {

// Device table exp(-2 pi i m / L), m in [0, L), evaluated in long double and rounded.
int make_twiddles(tg_ctx* c, int L) {
  if (L <= 0 || c->tw.count(L)) return TG_OK;
  std::vector<cx<double>> h(L);
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int m = 0; m < L; ++m) {
    const long double ang = two_pi * (long double)m / (long double)L;
    h[m].x = (double)cosl(ang);
    h[m].y = (double)(-sinl(ang));
  }
  cx<double>* d = nullptr;
  TG_CK(cudaMalloc(&d, sizeof(cx<double>) * L));
  c->bytes += sizeof(cx<double>) * L;
  TG_CK(cudaMemcpy(d, h.data(), sizeof(cx<double>) * L, cudaMemcpyHostToDevice));
  c->tw[L] = d;
  return TG_OK;
}

int dalloc(tg_ctx* c, void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_err(c, TG_ERR_OOM, "device allocation of " + std::to_string(bytes) + " bytes failed");
  }
  c->bytes += bytes;
  e = cudaMemsetAsync(*p, 0, bytes, c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "cudaMemsetAsync");
  return TG_OK;
}

// Stored wavenumbers of one axis under the 2/3 rule (Dealias_array universal_misc.cc:118-159)
void keep_axis(int N, int axis, int basis, int dealias, int& lo, int& hi) {
  lo = N;
  hi = 0;
  if (!dealias || N < 3) return;
  if (axis == 0) {
    if (basis == TG_FOUR) {
      lo = N / 3;          // kx = 0 .. N/3-1
      hi = N / 3 - 1;      // kx = -(N/3-1) .. -1
    } else {
      lo = 2 * N / 3;      // m = 0 .. 2N/3-1
      hi = 0;
    }
  } else {
    lo = N / 3;                      // l2 = 0 .. N/3-1
    hi = N - (2 * N / 3 + 2);        // l2 = 2N/3+2 .. N-1
    if (hi < 0) hi = 0;
  }
  if (hi < 0) hi = 0;
}

AxisMap full_map(int L) { return AxisMap{L, L, 0}; }

int max_radius_inside(const tg_ctx* c) {
  // Max_radius_inside_(de)aliased_FOUR four_inline.h:190-257
  const int d = c->cfg.dealias ? 3 : 2;
  const double* kf = c->cfg.kfactor;
  double km;
  if (c->basis == TG_FOUR) {
    km = std::min((c->N1 / d) * kf[0], (c->N2 / d) * kf[1]);
    if (c->N3 > 2) km = std::min(km, (c->N3 / d) * kf[2]);
  } else {
    // Max_radius_inside_(de)aliased_SCFT scft_inline.h:160-220: 2 N1/3 dealiased, N1 - 1 aliased
    const int nx = c->cfg.dealias ? (2 * c->N1 / 3) : c->N1 - 1;
    km = std::min(nx * kf[0], (c->N2 / d) * kf[1]);
    if (c->N3 > 2) km = std::min(km, (c->N3 / d) * kf[2]);
  }
  return (int)km;
}

// ------------------------------------------------------------------ pipeline
// X-inverse, Y-inverse, fused z-pass (c2r, products, r2c), Y-forward, X-forward.
// inputs: compact fields of precision inprec.  MHD: in[0..2] = U, in[3..5] = B, the x-pass
// forms z+ = U + B (fields 0..2) and z- = U - B (fields 3..5).
int run_pipeline(tg_ctx* c, const void* const* in, int inprec) {
  const void* src[6];
  const void* src2[6] = {};
  int comb[6] = {0, 0, 0, 0, 0, 0};
  for (int f = 0; f < c->nin; ++f) {
    if (c->phys == TG_MHD) {
      src[f] = in[f % 3];
      src2[f] = in[3 + f % 3];
      comb[f] = f < 3 ? +1 : -1;
    } else {
      src[f] = in[f];
    }
  }
  int rc = pipe_inverse_xy(c, c->nin, src, src2, comb, inprec, c->nstate, c->WX, c->WY);
  if (rc) return rc;
  return pipe_products_forward(c, c->nin, c->WY, c->nprod, c->pairs, c->PP, c->PY, c->PX);
}

// U: the c->nstate fields the force is computed from (the stage input)
int run_force(tg_ctx* c, const void* const* U, int uprec) {
  if (c->force_on != 1) return TG_OK;
  ForceArgs f{};
  f.g = c->g;
  f.ns = c->nstate;
  for (int i = 0; i < c->nstate; ++i) f.U[i] = U[i];
  f.uprec = uprec;
  f.mode = c->cfg.force_kind == TG_FORCE_ENERGY_HELICITY ? 2 : 1;
  // the fluid-only supply does not test the energy per mode (compute_force_ek_hk_supply.cc:120)
  f.gate = (f.mode == 2 || c->phys != TG_FLUID) ? 1 : 0;
  f.fx = c->fx;
  f.fy = c->fy;
  f.fz = c->fz;
  const double* fp = c->cfg.force_para;
  const double nf = c->nf_modes > 0 ? (double)c->nf_modes : 0.0;
  f.inner = fp[0];
  f.outer = fp[1];
  f.e_per_mode = nf > 0 ? fp[2] / nf : 0.0;
  f.eps_h = fp[3];
  f.e_per_mode_b = (nf > 0 && c->nstate > 3) ? fp[4] / nf : 0.0;
  f.eps_h_b = c->nstate == 6 ? fp[5] : 0.0;
  f.FB = c->FB;
  ProfScope pr(c, "force", 0.0);
  TG_CK(launch_force_supply(f, c->st));
  c->force_ever = true;
  return TG_OK;
}

}  // namespace

namespace tg {
RKArgs rk_args(tg_ctx* c, int stage) {
  RKArgs a{};
  a.g = c->g;
  a.stage = stage;
  a.nstate = c->nstate;
  for (int i = 0; i < 6; ++i) {
    a.nu[i] = c->nu_of[i];
    a.nuh[i] = c->nuh_of[i];
    a.U0[i] = c->U0[i];
    a.TOT[i] = c->TOT[i];
    a.US[i] = c->US[i];
    a.RHS[i] = c->NL[i];
  }
  for (int q = 0; q < 9; ++q) a.PX[q] = c->PX[q];
  a.dt = c->scal;
  a.FB = c->force_on ? c->FB : nullptr;
  a.fx = c->fx;
  a.fy = c->fy;
  a.fz = c->fz;
  a.part = stage_is_final(stage) ? c->part : nullptr;
  a.rb_buoy_u = c->rb_fu;
  a.rb_buoy_t = c->rb_ft;
  a.nact = c->nact;
  a.nu_tab = c->nu_tab;
  a.coriolis = c->coriolis ? 1 : 0;
  for (int i = 0; i < 3; ++i) a.om[i] = c->om[i];
  a.lm = c->lm ? 1 : 0;
  for (int i = 0; i < 3; ++i) a.b0[i] = c->b0[i];
  return a;
}

// reduce the partials of slots r0 .. r0+n-1 and apply the dt rule to each of them
int run_finalize(tg_ctx* c, int dt_mode, bool ring, int r0, int n) {
  if (n < 0) n = c->nact;
  FinalizeArgs f{};
  f.part = c->part + (size_t)r0 * 8 * c->npart_blocks;
  f.nblocks = c->npart_blocks;
  f.nslots = 8;
  f.out = c->red_out + (size_t)r0 * 8;
  f.scal = c->scal + (size_t)r0 * 8;
  f.ering = (ring && r0 == 0) ? c->ering : nullptr;
  f.ering_pos = c->ering_pos;
  f.dt_mode = dt_mode;
  f.dx = c->dx_cfl;
  f.Tdt = c->cfg.dt;
  f.mhd = (c->phys == TG_MHD);
  f.nact = n;
  f.S = c->S;
  if (f.mhd) {
    // mean field B0 = real(B(0,0,0)) (compute_dt.cc:86-93): compact index 0 is the origin
    for (int i = 0; i < 3; ++i) f.B0[i] = c->U0[3 + i] + (size_t)r0 * c->S;
  }
  ProfScope pr(c, "finalize", 0.0);
  TG_CK(launch_finalize(f, c->st));
  return TG_OK;
}

}  // namespace tg

namespace tg {
// energy partials of the master state of slots r0 .. r0+n-1 into reduction slots (U: 0,1;
// B: 2,3; T: 4,5), then finalize
int run_energy_slots(tg_ctx* c, int dt_mode, int r0, int n) {
  const size_t o = (size_t)r0 * c->S;
  double* part = c->part + (size_t)r0 * 8 * c->npart_blocks;
  TG_CK(cudaMemsetAsync(part, 0, sizeof(double) * 8 * (size_t)c->npart_blocks * n, c->st));
  int nb = 0;
  const cx<double>* F[3] = {c->U0[0] + o, c->U0[1] + o, c->U0[2] + o};
  TG_CK(launch_energy_partials(c->g, F, 3, part, 0, 8, c->st, &nb, n));
  if (c->phys == TG_MHD) {
    const cx<double>* B[3] = {c->U0[3] + o, c->U0[4] + o, c->U0[5] + o};
    TG_CK(launch_energy_partials(c->g, B, 3, part, 2, 8, c->st, &nb, n));
  } else if (c->phys == TG_SCALAR || c->phys == TG_RB) {
    const cx<double>* T[1] = {c->U0[3] + o};
    TG_CK(launch_energy_partials(c->g, T, 1, part, 4, 8, c->st, &nb, n));
  }
  return run_finalize(c, dt_mode, false, r0, n);
}

int run_energy(tg_ctx* c, int dt_mode) { return run_energy_slots(c, dt_mode, 0, c->nact); }

int ensure_dt(tg_ctx* c) {
  if (c->energy_valid) return TG_OK;
  int rc = run_energy(c, 2);
  if (rc) return rc;
  c->energy_valid = true;
  return TG_OK;
}

int scheme_stages(int scheme, int out[4]) {
  if (scheme == TG_EULER) {
    out[0] = 5;
    return 1;
  }
  if (scheme == TG_RK2) {
    out[0] = 7;
    out[1] = 6;
    return 2;
  }
  for (int i = 0; i < 4; ++i) out[i] = i + 1;
  return 4;
}

// the stages first..last of the configured scheme's step on the fused path (first = 1: the
// whole step; 2: after a first stage from precomputed right-hand sides); `ring` records the
// step's energy
int run_stages(tg_ctx* c, int first, bool ring) {
  int st[4];
  const int ns_stages = scheme_stages(c->cfg.scheme, st);
  for (int si = first - 1; si < ns_stages; ++si) {
    const int stage = st[si];
    const void* in[6];
    int inprec;
    if (si == 0) {
      for (int i = 0; i < c->nstate; ++i) in[i] = c->U0[i];
      inprec = F64;
    } else {
      for (int i = 0; i < c->nstate; ++i) in[i] = c->US[i];
      inprec = c->tprec;
    }
    int rc = run_force(c, in, inprec);
    if (rc) return rc;
    rc = run_pipeline(c, in, inprec);
    if (rc) return rc;
    RKArgs a = rk_args(c, stage);
    for (int i = 0; i < c->nstate; ++i) a.IN[i] = in[i];
    a.inprec = (inprec == F64) ? 0 : 1;
    {
      // bytes: products and U0 read; TOT read (RK4 stages 2-4) and written (1-3); the stage
      // field written (1-3, 7) or U0 (final stages)
      const double ns = c->nstate, e = el_compact(c);
      const bool tot_rd = stage >= 2 && stage <= 4, tot_wr = stage >= 1 && stage <= 3;
      const double rd = c->nprod * e * c->tsz + ns * e * 16 + (tot_rd ? ns * e * 16 : 0);
      const double wr = (stage_is_final(stage) ? ns * e * 16 : ns * e * c->tsz) + (tot_wr ? ns * e * 16 : 0);
      ProfScope pr(c, "rk_stage", rd + wr);
      TG_CK(launch_rk(a, c->phys, c->tprec, c->tprec, 0, c->st, nullptr));
    }
  }
  return run_finalize(c, 1, ring);
}

int enqueue_step(tg_ctx* c, bool ring) { return run_stages(c, 1, ring); }
}  // namespace tg

namespace {

int field_state_index(const tg_ctx* c, int field) {
  if (field >= TG_V1 && field <= TG_V3) return field - TG_V1;
  if (field >= TG_W1 && field <= TG_W3 && c->phys == TG_MHD) return 3 + field - TG_W1;
  if (field == TG_T && (c->phys == TG_SCALAR || c->phys == TG_RB)) return 3;
  return -1;
}
int field_nl_index(const tg_ctx* c, int field) {
  if (field >= TG_NLIN1 && field <= TG_NLIN3) return field - TG_NLIN1;
  if (field >= TG_WNLIN1 && field <= TG_WNLIN3 && c->phys == TG_MHD) return 3 + field - TG_WNLIN1;
  if (field == TG_TNLIN && (c->phys == TG_SCALAR || c->phys == TG_RB)) return 3;
  return -1;
}

int ensure_dense(tg_ctx* c, int field) {
  if (c->dense[field]) return TG_OK;
  void* p = nullptr;
  int rc = dalloc(c, &p, sizeof(cx<double>) * (size_t)c->D);
  if (rc) return rc;
  c->dense[field] = (cx<double>*)p;
  return TG_OK;
}
int ensure_staging(tg_ctx* c) {
  if (c->staging) return TG_OK;
  void* p = nullptr;
  int rc = dalloc(c, &p, sizeof(cx<double>) * (size_t)c->D);
  if (rc) return rc;
  c->staging = (cx<double>*)p;
  return TG_OK;
}

// dense transforms of a work field, in place: FOUR (ArrayFFT_FOUR / ArrayIFFT_FOUR) or SCFT with
// parity 0 cos / 1 sin along x (ArrayCFT/SFT_SCFT, ArrayICFT/ISFT_SCFT)
int dense_transform(tg_ctx* c, cx<double>* f, int forward, int parity) {
  const int wp = (c->prec == TG_FP64) ? F64 : F32;
  const long long M3 = c->M3;
  if (forward) {
    ZLaunch z;
    z.M = c->Mz;
    z.kind = 1;
    z.pin = F64;
    z.pout = F64;
    z.pwork = wp;
    z.a.nrows = (long long)c->N1 * c->N2;
    z.a.ss = M3;
    z.a.ds = M3;
    z.a.nout = (int)M3;
    z.a.nfill = (int)M3;
    z.a.scale = 1.0 / ((double)c->N1 * c->N2 * c->N3);
    z.a.twM = c->tw[c->Mz];
    z.a.twN = c->tw[c->N3];
    z.ps.src[0] = f;
    z.ps.dst[0] = f;
    TG_CK(launch_z(z, c->st));
  }
  for (int pass = 0; pass < 2; ++pass) {
    // inverse: x then y; forward: y then x
    const bool xpass = forward ? (pass == 1) : (pass == 0);
    AxisLaunch l;
    wait_args(c, l.a);
    l.dir = forward ? -1 : +1;
    l.pin = F64;
    l.pout = F64;
    l.pwork = wp;
    l.nfields = 1;
    l.a.scale = 1.0;
    l.ps.src[0] = f;
    l.ps.dst[0] = f;
    if (xpass) {
      l.L = c->N1;
      l.nbatch = 1;
      l.a.sb = l.a.db = 0;
      l.a.sr = l.a.dr = (long long)c->N2 * M3;
      l.a.ncols = (int)(c->N2 * M3);
      l.a.in = l.a.out = full_map(c->N1);
      l.a.tw = c->tw[c->N1];
    } else {
      l.L = c->N2;
      l.nbatch = c->N1;
      l.a.sb = l.a.db = (long long)c->N2 * M3;
      l.a.sr = l.a.dr = M3;
      l.a.ncols = (int)M3;
      l.a.in = l.a.out = full_map(c->N2);
      l.a.tw = c->tw[c->N2];
    }
    if (xpass && c->basis == TG_SCFT) {
      R2RArgs r{};
      r.kind[0] = forward ? (parity ? 1 : 0) : (parity ? 3 : 2);
      r.trig = c->trigx;
      if (forward) l.a.scale = 0.5;  // Norm_SCFT 1/(2 N1 N2 N3)
      TG_CK(launch_r2r(l, r, c->st));
    } else {
      TG_CK(launch_axis(l, c->st));
    }
  }
  if (!forward) {
    ZLaunch z;
    z.M = c->Mz;
    z.kind = 0;
    z.pin = F64;
    z.pout = F64;
    z.pwork = wp;
    z.a.nrows = (long long)c->N1 * c->N2;
    z.a.ss = M3;
    z.a.ds = M3;
    z.a.nin = (int)M3;
    z.a.pad = 1;
    z.a.scale = 1.0;
    z.a.twM = c->tw[c->Mz];
    z.a.twN = c->tw[c->N3];
    z.ps.src[0] = f;
    z.ps.dst[0] = f;
    TG_CK(launch_z(z, c->st));
  }
  return TG_OK;
}

void free_ctx(tg_ctx* c) {
  if (!c) return;
  if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
  auto fr = [](void* p) {
    if (p) cudaFree(p);
  };
  for (auto& kv : c->tw) fr(kv.second);
  for (int i = 0; i < 6; ++i) {
    fr(c->U0[i]);
    fr(c->TOT[i]);
    fr(c->US[i]);
    fr(c->NL[i]);
    fr(c->WX[i]);
    fr(c->WY[i]);
  }
  for (int i = 0; i < 9; ++i) {
    fr(c->PP[i]);
    fr(c->PY[i]);
    fr(c->PX[i]);
    fr(c->SA[i]);
    fr(c->SB[i]);
  }
  for (int i = 0; i < 6; ++i) fr(c->SR[i]);
  fr(c->gsum);
  fr(c->PR);
  fr(c->FB);
  fr(c->trigx);
  fr(c->zoct);
  for (int k = 0; k < 4; ++k) fr(c->xmat[k]);
  fr(c->scal);
  fr(c->nu_tab);
  fr(c->red_out);
  fr(c->part);
  fr(c->ering);
  fr(c->ering_pos);
  fr(c->diag);
  for (int i = 0; i < 3; ++i) fr(c->etG[i]);
  for (int i = 0; i < c->n_et_own; ++i) fr(c->et_own[i]);
  for (int i = 0; i < TG_NFIELDS; ++i) fr(c->dense[i]);
  fr(c->staging);
  for (auto& r : c->prof_recs) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (auto e : c->ev_pool) cudaEventDestroy(e);
  if (c->h_pinned) cudaFreeHost(c->h_pinned);
  if (c->h_wait) cudaFreeHost(c->h_wait);
  if (c->own_stream && c->st) cudaStreamDestroy(c->st);
  delete c;
}

// Get_number_modes_in_shell_FOUR (four_basic.cc:48-105): inner <= |K| < outer, kz = 0 once,
// kz > 0 twice
int count_force_modes(const tg_config& cfg) {
  const double inner = cfg.force_para[0], outer = cfg.force_para[1];
  const int kxm = (int)std::ceil(outer / cfg.kfactor[0]);
  const int kym = (int)std::ceil(outer / cfg.kfactor[1]);
  const int kzm = (int)std::ceil(outer / cfg.kfactor[2]);
  int cnt = 0;
  // Get_number_modes_in_shell_FOUR / _SCFT (four_basic.cc:48-105, scft_basic.cc:48-106): SCFT
  // counts kx >= 0 only
  for (int kx = cfg.basis == TG_SCFT ? 0 : -kxm; kx <= kxm; ++kx)
    for (int ky = -kym; ky <= kym; ++ky)
      for (int kz = 0; kz <= kzm; ++kz) {
        const double a = kx * cfg.kfactor[0], b = ky * cfg.kfactor[1], d = kz * cfg.kfactor[2];
        const double km = std::sqrt(a * a + b * b + d * d);
        if (km >= inner && km < outer) cnt += (kz == 0) ? 1 : 2;
      }
  return cnt;
}

}  // namespace

// =====================================================================================
// C ABI
// =====================================================================================
extern "C" {

void tg_config_default(tg_config* cfg) {
  if (!cfg) return;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->N[0] = cfg->N[1] = cfg->N[2] = 64;
  cfg->basis = TG_FOUR;
  cfg->physics = TG_FLUID;
  cfg->precision = TG_FP64;
  cfg->dealias = 1;
  cfg->scheme = TG_RK4;
  cfg->kfactor[0] = cfg->kfactor[1] = cfg->kfactor[2] = 1.0;
  cfg->nu = 0.01;
  cfg->eta = 0.01;
  cfg->kappa = 0.01;
  cfg->dt = 1e-3;
  cfg->force_kind = TG_FORCE_DECAY;
  cfg->n_shells = 12;
  cfg->rb_temp_grad = 1.0;
  cfg->device = 0;
  cfg->stream = nullptr;
}

const char* tg_last_error(const tg_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

}  // extern "C"

namespace tg {
int ctx_create_batch(const tg_config* cfg, int B, tg_ctx** out, int slab_W, int slab_r) {
  if (!cfg || !out || B < 1) return TG_ERR_ARG;
  if (slab_W < 0 || (slab_W > 0 && (B != 1 || slab_r < 0 || slab_r >= slab_W))) return TG_ERR_ARG;
  *out = nullptr;
  {
    const int v = validate_config(cfg);
    if (v) return v;
  }
  const int N1 = cfg->N[0], N2 = cfg->N[1], N3 = cfg->N[2];
  // the fused product z-pass needs N3/2 in {4..256} (a power of two); other grids get the
  // transform API only.  The x and y passes take any length.
  const int Mz = N3 / 2;
  const bool pipeline_ok = is_pow2(Mz) && Mz >= 4 && Mz <= 256;

  tg_ctx* c = new tg_ctx();
  c->cfg = *cfg;
  c->dev = cfg->device;
  cudaError_t e = cudaSetDevice(c->dev);
  if (e != cudaSuccess) {
    delete c;
    return TG_ERR_CUDA;
  }
  if (cfg->stream) {
    c->st = (cudaStream_t)cfg->stream;
  } else {
    if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) {
      delete c;
      return TG_ERR_CUDA;
    }
    c->own_stream = true;
  }
  c->pipeline_ok = pipeline_ok;
  c->N1 = N1;
  c->N2 = N2;
  c->N3 = N3;
  c->M3 = N3 / 2 + 1;
  c->Mz = Mz;
  c->phys = cfg->physics;
  c->basis = cfg->basis;
  c->prec = cfg->precision;
  c->tprec = (c->prec == TG_FP64) ? F64 : F32;
  c->tsz = (c->tprec == F64) ? sizeof(cx<double>) : sizeof(cx<float>);
  int lo, hi;
  Geo& g = c->g;
  g.N1 = N1;
  g.N2 = N2;
  g.N3 = N3;
  keep_axis(N1, 0, c->basis, cfg->dealias, lo, hi);
  g.ax = AxisMap{N1, lo, hi};
  keep_axis(N2, 1, c->basis, cfg->dealias, lo, hi);
  g.ay = AxisMap{N2, lo, hi};
  g.nkx = amap_count(g.ax);
  g.nky = amap_count(g.ay);
  g.nkz = (cfg->dealias && N3 >= 3) ? N3 / 3 : N3 / 2 + 1;
  g.kzp = (g.nkz + 7) / 8 * 8;
  g.S = (long long)g.nkx * g.nky * g.kzp;
  g.kf0 = cfg->kfactor[0];
  g.kf1 = cfg->kfactor[1];
  g.kf2 = cfg->kfactor[2];
  g.basis = c->basis;
  g.x0 = 0;
  if (slab_W > 0) {
    // rank slab_r's compact kx rows and real y planes (the reference's slab decomposition,
    // basis_basicfn.cc:49-281: x slabs in spectral space, y slabs in real space)
    if (g.nkx < slab_W || N2 < slab_W) {
      free_ctx(c);
      return TG_ERR_ARG;
    }
    c->slab_W = slab_W;
    c->slab_r = slab_r;
    c->slab_x.resize(slab_W);
    c->slab_nx.resize(slab_W);
    c->slab_y.resize(slab_W);
    c->slab_ny.resize(slab_W);
    for (int i = 0; i < slab_W; ++i) {
      split_range(g.nkx, slab_W, i, c->slab_x[i], c->slab_nx[i]);
      split_range(N2, slab_W, i, c->slab_y[i], c->slab_ny[i]);
    }
    g.x0 = c->slab_x[slab_r];
    g.S = (long long)c->slab_nx[slab_r] * g.nky * g.kzp;
  }
  c->S = g.S;
  c->D = (long long)N1 * N2 * c->M3;

  // physics layout of the pipeline
  ProdPairs& pp = c->pairs;
  if (c->phys == TG_FLUID) {
    c->nstate = 3;
    c->nin = 3;
    c->nprod = 6;
    const signed char PA[6] = {0, 1, 2, 0, 1, 2}, PB[6] = {0, 1, 2, 1, 2, 0};
    for (int q = 0; q < 6; ++q) {
      pp.a[q] = PA[q];
      pp.b[q] = PB[q];
    }
  } else if (c->phys == TG_MHD) {
    c->nstate = 6;
    c->nin = 6;
    c->nprod = 9;
    // inputs 0..2 = z+, 3..5 = z-
    const signed char PA[9] = {0, 1, 2, 0, 3, 1, 4, 2, 5}, PB[9] = {3, 4, 5, 4, 1, 5, 2, 3, 0};
    for (int q = 0; q < 9; ++q) {
      pp.a[q] = PA[q];
      pp.b[q] = PB[q];
    }
  } else {
    c->nstate = 4;
    c->nin = 4;
    c->nprod = 9;
    const signed char PA[9] = {0, 1, 2, 0, 1, 2, 0, 1, 2}, PB[9] = {0, 1, 2, 1, 2, 0, 3, 3, 3};
    for (int q = 0; q < 9; ++q) {
      pp.a[q] = PA[q];
      pp.b[q] = PB[q];
    }
    if (c->phys == TG_RB && (cfg->force_kind == TG_FORCE_RB || cfg->force_kind == TG_FORCE_RB_ROTATION)) {
      // Compute_force_RB: Force1 = fu theta, T.Force = ft u1
      const RBCoef r = rb_coefficients(cfg);
      c->rb_fu = r.fu;
      c->rb_ft = r.ft;
    }
  }

  state_viscosities(cfg, c->nu_of);
  state_hyper(cfg, c->nuh_of);

  int rc = TG_OK;
  auto fail = [&](int code) {
    std::string m = c->err;
    free_ctx(c);
    return code;
  };
  // SCFT x-pass kinds by field parity: u1, theta sine; u2, u3 cosine (Rvf.cc:135-186,
  // compute_nlin_SF.cc:80-115); products u1u1, u2u2, u3u3, u2u3, u1 theta cos; u1u2, u3u1,
  // u2 theta, u3 theta sin
  {
    const int inv[6] = {3, 2, 2, 3, 0, 0};
    const int fwd[9] = {0, 0, 0, 1, 0, 1, 0, 1, 1};
    for (int i = 0; i < 6; ++i) c->xinv_kind[i] = inv[i];
    for (int q = 0; q < 9; ++q) c->xfwd_kind[q] = fwd[q];
  }
  if (c->basis == TG_SCFT) {
    std::vector<cx<double>> h(4 * (size_t)N1);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int j = 0; j < 4 * N1; ++j) {
      const long double ang = pi * (long double)j / (2.0L * N1);
      h[j].x = (double)cosl(ang);
      h[j].y = (double)sinl(ang);
    }
    if ((rc = dalloc(c, (void**)&c->trigx, sizeof(cx<double>) * h.size()))) return fail(rc);
    e = cudaMemcpy(c->trigx, h.data(), sizeof(cx<double>) * h.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(cuda_err(c, e, "trig table"));
    // the x-pass of the pipeline as matrices [stored input row][output row] (the coefficients
    // of k_axis_r2r): inverse kinds 2, 3 map the nkx stored slots m to all N1 points,
    // forward kinds 0, 1 map the N1 points to the nkx kept slots
    const int nk = g.nkx, fourN = 4 * N1;
    for (int kind = 0; kind < 4; ++kind) {
      const bool sine = (kind == 1 || kind == 3);
      const bool fwd = kind <= 1;
      const int nin = fwd ? N1 : nk, nout = fwd ? nk : N1;
      std::vector<double> m((size_t)nin * nout);
      for (int rr = 0; rr < nin; ++rr)
        for (int ko = 0; ko < nout; ++ko) {
          double t;
          if (fwd) {
            const int j = (int)(((long long)(2 * rr + 1) * ko) % fourN);
            t = 2.0 * (sine ? h[j].y : h[j].x);
          } else {
            const int mm = amap_index(g.ax, rr);
            const int j = (int)(((long long)mm * (2 * ko + 1)) % fourN);
            t = (sine ? h[j].y : h[j].x) * ((mm == 0 && !sine) ? 1.0 : 2.0);
          }
          m[(size_t)rr * nout + ko] = t;
        }
      if ((rc = dalloc(c, (void**)&c->xmat[kind], sizeof(double) * m.size()))) return fail(rc);
      e = cudaMemcpy(c->xmat[kind], m.data(), sizeof(double) * m.size(), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) return fail(cuda_err(c, e, "x-pass matrices"));
      c->xmat_rows[kind] = nout;
      c->xmat_cols[kind] = nin;
    }
  }
  for (int L : {N1, N2, Mz, N3}) {
    rc = make_twiddles(c, L);
    if (rc) return fail(rc);
  }
  if (N3 == 256 || N3 == 128) {
    std::vector<cx<double>> t(kZoctTableLen);
    zoct_table(N3 / 2, t.data());
    if ((rc = dalloc(c, (void**)&c->zoct, sizeof(cx<double>) * t.size()))) return fail(rc);
    e = cudaMemcpy(c->zoct, t.data(), sizeof(cx<double>) * t.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(cuda_err(c, e, "z-pass table"));
  }
  // a batch of B same-shape requests stores request r of every field at offset r * S
  c->B = B;
  c->nact = 1;
  const size_t Sd1 = sizeof(cx<double>) * (size_t)g.S;
  const size_t Sd = Sd1 * B;
  const size_t St = c->tsz * (size_t)g.S * B;
  size_t WXb = c->tsz * (size_t)N1 * g.nky * g.kzp * B;
  const size_t WYb = c->tsz * (size_t)N1 * N2 * g.kzp * B;
  size_t PPb = WYb, PYb = WXb;
  if (slab_W > 0) {
    // between the exchanges: [N1][ny][kzp] (x-inverse outputs, products), [nkx][ny][kzp]
    // (x-forward outputs = forward send)
    const size_t ny = (size_t)c->slab_ny[slab_r], nx = (size_t)c->slab_nx[slab_r];
    WXb = PPb = c->tsz * (size_t)N1 * ny * g.kzp;
    PYb = c->tsz * (size_t)g.nkx * ny * g.kzp;
    const size_t Ab = c->tsz * nx * N2 * g.kzp;
    for (int q = 0; q < c->nprod; ++q) {
      if ((rc = dalloc(c, &c->SA[q], Ab))) return fail(rc);
      if ((rc = dalloc(c, &c->SB[q], Ab))) return fail(rc);
    }
    for (int i = 0; i < c->nin; ++i)
      if ((rc = dalloc(c, &c->SR[i], PYb))) return fail(rc);
    if ((rc = dalloc(c, (void**)&c->gsum, sizeof(double) * 16))) return fail(rc);
  }
  for (int i = 0; i < c->nstate; ++i) {
    if ((rc = dalloc(c, (void**)&c->U0[i], Sd))) return fail(rc);
    if ((rc = dalloc(c, (void**)&c->TOT[i], Sd))) return fail(rc);
    if ((rc = dalloc(c, &c->US[i], St))) return fail(rc);
    if ((rc = dalloc(c, (void**)&c->NL[i], Sd1))) return fail(rc);
  }
  if ((rc = dalloc(c, (void**)&c->PR, Sd1))) return fail(rc);
  for (int i = 0; i < c->nin; ++i) {
    if ((rc = dalloc(c, &c->WX[i], WXb))) return fail(rc);
    if (slab_W == 0 && (rc = dalloc(c, &c->WY[i], WYb))) return fail(rc);
  }
  for (int q = 0; q < c->nprod; ++q) {
    if ((rc = dalloc(c, &c->PP[q], PPb))) return fail(rc);
    if ((rc = dalloc(c, &c->PY[q], PYb))) return fail(rc);
    if ((rc = dalloc(c, &c->PX[q], St))) return fail(rc);
  }
  c->npart_blocks = reduction_blocks(g.S);
  if ((rc = dalloc(c, (void**)&c->part, sizeof(double) * 8 * (size_t)c->npart_blocks * B))) return fail(rc);
  if ((rc = dalloc(c, (void**)&c->scal, sizeof(double) * 8 * B))) return fail(rc);
  if ((rc = dalloc(c, (void**)&c->red_out, sizeof(double) * 8 * B))) return fail(rc);
  if ((rc = dalloc(c, (void**)&c->nu_tab, sizeof(double) * 6 * B))) return fail(rc);
  {
    std::vector<double> nut((size_t)6 * B);
    for (int r = 0; r < B; ++r)
      for (int i = 0; i < 6; ++i) nut[(size_t)r * 6 + i] = c->nu_of[i];
    e = cudaMemcpyAsync(c->nu_tab, nut.data(), sizeof(double) * nut.size(), cudaMemcpyHostToDevice, c->st);
    if (e != cudaSuccess) return fail(cuda_err(c, e, "init viscosities"));
  }
  c->ering_cap = 1 << 16;
  if ((rc = dalloc(c, (void**)&c->ering, sizeof(double) * c->ering_cap))) return fail(rc);
  if ((rc = dalloc(c, (void**)&c->ering_pos, sizeof(int) * 4))) return fail(rc);
  c->wait_status = c->ering_pos + 2;
  if (cudaMallocHost(&c->h_pinned, sizeof(double) * 1024) != cudaSuccess) return fail(TG_ERR_OOM);
  if (cudaMallocHost(&c->h_wait, sizeof(int) * 4) != cudaSuccess) return fail(TG_ERR_OOM);
  *c->h_wait = 0;
  {
    // per request: dt, t, steps, non-finite flag, Tdt
    std::vector<double> init((size_t)8 * B, 0.0);
    for (int r = 0; r < B; ++r) {
      init[(size_t)r * 8 + 0] = cfg->dt;
      init[(size_t)r * 8 + 4] = cfg->dt;
    }
    e = cudaMemcpyAsync(c->scal, init.data(), sizeof(double) * init.size(), cudaMemcpyHostToDevice, c->st);
    if (e != cudaSuccess) return fail(cuda_err(c, e, "init scalars"));
    e = cudaStreamSynchronize(c->st);
    if (e != cudaSuccess) return fail(cuda_err(c, e, "init scalars"));
  }
  c->dx_cfl = 2 * M_PI / std::max(1, max_radius_inside(c));
  if (cfg->force_kind == TG_FORCE_ENERGY_SUPPLY || cfg->force_kind == TG_FORCE_ENERGY_HELICITY) {
    if (B != 1) return fail(set_err(c, TG_ERR_UNSUPPORTED, "forced requests are not batched"));
    c->force_on = 1;
    const double outer = cfg->force_para[1];
    c->fx = (int)std::ceil(outer / cfg->kfactor[0]);
    c->fy = (int)std::ceil(outer / cfg->kfactor[1]);
    c->fz = (int)std::ceil(outer / cfg->kfactor[2]);
    c->fbox = (2 * c->fx + 1) * (2 * c->fy + 1) * (c->fz + 1);
    c->nf_modes = count_force_modes(*cfg);
    if (c->nf_modes <= 0) return fail(set_err(c, TG_ERR_ARG, "forcing shell holds no modes"));
    if ((rc = dalloc(c, (void**)&c->FB, sizeof(cx<double>) * c->nstate * (size_t)c->fbox))) return fail(rc);
  } else if (cfg->force_kind == TG_FORCE_MODES) {
    if (B != 1) return fail(set_err(c, TG_ERR_UNSUPPORTED, "forced requests are not batched"));
    c->force_on = 2;  // the box is allocated by tg_set_force_modes
  } else if (cfg->force_kind == TG_FORCE_LIQUID_METAL) {
    c->lm = true;
    for (int i = 0; i < 3; ++i) c->b0[i] = cfg->force_para[i];
  } else if (cfg->force_kind == TG_FORCE_CORIOLIS || cfg->force_kind == TG_FORCE_RB_ROTATION) {
    c->coriolis = true;
    // Compute_force_RB_rotation scales the Coriolis force with the nondimensionalisation
    double sc = 1.0;
    if (cfg->force_kind == TG_FORCE_RB_ROTATION) {
      if (cfg->rb_u_scaling == TG_RB_ULARGE) sc = std::sqrt(cfg->rb_pr / cfg->rb_ra);
      else if (cfg->rb_pr_switch == TG_RB_PRLARGE) sc = cfg->rb_pr;
    }
    for (int i = 0; i < 3; ++i) c->om[i] = sc * cfg->force_para[i];
  }
  e = cudaStreamSynchronize(c->st);
  if (e != cudaSuccess) return fail(cuda_err(c, e, "create"));
  *out = c;
  return TG_OK;
}

int validate_config(const tg_config* cfg) {
  if (!cfg) return TG_ERR_ARG;
  const int N1 = cfg->N[0], N2 = cfg->N[1], N3 = cfg->N[2];
  if (N1 < 2 || N2 < 2 || N3 < 4 || (N3 & 1)) return TG_ERR_ARG;
  if (cfg->basis != TG_FOUR && cfg->basis != TG_SCFT) return TG_ERR_ARG;
  if (cfg->physics < TG_FLUID || cfg->physics > TG_RB) return TG_ERR_ARG;
  if (cfg->basis == TG_SCFT && cfg->physics == TG_MHD) return TG_ERR_UNSUPPORTED;
  if (cfg->physics == TG_RB && !(cfg->rb_ra > 0 && cfg->rb_pr > 0)) return TG_ERR_ARG;
  if (cfg->physics == TG_RB &&
      ((cfg->rb_pr_switch != TG_RB_PRLARGE && cfg->rb_pr_switch != TG_RB_PRSMALL) ||
       (cfg->rb_u_scaling != TG_RB_ULARGE && cfg->rb_u_scaling != TG_RB_USMALL) || !std::isfinite(cfg->rb_temp_grad)))
    return TG_ERR_ARG;
  if (cfg->precision != TG_FP64 && cfg->precision != TG_FP32_MIXED) return TG_ERR_ARG;
  if (cfg->scheme != TG_RK4 && cfg->scheme != TG_RK2 && cfg->scheme != TG_EULER) return TG_ERR_UNSUPPORTED;
  if (!(cfg->hyper_nu >= 0 && cfg->hyper_eta >= 0 && cfg->hyper_kappa >= 0) || !std::isfinite(cfg->hyper_nu) ||
      !std::isfinite(cfg->hyper_eta) || !std::isfinite(cfg->hyper_kappa))
    return TG_ERR_ARG;
  if (cfg->force_kind != TG_FORCE_DECAY && cfg->force_kind != TG_FORCE_ENERGY_SUPPLY &&
      cfg->force_kind != TG_FORCE_ENERGY_HELICITY && cfg->force_kind != TG_FORCE_RB &&
      cfg->force_kind != TG_FORCE_LIQUID_METAL &&
      cfg->force_kind != TG_FORCE_MODES && cfg->force_kind != TG_FORCE_CORIOLIS && cfg->force_kind != TG_FORCE_RB_ROTATION)
    return TG_ERR_UNSUPPORTED;
  if ((cfg->force_kind == TG_FORCE_RB || cfg->force_kind == TG_FORCE_RB_ROTATION) && cfg->physics != TG_RB)
    return TG_ERR_ARG;
  if (cfg->force_kind == TG_FORCE_RB_ROTATION)
    for (int i = 0; i < 3; ++i)
      if (!std::isfinite(cfg->force_para[i])) return TG_ERR_ARG;
  // convection has its own force (force_field_proc 51)
  if ((cfg->force_kind == TG_FORCE_MODES || cfg->force_kind == TG_FORCE_CORIOLIS) && cfg->physics == TG_RB)
    return TG_ERR_UNSUPPORTED;
  if (cfg->force_kind == TG_FORCE_CORIOLIS || cfg->force_kind == TG_FORCE_LIQUID_METAL)
    for (int i = 0; i < 3; ++i)
      if (!std::isfinite(cfg->force_para[i])) return TG_ERR_ARG;
  // the liquid-metal force is the fluid's force_field_proc 101 (FOUR: Array_mult_V0_khat_sqr_FOUR)
  if (cfg->force_kind == TG_FORCE_LIQUID_METAL && (cfg->physics != TG_FLUID || cfg->basis != TG_FOUR))
    return TG_ERR_UNSUPPORTED;
  if (cfg->force_kind == TG_FORCE_ENERGY_SUPPLY || cfg->force_kind == TG_FORCE_ENERGY_HELICITY) {
    // band forcings: fluid, MHD and passive scalar (convection has its own force); FOUR, and
    // SCFT for the fluid and the passive scalar (MHD runs FOUR only here)
    if (cfg->physics == TG_RB) return TG_ERR_UNSUPPORTED;
    if (!(cfg->force_para[1] > cfg->force_para[0])) return TG_ERR_ARG;
    for (int i = 0; i < 6; ++i)
      if (!std::isfinite(cfg->force_para[i])) return TG_ERR_ARG;
  }
  for (int i = 0; i < 3; ++i)
    if (!(cfg->kfactor[i] > 0)) return TG_ERR_ARG;
  if (!(cfg->dt > 0)) return TG_ERR_ARG;
  return TG_OK;
}

// RB coefficients of a nondimensionalisation (RB_slip_main.cc:222-262, compute_force_RB.cc:
// 50-105, nusselt.cc:53-89): nu (grad^2 u), kappa (grad^2 theta), Force1 = fu theta,
// T.Force = ft u1, Nu = 1 + nuf <u1, theta> (nuf times the Get_total_energy cross term)
RBCoef rb_coefficients(const tg_config* cfg) {
  const double Ra = cfg->rb_ra, Pr = cfg->rb_pr, g = cfg->rb_temp_grad;
  RBCoef r{};
  const bool small_u = cfg->rb_u_scaling == TG_RB_USMALL;
  if (cfg->rb_pr_switch == TG_RB_PRSMALL) {
    r.nu = small_u ? 1.0 : std::sqrt(Pr / Ra);
    r.kappa = small_u ? 1.0 / Pr : 1.0 / std::sqrt(Pr * Ra);
    r.fu = small_u ? Ra : Pr;
    r.ft = g / Pr;
    r.nuf = small_u ? 2 * Pr * Pr : 2 * Pr * std::sqrt(Ra * Pr);
  } else {
    r.nu = small_u ? Pr : std::sqrt(Pr / Ra);
    r.kappa = small_u ? 1.0 : 1.0 / std::sqrt(Pr * Ra);
    r.fu = small_u ? Ra * Pr : 1.0;
    r.ft = g;
    r.nuf = small_u ? 2.0 : 2 * std::sqrt(Ra * Pr);
  }
  return r;
}

void state_hyper(const tg_config* cfg, double nuh[6]) {
  for (int i = 0; i < 6; ++i) nuh[i] = 0.0;
  for (int i = 0; i < 3; ++i) nuh[i] = cfg->hyper_nu;
  if (cfg->physics == TG_MHD) {
    for (int i = 0; i < 3; ++i) nuh[3 + i] = cfg->hyper_eta;
  } else if (cfg->physics == TG_SCALAR || cfg->physics == TG_RB) {
    nuh[3] = cfg->hyper_kappa;
  }
}

void state_viscosities(const tg_config* cfg, double nu[6]) {
  for (int i = 0; i < 6; ++i) nu[i] = 0.0;
  for (int i = 0; i < 3; ++i) nu[i] = cfg->nu;
  if (cfg->physics == TG_MHD) {
    for (int i = 0; i < 3; ++i) nu[3 + i] = cfg->eta;
  } else if (cfg->physics == TG_SCALAR) {
    nu[3] = cfg->kappa;
  } else if (cfg->physics == TG_RB) {
    const RBCoef r = rb_coefficients(cfg);
    for (int i = 0; i < 3; ++i) nu[i] = r.nu;
    nu[3] = r.kappa;
  }
}

int ensure_staging_ctx(tg_ctx* c) { return ensure_staging(c); }

int radius_inside(const tg_ctx* c) { return max_radius_inside(c); }

int ensure_force_box(tg_ctx* c) {
  if (c->force_on != 1 || c->force_ever) return TG_OK;
  const void* U[6];
  for (int i = 0; i < c->nstate; ++i) U[i] = c->U0[i];
  return run_force(c, U, F64);
}

// Device bytes that ctx_create_batch(cfg, B) allocates (same sizes, same order), plus the dense
// staging field that uploads and downloads add (with_staging).  0 for a configuration that
// ctx_create_batch rejects on its shape.
size_t ctx_bytes_estimate(const tg_config* cfg, int B, bool with_staging) {
  if (!cfg || B < 1) return 0;
  const int N1 = cfg->N[0], N2 = cfg->N[1], N3 = cfg->N[2];
  if (N1 < 2 || N2 < 2 || N3 < 4 || (N3 & 1)) return 0;
  const int Mz = N3 / 2;
  int lo, hi;
  keep_axis(N1, 0, cfg->basis, cfg->dealias, lo, hi);
  const int nkx = amap_count(AxisMap{N1, lo, hi});
  keep_axis(N2, 1, cfg->basis, cfg->dealias, lo, hi);
  const int nky = amap_count(AxisMap{N2, lo, hi});
  const int nkz = (cfg->dealias && N3 >= 3) ? N3 / 3 : N3 / 2 + 1;
  const int kzp = (nkz + 7) / 8 * 8;
  const size_t S = (size_t)nkx * nky * kzp;
  const size_t tsz = cfg->precision == TG_FP64 ? sizeof(cx<double>) : sizeof(cx<float>);
  int nstate = 3, nin = 3, nprod = 6;
  if (cfg->physics == TG_MHD) {
    nstate = nin = 6;
    nprod = 9;
  } else if (cfg->physics == TG_SCALAR || cfg->physics == TG_RB) {
    nstate = nin = 4;
    nprod = 9;
  }
  size_t b = 0;
  std::vector<int> lens;
  for (int L : {N1, N2, Mz, N3})
    if (std::find(lens.begin(), lens.end(), L) == lens.end()) {
      lens.push_back(L);
      b += sizeof(cx<double>) * (size_t)L;
    }
  if (cfg->basis == TG_SCFT) b += sizeof(cx<double>) * 4 * (size_t)N1 + sizeof(double) * 4 * (size_t)N1 * nkx;
  if (N3 == 256 || N3 == 128) b += sizeof(cx<double>) * (size_t)kZoctTableLen;
  const size_t Sd1 = sizeof(cx<double>) * S;
  const size_t WXb = tsz * (size_t)N1 * nky * kzp * B;
  const size_t WYb = tsz * (size_t)N1 * N2 * kzp * B;
  b += (size_t)nstate * (2 * Sd1 * B + tsz * S * B + Sd1) + Sd1;
  b += (size_t)nin * (WXb + WYb);
  b += (size_t)nprod * (WYb + WXb + tsz * S * B);
  b += sizeof(double) * 8 * (size_t)reduction_blocks((long long)S) * B;
  b += sizeof(double) * (8 + 8 + 6) * (size_t)B;
  b += sizeof(double) * (1 << 16) + sizeof(int) * 4;
  if (cfg->force_kind == TG_FORCE_ENERGY_SUPPLY || cfg->force_kind == TG_FORCE_ENERGY_HELICITY) {
    const double outer = cfg->force_para[1];
    const int fx = (int)std::ceil(outer / cfg->kfactor[0]), fy = (int)std::ceil(outer / cfg->kfactor[1]),
              fz = (int)std::ceil(outer / cfg->kfactor[2]);
    b += sizeof(cx<double>) * nstate * (size_t)(2 * fx + 1) * (2 * fy + 1) * (fz + 1);
  }
  if (with_staging) b += sizeof(cx<double>) * (size_t)N1 * N2 * (N3 / 2 + 1);
  return b;
}
}  // namespace tg

extern "C" {

int tg_ctx_create(const tg_config* cfg, tg_ctx** out) { return tg::ctx_create_batch(cfg, 1, out); }

int tg_ctx_destroy(tg_ctx* c) {
  if (!c) return TG_ERR_ARG;
  cudaSetDevice(c->dev);
  cudaStreamSynchronize(c->st);
  free_ctx(c);
  return TG_OK;
}

int tg_debug_set(tg_ctx* c, int what, long long value) {
  if (!c) return TG_ERR_ARG;
  if (what != TG_DEBUG_SHORT_TMA_WAIT || (value != 0 && value != 1)) return TG_ERR_ARG;
  cudaSetDevice(c->dev);
  TG_SYNC(c, "tg_debug_set");
  c->wait_short = (int)value;
  // the step graph holds the pass arguments it was captured with
  if (c->step_graph) {
    cudaGraphExecDestroy(c->step_graph);
    c->step_graph = nullptr;
  }
  return TG_OK;
}

int tg_synchronize(tg_ctx* c) {
  if (!c) return TG_ERR_ARG;
  TG_SYNC(c, __func__);
  return TG_OK;
}

int tg_device_bytes(const tg_ctx* c, size_t* bytes) {
  if (!c || !bytes) return TG_ERR_ARG;
  *bytes = c->bytes;
  return TG_OK;
}

namespace {

// The stored modes of a dense reference-layout field [l1][l2][0..N3/2] are up to four boxes
// (kept x rows [0, lo) and [N1 - hi, N1), the same for y, kz < nkz); each box is one 3-D
// pitched copy between the dense array and the compact rows [r1][r2][0..kzp).
cudaError_t copy_stored(tg_ctx* c, cx<double>* compact, double* dense, bool to_device) {
  const Geo& g = c->g;
  const size_t e = sizeof(cx<double>);
  const int xs[2][2] = {{0, g.ax.lo}, {g.ax.L - g.ax.hi, g.ax.hi}};
  const int ys[2][2] = {{0, g.ay.lo}, {g.ay.L - g.ay.hi, g.ay.hi}};
  int r1 = 0;
  for (int bx = 0; bx < 2; ++bx) {
    const int x0 = xs[bx][0], nx = xs[bx][1];
    if (nx <= 0) continue;
    int r2 = 0;
    for (int by = 0; by < 2; ++by) {
      const int y0 = ys[by][0], ny = ys[by][1];
      if (ny <= 0) continue;
      cudaMemcpy3DParms p = {};
      cudaPitchedPtr hp = make_cudaPitchedPtr(dense, (size_t)c->M3 * e, (size_t)c->M3 * e, (size_t)c->N2);
      cudaPitchedPtr dp = make_cudaPitchedPtr(compact, (size_t)g.kzp * e, (size_t)g.kzp * e, (size_t)g.nky);
      const cudaPos hpos = make_cudaPos(0, (size_t)y0, (size_t)x0), dpos = make_cudaPos(0, (size_t)r2, (size_t)r1);
      if (to_device) {
        p.srcPtr = hp;
        p.srcPos = hpos;
        p.dstPtr = dp;
        p.dstPos = dpos;
        p.kind = cudaMemcpyHostToDevice;
      } else {
        p.srcPtr = dp;
        p.srcPos = dpos;
        p.dstPtr = hp;
        p.dstPos = hpos;
        p.kind = cudaMemcpyDeviceToHost;
      }
      p.extent = make_cudaExtent((size_t)g.nkz * e, (size_t)ny, (size_t)nx);
      cudaError_t err = cudaMemcpy3DAsync(&p, c->st);
      if (err != cudaSuccess) return err;
      r2 += ny;
    }
    r1 += nx;
  }
  return cudaSuccess;
}

}  // namespace

int tg_field_download_stored(tg_ctx* c, int field, double* host, size_t n) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c || !host || field < 0 || field >= TG_NFIELDS) return TG_ERR_ARG;
  if (n != 2 * (size_t)c->D) return set_err(c, TG_ERR_ARG, "download: n_doubles must be 2*N1*N2*(N3/2+1)");
  const int si = field_state_index(c, field);
  if (si < 0) return set_err(c, TG_ERR_ARG, "download_stored: state fields only");
  cudaSetDevice(c->dev);
  TG_CK(copy_stored(c, c->U0[si], host, false));
  TG_SYNC(c, __func__);
  return TG_OK;
}

int tg_field_upload(tg_ctx* c, int field, const double* host, size_t n) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c || !host || field < 0 || field >= TG_NFIELDS) return TG_ERR_ARG;
  if (n != 2 * (size_t)c->D) return set_err(c, TG_ERR_ARG, "upload: n_doubles must be 2*N1*N2*(N3/2+1)");
  cudaSetDevice(c->dev);
  const int si = field_state_index(c, field);
  const int ni = field_nl_index(c, field);
  if (field >= TG_WORK0 && field < TG_WORK0 + TG_NWORK) {
    int rc = ensure_dense(c, field);
    if (rc) return rc;
    TG_CK(cudaMemcpyAsync(c->dense[field], host, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
    TG_SYNC(c, __func__);
    return TG_OK;
  }
  if (si >= 0) {
    // state fields: only the stored modes cross the bus, straight into the compact rows
    TG_CK(copy_stored(c, c->U0[si], const_cast<double*>(host), true));
    TG_SYNC(c, __func__);
    c->energy_valid = false;
    c->have_nlin = c->have_pressure = c->have_force = false;
    return TG_OK;
  }
  cx<double>* target = nullptr;
  if (ni >= 0) target = c->NL[ni];
  else if (field == TG_PRESSURE) target = c->PR;
  else return set_err(c, TG_ERR_ARG, "upload: field not stored by this context");
  int rc = ensure_staging(c);
  if (rc) return rc;
  TG_CK(cudaMemcpyAsync(c->staging, host, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
  TG_CK(launch_dense_to_compact(c->g, c->staging, target, 0, c->st));
  TG_SYNC(c, __func__);
  if (si >= 0) {
    c->energy_valid = false;
    c->have_nlin = c->have_pressure = c->have_force = false;
  }
  return TG_OK;
}

int tg_field_download(tg_ctx* c, int field, double* host, size_t n) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c || !host || field < 0 || field >= TG_NFIELDS) return TG_ERR_ARG;
  if (n != 2 * (size_t)c->D) return set_err(c, TG_ERR_ARG, "download: n_doubles must be 2*N1*N2*(N3/2+1)");
  cudaSetDevice(c->dev);
  if (field >= TG_WORK0 && field < TG_WORK0 + TG_NWORK) {
    if (!c->dense[field]) return set_err(c, TG_ERR_STATE, "download: work field never written");
    TG_CK(cudaMemcpyAsync(host, c->dense[field], sizeof(double) * n, cudaMemcpyDeviceToHost, c->st));
    TG_SYNC(c, __func__);
    return TG_OK;
  }
  if (field >= TG_FORCE1 && field <= TG_FORCE3) {
    std::memset(host, 0, sizeof(double) * n);
    if (c->coriolis && c->have_force) {
      // Force = V x Omega of the current velocity
      std::vector<double> v[3];
      for (int i = 0; i < 3; ++i) {
        v[i].resize(n);
        int rc = tg_field_download(c, TG_V1 + i, v[i].data(), n);
        if (rc) return rc;
      }
      const int a = (field - TG_FORCE1 + 1) % 3, b = (field - TG_FORCE1 + 2) % 3;
      for (size_t q = 0; q < n; ++q) host[q] = c->om[a] * v[b][q] - c->om[b] * v[a][q];
      return TG_OK;
    }
    if (c->lm && c->have_force) {
      // Force = -(B0 . K)^2/K^2 V of the current velocity
      int rc = tg_field_download(c, TG_V1 + (field - TG_FORCE1), host, n);
      if (rc) return rc;
      for (int l1 = 0; l1 < c->N1; ++l1)
        for (int l2 = 0; l2 < c->N2; ++l2)
          for (int l3 = 0; l3 < c->M3; ++l3) {
            const double kx = (l1 <= c->N1 / 2 ? l1 : l1 - c->N1) * c->cfg.kfactor[0];
            const double ky = (l2 <= c->N2 / 2 ? l2 : l2 - c->N2) * c->cfg.kfactor[1];
            const double kz = l3 * c->cfg.kfactor[2];
            const double K2 = kx * kx + ky * ky + kz * kz, bk = c->b0[0] * kx + c->b0[1] * ky + c->b0[2] * kz;
            const double f = K2 > 0 ? -bk * bk / K2 : 0.0;
            const size_t o = (((size_t)l1 * c->N2 + l2) * c->M3 + l3) * 2;
            host[o] *= f;
            host[o + 1] *= f;
          }
      return TG_OK;
    }
    if (!c->force_on || !c->FB || (c->force_on == 1 && !c->have_force)) return TG_OK;
    std::vector<cx<double>> box((size_t)c->fbox);
    const int comp = field - TG_FORCE1;
    TG_CK(cudaMemcpyAsync(box.data(), c->FB + (size_t)comp * c->fbox, sizeof(cx<double>) * c->fbox,
                          cudaMemcpyDeviceToHost, c->st));
    TG_SYNC(c, __func__);
    const int ny = 2 * c->fy + 1, nz = c->fz + 1;
    for (int p = 0; p < c->fbox; ++p) {
      const int kz = p % nz, ky = (p / nz) % ny - c->fy, kx = p / (nz * ny) - c->fx;
      if (c->basis == TG_SCFT && kx < 0) continue;  // SCFT: kx >= 0
      const int lx = kx >= 0 ? kx : kx + c->N1, ly = ky >= 0 ? ky : ky + c->N2;
      if (lx < 0 || lx >= c->N1 || ly < 0 || ly >= c->N2 || kz >= c->M3) continue;
      const size_t o = (((size_t)lx * c->N2 + ly) * c->M3 + kz) * 2;
      host[o] = box[p].x;
      host[o + 1] = box[p].y;
    }
    return TG_OK;
  }
  const void* src = nullptr;
  int sp = 0;
  const int si = field_state_index(c, field);
  const int ni = field_nl_index(c, field);
  if (si >= 0) src = c->U0[si];
  else if (ni >= 0) src = c->NL[ni];
  else if (field == TG_PRESSURE) src = c->PR;
  else return set_err(c, TG_ERR_ARG, "download: field not stored by this context");
  int rc = ensure_staging(c);
  if (rc) return rc;
  TG_CK(launch_compact_to_dense(c->g, src, sp, c->staging, c->st));
  TG_CK(cudaMemcpyAsync(host, c->staging, sizeof(double) * n, cudaMemcpyDeviceToHost, c->st));
  TG_SYNC(c, __func__);
  return TG_OK;
}

int tg_field_alloc(tg_ctx* c, int* field) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c || !field) return TG_ERR_ARG;
  *field = -1;
  cudaSetDevice(c->dev);
  for (int i = 0; i < TG_NWORK; ++i) {
    if (c->work_reserved[i]) continue;
    const int f = TG_WORK0 + i;
    int rc = ensure_dense(c, f);  // zeroed by dalloc when new
    if (rc) return rc;
    TG_CK(cudaMemsetAsync(c->dense[f], 0, sizeof(cx<double>) * (size_t)c->D, c->st));
    c->work_reserved[i] = true;
    *field = f;
    return TG_OK;
  }
  return set_err(c, TG_ERR_BUSY, "all work fields are reserved");
}

int tg_field_free(tg_ctx* c, int field) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c || field < TG_WORK0 || field >= TG_WORK0 + TG_NWORK) return TG_ERR_ARG;
  const int i = field - TG_WORK0;
  if (!c->work_reserved[i]) return set_err(c, TG_ERR_STATE, "free: work field not reserved");
  cudaSetDevice(c->dev);
  TG_SYNC(c, __func__);
  if (c->dense[field]) {
    cudaFree(c->dense[field]);
    c->bytes -= sizeof(cx<double>) * (size_t)c->D;
    c->dense[field] = nullptr;
  }
  c->work_reserved[i] = false;
  return TG_OK;
}

int tg_field_copy(tg_ctx* c, int dst, int src) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c || dst < 0 || dst >= TG_NFIELDS || src < 0 || src >= TG_NFIELDS) return TG_ERR_ARG;
  cudaSetDevice(c->dev);
  const bool dwork = dst >= TG_WORK0 && dst < TG_WORK0 + TG_NWORK;
  const bool swork = src >= TG_WORK0 && src < TG_WORK0 + TG_NWORK;
  auto compact_of = [&](int f) -> cx<double>* {
    int si = field_state_index(c, f), ni = field_nl_index(c, f);
    if (si >= 0) return c->U0[si];
    if (ni >= 0) return c->NL[ni];
    if (f == TG_PRESSURE) return c->PR;
    return nullptr;
  };
  if (dwork) {
    int rc = ensure_dense(c, dst);
    if (rc) return rc;
    if (swork) {
      if (!c->dense[src]) return set_err(c, TG_ERR_STATE, "copy: source work field never written");
      TG_CK(cudaMemcpyAsync(c->dense[dst], c->dense[src], sizeof(cx<double>) * c->D, cudaMemcpyDeviceToDevice, c->st));
    } else {
      cx<double>* s = compact_of(src);
      if (!s) return TG_ERR_ARG;
      TG_CK(launch_compact_to_dense(c->g, s, 0, c->dense[dst], c->st));
    }
    return TG_OK;
  }
  cx<double>* d = compact_of(dst);
  if (!d) return TG_ERR_ARG;
  if (swork) {
    if (!c->dense[src]) return set_err(c, TG_ERR_STATE, "copy: source work field never written");
    TG_CK(launch_dense_to_compact(c->g, c->dense[src], d, 0, c->st));
  } else {
    cx<double>* s = compact_of(src);
    if (!s) return TG_ERR_ARG;
    TG_CK(cudaMemcpyAsync(d, s, sizeof(cx<double>) * c->S, cudaMemcpyDeviceToDevice, c->st));
  }
  if (field_state_index(c, dst) >= 0) {
    c->energy_valid = false;
    c->have_nlin = c->have_pressure = c->have_force = false;
  }
  return TG_OK;
}

int tg_forward_transform(tg_ctx* c, int field, int parity) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c || field < TG_WORK0 || field >= TG_WORK0 + TG_NWORK) return TG_ERR_ARG;
  cudaSetDevice(c->dev);
  if (!c->dense[field]) return set_err(c, TG_ERR_STATE, "transform: work field never written");
  if (c->basis == TG_SCFT && parity != 0 && parity != 1) return TG_ERR_ARG;
  return dense_transform(c, c->dense[field], 1, parity);
}

int tg_inverse_transform(tg_ctx* c, int field, int parity) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c || field < TG_WORK0 || field >= TG_WORK0 + TG_NWORK) return TG_ERR_ARG;
  cudaSetDevice(c->dev);
  if (!c->dense[field]) return set_err(c, TG_ERR_STATE, "transform: work field never written");
  if (c->basis == TG_SCFT && parity != 0 && parity != 1) return TG_ERR_ARG;
  return dense_transform(c, c->dense[field], 0, parity);
}

int tg_compute_force(tg_ctx* c) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c) return TG_ERR_ARG;
  cudaSetDevice(c->dev);
  if (c->force_on) {
    const void* in[6];
    for (int i = 0; i < c->nstate; ++i) in[i] = c->U0[i];
    int rc = run_force(c, in, F64);
    if (rc) return rc;
  }
  c->have_force = true;
  return TG_OK;
}

int tg_set_force_modes(tg_ctx* c, int n, const int* k, const double* F) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c || n < 0 || (n > 0 && (!k || !F))) return TG_ERR_ARG;
  if (c->cfg.force_kind != TG_FORCE_MODES) return set_err(c, TG_ERR_STATE, "set_force_modes: force_kind is not TG_FORCE_MODES");
  cudaSetDevice(c->dev);
  const int ns = c->nstate, K = TG_FORCE_MODES_KMAX;
  int fx = 0, fy = 0, fz = 0;
  for (int i = 0; i < n; ++i) {
    const int kx = k[3 * i], ky = k[3 * i + 1], kz = k[3 * i + 2];
    if (std::abs(kx) > K || std::abs(ky) > K || kz < 0 || kz > K)
      return set_err(c, TG_ERR_ARG, "set_force_modes: wavenumber out of range");
    // the mode must be one the context stores, named by the wavenumber the kernels see for it
    const int lx = c->basis == TG_FOUR ? (kx >= 0 ? kx : kx + c->N1) : kx;
    const int ly = ky >= 0 ? ky : ky + c->N2;
    const int r1 = (lx >= 0 && lx < c->N1) ? amap_row(c->g.ax, lx) : -1;
    const int r2 = (ly >= 0 && ly < c->N2) ? amap_row(c->g.ay, ly) : -1;
    if (r1 < 0 || r2 < 0 || geo_kx(c->g, r1) != kx || geo_ky(c->g, r2) != ky || kz >= c->g.nkz)
      return set_err(c, TG_ERR_ARG, "set_force_modes: mode (" + std::to_string(kx) + "," + std::to_string(ky) + "," +
                                        std::to_string(kz) + ") is not stored");
    for (int q = 0; q < 2 * ns; ++q)
      if (!std::isfinite(F[(size_t)2 * ns * i + q])) return set_err(c, TG_ERR_ARG, "set_force_modes: force not finite");
    fx = std::max(fx, std::abs(kx));
    fy = std::max(fy, std::abs(ky));
    fz = std::max(fz, kz);
  }
  const int ny = 2 * fy + 1, nz = fz + 1, box = n > 0 ? (2 * fx + 1) * ny * nz : 0;
  std::vector<cx<double>> h((size_t)ns * box);
  for (int i = 0; i < n; ++i) {
    const int p = ((k[3 * i] + fx) * ny + (k[3 * i + 1] + fy)) * nz + k[3 * i + 2];
    for (int q = 0; q < ns; ++q) {
      h[(size_t)q * box + p].x = F[(size_t)2 * ns * i + 2 * q];
      h[(size_t)q * box + p].y = F[(size_t)2 * ns * i + 2 * q + 1];
    }
  }
  TG_SYNC(c, __func__);
  // a captured step reads the box's address and extents
  if (c->step_graph) {
    cudaGraphExecDestroy(c->step_graph);
    c->step_graph = nullptr;
  }
  if (c->FB && box != c->fbox) {
    TG_CK(cudaFree(c->FB));
    c->bytes -= sizeof(cx<double>) * (size_t)ns * c->fbox;
    c->FB = nullptr;
  }
  c->fx = fx;
  c->fy = fy;
  c->fz = fz;
  c->fbox = box;
  if (box > 0) {
    if (!c->FB) {
      int rc = dalloc(c, (void**)&c->FB, sizeof(cx<double>) * (size_t)ns * box);
      if (rc) return rc;
    }
    TG_CK(cudaMemcpyAsync(c->FB, h.data(), sizeof(cx<double>) * h.size(), cudaMemcpyHostToDevice, c->st));
    TG_SYNC(c, __func__);
  }
  c->force_ever = true;
  return TG_OK;
}

int tg_compute_nlin(tg_ctx* c) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c) return TG_ERR_ARG;
  cudaSetDevice(c->dev);
  const void* in[6];
  for (int i = 0; i < c->nstate; ++i) in[i] = c->U0[i];
  int rc = run_pipeline(c, in, F64);
  if (rc) return rc;
  TG_CK(launch_assemble_nlin(c->g, c->phys, c->tprec, (const void* const*)c->PX, c->NL, c->st));
  c->have_nlin = true;
  c->have_pressure = false;
  return TG_OK;
}

int tg_add_force(tg_ctx* c) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c) return TG_ERR_ARG;
  if (!c->have_nlin) return set_err(c, TG_ERR_STATE, "Add_force before Compute_nlin");
  cudaSetDevice(c->dev);
  if ((c->force_on || c->coriolis || c->lm) && !c->have_force)
    return set_err(c, TG_ERR_STATE, "Add_force before Compute_force");
  if (c->force_on && c->FB) TG_CK(launch_sub_force_box(c->g, c->nstate, c->FB, c->fx, c->fy, c->fz, c->NL, c->st));
  if (c->coriolis) {
    const cx<double>* U[3] = {c->U0[0], c->U0[1], c->U0[2]};
    TG_CK(launch_sub_coriolis(c->g, c->NL, U, c->om, c->st));
  }
  if (c->lm) {
    const cx<double>* U[3] = {c->U0[0], c->U0[1], c->U0[2]};
    TG_CK(launch_sub_liquid_metal(c->g, c->NL, U, c->b0, c->st));
  }
  if (c->phys == TG_RB) {
    TG_CK(launch_rb_sub_force(c->g, c->NL, c->U0[0], c->U0[3], c->rb_fu, c->rb_ft, c->st));
  }
  return TG_OK;
}

int tg_compute_pressure(tg_ctx* c) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c) return TG_ERR_ARG;
  if (!c->have_nlin) return set_err(c, TG_ERR_STATE, "Compute_pressure before Compute_nlin");
  cudaSetDevice(c->dev);
  TG_CK(launch_pressure(c->g, c->NL, c->PR, c->st));
  c->have_pressure = true;
  return TG_OK;
}

int tg_compute_rhs(tg_ctx* c) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c) return TG_ERR_ARG;
  if (!c->have_nlin || !c->have_pressure) return set_err(c, TG_ERR_STATE, "Compute_rhs before Compute_pressure");
  cudaSetDevice(c->dev);
  TG_CK(launch_rhs_from_nlin(c->g, c->phys, c->NL, c->PR, c->st));
  return TG_OK;
}

int tg_get_dt(tg_ctx* c, double* dt) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c) return TG_ERR_ARG;
  cudaSetDevice(c->dev);
  int rc = run_energy(c, 2);
  if (rc) return rc;
  c->energy_valid = true;
  if (dt) {
    TG_CK(cudaMemcpyAsync(c->h_pinned, c->scal, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    TG_SYNC(c, __func__);
    *dt = c->h_pinned[0];
  }
  return TG_OK;
}

int tg_time_advance(tg_ctx* c) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c) return TG_ERR_ARG;
  if (!c->have_nlin || !c->have_pressure) return set_err(c, TG_ERR_STATE, "Time_advance needs Compute_nlin and Compute_pressure");
  cudaSetDevice(c->dev);
  int rc = ensure_dt(c);
  if (rc) return rc;
  // the scheme's first stage from the caller's nlin and pressure (Compute_rhs inside
  // Time_advance), then the rest of the step
  TG_CK(launch_rhs_from_nlin(c->g, c->phys, c->NL, c->PR, c->st));
  int st[4];
  const int nst = scheme_stages(c->cfg.scheme, st);
  RKArgs a = rk_args(c, st[0]);
  TG_CK(launch_rk(a, c->phys, c->tprec, c->tprec, 1, c->st, nullptr));
  if (nst == 1) {
    rc = run_finalize(c, 1, false);
  } else {
    rc = run_stages(c, 2, false);
  }
  if (rc) return rc;
  c->have_nlin = c->have_pressure = c->have_force = false;
  return TG_OK;
}

int tg_step(tg_ctx* c, int n, double* energies) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c || n < 0) return TG_ERR_ARG;
  if (n == 0) return TG_OK;
  cudaSetDevice(c->dev);
  int rc = ensure_dt(c);
  if (rc) return rc;
  int done = 0;
  while (done < n) {
    const int chunk = std::min(n - done, c->ering_cap);
    TG_CK(cudaMemsetAsync(c->ering_pos, 0, sizeof(int), c->st));
    for (int i = 0; i < chunk; ++i) {
      if (c->graphs && !c->prof && c->eager_steps >= 1) {
        if (!c->step_graph) {
          cudaGraph_t gr = nullptr;
          TG_CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
          rc = enqueue_step(c, true);
          cudaError_t e2 = cudaStreamEndCapture(c->st, &gr);
          if (rc) {
            if (gr) cudaGraphDestroy(gr);
            return rc;
          }
          if (e2 != cudaSuccess) return cuda_err(c, e2, "cudaStreamEndCapture");
          cudaError_t e3 = cudaGraphInstantiate(&c->step_graph, gr, 0);
          cudaGraphDestroy(gr);
          if (e3 != cudaSuccess) return cuda_err(c, e3, "cudaGraphInstantiate");
        }
        TG_CK(cudaGraphLaunch(c->step_graph, c->st));
      } else {
        rc = enqueue_step(c, true);
        if (rc) return rc;
        c->eager_steps++;
      }
    }
    if (energies) {
      TG_CK(cudaMemcpyAsync(energies + done, c->ering, sizeof(double) * chunk, cudaMemcpyDeviceToHost, c->st));
    }
    TG_CK(cudaMemcpyAsync(c->h_pinned, c->scal, sizeof(double) * 8, cudaMemcpyDeviceToHost, c->st));
    TG_SYNC(c, __func__);
    done += chunk;
    if (c->h_pinned[3] != 0.0) return set_err(c, TG_ERR_NONFINITE, "ERROR: Numerical Overflow (total energy is not finite)");
  }
  c->have_nlin = c->have_pressure = c->have_force = false;
  return TG_OK;
}

int tg_time(const tg_ctx* c, double* t, long long* steps) {
  if (!c) return TG_ERR_ARG;
  double h[8];
  tg_ctx* cc = const_cast<tg_ctx*>(c);
  cudaSetDevice(c->dev);
  cudaError_t e = cudaMemcpyAsync(h, c->scal, sizeof(h), cudaMemcpyDeviceToHost, c->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
  if (e != cudaSuccess) return cuda_err(cc, e, "tg_time");
  if (t) *t = h[1];
  if (steps) *steps = (long long)h[2];
  return TG_OK;
}

int tg_energy(tg_ctx* c, int group, double* energy, double* diss) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c) return TG_ERR_ARG;
  if (group < 0 || group > 2) return TG_ERR_ARG;
  if (group == 1 && c->phys != TG_MHD) return TG_ERR_ARG;
  if (group == 2 && c->phys != TG_SCALAR && c->phys != TG_RB) return TG_ERR_ARG;
  cudaSetDevice(c->dev);
  int rc = run_energy(c, 0);
  if (rc) return rc;
  TG_CK(cudaMemcpyAsync(c->h_pinned, c->red_out, sizeof(double) * 8, cudaMemcpyDeviceToHost, c->st));
  TG_SYNC(c, __func__);
  const int s = group * 2;
  // CV_total_energy and CV_total_dissipation = 2 sum mult K^2 |u|^2 (Cvf.cc:385-397)
  if (energy) *energy = c->h_pinned[s];
  if (diss) *diss = 2.0 * c->h_pinned[s + 1];
  return TG_OK;
}

int tg_shell_spectrum(tg_ctx* c, int group, double* ek, double* dissk, int n) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c || !ek) return TG_ERR_ARG;
  if (group < 0 || group > 2) return TG_ERR_ARG;
  if (group == 1 && c->phys != TG_MHD) return TG_ERR_ARG;
  if (group == 2 && c->phys != TG_SCALAR && c->phys != TG_RB) return TG_ERR_ARG;
  cudaSetDevice(c->dev);
  // Min_radius_outside / Max_radius_inside (four_inline.h:172-257)
  const int d = c->cfg.dealias ? 3 : 2;
  const double* kf = c->cfg.kfactor;
  // SCFT: kx extent 2 N1/3 dealiased, N1 - 1 aliased (scft_inline.h:144-200)
  const int nx = (c->basis == TG_FOUR) ? c->N1 / d : (c->cfg.dealias ? 2 * c->N1 / 3 : c->N1 - 1);
  const double a0 = nx * kf[0], a1 = (c->N2 / d) * kf[1], a2 = (c->N3 / d) * kf[2];
  const int kkmax = (int)std::ceil(std::sqrt(a0 * a0 + a1 * a1 + a2 * a2));
  const int kin = max_radius_inside(c);
  const int nbins = kkmax + 1;
  if (n < nbins) return set_err(c, TG_ERR_ARG, "shell spectrum: n < kmax_outside + 1");
  const int nf = (group == 2) ? 1 : 3;
  const cx<double>* F[3];
  for (int i = 0; i < nf; ++i) F[i] = c->U0[(group == 0 ? 0 : 3) + i];
  // scratch: [nf*nbins] ek, [nbins] cnt, [nbins] diss, [nbins] cnt2, then the kernels' block sums
  const size_t need = (size_t)(nf + 3) * nbins;
  const size_t part_n = (size_t)shell_spectrum_blocks(c->g) * (nf + 1) * nbins;
  if (c->diag_cap < need + part_n) {
    if (c->diag) {
      cudaFree(c->diag);
      c->bytes -= sizeof(double) * c->diag_cap;
    }
    c->diag = nullptr;
    c->diag_cap = 0;
    int rc = dalloc(c, (void**)&c->diag, sizeof(double) * (need + part_n));
    if (rc) return rc;
    c->diag_cap = need + part_n;
  }
  double* dbuf = c->diag;
  double* part = c->diag + need;
  TG_CK(cudaMemsetAsync(dbuf, 0, sizeof(double) * need, c->st));
  TG_CK(launch_shell_spectrum(c->g, F, nf, 0.0, dbuf, dbuf + (size_t)nf * nbins, nbins, part, c->st));
  // dissipation spectrum: sum over components of K^2-weighted, times 2 (Cvf.cc:430-448)
  double* dk = dbuf + (size_t)(nf + 1) * nbins;
  double* dcnt = dk + nbins;
  {
    // accumulate all components into one row by summing separate passes
    for (int i = 0; i < nf; ++i) {
      const cx<double>* Fi[1] = {F[i]};
      TG_CK(launch_shell_spectrum(c->g, Fi, 1, 2.0, dk, dcnt, nbins, part, c->st));
    }
  }
  std::vector<double> h(need);
  TG_CK(cudaMemcpyAsync(h.data(), dbuf, sizeof(double) * need, cudaMemcpyDeviceToHost, c->st));
  TG_SYNC(c, __func__);
  // Sk_count of the reference runs over every mode of its dense array, the dealiased zeros
  // included (four_energy.cc:271-286, scft_energy.cc:266-281): geometry only, computed once
  if ((int)c->shell_count.size() != nbins) {
    c->shell_count.assign(nbins, 0.0);
    for (int l1 = 0; l1 < c->N1; ++l1) {
      const int kxi = (c->basis == TG_FOUR && l1 > c->N1 / 2) ? l1 - c->N1 : l1;
      for (int l2 = 0; l2 < c->N2; ++l2) {
        const int kyi = l2 <= c->N2 / 2 ? l2 : l2 - c->N2;
        for (int l3 = 0; l3 < c->M3; ++l3) {
          const double kx = kxi * kf[0], ky = kyi * kf[1], kz = l3 * kf[2];
          const int b = (int)std::ceil(std::sqrt(kx * kx + ky * ky + kz * kz));
          if (b >= nbins) continue;
          c->shell_count[b] += (c->basis == TG_FOUR) ? mult_four(l1, l2, l3, c->N1, c->N2)
                                                     : 0.5 * mult_scft(l1, l2, l3, c->N2);
        }
      }
    }
  }
  const double* cnt = c->shell_count.data();
  // Approx_number_modes_in_shell: FOUR hemisphere 2 pi r^2, SCFT quarter sphere pi r^2
  const double approx_fac = (c->basis == TG_FOUR ? 2 * M_PI : M_PI) / (kf[0] * kf[1] * kf[2]);
  for (int i = 0; i < nf; ++i)
    for (int b = 0; b < n; ++b) ek[(size_t)i * n + b] = 0.0;
  if (dissk)
    for (int b = 0; b < n; ++b) dissk[b] = 0.0;
  for (int b = 0; b < nbins; ++b) {
    // partial shells (kmax_inside, kmax] rescaled (four_energy.cc:324-336)
    const bool resc = (b > kin) && (cnt[b] >= 1);
    const double f = resc ? approx_fac * b * b / cnt[b] : 1.0;
    for (int i = 0; i < nf; ++i) ek[(size_t)i * n + b] = h[(size_t)i * nbins + b] * f;
    if (dissk) dissk[b] = 2.0 * h[(size_t)(nf + 1) * nbins + b] * f;
  }
  return TG_OK;
}

int tg_profile_enable(tg_ctx* c, int enable) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c) return TG_ERR_ARG;
  c->prof = enable != 0;
  return TG_OK;
}

int tg_profile_read(tg_ctx* c, tg_kernel_stat* out, int max, int* n) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c || (max > 0 && !out)) return TG_ERR_ARG;
  cudaSetDevice(c->dev);
  TG_SYNC(c, __func__);
  std::vector<tg_kernel_stat> agg;
  for (auto& r : c->prof_recs) {
    float ms = 0;
    cudaEventElapsedTime(&ms, r.a, r.b);
    size_t k = 0;
    for (; k < agg.size(); ++k)
      if (std::strncmp(agg[k].name, r.name, sizeof(agg[k].name)) == 0) break;
    if (k == agg.size()) {
      tg_kernel_stat st{};
      std::strncpy(st.name, r.name, sizeof(st.name) - 1);
      agg.push_back(st);
    }
    agg[k].launches += 1;
    agg[k].total_ms += ms;
    agg[k].bytes_per_launch += r.bytes;
    c->ev_pool.push_back(r.a);
    c->ev_pool.push_back(r.b);
  }
  c->prof_recs.clear();
  for (auto& a : agg)
    if (a.launches) a.bytes_per_launch /= a.launches;
  const int m = std::min<int>(max, (int)agg.size());
  for (int i = 0; i < m; ++i) out[i] = agg[i];
  if (n) *n = (int)agg.size();
  return TG_OK;
}

int tg_nusselt(tg_ctx* c, double* nu) {
  if (c && c->slab_W) return slab_refuse(c);
  if (!c || !nu) return TG_ERR_ARG;
  if (c->phys != TG_RB) return set_err(c, TG_ERR_ARG, "Nusselt number needs the RB physics");
  cudaSetDevice(c->dev);
  // Get_Nusselt_no (nusselt.cc:53-89), PRLARGE + ULARGE: 1 + 2 sqrt(Ra Pr) <u1, theta>
  int nb = 0;
  TG_CK(launch_cross_partials(c->g, c->U0[0], c->U0[3], c->part, 0, 8, c->st, &nb));
  std::vector<double> h((size_t)nb * 8);
  TG_CK(cudaMemcpyAsync(h.data(), c->part, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->st));
  TG_SYNC(c, __func__);
  double cross = 0;
  for (int b = 0; b < nb; ++b) cross += h[(size_t)b * 8];
  *nu = 1.0 + rb_coefficients(&c->cfg).nuf * cross;
  return TG_OK;
}

}  // extern "C"
