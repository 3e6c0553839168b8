// The pass sequence of a nonlinear product term on the compact layout:
//   x-inverse -> y-inverse (pipe_inverse_xy) and
//   fused z-pass (c2r, pointwise products, r2c) -> y-forward -> x-forward (pipe_products_forward).
// Used by the time step (IncVF::Compute_nlin) and by the energy-transfer diagnostics
// (IncVF::EnergyTr_Compute_nlin).
#include <algorithm>

#include "tg_ctx.h"

namespace tg {

namespace {
AxisMap full_map(int L) { return AxisMap{L, L, 0}; }
}  // namespace

cudaEvent_t prof_event(tg_ctx* c) {
  if (!c->ev_pool.empty()) {
    cudaEvent_t e = c->ev_pool.back();
    c->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

ProfScope::ProfScope(tg_ctx* c_, const char* name, double bytes) : c(c_) {
  if (!c->prof) return;
  tg_ctx::ProfRec r{name, prof_event(c), prof_event(c), bytes};
  cudaEventRecord(r.a, c->st);
  c->prof_recs.push_back(r);
  idx = (long)c->prof_recs.size() - 1;
}
ProfScope::~ProfScope() {
  if (idx >= 0) cudaEventRecord(c->prof_recs[idx].b, c->st);
}

double el_compact(const tg_ctx* c) { return (double)c->g.nkx * c->g.nky * c->g.nkz; }
double el_xstage(const tg_ctx* c) { return (double)c->N1 * c->g.nky * c->g.nkz; }
double el_ystage(const tg_ctx* c) { return (double)c->N1 * c->N2 * c->g.nkz; }

int pipe_inverse_xy(tg_ctx* c, int nf, const void* const* in, const void* const* in2, const int* comb,
                    int inprec, int nread, void* const* WX, void* const* WY) {
  if (!c->pipeline_ok) return set_err(c, TG_ERR_UNSUPPORTED, "nonlinear term needs N3/2 a power of two in [4, 256]");
  const Geo& g = c->g;
  {
    AxisLaunch l;
    wait_args(c, l.a);
    l.L = c->N1;
    l.dir = +1;
    l.pin = inprec;
    l.pout = c->tprec;
    l.pwork = c->tprec;
    l.nbatch = c->nact;
    l.nfields = nf;
    l.a.sb = g.S;  // request stride of the batch
    l.a.sr = (long long)g.nky * g.kzp;
    l.a.db = (long long)c->N1 * g.nky * g.kzp;
    l.a.dr = (long long)g.nky * g.kzp;
    l.a.ncols = g.nky * g.kzp;
    l.a.in = g.ax;
    l.a.out = full_map(c->N1);
    l.a.scale = 1.0;
    l.a.tw = c->tw[c->N1];
    for (int f = 0; f < nf; ++f) {
      l.ps.src[f] = in[f];
      l.ps.dst[f] = WX[f];
      l.a.comb[f] = comb ? comb[f] : 0;
      l.ps.src2[f] = (comb && comb[f]) ? in2[f] : nullptr;
    }
    const double insz = inprec == F64 ? 16.0 : 8.0;
    ProfScope pr(c, "x_inverse", nread * el_compact(c) * insz + nf * el_xstage(c) * c->tsz);
    cudaError_t e;
    if (c->basis == TG_SCFT) {
      // ISFT / ICFT along x (scft_tr.cc:440-639) on the stored sin/cos slots
      R2RArgs r{};
      for (int f = 0; f < nf; ++f) r.kind[f] = c->xinv_kind[f];
      r.trig = c->trigx;
      for (int k = 0; k < 4; ++k) {
        r.mat[k] = c->xmat[k];
        r.mat_rows[k] = c->xmat_rows[k];
        r.mat_cols[k] = c->xmat_cols[k];
      }
      e = launch_r2r(l, r, c->st);
    } else {
      e = launch_axis(l, c->st);
    }
    if (e != cudaSuccess) return cuda_err(c, e, "x inverse");
  }
  {
    AxisLaunch l;
    wait_args(c, l.a);
    l.L = c->N2;
    l.dir = +1;
    l.pin = l.pout = l.pwork = c->tprec;
    l.nbatch = c->nact * c->N1;
    l.nfields = nf;
    l.a.sb = (long long)g.nky * g.kzp;
    l.a.sr = g.kzp;
    l.a.db = (long long)c->N2 * g.kzp;
    l.a.dr = g.kzp;
    l.a.ncols = g.kzp;
    l.a.in = g.ay;
    l.a.out = full_map(c->N2);
    l.a.scale = 1.0;
    l.a.tw = c->tw[c->N2];
    for (int f = 0; f < nf; ++f) {
      l.ps.src[f] = WX[f];
      l.ps.dst[f] = WY[f];
    }
    ProfScope pr(c, "y_inverse", nf * (el_xstage(c) + el_ystage(c)) * c->tsz);
    cudaError_t e = launch_axis(l, c->st);
    if (e != cudaSuccess) return cuda_err(c, e, "y inverse");
  }
  return TG_OK;
}

int pipe_products_forward(tg_ctx* c, int nin, const void* const* WY, int nprod, const ProdPairs& pp,
                          void* const* PP, void* const* PY, void* const* PX, const int* xkinds) {
  if (!c->pipeline_ok) return set_err(c, TG_ERR_UNSUPPORTED, "nonlinear term needs N3/2 a power of two in [4, 256]");
  const Geo& g = c->g;
  {
    ZProdLaunch l;
    l.M = c->Mz;
    l.nin = nin;
    l.nprod = nprod;
    l.pin = l.pout = l.pwork = c->tprec;
    l.a.nrows = (long long)c->nact * c->N1 * c->N2;
    l.a.ss = g.kzp;
    l.a.ds = g.kzp;
    l.a.nin = g.nkz;
    l.a.nout = g.nkz;
    l.a.nfill = g.kzp;
    l.a.pad = 0;
    l.a.scale = 1.0 / ((double)c->N1 * c->N2 * c->N3);
    l.a.twM = c->tw[c->Mz];
    l.a.twN = c->tw[c->N3];
    l.a.oct = c->zoct;
    for (int f = 0; f < nin; ++f) l.ps.src[f] = WY[f];
    for (int q = 0; q < nprod; ++q) l.ps.dst[q] = PP[q];
    l.pp = pp;
    ProfScope pr(c, "z_products", (nin + nprod) * el_ystage(c) * c->tsz);
    cudaError_t e = launch_zprod(l, c->st);
    if (e != cudaSuccess) return cuda_err(c, e, "z products");
  }
  {
    AxisLaunch l;
    wait_args(c, l.a);
    l.L = c->N2;
    l.dir = -1;
    l.pin = l.pout = l.pwork = c->tprec;
    l.nbatch = c->nact * c->N1;
    l.nfields = nprod;
    l.a.sb = (long long)c->N2 * g.kzp;
    l.a.sr = g.kzp;
    l.a.db = (long long)g.nky * g.kzp;
    l.a.dr = g.kzp;
    l.a.ncols = g.kzp;
    l.a.in = full_map(c->N2);
    l.a.out = g.ay;
    l.a.scale = 1.0;
    l.a.tw = c->tw[c->N2];
    for (int q = 0; q < nprod; ++q) {
      l.ps.src[q] = PP[q];
      l.ps.dst[q] = PY[q];
    }
    ProfScope pr(c, "y_forward", nprod * (el_ystage(c) + el_xstage(c)) * c->tsz);
    cudaError_t e = launch_axis(l, c->st);
    if (e != cudaSuccess) return cuda_err(c, e, "y forward");
  }
  {
    AxisLaunch l;
    wait_args(c, l.a);
    l.L = c->N1;
    l.dir = -1;
    l.pin = l.pout = l.pwork = c->tprec;
    l.nbatch = c->nact;
    l.nfields = nprod;
    l.a.sb = (long long)c->N1 * g.nky * g.kzp;
    l.a.sr = (long long)g.nky * g.kzp;
    l.a.db = g.S;
    l.a.dr = (long long)g.nky * g.kzp;
    l.a.ncols = g.nky * g.kzp;
    l.a.in = full_map(c->N1);
    l.a.out = g.ax;
    l.a.scale = 1.0;
    l.a.tw = c->tw[c->N1];
    for (int q = 0; q < nprod; ++q) {
      l.ps.src[q] = PY[q];
      l.ps.dst[q] = PX[q];
    }
    ProfScope pr(c, "x_forward", nprod * (el_xstage(c) + el_compact(c)) * c->tsz);
    cudaError_t e;
    if (c->basis == TG_SCFT) {
      // SFT / CFT along x with Norm_SCFT's extra 1/2 (scft_tr.cc:89-92; the z-pass applied
      // 1/(N1 N2 N3))
      R2RArgs r{};
      for (int q = 0; q < nprod; ++q) r.kind[q] = xkinds ? xkinds[q] : c->xfwd_kind[q];
      r.trig = c->trigx;
      for (int k = 0; k < 4; ++k) {
        r.mat[k] = c->xmat[k];
        r.mat_rows[k] = c->xmat_rows[k];
        r.mat_cols[k] = c->xmat_cols[k];
      }
      l.a.scale = 0.5;
      e = launch_r2r(l, r, c->st);
    } else {
      e = launch_axis(l, c->st);
    }
    if (e != cudaSuccess) return cuda_err(c, e, "x forward");
  }
  return TG_OK;
}

}  // namespace tg
