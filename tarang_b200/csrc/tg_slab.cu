// Slab-sharded single solve: one context per rank, each holding a slab of the compact kx rows
// of the spectral state; the exchanges between the passes are the caller's (an NCCL all-to-all
// through torch.distributed, one process per GPU; or device copies between contexts that share
// one GPU).
//
// Reference: the MPI slab decomposition of basis_basicfn.cc:49-281 — local_N1 kx planes of the
// spectral arrays per rank, local_N2 y planes in real space, and an all-to-all transpose inside
// every 3-D transform (FFTW-MPI in four_tr.cc / scft_tr.cc) — with the time step of
// Ifluid_main.cc:258-301.
//
// One RHS evaluation of RK stage s (tg_slab_phase):
//   phase 0  y-inverse of the stage input's kx rows [nx][nky][kzp] -> [nx][N2][kzp], packed into
//            W chunks [nx][ny_d][kzp] (chunk d for rank d)                  -> inverse send
//   (caller) all-to-all: rank r receives chunk r of every rank s, in rank order, which is
//            [nkx][ny][kzp]: all stored kx rows of its y planes            -> inverse receive
//   phase 1  x-inverse [nkx][ny][kzp] -> [N1][ny][kzp], the fused z-pass (c2r, products, r2c) on
//            the N1 ny rows, x-forward -> [nkx][ny][kzp]; rows of rank d are chunk d -> forward send
//   (caller) all-to-all: rank r receives its kx rows of every rank's y planes -> forward receive
//   phase 2  unpack the W chunks [nx][ny_s][kzp] into [nx][N2][kzp], y-forward -> [nx][nky][kzp],
//            the RK stage kernel (nonlinear term, projection, IF-RK4 update) on the rank's modes;
//            after stage 4 the rank's energy sums -> reduction buffer
//   (caller) all-reduce (sum) of the 8 reduction values into the summed buffer
//   phase 3  Get_dt and the step count from the summed reductions (end of a step); phase 5 sets
//            dt only (before the first step, after phase 4 = the energy sums of the uploaded state)
// Every pass is the whole-grid context's kernel (the same per-row transforms), so a slab solve
// with any number of ranks gives the same fields bit for bit when dt is the fixed ceiling; the
// energies are sums in another order.
#include <cstring>
#include <vector>

#include "tg_ctx.h"

using namespace tg;

namespace {

constexpr int TPB = 256;

AxisMap full_axis(int L) { return AxisMap{L, L, 0}; }

struct ChunkMap {
  int W, nx, N2, kzp;
  int y0[TG_SLAB_MAX_RANKS], ny[TG_SLAB_MAX_RANKS];
  long long off[TG_SLAB_MAX_RANKS];  // element offset of chunk d
};

// owner of y plane y under split_range(N2, W, .)
__device__ __forceinline__ int y_owner(int y, int N2, int W) {
  const int b = N2 / W, rem = N2 % W;
  const int big = rem * (b + 1);
  return y < big ? y / (b + 1) : rem + (y - big) / b;
}

// pack (to_chunks = 1): chunked[d] [nx][ny_d][kzp] <- natural [nx][N2][kzp]; unpack (0): back
template <typename T>
__global__ void __launch_bounds__(TPB) k_slab_chunks(const T* __restrict__ src, T* __restrict__ dst, ChunkMap m,
                                                     int to_chunks) {
  const long long n = (long long)m.nx * m.N2 * m.kzp;
  const long long stride = (long long)gridDim.x * TPB;
  for (long long i = (long long)blockIdx.x * TPB + threadIdx.x; i < n; i += stride) {
    const int kz = (int)(i % m.kzp);
    const long long rr = i / m.kzp;
    const int y = (int)(rr % m.N2);
    const int kx = (int)(rr / m.N2);
    const int d = y_owner(y, m.N2, m.W);
    const long long j = m.off[d] + ((long long)kx * m.ny[d] + (y - m.y0[d])) * m.kzp + kz;
    if (to_chunks) dst[j] = src[i];
    else dst[i] = src[j];
  }
}

ChunkMap chunk_map(const tg_ctx* c) {
  ChunkMap m{};
  m.W = c->slab_W;
  m.nx = c->slab_nx[c->slab_r];
  m.N2 = c->N2;
  m.kzp = c->g.kzp;
  long long off = 0;
  for (int d = 0; d < c->slab_W; ++d) {
    m.y0[d] = c->slab_y[d];
    m.ny[d] = c->slab_ny[d];
    m.off[d] = off;
    off += (long long)m.nx * m.ny[d] * m.kzp;
  }
  return m;
}

cudaError_t launch_chunks(const tg_ctx* c, const void* src, void* dst, int to_chunks) {
  const ChunkMap m = chunk_map(c);
  const long long n = (long long)m.nx * m.N2 * m.kzp;
  long long blocks = (n + TPB - 1) / TPB;
  if (blocks > 148LL * 16) blocks = 148LL * 16;
  if (blocks < 1) return cudaSuccess;
  if (c->tprec == F64)
    k_slab_chunks<cx<double>><<<(unsigned)blocks, TPB, 0, c->st>>>((const cx<double>*)src, (cx<double>*)dst, m, to_chunks);
  else
    k_slab_chunks<cx<float>><<<(unsigned)blocks, TPB, 0, c->st>>>((const cx<float>*)src, (cx<float>*)dst, m, to_chunks);
  return cudaGetLastError();
}

int slab_ok(tg_ctx* c) {
  if (!c) return TG_ERR_ARG;
  if (c->slab_W <= 0) return set_err(c, TG_ERR_STATE, "not a slab context (tg_slab_create)");
  return TG_OK;
}

// x pass over [rows_in][ny][kzp] -> [rows_out][ny][kzp] of nf fields (FOUR c2c, SCFT r2r)
int slab_xpass(tg_ctx* c, int dir, int nf, void* const* src, void* const* dst, const int* xkinds) {
  const Geo& g = c->g;
  const long long ny = c->slab_ny[c->slab_r];
  AxisLaunch l;
  wait_args(c, l.a);
  l.L = c->N1;
  l.dir = dir;
  l.pin = l.pout = l.pwork = c->tprec;
  l.nbatch = 1;
  l.nfields = nf;
  const long long col = ny * g.kzp;
  l.a.sr = col;
  l.a.dr = col;
  l.a.ncols = (int)col;
  if (dir > 0) {
    l.a.sb = (long long)g.nkx * col;
    l.a.db = (long long)c->N1 * col;
    l.a.in = g.ax;
    l.a.out = full_axis(c->N1);
  } else {
    l.a.sb = (long long)c->N1 * col;
    l.a.db = (long long)g.nkx * col;
    l.a.in = full_axis(c->N1);
    l.a.out = g.ax;
  }
  l.a.scale = 1.0;
  l.a.tw = c->tw[c->N1];
  for (int f = 0; f < nf; ++f) {
    l.ps.src[f] = src[f];
    l.ps.dst[f] = dst[f];
  }
  cudaError_t e;
  if (c->basis == TG_SCFT) {
    R2RArgs r{};
    for (int f = 0; f < nf; ++f) r.kind[f] = xkinds[f];
    r.trig = c->trigx;
    for (int k = 0; k < 4; ++k) {
      r.mat[k] = c->xmat[k];
      r.mat_rows[k] = c->xmat_rows[k];
      r.mat_cols[k] = c->xmat_cols[k];
    }
    if (dir < 0) l.a.scale = 0.5;  // Norm_SCFT's extra 1/2 (scft_tr.cc:89-92)
    e = launch_r2r(l, r, c->st);
  } else {
    e = launch_axis(l, c->st);
  }
  return e == cudaSuccess ? TG_OK : cuda_err(c, e, dir > 0 ? "slab x inverse" : "slab x forward");
}

// y pass over the rank's kx rows: inverse [nx][nky][kzp] -> [nx][N2][kzp], forward back
int slab_ypass(tg_ctx* c, int dir, int nf, int pin, const void* const* src, void* const* dst) {
  const Geo& g = c->g;
  AxisLaunch l;
  wait_args(c, l.a);
  l.L = c->N2;
  l.dir = dir;
  l.pin = pin;
  l.pout = l.pwork = c->tprec;
  l.nbatch = c->slab_nx[c->slab_r];
  l.nfields = nf;
  l.a.sr = g.kzp;
  l.a.dr = g.kzp;
  l.a.ncols = g.kzp;
  if (dir > 0) {
    l.a.sb = (long long)g.nky * g.kzp;
    l.a.db = (long long)c->N2 * g.kzp;
    l.a.in = g.ay;
    l.a.out = full_axis(c->N2);
  } else {
    l.a.sb = (long long)c->N2 * g.kzp;
    l.a.db = (long long)g.nky * g.kzp;
    l.a.in = full_axis(c->N2);
    l.a.out = g.ay;
  }
  l.a.scale = 1.0;
  l.a.tw = c->tw[c->N2];
  for (int f = 0; f < nf; ++f) {
    l.ps.src[f] = src[f];
    l.ps.dst[f] = dst[f];
  }
  const cudaError_t e = launch_axis(l, c->st);
  return e == cudaSuccess ? TG_OK : cuda_err(c, e, dir > 0 ? "slab y inverse" : "slab y forward");
}

void stage_inputs(tg_ctx* c, int stage, const void* in[6], int& inprec) {
  for (int i = 0; i < c->nstate; ++i) in[i] = stage == 1 ? (const void*)c->U0[i] : (const void*)c->US[i];
  inprec = stage == 1 ? F64 : c->tprec;
}

int phase0(tg_ctx* c, int stage) {
  const void* in[6];
  int inprec;
  stage_inputs(c, stage, in, inprec);
  int rc = slab_ypass(c, +1, c->nin, inprec, in, c->SA);
  if (rc) return rc;
  for (int f = 0; f < c->nin; ++f) {
    const cudaError_t e = launch_chunks(c, c->SA[f], c->SB[f], 1);
    if (e != cudaSuccess) return cuda_err(c, e, "slab pack");
  }
  return TG_OK;
}

int phase1(tg_ctx* c) {
  const Geo& g = c->g;
  int rc = slab_xpass(c, +1, c->nin, c->SR, c->WX, c->xinv_kind);
  if (rc) return rc;
  ZProdLaunch z;
  z.M = c->Mz;
  z.nin = c->nin;
  z.nprod = c->nprod;
  z.pin = z.pout = z.pwork = c->tprec;
  z.a.nrows = (long long)c->N1 * c->slab_ny[c->slab_r];
  z.a.ss = g.kzp;
  z.a.ds = g.kzp;
  z.a.nin = g.nkz;
  z.a.nout = g.nkz;
  z.a.nfill = g.kzp;
  z.a.pad = 0;
  z.a.scale = 1.0 / ((double)c->N1 * c->N2 * c->N3);
  z.a.twM = c->tw[c->Mz];
  z.a.twN = c->tw[c->N3];
  z.a.oct = c->zoct;
  for (int f = 0; f < c->nin; ++f) z.ps.src[f] = c->WX[f];
  for (int q = 0; q < c->nprod; ++q) z.ps.dst[q] = c->PP[q];
  z.pp = c->pairs;
  const cudaError_t e = launch_zprod(z, c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "slab z products");
  return slab_xpass(c, -1, c->nprod, c->PP, c->PY, c->xfwd_kind);
}

int phase2(tg_ctx* c, int stage) {
  for (int q = 0; q < c->nprod; ++q) {
    const cudaError_t e = launch_chunks(c, c->SB[q], c->SA[q], 0);
    if (e != cudaSuccess) return cuda_err(c, e, "slab unpack");
  }
  const void* sa[9];
  for (int q = 0; q < c->nprod; ++q) sa[q] = c->SA[q];
  int rc = slab_ypass(c, -1, c->nprod, c->tprec, sa, c->PX);
  if (rc) return rc;
  const void* in[6];
  int inprec;
  stage_inputs(c, stage, in, inprec);
  RKArgs a = rk_args(c, stage);
  for (int i = 0; i < c->nstate; ++i) a.IN[i] = in[i];
  a.inprec = (inprec == F64) ? 0 : 1;
  TG_CK(launch_rk(a, c->phys, c->tprec, c->tprec, 0, c->st, nullptr));
  // after stage 4: this rank's energy sums (no dt yet: that needs every rank's sums)
  if (stage == 4) return run_finalize(c, 0, false);
  return TG_OK;
}

// Get_dt from the reductions summed over the ranks (c->gsum): dt_mode 1 also advances t and the
// step count (the end of a step), 2 sets dt only
int phase_global(tg_ctx* c, int dt_mode) {
  FinalizeArgs f{};
  f.part = c->gsum;
  f.nblocks = 1;
  f.nslots = 8;
  f.out = c->red_out;
  f.scal = c->scal;
  f.ering = nullptr;
  f.ering_pos = c->ering_pos;
  f.dt_mode = dt_mode;
  f.dx = c->dx_cfl;
  f.Tdt = c->cfg.dt;
  f.mhd = 0;
  f.nact = 1;
  f.S = c->S;
  TG_CK(launch_finalize(f, c->st));
  return TG_OK;
}

}  // namespace

namespace tg {
int slab_refuse(tg_ctx* c) {
  return set_err(c, TG_ERR_STATE, "a slab context answers the tg_slab_* calls only");
}
}  // namespace tg

extern "C" {

int tg_slab_create(const tg_config* cfg, int world, int rank, tg_ctx** out) {
  if (!cfg || !out || world < 1 || world > TG_SLAB_MAX_RANKS || rank < 0 || rank >= world) return TG_ERR_ARG;
  // slabs cover the equations whose forces are local in K (none, convection's buoyancy, the
  // Coriolis and liquid-metal forces, fixed modes); the band forcings need band sums over all
  // ranks and MHD's Get_dt the mean field of rank 0: not built for slabs
  if (cfg->physics == TG_MHD || cfg->force_kind == TG_FORCE_ENERGY_SUPPLY ||
      cfg->force_kind == TG_FORCE_ENERGY_HELICITY)
    return TG_ERR_UNSUPPORTED;
  // the phases run the four RK4 stages (tg_slab_phase stage 1..4)
  if (cfg->scheme != TG_RK4) return TG_ERR_UNSUPPORTED;
  const int Mz = cfg->N[2] / 2;
  if (Mz < 4 || Mz > 256 || (Mz & (Mz - 1))) return TG_ERR_UNSUPPORTED;
  return ctx_create_batch(cfg, 1, out, world, rank);
}

int tg_slab_info_get(const tg_ctx* c, tg_slab_info* info) {
  if (!c || !info || c->slab_W <= 0) return TG_ERR_ARG;
  std::memset(info, 0, sizeof(*info));
  info->world = c->slab_W;
  info->rank = c->slab_r;
  info->x0 = c->slab_x[c->slab_r];
  info->nx = c->slab_nx[c->slab_r];
  info->y0 = c->slab_y[c->slab_r];
  info->ny = c->slab_ny[c->slab_r];
  for (int d = 0; d < c->slab_W; ++d) {
    info->xs[d] = c->slab_x[d];
    info->xn[d] = c->slab_nx[d];
    info->ys[d] = c->slab_y[d];
    info->yn[d] = c->slab_ny[d];
  }
  info->nkx = c->g.nkx;
  info->nky = c->g.nky;
  info->nkz = c->g.nkz;
  info->kzp = c->g.kzp;
  info->nin = c->nin;
  info->nprod = c->nprod;
  info->elem_bytes = c->tsz;
  return TG_OK;
}

int tg_slab_buffer(tg_ctx* c, int which, int field, void** ptr) {
  int rc = slab_ok(c);
  if (rc) return rc;
  if (!ptr) return TG_ERR_ARG;
  *ptr = nullptr;
  switch (which) {
    case TG_SLAB_INV_SEND:
      if (field < 0 || field >= c->nin) return TG_ERR_ARG;
      *ptr = c->SB[field];
      break;
    case TG_SLAB_INV_RECV:
      if (field < 0 || field >= c->nin) return TG_ERR_ARG;
      *ptr = c->SR[field];
      break;
    case TG_SLAB_FWD_SEND:
      if (field < 0 || field >= c->nprod) return TG_ERR_ARG;
      *ptr = c->PY[field];
      break;
    case TG_SLAB_FWD_RECV:
      if (field < 0 || field >= c->nprod) return TG_ERR_ARG;
      *ptr = c->SB[field];
      break;
    case TG_SLAB_SUMS:
      *ptr = c->red_out;
      break;
    case TG_SLAB_GLOBAL_SUMS:
      *ptr = c->gsum;
      break;
    default:
      return TG_ERR_ARG;
  }
  return TG_OK;
}

int tg_slab_phase(tg_ctx* c, int phase, int stage) {
  int rc = slab_ok(c);
  if (rc) return rc;
  if ((phase == 0 || phase == 2) && (stage < 1 || stage > 4)) return TG_ERR_ARG;
  cudaSetDevice(c->dev);
  switch (phase) {
    case 0: return phase0(c, stage);
    case 1: return phase1(c);
    case 2: return phase2(c, stage);
    case 3: return phase_global(c, 1);
    case 4: {
      // energy sums of the current state (before the first step)
      TG_CK(cudaMemsetAsync(c->part, 0, sizeof(double) * 8 * (size_t)c->npart_blocks, c->st));
      int nb = 0;
      const cx<double>* F[3] = {c->U0[0], c->U0[1], c->U0[2]};
      TG_CK(launch_energy_partials(c->g, F, 3, c->part, 0, 8, c->st, &nb, 1));
      if (c->phys == TG_SCALAR || c->phys == TG_RB) {
        const cx<double>* T[1] = {c->U0[3]};
        TG_CK(launch_energy_partials(c->g, T, 1, c->part, 4, 8, c->st, &nb, 1));
      }
      return run_finalize(c, 0, false);
    }
    case 5: return phase_global(c, 2);
    default: return TG_ERR_ARG;
  }
}

int tg_slab_upload(tg_ctx* c, int field, const double* host) {
  int rc = slab_ok(c);
  if (rc) return rc;
  if (!host || field < 0 || field >= c->nstate) return TG_ERR_ARG;
  const Geo& g = c->g;
  const int nx = c->slab_nx[c->slab_r];
  const long long M3 = c->M3;
  std::vector<cx<double>> h((size_t)c->S);
  const cx<double>* src = reinterpret_cast<const cx<double>*>(host);
  for (int r = 0; r < nx; ++r) {
    const int l1 = amap_index(g.ax, g.x0 + r);
    for (int r2 = 0; r2 < g.nky; ++r2) {
      const int l2 = amap_index(g.ay, r2);
      cx<double>* d = h.data() + ((size_t)r * g.nky + r2) * g.kzp;
      const cx<double>* s = src + ((size_t)l1 * c->N2 + l2) * M3;
      for (int k = 0; k < g.kzp; ++k) d[k] = k < g.nkz ? s[k] : cx<double>{0.0, 0.0};
    }
  }
  cudaSetDevice(c->dev);
  cudaError_t e = cudaMemcpyAsync(c->U0[field], h.data(), sizeof(cx<double>) * h.size(), cudaMemcpyHostToDevice, c->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "slab upload");
  c->energy_valid = false;
  return TG_OK;
}

int tg_slab_download(tg_ctx* c, int field, double* host) {
  int rc = slab_ok(c);
  if (rc) return rc;
  if (!host || field < 0 || field >= c->nstate) return TG_ERR_ARG;
  const Geo& g = c->g;
  const int nx = c->slab_nx[c->slab_r];
  const long long M3 = c->M3;
  std::vector<cx<double>> h((size_t)c->S);
  cudaSetDevice(c->dev);
  cudaError_t e = cudaMemcpyAsync(h.data(), c->U0[field], sizeof(cx<double>) * h.size(), cudaMemcpyDeviceToHost, c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "slab download");
  TG_SYNC(c, "slab download");
  cx<double>* dst = reinterpret_cast<cx<double>*>(host);
  for (int r = 0; r < nx; ++r) {
    const int l1 = amap_index(g.ax, g.x0 + r);
    for (int r2 = 0; r2 < g.nky; ++r2) {
      const int l2 = amap_index(g.ay, r2);
      const cx<double>* s = h.data() + ((size_t)r * g.nky + r2) * g.kzp;
      cx<double>* d = dst + ((size_t)l1 * c->N2 + l2) * M3;
      for (int k = 0; k < g.nkz; ++k) d[k] = s[k];
    }
  }
  return TG_OK;
}

int tg_slab_scalars(tg_ctx* c, double* sums, double* scalars) {
  int rc = slab_ok(c);
  if (rc) return rc;
  cudaSetDevice(c->dev);
  TG_CK(cudaMemcpyAsync(c->h_pinned, c->red_out, sizeof(double) * 8, cudaMemcpyDeviceToHost, c->st));
  TG_CK(cudaMemcpyAsync(c->h_pinned + 8, c->scal, sizeof(double) * 8, cudaMemcpyDeviceToHost, c->st));
  TG_SYNC(c, "slab scalars");
  if (sums) std::memcpy(sums, c->h_pinned, sizeof(double) * 8);
  if (scalars) std::memcpy(scalars, c->h_pinned + 8, sizeof(double) * 8);
  return TG_OK;
}

}  // extern "C"
