// Internal definition of a solver context (the device-side state of one IncFluid/IncVF/IncSF
// set of objects in the reference).
#pragma once

#include <map>
#include <string>
#include <vector>

#include "../../include/tarang_gpu.h"
#include "tg_fft_launch.h"
#include "tg_spectral.cuh"

struct tg_ctx {
  tg_config cfg{};
  std::string err;
  int dev = 0;
  cudaStream_t st = nullptr;
  bool own_stream = false;

  // geometry
  int N1 = 0, N2 = 0, N3 = 0, M3 = 0, Mz = 0;
  int phys = 0, basis = 0, prec = 0;
  int tprec = 0;            // transform precision (tg::F64 / tg::F32)
  size_t tsz = 16;          // bytes per complex at transform precision
  tg::Geo g{};
  long long S = 0;          // compact elements per field
  long long D = 0;          // dense elements per field
  int nstate = 3, nin = 3, nprod = 6;
  tg::ProdPairs pairs{};
  double nu_of[6] = {0, 0, 0, 0, 0, 0};
  double nuh_of[6] = {0, 0, 0, 0, 0, 0};  // hyper coefficients per state field (0: off)
  // batch of same-shape requests (serving): B slots, the first nact of them advanced by a step;
  // slot r of every state and pipeline buffer at offset r * S (or r * stage size)
  int B = 1;
  int nact = 1;
  double* nu_tab = nullptr;  // [B][6] viscosity per slot and state field

  // twiddle tables: length -> exp(-2 pi i m / L)
  std::map<int, tg::cx<double>*> tw;
  // SCFT: (cos, sin)(pi j / 2 N1), j < 4 N1, and the x-pass kind of every pipeline field
  // (0 CFT, 1 SFT forward; 2 ICFT, 3 ISFT inverse)
  tg::cx<double>* zoct = nullptr;  // N3 = 256 or 128: coefficient table of the eight-lane z-pass
  tg::cx<double>* trigx = nullptr;
  double* xmat[4] = {};  // SCFT x-pass of the pipeline as matrices, per kind (see ctx creation)
  int xmat_rows[4] = {}, xmat_cols[4] = {};
  int xinv_kind[6] = {};
  int xfwd_kind[9] = {};
  double rb_fu = 0, rb_ft = 0;  // RB: Force1 = rb_fu theta, T.Force = rb_ft u1

  // compact solver state
  tg::cx<double>* U0[6] = {};
  tg::cx<double>* TOT[6] = {};
  void* US[6] = {};
  tg::cx<double>* NL[6] = {};
  tg::cx<double>* PR = nullptr;
  // pipeline intermediates (transform precision)
  void* WX[6] = {};
  void* WY[6] = {};
  void* PP[9] = {};
  void* PY[9] = {};
  void* PX[9] = {};

  // forcing box [nstate][(2 fx + 1)(2 fy + 1)(fz + 1)] over kx in [-fx, fx], ky in [-fy, fy],
  // kz in [0, fz]; force_on 1: energy supply (recomputed every stage), 2: fixed modes
  int force_on = 0;
  int fx = 0, fy = 0, fz = 0, fbox = 0;
  int nf_modes = 0;
  tg::cx<double>* FB = nullptr;
  bool force_ever = false;  // FB holds a force computed by this context
  bool coriolis = false;    // Force = V x om of every stage's velocity
  double om[3] = {0, 0, 0};
  bool lm = false;  // liquid-metal force (force_field_proc 101, fluid)
  double b0[3] = {0, 0, 0};

  // scalars and reductions
  double* scal = nullptr;   // per slot [8]: [0] dt, [1] t_now, [2] steps, [3] nonfinite, [4] Tdt
  double* red_out = nullptr;  // per slot [8]
  double* part = nullptr;   // per slot [nblocks][8]
  int npart_blocks = 0;
  double* ering = nullptr;  // energy per step of the current tg_step call
  int* ering_pos = nullptr;   // [0] ring position, [2] bounded-wait status (wait_status)
  // 1 when a TMA-staged pass of this context gave up waiting for its tile since the last
  // check (points into the ering_pos allocation); read and cleared by ctx_sync
  int* wait_status = nullptr;
  int* h_wait = nullptr;      // pinned host copy of *wait_status
  int wait_short = 0;         // test hook (tg_debug_set): first TMA wait gets no polls
  int ering_cap = 0;
  double* h_pinned = nullptr;  // small pinned host buffer
  double* diag = nullptr;      // diagnostics scratch (spectra, transfer tables)
  size_t diag_cap = 0;
  std::vector<double> shell_count;  // Sk_count over the dense grid (geometry only)

  // energy-transfer buffers (pipeline buffers reused where the physics already has them)
  bool et_ready = false;
  tg::cx<double>* etG[3] = {};
  tg::cx<double>* etVort[3] = {};  // vorticity of the velocity (helicity flux), owned via et_own
  tg::cx<double>* etZ[6] = {};     // Elsasser fields Z+ = U + B, Z- = U - B (MHD), via et_own
  tg::cx<double>* etZero = nullptr;  // a compact field of zeros (scalar transfers), via et_own
  void* etWY[6] = {};
  void* etPP[9] = {};
  void* etPY[9] = {};
  void* etPX[9] = {};
  void* et_own[32] = {};
  int n_et_own = 0;
  double dx_cfl = 0;

  // dense fields (reference layout, FP64), allocated on demand
  tg::cx<double>* dense[TG_NFIELDS] = {};
  tg::cx<double>* staging = nullptr;
  bool work_reserved[TG_NWORK] = {};  // tg_field_alloc

  // status
  bool energy_valid = false;  // scal[0] holds Get_dt of the current state
  bool have_nlin = false, have_pressure = false, have_force = false;
  size_t bytes = 0;

  // profiling: per-launch events on st
  struct ProfRec {
    const char* name;
    cudaEvent_t a, b;
    double bytes;
  };
  bool prof = false;
  std::vector<ProfRec> prof_recs;
  std::vector<cudaEvent_t> ev_pool;

  // slab-sharded single solve (tg_slab_*): this context is rank slab_r of slab_W; its spectral
  // state holds compact kx rows [slab_x[r], slab_x[r] + slab_nx[r]) (g.x0, g.S local) and between
  // the two exchanges of an RHS evaluation its pass buffers hold real y planes
  // [slab_y[r], slab_y[r] + slab_ny[r]).  slab_W = 0: a whole-grid context.
  int slab_W = 0, slab_r = 0;
  std::vector<int> slab_x, slab_nx, slab_y, slab_ny;
  void* SA[9] = {};   // [nx][N2][kzp]: y-inverse outputs of the inputs; unpacked products
  void* SB[9] = {};   // [nx][N2][kzp] as W chunks [nx][ny_d][kzp]: inverse send, forward receive
  void* SR[6] = {};   // [nkx][ny][kzp]: inverse receive (sources in rank order)
  double* gsum = nullptr;  // [8] reductions summed over the ranks (written by the host's all-reduce)

  // graph of one fused step
  cudaGraphExec_t step_graph = nullptr;
  bool graphs = true;
  bool pipeline_ok = true;
  int eager_steps = 0;
};

namespace tg {
int set_err(tg_ctx* c, int code, const std::string& msg);
int cuda_err(tg_ctx* c, cudaError_t e, const char* where);
// the context's bounded-wait status word and test hook, into the arguments of an axis pass
void wait_args(const tg_ctx* c, AxisArgs& a);
// synchronises the context's stream, then reports a TMA-staged pass that gave up waiting for
// its tile since the last check (TG_ERR_TIMEOUT: the results of that work are not valid; the
// word is cleared, so the context stays usable) or a CUDA error
int ctx_sync(tg_ctx* c, const char* where);
// a slab context (tg_slab_create) answers only the tg_slab_* calls: TG_ERR_STATE with a message
int slab_refuse(tg_ctx* c);
// a CUDA call inside a function with a context `c` in scope: its error becomes the call's status
#define TG_CK(call)                                        \
  do {                                                     \
    cudaError_t _e = (call);                               \
    if (_e != cudaSuccess) return cuda_err(c, _e, #call);  \
  } while (0)
#define TG_SYNC(c, where)                      \
  do {                                         \
    const int _rs = tg::ctx_sync((c), (where)); \
    if (_rs) return _rs;                       \
  } while (0)

// per-launch CUDA events while profiling is enabled (tg_profile_enable)
struct ProfScope {
  tg_ctx* c;
  long idx = -1;
  ProfScope(tg_ctx* c_, const char* name, double bytes);
  ~ProfScope();
};
double el_compact(const tg_ctx* c);
double el_xstage(const tg_ctx* c);
double el_ystage(const tg_ctx* c);

// x- and y-inverse passes of nf compact fields (field f read as in[f] + comb[f] * in2[f]);
// nread = number of distinct compact fields read (for the byte count)
int pipe_inverse_xy(tg_ctx* c, int nf, const void* const* in, const void* const* in2, const int* comb,
                    int inprec, int nread, void* const* WX, void* const* WY);
// fused z-pass products (pairs pp of the nin inputs), then y- and x-forward passes into PX;
// SCFT: product q takes the x transform xkinds[q] (0 cosine, 1 sine; default c->xfwd_kind)
int pipe_products_forward(tg_ctx* c, int nin, const void* const* WY, int nprod, const ProdPairs& pp,
                          void* const* PP, void* const* PY, void* const* PX, const int* xkinds = nullptr);
int dalloc_ctx(tg_ctx* c, void** p, size_t bytes);
// a context holding B same-shape request slots (B = 1: tg_ctx_create); with slab_W > 0, rank
// slab_r's share of a slab-sharded solve (B = 1)
int ctx_create_batch(const tg_config* cfg, int B, tg_ctx** out, int slab_W = 0, int slab_r = 0);
// arguments of the RK stage kernel for the context's current buffers
RKArgs rk_args(tg_ctx* c, int stage);
// reduce the partials of slots r0 .. r0+n-1 (n < 0: all active) and apply the dt rule
int run_finalize(tg_ctx* c, int dt_mode, bool ring, int r0 = 0, int n = -1);
// start and count of part i of n items split over W parts (the first n % W parts one larger)
inline void split_range(int n, int W, int i, int& start, int& count) {
  const int b = n / W, rem = n % W;
  count = b + (i < rem ? 1 : 0);
  start = i * b + (i < rem ? i : rem);
}
size_t ctx_bytes_estimate(const tg_config* cfg, int B, bool with_staging);
int ensure_staging_ctx(tg_ctx* c);
// TG_OK or the code tg_ctx_create returns for cfg before allocating anything
int validate_config(const tg_config* cfg);
// viscosity of each state field (nu, eta, kappa; RB: from Ra and Pr)
void state_viscosities(const tg_config* cfg, double nu[6]);
void state_hyper(const tg_config* cfg, double nuh[6]);
// the RK kernel's stages of one step of the configured scheme, in order (k_rk STAGE codes):
// RK4 1, 2, 3, 4; EULER 5; RK2 7, 6
int scheme_stages(int scheme, int out[4]);
// the stage that ends a step (energy partials, U0 written)
inline bool stage_is_final(int stage) { return stage == 4 || stage == 5 || stage == 6; }
struct RBCoef {
  double nu, kappa, fu, ft, nuf;
};
RBCoef rb_coefficients(const tg_config* cfg);
// one fused RK4 step of the first nact slots, enqueued on c->st; ring: record slot 0's energy
int enqueue_step(tg_ctx* c, bool ring);
// energies of the master state of all active slots, or of slots r0 .. r0+n-1; dt_mode 2 sets
// each slot's dt by the Get_dt rule without advancing its time
int run_energy(tg_ctx* c, int dt_mode);
int run_energy_slots(tg_ctx* c, int dt_mode, int r0, int n);
// the force box from the current state if this context never computed a force (else unchanged)
int ensure_force_box(tg_ctx* c);
// Max_radius_inside (four_inline.h:190-257, scft_inline.h) of the context's grid
int radius_inside(const tg_ctx* c);
// the diagnostics scratch c->diag grown to at least `need` doubles
int ensure_diag(tg_ctx* c, size_t need);
// energy-transfer buffers (giver fields etG, helper transforms etWY, products etPP/PY/PX)
int ensure_et_buffers(tg_ctx* c);
// SCFT x transforms of P(i, j) = F(H_j G_i), q = 3 i + j, with H and G of parities (sin, cos,
// cos) along x: sin x sin and cos x cos products are cosine series (0), mixed ones sine (1)
// (ET_Forward_transform_RSprod_G ET_transform.cc:49-113 with the parities of ET_RSprod.cc:49-169)
constexpr int kEtXKinds[9] = {0, 1, 1, 1, 0, 0, 1, 0, 0};
// helper, giver and receiver fields of an energy-transfer kind (TG_ET_*) and its sign; Elsasser
// kinds fill scratch fields first (tg_et.cu)
int et_kind_fields(tg_ctx* c, int kind, const cx<double>* H[3], const cx<double>* F[3], const cx<double>* R[3],
                   double& sign);
}  // namespace tg
