// Serving loop: continuous batching of independent solves on one GPU.
//
// A batch is a context created with B request slots (ctx_create_batch): every state and
// pipeline buffer holds B copies at a fixed slot stride, and every kernel of the step takes the
// slot as a grid dimension, so one launch per pass advances the first nact slots.  Active slots
// are kept dense (0 .. nact-1): a request that leaves hands its slot to the last one.  A step of
// a batch with nact active slots is one CUDA graph, captured once per (batch, nact).
//
// Per request, the slot carries its own viscosities (nu_tab row), dt, time, step count,
// non-finite flag and dt ceiling (scal row); the energy reduction of each slot runs in its own
// blocks in a fixed order.  So a request's fields after n steps are the same bits whatever else
// shares its batch, and the same as tg_step on a lone context.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "tg_ctx.h"

using namespace tg;

namespace {

struct Req {
  long long id = 0;
  tg_config cfg{};
  int n_steps = 0;
  int nstate = 3;
  std::vector<double> init;    // dropped at admission (when the pinned pool was full at submit)
  double* init_pin = nullptr;  // pinned block of the pool holding the fields (usual case)
  const double* init_borrow = nullptr;  // the caller's fields (borrow_inputs), until admission
  size_t n_init = 0;
  double* result = nullptr;    // kept fields (reference layout): a device block, or a pinned host
  size_t n_result = 0;         // block when the device had no room
  bool result_host = false;
  cudaEvent_t result_ev = nullptr;  // the result's copies into `result` are done past this event
  tg_request_status st{};
  std::string key;
  long long batch = -1;        // batch id while running
};

struct Batch {
  long long id = 0;
  std::string key;
  tg_ctx* c = nullptr;
  int B = 0;
  bool solo = false;                 // forced request: one slot, never shared
  std::vector<long long> slot_req;   // request id of active slot r
  std::map<int, cudaGraphExec_t> graphs;  // per active count
  bool warmed = false;               // one eager step ran (module loading outside capture)
  double* h = nullptr;               // pinned: scal [B][8], red_out [B][8], load rows [B][16]
  std::vector<std::pair<double*, size_t>> loading;  // pinned init blocks of loads in flight
  size_t bytes = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;  // around the steps of the current round
  int launched_steps = 0;
  bool launched_graph = false;       // the round's steps were graph replays (their timing counts)
  double device_ms = 0;              // all timed steps so far
  long long steps_run = 0;
  double step_ms = 0;                // measured time of one step at the current active count
  int step_ms_nact = 0;
  double idle_since = -1;            // server clock when the batch last became empty
};

// Page-locked host blocks, reused by size: initial fields on their way to the device and
// finished fields on their way back, so that neither copy waits for the batch's stream.
struct PinnedPool {
  std::map<size_t, std::vector<double*>> free_;
  size_t held = 0;
  static constexpr size_t kCap = (size_t)16 << 30;  // page-locked bytes held at most
  double* get(size_t n) {
    auto it = free_.find(n);
    if (it != free_.end() && !it->second.empty()) {
      double* p = it->second.back();
      it->second.pop_back();
      return p;
    }
    void* p = nullptr;
    if (held + sizeof(double) * n > kCap) return nullptr;
    if (cudaMallocHost(&p, sizeof(double) * n) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    held += sizeof(double) * n;
    return (double*)p;
  }
  void put(double* p, size_t n) {
    if (p) free_[n].push_back(p);
  }
  void clear() {
    for (auto& kv : free_)
      for (double* p : kv.second) cudaFreeHost(p);
    free_.clear();
    held = 0;
  }
};

}  // namespace

struct tg_server {
  tg_server_config cfg{};
  int dev = 0;
  std::chrono::steady_clock::time_point t0;
  long long next_id = 1, next_batch = 1;
  std::map<long long, Req> reqs;
  std::vector<long long> queue;        // FIFO of queued request ids
  std::vector<long long> finished;     // finished since the last tg_server_take_finished
  std::map<long long, Batch> batches;
  PinnedPool pinned;
  size_t bytes = 0, bytes_peak = 0;
  long long rounds = 0, request_steps = 0, graph_launches = 0, eager_steps = 0;
  std::string err;
  bool round_open = false;                                // between pump_begin and pump_end
  cudaStream_t aux = nullptr;  // result downloads and frees (non-blocking)
  cudaMemPool_t pool = nullptr;  // device blocks of kept results: freed blocks stay for reuse
  cudaEvent_t chain = nullptr;                            // end of the last batch launched
  std::map<long long, std::pair<int, int>> launched;      // batch -> (slots stepped, launch code)
};

namespace {

double now_s(const tg_server* s) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - s->t0).count();
}

int state_fields(int physics) {
  if (physics == TG_MHD) return 6;
  if (physics == TG_SCALAR || physics == TG_RB) return 4;
  return 3;
}

// Requests share a batch when they agree on everything that the kernels or the geometry read
// from the context; the per-slot coefficients (viscosities, dt) may differ.
std::string batch_key(const tg_config& c, long long id) {
  char buf[512];
  std::snprintf(buf, sizeof(buf), "%d,%d,%d|b%d|p%d|x%d|d%d|s%d|k%a,%a,%a|f%d|h%a,%a,%a", c.N[0], c.N[1], c.N[2],
                c.basis, c.physics, c.precision, c.dealias, c.scheme, c.kfactor[0], c.kfactor[1], c.kfactor[2],
                c.force_kind, c.hyper_nu, c.hyper_eta, c.hyper_kappa);
  std::string k(buf);
  if (c.force_kind == TG_FORCE_ENERGY_SUPPLY || c.force_kind == TG_FORCE_ENERGY_HELICITY)
    k += "|solo" + std::to_string(id);
  if (c.force_kind == TG_FORCE_CORIOLIS || c.force_kind == TG_FORCE_RB_ROTATION ||
      c.force_kind == TG_FORCE_LIQUID_METAL) {
    // Omega (Coriolis) or B0 (liquid metal): one value per batch
    std::snprintf(buf, sizeof(buf), "|om%a,%a,%a", c.force_para[0], c.force_para[1], c.force_para[2]);
    k += buf;
  }
  if (c.physics == TG_RB && (c.force_kind == TG_FORCE_RB || c.force_kind == TG_FORCE_RB_ROTATION)) {
    // the buoyancy coefficients are per context: requests share a batch only when they agree
    const RBCoef r = rb_coefficients(&c);
    std::snprintf(buf, sizeof(buf), "|rb%a,%a", r.fu, r.ft);
    k += buf;
  }
  return k;
}

void destroy_batch(tg_server* s, Batch& b) {
  if (b.c) {
    cudaSetDevice(b.c->dev);
    cudaStreamSynchronize(b.c->st);
    for (auto& kv : b.graphs) cudaGraphExecDestroy(kv.second);
    b.graphs.clear();
    if (b.ev0) cudaEventDestroy(b.ev0);
    if (b.ev1) cudaEventDestroy(b.ev1);
    b.ev0 = b.ev1 = nullptr;
    tg_ctx_destroy(b.c);
    b.c = nullptr;
  }
  for (auto& blk : b.loading) s->pinned.put(blk.first, blk.second);
  b.loading.clear();
  if (b.h) cudaFreeHost(b.h);
  b.h = nullptr;
  s->bytes -= b.bytes;
  b.bytes = 0;
}

void finish_req(tg_server* s, Req& r, int state, int error) {
  s->finished.push_back(r.id);
  r.st.state = state;
  r.st.error = error;
  r.st.finish_s = now_s(s);
  r.batch = -1;
  std::vector<double>().swap(r.init);
  if (r.init_pin) s->pinned.put(r.init_pin, r.n_init);
  r.init_pin = nullptr;
  r.init_borrow = nullptr;
}

// Enqueue, on the batch stream, the copy of a request's fields into slot `slot` and the set-up
// of the slot's coefficients, time and dt (Get_dt of the initial state, compute_dt.cc:47-108).
// The host only copies into a pinned block; the stream runs the rest after the batch's step.
int load_slot(tg_server* s, Batch& b, int slot, Req& r) {
  tg_ctx* c = b.c;
  const size_t D2 = 2 * (size_t)c->D;
  const size_t n = D2 * c->nstate;
  const double* src = r.init_borrow;
  if (src) {
    // the caller's (pageable) memory: each copy returns once the driver has staged it, so the
    // caller's buffer is free again when this function returns
    r.init_borrow = nullptr;
  } else {
    double* pin = r.init_pin;
    if (pin) {
      r.init_pin = nullptr;  // from here on the batch releases it (after the copies ran)
    } else {
      pin = s->pinned.get(n);
      if (!pin) return set_err(c, TG_ERR_OOM, "pinned host block for a request's fields");
      std::memcpy(pin, r.init.data(), sizeof(double) * n);
      std::vector<double>().swap(r.init);
    }
    b.loading.emplace_back(pin, n);
    src = pin;
  }
  cudaError_t e;
  for (int i = 0; i < c->nstate; ++i) {
    e = cudaMemcpyAsync(c->staging, src + (size_t)i * D2, sizeof(double) * D2, cudaMemcpyHostToDevice, c->st);
    if (e != cudaSuccess) return cuda_err(c, e, "slot upload");
    e = launch_dense_to_compact(c->g, c->staging, c->U0[i] + (size_t)slot * c->S, 0, c->st);
    if (e != cudaSuccess) return cuda_err(c, e, "slot upload");
  }
  double nu[6];
  state_viscosities(&r.cfg, nu);
  double* row = b.h + 16 * (size_t)b.B + 16 * (size_t)slot;  // this slot's load row
  for (int i = 0; i < 6; ++i) row[i] = nu[i];
  const double sc[8] = {r.cfg.dt, 0, 0, 0, r.cfg.dt, 0, 0, 0};
  for (int i = 0; i < 8; ++i) row[8 + i] = sc[i];
  e = cudaMemcpyAsync(c->nu_tab + (size_t)slot * 6, row, sizeof(double) * 6, cudaMemcpyHostToDevice, c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "slot coefficients");
  e = cudaMemcpyAsync(c->scal + (size_t)slot * 8, row + 8, sizeof(double) * 8, cudaMemcpyHostToDevice, c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "slot scalars");
  return run_energy_slots(c, 2, slot, 1);
}

// fields of slot `slot` into a device block held by the request (reference layout), queued on
// the batch stream ahead of anything that reuses the slot or the staging buffer; no host work and
// no page-locking: the block goes to the host only when tg_server_result asks for it
int store_slot(tg_server* s, Batch& b, int slot, Req& r) {
  tg_ctx* c = b.c;
  if (!s->cfg.keep_results) return TG_OK;
  const size_t D2 = 2 * (size_t)c->D;
  const size_t n = D2 * c->nstate;
  // kept results are outside the batch budget (the caller releases them); a pinned host block
  // where the device has no room
  double* res = nullptr;
  bool on_host = false;
  if (cudaMallocFromPoolAsync(reinterpret_cast<void**>(&res), sizeof(double) * n, s->pool, c->st) != cudaSuccess) {
    cudaGetLastError();
    res = s->pinned.get(n);
    if (!res) return set_err(c, TG_ERR_OOM, "block for a result");
    on_host = true;
  }
  const cudaMemcpyKind kind = on_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < c->nstate && e == cudaSuccess; ++i) {
    e = launch_compact_to_dense(c->g, c->U0[i] + (size_t)slot * c->S, 0, c->staging, c->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(res + (size_t)i * D2, c->staging, sizeof(double) * D2, kind, c->st);
  }
  cudaEvent_t ev = nullptr;
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord(ev, c->st);
  if (e != cudaSuccess) {
    cudaStreamSynchronize(c->st);  // no copy into the block may still be running
    if (ev) cudaEventDestroy(ev);
    if (on_host) s->pinned.put(res, n);
    else cudaFree(res);
    return cuda_err(c, e, "slot result");
  }
  r.result = res;
  r.n_result = n;
  r.result_host = on_host;
  r.result_ev = ev;
  return TG_OK;
}

// the request's result copies have landed (a no-op once waited for)
void wait_result(Req& r) {
  if (r.result_ev) {
    cudaEventSynchronize(r.result_ev);
    cudaEventDestroy(r.result_ev);
    r.result_ev = nullptr;
  }
}

// slot `to` takes the request in slot `from` (device copies on the batch stream)
int move_slot(Batch& b, int from, int to) {
  tg_ctx* c = b.c;
  const size_t Sd = sizeof(cx<double>) * (size_t)c->S;
  cudaError_t e;
  for (int i = 0; i < c->nstate; ++i) {
    e = cudaMemcpyAsync(c->U0[i] + (size_t)to * c->S, c->U0[i] + (size_t)from * c->S, Sd, cudaMemcpyDeviceToDevice, c->st);
    if (e != cudaSuccess) return cuda_err(c, e, "slot move");
  }
  e = cudaMemcpyAsync(c->scal + (size_t)to * 8, c->scal + (size_t)from * 8, sizeof(double) * 8, cudaMemcpyDeviceToDevice, c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "slot move");
  e = cudaMemcpyAsync(c->red_out + (size_t)to * 8, c->red_out + (size_t)from * 8, sizeof(double) * 8, cudaMemcpyDeviceToDevice, c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "slot move");
  e = cudaMemcpyAsync(c->nu_tab + (size_t)to * 6, c->nu_tab + (size_t)from * 6, sizeof(double) * 6, cudaMemcpyDeviceToDevice, c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "slot move");
  return TG_OK;
}

// a new batch for request r's key: as many slots as fit in a quarter of the budget (at least
// one) and in what is left of it, at most max_batch
int open_batch(tg_server* s, const Req& r, long long* bid) {
  const bool solo = r.cfg.force_kind == TG_FORCE_ENERGY_SUPPLY || r.cfg.force_kind == TG_FORCE_ENERGY_HELICITY;
  const size_t budget = s->cfg.hbm_budget_bytes;
  const size_t left = budget > s->bytes ? budget - s->bytes : 0;
  const size_t one = ctx_bytes_estimate(&r.cfg, 1, true);
  if (one == 0 || one > left) return TG_ERR_OOM;
  const size_t cap = std::min(left, std::max(budget / 4, one));
  int B = 1;
  if (!solo) {
    B = std::max(1, s->cfg.max_batch);
    while (B > 1 && ctx_bytes_estimate(&r.cfg, B, true) > cap) --B;
  }
  tg_config cc = r.cfg;
  cc.device = s->dev;
  cc.stream = nullptr;
  tg_ctx* c = nullptr;
  int rc = ctx_create_batch(&cc, B, &c);
  if (rc) return rc;
  rc = ensure_staging_ctx(c);
  if (rc) {
    tg_ctx_destroy(c);
    return rc;
  }
  Batch b;
  b.id = s->next_batch++;
  b.key = r.key;
  b.c = c;
  b.B = B;
  b.solo = solo;
  c->graphs = s->cfg.use_graphs != 0;
  if (cudaMallocHost(&b.h, sizeof(double) * 32 * (size_t)B) != cudaSuccess) {
    tg_ctx_destroy(c);
    return TG_ERR_OOM;
  }
  b.bytes = c->bytes;
  s->bytes += b.bytes;
  s->bytes_peak = std::max(s->bytes_peak, s->bytes);
  *bid = b.id;
  s->batches.emplace(b.id, std::move(b));
  return TG_OK;
}

// release the idle batch that has been idle longest; false if there is none
bool evict_idle_batch(tg_server* s) {
  auto victim = s->batches.end();
  for (auto it = s->batches.begin(); it != s->batches.end(); ++it) {
    const Batch& b = it->second;
    if (!b.slot_req.empty() || !b.loading.empty()) continue;
    if (victim == s->batches.end() || b.idle_since < victim->second.idle_since) victim = it;
  }
  if (victim == s->batches.end()) return false;
  destroy_batch(s, victim->second);
  s->batches.erase(victim);
  return true;
}

// admit queued requests in arrival order into batches with free slots or into new batches
int admit(tg_server* s) {
  std::vector<long long> still;
  for (size_t qi = 0; qi < s->queue.size(); ++qi) {
    Req& r = s->reqs[s->queue[qi]];
    long long bid = -1;
    for (auto& kv : s->batches) {
      Batch& b = kv.second;
      if (b.key == r.key && !b.solo && (int)b.slot_req.size() < b.B) {
        bid = kv.first;
        break;
      }
    }
    if (bid < 0) {
      int rc = open_batch(s, r, &bid);
      while (rc == TG_ERR_OOM && evict_idle_batch(s)) rc = open_batch(s, r, &bid);
      if (rc == TG_ERR_OOM) {
        if (s->batches.empty()) {
          // nothing resident and still no room: the allocation itself failed
          finish_req(s, r, TG_REQ_FAILED, TG_ERR_OOM);
        } else {
          still.push_back(r.id);  // waits for room
        }
        continue;
      }
      if (rc) {
        finish_req(s, r, TG_REQ_FAILED, rc);
        continue;
      }
    }
    Batch& b = s->batches[bid];
    const int slot = (int)b.slot_req.size();
    r.st.start_s = now_s(s);
    int rc = load_slot(s, b, slot, r);
    if (rc) {
      s->err = b.c->err;
      finish_req(s, r, TG_REQ_FAILED, rc);
      continue;
    }
    r.st.state = TG_REQ_RUNNING;
    r.batch = bid;
    b.slot_req.push_back(r.id);  // a request of 0 steps leaves at the collect that follows
  }
  s->queue.swap(still);
  return TG_OK;
}

// one step of the active slots of batch b, then the slot scalars into pinned memory
// k steps of the active slots of batch b (one graph replay each, captured per active count;
// the first step of a batch runs eagerly), timed by events on the batch stream, then the slot
// scalars and energies into pinned memory
int launch_batch(tg_server* s, Batch& b, int k) {
  tg_ctx* c = b.c;
  const int nact = (int)b.slot_req.size();
  c->nact = nact;
  cudaError_t e;
  if (!b.ev0) {
    if (cudaEventCreate(&b.ev0) != cudaSuccess || cudaEventCreate(&b.ev1) != cudaSuccess)
      return cuda_err(c, cudaGetLastError(), "cudaEventCreate");
  }
  // the graph of this active count first, so that a capture stays outside the timed steps
  cudaGraphExec_t ex = nullptr;
  if (s->cfg.use_graphs && b.warmed) {
    auto it = b.graphs.find(nact);
    if (it == b.graphs.end()) {
      cudaGraph_t gr = nullptr;
      e = cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) return cuda_err(c, e, "cudaStreamBeginCapture");
      int rc = enqueue_step(c, false);
      cudaError_t e2 = cudaStreamEndCapture(c->st, &gr);
      if (rc) {
        if (gr) cudaGraphDestroy(gr);
        return rc;
      }
      if (e2 != cudaSuccess) return cuda_err(c, e2, "cudaStreamEndCapture");
      cudaGraphExec_t g = nullptr;
      e = cudaGraphInstantiate(&g, gr, 0);
      cudaGraphDestroy(gr);
      if (e != cudaSuccess) return cuda_err(c, e, "cudaGraphInstantiate");
      it = b.graphs.emplace(nact, g).first;
    }
    ex = it->second;
  }
  e = cudaEventRecord(b.ev0, c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "cudaEventRecord");
  for (int step = 0; step < k; ++step) {
    if (ex) {
      e = cudaGraphLaunch(ex, c->st);
      if (e != cudaSuccess) return cuda_err(c, e, "cudaGraphLaunch");
      s->graph_launches++;
    } else {
      int rc = enqueue_step(c, false);
      if (rc) return rc;
      b.warmed = true;
      s->eager_steps++;
    }
  }
  e = cudaEventRecord(b.ev1, c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "cudaEventRecord");
  b.launched_steps = k;
  b.launched_graph = ex != nullptr;
  e = cudaMemcpyAsync(b.h, c->scal, sizeof(double) * 8 * nact, cudaMemcpyDeviceToHost, c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "slot scalars");
  e = cudaMemcpyAsync(b.h + 8 * (size_t)b.B, c->red_out, sizeof(double) * 8 * nact, cudaMemcpyDeviceToHost, c->st);
  if (e != cudaSuccess) return cuda_err(c, e, "slot energies");
  return TG_OK;
}

// Steps per round of each batch: the slowest batch runs one, a faster one about as many as fit
// in that time (at most kMaxStepsPerRound), never past the fewest steps any of its requests
// still needs.  Until a batch has a measured step time it runs one.
constexpr int kMaxStepsPerRound = 16;

int steps_this_round(const tg_server* s, const Batch& b, double slowest_ms) {
  int left = 1 << 30;
  for (long long id : b.slot_req) {
    const Req& q = s->reqs.at(id);
    left = std::min(left, std::max(1, q.n_steps - q.st.steps_done));
  }
  int k = 1;
  if (b.step_ms > 0 && slowest_ms > 0) k = (int)std::floor(slowest_ms / b.step_ms);
  k = std::max(1, std::min(k, kMaxStepsPerRound));
  return std::min(k, left);
}

// after the round: count the step of the first nl slots (those that were launched), retire
// finished and non-finite requests, keep the slots dense
int collect_batch(tg_server* s, Batch& b, int nl, int launch_rc) {
  tg_ctx* c = b.c;
  // a bounded wait that ran out (TG_ERR_TIMEOUT) fails every request of this batch; the
  // batch itself stays usable for later requests
  const int sync_rc = ctx_sync(c, "batch step");
  for (auto& blk : b.loading) s->pinned.put(blk.first, blk.second);
  b.loading.clear();
  if (launch_rc || sync_rc) {
    const int code = launch_rc ? launch_rc : sync_rc;
    s->err = c->err;
    for (long long id : b.slot_req) finish_req(s, s->reqs[id], TG_REQ_FAILED, code);
    b.slot_req.clear();
    return code;
  }
  // only graph replays time a step: an eager step's events also span its host-side launches
  // (module loading, first-use set-up) and would make the batch look far slower than it is
  if (nl > 0 && b.launched_steps > 0) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, b.ev0, b.ev1) == cudaSuccess) {
      b.device_ms += ms;
      b.steps_run += b.launched_steps;
    }
  }
  if (nl > 0 && b.launched_steps > 0 && b.launched_graph) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, b.ev0, b.ev1) == cudaSuccess) {
      const double per = ms / b.launched_steps;
      b.step_ms = (b.step_ms_nact == nl && b.step_ms > 0) ? 0.5 * (b.step_ms + per) : per;
      b.step_ms_nact = nl;
    }
  }
  std::vector<int> leave;
  const int n = (int)b.slot_req.size();
  for (int r = 0; r < n; ++r) {
    Req& q = s->reqs[b.slot_req[r]];
    if (r < nl) {
      const double* sc = b.h + 8 * (size_t)r;
      const double* ro = b.h + 8 * (size_t)b.B + 8 * (size_t)r;
      const int now = (int)sc[2];  // the slot's step counter (Get_dt's finalize counts every step)
      s->request_steps += now - q.st.steps_done;
      q.st.steps_done = now;
      q.st.t_final = sc[1];
      q.st.final_energy = ro[0] + (c->phys == TG_MHD ? ro[2] : 0.0);
      if (sc[3] != 0.0) {
        finish_req(s, q, TG_REQ_FAILED, TG_ERR_NONFINITE);
        leave.push_back(r);
        continue;
      }
    }
    if (q.st.steps_done >= q.n_steps) {
      const int rc = store_slot(s, b, r, q);
      finish_req(s, q, rc ? TG_REQ_FAILED : TG_REQ_DONE, rc);
      leave.push_back(r);
    }
  }
  // fill each hole from the end, highest hole first
  for (auto it = leave.rbegin(); it != leave.rend(); ++it) {
    const int hole = *it;
    const int last = (int)b.slot_req.size() - 1;
    if (hole != last) {
      int rc = move_slot(b, last, hole);
      if (rc) return rc;
      b.slot_req[hole] = b.slot_req[last];
    }
    b.slot_req.pop_back();
  }
  return TG_OK;
}

}  // namespace

extern "C" {

int tg_request_bytes(const tg_config* cfg, int batch, size_t* bytes) {
  if (!cfg || !bytes || batch < 1) return TG_ERR_ARG;
  const int v = validate_config(cfg);
  if (v) return v;
  *bytes = ctx_bytes_estimate(cfg, batch, true);
  return *bytes ? TG_OK : TG_ERR_ARG;
}

int tg_server_create(const tg_server_config* cfg, tg_server** out) {
  if (!cfg || !out) return TG_ERR_ARG;
  *out = nullptr;
  if (cfg->hbm_budget_bytes == 0 || cfg->max_batch < 1) return TG_ERR_ARG;
  if (cudaSetDevice(cfg->device) != cudaSuccess) return TG_ERR_CUDA;
  tg_server* s = new tg_server();
  s->cfg = *cfg;
  s->dev = cfg->device;
  if (cudaStreamCreateWithFlags(&s->aux, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    delete s;
    return TG_ERR_CUDA;
  }
  // the kept results' pool keeps freed memory mapped (a pool that hands memory back at every
  // synchronisation maps it again for the next result)
  cudaMemPoolProps pp{};
  pp.allocType = cudaMemAllocationTypePinned;
  pp.location.type = cudaMemLocationTypeDevice;
  pp.location.id = s->dev;
  if (cudaMemPoolCreate(&s->pool, &pp) != cudaSuccess) {
    cudaGetLastError();
    cudaStreamDestroy(s->aux);
    delete s;
    return TG_ERR_CUDA;
  }
  unsigned long long keep = ~0ull;
  cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  s->t0 = std::chrono::steady_clock::now();
  *out = s;
  return TG_OK;
}

int tg_server_destroy(tg_server* s) {
  if (!s) return TG_ERR_ARG;
  cudaSetDevice(s->dev);
  if (s->round_open) tg_server_pump_end(s, nullptr);
  for (auto& kv : s->reqs) wait_result(kv.second);
  for (auto& kv : s->batches) destroy_batch(s, kv.second);
  if (s->chain) cudaEventDestroy(s->chain);
  if (s->aux) cudaStreamSynchronize(s->aux);  // frees and downloads of results queued there
  for (auto& kv : s->reqs) {
    if (!kv.second.result) continue;
    if (kv.second.result_host) cudaFreeHost(kv.second.result);
    else cudaFree(kv.second.result);
  }
  if (s->aux) cudaStreamDestroy(s->aux);
  if (s->pool) cudaMemPoolDestroy(s->pool);
  for (auto& kv : s->reqs)
    if (kv.second.init_pin) cudaFreeHost(kv.second.init_pin);
  s->pinned.clear();
  delete s;
  return TG_OK;
}

int tg_server_submit(tg_server* s, const tg_request* rq, long long* id) {
  if (!s || !rq || !id) return TG_ERR_ARG;
  *id = -1;
  const int v = validate_config(&rq->cfg);
  if (v) return v;
  // a request carries no force modes (tg_set_force_modes is a context call)
  if (rq->cfg.force_kind == TG_FORCE_MODES) return TG_ERR_UNSUPPORTED;
  const int Mz = rq->cfg.N[2] / 2;
  if (!(Mz >= 4 && Mz <= 256 && (Mz & (Mz - 1)) == 0)) return TG_ERR_UNSUPPORTED;
  if (rq->n_steps < 0) return TG_ERR_ARG;
  const int ns = state_fields(rq->cfg.physics);
  const size_t D2 = 2 * (size_t)rq->cfg.N[0] * rq->cfg.N[1] * (rq->cfg.N[2] / 2 + 1);
  if (!rq->init || rq->n_doubles != D2 * ns) return TG_ERR_ARG;
  Req r;
  r.id = s->next_id++;
  r.cfg = rq->cfg;
  r.n_steps = rq->n_steps;
  r.nstate = ns;
  r.key = batch_key(r.cfg, r.id);
  r.st.state = TG_REQ_QUEUED;
  r.st.submit_s = now_s(s);
  if (ctx_bytes_estimate(&r.cfg, 1, true) > s->cfg.hbm_budget_bytes) {
    r.st.state = TG_REQ_FAILED;
    r.st.error = TG_ERR_OOM;
    r.st.finish_s = r.st.submit_s;
    s->finished.push_back(r.id);
  } else if (s->cfg.borrow_inputs) {
    // no copy: admission uploads from the caller's memory (valid until the request runs)
    r.n_init = rq->n_doubles;
    r.init_borrow = rq->init;
    s->queue.push_back(r.id);
  } else {
    // into a reused page-locked block when the pool has room (no page faults, and the upload
    // at admission is a plain asynchronous copy), else into ordinary memory
    r.n_init = rq->n_doubles;
    r.init_pin = s->pinned.get(r.n_init);
    if (r.init_pin) std::memcpy(r.init_pin, rq->init, sizeof(double) * r.n_init);
    else r.init.assign(rq->init, rq->init + rq->n_doubles);
    s->queue.push_back(r.id);
  }
  *id = r.id;
  s->reqs.emplace(r.id, std::move(r));
  return TG_OK;
}

// The round's launches: the steps of every running batch go to the device first, so that the
// host work that follows (submissions between pump_begin and pump_end, then admission: copies
// into pinned blocks, new contexts) overlaps them.  The batches run one after another on the
// device (each batch's stream waits for the previous batch's steps): a batch of requests
// saturates the device alone, and batches overlapping on their streams measured slower in sum
// (L2 shared by unrelated working sets) than the same batches in sequence.  Each batch's step
// time (events on its stream, after the wait) is then its own, which steps_this_round needs.
int tg_server_pump_begin(tg_server* s) {
  if (!s) return TG_ERR_ARG;
  if (s->round_open) return TG_ERR_STATE;
  cudaSetDevice(s->dev);
  auto& launched = s->launched;
  launched.clear();
  if (!s->chain && cudaEventCreateWithFlags(&s->chain, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    s->chain = nullptr;
    return TG_ERR_CUDA;
  }
  double slowest = 0;
  for (auto& kv : s->batches)
    if (!kv.second.slot_req.empty()) slowest = std::max(slowest, kv.second.step_ms);
  // (the chain orders independent work only: where a wait or record fails the batches overlap)
  bool chained = false;
  for (auto& kv : s->batches) {
    Batch& b = kv.second;
    if (b.slot_req.empty()) continue;
    if (chained && cudaStreamWaitEvent(b.c->st, s->chain, 0) != cudaSuccess) cudaGetLastError();
    const int nl = (int)b.slot_req.size();
    const int k = s->cfg.use_graphs ? steps_this_round(s, b, slowest) : 1;
    launched[kv.first] = {nl, launch_batch(s, b, k)};
    chained = cudaEventRecord(s->chain, b.c->st) == cudaSuccess;
    if (!chained) cudaGetLastError();
  }
  s->round_open = true;
  return TG_OK;
}

// admission, then the wait for the round's steps and the retirement of finished requests
int tg_server_pump_end(tg_server* s, int* n_active) {
  if (!s) return TG_ERR_ARG;
  cudaSetDevice(s->dev);

  if (!s->round_open) s->launched.clear();  // a round without launches: admission only
  s->round_open = false;
  const auto& launched = s->launched;
  int first_err = admit(s);
  for (auto& kv : s->batches) {
    Batch& b = kv.second;
    auto it = launched.find(kv.first);
    if (it == launched.end() && b.slot_req.empty() && b.loading.empty()) continue;
    const int nl = it == launched.end() ? 0 : it->second.first;
    const int lrc = it == launched.end() ? TG_OK : it->second.second;
    const int r2 = collect_batch(s, b, nl, lrc);
    if (r2 && !first_err) first_err = r2;
  }
  if (!launched.empty()) s->rounds++;
  // an idle batch stays resident for later requests of its shape (creating and releasing a
  // context costs far more than a step) until admission needs its memory; a forced request's
  // batch serves nobody else and goes at once
  for (auto it = s->batches.begin(); it != s->batches.end();) {
    Batch& b = it->second;
    if (b.slot_req.empty() && b.idle_since < 0) b.idle_since = now_s(s);
    if (!b.slot_req.empty()) b.idle_since = -1;
    if (b.slot_req.empty() && b.solo) {
      destroy_batch(s, b);
      it = s->batches.erase(it);
    } else {
      ++it;
    }
  }
  s->launched.clear();
  if (n_active) {
    int n = (int)s->queue.size();
    for (auto& kv : s->batches) n += (int)kv.second.slot_req.size();
    *n_active = n;
  }
  return first_err;
}

int tg_server_pump(tg_server* s, int* n_active) {
  const int rc = tg_server_pump_begin(s);
  if (rc) return rc;
  return tg_server_pump_end(s, n_active);
}

int tg_server_drain(tg_server* s, long long max_rounds) {
  if (!s) return TG_ERR_ARG;
  int first_err = TG_OK;
  if (s->round_open) {
    int n = 0;
    first_err = tg_server_pump_end(s, &n);
    if (n == 0) return first_err;
  }
  for (long long i = 0; max_rounds <= 0 || i < max_rounds; ++i) {
    int n = 0;
    const int rc = tg_server_pump(s, &n);
    if (rc && !first_err) first_err = rc;
    if (n == 0) return first_err;
  }
  return first_err ? first_err : TG_ERR_TIMEOUT;
}

int tg_server_poll(tg_server* s, long long id, tg_request_status* st) {
  if (!s || !st) return TG_ERR_ARG;
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return TG_ERR_ARG;
  *st = it->second.st;
  return TG_OK;
}

int tg_server_result(tg_server* s, long long id, double* host, size_t n) {
  if (!s || !host) return TG_ERR_ARG;
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return TG_ERR_ARG;
  Req& r = it->second;
  if (r.st.state != TG_REQ_DONE || !r.result) return TG_ERR_STATE;
  if (n != r.n_result) return TG_ERR_ARG;
  cudaSetDevice(s->dev);
  if (r.result_host) {
    wait_result(r);
    std::memcpy(host, r.result, sizeof(double) * n);
    return TG_OK;
  }
  // on the server's own non-blocking stream, after the result's copies, so that the batches'
  // streams go on
  cudaError_t e = r.result_ev ? cudaStreamWaitEvent(s->aux, r.result_ev, 0) : cudaSuccess;
  if (e == cudaSuccess) e = cudaMemcpyAsync(host, r.result, sizeof(double) * n, cudaMemcpyDeviceToHost, s->aux);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->aux);
  if (e != cudaSuccess) {
    s->err = std::string("result download: ") + cudaGetErrorString(e);
    return TG_ERR_CUDA;
  }
  return TG_OK;
}

int tg_server_release(tg_server* s, long long id) {
  if (!s) return TG_ERR_ARG;
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return TG_ERR_ARG;
  Req& r = it->second;
  cudaSetDevice(s->dev);
  if (r.result && r.result_host) {
    wait_result(r);
    s->pinned.put(r.result, r.n_result);
  } else if (r.result) {
    // freed on the server's stream once the result's copies have run (no host wait)
    if (r.result_ev) cudaStreamWaitEvent(s->aux, r.result_ev, 0);
    cudaFreeAsync(r.result, s->aux);
  }
  if (r.result_ev) {
    cudaEventDestroy(r.result_ev);
    r.result_ev = nullptr;
  }
  r.result = nullptr;
  r.n_result = 0;
  return TG_OK;
}

int tg_server_take_finished(tg_server* s, long long* ids, int max, int* n) {
  if (!s || !n || max < 0 || (max > 0 && !ids)) return TG_ERR_ARG;
  const int k = (int)std::min<size_t>((size_t)max, s->finished.size());
  for (int i = 0; i < k; ++i) ids[i] = s->finished[i];
  s->finished.erase(s->finished.begin(), s->finished.begin() + k);
  *n = k;
  return TG_OK;
}

int tg_server_stats_get(tg_server* s, tg_server_stats* st) {
  if (!s || !st) return TG_ERR_ARG;
  std::memset(st, 0, sizeof(*st));
  st->bytes_resident = s->bytes;
  st->bytes_peak = s->bytes_peak;
  st->n_batches = (int)s->batches.size();
  for (auto& kv : s->batches) st->n_running += (int)kv.second.slot_req.size();
  st->n_queued = (int)s->queue.size();
  st->rounds = s->rounds;
  st->request_steps = s->request_steps;
  st->graph_launches = s->graph_launches;
  st->eager_steps = s->eager_steps;
  return TG_OK;
}

int tg_server_batch_stats(tg_server* s, tg_batch_stat* out, int max, int* n) {
  if (!s || !n || max < 0 || (max > 0 && !out)) return TG_ERR_ARG;
  int k = 0;
  for (auto& kv : s->batches) {
    if (k >= max) break;
    const Batch& b = kv.second;
    tg_batch_stat& o = out[k++];
    std::memset(&o, 0, sizeof(o));
    for (int i = 0; i < 3; ++i) o.N[i] = b.c->cfg.N[i];
    o.basis = b.c->cfg.basis;
    o.physics = b.c->cfg.physics;
    o.precision = b.c->cfg.precision;
    o.capacity = b.B;
    o.n_active = (int)b.slot_req.size();
    o.step_ms_n_active = b.step_ms > 0 ? b.step_ms_nact : 0;
    o.step_ms = b.step_ms;
    o.device_ms = b.device_ms;
    o.steps = b.steps_run;
  }
  *n = k;
  return TG_OK;
}

double tg_server_clock(tg_server* s) { return s ? now_s(s) : 0.0; }

}  // extern "C"
