// Serving loop (continuous batching of independent solves): see tg_server_impl below.
#include "tg_ctx.h"

extern "C" {

int tg_server_create(const tg_server_config* cfg, tg_server** out) {
  (void)cfg;
  if (out) *out = nullptr;
  return TG_ERR_UNSUPPORTED;
}
int tg_server_destroy(tg_server* srv) { return srv ? TG_ERR_UNSUPPORTED : TG_ERR_ARG; }
int tg_server_submit(tg_server* srv, const tg_request* req, long long* id) {
  (void)srv; (void)req; (void)id;
  return TG_ERR_UNSUPPORTED;
}
int tg_server_pump(tg_server* srv, int* n_active) {
  (void)srv; (void)n_active;
  return TG_ERR_UNSUPPORTED;
}
int tg_server_drain(tg_server* srv, long long max_rounds) {
  (void)srv; (void)max_rounds;
  return TG_ERR_UNSUPPORTED;
}
int tg_server_poll(tg_server* srv, long long id, tg_request_status* st) {
  (void)srv; (void)id; (void)st;
  return TG_ERR_UNSUPPORTED;
}
int tg_server_result(tg_server* srv, long long id, double* host, size_t n) {
  (void)srv; (void)id; (void)host; (void)n;
  return TG_ERR_UNSUPPORTED;
}
double tg_server_clock(tg_server* srv) {
  (void)srv;
  return 0.0;
}

}  // extern "C"
