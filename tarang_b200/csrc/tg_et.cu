// Energy transfer diagnostics: shell radii, flux Pi(R) and shell-to-shell transfer.
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

}  // namespace tg

extern "C" {

int tg_et_radii(tg_ctx* c, double* radii, int n) {
  if (!c || !radii) return TG_ERR_ARG;
  const int S = c->cfg.n_shells;
  if (S < 6) return set_err(c, TG_ERR_ARG, "energy transfer needs at least 6 shells");
  if (n < S + 1) return TG_ERR_ARG;
  std::vector<double> R = et_radii(c);
  for (int i = 0; i <= S; ++i) radii[i] = R[i];
  return TG_OK;
}

int tg_flux(tg_ctx* c, int kind, double* flux, int n) {
  (void)kind;
  (void)flux;
  (void)n;
  if (!c) return TG_ERR_ARG;
  return set_err(c, TG_ERR_UNSUPPORTED, "flux not built yet");
}

int tg_shell_to_shell(tg_ctx* c, int kind, double* tr, int n) {
  (void)kind;
  (void)tr;
  (void)n;
  if (!c) return TG_ERR_ARG;
  return set_err(c, TG_ERR_UNSUPPORTED, "shell-to-shell not built yet");
}

}  // extern "C"
