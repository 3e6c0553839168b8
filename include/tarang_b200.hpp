/*
 * tarang_b200.hpp -- header-only C++ host classes over the C ABI (tarang_gpu.h) that keep the
 * names and call order of Tarang-4.0's solver objects, so a C++ driver written against the
 * reference's IncFluid / IncVF / IncSF / CVF / CSF interface ports by changing its declarations:
 *
 *   reference (trunk/lib/...)                              here
 *   CVF   fields/Cvf.h:82-445   V1..V3, CV_Forward/Inverse_transform (:292-343),
 *                               CV_Compute_totalenergy_diss (:349),
 *                               CV_Compute_shell_spectrum (:364), CV_total_energy,
 *                               CV_total_dissipation, CV_shell_ek1..3, CV_shell_dissk   CVF
 *   CSF   fields/Csf.h:79-327   F, CS_Compute_totalenergy_diss, CS_Compute_shell_spectrum,
 *                               CS_total_energy, CS_shell_ek, CS_shell_dissk             CSF
 *   IncVF IncFlow/IncVF.h:75-531  nlin1..3 (Nlin.h:51-88), Compute_nlin (:274-287),
 *                               Compute_pressure (:289), Dealias (:202-215),
 *                               Compute_flux (:404-409), Compute_shell_tr (:418-423),
 *                               Compute_force_feed_shell; flux_self, shelltoshell_self,
 *                               forceV_shell (EnergyTr.h:182-226)                        IncVF
 *   IncSF IncFlow/IncSF.h:66-142  the scalar T of a passive-scalar or convection run      IncSF
 *   IncFluid IncFluid/IncFluid.h:82-606  Compute_force (:246-249), Add_force (:302-305),
 *                               Compute_rhs (:309-314), Get_dt (:317-320), Time_advance
 *                               (:351-356), Tnow, Tdt; Get_Nusselt_no (nusselt.cc:53-89)  IncFluid
 *
 * Where the reference's objects own blitz arrays in host memory, here the state lives on the
 * GPU in a tg_ctx owned by IncFluid; the V1..V3 / F / nlin host arrays of these classes are the
 * reference layout (complex<double> interleaved, [l1][l2][l3], l3 <= N3/2) and move to and from
 * the device with Upload() / Download().  A method that computes on the device leaves its
 * result on the device: call Download() where the reference would read V1..V3 afterwards.
 * Results that the reference keeps as member arrays (energies, spectra, fluxes) are copied to
 * the members of the same names.  Every failing call throws tarang_b200::Error with the
 * status code and the context's message (the reference exits or prints instead).
 *
 * Requires C++17 and linking with libtarang_gpu.so.
 */
#ifndef TARANG_B200_HPP
#define TARANG_B200_HPP

#include <cmath>
#include <cstddef>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "tarang_gpu.h"

namespace tarang_b200 {

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& what) : std::runtime_error(what), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

inline void check(int rc, const tg_ctx* c, const char* what) {
  if (rc == TG_OK) return;
  std::string m = std::string(what) + " failed (status " + std::to_string(rc) + ")";
  if (c) {
    const char* e = tg_last_error(c);
    if (e && *e) m += ": " + std::string(e);
  }
  throw Error(rc, m);
}

// The device-side state of one solve (an IncFluid with its fields): owns the tg_ctx.
class Context {
 public:
  explicit Context(const tg_config& cfg) : cfg_(cfg) { check(tg_ctx_create(&cfg_, &h_), nullptr, "tg_ctx_create"); }
  ~Context() {
    if (h_) tg_ctx_destroy(h_);
  }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;

  tg_ctx* get() const { return h_; }
  const tg_config& config() const { return cfg_; }
  int N(int i) const { return cfg_.N[i]; }
  // doubles per dense field in the reference layout: 2 N1 N2 (N3/2 + 1)
  size_t field_doubles() const { return 2 * (size_t)cfg_.N[0] * cfg_.N[1] * (cfg_.N[2] / 2 + 1); }
  void synchronize() { check(tg_synchronize(h_), h_, "tg_synchronize"); }

 private:
  tg_config cfg_;
  tg_ctx* h_ = nullptr;
};

// A field of the reference layout held on the host (allocated on first use), bound to one
// context field id.
class Field {
 public:
  Field() = default;
  Field(Context* c, int id) : ctx_(c), id_(id) {}
  std::vector<double>& data() {
    if (data_.empty()) data_.assign(ctx_->field_doubles(), 0.0);
    return data_;
  }
  // complex<double> entry (l1, l2, l3) as (re, im) in the reference layout
  double* at(int l1, int l2, int l3) {
    const size_t M3 = (size_t)ctx_->N(2) / 2 + 1;
    return data().data() + 2 * (((size_t)l1 * ctx_->N(1) + l2) * M3 + l3);
  }
  void Upload() {
    std::vector<double>& d = data();
    check(tg_field_upload(ctx_->get(), id_, d.data(), d.size()), ctx_->get(), "tg_field_upload");
  }
  void Download() {
    std::vector<double>& d = data();
    check(tg_field_download(ctx_->get(), id_, d.data(), d.size()), ctx_->get(), "tg_field_download");
  }
  int id() const { return id_; }

 private:
  Context* ctx_ = nullptr;
  int id_ = -1;
  std::vector<double> data_;
};

namespace detail {
// Forward_transform_array / Inverse_transform_array (universal_tr.cc:66-146) of a host array
// through a work field of the context
inline void transform(Context* c, std::vector<double>& a, bool forward, int parity) {
  int w = -1;
  check(tg_field_alloc(c->get(), &w), c->get(), "tg_field_alloc");
  try {
    check(tg_field_upload(c->get(), w, a.data(), a.size()), c->get(), "tg_field_upload");
    check(forward ? tg_forward_transform(c->get(), w, parity) : tg_inverse_transform(c->get(), w, parity), c->get(),
          forward ? "tg_forward_transform" : "tg_inverse_transform");
    check(tg_field_download(c->get(), w, a.data(), a.size()), c->get(), "tg_field_download");
  } catch (...) {
    tg_field_free(c->get(), w);
    throw;
  }
  check(tg_field_free(c->get(), w), c->get(), "tg_field_free");
}
inline std::vector<double> spectrum_out(Context* c) {
  // kmax_outside + 1 entries suffice; the largest grid radius bounds it from above
  const double n1 = c->N(0), n2 = c->N(1), n3 = c->N(2);
  const double k0 = c->config().kfactor[0], k1 = c->config().kfactor[1], k2 = c->config().kfactor[2];
  const double r = std::sqrt((n1 * k0) * (n1 * k0) + (n2 * k1) * (n2 * k1) + (n3 * k2) * (n3 * k2));
  return std::vector<double>((size_t)r + 4, 0.0);
}
}  // namespace detail

// CVF: a complex vector field (V1, V2, V3) of a context, group 0 (U) or 1 (W of MHD).
class CVF {
 public:
  CVF(Context* c, int group)
      : ctx_(c),
        group_(group),
        V1(c, group == 1 ? TG_W1 : TG_V1),
        V2(c, group == 1 ? TG_W2 : TG_V2),
        V3(c, group == 1 ? TG_W3 : TG_V3) {}

  void Upload() {
    V1.Upload();
    V2.Upload();
    V3.Upload();
  }
  void Download() {
    V1.Download();
    V2.Download();
    V3.Download();
  }

  // In place on the host arrays (real space in the reference's packed layout <-> spectrum):
  // FOUR: Fourier transforms; SCFT: SFT(V1), CFT(V2), CFT(V3) and their inverses (Cvf.h:292-343)
  void CV_Forward_transform() {
    const bool scft = ctx_->config().basis == TG_SCFT;
    detail::transform(ctx_, V1.data(), true, scft ? 1 : 0);
    detail::transform(ctx_, V2.data(), true, 0);
    detail::transform(ctx_, V3.data(), true, 0);
  }
  void CV_Inverse_transform() {
    const bool scft = ctx_->config().basis == TG_SCFT;
    detail::transform(ctx_, V1.data(), false, scft ? 1 : 0);
    detail::transform(ctx_, V2.data(), false, 0);
    detail::transform(ctx_, V3.data(), false, 0);
  }

  // of the device state
  void CV_Compute_totalenergy_diss() {
    check(tg_energy(ctx_->get(), group_, &CV_total_energy, &CV_total_dissipation), ctx_->get(), "tg_energy");
  }
  void CV_Compute_shell_spectrum() {
    std::vector<double> d = detail::spectrum_out(ctx_);
    const int n = (int)d.size();
    std::vector<double> ek(3 * (size_t)n, 0.0);
    check(tg_shell_spectrum(ctx_->get(), group_, ek.data(), d.data(), n), ctx_->get(), "tg_shell_spectrum");
    CV_shell_ek1.assign(ek.begin(), ek.begin() + n);
    CV_shell_ek2.assign(ek.begin() + n, ek.begin() + 2 * n);
    CV_shell_ek3.assign(ek.begin() + 2 * n, ek.end());
    CV_shell_ek.resize(n);
    for (int i = 0; i < n; ++i) CV_shell_ek[i] = CV_shell_ek1[i] + CV_shell_ek2[i] + CV_shell_ek3[i];
    CV_shell_dissk = std::move(d);
  }

  Context* context() const { return ctx_; }
  int group() const { return group_; }

 protected:
  Context* ctx_;
  int group_;

 public:
  Field V1, V2, V3;
  double CV_total_energy = 0, CV_total_dissipation = 0;
  std::vector<double> CV_shell_ek1, CV_shell_ek2, CV_shell_ek3, CV_shell_ek, CV_shell_dissk;
};

// CSF: a complex scalar field F (the temperature / passive scalar, group 2).
class CSF {
 public:
  explicit CSF(Context* c) : ctx_(c), F(c, TG_T) {}
  void Upload() { F.Upload(); }
  void Download() { F.Download(); }
  // SCFT: SFT (the temperature's parity); FOUR: Fourier
  void CS_Forward_transform() { detail::transform(ctx_, F.data(), true, ctx_->config().basis == TG_SCFT ? 1 : 0); }
  void CS_Inverse_transform() { detail::transform(ctx_, F.data(), false, ctx_->config().basis == TG_SCFT ? 1 : 0); }
  void CS_Compute_totalenergy_diss() {
    check(tg_energy(ctx_->get(), 2, &CS_total_energy, &CS_total_dissipation), ctx_->get(), "tg_energy");
  }
  void CS_Compute_shell_spectrum() {
    std::vector<double> d = detail::spectrum_out(ctx_);
    CS_shell_ek.assign(d.size(), 0.0);
    check(tg_shell_spectrum(ctx_->get(), 2, CS_shell_ek.data(), d.data(), (int)d.size()), ctx_->get(),
          "tg_shell_spectrum");
    CS_shell_dissk = std::move(d);
  }

 protected:
  Context* ctx_;

 public:
  Field F;
  double CS_total_energy = 0, CS_total_dissipation = 0;
  std::vector<double> CS_shell_ek, CS_shell_dissk;
};

// IncSF: the scalar of a passive-scalar or convection run, with its nlin.
class IncSF : public CSF {
 public:
  explicit IncSF(Context* c) : CSF(c), nlin(c, TG_TNLIN) {}
  Field nlin;
};

// IncVF: an incompressible vector field with its nonlinear term and energy-transfer tables.
class IncVF : public CVF {
 public:
  IncVF(Context* c, int group)
      : CVF(c, group),
        nlin1(c, group == 1 ? TG_WNLIN1 : TG_NLIN1),
        nlin2(c, group == 1 ? TG_WNLIN2 : TG_NLIN2),
        nlin3(c, group == 1 ? TG_WNLIN3 : TG_NLIN3),
        F(c, TG_PRESSURE) {}

  // nlin = FT(u.grad u) (and the W / T parts of the same context), dealiased (IncVF.h:274-287);
  // the overloads name the fields the reference passes; the context computes them all at once
  void Compute_nlin() { check(tg_compute_nlin(ctx_->get()), ctx_->get(), "tg_compute_nlin"); }
  void Compute_nlin(IncVF&) { Compute_nlin(); }
  void Compute_nlin(IncSF&) { Compute_nlin(); }
  void Compute_nlin(IncVF&, IncSF&) { Compute_nlin(); }
  void Compute_pressure() { check(tg_compute_pressure(ctx_->get()), ctx_->get(), "tg_compute_pressure"); }
  // The device state keeps only the 2/3-dealiased modes (every upload drops the rest), so the
  // state is dealiased at all times; Dealias() checks nothing further.
  void Dealias() {}
  void Dealias(IncVF&) {}
  void Dealias(IncSF&) {}

  // energy transfer over the context's n_shells spheres / shells (EnergyTr.cc:136-160 radii)
  void Compute_flux(int kind = TG_ET_UU) {
    const int S = ctx_->config().n_shells;
    flux_self.assign((size_t)S + 1, 0.0);
    check(tg_flux(ctx_->get(), kind, flux_self.data(), S + 1), ctx_->get(), "tg_flux");
  }
  void Compute_shell_tr(int kind = TG_ET_UU) {
    const int S = ctx_->config().n_shells;
    shelltoshell_self.assign((size_t)(S + 1) * (S + 1), 0.0);
    check(tg_shell_to_shell(ctx_->get(), kind, shelltoshell_self.data(), S + 1), ctx_->get(), "tg_shell_to_shell");
  }
  void Compute_force_feed_shell() {
    const int S = ctx_->config().n_shells;
    forceV_shell.assign((size_t)S + 1, 0.0);
    check(tg_force_feed_group(ctx_->get(), group_, forceV_shell.data(), S + 1), ctx_->get(), "tg_force_feed_group");
  }
  std::vector<double> ET_shell_radii() {
    const int S = ctx_->config().n_shells;
    std::vector<double> r((size_t)S + 1, 0.0);
    check(tg_et_radii(ctx_->get(), r.data(), S + 1), ctx_->get(), "tg_et_radii");
    return r;
  }

  Field nlin1, nlin2, nlin3;
  Field F;  // the pressure (NLIN's CSF F)
  std::vector<double> flux_self, shelltoshell_self, forceV_shell;
};

// IncFluid: the velocity field of a solve and its time stepping; owns the context.  For MHD the
// magnetic field is W(), for a passive scalar or convection the scalar is T(): they live in the
// same context, and the methods that take them advance them together as the reference's
// overloads do.
class IncFluid : public IncVF {
 public:
  explicit IncFluid(const tg_config& cfg) : IncFluid(new Context(cfg)) {}
  ~IncFluid() { delete own_; }
  IncFluid(const IncFluid&) = delete;
  IncFluid& operator=(const IncFluid&) = delete;

  IncVF& W() { return W_; }
  IncSF& T() { return T_; }

  void Compute_force() { check(tg_compute_force(ctx_->get()), ctx_->get(), "tg_compute_force"); }
  void Compute_force(IncVF&) { Compute_force(); }
  void Compute_force(IncSF&) { Compute_force(); }
  void Add_force() { check(tg_add_force(ctx_->get()), ctx_->get(), "tg_add_force"); }
  void Add_force(IncVF&) { Add_force(); }
  void Add_force(IncSF&) { Add_force(); }
  void Compute_rhs() { check(tg_compute_rhs(ctx_->get()), ctx_->get(), "tg_compute_rhs"); }
  void Compute_rhs(IncVF&) { Compute_rhs(); }
  void Compute_rhs(IncSF&) { Compute_rhs(); }
  double Get_dt() {
    double dt = 0;
    check(tg_get_dt(ctx_->get(), &dt), ctx_->get(), "tg_get_dt");
    return dt;
  }
  double Get_dt(IncVF&) { return Get_dt(); }
  double Get_dt(IncSF&) { return Get_dt(); }
  void Time_advance() { check(tg_time_advance(ctx_->get()), ctx_->get(), "tg_time_advance"); }
  void Time_advance(IncVF&) { Time_advance(); }
  void Time_advance(IncSF&) { Time_advance(); }
  void Time_advance(IncVF&, IncSF&) { Time_advance(); }
  double Get_Nusselt_no() {
    double nu = 0;
    check(tg_nusselt(ctx_->get(), &nu), ctx_->get(), "tg_nusselt");
    return nu;
  }

  // n iterations of the loop body of Ifluid_main.cc:261-286 fused on the device (one captured
  // CUDA graph per step); the total energy after each step is returned.  Tnow advances by the
  // steps' dt.  Throws Error(TG_ERR_NONFINITE) where the reference breaks on isnan(E).
  std::vector<double> Step(int n) {
    std::vector<double> E((size_t)(n > 0 ? n : 0), 0.0);
    check(tg_step(ctx_->get(), n, E.data()), ctx_->get(), "tg_step");
    long long steps = 0;
    check(tg_time(ctx_->get(), &Tnow, &steps), ctx_->get(), "tg_time");
    return E;
  }

  double Tnow = 0, Tdt = 0;

 private:
  explicit IncFluid(Context* c) : IncVF(c, 0), own_(c), W_(c, 1), T_(c) { Tdt = c->config().dt; }
  Context* own_;
  IncVF W_;
  IncSF T_;
};

}  // namespace tarang_b200

#endif  // TARANG_B200_HPP
