// A C++ driver of the reference's fluid loop (trunk/src/IFluid/Ifluid_main.cc:258-301) written
// against the mirror classes of tarang_b200.hpp, for the tests.
//
//   ifluid_driver <in.bin> <out.bin> N1 N2 N3 nu dt steps mode
//
// in.bin holds V1, V2, V3 in the reference layout (3 x 2 N1 N2 (N3/2+1) doubles).  The run is
// forced (constant energy supply on 2 < k <= 3 at eps = 0.1).  mode 0 calls the loop body
// method by method (Compute_force, Compute_nlin, Add_force, Compute_pressure, Get_dt,
// Time_advance, CV_Compute_totalenergy_diss with the isnan break); mode 1 runs the fused
// IncFluid::Step.  out.bin receives V1, V2, V3 after the steps, then the energy after each step,
// then the 16-shell flux and shell-to-shell tables of the final field (17 + 17 x 17 doubles).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "tarang_b200.hpp"

int main(int argc, char** argv) {
  if (argc != 10) {
    std::fprintf(stderr, "usage: %s in.bin out.bin N1 N2 N3 nu dt steps mode\n", argv[0]);
    return 2;
  }
  tg_config cfg;
  tg_config_default(&cfg);
  cfg.N[0] = std::atoi(argv[3]);
  cfg.N[1] = std::atoi(argv[4]);
  cfg.N[2] = std::atoi(argv[5]);
  cfg.nu = std::atof(argv[6]);
  cfg.dt = std::atof(argv[7]);
  const int steps = std::atoi(argv[8]), mode = std::atoi(argv[9]);
  cfg.force_kind = TG_FORCE_ENERGY_SUPPLY;
  const double fp[6] = {2.0, 3.0, 0.1, 0.0, 0.0, 0.0};
  for (int i = 0; i < 6; ++i) cfg.force_para[i] = fp[i];
  cfg.n_shells = 16;
  try {
    tarang_b200::IncFluid U(cfg);
    FILE* in = std::fopen(argv[1], "rb");
    if (!in) return 3;
    for (tarang_b200::Field* f : {&U.V1, &U.V2, &U.V3}) {
      std::vector<double>& d = f->data();
      if (std::fread(d.data(), sizeof(double), d.size(), in) != d.size()) return 3;
    }
    std::fclose(in);
    U.Upload();
    std::vector<double> energy;
    if (mode == 0) {
      for (int it = 0; it < steps; ++it) {
        U.Compute_force();
        U.Compute_nlin();
        U.Add_force();
        U.Compute_pressure();
        U.Tdt = U.Get_dt();
        U.Tnow = U.Tnow + U.Tdt;
        U.Time_advance();
        U.CV_Compute_totalenergy_diss();
        if (std::isnan(U.CV_total_energy)) {
          std::fprintf(stderr, "ERROR: Numerical Overflow\n");
          return 4;
        }
        energy.push_back(U.CV_total_energy);
      }
    } else {
      energy = U.Step(steps);
    }
    U.Download();
    U.Compute_flux();
    U.Compute_shell_tr();
    FILE* out = std::fopen(argv[2], "wb");
    if (!out) return 3;
    for (tarang_b200::Field* f : {&U.V1, &U.V2, &U.V3}) std::fwrite(f->data().data(), sizeof(double), f->data().size(), out);
    std::fwrite(energy.data(), sizeof(double), energy.size(), out);
    std::fwrite(U.flux_self.data(), sizeof(double), U.flux_self.size(), out);
    std::fwrite(U.shelltoshell_self.data(), sizeof(double), U.shelltoshell_self.size(), out);
    std::fclose(out);
    std::printf("ok %d steps, E = %.15e, t = %.6e\n", steps, energy.empty() ? 0.0 : energy.back(), U.Tnow);
  } catch (const tarang_b200::Error& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 5;
  }
  return 0;
}
