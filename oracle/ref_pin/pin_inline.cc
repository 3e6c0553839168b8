// Test infrastructure only (the oracle's checker, never part of the product): runs the reference's
// own inline wavenumber code -- trunk/lib/four/four_inline.h and trunk/lib/scft/scft_inline.h,
// included from the reference tree, not copied -- on a set of grids, one process (local_N1_start =
// 0), actual wavenumbers (globalvar_waveno_switch = 0), and prints a JSON document: per mode the
// grid wavenumbers, |K| and the multiplicity factor; per grid the aliased and dealiased radii
// (Min_radius_outside, Max_radius_inside), Approx_number_modes_in_shell; per anisotropy axis the
// parallel / perpendicular wavenumbers and polar angle per mode and the extents Anis_min_Kpll,
// Anis_max_Kpll, Anis_max_Krho_radius_inside.  The MPI, FFTW and blitz++ headers those files
// include are replaced by declaration-only stand-ins (oracle/ref_pin/stubs): no function of
// those libraries is called.  tests/golden/make_ref_inline_fixtures.py builds and runs it and
// stores the output as tests/golden/ref_inline.json, which tests/test_oracle_ref_inline.py
// compares with the oracle's restatement.
#include <cstdio>
#include <string>
#include <vector>

#include "four_inline.h"
#include "scft_inline.h"

int my_id = 0;
int numprocs = 1;
extern const int master_id = 0;
ptrdiff_t local_N1 = 0, local_N1_start = 0, local_N2 = 0, local_N2_start = 0;
MPI_Status status;
fftw_plan r2c_plan_FOUR, c2r_plan_FOUR, r2c_2d_plan_FOUR, c2r_2d_plan_FOUR, c2c_1d_forward_plan_FOUR,
    c2c_1d_inverse_plan_FOUR, r2c_plan_SCFT, c2r_plan_SCFT, sintr_plan_SCFT, costr_plan_SCFT, isintr_plan_SCFT,
    icostr_plan_SCFT, r2c_1d_plan_SCFT, c2r_1d_plan_SCFT;
int globalvar_fftw_original_switch = 1;
int globalvar_anisotropy_switch = 3;
int globalvar_waveno_switch = 0;

namespace {

struct Case {
  const char* basis;
  int n[3];
  double kf[3];
  bool modes;       // per-mode wavenumbers, |K| and multiplicity (small grids only)
  bool anis_modes;  // per-mode parallel / perpendicular wavenumbers and polar angle
};

void list_d(const char* key, const std::vector<double>& v, bool last = false) {
  std::printf("\"%s\": [", key);
  for (size_t i = 0; i < v.size(); ++i) std::printf("%s%.17g", i ? ", " : "", v[i]);
  std::printf("]%s", last ? "" : ", ");
}

void one(const Case& c, bool last) {
  const bool four = std::string(c.basis) == "FOUR";
  int N[4] = {0, c.n[0], c.n[1], c.n[2]};
  double kf[4] = {0.0, c.kf[0], c.kf[1], c.kf[2]};
  local_N1 = N[1];
  std::printf("{\"basis\": \"%s\", \"N\": [%d, %d, %d], \"kfactor\": [%.17g, %.17g, %.17g], ", c.basis, N[1], N[2],
              N[3], kf[1], kf[2], kf[3]);
  for (const char* al : {"ALIAS", "DEALIAS"}) {
    const std::string a(al);
    std::printf("\"min_radius_outside_%s\": %d, \"max_radius_inside_%s\": %d, ", al,
                four ? Min_radius_outside_FOUR(a, N, kf) : Min_radius_outside_SCFT(a, N, kf), al,
                four ? Max_radius_inside_FOUR(a, N, kf) : Max_radius_inside_SCFT(a, N, kf));
  }
  std::vector<double> approx;
  for (int r = 1; r <= 6; ++r)
    approx.push_back(four ? Approx_number_modes_in_shell_FOUR(N, r, kf) : Approx_number_modes_in_shell_SCFT(N, r, kf));
  list_d("approx_number_modes_in_shell_r1_6", approx);
  std::printf("\"anis\": [");
  for (int ax = 1; ax <= 3; ++ax) {
    globalvar_anisotropy_switch = ax;
    std::printf("%s{\"axis\": %d", ax > 1 ? ", " : "", ax);
    for (const char* al : {"ALIAS", "DEALIAS"}) {
      const std::string a(al);
      std::printf(", \"min_kpll_%s\": %.17g, \"max_kpll_%s\": %.17g, \"max_krho_inside_%s\": %d", al,
                  four ? Anis_min_Kpll_FOUR(a, N, kf) : Anis_min_Kpll_SCFT(a, N, kf), al,
                  four ? Anis_max_Kpll_FOUR(a, N, kf) : Anis_max_Kpll_SCFT(a, N, kf), al,
                  four ? Anis_max_Krho_radius_inside_FOUR(a, N, kf) : Anis_max_Krho_radius_inside_SCFT(a, N, kf));
    }
    if (c.anis_modes) {
      std::vector<double> kpll, kperp, polar;
      for (int l1 = 0; l1 < N[1]; ++l1)
        for (int l2 = 0; l2 < N[2]; ++l2)
          for (int l3 = 0; l3 <= N[3] / 2; ++l3) {
            kpll.push_back(four ? AnisKpll_FOUR(l1, l2, l3, N, kf) : AnisKpll_SCFT(l1, l2, l3, N, kf));
            kperp.push_back(four ? AnisKperp_FOUR(l1, l2, l3, N, kf) : AnisKperp_SCFT(l1, l2, l3, N, kf));
            polar.push_back(four ? AnisKvect_polar_angle_FOUR(l1, l2, l3, N, kf)
                                 : AnisKvect_polar_angle_SCFT(l1, l2, l3, N, kf));
          }
      std::printf(", ");
      list_d("kpll", kpll);
      list_d("kperp", kperp);
      list_d("polar_angle", polar, true);
    }
    std::printf("}");
  }
  std::printf("]");
  if (c.modes) {
    std::vector<double> kx, ky, kmag, mult;
    for (int l1 = 0; l1 < N[1]; ++l1) kx.push_back(four ? Get_kx_FOUR(l1, N) : Get_kx_SCFT(l1, N));
    for (int l2 = 0; l2 < N[2]; ++l2) ky.push_back(four ? Get_ky3D_FOUR(l2, N) : Get_ky3D_SCFT(l2, N));
    for (int l1 = 0; l1 < N[1]; ++l1)
      for (int l2 = 0; l2 < N[2]; ++l2)
        for (int l3 = 0; l3 <= N[3] / 2; ++l3) {
          kmag.push_back(four ? Kmagnitude_FOUR(l1, l2, l3, N, kf) : Kmagnitude_SCFT(l1, l2, l3, N, kf));
          mult.push_back(four ? Multiplicity_factor_FOUR(l1, l2, l3, N) : Multiplicity_factor_SCFT(l1, l2, l3, N));
        }
    std::printf(", ");
    list_d("kx", kx);
    list_d("ky", ky);
    list_d("kmag", kmag);
    list_d("multiplicity", mult, true);
  }
  std::printf("}%s\n", last ? "" : ",");
}

}  // namespace

int main() {
  const double pi = 3.14159265358979323846;
  const double r2 = 1.4142135623730951;
  const Case cases[] = {
      {"FOUR", {8, 8, 8}, {1.0, 1.0, 1.0}, true, false},
      {"FOUR", {10, 6, 8}, {1.0, 0.7, 2.3}, true, true},
      {"FOUR", {6, 16, 4}, {0.5, 1.0, 1.5}, true, false},
      {"FOUR", {64, 64, 64}, {1.0, 1.0, 1.0}, false, false},
      {"FOUR", {256, 256, 256}, {1.0, 1.0, 1.0}, false, false},
      {"FOUR", {32, 128, 64}, {2.0, 0.5, 1.0}, false, false},
      {"SCFT", {9, 8, 8}, {pi, pi / r2, pi / r2}, true, false},
      {"SCFT", {11, 6, 8}, {1.0, 1.0, 1.0}, true, false},
      {"SCFT", {8, 6, 10}, {1.0, 2.0, 0.5}, true, true},
      {"SCFT", {129, 256, 256}, {pi, pi / r2, pi / r2}, false, false},
      {"SCFT", {65, 128, 128}, {pi, pi / r2, pi / r2}, false, false},
      {"SCFT", {128, 256, 256}, {1.0, 1.0, 1.0}, false, false},
  };
  const int n = (int)(sizeof(cases) / sizeof(cases[0]));
  std::printf("{\"source\": \"trunk/lib/four/four_inline.h, trunk/lib/scft/scft_inline.h\", \"cases\": [\n");
  for (int i = 0; i < n; ++i) one(cases[i], i == n - 1);
  std::printf("]}\n");
  return 0;
}
