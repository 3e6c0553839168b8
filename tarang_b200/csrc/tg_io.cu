// Field files in the reference's text format (host only; no device code).
//
// Writer: IncFluid::Output_field / Output_field_scalar (output_field.cc:43-108) with
// Write_data_MPI and Write_data_kz0plane_MPI (array_basic.cc:814-898) on one rank: the line
// "%% Time = t", then every array as "(re,im) " per mode in [l1][l2][l3] order, each array
// followed by two newlines, on a stream of precision MY_PRECISION = 12 (file_operations.cc:
// 222-236, extern_def_vars.h:78).  With vx_vy = 1 the third component is written as its kz = 0
// plane only (each vector's: V3, and W3 of MHD).
// Reader: IncFluid::Init_cond (init_cond_field.cc:47-88) with Read_data_MPI /
// Read_data_kz0plane_MPI (array_basic.cc:294-383): the same values read with the stream's
// complex extractor; with vx_vy = 1, V3 for kz >= 1 is rebuilt from incompressibility
// (IncVF::Last_component field_k_fns.cc:79-87, DxVx_plus_DyVy universal_inline.h:435-451).
// Lines that start with '%' are skipped, so a written file reads back.
#include <complex>
#include <fstream>
#include <string>
#include <vector>

#include "../../include/tarang_gpu.h"

namespace {

using cplx = std::complex<double>;

// next non-comment token stream position: skips whitespace and whole lines starting with '%'
void skip_comments(std::istream& in) {
  for (;;) {
    in >> std::ws;
    if (in.peek() != '%') return;
    std::string line;
    std::getline(in, line);
  }
}

bool read_values(std::istream& in, cplx* out, size_t n) {
  for (size_t i = 0; i < n; ++i) {
    skip_comments(in);
    if (!(in >> out[i])) return false;
  }
  return true;
}

int geo_k(int l, int N, bool fourier) { return (!fourier || l <= N / 2) ? l : l - N; }

}  // namespace

extern "C" {

int tg_write_field_file(const char* path, double time, const int N[3], int n_fields,
                        const double* const* fields, int vx_vy, int append) {
  if (!path || !N || !fields || n_fields < 1 || n_fields > 8) return TG_ERR_ARG;
  if (N[0] < 1 || N[1] < 1 || N[2] < 2 || (N[2] & 1)) return TG_ERR_ARG;
  if (vx_vy && n_fields < 3) return TG_ERR_ARG;
  for (int f = 0; f < n_fields; ++f)
    if (!fields[f]) return TG_ERR_ARG;
  std::ofstream out(path, append ? std::ios::app : std::ios::trunc);
  if (!out.is_open()) return TG_ERR_ARG;
  out.precision(12);
  const int N1 = N[0], N2 = N[1], M3 = N[2] / 2 + 1;
  out << "%% Time = " << time << std::endl;
  for (int f = 0; f < n_fields; ++f) {
    const cplx* A = reinterpret_cast<const cplx*>(fields[f]);
    const bool plane = vx_vy && (f == 2 || f == 5);  // Write_data_kz0plane_MPI
    for (int i = 0; i < N1; ++i)
      for (int j = 0; j < N2; ++j) {
        const size_t row = ((size_t)i * N2 + j) * M3;
        if (plane) {
          out << A[row] << " ";
        } else {
          for (int k = 0; k < M3; ++k) out << A[row + k] << " ";
        }
      }
    out << std::endl << std::endl;
  }
  out.flush();
  return out.good() ? TG_OK : TG_ERR_ARG;
}

int tg_read_field_file(const char* path, const int N[3], int basis, const double kfactor[3], int n_fields,
                       double* const* fields, int vx_vy) {
  if (!path || !N || !fields || n_fields < 1 || n_fields > 8) return TG_ERR_ARG;
  if (N[0] < 1 || N[1] < 1 || N[2] < 2 || (N[2] & 1)) return TG_ERR_ARG;
  if (basis != TG_FOUR && basis != TG_SCFT) return TG_ERR_ARG;
  if (vx_vy && (n_fields < 3 || !kfactor)) return TG_ERR_ARG;
  for (int f = 0; f < n_fields; ++f)
    if (!fields[f]) return TG_ERR_ARG;
  std::ifstream in(path);
  if (!in.is_open()) return TG_ERR_ARG;
  const int N1 = N[0], N2 = N[1], M3 = N[2] / 2 + 1;
  const size_t D = (size_t)N1 * N2 * M3;
  for (int f = 0; f < n_fields; ++f) {
    cplx* A = reinterpret_cast<cplx*>(fields[f]);
    if (vx_vy && (f == 2 || f == 5)) {
      // the kz = 0 plane, then kz >= 1 from i K . V = 0 with the vector's first two components
      std::vector<cplx> plane((size_t)N1 * N2);
      if (!read_values(in, plane.data(), plane.size())) return TG_ERR_ARG;
      const cplx* V1 = reinterpret_cast<const cplx*>(fields[f - 2]);
      const cplx* V2 = reinterpret_cast<const cplx*>(fields[f - 1]);
      const bool four = (basis == TG_FOUR);
      for (int i = 0; i < N1; ++i)
        for (int j = 0; j < N2; ++j) {
          const size_t row = ((size_t)i * N2 + j) * M3;
          A[row] = plane[(size_t)i * N2 + j];
          const int kx = geo_k(i, N1, four), ky = geo_k(j, N2, true);
          for (int k = 1; k < M3; ++k) {
            const cplx dx = four ? cplx(0, kx * kfactor[0]) * V1[row + k] : cplx(kx * kfactor[0], 0) * V1[row + k];
            const cplx temp = dx + cplx(0, ky * kfactor[1]) * V2[row + k];
            A[row + k] = temp / cplx(0, -k * kfactor[2]);
          }
        }
    } else if (!read_values(in, A, D)) {
      return TG_ERR_ARG;
    }
  }
  return TG_OK;
}

}  // extern "C"
