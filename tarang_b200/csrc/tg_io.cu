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
// Reduced-size files (output of Output_field_reduced, input of Init_cond_reduced) hold the
// low-wavenumber corner Nr of an N grid in the same text, without separators between values.
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

// Rows of a reduced-size array (Nr of N) in file order (Write_data_MPI with Nreduced,
// array_basic.cc:997-1175): FOUR x rows 0..Nr/2 then N-Nr/2+1..N-1; SCFT x rows 0..Nr-1;
// y rows (both bases) 0..Nr/2 then N-Nr/2+1..N-1.
std::vector<int> reduced_rows(int N, int Nr, bool fourier) {
  std::vector<int> r;
  if (!fourier) {
    for (int i = 0; i < Nr; ++i) r.push_back(i);
    return r;
  }
  for (int i = 0; i <= Nr / 2; ++i) r.push_back(i);
  for (int i = N - Nr / 2 + 1; i < N; ++i) r.push_back(i);
  return r;
}

bool valid_reduced(const int N[3], const int Nr[3], int basis) {
  if (basis != TG_FOUR && basis != TG_SCFT) return false;
  if (Nr[0] < 1 || Nr[0] > N[0] || Nr[1] < 2 || Nr[1] > N[1] || Nr[2] < 2 || Nr[2] > N[2]) return false;
  if ((Nr[1] & 1) || (Nr[2] & 1)) return false;
  if (basis == TG_FOUR && ((Nr[0] & 1) || Nr[0] < 2)) return false;
  return true;
}

// V3 (or W3) for kz >= 1 from i K . V = 0 with the vector's first two components
// (IncVF::Last_component field_k_fns.cc:79-87); the kz = 0 plane is kept
void rebuild_last(const int N[3], int basis, const double kfactor[3], const cplx* V1, const cplx* V2, cplx* A) {
  const int N1 = N[0], N2 = N[1], M3 = N[2] / 2 + 1;
  const bool four = (basis == TG_FOUR);
  for (int i = 0; i < N1; ++i)
    for (int j = 0; j < N2; ++j) {
      const size_t row = ((size_t)i * N2 + j) * M3;
      const int kx = geo_k(i, N1, four), ky = geo_k(j, N2, true);
      for (int k = 1; k < M3; ++k) {
        const cplx dx = four ? cplx(0, kx * kfactor[0]) * V1[row + k] : cplx(kx * kfactor[0], 0) * V1[row + k];
        const cplx temp = dx + cplx(0, ky * kfactor[1]) * V2[row + k];
        A[row + k] = temp / cplx(0, -k * kfactor[2]);
      }
    }
}

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
      for (int i = 0; i < N1; ++i)
        for (int j = 0; j < N2; ++j) A[((size_t)i * N2 + j) * M3] = plane[(size_t)i * N2 + j];
      rebuild_last(N, basis, kfactor, V1, V2, A);
    } else if (!read_values(in, A, D)) {
      return TG_ERR_ARG;
    }
  }
  return TG_OK;
}

int tg_write_field_file_reduced(const char* path, double time, const int N[3], const int Nr[3], int basis,
                                int n_fields, const double* const* fields, int vx_vy, int append) {
  if (!path || !N || !Nr || !fields || n_fields < 1 || n_fields > 8) return TG_ERR_ARG;
  if (N[0] < 1 || N[1] < 1 || N[2] < 2 || (N[2] & 1) || !valid_reduced(N, Nr, basis)) return TG_ERR_ARG;
  if (vx_vy && n_fields < 3) return TG_ERR_ARG;
  for (int f = 0; f < n_fields; ++f)
    if (!fields[f]) return TG_ERR_ARG;
  std::ofstream out(path, append ? std::ios::app : std::ios::trunc);
  if (!out.is_open()) return TG_ERR_ARG;
  out.precision(12);
  const int N2 = N[1], M3 = N[2] / 2 + 1, K = Nr[2] / 2;
  const std::vector<int> xs = reduced_rows(N[0], Nr[0], basis == TG_FOUR), ys = reduced_rows(N2, Nr[1], true);
  out << "%% Time = " << time << std::endl;
  for (int f = 0; f < n_fields; ++f) {
    const cplx* A = reinterpret_cast<const cplx*>(fields[f]);
    const bool plane = vx_vy && (f == 2 || f == 5);  // Write_data_kz0plane_MPI (array_basic.cc:1176-1347)
    for (int i : xs)
      for (int j : ys) {
        const size_t row = ((size_t)i * N2 + j) * M3;
        for (int k = 0; k <= (plane ? 0 : K); ++k) out << A[row + k];
      }
    out << std::endl << std::endl;
  }
  out.flush();
  return out.good() ? TG_OK : TG_ERR_ARG;
}

int tg_read_field_file_reduced(const char* path, const int N[3], const int Nr[3], int basis, const double kfactor[3],
                               int n_fields, double* const* fields, int vx_vy) {
  if (!path || !N || !Nr || !fields || n_fields < 1 || n_fields > 8) return TG_ERR_ARG;
  if (N[0] < 1 || N[1] < 1 || N[2] < 2 || (N[2] & 1) || !valid_reduced(N, Nr, basis)) return TG_ERR_ARG;
  if (vx_vy && (n_fields < 3 || !kfactor)) return TG_ERR_ARG;
  for (int f = 0; f < n_fields; ++f)
    if (!fields[f]) return TG_ERR_ARG;
  std::ifstream in(path);
  if (!in.is_open()) return TG_ERR_ARG;
  const int N1 = N[0], N2 = N[1], M3 = N[2] / 2 + 1, K = Nr[2] / 2;
  const bool four = (basis == TG_FOUR);
  const std::vector<int> xs = reduced_rows(N1, Nr[0], four), ys = reduced_rows(N2, Nr[1], true);
  const size_t D = (size_t)N1 * N2 * M3;
  for (int f = 0; f < n_fields; ++f) {
    cplx* A = reinterpret_cast<cplx*>(fields[f]);
    for (size_t q = 0; q < D; ++q) A[q] = 0;
    const bool plane = vx_vy && (f == 2 || f == 5);
    const int nk = plane ? 1 : K + 1;
    std::vector<cplx> buf(xs.size() * ys.size() * nk);
    if (!read_values(in, buf.data(), buf.size())) return TG_ERR_ARG;
    // Read_data_MPI with Nreduced (array_basic.cc:388-601): the kx = +Nr1/2 (FOUR) and
    // ky = +Nr2/2 rows of the file also fill the -Nr/2 rows of the larger array
    auto put = [&](int i, int j, const cplx* v) {
      const size_t row = ((size_t)i * N2 + j) * M3;
      for (int k = 0; k < nk; ++k) A[row + k] = v[k];
    };
    for (size_t a = 0; a < xs.size(); ++a)
      for (size_t b = 0; b < ys.size(); ++b) {
        const cplx* v = &buf[(a * ys.size() + b) * nk];
        const int i = xs[a], j = ys[b];
        const bool xny = four && i == Nr[0] / 2 && Nr[0] < N1, yny = j == Nr[1] / 2 && Nr[1] < N2;
        put(i, j, v);
        if (xny) put(N1 - Nr[0] / 2, j, v);
        if (yny) put(i, N2 - Nr[1] / 2, v);
        if (xny && yny) put(N1 - Nr[0] / 2, N2 - Nr[1] / 2, v);
      }
    if (plane) {
      rebuild_last(N, basis, kfactor, reinterpret_cast<const cplx*>(fields[f - 2]),
                   reinterpret_cast<const cplx*>(fields[f - 1]), A);
    }
  }
  return TG_OK;
}

}  // extern "C"
