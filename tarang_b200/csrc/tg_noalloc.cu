// tg_energy_noalloc: the energy / dissipation reduction of tg_energy for callers that cannot
// allocate device memory.  Its per-block partial sums live in a fixed file-scope device array
// instead of context-owned scratch, so the call allocates nothing.
#include <cuda.h>

#include <map>
#include <mutex>

#include "../../include/tarang_gpu.h"
#include "tg_spectral.cuh"

using namespace tg;

namespace {

constexpr int kBlocks = 148 * 8;          // reduction grid (one wave of 8 blocks per SM)
constexpr int kThreads = 256;
constexpr int kMaxFields = TG_NOALLOC_MAX_FIELDS;

// Scratch: [field][block][2] partial sums; 8 x 1184 x 2 doubles = 151,552 bytes.  Shared by
// every call on a device and left holding the last call's partials.
static __device__ __align__(256) double g_energy_partials[kMaxFields * kBlocks * 2];

// Device address of g_energy_partials per CUDA context (the host-side name is only a
// stand-in).  The address belongs to the context that loaded the module, so the cache is keyed
// on the context's unique id (cuCtxGetId never repeats within a process), not on the device
// ordinal: after cudaDeviceReset, or with a caller's own non-primary context current, the
// lookup runs again.
std::mutex g_partials_mu;
std::map<unsigned long long, double*> g_partials_addr;

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

template <typename Fn>
Fn driver_fn(const char* name) {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
    return reinterpret_cast<Fn>(p);
  cudaGetLastError();
  return nullptr;
}

// unique id of the context current on this thread; with none current yet, the symbol lookup
// (which initialises the runtime's primary context of the current device) runs first
int current_context_id(unsigned long long* id) {
  static CtxGetCurrentFn get_current = driver_fn<CtxGetCurrentFn>("cuCtxGetCurrent");
  static CtxGetIdFn get_id = driver_fn<CtxGetIdFn>("cuCtxGetId");
  if (!get_current || !get_id) return TG_ERR_CUDA;
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS) return TG_ERR_CUDA;
  if (ctx == nullptr) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_energy_partials) != cudaSuccess) {
      cudaGetLastError();
      return TG_ERR_CUDA;
    }
    if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return TG_ERR_CUDA;
  }
  if (get_id(ctx, id) != CUDA_SUCCESS) return TG_ERR_CUDA;
  return TG_OK;
}

struct DenseArgs {
  const cx<double>* f;   // n_fields consecutive fields, reference layout
  int nf;
  int N1, N2, M3;
  long long D;           // elements per field
  double kf0, kf1, kf2;
  double kkmax;          // Min_radius_outside
  double* part;
};

// Get_local_energy_FOUR (four_energy.cc:48-86) and Get_local_Sn_FOUR with n = 2
// (four_energy.cc:179-211) on the dense reference layout, per field
__global__ void __launch_bounds__(kThreads) k_energy_dense(DenseArgs a) {
  double e[kMaxFields], d[kMaxFields];
#pragma unroll
  for (int f = 0; f < kMaxFields; ++f) e[f] = d[f] = 0.0;
  const long long stride = (long long)gridDim.x * kThreads;
  for (long long idx = (long long)blockIdx.x * kThreads + threadIdx.x; idx < a.D; idx += stride) {
    const int l3 = (int)(idx % a.M3);
    const long long rr = idx / a.M3;
    const int l2 = (int)(rr % a.N2), l1 = (int)(rr / a.N2);
    const int kxi = l1 <= a.N1 / 2 ? l1 : l1 - a.N1;
    const int kyi = l2 <= a.N2 / 2 ? l2 : l2 - a.N2;
    const double kx = kxi * a.kf0, ky = kyi * a.kf1, kz = l3 * a.kf2;
    const double K2 = kx * kx + ky * ky + kz * kz;
    const double w = energy_weight_four(l1, l2, l3, a.N1, a.N2);
    const double m = (sqrt(K2) <= a.kkmax) ? mult_four(l1, l2, l3, a.N1, a.N2) * K2 : 0.0;
#pragma unroll
    for (int f = 0; f < kMaxFields; ++f) {
      if (f < a.nf) {
        const cx<double> u = a.f[(long long)f * a.D + idx];
        const double m2 = u.x * u.x + u.y * u.y;
        e[f] += w * m2;
        d[f] += m * m2;
      }
    }
  }
  __shared__ double red[kThreads / 32][2 * kMaxFields];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int f = 0; f < kMaxFields; ++f) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      e[f] += __shfl_down_sync(0xffffffffu, e[f], o);
      d[f] += __shfl_down_sync(0xffffffffu, d[f], o);
    }
    if (lane == 0) {
      red[wid][2 * f] = e[f];
      red[wid][2 * f + 1] = d[f];
    }
  }
  __syncthreads();
  // every block writes its own slot for every requested field: nothing has to start at zero
  if (threadIdx.x < 2 * a.nf) {
    double s = 0;
    for (int w2 = 0; w2 < kThreads / 32; ++w2) s += red[w2][threadIdx.x];
    const int f = threadIdx.x / 2, j = threadIdx.x % 2;
    a.part[((long long)f * kBlocks + blockIdx.x) * 2 + j] = s;
  }
}

// sums the partials of field blockIdx.x over the nb blocks of the first kernel, fixed order
__global__ void __launch_bounds__(kThreads) k_energy_dense_final(const double* part, int nb, double* out) {
  __shared__ double red[2][kThreads];
  const int f = blockIdx.x;
  double s0 = 0, s1 = 0;
  for (int b = threadIdx.x; b < nb; b += kThreads) {
    s0 += part[((long long)f * kBlocks + b) * 2];
    s1 += part[((long long)f * kBlocks + b) * 2 + 1];
  }
  red[0][threadIdx.x] = s0;
  red[1][threadIdx.x] = s1;
  __syncthreads();
  for (int o = kThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      red[0][threadIdx.x] += red[0][threadIdx.x + o];
      red[1][threadIdx.x] += red[1][threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[2 * f] = red[0][0];
    out[2 * f + 1] = 2.0 * red[1][0];  // CV_total_dissipation = 2 sum mult K^2 |A|^2 (Cvf.cc:385-397)
  }
}

// once per context, with that context current
int partials_address(double** out) {
  unsigned long long id = 0;
  int rc = current_context_id(&id);
  if (rc) return rc;
  std::lock_guard<std::mutex> lock(g_partials_mu);
  auto it = g_partials_addr.find(id);
  if (it == g_partials_addr.end()) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_energy_partials) != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return TG_ERR_CUDA;
    }
    if (g_partials_addr.size() >= 4096) g_partials_addr.clear();
    it = g_partials_addr.emplace(id, static_cast<double*>(p)).first;
  }
  *out = it->second;
  return TG_OK;
}

}  // namespace

extern "C" int tg_energy_noalloc(const double* d_fields, int n_fields, const int N[3], const double kfactor[3],
                                 int dealias, double* d_out, void* stream) {
  if (!d_fields || !d_out || !N || !kfactor) return TG_ERR_ARG;
  if (n_fields < 1 || n_fields > kMaxFields) return TG_ERR_ARG;   // scratch holds 8 fields
  // the fields are read as 16-byte complex values, the output written as doubles
  if (((uintptr_t)d_fields & 15) != 0 || ((uintptr_t)d_out & 7) != 0) return TG_ERR_ARG;
  if (N[0] < 2 || N[1] < 2 || N[2] < 2 || (N[2] & 1)) return TG_ERR_ARG;
  if (!(kfactor[0] > 0 && kfactor[1] > 0 && kfactor[2] > 0)) return TG_ERR_ARG;
  double* part = nullptr;
  int rc = partials_address(&part);
  if (rc) return rc;
  DenseArgs a{};
  a.f = reinterpret_cast<const cx<double>*>(d_fields);
  a.nf = n_fields;
  a.N1 = N[0];
  a.N2 = N[1];
  a.M3 = N[2] / 2 + 1;
  a.D = (long long)N[0] * N[1] * a.M3;
  a.kf0 = kfactor[0];
  a.kf1 = kfactor[1];
  a.kf2 = kfactor[2];
  // Min_radius_outside_(de)aliased_FOUR (four_inline.h:172-228)
  const int d = dealias ? 3 : 2;
  const double r0 = (N[0] / d) * kfactor[0], r1 = (N[1] / d) * kfactor[1], r2 = (N[2] / d) * kfactor[2];
  a.kkmax = ceil(sqrt(r0 * r0 + r1 * r1 + r2 * r2));
  a.part = part;
  long long nb = (a.D + kThreads - 1) / kThreads;
  if (nb > kBlocks) nb = kBlocks;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_energy_dense<<<(int)nb, kThreads, 0, s>>>(a);
  if (cudaGetLastError() != cudaSuccess) return TG_ERR_CUDA;
  k_energy_dense_final<<<n_fields, kThreads, 0, s>>>(part, (int)nb, d_out);
  if (cudaGetLastError() != cudaSuccess) return TG_ERR_CUDA;
  return TG_OK;
}
