// Host side of the TMA primitives: tensor-map encoding through the driver entry point, cached.
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "tg_tma.cuh"

namespace tg {

namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
    else
      cudaGetLastError();
  });
  return fn;
}

using Key = std::tuple<const void*, unsigned long long, unsigned long long, unsigned long long, unsigned long long,
                       unsigned long long, unsigned, unsigned>;
std::mutex g_mu;
std::map<Key, CUtensorMap> g_maps;

}  // namespace

bool tma_map_3d(CUtensorMap* out, const void* base, unsigned long long d0, unsigned long long d1,
                unsigned long long d2, unsigned long long stride1, unsigned long long stride2, unsigned box0,
                unsigned box1) {
  // the rules cuTensorMapEncodeTiled checks, checked here first so a refusal is a fallback
  if (!base || ((uintptr_t)base & 15) != 0) return false;
  if (d0 == 0 || d1 == 0 || d2 == 0) return false;
  if ((stride1 & 15) != 0 || (stride2 & 15) != 0 || stride1 >= (1ull << 40) || stride2 >= (1ull << 40)) return false;
  if (box0 == 0 || box1 == 0 || box0 > 256 || box1 > 256 || ((box0 * 8u) & 15u) != 0) return false;
  const Key k{base, d0, d1, d2, stride1, stride2, box0, box1};
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_maps.find(k);
  if (it != g_maps.end()) {
    *out = it->second;
    return true;
  }
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  CUtensorMap m;
  std::memset(&m, 0, sizeof(m));
  const cuuint64_t dims[3] = {d0, d1, d2};
  const cuuint64_t strides[2] = {stride1, stride2};
  const cuuint32_t box[3] = {box0, box1, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = fn(&m, CU_TENSOR_MAP_DATA_TYPE_INT64, 3, const_cast<void*>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return false;
  if (g_maps.size() > 8192) g_maps.clear();
  g_maps.emplace(k, m);
  *out = m;
  return true;
}

}  // namespace tg
