// Tensor-map encoding for the TMA pencil kernels.
//
// cuTensorMapEncodeTiled is a driver entry point; it is fetched through the
// runtime (cudaGetDriverEntryPoint) so the library does not link libcuda and
// still loads on hosts without a GPU driver.  Encoded maps are cached by every
// parameter they encode (base address, extents, element size, box), so a cached
// map is valid for any buffer that matches its key, including a freed and
// re-allocated one at the same address.
#include <cudaTypedefs.h>

#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>

#include "kernels.h"

namespace sb200 {

namespace {

using Key = std::tuple<uintptr_t, int64_t, int64_t, int64_t, int, int, int>;

std::mutex g_mu;
std::map<Key, std::unique_ptr<CUtensorMap>>* g_cache = nullptr;
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

PFN_cuTensorMapEncodeTiled_v12000 encoder() {
    if (!g_encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    return g_encode;
}

}  // namespace

int tensor_map_3d(CUtensorMap* out, const void* base, int64_t nx, int64_t ny, int64_t nz,
                  int esize, int box_x, int box_y) {
    const Key key{reinterpret_cast<uintptr_t>(base), nx, ny, nz, esize, box_x, box_y};
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_cache) g_cache = new std::map<Key, std::unique_ptr<CUtensorMap>>();
    auto it = g_cache->find(key);
    if (it != g_cache->end()) {
        *out = *it->second;
        return 0;
    }

    auto enc = encoder();
    if (!enc) return -1;
    if (g_cache->size() > 4096) g_cache->clear();  // bound host memory for long sessions

    auto map = std::make_unique<CUtensorMap>();
    std::memset(map.get(), 0, sizeof(CUtensorMap));
    const cuuint64_t dims[3] = {static_cast<cuuint64_t>(nx), static_cast<cuuint64_t>(ny),
                                static_cast<cuuint64_t>(nz)};
    const cuuint64_t strides[2] = {static_cast<cuuint64_t>(nx) * esize,
                                   static_cast<cuuint64_t>(nx) * ny * esize};
    const cuuint32_t box[3] = {static_cast<cuuint32_t>(box_x), static_cast<cuuint32_t>(box_y), 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUtensorMapDataType dt =
        esize == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_UINT16;
    const CUresult r = enc(map.get(), dt, 3, const_cast<void*>(base), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return static_cast<int>(r);
    *out = *map;
    (*g_cache)[key] = std::move(map);
    return 0;
}

}  // namespace sb200
