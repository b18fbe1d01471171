// Tensor maps for TMA (cp.async.bulk.tensor) plane loads of level arrays.
//
// A level array of Nx x Ny x Nz doubles is described as a 3-D tensor with
// x innermost; one box is a window of kTmaBoxX x kTmaBoxY cells of one
// z-plane.  The driver entry point is looked up through the runtime, so the
// library does not link libcuda.  Maps are cached per (array, level): the
// encoding is a host call and the colored Gauss-Seidel solve alternates
// between the same few arrays.
#include "internal.cuh"

#include <cudaTypedefs.h>
#include <mutex>

namespace artss {

namespace {
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;
}  // namespace

bool tma_level_ok(const artss_ctx *ctx, int level) {
    // row and plane strides must be multiples of 16 bytes
    return (ctx->lvl[level].Nx % 2) == 0;
}

int tensor_map_3d(artss_ctx *ctx, const double *base, int level, const CUtensorMap **out, int box_x, int box_y) {
    // cached per (array, level, box)
    const auto key = std::make_pair((const void *) base, level | (box_x << 8) | (box_y << 20));
    auto it = ctx->tmaps.find(key);
    if (it != ctx->tmaps.end()) {
        *out = &it->second;
        return ARTSS_OK;
    }
    std::call_once(g_encode_once, [] {
        cudaDriverEntryPointQueryResult q;
        void *fn = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_encode = (PFN_cuTensorMapEncodeTiled_v12000) fn;
    });
    if (!g_encode) { set_error("cuTensorMapEncodeTiled is not available"); return ARTSS_ERR_CUDA; }
    if (((uintptr_t) base & 15) != 0 || !tma_level_ok(ctx, level)) {
        set_error("array not aligned for TMA plane loads"); return ARTSS_ERR_ARG;
    }
    const Level &L = ctx->lvl[level];
    CUtensorMap m;
    const cuuint64_t dim[3] = {(cuuint64_t) L.Nx, (cuuint64_t) L.Ny, (cuuint64_t) L.Nz};
    const cuuint64_t stride[2] = {(cuuint64_t) L.Nx * sizeof(double), (cuuint64_t) L.Nx * L.Ny * sizeof(double)};
    if ((box_x * (int) sizeof(double)) % 16 != 0 || box_x > 256 || box_y > 256) {
        set_error("TMA box not a multiple of 16 bytes"); return ARTSS_ERR_ARG;
    }
    const cuuint32_t box[3] = {(cuuint32_t) box_x, (cuuint32_t) box_y, 1};
    const cuuint32_t estride[3] = {1, 1, 1};
    const CUresult r = g_encode(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void *) base, dim, stride, box, estride,
                                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) { set_error("cuTensorMapEncodeTiled failed"); return ARTSS_ERR_CUDA; }
    auto ins = ctx->tmaps.emplace(key, m);
    *out = &ins.first->second;
    return ARTSS_OK;
}

}  // namespace artss
