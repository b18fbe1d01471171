// BF16 implicit-GEMM 3-D convolution on the 5th-generation tensor cores
// (tcgen05.mma, FP32 accumulation in tensor memory) for the learned
// initial guess of the pressure solve.  No counterpart in the reference.
//
// Activations are channels-last, [D][H][W][C] bf16, C a multiple of 16.
// Kernel 3x3x3, stride 1, zero padding 1 (cross-correlation):
//     y[z,y,x,co] = bias[co] + sum_{t, ci} w[t][co][ci] * x[z+dz, y+dy, x+dx, ci]
// with tap t = 9 (dz+1) + 3 (dy+1) + (dx+1).
//
// GEMM view: M = 128 output voxels (a run of x, several y rows and z planes
// when W or W*H is below 128),
// N = C_out, K = 27 taps x C_in.  Per tap one TMA load brings the 128 shifted
// input rows (out-of-range voxels arrive as zeros, which is the padding) in
// the K-major core-matrix layout [C_in/8][128][8] (the tensor map orders the
// dimensions channel-in-group, x, y, z, channel group), and one bulk copy brings
// the tap's weights, pre-packed as [C_in/8][C_out][8]; one thread issues the
// C_in/16 MMAs of the tap and commits them to the stage's "empty" barrier.
// After the 27th tap the accumulator (128 lanes x C_out FP32 columns) is read
// by warps 0-3 with tcgen05.ld: bias, optional ReLU, BF16, store.  Warp 4
// loads and issues: two accumulators in tensor memory alternate between tiles,
// so the MMAs of tile n+1 run while tile n is read out.  Blocks are persistent
// over output tiles; loads run as many taps ahead as shared memory holds
// stages (ConvShape::stages, at most kConvMaxStages), across tile boundaries.
// Every wait is bounded and raises an error flag.
#include "internal.cuh"
#include "tc.cuh"

#include <cuda_bf16.h>
#include <cudaTypedefs.h>
#include <mutex>
#include <tuple>

namespace artss {

namespace {

constexpr int kConvThreads = 128;
constexpr int kConvFwdThreads = 160;  // warps 0-3: epilogue (tensor-memory lanes 0..127); warp 4: loads and MMAs
constexpr int kConvMaxStages = 16;
constexpr int kConvPolls = 1 << 20;
constexpr size_t kConvGuard = 64 * 1024;           // shared memory past the last stage, never addressed by a correct descriptor
constexpr size_t kConvSmemMax = 227 * 1024 - 2048;  // dynamic limit minus the kernels' static shared memory

struct ConvShape {
    int D, H, W, cin, cout;
    int tw, th, tz;           // tile: tw x th x tz voxels, tw * th * tz = 128 (x fastest)
    int tiles_x, tiles_y, tiles_z, tiles;
    unsigned a_bytes, b_bytes, stage_bytes;
    int stages;               // ring depth (taps in flight)
};

__global__ void __launch_bounds__(kConvFwdThreads, 1)
k_conv3d_fwd(const __grid_constant__ CUtensorMap tm_x, const __nv_bfloat16 *__restrict__ wp,
             const float *__restrict__ bias, __nv_bfloat16 *__restrict__ y, ConvShape s, int relu,
             int *__restrict__ err) {
    extern __shared__ __align__(1024) uint8_t cv_sm[];
    // full / empty: the stage ring; accf[a]: accumulator a holds a finished tile;
    // acce[a]: the four epilogue warps have read accumulator a out
    __shared__ __align__(8) uint64_t full[kConvMaxStages], empty[kConvMaxStages], accf[2], acce[2];
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int S = s.stages;
    const unsigned tcols = s.cout <= 32 ? 32u : (s.cout <= 64 ? 64u : (s.cout <= 128 ? 128u : 256u));
    if (tid == 0) {
        for (int i = 0; i < S; i++) {
            tc::mbar_init(&full[i], 1);
            tc::mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; i++) {
            tc::mbar_init(&accf[i], 1);
            tc::mbar_init(&acce[i], 4);
        }
        tc::fence_barrier_init();
    }
    if (warp == 0) {
        tc::tmem_alloc(&tmem_base, 2 * tcols);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = tmem_base;
    const int my_tiles = (s.tiles - (int) blockIdx.x + (int) gridDim.x - 1) / (int) gridDim.x;
    const int nsteps = my_tiles * 27;

    if (warp == 4) {
        if (lane == 0) {
            const int kk_n = s.cin / 16;
            const uint32_t idesc = tc::idesc_bf16(128, s.cout, 0, 0);
            const unsigned lbo_a = 128 * 16, lbo_b = (unsigned) s.cout * 16;
            // the loads of step p (tile p / 27, tap p % 27)
            auto produce = [&](int p) {
                const int st = p % S;
                if (p >= S && !tc::mbar_wait(&empty[st], (unsigned) ((p / S - 1) & 1), kConvPolls)) return false;
                const int tile = (int) blockIdx.x + (p / 27) * (int) gridDim.x, tap = p % 27;
                const int tx = tile % s.tiles_x, ty = (tile / s.tiles_x) % s.tiles_y, tzi = tile / (s.tiles_x * s.tiles_y);
                const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
                uint8_t *a = cv_sm + (size_t) st * s.stage_bytes;
                tc::mbar_expect_tx(&full[st], s.a_bytes + s.b_bytes);
                tc::tma_load_5d(a, &tm_x, 0, tx * s.tw + dx, ty * s.th + dy, tzi * s.tz + dz, 0, &full[st]);
                tc::bulk_load(a + s.a_bytes, wp + (size_t) tap * s.cout * s.cin, s.b_bytes, &full[st]);
                return true;
            };
            bool ok = true;
            int issued = 0;  // steps whose loads were issued
            for (int p = 0; p < S - 1 && p < nsteps && ok; p++)
                if ((ok = produce(p))) issued = p + 1;
            int step = 0;
            for (int it = 0; it < my_tiles && ok; it++) {
                const int acc = it & 1;
                const uint32_t d = tmem + (uint32_t) acc * tcols;
                // accumulator acc last held tile it - 2: wait until it was read out
                if (it >= 2) ok = tc::mbar_wait(&acce[acc], (unsigned) (((it >> 1) - 1) & 1), kConvPolls);
                tc::tc_fence_after();
                for (int tap = 0; tap < 27 && ok; tap++, step++) {
                    if (step + S - 1 < nsteps && (ok = produce(step + S - 1))) issued = step + S;
                    const int st = step % S;
                    if (ok) ok = tc::mbar_wait(&full[st], (unsigned) ((step / S) & 1), kConvPolls);
                    if (!ok) break;
                    tc::tc_fence_after();
                    const uint8_t *a = cv_sm + (size_t) st * s.stage_bytes;
                    const uint8_t *b = a + s.a_bytes;
                    for (int kk = 0; kk < kk_n; kk++) {
                        const uint64_t da = tc::smem_desc(a + 2 * kk * lbo_a, lbo_a, 128);
                        const uint64_t db = tc::smem_desc(b + 2 * kk * lbo_b, lbo_b, 128);
                        tc::mma_bf16(d, da, db, idesc, (tap | kk) != 0);
                    }
                    tc::mma_commit(&empty[st]);
                }
                if (ok) tc::mma_commit(&accf[acc]);
            }
            if (!ok) {
                if (err) atomicExch(err, 1);
                // let this block's loads and MMAs in flight finish before it leaves
                for (int p = step; p < issued; p++)
                    (void) tc::mbar_wait(&full[p % S], (unsigned) ((p / S) & 1), kConvPolls);
                if (step > 0)
                    (void) tc::mbar_wait(&empty[(step - 1) % S], (unsigned) (((step - 1) / S) & 1), kConvPolls);
            }
        }
    } else {
        // epilogue: lane = voxel of the tile, columns = output channels
        for (int it = 0; it < my_tiles; it++) {
            const int acc = it & 1;
            if (!tc::mbar_wait(&accf[acc], (unsigned) ((it >> 1) & 1), kConvPolls)) {
                if (lane == 0 && err) atomicExch(err, 1);
                break;
            }
            tc::tc_fence_after();
            const int tile = (int) blockIdx.x + it * (int) gridDim.x;
            const int tx = tile % s.tiles_x, ty = (tile / s.tiles_x) % s.tiles_y, tzi = tile / (s.tiles_x * s.tiles_y);
            const int vx = tx * s.tw + tid % s.tw, vy = ty * s.th + (tid / s.tw) % s.th,
                      vz = tzi * s.tz + tid / (s.tw * s.th);
            __nv_bfloat16 *yo = y + (((size_t) vz * s.H + vy) * s.W + vx) * s.cout;
            const uint32_t src = tmem + (uint32_t) acc * tcols + ((uint32_t) (32 * warp) << 16);
            for (int c0 = 0; c0 < s.cout; c0 += 16) {
                float v[16];
                tc::tmem_ld16(src + (uint32_t) c0, v);
                __align__(16) __nv_bfloat16 o[16];
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    float r = v[i] + (bias ? bias[c0 + i] : 0.f);
                    if (relu) r = fmaxf(r, 0.f);
                    o[i] = __float2bfloat16_rn(r);
                }
                uint4 *dst = reinterpret_cast<uint4 *>(yo + c0);
                dst[0] = reinterpret_cast<const uint4 *>(o)[0];
                dst[1] = reinterpret_cast<const uint4 *>(o)[1];
            }
            tc::tc_fence_before();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&acce[acc]);
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    if (warp == 0) tc::tmem_dealloc(tmem, 2 * tcols);
}

// Weight gradient dW[t][co][ci] += sum_v dY[v][co] x[v + off_t][ci] as a GEMM
// with M = C_out (padded to 128 by TMA's zero fill), N = C_in, K = voxels.
// The activation tiles keep the forward's shared-memory layout
// [channel/8][128 voxels][8], which read as MN-major operands is exactly the
// canonical layout: 8 voxels (K) x 8 channels (M or N) per core matrix, the
// core matrices of one channel group 128 bytes apart (LBO), channel groups
// 2048 bytes apart (SBO).  A block accumulates one tap over its range of
// voxel tiles in tensor memory, then adds the C_out x C_in block to dW with
// FP32 atomics (dW must be zeroed by the caller), and moves to the next tap.
constexpr int kWgradMRows = 128;

__global__ void __launch_bounds__(kConvThreads, 1)
k_conv3d_wgrad(const __grid_constant__ CUtensorMap tm_x, const __grid_constant__ CUtensorMap tm_dy,
               float *__restrict__ dw, ConvShape s, int tiles_per_block, int *__restrict__ err) {
    extern __shared__ __align__(1024) uint8_t cv_sm[];
    __shared__ __align__(8) uint64_t full[kConvMaxStages], empty[kConvMaxStages], accb;
    __shared__ uint32_t tmem_base;
    __shared__ int s_fail;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int S = s.stages;
    const unsigned tcols = s.cin <= 32 ? 32u : (s.cin <= 64 ? 64u : (s.cin <= 128 ? 128u : 256u));
    const int t_begin = (int) blockIdx.x * tiles_per_block;
    const int t_end = min(s.tiles, t_begin + tiles_per_block);
    const int ntile = t_end - t_begin;
    if (ntile <= 0) return;
    if (tid == 0) {
        for (int i = 0; i < S; i++) {
            tc::mbar_init(&full[i], 1);
            tc::mbar_init(&empty[i], 1);
        }
        tc::mbar_init(&accb, 1);
        tc::fence_barrier_init();
        s_fail = 0;
    }
    if (warp == 0) {
        tc::tmem_alloc(&tmem_base, tcols);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = tmem_base;
    const int nsteps = 27 * ntile;
    const uint32_t idesc = tc::idesc_bf16(kWgradMRows, s.cin, 1, 1);
    const unsigned a_bytes = (unsigned) kWgradMRows * 128u * 2u;  // dY tile, 16 channel groups
    const unsigned b_bytes = s.a_bytes;                            // x tile, C_in/8 channel groups

    auto produce = [&](int p) {
        const int st = p % S;
        if (p >= S && !tc::mbar_wait(&empty[st], (unsigned) ((p / S - 1) & 1), kConvPolls)) return false;
        const int tap = p / ntile, tile = t_begin + p % ntile;
        const int tx = tile % s.tiles_x, ty = (tile / s.tiles_x) % s.tiles_y, tzi = tile / (s.tiles_x * s.tiles_y);
        const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
        uint8_t *a = cv_sm + (size_t) st * s.stage_bytes;
        tc::mbar_expect_tx(&full[st], a_bytes + b_bytes);
        tc::tma_load_5d(a, &tm_dy, 0, tx * s.tw, ty * s.th, tzi * s.tz, 0, &full[st]);
        tc::tma_load_5d(a + a_bytes, &tm_x, 0, tx * s.tw + dx, ty * s.th + dy, tzi * s.tz + dz, 0, &full[st]);
        return true;
    };

    bool ok = true;
    int step = 0;
    if (tid == 0)
        for (int p = 0; p < S - 1 && p < nsteps && ok; p++) ok = produce(p);
    for (int tap = 0; tap < 27; tap++) {
        if (tid == 0 && ok) {
            for (int i = 0; i < ntile && ok; i++, step++) {
                if (step + S - 1 < nsteps) ok = produce(step + S - 1);
                const int st = step % S;
                if (ok) ok = tc::mbar_wait(&full[st], (unsigned) ((step / S) & 1), kConvPolls);
                if (!ok) break;
                tc::tc_fence_after();
                const uint8_t *a = cv_sm + (size_t) st * s.stage_bytes;
                const uint8_t *b = a + a_bytes;
#pragma unroll
                for (int kk = 0; kk < 8; kk++) {  // 16 voxels per MMA
                    const uint64_t da = tc::smem_desc(a + kk * 256, 128, 2048);
                    const uint64_t db = tc::smem_desc(b + kk * 256, 128, 2048);
                    tc::mma_bf16(tmem, da, db, idesc, (i | kk) != 0);
                }
                tc::mma_commit(&empty[st]);
                if (i == ntile - 1) tc::mma_commit(&accb);
            }
            if (!ok) s_fail = 1;
        }
        bool acc_ok = true;
        if (tid == 0) acc_ok = ok && tc::mbar_wait(&accb, (unsigned) (tap & 1), kConvPolls);
        if (__syncthreads_or(!acc_ok || s_fail)) {
            if (tid == 0 && err) atomicExch(err, 1);
            break;
        }
        tc::tc_fence_after();
        // lane = output channel co, columns = input channels
        for (int c0 = 0; c0 < s.cin; c0 += 16) {
            float v[16];
            tc::tmem_ld16(tmem + ((uint32_t) (32 * warp) << 16) + (uint32_t) c0, v);
            if (tid < s.cout) {
                float *d = dw + ((size_t) tap * s.cout + tid) * s.cin + c0;
#pragma unroll
                for (int i = 0; i < 16; i++) atomicAdd(d + i, v[i]);
            }
        }
        tc::tc_fence_before();
        __syncthreads();
    }
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, tcols);
}

PFN_cuTensorMapEncodeTiled_v12000 g_enc = nullptr;
std::once_flag g_enc_once;

// map of a [D][H][W][c] activation whose box lands as [box_chunks][th][tw][8]
int encode_act_map(const __nv_bfloat16 *x, const ConvShape &s, int c, int box_chunks, CUtensorMap *m);

int encode_x_map(const __nv_bfloat16 *x, const ConvShape &s, CUtensorMap *m) {
    return encode_act_map(x, s, s.cin, s.cin / 8, m);
}

int encode_act_map(const __nv_bfloat16 *x, const ConvShape &s, int c, int box_chunks, CUtensorMap *m) {
    std::call_once(g_enc_once, [] {
        cudaDriverEntryPointQueryResult q;
        void *fn = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_enc = (PFN_cuTensorMapEncodeTiled_v12000) fn;
    });
    if (!g_enc) { set_error("cuTensorMapEncodeTiled is not available"); return ARTSS_ERR_CUDA; }
    // dims: channel-in-chunk (8), x, y, z, chunk -> a box lands as [chunk][z][y][x][8]
    const cuuint64_t dim[5] = {8, (cuuint64_t) s.W, (cuuint64_t) s.H, (cuuint64_t) s.D, (cuuint64_t) (c / 8)};
    const cuuint64_t es = 2;
    const cuuint64_t stride[4] = {(cuuint64_t) c * es, (cuuint64_t) s.W * c * es, (cuuint64_t) s.H * s.W * c * es, 16};
    const cuuint32_t box[5] = {8, (cuuint32_t) s.tw, (cuuint32_t) s.th, (cuuint32_t) s.tz, (cuuint32_t) box_chunks};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    const CUresult r = g_enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, (void *) x, dim, stride, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) { set_error("conv3d: input tensor map rejected"); return ARTSS_ERR_ARG; }
    return ARTSS_OK;
}

// stages of `bytes` each that fit the dynamic shared memory with kConvGuardMin
// left over, at most kConvMaxStages
constexpr size_t kConvGuardMin = 16 * 1024;
int conv_stages(size_t bytes) {
    return (int) std::min<size_t>(kConvMaxStages, (kConvSmemMax - kConvGuardMin) / bytes);
}

int conv_shape(const artss_conv_desc *d, ConvShape *s) {
    if (d->D < 1 || d->H < 1 || d->W < 1 || d->cin < 16 || d->cin % 16 || d->cin > 256 ||
        d->cout < 16 || d->cout % 16 || d->cout > 256) {
        set_error("conv3d: channels must be multiples of 16, at most 256");
        return ARTSS_ERR_ARG;
    }
    s->D = d->D; s->H = d->H; s->W = d->W; s->cin = d->cin; s->cout = d->cout;
    s->tz = 1;
    if (d->W % 128 == 0) { s->tw = 128; s->th = 1; }
    else if (128 % d->W == 0 && d->W * d->H >= 128 && d->H % (128 / d->W) == 0) { s->tw = d->W; s->th = 128 / d->W; }
    else if (128 % (d->W * d->H) == 0 && d->D % (128 / (d->W * d->H)) == 0) {
        s->tw = d->W; s->th = d->H; s->tz = 128 / (d->W * d->H);
    } else {
        set_error("conv3d: 128-voxel tiles must fit: W a multiple of 128, or W dividing 128 with H a multiple of "
                  "128/W, or W*H dividing 128 with D a multiple of 128/(W*H)");
        return ARTSS_ERR_ARG;
    }
    s->tiles_x = d->W / s->tw;
    s->tiles_y = d->H / s->th;
    s->tiles_z = d->D / s->tz;
    s->tiles = s->tiles_x * s->tiles_y * s->tiles_z;
    s->a_bytes = 128u * (unsigned) d->cin * 2u;
    s->b_bytes = (unsigned) d->cout * (unsigned) d->cin * 2u;
    s->stage_bytes = (s->a_bytes + s->b_bytes + 1023u) & ~1023u;
    s->stages = conv_stages(s->stage_bytes);
    if (s->stages < 2) { set_error("conv3d: stages too large"); return ARTSS_ERR_LIMIT; }
    return ARTSS_OK;
}

}  // namespace

int conv3d_wgrad(artss_ctx *ctx, const artss_conv_desc *d, const void *x, const void *dy, float *dw) {
    ConvShape s;
    int st = conv_shape(d, &s);
    if (st) return st;
    if (d->cout > kWgradMRows || d->cin > 128) { set_error("conv3d wgrad: C_out and C_in at most 128"); return ARTSS_ERR_ARG; }
    if (((uintptr_t) x & 15) || ((uintptr_t) dy & 15)) { set_error("conv3d: arrays must be 16-byte aligned"); return ARTSS_ERR_ARG; }
    CUtensorMap mx, mdy;
    if ((st = encode_act_map((const __nv_bfloat16 *) x, s, s.cin, s.cin / 8, &mx))) return st;
    if ((st = encode_act_map((const __nv_bfloat16 *) dy, s, s.cout, kWgradMRows / 8, &mdy))) return st;
    // stage: dY tile (128 voxels x 128 padded channels) + x tile
    const unsigned stage = ((unsigned) kWgradMRows * 128u * 2u + s.a_bytes + 1023u) & ~1023u;
    s.stage_bytes = stage;
    s.stages = conv_stages(stage);
    if (s.stages < 2) { set_error("conv3d wgrad: stages too large"); return ARTSS_ERR_LIMIT; }
    const size_t stages = (size_t) stage * s.stages;
    const size_t smem = stages + std::min<size_t>(kConvGuard, kConvSmemMax - stages);
    ARTSS_CK(cudaFuncSetAttribute(k_conv3d_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    const int grid = std::min(s.tiles, sms);
    const int per = (s.tiles + grid - 1) / grid;
    const int blocks = (s.tiles + per - 1) / per;
    ARTSS_LAUNCH(ctx, FAM_CONV, k_conv3d_wgrad<<<blocks, kConvThreads, smem, ctx->stream>>>(
                                    mx, mdy, dw, s, per, &ctx->d_loop[kNnErrSlot].pad));
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

int conv3d_fwd(artss_ctx *ctx, const artss_conv_desc *d, const void *x, const void *wp, const float *bias, void *y) {
    ConvShape s;
    int st = conv_shape(d, &s);
    if (st) return st;
    if (((uintptr_t) x & 15) || ((uintptr_t) wp & 15) || ((uintptr_t) y & 15)) {
        set_error("conv3d: arrays must be 16-byte aligned"); return ARTSS_ERR_ARG;
    }
    CUtensorMap m;
    if ((st = encode_x_map((const __nv_bfloat16 *) x, s, &m))) return st;
    const size_t stages = (size_t) s.stage_bytes * s.stages;
    const size_t smem = stages + std::min<size_t>(kConvGuard, kConvSmemMax - stages);
    ARTSS_CK(cudaFuncSetAttribute(k_conv3d_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    const int grid = std::min(s.tiles, sms);
    ARTSS_LAUNCH(ctx, FAM_CONV, k_conv3d_fwd<<<grid, kConvFwdThreads, smem, ctx->stream>>>(
                                    m, (const __nv_bfloat16 *) wp, bias, (__nv_bfloat16 *) y, s, d->relu,
                                    &ctx->d_loop[kNnErrSlot].pad));
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

}  // namespace artss

using namespace artss;

extern "C" int artss_conv3d_fwd(artss_ctx *ctx, const artss_conv_desc *d, const void *x, const void *w_packed,
                                const float *bias, void *y) {
    if (!ctx || !d || !x || !w_packed || !y) { set_error("null argument"); return ARTSS_ERR_ARG; }
    return conv3d_fwd(ctx, d, x, w_packed, bias, y);
}

extern "C" int artss_nn_check(artss_ctx *ctx) {
    if (!ctx) { set_error("null argument"); return ARTSS_ERR_ARG; }
    LoopState ls{};
    int st = read_loop(ctx, kNnErrSlot, &ls);
    if (st) return st;
    if (ls.pad) {
        ARTSS_CK(cudaMemsetAsync(&ctx->d_loop[kNnErrSlot].pad, 0, sizeof(int), ctx->stream));
        ARTSS_CK(cudaStreamSynchronize(ctx->stream));
        set_error("a network kernel gave up waiting for its operands");
        return ARTSS_ERR_CUDA;
    }
    return ARTSS_OK;
}

extern "C" int artss_conv3d_wgrad(artss_ctx *ctx, const artss_conv_desc *d, const void *x, const void *dy, float *dw) {
    if (!ctx || !d || !x || !dy || !dw) { set_error("null argument"); return ARTSS_ERR_ARG; }
    return conv3d_wgrad(ctx, d, x, dy, dw);
}
