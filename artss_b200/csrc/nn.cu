// Element-wise and data-movement kernels of the learned initial guess (the
// 3-D U-Net around artss_conv3d_*).  No counterpart in the reference.
// Activations: channels-last [D][H][W][C] bf16; parameters, gradients and
// optimizer moments: FP32.
#include "internal.cuh"

#include <cuda_bf16.h>

namespace artss {
namespace {

__device__ __forceinline__ float bf(const __nv_bfloat16 v) { return __bfloat162float(v); }

inline unsigned nblk(int64_t n, int t = 256) {
    int64_t b = (n + t - 1) / t;
    return (unsigned) std::max<int64_t>(1, std::min<int64_t>(b, 148 * 32));
}

#define NN_LOOP(n) for (int64_t q = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; q < (n); q += (int64_t) gridDim.x * blockDim.x)

// dy *= (y > 0): ReLU backward through the stored forward output
__global__ void k_relu_bwd(__nv_bfloat16 *__restrict__ dy, const __nv_bfloat16 *__restrict__ y, int64_t n) {
    NN_LOOP(n) if (!(bf(y[q]) > 0.f)) dy[q] = __float2bfloat16_rn(0.f);
}

// 2x2x2 average pooling, [D][H][W][C] -> [D/2][H/2][W/2][C]
__global__ void k_pool2(const __nv_bfloat16 *__restrict__ x, __nv_bfloat16 *__restrict__ y, int D, int H, int W, int C) {
    const int64_t n = (int64_t) (D / 2) * (H / 2) * (W / 2) * C;
    NN_LOOP(n) {
        const int c = (int) (q % C);
        int64_t v = q / C;
        const int xo = (int) (v % (W / 2)); v /= (W / 2);
        const int yo = (int) (v % (H / 2));
        const int zo = (int) (v / (H / 2));
        float s = 0.f;
#pragma unroll
        for (int o = 0; o < 8; o++)
            s += bf(x[(((int64_t) (2 * zo + (o >> 2)) * H + 2 * yo + ((o >> 1) & 1)) * W + 2 * xo + (o & 1)) * C + c]);
        y[q] = __float2bfloat16_rn(0.125f * s);
    }
}

// backward of the pooling: dx = dy / 8 on each of the 8 children
__global__ void k_pool2_bwd(const __nv_bfloat16 *__restrict__ dy, __nv_bfloat16 *__restrict__ dx, int D, int H, int W,
                            int C) {
    const int64_t n = (int64_t) D * H * W * C;
    NN_LOOP(n) {
        const int c = (int) (q % C);
        int64_t v = q / C;
        const int x = (int) (v % W); v /= W;
        const int y = (int) (v % H);
        const int z = (int) (v / H);
        dx[q] = __float2bfloat16_rn(0.125f * bf(dy[(((int64_t) (z / 2) * (H / 2) + y / 2) * (W / 2) + x / 2) * C + c]));
    }
}

// nearest 2x upsampling of [D][H][W][C] into channels [c_off, c_off + C) of a
// [2D][2H][2W][c_total] tensor (the concatenation with a skip connection)
__global__ void k_up2(const __nv_bfloat16 *__restrict__ x, __nv_bfloat16 *__restrict__ y, int D, int H, int W, int C,
                      int c_total, int c_off) {
    const int64_t n = (int64_t) 8 * D * H * W * C;
    NN_LOOP(n) {
        const int c = (int) (q % C);
        int64_t v = q / C;
        const int xf = (int) (v % (2 * W)); v /= (2 * W);
        const int yf = (int) (v % (2 * H));
        const int zf = (int) (v / (2 * H));
        y[(((int64_t) zf * 2 * H + yf) * 2 * W + xf) * c_total + c_off + c] =
            x[(((int64_t) (zf / 2) * H + yf / 2) * W + xf / 2) * C + c];
    }
}

// backward of k_up2: dx = sum of the 8 children's gradients
__global__ void k_up2_bwd(const __nv_bfloat16 *__restrict__ dy, __nv_bfloat16 *__restrict__ dx, int D, int H, int W,
                          int C, int c_total, int c_off) {
    const int64_t n = (int64_t) D * H * W * C;
    NN_LOOP(n) {
        const int c = (int) (q % C);
        int64_t v = q / C;
        const int x = (int) (v % W); v /= W;
        const int y = (int) (v % H);
        const int z = (int) (v / H);
        float s = 0.f;
#pragma unroll
        for (int o = 0; o < 8; o++)
            s += bf(dy[(((int64_t) (2 * z + (o >> 2)) * 2 * H + 2 * y + ((o >> 1) & 1)) * 2 * W + 2 * x + (o & 1)) * c_total +
                       c_off + c]);
        dx[q] = __float2bfloat16_rn(s);
    }
}

// copy channels: dst[v][d_off + c] = src[v][s_off + c], c < C (concat / split)
__global__ void k_copy_channels(const __nv_bfloat16 *__restrict__ src, int s_total, int s_off,
                                __nv_bfloat16 *__restrict__ dst, int d_total, int d_off, int C, int64_t voxels,
                                int accumulate) {
    const int64_t n = voxels * C;
    NN_LOOP(n) {
        const int c = (int) (q % C);
        const int64_t v = q / C;
        const __nv_bfloat16 s = src[v * s_total + s_off + c];
        __nv_bfloat16 &d = dst[v * d_total + d_off + c];
        d = accumulate ? __float2bfloat16_rn(bf(d) + bf(s)) : s;
    }
}

// db[c] += sum_v dy[v][c]
__global__ void k_bias_grad(const __nv_bfloat16 *__restrict__ dy, float *__restrict__ db, int64_t voxels, int C) {
    // one block per channel slice: threads stride over voxels
    for (int c = blockIdx.y; c < C; c += gridDim.y) {
        float s = 0.f;
        for (int64_t v = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; v < voxels; v += (int64_t) gridDim.x * blockDim.x)
            s += bf(dy[v * C + c]);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(db + c, s);
    }
}

// FP32 master weights w[27][co][ci] -> packed BF16 operands of the
// convolution kernels.  flip = 0: [27][ci/8][co][8] (forward);
// flip = 1: [27][co/8][ci][8] holding w[26-t][co][ci], the weights of the
// input-gradient convolution (input channels co, output channels ci).
__global__ void k_pack_weights(const float *__restrict__ w, __nv_bfloat16 *__restrict__ p, int co, int ci, int flip) {
    const int n_out = flip ? ci : co, n_in = flip ? co : ci;
    const int64_t n = (int64_t) 27 * n_in * n_out;
    NN_LOOP(n) {
        const int e = (int) (q % 8);
        int64_t r = q / 8;
        const int o = (int) (r % n_out); r /= n_out;
        const int g = (int) (r % (n_in / 8));
        const int t = (int) (r / (n_in / 8));
        const int i = 8 * g + e;
        const float v = flip ? w[((int64_t) (26 - t) * co + i) * ci + o] : w[((int64_t) t * co + o) * ci + i];
        p[q] = __float2bfloat16_rn(v);
    }
}

// Adam (Kingma & Ba 2015) with bias correction, FP32
__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       int64_t n, float lr, float b1, float b2, float eps, float c1, float c2) {
    NN_LOOP(n) {
        const float gq = g[q];
        const float mq = b1 * m[q] + (1.f - b1) * gq;
        const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
        m[q] = mq;
        v[q] = vq;
        w[q] -= lr * (mq / c1) / (sqrtf(vq / c2) + eps);
    }
}

// Network input from level arrays of the pressure problem A p = rhs, for the
// inner box [i1..i2] x [j1..j2] x [k1..k2] (x fastest):
//   ch0 = s_r (rhs - A p_prev)   (the residual of the previous pressure; p_prev
//                                 must carry its boundary values)
//   ch1 = inner-cell mask,  ch2 = s_b rhs,  ch3.. = 0;  zeros off the inner list.
__global__ void k_nn_inputs(const double *__restrict__ rhs, const double *__restrict__ p,
                            const uint8_t *__restrict__ flags, Level L, int D, int H, int W, double s_r, double s_b,
                            double rx, double ry, double rz, __nv_bfloat16 *__restrict__ out, int C) {
    const int64_t n = (int64_t) D * H * W;
    const int64_t nj = L.Nx, nk = L.nxy();
    NN_LOOP(n) {
        const int x = (int) (q % W);
        const int y = (int) ((q / W) % H);
        const int z = (int) (q / ((int64_t) W * H));
        const int64_t a = (L.i1 + x) + nj * (L.j1 + y) + nk * (L.k1 + z);
        const bool in = (flags[a] & kInner) != 0;
        float r = 0.f, bb = 0.f;
        if (in) {
            const double c2 = 2 * p[a];
            const double lap = rx * (p[a - 1] - c2 + p[a + 1]) + ry * (p[a - nj] - c2 + p[a + nj]) +
                               rz * (p[a - nk] - c2 + p[a + nk]);
            r = (float) (s_r * (rhs[a] - lap));
            bb = (float) (s_b * rhs[a]);
        }
        __nv_bfloat16 *o = out + q * C;
        o[0] = __float2bfloat16_rn(r);
        o[1] = __float2bfloat16_rn(in ? 1.f : 0.f);
        o[2] = __float2bfloat16_rn(bb);
        for (int c = 3; c < C; c++) o[c] = __float2bfloat16_rn(0.f);
    }
}

// guess: p[a] = p_prev[a] + scale * y[v][0] on inner cells (other cells keep p)
__global__ void k_nn_apply(const __nv_bfloat16 *__restrict__ y, int C, const double *__restrict__ p_prev,
                           const uint8_t *__restrict__ flags, Level L, int D, int H, int W, double scale,
                           double *__restrict__ p) {
    const int64_t n = (int64_t) D * H * W;
    NN_LOOP(n) {
        const int x = (int) (q % W);
        const int yy = (int) ((q / W) % H);
        const int z = (int) (q / ((int64_t) W * H));
        const int64_t a = (L.i1 + x) + L.Nx * (L.j1 + yy) + L.nxy() * (L.k1 + z);
        if (flags[a] & kInner) p[a] = p_prev[a] + scale * (double) bf(y[q * C]);
    }
}

// training target: t[v] = scale * (p_star[a] - p_prev[a]) over the inner box
// (0 outside the inner list), voxel order x fastest
__global__ void k_nn_target(const double *__restrict__ p_star, const double *__restrict__ p_prev,
                            const uint8_t *__restrict__ flags, Level L, int D, int H, int W, double scale,
                            float *__restrict__ t) {
    const int64_t n = (int64_t) D * H * W;
    NN_LOOP(n) {
        const int x = (int) (q % W);
        const int y = (int) ((q / W) % H);
        const int z = (int) (q / ((int64_t) W * H));
        const int64_t a = (L.i1 + x) + L.Nx * (L.j1 + y) + L.nxy() * (L.k1 + z);
        t[q] = (flags[a] & kInner) ? (float) (scale * (p_star[a] - p_prev[a])) : 0.f;
    }
}

// loss 0.5 * sum over inner cells (y[v][0] - t[v])^2 and its gradient into
// channel 0 of dy (other channels zero); block partials of the loss
__global__ void k_mse(const __nv_bfloat16 *__restrict__ y, int C, const float *__restrict__ t,
                      const __nv_bfloat16 *__restrict__ mask_in, __nv_bfloat16 *__restrict__ dy, int64_t voxels,
                      float inv_n, float *__restrict__ partials) {
    __shared__ float sm[32];
    float acc = 0.f;
    NN_LOOP(voxels) {
        const bool in = bf(mask_in[q * C + 1]) > 0.5f;
        const float d = in ? bf(y[q * C]) - t[q] : 0.f;
        acc += 0.5f * d * d;
        dy[q * C] = __float2bfloat16_rn(d * inv_n);
        for (int c = 1; c < C; c++) dy[q * C + c] = __float2bfloat16_rn(0.f);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        acc = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0.f;
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (threadIdx.x == 0) partials[blockIdx.x] = acc;
    }
}

}  // namespace
}  // namespace artss

using namespace artss;

#define NN_CK(ctx) ARTSS_LAUNCH_CK(ctx)
#define NN_ARGS_OK(...) do { if (!(__VA_ARGS__)) { set_error("invalid argument"); return ARTSS_ERR_ARG; } } while (0)

extern "C" {

int artss_nn_zero(artss_ctx *ctx, void *p, int64_t bytes) {
    NN_ARGS_OK(ctx && p && bytes >= 0);
    ARTSS_CK(cudaMemsetAsync(p, 0, (size_t) bytes, ctx->stream));
    return ARTSS_OK;
}

int artss_nn_relu_bwd(artss_ctx *ctx, void *dy, const void *y, int64_t n) {
    NN_ARGS_OK(ctx && dy && y && n >= 0);
    ARTSS_LAUNCH(ctx, FAM_NN, k_relu_bwd<<<nblk(n), 256, 0, ctx->stream>>>((__nv_bfloat16 *) dy, (const __nv_bfloat16 *) y, n));
    NN_CK(ctx);
    return ARTSS_OK;
}

int artss_nn_pool2(artss_ctx *ctx, const void *x, void *y, int D, int H, int W, int C, int backward) {
    NN_ARGS_OK(ctx && x && y && D % 2 == 0 && H % 2 == 0 && W % 2 == 0 && C > 0);
    const int64_t n = backward ? (int64_t) D * H * W * C : (int64_t) D * H * W * C / 8;
    if (backward)
        ARTSS_LAUNCH(ctx, FAM_NN, k_pool2_bwd<<<nblk(n), 256, 0, ctx->stream>>>((const __nv_bfloat16 *) x, (__nv_bfloat16 *) y, D, H, W, C));
    else
        ARTSS_LAUNCH(ctx, FAM_NN, k_pool2<<<nblk(n), 256, 0, ctx->stream>>>((const __nv_bfloat16 *) x, (__nv_bfloat16 *) y, D, H, W, C));
    NN_CK(ctx);
    return ARTSS_OK;
}

int artss_nn_up2(artss_ctx *ctx, const void *x, void *y, int D, int H, int W, int C, int c_total, int c_off,
                 int backward) {
    NN_ARGS_OK(ctx && x && y && C > 0 && c_off >= 0 && c_off + C <= c_total);
    if (backward)
        ARTSS_LAUNCH(ctx, FAM_NN, k_up2_bwd<<<nblk((int64_t) D * H * W * C), 256, 0, ctx->stream>>>(
                                     (const __nv_bfloat16 *) x, (__nv_bfloat16 *) y, D, H, W, C, c_total, c_off));
    else
        ARTSS_LAUNCH(ctx, FAM_NN, k_up2<<<nblk((int64_t) 8 * D * H * W * C), 256, 0, ctx->stream>>>(
                                     (const __nv_bfloat16 *) x, (__nv_bfloat16 *) y, D, H, W, C, c_total, c_off));
    NN_CK(ctx);
    return ARTSS_OK;
}

int artss_nn_copy_channels(artss_ctx *ctx, const void *src, int s_total, int s_off, void *dst, int d_total, int d_off,
                           int C, int64_t voxels, int accumulate) {
    NN_ARGS_OK(ctx && src && dst && C > 0 && s_off + C <= s_total && d_off + C <= d_total && voxels >= 0);
    ARTSS_LAUNCH(ctx, FAM_NN, k_copy_channels<<<nblk(voxels * C), 256, 0, ctx->stream>>>(
                                 (const __nv_bfloat16 *) src, s_total, s_off, (__nv_bfloat16 *) dst, d_total, d_off, C,
                                 voxels, accumulate));
    NN_CK(ctx);
    return ARTSS_OK;
}

int artss_nn_bias_grad(artss_ctx *ctx, const void *dy, float *db, int64_t voxels, int C) {
    NN_ARGS_OK(ctx && dy && db && C > 0);
    const dim3 g((unsigned) std::min<int64_t>(512, (voxels + 255) / 256 + 1), (unsigned) C);
    ARTSS_LAUNCH(ctx, FAM_NN, k_bias_grad<<<g, 256, 0, ctx->stream>>>((const __nv_bfloat16 *) dy, db, voxels, C));
    NN_CK(ctx);
    return ARTSS_OK;
}

int artss_nn_pack_weights(artss_ctx *ctx, const float *w, void *packed, int cout, int cin, int flip) {
    NN_ARGS_OK(ctx && w && packed && cin % 16 == 0 && cout % 16 == 0);
    const int64_t n = (int64_t) 27 * cout * cin;
    ARTSS_LAUNCH(ctx, FAM_NN, k_pack_weights<<<nblk(n), 256, 0, ctx->stream>>>(w, (__nv_bfloat16 *) packed, cout, cin,
                                                                               flip));
    NN_CK(ctx);
    return ARTSS_OK;
}

int artss_nn_adam(artss_ctx *ctx, float *w, const float *g, float *m, float *v, int64_t n, float lr, float b1, float b2,
                  float eps, int step) {
    NN_ARGS_OK(ctx && w && g && m && v && step >= 1);
    const float c1 = 1.f - powf(b1, (float) step), c2 = 1.f - powf(b2, (float) step);
    ARTSS_LAUNCH(ctx, FAM_NN, k_adam<<<nblk(n), 256, 0, ctx->stream>>>(w, g, m, v, n, lr, b1, b2, eps, c1, c2));
    NN_CK(ctx);
    return ARTSS_OK;
}

int artss_nn_inputs(artss_ctx *ctx, int level, const double *rhs, const double *p_prev, double s_r, double s_b,
                    void *out, int C) {
    NN_ARGS_OK(ctx && rhs && p_prev && out && C >= 3);
    int st = check_level(ctx, level);
    if (st) return st;
    const Level &L = ctx->lvl[level];
    const artss_grid_desc &g = ctx->grid;
    const int W = (int) (L.i2 - L.i1 + 1), H = (int) (L.j2 - L.j1 + 1), D = (int) (L.k2 - L.k1 + 1);
    ARTSS_LAUNCH(ctx, FAM_NN, k_nn_inputs<<<nblk((int64_t) D * H * W), 256, 0, ctx->stream>>>(
                                 rhs, p_prev, ctx->d_flags[level], L, D, H, W, s_r, s_b,
                                 1. / (g.dx[level] * g.dx[level]), 1. / (g.dy[level] * g.dy[level]),
                                 1. / (g.dz[level] * g.dz[level]), (__nv_bfloat16 *) out, C));
    NN_CK(ctx);
    return ARTSS_OK;
}

int artss_nn_apply(artss_ctx *ctx, int level, const void *y, int C, const double *p_prev, double scale, double *p) {
    NN_ARGS_OK(ctx && y && p_prev && p && C >= 1);
    int st = check_level(ctx, level);
    if (st) return st;
    const Level &L = ctx->lvl[level];
    const int W = (int) (L.i2 - L.i1 + 1), H = (int) (L.j2 - L.j1 + 1), D = (int) (L.k2 - L.k1 + 1);
    ARTSS_LAUNCH(ctx, FAM_NN, k_nn_apply<<<nblk((int64_t) D * H * W), 256, 0, ctx->stream>>>(
                                 (const __nv_bfloat16 *) y, C, p_prev, ctx->d_flags[level], L, D, H, W, scale, p));
    NN_CK(ctx);
    return ARTSS_OK;
}

int artss_nn_target(artss_ctx *ctx, int level, const double *p_star, const double *p_prev, double scale, float *t) {
    NN_ARGS_OK(ctx && p_star && p_prev && t);
    int st = check_level(ctx, level);
    if (st) return st;
    const Level &L = ctx->lvl[level];
    const int W = (int) (L.i2 - L.i1 + 1), H = (int) (L.j2 - L.j1 + 1), D = (int) (L.k2 - L.k1 + 1);
    ARTSS_LAUNCH(ctx, FAM_NN, k_nn_target<<<nblk((int64_t) D * H * W), 256, 0, ctx->stream>>>(
                                 p_star, p_prev, ctx->d_flags[level], L, D, H, W, scale, t));
    NN_CK(ctx);
    return ARTSS_OK;
}

int artss_nn_mse(artss_ctx *ctx, const void *y, int C, const float *target, const void *inputs, void *dy,
                 int64_t voxels, float inv_n, float *partials, int n_partials) {
    NN_ARGS_OK(ctx && y && target && inputs && dy && partials && n_partials >= 1);
    ARTSS_LAUNCH(ctx, FAM_NN, k_mse<<<(unsigned) n_partials, 256, 0, ctx->stream>>>(
                                 (const __nv_bfloat16 *) y, C, target, (const __nv_bfloat16 *) inputs,
                                 (__nv_bfloat16 *) dy, voxels, inv_n, partials));
    NN_CK(ctx);
    return ARTSS_OK;
}

}  // extern "C"
