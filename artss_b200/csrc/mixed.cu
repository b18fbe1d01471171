// Mixed-precision pressure solve: FP64 defect correction around FP32 V-cycles.
//
// No counterpart in the reference; it plugs in where IPressure::pressure
// (src/interfaces/IPressure.h:17) is called and is judged against VCycleMG
// (src/pressure/VCycleMG.cpp) iterated to the same relative residual.
//
// Outer loop, FP64 on level 0:
//     r = b - A p                      stop when ||r||_2 <= rel_tol * ||b||_2
//     e = V(r)                         FP32 V-cycle on A e = r, e = 0 at start
//     p += e                           FP64
// and, for pure-Neumann problems (A 1 = 0), the mean of p over the inner
// cells is removed at the end.  b must lie in the range of A: with the
// reference's obstacle boundary programs (edge and corner cells copy one of
// their fluid neighbours) A is not symmetric, so a mean-free b is not enough
// for a pure-Neumann problem; artss_laplacian builds consistent right-hand
// sides.  The V-cycle has the structure of VCycleMG::VCycleMultigrid
// (n_relax weighted-Jacobi sweeps, each followed by the level's boundary
// program, residual, restriction, prolongation with the trilinear weights of
// VCycleMG::Prolongate), all in FP32 with the boundary values set to zero
// (the correction equation is homogeneous), and the coarsest level solved in
// FP64 by the cluster kernel to a relative tolerance.  Because the outer
// residual is FP64, the FP32 round-off limits only the convergence rate per
// cycle, not the final accuracy.
//
// All outer iterations run as predicated batches: every kernel of an
// iteration returns at once when the device loop state says the solve has
// converged, and the host reads that state once per batch.
#include "internal.cuh"

#include <algorithm>

struct artss_mixed {
    artss_ctx *ctx = nullptr;
    artss_mixed_cfg cfg{};
    int L = 0;  // levels 0 .. L-1
    float *r[artss::kMaxLevel + 1]{};    // right-hand side of level l
    float *q[artss::kMaxLevel + 1]{};    // residual of level l
    float *e[artss::kMaxLevel + 1]{};    // correction of level l
    float *t[artss::kMaxLevel + 1]{};    // Jacobi ping-pong partner of e
    int64_t n_inner0 = 0;
    int64_t hint = 1;                    // outer iterations of the last solve
};

namespace artss {

namespace {

inline dim3 mx_grid(const Box3 &b) {
    dim3 g = box_grid(b);
    const int64_t xy = (int64_t) g.x * g.y;
    int64_t gz = b.nz();
    const int64_t cap = std::max<int64_t>(1, 2048 / std::max<int64_t>(xy, 1));
    if (gz > cap) gz = cap;
    g.z = (unsigned) std::max<int64_t>(gz, 1);
    return g;
}

#define MX_COLUMN(box)                                                            \
    const int64_t i = (box).x0 + (int64_t) blockIdx.x * blockDim.x + threadIdx.x; \
    const int64_t j = (box).y0 + (int64_t) blockIdx.y * blockDim.y + threadIdx.y; \
    const bool col = (i <= (box).x1) && (j <= (box).y1)

struct CoefF {
    float ax, ay, az, beta, w, omw;
};

// weighted Jacobi sweep of the pressure operator (the multigrid variant of
// JacobiDiffuse::JacobiStep, dsign = -1), FP32
__global__ void k_mx_jacobi(float *__restrict__ out, const float *__restrict__ in, const float *__restrict__ b,
                            const uint8_t *__restrict__ flags, Level L, Box3 box, CoefF c,
                            const LoopState *__restrict__ pred) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    if (pred && !pred->cond) return;
    MX_COLUMN(box);
    if (!col) return;
    const int64_t nj = L.Nx, nk = L.nxy();
    for (int64_t k = box.z0 + blockIdx.z; k <= box.z1; k += gridDim.z) {
        const int64_t x = i + nj * j + nk * k;
        if (!(flags[x] & kInner)) continue;
        const float h = c.beta * (-b[x] + c.ax * (in[x + 1] + in[x - 1]) + c.ay * (in[x + nj] + in[x - nj]) +
                                  c.az * (in[x + nk] + in[x - nk]));
        out[x] = c.omw * in[x] + c.w * h;
    }
}

// residual q = b - A e on inner cells, FP32 (VCycleMG::Residuum)
__global__ void k_mx_residuum(float *__restrict__ out, const float *__restrict__ e, const float *__restrict__ b,
                              const uint8_t *__restrict__ flags, Level L, Box3 box, float rx, float ry, float rz,
                              const LoopState *__restrict__ pred) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    if (pred && !pred->cond) return;
    MX_COLUMN(box);
    if (!col) return;
    const int64_t nj = L.Nx, nk = L.nxy();
    for (int64_t k = box.z0 + blockIdx.z; k <= box.z1; k += gridDim.z) {
        const int64_t x = i + nj * j + nk * k;
        if (!(flags[x] & kInner)) continue;
        const float c2 = 2.f * e[x];
        out[x] = b[x] - (rx * (e[x - 1] - c2 + e[x + 1]) + ry * (e[x - nj] - c2 + e[x + nj]) +
                         rz * (e[x - nk] - c2 + e[x + nk]));
    }
}

// coarse inner cell = mean of its 8 children (VCycleMG::Restrict), FP32
__global__ void k_mx_restrict(float *__restrict__ out, const float *__restrict__ in,
                              const uint8_t *__restrict__ flags, Level C, Level F, Box3 box,
                              const LoopState *__restrict__ pred) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    if (pred && !pred->cond) return;
    MX_COLUMN(box);
    if (!col) return;
    const int64_t fx = F.Nx, fxy = F.nxy();
    for (int64_t k = box.z0 + blockIdx.z; k <= box.z1; k += gridDim.z) {
        const int64_t x = i + C.Nx * j + C.nxy() * k;
        if (!(flags[x] & kInner)) continue;
        const int64_t f = (2 * i - 1) + fx * (2 * j - 1) + fxy * (2 * k - 1);
        out[x] = 0.125f * (in[f] + in[f + 1] + in[f + fx] + in[f + fx + 1] + in[f + fxy] + in[f + fxy + 1] +
                           in[f + fxy + fx] + in[f + fxy + fx + 1]);
    }
}

// first Jacobi sweep from a zero correction: every neighbour is zero, so
// e = w * beta * (-b) on the inner cells
__global__ void k_mx_jacobi0(float *__restrict__ out, const float *__restrict__ b, const uint8_t *__restrict__ flags,
                             Level L, Box3 box, CoefF c, const LoopState *__restrict__ pred) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    if (pred && !pred->cond) return;
    MX_COLUMN(box);
    if (!col) return;
    const int64_t nj = L.Nx, nk = L.nxy();
    for (int64_t k = box.z0 + blockIdx.z; k <= box.z1; k += gridDim.z) {
        const int64_t x = i + nj * j + nk * k;
        if (!(flags[x] & kInner)) continue;
        out[x] = c.w * (c.beta * -b[x]);
    }
}

// fine correction += trilinear prolongation of the coarse correction
// (weights 27/9/3/1 over 64 of VCycleMG::Prolongate), on the fine inner
// children of each coarse inner cell, FP32
__global__ void k_mx_prolong_add(float *__restrict__ fine, const float *__restrict__ in,
                                 const uint8_t *__restrict__ cflags, const uint8_t *__restrict__ fflags, Level C,
                                 Level F, Box3 box, const LoopState *__restrict__ pred) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    if (pred && !pred->cond) return;
    MX_COLUMN(box);
    if (!col) return;
    const int64_t nj = C.Nx, nk = C.nxy();
    const int64_t fx = F.Nx, fxy = F.nxy();
    for (int64_t k = box.z0 + blockIdx.z; k <= box.z1; k += gridDim.z) {
        const int64_t x = i + nj * j + nk * k;
        if (!(cflags[x] & kInner)) continue;
#pragma unroll
        for (int c = 0; c < 8; c++) {
            const int sx = (c & 1) ? 1 : -1, sy = (c & 2) ? 1 : -1, sz = (c & 4) ? 1 : -1;
            const int64_t f = (2 * i - (sx < 0)) + fx * (2 * j - (sy < 0)) + fxy * (2 * k - (sz < 0));
            if (!(fflags[f] & kInner)) continue;
            const float v = 0.015625f * (27.f * in[x] + 9.f * in[x + sx] + 9.f * in[x + sy * nj] + 9.f * in[x + sz * nk] +
                                         3.f * in[x + sx + sy * nj] + 3.f * in[x + sx + sz * nk] +
                                         3.f * in[x + sy * nj + sz * nk] + in[x + sx + sy * nj + sz * nk]);
            fine[f] += v;
        }
    }
}

// FP64 outer residual r = b - A p on level 0, stored as the FP32 right-hand
// side of the correction equation; block partials of ||r||^2
__global__ void k_mx_outer_residual(const double *__restrict__ p, const double *__restrict__ b,
                                    float *__restrict__ r, const uint8_t *__restrict__ flags, Level L, Box3 box,
                                    double rx, double ry, double rz, double *__restrict__ partials,
                                    const LoopState *__restrict__ pred) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    __shared__ double smem[32];
    if (pred && !pred->cond) return;
    MX_COLUMN(box);
    const int64_t nj = L.Nx, nk = L.nxy();
    double acc = 0.0;
    if (col) {
        for (int64_t k = box.z0 + blockIdx.z; k <= box.z1; k += gridDim.z) {
            const int64_t x = i + nj * j + nk * k;
            if (!(flags[x] & kInner)) continue;
            const double c2 = 2 * p[x];
            const double v = b[x] - (rx * (p[x - 1] - c2 + p[x + 1]) + ry * (p[x - nj] - c2 + p[x + nj]) +
                                     rz * (p[x - nk] - c2 + p[x + nk]));
            r[x] = (float) v;
            acc += v * v;
        }
    }
    acc = artss_block_sum(acc, smem);
    if (threadIdx.x == 0 && threadIdx.y == 0)
        partials[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = acc;
}

// p += e on the inner cells (FP64 += FP32)
__global__ void k_mx_correct(double *__restrict__ p, const float *__restrict__ e, const uint8_t *__restrict__ flags,
                             Level L, Box3 box, const LoopState *__restrict__ pred) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    if (pred && !pred->cond) return;
    MX_COLUMN(box);
    if (!col) return;
    const int64_t nj = L.Nx, nk = L.nxy();
    for (int64_t k = box.z0 + blockIdx.z; k <= box.z1; k += gridDim.z) {
        const int64_t x = i + nj * j + nk * k;
        if (!(flags[x] & kInner)) continue;
        p[x] += (double) e[x];
    }
}

// block partials of sum(x - shift) and sum((x - shift)^2) over the inner cells
__global__ void k_mx_moments(const double *__restrict__ x, double shift, const uint8_t *__restrict__ flags, Level L,
                             Box3 box, double *__restrict__ p1, double *__restrict__ p2) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    __shared__ double smem[32];
    MX_COLUMN(box);
    const int64_t nj = L.Nx, nk = L.nxy();
    double s1 = 0.0, s2 = 0.0;
    if (col) {
        for (int64_t k = box.z0 + blockIdx.z; k <= box.z1; k += gridDim.z) {
            const int64_t q = i + nj * j + nk * k;
            if (!(flags[q] & kInner)) continue;
            const double v = x[q] - shift;
            s1 += v;
            s2 += v * v;
        }
    }
    const int bl = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    s1 = artss_block_sum(s1, smem);
    if (threadIdx.x == 0 && threadIdx.y == 0) p1[bl] = s1;
    __syncthreads();
    s2 = artss_block_sum(s2, smem);
    if (threadIdx.x == 0 && threadIdx.y == 0) p2[bl] = s2;
}

// out = A p on the inner cells (FP64)
__global__ void k_mx_laplacian(double *__restrict__ out, const double *__restrict__ p,
                               const uint8_t *__restrict__ flags, Level L, Box3 box, double rx, double ry, double rz) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    MX_COLUMN(box);
    if (!col) return;
    const int64_t nj = L.Nx, nk = L.nxy();
    for (int64_t k = box.z0 + blockIdx.z; k <= box.z1; k += gridDim.z) {
        const int64_t x = i + nj * j + nk * k;
        if (!(flags[x] & kInner)) continue;
        const double c2 = 2 * p[x];
        out[x] = rx * (p[x - 1] - c2 + p[x + 1]) + ry * (p[x - nj] - c2 + p[x + nj]) + rz * (p[x - nk] - c2 + p[x + nk]);
    }
}

__global__ void k_mx_fill(float *__restrict__ f, int64_t n, const LoopState *__restrict__ pred) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    if (pred && !pred->cond) return;
    for (int64_t q = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; q < n; q += (int64_t) gridDim.x * blockDim.x)
        f[q] = 0.f;
}

}  // namespace

namespace {

constexpr int kSlotOuter = 6;  // device loop state of the outer iteration
constexpr int kSlotSum = 7;    // plain sums

CoefF coef_f(const artss_ctx *ctx, int level, double w) {
    const artss_grid_desc &g = ctx->grid;
    const double ax = 1. / (g.dx[level] * g.dx[level]), ay = 1. / (g.dy[level] * g.dy[level]),
                 az = 1. / (g.dz[level] * g.dz[level]);
    return CoefF{(float) ax, (float) ay, (float) az, (float) (1. / (2. * (ax + ay + az))), (float) w, (float) (1. - w)};
}

int mx_bc(artss_mixed *m, float *f, int level, const LoopState *pred) {
    return apply_bc_f32(m->ctx, f, level, ARTSS_FIELD_P, pred);
}

// n_relax weighted-Jacobi sweeps from e = 0 on level l, each followed by the
// boundary program; the result is left in m->e[l]
int mx_smooth_from_zero(artss_mixed *m, int l, const LoopState *pred) {
    artss_ctx *ctx = m->ctx;
    const Level &L = ctx->lvl[l];
    const Box3 box = inner_box(L);
    const CoefF c = coef_f(ctx, l, m->cfg.w);
    int st;
    ARTSS_LAUNCH_PDL(ctx, FAM_MG_JACOBI, k_mx_jacobi0, mx_grid(box), box_block(), 0, 
                                         m->e[l], m->r[l], ctx->d_flags[l], L, box, c, pred);
    ARTSS_LAUNCH_CK(ctx);
    if ((st = mx_bc(m, m->e[l], l, pred))) return st;
    for (int s = 1; s < m->cfg.n_relax; s++) {
        ARTSS_LAUNCH_PDL(ctx, FAM_MG_JACOBI, k_mx_jacobi, mx_grid(box), box_block(), 0, 
                                             m->t[l], m->e[l], m->r[l], ctx->d_flags[l], L, box, c, pred);
        ARTSS_LAUNCH_CK(ctx);
        std::swap(m->e[l], m->t[l]);
        if ((st = mx_bc(m, m->e[l], l, pred))) return st;
    }
    return ARTSS_OK;
}

// n_relax weighted-Jacobi sweeps continuing from m->e[l]
int mx_smooth(artss_mixed *m, int l, const LoopState *pred) {
    artss_ctx *ctx = m->ctx;
    const Level &L = ctx->lvl[l];
    const Box3 box = inner_box(L);
    const CoefF c = coef_f(ctx, l, m->cfg.w);
    int st;
    for (int s = 0; s < m->cfg.n_relax; s++) {
        ARTSS_LAUNCH_PDL(ctx, FAM_MG_JACOBI, k_mx_jacobi, mx_grid(box), box_block(), 0, 
                                             m->t[l], m->e[l], m->r[l], ctx->d_flags[l], L, box, c, pred);
        ARTSS_LAUNCH_CK(ctx);
        std::swap(m->e[l], m->t[l]);
        if ((st = mx_bc(m, m->e[l], l, pred))) return st;
    }
    return ARTSS_OK;
}

// FP32 V-cycle on A e = r[0] with e = 0 at start; result in m->e[0]
int mx_vcycle(artss_mixed *m, const LoopState *pred) {
    artss_ctx *ctx = m->ctx;
    const int Lc = m->L - 1;  // coarsest level
    const artss_grid_desc &g = ctx->grid;
    int st;
    for (int l = 0; l < Lc; l++) {
        if ((st = mx_smooth_from_zero(m, l, pred))) return st;
        const Level &L = ctx->lvl[l];
        const Box3 box = inner_box(L);
        ARTSS_LAUNCH_PDL(ctx, FAM_MG_RESIDUUM, k_mx_residuum, mx_grid(box), box_block(), 0, 
                                               m->q[l], m->e[l], m->r[l], ctx->d_flags[l], L, box,
                                               (float) (1. / (g.dx[l] * g.dx[l])), (float) (1. / (g.dy[l] * g.dy[l])),
                                               (float) (1. / (g.dz[l] * g.dz[l])), pred);
        ARTSS_LAUNCH_CK(ctx);
        if ((st = mx_bc(m, m->q[l], l, pred))) return st;
        const Level &C = ctx->lvl[l + 1];
        const Box3 cbox = inner_box(C);
        ARTSS_LAUNCH_PDL(ctx, FAM_MG_RESTRICT, k_mx_restrict, mx_grid(cbox), box_block(), 0, 
                                               m->r[l + 1], m->q[l], ctx->d_flags[l + 1], C, L, cbox, pred);
        ARTSS_LAUNCH_CK(ctx);
    }
    // coarsest level: FP64 solve from zero
    {
        const int64_t n = ctx->lvl[Lc].size();
        ARTSS_LAUNCH_PDL(ctx, FAM_FIELD_OP, k_mx_fill, flat_blocks(n), 256, 0, m->e[Lc], n, pred);
        ARTSS_LAUNCH_CK(ctx);
        double w = m->cfg.coarse_w;
        if (w <= 0) {
            // red-black SOR with the optimal weight of the model problem on this grid
            const Level &C = ctx->lvl[Lc];
            const double n = (double) std::max({C.i2 - C.i1 + 1, C.j2 - C.j1 + 1, C.k2 - C.k1 + 1});
            w = m->cfg.coarse_smoother == ARTSS_SMOOTHER_CGS ? 2. / (1. + sin(M_PI / (n + 1.))) : 0.6666666667;
        }
        if ((st = coarse_cluster_f32(ctx, m->e[Lc], m->r[Lc], Lc, m->cfg.coarse_smoother, w, m->cfg.coarse_rel_tol,
                                     m->cfg.coarse_max_iter, pred)))
            return st;
    }
    for (int l = Lc - 1; l >= 0; l--) {
        const Level &C = ctx->lvl[l + 1], &F = ctx->lvl[l];
        const Box3 cbox = inner_box(C);
        ARTSS_LAUNCH_PDL(ctx, FAM_MG_PROLONGATE, k_mx_prolong_add, mx_grid(cbox), box_block(), 0, 
                                                 m->e[l], m->e[l + 1], ctx->d_flags[l + 1], ctx->d_flags[l], C, F,
                                                 cbox, pred);
        ARTSS_LAUNCH_CK(ctx);
        if ((st = mx_bc(m, m->e[l], l, pred))) return st;
        if ((st = mx_smooth(m, l, pred))) return st;
    }
    return ARTSS_OK;
}

// sum(x - shift) and sum((x - shift)^2) over level-0 inner cells, read back
int mx_moments(artss_mixed *m, const double *x, double shift, double *s1, double *s2) {
    artss_ctx *ctx = m->ctx;
    const Level &L = ctx->lvl[0];
    const Box3 box = inner_box(L);
    const dim3 grid = mx_grid(box);
    int st;
    if ((st = check_reduce_blocks(grid))) return st;
    const int nb = (int) (grid.x * grid.y * grid.z);
    ARTSS_LAUNCH_PDL(ctx, FAM_MG_RESNORM, k_mx_moments, grid, box_block(), 0, 
                                          x, shift, ctx->d_flags[0], L, box, ctx->d_partials, ctx->d_partials + nb);
    ARTSS_LAUNCH_CK(ctx);
    LoopState a{}, b{};
    if ((st = finalize_sum(ctx, kSlotSum, nb))) return st;
    if ((st = read_loop(ctx, kSlotSum, &a))) return st;
    ARTSS_CK(cudaMemcpyAsync(ctx->d_partials, ctx->d_partials + nb, nb * sizeof(double), cudaMemcpyDeviceToDevice,
                             ctx->stream));
    if ((st = finalize_sum(ctx, kSlotSum, nb))) return st;
    if ((st = read_loop(ctx, kSlotSum, &b))) return st;
    *s1 = a.sum;
    *s2 = b.sum;
    return ARTSS_OK;
}

}  // namespace
}  // namespace artss

using namespace artss;

extern "C" {

int artss_mixed_create(artss_ctx *ctx, const artss_mixed_cfg *cfg, artss_mixed **out) {
    if (!ctx || !cfg || !out) { set_error("null argument"); return ARTSS_ERR_ARG; }
    *out = nullptr;
    if (cfg->n_level < 2 || cfg->n_level > ctx->grid.n_levels + 1) {
        set_error("n_level must be at least 2 and at most the context's levels + 1"); return ARTSS_ERR_ARG;
    }
    if (cfg->n_relax < 1 || cfg->max_cycles < 0 || cfg->coarse_max_iter < 0 || !(cfg->rel_tol >= 0) ||
        (cfg->coarse_smoother != ARTSS_SMOOTHER_JACOBI && cfg->coarse_smoother != ARTSS_SMOOTHER_CGS)) {
        set_error("invalid mixed-precision settings"); return ARTSS_ERR_ARG;
    }
    auto *m = new artss_mixed();
    m->ctx = ctx;
    m->cfg = *cfg;
    m->L = cfg->n_level;
    int st = ARTSS_OK;
    for (int l = 0; l < m->L && !st; l++) {
        const size_t bytes = (size_t) ctx->lvl[l].size() * sizeof(float);
        for (float **f : {&m->r[l], &m->q[l], &m->e[l], &m->t[l]}) {
            cudaError_t e = cudaMalloc((void **) f, bytes);
            if (e == cudaSuccess) e = cudaMemsetAsync(*f, 0, bytes, ctx->stream);
            if (e != cudaSuccess) { st = cuda_fail(e, "mixed-precision level arrays"); break; }
        }
    }
    if (!st) {
        int cap = 0;
        int64_t smem = 0;
        if (!cluster_fits(ctx, m->L - 1, cfg->coarse_smoother == ARTSS_SMOOTHER_CGS ? 1 : 2, &cap, &smem)) {
            set_error("the coarsest level is too large for the cluster coarse solve; use more levels");
            st = ARTSS_ERR_LIMIT;
        }
    }
    if (!st) st = cudaStreamSynchronize(ctx->stream) == cudaSuccess ? ARTSS_OK : cuda_fail(cudaGetLastError(), "sync");
    if (st) { artss_mixed_destroy(m); return st; }
    *out = m;
    return ARTSS_OK;
}

int artss_mixed_destroy(artss_mixed *m) {
    if (!m) return ARTSS_OK;
    cudaStreamSynchronize(m->ctx->stream);
    for (int l = 0; l <= kMaxLevel; l++)
        for (float *f : {m->r[l], m->q[l], m->e[l], m->t[l]})
            if (f) cudaFree(f);
    delete m;
    return ARTSS_OK;
}

int artss_laplacian(artss_ctx *ctx, double *out, double *p, int level) {
    if (!ctx || !out || !p || out == p) { set_error("null or aliased argument"); return ARTSS_ERR_ARG; }
    int st = check_level(ctx, level);
    if (st) return st;
    if ((st = apply_bc(ctx, p, level, ARTSS_FIELD_P))) return st;
    const Level &L = ctx->lvl[level];
    const Box3 box = inner_box(L);
    const artss_grid_desc &g = ctx->grid;
    ARTSS_LAUNCH_PDL(ctx, FAM_MG_RESIDUUM, k_mx_laplacian, mx_grid(box), box_block(), 0, 
                                           out, p, ctx->d_flags[level], L, box, 1. / (g.dx[level] * g.dx[level]),
                                           1. / (g.dy[level] * g.dy[level]), 1. / (g.dz[level] * g.dz[level]));
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

int artss_mixed_solve(artss_mixed *m, double *p, const double *b, artss_solve_stats *stats) {
    if (!m || !p || !b) { set_error("null argument"); return ARTSS_ERR_ARG; }
    artss_ctx *ctx = m->ctx;
    const Level &L = ctx->lvl[0];
    const Box3 box = inner_box(L);
    const artss_grid_desc &g = ctx->grid;
    const bool remove_mean = (m->cfg.flags & ARTSS_MIXED_REMOVE_MEAN) != 0;
    const int64_t n_inner = ctx->n_inner[0];
    int st;
    const dim3 grid = mx_grid(box);
    if ((st = check_reduce_blocks(grid))) return st;
    const int nb = (int) (grid.x * grid.y * grid.z);
    // ||b|| for the relative stopping rule: on the host, or (inside a capture)
    // kept in loop slot kSlotSum and applied by the loop step on the device
    double s1 = 0, s2 = 0;
    if (ctx->capturing) {
        if (remove_mean) { set_error("the mean removal reads sums on the host and cannot be captured"); return ARTSS_ERR_ARG; }
        ARTSS_LAUNCH_PDL(ctx, FAM_MG_RESNORM, k_mx_moments, grid, box_block(), 0, 
                                              b, 0.0, ctx->d_flags[0], L, box, ctx->d_partials, ctx->d_partials + nb);
        ARTSS_LAUNCH_CK(ctx);
        ARTSS_CK(cudaMemcpyAsync(ctx->d_partials, ctx->d_partials + nb, nb * sizeof(double), cudaMemcpyDeviceToDevice,
                                 ctx->stream));
        if ((st = finalize_sum(ctx, kSlotSum, nb))) return st;
    } else if ((st = mx_moments(m, b, 0.0, &s1, &s2))) {
        return st;
    }
    const double b_norm = sqrt(s2);
    const double tol = m->cfg.rel_tol * b_norm;
    if ((st = apply_bc(ctx, p, 0, ARTSS_FIELD_P))) return st;

    const double rx = 1. / (g.dx[0] * g.dx[0]), ry = 1. / (g.dy[0] * g.dy[0]), rz = 1. / (g.dz[0] * g.dz[0]);
    const long long max_eval = m->cfg.max_cycles + 1;
    if ((st = init_loop(ctx, kSlotOuter, 1e300, 0, 1))) return st;
    const LoopState *pred = ctx->d_loop + kSlotOuter;
    LoopState ls{};
    long long it = 0;
    bool cond = true;
    int64_t batch = std::max<int64_t>(1, std::min<int64_t>(m->hint, max_eval));
    GraphLoop gl;
    if (ctx->capturing) {
        // one outer iteration per body of a WHILE node decided on the device
        if ((st = gl.begin(ctx, 1))) return st;
        batch = 1;
    }
    while (cond) {
        for (int64_t r = 0; r < batch; r++) {
            ARTSS_LAUNCH_PDL(ctx, FAM_MG_RESNORM, k_mx_outer_residual, grid, box_block(), 0, 
                                                  p, b, m->r[0], ctx->d_flags[0], L, box, rx, ry, rz,
                                                  ctx->d_partials, pred);
            ARTSS_LAUNCH_CK(ctx);
            if (ctx->capturing) st = finalize_loop_rel(ctx, kSlotOuter, nb, m->cfg.rel_tol, kSlotSum, max_eval);
            else st = finalize_loop(ctx, kSlotOuter, nb, tol, max_eval);
            if (st) return st;
            if ((st = mx_vcycle(m, pred))) return st;
            ARTSS_LAUNCH_PDL(ctx, FAM_FIELD_OP, k_mx_correct, grid, box_block(), 0, 
                                                p, m->e[0], ctx->d_flags[0], L, box, pred);
            ARTSS_LAUNCH_CK(ctx);
            if ((st = apply_bc(ctx, p, 0, ARTSS_FIELD_P, pred))) return st;
        }
        if (ctx->capturing) {
            if ((st = gl.end(kSlotOuter, max_eval + 2))) return st;
            if (stats) *stats = artss_solve_stats{-1, -1.0, -1.0, -1.0};
            return ARTSS_OK;
        }
        if ((st = read_loop(ctx, kSlotOuter, &ls))) return st;
        it = ls.it;
        cond = ls.cond != 0;
        batch = std::max<int64_t>(1, std::min<int64_t>(2 * batch, max_eval - it));
    }
    m->hint = std::max<int64_t>(1, it);
    if (remove_mean && n_inner > 0) {
        double p1 = 0, p2 = 0;
        if ((st = mx_moments(m, p, 0.0, &p1, &p2))) return st;
        // a uniform shift keeps every Neumann ghost relation
        if ((st = artss_add_scalar(ctx, p, -p1 / (double) n_inner, 0))) return st;
    }
    if (stats) {
        stats->cycles = it - 1;
        stats->residual = ls.residual;
        stats->rel_residual = b_norm > 0 ? ls.residual / b_norm : ls.residual;
        stats->b_norm = b_norm;
    }
    return ARTSS_OK;
}

}  // extern "C"
