// Geometric multigrid pressure solver, VCycleMG of ARTSS
// (src/pressure/VCycleMG.cpp:17-798), FP64.
//
// The V-cycle visits the levels in the reference's order with the reference's
// quirks preserved: the "coarse solve" runs on level n_level-1 while the
// coarsest level only carries the restricted residual (VCycleMG.cpp:229-281);
// Jacobi smoothing ping-pongs two arrays and, for an even number of sweeps,
// hands back the second-to-last iterate (:699-722, pointer swaps); every
// smoothing sweep and transfer is followed by the level's boundary program.
#include "internal.cuh"

#include <algorithm>

struct artss_mg {
    artss_ctx *ctx = nullptr;
    artss_mg_cfg cfg{};
    int L = 0;
    double *r0[artss::kMaxLevel + 1]{};   // residuum0[level]   (levels 0..L-1)
    double *r1[artss::kMaxLevel + 1]{};   // residuum1[level]   (levels 0..L)
    double *e0[artss::kMaxLevel + 1]{};   // error0[level]      (levels 0..L-1)
    double *e1[artss::kMaxLevel + 1]{};   // error1[level]      (levels 0..L)
    double *tmp[artss::kMaxLevel + 1]{};  // temporal solution  (levels 0..L)
};

namespace artss {

inline dim3 mg_grid(const Box3 &b) {
    dim3 g = box_grid(b);
    const int64_t xy = (int64_t) g.x * g.y;
    int64_t gz = b.nz();
    const int64_t cap = std::max<int64_t>(1, 2048 / std::max<int64_t>(xy, 1));
    if (gz > cap) gz = cap;
    g.z = (unsigned) std::max<int64_t>(gz, 1);
    return g;
}

#define MG_COLUMN(box)                                                     \
    const int64_t i = (box).x0 + (int64_t) blockIdx.x * blockDim.x + threadIdx.x; \
    const int64_t j = (box).y0 + (int64_t) blockIdx.y * blockDim.y + threadIdx.y; \
    const bool col = (i <= (box).x1) && (j <= (box).y1)

struct MgCoef {
    double ax, ay, az;   // 1/(dx*dx) ... of the level (VCycleMG.cpp:595-601)
    double beta;         // 1/(2 (ax+ay+az))
    double dsign, w, omw;
};

// JacobiDiffuse::JacobiStep, multigrid variant (JacobiDiffuse.cpp:274-305)
__global__ void k_mg_jacobi(double *__restrict__ out, const double *__restrict__ in, const double *__restrict__ b,
                            const uint8_t *__restrict__ flags, Level L, Box3 box, MgCoef c) {
    MG_COLUMN(box);
    if (!col) return;
    const int64_t nj = L.Nx, nk = L.nxy();
    for (int64_t k = box.z0 + blockIdx.z; k <= box.z1; k += gridDim.z) {
        const int64_t q = i + L.Nx * j + nk * k;
        if (!(flags[q] & kInner)) continue;
        const double out_h = c.beta * (c.dsign * b[q] + c.ax * (in[q + 1] + in[q - 1]) +
                                       c.ay * (in[q + nj] + in[q - nj]) + c.az * (in[q + nk] + in[q - nk]));
        out[q] = c.omw * in[q] + c.w * out_h;
    }
}

// colored Gauss-Seidel stencil with the multigrid coefficients
// (ColoredGaussSeidelDiffuse.cpp:316-341 called from VCycleMG.cpp:608-616)
__global__ void k_mg_cgs_color(double *__restrict__ out, const double *__restrict__ b,
                               const uint8_t *__restrict__ flags, Level L, Box3 box, int color, MgCoef c) {
    MG_COLUMN(box);
    if (!col) return;
    const int64_t nj = L.Nx, nk = L.nxy();
    for (int64_t k = box.z0 + blockIdx.z; k <= box.z1; k += gridDim.z) {
        if (((i + j + k) & 1) != color) continue;
        const int64_t q = i + L.Nx * j + nk * k;
        if (!(flags[q] & kInner)) continue;
        const double out_h = c.beta * (c.dsign * b[q] + c.ax * (out[q + 1] + out[q - 1]) +
                                       c.ay * (out[q + nj] + out[q - nj]) + c.az * (out[q + nk] + out[q - nk]));
        out[q] = c.omw * out[q] + c.w * out_h;
    }
}

// VCycleMG::Residuum (VCycleMG.cpp:346-354)
__global__ void k_mg_residuum(double *__restrict__ out, const double *__restrict__ in, const double *__restrict__ b,
                              const uint8_t *__restrict__ flags, Level L, Box3 box, double rx, double ry, double rz) {
    MG_COLUMN(box);
    if (!col) return;
    const int64_t nj = L.Nx, nk = L.nxy();
    for (int64_t k = box.z0 + blockIdx.z; k <= box.z1; k += gridDim.z) {
        const int64_t q = i + L.Nx * j + nk * k;
        if (!(flags[q] & kInner)) continue;
        const double weighted = (rx * (in[q - 1] - 2 * in[q] + in[q + 1]) + ry * (in[q - nj] - 2 * in[q] + in[q + nj]) +
                                 rz * (in[q - nk] - 2 * in[q] + in[q + nk]));
        out[q] = b[q] - weighted;
    }
}

// block partials of sum (b - A x)^2 over the level's inner cells
// (VCycleMG.cpp:186-194, :668-679, :777-788)
__global__ void k_mg_resnorm(const double *__restrict__ x, const double *__restrict__ b,
                             const uint8_t *__restrict__ flags, Level L, Box3 box, double rx, double ry, double rz,
                             double *__restrict__ partials, double *__restrict__ partials_b) {
    __shared__ double smem[32];
    MG_COLUMN(box);
    const int64_t nj = L.Nx, nk = L.nxy();
    double acc = 0.0, accb = 0.0;
    if (col) {
        for (int64_t k = box.z0 + blockIdx.z; k <= box.z1; k += gridDim.z) {
            const int64_t q = i + L.Nx * j + nk * k;
            if (!(flags[q] & kInner)) continue;
            const double r = b[q] - (rx * (x[q - 1] - 2 * x[q] + x[q + 1]) + ry * (x[q - nj] - 2 * x[q] + x[q + nj]) +
                                     rz * (x[q - nk] - 2 * x[q] + x[q + nk]));
            acc += r * r;
            accb += b[q] * b[q];
        }
    }
    const int bl = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    acc = artss_block_sum(acc, smem);
    if (threadIdx.x == 0 && threadIdx.y == 0) partials[bl] = acc;
    if (partials_b) {
        __syncthreads();
        accb = artss_block_sum(accb, smem);
        if (threadIdx.x == 0 && threadIdx.y == 0) partials_b[bl] = accb;
    }
}

// VCycleMG::Restrict (VCycleMG.cpp:402-421), over coarse inner cells
__global__ void k_mg_restrict(double *__restrict__ out, const double *__restrict__ in,
                              const uint8_t *__restrict__ flags, Level C, Level F, Box3 box) {
    MG_COLUMN(box);
    if (!col) return;
    const int64_t fx = F.Nx, fxy = F.nxy();
    for (int64_t k = box.z0 + blockIdx.z; k <= box.z1; k += gridDim.z) {
        const int64_t q = i + C.Nx * j + C.nxy() * k;
        if (!(flags[q] & kInner)) continue;
        const int64_t a = 2 * i - 1, bx = 2 * i, c = 2 * j - 1, d = 2 * j, e = 2 * k - 1, f = 2 * k;
        out[q] = 0.125 * (in[a + fx * c + fxy * e] + in[bx + fx * c + fxy * e] + in[a + fx * d + fxy * e] +
                          in[bx + fx * d + fxy * e] + in[a + fx * c + fxy * f] + in[bx + fx * c + fxy * f] +
                          in[a + fx * d + fxy * f] + in[bx + fx * d + fxy * f]);
    }
}

// VCycleMG::Prolongate (VCycleMG.cpp:464-546): 8 fine cells per coarse inner cell
__global__ void k_mg_prolongate(double *__restrict__ out, const double *__restrict__ in,
                                const uint8_t *__restrict__ flags, Level C, Level F, Box3 box) {
    MG_COLUMN(box);
    if (!col) return;
    const int64_t ni = 1, nj = C.Nx, nk = C.nxy();
    const int64_t fx = F.Nx, fxy = F.nxy();
    for (int64_t k = box.z0 + blockIdx.z; k <= box.z1; k += gridDim.z) {
        const int64_t q = i + C.Nx * j + C.nxy() * k;
        if (!(flags[q] & kInner)) continue;
        // sx, sy, sz in {+1, -1}: fine cell 2i (+) or 2i-1 (-) per axis
#define ARTSS_PROLONG(SX, SY, SZ, FI, FJ, FK)                                                         \
        out[(FI) + fx * (FJ) + fxy * (FK)] =                                                          \
            0.015625 * (27 * in[q] + 9 * in[q + (SX) * ni] + 9 * in[q + (SY) * nj] + 9 * in[q + (SZ) * nk] \
                        + 3 * in[q + (SX) * ni + (SY) * nj] + 3 * in[q + (SX) * ni + (SZ) * nk]        \
                        + 3 * in[q + (SY) * nj + (SZ) * nk] + in[q + (SX) * ni + (SY) * nj + (SZ) * nk]);
        ARTSS_PROLONG(1, 1, 1, 2 * i, 2 * j, 2 * k)
        ARTSS_PROLONG(1, 1, -1, 2 * i, 2 * j, 2 * k - 1)
        ARTSS_PROLONG(1, -1, 1, 2 * i, 2 * j - 1, 2 * k)
        ARTSS_PROLONG(1, -1, -1, 2 * i, 2 * j - 1, 2 * k - 1)
        ARTSS_PROLONG(-1, 1, 1, 2 * i - 1, 2 * j, 2 * k)
        ARTSS_PROLONG(-1, 1, -1, 2 * i - 1, 2 * j, 2 * k - 1)
        ARTSS_PROLONG(-1, -1, 1, 2 * i - 1, 2 * j - 1, 2 * k)
        ARTSS_PROLONG(-1, -1, -1, 2 * i - 1, 2 * j - 1, 2 * k - 1)
#undef ARTSS_PROLONG
    }
}

MgCoef mg_coef(const artss_mg *mg, int level) {
    const artss_grid_desc &g = mg->ctx->grid;
    MgCoef c{};
    c.ax = 1. / (g.dx[level] * g.dx[level]);
    c.ay = 1. / (g.dy[level] * g.dy[level]);
    c.az = 1. / (g.dz[level] * g.dz[level]);
    const double rbeta = 2. * (c.ax + c.ay + c.az);
    c.beta = 1. / rbeta;
    c.dsign = -1;
    c.w = mg->cfg.smoother_w;
    c.omw = 1 - mg->cfg.smoother_w;
    return c;
}

int mg_bc(artss_mg *mg, double *f, int level) { return apply_bc(mg->ctx, f, level, ARTSS_FIELD_P); }

int mg_jacobi_step(artss_mg *mg, double *out, const double *in, const double *b, int level) {
    artss_ctx *ctx = mg->ctx;
    const Level &L = ctx->lvl[level];
    const Box3 box = inner_box(L);
    ARTSS_LAUNCH(ctx, FAM_MG_JACOBI, k_mg_jacobi<<<mg_grid(box), box_block(), 0, ctx->stream>>>(out, in, b, ctx->d_flags[level], L, box,
                                                               mg_coef(mg, level)));
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

int mg_cgs_step(artss_mg *mg, double *out, const double *b, int level) {
    artss_ctx *ctx = mg->ctx;
    const Level &L = ctx->lvl[level];
    const Box3 box = inner_box(L);
    const MgCoef c = mg_coef(mg, level);
    for (int color = 0; color < 2; color++) {
        ARTSS_LAUNCH(ctx, FAM_MG_CGS, k_mg_cgs_color<<<mg_grid(box), box_block(), 0, ctx->stream>>>(out, b, ctx->d_flags[level], L, box, color, c));
        ARTSS_LAUNCH_CK(ctx);
    }
    return ARTSS_OK;
}

// ||b - A x||_2 over the level's inner cells into loop slot `slot`
int mg_resnorm(artss_mg *mg, const double *x, const double *b, int level, int slot, double tol, long long max_it,
               bool iterate) {
    artss_ctx *ctx = mg->ctx;
    const Level &L = ctx->lvl[level];
    const Box3 box = inner_box(L);
    const artss_grid_desc &g = ctx->grid;
    const dim3 grid = mg_grid(box);
    int st = check_reduce_blocks(grid);
    if (st) return st;
    ARTSS_LAUNCH(ctx, FAM_MG_RESNORM, k_mg_resnorm<<<grid, box_block(), 0, ctx->stream>>>(x, b, ctx->d_flags[level], L, box,
                                                        1. / (g.dx[level] * g.dx[level]),
                                                        1. / (g.dy[level] * g.dy[level]),
                                                        1. / (g.dz[level] * g.dz[level]), ctx->d_partials, nullptr));
    ARTSS_LAUNCH_CK(ctx);
    const int nb = (int) (grid.x * grid.y * grid.z);
    if (iterate) return finalize_loop(ctx, slot, nb, tol, max_it);
    return finalize_loop(ctx, slot, nb, -1.0, 1);  // residual only
}

// VCycleMG::Smooth + call_smooth_{jacobi,colored_gauss_seidel} (VCycleMG.cpp:299-305, :583-723)
int mg_smooth(artss_mg *mg, double *out, double *tmp, const double *b, int level) {
    int st;
    if ((st = mg_bc(mg, out, level))) return st;   // Smooth
    if ((st = mg_bc(mg, out, level))) return st;   // call_smooth_*
    if (mg->cfg.smoother == ARTSS_SMOOTHER_CGS) {
        for (int r = 0; r < mg->cfg.n_relax; r++) {
            if ((st = mg_cgs_step(mg, out, b, level))) return st;
            if ((st = mg_bc(mg, out, level))) return st;
        }
        return ARTSS_OK;
    }
    if ((st = artss_copy(mg->ctx, tmp, out, level))) return st;
    double *A = out, *B = tmp;   // Field data pointers as swapped by Field::swap
    for (int r = 0; r < mg->cfg.n_relax; r++) {
        if ((st = mg_jacobi_step(mg, A, B, b, level))) return st;
        if ((st = mg_bc(mg, A, level))) return st;
        std::swap(A, B);
    }
    return ARTSS_OK;
}

// VCycleMG::Solve + call_solve_{jacobi,colored_gauss_seidel} (VCycleMG.cpp:562-581, :620-798)
int mg_solve(artss_mg *mg, double *out, double *tmp, const double *b, int level, int64_t *iterations) {
    artss_ctx *ctx = mg->ctx;
    const Level &L = ctx->lvl[level];
    if (L.Nx <= 4 && L.Ny <= 4) {
        if (iterations) *iterations = 0;
        return mg_smooth(mg, out, tmp, b, level);
    }
    int st;
    const int slot = 1;
    const long long max_it = mg->cfg.smoother_max_iter;
    const double tol = mg->cfg.smoother_tol_res;
    if ((st = mg_bc(mg, out, level))) return st;
    long long it = 0;
    double res = 10000.;
    bool cond = res > tol && it < max_it;
    if ((st = init_loop(ctx, slot, res, 0, cond ? 1 : 0))) return st;
    LoopState ls{};
    if (mg->cfg.smoother == ARTSS_SMOOTHER_CGS) {
        while (cond) {
            if ((st = mg_cgs_step(mg, out, b, level))) return st;
            if ((st = mg_bc(mg, out, level))) return st;
            if ((st = mg_resnorm(mg, out, b, level, slot, tol, max_it, true))) return st;
            if ((st = read_loop(ctx, slot, &ls))) return st;
            it = ls.it;
            cond = ls.cond != 0;
        }
    } else {
        if ((st = artss_copy(ctx, tmp, out, level))) return st;
        double *A = out, *B = tmp;
        while (cond) {
            if ((st = mg_jacobi_step(mg, A, B, b, level))) return st;
            if ((st = mg_bc(mg, A, level))) return st;
            if ((st = mg_resnorm(mg, A, b, level, slot, tol, max_it, true))) return st;
            std::swap(A, B);
            if ((st = read_loop(ctx, slot, &ls))) return st;
            it = ls.it;
            cond = ls.cond != 0;
        }
    }
    if (iterations) *iterations = it;
    return ARTSS_OK;
}

int mg_restrict(artss_mg *mg, double *coarse, const double *fine, int coarse_level) {
    artss_ctx *ctx = mg->ctx;
    const Level &C = ctx->lvl[coarse_level];
    const Box3 box = inner_box(C);
    ARTSS_LAUNCH(ctx, FAM_MG_RESTRICT, k_mg_restrict<<<mg_grid(box), box_block(), 0, ctx->stream>>>(coarse, fine, ctx->d_flags[coarse_level], C,
                                                                 ctx->lvl[coarse_level - 1], box));
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

int mg_prolongate(artss_mg *mg, double *fine, const double *coarse, int coarse_level) {
    artss_ctx *ctx = mg->ctx;
    const Level &C = ctx->lvl[coarse_level];
    const Box3 box = inner_box(C);
    ARTSS_LAUNCH(ctx, FAM_MG_PROLONGATE, k_mg_prolongate<<<mg_grid(box), box_block(), 0, ctx->stream>>>(fine, coarse, ctx->d_flags[coarse_level], C,
                                                                   ctx->lvl[coarse_level - 1], box));
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

int mg_residuum(artss_mg *mg, double *out, const double *in, const double *b, int level) {
    artss_ctx *ctx = mg->ctx;
    const Level &L = ctx->lvl[level];
    const Box3 box = inner_box(L);
    const artss_grid_desc &g = ctx->grid;
    ARTSS_LAUNCH(ctx, FAM_MG_RESIDUUM, k_mg_residuum<<<mg_grid(box), box_block(), 0, ctx->stream>>>(out, in, b, ctx->d_flags[level], L, box,
                                                                 1. / (g.dx[level] * g.dx[level]),
                                                                 1. / (g.dy[level] * g.dy[level]),
                                                                 1. / (g.dz[level] * g.dz[level])));
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

// VCycleMG::VCycleMultigrid (VCycleMG.cpp:215-288)
int mg_vcycle(artss_mg *mg, double *out, int64_t *coarse_its) {
    artss_ctx *ctx = mg->ctx;
    const int L = mg->L;
    int st;
    if (L == 0) return mg_solve(mg, out, mg->tmp[0], mg->r1[0], 0, coarse_its);
    if ((st = artss_copy(ctx, mg->e1[0], out, 0))) return st;
    for (int l = 0; l < L; l++) {
        if ((st = mg_smooth(mg, mg->e1[l], mg->tmp[l], mg->r1[l], l))) return st;
        if ((st = mg_residuum(mg, mg->r0[l], mg->e1[l], mg->r1[l], l))) return st;
        if ((st = mg_bc(mg, mg->r0[l], l))) return st;
        if ((st = mg_restrict(mg, mg->r1[l + 1], mg->r0[l], l + 1))) return st;
        if ((st = mg_bc(mg, mg->r1[l + 1], l + 1))) return st;
        if ((st = artss_fill(ctx, mg->e1[l + 1], l + 1, 0.0))) return st;
    }
    // out.copy_data(*m_error0[0]) at VCycleMG.cpp:254 is overwritten below
    // before anything reads it
    for (int l = L; l > 0; l--) {
        if ((st = mg_prolongate(mg, mg->e0[l - 1], mg->e1[l], l))) return st;
        if ((st = mg_bc(mg, mg->e0[l - 1], l - 1))) return st;
        if ((st = artss_add_field(ctx, mg->e1[l - 1], mg->e0[l - 1], l - 1))) return st;
        if (l == L) {
            if ((st = mg_solve(mg, mg->e1[l - 1], mg->tmp[l - 1], mg->r1[l - 1], l - 1, coarse_its))) return st;
        } else {
            if ((st = mg_smooth(mg, mg->e1[l - 1], mg->tmp[l - 1], mg->r1[l - 1], l - 1))) return st;
        }
    }
    if ((st = artss_copy(ctx, out, mg->e1[0], 0))) return st;
    return mg_bc(mg, out, 0);
}

}  // namespace artss

using namespace artss;

extern "C" {

int artss_mg_create(artss_ctx *ctx, const artss_mg_cfg *cfg, artss_mg **out) {
    if (!ctx || !cfg || !out) { set_error("null argument"); return ARTSS_ERR_ARG; }
    *out = nullptr;
    if (cfg->n_level < 0 || cfg->n_level > ctx->grid.n_levels) {
        set_error("n_level exceeds the context's levels"); return ARTSS_ERR_ARG;
    }
    if (cfg->n_cycle < 0 || cfg->n_relax < 0 || cfg->max_cycle < 0 || cfg->smoother_max_iter < 0 ||
        (cfg->smoother != ARTSS_SMOOTHER_JACOBI && cfg->smoother != ARTSS_SMOOTHER_CGS)) {
        set_error("invalid multigrid settings"); return ARTSS_ERR_ARG;
    }
    auto *mg = new artss_mg();
    mg->ctx = ctx;
    mg->cfg = *cfg;
    mg->L = cfg->n_level;
    int st = ARTSS_OK;
    // VCycleMG.cpp:51-99: level-0 r1/e1/tmp, levels 0..L-1 r0/e0, 1..L r1/e1/tmp
    st = st ? st : artss_field_alloc(ctx, 0, &mg->r1[0]);
    st = st ? st : artss_field_alloc(ctx, 0, &mg->e1[0]);
    st = st ? st : artss_field_alloc(ctx, 0, &mg->tmp[0]);
    for (int l = 0; l < mg->L && !st; l++) {
        st = st ? st : artss_field_alloc(ctx, l, &mg->r0[l]);
        st = st ? st : artss_field_alloc(ctx, l + 1, &mg->r1[l + 1]);
        st = st ? st : artss_field_alloc(ctx, l, &mg->e0[l]);
        st = st ? st : artss_field_alloc(ctx, l + 1, &mg->e1[l + 1]);
        st = st ? st : artss_field_alloc(ctx, l + 1, &mg->tmp[l + 1]);
    }
    if (st) { artss_mg_destroy(mg); return st; }
    *out = mg;
    return ARTSS_OK;
}

int artss_mg_destroy(artss_mg *mg) {
    if (!mg) return ARTSS_OK;
    for (int l = 0; l <= kMaxLevel; l++) {
        for (double *p : {mg->r0[l], mg->r1[l], mg->e0[l], mg->e1[l], mg->tmp[l]})
            if (p) artss_field_free(mg->ctx, p);
    }
    delete mg;
    return ARTSS_OK;
}

int artss_mg_set_rhs(artss_mg *mg, const double *p, const double *rhs) {
    if (!mg || !p || !rhs) { set_error("null argument"); return ARTSS_ERR_ARG; }
    // VCycleMG::UpdateInput (VCycleMG.cpp:125-132)
    int st;
    if ((st = artss_copy(mg->ctx, mg->e1[0], p, 0))) return st;
    if ((st = artss_copy(mg->ctx, mg->tmp[0], p, 0))) return st;
    return artss_copy(mg->ctx, mg->r1[0], rhs, 0);
}

int artss_mg_vcycle(artss_mg *mg, double *p) {
    if (!mg || !p) { set_error("null argument"); return ARTSS_ERR_ARG; }
    return mg_vcycle(mg, p, nullptr);
}

int artss_mg_pressure(artss_mg *mg, double *p, const double *rhs, int first_step, artss_mg_stats *stats) {
    if (!mg || !p || !rhs) { set_error("null argument"); return ARTSS_ERR_ARG; }
    int st;
    if ((st = artss_mg_set_rhs(mg, p, rhs))) return st;
    int64_t cycles = 0, coarse = 0;
    double residual = -1.0;
    if (first_step) {
        // VCycleMG.cpp:150-197
        const long long max_cycles = mg->cfg.max_cycle;
        const long long max_relaxs = mg->cfg.smoother_max_iter;
        long long set_relax = mg->cfg.n_relax;
        double r = 10000.;
        const double tol = mg->cfg.tol_res;
        const int slot = 2;
        while (r > tol && cycles < max_cycles && set_relax < max_relaxs) {
            for (int c = 0; c < mg->cfg.n_cycle; c++) {
                if ((st = mg_vcycle(mg, p, &coarse))) return st;
                cycles++;
            }
            if ((st = mg_resnorm(mg, p, rhs, 0, slot, -1.0, 1, false))) return st;
            LoopState ls{};
            if ((st = read_loop(mg->ctx, slot, &ls))) return st;
            r = ls.residual;
            set_relax += mg->cfg.n_relax;
        }
        residual = r;
    } else {
        for (int c = 0; c < mg->cfg.n_cycle; c++) {
            if ((st = mg_vcycle(mg, p, &coarse))) return st;
            cycles++;
        }
    }
    if (stats) {
        stats->cycles = cycles;
        stats->coarse_iterations = coarse;
        stats->residual = residual;
    }
    return ARTSS_OK;
}

int artss_residual_norm(artss_ctx *ctx, const double *p, const double *b, double *res_out, double *b_norm_out) {
    if (!ctx || !p || !b) { set_error("null argument"); return ARTSS_ERR_ARG; }
    const Level &L = ctx->lvl[0];
    const Box3 box = inner_box(L);
    const artss_grid_desc &g = ctx->grid;
    const dim3 grid = mg_grid(box);
    if (int st0 = check_reduce_blocks(grid)) return st0;
    const int nb = (int) (grid.x * grid.y * grid.z);
    ARTSS_LAUNCH(ctx, FAM_MG_RESNORM, k_mg_resnorm<<<grid, box_block(), 0, ctx->stream>>>(p, b, ctx->d_flags[0], L, box, 1. / (g.dx[0] * g.dx[0]),
                                                        1. / (g.dy[0] * g.dy[0]), 1. / (g.dz[0] * g.dz[0]),
                                                        ctx->d_partials, ctx->d_partials + nb));
    ARTSS_LAUNCH_CK(ctx);
    int st;
    LoopState a{}, c{};
    if ((st = finalize_sum(ctx, 3, nb))) return st;
    if ((st = read_loop(ctx, 3, &a))) return st;
    // second pass over the b partials
    cudaError_t e = cudaMemcpyAsync(ctx->d_partials, ctx->d_partials + nb, nb * sizeof(double),
                                    cudaMemcpyDeviceToDevice, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "partials");
    if ((st = finalize_sum(ctx, 4, nb))) return st;
    if ((st = read_loop(ctx, 4, &c))) return st;
    if (res_out) *res_out = sqrt(a.sum);
    if (b_norm_out) *b_norm_out = sqrt(c.sum);
    return ARTSS_OK;
}

}  // extern "C"
