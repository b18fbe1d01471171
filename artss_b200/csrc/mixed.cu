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
#include <unordered_map>

struct artss_mixed {
    artss_ctx *ctx = nullptr;
    artss_mixed_cfg cfg{};
    int L = 0;  // levels 0 .. L-1
    float *r[artss::kMaxLevel + 1]{};    // right-hand side of level l
    float *q[artss::kMaxLevel + 1]{};    // residual of level l
    float *e[artss::kMaxLevel + 1]{};    // correction of level l
    float *t[artss::kMaxLevel + 1]{};    // Jacobi ping-pong partner of e
    // the level's homogeneous pressure program applied by the writers of the
    // inner cells instead of by a launch after each sweep (levels 0 .. L-2, when
    // fold[l]): nbm[l][x] bit 0 = inner, bits 1..7 = index of the cell's push
    // pattern in push[l]; bits 2d .. 2d + 1 of a pattern = what the boundary cell
    // x + off[d] (d: -x, +x, -y, +y, -z, +z) takes from inner cell x with value v:
    // 0 nothing, 1 +v, 2 -v
    uint8_t *nbm[artss::kMaxLevel + 1]{};
    uint16_t *push[artss::kMaxLevel + 1]{};  // 128 patterns per level (pattern 0: none)
    bool fold[artss::kMaxLevel + 1]{};
    uint64_t geom_version = ~0ull;       // ctx->geom_version the tables describe
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

// 32-bit cell indices: artss_ctx_create rejects levels of 2^31 cells or more
#define MX_COLUMN(box)                                                             \
    const int i = (int) (box).x0 + (int) (blockIdx.x * blockDim.x + threadIdx.x); \
    const int j = (int) (box).y0 + (int) (blockIdx.y * blockDim.y + threadIdx.y); \
    const bool col = (i <= (int) (box).x1) && (j <= (int) (box).y1)

struct CoefF {
    float ax, ay, az, beta, w, omw;
};

// weighted Jacobi sweep of the pressure operator (the multigrid variant of
// JacobiDiffuse::JacobiStep, dsign = -1), FP32
// store v at inner cell x and the boundary cells whose homogeneous program
// value is +-x (push bits of the neighbour mask)
__device__ __forceinline__ void mx_store(float *__restrict__ out, uint8_t mask, const uint16_t *__restrict__ push,
                                         int x, float v, int nj, int nk) {
    out[x] = v;
    if (mask >> 1) {
        const unsigned mm = __ldg(push + (mask >> 1));
        const int off[6] = {-1, 1, -nj, nj, -nk, nk};
#pragma unroll
        for (int d = 0; d < 6; d++) {
            const unsigned kind = (mm >> (2 * d)) & 3u;
            if (kind) out[x + off[d]] = kind == 1u ? v : -v;
        }
    }
}

// CORRECT (the last sweep of level 0 in a V-cycle): instead of storing the
// sweep's value v, add it to the FP64 iterate, p[x] += (double) v, which is
// k_mx_correct's update of the same value (out and push unused)
template <bool CORRECT>
__global__ void __launch_bounds__(256, 8) k_mx_jacobi(float *__restrict__ out, const float *__restrict__ in, const float *__restrict__ b,
                            const uint8_t *__restrict__ nbm, const uint16_t *__restrict__ push, Level L, Box3 box,
                            CoefF c, const LoopState *__restrict__ pred, double *__restrict__ p) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    if (pred && !pred->cond) return;
    MX_COLUMN(box);
    if (!col) return;
    const int nj = (int) L.Nx, nk = (int) L.nxy();
    column_march<2>(in, i + nj * j, nk, (int) box.z0, (int) box.z1, nbm,
        [&](int x, int, float km, float c0, float kp) {
            const float h = c.beta * (-b[x] + c.ax * (in[x + 1] + in[x - 1]) + c.ay * (in[x + nj] + in[x - nj]) +
                                      c.az * (kp + km));
            return c.omw * c0 + c.w * h;
        },
        [&](int x, int, float v, uint8_t fl) {
            if (CORRECT) p[x] = p[x] + (double) v;
            else mx_store(out, fl, push, x, v, nj, nk);
        });
}

// one colour of an in-place red-black Gauss-Seidel sweep of the same operator,
// FP32: cells with (i + j + k) % 2 == color; first != 0: the sweep starts from a
// zero correction, so the red cells get w * beta * (-b) and the black cells 0
__global__ void k_mx_rbgs(float *__restrict__ e, const float *__restrict__ b, const uint8_t *__restrict__ flags,
                          Level L, Box3 box, CoefF c, int color, int first, const LoopState *__restrict__ pred) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    if (pred && !pred->cond) return;
    MX_COLUMN(box);
    if (!col) return;
    const int nj = (int) L.Nx, nk = (int) L.nxy();
    // the cells of one colour read only cells of the other: no cell of the
    // launch is both read and written
    column_march((const float *) e, i + nj * j, nk, (int) box.z0, (int) box.z1, flags,
        [&](int x, int, float km, float c0, float kp) {
            if (first) return c.w * (c.beta * -b[x]);
            const float h = c.beta * (-b[x] + c.ax * (e[x + 1] + e[x - 1]) + c.ay * (e[x + nj] + e[x - nj]) +
                                      c.az * (kp + km));
            return c.omw * c0 + c.w * h;
        },
        [&](int x, int k, float v, auto) {
            if (((i + j + k) & 1) == color) e[x] = v;
            else if (first) e[x] = 0.f;
        });
}

// residual q = b - A e on inner cells, FP32 (VCycleMG::Residuum)
__global__ void __launch_bounds__(256, 8) k_mx_residuum(float *__restrict__ out, const float *__restrict__ e, const float *__restrict__ b,
                              const uint8_t *__restrict__ nbm, Level L, Box3 box, float rx, float ry, float rz,
                              const LoopState *__restrict__ pred) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    if (pred && !pred->cond) return;
    MX_COLUMN(box);
    if (!col) return;
    const int nj = (int) L.Nx, nk = (int) L.nxy();
    column_march<2>(e, i + nj * j, nk, (int) box.z0, (int) box.z1, nbm,
        [&](int x, int, float km, float c0, float kp) {
            const float c2 = 2.f * c0;
            return b[x] - (rx * (e[x - 1] - c2 + e[x + 1]) + ry * (e[x - nj] - c2 + e[x + nj]) +
                           rz * (km - c2 + kp));
        },
        [&](int x, int, float v, auto) { out[x] = v; });
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
    const int fx = (int) F.Nx, fxy = (int) F.nxy();
    column_planes(i + (int) C.Nx * j, (int) C.nxy(), (int) box.z0, (int) box.z1, flags,
        [&](int, int k) {
            const int f = (2 * i - 1) + fx * (2 * j - 1) + fxy * (2 * k - 1);
            return 0.125f * (in[f] + in[f + 1] + in[f + fx] + in[f + fx + 1] + in[f + fxy] + in[f + fxy + 1] +
                             in[f + fxy + fx] + in[f + fxy + fx + 1]);
        },
        [&](int x, int, float v, auto) { out[x] = v; });
}

// first Jacobi sweep from a zero correction: every neighbour is zero, so
// e = w * beta * (-b) on the inner cells
__global__ void k_mx_jacobi0(float *__restrict__ out, const float *__restrict__ b, const uint8_t *__restrict__ flags,
                             const uint16_t *__restrict__ push, Level L, Box3 box, CoefF c,
                             const LoopState *__restrict__ pred) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    if (pred && !pred->cond) return;
    MX_COLUMN(box);
    if (!col) return;
    const int nj = (int) L.Nx, nk = (int) L.nxy();
    column_planes(i + nj * j, nk, (int) box.z0, (int) box.z1, flags,
        [&](int x, int) { return c.w * (c.beta * -b[x]); },
        [&](int x, int, float v, uint8_t fl) { mx_store(out, fl, push, x, v, nj, nk); });
}

// fine correction += trilinear prolongation of the coarse correction
// (weights 27/9/3/1 over 64 of VCycleMG::Prolongate), on the fine inner
// children of each coarse inner cell, FP32
__global__ void k_mx_prolong_add(float *__restrict__ fine, const float *__restrict__ in,
                                 const uint8_t *__restrict__ cflags, const uint8_t *__restrict__ fflags,
                                 const uint16_t *__restrict__ push, Level C, Level F, Box3 fbox,
                                 const LoopState *__restrict__ pred) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    if (pred && !pred->cond) return;
    MX_COLUMN(fbox);  // one thread per fine column: fine cell 2c (side +1) or 2c - 1 (side -1) of coarse cell c
    if (!col) return;
    const int nj = (int) C.Nx, nk = (int) C.nxy();
    const int fx = (int) F.Nx, fxy = (int) F.nxy();
    const int ci = (i + 1) >> 1, cj = (j + 1) >> 1;
    const int sx = (i & 1) ? -1 : 1, sy = (j & 1) ? -1 : 1;
    struct Out { float v; uint8_t cf; };
    column_planes(i + fx * j, fxy, (int) fbox.z0, (int) fbox.z1, fflags,
        [&](int f, int k) {
            const int sz = (k & 1) ? -1 : 1;
            const int x = ci + nj * cj + nk * ((k + 1) >> 1);
            const float v = 0.015625f * (27.f * in[x] + 9.f * in[x + sx] + 9.f * in[x + sy * nj] + 9.f * in[x + sz * nk] +
                                         3.f * in[x + sx + sy * nj] + 3.f * in[x + sx + sz * nk] +
                                         3.f * in[x + sy * nj + sz * nk] + in[x + sx + sy * nj + sz * nk]);
            return Out{fine[f] + v, cflags[x]};
        },
        [&](int f, int, Out o, uint8_t fl) {
            if (o.cf & kInner) mx_store(fine, fl, push, f, o.v, fx, fxy);
        });
}

// The same prolongation, one thread per coarse column: the thread marches up
// its contiguous run of coarse planes keeping the 3 x 3 x 3 coarse
// neighbourhood in registers (one new 3 x 3 plane per step) and updates the 8
// fine children of each coarse inner cell, each with k_mx_prolong_add's
// expression, so every fine value is the same bit for bit.  The fine x pairs
// of a warp's 32 coarse columns are 64 consecutive cells.
__global__ void __launch_bounds__(256) k_mx_prolong_add8(float *__restrict__ fine, const float *__restrict__ in,
                                                         const uint8_t *__restrict__ cflags,
                                                         const uint8_t *__restrict__ fflags,
                                                         const uint16_t *__restrict__ push, Level C, Level F,
                                                         Box3 cbox, Box3 fbox, const LoopState *__restrict__ pred) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    if (pred && !pred->cond) return;
    MX_COLUMN(cbox);  // (i, j): the coarse column
    if (!col) return;
    const int nj = (int) C.Nx, nk = (int) C.nxy();
    const int fx = (int) F.Nx, fxy = (int) F.nxy();
    const int nzc = (int) cbox.nz();
    const int chunk = (nzc + (int) gridDim.z - 1) / (int) gridDim.z;
    const int k0 = (int) cbox.z0 + (int) blockIdx.z * chunk;
    const int k1 = min((int) cbox.z1, k0 + chunk - 1);
    if (k0 > k1) return;
    // w[p][b][a]: coarse value at (i + a - 1, j + b - 1, k + p - 1) for the current plane k
    float w[3][3][3];
    auto load_plane = [&](int k, float (&pl)[3][3]) {
        const int x = i + nj * j + nk * k;
#pragma unroll
        for (int b = 0; b < 3; b++)
#pragma unroll
            for (int a = 0; a < 3; a++) pl[b][a] = in[x + (a - 1) + nj * (b - 1)];
    };
    load_plane(k0 - 1, w[0]);
    load_plane(k0, w[1]);
    // fine children of this column that lie in the fine box
    const int fi0 = 2 * i - 1, fj0 = 2 * j - 1;
    const bool xa = fi0 >= (int) fbox.x0 && fi0 <= (int) fbox.x1, xb = fi0 + 1 >= (int) fbox.x0 && fi0 + 1 <= (int) fbox.x1;
    const bool ya = fj0 >= (int) fbox.y0 && fj0 <= (int) fbox.y1, yb = fj0 + 1 >= (int) fbox.y0 && fj0 + 1 <= (int) fbox.y1;
    for (int k = k0; k <= k1; k++) {
        // every load of the step first (the children lie in the fine array: 2 c <=
        // the fine inner box's end + 1), then the arithmetic and the stores
        const bool cin = (cflags[i + nj * j + nk * k] & kInner) != 0;
        uint8_t fl[8];
        float fv[8];
#pragma unroll
        for (int c = 0; c < 8; c++) {
            const int f = fi0 + (c & 1) + fx * (fj0 + ((c >> 1) & 1)) + fxy * (2 * k - 1 + (c >> 2));
            fl[c] = fflags[f];
            fv[c] = fine[f];
        }
        load_plane(k + 1, w[2]);
        if (cin) {
#pragma unroll
            for (int c = 0; c < 8; c++) {
                const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
                const int fk = 2 * k - 1 + dz;
                if (fk < (int) fbox.z0 || fk > (int) fbox.z1 || !(dy ? yb : ya) || !(dx ? xb : xa) || !(fl[c] & kInner))
                    continue;
                const int px = dx ? 2 : 0, py = dy ? 2 : 0, pz = dz ? 2 : 0;  // s = +1 for the even child
                const int f = fi0 + dx + fx * (fj0 + dy) + fxy * fk;
                const float v = 0.015625f * (27.f * w[1][1][1] + 9.f * w[1][1][px] + 9.f * w[1][py][1] +
                                             9.f * w[pz][1][1] + 3.f * w[1][py][px] + 3.f * w[pz][1][px] +
                                             3.f * w[pz][py][1] + w[pz][py][px]);
                mx_store(fine, fl[c], push, f, fv[c] + v, fx, fxy);
            }
        }
#pragma unroll
        for (int b = 0; b < 3; b++)
#pragma unroll
            for (int a = 0; a < 3; a++) {
                w[0][b][a] = w[1][b][a];
                w[1][b][a] = w[2][b][a];
            }
    }
}

// FP64 outer residual r = b - A p on level 0, stored as the FP32 right-hand
// side of the correction equation; block partials of ||r||^2
__global__ void __launch_bounds__(256, 8) k_mx_outer_residual(const double *__restrict__ p, const double *__restrict__ b,
                                    float *__restrict__ r, const uint8_t *__restrict__ flags, Level L, Box3 box,
                                    double rx, double ry, double rz, double *__restrict__ partials,
                                    const LoopState *__restrict__ pred) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    __shared__ double smem[32];
    if (pred && !pred->cond) return;
    MX_COLUMN(box);
    const int nj = (int) L.Nx, nk = (int) L.nxy();
    double acc = 0.0;
    if (col) {
        column_march<2>(p, i + nj * j, nk, (int) box.z0, (int) box.z1, flags,
            [&](int x, int, double km, double c0, double kp) {
                const double c2 = 2 * c0;
                return b[x] - (rx * (p[x - 1] - c2 + p[x + 1]) + ry * (p[x - nj] - c2 + p[x + nj]) +
                               rz * (km - c2 + kp));
            },
            [&](int x, int, double v, auto) {
                r[x] = (float) v;
                acc += v * v;
            });
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
    const int nj = (int) L.Nx, nk = (int) L.nxy();
    column_planes(i + nj * j, nk, (int) box.z0, (int) box.z1, flags,
        [&](int x, int) { return p[x] + (double) e[x]; },
        [&](int x, int, double v, auto) { p[x] = v; });
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

// the boundary program after a smoothing sweep, unless the level's stencils
// read their boundary neighbours through the program (m->fold[l])
int mx_bc_sweep(artss_mixed *m, float *f, int level, const LoopState *pred) {
    return m->fold[level] ? ARTSS_OK : mx_bc(m, f, level, pred);
}

// n_relax red-black Gauss-Seidel sweeps (ARTSS_MIXED_RBGS), in place on
// m->e[l], each colour followed by the level's boundary program
int mx_smooth_rbgs(artss_mixed *m, int l, bool from_zero, const LoopState *pred) {
    artss_ctx *ctx = m->ctx;
    const Level &L = ctx->lvl[l];
    const Box3 box = inner_box(L);
    const CoefF c = coef_f(ctx, l, m->cfg.w);
    int st;
    for (int s = 0; s < m->cfg.n_relax; s++) {
        for (int color = 0; color < 2; color++) {
            const int first = (from_zero && s == 0 && color == 0) ? 1 : 0;
            ARTSS_LAUNCH_PDL(ctx, FAM_MG_JACOBI, k_mx_rbgs, mx_grid(box), box_block(), 0, m->e[l],
                             (const float *) m->r[l], ctx->d_flags[l], L, box, c, color, first, pred);
            ARTSS_LAUNCH_CK(ctx);
            if ((st = mx_bc(m, m->e[l], l, pred))) return st;
        }
    }
    return ARTSS_OK;
}

// one weighted-Jacobi sweep m->t[l] <- m->e[l] (p: added to p instead, see
// k_mx_jacobi), in the launch shape tuned for the level (the p form repeats
// no launch, so it takes the shape the plain form was tuned to)
int mx_jacobi(artss_mixed *m, int l, const CoefF &c, const LoopState *pred, double *p) {
    artss_ctx *ctx = m->ctx;
    const Level &L = ctx->lvl[l];
    const Box3 box = inner_box(L);
    return tuned_column_launch(ctx, kTuneMxJacobi, l, box, p == nullptr, [&](dim3 g, dim3 bl) -> int {
        if (p)
            ARTSS_LAUNCH_PDL(ctx, FAM_MG_JACOBI, k_mx_jacobi<true>, g, bl, 0, m->t[l], (const float *) m->e[l],
                             (const float *) m->r[l], (const uint8_t *) m->nbm[l], (const uint16_t *) m->push[l], L,
                             box, c, pred, p);
        else
            ARTSS_LAUNCH_PDL(ctx, FAM_MG_JACOBI, k_mx_jacobi<false>, g, bl, 0, m->t[l], (const float *) m->e[l],
                             (const float *) m->r[l], (const uint8_t *) m->nbm[l], (const uint16_t *) m->push[l], L,
                             box, c, pred, (double *) nullptr);
        ARTSS_LAUNCH_CK(ctx);
        return ARTSS_OK;
    }, 256);
}

// n_relax weighted-Jacobi sweeps from e = 0 on level l, each followed by the
// boundary program; the result is left in m->e[l]
int mx_smooth_from_zero(artss_mixed *m, int l, const LoopState *pred) {
    if (m->cfg.flags & ARTSS_MIXED_RBGS) return mx_smooth_rbgs(m, l, true, pred);
    artss_ctx *ctx = m->ctx;
    const Level &L = ctx->lvl[l];
    const Box3 box = inner_box(L);
    const CoefF c = coef_f(ctx, l, m->cfg.w);
    int st;
    if ((st = tuned_column_launch(ctx, kTuneMxJacobi0, l, box, true, [&](dim3 g, dim3 bl) -> int {
             ARTSS_LAUNCH_PDL(ctx, FAM_MG_JACOBI, k_mx_jacobi0, g, bl, 0, m->e[l], (const float *) m->r[l],
                              (const uint8_t *) m->nbm[l], (const uint16_t *) m->push[l], L, box, c, pred);
             ARTSS_LAUNCH_CK(ctx);
             return ARTSS_OK;
         })))
        return st;
    if ((st = mx_bc_sweep(m, m->e[l], l, pred))) return st;
    for (int s = 1; s < m->cfg.n_relax; s++) {
        if ((st = mx_jacobi(m, l, c, pred, nullptr))) return st;
        std::swap(m->e[l], m->t[l]);
        if ((st = mx_bc_sweep(m, m->e[l], l, pred))) return st;
    }
    return ARTSS_OK;
}

// n_relax weighted-Jacobi sweeps continuing from m->e[l]; p: the last sweep
// adds its values to p (FP64) instead of storing them (the correction p += e
// of the outer loop, whose e is not read again); *corrected tells whether it did
int mx_smooth(artss_mixed *m, int l, const LoopState *pred, double *p = nullptr, bool *corrected = nullptr) {
    if (corrected) *corrected = false;
    if (m->cfg.flags & ARTSS_MIXED_RBGS) return mx_smooth_rbgs(m, l, false, pred);
    artss_ctx *ctx = m->ctx;
    const Level &L = ctx->lvl[l];
    const Box3 box = inner_box(L);
    const CoefF c = coef_f(ctx, l, m->cfg.w);
    int st;
    for (int s = 0; s < m->cfg.n_relax; s++) {
        if (p && s + 1 == m->cfg.n_relax) {
            if ((st = mx_jacobi(m, l, c, pred, p))) return st;
            if (corrected) *corrected = true;
            break;
        }
        if ((st = mx_jacobi(m, l, c, pred, nullptr))) return st;
        std::swap(m->e[l], m->t[l]);
        if ((st = mx_bc_sweep(m, m->e[l], l, pred))) return st;
    }
    return ARTSS_OK;
}

// Push masks of levels 0 .. L-2 from the inner bitmaps and the pressure
// boundary programs with every value zero (x_t = +-x_root after chain
// folding).  Every boundary cell that a smoothing or residual stencil reads
// (a face neighbour of an inner cell) must take its value from an inner face
// neighbour, which then writes it with each of its own values.  A level where
// that fails (a root that is not inner, not face-adjacent or itself written by
// the program, an inner target) or a solver with ARTSS_MIXED_RBGS /
// ARTSS_MIXED_BC_LAUNCH launches the program after each sweep instead, with a
// mask of inner bits only.
int mx_build_tables(artss_mixed *m) {
    artss_ctx *ctx = m->ctx;
    const bool allow = !(m->cfg.flags & (ARTSS_MIXED_RBGS | ARTSS_MIXED_BC_LAUNCH));
    for (int l = 0; l + 1 < m->L; l++) {
        const Level &L = ctx->lvl[l];
        const int64_t n = L.size();
        std::vector<uint16_t> pat((size_t) n, 0);  // 2 bits per direction, as a push pattern
        const std::vector<bool> &inner = ctx->h_inner[l];
        const bool have_inner = (int64_t) inner.size() == n;
        bool fold = allow && have_inner;
        const BcProgram &p = ctx->bc[l][ARTSS_FIELD_P];
        if (fold && p.present && p.n) {
            // final (root, sign) of every target, the program applied wave by wave
            std::unordered_map<int64_t, std::pair<int64_t, int>> res;
            res.reserve((size_t) p.n * 2);
            for (int64_t a = 0; a < p.n; a++) {
                int64_t r = p.h_root[(size_t) a];
                int sg = p.h_sign[(size_t) a];
                const auto it = res.find(r);
                if (it != res.end()) {
                    r = it->second.first;
                    sg *= it->second.second;
                }
                res[p.h_target[(size_t) a]] = {r, sg};
            }
            const int64_t off[6] = {-1, 1, -L.Nx, L.Nx, -L.nxy(), L.nxy()};
            for (const auto &kv : res) {
                const int64_t t = kv.first, r = kv.second.first;
                const int sg = kv.second.second;
                if (inner[(size_t) t]) { fold = false; break; }
                bool read = false;  // t is a face neighbour of an inner cell
                for (int d = 0; d < 6 && !read; d++) {
                    const int64_t x = t - off[d];
                    read = x >= 0 && x < n && inner[(size_t) x];
                }
                if (!read) continue;
                int dir = -1;  // t = r + off[dir]
                for (int d = 0; d < 6; d++)
                    if (r + off[d] == t) dir = d;
                if (dir < 0 || r < 0 || r >= n || !inner[(size_t) r] || res.count(r)) { fold = false; break; }
                pat[(size_t) r] = (uint16_t) (pat[(size_t) r] | ((sg > 0 ? 1u : 2u) << (2 * dir)));
            }
        }
        // distinct patterns -> ids 1..127
        std::vector<uint8_t> nbm((size_t) n, 0);
        std::vector<uint16_t> push(128, 0);
        std::unordered_map<uint16_t, int> ids;
        for (int64_t x = 0; x < n && fold; x++) {
            const uint16_t pv = pat[(size_t) x];
            if (!pv) continue;
            auto it = ids.find(pv);
            if (it == ids.end()) {
                if (ids.size() >= 127) { fold = false; break; }
                it = ids.emplace(pv, (int) ids.size() + 1).first;
                push[(size_t) it->second] = pv;
            }
            nbm[(size_t) x] = (uint8_t) (it->second << 1);
        }
        if (!fold) {
            std::fill(push.begin(), push.end(), (uint16_t) 0);
            std::fill(nbm.begin(), nbm.end(), (uint8_t) 0);
        }
        if (have_inner)
            for (int64_t x = 0; x < n; x++)
                if (inner[(size_t) x]) nbm[(size_t) x] = (uint8_t) (nbm[(size_t) x] | 1u);
        m->fold[l] = fold;
        if (!m->nbm[l]) ARTSS_CK(cudaMalloc(&m->nbm[l], (size_t) n));
        if (!m->push[l]) ARTSS_CK(cudaMalloc(&m->push[l], 128 * sizeof(uint16_t)));
        ARTSS_CK(cudaMemcpyAsync(m->push[l], push.data(), 128 * sizeof(uint16_t), cudaMemcpyHostToDevice, ctx->stream));
        ARTSS_CK(cudaMemcpyAsync(m->nbm[l], nbm.data(), (size_t) n, cudaMemcpyHostToDevice, ctx->stream));
        // the host vectors die with this iteration
        ARTSS_CK(cudaStreamSynchronize(ctx->stream));
    }
    m->geom_version = ctx->geom_version;
    return ARTSS_OK;
}

// FP32 V-cycle on A e = r[0] with e = 0 at start; result in m->e[0], or, with p,
// added to p by the last smoothing sweep where *corrected says so
int mx_vcycle(artss_mixed *m, const LoopState *pred, double *p = nullptr, bool *corrected = nullptr) {
    artss_ctx *ctx = m->ctx;
    const int Lc = m->L - 1;  // coarsest level
    const artss_grid_desc &g = ctx->grid;
    int st;
    for (int l = 0; l < Lc; l++) {
        if ((st = mx_smooth_from_zero(m, l, pred))) return st;
        const Level &L = ctx->lvl[l];
        const Box3 box = inner_box(L);
        if ((st = tuned_column_launch(ctx, kTuneMxResiduum, l, box, true, [&](dim3 gr, dim3 bl) -> int {
                 ARTSS_LAUNCH_PDL(ctx, FAM_MG_RESIDUUM, k_mx_residuum, gr, bl, 0, m->q[l], (const float *) m->e[l],
                                  (const float *) m->r[l], (const uint8_t *) m->nbm[l], L, box,
                                  (float) (1. / (g.dx[l] * g.dx[l])), (float) (1. / (g.dy[l] * g.dy[l])),
                                  (float) (1. / (g.dz[l] * g.dz[l])), pred);
                 ARTSS_LAUNCH_CK(ctx);
                 return ARTSS_OK;
             }, 256)))
            return st;
        if ((st = mx_bc(m, m->q[l], l, pred))) return st;
        const Level &C = ctx->lvl[l + 1];
        const Box3 cbox = inner_box(C);
        if ((st = tuned_column_launch(ctx, kTuneMxRestrict, l + 1, cbox, true, [&](dim3 gr, dim3 bl) -> int {
                 ARTSS_LAUNCH_PDL(ctx, FAM_MG_RESTRICT, k_mx_restrict, gr, bl, 0, m->r[l + 1], m->q[l],
                                  ctx->d_flags[l + 1], C, L, cbox, pred);
                 ARTSS_LAUNCH_CK(ctx);
                 return ARTSS_OK;
             })))
            return st;
    }
    // coarsest level: FP64 solve from zero
    {
        double w = m->cfg.coarse_w;
        if (w <= 0) {
            // red-black SOR with the optimal weight of the model problem on this grid
            const Level &C = ctx->lvl[Lc];
            const double n = (double) std::max({C.i2 - C.i1 + 1, C.j2 - C.j1 + 1, C.k2 - C.k1 + 1});
            w = m->cfg.coarse_smoother == ARTSS_SMOOTHER_CGS ? 2. / (1. + sin(M_PI / (n + 1.))) : 0.6666666667;
        }
        if ((st = coarse_cluster_f32(ctx, m->e[Lc], m->r[Lc], Lc, m->cfg.coarse_smoother, w, m->cfg.coarse_rel_tol,
                                     m->cfg.coarse_max_iter, pred, !(m->cfg.flags & ARTSS_MIXED_CLUSTER_COARSE),
                                     true)))
            return st;
    }
    for (int l = Lc - 1; l >= 0; l--) {
        // the prolongation reads the coarse correction's boundary cells (edges
        // and corners too): the level's program once, where the sweeps skipped it
        if (l + 1 < Lc && m->fold[l + 1] && (st = mx_bc(m, m->e[l + 1], l + 1, pred))) return st;
        const Level &C = ctx->lvl[l + 1], &F = ctx->lvl[l];
        // the fine children 2c - 1, 2c of the coarse inner box, within the fine inner box
        const Box3 fbox{std::max(F.i1, 2 * C.i1 - 1), std::min(F.i2, 2 * C.i2), std::max(F.j1, 2 * C.j1 - 1),
                        std::min(F.j2, 2 * C.j2), std::max(F.k1, 2 * C.k1 - 1), std::min(F.k2, 2 * C.k2)};
        const Box3 cbox = inner_box(C);
        if (m->cfg.flags & ARTSS_MIXED_FINE_PROLONG) {
            ARTSS_LAUNCH_PDL(ctx, FAM_MG_PROLONGATE, k_mx_prolong_add, mx_grid(fbox), box_block(), 0,
                             m->e[l], (const float *) m->e[l + 1], (const uint8_t *) ctx->d_flags[l + 1],
                             (const uint8_t *) m->nbm[l], (const uint16_t *) m->push[l], C, F, fbox, pred);
        } else {
            ARTSS_LAUNCH_PDL(ctx, FAM_MG_PROLONGATE, k_mx_prolong_add8, mx_grid(cbox), box_block(), 0,
                             m->e[l], (const float *) m->e[l + 1], (const uint8_t *) ctx->d_flags[l + 1],
                             (const uint8_t *) m->nbm[l], (const uint16_t *) m->push[l], C, F, cbox, fbox, pred);
        }
        ARTSS_LAUNCH_CK(ctx);
        if ((st = mx_bc_sweep(m, m->e[l], l, pred))) return st;
        if ((st = mx_smooth(m, l, pred, l == 0 ? p : nullptr, l == 0 ? corrected : nullptr))) return st;
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
        const int buffers = cfg->coarse_smoother == ARTSS_SMOOTHER_CGS ? 1 : 2;
        if (!cluster_fits(ctx, m->L - 1, buffers, &cap, &smem) &&
            ((cfg->flags & ARTSS_MIXED_CLUSTER_COARSE) || !block_fits(ctx, m->L - 1, buffers, &smem))) {
            set_error("the coarsest level is too large for the cluster coarse solve; use more levels");
            st = ARTSS_ERR_LIMIT;
        }
    }
    if (!st) st = cudaStreamSynchronize(ctx->stream) == cudaSuccess ? ARTSS_OK : cuda_fail(cudaGetLastError(), "sync");
    if (!st) st = mx_build_tables(m);
    if (st) { artss_mixed_destroy(m); return st; }
    *out = m;
    return ARTSS_OK;
}

int artss_mixed_destroy(artss_mixed *m) {
    if (!m) return ARTSS_OK;
    cudaStreamSynchronize(m->ctx->stream);
    for (int l = 0; l <= kMaxLevel; l++) {
        for (float *f : {m->r[l], m->q[l], m->e[l], m->t[l]})
            if (f) cudaFree(f);
        if (m->nbm[l]) cudaFree(m->nbm[l]);
        if (m->push[l]) cudaFree(m->push[l]);
    }
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
    if (m->geom_version != ctx->geom_version) {
        // cell lists or boundary programs changed since the tables were built
        if (ctx->capturing) { set_error("the mixed solver's boundary tables are stale; solve once before capturing"); return ARTSS_ERR_ARG; }
        if ((st = mx_build_tables(m))) return st;
    }
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
            bool corrected = false;
            if ((st = mx_vcycle(m, pred, p, &corrected))) return st;
            if (!corrected) {
                ARTSS_LAUNCH_PDL(ctx, FAM_FIELD_OP, k_mx_correct, grid, box_block(), 0,
                                                    p, m->e[0], ctx->d_flags[0], L, box, pred);
                ARTSS_LAUNCH_CK(ctx);
            }
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
