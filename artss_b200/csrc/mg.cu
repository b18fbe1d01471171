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
#include "tc.cuh"

#include <algorithm>
#include <cooperative_groups.h>

struct artss_mg {
    artss_ctx *ctx = nullptr;
    artss_mg_cfg cfg{};
    int L = 0;
    bool fused_coarse = true;
    bool cluster_coarse = true;
    bool pipelined_coarse = true;
    double *r0[artss::kMaxLevel + 1]{};   // residuum0[level]   (levels 0..L-1)
    double *r1[artss::kMaxLevel + 1]{};   // residuum1[level]   (levels 0..L)
    double *e0[artss::kMaxLevel + 1]{};   // error0[level]      (levels 0..L-1)
    double *e1[artss::kMaxLevel + 1]{};   // error1[level]      (levels 0..L)
    double *tmp[artss::kMaxLevel + 1]{};  // temporal solution  (levels 0..L)
    // CUDA graphs of the fixed launch sequence of a later-step pressure call
    // (set_rhs + n_cycle V-cycles), one per (p, rhs) pair
    struct Graph {
        const double *p, *rhs;
        cudaGraphExec_t exec;
        int64_t launches, fam[artss::FAM_COUNT];
    };
    std::vector<Graph> graphs;
    bool use_graphs = true;
    // the restriction of level l+1's inner cells reads no target of level l's
    // boundary program: the program on residuum0[l] has no reader
    bool r0_bc_dead[artss::kMaxLevel + 1]{};
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

// 32-bit cell indices: artss_ctx_create rejects levels of 2^31 cells or more
#define MG_COLUMN(box)                                                                    \
    const int i = (int) (box).x0 + (int) (blockIdx.x * blockDim.x + threadIdx.x);        \
    const int j = (int) (box).y0 + (int) (blockIdx.y * blockDim.y + threadIdx.y);        \
    const bool col = (i <= (int) (box).x1) && (j <= (int) (box).y1)

struct MgCoef {
    double ax, ay, az;   // 1/(dx*dx) ... of the level (VCycleMG.cpp:595-601)
    double beta;         // 1/(2 (ax+ay+az))
    double dsign, w, omw;
};

// JacobiDiffuse::JacobiStep, multigrid variant (JacobiDiffuse.cpp:274-305)
__global__ void __launch_bounds__(256, 8) k_mg_jacobi(double *__restrict__ out, const double *__restrict__ in, const double *__restrict__ b,
                            const uint8_t *__restrict__ flags, Level L, Box3 box, MgCoef c) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    MG_COLUMN(box);
    if (!col) return;
    const int nj = (int) L.Nx, nk = (int) L.nxy();
    column_march<2>(in, i + nj * j, nk, (int) box.z0, (int) box.z1, flags,
        [&](int q, int, double km, double c0, double kp) {
            const double out_h = c.beta * (c.dsign * b[q] + c.ax * (in[q + 1] + in[q - 1]) +
                                           c.ay * (in[q + nj] + in[q - nj]) + c.az * (kp + km));
            return c.omw * c0 + c.w * out_h;
        },
        [&](int q, int, double v, auto) { out[q] = v; });
}

// colored Gauss-Seidel stencil with the multigrid coefficients
// (ColoredGaussSeidelDiffuse.cpp:316-341 called from VCycleMG.cpp:608-616)
__global__ void k_mg_cgs_color(double *__restrict__ out, const double *__restrict__ b,
                               const uint8_t *__restrict__ flags, Level L, Box3 box, int color, MgCoef c) {
    MG_COLUMN(box);
    if (!col) return;
    const int nj = (int) L.Nx, nk = (int) L.nxy();
    for (int k = (int) box.z0 + (int) blockIdx.z; k <= (int) box.z1; k += (int) gridDim.z) {
        if (((i + j + k) & 1) != color) continue;
        const int q = i + (int) L.Nx * j + nk * k;
        if (!(flags[q] & kInner)) continue;
        const double out_h = c.beta * (c.dsign * b[q] + c.ax * (out[q + 1] + out[q - 1]) +
                                       c.ay * (out[q + nj] + out[q - nj]) + c.az * (out[q + nk] + out[q - nk]));
        out[q] = c.omw * out[q] + c.w * out_h;
    }
}

// VCycleMG::Residuum (VCycleMG.cpp:346-354)
__global__ void __launch_bounds__(256, 8) k_mg_residuum(double *__restrict__ out, const double *__restrict__ in, const double *__restrict__ b,
                              const uint8_t *__restrict__ flags, Level L, Box3 box, double rx, double ry, double rz) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    MG_COLUMN(box);
    if (!col) return;
    const int nj = (int) L.Nx, nk = (int) L.nxy();
    column_march<2>(in, i + nj * j, nk, (int) box.z0, (int) box.z1, flags,
        [&](int q, int, double km, double c0, double kp) {
            const double weighted = (rx * (in[q - 1] - 2 * c0 + in[q + 1]) +
                                     ry * (in[q - nj] - 2 * c0 + in[q + nj]) +
                                     rz * (km - 2 * c0 + kp));
            return b[q] - weighted;
        },
        [&](int q, int, double v, auto) { out[q] = v; });
}

// block partials of sum (b - A x)^2 over the level's inner cells
// (VCycleMG.cpp:186-194, :668-679, :777-788)
__global__ void __launch_bounds__(256, 8) k_mg_resnorm(const double *__restrict__ x, const double *__restrict__ b,
                             const uint8_t *__restrict__ flags, Level L, Box3 box, double rx, double ry, double rz,
                             double *__restrict__ partials, double *__restrict__ partials_b) {
    __shared__ double smem[32];
    MG_COLUMN(box);
    const int nj = (int) L.Nx, nk = (int) L.nxy();
    double acc = 0.0, accb = 0.0;
    if (col) {
        struct RB { double r, b; };
        column_march<2>(x, i + nj * j, nk, (int) box.z0, (int) box.z1, flags,
            [&](int q, int, double km, double c0, double kp) {
                const double r = b[q] - (rx * (x[q - 1] - 2 * c0 + x[q + 1]) +
                                         ry * (x[q - nj] - 2 * c0 + x[q + nj]) +
                                         rz * (km - 2 * c0 + kp));
                return RB{r, b[q]};
            },
            [&](int, int, RB v, auto) {
                acc += v.r * v.r;
                accb += v.b * v.b;
            });
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
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    MG_COLUMN(box);
    if (!col) return;
    const int fx = (int) F.Nx, fxy = (int) F.nxy();
    column_planes(i + (int) C.Nx * j, (int) C.nxy(), (int) box.z0, (int) box.z1, flags,
        [&](int, int k) {
            const int a = 2 * i - 1, bx = 2 * i, c = 2 * j - 1, d = 2 * j, e = 2 * k - 1, f = 2 * k;
            return 0.125 * (in[a + fx * c + fxy * e] + in[bx + fx * c + fxy * e] + in[a + fx * d + fxy * e] +
                            in[bx + fx * d + fxy * e] + in[a + fx * c + fxy * f] + in[bx + fx * c + fxy * f] +
                            in[a + fx * d + fxy * f] + in[bx + fx * d + fxy * f]);
        },
        [&](int q, int, double v, auto) { out[q] = v; });
}

// VCycleMG::Prolongate (VCycleMG.cpp:464-546): 8 fine cells per coarse inner cell
__global__ void k_mg_prolongate(double *__restrict__ out, const double *__restrict__ in,
                                const uint8_t *__restrict__ flags, Level C, Level F, Box3 box) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    MG_COLUMN(box);
    if (!col) return;
    const int ni = 1, nj = (int) C.Nx, nk = (int) C.nxy();
    const int fx = (int) F.Nx, fxy = (int) F.nxy();
    for (int k = (int) box.z0 + (int) blockIdx.z; k <= (int) box.z1; k += (int) gridDim.z) {
        const int q = i + (int) C.Nx * j + (int) C.nxy() * k;
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
    const MgCoef c = mg_coef(mg, level);
    return tuned_column_launch(ctx, kTuneMgJacobi, level, box, out != in && out != b, [&](dim3 g, dim3 bl) -> int {
        ARTSS_LAUNCH_PDL(ctx, FAM_MG_JACOBI, k_mg_jacobi, g, bl, 0, out, in, b, ctx->d_flags[level], L, box, c);
        ARTSS_LAUNCH_CK(ctx);
        return ARTSS_OK;
    }, 256);
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
    return finalize_residual(ctx, slot, nb);
}

// VCycleMG::Smooth + call_smooth_{jacobi,colored_gauss_seidel} (VCycleMG.cpp:299-305, :583-723)
int mg_smooth(artss_mg *mg, double *out, double *tmp, const double *b, int level, bool out_satisfies_bc = false) {
    int st;
    // VCycleMG::Smooth and call_smooth_* each apply the boundary program first;
    // the program is idempotent (ghost values are functions of inner values it
    // does not write), so one application gives the same array.  With every
    // value +0.0 (x_t = +-x_r + 0) an array of zeros, and the sum of two arrays
    // that satisfy the program, satisfy it bit for bit (sign flips commute with
    // round-to-nearest addition; the + 0 turns -0 into +0 on both sides): the
    // caller says so and the application is left out.
    if (!(out_satisfies_bc && mg->ctx->bc[level][ARTSS_FIELD_P].zero_values) && (st = mg_bc(mg, out, level)))
        return st;
    if (mg->cfg.smoother == ARTSS_SMOOTHER_CGS) {
        for (int r = 0; r < mg->cfg.n_relax; r++) {
            if ((st = mg_cgs_step(mg, out, b, level))) return st;
            if ((st = mg_bc(mg, out, level))) return st;
        }
        return ARTSS_OK;
    }
    if ((st = artss_copy(mg->ctx, tmp, out, level))) return st;
    double *A = out, *B = tmp;   // Field data pointers as swapped by Field::swap
    // VCycleMG::call_smooth_jacobi (VCycleMG.cpp:710-721) leaves `out` with
    // iterate n_relax - 1 when n_relax is even: the last relaxation writes only
    // tmp, which the next smoothing or coarse solve overwrites before reading
    // it.  That relaxation and its boundary program are left out.
    const int n_relax = mg->cfg.n_relax - (mg->cfg.n_relax > 0 && mg->cfg.n_relax % 2 == 0 ? 1 : 0);
    for (int r = 0; r < n_relax; r++) {
        if ((st = mg_jacobi_step(mg, A, B, b, level))) return st;
        if ((st = mg_bc(mg, A, level))) return st;
        std::swap(A, B);
    }
    return ARTSS_OK;
}

// VCycleMG::Solve + call_solve_{jacobi,colored_gauss_seidel} (VCycleMG.cpp:562-581, :620-798)
// ---------------------------------------------------------------- single-block coarse solve
//
// VCycleMG::Solve on a small level runs up to smoother_max_iter sweeps, each
// followed by the boundary program and a residual norm that decides whether
// to continue (VCycleMG.cpp:725-798).  On a level of a few thousand cells
// every one of these passes is launch- and latency-bound, so one 1024-thread
// block runs the whole loop: sweep, __syncthreads, boundary waves, residual
// reduced inside the block, decision, next sweep.  The arithmetic per cell is
// the multigrid Jacobi / colored Gauss-Seidel stencil of the multi-block path.

constexpr int kCoarseThreads = 1024;
constexpr int64_t kCoarseMaxCells = 1 << 17;  // level array size handled by one block
constexpr int kCoarseMaxWaves = 8;

struct BcView {
    const int64_t *target, *root;
    const uint8_t *depth, *neg;
    const double *value;
    int64_t n;
    int waves;
    int64_t begin[kCoarseMaxWaves + 1];
};

// The level's boundary program executed by one block, wave after wave.
__device__ __forceinline__ void coarse_bc(double *__restrict__ f, const BcView &bc, int tid, int nthr) {
    for (int w = 0; w < bc.waves; w++) {
        for (int64_t q = bc.begin[w] + tid; q < bc.begin[w + 1]; q += nthr) {
            double x = f[bc.root[q]];
            const int d = bc.depth[q];
            const uint8_t m = bc.neg[q];
#pragma unroll
            for (int s = 0; s < kBcMaxDepth; s++)
                if (s < d) x = ((m >> s) & 1 ? -x : x) + bc.value[s * bc.n + q];
            f[bc.target[q]] = x;
        }
        __syncthreads();
    }
}

// VCycleMG::Solve loop of one level inside one block.  SMEM: the level's
// arrays (out, and tmp for Jacobi) are copied into shared memory, iterated
// there, and written back; otherwise they are iterated in global memory.
template <bool CGS, bool SMEM>
__global__ void __launch_bounds__(kCoarseThreads)
k_mg_coarse_solve(double *__restrict__ out, double *__restrict__ tmp, const double *__restrict__ b,
                  const uint8_t *__restrict__ flags, Level L, Box3 box, MgCoef c, double rx, double ry, double rz,
                  BcView bc, double tol, long long max_it, LoopState *__restrict__ st) {
    extern __shared__ double sm[];
    __shared__ double red[32];
    __shared__ double s_res;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int nj = (int) L.Nx, nk = (int) (L.Nx * L.Ny), ntot = (int) (L.Nx * L.Ny * L.Nz);
    const int nx = (int) box.nx(), nxy = (int) (box.nx() * box.ny()), ncell = (int) (nxy * box.nz());
    const int x0 = (int) box.x0, y0 = (int) box.y0, z0 = (int) box.z0;
    double *A = out, *B = tmp;
    if (SMEM) {
        A = sm;
        B = sm + ntot;
        for (int q = tid; q < ntot; q += nthr) A[q] = out[q];
        __syncthreads();
    }
    coarse_bc(A, bc, tid, nthr);
    if (!CGS) {
        for (int q = tid; q < ntot; q += nthr) B[q] = A[q];
        __syncthreads();
    }
    double res = 10000.;
    long long it = 0;
    while (res > tol && it < max_it) {
        if (CGS) {
            for (int color = 0; color < 2; color++) {
                for (int lin = tid; lin < ncell; lin += nthr) {
                    const int k = z0 + lin / nxy, r = lin % nxy, j = y0 + r / nx, i = x0 + r % nx;
                    if (((i + j + k) & 1) != color) continue;
                    const int q = i + nj * j + nk * k;
                    if (!(__ldg(flags + q) & kInner)) continue;
                    const double out_h = c.beta * (c.dsign * __ldg(b + q) + c.ax * (A[q + 1] + A[q - 1]) +
                                                   c.ay * (A[q + nj] + A[q - nj]) + c.az * (A[q + nk] + A[q - nk]));
                    A[q] = c.omw * A[q] + c.w * out_h;
                }
                __syncthreads();
            }
        } else {
            for (int lin = tid; lin < ncell; lin += nthr) {
                const int k = z0 + lin / nxy, r = lin % nxy, j = y0 + r / nx, i = x0 + r % nx;
                const int q = i + nj * j + nk * k;
                if (!(__ldg(flags + q) & kInner)) continue;
                const double out_h = c.beta * (c.dsign * __ldg(b + q) + c.ax * (B[q + 1] + B[q - 1]) +
                                               c.ay * (B[q + nj] + B[q - nj]) + c.az * (B[q + nk] + B[q - nk]));
                A[q] = c.omw * B[q] + c.w * out_h;
            }
            __syncthreads();
        }
        coarse_bc(A, bc, tid, nthr);
        double acc = 0.0;
        for (int lin = tid; lin < ncell; lin += nthr) {
            const int k = z0 + lin / nxy, r = lin % nxy, j = y0 + r / nx, i = x0 + r % nx;
            const int q = i + nj * j + nk * k;
            if (!(__ldg(flags + q) & kInner)) continue;
            const double rr = __ldg(b + q) - (rx * (A[q - 1] - 2 * A[q] + A[q + 1]) +
                                             ry * (A[q - nj] - 2 * A[q] + A[q + nj]) +
                                             rz * (A[q - nk] - 2 * A[q] + A[q + nk]));
            acc += rr * rr;
        }
        acc = artss_block_sum(acc, red);
        if (tid == 0) s_res = sqrt(acc);
        __syncthreads();
        res = s_res;
        __syncthreads();
        if (!CGS) {
            double *t = A;
            A = B;
            B = t;
        }
        it++;
    }
    if (SMEM) {
        // sm[0..ntot) is out's storage and sm[ntot..) tmp's, whatever the swaps did
        for (int q = tid; q < ntot; q += nthr) out[q] = sm[q];
        if (!CGS)
            for (int q = tid; q < ntot; q += nthr) tmp[q] = sm[ntot + q];
    }
    if (tid == 0 && st) {
        st->it = it;
        st->residual = res;
        st->cond = 0;
    }
}

constexpr int64_t kCoarseSmemBytes = 200 * 1024;

// ---------------------------------------------------------------- cluster coarse solve
//
// The same VCycleMG::Solve loop spread over a thread-block cluster: rank r
// keeps the z-planes [kb[r], kb[r+1]) of the level's arrays in its shared
// memory and reaches the other ranks' planes through distributed shared
// memory (a per-plane pointer table).  Each rank sweeps its own inner cells,
// whose indices and right-hand side stay in registers for the whole loop; the
// boundary assignments are dealt out over all ranks; the residual is reduced
// per block, every rank receives all partial sums and adds them in rank
// order, so all ranks take the same loop decision.  Cluster barriers separate
// sweep, boundary waves and reduction.  Per cell the arithmetic is that of
// k_mg_coarse_solve.

constexpr int kClusterSize = 8;
constexpr int kClusterThreads = 512;
constexpr int kClusterCells = 8;        // inner cells per thread
constexpr int kClusterMaxPlanes = 256;  // z-planes of the level

// Boundary waves over the whole cluster; T maps a z-plane to its storage.
__device__ __forceinline__ void cluster_bc(double *const *T, const int64_t *begin, int waves, const int64_t *root,
                                           const int64_t *target, const uint8_t *depth, const uint8_t *neg,
                                           const double *value, int64_t n, int gtid, int nthr, int nk,
                                           cooperative_groups::cluster_group &cl) {
    for (int w = 0; w < waves; w++) {
        for (int64_t q = begin[w] + gtid; q < begin[w + 1]; q += nthr) {
            const int r = (int) __ldg(root + q), t = (int) __ldg(target + q);
            const int kr = r / nk, kt = t / nk;
            double x = T[kr][r - kr * nk];
            const int d = __ldg(depth + q);
            const uint8_t m = __ldg(neg + q);
#pragma unroll
            for (int s = 0; s < kBcMaxDepth; s++)
                if (s < d) x = ((m >> s) & 1 ? -x : x) + (value ? __ldg(value + s * n + q) : 0.0);
            T[kt][t - kt * nk] = x;
        }
        cl.sync();
    }
}

// ||b - A x||_2 over the cluster's inner cells, identical in every rank
template <int NC>
__device__ __forceinline__ double cluster_resnorm(double *const *T, const int (&ck)[NC], const int (&co)[NC],
                                                  const double (&cb)[NC], unsigned mask, int nj, double rx, double ry,
                                                  double rz, double *red, double *s_acc, double *parts, int rank,
                                                  int cs, cooperative_groups::cluster_group &cl) {
    double acc = 0.0;
#pragma unroll
    for (int m = 0; m < NC; m++) {
        if (!(mask >> m & 1)) continue;
        const double *A = T[ck[m]], *Am = T[ck[m] - 1], *Ap = T[ck[m] + 1];
        const int o = co[m];
        const double rr = cb[m] - (rx * (A[o - 1] - 2 * A[o] + A[o + 1]) + ry * (A[o - nj] - 2 * A[o] + A[o + nj]) +
                                   rz * (Am[o] - 2 * A[o] + Ap[o]));
        acc += rr * rr;
    }
    acc = artss_block_sum(acc, red);
    if (threadIdx.x == 0) *s_acc = acc;
    __syncthreads();
    // thread r sends this rank's sum to rank r
    if ((int) threadIdx.x < cs) cl.map_shared_rank(parts, (int) threadIdx.x)[rank] = *s_acc;
    cl.sync();
    double s = 0.0;
    for (int r = 0; r < cs; r++) s += parts[r];
    return sqrt(s);
}

// TS: storage type of out / tmp / b (the arithmetic is FP64 either way).
// rel: tol is relative to the residual of the initial iterate.
// pred: the launch does nothing when pred->cond == 0 (predicated loops).
template <bool CGS, typename TS>
__global__ void __launch_bounds__(kClusterThreads, 1)
k_mg_coarse_cluster(TS *__restrict__ out, TS *__restrict__ tmp, const TS *__restrict__ b,
                    const uint8_t *__restrict__ flags, Level L, Box3 box, MgCoef c, double rx, double ry, double rz,
                    BcView bc, double tol, int rel, long long max_it, int plane_cap, LoopState *__restrict__ st,
                    const LoopState *__restrict__ pred) {
    namespace cg = cooperative_groups;
    if (pred && !pred->cond) return;  // every rank reads the same flag
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ double sm[];
    __shared__ double *tab0[kClusterMaxPlanes];
    __shared__ double *tab1[kClusterMaxPlanes];
    __shared__ double red[32];
    __shared__ double parts[kClusterSize];
    __shared__ double s_acc;
    __shared__ int64_t s_begin[kCoarseMaxWaves + 1];
    const int tid = threadIdx.x;
    const int rank = (int) cl.block_rank();
    const int cs = (int) cl.num_blocks();
    const int nj = (int) L.Nx, nk = (int) (L.Nx * L.Ny), nz = (int) L.Nz;
    const int kb0 = (int) ((int64_t) rank * nz / cs), kb1 = (int) ((int64_t) (rank + 1) * nz / cs);
    double *X0 = sm, *X1 = sm + (int64_t) plane_cap * nk;
#pragma unroll
    for (int w = 0; w <= kCoarseMaxWaves; w++)
        if (tid == w) s_begin[w] = bc.begin[w];

    // own planes of out (and, for Jacobi, nothing yet of tmp)
    for (int q = tid; q < (kb1 - kb0) * nk; q += kClusterThreads) X0[q] = (double) out[(int64_t) kb0 * nk + q];
    // plane k lives on rank r with kb(r) <= k < kb(r+1)
    for (int k = tid; k < nz; k += kClusterThreads) {
        for (int r = 0; r < cs; r++) {
            const int a = (int) ((int64_t) r * nz / cs), e = (int) ((int64_t) (r + 1) * nz / cs);
            if (k >= a && k < e) {
                tab0[k] = cl.map_shared_rank(X0, r) + (int64_t) (k - a) * nk;
                tab1[k] = cl.map_shared_rank(X1, r) + (int64_t) (k - a) * nk;
            }
        }
    }
    // this thread's inner cells: plane, in-plane offset and b, in registers
    int ck[kClusterCells], co[kClusterCells];
    double cb[kClusterCells];
    unsigned m0 = 0, m1 = 0;  // cells of colour 0 / 1 (Jacobi: all in m0)
    {
        const int z0 = max((int) box.z0, kb0), z1 = min((int) box.z1, kb1 - 1);
        const int nx = (int) box.nx(), nxy = (int) (box.nx() * box.ny());
        const int ncell = z1 >= z0 ? (z1 - z0 + 1) * nxy : 0;
#pragma unroll
        for (int m = 0; m < kClusterCells; m++) {
            const int lin = tid + m * kClusterThreads;
            ck[m] = 0;
            co[m] = 0;
            cb[m] = 0.0;
            if (lin < ncell) {
                const int k = z0 + lin / nxy, r = lin % nxy, j = (int) box.y0 + r / nx, i = (int) box.x0 + r % nx;
                const int o = i + nj * j;
                const int64_t q = (int64_t) k * nk + o;
                if (__ldg(flags + q) & kInner) {
                    ck[m] = k;
                    co[m] = o;
                    cb[m] = (double) b[q];
                    if (!CGS || ((i + j + k) & 1) == 0) m0 |= 1u << m;
                    else m1 |= 1u << m;
                }
            }
        }
    }
    cl.sync();

    double **TA = tab0, **TB = tab1;
    const int nthr = cs * kClusterThreads, gtid = rank * kClusterThreads + tid;
    cluster_bc(TA, s_begin, bc.waves, bc.root, bc.target, bc.depth, bc.neg, bc.value, bc.n, gtid, nthr, nk, cl);
    if (!CGS) {
        for (int q = tid; q < (kb1 - kb0) * nk; q += kClusterThreads) X1[q] = X0[q];
        cl.sync();
    }
    double res = 10000.;
    long long it = 0;
    if (rel) tol *= cluster_resnorm(TA, ck, co, cb, m0 | m1, nj, rx, ry, rz, red, &s_acc, parts, rank, cs, cl);
    while (res > tol && it < max_it) {
        if (CGS) {
#pragma unroll
            for (int color = 0; color < 2; color++) {
                const unsigned mask = color ? m1 : m0;
#pragma unroll
                for (int m = 0; m < kClusterCells; m++) {
                    if (!(mask >> m & 1)) continue;
                    double *A = TA[ck[m]];
                    const double *Am = TA[ck[m] - 1], *Ap = TA[ck[m] + 1];
                    const int o = co[m];
                    const double out_h = c.beta * (c.dsign * cb[m] + c.ax * (A[o + 1] + A[o - 1]) +
                                                   c.ay * (A[o + nj] + A[o - nj]) + c.az * (Ap[o] + Am[o]));
                    A[o] = c.omw * A[o] + c.w * out_h;
                }
                cl.sync();
            }
        } else {
#pragma unroll
            for (int m = 0; m < kClusterCells; m++) {
                if (!(m0 >> m & 1)) continue;
                const double *B = TB[ck[m]], *Bm = TB[ck[m] - 1], *Bp = TB[ck[m] + 1];
                const int o = co[m];
                const double out_h = c.beta * (c.dsign * cb[m] + c.ax * (B[o + 1] + B[o - 1]) +
                                               c.ay * (B[o + nj] + B[o - nj]) + c.az * (Bp[o] + Bm[o]));
                TA[ck[m]][o] = c.omw * B[o] + c.w * out_h;
            }
            cl.sync();
        }
        cluster_bc(TA, s_begin, bc.waves, bc.root, bc.target, bc.depth, bc.neg, bc.value, bc.n, gtid, nthr, nk, cl);
        res = cluster_resnorm(TA, ck, co, cb, m0 | m1, nj, rx, ry, rz, red, &s_acc, parts, rank, cs, cl);
        if (!CGS) {
            double **t = TA;
            TA = TB;
            TB = t;
        }
        it++;
    }
    // X0 is out's storage and X1 tmp's, whatever the swaps did
    for (int q = tid; q < (kb1 - kb0) * nk; q += kClusterThreads) {
        out[(int64_t) kb0 * nk + q] = (TS) X0[q];
        if (!CGS && tmp) tmp[(int64_t) kb0 * nk + q] = (TS) X1[q];
    }
    if (rank == 0 && tid == 0 && st) {
        st->it = it;
        st->residual = res;
        st->cond = 0;
    }
    cl.sync();
}

// ---------------------------------------------------------------- one-block coarse solve
//
// The loop of k_mg_coarse_cluster on ONE block for a level that fits its
// shared memory (a few thousand inner cells, the coarsest grid of a deep
// V-cycle): the whole level array (and tmp's for Jacobi) lives in shared
// memory, each thread keeps its cells' offsets and right-hand side and its
// boundary assignments (target, root, chain) in registers, and the barriers
// are block barriers.  Cell slots 0 .. kBlkCells/2 - 1 of a thread hold cells
// of colour 0, the others colour 1, numbered so that the 32 lanes of a warp
// hold cells of one colour: a colour pass runs without divergence.  The
// residual's warp sums are added by every warp in the same butterfly order,
// and the loop test compares the squared sum with tol^2 outside a guard band
// (the square root only inside it).  Same iterates as the cluster kernel; only
// the order of the residual sums differs.  The set-up that reads no result of
// the previous kernel (cell slots, boundary slots) runs before the
// programmatic-launch wait.

constexpr int kBlkThreads = 1024;
constexpr int kBlkCells = 4;     // cell slots per thread, half per colour: at most 2048 cells per colour
constexpr int kBlkTargets = 4;   // boundary assignments per thread, all waves together

// box cells of colour col ((i + j + k) % 2) in slot order: slot s = (k, j, t)
// row-major over ceil(nx / 2) pairs per row, x = x0 + 2 t + the row's offset
__host__ __device__ inline int64_t blk_slots(const Box3 &box) {
    return ((box.nx() + 1) / 2) * box.ny() * box.nz();
}

template <bool CGS, typename TS>
__global__ void __launch_bounds__(kBlkThreads, 1)
k_mg_coarse_block(TS *__restrict__ out, TS *__restrict__ tmp, const TS *__restrict__ b,
                  const uint8_t *__restrict__ flags, Level L, Box3 box, MgCoef c, double rx, double ry, double rz,
                  const __grid_constant__ BcView bc, double tol, int rel, long long max_it, LoopState *__restrict__ st,
                  const LoopState *__restrict__ pred, int zero_start) {
    extern __shared__ double sm[];
    __shared__ double red[kBlkThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31;
    const int nj = (int) L.Nx, nk = (int) (L.Nx * L.Ny), ntot = (int) (L.Nx * L.Ny * L.Nz);
    constexpr int H = kBlkCells / 2;
    // this thread's cells (static: the level's flags): offsets and colour masks
    int co[kBlkCells];
    unsigned m0 = 0, m1 = 0;
    {
        const int np = (int) ((box.nx() + 1) / 2), nrow = np * (int) box.ny(), nslot = nrow * (int) box.nz();
#pragma unroll
        for (int m = 0; m < kBlkCells; m++) {
            const int col = m < H ? 0 : 1;
            const int s = tid + (m % H) * kBlkThreads;
            co[m] = 0;
            if (s < nslot) {
                const int k = (int) box.z0 + s / nrow, r = s % nrow, j = (int) box.y0 + r / np;
                const int x0 = (int) box.x0;
                const int i = x0 + 2 * (r % np) + ((x0 + j + k + col) & 1);
                if (i <= (int) box.x1) {
                    const int q = i + nj * j + nk * k;
                    if (__ldg(flags + q) & kInner) {
                        co[m] = q;
                        if (!CGS || col == 0) m0 |= 1u << m;
                        else m1 |= 1u << m;
                    }
                }
            }
        }
    }
    // this thread's boundary assignments, in wave order: slot u is its u-th
    // assignment begin[w] + tid + v * threads over the waves w (a slot index known
    // at compile time, so the slots stay in registers); bdn = depth | neg << 8 |
    // (wave + 1) << 16, 0 for an empty slot
    int bt[kBlkTargets], br[kBlkTargets], bq[kBlkTargets];
    uint32_t bdn[kBlkTargets];
    {
        // slot -> assignment first (no loads), then all slots' loads at once
        int wv[kBlkTargets];
#pragma unroll
        for (int u = 0; u < kBlkTargets; u++) {
            bq[u] = -1;
            wv[u] = 0;
            int before = 0;
            for (int w = 0; w < bc.waves; w++) {
                const int64_t n_w = bc.begin[w + 1] - bc.begin[w] - tid;
                const int cnt = n_w > 0 ? (int) ((n_w + kBlkThreads - 1) / kBlkThreads) : 0;
                if (bq[u] < 0 && u < before + cnt) {
                    bq[u] = (int) (bc.begin[w] + tid + (int64_t) (u - before) * kBlkThreads);
                    wv[u] = w + 1;
                }
                before += cnt;
            }
        }
#pragma unroll
        for (int u = 0; u < kBlkTargets; u++) {
            bt[u] = br[u] = 0;
            bdn[u] = 0;
            if (bq[u] >= 0) {
                bt[u] = (int) __ldg(bc.target + bq[u]);
                br[u] = (int) __ldg(bc.root + bq[u]);
                bdn[u] = (uint32_t) __ldg(bc.depth + bq[u]) | (uint32_t) __ldg(bc.neg + bq[u]) << 8 |
                         (uint32_t) wv[u] << 16;
            }
        }
    }
    pdl_wait();  // launched by launch_pdl: the predecessor's writes (b, out, pred) are visible after this
    pdl_trigger();
    if (pred && !pred->cond) return;
    double cb[kBlkCells];
#pragma unroll
    for (int m = 0; m < kBlkCells; m++) cb[m] = ((m0 | m1) >> m & 1) ? (double) b[co[m]] : 0.0;
    // zero_start: the iterate starts at zero (out is not read)
    for (int q = tid; q < ntot; q += kBlkThreads) sm[q] = zero_start ? 0.0 : (double) out[q];
#define BLK_APPLY_BC(base)                                                                                     \
    for (int w = 0; w < bc.waves; w++) {                                                                       \
        _Pragma("unroll") for (int u = 0; u < kBlkTargets; u++) {                                              \
            if ((int) (bdn[u] >> 16) != w + 1) continue;                                                       \
            double x = sm[(base) + br[u]];                                                                     \
            const int d = (int) (bdn[u] & 0xffu);                                                              \
            const uint32_t mneg = (bdn[u] >> 8) & 0xffu;                                                       \
            _Pragma("unroll") for (int e = 0; e < kBcMaxDepth; e++) if (e < d) x =                             \
                ((mneg >> e) & 1 ? -x : x) + (bc.value ? __ldg(bc.value + e * bc.n + bq[u]) : 0.0);            \
            sm[(base) + bt[u]] = x;                                                                            \
        }                                                                                                      \
        __syncthreads();                                                                                       \
    }
    // sum of ||b - A x||^2 over the inner cells (x at sm[base ..]), the same in
    // every thread
    auto ressum = [&](int base) {
        double acc = 0.0;
#pragma unroll
        for (int m = 0; m < kBlkCells; m++) {
            if (!((m0 | m1) >> m & 1)) continue;
            const int o = base + co[m];
            const double c0 = sm[o];
            const double rr = cb[m] - (rx * (sm[o - 1] - 2 * c0 + sm[o + 1]) + ry * (sm[o - nj] - 2 * c0 + sm[o + nj]) +
                                       rz * (sm[o - nk] - 2 * c0 + sm[o + nk]));
            acc += rr * rr;
        }
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (lane == 0) red[tid >> 5] = acc;
        __syncthreads();
        double v = red[lane];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        return v;
    };
    __syncthreads();
    BLK_APPLY_BC(0);
    if (!CGS) {
        for (int q = tid; q < ntot; q += kBlkThreads) sm[ntot + q] = sm[q];
        __syncthreads();
    }
    int A = 0, B = ntot;  // offsets of the two arrays (Field::swap of the reference)
    double res = 10000.;
    long long it = 0;
    if (rel) {
        tol *= sqrt(ressum(A));
        __syncthreads();  // red is rewritten by the next reduction
    }
    // res > tol decided on the squared sum s where that is exact: outside +-16
    // units of roundoff around tol^2 sqrt(s) lies on the same side of tol
    const double tol2 = tol * tol;
    const bool fast = tol2 > 1e-280 && tol2 < 1e280;
    bool above = res > tol;
    double s_last = -1.0;
    while (above && it < max_it) {
        if (CGS) {
#pragma unroll
            for (int color = 0; color < 2; color++) {
#pragma unroll
                for (int m = color * H; m < (color + 1) * H; m++) {
                    if (!((color ? m1 : m0) >> m & 1)) continue;
                    const int o = co[m];
                    const double out_h = c.beta * (c.dsign * cb[m] + c.ax * (sm[o + 1] + sm[o - 1]) +
                                                   c.ay * (sm[o + nj] + sm[o - nj]) + c.az * (sm[o + nk] + sm[o - nk]));
                    sm[o] = c.omw * sm[o] + c.w * out_h;
                }
                __syncthreads();
            }
        } else {
#pragma unroll
            for (int m = 0; m < kBlkCells; m++) {
                if (!(m0 >> m & 1)) continue;
                const int o = co[m];
                const double out_h = c.beta * (c.dsign * cb[m] + c.ax * (sm[B + o + 1] + sm[B + o - 1]) +
                                               c.ay * (sm[B + o + nj] + sm[B + o - nj]) +
                                               c.az * (sm[B + o + nk] + sm[B + o - nk]));
                sm[A + o] = c.omw * sm[B + o] + c.w * out_h;
            }
            __syncthreads();
        }
        BLK_APPLY_BC(A);
        const double s = ressum(A);
        s_last = s;
        if (fast && s > tol2 * (1.0 + 0x1p-49)) above = true;
        else if (fast && s < tol2 * (1.0 - 0x1p-49)) above = false;
        else above = sqrt(s) > tol;
        if (!CGS) {
            const int t = A;
            A = B;
            B = t;
        }
        it++;
    }
#undef BLK_APPLY_BC
    if (s_last >= 0) res = sqrt(s_last);
    __syncthreads();
    // sm[0 ..) is out's storage and sm[ntot ..) tmp's, whatever the swaps did
    for (int q = tid; q < ntot; q += kBlkThreads) {
        out[q] = (TS) sm[q];
        if (!CGS && tmp) tmp[q] = (TS) sm[ntot + q];
    }
    if (tid == 0 && st) {
        st->it = it;
        st->residual = res;
        st->cond = 0;
    }
}

// ---------------------------------------------------------------- pipelined Jacobi coarse solve
//
// VCycleMG::call_solve_jacobi (src/pressure/VCycleMG.cpp:725-798) on the
// cluster with every access to the rank's own shared memory and one cluster
// barrier per sweep, for boundary programs of a single wave (every
// configuration of the reference's tests):
//  * rank r owns the z-planes [kb[r], kb[r+1]) of a split chosen on the host
//    so that no boundary assignment with an inner root crosses a rank; it
//    keeps them plus one halo plane on each side, in three buffers of the
//    same layout in every rank;
//  * after a sweep each rank sends its two edge planes to the neighbours'
//    halos as two bulk shared-memory copies that complete on the receiver's
//    mbarrier (point to point, no multicast); the receiver waits on it
//    before the next sweep reads the halo;
//  * the boundary program runs inside the sweep: in a single-wave program no
//    root is ever a target, so a root is either an inner cell, and the thread
//    that computes the root's new value also evaluates the target's chain
//    from it (a per-thread target list built at launch), or a cell that
//    nothing writes, whose targets are set once before the loop;
//  * the residual of iterate k-1 is summed in the pass that computes iterate
//    k (both read only iterate k-1), so the loop decision for k arrives one
//    sweep late.  Three buffers keep iterates k-2, k-1 and k apart and the
//    reference's result is still there when the loop stops: after `it`
//    sweeps and swaps, out holds iterate it when it is odd and iterate it-1
//    when it is even, tmp the other one.
// Values, iteration count and residual are those of k_mg_coarse_cluster.

// boundary assignment with an inner root in the rank's planes: the target's
// and the root's local index in a buffer, the chain
struct HaloTarget {
    double val[kBcMaxDepth];
    uint32_t dst, root;
    uint32_t depth_neg;  // depth | neg << 8
    uint32_t pad;
};

// ranks of the pipelined coarse solve: up to 16 CTAs (a non-portable cluster size)
constexpr int kPipeMaxRanks = 16;

// z-planes of each rank: rank r owns [kb[r], kb[r+1])
struct PlaneSplit {
    int kb[kPipeMaxRanks + 1];
};

// smem -> the same-layout smem of a peer CTA, completing on the peer's
// mbarrier (a point-to-point bulk copy, no multicast)
__device__ __forceinline__ void bulk_copy_to_peer(uint32_t dst, uint32_t src, uint32_t bytes, uint32_t mbar) {
    asm volatile("cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     dst),
                 "r"(src), "r"(bytes), "r"(mbar)
                 : "memory");
}
__device__ __forceinline__ uint32_t mapa_u32(uint32_t a, int rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
    return r;
}

constexpr int kHaloPolls = 1 << 20;  // mbarrier polls before a halo wait gives up
constexpr int kPipeCells = 4;        // inner cells per thread of k_mg_coarse_jacobi_pipe

template <typename TS>
__global__ void __launch_bounds__(kClusterThreads, 1)
k_mg_coarse_jacobi_pipe(TS *__restrict__ out, TS *__restrict__ tmp, const TS *__restrict__ b,
                        const uint8_t *__restrict__ flags, Level L, Box3 box, MgCoef c, double rx, double ry, double rz,
                        BcView bc, double tol, int rel, long long max_it, PlaneSplit sp, int plane_cap,
                        int target_cap, int fix_cap, LoopState *__restrict__ st, const LoopState *__restrict__ pred) {
    namespace cg = cooperative_groups;
    if (pred && !pred->cond) return;  // every rank reads the same flag
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ __align__(16) double sm[];
    __shared__ double red[32];
    __shared__ double parts[2][kPipeMaxRanks];
    __shared__ int s_nt, s_nf, s_over, s_overs[kPipeMaxRanks], s_fail;
    __shared__ __align__(8) uint64_t hb[3];  // halo arrivals per buffer
    const int tid = threadIdx.x;
    const int rank = (int) cl.block_rank();
    const int cs = (int) cl.num_blocks();
    const int nj = (int) L.Nx, nk = (int) (L.Nx * L.Ny);
    const int kb0 = sp.kb[rank], kb1 = sp.kb[rank + 1], own = kb1 - kb0;
    const int bstride = (plane_cap + 2) * nk;  // doubles per buffer (nk even: 16-byte planes)
    double *X = sm;
    HaloTarget *tg = (HaloTarget *) (sm + 3 * (int64_t) bstride);  // targets and roots in own planes
    HaloTarget *fx = tg + target_cap;                                  // the chain crosses to a neighbour
    const uint32_t base = (uint32_t) __cvta_generic_to_shared(sm);
    if (tid == 0) {
        s_nt = 0;
        s_nf = 0;
        s_over = 0;
        s_fail = 0;
        for (int s = 0; s < 3; s++) tc::mbar_init(&hb[s], 1);
        tc::fence_barrier_init();
    }
    // buffer 0: planes kb0-1 .. kb1 of out (local plane lp = k - kb0 + 1)
    for (int q = tid; q < (own + 2) * nk; q += kClusterThreads) {
        const int k = kb0 - 1 + q / nk;
        X[q] = (k >= 0 && k < (int) L.Nz) ? (double) out[(int64_t) k * nk + q % nk] : 0.0;
    }
    // this thread's inner cells: slot m holds box cell lin = tid + m * threads
    // of the rank's planes; local index and right-hand side
    const int z0 = max((int) box.z0, kb0), z1 = min((int) box.z1, kb1 - 1);
    const int nx = (int) box.nx(), nxy = (int) (box.nx() * box.ny());
    int ca[kPipeCells];
    double cb[kPipeCells];
    unsigned m0 = 0;
    {
        const int ncell = z1 >= z0 ? (z1 - z0 + 1) * nxy : 0;
#pragma unroll
        for (int m = 0; m < kPipeCells; m++) {
            const int lin = tid + m * kClusterThreads;
            ca[m] = nk;
            cb[m] = 0.0;
            if (lin < ncell) {
                const int k = z0 + lin / nxy, r = lin % nxy, j = (int) box.y0 + r / nx, i = (int) box.x0 + r % nx;
                const int o = i + nj * j;
                const int64_t q = (int64_t) k * nk + o;
                if (__ldg(flags + q) & kInner) {
                    ca[m] = (k - kb0 + 1) * nk + o;
                    cb[m] = (double) b[q];
                    m0 |= 1u << m;
                }
            }
        }
    }
    __syncthreads();
    // The boundary program on iterate 0 for the targets in own planes (roots
    // lie within one plane, in own or halo planes, and are never targets), and
    // two tables of the targets whose root is an inner cell: target and root in
    // own planes (re-evaluated in the sweep from the root's new value), and a
    // chain that crosses to a neighbouring rank, target or root in a halo plane
    // (re-evaluated at the start of the next sweep, once the halo has arrived,
    // by both ranks); targets of constant roots stay as set here.
    const int64_t q_begin = bc.waves > 0 ? bc.begin[0] : 0, q_end = bc.waves > 0 ? bc.begin[1] : 0;
    for (int64_t q0 = q_begin; q0 < q_end; q0 += kClusterThreads) {
        const int64_t qq = q0 + tid;
        if (qq >= q_end) continue;
        const int t = (int) __ldg(bc.target + qq), kt = t / nk;
        const int r = (int) __ldg(bc.root + qq), kr = r / nk;
        const bool own_t = kt >= kb0 && kt < kb1, own_r = kr >= kb0 && kr < kb1;
        const bool halo_t = kt == kb0 - 1 || kt == kb1, halo_r = kr == kb0 - 1 || kr == kb1;
        if (!own_t && !own_r) continue;
        const int d = __ldg(bc.depth + qq);
        const uint8_t mneg = __ldg(bc.neg + qq);
        if (own_t) {
            double x = X[(kr - kb0 + 1) * nk + (r - kr * nk)];
#pragma unroll
            for (int s = 0; s < kBcMaxDepth; s++)
                if (s < d) x = ((mneg >> s) & 1 ? -x : x) + (bc.value ? __ldg(bc.value + s * bc.n + qq) : 0.0);
            X[(kt - kb0 + 1) * nk + (t - kt * nk)] = x;
        }
        if (!(__ldg(flags + r) & kInner)) continue;  // constant root: set once above
        HaloTarget *h = nullptr;
        if (own_t && own_r) {
            const int slot = atomicAdd(&s_nt, 1);
            if (slot < target_cap) h = &tg[slot];
        } else if ((own_t && halo_r) || (own_r && halo_t)) {
            const int slot = atomicAdd(&s_nf, 1);
            if (slot < fix_cap) h = &fx[slot];
        }
        if (!h) {
            s_over = 1;  // a table overflowed, or a chain spans more than one plane
            continue;
        }
#pragma unroll
        for (int s = 0; s < kBcMaxDepth; s++) h->val[s] = (s < d && bc.value) ? __ldg(bc.value + s * bc.n + qq) : 0.0;
        h->dst = (uint32_t) ((kt - kb0 + 1) * nk + (t - kt * nk));
        h->root = (uint32_t) ((kr - kb0 + 1) * nk + (r - kr * nk));
        h->depth_neg = (uint32_t) d | (uint32_t) mneg << 8;
        h->pad = 0;
    }
    __syncthreads();
    const int nt = min(s_nt, target_cap), nf = min(s_nf, fix_cap);
    cl.sync();
    // every rank learns every rank's error flag, so all take the same path
    if (tid < cs) cl.map_shared_rank(s_overs, tid)[rank] = s_over;
    // halo planes of iterate 0 from the neighbours' own planes
    if (rank > 0) {
        const double *src = cl.map_shared_rank(X, rank - 1) + (int64_t) (kb0 - sp.kb[rank - 1]) * nk;
        for (int q = tid; q < nk; q += kClusterThreads) X[q] = src[q];
    }
    if (rank < cs - 1) {
        const double *src = cl.map_shared_rank(X, rank + 1) + nk;
        for (int q = tid; q < nk; q += kClusterThreads) X[(own + 1) * nk + q] = src[q];
    }
    __syncthreads();
    for (int q = tid; q < (own + 2) * nk; q += kClusterThreads) X[2 * bstride + q] = X[bstride + q] = X[q];
    cl.sync();
    int over = 0;
    for (int r = 0; r < cs; r++) over |= s_overs[r];

    // edge planes sent per sweep: own plane 1 to rank-1's upper halo (its local
    // plane own(rank-1) + 1), own plane `own` to rank+1's lower halo (plane 0)
    const uint32_t plane_bytes = (uint32_t) nk * 8u;
    const uint32_t halo_bytes = plane_bytes * (uint32_t) ((rank > 0) + (rank < cs - 1));
    uint32_t dst_lo = 0, dst_hi = 0, bar_lo = 0, bar_hi = 0;
    if (tid == 0) {
        if (rank > 0) {
            const int own_lo = kb0 - sp.kb[rank - 1];
            dst_lo = mapa_u32(base + (uint32_t) ((own_lo + 1) * nk) * 8u, rank - 1);
            bar_lo = mapa_u32((uint32_t) __cvta_generic_to_shared(hb), rank - 1);
        }
        if (rank < cs - 1) {
            dst_hi = mapa_u32(base, rank + 1);
            bar_hi = mapa_u32((uint32_t) __cvta_generic_to_shared(hb), rank + 1);
        }
    }
    unsigned par = 0;       // bit s: parity of the pending phase of hb[s]
    long long unwaited = 0; // a phase whose halos were sent and not yet waited for (0: none)

    double res = 10000.;
    long long it = 0;
    if (over) {
        it = -1;  // target table too small or split violated: nothing computed, reported as an error
    } else if (rel || (res > tol && it < max_it)) {
        // phase k: iterate k from iterate k-1 (unless k-1 == max_it) and the
        // residual of iterate k-1 (k >= 2, or k = 1 for the relative
        // tolerance); iterate k-1 is accepted on entry
        // res > tol is decided on the squared sum where that is exact: outside
        // +-16 units of roundoff around tol^2 the rounded square root lies on
        // the same side of tol; inside that band, or for tol^2 outside the
        // normal range, the square root is taken.  Buffers rotate without a
        // 64-bit modulo.
        double tol2 = tol * tol;
        bool have_s = false;
        double s_last = 0.0;
        int sp_ = 0, sn = 1;
        for (long long k = 1;; k++, sp_ = sn, sn = sn == 2 ? 0 : sn + 1) {
            const double *P = X + sp_ * bstride;
            double *N = X + sn * bstride;
            const bool sweep = k - 1 < max_it, resid = k >= 2 || rel;
            if (unwaited) {
                // halos of iterate k-1 (sent in phase k-1) must have landed
                if (tid == 0) {
                    if (!tc::mbar_wait(&hb[sp_], (par >> sp_) & 1u, kHaloPolls)) s_fail = 1;
                    par ^= 1u << sp_;
                }
                unwaited = 0;
                __syncthreads();
                if (nf > 0) {
                    // chains across ranks: iterate k-1's targets from its roots, now all present
                    double *Pw = X + sp_ * bstride;
                    for (int t = tid; t < nf; t += kClusterThreads) {
                        const HaloTarget &h = fx[t];
                        double x = Pw[h.root];
                        const int d = (int) (h.depth_neg & 0xffu);
                        const uint32_t mneg = h.depth_neg >> 8;
#pragma unroll
                        for (int s = 0; s < kBcMaxDepth; s++)
                            if (s < d) x = ((mneg >> s) & 1 ? -x : x) + h.val[s];
                        Pw[h.dst] = x;
                    }
                    __syncthreads();
                }
            }
            double acc = 0.0, v[kPipeCells];
#pragma unroll
            for (int m = 0; m < kPipeCells; m++) {
                v[m] = 0.0;
                if (!(m0 >> m & 1)) continue;
                const int a = ca[m];
                const double c0 = P[a], xm = P[a - 1], xp = P[a + 1], ym = P[a - nj], yp = P[a + nj],
                             zm = P[a - nk], zp = P[a + nk];
                if (resid) {
                    const double rr = cb[m] - (rx * (xm - 2 * c0 + xp) + ry * (ym - 2 * c0 + yp) +
                                               rz * (zm - 2 * c0 + zp));
                    acc += rr * rr;
                }
                const double out_h = c.beta * (c.dsign * cb[m] + c.ax * (xp + xm) + c.ay * (yp + ym) + c.az * (zp + zm));
                v[m] = c.omw * c0 + c.w * out_h;
            }
            bool reduced = false;
            if (sweep) {
#pragma unroll
                for (int m = 0; m < kPipeCells; m++)
                    if (m0 >> m & 1) N[ca[m]] = v[m];
                if (resid) {
                    // first stage of artss_block_sum, second stage below by warp 0
                    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
                    if ((tid & 31) == 0) red[tid >> 5] = acc;
                }
                __syncthreads();  // the roots' new values are in N, the warp sums in red
                if (resid && tid < 32) {
                    acc = tid < kClusterThreads / 32 ? red[tid] : 0.0;
                    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
                    acc = __shfl_sync(0xffffffffu, acc, 0);
                    if (tid < cs) cl.map_shared_rank(parts[k & 1], tid)[rank] = acc;
                }
                reduced = resid;
                for (int t = tid; t < nt; t += kClusterThreads) {
                    const HaloTarget &h = tg[t];
                    double x = N[h.root];
                    const int d = (int) (h.depth_neg & 0xffu);
                    const uint32_t mneg = h.depth_neg >> 8;
#pragma unroll
                    for (int s = 0; s < kBcMaxDepth; s++)
                        if (s < d) x = ((mneg >> s) & 1 ? -x : x) + h.val[s];
                    N[h.dst] = x;
                }
                if (tid == 0) tc::mbar_expect_tx(&hb[sn], halo_bytes);  // this rank's incoming halos
                __syncthreads();  // the edge planes are complete
                if (tid == 0) {
                    tc::fence_proxy_async();
                    const uint32_t nb = base + (uint32_t) (sn * bstride) * 8u;
                    if (rank > 0)
                        bulk_copy_to_peer(dst_lo + (uint32_t) (sn * bstride) * 8u, nb + plane_bytes, plane_bytes,
                                          bar_lo + (uint32_t) sn * 8u);
                    if (rank < cs - 1)
                        bulk_copy_to_peer(dst_hi + (uint32_t) (sn * bstride) * 8u, nb + (uint32_t) own * plane_bytes,
                                          plane_bytes, bar_hi + (uint32_t) sn * 8u);
                }
                unwaited = k;
            }
            if (resid && !reduced) {
                acc = artss_block_sum(acc, red);  // complete in thread 0
                acc = __shfl_sync(0xffffffffu, acc, 0);
                if (tid < cs) cl.map_shared_rank(parts[k & 1], tid)[rank] = acc;
            }
            cl.sync();
            if (!resid) {
                it = k;  // cond(0): res = 10000 > tol and 0 < max_it
                continue;
            }
            double s = 0.0;
            for (int r = 0; r < cs; r++) s += parts[k & 1][r];
            if (k == 1) {
                // relative tolerance: scaled by the residual of iterate 0
                tol *= sqrt(s);
                tol2 = tol * tol;
                if (!(res > tol && 0 < max_it)) break;
                it = 1;
                continue;
            }
            // residual of iterate k-1: sqrt(s)
            const bool fast = tol2 > 1e-280 && tol2 < 1e280;
            bool above;
            if (fast && s > tol2 * (1.0 + 0x1p-49)) above = true;
            else if (fast && s < tol2 * (1.0 - 0x1p-49)) above = false;
            else above = sqrt(s) > tol;
            have_s = true;
            s_last = s;
            if (!(above && k - 1 < max_it)) break;  // it = k-1 stands
            it = k;
        }
        if (have_s) res = sqrt(s_last);
    }
    // the last halos sent must land before any rank leaves (their source and
    // destination are shared memory)
    if (unwaited && tid == 0) {
        const int s = (int) (unwaited % 3);
        if (!tc::mbar_wait(&hb[s], (par >> s) & 1u, kHaloPolls)) s_fail = 1;
    }
    // iterate `it` lives in buffer it%3, iterate it-1 in (it-1)%3 (it >= 1)
    if (it >= 0) {
        const double *Xo = X + (it % 3) * bstride, *Xt = Xo;
        if (it >= 1) {
            const double *Xprev = X + ((it - 1) % 3) * bstride;
            if (it % 2 == 0) Xo = Xprev;
            else Xt = Xprev;
        }
        for (int q = tid; q < own * nk; q += kClusterThreads) {
            out[(int64_t) kb0 * nk + q] = (TS) Xo[nk + q];
            if (tmp) tmp[(int64_t) kb0 * nk + q] = (TS) Xt[nk + q];
        }
    }
    __syncthreads();
    if (st && tid == 0 && (s_fail || it < 0)) st->pad = 1;
    if (rank == 0 && tid == 0 && st) {
        st->it = it < 0 ? 0 : it;
        st->residual = res;
        st->cond = 0;
    }
    cl.sync();
}

// Launch shape of the cluster coarse solve, or false when the level does not fit it.
// ranks of the cluster for a level: one per z-plane up to kClusterSize
inline int cluster_ranks(const Level &L) { return (int) std::min<int64_t>(kClusterSize, L.Nz); }

bool cluster_fits(const artss_ctx *ctx, int level, int buffers, int *plane_cap, int64_t *smem) {
    const Level &L = ctx->lvl[level];
    const BcProgram &p = ctx->bc[level][ARTSS_FIELD_P];
    if (p.present && p.waves > kCoarseMaxWaves) return false;
    const int cs = cluster_ranks(L);
    if (cs < 2 || L.Nz > kClusterMaxPlanes || L.size() > (int64_t) 1 << 24) return false;
    int cap = 0;
    for (int r = 0; r < cs; r++) {
        const int64_t a = (int64_t) r * L.Nz / cs, e = (int64_t) (r + 1) * L.Nz / cs;
        cap = std::max<int>(cap, (int) (e - a));
        // inner cells of the rank's planes, one thread each per register slot
        const int64_t z0 = std::max<int64_t>(a, L.k1), z1 = std::min<int64_t>(e - 1, L.k2);
        const int64_t cells = z1 >= z0 ? (z1 - z0 + 1) * (L.i2 - L.i1 + 1) * (L.j2 - L.j1 + 1) : 0;
        if (cells > (int64_t) kClusterThreads * kClusterCells) return false;
    }
    const int64_t bytes = buffers * (int64_t) cap * L.nxy() * (int64_t) sizeof(double);
    if (bytes > kCoarseSmemBytes) return false;
    *plane_cap = cap;
    *smem = bytes;
    return true;
}

// Launch data of k_mg_coarse_jacobi_pipe for the level, or false when its
// pressure boundary program does not qualify (more than one wave, an inner
// target, a chain leaving its target's neighbouring planes, no plane split
// that keeps every inner root with its target) or the level does not fit.
// The split cuts the planes as evenly as the forbidden cuts allow.
struct PipeLaunch {
    PlaneSplit split;
    int ranks, plane_cap, target_cap, fix_cap;
    int64_t smem;
};

bool coarse_pipe_plan_new(artss_ctx *ctx, int level, PipeLaunch *pl);

bool coarse_pipe_plan(artss_ctx *ctx, int level, PipeLaunch *pl) {
    BcProgram &p = ctx->bc[level][ARTSS_FIELD_P];
    if (p.pipe_state == -2) {
        PipeLaunch fresh{};
        const bool ok = coarse_pipe_plan_new(ctx, level, &fresh);
        p.pipe_state = ok ? 1 : -1;
        if (ok) {
            p.pipe_kb.assign(fresh.split.kb, fresh.split.kb + kPipeMaxRanks + 1);
            p.pipe_ranks = fresh.ranks;
            p.pipe_cap = fresh.plane_cap;
            p.pipe_tcap = fresh.target_cap;
            p.pipe_fcap = fresh.fix_cap;
            p.pipe_smem = fresh.smem;
        }
    }
    if (p.pipe_state != 1) return false;
    for (int r = 0; r <= kPipeMaxRanks; r++) pl->split.kb[r] = p.pipe_kb[r];
    pl->ranks = p.pipe_ranks;
    pl->plane_cap = p.pipe_cap;
    pl->target_cap = p.pipe_tcap;
    pl->fix_cap = p.pipe_fcap;
    pl->smem = p.pipe_smem;
    return true;
}

bool coarse_pipe_plan_new(artss_ctx *ctx, int level, PipeLaunch *pl) {
    BcProgram &p = ctx->bc[level][ARTSS_FIELD_P];
    const Level &L = ctx->lvl[level];
    const std::vector<bool> &in = ctx->h_inner[level];
    const int nz = (int) L.Nz;
    if (cluster_ranks(L) < 2 || L.nxy() % 2 || in.empty() || (int64_t) in.size() != L.size()) return false;
    if (p.present && p.waves > 1) return false;
    // forbidden[c]: no rank boundary between planes c-1 and c; the ghost planes
    // stay with their neighbour (a rank of a ghost plane alone has no cells)
    std::vector<char> forbidden(nz + 1, 0);
    forbidden[1] = forbidden[nz - 1] = 1;
    const int64_t n = p.present ? p.n : 0;
    for (int64_t q = 0; q < n; q++) {
        const int64_t t = p.h_target[q], r = p.h_root[q];
        const int kt = (int) (t / L.nxy()), kr = (int) (r / L.nxy());
        if (in[(size_t) t] || kr < kt - 1 || kr > kt + 1) return false;
    }
    static bool attr_set = false;
    if (!attr_set) {
        if (cudaFuncSetAttribute(k_mg_coarse_jacobi_pipe<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int) kCoarseSmemBytes) != cudaSuccess ||
            cudaFuncSetAttribute(k_mg_coarse_jacobi_pipe<double>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        attr_set = true;
    }
    // the most ranks (up to one per plane, at most kPipeMaxRanks) that admit a
    // split, fit the rank's cell slots and shared memory and can be placed
    const int64_t nxy_in = (L.i2 - L.i1 + 1) * (L.j2 - L.j1 + 1);
    for (int cs = (int) std::min<int64_t>(kPipeMaxRanks, L.Nz); cs >= 2; cs--) {
        PlaneSplit sp{};
        bool ok = true;
        for (int r = 1; r < cs && ok; r++) {
            const int ideal = (int) ((int64_t) r * nz / cs);
            const int lo = sp.kb[r - 1] + 1, hi = nz - (cs - r);  // every rank keeps at least one plane
            int best = -1;
            for (int cut = lo; cut <= hi; cut++)
                if (!forbidden[cut] && (best < 0 || std::abs(cut - ideal) < std::abs(best - ideal))) best = cut;
            if (best < 0) ok = false;
            else sp.kb[r] = best;
        }
        if (!ok) continue;
        sp.kb[cs] = nz;
        int cap = 0, tcap = 0, fcap = 0;
        for (int r = 0; r < cs && ok; r++) {
            const int a = sp.kb[r], e = sp.kb[r + 1];
            cap = std::max(cap, e - a);
            const int64_t z0 = std::max<int64_t>(a, L.k1), z1 = std::min<int64_t>(e - 1, L.k2);
            if (z1 >= z0 && (z1 - z0 + 1) * nxy_in > (int64_t) kClusterThreads * kPipeCells) ok = false;
            int nt = 0, nf = 0;
            for (int64_t q = 0; q < n; q++) {
                if (!in[(size_t) p.h_root[q]]) continue;
                const int kt = (int) (p.h_target[q] / L.nxy()), kr = (int) (p.h_root[q] / L.nxy());
                const bool own_t = kt >= a && kt < e, own_r = kr >= a && kr < e;
                if (own_t && own_r) nt++;
                else if ((own_t && (kr == a - 1 || kr == e)) || (own_r && (kt == a - 1 || kt == e))) nf++;
                // a rank of one plane sends its plane both ways before such a
                // target is set, and the far neighbour cannot set it itself
                if (own_t && !own_r && e - a == 1) ok = false;
            }
            tcap = std::max(tcap, nt);
            fcap = std::max(fcap, nf);
        }
        const int64_t smem = 3 * (int64_t) (cap + 2) * L.nxy() * (int64_t) sizeof(double) +
                             (int64_t) (tcap + fcap) * (int64_t) sizeof(HaloTarget);
        if (!ok || smem > kCoarseSmemBytes) continue;
        // the device must be able to place a cluster of this size (more than 8 is non-portable)
        cudaLaunchConfig_t lc = {};
        cudaLaunchAttribute at[1];
        lc.gridDim = dim3(cs, 1, 1);
        lc.blockDim = dim3(kClusterThreads, 1, 1);
        lc.dynamicSmemBytes = (size_t) smem;
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = cs;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        lc.attrs = at;
        lc.numAttrs = 1;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, k_mg_coarse_jacobi_pipe<double>, &lc) != cudaSuccess ||
            clusters < 1) {
            cudaGetLastError();
            continue;
        }
        pl->split = sp;
        pl->ranks = cs;
        pl->plane_cap = cap;
        pl->target_cap = tcap;
        pl->fix_cap = fcap;
        pl->smem = smem;
        return true;
    }
    return false;
}

inline cudaLaunchConfig_t cluster_config(artss_ctx *ctx, int cs, int64_t smem, cudaLaunchAttribute *at) {
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(cs, 1, 1);
    lc.blockDim = dim3(kClusterThreads, 1, 1);
    lc.dynamicSmemBytes = (size_t) smem;
    lc.stream = ctx->stream;
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    return lc;
}

template <bool CGS, typename TS>
int launch_coarse_cluster(artss_ctx *ctx, TS *out, TS *tmp, const TS *b, int level, const MgCoef &c, double rx,
                          double ry, double rz, const BcView &v, double tol, int rel, long long mi, int cap,
                          int64_t smem, LoopState *st, const LoopState *pred) {
    static bool attr_set = false;
    if (!attr_set) {
        ARTSS_CK(cudaFuncSetAttribute(k_mg_coarse_cluster<CGS, TS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int) kCoarseSmemBytes));
        attr_set = true;
    }
    const Level &L = ctx->lvl[level];
    cudaLaunchAttribute at[1];
    cudaLaunchConfig_t lc = cluster_config(ctx, cluster_ranks(L), smem, at);
    ARTSS_LAUNCH(ctx, FAM_MG_COARSE, ARTSS_CK(cudaLaunchKernelEx(&lc, k_mg_coarse_cluster<CGS, TS>, out, tmp, b,
                                                                  (const uint8_t *) ctx->d_flags[level], L,
                                                                  inner_box(L), c, rx, ry, rz, v, tol, rel, mi, cap,
                                                                  st, pred)));
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

template <typename TS>
int launch_coarse_pipe(artss_ctx *ctx, TS *out, TS *tmp, const TS *b, int level, const MgCoef &c, double rx,
                       double ry, double rz, const BcView &v, double tol, int rel, long long mi, const PipeLaunch &pl,
                       LoopState *st, const LoopState *pred) {
    static bool attr_set = false;
    if (!attr_set) {
        ARTSS_CK(cudaFuncSetAttribute(k_mg_coarse_jacobi_pipe<TS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int) kCoarseSmemBytes));
        ARTSS_CK(cudaFuncSetAttribute(k_mg_coarse_jacobi_pipe<TS>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        attr_set = true;
    }
    const Level &L = ctx->lvl[level];
    cudaLaunchAttribute at[1];
    cudaLaunchConfig_t lc = cluster_config(ctx, pl.ranks, pl.smem, at);
    ARTSS_LAUNCH(ctx, FAM_MG_COARSE, ARTSS_CK(cudaLaunchKernelEx(&lc, k_mg_coarse_jacobi_pipe<TS>, out, tmp, b,
                                                                  (const uint8_t *) ctx->d_flags[level], L,
                                                                  inner_box(L), c, rx, ry, rz, v, tol, rel, mi,
                                                                  pl.split, pl.plane_cap, pl.target_cap, pl.fix_cap,
                                                                  st, pred)));
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

BcView bc_view(const artss_ctx *ctx, int level) {
    const BcProgram &p = ctx->bc[level][ARTSS_FIELD_P];
    BcView v{};
    if (p.present && p.n > 0) {
        v = BcView{p.d_target, p.d_root, p.d_depth, p.d_neg, p.d_value, p.n, p.waves, {}};
        for (int w = 0; w <= p.waves; w++) v.begin[w] = p.wave_begin[w];
    }
    return v;
}

// out = 0 (the coarse solve's start on the cluster path)
__global__ void k_fill_f32(float *__restrict__ f, int64_t n, const LoopState *__restrict__ pred) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    if (pred && !pred->cond) return;
    for (int64_t q = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; q < n; q += (int64_t) gridDim.x * blockDim.x)
        f[q] = 0.f;
}

// true when the level fits k_mg_coarse_block: its inner box in the threads'
// cell slots, its array (and tmp's) in shared memory, its boundary program in
// the threads' assignment slots
bool block_fits(const artss_ctx *ctx, int level, int buffers, int64_t *smem) {
    const Level &L = ctx->lvl[level];
    const BcProgram &p = ctx->bc[level][ARTSS_FIELD_P];
    if (p.present && p.waves > kCoarseMaxWaves) return false;
    const Box3 box = inner_box(L);
    if (blk_slots(box) > (int64_t) kBlkThreads * (kBlkCells / 2)) return false;
    const int64_t bytes = buffers * L.size() * (int64_t) sizeof(double);
    if (bytes > kCoarseSmemBytes) return false;
    if (p.present && p.n > 0) {
        int64_t per_thread = 0;
        for (int w = 0; w < p.waves; w++)
            per_thread += (p.wave_begin[w + 1] - p.wave_begin[w] + kBlkThreads - 1) / kBlkThreads;
        if (per_thread > kBlkTargets) return false;
    }
    *smem = bytes;
    return true;
}

template <bool CGS, typename TS>
int launch_coarse_block(artss_ctx *ctx, TS *out, TS *tmp, const TS *b, int level, const MgCoef &c, double rx,
                        double ry, double rz, const BcView &v, double tol, int rel, long long mi, int64_t smem,
                        LoopState *st, const LoopState *pred, bool zero_start) {
    static bool attr_set = false;
    if (!attr_set) {
        ARTSS_CK(cudaFuncSetAttribute(k_mg_coarse_block<CGS, TS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int) kCoarseSmemBytes));
        attr_set = true;
    }
    const Level &L = ctx->lvl[level];
    ARTSS_LAUNCH_PDL(ctx, FAM_MG_COARSE, (k_mg_coarse_block<CGS, TS>), 1, kBlkThreads, smem, out, tmp, b,
                     (const uint8_t *) ctx->d_flags[level], L, inner_box(L), c, rx, ry, rz, v, tol, rel, mi, st, pred, zero_start ? 1 : 0);
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

// FP64 solve of one level's pressure system by the cluster kernel on FP32
// storage (the coarsest-grid solve of the mixed-precision V-cycle); the
// level's boundary values are taken as zero, tol is relative to the initial
// residual.  block: by k_mg_coarse_block where the level fits one block;
// zero_start: the solve starts from zero (out's contents are not read).
int coarse_cluster_f32(artss_ctx *ctx, float *out, const float *b, int level, int smoother, double w, double tol,
                       long long max_it, const LoopState *pred, bool block, bool zero_start) {
    const bool cgs = smoother == ARTSS_SMOOTHER_CGS;
    int cap = 0;
    int64_t smem = 0;
    PipeLaunch pl{};
    const bool pipe = !cgs && coarse_pipe_plan(ctx, level, &pl);
    int64_t bs = 0;
    if (!pipe && !cluster_fits(ctx, level, cgs ? 1 : 2, &cap, &smem) &&
        !(block && block_fits(ctx, level, cgs ? 1 : 2, &bs))) {
        set_error("the coarsest level does not fit the cluster coarse solve");
        return ARTSS_ERR_LIMIT;
    }
    const artss_grid_desc &g = ctx->grid;
    MgCoef c{};
    c.ax = 1. / (g.dx[level] * g.dx[level]);
    c.ay = 1. / (g.dy[level] * g.dy[level]);
    c.az = 1. / (g.dz[level] * g.dz[level]);
    c.beta = 1. / (2. * (c.ax + c.ay + c.az));
    c.dsign = -1;
    c.w = w;
    c.omw = 1 - w;
    BcView v = bc_view(ctx, level);
    v.value = nullptr;  // homogeneous: the correction equation has zero boundary values
    int64_t bsmem = 0;
    if (block && block_fits(ctx, level, cgs ? 1 : 2, &bsmem)) {
        if (cgs)
            return launch_coarse_block<true, float>(ctx, out, nullptr, b, level, c, c.ax, c.ay, c.az, v, tol, 1, max_it,
                                                    bsmem, nullptr, pred, zero_start);
        return launch_coarse_block<false, float>(ctx, out, nullptr, b, level, c, c.ax, c.ay, c.az, v, tol, 1, max_it,
                                                 bsmem, nullptr, pred, zero_start);
    }
    if (zero_start) {
        const int64_t n = ctx->lvl[level].size();
        ARTSS_LAUNCH_PDL(ctx, FAM_FIELD_OP, k_fill_f32, flat_blocks(n), 256, 0, out, n, pred);
        ARTSS_LAUNCH_CK(ctx);
    }
    if (cgs)
        return launch_coarse_cluster<true, float>(ctx, out, nullptr, b, level, c, c.ax, c.ay, c.az, v, tol, 1, max_it,
                                                  cap, smem, nullptr, pred);
    if (pipe)
        return launch_coarse_pipe<float>(ctx, out, nullptr, b, level, c, c.ax, c.ay, c.az, v, tol, 1, max_it, pl, nullptr,
                                         pred);
    return launch_coarse_cluster<false, float>(ctx, out, nullptr, b, level, c, c.ax, c.ay, c.az, v, tol, 1, max_it, cap,
                                               smem, nullptr, pred);
}

// true when the level is handled by k_mg_coarse_solve
bool coarse_fits(const artss_ctx *ctx, int level) {
    const BcProgram &p = ctx->bc[level][ARTSS_FIELD_P];
    return ctx->lvl[level].size() <= kCoarseMaxCells && (!p.present || p.waves <= kCoarseMaxWaves);
}

int mg_coarse_solve(artss_mg *mg, double *out, double *tmp, const double *b, int level) {
    artss_ctx *ctx = mg->ctx;
    const Level &L = ctx->lvl[level];
    const Box3 box = inner_box(L);
    const BcProgram &p = ctx->bc[level][ARTSS_FIELD_P];
    BcView v{};
    if (p.present && p.n > 0) {
        v = BcView{p.d_target, p.d_root, p.d_depth, p.d_neg, p.d_value, p.n, p.waves, {}};
        for (int w = 0; w <= p.waves; w++) v.begin[w] = p.wave_begin[w];
    }
    const artss_grid_desc &g = ctx->grid;
    const double rx = 1. / (g.dx[level] * g.dx[level]), ry = 1. / (g.dy[level] * g.dy[level]),
                 rz = 1. / (g.dz[level] * g.dz[level]);
    const MgCoef c = mg_coef(mg, level);
    const bool cgs = mg->cfg.smoother == ARTSS_SMOOTHER_CGS;
    const int64_t smem = (cgs ? 1 : 2) * L.size() * (int64_t) sizeof(double);
    const double tol = mg->cfg.smoother_tol_res;
    const long long mi = mg->cfg.smoother_max_iter;
    int cap = 0;
    int64_t csmem = 0;
    PipeLaunch pl{};
    if (mg->cluster_coarse && !cgs && mg->pipelined_coarse && coarse_pipe_plan(ctx, level, &pl))
        return launch_coarse_pipe<double>(ctx, out, tmp, b, level, c, rx, ry, rz, v, tol, 0, mi, pl, ctx->d_loop + 1,
                                          nullptr);
    if (mg->cluster_coarse && cluster_fits(ctx, level, cgs ? 1 : 2, &cap, &csmem)) {
        if (cgs)
            return launch_coarse_cluster<true, double>(ctx, out, tmp, b, level, c, rx, ry, rz, v, tol, 0, mi, cap, csmem,
                                                       ctx->d_loop + 1, nullptr);
        return launch_coarse_cluster<false, double>(ctx, out, tmp, b, level, c, rx, ry, rz, v, tol, 0, mi, cap, csmem,
                                                    ctx->d_loop + 1, nullptr);
    }
    if (smem <= kCoarseSmemBytes) {
        static bool attr_set[2] = {false, false};
        if (!attr_set[cgs]) {
            if (cgs) ARTSS_CK(cudaFuncSetAttribute(k_mg_coarse_solve<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) kCoarseSmemBytes));
            else ARTSS_CK(cudaFuncSetAttribute(k_mg_coarse_solve<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) kCoarseSmemBytes));
            attr_set[cgs] = true;
        }
        if (cgs)
            ARTSS_LAUNCH(ctx, FAM_MG_COARSE, k_mg_coarse_solve<true, true><<<1, kCoarseThreads, smem, ctx->stream>>>(
                out, tmp, b, ctx->d_flags[level], L, box, c, rx, ry, rz, v, tol, mi, ctx->d_loop + 1));
        else
            ARTSS_LAUNCH(ctx, FAM_MG_COARSE, k_mg_coarse_solve<false, true><<<1, kCoarseThreads, smem, ctx->stream>>>(
                out, tmp, b, ctx->d_flags[level], L, box, c, rx, ry, rz, v, tol, mi, ctx->d_loop + 1));
    } else if (cgs) {
        ARTSS_LAUNCH(ctx, FAM_MG_COARSE, k_mg_coarse_solve<true, false><<<1, kCoarseThreads, 0, ctx->stream>>>(
            out, tmp, b, ctx->d_flags[level], L, box, c, rx, ry, rz, v, tol, mi, ctx->d_loop + 1));
    } else {
        ARTSS_LAUNCH(ctx, FAM_MG_COARSE, k_mg_coarse_solve<false, false><<<1, kCoarseThreads, 0, ctx->stream>>>(
            out, tmp, b, ctx->d_flags[level], L, box, c, rx, ry, rz, v, tol, mi, ctx->d_loop + 1));
    }
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

int mg_solve(artss_mg *mg, double *out, double *tmp, const double *b, int level, int64_t *iterations) {
    artss_ctx *ctx = mg->ctx;
    const Level &L = ctx->lvl[level];
    if (L.Nx <= 4 && L.Ny <= 4) {
        if (iterations) *iterations = 0;
        return mg_smooth(mg, out, tmp, b, level);
    }
    if (mg->fused_coarse && coarse_fits(ctx, level)) {
        if (iterations) *iterations = -1;  // kept on the device (loop slot 1), read on demand
        return mg_coarse_solve(mg, out, tmp, b, level);
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
    return tuned_column_launch(ctx, kTuneMgRestrict, coarse_level, box, true, [&](dim3 g, dim3 b) -> int {
        ARTSS_LAUNCH_PDL(ctx, FAM_MG_RESTRICT, k_mg_restrict, g, b, 0, coarse, fine, ctx->d_flags[coarse_level], C,
                         ctx->lvl[coarse_level - 1], box);
        ARTSS_LAUNCH_CK(ctx);
        return ARTSS_OK;
    });
}

int mg_prolongate(artss_mg *mg, double *fine, const double *coarse, int coarse_level) {
    artss_ctx *ctx = mg->ctx;
    const Level &C = ctx->lvl[coarse_level];
    const Box3 box = inner_box(C);
    return tuned_column_launch(ctx, kTuneMgProlongate, coarse_level, box, true, [&](dim3 g, dim3 b) -> int {
        ARTSS_LAUNCH_PDL(ctx, FAM_MG_PROLONGATE, k_mg_prolongate, g, b, 0, fine, coarse, ctx->d_flags[coarse_level], C,
                         ctx->lvl[coarse_level - 1], box);
        ARTSS_LAUNCH_CK(ctx);
        return ARTSS_OK;
    });
}

int mg_residuum(artss_mg *mg, double *out, const double *in, const double *b, int level) {
    artss_ctx *ctx = mg->ctx;
    const Level &L = ctx->lvl[level];
    const Box3 box = inner_box(L);
    const artss_grid_desc &g = ctx->grid;
    const double rx = 1. / (g.dx[level] * g.dx[level]), ry = 1. / (g.dy[level] * g.dy[level]),
                 rz = 1. / (g.dz[level] * g.dz[level]);
    return tuned_column_launch(ctx, kTuneMgResiduum, level, box, out != in && out != b, [&](dim3 gr, dim3 bl) -> int {
        ARTSS_LAUNCH_PDL(ctx, FAM_MG_RESIDUUM, k_mg_residuum, gr, bl, 0, out, in, b, ctx->d_flags[level], L, box, rx,
                         ry, rz);
        ARTSS_LAUNCH_CK(ctx);
        return ARTSS_OK;
    }, 256);
}

// VCycleMG::VCycleMultigrid (VCycleMG.cpp:215-288).  The reference copies out
// into error1[0], works on error1[0] and copies it back; nothing reads out in
// between, so level 0's error1 is out itself here.  b0: the level-0 right-hand
// side (residuum1[0] when null).
int mg_vcycle(artss_mg *mg, double *out, int64_t *coarse_its, const double *b0 = nullptr) {
    artss_ctx *ctx = mg->ctx;
    const int L = mg->L;
    int st;
    const double *R0 = b0 ? b0 : mg->r1[0];
    if (L == 0) return mg_solve(mg, out, mg->tmp[0], R0, 0, coarse_its);
    auto e1 = [&](int l) { return l == 0 ? out : mg->e1[l]; };
    auto r1 = [&](int l) { return l == 0 ? R0 : (const double *) mg->r1[l]; };
    for (int l = 0; l < L; l++) {
        // levels >= 1 start from the zeros set below
        if ((st = mg_smooth(mg, e1(l), mg->tmp[l], r1(l), l, l > 0))) return st;
        if ((st = mg_residuum(mg, mg->r0[l], e1(l), r1(l), l))) return st;
        if (!mg->r0_bc_dead[l] && (st = mg_bc(mg, mg->r0[l], l))) return st;
        if ((st = mg_restrict(mg, mg->r1[l + 1], mg->r0[l], l + 1))) return st;
        // the reference also applies the boundary program to the restricted
        // residual; nothing reads r1's boundary cells (it is only a right-hand
        // side, read on inner cells), so that launch is left out
        if ((st = artss_fill(ctx, mg->e1[l + 1], l + 1, 0.0))) return st;
    }
    // out.copy_data(*m_error0[0]) at VCycleMG.cpp:254 is overwritten below
    // before anything reads it
    for (int l = L; l > 0; l--) {
        if ((st = mg_prolongate(mg, mg->e0[l - 1], e1(l), l))) return st;
        if ((st = mg_bc(mg, mg->e0[l - 1], l - 1))) return st;
        if ((st = artss_add_field(ctx, e1(l - 1), mg->e0[l - 1], l - 1))) return st;
        if (l == L) {
            if ((st = mg_solve(mg, e1(l - 1), mg->tmp[l - 1], r1(l - 1), l - 1, coarse_its))) return st;
        } else {
            // e1 (smoothed, the program applied last) plus e0 (the program applied last)
            if ((st = mg_smooth(mg, e1(l - 1), mg->tmp[l - 1], r1(l - 1), l - 1, true))) return st;
        }
    }
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
    mg->fused_coarse = !(cfg->flags & ARTSS_MG_NO_FUSED_COARSE);
    mg->cluster_coarse = !(cfg->flags & ARTSS_MG_NO_CLUSTER_COARSE);
    mg->pipelined_coarse = !(cfg->flags & ARTSS_MG_NO_PIPELINED_COARSE);
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
    // residuum0[l] is read only by the restriction to level l+1, at the 8 fine
    // cells of each coarse inner cell
    for (int l = 0; l < mg->L; l++) {
        const BcProgram &p = ctx->bc[l][ARTSS_FIELD_P];
        const Level &F = ctx->lvl[l], &Cl = ctx->lvl[l + 1];
        const std::vector<bool> &cin = ctx->h_inner[l + 1];
        if (!p.present || (int64_t) cin.size() != Cl.size()) continue;
        std::vector<bool> is_target((size_t) F.size(), false);
        for (int64_t t : p.h_target) is_target[(size_t) t] = true;
        bool read = false;
        for (int64_t k = 0; k < Cl.Nz && !read; k++)
            for (int64_t j = 0; j < Cl.Ny && !read; j++)
                for (int64_t i = 0; i < Cl.Nx && !read; i++) {
                    if (!cin[(size_t) (i + Cl.Nx * j + Cl.nxy() * k)]) continue;
                    for (int c = 0; c < 8 && !read; c++) {
                        const int64_t fi = 2 * i - 1 + (c & 1), fj = 2 * j - 1 + (c >> 1 & 1), fk = 2 * k - 1 + (c >> 2);
                        if (fi < 0 || fj < 0 || fk < 0 || fi >= F.Nx || fj >= F.Ny || fk >= F.Nz) read = true;
                        else read = is_target[(size_t) (fi + F.Nx * fj + F.nxy() * fk)];
                    }
                }
        mg->r0_bc_dead[l] = !read;
    }
    *out = mg;
    return ARTSS_OK;
}

int artss_mg_destroy(artss_mg *mg) {
    if (!mg) return ARTSS_OK;
    for (auto &g : mg->graphs) cudaGraphExecDestroy(g.exec);
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

// kernel families a V-cycle launches: event profiling of any of them needs eager launches
constexpr uint64_t kMgFamilies = (1ull << FAM_FIELD_OP) | (1ull << FAM_BC) | (1ull << FAM_MG_JACOBI) |
                                 (1ull << FAM_MG_CGS) | (1ull << FAM_MG_RESIDUUM) | (1ull << FAM_MG_RESTRICT) |
                                 (1ull << FAM_MG_PROLONGATE) | (1ull << FAM_MG_COARSE) | (1ull << FAM_REDUCE);

// Captures set_rhs + n_cycle V-cycles for (p, rhs) into a graph of mg->graphs
// (at most 8 are kept; the oldest is dropped).
static int mg_capture(artss_mg *mg, double *p, const double *rhs) {
    artss_ctx *ctx = mg->ctx;
    const int64_t l0 = ctx->launches;
    int64_t f0[FAM_COUNT];
    for (int f = 0; f < FAM_COUNT; f++) f0[f] = ctx->prof.launches[f];
    ARTSS_CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    // VCycleMG::UpdateInput's copies are not needed: level 0 works on p and
    // reads rhs directly, and the smoother sets its scratch itself
    int st = ARTSS_OK;
    int64_t coarse = 0;
    for (int c = 0; c < mg->cfg.n_cycle && !st; c++) st = mg_vcycle(mg, p, &coarse, rhs);
    cudaGraph_t graph = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(ctx->stream, &graph);
    if (st) { if (graph) cudaGraphDestroy(graph); return st; }
    if (ec != cudaSuccess) return cuda_fail(ec, "V-cycle capture");
    artss_mg::Graph g{};
    g.p = p;
    g.rhs = rhs;
    const cudaError_t ei = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) return cuda_fail(ei, "V-cycle graph");
    // the capture only recorded the launches: count them per replay instead
    g.launches = ctx->launches - l0;
    ctx->launches = l0;
    for (int f = 0; f < FAM_COUNT; f++) {
        g.fam[f] = ctx->prof.launches[f] - f0[f];
        ctx->prof.launches[f] = f0[f];
    }
    if (mg->graphs.size() >= 8) {
        cudaGraphExecDestroy(mg->graphs.front().exec);
        mg->graphs.erase(mg->graphs.begin());
    }
    mg->graphs.push_back(g);
    return ARTSS_OK;
}

int artss_mg_pressure(artss_mg *mg, double *p, const double *rhs, int first_step, artss_mg_stats *stats) {
    if (mg && mg->ctx && mg->ctx->capturing && first_step) {
        set_error("the first-step pressure solve reads its residual on the host and cannot be captured");
        return ARTSS_ERR_ARG;
    }
    if (!mg || !p || !rhs) { set_error("null argument"); return ARTSS_ERR_ARG; }
    int st;
    int64_t cycles = 0, coarse = 0;
    double residual = -1.0;
    if (first_step) {
        if ((st = artss_mg_set_rhs(mg, p, rhs))) return st;
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
    } else if (mg->use_graphs && !(mg->ctx->prof.mask & kMgFamilies) && mg->fused_coarse && !mg->ctx->capturing) {
        // the later-step call is a fixed launch sequence: replay it as one graph
        artss_ctx *ctx = mg->ctx;
        artss_mg::Graph *g = nullptr;
        for (auto &e : mg->graphs)
            if (e.p == p && e.rhs == rhs) g = &e;
        if (!g) {
            if ((st = mg_capture(mg, p, rhs))) return st;
            g = &mg->graphs.back();
        }
        ARTSS_CK(cudaGraphLaunch(g->exec, ctx->stream));
        ctx->launches += g->launches;
        for (int f = 0; f < FAM_COUNT; f++) ctx->prof.launches[f] += g->fam[f];
        cycles = mg->cfg.n_cycle;
        coarse = -1;
    } else {
        for (int c = 0; c < mg->cfg.n_cycle; c++) {
            if ((st = mg_vcycle(mg, p, &coarse, rhs))) return st;
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

int artss_coarse_project(artss_ctx *ctx, double *d, int levels) {
    if (!ctx || !d) { set_error("null argument"); return ARTSS_ERR_ARG; }
    if (levels < 1 || levels > ctx->grid.n_levels) { set_error("levels out of range"); return ARTSS_ERR_ARG; }
    int st;
    double *arr[kMaxLevel + 1] = {d};
    for (int l = 1; l <= levels; l++) {
        if (!ctx->proj[l] && (st = artss_field_alloc(ctx, l, &ctx->proj[l]))) return st;
        arr[l] = ctx->proj[l];
    }
    // restrict: coarse inner cell = mean of its 8 children (VCycleMG::Restrict)
    for (int l = 1; l <= levels; l++) {
        const Level &C = ctx->lvl[l];
        const Box3 box = inner_box(C);
        if ((st = artss_fill(ctx, arr[l], l, 0.0))) return st;
        ARTSS_LAUNCH_PDL(ctx, FAM_MG_RESTRICT, k_mg_restrict, mg_grid(box), box_block(), 0, 
                                               arr[l], arr[l - 1], ctx->d_flags[l], C, ctx->lvl[l - 1], box);
        ARTSS_LAUNCH_CK(ctx);
    }
    // prolongate back (VCycleMG::Prolongate), the coarse level's boundary values first
    for (int l = levels; l >= 1; l--) {
        if ((st = apply_bc(ctx, arr[l], l, ARTSS_FIELD_P))) return st;
        if ((st = artss_fill(ctx, arr[l - 1], l - 1, 0.0))) return st;
        const Level &C = ctx->lvl[l];
        const Box3 box = inner_box(C);
        ARTSS_LAUNCH_PDL(ctx, FAM_MG_PROLONGATE, k_mg_prolongate, mg_grid(box), box_block(), 0, 
                                                 arr[l - 1], arr[l], ctx->d_flags[l], C, ctx->lvl[l - 1], box);
        ARTSS_LAUNCH_CK(ctx);
    }
    return ARTSS_OK;
}

int artss_mg_solve_rel(artss_mg *mg, double *p, const double *rhs, double rel_tol, int64_t max_cycles,
                       artss_solve_stats *stats) {
    if (!mg || !p || !rhs) { set_error("null argument"); return ARTSS_ERR_ARG; }
    if (max_cycles < 0 || !(rel_tol >= 0)) { set_error("invalid tolerance or cycle limit"); return ARTSS_ERR_ARG; }
    int st;
    if ((st = artss_mg_set_rhs(mg, p, rhs))) return st;
    double res = 0, b_norm = 0;
    if ((st = artss_residual_norm(mg->ctx, p, rhs, &res, &b_norm))) return st;
    const double tol = rel_tol * b_norm;
    int64_t cycles = 0, coarse = 0;
    const int slot = 2;
    while (res > tol && cycles < max_cycles) {
        if ((st = mg_vcycle(mg, p, &coarse))) return st;
        cycles++;
        if ((st = mg_resnorm(mg, p, rhs, 0, slot, -1.0, 1, false))) return st;
        LoopState ls{};
        if ((st = read_loop(mg->ctx, slot, &ls))) return st;
        res = ls.residual;
    }
    if (stats) {
        stats->cycles = cycles;
        stats->residual = res;
        stats->rel_residual = b_norm > 0 ? res / b_norm : res;
        stats->b_norm = b_norm;
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
