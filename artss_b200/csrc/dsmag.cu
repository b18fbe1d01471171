// DynamicSmagorinsky (src/turbulence/DynamicSmagorinsky.cpp:172-427): eddy
// viscosity of the dynamic Smagorinsky-Lilly model on level 0, FP64, with the
// reference's loops restated as passes over the inner cells:
//   1. u_f, v_f, w_f = explicit filter of u, v, w (trapezoidal 3x3x3 weights,
//      the sum over x offsets outermost and z offsets innermost, :384-427);
//   2. products of the filtered velocities (the reference's "velocity
//      products" are the filtered ones too), strain tensor S_ij of the filtered
//      velocities, |S| and P_ij = |S| S_ij (:200-282);
//   3. filters of the products (uu, vv, ww, uv, vw; the reference filters ww
//      twice and never uw, whose filter stays zero), of S_ij and of P_ij;
//   4. Leonard stress, M_ij and Cs = num / den with the reference's products
//      of the 22 and 33 terms in num and den (:298-344);
//   5. the 27-cell average of Cs in place in list order, so that a cell sees
//      the averaged values of every neighbour before it in the list, then
//      ev = 2 Cs delta_s^2 |S| and ev = 0 where ev + nu < 0 (:350-376).
// Step 5 is sequential in the reference.  Here it runs as one cooperative
// launch over hyperplanes t = i + 2j + 4k: every neighbour that precedes a
// cell in the list has a smaller t, every one that follows has a larger t and
// no two neighbours share a t, so updating Cs in place one hyperplane at a
// time (a grid barrier between hyperplanes) reads exactly what the sequential
// loop reads.  The work fields live in the context, zero outside the inner
// cells (the reference's fields start zero and only inner cells are written).
#include "internal.cuh"

#include <cmath>
#include <cooperative_groups.h>

namespace cg = cooperative_groups;

namespace artss {
namespace {

enum DsArr : int {
    UF, VF, WF, UU, VV, WW, UV, UW, VW, UUF, VVF, WWF, UVF, VWF,
    S11, S22, S33, S12, S13, S23, SBAR, P11, P22, P33, P12, P13, P23,
    S11F, S22F, S33F, S12F, S13F, S23F, P11F, P22F, P33F, P12F, P13F, P23F,
    CS, DS_ARRAYS
};

#define DS_COLUMN(box)                                                             \
    const int i = (int) (box).x0 + (int) (blockIdx.x * blockDim.x + threadIdx.x); \
    const int j = (int) (box).y0 + (int) (blockIdx.y * blockDim.y + threadIdx.y); \
    if (i > (int) (box).x1 || j > (int) (box).y1) return

inline dim3 ds_grid(const Box3 &b) {
    dim3 g = box_grid(b);
    const int64_t xy = (int64_t) g.x * g.y;
    int64_t gz = b.nz();
    const int64_t cap = std::max<int64_t>(1, 2048 / std::max<int64_t>(xy, 1));
    if (gz > cap) gz = cap;
    g.z = (unsigned) std::max<int64_t>(gz, 1);
    return g;
}

struct DsFilter {
    const double *in[12];
    double *out[12];
    int n;
};

// explicit_filtering of up to 12 fields: sum over l (x), m (y), n (z) of
// a[l] a[m] a[n] in[...], a = (1/4, 1/2, 1/4); the weight products are powers of
// two, so w * in is exact and only the order of the additions matters
__global__ void k_ds_filter(DsFilter f, const uint8_t *__restrict__ flags, Level L, Box3 box) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    DS_COLUMN(box);
    const int nj = (int) L.Nx, nk = (int) L.nxy();
    const double a[3] = {1. / 4., 1. / 2., 1. / 4.};
    for (int k = (int) box.z0 + (int) blockIdx.z; k <= (int) box.z1; k += (int) gridDim.z) {
        const int q = i + nj * j + nk * k;
        if (!(flags[q] & kInner)) continue;
        for (int fi = 0; fi < f.n; fi++) {
            const double *in = f.in[fi];
            double sum = 0;
#pragma unroll
            for (int l = 0; l < 3; l++)
#pragma unroll
                for (int m = 0; m < 3; m++)
#pragma unroll
                    for (int n = 0; n < 3; n++)
                        sum = sum + a[l] * a[m] * a[n] * in[q - 1 + l + nj * (m - 1) + nk * (n - 1)];
            f.out[fi][q] = sum;
        }
    }
}

// products of the filtered velocities, strain tensor, |S| and |S| S_ij
__global__ void k_ds_strain(double *__restrict__ A, const uint8_t *__restrict__ flags, Level L, Box3 box, int64_t N,
                            double rdx, double rdy, double rdz) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    DS_COLUMN(box);
    const int nj = (int) L.Nx, nk = (int) L.nxy();
    const double *uf = A + UF * N, *vf = A + VF * N, *wf = A + WF * N;
    for (int k = (int) box.z0 + (int) blockIdx.z; k <= (int) box.z1; k += (int) gridDim.z) {
        const int q = i + nj * j + nk * k;
        if (!(flags[q] & kInner)) continue;
        A[UU * N + q] = uf[q] * uf[q];
        A[VV * N + q] = vf[q] * vf[q];
        A[WW * N + q] = wf[q] * wf[q];
        A[UV * N + q] = uf[q] * vf[q];
        A[UW * N + q] = uf[q] * wf[q];
        A[VW * N + q] = vf[q] * wf[q];
        const double s11 = (uf[q + 1] - uf[q - 1]) * 0.5 * rdx;
        const double s22 = (vf[q + nj] - vf[q - nj]) * 0.5 * rdy;
        const double s33 = (wf[q + nk] - wf[q - nk]) * 0.5 * rdz;
        const double s12 = 0.5 * ((uf[q + nj] - uf[q - nj]) * 0.5 * rdy + (vf[q + 1] - vf[q - 1]) * 0.5 * rdx);
        const double s13 = 0.5 * ((uf[q + nk] - uf[q - nk]) * 0.5 * rdz + (wf[q + 1] - wf[q - 1]) * 0.5 * rdx);
        const double s23 = 0.5 * ((vf[q + nk] - vf[q - nk]) * 0.5 * rdz + (wf[q + nj] - wf[q - nj]) * 0.5 * rdy);
        const double sb = sqrt(2. * (s11 * s11 + s22 * s22 + s33 * s33 + 2. * (s12 * s12) + 2. * (s13 * s13) +
                                     2. * (s23 * s23)));
        A[S11 * N + q] = s11;
        A[S22 * N + q] = s22;
        A[S33 * N + q] = s33;
        A[S12 * N + q] = s12;
        A[S13 * N + q] = s13;
        A[S23 * N + q] = s23;
        A[SBAR * N + q] = sb;
        A[P11 * N + q] = sb * s11;
        A[P22 * N + q] = sb * s22;
        A[P33 * N + q] = sb * s33;
        A[P12 * N + q] = sb * s12;
        A[P13 * N + q] = sb * s13;
        A[P23 * N + q] = sb * s23;
    }
}

// Leonard stress, M_ij and the dynamic coefficient Cs = num / den
__global__ void k_ds_coefficient(double *__restrict__ A, const uint8_t *__restrict__ flags, Level L, Box3 box,
                                 int64_t N, double delta_s) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    DS_COLUMN(box);
    const int nj = (int) L.Nx, nk = (int) L.nxy();
    const double alpha = 2.0;
    for (int k = (int) box.z0 + (int) blockIdx.z; k <= (int) box.z1; k += (int) gridDim.z) {
        const int q = i + nj * j + nk * k;
        if (!(flags[q] & kInner)) continue;
        const double l11 = A[UUF * N + q] - A[UU * N + q];
        const double l22 = A[VVF * N + q] - A[VV * N + q];
        const double l33 = A[WWF * N + q] - A[WW * N + q];
        const double l12 = A[UVF * N + q] - A[UV * N + q];
        const double l13 = 0.0 - A[UW * N + q];  // the filter of uw is never formed: zero
        const double l23 = A[VWF * N + q] - A[VW * N + q];
        const double f11 = A[S11F * N + q], f22 = A[S22F * N + q], f33 = A[S33F * N + q];
        const double f12 = A[S12F * N + q], f13 = A[S13F * N + q], f23 = A[S23F * N + q];
        const double sbf = sqrt(2. * (f11 * f11 + f22 * f22 + f33 * f33 + 2. * (f12 * f12) + 2. * (f13 * f13) +
                                      2. * (f23 * f23)));
        const double m11 = 2.0 * delta_s * delta_s * (A[P11F * N + q] - alpha * alpha * sbf * f11);
        const double m22 = 2.0 * delta_s * delta_s * (A[P22F * N + q] - alpha * alpha * sbf * f22);
        const double m33 = 2.0 * delta_s * delta_s * (A[P33F * N + q] - alpha * alpha * sbf * f33);
        const double m12 = 2.0 * delta_s * delta_s * (A[P12F * N + q] - alpha * alpha * sbf * f12);
        const double m13 = 2.0 * delta_s * delta_s * (A[P13F * N + q] - alpha * alpha * sbf * f13);
        const double m23 = 2.0 * delta_s * delta_s * (A[P23F * N + q] - alpha * alpha * sbf * f23);
        const double num = l11 * m11 + l22 * m22 * l33 * m33 + 2.0 * l12 * m12 + 2.0 * l13 * m13 + 2.0 * l23 * m23;
        const double den = m11 * m11 + m22 * m22 * m33 * m33 + 2.0 * m12 * m12 + 2.0 * m13 * m13 + 2.0 * m23 * m23;
        A[CS * N + q] = num / den;
    }
}

// the in-place 27-cell average of Cs, hyperplane by hyperplane, and ev
__global__ void k_ds_average(double *__restrict__ Cs, double *__restrict__ ev, const double *__restrict__ sbar,
                             const uint8_t *__restrict__ flags, Level L, Box3 box, double delta_s, double nu) {
    cg::grid_group grid = cg::this_grid();
    const int nj = (int) L.Nx, nk = (int) L.nxy();
    const int x0 = (int) box.x0, x1 = (int) box.x1, y0 = (int) box.y0, z0 = (int) box.z0;
    const int ny = (int) box.ny(), nz = (int) box.nz();
    const int pairs = ny * nz;
    const int t0 = x0 + 2 * y0 + 4 * z0, t1 = x1 + 2 * (int) box.y1 + 4 * (int) box.z1;
    const int stride = (int) (gridDim.x * blockDim.x);
    const int first = (int) (blockIdx.x * blockDim.x + threadIdx.x);
    for (int t = t0; t <= t1; t++) {
        for (int p = first; p < pairs; p += stride) {
            const int j = y0 + p % ny, k = z0 + p / ny;
            const int i = t - 2 * j - 4 * k;
            if (i < x0 || i > x1) continue;
            const int q = i + nj * j + nk * k;
            if (!(flags[q] & kInner)) continue;
            double sum = 0;
#pragma unroll
            for (int l = 0; l < 3; l++)
#pragma unroll
                for (int m = 0; m < 3; m++)
#pragma unroll
                    for (int n = 0; n < 3; n++) sum = sum + Cs[q - 1 + l + nj * (m - 1) + nk * (n - 1)];
            const double c = sum / 27.0;
            Cs[q] = c;
            double e = 2.0 * c * delta_s * delta_s * sbar[q];
            if ((e + nu) < 0) e = 0;
            ev[q] = e;
        }
        grid.sync();
    }
}

}  // namespace
}  // namespace artss

using namespace artss;

extern "C" {

int artss_turb_dynamic_smagorinsky(artss_ctx *ctx, double *ev, const double *u, const double *v, const double *w,
                                   double nu) {
    if (!ctx || !ev || !u || !v || !w) { set_error("null argument"); return ARTSS_ERR_ARG; }
    const Level &L = ctx->lvl[0];
    const int64_t N = L.size();
    if (!ctx->dsmag || ctx->dsmag_version != ctx->geom_version) {
        if (ctx->capturing) {
            set_error("the dynamic Smagorinsky work fields are set up on an eager call; call it once before capturing");
            return ARTSS_ERR_ARG;
        }
        if (!ctx->dsmag) ARTSS_CK(cudaMalloc(&ctx->dsmag, (size_t) DS_ARRAYS * N * sizeof(double)));
        // zero outside the inner cells, also after the inner set changed
        ARTSS_CK(cudaMemsetAsync(ctx->dsmag, 0, (size_t) DS_ARRAYS * N * sizeof(double), ctx->stream));
        ctx->dsmag_version = ctx->geom_version;
    }
    double *A = ctx->dsmag;
    const Box3 box = inner_box(L);
    const artss_grid_desc &g = ctx->grid;
    const double dx = g.dx[0], dy = g.dy[0], dz = g.dz[0];
    const double rdx = 1. / dx, rdy = 1. / dy, rdz = 1. / dz;
    const double delta_s = cbrt(dx * dy * dz);
    const dim3 grid = ds_grid(box), block = box_block();
    const uint8_t *flags = ctx->d_flags[0];

    DsFilter f{};
    f.n = 3;
    f.in[0] = u; f.in[1] = v; f.in[2] = w;
    f.out[0] = A + UF * N; f.out[1] = A + VF * N; f.out[2] = A + WF * N;
    ARTSS_LAUNCH_PDL(ctx, FAM_SMAGORINSKY, k_ds_filter, grid, block, 0, f, flags, L, box);
    ARTSS_LAUNCH_CK(ctx);
    ARTSS_LAUNCH_PDL(ctx, FAM_SMAGORINSKY, k_ds_strain, grid, block, 0, A, flags, L, box, N, rdx, rdy, rdz);
    ARTSS_LAUNCH_CK(ctx);
    // filters of the products (uu, vv, ww, uv, vw), of S_ij and of |S| S_ij
    DsFilter g1{};
    const int src1[5] = {UU, VV, WW, UV, VW}, dst1[5] = {UUF, VVF, WWF, UVF, VWF};
    for (int a = 0; a < 5; a++) { g1.in[a] = A + src1[a] * N; g1.out[a] = A + dst1[a] * N; }
    g1.n = 5;
    ARTSS_LAUNCH_PDL(ctx, FAM_SMAGORINSKY, k_ds_filter, grid, block, 0, g1, flags, L, box);
    ARTSS_LAUNCH_CK(ctx);
    DsFilter g2{};
    for (int a = 0; a < 6; a++) {
        g2.in[a] = A + (S11 + a) * N; g2.out[a] = A + (S11F + a) * N;
        g2.in[6 + a] = A + (P11 + a) * N; g2.out[6 + a] = A + (P11F + a) * N;
    }
    g2.n = 12;
    ARTSS_LAUNCH_PDL(ctx, FAM_SMAGORINSKY, k_ds_filter, grid, block, 0, g2, flags, L, box);
    ARTSS_LAUNCH_CK(ctx);
    ARTSS_LAUNCH_PDL(ctx, FAM_SMAGORINSKY, k_ds_coefficient, grid, block, 0, A, flags, L, box, N, delta_s);
    ARTSS_LAUNCH_CK(ctx);
    // the averaging: one cooperative launch, every block resident
    static int blocks_per_sm = -1;
    const int threads = 256;
    if (blocks_per_sm < 0) {
        int nb = 0;
        ARTSS_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_ds_average, threads, 0));
        blocks_per_sm = std::max(1, std::min(nb, 4));
    }
    double *Cs = A + CS * N;
    const double *sb = A + SBAR * N;
    Level Lc = L;
    Box3 bc = box;
    double ds = delta_s, nuv = nu;
    void *args[] = {&Cs, &ev, (void *) &sb, (void *) &flags, &Lc, &bc, &ds, &nuv};
    cudaError_t err;
    ARTSS_LAUNCH(ctx, FAM_SMAGORINSKY,
                 err = cudaLaunchCooperativeKernel((const void *) k_ds_average,
                                                   dim3((unsigned) (blocks_per_sm * std::max(ctx->sm_count, 1))),
                                                   dim3(threads), args, 0, ctx->stream));
    if (err != cudaSuccess) return cuda_fail(err, "cooperative launch");
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

}  // extern "C"
