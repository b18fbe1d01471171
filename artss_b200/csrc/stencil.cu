// Level-0 plugin kernels: semi-Lagrangian advection, constant Smagorinsky,
// divergence / projection, buoyancy and explicit-Euler sources, and the
// colored Gauss-Seidel and Jacobi diffusion solvers.
//
// Iteration space: the reference loops over index lists (domain inner list,
// domain list).  Here every kernel sweeps the computational-domain box of the
// level in x-fastest order and tests the per-cell flags built from those same
// lists, so the set of cells and the per-cell arithmetic are identical while
// loads along x stay coalesced.  Threads own one (i, j) column and walk z in
// strides of gridDim.z.
#include "internal.cuh"

namespace artss {

// launch shape of box kernels: at most ~2048 blocks so that per-block partial
// sums of a reduction fit ctx->d_partials
inline dim3 zgrid(const Box3 &b) {
    dim3 g = box_grid(b);
    const int64_t xy = (int64_t) g.x * g.y;
    int64_t gz = b.nz();
    const int64_t cap = std::max<int64_t>(1, 2048 / std::max<int64_t>(xy, 1));
    if (gz > cap) gz = cap;
    g.z = (unsigned) std::max<int64_t>(gz, 1);
    return g;
}
inline int nblocks(const dim3 &g) { return (int) (g.x * g.y * g.z); }

// 32-bit cell indices: artss_ctx_create rejects levels of 2^31 cells or more
#define ARTSS_COLUMN(box)                                                                 \
    const int i = (int) (box).x0 + (int) (blockIdx.x * blockDim.x + threadIdx.x);        \
    const int j = (int) (box).y0 + (int) (blockIdx.y * blockDim.y + threadIdx.y);        \
    const bool col = (i <= (int) (box).x1) && (j <= (int) (box).y1)

__device__ __forceinline__ int block_linear() { return blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z); }

// ------------------------------------------------------------ advection

struct AdvCoef {
    double dtx, dty, dtz;                 // dt/dx, dt/dy, dt/dz (SLAdvect.cpp:53-55)
    int64_t is, ie, js, je, ks, ke;       // computational-domain inner index range
};

// Backtrace of SLAdvect.cpp:79-126 for one axis.
// fmod(x, 1.0) for x >= 0: x - trunc(x), the exact remainder fmod returns,
// without the general fmod
__device__ __forceinline__ double frac1(double x) { return x < 1.0 ? x : x - trunc(x); }

// 32-bit indices: the host runs the advection only on levels below 2^31 cells
__device__ __forceinline__ void sl_axis(double C, int c, int cs, int ce, int &c0, int &c1, double &r) {
    const double eps = 1e-6;
    c0 = c; c1 = c; r = 1.0;
    if (C > eps) {
        const int t = c - (int) C;
        c0 = t > cs ? t : cs;
        c1 = c0 - 1;
        r = frac1(C);
    } else if (C < -eps) {
        const int t = c - (int) C;
        c0 = t < ce ? t : ce;
        c1 = c0 + 1;
        r = frac1(-C);
    }
}

// Trilinear blend of SLAdvect.cpp:131-162, same operation order.
__device__ __forceinline__ double sl_interp(const double *__restrict__ in, int Nx, int nxy, int i0, int i1, int j0,
                                            int j1, int k0, int k1, double r, double s, double t) {
    const double d000 = in[i0 + Nx * j0 + nxy * k0];
    const double d100 = in[i1 + Nx * j0 + nxy * k0];
    const double d010 = in[i0 + Nx * j1 + nxy * k0];
    const double d110 = in[i1 + Nx * j1 + nxy * k0];
    const double d001 = in[i0 + Nx * j0 + nxy * k1];
    const double d101 = in[i1 + Nx * j0 + nxy * k1];
    const double d011 = in[i0 + Nx * j1 + nxy * k1];
    const double d111 = in[i1 + Nx * j1 + nxy * k1];
    const double r100 = d000 + r * (d100 - d000);
    const double r110 = d010 + r * (d110 - d010);
    const double r101 = d001 + r * (d101 - d001);
    const double r111 = d011 + r * (d111 - d011);
    const double s110 = r100 + s * (r110 - r100);
    const double s111 = r101 + s * (r111 - r101);
    return s110 + t * (s111 - s110);
}

template <int NF>
__global__ void k_advect(double *__restrict__ o0, double *__restrict__ o1, double *__restrict__ o2,
                         const double *__restrict__ n0, const double *__restrict__ n1, const double *__restrict__ n2,
                         const double *__restrict__ u, const double *__restrict__ v, const double *__restrict__ w,
                         const uint8_t *__restrict__ flags, Level L, Box3 box, AdvCoef c) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    ARTSS_COLUMN(box);
    if (!col) return;
    const int Nx = (int) L.Nx, nxy = (int) L.nxy();
    const int is = (int) c.is, ie = (int) c.ie, js = (int) c.js, je = (int) c.je, ks = (int) c.ks, ke = (int) c.ke;
    for (int k = (int) box.z0 + (int) blockIdx.z; k <= (int) box.z1; k += (int) gridDim.z) {
        const int idx = (int) i + Nx * (int) j + nxy * k;
        if (!(flags[idx] & kInner)) continue;
        int i0, i1, j0, j1, k0, k1;
        double r, s, t;
        sl_axis(c.dtx * u[idx], (int) i, is, ie, i0, i1, r);
        sl_axis(c.dty * v[idx], (int) j, js, je, j0, j1, s);
        sl_axis(c.dtz * w[idx], k, ks, ke, k0, k1, t);
        o0[idx] = sl_interp(n0, Nx, nxy, i0, i1, j0, j1, k0, k1, r, s, t);
        if (NF == 3) {
            o1[idx] = sl_interp(n1, Nx, nxy, i0, i1, j0, j1, k0, k1, r, s, t);
            o2[idx] = sl_interp(n2, Nx, nxy, i0, i1, j0, j1, k0, k1, r, s, t);
        }
    }
}

// ------------------------------------------------------------ turbulence

// ConstSmagorinsky.cpp:60-80; cs2d2 = Cs * Cs * delta_s * delta_s (host).
__global__ void k_smagorinsky(double *__restrict__ ev, const double *__restrict__ u, const double *__restrict__ v,
                              const double *__restrict__ w, const uint8_t *__restrict__ flags, Level L, Box3 box,
                              double rdx, double rdy, double rdz, double cs2d2) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    ARTSS_COLUMN(box);
    if (!col) return;
    const int ni = 1, nj = (int) L.Nx, nk = (int) L.nxy();
    column_planes<2>(i + nj * j, nk, (int) box.z0, (int) box.z1, flags,
        [&](int q, int) {
            const double S11 = (u[q + ni] - u[q - ni]) * 0.5 * rdx;
            const double S22 = (v[q + nj] - v[q - nj]) * 0.5 * rdy;
            const double S33 = (w[q + nk] - w[q - nk]) * 0.5 * rdz;
            const double S12 = 0.5 * ((u[q + nj] - u[q - nj]) * 0.5 * rdy + (v[q + ni] - v[q - ni]) * 0.5 * rdx);
            const double S13 = 0.5 * ((u[q + nk] - u[q - nk]) * 0.5 * rdz + (w[q + ni] - w[q - ni]) * 0.5 * rdx);
            const double S23 = 0.5 * ((v[q + nk] - v[q - nk]) * 0.5 * rdz + (w[q + nj] - w[q - nj]) * 0.5 * rdy);
            const double S_bar = sqrt(2. * (S11 * S11 + S22 * S22 + S33 * S33
                                            + 2. * (S12 * S12) + 2. * (S13 * S13) + 2. * (S23 * S23)));
            return cs2d2 * S_bar;
        },
        [&](int q, int, double v_, uint8_t) { ev[q] = v_; });
}

// ExplicitDiffuse::ExplicitStep: laminar (ExplicitDiffuse.cpp:50-76, rd* = D / (d* d*)
// on the host) and turbulent (:79-124: face viscosities 0.5 (EV_nb + EV) + D, no
// division by the spacing, as the reference writes it); inner cells, same order
template <bool TURB>
__global__ void k_explicit_diffuse(double *__restrict__ out, const double *__restrict__ in,
                                   const double *__restrict__ ev, const uint8_t *__restrict__ flags, Level L, Box3 box,
                                   double D, double dt, double rdx, double rdy, double rdz) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    ARTSS_COLUMN(box);
    if (!col) return;
    const int ni = 1, nj = (int) L.Nx, nk = (int) L.nxy();
    for (int k = (int) box.z0 + (int) blockIdx.z; k <= (int) box.z1; k += (int) gridDim.z) {
        const int q = i + nj * j + nk * k;
        if (!(flags[q] & kInner)) continue;
        if (!TURB) {
            out[q] = in[q] + dt * ((in[q + ni] - 2 * in[q] + in[q - ni]) * rdx + (in[q + nj] - 2 * in[q] + in[q - nj]) * rdy +
                                   (in[q + nk] - 2 * in[q] + in[q - nk]) * rdz);
        } else {
            const double e0 = ev[q];
            const double nu_x1 = 0.5 * (ev[q + ni] + e0) + D, nu_x2 = 0.5 * (ev[q - ni] + e0) + D;
            const double nu_y1 = 0.5 * (ev[q + nj] + e0) + D, nu_y2 = 0.5 * (ev[q - nj] + e0) + D;
            const double nu_z1 = 0.5 * (ev[q + nk] + e0) + D, nu_z2 = 0.5 * (ev[q - nk] + e0) + D;
            const double c = in[q];
            const double di0 = c - in[q - ni], di1 = in[q + ni] - c;
            const double dj0 = c - in[q - nj], dj1 = in[q + nj] - c;
            const double dk0 = c - in[q - nk], dk1 = in[q + nk] - c;
            out[q] = c + dt * ((nu_x1 * di0 - nu_x2 * di1) + (nu_y1 * dj0 - nu_y2 * dj1) + (nu_z1 * dk0 - nu_z2 * dk1));
        }
    }
}

// ISource::dissipate (ISource.cpp:94-114): out += dt * nu * Phi on inner cells;
// h* = 0.5 * (1 / d*) on the host (the reference's 0.5 * reciprocal_d*, the same
// product), every sub-expression evaluated as the reference writes it
__global__ void k_dissipate(double *__restrict__ out, const double *__restrict__ u, const double *__restrict__ v,
                            const double *__restrict__ w, const uint8_t *__restrict__ flags, Level L, Box3 box,
                            double nu, double dt, double hx, double hy, double hz) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    ARTSS_COLUMN(box);
    if (!col) return;
    const int ni = 1, nj = (int) L.Nx, nk = (int) L.nxy();
    for (int k = (int) box.z0 + (int) blockIdx.z; k <= (int) box.z1; k += (int) gridDim.z) {
        const int q = i + nj * j + nk * k;
        if (!(flags[q] & kInner)) continue;
        const double ux = hx * (u[q + ni] - u[q - ni]), vy = hy * (v[q + nj] - v[q - nj]);
        const double wz = hz * (w[q + nk] - w[q - nk]);
        const double s12 = hx * (v[q + ni] - v[q - ni]) + hy * (u[q + nj] - u[q - nj]);
        const double s23 = hy * (w[q + nj] - w[q - nj]) + hz * (v[q + nk] - v[q - nk]);
        const double s31 = hz * (u[q + nk] - u[q - nk]) + hx * (w[q + ni] - w[q - ni]);
        const double out_h = nu * (2 * ux * ux + 2 * vy * vy + 2 * wz * wz + s12 * s12 + s23 * s23 + s31 * s31);
        out[q] += dt * out_h;
    }
}

// Analysis::calc_CFL (Analysis.cpp:322-351): per block the largest
// |u|/dx + |v|/dy + |w|/dz over inner cells; a maximum is exact in any order
__global__ void k_cfl_max(const double *__restrict__ u, const double *__restrict__ v, const double *__restrict__ w,
                          const uint8_t *__restrict__ flags, Level L, Box3 box, double dx, double dy, double dz,
                          double *__restrict__ partials) {
    __shared__ double sm[32];
    double m = 0.0;  // C >= 0
    const int i = (int) box.x0 + (int) (blockIdx.x * blockDim.x + threadIdx.x);
    const int j = (int) box.y0 + (int) (blockIdx.y * blockDim.y + threadIdx.y);
    if (i <= (int) box.x1 && j <= (int) box.y1) {
        const int nj = (int) L.Nx, nk = (int) L.nxy();
        for (int k = (int) box.z0 + (int) blockIdx.z; k <= (int) box.z1; k += (int) gridDim.z) {
            const int q = i + nj * j + nk * k;
            if (!(flags[q] & kInner)) continue;
            m = fmax(m, fabs(u[q]) / dx + fabs(v[q]) / dy + fabs(w[q]) / dz);
        }
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    const int tid = threadIdx.x + blockDim.x * threadIdx.y, lane = tid & 31, wid = tid >> 5;
    if (lane == 0) sm[wid] = m;
    __syncthreads();
    if (wid == 0) {
        const int nw = (blockDim.x * blockDim.y + 31) >> 5;
        m = lane < nw ? sm[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
        if (lane == 0) partials[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = m;
    }
}

// ------------------------------------------------------------ pressure coupling

// IPressure.cpp:58-66; h* = 0.5 * (1/d*) (host)
__global__ void k_divergence(double *__restrict__ out, const double *__restrict__ u, const double *__restrict__ v,
                             const double *__restrict__ w, const uint8_t *__restrict__ flags, Level L, Box3 box,
                             double hx, double hy, double hz) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    ARTSS_COLUMN(box);
    if (!col) return;
    const int nj = (int) L.Nx, nk = (int) L.nxy();
    column_planes(i + nj * j, nk, (int) box.z0, (int) box.z1, flags,
        [&](int q, int) {
            const double a = hx * (u[q + 1] - u[q - 1]);
            const double b = hy * (v[q + nj] - v[q - nj]);
            const double c = hz * (w[q + nk] - w[q - nk]);
            return a + b + c;
        },
        [&](int q, int, double v_, uint8_t) { out[q] = v_; });
}

// zero the ghost ring of the computational domain (IPressure.cpp:69-104)
__global__ void k_ghost_ring_zero(double *__restrict__ out, Level L, Box3 ring) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    ARTSS_COLUMN(ring);
    if (!col) return;
    for (int k = (int) ring.z0 + (int) blockIdx.z; k <= (int) ring.z1; k += (int) gridDim.z) {
        if (i == ring.x0 || i == ring.x1 || j == ring.y0 || j == ring.y1 || k == ring.z0 || k == ring.z1)
            out[i + (int) L.Nx * j + (int) L.nxy() * k] = 0.0;
    }
}

// IPressure.cpp:154-161
__global__ void k_projection(double *__restrict__ ou, double *__restrict__ ov, double *__restrict__ ow,
                             const double *__restrict__ us, const double *__restrict__ vs,
                             const double *__restrict__ ws, const double *__restrict__ p,
                             const uint8_t *__restrict__ flags, Level L, Box3 box, double hx, double hy, double hz) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    ARTSS_COLUMN(box);
    if (!col) return;
    const int nj = (int) L.Nx, nk = (int) L.nxy();
    struct UVW { double u, v, w; };
    column_planes<2>(i + nj * j, nk, (int) box.z0, (int) box.z1, flags,
        [&](int q, int) {
            return UVW{us[q] - hx * (p[q + 1] - p[q - 1]), vs[q] - hy * (p[q + nj] - p[q - nj]),
                       ws[q] - hz * (p[q + nk] - p[q - nk])};
        },
        [&](int q, int, UVW r, uint8_t) {
            ou[q] = r.u;
            ov[q] = r.v;
            ow[q] = r.w;
        });
}

// ------------------------------------------------------------ sources

// ISource.cpp:41-46 on the domain list; nbeta = -beta (host)
__global__ void k_buoyancy(double *__restrict__ f, const double *__restrict__ T, const double *__restrict__ Ta,
                           const uint8_t *__restrict__ flags, Level L, Box3 box, double nbeta, double g) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    ARTSS_COLUMN(box);
    if (!col) return;
    column_planes(i + (int) L.Nx * j, (int) L.nxy(), (int) box.z0, (int) box.z1, flags,
        [&](int q, int) { return nbeta * (T[q] - Ta[q]) * g; },
        [&](int q, int, double v_, uint8_t) { f[q] = v_; }, kDomain);
}

// ExplicitEulerSource.cpp:92-96
__global__ void k_add_source(double *__restrict__ out, const double *__restrict__ S,
                             const uint8_t *__restrict__ flags, Level L, Box3 box, double dt) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    ARTSS_COLUMN(box);
    if (!col) return;
    column_planes(i + (int) L.Nx * j, (int) L.nxy(), (int) box.z0, (int) box.z1, flags,
        [&](int q, int) { return out[q] + dt * S[q]; },
        [&](int q, int, double v_, uint8_t) { out[q] = v_; });
}

// ------------------------------------------------------------ diffusion

struct DiffCoef {
    double ax, ay, az;         // laminar alphas  D*dt/dx^2 ... (ColoredGaussSeidelDiffuse.cpp:58-60)
    double beta;               // 1/(1 + 2 sum alpha)
    double rbeta;              // 1 + 2 sum alpha
    double dsign, w, omw;      // sign of b, relaxation weight, (1 - w)
    double D, dt, rdx, rdy, rdz;  // turbulent variant: alphas from D + EV per cell
};

// alpha / beta of the turbulent variant (ColoredGaussSeidelDiffuse.cpp:273-278)
__device__ __forceinline__ void turb_alpha(const DiffCoef &c, double ev, double &ax, double &ay, double &az,
                                           double &rb) {
    ax = (c.D + ev) * c.dt * c.rdx * c.rdx;
    ay = (c.D + ev) * c.dt * c.rdy * c.rdy;
    az = (c.D + ev) * c.dt * c.rdz * c.rdz;
    rb = (1. + 2. * (ax + ay + az));
}

// One colored Gauss-Seidel iteration, red then black (stencil at
// ColoredGaussSeidelDiffuse.cpp:316-341, sweep order :190-295), in ONE pass
// over the arrays, out of place: `in` holds iterate n (never written), `out`
// receives iterate n+1 on the inner box; also writes the block partial of
// sum (rbeta * (new - old))^2 over both colours, the convergence measure of
// ColoredGaussSeidelDiffuse.cpp:77-85.  The values equal the in-place
// two-colour sweep: red cells read only black neighbours (old), black cells
// read only red neighbours (new).
//
// A block owns a tile of kSwTx x kSwTy columns over kSwZ planes and marches
// up in z.  At plane step k it computes red on plane k for the tile plus a
// one-cell ring (the ring's red values feed the tile's black cells; they are
// recomputed, never written), then black on plane k-1 for the tile, and
// writes plane k-1 of the tile to `out`.  Planes of `in`, `b` and `EV` (tile
// plus a two-cell ring) stream through shared-memory ring buffers by
// cp.async, kSwD planes ahead of use; a tile's red values replace the old
// ones in the `in` plane buffer, since only black cells read them afterwards.
// Non-inner cells of the tile are copied from `in`; the boundary program
// rewrites the ones anything reads.
constexpr int kSwTx = 64, kSwTy = 8, kSwZ = 16, kSwD = 2;
constexpr int kSwThreads = (kSwTx / 2) * kSwTy;            // one thread per x-pair of the tile
constexpr int kSwWx = kSwTx + 4, kSwWy = kSwTy + 4;         // staged window: tile + 2-cell ring
constexpr int kSwPlane = kSwWx * kSwWy;
constexpr int kSwSlotsX = kSwD + 4;                         // x planes k-2 .. k+1+D
constexpr int kSwSlotsB = kSwD + 3;                         // b / EV planes k-1 .. k+1+D
constexpr int kSwRedPairs = ((kSwTx + 2) / 2) * (kSwTy + 2);  // x-pairs of the tile + 1-cell ring

inline dim3 sweep_grid(const Box3 &b) {
    return dim3((unsigned) ((b.nx() + kSwTx - 1) / kSwTx), (unsigned) ((b.ny() + kSwTy - 1) / kSwTy),
                (unsigned) ((b.nz() + kSwZ - 1) / kSwZ));
}
inline size_t sweep_smem(bool turb) {
    return sizeof(double) * (size_t) kSwPlane * (kSwSlotsX + (turb ? 2 : 1) * kSwSlotsB);
}

__device__ __forceinline__ void cp_async8(double *dst, const double *src) {
    const unsigned d = (unsigned) __cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <bool TURB>
__global__ void __launch_bounds__(kSwThreads, 2)
k_cgs_sweep(double *__restrict__ out, const double *__restrict__ in, const double *__restrict__ b,
            const double *__restrict__ ev, const uint8_t *__restrict__ flags, Level L, Box3 box, DiffCoef c,
            double *__restrict__ partials, const LoopState *__restrict__ pred) {
    extern __shared__ double sw[];
    __shared__ double smem[32];
    if (pred && !pred->cond) return;  // iteration enqueued past convergence
    if (blockDim.x != kSwTx / 2 || blockDim.y != kSwTy || blockDim.z != 1) return;  // launch shape is fixed
    double *X = sw;                                  // [kSwSlotsX][kSwPlane]
    double *B = sw + kSwSlotsX * kSwPlane;           // [kSwSlotsB][kSwPlane]
    double *E = B + kSwSlotsB * kSwPlane;            // [kSwSlotsB][kSwPlane] (TURB)
    const int tid = threadIdx.x + (kSwTx / 2) * threadIdx.y;
    const int64_t nj = L.Nx, nk = L.nxy();
    const int64_t wx0 = box.x0 + (int64_t) blockIdx.x * kSwTx - 2;  // global i of window column 0
    const int64_t wy0 = box.y0 + (int64_t) blockIdx.y * kSwTy - 2;
    const int64_t kc0 = box.z0 + (int64_t) blockIdx.z * kSwZ;
    const int64_t kc1 = min(kc0 + kSwZ - 1, box.z1);

    // stage plane p of x, b (and EV) into their ring slots; one commit group per plane
    auto stage = [&](int64_t p) {
        // planes kc0-2 .. kc1+2 are read; the ring is kept in step past them
        if (p >= 0 && p < L.Nz && p <= kc1 + 2) {
            double *xs = X + (int) ((p - kc0 + 2 + 2 * kSwSlotsX) % kSwSlotsX) * kSwPlane;
            double *bs = B + (int) ((p - kc0 + 2 + 2 * kSwSlotsB) % kSwSlotsB) * kSwPlane;
            double *es = E + (int) ((p - kc0 + 2 + 2 * kSwSlotsB) % kSwSlotsB) * kSwPlane;
            for (int e = tid; e < kSwPlane; e += kSwThreads) {
                const int ly = e / kSwWx, lx = e - ly * kSwWx;
                const int64_t gi = wx0 + lx, gj = wy0 + ly;
                if (gi < 0 || gi >= L.Nx || gj < 0 || gj >= L.Ny) continue;
                const int64_t q = gi + nj * gj + nk * p;
                cp_async8(xs + e, in + q);
                // b and EV are read on the tile and its 1-cell ring only
                if (lx >= 1 && lx <= kSwTx + 2 && ly >= 1 && ly <= kSwTy + 2) {
                    cp_async8(bs + e, b + q);
                    if (TURB) cp_async8(es + e, ev + q);
                }
            }
        }
        cp_async_commit();
    };
    auto xslot = [&](int64_t p) { return X + ((unsigned) (p - kc0 + 2) % (unsigned) kSwSlotsX) * kSwPlane; };
    auto bslot = [&](int64_t p) { return (int) (((unsigned) (p - kc0 + 2) % (unsigned) kSwSlotsB) * kSwPlane); };

    // one stencil update; returns the new value and the residual term
    auto update = [&](const double *xm, const double *x0, const double *xp, int e, int bo, double &res2) {
        double ax = c.ax, ay = c.ay, az = c.az, beta = c.beta, rb = c.rbeta;
        if (TURB) {
            turb_alpha(c, E[bo + e], ax, ay, az, rb);
            beta = 1. / rb;
        }
        const double old = x0[e];
        const double out_h = beta * (c.dsign * B[bo + e] + ax * (x0[e + 1] + x0[e - 1]) +
                                     ay * (x0[e + kSwWx] + x0[e - kSwWx]) + az * (xp[e] + xm[e]));
        const double nw = c.omw * old + c.w * out_h;
        const double r = rb * (nw - old);
        res2 = r * r;
        return nw;
    };

    for (int64_t p = kc0 - 2; p <= kc0 - 1 + kSwD; p++) stage(p);
    double acc = 0.0;
    for (int64_t k = kc0 - 1; k <= kc1 + 1; k++) {
        cp_async_wait<kSwD - 1>();  // planes up to k+1 have landed
        __syncthreads();            // ... and step k-1 is done with the slots refilled next
        stage(k + 1 + kSwD);
        // red on plane k, tile + 1-cell ring
        if (k >= box.z0 && k <= box.z1) {
            const double *xm = xslot(k - 1), *xp = xslot(k + 1);
            double *x0 = xslot(k);
            const int bo = bslot(k);
            for (int pr = tid; pr < kSwRedPairs; pr += kSwThreads) {
                const int ry = 1 + pr / ((kSwTx + 2) / 2);
                const int px = pr - (ry - 1) * ((kSwTx + 2) / 2);
                const int64_t gj = wy0 + ry;
                const int rx = 1 + 2 * px + (int) ((wx0 + 1 + gj + k) & 1);  // (i + j + k) even
                const int64_t gi = wx0 + rx;
                if (gi < box.x0 || gi > box.x1 || gj < box.y0 || gj > box.y1) continue;
                if (!(__ldg(flags + gi + nj * gj + nk * k) & kInner)) continue;
                const int e = rx + kSwWx * ry;
                double r2;
                const double nw = update(xm, x0, xp, e, bo, r2);
                x0[e] = nw;
                if (rx >= 2 && rx < kSwTx + 2 && ry >= 2 && ry < kSwTy + 2 && k >= kc0 && k <= kc1) acc += r2;
            }
        }
        __syncthreads();
        // black on plane k-1, tile only, and the tile's plane k-1 out
        const int64_t kb = k - 1;
        if (kb >= kc0 && kb <= kc1) {
            const double *xm = xslot(kb - 1), *xp = xslot(kb + 1);
            const double *x0 = xslot(kb);
            const int bo = bslot(kb);
            const int ty = threadIdx.y, tx = threadIdx.x;
            const int64_t gj = wy0 + 2 + ty;
            const int lx0 = 2 + 2 * tx;
            const int par = (int) ((wx0 + lx0 + gj + kb + 1) & 1);  // (i + j + k) odd
            const int e0 = lx0 + kSwWx * (2 + ty);
            if (gj <= box.y1) {
#pragma unroll
                for (int s = 0; s < 2; s++) {
                    const int64_t gi = wx0 + lx0 + s;
                    if (gi > box.x1) continue;
                    const int64_t q = gi + nj * gj + nk * kb;
                    double v = x0[e0 + s];
                    if (s == par && (__ldg(flags + q) & kInner)) {
                        double r2;
                        v = update(xm, x0, xp, e0 + s, bo, r2);
                        acc += r2;
                    }
                    out[q] = v;
                }
            }
        }
    }
    cp_async_wait<0>();
    acc = artss_block_sum(acc, smem);
    if (partials && tid == 0) partials[block_linear()] = acc;
}

// ---- the same sweep with TMA plane staging -------------------------------
//
// One thread issues, per z-plane, one cp.async.bulk.tensor load of the
// kTmaBoxX x kTmaBoxY window of x, b (and EV) into the plane's ring slot;
// the loads complete on the slot's mbarrier.  The window starts at an even x
// (a TMA box must start on a 16-byte boundary), so the tile sits ox = 0 or 1
// cells further right in it than in the cp.async variant.  Red work is one
// x-pair per thread (33 x 10 pairs: tile plus ring), black one x-pair per
// thread of the first 256.  Waits on an mbarrier give up after a bounded
// number of polls and raise the loop state's error flag instead of hanging.
constexpr int kStThreads = ((kSwTx + 2) / 2) * (kSwTy + 2);  // 330 red pairs
constexpr int kStPlane = kTmaBoxX * kTmaBoxY;                 // doubles per slot
constexpr int kStSlotsX = kSwD + 4, kStSlotsB = kSwD + 3;
constexpr unsigned kStPlaneBytes = kStPlane * sizeof(double);
static_assert(kTmaBoxX >= kSwTx + 5 && kTmaBoxY == kSwTy + 4, "TMA window covers tile + ring + alignment");
static_assert(kStPlaneBytes % 128 == 0, "slots stay 128-byte aligned");

// z-planes per block of the TMA sweep: the autotuned choice among these
constexpr int kStDepths[3] = {8, 16, 32};
inline dim3 sweep_tma_grid(const Box3 &b, int zb) {
    return dim3((unsigned) ((b.nx() + kSwTx - 1) / kSwTx), (unsigned) ((b.ny() + kSwTy - 1) / kSwTy),
                (unsigned) ((b.nz() + zb - 1) / zb));
}

inline size_t sweep_tma_smem(bool turb) {
    return (size_t) kStPlaneBytes * (kStSlotsX + (turb ? 2 : 1) * kStSlotsB);
}

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned) __cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// true once the phase with the given parity has completed; gives up after `polls` tries
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, int polls) {
    for (int n = 0; n < polls; n++) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
__device__ __forceinline__ void tma_load_plane(double *dst, const CUtensorMap *map, int x, int y, int z,
                                               uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];\n" ::"r"(smem_u32(dst)),
        "l"((uint64_t) map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

constexpr int kStPolls = 1 << 22;  // mbarrier polls before a wait gives up

template <bool TURB, int ZB>
__global__ void __launch_bounds__(kStThreads, 2)
k_cgs_sweep_tma(const __grid_constant__ CUtensorMap tm_x, const __grid_constant__ CUtensorMap tm_b,
                const __grid_constant__ CUtensorMap tm_e, double *__restrict__ out,
                const uint8_t *__restrict__ flags, Level L, Box3 box, DiffCoef c, double *__restrict__ partials,
                LoopState *__restrict__ pred) {
    extern __shared__ __align__(1024) double st_sm[];
    __shared__ double smem[32];
    __shared__ __align__(8) uint64_t bars[kStSlotsX];
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    if (pred && !pred->cond) return;  // iteration enqueued past convergence
    if (blockDim.x != kStThreads || blockDim.y != 1 || blockDim.z != 1) return;  // launch shape is fixed
    double *X = st_sm;                          // [kStSlotsX][kStPlane]
    double *B = st_sm + kStSlotsX * kStPlane;   // [kStSlotsB][kStPlane]
    double *E = B + kStSlotsB * kStPlane;       // [kStSlotsB][kStPlane] (TURB)
    const int tid = threadIdx.x;
    // 32-bit indices: the host takes this kernel only for levels of fewer than 2^31 cells
    const int nj = (int) L.Nx, nk = (int) L.nxy();
    const int bx0 = (int) box.x0, bx1 = (int) box.x1, by0 = (int) box.y0, by1 = (int) box.y1;
    const int bz0 = (int) box.z0, bz1 = (int) box.z1;
    const int wx0 = bx0 + (int) blockIdx.x * kSwTx - 2;  // global i of ring column 0
    const int wxa = wx0 - (wx0 & 1);                      // TMA window start, even
    const int ox = wx0 - wxa;
    const int wy0 = by0 + (int) blockIdx.y * kSwTy - 2;
    const int kc0 = bz0 + (int) blockIdx.z * ZB;
    const int kc1 = min(kc0 + ZB - 1, bz1);
    const int pbase = kc0 - 2, plast = kc1 + 2;  // staged planes

    if (tid == 0) {
        for (int s = 0; s < kStSlotsX; s++) mbar_init(&bars[s], 1);
        fence_proxy_async();
    }
    __syncthreads();
    // thread 0: load plane p into its slots
    auto issue = [&](int p) {
        if (p > plast) return;
        const unsigned u = (unsigned) (p - pbase);
        uint64_t *bar = &bars[u % kStSlotsX];
        mbar_expect_tx(bar, kStPlaneBytes * (TURB ? 3u : 2u));
        tma_load_plane(X + (u % kStSlotsX) * kStPlane, &tm_x, wxa, wy0, p, bar);
        tma_load_plane(B + (u % kStSlotsB) * kStPlane, &tm_b, wxa, wy0, p, bar);
        if (TURB) tma_load_plane(E + (u % kStSlotsB) * kStPlane, &tm_e, wxa, wy0, p, bar);
    };
    auto ready = [&](int p) -> bool {
        const unsigned u = (unsigned) (p - pbase);
        return mbar_wait(&bars[u % kStSlotsX], (u / kStSlotsX) & 1u, kStPolls);
    };
    // ring slots by local plane number (32-bit, constant divisors)
    auto xslot = [&](int p) { return X + ((unsigned) (p - pbase) % (unsigned) kStSlotsX) * kStPlane; };
    auto bslot = [&](int p) { return (int) (((unsigned) (p - pbase) % (unsigned) kStSlotsB) * kStPlane); };
    auto update = [&](const double *xm, const double *x0, const double *xp, int e, int bo, double &res2) {
        double ax = c.ax, ay = c.ay, az = c.az, beta = c.beta, rb = c.rbeta;
        if (TURB) {
            turb_alpha(c, E[bo + e], ax, ay, az, rb);
            beta = 1. / rb;
        }
        const double old = x0[e];
        const double out_h = beta * (c.dsign * B[bo + e] + ax * (x0[e + 1] + x0[e - 1]) +
                                     ay * (x0[e + kTmaBoxX] + x0[e - kTmaBoxX]) + az * (xp[e] + xm[e]));
        const double nw = c.omw * old + c.w * out_h;
        const double r = rb * (nw - old);
        res2 = r * r;
        return nw;
    };

    // this thread's red x-pair (tile + ring) and black x-pair (tile)
    const int ry = 1 + tid / ((kSwTx + 2) / 2), px = tid % ((kSwTx + 2) / 2);
    const int gjr = wy0 + ry;
    const bool red_row_ok = gjr >= by0 && gjr <= by1;
    const int red_row = nj * gjr;
    const bool red_tile = ry >= 2 && ry < kSwTy + 2;
    const bool has_black = tid < (kSwTx / 2) * kSwTy;
    const int tx = tid % (kSwTx / 2), ty = tid / (kSwTx / 2);
    const int gjb = wy0 + 2 + ty;
    const int black_row = nj * gjb;
    const int lx0 = 2 + 2 * tx;
    auto red_x = [&](int k) { return 1 + 2 * px + ((wx0 + 1 + gjr + k) & 1); };  // (i + j + k) even
    auto red_flag = [&](int k) -> uint8_t {
        if (!red_row_ok || k < bz0 || k > bz1) return 0;
        const int gi = wx0 + red_x(k);
        if (gi < bx0 || gi > bx1) return 0;
        return __ldg(flags + gi + red_row + nk * k);
    };
    auto black_par = [&](int kb) { return (wx0 + lx0 + gjb + kb + 1) & 1; };  // (i + j + k) odd
    auto black_flag = [&](int kb) -> uint8_t {
        if (!has_black || gjb > by1 || kb < kc0 || kb > kc1) return 0;
        const int gi = wx0 + lx0 + black_par(kb);
        if (gi > bx1) return 0;
        return __ldg(flags + gi + black_row + nk * kb);
    };

    double acc = 0.0;
    int issued = kc0 - 1 + kSwD;  // thread 0's last issued plane
    if (tid == 0)
        for (int p = pbase; p <= issued; p++) issue(p);
    bool ok = tid != 0 || (ready(pbase) && ready(pbase + 1));
    uint8_t fr = red_flag(kc0 - 1), fb = black_flag(kc0 - 2);
    bool failed = false;
    int waited = pbase + 1;  // planes up to here have landed
    for (int k = kc0 - 1; k <= kc1 + 1; k++) {
        // the next step's flags, loaded early
        const uint8_t fr_next = red_flag(k + 1), fb_next = black_flag(k);
        // thread 0 waits for plane k+1; the barrier below publishes it to the block
        if (tid == 0) ok = ok && ready(k + 1);
        fence_proxy_async();  // this thread's shared-memory writes before the slot refill below
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        waited = k + 1;
        if (tid == 0 && k + 1 + kSwD <= plast) {
            issue(k + 1 + kSwD);
            issued = k + 1 + kSwD;
        }
        // red on plane k, tile + 1-cell ring
        if (fr & kInner) {
            const int rx = red_x(k);
            const int e = rx + ox + kTmaBoxX * ry;
            double *x0 = xslot(k);
            double r2;
            const double nw = update(xslot(k - 1), x0, xslot(k + 1), e, bslot(k), r2);
            x0[e] = nw;
            if (red_tile && rx >= 2 && rx < kSwTx + 2 && k >= kc0 && k <= kc1) acc += r2;
        }
        __syncthreads();
        // black on plane k-1, tile only, and the tile's plane k-1 out
        const int kb = k - 1;
        if (has_black && kb >= kc0 && kb <= kc1 && gjb <= by1) {
            const double *x0 = xslot(kb);
            const int par = black_par(kb);
            const int e0 = lx0 + ox + kTmaBoxX * (2 + ty);
#pragma unroll
            for (int s = 0; s < 2; s++) {
                const int gi = wx0 + lx0 + s;
                if (gi > bx1) continue;
                double v = x0[e0 + s];
                if (s == par && (fb & kInner)) {
                    double r2;
                    v = update(xslot(kb - 1), x0, xslot(kb + 1), e0 + s, bslot(kb), r2);
                    acc += r2;
                }
                out[gi + black_row + nk * kb] = v;
            }
        }
        fr = fr_next;
        fb = fb_next;
    }
    if (failed) {
        // a plane never arrived: flag it, let the loads in flight land, leave
        if (tid == 0) {
            if (pred) *(volatile int *) &pred->pad = 1;
            for (int p = waited + 1; p <= issued; p++) (void) ready(p);
        }
        __syncthreads();
        return;
    }
    acc = artss_block_sum(acc, smem);
    if (partials && tid == 0) partials[block_linear()] = acc;
}

// ---- the sweep with red and black in one phase ------------------------------
//
// The same iteration with black two planes behind red: at plane step k a
// block updates red on plane k (tile + 1-cell ring) and black on plane k-2
// (tile).  Black on k-2 reads only red values that are final (planes k-3..k-1,
// red on k-1 done in the previous step) and none that this step's red update
// writes; red on k reads planes k-1..k+1, whose black cells are still the old
// ones.  One block barrier per step therefore separates the steps, and every
// thread has two independent updates in the phase between them.  x arrives in
// a 70 x 12 window (tile + 2-cell ring from the even x at or below the ring),
// b and EV in 66 x 10 windows (tile + 1-cell ring, which starts at an even x
// when the inner box starts at an odd one), seven and six planes deep, two
// planes ahead; all three loads of a plane complete on its mbarrier, whose
// waits are bounded.
constexpr int kSt2BoxX = 70, kSt2BoxBX = kSwTx + 2, kSt2BoxBY = kSwTy + 2;
constexpr int kSt2SlotsX = 7, kSt2SlotsB = 6;
constexpr int kSt2PlaneX = 848;  // doubles per x slot: 70 x 12 = 840, padded to a 128-byte multiple
constexpr int kSt2PlaneB = 672;  // doubles per b / EV slot: 66 x 10 = 660, padded
constexpr unsigned kSt2BytesX = kSt2BoxX * kTmaBoxY * sizeof(double);
constexpr unsigned kSt2BytesB = kSt2BoxBX * kSt2BoxBY * sizeof(double);
static_assert(kSt2BoxX >= kSwTx + 5 && (kSt2PlaneX * 8) % 128 == 0 && (kSt2PlaneB * 8) % 128 == 0, "slots");
static_assert(kSt2BoxX * kTmaBoxY <= kSt2PlaneX && kSt2BoxBX * kSt2BoxBY <= kSt2PlaneB, "windows fit their slots");

inline size_t sweep_tma2_smem(bool turb) {
    return (size_t) kSt2PlaneX * kSt2SlotsX * sizeof(double) +
           (size_t) kSt2PlaneB * kSt2SlotsB * (turb ? 2 : 1) * sizeof(double);
}

template <bool TURB, int ZB>
__global__ void __launch_bounds__(kStThreads, 2)
k_cgs_sweep_tma2(const __grid_constant__ CUtensorMap tm_x, const __grid_constant__ CUtensorMap tm_b,
                 const __grid_constant__ CUtensorMap tm_e, double *__restrict__ out,
                 const uint8_t *__restrict__ flags, Level L, Box3 box, DiffCoef c, double *__restrict__ partials,
                 LoopState *__restrict__ pred) {
    extern __shared__ __align__(1024) double st_sm[];
    __shared__ double smem[32];
    __shared__ __align__(8) uint64_t bars[kSt2SlotsX];
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    if (pred && !pred->cond) return;  // iteration enqueued past convergence
    if (blockDim.x != kStThreads || blockDim.y != 1 || blockDim.z != 1) return;  // launch shape is fixed
    double *X = st_sm;                                // [kSt2SlotsX][kSt2PlaneX]
    double *B = st_sm + kSt2SlotsX * kSt2PlaneX;      // [kSt2SlotsB][kSt2PlaneB]
    double *E = B + kSt2SlotsB * kSt2PlaneB;          // [kSt2SlotsB][kSt2PlaneB] (TURB)
    const int tid = threadIdx.x;
    // 32-bit indices: the host takes this kernel only for levels of fewer than 2^31 cells
    const int nj = (int) L.Nx, nk = (int) L.nxy();
    const int bx0 = (int) box.x0, bx1 = (int) box.x1, by0 = (int) box.y0, by1 = (int) box.y1;
    const int bz0 = (int) box.z0, bz1 = (int) box.z1;
    const int wx0 = bx0 + (int) blockIdx.x * kSwTx - 2;  // global i of ring column 0
    const int wxa = wx0 - (wx0 & 1);                      // x window start, even
    const int ox = wx0 - wxa;
    const int wb = wx0 + 1;                               // b / EV window start (even: box.x0 odd)
    const int wy0 = by0 + (int) blockIdx.y * kSwTy - 2;
    const int kc0 = bz0 + (int) blockIdx.z * ZB;
    const int kc1 = min(kc0 + ZB - 1, bz1);
    const int pbase = kc0 - 2, plast = kc1 + 2;  // staged planes

    if (tid == 0) {
        for (int s = 0; s < kSt2SlotsX; s++) mbar_init(&bars[s], 1);
        fence_proxy_async();
    }
    __syncthreads();
    // thread 0: load plane p into its slots
    auto issue = [&](int p) {
        if (p > plast) return;
        const unsigned u = (unsigned) (p - pbase);
        uint64_t *bar = &bars[u % kSt2SlotsX];
        mbar_expect_tx(bar, kSt2BytesX + kSt2BytesB * (TURB ? 2u : 1u));
        tma_load_plane(X + (u % kSt2SlotsX) * kSt2PlaneX, &tm_x, wxa, wy0, p, bar);
        tma_load_plane(B + (u % kSt2SlotsB) * kSt2PlaneB, &tm_b, wb, wy0 + 1, p, bar);
        if (TURB) tma_load_plane(E + (u % kSt2SlotsB) * kSt2PlaneB, &tm_e, wb, wy0 + 1, p, bar);
    };
    auto ready = [&](int p) -> bool {
        const unsigned u = (unsigned) (p - pbase);
        return mbar_wait(&bars[u % kSt2SlotsX], (u / kSt2SlotsX) & 1u, kStPolls);
    };
    // ring slots by local plane number (32-bit, constant divisors)
    auto xslot = [&](int p) { return X + ((unsigned) (p - pbase) % (unsigned) kSt2SlotsX) * kSt2PlaneX; };
    auto bslot = [&](int p) { return (int) (((unsigned) (p - pbase) % (unsigned) kSt2SlotsB) * kSt2PlaneB); };
    // e: the cell in the x window, eb: in the b / EV window
    auto update = [&](const double *xm, const double *x0, const double *xp, int e, int eb, double &res2) {
        double ax = c.ax, ay = c.ay, az = c.az, beta = c.beta, rb = c.rbeta;
        if (TURB) {
            turb_alpha(c, E[eb], ax, ay, az, rb);
            beta = 1. / rb;
        }
        const double old = x0[e];
        const double out_h = beta * (c.dsign * B[eb] + ax * (x0[e + 1] + x0[e - 1]) +
                                     ay * (x0[e + kSt2BoxX] + x0[e - kSt2BoxX]) + az * (xp[e] + xm[e]));
        const double nw = c.omw * old + c.w * out_h;
        const double r = rb * (nw - old);
        res2 = r * r;
        return nw;
    };

    // this thread's red x-pair (tile + ring) and black x-pair (tile)
    const int ry = 1 + tid / ((kSwTx + 2) / 2), px = tid % ((kSwTx + 2) / 2);
    const int gjr = wy0 + ry;
    const bool red_row_ok = gjr >= by0 && gjr <= by1;
    const int red_row = nj * gjr;
    const bool red_tile = ry >= 2 && ry < kSwTy + 2;
    const bool has_black = tid < (kSwTx / 2) * kSwTy;
    const int tx = tid % (kSwTx / 2), ty = tid / (kSwTx / 2);
    const int gjb = wy0 + 2 + ty;
    const int black_row = nj * gjb;
    const int lx0 = 2 + 2 * tx;
    auto red_x = [&](int k) { return 1 + 2 * px + ((wx0 + 1 + gjr + k) & 1); };  // (i + j + k) even
    auto red_flag = [&](int k) -> uint8_t {
        if (!red_row_ok || k < bz0 || k > bz1) return 0;
        const int gi = wx0 + red_x(k);
        if (gi < bx0 || gi > bx1) return 0;
        return __ldg(flags + gi + red_row + nk * k);
    };
    auto black_par = [&](int kb) { return (wx0 + lx0 + gjb + kb + 1) & 1; };  // (i + j + k) odd
    auto black_flag = [&](int kb) -> uint8_t {
        if (!has_black || gjb > by1 || kb < kc0 || kb > kc1) return 0;
        const int gi = wx0 + lx0 + black_par(kb);
        if (gi > bx1) return 0;
        return __ldg(flags + gi + black_row + nk * kb);
    };

    double acc = 0.0;
    int issued = kc0 - 1 + kSwD;  // thread 0's last issued plane
    if (tid == 0)
        for (int p = pbase; p <= issued; p++) issue(p);
    bool ok = tid != 0 || (ready(pbase) && ready(pbase + 1));
    uint8_t fr = red_flag(kc0 - 1), fb = black_flag(kc0 - 3);
    bool failed = false;
    int waited = pbase + 1;  // planes up to here have landed
    for (int k = kc0 - 1; k <= kc1 + 2; k++) {
        // the next step's flags, loaded early
        const uint8_t fr_next = red_flag(k + 1), fb_next = black_flag(k - 1);
        // thread 0 waits for plane k+1; the barrier below publishes it (and the
        // previous step's red writes) to the block
        if (tid == 0 && k + 1 <= plast) ok = ok && ready(k + 1);
        fence_proxy_async();  // this thread's shared-memory writes before the slot refill below
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        if (k + 1 <= plast) waited = k + 1;
        if (tid == 0 && k + 1 + kSwD <= plast) {
            issue(k + 1 + kSwD);
            issued = k + 1 + kSwD;
        }
        // red on plane k, tile + 1-cell ring (planes up to kc1 + 1 are staged around it)
        if ((fr & kInner) && k <= kc1 + 1) {
            const int rx = red_x(k);
            const int e = rx + ox + kSt2BoxX * ry;
            const int eb = bslot(k) + (rx - 1) + kSt2BoxBX * (ry - 1);
            double *x0 = xslot(k);
            double r2;
            const double nw = update(xslot(k - 1), x0, xslot(k + 1), e, eb, r2);
            x0[e] = nw;
            if (red_tile && rx >= 2 && rx < kSwTx + 2 && k >= kc0 && k <= kc1) acc += r2;
        }
        // black on plane k-2, tile only, and the tile's plane k-2 out
        const int kb = k - 2;
        if (has_black && kb >= kc0 && kb <= kc1 && gjb <= by1) {
            const double *x0 = xslot(kb);
            const int par = black_par(kb);
            const int e0 = lx0 + ox + kSt2BoxX * (2 + ty);
            const int eb0 = bslot(kb) + (lx0 - 1) + kSt2BoxBX * (1 + ty);
#pragma unroll
            for (int s = 0; s < 2; s++) {
                const int gi = wx0 + lx0 + s;
                if (gi > bx1) continue;
                double v = x0[e0 + s];
                if (s == par && (fb & kInner)) {
                    double r2;
                    v = update(xslot(kb - 1), x0, xslot(kb + 1), e0 + s, eb0 + s, r2);
                    acc += r2;
                }
                out[gi + black_row + nk * kb] = v;
            }
        }
        fr = fr_next;
        fb = fb_next;
    }
    if (failed) {
        // a plane never arrived: flag it, let the loads in flight land, leave
        if (tid == 0) {
            if (pred) *(volatile int *) &pred->pad = 1;
            for (int p = waited + 1; p <= issued; p++) (void) ready(p);
        }
        __syncthreads();
        return;
    }
    acc = artss_block_sum(acc, smem);
    if (partials && tid == 0) partials[block_linear()] = acc;
}

// ---- the sweep on row-pair threads with mbarrier pipelines ------------------
//
// The one-phase iteration of k_cgs_sweep_tma2 (red on plane k, black on plane
// k-2), organised for fewer instructions per cell and no block-wide barrier:
//  * a lane owns two x columns (x and x + 32) of a pair of rows (j, j+1): on
//    every plane one of a column's two cells is red and the other black, so each
//    step it makes two red updates (plane k) and two black updates (plane k-2),
//    four independent chains computed together.  Lanes are consecutive in x, so
//    every shared-memory access of a warp is conflict-free.  One warp per row
//    pair covers rows y0-1 .. y0+TY of a 64 x TY tile (the tile and the red ring
//    rows); a side warp covers the ring columns x0-1 and x0+64, whose two cells
//    of a row have opposite colours (one red update per lane and plane);
//  * x (tile + 2-cell ring, 72 x (TY+4) from the even x at x0-3), b and EV
//    (tile + 1-cell ring, 66 x (TY+2) from x0-1) arrive by TMA in shared-memory
//    rings, AHEAD steps ahead, each plane completing on its full mbarrier; lane
//    31 of the side warp issues a plane once every warp has arrived on the step
//    mbarrier of the step that last read the slots it refills;
//  * red results overwrite their cells of the x ring in place (red updates read
//    only black cells of plane k, which stay old); a black update waits on the
//    red mbarrier of the step that computed its plane's red cells, on which
//    every warp arrives after its red updates; waiting threads sleep in
//    mbarrier.try_wait instead of spinning;
//  * blocks are persistent: the (tile column, plane) units of the level are
//    split evenly over the grid, a block taking consecutive planes of one or
//    two columns (segments); planes ka-2 .. kb+2 of a segment [ka, kb] are
//    staged, red runs on ka-1 .. kb+1 and black on ka .. kb.
// Each iteration's values equal the in-place red-then-black sweep; out receives
// iterate n+1 on the inner box (old values on cells that are not inner).
// Every mbarrier wait is bounded: a wait that gives up raises the loop state's
// error flag and the block leaves after the loads it issued have landed.
// Tile rows, ring depths (planes) and lookahead (steps) of one instance.  The
// slot of plane I is refilled once every warp has finished the step that last
// read its previous plane (I - NSX for x, I - NSB for b and EV); with
// NSX >= AHEAD + 5 and NSB >= AHEAD + 4 that step lies before the producer's
// current one, so the producer waits for warps at most one step behind it.
template <int TY_, int NSX_, int NSB_, int AHEAD_, int BPS_ = 2>
struct S3Cfg {
    static constexpr int TY = TY_, NSX = NSX_, NSB = NSB_, AHEAD = AHEAD_;
    static constexpr int BPS = BPS_;                // resident blocks per multiprocessor
    static constexpr int Pairs = (TY + 2) / 2;      // row pairs (tile + ring rows)
    static constexpr int Warps = Pairs + 1;         // row-pair warps (two x columns per lane) + side warp
    static constexpr int Threads = 32 * Warps;
    static constexpr int XW = 72, XH = TY + 4;      // x window (cells), from the even x at x0 - 3
    static constexpr int BW = 66, BH = TY + 2;      // b / EV window, from x0 - 1
    static constexpr int PlaneX = XW * XH;          // doubles per x slot
    static constexpr int PlaneB = (BW * BH + 15) / 16 * 16;  // doubles per b / EV slot, 128-byte multiple
    static constexpr unsigned BytesX = XW * XH * sizeof(double), BytesB = BW * BH * sizeof(double);
    static_assert(TY % 2 == 0 && TY + 2 <= 31, "row pairs; side lanes and the producer lane fit one warp");
    static_assert((PlaneX * 8) % 128 == 0 && (PlaneB * 8) % 128 == 0, "slots stay 128-byte aligned");
    static_assert(NSX >= AHEAD + 5 && NSB >= AHEAD + 4 && NSX <= 16, "ring depths (barrier rings of 16)");
    static size_t smem(bool turb) {
        return (size_t) PlaneX * NSX * sizeof(double) + (size_t) PlaneB * NSB * (turb ? 2 : 1) * sizeof(double);
    }
};
using S3Tall = S3Cfg<8, 7, 6, 2>;   // 64 x 8 tiles, 192 threads, 112.9 KB (turbulent)
using S3Flat = S3Cfg<6, 8, 7, 3>;   // 64 x 6 tiles, 160 threads, 105.2 KB, one step more lookahead
using S3Wide = S3Cfg<16, 8, 7, 3, 1>;    // 64 x 16 tiles, 320 threads, one block per multiprocessor (226 KB)
constexpr int kS3Bars = 16;         // mbarriers per ring (full, step, red)
constexpr int kS3MinPlanes = 8;     // planes per block at least
static_assert(S3Tall::XH == kTmaBoxY && S3Tall::BW == kSt2BoxBX && S3Tall::BH == kSt2BoxBY, "maps shared");

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

// one stencil update at x-window offset e (row pitch 72)
template <bool TURB>
__device__ __forceinline__ double cgs3_update(const DiffCoef &c, const double *__restrict__ xm,
                                              const double *__restrict__ x0, const double *__restrict__ xp, const int e,
                                              double bv, double ev, double &res2) {
    double ax = c.ax, ay = c.ay, az = c.az, beta = c.beta, rb = c.rbeta;
    if (TURB) {
        turb_alpha(c, ev, ax, ay, az, rb);
        beta = 1. / rb;
    }
    const double old = x0[e];
    const double out_h = beta * (c.dsign * bv + ax * (x0[e + 1] + x0[e - 1]) + ay * (x0[e + 72] + x0[e - 72]) +
                                 az * (xp[e] + xm[e]));
    const double nw = c.omw * old + c.w * out_h;
    const double r = rb * (nw - old);
    res2 = r * r;
    return nw;
}

// the block's segments: units [u0, u1) of (tile column, plane), column-major
struct S3Walk {
    int64_t u, u1;
    int nz, ncx;
    __device__ bool next(int &col, int &ka, int &kb, int bz0) {
        if (u >= u1) return false;
        col = (int) (u / nz);
        const int k0 = (int) (u - (int64_t) col * nz);
        const int64_t left = u1 - u;
        const int k1 = (int) (left < (int64_t) (nz - k0) ? k0 + left - 1 : nz - 1);
        ka = bz0 + k0;
        kb = bz0 + k1;
        u += k1 - k0 + 1;
        return true;
    }
};

template <int V>
struct S3Par {
    static constexpr int value = V;
};

// Waits on phase (g >> 4) & 1 of a ring barrier (kS3Bars = 16 per ring): each
// try_wait may suspend the thread in hardware for up to kS3SuspendNs until the
// phase completes, so a waiting warp does not spin on the issue slots; bounded
// by kS3Polls tries.
constexpr unsigned kS3SuspendNs = 2000;
constexpr int kS3Polls = 1 << 19;
__device__ __forceinline__ bool mbar_try_sleep(uint64_t *bar, unsigned parity) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity), "r"(kS3SuspendNs)
        : "memory");
    return done != 0;
}
__device__ __noinline__ bool mbar_wait_s3_slow(uint64_t *bar, unsigned parity) {
    for (int n = 0; n < kS3Polls; n++)
        if (mbar_try_sleep(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ bool mbar_wait_s3(uint64_t *bar, int g) {
    const unsigned parity = (unsigned) (g >> 4) & 1u;
    return mbar_try_sleep(bar, parity) || mbar_wait_s3_slow(bar, parity);
}
static_assert(kS3Bars == 16, "barrier rings are indexed with & 15 and >> 4");

template <bool TURB, class G3>
__global__ void __launch_bounds__(G3::Threads, G3::BPS)
k_cgs_sweep3(const __grid_constant__ CUtensorMap tm_x, const __grid_constant__ CUtensorMap tm_b,
             const __grid_constant__ CUtensorMap tm_e, double *__restrict__ out, const uint8_t *__restrict__ flags,
             const uint8_t *__restrict__ obst, Level L, Box3 box, DiffCoef c, int ncx, int ncy,
             double *__restrict__ partials, LoopState *__restrict__ pred) {
    extern __shared__ __align__(1024) double s3[];
    __shared__ double red_sm[32];
    __shared__ __align__(8) uint64_t full[kS3Bars], stepdone[kS3Bars], reddone[kS3Bars];
    __shared__ int deathx[kS3Bars], deathb[kS3Bars];  // producer: last step reading each plane's x / b, EV
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    if (pred && !pred->cond) return;  // iteration enqueued past convergence
    if (blockDim.x != G3::Threads || blockDim.y != 1 || blockDim.z != 1) return;  // launch shape is fixed
    double *X = s3;                                   // [NSX][PlaneX]
    const double *B = s3 + G3::NSX * G3::PlaneX;      // [NSB][PlaneB]
    const double *E = B + G3::NSB * G3::PlaneB;       // [NSB][PlaneB] (TURB)
    constexpr int XW = G3::XW, BW = G3::BW, TY = G3::TY;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool side = warp == G3::Pairs;
    // 32-bit indices: the host takes this kernel only for levels of fewer than 2^31 cells
    const int nj = (int) L.Nx, nk = (int) L.nxy(), nzl = (int) L.Nz;
    const int bx0 = (int) box.x0, bx1 = (int) box.x1, by0 = (int) box.y0, by1 = (int) box.y1;
    const int bz0 = (int) box.z0, bz1 = (int) box.z1;
    const int nz = bz1 - bz0 + 1;
    const int64_t units = (int64_t) ncx * ncy * nz;
    const int64_t u0 = units * blockIdx.x / gridDim.x, u1 = units * (blockIdx.x + 1) / gridDim.x;

    // producer (lane 31 of the side warp): its own walk over the segments, state
    // in shared memory so that it holds no registers of the other threads
    struct Prod {
        S3Walk w;
        int col, ka, kb, q, S0, issued, more;
    };
    __shared__ Prod pr;
    if (tid == 0) {
        for (int s = 0; s < kS3Bars; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&stepdone[s], G3::Warps);
            mbar_init(&reddone[s], G3::Warps);
        }
        fence_proxy_async();
        pr.w = S3Walk{u0, u1, nz, ncx};
        pr.kb = -1;
        pr.q = pr.S0 = pr.issued = 0;
        pr.more = pr.w.next(pr.col, pr.ka, pr.kb, bz0);
    }
    __syncthreads();

    double acc = 0.0;
    bool ok = true;
    auto issue_upto = [&](int target) {
        while (pr.more && pr.issued <= target && ok) {
            const int I = pr.issued, n = pr.kb - pr.ka + 1;
            // the slots of plane I held planes I-NSX (x) and I-NSB (b, EV): wait
            // until every warp has finished the last step that read them
            int d = -1;
            if (I >= G3::NSX) d = deathx[(I - G3::NSX) & 15];
            if (I >= G3::NSB) d = max(d, deathb[(I - G3::NSB) & 15]);
            if (d >= 0 && !(ok = mbar_wait_s3(&stepdone[d & 15], d))) break;
            const int x0 = bx0 + 64 * (pr.col % ncx), y0 = by0 + TY * (pr.col / ncx);
            const int k = pr.ka - 2 + pr.q;
            const int bar = I & 15;
            // x of local plane q is read on steps q-2 .. q+2, b and EV on q-1 and q+1 (within 0 .. n+2)
            deathx[bar] = pr.S0 + min(pr.q + 2, n + 2);
            deathb[bar] = pr.S0 + min(pr.q + 1, n + 2);
            mbar_expect_tx(&full[bar], G3::BytesX + G3::BytesB * (TURB ? 2u : 1u));
            tma_load_plane(X + (I % G3::NSX) * G3::PlaneX, &tm_x, x0 - 3, y0 - 2, k, &full[bar]);
            tma_load_plane((double *) B + (I % G3::NSB) * G3::PlaneB, &tm_b, x0 - 1, y0 - 1, k, &full[bar]);
            if (TURB) tma_load_plane((double *) E + (I % G3::NSB) * G3::PlaneB, &tm_e, x0 - 1, y0 - 1, k, &full[bar]);
            pr.issued = I + 1;
            if (++pr.q == n + 4) {  // segment staged: the next one starts n + 3 steps later
                pr.S0 += n + 3;
                pr.q = 0;
                pr.more = pr.w.next(pr.col, pr.ka, pr.kb, bz0);
            }
        }
    };

    // Cells of this thread.  Row-pair warp rp: lane l owns x = x0 + l and
    // x0 + 32 + l (columns 0 and 1) of rows A = y0 + 2 rp - 1 and B = A + 1; the
    // red cell of a column on even local steps is er[0] (x-window offset of
    // column 0), on odd steps er[1]; the black cell is the other.  Side lane l
    // (l <= TY + 1): A = (x0 - 1, y0 - 1 + l), B = (x0 + 64, same row).
    const int rowA = side ? lane - 1 : 2 * warp - 1;  // relative to y0
    const int lrow = side ? min(lane, TY + 1) : 0;   // side lanes past the ring keep in-window offsets
    const int xoA = side ? 2 + XW * (lrow + 1) : lane + 3 + XW * (rowA + 2);
    const int xoB = side ? xoA + 65 : xoA + XW;
    const int boA = side ? BW * lrow : lane + 1 + BW * (rowA + 1);
    const int boB = side ? boA + 65 : boA + BW;
    const bool tileA = !side && rowA >= 0, tileB = !side && rowA + 1 < TY;
    const int gdB = side ? 65 : nj;  // global index of B minus A

    S3Walk cw{u0, u1, nz, ncx};
    int col, ka, kb, S = 0, P = 0;  // segment; its first step and first plane
    while (ok && cw.next(col, ka, kb, bz0)) {
        const int n = kb - ka + 1;
        const int x0 = bx0 + 64 * (col % ncx), y0 = by0 + TY * (col / ncx);
        const int gx = side ? x0 - 1 : x0 + lane, gy = y0 + rowA;
        const bool yA = gy >= by0 && gy <= by1, yB = side ? yA : (gy + 1 >= by0 && gy + 1 <= by1);
        const bool xin0 = side ? (lane <= TY + 1 && gx >= bx0) : gx <= bx1;
        const bool xin1 = side ? (lane <= TY + 1 && x0 + 64 <= bx1) : gx + 32 <= bx1;
        const bool okA0 = xin0 && yA, okB0 = (side ? xin1 : xin0) && yB;  // column 0 (side: left A, right B)
        const bool okA1 = !side && xin1 && yA, okB1 = !side && xin1 && yB;  // column 1
        const bool redA0 = ((gx + gy + ka - 1) & 1) == 0;  // A red on even local steps (both columns)
        const int er[2] = {redA0 ? xoA : xoB, redA0 ? xoB : xoA};
        const int ebr[2] = {redA0 ? boA : boB, redA0 ? boB : boA};
        const bool ok0[2] = {redA0 ? okA0 : okB0, redA0 ? okB0 : okA0};
        const bool ok1[2] = {redA0 ? okA1 : okB1, redA0 ? okB1 : okA1};
        const bool tr[2] = {redA0 ? tileA : tileB, redA0 ? tileB : tileA};  // the cell lies in a tile row
        const int gA = gx + nj * gy;
        const bool wA0 = tileA && okA0, wB0 = tileB && okB0, wA1 = tileA && okA1, wB1 = tileB && okB1;
        const uint8_t *ob = obst ? obst + (int64_t) col * nzl : nullptr;
        // slot offsets (doubles) of planes qr+1, qr, qr-1, qr-2, qr-3 with qr = P + s + 1 the red plane
        int xp1 = ((P + 2) % G3::NSX) * G3::PlaneX, x00 = ((P + 1) % G3::NSX) * G3::PlaneX;
        int xm1 = (P % G3::NSX) * G3::PlaneX, xm2 = ((P + G3::NSX - 1) % G3::NSX) * G3::PlaneX,
            xm3 = ((P + G3::NSX - 2) % G3::NSX) * G3::PlaneX;  // before P: unused until they hold this segment's planes
        int b00 = ((P + 1) % G3::NSB) * G3::PlaneB, bm1 = (P % G3::NSB) * G3::PlaneB,
            bm2 = ((P + G3::NSB - 1) % G3::NSB) * G3::PlaneB;
        // obstacle bytes of the red planes of steps s, s-1, s-2 (the last is black's plane)
        int o0 = (ob && ka - 1 >= 0) ? ob[ka - 1] : 0, o1 = 0, o2 = 0;

        // the red (R) and black (K) updates of one step, computed together (independent
        // chains: red writes plane qr, black reads planes qr-1 .. qr-3)
        auto updates = [&](auto par, auto do_r, auto do_k, int kr) {
            constexpr int Q = decltype(par)::value;
            constexpr bool R = decltype(do_r)::value, K = decltype(do_k)::value;
            double nr0 = 0, nr1 = 0, rr0 = 0, rr1 = 0, nb0 = 0, nb1 = 0, rb0 = 0, rb1 = 0, ob0 = 0, ob1 = 0;
            bool onr0 = false, onr1 = false, onb0 = false, onb1 = false;
            if (R) {
                const int e = er[Q], eb = b00 + ebr[Q];
                onr0 = ok0[Q];
                onr1 = ok1[Q];
                if (o0) {
                    const int g = gA + (e == xoA ? 0 : gdB) + nk * kr;
                    onr0 = onr0 && (__ldg(flags + g) & kInner);
                    if (!side) onr1 = onr1 && (__ldg(flags + g + 32) & kInner);
                }
                double *pc = X + x00 + e;
                nr0 = cgs3_update<TURB>(c, X + xm1 + e, pc, X + xp1 + e, 0, B[eb], TURB ? E[eb] : 0.0, rr0);
                if (!side) nr1 = cgs3_update<TURB>(c, X + xm1 + e, pc, X + xp1 + e, 32, B[eb + 32],
                                                   TURB ? E[eb + 32] : 0.0, rr1);
            }
            if (K) {
                const int e = er[Q ^ 1], eb = bm2 + ebr[Q ^ 1];
                onb0 = tr[Q ^ 1] && ok0[Q ^ 1];
                onb1 = tr[Q ^ 1] && ok1[Q ^ 1];
                if (o2) {
                    const int g = gA + (e == xoA ? 0 : gdB) + nk * (kr - 2);
                    onb0 = onb0 && (__ldg(flags + g) & kInner);
                    onb1 = onb1 && (__ldg(flags + g + 32) & kInner);
                }
                const double *pc = X + xm2 + e;
                ob0 = pc[0];
                ob1 = pc[32];
                nb0 = cgs3_update<TURB>(c, X + xm3 + e, pc, X + xm1 + e, 0, B[eb], TURB ? E[eb] : 0.0, rb0);
                nb1 = cgs3_update<TURB>(c, X + xm3 + e, pc, X + xm1 + e, 32, B[eb + 32], TURB ? E[eb + 32] : 0.0,
                                        rb1);
            }
            if (R) {
                double *pc = X + x00 + er[Q];
                if (onr0) pc[0] = nr0;
                if (onr1) pc[32] = nr1;
                if (tr[Q] && kr >= ka && kr <= kb) acc += (onr0 ? rr0 : 0.0) + (onr1 ? rr1 : 0.0);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&reddone[(S + (kr - ka + 1)) & 15]);
            if (K) {
                acc += (onb0 ? rb0 : 0.0) + (onb1 ? rb1 : 0.0);
                const double vb0 = onb0 ? nb0 : ob0, vb1 = onb1 ? nb1 : ob1;
                const double *pr0 = X + xm2 + er[Q];  // the red cells of the same plane
                const double vr0 = pr0[0], vr1 = pr0[32];
                const bool aRed = er[Q] == xoA;
                double *o = out + gA + nk * (kr - 2);
                if (wA0) o[0] = aRed ? vr0 : vb0;
                if (wB0) o[nj] = aRed ? vb0 : vr0;
                if (wA1) o[32] = aRed ? vr1 : vb1;
                if (wB1) o[nj + 32] = aRed ? vb1 : vr1;
            }
        };

        auto step = [&](int s, auto par) {
            const int Sg = S + s;
            const int kr = ka - 1 + s;
            const int onext = (ob && kr + 1 < nzl) ? __ldg(ob + kr + 1) : 0;  // next step's, loaded early
            if (side) {
                if (lane == 31) issue_upto(P + min(s + 2, n + 3) + G3::AHEAD);
                ok = __all_sync(0xffffffffu, ok);  // the side warp leaves together
            }
            if (ok) {
                if (s == 0)
                    ok = mbar_wait_s3(&full[P & 15], P) && mbar_wait_s3(&full[(P + 1) & 15], P + 1) &&
                         mbar_wait_s3(&full[(P + 2) & 15], P + 2);
                else if (s + 2 <= n + 3)
                    ok = mbar_wait_s3(&full[(P + s + 2) & 15], P + s + 2);
            }
            const bool do_k = !side && s >= 3;  // black on plane kr - 2 (local plane s - 1)
            if (ok && do_k) ok = mbar_wait_s3(&reddone[(Sg - 2) & 15], Sg - 2);
            if (!ok) return;
            const bool do_r = s <= n + 1 && kr >= bz0 && kr <= bz1;  // red on plane kr (local plane s + 1)
            using T = S3Par<1>;
            using F = S3Par<0>;
            if (do_r && do_k) updates(par, T{}, T{}, kr);
            else if (do_r) updates(par, T{}, F{}, kr);
            else if (do_k) updates(par, F{}, T{}, kr);
            else updates(par, F{}, F{}, kr);
            fence_proxy_async();  // this thread's shared-memory writes before slot refills
            __syncwarp();
            if (lane == 0) mbar_arrive(&stepdone[Sg & 15]);
            // rotate the slot rings and the obstacle history to step s + 1
            xm3 = xm2; xm2 = xm1; xm1 = x00; x00 = xp1;
            xp1 = xp1 + G3::PlaneX == G3::NSX * G3::PlaneX ? 0 : xp1 + G3::PlaneX;
            bm2 = bm1; bm1 = b00;
            b00 = b00 + G3::PlaneB == G3::NSB * G3::PlaneB ? 0 : b00 + G3::PlaneB;
            o2 = o1; o1 = o0; o0 = onext;
        };
        for (int s = 0; s <= n + 2 && ok; s += 2) {
            step(s, S3Par<0>{});
            if (s + 1 <= n + 2 && ok) step(s + 1, S3Par<1>{});
        }
        S += n + 3;
        P += n + 4;
    }
    if (!ok) {
        // a wait gave up: flag it, let the loads this block issued land, leave
        if (pred) *(volatile int *) &pred->pad = 1;
        if (side && lane == 31)
            for (int g = max(0, pr.issued - kS3Bars); g < pr.issued; g++) (void) mbar_wait_s3(&full[g & 15], g);
        return;
    }
    acc = artss_block_sum(acc, red_sm);
    if (partials && tid == 0) partials[blockIdx.x] = acc;
}

// ---- colored Gauss-Seidel with FP32 sweeps inside FP64 defect correction ----
//
// One iteration of the reference's red-then-black sweep (stencil at
// ColoredGaussSeidelDiffuse.cpp:316-341) written as a correction of x: with
// the system rb x - sum(alpha x_nb) = dsign b and the defect r = dsign b -
// (rb x - sum(alpha x_nb)) of the current x (FP64), the red update is
// e = r / rb and the black update e = (r + sum(alpha e_red,nb)) / rb, then
// x += e, which in exact arithmetic is the in-place sweep (w = 1).  The
// defect and the correction are FP32 values in one scratch array (red cells:
// e, black cells: r) and the black update is FP32 arithmetic; the defect and
// x stay FP64.  The loop stops on the reference's measure ||rb (x_new - x)||_2
// = ||rb e||_2.
template <bool TURB>
__device__ __forceinline__ void cgsm_coef(const DiffCoef &c, const double *__restrict__ ev, int q, double &ax,
                                          double &ay, double &az, double &rb) {
    ax = c.ax, ay = c.ay, az = c.az, rb = c.rbeta;
    if (TURB) turb_alpha(c, ev[q], ax, ay, az, rb);
}

// red cells: w = (float) (r / rb); black cells: w = (float) r
template <bool TURB>
__global__ void k_cgsm_defect(float *__restrict__ wv, const double *__restrict__ x, const double *__restrict__ b,
                              const double *__restrict__ ev, const uint8_t *__restrict__ flags, Level L, Box3 box,
                              DiffCoef c, const LoopState *__restrict__ pred) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    if (pred && !pred->cond) return;  // iteration enqueued past convergence
    ARTSS_COLUMN(box);
    if (!col) return;
    const int nj = (int) L.Nx, nk = (int) L.nxy();
    for (int k = (int) box.z0 + (int) blockIdx.z; k <= (int) box.z1; k += (int) gridDim.z) {
        const int q = i + nj * j + nk * k;
        if (!(flags[q] & kInner)) continue;
        double ax, ay, az, rb;
        cgsm_coef<TURB>(c, ev, q, ax, ay, az, rb);
        const double r = c.dsign * b[q] + ax * (x[q + 1] + x[q - 1]) + ay * (x[q + nj] + x[q - nj]) +
                         az * (x[q + nk] + x[q - nk]) - rb * x[q];
        wv[q] = ((i + j + k) & 1) == 0 ? (float) (r / rb) : (float) r;
    }
}

// black cells: e = (r + sum(alpha e_red,nb)) / rb in FP32; every inner cell
// x += e; block partial of sum (rb e)^2
template <bool TURB>
__global__ void k_cgsm_correct(double *__restrict__ x, const float *__restrict__ wv, const double *__restrict__ ev,
                               const uint8_t *__restrict__ flags, Level L, Box3 box, DiffCoef c,
                               double *__restrict__ partials, const LoopState *__restrict__ pred) {
    __shared__ double smem[32];
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    if (pred && !pred->cond) return;  // iteration enqueued past convergence
    ARTSS_COLUMN(box);
    double acc = 0.0;
    if (col) {
        const int nj = (int) L.Nx, nk = (int) L.nxy();
        for (int k = (int) box.z0 + (int) blockIdx.z; k <= (int) box.z1; k += (int) gridDim.z) {
            const int q = i + nj * j + nk * k;
            if (!(flags[q] & kInner)) continue;
            double ax, ay, az, rb;
            cgsm_coef<TURB>(c, ev, q, ax, ay, az, rb);
            float e = wv[q];
            if (((i + j + k) & 1) != 0) {
                // red neighbours that are not inner carry no correction
                auto er = [&](int n) { return (flags[n] & kInner) ? wv[n] : 0.0f; };
                e = (e + (float) ax * (er(q + 1) + er(q - 1)) + (float) ay * (er(q + nj) + er(q - nj)) +
                     (float) az * (er(q + nk) + er(q - nk))) /
                    (float) rb;
            }
            x[q] += (double) e;
            const double rr = rb * (double) e;
            acc += rr * rr;
        }
    }
    acc = artss_block_sum(acc, smem);
    if (partials && threadIdx.x == 0 && threadIdx.y == 0) partials[block_linear()] = acc;
}

// One Jacobi step of JacobiDiffuse (laminar: JacobiDiffuse.cpp:241-249, note
// the division by reciprocal_beta; turbulent: :345-362) + residual partials
// of sum (rbeta * (out - in))^2 (:72-79).
template <bool TURB>
__global__ void k_jacobi_diffuse(double *__restrict__ out, const double *__restrict__ in, const double *__restrict__ b,
                                 const double *__restrict__ ev, const uint8_t *__restrict__ flags, Level L, Box3 box,
                                 DiffCoef c, double *__restrict__ partials, const LoopState *__restrict__ pred) {
    __shared__ double smem[32];
    if (pred && !pred->cond) return;  // iteration enqueued past convergence
    ARTSS_COLUMN(box);
    const int nj = (int) L.Nx, nk = (int) L.nxy();
    double acc = 0.0;
    if (col) {
        for (int k = (int) box.z0 + (int) blockIdx.z; k <= (int) box.z1; k += (int) gridDim.z) {
            const int q = i + (int) L.Nx * j + nk * k;
            if (!(flags[q] & kInner)) continue;
            double out_h, rb;
            if (TURB) {
                double ax, ay, az;
                turb_alpha(c, ev[q], ax, ay, az, rb);
                const double bb = 1. / rb;
                const double d_ax = ax * (in[q + 1] + in[q - 1]);
                const double d_ay = ay * (in[q + nj] + in[q - nj]);
                const double d_az = az * (in[q + nk] + in[q - nk]);
                out_h = bb * (c.dsign * b[q] + d_ax + d_ay + d_az);
            } else {
                rb = c.rbeta;
                out_h = (c.dsign * b[q] + c.ax * (in[q + 1] + in[q - 1]) + c.ay * (in[q + nj] + in[q - nj])
                         + c.az * (in[q + nk] + in[q - nk])) / c.rbeta;
            }
            const double nw = c.omw * in[q] + c.w * out_h;
            out[q] = nw;
            const double res = rb * (nw - in[q]);
            acc += res * res;
        }
    }
    acc = artss_block_sum(acc, smem);
    if (threadIdx.x == 0 && threadIdx.y == 0) partials[block_linear()] = acc;
}

// in = out over the domain list (JacobiDiffuse.cpp:85-89)
__global__ void k_copy_domain(double *__restrict__ dst, const double *__restrict__ src,
                              const uint8_t *__restrict__ flags, Level L, Box3 box, const LoopState *__restrict__ pred) {
    if (pred && !pred->cond) return;
    ARTSS_COLUMN(box);
    if (!col) return;
    for (int k = (int) box.z0 + (int) blockIdx.z; k <= (int) box.z1; k += (int) gridDim.z) {
        const int q = i + (int) L.Nx * j + (int) L.nxy() * k;
        if (flags[q] & kDomain) dst[q] = src[q];
    }
}

// exchanges two arrays element by element
// After a captured colored Gauss-Seidel loop: the last iterate sits in `in`
// when (s0 + it) is odd; exchange the arrays (the caller keeps in) or copy it
// back, as the host does after an uncaptured loop.
__global__ void k_cgs_fixup(double *__restrict__ out, double *__restrict__ in, const LoopState *__restrict__ st,
                            int s0, int in_is_scratch, int64_t n) {
    const long long it = st->it;
    if (it <= 0 || !((s0 + it) & 1)) return;
    for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
        const double v = in[i];
        if (!in_is_scratch) in[i] = out[i];
        out[i] = v;
    }
}

__global__ void k_swap(double *__restrict__ x, double *__restrict__ y, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
        const double t = x[i];
        x[i] = y[i];
        y[i] = t;
    }
}

// Iterations enqueued per host round trip of a predicated loop: the count the
// same call site needed last time (usually exact, one round trip), doubled
// when a batch ends without convergence.
inline int64_t& loop_hint(artss_ctx *ctx, int site, int field_type) {
    return ctx->loop_hint[site][field_type & 15];
}

int check_field_args(artss_ctx *ctx, std::initializer_list<const void *> ptrs) {
    if (!ctx) { set_error("null context"); return ARTSS_ERR_ARG; }
    for (const void *p : ptrs)
        if (!p) { set_error("null field pointer"); return ARTSS_ERR_ARG; }
    return ARTSS_OK;
}

DiffCoef diff_coef(const artss_ctx *ctx, double D, double dt, double w, double dsign) {
    // ColoredGaussSeidelDiffuse.cpp:49-62 / JacobiDiffuse.cpp:46-60, level 0
    DiffCoef c{};
    const double dx = ctx->grid.dx[0], dy = ctx->grid.dy[0], dz = ctx->grid.dz[0];
    c.rdx = 1. / dx;
    c.rdy = 1. / dy;
    c.rdz = 1. / dz;
    c.ax = D * dt * c.rdx * c.rdx;
    c.ay = D * dt * c.rdy * c.rdy;
    c.az = D * dt * c.rdz * c.rdz;
    c.rbeta = (1. + 2. * (c.ax + c.ay + c.az));
    c.beta = 1. / c.rbeta;
    c.dsign = dsign;
    c.w = w;
    c.omw = 1 - w;
    c.D = D;
    c.dt = dt;
    return c;
}

}  // namespace artss

using namespace artss;

extern "C" {

int artss_advect_sl(artss_ctx *ctx, double *out, const double *in, const double *u, const double *v,
                    const double *w, double dt, int out_field_type) {
    int st = check_field_args(ctx, {out, in, u, v, w});
    if (st || (st = check_field_type(out_field_type))) return st;
    const Level &L = ctx->lvl[0];
    if (L.size() >= ((int64_t) 1 << 31)) { set_error("advection: level of 2^31 cells or more"); return ARTSS_ERR_LIMIT; }
    const Box3 box = inner_box(L);
    AdvCoef c{dt / ctx->grid.dx[0], dt / ctx->grid.dy[0], dt / ctx->grid.dz[0], L.i1, L.i2, L.j1, L.j2, L.k1, L.k2};
    const bool fresh = out != in && out != u && out != v && out != w;
    if ((st = tuned_column_launch(ctx, kTuneAdvect1, 0, box, fresh, [&](dim3 g, dim3 b) -> int {
             ARTSS_LAUNCH_PDL(ctx, FAM_ADVECT, (k_advect<1>), g, b, 0, out, nullptr, nullptr, in, nullptr, nullptr, u,
                              v, w, ctx->d_flags[0], L, box, c);
             ARTSS_LAUNCH_CK(ctx);
             return ARTSS_OK;
         })))
        return st;
    return apply_bc(ctx, out, 0, out_field_type);
}

int artss_advect_sl_uvw(artss_ctx *ctx, double *out_u, double *out_v, double *out_w, const double *in_u,
                        const double *in_v, const double *in_w, const double *u, const double *v, const double *w,
                        double dt) {
    int st = check_field_args(ctx, {out_u, out_v, out_w, in_u, in_v, in_w, u, v, w});
    if (st) return st;
    const Level &L = ctx->lvl[0];
    if (L.size() >= ((int64_t) 1 << 31)) { set_error("advection: level of 2^31 cells or more"); return ARTSS_ERR_LIMIT; }
    const Box3 box = inner_box(L);
    AdvCoef c{dt / ctx->grid.dx[0], dt / ctx->grid.dy[0], dt / ctx->grid.dz[0], L.i1, L.i2, L.j1, L.j2, L.k1, L.k2};
    bool fresh = true;
    for (const double *o : {(const double *) out_u, (const double *) out_v, (const double *) out_w})
        for (const double *x : {in_u, in_v, in_w, u, v, w}) fresh = fresh && o != x;
    if ((st = tuned_column_launch(ctx, kTuneAdvect3, 0, box, fresh, [&](dim3 g, dim3 b) -> int {
             ARTSS_LAUNCH_PDL(ctx, FAM_ADVECT, (k_advect<3>), g, b, 0, out_u, out_v, out_w, in_u, in_v, in_w, u, v, w,
                              ctx->d_flags[0], L, box, c);
             ARTSS_LAUNCH_CK(ctx);
             return ARTSS_OK;
         })))
        return st;
    if ((st = apply_bc(ctx, out_u, 0, ARTSS_FIELD_U))) return st;
    if ((st = apply_bc(ctx, out_v, 0, ARTSS_FIELD_V))) return st;
    return apply_bc(ctx, out_w, 0, ARTSS_FIELD_W);
}

int artss_turb_const_smagorinsky(artss_ctx *ctx, double *nu_t, const double *u, const double *v, const double *w,
                                 double cs) {
    int st = check_field_args(ctx, {nu_t, u, v, w});
    if (st) return st;
    const Level &L = ctx->lvl[0];
    const Box3 box = inner_box(L);
    const double dx = ctx->grid.dx[0], dy = ctx->grid.dy[0], dz = ctx->grid.dz[0];
    const double delta_s = cbrt(dx * dy * dz);
    const double cs2d2 = cs * cs * delta_s * delta_s;
    const bool fresh = nu_t != u && nu_t != v && nu_t != w;
    if ((st = tuned_column_launch(ctx, kTuneSmagorinsky, 0, box, fresh, [&](dim3 g, dim3 b) -> int {
             ARTSS_LAUNCH_PDL(ctx, FAM_SMAGORINSKY, k_smagorinsky, g, b, 0, nu_t, u, v, w, ctx->d_flags[0], L, box,
                              1. / dx, 1. / dy, 1. / dz, cs2d2);
             ARTSS_LAUNCH_CK(ctx);
             return ARTSS_OK;
         })))
        return st;
    return apply_bc(ctx, nu_t, 0, ARTSS_FIELD_NU);
}

int artss_divergence(artss_ctx *ctx, double *rhs, const double *u, const double *v, const double *w) {
    int st = check_field_args(ctx, {rhs, u, v, w});
    if (st) return st;
    const Level &L = ctx->lvl[0];
    const Box3 box = inner_box(L);
    const double hx = 0.5 * (1. / ctx->grid.dx[0]);
    const double hy = 0.5 * (1. / ctx->grid.dy[0]);
    const double hz = 0.5 * (1. / ctx->grid.dz[0]);
    const bool fresh = rhs != u && rhs != v && rhs != w;
    if ((st = tuned_column_launch(ctx, kTuneDivergence, 0, box, fresh, [&](dim3 g, dim3 b) -> int {
             ARTSS_LAUNCH_PDL(ctx, FAM_DIVERGENCE, k_divergence, g, b, 0, rhs, u, v, w, ctx->d_flags[0], L, box, hx,
                              hy, hz);
             ARTSS_LAUNCH_CK(ctx);
             return ARTSS_OK;
         })))
        return st;
    const Box3 ring = domain_box(L);
    ARTSS_LAUNCH_PDL(ctx, FAM_DIVERGENCE, k_ghost_ring_zero, zgrid(ring), box_block(), 0, rhs, L, ring);
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

int artss_projection(artss_ctx *ctx, double *u, double *v, double *w, const double *us, const double *vs,
                     const double *ws, const double *p) {
    int st = check_field_args(ctx, {u, v, w, us, vs, ws, p});
    if (st) return st;
    const Level &L = ctx->lvl[0];
    const Box3 box = inner_box(L);
    const double hx = 0.5 * (1. / ctx->grid.dx[0]);
    const double hy = 0.5 * (1. / ctx->grid.dy[0]);
    const double hz = 0.5 * (1. / ctx->grid.dz[0]);
    bool fresh = true;
    for (const double *o : {(const double *) u, (const double *) v, (const double *) w})
        for (const double *x : {us, vs, ws, p}) fresh = fresh && o != x;
    if ((st = tuned_column_launch(ctx, kTuneProjection, 0, box, fresh, [&](dim3 g, dim3 b) -> int {
             ARTSS_LAUNCH_PDL(ctx, FAM_PROJECTION, k_projection, g, b, 0, u, v, w, us, vs, ws, p, ctx->d_flags[0], L,
                              box, hx, hy, hz);
             ARTSS_LAUNCH_CK(ctx);
             return ARTSS_OK;
         })))
        return st;
    if ((st = apply_bc(ctx, u, 0, ARTSS_FIELD_U))) return st;
    if ((st = apply_bc(ctx, v, 0, ARTSS_FIELD_V))) return st;
    return apply_bc(ctx, w, 0, ARTSS_FIELD_W);
}

int artss_buoyancy_force(artss_ctx *ctx, double *force, const double *T, const double *Ta, double beta, double g) {
    int st = check_field_args(ctx, {force, T, Ta});
    if (st) return st;
    const Level &L = ctx->lvl[0];
    const Box3 box = domain_box(L);
    const bool fresh = force != T && force != Ta;
    return tuned_column_launch(ctx, kTuneBuoyancy, 0, box, fresh, [&](dim3 gr, dim3 b) -> int {
        ARTSS_LAUNCH_PDL(ctx, FAM_BUOYANCY, k_buoyancy, gr, b, 0, force, T, Ta, ctx->d_flags[0], L, box, -beta, g);
        ARTSS_LAUNCH_CK(ctx);
        return ARTSS_OK;
    });
}

int artss_cfl(artss_ctx *ctx, const double *u, const double *v, const double *w, double dt, double *cfl) {
    int st = check_field_args(ctx, {u, v, w, cfl});
    if (st) return st;
    const Level &L = ctx->lvl[0];
    const Box3 box = inner_box(L);
    const dim3 g = zgrid(box);
    if ((st = check_reduce_blocks(g))) return st;
    const int nb = nblocks(g);
    ARTSS_LAUNCH(ctx, FAM_REDUCE, k_cfl_max<<<g, box_block(), 0, ctx->stream>>>(
                                      u, v, w, ctx->d_flags[0], L, box, ctx->grid.dx[0], ctx->grid.dy[0],
                                      ctx->grid.dz[0], ctx->d_partials));
    ARTSS_LAUNCH_CK(ctx);
    std::vector<double> part((size_t) nb);
    ARTSS_CK(cudaMemcpyAsync(part.data(), ctx->d_partials, (size_t) nb * sizeof(double), cudaMemcpyDeviceToHost,
                             ctx->stream));
    ARTSS_CK(cudaStreamSynchronize(ctx->stream));
    double m = 0.0;
    for (double x : part) m = std::max(m, x);
    *cfl = dt * m;
    return ARTSS_OK;
}

int artss_diffuse_explicit(artss_ctx *ctx, double *out, const double *in, double D, const double *ev, double dt,
                           int field_type) {
    int st = check_field_args(ctx, {out, in});
    if (st || (st = check_field_type(field_type))) return st;
    if (out == in) { set_error("out and in must be distinct arrays"); return ARTSS_ERR_ARG; }
    const Level &L = ctx->lvl[0];
    const Box3 box = inner_box(L);
    const double dx = ctx->grid.dx[0], dy = ctx->grid.dy[0], dz = ctx->grid.dz[0];
    // ExplicitDiffuse.cpp:64-66 (laminar); the turbulent step uses D and EV only
    const double rdx = D / (dx * dx), rdy = D / (dy * dy), rdz = D / (dz * dz);
    if (ev)
        ARTSS_LAUNCH_PDL(ctx, FAM_JACOBI, k_explicit_diffuse<true>, zgrid(box), box_block(), 0, out, in, ev,
                         (const uint8_t *) ctx->d_flags[0], L, box, D, dt, rdx, rdy, rdz);
    else
        ARTSS_LAUNCH_PDL(ctx, FAM_JACOBI, k_explicit_diffuse<false>, zgrid(box), box_block(), 0, out, in,
                         (const double *) nullptr, (const uint8_t *) ctx->d_flags[0], L, box, D, dt, rdx, rdy, rdz);
    ARTSS_LAUNCH_CK(ctx);
    return apply_bc(ctx, out, 0, field_type, nullptr);
}

int artss_dissipate(artss_ctx *ctx, double *out, const double *u, const double *v, const double *w, double nu,
                    double dt, int field_type) {
    int st = check_field_args(ctx, {out, u, v, w});
    if (st || (st = check_field_type(field_type))) return st;
    const Level &L = ctx->lvl[0];
    const Box3 box = inner_box(L);
    const double hx = 0.5 * (1. / ctx->grid.dx[0]), hy = 0.5 * (1. / ctx->grid.dy[0]), hz = 0.5 * (1. / ctx->grid.dz[0]);
    ARTSS_LAUNCH_PDL(ctx, FAM_ADD_SOURCE, k_dissipate, zgrid(box), box_block(), 0, out, u, v, w,
                     (const uint8_t *) ctx->d_flags[0], L, box, nu, dt, hx, hy, hz);
    ARTSS_LAUNCH_CK(ctx);
    return apply_bc(ctx, out, 0, field_type, nullptr);
}

int artss_add_source(artss_ctx *ctx, double *out, const double *S, double dt, int field_type) {
    int st = check_field_args(ctx, {out, S});
    if (st || (st = check_field_type(field_type))) return st;
    const Level &L = ctx->lvl[0];
    const Box3 box = inner_box(L);
    ARTSS_LAUNCH_PDL(ctx, FAM_ADD_SOURCE, k_add_source, zgrid(box), box_block(), 0, out, S, ctx->d_flags[0], L, box, dt);
    ARTSS_LAUNCH_CK(ctx);
    return apply_bc(ctx, out, 0, field_type);
}

namespace {

// TMA descriptors of one sweep: x (the array read), b, EV, for the kernel with
// 72 x 12 windows and for the one-phase kernel (70 x 12 and 66 x 10)
// variant number of k_cgs_sweep3 with 64 x 8 tiles; + 1: 64 x 6 tiles; + 2: 64 x 16
// tiles, one block per multiprocessor
constexpr int kSweepRowPair = 6;
constexpr int kSweepVariants = kSweepRowPair + 3;
struct SweepMaps {
    const CUtensorMap *x = nullptr, *b = nullptr, *e = nullptr;
    const CUtensorMap *x2 = nullptr, *b2 = nullptr, *e2 = nullptr;
    const CUtensorMap *x3 = nullptr, *b3 = nullptr, *e3 = nullptr;  // 72 x 10 and 66 x 8 windows
    const CUtensorMap *x4 = nullptr, *b4 = nullptr, *e4 = nullptr;  // 72 x 20 and 66 x 18 windows
};

// Obstacle table of the row-pair sweep (k_cgs_sweep3) with tiles of 64 x ty
// cells (table t of the context): per tile column (column-major over the inner
// box) and plane of level 0, 1 where the tile or its 1-cell ring holds a box
// cell that is not inner (the kernel reads cell flags there only).
// *out = nullptr when every box cell is inner.  Built on the host from the
// inner-cell bitmap on first use.
int sweep3_obst(artss_ctx *ctx, const Box3 &box, int t, int ty_rows, int ncx, int ncy, const uint8_t **out) {
    if (ctx->sweep3_obst_state[t] == 0) {
        const Level &L = ctx->lvl[0];
        const std::vector<bool> &in = ctx->h_inner[0];
        if (!in.empty() && ctx->n_inner[0] == box.nx() * box.ny() * box.nz()) {
            ctx->sweep3_obst_state[t] = 2;
        } else {
            // no lists uploaded: every cell goes through its flag
            std::vector<uint8_t> tab((size_t) ncx * ncy * L.Nz, in.empty() ? 1 : 0);
            if (!in.empty()) {
                for (int64_t k = box.z0; k <= box.z1; k++)
                    for (int64_t y = box.y0; y <= box.y1; y++)
                        for (int64_t x = box.x0; x <= box.x1; x++) {
                            if (in[(size_t) (x + L.Nx * y + L.nxy() * k)]) continue;
                            const int64_t cx = (x - box.x0) / 64, cy = (y - box.y0) / ty_rows;
                            for (int64_t ty = std::max<int64_t>(0, cy - 1); ty <= std::min<int64_t>(ncy - 1, cy + 1); ty++)
                                for (int64_t tx = std::max<int64_t>(0, cx - 1); tx <= std::min<int64_t>(ncx - 1, cx + 1);
                                     tx++) {
                                    const int64_t x0 = box.x0 + 64 * tx, y0 = box.y0 + ty_rows * ty;
                                    if (x >= x0 - 1 && x <= x0 + 64 && y >= y0 - 1 && y <= y0 + ty_rows)
                                        tab[(size_t) ((tx + ncx * ty) * L.Nz + k)] = 1;
                                }
                        }
            }
            if (ctx->capturing) { set_error("sweep obstacle table built inside a capture"); return ARTSS_ERR_STATE; }
            ARTSS_CK(cudaMalloc(&ctx->d_sweep3_obst[t], tab.size()));
            ARTSS_CK(cudaMemcpy(ctx->d_sweep3_obst[t], tab.data(), tab.size(), cudaMemcpyHostToDevice));
            ctx->sweep3_obst_state[t] = 1;
        }
    }
    *out = ctx->sweep3_obst_state[t] == 1 ? ctx->d_sweep3_obst[t] : nullptr;
    return ARTSS_OK;
}

// the row-pair sweep: persistent blocks, G3::BPS per multiprocessor, at least
// kS3MinPlanes (tile column, plane) units each
extern "C++" {  // a template inside the extern "C" block of this file
template <class G3>
int launch_sweep3(artss_ctx *ctx, bool turb, int t, const Box3 &box, const CUtensorMap *mx, const CUtensorMap *mb,
                  const CUtensorMap *me, double *w, const Level &L, const DiffCoef &c, LoopState *pred, int *nb) {
    const int ncx = (int) ((box.nx() + 63) / 64), ncy = (int) ((box.ny() + G3::TY - 1) / G3::TY);
    const int64_t units = (int64_t) ncx * ncy * box.nz();
    const int G = (int) std::min<int64_t>(std::min<int64_t>(G3::BPS * std::max(ctx->sm_count, 1), kMaxPartials / 2),
                                          std::max<int64_t>(1, units / kS3MinPlanes));
    const uint8_t *obst = nullptr;
    int st = sweep3_obst(ctx, box, t, G3::TY, ncx, ncy, &obst);
    if (st) return st;
    const size_t smem = G3::smem(turb);
    if (turb)
        ARTSS_LAUNCH_PDL(ctx, FAM_CGS, (k_cgs_sweep3<true, G3>), dim3(G), G3::Threads, smem, *mx, *mb, *me, w,
                         (const uint8_t *) ctx->d_flags[0], obst, L, box, c, ncx, ncy, ctx->d_partials, pred);
    else
        ARTSS_LAUNCH_PDL(ctx, FAM_CGS, (k_cgs_sweep3<false, G3>), dim3(G), G3::Threads, smem, *mx, *mb, *mb, w,
                         (const uint8_t *) ctx->d_flags[0], obst, L, box, c, ncx, ncy, ctx->d_partials, pred);
    ARTSS_LAUNCH_CK(ctx);
    *nb = G;
    return ARTSS_OK;
}
}  // extern "C++"

// Variants of the TMA sweep: v < 3 the kernel with two barriers per plane step
// and z-depth kStDepths[v]; 3 <= v < 6 the one-phase kernel with
// kStDepths[v - 3]; v = 6, 7 the row-pair kernel with 64 x 8 and 64 x 6 tiles; v >= 3 only
// where the b / EV window starts at an even x.  Returns the number of blocks
// (partials) in *nb.
int launch_sweep_tma(artss_ctx *ctx, bool turb, int v, const Box3 &box, const SweepMaps &m, double *w,
                     const Level &L, const DiffCoef &c, LoopState *pred, int *nb) {
    if (v == kSweepRowPair) return launch_sweep3<S3Tall>(ctx, turb, 0, box, m.x, m.b2, m.e2, w, L, c, pred, nb);
    if (v == kSweepRowPair + 1) return launch_sweep3<S3Flat>(ctx, turb, 1, box, m.x3, m.b3, m.e3, w, L, c, pred, nb);
    if (v == kSweepRowPair + 2) return launch_sweep3<S3Wide>(ctx, turb, 2, box, m.x4, m.b4, m.e4, w, L, c, pred, nb);
    const int zb = kStDepths[v % 3];
    const dim3 g = sweep_tma_grid(box, zb);
    *nb = nblocks(g);
    const size_t smem1 = sweep_tma_smem(turb), smem2 = sweep_tma2_smem(turb);
#define ARTSS_SWEEP_TMA(K, T, Z, SM, MX, MB, ME)                                                      \
    ARTSS_LAUNCH_PDL(ctx, FAM_CGS, (K<T, Z>), g, kStThreads, SM, *MX, *MB, *ME, w,                     \
                     (const uint8_t *) ctx->d_flags[0], L, box, c, ctx->d_partials, pred)
    switch (v * 2 + (turb ? 1 : 0)) {
        case 0: ARTSS_SWEEP_TMA(k_cgs_sweep_tma, false, 8, smem1, m.x, m.b, m.e); break;
        case 1: ARTSS_SWEEP_TMA(k_cgs_sweep_tma, true, 8, smem1, m.x, m.b, m.e); break;
        case 2: ARTSS_SWEEP_TMA(k_cgs_sweep_tma, false, 16, smem1, m.x, m.b, m.e); break;
        case 3: ARTSS_SWEEP_TMA(k_cgs_sweep_tma, true, 16, smem1, m.x, m.b, m.e); break;
        case 4: ARTSS_SWEEP_TMA(k_cgs_sweep_tma, false, 32, smem1, m.x, m.b, m.e); break;
        case 5: ARTSS_SWEEP_TMA(k_cgs_sweep_tma, true, 32, smem1, m.x, m.b, m.e); break;
        case 6: ARTSS_SWEEP_TMA(k_cgs_sweep_tma2, false, 8, smem2, m.x2, m.b2, m.e2); break;
        case 7: ARTSS_SWEEP_TMA(k_cgs_sweep_tma2, true, 8, smem2, m.x2, m.b2, m.e2); break;
        case 8: ARTSS_SWEEP_TMA(k_cgs_sweep_tma2, false, 16, smem2, m.x2, m.b2, m.e2); break;
        case 9: ARTSS_SWEEP_TMA(k_cgs_sweep_tma2, true, 16, smem2, m.x2, m.b2, m.e2); break;
        case 10: ARTSS_SWEEP_TMA(k_cgs_sweep_tma2, false, 32, smem2, m.x2, m.b2, m.e2); break;
        default: ARTSS_SWEEP_TMA(k_cgs_sweep_tma2, true, 32, smem2, m.x2, m.b2, m.e2); break;
    }
#undef ARTSS_SWEEP_TMA
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

int set_sweep_smem(bool turb) {
    static bool done[2] = {false, false};
    if (done[turb]) return ARTSS_OK;
    const int b1 = (int) sweep_tma_smem(turb), b2 = (int) sweep_tma2_smem(turb);
    const auto attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
    const int b3 = (int) S3Tall::smem(turb), b4 = (int) S3Flat::smem(turb);
    const int b6 = (int) S3Wide::smem(turb);
    if (turb) {
        ARTSS_CK(cudaFuncSetAttribute(k_cgs_sweep3<true, S3Tall>, attr, b3));
        ARTSS_CK(cudaFuncSetAttribute(k_cgs_sweep3<true, S3Flat>, attr, b4));
        ARTSS_CK(cudaFuncSetAttribute(k_cgs_sweep3<true, S3Wide>, attr, b6));
        ARTSS_CK(cudaFuncSetAttribute(k_cgs_sweep_tma<true, 8>, attr, b1));
        ARTSS_CK(cudaFuncSetAttribute(k_cgs_sweep_tma<true, 16>, attr, b1));
        ARTSS_CK(cudaFuncSetAttribute(k_cgs_sweep_tma<true, 32>, attr, b1));
        ARTSS_CK(cudaFuncSetAttribute(k_cgs_sweep_tma2<true, 8>, attr, b2));
        ARTSS_CK(cudaFuncSetAttribute(k_cgs_sweep_tma2<true, 16>, attr, b2));
        ARTSS_CK(cudaFuncSetAttribute(k_cgs_sweep_tma2<true, 32>, attr, b2));
    } else {
        ARTSS_CK(cudaFuncSetAttribute(k_cgs_sweep3<false, S3Tall>, attr, b3));
        ARTSS_CK(cudaFuncSetAttribute(k_cgs_sweep3<false, S3Flat>, attr, b4));
        ARTSS_CK(cudaFuncSetAttribute(k_cgs_sweep3<false, S3Wide>, attr, b6));
        ARTSS_CK(cudaFuncSetAttribute(k_cgs_sweep_tma<false, 8>, attr, b1));
        ARTSS_CK(cudaFuncSetAttribute(k_cgs_sweep_tma<false, 16>, attr, b1));
        ARTSS_CK(cudaFuncSetAttribute(k_cgs_sweep_tma<false, 32>, attr, b1));
        ARTSS_CK(cudaFuncSetAttribute(k_cgs_sweep_tma2<false, 8>, attr, b2));
        ARTSS_CK(cudaFuncSetAttribute(k_cgs_sweep_tma2<false, 16>, attr, b2));
        ARTSS_CK(cudaFuncSetAttribute(k_cgs_sweep_tma2<false, 32>, attr, b2));
    }
    done[turb] = true;
    return ARTSS_OK;
}

// Autotuner of the sweep: the first solve on a level shape times every
// variant (kernel and z-depth) on that solve's first iteration (the sweep
// reads `rd`, b, EV and writes only `w` and the partials, so repeating it
// changes nothing) and keeps the fastest for the context.
int tune_sweep(artss_ctx *ctx, bool turb, bool one_phase, const Box3 &box, const SweepMaps &m, double *w,
               const Level &L, const DiffCoef &c, LoopState *pred, int *choice) {
    if (ctx->sweep_force >= 0) {
        if (ctx->sweep_force >= 3 && !one_phase) {
            set_error("sweep variant needs an inner box starting at an odd x");
            return ARTSS_ERR_ARG;
        }
        *choice = ctx->sweep_force;
        return ARTSS_OK;
    }
    const TuneKey key{0, L.Nx, L.Ny, L.Nz, turb ? 1 : 0};
    auto it = ctx->tuned.find(key);
    if (it != ctx->tuned.end() && (one_phase || it->second < 3)) { *choice = it->second; return ARTSS_OK; }
    const int fallback = one_phase ? kSweepRowPair : 1;
    if (!ctx->autotune || ctx->capturing) { *choice = fallback; return ARTSS_OK; }
    cudaEvent_t e0, e1;
    ARTSS_CK(cudaEventCreate(&e0));
    ARTSS_CK(cudaEventCreate(&e1));
    int best = fallback, st = ARTSS_OK, nb = 0;
    float best_ms = 1e30f;
    for (int v = 0; v < (one_phase ? kSweepVariants : 3) && !st; v++) {
        if ((st = launch_sweep_tma(ctx, turb, v, box, m, w, L, c, pred, &nb))) break;  // warm
        cudaEventRecord(e0, ctx->stream);
        for (int r = 0; r < 3 && !st; r++) st = launch_sweep_tma(ctx, turb, v, box, m, w, L, c, pred, &nb);
        cudaEventRecord(e1, ctx->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) { st = cuda_fail(cudaGetLastError(), "autotune"); break; }
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) { best_ms = ms; best = v; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    ctx->tuned[key] = best;
    *choice = best;
    return ARTSS_OK;
}

}  // namespace

int artss_ctx_autotune(artss_ctx *ctx, int enable) {
    if (!ctx) { set_error("null argument"); return ARTSS_ERR_ARG; }
    ctx->autotune = enable != 0;
    if (!enable) ctx->tuned.clear();
    return ARTSS_OK;
}

int artss_ctx_pdl(artss_ctx *ctx, int enable) {
    if (!ctx) { set_error("null argument"); return ARTSS_ERR_ARG; }
    if (enable < 0 || enable > 2) { set_error("pdl mode is 0, 1 or 2"); return ARTSS_ERR_ARG; }
    ctx->pdl = enable;
    return ARTSS_OK;
}

int artss_ctx_sweep_variant(artss_ctx *ctx, int variant) {
    if (!ctx) { set_error("null argument"); return ARTSS_ERR_ARG; }
    if (variant < -1 || variant >= kSweepVariants) { set_error("sweep variant is -1 .. 8"); return ARTSS_ERR_ARG; }
    ctx->sweep_force = variant;
    return ARTSS_OK;
}

int artss_cgs_sweep_variant(artss_ctx *ctx, int turbulent) {
    if (!ctx) return -1;
    const Level &L = ctx->lvl[0];
    auto it = ctx->tuned.find(TuneKey{0, L.Nx, L.Ny, L.Nz, turbulent ? 1 : 0});
    return it == ctx->tuned.end() ? -1 : it->second;
}

int artss_cgs_sweep_depth(artss_ctx *ctx, int turbulent) {
    if (!ctx) return 0;
    const Level &L = ctx->lvl[0];
    auto it = ctx->tuned.find(TuneKey{0, L.Nx, L.Ny, L.Nz, turbulent ? 1 : 0});
    return it == ctx->tuned.end() ? 0 : it->second >= kSweepRowPair ? -1 : kStDepths[it->second % 3];
}

int artss_diffuse_cgs(artss_ctx *ctx, double *out, double *in, const double *b, double D, const double *ev,
                      double dt, int field_type, const artss_iter_cfg *cfg, int flags,
                      artss_iter_stats *stats) {
    const int in_is_scratch = flags & ARTSS_DIFFUSE_IN_SCRATCH;
    int st = check_field_args(ctx, {out, in, b, cfg});
    if (st || (st = check_field_type(field_type))) return st;
    if (cfg->max_iter < 0) { set_error("max_iter < 0"); return ARTSS_ERR_ARG; }
    if (out == in || b == out || b == in) { set_error("out, in and b must be distinct arrays"); return ARTSS_ERR_ARG; }
    const Level &L = ctx->lvl[0];
    const Box3 box = inner_box(L);
    const dim3 g = sweep_grid(box);
    if ((st = check_reduce_blocks(g))) return st;
    if ((st = check_reduce_blocks(sweep_tma_grid(box, kStDepths[0])))) return st;
    int nb = nblocks(g);
    // TMA plane staging where the row pitch allows it, cp.async otherwise
    const bool tma = tma_level_ok(ctx, 0) && L.size() < ((int64_t) 1 << 31);
    const size_t smem = tma ? sweep_tma_smem(ev != nullptr) : sweep_smem(ev != nullptr);
    if (tma) {
        if ((st = set_sweep_smem(ev != nullptr))) return st;
    } else {
        if (ev) ARTSS_CK(cudaFuncSetAttribute(k_cgs_sweep<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
        else ARTSS_CK(cudaFuncSetAttribute(k_cgs_sweep<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    }
    // one-phase kernel: its b / EV window starts at an even x when the inner box starts at an odd one
    const bool one_phase = tma && (box.x0 & 1) == 1;
    SweepMaps maps[2];  // by the array read: buf[0] = out, buf[1] = in
    const DiffCoef c = diff_coef(ctx, D, dt, cfg->w, 1.0);
    // out.copy_data(in) (ColoredGaussSeidelDiffuse.cpp:41,114), unless out holds in already
    if (!(flags & ARTSS_DIFFUSE_OUT_HOLDS_IN) && (st = artss_copy(ctx, out, in, 0))) return st;
    const int slot = 0;
    // while (res > tol_res && it < max_iter), res starts at 1
    long long it = 0;
    double res = 1.;
    bool cond = res > cfg->tol_res && it < cfg->max_iter;
    if ((st = init_loop(ctx, slot, res, 0, cond ? 1 : 0))) return st;
    LoopState ls{};
    const LoopState *pred = ctx->d_loop + slot;
    int64_t batch = std::max<int64_t>(1, std::min<int64_t>(loop_hint(ctx, 0, field_type), cfg->max_iter));
    // The reference sweeps `out` in place after in.copy_data(out) (:69-76); here
    // iteration n reads iterate n-1 from one of {out, in} and writes iterate n
    // into the other, so after n iterations the two arrays hold exactly what the
    // reference's out and in hold, possibly exchanged.  The first direction is
    // chosen so that a solve of the predicted length ends in out.
    double *buf[2] = {out, in};
    const int s0 = (int) (batch & 1);  // iteration n writes buf[(s0 + n) & 1]
    if (tma) {
        for (int r = 0; r < 2; r++) {
            SweepMaps &m = maps[r];
            if ((st = tensor_map_3d(ctx, buf[r], 0, &m.x))) return st;
            if ((st = tensor_map_3d(ctx, b, 0, &m.b))) return st;
            m.e = m.b;
            if (ev && (st = tensor_map_3d(ctx, ev, 0, &m.e))) return st;
            if (one_phase) {
                if ((st = tensor_map_3d(ctx, buf[r], 0, &m.x2, kSt2BoxX, kTmaBoxY))) return st;
                if ((st = tensor_map_3d(ctx, b, 0, &m.b2, kSt2BoxBX, kSt2BoxBY))) return st;
                m.e2 = m.b2;
                if (ev && (st = tensor_map_3d(ctx, ev, 0, &m.e2, kSt2BoxBX, kSt2BoxBY))) return st;
                if ((st = tensor_map_3d(ctx, buf[r], 0, &m.x3, S3Flat::XW, S3Flat::XH))) return st;
                if ((st = tensor_map_3d(ctx, b, 0, &m.b3, S3Flat::BW, S3Flat::BH))) return st;
                m.e3 = m.b3;
                if (ev && (st = tensor_map_3d(ctx, ev, 0, &m.e3, S3Flat::BW, S3Flat::BH))) return st;
                if ((st = tensor_map_3d(ctx, buf[r], 0, &m.x4, S3Wide::XW, S3Wide::XH))) return st;
                if ((st = tensor_map_3d(ctx, b, 0, &m.b4, S3Wide::BW, S3Wide::BH))) return st;
                m.e4 = m.b4;
                if (ev && (st = tensor_map_3d(ctx, ev, 0, &m.e4, S3Wide::BW, S3Wide::BH))) return st;
            }
        }
    }
    LoopState *pred_rw = ctx->d_loop + slot;
    int depth = 1;  // the sweep variant (launch_sweep_tma)
    if (tma && cond) {
        const int n1 = (s0 + 1) & 1;
        if ((st = tune_sweep(ctx, ev != nullptr, one_phase, box, maps[1 - n1], buf[n1], L, c, pred_rw, &depth)))
            return st;
    }
    if (ctx->capturing) {
        // a WHILE node whose body is two iterations (the second writes back into
        // the first's source); the loop state decides on the device
        if (cond) {
            GraphLoop gl;
            if ((st = gl.begin(ctx, 1))) return st;
            for (int n = 1; n <= 2; n++) {
                double *w = buf[(s0 + n) & 1];
                const double *rd = buf[(s0 + n + 1) & 1];
                if (tma) {
                    if ((st = launch_sweep_tma(ctx, ev != nullptr, depth, box, maps[(s0 + n + 1) & 1], w, L, c,
                                               pred_rw, &nb)))
                        return st;
                } else if (ev)
                    ARTSS_LAUNCH(ctx, FAM_CGS, k_cgs_sweep<true><<<g, dim3(kSwTx / 2, kSwTy), smem, ctx->stream>>>(
                        w, rd, b, ev, ctx->d_flags[0], L, box, c, ctx->d_partials, pred));
                else
                    ARTSS_LAUNCH(ctx, FAM_CGS, k_cgs_sweep<false><<<g, dim3(kSwTx / 2, kSwTy), smem, ctx->stream>>>(
                        w, rd, b, nullptr, ctx->d_flags[0], L, box, c, ctx->d_partials, pred));
                if (!tma) ARTSS_LAUNCH_CK(ctx);
                if ((st = apply_bc(ctx, w, 0, field_type, pred))) return st;
                if ((st = finalize_loop(ctx, slot, nb, cfg->tol_res, cfg->max_iter))) return st;
            }
            if ((st = gl.end(slot, cfg->max_iter / 2 + 2))) return st;
            const int64_t n = L.size();
            ARTSS_LAUNCH(ctx, FAM_FIELD_OP, k_cgs_fixup<<<flat_blocks(n), 256, 0, ctx->stream>>>(
                                                out, in, ctx->d_loop + slot, s0, in_is_scratch, n));
            ARTSS_LAUNCH_CK(ctx);
        }
        if (stats) { stats->iterations = -1; stats->residual = -1.0; }
        return ARTSS_OK;
    }
    while (cond) {
        // `batch` iterations per host round trip; iterations past convergence skip themselves
        for (int64_t r = 0; r < batch; r++) {
            const long long n = it + 1 + r;
            double *w = buf[(s0 + n) & 1];
            const double *rd = buf[(s0 + n + 1) & 1];
            if (tma) {
                if ((st = launch_sweep_tma(ctx, ev != nullptr, depth, box, maps[(s0 + n + 1) & 1], w, L, c, pred_rw,
                                           &nb)))
                    return st;
            } else if (ev)
                ARTSS_LAUNCH(ctx, FAM_CGS, k_cgs_sweep<true><<<g, dim3(kSwTx / 2, kSwTy), smem, ctx->stream>>>(
                    w, rd, b, ev, ctx->d_flags[0], L, box, c, ctx->d_partials, pred));
            else
                ARTSS_LAUNCH(ctx, FAM_CGS, k_cgs_sweep<false><<<g, dim3(kSwTx / 2, kSwTy), smem, ctx->stream>>>(
                    w, rd, b, nullptr, ctx->d_flags[0], L, box, c, ctx->d_partials, pred));
            if (!tma) ARTSS_LAUNCH_CK(ctx);
            if ((st = apply_bc(ctx, w, 0, field_type, pred))) return st;
            if ((st = finalize_loop(ctx, slot, nb, cfg->tol_res, cfg->max_iter))) return st;
        }
        if ((st = read_loop(ctx, slot, &ls))) return st;
        if (ls.pad) { set_error("colored Gauss-Seidel sweep: a TMA plane load did not arrive"); return ARTSS_ERR_CUDA; }
        it = ls.it;
        res = ls.residual;
        cond = ls.cond != 0;
        batch = std::min<int64_t>(2 * batch, std::max<int64_t>(1, cfg->max_iter - it));
    }
    if (it > 0 && ((s0 + it) & 1)) {
        // the last iterate sits in `in`: exchange (the caller keeps in) or copy back
        const int64_t n = L.size();
        if (in_is_scratch) {
            if ((st = artss_copy(ctx, out, in, 0))) return st;
        } else {
            ARTSS_LAUNCH(ctx, FAM_FIELD_OP, k_swap<<<flat_blocks(n), 256, 0, ctx->stream>>>(out, in, n));
            ARTSS_LAUNCH_CK(ctx);
        }
    }
    loop_hint(ctx, 0, field_type) = std::max<int64_t>(1, it);
    if (stats) { stats->iterations = it; stats->residual = res; }
    return ARTSS_OK;
}

int artss_diffuse_cgs_mixed(artss_ctx *ctx, double *out, double *in, const double *b, double D, const double *ev,
                            double dt, int field_type, const artss_iter_cfg *cfg, int flags,
                            artss_iter_stats *stats) {
    int st = check_field_args(ctx, {out, in, b, cfg});
    if (st || (st = check_field_type(field_type))) return st;
    if (cfg->max_iter < 0) { set_error("max_iter < 0"); return ARTSS_ERR_ARG; }
    if (cfg->w != 1.0) { set_error("the defect-correction sweep reproduces the relaxation weight 1 only"); return ARTSS_ERR_ARG; }
    if (out == in || b == out || b == in) { set_error("out, in and b must be distinct arrays"); return ARTSS_ERR_ARG; }
    if (ctx->capturing) { set_error("the mixed-precision diffusion is not captured into graphs"); return ARTSS_ERR_STATE; }
    const Level &L = ctx->lvl[0];
    const Box3 box = inner_box(L);
    const dim3 g = zgrid(box);
    if ((st = check_reduce_blocks(g))) return st;
    const int nb = nblocks(g);
    if (!ctx->cgsm_w || ctx->cgsm_n != L.size()) {
        if (ctx->cgsm_w) cudaFree(ctx->cgsm_w);
        ctx->cgsm_w = nullptr;
        ARTSS_CK(cudaMalloc(&ctx->cgsm_w, (size_t) L.size() * sizeof(float)));
        ctx->cgsm_n = L.size();
    }
    float *wv = ctx->cgsm_w;
    const DiffCoef c = diff_coef(ctx, D, dt, cfg->w, 1.0);
    // out.copy_data(in) (ColoredGaussSeidelDiffuse.cpp:41,114)
    if (!(flags & ARTSS_DIFFUSE_OUT_HOLDS_IN) && (st = artss_copy(ctx, out, in, 0))) return st;
    const int slot = 0;
    long long it = 0;
    double res = 1.;
    bool cond = res > cfg->tol_res && it < cfg->max_iter;
    if ((st = init_loop(ctx, slot, res, 0, cond ? 1 : 0))) return st;
    LoopState ls{};
    const LoopState *pred = ctx->d_loop + slot;
    int64_t batch = std::max<int64_t>(1, std::min<int64_t>(loop_hint(ctx, 2, field_type), cfg->max_iter));
    while (cond) {
        for (int64_t r = 0; r < batch; r++) {
            if (ev) {
                ARTSS_LAUNCH_PDL(ctx, FAM_CGS, k_cgsm_defect<true>, g, box_block(), 0, wv, (const double *) out, b, ev,
                                 (const uint8_t *) ctx->d_flags[0], L, box, c, pred);
                ARTSS_LAUNCH_PDL(ctx, FAM_CGS, k_cgsm_correct<true>, g, box_block(), 0, out, (const float *) wv, ev,
                                 (const uint8_t *) ctx->d_flags[0], L, box, c, ctx->d_partials, pred);
            } else {
                ARTSS_LAUNCH_PDL(ctx, FAM_CGS, k_cgsm_defect<false>, g, box_block(), 0, wv, (const double *) out, b,
                                 (const double *) nullptr, (const uint8_t *) ctx->d_flags[0], L, box, c, pred);
                ARTSS_LAUNCH_PDL(ctx, FAM_CGS, k_cgsm_correct<false>, g, box_block(), 0, out, (const float *) wv,
                                 (const double *) nullptr, (const uint8_t *) ctx->d_flags[0], L, box, c,
                                 ctx->d_partials, pred);
            }
            ARTSS_LAUNCH_CK(ctx);
            if ((st = apply_bc(ctx, out, 0, field_type, pred))) return st;
            if ((st = finalize_loop(ctx, slot, nb, cfg->tol_res, cfg->max_iter))) return st;
        }
        if ((st = read_loop(ctx, slot, &ls))) return st;
        it = ls.it;
        res = ls.residual;
        cond = ls.cond != 0;
        batch = std::min<int64_t>(2 * batch, std::max<int64_t>(1, cfg->max_iter - it));
    }
    loop_hint(ctx, 2, field_type) = std::max<int64_t>(1, it);
    // the reference leaves in = out after every iteration (:79)
    if (!(flags & ARTSS_DIFFUSE_IN_SCRATCH) && (st = artss_copy(ctx, in, out, 0))) return st;
    if (stats) { stats->iterations = it; stats->residual = res; }
    return ARTSS_OK;
}

int artss_diffuse_jacobi(artss_ctx *ctx, double *out, double *in, const double *b, double D, const double *ev,
                         double dt, int field_type, const artss_iter_cfg *cfg, artss_iter_stats *stats) {
    int st = check_field_args(ctx, {out, in, b, cfg});
    if (st || (st = check_field_type(field_type))) return st;
    if (cfg->max_iter < 0) { set_error("max_iter < 0"); return ARTSS_ERR_ARG; }
    const Level &L = ctx->lvl[0];
    const Box3 box = inner_box(L);
    const Box3 dbox = domain_box(L);
    const dim3 g = zgrid(box);
    if ((st = check_reduce_blocks(g))) return st;
    const int nb = nblocks(g);
    const DiffCoef c = diff_coef(ctx, D, dt, cfg->w, 1.0);
    const int slot = 0;
    long long it = 0;
    double res = 1.;
    bool cond = res > cfg->tol_res && it < cfg->max_iter;
    if ((st = init_loop(ctx, slot, res, 0, cond ? 1 : 0))) return st;
    LoopState ls{};
    const LoopState *pred = ctx->d_loop + slot;
    int64_t batch = std::max<int64_t>(1, std::min<int64_t>(loop_hint(ctx, 1, field_type), cfg->max_iter));
    GraphLoop gl;
    if (ctx->capturing) {
        // one iteration per body of a WHILE node decided on the device
        if (!cond) {
            if (stats) { stats->iterations = 0; stats->residual = res; }
            return ARTSS_OK;
        }
        if ((st = gl.begin(ctx, 1))) return st;
        batch = 1;
    }
    while (cond) {
        for (int64_t r = 0; r < batch; r++) {
            if (ev)
                ARTSS_LAUNCH(ctx, FAM_JACOBI, k_jacobi_diffuse<true><<<g, box_block(), 0, ctx->stream>>>(
                    out, in, b, ev, ctx->d_flags[0], L, box, c, ctx->d_partials, pred));
            else
                ARTSS_LAUNCH(ctx, FAM_JACOBI, k_jacobi_diffuse<false><<<g, box_block(), 0, ctx->stream>>>(
                    out, in, b, nullptr, ctx->d_flags[0], L, box, c, ctx->d_partials, pred));
            ARTSS_LAUNCH_CK(ctx);
            if ((st = apply_bc(ctx, out, 0, field_type, pred))) return st;
            // in = out before the loop decision: the residual partials are already taken
            ARTSS_LAUNCH(ctx, FAM_COPY_DOMAIN, k_copy_domain<<<zgrid(dbox), box_block(), 0, ctx->stream>>>(
                in, out, ctx->d_flags[0], L, dbox, pred));
            ARTSS_LAUNCH_CK(ctx);
            if ((st = finalize_loop(ctx, slot, nb, cfg->tol_res, cfg->max_iter))) return st;
        }
        if (ctx->capturing) {
            if ((st = gl.end(slot, cfg->max_iter + 2))) return st;
            if (stats) { stats->iterations = -1; stats->residual = -1.0; }
            return ARTSS_OK;
        }
        if ((st = read_loop(ctx, slot, &ls))) return st;
        it = ls.it;
        res = ls.residual;
        cond = ls.cond != 0;
        batch = std::min<int64_t>(2 * batch, std::max<int64_t>(1, cfg->max_iter - it));
    }
    loop_hint(ctx, 1, field_type) = std::max<int64_t>(1, it);
    // the final odd-count copy of JacobiDiffuse.cpp:92-99 repeats the last
    // in = out over the domain list and changes nothing
    if (stats) { stats->iterations = it; stats->residual = res; }
    return ARTSS_OK;
}

}  // extern "C"
