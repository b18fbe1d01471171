// Residual norm that allocates nothing.
//
// Some callers cannot allocate device memory at the point where they need a
// residual: code running inside a memory pool that must not grow, or a host
// application whose allocator owns the device (a coupled solver that hands us
// only its arrays).  For them artss_residual_norm_static computes the same
// ||b - A p||_2 and ||b||_2 as artss_residual_norm without a context: the
// per-block partial sums go to the fixed array below, which every GPU that
// loads this library keeps until the process exits.  The call waits for its
// result, so it refuses a stream that is being captured into a graph.
//
// Host code cannot use `g_static_partials` as a device address (it names a
// host-side shadow); the device address is looked up once per device with
// cudaGetSymbolAddress on the first call made with that device current, and
// kept for the life of the process: after a cudaDeviceReset of that device
// the kept address is stale, so the entry point must not be used across one.
#include "internal.cuh"

#include <cmath>
#include <mutex>

namespace artss {

constexpr int kStaticPartials = 8192;  // blocks per call; two sums per block + 2 results
static __device__ __align__(256) double g_static_partials[2 * kStaticPartials + 2];

constexpr int kStaticMaxDevices = 64;
static double *g_static_ptr[kStaticMaxDevices] = {};
static std::mutex g_static_mutex;

// ||b - A p||^2 and ||b||^2 partial sums of one block, cells of the
// computational domain whose flag has bit 0 set (all of them when flags == NULL)
__global__ void k_static_resnorm(const double *__restrict__ p, const double *__restrict__ b,
                                 const uint8_t *__restrict__ flags, Level L, Box3 box, double rx, double ry, double rz,
                                 double *__restrict__ partials) {
    __shared__ double smem[32];
    const int64_t i = box.x0 + (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t j = box.y0 + (int64_t) blockIdx.y * blockDim.y + threadIdx.y;
    const int64_t nj = L.Nx, nk = L.Nx * L.Ny;
    double acc = 0.0, accb = 0.0;
    if (i <= box.x1 && j <= box.y1) {
        for (int64_t k = box.z0 + blockIdx.z; k <= box.z1; k += gridDim.z) {
            const int64_t q = i + nj * j + nk * k;
            if (flags && !(flags[q] & kInner)) continue;
            const double r = b[q] - (rx * (p[q - 1] - 2 * p[q] + p[q + 1]) + ry * (p[q - nj] - 2 * p[q] + p[q + nj]) +
                                     rz * (p[q - nk] - 2 * p[q] + p[q + nk]));
            acc += r * r;
            accb += b[q] * b[q];
        }
    }
    const int bl = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    const int nb = gridDim.x * gridDim.y * gridDim.z;
    acc = artss_block_sum(acc, smem);
    if (threadIdx.x == 0 && threadIdx.y == 0) partials[bl] = acc;
    __syncthreads();
    accb = artss_block_sum(accb, smem);
    if (threadIdx.x == 0 && threadIdx.y == 0) partials[nb + bl] = accb;
}

// sums the partials in a fixed order; results at partials[2 * kStaticPartials + {0, 1}]
__global__ void k_static_finalize(double *__restrict__ partials, int nb) {
    __shared__ double smem[32];
    double a = 0.0, c = 0.0;
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
        a += partials[k];
        c += partials[nb + k];
    }
    a = artss_block_sum(a, smem);
    __syncthreads();
    c = artss_block_sum(c, smem);
    if (threadIdx.x == 0) {
        partials[2 * kStaticPartials] = sqrt(a);
        partials[2 * kStaticPartials + 1] = sqrt(c);
    }
}

static int static_scratch(double **out) {
    int dev = 0;
    ARTSS_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kStaticMaxDevices) { set_error("device ordinal beyond the static table"); return ARTSS_ERR_LIMIT; }
    std::lock_guard<std::mutex> lock(g_static_mutex);
    if (!g_static_ptr[dev]) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_partials);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_static_partials)");
        g_static_ptr[dev] = static_cast<double *>(ptr);
    }
    *out = g_static_ptr[dev];
    return ARTSS_OK;
}

}  // namespace artss

using namespace artss;

extern "C" int artss_residual_norm_static(const artss_grid_desc *grid, const uint8_t *flags, const double *p,
                                          const double *b, void *stream, double *res_out, double *b_norm_out) {
    if (!grid || !p || !b || !res_out || !b_norm_out) { set_error("null argument"); return ARTSS_ERR_ARG; }
    const Level L{grid->Nx[0], grid->Ny[0], grid->Nz[0], grid->i1[0], grid->i2[0],
                  grid->j1[0], grid->j2[0], grid->k1[0], grid->k2[0]};
    if (L.Nx < 3 || L.Ny < 3 || L.Nz < 3 || L.i1 < 1 || L.i2 > L.Nx - 2 || L.i1 > L.i2 || L.j1 < 1 ||
        L.j2 > L.Ny - 2 || L.j1 > L.j2 || L.k1 < 1 || L.k2 > L.Nz - 2 || L.k1 > L.k2) {
        set_error("inconsistent grid description");
        return ARTSS_ERR_ARG;
    }
    const double dx = grid->dx[0], dy = grid->dy[0], dz = grid->dz[0];
    if (!(dx > 0.0) || !(dy > 0.0) || !(dz > 0.0) || !std::isfinite(dx) || !std::isfinite(dy) ||
        !std::isfinite(dz)) {
        set_error("cell spacing must be positive and finite");
        return ARTSS_ERR_ARG;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    ARTSS_CK(cudaStreamIsCapturing(s, &cap));
    if (cap != cudaStreamCaptureStatusNone) {
        set_error("artss_residual_norm_static waits for its result and cannot run on a capturing stream");
        return ARTSS_ERR_ARG;
    }
    const Box3 box{L.i1, L.i2, L.j1, L.j2, L.k1, L.k2};
    dim3 g = box_grid(box);
    const int64_t xy = (int64_t) g.x * g.y;
    if (xy > kStaticPartials) {
        set_error("grid too large for artss_residual_norm_static: more than " + std::to_string(kStaticPartials) +
                  " tiles of 64x4 cells in an x-y plane");
        return ARTSS_ERR_LIMIT;
    }
    g.z = (unsigned) std::min<int64_t>(box.nz(), std::max<int64_t>(1, kStaticPartials / xy));
    const int nb = (int) (xy * g.z);
    double *scratch = nullptr;
    int st = static_scratch(&scratch);
    if (st) return st;
    k_static_resnorm<<<g, box_block(), 0, s>>>(p, b, flags, L, box, 1. / (dx * dx), 1. / (dy * dy), 1. / (dz * dz),
                                               scratch);
    ARTSS_CK(cudaGetLastError());
    k_static_finalize<<<1, kReduceThreads, 0, s>>>(scratch, nb);
    ARTSS_CK(cudaGetLastError());
    double out[2];
    ARTSS_CK(cudaMemcpyAsync(out, scratch + 2 * kStaticPartials, sizeof(out), cudaMemcpyDeviceToHost, s));
    ARTSS_CK(cudaStreamSynchronize(s));
    *res_out = out[0];
    *b_norm_out = out[1];
    return ARTSS_OK;
}
