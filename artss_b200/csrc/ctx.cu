// Context, device memory, cell flags and whole-array field operations.
#include "internal.cuh"

#include <algorithm>
#include <cstdio>
#include <cstring>

namespace artss {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

int cuda_fail(cudaError_t e, const char *what) {
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    // a failed runtime call also sets the thread's last error; clear it so the
    // next launch check does not report it again (sticky errors stay)
    (void) cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? ARTSS_ERR_NOMEM
         : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? ARTSS_ERR_NO_DEVICE
         : ARTSS_ERR_CUDA;
}

int check_level(const artss_ctx *ctx, int level) {
    if (!ctx) { set_error("null context"); return ARTSS_ERR_ARG; }
    if (level < 0 || level > ctx->grid.n_levels) {
        set_error("level " + std::to_string(level) + " outside 0.." + std::to_string(ctx->grid.n_levels));
        return ARTSS_ERR_ARG;
    }
    return ARTSS_OK;
}

int check_field_type(int ft) {
    if (ft < 0 || ft >= kFieldTypes) { set_error("unknown field type " + std::to_string(ft)); return ARTSS_ERR_ARG; }
    return ARTSS_OK;
}

// ---------------------------------------------------------------- kernels

__global__ void k_fill(double *__restrict__ f, int64_t n, double v) {
    artss::pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    artss::pdl_trigger();
    for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
        f[i] = v;
}

__global__ void k_copy(double *__restrict__ d, const double *__restrict__ s, int64_t n) {
    artss::pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    artss::pdl_trigger();
    for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
        d[i] = s[i];
}

__global__ void k_add_field(double *__restrict__ d, const double *__restrict__ s, int64_t n) {
    artss::pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    artss::pdl_trigger();
    for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
        d[i] += s[i];
}

__global__ void k_add_scalar(double *__restrict__ d, double x, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
        d[i] += x;
}

__global__ void k_scale(double *__restrict__ d, double x, int64_t n) {
    artss::pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    artss::pdl_trigger();
    for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
        d[i] *= x;
}

__global__ void k_scale_copy(double *__restrict__ d, const double *__restrict__ s, double x, int64_t n) {
    artss::pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    artss::pdl_trigger();
    for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
        d[i] = s[i] * x;
}

// a0 = a (unless a0 is null), a_tmp = a for up to three vectors in one pass
// (couple_vector).
__global__ void k_couple3(const double *__restrict__ a, double *__restrict__ a0, double *__restrict__ at,
                          const double *__restrict__ b, double *__restrict__ b0, double *__restrict__ bt,
                          const double *__restrict__ c, double *__restrict__ c0, double *__restrict__ ct,
                          int64_t n) {
    artss::pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    artss::pdl_trigger();
    for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
        if (a) { const double x = a[i]; if (a0) a0[i] = x; at[i] = x; }
        if (b) { const double x = b[i]; if (b0) b0[i] = x; bt[i] = x; }
        if (c) { const double x = c[i]; if (c0) c0[i] = x; ct[i] = x; }
    }
}

// Mark the cells of a sorted index list with `bit`.
__global__ void k_mark(uint8_t *__restrict__ flags, const int64_t *__restrict__ list, int64_t n, uint8_t bit) {
    for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
        flags[list[i]] |= bit;
}

cudaEvent_t prof_event(artss_ctx *ctx) {
    Profile &p = ctx->prof;
    if (!p.pool.empty()) {
        cudaEvent_t e = p.pool.back();
        p.pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
}

static const char *const kFamilyNames[FAM_COUNT] = {
    "advect", "smagorinsky", "divergence", "projection", "buoyancy", "add_source", "cgs_sweep",
    "jacobi_diffuse", "copy_domain", "bc_wave", "field_op", "couple", "mg_jacobi", "mg_cgs", "mg_residuum",
    "mg_restrict", "mg_prolongate", "mg_resnorm", "reduce", "mg_coarse", "conv3d", "nn_elementwise"};

}  // namespace artss

using namespace artss;

extern "C" {

const char *artss_last_error(void) { return g_last_error.c_str(); }

const char *artss_kernel_family_name(int family) {
    return family >= 0 && family < FAM_COUNT ? kFamilyNames[family] : "";
}

int artss_ctx_profile(artss_ctx *ctx, uint64_t mask) {
    if (!ctx) { set_error("null context"); return ARTSS_ERR_ARG; }
    ctx->prof.mask = mask;
    return ARTSS_OK;
}

int artss_ctx_profile_reset(artss_ctx *ctx) {
    if (!ctx) { set_error("null context"); return ARTSS_ERR_ARG; }
    ARTSS_CK(cudaStreamSynchronize(ctx->stream));
    Profile &p = ctx->prof;
    for (auto &pe : p.pending) p.pool.push_back(pe.first);
    for (auto e : p.events) p.pool.push_back(e);
    p.pending.clear();
    p.events.clear();
    for (int f = 0; f < FAM_COUNT; f++) { p.launches[f] = 0; p.ms[f] = 0.0; }
    return ARTSS_OK;
}

int artss_ctx_profile_read(artss_ctx *ctx, int64_t *launches, double *ms, int n_families) {
    if (!ctx) { set_error("null context"); return ARTSS_ERR_ARG; }
    ARTSS_CK(cudaStreamSynchronize(ctx->stream));
    Profile &p = ctx->prof;
    for (size_t q = 0; q < p.pending.size(); q++) {
        float t = 0.f;
        ARTSS_CK(cudaEventElapsedTime(&t, p.pending[q].first, p.events[q]));
        p.ms[p.pending[q].second] += t;
        p.pool.push_back(p.pending[q].first);
        p.pool.push_back(p.events[q]);
    }
    p.pending.clear();
    p.events.clear();
    for (int f = 0; f < n_families && f < FAM_COUNT; f++) {
        if (launches) launches[f] = p.launches[f];
        if (ms) ms[f] = p.ms[f];
    }
    return ARTSS_OK;
}

int artss_ctx_stage_timing(artss_ctx *ctx, int enable) {
    if (!ctx) { set_error("null context"); return ARTSS_ERR_ARG; }
    ARTSS_CK(cudaStreamSynchronize(ctx->stream));
    Profile &p = ctx->prof;
    for (auto &m : p.marks) p.pool.push_back(m.first);
    p.marks.clear();
    for (int s = 0; s < ARTSS_STAGES; s++) p.stage_ms[s] = 0.0;
    p.stages = enable != 0;
    return ARTSS_OK;
}

int artss_ctx_stage_mark(artss_ctx *ctx, int stage) {
    if (!ctx) { set_error("null context"); return ARTSS_ERR_ARG; }
    if (stage < ARTSS_STAGE_END || stage >= ARTSS_STAGES) { set_error("stage out of range"); return ARTSS_ERR_ARG; }
    Profile &p = ctx->prof;
    if (!p.stages || ctx->capturing) return ARTSS_OK;
    cudaEvent_t e = prof_event(ctx);
    if (!e) { set_error("cudaEventCreate failed"); return ARTSS_ERR_CUDA; }
    ARTSS_CK(cudaEventRecord(e, ctx->stream));
    p.marks.push_back({e, stage});
    return ARTSS_OK;
}

int artss_ctx_stage_read(artss_ctx *ctx, double *ms, int n_stages) {
    if (!ctx) { set_error("null context"); return ARTSS_ERR_ARG; }
    ARTSS_CK(cudaStreamSynchronize(ctx->stream));
    Profile &p = ctx->prof;
    // the interval from one mark to the next belongs to the stage the first opens
    for (size_t q = 0; q + 1 < p.marks.size(); q++) {
        if (p.marks[q].second >= 0) {
            float t = 0.f;
            ARTSS_CK(cudaEventElapsedTime(&t, p.marks[q].first, p.marks[q + 1].first));
            p.stage_ms[p.marks[q].second] += t;
        }
        p.pool.push_back(p.marks[q].first);
    }
    if (!p.marks.empty()) p.marks.erase(p.marks.begin(), p.marks.end() - 1);  // the last mark opens the next interval
    for (int s = 0; s < n_stages && s < ARTSS_STAGES; s++) ms[s] = p.stage_ms[s];
    return ARTSS_OK;
}

int artss_ctx_create(const artss_grid_desc *grid, int device, artss_ctx **out) {
    if (!grid || !out) { set_error("null argument"); return ARTSS_ERR_ARG; }
    *out = nullptr;
    if (grid->n_levels < 0 || grid->n_levels > kMaxLevel) {
        set_error("n_levels " + std::to_string(grid->n_levels) + " outside 0.." + std::to_string(kMaxLevel));
        return ARTSS_ERR_LIMIT;
    }
    for (int l = 0; l <= grid->n_levels; l++) {
        if (grid->Nx[l] < 3 || grid->Ny[l] < 3 || grid->Nz[l] < 3 ||
            grid->i1[l] < 1 || grid->i2[l] > grid->Nx[l] - 2 || grid->i1[l] > grid->i2[l] ||
            grid->j1[l] < 1 || grid->j2[l] > grid->Ny[l] - 2 || grid->j1[l] > grid->j2[l] ||
            grid->k1[l] < 1 || grid->k2[l] > grid->Nz[l] - 2 || grid->k1[l] > grid->k2[l]) {
            set_error("inconsistent grid description at level " + std::to_string(l));
            return ARTSS_ERR_ARG;
        }
        // kernels index cells with 32-bit integers
        if ((int64_t) grid->Nx[l] * grid->Ny[l] * grid->Nz[l] >= ((int64_t) 1 << 31)) {
            set_error("level " + std::to_string(l) + " has 2^31 cells or more");
            return ARTSS_ERR_LIMIT;
        }
    }
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        set_error(std::string("no CUDA device: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "count 0"));
        return ARTSS_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) { set_error("device ordinal out of range"); return ARTSS_ERR_ARG; }
    ARTSS_CK(cudaSetDevice(device));
    auto *ctx = new artss_ctx();
    ctx->device = device;
    ctx->grid = *grid;
    for (int l = 0; l <= grid->n_levels; l++) {
        ctx->lvl[l] = Level{grid->Nx[l], grid->Ny[l], grid->Nz[l], grid->i1[l], grid->i2[l],
                            grid->j1[l], grid->j2[l], grid->k1[l], grid->k2[l]};
    }
    auto fail = [&](cudaError_t err, const char *what) {
        int st = cuda_fail(err, what);
        artss_ctx_destroy(ctx);
        return st;
    };
    if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "stream");
    if ((e = cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess)
        return fail(e, "multiprocessor count");
    if ((e = cudaMalloc(&ctx->d_partials, kMaxPartials * sizeof(double))) != cudaSuccess) return fail(e, "partials");
    if ((e = cudaMalloc(&ctx->d_loop, 16 * sizeof(LoopState))) != cudaSuccess) return fail(e, "loop state");
    if ((e = cudaMalloc(&ctx->d_param, kParams * sizeof(double))) != cudaSuccess) return fail(e, "parameters");
    if ((e = cudaMemset(ctx->d_param, 0, kParams * sizeof(double))) != cudaSuccess) return fail(e, "parameters");
    if ((e = cudaStreamCreateWithFlags(&ctx->body_stream, cudaStreamNonBlocking)) != cudaSuccess)
        return fail(e, "capture stream");
    if ((e = cudaMemset(ctx->d_loop, 0, 16 * sizeof(LoopState))) != cudaSuccess) return fail(e, "loop state");
    if ((e = cudaMallocHost(&ctx->h_loop, 16 * sizeof(LoopState))) != cudaSuccess) return fail(e, "pinned loop state");
    for (int l = 0; l <= grid->n_levels; l++) {
        const int64_t n = ctx->lvl[l].size();
        if ((e = cudaMalloc(&ctx->d_flags[l], n)) != cudaSuccess) return fail(e, "cell flags");
        if ((e = cudaMemset(ctx->d_flags[l], 0, n)) != cudaSuccess) return fail(e, "cell flags");
    }
    // the memsets above ran on the legacy stream, which the context's
    // non-blocking stream does not order against
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return fail(e, "set-up");
    *out = ctx;
    return ARTSS_OK;
}

int artss_ctx_destroy(artss_ctx *ctx) {
    if (!ctx) return ARTSS_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (double *f : ctx->fields) cudaFree(f);
    for (int l = 0; l <= kMaxLevel; l++) {
        if (ctx->d_flags[l]) cudaFree(ctx->d_flags[l]);
        for (int t = 0; t < kFieldTypes; t++) {
            BcProgram &p = ctx->bc[l][t];
            cudaFree(p.d_target); cudaFree(p.d_root); cudaFree(p.d_depth); cudaFree(p.d_neg); cudaFree(p.d_value);
        }
    }
    for (uint8_t *t : ctx->d_sweep3_obst) if (t) cudaFree(t);
    if (ctx->cgsm_w) cudaFree(ctx->cgsm_w);
    if (ctx->dsmag) cudaFree(ctx->dsmag);
    if (ctx->rb_stream) cudaStreamSynchronize(ctx->rb_stream);
    for (auto &r : ctx->rb) {
        for (double *a : r.dev) cudaFree(a);
        for (double *a : r.host) cudaFreeHost(a);
        if (r.done) cudaEventDestroy(r.done);
    }
    if (ctx->rb_stream) cudaStreamDestroy(ctx->rb_stream);
    for (auto &m : ctx->prof.marks) cudaEventDestroy(m.first);
    for (auto &pe : ctx->prof.pending) cudaEventDestroy(pe.first);
    for (auto e : ctx->prof.events) cudaEventDestroy(e);
    for (auto e : ctx->prof.pool) cudaEventDestroy(e);
    if (ctx->copy_stream) {
        cudaStreamSynchronize(ctx->copy_stream);
        for (auto e : ctx->copy_ev) cudaEventDestroy(e);
        cudaEventDestroy(ctx->copy_mark);
        cudaEventDestroy(ctx->copy_tail);
        cudaStreamDestroy(ctx->copy_stream);
    }
    if (ctx->io_up) {
        cudaStreamSynchronize(ctx->io_up);
        cudaStreamSynchronize(ctx->io_down);
        for (double *a : ctx->io_stage_in) cudaFree(a);
        for (auto &v : ctx->io_stage_out)
            for (double *a : v) cudaFree(a);
        cudaEventDestroy(ctx->io_in_ready);
        cudaEventDestroy(ctx->io_in_free);
        for (int b = 0; b < 2; b++) {
            cudaEventDestroy(ctx->io_out_ready[b]);
            cudaEventDestroy(ctx->io_out_free[b]);
        }
        cudaStreamDestroy(ctx->io_up);
        cudaStreamDestroy(ctx->io_down);
    }
    cudaFree(ctx->d_partials);
    cudaFree(ctx->d_loop);
    cudaFree(ctx->d_param);
    if (ctx->body_stream) cudaStreamDestroy(ctx->body_stream);
    if (ctx->h_loop) cudaFreeHost(ctx->h_loop);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return ARTSS_OK;
}

void *artss_ctx_stream(artss_ctx *ctx) { return ctx ? (void *) ctx->stream : nullptr; }

int artss_ctx_sync(artss_ctx *ctx) {
    if (!ctx) { set_error("null context"); return ARTSS_ERR_ARG; }
    ARTSS_CK(cudaStreamSynchronize(ctx->stream));
    return ARTSS_OK;
}

int64_t artss_ctx_kernel_launches(artss_ctx *ctx) { return ctx ? ctx->launches : -1; }

int64_t artss_field_size(artss_ctx *ctx, int level) {
    if (check_level(ctx, level) != ARTSS_OK) return -1;
    return ctx->lvl[level].size();
}

int artss_field_alloc(artss_ctx *ctx, int level, double **out) {
    int st = check_level(ctx, level);
    if (st) return st;
    if (!out) { set_error("null output pointer"); return ARTSS_ERR_ARG; }
    const int64_t n = ctx->lvl[level].size();
    double *p = nullptr;
    ARTSS_CK(cudaMalloc(&p, n * sizeof(double)));
    cudaError_t e = cudaMemsetAsync(p, 0, n * sizeof(double), ctx->stream);
    if (e != cudaSuccess) { cudaFree(p); return cuda_fail(e, "field zero fill"); }
    ctx->fields.insert(p);
    *out = p;
    return ARTSS_OK;
}

int artss_field_free(artss_ctx *ctx, double *field) {
    if (!ctx) { set_error("null context"); return ARTSS_ERR_ARG; }
    auto it = ctx->fields.find(field);
    if (it == ctx->fields.end()) { set_error("pointer is not a field of this context"); return ARTSS_ERR_ARG; }
    ARTSS_CK(cudaStreamSynchronize(ctx->stream));
    ARTSS_CK(cudaFree(field));
    ctx->fields.erase(it);
    return ARTSS_OK;
}

int artss_upload(artss_ctx *ctx, double *dst, const double *host, int64_t n) {
    if (!ctx || !dst || !host || n < 0) { set_error("bad upload arguments"); return ARTSS_ERR_ARG; }
    ARTSS_CK(cudaMemcpyAsync(dst, host, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    ARTSS_CK(cudaStreamSynchronize(ctx->stream));
    return ARTSS_OK;
}

int artss_download(artss_ctx *ctx, double *host, const double *src, int64_t n) {
    if (!ctx || !src || !host || n < 0) { set_error("bad download arguments"); return ARTSS_ERR_ARG; }
    ARTSS_CK(cudaMemcpyAsync(host, src, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    ARTSS_CK(cudaStreamSynchronize(ctx->stream));
    return ARTSS_OK;
}

int artss_upload_async(artss_ctx *ctx, double *dst, const double *host, int64_t n) {
    if (!ctx || !dst || !host || n < 0) { set_error("bad upload arguments"); return ARTSS_ERR_ARG; }
    ARTSS_CK(cudaMemcpyAsync(dst, host, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    return ARTSS_OK;
}

int artss_download_async(artss_ctx *ctx, double *host, const double *src, int64_t n) {
    if (!ctx || !src || !host || n < 0) { set_error("bad download arguments"); return ARTSS_ERR_ARG; }
    ARTSS_CK(cudaMemcpyAsync(host, src, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    return ARTSS_OK;
}

namespace {
// the copy stream and its events, created on first use
int copy_stream_ready(artss_ctx *ctx) {
    if (ctx->copy_stream) return ARTSS_OK;
    ARTSS_CK(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    for (auto &e : ctx->copy_ev) ARTSS_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ARTSS_CK(cudaEventCreateWithFlags(&ctx->copy_mark, cudaEventDisableTiming));
    ARTSS_CK(cudaEventCreateWithFlags(&ctx->copy_tail, cudaEventDisableTiming));
    return ARTSS_OK;
}
// the copy stream continues after the main stream's work enqueued so far
int copy_after_main(artss_ctx *ctx) {
    int st = copy_stream_ready(ctx);
    if (st) return st;
    ARTSS_CK(cudaEventRecord(ctx->copy_mark, ctx->stream));
    ARTSS_CK(cudaStreamWaitEvent(ctx->copy_stream, ctx->copy_mark, 0));
    return ARTSS_OK;
}
}  // namespace

// ---------------------------------------------------------------- whole-step graphs

struct artss_graph {
    artss_ctx *ctx = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t launches = 0;
    int64_t fam[artss::FAM_COUNT]{};
};

namespace {
int64_t g_capture_launches0 = 0;
int64_t g_capture_fam0[artss::FAM_COUNT]{};
__global__ void k_set_param(double *slot, double v) { *slot = v; }
__global__ void k_scale_copy_param(double *__restrict__ dst, const double *__restrict__ src,
                                   const double *__restrict__ x, int64_t n) {
    const double f = *x;
    for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
        dst[i] = src[i] * f;
}
}  // namespace

int artss_graph_begin(artss_ctx *ctx) {
    if (!ctx) { set_error("null argument"); return ARTSS_ERR_ARG; }
    if (ctx->capturing) { set_error("a capture is already running"); return ARTSS_ERR_ARG; }
    if (ctx->prof.mask) { set_error("kernel-family timing cannot run inside a captured graph"); return ARTSS_ERR_ARG; }
    ARTSS_CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
    ctx->capturing = true;
    g_capture_launches0 = ctx->launches;
    for (int f = 0; f < FAM_COUNT; f++) g_capture_fam0[f] = ctx->prof.launches[f];
    return ARTSS_OK;
}

int artss_graph_end(artss_ctx *ctx, int discard, artss_graph **out) {
    if (!ctx || (!discard && !out)) { set_error("null argument"); return ARTSS_ERR_ARG; }
    if (!ctx->capturing) { set_error("no capture is running"); return ARTSS_ERR_ARG; }
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    ctx->capturing = false;
    // the captured work did not run: its launches are counted when the graph is
    const int64_t launches = ctx->launches - g_capture_launches0;
    int64_t fam[FAM_COUNT];
    for (int f = 0; f < FAM_COUNT; f++) {
        fam[f] = ctx->prof.launches[f] - g_capture_fam0[f];
        ctx->prof.launches[f] = g_capture_fam0[f];
    }
    ctx->launches = g_capture_launches0;
    if (e != cudaSuccess || discard) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        if (discard) return ARTSS_OK;
        return cuda_fail(e, "capture");
    }
    auto *gr = new artss_graph();
    gr->ctx = ctx;
    gr->graph = g;
    gr->launches = launches;
    for (int f = 0; f < FAM_COUNT; f++) gr->fam[f] = fam[f];
    const cudaError_t ei = cudaGraphInstantiate(&gr->exec, g, 0);
    if (ei != cudaSuccess) {
        cudaGraphDestroy(g);
        delete gr;
        return cuda_fail(ei, "graph instantiate");
    }
    *out = gr;
    return ARTSS_OK;
}

int artss_graph_launch(artss_graph *g) {
    if (!g) { set_error("null graph"); return ARTSS_ERR_ARG; }
    artss_ctx *ctx = g->ctx;
    ARTSS_CK(cudaGraphLaunch(g->exec, ctx->stream));
    ctx->launches += g->launches;
    for (int f = 0; f < FAM_COUNT; f++) ctx->prof.launches[f] += g->fam[f];
    return ARTSS_OK;
}

int artss_graph_destroy(artss_graph *g) {
    if (!g) return ARTSS_OK;
    if (g->ctx && g->ctx->stream) cudaStreamSynchronize(g->ctx->stream);
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return ARTSS_OK;
}

int artss_graph_capturing(artss_ctx *ctx) { return ctx && ctx->capturing ? 1 : 0; }

int artss_param_set(artss_ctx *ctx, int slot, double value) {
    if (!ctx || slot < 0 || slot >= kParams) { set_error("bad parameter slot"); return ARTSS_ERR_ARG; }
    if (ctx->capturing) { set_error("parameters are set outside a capture"); return ARTSS_ERR_ARG; }
    ARTSS_LAUNCH(ctx, FAM_FIELD_OP, k_set_param<<<1, 1, 0, ctx->stream>>>(ctx->d_param + slot, value));
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

int artss_scale_copy_param(artss_ctx *ctx, double *dst, const double *src, int slot, int level) {
    if (!ctx || !dst || !src || slot < 0 || slot >= kParams) { set_error("bad arguments"); return ARTSS_ERR_ARG; }
    int st = check_level(ctx, level);
    if (st) return st;
    const int64_t n = ctx->lvl[level].size();
    ARTSS_LAUNCH(ctx, FAM_FIELD_OP,
                 k_scale_copy_param<<<flat_blocks(n), 256, 0, ctx->stream>>>(dst, src, ctx->d_param + slot, n));
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

int artss_copy_upload(artss_ctx *ctx, int slot, double *dst, const double *host, int64_t n) {
    if (!ctx || !dst || !host || n < 0 || slot < 0 || slot >= kCopySlots) {
        set_error("bad copy upload arguments");
        return ARTSS_ERR_ARG;
    }
    int st = copy_after_main(ctx);
    if (st) return st;
    ARTSS_CK(cudaMemcpyAsync(dst, host, n * sizeof(double), cudaMemcpyHostToDevice, ctx->copy_stream));
    ARTSS_CK(cudaEventRecord(ctx->copy_ev[slot], ctx->copy_stream));
    return ARTSS_OK;
}

int artss_copy_wait(artss_ctx *ctx, int slot) {
    if (!ctx || slot < 0 || slot >= kCopySlots || !ctx->copy_stream) {
        set_error("bad copy wait arguments");
        return ARTSS_ERR_ARG;
    }
    ARTSS_CK(cudaStreamWaitEvent(ctx->stream, ctx->copy_ev[slot], 0));
    return ARTSS_OK;
}

int artss_copy_download(artss_ctx *ctx, double *host, const double *src, int64_t n) {
    if (!ctx || !src || !host || n < 0) { set_error("bad copy download arguments"); return ARTSS_ERR_ARG; }
    int st = copy_after_main(ctx);
    if (st) return st;
    ARTSS_CK(cudaMemcpyAsync(host, src, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->copy_stream));
    return ARTSS_OK;
}

int artss_copy_join(artss_ctx *ctx) {
    if (!ctx) { set_error("null argument"); return ARTSS_ERR_ARG; }
    if (!ctx->copy_stream) return ARTSS_OK;
    ARTSS_CK(cudaEventRecord(ctx->copy_tail, ctx->copy_stream));
    ARTSS_CK(cudaStreamWaitEvent(ctx->stream, ctx->copy_tail, 0));
    return ARTSS_OK;
}

}  // extern "C"

namespace {
// the pipeline's streams and events on first use; staging arrays of n doubles
int io_ready(artss_ctx *ctx, int64_t n, int n_in, int n_out) {
    if (!ctx->io_up) {
        ARTSS_CK(cudaStreamCreateWithFlags(&ctx->io_up, cudaStreamNonBlocking));
        ARTSS_CK(cudaStreamCreateWithFlags(&ctx->io_down, cudaStreamNonBlocking));
        ARTSS_CK(cudaEventCreateWithFlags(&ctx->io_in_ready, cudaEventDisableTiming));
        ARTSS_CK(cudaEventCreateWithFlags(&ctx->io_in_free, cudaEventDisableTiming));
        for (int b = 0; b < 2; b++) {
            ARTSS_CK(cudaEventCreateWithFlags(&ctx->io_out_ready[b], cudaEventDisableTiming));
            ARTSS_CK(cudaEventCreateWithFlags(&ctx->io_out_free[b], cudaEventDisableTiming));
        }
    }
    if (n != ctx->io_n) {
        // a new field size: every transfer in flight ends before the staging changes
        ARTSS_CK(cudaStreamSynchronize(ctx->io_up));
        ARTSS_CK(cudaStreamSynchronize(ctx->io_down));
        ARTSS_CK(cudaStreamSynchronize(ctx->stream));
        for (double *a : ctx->io_stage_in) cudaFree(a);
        ctx->io_stage_in.clear();
        for (auto &v : ctx->io_stage_out) {
            for (double *a : v) cudaFree(a);
            v.clear();
        }
        ctx->io_n = n;
    }
    while ((int) ctx->io_stage_in.size() < n_in) {
        double *a = nullptr;
        ARTSS_CK(cudaMalloc(&a, (size_t) n * sizeof(double)));
        ctx->io_stage_in.push_back(a);
    }
    for (auto &v : ctx->io_stage_out)
        while ((int) v.size() < n_out) {
            double *a = nullptr;
            ARTSS_CK(cudaMalloc(&a, (size_t) n * sizeof(double)));
            v.push_back(a);
        }
    return ARTSS_OK;
}
}  // namespace

extern "C" {

int artss_io_in(artss_ctx *ctx, int n_in, double *const *fields, const double *const *host, int64_t n) {
    if (!ctx || n_in < 0 || n < 0 || (n_in && (!fields || !host))) {
        set_error("bad io_in arguments");
        return ARTSS_ERR_ARG;
    }
    for (int k = 0; k < n_in; k++)
        if (!fields[k] || !host[k]) { set_error("null io_in array"); return ARTSS_ERR_ARG; }
    if (ctx->capturing) { set_error("io_in while a graph is captured"); return ARTSS_ERR_ARG; }
    if (n_in == 0) return ARTSS_OK;
    int st = io_ready(ctx, n, n_in, 0);
    if (st) return st;
    // the staging is overwritten once the previous call's inputs have left it
    ARTSS_CK(cudaStreamWaitEvent(ctx->io_up, ctx->io_in_free, 0));
    for (int k = 0; k < n_in; k++)
        ARTSS_CK(cudaMemcpyAsync(ctx->io_stage_in[k], host[k], (size_t) n * sizeof(double), cudaMemcpyHostToDevice,
                                 ctx->io_up));
    ARTSS_CK(cudaEventRecord(ctx->io_in_ready, ctx->io_up));
    ARTSS_CK(cudaStreamWaitEvent(ctx->stream, ctx->io_in_ready, 0));
    for (int k = 0; k < n_in; k++) {
        ARTSS_LAUNCH_PDL(ctx, FAM_FIELD_OP, k_copy, flat_blocks(n), 256, 0, fields[k],
                         (const double *) ctx->io_stage_in[k], n);
        ARTSS_LAUNCH_CK(ctx);
    }
    ARTSS_CK(cudaEventRecord(ctx->io_in_free, ctx->stream));
    return ARTSS_OK;
}

int artss_io_out(artss_ctx *ctx, int n_out, const double *const *fields, double *const *host, int64_t n) {
    if (!ctx || n_out < 0 || n < 0 || (n_out && (!fields || !host))) {
        set_error("bad io_out arguments");
        return ARTSS_ERR_ARG;
    }
    for (int k = 0; k < n_out; k++)
        if (!fields[k] || !host[k]) { set_error("null io_out array"); return ARTSS_ERR_ARG; }
    if (ctx->capturing) { set_error("io_out while a graph is captured"); return ARTSS_ERR_ARG; }
    int st = io_ready(ctx, n, 0, n_out);
    if (st) return st;
    const int b = (int) (ctx->io_calls & 1);
    ctx->io_calls++;
    // call k returns once call k-2 (the last user of this parity's staging) is
    // complete: its host arrays are then free
    ARTSS_CK(cudaEventSynchronize(ctx->io_out_free[b]));
    if (n_out == 0) return ARTSS_OK;
    for (int k = 0; k < n_out; k++) {
        ARTSS_LAUNCH_PDL(ctx, FAM_FIELD_OP, k_copy, flat_blocks(n), 256, 0, ctx->io_stage_out[b][k], fields[k], n);
        ARTSS_LAUNCH_CK(ctx);
    }
    ARTSS_CK(cudaEventRecord(ctx->io_out_ready[b], ctx->stream));
    ARTSS_CK(cudaStreamWaitEvent(ctx->io_down, ctx->io_out_ready[b], 0));
    for (int k = 0; k < n_out; k++)
        ARTSS_CK(cudaMemcpyAsync(host[k], ctx->io_stage_out[b][k], (size_t) n * sizeof(double), cudaMemcpyDeviceToHost,
                                 ctx->io_down));
    ARTSS_CK(cudaEventRecord(ctx->io_out_free[b], ctx->io_down));
    return ARTSS_OK;
}

int artss_readback(artss_ctx *ctx, int n, const double *const *fields, int64_t count, int64_t *ticket) {
    if (!ctx || n < 1 || count < 1 || !fields || !ticket) { set_error("bad readback arguments"); return ARTSS_ERR_ARG; }
    for (int k = 0; k < n; k++)
        if (!fields[k]) { set_error("null readback field"); return ARTSS_ERR_ARG; }
    if (ctx->capturing) { set_error("readback while a graph is captured"); return ARTSS_ERR_ARG; }
    const int64_t t = ctx->rb_next;
    artss_ctx::Readback &r = ctx->rb[t & 1];
    {
        // the slot's previous ticket (t - 2) must be released by its user
        std::unique_lock<std::mutex> lock(ctx->rb_mutex);
        ctx->rb_cv.wait(lock, [&] { return r.released; });
    }
    if (!ctx->rb_stream) ARTSS_CK(cudaStreamCreateWithFlags(&ctx->rb_stream, cudaStreamNonBlocking));
    if (!r.done) ARTSS_CK(cudaEventCreateWithFlags(&r.done, cudaEventDisableTiming));
    ARTSS_CK(cudaEventSynchronize(r.done));  // the slot's previous copies are complete
    if (r.count != count || (int) r.dev.size() < n) {
        for (double *a : r.dev) cudaFree(a);
        for (double *a : r.host) cudaFreeHost(a);
        r.dev.clear();
        r.host.clear();
        r.count = count;
    }
    while ((int) r.dev.size() < n) {
        double *d = nullptr, *h = nullptr;
        ARTSS_CK(cudaMalloc(&d, (size_t) count * sizeof(double)));
        ARTSS_CK(cudaMallocHost(&h, (size_t) count * sizeof(double)));
        r.dev.push_back(d);
        r.host.push_back(h);
    }
    // snapshot on the context stream (ordered after the work enqueued so far),
    // device-to-host beside the context's later work
    for (int k = 0; k < n; k++) {
        ARTSS_LAUNCH_PDL(ctx, FAM_FIELD_OP, k_copy, flat_blocks(count), 256, 0, r.dev[k], fields[k], count);
        ARTSS_LAUNCH_CK(ctx);
    }
    cudaEvent_t snap = prof_event(ctx);
    if (!snap) { set_error("cudaEventCreate failed"); return ARTSS_ERR_CUDA; }
    ARTSS_CK(cudaEventRecord(snap, ctx->stream));
    ARTSS_CK(cudaStreamWaitEvent(ctx->rb_stream, snap, 0));
    ctx->prof.pool.push_back(snap);  // reusable once recorded and waited on
    for (int k = 0; k < n; k++)
        ARTSS_CK(cudaMemcpyAsync(r.host[k], r.dev[k], (size_t) count * sizeof(double), cudaMemcpyDeviceToHost,
                                 ctx->rb_stream));
    ARTSS_CK(cudaEventRecord(r.done, ctx->rb_stream));
    {
        std::lock_guard<std::mutex> lock(ctx->rb_mutex);
        r.ticket = t;
        r.released = false;
    }
    ctx->rb_next = t + 1;
    *ticket = t;
    return ARTSS_OK;
}

int artss_readback_wait(artss_ctx *ctx, int64_t ticket, const double **host, int n) {
    if (!ctx || ticket < 0 || (n > 0 && !host)) { set_error("bad readback_wait arguments"); return ARTSS_ERR_ARG; }
    artss_ctx::Readback &r = ctx->rb[ticket & 1];
    cudaEvent_t done;
    {
        std::lock_guard<std::mutex> lock(ctx->rb_mutex);
        if (r.ticket != ticket || r.released) { set_error("readback ticket not pending"); return ARTSS_ERR_STATE; }
        if (n > (int) r.host.size()) { set_error("more arrays than the readback holds"); return ARTSS_ERR_ARG; }
        done = r.done;
        for (int k = 0; k < n; k++) host[k] = r.host[k];
    }
    ARTSS_CK(cudaEventSynchronize(done));
    return ARTSS_OK;
}

int artss_readback_release(artss_ctx *ctx, int64_t ticket) {
    if (!ctx || ticket < 0) { set_error("bad readback_release arguments"); return ARTSS_ERR_ARG; }
    artss_ctx::Readback &r = ctx->rb[ticket & 1];
    {
        std::lock_guard<std::mutex> lock(ctx->rb_mutex);
        if (r.ticket != ticket || r.released) { set_error("readback ticket not pending"); return ARTSS_ERR_STATE; }
        r.released = true;
    }
    ctx->rb_cv.notify_all();
    return ARTSS_OK;
}

int artss_io_sync(artss_ctx *ctx) {
    if (!ctx) { set_error("null argument"); return ARTSS_ERR_ARG; }
    if (ctx->io_up) {
        ARTSS_CK(cudaStreamSynchronize(ctx->io_up));
        ARTSS_CK(cudaStreamSynchronize(ctx->io_down));
    }
    ARTSS_CK(cudaStreamSynchronize(ctx->stream));
    return ARTSS_OK;
}

int artss_set_cell_lists(artss_ctx *ctx, int level, const int64_t *inner, int64_t n_inner,
                         const int64_t *domain, int64_t n_domain) {
    int st = check_level(ctx, level);
    if (st) return st;
    if ((n_inner && !inner) || (n_domain && !domain) || n_inner < 0 || n_domain < 0) {
        set_error("bad list arguments"); return ARTSS_ERR_ARG;
    }
    const Level &L = ctx->lvl[level];
    ctx->n_inner[level] = n_inner;
    ctx->geom_version++;
    if (level == 0) {
        // the sweep's obstacle table describes the old lists
        for (int t = 0; t < 3; t++) {
            if (ctx->d_sweep3_obst[t]) cudaFree(ctx->d_sweep3_obst[t]);
            ctx->d_sweep3_obst[t] = nullptr;
            ctx->sweep3_obst_state[t] = 0;
        }
    }
    // every inner cell must lie in the computational domain, every domain-list
    // cell in the box one layer larger; lists are strictly ascending
    auto check = [&](const int64_t *list, int64_t n, int64_t grow, const char *name) -> bool {
        for (int64_t q = 0; q < n; q++) {
            const int64_t idx = list[q];
            if (idx < 0 || idx >= L.size() || (q && list[q - 1] >= idx)) {
                set_error(std::string(name) + " list not ascending or out of range"); return false;
            }
            const int64_t k = idx / L.nxy(), j = (idx - k * L.nxy()) / L.Nx, i = idx - k * L.nxy() - j * L.Nx;
            if (i < L.i1 - grow || i > L.i2 + grow || j < L.j1 - grow || j > L.j2 + grow ||
                k < L.k1 - grow || k > L.k2 + grow) {
                set_error(std::string(name) + " list cell outside its box"); return false;
            }
        }
        return true;
    };
    if (!check(inner, n_inner, 0, "inner") || !check(domain, n_domain, 1, "domain")) return ARTSS_ERR_ARG;
    ctx->h_inner[level].assign((size_t) L.size(), false);
    for (int64_t q = 0; q < n_inner; q++) ctx->h_inner[level][(size_t) inner[q]] = true;
    for (auto &prog : ctx->bc[level]) prog.pipe_state = -2;
    int64_t *d_list = nullptr;
    const int64_t nmax = std::max<int64_t>(std::max(n_inner, n_domain), 1);
    ARTSS_CK(cudaMalloc(&d_list, nmax * sizeof(int64_t)));
    cudaError_t e = cudaMemsetAsync(ctx->d_flags[level], 0, L.size(), ctx->stream);
    if (e == cudaSuccess && n_inner) e = cudaMemcpyAsync(d_list, inner, n_inner * sizeof(int64_t), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess && n_inner) {
        ARTSS_LAUNCH(ctx, FAM_FIELD_OP, k_mark<<<flat_blocks(n_inner), 256, 0, ctx->stream>>>(ctx->d_flags[level], d_list, n_inner, kInner));
        ctx->launches++;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess && n_domain) e = cudaMemcpyAsync(d_list, domain, n_domain * sizeof(int64_t), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess && n_domain) {
        ARTSS_LAUNCH(ctx, FAM_FIELD_OP, k_mark<<<flat_blocks(n_domain), 256, 0, ctx->stream>>>(ctx->d_flags[level], d_list, n_domain, kDomain));
        ctx->launches++;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d_list);
    if (e != cudaSuccess) return cuda_fail(e, "cell flags");
    return ARTSS_OK;
}

int artss_get_cell_flags(artss_ctx *ctx, int level, uint8_t *host_out, int64_t n) {
    int st = check_level(ctx, level);
    if (st) return st;
    if (!host_out || n != ctx->lvl[level].size()) { set_error("flag buffer size mismatch"); return ARTSS_ERR_ARG; }
    ARTSS_CK(cudaMemcpyAsync(host_out, ctx->d_flags[level], n, cudaMemcpyDeviceToHost, ctx->stream));
    ARTSS_CK(cudaStreamSynchronize(ctx->stream));
    return ARTSS_OK;
}

#define ARTSS_FIELD_OP(...)                                           \
    int st = check_level(ctx, level);                                 \
    if (st) return st;                                                \
    const int64_t n = ctx->lvl[level].size();                         \
    __VA_ARGS__;                                                      \
    ARTSS_LAUNCH_CK(ctx);                                             \
    return ARTSS_OK;

int artss_fill(artss_ctx *ctx, double *f, int level, double value) {
    if (!f) { set_error("null field"); return ARTSS_ERR_ARG; }
    ARTSS_FIELD_OP(ARTSS_LAUNCH_PDL(ctx, FAM_FIELD_OP, k_fill, flat_blocks(n), 256, 0, f, n, value))
}

int artss_copy(artss_ctx *ctx, double *dst, const double *src, int level) {
    if (!dst || !src) { set_error("null field"); return ARTSS_ERR_ARG; }
    if (dst == src) return check_level(ctx, level);
    ARTSS_FIELD_OP(ARTSS_LAUNCH_PDL(ctx, FAM_FIELD_OP, k_copy, flat_blocks(n), 256, 0, dst, src, n))
}

int artss_add_field(artss_ctx *ctx, double *dst, const double *src, int level) {
    if (!dst || !src) { set_error("null field"); return ARTSS_ERR_ARG; }
    ARTSS_FIELD_OP(ARTSS_LAUNCH_PDL(ctx, FAM_FIELD_OP, k_add_field, flat_blocks(n), 256, 0, dst, src, n))
}

int artss_add_scalar(artss_ctx *ctx, double *dst, double x, int level) {
    if (!dst) { set_error("null field"); return ARTSS_ERR_ARG; }
    ARTSS_FIELD_OP(ARTSS_LAUNCH(ctx, FAM_FIELD_OP, k_add_scalar<<<flat_blocks(n), 256, 0, ctx->stream>>>(dst, x, n)))
}

int artss_scale(artss_ctx *ctx, double *dst, double x, int level) {
    if (!dst) { set_error("null field"); return ARTSS_ERR_ARG; }
    ARTSS_FIELD_OP(ARTSS_LAUNCH_PDL(ctx, FAM_FIELD_OP, k_scale, flat_blocks(n), 256, 0, dst, x, n))
}

int artss_scale_copy(artss_ctx *ctx, double *dst, const double *src, double x, int level) {
    if (!dst || !src) { set_error("null field"); return ARTSS_ERR_ARG; }
    ARTSS_FIELD_OP(ARTSS_LAUNCH_PDL(ctx, FAM_FIELD_OP, k_scale_copy, flat_blocks(n), 256, 0, dst, src, x, n))
}

int artss_couple(artss_ctx *ctx, const double *a, double *a0, double *a_tmp,
                 const double *b, double *b0, double *b_tmp,
                 const double *c, double *c0, double *c_tmp) {
    if ((a && !a_tmp) || (b && !b_tmp) || (c && !c_tmp)) {
        set_error("couple: incomplete triple"); return ARTSS_ERR_ARG;
    }
    const int level = 0;
    ARTSS_FIELD_OP(ARTSS_LAUNCH_PDL(ctx, FAM_COUPLE, k_couple3, flat_blocks(n), 256, 0, a, a0, a_tmp, b, b0, b_tmp, c, c0, c_tmp, n))
}

}  // extern "C"
