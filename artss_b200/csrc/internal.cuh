// Internal declarations shared by the translation units of libartss_cuda.so.
// The arithmetic of every kernel reproduces the reference expression order
// operation by operation; the library is compiled with --fmad=false so each
// a*b+c rounds twice, as the reference serial build does.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <condition_variable>
#include <map>
#include <mutex>
#include <utility>
#include <string>
#include <vector>
#include <set>

#include "../../include/artss_cuda.h"

namespace artss {

constexpr int kMaxLevel = ARTSS_MAX_LEVEL;
constexpr int kFieldTypes = ARTSS_NUM_FIELD_TYPES;
constexpr int kCopySlots = 8;           // uploads on the copy stream waited for by slot
constexpr int kParams = 16;             // parameter slots of captured steps
constexpr int kBcMaxDepth = 4;          // boundary assignments folded per thread
constexpr int kReduceThreads = 256;
constexpr int kMaxPartials = 1 << 16;   // per-block partial sums of up to two reduction passes
constexpr int kNnErrSlot = 15;          // loop slot whose error flag the network kernels raise
constexpr int kTmaBoxX = 72, kTmaBoxY = 12;  // TMA plane window (cells): a 64 x 8 tile, a 2-cell ring, x aligned to 2

enum CellFlag : uint8_t { kInner = 1, kDomain = 2 };

// Geometry of one multigrid level, passed to kernels by value.
struct Level {
    int64_t Nx, Ny, Nz;
    int64_t i1, i2, j1, j2, k1, k2;  // computational-domain inner cells, inclusive
    __host__ __device__ int64_t nxy() const { return Nx * Ny; }
    __host__ __device__ int64_t size() const { return Nx * Ny * Nz; }
};

// Compiled boundary program of one (level, field type): `waves` groups of
// assignments; within a group no assignment reads a cell another one writes.
struct BcProgram {
    bool present = false;
    int waves = 0;
    std::vector<int64_t> wave_begin;  // waves+1 offsets
    int64_t n = 0;
    int64_t *d_target = nullptr;
    int64_t *d_root = nullptr;
    uint8_t *d_depth = nullptr;
    uint8_t *d_neg = nullptr;          // bit d: step d negates
    double *d_value = nullptr;         // [kBcMaxDepth][n]
    std::vector<int64_t> h_target;     // targets, host copy
    std::vector<int64_t> h_root;       // roots, host copy
    std::vector<int8_t> h_sign;        // sign of x_t = +-x_r with every value zero, host copy
    bool zero_values = false;          // every value of the program is +0.0: x_t = +-x_r + 0
    // plan of the pipelined coarse solve: state -2 unknown, -1 not eligible, 1 planned
    int pipe_state = -2;
    std::vector<int> pipe_kb;          // plane split, ranks + 1 entries
    int pipe_ranks = 0, pipe_cap = 0, pipe_tcap = 0, pipe_fcap = 0;
    int64_t pipe_smem = 0;
};

// Device-resident control block of one bounded iteration loop.
struct LoopState {
    double sum;        // reduction result of the last pass
    double residual;   // sqrt(sum) (or caller-defined)
    long long it;      // iterations done
    int cond;          // loop continues
    int pad;           // error flag: a bounded wait in a kernel of the loop gave up (2: a graph loop hit its cap)
    int guard;         // bodies run by a graph loop (conditional node) since the loop's init
    int unused;
};

// Kernel families for launch counting and event timing (artss_ctx_profile).
enum Family : int {
    FAM_ADVECT = 0, FAM_SMAGORINSKY, FAM_DIVERGENCE, FAM_PROJECTION, FAM_BUOYANCY, FAM_ADD_SOURCE,
    FAM_CGS, FAM_JACOBI, FAM_COPY_DOMAIN, FAM_BC, FAM_FIELD_OP, FAM_COUPLE, FAM_MG_JACOBI, FAM_MG_CGS,
    FAM_MG_RESIDUUM, FAM_MG_RESTRICT, FAM_MG_PROLONGATE, FAM_MG_RESNORM, FAM_REDUCE, FAM_MG_COARSE,
    FAM_CONV, FAM_NN,
    FAM_COUNT
};
static_assert(FAM_COUNT == ARTSS_KERNEL_FAMILIES, "family table");

// Autotuner key: kernel id, level shape, kernel flavour.
struct TuneKey {
    int kernel;
    int64_t nx, ny, nz;
    int flavour;
    bool operator<(const TuneKey &o) const {
        if (kernel != o.kernel) return kernel < o.kernel;
        if (nx != o.nx) return nx < o.nx;
        if (ny != o.ny) return ny < o.ny;
        if (nz != o.nz) return nz < o.nz;
        return flavour < o.flavour;
    }
};

struct Profile {
    uint64_t mask = 0;
    int64_t launches[FAM_COUNT] = {};
    double ms[FAM_COUNT] = {};
    std::vector<std::pair<cudaEvent_t, int>> pending;  // start event (end = next) + family
    std::vector<cudaEvent_t> events;                    // recorded, in order
    std::vector<cudaEvent_t> pool;                      // free events
    bool stages = false;                                // stage marks recorded (artss_ctx_stage_timing)
    std::vector<std::pair<cudaEvent_t, int>> marks;     // stage boundary events, in order, with the stage they open
    double stage_ms[ARTSS_STAGES] = {};
};

}  // namespace artss

struct artss_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    artss_grid_desc grid{};
    artss::Level lvl[artss::kMaxLevel + 1]{};
    uint8_t *d_flags[artss::kMaxLevel + 1]{};
    std::vector<bool> h_inner[artss::kMaxLevel + 1];  // inner-cell bitmap per level, host copy
    int64_t n_inner[artss::kMaxLevel + 1]{};  // inner cells per level (artss_set_cell_lists)
    double *proj[artss::kMaxLevel + 1]{};     // scratch of artss_coarse_project (lazily, freed with fields)
    artss::BcProgram bc[artss::kMaxLevel + 1][artss::kFieldTypes];
    double *d_partials = nullptr;       // kMaxPartials doubles
    artss::LoopState *d_loop = nullptr; // device loop blocks (16)
    artss::LoopState *h_loop = nullptr; // pinned mirror
    int64_t launches = 0;
    std::set<double *> fields;
    artss::Profile prof;
    std::map<std::pair<const void *, int>, CUtensorMap> tmaps;  // TMA descriptors per (array, level)
    bool autotune = true;                                        // time kernel variants on first use
    int sweep_force = -1;                                        // colored Gauss-Seidel sweep variant pinned (-1: tuned)
    int sm_count = 0;                                            // multiprocessors of the device
    uint64_t geom_version = 0;                                   // bumped by every cell-list or boundary-program change
    // tile columns x planes of level 0 whose row-pair sweep tile (+ ring) holds a
    // box cell that is not inner (k_cgs_sweep3); built on first use
    uint8_t *d_sweep3_obst[3] = {nullptr, nullptr, nullptr};     // per tile height (64 x 8, 64 x 6, 64 x 16)
    int sweep3_obst_state[3] = {0, 0, 0};                        // 0 not built, 1 built, 2 every box cell inner
    double *dsmag = nullptr;                                     // work arrays of artss_turb_dynamic_smagorinsky
    uint64_t dsmag_version = 0;                                  // geom_version they were zeroed for
    float *cgsm_w = nullptr;                                     // FP32 defect / correction of artss_diffuse_cgs_mixed
    int64_t cgsm_n = 0;
    std::map<artss::TuneKey, int> tuned;                         // autotuned variant per kernel and shape
    // host transfers overlapped with the step: a second stream, completion
    // events of its uploads by slot, a mark of the main stream, its tail
    // whole-step capture (artss_graph_begin .. artss_graph_end): loops become
    // conditional WHILE nodes whose bodies are captured on body_stream
    bool capturing = false;
    int pdl = 2;  // launch_pdl overlaps a launch with its predecessor's tail: 1 eager runs, 2 also captured graphs
    cudaStream_t body_stream = nullptr;
    double *d_param = nullptr;  // per-launch parameters of captured work (artss_param_set), kParams doubles
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t copy_ev[artss::kCopySlots]{};
    cudaEvent_t copy_mark = nullptr, copy_tail = nullptr;
    // pipelined whole-field transfers (artss_io_in / artss_io_out): uploads on
    // io_up, read-backs on io_down (one copy engine each), device staging
    cudaStream_t io_up = nullptr, io_down = nullptr;
    std::vector<double *> io_stage_in, io_stage_out[2];
    // snapshot read-backs for output writers (artss_readback): per slot device
    // staging, page-locked host copies, completion event; slot t % 2 of ticket t
    struct Readback {
        std::vector<double *> dev;
        std::vector<double *> host;
        int64_t count = 0;
        cudaEvent_t done = nullptr;
        int64_t ticket = -1;   // ticket occupying the slot
        bool released = true;  // its user has finished with the host copies
    } rb[2];
    int64_t rb_next = 0;
    cudaStream_t rb_stream = nullptr;
    std::mutex rb_mutex;
    std::condition_variable rb_cv;
    int64_t io_n = 0, io_calls = 0;
    cudaEvent_t io_in_ready = nullptr, io_in_free = nullptr, io_out_ready[2]{}, io_out_free[2]{};
    int64_t loop_hint[4][8] = {{1, 1, 1, 1, 1, 1, 1, 1}, {1, 1, 1, 1, 1, 1, 1, 1},
                               {1, 1, 1, 1, 1, 1, 1, 1}, {1, 1, 1, 1, 1, 1, 1, 1}};
};

namespace artss {
cudaEvent_t prof_event(artss_ctx *ctx);

// Programmatic dependent launch.  A kernel started by launch_pdl may begin while
// its predecessor on the stream is still running: before pdl_wait() returns (the
// predecessor complete, its writes visible) it reads only data that no kernel of
// the step writes.  pdl_trigger() in a predecessor lets its dependent launch
// once every block of the predecessor has passed it.  Both are no-ops for
// ordinary launches.  Whether launch_pdl also sets the attribute while a graph
// is captured (a programmatic edge in the graph) is the context's pdl mode.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... K, typename... A>
cudaError_t launch_pdl(artss_ctx *ctx, void (*kern)(K...), dim3 grid, dim3 block, size_t smem, A &&...args) {
    cudaLaunchConfig_t lc = {};
    lc.gridDim = grid;
    lc.blockDim = block;
    lc.dynamicSmemBytes = smem;
    lc.stream = ctx->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    lc.attrs = at;
    lc.numAttrs = (ctx->pdl == 2 || (ctx->pdl == 1 && !ctx->capturing)) ? 1 : 0;
    return cudaLaunchKernelEx(&lc, kern, std::forward<A>(args)...);
}
// Brackets one kernel launch: counts it under its family and, when the
// family is profiled, records an event pair around it on the context stream.
struct ProfScope {
    artss_ctx *ctx;
    int fam;
    cudaEvent_t start = nullptr;
    ProfScope(artss_ctx *c, int f) : ctx(c), fam(f) {
        if (ctx->prof.mask >> fam & 1) {
            start = prof_event(ctx);
            if (start) cudaEventRecord(start, ctx->stream);
        }
    }
    ~ProfScope() {
        ctx->prof.launches[fam]++;
        if (start) {
            cudaEvent_t stop = prof_event(ctx);
            if (stop) {
                cudaEventRecord(stop, ctx->stream);
                ctx->prof.pending.push_back({start, fam});
                ctx->prof.events.push_back(stop);
            }
        }
    }
};
}  // namespace artss

namespace artss {

// thread-local error message of the last failing call
void set_error(const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);

#define ARTSS_CK(call)                                                   \
    do {                                                                 \
        cudaError_t e_ = (call);                                         \
        if (e_ != cudaSuccess) return artss::cuda_fail(e_, #call);       \
    } while (0)

#define ARTSS_LAUNCH_CK(ctx)                                             \
    do {                                                                 \
        (ctx)->launches++;                                               \
        cudaError_t e_ = cudaGetLastError();                             \
        if (e_ != cudaSuccess) return artss::cuda_fail(e_, "kernel launch"); \
    } while (0)

int check_level(const artss_ctx *ctx, int level);
int check_field_type(int ft);

// 3-D launch shape over an index box [x0..x1] x [y0..y1] x [z0..z1].
struct Box3 {
    int64_t x0, x1, y0, y1, z0, z1;
    __host__ __device__ int64_t nx() const { return x1 - x0 + 1; }
    __host__ __device__ int64_t ny() const { return y1 - y0 + 1; }
    __host__ __device__ int64_t nz() const { return z1 - z0 + 1; }
};
constexpr int kBx = 64, kBy = 4;
inline dim3 box_grid(const Box3 &b) {
    return dim3((unsigned) ((b.nx() + kBx - 1) / kBx), (unsigned) ((b.ny() + kBy - 1) / kBy), (unsigned) b.nz());
}
inline dim3 box_block() { return dim3(kBx, kBy, 1); }
inline Box3 inner_box(const Level &L) { return {L.i1, L.i2, L.j1, L.j2, L.k1, L.k2}; }
inline Box3 domain_box(const Level &L) { return {L.i1 - 1, L.i2 + 1, L.j1 - 1, L.j2 + 1, L.k1 - 1, L.k2 + 1}; }

// Plane loop of one (i, j) column over planes k = z0 + blockIdx.z + t * gridDim.z,
// U (default kColU) planes per round.  For every plane of a round `value(q, k)` runs first
// (the cells of a column are independent, so their loads are in flight
// together), then `put(q, k, v, flag)` for the planes whose cell carries kInner, in
// ascending k, with the flag value already loaded (`bit`: the flag bit that
// selects the cells, kInner by default).  A round's planes past z1 evaluate the round's first plane again
// and store nothing.  Every cell of an inner box has its six neighbours inside
// the level's array, so `value` reads them without a check.  32-bit indices:
// artss_ctx_create rejects levels of 2^31 cells or more.
constexpr int kColU = 4;
template <int U = kColU, class FlagT, class V, class P>
__device__ __forceinline__ void column_planes(int base, int nk, int z0, int z1, const FlagT *__restrict__ flags,
                                              V value, P put, unsigned bit = kInner) {
    const int gz = (int) gridDim.z;
    using T = decltype(value(0, 0));
    for (int k0 = z0 + (int) blockIdx.z; k0 <= z1; k0 += U * gz) {
        T v[U];
        int q[U], kk[U];
        FlagT fl[U];
        bool ok[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int k = k0 + u * gz;
            const bool in = k <= z1;
            kk[u] = in ? k : k0;
            q[u] = base + nk * kk[u];
            fl[u] = flags[q[u]];
            ok[u] = in && (fl[u] & bit);
            v[u] = value(q[u], kk[u]);
        }
#pragma unroll
        for (int u = 0; u < U; u++)
            if (ok[u]) put(q[u], kk[u], v[u], fl[u]);
    }
}

// z-marching variant for 7-point stencils of one array f: the block's planes
// are the contiguous run [z0 + blockIdx.z * chunk, ...] of chunk =
// ceil(nz / gridDim.z) planes, and the thread walks its column through them
// U (default kColU) planes per round.  The centre values f[q] of planes k-1 .. k+U are
// loaded once per round and handed to `value(q, k, f_km1, f_k, f_kp1)` as the
// z-neighbours, so a cell costs one f load less than its stencil has z terms,
// and each block streams through consecutive planes.  Planes past the run end
// are clamped to the plane after it (a ghost or inner plane of the array) and
// store nothing; `put` as in column_planes.
template <int U = kColU, class T, class FlagT, class V, class P>
__device__ __forceinline__ void column_march(const T *__restrict__ f, int base, int nk, int z0, int z1,
                                             const FlagT *__restrict__ flags, V value, P put) {
    const int nz = z1 - z0 + 1, gz = (int) gridDim.z;
    const int chunk = (nz + gz - 1) / gz;
    const int kb = z0 + (int) blockIdx.z * chunk;
    if (kb > z1) return;
    const int ke = min(kb + chunk - 1, z1);
    T c[U + 2];
    c[0] = f[base + nk * (kb - 1)];
    c[1] = f[base + nk * kb];
    using R = decltype(value(0, 0, c[0], c[1], c[1]));
    for (int k0 = kb; k0 <= ke; k0 += U) {
#pragma unroll
        for (int u = 0; u < U; u++) c[2 + u] = f[base + nk * min(k0 + 1 + u, ke + 1)];
        R v[U];
        int q[U];
        FlagT fl[U];
        bool ok[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int k = k0 + u;
            const bool in = k <= ke;
            q[u] = base + nk * (in ? k : ke);
            fl[u] = flags[q[u]];
            ok[u] = in && (fl[u] & kInner);
            v[u] = value(q[u], in ? k : ke, c[u], c[u + 1], c[u + 2]);
        }
#pragma unroll
        for (int u = 0; u < U; u++)
            if (ok[u]) put(q[u], k0 + u, v[u], fl[u]);
        c[0] = c[U];
        c[1] = c[U + 1];
    }
}

// Launch shapes the autotuner tries for column kernels: threads of a block in
// x and y, and the cap on the number of blocks (the z extent of the grid is
// the box's planes, capped so that x * y * z blocks stay within it).  Shape 0
// is the untuned default.
struct ColShape {
    unsigned bx, by, cap;
};
constexpr ColShape kColShapes[] = {{64, 4, 2048}, {32, 8, 2048}, {128, 2, 2048}, {32, 4, 4096},
                                   {64, 4, 4096}, {64, 4, 1024}, {128, 4, 1024}, {256, 1, 2048}};
constexpr int kColShapeCount = (int) (sizeof(kColShapes) / sizeof(kColShapes[0]));
inline dim3 col_grid(const Box3 &b, const ColShape &s) {
    const int64_t gx = (b.nx() + s.bx - 1) / s.bx, gy = (b.ny() + s.by - 1) / s.by;
    const int64_t cap = std::max<int64_t>(1, (int64_t) s.cap / std::max<int64_t>(gx * gy, 1));
    return dim3((unsigned) gx, (unsigned) gy, (unsigned) std::max<int64_t>(1, std::min<int64_t>(b.nz(), cap)));
}
// Kernel ids of the launch-shape tuner (TuneKey::kernel; 0 is the sweep variant)
enum ColKernel : int {
    kTuneAdvect1 = 101, kTuneAdvect3, kTuneSmagorinsky, kTuneDivergence, kTuneProjection, kTuneBuoyancy,
    kTuneMgJacobi, kTuneMgResiduum, kTuneMgRestrict, kTuneMgProlongate,
    kTuneMxJacobi0, kTuneMxJacobi, kTuneMxResiduum, kTuneMxRestrict
};

// Launches a column kernel, `launch(grid, block)` returning a status, with the
// tuned shape of (kernel, level shape).  The first eager call of a key times
// every shape (one warm launch, then three) and keeps the fastest in the
// context; the kernel must write the same values when it runs again with the
// same arguments (its output is not its input) and must not reduce (a
// reduction's order would follow the choice; a call whose output aliases an
// input passes may_tune = false).  Inside a capture, with the autotuner off or
// without may_tune, an untuned key launches shape 0.  max_threads: the
// kernel's __launch_bounds__ (shapes with larger blocks are not tried).
template <class F>
int tuned_column_launch(artss_ctx *ctx, int kernel, int level, const Box3 &box, bool may_tune, F launch,
                        unsigned max_threads = 1024) {
    const Level &L = ctx->lvl[level];
    const TuneKey key{kernel, L.Nx, L.Ny, L.Nz, level};
    auto it = ctx->tuned.find(key);
    if (it != ctx->tuned.end()) {
        const ColShape &s = kColShapes[it->second];
        return launch(col_grid(box, s), dim3(s.bx, s.by, 1));
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    // captures that other code opened on the stream count too
    if (!ctx->autotune || ctx->capturing || !may_tune || cudaStreamIsCapturing(ctx->stream, &cs) != cudaSuccess ||
        cs != cudaStreamCaptureStatusNone)
        return launch(col_grid(box, kColShapes[0]), dim3(kBx, kBy, 1));
    cudaEvent_t e0, e1;
    ARTSS_CK(cudaEventCreate(&e0));
    ARTSS_CK(cudaEventCreate(&e1));
    int best = 0, st = ARTSS_OK;
    float best_ms = 1e30f;
    for (int v = 0; v < kColShapeCount && !st; v++) {
        const ColShape &s = kColShapes[v];
        if (s.bx * s.by > max_threads) continue;
        const dim3 g = col_grid(box, s), b(s.bx, s.by, 1);
        if ((st = launch(g, b))) break;
        cudaEventRecord(e0, ctx->stream);
        for (int r = 0; r < 3 && !st; r++) st = launch(g, b);
        cudaEventRecord(e1, ctx->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) { st = cuda_fail(cudaGetLastError(), "launch-shape tuning"); break; }
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) { best_ms = ms; best = v; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    ctx->tuned[key] = best;
    return ARTSS_OK;
}

// Grid-size helper for flat (1-D) loops over n elements.
inline unsigned flat_blocks(int64_t n, int threads = 256) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148 * 16) b = 148 * 16;
    return (unsigned) b;
}

// A reduction pass writes one partial per block; two passes share d_partials.
inline int check_reduce_blocks(const dim3 &g) {
    if (2 * (int64_t) g.x * g.y * g.z > kMaxPartials) {
        set_error("x-y plane too large for the reduction buffer");
        return ARTSS_ERR_LIMIT;
    }
    return ARTSS_OK;
}

// Boundary program execution (bc.cu).
// pred != NULL: every launch returns at once when pred->cond == 0 (predicated loop body)
int apply_bc(artss_ctx *ctx, double *f, int level, int field_type, const LoopState *pred = nullptr);

// Homogeneous boundary program (values zero) on FP32 storage (bc.cu).
int apply_bc_f32(artss_ctx *ctx, float *f, int level, int field_type, const LoopState *pred = nullptr);
// FP64 cluster (block: one-block where the level fits) solve of a level's
// pressure equation on FP32 storage, zero boundary values, tolerance relative
// to the initial residual (mg.cu).
bool cluster_fits(const artss_ctx *ctx, int level, int buffers, int *plane_cap, int64_t *smem);
bool block_fits(const artss_ctx *ctx, int level, int buffers, int64_t *smem);
int coarse_cluster_f32(artss_ctx *ctx, float *out, const float *b, int level, int smoother, double w, double tol,
                       long long max_it, const LoopState *pred, bool block, bool zero_start);

// TMA descriptor of a level array for kTmaBoxX x kTmaBoxY plane windows (tma.cu);
// tma_level_ok: the level's row pitch allows TMA (Nx even).
bool tma_level_ok(const artss_ctx *ctx, int level);
int tensor_map_3d(artss_ctx *ctx, const double *base, int level, const CUtensorMap **out, int box_x = kTmaBoxX,
                  int box_y = kTmaBoxY);

// Reductions (reduce.cu): sum of per-block partials -> loop state `slot`.
//   mode 0: residual = sqrt(sum); it += 1; cond = residual > tol && it < max_it
int finalize_loop(artss_ctx *ctx, int slot, int nblocks, double tol, long long max_it);
int init_loop(artss_ctx *ctx, int slot, double residual0, long long it0, int cond0);
// loop step whose tolerance is rel_tol * sqrt(sum of loop slot ref_slot), on the device
int finalize_loop_rel(artss_ctx *ctx, int slot, int nblocks, double rel_tol, int ref_slot, long long max_it);
int read_loop(artss_ctx *ctx, int slot, LoopState *out);

// A loop inside a whole-step capture: a WHILE conditional node whose body is
// everything enqueued on the context between begin and end (the context's
// stream is the body's capture stream meanwhile).  end() appends the kernel
// that sets the node's condition from loop slot `slot`'s cond, or stops the
// loop (error flag 2) after `cap` bodies.
struct GraphLoop {
    artss_ctx *ctx = nullptr;
    cudaStream_t outer = nullptr;
    cudaGraphNode_t node = nullptr;
    cudaGraphConditionalHandle handle = 0;
    int begin(artss_ctx *c, int cond0);
    int end(int slot, long long cap);
};
// Plain sum of partials into loop slot (no iteration bookkeeping).
int finalize_sum(artss_ctx *ctx, int slot, int nblocks);
// sum of partials -> residual = sqrt(sum), no loop bookkeeping
int finalize_residual(artss_ctx *ctx, int slot, int nblocks);

}  // namespace artss

// Block-wide sum of one double per thread; result valid in thread 0.
__device__ __forceinline__ double artss_block_sum(double v, double *smem) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int nwarps = (blockDim.x * blockDim.y * blockDim.z + 31) >> 5;
    if (lane == 0) smem[warp] = v;
    __syncthreads();
    v = 0.0;
    if (tid < 32) {
        v = (tid < nwarps) ? smem[tid] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    return v;
}

// Launches a kernel inside a ProfScope of the given family.
#define ARTSS_LAUNCH(ctx, fam, ...)                 \
    do {                                            \
        artss::ProfScope ps_((ctx), (fam));         \
        __VA_ARGS__;                                \
    } while (0)

// ARTSS_LAUNCH of a kernel that begins with pdl_wait() (artss::launch_pdl)
#define ARTSS_LAUNCH_PDL(ctx, fam, kern, grid, block, smem, ...)                                       \
    do {                                                                                             \
        cudaError_t e_pdl_;                                                                          \
        {                                                                                            \
            artss::ProfScope ps_((ctx), (fam));                                                      \
            e_pdl_ = artss::launch_pdl((ctx), kern, dim3(grid), dim3(block), (size_t) (smem), __VA_ARGS__); \
        }                                                                                            \
        if (e_pdl_ != cudaSuccess) return artss::cuda_fail(e_pdl_, "kernel launch");                \
    } while (0)
