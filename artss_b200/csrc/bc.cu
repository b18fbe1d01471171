// Boundary conditions as compiled assignment programs.
//
// The reference applies boundary conditions as a sequence of per-patch loops
// (ARTSS src/domain/Multigrid.cpp:555-572): obstacles in id order, each over
// its six patches, then the six domain patches LEFT..BACK, each cell doing
// x[t] = sign * x[t + ref] + value.  Later writes win on edges and corners and
// some assignments read cells an earlier one wrote.  Running that sequence as
// one GPU pass per patch would cost 6 + 6*obstacles launches per call.
//
// Here the host compiles the sequence once per (level, field type):
//   1. dead writes (overwritten before anyone reads them) are dropped;
//   2. read-after-write chains are folded: an assignment whose source was
//      written earlier re-evaluates that chain from its root cell, step by
//      step with the same roundings, so it no longer reads the intermediate;
//   3. the remaining ordering constraints (a cell read before it is written,
//      chains longer than kBcMaxDepth) are resolved by wave numbers.
// The device executes one kernel per wave (one wave in every configuration
// of the reference tests and benchmarks).  Results are identical to the
// sequential loops.
#include "internal.cuh"

#include <algorithm>
#include <cstring>
#include <unordered_map>

namespace artss {

__global__ void k_bc_wave(double *__restrict__ f, const int64_t *__restrict__ target,
                          const int64_t *__restrict__ root, const uint8_t *__restrict__ depth,
                          const uint8_t *__restrict__ neg, const double *__restrict__ value,
                          int64_t begin, int64_t end, int64_t n_total, const LoopState *__restrict__ pred) {
    // the program's tables are constant: the first assignment's entries are
    // read before waiting for the kernel that wrote f
    const int64_t stride = (int64_t) gridDim.x * blockDim.x;
    int64_t q = begin + blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
    int64_t t = 0, r = 0;
    int d = 0;
    uint8_t m = 0;
    double val[kBcMaxDepth];
    if (q < end) {
        t = target[q];
        r = root[q];
        d = depth[q];
        m = neg[q];
    }
#pragma unroll
    for (int s = 0; s < kBcMaxDepth; s++) val[s] = (q < end && s < d) ? value[s * n_total + q] : 0.0;
    pdl_wait();
    pdl_trigger();
    if (pred && !pred->cond) return;
    while (q < end) {
        double x = f[r];
#pragma unroll
        for (int s = 0; s < kBcMaxDepth; s++) {
            if (s < d) x = ((m >> s) & 1 ? -x : x) + val[s];
        }
        f[t] = x;
        q += stride;
        if (q >= end) break;
        t = target[q];
        r = root[q];
        d = depth[q];
        m = neg[q];
#pragma unroll
        for (int s = 0; s < kBcMaxDepth; s++) val[s] = s < d ? value[s * n_total + q] : 0.0;
    }
}

int apply_bc(artss_ctx *ctx, double *f, int level, int field_type, const LoopState *pred) {
    const BcProgram &p = ctx->bc[level][field_type];
    if (!p.present || p.n == 0) return ARTSS_OK;
    for (int w = 0; w < p.waves; w++) {
        const int64_t b = p.wave_begin[w], e = p.wave_begin[w + 1];
        if (e <= b) continue;
        cudaError_t err;
        ARTSS_LAUNCH(ctx, FAM_BC,
                     err = launch_pdl(ctx, k_bc_wave, dim3((unsigned) flat_blocks(e - b)), dim3(256), 0, f,
                                      (const int64_t *) p.d_target, (const int64_t *) p.d_root,
                                      (const uint8_t *) p.d_depth, (const uint8_t *) p.d_neg,
                                      (const double *) p.d_value, b, e, p.n, pred));
        if (err != cudaSuccess) return cuda_fail(err, "kernel launch");
        ARTSS_LAUNCH_CK(ctx);
    }
    return ARTSS_OK;
}

// The boundary program with every value taken as zero, on FP32 storage: the
// homogeneous conditions of a correction equation (mixed-precision pressure
// solve); only the sign chain of each folded assignment remains.
__global__ void k_bc_wave_f32(float *__restrict__ f, const int64_t *__restrict__ target,
                              const int64_t *__restrict__ root, const uint8_t *__restrict__ depth,
                              const uint8_t *__restrict__ neg, int64_t begin, int64_t end,
                              const LoopState *__restrict__ pred) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    if (pred && !pred->cond) return;
    for (int64_t q = begin + blockIdx.x * (int64_t) blockDim.x + threadIdx.x; q < end;
         q += (int64_t) gridDim.x * blockDim.x) {
        const int d = depth[q];
        const unsigned flips = __popc((unsigned) neg[q] & ((1u << d) - 1u));
        const float x = f[root[q]];
        f[target[q]] = (flips & 1u) ? -x : x;
    }
}

int apply_bc_f32(artss_ctx *ctx, float *f, int level, int field_type, const LoopState *pred) {
    const BcProgram &p = ctx->bc[level][field_type];
    if (!p.present || p.n == 0) return ARTSS_OK;
    for (int w = 0; w < p.waves; w++) {
        const int64_t b = p.wave_begin[w], e = p.wave_begin[w + 1];
        if (e <= b) continue;
        ARTSS_LAUNCH_PDL(ctx, FAM_BC, k_bc_wave_f32, flat_blocks(e - b), 256, 0, 
                                      f, p.d_target, p.d_root, p.d_depth, p.d_neg, b, e, pred);
        ARTSS_LAUNCH_CK(ctx);
    }
    return ARTSS_OK;
}

namespace {

struct Folded {
    int64_t target;
    int64_t root;
    int depth;
    uint8_t neg;
    double value[kBcMaxDepth];
    int wave;
};

}  // namespace

// Compile the ordered assignment list; exposed for the host-side unit test.
int compile_bc(const artss_bc_assign *ops, int64_t n, std::vector<Folded> &out, int &waves) {
    out.clear();
    waves = 0;
    // 1. dead-write elimination, scanning backwards
    std::vector<char> live(n, 0);
    {
        std::unordered_map<int64_t, char> overwritten;  // true: a later live write precedes any read
        overwritten.reserve(n * 2 + 1);
        for (int64_t k = n - 1; k >= 0; k--) {
            auto it = overwritten.find(ops[k].target);
            if (it != overwritten.end() && it->second) continue;  // dead
            live[k] = 1;
            overwritten[ops[k].target] = 1;
            overwritten[ops[k].source] = 0;
        }
    }
    // 2./3. forward pass: fold chains, assign waves
    std::unordered_map<int64_t, int64_t> last_writer;  // cell -> index in out
    std::unordered_map<int64_t, int> max_reader_wave;  // cell -> max wave of ops reading it
    std::unordered_map<int64_t, int> last_write_wave;  // cell -> wave of last write
    out.reserve(n);
    for (int64_t k = 0; k < n; k++) {
        if (!live[k]) continue;
        const artss_bc_assign &a = ops[k];
        Folded f{};
        f.target = a.target;
        int wave = 0;
        auto lw = last_writer.find(a.source);
        bool folded = false;
        if (lw != last_writer.end()) {
            const Folded &prev = out[lw->second];
            // fold only if the chain's root has not been written since it was read
            const bool root_written = last_writer.count(prev.root) != 0;
            if (prev.depth < kBcMaxDepth && !root_written) {
                f.root = prev.root;
                f.depth = prev.depth + 1;
                f.neg = prev.neg;
                for (int s = 0; s < prev.depth; s++) f.value[s] = prev.value[s];
                f.neg |= (a.sign < 0 ? 1 : 0) << prev.depth;
                f.value[prev.depth] = a.value;
                folded = true;
            } else {
                wave = std::max(wave, prev.wave + 1);
            }
        }
        if (!folded) {
            f.root = a.source;
            f.depth = 1;
            f.neg = a.sign < 0 ? 1 : 0;
            f.value[0] = a.value;
        }
        auto mr = max_reader_wave.find(a.target);
        if (mr != max_reader_wave.end()) wave = std::max(wave, mr->second + 1);
        auto ww = last_write_wave.find(a.target);
        if (ww != last_write_wave.end()) wave = std::max(wave, ww->second + 1);
        f.wave = wave;
        last_writer[a.target] = (int64_t) out.size();
        last_write_wave[a.target] = wave;
        auto &r = max_reader_wave[f.root];
        r = std::max(r, wave);
        waves = std::max(waves, wave + 1);
        out.push_back(f);
    }
    return ARTSS_OK;
}

}  // namespace artss

using namespace artss;

extern "C" {

int artss_set_boundary_program(artss_ctx *ctx, int level, int field_type, const artss_bc_assign *ops, int64_t n_ops) {
    int st = check_level(ctx, level);
    if (st) return st;
    if ((st = check_field_type(field_type))) return st;
    if (n_ops < 0 || (n_ops && !ops)) { set_error("bad boundary program"); return ARTSS_ERR_ARG; }
    const Level &L = ctx->lvl[level];
    for (int64_t k = 0; k < n_ops; k++) {
        if (ops[k].target < 0 || ops[k].target >= L.size() || ops[k].source < 0 || ops[k].source >= L.size() ||
            (ops[k].sign != 1 && ops[k].sign != -1)) {
            set_error("boundary assignment " + std::to_string(k) + " out of range");
            return ARTSS_ERR_ARG;
        }
    }
    std::vector<Folded> folded;
    int waves = 0;
    compile_bc(ops, n_ops, folded, waves);
    // group by wave, targets ascending within a wave
    std::stable_sort(folded.begin(), folded.end(), [](const Folded &a, const Folded &b) {
        return a.wave != b.wave ? a.wave < b.wave : a.target < b.target;
    });
    const int64_t n = (int64_t) folded.size();
    std::vector<int64_t> tgt(n), root(n);
    std::vector<int8_t> sign(n);
    std::vector<uint8_t> depth(n), neg(n);
    std::vector<double> val((size_t) kBcMaxDepth * std::max<int64_t>(n, 1), 0.0);
    std::vector<int64_t> begin(waves + 1, 0);
    for (int64_t q = 0; q < n; q++) {
        tgt[q] = folded[q].target;
        root[q] = folded[q].root;
        depth[q] = (uint8_t) folded[q].depth;
        neg[q] = folded[q].neg;
        sign[q] = (__builtin_popcount((unsigned) folded[q].neg & ((1u << folded[q].depth) - 1u)) & 1) ? -1 : 1;
        for (int s = 0; s < kBcMaxDepth; s++) val[s * n + q] = s < folded[q].depth ? folded[q].value[s] : 0.0;
        begin[folded[q].wave + 1] = q + 1;
    }
    for (int w = 1; w <= waves; w++) begin[w] = std::max(begin[w], begin[w - 1]);

    BcProgram &p = ctx->bc[level][field_type];
    ARTSS_CK(cudaStreamSynchronize(ctx->stream));
    cudaFree(p.d_target); cudaFree(p.d_root); cudaFree(p.d_depth); cudaFree(p.d_neg); cudaFree(p.d_value);
    p = BcProgram{};
    p.present = true;
    p.waves = waves;
    p.wave_begin = begin;
    p.n = n;
    p.h_target = tgt;
    p.h_root = root;
    p.h_sign = sign;
    ctx->geom_version++;
    p.zero_values = true;
    for (double v : val) {
        uint64_t bits;
        std::memcpy(&bits, &v, sizeof bits);
        if (bits != 0) p.zero_values = false;
    }
    if (n == 0) return ARTSS_OK;
    ARTSS_CK(cudaMalloc(&p.d_target, n * sizeof(int64_t)));
    ARTSS_CK(cudaMalloc(&p.d_root, n * sizeof(int64_t)));
    ARTSS_CK(cudaMalloc(&p.d_depth, n));
    ARTSS_CK(cudaMalloc(&p.d_neg, n));
    ARTSS_CK(cudaMalloc(&p.d_value, kBcMaxDepth * n * sizeof(double)));
    ARTSS_CK(cudaMemcpyAsync(p.d_target, tgt.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice, ctx->stream));
    ARTSS_CK(cudaMemcpyAsync(p.d_root, root.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice, ctx->stream));
    ARTSS_CK(cudaMemcpyAsync(p.d_depth, depth.data(), n, cudaMemcpyHostToDevice, ctx->stream));
    ARTSS_CK(cudaMemcpyAsync(p.d_neg, neg.data(), n, cudaMemcpyHostToDevice, ctx->stream));
    ARTSS_CK(cudaMemcpyAsync(p.d_value, val.data(), kBcMaxDepth * n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    // the host vectors die with this call
    ARTSS_CK(cudaStreamSynchronize(ctx->stream));
    return ARTSS_OK;
}

int artss_boundary_program_waves(artss_ctx *ctx, int level, int field_type) {
    if (check_level(ctx, level) || check_field_type(field_type)) return -1;
    return ctx->bc[level][field_type].present ? ctx->bc[level][field_type].waves : 0;
}

int artss_apply_boundary(artss_ctx *ctx, double *field, int level, int field_type) {
    int st = check_level(ctx, level);
    if (st) return st;
    if ((st = check_field_type(field_type))) return st;
    if (!field) { set_error("null field"); return ARTSS_ERR_ARG; }
    return apply_bc(ctx, field, level, field_type);
}

}  // extern "C"
