// Deterministic two-pass reductions and the device-side loop-control block.
//
// Pass 1 (inside the stencil kernels): every block writes one partial sum to
// ctx->d_partials[block].  Pass 2 (here, one block): partials are summed in a
// fixed order, so a residual is reproducible run to run for a given launch
// shape.  The loop block then holds what the reference keeps in host scalars
// (`res`, `it`, the while-condition) of its bounded iteration loops, e.g.
// ARTSS src/diffusion/ColoredGaussSeidelDiffuse.cpp:69-88.
#include "internal.cuh"

namespace artss {

// mode 0: loop step with tolerance tol; 3: the same with tol * sqrt(ref->sum);
// 1: plain sum; 2: sum and its square root
__global__ void k_finalize_loop(const double *__restrict__ partials, int nblocks, LoopState *__restrict__ st,
                                double tol, long long max_it, int mode, const LoopState *__restrict__ ref) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    __shared__ double smem[32];
    if (mode == 3) {
        tol = tol * sqrt(ref->sum);
        mode = 0;
    }
    // a predicated iteration enqueued after the loop ended changes nothing
    if (mode == 0 && !st->cond) return;
    double v = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v += partials[b];
    v = artss_block_sum(v, smem);
    if (threadIdx.x == 0) {
        st->sum = v;
        if (mode == 0) {
            const double r = sqrt(v);
            st->residual = r;
            st->it += 1;
            st->cond = (r > tol && st->it < max_it) ? 1 : 0;
        } else if (mode == 2) {
            st->residual = sqrt(v);
        }
    }
}

__global__ void k_init_loop(LoopState *st, double r0, long long it0, int cond0) {
    pdl_wait();  // launched by launch_pdl: the predecessor's writes are visible after this
    pdl_trigger();
    st->sum = 0.0;
    st->residual = r0;
    st->it = it0;
    st->cond = cond0;
    st->pad = 0;  // error flag of kernels with bounded waits
    st->guard = 0;
}

// last kernel of a graph loop's body: continue while the loop state says so,
// at most `cap` bodies
__global__ void k_loop_continue(LoopState *st, cudaGraphConditionalHandle h, long long cap) {
    int c = st->cond;
    if (++st->guard >= cap && c) {
        c = 0;
        st->cond = 0;
        st->pad = 2;
    }
    cudaGraphSetConditional(h, c ? 1u : 0u);
}

int finalize_loop(artss_ctx *ctx, int slot, int nblocks, double tol, long long max_it) {
    ARTSS_LAUNCH_PDL(ctx, FAM_REDUCE, k_finalize_loop, 1, kReduceThreads, 0, ctx->d_partials, nblocks, ctx->d_loop + slot, tol, max_it, 0, nullptr);
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

int finalize_loop_rel(artss_ctx *ctx, int slot, int nblocks, double rel_tol, int ref_slot, long long max_it) {
    ARTSS_LAUNCH_PDL(ctx, FAM_REDUCE, k_finalize_loop, 1, kReduceThreads, 0, 
                                      ctx->d_partials, nblocks, ctx->d_loop + slot, rel_tol, max_it, 3,
                                      ctx->d_loop + ref_slot);
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

int finalize_sum(artss_ctx *ctx, int slot, int nblocks) {
    ARTSS_LAUNCH_PDL(ctx, FAM_REDUCE, k_finalize_loop, 1, kReduceThreads, 0, ctx->d_partials, nblocks, ctx->d_loop + slot, 0.0, 0, 1, nullptr);
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

int finalize_residual(artss_ctx *ctx, int slot, int nblocks) {
    ARTSS_LAUNCH_PDL(ctx, FAM_REDUCE, k_finalize_loop, 1, kReduceThreads, 0, ctx->d_partials, nblocks, ctx->d_loop + slot, 0.0, 0, 2, nullptr);
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

int init_loop(artss_ctx *ctx, int slot, double r0, long long it0, int cond0) {
    ARTSS_LAUNCH_PDL(ctx, FAM_REDUCE, k_init_loop, 1, 1, 0, ctx->d_loop + slot, r0, it0, cond0);
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

int GraphLoop::begin(artss_ctx *c, int cond0) {
    ctx = c;
    cudaStreamCaptureStatus status;
    cudaGraph_t graph;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    ARTSS_CK(cudaStreamGetCaptureInfo(ctx->stream, &status, nullptr, &graph, &deps, &ndeps));
    if (status != cudaStreamCaptureStatusActive) {
        set_error("a graph loop outside a capture");
        return ARTSS_ERR_ARG;
    }
    ARTSS_CK(cudaGraphConditionalHandleCreate(&handle, graph, cond0 ? 1u : 0u, cudaGraphCondAssignDefault));
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = handle;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    ARTSS_CK(cudaGraphAddNode(&node, graph, deps, ndeps, &p));
    ARTSS_CK(cudaStreamBeginCaptureToGraph(ctx->body_stream, p.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                           cudaStreamCaptureModeRelaxed));
    outer = ctx->stream;
    ctx->stream = ctx->body_stream;
    return ARTSS_OK;
}

int GraphLoop::end(int slot, long long cap) {
    ARTSS_LAUNCH(ctx, FAM_REDUCE, k_loop_continue<<<1, 1, 0, ctx->stream>>>(ctx->d_loop + slot, handle, cap));
    cudaGraph_t body;
    const cudaError_t e = cudaStreamEndCapture(ctx->body_stream, &body);
    ctx->stream = outer;
    ARTSS_CK(e);
    ARTSS_CK(cudaStreamUpdateCaptureDependencies(ctx->stream, &node, 1, cudaStreamSetCaptureDependencies));
    return ARTSS_OK;
}

int read_loop(artss_ctx *ctx, int slot, LoopState *out) {
    ARTSS_CK(cudaMemcpyAsync(ctx->h_loop + slot, ctx->d_loop + slot, sizeof(LoopState), cudaMemcpyDeviceToHost,
                             ctx->stream));
    ARTSS_CK(cudaStreamSynchronize(ctx->stream));
    *out = ctx->h_loop[slot];
    return ARTSS_OK;
}

}  // namespace artss
