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

__global__ void k_finalize_loop(const double *__restrict__ partials, int nblocks, LoopState *__restrict__ st,
                                double tol, long long max_it, int mode) {
    __shared__ double smem[32];
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
    st->sum = 0.0;
    st->residual = r0;
    st->it = it0;
    st->cond = cond0;
    st->pad = 0;  // error flag of kernels with bounded waits
}

int finalize_loop(artss_ctx *ctx, int slot, int nblocks, double tol, long long max_it) {
    ARTSS_LAUNCH(ctx, FAM_REDUCE, k_finalize_loop<<<1, kReduceThreads, 0, ctx->stream>>>(ctx->d_partials, nblocks, ctx->d_loop + slot, tol, max_it, 0));
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

int finalize_sum(artss_ctx *ctx, int slot, int nblocks) {
    ARTSS_LAUNCH(ctx, FAM_REDUCE, k_finalize_loop<<<1, kReduceThreads, 0, ctx->stream>>>(ctx->d_partials, nblocks, ctx->d_loop + slot, 0.0, 0, 1));
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

int finalize_residual(artss_ctx *ctx, int slot, int nblocks) {
    ARTSS_LAUNCH(ctx, FAM_REDUCE, k_finalize_loop<<<1, kReduceThreads, 0, ctx->stream>>>(ctx->d_partials, nblocks, ctx->d_loop + slot, 0.0, 0, 2));
    ARTSS_LAUNCH_CK(ctx);
    return ARTSS_OK;
}

int init_loop(artss_ctx *ctx, int slot, double r0, long long it0, int cond0) {
    ARTSS_LAUNCH(ctx, FAM_REDUCE, k_init_loop<<<1, 1, 0, ctx->stream>>>(ctx->d_loop + slot, r0, it0, cond0));
    ARTSS_LAUNCH_CK(ctx);
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
