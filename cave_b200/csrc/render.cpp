// render.cpp -- cave_render_*: the render mode's tick on its own cell buffers.
//
// Render mode (rayMarchCompute.slang:211-280) steps the same rule as search mode but on the
// Morton-tiled, two-cells-per-texel buffer of cellStateUtils.slang:18-54, and wraps around
// every axis when the W neighbourhood flag is set (simulationRenderer.cpp:595, :623). The
// entry point converts that buffer into the strip layout -- with a one-cell ghost shell
// holding the opposite faces when wrapping -- runs the streaming tick kernel, refreshing the
// shell before every tick, and converts back; the skip grid of the last tick is optional.
#include <cuda_runtime.h>

#include <cstring>

#include "../../include/cave_ca.h"
#include "context.h"
#include "jit.h"
#include "kernels.h"
#include "rules.h"
#include "trace.h"

using namespace cave;

extern "C" {

uint64_t cave_render_buffer_elements(uint32_t X, uint32_t Y, uint32_t Z) {
    return render_geometry(X, Y, Z, 0).elements;
}

uint64_t cave_render_skip_elements(uint32_t X, uint32_t Y, uint32_t Z) {
    return render_geometry(X, Y, Z, 0).skip_elements;
}

cave_status cave_render_step(cave_ctx* ctx, const uint32_t* d_in, uint32_t* d_out, uint32_t X, uint32_t Y, uint32_t Z,
                             const cave_sim_params* params, uint32_t nticks, uint32_t* d_skip) {
    if (!ctx || !params || !d_in || !d_out) return CAVE_ERR_INVALID_ARG;
    TraceRange trace("cave_render_step");
    if (X == 0 || Y == 0 || Z == 0 || (uint64_t)X * Y * Z >= (1ull << 32))
        return set_error(ctx, CAVE_ERR_INVALID_ARG, "grid volume must be in [1, 2^32)");
    DecodedRule d;
    decode_params(*params, nullptr, 0, 0, d);
    const uint32_t pad = (d.flags & 8u) ? 1u : 0u;  // W flag: WRAP_AT_BOUNDARY
    const RenderGeom g = render_geometry(X, Y, Z, pad);
    CAVE_CUDA(ctx, cudaSetDevice(ctx->device));
    // the rule-specialised kernels when ready (jit.h; kJitRowsPerThread rows per thread, one CTA
    // per SM-equivalent), else the generic one
    const JitKernels jk = nticks ? jit_stream_kernel(jit_key(make_device_rule(d)), jit_mode(),
                                                     (uint64_t)X * Y * Z >= kJitMinCells)
                                 : JitKernels{};
    StreamPlan plan;
    bool planned = jk ? plan_stream(0, g.Xp, g.Yp, g.Zp, (uint32_t)ctx->sm_count, 0, plan, kJitRowsPerThread)
                      : plan_stream(0, g.Xp, g.Yp, g.Zp, (uint32_t)ctx->sm_count * 2u, 0, plan);
    if (planned && jk && plan.threads < (uint32_t)kJitMaxThreads)
        planned = plan_stream(0, g.Xp, g.Yp, g.Zp, (uint32_t)ctx->sm_count * ((uint32_t)kJitMaxThreads / plan.threads),
                              plan.rows, plan, kJitRowsPerThread);
    if (!planned)
        return set_error(ctx, CAVE_ERR_INVALID_ARG, "render grid too large for the streaming kernel (X <= 1022)");
    const uint64_t nstrips = (uint64_t)g.SX * g.Yp * g.Zp;
    uint4* strips = nullptr;
    StripSim* rec = nullptr;
    StreamItem* items = nullptr;
    struct Free {
        void* p[4];
        ~Free() {
            for (void* q : p) cudaFree(q);
        }
    } fr{{nullptr, nullptr, nullptr, nullptr}};
    CAVE_CUDA(ctx, cudaMalloc(&strips, nstrips * 16 * 2));
    fr.p[0] = strips;
    CAVE_CUDA(ctx, cudaMalloc(&rec, sizeof(StripSim)));
    fr.p[1] = rec;
    CAVE_CUDA(ctx, cudaMalloc(&items, sizeof(StreamItem) * plan.items.size()));
    fr.p[2] = items;
    TickTotals* tt = nullptr;  // per-tick totals, folded after the last tick
    if (nticks) {
        CAVE_CUDA(ctx, cudaMalloc(&tt, sizeof(TickTotals) * nticks));
        fr.p[3] = tt;
        CAVE_CUDA(ctx, cudaMemsetAsync(tt, 0, sizeof(TickTotals) * nticks, ctx->stream));
    }
    StripSim s;
    std::memset(&s, 0, sizeof(s));
    s.rule = make_device_rule(d);
    s.X = g.Xp;
    s.Y = g.Yp;
    s.Z = g.Zp;
    s.SX = g.SX;
    s.buf[0] = 0;
    s.buf[1] = nstrips * 16;
    s.max_ticks = nticks;
    s.tick_limit = nticks;
    s.stop_on_status = 0;
    s.n_items = (uint32_t)plan.items.size();
    for (int k = 0; k < 3; k++) s.acc_bmin[k] = 0xFFFFFFFFu;
    s.deferred = tt;
    cudaError_t e = cudaMemcpyAsync(rec, &s, sizeof(s), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(items, plan.items.data(), sizeof(StreamItem) * plan.items.size(), cudaMemcpyHostToDevice,
                            ctx->stream);
    if (e == cudaSuccess) e = launch_render_to_strips(d_in, strips, g, ctx->stream);
    // (the first tick of the specialised kernels counts every statistic; later ticks leave the
    // zero cells to the fold)
    for (uint32_t t = 0; t < nticks && e == cudaSuccess; t++) {
        if (pad) e = launch_ghost_fill(strips + (uint64_t)(t & 1u) * nstrips, g, ctx->stream);
        const bool pdl = t > 0 && !pad;
        if (e == cudaSuccess)
            e = jk ? launch_stream_tick_jit(jk.pick(t == 0, plan.SX == plan.SXp), items, (uint32_t)plan.items.size(), rec, strips, plan.SX, plan.SXp,
                                            plan.threads, ctx->stream, pdl, (int)t)
                   : launch_stream_tick((int)(d.flags & 7u), (int)s.rule.nterms, &s.rule, items,
                                        (uint32_t)plan.items.size(), rec, strips, plan.SX, plan.SXp, plan.threads,
                                        ctx->stream, pdl, (int)t);
    }
    if (e == cudaSuccess && nticks && jk)  // the last tick's population comes from the final grid
        e = launch_strip_stats(strips + (uint64_t)(nticks & 1u) * nstrips, g.Yp, g.Zp, g.SX, tt + (nticks - 1),
                               (uint32_t)ctx->sm_count, ctx->stream);
    if (e == cudaSuccess && nticks) e = launch_fold_deferred(rec, tt, nticks, (bool)jk, ctx->stream);
    const uint4* last = strips + (uint64_t)(nticks & 1u) * nstrips;
    if (e == cudaSuccess) e = launch_strips_to_render(last, d_out, g, ctx->stream);
    if (e == cudaSuccess && d_skip) e = launch_render_skip(last, d_skip, g, ctx->stream);
    StripSim back;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&back, rec, sizeof(back), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return check_cuda(ctx, e, "cave_render_step");
    if (back.error & kErrBounds) return set_error(ctx, CAVE_ERR_INTERNAL, "streaming kernel: an index check failed");
    if (back.error & kErrWaitTimeout) return set_error(ctx, CAVE_ERR_TIMEOUT, "streaming kernel: bulk-copy wait timed out");
    if (back.error) return set_error(ctx, CAVE_ERR_INTERNAL, "streaming kernel raised an error flag");
    if (back.tick != nticks) return set_error(ctx, CAVE_ERR_INTERNAL, "render step ran a different number of ticks");
    return CAVE_OK;
}

}  // extern "C"
