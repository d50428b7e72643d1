// noalloc.cu -- cave_run_noalloc: the streaming run of cave_run on caller-owned device
// buffers, with the library's scratch (bit-plane copies, simulation record, work items) in one
// file-scope device array instead of memory allocated per grid.
//
// For callers that must not allocate device memory while they run: a serving loop whose
// memory belongs to another allocator (a caching allocator that has reserved the HBM, where a
// cudaMalloc can fail), or one that cannot afford cudaFree's device-wide synchronisation
// between requests. This entry point calls no cudaMalloc, cudaFree or other allocating
// routine; its scratch array is part of the library's device image, so every GPU that loads
// the library holds it (CAVE_NOALLOC_SCRATCH_BYTES) until the process exits.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "../../include/cave_ca.h"
#include "context.h"
#include "kernels.h"
#include "rules.h"
#include "trace.h"

namespace cave {
namespace {

constexpr size_t kScratchBytes = CAVE_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

// The shared scratch. Host code never touches it by name: the device address comes from
// cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mu;
unsigned char* g_scratch_base[kMaxDevices] = {};

constexpr uint64_t align256(uint64_t v) { return (v + 255u) & ~uint64_t(255u); }

// Writes the simulation record into the scratch array. Every field is rewritten, so nothing
// from an earlier call survives in it.
__global__ void k_noalloc_setup(StripSim rec, StripSim* dst) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *dst = rec;
}

// Device address of the scratch array on ctx's device, looked up on the first call there.
cave_status scratch_base(cave_ctx* ctx, unsigned char** out) {
    if (ctx->device < 0 || ctx->device >= kMaxDevices)
        return set_error(ctx, CAVE_ERR_INVALID_ARG, "cave_run_noalloc: device index above 63");
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_base[ctx->device]) {
        void* p = nullptr;
        // With lazy module loading (the CUDA default) this is where the module holding the array
        // is loaded on this device, so this is where its memory is taken.
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);  // ctx's device is current
        if (e == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            return set_error(ctx, CAVE_ERR_OUT_OF_MEMORY,
                             "cave_run_noalloc: the device could not hold the static scratch array "
                             "g_noalloc_scratch (" + std::to_string((uint64_t)kScratchBytes) +
                                 " bytes); make the first call on a device before another allocator "
                                 "reserves its memory");
        }
        if (e != cudaSuccess) return check_cuda(ctx, e, "cudaGetSymbolAddress(scratch)");
        if (!p) return set_error(ctx, CAVE_ERR_CUDA, "cave_run_noalloc: scratch array has no device address");
        g_scratch_base[ctx->device] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_base[ctx->device];
    return CAVE_OK;
}

// Device memory of `device` itself, or managed memory (reachable from every device). Memory of
// another GPU is rejected: without peer access the kernels would fault on it.
bool is_device_pointer(const void* p, int device) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type == cudaMemoryTypeManaged) return true;
    return a.type == cudaMemoryTypeDevice && a.device == device;
}

}  // namespace
}  // namespace cave

using namespace cave;

extern "C" cave_status cave_run_noalloc(cave_ctx* ctx, const uint32_t* d_in, uint32_t* d_out, uint32_t X,
                                        uint32_t Y, uint32_t Z, const cave_sim_params* params,
                                        const uint64_t* validBitmasks, uint32_t nValid, uint32_t maxRuleBits,
                                        uint32_t nticks, uint32_t maxTicks, cave_tick_stats* d_per_tick,
                                        cave_grid_info* info) {
    if (!ctx || !params || !d_in || !d_out) return CAVE_ERR_INVALID_ARG;
    TraceRange trace("cave_run_noalloc");
    DecodedRule d;
    if (!decode_params(*params, validBitmasks, nValid, maxRuleBits, d))
        return set_error(ctx, CAVE_ERR_INVALID_ARG, "rule index outside the valid-bitmask table");
    // the tile shape cave_run uses by default with the library's tick kernel (two CTAs per SM);
    // plan_stream builds the work items in host memory only
    StreamPlan plan;
    if (!plan_stream(0, X, Y, Z, (uint32_t)ctx->sm_count * 2u, 0, plan, 1))
        return set_error(ctx, CAVE_ERR_INVALID_ARG,
                         "grid shape not supported by the streaming kernel (X <= 1024, Y, Z <= 65535)");
    const uint64_t nstrips = (uint64_t)plan.SX * Y * Z;
    const uint64_t n_items = plan.items.size();
    const uint64_t items_off = align256(sizeof(StripSim));
    const uint64_t strips_off = align256(items_off + n_items * sizeof(StreamItem));
    const uint64_t need = strips_off + 2 * nstrips * 16;
    if (need > kScratchBytes)
        return set_error(ctx, CAVE_ERR_INVALID_ARG,
                         "cave_run_noalloc: grid needs " + std::to_string(need) + " bytes of scratch, above the " +
                             std::to_string((uint64_t)kScratchBytes) +
                             "-byte maximum (two bit-plane copies of 16 bytes per 32 x-cells)");
    if ((reinterpret_cast<uintptr_t>(d_in) | reinterpret_cast<uintptr_t>(d_out)) & 3u)
        return set_error(ctx, CAVE_ERR_INVALID_ARG, "cave_run_noalloc: grid buffers must be 4-byte aligned");
    if (d_per_tick && (reinterpret_cast<uintptr_t>(d_per_tick) & 7u))
        return set_error(ctx, CAVE_ERR_INVALID_ARG, "cave_run_noalloc: per-tick buffer must be 8-byte aligned");
    CAVE_CUDA(ctx, cudaSetDevice(ctx->device));
    if (!is_device_pointer(d_in, ctx->device) || !is_device_pointer(d_out, ctx->device) ||
        (d_per_tick && !is_device_pointer(d_per_tick, ctx->device)))
        return set_error(ctx, CAVE_ERR_INVALID_ARG,
                         "cave_run_noalloc: buffers must be device memory of the context's device");
    unsigned char* base = nullptr;
    if (cave_status s = scratch_base(ctx, &base); s != CAVE_OK) return s;

    StripSim* rec_dev = reinterpret_cast<StripSim*>(base);
    StreamItem* items = reinterpret_cast<StreamItem*>(base + items_off);
    uint4* pool = reinterpret_cast<uint4*>(base + strips_off);

    StripSim s;
    std::memset(&s, 0, sizeof(s));
    s.rule = make_device_rule(d);
    s.X = X;
    s.Y = Y;
    s.Z = Z;
    s.SX = plan.SX;
    s.buf[0] = 0;
    s.buf[1] = nstrips * 16;
    s.max_ticks = maxTicks;
    s.tick_limit = nticks;
    s.stop_on_status = 0;
    s.n_items = (uint32_t)n_items;
    for (int k = 0; k < 3; k++) s.acc_bmin[k] = 0xFFFFFFFFu;
    s.per_tick = nticks ? d_per_tick : nullptr;

    // the work items travel by a copy from pageable host memory (staged by the driver in host
    // memory; no device allocation), the record by a one-thread kernel
    cudaError_t e = cudaMemcpyAsync(items, plan.items.data(), sizeof(StreamItem) * n_items, cudaMemcpyHostToDevice,
                                    ctx->stream);
    if (e == cudaSuccess) {
        k_noalloc_setup<<<1, 32, 0, ctx->stream>>>(s, rec_dev);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = launch_nib_to_strips(d_in, pool, X, Y, Z, ctx->stream);
    for (uint32_t k = 0; k < nticks && e == cudaSuccess; k++)
        e = launch_stream_tick((int)(d.flags & 7u), (int)s.rule.nterms, &s.rule, items, (uint32_t)n_items, rec_dev,
                               pool, plan.SX, plan.SXp, plan.threads, ctx->stream);
    // Raw stepping never stops early, so the result is in copy (nticks & 1).
    if (e == cudaSuccess) e = launch_strips_to_nib(pool + (uint64_t)(nticks & 1u) * nstrips, d_out, X, Y, Z, ctx->stream);
    StripSim back;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&back, rec_dev, sizeof(back), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return check_cuda(ctx, e, "cave_run_noalloc");
    if (back.error & kErrBounds) return set_error(ctx, CAVE_ERR_INTERNAL, "streaming kernel: an index check failed");
    if (back.error & kErrWaitTimeout)
        return set_error(ctx, CAVE_ERR_TIMEOUT, "streaming kernel: bulk-copy wait timed out");
    if (back.error) return set_error(ctx, CAVE_ERR_INTERNAL, "streaming kernel raised an error flag");
    if (back.tick != nticks) return set_error(ctx, CAVE_ERR_INTERNAL, "streaming run stopped early");
    if (info) *info = back.info;
    return CAVE_OK;
}
