// Persistent-warp closest-hit / any-hit traversal of the 64-byte binary BVH.
//
// Reference: HipTracer::trace (rt/tracer/HipTracer.cpp:13-52) and the Aila-Laine
// while-while kernel `trace` / `traceStats` (rt/tracer/HipTracerBinKernels.cu:19-286,
// 290-568): persistent warps that take rays from a global counter, near child
// first, a per-ray stack with a sentinel bottom entry, slab tests against both
// children of a node, Woop triangle tests, and a refill of finished lanes when
// fewer than 20 lanes of a warp still traverse.
//
// Differences by design:
//   * the traversal stack (64 entries) is split: its first SST entries (16 by
//     default; 8 or 32 as a tuning choice) live in shared memory
//     (bank-conflict-free, one column per thread), deeper entries in local memory;
//   * every floating-point step is written out (fma, IEEE reciprocal), so a CPU
//     restatement of the per-ray algorithm reproduces the results bit for bit;
//     the first leaf a lane meets is postponed as in the reference, which can
//     change the order in which a ray tests its leaves but not its closest hit
//     unless two candidate hits lie within rounding of a node's slab distance;
//   * closest-hit ties in t are resolved to the lower triangle id.
#include <cuda_runtime.h>
#include "hp_device.cuh"
#include "hp_internal.h"

namespace {

#define HP_TRACE_RCP(x) __frcp_rn(x)
#include "k_trace_impl.cuh"

// Empty BVH: every ray misses.
__global__ void k_trace_empty(const float4* rays, int64_t num_rays, int4* results, int2* stats) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= num_rays) return;
    reinterpret_cast<int2*>(results)[2 * i] = make_int2(-1, __float_as_int(rays[2 * i + 1].w));
    if (stats) stats[i] = make_int2(0, 0);
}

template <bool A, bool S, int SST>
hp_status launch_batch_t(hp_ctx* ctx, const hp_batch_trace_args& t, unsigned long long* counter, cudaStream_t s) {
    int per_sm = 0;
    HP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace<A, S, true, SST>, TRACE_BLOCK, 0));
    k_trace<A, S, true, SST><<<trace_grid(ctx, per_sm, t.num_rays), TRACE_BLOCK, 0, s>>>(
        reinterpret_cast<const float4*>(t.rays), t.num_rays, reinterpret_cast<int4*>(t.results),
        reinterpret_cast<int2*>(t.stats), reinterpret_cast<const float4*>(t.nodes), t.woop, t.tri_idx, 0, 0,
        counter, ctx->d_status, t.segs, t.ray_off, t.num_segs, nullptr);
    HP_CUDA(cudaGetLastError());
    hp_count_launch();
    return HP_OK;
}

template <bool A, bool S>
hp_status launch_batch_st(hp_ctx* ctx, const hp_batch_trace_args& t, unsigned long long* counter, cudaStream_t s) {
    switch (ctx->tune.trace_stack) {
        case 8: return launch_batch_t<A, S, 8>(ctx, t, counter, s);
        case 32: return launch_batch_t<A, S, 32>(ctx, t, counter, s);
        default: return launch_batch_t<A, S, 16>(ctx, t, counter, s);
    }
}

}  // namespace

hp_status hp_trace_batch_launch(hp_ctx* ctx, const hp_batch_trace_args& t, uint32_t flags, cudaStream_t s) {
    if (t.num_rays <= 0) return HP_OK;
    unsigned long long* counter = reinterpret_cast<unsigned long long*>(ctx->d_status + 16);
    HP_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s));
    const bool any = flags & HP_TRACE_ANY_HIT, st = (flags & HP_TRACE_STATS) && t.stats;
    if (any && st) return launch_batch_st<true, true>(ctx, t, counter, s);
    if (any) return launch_batch_st<true, false>(ctx, t, counter, s);
    if (st) return launch_batch_st<false, true>(ctx, t, counter, s);
    return launch_batch_st<false, false>(ctx, t, counter, s);
}

hp_status hp_trace_launch(hp_ctx* ctx, const hp_bvh_impl* b, int64_t n_refs, const float* rays,
                          int64_t num_rays, int32_t* results, int32_t* stats, uint32_t flags,
                          cudaStream_t s, const int32_t* order, unsigned long long* counter) {
    if (num_rays <= 0) return HP_OK;
    if (n_refs <= 0) {
        k_trace_empty<<<hp_div_up(num_rays, 256), 256, 0, s>>>(
            reinterpret_cast<const float4*>(rays), num_rays, reinterpret_cast<int4*>(results),
            reinterpret_cast<int2*>(stats));
        HP_CUDA(cudaGetLastError());
        hp_count_launch();
        return HP_OK;
    }
    if (!counter) counter = reinterpret_cast<unsigned long long*>(ctx->d_status + 16);
    HP_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s));
    hp_mark(ctx, s, "trace_begin");
    if (b->layout != 2)
        return hp_trace_wide_launch(ctx, b, n_refs, rays, num_rays, results, stats, flags, counter, order, s);
    if (ctx->arith == HP_ARITH_REFERENCE)
        return hp_trace_ref_launch(ctx, b, n_refs, rays, num_rays, results, stats, flags, counter, order, s);
    const bool any = flags & HP_TRACE_ANY_HIT, st = (flags & HP_TRACE_STATS) && stats;
    if (any && st) return launch_st<true, true>(ctx, b, n_refs, rays, num_rays, results, stats, counter, order, s);
    if (any) return launch_st<true, false>(ctx, b, n_refs, rays, num_rays, results, stats, counter, order, s);
    if (st) return launch_st<false, true>(ctx, b, n_refs, rays, num_rays, results, stats, counter, order, s);
    return launch_st<false, false>(ctx, b, n_refs, rays, num_rays, results, stats, counter, order, s);
}
