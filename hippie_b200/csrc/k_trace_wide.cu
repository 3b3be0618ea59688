// Closest-hit / any-hit traversal of the N-wide layouts (Quad: N = 4, Oct: N = 8).
//
// Reference: the Quad and Oct tracer kernels (rt/tracer/HipTracerQuadKernels.cu,
// rt/tracer/HipTracerOctKernels.cu): a sub-warp of N lanes per ray, lane i
// testing child i of the node, hits ordered by entry distance and pushed on a
// shared-memory stack so that the nearest child is visited next; a leaf's
// triangles are shared among the lanes and the sub-warp keeps the closest hit.
//
// Here:
//   * the child count of a node decides which lanes test a box, so the empty
//     boxes that fill unused child slots are never visited;
//   * each lane's place on the stack is its rank among the hitting lanes by
//     (entry distance, child slot), nearest on top;
//   * the per-ray stack (STACK_N entries in shared memory) reports an overflow
//     as a device error instead of overrunning;
//   * persistent warps refill finished sub-warps with one atomic per warp when
//     fewer than half of them still traverse;
//   * the slab and Woop arithmetic is the binary tracer's, written out step by
//     step, and closest-hit ties in t go to the lower triangle id, so both
//     layouts return the same hits.
#include <algorithm>
#include <climits>
#include <cuda_runtime.h>
#include "hp_device.cuh"
#include "hp_internal.h"

namespace {

constexpr int TB = 128;
constexpr int TRAVERSAL_LIMIT = 1 << 22;

__device__ __forceinline__ float safe_rcp(float d) {
    const float ooeps = 8.2718061255302767e-25f;  // 2^-80 (HipTracerQuadKernels.cu, ray setup)
    return __frcp_rn(fabsf(d) > ooeps ? d : copysignf(ooeps, d));
}

template <int N> struct wide_cfg;
template <> struct wide_cfg<4> { static constexpr int STACK = 96; };
template <> struct wide_cfg<8> { static constexpr int STACK = 128; };

template <int N, bool ANY_HIT, bool STATS>
__global__ void __launch_bounds__(TB, 12) k_trace_wide(const float4* __restrict__ rays, int64_t num_rays,
                                                   int4* __restrict__ results, int2* __restrict__ stats,
                                                   const int4* __restrict__ nodes, const float4* __restrict__ woop,
                                                   const int32_t* __restrict__ tri_idx, int max_nodes, int num_refs,
                                                   unsigned long long* ray_counter, int* err,
                                                   const int32_t* __restrict__ order) {
    constexpr int R = 32 / N;  // rays per warp
    constexpr int SD = wide_cfg<N>::STACK;
    __shared__ int s_stack[TB / 32][R][SD];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int sub = lane / N, off = lane % N, first = sub * N;
    const unsigned submask = ((N == 32) ? 0xFFFFFFFFu : ((1u << N) - 1u)) << first;
    int* stack = s_stack[warp][sub];

    float ox = 0, oy = 0, oz = 0, tmin = 0, dx = 0, dy = 0, dz = 0;
    float ix = 0, iy = 0, iz = 0, oodx = 0, oody = 0, oodz = 0;
    float hit_t = 0, hit_u = 0, hit_v = 0;
    int hit = -1, hit_id = INT_MAX;  // leaf-ordered reference and its triangle id
    int64_t ray = -1;
    int sp = -1;  // top of the ray's stack; -1 when the sub-warp holds no ray
    int steps = 0, n_nodes = 0, n_tris = 0;
    bool exhausted = false;

    while (true) {
        // Refill sub-warps whose ray is finished (one atomic per warp).
        const bool need = sp < 0 && !exhausted;
        const unsigned need_mask = __ballot_sync(HP_FULL_MASK, need && off == 0);
        if (need_mask) {
            const int leader = __ffs(need_mask) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(ray_counter, (unsigned long long)__popc(need_mask));
            base = __shfl_sync(HP_FULL_MASK, base, leader);
            if (need) {
                const int64_t slot = (int64_t)base + __popc(need_mask & ((1u << first) - 1u));
                const int64_t id = (order && slot < num_rays) ? (int64_t)__ldg(order + slot) : slot;
                if (slot < num_rays && (uint64_t)id >= (uint64_t)num_rays) {
                    if (off == 0) hp_report(err, HP_DEV_BAD_INDEX, (int)slot);
                    exhausted = true;
                } else if (id < num_rays) {
                    ray = id;
                    const float4 o = __ldg(rays + 2 * id), d = __ldg(rays + 2 * id + 1);
                    ox = o.x; oy = o.y; oz = o.z; tmin = o.w;
                    dx = d.x; dy = d.y; dz = d.z; hit_t = d.w;
                    ix = safe_rcp(d.x); iy = safe_rcp(d.y); iz = safe_rcp(d.z);
                    oodx = __fmul_rn(o.x, ix); oody = __fmul_rn(o.y, iy); oodz = __fmul_rn(o.z, iz);
                    hit = -1; hit_id = INT_MAX; hit_u = hit_v = 0.0f;
                    steps = n_nodes = n_tris = 0;
                    if (off == 0) stack[0] = 0;
                    sp = 0;
                } else {
                    exhausted = true;
                }
            }
        }
        if (__all_sync(HP_FULL_MASK, sp < 0)) break;
        __syncwarp();

        // Traverse until fewer than half of the warp's sub-warps hold a ray.
        while (true) {
            if (sp >= 0) {
                const int curr = stack[sp];
                __syncwarp(submask);
                --sp;
                if (++steps > TRAVERSAL_LIMIT) {
                    if (off == 0) hp_report(err, HP_DEV_BAD_INDEX, (int)ray);
                    sp = -1;
                } else if (curr >= 0) {
                    // interior node: lane `off` tests child `off`
                    if (curr >= max_nodes) {
                        if (off == 0) hp_report(err, HP_DEV_BAD_INDEX, curr);
                        sp = -1;
                    } else {
                        if (STATS) ++n_nodes;
                        const int4* np = nodes + (size_t)curr * 2 * N;
                        const float4 xy = __ldg(reinterpret_cast<const float4*>(np) + off);
                        const int4 zq = __ldg(np + N + off);
                        const int nch = __shfl_sync(submask, zq.w, first + N - 3);
                        const float lox = __fmaf_rn(xy.x, ix, -oodx), hix = __fmaf_rn(xy.y, ix, -oodx);
                        const float loy = __fmaf_rn(xy.z, iy, -oody), hiy = __fmaf_rn(xy.w, iy, -oody);
                        const float loz = __fmaf_rn(__int_as_float(zq.x), iz, -oodz);
                        const float hiz = __fmaf_rn(__int_as_float(zq.y), iz, -oodz);
                        const float cmin = fmaxf(fmaxf(fminf(lox, hix), fminf(loy, hiy)), fmaxf(fminf(loz, hiz), tmin));
                        const float cmax = fminf(fminf(fmaxf(lox, hix), fmaxf(loy, hiy)), fminf(fmaxf(loz, hiz), hit_t));
                        const bool h = off < nch && cmax >= cmin;
                        const unsigned hm = (__ballot_sync(submask, h) >> first) & ((1u << N) - 1u);
                        const int nh = __popc(hm);
                        int rank = 0;
#pragma unroll
                        for (int j = 0; j < N; ++j) {
                            const float dj = __shfl_sync(submask, cmin, first + j);
                            rank += ((hm >> j) & 1u) && (dj < cmin || (dj == cmin && j < off));
                        }
                        if (h) {
                            const int pos = sp + nh - rank;
                            if (pos < SD) stack[pos] = zq.z;
                            else hp_report(err, HP_DEV_STACK_OVERFLOW, (int)ray);
                        }
                        sp = min(sp + nh, SD - 1);
                        __syncwarp(submask);
                    }
                } else {
                    // leaf: the lanes share its references
                    const int leaf = ~curr;
                    if (leaf >= max_nodes) {
                        if (off == 0) hp_report(err, HP_DEV_BAD_INDEX, leaf);
                        sp = -1;
                    } else {
                        const int4 q = __ldg(nodes + (size_t)leaf * 2 * N + N);
                        int begin = q.z, end = q.w;
                        if (begin < 0 || end > num_refs || begin > end) {
                            if (off == 0) hp_report(err, HP_DEV_BAD_INDEX, begin);
                            begin = end = 0;
                        }
                        float bt = hit_t, bu = hit_u, bv = hit_v;
                        int bh = hit, bid = hit_id;
                        for (int tri = begin + off; tri < end; tri += N) {
                            if (STATS) ++n_tris;
                            const float4 v0 = __ldg(woop + 3 * (int64_t)tri);
                            const float ozz = __fmaf_rn(-oz, v0.z, __fmaf_rn(-oy, v0.y, __fmaf_rn(-ox, v0.x, v0.w)));
                            const float den = __fmaf_rn(dz, v0.z, __fmaf_rn(dx, v0.x, __fmul_rn(dy, v0.y)));
                            const float t = __fmul_rn(ozz, __frcp_rn(den));
                            if (!(t > tmin) || t > bt) continue;
                            int id = INT_MAX;
                            if (t == bt) {
                                if (bh < 0) continue;  // equal to tmax: not a hit
                                id = __ldg(tri_idx + tri);
                                if (id >= bid) continue;
                            }
                            const float4 v1 = __ldg(woop + 3 * (int64_t)tri + 1);
                            const float oxx = __fmaf_rn(oz, v1.z, __fmaf_rn(oy, v1.y, __fmaf_rn(ox, v1.x, v1.w)));
                            const float dxx = __fmaf_rn(dz, v1.z, __fmaf_rn(dy, v1.y, __fmul_rn(dx, v1.x)));
                            const float u = __fmaf_rn(t, dxx, oxx);
                            if (!(u >= 0.0f)) continue;
                            const float4 v2 = __ldg(woop + 3 * (int64_t)tri + 2);
                            const float oyy = __fmaf_rn(oz, v2.z, __fmaf_rn(oy, v2.y, __fmaf_rn(ox, v2.x, v2.w)));
                            const float dyy = __fmaf_rn(dz, v2.z, __fmaf_rn(dx, v2.x, __fmul_rn(dy, v2.y)));
                            const float v = __fmaf_rn(t, dyy, oyy);
                            if (!(v >= 0.0f) || !(__fadd_rn(u, v) <= 1.0f)) continue;
                            bt = t; bu = u; bv = v; bh = tri;
                            bid = id != INT_MAX ? id : __ldg(tri_idx + tri);
                        }
                        // the closest over the sub-warp: smallest t, then smallest triangle id
#pragma unroll
                        for (int o = N / 2; o > 0; o >>= 1) {
                            const float ot = __shfl_xor_sync(submask, bt, o);
                            const int oid = __shfl_xor_sync(submask, bid, o);
                            const int oh = __shfl_xor_sync(submask, bh, o);
                            const float ou = __shfl_xor_sync(submask, bu, o);
                            const float ov = __shfl_xor_sync(submask, bv, o);
                            if (oh >= 0 && (bh < 0 || ot < bt || (ot == bt && oid < bid))) {
                                bt = ot; bid = oid; bh = oh; bu = ou; bv = ov;
                            }
                        }
                        const bool found = bh != hit;
                        hit_t = bt; hit_u = bu; hit_v = bv; hit = bh; hit_id = bid;
                        if (ANY_HIT && found) sp = -1;
                    }
                }
                if (sp < 0) {
                    int nt = n_tris;
                    if (STATS) {
#pragma unroll
                        for (int o = N / 2; o > 0; o >>= 1) nt += __shfl_xor_sync(submask, nt, o);
                    }
                    if (off == 0) {
                        if (hit < 0) {
                            reinterpret_cast<int2*>(results)[2 * ray] = make_int2(-1, __float_as_int(hit_t));
                            if (STATS) stats[ray] = make_int2(0, 0);
                        } else {
                            results[ray] = make_int4(hit_id, __float_as_int(hit_t), __float_as_int(hit_u),
                                                     __float_as_int(hit_v));
                            if (STATS) stats[ray] = make_int2(n_nodes, nt);
                        }
                    }
                }
            }
            __syncwarp();
            if (__popc(__ballot_sync(HP_FULL_MASK, sp >= 0 && off == 0)) * 2 < R) break;
        }
    }
}

template <int N, bool A, bool S>
hp_status launch_wide_t(hp_ctx* ctx, const hp_bvh_impl* b, int64_t n_refs, const float* rays, int64_t num_rays,
                        int32_t* results, int32_t* stats, unsigned long long* counter, const int32_t* order,
                        cudaStream_t s) {
    int per_sm = 0;
    HP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace_wide<N, A, S>, TB, 0));
    int k = std::max(per_sm, 1);
    if (ctx->tune.trace_ctas_per_sm > 0) k = std::min(k, (int)ctx->tune.trace_ctas_per_sm);
    const int64_t rays_per_cta = TB / N;
    const int64_t grid = std::max<int64_t>(
        1, std::min<int64_t>((int64_t)ctx->sm_count * k, (num_rays + rays_per_cta - 1) / rays_per_cta));
    const int max_nodes = (int)std::max<int64_t>(2 * b->capacity - 1, 3);
    k_trace_wide<N, A, S><<<(unsigned)grid, TB, 0, s>>>(
        reinterpret_cast<const float4*>(rays), num_rays, reinterpret_cast<int4*>(results),
        reinterpret_cast<int2*>(stats), reinterpret_cast<const int4*>(b->nodes), b->woop, b->tri_idx, max_nodes,
        (int)n_refs, counter, ctx->d_status, order);
    HP_CUDA(cudaGetLastError());
    hp_count_launch();
    hp_mark(ctx, s, "trace");
    return HP_OK;
}

template <int N>
hp_status launch_wide_n(hp_ctx* ctx, const hp_bvh_impl* b, int64_t n_refs, const float* rays, int64_t num_rays,
                        int32_t* results, int32_t* stats, uint32_t flags, unsigned long long* counter,
                        const int32_t* order, cudaStream_t s) {
    const bool any = flags & HP_TRACE_ANY_HIT, st = (flags & HP_TRACE_STATS) && stats;
    if (any && st) return launch_wide_t<N, true, true>(ctx, b, n_refs, rays, num_rays, results, stats, counter, order, s);
    if (any) return launch_wide_t<N, true, false>(ctx, b, n_refs, rays, num_rays, results, stats, counter, order, s);
    if (st) return launch_wide_t<N, false, true>(ctx, b, n_refs, rays, num_rays, results, stats, counter, order, s);
    return launch_wide_t<N, false, false>(ctx, b, n_refs, rays, num_rays, results, stats, counter, order, s);
}

}  // namespace

hp_status hp_trace_wide_launch(hp_ctx* ctx, const hp_bvh_impl* b, int64_t n_refs, const float* rays,
                               int64_t num_rays, int32_t* results, int32_t* stats, uint32_t flags,
                               unsigned long long* counter, const int32_t* order, cudaStream_t s) {
    if (b->layout == 4)
        return launch_wide_n<4>(ctx, b, n_refs, rays, num_rays, results, stats, flags, counter, order, s);
    if (b->layout == 8)
        return launch_wide_n<8>(ctx, b, n_refs, rays, num_rays, results, stats, flags, counter, order, s);
    return hp_fail(HP_ERR_UNSUPPORTED, "trace: unknown node layout");
}
