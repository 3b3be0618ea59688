// Closest-hit / any-hit traversal of the N-wide layouts (Quad: N = 4, Oct: N = 8).
//
// Reference: the Quad and Oct tracer kernels (rt/tracer/HipTracerQuadKernels.cu,
// rt/tracer/HipTracerOctKernels.cu), which give each ray a sub-warp of N lanes
// (lane i tests child i), order the hit children by entry distance on a
// shared-memory stack, and share a leaf's triangles among the lanes.
//
// Here one lane traces one ray (k_trace_wide1):
//   * the lane loads the whole node record with 256-bit loads, tests the
//     node's child boxes (its child count says how many; the empty boxes of
//     unused slots are never visited), continues with the nearest hit child
//     and pushes the other hits farthest first, so the nearest of them is
//     popped next; a sub-warp per ray left most lanes idle on nodes with few
//     hit children and made every leaf's few triangles a shuffle reduction;
//   * the first leaf a lane reaches is postponed until every lane still
//     traversing holds one, then the leaves are tested together (as in the
//     binary tracer);
//   * persistent warps take rays with one atomic per warp when fewer than 20
//     lanes still hold one, as in the binary tracer; the per-ray stack keeps
//     its first entries in shared memory and the rest in local memory, and an
//     overflow is reported as a device error instead of overrunning;
//   * the slab and Woop arithmetic is the binary tracer's, written out step by
//     step, and closest-hit ties in t go to the lower triangle id, so both
//     layouts return the same hits.
#include <algorithm>
#include <climits>
#include <cuda_runtime.h>
#include "hp_device.cuh"
#include "hp_internal.h"

namespace {

constexpr int TRAVERSAL_LIMIT = 1 << 22;

__device__ __forceinline__ float safe_rcp(float d) {
    const float ooeps = 8.2718061255302767e-25f;  // 2^-80 (HipTracerQuadKernels.cu, ray setup)
    return __frcp_rn(fabsf(d) > ooeps ? d : copysignf(ooeps, d));
}

// One lane per ray: the lane loads the whole node (32 N bytes, as 256-bit
// loads), tests its N child boxes itself, continues with the nearest hit
// child and pushes the other hits farthest first, so the nearest of them is
// popped next. Rays are taken by persistent warps as in the binary tracer
// (refill when fewer than RF lanes still hold a ray); each lane's stack keeps
// SST entries in shared memory (one column per thread) and the rest in local
// memory. Leaves are tested by the lane, with the binary tracer's Woop
// arithmetic and tie rule, so the hits equal the binary layout's.
constexpr int TB1 = 128;
constexpr int SST1 = 16;
constexpr int RF1 = 20;
constexpr int SENT1 = 0x76543210;
template <int N> struct wide1_cfg;
template <> struct wide1_cfg<4> { static constexpr int STACK = 64; };
template <> struct wide1_cfg<8> { static constexpr int STACK = 96; };

template <int N, bool ANY_HIT, bool STATS>
__global__ void __launch_bounds__(TB1, N == 4 ? 10 : 8) k_trace_wide1(const float4* __restrict__ rays, int64_t num_rays,
                                                   int4* __restrict__ results, int2* __restrict__ stats,
                                                   const int4* __restrict__ nodes, const float4* __restrict__ woop,
                                                   const int32_t* __restrict__ tri_idx, int max_nodes, int num_refs,
                                                   unsigned long long* ray_counter, int* err,
                                                   const int32_t* __restrict__ order) {
    constexpr int STACK = wide1_cfg<N>::STACK, LST = STACK - SST1;
    __shared__ int s_stack[SST1 * TB1];
    int* sstack = s_stack + threadIdx.x;
    // Entries past the shared part. Left uninitialised: sp counts the pushes
    // that were stored (an overflowing push is dropped and reported), so a pop
    // reads only entries a push wrote.
    int lstack[LST];
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;

    float ox = 0, oy = 0, oz = 0, tmin = 0, dx = 0, dy = 0, dz = 0;
    float ix = 0, iy = 0, iz = 0, oodx = 0, oody = 0, oodz = 0;
    float hit_t = 0, hit_u = 0, hit_v = 0;
    int hit = -1;  // leaf-ordered reference of the closest hit
    int64_t ray = -1;
    int node = SENT1, sp = 0, steps = 0, n_nodes = 0, n_tris = 0;
    int leaf = 0;  // postponed leaf (~index), >= 0 when none
    bool exhausted = false;
    auto pop = [&]() {
        if (sp == 0) {
            node = SENT1;
        } else {
            --sp;
            node = sp < SST1 ? sstack[sp * TB1] : lstack[sp - SST1];
        }
    };
    auto push = [&](int v) {
        if (sp < SST1) sstack[sp * TB1] = v;
        else if (sp < STACK) lstack[sp - SST1] = v;
        else { hp_report(err, HP_DEV_STACK_OVERFLOW, (int)ray); --sp; }
        ++sp;
    };

    while (true) {
        // Refill lanes whose ray is finished (one atomic per warp).
        const bool need = node == SENT1 && !exhausted;
        const unsigned need_mask = __ballot_sync(HP_FULL_MASK, need);
        if (need_mask) {
            const int leader = __ffs(need_mask) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(ray_counter, (unsigned long long)__popc(need_mask));
            base = __shfl_sync(HP_FULL_MASK, base, leader);
            if (need) {
                const int64_t slot = (int64_t)base + __popc(need_mask & lt_mask);
                const int64_t id = (order && slot < num_rays) ? (int64_t)__ldg(order + slot) : slot;
                if (slot < num_rays && (uint64_t)id >= (uint64_t)num_rays) {
                    hp_report(err, HP_DEV_BAD_INDEX, (int)slot);
                    exhausted = true;
                } else if (id < num_rays) {
                    ray = id;
                    const float4 o = __ldg(rays + 2 * id), d = __ldg(rays + 2 * id + 1);
                    ox = o.x; oy = o.y; oz = o.z; tmin = o.w;
                    dx = d.x; dy = d.y; dz = d.z; hit_t = d.w;
                    ix = safe_rcp(d.x); iy = safe_rcp(d.y); iz = safe_rcp(d.z);
                    oodx = __fmul_rn(o.x, ix); oody = __fmul_rn(o.y, iy); oodz = __fmul_rn(o.z, iz);
                    hit = -1; hit_u = hit_v = 0.0f;
                    sp = 0; steps = 0; n_nodes = n_tris = 0;
                    node = 0;
                    leaf = 0;
                } else {
                    exhausted = true;
                }
            }
        }
        if (__all_sync(HP_FULL_MASK, node == SENT1)) break;

        while (true) {
            if (node != SENT1) {
                // interior nodes
                while ((unsigned)node < (unsigned)SENT1) {
                    if (node >= max_nodes || ++steps > TRAVERSAL_LIMIT) {
                        hp_report(err, HP_DEV_BAD_INDEX, node);
                        node = SENT1;
                        leaf = 0;
                        break;
                    }
                    if (STATS) ++n_nodes;
                    const int4* np = nodes + (size_t)node * 2 * N;
                    float4 xy[N];
                    int4 zq[N];
#pragma unroll
                    for (int i = 0; i < N; i += 2) {
                        asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                                     : "=f"(xy[i].x), "=f"(xy[i].y), "=f"(xy[i].z), "=f"(xy[i].w),
                                       "=f"(xy[i + 1].x), "=f"(xy[i + 1].y), "=f"(xy[i + 1].z), "=f"(xy[i + 1].w)
                                     : "l"(np + i));
                        asm volatile("ld.global.nc.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                                     : "=r"(zq[i].x), "=r"(zq[i].y), "=r"(zq[i].z), "=r"(zq[i].w),
                                       "=r"(zq[i + 1].x), "=r"(zq[i + 1].y), "=r"(zq[i + 1].z), "=r"(zq[i + 1].w)
                                     : "l"(np + N + i));
                    }
                    const int nch = zq[N - 3].w;
                    // sort keys: entry distance as an order-preserving uint, misses last
                    uint32_t key[N];
                    int ref[N];
#pragma unroll
                    for (int i = 0; i < N; ++i) {
                        const float lox = __fmaf_rn(xy[i].x, ix, -oodx), hix = __fmaf_rn(xy[i].y, ix, -oodx);
                        const float loy = __fmaf_rn(xy[i].z, iy, -oody), hiy = __fmaf_rn(xy[i].w, iy, -oody);
                        const float loz = __fmaf_rn(__int_as_float(zq[i].x), iz, -oodz);
                        const float hiz = __fmaf_rn(__int_as_float(zq[i].y), iz, -oodz);
                        const float cmin = fmaxf(fmaxf(fminf(lox, hix), fminf(loy, hiy)), fmaxf(fminf(loz, hiz), tmin));
                        const float cmax = fminf(fminf(fmaxf(lox, hix), fmaxf(loy, hiy)), fminf(fmaxf(loz, hiz), hit_t));
                        const bool h = i < nch && cmax >= cmin;
                        key[i] = h ? hp_f2ord(cmin) : 0xFFFFFFFFu;
                        ref[i] = zq[i].z;
                    }
                    // ascending by entry distance (misses last): odd-even transposition
#pragma unroll
                    for (int rd = 0; rd < N; ++rd) {
#pragma unroll
                        for (int i = rd & 1; i + 1 < N; i += 2) {
                            if (key[i + 1] < key[i]) {
                                const uint32_t tk = key[i]; key[i] = key[i + 1]; key[i + 1] = tk;
                                const int tr = ref[i]; ref[i] = ref[i + 1]; ref[i + 1] = tr;
                            }
                        }
                    }
                    if (key[0] == 0xFFFFFFFFu) {
                        pop();
                    } else {
#pragma unroll
                        for (int i = N - 1; i >= 1; --i)
                            if (key[i] != 0xFFFFFFFFu) push(ref[i]);
                        node = ref[0];
                    }
                    // The first leaf a lane reaches waits until every lane still
                    // traversing holds one; then the leaves are tested together.
                    if (node < 0 && leaf >= 0) {
                        leaf = node;
                        pop();
                    }
                    if (!__any_sync(__activemask(), leaf >= 0)) break;
                }
                // leaves: the postponed one, then `node` if it is a leaf too
                while (leaf < 0) {
                    const int li = ~leaf;
                    if (li >= max_nodes || ++steps > TRAVERSAL_LIMIT) {
                        hp_report(err, HP_DEV_BAD_INDEX, li);
                        node = SENT1;
                        leaf = 0;
                        break;
                    }
                    const int4 q = __ldg(nodes + (size_t)li * 2 * N + N);
                    int begin = q.z, end = q.w;
                    if (begin < 0 || end > num_refs || begin > end) {
                        hp_report(err, HP_DEV_BAD_INDEX, begin);
                        begin = end = 0;
                    }
                    bool done = false;
                    for (int tri = begin; tri < end; ++tri) {
                        if (STATS) ++n_tris;
                        const float4 v0 = __ldg(woop + 3 * (int64_t)tri);
                        const float4 v1 = __ldg(woop + 3 * (int64_t)tri + 1);
                        const float ozz = __fmaf_rn(-oz, v0.z, __fmaf_rn(-oy, v0.y, __fmaf_rn(-ox, v0.x, v0.w)));
                        const float den = __fmaf_rn(dz, v0.z, __fmaf_rn(dx, v0.x, __fmul_rn(dy, v0.y)));
                        const float t = __fmul_rn(ozz, __frcp_rn(den));
                        bool closer = t < hit_t;
                        if (!closer && t == hit_t && hit >= 0) closer = __ldg(tri_idx + tri) < __ldg(tri_idx + hit);
                        if (t > tmin && closer) {
                            const float oxx = __fmaf_rn(oz, v1.z, __fmaf_rn(oy, v1.y, __fmaf_rn(ox, v1.x, v1.w)));
                            const float dxx = __fmaf_rn(dz, v1.z, __fmaf_rn(dy, v1.y, __fmul_rn(dx, v1.x)));
                            const float u = __fmaf_rn(t, dxx, oxx);
                            if (u >= 0.0f) {
                                const float4 v2 = __ldg(woop + 3 * (int64_t)tri + 2);
                                const float oyy = __fmaf_rn(oz, v2.z, __fmaf_rn(oy, v2.y, __fmaf_rn(ox, v2.x, v2.w)));
                                const float dyy = __fmaf_rn(dz, v2.z, __fmaf_rn(dx, v2.x, __fmul_rn(dy, v2.y)));
                                const float v = __fmaf_rn(t, dyy, oyy);
                                if (v >= 0.0f && __fadd_rn(u, v) <= 1.0f) {
                                    hit_t = t; hit = tri; hit_u = u; hit_v = v;
                                    if (ANY_HIT) { done = true; break; }
                                }
                            }
                        }
                    }
                    if (done) { sp = 0; node = SENT1; leaf = 0; break; }
                    leaf = node;
                    if (node < 0) pop();
                }
                if (node == SENT1) {
                    if (hit < 0) {
                        reinterpret_cast<int2*>(results)[2 * ray] = make_int2(-1, __float_as_int(hit_t));
                        if (STATS) stats[ray] = make_int2(0, 0);
                    } else {
                        results[ray] = make_int4(__ldg(tri_idx + hit), __float_as_int(hit_t), __float_as_int(hit_u),
                                                 __float_as_int(hit_v));
                        if (STATS) stats[ray] = make_int2(n_nodes, n_tris);
                    }
                }
            }
            __syncwarp();
            if (__popc(__ballot_sync(HP_FULL_MASK, node != SENT1)) < RF1) break;
        }
    }
}

template <int N, bool A, bool S>
hp_status launch_wide_t(hp_ctx* ctx, const hp_bvh_impl* b, int64_t n_refs, const float* rays, int64_t num_rays,
                        int32_t* results, int32_t* stats, unsigned long long* counter, const int32_t* order,
                        cudaStream_t s) {
    int per_sm = 0;
    HP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace_wide1<N, A, S>, TB1, 0));
    int k = std::max(per_sm, 1);
    if (ctx->tune.trace_ctas_per_sm > 0) k = std::min(k, (int)ctx->tune.trace_ctas_per_sm);
    const int64_t rays_per_cta = TB1;
    const int64_t grid = std::max<int64_t>(
        1, std::min<int64_t>((int64_t)ctx->sm_count * k, (num_rays + rays_per_cta - 1) / rays_per_cta));
    const int max_nodes = (int)std::max<int64_t>(2 * b->capacity - 1, 3);
    k_trace_wide1<N, A, S><<<(unsigned)grid, TB1, 0, s>>>(
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
