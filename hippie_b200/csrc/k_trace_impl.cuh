// The persistent-warp binary-BVH tracer, shared by two translation units that
// differ only in their reciprocal and compiler flags:
//   k_trace.cu      HP_TRACE_RCP(x) = __frcp_rn(x), IEEE round-to-nearest (the
//                   library's default arithmetic, reproduced bit for bit by the
//                   CPU oracle);
//   k_refarith.cu   HP_TRACE_RCP(x) = 1.0f / x compiled with -use_fast_math:
//                   the quotient and denormal flushing of the reference's
//                   fast-math build (gpu/HipCompiler.cpp:127-129), so that its
//                   hits can be reproduced bit for bit. Every other operation
//                   here is an explicit __fmaf_rn / __fmul_rn / __fadd_rn,
//                   which that flag does not contract further.
// Included inside an anonymous namespace after hp_device.cuh / hp_internal.h,
// with HP_TRACE_RCP defined.
#ifndef HP_TRACE_RCP
#error "define HP_TRACE_RCP before including k_trace_impl.cuh"
#endif

constexpr int TRACE_BLOCK = 128;
constexpr int STACK = 64;         // traversal stack entries per ray: SST in shared memory, the rest local
constexpr int SENTINEL = 0x76543210;
constexpr int FETCH_THRESHOLD = 20;
constexpr int TRAVERSAL_LIMIT = 1 << 22;  // visits per ray before the ray is abandoned with an error

struct ray_state {
    float ox, oy, oz, tmin, dx, dy, dz;
    float idx_, idy, idz, oodx, oody, oodz;
    float hit_t, hit_u, hit_v;
    int hit;       // woop / leaf-ordered reference index of the closest hit, -1 if none
    int nodes, tris;
};

// One 32-byte read-only load (sm_100 vector width); p must be 32-byte aligned.
__device__ __forceinline__ void ld32(const float4* p, float4& a, float4& b) {
    asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
                 : "l"(p));
}

__device__ __forceinline__ float safe_rcp(float d) {
    // idir = 1 / (|d| > 2^-80 ? d : copysign(2^-80, d)) (HipTracerBinKernels.cu:83-86)
    const float ooeps = 8.2718061255302767e-25f;  // 2^-80
    return HP_TRACE_RCP(fabsf(d) > ooeps ? d : copysignf(ooeps, d));
}

// Index of the segment containing element g: the last m with off[m] <= g.
__device__ __forceinline__ int seg_search(const int64_t* __restrict__ off, int num_segs, int64_t g) {
    int lo = 0, hi = num_segs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(off + mid) <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// BATCH: rays of many meshes in one launch; ray g belongs to the segment whose
// ray range holds it, and the lane traverses that mesh's BVH.
template <bool ANY_HIT, bool STATS, bool BATCH, int SST>
__global__ void __launch_bounds__(TRACE_BLOCK, BATCH ? 9 : 12) k_trace(
    const float4* __restrict__ rays, int64_t num_rays, int4* __restrict__ results,
    int2* __restrict__ stats, const float4* __restrict__ nodes_all, const float4* __restrict__ woop_all,
    const int32_t* __restrict__ tri_all, int max_nodes_all, int num_refs_all,
    unsigned long long* ray_counter, int* err, const hp_batch_seg* __restrict__ segs,
    const int64_t* __restrict__ ray_off, int num_segs, const int32_t* __restrict__ order) {
    constexpr int SSTACK = SST, LSTACK = STACK - SST;
    __shared__ int s_stack[SSTACK * TRACE_BLOCK];
    int* sstack = s_stack + threadIdx.x;
    int lstack[LSTACK];
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;

    ray_state r;
    int64_t ray = -1;
    int node = SENTINEL;
    int leaf = 0;   // postponed leaf (~index), >= 0 when none
    int sp = 0;
    int steps = 0;  // node + leaf visits of the current ray (bounded)
    bool exhausted = false;
    const float4* nodes = nodes_all;
    const float4* woop = woop_all;
    const int32_t* tri_idx = tri_all;
    int max_nodes = max_nodes_all, num_refs = num_refs_all;

    while (true) {
        // Refill lanes whose ray is finished (one atomic per warp).
        const bool need = (node == SENTINEL) && !exhausted;
        const unsigned need_mask = __ballot_sync(HP_FULL_MASK, need);
        if (need_mask) {
            const int leader = __ffs(need_mask) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(ray_counter, (unsigned long long)__popc(need_mask));
            base = __shfl_sync(HP_FULL_MASK, base, leader);
            if (need) {
                const int64_t slot = (int64_t)base + __popc(need_mask & lt_mask);
                // traceSort: slot k traces ray order[k] (rays in Morton order)
                const int64_t id = (order && slot < num_rays) ? (int64_t)__ldg(order + slot) : slot;
                if (slot < num_rays && (uint64_t)id >= (uint64_t)num_rays) {
                    hp_report(err, HP_DEV_BAD_INDEX, (int)slot);
                    exhausted = true;
                } else if (id < num_rays) {
                    ray = id;
                    const float4 o = __ldg(rays + 2 * id), d = __ldg(rays + 2 * id + 1);
                    r.ox = o.x; r.oy = o.y; r.oz = o.z; r.tmin = o.w;
                    r.dx = d.x; r.dy = d.y; r.dz = d.z; r.hit_t = d.w;
                    r.idx_ = safe_rcp(d.x); r.idy = safe_rcp(d.y); r.idz = safe_rcp(d.z);
                    r.oodx = __fmul_rn(o.x, r.idx_);
                    r.oody = __fmul_rn(o.y, r.idy);
                    r.oodz = __fmul_rn(o.z, r.idz);
                    r.hit = -1;
                    r.hit_u = r.hit_v = 0.0f;
                    r.nodes = r.tris = 0;
                    sp = 0;
                    steps = 0;
                    leaf = 0;
                    node = 0;
                    if (BATCH) {
                        const hp_batch_seg& g = segs[seg_search(ray_off, num_segs, id)];
                        nodes = nodes_all + 4 * g.node_off;
                        woop = woop_all + 3 * (int64_t)g.tri_off;
                        tri_idx = tri_all + g.tri_off;
                        num_refs = g.n;
                        max_nodes = max(2 * g.n - 1, 3);
                        if (g.n == 0) {  // empty mesh: the ray misses
                            reinterpret_cast<int2*>(results)[2 * id] = make_int2(-1, __float_as_int(d.w));
                            if (STATS) stats[id] = make_int2(0, 0);
                            node = SENTINEL;
                        }
                    }
                } else {
                    exhausted = true;
                }
            }
        }
        if (__all_sync(HP_FULL_MASK, node == SENTINEL)) {
            if (!BATCH || __all_sync(HP_FULL_MASK, exhausted)) break;
            continue;  // every lane drew a ray of an empty mesh
        }

        // Traverse until fewer than FETCH_THRESHOLD lanes of the warp still hold
        // a ray; the warp reconverges after every round so that the decision
        // (and the refill that follows) is taken by all 32 lanes together.
        while (true) {
          if (node != SENTINEL) {
            // Interior nodes. The first leaf a lane reaches is postponed and the
            // lane keeps traversing until every lane still traversing holds a
            // leaf (or finishes); then the leaves are tested together.
            while ((unsigned)node < (unsigned)SENTINEL) {
                if (node >= max_nodes || ++steps > TRAVERSAL_LIMIT) {
                    hp_report(err, HP_DEV_BAD_INDEX, node);
                    node = SENTINEL;
                    leaf = 0;
                    break;
                }
                if (STATS) ++r.nodes;
                const float4* np = nodes + 4 * (int64_t)node;
                float4 n0, n1, nz, nm;
                ld32(np, n0, n1);
                ld32(np + 2, nz, nm);
                const float c0lox = __fmaf_rn(n0.x, r.idx_, -r.oodx);
                const float c0hix = __fmaf_rn(n0.y, r.idx_, -r.oodx);
                const float c0loy = __fmaf_rn(n0.z, r.idy, -r.oody);
                const float c0hiy = __fmaf_rn(n0.w, r.idy, -r.oody);
                const float c0loz = __fmaf_rn(nz.x, r.idz, -r.oodz);
                const float c0hiz = __fmaf_rn(nz.y, r.idz, -r.oodz);
                const float c1loz = __fmaf_rn(nz.z, r.idz, -r.oodz);
                const float c1hiz = __fmaf_rn(nz.w, r.idz, -r.oodz);
                const float c1lox = __fmaf_rn(n1.x, r.idx_, -r.oodx);
                const float c1hix = __fmaf_rn(n1.y, r.idx_, -r.oodx);
                const float c1loy = __fmaf_rn(n1.z, r.idy, -r.oody);
                const float c1hiy = __fmaf_rn(n1.w, r.idy, -r.oody);
                const float c0min = fmaxf(fmaxf(fminf(c0lox, c0hix), fminf(c0loy, c0hiy)),
                                          fmaxf(fminf(c0loz, c0hiz), r.tmin));
                const float c0max = fminf(fminf(fmaxf(c0lox, c0hix), fmaxf(c0loy, c0hiy)),
                                          fminf(fmaxf(c0loz, c0hiz), r.hit_t));
                const float c1min = fmaxf(fmaxf(fminf(c1lox, c1hix), fminf(c1loy, c1hiy)),
                                          fmaxf(fminf(c1loz, c1hiz), r.tmin));
                const float c1max = fminf(fminf(fmaxf(c1lox, c1hix), fmaxf(c1loy, c1hiy)),
                                          fminf(fmaxf(c1loz, c1hiz), r.hit_t));
                const bool t0 = c0max >= c0min, t1 = c1max >= c1min;
                int c0 = __float_as_int(nm.x), c1 = __float_as_int(nm.y);
                if (!t0 && !t1) {
                    if (sp == 0) node = SENTINEL;
                    else { --sp; node = sp < SSTACK ? sstack[sp * TRACE_BLOCK] : lstack[sp - SSTACK]; }
                } else {
                    node = t0 ? c0 : c1;
                    if (t0 && t1) {
                        int far = c1;
                        if (c1min < c0min) { node = c1; far = c0; }
                        if (sp < SSTACK) sstack[sp * TRACE_BLOCK] = far;
                        else if (sp < SSTACK + LSTACK) lstack[sp - SSTACK] = far;
                        else { hp_report(err, HP_DEV_STACK_OVERFLOW, (int)ray); --sp; }
                        ++sp;
                    }
                }
                if (node < 0 && leaf >= 0) {  // postpone the first leaf
                    leaf = node;
                    if (sp == 0) node = SENTINEL;
                    else { --sp; node = sp < SSTACK ? sstack[sp * TRACE_BLOCK] : lstack[sp - SSTACK]; }
                }
                if (!__any_sync(__activemask(), leaf >= 0)) break;
            }
            // Leaves: the postponed one, then `node` if it is a leaf too.
            while (leaf < 0) {
                if (~leaf >= max_nodes || ++steps > TRAVERSAL_LIMIT) {
                    hp_report(err, HP_DEV_BAD_INDEX, leaf);
                    node = SENTINEL;
                    leaf = 0;
                    break;
                }
                const float4 lm = __ldg(nodes + 4 * (int64_t)(~leaf) + 3);
                int begin = __float_as_int(lm.x), end = __float_as_int(lm.y);
                if (begin < 0 || end > num_refs || begin > end) {
                    hp_report(err, HP_DEV_BAD_INDEX, begin);
                    begin = end = 0;
                }
                for (int tri = begin; tri < end; ++tri) {
                    if (STATS) ++r.tris;
                    // The first two Woop rows at once (the second is needed whenever the
                    // plane is hit in range): one round trip fewer per tested triangle;
                    // the third when u >= 0.
                    const float4 v0 = __ldg(woop + 3 * (int64_t)tri);
                    const float4 v1 = __ldg(woop + 3 * (int64_t)tri + 1);
                    const float oz = __fmaf_rn(-r.oz, v0.z, __fmaf_rn(-r.oy, v0.y, __fmaf_rn(-r.ox, v0.x, v0.w)));
                    // The roundings of the reference's fast-math tracer, measured
                    // against its output on sm_100a: the chains o.w +- ... are
                    // contracted term by term from the left; of the three-term dot
                    // products d.w, the denominator and the v term fuse the x
                    // product over the rounded y product, the u term the y product
                    // over the rounded x product (nvcc's choice depends on context).
                    const float den = __fmaf_rn(r.dz, v0.z, __fmaf_rn(r.dx, v0.x, __fmul_rn(r.dy, v0.y)));
                    const float t = __fmul_rn(oz, HP_TRACE_RCP(den));
                    bool closer = t < r.hit_t;
                    if (!closer && t == r.hit_t && r.hit >= 0)
                        closer = __ldg(tri_idx + tri) < __ldg(tri_idx + r.hit);
                    if (t > r.tmin && closer) {
                        const float ox = __fmaf_rn(r.oz, v1.z, __fmaf_rn(r.oy, v1.y, __fmaf_rn(r.ox, v1.x, v1.w)));
                        const float dx = __fmaf_rn(r.dz, v1.z, __fmaf_rn(r.dy, v1.y, __fmul_rn(r.dx, v1.x)));
                        const float u = __fmaf_rn(t, dx, ox);
                        if (u >= 0.0f) {
                            const float4 v2 = __ldg(woop + 3 * (int64_t)tri + 2);
                            const float oy = __fmaf_rn(r.oz, v2.z, __fmaf_rn(r.oy, v2.y, __fmaf_rn(r.ox, v2.x, v2.w)));
                            const float dy = __fmaf_rn(r.dz, v2.z, __fmaf_rn(r.dx, v2.x, __fmul_rn(r.dy, v2.y)));
                            const float v = __fmaf_rn(t, dy, oy);
                            if (v >= 0.0f && __fadd_rn(u, v) <= 1.0f) {
                                r.hit_t = t;
                                r.hit = tri;
                                r.hit_u = u;
                                r.hit_v = v;
                                if (ANY_HIT) { sp = 0; break; }
                            }
                        }
                    }
                }
                if (ANY_HIT && r.hit >= 0) { node = SENTINEL; leaf = 0; break; }
                leaf = node;
                if (node < 0) {
                    if (sp == 0) node = SENTINEL;
                    else { --sp; node = sp < SSTACK ? sstack[sp * TRACE_BLOCK] : lstack[sp - SSTACK]; }
                }
            }
            if (node == SENTINEL) {
                if (r.hit < 0) {
                    reinterpret_cast<int2*>(results)[2 * ray] = make_int2(-1, __float_as_int(r.hit_t));
                    if (STATS) stats[ray] = make_int2(0, 0);
                } else {
                    results[ray] = make_int4(__ldg(tri_idx + r.hit), __float_as_int(r.hit_t),
                                             __float_as_int(r.hit_u), __float_as_int(r.hit_v));
                    if (STATS) stats[ray] = make_int2(r.nodes, r.tris);
                }
            }
          }
          __syncwarp();
          if (__popc(__ballot_sync(HP_FULL_MASK, node != SENTINEL)) < FETCH_THRESHOLD) break;
        }
    }
}

// Persistent grid: the tuned CTAs per SM, or as many as fit.
int trace_grid(const hp_ctx* ctx, int per_sm, int64_t num_rays) {
    int k = std::max(per_sm, 1);
    if (ctx->tune.trace_ctas_per_sm > 0) k = std::min(k, (int)ctx->tune.trace_ctas_per_sm);
    const int64_t grid = std::min<int64_t>((int64_t)ctx->sm_count * k, (num_rays + TRACE_BLOCK - 1) / TRACE_BLOCK);
    return (int)std::max<int64_t>(grid, 1);
}

template <bool A, bool S, int SST>
hp_status launch_t(hp_ctx* ctx, const hp_bvh_impl* b, int64_t n_refs, const float* rays,
                   int64_t num_rays, int32_t* results, int32_t* stats, unsigned long long* counter,
                   const int32_t* order, cudaStream_t s) {
    int per_sm = 0;
    HP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace<A, S, false, SST>, TRACE_BLOCK, 0));
    const int max_nodes = (int)std::max<int64_t>(2 * b->capacity - 1, 3);
    k_trace<A, S, false, SST><<<trace_grid(ctx, per_sm, num_rays), TRACE_BLOCK, 0, s>>>(
        reinterpret_cast<const float4*>(rays), num_rays, reinterpret_cast<int4*>(results),
        reinterpret_cast<int2*>(stats), reinterpret_cast<const float4*>(b->nodes), b->woop, b->tri_idx,
        max_nodes, (int)n_refs, counter, ctx->d_status, nullptr, nullptr, 0, order);
    HP_CUDA(cudaGetLastError());
    hp_count_launch();
    hp_mark(ctx, s, "trace");
    return HP_OK;
}

template <bool A, bool S>
hp_status launch_st(hp_ctx* ctx, const hp_bvh_impl* b, int64_t n_refs, const float* rays,
                    int64_t num_rays, int32_t* results, int32_t* stats, unsigned long long* counter,
                    const int32_t* order, cudaStream_t s) {
    switch (ctx->tune.trace_stack) {
        case 8: return launch_t<A, S, 8>(ctx, b, n_refs, rays, num_rays, results, stats, counter, order, s);
        case 32: return launch_t<A, S, 32>(ctx, b, n_refs, rays, num_rays, results, stats, counter, order, s);
        default: return launch_t<A, S, 16>(ctx, b, n_refs, rays, num_rays, results, stats, counter, order, s);
    }
}

