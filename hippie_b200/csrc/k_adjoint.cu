// Closest-hit adjoint and refit-only BVH update.
//
// Adjoint: a hit satisfies O + t D = u v0 + v v1 + (1-u-v) v2 (u weights v0 and
// v weights v1, the barycentric convention of rt/HipUtil.h:190-195), i.e.
// A x = O - v2 with A = [v0-v2, v1-v2, -D] and x = (u, v, t). Differentiating,
// dx/dv0 = -u A^-1, dx/dv1 = -v A^-1, dx/dv2 = -(1-u-v) A^-1, so with
// q = A^-T (dL/du, dL/dv, dL/dt):
//   dL/dv0 = -u q,  dL/dv1 = -v q,  dL/dv2 = -(1-u-v) q,
// and A^-T g = (g_u (b x c) + g_v (c x a) + g_t (a x b)) / det(A) for A = [a b c].
// Lanes of a warp whose rays touch the same vertex add their contributions
// with shuffles first, so each distinct vertex costs one set of atomics per warp.
//
// Refit: HipBVH::update (rt/bvh/HipBVH.cpp:472-477) = woopifyTriangles +
// refitLeavesBin + refitInteriorsBin (rt/bvh/HipBVHKernels.cu:240-326). The
// reference launches refitLeaves with 4 of its 6 arguments (HipBVH.cpp:43-48);
// this version passes the mesh, so leaf boxes come from the current vertices.
#include <cuda_runtime.h>
#include "hp_device.cuh"
#include "hp_internal.h"

namespace {

constexpr int AB = 256;

__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return make_float3(__fmaf_rn(a.y, b.z, -__fmul_rn(a.z, b.y)), __fmaf_rn(a.z, b.x, -__fmul_rn(a.x, b.z)),
                       __fmaf_rn(a.x, b.y, -__fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float dot3(float3 a, float3 b) {
    return __fmaf_rn(a.z, b.z, __fmaf_rn(a.y, b.y, __fmul_rn(a.x, b.x)));
}
// g0 * x + g1 * y + g2 * z
__device__ __forceinline__ float comb3(float g0, float x, float g1, float y, float g2, float z) {
    return __fmaf_rn(g2, z, __fmaf_rn(g1, y, __fmul_rn(g0, x)));
}

// Sum `val` over the lanes in `peers` (all of which call this with the same mask).
__device__ __forceinline__ float group_sum(unsigned peers, float val) {
    float s = 0.0f;
    unsigned m = peers;
    while (m) {
        const int j = __ffs(m) - 1;
        s += __shfl_sync(peers, val, j);
        m &= m - 1;
    }
    return s;
}

__global__ void __launch_bounds__(AB) k_adjoint(const float* __restrict__ verts, int64_t nv,
                                                const int32_t* __restrict__ tris, int64_t ntri,
                                                const float4* __restrict__ rays,
                                                const int4* __restrict__ results,
                                                const float* __restrict__ dl, int64_t num_rays,
                                                float* __restrict__ dverts, int* err) {
    const int64_t i = blockIdx.x * (int64_t)AB + threadIdx.x;
    const int lane = threadIdx.x & 31;
    int vid[3] = {-1, -1, -1};
    float gx[3] = {0, 0, 0}, gy[3] = {0, 0, 0}, gz[3] = {0, 0, 0};
    if (i < num_rays) {
        const int4 res = results[i];
        const int tri = res.x;
        if (tri >= 0 && tri < ntri) {
            const float u = __int_as_float(res.z), v = __int_as_float(res.w);
            const float gu = dl[3 * i + 1], gv = dl[3 * i + 2], gt = dl[3 * i + 0];
            const float4 d4 = rays[2 * i + 1];
            int idx[3];
            float3 p[3];
            bool ok = true;
            for (int k = 0; k < 3; ++k) {
                idx[k] = tris[3 * (int64_t)tri + k];
                if (idx[k] < 0 || idx[k] >= nv) { ok = false; idx[k] = 0; }
                p[k] = make_float3(verts[3 * (int64_t)idx[k]], verts[3 * (int64_t)idx[k] + 1],
                                   verts[3 * (int64_t)idx[k] + 2]);
            }
            if (!ok) hp_report(err, HP_DEV_BAD_INPUT, tri);
            const float3 a = make_float3(p[0].x - p[2].x, p[0].y - p[2].y, p[0].z - p[2].z);
            const float3 b = make_float3(p[1].x - p[2].x, p[1].y - p[2].y, p[1].z - p[2].z);
            const float3 c = make_float3(-d4.x, -d4.y, -d4.z);
            const float3 bc = cross3(b, c), ca = cross3(c, a), ab = cross3(a, b);
            const float det = dot3(a, bc);
            if (ok && det != 0.0f) {
                const float qx = __fdiv_rn(comb3(gu, bc.x, gv, ca.x, gt, ab.x), det);
                const float qy = __fdiv_rn(comb3(gu, bc.y, gv, ca.y, gt, ab.y), det);
                const float qz = __fdiv_rn(comb3(gu, bc.z, gv, ca.z, gt, ab.z), det);
                const float w[3] = {u, v, __fsub_rn(__fsub_rn(1.0f, u), v)};
                for (int k = 0; k < 3; ++k) {
                    vid[k] = idx[k];
                    gx[k] = -__fmul_rn(w[k], qx);
                    gy[k] = -__fmul_rn(w[k], qy);
                    gz[k] = -__fmul_rn(w[k], qz);
                }
            }
        }
    }
    // Warp-aggregated scatter, one round per triangle corner.
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const unsigned peers = __match_any_sync(HP_FULL_MASK, vid[k]);
        const float sx = group_sum(peers, gx[k]);
        const float sy = group_sum(peers, gy[k]);
        const float sz = group_sum(peers, gz[k]);
        if (vid[k] >= 0 && lane == __ffs(peers) - 1) {
            atomicAdd(dverts + 3 * (int64_t)vid[k] + 0, sx);
            atomicAdd(dverts + 3 * (int64_t)vid[k] + 1, sy);
            atomicAdd(dverts + 3 * (int64_t)vid[k] + 2, sz);
        }
    }
}

// One thread per leaf node: re-woopify its triangles, store its box, then
// climb through parent links; the second child to arrive at a node finishes it.
__global__ void __launch_bounds__(AB) k_refit(const float* __restrict__ verts, int64_t nv,
                                              const int32_t* __restrict__ tris,
                                              const int32_t* __restrict__ tri_idx,
                                              hp_node_bin* nodes, float4* __restrict__ woop,
                                              int* counters, const hp_bvh_info* info, int n_refs,
                                              int* err) {
    const int num_int = info->num_interior, num_leaf = info->num_leaf;
    const int li = blockIdx.x * AB + threadIdx.x;
    if (li >= num_leaf) return;
    const int leaf = num_int + li;
    const int4 meta = nodes[leaf].meta;
    if (meta.x < 0 || meta.y > n_refs || meta.x > meta.y) {
        hp_report(err, HP_DEV_BAD_INDEX, leaf);
        return;
    }
    float mn[3] = {HP_MAX_FLOAT, HP_MAX_FLOAT, HP_MAX_FLOAT};
    float mx[3] = {-HP_MAX_FLOAT, -HP_MAX_FLOAT, -HP_MAX_FLOAT};
    for (int r = meta.x; r < meta.y; ++r) {
        const int tri = tri_idx[r];
        float p[9];
        for (int k = 0; k < 3; ++k) {
            int vi = tris[3 * (int64_t)tri + k];
            if (vi < 0 || vi >= nv) { hp_report(err, HP_DEV_BAD_INPUT, tri); vi = 0; }
            for (int c = 0; c < 3; ++c) {
                p[3 * k + c] = verts[3 * (int64_t)vi + c];
                mn[c] = fminf(mn[c], p[3 * k + c]);
                mx[c] = fmaxf(mx[c], p[3 * k + c]);
            }
        }
        float4 w0, w1, w2;
        hp_woop(p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], p[8], w0, w1, w2);
        woop[3 * (int64_t)r] = w0;
        woop[3 * (int64_t)r + 1] = w1;
        woop[3 * (int64_t)r + 2] = w2;
    }
    if (meta.x >= meta.y) return;  // empty leaf (single-triangle BVH): keeps its inverted box
    float4 bmn = make_float4(mn[0], mn[1], mn[2], 0.0f), bmx = make_float4(mx[0], mx[1], mx[2], 0.0f);
    nodes[leaf].c0xy = make_float4(bmn.x, bmx.x, bmn.y, bmx.y);
    nodes[leaf].c1xy = make_float4(bmn.x, bmx.x, bmn.y, bmx.y);
    nodes[leaf].cz = make_float4(bmn.z, bmx.z, bmn.z, bmx.z);
    int child = leaf;
    int node = meta.w;
    int guard = 0;
    while (node >= 0) {
        if (node >= num_int || ++guard > num_int) {
            hp_report(err, HP_DEV_BAD_INDEX, node);
            return;
        }
        hp_node_bin* pn = nodes + node;
        const int4 pm = __ldcg(&pn->meta);
        const int c0 = pm.x < 0 ? ~pm.x : pm.x;
        if (c0 == child) {
            __stcg(&pn->c0xy, make_float4(bmn.x, bmx.x, bmn.y, bmx.y));
            __stcg(reinterpret_cast<float2*>(&pn->cz), make_float2(bmn.z, bmx.z));
        } else {
            __stcg(&pn->c1xy, make_float4(bmn.x, bmx.x, bmn.y, bmx.y));
            __stcg(reinterpret_cast<float2*>(&pn->cz) + 1, make_float2(bmn.z, bmx.z));
        }
        __threadfence();
        if (atomicAdd(&counters[node], 1) == 0) return;
        __threadfence();
        const float4 a = __ldcg(&pn->c0xy), b = __ldcg(&pn->c1xy), z = __ldcg(&pn->cz);
        bmn = make_float4(fminf(a.x, b.x), fminf(a.z, b.z), fminf(z.x, z.z), 0.0f);
        bmx = make_float4(fmaxf(a.y, b.y), fmaxf(a.w, b.w), fmaxf(z.y, z.w), 0.0f);
        child = node;
        node = pm.w;
    }
}

}  // namespace

hp_status hp_adjoint_launch(hp_ctx* ctx, const hp_mesh* m, const float* rays, const int32_t* results,
                            const float* dl_dtuv, int64_t num_rays, float* dl_dvertices,
                            cudaStream_t s) {
    if (num_rays <= 0) return HP_OK;
    k_adjoint<<<hp_div_up(num_rays, AB), AB, 0, s>>>(
        m->vertices, m->num_vertices, m->triangles, m->num_triangles,
        reinterpret_cast<const float4*>(rays), reinterpret_cast<const int4*>(results), dl_dtuv,
        num_rays, dl_dvertices, ctx->d_status);
    HP_CUDA(cudaGetLastError());
    hp_count_launch();
    hp_mark(ctx, s, "adjoint");
    return HP_OK;
}

hp_status hp_refit_launch(hp_ctx* ctx, hp_bvh_impl* b, int64_t n_refs, const hp_mesh* m,
                          cudaStream_t s) {
    if (n_refs <= 0) return HP_OK;
    HP_CUDA(cudaMemsetAsync(b->counters, 0, sizeof(int) * std::max<int64_t>(n_refs, 2), s));
    const int64_t max_leaves = std::max<int64_t>(n_refs, 2);
    k_refit<<<hp_div_up(max_leaves, AB), AB, 0, s>>>(m->vertices, m->num_vertices, m->triangles,
                                                     b->tri_idx, b->nodes, b->woop, b->counters,
                                                     b->info, (int)n_refs, ctx->d_status);
    HP_CUDA(cudaGetLastError());
    hp_count_launch();
    hp_mark(ctx, s, "refit");
    return HP_OK;
}
