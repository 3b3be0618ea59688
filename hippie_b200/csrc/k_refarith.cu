// Reference arithmetic: the reciprocals of the reference's fast-math build.
//
// This translation unit is compiled with -use_fast_math (hippie_b200/build.py),
// the flag the reference compiles its kernels with (gpu/HipCompiler.cpp:127-129):
// `1.0f / x` lowers to the same approximate quotient, every float operation
// flushes denormals, and the compiler contracts multiply-add pairs. Two
// pieces use it:
//   * k_woop_ref: the Woop rows of every reference, HipBVH::woopifyTriangles
//     (rt/bvh/HipBVH.cpp:95-116, rt/bvh/HipBVHKernels.cu:12-65). Which
//     products the compiler fuses depends on the shape of each expression, so
//     woop_fast() writes the cross product, the 3x3 minors and the cofactor
//     inverse with the reference's expression trees (util/Math.h:178, 326-330,
//     350-368) and leaves the contraction to the compiler, as in the
//     reference's build; rcp(d) is 1/d, 0 for a singular matrix (Math.h:20);
//   * the binary tracer (k_trace_impl.cuh) with idir = 1/d and the triangle
//     test's 1/(d.n) as in rt/tracer/HipTracerBinKernels.cu:87-89,219-220.
//     Its other arithmetic is written with __fmaf_rn / __fmul_rn / __fadd_rn,
//     which the compiler never contracts further, so only the reciprocals and
//     denormal flushing change.
#include <algorithm>
#include <cuda_runtime.h>
#include "hp_device.cuh"
#include "hp_internal.h"

namespace {

#define HP_TRACE_RCP(x) (1.0f / (x))
#include "k_trace_impl.cuh"

// Determinant of a 3x3 minor a(r, c) = a[r + 3c], as detImpl<3>: six triple
// products summed left to right.
__device__ __forceinline__ float det3_fast(const float* a) {
#define A(r, c) a[(r) + 3 * (c)]
    return A(0, 0) * A(1, 1) * A(2, 2) - A(0, 0) * A(1, 2) * A(2, 1) +
           A(1, 0) * A(2, 1) * A(0, 2) - A(1, 0) * A(2, 2) * A(0, 1) +
           A(2, 0) * A(0, 1) * A(1, 2) - A(2, 0) * A(0, 2) * A(1, 1);
#undef A
}

// Woop rows of one triangle: M has columns (v0-v2, 0), (v1-v2, 0),
// ((v0-v2) x (v1-v2), 0), (v2, 1); its inverse by cofactors, r * rcp(d) * 4
// with d the sum of all 16 cofactor products (4 det M).
__device__ __forceinline__ void woop_fast(const tri_verts& t, float4& w0, float4& w1, float4& w2) {
    const float ax = t.x0 - t.x2, ay = t.y0 - t.y2, az = t.z0 - t.z2;
    const float bx = t.x1 - t.x2, by = t.y1 - t.y2, bz = t.z1 - t.z2;
    const float nx = ay * bz - az * by, ny = az * bx - ax * bz, nz = ax * by - ay * bx;
    const float M[16] = {ax, ay, az, 0.0f, bx, by, bz, 0.0f, nx, ny, nz, 0.0f, t.x2, t.y2, t.z2, 1.0f};
    float R[16];
    float d = 0.0f, si = 1.0f;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        float sj = si;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float sub[9];
#pragma unroll
            for (int k = 0; k < 3; ++k)
#pragma unroll
                for (int l = 0; l < 3; ++l)
                    sub[k + 3 * l] = M[((k < j) ? k : k + 1) + 4 * ((l < i) ? l : l + 1)];
            const float dd = det3_fast(sub) * sj;
            R[i + 4 * j] = dd;
            d += dd * M[j + 4 * i];
            sj = -sj;
        }
        si = -si;
    }
    const float rd = d ? 1.0f / d : 0.0f;
#pragma unroll
    for (int k = 0; k < 16; ++k) R[k] = R[k] * rd * 4.0f;
    w0 = make_float4(R[2], R[6], R[10], -R[14]);
    w1 = make_float4(R[0], R[4], R[8], R[12]);
    w2 = make_float4(R[1], R[5], R[9], R[13]);
}

constexpr int WB = 256;

// Woop rows of leaf-ordered reference k from scene triangle tri_idx[k].
__global__ void __launch_bounds__(WB) k_woop_ref(const float* __restrict__ verts, int64_t nv,
                                                 const int32_t* __restrict__ tris, int64_t num_tris,
                                                 const int32_t* __restrict__ tri_idx, int64_t n,
                                                 float4* __restrict__ woop, int* err) {
    const int64_t k = blockIdx.x * (int64_t)WB + threadIdx.x;
    if (k >= n) return;
    int tri = __ldg(tri_idx + k);
    if (tri < 0 || tri >= num_tris) {
        hp_report(err, HP_DEV_BAD_INDEX, tri);
        return;
    }
    const tri_verts v = load_tri(verts, nv, tris, tri, err);
    float4 w0, w1, w2;
    woop_fast(v, w0, w1, w2);
    woop[3 * k + 0] = w0;
    woop[3 * k + 1] = w1;
    woop[3 * k + 2] = w2;
}

}  // namespace

hp_status hp_woop_ref_launch(hp_ctx* ctx, hp_bvh_impl* b, int64_t n_refs, const hp_mesh* m, cudaStream_t s) {
    if (n_refs <= 0) return HP_OK;
    k_woop_ref<<<(unsigned)hp_div_up(n_refs, WB), WB, 0, s>>>(m->vertices, m->num_vertices, m->triangles,
                                                             m->num_triangles, b->tri_idx, n_refs, b->woop,
                                                             ctx->d_status);
    HP_CUDA(cudaGetLastError());
    hp_count_launch();
    hp_mark(ctx, s, "woop_ref");
    return HP_OK;
}

hp_status hp_trace_ref_launch(hp_ctx* ctx, const hp_bvh_impl* b, int64_t n_refs, const float* rays,
                              int64_t num_rays, int32_t* results, int32_t* stats, uint32_t flags,
                              unsigned long long* counter, const int32_t* order, cudaStream_t s) {
    const bool any = flags & HP_TRACE_ANY_HIT, st = (flags & HP_TRACE_STATS) && stats;
    if (any && st) return launch_st<true, true>(ctx, b, n_refs, rays, num_rays, results, stats, counter, order, s);
    if (any) return launch_st<true, false>(ctx, b, n_refs, rays, num_rays, results, stats, counter, order, s);
    if (st) return launch_st<false, true>(ctx, b, n_refs, rays, num_rays, results, stats, counter, order, s);
    return launch_st<false, false>(ctx, b, n_refs, rays, num_rays, results, stats, counter, order, s);
}
