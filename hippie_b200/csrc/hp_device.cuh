// Device-side helpers shared by the build, trace and adjoint kernels.
//
// Floating-point policy: every translation unit is compiled with
// -fmad=false, so the compiler never contracts a*b+c on its own. Wherever the
// reference's fast-math build contracts (rt/bvh/*Kernels.cu, compiled with
// -use_fast_math by src/hippie/gpu/HipCompiler.cpp:109-161) the contraction is
// written out with __fmaf_rn, and the CPU oracle writes the same fmaf calls.
// That makes GPU and oracle results bit-identical.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define HP_WARP 32
#define HP_FULL_MASK 0xffffffffu
#define HP_MAX_FLOAT 3.402823466e+38f

// Error words written by kernels into the context's status buffer.
enum hp_dev_error {
    HP_DEV_OK = 0,
    HP_DEV_SPIN_LIMIT = 1,      // a bounded wait (look-back, barrier) gave up
    HP_DEV_BAD_INDEX = 2,       // an index read from memory was out of range
    HP_DEV_STACK_OVERFLOW = 3,  // traversal stack exceeded its capacity
    HP_DEV_BAD_INPUT = 4,       // e.g. a triangle references a vertex out of range
    HP_DEV_CHECK_FAILED = 5     // checked mode: an output failed its verification
};

// Upper bound on iterations of any spin-wait in this library.
#define HP_SPIN_LIMIT (1u << 24)

__device__ __forceinline__ void hp_report(int* status, int code, int info) {
    if (status) {
        if (atomicCAS(status, 0, code) == 0) status[1] = info;
    }
}

// Arrival at a node in a bottom-up climb: returns the count before this
// arrival. The add is acq_rel at GPU scope, so the second thread to arrive sees
// every write the first one made before its arrival.
__device__ __forceinline__ int hp_arrive(int* counter) {
    int old;
    asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], 1;" : "=r"(old) : "l"(counter) : "memory");
    return old;
}

// Bounded grid barrier for cooperative launches: bar[0] counts arrivals,
// bar[1] is the generation (both zero before the launch). Every thread of every
// CTA calls it. Returns false, with HP_DEV_SPIN_LIMIT reported, when the wait
// gave up: after `limit` polls, or early once another CTA has reported an
// error; the caller then leaves the kernel.
__device__ __forceinline__ bool hp_grid_barrier(unsigned* bar, int* err, unsigned limit) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        s_ok = 1;
        const unsigned gen = *((volatile unsigned*)(bar + 1));
        __threadfence();
        if (atomicAdd(bar, 1u) == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            unsigned spins = 0;
            while (*((volatile unsigned*)(bar + 1)) == gen) {
                if (++spins > limit || ((spins & 255u) == 0 && *((volatile int*)err) != 0)) {
                    hp_report(err, HP_DEV_SPIN_LIMIT, -1);
                    s_ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return s_ok != 0;
}

// ---- float <-> order-preserving uint (for atomicMin/atomicMax on floats) ----
__device__ __forceinline__ uint32_t hp_f2ord(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float hp_ord2f(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// ---- Morton codes (rt/HipUtil.h:35-106) ------------------------------------
// 10-bit spread into every third bit; x in the least significant position.
__device__ __forceinline__ uint32_t hp_spread10(uint32_t x) {
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}
__device__ __forceinline__ uint32_t hp_morton30(uint32_t x, uint32_t y, uint32_t z) {
    return hp_spread10(x) | (hp_spread10(y) << 1) | (hp_spread10(z) << 2);
}
// 60-bit code of 20-bit coordinates: high 10 bits of each axis form the upper
// 30 key bits, low 10 bits the lower 30 (rt/HipUtil.h:72-82).
__device__ __forceinline__ uint64_t hp_morton60(uint32_t x, uint32_t y, uint32_t z) {
    uint64_t lo = hp_morton30(x & 1023u, y & 1023u, z & 1023u);
    uint64_t hi = hp_morton30(x >> 10, y >> 10, z >> 10);
    return (hi << 30) | lo;
}

// Quantise a box centroid the way computeMortonCodes60 does
// (rt/bvh/LBVHBuilderKernels.cu:131-160, rt/HipUtil.h:92-98):
// c = (mn + mx) * 0.5; q = (uint)(((c - sceneMin) * scale) * 1048575.0f).
// The float->uint conversion truncates toward zero and saturates (cvt.rzi.u32.f32).
__device__ __forceinline__ uint64_t hp_morton_key(float mnx, float mny, float mnz,
                                                  float mxx, float mxy, float mxz,
                                                  const float* smin, const float* scale,
                                                  int bits) {
    const float q20 = 1048575.0f;
    float cx = __fmul_rn(__fadd_rn(mnx, mxx), 0.5f);
    float cy = __fmul_rn(__fadd_rn(mny, mxy), 0.5f);
    float cz = __fmul_rn(__fadd_rn(mnz, mxz), 0.5f);
    uint32_t x = __float2uint_rz(__fmul_rn(__fmul_rn(__fsub_rn(cx, smin[0]), scale[0]), q20));
    uint32_t y = __float2uint_rz(__fmul_rn(__fmul_rn(__fsub_rn(cy, smin[1]), scale[1]), q20));
    uint32_t z = __float2uint_rz(__fmul_rn(__fmul_rn(__fsub_rn(cz, smin[2]), scale[2]), q20));
    return hp_morton60(x, y, z) >> (60 - bits);
}

// ---- triangle vertices (indexed mesh, 3 vertex indices per triangle) --------
__device__ __forceinline__ void load_vertex(const float* __restrict__ v, int64_t nv, int idx,
                                            float& x, float& y, float& z, int* err) {
    if (idx < 0 || idx >= nv) {
        hp_report(err, HP_DEV_BAD_INPUT, idx);
        idx = 0;
    }
    x = __ldg(v + 3 * (int64_t)idx + 0);
    y = __ldg(v + 3 * (int64_t)idx + 1);
    z = __ldg(v + 3 * (int64_t)idx + 2);
}

struct tri_verts {
    float x0, y0, z0, x1, y1, z1, x2, y2, z2;
};

__device__ __forceinline__ tri_verts load_tri(const float* __restrict__ v, int64_t nv,
                                              const int32_t* __restrict__ t, int64_t tri, int* err) {
    tri_verts r;
    int a = __ldg(t + 3 * tri + 0), b = __ldg(t + 3 * tri + 1), c = __ldg(t + 3 * tri + 2);
    load_vertex(v, nv, a, r.x0, r.y0, r.z0, err);
    load_vertex(v, nv, b, r.x1, r.y1, r.z1, err);
    load_vertex(v, nv, c, r.x2, r.y2, r.z2, err);
    return r;
}

// ---- surface area with the reference's contraction ------------------------
// AABB::area (util/AABB.h:33): 2 * (d.x*d.y + d.y*d.z + d.z*d.x) under fast-math
// FMA contraction = 2 * fma(dz, dx, fma(dx, dy, dy*dz)).
__device__ __forceinline__ float hp_area(float mnx, float mny, float mnz,
                                         float mxx, float mxy, float mxz) {
    float dx = __fsub_rn(mxx, mnx), dy = __fsub_rn(mxy, mny), dz = __fsub_rn(mxz, mnz);
    if (!(mnx <= mxx && mny <= mxy && mnz <= mxz)) return 0.0f;
    float s = __fmaf_rn(dz, dx, __fmaf_rn(dx, dy, __fmul_rn(dy, dz)));
    return __fmul_rn(2.0f, s);
}

// ---- 64-byte binary node (rt/bvh/HipBVHNode.h:116-218) -----------------------
struct __align__(16) hp_node_bin {
    float4 c0xy;   // c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y
    float4 c1xy;   // c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y
    float4 cz;     // c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z
    int4 meta;     // child0 / begin, child1 / end, size (~size for a leaf), parent
};
static_assert(sizeof(hp_node_bin) == 64, "binary node must be 64 bytes");

__device__ __forceinline__ hp_node_bin hp_make_node(float4 amn, float4 amx, float4 bmn, float4 bmx,
                                                    int c0, int c1, int size, int parent) {
    hp_node_bin n;
    n.c0xy = make_float4(amn.x, amx.x, amn.y, amx.y);
    n.c1xy = make_float4(bmn.x, bmx.x, bmn.y, bmx.y);
    n.cz = make_float4(amn.z, amx.z, bmn.z, bmx.z);
    n.meta = make_int4(c0, c1, size, parent);
    return n;
}

// ---- Woop transform (rt/bvh/HipBVHKernels.cu:12-65, util/Math.h:318-367) -----
// The matrix M has columns (v0-v2, 0), (v1-v2, 0), ((v0-v2)x(v1-v2), 0), (v2, 1);
// its inverse is taken by cofactors exactly as Math.h's inverse(): the 3x3
// minors, d accumulated over all L*L cofactor products (= 4 det), then
// r * (1/d) * 4. Every product-sum is written with the contraction the
// fast-math build applies.
struct hp_mat4 { float m[16]; };  // column-major: m[r + 4*c]

__device__ __forceinline__ float hp_det3(const float* a /* 3x3 column-major */) {
    // detImpl<3> (Math.h:326-330): the six products summed left to right,
    //   a00 a11 a22 - a00 a12 a21 + a10 a21 a02 - a10 a22 a01 + a20 a01 a12 - a20 a02 a11,
    // contracted as nvcc contracts that expression under fast math (measured on
    // sm_100a): the first difference fuses the first product over the rounded
    // second, each later product is folded into the running sum with one fma.
#define A(r, c) a[(r) + 3 * (c)]
    float acc = __fmaf_rn(__fmul_rn(A(0, 0), A(1, 1)), A(2, 2), -__fmul_rn(__fmul_rn(A(0, 0), A(1, 2)), A(2, 1)));
    acc = __fmaf_rn(__fmul_rn(A(1, 0), A(2, 1)), A(0, 2), acc);
    acc = __fmaf_rn(-__fmul_rn(A(1, 0), A(2, 2)), A(0, 1), acc);
    acc = __fmaf_rn(__fmul_rn(A(2, 0), A(0, 1)), A(1, 2), acc);
    acc = __fmaf_rn(-__fmul_rn(A(2, 0), A(0, 2)), A(1, 1), acc);
#undef A
    return acc;
}

__device__ __forceinline__ void hp_woop(float v0x, float v0y, float v0z,
                                        float v1x, float v1y, float v1z,
                                        float v2x, float v2y, float v2z,
                                        float4& w0, float4& w1, float4& w2) {
    float ax = __fsub_rn(v0x, v2x), ay = __fsub_rn(v0y, v2y), az = __fsub_rn(v0z, v2z);
    float bx = __fsub_rn(v1x, v2x), by = __fsub_rn(v1y, v2y), bz = __fsub_rn(v1z, v2z);
    // cross(u, v) = (u.y*v.z - u.z*v.y, u.z*v.x - u.x*v.z, u.x*v.y - u.y*v.x)
    float nx = __fmaf_rn(ay, bz, -__fmul_rn(az, by));
    float ny = __fmaf_rn(az, bx, -__fmul_rn(ax, bz));
    float nz = __fmaf_rn(ax, by, -__fmul_rn(ay, bx));
    float M[16] = {ax, ay, az, 0.0f, bx, by, bz, 0.0f, nx, ny, nz, 0.0f, v2x, v2y, v2z, 1.0f};
    float R[16];
    float d = 0.0f;
    float si = 1.0f;
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
            float dd = __fmul_rn(hp_det3(sub), sj);
            R[i + 4 * j] = dd;
            d = __fmaf_rn(dd, M[j + 4 * i], d);
            sj = -sj;
        }
        si = -si;
    }
    float rd = (d != 0.0f) ? __frcp_rn(d) : 0.0f;  // rcp() (Math.h:20): 0 for a singular matrix
#pragma unroll
    for (int k = 0; k < 16; ++k) R[k] = __fmul_rn(__fmul_rn(R[k], rd), 4.0f);
    // im[c][r] in the reference is column c, row r: R[r + 4c].
#define IM(c, r) R[(r) + 4 * (c)]
    w0 = make_float4(IM(0, 2), IM(1, 2), IM(2, 2), -IM(3, 2));
    w1 = make_float4(IM(0, 0), IM(1, 0), IM(2, 0), IM(3, 0));
    w2 = make_float4(IM(0, 1), IM(1, 1), IM(2, 1), IM(3, 1));
#undef IM
}
