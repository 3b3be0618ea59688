// Ray generation and ray sorting.
//
// Primary rays: RayGen::primary (rt/ray/RayGen.cpp:35-62) and its kernel
// generatePrimaryRays (rt/ray/RayGenKernels.cu:106-153): one ray per pixel of a
// pinhole camera, jittered by the Halton point of the sample index (bases 2 and
// 3, RayGenKernels.cu:20-39), unprojected through inverse(projection * view),
// written in the order of the pixel table (PixelTable::recalculate,
// rt/ray/PixelTable.cpp:10-80: 8x8 pixel blocks in Morton order, pixels
// swizzled inside a block, then the stripes below and right of the blocks).
// Every step is IEEE-rounded (the reference's fast-math build approximates the
// divisions and the normalisation), so the CPU oracle reproduces the rays bit
// for bit.
//
// Ray sorting: RayBuffer::mortonSort (rt/ray/RayBuffer.cpp:31-131) with the
// default method computeMortonCodesAila64 (rt/ray/RayBufferKernels.cu:556-615):
// the origin normalised to the ray box (the reference fixes it to [0,1]^3) and
// the direction mapped to [0,1]^3, both quantised to 13 bits per axis and
// interleaved (origin bits 12..10 first, then origin and direction bits in
// alternating triples); the key keeps the top `bits` of the 64-bit code. The
// rays are then traced in key order (HipTracer::traceSort, rt/tracer/
// HipTracer.cpp:109-125): slot k of the traversal takes ray order[k], results
// stay at the rays' own indices.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <utility>
#include <vector>
#include <cuda_runtime.h>
#include "hp_device.cuh"
#include "hp_internal.h"

namespace {

struct cam_args {
    float ox, oy, oz;
    float m[16];  // screen -> world, row-major: world4 = M * (x, y, 0, 1)
    int width, height;
    float hx, hy;  // Halton jitter of the sample
    float max_dist;
};

__global__ void __launch_bounds__(256) k_primary_rays(cam_args c, const int32_t* __restrict__ index_to_pixel,
                                                      float4* __restrict__ rays, int64_t n, int* err) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t pixel = index_to_pixel ? (int64_t)index_to_pixel[i] : i;
    if (pixel < 0 || pixel >= n) {
        hp_report(err, HP_DEV_BAD_INDEX, (int)i);
        pixel = 0;
    }
    const float x = __fadd_rn((float)(pixel % c.width), c.hx);
    const float y = __fadd_rn((float)(pixel / c.width), c.hy);
    const float nx = __fsub_rn(__fdiv_rn(__fmul_rn(2.0f, x), (float)c.width), 1.0f);
    const float ny = __fsub_rn(__fdiv_rn(__fmul_rn(2.0f, y), (float)c.height), 1.0f);
    float w[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) w[r] = __fmaf_rn(c.m[4 * r + 0], nx, __fmaf_rn(c.m[4 * r + 1], ny, c.m[4 * r + 3]));
    const float px = __fdiv_rn(w[0], w[3]), py = __fdiv_rn(w[1], w[3]), pz = __fdiv_rn(w[2], w[3]);
    const float dx = __fsub_rn(px, c.ox), dy = __fsub_rn(py, c.oy), dz = __fsub_rn(pz, c.oz);
    const float len = __fsqrt_rn(__fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx))));
    rays[2 * i] = make_float4(c.ox, c.oy, c.oz, 0.0f);
    rays[2 * i + 1] = make_float4(__fdiv_rn(dx, len), __fdiv_rn(dy, len), __fdiv_rn(dz, len), c.max_dist);
}

struct key_args {
    float mn[3], mx[3], inv[3];  // ray box min, max and 1 / extent
    float ray_length;            // RayBuffer::rayLength (two-point keys)
    int bits;
};

// Float to int by truncation, saturating as the GPU conversion does (NaN: 0).
__device__ __forceinline__ int qz(float a, float scale) { return __float2int_rz(__fmul_rn(a, scale)); }

// Own atan2 and acos for the Costa and Reis keys (the reference calls the CUDA
// math library under fast math): octant reduction and atan(t) ~ t * P(t^2) on
// [0, 1], P of degree 8 fitted by iteratively reweighted least squares at
// Chebyshev nodes (max error 1e-7 rad in float); every step IEEE-rounded.
__device__ __forceinline__ float rk_atan01(float t) {
    const float s = __fmul_rn(t, t);
    float p = 0.0024567153304815292f;
    p = __fmaf_rn(p, s, -0.014401324093341827f);
    p = __fmaf_rn(p, s, 0.039781175553798676f);
    p = __fmaf_rn(p, s, -0.07234854251146317f);
    p = __fmaf_rn(p, s, 0.10498945415019989f);
    p = __fmaf_rn(p, s, -0.14161229133605957f);
    p = __fmaf_rn(p, s, 0.19985906779766083f);
    p = __fmaf_rn(p, s, -0.33332598209381104f);
    p = __fmaf_rn(p, s, 0.9999998807907104f);
    return __fmul_rn(t, p);
}
__device__ __forceinline__ float rk_atan2(float y, float x) {
    const float ax = fabsf(x), ay = fabsf(y);
    const float hi = fmaxf(ax, ay), lo = fminf(ax, ay);
    if (!(hi > 0.0f)) return 0.0f;
    float r = rk_atan01(__fdiv_rn(lo, hi));
    if (ay > ax) r = __fsub_rn(1.5707963705062866f, r);
    if (x < 0.0f) r = __fsub_rn(3.1415927410125732f, r);
    return y < 0.0f ? -r : r;
}
__device__ __forceinline__ float rk_acos(float z) {
    return rk_atan2(__fsqrt_rn(fmaxf(__fmaf_rn(-z, z, 1.0f), 0.0f)), z);
}

// Ray-box entry distance of the two-point keys (intersect, RayBufferKernels.cu:11-56).
__device__ __forceinline__ float rk_intersect(float4 o, float4 d, const key_args& k) {
    const float dd[3] = {d.x, d.y, d.z}, oo[3] = {o.x, o.y, o.z};
    float t0[3], t1[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float lo = dd[a] >= 0.0f ? k.mn[a] : k.mx[a], hi = dd[a] >= 0.0f ? k.mx[a] : k.mn[a];
        t0[a] = __fdiv_rn(__fsub_rn(lo, oo[a]), dd[a]);
        t1[a] = __fdiv_rn(__fsub_rn(hi, oo[a]), dd[a]);
    }
    const float tmin = fmaxf(t0[2], fmaxf(t0[0], t0[1]));
    const float tmax = fminf(t1[2], fminf(t1[0], t1[1]));
    if (tmin > tmax) return -1.0f;
    return __fmul_rn(1.0f - 1.0e-3f, tmin >= 0.0f ? tmin : tmax);
}

template <int M>
__device__ __forceinline__ uint64_t ray_code(float4 o, float4 d, const key_args& k) {
    const float a0 = __fmul_rn(__fsub_rn(o.x, k.mn[0]), k.inv[0]);
    const float a1 = __fmul_rn(__fsub_rn(o.y, k.mn[1]), k.inv[1]);
    const float a2 = __fmul_rn(__fsub_rn(o.z, k.mn[2]), k.inv[2]);
    uint64_t c = 0;
    if (M == HP_RAY_KEYS_TWO_POINT) {  // computeMortonCodesTwoPoint64 (RayBufferKernels.cu:492-554)
        float len = fminf(k.ray_length, fmaxf(d.w, 0.0f));
        len = fminf(len, rk_intersect(o, d, k));
        const float e0 = __fmaf_rn(len, d.x, o.x), e1 = __fmaf_rn(len, d.y, o.y), e2 = __fmaf_rn(len, d.z, o.z);
        const int ia[3] = {qz(a0, 8191.0f), qz(a1, 8191.0f), qz(a2, 8191.0f)};
        const int ib[3] = {qz(__fmul_rn(__fsub_rn(e0, k.mn[0]), k.inv[0]), 8191.0f),
                           qz(__fmul_rn(__fsub_rn(e1, k.mn[1]), k.inv[1]), 8191.0f),
                           qz(__fmul_rn(__fsub_rn(e2, k.mn[2]), k.inv[2]), 8191.0f)};
#pragma unroll
        for (int i = 12; i >= 2; --i)
            for (int a = 0; a < 3; ++a) c |= (uint64_t)((ia[a] >> i) & 1) << (6 * i - 9 - a);
#pragma unroll
        for (int i = 12; i >= 3; --i)
            for (int a = 0; a < 3; ++a) c |= (uint64_t)((ib[a] >> i) & 1) << (6 * i - 12 - a);
        c |= (uint64_t)(ib[0] & 1);
        return c;
    }
    if (M == HP_RAY_KEYS_ORIGIN) {  // computeMortonCodesOrigin64 (RayBufferKernels.cu:775-814)
        const int ia[3] = {qz(a0, 8388607.0f), qz(a1, 8388607.0f), qz(a2, 8388607.0f)};
#pragma unroll
        for (int i = 22; i >= 2; --i)
            for (int a = 0; a < 3; ++a) c |= (uint64_t)((ia[a] >> i) & 1) << (3 * i - 3 - a);
        c |= (uint64_t)(ia[0] & 1);
        return c;
    }
    const float len = __fsqrt_rn(__fmaf_rn(d.z, d.z, __fmaf_rn(d.y, d.y, __fmul_rn(d.x, d.x))));
    const float nx = __fdiv_rn(d.x, len), ny = __fdiv_rn(d.y, len), nz = __fdiv_rn(d.z, len);
    if (M == HP_RAY_KEYS_PARABOLOID || M == HP_RAY_KEYS_OCTAHEDRON) {
        // computeMortonCodesParaboloid64 / Octahedron64 (RayBufferKernels.cu:616-773)
        float bx, by;
        if (M == HP_RAY_KEYS_PARABOLOID) {
            if (nz < 0.0f) {
                const float dd = __fadd_rn(-nz, 1.0f);
                bx = __fadd_rn(__fdiv_rn(__fmul_rn(0.25f, nx), dd), 0.25f);
                by = __fadd_rn(__fdiv_rn(__fmul_rn(0.5f, ny), dd), 0.5f);
            } else {
                const float dd = __fadd_rn(nz, 1.0f);
                bx = __fadd_rn(__fdiv_rn(__fmul_rn(0.25f, nx), dd), 0.75f);
                by = __fadd_rn(__fdiv_rn(__fmul_rn(0.5f, ny), dd), 0.5f);
            }
        } else {
            const float ax = fabsf(nx), ay = fabsf(ny), az = fabsf(nz);
            const float fact = __fdiv_rn(1.0f, __fadd_rn(__fadd_rn(ax, ay), az));
            if (nz >= 0.0f) {
                bx = __fmul_rn(nx, fact);
                by = __fmul_rn(ny, fact);
            } else {
                bx = __fmul_rn(__fsub_rn(1.0f, __fmul_rn(ay, fact)), nx <= 0.0f ? -1.0f : 1.0f);
                by = __fmul_rn(__fsub_rn(1.0f, __fmul_rn(ax, fact)), ny <= 0.0f ? -1.0f : 1.0f);
            }
            bx = __fmul_rn(__fadd_rn(bx, 1.0f), 0.5f);
            by = __fmul_rn(__fadd_rn(by, 1.0f), 0.5f);
        }
        const int ia[3] = {qz(a0, 32767.0f), qz(a1, 32767.0f), qz(a2, 32767.0f)};
        const int ib[2] = {qz(bx, 32767.0f), qz(by, 32767.0f)};
#pragma unroll
        for (int i = 14; i >= 11; --i)
            for (int a = 0; a < 3; ++a) c |= (uint64_t)((ia[a] >> i) & 1) << (63 - 3 * (14 - i) - a);
#pragma unroll
        for (int i = 10; i >= 0; --i) {
            c |= (uint64_t)((ia[0] >> i) & 1) << (5 * i + 1);
            c |= (uint64_t)((ia[1] >> i) & 1) << (5 * i);
            if (i > 0) c |= (uint64_t)((ia[2] >> i) & 1) << (5 * i - 1);
        }
#pragma unroll
        for (int i = 14; i >= 5; --i) {
            c |= (uint64_t)((ib[0] >> i) & 1) << (5 * i - 22);
            c |= (uint64_t)((ib[1] >> i) & 1) << (5 * i - 23);
        }
        return c;
    }
    if (M == HP_RAY_KEYS_COSTA || M == HP_RAY_KEYS_REIS) {
        // computeMortonCodesCosta64 / Reis64 (RayBufferKernels.cu:816-921)
        const float bx = __fadd_rn(__fdiv_rn(rk_atan2(ny, nx), 6.2831854820251465f), 0.5f);
        const float by = __fdiv_rn(rk_acos(nz), 3.1415927410125732f);
        if (M == HP_RAY_KEYS_COSTA) {
            const int ia[3] = {qz(a0, 32767.0f), qz(a1, 32767.0f), qz(a2, 32767.0f)};
            const int ib[2] = {qz(bx, 32767.0f), qz(by, 32767.0f)};
#pragma unroll
            for (int i = 14; i >= 11; --i) {
                c |= (uint64_t)((ib[0] >> i) & 1) << (2 * i + 35);
                c |= (uint64_t)((ib[1] >> i) & 1) << (2 * i + 34);
            }
#pragma unroll
            for (int i = 14; i >= 0; --i)
                for (int a = 0; a < 3; ++a) c |= (uint64_t)((ia[a] >> i) & 1) << (3 * i + 13 - a);
        } else {
            const int ia[3] = {qz(a0, 2097151.0f), qz(a1, 2097151.0f), qz(a2, 2097151.0f)};
            const int ib[2] = {qz(bx, 2097151.0f), qz(by, 2097151.0f)};
#pragma unroll
            for (int i = 20; i >= 14; --i)
                for (int a = 0; a < 3; ++a) c |= (uint64_t)((ia[a] >> i) & 1) << (3 * i + 3 - a);
            c |= (uint64_t)((ia[0] >> 13) & 1) << 42;
#pragma unroll
            for (int i = 20; i >= 0; --i) {
                c |= (uint64_t)((ib[0] >> i) & 1) << (2 * i + 1);
                c |= (uint64_t)((ib[1] >> i) & 1) << (2 * i);
            }
        }
        return c;
    }
    // computeMortonCodesAila64 (RayBufferKernels.cu:556-615)
    const int ax = qz(a0, 8191.0f), ay = qz(a1, 8191.0f), az = qz(a2, 8191.0f);
    const int bx = qz(__fmul_rn(__fadd_rn(nx, 1.0f), 0.5f), 8191.0f);
    const int by = qz(__fmul_rn(__fadd_rn(ny, 1.0f), 0.5f), 8191.0f);
    const int bz = qz(__fmul_rn(__fadd_rn(nz, 1.0f), 0.5f), 8191.0f);
#pragma unroll
    for (int b = 12; b >= 10; --b) {
        const int sh = 63 - 3 * (12 - b);
        c |= (uint64_t)((ax >> b) & 1) << sh;
        c |= (uint64_t)((ay >> b) & 1) << (sh - 1);
        c |= (uint64_t)((az >> b) & 1) << (sh - 2);
    }
#pragma unroll
    for (int b = 9; b >= 1; --b) {
        c |= (uint64_t)((ax >> b) & 1) << (6 * b);
        c |= (uint64_t)((ay >> b) & 1) << (6 * b - 1);
        c |= (uint64_t)((az >> b) & 1) << (6 * b - 2);
    }
#pragma unroll
    for (int b = 12; b >= 4; --b) {
        c |= (uint64_t)((bx >> b) & 1) << (6 * b - 21);
        c |= (uint64_t)((by >> b) & 1) << (6 * b - 22);
        c |= (uint64_t)((bz >> b) & 1) << (6 * b - 23);
    }
    return c;
}

template <int M>
__global__ void __launch_bounds__(256) k_ray_keys(const float4* __restrict__ rays, int64_t n, key_args k,
                                                  uint64_t* __restrict__ keys) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t c = ray_code<M>(__ldg(rays + 2 * i), __ldg(rays + 2 * i + 1), k);
    keys[i] = k.bits == 64 ? c : c >> (64 - k.bits);
}

// Keys of at most 32 bits for a sorted trace, with the sort's digit histograms
// (passes x 256, digit p at bits 8p) counted in shared memory as they are made.
template <int M>
__global__ void __launch_bounds__(256) k_ray_keys32(const float4* __restrict__ rays, int64_t n, key_args k,
                                                    uint32_t* __restrict__ keys, uint32_t* hist, int passes) {
    __shared__ uint32_t sh[4 * 256];
    for (int i = threadIdx.x; i < passes * 256; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t c = ray_code<M>(__ldg(rays + 2 * i), __ldg(rays + 2 * i + 1), k);
        const uint32_t key = (uint32_t)(c >> (64 - k.bits));
        keys[i] = key;
        for (int p = 0; p < passes; ++p) atomicAdd(&sh[p * 256 + ((key >> (8 * p)) & 255u)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += blockDim.x)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// halton (RayGenKernels.cu:20-30): radical inverse of i in the given base.
float halton(int i, int base) {
    double r = 0.0, f = 1.0 / base;
    while (i > 0) {
        r += f * (i % base);
        i /= base;
        f /= base;
    }
    return (float)r;
}

bool invert4(const double* a, double* inv) {
    double m[4][8];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 8; ++c) m[r][c] = c < 4 ? a[4 * r + c] : (c - 4 == r ? 1.0 : 0.0);
    for (int c = 0; c < 4; ++c) {
        int p = c;
        for (int r = c + 1; r < 4; ++r)
            if (std::fabs(m[r][c]) > std::fabs(m[p][c])) p = r;
        if (std::fabs(m[p][c]) < 1e-300) return false;
        if (p != c)
            for (int k = 0; k < 8; ++k) std::swap(m[p][k], m[c][k]);
        const double d = m[c][c];
        for (int k = 0; k < 8; ++k) m[c][k] /= d;
        for (int r = 0; r < 4; ++r) {
            if (r == c) continue;
            const double f = m[r][c];
            for (int k = 0; k < 8; ++k) m[r][k] -= f * m[c][k];
        }
    }
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) inv[4 * r + c] = m[r][4 + c];
    return true;
}

void matmul4(const double* a, const double* b, double* o) {
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            double s = 0.0;
            for (int k = 0; k < 4; ++k) s += a[4 * r + k] * b[4 * k + c];
            o[4 * r + c] = s;
        }
}

// rotate (util/Math.cpp:22-30): rotation by `angle` about a unit axis.
void rot4(double angle, double x, double y, double z, double* R) {
    const double c = std::cos(angle), s = std::sin(angle), t = 1.0 - c;
    const double v[16] = {c + x * x * t,     x * y * t - z * s, x * z * t + y * s, 0,
                          x * y * t + z * s, c + y * y * t,     y * z * t - x * s, 0,
                          z * x * t - y * s, z * y * t + x * s, c + z * z * t,     0,
                          0,                 0,                 0,                 1};
    std::memcpy(R, v, sizeof(v));
}

}  // namespace

extern "C" hp_status hp_pixel_table(int32_t width, int32_t height, int32_t* index_to_pixel) {
    if (width <= 0 || height <= 0 || !index_to_pixel || (int64_t)width * height >= (int64_t(1) << 31))
        return hp_fail(HP_ERR_ARG, "hp_pixel_table: bad size or null output");
    const int bw = width & ~7, bh = height & ~7;
    const int w8 = bw >> 3, h8 = bh >> 3;
    // The reference walks Morton indices over a square of block coordinates and
    // keeps those inside the image; sorting the image's blocks by their Morton
    // code (x bits at even positions) visits them in the same order.
    std::vector<std::pair<uint64_t, int>> blocks;
    blocks.reserve((size_t)w8 * h8);
    for (int ty = 0; ty < h8; ++ty)
        for (int tx = 0; tx < w8; ++tx) {
            uint64_t code = 0;
            for (int k = 0; k < 31; ++k)
                code |= (uint64_t)((tx >> k) & 1) << (2 * k) | (uint64_t)((ty >> k) & 1) << (2 * k + 1);
            blocks.push_back({code, ty * w8 + tx});
        }
    std::sort(blocks.begin(), blocks.end());
    int64_t idx = 0;
    for (const auto& bk : blocks) {
        const int tx = bk.second % w8, ty = bk.second / w8;
        for (int inner = 0; inner < 64; ++inner) {
            const int ix = (inner & 1) | ((inner & 4) >> 1) | ((inner & 16) >> 2);
            const int iy = ((inner & 2) >> 1) | ((inner & 8) >> 2) | ((inner & 32) >> 3);
            index_to_pixel[idx++] = (ty * 8 + iy) * width + (tx * 8 + ix);
        }
    }
    for (int px = 0; px < bw; ++px)
        for (int py = bh; py < height; ++py) index_to_pixel[idx++] = px + py * width;
    for (int py = 0; py < height; ++py)
        for (int px = bw; px < width; ++px) index_to_pixel[idx++] = px + py * width;
    if (idx != (int64_t)width * height) return hp_fail(HP_ERR_ARG, "hp_pixel_table: table incomplete");
    return HP_OK;
}

// inverse(Camera::getProjectionMatrix() * getViewMatrix()) (rt/scene/Camera.cpp:95-109):
// view = Rx(-elev) * Ry(view) * T(-position) with elev = asin(dir.y) and
// view = atan2(dir.x, -dir.z) (Camera::setDirection), no wheel rotation;
// projection = perspective(fovy, width / height, near, far) (util/Math.cpp:10-20).
extern "C" hp_status hp_camera_screen_to_world(const float* position, const float* direction, float fov_deg,
                                               int32_t width, int32_t height, float near_plane, float far_plane,
                                               float* out16) {
    if (!position || !direction || !out16 || width <= 0 || height <= 0 || !(near_plane > 0.0f) ||
        !(far_plane > near_plane) || !(fov_deg > 0.0f && fov_deg < 180.0f))
        return hp_fail(HP_ERR_ARG, "hp_camera_screen_to_world: bad camera");
    double d[3] = {direction[0], direction[1], direction[2]};
    const double len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if (!(len > 0.0)) return hp_fail(HP_ERR_ARG, "hp_camera_screen_to_world: zero direction");
    for (double& x : d) x /= len;
    const double elev = std::asin(d[1]), view = std::atan2(d[0], -d[2]);
    double Rx[16], Ry[16], T[16] = {1, 0, 0, -position[0], 0, 1, 0, -position[1], 0, 0, 1, -position[2], 0, 0, 0, 1};
    rot4(-elev, 1, 0, 0, Rx);
    rot4(view, 0, 1, 0, Ry);
    double RyT[16], V[16], P[16] = {0}, PV[16], inv[16];
    matmul4(Ry, T, RyT);
    matmul4(Rx, RyT, V);
    const double fovy = fov_deg * 3.14159265358979323846 / 180.0;
    const double fy = 1.0 / std::tan(0.5 * fovy), fx = fy / ((double)width / height);
    const double dd = 1.0 / ((double)near_plane - far_plane);
    P[0] = fx;
    P[5] = fy;
    P[10] = ((double)near_plane + far_plane) * dd;
    P[11] = 2.0 * near_plane * far_plane * dd;
    P[14] = -1.0;
    matmul4(P, V, PV);
    if (!invert4(PV, inv)) return hp_fail(HP_ERR_ARG, "hp_camera_screen_to_world: singular matrix");
    for (int k = 0; k < 16; ++k) out16[k] = (float)inv[k];
    return HP_OK;
}

extern "C" hp_status hp_gen_primary_rays(hp_ctx* ctx, const float* position, const float* screen_to_world16,
                                         int32_t width, int32_t height, float max_dist, int32_t sample_index,
                                         const int32_t* index_to_pixel, float* rays, void* stream) {
    if (!ctx || !position || !screen_to_world16 || !rays || width <= 0 || height <= 0 || sample_index < 0)
        return hp_fail(HP_ERR_ARG, "hp_gen_primary_rays: bad argument");
    cam_args c{};
    c.ox = position[0];
    c.oy = position[1];
    c.oz = position[2];
    std::memcpy(c.m, screen_to_world16, sizeof(c.m));
    c.width = width;
    c.height = height;
    c.hx = halton(sample_index, 2);
    c.hy = halton(sample_index, 3);
    c.max_dist = max_dist;
    const int64_t n = (int64_t)width * height;
    k_primary_rays<<<hp_div_up(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        c, index_to_pixel, reinterpret_cast<float4*>(rays), n, ctx->d_status);
    HP_CUDA(cudaGetLastError());
    hp_count_launch();
    return HP_OK;
}

extern "C" hp_status hp_ray_keys(hp_ctx* ctx, const float* rays, int64_t num_rays, const float* ray_box6,
                                 int32_t bits, uint64_t* keys, void* stream) {
    if (!ctx || (num_rays > 0 && (!rays || !keys)) || num_rays < 0 || bits < 1 || bits > 64)
        return hp_fail(HP_ERR_ARG, "hp_ray_keys: bad argument");
    key_args k{};
    const float def[6] = {0.0f, 0.0f, 0.0f, 1.0f, 1.0f, 1.0f};
    const float* b = ray_box6 ? ray_box6 : def;
    for (int a = 0; a < 3; ++a) {
        k.mn[a] = b[a];
        k.mx[a] = b[3 + a];
        const float ext = b[3 + a] - b[a];
        k.inv[a] = ext > 0.0f ? 1.0f / ext : 0.0f;
    }
    k.bits = bits;
    k.ray_length = ctx->ray_length;
    if (num_rays == 0) return HP_OK;
    const unsigned grid = (unsigned)hp_div_up(num_rays, 256);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const float4* r4 = reinterpret_cast<const float4*>(rays);
    switch (ctx->ray_key_method) {
        case HP_RAY_KEYS_TWO_POINT: k_ray_keys<HP_RAY_KEYS_TWO_POINT><<<grid, 256, 0, s>>>(r4, num_rays, k, keys); break;
        case HP_RAY_KEYS_PARABOLOID: k_ray_keys<HP_RAY_KEYS_PARABOLOID><<<grid, 256, 0, s>>>(r4, num_rays, k, keys); break;
        case HP_RAY_KEYS_OCTAHEDRON: k_ray_keys<HP_RAY_KEYS_OCTAHEDRON><<<grid, 256, 0, s>>>(r4, num_rays, k, keys); break;
        case HP_RAY_KEYS_ORIGIN: k_ray_keys<HP_RAY_KEYS_ORIGIN><<<grid, 256, 0, s>>>(r4, num_rays, k, keys); break;
        case HP_RAY_KEYS_COSTA: k_ray_keys<HP_RAY_KEYS_COSTA><<<grid, 256, 0, s>>>(r4, num_rays, k, keys); break;
        case HP_RAY_KEYS_REIS: k_ray_keys<HP_RAY_KEYS_REIS><<<grid, 256, 0, s>>>(r4, num_rays, k, keys); break;
        default: k_ray_keys<HP_RAY_KEYS_AILA><<<grid, 256, 0, s>>>(r4, num_rays, k, keys); break;
    }
    HP_CUDA(cudaGetLastError());
    hp_count_launch();
    return HP_OK;
}

namespace {

key_args unit_key_args(const hp_ctx* ctx, int bits) {
    key_args k{};
    for (int a = 0; a < 3; ++a) {
        k.mn[a] = 0.0f;
        k.mx[a] = 1.0f;
        k.inv[a] = 1.0f;
    }
    k.bits = bits;
    k.ray_length = ctx->ray_length;
    return k;
}

}  // namespace

size_t hp_ray_order_scratch_bytes(int64_t n, int bits, int block) {
    const int kb = bits <= 32 ? 4 : 8;
    const hp_sort_plan plan = hp_sort_make_plan(std::max<int64_t>(n, 1), kb, bits, block);
    return 2 * hp_carve::pad((size_t)n * kb) + hp_carve::pad(plan.scratch_bytes) +
           hp_carve::pad(hp_sort_hist_bytes(plan.passes));
}

hp_status hp_ray_order(hp_ctx* ctx, const float* rays, int64_t n, int bits, int32_t* order, void* scratch,
                       cudaStream_t s) {
    if (n <= 0) return HP_OK;
    const int kb = bits <= 32 ? 4 : 8;
    const hp_sort_plan plan = hp_sort_make_plan(n, kb, bits, ctx->tune.sort_block);
    hp_carve cv(reinterpret_cast<char*>(scratch));
    void* keys = cv.take<char>((size_t)n * kb);
    void* skeys = cv.take<char>((size_t)n * kb);
    void* sort_scratch = cv.take<char>(plan.scratch_bytes);
    uint32_t* hist = cv.take<uint32_t>((size_t)plan.passes * 256);
    if (kb == 8) {  // wide keys: the public key kernel, histograms by the sort
        HP_TRY(hp_ray_keys(ctx, rays, n, nullptr, bits, reinterpret_cast<uint64_t*>(keys), s));
        hp_sort_args sa{keys, nullptr, skeys, order, sort_scratch, hist, false, ctx->d_status, nullptr};
        return hp_sort_run(plan, sa, s);
    }
    HP_CUDA(cudaMemsetAsync(hist, 0, hp_sort_hist_bytes(plan.passes), s));
    const key_args k = unit_key_args(ctx, bits);
    const unsigned grid = (unsigned)std::min<int64_t>(hp_div_up(n, 256), (int64_t)ctx->sm_count * 8);
    const float4* r4 = reinterpret_cast<const float4*>(rays);
    uint32_t* k32 = reinterpret_cast<uint32_t*>(keys);
    const int P = plan.passes;
    switch (ctx->ray_key_method) {
        case HP_RAY_KEYS_TWO_POINT: k_ray_keys32<HP_RAY_KEYS_TWO_POINT><<<grid, 256, 0, s>>>(r4, n, k, k32, hist, P); break;
        case HP_RAY_KEYS_PARABOLOID: k_ray_keys32<HP_RAY_KEYS_PARABOLOID><<<grid, 256, 0, s>>>(r4, n, k, k32, hist, P); break;
        case HP_RAY_KEYS_OCTAHEDRON: k_ray_keys32<HP_RAY_KEYS_OCTAHEDRON><<<grid, 256, 0, s>>>(r4, n, k, k32, hist, P); break;
        case HP_RAY_KEYS_ORIGIN: k_ray_keys32<HP_RAY_KEYS_ORIGIN><<<grid, 256, 0, s>>>(r4, n, k, k32, hist, P); break;
        case HP_RAY_KEYS_COSTA: k_ray_keys32<HP_RAY_KEYS_COSTA><<<grid, 256, 0, s>>>(r4, n, k, k32, hist, P); break;
        case HP_RAY_KEYS_REIS: k_ray_keys32<HP_RAY_KEYS_REIS><<<grid, 256, 0, s>>>(r4, n, k, k32, hist, P); break;
        default: k_ray_keys32<HP_RAY_KEYS_AILA><<<grid, 256, 0, s>>>(r4, n, k, k32, hist, P); break;
    }
    HP_CUDA(cudaGetLastError());
    hp_count_launch();
    hp_sort_args sa{keys, nullptr, skeys, order, sort_scratch, hist, true, ctx->d_status, nullptr};
    return hp_sort_run(plan, sa, s);
}

// RayBuffer::setMortonCodeMethod / setRayLength (rt/ray/RayBuffer.cpp:167-195).
extern "C" hp_status hp_ctx_set_ray_keys(hp_ctx* ctx, int32_t method, float ray_length) {
    if (!ctx) return hp_fail(HP_ERR_ARG, "hp_ctx_set_ray_keys: null context");
    if (method < HP_RAY_KEYS_TWO_POINT || method > HP_RAY_KEYS_REIS)
        return hp_fail(HP_ERR_ARG, "hp_ctx_set_ray_keys: unknown method");
    if (!(ray_length >= 0.0f)) return hp_fail(HP_ERR_ARG, "hp_ctx_set_ray_keys: ray length must be >= 0");
    ctx->ray_key_method = method;
    ctx->ray_length = ray_length;
    return HP_OK;
}

// Renderer::stringToMortonCodeMethod (rt/renderer/Renderer.cpp:37-52): the
// Reis method is spelled "reise"; any other string selects the two-point method.
extern "C" int32_t hp_ray_keys_method(const char* name) {
    if (!name) return HP_RAY_KEYS_TWO_POINT;
    if (!std::strcmp(name, "aila")) return HP_RAY_KEYS_AILA;
    if (!std::strcmp(name, "paraboloid")) return HP_RAY_KEYS_PARABOLOID;
    if (!std::strcmp(name, "octahedron")) return HP_RAY_KEYS_OCTAHEDRON;
    if (!std::strcmp(name, "origin")) return HP_RAY_KEYS_ORIGIN;
    if (!std::strcmp(name, "costa")) return HP_RAY_KEYS_COSTA;
    if (!std::strcmp(name, "reise")) return HP_RAY_KEYS_REIS;
    return HP_RAY_KEYS_TWO_POINT;
}

extern "C" hp_status hp_trace_sorted(hp_ctx* ctx, const hp_bvh* bvh, const float* rays, int64_t num_rays,
                                     int32_t* results, int32_t* stats, uint32_t flags, int32_t bits,
                                     int32_t* order_out, void* stream) {
    if (!ctx || !bvh || !bvh->impl || num_rays < 0 || (num_rays > 0 && (!rays || !results)))
        return hp_fail(HP_ERR_ARG, "hp_trace_sorted: bad argument");
    if (bits < 1 || bits > 64) return hp_fail(HP_ERR_ARG, "hp_trace_sorted: bits must be in [1,64]");
    if (num_rays >= (int64_t(1) << 30)) return hp_fail(HP_ERR_ARG, "hp_trace_sorted: too many rays");
    if (num_rays == 0) return HP_OK;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const size_t key_bytes = hp_ray_order_scratch_bytes(num_rays, bits, ctx->tune.sort_block);
    HP_TRY(hp_ctx_reserve(ctx, hp_carve::pad(num_rays * 4) + key_bytes, s));
    hp_carve cv(ctx->arena);
    int32_t* order_tmp = cv.take<int32_t>(num_rays);
    int32_t* order = order_out ? order_out : order_tmp;
    void* scratch = cv.take<char>(key_bytes);
    hp_mark(ctx, s, "ray_sort_begin");
    HP_TRY(hp_ray_order(ctx, rays, num_rays, bits, order, scratch, s));
    hp_mark(ctx, s, "ray_sort");
    return hp_trace_launch(ctx, reinterpret_cast<const hp_bvh_impl*>(bvh->impl), bvh->num_refs, rays, num_rays,
                           results, stats, flags, s, order);
}
