// Synthetic meshes and rays. Every random number is a pure function of
// (seed, item, slot) -- a SplitMix64 finaliser over a counter -- so the output
// is identical for any number of OpenMP threads, and the oracle, the benchmark
// and the tests all see the same bytes. Uniform floats are (h >> 40) * 2^-24.
// The reference's scenes are not available; these generators stand in for them
// with the shapes and value distributions of the benchmark configurations.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include "hp_internal.h"

namespace {

inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

inline float u01(uint64_t seed, uint64_t item, uint32_t slot) {
    uint64_t h = mix64((seed * 0xD1B54A32D192ED03ull) ^ (item * 64u + slot));
    return (float)((double)(h >> 40) * (1.0 / 16777216.0));
}

inline double u01d(uint64_t seed, uint64_t item, uint32_t slot) { return (double)u01(seed, item, slot); }

// Box-Muller normal from two uniforms (the first shifted into (0, 1]).
inline double normal(uint64_t seed, uint64_t item, uint32_t slot) {
    double a = 1.0 - u01d(seed, item, slot);
    double b = u01d(seed, item, slot + 1);
    return std::sqrt(-2.0 * std::log(a)) * std::cos(6.283185307179586 * b);
}

const double TWO_PI = 6.283185307179586;

}  // namespace

extern "C" {

hp_status hp_gen_uniform_mesh(uint64_t seed, int64_t n, float h, float* v, int32_t* t) {
    if (n < 0 || (n > 0 && (!v || !t))) return hp_fail(HP_ERR_ARG, "hp_gen_uniform_mesh: bad argument");
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const float c[3] = {u01(seed, i, 0), u01(seed, i, 1), u01(seed, i, 2)};
        for (int k = 0; k < 3; ++k) {
            for (int a = 0; a < 3; ++a) {
                float r = u01(seed, i, 3 + 3 * k + a);
                v[9 * i + 3 * k + a] = c[a] + (2.0f * r - 1.0f) * h;
            }
            t[3 * i + k] = (int32_t)(3 * i + k);
        }
    }
    return HP_OK;
}

hp_status hp_gen_clustered_mesh(uint64_t seed, int64_t n, int32_t n_clusters, float sigma, float h,
                                float* v, int32_t* t) {
    if (n < 0 || n_clusters <= 0 || (n > 0 && (!v || !t)))
        return hp_fail(HP_ERR_ARG, "hp_gen_clustered_mesh: bad argument");
    const uint64_t cseed = seed ^ 0xA5A5A5A55A5A5A5Aull;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const int64_t cl = i % n_clusters;
        float c[3];
        for (int a = 0; a < 3; ++a)
            c[a] = u01(cseed, cl, a) + (float)((double)sigma * normal(seed, i, 2 * a));
        for (int k = 0; k < 3; ++k) {
            for (int a = 0; a < 3; ++a) {
                float r = u01(seed, i, 8 + 3 * k + a);
                v[9 * i + 3 * k + a] = c[a] + (2.0f * r - 1.0f) * h;
            }
            t[3 * i + k] = (int32_t)(3 * i + k);
        }
    }
    return HP_OK;
}

hp_status hp_gen_heightfield(uint64_t seed, int32_t nx, int32_t ny, float sx, float sy, int32_t n_waves,
                             float* v, int32_t* t) {
    if (nx < 2 || ny < 2 || n_waves < 0 || !v || !t) return hp_fail(HP_ERR_ARG, "hp_gen_heightfield: bad argument");
    double amp[64], freq[64], ux[64], uy[64], phase[64];
    if (n_waves > 64) return hp_fail(HP_ERR_ARG, "hp_gen_heightfield: at most 64 waves");
    for (int k = 0; k < n_waves; ++k) {
        amp[k] = 0.05 * u01d(seed, k, 0);
        freq[k] = 1.0 + 31.0 * u01d(seed, k, 1);
        double th = TWO_PI * u01d(seed, k, 2);
        ux[k] = std::cos(th);
        uy[k] = std::sin(th);
        phase[k] = TWO_PI * u01d(seed, k, 3);
    }
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < ny; ++j) {
        for (int64_t i = 0; i < nx; ++i) {
            double x = (double)sx * (double)i / (double)(nx - 1);
            double y = (double)sy * (double)j / (double)(ny - 1);
            double z = 0.0;
            for (int k = 0; k < n_waves; ++k)
                z += amp[k] * std::sin(TWO_PI * freq[k] * (ux[k] * x + uy[k] * y) + phase[k]);
            int64_t id = j * nx + i;
            v[3 * id + 0] = (float)x;
            v[3 * id + 1] = (float)y;
            v[3 * id + 2] = (float)z;
        }
    }
    const int64_t cx = nx - 1;
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < ny - 1; ++j) {
        for (int64_t i = 0; i < cx; ++i) {
            int64_t c = j * cx + i;
            int32_t v00 = (int32_t)(j * nx + i), v10 = v00 + 1, v01 = (int32_t)(v00 + nx), v11 = v01 + 1;
            int32_t* a = t + 6 * c;
            a[0] = v00; a[1] = v10; a[2] = v11;
            a[3] = v00; a[4] = v11; a[5] = v01;
        }
    }
    return HP_OK;
}

hp_status hp_gen_rays_targeted(uint64_t seed, int64_t n, float lo, float hi, float* rays) {
    if (n < 0 || (n > 0 && !rays)) return hp_fail(HP_ERR_ARG, "hp_gen_rays_targeted: bad argument");
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double o[3], d[3], len = 0.0;
        for (int a = 0; a < 3; ++a) {
            o[a] = (double)(lo + (hi - lo) * u01(seed, i, a));
            double tg = u01d(seed, i, 3 + a);
            d[a] = tg - o[a];
            len += d[a] * d[a];
        }
        len = std::sqrt(len);
        if (len == 0.0) { d[0] = 0.0; d[1] = 0.0; d[2] = 1.0; len = 1.0; }
        float* r = rays + 8 * i;
        r[0] = (float)o[0]; r[1] = (float)o[1]; r[2] = (float)o[2]; r[3] = 0.0f;
        r[4] = (float)(d[0] / len); r[5] = (float)(d[1] / len); r[6] = (float)(d[2] / len);
        r[7] = INFINITY;
    }
    return HP_OK;
}

hp_status hp_gen_rays_sphere(uint64_t seed, int64_t n, const float* box, float* rays) {
    if (n < 0 || !box || (n > 0 && !rays)) return hp_fail(HP_ERR_ARG, "hp_gen_rays_sphere: bad argument");
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        float* r = rays + 8 * i;
        for (int a = 0; a < 3; ++a) r[a] = box[a] + (box[3 + a] - box[a]) * u01(seed, i, a);
        r[3] = 0.0f;
        double z = 2.0 * u01d(seed, i, 3) - 1.0;
        double phi = TWO_PI * u01d(seed, i, 4);
        double s = std::sqrt(std::max(0.0, 1.0 - z * z));
        r[4] = (float)(s * std::cos(phi));
        r[5] = (float)(s * std::sin(phi));
        r[6] = (float)z;
        r[7] = INFINITY;
    }
    return HP_OK;
}

hp_status hp_gen_rays_grid_down(uint64_t seed, int32_t nx, int32_t ny, float sx, float sy, float z0,
                                float* rays) {
    if (nx <= 0 || ny <= 0 || !rays) return hp_fail(HP_ERR_ARG, "hp_gen_rays_grid_down: bad argument");
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < ny; ++j) {
        for (int64_t i = 0; i < nx; ++i) {
            int64_t id = j * nx + i;
            float* r = rays + 8 * id;
            r[0] = (float)(((double)i + u01d(seed, id, 0)) * (double)sx / (double)nx);
            r[1] = (float)(((double)j + u01d(seed, id, 1)) * (double)sy / (double)ny);
            r[2] = z0;
            r[3] = 0.0f;
            r[4] = 0.0f; r[5] = 0.0f; r[6] = -1.0f;
            r[7] = INFINITY;
        }
    }
    return HP_OK;
}

}  // extern "C"
