// CPU ORACLE — test infrastructure only.
//
// A plain C++/OpenMP restatement of the reference's build-and-trace path
// (meistdan/hippie, paths relative to src/hippie/). It is the checker the
// parity tests compare the CUDA library against, and the CPU baseline the
// benchmark times; nothing in the shipped library calls it.
//
// Each function cites the reference code it restates. Floating-point
// expressions are written with the same explicit fmaf calls the CUDA kernels
// use (this file is compiled with -ffp-contract=off), so oracle and GPU agree
// bit for bit. Two places differ from the reference's fast-math JIT build and
// are handled explicitly:
//   * the Morton scale 1/diagonal is an approximate quotient on the GPU; the
//     oracle takes that value as an input (or uses the IEEE quotient when run
//     alone);
//   * reciprocals in woopify and traversal use IEEE 1/x on both sides.
// Parity pin: the reference ships no tests, fixtures or golden vectors (its
// test/ folder holds benchmark sweep scripts only), so this restatement is
// pinned by known-answer vectors derived by hand from the reference formulas
// (tests/golden/) and by structural invariants; see the tests.
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const float MAXF = 3.402823466e+38f;

// cvt.rzi.u32.f32: truncate toward zero, saturate, NaN -> 0.
inline uint32_t f2u_rz_sat(float x) {
    if (!(x > 0.0f)) return 0u;
    if (x >= 4294967296.0f) return 0xffffffffu;
    return (uint32_t)x;
}

// rt/HipUtil.h:35-49
inline uint32_t spread10(uint32_t x) {
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}
inline uint32_t morton30(uint32_t x, uint32_t y, uint32_t z) {
    return spread10(x) | (spread10(y) << 1) | (spread10(z) << 2);
}
// rt/HipUtil.h:72-82
inline uint64_t morton60(uint32_t x, uint32_t y, uint32_t z) {
    uint64_t lo = morton30(x & 1023u, y & 1023u, z & 1023u);
    uint64_t hi = morton30(x >> 10, y >> 10, z >> 10);
    return (hi << 30) | lo;
}

// util/AABB.h:33 with the fast-math contraction 2*fma(dz,dx,fma(dx,dy,dy*dz)).
inline float area6(float mnx, float mny, float mnz, float mxx, float mxy, float mxz) {
    if (!(mnx <= mxx && mny <= mxy && mnz <= mxz)) return 0.0f;
    float dx = mxx - mnx, dy = mxy - mny, dz = mxz - mnz;
    return 2.0f * std::fmaf(dz, dx, std::fmaf(dx, dy, dy * dz));
}

// detImpl<3> (util/Math.h:326-330), terms in reference order with the
// contraction nvcc applies to that expression under fast math: the first
// difference fuses the first product over the second, each later term is one fma.
inline float det3(const float* a) {
#define A(r, c) a[(r) + 3 * (c)]
    float acc = std::fmaf(A(0, 0) * A(1, 1), A(2, 2), -((A(0, 0) * A(1, 2)) * A(2, 1)));
    acc = std::fmaf(A(1, 0) * A(2, 1), A(0, 2), acc);
    acc = std::fmaf(-(A(1, 0) * A(2, 2)), A(0, 1), acc);
    acc = std::fmaf(A(2, 0) * A(0, 1), A(1, 2), acc);
    acc = std::fmaf(-(A(2, 0) * A(0, 2)), A(1, 1), acc);
#undef A
    return acc;
}

// woopifyTriangle (rt/bvh/HipBVHKernels.cu:12-33) with inverse() (util/Math.h:350-367).
void woop(const float* v0, const float* v1, const float* v2, float* w /*12*/) {
    float ax = v0[0] - v2[0], ay = v0[1] - v2[1], az = v0[2] - v2[2];
    float bx = v1[0] - v2[0], by = v1[1] - v2[1], bz = v1[2] - v2[2];
    float nx = std::fmaf(ay, bz, -(az * by));
    float ny = std::fmaf(az, bx, -(ax * bz));
    float nz = std::fmaf(ax, by, -(ay * bx));
    float M[16] = {ax, ay, az, 0.0f, bx, by, bz, 0.0f, nx, ny, nz, 0.0f, v2[0], v2[1], v2[2], 1.0f};
    float R[16];
    float d = 0.0f, si = 1.0f;
    for (int i = 0; i < 4; ++i) {
        float sj = si;
        for (int j = 0; j < 4; ++j) {
            float sub[9];
            for (int k = 0; k < 3; ++k)
                for (int l = 0; l < 3; ++l)
                    sub[k + 3 * l] = M[((k < j) ? k : k + 1) + 4 * ((l < i) ? l : l + 1)];
            float dd = det3(sub) * sj;
            R[i + 4 * j] = dd;
            d = std::fmaf(dd, M[j + 4 * i], d);
            sj = -sj;
        }
        si = -si;
    }
    float rd = (d != 0.0f) ? 1.0f / d : 0.0f;
    for (int k = 0; k < 16; ++k) R[k] = (R[k] * rd) * 4.0f;
#define IM(c, r) R[(r) + 4 * (c)]
    w[0] = IM(0, 2); w[1] = IM(1, 2); w[2] = IM(2, 2); w[3] = -IM(3, 2);
    w[4] = IM(0, 0); w[5] = IM(1, 0); w[6] = IM(2, 0); w[7] = IM(3, 0);
    w[8] = IM(0, 1); w[9] = IM(1, 1); w[10] = IM(2, 1); w[11] = IM(3, 1);
#undef IM
}

template <typename K> inline int clz_k(K x);
template <> inline int clz_k<uint64_t>(uint64_t x) { return x ? __builtin_clzll(x) : 64; }

// delta<unsigned long long> (rt/bvh/HipBVHUtil.h:17-25).
inline int delta(const uint64_t* k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    uint64_t a = k[i], b = k[j];
    if (a != b) return clz_k<uint64_t>(a ^ b);
    return clz_k<uint64_t>((uint64_t)(int64_t)(i ^ j)) + 64;
}

inline void tri_box(const float* verts, const int32_t* tris, int64_t t, float* mn, float* mx) {
    for (int a = 0; a < 3; ++a) { mn[a] = MAXF; mx[a] = -MAXF; }
    for (int k = 0; k < 3; ++k) {
        const float* p = verts + 3 * (int64_t)tris[3 * t + k];
        for (int a = 0; a < 3; ++a) {
            mn[a] = std::min(mn[a], p[a]);
            mx[a] = std::max(mx[a], p[a]);
        }
    }
}

struct bin_node {
    float f[12];
    int32_t c0, c1, size, parent;
};
static_assert(sizeof(bin_node) == 64, "node");

void make_node(bin_node& n, const float* amn, const float* amx, const float* bmn, const float* bmx,
               int c0, int c1, int size, int parent) {
    n.f[0] = amn[0]; n.f[1] = amx[0]; n.f[2] = amn[1]; n.f[3] = amx[1];
    n.f[4] = bmn[0]; n.f[5] = bmx[0]; n.f[6] = bmn[1]; n.f[7] = bmx[1];
    n.f[8] = amn[2]; n.f[9] = amx[2]; n.f[10] = bmn[2]; n.f[11] = bmx[2];
    n.c0 = c0; n.c1 = c1; n.size = size; n.parent = parent;
}

}  // namespace

extern "C" {

// ---- A1/A2: setupBoxes (rt/bvh/LBVHBuilderKernels.cu:65-98) + scene box ----------
void or_tri_boxes(const float* verts, const int32_t* tris, int64_t n, float* bmin4, float* bmax4,
                  float* scene_box) {
    float smn[3] = {MAXF, MAXF, MAXF}, smx[3] = {-MAXF, -MAXF, -MAXF};
    for (int64_t i = 0; i < n; ++i) {
        float mn[3], mx[3];
        tri_box(verts, tris, i, mn, mx);
        for (int a = 0; a < 3; ++a) {
            bmin4[4 * i + a] = mn[a];
            bmax4[4 * i + a] = mx[a];
            smn[a] = std::min(smn[a], mn[a]);
            smx[a] = std::max(smx[a], mx[a]);
        }
        bmin4[4 * i + 3] = 0.0f;
        bmax4[4 * i + 3] = 0.0f;
    }
    for (int a = 0; a < 3; ++a) { scene_box[a] = smn[a]; scene_box[3 + a] = smx[a]; }
}

// ---- A3: computeMortonCodes60 (rt/bvh/LBVHBuilderKernels.cu:131-160) --------------
// scale: the per-axis 1/diagonal to use; if null, the IEEE quotient.
void or_morton(int64_t n, const float* bmin4, const float* bmax4, const float* scene_box,
               const float* scale_in, int bits, uint64_t* keys, float* scale_out) {
    float scale[3];
    for (int a = 0; a < 3; ++a)
        scale[a] = scale_in ? scale_in[a] : 1.0f / (scene_box[3 + a] - scene_box[a]);
    if (scale_out) for (int a = 0; a < 3; ++a) scale_out[a] = scale[a];
    const float q20 = 1048575.0f;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        uint32_t q[3];
        for (int a = 0; a < 3; ++a) {
            float c = (bmin4[4 * i + a] + bmax4[4 * i + a]) * 0.5f;
            q[a] = f2u_rz_sat(((c - scene_box[a]) * scale[a]) * q20);
        }
        keys[i] = morton60(q[0], q[1], q[2]) >> (60 - bits);
    }
}

// ---- A4: stable sort (RadixSort::sort, radix_sort/RadixSort.cpp:181-238) -----------
// Stable LSD radix sort by key bits [0, bits), 8-bit digits, OpenMP histograms.
// sorted_refs receives the original index of every sorted position.
void or_sort(int64_t n, const uint64_t* keys, int bits, uint64_t* sorted_keys, int32_t* sorted_refs) {
    std::vector<uint64_t> ka(keys, keys + n), kb(n);
    std::vector<int32_t> va(n), vb(n);
    for (int64_t i = 0; i < n; ++i) va[i] = (int32_t)i;
    const int passes = (bits + 7) / 8;
    for (int p = 0; p < passes; ++p) {
        const int shift = 8 * p;
        int nt = 1;
#ifdef _OPENMP
        nt = omp_get_max_threads();
#endif
        std::vector<int64_t> hist((size_t)nt * 256, 0);
        const int64_t chunk = (n + nt - 1) / nt;
#pragma omp parallel num_threads(nt)
        {
            int t = 0;
#ifdef _OPENMP
            t = omp_get_thread_num();
#endif
            int64_t b = std::min(n, t * chunk), e = std::min(n, b + chunk);
            int64_t* h = &hist[(size_t)t * 256];
            for (int64_t i = b; i < e; ++i) h[(ka[i] >> shift) & 255]++;
        }
        int64_t run = 0;
        for (int d = 0; d < 256; ++d)
            for (int t = 0; t < nt; ++t) {
                int64_t c = hist[(size_t)t * 256 + d];
                hist[(size_t)t * 256 + d] = run;
                run += c;
            }
#pragma omp parallel num_threads(nt)
        {
            int t = 0;
#ifdef _OPENMP
            t = omp_get_thread_num();
#endif
            int64_t b = std::min(n, t * chunk), e = std::min(n, b + chunk);
            int64_t* h = &hist[(size_t)t * 256];
            for (int64_t i = b; i < e; ++i) {
                int64_t pos = h[(ka[i] >> shift) & 255]++;
                kb[pos] = ka[i];
                vb[pos] = va[i];
            }
        }
        ka.swap(kb);
        va.swap(vb);
    }
    std::memcpy(sorted_keys, ka.data(), n * 8);
    std::memcpy(sorted_refs, va.data(), n * 4);
}

// ---- A6: construct<T> (rt/bvh/LBVHBuilderKernels.cu:11-63) ----------------------------
void or_karras(int n, const uint64_t* keys, int32_t* parent, int32_t* left, int32_t* right) {
    if (n >= 1) parent[0] = -1;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n - 1; ++i) {
        const int dr = delta(keys, n, i, i + 1), dl = delta(keys, n, i, i - 1);
        const int d = (dr - dl > 0) - (dr - dl < 0);
        const int dmin = delta(keys, n, i, i - d);
        int lmax = 2;
        while (delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
        int l = 0;
        for (int t = lmax >> 1; t >= 1; t >>= 1)
            if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
        const int j = i + l * d;
        const int dnode = delta(keys, n, i, j);
        int s = 0, k = 2, t;
        do {
            t = (l + k - 1) / k;
            k <<= 1;
            if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
        } while (t > 1);
        const int gamma = i + s * d + std::min(d, 0);
        int lc = gamma, rc = gamma + 1;
        if (std::min(i, j) == gamma) lc += n - 1;
        if (std::max(i, j) == gamma + 1) rc += n - 1;
        left[i] = lc;
        right[i] = rc;
        parent[lc] = i;
        parent[rc] = i;
    }
    // leaf nodes (setupLeaves, LBVHBuilderKernels.cu:162-195): left = i, right = i + 1
    for (int i = 0; i < n; ++i) {
        left[n - 1 + i] = i;
        right[n - 1 + i] = i + 1;
    }
}

// ---- A5/A7 + collapse DP: refit (LBVHBuilderKernels.cu:254-305),
// computeSizes (BVHCollapserKernels.cu:11-56), computeNodeStatesAdaptive (:58-136),
// computeNodeStates (:138-184). Post-order over the tree from the root.
// Outputs per node (2n-1): box min/max (4 floats, w = 0), size, cost, state.
void or_refit(int n, const float* verts, const int32_t* tris, const int32_t* sorted_tri,
              const int32_t* parent, const int32_t* left, const int32_t* right, float ct, float ci,
              int adaptive, int max_leaf, float* bmin4, float* bmax4, int32_t* size, float* cost,
              int32_t* state) {
    (void)parent;
    const int nn = 2 * n - 1;
    for (int p = 0; p < n; ++p) {
        const int j = n - 1 + p;
        float mn[3], mx[3];
        tri_box(verts, tris, sorted_tri[p], mn, mx);
        for (int a = 0; a < 3; ++a) { bmin4[4 * j + a] = mn[a]; bmax4[4 * j + a] = mx[a]; }
        bmin4[4 * j + 3] = bmax4[4 * j + 3] = 0.0f;
        size[j] = 1;
        cost[j] = adaptive ? ci * area6(mn[0], mn[1], mn[2], mx[0], mx[1], mx[2]) : 0.0f;
        state[j] = 0;
    }
    if (n < 2) return;
    // iterative post-order
    std::vector<int> stack;
    std::vector<char> expanded(nn, 0);
    stack.push_back(0);
    while (!stack.empty()) {
        int v = stack.back();
        if (v >= n - 1) { stack.pop_back(); continue; }
        if (!expanded[v]) {
            expanded[v] = 1;
            stack.push_back(right[v]);
            stack.push_back(left[v]);
            continue;
        }
        stack.pop_back();
        const int l = left[v], r = right[v];
        float mn[3], mx[3];
        for (int a = 0; a < 3; ++a) {
            mn[a] = std::min(bmin4[4 * l + a], bmin4[4 * r + a]);
            mx[a] = std::max(bmax4[4 * l + a], bmax4[4 * r + a]);
            bmin4[4 * v + a] = mn[a];
            bmax4[4 * v + a] = mx[a];
        }
        bmin4[4 * v + 3] = bmax4[4 * v + 3] = 0.0f;
        size[v] = size[l] + size[r];
        if (adaptive) {
            const float A = area6(mn[0], mn[1], mn[2], mx[0], mx[1], mx[2]);
            const float c_int = std::fmaf(ct, A, cost[l]) + cost[r];
            const float c_leaf = (ci * A) * (float)size[v];
            state[v] = (c_leaf < c_int) ? 0 : 1;
            cost[v] = state[v] ? c_int : c_leaf;
        } else {
            state[v] = (size[v] <= max_leaf) ? 0 : 1;
            cost[v] = 0.0f;
        }
    }
}

// ---- A9/A10: collapse into 64-byte binary nodes ----------------------------------------
// Leaf assignment as computeLeafIndices (BVHCollapserKernels.cu:186-217): the
// leaf of a reference is its topmost state-0 ancestor below the root (the
// root is always interior). Node numbering is the canonical order for trees
// over contiguous reference ranges: interior nodes by split position with the
// root moved to 0, leaves by their first reference; triangles stay in sorted
// order. Returns the node count; counts[0] = interior, counts[1] = leaves.
int64_t or_collapse(int n, const int32_t* parent, const int32_t* left, const int32_t* right,
                    const float* bmin4, const float* bmax4, const int32_t* size, const int32_t* state,
                    void* nodes_out, int32_t* counts) {
    bin_node* out = reinterpret_cast<bin_node*>(nodes_out);
    if (n < 2) { counts[0] = counts[1] = 0; return 0; }
    const int nn = 2 * n - 1;
    // lo/hi range of every node
    std::vector<int> lo(nn), hi(nn);
    for (int p = 0; p < n; ++p) lo[n - 1 + p] = hi[n - 1 + p] = p;
    {
        std::vector<int> st{0};
        std::vector<char> ex(nn, 0);
        while (!st.empty()) {
            int v = st.back();
            if (v >= n - 1) { st.pop_back(); continue; }
            if (!ex[v]) { ex[v] = 1; st.push_back(right[v]); st.push_back(left[v]); continue; }
            st.pop_back();
            lo[v] = lo[left[v]];
            hi[v] = hi[right[v]];
        }
    }
    // leaf index of every reference (walk to the root)
    std::vector<int> leaf_of(n);
    for (int p = 0; p < n; ++p) {
        int node = n - 1 + p, leaf = node, par = parent[node];
        while (par > 0) {
            if (state[par] == 0) leaf = par;
            node = par;
            par = parent[node];
        }
        leaf_of[p] = leaf;
    }
    std::vector<char> is_leaf(nn, 0), alive(nn, 0);
    for (int p = 0; p < n; ++p) is_leaf[leaf_of[p]] = 1;
    // surviving interior nodes: ancestors of collapsed leaves
    for (int v = 0; v < nn; ++v)
        if (is_leaf[v]) {
            alive[v] = 1;
            for (int a = parent[v]; a >= 0 && !alive[a]; a = parent[a]) alive[a] = 1;
        }
    // numbering
    std::vector<int> split_rank(n - 1, -1);  // by split position gamma
    int num_int = 0;
    std::vector<int> gamma_of(n - 1);
    for (int v = 0; v < n - 1; ++v) gamma_of[v] = hi[left[v]];
    std::vector<int> int_at(n - 1, -1);
    for (int v = 0; v < n - 1; ++v)
        if (alive[v] && !is_leaf[v]) int_at[gamma_of[v]] = v;
    std::vector<int> new_int(nn, -1);
    for (int g = 0; g < n - 1; ++g)
        if (int_at[g] >= 0) split_rank[g] = num_int++;
    const int root_rank = split_rank[gamma_of[0]];
    for (int v = 0; v < n - 1; ++v)
        if (alive[v] && !is_leaf[v]) {
            int r = split_rank[gamma_of[v]];
            new_int[v] = (v == 0) ? 0 : (r < root_rank ? r + 1 : r);
        }
    std::vector<int> leaf_rank(n, -1);
    int num_leaf = 0;
    std::vector<int> leaf_at(n, -1);
    for (int v = 0; v < nn; ++v)
        if (is_leaf[v]) leaf_at[lo[v]] = v;
    for (int p = 0; p < n; ++p)
        if (leaf_at[p] >= 0) leaf_rank[p] = num_leaf++;
    auto ref_of = [&](int v) -> int {
        if (is_leaf[v]) return ~(num_int + leaf_rank[lo[v]]);
        return new_int[v];
    };
    auto box = [&](int v, float* mn, float* mx) {
        for (int a = 0; a < 3; ++a) { mn[a] = bmin4[4 * v + a]; mx[a] = bmax4[4 * v + a]; }
    };
    for (int v = 0; v < nn; ++v) {
        if (!alive[v]) continue;
        const int par = (v == 0) ? -1 : new_int[parent[v]];
        if (is_leaf[v]) {
            float mn[3], mx[3];
            box(v, mn, mx);
            make_node(out[num_int + leaf_rank[lo[v]]], mn, mx, mn, mx, lo[v], hi[v] + 1, ~size[v], par);
        } else {
            float amn[3], amx[3], bmn[3], bmx[3];
            box(left[v], amn, amx);
            box(right[v], bmn, bmx);
            make_node(out[new_int[v]], amn, amx, bmn, bmx, ref_of(left[v]), ref_of(right[v]), size[v], par);
        }
    }
    counts[0] = num_int;
    counts[1] = num_leaf;
    return (int64_t)num_int + num_leaf;
}

// ---- A11: woopifyTriangles (rt/bvh/HipBVHKernels.cu:35-65) ---------------------------------
void or_woopify(int64_t n, const float* verts, const int32_t* tris, const int32_t* tri_idx, float* woop4) {
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n; ++r) {
        const int32_t* t = tris + 3 * (int64_t)tri_idx[r];
        woop(verts + 3 * (int64_t)t[0], verts + 3 * (int64_t)t[1], verts + 3 * (int64_t)t[2], woop4 + 12 * r);
    }
}

// Single-triangle BVH: root with the triangle's leaf and an empty leaf.
int64_t or_single(const float* verts, const int32_t* tris, void* nodes_out, int32_t* counts) {
    bin_node* out = reinterpret_cast<bin_node*>(nodes_out);
    float mn[3], mx[3], emn[3] = {MAXF, MAXF, MAXF}, emx[3] = {-MAXF, -MAXF, -MAXF};
    tri_box(verts, tris, 0, mn, mx);
    make_node(out[0], mn, mx, emn, emx, ~1, ~2, 1, -1);
    make_node(out[1], mn, mx, mn, mx, 0, 1, ~1, 0);
    make_node(out[2], emn, emx, emn, emx, 1, 1, ~0, 0);
    counts[0] = 1;
    counts[1] = 2;
    return 3;
}

// ---- whole LBVH build (LBVHBuilder::build, rt/bvh/LBVHBuilder.cpp:183-241) -----------------
// nodes_out: (2n-1 or 3) * 64 bytes; woop4: 12 floats per reference.
int64_t or_build_lbvh(const float* verts, const int32_t* tris, int64_t n64, int bits, float ct, float ci,
                      int adaptive, int max_leaf, const float* scale_in, void* nodes_out, float* woop4,
                      int32_t* tri_idx, int32_t* counts, float* scene_box, float* scale_out) {
    const int n = (int)n64;
    if (n == 0) { counts[0] = counts[1] = 0; return 0; }
    if (n == 1) {
        tri_idx[0] = 0;
        or_woopify(1, verts, tris, tri_idx, woop4);
        float mn[3], mx[3];
        tri_box(verts, tris, 0, mn, mx);
        for (int a = 0; a < 3; ++a) { scene_box[a] = mn[a]; scene_box[3 + a] = mx[a]; }
        return or_single(verts, tris, nodes_out, counts);
    }
    std::vector<float> bmin(4 * (size_t)n), bmax(4 * (size_t)n);
    or_tri_boxes(verts, tris, n, bmin.data(), bmax.data(), scene_box);
    std::vector<uint64_t> keys(n), skeys(n);
    or_morton(n, bmin.data(), bmax.data(), scene_box, scale_in, bits, keys.data(), scale_out);
    or_sort(n, keys.data(), bits, skeys.data(), tri_idx);
    const int nn = 2 * n - 1;
    std::vector<int32_t> parent(nn), left(nn), right(nn), size(nn), state(nn);
    or_karras(n, skeys.data(), parent.data(), left.data(), right.data());
    std::vector<float> nbmin(4 * (size_t)nn), nbmax(4 * (size_t)nn), cost(nn);
    or_refit(n, verts, tris, tri_idx, parent.data(), left.data(), right.data(), ct, ci, adaptive, max_leaf,
             nbmin.data(), nbmax.data(), size.data(), cost.data(), state.data());
    or_woopify(n, verts, tris, tri_idx, woop4);
    return or_collapse(n, parent.data(), left.data(), right.data(), nbmin.data(), nbmax.data(), size.data(),
                       state.data(), nodes_out, counts);
}

// ---- A8: PLOC (PLOCBuilder::clustering, rt/bvh/PLOCBuilder.cpp:21-159) -----------------
// Clusters start as the sorted leaves. Each iteration: every cluster finds its
// nearest neighbour within +-r by the surface area of the union box, scanning
// the left side then the right side and keeping the first strict minimum
// (generateNeighbours(Cached), PLOCBuilderKernels.cu:11-195); mutual pairs merge
// with the lower cluster as the left child into node (count - 2) - k, k the
// number of merges at lower cluster positions (merge, :197-288; the reference
// takes k from warp-level atomics), and the surviving clusters are compacted in
// order (:290-389). The collapse costs of computeNodeStatesAdaptive are
// evaluated when a node is created, since its children are final then.
// Outputs the binary tree over node indices 0..2n-2 (root 0), the per-node box,
// size, cost and state, and the number of iterations.
int or_ploc(int n, const float* verts, const int32_t* tris, const int32_t* sorted_tri, int radius,
            int max_radius, int adaptive_r, float ct, float ci, int adaptive_leaf, int max_leaf,
            int32_t* parent, int32_t* left, int32_t* right, float* bmin4, float* bmax4, int32_t* size,
            float* cost, int32_t* state) {
    const int nn = 2 * n - 1;
    for (int p = 0; p < n; ++p) {
        const int j = n - 1 + p;
        float mn[3], mx[3];
        tri_box(verts, tris, sorted_tri[p], mn, mx);
        for (int a = 0; a < 3; ++a) { bmin4[4 * j + a] = mn[a]; bmax4[4 * j + a] = mx[a]; }
        bmin4[4 * j + 3] = bmax4[4 * j + 3] = 0.0f;
        size[j] = 1;
        cost[j] = adaptive_leaf ? ci * area6(mn[0], mn[1], mn[2], mx[0], mx[1], mx[2]) : 0.0f;
        state[j] = 0;
        left[j] = p;
        right[j] = p + 1;
    }
    if (n >= 1) parent[0] = -1;
    std::vector<int> cl(n), cl2(n), nbr(n);
    for (int p = 0; p < n; ++p) cl[p] = n - 1 + p;
    int count = n, iters = 0, r = radius;
    auto union_area = [&](int a, int b) {
        float mn[3], mx[3];
        for (int k = 0; k < 3; ++k) {
            mn[k] = std::min(bmin4[4 * a + k], bmin4[4 * b + k]);
            mx[k] = std::max(bmax4[4 * a + k], bmax4[4 * b + k]);
        }
        return area6(mn[0], mn[1], mn[2], mx[0], mx[1], mx[2]);
    };
    while (count > 1) {
        ++iters;
        if (adaptive_r) r = std::min(r + 1, max_radius);
#pragma omp parallel for schedule(static)
        for (int i = 0; i < count; ++i) {
            float best = MAXF;
            int bi = -1;
            for (int j = std::max(0, i - r); j < i; ++j) {
                float d = union_area(cl[i], cl[j]);
                if (best > d) { best = d; bi = j; }
            }
            for (int j = i + 1; j < std::min(count, i + r + 1); ++j) {
                float d = union_area(cl[i], cl[j]);
                if (best > d) { best = d; bi = j; }
            }
            nbr[i] = bi;
        }
        const int offset = count - 2;
        int merges = 0, kept = 0;
        for (int i = 0; i < count; ++i) {
            const int j = nbr[i];
            const bool mutual = j >= 0 && nbr[j] == i;
            if (mutual && i < j) {
                const int node = offset - merges++;
                const int a = cl[i], b = cl[j];
                float mn[3], mx[3];
                for (int k = 0; k < 3; ++k) {
                    mn[k] = std::min(bmin4[4 * a + k], bmin4[4 * b + k]);
                    mx[k] = std::max(bmax4[4 * a + k], bmax4[4 * b + k]);
                    bmin4[4 * node + k] = mn[k];
                    bmax4[4 * node + k] = mx[k];
                }
                bmin4[4 * node + 3] = bmax4[4 * node + 3] = 0.0f;
                left[node] = a;
                right[node] = b;
                parent[a] = parent[b] = node;
                size[node] = size[a] + size[b];
                if (adaptive_leaf) {
                    const float A = area6(mn[0], mn[1], mn[2], mx[0], mx[1], mx[2]);
                    const float c_int = std::fmaf(ct, A, cost[a]) + cost[b];
                    const float c_leaf = (ci * A) * (float)size[node];
                    state[node] = (c_leaf < c_int) ? 0 : 1;
                    cost[node] = state[node] ? c_int : c_leaf;
                } else {
                    state[node] = (size[node] <= max_leaf) ? 0 : 1;
                    cost[node] = 0.0f;
                }
                cl2[kept++] = node;
            } else if (!(mutual && j < i)) {
                cl2[kept++] = cl[i];
            }
        }
        count -= merges;
        std::swap(cl, cl2);
    }
    (void)nn;
    return iters;
}

// ---- collapse of a general binary tree (BVHCollapser::collapseAdaptive,
// rt/bvh/BVHCollapser.cpp:521-597) into binary nodes with the canonical
// depth-first order: interior nodes numbered in preorder (root 0, left
// subtree before right), leaves and their triangles in left-to-right order.
// A node is a leaf of the collapsed tree iff it is an original leaf or its
// state is 0, and no proper ancestor below the root is one (the root stays
// interior, as computeLeafIndices never collapses it). Writes nodes, the
// triangle order (tri_idx_out) and the Woop triangles in that order.
int64_t or_collapse_dfs(int n, const float* verts, const int32_t* tris, const int32_t* sorted_tri,
                        const int32_t* left, const int32_t* right, const float* bmin4, const float* bmax4,
                        const int32_t* size, const int32_t* state, void* nodes_out, int32_t* tri_idx_out,
                        float* woop4, int32_t* counts) {
    bin_node* out = reinterpret_cast<bin_node*>(nodes_out);
    if (n < 2) { counts[0] = counts[1] = 0; return 0; }
    auto is_leaf = [&](int v) { return v >= n - 1 || state[v] == 0; };
    // pass 1: preorder numbering of interior nodes and left-to-right leaves
    std::vector<int> iidx(2 * n - 1, -1), lidx(2 * n - 1, -1), toff(2 * n - 1, -1);
    int ni = 0, nl = 0, nt = 0;
    std::vector<int> st{0};
    while (!st.empty()) {
        int v = st.back();
        st.pop_back();
        if (v != 0 && is_leaf(v)) {
            lidx[v] = nl++;
            toff[v] = nt;
            nt += size[v];
            continue;
        }
        iidx[v] = ni++;
        st.push_back(right[v]);
        st.push_back(left[v]);
    }
    // pass 2: triangles of every leaf in left-to-right order of the original leaves
    for (int v = 0; v < 2 * n - 1; ++v) {
        if (lidx[v] < 0) continue;
        int pos = toff[v];
        std::vector<int> s{v};
        while (!s.empty()) {
            int x = s.back();
            s.pop_back();
            if (x >= n - 1) { tri_idx_out[pos++] = sorted_tri[x - (n - 1)]; continue; }
            s.push_back(right[x]);
            s.push_back(left[x]);
        }
    }
    auto box = [&](int v, float* mn, float* mx) {
        for (int a = 0; a < 3; ++a) { mn[a] = bmin4[4 * v + a]; mx[a] = bmax4[4 * v + a]; }
    };
    auto ref_of = [&](int c) { return iidx[c] >= 0 ? iidx[c] : ~(ni + lidx[c]); };
    std::vector<int> par_of(2 * n - 1, -1);
    for (int v = 0; v < 2 * n - 1; ++v)
        if (iidx[v] >= 0) { par_of[left[v]] = iidx[v]; par_of[right[v]] = iidx[v]; }
    for (int v = 0; v < 2 * n - 1; ++v) {
        if (iidx[v] >= 0) {
            float amn[3], amx[3], bmn[3], bmx[3];
            box(left[v], amn, amx);
            box(right[v], bmn, bmx);
            make_node(out[iidx[v]], amn, amx, bmn, bmx, ref_of(left[v]), ref_of(right[v]), size[v],
                      v == 0 ? -1 : par_of[v]);
        } else if (lidx[v] >= 0) {
            float mn[3], mx[3];
            box(v, mn, mx);
            make_node(out[ni + lidx[v]], mn, mx, mn, mx, toff[v], toff[v] + size[v], ~size[v], par_of[v]);
        }
    }
    or_woopify(n, verts, tris, tri_idx_out, woop4);
    counts[0] = ni;
    counts[1] = nl;
    return (int64_t)ni + nl;
}

// Whole PLOC build (PLOCBuilder::build, rt/bvh/PLOCBuilder.cpp:161-208).
int64_t or_build_ploc(const float* verts, const int32_t* tris, int64_t n64, int bits, int radius, int max_radius,
                      int adaptive_r, float ct, float ci, int adaptive, int max_leaf, const float* scale_in,
                      void* nodes_out, float* woop4, int32_t* tri_idx, int32_t* counts, float* scene_box,
                      float* scale_out, int32_t* iterations) {
    const int n = (int)n64;
    if (n < 2)
        return or_build_lbvh(verts, tris, n64, bits, ct, ci, adaptive, max_leaf, scale_in, nodes_out, woop4,
                             tri_idx, counts, scene_box, scale_out);
    std::vector<float> bmin(4 * (size_t)n), bmax(4 * (size_t)n);
    or_tri_boxes(verts, tris, n, bmin.data(), bmax.data(), scene_box);
    std::vector<uint64_t> keys(n), skeys(n);
    or_morton(n, bmin.data(), bmax.data(), scene_box, scale_in, bits, keys.data(), scale_out);
    std::vector<int32_t> sorted(n);
    or_sort(n, keys.data(), bits, skeys.data(), sorted.data());
    const int nn = 2 * n - 1;
    std::vector<int32_t> parent(nn), left(nn), right(nn), size(nn), state(nn);
    std::vector<float> nbmin(4 * (size_t)nn), nbmax(4 * (size_t)nn), cost(nn);
    int it = or_ploc(n, verts, tris, sorted.data(), radius, max_radius, adaptive_r, ct, ci, adaptive, max_leaf,
                     parent.data(), left.data(), right.data(), nbmin.data(), nbmax.data(), size.data(), cost.data(),
                     state.data());
    if (iterations) *iterations = it;
    return or_collapse_dfs(n, verts, tris, sorted.data(), left.data(), right.data(), nbmin.data(), nbmax.data(),
                           size.data(), state.data(), nodes_out, tri_idx, woop4, counts);
}

// ---- A15: ATR, agglomerative treelet restructuring (ATRBuilder::optimize,
// rt/bvh/ATRBuilder.cpp:80-178; kernels optimize / optimizeSmall,
// rt/bvh/ATRBuilderKernels.cu:12-554; formTreelet, rt/bvh/TRBuilderUtil.h:141-216).
//
// Per iteration (gamma = treelet size, doubled after each one) the reference
// climbs from the leaves; at every node reached by its second child it sets
// refs = refs(l) + refs(r), cost = ct*A + cost(l) + cost(r) (leaves: ci*A),
// and a node with refs >= gamma becomes a treelet root right away. Every node
// below a treelet root is final when the root is reached and concurrent
// treelets are disjoint, so a sequential post-order gives the same result.
// A treelet: starting from the root's two children, the treelet leaf with the
// largest area that is not a BVH leaf is expanded until there are T leaves
// (T-1 internal nodes, the root first); the leaves are then merged
// agglomeratively by the area of the union box, the smallest pair first, the
// new cluster taking the column slot and the last slot moving into the row
// slot. The new topology is kept iff its cost is strictly below the old cost.
// Ties in the two searches are broken by the reference's warp reductions,
// simulated here lane by lane. Areas use the formula of the ATR kernels,
// 2*(x*y + x*z + y*z), which the fast-math build contracts to
// 2*fma(y, z, fma(x, y, x*z)).
}  // extern "C"

namespace {

inline float atr_area(const float* mn, const float* mx) {
    const float x = mx[0] - mn[0], y = mx[1] - mn[1], z = mx[2] - mn[2];
    return 2.0f * std::fmaf(y, z, std::fmaf(x, y, x * z));
}

inline int tri_index(int row, int col) { return row * (row - 1) / 2 + col; }

inline void tri_decode(int e, int& row, int& col) {
    int r = (int)((1.0 + std::sqrt(8.0 * e + 1.0)) * 0.5);
    while (r * (r - 1) / 2 > e) --r;
    while ((r + 1) * r / 2 <= e) ++r;
    row = r;
    col = e - r * (r - 1) / 2;
}

struct atr_state {
    int n, T;
    float ct, ci;
    int32_t *parent, *left, *right;
    float *bmin4, *bmax4;
    std::vector<float> cost;
    std::vector<int> refs;
};

// findLeafToExpand (TRBuilderUtil.h:141-153) over `count` lanes: shuffles down
// by count/2, the lower lane keeping its value unless the other is strictly
// larger; repeated on ceil(count/2) lanes until one is left. Returns lane 0's index.
int warp_argmax(const float* a_in, int count) {
    float a[32];
    int idx[32];
    for (int k = 0; k < 32; ++k) { a[k] = k < count ? a_in[k] : -MAXF; idx[k] = k; }
    int cnt = count, sh = cnt / 2;
    while (cnt > 1) {
        float na[32];
        int ni[32];
        for (int k = 0; k < 32; ++k) {
            na[k] = a[k];
            ni[k] = idx[k];
            if (k + sh < 32 && a[k + sh] > a[k]) { na[k] = a[k + sh]; ni[k] = idx[k + sh]; }
        }
        std::memcpy(a, na, sizeof(a));
        std::memcpy(idx, ni, sizeof(idx));
        cnt = (cnt + 1) / 2;
        sh = cnt / 2;
    }
    return idx[0];
}

// findMinimumDistance (ATRBuilderKernels.cu:68-94): lane l scans entries l,
// l+32, ... keeping the first strict minimum; then a 32-lane reduction by
// offsets 16..1 where the lower lane keeps its value unless the other is
// strictly smaller. Returns the entry lane 0 ends with.
int warp_argmin(const float* d, int m) {
    float best[32];
    int bi[32];
    for (int l = 0; l < 32; ++l) {
        best[l] = MAXF;
        bi[l] = 0;
        for (int e = l; e < m; e += 32)
            if (d[e] < best[l]) { best[l] = d[e]; bi[l] = e; }
    }
    for (int off = 16; off > 0; off >>= 1) {
        float nb[32];
        int ni[32];
        for (int l = 0; l < 32; ++l) {
            nb[l] = best[l];
            ni[l] = bi[l];
            if (l + off < 32 && best[l + off] < best[l]) { nb[l] = best[l + off]; ni[l] = bi[l + off]; }
        }
        std::memcpy(best, nb, sizeof(best));
        std::memcpy(bi, ni, sizeof(bi));
    }
    return bi[0];
}

void atr_treelet(atr_state& S, int root) {
    const int T = S.T, n = S.n;
    auto box = [&](int v, float* mn, float* mx) {
        for (int a = 0; a < 3; ++a) { mn[a] = S.bmin4[4 * v + a]; mx[a] = S.bmax4[4 * v + a]; }
    };
    auto node_area = [&](int v) {
        float mn[3], mx[3];
        box(v, mn, mx);
        return atr_area(mn, mx);
    };
    // formTreelet
    std::vector<int> tl(T), ti(T - 1);
    std::vector<float> ta(T);
    tl[0] = S.left[root];
    tl[1] = S.right[root];
    ta[0] = node_area(tl[0]);
    ta[1] = node_area(tl[1]);
    ti[0] = root;
    for (int it = 0; it < T - 2; ++it) {
        const int m = it + 2;
        float a[32];
        for (int k = 0; k < m; ++k) a[k] = tl[k] >= n - 1 ? -MAXF : ta[k];
        const int idx = warp_argmax(a, m);
        const int rep = tl[idx];
        ti[it + 1] = rep;
        tl[idx] = S.left[rep];
        tl[m] = S.right[rep];
        ta[idx] = node_area(tl[idx]);
        ta[m] = node_area(tl[m]);
    }
    // slot state and the distance matrix
    std::vector<int> sn(T), sr(T);
    std::vector<float> sc(T), smn(3 * T), smx(3 * T);
    for (int k = 0; k < T; ++k) {
        sn[k] = tl[k];
        sc[k] = S.cost[tl[k]];
        sr[k] = S.refs[tl[k]];
        box(tl[k], &smn[3 * k], &smx[3 * k]);
    }
    auto union_area = [&](int i, int j) {
        float mn[3], mx[3];
        for (int a = 0; a < 3; ++a) {
            mn[a] = std::min(smn[3 * i + a], smn[3 * j + a]);
            mx[a] = std::max(smx[3 * i + a], smx[3 * j + a]);
        }
        return atr_area(mn, mx);
    };
    std::vector<float> d(T * (T - 1) / 2);
    for (int i = 1; i < T; ++i)
        for (int j = 0; j < i; ++j) d[tri_index(i, j)] = union_area(i, j);
    // outputs: internal node ti[k-1] is created at step k
    std::vector<int> ol(T), orr(T), orf(T);
    std::vector<float> oc(T), omn(3 * T), omx(3 * T);
    for (int last = T - 1; last >= 1; --last) {
        int row, col;
        tri_decode(warp_argmin(d.data(), last * (last + 1) / 2), row, col);
        float umn[3], umx[3];
        for (int a = 0; a < 3; ++a) {
            umn[a] = std::min(smn[3 * row + a], smn[3 * col + a]);
            umx[a] = std::max(smx[3 * row + a], smx[3 * col + a]);
        }
        const float uc = std::fmaf(S.ct, atr_area(umn, umx), sc[row] + sc[col]);
        ol[last] = sn[row];
        orr[last] = sn[col];
        oc[last] = uc;
        orf[last] = sr[row] + sr[col];
        for (int a = 0; a < 3; ++a) { omn[3 * last + a] = umn[a]; omx[3 * last + a] = umx[a]; }
        // the last slot moves into the row slot, the new cluster takes the column slot
        if (row != last) {
            sn[row] = sn[last];
            sc[row] = sc[last];
            sr[row] = sr[last];
            for (int a = 0; a < 3; ++a) { smn[3 * row + a] = smn[3 * last + a]; smx[3 * row + a] = smx[3 * last + a]; }
        }
        sn[col] = ti[last - 1];
        sc[col] = uc;
        sr[col] = orf[last];
        for (int a = 0; a < 3; ++a) { smn[3 * col + a] = umn[a]; smx[3 * col + a] = umx[a]; }
        if (last > 1) {
            for (int t = 0; t < last; ++t)
                if (t != row) d[tri_index(std::max(row, t), std::min(row, t))] = d[tri_index(last, t)];
            for (int t = 0; t < last; ++t)
                if (t != col) d[tri_index(std::max(col, t), std::min(col, t))] = union_area(t, col);
        }
    }
    // updateTreelet (ATRBuilderKernels.cu:197-229)
    if (!(oc[1] < S.cost[root])) return;
    for (int k = 1; k < T; ++k) {
        const int v = ti[k - 1];
        S.left[v] = ol[k];
        S.right[v] = orr[k];
        S.parent[ol[k]] = v;
        S.parent[orr[k]] = v;
        S.cost[v] = oc[k];
        S.refs[v] = orf[k];
        for (int a = 0; a < 3; ++a) { S.bmin4[4 * v + a] = omn[3 * k + a]; S.bmax4[4 * v + a] = omx[3 * k + a]; }
    }
}

}  // namespace

extern "C" {

// Runs the ATR iterations on a refitted LBVH (parent / left / right / boxes over
// 2n-1 nodes, leaves n-1..2n-2) in place. Returns the number of iterations run.
int or_atr(int n, int treelet, int iterations, float ct, float ci, int32_t* parent, int32_t* left,
           int32_t* right, float* bmin4, float* bmax4) {
    if (n < 2 || treelet < 3 || treelet > 32) return 0;
    atr_state S;
    S.n = n; S.T = treelet; S.ct = ct; S.ci = ci;
    S.parent = parent; S.left = left; S.right = right; S.bmin4 = bmin4; S.bmax4 = bmax4;
    S.cost.assign(2 * n - 1, 0.0f);
    S.refs.assign(2 * n - 1, 0);
    for (int p = 0; p < n; ++p) {
        const int j = n - 1 + p;
        S.cost[j] = ci * atr_area(&bmin4[4 * j], &bmax4[4 * j]);
        S.refs[j] = 1;
    }
    int gamma = treelet, done = 0;
    for (int i = 0; i < iterations; ++i) {
        ++done;
        std::vector<std::pair<int, bool>> st{{0, false}};
        while (!st.empty()) {
            auto [v, expanded] = st.back();
            if (v >= n - 1) { st.pop_back(); continue; }
            if (!expanded) {
                st.back().second = true;
                st.push_back({right[v], false});
                st.push_back({left[v], false});
                continue;
            }
            st.pop_back();
            const int l = left[v], r = right[v];
            for (int a = 0; a < 3; ++a) {
                bmin4[4 * v + a] = std::min(bmin4[4 * l + a], bmin4[4 * r + a]);
                bmax4[4 * v + a] = std::max(bmax4[4 * l + a], bmax4[4 * r + a]);
            }
            S.refs[v] = S.refs[l] + S.refs[r];
            S.cost[v] = std::fmaf(ct, atr_area(&bmin4[4 * v], &bmax4[4 * v]), S.cost[l]) + S.cost[r];
            if (S.refs[v] >= gamma) atr_treelet(S, v);
        }
        gamma *= 2;
        if (gamma > n) break;
    }
    return done;
}

// ---- TRBVH: treelet restructuring by dynamic programming over subsets
// (TRBuilder::optimize, rt/bvh/TRBuilder.cpp:137-205; kernel optimize with
// calculateSubsetSurfaceAreas, processSchedule, processSubsets, updateTreelet,
// rt/bvh/TRBuilderKernels.cu:12-470; formTreelet, TRBuilderUtil.h:141-216).
//
// The climb is ATR's (refs, cost = ct*A + cost(l) + cost(r), leaves ci*A; a
// node with refs >= gamma is a treelet root, gamma = 7 doubled per
// iteration). A treelet has T = 7 leaves formed as in ATR. Every subset s of
// them gets the box of its leaves and A(s); singletons cost their node's cost;
// then, by increasing size, cost(s) = min(ct*A(s) + best split, ci*A(s)*R)
// with R the treelet root's reference count, the best split over partitions
// (p, s^p) in the kernel's enumeration order, first strict minimum kept:
//   * sizes 2..T-2: p runs over (−delta)&s, then (p − delta)&s, delta =
//     (s−1)&s;
//   * size T-1 (bit k cleared): four lanes q take bases q+1, q+5, ..., each
//     mapped to ((b & m) << 1 | (b & ~m)) << 1, m = −(1 << max(k−1, 0)); the
//     lanes' minima are reduced q0:q2, q1:q3, then the two winners;
//   * the full set: lane l takes p = 2(l+1) and p + 64 (while below 127), the
//     32 minima reduced by shuffle-down halving, the lower lane winning ties.
// If cost(full) < the root's cost, the treelet is rebuilt top-down from the
// splits: internal nodes are reused in the order the rounds hand them out
// (all left children of a round, then all right children), each takes its
// subset's box, and its cost becomes cost(split) — for a right child as well:
// the kernel stores costs[partition], not costs[partition ^ subset], and that
// value feeds later treelets, so it is kept. The root keeps its cost.
namespace {

void tr_treelet(atr_state& S, int root) {
    const int T = 7, n = S.n, FULL = (1 << T) - 1;
    auto box = [&](int v, float* mn, float* mx) {
        for (int a = 0; a < 3; ++a) { mn[a] = S.bmin4[4 * v + a]; mx[a] = S.bmax4[4 * v + a]; }
    };
    auto node_area = [&](int v) {
        float mn[3], mx[3];
        box(v, mn, mx);
        return atr_area(mn, mx);
    };
    // formTreelet
    int tl[T], ti[T - 1];
    float ta[T];
    tl[0] = S.left[root];
    tl[1] = S.right[root];
    ta[0] = node_area(tl[0]);
    ta[1] = node_area(tl[1]);
    ti[0] = root;
    for (int it = 0; it < T - 2; ++it) {
        const int m = it + 2;
        float a[32];
        for (int k = 0; k < m; ++k) a[k] = tl[k] >= n - 1 ? -MAXF : ta[k];
        const int idx = warp_argmax(a, m);
        const int rep = tl[idx];
        ti[it + 1] = rep;
        tl[idx] = S.left[rep];
        tl[m] = S.right[rep];
        ta[idx] = node_area(tl[idx]);
        ta[m] = node_area(tl[m]);
    }
    // subset boxes and areas
    float smn[128][3], smx[128][3], cost[128];
    int mask[128];
    for (int s = 0; s <= FULL; ++s) {
        for (int a = 0; a < 3; ++a) { smn[s][a] = MAXF; smx[s][a] = -MAXF; }
        for (int i = 0; i < T; ++i)
            if (s & (1 << i)) {
                float mn[3], mx[3];
                box(tl[i], mn, mx);
                for (int a = 0; a < 3; ++a) {
                    smn[s][a] = std::min(smn[s][a], mn[a]);
                    smx[s][a] = std::max(smx[s][a], mx[a]);
                }
            }
        cost[s] = atr_area(smn[s], smx[s]);
        mask[s] = 0;
    }
    float area[128];
    std::memcpy(area, cost, sizeof(area));
    for (int i = 0; i < T; ++i) cost[1 << i] = S.cost[tl[i]];
    const float refs = (float)S.refs[root];
    auto finish = [&](int s, float opt, int p) {
        cost[s] = std::min(std::fmaf(S.ct, area[s], opt), (S.ci * area[s]) * refs);
        mask[s] = p;
    };
    // sizes 2 .. T-2
    for (int size = 2; size <= T - 2; ++size)
        for (int s = 1; s < FULL; ++s) {
            if (__builtin_popcount(s) != size) continue;
            float opt = MAXF;
            int optp = 0;
            const int delta = (s - 1) & s;
            int p = (-delta) & s;
            while (p != 0) {
                const float c = cost[p] + cost[p ^ s];
                if (c < opt) { opt = c; optp = p; }
                p = (p - delta) & s;
            }
            finish(s, opt, optp);
        }
    // size T-1
    for (int k = 0; k < T; ++k) {
        const int s = FULL & ~(1 << k);
        const int lm = -(1 << std::max(k - 1, 0));
        const int np = (1 << (T - 2)) - 1;
        float qo[4];
        int qp[4];
        for (int q = 0; q < 4; ++q) {
            int base = q + 1;
            float opt = MAXF;
            int optp = 0;
            int p = (((base & lm) << 1) | (base & ~lm)) << 1;
            for (int j = q; j < np; j += 4) {
                const float c = cost[p] + cost[p ^ s];
                if (c < opt) { opt = c; optp = p; }
                base += 4;
                p = (((base & lm) << 1) | (base & ~lm)) << 1;
            }
            qo[q] = opt;
            qp[q] = optp;
        }
        for (int q = 0; q < 2; ++q)
            if (qo[q + 2] < qo[q]) { qo[q] = qo[q + 2]; qp[q] = qp[q + 2]; }
        if (qo[1] < qo[0]) { qo[0] = qo[1]; qp[0] = qp[1]; }
        finish(s, qo[0], qp[0]);
    }
    // the full set
    {
        float lo[32];
        int lp[32];
        const int np = (1 << (T - 1)) - 1;
        for (int l = 0; l < 32; ++l) {
            float opt = MAXF;
            int optp = 0;
            int p = (l + 1) * 2;
            for (int j = l; j < np; j += 32) {
                const float c = cost[p] + cost[p ^ FULL];
                if (c < opt) { opt = c; optp = p; }
                p += 64;
            }
            lo[l] = opt;
            lp[l] = optp;
        }
        for (int off = 16; off > 0; off >>= 1)
            for (int l = 0; l < 32; ++l)
                if (l + off < 32 && lo[l + off] < lo[l]) { lo[l] = lo[l + off]; lp[l] = lp[l + off]; }
        finish(FULL, lo[0], lp[0]);
    }
    // updateTreelet
    if (!(cost[FULL] < S.cost[root])) return;
    std::vector<std::pair<int, int>> round{{root, FULL}};
    int next = 1;
    auto leaf_refs = [&](int s) {
        int r = 0;
        for (int i = 0; i < T; ++i)
            if (s & (1 << i)) r += S.refs[tl[i]];
        return r;
    };
    auto place = [&](int node, int s, int from, bool left_side, std::vector<std::pair<int, int>>& out) {
        int child;
        if (__builtin_popcount(s) > 1) {
            child = ti[next++];
            for (int a = 0; a < 3; ++a) { S.bmin4[4 * child + a] = smn[s][a]; S.bmax4[4 * child + a] = smx[s][a]; }
            S.cost[child] = cost[from];
            S.refs[child] = leaf_refs(s);
            out.push_back({child, s});
        } else {
            child = tl[__builtin_ctz(s)];
        }
        (left_side ? S.left : S.right)[node] = child;
        S.parent[child] = node;
    };
    while (!round.empty()) {
        std::vector<std::pair<int, int>> out;
        for (auto [node, s] : round) place(node, mask[s], mask[s], true, out);
        for (auto [node, s] : round) place(node, mask[s] ^ s, mask[s], false, out);
        round.swap(out);
    }
}

}  // namespace

extern "C" {

// TRBVH iterations (treelet 7) on a refitted LBVH in place; returns the count run.
int or_tr(int n, int iterations, float ct, float ci, int32_t* parent, int32_t* left, int32_t* right, float* bmin4,
          float* bmax4) {
    const int T = 7;
    if (n < 2) return 0;
    atr_state S;
    S.n = n; S.T = T; S.ct = ct; S.ci = ci;
    S.parent = parent; S.left = left; S.right = right; S.bmin4 = bmin4; S.bmax4 = bmax4;
    S.cost.assign(2 * n - 1, 0.0f);
    S.refs.assign(2 * n - 1, 0);
    for (int p = 0; p < n; ++p) {
        const int j = n - 1 + p;
        S.cost[j] = ci * atr_area(&bmin4[4 * j], &bmax4[4 * j]);
        S.refs[j] = 1;
    }
    int gamma = T, done = 0;
    for (int i = 0; i < iterations; ++i) {
        ++done;
        std::vector<std::pair<int, bool>> st{{0, false}};
        while (!st.empty()) {
            auto [v, expanded] = st.back();
            if (v >= n - 1) { st.pop_back(); continue; }
            if (!expanded) {
                st.back().second = true;
                st.push_back({right[v], false});
                st.push_back({left[v], false});
                continue;
            }
            st.pop_back();
            const int l = left[v], r = right[v];
            for (int a = 0; a < 3; ++a) {
                bmin4[4 * v + a] = std::min(bmin4[4 * l + a], bmin4[4 * r + a]);
                bmax4[4 * v + a] = std::max(bmax4[4 * l + a], bmax4[4 * r + a]);
            }
            S.refs[v] = S.refs[l] + S.refs[r];
            S.cost[v] = std::fmaf(ct, atr_area(&bmin4[4 * v], &bmax4[4 * v]), S.cost[l]) + S.cost[r];
            if (S.refs[v] >= gamma) tr_treelet(S, v);
        }
        gamma *= 2;
        if (gamma > n) break;
    }
    return done;
}

}  // extern "C"

// Whole ATR build (ATRBuilder::build, rt/bvh/ATRBuilder.cpp:180-236): the LBVH
// stages, the ATR iterations, then the collapse of the restructured tree.
int64_t or_build_atr(const float* verts, const int32_t* tris, int64_t n64, int bits, int treelet, int iterations,
                     float ct, float ci, int adaptive, int max_leaf, const float* scale_in, void* nodes_out,
                     float* woop4, int32_t* tri_idx, int32_t* counts, float* scene_box, float* scale_out) {
    const int n = (int)n64;
    if (n < 2)
        return or_build_lbvh(verts, tris, n64, bits, ct, ci, adaptive, max_leaf, scale_in, nodes_out, woop4,
                             tri_idx, counts, scene_box, scale_out);
    std::vector<float> bmin(4 * (size_t)n), bmax(4 * (size_t)n);
    or_tri_boxes(verts, tris, n, bmin.data(), bmax.data(), scene_box);
    std::vector<uint64_t> keys(n), skeys(n);
    or_morton(n, bmin.data(), bmax.data(), scene_box, scale_in, bits, keys.data(), scale_out);
    std::vector<int32_t> sorted(n);
    or_sort(n, keys.data(), bits, skeys.data(), sorted.data());
    const int nn = 2 * n - 1;
    std::vector<int32_t> parent(nn), left(nn), right(nn), size(nn), state(nn);
    or_karras(n, skeys.data(), parent.data(), left.data(), right.data());
    std::vector<float> nbmin(4 * (size_t)nn), nbmax(4 * (size_t)nn), cost(nn);
    or_refit(n, verts, tris, sorted.data(), parent.data(), left.data(), right.data(), ct, ci, adaptive, max_leaf,
             nbmin.data(), nbmax.data(), size.data(), cost.data(), state.data());
    or_atr(n, treelet, iterations, ct, ci, parent.data(), left.data(), right.data(), nbmin.data(), nbmax.data());
    or_refit(n, verts, tris, sorted.data(), parent.data(), left.data(), right.data(), ct, ci, adaptive, max_leaf,
             nbmin.data(), nbmax.data(), size.data(), cost.data(), state.data());
    return or_collapse_dfs(n, verts, tris, sorted.data(), left.data(), right.data(), nbmin.data(), nbmax.data(),
                           size.data(), state.data(), nodes_out, tri_idx, woop4, counts);
}

// ---- HLBVH: LBVH clusters below the top Morton bits, binned SAH above them
// (HLBVHBuilder::build, rt/bvh/HLBVHBuilder.cpp:330-395; kernels
// computeNodeStates, computeLeafClusterIndices, computeClusters, binClusters,
// split, distributeClusters, rt/bvh/HLBVHBuilderKernels.cu:35-704).
//
// An interior LBVH node whose split prefix delta(g, g+1) is at least
// 64 - bits + sahBits lies inside a cluster (state 0; leaves too); the clusters
// are the highest state-0 nodes below the root. Each cluster is binned by the
// (x, y, z) coordinates of its top sahBits Morton bits (2^(sahBits/3) bins
// per axis). The top tree is built top-down over the clusters: per task and
// axis the bins are swept from the left against suffix unions from the
// right; a split needs clusters on both sides and costs
// count_l * A_l + count_r * A_r (the kernel's fused form
// fma(count_l, A_l, count_r * A_r), A = 2 * fma(y, z, fma(x, y, x * z))), the
// first strictly lowest cost over (axis, bin) wins, clusters at or below the
// split bin go left; a side with one cluster takes the cluster's subtree. With
// sahBits a multiple of 3 every cluster has its own cell except a leaf
// cluster at the last sorted position, which the kernel bins with key 0's
// cell (below); that leaf and the cluster holding position 0 are never
// separated by a bin split and end as the two clusters of the kernel's
// object-median fallback. The new top nodes reuse the indices of the LBVH's
// state-1 nodes in increasing order (the root stays 0). When the root itself
// lies inside a cluster (every key shares the top sahBits) the LBVH is kept.
// Bin boxes are float min / max; the kernel's integer atomics on float bits
// agree with them for non-negative coordinates (the reference's scene loader
// scales scenes into [0, 1]^3, rt/scene/SceneLoader.cpp:136-140), not for
// negative ones.
namespace {

inline void morton_coords(uint32_t code, int* c) {
    c[0] = c[1] = c[2] = 0;
    for (int i = 0; i < 10; ++i) {
        c[0] += ((code >> (3 * i + 0)) & 1) << i;
        c[1] += ((code >> (3 * i + 1)) & 1) << i;
        c[2] += ((code >> (3 * i + 2)) & 1) << i;
    }
}

}  // namespace

extern "C" {

// HLBVH top-level rebuild in place on a Karras LBVH (parent / left / right /
// refitted boxes over 2n-1 nodes) with its sorted keys. Returns the number of
// clusters, or -1 for an unsupported sahBits.
int or_hlbvh(int n, const uint64_t* skeys, int bits, int sah_bits, int32_t* parent, int32_t* left, int32_t* right,
             float* bmin4, float* bmax4) {
    if (sah_bits % 3 != 0 || sah_bits < 6 || sah_bits > 15 || sah_bits > bits) return -1;
    if (n < 2) return 0;
    const int nn = 2 * n - 1, off = 64 - bits + sah_bits, NB = 1 << (sah_bits / 3);
    std::vector<int> state(nn, 0), gamma(n - 1, 0), last(nn, 0);
    // split position of each interior node: the last sorted position of its left child
    for (int p = 0; p < n; ++p) last[n - 1 + p] = p;
    {
        std::vector<int> st{0};
        std::vector<char> ex(nn, 0);
        while (!st.empty()) {
            const int v = st.back();
            if (v >= n - 1) { st.pop_back(); continue; }
            if (!ex[v]) { ex[v] = 1; st.push_back(right[v]); st.push_back(left[v]); continue; }
            st.pop_back();
            last[v] = last[right[v]];
            gamma[v] = last[left[v]];
        }
    }
    for (int v = 0; v < n - 1; ++v) state[v] = delta(skeys, n, gamma[v], gamma[v] + 1) >= off ? 0 : 1;
    // clusters, in order of their first sorted position
    std::vector<int> clusters;
    {
        std::vector<int> st{0};
        while (!st.empty()) {
            const int v = st.back();
            st.pop_back();
            if (v != 0 && state[v] == 0) { clusters.push_back(v); continue; }
            st.push_back(right[v]);
            st.push_back(left[v]);
        }
    }
    const int C = (int)clusters.size();
    std::vector<int> free_idx;  // state-1 interior nodes, root first
    for (int v = 0; v < n - 1; ++v)
        if (state[v] == 1) free_idx.push_back(v);
    if (C < 2 || free_idx.empty() || free_idx[0] != 0) return C;
    // computeClusters reads the key at the node's left index with leaf indices
    // mapped by subtracting n-1; a leaf's left index is its sorted position, so
    // the leaf at the last position n-1 reads key 0 (rt/bvh/HLBVHBuilderKernels.cu:
    // 325-327 with setupLeaves, rt/bvh/LBVHBuilderKernels.cu:186).
    std::vector<std::array<int, 3>> coord(C);
    for (int c = 0; c < C; ++c) {
        const int v = clusters[c];
        int pos = v >= n - 1 ? v - (n - 1) : gamma[v];
        if (v == 2 * n - 2) pos = 0;
        morton_coords((uint32_t)((skeys[pos] >> (bits - sah_bits)) & ((1u << sah_bits) - 1)), coord[c].data());
    }
    struct bin {
        float mn[3], mx[3];
        int cnt;
        void reset() { for (int a = 0; a < 3; ++a) { mn[a] = MAXF; mx[a] = -MAXF; } cnt = 0; }
        void add(const float* bmn, const float* bmx, int k) {
            for (int a = 0; a < 3; ++a) { mn[a] = std::min(mn[a], bmn[a]); mx[a] = std::max(mx[a], bmx[a]); }
            cnt += k;
        }
        float cost() const {
            return (float)cnt * atr_area(mn, mx);  // only the product; the sum below is fused
        }
    };
    auto area = [](const bin& b) { return atr_area(b.mn, b.mx); };
    // tasks: (node to write, parent), each with its clusters (in cluster order)
    std::vector<int> task_node{0}, task_parent{-1};
    std::vector<int> task_of(C, 0);
    size_t next_free = 1;
    std::vector<int> node_of_task(1, 0);
    while (!task_node.empty()) {
        const int T = (int)task_node.size();
        std::vector<bin> bins((size_t)T * 3 * NB);
        for (auto& b : bins) b.reset();
        for (int c = 0; c < C; ++c) {
            const int t = task_of[c];
            if (t < 0) continue;
            const int v = clusters[c];
            for (int a = 0; a < 3; ++a) bins[((size_t)t * 3 + a) * NB + coord[c][a]].add(&bmin4[4 * v], &bmax4[4 * v], 1);
        }
        std::vector<int> new_node, new_parent;
        std::vector<int> best_axis(T, -1), best_bin(T, -1), left_task(T, -1), right_task(T, -1);
        std::vector<int> left_cnt(T, 0), right_cnt(T, 0), total(T, 0), rank(T, 0);
        for (int c = 0; c < C; ++c)
            if (task_of[c] >= 0) ++total[task_of[c]];
        for (int t = 0; t < T; ++t) {
            float best = MAXF;
            bin bl{}, br{};
            for (int a = 0; a < 3; ++a) {
                const bin* B = &bins[((size_t)t * 3 + a) * NB];
                std::vector<bin> suffix(NB);
                suffix[NB - 1] = B[NB - 1];
                for (int b = NB - 2; b >= 0; --b) {
                    suffix[b] = suffix[b + 1];
                    suffix[b].add(B[b].mn, B[b].mx, B[b].cnt);
                }
                bin lft = B[0];
                for (int b = 0; b < NB - 1; ++b) {
                    if (lft.cnt > 0 && suffix[b + 1].cnt > 0) {
                        const float cost = std::fmaf((float)lft.cnt, area(lft), (float)suffix[b + 1].cnt * area(suffix[b + 1]));
                        if (cost < best) {
                            best = cost;
                            best_axis[t] = a;
                            best_bin[t] = b;
                            bl = lft;
                            br = suffix[b + 1];
                        }
                    }
                    lft.add(B[b + 1].mn, B[b + 1].mx, B[b + 1].cnt);
                }
            }
            if (best_axis[t] < 0) {
                // Every cluster in one bin (only the leaf above and the cluster of
                // key 0 share a cell): an object median, the first half of the
                // clusters left. The kernel orders them by atomic arrival; here
                // they go in sorted order.
                best_axis[t] = 3;
                best_bin[t] = total[t] / 2;
                bl.reset();
                br.reset();
                int k = 0;
                for (int c = 0; c < C; ++c) {
                    if (task_of[c] != t) continue;
                    const int v = clusters[c];
                    (k++ < best_bin[t] ? bl : br).add(&bmin4[4 * v], &bmax4[4 * v], 1);
                }
            }
            const int node = task_node[t];
            for (int a = 0; a < 3; ++a) {
                bmin4[4 * node + a] = std::min(bl.mn[a], br.mn[a]);
                bmax4[4 * node + a] = std::max(bl.mx[a], br.mx[a]);
            }
            parent[node] = task_parent[t];
            left_cnt[t] = bl.cnt;
            right_cnt[t] = br.cnt;
            // interior children take the next free indices, left then right
            if (bl.cnt > 1) {
                left_task[t] = (int)new_node.size();
                new_node.push_back(free_idx[next_free++]);
                new_parent.push_back(node);
                left[node] = new_node.back();
            }
            if (br.cnt > 1) {
                right_task[t] = (int)new_node.size();
                new_node.push_back(free_idx[next_free++]);
                new_parent.push_back(node);
                right[node] = new_node.back();
            }
        }
        // distribute the clusters; a single cluster becomes its side's child
        for (int c = 0; c < C; ++c) {
            const int t = task_of[c];
            if (t < 0) continue;
            const bool go_left =
                best_axis[t] == 3 ? rank[t]++ < best_bin[t] : coord[c][best_axis[t]] <= best_bin[t];
            const int nt = go_left ? left_task[t] : right_task[t];
            if (nt >= 0) {
                task_of[c] = nt;
            } else {
                const int node = task_node[t], v = clusters[c];
                (go_left ? left : right)[node] = v;
                parent[v] = node;
                task_of[c] = -1;
            }
        }
        task_node.swap(new_node);
        task_parent.swap(new_parent);
    }
    return C;
}

// Whole HLBVH build: the LBVH stages, the top-level rebuild, then the collapse.
int64_t or_build_hlbvh(const float* verts, const int32_t* tris, int64_t n64, int bits, int sah_bits, float ct, float ci,
                       int adaptive, int max_leaf, const float* scale_in, void* nodes_out, float* woop4,
                       int32_t* tri_idx, int32_t* counts, float* scene_box, float* scale_out) {
    const int n = (int)n64;
    if (n < 2)
        return or_build_lbvh(verts, tris, n64, bits, ct, ci, adaptive, max_leaf, scale_in, nodes_out, woop4,
                             tri_idx, counts, scene_box, scale_out);
    std::vector<float> bmin(4 * (size_t)n), bmax(4 * (size_t)n);
    or_tri_boxes(verts, tris, n, bmin.data(), bmax.data(), scene_box);
    std::vector<uint64_t> keys(n), skeys(n);
    or_morton(n, bmin.data(), bmax.data(), scene_box, scale_in, bits, keys.data(), scale_out);
    std::vector<int32_t> sorted(n);
    or_sort(n, keys.data(), bits, skeys.data(), sorted.data());
    const int nn = 2 * n - 1;
    std::vector<int32_t> parent(nn), left(nn), right(nn), size(nn), state(nn);
    or_karras(n, skeys.data(), parent.data(), left.data(), right.data());
    std::vector<float> nbmin(4 * (size_t)nn), nbmax(4 * (size_t)nn), cost(nn);
    or_refit(n, verts, tris, sorted.data(), parent.data(), left.data(), right.data(), ct, ci, adaptive, max_leaf,
             nbmin.data(), nbmax.data(), size.data(), cost.data(), state.data());
    if (or_hlbvh(n, skeys.data(), bits, sah_bits, parent.data(), left.data(), right.data(), nbmin.data(),
                 nbmax.data()) < 0) {
        counts[0] = counts[1] = 0;
        return -1;
    }
    or_refit(n, verts, tris, sorted.data(), parent.data(), left.data(), right.data(), ct, ci, adaptive, max_leaf,
             nbmin.data(), nbmax.data(), size.data(), cost.data(), state.data());
    return or_collapse_dfs(n, verts, tris, sorted.data(), left.data(), right.data(), nbmin.data(), nbmax.data(),
                           size.data(), state.data(), nodes_out, tri_idx, woop4, counts);
}

}  // extern "C"

// Whole TRBVH build (TRBuilder::build, rt/bvh/TRBuilder.cpp:207-260): the LBVH
// stages, the TR iterations, then the collapse of the restructured tree.
int64_t or_build_tr(const float* verts, const int32_t* tris, int64_t n64, int bits, int iterations, float ct,
                    float ci, int adaptive, int max_leaf, const float* scale_in, void* nodes_out, float* woop4,
                    int32_t* tri_idx, int32_t* counts, float* scene_box, float* scale_out) {
    const int n = (int)n64;
    if (n < 2)
        return or_build_lbvh(verts, tris, n64, bits, ct, ci, adaptive, max_leaf, scale_in, nodes_out, woop4,
                             tri_idx, counts, scene_box, scale_out);
    std::vector<float> bmin(4 * (size_t)n), bmax(4 * (size_t)n);
    or_tri_boxes(verts, tris, n, bmin.data(), bmax.data(), scene_box);
    std::vector<uint64_t> keys(n), skeys(n);
    or_morton(n, bmin.data(), bmax.data(), scene_box, scale_in, bits, keys.data(), scale_out);
    std::vector<int32_t> sorted(n);
    or_sort(n, keys.data(), bits, skeys.data(), sorted.data());
    const int nn = 2 * n - 1;
    std::vector<int32_t> parent(nn), left(nn), right(nn), size(nn), state(nn);
    or_karras(n, skeys.data(), parent.data(), left.data(), right.data());
    std::vector<float> nbmin(4 * (size_t)nn), nbmax(4 * (size_t)nn), cost(nn);
    or_refit(n, verts, tris, sorted.data(), parent.data(), left.data(), right.data(), ct, ci, adaptive, max_leaf,
             nbmin.data(), nbmax.data(), size.data(), cost.data(), state.data());
    or_tr(n, iterations, ct, ci, parent.data(), left.data(), right.data(), nbmin.data(), nbmax.data());
    or_refit(n, verts, tris, sorted.data(), parent.data(), left.data(), right.data(), ct, ci, adaptive, max_leaf,
             nbmin.data(), nbmax.data(), size.data(), cost.data(), state.data());
    return or_collapse_dfs(n, verts, tris, sorted.data(), left.data(), right.data(), nbmin.data(), nbmax.data(),
                           size.data(), state.data(), nodes_out, tri_idx, woop4, counts);
}

// ---- wide layouts (Quad / Oct) ------------------------------------------------------
// BVHCollapser::collapseAdaptive / collapse for layouts other than Bin
// (rt/bvh/BVHCollapser.cpp:521-660): the binary tree becomes a host BVH whose
// references are renumbered in left-first depth-first order (convert,
// :339-413; writeTriangleIndices, :497-519), BVH::collapseAdaptiveWide(N) /
// collapseWide(N, maxLeafSize) (rt/bvh/BVH.h:94-160, 228-292, 401-423) turns
// it into an N-wide tree, and BVHConverter::convert (rt/bvh/BVHConverter.cpp:
// 13-89) numbers it breadth first (interior nodes from 0, leaves after them).
//
// Cost model per binary node v and child budget j = 1..N-1 (recomputeCostsWide):
//   leaf(v)    = ci * A(v) / A(root) * ceil(size/N) * N   (MAX_FLOAT if size > maxLeaf)
//   cost[0]    = min(leaf(v), ct * A(v) / A(root) + min_k cost_l[k-1] + cost_r[N-k-1])
//   cost[j-1]  = min(cost[j-2], min_k cost_l[k-1] + cost_r[j-k-1])        j >= 2
// with the first minimum kept on ties and counts (k, j-k) or (-1, -1) for a
// leaf. A = AABB::area, 2 * (dx*dy + dy*dz + dz*dx), evaluated as written.
// collapseWide: a node with budget k starts from its two children with the
// counts of count[k-1]; while it has fewer than N children, the first child
// whose counts (l, r) are both positive with l + r < N is replaced by its
// two children; children whose counts are (-1, -1) become leaves.
// One deviation: when the root's best choice is a leaf (small meshes), the
// reference reads count[-2] of the root's children (undefined); here the root
// then takes its best interior split.
namespace {

inline float host_area(const float* mn, const float* mx) {
    if (!(mn[0] <= mx[0] && mn[1] <= mx[1] && mn[2] <= mx[2])) return 0.0f;
    const float dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
    return 2.0f * (dx * dy + dy * dz + dz * dx);
}

struct wide_dp {
    std::vector<float> cost;   // [nn][N-1]
    std::vector<int8_t> cl, cr; // counts, -1 for a leaf
    std::vector<int8_t> bl, br; // best interior split of budget 1 (root fallback)
};

}  // namespace

extern "C" {

// nodes_out: count * 8 * width int32; tri_idx_out: n. Returns the node count.
int64_t or_collapse_wide(int n, const int32_t* sorted_tri, const int32_t* left, const int32_t* right,
                         const float* bmin4, const float* bmax4, int width, float ct, float ci, int max_leaf,
                         int32_t* nodes_out, int32_t* tri_idx_out, int32_t* counts) {
    const int N = width, W = 8 * width;
    counts[0] = counts[1] = 0;
    if (n < 1 || (N != 4 && N != 8)) return 0;
    auto box = [&](int v, float* mn, float* mx) {
        for (int a = 0; a < 3; ++a) { mn[a] = bmin4[4 * v + a]; mx[a] = bmax4[4 * v + a]; }
    };
    auto put_box = [&](int32_t* nd, int i, const float* mn, const float* mx) {
        std::memcpy(&nd[4 * i + 0], &mn[0], 4); std::memcpy(&nd[4 * i + 1], &mx[0], 4);
        std::memcpy(&nd[4 * i + 2], &mn[1], 4); std::memcpy(&nd[4 * i + 3], &mx[1], 4);
        std::memcpy(&nd[4 * (N + i) + 0], &mn[2], 4); std::memcpy(&nd[4 * (N + i) + 1], &mx[2], 4);
    };
    if (n == 1) {  // root with the single triangle's leaf
        tri_idx_out[0] = sorted_tri[0];
        float mn[3], mx[3];
        box(0, mn, mx);
        int32_t* root = nodes_out;
        int32_t* leaf = nodes_out + W;
        std::memset(root, 0, 2 * W * 4);
        const float dmx[3] = {mn[0], mn[1], mn[2]};
        for (int i = 0; i < N; ++i) {
            put_box(root, i, mn, i == 0 ? mx : dmx);
            root[4 * (N + i) + 2] = i == 0 ? ~1 : 1;  // unused slots: child 0's decoded index
            put_box(leaf, i, mn, mx);
        }
        root[8 * N - 9] = 1; root[8 * N - 5] = 1; root[8 * N - 1] = -1;
        leaf[4 * N + 2] = 0; leaf[4 * N + 3] = 1; leaf[8 * N - 9] = 0; leaf[8 * N - 5] = ~1; leaf[8 * N - 1] = 0;
        counts[0] = 1; counts[1] = 1;
        return 2;
    }
    const int nn = 2 * n - 1;
    // depth-first (left first) reference order: begin/end of every node
    std::vector<int> beg(nn), end(nn), order;
    order.reserve(nn);
    {
        int pos = 0;
        std::vector<int> st{0};
        while (!st.empty()) {
            int v = st.back();
            st.pop_back();
            order.push_back(v);  // preorder
            if (v >= n - 1) { tri_idx_out[pos] = sorted_tri[v - (n - 1)]; beg[v] = pos; end[v] = ++pos; continue; }
            st.push_back(right[v]);
            st.push_back(left[v]);
        }
        for (int k = nn - 1; k >= 0; --k) {
            const int v = order[k];
            if (v < n - 1) { beg[v] = beg[left[v]]; end[v] = end[right[v]]; }
        }
    }
    // recomputeCostsWide, children before parents (reverse preorder)
    const int J = N - 1;
    wide_dp D;
    D.cost.assign((size_t)nn * J, 0.0f);
    D.cl.assign((size_t)nn * J, -1); D.cr.assign((size_t)nn * J, -1);
    D.bl.assign(nn, -1); D.br.assign(nn, -1);
    float rmn[3], rmx[3];
    box(0, rmn, rmx);
    const float root_area = host_area(rmn, rmx);
    for (int k = nn - 1; k >= 0; --k) {
        const int v = order[k];
        float mn[3], mx[3];
        box(v, mn, mx);
        const float A = host_area(mn, mx);
        const int size = end[v] - beg[v];
        float* c = &D.cost[(size_t)v * J];
        int8_t* xl = &D.cl[(size_t)v * J];
        int8_t* xr = &D.cr[(size_t)v * J];
        if (v >= n - 1) {
            for (int j = 1; j < N; ++j) {
                c[j - 1] = ci * A / root_area * (float)((size + N - 1) / N) * (float)N;
                xl[j - 1] = xr[j - 1] = -1;
            }
            continue;
        }
        const float* c0 = &D.cost[(size_t)left[v] * J];
        const float* c1 = &D.cost[(size_t)right[v] * J];
        const float leaf_cost = size > max_leaf ? MAXF : ci * A / root_area * (float)((size + N - 1) / N) * (float)N;
        float sub = ct * A / root_area;
        float dist = MAXF;
        int bk = 0;
        for (int kk = 1; kk < N; ++kk) {
            const float cc = c0[kk - 1] + c1[N - kk - 1];
            if (dist > cc) { dist = cc; bk = kk; }
        }
        sub += dist;
        D.bl[v] = (int8_t)bk;
        D.br[v] = (int8_t)(N - bk);
        if (leaf_cost > sub) { c[0] = sub; xl[0] = (int8_t)bk; xr[0] = (int8_t)(N - bk); }
        else { c[0] = leaf_cost; xl[0] = xr[0] = -1; }
        for (int j = 2; j < N; ++j) {
            dist = MAXF;
            for (int kk = 1; kk < j; ++kk) {
                const float cc = c0[kk - 1] + c1[j - kk - 1];
                if (dist > cc) { dist = cc; bk = kk; }
            }
            if (c[j - 2] <= dist) { c[j - 1] = c[j - 2]; xl[j - 1] = xl[j - 2]; xr[j - 1] = xr[j - 2]; }
            else { c[j - 1] = dist; xl[j - 1] = (int8_t)bk; xr[j - 1] = (int8_t)(j - bk); }
        }
    }
    // collapseWide: children (binary node, budget) of every wide interior node, breadth first
    struct kid { int v, k; bool leaf; };
    auto is_leaf_at = [&](int v, int k) { return D.cl[(size_t)v * J + k - 1] < 0; };
    std::vector<std::vector<kid>> kids;
    std::vector<int> wnode, wparent;  // binary node of each wide interior node, its wide parent
    std::vector<std::pair<int, int>> queue{{0, 1}};
    std::vector<int> qparent{-1};
    for (size_t h = 0; h < queue.size(); ++h) {
        const int v = queue[h].first, budget = queue[h].second;
        int kl = D.cl[(size_t)v * J + budget - 1], kr = D.cr[(size_t)v * J + budget - 1];
        if (kl < 0) { kl = D.bl[v]; kr = D.br[v]; }  // root whose best choice is a leaf
        std::vector<int> cv{left[v], right[v]}, ck{kl, kr};
        while ((int)cv.size() < N) {
            int sidx = -1;
            for (int i = 0; i < (int)cv.size(); ++i) {
                const int lc = D.cl[(size_t)cv[i] * J + ck[i] - 1], rc = D.cr[(size_t)cv[i] * J + ck[i] - 1];
                if (lc > 0 && rc > 0 && lc + rc < N) { sidx = i; break; }
            }
            if (sidx < 0) break;
            const int x = cv[sidx], b = ck[sidx];
            const int lc = D.cl[(size_t)x * J + b - 1], rc = D.cr[(size_t)x * J + b - 1];
            cv[sidx] = left[x]; ck[sidx] = lc;
            cv.insert(cv.begin() + sidx + 1, right[x]);
            ck.insert(ck.begin() + sidx + 1, rc);
        }
        std::vector<kid> ks;
        for (size_t i = 0; i < cv.size(); ++i) {
            const bool lf = is_leaf_at(cv[i], ck[i]);
            ks.push_back({cv[i], ck[i], lf});
        }
        kids.push_back(ks);
        wnode.push_back(v);
        wparent.push_back(qparent[h]);
        for (const kid& c : ks)
            if (!c.leaf) { queue.push_back({c.v, c.k}); qparent.push_back((int)h); }
    }
    // BVHConverter::convert: breadth-first numbering, interior nodes first
    const int ni = (int)kids.size();
    int nl = 0;
    for (const auto& ks : kids)
        for (const kid& c : ks) nl += c.leaf;
    std::memset(nodes_out, 0, (size_t)(ni + nl) * W * 4);
    int next_int = 1, next_leaf = ni;
    for (int w = 0; w < ni; ++w) {
        int32_t* nd = nodes_out + (size_t)w * W;
        const auto& ks = kids[w];
        for (int i = 0; i < (int)ks.size(); ++i) {
            float mn[3], mx[3];
            box(ks[i].v, mn, mx);
            put_box(nd, i, mn, mx);
            if (ks[i].leaf) {
                const int li = next_leaf++;
                nd[4 * (N + i) + 2] = ~li;
                int32_t* lf = nodes_out + (size_t)li * W;
                for (int q = 0; q < N; ++q) put_box(lf, q, mn, mx);
                lf[4 * N + 2] = beg[ks[i].v];
                lf[4 * N + 3] = end[ks[i].v];
                lf[8 * N - 9] = 0;
                lf[8 * N - 5] = ~(end[ks[i].v] - beg[ks[i].v]);
                lf[8 * N - 1] = w;
            } else {
                nd[4 * (N + i) + 2] = next_int++;  // children are queued in this order
            }
        }
        {  // unused slots: the degenerate box at child 0's minimum corner and child 0's
           // index as getChildIndex returns it (decoded, also for a leaf child)
            float mn0[3], mx0[3];
            box(ks[0].v, mn0, mx0);
            const int32_t d0 = nd[4 * N + 2];
            for (int i = (int)ks.size(); i < N; ++i) {
                put_box(nd, i, mn0, mn0);
                nd[4 * (N + i) + 2] = d0 < 0 ? ~d0 : d0;
            }
        }
        nd[8 * N - 9] = (int)ks.size();
        nd[8 * N - 5] = end[wnode[w]] - beg[wnode[w]];
        nd[8 * N - 1] = wparent[w];
    }
    counts[0] = ni;
    counts[1] = nl;
    return (int64_t)ni + nl;
}

}  // extern "C"

// The final binary tree of a build (method 0 LBVH, 1 PLOC, 2 ATR, 3 TRBVH, 4 HLBVH) before its
// collapse: children, refitted boxes and the sorted reference order.
void or_binary_tree(const float* verts, const int32_t* tris, int64_t n64, int method, int bits, int radius,
                    int max_radius, int adaptive_r, int treelet, int iterations, int sah_bits, float ct, float ci,
                    const float* scale_in, int32_t* left, int32_t* right, float* nbmin4, float* nbmax4,
                    int32_t* sorted_tri, float* scene_box, float* scale_out) {
    const int n = (int)n64;
    std::vector<float> bmin(4 * (size_t)n), bmax(4 * (size_t)n);
    or_tri_boxes(verts, tris, n, bmin.data(), bmax.data(), scene_box);
    std::vector<uint64_t> keys(n), skeys(n);
    or_morton(n, bmin.data(), bmax.data(), scene_box, scale_in, bits, keys.data(), scale_out);
    or_sort(n, keys.data(), bits, skeys.data(), sorted_tri);
    const int nn = 2 * n - 1;
    std::vector<int32_t> parent(nn), size(nn), state(nn);
    std::vector<float> cost(nn);
    if (n == 1) {
        tri_box(verts, tris, sorted_tri[0], nbmin4, nbmax4);
        nbmin4[3] = nbmax4[3] = 0.0f;
        left[0] = 0;
        right[0] = 1;
        return;
    }
    if (method == 1) {
        or_ploc(n, verts, tris, sorted_tri, radius, max_radius, adaptive_r, ct, ci, 1, 8, parent.data(), left, right,
                nbmin4, nbmax4, size.data(), cost.data(), state.data());
        return;
    }
    or_karras(n, skeys.data(), parent.data(), left, right);
    or_refit(n, verts, tris, sorted_tri, parent.data(), left, right, ct, ci, 1, 8, nbmin4, nbmax4, size.data(),
             cost.data(), state.data());
    if (method == 2 || method == 3 || method == 4) {
        if (method == 2) or_atr(n, treelet, iterations, ct, ci, parent.data(), left, right, nbmin4, nbmax4);
        else if (method == 3) or_tr(n, iterations, ct, ci, parent.data(), left, right, nbmin4, nbmax4);
        else or_hlbvh(n, skeys.data(), bits, sah_bits, parent.data(), left, right, nbmin4, nbmax4);
        or_refit(n, verts, tris, sorted_tri, parent.data(), left, right, ct, ci, 1, 8, nbmin4, nbmax4, size.data(),
                 cost.data(), state.data());
    }
}

// Whole build into an N-wide layout: the binary tree of the method, the wide
// collapse, then the Woop triangles in the collapsed reference order.
int64_t or_build_wide(const float* verts, const int32_t* tris, int64_t n64, int method, int bits, int radius,
                      int max_radius, int adaptive_r, int treelet, int iterations, int sah_bits, float ct, float ci,
                      int adaptive,
                      int max_leaf, int width, const float* scale_in, int32_t* nodes_out, float* woop4,
                      int32_t* tri_idx, int32_t* counts, float* scene_box, float* scale_out) {
    const int n = (int)n64;
    counts[0] = counts[1] = 0;
    if (n == 0) return 0;
    const int nn = 2 * n - 1;
    std::vector<int32_t> left(nn), right(nn), sorted(n);
    std::vector<float> nbmin(4 * (size_t)nn), nbmax(4 * (size_t)nn);
    or_binary_tree(verts, tris, n64, method, bits, radius, max_radius, adaptive_r, treelet, iterations, sah_bits, ct,
                   ci, scale_in, left.data(), right.data(), nbmin.data(), nbmax.data(), sorted.data(), scene_box,
                   scale_out);
    const int64_t c = or_collapse_wide(n, sorted.data(), left.data(), right.data(), nbmin.data(), nbmax.data(),
                                       width, ct, ci, adaptive ? 0x7fffffff : max_leaf, nodes_out, tri_idx, counts);
    or_woopify(n, verts, tris, tri_idx, woop4);
    return c;
}

// ---- ray generation and ray keys ---------------------------------------------------
// PixelTable::recalculate (rt/ray/PixelTable.cpp:10-80), walked as the reference
// does: Morton indices over a square of block coordinates whose side is the
// power of two the reference's bit-smearing gives, keeping blocks inside the
// image, then the bottom stripe column by column and the right stripe row by row.
int32_t or_pixel_table(int32_t width, int32_t height, int32_t* idxtopos) {
    int idx = 0;
    const int bheight = height & ~7, bwidth = width & ~7;
    int maxdim = bwidth > bheight ? bwidth : bheight;
    maxdim |= maxdim >> 1;
    maxdim |= maxdim >> 2;
    maxdim |= maxdim >> 4;
    maxdim |= maxdim >> 8;
    maxdim |= maxdim >> 16;
    maxdim = (maxdim + 1) >> 1;
    const int width8 = bwidth >> 3, height8 = bheight >> 3;
    for (int64_t i = 0; i < (int64_t)maxdim * maxdim; ++i) {
        int tx = 0, ty = 0, bit = 1;
        int64_t val = i;
        while (val) {
            if (val & 1) tx |= bit;
            if (val & 2) ty |= bit;
            bit += bit;
            val >>= 2;
        }
        if (tx < width8 && ty < height8) {
            for (int inner = 0; inner < 64; inner++) {
                const int ix = ((inner & 1) >> 0) | ((inner & 4) >> 1) | ((inner & 16) >> 2);
                const int iy = ((inner & 2) >> 1) | ((inner & 8) >> 2) | ((inner & 32) >> 3);
                idxtopos[idx++] = (ty * 8 + iy) * width + (tx * 8 + ix);
            }
        }
    }
    for (int px = 0; px < bwidth; px++)
        for (int py = bheight; py < height; py++) idxtopos[idx++] = px + py * width;
    for (int py = 0; py < height; py++)
        for (int px = bwidth; px < width; px++) idxtopos[idx++] = px + py * width;
    return idx;
}

// generatePrimaryRays (rt/ray/RayGenKernels.cu:106-153) with IEEE rounding and
// the fma order of the CUDA kernel; hx, hy: the sample's Halton point.
void or_primary_rays(const float* origin, const float* m, int32_t width, int32_t height, float hx, float hy,
                     float max_dist, const int32_t* index_to_pixel, float* rays) {
    const int64_t n = (int64_t)width * height;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const int64_t pixel = index_to_pixel ? index_to_pixel[i] : i;
        const float x = (float)(pixel % width) + hx, y = (float)(pixel / width) + hy;
        const float nx = (2.0f * x) / (float)width - 1.0f, ny = (2.0f * y) / (float)height - 1.0f;
        float w[4];
        for (int r = 0; r < 4; ++r) w[r] = std::fmaf(m[4 * r], nx, std::fmaf(m[4 * r + 1], ny, m[4 * r + 3]));
        const float dx = w[0] / w[3] - origin[0], dy = w[1] / w[3] - origin[1], dz = w[2] / w[3] - origin[2];
        const float len = std::sqrt(std::fmaf(dz, dz, std::fmaf(dy, dy, dx * dx)));
        float* r = rays + 8 * i;
        r[0] = origin[0]; r[1] = origin[1]; r[2] = origin[2]; r[3] = 0.0f;
        r[4] = dx / len; r[5] = dy / len; r[6] = dz / len; r[7] = max_dist;
    }
}

// ---- ray Morton keys: the 64-bit kernels computeMortonCodes*64 of
// rt/ray/RayBufferKernels.cu:492-921 (method order of RayBuffer::
// MortonCodeMethod, rt/ray/RayBuffer.h:20-28), every step IEEE-rounded; the
// origin is normalised by the box's inverse extent; Costa and Reis use the
// library's own atan2 / acos (an odd polynomial of degree 17 for atan on
// [0, 1], coefficients fitted by reweighted least squares at Chebyshev nodes).
namespace {

inline int sat_trunc(float v) {  // float -> int by truncation, saturating, NaN -> 0 (as cvt.rzi on the GPU)
    if (!(v == v)) return 0;
    if (v >= 2147483648.0f) return 2147483647;
    if (v <= -2147483648.0f) return (int)0x80000000u;
    return (int)std::trunc(v);
}
inline int qz(float a, float scale) { return sat_trunc(a * scale); }

inline float rk_atan01(float t) {
    const float s = t * t;
    float p = 0.0024567153304815292f;
    p = std::fmaf(p, s, -0.014401324093341827f);
    p = std::fmaf(p, s, 0.039781175553798676f);
    p = std::fmaf(p, s, -0.07234854251146317f);
    p = std::fmaf(p, s, 0.10498945415019989f);
    p = std::fmaf(p, s, -0.14161229133605957f);
    p = std::fmaf(p, s, 0.19985906779766083f);
    p = std::fmaf(p, s, -0.33332598209381104f);
    p = std::fmaf(p, s, 0.9999998807907104f);
    return t * p;
}
inline float rk_atan2(float y, float x) {
    const float ax = std::fabs(x), ay = std::fabs(y);
    const float hi = std::fmax(ax, ay), lo = std::fmin(ax, ay);
    if (!(hi > 0.0f)) return 0.0f;
    float r = rk_atan01(lo / hi);
    if (ay > ax) r = 1.5707963705062866f - r;
    if (x < 0.0f) r = 3.1415927410125732f - r;
    return y < 0.0f ? -r : r;
}
inline float rk_acos(float z) { return rk_atan2(std::sqrt(std::fmax(std::fmaf(-z, z, 1.0f), 0.0f)), z); }

uint64_t ray_code(const float* r, int method, const float* mn, const float* mx, const float* inv, float ray_length) {
    const float a0 = (r[0] - mn[0]) * inv[0], a1 = (r[1] - mn[1]) * inv[1], a2 = (r[2] - mn[2]) * inv[2];
    uint64_t c = 0;
    if (method == 0) {  // two point (RayBufferKernels.cu:492-554; intersect :11-56)
        float t0[3], t1[3];
        for (int a = 0; a < 3; ++a) {
            const float lo = r[4 + a] >= 0.0f ? mn[a] : mx[a], hi = r[4 + a] >= 0.0f ? mx[a] : mn[a];
            t0[a] = (lo - r[a]) / r[4 + a];
            t1[a] = (hi - r[a]) / r[4 + a];
        }
        const float tmin = std::fmax(t0[2], std::fmax(t0[0], t0[1]));
        const float tmax = std::fmin(t1[2], std::fmin(t1[0], t1[1]));
        const float hit = tmin > tmax ? -1.0f : (1.0f - 1.0e-3f) * (tmin >= 0.0f ? tmin : tmax);
        float len = std::fmin(ray_length, std::fmax(r[7], 0.0f));
        len = std::fmin(len, hit);
        int ia[3], ib[3];
        const float aa[3] = {a0, a1, a2};
        for (int a = 0; a < 3; ++a) {
            ia[a] = qz(aa[a], 8191.0f);
            ib[a] = qz((std::fmaf(len, r[4 + a], r[a]) - mn[a]) * inv[a], 8191.0f);
        }
        for (int i = 12; i >= 2; --i)
            for (int a = 0; a < 3; ++a) c |= (uint64_t)((ia[a] >> i) & 1) << (6 * i - 9 - a);
        for (int i = 12; i >= 3; --i)
            for (int a = 0; a < 3; ++a) c |= (uint64_t)((ib[a] >> i) & 1) << (6 * i - 12 - a);
        c |= (uint64_t)(ib[0] & 1);
        return c;
    }
    if (method == 4) {  // origin (RayBufferKernels.cu:775-814)
        const int ia[3] = {qz(a0, 8388607.0f), qz(a1, 8388607.0f), qz(a2, 8388607.0f)};
        for (int i = 22; i >= 2; --i)
            for (int a = 0; a < 3; ++a) c |= (uint64_t)((ia[a] >> i) & 1) << (3 * i - 3 - a);
        c |= (uint64_t)(ia[0] & 1);
        return c;
    }
    const float len = std::sqrt(std::fmaf(r[6], r[6], std::fmaf(r[5], r[5], r[4] * r[4])));
    const float nx = r[4] / len, ny = r[5] / len, nz = r[6] / len;
    if (method == 2 || method == 3) {  // paraboloid / octahedron (RayBufferKernels.cu:616-773)
        float bx, by;
        if (method == 2) {
            if (nz < 0.0f) {
                const float dd = -nz + 1.0f;
                bx = (0.25f * nx) / dd + 0.25f;
                by = (0.5f * ny) / dd + 0.5f;
            } else {
                const float dd = nz + 1.0f;
                bx = (0.25f * nx) / dd + 0.75f;
                by = (0.5f * ny) / dd + 0.5f;
            }
        } else {
            const float ax = std::fabs(nx), ay = std::fabs(ny), az = std::fabs(nz);
            const float fact = 1.0f / ((ax + ay) + az);
            if (nz >= 0.0f) {
                bx = nx * fact;
                by = ny * fact;
            } else {
                bx = (1.0f - ay * fact) * (nx <= 0.0f ? -1.0f : 1.0f);
                by = (1.0f - ax * fact) * (ny <= 0.0f ? -1.0f : 1.0f);
            }
            bx = (bx + 1.0f) * 0.5f;
            by = (by + 1.0f) * 0.5f;
        }
        const int ia[3] = {qz(a0, 32767.0f), qz(a1, 32767.0f), qz(a2, 32767.0f)};
        const int ib[2] = {qz(bx, 32767.0f), qz(by, 32767.0f)};
        for (int i = 14; i >= 11; --i)
            for (int a = 0; a < 3; ++a) c |= (uint64_t)((ia[a] >> i) & 1) << (63 - 3 * (14 - i) - a);
        for (int i = 10; i >= 0; --i) {
            c |= (uint64_t)((ia[0] >> i) & 1) << (5 * i + 1);
            c |= (uint64_t)((ia[1] >> i) & 1) << (5 * i);
            if (i > 0) c |= (uint64_t)((ia[2] >> i) & 1) << (5 * i - 1);
        }
        for (int i = 14; i >= 5; --i) {
            c |= (uint64_t)((ib[0] >> i) & 1) << (5 * i - 22);
            c |= (uint64_t)((ib[1] >> i) & 1) << (5 * i - 23);
        }
        return c;
    }
    if (method == 5 || method == 6) {  // Costa / Reis (RayBufferKernels.cu:816-921)
        const float bx = rk_atan2(ny, nx) / 6.2831854820251465f + 0.5f;
        const float by = rk_acos(nz) / 3.1415927410125732f;
        if (method == 5) {
            const int ia[3] = {qz(a0, 32767.0f), qz(a1, 32767.0f), qz(a2, 32767.0f)};
            const int ib[2] = {qz(bx, 32767.0f), qz(by, 32767.0f)};
            for (int i = 14; i >= 11; --i) {
                c |= (uint64_t)((ib[0] >> i) & 1) << (2 * i + 35);
                c |= (uint64_t)((ib[1] >> i) & 1) << (2 * i + 34);
            }
            for (int i = 14; i >= 0; --i)
                for (int a = 0; a < 3; ++a) c |= (uint64_t)((ia[a] >> i) & 1) << (3 * i + 13 - a);
        } else {
            const int ia[3] = {qz(a0, 2097151.0f), qz(a1, 2097151.0f), qz(a2, 2097151.0f)};
            const int ib[2] = {qz(bx, 2097151.0f), qz(by, 2097151.0f)};
            for (int i = 20; i >= 14; --i)
                for (int a = 0; a < 3; ++a) c |= (uint64_t)((ia[a] >> i) & 1) << (3 * i + 3 - a);
            c |= (uint64_t)((ia[0] >> 13) & 1) << 42;
            for (int i = 20; i >= 0; --i) {
                c |= (uint64_t)((ib[0] >> i) & 1) << (2 * i + 1);
                c |= (uint64_t)((ib[1] >> i) & 1) << (2 * i);
            }
        }
        return c;
    }
    // Aila (RayBufferKernels.cu:556-615)
    const int ia[3] = {qz(a0, 8191.0f), qz(a1, 8191.0f), qz(a2, 8191.0f)};
    const int ib[3] = {qz((nx + 1.0f) * 0.5f, 8191.0f), qz((ny + 1.0f) * 0.5f, 8191.0f),
                       qz((nz + 1.0f) * 0.5f, 8191.0f)};
    for (int b = 12; b >= 10; --b)
        for (int a = 0; a < 3; ++a) c |= (uint64_t)((ia[a] >> b) & 1) << (63 - 3 * (12 - b) - a);
    for (int b = 9; b >= 1; --b)
        for (int a = 0; a < 3; ++a) c |= (uint64_t)((ia[a] >> b) & 1) << (6 * b - a);
    for (int b = 12; b >= 4; --b)
        for (int a = 0; a < 3; ++a) c |= (uint64_t)((ib[a] >> b) & 1) << (6 * b - 21 - a);
    return c;
}

}  // namespace

void or_ray_keys_method(const float* rays, int64_t n, const float* box6, int32_t bits, int32_t method,
                        float ray_length, uint64_t* keys) {
    float mn[3], mx[3], inv[3];
    for (int a = 0; a < 3; ++a) {
        mn[a] = box6[a];
        mx[a] = box6[3 + a];
        const float ext = box6[3 + a] - box6[a];
        inv[a] = ext > 0.0f ? 1.0f / ext : 0.0f;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const uint64_t c = ray_code(rays + 8 * i, method, mn, mx, inv, ray_length);
        keys[i] = bits == 64 ? c : c >> (64 - bits);
    }
}

// The default method (Aila).
void or_ray_keys(const float* rays, int64_t n, const float* box6, int32_t bits, uint64_t* keys) {
    or_ray_keys_method(rays, n, box6, bits, 1, 0.25f, keys);
}

// ---- A12: HipBVH::getCost (rt/bvh/HipBVH.cpp:346-370, HipBVHKernels.cu:184-238) ----------
double or_cost(const void* nodes_in, int64_t count, const float* scene_box, float ct, float ci) {
    const bin_node* nd = reinterpret_cast<const bin_node*>(nodes_in);
    const double sa = area6(scene_box[0], scene_box[1], scene_box[2], scene_box[3], scene_box[4], scene_box[5]);
    double c = 0.0;
    for (int64_t i = 0; i < count; ++i) {
        const float* f = nd[i].f;
        float mn[3] = {std::min(f[0], f[4]), std::min(f[2], f[6]), std::min(f[8], f[10])};
        float mx[3] = {std::max(f[1], f[5]), std::max(f[3], f[7]), std::max(f[9], f[11])};
        double a = area6(mn[0], mn[1], mn[2], mx[0], mx[1], mx[2]) / sa;
        if (nd[i].size < 0) c += (double)ci * a * (double)(~nd[i].size);
        else c += (double)ct * a;
    }
    return c;
}

// ---- A13: closest-hit traversal (rt/tracer/HipTracerBinKernels.cu:19-286) ------------------
// Per ray: near child first, far child pushed; leaves handled as they are reached;
// Woop test with the kernel's fma order; ties in t go to the lower triangle id.
void or_trace(const void* nodes_in, const float* woop4, const int32_t* tri_idx, int64_t num_refs,
              const float* rays, int64_t num_rays, int32_t* results, int32_t* stats, int any_hit) {
    const bin_node* nodes = reinterpret_cast<const bin_node*>(nodes_in);
    const float ooeps = 8.2718061255302767e-25f;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t ri = 0; ri < num_rays; ++ri) {
        const float* ry = rays + 8 * ri;
        const float ox = ry[0], oy = ry[1], oz = ry[2], tmin = ry[3];
        const float dx = ry[4], dy = ry[5], dz = ry[6];
        float hit_t = ry[7], hit_u = 0.0f, hit_v = 0.0f;
        int hit = -1, n_nodes = 0, n_tris = 0;
        auto srcp = [&](float d) { return 1.0f / (std::fabs(d) > ooeps ? d : std::copysign(ooeps, d)); };
        const float idx = srcp(dx), idy = srcp(dy), idz = srcp(dz);
        const float oodx = ox * idx, oody = oy * idy, oodz = oz * idz;
        int stack[64];
        int sp = 0;
        int node = num_refs > 0 ? 0 : -0x7fffffff;
        bool done = num_refs <= 0;
        while (!done) {
            if (node >= 0) {
                ++n_nodes;
                const float* f = nodes[node].f;
                auto slab = [&](float b, float id, float ood) { return std::fmaf(b, id, -ood); };
                const float c0lox = slab(f[0], idx, oodx), c0hix = slab(f[1], idx, oodx);
                const float c0loy = slab(f[2], idy, oody), c0hiy = slab(f[3], idy, oody);
                const float c0loz = slab(f[8], idz, oodz), c0hiz = slab(f[9], idz, oodz);
                const float c1lox = slab(f[4], idx, oodx), c1hix = slab(f[5], idx, oodx);
                const float c1loy = slab(f[6], idy, oody), c1hiy = slab(f[7], idy, oody);
                const float c1loz = slab(f[10], idz, oodz), c1hiz = slab(f[11], idz, oodz);
                const float c0min = std::max(std::max(std::min(c0lox, c0hix), std::min(c0loy, c0hiy)),
                                             std::max(std::min(c0loz, c0hiz), tmin));
                const float c0max = std::min(std::min(std::max(c0lox, c0hix), std::max(c0loy, c0hiy)),
                                             std::min(std::max(c0loz, c0hiz), hit_t));
                const float c1min = std::max(std::max(std::min(c1lox, c1hix), std::min(c1loy, c1hiy)),
                                             std::max(std::min(c1loz, c1hiz), tmin));
                const float c1max = std::min(std::min(std::max(c1lox, c1hix), std::max(c1loy, c1hiy)),
                                             std::min(std::max(c1loz, c1hiz), hit_t));
                const bool t0 = c0max >= c0min, t1 = c1max >= c1min;
                const int c0 = nodes[node].c0, c1 = nodes[node].c1;
                if (!t0 && !t1) {
                    if (sp == 0) { done = true; continue; }
                    node = stack[--sp];
                } else {
                    node = t0 ? c0 : c1;
                    if (t0 && t1) {
                        int far = c1;
                        if (c1min < c0min) { node = c1; far = c0; }
                        if (sp < 64) stack[sp++] = far;
                    }
                }
            } else {
                const bin_node& lf = nodes[~node];
                for (int tri = lf.c0; tri < lf.c1; ++tri) {
                    ++n_tris;
                    const float* v0 = woop4 + 12 * (int64_t)tri;
                    const float* v1 = v0 + 4;
                    const float* v2 = v0 + 8;
                    // The fast-math roundings of HipTracerBinKernels.cu:216-241 as the
                    // kernels write them: left-to-right chains for o.w; the
                    // denominator and the v term fuse x over the rounded y product,
                    // the u term y over the rounded x product.
                    const float Oz = std::fmaf(-oz, v0[2], std::fmaf(-oy, v0[1], std::fmaf(-ox, v0[0], v0[3])));
                    const float den = std::fmaf(dz, v0[2], std::fmaf(dx, v0[0], dy * v0[1]));
                    const float t = Oz * (1.0f / den);
                    bool closer = t < hit_t;
                    if (!closer && t == hit_t && hit >= 0) closer = tri_idx[tri] < tri_idx[hit];
                    if (t > tmin && closer) {
                        const float Ox = std::fmaf(oz, v1[2], std::fmaf(oy, v1[1], std::fmaf(ox, v1[0], v1[3])));
                        const float Dx = std::fmaf(dz, v1[2], std::fmaf(dy, v1[1], dx * v1[0]));
                        const float u = std::fmaf(t, Dx, Ox);
                        if (u >= 0.0f) {
                            const float Oy = std::fmaf(oz, v2[2], std::fmaf(oy, v2[1], std::fmaf(ox, v2[0], v2[3])));
                            const float Dy = std::fmaf(dz, v2[2], std::fmaf(dx, v2[0], dy * v2[1]));
                            const float v = std::fmaf(t, Dy, Oy);
                            if (v >= 0.0f && u + v <= 1.0f) {
                                hit_t = t; hit = tri; hit_u = u; hit_v = v;
                                if (any_hit) break;
                            }
                        }
                    }
                }
                if (any_hit && hit >= 0) break;
                if (sp == 0) break;
                node = stack[--sp];
            }
        }
        int32_t* res = results + 4 * ri;
        if (hit < 0) {
            res[0] = -1;
            std::memcpy(&res[1], &hit_t, 4);
            if (stats) { stats[2 * ri] = 0; stats[2 * ri + 1] = 0; }
        } else {
            res[0] = tri_idx[hit];
            std::memcpy(&res[1], &hit_t, 4);
            std::memcpy(&res[2], &hit_u, 4);
            std::memcpy(&res[3], &hit_v, 4);
            if (stats) { stats[2 * ri] = n_nodes; stats[2 * ri + 1] = n_tris; }
        }
    }
}

// Double-precision intersection of one ray with one triangle, in the
// reference's barycentric convention (u weights v0, v weights v1). Returns 1
// on a hit with t > tmin.
int or_intersect64(const double* v0, const double* v1, const double* v2, const double* o, const double* d,
                   double tmin, double* tuv) {
    double a[3], b[3], c[3], rhs[3];
    for (int k = 0; k < 3; ++k) {
        a[k] = v0[k] - v2[k];
        b[k] = v1[k] - v2[k];
        c[k] = -d[k];
        rhs[k] = o[k] - v2[k];
    }
    auto cross = [](const double* x, const double* y, double* r) {
        r[0] = x[1] * y[2] - x[2] * y[1];
        r[1] = x[2] * y[0] - x[0] * y[2];
        r[2] = x[0] * y[1] - x[1] * y[0];
    };
    double bc[3], ca[3], ab[3];
    cross(b, c, bc); cross(c, a, ca); cross(a, b, ab);
    double det = a[0] * bc[0] + a[1] * bc[1] + a[2] * bc[2];
    if (det == 0.0) return 0;
    double u = (rhs[0] * bc[0] + rhs[1] * bc[1] + rhs[2] * bc[2]) / det;
    double v = (rhs[0] * ca[0] + rhs[1] * ca[1] + rhs[2] * ca[2]) / det;
    double t = (rhs[0] * ab[0] + rhs[1] * ab[1] + rhs[2] * ab[2]) / det;
    tuv[0] = t; tuv[1] = u; tuv[2] = v;
    return (t > tmin && u >= 0.0 && v >= 0.0 && u + v <= 1.0) ? 1 : 0;
}

// Brute-force closest hit in double precision (small cases): results as
// (triangle id, t, u, v) in doubles; id -1 on a miss. Ties go to the lower id.
void or_brute64(const float* verts, const int32_t* tris, int64_t n, const float* rays, int64_t num_rays,
                double* out) {
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t ri = 0; ri < num_rays; ++ri) {
        const float* ry = rays + 8 * ri;
        double o[3] = {ry[0], ry[1], ry[2]}, d[3] = {ry[4], ry[5], ry[6]};
        double best_t = ry[7], bu = 0, bv = 0;
        int64_t best = -1;
        for (int64_t i = 0; i < n; ++i) {
            double p[3][3];
            for (int k = 0; k < 3; ++k)
                for (int a = 0; a < 3; ++a) p[k][a] = verts[3 * (int64_t)tris[3 * i + k] + a];
            double tuv[3];
            if (or_intersect64(p[0], p[1], p[2], o, d, ry[3], tuv) && tuv[0] < best_t) {
                best_t = tuv[0]; bu = tuv[1]; bv = tuv[2]; best = i;
            }
        }
        out[4 * ri] = (double)best;
        out[4 * ri + 1] = best_t;
        out[4 * ri + 2] = bu;
        out[4 * ri + 3] = bv;
    }
}

// Adjoint in double precision: dL/dvertices of sum_r (g_t t + g_u u + g_v v) for
// the hit triangles of `results` (ids), with (t, u, v) recomputed in double.
void or_adjoint64(const float* verts, const int32_t* tris, const float* rays, const int32_t* results,
                  const float* dl, int64_t num_rays, double* dverts) {
    for (int64_t ri = 0; ri < num_rays; ++ri) {
        const int tri = results[4 * ri];
        if (tri < 0) continue;
        const float* ry = rays + 8 * ri;
        double p[3][3];
        int vid[3];
        for (int k = 0; k < 3; ++k) {
            vid[k] = tris[3 * (int64_t)tri + k];
            for (int a = 0; a < 3; ++a) p[k][a] = verts[3 * (int64_t)vid[k] + a];
        }
        double a[3], b[3], c[3], rhs[3];
        for (int k = 0; k < 3; ++k) {
            a[k] = p[0][k] - p[2][k]; b[k] = p[1][k] - p[2][k]; c[k] = -(double)ry[4 + k];
            rhs[k] = (double)ry[k] - p[2][k];
        }
        auto cross = [](const double* x, const double* y, double* r) {
            r[0] = x[1] * y[2] - x[2] * y[1];
            r[1] = x[2] * y[0] - x[0] * y[2];
            r[2] = x[0] * y[1] - x[1] * y[0];
        };
        double bc[3], ca[3], ab[3];
        cross(b, c, bc); cross(c, a, ca); cross(a, b, ab);
        double det = a[0] * bc[0] + a[1] * bc[1] + a[2] * bc[2];
        if (det == 0.0) continue;
        double u = (rhs[0] * bc[0] + rhs[1] * bc[1] + rhs[2] * bc[2]) / det;
        double v = (rhs[0] * ca[0] + rhs[1] * ca[1] + rhs[2] * ca[2]) / det;
        const double gt = dl[3 * ri], gu = dl[3 * ri + 1], gv = dl[3 * ri + 2];
        double q[3];
        for (int k = 0; k < 3; ++k) q[k] = (gu * bc[k] + gv * ca[k] + gt * ab[k]) / det;
        const double w[3] = {u, v, 1.0 - u - v};
        for (int k = 0; k < 3; ++k)
            for (int x = 0; x < 3; ++x) dverts[3 * (int64_t)vid[k] + x] -= w[k] * q[x];
    }
}

}  // extern "C"

// ---- canonical form of a collapsed binary BVH ---------------------------------
// Builders that number nodes by atomics (the reference's collapser,
// rt/bvh/BVHCollapserKernels.cu:268-433) leave node order and the order of
// triangles inside a leaf undefined; the tree itself is defined. Its canonical
// form: nodes in depth-first order from the root, child 0 before child 1;
// per node its 12 child-box words and its size word (~size for a leaf), and
// per leaf its triangle ids in ascending order, appended in visit order.
// Returns the number of nodes visited, or -1 if an index leaves the arrays or
// a node is reached twice.
extern "C" int64_t or_canonical(const int32_t* nodes, int64_t num_nodes, const int32_t* tri_idx, int64_t num_refs,
                                int32_t* rows /* [num_nodes][13] */, int32_t* tris /* [num_refs] */) {
    if (num_nodes <= 0) return 0;
    std::vector<int32_t> stack{0};
    std::vector<char> seen((size_t)num_nodes, 0);
    int64_t count = 0, nt = 0;
    while (!stack.empty()) {
        const int32_t i = stack.back();
        stack.pop_back();
        if (i < 0 || i >= num_nodes || seen[(size_t)i]) return -1;
        seen[(size_t)i] = 1;
        const int32_t* nd = nodes + 16 * (int64_t)i;
        int32_t* row = rows + 13 * count++;
        for (int k = 0; k < 12; ++k) row[k] = nd[k];
        row[12] = nd[14];
        if (nd[14] < 0) {
            const int32_t b = nd[12], e = nd[13];
            if (b < 0 || e < b || e > num_refs || nt + (e - b) > num_refs) return -1;
            std::copy(tri_idx + b, tri_idx + e, tris + nt);
            std::sort(tris + nt, tris + nt + (e - b));
            nt += e - b;
        } else {
            stack.push_back(nd[13] < 0 ? ~nd[13] : nd[13]);
            stack.push_back(nd[12] < 0 ? ~nd[12] : nd[12]);
        }
    }
    return count;
}

// ---- synthetic inputs, without the library ------------------------------------
// The same streams as the library's generators (hippie_b200/csrc/gen.cpp), so
// that the CPU arm of the benchmark builds its inputs without loading the GPU
// library: a SplitMix64 finaliser over (seed, item, slot), uniforms
// (h >> 40) * 2^-24, Box-Muller normals in double. tests/test_raygen.py checks
// that both produce the same bytes.
namespace {
inline uint64_t gn_mix(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
inline float gn_u(uint64_t seed, uint64_t item, uint32_t slot) {
    const uint64_t h = gn_mix((seed * 0xD1B54A32D192ED03ull) ^ (item * 64u + slot));
    return (float)((double)(h >> 40) * (1.0 / 16777216.0));
}
inline double gn_normal(uint64_t seed, uint64_t item, uint32_t slot) {
    const double a = 1.0 - (double)gn_u(seed, item, slot);
    const double b = (double)gn_u(seed, item, slot + 1);
    return std::sqrt(-2.0 * std::log(a)) * std::cos(6.283185307179586 * b);
}
}  // namespace

extern "C" {

void or_gen_uniform_mesh(uint64_t seed, int64_t n, float h, float* v, int32_t* t) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        float c[3];
        for (int a = 0; a < 3; ++a) c[a] = gn_u(seed, i, a);
        for (int k = 0; k < 3; ++k) {
            for (int a = 0; a < 3; ++a) v[9 * i + 3 * k + a] = c[a] + (2.0f * gn_u(seed, i, 3 + 3 * k + a) - 1.0f) * h;
            t[3 * i + k] = (int32_t)(3 * i + k);
        }
    }
}

void or_gen_clustered_mesh(uint64_t seed, int64_t n, int32_t clusters, float sigma, float h, float* v,
                           int32_t* t) {
    const uint64_t cseed = seed ^ 0xA5A5A5A55A5A5A5Aull;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const int64_t cl = i % clusters;
        float c[3];
        for (int a = 0; a < 3; ++a) c[a] = gn_u(cseed, cl, a) + (float)((double)sigma * gn_normal(seed, i, 2 * a));
        for (int k = 0; k < 3; ++k) {
            for (int a = 0; a < 3; ++a) v[9 * i + 3 * k + a] = c[a] + (2.0f * gn_u(seed, i, 8 + 3 * k + a) - 1.0f) * h;
            t[3 * i + k] = (int32_t)(3 * i + k);
        }
    }
}

void or_gen_rays_targeted(uint64_t seed, int64_t n, float lo, float hi, float* rays) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double o[3], d[3], len = 0.0;
        for (int a = 0; a < 3; ++a) {
            o[a] = (double)(lo + (hi - lo) * gn_u(seed, i, a));
            d[a] = (double)gn_u(seed, i, 3 + a) - o[a];
            len += d[a] * d[a];
        }
        len = std::sqrt(len);
        if (len == 0.0) { d[0] = 0.0; d[1] = 0.0; d[2] = 1.0; len = 1.0; }
        float* r = rays + 8 * i;
        r[0] = (float)o[0]; r[1] = (float)o[1]; r[2] = (float)o[2]; r[3] = 0.0f;
        r[4] = (float)(d[0] / len); r[5] = (float)(d[1] / len); r[6] = (float)(d[2] / len);
        r[7] = INFINITY;
    }
}

void or_gen_rays_sphere(uint64_t seed, int64_t n, const float* box, float* rays) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        float* r = rays + 8 * i;
        for (int a = 0; a < 3; ++a) r[a] = box[a] + (box[3 + a] - box[a]) * gn_u(seed, i, a);
        r[3] = 0.0f;
        const double z = 2.0 * (double)gn_u(seed, i, 3) - 1.0;
        const double phi = 6.283185307179586 * (double)gn_u(seed, i, 4);
        const double s = std::sqrt(std::max(0.0, 1.0 - z * z));
        r[4] = (float)(s * std::cos(phi));
        r[5] = (float)(s * std::sin(phi));
        r[6] = (float)z;
        r[7] = INFINITY;
    }
}

}  // extern "C"
