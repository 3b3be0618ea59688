// Batched LBVH build and trace of many meshes of uneven size in a fixed number
// of launches (independent of the number of meshes).
//
// Every mesh is an independent LBVH (LBVHBuilder::build, rt/bvh/LBVHBuilder.cpp:
// 183-241) and gets exactly the tree, nodes and Woop triangles the single-mesh
// path builds for it. The meshes are laid out back to back: mesh m owns sorted
// positions / Woop rows / triangle-index slots [tri_off, tri_off + n) and node
// slots [node_off, node_off + max(2n-1, 3)). Each kernel runs over all meshes at
// once and finds an element's mesh from the segment table:
//   * boxes: triangle boxes, and per-mesh scene boxes reduced per warp over the
//     lanes of the same mesh (__match_any_sync + __reduce_*_sync);
//   * Morton keys carry the mesh index above the Morton bits, so one radix sort
//     of all keys sorts every mesh on its own (stably, by original index);
//     with the mesh bits zero in the XOR of two keys of one mesh, the Karras
//     deltas are those of the mesh's own keys, so the hierarchy is identical;
//   * Karras emission, the bottom-up climb (refit, sizes, collapse rule,
//     Woop) and the collapse use mesh-local node indices;
//   * the collapse's max-scan runs over global positions (a state-0 range of
//     one mesh never reaches into the next), and its two counting scans over
//     all meshes, each mesh subtracting the count at its first position.
// Tracing is one persistent launch over the rays of all meshes (k_trace in
// batch mode). The whole sequence is captured once into a CUDA graph and
// replayed.
#include <algorithm>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>
#include "hp_device.cuh"
#include "hp_internal.h"

namespace {

constexpr int TB = 256;

__device__ __forceinline__ int seg_of(const int32_t* __restrict__ off, int num_segs, int64_t g) {
    int lo = 0, hi = num_segs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(off + mid) <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

struct bargs {
    const hp_batch_seg* seg;
    const int32_t* tri_off;  // [M + 1]
    int M;
    int64_t N;
    int bits;                // Morton bits (the mesh index sits above them)
    int passes;  // digits counted for the sort (hp_sort_hist_digits) from shift hshift
    int hshift;
    hp_bvh_info* info;       // [M]
    float4* tbmin;
    float4* tbmax;
    uint64_t* keys;
    const uint64_t* skeys;
    const int32_t* sorted;   // global triangle index per sorted position
    int* parent;             // node slots
    int* left;               // interior slots (tri_off + i)
    int* right;
    int2* range;
    float4* nbmin;           // node slots
    float4* nbmax;
    int* counters;           // interior slots
    int* max_hi;             // positions (global values)
    const int* reach;
    uint8_t* state;          // interior slots
    int* flag_int;           // positions
    int* flag_leaf;
    const int* rank_int;
    const int* rank_leaf;
    const int* totals;       // [2]: all surviving interior nodes, all leaves
    hp_node_bin* nodes;      // output node slots
    float4* woop;            // output, 3 per position
    int32_t* tri_idx;        // output, mesh-local triangle ids
    uint32_t* hist;
    float ct, ci;
    int adaptive, max_leaf;
    int* err;
};

__global__ void k_b_init(bargs B, int hist_words) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < hist_words) B.hist[i] = 0;
    if (i < B.M) {
        for (int k = 0; k < 6; ++k) B.info[i].box_ord[k] = (k < 3) ? 0xffffffffu : 0u;
        B.info[i].num_interior = 0;
        B.info[i].num_leaf = 0;
    }
}

// setupBoxes per triangle; per-mesh scene boxes.
__global__ void __launch_bounds__(TB) k_b_boxes(bargs B) {
    const int64_t g = blockIdx.x * (int64_t)TB + threadIdx.x;
    const bool live = g < B.N;
    const int m = live ? seg_of(B.tri_off, B.M, g) : -1;
    uint32_t o[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    if (live) {
        const hp_batch_seg sg = B.seg[m];
        const tri_verts t = load_tri(sg.verts, sg.nv, sg.tris, g - sg.tri_off, B.err);
        const float ax = fminf(fminf(t.x0, t.x1), t.x2), ay = fminf(fminf(t.y0, t.y1), t.y2),
                    az = fminf(fminf(t.z0, t.z1), t.z2);
        const float bx = fmaxf(fmaxf(t.x0, t.x1), t.x2), by = fmaxf(fmaxf(t.y0, t.y1), t.y2),
                    bz = fmaxf(fmaxf(t.z0, t.z1), t.z2);
        B.tbmin[g] = make_float4(ax, ay, az, 0.0f);
        B.tbmax[g] = make_float4(bx, by, bz, 0.0f);
        o[0] = hp_f2ord(ax); o[1] = hp_f2ord(ay); o[2] = hp_f2ord(az);
        o[3] = hp_f2ord(bx); o[4] = hp_f2ord(by); o[5] = hp_f2ord(bz);
    }
    const unsigned grp = __match_any_sync(HP_FULL_MASK, m);
    uint32_t r[6];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        r[k] = __reduce_min_sync(grp, o[k]);
        r[3 + k] = __reduce_max_sync(grp, o[3 + k]);
    }
    if (live && (threadIdx.x & 31) == __ffs(grp) - 1) {
        uint32_t* bo = B.info[m].box_ord;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            atomicMin(bo + k, r[k]);
            atomicMax(bo + 3 + k, r[3 + k]);
        }
    }
}

// computeMortonCodes60 per mesh (its own box and scale), mesh index above the
// Morton bits, fused with the sort's digit histograms.
__global__ void __launch_bounds__(TB) k_b_morton(bargs B) {
    __shared__ uint32_t sh[8 * 256];
    for (int i = threadIdx.x; i < B.passes * 256; i += TB) sh[i] = 0;
    __syncthreads();
    const int64_t g = blockIdx.x * (int64_t)TB + threadIdx.x;
    if (g < B.N) {
        const int m = seg_of(B.tri_off, B.M, g);
        const hp_bvh_info& in = B.info[m];
        float smin[3], scale[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            smin[k] = hp_ord2f(in.box_ord[k]);
            scale[k] = __fdividef(1.0f, __fsub_rn(hp_ord2f(in.box_ord[3 + k]), smin[k]));
        }
        const float4 a = B.tbmin[g], b = B.tbmax[g];
        const uint64_t key = ((uint64_t)m << B.bits) |
                             hp_morton_key(a.x, a.y, a.z, b.x, b.y, b.z, smin, scale, B.bits);
        B.keys[g] = key;
        for (int p = 0; p < B.passes; ++p)  // bits above the key width are zero
            atomicAdd(&sh[p * 256 + (uint32_t)((key >> (B.hshift + 8 * p)) & 0xffu)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < B.passes * 256; i += TB)
        if (sh[i]) atomicAdd(&B.hist[i], sh[i]);
}

// Per-mesh scale as the single-mesh path records it.
__global__ void k_b_scale(bargs B) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= B.M) return;
    hp_bvh_info& in = B.info[m];
    for (int k = 0; k < 3; ++k)
        in.scale[k] = __fdividef(1.0f, __fsub_rn(hp_ord2f(in.box_ord[3 + k]), hp_ord2f(in.box_ord[k])));
}

__device__ __forceinline__ int ldelta(const uint64_t* k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    const uint64_t a = __ldg(k + i), b = __ldg(k + j);
    if (a != b) return __clzll((long long)(a ^ b));
    return __clzll((long long)(i ^ j)) + 64;
}

// construct<T> (LBVHBuilderKernels.cu:11-63) on each mesh's keys.
__global__ void __launch_bounds__(TB) k_b_karras(bargs B) {
    const int64_t g = blockIdx.x * (int64_t)TB + threadIdx.x;
    if (g >= B.N) return;
    const int m = seg_of(B.tri_off, B.M, g);
    const hp_batch_seg sg = B.seg[m];
    const int n = sg.n, i = (int)(g - sg.tri_off);
    int* parent = B.parent + sg.node_off;
    if (n < 2) return;
    if (i == 0) parent[0] = -1;
    if (i >= n - 1) return;
    const uint64_t* keys = B.skeys + sg.tri_off;
    const int dr = ldelta(keys, n, i, i + 1), dl = ldelta(keys, n, i, i - 1);
    const int d = (dr - dl > 0) - (dr - dl < 0);
    const int dmin = ldelta(keys, n, i, i - d);
    int lmax = 2;
    while (ldelta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (ldelta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = ldelta(keys, n, i, j);
    int s = 0, k = 2, t;
    do {
        t = (l + k - 1) / k;
        k <<= 1;
        if (ldelta(keys, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    const int gamma = i + s * d + min(d, 0);
    int lc = gamma, rc = gamma + 1;
    if (min(i, j) == gamma) lc += n - 1;
    if (max(i, j) == gamma + 1) rc += n - 1;
    B.left[sg.tri_off + i] = lc;
    B.right[sg.tri_off + i] = rc;
    parent[lc] = i;
    parent[rc] = i;
    B.range[sg.tri_off + i] = make_int2(min(i, j), max(i, j));
}

// Woopify, leaf box, then the bottom-up climb of each mesh (refit, sizes,
// computeNodeStatesAdaptive / computeNodeStates). Single-triangle meshes get
// the single-mesh path's three-node tree here.
__global__ void __launch_bounds__(TB) k_b_climb(bargs B) {
    const int64_t g = blockIdx.x * (int64_t)TB + threadIdx.x;
    if (g >= B.N) return;
    const int m = seg_of(B.tri_off, B.M, g);
    const hp_batch_seg sg = B.seg[m];
    const int n = sg.n, p = (int)(g - sg.tri_off);
    const int tri = B.sorted[g] - sg.tri_off;
    if ((unsigned)tri >= (unsigned)n) {
        hp_report(B.err, HP_DEV_BAD_INDEX, (int)g);
        return;
    }
    const tri_verts t = load_tri(sg.verts, sg.nv, sg.tris, tri, B.err);
    float4 w0, w1, w2;
    hp_woop(t.x0, t.y0, t.z0, t.x1, t.y1, t.z1, t.x2, t.y2, t.z2, w0, w1, w2);
    B.woop[3 * g + 0] = w0;
    B.woop[3 * g + 1] = w1;
    B.woop[3 * g + 2] = w2;
    B.tri_idx[g] = tri;
    const float ax = fminf(fminf(t.x0, t.x1), t.x2), ay = fminf(fminf(t.y0, t.y1), t.y2),
                az = fminf(fminf(t.z0, t.z1), t.z2);
    const float bx = fmaxf(fmaxf(t.x0, t.x1), t.x2), by = fmaxf(fmaxf(t.y0, t.y1), t.y2),
                bz = fmaxf(fmaxf(t.z0, t.z1), t.z2);
    if (n == 1) {
        hp_node_bin* nodes = B.nodes + sg.node_off;
        const float4 mn = make_float4(ax, ay, az, 0.0f), mx = make_float4(bx, by, bz, 0.0f);
        const float4 emn = make_float4(HP_MAX_FLOAT, HP_MAX_FLOAT, HP_MAX_FLOAT, 0.0f);
        const float4 emx = make_float4(-HP_MAX_FLOAT, -HP_MAX_FLOAT, -HP_MAX_FLOAT, 0.0f);
        nodes[0] = hp_make_node(mn, mx, emn, emx, ~1, ~2, 1, -1);
        nodes[1] = hp_make_node(mn, mx, mn, mx, 0, 1, ~1, 0);
        nodes[2] = hp_make_node(emn, emx, emn, emx, 1, 1, ~0, 0);
        return;
    }
    int* parent = B.parent + sg.node_off;
    const int* left = B.left + sg.tri_off;
    const int* right = B.right + sg.tri_off;
    const int2* range = B.range + sg.tri_off;
    float4* nbmin = B.nbmin + sg.node_off;
    float4* nbmax = B.nbmax + sg.node_off;
    int* counters = B.counters + sg.tri_off;
    uint8_t* state = B.state + sg.tri_off;
    const float cost = B.adaptive ? __fmul_rn(B.ci, hp_area(ax, ay, az, bx, by, bz)) : 0.0f;
    const int leaf = n - 1 + p;
    nbmin[leaf] = make_float4(ax, ay, az, cost);
    nbmax[leaf] = make_float4(bx, by, bz, __int_as_float(1));
    int node = parent[leaf];
    int guard = 0;
    while (node >= 0) {
        if (node >= n - 1 || ++guard > n) {
            hp_report(B.err, HP_DEV_BAD_INDEX, node);
            return;
        }
        __threadfence();
        if (atomicAdd(&counters[node], 1) == 0) return;
        __threadfence();
        const int l = left[node], r = right[node];
        if ((unsigned)l >= (unsigned)(2 * n - 1) || (unsigned)r >= (unsigned)(2 * n - 1)) {
            hp_report(B.err, HP_DEV_BAD_INDEX, node);
            return;
        }
        const float4 lmn = __ldcg(nbmin + l), lmx = __ldcg(nbmax + l);
        const float4 rmn = __ldcg(nbmin + r), rmx = __ldcg(nbmax + r);
        const float mnx = fminf(lmn.x, rmn.x), mny = fminf(lmn.y, rmn.y), mnz = fminf(lmn.z, rmn.z);
        const float mxx = fmaxf(lmx.x, rmx.x), mxy = fmaxf(lmx.y, rmx.y), mxz = fmaxf(lmx.z, rmx.z);
        const int size = __float_as_int(lmx.w) + __float_as_int(rmx.w);
        int st;
        float c;
        if (B.adaptive) {
            const float area = hp_area(mnx, mny, mnz, mxx, mxy, mxz);
            const float c_int = __fadd_rn(__fmaf_rn(B.ct, area, lmn.w), rmn.w);
            const float c_leaf = __fmul_rn(__fmul_rn(B.ci, area), (float)size);
            st = (c_leaf < c_int) ? 0 : 1;
            c = st ? c_int : c_leaf;
        } else {
            st = (size <= B.max_leaf) ? 0 : 1;
            c = 0.0f;
        }
        __stcg(nbmin + node, make_float4(mnx, mny, mnz, c));
        __stcg(nbmax + node, make_float4(mxx, mxy, mxz, __int_as_float(size)));
        state[node] = (uint8_t)st;
        if (st == 0 && node != 0) {
            const int2 rg = range[node];
            atomicMax(&B.max_hi[sg.tri_off + rg.x], sg.tri_off + rg.y);
        }
        node = parent[node];
    }
}

__device__ __forceinline__ int split_of(const int* left, int n, int i) {
    const int l = left[i];
    return l >= n - 1 ? l - (n - 1) : l;
}

// Collapse flags over global positions: interior node i of mesh m survives iff no
// state-0 range strictly contains its range; position p starts a collapsed leaf.
__global__ void __launch_bounds__(TB) k_b_flags(bargs B) {
    const int64_t g = blockIdx.x * (int64_t)TB + threadIdx.x;
    if (g >= B.N) return;
    const int m = seg_of(B.tri_off, B.M, g);
    const hp_batch_seg sg = B.seg[m];
    const int n = sg.n, i = (int)(g - sg.tri_off);
    const int o = sg.tri_off;
    if (n < 2) {
        B.flag_int[g] = 0;
        B.flag_leaf[g] = 0;
        return;
    }
    if (i == n - 1) B.flag_int[g] = 0;  // the split position no interior node takes
    if (i < n - 1) {
        const int2 rg = B.range[o + i];
        const bool alive = (i == 0) || !(B.reach[o + rg.x] >= o + rg.y || B.max_hi[o + rg.x] > o + rg.y);
        B.flag_int[o + split_of(B.left + o, n, i)] = (alive && (i == 0 || B.state[o + i] == 1)) ? 1 : 0;
    }
    B.flag_leaf[g] = (B.reach[g] < g) ? 1 : 0;
}

// Per-mesh node counts from the counting scans.
__global__ void k_b_counts(bargs B) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= B.M) return;
    const hp_batch_seg sg = B.seg[m];
    if (sg.n < 2) {
        B.info[m].num_interior = sg.n == 1 ? 1 : 0;
        B.info[m].num_leaf = sg.n == 1 ? 2 : 0;
        return;
    }
    const int64_t end = (int64_t)sg.tri_off + sg.n;
    const int ri_end = end < B.N ? B.rank_int[end] : B.totals[0];
    const int rl_end = end < B.N ? B.rank_leaf[end] : B.totals[1];
    B.info[m].num_interior = ri_end - B.rank_int[sg.tri_off];
    B.info[m].num_leaf = rl_end - B.rank_leaf[sg.tri_off];
}

struct mesh_view {
    int n, o;
    const int* left;
    const int* right;
    const int* parent;
    const int2* range;
    const uint8_t* state;
    const int* rank_int;   // global ranks; the mesh's base is subtracted
    const int* rank_leaf;
    int base_int, base_leaf, root_rank, num_int;
};

__device__ __forceinline__ int new_interior(const mesh_view& e, int i) {
    if (i == 0) return 0;
    const int r = e.rank_int[e.o + split_of(e.left, e.n, i)] - e.base_int;
    return r < e.root_rank ? r + 1 : r;
}

__device__ __forceinline__ int child_ref(const mesh_view& e, int c) {
    if (c >= e.n - 1) return ~(e.num_int + e.rank_leaf[e.o + c - (e.n - 1)] - e.base_leaf);
    if (e.state[c] == 0) return ~(e.num_int + e.rank_leaf[e.o + e.range[c].x] - e.base_leaf);
    return new_interior(e, c);
}

__device__ __forceinline__ void put(hp_node_bin* nodes, int idx, int max_nodes, const hp_node_bin& nd, int* err) {
    if ((unsigned)idx < (unsigned)max_nodes) nodes[idx] = nd;
    else hp_report(err, HP_DEV_BAD_INDEX, idx);
}

// Emission of each mesh's collapsed nodes (interior node i and leaf n-1+i for
// position i), numbered as the single-mesh path numbers them.
__global__ void __launch_bounds__(TB) k_b_emit(bargs B) {
    const int64_t g = blockIdx.x * (int64_t)TB + threadIdx.x;
    if (g >= B.N) return;
    const int m = seg_of(B.tri_off, B.M, g);
    const hp_batch_seg sg = B.seg[m];
    const int n = sg.n, i = (int)(g - sg.tri_off);
    if (n < 2) return;
    const int o = sg.tri_off;
    mesh_view e;
    e.n = n;
    e.o = o;
    e.left = B.left + o;
    e.right = B.right + o;
    e.parent = B.parent + sg.node_off;
    e.range = B.range + o;
    e.state = B.state + o;
    e.rank_int = B.rank_int;
    e.rank_leaf = B.rank_leaf;
    e.base_int = B.rank_int[o];
    e.base_leaf = B.rank_leaf[o];
    e.root_rank = B.rank_int[o + split_of(e.left, n, 0)] - e.base_int;
    e.num_int = B.info[m].num_interior;
    const float4* nbmin = B.nbmin + sg.node_off;
    const float4* nbmax = B.nbmax + sg.node_off;
    hp_node_bin* nodes = B.nodes + sg.node_off;
    const int max_nodes = 2 * n - 1;
    if (i < n - 1) {
        const int2 rg = e.range[i];
        const bool alive = (i == 0) || !(B.reach[o + rg.x] >= o + rg.y || B.max_hi[o + rg.x] > o + rg.y);
        if (alive) {
            const int par = (i == 0) ? -1 : new_interior(e, e.parent[i]);
            const float4 mn = nbmin[i], mx = nbmax[i];
            const int size = __float_as_int(mx.w);
            if (i == 0 || e.state[i] == 1) {
                const int l = e.left[i], r = e.right[i];
                put(nodes, new_interior(e, i), max_nodes,
                    hp_make_node(nbmin[l], nbmax[l], nbmin[r], nbmax[r], child_ref(e, l), child_ref(e, r), size, par),
                    B.err);
            } else {
                put(nodes, e.num_int + e.rank_leaf[o + rg.x] - e.base_leaf, max_nodes,
                    hp_make_node(mn, mx, mn, mx, rg.x, rg.y + 1, ~size, par), B.err);
            }
        }
    }
    if (B.reach[g] < g && B.max_hi[g] < g) {
        const int leaf = n - 1 + i;
        const float4 mn = nbmin[leaf], mx = nbmax[leaf];
        const int par = new_interior(e, e.parent[leaf]);
        put(nodes, e.num_int + e.rank_leaf[g] - e.base_leaf, max_nodes,
            hp_make_node(mn, mx, mn, mx, i, i + 1, ~1, par), B.err);
    }
}

}  // namespace

// ---- host side ----------------------------------------------------------------------------

struct hp_batch {
    int device = 0;
    int M = 0;
    int64_t N = 0, R = 0, NN = 0;
    int bits = 30, key_bits = 30;
    hp_build_params params{};
    std::vector<hp_batch_seg> segs;
    std::vector<int64_t> ray_off;        // host copy [M + 1]
    hp_batch_seg* d_seg = nullptr;
    int32_t* d_tri_off = nullptr;        // [M + 1]
    int64_t* d_ray_off = nullptr;        // [M + 1]
    hp_bvh_info* d_info = nullptr;       // [M]
    hp_node_bin* nodes = nullptr;
    float4* woop = nullptr;
    int32_t* tri_idx = nullptr;
    std::vector<hp_bvh_impl> views;
    size_t scratch = 0;
    cudaGraphExec_t exec = nullptr;
    const float* g_rays = nullptr;
    int32_t* g_results = nullptr;
    int32_t* g_stats = nullptr;
    uint32_t g_flags = 0;
    int g_mode = -1;                     // 0 build, 1 trace, 2 both
    const hp_ctx* g_ctx = nullptr;       // context, scratch arena and launch choices of the capture
    const char* g_arena = nullptr;
    int g_tune[4] = {0, 0, 0, 0};
    int64_t graph_launches = 0;
};

namespace {

size_t batch_scratch(const hp_batch& b, hp_sort_plan& plan, int sort_block) {
    const int64_t N = std::max<int64_t>(b.N, 1), NN = std::max<int64_t>(b.NN, 1);
    plan = hp_sort_make_plan(N, 8, b.key_bits, sort_block);
    size_t need = 0;
    need += 2 * hp_carve::pad(N * 16);                 // triangle boxes
    need += 2 * hp_carve::pad(N * 8);                  // keys, sorted keys
    need += hp_carve::pad(plan.scratch_bytes) + hp_carve::pad(hp_sort_hist_bytes(plan.passes));
    need += hp_carve::pad(N * 4);                      // sorted
    need += hp_carve::pad(NN * 4);                     // parent
    need += 2 * hp_carve::pad(N * 4) + hp_carve::pad(N * 8);  // left, right, range
    need += 2 * hp_carve::pad(NN * 16);                // node boxes
    need += hp_carve::pad(N * 4) * 7 + hp_carve::pad(N);  // counters, max_hi, reach, flags x2, ranks x2, state
    need += 2 * hp_scan2_scratch_bytes(N + 1) + hp_carve::pad(64);
    return need;
}

hp_status batch_build_seq(hp_ctx* ctx, hp_batch* b, cudaStream_t s) {
    if (b->N == 0) {
        HP_CUDA(cudaMemsetAsync(b->d_info, 0, sizeof(hp_bvh_info) * b->M, s));
        return HP_OK;
    }
    hp_sort_plan plan;
    batch_scratch(*b, plan, ctx->tune.sort_block);
    hp_carve cv(ctx->arena);
    const int64_t N = b->N, NN = b->NN;
    bargs B{};
    B.seg = b->d_seg;
    B.tri_off = b->d_tri_off;
    B.M = b->M;
    B.N = N;
    B.bits = b->bits;
    hp_sort_hist_digits(plan, &B.hshift, &B.passes);
    B.info = b->d_info;
    B.tbmin = cv.take<float4>(N);
    B.tbmax = cv.take<float4>(N);
    B.keys = cv.take<uint64_t>(N);
    uint64_t* skeys = cv.take<uint64_t>(N);
    B.skeys = skeys;
    void* sort_scratch = cv.take<char>(plan.scratch_bytes);
    B.hist = cv.take<uint32_t>(plan.passes * 256);
    int32_t* sorted = cv.take<int32_t>(N);
    B.sorted = sorted;
    B.parent = cv.take<int>(NN);
    B.left = cv.take<int>(N);
    B.right = cv.take<int>(N);
    B.range = cv.take<int2>(N);
    B.nbmin = cv.take<float4>(NN);
    B.nbmax = cv.take<float4>(NN);
    B.counters = cv.take<int>(N);
    B.max_hi = cv.take<int>(N);
    int* reach = cv.take<int>(N);
    B.reach = reach;
    B.flag_int = cv.take<int>(N);
    B.flag_leaf = cv.take<int>(N);
    int* rank_int = cv.take<int>(N);
    int* rank_leaf = cv.take<int>(N);
    B.rank_int = rank_int;
    B.rank_leaf = rank_leaf;
    B.state = cv.take<uint8_t>(N);
    void* scan_a = cv.take<char>(hp_scan2_scratch_bytes(N + 1));
    void* scan_b = cv.take<char>(hp_scan2_scratch_bytes(N + 1));
    int* totals = cv.take<int>(16);
    B.totals = totals;
    B.nodes = b->nodes;
    B.woop = b->woop;
    B.tri_idx = b->tri_idx;
    B.ct = b->params.ct;
    B.ci = b->params.ci;
    B.adaptive = b->params.adaptive_leaf;
    B.max_leaf = b->params.max_leaf_size;
    B.err = ctx->d_status;
    const int grid = hp_div_up(N, TB);
    const int hist_words = plan.passes * 256;
    k_b_init<<<hp_div_up(std::max<int64_t>(hist_words, b->M), TB), TB, 0, s>>>(B, hist_words);
    HP_CUDA(cudaMemsetAsync(B.counters, 0, N * 4, s));
    HP_CUDA(cudaMemsetAsync(B.max_hi, 0xff, N * 4, s));
    k_b_boxes<<<grid, TB, 0, s>>>(B);
    k_b_morton<<<grid, TB, 0, s>>>(B);
    k_b_scale<<<hp_div_up(b->M, TB), TB, 0, s>>>(B);
    HP_CUDA(cudaGetLastError());
    hp_count_launch(4);
    hp_mark(ctx, s, "batch_keys");
    hp_sort_args sa{B.keys, nullptr, skeys, sorted, sort_scratch, B.hist, true, ctx->d_status, ctx};
    HP_TRY(hp_sort_run(plan, sa, s));
    k_b_karras<<<grid, TB, 0, s>>>(B);
    k_b_climb<<<grid, TB, 0, s>>>(B);
    HP_CUDA(cudaGetLastError());
    hp_count_launch(2);
    hp_mark(ctx, s, "batch_climb");
    hp_scan_max_excl(B.max_hi, N, reach, scan_a, ctx->d_status, s);
    k_b_flags<<<grid, TB, 0, s>>>(B);
    hp_scan2_sum(B.flag_int, N, B.flag_leaf, N, rank_int, rank_leaf, totals, scan_b, ctx->d_status, s);
    k_b_counts<<<hp_div_up(b->M, TB), TB, 0, s>>>(B);
    k_b_emit<<<grid, TB, 0, s>>>(B);
    HP_CUDA(cudaGetLastError());
    hp_count_launch(3);
    hp_mark(ctx, s, "batch_collapse");
    return HP_OK;
}

hp_status batch_trace_seq(hp_ctx* ctx, hp_batch* b, const float* rays, int32_t* results, int32_t* stats,
                          uint32_t flags, cudaStream_t s) {
    hp_batch_trace_args t{};
    t.rays = rays;
    t.num_rays = b->R;
    t.results = results;
    t.stats = stats;
    t.nodes = b->nodes;
    t.woop = b->woop;
    t.tri_idx = b->tri_idx;
    t.segs = b->d_seg;
    t.ray_off = b->d_ray_off;
    t.num_segs = b->M;
    HP_TRY(hp_trace_batch_launch(ctx, t, flags, s));
    hp_mark(ctx, s, "batch_trace");
    return HP_OK;
}

void drop_graph(hp_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    b->g_mode = -1;
}

// Run the build and/or trace sequence, from a CUDA graph unless HP_BATCH_NO_GRAPH.
hp_status batch_run(hp_ctx* ctx, hp_batch* b, int mode, const float* rays, int32_t* results, int32_t* stats,
                    uint32_t flags, cudaStream_t s) {
    const bool use_graph = !(flags & HP_BATCH_NO_GRAPH) && !ctx->profiling;
    auto seq = [&]() -> hp_status {
        if (mode != 1) HP_TRY(batch_build_seq(ctx, b, s));
        if (mode != 0 && b->R > 0) HP_TRY(batch_trace_seq(ctx, b, rays, results, stats, flags, s));
        return HP_OK;
    };
    if (!use_graph) return seq();
    if (s == nullptr) return hp_fail(HP_ERR_ARG, "batched launches from a CUDA graph need a non-default stream");
    const uint32_t gflags = flags & (HP_TRACE_ANY_HIT | HP_TRACE_STATS);
    if (!b->exec || b->g_mode != mode || b->g_rays != rays || b->g_results != results || b->g_stats != stats ||
        b->g_flags != gflags || b->g_ctx != ctx || b->g_arena != ctx->arena ||
        b->g_tune[0] != ctx->tune.sort_block || b->g_tune[1] != ctx->tune.trace_ctas_per_sm ||
        b->g_tune[2] != ctx->tune.trace_stack) {
        drop_graph(b);
        cudaGraph_t graph = nullptr;
        HP_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        const int64_t l0 = hp_launch_count();
        const hp_status st = seq();
        cudaError_t e = cudaStreamEndCapture(s, &graph);
        if (st != HP_OK) {
            if (graph) cudaGraphDestroy(graph);
            return st;
        }
        if (e != cudaSuccess) return hp_cuda_fail(e, "cudaStreamEndCapture");
        b->graph_launches = hp_launch_count() - l0;
        e = cudaGraphInstantiate(&b->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            b->exec = nullptr;
            return hp_cuda_fail(e, "cudaGraphInstantiate");
        }
        b->g_mode = mode;
        b->g_rays = rays;
        b->g_results = results;
        b->g_stats = stats;
        b->g_flags = gflags;
        b->g_ctx = ctx;
        b->g_arena = ctx->arena;
        b->g_tune[0] = ctx->tune.sort_block;
        b->g_tune[1] = ctx->tune.trace_ctas_per_sm;
        b->g_tune[2] = ctx->tune.trace_stack;
        hp_count_launch(-(int)b->graph_launches);  // counted when the graph runs
    }
    HP_CUDA(cudaGraphLaunch(b->exec, s));
    hp_count_launch((int)b->graph_launches);
    return HP_OK;
}

}  // namespace

hp_status hp_batch_create(hp_ctx* ctx, const hp_mesh* meshes, int32_t num_meshes, const int64_t* rays_per_mesh,
                          const hp_build_params* p, hp_batch** out) {
    if (!ctx || !out || (!meshes && num_meshes > 0) || num_meshes < 0 || !p)
        return hp_fail(HP_ERR_ARG, "hp_batch_create: null or negative argument");
    *out = nullptr;
    if (p->method != HP_METHOD_LBVH)
        return hp_fail(HP_ERR_UNSUPPORTED, "batched builds use the LBVH method");
    if (p->layout != 0 && p->layout != HP_LAYOUT_BIN)
        return hp_fail(HP_ERR_UNSUPPORTED, "batched builds use the binary layout");
    if (p->morton_bits < 6 || p->morton_bits > 60) return hp_fail(HP_ERR_ARG, "morton_bits must be in [6,60]");
    if (p->ct <= 0.0f || p->ci <= 0.0f) return hp_fail(HP_ERR_ARG, "ct and ci must be positive");
    if (p->max_leaf_size <= 0 || p->max_leaf_size > 1024) return hp_fail(HP_ERR_ARG, "max_leaf_size must be in (0,1024]");
    int mbits = 0;
    while ((1 << mbits) < std::max(num_meshes, 1)) ++mbits;
    if (p->morton_bits + mbits > 64)
        return hp_fail(HP_ERR_UNSUPPORTED, "batched build: Morton bits + log2(meshes) must fit in 64 bits");
    hp_batch* b = new hp_batch();
    b->device = ctx->device;
    b->M = num_meshes;
    b->params = *p;
    b->bits = p->morton_bits;
    b->key_bits = p->morton_bits + mbits;
    b->segs.resize(num_meshes);
    b->ray_off.resize(num_meshes + 1);
    std::vector<int32_t> tri_off(num_meshes + 1);
    int64_t N = 0, NN = 0, R = 0;
    for (int m = 0; m < num_meshes; ++m) {
        const hp_mesh& me = meshes[m];
        const int64_t rays = rays_per_mesh ? rays_per_mesh[m] : 0;
        if (me.num_triangles < 0 || me.num_vertices < 0 || rays < 0 ||
            (me.num_triangles > 0 && (!me.vertices || !me.triangles))) {
            delete b;
            return hp_fail(HP_ERR_ARG, "hp_batch_create: mesh " + std::to_string(m) + " is invalid");
        }
        hp_batch_seg& g = b->segs[m];
        g.verts = me.vertices;
        g.tris = me.triangles;
        g.nv = me.num_vertices;
        g.n = (int32_t)me.num_triangles;
        g.tri_off = (int32_t)N;
        g.node_off = NN;
        g.ray_off = R;
        tri_off[m] = (int32_t)N;
        b->ray_off[m] = R;
        N += me.num_triangles;
        NN += std::max<int64_t>(2 * me.num_triangles - 1, 3);
        R += rays;
        if (N >= (int64_t(1) << 30)) {
            delete b;
            return hp_fail(HP_ERR_ARG, "hp_batch_create: more than 2^30 triangles in a batch");
        }
    }
    tri_off[num_meshes] = (int32_t)N;
    b->ray_off[num_meshes] = R;
    b->N = N;
    b->NN = NN;
    b->R = R;
    cudaError_t e = cudaSuccess;
    const size_t M1 = (size_t)num_meshes + 1;
    if (e == cudaSuccess) e = cudaMalloc(&b->d_seg, std::max<size_t>(num_meshes, 1) * sizeof(hp_batch_seg));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_tri_off, M1 * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_ray_off, M1 * sizeof(int64_t));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_info, std::max<size_t>(num_meshes, 1) * sizeof(hp_bvh_info));
    if (e == cudaSuccess) e = cudaMalloc(&b->nodes, std::max<int64_t>(NN, 1) * sizeof(hp_node_bin));
    if (e == cudaSuccess) e = cudaMalloc(&b->woop, std::max<int64_t>(3 * N, 1) * sizeof(float4));
    if (e == cudaSuccess) e = cudaMalloc(&b->tri_idx, std::max<int64_t>(N, 1) * sizeof(int32_t));
    if (e == cudaSuccess && num_meshes > 0)
        e = cudaMemcpy(b->d_seg, b->segs.data(), num_meshes * sizeof(hp_batch_seg), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_tri_off, tri_off.data(), M1 * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(b->d_ray_off, b->ray_off.data(), M1 * sizeof(int64_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaGetLastError();
        hp_batch_destroy(b);
        return e == cudaErrorMemoryAllocation ? hp_fail(HP_ERR_OOM, "hp_batch_create: out of device memory")
                                              : hp_cuda_fail(e, "hp_batch_create");
    }
    b->views.resize(num_meshes);
    for (int m = 0; m < num_meshes; ++m) {
        hp_bvh_impl& v = b->views[m];
        v.nodes = b->nodes + b->segs[m].node_off;
        v.woop = b->woop + 3 * (int64_t)b->segs[m].tri_off;
        v.tri_idx = b->tri_idx + b->segs[m].tri_off;
        v.counters = nullptr;
        v.info = b->d_info + m;
        v.capacity = b->segs[m].n;
        v.view = true;
    }
    // reserve the scratch now (for either sort CTA size): nothing may allocate
    // inside a graph capture
    hp_sort_plan plan;
    b->scratch = std::max(batch_scratch(*b, plan, 512), batch_scratch(*b, plan, 256));
    const hp_status st = hp_ctx_reserve(ctx, b->scratch, nullptr);
    if (st != HP_OK) {
        hp_batch_destroy(b);
        return st;
    }
    *out = b;
    return HP_OK;
}

hp_status hp_batch_destroy(hp_batch* b) {
    if (!b) return HP_OK;
    drop_graph(b);
    cudaFree(b->d_seg);
    cudaFree(b->d_tri_off);
    cudaFree(b->d_ray_off);
    cudaFree(b->d_info);
    cudaFree(b->nodes);
    cudaFree(b->woop);
    cudaFree(b->tri_idx);
    delete b;
    return HP_OK;
}

hp_status hp_batch_info(const hp_batch* b, int32_t* num_meshes, int64_t* num_triangles, int64_t* num_rays) {
    if (!b) return hp_fail(HP_ERR_ARG, "hp_batch_info: null batch");
    if (num_meshes) *num_meshes = b->M;
    if (num_triangles) *num_triangles = b->N;
    if (num_rays) *num_rays = b->R;
    return HP_OK;
}

hp_status hp_batch_ray_offset(const hp_batch* b, int32_t mesh, int64_t* offset) {
    if (!b || !offset || mesh < 0 || mesh > b->M) return hp_fail(HP_ERR_ARG, "hp_batch_ray_offset: bad argument");
    *offset = b->ray_off[mesh];
    return HP_OK;
}

hp_status hp_batch_build(hp_ctx* ctx, hp_batch* b, uint32_t flags, void* stream) {
    if (!ctx || !b) return hp_fail(HP_ERR_ARG, "hp_batch_build: null argument");
    hp_nvtx_range nvtx_("hp_batch_build");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    HP_TRY(hp_ctx_reserve(ctx, b->scratch, s));
    HP_TRY(batch_run(ctx, b, 0, nullptr, nullptr, nullptr, flags, s));
    if (hp_checking(ctx, s)) HP_TRY(hp_ctx_check(ctx, stream));
    return HP_OK;
}

hp_status hp_batch_trace(hp_ctx* ctx, hp_batch* b, const float* rays, int32_t* results, int32_t* stats,
                         uint32_t flags, void* stream) {
    if (!ctx || !b || (b->R > 0 && (!rays || !results))) return hp_fail(HP_ERR_ARG, "hp_batch_trace: null argument");
    hp_nvtx_range nvtx_("hp_batch_trace");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    HP_TRY(batch_run(ctx, b, 1, rays, results, stats, flags, s));
    if (hp_checking(ctx, s)) HP_TRY(hp_ctx_check(ctx, stream));
    return HP_OK;
}

hp_status hp_batch_build_trace(hp_ctx* ctx, hp_batch* b, const float* rays, int32_t* results, int32_t* stats,
                               uint32_t flags, void* stream) {
    if (!ctx || !b || (b->R > 0 && (!rays || !results)))
        return hp_fail(HP_ERR_ARG, "hp_batch_build_trace: null argument");
    hp_nvtx_range nvtx_("hp_batch_build_trace");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    HP_TRY(hp_ctx_reserve(ctx, b->scratch, s));
    HP_TRY(batch_run(ctx, b, 2, rays, results, stats, flags, s));
    if (hp_checking(ctx, s)) HP_TRY(hp_ctx_check(ctx, stream));
    return HP_OK;
}

hp_status hp_batch_bvh(hp_batch* b, int32_t mesh, hp_bvh* out) {
    if (!b || !out || mesh < 0 || mesh >= b->M) return hp_fail(HP_ERR_ARG, "hp_batch_bvh: bad argument");
    std::memset(out, 0, sizeof(*out));
    hp_bvh_impl& v = b->views[mesh];
    out->nodes = v.nodes;
    out->woop = v.woop;
    out->tri_indices = v.tri_idx;
    out->num_refs = b->segs[mesh].n;
    out->capacity_refs = b->segs[mesh].n;
    out->num_interior = out->num_leaf = -1;
    out->method = HP_METHOD_LBVH;
    out->ct = b->params.ct;
    out->ci = b->params.ci;
    out->impl = &v;
    out->layout = HP_LAYOUT_BIN;
    out->node_bytes = 64;
    return HP_OK;
}
