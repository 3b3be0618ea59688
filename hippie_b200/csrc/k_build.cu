// LBVH construction: triangle boxes and scene box, Morton keys, radix sort,
// Karras hierarchy emission, one bottom-up climb that refits boxes, counts
// subtree sizes, evaluates the SAH collapse rule and woopifies triangles, and
// a collapse into the reference's 64-byte binary node layout.
//
// Reference path (src/hippie/): LBVHBuilder::build rt/bvh/LBVHBuilder.cpp:183-241
//   setupBoxes            rt/bvh/LBVHBuilderKernels.cu:65-98
//   computeMortonCodes60  rt/bvh/LBVHBuilderKernels.cu:131-160
//   RadixSort::sort       radix_sort/RadixSort.cpp:181-238
//   setupLeaves           rt/bvh/LBVHBuilderKernels.cu:162-195
//   construct60           rt/bvh/LBVHBuilderKernels.cu:11-63,226-252
//   refit                 rt/bvh/LBVHBuilderKernels.cu:254-305
//   BVHCollapser::collapseAdaptive rt/bvh/BVHCollapser.cpp:521-597 and its kernels
//                         rt/bvh/BVHCollapserKernels.cu:11-526
//   woopifyTriangles      rt/bvh/HipBVHKernels.cu:12-65
//
// Collapse numbering. The reference numbers the collapsed tree breadth-first
// with global atomics, so its node order depends on scheduling. Here every
// node of an LBVH covers a contiguous range [lo, hi] of sorted references, so
// the collapse is decided and numbered without any top-down pass:
//   * a node is removed iff a state-0 ("better as a leaf") node strictly
//     contains its range; state-0 ranges are scattered as maxHi[lo] = hi and
//     an exclusive max-scan over positions answers that query for any range;
//   * surviving interior nodes are numbered in order of their split position
//     (in-order), with the root moved to index 0; leaves are numbered by the
//     first sorted reference they hold;
//   * each collapsed leaf holds a contiguous range of sorted references, so
//     the sorted triangle order is already leaf-contiguous and no reordering
//     pass is needed.
// The tree this produces is the reference's tree up to node numbering and the
// order of triangles inside a leaf (which the reference leaves to atomics).
#include <algorithm>
#include <cuda_runtime.h>
#include "hp_device.cuh"
#include "hp_internal.h"

namespace {

constexpr int TB = 256;

// Per-triangle boxes (setupBoxes) and the scene box as their union
// (SceneLoader.cpp:144-153 computes it over triangle boxes at load time).
// woop (or null): the Woop rows of every triangle, in scene order, computed
// here from the vertices the boxes read anyway (the collapse then gathers one
// 48-byte record per reference instead of the triangle and its vertices).
__global__ void __launch_bounds__(TB) k_tri_boxes(const float* __restrict__ verts, int64_t nv,
                                                  const int32_t* __restrict__ tris, int64_t n,
                                                  float4* __restrict__ bmin, float4* __restrict__ bmax,
                                                  uint32_t* box_ord, int* err, float4* __restrict__ woop = nullptr) {
    float mn[3] = {HP_MAX_FLOAT, HP_MAX_FLOAT, HP_MAX_FLOAT};
    float mx[3] = {-HP_MAX_FLOAT, -HP_MAX_FLOAT, -HP_MAX_FLOAT};
    for (int64_t i = blockIdx.x * (int64_t)TB + threadIdx.x; i < n; i += (int64_t)gridDim.x * TB) {
        tri_verts t = load_tri(verts, nv, tris, i, err);
        float ax = fminf(fminf(t.x0, t.x1), t.x2), ay = fminf(fminf(t.y0, t.y1), t.y2),
              az = fminf(fminf(t.z0, t.z1), t.z2);
        float bx = fmaxf(fmaxf(t.x0, t.x1), t.x2), by = fmaxf(fmaxf(t.y0, t.y1), t.y2),
              bz = fmaxf(fmaxf(t.z0, t.z1), t.z2);
        bmin[2 * i] = make_float4(ax, ay, az, 0.0f);  // min / max interleaved (32 B per triangle)
        bmax[2 * i] = make_float4(bx, by, bz, 0.0f);
        if (woop) {
            float4 w0, w1, w2;
            hp_woop(t.x0, t.y0, t.z0, t.x1, t.y1, t.z1, t.x2, t.y2, t.z2, w0, w1, w2);
            woop[3 * i] = w0;
            woop[3 * i + 1] = w1;
            woop[3 * i + 2] = w2;
        }
        mn[0] = fminf(mn[0], ax); mn[1] = fminf(mn[1], ay); mn[2] = fminf(mn[2], az);
        mx[0] = fmaxf(mx[0], bx); mx[1] = fmaxf(mx[1], by); mx[2] = fmaxf(mx[2], bz);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            mn[k] = fminf(mn[k], __shfl_xor_sync(HP_FULL_MASK, mn[k], o));
            mx[k] = fmaxf(mx[k], __shfl_xor_sync(HP_FULL_MASK, mx[k], o));
        }
    }
    __shared__ float s[TB / 32][6];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
        for (int k = 0; k < 3; ++k) { s[warp][k] = mn[k]; s[warp][3 + k] = mx[k]; }
    __syncthreads();
    if (threadIdx.x < 6) {
        int k = threadIdx.x;
        float r = s[0][k];
        for (int w = 1; w < TB / 32; ++w) r = (k < 3) ? fminf(r, s[w][k]) : fmaxf(r, s[w][k]);
        if (k < 3) atomicMin(&box_ord[k], hp_f2ord(r));
        else atomicMax(&box_ord[k], hp_f2ord(r));
    }
}

__global__ void k_init_build(hp_bvh_info* info, uint32_t* hist, int hist_words) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < hist_words) hist[i] = 0;
    if (i < 6) info->box_ord[i] = (i < 3) ? 0xffffffffu : 0u;
    if (i == 0) { info->num_interior = 0; info->num_leaf = 0; }
}

// Morton keys (computeMortonCodes60) fused with the radix sort's per-pass digit
// histograms. scale = 1/diagonal is taken with __fdividef, the approximate
// quotient the reference's fast-math JIT build produces for `1.0f / diag`.
template <typename K>
__global__ void __launch_bounds__(TB) k_morton(const float4* __restrict__ bmin,
                                               const float4* __restrict__ bmax, int64_t n,
                                               hp_bvh_info* info, int bits, int hshift, int passes,
                                               K* __restrict__ keys, uint32_t* hist) {
    __shared__ uint32_t sh[8 * 256];
    for (int i = threadIdx.x; i < passes * 256; i += TB) sh[i] = 0;
    float smin[3], scale[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        smin[k] = hp_ord2f(info->box_ord[k]);
        float d = __fsub_rn(hp_ord2f(info->box_ord[3 + k]), smin[k]);
        scale[k] = __fdividef(1.0f, d);
    }
    if (blockIdx.x == 0 && threadIdx.x < 3) info->scale[threadIdx.x] = scale[threadIdx.x];
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)TB + threadIdx.x; i < n; i += (int64_t)gridDim.x * TB) {
        float4 a = bmin[2 * i], b = bmax[2 * i];
        uint64_t key = hp_morton_key(a.x, a.y, a.z, b.x, b.y, b.z, smin, scale, bits);
        keys[i] = (K)key;
        for (int p = 0; p < passes; ++p) {  // the sort's digits (hp_sort_hist_digits)
            const int sh_p = hshift + 8 * p, w = min(8, bits - sh_p);
            atomicAdd(&sh[p * 256 + (uint32_t)((key >> sh_p) & ((1u << w) - 1u))], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += TB)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// delta (rt/bvh/HipBVHUtil.h:17-33): common prefix length of keys i and j, with
// the index prefix appended for equal keys; -1 outside [0, n).
template <typename K> __device__ __forceinline__ int kdelta(const K* k, int n, int i, int j);
template <> __device__ __forceinline__ int kdelta<uint64_t>(const uint64_t* k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    uint64_t a = __ldg(k + i), b = __ldg(k + j);
    if (a != b) return __clzll((long long)(a ^ b));
    return __clzll((long long)(i ^ j)) + 64;
}
template <> __device__ __forceinline__ int kdelta<uint32_t>(const uint32_t* k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    uint32_t a = __ldg(k + i), b = __ldg(k + j);
    if (a != b) return __clz((int)(a ^ b));
    return __clz(i ^ j) + 32;
}

// Karras 2012 radix-tree emission (construct<T>, LBVHBuilderKernels.cu:11-63).
// Interior node i covers [min(i,j), max(i,j)] and splits after gamma; a child
// is a leaf (index + n-1) when its range has one reference.
template <typename K>
__global__ void __launch_bounds__(TB) k_karras(const K* __restrict__ keys, int n, int* parent,
                                               int* left, int* right, int2* range) {
    const int i = blockIdx.x * TB + threadIdx.x;
    if (i == 0) parent[0] = -1;
    if (i >= n - 1) return;
    const int dr = kdelta(keys, n, i, i + 1), dl = kdelta(keys, n, i, i - 1);
    const int d = (dr - dl > 0) - (dr - dl < 0);
    const int dmin = kdelta(keys, n, i, i - d);
    int lmax = 2;
    while (kdelta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (kdelta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = kdelta(keys, n, i, j);
    int s = 0, k = 2, t;
    do {
        t = (l + k - 1) / k;
        k <<= 1;
        if (kdelta(keys, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    const int gamma = i + s * d + min(d, 0);
    int lc = gamma, rc = gamma + 1;
    if (min(i, j) == gamma) lc += n - 1;
    if (max(i, j) == gamma + 1) rc += n - 1;
    left[i] = lc;
    right[i] = rc;
    parent[lc] = i;
    parent[rc] = i;
    range[i] = make_int2(min(i, j), max(i, j));
}

// Leaf records, one thread per sorted reference p (leaf node n-1+p): the Woop
// rows of its triangle (HipBVH::woopifyTriangles, rt/bvh/HipBVHKernels.cu:35-65),
// the leaf box (setupLeaves, rt/bvh/LBVHBuilderKernels.cu:162-195), its leaf
// cost ci*A and size 1. Node boxes keep the cost in min.w and the size (as int
// bits) in max.w. Coalesced stores; the triangle gather is the only random
// access.
__global__ void __launch_bounds__(TB) k_leaves(
    int n, const int32_t* __restrict__ sorted_tri, const float* __restrict__ verts, int64_t nv,
    const int32_t* __restrict__ tris, float4* __restrict__ nbmin, float4* __restrict__ nbmax,
    float4* __restrict__ woop, float ci, int adaptive, int* err) {
    const int p = blockIdx.x * TB + threadIdx.x;
    if (p >= n) return;
    const int tri = __ldg(sorted_tri + p);
    tri_verts t = load_tri(verts, nv, tris, tri, err);
    float4 w0, w1, w2;
    hp_woop(t.x0, t.y0, t.z0, t.x1, t.y1, t.z1, t.x2, t.y2, t.z2, w0, w1, w2);
    woop[3 * (int64_t)p + 0] = w0;
    woop[3 * (int64_t)p + 1] = w1;
    woop[3 * (int64_t)p + 2] = w2;
    float ax = fminf(fminf(t.x0, t.x1), t.x2), ay = fminf(fminf(t.y0, t.y1), t.y2),
          az = fminf(fminf(t.z0, t.z1), t.z2);
    float bx = fmaxf(fmaxf(t.x0, t.x1), t.x2), by = fmaxf(fmaxf(t.y0, t.y1), t.y2),
          bz = fmaxf(fmaxf(t.z0, t.z1), t.z2);
    const float cost = adaptive ? __fmul_rn(ci, hp_area(ax, ay, az, bx, by, bz)) : 0.0f;
    nbmin[n - 1 + p] = make_float4(ax, ay, az, cost);
    nbmax[n - 1 + p] = make_float4(bx, by, bz, __int_as_float(1));
}

// Bottom-up refit (refit, rt/bvh/LBVHBuilderKernels.cu:254-305). A thread
// arriving first at a node leaves; the second merges the children's boxes,
// sums sizes and evaluates the collapse rule of computeNodeStatesAdaptive
// (BVHCollapserKernels.cu:58-136):
//   leaf cost = ci*A, interior cost = ct*A + c(left) + c(right),
//   state 0 (collapse into a leaf) iff ci*A*size < interior cost;
// or, without adaptive leaves, computeNodeStates (:138-184): size <= maxLeafSize.
//
// Two phases, so that almost all memory traffic is coalesced. Every LBVH node
// covers a contiguous range [lo, hi] of sorted leaves and its index lies in
// that range; a CTA owning the CB = 512 leaves [base, base + CB) therefore owns every node
// whose range lies inside its own ("local" nodes: their indices, children and
// boxes are all in [base, base + CB)). Phase A (k_climb_local) loads the
// CTA's node indices and leaf boxes with coalesced loads, climbs the local
// nodes with shared-memory arrival counters and boxes (block-scope ordering),
// and writes their boxes, states and maxHi words back with coalesced stores;
// a thread whose next node is not local stops and appends its child to the
// frontier list. (Computing the local nodes in barrier-separated rounds
// instead was slower: the CTAs' local subtrees are deep.) Phase B
// (k_climb_frontier) climbs from the frontier entries through the non-local
// nodes (those whose ranges cross a CTA boundary: about depth per boundary)
// with the global counters and one acq_rel atomic per arrival.
constexpr int CB = 512;
constexpr size_t CLIMB_SMEM = (size_t)CB * (4 * sizeof(float4) + 7 * sizeof(int) + sizeof(int2)) + 2 * sizeof(int);

struct climb_args {
    int n;
    const int* parent;
    const int* left;
    const int* right;
    const int2* range;
    float4* nbmin;
    float4* nbmax;
    int* counters;     // arrivals at non-local nodes (zeroed)
    int* max_hi;       // maxHi words (initialised to -1)
    uint8_t* state;
    int* frontier;     // children whose parent is not local to their CTA
    unsigned* frontier_count;
    float ct, ci;
    int adaptive, max_leaf;
    int* err;
};

// Box, cost, size and state of a node from its left (l*) and right (r*) children.
__device__ __forceinline__ int merge_node(const climb_args& A, float4 lmn, float4 lmx, float4 rmn, float4 rmx,
                                          float4& omn, float4& omx) {
    const float mnx = fminf(lmn.x, rmn.x), mny = fminf(lmn.y, rmn.y), mnz = fminf(lmn.z, rmn.z);
    const float mxx = fmaxf(lmx.x, rmx.x), mxy = fmaxf(lmx.y, rmx.y), mxz = fmaxf(lmx.z, rmx.z);
    const int size = __float_as_int(lmx.w) + __float_as_int(rmx.w);
    int st;
    float c;
    if (A.adaptive) {
        const float area = hp_area(mnx, mny, mnz, mxx, mxy, mxz);
        const float c_int = __fadd_rn(__fmaf_rn(A.ct, area, lmn.w), rmn.w);
        const float c_leaf = __fmul_rn(__fmul_rn(A.ci, area), (float)size);
        st = (c_leaf < c_int) ? 0 : 1;
        c = st ? c_int : c_leaf;
    } else {
        st = (size <= A.max_leaf) ? 0 : 1;
        c = 0.0f;
    }
    omn = make_float4(mnx, mny, mnz, c);
    omx = make_float4(mxx, mxy, mxz, __int_as_float(size));
    return st;
}

__global__ void __launch_bounds__(CB, 4) k_climb_local(climb_args A) {
    extern __shared__ __align__(16) unsigned char climb_smem[];
    float4* s_imn = reinterpret_cast<float4*>(climb_smem);  // local interior node base + k
    float4* s_imx = s_imn + CB;
    float4* s_lmn = s_imx + CB;                             // leaf base + k
    float4* s_lmx = s_lmn + CB;
    int2* s_rng = reinterpret_cast<int2*>(s_lmx + CB);      // ranges of nodes base + k
    int* s_cnt = reinterpret_cast<int*>(s_rng + CB);        // arrivals at local nodes
    int* s_left = s_cnt + CB;
    int* s_right = s_left + CB;
    int* s_up = s_right + CB;                               // parents of nodes base + k
    int* s_mh = s_up + CB;                                  // maxHi of positions base + k
    int* s_st = s_mh + CB;                                  // state of local nodes
    int* s_front = s_st + CB;                               // this CTA's frontier entries
    int* s_fn = s_front + CB;                               // [0] their count, [1] their offset
    const int n = A.n;
    const int base = blockIdx.x * CB, k = threadIdx.x, p = base + k;
    const int last = min(base + CB, n) - 1;  // this CTA's last leaf
    s_cnt[k] = 0;
    s_mh[k] = -1;
    if (k == 0) s_fn[0] = 0;
    if (p < n - 1) {
        s_left[k] = __ldg(A.left + p);
        s_right[k] = __ldg(A.right + p);
        s_up[k] = __ldg(A.parent + p);
        s_rng[k] = __ldg(A.range + p);
    } else {
        s_rng[k] = make_int2(-1, -1);  // not an interior node: never local
    }
    float4 cmn = make_float4(0.0f, 0.0f, 0.0f, 0.0f), cmx = cmn;
    int node = -1;
    if (p < n) {
        cmn = A.nbmin[n - 1 + p];
        cmx = A.nbmax[n - 1 + p];
        s_lmn[k] = cmn;
        s_lmx[k] = cmx;
        node = __ldg(A.parent + n - 1 + p);
    }
    __syncthreads();
    int child = n - 1 + p;
    int guard = 0;
    while (p < n && node >= 0) {
        const int kn = node - base;
        const int2 rg = ((unsigned)kn < (unsigned)CB) ? s_rng[kn] : make_int2(-1, -1);
        if (!(rg.x >= base && rg.y <= last && kn <= rg.y - base && kn >= rg.x - base)) {
            // the next node's range crosses the CTA's: phase B continues from
            // child (collected here, one global reservation per CTA below)
            s_front[atomicAdd(s_fn, 1)] = child;  // one entry per leaf thread at most
            break;
        }
        if (++guard > CB) {
            hp_report(A.err, HP_DEV_BAD_INDEX, node);
            break;
        }
        const int l = s_left[kn], r = s_right[kn];
        if (l != child && r != child) {
            hp_report(A.err, HP_DEV_BAD_INDEX, node);
            break;
        }
        const bool is_left = l == child;
        const int sib = is_left ? r : l;
        const int ks = (sib >= n - 1) ? sib - (n - 1) - base : sib - base;
        if ((unsigned)ks >= (unsigned)CB) {
            hp_report(A.err, HP_DEV_BAD_INDEX, node);
            break;
        }
        __threadfence_block();
        if (atomicAdd(&s_cnt[kn], 1) == 0) break;
        __threadfence_block();
        const float4 smn = sib >= n - 1 ? s_lmn[ks] : s_imn[ks];
        const float4 smx = sib >= n - 1 ? s_lmx[ks] : s_imx[ks];
        float4 omn, omx;
        const int st = is_left ? merge_node(A, cmn, cmx, smn, smx, omn, omx)
                               : merge_node(A, smn, smx, cmn, cmx, omn, omx);
        s_imn[kn] = omn;
        s_imx[kn] = omx;
        s_st[kn] = st;
        if (st == 0 && node != 0) atomicMax(&s_mh[rg.x - base], rg.y);
        cmn = omn;
        cmx = omx;
        child = node;
        node = s_up[kn];
    }
    __syncthreads();
    if (k == 0) s_fn[1] = s_fn[0] ? (int)atomicAdd(A.frontier_count, (unsigned)s_fn[0]) : 0;
    __syncthreads();
    for (int i = k; i < s_fn[0]; i += CB) A.frontier[s_fn[1] + i] = s_front[i];
    // write back the local nodes (index base + k) and the maxHi words of the
    // CTA's positions; phase B raises maxHi further with global atomics
    const int2 rg = s_rng[k];
    if (p < n - 1 && rg.x >= base && rg.y <= last) {
        __stcg(A.nbmin + p, s_imn[k]);
        __stcg(A.nbmax + p, s_imx[k]);
        A.state[p] = (uint8_t)s_st[k];
    }
    if (p < n && s_mh[k] >= 0) A.max_hi[p] = s_mh[k];
}

__global__ void __launch_bounds__(TB) k_climb_frontier(climb_args A) {
    const unsigned count = *A.frontier_count;
    const int n = A.n;
    for (unsigned e = blockIdx.x * TB + threadIdx.x; e < count; e += gridDim.x * TB) {
        int child = A.frontier[e];
        if ((unsigned)child >= (unsigned)(2 * n - 1)) {
            hp_report(A.err, HP_DEV_BAD_INDEX, child);
            continue;
        }
        float4 cmn = __ldcg(A.nbmin + child), cmx = __ldcg(A.nbmax + child);
        int node = __ldg(A.parent + child);
        int guard = 0;
        while (node >= 0) {
            if (node >= n - 1 || ++guard > n) {
                hp_report(A.err, HP_DEV_BAD_INDEX, node);
                break;
            }
            const int l = __ldg(A.left + node), r = __ldg(A.right + node), up = __ldg(A.parent + node);
            const int2 rg = __ldg(A.range + node);
            if (hp_arrive(&A.counters[node]) == 0) break;
            if ((unsigned)l >= (unsigned)(2 * n - 1) || (unsigned)r >= (unsigned)(2 * n - 1) ||
                (l != child && r != child)) {
                hp_report(A.err, HP_DEV_BAD_INDEX, node);
                break;
            }
            const bool is_left = l == child;
            const int sib = is_left ? r : l;
            const float4 smn = __ldcg(A.nbmin + sib), smx = __ldcg(A.nbmax + sib);
            float4 omn, omx;
            const int st = is_left ? merge_node(A, cmn, cmx, smn, smx, omn, omx)
                                   : merge_node(A, smn, smx, cmn, cmx, omn, omx);
            __stcg(A.nbmin + node, omn);
            __stcg(A.nbmax + node, omx);
            A.state[node] = (uint8_t)st;
            if (st == 0 && node != 0) atomicMax(&A.max_hi[rg.x], rg.y);
            cmn = omn;
            cmx = omx;
            child = node;
            node = up;
        }
    }
}

__device__ __forceinline__ int split_of(const int* left, int n, int i) {
    int l = left[i];
    return l >= n - 1 ? l - (n - 1) : l;
}

// Collapse flags: interior split gamma survives as an interior node; sorted
// position p starts a leaf of the collapsed tree.
__global__ void __launch_bounds__(TB) k_collapse_flags(int n, const int* __restrict__ left,
                                                       const int2* __restrict__ range,
                                                       const uint8_t* __restrict__ state,
                                                       const int* __restrict__ max_hi,
                                                       const int* __restrict__ reach,
                                                       int* flag_int, int* flag_leaf) {
    const int t = blockIdx.x * TB + threadIdx.x;
    if (t < n - 1) {
        const int2 rg = range[t];
        const bool alive = (t == 0) || !(reach[rg.x] >= rg.y || max_hi[rg.x] > rg.y);
        flag_int[split_of(left, n, t)] = (alive && (t == 0 || state[t] == 1)) ? 1 : 0;
    } else if (t < 2 * n - 1) {
        const int p = t - (n - 1);
        flag_leaf[p] = (reach[p] < p) ? 1 : 0;
    }
}

struct emit_ctx {
    int n;
    const int* left;
    const int* right;
    const int* parent;
    const int2* range;
    const uint8_t* state;
    const int* rank_int;
    const int* rank_leaf;
    const float4* nbmin;
    const float4* nbmax;
    int root_rank;
    int num_int;
};

__device__ __forceinline__ int new_interior(const emit_ctx& e, int i) {
    if (i == 0) return 0;
    int r = e.rank_int[split_of(e.left, e.n, i)];
    return r < e.root_rank ? r + 1 : r;
}

// Encoded child reference of a surviving interior node: interior index, or
// ~(leaf node index) for a leaf child.
__device__ __forceinline__ int child_ref(const emit_ctx& e, int c) {
    if (c >= e.n - 1) return ~(e.num_int + e.rank_leaf[c - (e.n - 1)]);
    if (e.state[c] == 0) return ~(e.num_int + e.rank_leaf[e.range[c].x]);
    return new_interior(e, c);
}

__device__ __forceinline__ void put_node(hp_node_bin* nodes, int idx, int max_nodes,
                                         const hp_node_bin& nd, int* err) {
    if ((unsigned)idx < (unsigned)max_nodes) nodes[idx] = nd;
    else hp_report(err, HP_DEV_BAD_INDEX, idx);
}

__global__ void __launch_bounds__(TB) k_emit(emit_ctx e, const int* __restrict__ max_hi,
                                             const int* __restrict__ reach, hp_bvh_info* info,
                                             hp_node_bin* __restrict__ nodes, int max_nodes, int* err) {
    const int t = blockIdx.x * TB + threadIdx.x;
    const int n = e.n;
    if (t >= 2 * n - 1) return;
    e.root_rank = e.rank_int[split_of(e.left, n, 0)];
    e.num_int = info->num_interior;
    if (t < n - 1) {
        const int2 rg = e.range[t];
        const bool alive = (t == 0) || !(reach[rg.x] >= rg.y || max_hi[rg.x] > rg.y);
        if (!alive) return;
        const int par = (t == 0) ? -1 : new_interior(e, e.parent[t]);
        const float4 mn = e.nbmin[t], mx = e.nbmax[t];
        const int size = __float_as_int(mx.w);
        if (t == 0 || e.state[t] == 1) {
            const int l = e.left[t], r = e.right[t];
            put_node(nodes, new_interior(e, t), max_nodes,
                     hp_make_node(e.nbmin[l], e.nbmax[l], e.nbmin[r], e.nbmax[r], child_ref(e, l),
                                  child_ref(e, r), size, par), err);
        } else {
            put_node(nodes, e.num_int + e.rank_leaf[rg.x], max_nodes,
                     hp_make_node(mn, mx, mn, mx, rg.x, rg.y + 1, ~size, par), err);
        }
    } else {
        const int p = t - (n - 1);
        if (!(reach[p] < p && max_hi[p] < p)) return;
        const float4 mn = e.nbmin[t], mx = e.nbmax[t];
        const int par = new_interior(e, e.parent[t]);
        put_node(nodes, e.num_int + e.rank_leaf[p], max_nodes,
                 hp_make_node(mn, mx, mn, mx, p, p + 1, ~1, par), err);
    }
}

// A single triangle: root interior node whose second child is an empty leaf.
__global__ void k_single(const float* verts, int64_t nv, const int32_t* tris, hp_node_bin* nodes,
                         float4* woop, int32_t* tri_idx, hp_bvh_info* info, int* err) {
    if (threadIdx.x != 0) return;
    tri_verts t = load_tri(verts, nv, tris, 0, err);
    float4 w0, w1, w2;
    hp_woop(t.x0, t.y0, t.z0, t.x1, t.y1, t.z1, t.x2, t.y2, t.z2, w0, w1, w2);
    woop[0] = w0; woop[1] = w1; woop[2] = w2;
    tri_idx[0] = 0;
    float4 mn = make_float4(fminf(fminf(t.x0, t.x1), t.x2), fminf(fminf(t.y0, t.y1), t.y2),
                            fminf(fminf(t.z0, t.z1), t.z2), 0.0f);
    float4 mx = make_float4(fmaxf(fmaxf(t.x0, t.x1), t.x2), fmaxf(fmaxf(t.y0, t.y1), t.y2),
                            fmaxf(fmaxf(t.z0, t.z1), t.z2), 0.0f);
    float4 emn = make_float4(HP_MAX_FLOAT, HP_MAX_FLOAT, HP_MAX_FLOAT, 0.0f);
    float4 emx = make_float4(-HP_MAX_FLOAT, -HP_MAX_FLOAT, -HP_MAX_FLOAT, 0.0f);
    nodes[0] = hp_make_node(mn, mx, emn, emx, ~1, ~2, 1, -1);
    nodes[1] = hp_make_node(mn, mx, mn, mx, 0, 1, ~1, 0);
    nodes[2] = hp_make_node(emn, emx, emn, emx, 1, 1, ~0, 0);
    for (int k = 0; k < 3; ++k) {
        info->box_ord[k] = hp_f2ord((&mn.x)[k]);
        info->box_ord[3 + k] = hp_f2ord((&mx.x)[k]);
    }
    info->num_interior = 1;
    info->num_leaf = 2;
}

// ---- taps (intermediate results for parity tests) ----------------------------------
template <typename K>
__global__ void k_tap_keys(const K* in, uint64_t* out, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] = (uint64_t)in[i];
}
__global__ void k_tap_tree(int n, const int* parent, const int* left, const int* right,
                           const float4* nbmin, const float4* nbmax, int* tp, int* tl, int* tr,
                           float4* tmn, float4* tmx) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * n - 1) return;
    if (tp) tp[i] = parent[i];
    if (tl) tl[i] = (i < n - 1) ? left[i] : i - (n - 1);
    if (tr) tr[i] = (i < n - 1) ? right[i] : i - (n - 1) + 1;
    float4 a = nbmin[i], b = nbmax[i];
    if (tmn) tmn[i] = make_float4(a.x, a.y, a.z, 0.0f);
    if (tmx) tmx[i] = make_float4(b.x, b.y, b.z, 0.0f);
}
__global__ void k_tap_box(const hp_bvh_info* info, float* out) {
    int k = threadIdx.x;
    if (k < 6) out[k] = hp_ord2f(info->box_ord[k]);
}

template <typename K>
hp_status lbvh_t(hp_ctx* ctx, const hp_mesh* m, const hp_build_params* p, hp_bvh_impl* out,
                 const hp_build_taps* taps, cudaStream_t s) {
    const int64_t n = m->num_triangles;
    const int bits = p->morton_bits;
    const hp_sort_plan plan = hp_sort_make_plan(n, (int)sizeof(K), bits, ctx->tune.sort_block);
    int h_shift = 0, h_count = 0;  // digits the Morton kernel counts for the sort
    hp_sort_hist_digits(plan, &h_shift, &h_count);
    const int64_t nn = 2 * n - 1;
    const bool ploc = p->method == HP_METHOD_PLOC;
    const bool hlbvh = p->method == HP_METHOD_HLBVH;  // binned SAH above the clusters, then the ATR collapse
    const bool atr = p->method == HP_METHOD_ATR || p->method == HP_METHOD_TR || hlbvh;  // treelet restructuring
    const int layout = hp_layout_of(p);
    const bool wide = layout != 2;
    size_t need = 0;
    if (wide) need += hp_carve::pad(hp_wide_scratch_bytes(n, layout));
    need += 2 * hp_carve::pad(n * 16);                  // triangle boxes
    need += 2 * hp_carve::pad(n * sizeof(K));           // keys, sorted keys
    need += hp_carve::pad(plan.scratch_bytes);
    need += hp_carve::pad(hp_sort_hist_bytes(plan.passes));
    if (ploc) {
        need += hp_carve::pad(n * 4) + hp_ploc_scratch_bytes(n);  // sorted references, clustering
        if (!wide) need += hp_carve::pad(n * 48);                 // Woop rows in scene order
    } else if (atr) {
        need += hp_carve::pad(n * 4);                                                     // sorted references
        need += hp_carve::pad(nn * 4) + 2 * hp_carve::pad(n * 4) + hp_carve::pad(n * 8);  // parent, l, r, range
        need += 2 * hp_carve::pad(nn * 16) + hp_carve::pad(n * 4);                        // node boxes, counters
        need += std::max(hp_atr_scratch_bytes(n), hlbvh ? hp_hlbvh_scratch_bytes(n, p->hlbvh_sah_bits) : 0);
    } else {
        need += hp_carve::pad(nn * 4) + 2 * hp_carve::pad(n * 4) + hp_carve::pad(n * 8);  // parent, l, r, range
        need += 2 * hp_carve::pad(nn * 16);                   // node boxes
        need += hp_carve::pad(n * 4) * 8 + hp_carve::pad(n);  // counters, maxhi, reach, flags, ranks, frontier, state
        need += 2 * hp_scan2_scratch_bytes(n + 1);
    }
    HP_TRY(hp_ctx_reserve(ctx, need, s));
    hp_carve cv(ctx->arena);
    // triangle boxes, min and max corners interleaved: element i at [2 i] of
    // tbmin and tbmax, so that a gather in sorted order reads one 32-byte sector
    float4* tbox = cv.take<float4>(2 * n);
    float4* tbmin = tbox;
    float4* tbmax = tbox + 1;
    K* keys = cv.take<K>(n);
    K* skeys = cv.take<K>(n);
    void* sort_scratch = cv.take<char>(plan.scratch_bytes);
    uint32_t* hist = cv.take<uint32_t>(plan.passes * 256);
    void* wide_scratch = wide ? cv.take<char>(hp_wide_scratch_bytes(n, layout)) : nullptr;
    int* err = ctx->d_status;
    hp_bvh_info* info = out->info;
    const int grid_n = hp_div_up(n, TB);
    const int grid_red = (int)std::min<int64_t>(grid_n, (int64_t)ctx->sm_count * 8);
    // the Morton kernel's grid: the CTAs resident at once (a partial second
    // round of CTAs would run at a fraction of the SMs' occupancy)
    int occ_m = 0;
    HP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_m, k_morton<K>, TB, 0));
    const int grid_mor = (int)std::min<int64_t>(grid_n, (int64_t)ctx->sm_count * std::max(1, occ_m));
    if (ploc) {
        int32_t* sorted_refs = cv.take<int32_t>(n);
        void* ploc_scratch = cv.take<char>(hp_ploc_scratch_bytes(n));
        float4* woop_src = wide ? nullptr : cv.take<float4>(3 * n);
        k_init_build<<<hp_div_up(plan.passes * 256, TB), TB, 0, s>>>(info, hist, plan.passes * 256);
        k_tri_boxes<<<grid_red, TB, 0, s>>>(m->vertices, m->num_vertices, m->triangles, n, tbmin, tbmax,
                                            info->box_ord, err, woop_src);
        hp_count_launch(2);
        hp_mark(ctx, s, "boxes");
        k_morton<K><<<grid_mor, TB, 0, s>>>(tbmin, tbmax, n, info, bits, h_shift, h_count, keys, hist);
        HP_CUDA(cudaGetLastError());
        hp_count_launch();
        hp_mark(ctx, s, "morton");
        hp_sort_args sa{keys, nullptr, skeys, sorted_refs, sort_scratch, hist, true, err, ctx};
        HP_TRY(hp_sort_run(plan, sa, s));
        HP_TRY(hp_ploc_stage(ctx, m, p, out, sorted_refs, tbmin, tbmax, ploc_scratch, wide_scratch, s, woop_src));
        if (taps) {
            if (taps->morton_keys) k_tap_keys<K><<<grid_n, TB, 0, s>>>(keys, taps->morton_keys, n);
            if (taps->sorted_keys) k_tap_keys<K><<<grid_n, TB, 0, s>>>(skeys, taps->sorted_keys, n);
            if (taps->sorted_refs)
                HP_CUDA(cudaMemcpyAsync(taps->sorted_refs, sorted_refs, n * 4, cudaMemcpyDeviceToDevice, s));
            if (taps->scene_box) k_tap_box<<<1, 32, 0, s>>>(info, taps->scene_box);
            HP_CUDA(cudaGetLastError());
        }
        return HP_OK;
    }
    if (atr) {
        int32_t* sorted_refs = cv.take<int32_t>(n);
        int* parent = cv.take<int>(nn);
        int* left = cv.take<int>(n);
        int* right = cv.take<int>(n);
        int2* range = cv.take<int2>(n);
        float4* nbmin = cv.take<float4>(nn);
        float4* nbmax = cv.take<float4>(nn);
        int* counters = cv.take<int>(n);
        void* atr_scratch =
            cv.take<char>(std::max(hp_atr_scratch_bytes(n), hlbvh ? hp_hlbvh_scratch_bytes(n, p->hlbvh_sah_bits) : 0));
        k_init_build<<<hp_div_up(plan.passes * 256, TB), TB, 0, s>>>(info, hist, plan.passes * 256);
        k_tri_boxes<<<grid_red, TB, 0, s>>>(m->vertices, m->num_vertices, m->triangles, n, tbmin, tbmax,
                                            info->box_ord, err);
        hp_count_launch(2);
        hp_mark(ctx, s, "boxes");
        k_morton<K><<<grid_mor, TB, 0, s>>>(tbmin, tbmax, n, info, bits, h_shift, h_count, keys, hist);
        HP_CUDA(cudaGetLastError());
        hp_count_launch();
        hp_mark(ctx, s, "morton");
        hp_sort_args sa{keys, nullptr, skeys, sorted_refs, sort_scratch, hist, true, err, ctx};
        HP_TRY(hp_sort_run(plan, sa, s));
        k_karras<K><<<grid_n, TB, 0, s>>>(skeys, (int)n, parent, left, right, range);
        HP_CUDA(cudaGetLastError());
        hp_count_launch();
        hp_mark(ctx, s, "karras");
        hp_build_params q = *p;
        if (hlbvh) {  // the top-level rebuild; the ATR stage with no iterations refits and collapses
            HP_TRY(hp_hlbvh_stage(ctx, p, (int)n, skeys, (int)sizeof(K), sorted_refs, tbmin, tbmax, parent, left,
                                  right, range, nbmin, nbmax, counters, atr_scratch, s));
            q.method = HP_METHOD_ATR;
            q.atr_iterations = 0;
            q.atr_treelet = 9;
        }
        HP_TRY(hp_atr_stage(ctx, m, &q, out, (int)n, sorted_refs, parent, left, right, nbmin, nbmax, counters,
                            tbmin, tbmax, atr_scratch, wide_scratch, s));
        if (taps) {
            if (taps->morton_keys) k_tap_keys<K><<<grid_n, TB, 0, s>>>(keys, taps->morton_keys, n);
            if (taps->sorted_keys) k_tap_keys<K><<<grid_n, TB, 0, s>>>(skeys, taps->sorted_keys, n);
            if (taps->sorted_refs)
                HP_CUDA(cudaMemcpyAsync(taps->sorted_refs, sorted_refs, n * 4, cudaMemcpyDeviceToDevice, s));
            if (taps->node_parent || taps->node_left || taps->node_right || taps->node_box_min ||
                taps->node_box_max)
                k_tap_tree<<<hp_div_up(nn, TB), TB, 0, s>>>((int)n, parent, left, right, nbmin, nbmax,
                                                           taps->node_parent, taps->node_left,
                                                           taps->node_right, (float4*)taps->node_box_min,
                                                           (float4*)taps->node_box_max);
            if (taps->scene_box) k_tap_box<<<1, 32, 0, s>>>(info, taps->scene_box);
            HP_CUDA(cudaGetLastError());
        }
        return HP_OK;
    }
    int* parent = cv.take<int>(nn);
    int* left = cv.take<int>(n);
    int* right = cv.take<int>(n);
    int2* range = cv.take<int2>(n);
    float4* nbmin = cv.take<float4>(nn);
    float4* nbmax = cv.take<float4>(nn);
    int* counters = cv.take<int>(n);
    int* max_hi = cv.take<int>(n);
    int* reach = cv.take<int>(n);
    int* flag_int = cv.take<int>(n);
    int* flag_leaf = cv.take<int>(n);
    int* rank_int = cv.take<int>(n);
    int* rank_leaf = cv.take<int>(n);
    uint8_t* state = cv.take<uint8_t>(n);
    int* frontier = cv.take<int>(n);
    void* scan_a = cv.take<char>(hp_scan2_scratch_bytes(n + 1));
    void* scan_b = cv.take<char>(hp_scan2_scratch_bytes(n + 1));

    k_init_build<<<hp_div_up(plan.passes * 256, TB), TB, 0, s>>>(info, hist, plan.passes * 256);
    HP_CUDA(cudaMemsetAsync(counters, 0, n * 4, s));
    HP_CUDA(cudaMemsetAsync(max_hi, 0xff, n * 4, s));
    k_tri_boxes<<<grid_red, TB, 0, s>>>(m->vertices, m->num_vertices, m->triangles, n, tbmin, tbmax,
                                        info->box_ord, err);
    hp_count_launch(2);
    hp_mark(ctx, s, "boxes");
    k_morton<K><<<grid_mor, TB, 0, s>>>(tbmin, tbmax, n, info, bits, h_shift, h_count, keys, hist);
    HP_CUDA(cudaGetLastError());
    hp_count_launch();
    hp_mark(ctx, s, "morton");
    hp_sort_args sa{keys, nullptr, skeys, out->tri_idx, sort_scratch, hist, true, err, ctx};
    HP_TRY(hp_sort_run(plan, sa, s));
    k_karras<K><<<grid_n, TB, 0, s>>>(skeys, (int)n, parent, left, right, range);
    hp_count_launch();
    hp_mark(ctx, s, "karras");
    k_leaves<<<grid_n, TB, 0, s>>>((int)n, out->tri_idx, m->vertices, m->num_vertices, m->triangles, nbmin,
                                   nbmax, out->woop, p->ci, p->adaptive_leaf, err);
    hp_count_launch();
    hp_mark(ctx, s, "leaves");
    {
        climb_args A{(int)n, parent, left, right, range, nbmin, nbmax, counters, max_hi, state, frontier,
                     reinterpret_cast<unsigned*>(ctx->d_status + 32), p->ct, p->ci, p->adaptive_leaf,
                     p->max_leaf_size, err};
        HP_CUDA(cudaMemsetAsync(A.frontier_count, 0, sizeof(unsigned), s));
        HP_CUDA(cudaFuncSetAttribute(k_climb_local, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)CLIMB_SMEM));
        k_climb_local<<<(unsigned)hp_div_up(n, CB), CB, CLIMB_SMEM, s>>>(A);
        HP_CUDA(cudaGetLastError());
        hp_count_launch();
        hp_mark(ctx, s, "climb_local");
        k_climb_frontier<<<(unsigned)(ctx->sm_count * 8), TB, 0, s>>>(A);
        HP_CUDA(cudaGetLastError());
        hp_count_launch();
    }
    hp_count_launch();
    hp_mark(ctx, s, "climb");
    if (wide) {  // N-wide layouts: references stay in sorted (= depth-first) order
        hp_wide_in W;
        W.n = (int)n;
        W.width = layout;
        W.parent = parent;
        W.left = left;
        W.right = right;
        W.nbmin = nbmin;
        W.nbmax = nbmax;
        W.sorted_tri = out->tri_idx;
        W.reorder = false;
        W.ct = p->ct;
        W.ci = p->ci;
        W.max_leaf = p->adaptive_leaf ? 0x7fffffff : p->max_leaf_size;
        W.verts = m->vertices;
        W.nv = m->num_vertices;
        W.tris = m->triangles;
        HP_TRY(hp_wide_collapse(ctx, W, out, wide_scratch, s));
    } else {
    hp_scan_max_excl(max_hi, n, reach, scan_a, err, s);
    k_collapse_flags<<<hp_div_up(nn, TB), TB, 0, s>>>((int)n, left, range, state, max_hi, reach,
                                                     flag_int, flag_leaf);
    hp_scan2_sum(flag_int, n - 1, flag_leaf, n, rank_int, rank_leaf, &info->num_interior, scan_b, err, s);
    emit_ctx e{(int)n, left, right, parent, range, state, rank_int, rank_leaf, nbmin, nbmax, 0, 0};
    k_emit<<<hp_div_up(nn, TB), TB, 0, s>>>(e, max_hi, reach, info, out->nodes,
                                            (int)std::max<int64_t>(2 * out->capacity - 1, 3), err);
    HP_CUDA(cudaGetLastError());
    hp_count_launch(2);
    hp_mark(ctx, s, "collapse");
    }

    if (taps) {
        if (taps->morton_keys)
            k_tap_keys<K><<<grid_n, TB, 0, s>>>(keys, taps->morton_keys, n);
        if (taps->sorted_keys)
            k_tap_keys<K><<<grid_n, TB, 0, s>>>(skeys, taps->sorted_keys, n);
        if (taps->sorted_refs)
            HP_CUDA(cudaMemcpyAsync(taps->sorted_refs, out->tri_idx, n * 4, cudaMemcpyDeviceToDevice, s));
        if (taps->node_parent || taps->node_left || taps->node_right || taps->node_box_min ||
            taps->node_box_max)
            k_tap_tree<<<hp_div_up(nn, TB), TB, 0, s>>>((int)n, parent, left, right, nbmin, nbmax,
                                                       taps->node_parent, taps->node_left,
                                                       taps->node_right, (float4*)taps->node_box_min,
                                                       (float4*)taps->node_box_max);
        if (taps->scene_box) k_tap_box<<<1, 32, 0, s>>>(info, taps->scene_box);
        HP_CUDA(cudaGetLastError());
    }
    return HP_OK;
}

}  // namespace

hp_status hp_lbvh_build(hp_ctx* ctx, const hp_mesh* m, const hp_build_params* p, hp_bvh_impl* out,
                        const hp_build_taps* taps, cudaStream_t s) {
    const int64_t n = m->num_triangles;
    if (n == 1 && hp_layout_of(p) != 2) return hp_wide_single(ctx, m, hp_layout_of(p), out, s);
    if (n == 1) {
        k_single<<<1, 32, 0, s>>>(m->vertices, m->num_vertices, m->triangles, out->nodes, out->woop,
                                  out->tri_idx, out->info, ctx->d_status);
        HP_CUDA(cudaGetLastError());
        hp_count_launch();
        hp_mark(ctx, s, "single");
        return HP_OK;
    }
    if (p->morton_bits <= 32) return lbvh_t<uint32_t>(ctx, m, p, out, taps, s);
    return lbvh_t<uint64_t>(ctx, m, p, out, taps, s);
}
