// ATR: agglomerative treelet restructuring of the LBVH, then the collapse of the
// restructured tree into 64-byte binary nodes.
//
// Reference: ATRBuilder::build / optimize (rt/bvh/ATRBuilder.cpp:80-236), kernels
// optimize / optimizeSmall / computeSurfaceAreas (rt/bvh/ATRBuilderKernels.cu:
// 12-577) and formTreelet (rt/bvh/TRBuilderUtil.h:141-216).
//
// One launch per iteration (gamma = treelet size T, doubled after each one):
// every thread starts at a leaf and climbs; the second thread to reach a node
// sets refs = refs(l) + refs(r) and cost = ct*A + cost(l) + cost(r) (a leaf
// costs ci*A), and a node with refs >= gamma is restructured by its warp right
// away: the treelet grows from the root's children by expanding the treelet
// leaf of largest area that is not a BVH leaf until it has T leaves, then the
// leaves are merged agglomeratively, smallest union area first, and the new
// topology is written back iff its cost is strictly lower. Every node below a
// treelet root is final when the root is reached, and treelets restructured at
// the same time are disjoint, so the result does not depend on scheduling; the
// two warp searches keep the reference's shuffle-reduction order, which fixes
// how ties are broken.
//
// Differences in form, not in result:
//   * the first iteration also refits the boxes (the reference runs a refit
//     and a surface-area kernel before it), and areas are recomputed from the
//     boxes instead of being stored;
//   * the distance matrix is always in shared memory (up to T = 32);
//   * the row/column of a packed triangular index is decoded exactly with
//     integer arithmetic (the reference uses sqrtf);
//   * refs of restructured treelet nodes are updated too.
// Areas use the ATR kernels' formula 2*(x*y + x*z + y*z), which the
// reference's fast-math build contracts to 2*fma(y, z, fma(x, y, x*z)).
//
// Collapse. A final climb evaluates computeNodeStatesAdaptive
// (BVHCollapserKernels.cu:58-136) on the final topology and the per-subtree
// counts of surviving interior nodes and collapsed leaves. The depth-first
// collapse kernel then processes the nodes in an order where every parent
// comes first, so that each node can wait for its parent's record: interior
// nodes by decreasing subtree size (a radix sort of n - size), then the leaves.
// A parent is larger than its children and usually far larger, so the waits
// rarely chain. The output is numbered in left-first preorder.
#include <algorithm>
#include <type_traits>
#include <cuda_runtime.h>
#include "hp_device.cuh"
#include "hp_internal.h"

namespace {

constexpr int AB = 128;  // threads per CTA
constexpr int AW = AB / 32;
constexpr int TMAX = 32;
constexpr int DMAX = TMAX * (TMAX - 1) / 2;
constexpr float MAXF = 3.402823466e+38f;

__device__ __forceinline__ float atr_area(float mnx, float mny, float mnz, float mxx, float mxy, float mxz) {
    const float x = __fsub_rn(mxx, mnx), y = __fsub_rn(mxy, mny), z = __fsub_rn(mxz, mnz);
    return __fmul_rn(2.0f, __fmaf_rn(y, z, __fmaf_rn(x, y, __fmul_rn(x, z))));
}

__device__ __forceinline__ int tri_index(int row, int col) { return row * (row - 1) / 2 + col; }

__device__ __forceinline__ void tri_decode(int e, int& row, int& col) {
    int r = (int)((1.0f + sqrtf((float)(8 * e + 1))) * 0.5f);
    while (r * (r - 1) / 2 > e) --r;
    while ((r + 1) * r / 2 <= e) ++r;
    row = r;
    col = e - r * (r - 1) / 2;
}

struct atr_args {
    int n, T, gamma, init;
    float ct, ci;
    int* left;
    int* right;
    int* parent;
    float4* nbmin;  // w: ATR cost
    float4* nbmax;  // w: reference count (int bits)
    int* counters;
    const int32_t* sorted_tri;
    const float4* tbmin;
    const float4* tbmax;
    int* err;
};

struct box6 {
    float mn[3], mx[3];
};

__device__ __forceinline__ box6 shfl_box(const box6& b, int src) {
    box6 o;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        o.mn[a] = __shfl_sync(HP_FULL_MASK, b.mn[a], src);
        o.mx[a] = __shfl_sync(HP_FULL_MASK, b.mx[a], src);
    }
    return o;
}

__device__ __forceinline__ box6 join(const box6& a, const box6& b) {
    box6 o;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        o.mn[k] = fminf(a.mn[k], b.mn[k]);
        o.mx[k] = fmaxf(a.mx[k], b.mx[k]);
    }
    return o;
}

__device__ __forceinline__ float area_of(const box6& b) {
    return atr_area(b.mn[0], b.mn[1], b.mn[2], b.mx[0], b.mx[1], b.mx[2]);
}

// Per-warp treelet state in shared memory: the slots being merged (box, cost,
// refs, node), the record of the internal node made at each merge step, and the
// packed lower triangle of pairwise union areas.
struct atr_smem {
    float4 lo[TMAX];   // slot: min corner, cost
    float4 hi[TMAX];   // slot: max corner, refs (int bits)
    int node[TMAX];
    float4 olo[TMAX];  // record of merge step k: min corner, cost
    float4 ohi[TMAX];  // max corner, refs (int bits)
    int2 okids[TMAX];  // children
    float d[DMAX];
};

// TRBVH (treelet of 7 leaves): per-warp subset boxes, costs and best splits.
constexpr int TR_T = 7;
constexpr int TR_SUB = 1 << TR_T;
struct tr_smem {
    float4 smn[TR_SUB];  // subset boxes (w unused)
    float4 smx[TR_SUB];
    float cost[TR_SUB];
    uint8_t mask[TR_SUB];
    int refs[TR_T];      // reference counts of the treelet leaves
};

// Subsets of 2..5 of the 7 treelet leaves, by size (21, 35, 35, 21): each size
// depends only on smaller ones.
__constant__ uint8_t c_tr_subsets[112];
__constant__ int c_tr_size_off[5];

__device__ __forceinline__ box6 box_of(const float4& lo, const float4& hi) {
    box6 b;
    b.mn[0] = lo.x; b.mn[1] = lo.y; b.mn[2] = lo.z;
    b.mx[0] = hi.x; b.mx[1] = hi.y; b.mx[2] = hi.z;
    return b;
}

__device__ __forceinline__ void load_node(const atr_args& A, int v, box6& b, float& cost, int& refs) {
    const float4 mn = __ldcg(A.nbmin + v), mx = __ldcg(A.nbmax + v);
    b.mn[0] = mn.x; b.mn[1] = mn.y; b.mn[2] = mn.z;
    b.mx[0] = mx.x; b.mx[1] = mx.y; b.mx[2] = mx.z;
    cost = mn.w;
    refs = __float_as_int(mx.w);
}

__device__ __forceinline__ bool interior_ok(const atr_args& A, int v) { return (unsigned)v < (unsigned)(A.n - 1); }
__device__ __forceinline__ bool node_ok(const atr_args& A, int v) { return (unsigned)v < (unsigned)(2 * A.n - 1); }

// formTreelet (TRBuilderUtil.h:141-216) for a treelet of T leaves rooted at
// `root` with children l0, r0 (whole warp, converged): lane k ends with
// treelet leaf k (node, box, cost in lo.w, refs in hi.w) and internal node k
// (the root is internal node 0). Each lane fetches a new treelet leaf together
// with its children, so an expansion costs one dependent round trip. Returns
// false (after reporting) on an index out of range.
struct treelet_lane {
    int tl, ti;
    float4 lo, hi;
};

__device__ bool form_treelet(const atr_args& A, int T, int root, int l0, int r0, treelet_lane& L) {
    const int lane = threadIdx.x & 31;
    int tl = lane == 0 ? l0 : (lane == 1 ? r0 : -1);
    int ti = lane == 0 ? root : -1;
    int kl = -1, kr = -1;
    float4 lo = make_float4(0.0f, 0.0f, 0.0f, 0.0f), hi = lo;
    float ta = -MAXF;  // area of an interior treelet leaf
    bool bad = !node_ok(A, l0) || !node_ok(A, r0);
    if (!bad && lane < 2) {
        lo = __ldcg(A.nbmin + tl);
        hi = __ldcg(A.nbmax + tl);
        if (interior_ok(A, tl)) {
            kl = __ldcg(A.left + tl);
            kr = __ldcg(A.right + tl);
            ta = area_of(box_of(lo, hi));
        }
    }
    for (int it = 0; it < T - 2 && !bad; ++it) {
        const int m = it + 2;
        int idx = lane;
        float a = lane < m ? ta : -MAXF;
        // findLeafToExpand: strict '>' keeps the lower lane on ties
        int cnt = m, sh = cnt / 2;
        while (cnt > 1) {
            const int oi = __shfl_down_sync(HP_FULL_MASK, idx, sh);
            const float oa = __shfl_down_sync(HP_FULL_MASK, a, sh);
            if (oa > a) { a = oa; idx = oi; }
            cnt = (cnt + 1) / 2;
            sh = cnt / 2;
        }
        idx = __shfl_sync(HP_FULL_MASK, idx, 0);
        const int rep = __shfl_sync(HP_FULL_MASK, tl, idx);
        const int rl = __shfl_sync(HP_FULL_MASK, kl, idx), rr = __shfl_sync(HP_FULL_MASK, kr, idx);
        // a subtree of >= gamma refs always has an interior leaf to expand
        if (!interior_ok(A, rep) || !node_ok(A, rl) || !node_ok(A, rr)) { bad = true; break; }
        if (lane == it + 1) ti = rep;
        if (lane == idx || lane == m) {
            tl = lane == idx ? rl : rr;
            lo = __ldcg(A.nbmin + tl);
            hi = __ldcg(A.nbmax + tl);
            kl = kr = -1;
            ta = -MAXF;
            if (interior_ok(A, tl)) {
                kl = __ldcg(A.left + tl);
                kr = __ldcg(A.right + tl);
                ta = area_of(box_of(lo, hi));
            }
        }
    }
    if (bad) {
        if (lane == 0) hp_report(A.err, HP_DEV_BAD_INDEX, root);
        return false;
    }
    L.tl = tl;
    L.ti = ti;
    L.lo = lo;
    L.hi = hi;
    return true;
}

// Restructure the treelet rooted at `root` with children l0, r0 (whole warp,
// converged) by agglomerative merging. root_cost is the cost the climb just
// computed for the root.
__device__ void atr_treelet(const atr_args& A, int root, float root_cost, int l0, int r0, atr_smem& W,
                            const uint16_t* rc_of) {
    const int lane = threadIdx.x & 31;
    const int T = A.T;
    treelet_lane L;
    if (!form_treelet(A, T, root, l0, r0, L)) return;
    const int tl = L.tl, ti = L.ti;
    const float4 lo = L.lo, hi = L.hi;
    // ---- slots and the distance matrix
    if (lane < T) {
        W.lo[lane] = lo;
        W.hi[lane] = hi;
        W.node[lane] = tl;
    }
    __syncwarp();
    const int M = T * (T - 1) / 2;
    for (int e = lane; e < M; e += 32) {
        const int rc = rc_of[e], row = rc >> 8, col = rc & 255;
        W.d[e] = area_of(join(box_of(W.lo[row], W.hi[row]), box_of(W.lo[col], W.hi[col])));
    }
    __syncwarp();
    // ---- agglomerative merging; step `last` makes internal node ti[last - 1]
    for (int last = T - 1; last >= 1; --last) {
        const int mm = last * (last + 1) / 2;
        float best = MAXF;
        int bi = 0;
        for (int e = lane; e < mm; e += 32) {
            const float d = W.d[e];
            if (d < best) { best = d; bi = e; }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const float obst = __shfl_down_sync(HP_FULL_MASK, best, off);
            const int oi = __shfl_down_sync(HP_FULL_MASK, bi, off);
            if (obst < best) { best = obst; bi = oi; }
        }
        bi = __shfl_sync(HP_FULL_MASK, bi, 0);
        const int rc = rc_of[bi], row = rc >> 8, col = rc & 255;
        const float4 rlo = W.lo[row], rhi = W.hi[row], clo = W.lo[col], chi = W.hi[col];
        const box6 u = join(box_of(rlo, rhi), box_of(clo, chi));
        const float uc = __fmaf_rn(A.ct, area_of(u), __fadd_rn(rlo.w, clo.w));
        const float4 ulo = make_float4(u.mn[0], u.mn[1], u.mn[2], uc);
        const float4 uhi = make_float4(u.mx[0], u.mx[1], u.mx[2],
                                       __int_as_float(__float_as_int(rhi.w) + __float_as_int(chi.w)));
        const int n_r = W.node[row], n_c = W.node[col];
        const float4 llo = W.lo[last], lhi = W.hi[last];
        const int n_l = W.node[last];
        const int inode = __shfl_sync(HP_FULL_MASK, ti, last - 1);
        float dv = 0.0f;
        int dst = -1;
        if (last > 1 && lane < last && lane != row) {
            dv = W.d[tri_index(last, lane)];
            dst = tri_index(max(row, lane), min(row, lane));
        }
        __syncwarp();
        if (lane == 0) {
            W.olo[last] = ulo;
            W.ohi[last] = uhi;
            W.okids[last] = make_int2(n_r, n_c);
            W.lo[col] = ulo;
            W.hi[col] = uhi;
            W.node[col] = inode;
            W.lo[row] = llo;
            W.hi[row] = lhi;
            W.node[row] = n_l;
        }
        if (dst >= 0) W.d[dst] = dv;
        __syncwarp();
        if (last > 1 && lane < last && lane != col)
            W.d[tri_index(max(col, lane), min(col, lane))] = area_of(join(box_of(W.lo[lane], W.hi[lane]), u));
        __syncwarp();
    }
    // ---- updateTreelet: keep the new topology iff its cost is strictly lower
    const float newc = W.olo[1].w;
    const int node = __shfl_up_sync(HP_FULL_MASK, ti, 1);
    if (newc < root_cost && lane >= 1 && lane < T) {
        const float4 olo = W.olo[lane], ohi = W.ohi[lane];
        const int2 k = W.okids[lane];
        __stcg(A.left + node, k.x);
        __stcg(A.right + node, k.y);
        __stcg(A.parent + k.x, node);
        __stcg(A.parent + k.y, node);
        __stcg(A.nbmin + node, olo);
        __stcg(A.nbmax + node, ohi);
    }
    __threadfence();
    __syncwarp();
}

// TRBVH treelet optimisation (TRBuilderKernels.cu:12-300) for the treelet at
// `root` (whole warp, converged): subset boxes and areas, the dynamic
// programme over subsets in the kernel's partition order and tie rules, and
// the top-down rebuild when the best cost is below the root's. root_refs is
// the root's reference count (the leaf term of every subset uses it, as the
// kernel does), root_cost the cost the climb computed for it. The root keeps
// its cost; a new internal node takes cost(split of its parent's subset) —
// for a right child as well, as the kernel stores it.
__device__ void tr_treelet(const atr_args& A, int root, float root_cost, int root_refs, int l0, int r0, tr_smem& W) {
    const int lane = threadIdx.x & 31;
    constexpr int T = TR_T, FULL = TR_SUB - 1;
    treelet_lane L;
    if (!form_treelet(A, T, root, l0, r0, L)) return;
    // subset boxes and areas: lane l builds subsets 4l .. 4l+3
    box6 leaf[T];
#pragma unroll
    for (int i = 0; i < T; ++i) leaf[i] = shfl_box(box_of(L.lo, L.hi), i);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int sub = 4 * lane + q;
        box6 b;
        for (int a = 0; a < 3; ++a) { b.mn[a] = MAXF; b.mx[a] = -MAXF; }
#pragma unroll
        for (int i = 0; i < T; ++i)
            if (sub & (1 << i)) b = join(b, leaf[i]);
        W.smn[sub] = make_float4(b.mn[0], b.mn[1], b.mn[2], 0.0f);
        W.smx[sub] = make_float4(b.mx[0], b.mx[1], b.mx[2], 0.0f);
        W.cost[sub] = area_of(b);
        W.mask[sub] = 0;
    }
    __syncwarp();
    if (lane < T) {
        W.cost[1 << lane] = L.lo.w;
        W.refs[lane] = __float_as_int(L.hi.w);
    }
    __syncwarp();
    const float refs = (float)root_refs;
    auto finish = [&](int sub, float opt, int p) {
        const float a = W.cost[sub];
        W.cost[sub] = fminf(__fmaf_rn(A.ct, a, opt), __fmul_rn(__fmul_rn(A.ci, a), refs));
        W.mask[sub] = (uint8_t)p;
    };
    // sizes 2 .. T-2 (processSchedule): partitions (-delta)&s, then (p - delta)&s
    for (int size = 0; size < 4; ++size) {
        const int off = c_tr_size_off[size], cnt = c_tr_size_off[size + 1] - off;
        for (int b0 = 0; b0 < cnt; b0 += 32) {
            if (b0 + lane < cnt) {
                const int sub = c_tr_subsets[off + b0 + lane];
                const int delta = (sub - 1) & sub;
                int p = (-delta) & sub;
                float opt = MAXF;
                int optp = 0;
                while (p != 0) {
                    const float c = __fadd_rn(W.cost[p], W.cost[p ^ sub]);
                    if (c < opt) { opt = c; optp = p; }
                    p = (p - delta) & sub;
                }
                finish(sub, opt, optp);
            }
        }
        __syncwarp();
    }
    // size T-1 (processSubsets): four lanes per subset, reduced q0:q2, q1:q3, then 0:1
    {
        const int k = lane >> 2, q = lane & 3;
        const int sub = FULL & ~(1 << k);
        float opt = MAXF;
        int optp = 0;
        if (lane < 4 * T) {
            const int lm = -(1 << max(k - 1, 0));
            int base = q + 1;
            int p = (((base & lm) << 1) | (base & ~lm)) << 1;
            for (int j = q; j < (1 << (T - 2)) - 1; j += 4) {
                const float c = __fadd_rn(W.cost[p], W.cost[p ^ sub]);
                if (c < opt) { opt = c; optp = p; }
                base += 4;
                p = (((base & lm) << 1) | (base & ~lm)) << 1;
            }
        }
        for (int i = 2; i > 0; i >>= 1) {
            const float oo = __shfl_down_sync(HP_FULL_MASK, opt, i);
            const int op = __shfl_down_sync(HP_FULL_MASK, optp, i);
            if (oo < opt) { opt = oo; optp = op; }
        }
        if (lane < 4 * T && q == 0) finish(sub, opt, optp);
    }
    __syncwarp();
    // the full set: lane l takes 2(l+1) and 2(l+1) + 64, reduced over the warp
    {
        float opt = MAXF;
        int optp = 0;
        int p = (lane + 1) * 2;
        for (int j = lane; j < (1 << (T - 1)) - 1; j += 32) {
            const float c = __fadd_rn(W.cost[p], W.cost[p ^ FULL]);
            if (c < opt) { opt = c; optp = p; }
            p += 64;
        }
#pragma unroll
        for (int i = 16; i > 0; i >>= 1) {
            const float oo = __shfl_down_sync(HP_FULL_MASK, opt, i);
            const int op = __shfl_down_sync(HP_FULL_MASK, optp, i);
            if (oo < opt) { opt = oo; optp = op; }
        }
        if (lane == 0) finish(FULL, opt, optp);
    }
    __syncwarp();
    // updateTreelet: top-down rebuild by lane 0, rounds of left children then right children
    int ti_all[T - 1], tl_all[T];
#pragma unroll
    for (int i = 0; i < T - 1; ++i) ti_all[i] = __shfl_sync(HP_FULL_MASK, L.ti, i);
#pragma unroll
    for (int i = 0; i < T; ++i) tl_all[i] = __shfl_sync(HP_FULL_MASK, L.tl, i);
    if (lane == 0 && W.cost[FULL] < root_cost) {
        int rn[T - 1], rs[T - 1], nr = 1, next = 1;
        rn[0] = root;
        rs[0] = FULL;
        while (nr > 0) {
            int on[T - 1], os[T - 1], no = 0;
            for (int side = 0; side < 2; ++side)
                for (int e = 0; e < nr; ++e) {
                    const int node = rn[e], sub = rs[e];
                    const int p = W.mask[sub];
                    const int cs = side == 0 ? p : (p ^ sub);
                    int child;
                    if (__popc(cs) > 1) {
                        if (next >= T - 1 || no >= T - 1) { hp_report(A.err, HP_DEV_BAD_INDEX, root); return; }
                        child = ti_all[next++];
                        int r = 0;
                        for (int i = 0; i < T; ++i)
                            if (cs & (1 << i)) r += W.refs[i];
                        const float4 mn = W.smn[cs], mx = W.smx[cs];
                        __stcg(A.nbmin + child, make_float4(mn.x, mn.y, mn.z, W.cost[p]));
                        __stcg(A.nbmax + child, make_float4(mx.x, mx.y, mx.z, __int_as_float(r)));
                        on[no] = child;
                        os[no] = cs;
                        ++no;
                    } else {
                        child = tl_all[__ffs(cs) - 1];
                    }
                    __stcg((side == 0 ? A.left : A.right) + node, child);
                    __stcg(A.parent + child, node);
                }
            for (int e = 0; e < no; ++e) { rn[e] = on[e]; rs[e] = os[e]; }
            nr = no;
        }
    }
    __threadfence();
    __syncwarp();
}

template <bool TR>
__global__ void __launch_bounds__(AB) k_atr_iter(atr_args A) {
    using wsmem = typename std::conditional<TR, tr_smem, atr_smem>::type;
    __shared__ wsmem s_w[AW];
    __shared__ uint16_t s_rc[DMAX];  // packed triangle index -> (row << 8) | col
    if (!TR) {
        for (int e = threadIdx.x; e < DMAX; e += AB) {
            int row, col;
            tri_decode(e, row, col);
            s_rc[e] = (uint16_t)((row << 8) | col);
        }
        __syncthreads();
    }
    const int warp = threadIdx.x >> 5;
    const int p = blockIdx.x * AB + threadIdx.x;
    const int n = A.n;
    int cur = -1;
    if (p < n) {
        const int leaf = n - 1 + p;
        if (A.init) {
            const int tri = A.sorted_tri[p];
            if ((unsigned)tri >= (unsigned)n) {
                hp_report(A.err, HP_DEV_BAD_INDEX, p);
            } else {
                const float4 mn = A.tbmin[2 * (int64_t)tri], mx = A.tbmax[2 * (int64_t)tri];
                const float c = __fmul_rn(A.ci, atr_area(mn.x, mn.y, mn.z, mx.x, mx.y, mx.z));
                __stcg(A.nbmin + leaf, make_float4(mn.x, mn.y, mn.z, c));
                __stcg(A.nbmax + leaf, make_float4(mx.x, mx.y, mx.z, __int_as_float(1)));
            }
        }
        cur = __ldcg(A.parent + leaf);
    }
    int steps = 0;
    while (__any_sync(HP_FULL_MASK, cur >= 0)) {
        if (++steps > n + 1) {  // a valid tree is climbed in at most n - 1 steps
            if ((threadIdx.x & 31) == 0) hp_report(A.err, HP_DEV_BAD_INDEX, -1);
            break;
        }
        bool arrived = false;
        int refs = 0, l = -1, r = -1;
        float cost = 0.0f;
        if (cur >= 0) {
            if (!interior_ok(A, cur)) {
                hp_report(A.err, HP_DEV_BAD_INDEX, cur);
                cur = -1;
            } else {
                if (hp_arrive(A.counters + cur) == 0) cur = -1;
                else arrived = true;
            }
        }
        int up = -1;
        if (arrived) {
            l = __ldcg(A.left + cur);
            r = __ldcg(A.right + cur);
            up = __ldcg(A.parent + cur);  // a treelet rooted at cur keeps cur's parent
            if (!node_ok(A, l) || !node_ok(A, r)) {
                hp_report(A.err, HP_DEV_BAD_INDEX, cur);
                arrived = false;
                cur = -1;
            } else {
                box6 bl, br;
                float cl, cr;
                int rl, rr;
                load_node(A, l, bl, cl, rl);
                load_node(A, r, br, cr, rr);
                const box6 u = join(bl, br);
                refs = rl + rr;
                cost = __fadd_rn(__fmaf_rn(A.ct, area_of(u), cl), cr);
                __stcg(A.nbmin + cur, make_float4(u.mn[0], u.mn[1], u.mn[2], cost));
                __stcg(A.nbmax + cur, make_float4(u.mx[0], u.mx[1], u.mx[2], __int_as_float(refs)));
            }
        }
        unsigned vote = __ballot_sync(HP_FULL_MASK, arrived && refs >= A.gamma);
        while (vote) {
            const int src = __ffs(vote) - 1;
            const int root = __shfl_sync(HP_FULL_MASK, cur, src);
            const float rc = __shfl_sync(HP_FULL_MASK, cost, src);
            const int l0 = __shfl_sync(HP_FULL_MASK, l, src), r0 = __shfl_sync(HP_FULL_MASK, r, src);
            if constexpr (TR) {
                const int rr = __shfl_sync(HP_FULL_MASK, refs, src);
                tr_treelet(A, root, rc, rr, l0, r0, s_w[warp]);
            } else {
                atr_treelet(A, root, rc, l0, r0, s_w[warp], s_rc);
            }
            vote &= vote - 1;
        }
        cur = arrived ? up : -1;
    }
}

struct fin_args {
    int n, init, adaptive, max_leaf;
    float ct, ci;
    const int* left;
    const int* right;
    const int* parent;
    float4* nbmin;  // w: collapse cost
    float4* nbmax;  // w: size (int bits)
    int* counters;
    uint8_t* state;
    int2* counts;   // surviving interior nodes, collapsed leaves
    const int32_t* sorted_tri;
    const float4* tbmin;
    const float4* tbmax;
    int* err;
};

// computeSizes + computeNodeStatesAdaptive / computeNodeStates on the final
// topology, plus the per-subtree counts of the collapse.
__global__ void __launch_bounds__(256) k_atr_finish(fin_args F) {
    const int p = blockIdx.x * 256 + threadIdx.x;
    const int n = F.n;
    if (p >= n) return;
    const int leaf = n - 1 + p;
    float4 mn, mx;
    if (F.init) {
        const int tri = F.sorted_tri[p];
        if ((unsigned)tri >= (unsigned)n) { hp_report(F.err, HP_DEV_BAD_INDEX, p); return; }
        mn = F.tbmin[2 * (int64_t)tri];  // interleaved corners
        mx = F.tbmax[2 * (int64_t)tri];
    } else {
        mn = __ldcg(F.nbmin + leaf);
        mx = __ldcg(F.nbmax + leaf);
    }
    const float lc = F.adaptive ? __fmul_rn(F.ci, hp_area(mn.x, mn.y, mn.z, mx.x, mx.y, mx.z)) : 0.0f;
    __stcg(F.nbmin + leaf, make_float4(mn.x, mn.y, mn.z, lc));
    __stcg(F.nbmax + leaf, make_float4(mx.x, mx.y, mx.z, __int_as_float(1)));
    F.state[leaf] = 0;
    __stcg(F.counts + leaf, make_int2(0, 1));
    int node = __ldcg(F.parent + leaf);
    int guard = 0;
    while (node >= 0) {
        if (node >= n - 1 || ++guard > n) {
            hp_report(F.err, HP_DEV_BAD_INDEX, node);
            return;
        }
        __threadfence();
        if (atomicAdd(F.counters + node, 1) == 0) return;
        __threadfence();
        const int l = __ldcg(F.left + node), r = __ldcg(F.right + node);
        if ((unsigned)l >= (unsigned)(2 * n - 1) || (unsigned)r >= (unsigned)(2 * n - 1)) {
            hp_report(F.err, HP_DEV_BAD_INDEX, node);
            return;
        }
        const float4 lmn = __ldcg(F.nbmin + l), lmx = __ldcg(F.nbmax + l);
        const float4 rmn = __ldcg(F.nbmin + r), rmx = __ldcg(F.nbmax + r);
        const float mnx = fminf(lmn.x, rmn.x), mny = fminf(lmn.y, rmn.y), mnz = fminf(lmn.z, rmn.z);
        const float mxx = fmaxf(lmx.x, rmx.x), mxy = fmaxf(lmx.y, rmx.y), mxz = fmaxf(lmx.z, rmx.z);
        const int size = __float_as_int(lmx.w) + __float_as_int(rmx.w);
        int st;
        float c;
        if (F.adaptive) {
            const float area = hp_area(mnx, mny, mnz, mxx, mxy, mxz);
            const float c_int = __fadd_rn(__fmaf_rn(F.ct, area, lmn.w), rmn.w);
            const float c_leaf = __fmul_rn(__fmul_rn(F.ci, area), (float)size);
            st = (c_leaf < c_int) ? 0 : 1;
            c = st ? c_int : c_leaf;
        } else {
            st = (size <= F.max_leaf) ? 0 : 1;
            c = 0.0f;
        }
        const int2 cl = __ldcg(F.counts + l), cr = __ldcg(F.counts + r);
        __stcg(F.nbmin + node, make_float4(mnx, mny, mnz, c));
        __stcg(F.nbmax + node, make_float4(mxx, mxy, mxz, __int_as_float(size)));
        F.state[node] = (uint8_t)st;
        __stcg(F.counts + node, st ? make_int2(1 + cl.x + cr.x, cl.y + cr.y) : make_int2(0, 1));
        node = __ldcg(F.parent + node);
    }
}

// Sort keys of the interior nodes: n - size, so that a stable ascending sort
// lists larger subtrees first.
__global__ void __launch_bounds__(256) k_size_keys(int n, const float4* __restrict__ nbmax, uint32_t* keys) {
    const int v = blockIdx.x * 256 + threadIdx.x;
    if (v >= n - 1) return;
    keys[v] = (uint32_t)(n - __float_as_int(__ldg(&nbmax[v].w)));
}

__global__ void __launch_bounds__(256) k_leaf_order(int n, int* order) {
    const int p = blockIdx.x * 256 + threadIdx.x;
    if (p < n) order[n - 1 + p] = n - 1 + p;
}

}  // namespace

size_t hp_atr_scratch_bytes(int64_t n) {
    const int64_t nn = 2 * n - 1;
    size_t b = 0;
    b += hp_carve::pad(nn);                        // state
    b += hp_carve::pad(nn * 8);                    // counts
    b += 2 * hp_carve::pad(n * 4);                 // size keys, sorted keys
    b += hp_carve::pad(nn * 4);                    // order
    const hp_sort_plan plan = hp_sort_make_plan(n, 4, 32);
    b += hp_carve::pad(plan.scratch_bytes) + hp_carve::pad(hp_sort_hist_bytes(plan.passes));
    b += hp_topdown_scratch_bytes(n);
    return b;
}

// The subset table of the TRBVH kernel: subsets of 2..5 of 7 leaves by size,
// uploaded once per device.
hp_status tr_tables() {
    static bool done[64] = {};
    int dev = 0;
    HP_CUDA(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && done[dev]) return HP_OK;
    uint8_t subs[112];
    int off[5] = {0, 0, 0, 0, 0}, k = 0;
    for (int size = 2; size <= TR_T - 2; ++size) {
        off[size - 2] = k;
        for (int sub = 1; sub < TR_SUB - 1; ++sub)
            if (__builtin_popcount(sub) == size) subs[k++] = (uint8_t)sub;
    }
    off[4] = k;
    if (k != 112) return hp_fail(HP_ERR_ARG, "TRBVH subset table");
    HP_CUDA(cudaMemcpyToSymbol(c_tr_subsets, subs, sizeof(subs)));
    HP_CUDA(cudaMemcpyToSymbol(c_tr_size_off, off, sizeof(off)));
    if (dev >= 0 && dev < 64) done[dev] = true;
    return HP_OK;
}

hp_status hp_atr_stage(hp_ctx* ctx, const hp_mesh* m, const hp_build_params* p, hp_bvh_impl* out, int n,
                       const int32_t* sorted_tri, int* parent, int* left, int* right, float4* nbmin,
                       float4* nbmax, int* counters, const float4* tbmin, const float4* tbmax, void* scratch,
                       void* wide_scratch, cudaStream_t s) {
    const int64_t nn = 2 * (int64_t)n - 1;
    const bool tr = p->method == HP_METHOD_TR;  // TRBVH: dynamic programming over treelets of 7
    const int T = tr ? TR_T : p->atr_treelet;
    if (T < 3 || T > TMAX) return hp_fail(HP_ERR_ARG, "ATR treelet size must be in [3, 32]");
    if (tr) HP_TRY(tr_tables());
    if (p->atr_iterations < 0) return hp_fail(HP_ERR_ARG, "ATR iterations must be >= 0");
    hp_carve cv(reinterpret_cast<char*>(scratch));
    uint8_t* state = cv.take<uint8_t>(nn);
    int2* counts = cv.take<int2>(nn);
    uint32_t* keys = cv.take<uint32_t>(n);
    uint32_t* skeys = cv.take<uint32_t>(n);
    int* order = cv.take<int>(nn);
    int bits = 1;
    while ((int64_t(1) << bits) <= n) ++bits;
    const hp_sort_plan plan = hp_sort_make_plan(n - 1, 4, bits, 512);
    const hp_sort_plan pmax = hp_sort_make_plan(n, 4, 32);
    void* sort_scratch = cv.take<char>(pmax.scratch_bytes);
    uint32_t* hist = cv.take<uint32_t>(pmax.passes * 256);
    void* td_scratch = cv.take<char>(hp_topdown_scratch_bytes(n));
    int* err = ctx->d_status;

    atr_args A{};
    A.n = n; A.T = T; A.ct = p->ct; A.ci = p->ci;
    A.left = left; A.right = right; A.parent = parent; A.nbmin = nbmin; A.nbmax = nbmax;
    A.counters = counters; A.sorted_tri = sorted_tri; A.tbmin = tbmin; A.tbmax = tbmax; A.err = err;
    int gamma = T, runs = 0;
    for (int i = 0; i < p->atr_iterations; ++i) {
        A.gamma = gamma;
        A.init = (i == 0);
        HP_CUDA(cudaMemsetAsync(counters, 0, (size_t)n * 4, s));
        if (tr) k_atr_iter<true><<<hp_div_up(n, AB), AB, 0, s>>>(A);
        else k_atr_iter<false><<<hp_div_up(n, AB), AB, 0, s>>>(A);
        HP_CUDA(cudaGetLastError());
        hp_count_launch();
        hp_mark(ctx, s, tr ? "tr_iteration" : "atr_iteration");
        ++runs;
        gamma *= 2;
        if (gamma > n) break;
    }
    fin_args F{};
    F.n = n; F.init = runs == 0; F.adaptive = p->adaptive_leaf; F.max_leaf = p->max_leaf_size;
    F.ct = p->ct; F.ci = p->ci; F.left = left; F.right = right; F.parent = parent; F.nbmin = nbmin;
    F.nbmax = nbmax; F.counters = counters; F.state = state; F.counts = counts;
    F.sorted_tri = sorted_tri; F.tbmin = tbmin; F.tbmax = tbmax; F.err = err;
    HP_CUDA(cudaMemsetAsync(counters, 0, (size_t)n * 4, s));
    k_atr_finish<<<hp_div_up(n, 256), 256, 0, s>>>(F);
    HP_CUDA(cudaGetLastError());
    hp_mark(ctx, s, "atr_finish");
    if (hp_layout_of(p) != 2) {  // N-wide layouts: the final climb has set every box
        hp_wide_in W;
        W.n = n;
        W.width = hp_layout_of(p);
        W.parent = parent;
        W.left = left;
        W.right = right;
        W.nbmin = nbmin;
        W.nbmax = nbmax;
        W.sorted_tri = sorted_tri;
        W.reorder = true;
        W.ct = p->ct;
        W.ci = p->ci;
        W.max_leaf = p->adaptive_leaf ? 0x7fffffff : p->max_leaf_size;
        W.verts = m->vertices;
        W.nv = m->num_vertices;
        W.tris = m->triangles;
        return hp_wide_collapse(ctx, W, out, wide_scratch, s);
    }
    k_size_keys<<<hp_div_up(n, 256), 256, 0, s>>>(n, nbmax, keys);
    k_leaf_order<<<hp_div_up(n, 256), 256, 0, s>>>(n, order);
    HP_CUDA(cudaGetLastError());
    hp_count_launch(2);
    hp_sort_args sa{keys, nullptr, skeys, order, sort_scratch, hist, false, err, nullptr};
    HP_TRY(hp_sort_run(plan, sa, s));
    hp_topdown_in in{};
    in.n = n; in.left = left; in.right = right; in.parent = parent; in.counts = counts; in.state = state;
    in.nbmin = nbmin; in.nbmax = nbmax; in.order = order; in.sorted_tri = sorted_tri;
    HP_TRY(hp_topdown_collapse(ctx, m, in, out, td_scratch, s));
    hp_mark(ctx, s, "collapse");
    return HP_OK;
}
