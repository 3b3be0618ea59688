// HLBVH: LBVH clusters below the top Morton bits, a binned-SAH top tree above.
//
// Reference: HLBVHBuilder::build (rt/bvh/HLBVHBuilder.cpp:330-395) with the
// kernels computeNodeStates, computeLeafClusterIndices,
// invalidateIntermediateClusters, computeNodeOffsets, compact, computeClusters,
// binClusters, split and distributeClusters (rt/bvh/HLBVHBuilderKernels.cu:
// 35-704), and HLBVHBin (rt/bvh/HLBVHBin.h).
//
// After the Karras LBVH:
//   1. a climb refits the LBVH boxes;
//   2. an interior node whose split prefix delta(g, g+1) covers the top sahBits
//      of the key lies inside a cluster (state 0; leaves too); the clusters are
//      the highest state-0 nodes below the root, listed in sorted order, and
//      the nodes above them (state 1) are listed in index order: their indices
//      are reused for the top tree (the root keeps index 0);
//   3. one CTA builds the top tree over the clusters (at most 2^sahBits of
//      them) level by level. Every cluster bins its box into its task's bins
//      by the (x, y, z) coordinates of its top sahBits Morton bits
//      (2^(sahBits/3) bins per axis, order-preserving integer atomics for the
//      float bounds); a warp per task sweeps an axis at a time, lane b holding
//      bin b: left unions by a prefix scan, right unions by a suffix scan, the
//      cost fma(count_l, A_l, count_r * A_r) of the split after bin b when
//      both sides hold clusters, and the first strictly lowest cost over (axis,
//      bin); clusters at or below the split bin go left, a side with one
//      cluster takes that cluster's subtree, and interior children take the
//      next free indices, left before right, tasks in order;
//   4. the ATR stage with no iterations then refits the tree and collapses it.
// sahBits must be a multiple of 3 in [6, 15]: then every cluster has its own
// cell (for other values the reference's bin coordinates run past the bins of
// their axis), except that the reference's computeClusters reads a leaf
// cluster's key at its left index with n-1 subtracted, so a leaf cluster at the
// last sorted position takes key 0's cell. That leaf and the cluster holding
// position 0 are never separated by a bin split and end as a task of two
// clusters in one bin, which takes the reference's object-median fallback: the
// reference orders the two by atomic arrival, this kernel puts the first in
// sorted order left. When the root itself lies inside a cluster the LBVH is
// kept as it is.
#include <algorithm>
#include <cuda_runtime.h>
#include "hp_device.cuh"
#include "hp_internal.h"

namespace {

constexpr int HB = 256;       // threads per CTA of the per-node kernels
constexpr int TOPB = 512;     // threads of a top-tree CTA
constexpr float MAXF = 3.402823466e+38f;

template <typename K> __device__ __forceinline__ int key_prefix(const K* k, int i, int j, int bits);
// Common prefix length of keys i and j within the `bits` key bits; equal keys
// share all of them (the reference appends the index bits after them).
template <> __device__ __forceinline__ int key_prefix<uint64_t>(const uint64_t* k, int i, int j, int bits) {
    const uint64_t a = __ldg(k + i), b = __ldg(k + j);
    return a == b ? bits : __clzll((long long)(a ^ b)) - (64 - bits);
}
template <> __device__ __forceinline__ int key_prefix<uint32_t>(const uint32_t* k, int i, int j, int bits) {
    const uint32_t a = __ldg(k + i), b = __ldg(k + j);
    return a == b ? bits : __clz((int)(a ^ b)) - (32 - bits);
}

// Refit of the LBVH boxes (leaves from the sorted triangle boxes).
__global__ void __launch_bounds__(HB) k_hl_refit(int n, const int32_t* __restrict__ sorted_tri,
                                                 const float4* __restrict__ tbmin, const float4* __restrict__ tbmax,
                                                 const int* parent, const int* left, const int* right, float4* nbmin,
                                                 float4* nbmax, int* counters, int* err) {
    const int p = blockIdx.x * HB + threadIdx.x;
    if (p >= n) return;
    const int tri = __ldg(sorted_tri + p);
    if ((unsigned)tri >= (unsigned)n) { hp_report(err, HP_DEV_BAD_INDEX, p); return; }
    const int leaf = n - 1 + p;
    __stcg(nbmin + leaf, __ldg(tbmin + 2 * (int64_t)tri));  // interleaved corners
    __stcg(nbmax + leaf, __ldg(tbmax + 2 * (int64_t)tri));
    int node = __ldcg(parent + leaf), guard = 0;
    while (node >= 0) {
        if (node >= n - 1 || ++guard > n) { hp_report(err, HP_DEV_BAD_INDEX, node); return; }
        if (hp_arrive(counters + node) == 0) return;
        const int l = __ldcg(left + node), r = __ldcg(right + node);
        const float4 a = __ldcg(nbmin + l), b = __ldcg(nbmin + r), c = __ldcg(nbmax + l), d = __ldcg(nbmax + r);
        __stcg(nbmin + node, make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z), 0.0f));
        __stcg(nbmax + node, make_float4(fmaxf(c.x, d.x), fmaxf(c.y, d.y), fmaxf(c.z, d.z), 0.0f));
        node = __ldcg(parent + node);
    }
}

// State of every interior node: 1 when its split prefix delta(g, g+1) ends
// inside the top sahBits of the key (g = the split position, which is the left
// child's index, or its sorted position for a leaf), else 0.
template <typename K>
__global__ void __launch_bounds__(HB) k_hl_mark(int n, const K* __restrict__ skeys, int bits, int sah,
                                                const int* __restrict__ left, int* state, int* top_flag) {
    const int v = blockIdx.x * HB + threadIdx.x;
    if (v >= n - 1) return;
    const int lc = __ldg(left + v);
    const int g = lc >= n - 1 ? lc - (n - 1) : lc;
    const int st = key_prefix<K>(skeys, g, g + 1, bits) >= sah ? 0 : 1;
    state[v] = st;
    top_flag[v] = st;
}

// Cluster roots: state 0 (leaves are) with the root or a state-1 node as parent.
__global__ void __launch_bounds__(HB) k_hl_clusters(int n, const int* __restrict__ parent,
                                                    const int2* __restrict__ range, const int* __restrict__ state,
                                                    int* cluster_flag, int* cluster_at) {
    const int v = blockIdx.x * HB + threadIdx.x;
    if (v == 0 || v >= 2 * n - 1) return;
    const int sv = v >= n - 1 ? 0 : __ldg(state + v);
    if (sv != 0) return;
    const int p = __ldg(parent + v);
    if (p < 0) return;
    if (p != 0 && __ldg(state + p) != 1) return;
    const int first = v >= n - 1 ? v - (n - 1) : __ldg(range + v).x;
    cluster_flag[first] = 1;
    cluster_at[first] = v;
}

// Cluster list (node, packed cell coordinates) and the free index list.
template <typename K>
__global__ void __launch_bounds__(HB) k_hl_scatter(int n, const K* __restrict__ skeys, int bits, int sah,
                                                   const int* __restrict__ cluster_flag,
                                                   const int* __restrict__ cluster_at,
                                                   const int* __restrict__ cluster_off, const int* __restrict__ top_flag,
                                                   const int* __restrict__ top_off, int* cl_node, int* cl_cell,
                                                   int* free_idx) {
    const int i = blockIdx.x * HB + threadIdx.x;
    if (i < n && cluster_flag[i]) {
        const int c = cluster_off[i];
        cl_node[c] = cluster_at[i];
        // the leaf at the last position bins with key 0's cell, as the
        // reference's computeClusters reads it
        const uint32_t code = (uint32_t)((__ldg(skeys + (i == n - 1 ? 0 : i)) >> (bits - sah)) & ((1u << sah) - 1u));
        int x = 0, y = 0, z = 0;
#pragma unroll
        for (int b = 0; b < 10; ++b) {
            x += ((code >> (3 * b + 0)) & 1) << b;
            y += ((code >> (3 * b + 1)) & 1) << b;
            z += ((code >> (3 * b + 2)) & 1) << b;
        }
        cl_cell[c] = x | (y << 10) | (z << 20);
    }
    if (i < n - 1 && top_flag[i]) free_idx[top_off[i]] = i;
}

struct top_args {
    int n, NB, tmax;
    const int* totals;     // [0] clusters, [1] state-1 nodes
    const int* cl_node;
    const int* cl_cell;
    const int* free_idx;
    int* task_of;          // [C] task of each unassigned cluster, -1 once linked
    int2* tasks[2];        // [C/2] (node, parent) per task, by level parity
    uint32_t* bins;        // [C/2][3][NB][7]: ordered min xyz, ordered max xyz, count
    int4* split;           // [C/2] (axis, bin, left task, right task); axis 3: object median
    int* scan;             // [C/2] interior children per task
    int* first[2];         // [C/2] lowest cluster of each task, by level parity
    int* ctl;              // [0] tasks, [1] next free index; [2], [3] grid barrier
    float4* nbmin;
    float4* nbmax;
    int* parent;
    int* left;
    int* right;
    int* err;
};

// AABB area as the reference's kernels evaluate it under fast-math contraction.
__device__ __forceinline__ float bin_area(float mnx, float mny, float mnz, float mxx, float mxy, float mxz) {
    const float x = __fsub_rn(mxx, mnx), y = __fsub_rn(mxy, mny), z = __fsub_rn(mxz, mnz);
    return __fmul_rn(2.0f, __fmaf_rn(y, z, __fmaf_rn(x, y, __fmul_rn(x, z))));
}

struct sbin {
    float mn[3], mx[3];
    int cnt;
};

__device__ __forceinline__ sbin shfl_bin(const sbin& b, bool down, int delta) {
    sbin o;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        o.mn[a] = down ? __shfl_down_sync(HP_FULL_MASK, b.mn[a], delta) : __shfl_up_sync(HP_FULL_MASK, b.mn[a], delta);
        o.mx[a] = down ? __shfl_down_sync(HP_FULL_MASK, b.mx[a], delta) : __shfl_up_sync(HP_FULL_MASK, b.mx[a], delta);
    }
    o.cnt = down ? __shfl_down_sync(HP_FULL_MASK, b.cnt, delta) : __shfl_up_sync(HP_FULL_MASK, b.cnt, delta);
    return o;
}

__device__ __forceinline__ void bin_add(sbin& a, const sbin& b) {
#pragma unroll
    for (int k = 0; k < 3; ++k) { a.mn[k] = fminf(a.mn[k], b.mn[k]); a.mx[k] = fmaxf(a.mx[k], b.mx[k]); }
    a.cnt += b.cnt;
}

__device__ __forceinline__ void reset_bins(const top_args& A, int T, int gtid, int gthreads) {
    const int words = T * 3 * A.NB * 7;
    for (int w = gtid; w < words; w += gthreads) __stcg(A.bins + w, (w % 7) < 3 ? 0xFFFFFFFFu : 0u);
}

// The split of task t by one warp, lane b holding bin b of an axis: left unions
// by a prefix scan, right unions by a suffix scan, the first strictly lowest
// cost over (axis, bin); all clusters in one bin take the object median.
__device__ void split_task(const top_args& A, const int2* tasks, int t, int lane) {
    const int NB = A.NB;
    float best = MAXF;
    int best_axis = -1, best_bin = -1;
    sbin bl{}, br{};
    int total = 0;
    for (int a = 0; a < 3; ++a) {
        sbin b;
        if (lane < NB) {
            const uint32_t* w = A.bins + ((size_t)(t * 3 + a) * NB + lane) * 7;
            b.mn[0] = hp_ord2f(__ldcg(w + 0)); b.mn[1] = hp_ord2f(__ldcg(w + 1)); b.mn[2] = hp_ord2f(__ldcg(w + 2));
            b.mx[0] = hp_ord2f(__ldcg(w + 3)); b.mx[1] = hp_ord2f(__ldcg(w + 4)); b.mx[2] = hp_ord2f(__ldcg(w + 5));
            b.cnt = (int)__ldcg(w + 6);
        } else {
            for (int k = 0; k < 3; ++k) { b.mn[k] = MAXF; b.mx[k] = -MAXF; }
            b.cnt = 0;
        }
        sbin pre = b, suf = b;  // union of bins 0..lane / lane..NB-1
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const sbin up = shfl_bin(pre, false, o);
            const sbin dn = shfl_bin(suf, true, o);
            if (lane >= o) bin_add(pre, up);
            if (lane + o < 32) bin_add(suf, dn);
        }
        if (a == 0) total = __shfl_sync(HP_FULL_MASK, suf.cnt, 0);
        const sbin right = shfl_bin(suf, true, 1);  // bins lane+1 .. NB-1
        float cost = MAXF;
        if (lane < NB - 1 && pre.cnt > 0 && right.cnt > 0)
            cost = __fmaf_rn((float)pre.cnt, bin_area(pre.mn[0], pre.mn[1], pre.mn[2], pre.mx[0], pre.mx[1], pre.mx[2]),
                             __fmul_rn((float)right.cnt, bin_area(right.mn[0], right.mn[1], right.mn[2], right.mx[0],
                                                                  right.mx[1], right.mx[2])));
        if (!(cost < MAXF)) cost = MAXF;  // a NaN cost never wins
        float m = cost;
        int mb = lane;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float om = __shfl_down_sync(HP_FULL_MASK, m, o);
            const int ob = __shfl_down_sync(HP_FULL_MASK, mb, o);
            if (om < m || (om == m && ob < mb)) { m = om; mb = ob; }
        }
        m = __shfl_sync(HP_FULL_MASK, m, 0);
        mb = __shfl_sync(HP_FULL_MASK, mb, 0);
        if (m < best) {
            best = m;
            best_axis = a;
            best_bin = mb;
            for (int k = 0; k < 3; ++k) {
                bl.mn[k] = __shfl_sync(HP_FULL_MASK, pre.mn[k], mb);
                bl.mx[k] = __shfl_sync(HP_FULL_MASK, pre.mx[k], mb);
                br.mn[k] = __shfl_sync(HP_FULL_MASK, right.mn[k], mb);
                br.mx[k] = __shfl_sync(HP_FULL_MASK, right.mx[k], mb);
            }
            bl.cnt = __shfl_sync(HP_FULL_MASK, pre.cnt, mb);
            br.cnt = __shfl_sync(HP_FULL_MASK, right.cnt, mb);
        } else if (a == 0) {  // no split on x: keep the whole task's box for the median
            for (int k = 0; k < 3; ++k) {
                bl.mn[k] = __shfl_sync(HP_FULL_MASK, suf.mn[k], 0);
                bl.mx[k] = __shfl_sync(HP_FULL_MASK, suf.mx[k], 0);
            }
        }
    }
    if (lane != 0) return;
    const int2 task = __ldcg(tasks + t);
    if (best_axis < 0) {
        // All clusters in one bin: only the last-position leaf and the cluster
        // of key 0 share a cell, so the task holds those two; the object median
        // puts the first in sorted order left.
        if (total != 2) hp_report(A.err, HP_DEV_BAD_INDEX, -4);
        __stcg(A.split + t, make_int4(3, 0, -1, -1));
        __stcg(A.scan + t, 0);
        __stcg(A.nbmin + task.x, make_float4(bl.mn[0], bl.mn[1], bl.mn[2], 0.0f));
        __stcg(A.nbmax + task.x, make_float4(bl.mx[0], bl.mx[1], bl.mx[2], 0.0f));
    } else {
        __stcg(A.nbmin + task.x, make_float4(fminf(bl.mn[0], br.mn[0]), fminf(bl.mn[1], br.mn[1]),
                                             fminf(bl.mn[2], br.mn[2]), 0.0f));
        __stcg(A.nbmax + task.x, make_float4(fmaxf(bl.mx[0], br.mx[0]), fmaxf(bl.mx[1], br.mx[1]),
                                             fmaxf(bl.mx[2], br.mx[2]), 0.0f));
        __stcg(A.split + t, make_int4(best_axis, best_bin, bl.cnt > 1 ? 1 : -1, br.cnt > 1 ? 1 : -1));
        __stcg(A.scan + t, (bl.cnt > 1) + (br.cnt > 1));
    }
    __stcg(A.parent + task.x, task.y);
}

// Interior children of the level's tasks take the next free indices in task
// order, left before right (one CTA: an exclusive scan over the tasks).
__device__ void allocate_children(const top_args& A, const int2* tasks, int2* next, int T, int F) {
    __shared__ int s_chunk[TOPB / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int next_free = __ldcg(A.ctl + 1);
    int running = 0;
    for (int base = 0; base < T; base += TOPB) {
        const int t = base + tid;
        const int x = t < T ? __ldcg(A.scan + t) : 0;
        int inc = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(HP_FULL_MASK, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) s_chunk[warp] = inc;
        __syncthreads();
        int woff = 0, total = 0;
        for (int w = 0; w < TOPB / 32; ++w) {
            if (w < warp) woff += s_chunk[w];
            total += s_chunk[w];
        }
        if (t < T) {
            int4 sp = __ldcg(A.split + t);
            const int2 task = __ldcg(tasks + t);
            int k = running + woff + inc - x;
            if (next_free + k + x > F || k + x > A.tmax) {
                hp_report(A.err, HP_DEV_BAD_INDEX, -5);
                sp.z = sp.w = -1;
            } else {
                if (sp.z > 0) {
                    const int node = __ldcg(A.free_idx + next_free + k);
                    __stcg(next + k, make_int2(node, task.x));
                    __stcg(A.left + task.x, node);
                    sp.z = k++;
                }
                if (sp.w > 0) {
                    const int node = __ldcg(A.free_idx + next_free + k);
                    __stcg(next + k, make_int2(node, task.x));
                    __stcg(A.right + task.x, node);
                    sp.w = k++;
                }
            }
            __stcg(A.split + t, sp);
        }
        running += total;
        __syncthreads();
    }
    if (tid == 0) {
        __stcg(A.ctl + 0, running);
        __stcg(A.ctl + 1, next_free + running);
    }
}

// The top tree over the clusters: a cooperative grid, level by level, with four
// grid barriers a level (after binning, splitting, allocating, distributing).
__global__ void __launch_bounds__(TOPB) k_hl_top(top_args A) {
    const int C = __ldcg(A.totals), F = __ldcg(A.totals + 1);
    if (C < 2 || F != C - 1) return;  // a single cluster, or the root inside a cluster: keep the LBVH
    const int tid = threadIdx.x, lane = tid & 31;
    const int gtid = blockIdx.x * TOPB + tid, gthreads = gridDim.x * TOPB;
    unsigned* bar = reinterpret_cast<unsigned*>(A.ctl + 2);
    for (int c = gtid; c < C; c += gthreads) __stcg(A.task_of + c, 0);
    reset_bins(A, 1, gtid, gthreads);
    if (gtid == 0) {
        __stcg(A.first[0], 0x7fffffff);
        __stcg(A.tasks[0], make_int2(__ldcg(A.free_idx), -1));
        __stcg(A.ctl + 0, 1);
        __stcg(A.ctl + 1, 1);
    }
    if (!hp_grid_barrier(bar, A.err, HP_SPIN_LIMIT)) return;
    for (int level = 0;; ++level) {
        const int T = __ldcg(A.ctl);
        if (T == 0) break;
        if (level > C || T > A.tmax) {  // the same on every CTA
            if (gtid == 0) hp_report(A.err, HP_DEV_BAD_INDEX, -3);
            return;
        }
        const int2* tasks = A.tasks[level & 1];
        int2* next = A.tasks[(level + 1) & 1];
        int* first = A.first[level & 1];
        // bin the clusters
        for (int c = gtid; c < C; c += gthreads) {
            const int t = __ldcg(A.task_of + c);
            if (t < 0) continue;
            if (t >= T) { hp_report(A.err, HP_DEV_BAD_INDEX, -6); continue; }
            const int v = __ldcg(A.cl_node + c), cell = __ldcg(A.cl_cell + c);
            const float4 mn = __ldcg(A.nbmin + v), mx = __ldcg(A.nbmax + v);
            atomicMin(first + t, c);
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const int coord = (cell >> (10 * a)) & 1023;
                uint32_t* b = A.bins + ((size_t)(t * 3 + a) * A.NB + coord) * 7;
                atomicMin(b + 0, hp_f2ord(mn.x));
                atomicMin(b + 1, hp_f2ord(mn.y));
                atomicMin(b + 2, hp_f2ord(mn.z));
                atomicMax(b + 3, hp_f2ord(mx.x));
                atomicMax(b + 4, hp_f2ord(mx.y));
                atomicMax(b + 5, hp_f2ord(mx.z));
                atomicAdd(b + 6, 1u);
            }
        }
        if (!hp_grid_barrier(bar, A.err, HP_SPIN_LIMIT)) return;
        for (int t = gtid >> 5; t < T; t += gthreads >> 5) split_task(A, tasks, t, lane);
        if (!hp_grid_barrier(bar, A.err, HP_SPIN_LIMIT)) return;
        if (blockIdx.x == 0) allocate_children(A, tasks, next, T, F);
        if (!hp_grid_barrier(bar, A.err, HP_SPIN_LIMIT)) return;
        // hand the clusters to the child tasks; a single cluster is its side's child
        const int Tn = __ldcg(A.ctl);
        for (int c = gtid; c < C; c += gthreads) {
            const int t = __ldcg(A.task_of + c);
            if (t < 0 || t >= T) continue;
            const int4 sp = __ldcg(A.split + t);
            const bool go_left = sp.x == 3 ? c == __ldcg(first + t) : ((__ldcg(A.cl_cell + c) >> (10 * sp.x)) & 1023) <= sp.y;
            const int nt = go_left ? sp.z : sp.w;
            if (nt >= 0) {
                __stcg(A.task_of + c, nt);
            } else {
                const int node = __ldcg(tasks + t).x, v = __ldcg(A.cl_node + c);
                __stcg((go_left ? A.left : A.right) + node, v);
                __stcg(A.parent + v, node);
                __stcg(A.task_of + c, -1);
            }
        }
        if (Tn <= A.tmax) {
            reset_bins(A, Tn, gtid, gthreads);
            for (int t = gtid; t < Tn; t += gthreads) __stcg(A.first[(level + 1) & 1] + t, 0x7fffffff);
        }
        if (!hp_grid_barrier(bar, A.err, HP_SPIN_LIMIT)) return;
    }
}

template <typename K>
hp_status hlbvh_t(hp_ctx* ctx, const hp_build_params* p, int n, const K* skeys, const int32_t* sorted_tri,
                  const float4* tbmin, const float4* tbmax, int* parent, int* left, int* right, const int2* range,
                  float4* nbmin, float4* nbmax, int* counters, void* scratch, cudaStream_t s) {
    const int sah = p->hlbvh_sah_bits;
    const int NB = 1 << (sah / 3);
    const int cmax = std::min(n, 1 << sah);
    const int tmax = std::max(cmax / 2, 1);
    int* err = ctx->d_status;
    hp_carve cv(reinterpret_cast<char*>(scratch));
    int* state = cv.take<int>(n);
    int* cluster_flag = cv.take<int>(n);
    int* cluster_at = cv.take<int>(n);
    int* top_flag = cv.take<int>(n);
    int* cluster_off = cv.take<int>(n);
    int* top_off = cv.take<int>(n);
    int* totals = cv.take<int>(2);
    void* scan = cv.take<char>(hp_scan2_scratch_bytes(n));
    int* cl_node = cv.take<int>(cmax);
    int* cl_cell = cv.take<int>(cmax);
    int* free_idx = cv.take<int>(n);
    top_args A{};
    A.n = n;
    A.NB = NB;
    A.tmax = tmax;
    A.totals = totals;
    A.cl_node = cl_node;
    A.cl_cell = cl_cell;
    A.free_idx = free_idx;
    A.task_of = cv.take<int>(cmax);
    A.tasks[0] = cv.take<int2>(tmax);
    A.tasks[1] = cv.take<int2>(tmax);
    A.bins = cv.take<uint32_t>((size_t)tmax * 3 * NB * 7);
    A.split = cv.take<int4>(tmax);
    A.scan = cv.take<int>(tmax);
    A.first[0] = cv.take<int>(tmax);
    A.first[1] = cv.take<int>(tmax);
    A.ctl = cv.take<int>(4);
    A.nbmin = nbmin;
    A.nbmax = nbmax;
    A.parent = parent;
    A.left = left;
    A.right = right;
    A.err = err;

    HP_CUDA(cudaMemsetAsync(counters, 0, (size_t)n * 4, s));
    HP_CUDA(cudaMemsetAsync(cluster_flag, 0, (size_t)n * 4, s));
    k_hl_refit<<<hp_div_up(n, HB), HB, 0, s>>>(n, sorted_tri, tbmin, tbmax, parent, left, right, nbmin, nbmax,
                                              counters, err);
    k_hl_mark<K><<<hp_div_up(n, HB), HB, 0, s>>>(n, skeys, p->morton_bits, sah, left, state, top_flag);
    k_hl_clusters<<<hp_div_up(2 * n - 1, HB), HB, 0, s>>>(n, parent, range, state, cluster_flag, cluster_at);
    hp_scan2_sum(cluster_flag, n, top_flag, n - 1, cluster_off, top_off, totals, scan, err, s);
    k_hl_scatter<K><<<hp_div_up(n, HB), HB, 0, s>>>(n, skeys, p->morton_bits, sah, cluster_flag, cluster_at,
                                                    cluster_off, top_flag, top_off, cl_node, cl_cell, free_idx);
    HP_CUDA(cudaGetLastError());
    hp_count_launch(4);
    hp_mark(ctx, s, "hlbvh_clusters");
    // A cooperative grid sized to the clusters it may hold, every CTA resident.
    int per_sm = 0;
    HP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_hl_top, TOPB, 0));
    if (per_sm < 1) return hp_fail(HP_ERR_UNSUPPORTED, "HLBVH top-tree kernel does not fit on an SM");
    const int grid = std::max(1, std::min(ctx->sm_count * std::min(per_sm, 2), hp_div_up(cmax, 256)));
    HP_CUDA(cudaMemsetAsync(A.ctl, 0, 16, s));
    void* args[] = {&A};
    HP_CUDA(cudaLaunchCooperativeKernel((void*)k_hl_top, grid, TOPB, args, 0, s));
    hp_count_launch();
    hp_mark(ctx, s, "hlbvh_top");
    return HP_OK;
}

}  // namespace

size_t hp_hlbvh_scratch_bytes(int64_t n, int sah_bits) {
    const int64_t NB = 1 << (sah_bits / 3);
    const int64_t cmax = std::min<int64_t>(n, (int64_t)1 << sah_bits);
    const int64_t tmax = std::max<int64_t>(cmax / 2, 1);
    size_t b = 0;
    b += 6 * hp_carve::pad(n * 4) + hp_carve::pad(8) + hp_carve::pad(hp_scan2_scratch_bytes(n));
    b += 2 * hp_carve::pad(cmax * 4) + hp_carve::pad(n * 4);
    b += hp_carve::pad(cmax * 4) + 2 * hp_carve::pad(tmax * 8);
    b += hp_carve::pad((size_t)tmax * 3 * NB * 7 * 4) + hp_carve::pad(tmax * 16) + 3 * hp_carve::pad(tmax * 4);
    b += hp_carve::pad(16);
    return b;
}

hp_status hp_hlbvh_stage(hp_ctx* ctx, const hp_build_params* p, int n, const void* skeys, int key_bytes,
                         const int32_t* sorted_tri, const float4* tbmin, const float4* tbmax, int* parent, int* left,
                         int* right, const int2* range, float4* nbmin, float4* nbmax, int* counters, void* scratch,
                         cudaStream_t s) {
    const int sah = p->hlbvh_sah_bits;
    if (sah % 3 != 0 || sah < 6 || sah > 15 || sah > p->morton_bits)
        return hp_fail(HP_ERR_UNSUPPORTED, "HLBVH: Morton code SAH bits must be a multiple of 3 in [6,15] and at "
                                           "most the Morton code bits");
    if (n < 2) return HP_OK;
    if (key_bytes == 8)
        return hlbvh_t<uint64_t>(ctx, p, n, reinterpret_cast<const uint64_t*>(skeys), sorted_tri, tbmin, tbmax,
                                 parent, left, right, range, nbmin, nbmax, counters, scratch, s);
    return hlbvh_t<uint32_t>(ctx, p, n, reinterpret_cast<const uint32_t*>(skeys), sorted_tri, tbmin, tbmax, parent,
                             left, right, range, nbmin, nbmax, counters, scratch, s);
}
