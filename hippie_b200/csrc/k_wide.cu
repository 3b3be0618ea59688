// N-wide BVH layouts (Quad, N = 4; Oct, N = 8): the collapse of a built binary
// tree into N-wide nodes, and the closest-hit / any-hit tracer for them.
//
// Reference (paths relative to src/hippie/):
//   BVHCollapser::collapseAdaptive / collapse for Quad and Oct
//     (rt/bvh/BVHCollapser.cpp:521-660): the binary tree is copied to the host,
//     BVH::collapseAdaptiveWide(N) / collapseWide(N, maxLeafSize)
//     (rt/bvh/BVH.h:94-160, 228-292, 401-423) collapses it there, and
//     BVHConverter::convert (rt/bvh/BVHConverter.cpp:13-89) numbers the result
//     breadth first into HipBVHNodeN<N> records (rt/bvh/HipBVHNode.h:14-114);
//   HipTracer with the Quad / Oct kernels (rt/tracer/HipTracerQuadKernels.cu,
//     HipTracerOctKernels.cu): a sub-warp of lanes per ray, one lane per child.
//
// The collapse runs on the device:
//   1. a bottom-up climb (one thread per binary leaf, the second thread to
//      reach a node carries on) evaluates recomputeCostsWide: per node and
//      child budget j = 1..N-1 the cost and the split (k, j-k) of the budget
//      between the children, or "leaf"; leaf costs of the binary leaves are
//      formed where they are read;
//   2. the N-wide tree is expanded level by level from the root: each wide
//      node starts from its binary children with the split of its budget and
//      replaces, while it has fewer than N children, the first child whose
//      split (l, r) has l + r < N by that child's two children (collapseWide);
//      children whose budget says "leaf" become leaves. One cooperative
//      launch runs every level (k_wide_levels): the CTAs count the interior
//      and leaf children of their chunk of the level, and after a grid
//      barrier each scans its chunk from the totals of the CTAs before it and
//      writes the next level, so interior nodes are numbered in breadth-first
//      order and leaves after them in breadth-first order, as
//      BVHConverter::convert numbers them, with no host round trip;
//   3. one kernel writes every wide node and the leaves below it, and walks
//      each leaf's binary subtree (parent links, no stack) to write the leaf's
//      references in left-first depth-first order with their Woop triangles.
// Costs use AABB::area as written, 2 * (dx*dy + dy*dz + dz*dx), and the cost
// expressions in their source order (ci * A / A(root) * ceil(size/N) * N), each
// step rounded as IEEE single precision like the reference's host code.
// Where the root's best choice is a leaf (tiny meshes) the reference reads
// outside its count arrays; here the root then takes its best interior split.
//
// Node record (32*N bytes, HipBVHNodeN<N>): child i's x/y bounds in int4 i,
// its z bounds, index (~index for a leaf) and one spare word in int4 N+i; the
// spare words of children N-3, N-2, N-1 hold the child count, the size (~size
// for a leaf) and the parent; a leaf keeps its reference range in the index
// and spare words of child 0 and its box in every child slot. Unused child
// slots repeat child 0's minimum corner as an empty box and child 0's
// (decoded) index; the tracer never reads them.
#include <algorithm>
#include <vector>
#include <cuda_runtime.h>
#include "hp_device.cuh"
#include "hp_internal.h"

namespace {

constexpr int WB = 256;                 // threads per build CTA
constexpr uint16_t CNT_LEAF = 0xFFFF;  // split of a budget: leaf
constexpr float MAXF = 3.402823466e+38f;

// AABB::area (util/AABB.h:36) as the reference's host code evaluates it.
__device__ __forceinline__ float host_area(const float4& mn, const float4& mx) {
    if (!(mn.x <= mx.x && mn.y <= mx.y && mn.z <= mx.z)) return 0.0f;
    const float dx = __fsub_rn(mx.x, mn.x), dy = __fsub_rn(mx.y, mn.y), dz = __fsub_rn(mx.z, mn.z);
    return __fmul_rn(2.0f, __fadd_rn(__fadd_rn(__fmul_rn(dx, dy), __fmul_rn(dy, dz)), __fmul_rn(dz, dx)));
}

// ci * A / A(root) * ceil(size / N) * N
template <int N>
__device__ __forceinline__ float leaf_cost(float ci, float a, float root_a, int size) {
    return __fmul_rn(__fmul_rn(__fdiv_rn(__fmul_rn(ci, a), root_a), (float)((size + N - 1) / N)), (float)N);
}

struct wide_args {
    int n;
    const int* parent;
    const int* left;
    const int* right;
    const float4* nbmin;
    const float4* nbmax;
    float ct, ci;
    int max_leaf;
    int* counters;      // [n-1] arrival counters
    float* cost;        // [n-1][N-1]
    uint16_t* cnt;      // [n-1][N-1] split (l | r << 8) or CNT_LEAF
    int* size;          // [n-1]
    int* root_split;    // best interior split of the root's budget 1
    int* err;
};

// recomputeCostsWide (rt/bvh/BVH.h:94-143) in a bottom-up climb.
template <int N>
__global__ void __launch_bounds__(WB) k_wide_dp(wide_args A) {
    constexpr int J = N - 1;
    const int n = A.n;
    const int p = blockIdx.x * WB + threadIdx.x;
    if (p >= n) return;
    const float root_a = host_area(__ldg(A.nbmin), __ldg(A.nbmax));
    int cur = __ldg(A.parent + n - 1 + p);
    int steps = 0;
    while (cur >= 0) {
        if (cur >= n - 1 || ++steps > n) { hp_report(A.err, HP_DEV_BAD_INDEX, cur); return; }
        if (hp_arrive(A.counters + cur) == 0) return;
        const int ch[2] = {__ldcg(A.left + cur), __ldcg(A.right + cur)};
        float c[2][J];
        int sz[2];
        for (int s = 0; s < 2; ++s) {
            const int x = ch[s];
            if ((unsigned)x >= (unsigned)(2 * n - 1)) { hp_report(A.err, HP_DEV_BAD_INDEX, cur); return; }
            if (x >= n - 1) {
                const float lc = leaf_cost<N>(A.ci, host_area(__ldcg(A.nbmin + x), __ldcg(A.nbmax + x)), root_a, 1);
#pragma unroll
                for (int j = 0; j < J; ++j) c[s][j] = lc;
                sz[s] = 1;
            } else {
#pragma unroll
                for (int j = 0; j < J; ++j) c[s][j] = __ldcg(A.cost + (size_t)x * J + j);
                sz[s] = __ldcg(A.size + x);
            }
        }
        const int size = sz[0] + sz[1];
        const float a = host_area(__ldcg(A.nbmin + cur), __ldcg(A.nbmax + cur));
        float* oc = A.cost + (size_t)cur * J;
        uint16_t* on = A.cnt + (size_t)cur * J;
        const float lc = size > A.max_leaf ? MAXF : leaf_cost<N>(A.ci, a, root_a, size);
        float sub = __fdiv_rn(__fmul_rn(A.ct, a), root_a);
        float dist = MAXF;
        int bk = 0;
#pragma unroll
        for (int k = 1; k < N; ++k) {
            const float cc = __fadd_rn(c[0][k - 1], c[1][N - k - 1]);
            if (dist > cc) { dist = cc; bk = k; }
        }
        sub = __fadd_rn(sub, dist);
        if (cur == 0) *A.root_split = bk | ((N - bk) << 8);
        float prev;
        uint16_t prev_n;
        if (lc > sub) { prev = sub; prev_n = (uint16_t)(bk | ((N - bk) << 8)); }
        else { prev = lc; prev_n = CNT_LEAF; }
        __stcg(oc, prev);
        __stcg(on, prev_n);
#pragma unroll
        for (int j = 2; j < N; ++j) {
            dist = MAXF;
            for (int k = 1; k < j; ++k) {
                const float cc = __fadd_rn(c[0][k - 1], c[1][j - k - 1]);
                if (dist > cc) { dist = cc; bk = k; }
            }
            if (!(prev <= dist)) { prev = dist; prev_n = (uint16_t)(bk | ((j - bk) << 8)); }
            __stcg(oc + j - 1, prev);
            __stcg(on + j - 1, prev_n);
        }
        __stcg(A.size + cur, size);
        cur = __ldcg(A.parent + cur);
    }
}

struct wide_entry {
    int v, k, begin, parent;
};

struct expand_args {
    int n;
    const int* left;
    const int* right;
    const uint16_t* cnt;
    const int* size;
    const int* root_split;
    int* err;
};

template <int N>
__device__ __forceinline__ uint16_t cnt_of(const expand_args& E, int x, int k) {
    if (x >= E.n - 1) return CNT_LEAF;
    return __ldg(E.cnt + (size_t)x * (N - 1) + k - 1);
}
__device__ __forceinline__ int size_of(const expand_args& E, int x) { return x >= E.n - 1 ? 1 : __ldg(E.size + x); }

// collapseWide (rt/bvh/BVH.h:228-292) for one wide node: its children as
// (binary node, budget, first reference, leaf?). Returns the child count, 0 on
// a bad index.
template <int N>
__device__ int expand(const expand_args& E, const wide_entry& e, int* kv, int* kk, int* kb, bool* kl) {
    const int nn = 2 * E.n - 1;
    if ((unsigned)e.v >= (unsigned)(E.n - 1) || e.k < 1 || e.k >= N) return 0;
    uint16_t c = cnt_of<N>(E, e.v, e.k);
    if (c == CNT_LEAF) c = (uint16_t)__ldg(E.root_split);  // only the root can be here
    const int l0 = __ldg(E.left + e.v), r0 = __ldg(E.right + e.v);
    if ((unsigned)l0 >= (unsigned)nn || (unsigned)r0 >= (unsigned)nn) return 0;
    // each child's split is read once, when the child enters the list
    uint16_t cs[N];
    kv[0] = l0; kk[0] = c & 0xFF; kb[0] = e.begin;
    kv[1] = r0; kk[1] = c >> 8; kb[1] = e.begin + size_of(E, l0);
    cs[0] = cnt_of<N>(E, l0, kk[0]);
    cs[1] = cnt_of<N>(E, r0, kk[1]);
    int m = 2;
    while (m < N) {
        int s = -1, l = 0, r = 0;
        for (int i = 0; i < m; ++i) {
            const uint16_t ci = cs[i];
            if (ci == CNT_LEAF) continue;
            const int li = ci & 0xFF, ri = ci >> 8;
            if (li > 0 && ri > 0 && li + ri < N) { s = i; l = li; r = ri; break; }
        }
        if (s < 0) break;
        const int x = kv[s], b = kb[s];
        const int xl = __ldg(E.left + x), xr = __ldg(E.right + x);
        if ((unsigned)xl >= (unsigned)nn || (unsigned)xr >= (unsigned)nn) return 0;
        for (int i = m; i > s + 1; --i) { kv[i] = kv[i - 1]; kk[i] = kk[i - 1]; kb[i] = kb[i - 1]; cs[i] = cs[i - 1]; }
        kv[s] = xl; kk[s] = l; kb[s] = b;
        kv[s + 1] = xr; kk[s + 1] = r; kb[s + 1] = b + size_of(E, xl);
        cs[s] = cnt_of<N>(E, xl, l);
        cs[s + 1] = cnt_of<N>(E, xr, r);
        ++m;
    }
    for (int i = 0; i < m; ++i) kl[i] = cs[i] == CNT_LEAF;
    return m;
}

// All levels of the breadth-first expansion in one cooperative launch (the
// counts, the exclusive scans and the placement of every level, with two grid
// barriers a level instead of a host round trip). Level entries are split
// into one contiguous chunk per CTA: a CTA counts its entries' interior and
// leaf children, publishes its totals, and after the barrier takes its offset
// from the totals of the CTAs before it and scans and places its chunk in
// order. result[0] and result[1] receive the interior and leaf counts.
constexpr int LB = 256;
constexpr unsigned LEVEL_SPIN = 1u << 22;
constexpr int LEVEL_MAX_CTAS = 1024;

struct level_args {
    expand_args E;
    int n;
    wide_entry* entries;  // [n]: level after level; the root is entries[0]
    int2* kid_base;
    int* ni;
    int* nl;
    int2* cta_sum;        // [grid]
    unsigned* bar;        // [2] grid barrier words, zero
    int* result;          // [2]
    int* err;
};

__device__ __forceinline__ int2 lb_scan_excl(int x, int y, int2* s_w, int2& total) {
    // exclusive block scan of (x, y) over LB threads
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int ix = x, iy = y;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int ux = __shfl_up_sync(HP_FULL_MASK, ix, o), uy = __shfl_up_sync(HP_FULL_MASK, iy, o);
        if (lane >= o) { ix += ux; iy += uy; }
    }
    if (lane == 31) s_w[warp] = make_int2(ix, iy);
    __syncthreads();
    int bx = 0, by = 0, tx = 0, ty = 0;
#pragma unroll
    for (int w = 0; w < LB / 32; ++w) {
        const int2 v = s_w[w];
        if (w < warp) { bx += v.x; by += v.y; }
        tx += v.x; ty += v.y;
    }
    __syncthreads();
    total = make_int2(tx, ty);
    return make_int2(bx + ix - x, by + iy - y);
}

template <int N>
__global__ void __launch_bounds__(LB) k_wide_levels(level_args L) {
    __shared__ int2 s_w[LB / 32];
    __shared__ int s_pre[4];
    const int G = gridDim.x, cta = blockIdx.x, tid = threadIdx.x, lane = tid & 31;
    // the root entry (binary root 0 with the whole budget); the same thread
    // expands it in the first level (chunk 0 of one entry)
    if (cta == 0 && tid == 0) L.entries[0] = wide_entry{0, 1, 0, -1};
    int base = 0, m = 1, leaves = 0;
    while (m > 0) {
        if (base + m > L.n) {  // every CTA sees the same counts
            if (cta == 0 && tid == 0) hp_report(L.err, HP_DEV_BAD_INDEX, base + m);
            break;
        }
        const wide_entry* level = L.entries + base;
        const int chunk = (m + G - 1) / G;
        const int lo = min(m, cta * chunk), hi = min(m, lo + chunk);
        int a = 0, b = 0;
        for (int i = lo + tid; i < hi; i += LB) {
            int kv[N], kk[N], kb[N];
            bool kl[N];
            const int c = expand<N>(L.E, level[i], kv, kk, kb, kl);
            if (c == 0) hp_report(L.err, HP_DEV_BAD_INDEX, level[i].v);
            int x = 0, y = 0;
            for (int j = 0; j < c; ++j) (kl[j] ? y : x)++;
            L.ni[i] = x;
            L.nl[i] = y;
            a += x;
            b += y;
        }
        int2 tot;
        lb_scan_excl(a, b, s_w, tot);
        if (tid == 0) __stcg(L.cta_sum + cta, tot);
        if (!hp_grid_barrier(L.bar, L.err, LEVEL_SPIN)) return;
        if (tid < 32) {  // this CTA's offset and the level's totals
            int pa = 0, pb = 0, ta = 0, tb = 0;
            for (int j = lane; j < G; j += 32) {
                const int2 v = __ldcg(L.cta_sum + j);
                if (j < cta) { pa += v.x; pb += v.y; }
                ta += v.x;
                tb += v.y;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                pa += __shfl_xor_sync(HP_FULL_MASK, pa, o);
                pb += __shfl_xor_sync(HP_FULL_MASK, pb, o);
                ta += __shfl_xor_sync(HP_FULL_MASK, ta, o);
                tb += __shfl_xor_sync(HP_FULL_MASK, tb, o);
            }
            if (lane == 0) { s_pre[0] = pa; s_pre[1] = pb; s_pre[2] = ta; s_pre[3] = tb; }
        }
        __syncthreads();
        int run_a = s_pre[0], run_b = s_pre[1];
        const int tot_a = s_pre[2], tot_b = s_pre[3];
        const int next_base = base + m;
        if (next_base + tot_a > L.n) {
            if (cta == 0 && tid == 0) hp_report(L.err, HP_DEV_BAD_INDEX, next_base + tot_a);
            break;
        }
        for (int r0 = lo; r0 < hi; r0 += LB) {  // uniform over the CTA
            const int i = r0 + tid;
            const int x = i < hi ? __ldcg(L.ni + i) : 0, y = i < hi ? __ldcg(L.nl + i) : 0;
            int2 sum;
            const int2 ex = lb_scan_excl(x, y, s_w, sum);
            if (i < hi) {
                int kv[N], kk[N], kb[N];
                bool kl[N];
                const int c = expand<N>(L.E, level[i], kv, kk, kb, kl);
                int o = next_base + run_a + ex.x;
                for (int j = 0; j < c; ++j)
                    if (!kl[j]) L.entries[o++] = wide_entry{kv[j], kk[j], kb[j], base + i};
                L.kid_base[base + i] = make_int2(next_base + run_a + ex.x, leaves + run_b + ex.y);
            }
            run_a += sum.x;
            run_b += sum.y;
        }
        if (!hp_grid_barrier(L.bar, L.err, LEVEL_SPIN)) return;
        leaves += tot_b;
        base = next_base;
        m = tot_a;
    }
    if (cta == 0 && tid == 0) {
        L.result[0] = base;
        L.result[1] = leaves;
    }
}

struct emit_args {
    int n, num_refs;
    const int* counts;          // [0] interior records, [1] leaf records (k_wide_levels)
    int4* leaf_task;            // per leaf record: binary node, first reference, size, parent
    const wide_entry* entries;  // [num_interior], breadth-first
    const int2* kid_base;
    const int* parent;
    const int* left;
    const int* right;
    const float4* nbmin;
    const float4* nbmax;
    const int32_t* sorted_tri;  // sorted position -> triangle
    bool reorder;               // write the references in depth-first order (else kept)
    int32_t* tri_out;
    float4* woop;
    const float* verts;
    int64_t nv;
    const int32_t* tris;
    int4* nodes;
    int* err;
};

template <int N>
__device__ __forceinline__ void put_child(int4* nd, int i, const float4& mn, const float4& mx, int ref, int spare) {
    nd[i] = make_int4(__float_as_int(mn.x), __float_as_int(mx.x), __float_as_int(mn.y), __float_as_int(mx.y));
    nd[N + i] = make_int4(__float_as_int(mn.z), __float_as_int(mx.z), ref, spare);
}

template <int N>
__global__ void __launch_bounds__(WB) k_wide_emit(expand_args E, emit_args M) {
    const int w = blockIdx.x * WB + threadIdx.x;
    const int num_interior = __ldg(M.counts);
    if (w >= num_interior) return;
    const wide_entry e = M.entries[w];
    int kv[N], kk[N], kb[N];
    bool kl[N];
    const int c = expand<N>(E, e, kv, kk, kb, kl);
    if (c == 0) { hp_report(M.err, HP_DEV_BAD_INDEX, e.v); return; }
    const int2 base = M.kid_base[w];
    int ni = 0, nl = 0;
    int refs[N];
    for (int j = 0; j < c; ++j) refs[j] = kl[j] ? ~(num_interior + base.y + nl++) : base.x + ni++;
    // spare words: child N-3 -> count, N-2 -> size, N-1 -> parent
    int spare[N];
    for (int i = 0; i < N; ++i) spare[i] = 0;
    spare[N - 3] = c;
    spare[N - 2] = size_of(E, e.v);
    spare[N - 1] = e.parent;
    int4* nd = M.nodes + (size_t)w * 2 * N;
    const float4 mn0 = __ldg(M.nbmin + kv[0]);
    const int d0 = refs[0] < 0 ? ~refs[0] : refs[0];
    for (int i = 0; i < N; ++i) {
        if (i < c) put_child<N>(nd, i, __ldg(M.nbmin + kv[i]), __ldg(M.nbmax + kv[i]), refs[i], spare[i]);
        else put_child<N>(nd, i, mn0, mn0, d0, spare[i]);
    }
    // the leaves below this node: one task each for k_wide_leaf_emit
    for (int j = 0; j < c; ++j) {
        if (!kl[j]) continue;
        const int li = ~refs[j];
        M.leaf_task[li - num_interior] = make_int4(kv[j], kb[j], size_of(E, kv[j]), w);
    }
}

// One thread per leaf record: its N child slots (the leaf box in each, the
// reference range in slot 0, size and parent in the spare words), and, when
// the references are reordered, the binary subtree's leaves walked left first
// through the parent links (no stack) with their triangle ids and Woop rows.
template <int N>
__global__ void __launch_bounds__(WB) k_wide_leaf_emit(expand_args E, emit_args M) {
    const int t = blockIdx.x * WB + threadIdx.x;
    const int num_interior = __ldg(M.counts), num_leaf = __ldg(M.counts + 1);
    if (t >= num_leaf) return;
    const int4 task = M.leaf_task[t];
    const int li = num_interior + t, v = task.x, b = task.y, s = task.z, w = task.w;
    const int n = M.n;
    if ((unsigned)v >= (unsigned)(2 * n - 1)) { hp_report(M.err, HP_DEV_BAD_INDEX, v); return; }
    const float4 mn = __ldg(M.nbmin + v), mx = __ldg(M.nbmax + v);
    int4* lf = M.nodes + (size_t)li * 2 * N;
    for (int i = 0; i < N; ++i) {
        int sp = 0;
        if (i == N - 3) sp = 0;
        else if (i == N - 2) sp = ~s;
        else if (i == N - 1) sp = w;
        if (i == 0) put_child<N>(lf, 0, mn, mx, b, b + s);
        else put_child<N>(lf, i, mn, mx, 0, sp);
    }
    if (b < 0 || b + s > M.num_refs) { hp_report(M.err, HP_DEV_BAD_INDEX, v); return; }
    if (!M.reorder) return;
    int x = v, pos = b, guard = 0;
    while (x < n - 1) x = __ldg(M.left + x);
    while (true) {
        if (pos >= b + s || ++guard > 4 * s + 4) { hp_report(M.err, HP_DEV_BAD_INDEX, v); break; }
        const int tri = __ldg(M.sorted_tri + (x - (n - 1)));
        M.tri_out[pos] = tri;
        tri_verts tv = load_tri(M.verts, M.nv, M.tris, tri, M.err);
        float4 w0, w1, w2;
        hp_woop(tv.x0, tv.y0, tv.z0, tv.x1, tv.y1, tv.z1, tv.x2, tv.y2, tv.z2, w0, w1, w2);
        M.woop[3 * (int64_t)pos] = w0;
        M.woop[3 * (int64_t)pos + 1] = w1;
        M.woop[3 * (int64_t)pos + 2] = w2;
        ++pos;
        // next leaf: climb while x is a right child, then step right and descend left
        bool done = false;
        while (true) {
            if (x == v) { done = true; break; }
            const int p = __ldg(M.parent + x);
            if (p < 0) { done = true; break; }
            if (__ldg(M.left + p) == x) { x = __ldg(M.right + p); break; }
            x = p;
        }
        if (done) break;
        while (x < n - 1) x = __ldg(M.left + x);
    }
}

__global__ void k_wide_info(hp_bvh_info* info, const int* counts) {
    if (threadIdx.x == 0) {
        info->num_interior = counts[0];
        info->num_leaf = counts[1];
    }
}

// A single reference: a root with one leaf child.
template <int N>
__global__ void k_wide_single(const float* verts, int64_t nv, const int32_t* tris, int4* nodes, float4* woop,
                              int32_t* tri_idx, hp_bvh_info* info, int* err) {
    if (threadIdx.x != 0) return;
    tri_verts t = load_tri(verts, nv, tris, 0, err);
    float4 w0, w1, w2;
    hp_woop(t.x0, t.y0, t.z0, t.x1, t.y1, t.z1, t.x2, t.y2, t.z2, w0, w1, w2);
    woop[0] = w0; woop[1] = w1; woop[2] = w2;
    tri_idx[0] = 0;
    const float4 mn = make_float4(fminf(fminf(t.x0, t.x1), t.x2), fminf(fminf(t.y0, t.y1), t.y2),
                                  fminf(fminf(t.z0, t.z1), t.z2), 0.0f);
    const float4 mx = make_float4(fmaxf(fmaxf(t.x0, t.x1), t.x2), fmaxf(fmaxf(t.y0, t.y1), t.y2),
                                  fmaxf(fmaxf(t.z0, t.z1), t.z2), 0.0f);
    for (int i = 0; i < N; ++i) {
        const int sp = i == N - 3 ? 1 : (i == N - 2 ? 1 : (i == N - 1 ? -1 : 0));
        put_child<N>(nodes, i, mn, i == 0 ? mx : mn, i == 0 ? ~1 : 1, sp);
        const int lsp = i == N - 2 ? ~1 : (i == N - 1 ? 0 : 0);
        if (i == 0) put_child<N>(nodes + 2 * N, 0, mn, mx, 0, 1);
        else put_child<N>(nodes + 2 * N, i, mn, mx, 0, lsp);
    }
    for (int k = 0; k < 3; ++k) {
        info->box_ord[k] = hp_f2ord((&mn.x)[k]);
        info->box_ord[3 + k] = hp_f2ord((&mx.x)[k]);
    }
    info->num_interior = 1;
    info->num_leaf = 1;
}

template <int N>
hp_status wide_collapse_t(hp_ctx* ctx, const hp_wide_in& in, hp_bvh_impl* out, void* scratch, cudaStream_t s) {
    constexpr int J = N - 1;
    const int n = in.n;
    int* err = ctx->d_status;
    hp_carve cv(reinterpret_cast<char*>(scratch));
    int* counters = cv.take<int>(n);
    float* cost = cv.take<float>((size_t)n * J);
    uint16_t* cnt = cv.take<uint16_t>((size_t)n * J);
    int* size = cv.take<int>(n);
    int* root_split = cv.take<int>(1);
    wide_entry* entries = cv.take<wide_entry>(n);
    int2* kid_base = cv.take<int2>(n);
    int* ni = cv.take<int>(n);
    int* nl = cv.take<int>(n);
    int2* cta_sum = cv.take<int2>(LEVEL_MAX_CTAS);
    int* ctl = cv.take<int>(16);  // [0..1] grid barrier, [4..5] interior / leaf record counts
    int4* leaf_task = cv.take<int4>(n);

    HP_CUDA(cudaMemsetAsync(counters, 0, (size_t)n * 4, s));
    wide_args A{n, in.parent, in.left, in.right, in.nbmin, in.nbmax, in.ct, in.ci, in.max_leaf,
                counters, cost, cnt, size, root_split, err};
    k_wide_dp<N><<<hp_div_up(n, WB), WB, 0, s>>>(A);
    HP_CUDA(cudaGetLastError());
    hp_count_launch();
    hp_mark(ctx, s, "wide_costs");

    expand_args E{n, in.left, in.right, cnt, size, root_split, err};
    HP_CUDA(cudaMemsetAsync(ctl, 0, 16 * sizeof(int), s));
    int per_sm = 0;
    HP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_wide_levels<N>, LB, 0));
    if (per_sm < 1) return hp_fail(HP_ERR_UNSUPPORTED, "wide collapse: level kernel does not fit on an SM");
    const int grid = std::min(ctx->sm_count * std::min(per_sm, 4), LEVEL_MAX_CTAS);
    level_args L{E, n, entries, kid_base, ni, nl, cta_sum, reinterpret_cast<unsigned*>(ctl),
                 ctl + 4, err};
    void* largs[] = {&L};
    HP_CUDA(cudaLaunchCooperativeKernel((void*)k_wide_levels<N>, grid, LB, largs, 0, s));
    hp_count_launch();
    hp_mark(ctx, s, "wide_levels");
    emit_args M{n, n, ctl + 4, leaf_task, entries, kid_base, in.parent, in.left, in.right, in.nbmin, in.nbmax,
                in.sorted_tri, in.reorder, out->tri_idx, out->woop, in.verts, in.nv, in.tris,
                reinterpret_cast<int4*>(out->nodes), err};
    k_wide_emit<N><<<hp_div_up(n, WB), WB, 0, s>>>(E, M);  // threads beyond the interior count leave
    k_wide_leaf_emit<N><<<hp_div_up(n, WB), WB, 0, s>>>(E, M);  // threads beyond the leaf count leave
    k_wide_info<<<1, 32, 0, s>>>(out->info, ctl + 4);
    HP_CUDA(cudaGetLastError());
    hp_count_launch(3);
    hp_mark(ctx, s, "wide_collapse");
    return HP_OK;
}

}  // namespace

size_t hp_wide_scratch_bytes(int64_t n, int width) {
    const int J = width - 1;
    size_t b = 0;
    b += hp_carve::pad(n * 4);                       // counters
    b += hp_carve::pad((size_t)n * J * 4);           // costs
    b += hp_carve::pad((size_t)n * J * 2);           // splits
    b += hp_carve::pad(n * 4) + hp_carve::pad(4);    // sizes, root split
    b += hp_carve::pad(n * sizeof(wide_entry));      // breadth-first entries
    b += hp_carve::pad(n * 8);                       // child bases
    b += 2 * hp_carve::pad(n * 4);                   // child counts of a level
    b += hp_carve::pad(LEVEL_MAX_CTAS * 8) + hp_carve::pad(64);  // CTA totals, barrier and counts
    b += hp_carve::pad(n * 16);                      // leaf tasks
    return b;
}

hp_status hp_wide_collapse(hp_ctx* ctx, const hp_wide_in& in, hp_bvh_impl* out, void* scratch, cudaStream_t s) {
    if (in.n < 2) return hp_fail(HP_ERR_ARG, "wide collapse: needs at least two references");
    if (in.width == 4) return wide_collapse_t<4>(ctx, in, out, scratch, s);
    if (in.width == 8) return wide_collapse_t<8>(ctx, in, out, scratch, s);
    return hp_fail(HP_ERR_UNSUPPORTED, "wide collapse: width must be 4 or 8");
}

hp_status hp_wide_single(hp_ctx* ctx, const hp_mesh* m, int width, hp_bvh_impl* out, cudaStream_t s) {
    if (width == 4)
        k_wide_single<4><<<1, 32, 0, s>>>(m->vertices, m->num_vertices, m->triangles,
                                          reinterpret_cast<int4*>(out->nodes), out->woop, out->tri_idx, out->info,
                                          ctx->d_status);
    else
        k_wide_single<8><<<1, 32, 0, s>>>(m->vertices, m->num_vertices, m->triangles,
                                          reinterpret_cast<int4*>(out->nodes), out->woop, out->tri_idx, out->info,
                                          ctx->d_status);
    HP_CUDA(cudaGetLastError());
    hp_count_launch();
    hp_mark(ctx, s, "single");
    return HP_OK;
}
