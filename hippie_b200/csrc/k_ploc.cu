// PLOC: parallel locally-ordered clustering over Morton-sorted references, and
// the depth-first collapse of the resulting tree into 64-byte binary nodes.
//
// Reference: PLOCBuilder::build / clustering (rt/bvh/PLOCBuilder.cpp:21-208) and
// its kernels (rt/bvh/PLOCBuilderKernels.cu:11-389). Per iteration every
// cluster picks the neighbour within +-r whose union box has the smallest
// surface area (left side first, first strict minimum wins), mutual pairs
// merge with the lower cluster as the left child into node (count-2) - k, and
// the clusters are compacted in order. The reference runs ~5 kernels and a
// host read-back per iteration; here
//   * one persistent cooperative kernel runs every iteration while more than
//     TAIL clusters remain. A tile of clusters loads the boxes of the tile and
//     2r clusters on each side into shared memory and finds the nearest
//     neighbours of its clusters and of r clusters on each side (four
//     clusters per thread on long lists, one on shorter ones; a tile holds
//     4*LPB - 2r or LPB - 2r clusters so that it and its halo take every thread
//     once), so each mutual pair of the tile is decided without another
//     tile's results; it then flags the merges, takes the two prefix sums
//     (merges, survivors) by a decoupled look-back over lower tiles, creates
//     the new nodes and compacts the clusters. Each CTA takes its tiles in
//     increasing order; one grid barrier ends the iteration. Every wait is
//     bounded; a wait that gives up records an error and the kernel stops
//     iterating;
//   * one CTA finishes the last TAIL clusters in shared memory;
//   * merge numbering is by cluster order (k = merges at lower positions), so
//     the tree is deterministic; the reference takes k from warp atomics.
// The collapse costs of computeNodeStatesAdaptive (BVHCollapserKernels.cu:58-136)
// are evaluated when a node is created, its children being final then.
//
// Collapse: PLOC creates parents after their children, so a parent always has
// a lower index. One pass over node indices in ticket order lets every node
// wait for its parent's record and derive its own: whether it survives the
// collapse, its preorder interior index, its leaf index and the offset of its
// triangles (children of a node come left subtree first). The same pass emits
// the binary nodes, reorders the triangle indices and woopifies the triangles.
#include <algorithm>
#include <cuda_runtime.h>
#include "hp_device.cuh"
#include "hp_internal.h"

namespace {

constexpr int PB = 1024;            // threads of the tail CTA
constexpr int LPB = 512;            // threads per CTA of the iteration kernel (two CTAs per SM)
constexpr int MAXR = 512;           // largest radius kept in a shared-memory window
constexpr int NB4 = 4;              // clusters per thread of the neighbour search on large lists
constexpr int WIN = NB4 * LPB + 2 * MAXR;  // neighbour window
// Lists at least this long use 4 clusters per thread (long tiles, about half as
// many tiles as the loop has CTAs at this length). On a B200 this beat twice
// and four times the length, half and a quarter of it, and long tiles at every
// length, on clustered and uniform scenes of 1 M to 16 M triangles.
constexpr int NB4_MIN_N = 148 * NB4 * 512;
// Shorter lists run fused iterations: a tile of LPB clusters finds the nearest
// neighbours of its clusters and of r clusters on each side itself, so each
// iteration needs one grid barrier instead of two.
constexpr int NNF = NB4 * LPB + 2 * MAXR;       // neighbour slots of a tile and its halo
constexpr int MIN_TILE4 = NB4 * LPB - 2 * MAXR;  // fewest clusters of a tile of the long lists
// Clusters of a fused tile: LPB - 2r (one thread per cluster of the tile and its
// halo), at least LPB / 2.
__host__ __device__ constexpr int fused_tile(int r) { return 2 * r <= LPB / 2 ? LPB - 2 * r : LPB / 2; }
// Clusters of a tile of the long lists: 4*LPB - 2r, at least 2*LPB.
__host__ __device__ constexpr int long_tile(int r) { return 2 * r <= 2 * LPB ? NB4 * LPB - 2 * r : 2 * LPB; }
constexpr size_t LOOP_SMEM = 6 * WIN * sizeof(float) + NNF * sizeof(int);
constexpr int TAIL = 2048;          // clusters finished by a single CTA
constexpr int TAIL_ITEMS = TAIL / PB;
constexpr int MAX_ITER = 1 << 16;
constexpr unsigned SPIN = 1u << 22;

// Acquire load / release store at GPU scope: a record written before the
// release store is visible to a thread whose acquire load sees the flag.
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_vol_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.volatile.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_vol_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.volatile.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

struct ploc_args {
    int n;
    int radius, max_radius, adaptive_r;
    float ct, ci;
    int adaptive_leaf, max_leaf;
    float4* nbmin;  // w: collapse cost
    float4* nbmax;  // w: subtree size (int bits)
    int* left;
    int* right;
    int* parent;
    int2* counts;   // (surviving interior nodes, leaves) of the subtree if the node survives
    uint8_t* state;
    // What the binary collapse needs of a node's children, written when the
    // node is made (null for the wide layouts): the left child's counts, its
    // index, its size with bit 31 set when the right child ends as a leaf;
    // and the three box rows of the node's Bin record (children's boxes).
    int4* cinfo;
    float4* cbox;
    int* cl0;
    int* cl1;
    unsigned long long* status;    // look-back words of the iterations on long lists
    unsigned long long* status_f;  // look-back words of the iterations on shorter lists
    unsigned* tickets;  // [MAX_ITER]
    unsigned* bar;      // [0] arrivals, [1] generation
    int* g;             // [0] cluster count, [1] iterations done
    int* err;
};

__device__ __forceinline__ float half_area(float ax, float ay, float az, float bx, float by, float bz) {
    // surface area / 2 of the union; the factor 2 does not change comparisons
    float dx = __fsub_rn(bx, ax), dy = __fsub_rn(by, ay), dz = __fsub_rn(bz, az);
    return __fmaf_rn(dz, dx, __fmaf_rn(dx, dy, __fmul_rn(dy, dz)));
}

__device__ __forceinline__ int radius_at(const ploc_args& a, int it) {
    return a.adaptive_r ? min(a.radius + it + 1, a.max_radius) : a.radius;
}

// Bounded grid barrier (generation counter). Returns false if it gave up.
__device__ __forceinline__ bool grid_barrier(unsigned* bar, int* err) { return hp_grid_barrier(bar, err, SPIN); }

// Create node `node` = merge of clusters with node ids a (left) and b (right).
// From the children's boxes (w: cost / size bits) and counts; returns the new
// node's min corner with its cost, max corner with its size, and its counts.
__device__ __forceinline__ void make_parent_from(const ploc_args& A, int node, int a, int b, const float4& amn,
                                                 const float4& amx, const float4& bmn, const float4& bmx,
                                                 const int2& ca, const int2& cb, float4& omn, float4& omx,
                                                 int2& ocnt) {
    const float mnx = fminf(amn.x, bmn.x), mny = fminf(amn.y, bmn.y), mnz = fminf(amn.z, bmn.z);
    const float mxx = fmaxf(amx.x, bmx.x), mxy = fmaxf(amx.y, bmx.y), mxz = fmaxf(amx.z, bmx.z);
    const int size = __float_as_int(amx.w) + __float_as_int(bmx.w);
    int st;
    float c;
    if (A.adaptive_leaf) {
        const float area = hp_area(mnx, mny, mnz, mxx, mxy, mxz);
        const float c_int = __fadd_rn(__fmaf_rn(A.ct, area, amn.w), bmn.w);
        const float c_leaf = __fmul_rn(__fmul_rn(A.ci, area), (float)size);
        st = (c_leaf < c_int) ? 0 : 1;
        c = st ? c_int : c_leaf;
    } else {
        st = (size <= A.max_leaf) ? 0 : 1;
        c = 0.0f;
    }
    omn = make_float4(mnx, mny, mnz, c);
    omx = make_float4(mxx, mxy, mxz, __int_as_float(size));
    ocnt = st ? make_int2(1 + ca.x + cb.x, ca.y + cb.y) : make_int2(0, 1);
    __stcg(A.nbmin + node, omn);
    __stcg(A.nbmax + node, omx);
    __stcg(A.counts + node, ocnt);
    A.state[node] = (uint8_t)st;
    A.left[node] = a;
    A.right[node] = b;
    A.parent[a] = node;
    A.parent[b] = node;
    if (A.cinfo) {
        __stcg(A.cinfo + node, make_int4(ca.x, ca.y, a, __float_as_int(amx.w) | (cb.x == 0 ? (int)0x80000000 : 0)));
        float4* cbx = A.cbox + 3 * (int64_t)node;
        __stcg(cbx, make_float4(amn.x, amx.x, amn.y, amx.y));
        __stcg(cbx + 1, make_float4(bmn.x, bmx.x, bmn.y, bmx.y));
        __stcg(cbx + 2, make_float4(amn.z, amx.z, bmn.z, bmx.z));
    }
}

__device__ __forceinline__ void make_parent(const ploc_args& A, int node, int a, int b) {
    const float4 amn = __ldcg(A.nbmin + a), amx = __ldcg(A.nbmax + a);
    const float4 bmn = __ldcg(A.nbmin + b), bmx = __ldcg(A.nbmax + b);
    const int2 ca = __ldcg(A.counts + a), cb = __ldcg(A.counts + b);
    float4 omn, omx;
    int2 ocnt;
    make_parent_from(A, node, a, b, amn, amx, bmn, bmx, ca, cb, omn, omx, ocnt);
}

// Leaves: sorted reference p becomes leaf node n-1+p and cluster p.
__global__ void __launch_bounds__(256) k_ploc_leaves(ploc_args A, const int32_t* __restrict__ sorted_tri,
                                                     const float4* __restrict__ tbmin,
                                                     const float4* __restrict__ tbmax) {
    const int p = blockIdx.x * 256 + threadIdx.x;
    if (p >= A.n) return;
    const int tri = sorted_tri[p];
    const float4 mn = tbmin[2 * (int64_t)tri], mx = tbmax[2 * (int64_t)tri];  // interleaved corners
    const int j = A.n - 1 + p;
    const float cost = A.adaptive_leaf ? __fmul_rn(A.ci, hp_area(mn.x, mn.y, mn.z, mx.x, mx.y, mx.z)) : 0.0f;
    A.nbmin[j] = make_float4(mn.x, mn.y, mn.z, cost);
    A.nbmax[j] = make_float4(mx.x, mx.y, mx.z, __int_as_float(1));
    A.counts[j] = make_int2(0, 1);
    A.state[j] = 0;
    A.cl0[p] = j;
    if (p == 0) {
        A.parent[0] = -1;
        A.g[0] = A.n;
        A.g[1] = 0;
    }
}

// Nearest neighbour of every cluster of one tile of B*LPB clusters: the tile's
// boxes and r on each side in shared memory (a huge box, never the nearest,
// outside the cluster list); candidates c-r .. c+r in increasing order, the
// first strict minimum. With B = 4 a thread searches for 4 consecutive
// clusters at once and reads each candidate box once for all of them; the
// candidates are walked in five runs whose valid clusters are known without a
// test per pair (runs valid for r >= 4).
// Boxes of clusters [w0, w0 + wn) into the shared-memory window (a huge box,
// never the nearest, outside the cluster list). The cluster indices of a batch
// of elements are read first and their boxes after, so that a thread has a
// batch of loads in flight instead of one dependent pair at a time.
__device__ __forceinline__ void load_window(const ploc_args& A, const int* __restrict__ cl, int N, int w0, int wn,
                                            float* s) {
    constexpr int BATCH = 3;
    for (int k0 = threadIdx.x; k0 < wn; k0 += BATCH * LPB) {
        int node[BATCH];
#pragma unroll
        for (int u = 0; u < BATCH; ++u) {
            const int k = k0 + u * LPB, c = w0 + k;
            node[u] = (k < wn && c >= 0 && c < N) ? __ldcg(cl + c) : -1;
        }
        float4 mn[BATCH], mx[BATCH];
#pragma unroll
        for (int u = 0; u < BATCH; ++u) {
            if (node[u] >= 0) {
                mn[u] = __ldcg(A.nbmin + node[u]);
                mx[u] = __ldcg(A.nbmax + node[u]);
            } else {
                mn[u] = make_float4(-HP_MAX_FLOAT, -HP_MAX_FLOAT, -HP_MAX_FLOAT, 0.0f);
                mx[u] = make_float4(HP_MAX_FLOAT, HP_MAX_FLOAT, HP_MAX_FLOAT, 0.0f);
            }
        }
#pragma unroll
        for (int u = 0; u < BATCH; ++u) {
            const int k = k0 + u * LPB;
            if (k < wn) {
                s[k] = mn[u].x; s[WIN + k] = mn[u].y; s[2 * WIN + k] = mn[u].z;
                s[3 * WIN + k] = mx[u].x; s[4 * WIN + k] = mx[u].y; s[5 * WIN + k] = mx[u].z;
            }
        }
    }
}

template <int B>
__device__ void nn_tile(const ploc_args& A, const int* __restrict__ cl, int N, int r, int base, float* s,
                        int* s_nn) {
    float* smnx = s;
    float* smny = s + WIN;
    float* smnz = s + 2 * WIN;
    float* smxx = s + 3 * WIN;
    float* smxy = s + 4 * WIN;
    float* smxz = s + 5 * WIN;
    constexpr int TS = B * LPB;
    __syncthreads();
    load_window(A, cl, N, base - r, TS + 2 * r, s);
    __syncthreads();
    const int l0 = threadIdx.x * B;  // cluster base + l sits at window position l + r
    float ax[B], ay[B], az[B], bx[B], by[B], bz[B], best[B];
    int bi[B];
#pragma unroll
    for (int q = 0; q < B; ++q) {
        const int me = l0 + q + r;
        ax[q] = smnx[me]; ay[q] = smny[me]; az[q] = smnz[me];
        bx[q] = smxx[me]; by[q] = smxy[me]; bz[q] = smxz[me];
        best[q] = HP_MAX_FLOAT;
        bi[q] = -1;
    }
    auto upd = [&](int q, int k, float cx, float cy, float cz, float dx, float dy, float dz) {
        const float d = half_area(fminf(ax[q], cx), fminf(ay[q], cy), fminf(az[q], cz), fmaxf(bx[q], dx),
                                  fmaxf(by[q], dy), fmaxf(bz[q], dz));
        if (best[q] > d) {
            best[q] = d;
            bi[q] = base - r + k;
        }
    };
#define HP_PLOC_CAND(k) const float cx = smnx[k], cy = smny[k], cz = smnz[k], dx = smxx[k], dy = smxy[k], dz = smxz[k]
    if (B == 1 || r < 4) {
        for (int k = l0; k <= l0 + (B - 1) + 2 * r; ++k) {
            HP_PLOC_CAND(k);
#pragma unroll
            for (int q = 0; q < B; ++q)
                if (k >= l0 + q && k <= l0 + q + 2 * r && k != l0 + q + r) upd(q, k, cx, cy, cz, dx, dy, dz);
        }
    } else {
        // cluster q: candidates l0+q .. l0+q+2r, itself at l0+q+r
        for (int k = l0; k < l0 + 3; ++k) {  // q <= k - l0
            HP_PLOC_CAND(k);
#pragma unroll
            for (int q = 0; q < B; ++q)
                if (q <= k - l0) upd(q, k, cx, cy, cz, dx, dy, dz);
        }
        for (int k = l0 + 3; k < l0 + r; ++k) {  // every cluster, none itself
            HP_PLOC_CAND(k);
#pragma unroll
            for (int q = 0; q < B; ++q) upd(q, k, cx, cy, cz, dx, dy, dz);
        }
        for (int k = l0 + r; k < l0 + r + 4; ++k) {  // every cluster but the one at k
            HP_PLOC_CAND(k);
#pragma unroll
            for (int q = 0; q < B; ++q)
                if (q != k - l0 - r) upd(q, k, cx, cy, cz, dx, dy, dz);
        }
        for (int k = l0 + r + 4; k <= l0 + 2 * r; ++k) {  // every cluster, none itself
            HP_PLOC_CAND(k);
#pragma unroll
            for (int q = 0; q < B; ++q) upd(q, k, cx, cy, cz, dx, dy, dz);
        }
        for (int k = l0 + 2 * r + 1; k <= l0 + 2 * r + 3; ++k) {  // q >= k - l0 - 2r
            HP_PLOC_CAND(k);
#pragma unroll
            for (int q = 0; q < B; ++q)
                if (q >= k - l0 - 2 * r) upd(q, k, cx, cy, cz, dx, dy, dz);
        }
    }
#undef HP_PLOC_CAND
#pragma unroll
    for (int q = 0; q < B; ++q) {
        const int c = base + l0 + q;
        s_nn[l0 + q] = (c >= 0 && c < N) ? bi[q] : -1;
    }
    __syncthreads();
}

// Status word of a merge tile: [63:60] iteration tag, [59:58] flag, [57:29] merges, [28:0] survivors.
constexpr unsigned long long F_AGG = 1ull << 58, F_INC = 2ull << 58, F_MASK = 3ull << 58;
__device__ __forceinline__ unsigned long long mk_status(unsigned tag, unsigned long long flag, unsigned m,
                                                        unsigned k) {
    return ((unsigned long long)tag << 60) | flag | ((unsigned long long)(m & 0x1fffffffu) << 29) |
           (unsigned long long)(k & 0x1fffffffu);
}

// Block-wide exclusive scan of (a, b) over NT threads (NT <= 1024). Returns
// the totals. s_wa and s_wb hold NT / 32 + 1 entries.
template <int NT>
__device__ __forceinline__ int2 block_scan2(int& a, int& b, int* s_wa, int* s_wb) {
    constexpr int NW = NT / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int ia = a, ib = b;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int ya = __shfl_up_sync(HP_FULL_MASK, ia, o), yb = __shfl_up_sync(HP_FULL_MASK, ib, o);
        if (lane >= o) { ia += ya; ib += yb; }
    }
    __syncthreads();
    if (lane == 31) { s_wa[warp] = ia; s_wb[warp] = ib; }
    __syncthreads();
    if (warp == 0) {  // exclusive scan of the NW warp totals by one warp; totals at [NW]
        const int va = lane < NW ? s_wa[lane] : 0, vb = lane < NW ? s_wb[lane] : 0;
        int xa = va, xb = vb;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int ya = __shfl_up_sync(HP_FULL_MASK, xa, o), yb = __shfl_up_sync(HP_FULL_MASK, xb, o);
            if (lane >= o) { xa += ya; xb += yb; }
        }
        if (lane < NW) { s_wa[lane] = xa - va; s_wb[lane] = xb - vb; }
        if (lane == NW - 1) { s_wa[NW] = xa; s_wb[NW] = xb; }
    }
    __syncthreads();
    a = s_wa[warp] + ia - a;
    b = s_wb[warp] + ib - b;
    return make_int2(s_wa[NW], s_wb[NW]);
}

// Nearest neighbours of the clusters [tbase - r, tbase + tsz + r) of a fused
// tile (s_nn[l] for cluster tbase - r + l), from the boxes of clusters
// [tbase - 2r, tbase + tsz + 2r) in shared memory; candidates in increasing
// order, the first strict minimum, as in nn_tile.
__device__ void nn_halo(const ploc_args& A, const int* __restrict__ cl, int N, int r, int tbase, int tsz, float* s,
                        int* s_nn) {
    float* smnx = s;
    float* smny = s + WIN;
    float* smnz = s + 2 * WIN;
    float* smxx = s + 3 * WIN;
    float* smxy = s + 4 * WIN;
    float* smxz = s + 5 * WIN;
    const int w0 = tbase - 2 * r;
    load_window(A, cl, N, w0, tsz + 4 * r, s);
    __syncthreads();
    for (int l = threadIdx.x; l < tsz + 2 * r; l += LPB) {
        const int c = tbase - r + l;
        int bi = -1;
        if (c >= 0 && c < N) {
            const int me = l + r;  // window position of cluster c; its candidates are l .. l + 2r
            const float ax = smnx[me], ay = smny[me], az = smnz[me], bx = smxx[me], by = smxy[me], bz = smxz[me];
            float best = HP_MAX_FLOAT;
            for (int k = l; k <= l + 2 * r; ++k) {
                if (k == me) continue;
                const float d = half_area(fminf(ax, smnx[k]), fminf(ay, smny[k]), fminf(az, smnz[k]),
                                          fmaxf(bx, smxx[k]), fmaxf(by, smxy[k]), fmaxf(bz, smxz[k]));
                if (best > d) {
                    best = d;
                    bi = w0 + k;
                }
            }
        }
        s_nn[l] = bi;
    }
    __syncthreads();
}

// One merge tile of at most ITEMS*LPB clusters: flags, prefix sums (tile + look-back),
// new nodes, compaction. FUSED tiles (ITEMS 1) find their neighbours first;
// the others read the neighbour phase's results.
template <int ITEMS>
__device__ void merge_tile(const ploc_args& A, const int* __restrict__ cl_in, int* __restrict__ cl_out,
                           int N, int r, int it, unsigned tile, int TSZ, unsigned long long* status, float* s_win,
                           int* s_nn, int* s_wa, int* s_wb, unsigned* s_pref) {
    const unsigned tag = (unsigned)(it % 15) + 1u;
    const int tbase = (int)tile * TSZ;
    __syncthreads();  // the previous tile's shared memory is free
    if (ITEMS == 1) nn_halo(A, cl_in, N, r, tbase, TSZ, s_win, s_nn);
    else nn_tile<ITEMS>(A, cl_in, N, r, tbase - r, s_win, s_nn);  // TSZ + 2r <= ITEMS * LPB clusters
    const int nlo = tbase - r;  // cluster of s_nn[0]
    auto nn_of = [&](int c) { return s_nn[c - nlo]; };
    const int base = tbase + threadIdx.x * ITEMS;
    int kind[ITEMS];  // 0: dropped (higher partner), 1: kept, 2: merges with nn
    int nbr[ITEMS];
    int m = 0, k = 0;
#pragma unroll
    for (int q = 0; q < ITEMS; ++q) {
        const int c = base + q;
        kind[q] = 0;
        nbr[q] = -1;
        if (c < N && c < tbase + TSZ) {
            const int j = nn_of(c);
            nbr[q] = j;
            const bool mutual = j >= 0 && j < N && j >= nlo && j < tbase + TSZ + r && nn_of(j) == c;
            kind[q] = (mutual && c < j) ? 2 : ((mutual && j < c) ? 0 : 1);
            m += kind[q] == 2;
            k += kind[q] != 0;
        }
    }
    int em = m, ek = k;
    const int2 tot = block_scan2<LPB>(em, ek, s_wa, s_wb);
    if (threadIdx.x < 32) {
        // Decoupled look-back by one warp over windows of 32 earlier tiles: lane i
        // reads tile t-i; the window is summed up to the nearest tile whose
        // inclusive prefix is published, once every tile up to it has published.
        const int lane = threadIdx.x;
        unsigned long long* st = status + tile;
        if (lane == 0) st_vol_u64(st, mk_status(tag, tile == 0 ? F_INC : F_AGG, tot.x, tot.y));
        unsigned pm = 0, pk = 0;
        if (tile > 0) {
            long t = (long)tile - 1;
            unsigned spins = 0;
            while (true) {
                const long idx = t - lane;
                const unsigned long long s = idx >= 0 ? ld_vol_u64(status + idx) : mk_status(tag, F_INC, 0, 0);
                const bool ready = (unsigned)(s >> 60) == tag && (s & F_MASK) != 0;
                const unsigned inc = __ballot_sync(HP_FULL_MASK, ready && (s & F_MASK) == F_INC);
                const int stop = inc ? __ffs(inc) - 1 : 31;  // the window ends at the nearest inclusive tile
                const unsigned need = stop == 31 ? HP_FULL_MASK : ((1u << (stop + 1)) - 1u);
                if (__ballot_sync(HP_FULL_MASK, !ready) & need) {
                    if (++spins > SPIN) { if (lane == 0) hp_report(A.err, HP_DEV_SPIN_LIMIT, (int)tile); break; }
                    if ((spins & 1023u) == 0 && __shfl_sync(HP_FULL_MASK, *((volatile int*)A.err), 0) != 0) break;
                    continue;
                }
                unsigned vm = lane <= stop ? (unsigned)((s >> 29) & 0x1fffffffu) : 0u;
                unsigned vk = lane <= stop ? (unsigned)(s & 0x1fffffffu) : 0u;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    vm += __shfl_xor_sync(HP_FULL_MASK, vm, o);
                    vk += __shfl_xor_sync(HP_FULL_MASK, vk, o);
                }
                pm += vm;
                pk += vk;
                if (inc) break;
                t -= 32;
            }
            if (lane == 0) st_vol_u64(st, mk_status(tag, F_INC, pm + tot.x, pk + tot.y));
        }
        if (lane == 0) {
            s_pref[0] = pm;
            s_pref[1] = pk;
            const int tiles = (N + TSZ - 1) / TSZ;
            if ((int)tile == tiles - 1) A.g[0] = N - (int)(pm + tot.x);
        }
    }
    __syncthreads();
    int mr = (int)s_pref[0] + em, kr = (int)s_pref[1] + ek;
#pragma unroll
    for (int q = 0; q < ITEMS; ++q) {
        const int c = base + q;
        if (kind[q] == 0) continue;
        int node = cl_in[c];
        if (kind[q] == 2) {
            const int nb = cl_in[nbr[q]];
            const int idx = (N - 2) - mr;
            make_parent(A, idx, node, nb);
            node = idx;
            ++mr;
        }
        cl_out[kr++] = node;
    }
}

__global__ void __launch_bounds__(LPB, 2) k_ploc_loop(ploc_args A) {
    extern __shared__ float s_win[];
    int* s_nn = reinterpret_cast<int*>(s_win + 6 * WIN);
    __shared__ int s_wa[LPB / 32 + 1], s_wb[LPB / 32 + 1];
    __shared__ unsigned s_pref[2];
    __shared__ unsigned s_ticket;
    __shared__ int s_n;
    for (int it = 0; it < MAX_ITER; ++it) {
        if (threadIdx.x == 0) s_n = *((volatile int*)A.g);
        __syncthreads();
        const int N = s_n;
        if (N <= TAIL || *((volatile int*)A.err) != 0) break;
        const int r = radius_at(A, it);
        const int* cl_in = (it & 1) ? A.cl1 : A.cl0;
        int* cl_out = (it & 1) ? A.cl0 : A.cl1;
        // Tiles of ITEMS*LPB - 2r clusters, so that a tile and its halo take ITEMS
        // clusters per thread; every CTA takes its tiles in increasing order (all
        // CTAs are resident; tickets are handed out in order), so each look-back
        // waits only on lower tiles that are in progress.
        // Tile sizes use the largest radius of the build, so that the tile
        // count of an iteration never exceeds the previous one's (the look-back
        // words of lower tiles are then always this iteration's or older ones
        // with another tag).
        const int rt = A.adaptive_r ? A.max_radius : A.radius;
        if (N >= NB4_MIN_N) {
            // long tiles (~25 us each) go to whichever CTA is free, in ticket order
            const int tsz = long_tile(rt);
            while (true) {
                if (threadIdx.x == 0) s_ticket = atomicAdd(A.tickets + it, 1u);
                __syncthreads();
                const unsigned tile = s_ticket;
                __syncthreads();
                if ((long)tile * tsz >= N) break;
                merge_tile<NB4>(A, cl_in, cl_out, N, r, it, tile, tsz, A.status, s_win, s_nn, s_wa, s_wb, s_pref);
            }
        } else {
            const int tsz = fused_tile(rt);
            for (unsigned tile = blockIdx.x; (long)tile * tsz < N; tile += gridDim.x)
                merge_tile<1>(A, cl_in, cl_out, N, r, it, tile, tsz, A.status_f, s_win, s_nn, s_wa, s_wb, s_pref);
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) A.g[1] = it + 1;
        if (!grid_barrier(A.bar, A.err)) break;
    }
}

// Finish the last <= TAIL clusters in one CTA.
constexpr size_t TAIL_SMEM = 12 * TAIL * sizeof(float);

__global__ void __launch_bounds__(PB, 1) k_ploc_tail(ploc_args A) {
    extern __shared__ float s_tail[];
    float(*smn)[TAIL] = reinterpret_cast<float(*)[TAIL]>(s_tail);
    float(*smx)[TAIL] = reinterpret_cast<float(*)[TAIL]>(s_tail + 3 * TAIL);
    int* snode = reinterpret_cast<int*>(s_tail + 6 * TAIL);
    int* snn = reinterpret_cast<int*>(s_tail + 7 * TAIL);
    // the clusters' cost and size (the w words of their boxes) and counts, so
    // that a merge reads nothing from global memory
    float* scost = s_tail + 8 * TAIL;
    int* ssize = reinterpret_cast<int*>(s_tail + 9 * TAIL);
    int2* scnt = reinterpret_cast<int2*>(s_tail + 10 * TAIL);
    __shared__ int s_wa[PB / 32 + 1], s_wb[PB / 32 + 1];
    __shared__ int s_n;
    if (*((volatile int*)A.err) != 0) return;
    const int it0 = A.g[1];
    int N = A.g[0];
    if (N > TAIL) { hp_report(A.err, HP_DEV_BAD_INDEX, N); return; }
    const int* cl = (it0 & 1) ? A.cl1 : A.cl0;
    for (int c = threadIdx.x; c < N; c += PB) {
        const int node = cl[c];
        const float4 mn = __ldcg(A.nbmin + node), mx = __ldcg(A.nbmax + node);
        snode[c] = node;
        smn[0][c] = mn.x; smn[1][c] = mn.y; smn[2][c] = mn.z;
        smx[0][c] = mx.x; smx[1][c] = mx.y; smx[2][c] = mx.z;
        scost[c] = mn.w;
        ssize[c] = __float_as_int(mx.w);
        scnt[c] = __ldcg(A.counts + node);
    }
    __syncthreads();
    for (int it = it0; N > 1 && it < MAX_ITER; ++it) {
        const int r = radius_at(A, it);
        for (int i = threadIdx.x; i < N; i += PB) {
            const float ax = smn[0][i], ay = smn[1][i], az = smn[2][i];
            const float bx = smx[0][i], by = smx[1][i], bz = smx[2][i];
            float best = HP_MAX_FLOAT;
            int bi = -1;
            const int lo = max(0, i - r), hi = min(N, i + r + 1);
            for (int k = lo; k < hi; ++k) {
                if (k == i) continue;
                const float d = half_area(fminf(ax, smn[0][k]), fminf(ay, smn[1][k]), fminf(az, smn[2][k]),
                                          fmaxf(bx, smx[0][k]), fmaxf(by, smx[1][k]), fmaxf(bz, smx[2][k]));
                if (best > d) { best = d; bi = k; }
            }
            snn[i] = bi;
        }
        __syncthreads();
        int kind[TAIL_ITEMS];
        int m = 0, k = 0;
#pragma unroll
        for (int q = 0; q < TAIL_ITEMS; ++q) {
            const int c = threadIdx.x * TAIL_ITEMS + q;
            kind[q] = 0;
            if (c < N) {
                const int j = snn[c];
                const bool mutual = j >= 0 && snn[j] == c;
                kind[q] = (mutual && c < j) ? 2 : ((mutual && j < c) ? 0 : 1);
                m += kind[q] == 2;
                k += kind[q] != 0;
            }
        }
        int em = m, ek = k;
        const int2 tot = block_scan2<PB>(em, ek, s_wa, s_wb);
        // new entries in registers, then compaction
        int nnode[TAIL_ITEMS];
        float nmn[TAIL_ITEMS][3], nmx[TAIL_ITEMS][3];
        float ncost[TAIL_ITEMS];
        int nsize[TAIL_ITEMS];
        int2 ncnt[TAIL_ITEMS];
        int pos[TAIL_ITEMS];
        int mr = em, kr = ek;
#pragma unroll
        for (int q = 0; q < TAIL_ITEMS; ++q) {
            const int c = threadIdx.x * TAIL_ITEMS + q;
            pos[q] = -1;
            if (kind[q] == 0) continue;
            nnode[q] = snode[c];
            for (int a = 0; a < 3; ++a) { nmn[q][a] = smn[a][c]; nmx[q][a] = smx[a][c]; }
            ncost[q] = scost[c];
            nsize[q] = ssize[c];
            ncnt[q] = scnt[c];
            if (kind[q] == 2) {
                const int j = snn[c];
                const int idx = (N - 2) - mr++;
                const float4 amn = make_float4(smn[0][c], smn[1][c], smn[2][c], scost[c]);
                const float4 amx = make_float4(smx[0][c], smx[1][c], smx[2][c], __int_as_float(ssize[c]));
                const float4 bmn = make_float4(smn[0][j], smn[1][j], smn[2][j], scost[j]);
                const float4 bmx = make_float4(smx[0][j], smx[1][j], smx[2][j], __int_as_float(ssize[j]));
                float4 omn, omx;
                make_parent_from(A, idx, snode[c], snode[j], amn, amx, bmn, bmx, scnt[c], scnt[j], omn, omx,
                                 ncnt[q]);
                nnode[q] = idx;
                nmn[q][0] = omn.x; nmn[q][1] = omn.y; nmn[q][2] = omn.z;
                nmx[q][0] = omx.x; nmx[q][1] = omx.y; nmx[q][2] = omx.z;
                ncost[q] = omn.w;
                nsize[q] = __float_as_int(omx.w);
            }
            pos[q] = kr++;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < TAIL_ITEMS; ++q) {
            if (pos[q] < 0) continue;
            snode[pos[q]] = nnode[q];
            for (int a = 0; a < 3; ++a) { smn[a][pos[q]] = nmn[q][a]; smx[a][pos[q]] = nmx[q][a]; }
            scost[pos[q]] = ncost[q];
            ssize[pos[q]] = nsize[q];
            scnt[pos[q]] = ncnt[q];
        }
        if (threadIdx.x == 0) s_n = N - tot.x;
        __syncthreads();
        N = s_n;
        __syncthreads();
    }
    if (threadIdx.x == 0 && N != 1) hp_report(A.err, HP_DEV_BAD_INDEX, N);
}

// ---- depth-first collapse of a tree whose parents come first in processing order ----------
// Node v is processed at ticket position r with v = order[r] (order null: v = r,
// which needs parent indices below child indices, as PLOC's are).
struct td_args {
    int n;
    const int* order;
    const int* left;
    const int* right;
    const int* parent;
    const int2* counts;
    const uint8_t* state;
    const float4* nbmin;
    const float4* nbmax;
    const int4* cinfo;   // PLOC: per node, what its children contribute (ploc_args::cinfo)
    const float4* cbox;  // PLOC: per node, its Bin record's three box rows
    int4* rec;          // [n-1] interior records: preorder index, first leaf, first triangle, status
    int* flag;          // [n-1] record published (build epoch)
    int epoch;
    unsigned* ticket;
    const int32_t* sorted_tri;
    const float4* woop_src;  // Woop rows per scene triangle, or null: computed from the vertices
    const float* verts;
    int64_t nv;
    const int32_t* tris;
    hp_node_bin* nodes;
    float4* woop;
    int32_t* tri_idx;
    hp_bvh_info* info;
    int max_nodes;
    int* err;
};

enum { ST_DEAD = 0, ST_LEAF = 1, ST_INTERIOR = 2 };

__device__ __forceinline__ void td_put(const td_args& T, int idx, const hp_node_bin& nd) {
    if ((unsigned)idx < (unsigned)T.max_nodes) T.nodes[idx] = nd;
    else hp_report(T.err, HP_DEV_BAD_INDEX, idx);
}

// PRE: the PLOC build recorded, per node, its children's contribution
// (cinfo, cbox), so a node reads its own row and its parent's instead of
// gathering its sibling's and its children's counts, states and boxes.
template <bool PRE>
__global__ void __launch_bounds__(256) k_topdown(td_args T) {
    __shared__ unsigned s_tile;
    if (threadIdx.x == 0) s_tile = atomicAdd(T.ticket, 1u);
    __syncthreads();
    const int n = T.n;
    const int r = (int)s_tile * 256 + threadIdx.x;
    if (r >= 2 * n - 1) return;
    const int v = T.order ? __ldg(T.order + r) : r;
    if ((unsigned)v >= (unsigned)(2 * n - 1)) {
        hp_report(T.err, HP_DEV_BAD_INDEX, r);
        return;
    }
    const int2 c0 = T.counts[T.left[0]], c1 = T.counts[T.right[0]];
    const int num_int = 1 + c0.x + c1.x;
    int status, iidx = 0, lidx = 0, toff = 0, par = -1;
    if (v == 0) {
        status = ST_INTERIOR;
        T.info->num_interior = num_int;
        T.info->num_leaf = c0.y + c1.y;
    } else {
        const int p = T.parent[v];
        if (p < 0 || (!T.order && p >= v) || p >= n - 1) {
            hp_report(T.err, HP_DEV_BAD_INDEX, v);
            return;
        }
        // what does not depend on the parent's record is read before waiting for it
        bool is_left;
        int2 cs;    // the left sibling's counts (used by a right child)
        int ssize;  // the left sibling's size
        if (PRE) {
            const int4 ci = __ldcg(T.cinfo + p);
            is_left = ci.z == v;
            cs = make_int2(ci.x, ci.y);
            ssize = ci.w & 0x7fffffff;
        } else {
            is_left = T.left[p] == v;
            const int sib = is_left ? T.right[p] : T.left[p];
            cs = T.counts[sib];
            ssize = __float_as_int(T.nbmax[sib].w);
        }
        const bool leaf = v >= n - 1 || T.state[v] == 0;
        unsigned spins = 0;
        while (ld_acquire_u32(reinterpret_cast<const unsigned*>(T.flag + p)) != (unsigned)T.epoch) {
            if (++spins > SPIN) {
                hp_report(T.err, HP_DEV_SPIN_LIMIT, v);
                break;
            }
            if ((spins & 1023u) == 0 && *((volatile int*)T.err) != 0) return;
        }
        const int4 pr = __ldcg(T.rec + p);
        par = pr.x;
        if (pr.w == ST_INTERIOR) {
            status = leaf ? ST_LEAF : ST_INTERIOR;
            if (is_left) {
                iidx = pr.x + 1; lidx = pr.y; toff = pr.z;
            } else {
                iidx = pr.x + 1 + cs.x;
                lidx = pr.y + cs.y;
                toff = pr.z + ssize;
            }
        } else {
            status = ST_DEAD;
            toff = is_left ? pr.z : pr.z + ssize;
        }
    }
    if (v < n - 1) {
        __stcg(T.rec + v, make_int4(iidx, lidx, toff, status));
        st_release_u32(reinterpret_cast<unsigned*>(T.flag + v), (unsigned)T.epoch);  // orders the record before
    }
    const float4 mn = T.nbmin[v], mx = T.nbmax[v];
    const int size = __float_as_int(mx.w);
    if (status == ST_INTERIOR && PRE) {
        // a left child ends as a leaf exactly when its counts are (0, 1)
        const int4 ci = __ldcg(T.cinfo + v);
        const bool l_leaf = ci.x == 0, r_leaf = ci.w < 0;
        const int lref = l_leaf ? ~(num_int + lidx) : iidx + 1;
        const int rref = r_leaf ? ~(num_int + lidx + ci.y) : iidx + 1 + ci.x;
        const float4* cb = T.cbox + 3 * (int64_t)v;
        hp_node_bin nd;
        nd.c0xy = __ldcg(cb);
        nd.c1xy = __ldcg(cb + 1);
        nd.cz = __ldcg(cb + 2);
        nd.meta = make_int4(lref, rref, size, par);
        td_put(T, iidx, nd);
    } else if (status == ST_INTERIOR) {
        const int l = T.left[v], r = T.right[v];
        const bool l_leaf = l >= n - 1 || T.state[l] == 0;
        const bool r_leaf = r >= n - 1 || T.state[r] == 0;
        const int2 cl = T.counts[l];
        const int lref = l_leaf ? ~(num_int + lidx) : iidx + 1;
        const int rref = r_leaf ? ~(num_int + lidx + cl.y) : iidx + 1 + cl.x;
        td_put(T, iidx, hp_make_node(T.nbmin[l], T.nbmax[l], T.nbmin[r], T.nbmax[r], lref, rref, size, par));
    } else if (status == ST_LEAF) {
        td_put(T, num_int + lidx, hp_make_node(mn, mx, mn, mx, toff, toff + size, ~size, par));
    }
    if (v >= n - 1) {
        if (toff < 0 || toff >= n) {
            hp_report(T.err, HP_DEV_BAD_INDEX, toff);
            return;
        }
        const int tri = T.sorted_tri[v - (n - 1)];
        T.tri_idx[toff] = tri;
        if (T.woop_src) {
            if ((unsigned)tri >= (unsigned)n) {
                hp_report(T.err, HP_DEV_BAD_INDEX, tri);
                return;
            }
            T.woop[3 * (int64_t)toff] = __ldg(T.woop_src + 3 * (int64_t)tri);
            T.woop[3 * (int64_t)toff + 1] = __ldg(T.woop_src + 3 * (int64_t)tri + 1);
            T.woop[3 * (int64_t)toff + 2] = __ldg(T.woop_src + 3 * (int64_t)tri + 2);
            return;
        }
        float p[9];
        for (int k = 0; k < 3; ++k) {
            int vi = T.tris[3 * (int64_t)tri + k];
            if (vi < 0 || vi >= T.nv) { hp_report(T.err, HP_DEV_BAD_INPUT, tri); vi = 0; }
            for (int a = 0; a < 3; ++a) p[3 * k + a] = __ldg(T.verts + 3 * (int64_t)vi + a);
        }
        float4 w0, w1, w2;
        hp_woop(p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], p[8], w0, w1, w2);
        T.woop[3 * (int64_t)toff] = w0;
        T.woop[3 * (int64_t)toff + 1] = w1;
        T.woop[3 * (int64_t)toff + 2] = w2;
    }
}

}  // namespace

size_t hp_topdown_scratch_bytes(int64_t n) {
    return hp_carve::pad(n * 16) + hp_carve::pad(n * 4) + hp_carve::pad(64);
}

hp_status hp_topdown_collapse(hp_ctx* ctx, const hp_mesh* m, const hp_topdown_in& in, hp_bvh_impl* out,
                              void* scratch, cudaStream_t s) {
    const int n = in.n;
    const int64_t nn = 2 * (int64_t)n - 1;
    hp_carve cv(reinterpret_cast<char*>(scratch));
    int4* rec = cv.take<int4>(n);
    int* flag = cv.take<int>(n);
    unsigned* ticket = cv.take<unsigned>(16);
    HP_CUDA(cudaMemsetAsync(flag, 0, (size_t)n * 4, s));
    HP_CUDA(cudaMemsetAsync(ticket, 0, 64, s));
    td_args T{};
    T.n = n;
    T.order = in.order;
    T.left = in.left;
    T.right = in.right;
    T.parent = in.parent;
    T.counts = in.counts;
    T.state = in.state;
    T.nbmin = in.nbmin;
    T.nbmax = in.nbmax;
    T.rec = rec;
    T.flag = flag;
    T.epoch = 1;
    T.ticket = ticket;
    T.sorted_tri = in.sorted_tri;
    T.verts = m->vertices;
    T.nv = m->num_vertices;
    T.tris = m->triangles;
    T.nodes = out->nodes;
    T.woop = out->woop;
    T.tri_idx = out->tri_idx;
    T.info = out->info;
    T.max_nodes = (int)std::max<int64_t>(2 * out->capacity - 1, 3);
    T.err = ctx->d_status;
    k_topdown<false><<<hp_div_up(nn, 256), 256, 0, s>>>(T);
    HP_CUDA(cudaGetLastError());
    hp_count_launch();
    return HP_OK;
}

size_t hp_ploc_scratch_bytes(int64_t n) {
    const int64_t nn = 2 * n - 1;
    size_t b = 0;
    b += 2 * hp_carve::pad(nn * 16);   // node boxes
    b += 3 * hp_carve::pad(nn * 4);    // left, right, parent
    b += hp_carve::pad(nn * 8);        // counts
    b += hp_carve::pad(nn);            // state
    b += 2 * hp_carve::pad(n * 4);     // cl0, cl1
    b += hp_carve::pad(((n + MIN_TILE4 - 1) / MIN_TILE4 + 1) * 8);
    b += hp_carve::pad(((std::min<int64_t>(n, NB4_MIN_N) + LPB / 2 - 1) / (LPB / 2) + 1) * 8);
    b += hp_carve::pad(MAX_ITER * 4 + 64);
    b += hp_carve::pad(n * 16) + hp_carve::pad(n * 4);  // records, flags
    b += hp_carve::pad(n * 16) + hp_carve::pad(n * 48);  // children's counts and boxes per node
    return b;
}

hp_status hp_ploc_stage(hp_ctx* ctx, const hp_mesh* m, const hp_build_params* p, hp_bvh_impl* out,
                        const int32_t* sorted_tri, const float4* tbmin, const float4* tbmax, void* scratch,
                        void* wide_scratch, cudaStream_t s, const float4* woop_src) {
    const int n = (int)m->num_triangles;
    const int64_t nn = 2 * (int64_t)n - 1;
    const int r_max = p->ploc_adaptive ? p->ploc_max_radius : p->ploc_radius;
    if (r_max > MAXR)
        return hp_fail(HP_ERR_UNSUPPORTED, "PLOC radius above 512 is not supported");
    hp_carve cv(reinterpret_cast<char*>(scratch));
    ploc_args A{};
    A.n = n;
    A.radius = p->ploc_radius;
    A.max_radius = p->ploc_max_radius;
    A.adaptive_r = p->ploc_adaptive;
    A.ct = p->ct;
    A.ci = p->ci;
    A.adaptive_leaf = p->adaptive_leaf;
    A.max_leaf = p->max_leaf_size;
    A.nbmin = cv.take<float4>(nn);
    A.nbmax = cv.take<float4>(nn);
    A.left = cv.take<int>(nn);
    A.right = cv.take<int>(nn);
    A.parent = cv.take<int>(nn);
    A.counts = cv.take<int2>(nn);
    A.state = cv.take<uint8_t>(nn);
    A.cl0 = cv.take<int>(n);
    A.cl1 = cv.take<int>(n);
    const int64_t mtiles = (n + MIN_TILE4 - 1) / MIN_TILE4 + 1;
    A.status = cv.take<unsigned long long>(mtiles);
    const int64_t ftiles = (std::min<int64_t>(n, NB4_MIN_N) + LPB / 2 - 1) / (LPB / 2) + 1;
    A.status_f = cv.take<unsigned long long>(ftiles);
    unsigned* ctl = cv.take<unsigned>(MAX_ITER + 16);
    A.tickets = ctl;
    A.bar = ctl + MAX_ITER;
    A.g = reinterpret_cast<int*>(ctl + MAX_ITER + 4);
    A.err = ctx->d_status;
    int4* rec = cv.take<int4>(n);
    int* flag = cv.take<int>(n);
    if (hp_layout_of(p) == 2) {  // the binary collapse reads them
        A.cinfo = cv.take<int4>(n);
        A.cbox = cv.take<float4>(3 * (int64_t)n);
    }
    HP_CUDA(cudaMemsetAsync(A.status, 0, mtiles * 8, s));
    HP_CUDA(cudaMemsetAsync(A.status_f, 0, ftiles * 8, s));
    HP_CUDA(cudaMemsetAsync(ctl, 0, (MAX_ITER + 16) * 4, s));
    HP_CUDA(cudaMemsetAsync(flag, 0, (size_t)n * 4, s));
    k_ploc_leaves<<<hp_div_up(n, 256), 256, 0, s>>>(A, sorted_tri, tbmin, tbmax);
    HP_CUDA(cudaGetLastError());
    hp_count_launch();
    hp_mark(ctx, s, "ploc_leaves");
    if (n > TAIL) {
        const size_t smem = LOOP_SMEM;
        HP_CUDA(cudaFuncSetAttribute(k_ploc_loop, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0;
        HP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ploc_loop, LPB, smem));
        if (per_sm < 1) return hp_fail(HP_ERR_UNSUPPORTED, "PLOC loop kernel does not fit on an SM");
        int grid = ctx->sm_count * per_sm;
        void* args[] = {&A};
        HP_CUDA(cudaLaunchCooperativeKernel((void*)k_ploc_loop, grid, LPB, args, smem, s));
        hp_count_launch();
        hp_mark(ctx, s, "ploc_loop");
    }
    HP_CUDA(cudaFuncSetAttribute(k_ploc_tail, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TAIL_SMEM));
    k_ploc_tail<<<1, PB, TAIL_SMEM, s>>>(A);
    HP_CUDA(cudaGetLastError());
    hp_count_launch();
    hp_mark(ctx, s, "ploc_tail");
    if (hp_layout_of(p) != 2) {  // N-wide layouts
        hp_wide_in W;
        W.n = n;
        W.width = hp_layout_of(p);
        W.parent = A.parent;
        W.left = A.left;
        W.right = A.right;
        W.nbmin = A.nbmin;
        W.nbmax = A.nbmax;
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
    td_args T{};
    T.n = n;
    T.left = A.left;
    T.right = A.right;
    T.parent = A.parent;
    T.counts = A.counts;
    T.state = A.state;
    T.nbmin = A.nbmin;
    T.nbmax = A.nbmax;
    T.rec = rec;
    T.flag = flag;
    T.epoch = 1;
    T.ticket = ctl + MAX_ITER + 8;
    T.sorted_tri = sorted_tri;
    T.woop_src = woop_src;
    T.verts = m->vertices;
    T.nv = m->num_vertices;
    T.tris = m->triangles;
    T.nodes = out->nodes;
    T.woop = out->woop;
    T.tri_idx = out->tri_idx;
    T.info = out->info;
    T.max_nodes = (int)std::max<int64_t>(2 * out->capacity - 1, 3);
    T.err = ctx->d_status;
    T.cinfo = A.cinfo;
    T.cbox = A.cbox;
    k_topdown<true><<<hp_div_up(nn, 256), 256, 0, s>>>(T);
    HP_CUDA(cudaGetLastError());
    hp_count_launch();
    hp_mark(ctx, s, "collapse");
    return HP_OK;
}
