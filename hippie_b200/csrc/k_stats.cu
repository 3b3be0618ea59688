// BVH quality statistics and validation on the device.
//
// Reference: HipBVH::getCost, getAvgLeafSize, getLeafSizeHistogram
// (rt/bvh/HipBVH.cpp:346-442) with kernels computeCost, computeSumOfLeafSizes
// and computeLeafSizeHistogram (rt/bvh/HipBVHKernels.cu:124-238), and
// HipBVH::validate (rt/bvh/HipBVH.cpp:157-307), which the reference runs on
// the host over the downloaded buffers.
//
// Statistics: one grid-stride pass over the nodes. Each node adds
// ct * A / A(scene) (interior) or ci * A / A(scene) * size (leaf), A being the
// area of the union of its two stored child boxes; the sums are taken in FP64
// in a fixed order (per thread, then per block, then over blocks in one CTA),
// so the cost is reproducible bit for bit, where the reference's float
// atomicAdd is not. Leaf sizes are summed as integers and counted in a
// histogram of sizes 0..32 (MAX_LEAF_SIZE, rt/bvh/HipBVHKernels.h:13); larger
// leaves are left out of the histogram as in the reference.
//
// Validation checks what the reference's does, as independent per-node tests
// whose conjunction is equivalent to its depth-first walk: the root's parent
// is -1 and its size is the reference count; every interior node lies below
// the leaf range, its children are in range, carry the matching leaf flag,
// point back to it as parent and sum to its size, and its stored child boxes
// enclose the children's own boxes; every leaf lies in the leaf range, holds a
// non-empty range [begin, end) of size ~size, and its box encloses the
// vertices of its triangles; every node except the root is the child of
// exactly one node, and every triangle is referenced by exactly one leaf.
// Sizes strictly decrease from parent to child when n > 1 (leaves hold at
// least one reference), so these counts leave no room for a cycle or an
// unreachable node. The first failure is recorded as (code, node).
#include <algorithm>
#include <cuda_runtime.h>
#include "hp_device.cuh"
#include "hp_internal.h"

namespace {

constexpr int SB = 256;         // threads per statistics CTA
constexpr int SGRID = 592;      // statistics CTAs (fixed: the FP64 sum order depends on it)
constexpr int MAX_LEAF = 32;    // histogram bins 0..MAX_LEAF

struct stats_out {
    double cost;
    long long leaf_sum;
    unsigned hist[MAX_LEAF + 1];
};

// A node of width N (HipBVHNodeN<N>, rt/bvh/HipBVHNode.h): N = 2 is the 64-byte
// binary record, N = 4 / 8 the wide records.
template <int N>
struct node_ref {
    const int* c;
    __device__ __forceinline__ float lo(int i, int a) const {
        const int k = a == 0 ? 4 * i : (a == 1 ? 4 * i + 2 : (N == 2 ? 8 + 2 * i : 4 * (N + i)));
        return __int_as_float(__ldg(c + k));
    }
    __device__ __forceinline__ float hi(int i, int a) const {
        const int k = a == 0 ? 4 * i + 1 : (a == 1 ? 4 * i + 3 : (N == 2 ? 9 + 2 * i : 4 * (N + i) + 1));
        return __int_as_float(__ldg(c + k));
    }
    __device__ __forceinline__ int child(int i) const { return __ldg(c + (N == 2 ? 12 + i : 4 * (N + i) + 2)); }
    __device__ __forceinline__ int size() const { return __ldg(c + (N == 2 ? 14 : 8 * N - 5)); }
    __device__ __forceinline__ int parent() const { return __ldg(c + (N == 2 ? 15 : 8 * N - 1)); }
    __device__ __forceinline__ int count() const { return N == 2 ? 2 : __ldg(c + 8 * N - 9); }
    __device__ __forceinline__ int begin() const { return __ldg(c + (N == 2 ? 12 : 4 * N + 2)); }
    __device__ __forceinline__ int end() const { return __ldg(c + (N == 2 ? 13 : 4 * N + 3)); }
    // HipBVHNodeN::getBoundingBox: the union of all N stored child boxes
    __device__ __forceinline__ void box(float* mn, float* mx) const {
        for (int a = 0; a < 3; ++a) { mn[a] = lo(0, a); mx[a] = hi(0, a); }
        for (int i = 1; i < N; ++i)
            for (int a = 0; a < 3; ++a) { mn[a] = fminf(mn[a], lo(i, a)); mx[a] = fmaxf(mx[a], hi(i, a)); }
    }
};

template <int N>
__device__ __forceinline__ node_ref<N> node_at(const int* nodes, int64_t i) {
    return node_ref<N>{nodes + (size_t)i * 8 * N};
}

template <int N>
__global__ void __launch_bounds__(SB) k_node_stats(const int* __restrict__ nodes,
                                                   const hp_bvh_info* __restrict__ info, float ct, float ci,
                                                   double* part_cost, long long* part_leaf, stats_out* out) {
    __shared__ unsigned s_hist[MAX_LEAF + 1];
    __shared__ double s_c[SB / 32];
    __shared__ long long s_l[SB / 32];
    if (threadIdx.x <= MAX_LEAF) s_hist[threadIdx.x] = 0;
    __syncthreads();
    const int64_t num_int = info->num_interior;
    const int64_t count = num_int + info->num_leaf;
    const float smn[3] = {hp_ord2f(info->box_ord[0]), hp_ord2f(info->box_ord[1]), hp_ord2f(info->box_ord[2])};
    const float smx[3] = {hp_ord2f(info->box_ord[3]), hp_ord2f(info->box_ord[4]), hp_ord2f(info->box_ord[5])};
    const double scene = (double)hp_area(smn[0], smn[1], smn[2], smx[0], smx[1], smx[2]);
    double c = 0.0;
    long long leaf = 0;
    for (int64_t i = blockIdx.x * (int64_t)SB + threadIdx.x; i < count; i += (int64_t)SGRID * SB) {
        const node_ref<N> nd = node_at<N>(nodes, i);
        float mn[3], mx[3];
        nd.box(mn, mx);
        const double a = (double)hp_area(mn[0], mn[1], mn[2], mx[0], mx[1], mx[2]) / scene;
        const int sz = nd.size();
        if (sz < 0) {
            const int size = ~sz;
            // computeCost: leaves of wide layouts count ceil(size / N) * N references
            const int billed = N > 2 ? (size + N - 1) / N * N : size;
            c += (double)ci * a * (double)billed;
            if (i >= num_int) {
                leaf += size;
                if (size <= MAX_LEAF) atomicAdd(&s_hist[size], 1u);
            }
        } else {
            c += (double)ct * a;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        c += __shfl_down_sync(HP_FULL_MASK, c, o);
        leaf += __shfl_down_sync(HP_FULL_MASK, leaf, o);
    }
    if (lane == 0) { s_c[warp] = c; s_l[warp] = leaf; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double bc = 0.0;
        long long bl = 0;
        for (int w = 0; w < SB / 32; ++w) { bc += s_c[w]; bl += s_l[w]; }
        part_cost[blockIdx.x] = bc;
        part_leaf[blockIdx.x] = bl;
    }
    if (threadIdx.x <= MAX_LEAF && s_hist[threadIdx.x]) atomicAdd(&out->hist[threadIdx.x], s_hist[threadIdx.x]);
}

__global__ void __launch_bounds__(32) k_stats_final(const double* part_cost, const long long* part_leaf,
                                                    stats_out* out) {
    const int lane = threadIdx.x;
    double c = 0.0;
    long long l = 0;
    for (int b = lane; b < SGRID; b += 32) { c += part_cost[b]; l += part_leaf[b]; }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        c += __shfl_down_sync(HP_FULL_MASK, c, o);
        l += __shfl_down_sync(HP_FULL_MASK, l, o);
    }
    if (lane == 0) { out->cost = c; out->leaf_sum = l; }
}

// ---- validation ---------------------------------------------------------------
enum : int {
    V_ROOT_PARENT = 1, V_ROOT_SIZE, V_INTERIOR_IN_LEAF_RANGE, V_CHILD_RANGE, V_CHILD_FLAG, V_PARENT,
    V_SIZE, V_CHILD_BOX, V_LEAF_IN_INTERIOR_RANGE, V_LEAF_BOUNDS, V_LEAF_SIZE, V_TRI_INDEX,
    V_VERTEX_INDEX, V_TRI_BOX, V_NODE_REFS, V_TRI_REFS, V_NO_NODES
};

__device__ __forceinline__ void v_fail(int* err, int code, int64_t node) {
    if (atomicCAS(err, 0, code) == 0) err[1] = (int)node;
}

struct val_args {
    const int* nodes;
    const hp_bvh_info* info;
    const int32_t* tri_idx;
    int64_t n;  // references
    const int32_t* tris;
    const float* verts;
    int64_t nv;
    int64_t cap_nodes;  // length of node_refs
    int* node_refs;  // [cap_nodes]
    int* tri_refs;   // [n]
    int* err;        // [2]
};

template <int N>
__global__ void __launch_bounds__(256) k_validate_nodes(val_args V) {
    const int64_t num_int = V.info->num_interior;
    const int64_t count = num_int + V.info->num_leaf;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i == 0 && count == 0) v_fail(V.err, V_NO_NODES, 0);
    if (count > V.cap_nodes) {  // more nodes than a tree over n references can have
        if (i == 0) v_fail(V.err, V_NODE_REFS, count);
        return;
    }
    if (i >= count) return;
    const node_ref<N> nd = node_at<N>(V.nodes, i);
    const int nsz = nd.size();
    if (i == 0) {
        if (nd.parent() != -1) v_fail(V.err, V_ROOT_PARENT, 0);
        const int64_t rs = nsz < 0 ? ~nsz : nsz;
        if (rs != V.n) v_fail(V.err, V_ROOT_SIZE, 0);
    }
    if (nsz >= 0) {
        if (i >= num_int) { v_fail(V.err, V_INTERIOR_IN_LEAF_RANGE, i); return; }
        const int nch = nd.count();
        if (nch < 1 || nch > N || (nch < 2 && V.n > 1)) { v_fail(V.err, V_CHILD_RANGE, i); return; }
        int64_t size = 0;
        for (int c = 0; c < nch; ++c) {
            const int raw = nd.child(c);
            const int64_t ch = raw < 0 ? ~(int64_t)raw : raw;
            if (ch <= 0 || ch >= count) { v_fail(V.err, V_CHILD_RANGE, i); return; }
            const node_ref<N> cn = node_at<N>(V.nodes, ch);
            const int csz = cn.size();
            if ((raw < 0) != (csz < 0)) { v_fail(V.err, V_CHILD_FLAG, i); return; }
            if (cn.parent() != i) { v_fail(V.err, V_PARENT, i); return; }
            size += csz < 0 ? ~csz : csz;
            atomicAdd(V.node_refs + ch, 1);
            const bool empty_child = csz < 0 && cn.begin() == cn.end();
            if (!empty_child) {
                float cmn[3], cmx[3];
                cn.box(cmn, cmx);
                for (int a = 0; a < 3; ++a)
                    if (cmn[a] < nd.lo(c, a) || cmx[a] > nd.hi(c, a)) { v_fail(V.err, V_CHILD_BOX, i); return; }
            }
        }
        if (size != nsz) v_fail(V.err, V_SIZE, i);
    } else {
        if (i < num_int) { v_fail(V.err, V_LEAF_IN_INTERIOR_RANGE, i); return; }
        const int64_t b = nd.begin(), e = nd.end();
        if (b > e || b < 0 || e > V.n || (b == e && V.n != 1)) { v_fail(V.err, V_LEAF_BOUNDS, i); return; }
        if (e - b != ~nsz) { v_fail(V.err, V_LEAF_SIZE, i); return; }
        float mn[3], mx[3];
        nd.box(mn, mx);
        for (int64_t r = b; r < e; ++r) {
            const int32_t t = __ldg(V.tri_idx + r);
            if (t < 0 || t >= V.n) { v_fail(V.err, V_TRI_INDEX, i); return; }
            atomicAdd(V.tri_refs + t, 1);
            for (int k = 0; k < 3; ++k) {
                const int32_t vi = __ldg(V.tris + 3 * (int64_t)t + k);
                if (vi < 0 || vi >= V.nv) { v_fail(V.err, V_VERTEX_INDEX, i); return; }
                for (int a = 0; a < 3; ++a) {
                    const float x = __ldg(V.verts + 3 * (int64_t)vi + a);
                    if (x < mn[a] || x > mx[a]) { v_fail(V.err, V_TRI_BOX, i); return; }
                }
            }
        }
    }
}

__global__ void __launch_bounds__(256) k_validate_refs(val_args V) {
    const int64_t count = std::min<int64_t>((int64_t)V.info->num_interior + V.info->num_leaf, V.cap_nodes);
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < count && V.node_refs[i] != (i == 0 ? 0 : 1)) v_fail(V.err, V_NODE_REFS, i);
    if (i < V.n && V.tri_refs[i] != 1) v_fail(V.err, V_TRI_REFS, i);
}

const char* v_message(int code) {
    switch (code) {
    case V_ROOT_PARENT: return "root parent is not -1";
    case V_ROOT_SIZE: return "root size is not the reference count";
    case V_INTERIOR_IN_LEAF_RANGE: return "interior node in the leaf range";
    case V_CHILD_RANGE: return "child index out of range";
    case V_CHILD_FLAG: return "child leaf flag mismatch";
    case V_PARENT: return "invalid parent index";
    case V_SIZE: return "invalid node size";
    case V_CHILD_BOX: return "child box not enclosed";
    case V_LEAF_IN_INTERIOR_RANGE: return "leaf node in the interior range";
    case V_LEAF_BOUNDS: return "invalid leaf bounds";
    case V_LEAF_SIZE: return "leaf size does not match its range";
    case V_TRI_INDEX: return "invalid triangle index";
    case V_VERTEX_INDEX: return "vertex index out of range";
    case V_TRI_BOX: return "triangle is not in its leaf box";
    case V_NODE_REFS: return "node not referenced exactly once";
    case V_TRI_REFS: return "triangle not referenced exactly once";
    case V_NO_NODES: return "no nodes";
    default: return "unknown";
    }
}

}  // namespace

// Both read the nodes and triangle indices through the public hp_bvh fields
// and the counts from the library's record of the build.
hp_status hp_bvh_stats_run(hp_ctx* ctx, const hp_bvh* bvh, hp_bvh_stats* out, cudaStream_t s) {
    const hp_bvh_impl* b = reinterpret_cast<const hp_bvh_impl*>(bvh->impl);
    const size_t need = hp_carve::pad(SGRID * sizeof(double)) + hp_carve::pad(SGRID * sizeof(long long)) +
                        hp_carve::pad(sizeof(stats_out)) + hp_carve::pad(sizeof(hp_bvh_info));
    HP_TRY(hp_ctx_reserve(ctx, need, s));
    hp_carve cv(ctx->arena);
    double* pc = cv.take<double>(SGRID);
    long long* pl = cv.take<long long>(SGRID);
    stats_out* so = cv.take<stats_out>(1);
    hp_bvh_info* inf = cv.take<hp_bvh_info>(1);
    HP_CUDA(cudaMemsetAsync(so, 0, sizeof(stats_out), s));
    const int* nodes = reinterpret_cast<const int*>(bvh->nodes);
    if (b->layout == 4) k_node_stats<4><<<SGRID, SB, 0, s>>>(nodes, b->info, bvh->ct, bvh->ci, pc, pl, so);
    else if (b->layout == 8) k_node_stats<8><<<SGRID, SB, 0, s>>>(nodes, b->info, bvh->ct, bvh->ci, pc, pl, so);
    else k_node_stats<2><<<SGRID, SB, 0, s>>>(nodes, b->info, bvh->ct, bvh->ci, pc, pl, so);
    k_stats_final<<<1, 32, 0, s>>>(pc, pl, so);
    HP_CUDA(cudaGetLastError());
    hp_count_launch(2);
    HP_CUDA(cudaMemcpyAsync(inf, b->info, sizeof(hp_bvh_info), cudaMemcpyDeviceToDevice, s));
    stats_out h;
    hp_bvh_info hi;
    HP_CUDA(cudaMemcpyAsync(&h, so, sizeof(h), cudaMemcpyDeviceToHost, s));
    HP_CUDA(cudaMemcpyAsync(&hi, inf, sizeof(hi), cudaMemcpyDeviceToHost, s));
    HP_CUDA(cudaStreamSynchronize(s));
    out->sah_cost = h.cost;
    out->sum_of_leaf_sizes = h.leaf_sum;
    out->num_interior = hi.num_interior;
    out->num_leaf = hi.num_leaf;
    out->avg_leaf_size = hi.num_leaf > 0 ? (double)h.leaf_sum / (double)hi.num_leaf : 0.0;
    for (int k = 0; k <= MAX_LEAF; ++k)
        out->leaf_size_histogram[k] = hi.num_leaf > 0 ? (float)h.hist[k] / (float)hi.num_leaf : 0.0f;
    return HP_OK;
}

hp_status hp_bvh_validate_run(hp_ctx* ctx, const hp_bvh* bvh, const hp_mesh* m, int32_t* valid, cudaStream_t s) {
    const hp_bvh_impl* b = reinterpret_cast<const hp_bvh_impl*>(bvh->impl);
    const int64_t n = bvh->num_refs;
    const int64_t cap_nodes = 2 * n + 1;  // 2n - 1, or 3 for a single binary reference (root + two leaves)
    const size_t need = hp_carve::pad(cap_nodes * 4) + hp_carve::pad(std::max<int64_t>(n, 1) * 4) +
                        hp_carve::pad(2 * sizeof(int));
    HP_TRY(hp_ctx_reserve(ctx, need, s));
    hp_carve cv(ctx->arena);
    val_args V{};
    V.nodes = reinterpret_cast<const int*>(bvh->nodes);
    V.info = b->info;
    V.tri_idx = bvh->tri_indices;
    V.n = n;
    V.tris = m->triangles;
    V.verts = m->vertices;
    V.nv = m->num_vertices;
    V.cap_nodes = cap_nodes;
    V.node_refs = cv.take<int>(cap_nodes);
    V.tri_refs = cv.take<int>(std::max<int64_t>(n, 1));
    V.err = cv.take<int>(2);
    HP_CUDA(cudaMemsetAsync(ctx->arena, 0, cv.off, s));
    const int64_t grid = hp_div_up(cap_nodes, 256);
    if (b->layout == 4) k_validate_nodes<4><<<(unsigned)grid, 256, 0, s>>>(V);
    else if (b->layout == 8) k_validate_nodes<8><<<(unsigned)grid, 256, 0, s>>>(V);
    else k_validate_nodes<2><<<(unsigned)grid, 256, 0, s>>>(V);
    k_validate_refs<<<(unsigned)grid, 256, 0, s>>>(V);
    HP_CUDA(cudaGetLastError());
    hp_count_launch(2);
    int e[2];
    HP_CUDA(cudaMemcpyAsync(e, V.err, sizeof(e), cudaMemcpyDeviceToHost, s));
    HP_CUDA(cudaStreamSynchronize(s));
    HP_TRY(hp_ctx_check(ctx, s));
    *valid = e[0] == 0 ? 1 : 0;
    if (e[0]) hp_set_error(std::string("validate: ") + v_message(e[0]) + " (node " + std::to_string(e[1]) + ")");
    return HP_OK;
}
