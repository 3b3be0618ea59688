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

__device__ __forceinline__ void node_union(const hp_node_bin& n, float* mn, float* mx) {
    mn[0] = fminf(n.c0xy.x, n.c1xy.x); mx[0] = fmaxf(n.c0xy.y, n.c1xy.y);
    mn[1] = fminf(n.c0xy.z, n.c1xy.z); mx[1] = fmaxf(n.c0xy.w, n.c1xy.w);
    mn[2] = fminf(n.cz.x, n.cz.z);     mx[2] = fmaxf(n.cz.y, n.cz.w);
}

__device__ __forceinline__ hp_node_bin load_bin(const hp_node_bin* nodes, int64_t i) {
    const float4* p = reinterpret_cast<const float4*>(nodes + i);
    hp_node_bin n;
    n.c0xy = __ldg(p + 0);
    n.c1xy = __ldg(p + 1);
    n.cz = __ldg(p + 2);
    const float4 m = __ldg(p + 3);
    n.meta = make_int4(__float_as_int(m.x), __float_as_int(m.y), __float_as_int(m.z), __float_as_int(m.w));
    return n;
}

__global__ void __launch_bounds__(SB) k_node_stats(const hp_node_bin* __restrict__ nodes,
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
        const hp_node_bin nd = load_bin(nodes, i);
        float mn[3], mx[3];
        node_union(nd, mn, mx);
        const double a = (double)hp_area(mn[0], mn[1], mn[2], mx[0], mx[1], mx[2]) / scene;
        if (nd.meta.z < 0) {
            const int size = ~nd.meta.z;
            c += (double)ci * a * (double)size;
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
    const hp_node_bin* nodes;
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
    const hp_node_bin nd = load_bin(V.nodes, i);
    if (i == 0) {
        if (nd.meta.w != -1) v_fail(V.err, V_ROOT_PARENT, 0);
        const int64_t rs = nd.meta.z < 0 ? ~nd.meta.z : nd.meta.z;
        if (rs != V.n) v_fail(V.err, V_ROOT_SIZE, 0);
    }
    if (nd.meta.z >= 0) {
        if (i >= num_int) { v_fail(V.err, V_INTERIOR_IN_LEAF_RANGE, i); return; }
        int64_t size = 0;
        for (int c = 0; c < 2; ++c) {
            const int raw = c == 0 ? nd.meta.x : nd.meta.y;
            const int64_t ch = raw < 0 ? ~(int64_t)raw : raw;
            if (ch <= 0 || ch >= count) { v_fail(V.err, V_CHILD_RANGE, i); return; }
            const hp_node_bin cn = load_bin(V.nodes, ch);
            if ((raw < 0) != (cn.meta.z < 0)) { v_fail(V.err, V_CHILD_FLAG, i); return; }
            if (cn.meta.w != i) { v_fail(V.err, V_PARENT, i); return; }
            size += cn.meta.z < 0 ? ~cn.meta.z : cn.meta.z;
            atomicAdd(V.node_refs + ch, 1);
            const bool empty_child = cn.meta.z < 0 && cn.meta.x == cn.meta.y;
            if (!empty_child) {
                float cmn[3], cmx[3];
                node_union(cn, cmn, cmx);
                const float4 xy = c == 0 ? nd.c0xy : nd.c1xy;
                const float bmn[3] = {xy.x, xy.z, c == 0 ? nd.cz.x : nd.cz.z};
                const float bmx[3] = {xy.y, xy.w, c == 0 ? nd.cz.y : nd.cz.w};
                for (int a = 0; a < 3; ++a)
                    if (cmn[a] < bmn[a] || cmx[a] > bmx[a]) { v_fail(V.err, V_CHILD_BOX, i); return; }
            }
        }
        if (size != nd.meta.z) v_fail(V.err, V_SIZE, i);
    } else {
        if (i < num_int) { v_fail(V.err, V_LEAF_IN_INTERIOR_RANGE, i); return; }
        const int64_t b = nd.meta.x, e = nd.meta.y;
        if (b > e || b < 0 || e > V.n || (b == e && V.n != 1)) { v_fail(V.err, V_LEAF_BOUNDS, i); return; }
        if (e - b != ~nd.meta.z) { v_fail(V.err, V_LEAF_SIZE, i); return; }
        float mn[3], mx[3];
        node_union(nd, mn, mx);
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
    k_node_stats<<<SGRID, SB, 0, s>>>(reinterpret_cast<const hp_node_bin*>(bvh->nodes), b->info, bvh->ct, bvh->ci,
                                      pc, pl, so);
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
    const int64_t cap_nodes = 2 * n + 1;  // 2n - 1, or 3 for a single reference (root + two leaves)
    const size_t need = hp_carve::pad(cap_nodes * 4) + hp_carve::pad(std::max<int64_t>(n, 1) * 4) +
                        hp_carve::pad(2 * sizeof(int));
    HP_TRY(hp_ctx_reserve(ctx, need, s));
    hp_carve cv(ctx->arena);
    val_args V{};
    V.nodes = reinterpret_cast<const hp_node_bin*>(bvh->nodes);
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
    k_validate_nodes<<<(unsigned)grid, 256, 0, s>>>(V);
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
