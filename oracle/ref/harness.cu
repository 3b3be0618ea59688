// Host harness that drives the REFERENCE's own CUDA kernels (test
// infrastructure: it pins the oracle and gives the reference GPU timing).
//
// The sequences restate, without Qt or HIP, the reference host code:
//   LBVHBuilder::build          rt/bvh/LBVHBuilder.cpp:183-241
//   PLOCBuilder::clustering     rt/bvh/PLOCBuilder.cpp:21-159, build :161-208
//   ATRBuilder::build / optimize / generateSchedule
//                               rt/bvh/ATRBuilder.cpp:23-236
//   BVHCollapser::collapseAdaptive + computeNodeOffsets loop
//                               rt/bvh/BVHCollapser.cpp:14-306,521-597
//   HipBVH::woopifyTriangles    rt/bvh/HipBVH.cpp:95-116
//   HipBVH::getCost             rt/bvh/HipBVH.cpp:346-370
//   HipTracer::trace            rt/tracer/HipTracer.cpp:13-52
// Each kernel is timed like HipKernel::launchTimed (gpu/HipKernel.cpp:296-325):
// synchronise, event, launch, event, synchronise; the build time is the sum.
// Deliberate differences: PLOC never writes nodeParentIndices[0] (the root's
// parent) and the collapser reads it, so the harness sets it to -1; and the
// sort step uses CUB's stable radix sort instead of the reference's radix sort
// kernels (see the note at the sort below).
#include <algorithm>
#include <cstdio>
#include <vector>
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include "hpref.h"

namespace {

struct timer {
    cudaEvent_t a, b;
    double total = 0.0;
    timer() { cudaEventCreate(&a); cudaEventCreate(&b); }
    ~timer() { cudaEventDestroy(a); cudaEventDestroy(b); }
    template <typename F> void run(F f) {
        cudaDeviceSynchronize();
        cudaEventRecord(a, 0);
        f();
        cudaEventRecord(b, 0);
        cudaEventSynchronize(b);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, a, b);
        total += ms * 1e-3;
    }
};

template <typename T> T* dalloc(size_t count) {
    T* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) return nullptr;
    return p;
}

char g_err[512] = "";
int fail(int code, const char* where) {
    cudaError_t e = cudaGetLastError();
    std::snprintf(g_err, sizeof(g_err), "%s: %s", where, cudaGetErrorString(e));
    return code;
}

#define ROUND_UP(x, y) ((((x) + (y) - 1) / (y)) * (y))

// Host check of a binary tree over nodes 0..2n-2 (root 0, leaves n-1..):
// every interior node's children are in range, name it as parent, and every
// node but the root is a child exactly once, and a walk from the root reaches
// all 2n-1 nodes (no detached cycle). Kernels that climb these links only run
// on a tree that passes.
bool valid_tree(int n, const int* parent, const int* left, const int* right) {
    const int nn = 2 * n - 1;
    std::vector<int> hp(nn), hl(nn), hr(nn), uses(nn, 0);
    if (cudaMemcpy(hp.data(), parent, nn * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(hl.data(), left, nn * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(hr.data(), right, nn * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        return false;
    if (hp[0] != -1) return false;
    for (int i = 0; i < n - 1; ++i)
        for (int c : {hl[i], hr[i]})
            if (c <= 0 || c >= nn || hp[c] != i || uses[c]++) return false;
    int seen = 0;
    std::vector<int> st{0};
    while (!st.empty()) {
        const int v = st.back();
        st.pop_back();
        if (++seen > nn) return false;
        if (v < n - 1) { st.push_back(hl[v]); st.push_back(hr[v]); }
    }
    return seen == nn;
}

// BVHCollapser::collapseAdaptive (Bin layout).
void ref_collapse(timer& T, int n, int* parent, int* left, int* right, float4* nbmin, float4* nbmax, int* tri1,
                  int* tri_out, void* nodes, float ct, float ci, int* counts) {
    const int nn = 2 * n - 1;
    int* counters = dalloc<int>(n);
    int* sizes = dalloc<int>(nn);
    int* states = dalloc<int>(nn);
    float* costs = dalloc<float>(nn);
    int* leaf_idx = dalloc<int>(n);
    int* node_off = dalloc<int>(nn);
    int* node_idx = dalloc<int>(n);
    int* ref_off = dalloc<int>(nn);
    cudaMemset(counters, 0, n * 4);
    // computeNodeOffsets writes the offsets of children only; the compaction
    // reads the root's, which the reference's fresh buffer holds as 0.
    cudaMemset(node_off, 0, nn * 4);
    T.run([&] { hpref_collapse_sizes(nn, counters, parent, left, right, sizes); });
    cudaMemset(counters, 0, n * 4);
    T.run([&] { hpref_collapse_states(n, ci, ct, counters, costs, parent, left, right, sizes, states, nbmin, nbmax); });
    T.run([&] { hpref_collapse_leaf_indices(n, leaf_idx, parent, states); });
    cudaMemset(counters, 0, n * 4);
    T.run([&] { hpref_collapse_invalidate(n, counters, leaf_idx, parent, states); });
    hpref_collapse_offsets_begin();
    cudaMemset(node_idx, 0, 4);
    int task_offset = 0, tasks = 1;
    while (tasks > 0) {
        T.run([&] { hpref_collapse_offsets(task_offset, tasks, left, right, node_idx, node_off, states); });
        task_offset += tasks;
        tasks = hpref_collapse_interiors() - task_offset;
    }
    T.run([&] { hpref_collapse_ref_offsets(nn, states, sizes, ref_off); });
    const int n_int = hpref_collapse_interiors(), n_leaf = hpref_collapse_leaves();
    T.run([&] { hpref_collapse_compact(nn, n_int, states, node_off, parent, left, right, sizes, ref_off, nbmin,
                                       nbmax, nodes); });
    T.run([&] { hpref_collapse_reorder(n, left, ref_off, tri1, tri_out, leaf_idx); });
    counts[0] = n_int;
    counts[1] = n_leaf;
    cudaFree(counters); cudaFree(sizes); cudaFree(states); cudaFree(costs); cudaFree(leaf_idx);
    cudaFree(node_off); cudaFree(node_idx); cudaFree(ref_off);
}

// ATRBuilder::generateSchedule (rt/bvh/ATRBuilder.cpp:23-56): the pairs (i, j),
// j < i < T, packed two per int (a pair per 16 bits), 32 pairs per half-row.
std::vector<int> atr_schedule(int T) {
    const int elements = (T - 1) * T / 2;
    const int iters = (elements + 63) / 64;
    std::vector<int> s(iters * 32, 0);
    int count = 0;
    float mult = 0.0f;
    for (int i = 0; i < T; ++i) {
        for (int j = 0; j < i; ++j) {
            const int idx = count + static_cast<int>(mult) * 32;
            s[idx] = (s[idx] << 16) | (i << 8) | j;
            if (++count == 32) {
                mult += 0.5f;
                count = 0;
            }
        }
    }
    if (static_cast<int>(mult + 0.5f) > static_cast<int>(mult))
        for (int i = count; i < 32; ++i) s[i + static_cast<int>(mult) * 32] <<= 16;
    return s;
}

// ATRBuilder::computeSurfaceAreas + optimize on a refitted LBVH.
int ref_atr(timer& T, int n, int treelet, int iterations, float ct, float ci, int* parent, int* left, int* right,
            float4* nbmin, float4* nbmax) {
    const int nn = 2 * n - 1;
    const std::vector<int> hs = atr_schedule(treelet);
    int* schedule = dalloc<int>(hs.size());
    cudaMemcpy(schedule, hs.data(), hs.size() * 4, cudaMemcpyHostToDevice);
    const int dist_size = (treelet - 1) * treelet / 2;
    float* areas = dalloc<float>(nn);
    float* costs = dalloc<float>(nn);
    int* refs = dalloc<int>(nn);
    int* counters = dalloc<int>(n);
    float* dist = treelet > 20 ? dalloc<float>((size_t)dist_size * ((n + 31) / 32)) : nullptr;
    int smem = ((2 * treelet - 1) * 4 + treelet * 4) * 4;
    if (treelet <= 20) smem += dist_size * 4 * 4;
    T.run([&] { hpref_atr_areas(nn, areas, nbmin, nbmax); });
    int gamma = treelet;
    for (int i = 0; i < iterations; ++i) {
        cudaMemset(counters, 0, n * 4);
        T.run([&] { hpref_atr_optimize(n, treelet, (int)hs.size(), dist_size, gamma, ci, ct, costs, areas, dist,
                                       left, right, nbmin, nbmax, counters, parent, refs, schedule, smem); });
        // The next launch climbs parent links with no bound: it only runs on a
        // tree that is still valid.
        if (!valid_tree(n, parent, left, right)) {
            std::fprintf(stderr, "reference ATR produced an invalid tree (iteration %d)\n", i);
            cudaFree(schedule); cudaFree(areas); cudaFree(costs); cudaFree(refs); cudaFree(counters); cudaFree(dist);
            return 4;
        }
        gamma *= 2;
        if (gamma > n) break;
    }
    cudaError_t e = cudaDeviceSynchronize();
    cudaFree(schedule); cudaFree(areas); cudaFree(costs); cudaFree(refs); cudaFree(counters); cudaFree(dist);
    if (e != cudaSuccess) return fail(9, "after ATR optimize");
    return 0;
}

// HLBVHBuilder::build after construct (rt/bvh/HLBVHBuilder.cpp:359-391) and
// HLBVHBuilder::split (rt/bvh/HLBVHBuilder.cpp:237-328) on a Karras tree
// (parent / left / right, leaf boxes set) and its sorted keys. Writes the
// HLBVH topology into hparent / hleft / hright and its boxes into nbmin /
// nbmax. Only run where the reference's index bookkeeping holds: Morton SAH
// bits a multiple of 3 (else its bin coordinates run past their axis) and the
// root outside every cluster (else its compaction and its top-level node
// counter hand out the same indices).
int ref_hlbvh(timer& T, int n, int bits, int sah, int* parent, int* left, int* right, unsigned long long* keys,
              float4* nbmin, float4* nbmax, int* hparent, int* hleft, int* hright) {
    if (sah % 3 != 0 || sah < 6 || sah > 15 || sah > bits) {
        std::snprintf(g_err, sizeof(g_err), "HLBVH: Morton SAH bits must be 6, 9, 12 or 15 and at most the bits");
        return 10;
    }
    unsigned long long k0 = 0, k1 = 0;
    if (cudaMemcpy(&k0, keys, 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(&k1, keys + (n - 1), 8, cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(10, "reading the sorted keys");
    if (((k0 ^ k1) >> (bits - sah)) == 0) {
        std::snprintf(g_err, sizeof(g_err), "HLBVH: every key shares the top Morton SAH bits (root in a cluster)");
        return 11;
    }
    const int nn = 2 * n - 1;
    int* counters = dalloc<int>(n);
    int* states = dalloc<int>(nn);
    int* offsets = dalloc<int>(n);
    int* leaf_cluster = dalloc<int>(n);
    int* cl_tasks = dalloc<int>(n);
    int* cl_nodes = dalloc<int>(n);
    int4* cl_bins = dalloc<int4>(n);
    cudaMemset(cl_bins, 0, (size_t)n * 16);
    cudaMemset(counters, 0, (size_t)n * 4);
    T.run([&] { hpref_hl_node_states(n, bits, sah, counters, parent, left, right, states, keys); });
    T.run([&] { hpref_hl_leaf_clusters(n, leaf_cluster, parent, states); });
    cudaMemset(counters, 0, (size_t)n * 4);
    T.run([&] { hpref_hl_invalidate(n, counters, leaf_cluster, parent, states); });
    hpref_hl_set_counter(0);
    T.run([&] { hpref_hl_node_offsets(n, offsets, states); });
    T.run([&] { hpref_hl_compact(n, offsets, states, parent, left, right, hparent, hleft, hright); });
    hpref_hl_set_counter(0);
    T.run([&] { hpref_hl_clusters(n, bits, sah, states, offsets, left, cl_nodes, cl_bins, keys); });
    const int C = hpref_hl_counter();
    int rc = 0;
    if (cudaDeviceSynchronize() != cudaSuccess) rc = fail(9, "after the HLBVH cluster kernels");
    else if (C < 2 || C > n) rc = fail(12, "HLBVH cluster count out of range");
    if (!rc) {
        cudaMemset(counters, 0, (size_t)n * 4);
        T.run([&] { hpref_refit(nn, counters, hparent, hleft, hright, nbmin, nbmax); });
        cudaMemset(cl_tasks, 0, (size_t)n * 4);
        hpref_hl_set_counter(1);
        const int NB = 1 << (sah / 3);
        float4* bmin = dalloc<float4>((size_t)3 * C * NB);
        float4* bmax = dalloc<float4>((size_t)3 * C * NB);
        int* new_tasks = dalloc<int>(C);
        int* split_idx = dalloc<int>(C);
        int2* q[2] = {dalloc<int2>(C), dalloc<int2>(C)};
        int* out_size = dalloc<int>(1);
        const int2 root = make_int2(0, -1);
        cudaMemcpy(q[0], &root, sizeof(root), cudaMemcpyHostToDevice);
        int in = 1, cur = 0, levels = 0;
        while (in > 0) {
            if (++levels > 2 * C + 2) { rc = fail(13, "HLBVH split did not terminate"); break; }
            cudaMemset(out_size, 0, 4);
            T.run([&] { hpref_hl_reset_bins(3 * in * NB, bmin, bmax); });
            T.run([&] { hpref_hl_bin(in, NB, C, cl_tasks, cl_nodes, cl_bins, nbmin, nbmax, bmin, bmax); });
            T.run([&] { hpref_hl_split(NB, in, out_size, new_tasks, split_idx, hparent, hleft, hright, nbmin, nbmax,
                                       bmin, bmax, q[cur], q[cur ^ 1]); });
            T.run([&] { hpref_hl_distribute(in, NB, C, new_tasks, split_idx, hparent, hleft, hright, cl_tasks,
                                            cl_nodes, cl_bins, bmin, bmax, q[cur]); });
            if (cudaMemcpy(&in, out_size, 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
                rc = fail(9, "after an HLBVH split level");
                break;
            }
            if (in < 0 || in > C) { rc = fail(12, "HLBVH task count out of range"); break; }
            cur ^= 1;
        }
        cudaFree(bmin); cudaFree(bmax); cudaFree(new_tasks); cudaFree(split_idx); cudaFree(q[0]); cudaFree(q[1]);
        cudaFree(out_size);
    }
    cudaFree(counters); cudaFree(states); cudaFree(offsets); cudaFree(leaf_cluster); cudaFree(cl_tasks);
    cudaFree(cl_nodes); cudaFree(cl_bins);
    return rc;
}

}  // namespace

extern "C" {

const char* hpref_last_error(void) { return g_err; }

// Build a BVH with the reference's kernels. method 0 = LBVH, 1 = PLOC, 2 = ATR
// (LBVH + treelet restructuring; radius carries the treelet size, max_radius
// the iteration count), 3 = HLBVH (radius carries the Morton SAH bits).
// Device inputs: verts, tris. Device outputs: nodes (64 B x (2n-1)), woop
// (48 B x n), tri_idx (n). Optional device taps (null to skip): morton keys
// (u64 n) before sorting, sorted keys, sorted reference indices, and the
// pre-collapse parent / left / right (2n-1) and node boxes (2n-1 float4 x 2).
// Host outputs: counts[2] (interior, leaf nodes), seconds (summed kernel time),
// iterations (PLOC steps). Returns 0 on success.
int hpref_build(int method, const float* verts, const int* tris, int n, const float* scene_box, int bits,
                int radius, int max_radius, int adaptive_r, float ct, float ci, void* nodes, float4* woop,
                int* tri_idx, unsigned long long* tap_keys, unsigned long long* tap_sorted, int* tap_refs,
                int* tap_parent, int* tap_left, int* tap_right, float4* tap_bmin, float4* tap_bmax, int* counts,
                double* seconds, int* iterations) {
    if (n < 2) return 1;
    int dev = 0, sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev);
    const int nn = 2 * n - 1;
    timer T;
    float4* rbmin = dalloc<float4>(n);
    float4* rbmax = dalloc<float4>(n);
    // Sort buffers are padded, and the sorted order is checked on the host
    // before any kernel indexes memory with it.
    const size_t pad_n = 3 * (size_t)n + 65536;
    unsigned long long* keys0 = dalloc<unsigned long long>(pad_n);
    unsigned long long* keys1 = dalloc<unsigned long long>(pad_n);
    int* refs0 = dalloc<int>(pad_n);
    int* refs1 = dalloc<int>(pad_n);
    int* tri0 = tri_idx;  // bvh.getTriangleIndices(): setupBoxes writes 0..n-1, the collapser the final order
    int* tri1 = dalloc<int>(n);
    int* parent = dalloc<int>(nn);
    int* left = dalloc<int>(nn);
    int* right = dalloc<int>(nn);
    float4* nbmin = dalloc<float4>(nn);
    float4* nbmax = dalloc<float4>(nn);
    // LBVHBuilder::build
    T.run([&] { hpref_setup_boxes(n, tri0, tris, verts, rbmin, rbmax); });
    hpref_set_scene_box(scene_box);
    T.run([&] { hpref_morton60(n, bits, keys0, refs0, rbmin, rbmax); });
    if (tap_keys) cudaMemcpy(tap_keys, keys0, n * 8, cudaMemcpyDeviceToDevice);
    std::vector<unsigned long long> unsorted(n);
    if (cudaMemcpy(unsorted.data(), keys0, n * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(7, "after setupBoxes / computeMortonCodes60");
    // The reference's own radix sort kernels (radix_sort/RadixSortKernels.cu)
    // rank keys with pre-Volta warp-synchronous shared-memory scans; on this
    // GPU they failed for a 3000-key input, so they are not run. Their output is
    // by definition the stable sort of (key, index) pairs; CUB's stable radix
    // sort produces it (timed like every other kernel).
    {
        size_t temp_bytes = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, keys0, keys1, refs0, refs1, n, 0, bits);
        void* temp = nullptr;
        if (cudaMalloc(&temp, std::max<size_t>(temp_bytes, 1)) != cudaSuccess) return fail(5, "sort temp");
        T.run([&] { cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys0, keys1, refs0, refs1, n, 0, bits); });
        cudaFree(temp);
        if (cudaMemcpy(keys0, keys1, n * 8, cudaMemcpyDeviceToDevice) != cudaSuccess ||
            cudaMemcpy(refs0, refs1, n * 4, cudaMemcpyDeviceToDevice) != cudaSuccess)
            return fail(6, "after sort");
    }
    (void)sm;
    {
        // The later kernels index memory with this output: check that it is the
        // stable sort of the keys before any of them runs.
        std::vector<int> h(n), seen(n, 0);
        std::vector<unsigned long long> hk(n);
        if (cudaMemcpy(h.data(), refs0, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(hk.data(), keys0, n * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
            return fail(8, "reading the sorted keys");
        for (int i = 0; i < n; ++i) {
            bool ok = h[i] >= 0 && h[i] < n && !seen[h[i]]++ && hk[i] == unsorted[h[i]];
            if (ok && i > 0) ok = hk[i - 1] < hk[i] || (hk[i - 1] == hk[i] && h[i - 1] < h[i]);
            if (!ok) {
                std::fprintf(stderr, "reference sort output is not the stable sort of its keys (position %d)\n", i);
                return 3;
            }
        }
    }
    if (tap_sorted) cudaMemcpy(tap_sorted, keys0, n * 8, cudaMemcpyDeviceToDevice);
    if (tap_refs) cudaMemcpy(tap_refs, refs0, n * 4, cudaMemcpyDeviceToDevice);
    T.run([&] { hpref_setup_leaves(n, refs0, refs1, tri0, tri1, left, right, nbmin, nbmax, rbmin, rbmax); });
    int iters = 0;
    if (method == 3) {  // HLBVH: radius carries the Morton SAH bits
        T.run([&] { hpref_construct60(n, parent, left, right, keys0); });
        if (!valid_tree(n, parent, left, right)) {
            std::fprintf(stderr, "reference construct60 produced an invalid tree\n");
            return 4;
        }
        int* hparent = dalloc<int>(nn);
        int* hleft = dalloc<int>(nn);
        int* hright = dalloc<int>(nn);
        const int rc = ref_hlbvh(T, n, bits, radius, parent, left, right, keys0, nbmin, nbmax, hparent, hleft, hright);
        if (!rc) {
            cudaMemcpy(parent, hparent, nn * 4, cudaMemcpyDeviceToDevice);
            cudaMemcpy(left, hleft, nn * 4, cudaMemcpyDeviceToDevice);
            cudaMemcpy(right, hright, nn * 4, cudaMemcpyDeviceToDevice);
        }
        cudaFree(hparent); cudaFree(hleft); cudaFree(hright);
        if (rc) return rc;
        if (!valid_tree(n, parent, left, right)) {
            std::fprintf(stderr, "reference HLBVH produced an invalid tree\n");
            return 4;
        }
    } else if (method == 0 || method == 2) {
        T.run([&] { hpref_construct60(n, parent, left, right, keys0); });
        if (!valid_tree(n, parent, left, right)) {
            std::fprintf(stderr, "reference construct60 produced an invalid tree\n");
            return 4;
        }
        int* counters = dalloc<int>(n);
        cudaMemset(counters, 0, n * 4);
        T.run([&] { hpref_refit(nn, counters, parent, left, right, nbmin, nbmax); });
        cudaFree(counters);
        if (method == 2) {
            const int rc = ref_atr(T, n, radius, max_radius, ct, ci, parent, left, right, nbmin, nbmax);
            if (rc) return rc;
            if (!valid_tree(n, parent, left, right)) {
                std::fprintf(stderr, "reference ATR produced an invalid tree\n");
                return 4;
            }
        }
    } else {
        // PLOCBuilder::build: referenceIndices[0] = referenceIndices[1], then clustering
        cudaMemcpy(refs0, refs1, n * 4, cudaMemcpyDeviceToDevice);
        const int m1 = -1;
        cudaMemcpy(parent, &m1, 4, cudaMemcpyHostToDevice);
        float* dist = dalloc<float>(nn);
        int* nbr = dalloc<int>(nn);
        int* block_off = dalloc<int>((n + 1023) / 1024 + 1);
        int* thread_off = reinterpret_cast<int*>(keys0);  // mortonCodes[0] reused as scratch
        int* bufs[2] = {refs0, refs1};
        bool sw = false;
        int clusters = n, r = radius;
        while (clusters > 1) {
            ++iters;
            if (adaptive_r) r = std::min(r + 1, max_radius);
            T.run([&] { hpref_ploc_neighbours(clusters, r, dist, nbr, nbmin, nbmax, bufs[sw]); });
            hpref_ploc_reset();
            T.run([&] { hpref_ploc_merge(clusters, clusters - 2, nbr, bufs[sw], bufs[!sw], parent, left, right, nbmin,
                                         nbmax); });
            const int merged = hpref_ploc_merged();
            sw = !sw;
            T.run([&] { hpref_ploc_scan_compact(clusters, bufs[sw], bufs[!sw], thread_off, block_off); });
            clusters -= merged;
            sw = !sw;
            if (merged == 0) break;  // would never terminate
        }
        cudaFree(dist); cudaFree(nbr); cudaFree(block_off);
        if (clusters != 1 || !valid_tree(n, parent, left, right)) {
            std::fprintf(stderr, "reference PLOC clustering produced an invalid tree\n");
            return 4;
        }
    }
    if (tap_parent) cudaMemcpy(tap_parent, parent, nn * 4, cudaMemcpyDeviceToDevice);
    if (tap_left) cudaMemcpy(tap_left, left, nn * 4, cudaMemcpyDeviceToDevice);
    if (tap_right) cudaMemcpy(tap_right, right, nn * 4, cudaMemcpyDeviceToDevice);
    if (tap_bmin) cudaMemcpy(tap_bmin, nbmin, nn * 16, cudaMemcpyDeviceToDevice);
    if (tap_bmax) cudaMemcpy(tap_bmax, nbmax, nn * 16, cudaMemcpyDeviceToDevice);
    ref_collapse(T, n, parent, left, right, nbmin, nbmax, tri1, tri0, nodes, ct, ci, counts);
    T.run([&] { hpref_woopify(n, tri0, tris, verts, woop); });
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) fail(2, "after the collapse / woopify");
    cudaFree(rbmin); cudaFree(rbmax); cudaFree(keys0); cudaFree(keys1); cudaFree(refs0); cudaFree(refs1);
    cudaFree(tri1); cudaFree(parent); cudaFree(left); cudaFree(right); cudaFree(nbmin); cudaFree(nbmax);
    *seconds = T.total;
    if (iterations) *iterations = iters;
    return e == cudaSuccess ? 0 : 2;
}

// Closest-hit (any_hit = 0) or any-hit trace with the reference's tracer.
int hpref_trace(const void* nodes, const float4* woop, const int* tri_idx, const float4* rays, int num_rays,
                int4* results, int any_hit, double* seconds) {
    timer T;
    T.run([&] { hpref_trace_launch(num_rays, any_hit != 0, const_cast<float4*>(rays), results,
                                   (float4*)nodes, const_cast<float4*>(woop), nullptr, const_cast<int*>(tri_idx)); });
    *seconds = T.total;
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

float hpref_bvh_cost(void* nodes, int num_nodes, float scene_area, float ct, float ci) {
    return hpref_cost(num_nodes, scene_area, ct, ci, nodes);
}

}  // extern "C"
