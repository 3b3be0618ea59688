// Host harness that drives the REFERENCE's own CUDA kernels (test
// infrastructure: it pins the oracle and gives the reference GPU timing).
//
// The sequences restate, without Qt or HIP, the reference host code:
//   LBVHBuilder::build          rt/bvh/LBVHBuilder.cpp:183-241
//   PLOCBuilder::clustering     rt/bvh/PLOCBuilder.cpp:21-159, build :161-208
//   RadixSort::sort/dispatch    radix_sort/RadixSort.cpp:29-238
//   BVHCollapser::collapseAdaptive + computeNodeOffsets loop
//                               rt/bvh/BVHCollapser.cpp:14-306,521-597
//   HipBVH::woopifyTriangles    rt/bvh/HipBVH.cpp:95-116
//   HipBVH::getCost             rt/bvh/HipBVH.cpp:346-370
//   HipTracer::trace            rt/tracer/HipTracer.cpp:13-52
// Each kernel is timed like HipKernel::launchTimed (gpu/HipKernel.cpp:296-325):
// synchronise, event, launch, event, synchronise; the build time is the sum.
// One deliberate difference: PLOC never writes nodeParentIndices[0]
// (the root's parent) and the collapser reads it; the harness sets it to -1.
#include <algorithm>
#include <cstdio>
#include <vector>
#include <cuda_runtime.h>
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

#define ROUND_UP(x, y) ((((x) + (y) - 1) / (y)) * (y))

// RadixSort::getMaxGridSize for compute capability >= 3.0 with the reference's
// policy constants (radix_sort/RadixSortPolicy.h).
int max_grid_size(int sm_count) {
    int regs = 0, smem = 0;
    hpref_sort_attrs(&regs, &smem);
    const int warp_threads = 32, max_sm_blocks = 16, max_sm_warps = 2048 / 32, max_sm_regs = 64 * 1024;
    const int warp_alloc_unit = 4, smem_alloc_unit = 256, reg_alloc_unit = 256, smem_bytes = 48 * 1024,
              subscription = 5;
    const int block_warps = (128 + warp_threads - 1) / warp_threads;
    const int max_warp_occ = max_sm_warps / block_warps;
    const int regs_per_side = max_sm_regs / warp_alloc_unit;
    const int regs_per_warp = ROUND_UP(regs * warp_threads, reg_alloc_unit);
    const int warps = (regs_per_side / regs_per_warp) * warp_alloc_unit;
    const int max_reg_occ = warps / block_warps;
    const int block_smem = ROUND_UP(smem, smem_alloc_unit);
    const int max_smem_occ = block_smem > 0 ? smem_bytes / block_smem : max_sm_blocks;
    const int occ = std::min(std::min(max_sm_blocks, max_warp_occ), std::min(max_smem_occ, max_reg_occ));
    return occ * sm_count * subscription;
}

// RadixSort::dispatch: passes of `radix` bits over [begin_bit, end_bit).
void dispatch(timer& T, unsigned long long* k1, unsigned long long* k2, int* v1, int* v2, int* spine, bool& swap,
              int n, int spine_size, int begin_bit, int end_bit, bool alt, int max_grid) {
    const int tile = 128 * 7;
    const int total_grains = (n + tile - 1) / tile;
    const int grid = std::min(total_grains, max_grid);
    const int grains_per_block = total_grains / grid;
    const int big_blocks = total_grains - grains_per_block * grid;
    const int normal_share = grains_per_block * tile;
    const int normal_base = big_blocks * tile;
    const int big_share = normal_share + tile;
    for (int bit = begin_bit; bit < end_bit; bit += alt ? 4 : 5) {
        unsigned long long* kin = swap ? k2 : k1;
        unsigned long long* kout = swap ? k1 : k2;
        int* vin = swap ? v2 : v1;
        int* vout = swap ? v1 : v2;
        T.run([&] { hpref_upsweep(grid, n, bit, big_blocks, big_share, normal_share, normal_base, total_grains, kin,
                                  spine, alt); });
        T.run([&] { hpref_scan(spine_size, spine); });
        T.run([&] { hpref_downsweep(grid, bit, n, big_blocks, big_share, normal_share, normal_base, total_grains,
                                    spine, kin, kout, vin, vout, alt); });
        swap = !swap;
    }
}

// RadixSort::sort over [0, bits).
void ref_sort(timer& T, unsigned long long* k1, unsigned long long* k2, int* v1, int* v2, bool& swap, int n,
              int bits, int sm_count) {
    const int max_grid = max_grid_size(sm_count);
    const int scan_tile = 1024 * 4;
    const int spine_size = max_grid * 32 + scan_tile;
    const int alt_spine_size = max_grid * 16 + scan_tile;
    int* spine = dalloc<int>(std::max(spine_size, alt_spine_size));
    swap = false;
    int begin_bit = 0;
    const int rem = bits % 5;
    if (rem != 0) {
        const int max_alt = 5 - rem;
        const int alt_end = std::min(bits, begin_bit + max_alt * 4);
        dispatch(T, k1, k2, v1, v2, spine, swap, n, alt_spine_size, begin_bit, alt_end, true, max_grid);
        begin_bit = alt_end;
    }
    dispatch(T, k1, k2, v1, v2, spine, swap, n, spine_size, begin_bit, bits, false, max_grid);
    cudaFree(spine);
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

}  // namespace

extern "C" {

// Build a BVH with the reference's kernels. method 0 = LBVH, 1 = PLOC.
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
    // The reference sort ranks keys with pre-Volta warp-synchronous scans. Its
    // buffers are padded so that a mis-rank can only land in owned memory, and
    // its output is checked to be a permutation before anything reads it.
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
    bool swap = false;
    ref_sort(T, keys0, keys1, refs0, refs1, swap, n, bits, sm);
    if (swap) {  // the reference copies buffer 1 over buffer 0
        cudaMemcpy(keys0, keys1, n * 8, cudaMemcpyDeviceToDevice);
        cudaMemcpy(refs0, refs1, n * 4, cudaMemcpyDeviceToDevice);
    }
    {
        std::vector<int> h(n), seen(n, 0);
        cudaMemcpy(h.data(), refs0, n * 4, cudaMemcpyDeviceToHost);
        for (int i = 0; i < n; ++i) {
            if (h[i] < 0 || h[i] >= n || seen[h[i]]++) {
                std::fprintf(stderr, "reference sort output is not a permutation (position %d)\n", i);
                return 3;
            }
        }
    }
    if (tap_sorted) cudaMemcpy(tap_sorted, keys0, n * 8, cudaMemcpyDeviceToDevice);
    if (tap_refs) cudaMemcpy(tap_refs, refs0, n * 4, cudaMemcpyDeviceToDevice);
    T.run([&] { hpref_setup_leaves(n, refs0, refs1, tri0, tri1, left, right, nbmin, nbmax, rbmin, rbmax); });
    int iters = 0;
    if (method == 0) {
        T.run([&] { hpref_construct60(n, parent, left, right, keys0); });
        int* counters = dalloc<int>(n);
        cudaMemset(counters, 0, n * 4);
        T.run([&] { hpref_refit(nn, counters, parent, left, right, nbmin, nbmax); });
        cudaFree(counters);
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
    }
    if (tap_parent) cudaMemcpy(tap_parent, parent, nn * 4, cudaMemcpyDeviceToDevice);
    if (tap_left) cudaMemcpy(tap_left, left, nn * 4, cudaMemcpyDeviceToDevice);
    if (tap_right) cudaMemcpy(tap_right, right, nn * 4, cudaMemcpyDeviceToDevice);
    if (tap_bmin) cudaMemcpy(tap_bmin, nbmin, nn * 16, cudaMemcpyDeviceToDevice);
    if (tap_bmax) cudaMemcpy(tap_bmax, nbmax, nn * 16, cudaMemcpyDeviceToDevice);
    ref_collapse(T, n, parent, left, right, nbmin, nbmax, tri1, tri0, nodes, ct, ci, counts);
    T.run([&] { hpref_woopify(n, tri0, tris, verts, woop); });
    cudaError_t e = cudaDeviceSynchronize();
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
