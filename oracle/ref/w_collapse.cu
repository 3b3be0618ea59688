// BVH collapser kernels of the reference, built from its source tree
// (its device counter prefixScanOffset is renamed at compile time).
#include "rt/bvh/BVHCollapserKernels.cu"
#include "hpref.h"

static int grid_for(int threads, int block) { return (threads + block - 1) / block; }

void hpref_collapse_sizes(int nodes, int* counters, int* parent, int* left, int* right, int* sizes) {
    int b = hpref_default_block((const void*)computeSizes);
    computeSizes<<<grid_for((nodes + 1) / 2, b), b>>>(nodes, counters, parent, left, right, sizes);
}
void hpref_collapse_states(int n, float ci, float ct, int* counters, float* costs, int* parent, int* left,
                           int* right, int* sizes, int* states, float4* nbmin, float4* nbmax) {
    int b = hpref_default_block((const void*)computeNodeStatesAdaptive);
    computeNodeStatesAdaptive<<<grid_for(n, b), b>>>(n, ci, ct, counters, costs, parent, left, right, sizes,
                                                      states, (Vec4f*)nbmin, (Vec4f*)nbmax);
}
void hpref_collapse_leaf_indices(int n, int* leaf_idx, int* parent, int* states) {
    int b = hpref_default_block((const void*)computeLeafIndices);
    computeLeafIndices<<<grid_for(n, b), b>>>(n, leaf_idx, parent, states);
}
void hpref_collapse_invalidate(int n, int* counters, int* leaf_idx, int* parent, int* states) {
    int b = hpref_default_block((const void*)invalidateCollapsedNodes);
    invalidateCollapsedNodes<<<grid_for(n, b), b>>>(n, counters, leaf_idx, parent, states);
}
void hpref_collapse_offsets_begin(void) {
    int zero = 0, one = 1;
    cudaMemcpyToSymbol(leafPrefixScanOffset, &zero, sizeof(int));
    cudaMemcpyToSymbol(interiorPrefixScanOffset, &one, sizeof(int));
    cudaMemcpyToSymbol(prefixScanOffset, &zero, sizeof(int));
}
void hpref_collapse_offsets(int task_offset, int tasks, int* left, int* right, int* node_idx, int* node_off,
                            int* states) {
    int b = hpref_default_block((const void*)computeNodeOffsets);
    computeNodeOffsets<<<grid_for(tasks, b), b>>>(task_offset, tasks, left, right, node_idx, node_off, states);
}
int hpref_collapse_interiors(void) {
    int v = 0;
    cudaMemcpyFromSymbol(&v, interiorPrefixScanOffset, sizeof(int));
    return v;
}
int hpref_collapse_leaves(void) {
    int v = 0;
    cudaMemcpyFromSymbol(&v, leafPrefixScanOffset, sizeof(int));
    return v;
}
void hpref_collapse_ref_offsets(int nodes, int* states, int* sizes, int* ref_off) {
    int b = hpref_default_block((const void*)computeReferenceOffsets);
    computeReferenceOffsets<<<grid_for(nodes, b), b>>>(nodes, states, sizes, ref_off);
}
void hpref_collapse_compact(int nodes, int n_int, int* states, int* node_off, int* parent, int* left, int* right,
                            int* sizes, int* ref_off, float4* nbmin, float4* nbmax, void* out_nodes) {
    int b = hpref_default_block((const void*)compactBin);
    compactBin<<<grid_for(nodes, b), b>>>(nodes, n_int, states, node_off, parent, left, right, sizes, ref_off,
                                          (Vec4f*)nbmin, (Vec4f*)nbmax, (HipBVHNodeBin*)out_nodes);
}
void hpref_collapse_reorder(int n, int* left, int* ref_off, int* tri_in, int* tri_out, int* leaf_idx) {
    int b = hpref_default_block((const void*)reorderTriangleIndices);
    reorderTriangleIndices<<<grid_for(n, b), b>>>(n, left, ref_off, tri_in, tri_out, leaf_idx);
}
