// HLBVH kernels of the reference (rt/bvh/HLBVHBuilderKernels.cu), built from
// its source tree. Their extern "C" names that other kernel files also use
// (computeNodeStates, computeNodeOffsets, compact, ...) and the device counter
// prefixScanOffset are renamed at compile time (oracle/ref/Makefile).
#include "rt/bvh/HLBVHBuilderKernels.cu"
#include "hpref.h"

static int grid_for(int threads, int block) { return (threads + block - 1) / block; }

void hpref_hl_node_states(int n, int bits, int sah, int* counters, int* parent, int* left, int* right, int* states,
                          unsigned long long* keys) {
    int b = hpref_default_block((const void*)computeNodeStates);
    computeNodeStates<<<grid_for(n, b), b>>>(n, bits, sah, counters, parent, left, right, states, keys);
}
void hpref_hl_leaf_clusters(int n, int* leaf_cluster, int* parent, int* states) {
    int b = hpref_default_block((const void*)computeLeafClusterIndices);
    computeLeafClusterIndices<<<grid_for(n, b), b>>>(n, leaf_cluster, parent, states);
}
void hpref_hl_invalidate(int n, int* counters, int* leaf_cluster, int* parent, int* states) {
    int b = hpref_default_block((const void*)invalidateIntermediateClusters);
    invalidateIntermediateClusters<<<grid_for(n, b), b>>>(n, counters, leaf_cluster, parent, states);
}
void hpref_hl_set_counter(int v) { cudaMemcpyToSymbol(prefixScanOffset, &v, sizeof(int)); }
int hpref_hl_counter(void) {
    int v = 0;
    cudaMemcpyFromSymbol(&v, prefixScanOffset, sizeof(int));
    return v;
}
void hpref_hl_node_offsets(int n, int* offsets, int* states) {
    int b = hpref_default_block((const void*)computeNodeOffsets);
    computeNodeOffsets<<<grid_for(n - 1, b), b>>>(n, offsets, states);
}
void hpref_hl_compact(int n, int* offsets, int* states, int* in_parent, int* in_left, int* in_right, int* out_parent,
                      int* out_left, int* out_right) {
    int b = hpref_default_block((const void*)compact);
    compact<<<grid_for(2 * n - 1, b), b>>>(2 * n - 1, offsets, states, in_parent, in_left, in_right, out_parent,
                                           out_left, out_right);
}
void hpref_hl_clusters(int n, int bits, int sah, int* states, int* offsets, int* lbvh_left, int* cluster_nodes,
                       int4* cluster_bins, unsigned long long* keys) {
    int b = hpref_default_block((const void*)computeClusters);
    computeClusters<<<grid_for(2 * n - 1, b), b>>>(2 * n - 1, bits, sah, states, offsets, lbvh_left, cluster_nodes,
                                                   (Vec4i*)cluster_bins, keys);
}
void hpref_hl_reset_bins(int all_bins, float4* bmin, float4* bmax) {
    int b = hpref_default_block((const void*)resetBins);
    resetBins<<<grid_for(all_bins, b), b>>>(all_bins, (Vec4f*)bmin, (Vec4f*)bmax);
}
void hpref_hl_bin(int tasks, int bins, int clusters, int* cluster_tasks, int* cluster_nodes, int4* cluster_bins,
                  float4* nbmin, float4* nbmax, float4* bmin, float4* bmax) {
    int b = hpref_default_block((const void*)binClusters);
    binClusters<<<grid_for(clusters, b), b>>>(tasks, bins, clusters, cluster_tasks, cluster_nodes,
                                              (Vec4i*)cluster_bins, (Vec4f*)nbmin, (Vec4f*)nbmax, (Vec4f*)bmin,
                                              (Vec4f*)bmax);
}
// HipKernel launches whole blocks; the kernel rounds the task count up to whole
// warps itself, which the block size (a multiple of 32) covers.
void hpref_hl_split(int bins, int tasks, int* out_size, int* new_tasks, int* split_idx, int* parent, int* left,
                    int* right, float4* nbmin, float4* nbmax, float4* bmin, float4* bmax, int2* in_q, int2* out_q) {
    int b = hpref_default_block((const void*)split);
    split<<<grid_for(tasks, b), b>>>(bins, tasks, out_size, new_tasks, split_idx, parent, left, right, (Vec4f*)nbmin,
                                     (Vec4f*)nbmax, (Vec4f*)bmin, (Vec4f*)bmax, (HLBVHTask*)in_q,
                                     (HLBVHTask*)out_q);
}
void hpref_hl_distribute(int tasks, int bins, int clusters, int* new_tasks, int* split_idx, int* parent, int* left,
                         int* right, int* cluster_tasks, int* cluster_nodes, int4* cluster_bins, float4* bmin,
                         float4* bmax, int2* in_q) {
    int b = hpref_default_block((const void*)distributeClusters);
    distributeClusters<<<grid_for(clusters, b), b>>>(tasks, bins, clusters, new_tasks, split_idx, parent, left,
                                                     right, cluster_tasks, cluster_nodes, (Vec4i*)cluster_bins,
                                                     (Vec4f*)bmin, (Vec4f*)bmax, (HLBVHTask*)in_q);
}
