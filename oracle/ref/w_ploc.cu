// PLOC kernels of the reference, built from its source tree
// (its device counter prefixScanOffset is renamed at compile time).
#include "rt/bvh/PLOCBuilderKernels.cu"
#include "hpref.h"

static int grid_for(int threads, int block) { return (threads + block - 1) / block; }

void hpref_ploc_neighbours(int clusters, int r, float* dist, int* nbr, float4* nbmin, float4* nbmax, int* nodes) {
    if (r <= PLOC_GEN_BLOCK_THREADS / 2)
        generateNeighboursCached<<<grid_for(clusters, PLOC_GEN_BLOCK_THREADS), PLOC_GEN_BLOCK_THREADS>>>(
            clusters, r, dist, nbr, (Vec4f*)nbmin, (Vec4f*)nbmax, nodes);
    else
        generateNeighbours<<<grid_for(clusters, PLOC_GEN_BLOCK_THREADS), PLOC_GEN_BLOCK_THREADS>>>(
            clusters, r, dist, nbr, (Vec4f*)nbmin, (Vec4f*)nbmax, nodes);
}
void hpref_ploc_reset(void) {
    int z = 0;
    cudaMemcpyToSymbol(prefixScanOffset, &z, sizeof(int));
}
void hpref_ploc_merge(int clusters, int offset, int* nbr, int* in, int* out, int* parent, int* left, int* right,
                      float4* nbmin, float4* nbmax) {
    int b = hpref_default_block((const void*)merge);
    merge<<<grid_for(clusters, b), b>>>(clusters, offset, nbr, in, out, parent, left, right, (Vec4f*)nbmin,
                                        (Vec4f*)nbmax);
}
int hpref_ploc_merged(void) {
    int v = 0;
    cudaMemcpyFromSymbol(&v, prefixScanOffset, sizeof(int));
    return v;
}
void hpref_ploc_scan_compact(int clusters, int* in, int* out, int* thread_offsets, int* block_offsets) {
    int blocks = (clusters + PLOC_SCAN_BLOCK_THREADS - 1) / PLOC_SCAN_BLOCK_THREADS;
    localPrefixScan<<<blocks, PLOC_SCAN_BLOCK_THREADS>>>(clusters, in, thread_offsets, block_offsets);
    globalPrefixScan<<<1, PLOC_SCAN_BLOCK_THREADS>>>(blocks, block_offsets);
    compact<<<blocks, PLOC_SCAN_BLOCK_THREADS>>>(clusters, in, out, block_offsets, thread_offsets);
}
