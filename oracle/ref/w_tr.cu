// TRBVH kernels of the reference (optimize / computeSurfaceAreas), built from
// its source tree. Their extern "C" names are those of the ATR kernels, so the
// Makefile renames them for this translation unit.
#include "rt/bvh/TRBuilderKernels.cu"
#include "hpref.h"

void hpref_tr_areas(int nodes, float* areas, float4* nbmin, float4* nbmax) {
    int b = hpref_default_block((const void*)computeSurfaceAreas);
    computeSurfaceAreas<<<(nodes + b - 1) / b, b>>>(nodes, areas, nbmin, nbmax);
}

// TRBuilder::optimize (rt/bvh/TRBuilder.cpp:137-205): 128-thread blocks over
// the references, the treelet arrays in dynamic shared memory.
void hpref_tr_optimize(int n, int rounds, int treelet, int gamma, float ci, float ct, float* costs, float* areas,
                       int* left, int* right, float4* nbmin, float4* nbmax, int* counters, int* parent,
                       int* subtree_refs, float* subset_areas, float4* subset_min, float4* subset_max, int* schedule,
                       int* current_internal, int* stack_node, int* stack_size, char* stack_mask) {
    const int block = 128, blocks = (n + block - 1) / block;
    const int treelet_mem = (2 * treelet - 1) * 4 + treelet * 4;
    const int cost_mask = (1 << treelet) * 4 + (1 << treelet);
    const int smem = (treelet_mem + cost_mask) * (block / 32);
    optimize<<<blocks, block, smem>>>(n, rounds, treelet, gamma, ci, ct, costs, areas, left, right, nbmin, nbmax,
                                      counters, parent, subtree_refs, subset_areas, subset_min, subset_max, schedule,
                                      current_internal, stack_node, stack_size, stack_mask);
}
