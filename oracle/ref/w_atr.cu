// ATR kernels of the reference (optimize / optimizeSmall / computeSurfaceAreas),
// built from its source tree.
#include "rt/bvh/ATRBuilderKernels.cu"
#include "hpref.h"

void hpref_atr_areas(int nodes, float* areas, float4* nbmin, float4* nbmax) {
    int b = hpref_default_block((const void*)computeSurfaceAreas);
    computeSurfaceAreas<<<(nodes + b - 1) / b, b>>>(nodes, areas, nbmin, nbmax);
}

// ATRBuilder::optimize (rt/bvh/ATRBuilder.cpp:89-104): 128-thread blocks, the
// global-matrix kernel above 20 treelet leaves.
void hpref_atr_optimize(int n, int treelet, int schedule_size, int dist_size, int gamma, float ci, float ct,
                        float* costs, float* areas, float* dist_mats, int* left, int* right, float4* nbmin,
                        float4* nbmax, int* counters, int* parent, int* subtree_refs, int* schedule, int smem) {
    const int block = 128, blocks = (n + block - 1) / block;
    if (treelet > 20)
        optimize<<<blocks, block, smem>>>(n, treelet, schedule_size, dist_size, gamma, ci, ct, costs, areas,
                                          dist_mats, left, right, nbmin, nbmax, counters, parent, subtree_refs,
                                          schedule);
    else
        optimizeSmall<<<blocks, block, smem>>>(n, treelet, schedule_size, dist_size, gamma, ci, ct, costs, areas,
                                               left, right, nbmin, nbmax, counters, parent, subtree_refs, schedule);
}
