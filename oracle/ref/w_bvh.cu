// HipBVH kernels of the reference (woopify, SAH cost), built from its source tree.
#include "rt/bvh/HipBVHKernels.cu"
#include "hpref.h"

void hpref_woopify(int n, int* tri_idx, const int* tris, const float* verts, float4* woop) {
    int b = hpref_default_block((const void*)woopifyTriangles);
    woopifyTriangles<<<(n + b - 1) / b, b>>>(n, tri_idx, (Vec3i*)tris, (Vec3f*)verts, (Vec4f*)woop);
}
float hpref_cost(int nodes, float scene_area, float ct, float ci, void* bin_nodes) {
    float zero = 0.0f, c = 0.0f;
    cudaMemcpyToSymbol(cost, &zero, sizeof(float));
    computeCostBin<<<(nodes + REDUCTION_BLOCK_THREADS - 1) / REDUCTION_BLOCK_THREADS, REDUCTION_BLOCK_THREADS>>>(
        nodes, scene_area, ct, ci, (HipBVHNodeBin*)bin_nodes);
    cudaMemcpyFromSymbol(&c, cost, sizeof(float));
    return c;
}
