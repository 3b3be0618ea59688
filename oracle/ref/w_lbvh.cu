// LBVH kernels of the reference, built from its source tree.
#include "rt/bvh/LBVHBuilderKernels.cu"
#include "hpref.h"

int hpref_default_block(const void* kernel) {
    int min_grid = 0, block = 0;
    cudaOccupancyMaxPotentialBlockSize(&min_grid, &block, kernel, 0, 0);
    return block > 0 ? block : 256;
}
static int grid_for(int threads, int block) { return (threads + block - 1) / block; }

void hpref_set_scene_box(const float* box6) { cudaMemcpyToSymbol(sceneBox, box6, 6 * sizeof(float)); }
void hpref_setup_boxes(int n, int* tri_idx, const int* tris, const float* verts, float4* bmin, float4* bmax) {
    int b = hpref_default_block((const void*)setupBoxes);
    setupBoxes<<<grid_for(n, b), b>>>(n, tri_idx, (Vec3i*)tris, (Vec3f*)verts, (Vec4f*)bmin, (Vec4f*)bmax);
}
void hpref_morton60(int n, int bits, unsigned long long* keys, int* refs, float4* bmin, float4* bmax) {
    int b = hpref_default_block((const void*)computeMortonCodes60);
    computeMortonCodes60<<<grid_for(n, b), b>>>(n, bits, keys, refs, (Vec4f*)bmin, (Vec4f*)bmax);
}
void hpref_setup_leaves(int n, int* refs0, int* refs1, int* tri0, int* tri1, int* left, int* right,
                        float4* nbmin, float4* nbmax, float4* bmin, float4* bmax) {
    int b = hpref_default_block((const void*)setupLeaves);
    setupLeaves<<<grid_for(n, b), b>>>(n, refs0, refs1, tri0, tri1, left, right, (Vec4f*)nbmin, (Vec4f*)nbmax,
                                       (Vec4f*)bmin, (Vec4f*)bmax);
}
void hpref_construct60(int n, int* parent, int* left, int* right, unsigned long long* keys) {
    int b = hpref_default_block((const void*)construct60);
    construct60<<<grid_for(n, b), b>>>(n, parent, left, right, keys);
}
void hpref_refit(int nodes, int* counters, int* parent, int* left, int* right, float4* nbmin, float4* nbmax) {
    int b = hpref_default_block((const void*)refit);
    int n = (nodes + 1) / 2;
    refit<<<grid_for(n, b), b>>>(nodes, counters, parent, left, right, (Vec4f*)nbmin, (Vec4f*)nbmax);
}
