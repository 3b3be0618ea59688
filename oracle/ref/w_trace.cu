// The reference's binary-BVH tracer (patched copy, see prepare.sh).
#include "tracer/HipTracerBinKernels.cu"
#include "hpref.h"

// HipTracer::trace (rt/tracer/HipTracer.cpp:13-52): reset the warp counter,
// query the kernel's configuration, launch desiredWarps warps of blockWidth x blockHeight.
void hpref_trace_launch(int rays, bool any_hit, float4* rays_buf, int4* results, float4* nodes, float4* tris,
                        int2* stats, int* tri_idx) {
    int zero = 0;
    cudaMemcpyToSymbol(g_warpCounter, &zero, sizeof(int));
    queryConfig<<<1, 1>>>();
    KernelConfig c;
    cudaMemcpyFromSymbol(&c, g_config, sizeof(c));
    dim3 block(c.blockWidth, c.blockHeight);
    int block_warps = (c.blockWidth * c.blockHeight + 31) / 32;
    int blocks = (c.desiredWarps + block_warps - 1) / block_warps;
    trace<<<blocks, block>>>(rays, any_hit, rays_buf, results, nodes, tris, stats, nullptr, tri_idx);
}
