// Radix sort kernels of the reference, built from its source tree.
#include "radix_sort/RadixSortKernels.cu"
#include "hpref.h"

void hpref_sort_attrs(int* regs, int* smem) {
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, (const void*)downsweepKernel);
    *regs = a.numRegs;
    *smem = (int)a.sharedSizeBytes;
}
void hpref_upsweep(int grid, int n, int bit, int big_blocks, int big_share, int normal_share, int normal_base,
                   int total_grains, unsigned long long* keys, int* spine, bool alt) {
    upsweepKernel<<<grid, UPSWEEP_BLOCK_THREADS>>>(n, bit, big_blocks, big_share, normal_share, normal_base,
                                                   total_grains, keys, spine, alt);
}
void hpref_scan(int bins, int* spine) { scanKernel<<<1, SCAN_BLOCK_THREADS>>>(bins, (int4*)spine); }
void hpref_downsweep(int grid, int bit, int n, int big_blocks, int big_share, int normal_share, int normal_base,
                     int total_grains, int* spine, unsigned long long* kin, unsigned long long* kout, int* vin,
                     int* vout, bool alt) {
    downsweepKernel<<<grid, DOWNSWEEP_BLOCK_THREADS>>>(bit, n, big_blocks, big_share, normal_share, normal_base,
                                                       total_grains, spine, kin, kout, vin, vout, alt);
}
