// PLOC builder (placeholder until the clustering kernels land).
#include <cuda_runtime.h>
#include "hp_device.cuh"
#include "hp_internal.h"

hp_status hp_ploc_build(hp_ctx* ctx, const hp_mesh* m, const hp_build_params* p, hp_bvh_impl* out,
                        const hp_build_taps* taps, cudaStream_t s) {
    (void)ctx; (void)m; (void)p; (void)out; (void)taps; (void)s;
    return hp_fail(HP_ERR_UNSUPPORTED, "PLOC builder not available in this build");
}
