// Force-included into the reference's kernel sources when this harness builds
// them. The reference calls the pre-Volta warp intrinsics (__shfl, __ballot,
// ...), which no longer exist; they map here to the _sync forms over the lanes
// active at the call, which is what the unsynchronised forms meant on the GPUs
// the reference was written for. No full-warp mask is used, so a lane that has
// left a loop is never waited for.
#pragma once
#include <cuda_runtime.h>
#define __shfl(v, l) __shfl_sync(__activemask(), (v), (l))
#define __shfl_up(v, d) __shfl_up_sync(__activemask(), (v), (d))
#define __shfl_down(v, d) __shfl_down_sync(__activemask(), (v), (d))
#define __shfl_xor(v, m) __shfl_xor_sync(__activemask(), (v), (m))
#define __ballot(p) __ballot_sync(__activemask(), (p))
#define __any(p) __any_sync(__activemask(), (p))
#define __all(p) __all_sync(__activemask(), (p))
