// Stand-in for the HIP runtime header that the reference's Globals.h includes
// on the host: only the function-space qualifiers are needed by the host code
// this harness compiles (rt/bvh/BVH.h and the math types it uses), and the C
// math functions that the HIP runtime headers would have brought in.
#pragma once
#include <cmath>
#include <math.h>
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
