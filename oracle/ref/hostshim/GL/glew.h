// Empty stand-in: the reference's Globals.h includes this header on the host,
// but the host code compiled by this harness (rt/bvh/BVH.h) uses nothing from it.
#pragma once
