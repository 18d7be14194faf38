// Stand-in for KittenEngine/KittenGpuLBVH/lbvh.cuh, which the reference includes
// (YarnBall.h:11) but does not ship (an empty, un-vendored submodule directory).  Test
// infrastructure for the recipe that compiles the reference's simulator kernels.
//
// Only the interface is declared: the kernels are built device-only, and the host harness
// (oracle/refbuild/ref_host.cpp) answers the simulator's BVH query (collision.cu:101-111) with
// the brute-force overlapping-box pair kernel refk_pairs of ref_device.cu, which writes every
// pair of overlapping boxes once as (lower index, higher index).  The contact set after the
// simulator's own narrow-phase filter is the same as with any exact overlap query.
#pragma once
#include <cuda_runtime.h>

#include "KittenEngine/includes/modules/Bound.h"

namespace Kitten {
class LBVH {
   public:
    typedef Bound<3, float> aabb;
    aabb bounds();
    void compute(aabb* devicePtr, size_t size);
    void refit();
    size_t query(ivec2* d_res, size_t resSize);
};
}  // namespace Kitten
