// demag_yzy.hpp — the FP32 fused y forward / direct z / y inverse pass per kx
// plane (demag_yzy.cu), built in its own translation unit.
#pragma once

#include "backend.hpp"
#include "demag.cuh"

namespace fm {

// Sets b.use_yzy when the grid qualifies (3-D, direct z, FP32 caller, the plane
// fits in shared memory; FULLMAG_FDM_YZY=off keeps the split kernels).  False
// only on a CUDA error that leaves the backend unusable.
bool yzy_configure(Backend &b);
bool yzy_launch(Backend &b, const DemagArgs<float> &a);

}  // namespace fm
