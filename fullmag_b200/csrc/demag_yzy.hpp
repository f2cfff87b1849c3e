// demag_yzy.hpp — the fused y forward / direct z / y inverse pass per kx plane
// (demag_yzy.cu), built in its own translation unit.
#pragma once

#include "backend.hpp"
#include "demag.cuh"

namespace fm {

// Sets b.use_yzy and the cluster size b.yzy_P when the grid qualifies (3-D,
// direct z table, Ly = 2 ny in 256..2048, the plane's share fits in shared
// memory; FULLMAG_FDM_YZY=off keeps the split kernels, FULLMAG_FDM_YZY_P forces
// a cluster size, and is needed for FP64, which is slower fused).  False only on
// a CUDA error that leaves the backend unusable.
bool yzy_configure_f32(Backend &b);
bool yzy_configure_f64(Backend &b);
template <typename T> inline bool yzy_configure(Backend &b) {
    return sizeof(T) == 4 ? yzy_configure_f32(b) : yzy_configure_f64(b);
}
bool yzy_launch(Backend &b, const DemagArgs<float> &a);
bool yzy_launch(Backend &b, const DemagArgs<double> &a);

}  // namespace fm
