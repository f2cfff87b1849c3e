// demag_yz.hpp — entry points of the fused y-z convolution pass (demag_yz.cuh),
// one pair per storage precision, each built in its own translation unit.
#pragma once

#include "backend.hpp"
#include "demag.cuh"

namespace fm {

bool yz_configure_f32(Backend &b);
bool yz_configure_f64(Backend &b);
bool yz_launch_f32(Backend &b, const DemagArgs<float> &a);
bool yz_launch_f64(Backend &b, const DemagArgs<double> &a);

template <typename T> inline bool yz_configure(Backend &b) {
    return sizeof(T) == 4 ? yz_configure_f32(b) : yz_configure_f64(b);
}
inline bool yz_launch(Backend &b, const DemagArgs<float> &a) { return yz_launch_f32(b, a); }
inline bool yz_launch(Backend &b, const DemagArgs<double> &a) { return yz_launch_f64(b, a); }

}  // namespace fm
