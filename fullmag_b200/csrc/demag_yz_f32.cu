// demag_yz_f32.cu — FP32 instantiations of the fused y-z pass.
#include "demag_yz.cuh"

namespace fm {

bool yz_configure_f32(Backend &b) { return yz_configure_t<float>(b); }
bool yz_launch_f32(Backend &b, const DemagArgs<float> &a) { return yz_launch_t<float>(b, a); }

}  // namespace fm
