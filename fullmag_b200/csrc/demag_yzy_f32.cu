// demag_yzy_f32.cu — F32 instantiations of the fused kx-plane pass (demag_yzy.cuh).
#define FM_SCALAR_COMPLEX_ADD
#include "demag_yzy.cuh"

namespace fm {

bool yzy_configure_f32(Backend &b) { return yzy_configure_t<float>(b); }
bool yzy_launch(Backend &b, const DemagArgs<float> &a) { return yzy_launch_t<float>(b, a); }

}  // namespace fm
