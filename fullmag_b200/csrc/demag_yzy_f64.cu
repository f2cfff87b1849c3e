// demag_yzy_f64.cu — F64 instantiations of the fused kx-plane pass (demag_yzy.cuh).
#define FM_SCALAR_COMPLEX_ADD
#include "demag_yzy.cuh"

namespace fm {

bool yzy_configure_f64(Backend &b) { return yzy_configure_t<double>(b); }
bool yzy_launch(Backend &b, const DemagArgs<double> &a) { return yzy_launch_t<double>(b, a); }

}  // namespace fm
