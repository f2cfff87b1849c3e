// demag_yz_f64.cu — FP64 instantiations of the fused y-z pass.
#include "demag_yz.cuh"

namespace fm {

bool yz_configure_f64(Backend &b) { return yz_configure_t<double>(b); }
bool yz_launch_f64(Backend &b, const DemagArgs<double> &a) { return yz_launch_t<double>(b, a); }

}  // namespace fm
