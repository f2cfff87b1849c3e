// demag_row_f64.cu — double instantiations of the fused row pass (demag_row.cuh).
#define FM_ROW_HOST
#include "demag_row.cuh"

namespace fm {

bool row_configure_f64(Backend &b) { return row_configure_t<double>(b); }
bool row_launch(Backend &b, const DemagArgs<double> &d, const StageArgs<double> &s, int mode) {
    return row_launch_t<double>(b, d, s, mode);
}

}  // namespace fm
