// demag_row_f32.cu — float instantiations of the fused row pass (demag_row.cuh).
#define FM_ROW_HOST
#include "demag_row.cuh"

namespace fm {

bool row_configure_f32(Backend &b) { return row_configure_t<float>(b); }
bool row_launch(Backend &b, const DemagArgs<float> &d, const StageArgs<float> &s, int mode) {
    return row_launch_t<float>(b, d, s, mode);
}

}  // namespace fm
