// stage_vec.cu — the FP32-mixed path's 16-byte-group stage kernels (stage_vec.cuh).
#include <algorithm>

#include "stage_vec.cuh"
#include "stage_vec.hpp"

namespace fm {

bool stage_vec_launch(Backend &b, const StageArgs<float> &s, int mode) {
    const bool diag = s.partials != nullptr;
    const dim3 g = stage_vec_grid(b, (int)sizeof(float), diag), blk(32, kStageVecBY);
    const int zb = stage_vec_zb(b, (int)sizeof(float), diag);
    if (b.stage_vec_mk) {  // mask and / or Ms map
        switch (mode) {
            case MODE_EVAL: k_stage_vec<float, MODE_EVAL, true><<<g, blk, 0, b.stream>>>(s, zb); break;
            case MODE_HEUN_CORR: k_stage_vec<float, MODE_HEUN_CORR, true><<<g, blk, 0, b.stream>>>(s, zb); break;
            default: k_stage_vec<float, MODE_ERR_LAST, true><<<g, blk, 0, b.stream>>>(s, zb); break;
        }
        return true;
    }
    switch (mode) {
        case MODE_EVAL: k_stage_vec<float, MODE_EVAL><<<g, blk, 0, b.stream>>>(s, zb); break;
        case MODE_HEUN_CORR: k_stage_vec<float, MODE_HEUN_CORR><<<g, blk, 0, b.stream>>>(s, zb); break;
        default: k_stage_vec<float, MODE_ERR_LAST><<<g, blk, 0, b.stream>>>(s, zb); break;
    }
    return true;
}

bool combine_vec_launch(Backend &b, const CombineArgs<float> &a) {
    constexpr int V = 16 / (int)sizeof(float);
    const long long groups = b.n / V;
    const unsigned grid = (unsigned)std::max<long long>(1, std::min<long long>((groups + 255) / 256, 148LL * 16));
    k_combine_vec<float><<<grid, 256, 0, b.stream>>>(a);
    return true;
}

}  // namespace fm
