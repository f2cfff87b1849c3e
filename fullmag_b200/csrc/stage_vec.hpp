// stage_vec.hpp — the uniform-material stage kernels on 16-byte cell groups
// (stage_vec.cuh), built in their own translation units.
#pragma once

#include "backend.hpp"
#include "stages.cuh"

namespace fm {

// z planes per thread of k_stage_vec (scalar bytes s): one without diagnostics;
// with them (a block reduction and its fence per block) halved from nz until the
// grid has at least 12 blocks per SM (measured at 512 x 512 x 8: RHS with
// diagnostics 58 -> 52 us at 2 planes, the corrector 37 -> 41 us, so 1 there)
inline int stage_vec_zb(const Backend &b, int s, bool diag) {
    if (!diag) return 1;
    const int V = 16 / s;
    const long long plane = (long long)((b.nx / V + 31) / 32) * ((b.ny + 3) / 4);
    int zb = b.nz > 0 ? b.nz : 1;
    while (zb > 1 && plane * ((b.nz + zb - 1) / zb) < 148LL * 12) zb = (zb + 1) / 2;
    return zb;
}
// Grid of k_stage_vec for this backend's grid and precision.
inline dim3 stage_vec_grid(const Backend &b, int s, bool diag) {
    const int V = 16 / s, zb = stage_vec_zb(b, s, diag);
    return dim3((unsigned)((b.nx / V + 31) / 32), (unsigned)((b.ny + 3) / 4), (unsigned)((b.nz + zb - 1) / zb));
}
// One launch of k_stage_vec<float, mode> (MODE_EVAL, MODE_HEUN_CORR or
// MODE_ERR_LAST) on the backend's stream: the FP32-mixed path only (the FP64
// path keeps the one-value-per-load kernels, measured faster there).
bool stage_vec_launch(Backend &b, const StageArgs<float> &s, int mode);
// One launch of k_combine_vec<float> (n a multiple of 4).
bool combine_vec_launch(Backend &b, const CombineArgs<float> &a);

}  // namespace fm
