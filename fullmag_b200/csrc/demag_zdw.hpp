// demag_zdw.hpp — the FP32 direct z convolution for 8 < nz <= 16 (demag_zdw.cuh),
// built in its own translation unit (demag_zdw_f32.cu).
#pragma once

#include "backend.hpp"
#include "demag.cuh"

namespace fm {

// Whether the wide direct z sum takes the grid: FP32, 3-D, not the fused y-z
// FFT pass, and 8 < nz <= 16, or nz = 8 with FULLMAG_FDM_ZDW=on (for tests
// against k_zd); FULLMAG_FDM_ZCONV=fft keeps the z FFT.
bool zdw_wanted(const Backend &b, bool fp32);
// Sets b.use_zdw, b.grid_zdw and b.rsm_zdw (persistent grid: resident blocks
// x SMs), and b.zdw_win / b.zdw_kyp for the window form (Ly % 128 == 0; the
// table is then uploaded with rows of zdw_kyp values; FULLMAG_FDM_ZDW=elem
// keeps the element copies).  False only on a CUDA error that leaves the
// backend unusable.
bool zdw_configure(Backend &b);
void zdw_launch(Backend &b, const DemagArgs<float> &a);

}  // namespace fm
