// demag_row.hpp — the fused x inverse / stage / x forward row pass
// (demag_row.cuh), built in its own translation units.
#pragma once

#include "backend.hpp"
#include "demag.cuh"
#include "stages.cuh"

namespace fm {

// Mode of k_row that runs its x forward alone on the rows of s.m (a state that
// no row pass produced: the first step, after an upload or after a field read),
// so that S1 gets the same bits a fused launch would give it.
constexpr int MODE_ROW_XFWD = 3;

// Sets b.use_row and the slab height b.row_rb when the plan qualifies (Heun,
// uniform material, register FFT path, Lx = 2 nx, 16-byte rows, even ny) and
// FULLMAG_FDM_ROW=on asks for it (measured slower than the split kernels);
// FULLMAG_FDM_ROW_RB forces the slab height.  False only on a CUDA error.
bool row_configure_f32(Backend &b);
bool row_configure_f64(Backend &b);
template <typename T> inline bool row_configure(Backend &b) {
    return sizeof(T) == 4 ? row_configure_f32(b) : row_configure_f64(b);
}
// One launch over all slabs: mode MODE_EVAL (RHS, diagnostics, predictor) or
// MODE_HEUN_CORR (corrector); S1 in: the convolved spectrum of s.m; out: the x
// transform of the state the stage wrote.
bool row_launch(Backend &b, const DemagArgs<float> &d, const StageArgs<float> &s, int mode);
bool row_launch(Backend &b, const DemagArgs<double> &d, const StageArgs<double> &s, int mode);

}  // namespace fm
