// batch.cuh — persistent kernels over many independent problems (the batched
// ensemble, fullmag_fdm_batch_*; no counterpart in the reference).
//
// Every stage of a step is one launch for the whole batch: the blocks walk a
// work list of (problem, block coordinates) items in grid-stride order and
// run the same block bodies as the single-problem kernels (demag_reg.cuh,
// stages.cuh) on that problem's arguments.  The padded FFT lengths differ per
// problem, so each item dispatches on its problem's length; the switch is
// uniform across the block.  Work lists, per-problem arguments and the grid
// sizes (chosen by the batch autotuner) are set up by batch.cu.
#pragma once

#include "demag_reg.cuh"
#include "stages.cuh"

namespace fm {

// x passes: item (p, bx, z, c); 256 threads, lines_x = 256 / L2 per problem;
// Lx a power of two in 16..1024, or in FP32 3 * 2^k in 96..768 (batch.cu pads
// every in-plane axis to at least 16)
template <typename T, bool INV>
__global__ void __launch_bounds__(256) k_batch_x(const DemagArgs<T> *__restrict__ A, const int4 *__restrict__ work,
                                                 int nwork) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int4 it = work[w];
        const DemagArgs<T> &a = A[it.x];
        switch (a.Lx) {
#define FM_X(L1, L2)                                                             \
    if (INV) xi_body<T, L1, L2>(a, it.y, it.z, it.w, smem_raw);                  \
    else xf_body<T, L1, L2, true>(a, it.y, it.z, it.w, smem_raw);                \
    break;
            case 16: FM_X(16, 1)
            case 32: FM_X(32, 1)
            case 64: FM_X(8, 8)
            case 96: if constexpr (sizeof(T) == 4) { FM_X(24, 4) } break;
            case 128: FM_X(16, 8)
            case 192: if constexpr (sizeof(T) == 4) { FM_X(24, 8) } break;
            case 256: FM_X(16, 16)
            case 384: if constexpr (sizeof(T) == 4) { FM_X(48, 8) } break;
            case 512: FM_X(32, 16)
            case 768: if constexpr (sizeof(T) == 4) { FM_X(48, 16) } break;
            case 1024: FM_X(32, 32)
#undef FM_X
            default: break;
        }
        __syncthreads();  // the next item refills the shared tables
    }
}

// y passes: item (p, bx); 256 threads, lines_y = 256 / L2 per problem
template <typename T, bool INV>
__global__ void __launch_bounds__(256) k_batch_y(const DemagArgs<T> *__restrict__ A, const int4 *__restrict__ work,
                                                 int nwork) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int4 it = work[w];
        const DemagArgs<T> &a = A[it.x];
        switch (a.Ly) {
#define FM_Y(L1, L2)                                                             \
    if (INV) yi_body<T, L1, L2>(a, it.y, smem_raw);                              \
    else yf_body<T, L1, L2, true>(a, it.y, smem_raw);                            \
    break;
            case 16: FM_Y(16, 1)
            case 32: FM_Y(32, 1)
            case 64: FM_Y(8, 8)
            case 96: if constexpr (sizeof(T) == 4) { FM_Y(24, 4) } break;
            case 128: FM_Y(16, 8)
            case 192: if constexpr (sizeof(T) == 4) { FM_Y(24, 8) } break;
            case 256: FM_Y(16, 16)
            case 384: if constexpr (sizeof(T) == 4) { FM_Y(48, 8) } break;
            case 512: FM_Y(32, 16)
            case 768: if constexpr (sizeof(T) == 4) { FM_Y(48, 16) } break;
            case 1024: FM_Y(32, 32)
#undef FM_Y
            default: break;
        }
        __syncthreads();
    }
}

// z convolution: item (p, chunk) of 128 column tasks; 128 threads
template <typename T>
__global__ void __launch_bounds__(128) k_batch_z(const DemagArgs<T> *__restrict__ A, const int4 *__restrict__ work,
                                                 int nwork) {
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int4 it = work[w];
        const DemagArgs<T> &a = A[it.x];
        const int tid = it.y * 128 + threadIdx.x;
        switch (a.Lz) {
            case 2: zc_task<T, 2, 1>(a, tid, 0); break;
            case 4: zc_task<T, 4, 1>(a, tid, 0); break;
            case 8: zc_task<T, 8, 1>(a, tid, 0); break;
            case 16: zc_task<T, 16, 2>(a, tid, threadIdx.x & 1); break;
            default: break;
        }
    }
}

// stage kernel: item (p, bx, by, bz), block (32, 4); zb[p] planes per thread;
// no diagnostics (the batch reports states, not per-step statistics)
template <typename T, int MODE>
__global__ void __launch_bounds__(128, 4) k_batch_stage(const StageArgs<T> *__restrict__ S,
                                                        const int *__restrict__ zb,
                                                        const int4 *__restrict__ work, int nwork) {
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int4 it = work[w];
        double acc[NQ] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // unused: no diagnostics
        stage_plain_body<T, MODE>(S[it.x], zb[it.x], it.y, it.z, it.w, acc);
    }
}

// predictor combine: item (p, chunk) of 256 cells
template <typename T>
__global__ void __launch_bounds__(256) k_batch_combine(const CombineArgs<T> *__restrict__ A,
                                                       const int4 *__restrict__ work, int nwork) {
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int4 it = work[w];
        const CombineArgs<T> &a = A[it.x];
        const long long i = (long long)it.y * 256 + threadIdx.x;
        if (i < a.n) combine_cell(a, i);
    }
}

}  // namespace fm
