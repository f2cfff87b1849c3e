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

// Direct z sum of one column (col = kx Ly + ky) with the table of
// octant_to_z_direct: the arithmetic of k_zd in the same order per output,
// inputs and table entries read straight from global memory.
template <typename T, int NZ>
__device__ __forceinline__ void zd_col(const DemagArgs<T> &a, int col) {
    using C = cx<T>;
    const int Ly = a.Ly, KY = a.KY, cols = a.nkx * Ly;
    if (col >= cols) return;
    const int cs = NZ * cols, dstr = a.nkx * KY, tstr = NZ * dstr;
    const int kx = col / Ly, ky = col - kx * Ly;
    const bool ymir = ky > Ly / 2;
    const T sy = ymir ? T(-1) : T(1);
    const T *tp = a.spec + (kx * KY + (ymir ? Ly - ky : ky));
    C *base = a.s2 + col;
    C mx[NZ], my[NZ], mz[NZ], hx[NZ], hy[NZ], hz[NZ];
#pragma unroll
    for (int z = 0; z < NZ; ++z) {
        mx[z] = base[z * cols];
        my[z] = base[cs + z * cols];
        const C v = base[2 * cs + z * cols];
        mz[z] = mk<T>(v.y, -v.x);  // -i Mz
        hx[z] = mk<T>(0, 0); hy[z] = mk<T>(0, 0); hz[z] = mk<T>(0, 0);
    }
#pragma unroll
    for (int d = 0; d < NZ; ++d) {
        const T *qd = tp + d * dstr;
        const T cxx = qd[0], cyy = qd[tstr], czz = qd[2 * tstr], cxy = qd[3 * tstr] * sy;
        const T cxz = d > 0 ? qd[4 * tstr] : T(0), cyz = d > 0 ? qd[5 * tstr] * sy : T(0);
#pragma unroll
        for (int z = 0; z + d < NZ; ++z) {
            {   // output z + d from input z (offset +d)
                const int o = z + d;
                zd_fma(hx[o], cxx, mx[z]); zd_fma(hx[o], cxy, my[z]); zd_fma(hx[o], cxz, mz[z]);
                zd_fma(hy[o], cxy, mx[z]); zd_fma(hy[o], cyy, my[z]); zd_fma(hy[o], cyz, mz[z]);
                zd_fma(hz[o], -cxz, mx[z]); zd_fma(hz[o], -cyz, my[z]); zd_fma(hz[o], czz, mz[z]);
            }
            if (d > 0) {  // output z from input z + d (offset -d: odd-in-z entries flip)
                const int i = z + d;
                zd_fma(hx[z], cxx, mx[i]); zd_fma(hx[z], cxy, my[i]); zd_fma(hx[z], -cxz, mz[i]);
                zd_fma(hy[z], cxy, mx[i]); zd_fma(hy[z], cyy, my[i]); zd_fma(hy[z], -cyz, mz[i]);
                zd_fma(hz[z], cxz, mx[i]); zd_fma(hz[z], cyz, my[i]); zd_fma(hz[z], czz, mz[i]);
            }
        }
    }
#pragma unroll
    for (int z = 0; z < NZ; ++z) {
        base[z * cols] = hx[z];
        base[cs + z * cols] = hy[z];
        base[2 * cs + z * cols] = mk<T>(-hz[z].y, hz[z].x);  // Hz = i Hz'
    }
}

// z convolution: item (p, chunk) of 128 column tasks; 128 threads.  DIRECT: the
// direct sum per column for nz <= NZMAX (the kernel's registers are those of
// its largest case, so batches whose problems all have nz <= 4 take NZMAX = 4),
// else the z FFT pass (zc_task; with Lz = 16 a thread pair per column)
template <typename T, bool DIRECT, int NZMAX = 8>
__global__ void __launch_bounds__(128) k_batch_z(const DemagArgs<T> *__restrict__ A, const int4 *__restrict__ work,
                                                 int nwork) {
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int4 it = work[w];
        const DemagArgs<T> &a = A[it.x];
        const int tid = it.y * 128 + threadIdx.x;
        if constexpr (DIRECT) {
            switch (a.nz) {
                case 1: zd_col<T, 1>(a, tid); break;
                case 2: zd_col<T, 2>(a, tid); break;
                case 3: zd_col<T, 3>(a, tid); break;
                case 4: zd_col<T, 4>(a, tid); break;
                default:
                    if constexpr (NZMAX > 4) {
                        switch (a.nz) {
                            case 5: zd_col<T, 5>(a, tid); break;
                            case 6: zd_col<T, 6>(a, tid); break;
                            case 7: zd_col<T, 7>(a, tid); break;
                            case 8: zd_col<T, 8>(a, tid); break;
                            default: break;
                        }
                    }
                    break;
            }
        } else {
            switch (a.Lz) {
                case 2: zc_task<T, 2, 1>(a, tid, 0); break;
                case 4: zc_task<T, 4, 1>(a, tid, 0); break;
                case 8: zc_task<T, 8, 1>(a, tid, 0); break;
                case 16: zc_task<T, 16, 2>(a, tid, threadIdx.x & 1); break;
                default: break;
            }
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
