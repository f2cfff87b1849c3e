// demag_zdw.cuh — direct z convolution for 8 < nz <= 16 in FP32 (the split
// y / z / y path of 3-D grids whose z lines are too long for one thread).
//
// k_zd (demag_reg.cuh) sums the whole column in one thread: 3 nz inputs and
// 3 nz outputs in registers, which for nz = 16 would be 192 FP32 registers of
// data alone.  Here a column is split by output half over two warps of the
// block, so each thread holds the column's 3 nz inputs and 3 ceil(nz/2)
// accumulators (96 + 48 registers at nz = 16):
//   - a block of 4 warps takes 64 consecutive columns (col = kx Ly + ky) per
//     iteration of its persistent loop; warps 0-1 sum outputs z < H = ceil(nz/2)
//     of columns [c0, c0 + 64), warps 2-3 outputs z >= H of the same columns,
//     so the half index is warp-uniform and compile-time inside each branch;
//   - the 64 columns' inputs (3 nz complex) and table entries (6 nz reals) are
//     copied into shared memory with cp.async by all 128 threads, double
//     buffered: the next batch's copies run while this batch is summed, and
//     both halves read one copy.
// Per output the sum runs over offsets d ascending, +d then -d, as in k_zd, with
// the same table (tab[c][d][kx][ky'], newell_host.hpp octant_to_z_direct) and
// the same packed FMAs, so for nz <= 8 the result is bitwise k_zd's.
// Shared memory: 2 buffers x 64 columns x (3 nz complex + 6 nz reals),
// 96 KiB at nz = 16: two blocks per SM.  No TMA; plain cp.async element copies.
#pragma once

#include <algorithm>
#include <type_traits>

#include "backend_impl.hpp"
#include "cpasync.cuh"
#include "demag.cuh"
#include "demag_reg.cuh"
#include "demag_zdw.hpp"

namespace fm {

constexpr int kZdwCols = 64;     // columns per batch
constexpr int kZdwThreads = 128; // 4 warps: 2 column groups of 32 x 2 output halves

template <int NZ> __host__ __device__ constexpr size_t zdw_buf_bytes() {
    return (size_t)kZdwCols * (3 * NZ * sizeof(float2) + 6 * NZ * sizeof(float));
}
template <int NZ> __host__ __device__ constexpr size_t zdw_smem() { return 2 * zdw_buf_bytes<NZ>(); }

// outputs o in [HH H, HH H + H) of one column; si / st: the column's inputs and
// table entries in the batch buffer (slot stride kZdwCols)
template <int NZ, int HH>
__device__ __forceinline__ void zdw_half(const float2 *si, const float *st, bool ymir, float2 *base, int cols,
                                         bool store) {
    constexpr int H = (NZ + 1) / 2, CS = kZdwCols;
    float2 mx[NZ], my[NZ], mz[NZ];
#pragma unroll
    for (int z = 0; z < NZ; ++z) {
        mx[z] = si[z * CS];
        my[z] = si[(NZ + z) * CS];
        const float2 v = si[(2 * NZ + z) * CS];
        mz[z] = make_float2(v.y, -v.x);  // -i Mz
    }
    float2 hx[H], hy[H], hz[H];
#pragma unroll
    for (int j = 0; j < H; ++j) { hx[j] = make_float2(0.f, 0.f); hy[j] = hx[j]; hz[j] = hx[j]; }
    const float sy = ymir ? -1.f : 1.f;
#pragma unroll
    for (int d = 0; d < NZ; ++d) {
        const float cxx = st[d * CS], cyy = st[(NZ + d) * CS], czz = st[(2 * NZ + d) * CS];
        const float cxy = st[(3 * NZ + d) * CS] * sy;
        const float cxz = d > 0 ? st[(4 * NZ + d) * CS] : 0.f, cyz = d > 0 ? st[(5 * NZ + d) * CS] * sy : 0.f;
#pragma unroll
        for (int j = 0; j < H; ++j) {
            const int o = HH * H + j;
            if (o >= NZ) continue;
            if (o - d >= 0) {  // output o from input o - d (offset +d)
                const int z = o - d;
                zd_fma(hx[j], cxx, mx[z]); zd_fma(hx[j], cxy, my[z]); zd_fma(hx[j], cxz, mz[z]);
                zd_fma(hy[j], cxy, mx[z]); zd_fma(hy[j], cyy, my[z]); zd_fma(hy[j], cyz, mz[z]);
                zd_fma(hz[j], -cxz, mx[z]); zd_fma(hz[j], -cyz, my[z]); zd_fma(hz[j], czz, mz[z]);
            }
            if (d > 0 && o + d < NZ) {  // output o from input o + d (offset -d: odd-in-z entries flip)
                const int i = o + d;
                zd_fma(hx[j], cxx, mx[i]); zd_fma(hx[j], cxy, my[i]); zd_fma(hx[j], -cxz, mz[i]);
                zd_fma(hy[j], cxy, mx[i]); zd_fma(hy[j], cyy, my[i]); zd_fma(hy[j], -cyz, mz[i]);
                zd_fma(hz[j], cxz, mx[i]); zd_fma(hz[j], cyz, my[i]); zd_fma(hz[j], czz, mz[i]);
            }
        }
    }
    if (!store) return;
    const int cs = NZ * cols;
#pragma unroll
    for (int j = 0; j < H; ++j) {
        const int o = HH * H + j;
        if (o >= NZ) continue;
        base[o * cols] = hx[j];
        base[cs + o * cols] = hy[j];
        base[2 * cs + o * cols] = make_float2(-hz[j].y, hz[j].x);  // Hz = i Hz'
    }
}

template <int NZ>
__global__ void __launch_bounds__(kZdwThreads, 2) k_zdw(DemagArgs<float> a) {
    constexpr int NM = 3 * NZ, NT = 6 * NZ, CS = kZdwCols;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x;
    // 3 NZ nkx Ly and 6 NZ nkx KY < 2^31 for every supported grid: 32-bit offsets
    const int Ly = a.Ly, KY = a.KY, cols = a.nkx * Ly;
    const int dstr = a.nkx * KY, tstr = NZ * dstr;
    const int nbat = (cols + CS - 1) / CS;
    auto in_buf = [&](int buf) { return reinterpret_cast<float2 *>(smem_raw + buf * zdw_buf_bytes<NZ>()); };
    auto tab_buf = [&](int buf) { return reinterpret_cast<float *>(in_buf(buf) + NM * CS); };
    // copies of batch bt: element e = tid + 128 i has column e % 64 = tid % 64 and
    // slot e / 64 = tid / 64 + 2 i; columns past the end are left uncopied (their
    // sums are not stored)
    const int cl_copy = tid % CS, s0 = tid / CS;
    auto issue = [&](int bt, int buf) {
        const int col = bt * CS + cl_copy;
        if (col >= cols) return;
        const int kx = col / Ly, ky = col - kx * Ly;
        const float2 *src = a.s2 + col;
        const unsigned di = (unsigned)__cvta_generic_to_shared(in_buf(buf) + cl_copy);
#pragma unroll
        for (int s = s0; s < NM; s += kZdwThreads / CS)
            cp_async_elem<8>(di + s * CS * (unsigned)sizeof(float2), src + s * cols);
        const float *tp = a.spec + (kx * KY + (ky > Ly / 2 ? Ly - ky : ky));
        const unsigned dt = (unsigned)__cvta_generic_to_shared(tab_buf(buf) + cl_copy);
#pragma unroll
        for (int s = s0; s < NT; s += kZdwThreads / CS) {
            const int c = s / NZ, d = s - c * NZ;
            if (c < 4 || d > 0)  // tau(0) = 0 is not read
                cp_async_elem<4>(dt + s * CS * (unsigned)sizeof(float), tp + c * tstr + d * dstr);
        }
    };
    const int warp = tid >> 5, lane = tid & 31;
    const int cl = (warp & 1) * 32 + lane, half = warp >> 1;
    int bt = blockIdx.x, buf = 0;
    if (bt < nbat) issue(bt, 0);
    cp_async_commit();
    for (; bt < nbat; bt += gridDim.x, buf ^= 1) {
        if (bt + (int)gridDim.x < nbat) issue(bt + gridDim.x, buf ^ 1);
        cp_async_commit();  // possibly empty: "all but the newest" is this batch
        cp_async_wait_all_but_one();
        __syncthreads();  // every thread's copies of this batch are visible
        const int col = bt * CS + cl;
        const bool ok = col < cols;
        const int kx = ok ? col / Ly : 0, ky = ok ? col - kx * Ly : 0;
        const float2 *si = in_buf(buf) + cl;
        const float *st = tab_buf(buf) + cl;
        float2 *base = a.s2 + (ok ? col : 0);
        if (half == 0) zdw_half<NZ, 0>(si, st, ky > Ly / 2, base, cols, ok);
        else zdw_half<NZ, 1>(si, st, ky > Ly / 2, base, cols, ok);
        __syncthreads();  // this buffer is refilled by the next iteration's copies
    }
    cp_async_wait_all();
}

template <int N> using ZdwIC = std::integral_constant<int, N>;

// nz = 11 and 13 never get here: their padded length 2 nz has a prime factor > 7
template <class F>
bool zdw_with_nz(int nz, F &&f) {
    switch (nz) {
        case 8: f(ZdwIC<8>{}); return true;
        case 9: f(ZdwIC<9>{}); return true;
        case 10: f(ZdwIC<10>{}); return true;
        case 12: f(ZdwIC<12>{}); return true;
        case 14: f(ZdwIC<14>{}); return true;
        case 15: f(ZdwIC<15>{}); return true;
        case 16: f(ZdwIC<16>{}); return true;
        default: return false;
    }
}

}  // namespace fm
