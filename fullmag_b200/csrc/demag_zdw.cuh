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
//     of columns [c0, c0 + 64), warps 2-3 outputs z >= H of the same columns
//     (in the z-reversed frame, with the same code);
//   - the 64 columns' inputs (3 nz complex) and table entries (6 nz reals) are
//     copied into shared memory with cp.async by all 128 threads, double
//     buffered: the next batch's copies run while this batch is summed, and
//     both halves read one copy.
// Per output the sum runs over offsets d ascending with the table of k_zd
// (tab[c][d][kx][ky'], newell_host.hpp octant_to_z_direct) and the same packed
// FMAs; the lower half's outputs are bitwise k_zd's, the upper half's sum each
// pair of +d / -d terms in the other order.
// Shared memory: 2 buffers x 64 columns x (3 nz complex + 6 nz reals),
// 96 KiB at nz = 16 (99 KiB in the window form below): two blocks per SM.
// No TMA; plain cp.async copies.
//
// Window form (WIN, Ly a multiple of 128): the table is uploaded with its rows
// padded to kyp = KY rounded up to 4 values, and a batch of 64 columns lies in
// one kx row on one side of the ky mirror.  Its entries of one table slot are
// then one window of 68 values that starts on a 16-byte boundary (ky' from ky0,
// or from Ly - ky0 - 64 for a mirrored batch), so every copy of the batch is a
// 16-byte cp.async.cg (no L1 allocation): 12 input and 13 table copies per
// thread in place of 24 + 47 element copies.
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

constexpr int kZdwWin = 68;      // table window per slot in the window form (values)

// table values per slot in shared memory
template <bool WIN> __host__ __device__ constexpr int zdw_ts() { return WIN ? kZdwWin : kZdwCols; }
template <int NZ, bool WIN> __host__ __device__ constexpr size_t zdw_buf_bytes() {
    return (size_t)kZdwCols * 3 * NZ * sizeof(float2) + (size_t)6 * NZ * zdw_ts<WIN>() * sizeof(float);
}
template <int NZ, bool WIN> __host__ __device__ constexpr size_t zdw_smem() { return 2 * zdw_buf_bytes<NZ, WIN>(); }

// Outputs of one column: z < H = ceil(nz / 2) (rev = false), or z >= H summed
// in the z-reversed frame (rev = true).  Reversing z (z' = nz - 1 - z) maps
// offset d to -d, which flips the components odd in z (xz, yz), so the upper
// half runs the lower half's code on the inputs read in reverse order with
// those two entries negated, and stores its outputs in reverse order: one code
// path for both warps of a column (the fully unrolled sum is long enough that
// two paths compete for the instruction cache).  Per output the sum runs over
// offsets d ascending, the inputs below the output first.  si / st: the
// column's inputs and table entries in the batch buffer (slot strides
// kZdwCols and TS).
template <int NZ, int TS>
__device__ __forceinline__ void zdw_col(const float2 *si, const float *st, bool ymir, bool rev, float2 *base,
                                        int cols, bool store) {
    constexpr int H = (NZ + 1) / 2, CS = kZdwCols;
    float2 mx[NZ], my[NZ], mz[NZ];
#pragma unroll
    for (int z = 0; z < NZ; ++z) {
        const int zz = rev ? NZ - 1 - z : z;
        mx[z] = si[zz * CS];
        my[z] = si[(NZ + zz) * CS];
        const float2 v = si[(2 * NZ + zz) * CS];
        mz[z] = make_float2(v.y, -v.x);  // -i Mz
    }
    float2 hx[H], hy[H], hz[H];
#pragma unroll
    for (int j = 0; j < H; ++j) { hx[j] = make_float2(0.f, 0.f); hy[j] = hx[j]; hz[j] = hx[j]; }
    const float sy = ymir ? -1.f : 1.f, sz = rev ? -1.f : 1.f;
#pragma unroll
    for (int d = 0; d < NZ; ++d) {
        const float cxx = st[d * TS], cyy = st[(NZ + d) * TS], czz = st[(2 * NZ + d) * TS];
        const float cxy = st[(3 * NZ + d) * TS] * sy;
        const float cxz = d > 0 ? st[(4 * NZ + d) * TS] * sz : 0.f;
        const float cyz = d > 0 ? st[(5 * NZ + d) * TS] * (sy * sz) : 0.f;
#pragma unroll
        for (int o = 0; o < H; ++o) {
            if (o - d >= 0) {  // output o from input o - d (offset +d)
                const int z = o - d;
                zd_fma(hx[o], cxx, mx[z]); zd_fma(hx[o], cxy, my[z]); zd_fma(hx[o], cxz, mz[z]);
                zd_fma(hy[o], cxy, mx[z]); zd_fma(hy[o], cyy, my[z]); zd_fma(hy[o], cyz, mz[z]);
                zd_fma(hz[o], -cxz, mx[z]); zd_fma(hz[o], -cyz, my[z]); zd_fma(hz[o], czz, mz[z]);
            }
            if (d > 0 && o + d < NZ) {  // output o from input o + d (offset -d: odd-in-z entries flip)
                const int i = o + d;
                zd_fma(hx[o], cxx, mx[i]); zd_fma(hx[o], cxy, my[i]); zd_fma(hx[o], -cxz, mz[i]);
                zd_fma(hy[o], cxy, mx[i]); zd_fma(hy[o], cyy, my[i]); zd_fma(hy[o], -cyz, mz[i]);
                zd_fma(hz[o], cxz, mx[i]); zd_fma(hz[o], cyz, my[i]); zd_fma(hz[o], czz, mz[i]);
            }
        }
    }
    if (!store) return;
    const int cs = NZ * cols;
#pragma unroll
    for (int j = 0; j < H; ++j) {
        // odd nz: the reversed frame's last output is the lower half's
        if ((NZ & 1) && rev && j == H - 1) continue;
        const int o = rev ? NZ - 1 - j : j;
        base[o * cols] = hx[j];
        base[cs + o * cols] = hy[j];
        base[2 * cs + o * cols] = make_float2(-hz[j].y, hz[j].x);  // Hz = i Hz'
    }
}

template <int NZ, bool WIN>
__global__ void __launch_bounds__(kZdwThreads, 2) k_zdw(DemagArgs<float> a, int kyp) {
    constexpr int NM = 3 * NZ, NT = 6 * NZ, CS = kZdwCols, TS = zdw_ts<WIN>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x;
    // 3 NZ nkx Ly and 6 NZ nkx kyp < 2^31 for every supported grid: 32-bit offsets
    const int Ly = a.Ly, KY = a.KY, nkx = a.nkx, cols = nkx * Ly;
    const int dstr = nkx * KY, tstr = NZ * dstr;
    const int nbat = (cols + CS - 1) / CS;
    auto in_buf = [&](int buf) { return reinterpret_cast<float2 *>(smem_raw + buf * zdw_buf_bytes<NZ, WIN>()); };
    auto tab_buf = [&](int buf) { return reinterpret_cast<float *>(in_buf(buf) + NM * CS); };
    auto issue = [&](int bt, int buf) {
        const int c0 = bt * CS;
        if constexpr (WIN) {
            // Ly % 128 == 0: the batch is whole (cols % 64 == 0), in one kx row
            // and on one side of the mirror; inputs: 3 NZ slots x 32 chunks of
            // 16 bytes; table: 6 NZ slots x 17 chunks of its window
            const int kx = c0 / Ly, ky0 = c0 - kx * Ly;
            const int wstart = ky0 >= Ly / 2 ? Ly - ky0 - CS : ky0;
            float2 *di = in_buf(buf);
            for (int q = tid; q < NM * (CS / 2); q += kZdwThreads) {
                const int s = q / (CS / 2), p = q - s * (CS / 2);
                cp_async16(di + s * CS + 2 * p, a.s2 + (s * cols + c0 + 2 * p));
            }
            float *dt = tab_buf(buf);
            for (int q = tid; q < NT * (kZdwWin / 4); q += kZdwThreads) {
                const int t = q / (kZdwWin / 4), p = q - t * (kZdwWin / 4);
                cp_async16(dt + t * kZdwWin + 4 * p, a.spec + ((t * nkx + kx) * kyp + wstart + 4 * p));
            }
        } else {
            // element e = tid + 128 i has column e % 64 = tid % 64 and slot
            // e / 64 = tid / 64 + 2 i; columns past the end are left uncopied
            // (their sums are not stored)
            const int cl_copy = tid % CS, s0 = tid / CS;
            const int col = c0 + cl_copy;
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
        // the column's table entries: its own slot position, or in the window
        // form ky' - wstart (64 - cl for a mirrored batch)
        const int ti = WIN ? ((ky - cl) >= Ly / 2 ? CS - cl : cl) : cl;
        const float2 *si = in_buf(buf) + cl;
        const float *st = tab_buf(buf) + ti;
        float2 *base = a.s2 + (ok ? col : 0);
        zdw_col<NZ, TS>(si, st, ky > Ly / 2, half != 0, base, cols, ok);
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
