// fftreg.cuh — register-resident FFTs and the two-level (4-step) line FFT.
//
// fft_reg<N>: an N-point FFT (N <= 64, power of two) held entirely in one
// thread's registers, radix-2 decimation in frequency, fully unrolled so every
// index and twiddle is a compile-time constant; the output of element k sits
// at v[brev<N>(k)].  Twiddles come from a 64-entry constant table of
// exp(-2 pi i k / 64) (filled in FP64 on the host), read with compile-time
// indices, i.e. as constant-bank operands.
//
// fft4step<L1, L2>: one line of length L = L1 * L2 handled by L2 threads.
// Thread t loads x[t + L2 i] (i < L1), runs fft_reg<L1>, multiplies by
// W_L^{t k1}, and writes the L1 results to a padded shared-memory tile; after a
// barrier every thread gathers L1/L2 columns of L2 values, runs fft_reg<L2> on
// each and emits X[k1 + L1 k2].  One shared-memory round trip per line
// replaces the log4(L) passes of a shared-memory Stockham FFT, and both the
// loads (consecutive t -> consecutive j) and the stores (consecutive t ->
// consecutive k1) are coalesced.
#pragma once

#include <cmath>
#include <vector>

#include "common.cuh"

namespace fm {

// exp(-2 pi i k / 64), k < 64, filled per device by the host (upload_tw64).
// Defined here: one translation unit (backend.cu) includes this header.
__constant__ double2 c_tw64d[64];
__constant__ float2 c_tw64f[64];

template <typename C> __device__ __forceinline__ C tw64(int k);
template <> __device__ __forceinline__ double2 tw64<double2>(int k) { return c_tw64d[k]; }
template <> __device__ __forceinline__ float2 tw64<float2>(int k) { return c_tw64f[k]; }

template <int N> __host__ __device__ constexpr int ilog2() { return N <= 1 ? 0 : 1 + ilog2<N / 2>(); }

template <int N> __host__ __device__ constexpr int brev(int k) {
    int r = 0;
    for (int b = 0; b < ilog2<N>(); ++b) r |= ((k >> b) & 1) << (ilog2<N>() - 1 - b);
    return r;
}

// v <- v * W_64^idx (forward) or conj (inverse).  idx is a constant after the
// callers' loops are unrolled, so the branches fold and the table read is a
// constant-bank operand.
template <bool INV, typename C>
__device__ __forceinline__ C twiddle_c(C v, int idx) {
    if (idx == 0) return v;
    if (idx == 16) return rot_i<INV>(v);                  // W_64^16 = -i
    if (idx == 32) { C r; r.x = -v.x; r.y = -v.y; return r; }
    if (idx == 48) return rot_i<!INV>(v);                 // W_64^48 = +i
    const C w = tw64<C>(idx);
    return INV ? cmulc(v, w) : cmul(v, w);
}

template <int N, bool INV, typename C>
__device__ __forceinline__ void fft_reg(C (&v)[N]) {
    static_assert(N >= 1 && N <= 64 && (N & (N - 1)) == 0, "fft_reg size");
#pragma unroll
    for (int s = N / 2; s >= 1; s /= 2) {
#pragma unroll
        for (int g = 0; g < N; g += 2 * s) {
#pragma unroll
            for (int j = 0; j < s; ++j) {
                const C a = v[g + j], b = v[g + j + s];
                v[g + j] = cadd(a, b);
                // W_{2s}^j = W_64^{j * 32 / s}
                v[g + j + s] = twiddle_c<INV>(csub(a, b), j * (32 / s));
            }
        }
    }
}

// Inverse (or forward) FFT of bit-reversed-ordered input, natural-order
// output: radix-2 decimation in time, the transpose of fft_reg's network.
// Lets a caller go forward with fft_reg, work on the spectrum where it lies
// (position p holds frequency brev(p)) and come back without reordering.
template <int N, bool INV, typename C>
__device__ __forceinline__ void fft_reg_dit(C (&v)[N]) {
    static_assert(N >= 1 && N <= 64 && (N & (N - 1)) == 0, "fft_reg_dit size");
#pragma unroll
    for (int s = 1; s < N; s *= 2) {
#pragma unroll
        for (int g = 0; g < N; g += 2 * s) {
#pragma unroll
            for (int j = 0; j < s; ++j) {
                const C a = v[g + j];
                const C b = twiddle_c<INV>(v[g + j + s], j * (32 / s));
                v[g + j] = cadd(a, b);
                v[g + j + s] = csub(a, b);
            }
        }
    }
}

// Sizes of the two levels for a line length L (power of two, 2..4096):
// L1 values per thread in registers, L2 threads per line.
__host__ __device__ constexpr int l2_for(int L) {
    return L <= 32 ? 1 : L == 64 ? 8 : L == 128 ? 8 : L == 256 ? 16 : L == 512 ? 16
         : L == 1024 ? 32 : L == 2048 ? 32 : 64;
}

// Shared-memory tile (complex elements) one line needs for its transpose.
__host__ __device__ constexpr int tile_elems(int L1, int L2) { return L2 == 1 ? 0 : L1 * (L2 + 1); }

// The inter-level twiddles W_L^{t k1} in the order fft4step reads them,
// twT[k1 L2 + t]: the L2 threads of a line read consecutive words for each k1,
// where a plain W_L^k table read at t k1 puts the threads 2 t k1 banks apart
// (up to 16-way conflicts).  g[k] = W_{L stride}^k, so g[stride k] = W_L^k.
template <int L1, int L2, typename C>
__device__ __forceinline__ void fill_tw4(C *twT, const C *__restrict__ g, int stride) {
    for (int idx = threadIdx.x; idx < L1 * L2; idx += blockDim.x) {
        const int k1 = idx / L2, t = idx - k1 * L2;
        twT[idx] = g[stride * k1 * t];
    }
}

// Host: the same table for a power-of-two length L split as l2_for(L), each
// entry computed exactly like the plain table exp(-2 pi i k / L) at k = k1 t.
template <typename T>
inline std::vector<cx<T>> host_tw4(int L) {
    const int L2 = l2_for(L);
    std::vector<cx<T>> t(L);
    for (int idx = 0; idx < L; ++idx) {
        const int k = (idx / L2) * (idx % L2);
        const double a = 2.0 * kPi * (double)k / (double)L;
        t[idx] = mk<T>((T)std::cos(a), (T)(-std::sin(a)));
    }
    return t;
}

// One line, L2 threads; t = thread index within the line group.
//   in(j)        -> C   for j = t + L2 * i
//   out(k, v)           for k = k1 + L1 * k2 (this thread's k1 = t + L2 * r)
// tw: the table of fill_tw4 (shared memory); tile: this line's
// scratch (tile_elems); ALIAS_IN: the inputs live in memory the tile overlaps
// (barrier before the tile is written); ALIAS_OUT: out() writes memory the
// tile overlaps (barrier before the outputs are written).  All threads of the
// block must call this the same number of times (it contains barriers).
// HALF_IN: inputs j >= L/2 are known zero (zero padding); since j = t + L2 i
// with t < L2, that is exactly i >= L1/2, so those registers are constant zero
// and the first radix-2 stage of fft_reg folds away.
template <int L1, int L2, bool INV, bool ALIAS_IN, bool ALIAS_OUT, bool HALF_IN = false, typename C,
          class In, class Out>
__device__ __forceinline__ void fft4step(int t, const C *__restrict__ tw, C *tile, In in, Out out) {
    constexpr int L = L1 * L2;
    C v[L1];
#pragma unroll
    for (int i = 0; i < L1; ++i) {
        if (HALF_IN && i >= L1 / 2) { v[i].x = 0; v[i].y = 0; }
        else v[i] = in(t + L2 * i);
    }
    fft_reg<L1, INV>(v);
    if constexpr (L2 == 1) {
        if (ALIAS_OUT) __syncthreads();
#pragma unroll
        for (int k1 = 0; k1 < L1; ++k1) out(k1, v[brev<L1>(k1)]);
    } else {
        if (ALIAS_IN) __syncthreads();
#pragma unroll
        for (int k1 = 0; k1 < L1; ++k1) {
            C x = v[brev<L1>(k1)];
            if (k1 != 0 && t != 0) {
                const C w = tw[k1 * L2 + t];
                x = INV ? cmulc(x, w) : cmul(x, w);
            }
            tile[k1 * (L2 + 1) + t] = x;
        }
        __syncthreads();
        constexpr int R = L1 / L2;
        C u[R][L2];
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
            for (int s = 0; s < L2; ++s) u[r][s] = tile[(t + L2 * r) * (L2 + 1) + s];
        if (ALIAS_OUT) __syncthreads();
#pragma unroll
        for (int r = 0; r < R; ++r) {
            fft_reg<L2, INV>(u[r]);
#pragma unroll
            for (int k2 = 0; k2 < L2; ++k2) out(t + L2 * r + L1 * k2, u[r][brev<L2>(k2)]);
        }
    }
    (void)L;
}

}  // namespace fm
