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
// Every translation unit that includes this header holds its own copy and
// fills it.
__constant__ double2 c_tw64d[64];
__constant__ float2 c_tw64f[64];
// exp(-2 pi i k / 192), k < 192, for the radix-3 stage of fft_reg3 (filled by
// the units whose kernels use lengths 3 * 2^k: upload_tw192)
__constant__ double2 c_tw192d[192];
__constant__ float2 c_tw192f[192];

template <typename C> __device__ __forceinline__ C tw64(int k);
template <> __device__ __forceinline__ double2 tw64<double2>(int k) { return c_tw64d[k]; }
template <> __device__ __forceinline__ float2 tw64<float2>(int k) { return c_tw64f[k]; }
template <typename C> __device__ __forceinline__ C tw192(int k);
template <> __device__ __forceinline__ double2 tw192<double2>(int k) { return c_tw192d[k]; }
template <> __device__ __forceinline__ float2 tw192<float2>(int k) { return c_tw192f[k]; }

template <int N> __host__ __device__ constexpr int ilog2() { return N <= 1 ? 0 : 1 + ilog2<N / 2>(); }
template <int N> __host__ __device__ constexpr bool is_pow2c() { return N >= 1 && (N & (N - 1)) == 0; }

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

// N = 3 M (M a power of two <= 16) held in one thread's registers: a radix-3
// decimation-in-frequency stage over x[j], x[j + M], x[j + 2 M] (twiddles
// W_N^{j r} from the W_192 table, compile-time indices), then fft_reg<M> on each
// third.  Output of element k = 3 k' + r at v[r M + brev<M>(k')] (perm_any).
template <int N, bool INV, typename C>
__device__ __forceinline__ void fft_reg3(C (&v)[N]) {
    constexpr int M = N / 3;
    static_assert(N == 3 * M && is_pow2c<M>() && M <= 16, "fft_reg3 size");
    using T = decltype(v[0].x);
    const T h = T(0.8660254037844386);  // sin(pi / 3)
#pragma unroll
    for (int j = 0; j < M; ++j) {
        const C a = v[j], b = v[j + M], c = v[j + 2 * M];
        const C sm = cadd(b, c), df = csub(b, c);
        C t = a;
        t.x = a.x - T(0.5) * sm.x;
        t.y = a.y - T(0.5) * sm.y;
        C u = rot_i<INV>(df);  // -i (b - c) forward, +i inverse
        u.x *= h;
        u.y *= h;
        v[j] = cadd(a, sm);
        C x1 = cadd(t, u), x2 = csub(t, u);
        if (j != 0) {
            const C w1 = tw192<C>(j * (64 / M)), w2 = tw192<C>(2 * j * (64 / M));
            x1 = INV ? cmulc(x1, w1) : cmul(x1, w1);
            x2 = INV ? cmulc(x2, w2) : cmul(x2, w2);
        }
        v[j + M] = x1;
        v[j + 2 * M] = x2;
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        C g[M];
#pragma unroll
        for (int j = 0; j < M; ++j) g[j] = v[r * M + j];
        fft_reg<M, INV>(g);
#pragma unroll
        for (int j = 0; j < M; ++j) v[r * M + j] = g[j];
    }
}

// a power of two (fft_reg) or three times one (fft_reg3), and where output k sits
template <int N, bool INV, typename C>
__device__ __forceinline__ void fft_any(C (&v)[N]) {
    if constexpr (is_pow2c<N>()) fft_reg<N, INV>(v);
    else fft_reg3<N, INV>(v);
}
template <int N> __host__ __device__ constexpr int perm_any(int k) {
    if constexpr (is_pow2c<N>()) return brev<N>(k);
    else return (k % 3) * (N / 3) + brev<N / 3>(k / 3);
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

// Sizes of the two levels for a line length L (a power of two 2..4096, or
// 3 * 2^k: 48, 96, 192, 384, 768): L1 values per thread in registers (L1 = L /
// L2, a multiple of L2), L2 threads per line.
__host__ __device__ constexpr int l2_for(int L) {
    return L <= 32 || L == 48 ? 1 : L == 96 ? 4 : L == 192 || L == 384 ? 8 : L == 768 ? 16
         : L == 64 ? 8 : L == 128 ? 8 : L == 256 ? 16 : L == 512 ? 16
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

// Host: the W_192 table of fft_reg3 (double and float copies).
inline void host_tw192(double2 (&d)[192], float2 (&f)[192]) {
    for (int k = 0; k < 192; ++k) {
        const double a = 2.0 * kPi * (double)k / 192.0;
        d[k] = make_double2(std::cos(a), -std::sin(a));
        f[k] = make_float2((float)d[k].x, (float)d[k].y);
    }
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
    fft_any<L1, INV>(v);
    if constexpr (L2 == 1) {
        if (ALIAS_OUT) __syncthreads();
#pragma unroll
        for (int k1 = 0; k1 < L1; ++k1) out(k1, v[perm_any<L1>(k1)]);
    } else {
        if (ALIAS_IN) __syncthreads();
#pragma unroll
        for (int k1 = 0; k1 < L1; ++k1) {
            C x = v[perm_any<L1>(k1)];
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
