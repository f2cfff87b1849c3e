// fft.cuh — shared-memory Stockham FFT engine for batches of lines.
//
// A thread block holds `nlines` lines of length L in shared memory, element j
// of line b at buf[b * ld + j].  Every radix stage reads one buffer and writes
// the other (Stockham autosort, no bit reversal), so consecutive threads touch
// consecutive elements of a line.  Twiddles come from a per-length table
// tw[k] = exp(-2 pi i k / L), computed in FP64 on the host and staged in
// shared memory; the inverse transform uses conj(tw).  Transforms are
// unnormalised, like the reference's rustfft/cuFFT calls.
#pragma once

#include "common.cuh"

namespace fm {

constexpr int kMaxStages = 24;

// Radix sequence of one line length (product of radix[] == L).
struct LinePlan {
    int L;
    int nstages;
    int radix[kMaxStages];
};

// Small DFTs (forward sign -1; INV uses +1).
template <int R, bool INV, typename C>
__device__ __forceinline__ void dft_small(C (&v)[R], const C *__restrict__ tw, int L) {
    if constexpr (R == 2) {
        C a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 4) {
        C a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
        C c = cadd(v[1], v[3]), d = rot_i<INV>(csub(v[1], v[3]));
        v[0] = cadd(a, c);
        v[1] = cadd(b, d);
        v[2] = csub(a, c);
        v[3] = csub(b, d);
    } else {
        // generic odd radix: V[q] = sum_r v[r] W_R^{r q}, W_R from the length-L table
        C out[R];
        const int step = L / R;
#pragma unroll
        for (int q = 0; q < R; ++q) {
            C acc = v[0];
#pragma unroll
            for (int r = 1; r < R; ++r) {
                C w = tw[((r * q) % R) * step];
                acc = cadd(acc, INV ? cmulc(v[r], w) : cmul(v[r], w));
            }
            out[q] = acc;
        }
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = out[q];
    }
}

template <int R, bool INV, typename C>
__device__ __forceinline__ void stockham_stage(const C *__restrict__ src, C *__restrict__ dst,
                                               int L, int Ns, int nlines, int ld,
                                               const C *__restrict__ tw) {
    const int nb = L / R;
    const int total = nb * nlines;
    const int tstep = L / (Ns * R);
    for (int u = threadIdx.x; u < total; u += blockDim.x) {
        const int line = u / nb;
        const int j = u - line * nb;
        const C *s = src + line * ld;
        C *d = dst + line * ld;
        const int k = j % Ns;
        C v[R];
#pragma unroll
        for (int i = 0; i < R; ++i) v[i] = s[j + i * nb];
        if (k != 0) {
#pragma unroll
            for (int i = 1; i < R; ++i) {
                C w = tw[i * k * tstep];
                v[i] = INV ? cmulc(v[i], w) : cmul(v[i], w);
            }
        }
        dft_small<R, INV>(v, tw, L);
        const int base = (j - k) * R + k;
#pragma unroll
        for (int i = 0; i < R; ++i) d[base + i * Ns] = v[i];
    }
}

// Transform all lines; data starts in `a`, `b` is scratch of the same shape.
// Returns the buffer holding the result.  Caller must __syncthreads() after
// filling `a`; the function ends with a barrier.
template <bool INV, typename C>
__device__ C *fft_lines(C *a, C *b, const LinePlan &p, int nlines, int ld, const C *tw) {
    int Ns = 1;
    for (int s = 0; s < p.nstages; ++s) {
        const int R = p.radix[s];
        switch (R) {
            case 4: stockham_stage<4, INV>(a, b, p.L, Ns, nlines, ld, tw); break;
            case 2: stockham_stage<2, INV>(a, b, p.L, Ns, nlines, ld, tw); break;
            case 3: stockham_stage<3, INV>(a, b, p.L, Ns, nlines, ld, tw); break;
            case 5: stockham_stage<5, INV>(a, b, p.L, Ns, nlines, ld, tw); break;
            case 7: stockham_stage<7, INV>(a, b, p.L, Ns, nlines, ld, tw); break;
            default: break;  // rejected on the host
        }
        __syncthreads();
        C *t = a; a = b; b = t;
        Ns *= R;
    }
    return a;
}

}  // namespace fm
