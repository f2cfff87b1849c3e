// demag_yzy.cu — FP32 fused y forward, direct z convolution and y inverse of one
// kx plane per block (3-D grids with nz <= 8 whose plane fits in shared memory).
//
// The three split kernels move the plane's y spectrum S2 through HBM three
// times (written by the y forward pass, read and written by the z sum, read
// by the y inverse pass).  Here block kx keeps its 3 nz lines of Ly complex
// values in shared memory from the y forward FFT to the y inverse FFT:
//   1. one group of L2 threads per line (c, z): forward y (fft4step, the
//      zero-padded half of the input pruned) from S1 into the line's row;
//   2. block barrier; each thread sums the direct z convolution of its ky
//      columns (the arithmetic of k_zd, in the same order, one output
//      component at a time to stay within the register budget of 3 nz x L2
//      threads), writing the column back in place;
//   3. block barrier; inverse y (fft4step) from the row back into S1, y < ny.
// Every operation and its order equal those of k_yf_r, k_zd and k_yi_r, so the
// result is bitwise the split path's.  Shared memory: 3 nz rows (rounded up to
// whole passes) of tile_elems(L1, L2) complex, each row also its line's 4-step
// tile, then the Ly twiddles.  One block per SM at Ly = 1024, nz = 8 (206 KB).
// measured at 512 x 512 x 8: 112 us with scalar complex adds, 117 us with the
// packed FP32 pair (the x passes gain from the packed form)
#define FM_SCALAR_COMPLEX_ADD
#include <cmath>
#include <cstdlib>
#include <string>
#include <type_traits>

#include "backend_impl.hpp"
#include "demag.cuh"
#include "demag_reg.cuh"
#include "demag_yzy.hpp"

namespace fm {

// Lines per pass of the FFT phases: at most 384 threads per block, so that a
// thread has the registers of a 4-step line FFT without spilling.
template <int L2, int NZ> __host__ __device__ constexpr int yzy_lines() {
    return 3 * NZ * L2 <= 384 ? 3 * NZ : 384 / L2;
}
// Rows: the 3 nz lines rounded up to whole passes (the idle line groups of a
// last, partial pass use their own rows as 4-step scratch).
template <int L2, int NZ> __host__ __device__ constexpr int yzy_rows() {
    return (3 * NZ + yzy_lines<L2, NZ>() - 1) / yzy_lines<L2, NZ>() * yzy_lines<L2, NZ>();
}
template <int L1, int L2, int NZ>
__host__ __device__ constexpr size_t yzy_smem() {
    return ((size_t)yzy_rows<L2, NZ>() * tile_elems(L1, L2) + (size_t)L1 * L2) * sizeof(cx<float>);
}
constexpr size_t kYzySmemMax = 227 * 1024;

template <int L1, int L2, int NZ>
__global__ void __launch_bounds__(yzy_lines<L2, NZ>() * L2) k_yzy(DemagArgs<float> a) {
    using T = float;
    using C = cx<T>;
    constexpr int L = L1 * L2, TE = tile_elems(L1, L2), NL = 3 * NZ, LP = yzy_lines<L2, NZ>(), BT = LP * L2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *S = reinterpret_cast<C *>(smem_raw);
    C *tws = S + yzy_rows<L2, NZ>() * TE;
    for (int k = threadIdx.x; k < L; k += BT) tws[k] = a.twyT[k];
    __syncthreads();  // fft4step reads twiddles before its first barrier
    const int kx = blockIdx.x, nkx = a.nkx, ny = a.ny;
    const int qg = threadIdx.x / L2, t = threadIdx.x - qg * L2;
    // 1. forward y, LP lines per pass: inputs y < ny (= L/2; the upper half is the
    // zero padding).  Every thread takes part in every pass (fft4step has barriers).
#pragma unroll 1
    for (int q0 = 0; q0 < NL; q0 += LP) {
        const int q = q0 + qg;  // line q = c nz + z
        const bool valid = q < NL;
        const C *line1 = a.s1 + ((long long)(valid ? q : 0) * nkx + kx) * ny;  // S1 [c][z][kx][y]
        C *row = S + q * TE;
        auto in1 = [&](int j) -> C { return valid ? line1[j] : mk<T>(0, 0); };
        auto out1 = [&](int k, C v) { row[k] = v; };
        fft4step<L1, L2, false, false, true, true>(t, tws, row, in1, out1);
    }
    __syncthreads();
    // 2. direct z convolution per ky column (table and signs as in k_zd)
    {
        const int KY = a.KY, dstr = nkx * KY, tstr = NZ * dstr;
        for (int ky = threadIdx.x; ky < L; ky += BT) {
            const bool ymir = ky > L / 2;
            const T sy = ymir ? T(-1) : T(1);
            const T *tp = a.spec + (kx * KY + (ymir ? L - ky : ky));
            C mx[NZ], my[NZ], mz[NZ];
#pragma unroll
            for (int z = 0; z < NZ; ++z) {
                mx[z] = S[z * TE + ky];
                my[z] = S[(NZ + z) * TE + ky];
                const C v = S[(2 * NZ + z) * TE + ky];
                mz[z] = mk<T>(v.y, -v.x);  // -i Mz
            }
            // output component r: coefficients (on Mx, My, Mz') of offset +d; offset -d
            // flips the entries odd in z
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                C h[NZ];
#pragma unroll
                for (int z = 0; z < NZ; ++z) h[z] = mk<T>(0, 0);
#pragma unroll
                for (int d = 0; d < NZ; ++d) {
                    const T *qd = tp + d * dstr;
                    T c0, c1, c2;  // +d row entries
                    bool odd0, odd1, odd2;  // entries odd in z (sign flip at -d)
                    if (r == 0) {
                        c0 = qd[0]; c1 = qd[3 * tstr] * sy; c2 = d > 0 ? qd[4 * tstr] : T(0);
                        odd0 = false; odd1 = false; odd2 = true;
                    } else if (r == 1) {
                        c0 = qd[3 * tstr] * sy; c1 = qd[tstr]; c2 = d > 0 ? qd[5 * tstr] * sy : T(0);
                        odd0 = false; odd1 = false; odd2 = true;
                    } else {
                        const T cxz = d > 0 ? qd[4 * tstr] : T(0), cyz = d > 0 ? qd[5 * tstr] * sy : T(0);
                        c0 = -cxz; c1 = -cyz; c2 = qd[2 * tstr];
                        odd0 = true; odd1 = true; odd2 = false;
                    }
#pragma unroll
                    for (int z = 0; z < NZ; ++z) {
                        if (z - d >= 0) {
                            zd_fma(h[z], c0, mx[z - d]); zd_fma(h[z], c1, my[z - d]); zd_fma(h[z], c2, mz[z - d]);
                        }
                        if (d > 0 && z + d < NZ) {
                            zd_fma(h[z], odd0 ? -c0 : c0, mx[z + d]);
                            zd_fma(h[z], odd1 ? -c1 : c1, my[z + d]);
                            zd_fma(h[z], odd2 ? -c2 : c2, mz[z + d]);
                        }
                    }
                }
#pragma unroll
                for (int z = 0; z < NZ; ++z)
                    S[(r * NZ + z) * TE + ky] = r == 2 ? mk<T>(-h[z].y, h[z].x) : h[z];  // Hz = i Hz'
            }
        }
    }
    __syncthreads();
    // 3. inverse y, keep y < ny
#pragma unroll 1
    for (int q0 = 0; q0 < NL; q0 += LP) {
        const int q = q0 + qg;
        const bool valid = q < NL;
        C *line1 = a.s1 + ((long long)(valid ? q : 0) * nkx + kx) * ny;
        C *row = S + q * TE;
        auto in3 = [&](int j) -> C { return row[j]; };
        auto out3 = [&](int k, C v) { if (valid && k < ny) line1[k] = v; };
        fft4step<L1, L2, true, true, false>(t, tws, row, in3, out3);
    }
}

namespace {

template <int N> using YzyIC = std::integral_constant<int, N>;

template <class F>
bool yzy_dispatch(int Ly, int nz, F &&f) {
    bool hit = false;
    auto nzs = [&](auto l1, auto l2) {
        switch (nz) {
            case 1: f(l1, l2, YzyIC<1>{}); break;
            case 2: f(l1, l2, YzyIC<2>{}); break;
            case 3: f(l1, l2, YzyIC<3>{}); break;
            case 4: f(l1, l2, YzyIC<4>{}); break;
            case 5: f(l1, l2, YzyIC<5>{}); break;
            case 6: f(l1, l2, YzyIC<6>{}); break;
            case 7: f(l1, l2, YzyIC<7>{}); break;
            case 8: f(l1, l2, YzyIC<8>{}); break;
            default: return;
        }
        hit = true;
    };
    switch (Ly) {
        case 256: nzs(YzyIC<16>{}, YzyIC<16>{}); break;
        case 512: nzs(YzyIC<32>{}, YzyIC<16>{}); break;
        case 1024: nzs(YzyIC<32>{}, YzyIC<32>{}); break;
        case 2048: nzs(YzyIC<64>{}, YzyIC<32>{}); break;
        default: break;
    }
    return hit;
}

bool yzy_upload_tw64(Backend &b) {
    double2 d[64];
    float2 f[64];
    for (int k = 0; k < 64; ++k) {
        const double ang = 2.0 * 3.14159265358979323846 * (double)k / 64.0;
        d[k] = make_double2(std::cos(ang), -std::sin(ang));
        f[k] = make_float2((float)d[k].x, (float)d[k].y);
    }
    return cuda_ok(b, cudaMemcpyToSymbol(c_tw64d, d, sizeof(d)), "twiddle64 d (yzy)") &&
           cuda_ok(b, cudaMemcpyToSymbol(c_tw64f, f, sizeof(f)), "twiddle64 f (yzy)");
}

}  // namespace

bool yzy_configure(Backend &b) {
    b.use_yzy = false;
    if (b.thin || !b.zdirect || b.Ly != 2 * b.ny || std::getenv("FULLMAG_FDM_YZY") &&
        std::string(std::getenv("FULLMAG_FDM_YZY")) == "off")
        return true;
    bool ok = true;
    yzy_dispatch(b.Ly, b.nz, [&](auto l1, auto l2, auto nzc) {
        constexpr int L1 = decltype(l1)::value, L2 = decltype(l2)::value, NZ = decltype(nzc)::value;
        constexpr size_t smem = yzy_smem<L1, L2, NZ>();
        if constexpr (smem <= kYzySmemMax) {
            if (!yzy_upload_tw64(b)) { ok = false; return; }
            if (cudaFuncSetAttribute(k_yzy<L1, L2, NZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
                cudaSuccess) {
                cudaGetLastError();
                return;  // stays on the split kernels
            }
            b.rsm_yzy = smem;
            b.use_yzy = true;
        }
    });
    return ok;
}

bool yzy_launch(Backend &b, const DemagArgs<float> &a) {
    yzy_dispatch(b.Ly, b.nz, [&](auto l1, auto l2, auto nzc) {
        constexpr int L1 = decltype(l1)::value, L2 = decltype(l2)::value, NZ = decltype(nzc)::value;
        if constexpr (yzy_smem<L1, L2, NZ>() <= kYzySmemMax)
            k_yzy<L1, L2, NZ><<<a.nkx, yzy_lines<L2, NZ>() * L2, b.rsm_yzy, b.stream>>>(a);
    });
    return true;
}

}  // namespace fm
