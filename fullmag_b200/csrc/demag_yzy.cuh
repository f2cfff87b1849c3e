// demag_yzy.cuh — fused y forward, direct z convolution and y inverse of one kx
// plane per cluster of P CTAs (3-D grids with nz <= 8, direct z table).
//
// The three split kernels move the plane's y spectrum S2 through HBM three
// times (written by the y forward pass, read and written by the z sum, read
// by the y inverse pass).  Here the 3 nz lines (c, z) of plane kx stay in the
// shared memory of one thread-block cluster from the y forward FFT to the y
// inverse FFT.  CTA h of the cluster owns lines [h NLH, (h + 1) NLH):
//   1. one group of L2 threads per owned line: forward y (fft4step, the
//      zero-padded half of the input pruned) from S1 into the line's row;
//   2. cluster barrier; CTA h sums the direct z convolution of the ky columns
//      [h Ly/P, (h + 1) Ly/P), reading each column's 3 nz values from the
//      owners' rows (distributed shared memory for the other CTAs' lines) and
//      writing the results back there (k_zd's loop, all three components at once;
//      one component at a time measured 104.6 against 99.4 us at 512 x 512 x 8);
//   3. cluster barrier; inverse y (fft4step) from the owned rows back into S1,
//      keeping y < ny.
// The sums are those of k_zd, in the same order per output, and the FFTs are
// those of k_yf_r and k_yi_r, so the result is bitwise the split path's.
// Shared memory per CTA: NLH rows of tile_elems(L1, L2) complex (a row is also
// its line's 4-step tile), then the Ly twiddles.  P = 1 is one CTA per plane.
// No TMA; the remote rows are read and written with plain loads and stores.
//
// Measured at 512 x 512 x 8 (FP32, P = 1): 112 us with scalar complex adds,
// 117 us with the packed FP32 pair, so the units that include this header
// define FM_SCALAR_COMPLEX_ADD first.  One unit per precision
// (demag_yzy_f32.cu, demag_yzy_f64.cu), so that they compile in parallel.
#pragma once
#include <cooperative_groups.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <type_traits>

#include "backend_impl.hpp"
#include "demag.cuh"
#include "demag_reg.cuh"
#include "demag_yzy.hpp"

namespace cg = cooperative_groups;

namespace fm {

// lines owned by one CTA of a P-CTA cluster
template <int NZ, int P> __host__ __device__ constexpr int yzy_nlh() { return (3 * NZ + P - 1) / P; }
// lines per FFT pass: FP32 CTAs of at most 192 threads (168 registers each, so
// that two CTAs of 107 KB fit per SM), FP64 at most 384
template <typename T, int L2, int NZ, int P> __host__ __device__ constexpr int yzy_lpp() {
    return yzy_nlh<NZ, P>() * L2 <= (sizeof(T) == 4 ? 192 : 384) ? yzy_nlh<NZ, P>() : (sizeof(T) == 4 ? 192 : 384) / L2;
}
// rows: the owned lines rounded up to whole passes (the idle line groups of a
// last, partial pass use their own rows as 4-step scratch)
template <typename T, int L2, int NZ, int P> __host__ __device__ constexpr int yzy_rows() {
    return (yzy_nlh<NZ, P>() + yzy_lpp<T, L2, NZ, P>() - 1) / yzy_lpp<T, L2, NZ, P>() * yzy_lpp<T, L2, NZ, P>();
}
template <typename T, int L1, int L2, int NZ, int P>
__host__ __device__ constexpr size_t yzy_smem() {
    return ((size_t)yzy_rows<T, L2, NZ, P>() * tile_elems(L1, L2) + (size_t)L1 * L2) * sizeof(cx<T>);
}
constexpr size_t kYzySmemMax = 227 * 1024;
template <typename T, int L1, int L2, int NZ, int P>
__host__ __device__ constexpr bool yzy_fits() {
    return yzy_smem<T, L1, L2, NZ, P>() <= kYzySmemMax &&
           (sizeof(T) == 4 || L1 <= 32);  // FP64 4-step lines: 32 values per thread at most
}
template <typename T, int L2, int NZ, int P> __host__ __device__ constexpr int yzy_threads() {
    return yzy_lpp<T, L2, NZ, P>() * L2;
}

template <typename T, int L1, int L2, int NZ, int P>
__global__ void __launch_bounds__(yzy_threads<T, L2, NZ, P>()) k_yzy(DemagArgs<T> a) {
    using C = cx<T>;
    constexpr int L = L1 * L2, TE = tile_elems(L1, L2), NL = 3 * NZ, NLH = yzy_nlh<NZ, P>();
    constexpr int LPP = yzy_lpp<T, L2, NZ, P>(), ROWS = yzy_rows<T, L2, NZ, P>(), BT = LPP * L2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *S = reinterpret_cast<C *>(smem_raw);
    C *tws = S + ROWS * TE;
    const int h = P > 1 ? (int)cg::this_cluster().block_rank() : 0;
    auto cluster_sync = [&]() {
        if constexpr (P > 1) cg::this_cluster().sync();
        else __syncthreads();
    };
    for (int k = threadIdx.x; k < L; k += BT) tws[k] = a.twyT[k];
    __syncthreads();  // fft4step reads twiddles before its first barrier
    const int kx = blockIdx.x / P, nkx = a.nkx, ny = a.ny;
    const int qg = threadIdx.x / L2, t = threadIdx.x - qg * L2;
    {   // only the z sum reads the plane's table (6 NZ rows of KY values): bring it
        // into L2 while the y forward FFTs run, the rows split over the cluster's CTAs
        constexpr int LN = 128 / (int)sizeof(T);  // values per 128-byte line
        const int KY = a.KY, nln = (KY + LN - 1) / LN;
        const T *t0 = a.spec + (long long)kx * KY;
        for (int i = h * BT + threadIdx.x; i < 6 * NZ * nln; i += P * BT) {
            const int r = i / nln, j = i - r * nln;
            const T *p = t0 + (long long)r * nkx * KY + min(j * LN, KY - 1);
            asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
        }
    }
    // 1. forward y, LPP lines per pass: inputs y < ny (= L/2; the upper half is the
    // zero padding).  Every thread takes part in every pass (fft4step has barriers).
#pragma unroll 1
    for (int r0 = 0; r0 < ROWS; r0 += LPP) {
        const int lr = r0 + qg, q = h * NLH + lr;  // local row, line q = c nz + z
        const bool valid = lr < NLH && q < NL;     // spare rows are scratch
        const C *line1 = a.s1 + ((long long)(valid ? q : 0) * nkx + kx) * ny;  // S1 [c][z][kx][y]
        C *row = S + lr * TE;
        auto in1 = [&](int j) -> C { return valid ? line1[j] : mk<T>(0, 0); };
        auto out1 = [&](int k, C v) { row[k] = v; };
        fft4step<L1, L2, false, false, true, true>(t, tws, row, in1, out1);
    }
    cluster_sync();
    // 2. direct z convolution of this CTA's ky columns (table and signs as in k_zd)
    {
        C *own[P];  // row 0 of every CTA of the cluster
#pragma unroll
        for (int r = 0; r < P; ++r) {
            if constexpr (P > 1) own[r] = cg::this_cluster().map_shared_rank(S, r);
            else own[r] = S;
        }
        auto cell = [&](int line, int ky) -> C & { return own[line / NLH][(line % NLH) * TE + ky]; };
        const int KY = a.KY, dstr = nkx * KY, tstr = NZ * dstr;
        constexpr int KC = L / P;  // columns per CTA
        for (int kk = threadIdx.x; kk < KC; kk += BT) {
            const int ky = h * KC + kk;
            const bool ymir = ky > L / 2;
            const T sy = ymir ? T(-1) : T(1);
            const T *tp = a.spec + (kx * KY + (ymir ? L - ky : ky));
            C mx[NZ], my[NZ], mz[NZ];
#pragma unroll
            for (int z = 0; z < NZ; ++z) {
                mx[z] = cell(z, ky);
                my[z] = cell(NZ + z, ky);
                const C v = cell(2 * NZ + z, ky);
                mz[z] = mk<T>(v.y, -v.x);  // -i Mz
            }
            C hx[NZ], hy[NZ], hz[NZ];
#pragma unroll
            for (int z = 0; z < NZ; ++z) { hx[z] = mk<T>(0, 0); hy[z] = mk<T>(0, 0); hz[z] = mk<T>(0, 0); }
            // the loop of k_zd: per output, offsets d ascending, +d then -d
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
                cell(z, ky) = hx[z];
                cell(NZ + z, ky) = hy[z];
                cell(2 * NZ + z, ky) = mk<T>(-hz[z].y, hz[z].x);  // Hz = i Hz'
            }
        }
    }
    cluster_sync();  // after this no CTA touches another's shared memory
    // 3. inverse y, keep y < ny
#pragma unroll 1
    for (int r0 = 0; r0 < ROWS; r0 += LPP) {
        const int lr = r0 + qg, q = h * NLH + lr;
        const bool valid = lr < NLH && q < NL;
        C *line1 = a.s1 + ((long long)(valid ? q : 0) * nkx + kx) * ny;
        C *row = S + lr * TE;
        auto in3 = [&](int j) -> C { return row[j]; };
        auto out3 = [&](int k, C v) { if (valid && k < ny) line1[k] = v; };
        fft4step<L1, L2, true, true, false>(t, tws, row, in3, out3);
    }
}

template <int N> using YzyIC = std::integral_constant<int, N>;

// (L1, L2) of Ly in 256..1024 and NZ of nz as compile-time values
template <class F>
void yzy_dispatch(int Ly, int nz, F &&f) {
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
            default: break;
        }
    };
    switch (Ly) {
        case 256: nzs(YzyIC<16>{}, YzyIC<16>{}); break;
        case 512: nzs(YzyIC<32>{}, YzyIC<16>{}); break;
        case 1024: nzs(YzyIC<32>{}, YzyIC<32>{}); break;
        default: break;  // other lengths: the split kernels
    }
}

template <class F>
void yzy_with_p(int P, F &&f) {
    switch (P) {
        case 1: f(YzyIC<1>{}); break;
        case 2: f(YzyIC<2>{}); break;
        case 4: f(YzyIC<4>{}); break;
        case 8: f(YzyIC<8>{}); break;
        default: break;
    }
}

// static: every unit that includes this header has its own copy of the
// constant twiddle table (fftreg.cuh) and must fill that one
static bool yzy_upload_tw64(Backend &b) {
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

template <typename T, int L1, int L2, int NZ, int P>
cudaLaunchConfig_t yzy_config(const Backend &b, cudaLaunchAttribute *attr) {
    cudaLaunchConfig_t cfg = {};
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)P;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3((unsigned)(b.nkx * P));
    cfg.blockDim = dim3((unsigned)yzy_threads<T, L2, NZ, P>());
    cfg.dynamicSmemBytes = yzy_smem<T, L1, L2, NZ, P>();
    cfg.stream = b.stream;
    cfg.attrs = attr;
    cfg.numAttrs = P > 1 ? 1 : 0;
    return cfg;
}

template <typename T>
bool yzy_configure_t(Backend &b) {
    b.use_yzy = false;
    b.yzy_P = 0;
    const char *off = std::getenv("FULLMAG_FDM_YZY");
    if (b.thin || !b.zdirect || b.Ly != 2 * b.ny || (off && std::strcmp(off, "off") == 0)) return true;
    // cluster size: FULLMAG_FDM_YZY_P, else the smallest P whose CTA fits twice per SM
    int want = 0;
    if (const char *p = std::getenv("FULLMAG_FDM_YZY_P")) want = std::atoi(p);
    // FP64 only on request: at 512 x 512 x 8 its 8-CTA clusters ran 320 us against
    // 244 us for the three split kernels
    if (sizeof(T) == 8 && !want) return true;
    if (!yzy_upload_tw64(b)) return false;
    yzy_dispatch(b.Ly, b.nz, [&](auto l1, auto l2, auto nzc) {
        constexpr int L1 = decltype(l1)::value, L2 = decltype(l2)::value, NZ = decltype(nzc)::value;
        for (int P : {1, 2, 4, 8}) {
            if (b.use_yzy || (want && P != want)) continue;
            yzy_with_p(P, [&](auto pc) {
                constexpr int PP = decltype(pc)::value;
                if constexpr (yzy_fits<T, L1, L2, NZ, PP>()) {
                    constexpr size_t smem = yzy_smem<T, L1, L2, NZ, PP>();
                    if (!want && PP < 8 && smem > kYzySmemMax / 2) return;  // one CTA per SM: try a larger cluster
                    auto kern = k_yzy<T, L1, L2, NZ, PP>;
                    // the largest shared-memory carveout, so that two CTAs fit per SM
                    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
                        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                             (int)cudaSharedmemCarveoutMaxShared) != cudaSuccess) {
                        cudaGetLastError();
                        return;
                    }
                    if constexpr (PP > 1) {
                        cudaLaunchAttribute attr[1];
                        cudaLaunchConfig_t cfg = yzy_config<T, L1, L2, NZ, PP>(b, attr);
                        int nclusters = 0;
                        if (cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg) != cudaSuccess || nclusters < 1) {
                            cudaGetLastError();
                            return;
                        }
                    }
                    b.yzy_P = PP;
                    b.use_yzy = true;
                }
            });
        }
    });
    return true;
}

template <typename T>
bool yzy_launch_t(Backend &b, const DemagArgs<T> &a) {
    yzy_dispatch(b.Ly, b.nz, [&](auto l1, auto l2, auto nzc) {
        constexpr int L1 = decltype(l1)::value, L2 = decltype(l2)::value, NZ = decltype(nzc)::value;
        yzy_with_p(b.yzy_P, [&](auto pc) {
            constexpr int PP = decltype(pc)::value;
            if constexpr (yzy_fits<T, L1, L2, NZ, PP>()) {
                cudaLaunchAttribute attr[1];
                cudaLaunchConfig_t cfg = yzy_config<T, L1, L2, NZ, PP>(b, attr);
                cudaLaunchKernelEx(&cfg, k_yzy<T, L1, L2, NZ, PP>, a);
            }
        });
    });
    return true;
}

}  // namespace fm
