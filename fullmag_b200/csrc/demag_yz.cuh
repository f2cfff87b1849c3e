// demag_yz.cuh — the fused y-z convolution pass (3-D demag, register FFTs).
//
// Compiled in its own translation units (demag_yz_f32.cu, demag_yz_f64.cu) so
// its many (M, LZ) instantiations build in parallel with the rest of the
// library; each unit holds its own copy of the W_64 constant table and uploads
// it when a backend is configured.
#pragma once

#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <type_traits>

#include "backend_impl.hpp"
#include "demag.cuh"
#include "demag_yz.hpp"
#include "fftreg.cuh"

namespace fm {

// ---------------------------------------------------------------------------
// Fused y-z convolution (3-D): S1 -> S1 in place, one cluster of P CTAs per kx.
//
// CTA h of the cluster owns the wavenumbers ky = P m + h (m < M = Ly / P).
// With y = j + s M (j < M) and x[y] = 0 for y >= ny = P M / 2,
//   X[P m + h] = FFT_M(f)[m],  f[j] = W_Ly^{h j} sum_{s < P/2} x[j + s M] W_P^{h s},
// so every CTA reads the whole input line but transforms only M points, and
// the (ky, z) slab of all three components, 3 nz lines of M values, stays in
// its shared memory through the z transform, H = -N M and the inverse z
// transform (as in k_zc_r).  Coming back,
//   x'[j + s M] = sum_h W_P^{-h s} Y_h[j],  Y_h[j] = W_Ly^{-h j} IFFT_M(X'_h)[j],
// so each CTA forms its Y_h in place, the cluster synchronises, and CTA r sums
// the P contributions for its M / 2 outputs y in [r M / 2, (r + 1) M / 2) by
// reading its peers' shared memory (distributed shared memory, in rank order,
// so the sum is deterministic).  S1 is read once and written once; the padded
// y spectrum never leaves the chip.
//
// Shared memory: W_M^{k1 t} (M), W_Ly^{h j} (M), W_P^k (8), then the line slots of
// LD = M + M1 elements (each line's 4-step transpose tile overlaps the line):
// 3 nz slots when M2 = 1 (no tile), else ceil(3 nz / G) G, since idle groups
// still write their tile.
// block = G line groups of M2 threads; grid = nkx * P, cluster (P, 1, 1).
// ---------------------------------------------------------------------------
template <int M1, int M2> __host__ __device__ constexpr int yz_ld() {
    return M2 == 1 ? M1 : M1 * M2 + M1;
}

template <typename T, int M1, int M2, int LZ, int PZ>
__global__ void __launch_bounds__(384, sizeof(T) == 4 ? 2 : 1) k_yz_r(DemagArgs<T> a) {
    using C = cx<T>;
    namespace cg = cooperative_groups;
    constexpr int M = M1 * M2, LD = yz_ld<M1, M2>();
    constexpr int NZL = LZ / PZ;
    static_assert(PZ == 1 || PZ == 2, "z split");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cg::cluster_group cluster = cg::this_cluster();
    const int P = (int)cluster.num_blocks();
    const int h = (int)cluster.block_rank();
    const int kx = blockIdx.x / P;
    const int ny = a.ny, nz = a.nz, nkx = a.nkx;
    const int nthr = blockDim.x;
    C *twM = reinterpret_cast<C *>(smem_raw);  // W_M^{k1 t} (fill_tw4 order), W_M = W_Ly^P
    C *twist = twM + M;                         // W_Ly^{h j}
    C *rootP = twist + M;                       // W_P^k = W_Ly^{k M}
    C *buf = rootP + 8;
    fill_tw4<M1, M2>(twM, a.twy, P);
    for (int k = threadIdx.x; k < M; k += nthr) twist[k] = a.twy[h * k];
    if (threadIdx.x < 8) rootP[threadIdx.x] = a.twy[(threadIdx.x & (P - 1)) * M];
    __syncthreads();

    const int G = nthr / M2;
    const int q = threadIdx.x / M2, t = threadIdx.x - q * M2;
    const int nl = 3 * nz;
    const int iters = (nl + G - 1) / G;  // the buffer holds iters * G line slots

    // ---- y forward, this CTA's residue class ----
    for (int it = 0; it < iters; ++it) {
        const int line = it * G + q;  // = c * nz + z
        const bool valid = line < nl;
        const C *src = a.s1 + (valid ? ((long long)line * nkx + kx) * ny : 0);
        C *dst = buf + line * LD;
        auto in = [&](int j) -> C {
            C acc = mk<T>(0, 0);
            if (valid && (P > 1 || j < ny)) {
                acc = src[j];
                for (int s = 1; s < P / 2; ++s)
                    acc = cadd(acc, cmul(src[j + s * M], rootP[(h * s) & (P - 1)]));
                if (h) acc = cmul(acc, twist[j]);
            }
            return acc;
        };
        auto out = [&](int k, C v) { if (valid) dst[k] = v; };
        fft4step<M1, M2, false, false, true>(t, twM, dst, in, out);
    }
    __syncthreads();

    // ---- z convolution per local column m (ky = P m + h) ----
    {
        const int ntask = M * PZ;
        const int span = (ntask + 31) / 32 * 32;  // pairs and warps iterate together
        for (int task = threadIdx.x; task < span; task += nthr) {
            const int m = task / PZ;
            const bool valid = m < M;
            const int hz = (PZ == 2) ? (task & 1) : 0;
            const int ky = P * m + h;
            C *col = buf + (valid ? m : 0);
            const int cs = nz * LD;  // component stride in buf
            C vx[NZL], vy[NZL], vz[NZL];
#pragma unroll
            for (int z = 0; z < NZL; ++z) {
                const bool in = valid && z < nz;
                vx[z] = in ? col[z * LD] : mk<T>(0, 0);
                vy[z] = in ? col[cs + z * LD] : mk<T>(0, 0);
                vz[z] = in ? col[2 * cs + z * LD] : mk<T>(0, 0);
                if (PZ == 2 && hz == 1 && z > 0) {
                    const C w = tw64<C>(z * (64 / LZ));  // W_LZ^z
                    vx[z] = cmul(vx[z], w); vy[z] = cmul(vy[z], w); vz[z] = cmul(vz[z], w);
                }
            }
            fft_reg<NZL, false>(vx);
            fft_reg<NZL, false>(vy);
            fft_reg<NZL, false>(vz);
            if (valid) {
#pragma unroll
                for (int p = 0; p < NZL; ++p) {
                    const int kz = PZ * brev<NZL>(p) + hz;
                    tensor_apply(a, kx, ky, kz, vx[p], vy[p], vz[p]);
                }
            }
            fft_reg_dit<NZL, true>(vx);
            fft_reg_dit<NZL, true>(vy);
            fft_reg_dit<NZL, true>(vz);
            if constexpr (PZ == 1) {
                if (valid) {
#pragma unroll
                    for (int z = 0; z < NZL; ++z) {
                        if (z < nz) {
                            col[z * LD] = vx[z];
                            col[cs + z * LD] = vy[z];
                            col[2 * cs + z * LD] = vz[z];
                        }
                    }
                }
            } else {
#pragma unroll
                for (int zz = 0; zz < NZL / 2; ++zz) {
                    const int zlo = zz, zhi = zz + NZL / 2;
                    const int zmine = hz ? zhi : zlo;
                    C ox = hz ? vx[zhi] : vx[zlo], oy = hz ? vy[zhi] : vy[zlo], oz = hz ? vz[zhi] : vz[zlo];
                    C sx = hz ? vx[zlo] : vx[zhi], sy = hz ? vy[zlo] : vy[zhi], sz = hz ? vz[zlo] : vz[zhi];
                    if (hz == 1) {
                        const C w1 = tw64<C>(zhi * (64 / LZ));
                        ox = cmulc(ox, w1); oy = cmulc(oy, w1); oz = cmulc(oz, w1);
                        const C w2 = tw64<C>(zlo * (64 / LZ));
                        sx = cmulc(sx, w2); sy = cmulc(sy, w2); sz = cmulc(sz, w2);
                    }
                    C rx, ry, rz;
                    rx.x = __shfl_xor_sync(0xffffffffu, sx.x, 1); rx.y = __shfl_xor_sync(0xffffffffu, sx.y, 1);
                    ry.x = __shfl_xor_sync(0xffffffffu, sy.x, 1); ry.y = __shfl_xor_sync(0xffffffffu, sy.y, 1);
                    rz.x = __shfl_xor_sync(0xffffffffu, sz.x, 1); rz.y = __shfl_xor_sync(0xffffffffu, sz.y, 1);
                    // both threads of the pair have read the whole column (before the
                    // shuffles); order those reads before this thread's writes
                    __syncwarp();
                    if (valid && zmine < nz) {
                        col[zmine * LD] = cadd(ox, rx);
                        col[cs + zmine * LD] = cadd(oy, ry);
                        col[2 * cs + zmine * LD] = cadd(oz, rz);
                    }
                }
            }
        }
    }
    __syncthreads();

    // ---- y inverse of this CTA's residue class, twisted by W_Ly^{-h j} ----
    for (int it = 0; it < iters; ++it) {
        const int line = it * G + q;
        const bool valid = line < nl;
        C *dst = buf + line * LD;
        auto in = [&](int j) -> C { return valid ? dst[j] : mk<T>(0, 0); };
        auto out = [&](int k, C v) { if (valid) dst[k] = h ? cmulc(v, twist[k]) : v; };
        fft4step<M1, M2, true, true, true>(t, twM, dst, in, out);
    }
    cluster.sync();

    // ---- sum over the cluster for y in [h M/2, (h+1) M/2) and store ----
    {
        constexpr int YC = M / 2;
        const int y0 = h * YC;
        for (int u = threadIdx.x; u < nl * YC; u += nthr) {
            const int line = u / YC, y = y0 + (u - line * YC);
            const int s = y / M, yp = y - s * M;
            C acc = mk<T>(0, 0);
            for (int r = 0; r < P; ++r) {
                const C *rb = cluster.map_shared_rank(buf, r);
                C v = rb[line * LD + yp];
                if (s) v = cmulc(v, rootP[(r * s) & (P - 1)]);
                acc = cadd(acc, v);
            }
            a.s1[((long long)line * nkx + kx) * ny + y] = acc;
        }
    }
    // peers may still be reading this CTA's shared memory
    cluster.sync();
}


template <int V> using YzIC = std::integral_constant<int, V>;

// (M1, M2) of the per-CTA y length M, 16 <= M <= 1024 (fftreg.cuh's l2_for)
template <class F>
static bool yz_split(int M, F &&f) {
    switch (M) {
        case 16: f(YzIC<16>{}, YzIC<1>{}); return true;
        case 32: f(YzIC<32>{}, YzIC<1>{}); return true;
        case 64: f(YzIC<8>{}, YzIC<8>{}); return true;
        case 128: f(YzIC<16>{}, YzIC<8>{}); return true;
        case 256: f(YzIC<16>{}, YzIC<16>{}); return true;
        case 512: f(YzIC<32>{}, YzIC<16>{}); return true;
        case 1024: f(YzIC<32>{}, YzIC<32>{}); return true;
        default: return false;
    }
}

// (LZ, PZ) of the z transform: one thread per column up to 8 points, a pair above
template <typename T, class F>
static bool yz_lz(int Lz, F &&f) {
    switch (Lz) {
        case 2: f(YzIC<2>{}, YzIC<1>{}); return true;
        case 4: f(YzIC<4>{}, YzIC<1>{}); return true;
        case 8: f(YzIC<8>{}, YzIC<1>{}); return true;
        case 16: f(YzIC<16>{}, YzIC<2>{}); return true;
        case 32:
            if constexpr (sizeof(T) == 4) { f(YzIC<32>{}, YzIC<2>{}); return true; }
            return false;
        default: return false;
    }
}

static bool yz_upload_tw64(Backend &b) {
    double2 d[64];
    float2 f[64];
    for (int k = 0; k < 64; ++k) {
        const double a = 2.0 * 3.14159265358979323846 * (double)k / 64.0;
        d[k] = make_double2(std::cos(a), -std::sin(a));
        f[k] = make_float2((float)d[k].x, (float)d[k].y);
    }
    return cuda_ok(b, cudaMemcpyToSymbol(c_tw64d, d, sizeof(d)), "twiddle64 d (yz)") &&
           cuda_ok(b, cudaMemcpyToSymbol(c_tw64f, f, sizeof(f)), "twiddle64 f (yz)");
}

template <typename T>
static cudaLaunchConfig_t yz_config(const Backend &b, int P, int thr, size_t smem, cudaLaunchAttribute *attr) {
    cudaLaunchConfig_t cfg = {};
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)P;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3((unsigned)(b.nkx * P));
    cfg.blockDim = dim3((unsigned)thr);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = b.stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

// The smallest cluster size P whose per-CTA slab fits two CTAs per SM; the
// pass stays off (three y/z kernels) when none does.  False only on a CUDA
// error that leaves the backend unusable.
template <typename T>
static bool yz_configure_t(Backend &b) {
    b.use_yz = false;
    if (!yz_upload_tw64(b)) return false;
    const size_t sz = 2 * sizeof(T), budget = 113 * 1024;
    const int nl = 3 * b.nz;
    for (int P = b.yz_min_P; P <= 8 && !b.use_yz; P *= 2) {
        const int M = b.Ly / P;
        if (b.Ly % P) continue;
        yz_split(M, [&](auto m1, auto m2) {
            constexpr int M1 = decltype(m1)::value, M2 = decltype(m2)::value;
            yz_lz<T>(b.Lz, [&](auto lz, auto pz) {
                constexpr int LZ = decltype(lz)::value, PZ = decltype(pz)::value;
                const int unit = M2 >= 32 ? 1 : 32 / M2;  // whole warps
                int G = (nl + unit - 1) / unit * unit;
                while (G * M2 > 384 && G > unit) G = ((G + 1) / 2 + unit - 1) / unit * unit;
                if (G * M2 < 128) G = 128 / M2;
                const int iters = (nl + G - 1) / G;
                const int slots = M2 == 1 ? nl : iters * G;
                const size_t smem = (size_t)(2 * M + 8 + (size_t)slots * yz_ld<M1, M2>()) * sz;
                if (smem > budget || G * M2 > 384) return;
                auto kern = k_yz_r<T, M1, M2, LZ, PZ>;
                if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
                    cudaGetLastError();
                    return;
                }
                cudaLaunchAttribute attr[1];
                cudaLaunchConfig_t cfg = yz_config<T>(b, P, G * M2, smem, attr);
                int nclusters = 0;
                if (cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg) != cudaSuccess || nclusters < 1) {
                    cudaGetLastError();
                    return;
                }
                b.yz_P = P;
                b.thr_yz = G * M2;
                b.rsm_yz = smem;
                b.use_yz = true;
            });
        });
    }
    return true;
}

template <typename T>
static bool yz_launch_t(Backend &b, const DemagArgs<T> &a) {
    cudaError_t err = cudaErrorInvalidConfiguration;
    yz_split(b.Ly / b.yz_P, [&](auto m1, auto m2) {
        constexpr int M1 = decltype(m1)::value, M2 = decltype(m2)::value;
        yz_lz<T>(b.Lz, [&](auto lz, auto pz) {
            constexpr int LZ = decltype(lz)::value, PZ = decltype(pz)::value;
            cudaLaunchAttribute attr[1];
            cudaLaunchConfig_t cfg = yz_config<T>(b, b.yz_P, b.thr_yz, b.rsm_yz, attr);
            err = cudaLaunchKernelEx(&cfg, k_yz_r<T, M1, M2, LZ, PZ>, a);
        });
    });
    return cuda_ok(b, err, "demag_yz launch");
}

}  // namespace fm
