// demag_reg.cuh — register-FFT versions of the five demag passes.
//
// Same data flow and buffers as demag.cuh (S1 [c][z][kx][y], S2 [c][z][kx][ky],
// real octant spectra), but every line FFT is fft4step (fftreg.cuh): one
// shared-memory round trip per line instead of one per radix-4 stage, no
// integer division in the butterflies, compile-time twiddles inside each
// thread.  Used whenever all padded lengths are powers of two within the
// register limits; other lengths use demag.cuh.
#pragma once

#include "cpasync.cuh"
#include "demag.cuh"
#include "fftreg.cuh"

namespace fm {

// Per-line shared-memory region (tile, then the line's outputs), padded by one
// element so that consecutive lines start in different banks.
template <int L1, int L2> __host__ __device__ constexpr int line_region() {
    return (tile_elems(L1, L2) > L1 * L2 ? tile_elems(L1, L2) : L1 * L2) + 1;
}

// Line stride of the x passes whose threads each handle a pair of rows (the x
// inverse's gather, the pipelined x forward's transposed store): a warp touches
// 4 lines x 8 kx (FP32) or a quarter-warp 4 lines x 2 kx (FP64) at once, and a
// stride of 4 mod 16 (FP32) or 2 mod 8 (FP64) complex elements puts each phase
// in distinct banks (line_region's 1 mod 16 made them collide).  Lines of 32
// threads only: a warp then holds one line inside fft4step.
template <typename T, int L1, int L2> __host__ __device__ constexpr int pair_stride() {
    return L2 == 32 ? line_region<L1, L2>() + (sizeof(T) == 8 ? 1 : 3) : line_region<L1, L2>();
}
// the pipelined x forward: padded in FP32 only (measured at 1024-point lines:
// FP32 28.9 -> 26.9 us, FP64 57.5 -> 65.6 us with the pad)
template <typename T, int L1, int L2> __host__ __device__ constexpr int xf_stride() {
    return sizeof(T) == 4 ? pair_stride<T, L1, L2>() : line_region<L1, L2>();
}

// ---------------------------------------------------------------------------
// x forward: pack Ms*m (two rows per complex line), R2C, transposed store.
// block = lines_x line groups of L2 threads; grid (ceil(ny / 2 lines_x), nz, 3)
// ---------------------------------------------------------------------------
// Block body (bx, z, c); also run per work item by the batched kernels
// (batch.cuh).  PAD: the padded length may exceed 2 nx (batch), so inputs
// j >= nx are zero; otherwise Lx = 2 nx and the half-input pruning covers them.
template <typename T, int L1, int L2, bool PAD = false>
__device__ __forceinline__ void xf_body(const DemagArgs<T> &a, int bx, int z, int c, unsigned char *smem_raw) {
    using C = cx<T>;
    constexpr int L = L1 * L2, TE = line_region<L1, L2>();
    const C *tw = a.twxT;
    C *region = reinterpret_cast<C *>(smem_raw);
    const int LP = a.lines_x, RB = 2 * LP;
    const int y0 = bx * RB;
    const int q = threadIdx.x / L2, t = threadIdx.x - q * L2;
    const T *mc = a.m + (long long)c * a.n;
    const int ya = y0 + 2 * q, yb = ya + 1, nx = a.nx, ny = a.ny;
    const long long rowa = ((long long)z * ny + ya) * nx, rowb = rowa + nx;
    C *line = region + q * TE;
    // M = Ms m in the storage precision (Ms of the uniform material is exact in FP32)
    const T msT = a.unit_source ? T(1) : (T)a.ms;
    auto in = [&](int j) -> C {
        C v = mk<T>(0, 0);
        if (PAD && j >= nx) return v;  // zero padding beyond the row (Lx > 2 nx)
        if (!a.mask && !a.ms_map && !a.vf) {
            if (ya < ny) v.x = mc[rowa + j] * msT;
            if (yb < ny) v.y = mc[rowb + j] * msT;
        } else {
            if (ya < ny) v.x = demag_source(a, rowa + j, mc[rowa + j]);
            if (yb < ny) v.y = demag_source(a, rowb + j, mc[rowb + j]);
        }
        return v;
    };
    auto out = [&](int k, C v) { line[k] = v; };
    if (!PAD && a.mask && !a.ms_map && !a.vf && !a.unit_source && nx % 16 == 0) {
        // masked rows: each line group first copies its two rows of m and of the
        // mask into its own region with 16-byte loads (many in flight), then the
        // transform reads them from there; per-element global loads under the
        // mask test stalled on memory latency (issue active 9 % at 2048-point lines)
        // 8-byte chunks: a line region starts on 8 bytes (its stride is odd in FP32)
        T *rm = reinterpret_cast<T *>(line);                                 // m rows: reals [0, 2 nx)
        unsigned char *rk = reinterpret_cast<unsigned char *>(rm + 2 * nx);  // mask rows: bytes [0, 2 nx)
        constexpr int PT = 8 / (int)sizeof(T);
        const int cm = 2 * nx / PT, ck = 2 * nx / 8;
        for (int u = t; u < cm + ck; u += L2) {
            if (u < cm) {
                const int e = u * PT, r = e >= nx, x = e - r * nx, yy = r ? yb : ya;
                uint2 v = make_uint2(0u, 0u);
                if (yy < ny) v = *reinterpret_cast<const uint2 *>(mc + (r ? rowb : rowa) + x);
                *reinterpret_cast<uint2 *>(rm + e) = v;
            } else {
                const int e = (u - cm) * 8, r = e >= nx, x = e - r * nx, yy = r ? yb : ya;
                uint2 v = make_uint2(0u, 0u);
                if (yy < ny) v = *reinterpret_cast<const uint2 *>(a.mask + (r ? rowb : rowa) + x);
                *reinterpret_cast<uint2 *>(rk + e) = v;
            }
        }
        __syncthreads();
        // M = Ms m on active cells, the product as demag_source forms it
        auto in_s = [&](int j) -> C {
            C v = mk<T>(0, 0);
            if (rk[j]) v.x = (T)((double)rm[j] * a.ms);
            if (rk[nx + j]) v.y = (T)((double)rm[nx + j] * a.ms);
            return v;
        };
        fft4step<L1, L2, false, true, true, true>(t, tw, line, in_s, out);
    } else {
        fft4step<L1, L2, false, false, true, true>(t, tw, line, in, out);
    }
    __syncthreads();
    const int nkx = a.nkx;
    C *s1row = a.s1 + ((long long)c * a.nz + z) * nkx * ny;
    auto emit = [&](int k, int r) {
        const int y = y0 + r;
        if (y >= ny) return;
        const C *ln = region + (r >> 1) * TE;
        const C zk = ln[k];
        const C zm = ln[k == 0 ? 0 : L - k];
        C o;
        if ((r & 1) == 0) { o.x = T(0.5) * (zk.x + zm.x); o.y = T(0.5) * (zk.y - zm.y); }
        else { o.x = T(0.5) * (zk.y + zm.y); o.y = T(-0.5) * (zk.x - zm.x); }
        s1row[(long long)k * ny + y] = o;
    };
    if (ny % 2 == 0 && blockDim.x % LP == 0) {
        // a thread writes both rows of its line pair at one kx (adjacent in S1,
        // one 16-byte store in FP32): Z[k] and Z[L - k] are read once
        const int qq = threadIdx.x % LP, kstep = blockDim.x / LP, ya2 = y0 + 2 * qq;
        if (ya2 < ny) {  // ny even: ya2 + 1 < ny as well
            const C *ln = region + qq * TE;
            for (int k = threadIdx.x / LP; k < nkx; k += kstep) {
                const C zk = ln[k];
                const C zm = ln[k == 0 ? 0 : L - k];
                C o0, o1;
                o0.x = T(0.5) * (zk.x + zm.x); o0.y = T(0.5) * (zk.y - zm.y);
                o1.x = T(0.5) * (zk.y + zm.y); o1.y = T(-0.5) * (zk.x - zm.x);
                C *d = s1row + (long long)k * ny + ya2;
                if constexpr (sizeof(C) == 8) *reinterpret_cast<float4 *>(d) = make_float4(o0.x, o0.y, o1.x, o1.y);
                else { d[0] = o0; d[1] = o1; }
            }
        }
    } else if (blockDim.x % RB == 0) {
        // each thread keeps its row; k advances by blockDim / RB (no division in the loop)
        const int r = threadIdx.x % RB, kstep = blockDim.x / RB;
        for (int k = threadIdx.x / RB; k < nkx; k += kstep) emit(k, r);
    } else {
        for (int u = threadIdx.x; u < nkx * RB; u += blockDim.x) emit(u / RB, u % RB);
    }
}

template <typename T, int L1, int L2>
__global__ void __launch_bounds__(256) k_xf_r(DemagArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    xf_body<T, L1, L2>(a, blockIdx.x, blockIdx.y, blockIdx.z, smem_raw);
}

// ---------------------------------------------------------------------------
// x forward, uniform material (no mask, Ms map or volume fraction; Lx = 2 nx,
// rows of 16-byte multiples): persistent blocks walk the groups g = (c, z,
// y-block) of RB = 2 lines_x rows.  The RB rows of a group are one contiguous
// chunk of m; the next group's chunk is copied into shared memory with 16-byte
// cp.async while the current group is transformed (double buffer, one commit
// group per chunk), so the row loads no longer stall the FFT.  The transform
// and the transposed store are those of xf_body.
// Shared memory: lines_x line regions (xf_stride complex each), 2 x RB nx reals, then
// the Lx twiddles of fft4step (2 x RB nx reals keep them 16-byte aligned).
// ---------------------------------------------------------------------------

template <int L1, int L2, typename T>
__host__ __device__ constexpr size_t xpipe_region_bytes(int lines) {
    return ((size_t)lines * xf_stride<T, L1, L2>() * 2 * sizeof(T) + 15) / 16 * 16;
}

template <typename T, int L1, int L2>
__global__ void __launch_bounds__(256) k_xf_pipe(DemagArgs<T> a, int ngroups) {
    using C = cx<T>;
    constexpr int L = L1 * L2, TE = xf_stride<T, L1, L2>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int LP = a.lines_x, RB = 2 * LP, nx = a.nx, ny = a.ny, nz = a.nz, nkx = a.nkx;
    const int nyb = (ny + RB - 1) / RB;
    C *region = reinterpret_cast<C *>(smem_raw);
    T *stage = reinterpret_cast<T *>(smem_raw + xpipe_region_bytes<L1, L2, T>(LP));
    const size_t stage_elems = (size_t)RB * nx;
    // the 4-step twiddle table, copied once per (persistent) block
    C *tws = reinterpret_cast<C *>(stage + 2 * stage_elems);
    for (int k = threadIdx.x; k < L; k += blockDim.x) tws[k] = a.twxT[k];
    constexpr int PER = 16 / (int)sizeof(T);  // elements per 16-byte copy
    auto issue = [&](int g, int buf) {
        const int yb = g % nyb, cz = g / nyb, z = cz % nz, c = cz / nz;
        const int y0 = yb * RB, rows = min(RB, ny - y0);
        const T *src = a.m + (long long)c * a.n + ((long long)z * ny + y0) * nx;
        T *dst = stage + buf * stage_elems;
        const int chunks = rows * nx / PER;
        for (int u = threadIdx.x; u < chunks; u += blockDim.x) cp_async16(dst + u * PER, src + u * PER);
        cp_async_commit();
    };
    const int q = threadIdx.x / L2, t = threadIdx.x - q * L2;
    C *line = region + q * TE;
    const T msT = a.unit_source ? T(1) : (T)a.ms;
    int buf = 0;
    if (blockIdx.x < ngroups) issue(blockIdx.x, 0);
    for (int g = blockIdx.x; g < ngroups; g += gridDim.x) {
        const int gn = g + gridDim.x;
        if (gn < ngroups) issue(gn, buf ^ 1);
        else cp_async_commit();  // an empty group keeps "all but the newest" meaning this chunk
        cp_async_wait_all_but_one();
        __syncthreads();
        const int yb = g % nyb, cz = g / nyb, z = cz % nz, c = cz / nz;
        const int y0 = yb * RB, ya = y0 + 2 * q, yb1 = ya + 1;
        const T *ra = stage + buf * stage_elems + (size_t)(2 * q) * nx, *rb = ra + nx;
        auto in = [&](int j) -> C {
            C v = mk<T>(0, 0);
            if (ya < ny) v.x = ra[j] * msT;
            if (yb1 < ny) v.y = rb[j] * msT;
            return v;
        };
        auto out = [&](int k, C v) { line[k] = v; };
        fft4step<L1, L2, false, false, true, true>(t, tws, line, in, out);
        __syncthreads();
        C *s1row = a.s1 + ((long long)c * nz + z) * nkx * ny;
        auto emit = [&](int k, int r) {
            const int y = y0 + r;
            if (y >= ny) return;
            const C *ln = region + (r >> 1) * TE;
            const C zk = ln[k];
            const C zm = ln[k == 0 ? 0 : L - k];
            C o;
            if ((r & 1) == 0) { o.x = T(0.5) * (zk.x + zm.x); o.y = T(0.5) * (zk.y - zm.y); }
            else { o.x = T(0.5) * (zk.y + zm.y); o.y = T(-0.5) * (zk.x - zm.x); }
            s1row[(long long)k * ny + y] = o;
        };
        if (ny % 2 == 0 && blockDim.x % LP == 0) {
            // a thread writes both rows of its line pair at one kx (adjacent in S1,
            // one 16-byte store in FP32): Z[k] and Z[L - k] are read once
            const int qq = threadIdx.x % LP, kstep = blockDim.x / LP, ya2 = y0 + 2 * qq;
            if (ya2 < ny) {  // ny even: ya2 + 1 < ny as well
                const C *ln = region + qq * TE;
                for (int k = threadIdx.x / LP; k < nkx; k += kstep) {
                    const C zk = ln[k];
                    const C zm = ln[k == 0 ? 0 : L - k];
                    C o0, o1;
                    o0.x = T(0.5) * (zk.x + zm.x); o0.y = T(0.5) * (zk.y - zm.y);
                    o1.x = T(0.5) * (zk.y + zm.y); o1.y = T(-0.5) * (zk.x - zm.x);
                    C *d = s1row + (long long)k * ny + ya2;
                    if constexpr (sizeof(C) == 8) *reinterpret_cast<float4 *>(d) = make_float4(o0.x, o0.y, o1.x, o1.y);
                    else { d[0] = o0; d[1] = o1; }
                }
            }
        } else if (blockDim.x % RB == 0) {
            const int r = threadIdx.x % RB, kstep = blockDim.x / RB;
            for (int k = threadIdx.x / RB; k < nkx; k += kstep) emit(k, r);
        } else {
            for (int u = threadIdx.x; u < nkx * RB; u += blockDim.x) emit(u / RB, u % RB);
        }
        __syncthreads();  // the line regions and this buffer are reused
        buf ^= 1;
    }
    // retire the copy groups still in flight (none land in memory still read)
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// ---------------------------------------------------------------------------
// x inverse: gather A/B half spectra (transposed), form Z = A + iB on the full
// circle, C2R, crop, 1/P, mask.  Same grid as k_xf_r.
// ---------------------------------------------------------------------------
// TWS: the twiddles were copied into shared memory after the line regions
// (k_xi_r; the batched kernels read them from global memory).
// line stride of the x inverse's shared regions (pair_stride with the pair gather)
template <typename T, int L1, int L2, bool PAIR> __host__ __device__ constexpr int xi_stride() {
    return PAIR ? pair_stride<T, L1, L2>() : line_region<L1, L2>();
}

// PAIR (ny even): a thread loads both rows of its line pair at one kx (adjacent
// in S1) and writes Z[k], Z[L - k] itself, instead of the row-per-thread gather
// whose pairs meet by shuffles; same values, no idle lanes.
template <typename T, int L1, int L2, bool TWS = false, int U = 8, bool PAIR = false>
__device__ __forceinline__ void xi_body(const DemagArgs<T> &a, int bx, int z, int c, unsigned char *smem_raw) {
    using C = cx<T>;
    constexpr int L = L1 * L2, TE = xi_stride<T, L1, L2, PAIR>();
    C *region = reinterpret_cast<C *>(smem_raw);
    const C *tw = TWS ? region + a.lines_x * TE : a.twxT;
    const int LP = a.lines_x, RB = 2 * LP, nx = a.nx, ny = a.ny, nkx = a.nkx;
    const int y0 = bx * RB;
    // Z[k] = A[k] + i B[k] (k <= nx), Z[L-k] = conj(A[k]) + i conj(B[k]); DC and
    // Nyquist taken as real.  Row pairs (A, B) sit in adjacent lanes.
    const C *s1row = a.s1 + ((long long)c * a.nz + z) * nkx * ny;
    auto place = [&](int k, int r, bool ok, C v) {
        const T bx = __shfl_down_sync(0xffffffffu, v.x, 1);
        const T by = __shfl_down_sync(0xffffffffu, v.y, 1);
        if (ok && (r & 1) == 0) {
            C A = v, B = mk<T>(bx, by);
            C *ln = region + (r >> 1) * TE;
            if (k == 0 || k == L / 2) {
                ln[k] = mk<T>(A.x, B.x);
            } else {
                ln[k] = mk<T>(A.x - B.y, A.y + B.x);
                ln[L - k] = mk<T>(A.x + B.y, -A.y + B.x);
            }
        }
    };
    if (PAIR && blockDim.x % LP == 0) {
        const int qq = threadIdx.x % LP, kstep = blockDim.x / LP, k0 = threadIdx.x / LP;
        const int ya = y0 + 2 * qq;  // ny even: ya < ny implies ya + 1 < ny
        const bool rows = ya < ny;
        const int iters = (nkx + kstep - 1) / kstep;
        C *ln = region + qq * TE;
        for (int it0 = 0; it0 < iters; it0 += U) {
            C va[U], vb[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int k = k0 + (it0 + u) * kstep;
                if (k < nkx && rows) {
                    const C *p = s1row + (long long)k * ny + ya;
                    if constexpr (sizeof(C) == 8) {
                        const float4 v = *reinterpret_cast<const float4 *>(p);  // 16-byte aligned: ya, ny even
                        va[u] = mk<T>(v.x, v.y);
                        vb[u] = mk<T>(v.z, v.w);
                    } else {
                        va[u] = p[0];
                        vb[u] = p[1];
                    }
                } else {
                    va[u] = mk<T>(0, 0);
                    vb[u] = mk<T>(0, 0);
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int k = k0 + (it0 + u) * kstep;
                if (k < nkx) {
                    const C A = va[u], B = vb[u];
                    if (k == 0 || k == L / 2) {
                        ln[k] = mk<T>(A.x, B.x);
                    } else {
                        ln[k] = mk<T>(A.x - B.y, A.y + B.x);
                        ln[L - k] = mk<T>(A.x + B.y, -A.y + B.x);
                    }
                }
            }
        }
    } else if (blockDim.x % RB == 0) {
        // fixed row per thread, warp-uniform trip count (the shuffle needs whole
        // warps); U independent loads in flight per thread before they are placed
        const int r = threadIdx.x % RB, kstep = blockDim.x / RB, k0 = threadIdx.x / RB;
        const int y = y0 + r;
        const int iters = (nkx + kstep - 1) / kstep;
        for (int it0 = 0; it0 < iters; it0 += U) {
            C vv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int k = k0 + (it0 + u) * kstep;
                vv[u] = (k < nkx && y < ny) ? s1row[(long long)k * ny + y] : mk<T>(0, 0);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (it0 + u < iters) {
                    const int k = k0 + (it0 + u) * kstep;
                    place(k < nkx ? k : 0, r, k < nkx, vv[u]);
                }
            }
        }
    } else {
        const int total = nkx * RB;
        const int span = (total + 31) / 32 * 32;
        for (int u = threadIdx.x; u < span; u += blockDim.x) {
            const int k = u / RB, r = u % RB, y = y0 + r;
            const bool ok = u < total;
            const C v = (ok && y < ny) ? s1row[(long long)k * ny + y] : mk<T>(0, 0);
            place(k, r, ok, v);
        }
    }
    __syncthreads();
    const int q = threadIdx.x / L2, t = threadIdx.x - q * L2;
    const int ya = y0 + 2 * q, yb = ya + 1;
    C *line = region + q * TE;
    const T nrm = (T)a.norm;
    T *hc = a.hd + (long long)c * a.n;
    const long long rowa = ((long long)z * ny + ya) * nx, rowb = rowa + nx;
    auto in = [&](int j) -> C { return line[j]; };
    // no mask and no Ms map: every cell is active when Ms > 0 (cell_active's answer)
    const bool uniform = !a.mask && !a.ms_map;
    const bool uni_on = a.ms > 0.0;
    auto out = [&](int k, C v) {
        if (k >= nx) return;
        if (uniform) {
            if (ya < ny) hc[rowa + k] = uni_on ? v.x * nrm : T(0);
            if (yb < ny) hc[rowb + k] = uni_on ? v.y * nrm : T(0);
            return;
        }
        double msi;
        if (ya < ny) hc[rowa + k] = cell_active(a, rowa + k, msi) ? v.x * nrm : T(0);
        if (yb < ny) hc[rowb + k] = cell_active(a, rowb + k, msi) ? v.y * nrm : T(0);
    };
    fft4step<L1, L2, true, true, false>(t, tw, line, in, out);
}

// Shared memory: lines_x line regions, then the Lx twiddles.  U: gather loads
// in flight per thread (xi_gather: measured at 512 x 512 x 8 with S1 out of
// L2, FP32 U = 8 / 33: 57.4 / 52.3 us, FP64 U = 8 / 17: 102.7 / 94.8 us).
template <typename T> __host__ __device__ constexpr int xi_gather() { return sizeof(T) == 4 ? 33 : 17; }
// pair gather (two rows per load): 17 load slots, one round at 513 kx
template <typename T> __host__ __device__ constexpr int xi_gather_pair() { return 17; }

template <typename T, int L1, int L2, int U = 8, bool PAIR = false>
__global__ void __launch_bounds__(256) k_xi_r(DemagArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *tws = reinterpret_cast<cx<T> *>(smem_raw) + a.lines_x * xi_stride<T, L1, L2, PAIR>();
    for (int k = threadIdx.x; k < L1 * L2; k += blockDim.x) tws[k] = a.twxT[k];
    // the first barrier inside xi_body (after the gather) precedes every twiddle read
    xi_body<T, L1, L2, true, U, PAIR>(a, blockIdx.x, blockIdx.y, blockIdx.z, smem_raw);
}

// ---------------------------------------------------------------------------
// y forward (3-D): S1 -> S2, line g = (c, z, kx); block = lines_y groups of L2
// ---------------------------------------------------------------------------
template <typename T, int L1, int L2, bool PAD = false>
__device__ __forceinline__ void yf_body(const DemagArgs<T> &a, int bx, unsigned char *smem_raw) {
    using C = cx<T>;
    constexpr int L = L1 * L2, TE = tile_elems(L1, L2);
    const C *tw = a.twyT;
    C *region = reinterpret_cast<C *>(smem_raw);
    const int q = threadIdx.x / L2, t = threadIdx.x - q * L2, ny = a.ny;
    const long long total = 3LL * a.nz * a.nkx;
    const long long g = (long long)bx * a.lines_y + q;
    const bool valid = g < total;
    const C *src = a.s1 + g * ny;
    C *dst = a.s2 + g * L;
    auto in = [&](int j) -> C { return (valid && (!PAD || j < ny)) ? src[j] : mk<T>(0, 0); };
    auto out = [&](int k, C v) { if (valid) dst[k] = v; };
    fft4step<L1, L2, false, false, false, true>(t, tw, region + q * TE, in, out);
}

template <typename T, int L1, int L2>
__global__ void __launch_bounds__(256) k_yf_r(DemagArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    yf_body<T, L1, L2>(a, blockIdx.x, smem_raw);
}

// y inverse (3-D): S2 -> S1, keeps y < ny
template <typename T, int L1, int L2>
__device__ __forceinline__ void yi_body(const DemagArgs<T> &a, int bx, unsigned char *smem_raw) {
    using C = cx<T>;
    constexpr int L = L1 * L2, TE = tile_elems(L1, L2);
    const C *tw = a.twyT;
    C *region = reinterpret_cast<C *>(smem_raw);
    const int q = threadIdx.x / L2, t = threadIdx.x - q * L2, ny = a.ny;
    const long long total = 3LL * a.nz * a.nkx;
    const long long g = (long long)bx * a.lines_y + q;
    const bool valid = g < total;
    const C *src = a.s2 + g * L;
    C *dst = a.s1 + g * ny;
    auto in = [&](int j) -> C { return valid ? src[j] : mk<T>(0, 0); };
    auto out = [&](int k, C v) { if (valid && k < ny) dst[k] = v; };
    fft4step<L1, L2, true, false, false>(t, tw, region + q * TE, in, out);
}

template <typename T, int L1, int L2>
__global__ void __launch_bounds__(256) k_yi_r(DemagArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    yi_body<T, L1, L2>(a, blockIdx.x, smem_raw);
}

// ---------------------------------------------------------------------------
// z convolution (3-D): P threads per (kx, ky) column hold the three
// components' z lines in registers: forward FFT, H = -N M per kz, inverse FFT,
// keep z < nz.  With P = 2 the zero padding (x[z] = 0 for z >= nz = LZ/2) is
// used to split the transform by the parity h of kz:
//   X[2m + h] = FFT_nz(x[z] W_LZ^{h z})[m],
//   x'[z]     = sum_h W_LZ^{-h z} IFFT_nz(X'_h)[z]        (z < nz),
// so each thread of the pair holds 3 x nz values and the two halves are summed
// with one shuffle exchange.
// ---------------------------------------------------------------------------
// One column task tid (tid / P = column, h = tid % P = kz parity, passed in by
// the caller: it is the lane parity, invariant over the caller's loop); the task
// index of a warp's lanes must be contiguous and start at a multiple of 32.
template <typename T, int LZ, int P>
__device__ __forceinline__ void zc_task(const DemagArgs<T> &a, int tid, int h) {
    using C = cx<T>;
    constexpr int NZL = LZ / P;  // points per thread
    static_assert(P == 1 || P == 2, "z split");
    // nkx * Ly < 2^31 for every supported grid: 32-bit index math
    const int cols = a.nkx * a.Ly;
    const int nz = a.nz, Ly = a.Ly, nkx = a.nkx;
    const long long cs = (long long)nz * nkx * Ly;  // component stride in S2
    const long long zs = (long long)nkx * Ly;
    {
        const int col = tid / P;
        const bool valid = col < cols;
        const int kx = valid ? col / Ly : 0;
        const int ky = valid ? col - kx * Ly : 0;
        C *base = a.s2 + (long long)kx * Ly + ky;
        C vx[NZL], vy[NZL], vz[NZL];
#pragma unroll
        for (int z = 0; z < NZL; ++z) {
            const bool in = valid && z < nz;
            vx[z] = in ? base[z * zs] : mk<T>(0, 0);
            vy[z] = in ? base[cs + z * zs] : mk<T>(0, 0);
            vz[z] = in ? base[2 * cs + z * zs] : mk<T>(0, 0);
            if (P == 2 && h == 1 && z > 0) {
                const C w = tw64<C>(z * (64 / LZ));  // W_LZ^z
                vx[z] = cmul(vx[z], w); vy[z] = cmul(vy[z], w); vz[z] = cmul(vz[z], w);
            }
        }
        fft_reg<NZL, false>(vx);
        fft_reg<NZL, false>(vy);
        fft_reg<NZL, false>(vz);
        if (valid) {
            // tensor_apply for one (kx, ky) column: the ky mirror, its sign and the
            // column's offset in a kz plane of the octant are hoisted out of the kz
            // loop; 32-bit offsets (6 KZ nkx KY < 2^31 for every supported grid)
            const int KY = a.KY, plane_z = nkx * KY, cstr = a.KZ * plane_z;
            const bool ymir = ky > Ly / 2;
            const T sy = ymir ? T(-1) : T(1);
            const T *sp = a.spec + (kx * KY + (ymir ? Ly - ky : ky));
#pragma unroll
            for (int p = 0; p < NZL; ++p) {
                const int kz = P * brev<NZL>(p) + h;
                const bool zmir = kz > LZ / 2;
                const T sz = zmir ? T(-1) : T(1);
                const T *q = sp + (zmir ? LZ - kz : kz) * plane_z;
                const T nxx = q[0], nyy = q[cstr], nzz = q[2 * cstr];
                const T nxy = q[3 * cstr] * sy, nxz = q[4 * cstr] * sz, nyz = q[5 * cstr] * (sy * sz);
                const C mx = vx[p], my = vy[p], mz = vz[p];
                vx[p].x = -((nxx * mx.x + nxy * my.x) + nxz * mz.x);
                vx[p].y = -((nxx * mx.y + nxy * my.y) + nxz * mz.y);
                vy[p].x = -((nxy * mx.x + nyy * my.x) + nyz * mz.x);
                vy[p].y = -((nxy * mx.y + nyy * my.y) + nyz * mz.y);
                vz[p].x = -((nxz * mx.x + nyz * my.x) + nzz * mz.x);
                vz[p].y = -((nxz * mx.y + nyz * my.y) + nzz * mz.y);
            }
        }
        fft_reg_dit<NZL, true>(vx);
        fft_reg_dit<NZL, true>(vy);
        fft_reg_dit<NZL, true>(vz);
        if constexpr (P == 1) {
            if (valid) {
#pragma unroll
                for (int z = 0; z < NZL; ++z) {
                    if (z < nz) {
                        base[z * zs] = vx[z];
                        base[cs + z * zs] = vy[z];
                        base[2 * cs + z * zs] = vz[z];
                    }
                }
            }
        } else {
            // thread h keeps z in [h nz/2, (h+1) nz/2); the partner's half arrives by shuffle
#pragma unroll
            for (int zz = 0; zz < NZL / 2; ++zz) {
                // register selection by h without dynamic indexing
                const int zlo = zz, zhi = zz + NZL / 2;
                const int zmine = h ? zhi : zlo;
                C ox = h ? vx[zhi] : vx[zlo], oy = h ? vy[zhi] : vy[zlo], oz = h ? vz[zhi] : vz[zlo];
                C sx = h ? vx[zlo] : vx[zhi], sy = h ? vy[zlo] : vy[zhi], sz = h ? vz[zlo] : vz[zhi];
                if (h == 1) {
                    // this thread's values carry W_LZ^{-z}
                    const C w1 = tw64<C>(zhi * (64 / LZ));
                    ox = cmulc(ox, w1); oy = cmulc(oy, w1); oz = cmulc(oz, w1);
                    const C w2 = tw64<C>(zlo * (64 / LZ));
                    sx = cmulc(sx, w2); sy = cmulc(sy, w2); sz = cmulc(sz, w2);
                }
                C rx, ry, rz;
                rx.x = __shfl_xor_sync(0xffffffffu, sx.x, 1); rx.y = __shfl_xor_sync(0xffffffffu, sx.y, 1);
                ry.x = __shfl_xor_sync(0xffffffffu, sy.x, 1); ry.y = __shfl_xor_sync(0xffffffffu, sy.y, 1);
                rz.x = __shfl_xor_sync(0xffffffffu, sz.x, 1); rz.y = __shfl_xor_sync(0xffffffffu, sz.y, 1);
                if (valid && zmine < nz) {
                    base[zmine * zs] = cadd(ox, rx);
                    base[cs + zmine * zs] = cadd(oy, ry);
                    base[2 * cs + zmine * zs] = cadd(oz, rz);
                }
            }
        }
    }
}

template <typename T, int LZ, int P>
__global__ void __launch_bounds__(128) k_zc_r(DemagArgs<T> a) {
    const int span = ((a.nkx * a.Ly * P + 127) / 128) * 128;  // whole pairs and warps iterate together
    const int h = (P == 2) ? (threadIdx.x & 1) : 0;
    for (int tid = blockIdx.x * blockDim.x + threadIdx.x; tid < span; tid += gridDim.x * blockDim.x)
        zc_task<T, LZ, P>(a, tid, h);
}

// ---------------------------------------------------------------------------
// z convolution by direct summation (3-D, nz <= 8).  With the zero padding the
// FFT pass computes, per (kx, ky) column, the linear convolution
//   H(z) = -sum_{z' < nz} n(z - z') M(z'),   n(d) = sum_kz N(kx, ky, kz) W_Lz^{-kz d},
// and only offsets |d| < nz reach a kept output, so the same sum is taken here
// directly: nz^2 3x3 tensor products per column instead of the two z FFTs,
// no twiddles and no padded points.  The table (built on the host from the
// octant, newell_host.hpp octant_to_z_direct) holds n(d) for d in [0, nz):
// components even in z are real; xz and yz are i tau(d) with tau real and odd
// in d.  With Mz' = -i Mz and Hz' = -i Hz the product is a real matrix on
// complex vectors,
//   (Hx, Hy, Hz') = [[-nxx, -nxy, tau_xz], [-nxy, -nyy, tau_yz],
//                    [-tau_xz, -tau_yz, -nzz]] (Mx, My, Mz'),
// stored as tab[c][d][kx][ky'] = (-nxx, -nyy, -nzz, -nxy, tau_xz, tau_yz) for
// ky' <= Ly/2.  ky > Ly/2 reads the mirror with the sign of the components odd
// in y (xy, yz); d < 0 flips the components odd in z (xz, yz).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void zd_fma(float2 &h, float c, float2 m) {
    h = __ffma2_rn(make_float2(c, c), m, h);  // packed: one instruction for both parts
}
__device__ __forceinline__ void zd_fma(double2 &h, double c, double2 m) {
    h.x = fma(c, m.x, h.x);
    h.y = fma(c, m.y, h.y);
}

// Persistent threads, one column per thread per iteration; the
// next column's inputs and table entries are copied into the thread's own
// shared-memory slots (cp.async, double buffer) while the current one is
// summed, so the loads of one column overlap the arithmetic of the previous.
// A thread only reads back what it copied itself: no block barrier.
// Shared memory per thread: 2 x (3 nz complex + 6 nz reals), item-major with
// the thread index fastest (conflict-free).
template <typename T, int NZ>
__host__ __device__ constexpr size_t zd_smem_per_thread() {
    return 2 * (3 * NZ * sizeof(cx<T>) + 6 * NZ * sizeof(T));
}
template <typename T> __host__ __device__ constexpr int zd_threads() { return sizeof(T) == 8 ? 64 : 128; }

template <typename T, int NZ>
__global__ void __launch_bounds__(zd_threads<T>()) k_zd(DemagArgs<T> a) {
    using C = cx<T>;
    constexpr int NM = 3 * NZ, NT = 6 * NZ, BT = zd_threads<T>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x;
    C *mb0 = reinterpret_cast<C *>(smem_raw);
    T *tb0 = reinterpret_cast<T *>(mb0 + 2 * NM * BT);
    // 3 NZ nkx Ly and 6 NZ nkx KY < 2^31 for every supported grid: 32-bit offsets
    const int Ly = a.Ly, KY = a.KY, cols = a.nkx * Ly;
    const int cs = NZ * cols, dstr = a.nkx * KY, tstr = NZ * dstr;
    auto prefetch = [&](int col, int buf) {
        const int kx = col / Ly, ky = col - kx * Ly;
        const C *src = a.s2 + col;
        const unsigned dm = (unsigned)__cvta_generic_to_shared(mb0 + buf * NM * BT + tid);
#pragma unroll
        for (int s = 0; s < NM; ++s)
            cp_async_elem<sizeof(C)>(dm + s * BT * (unsigned)sizeof(C), src + (s / NZ) * cs + (s % NZ) * cols);
        const T *tp = a.spec + (kx * KY + (ky > Ly / 2 ? Ly - ky : ky));
        const unsigned dt = (unsigned)__cvta_generic_to_shared(tb0 + buf * NT * BT + tid);
#pragma unroll
        for (int c = 0; c < 6; ++c)
#pragma unroll
            for (int d = 0; d < NZ; ++d)
                if (c < 4 || d > 0)  // tau(0) = 0 is not read
                    cp_async_elem<sizeof(T)>(dt + (c * NZ + d) * BT * (unsigned)sizeof(T), tp + c * tstr + d * dstr);
    };
    const int stride = gridDim.x * BT;
    int col = blockIdx.x * BT + tid, buf = 0;
    if (col < cols) prefetch(col, 0);
    cp_async_commit();
    for (; col < cols; col += stride, buf ^= 1) {
        if (col + stride < cols) prefetch(col + stride, buf ^ 1);
        cp_async_commit();  // possibly empty: "all but the newest" is this column
        cp_async_wait_all_but_one();
        const C *sm = mb0 + buf * NM * BT + tid;
        const T *st = tb0 + buf * NT * BT + tid;
        const int kx = col / Ly, ky = col - kx * Ly;
        const T sy = ky > Ly / 2 ? T(-1) : T(1);
        C mx[NZ], my[NZ], mz[NZ], hx[NZ], hy[NZ], hz[NZ];
#pragma unroll
        for (int z = 0; z < NZ; ++z) {
            mx[z] = sm[z * BT];
            my[z] = sm[(NZ + z) * BT];
            const C v = sm[(2 * NZ + z) * BT];
            mz[z] = mk<T>(v.y, -v.x);  // -i Mz
            hx[z] = mk<T>(0, 0); hy[z] = mk<T>(0, 0); hz[z] = mk<T>(0, 0);
        }
#pragma unroll
        for (int d = 0; d < NZ; ++d) {
            const T cxx = st[d * BT], cyy = st[(NZ + d) * BT], czz = st[(2 * NZ + d) * BT];
            const T cxy = st[(3 * NZ + d) * BT] * sy;
            const T cxz = d > 0 ? st[(4 * NZ + d) * BT] : T(0), cyz = d > 0 ? st[(5 * NZ + d) * BT] * sy : T(0);
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
        C *base = a.s2 + col;
#pragma unroll
        for (int z = 0; z < NZ; ++z) {
            base[z * cols] = hx[z];
            base[cs + z * cols] = hy[z];
            base[2 * cs + z * cols] = mk<T>(-hz[z].y, hz[z].x);  // Hz = i Hz'
        }
    }
    cp_async_wait_all();
}


// ---------------------------------------------------------------------------
// y convolution (2-D thin film): block = kb_y kx columns x 3 components, each
// line a group of L2 threads: forward y, multiply with N(kx, ky, 0), inverse y.
// ---------------------------------------------------------------------------
template <typename T, int L1, int L2>
__global__ void __launch_bounds__(256) k_yc_r(DemagArgs<T> a) {
    using C = cx<T>;
    constexpr int L = L1 * L2, TE = line_region<L1, L2>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const C *tw = a.twyT;
    C *region = reinterpret_cast<C *>(smem_raw);
    const int KB = a.kb_y, ny = a.ny, nkx = a.nkx;
    const int q = threadIdx.x / L2, t = threadIdx.x - q * L2;
    const int comp = q / KB, kxl = q - comp * KB;
    const int kx0 = blockIdx.x * KB, kx = kx0 + kxl;
    const bool valid = kx < nkx;
    C *line = region + q * TE;
    C *g = a.s1 + ((long long)comp * nkx + kx) * ny;
    auto in_g = [&](int j) -> C { return valid ? g[j] : mk<T>(0, 0); };
    auto out_s = [&](int k, C v) { line[k] = v; };
    fft4step<L1, L2, false, false, true, true>(t, tw, line, in_g, out_s);
    __syncthreads();
    for (int u = threadIdx.x; u < KB * L; u += blockDim.x) {
        const int kl = u / L, ky = u - kl * L;
        if (kx0 + kl >= nkx) continue;
        C *lx = region + (0 * KB + kl) * TE, *lyy = region + (1 * KB + kl) * TE,
          *lz = region + (2 * KB + kl) * TE;
        C mx = lx[ky], my = lyy[ky], mz = lz[ky];
        tensor_apply(a, kx0 + kl, ky, 0, mx, my, mz);
        lx[ky] = mx; lyy[ky] = my; lz[ky] = mz;
    }
    __syncthreads();
    auto in_s = [&](int j) -> C { return line[j]; };
    auto out_g = [&](int k, C v) { if (valid && k < ny) g[k] = v; };
    fft4step<L1, L2, true, true, false>(t, tw, line, in_s, out_g);
}

}  // namespace fm
