// demag.cuh — zero-padded Newell-tensor convolution with an in-house FFT.
//
// Replaces the reference's pack -> 3 x cufftExecZ2Z -> tensor multiply ->
// 3 x cufftExecZ2Z -> unpack chain (native/backends/fdm/src/demag_fp64.cu:264-381)
// with five passes over pruned, half-spectrum buffers:
//
//   x_fwd   m (SoA, N cells)  -> S1 [c][z][kx][y]    pack Ms*m, two real rows per
//                                                   complex line, R2C, transposed store
//   y_fwd   S1                -> S2 [c][z][kx][ky]   ny nonzero inputs -> Ly outputs
//   z_conv  S2 in place                              fwd z, H = -N(k) M(k), inv z,
//                                                   only z < nz kept (3-D only)
//   y_inv   S2                -> S1                  keeps y < ny
//   x_inv   S1                -> H_demag (SoA)       C2R, crop, 1/P, mask
//
// Thin films (nz = 1, 2-D spectra) use x_fwd -> y_conv (fwd y, multiply, inv y)
// -> x_inv.  N(k) is real and even/odd per axis (the Newell tensor is even or odd
// in every coordinate), so only the octant kx <= nx, ky <= ny, kz <= nz of its
// real part is stored: spec[comp][kz][kx][ky], comp = xx, yy, zz, xy, xz, yz,
// and the odd components flip sign on the mirrored half of ky and kz.
#pragma once

#include "common.cuh"
#include "fft.cuh"

namespace fm {

template <typename T>
struct DemagArgs {
    int nx, ny, nz;
    long long n;
    int Lx, Ly, Lz, nkx;
    int KZ, KY;             // octant extents: kz in [0, KZ), ky in [0, KY)
    LinePlan px, py, pz;
    const cx<T> *twx, *twy, *twz;
    // register-FFT inter-level twiddles in the order fft4step reads them
    // (twT[k1 L2 + t] = W_L^{k1 t}, fill_tw4's layout), read from global memory
    const cx<T> *twxT, *twyT;
    cx<T> *s1, *s2;
    const T *spec;          // octant, 6 components
    const T *m;             // SoA magnetisation, component stride n
    const uint8_t *mask;    // may be null
    const double *ms_map;   // may be null (then ms)
    double ms;
    const double *vf;       // boundary tiers: volume fraction (M = phi Ms m), else null
    int unit_source;        // 1: source = m on active cells (the adjoint's -N * lambda)
    T *hd;                  // SoA demag field out
    double norm;            // 1 / (Lx Ly Lz)
    int lines_x;            // complex lines (= 2 rows) per x-pass block
    int lines_y;            // lines per y-pass block
    int kt_z;               // ky tile of the z pass
    int kb_y;               // kx per block of the 2-D y_conv pass
};

template <typename T>
__device__ __forceinline__ bool cell_active(const DemagArgs<T> &a, long long i, double &ms_i) {
    ms_i = a.ms_map ? a.ms_map[i] : a.ms;
    return (!a.mask || a.mask[i] != 0) && (ms_i > 0.0);
}

// Magnetisation component fed to the FFT: (phi_i Ms) m_i over every cell when
// a boundary tier weights it (demag_fp64.cu:79-85), else Ms_i m_i on active cells.
template <typename T>
__device__ __forceinline__ T demag_source(const DemagArgs<T> &a, long long i, T m) {
    if (a.vf) return (T)((a.vf[i] * a.ms) * (double)m);
    double msi;
    if (!cell_active(a, i, msi)) return T(0);
    return a.unit_source ? m : (T)((double)m * msi);
}

// Apply H = -N(k) M(k) for one frequency (kx, ky, kz); M is overwritten by H.
template <typename T>
__device__ __forceinline__ void tensor_apply(const DemagArgs<T> &a, int kx, int ky, int kz,
                                             cx<T> &mx, cx<T> &my, cx<T> &mz) {
    int kyo = ky, kzo = kz;
    T sy = T(1), sz = T(1);
    if (ky > a.Ly / 2) { kyo = a.Ly - ky; sy = T(-1); }
    if (kz > a.Lz / 2) { kzo = a.Lz - kz; sz = T(-1); }
    const long long plane = (long long)a.KZ * a.nkx * a.KY;
    const long long o = ((long long)kzo * a.nkx + kx) * a.KY + kyo;
    const T nxx = a.spec[o];
    const T nyy = a.spec[plane + o];
    const T nzz = a.spec[2 * plane + o];
    const T nxy = a.spec[3 * plane + o] * sy;
    const T nxz = a.spec[4 * plane + o] * sz;
    const T nyz = a.spec[5 * plane + o] * (sy * sz);
    cx<T> hx, hy, hz;
    hx.x = -((nxx * mx.x + nxy * my.x) + nxz * mz.x);
    hx.y = -((nxx * mx.y + nxy * my.y) + nxz * mz.y);
    hy.x = -((nxy * mx.x + nyy * my.x) + nyz * mz.x);
    hy.y = -((nxy * mx.y + nyy * my.y) + nyz * mz.y);
    hz.x = -((nxz * mx.x + nyz * my.x) + nzz * mz.x);
    hz.y = -((nxz * mx.y + nyz * my.y) + nzz * mz.y);
    mx = hx; my = hy; mz = hz;
}

// ---------------------------------------------------------------------------
// x_fwd: grid (ceil(ny / (2 lines_x)), nz, 3)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_x_fwd(DemagArgs<T> a) {
    using C = cx<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int LP = a.lines_x, RB = 2 * LP, Lx = a.Lx, ld = Lx + 3;
    C *tw = reinterpret_cast<C *>(smem_raw);
    C *bufA = tw + Lx;
    C *bufB = bufA + LP * ld;
    const int c = blockIdx.z, z = blockIdx.y, y0 = blockIdx.x * RB;
    for (int k = threadIdx.x; k < Lx; k += blockDim.x) tw[k] = a.twx[k];
    const T *mc = a.m + (long long)c * a.n;
    for (int u = threadIdx.x; u < RB * Lx; u += blockDim.x) {
        const int r = u / Lx, x = u - r * Lx, y = y0 + r;
        T v = T(0);
        if (x < a.nx && y < a.ny) {
            const long long i = ((long long)z * a.ny + y) * a.nx + x;
            v = demag_source(a, i, mc[i]);
        }
        T *line = reinterpret_cast<T *>(bufA + (r >> 1) * ld);
        line[2 * x + (r & 1)] = v;
    }
    __syncthreads();
    const C *res = fft_lines<false>(bufA, bufB, a.px, LP, ld, tw);
    const int nkx = a.nkx;
    for (int u = threadIdx.x; u < nkx * RB; u += blockDim.x) {
        const int k = u / RB, r = u - k * RB, y = y0 + r;
        if (y >= a.ny) continue;
        const C *line = res + (r >> 1) * ld;
        const C zk = line[k];
        const C zm = line[k == 0 ? 0 : Lx - k];
        C out;
        if ((r & 1) == 0) {  // A = (Z[k] + conj Z[-k]) / 2
            out.x = T(0.5) * (zk.x + zm.x);
            out.y = T(0.5) * (zk.y - zm.y);
        } else {             // B = -i (Z[k] - conj Z[-k]) / 2
            out.x = T(0.5) * (zk.y + zm.y);
            out.y = T(-0.5) * (zk.x - zm.x);
        }
        a.s1[(((long long)c * a.nz + z) * nkx + k) * a.ny + y] = out;
    }
}

// ---------------------------------------------------------------------------
// y_fwd (3-D): grid ceil(3 nz nkx / lines_y)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_y_fwd(DemagArgs<T> a) {
    using C = cx<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int Ly = a.Ly, ld = Ly + 1, ny = a.ny;
    C *tw = reinterpret_cast<C *>(smem_raw);
    C *bufA = tw + Ly;
    C *bufB = bufA + a.lines_y * ld;
    const long long total = 3LL * a.nz * a.nkx;
    const long long g0 = (long long)blockIdx.x * a.lines_y;
    const int nl = (int)min((long long)a.lines_y, total - g0);
    for (int k = threadIdx.x; k < Ly; k += blockDim.x) tw[k] = a.twy[k];
    for (int u = threadIdx.x; u < nl * Ly; u += blockDim.x) {
        const int line = u / Ly, j = u - line * Ly;
        bufA[line * ld + j] = j < ny ? a.s1[(g0 + line) * ny + j] : mk<T>(0, 0);
    }
    __syncthreads();
    const C *res = fft_lines<false>(bufA, bufB, a.py, nl, ld, tw);
    for (int u = threadIdx.x; u < nl * Ly; u += blockDim.x) {
        const int line = u / Ly, j = u - line * Ly;
        a.s2[(g0 + line) * Ly + j] = res[line * ld + j];
    }
}

// ---------------------------------------------------------------------------
// z_conv (3-D): grid (ceil(Ly / kt_z), nkx); in place on S2
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_z_conv(DemagArgs<T> a) {
    using C = cx<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int Lz = a.Lz, ld = Lz + 1, KT = a.kt_z, nz = a.nz, Ly = a.Ly, nkx = a.nkx;
    C *tw = reinterpret_cast<C *>(smem_raw);
    C *bufA = tw + Lz;
    C *bufB = bufA + 3 * KT * ld;
    const int kx = blockIdx.y, ky0 = blockIdx.x * KT;
    for (int k = threadIdx.x; k < Lz; k += blockDim.x) tw[k] = a.twz[k];
    for (int u = threadIdx.x; u < 3 * KT * Lz; u += blockDim.x) {
        const int kyl = u % KT, rest = u / KT, z = rest % Lz, c = rest / Lz, ky = ky0 + kyl;
        C v = mk<T>(0, 0);
        if (z < nz && ky < Ly) v = a.s2[(((long long)c * nz + z) * nkx + kx) * Ly + ky];
        bufA[(c * KT + kyl) * ld + z] = v;
    }
    __syncthreads();
    C *res = fft_lines<false>(bufA, bufB, a.pz, 3 * KT, ld, tw);
    C *other = (res == bufA) ? bufB : bufA;
    for (int u = threadIdx.x; u < KT * Lz; u += blockDim.x) {
        const int kyl = u % KT, kz = u / KT, ky = ky0 + kyl;
        if (ky >= Ly) continue;
        C mx = res[(0 * KT + kyl) * ld + kz];
        C my = res[(1 * KT + kyl) * ld + kz];
        C mz = res[(2 * KT + kyl) * ld + kz];
        tensor_apply(a, kx, ky, kz, mx, my, mz);
        res[(0 * KT + kyl) * ld + kz] = mx;
        res[(1 * KT + kyl) * ld + kz] = my;
        res[(2 * KT + kyl) * ld + kz] = mz;
    }
    __syncthreads();
    const C *out = fft_lines<true>(res, other, a.pz, 3 * KT, ld, tw);
    for (int u = threadIdx.x; u < 3 * KT * nz; u += blockDim.x) {
        const int kyl = u % KT, rest = u / KT, z = rest % nz, c = rest / nz, ky = ky0 + kyl;
        if (ky < Ly) a.s2[(((long long)c * nz + z) * nkx + kx) * Ly + ky] = out[(c * KT + kyl) * ld + z];
    }
}

// ---------------------------------------------------------------------------
// y_conv (2-D thin film): grid ceil(nkx / kb_y); in place on S1 ([c][kx][y])
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_y_conv(DemagArgs<T> a) {
    using C = cx<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int Ly = a.Ly, ld = Ly + 1, ny = a.ny, KB = a.kb_y, nkx = a.nkx;
    C *tw = reinterpret_cast<C *>(smem_raw);
    C *bufA = tw + Ly;
    C *bufB = bufA + 3 * KB * ld;
    const int kx0 = blockIdx.x * KB;
    const int nb = min(KB, nkx - kx0);
    for (int k = threadIdx.x; k < Ly; k += blockDim.x) tw[k] = a.twy[k];
    for (int u = threadIdx.x; u < 3 * nb * Ly; u += blockDim.x) {
        const int j = u % Ly, lc = u / Ly, kxl = lc % nb, c = lc / nb;
        bufA[(c * nb + kxl) * ld + j] =
            j < ny ? a.s1[((long long)c * nkx + kx0 + kxl) * ny + j] : mk<T>(0, 0);
    }
    __syncthreads();
    C *res = fft_lines<false>(bufA, bufB, a.py, 3 * nb, ld, tw);
    C *other = (res == bufA) ? bufB : bufA;
    for (int u = threadIdx.x; u < nb * Ly; u += blockDim.x) {
        const int ky = u % Ly, kxl = u / Ly;
        C mx = res[(0 * nb + kxl) * ld + ky];
        C my = res[(1 * nb + kxl) * ld + ky];
        C mz = res[(2 * nb + kxl) * ld + ky];
        tensor_apply(a, kx0 + kxl, ky, 0, mx, my, mz);
        res[(0 * nb + kxl) * ld + ky] = mx;
        res[(1 * nb + kxl) * ld + ky] = my;
        res[(2 * nb + kxl) * ld + ky] = mz;
    }
    __syncthreads();
    const C *out = fft_lines<true>(res, other, a.py, 3 * nb, ld, tw);
    for (int u = threadIdx.x; u < 3 * nb * ny; u += blockDim.x) {
        const int j = u % ny, lc = u / ny, kxl = lc % nb, c = lc / nb;
        a.s1[((long long)c * nkx + kx0 + kxl) * ny + j] = out[(c * nb + kxl) * ld + j];
    }
}

// ---------------------------------------------------------------------------
// y_inv (3-D): grid ceil(3 nz nkx / lines_y)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_y_inv(DemagArgs<T> a) {
    using C = cx<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int Ly = a.Ly, ld = Ly + 1, ny = a.ny;
    C *tw = reinterpret_cast<C *>(smem_raw);
    C *bufA = tw + Ly;
    C *bufB = bufA + a.lines_y * ld;
    const long long total = 3LL * a.nz * a.nkx;
    const long long g0 = (long long)blockIdx.x * a.lines_y;
    const int nl = (int)min((long long)a.lines_y, total - g0);
    for (int k = threadIdx.x; k < Ly; k += blockDim.x) tw[k] = a.twy[k];
    for (int u = threadIdx.x; u < nl * Ly; u += blockDim.x) {
        const int line = u / Ly, j = u - line * Ly;
        bufA[line * ld + j] = a.s2[(g0 + line) * Ly + j];
    }
    __syncthreads();
    const C *res = fft_lines<true>(bufA, bufB, a.py, nl, ld, tw);
    for (int u = threadIdx.x; u < nl * ny; u += blockDim.x) {
        const int line = u / ny, j = u - line * ny;
        a.s1[(g0 + line) * ny + j] = res[line * ld + j];
    }
}

// ---------------------------------------------------------------------------
// x_inv: grid (ceil(ny / (2 lines_x)), nz, 3) -> H_demag
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_x_inv(DemagArgs<T> a) {
    using C = cx<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int LP = a.lines_x, RB = 2 * LP, Lx = a.Lx, ld = Lx + 3, nx = a.nx, nkx = a.nkx;
    C *tw = reinterpret_cast<C *>(smem_raw);
    C *bufA = tw + Lx;
    C *bufB = bufA + LP * ld;
    const int c = blockIdx.z, z = blockIdx.y, y0 = blockIdx.x * RB;
    for (int k = threadIdx.x; k < Lx; k += blockDim.x) tw[k] = a.twx[k];
    // raw half spectra of the two rows of each line: A at [0, nkx), B at [nkx, 2 nkx)
    for (int u = threadIdx.x; u < nkx * RB; u += blockDim.x) {
        const int k = u / RB, r = u - k * RB, y = y0 + r;
        C v = mk<T>(0, 0);
        if (y < a.ny) v = a.s1[(((long long)c * a.nz + z) * nkx + k) * a.ny + y];
        bufB[(r >> 1) * ld + (r & 1) * nkx + k] = v;
    }
    __syncthreads();
    // Z = A + i B on the full circle; DC and Nyquist are taken as real (C2R)
    for (int u = threadIdx.x; u < LP * Lx; u += blockDim.x) {
        const int q = u / Lx, k = u - q * Lx;
        const C *raw = bufB + q * ld;
        C zv;
        if (k <= nx) {
            C A = raw[k], B = raw[nkx + k];
            if (k == 0 || k == nx) { A.y = T(0); B.y = T(0); }
            zv.x = A.x - B.y;
            zv.y = A.y + B.x;
        } else {
            const int kk = Lx - k;
            const C A = raw[kk], B = raw[nkx + kk];
            zv.x = A.x + B.y;
            zv.y = -A.y + B.x;
        }
        bufA[q * ld + k] = zv;
    }
    __syncthreads();
    const C *res = fft_lines<true>(bufA, bufB, a.px, LP, ld, tw);
    const T nrm = (T)a.norm;
    T *hc = a.hd + (long long)c * a.n;
    for (int u = threadIdx.x; u < RB * nx; u += blockDim.x) {
        const int r = u / nx, x = u - r * nx, y = y0 + r;
        if (y >= a.ny) continue;
        const C v = res[(r >> 1) * ld + x];
        const long long i = ((long long)z * a.ny + y) * nx + x;
        double msi;
        hc[i] = cell_active(a, i, msi) ? ((r & 1) ? v.y : v.x) * nrm : T(0);
    }
}

// ---------------------------------------------------------------------------
// Sparse demag boundary correction (demag_boundary_fp64.cu:20-76): for target
// t, H(t) += -sum_s dN(t, s) M(s) with M(s) = (phi_s Ms) m_s and the tensor
// components (xx, xy, xz, yy, yz, zz); negative indices are skipped.  One
// thread per target, FP64 arithmetic, added to the field in its precision.
// The targets are distinct cells (each is updated by one thread).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_demag_corr(const T *__restrict__ m, T *hd, long long n,
                                                    const double *__restrict__ vf,
                                                    const int32_t *__restrict__ tgt,
                                                    const int32_t *__restrict__ src,
                                                    const double *__restrict__ ten, double ms,
                                                    unsigned targets, unsigned stencil) {
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= targets) return;
    const int32_t ti = tgt[t];
    if (ti < 0) return;
    double cx_ = 0.0, cy_ = 0.0, cz_ = 0.0;
    for (unsigned q = 0; q < stencil; ++q) {
        const size_t pq = (size_t)t * stencil + q;
        const int32_t si = src[pq];
        if (si < 0) continue;
        const double *N = ten + pq * 6;
        const double w = vf[si] * ms;
        const double Mx = w * (double)m[si], My = w * (double)m[n + si], Mz = w * (double)m[2 * n + si];
        cx_ -= N[0] * Mx + N[1] * My + N[2] * Mz;
        cy_ -= N[1] * Mx + N[3] * My + N[4] * Mz;
        cz_ -= N[2] * Mx + N[4] * My + N[5] * Mz;
    }
    hd[ti] = (T)((double)hd[ti] + cx_);
    hd[n + ti] = (T)((double)hd[n + ti] + cy_);
    hd[2 * n + ti] = (T)((double)hd[2 * n + ti] + cz_);
}

}  // namespace fm
