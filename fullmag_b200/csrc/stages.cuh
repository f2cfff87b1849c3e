// stages.cuh — fused exchange + Zeeman + LLG stage kernels and reductions.
//
// One kernel evaluates, per cell, the 6-point exchange field with clamped
// (Neumann) neighbours, adds the demag field produced by the FFT passes and
// the (optionally time-dependent) Zeeman field, forms the Gilbert RHS and,
// depending on MODE, also applies the integrator update and the diagnostics
// reductions.  This replaces the reference's separate exchange, combine,
// llg_rhs, predictor/corrector and five reduction kernels
// (native/backends/fdm/src/exchange_fp64.cu, demag_fp64.cu:213-260,
// llg_fp64.cu:43-150, llg_dp45_fp64.cu:44-165, reductions_fp64.cu).
//
// Semantics follow the reference CPU engine (crates/fullmag-engine/src/lib.rs):
// exchange 2247-2299, H_eff = (H_ex + H_d) + H_ext (2836-2843), RHS 2589-2600,
// normalised() zero-preserving (vector.rs:12-19); the exchange energy uses the
// CUDA backend's forward-pair sum (reductions_fp64.cu:122-214) and the region
// LUT follows exchange_fp64.cu:80-114.  All reductions accumulate in FP64 with
// a fixed warp-shuffle tree, so repeated runs are bitwise identical.
#pragma once

#include "common.cuh"

namespace fm {

enum : int {
    Q_EEX = 0,     // sum of forward-pair exchange energy (J)
    Q_EDEMAG = 1,  // sum -1/2 mu0 Ms V m.H_d (J)
    Q_EEXT = 2,    // sum -mu0 Ms V m.H_ext (J)
    Q_HEFF2 = 3,   // max |H_eff|^2
    Q_HD2 = 4,     // max |H_d|^2
    Q_RHS2 = 5,    // max |dm/dt|^2
    Q_ERR2 = 6,    // max |DP45 error|^2
    NQ = 7,
};
__host__ __device__ constexpr bool q_is_max(int q) { return q >= Q_HEFF2; }

enum : int {
    MODE_EVAL = 0,        // k = RHS(m); optional observables / diagnostics
    MODE_HEUN_CORR = 1,   // k2 = RHS(m_p); m <- normalize(m0 + dt/2 (k1 + k2))
    MODE_DP45_LAST = 2,   // k7 = RHS(y); diagnostics + embedded error norm
};

template <typename T>
struct StageArgs {
    int nx, ny, nz;
    long long n;
    T idx2, idy2, idz2;             // 1/dx^2, 1/dy^2, 1/dz^2
    double dinv[3];                 // same, FP64 (energies)
    double aex, ms;                 // uniform A and Ms
    const double *ms_map;           // optional per-cell Ms
    const uint8_t *mask;            // optional
    const uint32_t *region;         // optional
    const double *lut;              // 256 x 256, with region
    int enable_exchange, enable_demag, has_ext;
    double hext[3], hac[3], ac_omega;
    double gamma_bar, alpha;
    int precession;
    double vol;
    double t;                       // stage time (Zeeman)
    // buffers (SoA, component stride n)
    const T *m;                     // state evaluated (stencil)
    const T *hd;                    // demag field of m
    T *kout;                        // RHS out
    T *hex_out, *heff_out;          // optional observables
    double *partials;               // [NQ][gridDim.x] or null
    // MODE_HEUN_CORR
    T *m0;                          // in: m0; out: corrected m (same buffer)
    const T *k1;
    double half_dt;
    // MODE_DP45_LAST: error weights on k1,k3,k4,k5,k6,k7
    const T *ke[5];
    double dt;
};

__device__ __forceinline__ double warp_reduce(double v, bool is_max) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double w = __shfl_down_sync(0xffffffffu, v, o);
        v = is_max ? fmax(v, w) : v + w;
    }
    return v;
}

// Reduce acc[NQ] over the block; thread 0 stores partials[q * gridDim.x + blockIdx.x].
__device__ __forceinline__ void block_reduce_store(double (&acc)[NQ], double *partials) {
    __shared__ double sred[NQ][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        double v = warp_reduce(acc[q], q_is_max(q));
        if (lane == 0) sred[q][warp] = v;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            double v = lane < nw ? sred[q][lane] : 0.0;
            v = warp_reduce(v, q_is_max(q));
            if (lane == 0) partials[(long long)q * gridDim.x + blockIdx.x] = v;
        }
    }
}

template <typename T>
__device__ __forceinline__ bool st_active(const StageArgs<T> &a, long long i, double &ms_i) {
    ms_i = a.ms_map ? a.ms_map[i] : a.ms;
    return (!a.mask || a.mask[i] != 0) && (ms_i > 0.0);
}

template <typename T, int MODE>
__global__ void __launch_bounds__(256) k_stage(StageArgs<T> a) {
    double acc[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) acc[q] = 0.0;
    const long long n = a.n;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const long long sxy = (long long)nx * ny;
    const T *mx = a.m, *my = a.m + n, *mz = a.m + 2 * n;
    const double s = a.t * a.ac_omega;
    const double sinv = (a.ac_omega != 0.0) ? sin(s) : 0.0;
    const double hx0 = a.has_ext ? a.hext[0] + a.hac[0] * sinv : 0.0;
    const double hx1 = a.has_ext ? a.hext[1] + a.hac[1] * sinv : 0.0;
    const double hx2 = a.has_ext ? a.hext[2] + a.hac[2] * sinv : 0.0;

    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        double ms_i;
        const bool act = st_active(a, i, ms_i);
        if (!act) {
            if (a.kout) { a.kout[i] = T(0); a.kout[n + i] = T(0); a.kout[2 * n + i] = T(0); }
            if (a.hex_out) { a.hex_out[i] = T(0); a.hex_out[n + i] = T(0); a.hex_out[2 * n + i] = T(0); }
            if (a.heff_out) { a.heff_out[i] = T(0); a.heff_out[n + i] = T(0); a.heff_out[2 * n + i] = T(0); }
            if (MODE == MODE_HEUN_CORR) {
                a.m0[i] = T(0); a.m0[n + i] = T(0); a.m0[2 * n + i] = T(0);
            }
            continue;
        }
        const int z = (int)(i / sxy);
        const long long rem = i - (long long)z * sxy;
        const int y = (int)(rem / nx);
        const int x = (int)(rem - (long long)y * nx);
        // arithmetic in FP64 from the stored values (FP64 or FP32)
        using R = double;
        const R cx_ = mx[i], cy_ = my[i], cz_ = mz[i];
        R h0 = 0.0, h1 = 0.0, h2 = 0.0;  // exchange field
        long long nb[6];
        nb[0] = x < nx - 1 ? i + 1 : i;      // xp
        nb[1] = x > 0 ? i - 1 : i;           // xm
        nb[2] = y < ny - 1 ? i + nx : i;     // yp
        nb[3] = y > 0 ? i - nx : i;          // ym
        nb[4] = z < nz - 1 ? i + sxy : i;    // zp
        nb[5] = z > 0 ? i - sxy : i;         // zm
        if (a.mask || a.ms_map) {
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                double msq;
                if (!st_active(a, nb[q], msq)) nb[q] = i;
            }
        }
        if (a.enable_exchange) {
            const R ix2 = a.dinv[0], iy2 = a.dinv[1], iz2 = a.dinv[2];
            if (!a.region) {
                const R pref = 2.0 * a.aex / (kMu0 * ms_i);
                const R lx = ((R)mx[nb[0]] - 2.0 * cx_ + (R)mx[nb[1]]) * ix2 +
                             ((R)mx[nb[2]] - 2.0 * cx_ + (R)mx[nb[3]]) * iy2 +
                             ((R)mx[nb[4]] - 2.0 * cx_ + (R)mx[nb[5]]) * iz2;
                const R ly = ((R)my[nb[0]] - 2.0 * cy_ + (R)my[nb[1]]) * ix2 +
                             ((R)my[nb[2]] - 2.0 * cy_ + (R)my[nb[3]]) * iy2 +
                             ((R)my[nb[4]] - 2.0 * cy_ + (R)my[nb[5]]) * iz2;
                const R lz = ((R)mz[nb[0]] - 2.0 * cz_ + (R)mz[nb[1]]) * ix2 +
                             ((R)mz[nb[2]] - 2.0 * cz_ + (R)mz[nb[3]]) * iy2 +
                             ((R)mz[nb[4]] - 2.0 * cz_ + (R)mz[nb[5]]) * iz2;
                h0 = lx * pref; h1 = ly * pref; h2 = lz * pref;
            } else {
                const R pref = 2.0 / (kMu0 * ms_i);
                const uint32_t rc = a.region[i];
                const R inv[3] = {ix2, iy2, iz2};
                R sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll
                for (int q = 0; q < 6; ++q) {
                    const R aq = a.lut[(size_t)rc * 256 + a.region[nb[q]]];
                    sx += aq * ((R)mx[nb[q]] - cx_) * inv[q >> 1];
                    sy += aq * ((R)my[nb[q]] - cy_) * inv[q >> 1];
                    sz += aq * ((R)mz[nb[q]] - cz_) * inv[q >> 1];
                }
                h0 = pref * sx; h1 = pref * sy; h2 = pref * sz;
            }
        }
        R d0 = 0.0, d1 = 0.0, d2 = 0.0;
        if (a.enable_demag) { d0 = a.hd[i]; d1 = a.hd[n + i]; d2 = a.hd[2 * n + i]; }
        const R e0 = (h0 + d0) + hx0, e1 = (h1 + d1) + hx1, e2 = (h2 + d2) + hx2;
        // Gilbert RHS: -gamma_bar (m x H + alpha m x (m x H))
        const R p0 = cy_ * e2 - cz_ * e1, p1 = cz_ * e0 - cx_ * e2, p2 = cx_ * e1 - cy_ * e0;
        const R q0 = cy_ * p2 - cz_ * p1, q1 = cz_ * p0 - cx_ * p2, q2 = cx_ * p1 - cy_ * p0;
        const R al = a.alpha, gb = -a.gamma_bar;
        const R pr = a.precession ? 1.0 : 0.0;
        const R r0 = (pr * p0 + q0 * al) * gb, r1 = (pr * p1 + q1 * al) * gb,
                r2 = (pr * p2 + q2 * al) * gb;
        if (a.kout) { a.kout[i] = (T)r0; a.kout[n + i] = (T)r1; a.kout[2 * n + i] = (T)r2; }
        if (a.hex_out) { a.hex_out[i] = (T)h0; a.hex_out[n + i] = (T)h1; a.hex_out[2 * n + i] = (T)h2; }
        if (a.heff_out) { a.heff_out[i] = (T)e0; a.heff_out[n + i] = (T)e1; a.heff_out[2 * n + i] = (T)e2; }

        if (MODE == MODE_HEUN_CORR) {
            // m = normalize(m0 + (k1 + k2) * (dt/2)), FP64 accumulation
            const double hd_ = a.half_dt;
            const double v0 = (double)a.m0[i] + ((double)a.k1[i] + r0) * hd_;
            const double v1 = (double)a.m0[n + i] + ((double)a.k1[n + i] + r1) * hd_;
            const double v2 = (double)a.m0[2 * n + i] + ((double)a.k1[2 * n + i] + r2) * hd_;
            const double nn = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
            const double inv = nn > 0.0 ? 1.0 / nn : 0.0;
            a.m0[i] = (T)(v0 * inv); a.m0[n + i] = (T)(v1 * inv); a.m0[2 * n + i] = (T)(v2 * inv);
        }
        if (a.partials) {
            if (MODE == MODE_DP45_LAST) {
                // err = dt * (E1 k1 + E3 k3 + E4 k4 + E5 k5 + E6 k6 + E7 k7), lib.rs:1653-1674
                const double E[6] = {71.0 / 57600.0, -71.0 / 16695.0, 71.0 / 1920.0,
                                     -17253.0 / 339200.0, 22.0 / 525.0, -1.0 / 40.0};
                double er[3] = {0.0, 0.0, 0.0};
                // the stored k7 (rounded to T) enters the error like the other stages
                const double rr[3] = {(double)(T)r0, (double)(T)r1, (double)(T)r2};
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    double e = 0.0;
#pragma unroll
                    for (int s = 0; s < 5; ++s) e += E[s] * (double)a.ke[s][c * n + i];
                    e += E[5] * rr[c];
                    er[c] = e * a.dt;
                }
                acc[Q_ERR2] = fmax(acc[Q_ERR2], er[0] * er[0] + er[1] * er[1] + er[2] * er[2]);
            }
            const double m0d = (double)cx_, m1d = (double)cy_, m2d = (double)cz_;
            if (a.enable_exchange) {
                // forward pairs (x+1, y+1, z+1) inside the grid, both active
                const long long fw[3] = {x + 1 < nx ? i + 1 : -1, y + 1 < ny ? i + nx : -1,
                                         z + 1 < nz ? i + sxy : -1};
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    const long long j = fw[q];
                    if (j < 0) continue;
                    double msj;
                    if (!st_active(a, j, msj)) continue;
                    const double coeff = a.region ? a.lut[(size_t)a.region[i] * 256 + a.region[j]] * a.vol
                                                  : a.aex * a.vol;
                    const double dx_ = (double)mx[j] - m0d, dy_ = (double)my[j] - m1d,
                                 dz_ = (double)mz[j] - m2d;
                    acc[Q_EEX] += coeff * (dx_ * dx_ + dy_ * dy_ + dz_ * dz_) * a.dinv[q];
                }
            }
            const double coef = ms_i * a.vol * kMu0;
            acc[Q_EDEMAG] += -0.5 * coef * (m0d * (double)d0 + m1d * (double)d1 + m2d * (double)d2);
            acc[Q_EEXT] += -coef * (m0d * hx0 + m1d * hx1 + m2d * hx2);
            const double E0 = e0, E1 = e1, E2 = e2;
            acc[Q_HEFF2] = fmax(acc[Q_HEFF2], E0 * E0 + E1 * E1 + E2 * E2);
            const double D0 = d0, D1 = d1, D2 = d2;
            acc[Q_HD2] = fmax(acc[Q_HD2], D0 * D0 + D1 * D1 + D2 * D2);
            const double R0 = r0, R1 = r1, R2 = r2;
            acc[Q_RHS2] = fmax(acc[Q_RHS2], R0 * R0 + R1 * R1 + R2 * R2);
        }
    }
    if (a.partials) block_reduce_store(acc, a.partials);
}

// m_out = normalize(m0 + sum_j c_j k_j) in the reference's per-stage order.
// `form` selects the grouping used by crates/fullmag-engine/src/lib.rs:1418-1520:
//   0: m0 + k1*(c0)                     (Heun predictor: c0 = dt; DP45 stage 2: A21*dt)
//   1: m0 + (k1 c0 + k2 c1) dt
//   2: m0 + ((k1 c0 + k2 c1) + k3 c2) dt
//   3: m0 + ((k1 c0 + k2 c1) + (k3 c2 + k4 c3)) dt
//   4: m0 + (((k1 c0 + k2 c1) + k3 c2) + (k4 c3 + k5 c4)) dt
template <typename T>
struct CombineArgs {
    long long n;
    const T *m0;
    const T *k[5];
    double c[5];
    double dt;
    int form;
    T *out;
    const uint8_t *mask;
    const double *ms_map;
};

template <typename T>
__global__ void __launch_bounds__(256) k_combine(CombineArgs<T> a) {
    const long long n = a.n;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        double v[3];
#pragma unroll
        for (int comp = 0; comp < 3; ++comp) {
            const long long o = comp * n + i;
            double inc;
            switch (a.form) {
                case 0: inc = (double)a.k[0][o] * a.c[0]; break;
                case 1: inc = ((double)a.k[0][o] * a.c[0] + (double)a.k[1][o] * a.c[1]) * a.dt; break;
                case 2:
                    inc = (((double)a.k[0][o] * a.c[0] + (double)a.k[1][o] * a.c[1]) +
                           (double)a.k[2][o] * a.c[2]) * a.dt;
                    break;
                case 3:
                    inc = (((double)a.k[0][o] * a.c[0] + (double)a.k[1][o] * a.c[1]) +
                           ((double)a.k[2][o] * a.c[2] + (double)a.k[3][o] * a.c[3])) * a.dt;
                    break;
                default:
                    inc = ((((double)a.k[0][o] * a.c[0] + (double)a.k[1][o] * a.c[1]) +
                            (double)a.k[2][o] * a.c[2]) +
                           ((double)a.k[3][o] * a.c[3] + (double)a.k[4][o] * a.c[4])) * a.dt;
                    break;
            }
            v[comp] = (double)a.m0[o] + inc;
        }
        const double nn = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        const double inv = nn > 0.0 ? 1.0 / nn : 0.0;
        a.out[i] = (T)(v[0] * inv);
        a.out[n + i] = (T)(v[1] * inv);
        a.out[2 * n + i] = (T)(v[2] * inv);
    }
}

// Deterministic final reduction of the per-block partials: one block.
__global__ void __launch_bounds__(256) k_finalize(const double *partials, int nblocks, double *out) {
    __shared__ double sred[32];
    for (int q = 0; q < NQ; ++q) {
        const bool mx = q_is_max(q);
        double v = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
            const double w = partials[(long long)q * nblocks + b];
            v = mx ? fmax(v, w) : v + w;
        }
        v = warp_reduce(v, mx);
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
        if (lane == 0) sred[warp] = v;
        __syncthreads();
        if (warp == 0) {
            double w = lane < nw ? sred[lane] : 0.0;
            w = warp_reduce(w, mx);
            if (lane == 0) out[q] = w;
        }
        __syncthreads();
    }
}

}  // namespace fm
