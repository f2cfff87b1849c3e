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
#include "cpasync.cuh"

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
    MODE_ERR_LAST = 2,    // k_last = RHS(y); diagnostics + embedded error norm (DP45, RK23)
};

template <typename T>
struct StageArgs {
    int nx, ny, nz;
    long long n;
    T idx2, idy2, idz2;             // 1/dx^2, 1/dy^2, 1/dz^2
    double dinv[3];                 // same, FP64 (energies)
    double aex, ms;                 // uniform A and Ms
    double ex_pref;                 // 2 A / (mu0 Ms) for the uniform material
    double ex_pref_lut;             // 2 / (mu0 Ms) for the uniform material (region LUT)
    const double *ms_map;           // optional per-cell Ms
    const uint8_t *mask;            // optional
    const uint32_t *region;         // optional
    const double *lut;              // 256 x 256, with region
    int ex_tier;                    // boundary tiers: 0 standard, 1 T0 face links, 2 T1 ECB stencil
    const double *vf;               // volume fraction [n] (tiers)
    const double *face;             // [6][n] face link fractions xp, xm, yp, ym, zp, zm (T0)
    const double *delta;            // [6][n] boundary distances, same order (T1)
    double phi_floor, delta_min;
    double cell[3];                 // dx, dy, dz
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
    double *partials;               // [NQ][blocks] or null (then no diagnostics)
    unsigned *counter;              // blocks finished (last block reduces; reset to 0)
    double *out;                    // [NQ] final diagnostics
    // MODE_HEUN_CORR
    T *m0;                          // in: m0; out: corrected m (same buffer)
    const T *k1;
    double half_dt;
    // MODE_ERR_LAST: err = dt (sum_j ew[j] ke[j] + ew[nke] k_last), accumulated
    // from zero in that order (max_error_norm_buf, lib.rs:1653-1674)
    const T *ke[5];
    double ew[6];
    int nke;
    double dt;
    // MODE_EVAL: also the next Heun predictor normalize(m + k dt) with the stored
    // k, the arithmetic of k_combine form 0 (null: not written)
    T *pred_out;
    double pred_dt;
};

__device__ __forceinline__ double warp_reduce(double v, bool is_max) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double w = __shfl_down_sync(0xffffffffu, v, o);
        v = is_max ? fmax(v, w) : v + w;
    }
    return v;
}

template <typename T>
__device__ __forceinline__ bool st_active(const StageArgs<T> &a, long long i, double &ms_i) {
    ms_i = a.ms_map ? a.ms_map[i] : a.ms;
    return (!a.mask || a.mask[i] != 0) && (ms_i > 0.0);
}

// The next Heun predictor of cell i from the state c (its stored values) and
// k (as stored in T): normalize(m + k dt), the arithmetic of k_combine form 0.
template <typename T>
__device__ __forceinline__ void store_predictor(const StageArgs<T> &a, size_t i, size_t n, const double (&c)[3],
                                                double r0, double r1, double r2) {
    // one explicit fused multiply-add, as every predictor site of the library
    // (the stage kernels and combine form 0), so that all give the same bits
    const double v0 = __fma_rn((double)(T)r0, a.pred_dt, c[0]);
    const double v1 = __fma_rn((double)(T)r1, a.pred_dt, c[1]);
    const double v2 = __fma_rn((double)(T)r2, a.pred_dt, c[2]);
    const double n2 = v0 * v0 + v1 * v1 + v2 * v2;
    double inv;
    if (sizeof(T) == 8) {
        const double nn = sqrt(n2);
        inv = nn > 0.0 ? 1.0 / nn : 0.0;
    } else {
        inv = n2 > 0.0 ? rsqrt(n2) : 0.0;
    }
    a.pred_out[i] = (T)(v0 * inv);
    a.pred_out[n + i] = (T)(v1 * inv);
    a.pred_out[2 * n + i] = (T)(v2 * inv);
}

// Exchange field of the boundary tiers at an active cell i = (x, y, z) with
// m = c.  T0 (exchange_t0_fp64.cu:22-133): sum over the faces -x, +x, -y, +y,
// -z, +z inside the grid of f (m_j - c) / d^2 with face link f > 0, times
// 2A / (mu0 Ms) / max(phi, phi_floor).  T1 (exchange_t1_fp64.cu:28-175): per
// neighbour with non-zero m, 2 (m_j - c) / (d (d + delta_opposite)), deltas
// clamped below by delta_min, times 2A / (mu0 Ms).  The z faces are skipped for
// nz = 1; cells with phi <= 0 or m = 0 get zero (the reference leaves them
// unwritten).
template <typename T>
__device__ __forceinline__ void tier_exchange(const StageArgs<T> &a, long long i, int x, int y, int z,
                                              const double (&c)[3], double (&h)[3]) {
    h[0] = h[1] = h[2] = 0.0;
    const double phi0 = a.vf[i];
    if (phi0 <= 0.0 || (c[0] == 0.0 && c[1] == 0.0 && c[2] == 0.0)) return;
    const long long n = a.n;
    const int xyz[3] = {x, y, z}, ext[3] = {a.nx, a.ny, a.nz};
    const long long str[3] = {1, a.nx, (long long)a.nx * a.ny};
    double b[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        if (ax == 2 && a.nz <= 1) break;
        const bool has_m = xyz[ax] > 0, has_p = xyz[ax] + 1 < ext[ax];
        const double d = a.cell[ax];
        if (a.ex_tier == 1) {
            const double fm = a.face[(2 * ax + 1) * n + i], fp = a.face[2 * ax * n + i];
            const double inv = a.dinv[ax];
            if (fm > 0.0 && has_m) {
                const long long j = i - str[ax];
#pragma unroll
                for (int k = 0; k < 3; ++k) b[k] += fm * inv * ((double)a.m[k * n + j] - c[k]);
            }
            if (fp > 0.0 && has_p) {
                const long long j = i + str[ax];
#pragma unroll
                for (int k = 0; k < 3; ++k) b[k] += fp * inv * ((double)a.m[k * n + j] - c[k]);
            }
        } else {
            const double dm = fmax(a.delta[(2 * ax + 1) * n + i], a.delta_min);
            const double dp = fmax(a.delta[2 * ax * n + i], a.delta_min);
            if (has_m && dm > 0.0) {
                const long long j = i - str[ax];
                const double mn[3] = {(double)a.m[j], (double)a.m[n + j], (double)a.m[2 * n + j]};
                if (mn[0] != 0.0 || mn[1] != 0.0 || mn[2] != 0.0) {
                    const double coeff = 2.0 / (d * (d + dp));
#pragma unroll
                    for (int k = 0; k < 3; ++k) b[k] += coeff * (mn[k] - c[k]);
                }
            }
            if (has_p && dp > 0.0) {
                const long long j = i + str[ax];
                const double mn[3] = {(double)a.m[j], (double)a.m[n + j], (double)a.m[2 * n + j]};
                if (mn[0] != 0.0 || mn[1] != 0.0 || mn[2] != 0.0) {
                    const double coeff = 2.0 / (d * (d + dm));
#pragma unroll
                    for (int k = 0; k < 3; ++k) b[k] += coeff * (mn[k] - c[k]);
                }
            }
        }
    }
    double sc = 2.0 * a.aex / (kMu0 * a.ms);
    if (a.ex_tier == 1) sc = sc * (1.0 / (phi0 > a.phi_floor ? phi0 : a.phi_floor));
#pragma unroll
    for (int k = 0; k < 3; ++k) h[k] = sc * b[k];
}

// Reduce acc[NQ] over the block and, in the last block to finish, over all
// blocks' partials in a fixed order (deterministic), writing out[NQ].
__device__ __forceinline__ void block_reduce_final(double (&acc)[NQ], double *partials,
                                                   unsigned *counter, double *out) {
    __shared__ double sred[NQ][32];
    __shared__ bool am_last;
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthr = blockDim.x * blockDim.y * blockDim.z;
    const int lane = tid & 31, warp = tid >> 5, nw = (nthr + 31) >> 5;
    const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    const int nblocks = gridDim.x * gridDim.y * gridDim.z;
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
            if (lane == 0) partials[(long long)q * nblocks + bid] = v;
        }
    }
    if (tid == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(counter, 1u);
        am_last = (prev == (unsigned)nblocks - 1);
    }
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    for (int q = 0; q < NQ; ++q) {
        const bool mx = q_is_max(q);
        const double *pq = partials + (long long)q * nblocks;
        // four independent accumulators per thread, combined in a fixed order
        double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
        int b = tid;
        for (; b + 3 * nthr < nblocks; b += 4 * nthr) {
            const double w0 = __ldcg(pq + b), w1 = __ldcg(pq + b + nthr);
            const double w2 = __ldcg(pq + b + 2 * nthr), w3 = __ldcg(pq + b + 3 * nthr);
            v0 = mx ? fmax(v0, w0) : v0 + w0;
            v1 = mx ? fmax(v1, w1) : v1 + w1;
            v2 = mx ? fmax(v2, w2) : v2 + w2;
            v3 = mx ? fmax(v3, w3) : v3 + w3;
        }
        for (; b < nblocks; b += nthr) {
            const double w = __ldcg(pq + b);
            v0 = mx ? fmax(v0, w) : v0 + w;
        }
        double v = mx ? fmax(fmax(v0, v1), fmax(v2, v3)) : (v0 + v1) + (v2 + v3);
        v = warp_reduce(v, mx);
        __syncthreads();
        if (lane == 0) sred[0][warp] = v;
        __syncthreads();
        if (warp == 0) {
            double w = lane < nw ? sred[0][lane] : 0.0;
            w = warp_reduce(w, mx);
            if (lane == 0) out[q] = w;
        }
    }
    if (tid == 0) *counter = 0u;
}

// One thread per cell; block (32, 4, 2), grid (ceil(nx/32), ceil(ny/4),
// ceil(nz/2)).  x/y neighbours mostly hit L1, z neighbours L2; many small
// independent threads keep enough loads in flight to stream HBM.
template <typename T, int MODE>
__global__ void __launch_bounds__(256, 3) k_stage(StageArgs<T> a) {
    using R = double;
    double acc[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) acc[q] = 0.0;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const long long n = a.n;
    const long long sxy = (long long)nx * ny;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    const T *mx = a.m, *my = a.m + n, *mz = a.m + 2 * n;
    const bool masked = a.mask || a.ms_map;

    if (x < nx && y < ny && z < nz) {
        const long long i = ((long long)z * ny + y) * nx + x;
        double ms_i;
        if (!st_active(a, i, ms_i)) {
            if (a.kout) { a.kout[i] = T(0); a.kout[n + i] = T(0); a.kout[2 * n + i] = T(0); }
            if (a.hex_out) { a.hex_out[i] = T(0); a.hex_out[n + i] = T(0); a.hex_out[2 * n + i] = T(0); }
            if (a.heff_out) { a.heff_out[i] = T(0); a.heff_out[n + i] = T(0); a.heff_out[2 * n + i] = T(0); }
            if (MODE == MODE_HEUN_CORR) { a.m0[i] = T(0); a.m0[n + i] = T(0); a.m0[2 * n + i] = T(0); }
            if (MODE == MODE_EVAL && a.pred_out) {
                const double c0[3] = {(double)mx[i], (double)my[i], (double)mz[i]};
                store_predictor(a, (size_t)i, (size_t)n, c0, 0.0, 0.0, 0.0);
            }
        } else {
            // neighbours: clamped at the grid edge, inactive -> centre (lib.rs:2255-2286)
            long long nb[6];
            nb[0] = x < nx - 1 ? i + 1 : i;     // xp
            nb[1] = x > 0 ? i - 1 : i;          // xm
            nb[2] = y < ny - 1 ? i + nx : i;    // yp
            nb[3] = y > 0 ? i - nx : i;         // ym
            nb[4] = z < nz - 1 ? i + sxy : i;   // zp
            nb[5] = z > 0 ? i - sxy : i;        // zm
            if (masked) {
#pragma unroll
                for (int q = 0; q < 6; ++q) {
                    double msq;
                    if (!st_active(a, nb[q], msq)) nb[q] = i;
                }
            }
            const R c3[3] = {(R)mx[i], (R)my[i], (R)mz[i]};
            const T *comp[3] = {mx, my, mz};
            R hxc[3] = {0.0, 0.0, 0.0};
            if (a.enable_exchange) {
                const R ix2 = a.dinv[0], iy2 = a.dinv[1], iz2 = a.dinv[2];
                if (a.ex_tier) {
                    tier_exchange(a, i, x, y, z, c3, hxc);
                } else if (!a.region) {
                    const R pref = a.ms_map ? 2.0 * a.aex / (kMu0 * ms_i) : a.ex_pref;
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const T *f = comp[c];
                        const R lap = ((R)f[nb[0]] - 2.0 * c3[c] + (R)f[nb[1]]) * ix2 +
                                      ((R)f[nb[2]] - 2.0 * c3[c] + (R)f[nb[3]]) * iy2 +
                                      ((R)f[nb[4]] - 2.0 * c3[c] + (R)f[nb[5]]) * iz2;
                        hxc[c] = lap * pref;
                    }
                } else {
                    const R pref = a.ms_map ? 2.0 / (kMu0 * ms_i) : a.ex_pref_lut;
                    const uint32_t rc = a.region[i];
                    R aq[6];
#pragma unroll
                    for (int q = 0; q < 6; ++q) aq[q] = a.lut[(size_t)rc * 256 + a.region[nb[q]]];
                    const R inv[3] = {ix2, iy2, iz2};
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        // order of exchange_fp64.cu:102-112: xp, xm, yp, ym, zp, zm
                        const T *f = comp[c];
                        R sm = 0.0;
#pragma unroll
                        for (int q = 0; q < 6; ++q) sm += aq[q] * ((R)f[nb[q]] - c3[c]) * inv[q >> 1];
                        hxc[c] = pref * sm;
                    }
                }
            }
            const double sinv = (a.ac_omega != 0.0) ? sin(a.t * a.ac_omega) : 0.0;
            const R hx0 = a.has_ext ? a.hext[0] + a.hac[0] * sinv : 0.0;
            const R hx1 = a.has_ext ? a.hext[1] + a.hac[1] * sinv : 0.0;
            const R hx2 = a.has_ext ? a.hext[2] + a.hac[2] * sinv : 0.0;
            const R cx_ = c3[0], cy_ = c3[1], cz_ = c3[2];
            const R h0 = hxc[0], h1 = hxc[1], h2 = hxc[2];
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
            if (MODE == MODE_EVAL && a.pred_out) store_predictor(a, (size_t)i, (size_t)n, c3, r0, r1, r2);
            if (a.hex_out) { a.hex_out[i] = (T)h0; a.hex_out[n + i] = (T)h1; a.hex_out[2 * n + i] = (T)h2; }
            if (a.heff_out) { a.heff_out[i] = (T)e0; a.heff_out[n + i] = (T)e1; a.heff_out[2 * n + i] = (T)e2; }
            if (MODE == MODE_HEUN_CORR) {
                // m = normalize(m0 + (k1 + k2) * (dt/2)), FP64 accumulation
                const double hd_ = a.half_dt;
                const double v0 = (double)a.m0[i] + ((double)a.k1[i] + r0) * hd_;
                const double v1 = (double)a.m0[n + i] + ((double)a.k1[n + i] + r1) * hd_;
                const double v2 = (double)a.m0[2 * n + i] + ((double)a.k1[2 * n + i] + r2) * hd_;
                const double n2 = v0 * v0 + v1 * v1 + v2 * v2;
                double inv;
                if (sizeof(T) == 8) {
                    const double nn = sqrt(n2);  // FP64 path: 1/sqrt rounded like the reference
                    inv = nn > 0.0 ? 1.0 / nn : 0.0;
                } else {
                    inv = n2 > 0.0 ? rsqrt(n2) : 0.0;  // result is stored in FP32
                }
                a.m0[i] = (T)(v0 * inv); a.m0[n + i] = (T)(v1 * inv); a.m0[2 * n + i] = (T)(v2 * inv);
            }
            if (a.partials) {
                if (MODE == MODE_ERR_LAST) {
                    // the stored last stage (rounded to T) enters the error like the others
                    const double rr[3] = {(double)(T)r0, (double)(T)r1, (double)(T)r2};
                    double er[3];
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        double e = 0.0;
                        for (int st = 0; st < a.nke; ++st) e += a.ew[st] * (double)a.ke[st][c * n + i];
                        e += a.ew[a.nke] * rr[c];
                        er[c] = e * a.dt;
                    }
                    acc[Q_ERR2] = fmax(acc[Q_ERR2], er[0] * er[0] + er[1] * er[1] + er[2] * er[2]);
                }
                if (a.enable_exchange) {
                    // forward pairs (x+1, y+1, z+1) inside the grid, both active
                    const bool has[3] = {x + 1 < nx, y + 1 < ny, z + 1 < nz};
                    const long long fw[3] = {i + 1, i + nx, i + sxy};
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        if (!has[q]) continue;
                        const long long j = fw[q];
                        double msj;
                        if (masked && !st_active(a, j, msj)) continue;
                        const double coeff = a.region ? a.lut[(size_t)a.region[i] * 256 + a.region[j]] * a.vol
                                                      : a.aex * a.vol;
                        const double ddx = (double)mx[j] - cx_, ddy = (double)my[j] - cy_,
                                     ddz = (double)mz[j] - cz_;
                        acc[Q_EEX] += coeff * (ddx * ddx + ddy * ddy + ddz * ddz) * a.dinv[q];
                    }
                }
                const double coef = ms_i * a.vol * kMu0;
                acc[Q_EDEMAG] += -0.5 * coef * (cx_ * d0 + cy_ * d1 + cz_ * d2);
                acc[Q_EEXT] += -coef * (cx_ * hx0 + cy_ * hx1 + cz_ * hx2);
                acc[Q_HEFF2] = fmax(acc[Q_HEFF2], e0 * e0 + e1 * e1 + e2 * e2);
                acc[Q_HD2] = fmax(acc[Q_HD2], d0 * d0 + d1 * d1 + d2 * d2);
                acc[Q_RHS2] = fmax(acc[Q_RHS2], r0 * r0 + r1 * r1 + r2 * r2);
            }
        }
    }
    if (a.partials) block_reduce_final(acc, a.partials, a.counter, a.out);
}

// ---------------------------------------------------------------------------
// Uniform material (no mask, no Ms map, no region LUT): the same per-cell
// arithmetic as k_stage, organised for instruction economy.  block
// (32, BY, 1): lane = x, threadIdx.y = y; each thread marches over the planes
// z in [z0, z0 + zb), keeping m at z-1, z, z+1 in registers, takes the x
// neighbours from the adjacent lanes by shuffles (the warp's edge lanes load
// theirs), loads the y neighbours (rows the adjacent warps also load) and the
// next plane's values one plane ahead, reuses the loaded neighbours for the
// forward-pair exchange energy, and reduces the diagnostics once per block.
// 32-bit cell indices (3 n < 2^32 is checked by the host).  Threads of cells
// outside the grid load the clamped edge cell and neither store nor
// accumulate, so every lane takes part in the shuffles.
// ---------------------------------------------------------------------------
constexpr int kStagePlainBY = 4;  // rows (warps) per block of k_stage_plain

template <typename T>
struct PlaneLoads {
    T up[3];   // m(x, y, z + 1)
    T yp[3];   // m(x, y + 1, z)
    T ym[3];   // m(x, y - 1, z)
    T hd[3];   // H_d(x, y, z)
};

// Cell-invariant values of the uniform-material stage kernels.
struct PlainConst {
    double ix2, iy2, iz2, pref, hx0, hx1, hx2, al, gb, pr, coef, pair;
};

template <typename T>
__device__ __forceinline__ PlainConst plain_const(const StageArgs<T> &a) {
    PlainConst k;
    k.ix2 = a.dinv[0]; k.iy2 = a.dinv[1]; k.iz2 = a.dinv[2];
    k.pref = a.ex_pref;
    const double sinv = (a.ac_omega != 0.0) ? sin(a.t * a.ac_omega) : 0.0;
    k.hx0 = a.has_ext ? a.hext[0] + a.hac[0] * sinv : 0.0;
    k.hx1 = a.has_ext ? a.hext[1] + a.hac[1] * sinv : 0.0;
    k.hx2 = a.has_ext ? a.hext[2] + a.hac[2] * sinv : 0.0;
    k.al = a.alpha; k.gb = -a.gamma_bar;
    k.pr = a.precession ? 1.0 : 0.0;
    k.coef = a.ms * a.vol * kMu0;
    k.pair = a.aex * a.vol;
    return k;
}

// Per-cell arithmetic of the uniform-material stage kernels, after the loads:
// cell i at plane z with m = c, m(z - 1) = dn, m(z + 1) = upT (only read when
// z + 1 < nz), x neighbours xpT / xmT (already the cell itself at the grid
// edge), y neighbours ypT / ymT (read only when they exist), H_d = hdT, and for
// the corrector m0v, k1v.  Stores the stage outputs and accumulates the
// diagnostics when inxy.
template <typename T, int MODE>
__device__ __forceinline__ void plain_cell(const StageArgs<T> &a, const PlainConst &k, unsigned i, unsigned n, int z,
                                           bool inxy, bool has_xp, bool has_yp, bool has_ym, const double (&c)[3],
                                           const double (&dn)[3], const T (&upT)[3], const T (&xpT)[3],
                                           const T (&xmT)[3], const T (&ypT)[3], const T (&ymT)[3],
                                           const T (&hdT)[3], const T (&m0v)[3], const T (&k1v)[3],
                                           double (&acc)[NQ]) {
    using R = double;
    const int nz = a.nz;
    const bool ex = a.enable_exchange;
    R up[3] = {(R)upT[0], (R)upT[1], (R)upT[2]};
    if (z + 1 >= nz) { up[0] = c[0]; up[1] = c[1]; up[2] = c[2]; }
    R h[3] = {0.0, 0.0, 0.0};
    R yp[3], xp[3];
    if (ex) {
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            xp[q] = (R)xpT[q];
            yp[q] = has_yp ? (R)ypT[q] : c[q];
            const R ym = has_ym ? (R)ymT[q] : c[q];
            const R lap = (xp[q] - 2.0 * c[q] + (R)xmT[q]) * k.ix2 + (yp[q] - 2.0 * c[q] + ym) * k.iy2 +
                          (up[q] - 2.0 * c[q] + dn[q]) * k.iz2;
            h[q] = lap * k.pref;
        }
    }
    const R d0 = hdT[0], d1 = hdT[1], d2 = hdT[2];
    const R e0 = (h[0] + d0) + k.hx0, e1 = (h[1] + d1) + k.hx1, e2 = (h[2] + d2) + k.hx2;
    const R cx_ = c[0], cy_ = c[1], cz_ = c[2];
    const R p0 = cy_ * e2 - cz_ * e1, p1 = cz_ * e0 - cx_ * e2, p2 = cx_ * e1 - cy_ * e0;
    const R q0 = cy_ * p2 - cz_ * p1, q1 = cz_ * p0 - cx_ * p2, q2 = cx_ * p1 - cy_ * p0;
    const R r0 = (k.pr * p0 + q0 * k.al) * k.gb, r1 = (k.pr * p1 + q1 * k.al) * k.gb,
            r2 = (k.pr * p2 + q2 * k.al) * k.gb;
    if (!inxy) return;
    if (a.kout) { a.kout[i] = (T)r0; a.kout[n + i] = (T)r1; a.kout[2 * (size_t)n + i] = (T)r2; }
    if (MODE == MODE_EVAL && a.pred_out) store_predictor(a, (size_t)i, (size_t)n, c, r0, r1, r2);
    if (a.hex_out) { a.hex_out[i] = (T)h[0]; a.hex_out[n + i] = (T)h[1]; a.hex_out[2 * (size_t)n + i] = (T)h[2]; }
    if (a.heff_out) { a.heff_out[i] = (T)e0; a.heff_out[n + i] = (T)e1; a.heff_out[2 * (size_t)n + i] = (T)e2; }
    if (MODE == MODE_HEUN_CORR) {
        const double hd_ = a.half_dt;
        const double v0 = (double)m0v[0] + ((double)k1v[0] + r0) * hd_;
        const double v1 = (double)m0v[1] + ((double)k1v[1] + r1) * hd_;
        const double v2 = (double)m0v[2] + ((double)k1v[2] + r2) * hd_;
        const double n2 = v0 * v0 + v1 * v1 + v2 * v2;
        double inv;
        if (sizeof(T) == 8) {
            const double nn = sqrt(n2);
            inv = nn > 0.0 ? 1.0 / nn : 0.0;
        } else {
            inv = n2 > 0.0 ? rsqrt(n2) : 0.0;
        }
        a.m0[i] = (T)(v0 * inv); a.m0[n + i] = (T)(v1 * inv); a.m0[2 * (size_t)n + i] = (T)(v2 * inv);
    }
    if (a.partials) {
        if (MODE == MODE_ERR_LAST) {
            const double rr[3] = {(double)(T)r0, (double)(T)r1, (double)(T)r2};
            double er[3];
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                double e = 0.0;
                for (int st = 0; st < a.nke; ++st) e += a.ew[st] * (double)a.ke[st][q * (size_t)n + i];
                e += a.ew[a.nke] * rr[q];
                er[q] = e * a.dt;
            }
            acc[Q_ERR2] = fmax(acc[Q_ERR2], er[0] * er[0] + er[1] * er[1] + er[2] * er[2]);
        }
        if (ex) {
            // forward pairs (x+1, y+1, z+1) inside the grid, from the loaded neighbours
            if (has_xp) {
                const double ddx = xp[0] - cx_, ddy = xp[1] - cy_, ddz = xp[2] - cz_;
                acc[Q_EEX] += k.pair * (ddx * ddx + ddy * ddy + ddz * ddz) * a.dinv[0];
            }
            if (has_yp) {
                const double ddx = yp[0] - cx_, ddy = yp[1] - cy_, ddz = yp[2] - cz_;
                acc[Q_EEX] += k.pair * (ddx * ddx + ddy * ddy + ddz * ddz) * a.dinv[1];
            }
            if (z + 1 < nz) {
                const double ddx = up[0] - cx_, ddy = up[1] - cy_, ddz = up[2] - cz_;
                acc[Q_EEX] += k.pair * (ddx * ddx + ddy * ddy + ddz * ddz) * a.dinv[2];
            }
        }
        acc[Q_EDEMAG] += -0.5 * k.coef * (cx_ * d0 + cy_ * d1 + cz_ * d2);
        acc[Q_EEXT] += -k.coef * (cx_ * k.hx0 + cy_ * k.hx1 + cz_ * k.hx2);
        acc[Q_HEFF2] = fmax(acc[Q_HEFF2], e0 * e0 + e1 * e1 + e2 * e2);
        acc[Q_HD2] = fmax(acc[Q_HD2], d0 * d0 + d1 * d1 + d2 * d2);
        acc[Q_RHS2] = fmax(acc[Q_RHS2], r0 * r0 + r1 * r1 + r2 * r2);
    }
}

// Block body (bx, by, bz); the diagnostics accumulate into acc.  Also run per
// work item by the batched kernels (batch.cuh).
template <typename T, int MODE>
__device__ __forceinline__ void stage_plain_body(const StageArgs<T> &a, int zb, int bx, int by, int bz,
                                                 double (&acc)[NQ]) {
    using R = double;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const unsigned n = (unsigned)a.n, sxy = (unsigned)nx * (unsigned)ny;
    const int lane = threadIdx.x;
    const int x = bx * 32 + lane, y = by * blockDim.y + threadIdx.y;
    const int z0 = bz * zb, z1 = min(z0 + zb, nz);
    const bool inxy = x < nx && y < ny;
    const int xc = min(x, nx - 1), yc = min(y, ny - 1);
    const T *f0 = a.m, *f1 = a.m + n, *f2 = a.m + 2 * (size_t)n;
    const bool has_xp = x + 1 < nx, has_xm = x > 0, has_yp = yc + 1 < ny, has_ym = yc > 0;
    const bool ex = a.enable_exchange, dm = a.enable_demag;
    auto ld3 = [&](unsigned j, T (&v)[3]) { v[0] = f0[j]; v[1] = f1[j]; v[2] = f2[j]; };
    auto load_plane = [&](int z, unsigned j, PlaneLoads<T> &L) {
        if (z + 1 < nz) ld3(j + sxy, L.up); else { L.up[0] = f0[j]; L.up[1] = f1[j]; L.up[2] = f2[j]; }
        if (ex) {
            if (has_yp) ld3(j + nx, L.yp);
            if (has_ym) ld3(j - nx, L.ym);
        }
        if (dm) { L.hd[0] = a.hd[j]; L.hd[1] = a.hd[n + j]; L.hd[2] = a.hd[2 * (size_t)n + j]; }
        else { L.hd[0] = T(0); L.hd[1] = T(0); L.hd[2] = T(0); }
    };
    const PlainConst k = plain_const(a);

    unsigned i = ((unsigned)z0 * (unsigned)ny + (unsigned)yc) * (unsigned)nx + (unsigned)xc;
    T cT[3];
    ld3(i, cT);
    R c[3] = {(R)cT[0], (R)cT[1], (R)cT[2]};
    R dn[3] = {c[0], c[1], c[2]};
    if (z0 > 0) { T t3[3]; ld3(i - sxy, t3); dn[0] = t3[0]; dn[1] = t3[1]; dn[2] = t3[2]; }
    PlaneLoads<T> L;
    load_plane(z0, i, L);
    for (int z = z0; z < z1; ++z, i += sxy) {
        PlaneLoads<T> Ln;
        if (z + 1 < z1) load_plane(z + 1, i + sxy, Ln);
        // the corrector's m0 and k1 of this cell, issued before the arithmetic
        T m0v[3] = {T(0), T(0), T(0)}, k1v[3] = {T(0), T(0), T(0)};
        if (MODE == MODE_HEUN_CORR && inxy) {
            m0v[0] = a.m0[i]; m0v[1] = a.m0[n + i]; m0v[2] = a.m0[2 * (size_t)n + i];
            k1v[0] = a.k1[i]; k1v[1] = a.k1[n + i]; k1v[2] = a.k1[2 * (size_t)n + i];
        }
        // x neighbours: adjacent lanes; the warp's edge lanes load theirs
        T xpT[3], xmT[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            xpT[q] = __shfl_down_sync(0xffffffffu, cT[q], 1);
            xmT[q] = __shfl_up_sync(0xffffffffu, cT[q], 1);
        }
        if (!has_xp) { xpT[0] = cT[0]; xpT[1] = cT[1]; xpT[2] = cT[2]; }
        else if (lane == 31) ld3(i + 1, xpT);
        if (!has_xm) { xmT[0] = cT[0]; xmT[1] = cT[1]; xmT[2] = cT[2]; }
        else if (lane == 0) ld3(i - 1, xmT);
        plain_cell<T, MODE>(a, k, i, n, z, inxy, has_xp, has_yp, has_ym, c, dn, L.up, xpT, xmT, L.yp, L.ym, L.hd,
                            m0v, k1v, acc);
        // advance one plane
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            dn[q] = c[q];
            cT[q] = (z + 1 < nz) ? L.up[q] : cT[q];
            c[q] = (R)cT[q];
        }
        L = Ln;
    }
}

// ---------------------------------------------------------------------------
// Uniform material, ring-fed: the body of stage_plain_body, but each thread
// copies the inputs of plane z + D - 1 (m above, the y neighbours, H_d, the
// warp-edge lane's outer x neighbour, and the corrector's m0 and k1) into its
// own D-slot shared-memory ring with cp.async while it computes plane z, so
// D - 1 planes of loads are in flight without holding registers.  A thread
// reads back only what it copied itself: no block barrier.  Ring layout
// [slot][item][thread], items of a slot:
//   0..2 up, 3..5 y+1, 6..8 y-1, 9..11 H_d, 12..14 outer x neighbour (lanes 0
//   and 31), 15..17 m0 and 18..20 k1 (corrector).
// ---------------------------------------------------------------------------
// Depth D and resident blocks per SM, chosen so that D x items x 128 threads of
// shared memory and the register budget allow that many blocks (measured).
template <int MODE> __host__ __device__ constexpr int ring_items() { return MODE == MODE_HEUN_CORR ? 21 : 15; }
template <typename T, int MODE> __host__ __device__ constexpr int ring_depth() {
    return sizeof(T) == 8 ? 2 : (MODE == MODE_HEUN_CORR ? 3 : 4);
}
template <typename T, int MODE> __host__ __device__ constexpr int ring_min_blocks() {
    return (sizeof(T) == 8 && MODE == MODE_HEUN_CORR) ? 4 : 5;
}
template <typename T, int MODE>
__host__ __device__ constexpr size_t ring_bytes(int threads) {
    return (size_t)ring_depth<T, MODE>() * ring_items<MODE>() * threads * sizeof(T);
}

template <typename T, int MODE>
__global__ void __launch_bounds__(128, ring_min_blocks<T, MODE>()) k_stage_ring(StageArgs<T> a, int zb) {
    using R = double;
    constexpr int D = ring_depth<T, MODE>(), NV = ring_items<MODE>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *ring = reinterpret_cast<T *>(smem_raw);
    double acc[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) acc[q] = 0.0;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const unsigned n = (unsigned)a.n, sxy = (unsigned)nx * (unsigned)ny;
    const int lane = threadIdx.x, BT = blockDim.x * blockDim.y, tid = lane + blockDim.x * threadIdx.y;
    const int x = blockIdx.x * 32 + lane, y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z0 = blockIdx.z * zb, z1 = min(z0 + zb, nz);
    const bool inxy = x < nx && y < ny;
    const int xc = min(x, nx - 1), yc = min(y, ny - 1);
    const T *f0 = a.m, *f1 = a.m + n, *f2 = a.m + 2 * (size_t)n;
    const bool has_xp = x + 1 < nx, has_xm = x > 0, has_yp = yc + 1 < ny, has_ym = yc > 0;
    const bool ex = a.enable_exchange, dm = a.enable_demag;
    const unsigned rbase = (unsigned)__cvta_generic_to_shared(ring + tid);
    auto item = [&](int z, int v) -> unsigned {  // shared address of item v of plane z's slot
        return rbase + (unsigned)((((z - z0) % D) * NV + v) * BT) * (unsigned)sizeof(T);
    };
    auto cp3 = [&](unsigned dst, const T *p0, const T *p1, const T *p2, unsigned j) {
        cp_async_elem<sizeof(T)>(dst, p0 + j);
        cp_async_elem<sizeof(T)>(dst + BT * (unsigned)sizeof(T), p1 + j);
        cp_async_elem<sizeof(T)>(dst + 2 * BT * (unsigned)sizeof(T), p2 + j);
    };
    const unsigned ic = (unsigned)yc * (unsigned)nx + (unsigned)xc;  // in-plane index
    auto issue = [&](int z) {
        const unsigned j = (unsigned)z * sxy + ic;
        if (z + 1 < nz) cp3(item(z, 0), f0, f1, f2, j + sxy);
        if (ex) {
            if (has_yp) cp3(item(z, 3), f0, f1, f2, j + nx);
            if (has_ym) cp3(item(z, 6), f0, f1, f2, j - nx);
            if (lane == 31 && has_xp) cp3(item(z, 12), f0, f1, f2, j + 1);
            if (lane == 0 && has_xm) cp3(item(z, 12), f0, f1, f2, j - 1);
        }
        if (dm) cp3(item(z, 9), a.hd, a.hd + n, a.hd + 2 * (size_t)n, j);
        if (MODE == MODE_HEUN_CORR && inxy) {
            cp3(item(z, 15), a.m0, a.m0 + n, a.m0 + 2 * (size_t)n, j);
            cp3(item(z, 18), a.k1, a.k1 + n, a.k1 + 2 * (size_t)n, j);
        }
    };
    const PlainConst k = plain_const(a);
    unsigned i = (unsigned)z0 * sxy + ic;
    T cT[3] = {f0[i], f1[i], f2[i]};
    R c[3] = {(R)cT[0], (R)cT[1], (R)cT[2]};
    R dn[3] = {c[0], c[1], c[2]};
    if (z0 > 0) { dn[0] = f0[i - sxy]; dn[1] = f1[i - sxy]; dn[2] = f2[i - sxy]; }
#pragma unroll
    for (int p = 0; p < D - 1; ++p) {
        if (z0 + p < z1) issue(z0 + p);
        cp_async_commit();
    }
    for (int z = z0; z < z1; ++z, i += sxy) {
        if (z + D - 1 < z1) issue(z + D - 1);
        cp_async_commit();    // possibly empty: the group D - 1 back is always plane z's
        cp_async_wait<D - 1>();
        const T *sl = ring + (((z - z0) % D) * NV) * BT + tid;
        auto rd3 = [&](int v, T (&o)[3]) { o[0] = sl[v * BT]; o[1] = sl[(v + 1) * BT]; o[2] = sl[(v + 2) * BT]; };
        T upT[3] = {cT[0], cT[1], cT[2]}, ypT[3] = {cT[0], cT[1], cT[2]}, ymT[3] = {cT[0], cT[1], cT[2]};
        T hdT[3] = {T(0), T(0), T(0)}, m0v[3] = {T(0), T(0), T(0)}, k1v[3] = {T(0), T(0), T(0)};
        if (z + 1 < nz) rd3(0, upT);
        if (ex) {
            if (has_yp) rd3(3, ypT);
            if (has_ym) rd3(6, ymT);
        }
        if (dm) rd3(9, hdT);
        if (MODE == MODE_HEUN_CORR && inxy) { rd3(15, m0v); rd3(18, k1v); }
        // x neighbours: adjacent lanes; the warp's edge lanes read their copy
        T xpT[3], xmT[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            xpT[q] = __shfl_down_sync(0xffffffffu, cT[q], 1);
            xmT[q] = __shfl_up_sync(0xffffffffu, cT[q], 1);
        }
        if (!has_xp) { xpT[0] = cT[0]; xpT[1] = cT[1]; xpT[2] = cT[2]; }
        else if (lane == 31 && ex) rd3(12, xpT);
        if (!has_xm) { xmT[0] = cT[0]; xmT[1] = cT[1]; xmT[2] = cT[2]; }
        else if (lane == 0 && ex) rd3(12, xmT);
        plain_cell<T, MODE>(a, k, i, n, z, inxy, has_xp, has_yp, has_ym, c, dn, upT, xpT, xmT, ypT, ymT, hdT, m0v,
                            k1v, acc);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            dn[q] = c[q];
            cT[q] = (z + 1 < nz) ? upT[q] : cT[q];
            c[q] = (R)cT[q];
        }
    }
    cp_async_wait_all();
    if (a.partials) block_reduce_final(acc, a.partials, a.counter, a.out);
}

template <typename T, int MODE>
__global__ void __launch_bounds__(128, 4) k_stage_plain(StageArgs<T> a, int zb) {
    double acc[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) acc[q] = 0.0;
    stage_plain_body<T, MODE>(a, zb, blockIdx.x, blockIdx.y, blockIdx.z, acc);
    if (a.partials) block_reduce_final(acc, a.partials, a.counter, a.out);
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
__device__ __forceinline__ void combine_cell(const CombineArgs<T> &a, long long i) {
    const long long n = a.n;
    {
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
            // form 0 is the predictor: one explicit fused multiply-add like the
            // stage kernels' predictor (store_predictor), the same bits
            v[comp] = a.form == 0 ? __fma_rn((double)a.k[0][o], a.c[0], (double)a.m0[o]) : (double)a.m0[o] + inc;
        }
        const double n2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        double inv;
        if (sizeof(T) == 8) {
            const double nn = sqrt(n2);
            inv = nn > 0.0 ? 1.0 / nn : 0.0;
        } else {
            inv = n2 > 0.0 ? rsqrt(n2) : 0.0;
        }
        a.out[i] = (T)(v[0] * inv);
        a.out[n + i] = (T)(v[1] * inv);
        a.out[2 * n + i] = (T)(v[2] * inv);
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_combine(CombineArgs<T> a) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n;
         i += (long long)gridDim.x * blockDim.x)
        combine_cell(a, i);
}

}  // namespace fm
