// demag_row.cuh — the x inverse of a demag evaluation, the stage arithmetic at
// that state and the x forward of the state it produces, fused per row slab
// (uniform material, power-of-two x length, register FFT path).
//
// Split, one field evaluation followed by a Heun stage is
//   x forward (state -> S1) | y / z passes (S1 -> S1) | x inverse (S1 -> H_d)
//   | stage (state, H_d -> k, next state)
// and the following evaluation begins with the x forward of the state the
// stage kernel has just written.  k_row runs the last two of these and the
// first of the next evaluation as one kernel over slabs (z, RB rows y0 ...
// y0 + RB - 1, all three components):
//   1. gather: the slab's S1 rows (3 RB/2 complex lines, each a pair of real
//      rows) are read into shared memory as the full-circle spectrum
//      Z = A + i B of the line pair, as k_xi_r's pair gather does;
//   2. x inverse: each line is C2R-transformed in place (fft4step), keeping
//      x < nx, times 1/(Lx Ly Lz): the slab's H_d rows, in shared memory;
//   3. stage: per group of V = 16 / sizeof(T) cells along x, the 6-point
//      exchange stencil from m in HBM (16-byte row loads, the group's x
//      neighbours in registers), H_d from shared memory, Zeeman, the Gilbert
//      RHS, and the Heun predictor normalize(m + k dt) (MODE_EVAL) or the
//      corrector normalize(m0 + (k1 + k2) dt/2) (MODE_HEUN_CORR) in FP64; the
//      new state goes to HBM (the next stencil reads its neighbours) and over
//      the cell's H_d in shared memory; diagnostics reduce once per block;
//   4. x forward: the new state's rows, times Ms, are R2C-transformed in place
//      (fft4step, the zero-padded half pruned) and stored over the slab's S1
//      rows (both rows of a line pair per 16-byte store).
// Every slab reads and writes only its own S1 rows, so S1 is updated in place.
// H_d never reaches HBM, and the new state is not read back for the x
// forward: per evaluation this saves 3N s (H_d written), 3N s (H_d read) and
// 3N s (state re-read), and two launches.
//
// Measured at 512 x 512 x 8 on the B200 it is slower than the split kernels
// it replaces (FP32: 134 + 117 us per step against 248 us for the split x
// passes and stage kernels; FP64: 292 + 283 against 382 us): a slab holds
// three components' lines (59 KB of shared memory, 159 registers per thread),
// so only 12 warps fit per SM, and the S1 gather and the stencil loads stall
// on memory latency (issue active 26 %, long-scoreboard 5.1 per issue).  It
// is therefore opt-in (FULLMAG_FDM_ROW=on) and tested against the split path.
//
// Arithmetic: the stencil, H_eff and the RHS run in the storage precision T
// (FP32 for the FP32-mixed path, FP64 for the plain path, where the order of
// every operation is that of plain_cell in stages.cuh, so FP64 results equal
// the split kernels' bit for bit); the predictor / corrector sums, their
// normalisation and every energy accumulate in FP64.
#pragma once

#include "demag_reg.cuh"
#include "demag_row.hpp"
#include "stages.cuh"

namespace fm {

template <typename T>
struct RowArgs {
    DemagArgs<T> d;   // S1 (in: the convolved spectrum of s.m; out: x transform of the new state), twiddles, norm, Ms
    StageArgs<T> s;   // stencil input s.m; kout; MODE_EVAL: pred_out, pred_dt; MODE_HEUN_CORR: m0 (in/out), k1, half_dt
};

// Line stride (complex elements): the pair gather's bank-spread stride, even in
// FP32 so that every row of a line region starts on 16 bytes.
template <typename T, int L1, int L2> __host__ __device__ constexpr int row_stride() {
    return sizeof(T) == 4 ? (pair_stride<T, L1, L2>() + 1) / 2 * 2 : pair_stride<T, L1, L2>();
}
template <int RB> __host__ __device__ constexpr int row_lines() { return 3 * RB / 2; }
template <int RB, int L2> __host__ __device__ constexpr int row_threads() { return row_lines<RB>() * L2; }
template <typename T, int L1, int L2, int RB> __host__ __device__ constexpr size_t row_smem() {
    return ((size_t)row_lines<RB>() * row_stride<T, L1, L2>() + (size_t)L1 * L2) * sizeof(cx<T>);
}
// gather loads in flight per thread
template <int L1> __host__ __device__ constexpr int row_gather_u() { return L1 / 2 + 1 < 17 ? L1 / 2 + 1 : 17; }

// 16-byte row vectors: 4 floats or 2 doubles
template <typename T> struct RowVec { T v[16 / sizeof(T)]; };
template <typename T> __device__ __forceinline__ RowVec<T> ldv(const T *p);
template <> __device__ __forceinline__ RowVec<float> ldv<float>(const float *p) {
    const float4 q = *reinterpret_cast<const float4 *>(p);
    return {{q.x, q.y, q.z, q.w}};
}
template <> __device__ __forceinline__ RowVec<double> ldv<double>(const double *p) {
    const double2 q = *reinterpret_cast<const double2 *>(p);
    return {{q.x, q.y}};
}
__device__ __forceinline__ void stv(float *p, const RowVec<float> &v) {
    *reinterpret_cast<float4 *>(p) = make_float4(v.v[0], v.v[1], v.v[2], v.v[3]);
}
__device__ __forceinline__ void stv(double *p, const RowVec<double> &v) {
    *reinterpret_cast<double2 *>(p) = make_double2(v.v[0], v.v[1]);
}

// 1 / |v| for the renormalisation, zero for v = 0: FP64 path as the reference
// (sqrt, then a division); FP32-mixed path, whose result is stored in FP32, a
// single-precision estimate refined by one Newton step in FP64.
template <typename T>
__device__ __forceinline__ double inv_norm(double n2) {
    if (sizeof(T) == 8) {
        const double nn = sqrt(n2);
        return nn > 0.0 ? 1.0 / nn : 0.0;
    }
    if (!(n2 > 0.0)) return 0.0;
    const double y = (double)rsqrtf((float)n2);
    return y * (1.5 - 0.5 * n2 * y * y);
}

template <typename T, int L1, int L2, int RB> __host__ __device__ constexpr int row_min_blocks() {
    return sizeof(T) == 4 ? (RB <= 2 ? 4 : 2) : 2;
}

template <typename T, int L1, int L2, int RB, int MODE>
__global__ void __launch_bounds__(row_threads<RB, L2>(), (row_min_blocks<T, L1, L2, RB>()))
    k_row(RowArgs<T> ra) {
    using C = cx<T>;
    using R = T;
    constexpr int L = L1 * L2, NL = row_lines<RB>(), TE = row_stride<T, L1, L2>(), BT = NL * L2;
    constexpr int V = 16 / (int)sizeof(T), HB = RB / 2, U = row_gather_u<L1>();
    static_assert(RB % 2 == 0, "row pairs");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *region = reinterpret_cast<C *>(smem_raw);
    C *tws = region + NL * TE;
    const DemagArgs<T> &a = ra.d;
    const StageArgs<T> &s = ra.s;
    const int tid = threadIdx.x;
    const int nx = a.nx, ny = a.ny, nz = a.nz, nkx = a.nkx;
    const int y0 = blockIdx.x * RB, z = blockIdx.y;
    for (int k = tid; k < L; k += BT) tws[k] = a.twxT[k];
    // line q: component q / HB, rows y0 + 2 (q % HB) and the next one; its S1 rows
    auto s1_of = [&](int q) -> C * {
        return a.s1 + ((long long)(q / HB) * nz + z) * nkx * ny + y0 + 2 * (q % HB);
    };

    const int q = tid / L2, t = tid - q * L2;
    C *line = region + q * TE;
    T *rows = reinterpret_cast<T *>(line);
    if constexpr (MODE == MODE_ROW_XFWD) {
        // the slab's rows of s.m, 16 bytes per load, into the rows phase 4 reads
        const size_t n = (size_t)s.n;
        const int vpr = nx / V;  // vectors per row
        for (int u = tid; u < NL * 2 * vpr; u += BT) {
            const int qq = u / (2 * vpr), rr = u - qq * 2 * vpr, h = rr / vpr, x0 = (rr - h * vpr) * V;
            const int c = qq / HB, y = y0 + 2 * (qq % HB) + h;
            const RowVec<T> v = ldv<T>(s.m + c * n + ((size_t)z * ny + y) * nx + x0);
            stv(reinterpret_cast<T *>(region + qq * TE) + h * nx + x0, v);
        }
    } else {
    // ---- 1. gather the slab's S1 rows as Z = A + i B on the full circle
    {
        const int qq = tid % NL, k0 = tid / NL;  // kx stride BT / NL = L2
        const C *src = s1_of(qq);
        C *ln = region + qq * TE;
        for (int it0 = k0; it0 < nkx; it0 += U * L2) {
            C va[U], vb[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int k = it0 + u * L2;
                if (k < nkx) {
                    const C *p = src + (long long)k * ny;
                    if constexpr (sizeof(C) == 8) {
                        const float4 v = *reinterpret_cast<const float4 *>(p);  // rows y, y + 1: 16-byte aligned
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
                const int k = it0 + u * L2;
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
    }
    __syncthreads();

    // ---- 2. x inverse in place: rows (y, y + 1) of H_d at reals [0, nx), [nx, 2 nx)
    {
        const T nrm = (T)a.norm;
        fft4step<L1, L2, true, true, true>(t, tws, line, [&](int j) -> C { return line[j]; },
                                           [&](int k, C v) {
                                               if (k < nx) {
                                                   rows[k] = v.x * nrm;
                                                   rows[nx + k] = v.y * nrm;
                                               }
                                           });
    }
    __syncthreads();

    // ---- 3. stage arithmetic per group of V cells along x
    {
        double acc[NQ];
#pragma unroll
        for (int qd = 0; qd < NQ; ++qd) acc[qd] = 0.0;
        const PlainConst kc = plain_const(s);
        const R ix2 = (R)kc.ix2, iy2 = (R)kc.iy2, iz2 = (R)kc.iz2, pref = (R)kc.pref;
        const R hx[3] = {(R)kc.hx0, (R)kc.hx1, (R)kc.hx2};
        const R al = (R)kc.al, gb = (R)kc.gb, pr = (R)kc.pr;
        const bool ex = s.enable_exchange, diag = s.partials != nullptr;
        const size_t n = (size_t)s.n, sxy = (size_t)nx * ny;
        const int gpr = nx / V;
        for (int g = tid; g < RB * gpr; g += BT) {
            const int r = g / gpr, x0 = (g - r * gpr) * V, y = y0 + r;
            const size_t i0 = ((size_t)z * ny + y) * nx + x0;
            const bool hxp = x0 + V < nx, hyp = y + 1 < ny, hzp = z + 1 < nz;
            T *hrow[3];
#pragma unroll
            for (int c = 0; c < 3; ++c)
                hrow[c] = reinterpret_cast<T *>(region + (c * HB + (r >> 1)) * TE) + (r & 1) * nx + x0;
            RowVec<T> cen[3], hd[3], rhs[3], nw[3];
            R he[3][V];  // H_eff (diagnostics)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const T *f = s.m + c * n;
                cen[c] = ldv<T>(f + i0);
                hd[c] = ldv<T>(hrow[c]);
                RowVec<T> yp = cen[c], ym = cen[c], up = cen[c], dn = cen[c];
                T xl = cen[c].v[0], xr = cen[c].v[V - 1];
                if (ex) {
                    if (hyp) yp = ldv<T>(f + i0 + nx);
                    if (y > 0) ym = ldv<T>(f + i0 - nx);
                    if (hzp) up = ldv<T>(f + i0 + sxy);
                    if (z > 0) dn = ldv<T>(f + i0 - sxy);
                    if (x0 > 0) xl = f[i0 - 1];
                    if (hxp) xr = f[i0 + V];
                }
#pragma unroll
                for (int j = 0; j < V; ++j) {
                    R h = R(0);
                    if (ex) {
                        const R cc = cen[c].v[j];
                        const R xp = j + 1 < V ? (R)cen[c].v[j + 1] : (R)xr;
                        const R xm = j > 0 ? (R)cen[c].v[j - 1] : (R)xl;
                        const R lap = (xp - R(2) * cc + xm) * ix2 + ((R)yp.v[j] - R(2) * cc + (R)ym.v[j]) * iy2 +
                                      ((R)up.v[j] - R(2) * cc + (R)dn.v[j]) * iz2;
                        h = lap * pref;
                        if (diag) {
                            // forward pairs (x+1, y+1, z+1) inside the grid, per component
                            R e = R(0);
                            if (j + 1 < V || hxp) e += (xp - cc) * (xp - cc) * ix2;
                            if (hyp) e += ((R)yp.v[j] - cc) * ((R)yp.v[j] - cc) * iy2;
                            if (hzp) e += ((R)up.v[j] - cc) * ((R)up.v[j] - cc) * iz2;
                            acc[Q_EEX] += (double)e;
                        }
                    }
                    he[c][j] = (h + (R)hd[c].v[j]) + hx[c];
                }
            }
            // Gilbert RHS per cell: -gamma_bar (m x H + alpha m x (m x H))
#pragma unroll
            for (int j = 0; j < V; ++j) {
                const R cx_ = cen[0].v[j], cy_ = cen[1].v[j], cz_ = cen[2].v[j];
                const R e0 = he[0][j], e1 = he[1][j], e2 = he[2][j];
                const R p0 = cy_ * e2 - cz_ * e1, p1 = cz_ * e0 - cx_ * e2, p2 = cx_ * e1 - cy_ * e0;
                const R q0 = cy_ * p2 - cz_ * p1, q1 = cz_ * p0 - cx_ * p2, q2 = cx_ * p1 - cy_ * p0;
                rhs[0].v[j] = (T)((pr * p0 + q0 * al) * gb);
                rhs[1].v[j] = (T)((pr * p1 + q1 * al) * gb);
                rhs[2].v[j] = (T)((pr * p2 + q2 * al) * gb);
                if (diag) {
                    const R d0 = hd[0].v[j], d1 = hd[1].v[j], d2 = hd[2].v[j];
                    acc[Q_EDEMAG] += (double)(cx_ * d0 + cy_ * d1 + cz_ * d2);
                    acc[Q_EEXT] += (double)(cx_ * hx[0] + cy_ * hx[1] + cz_ * hx[2]);
                    acc[Q_HEFF2] = fmax(acc[Q_HEFF2], (double)(e0 * e0 + e1 * e1 + e2 * e2));
                    acc[Q_HD2] = fmax(acc[Q_HD2], (double)(d0 * d0 + d1 * d1 + d2 * d2));
                    const R r0 = rhs[0].v[j], r1 = rhs[1].v[j], r2 = rhs[2].v[j];
                    acc[Q_RHS2] = fmax(acc[Q_RHS2], (double)(r0 * r0 + r1 * r1 + r2 * r2));
                }
            }
            if (s.kout) {
#pragma unroll
                for (int c = 0; c < 3; ++c) stv(s.kout + c * n + i0, rhs[c]);
            }
            // the new state: predictor or corrector, FP64 sums and normalisation
            RowVec<T> m0v[3], k1v[3];
            if (MODE == MODE_HEUN_CORR) {
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    m0v[c] = ldv<T>(s.m0 + c * n + i0);
                    k1v[c] = ldv<T>(s.k1 + c * n + i0);
                }
            }
#pragma unroll
            for (int j = 0; j < V; ++j) {
                double v[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    if (MODE == MODE_HEUN_CORR)
                        v[c] = (double)m0v[c].v[j] + ((double)k1v[c].v[j] + (double)rhs[c].v[j]) * s.half_dt;
                    else
                        v[c] = __fma_rn((double)rhs[c].v[j], s.pred_dt, (double)cen[c].v[j]);  // as store_predictor
                }
                const double inv = inv_norm<T>(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
#pragma unroll
                for (int c = 0; c < 3; ++c) nw[c].v[j] = (T)(v[c] * inv);
            }
            T *dst = MODE == MODE_HEUN_CORR ? s.m0 : s.pred_out;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                stv(dst + c * n + i0, nw[c]);
                stv(hrow[c], nw[c]);  // this group's H_d is consumed: its slot takes the new state
            }
        }
        if (s.partials) {
            // scale once per thread: energies as in plain_cell, in FP64
            acc[Q_EEX] *= kc.pair;
            acc[Q_EDEMAG] *= -0.5 * kc.coef;
            acc[Q_EEXT] *= -kc.coef;
            block_reduce_final(acc, s.partials, s.counter, s.out);
        }
    }
    }  // MODE != MODE_ROW_XFWD
    __syncthreads();

    // ---- 4. x forward of the new state (times Ms) in place, stored over the slab's S1 rows
    {
        const T msT = (T)a.ms;
        fft4step<L1, L2, false, true, true, true>(
            t, tws, line, [&](int j) -> C { return mk<T>(rows[j] * msT, rows[nx + j] * msT); },
            [&](int k, C v) { line[k] = v; });
    }
    __syncthreads();
    {
        const int qq = tid % NL, k0 = tid / NL;
        const C *ln = region + qq * TE;
        C *dst = s1_of(qq);
        for (int k = k0; k < nkx; k += L2) {
            const C zk = ln[k];
            const C zm = ln[k == 0 ? 0 : L - k];
            C o0, o1;
            o0.x = T(0.5) * (zk.x + zm.x); o0.y = T(0.5) * (zk.y - zm.y);
            o1.x = T(0.5) * (zk.y + zm.y); o1.y = T(-0.5) * (zk.x - zm.x);
            C *d = dst + (long long)k * ny;
            if constexpr (sizeof(C) == 8) *reinterpret_cast<float4 *>(d) = make_float4(o0.x, o0.y, o1.x, o1.y);
            else { d[0] = o0; d[1] = o1; }
        }
    }
}

}  // namespace fm

// ---------------------------------------------------------------------------
// Host side (included by demag_row_f32.cu / demag_row_f64.cu only)
// ---------------------------------------------------------------------------
#ifdef FM_ROW_HOST
#include <cstdlib>
#include <cstring>
#include <type_traits>

#include "backend_impl.hpp"
#include "demag_row.hpp"

namespace fm {

template <int V> using RowIC = std::integral_constant<int, V>;

// (L1, L2) split of the x length, as fftreg.cuh's l2_for
template <class F>
static bool row_with_split(int L, F &&f) {
    switch (L) {
        case 8: f(RowIC<8>{}, RowIC<1>{}); return true;
        case 16: f(RowIC<16>{}, RowIC<1>{}); return true;
        case 32: f(RowIC<32>{}, RowIC<1>{}); return true;
        case 64: f(RowIC<8>{}, RowIC<8>{}); return true;
        case 128: f(RowIC<16>{}, RowIC<8>{}); return true;
        case 256: f(RowIC<16>{}, RowIC<16>{}); return true;
        case 512: f(RowIC<32>{}, RowIC<16>{}); return true;
        case 1024: f(RowIC<32>{}, RowIC<32>{}); return true;
        case 2048: f(RowIC<64>{}, RowIC<32>{}); return true;
        case 4096: f(RowIC<64>{}, RowIC<64>{}); return true;
        default: return false;
    }
}

template <typename T, class F>
static void row_with_rb(int RB, F &&f) {
    if (RB == 2) f(RowIC<2>{});
    if constexpr (sizeof(T) == 4) {
        if (RB == 4) f(RowIC<4>{});
    }
}

// static: every unit that includes fftreg.cuh has its own copy of the constant
// twiddle table and must fill that one; the legacy-stream upload from pageable
// memory is followed by a device synchronisation, since the library's stream
// is non-blocking
static bool row_upload_tw64(Backend &b) {
    double2 d[64];
    float2 f[64];
    for (int k = 0; k < 64; ++k) {
        const double ang = 2.0 * 3.14159265358979323846 * (double)k / 64.0;
        d[k] = make_double2(std::cos(ang), -std::sin(ang));
        f[k] = make_float2((float)d[k].x, (float)d[k].y);
    }
    return cuda_ok(b, cudaMemcpyToSymbol(c_tw64d, d, sizeof(d)), "twiddle64 d (row)") &&
           cuda_ok(b, cudaMemcpyToSymbol(c_tw64f, f, sizeof(f)), "twiddle64 f (row)") &&
           cuda_ok(b, cudaDeviceSynchronize(), "twiddle64 (row) sync");
}

template <typename T, int L1, int L2, int RB>
constexpr bool row_fits() {
    return row_smem<T, L1, L2, RB>() <= 200 * 1024 && (sizeof(T) == 4 || L1 <= 32);
}

template <typename T>
bool row_configure_t(Backend &b) {
    b.use_row = false;
    b.row_rb = 0;
    // opt-in (FULLMAG_FDM_ROW=on): measured slower than the split kernels
    const char *on = std::getenv("FULLMAG_FDM_ROW");
    if (!on || std::strcmp(on, "on") != 0) return true;
    constexpr int V = 16 / (int)sizeof(T);
    const bool uniform = !b.has_mask && !b.has_ms_map && !b.has_regions && b.boundary_tier == 0 && b.corr_targets == 0;
    if (!b.use_reg || !b.enable_demag || !uniform || b.integrator != FULLMAG_FDM_INTEGRATOR_HEUN ||
        b.Lx != 2 * b.nx || b.nx % V != 0 || b.ny % 2 != 0 || 3LL * b.n >= (1LL << 31))
        return true;
    int want = sizeof(T) == 4 ? (b.ny % 4 == 0 ? 4 : 2) : 2;
    if (const char *p = std::getenv("FULLMAG_FDM_ROW_RB")) want = std::atoi(p);
    if (want <= 0 || b.ny % want != 0) return true;
    bool ok = true, any = false;
    row_with_split(b.Lx, [&](auto l1, auto l2) {
        constexpr int L1 = decltype(l1)::value, L2 = decltype(l2)::value;
        row_with_rb<T>(want, [&](auto rbc) {
            constexpr int RB = decltype(rbc)::value;
            if constexpr (row_fits<T, L1, L2, RB>()) {
                constexpr size_t smem = row_smem<T, L1, L2, RB>();
                if (cudaFuncSetAttribute(k_row<T, L1, L2, RB, MODE_EVAL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
                    cudaFuncSetAttribute(k_row<T, L1, L2, RB, MODE_HEUN_CORR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
                    cudaFuncSetAttribute(k_row<T, L1, L2, RB, MODE_ROW_XFWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
                    cudaGetLastError();
                    return;
                }
                b.rsm_row = smem;
                b.row_rb = RB;
                any = true;
            }
        });
    });
    if (!any) return true;
    ok = row_upload_tw64(b);
    b.use_row = ok;
    return ok;
}

template <typename T>
bool row_launch_t(Backend &b, const DemagArgs<T> &d, const StageArgs<T> &s, int mode) {
    RowArgs<T> ra{d, s};
    bool launched = false;
    row_with_split(b.Lx, [&](auto l1, auto l2) {
        constexpr int L1 = decltype(l1)::value, L2 = decltype(l2)::value;
        row_with_rb<T>(b.row_rb, [&](auto rbc) {
            constexpr int RB = decltype(rbc)::value;
            if constexpr (row_fits<T, L1, L2, RB>()) {
                const dim3 grid((unsigned)(b.ny / RB), (unsigned)b.nz);
                if (mode == MODE_HEUN_CORR)
                    k_row<T, L1, L2, RB, MODE_HEUN_CORR><<<grid, row_threads<RB, L2>(), b.rsm_row, b.stream>>>(ra);
                else if (mode == MODE_ROW_XFWD)
                    k_row<T, L1, L2, RB, MODE_ROW_XFWD><<<grid, row_threads<RB, L2>(), b.rsm_row, b.stream>>>(ra);
                else
                    k_row<T, L1, L2, RB, MODE_EVAL><<<grid, row_threads<RB, L2>(), b.rsm_row, b.stream>>>(ra);
                launched = true;
            }
        });
    });
    if (!launched) {
        b.last_error = "fused row pass: no kernel for this grid";
        return false;
    }
    return cuda_ok(b, cudaGetLastError(), "fused row pass");
}

}  // namespace fm
#endif  // FM_ROW_HOST
