// stage_vec.cuh — uniform-material stage kernels on 16-byte groups of cells.
//
// The per-cell model of k_stage / plain_cell (stages.cuh) for a uniform
// material (no mask, Ms map, region LUT or boundary tier) whose rows are a
// multiple of V = 16 / sizeof(T) cells: each thread owns V consecutive cells
// of one row of one z plane and reads every operand as one 16-byte load per
// component (the cells' m, the rows above and below in y and in z, H_d, and
// for the corrector m0 and k1, for DP45's last stage the earlier stages); the
// x neighbours inside the group are in registers, those at its ends come from
// the adjacent lanes by shuffles (the warp's edge lanes load theirs).  One
// plane per thread and about 80 registers, so many warps per SM hide the load
// latency without a software pipeline; per cell this executes a fifth of the
// instructions of the one-value-per-load ring kernel.
//
// MK: a mask and / or an Ms map (no region LUT or boundary tier): a cell is
// active when its mask byte is non-zero and its Ms is positive; an inactive
// neighbour is replaced by the centre, inactive cells get zero RHS, fields and
// (corrector) state, and stay out of every diagnostic, as in k_stage.
//
// Precision: the stencil, H_eff and the Gilbert RHS run in the storage type T,
// FP32 for the FP32-mixed path, the only one built (stage_vec.cu: in FP64 the
// one-value-per-load kernels measured faster); the Heun predictor and corrector
// sums and their renormalisation, the embedded error norm and every energy
// accumulate in FP64; the max-norms are exact in either precision.
#pragma once

#include "stages.cuh"

namespace fm {

// 16-byte groups of cells: 4 floats or 2 doubles
template <typename T> struct SVec { T v[16 / sizeof(T)]; };
template <typename T> __device__ __forceinline__ SVec<T> sv_ld(const T *p);
template <> __device__ __forceinline__ SVec<float> sv_ld<float>(const float *p) {
    const float4 q = *reinterpret_cast<const float4 *>(p);
    return {{q.x, q.y, q.z, q.w}};
}
template <> __device__ __forceinline__ SVec<double> sv_ld<double>(const double *p) {
    const double2 q = *reinterpret_cast<const double2 *>(p);
    return {{q.x, q.y}};
}
__device__ __forceinline__ void sv_st(float *p, const SVec<float> &v) {
    *reinterpret_cast<float4 *>(p) = make_float4(v.v[0], v.v[1], v.v[2], v.v[3]);
}
__device__ __forceinline__ void sv_st(double *p, const SVec<double> &v) {
    *reinterpret_cast<double2 *>(p) = make_double2(v.v[0], v.v[1]);
}

// 1 / |v| for the renormalisation, zero for v = 0: the FP64 path as the
// reference (sqrt, then a division); the FP32-mixed path, whose result is
// stored in FP32, a single-precision estimate refined by one Newton step in
// FP64 (relative error ~1e-14).
template <typename T>
__device__ __forceinline__ double sv_inv_norm(double n2) {
    if (sizeof(T) == 8) {
        const double nn = sqrt(n2);
        return nn > 0.0 ? 1.0 / nn : 0.0;
    }
    if (!(n2 > 0.0)) return 0.0;
    const double y = (double)rsqrtf((float)n2);
    return y * (1.5 - 0.5 * n2 * y * y);
}

constexpr int kStageVecBY = 4;  // rows (warps) per block

template <typename T, int MODE> __host__ __device__ constexpr int stage_vec_min_blocks() {
    return sizeof(T) == 4 ? 5 : 4;
}

// activity bits of V cells from index i (bit j: cell i + j)
template <int V, bool MK, typename T>
__device__ __forceinline__ unsigned sv_active(const StageArgs<T> &a, size_t i) {
    if (!MK) return (1u << V) - 1u;
    unsigned b = (1u << V) - 1u;
    if (a.mask) {
        if (V == 4) {
            const unsigned w = *reinterpret_cast<const unsigned *>(a.mask + i);  // 4-byte aligned: i % 4 == 0
#pragma unroll
            for (int j = 0; j < 4; ++j) if (((w >> (8 * j)) & 0xffu) == 0u) b &= ~(1u << j);
        } else if (V == 2) {
            const unsigned short w = *reinterpret_cast<const unsigned short *>(a.mask + i);
#pragma unroll
            for (int j = 0; j < 2; ++j) if (((w >> (8 * j)) & 0xffu) == 0u) b &= ~(1u << j);
        } else {
            if (a.mask[i] == 0) b = 0u;
        }
    }
    if (a.ms_map) {
#pragma unroll
        for (int j = 0; j < V; ++j) if (!(a.ms_map[i + j] > 0.0)) b &= ~(1u << j);
    }
    return b;
}

// Per-launch constants of k_stage_vec in the arithmetic precision R.
template <typename R>
struct SvConst {
    R ix2, iy2, iz2, pref, hx[3], al, gb, pr;
};

// One group: V cells of row y, plane z, from x0 (an owning thread: x0 < nx,
// y < ny; the others pass the last group of the row with own = false and only
// take part in the shuffles).  32-bit indices (3 n < 2^32, checked by the host).
template <typename T, int MODE, bool MK>
__device__ __forceinline__ void sv_group(const StageArgs<T> &a, const PlainConst &kc, const SvConst<T> &q,
                                         int lane, int xc, int yc, int z, bool own, double (&acc)[NQ], T &mx_heff,
                                         T &mx_hd, T &mx_rhs) {
    using R = T;
    constexpr int V = 16 / (int)sizeof(T);
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const unsigned n = (unsigned)a.n, sxy = (unsigned)nx * (unsigned)ny;
    const unsigned i0 = ((unsigned)z * (unsigned)ny + (unsigned)yc) * (unsigned)nx + (unsigned)xc;
    const bool hxp = xc + V < nx, hxm = xc > 0, hyp = yc + 1 < ny, hym = yc > 0, hzp = z + 1 < nz, hzm = z > 0;
    const bool ex = a.enable_exchange, diag = a.partials != nullptr;

    // activity: this group's cells and its neighbour rows (bit j: cell j of the row)
    const unsigned act = sv_active<V, MK>(a, i0);
    unsigned ayp = act, aym = act, azp = act, azm = act, axr = 1u, axl = 1u;
    if (MK) {
        if (hyp) ayp = sv_active<V, MK>(a, i0 + nx);
        if (hym) aym = sv_active<V, MK>(a, i0 - nx);
        if (hzp) azp = sv_active<V, MK>(a, i0 + sxy);
        if (hzm) azm = sv_active<V, MK>(a, i0 - sxy);
        axr = __shfl_down_sync(0xffffffffu, act, 1) & 1u;
        axl = (__shfl_up_sync(0xffffffffu, act, 1) >> (V - 1)) & 1u;
        if (!hxp) axr = 0u;
        else if (lane == 31) axr = sv_active<1, MK>(a, i0 + V) & 1u;
        if (!hxm) axl = 0u;
        else if (lane == 0) axl = sv_active<1, MK>(a, i0 - 1) & 1u;
    }
    // per-cell Ms (exchange prefactor, energies) where it varies
    const bool per_cell = MK && a.ms_map;
    R prefj[V];
    double coefj[V];
#pragma unroll
    for (int j = 0; j < V; ++j) {
        const double msj = per_cell ? a.ms_map[i0 + j] : a.ms;
        prefj[j] = per_cell ? (R)(msj > 0.0 ? 2.0 * a.aex / (kMu0 * msj) : 0.0) : q.pref;
        coefj[j] = per_cell ? msj * a.vol * kMu0 : kc.coef;
    }

    SVec<T> cen[3], hd[3];
    R he[3][V], hxo[3][V], eex[V];
#pragma unroll
    for (int j = 0; j < V; ++j) eex[j] = R(0);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const T *f = a.m + c * n;
        cen[c] = sv_ld<T>(f + i0);
        if (a.enable_demag) hd[c] = sv_ld<T>(a.hd + c * n + i0);
        else {
#pragma unroll
            for (int j = 0; j < V; ++j) hd[c].v[j] = T(0);
        }
        // x neighbours of the group's end cells: the adjacent lanes, the warp's
        // edge lanes from memory, the cell itself at the grid edge (Neumann)
        T xr = __shfl_down_sync(0xffffffffu, cen[c].v[0], 1);
        T xl = __shfl_up_sync(0xffffffffu, cen[c].v[V - 1], 1);
        if (!hxp) xr = cen[c].v[V - 1];
        else if (lane == 31) xr = f[i0 + V];
        if (!hxm) xl = cen[c].v[0];
        else if (lane == 0) xl = f[i0 - 1];
        SVec<T> yp = cen[c], ym = cen[c], up = cen[c], dn = cen[c];
        if (ex) {
            if (hyp) yp = sv_ld<T>(f + i0 + nx);
            if (hym) ym = sv_ld<T>(f + i0 - nx);
            if (hzp) up = sv_ld<T>(f + i0 + sxy);
            if (hzm) dn = sv_ld<T>(f + i0 - sxy);
        }
#pragma unroll
        for (int j = 0; j < V; ++j) {
            R h = R(0);
            const bool aj = (act >> j) & 1u;
            if (ex && aj) {
                // neighbours clamped at the grid edge; an inactive one is the centre
                const R cc = cen[c].v[j];
                const bool axp = j + 1 < V ? ((act >> (j + 1)) & 1u) : axr;
                const bool axm = j > 0 ? ((act >> (j - 1)) & 1u) : axl;
                R xp = j + 1 < V ? (R)cen[c].v[j + 1] : (R)xr;
                R xm = j > 0 ? (R)cen[c].v[j - 1] : (R)xl;
                R ypj = yp.v[j], ymj = ym.v[j], upj = up.v[j], dnj = dn.v[j];
                if (MK) {
                    if (!axp) xp = cc;
                    if (!axm) xm = cc;
                    if (!((ayp >> j) & 1u)) ypj = cc;
                    if (!((aym >> j) & 1u)) ymj = cc;
                    if (!((azp >> j) & 1u)) upj = cc;
                    if (!((azm >> j) & 1u)) dnj = cc;
                }
                const R lap = (xp - R(2) * cc + xm) * q.ix2 + (ypj - R(2) * cc + ymj) * q.iy2 +
                              (upj - R(2) * cc + dnj) * q.iz2;
                h = lap * prefj[j];
                if (diag) {
                    // forward pairs (x+1, y+1, z+1) inside the grid, both cells active
                    if ((j + 1 < V || hxp) && (!MK || axp)) eex[j] += (xp - cc) * (xp - cc) * q.ix2;
                    if (hyp && (!MK || ((ayp >> j) & 1u))) eex[j] += (ypj - cc) * (ypj - cc) * q.iy2;
                    if (hzp && (!MK || ((azp >> j) & 1u))) eex[j] += (upj - cc) * (upj - cc) * q.iz2;
                }
            }
            hxo[c][j] = h;
            he[c][j] = aj ? (h + (R)hd[c].v[j]) + q.hx[c] : R(0);
        }
    }
    // Gilbert RHS per cell: -gamma_bar (m x H + alpha m x (m x H)), rounded to T
    SVec<T> rhs[3];
#pragma unroll
    for (int j = 0; j < V; ++j) {
        const R cx_ = cen[0].v[j], cy_ = cen[1].v[j], cz_ = cen[2].v[j];
        const R e0 = he[0][j], e1 = he[1][j], e2 = he[2][j];
        const R p0 = cy_ * e2 - cz_ * e1, p1 = cz_ * e0 - cx_ * e2, p2 = cx_ * e1 - cy_ * e0;
        const R q0 = cy_ * p2 - cz_ * p1, q1 = cz_ * p0 - cx_ * p2, q2 = cx_ * p1 - cy_ * p0;
        const bool aj = (act >> j) & 1u;
        rhs[0].v[j] = aj ? (T)((q.pr * p0 + q0 * q.al) * q.gb) : T(0);
        rhs[1].v[j] = aj ? (T)((q.pr * p1 + q1 * q.al) * q.gb) : T(0);
        rhs[2].v[j] = aj ? (T)((q.pr * p2 + q2 * q.al) * q.gb) : T(0);
        if (diag && own && aj) {
            // per cell in R, accumulated in FP64
            const R d0 = hd[0].v[j], d1 = hd[1].v[j], d2 = hd[2].v[j];
            const double dd = (double)(cx_ * d0 + cy_ * d1 + cz_ * d2);
            const double de = (double)(cx_ * q.hx[0] + cy_ * q.hx[1] + cz_ * q.hx[2]);
            acc[Q_EEX] += (double)eex[j];
            acc[Q_EDEMAG] += per_cell ? coefj[j] * dd : dd;
            acc[Q_EEXT] += per_cell ? coefj[j] * de : de;
            mx_heff = fmax(mx_heff, e0 * e0 + e1 * e1 + e2 * e2);
            mx_hd = fmax(mx_hd, d0 * d0 + d1 * d1 + d2 * d2);
            const R r0 = rhs[0].v[j], r1 = rhs[1].v[j], r2 = rhs[2].v[j];
            mx_rhs = fmax(mx_rhs, r0 * r0 + r1 * r1 + r2 * r2);
        }
    }
    if (!own) return;
    if (a.kout) {
#pragma unroll
        for (int c = 0; c < 3; ++c) sv_st(a.kout + c * n + i0, rhs[c]);
    }
    if (MODE == MODE_EVAL && (a.hex_out || a.heff_out)) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            SVec<T> ho, eo;
#pragma unroll
            for (int j = 0; j < V; ++j) { ho.v[j] = (T)hxo[c][j]; eo.v[j] = (T)he[c][j]; }
            if (a.hex_out) sv_st(a.hex_out + c * n + i0, ho);
            if (a.heff_out) sv_st(a.heff_out + c * n + i0, eo);
        }
    }
    if ((MODE == MODE_EVAL && a.pred_out) || MODE == MODE_HEUN_CORR) {
        // the new state in FP64: predictor normalize(m + k dt), corrector
        // normalize(m0 + (k1 + k2) dt / 2)
        // the corrector's m0 and k1 here (issued with the stencil's loads at 120
        // registers the kernel measured 45.4 us against 41.0 at C2)
        SVec<T> m0v[3], k1v[3], nw[3];
        if (MODE == MODE_HEUN_CORR) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                m0v[c] = sv_ld<T>(a.m0 + c * n + i0);
                k1v[c] = sv_ld<T>(a.k1 + c * n + i0);
            }
        }
#pragma unroll
        for (int j = 0; j < V; ++j) {
            double v[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                if (MK && MODE == MODE_HEUN_CORR && !((act >> j) & 1u))
                    v[c] = 0.0;  // inactive cells: the corrected state is zero
                else if (MODE == MODE_HEUN_CORR)
                    v[c] = (double)m0v[c].v[j] + ((double)k1v[c].v[j] + (double)rhs[c].v[j]) * a.half_dt;
                else
                    v[c] = __fma_rn((double)rhs[c].v[j], a.pred_dt, (double)cen[c].v[j]);  // as store_predictor
            }
            const double inv = sv_inv_norm<T>(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
#pragma unroll
            for (int c = 0; c < 3; ++c) nw[c].v[j] = (T)(v[c] * inv);
        }
        T *dst = MODE == MODE_HEUN_CORR ? a.m0 : a.pred_out;
#pragma unroll
        for (int c = 0; c < 3; ++c) sv_st(dst + c * n + i0, nw[c]);
    }
    if (MODE == MODE_ERR_LAST && diag) {
        // err = dt (sum_j ew[j] ke[j] + ew[nke] k_last) in FP64, accumulated from
        // zero in that order (max_error_norm_buf, lib.rs:1653-1674)
        double e2[V];
#pragma unroll
        for (int j = 0; j < V; ++j) e2[j] = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double e[V];
#pragma unroll
            for (int j = 0; j < V; ++j) e[j] = 0.0;
            for (int st = 0; st < a.nke; ++st) {
                const SVec<T> kv = sv_ld<T>(a.ke[st] + c * n + i0);
#pragma unroll
                for (int j = 0; j < V; ++j) e[j] += a.ew[st] * (double)kv.v[j];
            }
#pragma unroll
            for (int j = 0; j < V; ++j) {
                const double ej = (e[j] + a.ew[a.nke] * (double)rhs[c].v[j]) * a.dt;
                e2[j] += ej * ej;
            }
        }
#pragma unroll
        for (int j = 0; j < V; ++j)
            if ((act >> j) & 1u) acc[Q_ERR2] = fmax(acc[Q_ERR2], e2[j]);
    }
}

// block (32, kStageVecBY); grid (ceil(nx / (32 V)), ceil(ny / BY), ceil(nz / zb)):
// each thread takes the planes [blockIdx.z zb, + zb) of its group in turn, so
// that the per-block reduction and its fence are paid once per zb planes.
template <typename T, int MODE, bool MK = false>
__global__ void __launch_bounds__(32 * kStageVecBY, (stage_vec_min_blocks<T, MODE>())) k_stage_vec(StageArgs<T> a,
                                                                                                   int zb) {
    using R = T;
    constexpr int V = 16 / (int)sizeof(T);
    const int lane = threadIdx.x;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int x0 = (blockIdx.x * 32 + lane) * V, y = blockIdx.y * kStageVecBY + threadIdx.y;
    const bool own = x0 < nx && y < ny;   // threads past the grid load the last group and only shuffle
    const int xc = min(x0, nx - V), yc = min(y, ny - 1);
    const PlainConst kc = plain_const(a);
    SvConst<R> q;
    q.ix2 = (R)kc.ix2; q.iy2 = (R)kc.iy2; q.iz2 = (R)kc.iz2; q.pref = (R)kc.pref;
    q.hx[0] = (R)kc.hx0; q.hx[1] = (R)kc.hx1; q.hx[2] = (R)kc.hx2;
    q.al = (R)kc.al; q.gb = (R)kc.gb; q.pr = (R)kc.pr;
    double acc[NQ];
#pragma unroll
    for (int k = 0; k < NQ; ++k) acc[k] = 0.0;
    R mx_heff = R(0), mx_hd = R(0), mx_rhs = R(0);
    const int z0 = blockIdx.z * zb, z1 = min(z0 + zb, nz);
    for (int z = z0; z < z1; ++z)
        sv_group<T, MODE, MK>(a, kc, q, lane, xc, yc, z, own, acc, mx_heff, mx_hd, mx_rhs);
    if (a.partials) {
        const bool per_cell = MK && a.ms_map;
        acc[Q_EEX] *= kc.pair;
        acc[Q_EDEMAG] *= per_cell ? -0.5 : -0.5 * kc.coef;
        acc[Q_EEXT] *= per_cell ? -1.0 : -kc.coef;
        acc[Q_HEFF2] = (double)mx_heff;
        acc[Q_HD2] = (double)mx_hd;
        acc[Q_RHS2] = (double)mx_rhs;
        block_reduce_final(acc, a.partials, a.counter, a.out);  // every thread of the block
    }
}

}  // namespace fm

namespace fm {

// normalize(m0 + sum_j c_j k_j) on 16-byte groups of cells: the sums and
// grouping of combine_cell (forms 0..4, FP64) and the renormalisation of the
// k_stage_vec kernels it runs with, every operand one 16-byte load per
// component.  Requires n to be a multiple of V.
template <typename T>
__global__ void __launch_bounds__(256) k_combine_vec(CombineArgs<T> a) {
    constexpr int V = 16 / (int)sizeof(T);
    const size_t n = (size_t)a.n, groups = n / V;
    for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < groups; g += (size_t)gridDim.x * blockDim.x) {
        const size_t i = g * V;
        double v[3][V];
#pragma unroll
        for (int comp = 0; comp < 3; ++comp) {
            const size_t o = comp * n + i;
            SVec<T> k0 = sv_ld<T>(a.k[0] + o), k1, k2, k3, k4;
            if (a.form >= 1) k1 = sv_ld<T>(a.k[1] + o);
            if (a.form >= 2) k2 = sv_ld<T>(a.k[2] + o);
            if (a.form >= 3) k3 = sv_ld<T>(a.k[3] + o);
            if (a.form >= 4) k4 = sv_ld<T>(a.k[4] + o);
            const SVec<T> m0 = sv_ld<T>(a.m0 + o);
#pragma unroll
            for (int j = 0; j < V; ++j) {
                double inc;
                switch (a.form) {
                    case 0: inc = (double)k0.v[j] * a.c[0]; break;
                    case 1: inc = ((double)k0.v[j] * a.c[0] + (double)k1.v[j] * a.c[1]) * a.dt; break;
                    case 2:
                        inc = (((double)k0.v[j] * a.c[0] + (double)k1.v[j] * a.c[1]) + (double)k2.v[j] * a.c[2]) * a.dt;
                        break;
                    case 3:
                        inc = (((double)k0.v[j] * a.c[0] + (double)k1.v[j] * a.c[1]) +
                               ((double)k2.v[j] * a.c[2] + (double)k3.v[j] * a.c[3])) * a.dt;
                        break;
                    default:
                        inc = ((((double)k0.v[j] * a.c[0] + (double)k1.v[j] * a.c[1]) + (double)k2.v[j] * a.c[2]) +
                               ((double)k3.v[j] * a.c[3] + (double)k4.v[j] * a.c[4])) * a.dt;
                        break;
                }
                // form 0 (the predictor): one explicit fused multiply-add, as every predictor site
                v[comp][j] = a.form == 0 ? __fma_rn((double)k0.v[j], a.c[0], (double)m0.v[j]) : (double)m0.v[j] + inc;
            }
        }
        SVec<T> o3[3];
#pragma unroll
        for (int j = 0; j < V; ++j) {
            // the renormalisation of the 16-byte-group stage kernels, so that a
            // predictor formed here has the bits the RHS kernel would give it
            const double inv = sv_inv_norm<T>(v[0][j] * v[0][j] + v[1][j] * v[1][j] + v[2][j] * v[2][j]);
#pragma unroll
            for (int comp = 0; comp < 3; ++comp) o3[comp].v[j] = (T)(v[comp][j] * inv);
        }
#pragma unroll
        for (int comp = 0; comp < 3; ++comp) sv_st(a.out + comp * n + i, o3[comp]);
    }
}

}  // namespace fm
