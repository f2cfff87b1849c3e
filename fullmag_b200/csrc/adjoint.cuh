// adjoint.cuh — discrete adjoint of the Heun-LLG step (exchange + demag + Zeeman).
//
// No counterpart in the reference.  For one Heun step (lib.rs:1217-1249)
//   k1 = f(m_n, t),  u = m_n + dt k1,  m_p = u / |u|,
//   k2 = f(m_p, t + dt),  w = m_n + dt/2 (k1 + k2),  m_{n+1} = w / |w|,
//   f(m, t) = -gb (pr m x H + alpha m x (m x H)),  H = K(Ms) m + H_ext(t),
// the cotangent lambda of m_{n+1} is pulled back to m_n:
//   normalisation:  lambda_w = (lambda - (m.lambda) m) / |w|   (m = w / |w|), likewise for u;
//   RHS, per cell:  with g the cotangent of f, gp = -gb pr g, gq = -gb alpha g,
//                   gP = gp + gq x m,  p = m x H:
//                   lambda_H = gP x m,  lambda_m(local) = p x gq + H x gP;
//   fields:         K^T lambda_H = L (c lambda_H) + Ms (-N * lambda_H), c = 2A / (mu0 Ms);
//                   the 6-point Neumann Laplacian L and the Newell convolution N are
//                   symmetric (N(-r) = N(r), N^T = N), so both transposes are the
//                   forward operators (the demag one with a unit source).
// Parameter cotangents accumulate per cell in FP64:
//   dL/dMs_i   += lambda_H,i . (-H_ex,i / Ms_i) + m_i . (-N * lambda_H)_i,
//   dL/dH_ext  += lambda_H,i,   dL/dH_ac += lambda_H,i sin(omega t_stage).
// Inactive cells (mask or Ms = 0) carry no cotangent.
#pragma once

#include "common.cuh"

namespace fm {

struct AdjArgs {
    long long n;
    int nx, ny, nz;
    double dinv[3];                   // 1/dx^2, 1/dy^2, 1/dz^2
    double aex, ms, gamma_bar, alpha, pr;
    const double *ms_map;             // optional
    const uint8_t *mask;              // optional
    double dt;
};

__device__ __forceinline__ bool adj_active(const AdjArgs &a, long long i, double &ms_i) {
    ms_i = a.ms_map ? a.ms_map[i] : a.ms;
    return (!a.mask || a.mask[i] != 0) && ms_i > 0.0;
}

__device__ __forceinline__ void cross3(const double *a, const double *b, double *o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

// Start of a step's pull-back: lambda_w from lambda (cotangent of m_{n+1}),
// w recomputed from m_n, k1, k2 as the corrector forms it.  Outputs
// acc = lambda_w (m_n's cotangent so far) and gk = dt/2 lambda_w (cotangent of k2
// and, so far, of k1).
template <typename T>
__global__ void __launch_bounds__(256) k_adj_start(AdjArgs a, const T *m, const T *k1, const T *k2,
                                                   const double *lam, double *acc, double *gk) {
    const long long n = a.n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double ms_i;
        if (!adj_active(a, i, ms_i)) {
            for (int c = 0; c < 3; ++c) { acc[c * n + i] = 0.0; gk[c * n + i] = 0.0; }
            continue;
        }
        const double hdt = 0.5 * a.dt;
        double w[3], l[3];
        for (int c = 0; c < 3; ++c) {
            w[c] = (double)m[c * n + i] + ((double)k1[c * n + i] + (double)k2[c * n + i]) * hdt;
            l[c] = lam[c * n + i];
        }
        const double nw = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
        const double inv = nw > 0.0 ? 1.0 / nw : 0.0;
        const double mh[3] = {w[0] * inv, w[1] * inv, w[2] * inv};
        const double d = mh[0] * l[0] + mh[1] * l[1] + mh[2] * l[2];
        for (int c = 0; c < 3; ++c) {
            const double lw = (l[c] - d * mh[c]) * inv;
            acc[c * n + i] = lw;
            gk[c * n + i] = hdt * lw;
        }
    }
}

// Local vector-Jacobian product of f at (m, H) with cotangent g: lambda_H
// (stored in the state precision: it is the source of the transposed demag
// convolution) and the local part of m's cotangent.
template <typename T>
__global__ void __launch_bounds__(256) k_adj_vjp(AdjArgs a, const T *m, const T *H, const double *g,
                                                 T *lh, double *lloc) {
    const long long n = a.n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double ms_i;
        if (!adj_active(a, i, ms_i)) {
            for (int c = 0; c < 3; ++c) { lh[c * n + i] = T(0); lloc[c * n + i] = 0.0; }
            continue;
        }
        double mm[3], hh[3], gg[3];
        for (int c = 0; c < 3; ++c) {
            mm[c] = (double)m[c * n + i];
            hh[c] = (double)H[c * n + i];
            gg[c] = g[c * n + i];
        }
        const double s = -a.gamma_bar;
        double gp[3], gq[3];
        for (int c = 0; c < 3; ++c) { gp[c] = s * a.pr * gg[c]; gq[c] = s * a.alpha * gg[c]; }
        double gqm[3], gP[3], p[3], lH[3], t1[3], t2[3];
        cross3(gq, mm, gqm);
        for (int c = 0; c < 3; ++c) gP[c] = gp[c] + gqm[c];
        cross3(mm, hh, p);
        cross3(gP, mm, lH);
        cross3(p, gq, t1);
        cross3(hh, gP, t2);
        for (int c = 0; c < 3; ++c) {
            lh[c * n + i] = (T)lH[c];
            lloc[c * n + i] = t1[c] + t2[c];
        }
    }
}

// m's cotangent at one stage: lambda_local + L(c lambda_H) + Ms (-N * lambda_H),
// with the parameter cotangents accumulated (sin_t = sin(omega t_stage)).
// hadj = -N * (P lambda_H) from the demag pipeline with a unit source.
template <typename T>
__global__ void __launch_bounds__(256) k_adj_apply(AdjArgs a, const T *m, const T *lh, const T *hadj,
                                                   const T *hex, const double *lloc, double *out,
                                                   double *g_ms, double *g_hext, double *g_hac,
                                                   double sin_t) {
    const long long n = a.n, sxy = (long long)a.nx * a.ny;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double ms_i;
        if (!adj_active(a, i, ms_i)) {
            for (int c = 0; c < 3; ++c) out[c * n + i] = 0.0;
            continue;
        }
        const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / sxy);
        // neighbours inside the grid and active (the forward's clamping makes the
        // others contribute zero)
        const long long nb[6] = {x + 1 < nx ? i + 1 : -1, x > 0 ? i - 1 : -1,
                                 y + 1 < ny ? i + nx : -1, y > 0 ? i - nx : -1,
                                 z + 1 < nz ? i + sxy : -1, z > 0 ? i - sxy : -1};
        const double ci = 2.0 * a.aex / (kMu0 * ms_i);
        double yc[3];
        for (int c = 0; c < 3; ++c) yc[c] = ci * (double)lh[c * n + i];
        double z3[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            const long long j = nb[q];
            double ms_j;
            if (j < 0 || !adj_active(a, j, ms_j)) continue;
            const double cj = 2.0 * a.aex / (kMu0 * ms_j);
            for (int c = 0; c < 3; ++c) z3[c] += (cj * (double)lh[c * n + j] - yc[c]) * a.dinv[q >> 1];
        }
        double gms = 0.0;
        for (int c = 0; c < 3; ++c) {
            const double lHc = (double)lh[c * n + i], hc = (double)hadj[c * n + i];
            const double mc = (double)m[c * n + i];
            out[c * n + i] = lloc[c * n + i] + z3[c] + ms_i * hc;
            gms += lHc * (-(double)hex[c * n + i] / ms_i) + mc * hc;
            g_hext[c * n + i] += lHc;
            g_hac[c * n + i] += lHc * sin_t;
        }
        g_ms[i] += gms;
    }
}

// Predictor normalisation pull-back: lambda_u = (lambda_mp - (m_p.lambda_mp) m_p) / |u|
// with u = m_n + dt k1 recomputed as the predictor forms it; acc += lambda_u and
// gk (cotangent of k1) += dt lambda_u.
template <typename T>
__global__ void __launch_bounds__(256) k_adj_pred(AdjArgs a, const T *m, const T *k1, const double *lmp,
                                                  double *acc, double *gk) {
    const long long n = a.n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double ms_i;
        if (!adj_active(a, i, ms_i)) continue;
        double u[3], l[3];
        for (int c = 0; c < 3; ++c) {
            u[c] = (double)m[c * n + i] + (double)k1[c * n + i] * a.dt;
            l[c] = lmp[c * n + i];
        }
        const double nu = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        const double inv = nu > 0.0 ? 1.0 / nu : 0.0;
        const double mh[3] = {u[0] * inv, u[1] * inv, u[2] * inv};
        const double d = mh[0] * l[0] + mh[1] * l[1] + mh[2] * l[2];
        for (int c = 0; c < 3; ++c) {
            const double lu = (l[c] - d * mh[c]) * inv;
            acc[c * n + i] += lu;
            gk[c * n + i] += a.dt * lu;
        }
    }
}

// lambda_n = acc + the last stage's field pull-back.
__global__ void __launch_bounds__(256) k_adj_finish(long long n3, const double *acc, const double *part,
                                                    double *lam) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n3; i += (long long)gridDim.x * blockDim.x)
        lam[i] = acc[i] + part[i];
}

}  // namespace fm
