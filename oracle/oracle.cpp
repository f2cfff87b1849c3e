/*
 * oracle.cpp — FP64 CPU oracle for the FDM Exchange + Demag + Zeeman + LLG path.
 *
 * TEST INFRASTRUCTURE ONLY: loaded by tests/, the smoke check and the CPU
 * baseline leg of bench.py.  The product library does not link or call it.
 *
 * Restates, in C++ with OpenMP where the reference uses rayon:
 *   - crates/fullmag-engine/src/lib.rs  ExchangeLlgProblem (fields 2247-2445,
 *     RHS 2509-2600, energies 2653-2703, Heun 1217-1249, DP45 1412-1568,
 *     error norm 1653-1674, FFT driver fft3_core 2768-2812)
 *   - crates/fullmag-engine/src/vector.rs:12-76 (normalized, cross, ...)
 *   - crates/fullmag-fdm-demag/src/newell.rs:21-519 (Newell f/g, Kahan stencil,
 *     asymptotic far field, octant placement)
 *   - crates/fullmag-engine/src/lib.rs:337-406,511-610 (spectra)
 *   - crates/fullmag-plan/src/lib.rs:1928-1957 (random unit vectors)
 * Where the CPU engine has no counterpart, the CUDA backend's semantics are
 * restated: region exchange LUT (native/backends/fdm/src/exchange_fp64.cu:80-114)
 * and the forward-pair exchange energy (reductions_fp64.cu:122-214).
 * Extensions beyond the reference (documented semantics, parity unpinned vs the
 * reference): per-cell Ms map (Ms_i = 0 -> inactive) and a sinusoidal Zeeman
 * term evaluated at each stage time.
 *
 * The reference FFT is rustfft 6.4.1 (not vendored); this oracle uses its own
 * mixed-radix FP64 FFT, checked against numpy.fft by the tests.
 */
#include "oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstring>
#include <memory>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using cplx = std::complex<double>;
using V3 = std::array<double, 3>;

constexpr double PI = 3.14159265358979323846;
// crates/fullmag-engine/src/lib.rs:26  MU0 = 4.0 * PI * 1e-7
const double MU0 = 4.0 * PI * 1e-7;

// ---------------------------------------------------------------------------
// vector helpers (crates/fullmag-engine/src/vector.rs:12-76)
// ---------------------------------------------------------------------------
inline V3 add(V3 a, V3 b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
inline V3 sub(V3 a, V3 b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
inline V3 scale(V3 v, double f) { return {v[0] * f, v[1] * f, v[2] * f}; }
inline double dot(V3 a, V3 b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline V3 cross(V3 a, V3 b) {
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
inline double norm(V3 v) { return std::sqrt(dot(v, v)); }
inline V3 normalized(V3 v) {  // vector.rs:12-19: zero stays zero
    double n = norm(v);
    if (n <= 0.0) return {0.0, 0.0, 0.0};
    return scale(v, 1.0 / n);
}

// ---------------------------------------------------------------------------
// FFT: unnormalised mixed-radix DIT with direct DFT for prime factors.
// ---------------------------------------------------------------------------
struct FftPlan {
    size_t n = 0;
    int sign = -1;
    std::vector<cplx> tw;          // exp(sign*2*pi*i*j/n), j < n
    std::vector<size_t> factors;   // radix sequence, product = n

    FftPlan() = default;
    FftPlan(size_t n_, bool inverse) : n(n_), sign(inverse ? +1 : -1) {
        tw.resize(n);
        for (size_t j = 0; j < n; ++j) {
            double a = 2.0 * PI * (double)j / (double)n;
            tw[j] = cplx(std::cos(a), sign * std::sin(a));
        }
        size_t m = n;
        while (m > 1 && m % 4 == 0) { factors.push_back(4); m /= 4; }
        while (m > 1 && m % 2 == 0) { factors.push_back(2); m /= 2; }
        for (size_t p = 3; m > 1; p += 2) {
            while (m % p == 0) { factors.push_back(p); m /= p; }
        }
    }

    // out[k] for length len, reading in[j*stride]; fi = index into factors.
    void rec(const cplx *in, cplx *out, size_t len, size_t stride, size_t fi,
             cplx *scratch) const {
        if (len == 1) { out[0] = in[0]; return; }
        size_t p = factors[fi];
        size_t m = len / p;
        for (size_t r = 0; r < p; ++r)
            rec(in + r * stride, out + r * m, m, stride * p, fi + 1, scratch);
        size_t step = n / len;  // twiddle table step for W_len
        cplx tmp[64];
        std::vector<cplx> big;
        cplx *t = tmp;
        if (p > 64) { big.resize(p); t = big.data(); }
        for (size_t k = 0; k < m; ++k) {
            // apply W_len^{r k} to each sub-result
            for (size_t r = 0; r < p; ++r) {
                cplx v = out[r * m + k];
                if (r != 0 && k != 0) v *= tw[((r * k) % len) * step];
                t[r] = v;
            }
            for (size_t q = 0; q < p; ++q) {
                cplx acc = t[0];
                for (size_t r = 1; r < p; ++r)
                    acc += t[r] * tw[((r * q) % p) * (n / p)];
                scratch[q] = acc;
            }
            for (size_t q = 0; q < p; ++q) out[k + q * m] = scratch[q];
        }
    }

    bool pow2() const { return n >= 2 && (n & (n - 1)) == 0; }

    // Iterative Stockham autosort, radix 4 (one radix-2 pass when log2 n is odd),
    // ping-pong between data and work; same twiddle table as the recursive path.
    void execute_pow2(cplx *data, std::vector<cplx> &work) const {
        work.resize(n);
        cplx *a = data, *b = work.data();
        for (size_t Ns = 1; Ns < n;) {
            const size_t R = ((n / Ns) % 4 == 0) ? 4 : 2;
            const size_t m = n / R;
            const size_t tstep = n / (Ns * R);
            for (size_t jb = 0; jb < m; jb += Ns) {
                for (size_t k = 0; k < Ns; ++k) {
                    const size_t j = jb + k;
                    if (R == 4) {
                        cplx v0 = a[j], v1 = a[j + m], v2 = a[j + 2 * m], v3 = a[j + 3 * m];
                        if (k) {
                            v1 *= tw[k * tstep];
                            v2 *= tw[2 * k * tstep];
                            v3 *= tw[3 * k * tstep];
                        }
                        const cplx s02 = v0 + v2, d02 = v0 - v2, s13 = v1 + v3, d13 = v1 - v3;
                        // multiply d13 by -i (forward) or +i (inverse)
                        const cplx rot = (sign < 0) ? cplx(d13.imag(), -d13.real())
                                                    : cplx(-d13.imag(), d13.real());
                        cplx *o = b + jb * 4 + k;
                        o[0] = s02 + s13;
                        o[Ns] = d02 + rot;
                        o[2 * Ns] = s02 - s13;
                        o[3 * Ns] = d02 - rot;
                    } else {
                        cplx v0 = a[j], v1 = a[j + m];
                        if (k) v1 *= tw[k * tstep];
                        cplx *o = b + jb * 2 + k;
                        o[0] = v0 + v1;
                        o[Ns] = v0 - v1;
                    }
                }
            }
            std::swap(a, b);
            Ns *= R;
        }
        if (a != data) std::memcpy((void *)data, (const void *)a, n * sizeof(cplx));
    }

    void execute(cplx *data, std::vector<cplx> &work) const {
        if (n <= 1) return;
        if (pow2()) { execute_pow2(data, work); return; }
        work.resize(2 * n + 64);
        cplx *in = work.data();
        cplx *scratch = work.data() + n;
        std::memcpy((void *)in, (const void *)data, n * sizeof(cplx));
        rec(in, data, n, 1, 0, scratch);
    }
};

// fft3_core (crates/fullmag-engine/src/lib.rs:2768-2812): x lines, then y, then z.
// Serial by default, as in the reference; lines may be split over threads.
bool g_parallel_fft = false;

void fft3(cplx *data, size_t nx, size_t ny, size_t nz, const FftPlan &fx, const FftPlan &fy,
          const FftPlan &fz) {
    auto idx = [&](size_t x, size_t y, size_t z) { return x + nx * (y + ny * z); };
#pragma omp parallel if (g_parallel_fft)
    {
        std::vector<cplx> work, line;
#pragma omp for collapse(2)
        for (size_t z = 0; z < nz; ++z)
            for (size_t y = 0; y < ny; ++y) fx.execute(data + idx(0, y, z), work);
        line.resize(std::max(ny, nz));
#pragma omp for collapse(2)
        for (size_t z = 0; z < nz; ++z)
            for (size_t x = 0; x < nx; ++x) {
                if (ny == 1) continue;
                for (size_t y = 0; y < ny; ++y) line[y] = data[idx(x, y, z)];
                fy.execute(line.data(), work);
                for (size_t y = 0; y < ny; ++y) data[idx(x, y, z)] = line[y];
            }
#pragma omp for collapse(2)
        for (size_t y = 0; y < ny; ++y)
            for (size_t x = 0; x < nx; ++x) {
                if (nz == 1) continue;
                for (size_t z = 0; z < nz; ++z) line[z] = data[idx(x, y, z)];
                fz.execute(line.data(), work);
                for (size_t z = 0; z < nz; ++z) data[idx(x, y, z)] = line[z];
            }
    }
}

// ---------------------------------------------------------------------------
// Newell tensor (crates/fullmag-fdm-demag/src/newell.rs)
// ---------------------------------------------------------------------------
double newell_f(double x, double y, double z) {  // newell.rs:21-57
    double x2 = x * x, y2 = y * y, z2 = z * z;
    double r2 = x2 + y2 + z2;
    if (r2 < 1e-300) return 0.0;
    double r = std::sqrt(r2);
    double result = (2.0 * x2 - y2 - z2) * r / 6.0;
    double rxz2 = x2 + z2;
    if (rxz2 > 1e-300) {
        double arg = 2.0 * y * (y + r) / rxz2;
        if (arg > -1.0) result += y * (z2 - x2) / 4.0 * std::log1p(arg);
    }
    double rxy2 = x2 + y2;
    if (rxy2 > 1e-300) {
        double arg = 2.0 * z * (z + r) / rxy2;
        if (arg > -1.0) result += z * (y2 - x2) / 4.0 * std::log1p(arg);
    }
    if (std::fabs(x) > 1e-300) result -= x * y * z * std::atan(y * z / (x * r));
    return result;
}

double newell_g(double x, double y, double z) {  // newell.rs:62-121
    double x2 = x * x, y2 = y * y, z2 = z * z;
    double r2 = x2 + y2 + z2;
    if (r2 < 1e-300) return 0.0;
    double r = std::sqrt(r2);
    double result = -x * y * r / 3.0;
    double rxy2 = x2 + y2;
    if (rxy2 > 1e-300) {
        double arg = 2.0 * z * (z + r) / rxy2;
        if (arg > -1.0) result += x * y * z * std::log1p(arg) / 2.0;
    }
    double ryz2 = y2 + z2;
    if (ryz2 > 1e-300) {
        double arg = 2.0 * x * (x + r) / ryz2;
        if (arg > -1.0) result += y * (3.0 * z2 - y2) * std::log1p(arg) / 12.0;
    }
    double rxz2 = x2 + z2;
    if (rxz2 > 1e-300) {
        double arg = 2.0 * y * (y + r) / rxz2;
        if (arg > -1.0) result += x * (3.0 * z2 - x2) * std::log1p(arg) / 12.0;
    }
    if (std::fabs(z) > 1e-300) result -= z2 * z / 6.0 * std::atan(x * y / (z * r));
    if (std::fabs(y) > 1e-300) result -= y2 * z / 2.0 * std::atan(x * z / (y * r));
    if (std::fabs(x) > 1e-300) result -= x2 * z / 2.0 * std::atan(y * z / (x * r));
    return result;
}

double kahan_sum(const double *terms, int n) {  // newell.rs:133-147 (Kahan–Neumaier)
    double sum = 0.0, comp = 0.0;
    for (int i = 0; i < n; ++i) {
        double val = terms[i];
        double t = sum + val;
        if (std::fabs(sum) >= std::fabs(val)) comp += (sum - t) + val;
        else comp += (val - t) + sum;
        sum = t;
    }
    return sum + comp;
}

// 27-point stencil, newell.rs:151-203; f is stored with a +1 index offset.
double ldia(size_t i, size_t j, size_t k, const std::vector<double> &f, size_t sx, size_t sy,
            double hx, double hy, double hz) {
    i += 1; j += 1; k += 1;
    auto F = [&](size_t a, size_t b, size_t c) { return f[c * sy * sx + b * sx + a]; };
    double t[27] = {
        8.0 * F(i, j, k),
        -4.0 * F(i + 1, j, k), -4.0 * F(i - 1, j, k), -4.0 * F(i, j + 1, k),
        -4.0 * F(i, j - 1, k), -4.0 * F(i, j, k + 1), -4.0 * F(i, j, k - 1),
        2.0 * F(i - 1, j - 1, k), 2.0 * F(i - 1, j + 1, k), 2.0 * F(i + 1, j - 1, k),
        2.0 * F(i + 1, j + 1, k), 2.0 * F(i - 1, j, k - 1), 2.0 * F(i - 1, j, k + 1),
        2.0 * F(i + 1, j, k - 1), 2.0 * F(i + 1, j, k + 1), 2.0 * F(i, j - 1, k - 1),
        2.0 * F(i, j - 1, k + 1), 2.0 * F(i, j + 1, k - 1), 2.0 * F(i, j + 1, k + 1),
        -F(i - 1, j - 1, k - 1), -F(i - 1, j - 1, k + 1), -F(i - 1, j + 1, k - 1),
        -F(i + 1, j - 1, k - 1), -F(i - 1, j + 1, k + 1), -F(i + 1, j - 1, k + 1),
        -F(i + 1, j + 1, k - 1), -F(i + 1, j + 1, k + 1),
    };
    return kahan_sum(t, 27) / (4.0 * PI * hx * hy * hz);
}

double asym_nxx(double x, double y, double z, double vol) {  // newell.rs:212-218
    double r2 = x * x + y * y + z * z;
    double r = std::sqrt(r2);
    double r3 = r2 * r;
    return (1.0 / r3 - 3.0 * x * x / (r3 * r2)) / (4.0 * PI) * vol;
}
double asym_nxy(double x, double y, double z, double vol) {  // newell.rs:222-228
    double r2 = x * x + y * y + z * z;
    double r = std::sqrt(r2);
    double r5 = r2 * r2 * r;
    return -3.0 * x * y / (4.0 * PI * r5) * vol;
}
constexpr size_t ASYMPTOTIC_DISTANCE = 40;  // newell.rs:231

// compute_newell_kernels (newell.rs:254-519): out6 = xx,yy,zz,xy,xz,yz on (2nx,2ny,2nz)
void newell_kernels(size_t nx, size_t ny, size_t nz, double dx, double dy, double dz,
                    double *out6) {
    size_t px = 2 * nx, py = 2 * ny, pz = 2 * nz;
    size_t plen = px * py * pz;
    size_t nxd = std::min(nx, ASYMPTOTIC_DISTANCE), nyd = std::min(ny, ASYMPTOTIC_DISTANCE),
           nzd = std::min(nz, ASYMPTOTIC_DISTANCE);
    size_t fsx = nxd + 2, fsy = nyd + 2, fsz = nzd + 2, flen = fsx * fsy * fsz;
    std::vector<double> fxx(flen), fyy(flen), fzz(flen), gxy(flen), gxz(flen), gyz(flen);
#pragma omp parallel for
    for (long kk = 0; kk < (long)fsz; ++kk)
        for (size_t j = 0; j < fsy; ++j)
            for (size_t i = 0; i < fsx; ++i) {
                double x = ((long)i - 1) * dx, y = ((long)j - 1) * dy, z = (kk - 1) * dz;
                size_t b = (size_t)kk * fsx * fsy + j * fsx + i;
                fxx[b] = newell_f(x, y, z);
                fyy[b] = newell_f(y, x, z);
                fzz[b] = newell_f(z, y, x);
                gxy[b] = newell_g(x, y, z);
                gxz[b] = newell_g(x, z, y);
                gyz[b] = newell_g(y, z, x);
            }
    double *nxx = out6, *nyy = out6 + plen, *nzz = out6 + 2 * plen, *nxy = out6 + 3 * plen,
           *nxz = out6 + 4 * plen, *nyz = out6 + 5 * plen;
    std::fill(out6, out6 + 6 * plen, 0.0);
#pragma omp parallel for
    for (long kl = 0; kl < (long)nz; ++kl) {
        size_t k = (size_t)kl;
        for (size_t j = 0; j < ny; ++j)
            for (size_t i = 0; i < nx; ++i) {
                double vxx, vyy, vzz, vxy, vxz, vyz;
                size_t d2 = i * i + j * j + k * k;
                bool asym = i >= ASYMPTOTIC_DISTANCE || j >= ASYMPTOTIC_DISTANCE ||
                            k >= ASYMPTOTIC_DISTANCE ||
                            d2 >= ASYMPTOTIC_DISTANCE * ASYMPTOTIC_DISTANCE;
                if (asym) {
                    double x = i * dx, y = j * dy, z = k * dz, vol = dx * dy * dz;
                    vxx = asym_nxx(x, y, z, vol);
                    vyy = asym_nxx(y, x, z, vol);
                    vzz = asym_nxx(z, y, x, vol);
                    vxy = asym_nxy(x, y, z, vol);
                    vxz = asym_nxy(x, z, y, vol);
                    vyz = asym_nxy(y, z, x, vol);
                } else {
                    vxx = ldia(i, j, k, fxx, fsx, fsy, dx, dy, dz);
                    vyy = ldia(i, j, k, fyy, fsx, fsy, dy, dx, dz);
                    vzz = ldia(i, j, k, fzz, fsx, fsy, dz, dy, dx);
                    vxy = ldia(i, j, k, gxy, fsx, fsy, dx, dy, dz);
                    vxz = ldia(i, j, k, gxz, fsx, fsy, dx, dz, dy);
                    vyz = ldia(i, j, k, gyz, fsx, fsy, dy, dz, dx);
                }
                // octant placement with parity (newell.rs:397-426)
                size_t xs[2] = {i, px - i}, ys[2] = {j, py - j}, zs[2] = {k, pz - k};
                double sxs[2] = {1.0, -1.0};
                int nxs = i == 0 ? 1 : 2, nys = j == 0 ? 1 : 2, nzs = k == 0 ? 1 : 2;
                for (int a = 0; a < nxs; ++a)
                    for (int b = 0; b < nys; ++b)
                        for (int c = 0; c < nzs; ++c) {
                            size_t p = zs[c] * py * px + ys[b] * px + xs[a];
                            nxx[p] = vxx;
                            nyy[p] = vyy;
                            nzz[p] = vzz;
                            nxy[p] = vxy * sxs[a] * sxs[b];
                            nxz[p] = vxz * sxs[a] * sxs[c];
                            nyz[p] = vyz * sxs[b] * sxs[c];
                        }
            }
    }
}

// ---------------------------------------------------------------------------
// Problem (ExchangeLlgProblem + state + workspace)
// ---------------------------------------------------------------------------
struct Problem {
    oracle_desc d{};
    size_t nx, ny, nz, n;
    std::vector<uint8_t> mask;      // empty = all active
    std::vector<uint32_t> region;   // empty = none
    std::vector<double> lut;        // 256*256 when regions present
    std::vector<double> msmap;      // empty = uniform
    std::vector<V3> m;
    double t = 0.0;
    bool fsal_valid = false;
    std::vector<V3> fsal;
    // ABM3 history (AbmHistory, lib.rs:628-687): f_n, f_{n-1}, f_{n-2}
    std::vector<V3> abm_fn, abm_fn1, abm_fn2;
    int abm_startup = 0;
    double abm_last_dt = 0.0;
    // FFT workspace (FftWorkspace, lib.rs:288-380)
    size_t px = 0, py = 0, pz = 0, plen = 0;
    FftPlan fwx, fwy, fwz, ivx, ivy, ivz;
    std::vector<cplx> kxx, kyy, kzz, kxy, kxz, kyz;
    std::vector<cplx> bmx, bmy, bmz, bhx, bhy, bhz;

    bool active(size_t i) const {
        if (!mask.empty() && mask[i] == 0) return false;
        if (!msmap.empty() && !(msmap[i] > 0.0)) return false;
        return true;
    }
    double ms_at(size_t i) const { return msmap.empty() ? d.ms : msmap[i]; }

    // Boundary tiers, with the reference's launch conditions
    // (exchange_fp64.cu:159-198, demag_fp64.cu:299, 364): the T0 exchange needs
    // the face links, the T1 exchange the distances; phi-weighted demag needs
    // only the volume fraction; the sparse correction needs a tier.
    std::vector<double> vf, face[6], delta[6];
    std::vector<int32_t> ctgt, csrc;
    std::vector<double> cten;
    int ex_tier = 0;
    double phi_floor = 0.05, delta_min = 0.0;
    size_t index(size_t x, size_t y, size_t z) const { return x + nx * (y + ny * z); }

    V3 hext_at(double time) const {
        V3 h = {d.h_ext[0], d.h_ext[1], d.h_ext[2]};
        if (d.ac_freq != 0.0 || d.h_ac[0] != 0.0 || d.h_ac[1] != 0.0 || d.h_ac[2] != 0.0) {
            double s = std::sin(2.0 * PI * d.ac_freq * time);
            h = add(h, scale(V3{d.h_ac[0], d.h_ac[1], d.h_ac[2]}, s));
        }
        return h;
    }
    bool has_ext() const {
        return d.has_external_field != 0;
    }

    void init_workspace() {
        if (!d.enable_demag) return;
        px = 2 * nx; py = 2 * ny; pz = d.thin_film_2d ? 1 : 2 * nz;
        plen = px * py * pz;
        fwx = FftPlan(px, false); fwy = FftPlan(py, false); fwz = FftPlan(pz, false);
        ivx = FftPlan(px, true); ivy = FftPlan(py, true); ivz = FftPlan(pz, true);
        std::vector<double> sp(12 * plen);
        oracle_newell_spectra((uint32_t)nx, (uint32_t)ny, (uint32_t)nz, d.dx, d.dy, d.dz,
                              d.thin_film_2d, sp.data(), sp.data() + 2 * plen,
                              sp.data() + 4 * plen, sp.data() + 6 * plen, sp.data() + 8 * plen,
                              sp.data() + 10 * plen);
        auto take = [&](int c, std::vector<cplx> &dst) {
            dst.resize(plen);
            const double *s = sp.data() + 2 * plen * c;
            for (size_t i = 0; i < plen; ++i) dst[i] = cplx(s[2 * i], s[2 * i + 1]);
        };
        if (d.symmetric_kernel) symmetrize(sp);
        take(0, kxx); take(1, kyy); take(2, kzz); take(3, kxy); take(4, kxz); take(5, kyz);
        for (auto *b : {&bmx, &bmy, &bmz, &bhx, &bhy, &bhz}) b->assign(plen, cplx(0, 0));
    }

    // Replace each interleaved spectrum by its exactly even/odd real part: the
    // value at the octant (k <= L/2 per axis) mirrored with the component's parity.
    void symmetrize(std::vector<double> &sp) const {
        const int oddx[6] = {0, 0, 0, 1, 1, 0}, oddy[6] = {0, 0, 0, 1, 0, 1}, oddz[6] = {0, 0, 0, 0, 1, 1};
        std::vector<double> re(plen);
        for (int c = 0; c < 6; ++c) {
            double *s = sp.data() + 2 * plen * c;
            const bool imag2d = d.thin_film_2d && (oddx[c] != oddy[c]);
            for (size_t i = 0; i < plen; ++i) re[i] = s[2 * i];
            for (size_t kz = 0; kz < pz; ++kz)
                for (size_t ky = 0; ky < py; ++ky)
                    for (size_t kx = 0; kx < px; ++kx) {
                        const size_t kxo = kx <= px / 2 ? kx : px - kx;
                        const size_t kyo = ky <= py / 2 ? ky : py - ky;
                        const size_t kzo = kz <= pz / 2 ? kz : pz - kz;
                        double sg = 1.0;
                        if (kx > px / 2 && oddx[c]) sg = -sg;
                        if (ky > py / 2 && oddy[c]) sg = -sg;
                        if (kz > pz / 2 && oddz[c]) sg = -sg;
                        const size_t i = kx + px * (ky + py * kz);
                        s[2 * i] = imag2d ? 0.0 : sg * re[kxo + px * (kyo + py * kzo)];
                        s[2 * i + 1] = 0.0;
                    }
        }
    }

    // exchange_field_from_vectors (lib.rs:2247-2299) + region LUT (exchange_fp64.cu:80-114)
    // T0, exchange_t0_fp64.cu:22-133: face-link-weighted differences over the
    // faces in the order -x, +x, -y, +y, -z, +z, normalised by max(phi, floor).
    // T1, exchange_t1_fp64.cu:28-175: the ECB stencil 2 / (d (d + delta_opposite))
    // per interior neighbour with non-zero m, deltas clamped below by delta_min.
    // Cells with phi <= 0 or m = 0 get H_ex = 0 (the reference leaves them unwritten).
    void exchange_tier(const std::vector<V3> &mm, std::vector<V3> &out) const {
        const double i2[3] = {1.0 / (d.dx * d.dx), 1.0 / (d.dy * d.dy), 1.0 / (d.dz * d.dz)};
        const double dd[3] = {d.dx, d.dy, d.dz};
        const double scale0 = 2.0 * d.aex / (MU0 * d.ms);
#pragma omp parallel for
        for (long fl = 0; fl < (long)n; ++fl) {
            size_t f = (size_t)fl;
            out[f] = {0, 0, 0};
            if (!active(f)) continue;
            const V3 c = mm[f];
            const double phi0 = vf[f];
            if (phi0 <= 0.0 || (c[0] == 0.0 && c[1] == 0.0 && c[2] == 0.0)) continue;
            size_t xyz[3] = {f % nx, (f / nx) % ny, f / (nx * ny)};
            const size_t ext[3] = {nx, ny, nz};
            const size_t stride[3] = {1, nx, nx * ny};
            V3 b = {0, 0, 0};
            for (int ax = 0; ax < 3; ++ax) {
                if (ax == 2 && nz <= 1) break;
                const bool has_m = xyz[ax] > 0, has_p = xyz[ax] + 1 < ext[ax];
                if (ex_tier == 1) {
                    const double fm = face[2 * ax + 1][f], fp = face[2 * ax][f];
                    if (fm > 0.0 && has_m) {
                        const V3 &mn = mm[f - stride[ax]];
                        for (int cc = 0; cc < 3; ++cc) b[cc] += fm * i2[ax] * (mn[cc] - c[cc]);
                    }
                    if (fp > 0.0 && has_p) {
                        const V3 &mn = mm[f + stride[ax]];
                        for (int cc = 0; cc < 3; ++cc) b[cc] += fp * i2[ax] * (mn[cc] - c[cc]);
                    }
                } else {
                    const double dm = std::max(delta[2 * ax + 1][f], delta_min);
                    const double dp = std::max(delta[2 * ax][f], delta_min);
                    if (has_m && dm > 0.0) {
                        const V3 &mn = mm[f - stride[ax]];
                        if (mn[0] != 0.0 || mn[1] != 0.0 || mn[2] != 0.0) {
                            const double coeff = 2.0 / (dd[ax] * (dd[ax] + dp));
                            for (int cc = 0; cc < 3; ++cc) b[cc] += coeff * (mn[cc] - c[cc]);
                        }
                    }
                    if (has_p && dp > 0.0) {
                        const V3 &mn = mm[f + stride[ax]];
                        if (mn[0] != 0.0 || mn[1] != 0.0 || mn[2] != 0.0) {
                            const double coeff = 2.0 / (dd[ax] * (dd[ax] + dm));
                            for (int cc = 0; cc < 3; ++cc) b[cc] += coeff * (mn[cc] - c[cc]);
                        }
                    }
                }
            }
            const double sc = ex_tier == 1 ? scale0 * (1.0 / (phi0 > phi_floor ? phi0 : phi_floor)) : scale0;
            out[f] = scale(b, sc);
        }
    }

    void exchange_field(const std::vector<V3> &mm, std::vector<V3> &out) const {
        out.assign(n, V3{0, 0, 0});
        if (!d.enable_exchange) return;
        if (ex_tier) { exchange_tier(mm, out); return; }
        double dx2 = d.dx * d.dx, dy2 = d.dy * d.dy, dz2 = d.dz * d.dz;
#pragma omp parallel for
        for (long fl = 0; fl < (long)n; ++fl) {
            size_t f = (size_t)fl;
            if (!active(f)) { out[f] = {0, 0, 0}; continue; }
            size_t x = f % nx, y = (f / nx) % ny, z = f / (nx * ny);
            V3 c = mm[f];
            size_t nb[6] = {index(x > 0 ? x - 1 : 0, y, z), index(std::min(x + 1, nx - 1), y, z),
                            index(x, y > 0 ? y - 1 : 0, z), index(x, std::min(y + 1, ny - 1), z),
                            index(x, y, z > 0 ? z - 1 : 0), index(x, y, std::min(z + 1, nz - 1))};
            V3 v[6];
            for (int q = 0; q < 6; ++q) v[q] = active(nb[q]) ? mm[nb[q]] : c;
            if (region.empty()) {
                double pref = 2.0 * d.aex / (MU0 * ms_at(f));
                V3 lap;
                for (int cc = 0; cc < 3; ++cc)
                    lap[cc] = (v[1][cc] - 2.0 * c[cc] + v[0][cc]) / dx2 +
                              (v[3][cc] - 2.0 * c[cc] + v[2][cc]) / dy2 +
                              (v[5][cc] - 2.0 * c[cc] + v[4][cc]) / dz2;
                out[f] = scale(lap, pref);
            } else {
                // Per-pair A_ij: neighbour replaced by the centre contributes zero.
                uint32_t rc = region[f];
                double a[6];
                for (int q = 0; q < 6; ++q) {
                    size_t nq = active(nb[q]) ? nb[q] : f;
                    a[q] = lut[(size_t)rc * 256 + region[nq]];
                }
                double inv[3] = {1.0 / dx2, 1.0 / dy2, 1.0 / dz2};
                double pref = 2.0 / (MU0 * ms_at(f));
                // summation order of exchange_fp64.cu:102-112: xp, xm, yp, ym, zp, zm
                const int order[6] = {1, 0, 3, 2, 5, 4};
                V3 h;
                for (int cc = 0; cc < 3; ++cc) {
                    double s = 0.0;
                    for (int o = 0; o < 6; ++o) {
                        const int q = order[o];
                        s += a[q] * (v[q][cc] - c[cc]) * inv[q / 2];
                    }
                    h[cc] = pref * s;
                }
                out[f] = h;
            }
        }
    }

    // demag_field_from_vectors_ws (lib.rs:2306-2400)
    void demag_field(const std::vector<V3> &mm, std::vector<V3> &out) {
        out.assign(n, V3{0, 0, 0});
        if (!d.enable_demag) return;
        for (auto *b : {&bmx, &bmy, &bmz, &bhx, &bhy, &bhz}) std::fill(b->begin(), b->end(), cplx(0, 0));
        for (size_t z = 0; z < nz; ++z)
            for (size_t y = 0; y < ny; ++y)
                for (size_t x = 0; x < nx; ++x) {
                    size_t s = index(x, y, z);
                    size_t dd = x + px * (y + py * z);
                    // phi-weighted packing M = (phi Ms) m over every cell when a tier
                    // is set (demag_fp64.cu:79-85), else the mask
                    V3 mo = !vf.empty() ? scale(mm[s], vf[s] * ms_at(s))
                            : active(s) ? scale(mm[s], ms_at(s)) : V3{0, 0, 0};
                    bmx[dd] = cplx(mo[0], 0.0);
                    bmy[dd] = cplx(mo[1], 0.0);
                    bmz[dd] = cplx(mo[2], 0.0);
                }
        fft3(bmx.data(), px, py, pz, fwx, fwy, fwz);
        fft3(bmy.data(), px, py, pz, fwx, fwy, fwz);
        fft3(bmz.data(), px, py, pz, fwx, fwy, fwz);
#pragma omp parallel for
        for (long il = 0; il < (long)plen; ++il) {
            size_t i = (size_t)il;
            cplx mx = bmx[i], my = bmy[i], mz = bmz[i];
            bhx[i] = -(kxx[i] * mx + kxy[i] * my + kxz[i] * mz);
            bhy[i] = -(kxy[i] * mx + kyy[i] * my + kyz[i] * mz);
            bhz[i] = -(kxz[i] * mx + kyz[i] * my + kzz[i] * mz);
        }
        fft3(bhx.data(), px, py, pz, ivx, ivy, ivz);
        fft3(bhy.data(), px, py, pz, ivx, ivy, ivz);
        fft3(bhz.data(), px, py, pz, ivx, ivy, ivz);
        double norm_ = 1.0 / (double)plen;
        for (size_t z = 0; z < nz; ++z)
            for (size_t y = 0; y < ny; ++y)
                for (size_t x = 0; x < nx; ++x) {
                    size_t s = x + px * (y + py * z);
                    size_t dd = index(x, y, z);
                    out[dd] = active(dd) ? V3{bhx[s].real() * norm_, bhy[s].real() * norm_,
                                              bhz[s].real() * norm_}
                                         : V3{0, 0, 0};
                }
        // sparse boundary correction H(t) -= dN(t, s) M(s), demag_boundary_fp64.cu:20-76
        const size_t S = d.corr_stencil;
        for (size_t t = 0; t < ctgt.size(); ++t) {
            const int32_t ti = ctgt[t];
            if (ti < 0) continue;
            V3 ch = {0, 0, 0};
            for (size_t q = 0; q < S; ++q) {
                const int32_t si = csrc[t * S + q];
                if (si < 0) continue;
                const double *N = &cten[(t * S + q) * 6];
                const V3 M = scale(mm[(size_t)si], vf[(size_t)si] * ms_at((size_t)si));
                ch[0] -= N[0] * M[0] + N[1] * M[1] + N[2] * M[2];
                ch[1] -= N[1] * M[0] + N[3] * M[1] + N[4] * M[2];
                ch[2] -= N[2] * M[0] + N[4] * M[1] + N[5] * M[2];
            }
            out[(size_t)ti] = add(out[(size_t)ti], ch);
        }
    }

    void external_field(double time, std::vector<V3> &out) const {
        V3 h = has_ext() ? hext_at(time) : V3{0, 0, 0};
        out.resize(n);
        for (size_t i = 0; i < n; ++i) out[i] = active(i) ? h : V3{0, 0, 0};
    }

    // llg_rhs_from_field (lib.rs:2589-2600)
    V3 rhs_from_field(V3 mv, V3 h) const {
        double alpha = d.alpha;
        double gamma_bar = d.gamma / (1.0 + alpha * alpha);
        V3 prec = cross(mv, h);
        V3 damp = cross(mv, prec);
        V3 pt = d.precession_enabled ? prec : V3{0, 0, 0};
        return scale(add(pt, scale(damp, alpha)), -gamma_bar);
    }

    struct Fields { std::vector<V3> ex, dm, ext, eff, rhs; };

    void evaluate(const std::vector<V3> &mm, double time, Fields &F) {
        exchange_field(mm, F.ex);
        demag_field(mm, F.dm);
        external_field(time, F.ext);
        F.eff.resize(n);
        F.rhs.resize(n);
#pragma omp parallel for
        for (long il = 0; il < (long)n; ++il) {
            size_t i = (size_t)il;
            F.eff[i] = add(add(F.ex[i], F.dm[i]), F.ext[i]);  // combine_fields, lib.rs:2836-2843
            F.rhs[i] = rhs_from_field(mm[i], F.eff[i]);
        }
    }

    void rhs_into(const std::vector<V3> &mm, double time, std::vector<V3> &out) {
        Fields F;
        evaluate(mm, time, F);
        out.swap(F.rhs);
    }

    static double max_norm(const std::vector<V3> &v) {
        double mx = 0.0;
#pragma omp parallel for reduction(max : mx)
        for (long i = 0; i < (long)v.size(); ++i) mx = std::max(mx, norm(v[(size_t)i]));
        return mx;
    }

    double exchange_pair_energy(const std::vector<V3> &mm) const {  // reductions_fp64.cu:122-214
        if (!d.enable_exchange) return 0.0;
        double vol = d.dx * d.dy * d.dz;
        double inv[3] = {1.0 / (d.dx * d.dx), 1.0 / (d.dy * d.dy), 1.0 / (d.dz * d.dz)};
        double e = 0.0;
#pragma omp parallel for reduction(+ : e)
        for (long fl = 0; fl < (long)n; ++fl) {
            size_t f = (size_t)fl;
            if (!active(f)) continue;
            size_t x = f % nx, y = (f / nx) % ny, z = f / (nx * ny);
            size_t nbs[3] = {x + 1 < nx ? f + 1 : f, y + 1 < ny ? f + nx : f,
                             z + 1 < nz ? f + nx * ny : f};
            for (int q = 0; q < 3; ++q) {
                size_t nq = nbs[q];
                if (nq == f || !active(nq)) continue;
                double coeff = region.empty() ? d.aex * vol
                                              : lut[(size_t)region[f] * 256 + region[nq]] * vol;
                V3 df = sub(mm[nq], mm[f]);
                e += coeff * dot(df, df) * inv[q];
            }
        }
        return e;
    }

    // llg_rhs_full_ws (lib.rs:2529-2582): energies and max norms at a state.
    void diagnostics(const std::vector<V3> &mm, double time, Fields &F, oracle_report &r) {
        evaluate(mm, time, F);
        double vol = d.dx * d.dy * d.dz;
        double eex = 0.0, edm = 0.0, eext = 0.0;
#pragma omp parallel for reduction(+ : eex, edm, eext)
        for (long il = 0; il < (long)n; ++il) {
            size_t i = (size_t)il;
            double ms = ms_at(i);
            eex += -0.5 * MU0 * ms * dot(mm[i], F.ex[i]) * vol;
            edm += -0.5 * MU0 * ms * dot(mm[i], F.dm[i]) * vol;
            eext += -MU0 * ms * dot(mm[i], F.ext[i]) * vol;
        }
        r.e_ex_field = d.enable_exchange ? eex : 0.0;
        r.e_ex_pair = exchange_pair_energy(mm);
        r.e_demag = d.enable_demag ? edm : 0.0;
        r.e_ext = has_ext() ? eext : 0.0;
        r.e_total = r.e_ex_field + r.e_demag + r.e_ext;
        r.max_h_eff = max_norm(F.eff);
        r.max_h_demag = max_norm(F.dm);
        r.max_rhs = max_norm(F.rhs);
    }

    // heun_step_buf (lib.rs:1217-1249)
    void heun(double dt, oracle_report &r) {
        std::vector<V3> m0 = m, k1, k2, mp(n);
        rhs_into(m0, t, k1);
#pragma omp parallel for
        for (long i = 0; i < (long)n; ++i)
            mp[(size_t)i] = normalized(add(m0[(size_t)i], scale(k1[(size_t)i], dt)));
        rhs_into(mp, t + dt, k2);
#pragma omp parallel for
        for (long il = 0; il < (long)n; ++il) {
            size_t i = (size_t)il;
            m[i] = normalized(add(m0[i], scale(add(k1[i], k2[i]), 0.5 * dt)));
        }
        t += dt;
        Fields F;
        diagnostics(m, t, F, r);
        r.time_seconds = t;
        r.dt_used = dt;
        r.suggested_next_dt = 0.0;
    }

    // Stage state normalize(m0 + inc(i)) into ms.
    template <class Inc>
    void stage_state(const std::vector<V3> &m0, Inc inc, std::vector<V3> &ms) {
#pragma omp parallel for
        for (long il = 0; il < (long)n; ++il) {
            size_t i = (size_t)il;
            ms[i] = normalized(add(m0[i], inc(i)));
        }
    }

    // rk4_step_buf (lib.rs:1253-1297); stage times t, t + dt/2, t + dt/2, t + dt
    // for the time-dependent Zeeman extension.
    void rk4(double dt, oracle_report &r) {
        std::vector<V3> m0 = m, k1, k2, k3, k4, ms(n);
        rhs_into(m0, t, k1);
        stage_state(m0, [&](size_t i) { return scale(k1[i], 0.5 * dt); }, ms);
        rhs_into(ms, t + 0.5 * dt, k2);
        stage_state(m0, [&](size_t i) { return scale(k2[i], 0.5 * dt); }, ms);
        rhs_into(ms, t + 0.5 * dt, k3);
        stage_state(m0, [&](size_t i) { return scale(k3[i], dt); }, ms);
        rhs_into(ms, t + dt, k4);
        stage_state(m0, [&](size_t i) {
            return scale(add(add(k1[i], scale(k2[i], 2.0)), add(scale(k3[i], 2.0), k4[i])), dt / 6.0);
        }, m);
        t += dt;
        Fields F;
        diagnostics(m, t, F, r);
        r.time_seconds = t;
        r.dt_used = dt;
        r.suggested_next_dt = 0.0;
    }

    // max_error_norm_buf (lib.rs:1653-1674): max_i |dt sum_j w_j k_j[i]|, the
    // sum accumulated from zero in the listed order.
    double error_norm(std::initializer_list<std::pair<const std::vector<V3> *, double>> ws, double dt) {
        double err = 0.0;
#pragma omp parallel for reduction(max : err)
        for (long il = 0; il < (long)n; ++il) {
            size_t i = (size_t)il;
            V3 e = {0, 0, 0};
            for (auto &w : ws) {
                e[0] += w.second * (*w.first)[i][0];
                e[1] += w.second * (*w.first)[i][1];
                e[2] += w.second * (*w.first)[i][2];
            }
            e[0] *= dt; e[1] *= dt; e[2] *= dt;
            err = std::max(err, norm(e));
        }
        return err;
    }

    // rk23_step_buf (lib.rs:1332-1407), Bogacki-Shampine 2(3): k1 is evaluated
    // at m0 on every attempt (the same values each time); stage times t,
    // t + dt/2, t + 3dt/4, t + dt.
    void rk23(double dt_in, oracle_report &r) {
        double max_error = d.max_error > 0 ? d.max_error : 1e-5;
        double dt_min = d.dt_min > 0 ? d.dt_min : 1e-18;
        double dt_max = d.dt_max > 0 ? d.dt_max : 1e-10;
        double headroom = d.headroom > 0 ? d.headroom : 0.8;
        double dt = std::max(std::min(dt_in, dt_max), dt_min);
        std::vector<V3> m0 = m, k1, k2, k3, k4, ms(n);
        int rejected = 0;
        for (;;) {
            rhs_into(m0, t, k1);
            stage_state(m0, [&](size_t i) { return scale(k1[i], 0.5 * dt); }, ms);
            rhs_into(ms, t + 0.5 * dt, k2);
            stage_state(m0, [&](size_t i) { return scale(k2[i], 0.75 * dt); }, ms);
            rhs_into(ms, t + 0.75 * dt, k3);
            stage_state(m0, [&](size_t i) {
                return scale(add(add(scale(k1[i], 2.0 / 9.0), scale(k2[i], 1.0 / 3.0)), scale(k3[i], 4.0 / 9.0)), dt);
            }, ms);
            rhs_into(ms, t + dt, k4);
            const double err = error_norm({{&k1, -5.0 / 72.0}, {&k2, 1.0 / 12.0}, {&k3, 1.0 / 9.0}, {&k4, -1.0 / 8.0}}, dt);
            if (err <= max_error || dt <= dt_min) {
                m = ms;
                t += dt;
                const double dt_next = std::min(
                    std::max(headroom * dt * std::pow(max_error / std::max(err, 1e-30), 1.0 / 3.0), dt_min), dt_max);
                Fields F;
                diagnostics(m, t, F, r);
                r.time_seconds = t;
                r.dt_used = dt;
                r.suggested_next_dt = dt_next;
                r.rejected_attempts = rejected;
                return;
            }
            ++rejected;
            const double dt_new = headroom * dt * std::pow(max_error / err, 1.0 / 3.0);
            dt = std::min(std::max(dt_new, dt_min), dt_max);
        }
    }

    // abm3_step_buf (lib.rs:1573-1648): three Heun start-up steps push
    // f(m_{n+1}); then AB3 predictor, f* = f(predicted), AM3 corrector, push f*.
    // A dt that differs from the last one by more than 10 % restarts the
    // history before the step, as the reference's CUDA backend does
    // (native/backends/fdm/src/llg_abm3_fp64.cu:177-180); the CPU engine checks
    // at the push after the step (lib.rs:672-676).  Both agree for constant dt.
    void abm_push(std::vector<V3> f, double dt) {
        abm_fn2 = std::move(abm_fn1);
        abm_fn1 = std::move(abm_fn);
        abm_fn = std::move(f);
        abm_startup = std::min(abm_startup + 1, 3);
        abm_last_dt = dt;
    }

    void abm3(double dt, oracle_report &r) {
        if (abm_last_dt > 0.0 && std::fabs(dt - abm_last_dt) / abm_last_dt > 0.1) abm_startup = 0;
        std::vector<V3> m0 = m, ms(n);
        if (abm_startup < 3) {
            std::vector<V3> k1, k2, fa;
            rhs_into(m0, t, k1);
            stage_state(m0, [&](size_t i) { return scale(k1[i], dt); }, ms);
            rhs_into(ms, t + dt, k2);
            stage_state(m0, [&](size_t i) { return scale(add(k1[i], k2[i]), 0.5 * dt); }, m);
            t += dt;
            rhs_into(m, t, fa);
            abm_push(std::move(fa), dt);
        } else {
            const std::vector<V3> &fn = abm_fn, &fn1 = abm_fn1, &fn2 = abm_fn2;
            std::vector<V3> fs;
            stage_state(m0, [&](size_t i) {
                return scale(add(add(scale(fn[i], 23.0 / 12.0), scale(fn1[i], -16.0 / 12.0)), scale(fn2[i], 5.0 / 12.0)), dt);
            }, ms);
            rhs_into(ms, t + dt, fs);
            stage_state(m0, [&](size_t i) {
                return scale(add(add(scale(fs[i], 5.0 / 12.0), scale(fn[i], 8.0 / 12.0)), scale(fn1[i], -1.0 / 12.0)), dt);
            }, m);
            t += dt;
            abm_push(std::move(fs), dt);
        }
        Fields F;
        diagnostics(m, t, F, r);
        r.time_seconds = t;
        r.dt_used = dt;
        r.suggested_next_dt = 0.0;
    }

    // rk45_step_buf (lib.rs:1412-1568) with max_error_norm_buf (lib.rs:1653-1674)
    void dp45(double dt_in, oracle_report &r) {
        double max_error = d.max_error > 0 ? d.max_error : 1e-5;
        double dt_min = d.dt_min > 0 ? d.dt_min : 1e-18;
        double dt_max = d.dt_max > 0 ? d.dt_max : 1e-10;
        double headroom = d.headroom > 0 ? d.headroom : 0.8;
        double dt = std::max(std::min(dt_in, dt_max), dt_min);
        const double A21 = 1.0 / 5.0;
        const double A31 = 3.0 / 40.0, A32 = 9.0 / 40.0;
        const double A41 = 44.0 / 45.0, A42 = -56.0 / 15.0, A43 = 32.0 / 9.0;
        const double A51 = 19372.0 / 6561.0, A52 = -25360.0 / 2187.0, A53 = 64448.0 / 6561.0,
                     A54 = -212.0 / 729.0;
        const double A61 = 9017.0 / 3168.0, A62 = -355.0 / 33.0, A63 = 46732.0 / 5247.0,
                     A64 = 49.0 / 176.0, A65 = -5103.0 / 18656.0;
        const double B1 = 35.0 / 384.0, B3 = 500.0 / 1113.0, B4 = 125.0 / 192.0,
                     B5 = -2187.0 / 6784.0, B6 = 11.0 / 84.0;
        const double E1 = 71.0 / 57600.0, E3 = -71.0 / 16695.0, E4 = 71.0 / 1920.0,
                     E5 = -17253.0 / 339200.0, E6 = 22.0 / 525.0, E7 = -1.0 / 40.0;
        std::vector<V3> m0 = m;
        std::vector<V3> k[7];
        std::vector<V3> ms(n);
        int rejected = 0;
        for (;;) {
            if (fsal_valid) { k[0] = fsal; fsal_valid = false; }
            else rhs_into(m0, t, k[0]);
            // increment(i) returns the dt-scaled stage increment, in the reference's order
            auto stage_inc = [&](auto inc, double c, std::vector<V3> &kout) {
#pragma omp parallel for
                for (long il = 0; il < (long)n; ++il) {
                    size_t i = (size_t)il;
                    ms[i] = normalized(add(m0[i], inc(i)));
                }
                rhs_into(ms, t + c * dt, kout);
            };
            auto stage = [&](auto comb, double c, std::vector<V3> &kout) {
                stage_inc([&](size_t i) { return scale(comb(i), dt); }, c, kout);
            };
            // stage 2 is m0 + k1 * (A21 * dt) in the reference (lib.rs:1459-1462)
            stage_inc([&](size_t i) { return scale(k[0][i], A21 * dt); }, 0.2, k[1]);
            stage([&](size_t i) { return add(scale(k[0][i], A31), scale(k[1][i], A32)); }, 0.3, k[2]);
            stage([&](size_t i) {
                return add(add(scale(k[0][i], A41), scale(k[1][i], A42)), scale(k[2][i], A43));
            }, 0.8, k[3]);
            stage([&](size_t i) {
                return add(add(scale(k[0][i], A51), scale(k[1][i], A52)),
                           add(scale(k[2][i], A53), scale(k[3][i], A54)));
            }, 8.0 / 9.0, k[4]);
            stage([&](size_t i) {
                return add(add(add(scale(k[0][i], A61), scale(k[1][i], A62)), scale(k[2][i], A63)),
                           add(scale(k[3][i], A64), scale(k[4][i], A65)));
            }, 1.0, k[5]);
#pragma omp parallel for
            for (long il = 0; il < (long)n; ++il) {
                size_t i = (size_t)il;
                V3 s = add(add(add(scale(k[0][i], B1), scale(k[2][i], B3)), scale(k[3][i], B4)),
                           add(scale(k[4][i], B5), scale(k[5][i], B6)));
                ms[i] = normalized(add(m0[i], scale(s, dt)));
            }
            rhs_into(ms, t + dt, k[6]);
            double err = 0.0;
            const std::pair<int, double> ws[6] = {{0, E1}, {2, E3}, {3, E4}, {4, E5}, {5, E6}, {6, E7}};
#pragma omp parallel for reduction(max : err)
            for (long il = 0; il < (long)n; ++il) {
                size_t i = (size_t)il;
                V3 e = {0, 0, 0};
                for (auto &w : ws) {
                    e[0] += w.second * k[w.first][i][0];
                    e[1] += w.second * k[w.first][i][1];
                    e[2] += w.second * k[w.first][i][2];
                }
                e[0] *= dt; e[1] *= dt; e[2] *= dt;
                err = std::max(err, norm(e));
            }
            if (err <= max_error || dt <= dt_min) {
                m = ms;
                t += dt;
                fsal = k[6];
                fsal_valid = true;
                double dt_next = std::min(
                    std::max(headroom * dt * std::pow(max_error / std::max(err, 1e-30), 0.2), dt_min),
                    dt_max);
                Fields F;
                diagnostics(m, t, F, r);
                r.time_seconds = t;
                r.dt_used = dt;
                r.suggested_next_dt = dt_next;
                r.rejected_attempts = rejected;
                return;
            }
            ++rejected;
            double dt_new = headroom * dt * std::pow(max_error / err, 0.2);
            dt = std::min(std::max(dt_new, dt_min), dt_max);
        }
    }
};

}  // namespace

// ---------------------------------------------------------------------------
// C interface
// ---------------------------------------------------------------------------
struct oracle_problem { Problem p; };

extern "C" {

void oracle_set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}

double oracle_newell_f(double x, double y, double z) { return newell_f(x, y, z); }
double oracle_newell_g(double x, double y, double z) { return newell_g(x, y, z); }

void oracle_fft(double *data, uint64_t n, int inverse) {
    FftPlan plan((size_t)n, inverse != 0);
    std::vector<cplx> work;
    plan.execute(reinterpret_cast<cplx *>(data), work);
}

void oracle_newell_kernels(uint32_t nx, uint32_t ny, uint32_t nz, double dx, double dy,
                           double dz, double *out6) {
    newell_kernels(nx, ny, nz, dx, dy, dz, out6);
}

void oracle_newell_spectra(uint32_t nx, uint32_t ny, uint32_t nz, double dx, double dy,
                           double dz, int thin_film_2d, double *xx, double *yy, double *zz,
                           double *xy, double *xz, double *yz) {
    size_t px = 2 * (size_t)nx, py = 2 * (size_t)ny, pz3 = 2 * (size_t)nz;
    size_t plen3 = px * py * pz3;
    std::vector<double> real6(6 * plen3);
    newell_kernels(nx, ny, nz, dx, dy, dz, real6.data());
    double *outs[6] = {xx, yy, zz, xy, xz, yz};
    size_t pz = thin_film_2d ? 1 : pz3;
    size_t plen = px * py * pz;
    FftPlan fx(px, false), fy(py, false), fz(pz, false);
    std::vector<cplx> buf(plen);
    for (int c = 0; c < 6; ++c) {
        // thin film: the z = 0 plane of the 3-D kernel (lib.rs:560-568)
        for (size_t i = 0; i < plen; ++i) buf[i] = cplx(real6[c * plen3 + i], 0.0);
        fft3(buf.data(), px, py, pz, fx, fy, fz);
        for (size_t i = 0; i < plen; ++i) {
            outs[c][2 * i] = buf[i].real();
            outs[c][2 * i + 1] = buf[i].imag();
        }
    }
}

void oracle_random_unit_vectors(uint64_t seed, uint64_t count, double *out) {
    uint64_t state = seed;
    for (uint64_t v = 0; v < count; ++v) {
        double c[3];
        for (;;) {
            for (int i = 0; i < 3; ++i) {
                state ^= state << 13;
                state ^= state >> 7;
                state ^= state << 17;
                c[i] = ((double)state / (double)UINT64_MAX) * 2.0 - 1.0;
            }
            double nrm = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
            if (nrm > 1e-10) {
                c[0] /= nrm; c[1] /= nrm; c[2] /= nrm;
                break;
            }
        }
        out[3 * v] = c[0]; out[3 * v + 1] = c[1]; out[3 * v + 2] = c[2];
    }
}

oracle_problem *oracle_create(const oracle_desc *desc, const double *m0) {
    if (!desc || !m0 || desc->nx == 0 || desc->ny == 0 || desc->nz == 0) return nullptr;
    auto *op = new oracle_problem();
    Problem &p = op->p;
    p.d = *desc;
    p.nx = desc->nx; p.ny = desc->ny; p.nz = desc->nz;
    p.n = p.nx * p.ny * p.nz;
    if (p.d.thin_film_2d && p.nz != 1) p.d.thin_film_2d = 0;
    if (desc->active_mask) p.mask.assign(desc->active_mask, desc->active_mask + p.n);
    if (desc->ms_map) p.msmap.assign(desc->ms_map, desc->ms_map + p.n);
    if (desc->region_mask) {
        p.region.assign(desc->region_mask, desc->region_mask + p.n);
        p.lut.assign(256 * 256, 0.0);
        if (desc->exchange_lut) std::memcpy(p.lut.data(), desc->exchange_lut, 256 * 256 * sizeof(double));
        else for (size_t r = 0; r < 256; ++r) p.lut[r * 256 + r] = desc->aex;
    }
    if (desc->boundary_tier > 0 && desc->volume_fraction) {
        p.vf.assign(desc->volume_fraction, desc->volume_fraction + p.n);
        p.phi_floor = desc->phi_floor > 0.0 ? desc->phi_floor : 0.05;
        p.delta_min = desc->delta_min > 0.0 ? desc->delta_min
                                            : 0.1 * std::min(std::min(desc->dx, desc->dy), desc->dz);
        bool faces = true, deltas = true;
        for (int q = 0; q < 6; ++q) {
            faces = faces && desc->face_link[q];
            deltas = deltas && desc->delta[q];
        }
        if (faces) for (int q = 0; q < 6; ++q) p.face[q].assign(desc->face_link[q], desc->face_link[q] + p.n);
        if (deltas) for (int q = 0; q < 6; ++q) p.delta[q].assign(desc->delta[q], desc->delta[q] + p.n);
        p.ex_tier = (desc->boundary_tier == 1 && faces) ? 1 : (desc->boundary_tier >= 2 && deltas) ? 2 : 0;
        if (desc->corr_target && desc->corr_source && desc->corr_tensor && desc->corr_targets > 0 &&
            desc->corr_stencil > 0) {
            const size_t T = desc->corr_targets, S = desc->corr_stencil;
            p.ctgt.assign(desc->corr_target, desc->corr_target + T);
            p.csrc.assign(desc->corr_source, desc->corr_source + T * S);
            p.cten.assign(desc->corr_tensor, desc->corr_tensor + T * S * 6);
        }
    }
    p.m.resize(p.n);
    for (size_t i = 0; i < p.n; ++i) {
        V3 v = {m0[3 * i], m0[3 * i + 1], m0[3 * i + 2]};
        p.m[i] = p.active(i) ? normalized(v) : V3{0, 0, 0};
    }
    p.init_workspace();
    return op;
}

void oracle_destroy(oracle_problem *p) { delete p; }

int oracle_step(oracle_problem *op, double dt, oracle_report *out) {
    if (!op || !out || !(dt > 0.0)) return -1;
    std::memset(out, 0, sizeof(*out));
    switch (op->p.d.integrator) {
        case ORACLE_DP45: op->p.dp45(dt, *out); break;
        case ORACLE_ABM3: op->p.abm3(dt, *out); break;
        case ORACLE_RK4: op->p.rk4(dt, *out); break;
        case ORACLE_RK23: op->p.rk23(dt, *out); break;
        default: op->p.heun(dt, *out); break;
    }
    return 0;
}

void oracle_get_m(const oracle_problem *op, double *out) {
    const Problem &p = op->p;
    for (size_t i = 0; i < p.n; ++i)
        for (int c = 0; c < 3; ++c) out[3 * i + c] = p.m[i][c];
}

void oracle_set_m(oracle_problem *op, const double *m) {
    Problem &p = op->p;
    for (size_t i = 0; i < p.n; ++i) {
        V3 v = {m[3 * i], m[3 * i + 1], m[3 * i + 2]};
        p.m[i] = p.active(i) ? normalized(v) : V3{0, 0, 0};
    }
    p.fsal_valid = false;
}

double oracle_time(const oracle_problem *op) { return op->p.t; }

void oracle_observe(oracle_problem *op, double *h_ex, double *h_demag, double *h_ext,
                    double *h_eff, double *rhs, oracle_report *out) {
    Problem &p = op->p;
    Problem::Fields F;
    oracle_report r{};
    p.diagnostics(p.m, p.t, F, r);
    r.time_seconds = p.t;
    auto put = [&](double *dst, const std::vector<V3> &v) {
        if (!dst) return;
        for (size_t i = 0; i < p.n; ++i)
            for (int c = 0; c < 3; ++c) dst[3 * i + c] = v[i][c];
    };
    put(h_ex, F.ex); put(h_demag, F.dm); put(h_ext, F.ext); put(h_eff, F.eff); put(rhs, F.rhs);
    if (out) *out = r;
}

}  // extern "C"
