// newell_host.cpp — FP64 Newell demag tensor and its octant spectrum (host).
//
// Real-space tensor: Newell, Williams & Dunlop (1993) f/g potentials with the
// 27-point second-difference stencil summed with Kahan–Neumaier compensation,
// and the point-dipole asymptote beyond 40 cells, as the reference does in
// crates/fullmag-fdm-demag/src/newell.rs:21-519 (the steps and the 40-cell
// switch are kept identical so the spectra agree with the reference's).
//
// Spectrum: the padded kernel is even or odd along every axis, so its DFT on
// the (2nx, 2ny, 2nz) grid is real and is fully described by the octant
// k <= n.  Per axis, with G(k) = sum_{x<n} f(x) exp(-2 pi i k x / 2n) (a
// zero-padded FFT of the first half):
//     even  : F(k) = 2 Re G(k) - f(0)
//     odd   : F(k) = -i S(k),  S(k) = -2 Im G(k)
// and the odd factors (-i)^2 = -1 of xy, xz, yz make the product real.  This
// never materialises the full complex spectra the reference stores.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <thread>
#include <vector>

#include "newell_host.hpp"

namespace fm {
namespace {

constexpr double PI = 3.14159265358979323846;

double nf(double x, double y, double z) {
    const double x2 = x * x, y2 = y * y, z2 = z * z, r2 = x2 + y2 + z2;
    if (r2 < 1e-300) return 0.0;
    const double r = std::sqrt(r2);
    double res = (2.0 * x2 - y2 - z2) * r / 6.0;
    const double rxz2 = x2 + z2;
    if (rxz2 > 1e-300) {
        const double arg = 2.0 * y * (y + r) / rxz2;
        if (arg > -1.0) res += y * (z2 - x2) / 4.0 * std::log1p(arg);
    }
    const double rxy2 = x2 + y2;
    if (rxy2 > 1e-300) {
        const double arg = 2.0 * z * (z + r) / rxy2;
        if (arg > -1.0) res += z * (y2 - x2) / 4.0 * std::log1p(arg);
    }
    if (std::fabs(x) > 1e-300) res -= x * y * z * std::atan(y * z / (x * r));
    return res;
}

double ng(double x, double y, double z) {
    const double x2 = x * x, y2 = y * y, z2 = z * z, r2 = x2 + y2 + z2;
    if (r2 < 1e-300) return 0.0;
    const double r = std::sqrt(r2);
    double res = -x * y * r / 3.0;
    const double rxy2 = x2 + y2;
    if (rxy2 > 1e-300) {
        const double arg = 2.0 * z * (z + r) / rxy2;
        if (arg > -1.0) res += x * y * z * std::log1p(arg) / 2.0;
    }
    const double ryz2 = y2 + z2;
    if (ryz2 > 1e-300) {
        const double arg = 2.0 * x * (x + r) / ryz2;
        if (arg > -1.0) res += y * (3.0 * z2 - y2) * std::log1p(arg) / 12.0;
    }
    const double rxz2 = x2 + z2;
    if (rxz2 > 1e-300) {
        const double arg = 2.0 * y * (y + r) / rxz2;
        if (arg > -1.0) res += x * (3.0 * z2 - x2) * std::log1p(arg) / 12.0;
    }
    if (std::fabs(z) > 1e-300) res -= z2 * z / 6.0 * std::atan(x * y / (z * r));
    if (std::fabs(y) > 1e-300) res -= y2 * z / 2.0 * std::atan(x * z / (y * r));
    if (std::fabs(x) > 1e-300) res -= x2 * z / 2.0 * std::atan(y * z / (x * r));
    return res;
}

// Second difference of the potential over the 27 neighbours of (i, j, k),
// weights 8 / -4 / 2 / -1 by the number of shifted axes, compensated sum.
double stencil27(const std::vector<double> &f, size_t sx, size_t sy, size_t i, size_t j,
                 size_t k, double vol) {
    i += 1; j += 1; k += 1;
    auto F = [&](size_t a, size_t b, size_t c) { return f[(c * sy + b) * sx + a]; };
    double sum = 0.0, comp = 0.0;
    auto add = [&](double v) {
        const double t = sum + v;
        comp += (std::fabs(sum) >= std::fabs(v)) ? (sum - t) + v : (v - t) + sum;
        sum = t;
    };
    // same term order as newell.rs:171-198 (centre, faces, edges, corners)
    add(8.0 * F(i, j, k));
    add(-4.0 * F(i + 1, j, k)); add(-4.0 * F(i - 1, j, k)); add(-4.0 * F(i, j + 1, k));
    add(-4.0 * F(i, j - 1, k)); add(-4.0 * F(i, j, k + 1)); add(-4.0 * F(i, j, k - 1));
    add(2.0 * F(i - 1, j - 1, k)); add(2.0 * F(i - 1, j + 1, k)); add(2.0 * F(i + 1, j - 1, k));
    add(2.0 * F(i + 1, j + 1, k)); add(2.0 * F(i - 1, j, k - 1)); add(2.0 * F(i - 1, j, k + 1));
    add(2.0 * F(i + 1, j, k - 1)); add(2.0 * F(i + 1, j, k + 1)); add(2.0 * F(i, j - 1, k - 1));
    add(2.0 * F(i, j - 1, k + 1)); add(2.0 * F(i, j + 1, k - 1)); add(2.0 * F(i, j + 1, k + 1));
    add(-F(i - 1, j - 1, k - 1)); add(-F(i - 1, j - 1, k + 1)); add(-F(i - 1, j + 1, k - 1));
    add(-F(i + 1, j - 1, k - 1)); add(-F(i - 1, j + 1, k + 1)); add(-F(i + 1, j - 1, k + 1));
    add(-F(i + 1, j + 1, k - 1)); add(-F(i + 1, j + 1, k + 1));
    return (sum + comp) / (4.0 * PI * vol);
}

double dip_diag(double x, double y, double z, double vol) {
    const double r2 = x * x + y * y + z * z, r = std::sqrt(r2), r3 = r2 * r;
    return (1.0 / r3 - 3.0 * x * x / (r3 * r2)) / (4.0 * PI) * vol;
}
double dip_off(double x, double y, double z, double vol) {
    const double r2 = x * x + y * y + z * z, r = std::sqrt(r2), r5 = r2 * r2 * r;
    return -3.0 * x * y / (4.0 * PI * r5) * vol;
}

template <typename F>
void parallel_for(size_t n, F &&fn) {
    unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (n < 64) nt = 1;
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t)
        th.emplace_back([&, t] {
            for (size_t i = t; i < n; i += nt) fn(i);
        });
    for (auto &x : th) x.join();
}

// Minimal host FFT (unnormalised, forward), mixed radix by recursion.
struct HostFft {
    size_t n;
    std::vector<std::complex<double>> tw;
    std::vector<size_t> fac;
    explicit HostFft(size_t n_) : n(n_), tw(n_) {
        for (size_t j = 0; j < n; ++j) {
            const double a = 2.0 * PI * (double)j / (double)n;
            tw[j] = {std::cos(a), -std::sin(a)};
        }
        size_t m = n;
        for (size_t p : {4, 2}) while (m % p == 0 && m > 1) { fac.push_back(p); m /= p; }
        for (size_t p = 3; m > 1; p += 2) while (m % p == 0) { fac.push_back(p); m /= p; }
    }
    void rec(const std::complex<double> *in, std::complex<double> *out, size_t len, size_t stride,
             size_t fi) const {
        if (len == 1) { out[0] = in[0]; return; }
        const size_t p = fac[fi], m = len / p;
        for (size_t r = 0; r < p; ++r) rec(in + r * stride, out + r * m, m, stride * p, fi + 1);
        std::vector<std::complex<double>> t(p), o(p);
        for (size_t k = 0; k < m; ++k) {
            for (size_t r = 0; r < p; ++r)
                t[r] = out[r * m + k] * tw[((r * k) % len) * (n / len)];
            for (size_t q = 0; q < p; ++q) {
                std::complex<double> acc = 0.0;
                for (size_t r = 0; r < p; ++r) acc += t[r] * tw[((r * q) % p) * (n / p)];
                o[q] = acc;
            }
            for (size_t q = 0; q < p; ++q) out[k + q * m] = o[q];
        }
    }
    void run(std::complex<double> *data) const {
        std::vector<std::complex<double>> in(data, data + n);
        rec(in.data(), data, n, 1, 0);
    }
};

// Per-axis even/odd transform of a line of n samples f(0..n-1), extended to
// the padded length L >= 2n with f(L - r) = +-f(r) and zeros between, into the
// L/2 + 1 outputs k = 0..L/2: 2 Re F - f(0) (even) or -2 Im F (odd), F the
// length-L DFT of f(0..n-1) followed by zeros.
void axis_transform(const double *src, double *dst, size_t n, size_t L, bool odd, const HostFft &fft) {
    std::vector<std::complex<double>> buf(L, 0.0);
    for (size_t x = 0; x < n; ++x) buf[x] = src[x];
    fft.run(buf.data());
    for (size_t k = 0; k <= L / 2; ++k)
        dst[k] = odd ? -2.0 * buf[k].imag() : 2.0 * buf[k].real() - src[0];
}

}  // namespace

void newell_real_octant(int nx, int ny, int nz, double dx, double dy, double dz,
                        std::vector<double> (&out)[6]) {
    const size_t AD = 40;  // asymptotic switch, newell.rs:231
    const size_t nxd = std::min<size_t>(nx, AD), nyd = std::min<size_t>(ny, AD),
                 nzd = std::min<size_t>(nz, AD);
    const size_t sx = nxd + 2, sy = nyd + 2, sz = nzd + 2;
    std::vector<double> fv[6];
    for (auto &v : fv) v.assign(sx * sy * sz, 0.0);
    parallel_for(sz, [&](size_t kk) {
        for (size_t j = 0; j < sy; ++j)
            for (size_t i = 0; i < sx; ++i) {
                const double x = ((double)i - 1.0) * dx, y = ((double)j - 1.0) * dy,
                             z = ((double)kk - 1.0) * dz;
                const size_t b = (kk * sy + j) * sx + i;
                fv[0][b] = nf(x, y, z);
                fv[1][b] = nf(y, x, z);
                fv[2][b] = nf(z, y, x);
                fv[3][b] = ng(x, y, z);
                fv[4][b] = ng(x, z, y);
                fv[5][b] = ng(y, z, x);
            }
    });
    const size_t n = (size_t)nx * ny * nz;
    for (auto &v : out) v.assign(n, 0.0);
    const double vol = dx * dy * dz;
    parallel_for((size_t)nz, [&](size_t k) {
        for (size_t j = 0; j < (size_t)ny; ++j)
            for (size_t i = 0; i < (size_t)nx; ++i) {
                const size_t o = (k * ny + j) * nx + i;
                const bool far = i >= AD || j >= AD || k >= AD || i * i + j * j + k * k >= AD * AD;
                if (far) {
                    const double x = i * dx, y = j * dy, z = k * dz;
                    out[0][o] = dip_diag(x, y, z, vol);
                    out[1][o] = dip_diag(y, x, z, vol);
                    out[2][o] = dip_diag(z, y, x, vol);
                    out[3][o] = dip_off(x, y, z, vol);
                    out[4][o] = dip_off(x, z, y, vol);
                    out[5][o] = dip_off(y, z, x, vol);
                } else {
                    // the stencil normalisation is the product hx*hy*hz = vol for every component
                    for (int c = 0; c < 6; ++c) out[c][o] = stencil27(fv[c], sx, sy, i, j, k, vol);
                }
            }
    });
}

void newell_octant_spectra(int nx, int ny, int nz, double dx, double dy, double dz, bool thin,
                           std::vector<double> (&spec)[6]) {
    newell_octant_spectra_padded(nx, ny, nz, dx, dy, dz, thin, 2 * nx, 2 * ny, 2 * nz, spec);
}

void newell_octant_spectra_padded(int nx, int ny, int nz, double dx, double dy, double dz, bool thin,
                                  int Lx, int Ly, int Lz, std::vector<double> (&spec)[6]) {
    std::vector<double> real[6];
    newell_real_octant(nx, ny, nz, dx, dy, dz, real);
    const int KX = Lx / 2 + 1, KY = Ly / 2 + 1, KZ = thin ? 1 : Lz / 2 + 1;
    // parity per component along (x, y, z): xx, yy, zz even; xy odd x,y; xz odd x,z; yz odd y,z
    const bool oddx[6] = {false, false, false, true, true, false};
    const bool oddy[6] = {false, false, false, true, false, true};
    const bool oddz[6] = {false, false, false, false, true, true};
    HostFft fx((size_t)Lx), fy((size_t)Ly), fz((size_t)(thin ? 2 * nz : Lz));
    for (int c = 0; c < 6; ++c) {
        // x: [z][y][x<nx] -> A[z][y][kx<=nx]
        std::vector<double> A((size_t)nz * ny * KX);
        parallel_for((size_t)nz * ny, [&](size_t line) {
            axis_transform(&real[c][line * nx], &A[line * KX], nx, Lx, oddx[c], fx);
        });
        // y: A[z][y][kx] -> B[z][kx][ky<=ny]
        std::vector<double> B((size_t)nz * KX * KY);
        parallel_for((size_t)nz * KX, [&](size_t line) {
            const size_t z = line / KX, kx = line % KX;
            std::vector<double> src(ny), dst(KY);
            for (int y = 0; y < ny; ++y) src[y] = A[(z * ny + y) * KX + kx];
            axis_transform(src.data(), dst.data(), ny, Ly, oddy[c], fy);
            for (int ky = 0; ky < KY; ++ky) B[(z * KX + kx) * KY + ky] = dst[ky];
        });
        // z: B[z][kx][ky] -> spec[kz][kx][ky]; thin films keep only the z = 0 plane
        spec[c].assign((size_t)KZ * KX * KY, 0.0);
        const double sign = (oddx[c] + oddy[c] + oddz[c]) == 2 ? -1.0 : 1.0;
        if (thin) {
            // 2-D spectra of the z = 0 plane (the nz = 1 runner path): xz and yz are odd in
            // exactly one in-plane axis, so their 2-D transform is imaginary and the real
            // octant holds zero; xy carries (-i)^2 = -1.
            const bool imaginary = (oddx[c] != oddy[c]);
            const double s2 = (oddx[c] && oddy[c]) ? -1.0 : 1.0;
            for (size_t o = 0; o < (size_t)KX * KY; ++o) spec[c][o] = imaginary ? 0.0 : s2 * B[o];
            continue;
        }
        parallel_for((size_t)KX * KY, [&](size_t line) {
            std::vector<double> src(nz), dst(KZ);
            for (int z = 0; z < nz; ++z) src[z] = B[(size_t)z * KX * KY + line];
            axis_transform(src.data(), dst.data(), nz, Lz, oddz[c], fz);
            for (int kz = 0; kz < KZ; ++kz) spec[c][(size_t)kz * KX * KY + line] = sign * dst[kz];
        });
    }
}

void octant_to_z_direct(int nkx, int KY, int nz, const std::vector<double> (&spec)[6],
                        std::vector<double> (&out)[6], int h) {
    if (h <= 0) h = nz;
    const size_t plane = (size_t)nkx * KY;
    const bool oddz[6] = {false, false, false, false, true, true};
    // cos / sin (pi k d / h) for d < nz, k < h
    std::vector<double> cs((size_t)nz * h), sn((size_t)nz * h);
    for (int d = 0; d < nz; ++d)
        for (int k = 0; k < h; ++k) {
            const double a = PI * (double)k * (double)d / (double)h;
            cs[(size_t)d * h + k] = std::cos(a);
            sn[(size_t)d * h + k] = std::sin(a);
        }
    for (int c = 0; c < 6; ++c) {
        out[c].assign((size_t)nz * plane, 0.0);
        const double *S = spec[c].data();
        double *O = out[c].data();
        const double sign = oddz[c] ? 1.0 : -1.0;
        parallel_for(plane, [&](size_t o) {
            for (int d = 0; d < nz; ++d) {
                double acc = 0.0;
                for (int k = 1; k < h; ++k)
                    acc += S[(size_t)k * plane + o] * (oddz[c] ? sn[(size_t)d * h + k] : cs[(size_t)d * h + k]);
                acc *= 2.0;
                if (!oddz[c]) acc += S[o] + ((d & 1) ? -1.0 : 1.0) * S[(size_t)h * plane + o];
                O[(size_t)d * plane + o] = sign * acc;
            }
        });
    }
}

}  // namespace fm
