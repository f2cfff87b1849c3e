// newell_host.hpp — FP64 Newell tensor setup on the host.
#pragma once

#include <vector>

namespace fm {

// First-octant real-space tensor N_c(i, j, k), i < nx, j < ny, k < nz,
// c = xx, yy, zz, xy, xz, yz; layout [k][j][i].
void newell_real_octant(int nx, int ny, int nz, double dx, double dy, double dz,
                        std::vector<double> (&out)[6]);

// Real octant of the (2nx, 2ny, 2nz) spectrum, layout [kz][kx][ky] with
// kx <= nx, ky <= ny, kz <= nz (thin: only kz = 0, 2-D spectra of the z = 0 plane).
void newell_octant_spectra(int nx, int ny, int nz, double dx, double dy, double dz, bool thin,
                           std::vector<double> (&spec)[6]);

// The same for padded lengths L >= 2n per axis (even): octant kx <= Lx/2,
// ky <= Ly/2, kz <= Lz/2.  Outputs at the physical cells use only kernel offsets
// |r| <= n - 1, so any such L gives the field of L = 2n in exact arithmetic.
void newell_octant_spectra_padded(int nx, int ny, int nz, double dx, double dy, double dz, bool thin,
                                  int Lx, int Ly, int Lz, std::vector<double> (&spec)[6]);

// Table of the direct z convolution (3-D grids) from a real octant spectrum
// [kz <= h][kx < nkx][ky < KY] of padded length Lz = 2 h >= 2 nz - 1 (h = nz
// unless given): per (kx, ky) the unnormalised z inverse
// n(d) = sum_kz N(kz) W_Lz^{-kz d} for d in [0, nz),
//   even in z (xx, yy, zz, xy): S(0) + (-1)^d S(h) + 2 sum_{0<k<h} S(k) cos(pi k d / h)
//   odd in z (xz, yz):          i tau(d), tau(d) = 2 sum_{0<k<h} S(k) sin(pi k d / h)
// (the kz = 0 and kz = h entries of an odd component are zero up to rounding
// and are left out).  Output layout [c][d][kx][ky], entries
// (-n_xx, -n_yy, -n_zz, -n_xy, tau_xz, tau_yz): the real matrix of H = -N M on
// (Mx, My, -i Mz) -> (Hx, Hy, -i Hz).  With zero padding, offsets |d| < nz
// never wrap for any Lz >= 2 nz - 1, so the sum over z' < nz of n(z - z') M(z')
// is the padded z convolution kept at z < nz.
void octant_to_z_direct(int nkx, int KY, int nz, const std::vector<double> (&spec)[6],
                        std::vector<double> (&out)[6], int h = 0);

}  // namespace fm
