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

}  // namespace fm
