// api.cu — the exported C ABI (include/fullmag_fdm.h, include/fullmag_fdm_ext.h).
//
// Contract kept from the reference implementation
// (native/backends/fdm/src/api.cpp:36-718):
//   - device chosen by FULLMAG_FDM_GPU_INDEX, else FULLMAG_CUDA_DEVICE_INDEX;
//   - create() returns a handle even on failure, with last_error set; it
//     returns NULL only when the plan pointer is NULL or allocation of the
//     handle itself fails;
//   - length mismatches give FULLMAG_FDM_ERR_INVALID and a message;
//   - last_error(NULL) is "null handle".
// Additional validation (reported through last_error, never silently
// accepted): non-positive cell sizes or Ms, region ids >= 256, unknown
// integrator or boundary-tier values, boundary tiers whose per-cell arrays are
// missing or of the wrong length, spectra that are not the real, even/odd
// Newell form, padded FFT lengths with prime factors > 7.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "backend.hpp"
#include "backend_impl.hpp"
#include "fullmag_fdm.h"
#include "fullmag_fdm_ext.h"
#include "newell_host.hpp"

struct fullmag_fdm_backend {
    fm::Backend b;
};
struct fullmag_fdm_field_snapshot {
    fm::Snapshot s;
};

namespace {

using fm::Backend;

bool env_device(int &out) {
    const char *s = std::getenv("FULLMAG_FDM_GPU_INDEX");
    if (!s || !*s) s = std::getenv("FULLMAG_CUDA_DEVICE_INDEX");
    if (!s || !*s) return false;
    char *end = nullptr;
    long v = std::strtol(s, &end, 10);
    if (end == s || *end != '\0' || v < 0) return false;
    out = (int)v;
    return true;
}

bool select_device(Backend &b) {
    int want;
    if (env_device(want)) {
        if (!fm::cuda_ok(b, cudaSetDevice(want), "cudaSetDevice")) return false;
        b.device = want;
        return true;
    }
    return fm::cuda_ok(b, cudaGetDevice(&b.device), "cudaGetDevice");
}

// Re-select the handle's device for calls made from any host thread.
bool bind(Backend &b) { return fm::cuda_ok(b, cudaSetDevice(b.device), "cudaSetDevice"); }

template <typename F>
void par_for(size_t n, F &&fn) {
    unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    if (n < 4096) nt = 1;
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t)
        th.emplace_back([&, t] {
            const size_t lo = n * t / nt, hi = n * (t + 1) / nt;
            for (size_t i = lo; i < hi; ++i) fn(i);
        });
    for (auto &x : th) x.join();
}

// Octant of the supplied spectra: real part at kx <= nx, ky <= ny, kz <= KZ-1,
// checked on a sample for reality and even/odd symmetry.
bool extract_octant(Backend &b, const fullmag_fdm_plan_desc *plan, int Lzs,
                    std::vector<double> (&spec)[6]) {
    const double *src[6] = {plan->demag_kernel_xx_spectrum, plan->demag_kernel_yy_spectrum,
                            plan->demag_kernel_zz_spectrum, plan->demag_kernel_xy_spectrum,
                            plan->demag_kernel_xz_spectrum, plan->demag_kernel_yz_spectrum};
    const int Lx = b.Lx, Ly = b.Ly, KX = b.nkx, KY = b.KY, KZ = b.KZ;
    auto at = [&](int c, long long kx, long long ky, long long kz, int part) {
        return src[c][2 * (kx + (long long)Lx * (ky + (long long)Ly * kz)) + part];
    };
    for (int c = 0; c < 6; ++c) {
        spec[c].assign((size_t)KZ * KX * KY, 0.0);
        par_for((size_t)KZ * KX, [&](size_t row) {
            const int kz = (int)(row / KX), kx = (int)(row % KX);
            double *dst = &spec[c][row * KY];
            for (int ky = 0; ky < KY; ++ky) dst[ky] = at(c, kx, ky, kz, 0);
        });
    }
    // sampled check: imaginary parts ~ 0 and mirrored entries = +/- octant values
    double scale = 0.0;
    for (int c = 0; c < 3; ++c) scale = std::max(scale, std::fabs(spec[c][0]));
    for (int c = 0; c < 6; ++c)
        for (size_t o = 0; o < spec[c].size(); o += std::max<size_t>(1, spec[c].size() / 2048))
            scale = std::max(scale, std::fabs(spec[c][o]));
    const double tol = 1e-8 * std::max(scale, 1e-300);
    const bool oddx[6] = {false, false, false, true, true, false};
    const bool oddy[6] = {false, false, false, true, false, true};
    const bool oddz[6] = {false, false, false, false, true, true};
    const bool thin2d = (Lzs == 1);
    const size_t total = (size_t)KZ * KX * KY;
    const size_t stride = std::max<size_t>(1, total / 4096);
    for (int c = 0; c < 6; ++c) {
        // in the 2-D form, components odd in exactly one in-plane axis are imaginary;
        // their real octant is zero and is checked as such
        const bool imag2d = thin2d && (oddx[c] != oddy[c]);
        for (size_t o = 0; o < total; o += stride) {
            const int kz = (int)(o / ((size_t)KX * KY));
            const int kx = (int)((o / KY) % KX), ky = (int)(o % KY);
            const double v = spec[c][o];
            bool bad = false;
            if (imag2d) {
                bad |= std::fabs(at(c, kx, ky, 0, 0)) > tol || std::fabs(at(c, kx, ky, 0, 1)) > tol;
            } else {
                bad |= std::fabs(at(c, kx, ky, kz, 1)) > tol;
                if (kx > 0 && kx < Lx / 2)
                    bad |= std::fabs(at(c, Lx - kx, ky, kz, 0) - (oddx[c] ? -v : v)) > tol;
                if (ky > 0 && ky < Ly / 2)
                    bad |= std::fabs(at(c, kx, Ly - ky, kz, 0) - (oddy[c] ? -v : v)) > tol;
                if (!thin2d && Lzs > 1 && kz > 0 && kz < Lzs / 2)
                    bad |= std::fabs(at(c, kx, ky, Lzs - kz, 0) - (oddz[c] ? -v : v)) > tol;
            }
            if (bad) {
                b.last_error = "demag kernel spectra are not the real, even/odd Newell-tensor form "
                               "this backend stores as an octant (component " + std::to_string(c) + ")";
                return false;
            }
        }
        if (imag2d) std::fill(spec[c].begin(), spec[c].end(), 0.0);
    }
    return true;
}

// k k^T / k^2 on the padded grid, the reference's fallback without spectra
// (native/backends/fdm/src/demag_fp64.cu:102-148).  The reference uses +k at
// Nyquist indices, so its tensor is not Hermitian there, and it keeps the real
// part of the inverse transform: that equals convolving with the Hermitian
// part of the tensor, whose off-diagonal term vanishes wherever exactly one of
// its two axes sits at a Nyquist index.  The octant below stores that part.
void projection_octant(Backend &b, std::vector<double> (&spec)[6]) {
    const int KX = b.nkx, KY = b.KY, KZ = b.KZ;
    for (auto &s : spec) s.assign((size_t)KZ * KX * KY, 0.0);
    const double lx = b.Lx * b.dx, ly = b.Ly * b.dy, lz = b.Lz * b.dz;
    for (int kz = 0; kz < KZ; ++kz)
        for (int kx = 0; kx < KX; ++kx)
            for (int ky = 0; ky < KY; ++ky) {
                const double qx = 2.0 * fm::kPi * kx / lx, qy = 2.0 * fm::kPi * ky / ly,
                             qz = 2.0 * fm::kPi * kz / lz;
                const double q2 = qx * qx + qy * qy + qz * qz;
                const size_t o = ((size_t)kz * KX + kx) * KY + ky;
                if (q2 == 0.0) continue;
                spec[0][o] = qx * qx / q2;
                spec[1][o] = qy * qy / q2;
                spec[2][o] = qz * qz / q2;
                const bool nyx = 2 * kx == b.Lx, nyy = 2 * ky == b.Ly, nyz = 2 * kz == b.Lz;
                spec[3][o] = (nyx != nyy) ? 0.0 : qx * qy / q2;
                spec[4][o] = (nyx != nyz) ? 0.0 : qx * qz / q2;
                spec[5][o] = (nyy != nyz) ? 0.0 : qy * qz / q2;
            }
}

// Boundary tiers (fullmag_fdm.h:151-187; api.cpp:247-290, context.cu:629-730).
// T0 uses the face links, T1 the intersection distances; both weight the demag
// magnetisation by the volume fraction; the sparse demag correction needs a
// tier.  Unlike the reference, which skips the tier silently when the volume
// fraction is missing or has the wrong length, and reads out of bounds on bad
// correction indices, these are errors here.
static bool parse_boundary(Backend &b, const fullmag_fdm_plan_desc *plan) {
    const int tier = (int)plan->boundary_correction;
    if (tier == FULLMAG_FDM_BOUNDARY_NONE) return true;
    if (tier != FULLMAG_FDM_BOUNDARY_VOLUME && tier != FULLMAG_FDM_BOUNDARY_FULL) {
        b.last_error = "unknown boundary_correction " + std::to_string(tier);
        return false;
    }
    if (!plan->volume_fraction) { b.last_error = "boundary_correction: volume_fraction is required"; return false; }
    if (plan->volume_fraction_len != (uint64_t)b.n) {
        b.last_error = "volume_fraction_len mismatch: expected " + std::to_string(b.n) + ", got " +
                       std::to_string(plan->volume_fraction_len);
        return false;
    }
    const size_t n = (size_t)b.n;
    b.boundary_tier = tier;
    b.phi_floor = plan->boundary_phi_floor > 0.0 ? plan->boundary_phi_floor : 0.05;
    b.delta_min = plan->boundary_delta_min > 0.0 ? plan->boundary_delta_min : 0.1 * std::min({b.dx, b.dy, b.dz});
    b.vf_host.assign(plan->volume_fraction, plan->volume_fraction + n);
    const double *faces[6] = {plan->face_link_xp, plan->face_link_xm, plan->face_link_yp,
                              plan->face_link_ym, plan->face_link_zp, plan->face_link_zm};
    const double *deltas[6] = {plan->delta_xp, plan->delta_xm, plan->delta_yp,
                               plan->delta_ym, plan->delta_zp, plan->delta_zm};
    bool have_faces = true, have_deltas = true;
    for (int q = 0; q < 6; ++q) {
        have_faces = have_faces && faces[q];
        have_deltas = have_deltas && deltas[q];
    }
    if (tier == FULLMAG_FDM_BOUNDARY_VOLUME && have_faces) {
        b.ex_tier = 1;
        b.face_host.resize(6 * n);
        for (int q = 0; q < 6; ++q) std::copy(faces[q], faces[q] + n, b.face_host.begin() + q * n);
    } else if (tier == FULLMAG_FDM_BOUNDARY_FULL && have_deltas) {
        b.ex_tier = 2;
        b.delta_host.resize(6 * n);
        for (int q = 0; q < 6; ++q) std::copy(deltas[q], deltas[q] + n, b.delta_host.begin() + q * n);
    }
    if (plan->has_demag_boundary_corr && plan->demag_corr_target_idx && plan->demag_corr_source_idx &&
        plan->demag_corr_tensor && plan->demag_corr_target_count > 0 && plan->demag_corr_stencil_size > 0) {
        const size_t T = plan->demag_corr_target_count, S = plan->demag_corr_stencil_size;
        b.corr_targets = (uint32_t)T;
        b.corr_stencil = (uint32_t)S;
        b.corr_tgt_host.assign(plan->demag_corr_target_idx, plan->demag_corr_target_idx + T);
        b.corr_src_host.assign(plan->demag_corr_source_idx, plan->demag_corr_source_idx + T * S);
        b.corr_ten_host.assign(plan->demag_corr_tensor, plan->demag_corr_tensor + T * S * 6);
        for (int32_t v : b.corr_tgt_host)
            if (v >= (int64_t)n) { b.last_error = "demag_corr_target_idx " + std::to_string(v) + " out of range"; return false; }
        for (int32_t v : b.corr_src_host)
            if (v >= (int64_t)n) { b.last_error = "demag_corr_source_idx " + std::to_string(v) + " out of range"; return false; }
    }
    return true;
}

bool create_impl(Backend &b, const fullmag_fdm_plan_desc *plan, const fullmag_fdm_plan_ext *ext) {
    // plan validation and host-side setup first: no CUDA call before the plan is accepted
    b.nx = (int)plan->grid.nx; b.ny = (int)plan->grid.ny; b.nz = (int)plan->grid.nz;
    b.n = (long long)plan->grid.nx * plan->grid.ny * plan->grid.nz;
    b.dx = plan->grid.dx; b.dy = plan->grid.dy; b.dz = plan->grid.dz;
    b.ms = plan->material.saturation_magnetisation;
    b.aex = plan->material.exchange_stiffness;
    b.alpha = plan->material.damping;
    b.gamma = plan->material.gyromagnetic_ratio;
    b.precision = plan->precision;
    b.integrator = plan->integrator;
    b.precession = plan->disable_precession == 0;
    b.enable_exchange = plan->enable_exchange != 0;
    b.enable_demag = plan->enable_demag != 0;
    b.has_ext = plan->has_external_field != 0;
    for (int c = 0; c < 3; ++c) b.hext[c] = plan->external_field_am[c];
    b.max_error = plan->adaptive_max_error > 0 ? plan->adaptive_max_error : 1e-5;
    b.dt_min = plan->adaptive_dt_min > 0 ? plan->adaptive_dt_min : 1e-18;
    b.dt_max = plan->adaptive_dt_max > 0 ? plan->adaptive_dt_max : 1e-10;
    b.headroom = plan->adaptive_headroom > 0 ? plan->adaptive_headroom : 0.8;

    if (b.n == 0) { b.last_error = "grid has zero cells"; return false; }
    if (!(b.dx > 0) || !(b.dy > 0) || !(b.dz > 0)) { b.last_error = "cell sizes must be positive"; return false; }
    if (b.precision != FULLMAG_FDM_PRECISION_SINGLE && b.precision != FULLMAG_FDM_PRECISION_DOUBLE) {
        b.last_error = "unknown precision"; return false;
    }
    if (b.integrator < FULLMAG_FDM_INTEGRATOR_HEUN || b.integrator > FULLMAG_FDM_INTEGRATOR_RK23) {
        b.last_error = "unknown integrator " + std::to_string((int)b.integrator);
        return false;
    }
    const uint64_t expected = (uint64_t)b.n * 3;
    if (plan->initial_magnetization_len != expected) {
        b.last_error = "initial_magnetization_len mismatch: expected " + std::to_string(expected) +
                       ", got " + std::to_string(plan->initial_magnetization_len);
        return false;
    }
    if (!plan->initial_magnetization_xyz) { b.last_error = "initial_magnetization_xyz is null"; return false; }
    b.has_mask = plan->active_mask != nullptr;
    if (b.has_mask && plan->active_mask_len != (uint64_t)b.n) {
        b.last_error = "active_mask_len mismatch: expected " + std::to_string(b.n) + ", got " +
                       std::to_string(plan->active_mask_len);
        return false;
    }
    b.has_regions = plan->region_mask != nullptr;
    if (b.has_regions && plan->region_mask_len != (uint64_t)b.n) {
        b.last_error = "region_mask_len mismatch: expected " + std::to_string(b.n) + ", got " +
                       std::to_string(plan->region_mask_len);
        return false;
    }
    if (b.has_regions)
        for (long long i = 0; i < b.n; ++i)
            if (plan->region_mask[i] >= FULLMAG_FDM_MAX_EXCHANGE_REGIONS) {
                b.last_error = "region id " + std::to_string(plan->region_mask[i]) + " at cell " +
                               std::to_string(i) + " exceeds the 256-entry exchange table";
                return false;
            }
    if (!parse_boundary(b, plan)) return false;
    fullmag_fdm_ext_demag_source demag_src = FULLMAG_FDM_EXT_DEMAG_FROM_PLAN;
    if (ext) {
        if (ext->struct_size < sizeof(fullmag_fdm_plan_ext)) { b.last_error = "fullmag_fdm_plan_ext.struct_size too small"; return false; }
        if (ext->ms_map) {
            if (ext->ms_map_len != (uint64_t)b.n) { b.last_error = "ms_map_len mismatch"; return false; }
            b.has_ms_map = true;
            b.ms_map_host.assign(ext->ms_map, ext->ms_map + b.n);
        }
        for (int c = 0; c < 3; ++c) b.hac[c] = ext->ac_field_am[c];
        b.ac_freq = ext->ac_frequency_hz;
        demag_src = ext->demag_source;
    }
    if (!b.has_ms_map && !(b.ms > 0)) { b.last_error = "saturation_magnetisation must be positive"; return false; }
    if (b.has_ms_map && b.boundary_tier) {
        b.last_error = "a per-cell Ms map cannot be combined with boundary correction tiers";
        return false;
    }
    {
        // FULLMAG_FDM_FFT=stockham keeps the shared-memory Stockham FFT even for
        // power-of-two lengths (both FFT paths are covered by the parity tests)
        const char *f = std::getenv("FULLMAG_FDM_FFT");
        b.force_stockham = f && std::strcmp(f, "stockham") == 0;
        const char *yz = std::getenv("FULLMAG_FDM_YZ");
        b.want_yz = yz && std::strcmp(yz, "fused") == 0;
        const char *yzp = std::getenv("FULLMAG_FDM_YZ_P");
        if (yzp) {
            const int v = std::atoi(yzp);
            if (v == 1 || v == 2 || v == 4 || v == 8) b.yz_min_P = v;
        }
    }
    if (b.has_mask) b.mask_host.assign(plan->active_mask, plan->active_mask + b.n);

    // demag geometry
    std::vector<double> spec[6];
    if (b.enable_demag) {
        const uint64_t p3 = (uint64_t)8 * b.n, p2 = (uint64_t)4 * b.nx * b.ny;
        const uint64_t len = plan->demag_kernel_spectrum_len;
        int Lzs = 0;
        if (demag_src == FULLMAG_FDM_EXT_DEMAG_NEWELL) {
            b.thin = (b.nz == 1);
        } else if (len != 0) {
            if (!plan->demag_kernel_xx_spectrum || !plan->demag_kernel_yy_spectrum ||
                !plan->demag_kernel_zz_spectrum || !plan->demag_kernel_xy_spectrum ||
                !plan->demag_kernel_xz_spectrum || !plan->demag_kernel_yz_spectrum) {
                b.last_error = "demag kernel spectra pointers must all be present when demag_kernel_spectrum_len is set";
                return false;
            }
            if (b.nz == 1 && len == 2 * p2) { b.thin = true; Lzs = 1; }
            else if (len == 2 * p3) { b.thin = (b.nz == 1); Lzs = 2 * b.nz; }
            else {
                b.last_error = "demag_kernel_spectrum_len mismatch: expected " + std::to_string(2 * p3) + " (3D)" +
                               (b.nz == 1 ? " or " + std::to_string(2 * p2) + " (thin-film 2D)" : std::string()) +
                               ", got " + std::to_string(len);
                return false;
            }
        } else {
            b.projection = true;
            b.thin = false;  // the fallback runs on the 3-D padded grid, also for nz = 1
        }
        b.Lx = 2 * b.nx; b.Ly = 2 * b.ny; b.Lz = b.thin ? 1 : 2 * b.nz;
        b.nkx = b.nx + 1; b.KY = b.ny + 1; b.KZ = b.thin ? 1 : b.nz + 1;
        for (int L : {b.Lx, b.Ly, b.Lz}) {
            fm::LinePlan tmp;
            if (!fm::make_line_plan(L, tmp)) {
                b.last_error = "padded FFT length " + std::to_string(L) + " has a prime factor > 7";
                return false;
            }
            if (L > 4096) { b.last_error = "padded FFT length " + std::to_string(L) + " exceeds 4096"; return false; }
        }
        fm::make_line_plan(b.Lx, b.px);
        fm::make_line_plan(b.Ly, b.py);
        fm::make_line_plan(b.Lz, b.pz);
        if (demag_src == FULLMAG_FDM_EXT_DEMAG_NEWELL) {
            fm::newell_octant_spectra(b.nx, b.ny, b.nz, b.dx, b.dy, b.dz, b.thin, spec);
        } else if (b.projection) {
            projection_octant(b, spec);
        } else {
            // a 3-D spectrum of an nz = 1 grid is constant along kz: its kz = 0 plane is the 2-D one
            if (!extract_octant(b, plan, b.thin && Lzs == 2 ? 2 : Lzs, spec)) return false;
        }
    }

    if (!select_device(b)) return false;
    if (!fm::cuda_ok(b, cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking), "cudaStreamCreate")) return false;
    if (!fm::backend_alloc(b)) return false;
    if (!fm::backend_configure(b)) return false;
    if (!fm::backend_upload_tables(b, spec)) return false;
    if (b.has_mask && !fm::cuda_ok(b, cudaMemcpy(b.d_mask, plan->active_mask, b.n, cudaMemcpyHostToDevice), "upload mask")) return false;
    if (b.has_regions) {
        if (!fm::cuda_ok(b, cudaMemcpy(b.d_region, plan->region_mask, b.n * 4, cudaMemcpyHostToDevice), "upload regions")) return false;
        std::vector<double> lut(256 * 256, 0.0);
        if (plan->exchange_lut && plan->exchange_lut_len == 256 * 256) std::memcpy(lut.data(), plan->exchange_lut, lut.size() * 8);
        else for (int r = 0; r < 256; ++r) lut[r * 256 + r] = b.aex;
        if (!fm::cuda_ok(b, cudaMemcpy(b.d_lut, lut.data(), lut.size() * 8, cudaMemcpyHostToDevice), "upload lut")) return false;
    }
    if (b.has_ms_map && !fm::cuda_ok(b, cudaMemcpy(b.d_msmap, b.ms_map_host.data(), b.n * 8, cudaMemcpyHostToDevice), "upload ms_map")) return false;
    if (b.boundary_tier) {
        auto up = [&](void *dst, const void *src, size_t bytes, const char *what) {
            return bytes == 0 || fm::cuda_ok(b, cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice), what);
        };
        if (!up(b.d_vf, b.vf_host.data(), b.vf_host.size() * 8, "upload volume_fraction") ||
            !up(b.d_face, b.face_host.data(), b.face_host.size() * 8, "upload face links") ||
            !up(b.d_delta, b.delta_host.data(), b.delta_host.size() * 8, "upload deltas") ||
            !up(b.d_corr_tgt, b.corr_tgt_host.data(), b.corr_tgt_host.size() * 4, "upload demag_corr_target_idx") ||
            !up(b.d_corr_src, b.corr_src_host.data(), b.corr_src_host.size() * 4, "upload demag_corr_source_idx") ||
            !up(b.d_corr_ten, b.corr_ten_host.data(), b.corr_ten_host.size() * 8, "upload demag_corr_tensor"))
            return false;
    }
    if (!fm::cuda_ok(b, cudaDeviceSynchronize(), "create sync")) return false;
    if (!fm::backend_upload_m_f64(b, plan->initial_magnetization_xyz, plan->initial_magnetization_len)) return false;
    if (!fm::backend_refresh(b)) return false;
    // device info
    cudaDeviceProp prop;
    if (fm::cuda_ok(b, cudaGetDeviceProperties(&prop, b.device), "cudaGetDeviceProperties")) {
        std::memset(&b.info, 0, sizeof(b.info));
        std::strncpy(b.info.name, prop.name, sizeof(b.info.name) - 1);
        b.info.compute_capability_major = prop.major;
        b.info.compute_capability_minor = prop.minor;
        cudaDriverGetVersion(&b.info.driver_version);
        cudaRuntimeGetVersion(&b.info.runtime_version);
        b.info_valid = true;
    }
    return true;
}

bool ready(Backend &b) {
    if (!b.arena) {
        if (b.last_error.empty()) b.last_error = "backend was not created successfully";
        return false;
    }
    return bind(b);
}

}  // namespace

extern "C" {

int fullmag_fdm_is_available(void) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
        cudaGetLastError();
        return 0;
    }
    int want;
    if (env_device(want) && want >= count) return 0;
    return 1;
}

fullmag_fdm_backend *fullmag_fdm_backend_create_ext(const fullmag_fdm_plan_desc *plan,
                                                    const fullmag_fdm_plan_ext *ext) {
    if (!plan) return nullptr;
    auto *h = new (std::nothrow) fullmag_fdm_backend();
    if (!h) return nullptr;
    if (!create_impl(h->b, plan, ext)) {
        std::string err = h->b.last_error;
        fm::backend_free(h->b);
        h->b.last_error = err.empty() ? "backend creation failed" : err;
    }
    return h;
}

fullmag_fdm_backend *fullmag_fdm_backend_create(const fullmag_fdm_plan_desc *plan) {
    return fullmag_fdm_backend_create_ext(plan, nullptr);
}

int fullmag_fdm_backend_step(fullmag_fdm_backend *h, double dt, fullmag_fdm_step_stats *out) {
    if (!h || !out) return FULLMAG_FDM_ERR_INVALID;
    Backend &b = h->b;
    if (!(dt > 0.0) || !std::isfinite(dt)) { b.last_error = "dt must be positive and finite"; return FULLMAG_FDM_ERR_INVALID; }
    if (!ready(b)) return FULLMAG_FDM_ERR_INVALID;
    const auto t0 = std::chrono::steady_clock::now();
    fullmag_fdm_step_stats st{};
    if (!fm::backend_step(b, dt, &st)) return FULLMAG_FDM_ERR_CUDA;
    st.wall_time_ns = (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
                          std::chrono::steady_clock::now() - t0).count();
    *out = st;
    return FULLMAG_FDM_OK;
}

int fullmag_fdm_backend_step_n(fullmag_fdm_backend *h, double dt, uint32_t n_steps,
                               fullmag_fdm_step_stats *out) {
    if (!h || !out || n_steps == 0) return FULLMAG_FDM_ERR_INVALID;
    Backend &b = h->b;
    if (!(dt > 0.0) || !std::isfinite(dt)) { b.last_error = "dt must be positive and finite"; return FULLMAG_FDM_ERR_INVALID; }
    if (!ready(b)) return FULLMAG_FDM_ERR_INVALID;
    const auto t0 = std::chrono::steady_clock::now();
    fullmag_fdm_step_stats st{};
    if (!fm::backend_step_n(b, dt, n_steps, &st)) return FULLMAG_FDM_ERR_CUDA;
    st.wall_time_ns = (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
                          std::chrono::steady_clock::now() - t0).count();
    *out = st;
    return FULLMAG_FDM_OK;
}

int fullmag_fdm_adjoint_forward(fullmag_fdm_backend *h, double dt, uint32_t n_steps,
                                uint32_t checkpoint_every, fullmag_fdm_step_stats *out) {
    if (!h || !out || n_steps == 0) return FULLMAG_FDM_ERR_INVALID;
    Backend &b = h->b;
    if (!(dt > 0.0) || !std::isfinite(dt)) { b.last_error = "dt must be positive and finite"; return FULLMAG_FDM_ERR_INVALID; }
    if (!ready(b)) return FULLMAG_FDM_ERR_INVALID;
    if (b.integrator != FULLMAG_FDM_INTEGRATOR_HEUN) {
        b.last_error = "the adjoint is implemented for the Heun integrator";
        return FULLMAG_FDM_ERR_INVALID;
    }
    if (b.has_regions || b.boundary_tier) {
        b.last_error = "the adjoint does not support region exchange tables or boundary tiers";
        return FULLMAG_FDM_ERR_INVALID;
    }
    const auto t0 = std::chrono::steady_clock::now();
    fullmag_fdm_step_stats st{};
    if (!fm::backend_adjoint_forward(b, dt, n_steps, checkpoint_every, &st)) return FULLMAG_FDM_ERR_CUDA;
    st.wall_time_ns = (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
                          std::chrono::steady_clock::now() - t0).count();
    *out = st;
    return FULLMAG_FDM_OK;
}

int fullmag_fdm_adjoint_backward(fullmag_fdm_backend *h, const double *dl_dm, uint64_t len, double *dl_dms,
                                 double *dl_dh_ext, double *dl_dh_ac, double *dl_dm0) {
    if (!h || !dl_dm) return FULLMAG_FDM_ERR_INVALID;
    Backend &b = h->b;
    if (len != (uint64_t)b.n * 3) { b.last_error = "out_len mismatch"; return FULLMAG_FDM_ERR_INVALID; }
    if (!ready(b)) return FULLMAG_FDM_ERR_INVALID;
    if (!b.adj_ready || b.step_count != b.adj_step_final || b.time != b.adj_t_final) {
        b.last_error = "no recorded trajectory ends at the current state (call fullmag_fdm_adjoint_forward first)";
        return FULLMAG_FDM_ERR_INVALID;
    }
    const size_t n = (size_t)b.n;
    std::vector<double> lam(3 * n), gms(n), ghext(3 * n), ghac(3 * n), lam0(3 * n);
    for (size_t i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) lam[c * n + i] = dl_dm[3 * i + c];
    if (!fm::backend_adjoint_backward(b, lam.data(), gms.data(), ghext.data(), ghac.data(), lam0.data()))
        return FULLMAG_FDM_ERR_CUDA;
    if (dl_dms) std::copy(gms.begin(), gms.end(), dl_dms);
    for (int c = 0; c < 3; ++c) {
        double se = 0.0, sa = 0.0;  // fixed order: deterministic
        for (size_t i = 0; i < n; ++i) { se += ghext[c * n + i]; sa += ghac[c * n + i]; }
        if (dl_dh_ext) dl_dh_ext[c] = se;
        if (dl_dh_ac) dl_dh_ac[c] = sa;
    }
    if (dl_dm0)
        for (size_t i = 0; i < n; ++i)
            for (int c = 0; c < 3; ++c) dl_dm0[3 * i + c] = lam0[c * n + i];
    return FULLMAG_FDM_OK;
}

int fullmag_fdm_backend_copy_field_f64(fullmag_fdm_backend *h, fullmag_fdm_observable obs,
                                       double *out, uint64_t len) {
    if (!h || !out) return FULLMAG_FDM_ERR_INVALID;
    Backend &b = h->b;
    if (len != (uint64_t)b.n * 3) { b.last_error = "out_len mismatch"; return FULLMAG_FDM_ERR_INVALID; }
    if (!ready(b)) return FULLMAG_FDM_ERR_INVALID;
    return fm::backend_download_f64(b, obs, out, len) ? FULLMAG_FDM_OK : FULLMAG_FDM_ERR_CUDA;
}

int fullmag_fdm_backend_copy_field_f32(fullmag_fdm_backend *h, fullmag_fdm_observable obs,
                                       float *out, uint64_t len) {
    if (!h || !out) return FULLMAG_FDM_ERR_INVALID;
    Backend &b = h->b;
    if (len != (uint64_t)b.n * 3) { b.last_error = "out_len mismatch"; return FULLMAG_FDM_ERR_INVALID; }
    if (!ready(b)) return FULLMAG_FDM_ERR_INVALID;
    return fm::backend_download_f32(b, obs, out, len) ? FULLMAG_FDM_OK : FULLMAG_FDM_ERR_CUDA;
}

int fullmag_fdm_backend_copy_field_preview_f64(fullmag_fdm_backend *h, fullmag_fdm_observable obs,
                                               uint32_t pnx, uint32_t pny, uint32_t pnz,
                                               uint32_t z_origin, uint32_t z_stride, double *out,
                                               uint64_t len) {
    if (!h || !out || pnx == 0 || pny == 0 || pnz == 0 || z_stride == 0) return FULLMAG_FDM_ERR_INVALID;
    Backend &b = h->b;
    if (len != (uint64_t)pnx * pny * pnz * 3) { b.last_error = "preview out_len mismatch"; return FULLMAG_FDM_ERR_INVALID; }
    if (!ready(b)) return FULLMAG_FDM_ERR_INVALID;
    return fm::backend_preview_f64(b, obs, pnx, pny, pnz, z_origin, z_stride, out, len) ? FULLMAG_FDM_OK
                                                                                         : FULLMAG_FDM_ERR_CUDA;
}

int fullmag_fdm_backend_copy_field_preview_f32(fullmag_fdm_backend *h, fullmag_fdm_observable obs,
                                               uint32_t pnx, uint32_t pny, uint32_t pnz,
                                               uint32_t z_origin, uint32_t z_stride, float *out,
                                               uint64_t len) {
    if (!h || !out || pnx == 0 || pny == 0 || pnz == 0 || z_stride == 0) return FULLMAG_FDM_ERR_INVALID;
    Backend &b = h->b;
    if (len != (uint64_t)pnx * pny * pnz * 3) { b.last_error = "preview out_len mismatch"; return FULLMAG_FDM_ERR_INVALID; }
    if (!ready(b)) return FULLMAG_FDM_ERR_INVALID;
    return fm::backend_preview_f32(b, obs, pnx, pny, pnz, z_origin, z_stride, out, len) ? FULLMAG_FDM_OK
                                                                                         : FULLMAG_FDM_ERR_CUDA;
}

fullmag_fdm_field_snapshot *fullmag_fdm_backend_begin_field_snapshot(fullmag_fdm_backend *h,
                                                                     fullmag_fdm_observable obs) {
    if (!h) return nullptr;
    Backend &b = h->b;
    if (!ready(b)) return nullptr;
    auto *s = new (std::nothrow) fullmag_fdm_field_snapshot();
    if (!s) { b.last_error = "failed to allocate async field snapshot"; return nullptr; }
    if (!fm::backend_snapshot_begin(b, obs, s->s)) {
        fm::snapshot_free(s->s);
        delete s;
        return nullptr;
    }
    return s;
}

int fullmag_fdm_field_snapshot_wait(fullmag_fdm_field_snapshot *snap, const void **out_data,
                                    uint64_t *out_len, fullmag_fdm_snapshot_desc *out_desc) {
    if (!snap || !out_data || !out_len || !out_desc) return FULLMAG_FDM_ERR_INVALID;
    fm::Snapshot &s = snap->s;
    if (s.pending) {
        cudaSetDevice(s.device);
        if (cudaEventSynchronize(s.done) != cudaSuccess) return FULLMAG_FDM_ERR_CUDA;
        s.pending = false;
    }
    *out_data = s.host;
    *out_len = (uint64_t)s.bytes;
    out_desc->cell_count = s.cell_count;
    out_desc->component_count = 3;
    out_desc->scalar_bytes = (uint32_t)s.scalar;
    out_desc->scalar_type = s.scalar == 4 ? FULLMAG_FDM_SNAPSHOT_SCALAR_F32 : FULLMAG_FDM_SNAPSHOT_SCALAR_F64;
    return FULLMAG_FDM_OK;
}

void fullmag_fdm_field_snapshot_destroy(fullmag_fdm_field_snapshot *snap) {
    if (!snap) return;
    if (snap->s.pending) {
        cudaSetDevice(snap->s.device);
        cudaEventSynchronize(snap->s.done);
    }
    fm::snapshot_free(snap->s);
    delete snap;
}

int fullmag_fdm_backend_upload_magnetization_f64(fullmag_fdm_backend *h, const double *m, uint64_t len) {
    if (!h || !m) return FULLMAG_FDM_ERR_INVALID;
    Backend &b = h->b;
    if (len != (uint64_t)b.n * 3) { b.last_error = "magnetization length mismatch"; return FULLMAG_FDM_ERR_INVALID; }
    if (!ready(b)) return FULLMAG_FDM_ERR_INVALID;
    return fm::backend_upload_m_f64(b, m, len) ? FULLMAG_FDM_OK : FULLMAG_FDM_ERR_CUDA;
}

int fullmag_fdm_backend_upload_magnetization_f32(fullmag_fdm_backend *h, const float *m, uint64_t len) {
    if (!h || !m) return FULLMAG_FDM_ERR_INVALID;
    Backend &b = h->b;
    if (len != (uint64_t)b.n * 3) { b.last_error = "magnetization length mismatch"; return FULLMAG_FDM_ERR_INVALID; }
    if (!ready(b)) return FULLMAG_FDM_ERR_INVALID;
    return fm::backend_upload_m_f32(b, m, len) ? FULLMAG_FDM_OK : FULLMAG_FDM_ERR_CUDA;
}

int fullmag_fdm_backend_refresh_observables(fullmag_fdm_backend *h) {
    if (!h) return FULLMAG_FDM_ERR_INVALID;
    Backend &b = h->b;
    if (!ready(b)) return FULLMAG_FDM_ERR_INVALID;
    return fm::backend_refresh(b) ? FULLMAG_FDM_OK : FULLMAG_FDM_ERR_CUDA;
}

int fullmag_fdm_backend_get_device_info(fullmag_fdm_backend *h, fullmag_fdm_device_info *out) {
    if (!h || !out) return FULLMAG_FDM_ERR_INVALID;
    Backend &b = h->b;
    if (!b.info_valid) {
        if (!ready(b)) return FULLMAG_FDM_ERR_CUDA;
        return FULLMAG_FDM_ERR_CUDA;
    }
    *out = b.info;
    return FULLMAG_FDM_OK;
}

const char *fullmag_fdm_backend_last_error(fullmag_fdm_backend *h) {
    if (!h) return "null handle";
    return h->b.last_error.empty() ? nullptr : h->b.last_error.c_str();
}

void fullmag_fdm_backend_destroy(fullmag_fdm_backend *h) {
    if (!h) return;
    if (h->b.arena) cudaSetDevice(h->b.device);
    fm::backend_free(h->b);
    delete h;
}

int fullmag_fdm_backend_set_profiling(fullmag_fdm_backend *h, int enable) {
    if (!h) return FULLMAG_FDM_ERR_INVALID;
    h->b.profiling = enable != 0;
    return FULLMAG_FDM_OK;
}

int fullmag_fdm_backend_profile_count(fullmag_fdm_backend *h) {
    return h ? (int)h->b.prof_names.size() : 0;
}

int fullmag_fdm_backend_profile_entry(fullmag_fdm_backend *h, int i, const char **name,
                                      double *total_ms, uint64_t *launches) {
    if (!h || i < 0 || i >= (int)h->b.prof_names.size()) return FULLMAG_FDM_ERR_INVALID;
    if (name) *name = h->b.prof_names[i].c_str();
    if (total_ms) *total_ms = h->b.prof_ms[i];
    if (launches) *launches = h->b.prof_count[i];
    return FULLMAG_FDM_OK;
}

void fullmag_fdm_backend_profile_reset(fullmag_fdm_backend *h) {
    if (!h) return;
    for (auto &v : h->b.prof_ms) v = 0.0;
    for (auto &v : h->b.prof_count) v = 0;
}

int fullmag_fdm_backend_memory_info(fullmag_fdm_backend *h, uint64_t *bytes, uint32_t *dims) {
    if (!h) return FULLMAG_FDM_ERR_INVALID;
    if (bytes) *bytes = h->b.arena_bytes;
    if (dims) { dims[0] = h->b.Lx; dims[1] = h->b.Ly; dims[2] = h->b.Lz; }
    return FULLMAG_FDM_OK;
}

int fullmag_fdm_backend_get_stream(fullmag_fdm_backend *h, void **out) {
    if (!h || !out) return FULLMAG_FDM_ERR_INVALID;
    *out = (void *)h->b.stream;
    return h->b.stream ? FULLMAG_FDM_OK : FULLMAG_FDM_ERR_INVALID;
}

void fullmag_fdm_random_unit_vectors(uint64_t seed, uint64_t count, double *out) {
    if (!out) return;
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
            const double nrm = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
            if (nrm > 1e-10) {
                out[3 * v] = c[0] / nrm;
                out[3 * v + 1] = c[1] / nrm;
                out[3 * v + 2] = c[2] / nrm;
                break;
            }
        }
    }
}

int fullmag_fdm_newell_spectra(uint32_t nx, uint32_t ny, uint32_t nz, double dx, double dy, double dz,
                               int thin_film_2d, double *xx, double *yy, double *zz, double *xy,
                               double *xz, double *yz) {
    if (nx == 0 || ny == 0 || nz == 0 || !(dx > 0) || !(dy > 0) || !(dz > 0)) return FULLMAG_FDM_ERR_INVALID;
    const bool thin = thin_film_2d && nz == 1;
    std::vector<double> spec[6];
    fm::newell_octant_spectra((int)nx, (int)ny, (int)nz, dx, dy, dz, thin, spec);
    const long long Lx = 2LL * nx, Ly = 2LL * ny, Lz = thin ? 1 : 2LL * nz;
    const long long KX = nx + 1, KY = ny + 1;
    const bool oddx[6] = {false, false, false, true, true, false};
    const bool oddy[6] = {false, false, false, true, false, true};
    const bool oddz[6] = {false, false, false, false, true, true};
    double *outs[6] = {xx, yy, zz, xy, xz, yz};
    for (int c = 0; c < 6; ++c) {
        double *o = outs[c];
        if (!o) continue;
        par_for((size_t)(Lz * Ly), [&](size_t row) {
            const long long kz = (long long)row / Ly, ky = (long long)row % Ly;
            const long long kyo = ky <= (long long)ny ? ky : Ly - ky;
            const long long kzo = kz <= (long long)(Lz / 2) ? kz : Lz - kz;
            const double sy = (ky > (long long)ny && oddy[c]) ? -1.0 : 1.0;
            const double sz = (kz > Lz / 2 && oddz[c]) ? -1.0 : 1.0;
            for (long long kx = 0; kx < Lx; ++kx) {
                const long long kxo = kx <= (long long)nx ? kx : Lx - kx;
                const double sx = (kx > (long long)nx && oddx[c]) ? -1.0 : 1.0;
                const double v = spec[c][((size_t)kzo * KX + kxo) * KY + kyo] * sx * sy * sz;
                const long long idx = kx + Lx * (ky + Ly * kz);
                o[2 * idx] = v;
                o[2 * idx + 1] = 0.0;
            }
        });
    }
    return FULLMAG_FDM_OK;
}

}  // extern "C"
