// backend.cu — create / step / transfer logic of the B200 FDM stepper.
//
// Behaviour mirrors the reference backend's C ABI contract
// (native/backends/fdm/src/api.cpp:87-376, context.cu:377-1316) and the CPU
// engine's step semantics (crates/fullmag-engine/src/lib.rs:1217-1249 Heun,
// 1412-1568 DP45).  Differences by design:
//   - one arena allocation per handle, one non-blocking stream, no blocking
//     device-wide syncs except the single stats read-back per step;
//   - the RHS at the accepted state is kept (k1 cache), so a Heun step costs
//     two demag evaluations instead of three and a rejected DP45 attempt does
//     not recompute stage 1;
//   - DP45's error max-norm is reduced on the device (FP64), not on the host.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>

#include "backend.hpp"
#include "backend_impl.hpp"
#include "demag.cuh"
#include "demag_reg.cuh"
#include "demag_yz.hpp"
#include "demag_row.hpp"
#include "stage_vec.hpp"
#include "demag_yzy.hpp"
#include "demag_zdw.hpp"
#include "newell_host.hpp"
#include "stages.cuh"
#include "adjoint.cuh"

namespace fm {

// exp(-2 pi i k / 64), k < 64, for the register FFTs (per device).
bool upload_tw64(Backend &b) {
    double2 d[64];
    float2 f[64];
    for (int k = 0; k < 64; ++k) {
        const double a = 2.0 * kPi * (double)k / 64.0;
        d[k] = make_double2(std::cos(a), -std::sin(a));
        f[k] = make_float2((float)d[k].x, (float)d[k].y);
    }
    return cuda_ok(b, cudaMemcpyToSymbol(c_tw64d, d, sizeof(d)), "twiddle64 d") &&
           cuda_ok(b, cudaMemcpyToSymbol(c_tw64f, f, sizeof(f)), "twiddle64 f");
}

template <int V> using IC = std::integral_constant<int, V>;

// (L1, L2) split of a power-of-two line length, as fftreg.cuh's l2_for.
template <class F>
static bool with_split(int L, F &&f) {
    switch (L) {
        case 2: f(IC<2>{}, IC<1>{}); return true;
        case 4: f(IC<4>{}, IC<1>{}); return true;
        case 8: f(IC<8>{}, IC<1>{}); return true;
        case 16: f(IC<16>{}, IC<1>{}); return true;
        case 32: f(IC<32>{}, IC<1>{}); return true;
        case 64: f(IC<8>{}, IC<8>{}); return true;
        case 128: f(IC<16>{}, IC<8>{}); return true;
        case 256: f(IC<16>{}, IC<16>{}); return true;
        case 512: f(IC<32>{}, IC<16>{}); return true;
        case 1024: f(IC<32>{}, IC<32>{}); return true;
        case 2048: f(IC<64>{}, IC<32>{}); return true;
        case 4096: f(IC<64>{}, IC<64>{}); return true;
        default: return false;
    }
}

static bool is_pow2(int L) { return L >= 2 && (L & (L - 1)) == 0; }

static bool env_is(const char *name, const char *value) {
    const char *v = std::getenv(name);
    return v && std::strcmp(v, value) == 0;
}

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
bool cuda_ok(Backend &b, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return true;
    char buf[512];
    std::snprintf(buf, sizeof(buf), "CUDA error in %s: %s (%d)", what, cudaGetErrorString(e), (int)e);
    b.last_error = buf;
    return false;
}

static bool check_launch(Backend &b, const char *what) {
    return cuda_ok(b, cudaGetLastError(), what);
}

bool make_line_plan(int L, LinePlan &p) {
    p.L = L;
    p.nstages = 0;
    int m = L;
    while (m % 4 == 0 && m > 1) { p.radix[p.nstages++] = 4; m /= 4; }
    while (m % 2 == 0 && m > 1) { p.radix[p.nstages++] = 2; m /= 2; }
    for (int r : {3, 5, 7})
        while (m % r == 0 && m > 1) {
            if (p.nstages >= kMaxStages) return false;
            p.radix[p.nstages++] = r;
            m /= r;
        }
    return m == 1;
}

// Timing of one launch group (extension API: per-kernel device time).
struct ProfScope {
    Backend &b;
    int id = -1;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ProfScope(Backend &b_, const char *name) : b(b_) {
        if (!b.profiling) return;
        for (size_t i = 0; i < b.prof_names.size(); ++i)
            if (b.prof_names[i] == name) { id = (int)i; break; }
        if (id < 0) {
            id = (int)b.prof_names.size();
            b.prof_names.emplace_back(name);
            b.prof_ms.push_back(0.0);
            b.prof_count.push_back(0);
        }
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, b.stream);
    }
    ~ProfScope() {
        if (!b.profiling || id < 0) return;
        cudaEventRecord(e1, b.stream);
        b.prof_pending.push_back({id, {e0, e1}});
    }
};

void prof_collect(Backend &b) {
    for (auto &p : b.prof_pending) {
        float ms = 0.f;
        cudaEventSynchronize(p.second.second);
        cudaEventElapsedTime(&ms, p.second.first, p.second.second);
        b.prof_ms[p.first] += ms;
        b.prof_count[p.first] += 1;
        cudaEventDestroy(p.second.first);
        cudaEventDestroy(p.second.second);
    }
    b.prof_pending.clear();
}

// ---------------------------------------------------------------------------
// typed implementation
// ---------------------------------------------------------------------------
template <typename T>
struct Impl {
    using C = cx<T>;

    static DemagArgs<T> demag_args(Backend &b, const void *m, void *hd, bool unit = false) {
        DemagArgs<T> a{};
        a.nx = b.nx; a.ny = b.ny; a.nz = b.nz; a.n = b.n;
        a.Lx = b.Lx; a.Ly = b.Ly; a.Lz = b.Lz; a.nkx = b.nkx;
        a.KZ = b.KZ; a.KY = b.KY;
        a.px = b.px; a.py = b.py; a.pz = b.pz;
        a.twx = (const C *)b.twx; a.twy = (const C *)b.twy; a.twz = (const C *)b.twz;
        a.twxT = (const C *)b.twxT; a.twyT = (const C *)b.twyT;
        a.s1 = (C *)b.s1; a.s2 = (C *)b.s2;
        a.spec = (const T *)b.spec;
        a.m = (const T *)m;
        a.mask = b.d_mask;
        a.ms_map = b.d_msmap;
        a.ms = b.ms;
        a.vf = b.boundary_tier ? b.d_vf : nullptr;
        a.unit_source = unit ? 1 : 0;
        a.hd = (T *)hd;
        a.norm = 1.0 / ((double)b.Lx * (double)b.Ly * (double)b.Lz);
        a.lines_x = b.lines_x; a.lines_y = b.lines_y; a.kt_z = b.kt_z; a.kb_y = b.kb_y;
        return a;
    }

    // direct z convolution for nz = NZ (runtime nz -> template)
    template <typename F>
    static void with_nz(int nz, F &&f) {
        switch (nz) {
            case 1: f(std::integral_constant<int, 1>{}); break;
            case 2: f(std::integral_constant<int, 2>{}); break;
            case 3: f(std::integral_constant<int, 3>{}); break;
            case 4: f(std::integral_constant<int, 4>{}); break;
            case 5: f(std::integral_constant<int, 5>{}); break;
            case 6: f(std::integral_constant<int, 6>{}); break;
            case 7: f(std::integral_constant<int, 7>{}); break;
            case 8: f(std::integral_constant<int, 8>{}); break;
            default: break;
        }
    }

    // Register-FFT path: power-of-two x/y lengths <= 1024 (FP64) or 4096 (FP32).
    // z: direct summation for nz <= 8 (any nz; FULLMAG_FDM_ZCONV=fft keeps the
    // z FFT) and in FP32 for nz <= 16 (k_zdw), else the register z FFT, Lz a
    // power of two <= 16 (FP64) or 32 (FP32) since a thread holds 3 z lines.
    static bool configure_reg(Backend &b) {
        const bool dbl = sizeof(T) == 8;
        const int maxxy = dbl ? 1024 : 4096, maxz = dbl ? 16 : 32;
        if (!is_pow2(b.Lx) || !is_pow2(b.Ly) || b.Lx > maxxy || b.Ly > maxxy) return false;
        const bool zdw = zdw_wanted(b, !dbl);
        b.use_zdw = false;
        b.zdirect = zdw || (!b.thin && b.nz <= 8 && !b.want_yz && !env_is("FULLMAG_FDM_ZCONV", "fft"));
        if (!b.thin && !b.zdirect && (!is_pow2(b.Lz) || b.Lz > maxz)) return false;
        const size_t sz = sizeof(C), maxs = 200 * 1024;
        const int target = 128;  // x passes: small blocks, several per SM
        bool ok = true;
        // x passes: lines_x complex lines (row pairs) of L2 threads
        with_split(b.Lx, [&](auto l1, auto l2) {
            constexpr int L1 = decltype(l1)::value, L2 = decltype(l2)::value;
            if constexpr (sizeof(T) == 8 && L1 > 32) { ok = false; } else {
                constexpr int TE = line_region<L1, L2>();
                const int unit = L2 >= 32 ? 1 : 32 / L2;    // lines per warp multiple
                int lp = std::max(1, target / L2);
                lp = std::min(lp, std::max(unit, ((b.ny + 1) / 2 + unit - 1) / unit * unit));
                while (lp > unit && (size_t)(lp * TE) * sz > maxs) lp -= unit;
                b.lines_x = lp;
                b.thr_x = lp * L2;
                b.rsm_x = (size_t)(lp * TE) * sz;
                ok &= cuda_ok(b, cudaFuncSetAttribute(k_xf_r<T, L1, L2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b.rsm_x), "attr xf_r");
                // even ny: the pair gather (both rows of a line pair per load)
                b.xi_pair = b.ny % 2 == 0;
                b.rsm_xi = (size_t)lp * (b.xi_pair ? xi_stride<T, L1, L2, true>() : xi_stride<T, L1, L2, false>()) * sz +
                           (size_t)L1 * L2 * sz;  // line regions + the twiddle table
                ok &= cuda_ok(b, cudaFuncSetAttribute(b.xi_pair ? k_xi_r<T, L1, L2, xi_gather_pair<T>(), true>
                                                                : k_xi_r<T, L1, L2, xi_gather<T>(), false>,
                                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b.rsm_xi), "attr xi_r");
                // pipelined x forward for a uniform material with 16-byte rows
                b.use_xpipe = false;
                if (ok && !b.has_mask && !b.has_ms_map && !b.boundary_tier && (b.nx * sizeof(T)) % 16 == 0) {
                    const int RB = 2 * lp;
                    const size_t smem = xpipe_region_bytes<L1, L2, T>(lp) + (size_t)2 * RB * b.nx * sizeof(T) +
                                        (size_t)L1 * L2 * sizeof(C);
                    int occ = 0, sms = 148;
                    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b.device);
                    if (smem <= 200 * 1024 &&
                        cudaFuncSetAttribute(k_xf_pipe<T, L1, L2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess &&
                        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_xf_pipe<T, L1, L2>, b.thr_x, smem) == cudaSuccess &&
                        occ > 0 && !env_is("FULLMAG_FDM_XPIPE", "off")) {
                        b.groups_x = 3 * b.nz * ((b.ny + RB - 1) / RB);
                        b.grid_xpipe = std::min(b.groups_x, occ * sms);
                        b.rsm_xpipe = smem;
                        b.use_xpipe = true;
                    }
                    cudaGetLastError();
                }
            }
        });
        if (!ok) return false;
        with_split(b.Ly, [&](auto l1, auto l2) {
            constexpr int L1 = decltype(l1)::value, L2 = decltype(l2)::value;
            if constexpr (sizeof(T) == 8 && L1 > 32) { ok = false; } else {
                if (b.thin) {
                    constexpr int TE = line_region<L1, L2>();
                    const int unit = L2 >= 32 ? 1 : 32 / L2;  // kb multiple so 3*kb*L2 % 32 == 0
                    int kb = std::max(unit, (256 / (3 * L2)) / unit * unit);
                    kb = std::min(kb, std::max(unit, (b.nkx + unit - 1) / unit * unit));
                    while (kb > unit && (size_t)(3 * kb * TE) * sz > maxs) kb -= unit;
                    b.kb_y = kb;
                    b.thr_yc = 3 * kb * L2;
                    b.rsm_yc = (size_t)(3 * kb * TE) * sz;
                    ok &= b.rsm_yc <= 227 * 1024 && b.thr_yc <= 256;
                    ok &= cuda_ok(b, cudaFuncSetAttribute(k_yc_r<T, L1, L2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b.rsm_yc), "attr yc_r");
                } else {
                    constexpr int TE = tile_elems(L1, L2);
                    // lines per block: for 32-thread lines 6 (FP32) or 4 (FP64) lines,
                    // measured at Ly = 1024 against 8 (FP32 -2 us per pass; FP64 8 lines
                    // leave one 135 KB block per SM: 86.5 -> 74.5 us forward); at most
                    // 68 KB of tiles per block otherwise
                    int lpb = L2 == 32 ? (sizeof(T) == 8 ? 4 : 6) : std::max(1, 256 / L2);
                    while (lpb > 1 && (size_t)(lpb * TE) * sz > 68 * 1024) lpb /= 2;
                    b.lines_y = lpb;
                    b.thr_y = lpb * L2;
                    b.rsm_y = (size_t)(lpb * TE) * sz;
                    ok &= cuda_ok(b, cudaFuncSetAttribute(k_yf_r<T, L1, L2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b.rsm_y), "attr yf_r");
                    ok &= cuda_ok(b, cudaFuncSetAttribute(k_yi_r<T, L1, L2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b.rsm_y), "attr yi_r");
                }
            }
        });
        if (ok && !b.thin && b.want_yz && !yz_configure<T>(b)) return false;
        if (ok && b.zdirect) {
            with_nz(b.nz, [&](auto nzc) {
                constexpr int NZ = decltype(nzc)::value;
                const size_t smem = (size_t)zd_threads<T>() * zd_smem_per_thread<T, NZ>();
                int occ = 0, sms = 148;
                cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b.device);
                ok &= cuda_ok(b, cudaFuncSetAttribute(k_zd<T, NZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "attr zd");
                ok &= cuda_ok(b, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_zd<T, NZ>, zd_threads<T>(), smem), "occupancy zd");
                const long long cols = (long long)b.nkx * b.Ly;
                b.grid_zd = (int)std::max<long long>(1, std::min<long long>((cols + zd_threads<T>() - 1) / zd_threads<T>(), (long long)std::max(occ, 1) * sms));
                b.rsm_zd = smem;
            });
        }
        b.use_yzy = false;
        if (ok && zdw) {
            ok &= zdw_configure(b);
            if (ok && !b.use_zdw) return false;  // no resident block: the generic path
        }
        if (ok && b.zdirect && !b.use_zdw) ok &= yzy_configure<T>(b);
        return ok;
    }

    static bool demag_reg(Backend &b, const void *m, void *hd, bool unit = false) {
        DemagArgs<T> a = demag_args(b, m, hd, unit);
        x_fwd_reg(b, a);
        if (!mid_reg(b, a)) return false;
        x_inv_reg(b, a);
        return check_launch(b, "demag (register FFT)");
    }

    // x forward: Ms m -> S1
    static void x_fwd_reg(Backend &b, const DemagArgs<T> &a) {
        const int RB = 2 * b.lines_x;
        dim3 gx((b.ny + RB - 1) / RB, b.nz, 3);
        with_split(b.Lx, [&](auto l1, auto l2) {
            constexpr int L1 = decltype(l1)::value, L2 = decltype(l2)::value;
            if constexpr (!(sizeof(T) == 8 && L1 > 32)) {
                ProfScope p(b, "demag_x_fwd");
                if (b.use_xpipe)
                    k_xf_pipe<T, L1, L2><<<b.grid_xpipe, b.thr_x, b.rsm_xpipe, b.stream>>>(a, b.groups_x);
                else
                    k_xf_r<T, L1, L2><<<gx, b.thr_x, b.rsm_x, b.stream>>>(a);
            }
        });
    }

    // the y (thin film) or y / z passes: S1 -> S1
    static bool mid_reg(Backend &b, const DemagArgs<T> &a) {
        if (b.thin) {
            with_split(b.Ly, [&](auto l1, auto l2) {
                constexpr int L1 = decltype(l1)::value, L2 = decltype(l2)::value;
                if constexpr (!(sizeof(T) == 8 && L1 > 32)) {
                    ProfScope p(b, "demag_y_conv");
                    k_yc_r<T, L1, L2><<<(b.nkx + b.kb_y - 1) / b.kb_y, b.thr_yc, b.rsm_yc, b.stream>>>(a);
                }
            });
        } else if (b.use_yz) {
            ProfScope p(b, "demag_yz");
            if (!yz_launch(b, a)) return false;
        } else if (b.use_yzy) {
            ProfScope p(b, "demag_yzy");
            if (!yzy_launch(b, a)) return false;
        } else {
            const long long lines = 3LL * b.nz * b.nkx;
            const unsigned gy = (unsigned)((lines + b.lines_y - 1) / b.lines_y);
            with_split(b.Ly, [&](auto l1, auto l2) {
                constexpr int L1 = decltype(l1)::value, L2 = decltype(l2)::value;
                if constexpr (!(sizeof(T) == 8 && L1 > 32)) {
                    ProfScope p(b, "demag_y_fwd");
                    k_yf_r<T, L1, L2><<<gy, b.thr_y, b.rsm_y, b.stream>>>(a);
                }
            });
            if (b.use_zdw) {
                ProfScope p(b, "demag_z_direct");
                if constexpr (sizeof(T) == 4) zdw_launch(b, a);
            } else if (b.zdirect) {
                ProfScope p(b, "demag_z_direct");
                with_nz(b.nz, [&](auto nzc) {
                    constexpr int NZ = decltype(nzc)::value;
                    k_zd<T, NZ><<<b.grid_zd, zd_threads<T>(), b.rsm_zd, b.stream>>>(a);
                });
            } else {
                ProfScope p(b, "demag_z_conv");
                const long long cols = (long long)b.nkx * b.Ly;
                // one thread per column up to 3 x 8 z points, a thread pair (split by
                // kz parity) above
                const int P = (b.Lz > 8) ? 2 : 1;
                const unsigned gz2 = (unsigned)std::min<long long>((cols * P + 127) / 128, 148LL * 64);
                switch (b.Lz * 10 + P) {
                    case 21: k_zc_r<T, 2, 1><<<gz2, 128, 0, b.stream>>>(a); break;
                    case 41: k_zc_r<T, 4, 1><<<gz2, 128, 0, b.stream>>>(a); break;
                    case 81: k_zc_r<T, 8, 1><<<gz2, 128, 0, b.stream>>>(a); break;
                    case 162: k_zc_r<T, 16, 2><<<gz2, 128, 0, b.stream>>>(a); break;
                    case 322: if constexpr (sizeof(T) == 4) k_zc_r<T, 32, 2><<<gz2, 128, 0, b.stream>>>(a); break;
                    default: break;
                }
            }
            with_split(b.Ly, [&](auto l1, auto l2) {
                constexpr int L1 = decltype(l1)::value, L2 = decltype(l2)::value;
                if constexpr (!(sizeof(T) == 8 && L1 > 32)) {
                    ProfScope p(b, "demag_y_inv");
                    k_yi_r<T, L1, L2><<<gy, b.thr_y, b.rsm_y, b.stream>>>(a);
                }
            });
        }
        return true;
    }

    // x inverse: S1 -> H_d
    static void x_inv_reg(Backend &b, const DemagArgs<T> &a) {
        const int RB = 2 * b.lines_x;
        dim3 gx((b.ny + RB - 1) / RB, b.nz, 3);
        with_split(b.Lx, [&](auto l1, auto l2) {
            constexpr int L1 = decltype(l1)::value, L2 = decltype(l2)::value;
            if constexpr (!(sizeof(T) == 8 && L1 > 32)) {
                ProfScope p(b, "demag_x_inv");
                if (b.xi_pair)
                    k_xi_r<T, L1, L2, xi_gather_pair<T>(), true><<<gx, b.thr_x, b.rsm_xi, b.stream>>>(a);
                else
                    k_xi_r<T, L1, L2, xi_gather<T>(), false><<<gx, b.thr_x, b.rsm_xi, b.stream>>>(a);
            }
        });
    }

    // the ring-fed stage kernels' shared memory (above 48 KB for FP64)
    static bool configure_stage(Backend &b) {
        // FP32-mixed: 16-byte cell groups with FP32 stencil and RHS when rows are
        // whole groups and the material has at most a mask and an Ms map
        // (FULLMAG_FDM_STAGE=ring or plain keeps the one-value-per-load kernels of
        // a uniform material, =cell the general one).  FP64 keeps those: measured
        // at 512 x 512 x 8 the FP64 group kernels took 84.5 / 74.2 us (RHS /
        // corrector) against the ring's 70.0 / 60.0 us.
        const bool rows16 = sizeof(T) == 4 && b.nx % (16 / (int)sizeof(T)) == 0;
        const bool simple = !b.has_regions && !b.boundary_tier;
        const bool keep = env_is("FULLMAG_FDM_STAGE", "ring") || env_is("FULLMAG_FDM_STAGE", "plain") ||
                          env_is("FULLMAG_FDM_STAGE", "cell");
        b.stage_vec = rows16 && simple && !keep && 3ULL * (unsigned long long)b.n < (1ULL << 32);
        b.stage_vec_mk = b.stage_vec && (b.has_mask || b.has_ms_map);
        if (!b.stage_plain) return true;
        b.stage_ring = !env_is("FULLMAG_FDM_STAGE", "plain");
        if (!b.stage_ring) return true;
        const int thr = 32 * kStagePlainBY;
        bool ok = true;
        ok &= cuda_ok(b, cudaFuncSetAttribute(k_stage_ring<T, MODE_EVAL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)ring_bytes<T, MODE_EVAL>(thr)), "attr stage ring");
        ok &= cuda_ok(b, cudaFuncSetAttribute(k_stage_ring<T, MODE_HEUN_CORR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)ring_bytes<T, MODE_HEUN_CORR>(thr)), "attr stage ring");
        ok &= cuda_ok(b, cudaFuncSetAttribute(k_stage_ring<T, MODE_ERR_LAST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)ring_bytes<T, MODE_ERR_LAST>(thr)), "attr stage ring");
        return ok;
    }

    static bool configure(Backend &b) {
        if (!upload_tw64(b)) return false;
        if (!b.force_stockham && configure_reg(b)) {
            b.use_reg = true;
            return row_configure<T>(b);
        }
        b.use_reg = false;
        b.zdirect = false;
        b.use_yzy = false;
        b.use_zdw = false;
        if (!b.last_error.empty()) return false;
        const int budget = 100 * 1024;
        const int sz = (int)sizeof(C);
        auto lines_for = [&](int ld, int L, int per_line_mult, int maxl) {
            int avail = budget - L * sz;
            int l = avail / (2 * ld * sz * per_line_mult);
            return std::max(1, std::min(maxl, l));
        };
        b.lines_x = lines_for(b.Lx + 3, b.Lx, 1, 8);
        b.smem_xf = (size_t)sz * (b.Lx + 2 * (size_t)b.lines_x * (b.Lx + 3));
        if (b.thin) {
            b.kb_y = lines_for(b.Ly + 1, b.Ly, 3, 8);
            b.kb_y = std::min(b.kb_y, b.nkx);
            b.smem_yc = (size_t)sz * (b.Ly + 2 * 3 * (size_t)b.kb_y * (b.Ly + 1));
        } else {
            b.lines_y = lines_for(b.Ly + 1, b.Ly, 1, 16);
            b.smem_yf = (size_t)sz * (b.Ly + 2 * (size_t)b.lines_y * (b.Ly + 1));
            b.kt_z = lines_for(b.Lz + 1, b.Lz, 3, 32);
            b.kt_z = std::min(b.kt_z, b.Ly);
            b.smem_z = (size_t)sz * (b.Lz + 2 * 3 * (size_t)b.kt_z * (b.Lz + 1));
        }
        const size_t maxs = 227 * 1024;
        if (b.smem_xf > maxs || b.smem_yf > maxs || b.smem_z > maxs || b.smem_yc > maxs) {
            b.last_error = "padded FFT length too large for the shared-memory FFT (max 4096 per axis)";
            return false;
        }
        bool ok = true;
        ok &= cuda_ok(b, cudaFuncSetAttribute(k_x_fwd<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b.smem_xf), "attr x_fwd");
        ok &= cuda_ok(b, cudaFuncSetAttribute(k_x_inv<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b.smem_xf), "attr x_inv");
        if (b.thin) {
            ok &= cuda_ok(b, cudaFuncSetAttribute(k_y_conv<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b.smem_yc), "attr y_conv");
        } else {
            ok &= cuda_ok(b, cudaFuncSetAttribute(k_y_fwd<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b.smem_yf), "attr y_fwd");
            ok &= cuda_ok(b, cudaFuncSetAttribute(k_y_inv<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b.smem_yf), "attr y_inv");
            ok &= cuda_ok(b, cudaFuncSetAttribute(k_z_conv<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b.smem_z), "attr z_conv");
        }
        return ok;
    }

    // H_d(m) into hd, then the sparse boundary correction when the plan has one.
    // unit: the source is m itself on active cells (no Ms), for the adjoint.
    static bool demag(Backend &b, const void *m, void *hd, bool unit = false) {
        if (!b.enable_demag) return true;
        b.s1_state = 0;  // S1 now holds this evaluation's convolved spectrum
        if (hd == b.hd) b.hd_stale = (m != b.m) || unit;
        if (!(b.use_reg ? demag_reg(b, m, hd, unit) : demag_stockham(b, m, hd, unit))) return false;
        if (b.corr_targets) {
            {
                ProfScope p(b, "demag_boundary_corr");
                k_demag_corr<T><<<(b.corr_targets + 255) / 256, 256, 0, b.stream>>>(
                    (const T *)m, (T *)hd, b.n, b.d_vf, b.d_corr_tgt, b.d_corr_src, b.d_corr_ten, b.ms,
                    b.corr_targets, b.corr_stencil);
            }
            return check_launch(b, "demag boundary correction");
        }
        return true;
    }

    static bool demag_stockham(Backend &b, const void *m, void *hd, bool unit) {
        DemagArgs<T> a = demag_args(b, m, hd, unit);
        const int RB = 2 * b.lines_x;
        dim3 gx((b.ny + RB - 1) / RB, b.nz, 3);
        {
            ProfScope p(b, "demag_x_fwd");
            k_x_fwd<T><<<gx, 256, b.smem_xf, b.stream>>>(a);
        }
        if (b.thin) {
            ProfScope p(b, "demag_y_conv");
            k_y_conv<T><<<(b.nkx + b.kb_y - 1) / b.kb_y, 256, b.smem_yc, b.stream>>>(a);
        } else {
            const long long lines = 3LL * b.nz * b.nkx;
            const unsigned gy = (unsigned)((lines + b.lines_y - 1) / b.lines_y);
            {
                ProfScope p(b, "demag_y_fwd");
                k_y_fwd<T><<<gy, 256, b.smem_yf, b.stream>>>(a);
            }
            {
                ProfScope p(b, "demag_z_conv");
                dim3 gz((b.Ly + b.kt_z - 1) / b.kt_z, b.nkx);
                k_z_conv<T><<<gz, 256, b.smem_z, b.stream>>>(a);
            }
            {
                ProfScope p(b, "demag_y_inv");
                k_y_inv<T><<<gy, 256, b.smem_yf, b.stream>>>(a);
            }
        }
        {
            ProfScope p(b, "demag_x_inv");
            k_x_inv<T><<<gx, 256, b.smem_xf, b.stream>>>(a);
        }
        return check_launch(b, "demag");
    }

    static StageArgs<T> stage_args(Backend &b, const void *m, double t) {
        StageArgs<T> s{};
        s.nx = b.nx; s.ny = b.ny; s.nz = b.nz; s.n = b.n;
        s.idx2 = (T)(1.0 / (b.dx * b.dx));
        s.idy2 = (T)(1.0 / (b.dy * b.dy));
        s.idz2 = (T)(1.0 / (b.dz * b.dz));
        s.dinv[0] = 1.0 / (b.dx * b.dx);
        s.dinv[1] = 1.0 / (b.dy * b.dy);
        s.dinv[2] = 1.0 / (b.dz * b.dz);
        s.aex = b.aex; s.ms = b.ms; s.ms_map = b.d_msmap;
        s.ex_pref = 2.0 * b.aex / (kMu0 * b.ms);
        s.ex_tier = b.ex_tier;
        s.vf = b.d_vf;
        s.face = b.d_face;
        s.delta = b.d_delta;
        s.phi_floor = b.phi_floor;
        s.delta_min = b.delta_min;
        s.cell[0] = b.dx; s.cell[1] = b.dy; s.cell[2] = b.dz;
        s.ex_pref_lut = 2.0 / (kMu0 * b.ms);
        s.mask = b.d_mask; s.region = b.d_region; s.lut = b.d_lut;
        s.enable_exchange = b.enable_exchange; s.enable_demag = b.enable_demag;
        s.has_ext = b.has_ext;
        for (int c = 0; c < 3; ++c) { s.hext[c] = b.hext[c]; s.hac[c] = b.hac[c]; }
        s.ac_omega = 2.0 * kPi * b.ac_freq;
        s.gamma_bar = b.gamma / (1.0 + b.alpha * b.alpha);
        s.alpha = b.alpha;
        s.precession = b.precession;
        s.vol = b.dx * b.dy * b.dz;
        s.t = t;
        s.m = (const T *)m;
        s.hd = (const T *)b.hd;
        return s;
    }

    static unsigned grid_cells(const Backend &b) {
        return (unsigned)std::min<long long>((b.n + 255) / 256, 148LL * 16);
    }
    // stage kernels: one thread per cell, block (32, 4, 2)
    static dim3 stage_grid(const Backend &b) {
        return dim3((b.nx + 31) / 32, (b.ny + 3) / 4, (b.nz + 1) / 2);
    }

    // One stage launch: the z-marching kernel for a uniform material, the
    // general one (mask, Ms map, region LUT) otherwise.
    template <int MODE>
    static void launch_stage(Backend &b, const StageArgs<T> &s) {
        if constexpr (sizeof(T) == 4) {
            if (b.stage_vec) {
                stage_vec_launch(b, s, MODE);
                return;
            }
        }
        if (b.stage_plain) {
            const dim3 g((b.nx + 31) / 32, (b.ny + kStagePlainBY - 1) / kStagePlainBY,
                         (b.nz + b.stage_zb - 1) / b.stage_zb);
            if (b.stage_ring)
                k_stage_ring<T, MODE><<<g, dim3(32, kStagePlainBY, 1), ring_bytes<T, MODE>(32 * kStagePlainBY),
                                        b.stream>>>(s, b.stage_zb);
            else
                k_stage_plain<T, MODE><<<g, dim3(32, kStagePlainBY, 1), 0, b.stream>>>(s, b.stage_zb);
        } else {
            k_stage<T, MODE><<<stage_grid(b), dim3(32, 4, 2), 0, b.stream>>>(s);
        }
    }

    // k = RHS(m, t); optional observables and diagnostics.
    static bool eval(Backend &b, const void *m, double t, void *kout, bool diag, bool obs,
                     void *pred_out = nullptr, double pred_dt = 0.0) {
        StageArgs<T> s = stage_args(b, m, t);
        s.kout = (T *)kout;
        s.pred_out = (T *)pred_out;
        s.pred_dt = pred_dt;
        s.hex_out = obs ? (T *)b.hex : nullptr;
        s.heff_out = obs ? (T *)b.heff : nullptr;
        s.partials = diag ? b.partials : nullptr;
        s.counter = b.counter;
        s.out = b.d_out;
        {
            ProfScope p(b, "stage_eval");
            launch_stage<MODE_EVAL>(b, s);
        }
        return check_launch(b, "stage_eval");
    }

    // k = RHS(m, t) with H_ex and H_eff written to the given buffers (adjoint).
    static bool eval_fields(Backend &b, const void *m, double t, void *kout, void *hex, void *heff) {
        StageArgs<T> s = stage_args(b, m, t);
        s.kout = (T *)kout;
        s.hex_out = (T *)hex;
        s.heff_out = (T *)heff;
        s.partials = nullptr;
        s.counter = b.counter;
        s.out = b.d_out;
        {
            ProfScope p(b, "stage_eval");
            launch_stage<MODE_EVAL>(b, s);
        }
        return check_launch(b, "stage_eval (adjoint)");
    }

    static bool combine(Backend &b, int form, const void *m0, std::initializer_list<void *> ks,
                        std::initializer_list<double> cs, double dt, void *out) {
        CombineArgs<T> a{};
        a.n = b.n;
        a.m0 = (const T *)m0;
        int i = 0;
        for (void *k : ks) a.k[i++] = (const T *)k;
        i = 0;
        for (double c : cs) a.c[i++] = c;
        a.dt = dt;
        a.form = form;
        a.out = (T *)out;
        {
            ProfScope p(b, "stage_combine");
            bool done = false;
            if constexpr (sizeof(T) == 4) {
                if (b.stage_vec && b.n % 4 == 0) {
                    combine_vec_launch(b, a);  // 16-byte groups of cells, the group kernels' renormalisation
                    done = true;
                }
            }
            if (!done) k_combine<T><<<grid_cells(b), 256, 0, b.stream>>>(a);
        }
        return check_launch(b, "combine");
    }

    // the reducing kernel wrote the statistics into the mapped host buffer h_out
    static bool read_stats(Backend &b) { return cuda_ok(b, cudaStreamSynchronize(b.stream), "stats sync"); }

    static void fill_stats(Backend &b, double dt, fullmag_fdm_step_stats *st) {
        const double *o = b.h_out;
        st->step = b.step_count;
        st->time_seconds = b.time;
        st->dt_seconds = dt;
        st->exchange_energy_joules = b.enable_exchange ? o[Q_EEX] : 0.0;
        st->demag_energy_joules = b.enable_demag ? o[Q_EDEMAG] : 0.0;
        st->external_energy_joules = b.has_ext ? o[Q_EEXT] : 0.0;
        st->total_energy_joules =
            st->exchange_energy_joules + st->demag_energy_joules + st->external_energy_joules;
        st->max_effective_field_amplitude = std::sqrt(o[Q_HEFF2]);
        st->max_demag_field_amplitude = b.enable_demag ? std::sqrt(o[Q_HD2]) : 0.0;
        st->max_rhs_amplitude = std::sqrt(o[Q_RHS2]);
    }

    static bool ensure_k1(Backend &b) {
        if (b.k1_valid) return true;
        if (!demag(b, b.m, b.hd)) return false;
        if (!eval(b, b.m, b.time, b.k[0], false, false)) return false;
        b.k1_valid = true;
        return true;
    }

    // One launch of the fused row pass (x inverse, stage, x forward of the new
    // state) on S1, which holds the convolved spectrum of s.m.
    static bool row_pass(Backend &b, int mode, const StageArgs<T> &s) {
        const DemagArgs<T> a = demag_args(b, s.m, nullptr);
        ProfScope p(b, mode == MODE_EVAL ? "row_eval" : mode == MODE_HEUN_CORR ? "row_heun_corr" : "row_x_fwd");
        return row_launch(b, a, s, mode);
    }

    // S1 = X(Ms m) of state m by the row pass's own x forward (phase 4 alone)
    static bool row_x_fwd(Backend &b, const void *m) {
        StageArgs<T> s = stage_args(b, m, b.time);
        return row_pass(b, MODE_ROW_XFWD, s);
    }

    // k1 = RHS(m) and the predictor normalize(m + k1 dt) into mstage by the row
    // pass, the arithmetic of every later step, leaving S1 = X(Ms m_p).
    static bool rows_k1(Backend &b, double dt) {
        const DemagArgs<T> a = demag_args(b, b.m, nullptr);
        if (!row_x_fwd(b, b.m) || !mid_reg(b, a)) return false;
        StageArgs<T> s = stage_args(b, b.m, b.time);
        s.kout = (T *)b.k[0];
        s.pred_out = (T *)b.mstage;
        s.pred_dt = dt;
        s.counter = b.counter;
        s.out = b.d_out;
        if (!row_pass(b, MODE_EVAL, s)) return false;
        b.k1_valid = b.pred_valid = true;
        b.pred_dt = dt;
        b.s1_state = 1;
        return true;
    }

    // Heun with the fused row pass: per field evaluation the y / z passes and
    // one k_row launch.  S1 carries the x transform of the predictor from one
    // step's last launch to the next step; H_d is never written (hd_stale).
    static bool heun_rows(Backend &b, double dt, fullmag_fdm_step_stats *st, bool readback) {
        // k1 and the predictor come from the row pass itself, so a run gives the
        // same bits whether it starts here or continues (checkpoint replays)
        if (!(b.k1_valid && b.pred_valid && b.pred_dt == dt) && !rows_k1(b, dt)) return false;
        DemagArgs<T> a = demag_args(b, b.mstage, nullptr);
        if (b.s1_state != 1 && !row_x_fwd(b, b.mstage)) return false;
        if (!mid_reg(b, a)) return false;
        // corrector at m_p: m <- normalize(m0 + (k1 + k2) dt/2), S1 = X(Ms m)
        StageArgs<T> s = stage_args(b, b.mstage, b.time + dt);
        s.kout = nullptr;
        s.m0 = (T *)b.m;
        s.k1 = (const T *)b.k[0];
        s.half_dt = 0.5 * dt;
        if (!row_pass(b, MODE_HEUN_CORR, s)) return false;
        b.s1_state = 0;
        b.pred_valid = false;
        if (!mid_reg(b, a)) return false;
        // RHS at the new state (the next k1), diagnostics, the next predictor
        StageArgs<T> e = stage_args(b, b.m, b.time + dt);
        e.kout = (T *)b.k[0];
        e.pred_out = (T *)b.mstage;
        e.pred_dt = dt;
        e.partials = b.partials;
        e.counter = b.counter;
        e.out = b.d_out;
        if (!row_pass(b, MODE_EVAL, e)) return false;
        b.s1_state = 1;
        b.pred_valid = true;
        b.pred_dt = dt;
        b.time += dt;
        b.step_count += 1;
        b.k1_valid = true;
        b.obs_valid = false;
        b.hd_stale = true;
        if (readback) {
            if (!read_stats(b)) return false;
            fill_stats(b, dt, st);
            st->suggested_next_dt = 0.0;
        }
        return true;
    }

    // One Heun step (lib.rs:1217-1249) with the cached k1.
    static bool heun(Backend &b, double dt, fullmag_fdm_step_stats *st, bool readback) {
        if (b.use_row) return heun_rows(b, dt, st, readback);
        if (!ensure_k1(b)) return false;
        // predictor m_p = normalize(m + k1 dt); the previous step's RHS kernel
        // already wrote it when this dt equals the previous one
        if (!(b.pred_valid && b.pred_dt == dt) && !combine(b, 0, b.m, {b.k[0]}, {dt}, dt, b.mstage)) return false;
        b.pred_valid = false;
        if (!demag(b, b.mstage, b.hd)) return false;
        // corrector at m_p: k2 and m <- normalize(m0 + (k1 + k2) dt/2)
        StageArgs<T> s = stage_args(b, b.mstage, b.time + dt);
        s.kout = nullptr;  // k2 is consumed in registers
        s.m0 = (T *)b.m;
        s.k1 = (const T *)b.k[0];
        s.half_dt = 0.5 * dt;
        {
            ProfScope p(b, "stage_heun_corr");
            launch_stage<MODE_HEUN_CORR>(b, s);
        }
        if (!check_launch(b, "heun corrector")) return false;
        // fields, RHS (next k1), the next predictor and diagnostics at the new state
        if (!demag(b, b.m, b.hd)) return false;
        if (!eval(b, b.m, b.time + dt, b.k[0], true, false, b.mstage, dt)) return false;
        b.pred_valid = true;
        b.pred_dt = dt;
        b.time += dt;
        b.step_count += 1;
        b.k1_valid = true;
        b.obs_valid = false;
        if (readback) {
            if (!read_stats(b)) return false;
            fill_stats(b, dt, st);
            st->suggested_next_dt = 0.0;
        }
        return true;
    }

    // One accepted DP45 step (lib.rs:1412-1568).
    static bool dp45(Backend &b, double dt_in, fullmag_fdm_step_stats *st) {
        b.pred_valid = false;  // the stages below use mstage
        const double A21 = 1.0 / 5.0;
        const double A31 = 3.0 / 40.0, A32 = 9.0 / 40.0;
        const double A41 = 44.0 / 45.0, A42 = -56.0 / 15.0, A43 = 32.0 / 9.0;
        const double A51 = 19372.0 / 6561.0, A52 = -25360.0 / 2187.0, A53 = 64448.0 / 6561.0,
                     A54 = -212.0 / 729.0;
        const double A61 = 9017.0 / 3168.0, A62 = -355.0 / 33.0, A63 = 46732.0 / 5247.0,
                     A64 = 49.0 / 176.0, A65 = -5103.0 / 18656.0;
        const double B1 = 35.0 / 384.0, B3 = 500.0 / 1113.0, B4 = 125.0 / 192.0,
                     B5 = -2187.0 / 6784.0, B6 = 11.0 / 84.0;
        // initial dt clamped like rk45_step_buf (lib.rs:1419): min(dt_max) then max(dt_min)
        double dt = std::max(std::min(dt_in, b.dt_max), b.dt_min);
        if (!ensure_k1(b)) return false;
        void **k = b.k;
        for (;;) {
            const double t = b.time;
            if (!combine(b, 0, b.m, {k[0]}, {A21 * dt}, dt, b.mstage)) return false;
            if (!demag(b, b.mstage, b.hd) || !eval(b, b.mstage, t + 0.2 * dt, k[1], false, false)) return false;
            if (!combine(b, 1, b.m, {k[0], k[1]}, {A31, A32}, dt, b.mstage)) return false;
            if (!demag(b, b.mstage, b.hd) || !eval(b, b.mstage, t + 0.3 * dt, k[2], false, false)) return false;
            if (!combine(b, 2, b.m, {k[0], k[1], k[2]}, {A41, A42, A43}, dt, b.mstage)) return false;
            if (!demag(b, b.mstage, b.hd) || !eval(b, b.mstage, t + 0.8 * dt, k[3], false, false)) return false;
            if (!combine(b, 3, b.m, {k[0], k[1], k[2], k[3]}, {A51, A52, A53, A54}, dt, b.mstage)) return false;
            if (!demag(b, b.mstage, b.hd) || !eval(b, b.mstage, t + 8.0 / 9.0 * dt, k[4], false, false)) return false;
            if (!combine(b, 4, b.m, {k[0], k[1], k[2], k[3], k[4]}, {A61, A62, A63, A64, A65}, dt, b.mstage)) return false;
            if (!demag(b, b.mstage, b.hd) || !eval(b, b.mstage, t + dt, k[5], false, false)) return false;
            // 5th-order solution and k7 = RHS(y5) with the embedded error norm
            if (!combine(b, 4, b.m, {k[0], k[2], k[3], k[4], k[5]}, {B1, B3, B4, B5, B6}, dt, b.mstage)) return false;
            if (!demag(b, b.mstage, b.hd)) return false;
            StageArgs<T> s = stage_args(b, b.mstage, t + dt);
            s.kout = (T *)k[6];
            s.partials = b.partials;
            s.counter = b.counter;
            s.out = b.d_out;
            // err = dt (E1 k1 + E3 k3 + E4 k4 + E5 k5 + E6 k6 + E7 k7), lib.rs:1653-1674
            s.ke[0] = (const T *)k[0]; s.ke[1] = (const T *)k[2]; s.ke[2] = (const T *)k[3];
            s.ke[3] = (const T *)k[4]; s.ke[4] = (const T *)k[5];
            s.nke = 5;
            s.ew[0] = 71.0 / 57600.0; s.ew[1] = -71.0 / 16695.0; s.ew[2] = 71.0 / 1920.0;
            s.ew[3] = -17253.0 / 339200.0; s.ew[4] = 22.0 / 525.0; s.ew[5] = -1.0 / 40.0;
            s.dt = dt;
            {
                ProfScope p(b, "stage_dp45_last");
                launch_stage<MODE_ERR_LAST>(b, s);
            }
            if (!check_launch(b, "dp45 last stage") || !read_stats(b)) return false;
            const double err = std::sqrt(b.h_out[Q_ERR2]);
            if (err <= b.max_error || dt <= b.dt_min) {
                std::swap(b.m, b.mstage);
                b.hd_stale = false;  // the last evaluation was at the accepted state
                std::swap(k[0], k[6]);  // FSAL: k7 is the next step's k1
                b.time += dt;
                b.step_count += 1;
                b.k1_valid = true;
                b.obs_valid = false;
                fill_stats(b, dt, st);
                st->suggested_next_dt = std::min(
                    std::max(b.headroom * dt * std::pow(b.max_error / std::max(err, 1e-30), 0.2), b.dt_min),
                    b.dt_max);
                return true;
            }
            const double dt_new = b.headroom * dt * std::pow(b.max_error / err, 0.2);
            dt = std::min(std::max(dt_new, b.dt_min), b.dt_max);
            // k[0] still equals RHS(m0, t): nothing to recompute for stage 1
        }
    }

    // Fields and RHS at the accepted state into k[0] (the next step's k1), with
    // the step diagnostics; advances the step counter.
    static bool finish_step(Backend &b, double dt, fullmag_fdm_step_stats *st, bool readback) {
        if (!demag(b, b.m, b.hd)) return false;
        if (!eval(b, b.m, b.time, b.k[0], true, false)) return false;
        b.step_count += 1;
        b.k1_valid = true;
        b.obs_valid = false;
        if (readback) {
            if (!read_stats(b)) return false;
            fill_stats(b, dt, st);
            st->suggested_next_dt = 0.0;
        }
        return true;
    }

    // One classical RK4 step (lib.rs:1253-1297) with the cached k1; stage
    // times t, t + dt/2, t + dt/2, t + dt.
    static bool rk4(Backend &b, double dt, fullmag_fdm_step_stats *st, bool readback) {
        b.pred_valid = false;  // the stages below use mstage
        if (!ensure_k1(b)) return false;
        void **k = b.k;
        const double t = b.time;
        if (!combine(b, 0, b.m, {k[0]}, {0.5 * dt}, dt, b.mstage)) return false;
        if (!demag(b, b.mstage, b.hd) || !eval(b, b.mstage, t + 0.5 * dt, k[1], false, false)) return false;
        if (!combine(b, 0, b.m, {k[1]}, {0.5 * dt}, dt, b.mstage)) return false;
        if (!demag(b, b.mstage, b.hd) || !eval(b, b.mstage, t + 0.5 * dt, k[2], false, false)) return false;
        if (!combine(b, 0, b.m, {k[2]}, {dt}, dt, b.mstage)) return false;
        if (!demag(b, b.mstage, b.hd) || !eval(b, b.mstage, t + dt, k[3], false, false)) return false;
        // m <- normalize(m0 + ((k1 + 2 k2) + (2 k3 + k4)) dt/6), in place
        if (!combine(b, 3, b.m, {k[0], k[1], k[2], k[3]}, {1.0, 2.0, 2.0, 1.0}, dt / 6.0, b.m)) return false;
        b.time += dt;
        return finish_step(b, dt, st, readback);
    }

    // One accepted Bogacki-Shampine 2(3) step (lib.rs:1332-1407).  The
    // reference evaluates k1 = RHS(m0) on every attempt; the cached k1 holds the
    // same values.  Stage times t, t + dt/2, t + 3dt/4, t + dt; k4 = RHS(y3) is
    // the next step's k1.
    static bool rk23(Backend &b, double dt_in, fullmag_fdm_step_stats *st) {
        b.pred_valid = false;  // the stages below use mstage
        double dt = std::max(std::min(dt_in, b.dt_max), b.dt_min);
        if (!ensure_k1(b)) return false;
        void **k = b.k;
        for (;;) {
            const double t = b.time;
            if (!combine(b, 0, b.m, {k[0]}, {0.5 * dt}, dt, b.mstage)) return false;
            if (!demag(b, b.mstage, b.hd) || !eval(b, b.mstage, t + 0.5 * dt, k[1], false, false)) return false;
            if (!combine(b, 0, b.m, {k[1]}, {0.75 * dt}, dt, b.mstage)) return false;
            if (!demag(b, b.mstage, b.hd) || !eval(b, b.mstage, t + 0.75 * dt, k[2], false, false)) return false;
            if (!combine(b, 2, b.m, {k[0], k[1], k[2]}, {2.0 / 9.0, 1.0 / 3.0, 4.0 / 9.0}, dt, b.mstage)) return false;
            if (!demag(b, b.mstage, b.hd)) return false;
            StageArgs<T> s = stage_args(b, b.mstage, t + dt);
            s.kout = (T *)k[3];
            s.partials = b.partials;
            s.counter = b.counter;
            s.out = b.d_out;
            s.ke[0] = (const T *)k[0]; s.ke[1] = (const T *)k[1]; s.ke[2] = (const T *)k[2];
            s.nke = 3;
            s.ew[0] = -5.0 / 72.0; s.ew[1] = 1.0 / 12.0; s.ew[2] = 1.0 / 9.0; s.ew[3] = -1.0 / 8.0;
            s.dt = dt;
            {
                ProfScope p(b, "stage_rk23_last");
                launch_stage<MODE_ERR_LAST>(b, s);
            }
            if (!check_launch(b, "rk23 last stage") || !read_stats(b)) return false;
            const double err = std::sqrt(b.h_out[Q_ERR2]);
            if (err <= b.max_error || dt <= b.dt_min) {
                std::swap(b.m, b.mstage);
                b.hd_stale = false;  // the last evaluation was at the accepted state
                std::swap(k[0], k[3]);
                b.time += dt;
                b.step_count += 1;
                b.k1_valid = true;
                b.obs_valid = false;
                fill_stats(b, dt, st);
                st->suggested_next_dt = std::min(
                    std::max(b.headroom * dt * std::pow(b.max_error / std::max(err, 1e-30), 1.0 / 3.0), b.dt_min),
                    b.dt_max);
                return true;
            }
            const double dt_new = b.headroom * dt * std::pow(b.max_error / err, 1.0 / 3.0);
            dt = std::min(std::max(dt_new, b.dt_min), b.dt_max);
        }
    }

    // ABM3 (lib.rs:1573-1648).  History f_n, f_{n-1}, f_{n-2} in k[2], k[3],
    // k[4] (pointer rotation), k[1] the slot the next entry is written to.
    // Three Heun start-up steps push RHS(m_{n+1}); then AB3 predictor,
    // f* = RHS(predicted) at t + dt, AM3 corrector, push f*.  A dt more than 10 %
    // away from the last one restarts the history before the step
    // (native/backends/fdm/src/llg_abm3_fp64.cu:177-180).  The history survives
    // magnetisation uploads, as in the reference.
    static void abm_push(Backend &b, double dt) {
        void **k = b.k;
        void *spare = k[4];
        k[4] = k[3];
        k[3] = k[2];
        k[2] = k[1];
        k[1] = spare;
        b.abm_startup = std::min(b.abm_startup + 1, 3);
        b.abm_last_dt = dt;
    }

    static bool abm3(Backend &b, double dt, fullmag_fdm_step_stats *st, bool readback) {
        if (b.abm_last_dt > 0.0 && std::fabs(dt - b.abm_last_dt) / b.abm_last_dt > 0.1) b.abm_startup = 0;
        void **k = b.k;
        if (b.abm_startup < 3) {
            if (b.abm_startup == 0) b.pred_valid = false;
            if (!heun(b, dt, st, readback)) return false;
            // heun() left RHS(m_{n+1}) in k[0]; the history keeps a copy
            if (!cuda_ok(b, cudaMemcpyAsync(k[1], k[0], (size_t)3 * b.n * sizeof(T), cudaMemcpyDeviceToDevice, b.stream),
                         "abm history"))
                return false;
            abm_push(b, dt);
            return true;
        }
        const double t = b.time;
        b.pred_valid = false;
        if (!combine(b, 2, b.m, {k[2], k[3], k[4]}, {23.0 / 12.0, -16.0 / 12.0, 5.0 / 12.0}, dt, b.mstage)) return false;
        if (!demag(b, b.mstage, b.hd) || !eval(b, b.mstage, t + dt, k[1], false, false)) return false;
        if (!combine(b, 2, b.m, {k[1], k[2], k[3]}, {5.0 / 12.0, 8.0 / 12.0, -1.0 / 12.0}, dt, b.m)) return false;
        b.time += dt;
        abm_push(b, dt);
        return finish_step(b, dt, st, readback);
    }

    // ------------------------------------------------------------------
    // Adjoint of a Heun trajectory (adjoint.cuh).  Device layout of adj_mem:
    // nck checkpoints and K segment states (3N T each), then the T work
    // buffers k1, k2, m_p, H1, hex1, H2, hex2, lambda_H, hadj, final (3N each), then
    // the FP64 buffers lambda, acc, gk, lloc, part, g_hext, g_hac (3N each) and
    // g_ms (N).
    // ------------------------------------------------------------------
    struct AdjPtrs {
        T *ck, *seg, *k1, *k2, *mp, *H1, *hex1, *H2, *hex2, *lh, *hadj, *fin;
        double *lam, *acc, *gk, *lloc, *part, *ghext, *ghac, *gms;
    };

    static size_t adj_need(const Backend &b, uint32_t nck, uint32_t K) {
        const size_t v = (size_t)3 * b.n;
        return (size_t)(nck + K + 10) * v * sizeof(T) + (7 * v + (size_t)b.n) * sizeof(double) + 1024;
    }

    static AdjPtrs adj_ptrs(Backend &b) {
        const size_t v = (size_t)3 * b.n;
        AdjPtrs p{};
        T *t = (T *)b.adj_mem;
        p.ck = t; t += (size_t)b.adj_nck * v;
        p.seg = t; t += (size_t)b.adj_K * v;
        T **tb[10] = {&p.k1, &p.k2, &p.mp, &p.H1, &p.hex1, &p.H2, &p.hex2, &p.lh, &p.hadj, &p.fin};
        for (T **q : tb) { *q = t; t += v; }
        uintptr_t al = ((uintptr_t)t + 255) & ~(uintptr_t)255;
        double *d = (double *)al;
        double **db[7] = {&p.lam, &p.acc, &p.gk, &p.lloc, &p.part, &p.ghext, &p.ghac};
        for (double **q : db) { *q = d; d += v; }
        p.gms = d;
        return p;
    }

    static AdjArgs adj_args(const Backend &b, double dt) {
        AdjArgs a{};
        a.n = b.n; a.nx = b.nx; a.ny = b.ny; a.nz = b.nz;
        a.dinv[0] = 1.0 / (b.dx * b.dx); a.dinv[1] = 1.0 / (b.dy * b.dy); a.dinv[2] = 1.0 / (b.dz * b.dz);
        a.aex = b.enable_exchange ? b.aex : 0.0;
        a.ms = b.ms;
        a.gamma_bar = b.gamma / (1.0 + b.alpha * b.alpha);
        a.alpha = b.alpha;
        a.pr = b.precession ? 1.0 : 0.0;
        a.ms_map = b.d_msmap;
        a.mask = b.d_mask;
        a.dt = dt;
        return a;
    }

    // Run n Heun steps from the current state, keeping every K-th state.
    static bool adjoint_forward(Backend &b, double dt, uint32_t n, uint32_t K, fullmag_fdm_step_stats *st) {
        if (K == 0) K = (uint32_t)std::ceil(std::sqrt((double)n));
        K = std::max<uint32_t>(1, std::min(K, n));
        const uint32_t nck = (n + K - 1) / K;
        const size_t need = adj_need(b, nck, K);
        if (need > b.adj_bytes) {
            if (b.adj_mem) cudaFree(b.adj_mem);
            b.adj_mem = nullptr;
            b.adj_bytes = 0;
            if (!cuda_ok(b, cudaMalloc(&b.adj_mem, need), "cudaMalloc(adjoint)")) return false;
            b.adj_bytes = need;
        }
        b.adj_n = n; b.adj_K = K; b.adj_nck = nck; b.adj_dt = dt;
        b.adj_ck_time.assign(nck, 0.0);
        b.adj_ck_step.assign(nck, 0);
        b.adj_ready = false;
        AdjPtrs p = adj_ptrs(b);
        const size_t vb = (size_t)3 * b.n * sizeof(T);
        for (uint32_t s = 0; s < n; ++s) {
            if (s % K == 0) {
                const uint32_t c = s / K;
                if (!cuda_ok(b, cudaMemcpyAsync(p.ck + (size_t)c * 3 * b.n, b.m, vb, cudaMemcpyDeviceToDevice, b.stream), "checkpoint"))
                    return false;
                b.adj_ck_time[c] = b.time;
                b.adj_ck_step[c] = b.step_count;
            }
            if (!heun(b, dt, st, s + 1 == n)) return false;
        }
        b.adj_t_final = b.time;
        b.adj_step_final = b.step_count;
        b.adj_ready = true;
        return true;
    }

    // One step's pull-back from lam (cotangent of m_{n+1}) to lam (of m_n).
    static bool adjoint_step(Backend &b, AdjPtrs &p, const T *mn, double tn, double dt) {
        const AdjArgs a = adj_args(b, dt);
        const unsigned g = grid_cells(b);
        const double omega = 2.0 * kPi * b.ac_freq;
        // forward quantities of the step
        if (!demag(b, mn, b.hd) || !eval_fields(b, mn, tn, p.k1, p.hex1, p.H1)) return false;
        if (!combine(b, 0, mn, {(void *)p.k1}, {dt}, dt, p.mp)) return false;
        const double t2 = tn + dt;
        if (!demag(b, p.mp, b.hd) || !eval_fields(b, p.mp, t2, p.k2, p.hex2, p.H2)) return false;
        // corrector normalisation, then stage 2 (at m_p, t + dt)
        k_adj_start<T><<<g, 256, 0, b.stream>>>(a, mn, p.k1, p.k2, p.lam, p.acc, p.gk);
        k_adj_vjp<T><<<g, 256, 0, b.stream>>>(a, p.mp, p.H2, p.gk, p.lh, p.lloc);
        if (!demag(b, p.lh, p.hadj, true)) return false;
        k_adj_apply<T><<<g, 256, 0, b.stream>>>(a, p.mp, p.lh, p.hadj, p.hex2, p.lloc, p.part, p.gms,
                                                p.ghext, p.ghac, omega != 0.0 ? std::sin(t2 * omega) : 0.0);
        // predictor normalisation, then stage 1 (at m_n, t)
        k_adj_pred<T><<<g, 256, 0, b.stream>>>(a, mn, p.k1, p.part, p.acc, p.gk);
        k_adj_vjp<T><<<g, 256, 0, b.stream>>>(a, mn, p.H1, p.gk, p.lh, p.lloc);
        if (!demag(b, p.lh, p.hadj, true)) return false;
        k_adj_apply<T><<<g, 256, 0, b.stream>>>(a, mn, p.lh, p.hadj, p.hex1, p.lloc, p.part, p.gms,
                                                p.ghext, p.ghac, omega != 0.0 ? std::sin(tn * omega) : 0.0);
        k_adj_finish<<<g, 256, 0, b.stream>>>(3LL * b.n, p.acc, p.part, p.lam);
        return check_launch(b, "adjoint step");
    }

    // Pull dL/dm(final) back through the recorded trajectory.  The seed and the
    // outputs are host FP64 buffers: lam (SoA 3N), dL/dMs per cell (N), the
    // per-cell dL/dH_ext and dL/dH_ac (SoA 3N, summed by the caller), dL/dm0 (SoA 3N).
    static bool adjoint_backward(Backend &b, const double *lam_soa_host, double *gms_host,
                                 double *ghext_host, double *ghac_host, double *lam0_host) {
        AdjPtrs p = adj_ptrs(b);
        const size_t v = (size_t)3 * b.n;
        const size_t vb = v * sizeof(T);
        if (!cuda_ok(b, cudaMemcpyAsync(p.lam, lam_soa_host, v * 8, cudaMemcpyHostToDevice, b.stream), "adjoint seed") ||
            !cuda_ok(b, cudaMemsetAsync(p.ghext, 0, v * 8, b.stream), "adjoint zero") ||
            !cuda_ok(b, cudaMemsetAsync(p.ghac, 0, v * 8, b.stream), "adjoint zero") ||
            !cuda_ok(b, cudaMemsetAsync(p.gms, 0, (size_t)b.n * 8, b.stream), "adjoint zero"))
            return false;
        // the final state is kept aside while the segments are replayed
        bool ok = cuda_ok(b, cudaMemcpyAsync(p.fin, b.m, vb, cudaMemcpyDeviceToDevice, b.stream), "save final");
        std::vector<double> seg_time(b.adj_K);
        fullmag_fdm_step_stats st{};
        for (int c = (int)b.adj_nck - 1; ok && c >= 0; --c) {
            const uint32_t s0 = (uint32_t)c * b.adj_K;
            const uint32_t len = std::min(b.adj_K, b.adj_n - s0);
            ok = cuda_ok(b, cudaMemcpyAsync(b.m, p.ck + (size_t)c * v, vb, cudaMemcpyDeviceToDevice, b.stream), "restore checkpoint");
            b.time = b.adj_ck_time[c];
            b.step_count = b.adj_ck_step[c];
            b.k1_valid = false;
            b.pred_valid = false;
            for (uint32_t j = 0; ok && j < len; ++j) {
                ok = cuda_ok(b, cudaMemcpyAsync(p.seg + (size_t)j * v, b.m, vb, cudaMemcpyDeviceToDevice, b.stream), "segment");
                seg_time[j] = b.time;
                if (ok && j + 1 < len) ok = heun(b, b.adj_dt, &st, false);
            }
            for (int j = (int)len - 1; ok && j >= 0; --j)
                ok = adjoint_step(b, p, p.seg + (size_t)j * v, seg_time[j], b.adj_dt);
        }
        // restore the final state
        if (ok) ok = cuda_ok(b, cudaMemcpyAsync(b.m, p.fin, vb, cudaMemcpyDeviceToDevice, b.stream), "restore final");
        b.time = b.adj_t_final;
        b.step_count = b.adj_step_final;
        b.k1_valid = false;
        b.pred_valid = false;
        b.obs_valid = false;
        if (!ok) return false;
        if (gms_host && !cuda_ok(b, cudaMemcpyAsync(gms_host, p.gms, (size_t)b.n * 8, cudaMemcpyDeviceToHost, b.stream), "dL/dMs")) return false;
        if (ghext_host && !cuda_ok(b, cudaMemcpyAsync(ghext_host, p.ghext, v * 8, cudaMemcpyDeviceToHost, b.stream), "dL/dH_ext")) return false;
        if (ghac_host && !cuda_ok(b, cudaMemcpyAsync(ghac_host, p.ghac, v * 8, cudaMemcpyDeviceToHost, b.stream), "dL/dH_ac")) return false;
        if (lam0_host && !cuda_ok(b, cudaMemcpyAsync(lam0_host, p.lam, v * 8, cudaMemcpyDeviceToHost, b.stream), "dL/dm0")) return false;
        return cuda_ok(b, cudaStreamSynchronize(b.stream), "adjoint sync");
    }

    // With the fused row pass k1 is left to the next step, which computes it
    // with the row pass's own arithmetic.
    static bool refresh(Backend &b) {
        if (!demag(b, b.m, b.hd)) return false;
        if (!eval(b, b.m, b.time, b.use_row ? nullptr : b.k[0], false, true)) return false;
        b.k1_valid = !b.use_row;
        b.obs_valid = true;
        return cuda_ok(b, cudaStreamSynchronize(b.stream), "refresh");
    }

    // H_d(m) into hd when the fused Heun steps left it stale.
    static bool ensure_hd(Backend &b) {
        return !b.hd_stale || demag(b, b.m, b.hd);
    }

    static bool ensure_obs(Backend &b) {
        if (b.obs_valid) return true;
        if (!ensure_hd(b)) return false;
        // H_ex / H_eff (and k1, unchanged; the row pass keeps its own k1)
        if (!eval(b, b.m, b.time, b.use_row ? nullptr : b.k[0], false, true)) return false;
        b.obs_valid = true;
        return true;
    }
};

// ---------------------------------------------------------------------------
// AoS <-> SoA conversion kernels
// ---------------------------------------------------------------------------
template <typename TI, typename TO>
__global__ void k_aos_to_soa(const TI *in, TO *out, long long n, const uint8_t *mask,
                             const double *ms_map) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        bool act = (!mask || mask[i] != 0) && (!ms_map || ms_map[i] > 0.0);
        out[i] = act ? (TO)in[3 * i] : TO(0);
        out[n + i] = act ? (TO)in[3 * i + 1] : TO(0);
        out[2 * n + i] = act ? (TO)in[3 * i + 2] : TO(0);
    }
}

template <typename TI, typename TO>
__global__ void k_soa_to_aos(const TI *in, TO *out, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        out[3 * i] = (TO)in[i];
        out[3 * i + 1] = (TO)in[n + i];
        out[3 * i + 2] = (TO)in[2 * n + i];
    }
}

// Box average of the preview bins, same binning as the reference
// (native/backends/fdm/src/context.cu:222-286).
template <typename TI, typename TO>
__global__ void k_preview(const TI *f, long long n, int fx, int fy, int fz, int px, int py,
                          int pz, int z_origin, int z_stride, TO *out) {
    const long long count = (long long)px * py * pz;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < count;
         p += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(p % px), iy = (int)((p / px) % py), iz = (int)(p / ((long long)px * py));
        int x0 = (int)(((long long)ix * fx) / px), x1 = (int)(((long long)(ix + 1) * fx) / px);
        if (x1 <= x0) x1 = x0 + 1;
        if (x1 > fx) x1 = fx;
        int y0 = (int)(((long long)iy * fy) / py), y1 = (int)(((long long)(iy + 1) * fy) / py);
        if (y1 <= y0) y1 = y0 + 1;
        if (y1 > fy) y1 = fy;
        long long zs = (long long)z_origin + (long long)iz * z_stride;
        if (zs >= fz) zs = fz - 1;
        long long ze = (long long)z_origin + (long long)(iz + 1) * z_stride;
        if (ze <= zs) ze = zs + 1;
        if (ze > fz) ze = fz;
        double ax = 0, ay = 0, az = 0, cnt = 0;
        for (long long z = zs; z < ze; ++z)
            for (int y = y0; y < y1; ++y)
                for (int x = x0; x < x1; ++x) {
                    const long long i = (z * fy + y) * fx + x;
                    ax += (double)f[i];
                    ay += (double)f[n + i];
                    az += (double)f[2 * n + i];
                    cnt += 1.0;
                }
        out[3 * p] = (TO)(ax / cnt);
        out[3 * p + 1] = (TO)(ay / cnt);
        out[3 * p + 2] = (TO)(az / cnt);
    }
}

// ---------------------------------------------------------------------------
// public (C++) entry points used by api.cu
// ---------------------------------------------------------------------------
static unsigned cgrid(long long n) {
    return (unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * 16));
}

bool backend_alloc(Backend &b) {
    const bool dbl = b.precision == FULLMAG_FDM_PRECISION_DOUBLE;
    b.scalar = dbl ? 8 : 4;
    const size_t cs = 2 * b.scalar;  // complex
    const size_t vec = (size_t)3 * b.n * b.scalar;
    // layout sizes
    struct Item { void **p; size_t bytes; };
    std::vector<Item> items;
    // k buffers: DP45 k1..k7; RK4 and RK23 k1..k4; ABM3 k1, the next history
    // slot and f_n, f_{n-1}, f_{n-2}; Heun k1 (k2 stays in registers) + 1
    const int nk = b.integrator == FULLMAG_FDM_INTEGRATOR_DP45   ? 7
                   : b.integrator == FULLMAG_FDM_INTEGRATOR_ABM3 ? 5
                   : (b.integrator == FULLMAG_FDM_INTEGRATOR_RK4 || b.integrator == FULLMAG_FDM_INTEGRATOR_RK23) ? 4
                                                                   : 2;
    items.push_back({&b.m, vec});
    items.push_back({&b.mstage, vec});
    items.push_back({&b.hd, vec});
    items.push_back({&b.hex, vec});
    items.push_back({&b.heff, vec});
    for (int i = 0; i < nk; ++i) items.push_back({&b.k[i], vec});
    if (b.enable_demag) {
        items.push_back({&b.twx, (size_t)b.Lx * cs});
        items.push_back({&b.twy, (size_t)b.Ly * cs});
        items.push_back({&b.twxT, (size_t)b.Lx * cs});
        items.push_back({&b.twyT, (size_t)b.Ly * cs});
        items.push_back({&b.twz, (size_t)b.Lz * cs});
        items.push_back({&b.s1, (size_t)3 * b.nz * b.nkx * b.ny * cs});
        if (!b.thin) items.push_back({&b.s2, (size_t)3 * b.nz * b.nkx * b.Ly * cs});
        items.push_back({&b.spec, (size_t)6 * b.KZ * b.nkx * b.KY * b.scalar});
    }
    items.push_back({&b.staging, (size_t)3 * b.n * sizeof(double)});
    if (b.has_mask) items.push_back({(void **)&b.d_mask, (size_t)b.n});
    if (b.has_regions) {
        items.push_back({(void **)&b.d_region, (size_t)b.n * 4});
        items.push_back({(void **)&b.d_lut, (size_t)256 * 256 * 8});
    }
    if (b.has_ms_map) items.push_back({(void **)&b.d_msmap, (size_t)b.n * 8});
    if (b.boundary_tier) {
        items.push_back({(void **)&b.d_vf, b.vf_host.size() * 8});
        if (!b.face_host.empty()) items.push_back({(void **)&b.d_face, b.face_host.size() * 8});
        if (!b.delta_host.empty()) items.push_back({(void **)&b.d_delta, b.delta_host.size() * 8});
        if (b.corr_targets) {
            items.push_back({(void **)&b.d_corr_tgt, b.corr_tgt_host.size() * 4});
            items.push_back({(void **)&b.d_corr_src, b.corr_src_host.size() * 4});
            items.push_back({(void **)&b.d_corr_ten, b.corr_ten_host.size() * 8});
        }
    }
    // stage kernels: the z-marching kernel serves a uniform material whose
    // 3 n fits 32-bit indices; its planes per thread (zb) are halved until the
    // grid has about 8 blocks per SM
    b.stage_plain = !b.has_mask && !b.has_ms_map && !b.has_regions && !b.boundary_tier &&
                    3ULL * (unsigned long long)b.n < (1ULL << 32);
    {
        auto blocks = [&](int zb) {
            return (long long)((b.nx + 31) / 32) * ((b.ny + kStagePlainBY - 1) / kStagePlainBY) * ((b.nz + zb - 1) / zb);
        };
        int zb = std::max(1, b.nz);
        while (zb > 1 && blocks(zb) < 148LL * 8) zb = (zb + 1) / 2;
        b.stage_zb = zb;
        const long long general = (long long)((b.nx + 31) / 32) * ((b.ny + 3) / 4) * ((b.nz + 1) / 2);
        const long long rows = (long long)((b.ny + 1) / 2) * b.nz;  // the row pass with 2-row slabs
        const dim3 gv = stage_vec_grid(b, (int)b.scalar, false);      // 16-byte-group stage kernels (largest grid)
        const long long vgrid = (long long)gv.x * gv.y * gv.z;
        b.red_blocks = (int)std::max(std::max(general, blocks(zb)), std::max(rows, vgrid));  // partials of any stage grid
    }
    items.push_back({(void **)&b.partials, (size_t)NQ * b.red_blocks * 8});
    items.push_back({(void **)&b.counter, 64});
    size_t total = 0;
    for (auto &it : items) total += (it.bytes + 255) / 256 * 256;
    if (!cuda_ok(b, cudaMalloc(&b.arena, total), "cudaMalloc(arena)")) return false;
    b.arena_bytes = total;
    char *p = (char *)b.arena;
    for (auto &it : items) {
        *it.p = p;
        p += (it.bytes + 255) / 256 * 256;
    }
    if (!cuda_ok(b, cudaMemsetAsync(b.arena, 0, total, b.stream), "arena memset")) return false;
    // step statistics: the last block of a reducing kernel writes them straight
    // into this mapped pinned buffer, so a step ends with a stream sync, no copy
    if (!cuda_ok(b, cudaHostAlloc((void **)&b.h_out, NQ * sizeof(double) + 64, cudaHostAllocMapped), "cudaHostAlloc(stats)"))
        return false;
    if (!cuda_ok(b, cudaHostGetDevicePointer((void **)&b.d_out, b.h_out, 0), "stats device pointer")) return false;
    return true;
}

template <typename T>
static bool upload_tables(Backend &b, const std::vector<double> (&spec)[6]) {
    auto tw = [&](int L, void *dst) {
        std::vector<cx<T>> t(L);
        for (int k = 0; k < L; ++k) {
            const double a = 2.0 * kPi * (double)k / (double)L;
            t[k] = mk<T>((T)std::cos(a), (T)(-std::sin(a)));
        }
        return cuda_ok(b, cudaMemcpy(dst, t.data(), L * sizeof(cx<T>), cudaMemcpyHostToDevice), "twiddles");
    };
    if (!tw(b.Lx, b.twx) || !tw(b.Ly, b.twy) || !tw(b.Lz, b.twz)) return false;
    auto tw4 = [&](int L, void *dst) {
        if (L < 2 || (L & (L - 1))) return true;  // register FFT only (powers of two)
        const std::vector<cx<T>> t = host_tw4<T>(L);
        return cuda_ok(b, cudaMemcpy(dst, t.data(), L * sizeof(cx<T>), cudaMemcpyHostToDevice), "twiddles (4-step)");
    };
    if (!tw4(b.Lx, b.twxT) || !tw4(b.Ly, b.twyT)) return false;
    // the octant, or for the direct z convolution its z-inverse table (nz planes)
    std::vector<double> zt[6];
    if (b.zdirect) octant_to_z_direct(b.nkx, b.KY, b.nz, spec, zt);
    const auto &src = b.zdirect ? zt : spec;
    const size_t plane = (size_t)(b.zdirect ? b.nz : b.KZ) * b.nkx * b.KY;
    std::vector<T> host;
    if (b.use_zdw && b.zdw_win) {
        // rows of zdw_kyp values (16-byte windows of k_zdw), the padding zero
        const size_t kyp = (size_t)b.zdw_kyp, rows = (size_t)b.nz * b.nkx;
        host.assign(6 * rows * kyp, T(0));
        for (int c = 0; c < 6; ++c)
            for (size_t r = 0; r < rows; ++r)
                for (int ky = 0; ky < b.KY; ++ky) host[(c * rows + r) * kyp + ky] = (T)src[c][r * b.KY + ky];
    } else {
        host.resize(6 * plane);
        for (int c = 0; c < 6; ++c)
            for (size_t o = 0; o < plane; ++o) host[c * plane + o] = (T)src[c][o];
    }
    return cuda_ok(b, cudaMemcpy(b.spec, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice), "spectra upload");
}

bool backend_upload_tables(Backend &b, const std::vector<double> (&spec)[6]) {
    if (!b.enable_demag) return true;
    return b.precision == FULLMAG_FDM_PRECISION_DOUBLE ? upload_tables<double>(b, spec)
                                                       : upload_tables<float>(b, spec);
}

bool backend_configure(Backend &b) {
    const bool dbl = b.precision == FULLMAG_FDM_PRECISION_DOUBLE;
    if (!(dbl ? Impl<double>::configure_stage(b) : Impl<float>::configure_stage(b))) return false;
    if (!b.enable_demag) return true;
    return b.precision == FULLMAG_FDM_PRECISION_DOUBLE ? Impl<double>::configure(b)
                                                       : Impl<float>::configure(b);
}

template <typename TI>
static bool upload_m_impl(Backend &b, const TI *host, uint64_t len) {
    if (!cuda_ok(b, cudaMemcpyAsync(b.staging, host, len * sizeof(TI), cudaMemcpyHostToDevice, b.stream), "upload m"))
        return false;
    if (b.precision == FULLMAG_FDM_PRECISION_DOUBLE)
        k_aos_to_soa<TI, double><<<cgrid(b.n), 256, 0, b.stream>>>((const TI *)b.staging, (double *)b.m, b.n, b.d_mask, b.d_msmap);
    else
        k_aos_to_soa<TI, float><<<cgrid(b.n), 256, 0, b.stream>>>((const TI *)b.staging, (float *)b.m, b.n, b.d_mask, b.d_msmap);
    if (!check_launch(b, "aos_to_soa")) return false;
    b.k1_valid = false;
    b.pred_valid = false;
    b.obs_valid = false;
    b.s1_state = 0;
    return cuda_ok(b, cudaStreamSynchronize(b.stream), "upload sync");
}

bool backend_upload_m_f64(Backend &b, const double *m, uint64_t len) { return upload_m_impl<double>(b, m, len); }
bool backend_upload_m_f32(Backend &b, const float *m, uint64_t len) { return upload_m_impl<float>(b, m, len); }

bool backend_refresh(Backend &b) {
    return b.precision == FULLMAG_FDM_PRECISION_DOUBLE ? Impl<double>::refresh(b) : Impl<float>::refresh(b);
}

// One step of the plan's integrator; `last` asks for the stats readback (the
// adaptive integrators always read back: their error decides acceptance).
template <typename T>
static bool step_once(Backend &b, double dt, fullmag_fdm_step_stats *st, bool last) {
    switch (b.integrator) {
        case FULLMAG_FDM_INTEGRATOR_DP45: return Impl<T>::dp45(b, dt, st);
        case FULLMAG_FDM_INTEGRATOR_RK23: return Impl<T>::rk23(b, dt, st);
        case FULLMAG_FDM_INTEGRATOR_RK4: return Impl<T>::rk4(b, dt, st, last);
        case FULLMAG_FDM_INTEGRATOR_ABM3: return Impl<T>::abm3(b, dt, st, last);
        default: return Impl<T>::heun(b, dt, st, last);
    }
}

static bool adaptive(const Backend &b) {
    return b.integrator == FULLMAG_FDM_INTEGRATOR_DP45 || b.integrator == FULLMAG_FDM_INTEGRATOR_RK23;
}

bool backend_step(Backend &b, double dt, fullmag_fdm_step_stats *st) {
    const bool ok = b.precision == FULLMAG_FDM_PRECISION_DOUBLE ? step_once<double>(b, dt, st, true)
                                                                : step_once<float>(b, dt, st, true);
    if (b.profiling) prof_collect(b);
    return ok;
}

bool backend_step_n(Backend &b, double dt, uint32_t nsteps, fullmag_fdm_step_stats *st) {
    bool ok = true;
    for (uint32_t i = 0; i < nsteps && ok; ++i) {
        const bool last = (i + 1 == nsteps);
        ok = b.precision == FULLMAG_FDM_PRECISION_DOUBLE ? step_once<double>(b, dt, st, last)
                                                         : step_once<float>(b, dt, st, last);
        if (ok && adaptive(b)) dt = st->suggested_next_dt;
    }
    if (b.profiling) prof_collect(b);
    return ok;
}

bool backend_adjoint_forward(Backend &b, double dt, uint32_t n, uint32_t K, fullmag_fdm_step_stats *st) {
    const bool ok = b.precision == FULLMAG_FDM_PRECISION_DOUBLE ? Impl<double>::adjoint_forward(b, dt, n, K, st)
                                                                : Impl<float>::adjoint_forward(b, dt, n, K, st);
    if (b.profiling) prof_collect(b);
    return ok;
}

bool backend_adjoint_backward(Backend &b, const double *lam_soa, double *gms, double *ghext, double *ghac,
                              double *lam0_soa) {
    const bool ok = b.precision == FULLMAG_FDM_PRECISION_DOUBLE
                        ? Impl<double>::adjoint_backward(b, lam_soa, gms, ghext, ghac, lam0_soa)
                        : Impl<float>::adjoint_backward(b, lam_soa, gms, ghext, ghac, lam0_soa);
    if (b.profiling) prof_collect(b);
    return ok;
}

// Field pointer for an observable (after making H_ex / H_eff current).
static const void *observable_ptr(Backend &b, fullmag_fdm_observable obs, bool &ok) {
    ok = true;
    switch (obs) {
        case FULLMAG_FDM_OBSERVABLE_M: return b.m;
        case FULLMAG_FDM_OBSERVABLE_H_DEMAG:
            ok = b.precision == FULLMAG_FDM_PRECISION_DOUBLE ? Impl<double>::ensure_hd(b) : Impl<float>::ensure_hd(b);
            return b.hd;
        case FULLMAG_FDM_OBSERVABLE_H_EX:
        case FULLMAG_FDM_OBSERVABLE_H_EFF:
            ok = b.precision == FULLMAG_FDM_PRECISION_DOUBLE ? Impl<double>::ensure_obs(b) : Impl<float>::ensure_obs(b);
            return obs == FULLMAG_FDM_OBSERVABLE_H_EX ? b.hex : b.heff;
        default: ok = false; return nullptr;
    }
}

// Host-side H_ext value of cell i (synthesised like context.cu:802-815).
static void hext_cell(const Backend &b, long long i, double out[3]) {
    const bool act = (!b.has_mask || b.mask_host[i] != 0) && (!b.has_ms_map || b.ms_map_host[i] > 0.0);
    const double s = (b.ac_freq != 0.0) ? std::sin(2.0 * kPi * b.ac_freq * b.time) : 0.0;
    for (int c = 0; c < 3; ++c) out[c] = (b.has_ext && act) ? b.hext[c] + b.hac[c] * s : 0.0;
}

template <typename TO>
static bool download_impl(Backend &b, fullmag_fdm_observable obs, TO *out, uint64_t len) {
    if (obs == FULLMAG_FDM_OBSERVABLE_H_EXT) {
        for (long long i = 0; i < b.n; ++i) {
            double h[3];
            hext_cell(b, i, h);
            out[3 * i] = (TO)h[0]; out[3 * i + 1] = (TO)h[1]; out[3 * i + 2] = (TO)h[2];
        }
        return true;
    }
    bool ok;
    const void *src = observable_ptr(b, obs, ok);
    if (!ok) {
        if (b.last_error.empty()) b.last_error = "unsupported observable";
        return false;
    }
    if (b.precision == FULLMAG_FDM_PRECISION_DOUBLE)
        k_soa_to_aos<double, TO><<<cgrid(b.n), 256, 0, b.stream>>>((const double *)src, (TO *)b.staging, b.n);
    else
        k_soa_to_aos<float, TO><<<cgrid(b.n), 256, 0, b.stream>>>((const float *)src, (TO *)b.staging, b.n);
    if (!check_launch(b, "soa_to_aos")) return false;
    if (!cuda_ok(b, cudaMemcpyAsync(out, b.staging, len * sizeof(TO), cudaMemcpyDeviceToHost, b.stream), "field D2H"))
        return false;
    return cuda_ok(b, cudaStreamSynchronize(b.stream), "field sync");
}

bool backend_download_f64(Backend &b, fullmag_fdm_observable o, double *out, uint64_t len) { return download_impl<double>(b, o, out, len); }
bool backend_download_f32(Backend &b, fullmag_fdm_observable o, float *out, uint64_t len) { return download_impl<float>(b, o, out, len); }

template <typename TO>
static bool preview_impl(Backend &b, fullmag_fdm_observable obs, uint32_t pnx, uint32_t pny,
                         uint32_t pnz, uint32_t z_origin, uint32_t z_stride, TO *out, uint64_t len) {
    if (z_origin >= (uint32_t)b.nz) { b.last_error = "preview z_origin out of range"; return false; }
    if ((int)pnx == b.nx && (int)pny == b.ny && (int)pnz == b.nz && z_origin == 0 && z_stride == 1)
        return download_impl<TO>(b, obs, out, len);
    const long long count = (long long)pnx * pny * pnz;
    if (obs == FULLMAG_FDM_OBSERVABLE_H_EXT) {
        // fraction of active cells in the bin times H_ext (context.cu:941-1000)
        for (long long p = 0; p < count; ++p) {
            const int ix = (int)(p % pnx), iy = (int)((p / pnx) % pny), iz = (int)(p / ((long long)pnx * pny));
            int x0 = (int)(((long long)ix * b.nx) / pnx), x1 = (int)(((long long)(ix + 1) * b.nx) / pnx);
            if (x1 <= x0) x1 = x0 + 1;
            if (x1 > b.nx) x1 = b.nx;
            int y0 = (int)(((long long)iy * b.ny) / pny), y1 = (int)(((long long)(iy + 1) * b.ny) / pny);
            if (y1 <= y0) y1 = y0 + 1;
            if (y1 > b.ny) y1 = b.ny;
            long long zs = (long long)z_origin + (long long)iz * z_stride;
            if (zs >= b.nz) zs = b.nz - 1;
            long long ze = (long long)z_origin + (long long)(iz + 1) * z_stride;
            if (ze <= zs) ze = zs + 1;
            if (ze > b.nz) ze = b.nz;
            double act = 0, cnt = 0;
            for (long long z = zs; z < ze; ++z)
                for (int y = y0; y < y1; ++y)
                    for (int x = x0; x < x1; ++x) {
                        const long long i = (z * b.ny + y) * b.nx + x;
                        act += ((!b.has_mask || b.mask_host[i]) && (!b.has_ms_map || b.ms_map_host[i] > 0)) ? 1.0 : 0.0;
                        cnt += 1.0;
                    }
            const double sc = (b.has_ext && cnt > 0) ? act / cnt : 0.0;
            const double s = (b.ac_freq != 0.0) ? std::sin(2.0 * kPi * b.ac_freq * b.time) : 0.0;
            for (int c = 0; c < 3; ++c) out[3 * p + c] = (TO)((b.hext[c] + b.hac[c] * s) * sc);
        }
        return true;
    }
    bool ok;
    const void *src = observable_ptr(b, obs, ok);
    if (!ok) {
        if (b.last_error.empty()) b.last_error = "unsupported observable";
        return false;
    }
    if ((uint64_t)count * 3 * sizeof(TO) > (uint64_t)3 * b.n * sizeof(double)) {
        b.last_error = "preview larger than the field";
        return false;
    }
    if (b.precision == FULLMAG_FDM_PRECISION_DOUBLE)
        k_preview<double, TO><<<cgrid(count), 256, 0, b.stream>>>((const double *)src, b.n, b.nx, b.ny, b.nz, pnx, pny, pnz, z_origin, z_stride, (TO *)b.staging);
    else
        k_preview<float, TO><<<cgrid(count), 256, 0, b.stream>>>((const float *)src, b.n, b.nx, b.ny, b.nz, pnx, pny, pnz, z_origin, z_stride, (TO *)b.staging);
    if (!check_launch(b, "preview")) return false;
    if (!cuda_ok(b, cudaMemcpyAsync(out, b.staging, count * 3 * sizeof(TO), cudaMemcpyDeviceToHost, b.stream), "preview D2H"))
        return false;
    return cuda_ok(b, cudaStreamSynchronize(b.stream), "preview sync");
}

bool backend_preview_f64(Backend &b, fullmag_fdm_observable o, uint32_t a, uint32_t c, uint32_t d, uint32_t zo, uint32_t zs, double *out, uint64_t len) {
    return preview_impl<double>(b, o, a, c, d, zo, zs, out, len);
}
bool backend_preview_f32(Backend &b, fullmag_fdm_observable o, uint32_t a, uint32_t c, uint32_t d, uint32_t zo, uint32_t zs, float *out, uint64_t len) {
    return preview_impl<float>(b, o, a, c, d, zo, zs, out, len);
}

// Snapshot: D2D copy on the compute stream, D2H on its own stream into pinned memory.
bool backend_snapshot_begin(Backend &b, fullmag_fdm_observable obs, Snapshot &s) {
    s.scalar = b.scalar;
    s.cell_count = (uint64_t)b.n;
    s.bytes = (size_t)3 * b.n * b.scalar;
    if (!cuda_ok(b, cudaMallocHost(&s.host, s.bytes), "cudaMallocHost(snapshot)")) return false;
    if (obs == FULLMAG_FDM_OBSERVABLE_H_EXT) {
        for (long long i = 0; i < b.n; ++i) {
            double h[3];
            hext_cell(b, i, h);
            for (int c = 0; c < 3; ++c) {
                if (b.scalar == 8) ((double *)s.host)[c * b.n + i] = h[c];
                else ((float *)s.host)[c * b.n + i] = (float)h[c];
            }
        }
        s.pending = false;
        return true;
    }
    bool ok;
    const void *src = observable_ptr(b, obs, ok);
    if (!ok) {
        if (b.last_error.empty()) b.last_error = "unsupported async snapshot observable";
        return false;
    }
    if (!cuda_ok(b, cudaMalloc(&s.dev, s.bytes), "cudaMalloc(snapshot)")) return false;
    if (!cuda_ok(b, cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking), "snapshot stream")) return false;
    if (!cuda_ok(b, cudaEventCreateWithFlags(&s.ready, cudaEventDisableTiming), "snapshot event")) return false;
    if (!cuda_ok(b, cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming), "snapshot event")) return false;
    if (!cuda_ok(b, cudaMemcpyAsync(s.dev, src, s.bytes, cudaMemcpyDeviceToDevice, b.stream), "snapshot D2D")) return false;
    if (!cuda_ok(b, cudaEventRecord(s.ready, b.stream), "snapshot record")) return false;
    if (!cuda_ok(b, cudaStreamWaitEvent(s.stream, s.ready, 0), "snapshot wait")) return false;
    if (!cuda_ok(b, cudaMemcpyAsync(s.host, s.dev, s.bytes, cudaMemcpyDeviceToHost, s.stream), "snapshot D2H")) return false;
    if (!cuda_ok(b, cudaEventRecord(s.done, s.stream), "snapshot record")) return false;
    s.device = b.device;
    s.pending = true;
    return true;
}

void snapshot_free(Snapshot &s) {
    if (s.done) cudaEventDestroy(s.done);
    if (s.ready) cudaEventDestroy(s.ready);
    if (s.stream) cudaStreamDestroy(s.stream);
    if (s.dev) cudaFree(s.dev);
    if (s.host) cudaFreeHost(s.host);
    s = Snapshot{};
}

void backend_free(Backend &b) {
    if (b.stream) cudaStreamSynchronize(b.stream);
    for (auto &p : b.prof_pending) {
        cudaEventDestroy(p.second.first);
        cudaEventDestroy(p.second.second);
    }
    b.prof_pending.clear();
    if (b.arena) cudaFree(b.arena);
    b.arena = nullptr;
    if (b.adj_mem) cudaFree(b.adj_mem);
    b.adj_mem = nullptr;
    if (b.h_out) cudaFreeHost(b.h_out);
    b.h_out = nullptr;
    if (b.stream) cudaStreamDestroy(b.stream);
    b.stream = nullptr;
}

}  // namespace fm
