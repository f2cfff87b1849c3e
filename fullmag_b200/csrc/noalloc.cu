// noalloc.cu — the demag field for callers that cannot allocate device memory.
//
// fullmag_fdm_demag_field_f64_noalloc computes H_demag = -IFFT(N(k) FFT(Ms m))
// exactly like the stepper's FP64 demag passes (demag_reg.cuh), but it makes
// no device allocation: the FFT work arrays (two half-spectrum buffers and the
// twiddle tables) live in g_fft_scratch, a file-scope __device__ array of
// kNoAllocScratchBytes (32 MiB).  Every GPU that loads this library holds that
// array until the process exits.  The caller owns and passes the inputs (m,
// the Newell octant) and the output (H); the library only launches kernels.
//
// Who needs this: code that runs inside a host framework which owns the
// whole device-memory budget and forbids allocations outside its own
// allocator, and latency-critical loops that must not pay the implicit device
// synchronisation cudaMalloc / cudaFree bring.  Such callers cannot use
// fullmag_fdm_backend_create, which allocates its arena.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <type_traits>

#include "demag_reg.cuh"
#include "fullmag_fdm.h"
#include "fullmag_fdm_ext.h"

namespace fm {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
constexpr int kMaxDevices = 64;

// FFT work arrays of the allocation-free entry point (shared by every call).
static __device__ __align__(256) unsigned char g_fft_scratch[kNoAllocScratchBytes];

struct DeviceSlot {
    bool ready = false;
    unsigned char *scratch = nullptr;  // device address of g_fft_scratch on that device
};
std::mutex g_mu;
DeviceSlot g_slots[kMaxDevices];

void put_error(char *buf, uint64_t len, const char *msg) {
    if (buf && len > 0) {
        std::strncpy(buf, msg, (size_t)len - 1);
        buf[len - 1] = '\0';
    }
}

// With the device current: resolve the array's device address (the host-side
// symbol is only a stand-in) on every call, which is cheap, and once per
// device (again if the address changed) fill this file's copy of the radix-64
// twiddle table.  The upload goes through the legacy default stream from
// pageable memory, which may return before the data reach the device, and a
// caller's non-blocking stream is not ordered after it: the device is
// synchronised once here, before the first kernel can read the table.
bool setup_device(int dev, unsigned char **out, char *err, uint64_t errlen) {
    std::lock_guard<std::mutex> lock(g_mu);
    DeviceSlot &s = g_slots[dev];
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_fft_scratch);
    if (e != cudaSuccess) {
        char m[256];
        std::snprintf(m, sizeof(m), "cudaGetSymbolAddress(g_fft_scratch): %s", cudaGetErrorString(e));
        put_error(err, errlen, m);
        return false;
    }
    if (!s.ready || s.scratch != p) {
        s.ready = false;
        double2 d[64];
        float2 f[64];
        for (int k = 0; k < 64; ++k) {
            const double a = 2.0 * kPi * (double)k / 64.0;
            d[k] = make_double2(std::cos(a), -std::sin(a));
            f[k] = make_float2((float)d[k].x, (float)d[k].y);
        }
        e = cudaMemcpyToSymbol(c_tw64d, d, sizeof(d));
        if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_tw64f, f, sizeof(f));
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            char m[256];
            std::snprintf(m, sizeof(m), "twiddle table upload: %s", cudaGetErrorString(e));
            put_error(err, errlen, m);
            return false;
        }
        s.scratch = static_cast<unsigned char *>(p);
        s.ready = true;
    }
    *out = s.scratch;
    return true;
}

// tw[k] = exp(-2 pi i k / L), computed on the device (no host staging copy);
// with L2 > 0 the 4-step table of fftreg.cuh (entry k1 L2 + t holds the value
// of k = k1 t).
__global__ void k_fill_twiddles(double2 *tw, int L, int L2) {
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < L; idx += gridDim.x * blockDim.x) {
        const int k = L2 > 0 ? (idx / L2) * (idx % L2) : idx;
        double sn, cs;
        sincospi(2.0 * (double)k / (double)L, &sn, &cs);
        tw[idx] = make_double2(cs, -sn);
    }
}

template <int V> using IC = std::integral_constant<int, V>;

template <class F>
bool split_for(int L, F &&f) {
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
        default: return false;
    }
}

bool pow2(int L) { return L >= 2 && (L & (L - 1)) == 0; }

}  // namespace
}  // namespace fm

extern "C" int fullmag_fdm_demag_field_f64_noalloc(uint32_t nx, uint32_t ny, uint32_t nz,
                                                   int thin_film_2d, const double *octant,
                                                   const double *m, double ms, double *h,
                                                   void *stream, char *error_out,
                                                   uint64_t error_out_len) {
    using namespace fm;
    using C = double2;
    if (!octant || !m || !h || nx == 0 || ny == 0 || nz == 0 || !(ms > 0.0)) {
        put_error(error_out, error_out_len, "null pointer, empty grid or non-positive Ms");
        return FULLMAG_FDM_ERR_INVALID;
    }
    // range first, so that the doubled lengths below cannot overflow
    if (nx > 512 || ny > 512 || nz > 8) {
        put_error(error_out, error_out_len,
                  "grid not supported: 2nx and 2ny must be powers of two <= 1024 and 2nz <= 16 (or nz = 1)");
        return FULLMAG_FDM_ERR_INVALID;
    }
    const bool thin = thin_film_2d && nz == 1;
    const int Lx = 2 * (int)nx, Ly = 2 * (int)ny, Lz = thin ? 1 : 2 * (int)nz;
    if (!pow2(Lx) || !pow2(Ly) || Lx > 1024 || Ly > 1024 || (!thin && (!pow2(Lz) || Lz > 16))) {
        put_error(error_out, error_out_len,
                  "grid not supported: 2nx and 2ny must be powers of two <= 1024 and 2nz <= 16 (or nz = 1)");
        return FULLMAG_FDM_ERR_INVALID;
    }
    const int nkx = (int)nx + 1;
    // scratch layout (complex elements): twx | twy | twz | twxT | twyT | S1 | S2
    const size_t s1 = (size_t)3 * nz * nkx * ny, s2 = thin ? 0 : (size_t)3 * nz * nkx * Ly;
    const size_t elems = (size_t)2 * Lx + 2 * Ly + Lz + s1 + s2 + 16;
    const size_t need = elems * sizeof(C);
    if (need > kNoAllocScratchBytes) {
        char msg[256];
        std::snprintf(msg, sizeof(msg),
                      "grid %ux%ux%u needs %zu bytes of FFT scratch; the allocation-free entry point "
                      "holds at most %zu bytes",
                      nx, ny, nz, need, kNoAllocScratchBytes);
        put_error(error_out, error_out_len, msg);
        return FULLMAG_FDM_ERR_INVALID;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        put_error(error_out, error_out_len, "no current CUDA device");
        return FULLMAG_FDM_ERR_CUDA;
    }
    unsigned char *base = nullptr;
    if (!setup_device(dev, &base, error_out, error_out_len)) return FULLMAG_FDM_ERR_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // a launch error left by earlier, unrelated work is not this call's: clear
    // it, so that the check after the launches reports only this call's own
    (void)cudaGetLastError();

    C *p = reinterpret_cast<C *>(base);
    C *twx = p, *twy = twx + Lx, *twz = twy + Ly;
    C *twxT = twz + Lz, *twyT = twxT + Lx;
    C *ps1 = twyT + Ly;
    C *ps2 = ps1 + s1;
    k_fill_twiddles<<<(Lx + 255) / 256, 256, 0, st>>>(twx, Lx, 0);
    k_fill_twiddles<<<(Ly + 255) / 256, 256, 0, st>>>(twy, Ly, 0);
    k_fill_twiddles<<<(Lz + 255) / 256, 256, 0, st>>>(twz, Lz, 0);
    k_fill_twiddles<<<(Lx + 255) / 256, 256, 0, st>>>(twxT, Lx, l2_for(Lx));
    k_fill_twiddles<<<(Ly + 255) / 256, 256, 0, st>>>(twyT, Ly, l2_for(Ly));

    DemagArgs<double> a{};
    a.nx = nx; a.ny = ny; a.nz = nz;
    a.n = (long long)nx * ny * nz;
    a.Lx = Lx; a.Ly = Ly; a.Lz = Lz; a.nkx = nkx;
    a.KZ = thin ? 1 : (int)nz + 1;
    a.KY = (int)ny + 1;
    a.twx = twx; a.twy = twy; a.twz = twz;
    a.twxT = twxT; a.twyT = twyT;
    a.s1 = ps1; a.s2 = thin ? nullptr : ps2;
    a.spec = octant;
    a.m = m;
    a.mask = nullptr;
    a.ms_map = nullptr;
    a.ms = ms;
    a.hd = h;
    a.norm = 1.0 / ((double)Lx * (double)Ly * (double)Lz);

    const size_t sz = sizeof(C);
    bool ok = true;
    // x passes: complex lines (row pairs) per block
    int thr_x = 0;
    size_t smx = 0, smxi = 0;
    split_for(Lx, [&](auto l1, auto l2) {
        constexpr int L1 = decltype(l1)::value, L2 = decltype(l2)::value;
        constexpr int TE = line_region<L1, L2>();
        const int unit = L2 >= 32 ? 1 : 32 / L2;
        int lp = std::max(unit, (128 / L2) / unit * unit);
        while (lp > unit && (size_t)(lp * TE) * sz > 200 * 1024) lp -= unit;
        a.lines_x = lp;
        thr_x = lp * L2;
        smx = (size_t)(lp * TE) * sz;
        smxi = smx + (size_t)L1 * L2 * sz;  // the x inverse also holds the twiddle table
        ok &= cudaFuncSetAttribute(k_xf_r<double, L1, L2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx) == cudaSuccess;
        ok &= cudaFuncSetAttribute(k_xi_r<double, L1, L2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smxi) == cudaSuccess;
    });
    int thr_y = 0;
    size_t smy = 0;
    split_for(Ly, [&](auto l1, auto l2) {
        constexpr int L1 = decltype(l1)::value, L2 = decltype(l2)::value;
        if (thin) {
            constexpr int TE = line_region<L1, L2>();
            const int unit = L2 >= 32 ? 1 : 32 / L2;
            int kb = std::max(unit, (192 / (3 * L2)) / unit * unit);
            while (kb > unit && (size_t)(3 * kb * TE) * sz > 200 * 1024) kb -= unit;
            a.kb_y = kb;
            thr_y = 3 * kb * L2;
            smy = (size_t)(3 * kb * TE) * sz;
            ok &= cudaFuncSetAttribute(k_yc_r<double, L1, L2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smy) == cudaSuccess;
        } else {
            constexpr int TE = tile_elems(L1, L2);
            const int lpb = std::max(1, 128 / L2);
            a.lines_y = lpb;
            thr_y = lpb * L2;
            smy = (size_t)(lpb * TE) * sz;
            ok &= cudaFuncSetAttribute(k_yf_r<double, L1, L2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smy) == cudaSuccess;
            ok &= cudaFuncSetAttribute(k_yi_r<double, L1, L2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smy) == cudaSuccess;
        }
    });
    if (!ok) {
        put_error(error_out, error_out_len, "cudaFuncSetAttribute failed");
        return FULLMAG_FDM_ERR_CUDA;
    }
    const int RB = 2 * a.lines_x;
    const dim3 gx((ny + RB - 1) / RB, nz, 3);
    split_for(Lx, [&](auto l1, auto l2) {
        constexpr int L1 = decltype(l1)::value, L2 = decltype(l2)::value;
        k_xf_r<double, L1, L2><<<gx, thr_x, smx, st>>>(a);
    });
    if (thin) {
        split_for(Ly, [&](auto l1, auto l2) {
            constexpr int L1 = decltype(l1)::value, L2 = decltype(l2)::value;
            k_yc_r<double, L1, L2><<<(nkx + a.kb_y - 1) / a.kb_y, thr_y, smy, st>>>(a);
        });
    } else {
        const long long lines = 3LL * nz * nkx;
        const unsigned gy = (unsigned)((lines + a.lines_y - 1) / a.lines_y);
        split_for(Ly, [&](auto l1, auto l2) {
            constexpr int L1 = decltype(l1)::value, L2 = decltype(l2)::value;
            k_yf_r<double, L1, L2><<<gy, thr_y, smy, st>>>(a);
        });
        const int cols = nkx * Ly;
        const int P = Lz > 8 ? 2 : 1;
        const unsigned gz = (unsigned)std::min<long long>(((long long)cols * P + 127) / 128, 148LL * 64);
        switch (Lz * 10 + P) {
            case 21: k_zc_r<double, 2, 1><<<gz, 128, 0, st>>>(a); break;
            case 41: k_zc_r<double, 4, 1><<<gz, 128, 0, st>>>(a); break;
            case 81: k_zc_r<double, 8, 1><<<gz, 128, 0, st>>>(a); break;
            case 162: k_zc_r<double, 16, 2><<<gz, 128, 0, st>>>(a); break;
            default: break;
        }
        split_for(Ly, [&](auto l1, auto l2) {
            constexpr int L1 = decltype(l1)::value, L2 = decltype(l2)::value;
            k_yi_r<double, L1, L2><<<gy, thr_y, smy, st>>>(a);
        });
    }
    split_for(Lx, [&](auto l1, auto l2) {
        constexpr int L1 = decltype(l1)::value, L2 = decltype(l2)::value;
        k_xi_r<double, L1, L2><<<gx, thr_x, smxi, st>>>(a);
    });
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        char msg[256];
        std::snprintf(msg, sizeof(msg), "kernel launch: %s", cudaGetErrorString(e));
        put_error(error_out, error_out_len, msg);
        return FULLMAG_FDM_ERR_CUDA;
    }
    return FULLMAG_FDM_OK;
}
