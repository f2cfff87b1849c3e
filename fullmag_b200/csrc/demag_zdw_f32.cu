// demag_zdw_f32.cu — configuration and launch of the FP32 direct z convolution
// for 8 < nz <= 16 (demag_zdw.cuh).
#include <cstdlib>
#include <cstring>

#include "demag_zdw.cuh"

namespace fm {

static bool zdw_env(const char *name, const char *value) {
    const char *v = std::getenv(name);
    return v && std::strcmp(v, value) == 0;
}

bool zdw_wanted(const Backend &b, bool fp32) {
    if (!fp32 || b.thin || b.want_yz || zdw_env("FULLMAG_FDM_ZCONV", "fft")) return false;
    return (b.nz > 8 && b.nz <= 16) || (b.nz == 8 && zdw_env("FULLMAG_FDM_ZDW", "on"));
}

bool zdw_configure(Backend &b) {
    b.use_zdw = false;
    // window form: Ly a multiple of 128 and the padded table within the octant's
    // allocation (6 KZ nkx KY values; KY >= 3 nz is enough)
    const int kyp = (b.KY + 3) / 4 * 4;
    b.zdw_win = b.Ly % 128 == 0 && (long long)b.nz * kyp <= (long long)b.KZ * b.KY &&
                !zdw_env("FULLMAG_FDM_ZDW", "elem");
    b.zdw_kyp = b.zdw_win ? kyp : 0;
    bool ok = true;
    zdw_with_nz(b.nz, [&](auto nzc) {
        constexpr int NZ = decltype(nzc)::value;
        auto cfg = [&](auto kern, size_t smem) {
            int occ = 0, sms = 148;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b.device);
            ok &= cuda_ok(b, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                          "attr zdw");
            // the largest shared-memory carveout, so that two blocks fit per SM
            ok &= cuda_ok(b, cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                                  (int)cudaSharedmemCarveoutMaxShared), "carveout zdw");
            ok &= cuda_ok(b, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kZdwThreads, smem),
                          "occupancy zdw");
            if (!ok || occ < 1) return;
            const long long batches = ((long long)b.nkx * b.Ly + kZdwCols - 1) / kZdwCols;
            b.grid_zdw = (int)std::max<long long>(1, std::min<long long>(batches, (long long)occ * sms));
            b.rsm_zdw = smem;
            b.use_zdw = true;
        };
        if (b.zdw_win) cfg(k_zdw<NZ, true>, zdw_smem<NZ, true>());
        else cfg(k_zdw<NZ, false>, zdw_smem<NZ, false>());
    });
    return ok;
}

void zdw_launch(Backend &b, const DemagArgs<float> &a) {
    zdw_with_nz(b.nz, [&](auto nzc) {
        constexpr int NZ = decltype(nzc)::value;
        if (b.zdw_win) k_zdw<NZ, true><<<b.grid_zdw, kZdwThreads, b.rsm_zdw, b.stream>>>(a, b.zdw_kyp);
        else k_zdw<NZ, false><<<b.grid_zdw, kZdwThreads, b.rsm_zdw, b.stream>>>(a, 0);
    });
}

}  // namespace fm
