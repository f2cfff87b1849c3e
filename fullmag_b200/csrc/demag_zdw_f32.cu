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
    bool ok = true;
    zdw_with_nz(b.nz, [&](auto nzc) {
        constexpr int NZ = decltype(nzc)::value;
        constexpr size_t smem = zdw_smem<NZ>();
        int occ = 0, sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b.device);
        ok &= cuda_ok(b, cudaFuncSetAttribute(k_zdw<NZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                      "attr zdw");
        ok &= cuda_ok(b, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_zdw<NZ>, kZdwThreads, smem),
                      "occupancy zdw");
        if (!ok || occ < 1) return;
        const long long batches = ((long long)b.nkx * b.Ly + kZdwCols - 1) / kZdwCols;
        b.grid_zdw = (int)std::max<long long>(1, std::min<long long>(batches, (long long)occ * sms));
        b.rsm_zdw = smem;
        b.use_zdw = true;
    });
    return ok;
}

void zdw_launch(Backend &b, const DemagArgs<float> &a) {
    zdw_with_nz(b.nz, [&](auto nzc) {
        constexpr int NZ = decltype(nzc)::value;
        k_zdw<NZ><<<b.grid_zdw, kZdwThreads, b.rsm_zdw, b.stream>>>(a);
    });
}

}  // namespace fm
