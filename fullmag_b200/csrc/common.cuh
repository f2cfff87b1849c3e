// common.cuh — scalar/complex helpers shared by the sm_100a kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fm {

constexpr double kPi = 3.14159265358979323846;
// MU0 = 4 pi 1e-7, evaluated in the same order as the reference
// (crates/fullmag-engine/src/lib.rs:26).
constexpr double kMu0 = 4.0 * kPi * 1e-7;

template <typename T> struct Cx;
template <> struct Cx<float> { using type = float2; };
template <> struct Cx<double> { using type = double2; };
template <typename T> using cx = typename Cx<T>::type;

template <typename T> __host__ __device__ __forceinline__ cx<T> mk(T a, T b) {
    cx<T> r; r.x = a; r.y = b; return r;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000 && !defined(FM_SCALAR_COMPLEX_ADD)
// FP32 pairs: one packed instruction (sm_100), each part rounded as the scalar
// op, so results do not change.  A translation unit whose kernels measured
// faster with the scalar pair defines FM_SCALAR_COMPLEX_ADD before any include.
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
#endif
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
    C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {
    C r; r.x = a.x * b.x + a.y * b.y; r.y = a.y * b.x - a.x * b.y; return r;
}
template <typename C> __device__ __forceinline__ C cconj(C a) { C r; r.x = a.x; r.y = -a.y; return r; }
// multiply by -i (forward) or +i (inverse)
template <bool INV, typename C> __device__ __forceinline__ C rot_i(C a) {
    C r;
    if (INV) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; }
    return r;
}

struct Dims {
    int nx, ny, nz;
    long long n;  // nx*ny*nz
};

}  // namespace fm
