// Shared device types and helpers for the FFCM sm_100a kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ffcm {

// Device-side sticky error bits (read back by the host after a sync).
enum : int {
    DEVERR_NONFINITE_POSITION = 1,
    DEVERR_INDEX_RANGE = 2,
    DEVERR_COPY_TIMEOUT = 4,   // a bounded wait for a bulk copy gave up
};

template <typename T>
struct cplx {
    T x, y;
};

template <typename T>
__device__ __forceinline__ cplx<T> cmul(cplx<T> a, cplx<T> b) {
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename T>
__device__ __forceinline__ cplx<T> cadd(cplx<T> a, cplx<T> b) { return {a.x + b.x, a.y + b.y}; }
template <typename T>
__device__ __forceinline__ cplx<T> csub(cplx<T> a, cplx<T> b) { return {a.x - b.x, a.y - b.y}; }
template <typename T>
__device__ __forceinline__ cplx<T> cconj(cplx<T> a) { return {a.x, -a.y}; }
// multiply by -i (forward) or +i (inverse)
template <typename T>
__device__ __forceinline__ cplx<T> mul_mi(cplx<T> a) { return {a.y, -a.x}; }
template <typename T>
__device__ __forceinline__ cplx<T> mul_pi(cplx<T> a) { return {-a.y, a.x}; }

// Four-wide particle record (x, y, z, pad), 16/32-byte aligned.
template <typename T> struct vec4;
template <> struct alignas(16) vec4<float> { float x, y, z, w; };
template <> struct alignas(32) vec4<double> { double x, y, z, w; };

// IEEE round-to-nearest operations that the compiler may not contract into a
// fused multiply-add. Used wherever a later integer decision (a cell index, a
// stencil anchor, the cutoff test) depends on the exact rounding the
// reference's unfused Julia arithmetic produces.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }

__device__ __forceinline__ float fmod_t(float a, float b) { return fmodf(a, b); }
__device__ __forceinline__ double fmod_t(double a, double b) { return fmod(a, b); }
__device__ __forceinline__ float rint_t(float a) { return rintf(a); }
__device__ __forceinline__ double rint_t(double a) { return rint(a); }
__device__ __forceinline__ float floor_t(float a) { return floorf(a); }
__device__ __forceinline__ double floor_t(double a) { return floor(a); }
__device__ __forceinline__ float fma_t(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float exp_t(float a) { return expf(a); }
__device__ __forceinline__ double exp_t(double a) { return exp(a); }
__device__ __forceinline__ float erf_t(float a) { return erff(a); }
__device__ __forceinline__ double erf_t(double a) { return erf(a); }
__device__ __forceinline__ float sqrt_t(float a) { return sqrtf(a); }
__device__ __forceinline__ double sqrt_t(double a) { return sqrt(a); }
__device__ __forceinline__ float pow_t(float a, float b) { return powf(a, b); }
__device__ __forceinline__ double pow_t(double a, double b) { return pow(a, b); }
__device__ __forceinline__ bool isfinite_t(float a) { return isfinite(a); }
__device__ __forceinline__ bool isfinite_t(double a) { return isfinite(a); }

// Julia `mod(x, y)` for floating point (rem, then shift by y on a sign
// mismatch; an exact zero takes y's sign). src/cell_list.jl:26.
template <typename T>
__device__ __forceinline__ T julia_fmod(T x, T y) {
    T r = fmod_t(x, y);
    if (r == T(0)) return copysign(T(0), y);
    if ((r > T(0)) != (y > T(0))) return add_rn(r, y);
    return r;
}

// Julia integer `mod(a, m)` for m > 0 (result in [0, m)).
__device__ __forceinline__ int imod(int a, int m) {
    int r = a % m;
    return r < 0 ? r + m : r;
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

}  // namespace ffcm
