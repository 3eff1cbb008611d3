// Host-side selection and launch of the FFT pass kernels: the register
// (power-of-two) path when the line length allows it, the generic
// shared-memory Stockham path otherwise.
#pragma once

#include "fft.cuh"
#include "fft_pow2.cuh"

namespace ffcm {

inline bool fast_len(int n) { return n >= 32 && n <= 1024 && (n & (n - 1)) == 0; }

template <typename T>
struct FastFft {
    // x pass: H = Mx/2 complex points; block = lpb * H/8 threads (<= 256).
    static int x_lpb(int H) { return std::max(1, 256 / (H / 8)); }
    static size_t x_smem(int H) {
        return (size_t)(2 * H + x_lpb(H) * padded_len(H)) * sizeof(cplx<T>);
    }
    static size_t yz_smem(int n, int B) { return (size_t)(n + B * padded_len(n)) * sizeof(cplx<T>); }
    static size_t zlr_smem(int n, int B) { return (size_t)(n + 3 * B * padded_len(n)) * sizeof(cplx<T>); }
};

// Function-pointer tables for the y and z kernels, indexed by (n, B).
template <typename T>
using YKernel = void (*)(cplx<T>*, int, int, int, int, int, const cplx<T>*, int);
template <typename T>
using ZKernel = void (*)(cplx<T>*, int, int, int, int, const cplx<T>*, const T*, const T*, const T*, T);
template <typename T>
using XfKernel = void (*)(const T*, cplx<T>*, int, int, const cplx<T>*, int);
template <typename T>
using XiKernel = void (*)(const cplx<T>*, T*, int, int, const cplx<T>*, int);

template <typename T>
YKernel<T> y_kernel(int n, int B) {
#define FFCM_Y(NN, BB) if (n == NN && B == BB) return k_fftp_y<T, NN, BB>;
    FFCM_Y(32, 8) FFCM_Y(32, 16) FFCM_Y(64, 8) FFCM_Y(64, 16) FFCM_Y(128, 8) FFCM_Y(128, 16)
    FFCM_Y(256, 8) FFCM_Y(256, 16) FFCM_Y(512, 8) FFCM_Y(512, 16) FFCM_Y(1024, 4) FFCM_Y(1024, 8)
#undef FFCM_Y
    return nullptr;
}

template <typename T>
ZKernel<T> z_kernel(int n, int B) {
#define FFCM_Z(NN, BB) if (n == NN && B == BB) return k_fftp_z_stokes<T, NN, BB>;
    FFCM_Z(32, 8) FFCM_Z(32, 16) FFCM_Z(64, 8) FFCM_Z(64, 16) FFCM_Z(128, 4) FFCM_Z(128, 8)
    FFCM_Z(256, 4) FFCM_Z(256, 8) FFCM_Z(512, 4) FFCM_Z(512, 8) FFCM_Z(1024, 2) FFCM_Z(1024, 4)
#undef FFCM_Z
    return nullptr;
}

template <typename T>
ZKernel<T> zlr_kernel(int n, int B) {
#define FFCM_ZL(NN, BB) if (n == NN && B == BB) return k_fftp_z_stokes_lr<T, NN, BB>;
    FFCM_ZL(64, 8) FFCM_ZL(64, 16) FFCM_ZL(128, 4) FFCM_ZL(128, 8) FFCM_ZL(256, 2) FFCM_ZL(256, 4)
    FFCM_ZL(256, 8) FFCM_ZL(512, 2) FFCM_ZL(512, 4) FFCM_ZL(1024, 2)
#undef FFCM_ZL
    return nullptr;
}

template <typename T>
XfKernel<T> xf_kernel(int H) {
#define FFCM_XF(HH) if (H == HH) return k_fftp_x_r2c<T, HH>;
    FFCM_XF(32) FFCM_XF(64) FFCM_XF(128) FFCM_XF(256) FFCM_XF(512) FFCM_XF(1024)
#undef FFCM_XF
    return nullptr;
}

template <typename T>
XiKernel<T> xi_kernel(int H) {
#define FFCM_XI(HH) if (H == HH) return k_fftp_x_c2r<T, HH>;
    FFCM_XI(32) FFCM_XI(64) FFCM_XI(128) FFCM_XI(256) FFCM_XI(512) FFCM_XI(1024)
#undef FFCM_XI
    return nullptr;
}

// Bundle widths with an instantiated kernel, for the y and z passes.
inline int y_bundles(int n, int* out) {
    int c = 0;
    for (int B : {4, 8, 16}) if (B * (n / 8) <= 1024 && y_kernel<float>(n, B)) out[c++] = B;
    return c;
}
inline int z_bundles(int n, int* out) {
    int c = 0;
    for (int B : {2, 4, 8, 16}) if (B * (n / 8) <= 512 && z_kernel<float>(n, B)) out[c++] = B;
    return c;
}

}  // namespace ffcm
