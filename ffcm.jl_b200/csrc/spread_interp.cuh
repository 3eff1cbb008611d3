// Steps 3 and 5: Gaussian spreading of forces to the grid and interpolation
// of the grid velocity back to the particles, over the same M_G^3 stencil.
//
// Reference: src/stencil.jl:80-112 (_fill_particle_stencil!: nearest anchor
// j = round(Y/h) ties-to-even, per axis x = (j - M_G/2 + k - 1) h - Y, weight
// inv_norm * exp(-x^2 inv_2S2), wrapped index mod(g, M)); src/spread_forces.jl
// :73-130 (w = (a0 + a2 (r2x + r2yz)) gx (gy gz), f_g += w F); src/interpolate.jl
// :322-376 (v = sum w u_g, V[:, original_index[s]] = h^3 v).
//
// Grid layout: three component planes (x, y, z) of Mx*My*Mz values, x fastest.
#pragma once

#include "common.cuh"

namespace ffcm {

template <typename T>
struct StencilParams {
    int Mx, My, Mz, MG, half;
    T h, inv_h, a0, a2, inv_norm, inv_2S2;
    // Float64-geometry stencils (opt-in, comp = 1): the spacing of the box as
    // the caller gave it, in double (inv_hd = 1 / (L / M)), and split into two
    // T values h_hi + h_lo
    double inv_hd;
    T h_hi, h_lo;
    int comp;
};

// Which grid points a particle's stencil covers and how far they are from it.
//  * reference arithmetic (comp = 0; src/stencil.jl:97-105): the anchor
//    j = round(Y inv_h) and the offsets x = T(g) h - Y in the working precision
//    T. In Float32 the anchor of a particle whose Y / h lies within a few
//    ulp(Y / h) of a half-integer can differ from the one Float64 arithmetic
//    picks (and, at a box length like 275.6 that Float32 cannot represent,
//    from the one of the box the caller meant); the truncated M_G-point
//    stencil then covers a neighbouring set of points. Those particles carry
//    most of the Float32 result's distance from the Float64 one (2.2e-4
//    relative at N = 500k, L = 275.6, 512^3).
//  * Float64 geometry (comp = 1): the anchor is rounded from the double product
//    Y inv_hd, so it is the Float64 reference's choice, and the offset is
//    fma(g, h_hi, -Y) + g h_lo, rounded once at its own size. The weights
//    themselves stay in T. Bit parity with the reference's Float32 arithmetic
//    is given up, so this is not the default.
template <typename T>
__device__ __forceinline__ int stencil_anchor(const StencilParams<T>& p, T y) {
    if (p.comp) return (int)rint(__dmul_rn((double)y, p.inv_hd));
    return (int)rint_t(mul_rn(y, p.inv_h));
}

template <typename T>
__device__ __forceinline__ T stencil_offset(const StencilParams<T>& p, int g, T y) {
    if (p.comp) return fma_t((T)g, p.h_hi, -y) + (T)g * p.h_lo;
    return sub_rn(mul_rn((T)g, p.h), y);
}

// Per-warp shared stencil: g[3][MG], r2[3][MG], idx[3][MG].
template <typename T>
struct WarpStencil {
    T* g;
    T* r2;
    int* idx;
};

// Fill the separable stencil of one particle; lanes cover the 3*MG entries.
template <typename T>
__device__ __forceinline__ void fill_stencil_warp(const StencilParams<T>& p, T y0, T y1, T y2,
                                                  WarpStencil<T> st) {
    const int lane = lane_id();
    for (int e = lane; e < 3 * p.MG; e += 32) {
        int axis = e / p.MG, k = e - axis * p.MG;
        T y = axis == 0 ? y0 : (axis == 1 ? y1 : y2);
        int M = axis == 0 ? p.Mx : (axis == 1 ? p.My : p.Mz);
        int j = stencil_anchor(p, y);
        int g = j + (k - p.half);
        T x = stencil_offset(p, g, y);
        T x2 = mul_rn(x, x);
        st.g[e] = p.inv_norm * exp_t(-x2 * p.inv_2S2);
        st.r2[e] = x2;
        st.idx[e] = imod(g, M);
    }
    __syncwarp();
}

// Reference-style global-atomic spread: one warp per particle. The grid must
// be zeroed first.
template <typename T>
__global__ void k_spread_atomic(int n_part, const vec4<T>* __restrict__ Ys,
                                const vec4<T>* __restrict__ Fs, T* __restrict__ grid,
                                StencilParams<T> p) {
    extern __shared__ unsigned char smem_raw[];
    const int warps = blockDim.x >> 5;
    const int w = threadIdx.x >> 5;
    const int MG = p.MG;
    T* gbase = reinterpret_cast<T*>(smem_raw);
    WarpStencil<T> st{gbase + w * 3 * MG, gbase + (warps + w) * 3 * MG,
                      reinterpret_cast<int*>(gbase + 2 * warps * 3 * MG) + w * 3 * MG};
    const int64_t plane = (int64_t)p.Mx * p.My * p.Mz;
    const int MG2 = MG * MG, MG3 = MG2 * MG;
    for (int s = blockIdx.x * warps + w; s < n_part; s += gridDim.x * warps) {
        vec4<T> y = Ys[s], f = Fs[s];
        fill_stencil_warp(p, y.x, y.y, y.z, st);
        for (int q = lane_id(); q < MG3; q += 32) {
            int kz = q / MG2;
            int r = q - kz * MG2;
            int ky = r / MG;
            int kx = r - ky * MG;
            const T gz = st.g[2 * MG + kz], r2z = st.r2[2 * MG + kz];
            const T gyz = st.g[MG + ky] * gz;
            const T r2yz = st.r2[MG + ky] + r2z;
            const T wgt = (p.a0 + p.a2 * (st.r2[kx] + r2yz)) * st.g[kx] * gyz;
            int64_t o = ((int64_t)st.idx[2 * MG + kz] * p.My + st.idx[MG + ky]) * p.Mx + st.idx[kx];
            atomicAdd(grid + o, wgt * f.x);
            atomicAdd(grid + plane + o, wgt * f.y);
            atomicAdd(grid + 2 * plane + o, wgt * f.z);
        }
        __syncwarp();
    }
}

// Interpolation: one warp per particle, lanes stride the stencil, shuffle
// reduction, lane 0 writes V[:, perm[s]] = h^3 v (overwrite).
template <typename T>
__global__ void k_interpolate_warp(int n_part, const vec4<T>* __restrict__ Ys,
                                   const int32_t* __restrict__ perm, const T* __restrict__ grid,
                                   T* __restrict__ V, StencilParams<T> p, T h3) {
    extern __shared__ unsigned char smem_raw[];
    const int warps = blockDim.x >> 5;
    const int w = threadIdx.x >> 5;
    const int MG = p.MG;
    T* gbase = reinterpret_cast<T*>(smem_raw);
    WarpStencil<T> st{gbase + w * 3 * MG, gbase + (warps + w) * 3 * MG,
                      reinterpret_cast<int*>(gbase + 2 * warps * 3 * MG) + w * 3 * MG};
    const int64_t plane = (int64_t)p.Mx * p.My * p.Mz;
    const int MG2 = MG * MG, MG3 = MG2 * MG;
    for (int s = blockIdx.x * warps + w; s < n_part; s += gridDim.x * warps) {
        vec4<T> y = Ys[s];
        fill_stencil_warp(p, y.x, y.y, y.z, st);
        T v0 = 0, v1 = 0, v2 = 0;
        for (int q = lane_id(); q < MG3; q += 32) {
            int kz = q / MG2;
            int r = q - kz * MG2;
            int ky = r / MG;
            int kx = r - ky * MG;
            const T gz = st.g[2 * MG + kz], r2z = st.r2[2 * MG + kz];
            const T gyz = st.g[MG + ky] * gz;
            const T r2yz = st.r2[MG + ky] + r2z;
            const T wgt = (p.a0 + p.a2 * (st.r2[kx] + r2yz)) * st.g[kx] * gyz;
            int64_t o = ((int64_t)st.idx[2 * MG + kz] * p.My + st.idx[MG + ky]) * p.Mx + st.idx[kx];
            v0 += wgt * __ldg(grid + o);
            v1 += wgt * __ldg(grid + plane + o);
            v2 += wgt * __ldg(grid + 2 * plane + o);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            v0 += __shfl_xor_sync(0xffffffffu, v0, o);
            v1 += __shfl_xor_sync(0xffffffffu, v1, o);
            v2 += __shfl_xor_sync(0xffffffffu, v2, o);
        }
        if (lane_id() == 0) {
            int64_t n = perm[s];
            V[3 * n] = h3 * v0;
            V[3 * n + 1] = h3 * v1;
            V[3 * n + 2] = h3 * v2;
        }
        __syncwarp();
    }
}

}  // namespace ffcm
