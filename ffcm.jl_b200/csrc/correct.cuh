// Step 6: real-space pair correction M - M~ over the 27 neighbour cells plus
// the self term.
//
// Reference: src/correct_velocities.jl:21-27 (_self_correction), :71-104
// (_correction_scalars: A(r) I + B(r) x x^T with two erf and two exp),
// :121-127 (_min_image, ties-to-even), :216-286 (the CPU kernel: cells in
// hash order, 27 wrapped neighbour cells dz/dy/dx, s2 != s, r^2 < R_c^2,
// V[:, original_index[s]] += v).
//
// One thread per sorted particle gathers over the 27 cells in the reference's
// loop order, so the accumulation order per particle is the reference's; no
// atomics. The separation, r^2 and the cutoff test use unfused IEEE
// operations, so the set of interacting pairs is exactly the reference's.
#pragma once

#include "common.cuh"

namespace ffcm {

// Constants of _correction_scalars that do not depend on r, computed on the
// host in the working precision with the reference's operation order.
template <typename T>
struct CorrConsts {
    T s2, s4, S2, S4, d, dq, fourpimu, eightpimu, mu;
    T two_sigma, two_Sigma, pref_s, pref_S, four_s2, four_S2;
    T self;
    T L0, L1, L2, Rc2, ic0, ic1, ic2;
    int m0, m1, m2;
};

template <typename T>
__device__ __forceinline__ void correction_scalars(T r, const CorrConsts<T>& c, T& A, T& B) {
    const T r2 = r * r;
    const T r3 = r * r * r;
    const T r4 = r2 * r2;
    const T r5 = r4 * r;
    const T erf_diff = erf_t(r / c.two_sigma) - erf_t(r / c.two_Sigma);
    const T Ds = c.pref_s * exp_t(-r2 / c.four_s2);
    const T DS = c.pref_S * exp_t(-r2 / c.four_S2);
    A = erf_diff * (T(1) / (c.eightpimu * r) + c.s2 / (c.fourpimu * r3)) -
        T(2) * c.s4 / (c.mu * r2) * Ds +
        (T(2) * c.S4 / (c.mu * r2) + c.d / c.mu * (T(1) + T(2) * c.S2 / r2) -
         c.dq * (T(2) - r2 / (T(2) * c.S2)) / (T(2) * c.mu * c.S2)) * DS;
    B = erf_diff * (T(1) / (c.eightpimu * r3) - T(3) * c.s2 / (c.fourpimu * r5)) +
        T(6) * c.s4 / (c.mu * r4) * Ds +
        (-T(6) * c.S4 / (c.mu * r4) - c.d / (c.mu * r2) * (T(1) + T(6) * c.S2 / r2) -
         c.dq / (T(4) * c.mu * c.S4)) * DS;
}

template <typename T>
__device__ __forceinline__ T min_image(T x, T L) {
    return sub_rn(x, mul_rn(L, rint_t(div_rn(x, L))));
}

template <typename T>
__global__ void k_correct(int n_part, const vec4<T>* __restrict__ Ys,
                          const vec4<T>* __restrict__ Fs, const int32_t* __restrict__ off,
                          const int32_t* __restrict__ perm, T* __restrict__ V, CorrConsts<T> c) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n_part; s += gridDim.x * blockDim.x) {
        const vec4<T> yn = Ys[s];
        const vec4<T> fn = Fs[s];
        int cx = (int)floor_t(mul_rn(yn.x, c.ic0));
        int cy = (int)floor_t(mul_rn(yn.y, c.ic1));
        int cz = (int)floor_t(mul_rn(yn.z, c.ic2));
        cx = max(0, min(cx, c.m0 - 1));
        cy = max(0, min(cy, c.m1 - 1));
        cz = max(0, min(cz, c.m2 - 1));
        T v0 = c.self * fn.x, v1 = c.self * fn.y, v2 = c.self * fn.z;
        for (int dz = -1; dz <= 1; ++dz) {
            const int nz = imod(cz + dz, c.m2);
            for (int dy = -1; dy <= 1; ++dy) {
                const int ny = imod(cy + dy, c.m1);
                for (int dx = -1; dx <= 1; ++dx) {
                    const int nx = imod(cx + dx, c.m0);
                    const int cn = nx + (ny + nz * c.m1) * c.m0;
                    const int e = off[cn + 1];
                    for (int s2 = off[cn]; s2 < e; ++s2) {
                        if (s2 == s) continue;
                        const vec4<T> ym = Ys[s2];
                        const T x0 = min_image(sub_rn(yn.x, ym.x), c.L0);
                        const T x1 = min_image(sub_rn(yn.y, ym.y), c.L1);
                        const T x2 = min_image(sub_rn(yn.z, ym.z), c.L2);
                        const T rr = add_rn(add_rn(mul_rn(x0, x0), mul_rn(x1, x1)), mul_rn(x2, x2));
                        if (!(rr < c.Rc2)) continue;
                        T A, B;
                        correction_scalars(sqrt_t(rr), c, A, B);
                        const vec4<T> fm = Fs[s2];
                        const T xF = x0 * fm.x + x1 * fm.y + x2 * fm.z;
                        const T bx = B * xF;
                        v0 += A * fm.x + bx * x0;
                        v1 += A * fm.y + bx * x1;
                        v2 += A * fm.z + bx * x2;
                    }
                }
            }
        }
        const int64_t n = perm[s];
        V[3 * n] += v0;
        V[3 * n + 1] += v1;
        V[3 * n + 2] += v2;
    }
}

}  // namespace ffcm
