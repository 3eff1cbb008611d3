// Step 6: real-space pair correction M - M~ over the 27 neighbour cells plus
// the self term.
//
// Reference: src/correct_velocities.jl:21-27 (_self_correction), :71-104
// (_correction_scalars: A(r) I + B(r) x x^T with two erf and two exp),
// :121-127 (_min_image, ties-to-even), :216-286 (the CPU kernel: cells in
// hash order, 27 wrapped neighbour cells dz/dy/dx, s2 != s, r^2 < R_c^2,
// V[:, original_index[s]] += v).
//
// A few threads per sorted particle gather over the 27 cells (no atomics,
// deterministic). The separation, r^2 and the cutoff test use unfused IEEE
// operations, so the set of interacting pairs is exactly the reference's.
#pragma once

#include "common.cuh"

namespace ffcm {

// Constants of _correction_scalars that do not depend on r, computed on the
// host in the working precision. The pair scalars below are the reference's
// expressions regrouped over powers of 1/r (one division per pair instead of
// fifteen); they agree with the reference to round-off.
template <typename T>
struct CorrConsts {
    T inv_two_sigma, inv_two_Sigma, pref_s, pref_S, inv_four_s2, inv_four_S2;
    T k1, k2, k3, k4, k5, k6, k7, k8, k9, k10, k11, k12, k13;
    T self;
    T L0, L1, L2, Rc2, ic0, ic1, ic2;
    int m0, m1, m2;
};

// src/correct_velocities.jl:71-104:
//   A = erf_diff (1/(8 pi mu r) + s2/(4 pi mu r^3)) - 2 s4/(mu r^2) D_s
//       + [2 S4/(mu r^2) + d/mu (1 + 2 S2/r^2) - dq (2 - r^2/(2 S2))/(2 mu S2)] D_S
//   B = erf_diff (1/(8 pi mu r^3) - 3 s2/(4 pi mu r^5)) + 6 s4/(mu r^4) D_s
//       + [-6 S4/(mu r^4) - d/(mu r^2) (1 + 6 S2/r^2) - dq/(4 mu S4)] D_S
template <typename T>
__device__ __forceinline__ void correction_scalars(T r, const CorrConsts<T>& c, T& A, T& B) {
    const T r2 = r * r;
    const T ir = T(1) / r;
    const T ir2 = ir * ir, ir3 = ir2 * ir, ir4 = ir2 * ir2, ir5 = ir4 * ir;
    const T erf_diff = erf_t(r * c.inv_two_sigma) - erf_t(r * c.inv_two_Sigma);
    const T Ds = c.pref_s * exp_t(-r2 * c.inv_four_s2);
    const T DS = c.pref_S * exp_t(-r2 * c.inv_four_S2);
    A = erf_diff * (c.k1 * ir + c.k2 * ir3) - c.k3 * ir2 * Ds +
        (c.k4 * ir2 + c.k5 * (T(1) + c.k6 * ir2) - c.k7 * (T(2) - r2 * c.k8)) * DS;
    B = erf_diff * (c.k1 * ir3 - c.k9 * ir5) + c.k10 * ir4 * Ds +
        (-c.k11 * ir4 - c.k5 * ir2 * (T(1) + c.k12 * ir2) - c.k13) * DS;
}

// x - L round(x / L), ties to even (src/correct_velocities.jl:121-127). For
// |x| <= L/2 the correctly rounded quotient is at most 1/2 in magnitude, so
// the rounded multiple is 0 and the reference's expression returns x (up to
// the sign of a zero x, which no later sum or comparison sees): the division
// is only evaluated for separations that may wrap.
template <typename T>
__device__ __forceinline__ T min_image(T x, T L) {
    if (fabs(x) <= T(0.5) * L) return x;
    return sub_rn(x, mul_rn(L, rint_t(div_rn(x, L))));
}

// TPP threads per sorted particle share its 27 neighbour cells (cell q of the
// reference's dz/dy/dx order goes to lane q mod TPP), so that small systems
// still fill the GPU; the lanes' sums are combined by shuffles. Large systems
// use one thread per particle (corr_tpp picks).
// Vs == nullptr: V[:, perm[s]] += dv (the step API, reference semantics).
// Vs != nullptr: V[:, perm[s]] = h3 * Vs[s] + dv (finishes the fused
// interpolation, which left its sums in sorted order in Vs).
inline int corr_tpp(int64_t n_part) { return n_part <= 200000 ? 4 : 1; }

// Self term plus the pair terms of sorted particle s over its 27 neighbour
// cells; lane `sub` of the particle's TPP-lane group takes cells q = sub,
// sub + TPP, ... of the reference's order, and after the shuffles every lane
// of the group holds the group's sum.
template <typename T, int TPP>
__device__ __forceinline__ void pair_velocity(int s, int sub, unsigned group, const vec4<T>* __restrict__ Ys,
                                              const vec4<T>* __restrict__ Fs, const int32_t* __restrict__ off,
                                              const CorrConsts<T>& c, T& v0, T& v1, T& v2) {
    const vec4<T> yn = Ys[s];
    const vec4<T> fn = Fs[s];
    int cx = (int)floor_t(mul_rn(yn.x, c.ic0));
    int cy = (int)floor_t(mul_rn(yn.y, c.ic1));
    int cz = (int)floor_t(mul_rn(yn.z, c.ic2));
    cx = max(0, min(cx, c.m0 - 1));
    cy = max(0, min(cy, c.m1 - 1));
    cz = max(0, min(cz, c.m2 - 1));
    v0 = 0;
    v1 = 0;
    v2 = 0;
    if (sub == 0) {
        v0 = c.self * fn.x;
        v1 = c.self * fn.y;
        v2 = c.self * fn.z;
    }
    auto visit = [&](int nx, int ny, int nz) {
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
    };
    if constexpr (TPP == 1) {
        // the reference's dz / dy / dx loop order
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx)
                    visit(imod(cx + dx, c.m0), imod(cy + dy, c.m1), imod(cz + dz, c.m2));
    } else {
        // cell q of that order goes to lane q mod TPP
        for (int q = sub; q < 27; q += TPP)
            visit(imod(cx + q % 3 - 1, c.m0), imod(cy + (q / 3) % 3 - 1, c.m1), imod(cz + q / 9 - 1, c.m2));
    }
#pragma unroll
    for (int o = 1; o < TPP; o <<= 1) {
        v0 += __shfl_xor_sync(group, v0, o);
        v1 += __shfl_xor_sync(group, v1, o);
        v2 += __shfl_xor_sync(group, v2, o);
    }
}

template <typename T, int TPP>
__global__ void k_correct(int n_part, const vec4<T>* __restrict__ Ys,
                          const vec4<T>* __restrict__ Fs, const int32_t* __restrict__ off,
                          const int32_t* __restrict__ perm, T* __restrict__ V, CorrConsts<T> c,
                          const T* __restrict__ Vs, T h3) {
    const int sub = threadIdx.x % TPP;
    const unsigned group = ((1u << TPP) - 1u) << (lane_id() & ~(TPP - 1));
    const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < (int64_t)n_part * TPP;
         t += nthreads) {
        const int s = (int)(t / TPP);
        T v0, v1, v2;
        pair_velocity<T, TPP>(s, sub, group, Ys, Fs, off, c, v0, v1, v2);
        if (sub == 0) {
            const int64_t n = perm[s];
            if (Vs) {
                V[3 * n] = h3 * Vs[3 * (int64_t)s] + v0;
                V[3 * n + 1] = h3 * Vs[3 * (int64_t)s + 1] + v1;
                V[3 * n + 2] = h3 * Vs[3 * (int64_t)s + 2] + v2;
            } else {
                V[3 * n] += v0;
                V[3 * n + 1] += v1;
                V[3 * n + 2] += v2;
            }
        }
    }
}

// The pair terms alone, dv[3 s + c] in sorted order, for a solve that runs
// them on a second stream beside its grid stages (they need only the sorted
// particles and the cell list); k_finish_velocity then adds the
// interpolation sums, with the same arithmetic as k_correct.
template <typename T, int TPP>
__global__ void k_correct_pairs(int n_part, const vec4<T>* __restrict__ Ys, const vec4<T>* __restrict__ Fs,
                                const int32_t* __restrict__ off, CorrConsts<T> c, T* __restrict__ dv) {
    const int sub = threadIdx.x % TPP;
    const unsigned group = ((1u << TPP) - 1u) << (lane_id() & ~(TPP - 1));
    const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < (int64_t)n_part * TPP;
         t += nthreads) {
        const int s = (int)(t / TPP);
        T v0, v1, v2;
        pair_velocity<T, TPP>(s, sub, group, Ys, Fs, off, c, v0, v1, v2);
        if (sub == 0) {
            dv[3 * (int64_t)s] = v0;
            dv[3 * (int64_t)s + 1] = v1;
            dv[3 * (int64_t)s + 2] = v2;
        }
    }
}

// V[:, perm[s]] = h^3 Vs[s] + dv[s].
template <typename T>
__global__ void k_finish_velocity(int n_part, const int32_t* __restrict__ perm, const T* __restrict__ Vs,
                                  const T* __restrict__ dv, T h3, T* __restrict__ V) {
    const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n_part; s += nthreads) {
        const int64_t n = perm[s];
        V[3 * n] = h3 * Vs[3 * s] + dv[3 * s];
        V[3 * n + 1] = h3 * Vs[3 * s + 1] + dv[3 * s + 1];
        V[3 * n + 2] = h3 * Vs[3 * s + 2] + dv[3 * s + 2];
    }
}

}  // namespace ffcm
