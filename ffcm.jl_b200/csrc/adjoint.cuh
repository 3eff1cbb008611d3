// Adjoint form: the vector-Jacobian product of V(Y, F) = M(Y) F with a
// cotangent lambda (for J = 0.5 |V - V_t|^2, lambda = V - V_t).
//
//   dF = M lambda                                    (M is symmetric)
//   dY_n = h^3 sum_g grad_Y w_n(g) [lambda_n . u_g + F_n . psi_g]
//        + sum_m d/dx [lambda_n . T(x) F_m + lambda_m . T(x) F_n],  x = Y_n - Y_m
//
// with u = L^-1 S F (the forward velocity grid, the only checkpoint),
// psi = L^-1 S lambda, w the modified-kernel stencil weight of
// src/spread_forces.jl:121-125, and T = A(r) I + B(r) x x^T the pair
// correction of src/correct_velocities.jl:71-104. The nearest-anchor stencil
// and the cutoff r < R_c are piecewise constant in Y; their jumps carry no
// derivative, as in any automatic differentiation of the reference.
//
// Per axis, with x = g h - Y: d/dY [(a0 + a2 r^2) gx gy gz]
//                             = gx gy gz x [(a0 + a2 r^2) / Sigma^2 - 2 a2].
#pragma once

#include "common.cuh"
#include "correct.cuh"
#include "spread_interp.cuh"

namespace ffcm {

// lambda = V - Vt (caller order) and J += 0.5 sum lambda^2 (double).
template <typename T>
__global__ void k_residual(int n3, const T* __restrict__ V, const T* __restrict__ Vt, T* __restrict__ lam,
                           double* __restrict__ J) {
    __shared__ double red[32];
    double acc = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
        const T d = V[i] - Vt[i];
        lam[i] = d;
        acc += (double)d * (double)d;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        acc = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (threadIdx.x == 0) atomicAdd(J, 0.5 * acc);
    }
}

// Grid part of the pullback: one warp per sorted particle, lanes stride the
// stencil, reading the forward velocity grid u and the adjoint grid psi:
//   dY[:, perm[s]] = h^3 sum_g grad w(g) [lam . u_g + F . psi_g]   (overwrite)
//   dF[:, perm[s]] = h^3 sum_g w(g) psi_g                          (overwrite)
// Shared memory per warp: g[3 M_G], x[3 M_G] (T) and idx[3 M_G] (int).
template <typename T>
__global__ void k_adjoint_gather(int n_part, const vec4<T>* __restrict__ Ys, const vec4<T>* __restrict__ Fs,
                                 const vec4<T>* __restrict__ Ls, const int32_t* __restrict__ perm,
                                 const T* __restrict__ u, const T* __restrict__ psi, T* __restrict__ dY,
                                 T* __restrict__ dF, StencilParams<T> p, T h3) {
    extern __shared__ unsigned char smem_raw[];
    const int warps = blockDim.x >> 5;
    const int w = threadIdx.x >> 5;
    const int MG = p.MG;
    T* base = reinterpret_cast<T*>(smem_raw);
    T* g = base + w * 3 * MG;
    T* xo = base + (warps + w) * 3 * MG;
    int* idx = reinterpret_cast<int*>(base + 2 * warps * 3 * MG) + w * 3 * MG;
    const int64_t plane = (int64_t)p.Mx * p.My * p.Mz;
    const int MG2 = MG * MG, MG3 = MG2 * MG;
    const T inv_S2 = T(2) * p.inv_2S2;
    const T two_a2 = T(2) * p.a2;
    for (int s = blockIdx.x * warps + w; s < n_part; s += gridDim.x * warps) {
        const vec4<T> y = Ys[s], f = Fs[s], l = Ls[s];
        for (int e = lane_id(); e < 3 * MG; e += 32) {
            const int axis = e / MG, k = e - axis * MG;
            const T yy = axis == 0 ? y.x : (axis == 1 ? y.y : y.z);
            const int M = axis == 0 ? p.Mx : (axis == 1 ? p.My : p.Mz);
            const int j = stencil_anchor(p, yy);
            const int gi = j + (k - p.half);
            // one rounding (fused multiply-add) instead of the forward's two:
            // the gradient sums cancel strongly, so the offset's accuracy
            // matters more here than in the forward; with Float64 stencil geometry
            // the forward's own (more accurate) offset
            const T x = p.comp ? stencil_offset(p, gi, yy) : fma_t((T)gi, p.h, -yy);
            g[e] = p.inv_norm * exp_t(-x * x * p.inv_2S2);
            xo[e] = x;
            idx[e] = imod(gi, M);
        }
        __syncwarp();
        T d0 = 0, d1 = 0, d2 = 0, v0 = 0, v1 = 0, v2 = 0;
        for (int q = lane_id(); q < MG3; q += 32) {
            const int kz = q / MG2, rr = q - kz * MG2;
            const int ky = rr / MG, kx = rr - ky * MG;
            const T x0 = xo[kx], x1 = xo[MG + ky], x2 = xo[2 * MG + kz];
            const T poly = p.a0 + p.a2 * (x0 * x0 + x1 * x1 + x2 * x2);
            const T gg = g[kx] * g[MG + ky] * g[2 * MG + kz];
            const int64_t o = ((int64_t)idx[2 * MG + kz] * p.My + idx[MG + ky]) * p.Mx + idx[kx];
            const T p0 = __ldg(psi + o), p1 = __ldg(psi + plane + o), p2 = __ldg(psi + 2 * plane + o);
            const T sg = l.x * __ldg(u + o) + l.y * __ldg(u + plane + o) + l.z * __ldg(u + 2 * plane + o) +
                         f.x * p0 + f.y * p1 + f.z * p2;
            const T c = gg * (poly * inv_S2 - two_a2) * sg;
            const T wgt = gg * poly;
            d0 += c * x0;
            d1 += c * x1;
            d2 += c * x2;
            v0 += wgt * p0;
            v1 += wgt * p1;
            v2 += wgt * p2;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            d0 += __shfl_xor_sync(0xffffffffu, d0, o);
            d1 += __shfl_xor_sync(0xffffffffu, d1, o);
            d2 += __shfl_xor_sync(0xffffffffu, d2, o);
            v0 += __shfl_xor_sync(0xffffffffu, v0, o);
            v1 += __shfl_xor_sync(0xffffffffu, v1, o);
            v2 += __shfl_xor_sync(0xffffffffu, v2, o);
        }
        if (lane_id() == 0) {
            const int64_t n = perm[s];
            dY[3 * n] = h3 * d0;
            dY[3 * n + 1] = h3 * d1;
            dY[3 * n + 2] = h3 * d2;
            dF[3 * n] = h3 * v0;
            dF[3 * n + 1] = h3 * v1;
            dF[3 * n + 2] = h3 * v2;
        }
        __syncwarp();
    }
}

// Constants of the r-derivatives of the pair scalars.
template <typename T>
struct CorrGradConsts {
    T e_s, e_S;       // 1/(sigma sqrt(pi)), 1/(Sigma sqrt(pi)): d/dr erf(r/(2w)) = exp(-r^2/(4w^2))/(w sqrt(pi))
    T ds_s, ds_S;     // 1/(2 sigma^2), 1/(2 Sigma^2): D' = -r D / (2 w^2)
};

// A(r), B(r) and their r-derivatives (regrouped over powers of 1/r as in
// correction_scalars).
template <typename T>
__device__ __forceinline__ void correction_scalars_d(T r, const CorrConsts<T>& c, const CorrGradConsts<T>& cg,
                                                     T& A, T& B, T& dA, T& dB) {
    const T r2 = r * r;
    const T ir = T(1) / r;
    const T ir2 = ir * ir, ir3 = ir2 * ir, ir4 = ir2 * ir2, ir5 = ir4 * ir, ir6 = ir3 * ir3;
    const T es = exp_t(-r2 * c.inv_four_s2), eS = exp_t(-r2 * c.inv_four_S2);
    const T E = erf_t(r * c.inv_two_sigma) - erf_t(r * c.inv_two_Sigma);
    const T dE = cg.e_s * es - cg.e_S * eS;
    const T Ds = c.pref_s * es, DS = c.pref_S * eS;
    const T dDs = -r * cg.ds_s * Ds, dDS = -r * cg.ds_S * DS;
    const T PA = c.k4 * ir2 + c.k5 * (T(1) + c.k6 * ir2) - c.k7 * (T(2) - r2 * c.k8);
    const T PB = -c.k11 * ir4 - c.k5 * ir2 * (T(1) + c.k12 * ir2) - c.k13;
    A = E * (c.k1 * ir + c.k2 * ir3) - c.k3 * ir2 * Ds + PA * DS;
    B = E * (c.k1 * ir3 - c.k9 * ir5) + c.k10 * ir4 * Ds + PB * DS;
    dA = dE * (c.k1 * ir + c.k2 * ir3) + E * (-c.k1 * ir2 - T(3) * c.k2 * ir4) -
         c.k3 * (dDs * ir2 - T(2) * Ds * ir3) +
         (-T(2) * c.k4 * ir3 - T(2) * c.k5 * c.k6 * ir3 + T(2) * c.k7 * c.k8 * r) * DS + PA * dDS;
    dB = dE * (c.k1 * ir3 - c.k9 * ir5) + E * (-T(3) * c.k1 * ir4 + T(5) * c.k9 * ir6) +
         c.k10 * (dDs * ir4 - T(4) * Ds * ir5) +
         (T(4) * c.k11 * ir5 + T(2) * c.k5 * ir3 + T(4) * c.k5 * c.k12 * ir5) * DS + PB * dDS;
}

// Pair part of the pullback, one thread per sorted particle over the 27
// neighbour cells of the forward correction (same pair set):
//   dF[:, perm[s]] += self lam_n + sum_m T(x) lam_m
//   dY[:, perm[s]] += sum_m grad_x [lam_n . T(x) F_m + lam_m . T(x) F_n]
template <typename T, int TPP>
__global__ void k_correct_adjoint(int n_part, const vec4<T>* __restrict__ Ys, const vec4<T>* __restrict__ Fs,
                                  const vec4<T>* __restrict__ Ls, const int32_t* __restrict__ off,
                                  const int32_t* __restrict__ perm, T* __restrict__ dY, T* __restrict__ dF,
                                  CorrConsts<T> c, CorrGradConsts<T> cg) {
    // TPP lanes per particle share its 27 neighbour cells (as in k_correct)
    const int sub = threadIdx.x % TPP;
    const unsigned group = ((1u << TPP) - 1u) << (lane_id() & ~(TPP - 1));
    const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < (int64_t)n_part * TPP;
         t += nthreads) {
        const int s = (int)(t / TPP);
        const vec4<T> yn = Ys[s], fn = Fs[s], ln = Ls[s];
        int cx = (int)floor_t(mul_rn(yn.x, c.ic0));
        int cy = (int)floor_t(mul_rn(yn.y, c.ic1));
        int cz = (int)floor_t(mul_rn(yn.z, c.ic2));
        cx = max(0, min(cx, c.m0 - 1));
        cy = max(0, min(cy, c.m1 - 1));
        cz = max(0, min(cz, c.m2 - 1));
        T g0 = 0, g1 = 0, g2 = 0;
        T v0 = 0, v1 = 0, v2 = 0;
        if (sub == 0) {
            v0 = c.self * ln.x;
            v1 = c.self * ln.y;
            v2 = c.self * ln.z;
        }
        for (int q = sub; q < 27; q += TPP) {
            const int nz = imod(cz + q / 9 - 1, c.m2);
            const int ny = imod(cy + (q / 3) % 3 - 1, c.m1);
            const int nx = imod(cx + q % 3 - 1, c.m0);
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
                const T r = sqrt_t(rr);
                T A, B, dA, dB;
                correction_scalars_d(r, c, cg, A, B, dA, dB);
                const vec4<T> fm = Fs[s2], lm = Ls[s2];
                const T lnx = ln.x * x0 + ln.y * x1 + ln.z * x2;
                const T lmx = lm.x * x0 + lm.y * x1 + lm.z * x2;
                const T xfm = x0 * fm.x + x1 * fm.y + x2 * fm.z;
                const T xfn = x0 * fn.x + x1 * fn.y + x2 * fn.z;
                const T P = ln.x * fm.x + ln.y * fm.y + ln.z * fm.z + lm.x * fn.x + lm.y * fn.y +
                            lm.z * fn.z;
                const T radial = (dA * P + dB * (lnx * xfm + lmx * xfn)) / r;
                g0 += radial * x0 + B * (ln.x * xfm + fm.x * lnx + lm.x * xfn + fn.x * lmx);
                g1 += radial * x1 + B * (ln.y * xfm + fm.y * lnx + lm.y * xfn + fn.y * lmx);
                g2 += radial * x2 + B * (ln.z * xfm + fm.z * lnx + lm.z * xfn + fn.z * lmx);
                const T bl = B * lmx;
                v0 += A * lm.x + bl * x0;
                v1 += A * lm.y + bl * x1;
                v2 += A * lm.z + bl * x2;
            }
        }
#pragma unroll
        for (int o = 1; o < TPP; o <<= 1) {
            g0 += __shfl_xor_sync(group, g0, o);
            g1 += __shfl_xor_sync(group, g1, o);
            g2 += __shfl_xor_sync(group, g2, o);
            v0 += __shfl_xor_sync(group, v0, o);
            v1 += __shfl_xor_sync(group, v1, o);
            v2 += __shfl_xor_sync(group, v2, o);
        }
        if (sub == 0) {
            const int64_t n = perm[s];
            dY[3 * n] += g0;
            dY[3 * n + 1] += g1;
            dY[3 * n + 2] += g2;
            dF[3 * n] += v0;
            dF[3 * n + 1] += v1;
            dF[3 * n + 2] += v2;
        }
    }
}

}  // namespace ffcm
