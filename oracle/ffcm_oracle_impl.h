/*
 * Type-generic body of the CPU oracle. Included twice by ffcm_oracle.c, once
 * with FT = float (suffix _f) and once with FT = double (suffix _d).
 *
 * TEST INFRASTRUCTURE ONLY. This is a restatement of the reference Julia
 * package ForceCouplingMethod.jl (the src directory), loop for loop, used by the test
 * suite and by the CPU-baseline leg of bench.py as the checker. Nothing in
 * the product library links or calls it.
 *
 * Layouts follow the reference exactly:
 *   - 3xN Julia matrices (column-major) = N consecutive (x, y, z) triples;
 *   - (M_x, M_y, M_z) Julia arrays (column-major) = x fastest, z slowest;
 *   - index buffers are 1-based as in Julia.
 * Arithmetic is written in the reference's operation order; the file is
 * compiled with -ffp-contract=off so no multiply-add is fused (Julia does
 * not contract either).
 */

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(name, SFX)

/* Julia `mod(x, y)` for floats (rem, then shift by y on a sign mismatch).
 * src/cell_list.jl:26 calls it as `mod.(source, L)`. */
static FT FN(julia_fmod)(FT x, FT y) {
    FT r = (FT)FMOD(x, y);
    if (r == (FT)0) return (FT)COPYSIGN((FT)0, y);
    if ((r > (FT)0) != (y > (FT)0)) return r + y;
    return r;
}

/* src/cell_list.jl:22-31  wrap_positions!(destination, source, L) */
void FN(oracle_wrap_positions)(FT* dst, const FT* src, int64_t N, const FT* L) {
    for (int64_t n = 0; n < N; ++n)
        for (int i = 0; i < 3; ++i)
            dst[3 * n + i] = FN(julia_fmod)(src[3 * n + i], L[i]);
}

/* src/cell_list.jl:222-238  _assign_cells_kernel! */
void FN(oracle_assign_cells)(int32_t* cell_hash, const FT* Y, int64_t N,
                            const FT* inv_cell_size, const int32_t* num_cells) {
    for (int64_t n = 0; n < N; ++n) {
        int32_t c[3];
        for (int i = 0; i < 3; ++i) {
            FT s = Y[3 * n + i] * inv_cell_size[i];
            int32_t v = (int32_t)FLOOR(s);
            if (v > num_cells[i] - 1) v = num_cells[i] - 1;
            c[i] = v;
        }
        cell_hash[n] = c[0] + (c[1] + c[2] * num_cells[1]) * num_cells[0];
    }
}

/* src/cell_list.jl:159-176  _gather_particles_kernel! (original_index 1-based) */
void FN(oracle_gather)(FT* Y_sorted, FT* F_sorted, const FT* Y, const FT* F,
                      const int32_t* original_index, int64_t N) {
    for (int64_t s = 0; s < N; ++s) {
        int64_t n = (int64_t)original_index[s] - 1;
        for (int i = 0; i < 3; ++i) {
            Y_sorted[3 * s + i] = Y[3 * n + i];
            F_sorted[3 * s + i] = F[3 * n + i];
        }
    }
}

/* src/stencil.jl:22-31  _modified_kernel_coefficients(σ, Σ) -> (a0, a2, inv_norm, inv_2Σ²) */
void FN(oracle_modified_kernel_coefficients)(FT sigma, FT Sigma, FT* out4) {
    FT S2 = Sigma * Sigma;
    FT S4 = S2 * S2;
    FT d = sigma * sigma - S2;
    FT a0 = (FT)1 - (FT)3 * d / ((FT)2 * S2);
    FT a2 = d / ((FT)2 * S4);
    FT inv_norm = (FT)1 / (FT)SQRT((FT)2 * (FT)PI_T * S2);
    FT inv_2S2 = (FT)1 / ((FT)2 * S2);
    out4[0] = a0; out4[1] = a2; out4[2] = inv_norm; out4[3] = inv_2S2;
}

/* Anchor round(Y / h) and offset g h - Y of the stencil (src/stencil.jl:97-105),
 * or the Float64 geometry when g_geom_hd is set (see ffcm_oracle.c). */
static int32_t FN(stencil_anchor)(FT y, FT inv_h) {
    if (g_geom_hd > 0) return (int32_t)rint((double)y * (1.0 / g_geom_hd));
    return (int32_t)RINT(y * inv_h);
}
static FT FN(stencil_offset)(int32_t gi, FT y, FT h) {
    if (g_geom_hd > 0) {
        const FT hh = (FT)g_geom_hd;
        const FT hl = (FT)(g_geom_hd - (double)hh);
        return FMA((FT)gi, hh, -y) + (FT)gi * hl;
    }
    return (FT)gi * h - y;
}

/* src/stencil.jl:80-112  _fill_particle_stencil! for one particle.
 * g[axis*MG+k], r2[axis*MG+k], idx[axis*MG+k] (0-based wrapped index). */
static void FN(fill_stencil)(FT* g, FT* r2, int32_t* idx, const FT* Y, FT inv_norm,
                            FT inv_2S2, FT h, FT inv_h, const int32_t* M, int32_t MG) {
    int32_t half = MG / 2;
    for (int i = 0; i < 3; ++i) {
        int32_t j = FN(stencil_anchor)(Y[i], inv_h);
        for (int32_t k = 1; k <= MG; ++k) {
            int32_t off = k - 1 - half;
            int32_t gi = j + off;
            FT x = FN(stencil_offset)(gi, Y[i], h);
            FT x2 = x * x;
            g[i * MG + k - 1] = inv_norm * (FT)EXP(-x2 * inv_2S2);
            r2[i * MG + k - 1] = x2;
            int32_t w = gi % M[i];
            if (w < 0) w += M[i];
            idx[i * MG + k - 1] = w;
        }
    }
}

/* src/spread_forces.jl:73-130  _spread_forces_kernel!
 * f: three (M_x, M_y, M_z) component arrays, contiguous one after another. */
void FN(oracle_spread)(FT* f, const FT* Y_sorted, const FT* F_sorted, int64_t N,
                      FT sigma, FT Sigma, FT h, FT inv_h, const int32_t* M, int32_t MG) {
    int64_t Mtot = (int64_t)M[0] * M[1] * M[2];
    FT* fx = f; FT* fy = f + Mtot; FT* fz = f + 2 * Mtot;
    for (int64_t q = 0; q < 3 * Mtot; ++q) f[q] = (FT)0;
    FT c4[4];
    FN(oracle_modified_kernel_coefficients)(sigma, Sigma, c4);
    FT a0 = c4[0], a2 = c4[1], inv_norm = c4[2], inv_2S2 = c4[3];
    FT* g = (FT*)malloc(sizeof(FT) * 3 * MG);
    FT* r2 = (FT*)malloc(sizeof(FT) * 3 * MG);
    int32_t* idx = (int32_t*)malloc(sizeof(int32_t) * 3 * MG);
    for (int64_t s = 0; s < N; ++s) {
        FT Fn0 = F_sorted[3 * s], Fn1 = F_sorted[3 * s + 1], Fn2 = F_sorted[3 * s + 2];
        FN(fill_stencil)(g, r2, idx, Y_sorted + 3 * s, inv_norm, inv_2S2, h, inv_h, M, MG);
        for (int32_t kz = 0; kz < MG; ++kz) {
            int64_t iz = idx[2 * MG + kz];
            FT gz = g[2 * MG + kz];
            FT r2z = r2[2 * MG + kz];
            for (int32_t ky = 0; ky < MG; ++ky) {
                int64_t iy = idx[MG + ky];
                FT gyz = g[MG + ky] * gz;
                FT r2yz = r2[MG + ky] + r2z;
                int64_t row = (iy + iz * M[1]) * M[0];
                for (int32_t kx = 0; kx < MG; ++kx) {
                    int64_t ix = idx[kx];
                    FT w = (a0 + a2 * (r2[kx] + r2yz)) * g[kx] * gyz;
                    fx[row + ix] += w * Fn0;
                    fy[row + ix] += w * Fn1;
                    fz[row + ix] += w * Fn2;
                }
            }
        }
    }
    free(g); free(r2); free(idx);
}

/* src/interpolate.jl:82-136  _interpolate_velocities_kernel!
 * Writes V[:, original_index[s]] = h^3 * v (overwrite). */
void FN(oracle_interpolate)(FT* V, const FT* u, const FT* Y_sorted, const int32_t* original_index,
                           int64_t N, FT sigma, FT Sigma, FT h, FT inv_h, const int32_t* M,
                           int32_t MG) {
    int64_t Mtot = (int64_t)M[0] * M[1] * M[2];
    const FT* ux = u; const FT* uy = u + Mtot; const FT* uz = u + 2 * Mtot;
    FT c4[4];
    FN(oracle_modified_kernel_coefficients)(sigma, Sigma, c4);
    FT a0 = c4[0], a2 = c4[1], inv_norm = c4[2], inv_2S2 = c4[3];
    FT h3 = h * h * h;
    FT* g = (FT*)malloc(sizeof(FT) * 3 * MG);
    FT* r2 = (FT*)malloc(sizeof(FT) * 3 * MG);
    int32_t* idx = (int32_t*)malloc(sizeof(int32_t) * 3 * MG);
    for (int64_t s = 0; s < N; ++s) {
        FN(fill_stencil)(g, r2, idx, Y_sorted + 3 * s, inv_norm, inv_2S2, h, inv_h, M, MG);
        FT v0 = 0, v1 = 0, v2 = 0;
        for (int32_t kz = 0; kz < MG; ++kz) {
            int64_t iz = idx[2 * MG + kz];
            FT gz = g[2 * MG + kz];
            FT r2z = r2[2 * MG + kz];
            for (int32_t ky = 0; ky < MG; ++ky) {
                int64_t iy = idx[MG + ky];
                FT gyz = g[MG + ky] * gz;
                FT r2yz = r2[MG + ky] + r2z;
                int64_t row = (iy + iz * M[1]) * M[0];
                for (int32_t kx = 0; kx < MG; ++kx) {
                    int64_t ix = idx[kx];
                    FT w = (a0 + a2 * (r2[kx] + r2yz)) * g[kx] * gyz;
                    v0 += w * ux[row + ix];
                    v1 += w * uy[row + ix];
                    v2 += w * uz[row + ix];
                }
            }
        }
        int64_t n = (int64_t)original_index[s] - 1;
        V[3 * n] = h3 * v0;
        V[3 * n + 1] = h3 * v1;
        V[3 * n + 2] = h3 * v2;
    }
    free(g); free(r2); free(idx);
}

/* src/stokes_solve.jl:70-110  _apply_inverse_stokes_kernel!
 * fh: three half-complex arrays of shape (nkx, nky, nkz), interleaved (re, im). */
void FN(oracle_apply_inverse_stokes)(FT* fh, const FT* kx, const FT* ky, const FT* kz,
                                    int64_t nkx, int64_t nky, int64_t nkz, FT mu, FT inv_M) {
    int64_t tot = nkx * nky * nkz;
    FT* fxh = fh; FT* fyh = fh + 2 * tot; FT* fzh = fh + 4 * tot;
    FT inv_mu_M = inv_M / mu;
    for (int64_t iz = 0; iz < nkz; ++iz) {
        FT k3 = kz[iz];
        for (int64_t iy = 0; iy < nky; ++iy) {
            FT k2 = ky[iy];
            for (int64_t ix = 0; ix < nkx; ++ix) {
                FT k1 = kx[ix];
                int64_t q = 2 * (ix + nkx * (iy + nky * iz));
                FT ksq = k1 * k1 + k2 * k2 + k3 * k3;
                if (ksq == (FT)0) {
                    fxh[q] = fxh[q + 1] = 0;
                    fyh[q] = fyh[q + 1] = 0;
                    fzh[q] = fzh[q + 1] = 0;
                    continue;
                }
                FT inv_k2 = (FT)1 / ksq;
                FT scale = inv_mu_M * inv_k2;
                /* dot(k, f̂) for real k: k1*f1 + k2*f2 + k3*f3 per real/imag part */
                FT dre = k1 * fxh[q] + k2 * fyh[q] + k3 * fzh[q];
                FT dim = k1 * fxh[q + 1] + k2 * fyh[q + 1] + k3 * fzh[q + 1];
                FT cre = dre * inv_k2, cim = dim * inv_k2;
                FT nx_re = scale * (fxh[q] - k1 * cre), nx_im = scale * (fxh[q + 1] - k1 * cim);
                FT ny_re = scale * (fyh[q] - k2 * cre), ny_im = scale * (fyh[q + 1] - k2 * cim);
                FT nz_re = scale * (fzh[q] - k3 * cre), nz_im = scale * (fzh[q + 1] - k3 * cim);
                fxh[q] = nx_re; fxh[q + 1] = nx_im;
                fyh[q] = ny_re; fyh[q + 1] = ny_im;
                fzh[q] = nz_re; fzh[q + 1] = nz_im;
            }
        }
    }
}

/* src/correct_velocities.jl:21-27  _self_correction(σ, Σ, a, μ) */
FT FN(oracle_self_correction)(FT sigma, FT Sigma, FT a, FT mu) {
    FT d = sigma * sigma - Sigma * Sigma;
    FT Ssp = Sigma * (FT)SQRT((FT)PI_T);
    FT pi = (FT)PI_T;
    FT S5 = (FT)POW(Sigma, (FT)5);
    return (FT)1 / ((FT)6 * pi * mu * a) - (FT)1 / ((FT)6 * pi * mu * Ssp) +
           d / ((FT)12 * mu * (Ssp * Ssp * Ssp)) -
           (d * d) / ((FT)32 * mu * S5 * (FT)SQRT(pi * pi * pi));
}

/* src/correct_velocities.jl:71-104  _correction_scalars(r, σ, Σ, μ) -> (A, B) */
void FN(oracle_correction_scalars)(FT r, FT sigma, FT Sigma, FT mu, FT* A, FT* B) {
    FT r2 = r * r;
    FT r3 = r * r * r;
    FT r4 = r2 * r2;
    FT r5 = r4 * r;
    FT s2 = sigma * sigma;
    FT s4 = s2 * s2;
    FT S2 = Sigma * Sigma;
    FT S4 = S2 * S2;
    FT d = s2 - S2;
    FT dq = d * d / (FT)4;
    FT pi = (FT)PI_T;
    FT fourpimu = (FT)4 * pi * mu;
    FT eightpimu = (FT)8 * pi * mu;
    FT erf_diff = (FT)ERF(r / ((FT)2 * sigma)) - (FT)ERF(r / ((FT)2 * Sigma));
    FT Ds = (FT)POW((FT)4 * pi * s2, -(FT)3 / (FT)2) * (FT)EXP(-r2 / ((FT)4 * s2));
    FT DS = (FT)POW((FT)4 * pi * S2, -(FT)3 / (FT)2) * (FT)EXP(-r2 / ((FT)4 * S2));
    *A = erf_diff * ((FT)1 / (eightpimu * r) + s2 / (fourpimu * r3)) -
         (FT)2 * s4 / (mu * r2) * Ds +
         ((FT)2 * S4 / (mu * r2) + d / mu * ((FT)1 + (FT)2 * S2 / r2) -
          dq * ((FT)2 - r2 / ((FT)2 * S2)) / ((FT)2 * mu * S2)) * DS;
    *B = erf_diff * ((FT)1 / (eightpimu * r3) - (FT)3 * s2 / (fourpimu * r5)) +
         (FT)6 * s4 / (mu * r4) * Ds +
         (-(FT)6 * S4 / (mu * r4) - d / (mu * r2) * ((FT)1 + (FT)6 * S2 / r2) -
          dq / ((FT)4 * mu * S4)) * DS;
}

/* src/correct_velocities.jl:216-286  _correct_velocities_kernel! (CPU method).
 * cell_start/cell_end are 1-based inclusive; V is accumulated (+=). */
void FN(oracle_correct)(FT* V, const FT* Y_sorted, const FT* F_sorted, const int32_t* cell_start,
                       const int32_t* cell_end, const int32_t* original_index,
                       const int32_t* num_cells, const FT* L, FT sigma, FT Sigma, FT a, FT mu,
                       FT R_c) {
    FT self = FN(oracle_self_correction)(sigma, Sigma, a, mu);
    FT Rc2 = R_c * R_c;
    int32_t mx = num_cells[0], my = num_cells[1], mz = num_cells[2];
    for (int32_t cz = 0; cz < mz; ++cz)
    for (int32_t cy = 0; cy < my; ++cy)
    for (int32_t cx = 0; cx < mx; ++cx) {
        int32_t c = cx + (cy + cz * my) * mx;
        for (int32_t s = cell_start[c]; s <= cell_end[c]; ++s) {
            const FT* Yn = Y_sorted + 3 * (int64_t)(s - 1);
            const FT* Fn = F_sorted + 3 * (int64_t)(s - 1);
            FT v0 = self * Fn[0], v1 = self * Fn[1], v2 = self * Fn[2];
            for (int32_t dz = -1; dz <= 1; ++dz) {
                int32_t nz = ((cz + dz) % mz + mz) % mz;
                for (int32_t dy = -1; dy <= 1; ++dy) {
                    int32_t ny = ((cy + dy) % my + my) % my;
                    for (int32_t dx = -1; dx <= 1; ++dx) {
                        int32_t nx = ((cx + dx) % mx + mx) % mx;
                        int32_t cn = nx + (ny + nz * my) * mx;
                        for (int32_t s2 = cell_start[cn]; s2 <= cell_end[cn]; ++s2) {
                            if (s2 == s) continue;
                            const FT* Ym = Y_sorted + 3 * (int64_t)(s2 - 1);
                            FT x[3];
                            for (int i = 0; i < 3; ++i) {
                                FT t = Yn[i] - Ym[i];
                                x[i] = t - L[i] * (FT)RINT(t / L[i]);
                            }
                            FT rr = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
                            if (!(rr < Rc2)) continue;
                            FT A, B;
                            FN(oracle_correction_scalars)((FT)SQRT(rr), sigma, Sigma, mu, &A, &B);
                            const FT* Fm = F_sorted + 3 * (int64_t)(s2 - 1);
                            FT xF = x[0] * Fm[0] + x[1] * Fm[1] + x[2] * Fm[2];
                            FT bx = B * xF;
                            v0 += A * Fm[0] + bx * x[0];
                            v1 += A * Fm[1] + bx * x[1];
                            v2 += A * Fm[2] + bx * x[2];
                        }
                    }
                }
            }
            int64_t n = (int64_t)original_index[s - 1] - 1;
            V[3 * n] += v0;
            V[3 * n + 1] += v1;
            V[3 * n + 2] += v2;
        }
    }
}

/* ---------------------------------------------------------------------------
 * Adjoint of the mobility product (the reference has no derivative code; this
 * differentiates the forward restatement above, and the test suite pins it
 * with central finite differences of that forward in Float64).
 *
 * For the cotangent lam of V = M(Y) F:
 *   dY_n = h^3 sum_g grad_Y w_n(g) [lam_n . u_g + F_n . psi_g]
 *        + sum_m grad_x [lam_n . T(x) F_m + lam_m . T(x) F_n],  x = Y_n - Y_m
 * with u = L^-1 S F, psi = L^-1 S lam and T(x) = A(r) I + B(r) x x^T.
 * ------------------------------------------------------------------------- */

/* r-derivatives of the pair scalars of src/correct_velocities.jl:71-104,
 * term by term from the expression above (product and chain rules). */
void FN(oracle_correction_scalars_d)(FT r, FT sigma, FT Sigma, FT mu, FT* A, FT* B, FT* dA,
                                     FT* dB) {
    FN(oracle_correction_scalars)(r, sigma, Sigma, mu, A, B);
    FT r2 = r * r, r3 = r2 * r, r4 = r2 * r2, r5 = r4 * r, r6 = r3 * r3;
    FT s2 = sigma * sigma, s4 = s2 * s2, S2 = Sigma * Sigma, S4 = S2 * S2;
    FT d = s2 - S2;
    FT dq = d * d / (FT)4;
    FT pi = (FT)PI_T;
    FT fourpimu = (FT)4 * pi * mu;
    FT eightpimu = (FT)8 * pi * mu;
    FT erf_diff = (FT)ERF(r / ((FT)2 * sigma)) - (FT)ERF(r / ((FT)2 * Sigma));
    FT es = (FT)EXP(-r2 / ((FT)4 * s2)), eS = (FT)EXP(-r2 / ((FT)4 * S2));
    /* d/dr erf(r / (2w)) = exp(-r^2 / (4 w^2)) / (w sqrt(pi)) */
    FT derf = es / (sigma * (FT)SQRT(pi)) - eS / (Sigma * (FT)SQRT(pi));
    FT Ds = (FT)POW((FT)4 * pi * s2, -(FT)3 / (FT)2) * es;
    FT DS = (FT)POW((FT)4 * pi * S2, -(FT)3 / (FT)2) * eS;
    FT dDs = -r / ((FT)2 * s2) * Ds, dDS = -r / ((FT)2 * S2) * DS;
    FT PA = (FT)2 * S4 / (mu * r2) + d / mu * ((FT)1 + (FT)2 * S2 / r2) -
            dq * ((FT)2 - r2 / ((FT)2 * S2)) / ((FT)2 * mu * S2);
    FT dPA = -(FT)4 * S4 / (mu * r3) - (FT)4 * d * S2 / (mu * r3) + dq * r / ((FT)2 * mu * S2 * S2);
    FT PB = -(FT)6 * S4 / (mu * r4) - d / (mu * r2) * ((FT)1 + (FT)6 * S2 / r2) - dq / ((FT)4 * mu * S4);
    FT dPB = (FT)24 * S4 / (mu * r5) + (FT)2 * d / (mu * r3) + (FT)24 * d * S2 / (mu * r5);
    *dA = derf * ((FT)1 / (eightpimu * r) + s2 / (fourpimu * r3)) +
          erf_diff * (-(FT)1 / (eightpimu * r2) - (FT)3 * s2 / (fourpimu * r4)) -
          (FT)2 * s4 / mu * (dDs / r2 - (FT)2 * Ds / r3) + dPA * DS + PA * dDS;
    *dB = derf * ((FT)1 / (eightpimu * r3) - (FT)3 * s2 / (fourpimu * r5)) +
          erf_diff * (-(FT)3 / (eightpimu * r4) + (FT)15 * s2 / (fourpimu * r6)) +
          (FT)6 * s4 / mu * (dDs / r4 - (FT)4 * Ds / r5) + dPB * DS + PB * dDS;
}

/* Grid part of dY (overwrite): one pass over each particle's stencil, with
 * the weight gradient per axis  d w / d Y_i = w_g * x_i * [(a0 + a2 r^2)/Sigma^2 - 2 a2]
 * where w_g = g_x g_y g_z and x = grid point - Y (stencil of src/stencil.jl:80-112). */
void FN(oracle_grad_gather)(FT* dY, const FT* u, const FT* psi, const FT* Y_sorted,
                            const FT* F_sorted, const FT* L_sorted, const int32_t* original_index,
                            int64_t N, FT sigma, FT Sigma, FT h, FT inv_h, const int32_t* M,
                            int32_t MG) {
    int64_t Mtot = (int64_t)M[0] * M[1] * M[2];
    FT c4[4];
    FN(oracle_modified_kernel_coefficients)(sigma, Sigma, c4);
    FT a0 = c4[0], a2 = c4[1], inv_norm = c4[2], inv_2S2 = c4[3];
    FT inv_S2 = (FT)2 * inv_2S2;
    FT h3 = h * h * h;
    FT* g = (FT*)malloc(sizeof(FT) * 3 * MG);
    FT* r2 = (FT*)malloc(sizeof(FT) * 3 * MG);
    FT* xo = (FT*)malloc(sizeof(FT) * 3 * MG);
    int32_t* idx = (int32_t*)malloc(sizeof(int32_t) * 3 * MG);
    int32_t half = MG / 2;
    for (int64_t s = 0; s < N; ++s) {
        const FT* Yn = Y_sorted + 3 * s;
        const FT* Fn = F_sorted + 3 * s;
        const FT* Ln = L_sorted + 3 * s;
        FN(fill_stencil)(g, r2, idx, Yn, inv_norm, inv_2S2, h, inv_h, M, MG);
        for (int i = 0; i < 3; ++i) {
            int32_t j = FN(stencil_anchor)(Yn[i], inv_h);
            for (int32_t k = 0; k < MG; ++k) xo[i * MG + k] = FN(stencil_offset)(j + k - half, Yn[i], h);
        }
        FT d0 = 0, d1 = 0, d2 = 0;
        for (int32_t kz = 0; kz < MG; ++kz)
            for (int32_t ky = 0; ky < MG; ++ky)
                for (int32_t kx = 0; kx < MG; ++kx) {
                    int64_t o = (idx[2 * MG + kz] * (int64_t)M[1] + idx[MG + ky]) * M[0] + idx[kx];
                    FT rr = r2[kx] + r2[MG + ky] + r2[2 * MG + kz];
                    FT gg = g[kx] * g[MG + ky] * g[2 * MG + kz];
                    FT fac = gg * ((a0 + a2 * rr) * inv_S2 - (FT)2 * a2);
                    FT sg = Ln[0] * u[o] + Ln[1] * u[Mtot + o] + Ln[2] * u[2 * Mtot + o] +
                            Fn[0] * psi[o] + Fn[1] * psi[Mtot + o] + Fn[2] * psi[2 * Mtot + o];
                    FT c = fac * sg;
                    d0 += c * xo[kx];
                    d1 += c * xo[MG + ky];
                    d2 += c * xo[2 * MG + kz];
                }
        int64_t n = (int64_t)original_index[s] - 1;
        dY[3 * n] = h3 * d0;
        dY[3 * n + 1] = h3 * d1;
        dY[3 * n + 2] = h3 * d2;
    }
    free(g); free(r2); free(xo); free(idx);
}

/* Pair part of dY (accumulate): the neighbour loop of oracle_correct with
 * grad_x [lam_n.T F_m + lam_m.T F_n]
 *   = (A' P + B' Q) x / r + B [lam_n (x.F_m) + F_m (lam_n.x) + lam_m (x.F_n) + F_n (lam_m.x)],
 * P = lam_n.F_m + lam_m.F_n, Q = (lam_n.x)(x.F_m) + (lam_m.x)(x.F_n). */
void FN(oracle_correct_grad)(FT* dY, const FT* Y_sorted, const FT* F_sorted, const FT* L_sorted,
                             const int32_t* cell_start, const int32_t* cell_end,
                             const int32_t* original_index, const int32_t* num_cells, const FT* L,
                             FT sigma, FT Sigma, FT mu, FT R_c) {
    FT Rc2 = R_c * R_c;
    int32_t mx = num_cells[0], my = num_cells[1], mz = num_cells[2];
    for (int32_t cz = 0; cz < mz; ++cz)
    for (int32_t cy = 0; cy < my; ++cy)
    for (int32_t cx = 0; cx < mx; ++cx) {
        int32_t c = cx + (cy + cz * my) * mx;
        for (int32_t s = cell_start[c]; s <= cell_end[c]; ++s) {
            const FT* Yn = Y_sorted + 3 * (int64_t)(s - 1);
            const FT* Fn = F_sorted + 3 * (int64_t)(s - 1);
            const FT* Ln = L_sorted + 3 * (int64_t)(s - 1);
            FT gr[3] = {0, 0, 0};
            for (int32_t dz = -1; dz <= 1; ++dz) {
                int32_t nz = ((cz + dz) % mz + mz) % mz;
                for (int32_t dy = -1; dy <= 1; ++dy) {
                    int32_t ny = ((cy + dy) % my + my) % my;
                    for (int32_t dx = -1; dx <= 1; ++dx) {
                        int32_t nx = ((cx + dx) % mx + mx) % mx;
                        int32_t cn = nx + (ny + nz * my) * mx;
                        for (int32_t s2 = cell_start[cn]; s2 <= cell_end[cn]; ++s2) {
                            if (s2 == s) continue;
                            const FT* Ym = Y_sorted + 3 * (int64_t)(s2 - 1);
                            FT x[3];
                            for (int i = 0; i < 3; ++i) {
                                FT t = Yn[i] - Ym[i];
                                x[i] = t - L[i] * (FT)RINT(t / L[i]);
                            }
                            FT rr = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
                            if (!(rr < Rc2)) continue;
                            FT r = (FT)SQRT(rr);
                            FT A, B, dA, dB;
                            FN(oracle_correction_scalars_d)(r, sigma, Sigma, mu, &A, &B, &dA, &dB);
                            const FT* Fm = F_sorted + 3 * (int64_t)(s2 - 1);
                            const FT* Lm = L_sorted + 3 * (int64_t)(s2 - 1);
                            FT P = Ln[0] * Fm[0] + Ln[1] * Fm[1] + Ln[2] * Fm[2] +
                                   Lm[0] * Fn[0] + Lm[1] * Fn[1] + Lm[2] * Fn[2];
                            FT lnx = Ln[0] * x[0] + Ln[1] * x[1] + Ln[2] * x[2];
                            FT lmx = Lm[0] * x[0] + Lm[1] * x[1] + Lm[2] * x[2];
                            FT xfm = x[0] * Fm[0] + x[1] * Fm[1] + x[2] * Fm[2];
                            FT xfn = x[0] * Fn[0] + x[1] * Fn[1] + x[2] * Fn[2];
                            FT Q = lnx * xfm + lmx * xfn;
                            FT radial = (dA * P + dB * Q) / r;
                            for (int i = 0; i < 3; ++i)
                                gr[i] += radial * x[i] +
                                         B * (Ln[i] * xfm + Fm[i] * lnx + Lm[i] * xfn + Fn[i] * lmx);
                        }
                    }
                }
            }
            int64_t n = (int64_t)original_index[s - 1] - 1;
            dY[3 * n] += gr[0];
            dY[3 * n + 1] += gr[1];
            dY[3 * n + 2] += gr[2];
        }
    }
}

#undef FN
#undef CAT
#undef CAT_
