/*
 * CPU oracle for the FFCM mobility hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A restatement, in plain C, of the reference Julia package
 * ForceCouplingMethod.jl v0.1.0 (Biofluid-Dynamics-Group/FFCM.jl), following
 * the loops of src/cell_list.jl, src/stencil.jl, src/spread_forces.jl,
 * src/stokes_solve.jl (the per-mode projector), src/interpolate.jl and
 * src/correct_velocities.jl. The FFTs of src/stokes_solve.jl are done by the
 * Python driver (oracle/ffcm_oracle.py) with pocketfft.
 *
 * Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py
 * load this library, always as the checker or the timed CPU stand-in for the
 * reference; the product library never links it.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#define PI_D 3.14159265358979323846

/* Float32 instantiation. T(π) in Julia is Float32(π), the rounding of π. */
/* Stencil geometry (a test option, not the reference): 0 selects the
 * reference's arithmetic in the working precision; otherwise the double
 * spacing hd of the box as the caller gave it: anchors rounded from
 * Y * (1 / hd) in double, offsets fma(g, h_hi, -Y) + g h_lo with
 * h_hi + h_lo = hd in the working precision (the library's
 * FFCM_STENCIL_FLOAT64 mode). */
static double g_geom_hd = 0.0;
void oracle_set_stencil_geometry(double hd) { g_geom_hd = hd; }

#define FT float
#define SFX _f
#define FMOD fmodf
#define COPYSIGN copysignf
#define FLOOR floorf
#define RINT rintf
#define FMA fmaf
#define EXP expf
#define SQRT sqrtf
#define POW powf
#define ERF erff
#define PI_T ((float)PI_D)
#include "ffcm_oracle_impl.h"
#undef FT
#undef SFX
#undef FMOD
#undef COPYSIGN
#undef FLOOR
#undef RINT
#undef FMA
#undef EXP
#undef SQRT
#undef POW
#undef ERF
#undef PI_T

/* Float64 instantiation. */
#define FT double
#define SFX _d
#define FMOD fmod
#define COPYSIGN copysign
#define FLOOR floor
#define RINT rint
#define FMA fma
#define EXP exp
#define SQRT sqrt
#define POW pow
#define ERF erf
#define PI_T PI_D
#include "ffcm_oracle_impl.h"

/* src/cell_list.jl:64-93  _build_cell_list_kernel!: stable counting sort.
 * original_index, cell_start, cell_end are 1-based as in Julia; an empty
 * cell has cell_end = cell_start - 1. */
void oracle_build_cell_list(int32_t* original_index, int32_t* cell_start, int32_t* cell_end,
                            int32_t* scratch, const int32_t* cell_hash, int64_t N,
                            int64_t total) {
    for (int64_t c = 0; c < total; ++c) scratch[c] = 0;
    for (int64_t n = 0; n < N; ++n) scratch[cell_hash[n]] += 1;
    int32_t acc = 1;
    for (int64_t c = 0; c < total; ++c) {
        cell_start[c] = acc;
        acc += scratch[c];
        cell_end[c] = acc - 1;
        scratch[c] = cell_start[c];
    }
    for (int64_t n = 0; n < N; ++n) {
        int32_t c = cell_hash[n];
        original_index[scratch[c] - 1] = (int32_t)(n + 1);
        scratch[c] += 1;
    }
}

/* src/cell_list.jl:258-289  _build_neighbor_map: 13 forward half-shell
 * neighbours per cell, 0-based cell indices. */
void oracle_build_neighbor_map(int32_t* out, const int32_t* num_cells) {
    static const int32_t off[13][3] = {
        {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {-1, 1, 0}, {1, 0, -1}, {1, 1, -1}, {0, 1, -1},
        {-1, 1, -1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}, {-1, 1, 1}, {0, 0, 1}};
    int32_t mx = num_cells[0], my = num_cells[1], mz = num_cells[2];
    for (int32_t cz = 0; cz < mz; ++cz)
    for (int32_t cy = 0; cy < my; ++cy)
    for (int32_t cx = 0; cx < mx; ++cx) {
        int64_t base = 13 * (int64_t)(cx + (cy + cz * my) * mx);
        for (int k = 0; k < 13; ++k) {
            int32_t nx = ((cx + off[k][0]) % mx + mx) % mx;
            int32_t ny = ((cy + off[k][1]) % my + my) % my;
            int32_t nz = ((cz + off[k][2]) % mz + mz) % mz;
            out[base + k] = nx + (ny + nz * my) * mx;
        }
    }
}
