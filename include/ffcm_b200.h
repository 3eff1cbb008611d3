/*
 * libffcm_b200 -- C ABI of the B200 (sm_100a) FFCM mobility library.
 *
 * The library is the device backend of the reference Julia package
 * ForceCouplingMethod.jl (Biofluid-Dynamics-Group/FFCM.jl). Every entry point
 * below replaces one reference function on the hot path; the citation after
 * each declaration names it (file:line inside the reference project). Julia
 * binds these with `ccall`; any other host binds them with its C FFI.
 *
 * Conventions
 *  - Every call returns an int status (FFCM_OK = 0). On failure the message is
 *    available from ffcm_last_error() (thread-local, valid until the next call
 *    on the same thread).
 *  - Scalars are passed as double; for FFCM_FLOAT32 handles the library rounds
 *    them to float exactly once, as Julia's `T(x)` does, so a Float32 caller
 *    passing its Float32 values gets bit-identical derived scalars.
 *  - Particle arrays are the reference's 3xN column-major matrices: N
 *    consecutive (x, y, z) triples of the handle's element type.
 *  - `memory` says whether a pointer is host (FFCM_HOST) or device
 *    (FFCM_DEVICE) memory. Host calls copy through the handle and return after
 *    the result is in host memory; device calls are asynchronous on `stream`.
 *  - `stream` is a cudaStream_t: NULL = the handle's own stream; the
 *    special handles cudaStreamLegacy / cudaStreamPerThread are accepted.
 *    Inside one call the library may fork work onto a second stream of the
 *    handle (the pair correction of a solve, forked from `stream` after the
 *    spread and joined back before the call's last kernel; not while
 *    `stream` is being captured into a CUDA graph), so the call stays
 *    ordered on `stream` as a whole. A handle's first solve times its
 *    correction against its y pass and later solves fork only when the
 *    correction is the shorter by half; FFCM_OVERLAP_PAIRS=0 (never) or 1
 *    (always) in the environment at ffcm_create overrides that.
 *  - Index buffers exchanged through ffcm_get_buffer/ffcm_set_buffer are
 *    1-based, as in the reference (`original_index`, `cell_start`,
 *    `cell_end`); cell hashes are 0-based as in the reference.
 *  - A handle is not re-entrant: one host thread at a time, as the reference
 *    FFCMConfig (src/config.jl:196-215).
 */
#ifndef FFCM_B200_H
#define FFCM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define FFCM_OK 0
#define FFCM_ERR_ARGUMENT 1    /* Julia ArgumentError (src/config.jl:267-312)      */
#define FFCM_ERR_DIMENSION 2   /* Julia DimensionMismatch (src/mobility.jl:29-34) */
#define FFCM_ERR_OOM 3         /* device or host allocation failed                 */
#define FFCM_ERR_CUDA 4        /* CUDA runtime error                                */
#define FFCM_ERR_TIMEOUT 5     /* a bounded device-side wait gave up                */
#define FFCM_ERR_UNSUPPORTED 6 /* valid for the reference, not for this backend     */
#define FFCM_ERR_STATE 7       /* null handle, or a step called out of order        */

/* ---- element types ------------------------------------------------------ */
#define FFCM_FLOAT32 0
#define FFCM_FLOAT64 1

/* ---- fft_planning (src/config.jl:168-172); accepted and validated only ---- */
#define FFCM_FFT_ESTIMATE 0
#define FFCM_FFT_MEASURE 1
#define FFCM_FFT_PATIENT 2

/* ---- memory kinds -------------------------------------------------------- */
#define FFCM_HOST 0
#define FFCM_DEVICE 1

/* ---- buffers reachable by ffcm_get_buffer / ffcm_set_buffer --------------
 * Sizes in elements; T is the handle's element type.                        */
#define FFCM_BUF_Y_WRAPPED 0      /* 3N T    particles.Y_wrapped (src/config.jl:54-61)   */
#define FFCM_BUF_Y_SORTED 1       /* 3N T    particles.Y_sorted                          */
#define FFCM_BUF_F_SORTED 2       /* 3N T    particles.F_sorted                          */
#define FFCM_BUF_CELL_HASH 3      /* N int32 cells.cell_hash, 0-based (src/config.jl:24-31) */
#define FFCM_BUF_ORIGINAL_INDEX 4 /* N int32 cells.original_index, 1-based               */
#define FFCM_BUF_CELL_START 5     /* ncell int32, 1-based inclusive                      */
#define FFCM_BUF_CELL_END 6       /* ncell int32, 1-based inclusive (empty: end=start-1) */
#define FFCM_BUF_FORCE_DENSITY 7  /* 3*Mx*My*Mz T, grid.force_density, x fastest, SoA    */
#define FFCM_BUF_FLUID_VELOCITY 8 /* 3*Mx*My*Mz T, grid.fluid_velocity                   */
#define FFCM_BUF_K_X 9            /* Mx/2+1 T  solver.k_x (src/config.jl:353-356)        */
#define FFCM_BUF_K_Y 10           /* My T      solver.k_y                                */
#define FFCM_BUF_K_Z 11           /* Mz T      solver.k_z                                */
#define FFCM_BUF_NEIGHBOR_MAP 12  /* 13*ncell int32, half-shell map, 0-based, get only
                                     (src/cell_list.jl:258-289)                          */
#define FFCM_BUF_COUNT 13

/* ---- profiling stages (ffcm_profile_end) --------------------------------- */
#define FFCM_STAGE_H2D 0
#define FFCM_STAGE_CELL_LIST 1
#define FFCM_STAGE_SPREAD 2
#define FFCM_STAGE_FFT_X_FWD 3
#define FFCM_STAGE_FFT_Y_FWD 4
#define FFCM_STAGE_FFT_Z_STOKES 5
#define FFCM_STAGE_FFT_Y_INV 6
#define FFCM_STAGE_FFT_X_INV 7
#define FFCM_STAGE_INTERPOLATE 8
#define FFCM_STAGE_CORRECT 9
#define FFCM_STAGE_D2H 10
#define FFCM_STAGE_COUNT 11

typedef struct ffcm_handle ffcm_handle;

/* Message of the last failing call on this thread ("" if none). */
const char* ffcm_last_error(void);

/* Library ABI version (major * 10000 + minor * 100 + patch). */
int ffcm_version(void);

/* Parameter validation of the cold path, no device work.
 * Replaces _validate_config_parameters (src/config.jl:267-312) and the
 * anisotropy check inside _derive_scalars (lines 341-348 of the same file). */
int ffcm_validate_config(int32_t dtype, const double* L, double R_c, int64_t N, double a,
                         double kernel_widths_ratio, const int32_t* num_grid_points,
                         int32_t M_G, double viscosity, int32_t fft_planning,
                         int32_t fft_threads);

/* Derived scalars in the working precision (returned widened to double,
 * exactly). Replaces _derive_scalars (src/config.jl:326-359); lets the Julia
 * side cache them in its FFCMConfig fields. Any output pointer may be NULL. */
int ffcm_derive_scalars(int32_t dtype, const double* L, double R_c, double a,
                        double kernel_widths_ratio, const int32_t* num_grid_points,
                        int32_t* num_cells /*3*/, double* cell_size /*3*/,
                        double* inv_cell_size /*3*/, double* sigma, double* Sigma, double* h,
                        double* inv_h);

/* Build a configuration on `device`: validates, derives scalars, allocates
 * every hot-path buffer and the FFT tables. Replaces the GPU arm of
 * FFCMConfig{T}(...) (src/config.jl:466-546; ext/ForceCouplingMethodCUDAExt/
 * config.jl:19-103). */
int ffcm_create(ffcm_handle** out, int32_t dtype, const double* L, double R_c, int64_t N,
                double a, double kernel_widths_ratio, const int32_t* num_grid_points,
                int32_t M_G, double viscosity, int32_t fft_planning, int32_t fft_threads,
                int32_t device);

/* Release a configuration (finalizer of FFCMConfig). */
int ffcm_destroy(ffcm_handle* h);

/* ---- stencil arithmetic ----------------------------------------------------
 * FFCM_STENCIL_REFERENCE (the default): the stencil anchor j = round(Y inv_h)
 * and the offsets x = T(g) * h - Y are computed in the working precision T, as
 * the reference does (src/stencil.jl:97-105), so Float32 results match the
 * reference's Float32 CPU backend to round-off. Where Y / h lies within a few
 * Float32 ulps of a half-integer, that anchor can differ from the one Float64
 * arithmetic picks (and from the one of the box the caller meant, when L is
 * not representable in Float32), and the truncated M_G-point stencil then
 * covers neighbouring points: at N = 500k, L = 275.6, 512^3 those few dozen
 * particles put the Float32 answer 2.2e-4 (relative L2) from the Float64 one.
 * FFCM_STENCIL_FLOAT64: anchors rounded from the double product Y * (M / L),
 * with L as passed to ffcm_create, and offsets fma(g, h_hi, -Y) + g * h_lo
 * with h_hi + h_lo the double spacing; the weights stay in T. The Float32
 * solve then follows the Float64 one to round-off (3.6e-7 at that size) and
 * no longer matches the reference's Float32 arithmetic (the cell list and its
 * permutation are unchanged). No reference counterpart.
 * The mode applies to every later call on the handle (the environment
 * variable FFCM_STENCIL=float64 sets it at ffcm_create); changing it waits for
 * the handle's stream and drops a pending adjoint checkpoint. */
#define FFCM_STENCIL_REFERENCE 0
#define FFCM_STENCIL_FLOAT64 1
int ffcm_set_stencil(ffcm_handle* h, int32_t mode);
int ffcm_get_stencil(const ffcm_handle* h, int32_t* mode);

/* Particle count, element type and cell count of a handle. */
int ffcm_get_info(const ffcm_handle* h, int64_t* N, int32_t* dtype, int64_t* num_cells_total);

/* ---- launch-shape wisdom --------------------------------------------------
 * The analogue of FFTW wisdom for the reference's `fft_planning = :measure`
 * (src/config.jl:416-423; its cost is the cold path of FFCMConfig): at
 * ffcm_create the library times the variants of its y and z passes and keeps
 * the fastest per (device, precision, grid); later configurations of the same
 * shape in the process reuse it. These entry points carry the choices across
 * processes, as FFTW's wisdom export/import does.
 *
 * ffcm_get_tuning: the variant a handle uses, out[7] = {y kind, y columns per
 * tile, y grid, z kind, z columns per tile, z grid, kx chunk} (-1 for an axis
 * without the power-of-two passes).
 * ffcm_wisdom_export: all choices of this process as text, one line each;
 * writes at most cap bytes including the terminating NUL into buf (buf may be
 * NULL) and returns the full length without the NUL.
 * ffcm_wisdom_import: adds the choices of such text (replacing those of the
 * same key); nothing is imported from text with a malformed line
 * (FFCM_ERR_ARGUMENT). A configuration uses an imported choice only if it
 * names variants that configuration can run; otherwise it times them itself.
 * The key holds the device ordinal and its SM count: wisdom is for the
 * machine that made it, and a line made on another GPU model is not used.
 * Text format: one line per choice, "ffcm-wisdom-2" followed by 13 integers
 * (ordinal, element size, Mx, My, Mz, SM count, then the 7 fields of
 * ffcm_get_tuning). */
int ffcm_get_tuning(const ffcm_handle* h, int32_t* out);
int64_t ffcm_wisdom_export(char* buf, int64_t cap);
int ffcm_wisdom_import(const char* text);

/* The assembled operator V = M^VF(Y) F. Replaces mobility!(V, config, Y, F)
 * (src/mobility.jl:23-45) including its staging seam
 * (ext/ForceCouplingMethodCUDAExt/mobility.jl:10-23). Shapes are Julia's
 * (rows, cols) of V, Y, F; anything but (3, N) is FFCM_ERR_DIMENSION. Y and F
 * are never written; V is overwritten in the caller's original order. */
int ffcm_mobility(ffcm_handle* h, void* V, int64_t v_rows, int64_t v_cols, const void* Y,
                  int64_t y_rows, int64_t y_cols, const void* F, int64_t f_rows,
                  int64_t f_cols, int32_t memory, void* stream);

/* ---- the six steps, for step-isolated parity ----------------------------- */

/* Y_wrapped = mod.(Y, L). Replaces wrap_positions!(Y_wrapped, Y, L)
 * (src/cell_list.jl:22-31). */
int ffcm_wrap_positions(ffcm_handle* h, const void* Y, int32_t memory, void* stream);

/* cell_hash from Y_wrapped. Replaces assign_cells! (src/cell_list.jl:193-238). */
int ffcm_assign_cells(ffcm_handle* h, void* stream);

/* Stable counting sort by cell_hash, cell ranges, and gather of Y_wrapped and
 * F into sorted order. Replaces sort_particles_by_cell!(config, Y_wrapped, F)
 * (src/cell_list.jl:119-176). */
int ffcm_sort_particles_by_cell(ffcm_handle* h, const void* F, int32_t memory, void* stream);

/* force_density from Y_sorted/F_sorted. Replaces spread_forces!
 * (src/spread_forces.jl:17-130). */
int ffcm_spread_forces(ffcm_handle* h, void* stream);

/* fluid_velocity = L^-1 force_density. Replaces stokes_solve!
 * (src/stokes_solve.jl:21-110). */
int ffcm_stokes_solve(ffcm_handle* h, void* stream);

/* V[:, original_index[s]] = h^3 * gather. Replaces interpolate_velocities!
 * (src/interpolate.jl:23-136). V is 3xN. */
int ffcm_interpolate_velocities(ffcm_handle* h, void* V, int32_t memory, void* stream);

/* V += self and pair correction. Replaces correct_velocities!
 * (src/correct_velocities.jl:154-286). V is 3xN. */
int ffcm_correct_velocities(ffcm_handle* h, void* V, int32_t memory, void* stream);

/* ---- fixed-position operator ----------------------------------------------
 * FFCMMobility(config, Y) applied many times (src/mobility.jl:88-155): the
 * positions are wrapped, hashed and sorted once; every apply re-gathers the
 * forces into that order and solves. The results equal ffcm_mobility's. */

/* Fix the positions (Julia 3xN Y) for the following applies. */
int ffcm_set_positions(ffcm_handle* h, const void* Y, int32_t memory, void* stream);
/* V = M(Y) F for the positions of the last ffcm_set_positions; replaces
 * mul!(v, M, f) / M * F. FFCM_ERR_STATE if any other solve or step call ran
 * on the handle since. */
int ffcm_mobility_apply(ffcm_handle* h, void* V, const void* F, int32_t memory, void* stream);

/* ---- resistance problem (conjugate gradients on the operator) -------------
 * Solves M(Y) F = V for F, M the operator of the last ffcm_set_positions,
 * by conjugate gradients run on the device: the whole iteration loop is one
 * CUDA-graph launch (a while node whose condition the device sets), with no
 * host round trip per iteration. Replaces `cg(M, V)` / `cg!(F, M, V)` of a
 * Julia Krylov package on FFCMMobility, which the reference declares
 * symmetric positive definite for this use (src/mobility.jl:161-162).
 * Iteration and stopping rule as IterativeSolvers.jl's cg: stop once
 * |r| <= max(reltol |r0|, abstol) or after maxiter iterations, r0 = V - M F0.
 *   F        3xN: the initial guess F0 when flags has FFCM_CG_INITIAL_GUESS
 *            (else F0 = 0, initially_zero = true); the solution on return
 *   reltol   < 0 selects sqrt(eps(T)), IterativeSolvers' default
 *   maxiter  < 0 selects 3N (size(M, 2)), IterativeSolvers' default
 *   iterations, residual (|r| of the recursion), cg_status (FFCM_CG_*): any
 *            may be NULL.
 * Synchronous on `stream`. FFCM_ERR_STATE without a preceding
 * ffcm_set_positions; the positions stay set for further applies/solves. */
#define FFCM_CG_INITIAL_GUESS 1
#define FFCM_CG_CONVERGED 1
#define FFCM_CG_MAXITER 2
#define FFCM_CG_BREAKDOWN 3 /* p.q <= 0 or non-finite: the operator is not SPD on these inputs */
int ffcm_cg_solve(ffcm_handle* h, void* F, const void* V, int32_t memory, double reltol, double abstol,
                  int32_t maxiter, int32_t flags, int32_t* iterations, double* residual, int32_t* cg_status,
                  void* stream);

/* ---- buffer access (step isolation, as test/cuda/ does) ------------------ */
int64_t ffcm_buffer_bytes(const ffcm_handle* h, int32_t which);
int ffcm_get_buffer(ffcm_handle* h, int32_t which, void* dst, int64_t nbytes, int32_t memory,
                    void* stream);
int ffcm_set_buffer(ffcm_handle* h, int32_t which, const void* src, int64_t nbytes,
                    int32_t memory, void* stream);

/* Wait for the handle's work on `stream` and report any sticky device-side
 * error (non-finite position, a bounded wait that gave up). */
int ffcm_synchronize(ffcm_handle* h, void* stream);

/* ---- batched form ---------------------------------------------------------
 * Many independent suspensions (each one FFCMConfig of the reference), each
 * with nrhs force right-hand sides, solved by one launch of a CUDA graph
 * built on the first call. No reference counterpart: the reference solves
 * one system and one right-hand side per mobility! call; a batch is
 * equivalent to calling mobility!(V[i][r], config[i], Y[i], F[i][r]) for every
 * system i and right-hand side r (src/mobility.jl:23-45).
 *
 * Shared by all systems: dtype, a, kernel_widths_ratio, M_G, viscosity.
 * Per system i: L[3i..3i+2], R_c[i], N[i], num_grid_points[3i..3i+2].
 * Layouts (elements of the handle's type T): system i's positions start at
 * 3 * sum_{j<i} N[j] of Y; its forces and velocities at
 * 3 * nrhs * sum_{j<i} N[j] of F and V, right-hand side r at that offset plus
 * 3 * r * N[i]; each block is the reference's 3xN column-major matrix. */
typedef struct ffcm_batch ffcm_batch;

int ffcm_batch_create(ffcm_batch** out, int32_t dtype, int64_t nsys, const double* L,
                      const double* R_c, const int64_t* N, double a, double kernel_widths_ratio,
                      const int32_t* num_grid_points, int32_t M_G, double viscosity,
                      int32_t nrhs, int32_t device);
int ffcm_batch_destroy(ffcm_batch* b);
/* Solve every system and right-hand side. Host memory: returns with V filled.
 * Device memory: asynchronous on `stream`. */
int ffcm_batch_mobility(ffcm_batch* b, void* V, const void* Y, const void* F, int32_t memory,
                        void* stream);
/* Totals of a batch: particles over all systems, systems, right-hand sides,
 * and the kernels one ffcm_batch_mobility launches (graph nodes). */
int ffcm_batch_get_info(const ffcm_batch* b, int64_t* total_particles, int64_t* nsys,
                        int32_t* nrhs, int64_t* kernels_per_call);

/* ---- adjoint form ---------------------------------------------------------
 * Reverse-mode derivative of V = M(Y) F. No reference counterpart: the
 * reference has no derivative; these are the two halves of a
 * ChainRulesCore.rrule for mobility (src/mobility.jl:23-45), the forward
 * half keeping only the velocity grid u = L^-1 S F (plus the cell list and
 * sorted particles it already holds) and the pullback recomputing stencil
 * weights. All arrays are 3xN in the handle's type. */

/* Forward solve exactly as ffcm_mobility, which also keeps the checkpoint. */
int ffcm_mobility_checkpoint(ffcm_handle* h, void* V, const void* Y, const void* F, int32_t memory,
                             void* stream);
/* Pullback at the cotangent lambda = dJ/dV of the last ffcm_mobility_checkpoint
 * on this handle: dJdF = M lambda (M is symmetric) and
 * dJdY_n = h^3 sum_g grad w_n(g) [lambda_n . u_g + F_n . psi_g]
 *        + sum_m grad_x [lambda_n . T(x) F_m + lambda_m . T(x) F_n],
 * psi = L^-1 S lambda, T the pair correction. FFCM_ERR_STATE if any other
 * solve or step call ran on the handle since the checkpoint. */
int ffcm_adjoint(ffcm_handle* h, void* dJdY, void* dJdF, const void* lambda, int32_t memory, void* stream);
/* J = 0.5 |M(Y) F - V_target|^2 with dJ/dY, dJ/dF and V in one call
 * (checkpointed forward, residual, pullback). J is a double in the same
 * memory space as the arrays. */
int ffcm_objective_gradient(ffcm_handle* h, double* J, void* dJdY, void* dJdF, void* V, const void* Y,
                            const void* F, const void* V_target, int32_t memory, void* stream);

/* ---- one system over several GPUs (z-slab decomposition) -------------------
 * For grids beyond one GPU's memory: R ranks (one process and GPU each) share
 * one system. Rank r holds the z planes [z_begin, z_end) of the grid (whole
 * spread slabs) for the spread, the y passes and the interpolation, and the
 * kx columns [kx_begin, kx_end) of every plane for the z pass and the
 * projector; the particles (24 bytes each) are replicated on every rank. The
 * library never communicates: the host moves the data with its own
 * collectives (NCCL through torch.distributed, MPI, ...) between the calls:
 *
 *   ffcm_dist_forward      cell list, own slabs' spread, y forward; fills the
 *                          send buffer with R equal blocks (block q for rank q)
 *   <all-to-all>           recv block q <- rank q's send block r
 *   ffcm_dist_stokes       z pass + projector on the own kx columns; fills
 *                          the send buffer again
 *   <all-to-all>           the same exchange
 *   ffcm_dist_interpolate  y inverse, own slabs' interpolation into the
 *                          partial buffer (3N, this rank's share)
 *   <all-reduce, sum>      of the partial buffer over the ranks
 *   ffcm_dist_correct      V = h^3 partial + pair correction (every rank
 *                          computes all N velocities)
 *
 * The result equals ffcm_mobility's to round-off (the sums are the same, in
 * another order). No reference counterpart (the reference solves one system
 * per GPU); the ranges below are contiguous and as even as possible.
 * ffcm_dist_partition: ranges[4] = {z_begin, z_end, kx_begin, kx_end} of a
 * rank (host only, no device work). ffcm_dist_buffers: device pointers of the
 * send and receive buffers (R blocks of block_bytes each), of the partial
 * buffer, and the rank's ranges; any output may be NULL. A distributed handle
 * accepts only these calls (and ffcm_get_info, ffcm_destroy, profiling). */
int ffcm_dist_partition(int32_t dtype, const int32_t* num_grid_points, int32_t nranks, int32_t rank,
                        int32_t* ranges);
int ffcm_dist_create(ffcm_handle** out, int32_t dtype, const double* L, double R_c, int64_t N, double a,
                     double kernel_widths_ratio, const int32_t* num_grid_points, int32_t M_G, double viscosity,
                     int32_t nranks, int32_t rank, int32_t device);
int ffcm_dist_buffers(const ffcm_handle* h, void** send, void** recv, int64_t* block_bytes, void** partial,
                      int32_t* ranges);
int ffcm_dist_forward(ffcm_handle* h, const void* Y, const void* F, int32_t memory, void* stream);
int ffcm_dist_stokes(ffcm_handle* h, void* stream);
int ffcm_dist_interpolate(ffcm_handle* h, void* stream);
int ffcm_dist_correct(ffcm_handle* h, void* V, int32_t memory, void* stream);

/* ---- cell-list sort without allocation -------------------------------------
 * No counterpart in the reference. Computes the reference's cell-list buffers
 * (original_index, 1-based; cell_start and cell_end, 1-based inclusive, an
 * empty cell having start = end + 1; src/cell_list.jl:64-93) from a device
 * array of 0-based cell hashes, with the same stable order as
 * ffcm_sort_particles_by_cell. It allocates no memory: its scratch is a fixed
 * array inside the library, so callers that must not allocate per call (a
 * host language that owns the device memory pool, or a program that cannot
 * afford the device-wide synchronisation of cudaFree) can still build cell
 * lists for systems of any N. Limits: ncell <= FFCM_NOALLOC_MAX_CELLS; one
 * scratch per device, so calls that overlap in time on one device race and
 * must be serialised by the caller; the first call on a device sets the
 * scratch up and should come before any stream capture. All pointers are
 * device pointers on the calling thread's current device; the call returns
 * when the sort is complete. A hash outside [0, ncell) gives
 * FFCM_ERR_ARGUMENT. */
#define FFCM_NOALLOC_MAX_CELLS (1 << 21)
int ffcm_sort_cells_noalloc(const int32_t* cell_hash, int64_t N, int32_t ncell, int32_t* original_index,
                            int32_t* cell_start, int32_t* cell_end, void* stream);

/* ---- measurement --------------------------------------------------------- */

/* Start recording CUDA events around every stage of every call. */
int ffcm_profile_begin(ffcm_handle* h);
/* Stop recording; waits for the recorded work and returns, per stage, the
 * summed milliseconds and the number of timed launches (arrays of
 * FFCM_STAGE_COUNT). */
int ffcm_profile_end(ffcm_handle* h, double* stage_ms, int64_t* stage_calls);
/* Number of kernels this handle has launched since creation. */
int64_t ffcm_launch_count(const ffcm_handle* h);

#ifdef __cplusplus
}
#endif

#endif /* FFCM_B200_H */
