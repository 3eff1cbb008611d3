// Steps 1-2: periodic wrap, cell hash, stable counting sort, gather.
//
// Reference: src/cell_list.jl (wrap_positions! :22-31, _assign_cells_kernel!
// :222-238, _build_cell_list_kernel! :64-93, _gather_particles_kernel!
// :159-176). The permutation produced here is bit-identical to the reference's
// serial stable counting sort: a per-cell histogram and exclusive scan give
// the cell ranges, an atomic-cursor scatter groups each cell's particles, and
// one thread per slot moves its particle to its rank (by original index)
// inside the cell, which restores the stable order whatever the occupancy.
#pragma once

#include "common.cuh"

namespace ffcm {

// Cell coordinate floor(y * inv_cell), clamped to [0, m-1]. The multiply is
// a single IEEE rounding (no fusion possible), as in the reference.
template <typename T>
__device__ __forceinline__ int cell_coord(T y, T inv_cell, int m) {
    int c = (int)floor_t(mul_rn(y, inv_cell));
    c = c > m - 1 ? m - 1 : c;
    return c < 0 ? 0 : c;
}

// Fused wrap + hash. Y, Yw: N (x,y,z) triples.
template <typename T>
__global__ void k_wrap_hash(int n_part, const T* __restrict__ Y, T* __restrict__ Yw,
                            int32_t* __restrict__ key, T L0, T L1, T L2, T ic0, T ic1, T ic2,
                            int m0, int m1, int m2, int* __restrict__ err, int do_wrap,
                            int do_hash) {
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < n_part; n += gridDim.x * blockDim.x) {
        T y0, y1, y2;
        if (do_wrap) {
            y0 = Y[3 * (int64_t)n];
            y1 = Y[3 * (int64_t)n + 1];
            y2 = Y[3 * (int64_t)n + 2];
            y0 = julia_fmod(y0, L0);
            y1 = julia_fmod(y1, L1);
            y2 = julia_fmod(y2, L2);
            Yw[3 * (int64_t)n] = y0;
            Yw[3 * (int64_t)n + 1] = y1;
            Yw[3 * (int64_t)n + 2] = y2;
        } else {
            y0 = Yw[3 * (int64_t)n];
            y1 = Yw[3 * (int64_t)n + 1];
            y2 = Yw[3 * (int64_t)n + 2];
        }
        if (do_hash) {
            int c0 = 0, c1 = 0, c2 = 0;
            if (isfinite_t(y0) && isfinite_t(y1) && isfinite_t(y2)) {
                c0 = cell_coord(y0, ic0, m0);
                c1 = cell_coord(y1, ic1, m1);
                c2 = cell_coord(y2, ic2, m2);
            } else {
                atomicOr(err, DEVERR_NONFINITE_POSITION);
            }
            key[n] = c0 + (c1 + c2 * m1) * m0;
        }
    }
}

__global__ void k_count_cells(int n_part, const int32_t* __restrict__ key,
                              int32_t* __restrict__ count) {
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < n_part; n += gridDim.x * blockDim.x)
        atomicAdd(&count[key[n]], 1);
}

// ---- exclusive scan of `count` (length n) into `off` (length n+1) ---------
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ int block_exclusive_scan(int v, int* smem, int* total) {
    // warp inclusive scan
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) smem[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int nw = blockDim.x >> 5;
        int w = lane < nw ? smem[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < nw) smem[lane] = w;
    }
    __syncthreads();
    int warp_prefix = warp > 0 ? smem[warp - 1] : 0;
    *total = smem[(blockDim.x >> 5) - 1];
    __syncthreads();
    return warp_prefix + x - v;
}

__global__ void k_scan_tiles(const int32_t* __restrict__ count, int n, int32_t* __restrict__ tile_sum) {
    __shared__ int smem[32];
    int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    int s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) s += (base + i < n) ? count[base + i] : 0;
    int total;
    block_exclusive_scan(s, smem, &total);
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = total;
}

// Single block: exclusive scan of the tile sums, in place.
__global__ void k_scan_tile_sums(int32_t* __restrict__ tile_sum, int ntiles) {
    __shared__ int smem[32];
    int carry = 0;
    for (int base = 0; base < ntiles; base += blockDim.x) {
        int i = base + threadIdx.x;
        int v = i < ntiles ? tile_sum[i] : 0;
        int total;
        int ex = block_exclusive_scan(v, smem, &total);
        if (i < ntiles) tile_sum[i] = carry + ex;
        carry += total;
    }
}

__global__ void k_scan_apply(const int32_t* __restrict__ count, int n,
                             const int32_t* __restrict__ tile_prefix, int32_t* __restrict__ off) {
    __shared__ int smem[32];
    int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    int s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        v[i] = (base + i < n) ? count[base + i] : 0;
        s += v[i];
    }
    int total;
    int ex = block_exclusive_scan(s, smem, &total) + tile_prefix[blockIdx.x];
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        if (base + i < n) off[base + i] = ex;
        ex += v[i];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) off[n] = ex;
}

// Group each cell's particles at its range (order inside a cell arbitrary).
__global__ void k_scatter_cells(int n_part, const int32_t* __restrict__ key,
                                const int32_t* __restrict__ off, int32_t* __restrict__ cursor,
                                int32_t* __restrict__ slot_of) {
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < n_part; n += gridDim.x * blockDim.x) {
        int c = key[n];
        int s = off[c] + atomicAdd(&cursor[c], 1);
        slot_of[s] = n;
    }
}

// Stable order inside each cell without a per-cell serial sort: slot_of holds
// the cell-grouped particle indices in the arbitrary order of the atomic
// scatter; the particle at slot i moves to off[c] + (the number of particles of
// its cell with a smaller index), which is its place in the reference's stable
// counting sort (src/cell_list.jl:64-93). One thread per slot; the cost is the
// size of the slot's cell, so crowded cells spread over as many threads as
// they hold particles (the threads of a cell read the same indices, served as
// broadcasts). Positions and forces are gathered into vec4 records on the way.
template <typename T>
__global__ void k_rank_gather(int n_part, const int32_t* __restrict__ key, const int32_t* __restrict__ off,
                              const int32_t* __restrict__ slot_of, int32_t* __restrict__ perm,
                              const T* __restrict__ Yw, const T* __restrict__ F, vec4<T>* __restrict__ Ys,
                              vec4<T>* __restrict__ Fs) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_part; i += gridDim.x * blockDim.x) {
        const int n = slot_of[i];
        const int c = key[n];
        const int b = off[c], e = off[c + 1];
        int rank = 0;
        for (int j = b; j < e; ++j) rank += __ldg(slot_of + j) < n ? 1 : 0;
        const int dst = b + rank;
        perm[dst] = n;
        const int64_t n3 = 3 * (int64_t)n;
        Ys[dst] = vec4<T>{Yw[n3], Yw[n3 + 1], Yw[n3 + 2], T(0)};
        if (F) Fs[dst] = vec4<T>{F[n3], F[n3 + 1], F[n3 + 2], T(0)};   // F null: positions only
    }
}

// Re-gather forces only (a further right-hand side on the same positions).
template <typename T>
__global__ void k_gather_forces(int n_part, const int32_t* __restrict__ perm, const T* __restrict__ F,
                                vec4<T>* __restrict__ Fs) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n_part; s += gridDim.x * blockDim.x) {
        const int64_t n = perm[s];
        Fs[s] = vec4<T>{F[3 * n], F[3 * n + 1], F[3 * n + 2], T(0)};
    }
}

}  // namespace ffcm
