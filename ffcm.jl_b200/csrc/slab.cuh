// Steps 3 and 5 fused with the x-axis transforms (the fast path of the
// assembled operator): grids whose x length is a power of two (64..2048) and
// stencils of M_G = 8 points per axis.
//
// A block owns a slab: BY x BZ full x-rows of the grid, all three components,
// held in shared memory. The particles whose stencil can touch the slab are
// listed once per solve by k_slab_lists (one warp per slab, over the few
// (cy, cz) rows of cells that can reach it, in cell-sorted order, with the
// reference's integer anchor arithmetic).
//
//  * k_spread_slab: the list is replayed in windows of SLAB_CAP entries; one
//    thread per entry stores the entry's per-row weights gy gz and r^2 parts
//    (src/stencil.jl:80-112); the window is ordered by the first x point of
//    each stencil (a stable counting sort), and each thread then owns grid
//    points x and gathers F (a0 + a2 r^2) gx gy gz from the entries covering
//    x into registers (src/spread_forces.jl:73-130; gx is evaluated by the
//    one thread that uses it) — no floating-point atomics, deterministic.
//    Each slab row is then x-r2c transformed in shared memory and written
//    straight to the spectrum.
//  * k_interp_slab: the slab's spectrum rows are x-c2r transformed into shared
//    memory; one thread per listed particle gathers its partial velocity over
//    the slab rows from registers (src/interpolate.jl:82-136) and adds it,
//    with an L2 reduction, to a sorted-order velocity buffer that the
//    correction kernel finishes (h^3 scale, correction, scatter to the
//    caller's order).
//
// A slab whose list did not fit its capacity is scanned by the slab kernel
// itself (same candidates, same order).
#pragma once

#include "bulk_copy.cuh"
#include "common.cuh"
#include "fft_pow2.cuh"
#include "spread_interp.cuh"

namespace ffcm {

constexpr int SLAB_MG = 8;        // stencil width of the fused path
constexpr int SLAB_CAP = 128;     // entries per spread window (shared memory)
constexpr int SLAB_PAIRMAX = 512; // cell rows one slab may scan

struct SlabGeom {
    int m0, m1, m2;   // cell grid
    double cs1, cs2;  // cell sizes (y, z)
    double h;         // grid spacing
    int nty, ntz;     // slabs along y and z (z: the slabs this grid holds)
    int lcap;         // capacity of a slab's stored particle list
    // z slabs [zs0, zs0 + ntz) of the grid, held as mz_loc z planes of the
    // spectrum (one GPU: zs0 = 0, mz_loc = Mz; a rank of a z-slab decomposition
    // holds its own planes only)
    int zs0, mz_loc;
};

// Row pitch (in T) of a slab row: holds Mx reals and, during the FFT, the
// padded exchange of Mx/2 complex values; pitch = 8 (mod 32) spreads the
// 8-wide x runs of 4 consecutive rows over 32 distinct banks.
__host__ __device__ constexpr int slab_pitch(int Mx) {
    return ((2 * padded_len(Mx / 2) + 23) / 32) * 32 + 8;
}

// Slab shape per element type and x length (3*BY*BZ rows in shared memory).
template <typename T, int H>
struct SlabShape {
    static constexpr int BY = sizeof(T) == 4 ? 4 : 2;
    static constexpr int BZ = (2 * H >= 1024) ? 1 : 2;
};

// Range of cell indices (along one axis) that can hold a particle whose
// stencil anchor lies in [lo_anchor, hi_anchor] (unwrapped). The 1e-3 h slack
// covers the Float32 rounding of y / h and of the cell assignment.
__device__ __forceinline__ void cell_span(int lo_anchor, int hi_anchor, double h, double cs, int m,
                                          int& c_lo, int& count) {
    const double ylo = ((double)lo_anchor - 0.5) * h - 1e-3 * h;
    const double yhi = ((double)hi_anchor + 0.5) * h + 1e-3 * h;
    c_lo = (int)floor(ylo / cs);
    const int c_hi = (int)floor(yhi / cs);
    count = c_hi - c_lo + 1;
    if (count >= m) {
        c_lo = 0;
        count = m;
    }
}

// The (cy, cz) cell rows a slab's candidates come from.
struct SlabRows {
    int cy_lo, ny, cz_lo, nz;
};

template <int BY, int BZ>
__device__ __forceinline__ SlabRows slab_rows(const SlabGeom& g, int y0r, int z0r) {
    constexpr int half = SLAB_MG / 2;
    SlabRows r;
    cell_span(y0r - SLAB_MG + 1 + half, y0r + BY - 1 + half, g.h, g.cs1, g.m1, r.cy_lo, r.ny);
    cell_span(z0r - SLAB_MG + 1 + half, z0r + BZ - 1 + half, g.h, g.cs2, g.m2, r.cz_lo, r.nz);
    return r;
}

// First cell of cell row pi (x = 0), pi = iy + ny * iz.
__device__ __forceinline__ int slab_row_cell(const SlabGeom& g, const SlabRows& r, int pi) {
    const int cy = imod(r.cy_lo + pi % r.ny, g.m1);
    const int cz = imod(r.cz_lo + pi / r.ny, g.m2);
    return (cy + cz * g.m1) * g.m0;
}

// a mod M for a in (-M, 2M).
__device__ __forceinline__ int wrap1(int a, int M) { return a < 0 ? a + M : (a >= M ? a - M : a); }

// Bit b set when slab row r0 + b lies in the stencil starting at row s (s is
// anchor - half of a wrapped position, so r0 + b - s lies in (-M, 2M)).
template <int NB>
__device__ __forceinline__ unsigned rows_hit(int s, int r0, int M) {
    unsigned m = 0;
#pragma unroll
    for (int b = 0; b < NB; ++b)
        if (wrap1(r0 + b - s, M) < SLAB_MG) m |= 1u << b;
    return m;
}

// Block-wide exclusive scan of one int per thread (blockDim.x <= 1024).
__device__ __forceinline__ int block_scan(int v, int* sm, int& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sm[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < nw ? sm[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < nw) sm[lane] = w;
    }
    __syncthreads();
    const int pre = (warp > 0 ? sm[warp - 1] : 0) + x - v;
    total = sm[nw - 1];
    __syncthreads();
    return pre;
}

// Anchors and slab-row masks of a particle at y (a wrapped position).
template <typename T, int BY, int BZ>
__device__ __forceinline__ void slab_anchor(const StencilParams<T>& p, const vec4<T>& y, int y0r, int z0r,
                                            int& sx, int& sy, int& sz, unsigned& m) {
    constexpr int half = SLAB_MG / 2;
    sx = stencil_anchor(p, y.x) - half;
    sy = stencil_anchor(p, y.y) - half;
    sz = stencil_anchor(p, y.z) - half;
    const unsigned my = rows_hit<BY>(sy, y0r, p.My);
    const unsigned mz = rows_hit<BZ>(sz, z0r, p.Mz);
    m = (my && mz) ? (my | (mz << 8)) : 0u;
}

// Gaussian factor and squared offset of stencil point g along one axis, with
// the reference's x = g h - Y (src/stencil.jl:80-112; stencil_offset).
template <typename T>
__device__ __forceinline__ void axis_weight(const StencilParams<T>& p, int g, T y, T& gw, T& r2) {
    const T x = stencil_offset(p, g, y);
    r2 = mul_rn(x, x);
    gw = p.inv_norm * exp_t(-r2 * p.inv_2S2);
}

// Per slab row r = d * BY + b: gy gz and r2y + r2z of a particle (zero for
// rows the particle does not reach; the mask skips those).
template <typename T, int BY, int BZ>
__device__ __forceinline__ void row_weights(const StencilParams<T>& p, const vec4<T>& y, int sy, int sz,
                                            unsigned m, int y0r, int z0r, T (&gyz)[BY * BZ],
                                            T (&r2yz)[BY * BZ]) {
    T gy[BY], r2y[BY], gz[BZ], r2z[BZ];
#pragma unroll
    for (int b = 0; b < BY; ++b) {
        gy[b] = T(0);
        r2y[b] = T(0);
        if ((m >> b) & 1u) axis_weight(p, sy + wrap1(y0r + b - sy, p.My), y.y, gy[b], r2y[b]);
    }
#pragma unroll
    for (int d = 0; d < BZ; ++d) {
        gz[d] = T(0);
        r2z[d] = T(0);
        if ((m >> (8 + d)) & 1u) axis_weight(p, sz + wrap1(z0r + d - sz, p.Mz), y.z, gz[d], r2z[d]);
    }
#pragma unroll
    for (int d = 0; d < BZ; ++d)
#pragma unroll
        for (int b = 0; b < BY; ++b) {
            gyz[d * BY + b] = gy[b] * gz[d];
            r2yz[d * BY + b] = r2y[b] + r2z[d];
        }
}

// Per-slab particle lists, one warp per slab: the candidates (particles of
// the slab's cell rows, in sorted order) are tested with the same integer
// anchor arithmetic as the slab kernels and the touching ones appended, in
// candidate order, with a warp ballot. lists[slab][0, lcap), counts[slab]
// (-1 when the list did not fit; the slab kernels then scan for themselves).
template <typename T, int BY, int BZ>
__global__ void k_slab_lists(const vec4<T>* __restrict__ Ys, const int32_t* __restrict__ off,
                             StencilParams<T> p, SlabGeom g, int* __restrict__ lists, int* __restrict__ counts) {
    const int lane = threadIdx.x & 31;
    const int slab = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    if (slab >= g.nty * g.ntz) return;   // whole warps leave together
    const int y0r = (slab % g.nty) * BY, z0r = (slab / g.nty + g.zs0) * BZ;
    const SlabRows rows = slab_rows<BY, BZ>(g, y0r, z0r);
    int* out = lists + (int64_t)slab * g.lcap;
    const unsigned lt = (1u << lane) - 1u;
    int total = 0;
    for (int pi = 0; pi < rows.ny * rows.nz; ++pi) {
        const int c0 = slab_row_cell(g, rows, pi);
        const int sb = off[c0], se = off[c0 + g.m0];
        for (int b = sb; b < se; b += 32) {
            const int s = b + lane;
            unsigned m = 0;
            if (s < se) {
                int sx, sy, sz;
                slab_anchor<T, BY, BZ>(p, Ys[s], y0r, z0r, sx, sy, sz, m);
            }
            const unsigned bal = __ballot_sync(0xffffffffu, m != 0);
            if (m) {
                const int pos = total + __popc(bal & lt);
                if (pos < g.lcap) out[pos] = s;
            }
            total += __popc(bal);
        }
    }
    if (lane == 0) counts[slab] = total <= g.lcap ? total : -1;
}

// n values of T from / to shared memory in 16-byte loads and stores
// (p 16-byte aligned, n * sizeof(T) a multiple of 16).
template <typename T, int n>
__device__ __forceinline__ void load16(const T* p, T (&v)[n]) {
    if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (int q = 0; q < n / 4; ++q) {
            const float4 c = reinterpret_cast<const float4*>(p)[q];
            v[4 * q] = c.x; v[4 * q + 1] = c.y; v[4 * q + 2] = c.z; v[4 * q + 3] = c.w;
        }
    } else {
#pragma unroll
        for (int q = 0; q < n / 2; ++q) {
            const double2 c = reinterpret_cast<const double2*>(p)[q];
            v[2 * q] = c.x; v[2 * q + 1] = c.y;
        }
    }
}
template <typename T, int n>
__device__ __forceinline__ void store16(T* p, const T (&v)[n]) {
    if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (int q = 0; q < n / 4; ++q)
            reinterpret_cast<float4*>(p)[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    } else {
#pragma unroll
        for (int q = 0; q < n / 2; ++q) reinterpret_cast<double2*>(p)[q] = make_double2(v[2 * q], v[2 * q + 1]);
    }
}

// One window of the spread: per entry the first x point of its stencil, the
// slab rows it reaches, its x position, force, and per-row weight parts.
template <typename T, int BY, int BZ, int H>
struct SpreadWin {
    static constexpr int NRP = BY * BZ;
    // per entry, read with 16-byte loads: gy gz of each slab row, then
    // gy gz (r2y + r2z) of each row, then one 16-byte pad, so that the
    // entries of a quarter-warp's loads start in distinct bank groups
    static constexpr int WYZ = 2 * NRP + 16 / (int)sizeof(T);
    static_assert((2 * NRP * sizeof(T)) % 16 == 0, "rows of an entry fill whole 16-byte chunks");
    vec4<T> fy[SLAB_CAP];     // the force (x, y, z) and the particle's x position (w)
    T wyz[SLAB_CAP][WYZ];
    int key[SLAB_CAP];        // first x point of the stencil, in [0, Mx)
    unsigned msk[SLAB_CAP];   // y rows hit (bits 0..7) | z rows hit (bits 8..15) | first x + 32768 (16..31)
    unsigned sk[SLAB_CAP];    // sort keys (key << 7 | entry), in sorted order
    int first[2 * H + 1];     // counting-sort bins: entries with key <= v
    int scan[32];
};

// Bytes of the spread window region: the window, or the idle-lane FFT line
// that aliases it, whichever is larger (16-byte multiple).
template <typename T, int BY, int BZ, int H>
__host__ __device__ constexpr size_t spread_win_bytes() {
    return ((sizeof(SpreadWin<T, BY, BZ, H>) > (size_t)padded_len(H) * sizeof(cplx<T>)
                 ? sizeof(SpreadWin<T, BY, BZ, H>)
                 : (size_t)padded_len(H) * sizeof(cplx<T>)) + 15) / 16 * 16;
}

template <typename T, int BY, int BZ, int H>
__device__ __forceinline__ void spread_put(const StencilParams<T>& p, SpreadWin<T, BY, BZ, H>& W, int i,
                                           const vec4<T>& y, const vec4<T>& f, int sx, int sy, int sz,
                                           unsigned m, int y0r, int z0r) {
    constexpr int NRP = BY * BZ;
    W.key[i] = wrap1(sx, 2 * H);
    W.msk[i] = m | ((unsigned)(sx + 32768) << 16);   // the stencil's first x point, offset into bits 16..31
    W.fy[i] = vec4<T>{f.x, f.y, f.z, y.x};
    T gyz[NRP], r2yz[NRP];
    row_weights<T, BY, BZ>(p, y, sy, sz, m, y0r, z0r, gyz, r2yz);
    T w[2 * NRP];
#pragma unroll
    for (int r = 0; r < NRP; ++r) {
        w[r] = gyz[r];
        w[NRP + r] = gyz[r] * r2yz[r];
    }
    store16<T, 2 * NRP>(&W.wyz[i][0], w);
}

// x-r2c of every row of a spread slab (3 BY BZ rows of Mx reals, pitch P, in
// shared memory), written straight to the spectrum rows (c, z0r + d, y0r + b).
// `dummy` is a scratch line of padded_len(H) complex values for idle lanes of
// the generic path. All threads of the block call it after a barrier.
template <typename T, int H, int BY, int BZ>
__device__ __forceinline__ void slab_x_r2c(T* acc, cplx<T>* __restrict__ spec, int hxp,
                                           const StencilParams<T>& p, const cplx<T>* tw, cplx<T>* dummy,
                                           int y0r, int zl0, int mz_loc) {
    constexpr int Mx = 2 * H, P = slab_pitch(Mx), NRP = BY * BZ, ROWS = 3 * NRP;
    (void)Mx;
    if constexpr (sizeof(T) == 4 && (H == 64 || H == 128 || H == 256)) {
        // x lengths 128..512: L = H / 16 threads per row with 16 values each,
        // 32 / L rows per warp (ROWS is a multiple of 32 / L, so a warp's rows
        // are all present or all absent); the row is its own exchange scratch;
        // the r2c split takes Z[H - k] from the partner lane by shuffle
        constexpr int L = H / 16;
        static_assert(ROWS % (32 / L) == 0, "a warp's rows must be all present or all absent");
        static_assert(2 * 16 * (L + 1) <= P, "the exchange scratch must fit a slab row");
        const int t = threadIdx.x & (L - 1);
        for (int r = (int)(threadIdx.x / L); r < ROWS; r += (int)(blockDim.x / L)) {
            cplx<T>* rowc = reinterpret_cast<cplx<T>*>(acc + r * P);
            cplx<T> v[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) v[q] = rowc[t + L * q];
            fft_16xL<T, L>(v, t, rowc, tw, 2, false);
            const int c = r / NRP, bd = r % NRP;
            const int b = bd % BY, d = bd / BY;
            cplx<T>* dst = spec + (((int64_t)c * mz_loc + zl0 + d) * p.My + y0r + b) * hxp;
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int k = t + L * q;
                const cplx<T> other = shfl_seg<T, L>(v[15 - q], (L - t) & (L - 1));
                const cplx<T> Zk = v[q];
                const cplx<T> Zc = cconj(t == 0 ? v[(16 - q) & 15] : other);
                const cplx<T> S = cadd(Zk, Zc), D = cmul(tw[k], csub(Zk, Zc));
                dst[k] = cplx<T>{T(0.5) * (S.x + D.y), T(0.5) * (S.y - D.x)};
            }
            if (t == 0) dst[H] = cplx<T>{v[0].x - v[0].y, T(0)};
        }
        return;
    }
    // x r2c of every slab row (H/8 threads per row), output straight to spec.
    // A row that fits one warp is transformed with warp-level synchronisation
    // only (rows are disjoint between warps; idle lanes exchange through a
    // scratch line whose contents are never used).
    constexpr int TPL = H / 8, Q = H / 8;
    constexpr bool WARP = TPL <= 32;
    const int lines_per_round = blockDim.x / TPL;
    const int lr = threadIdx.x / TPL, j = threadIdx.x - lr * TPL;
    for (int r0 = 0; r0 < ROWS; r0 += lines_per_round) {
        const int r = r0 + lr;
        const bool active = r < ROWS && lr < lines_per_round;
        cplx<T>* rowc = reinterpret_cast<cplx<T>*>(acc + (active ? r : 0) * P);
        cplx<T> v[8];
#pragma unroll
        for (int qq = 0; qq < 8; ++qq) v[qq] = active ? rowc[j + qq * Q] : cplx<T>{T(0), T(0)};
        Exchange<T> ex{active ? rowc : dummy, 0, 1};
        fft_line_regs<T, H, WARP>(v, j, ex, tw, 2, false);
        if (WARP) __syncwarp(); else __syncthreads();
        if (active) {
#pragma unroll
            for (int qq = 0; qq < 8; ++qq) ex.at(j + qq * Q) = v[qq];
        }
        if (WARP) __syncwarp(); else __syncthreads();
        if (active) {
            const int c = r / NRP, bd = r % NRP;
            const int b = bd % BY, d = bd / BY;
            cplx<T>* dst = spec + (((int64_t)c * mz_loc + zl0 + d) * p.My + y0r + b) * hxp;
#pragma unroll
            for (int qq = 0; qq < 8; ++qq) {
                const int k = j + qq * Q;
                const cplx<T> Zk = v[qq];
                const cplx<T> Zc = cconj(ex.at((H - k) & (H - 1)));
                const cplx<T> S = cadd(Zk, Zc), D = cmul(tw[k], csub(Zk, Zc));
                dst[k] = cplx<T>{T(0.5) * (S.x + D.y), T(0.5) * (S.y - D.x)};
            }
            if (j == 0) {
                const cplx<T> Z0 = ex.at(0);
                dst[H] = cplx<T>{Z0.x - Z0.y, T(0)};
            }
        }
        if (WARP) __syncwarp(); else __syncthreads();
    }
}

// ---- spread into a slab, then x-r2c straight into the spectrum -----------
template <typename T, int H, int BY, int BZ>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 3 : 2) k_spread_slab(const vec4<T>* __restrict__ Ys,
                                                     const vec4<T>* __restrict__ Fs,
                                                     const int32_t* __restrict__ off,
                                                     cplx<T>* __restrict__ spec, int hxp,
                                                     StencilParams<T> p, SlabGeom g,
                                                     const cplx<T>* __restrict__ twx,
                                                     const int* __restrict__ lists,
                                                     const int* __restrict__ counts) {
    constexpr int Mx = 2 * H, P = slab_pitch(Mx), NRP = BY * BZ, ROWS = 3 * NRP;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* acc = reinterpret_cast<T*>(smem_raw);
    SpreadWin<T, BY, BZ, H>& W = *reinterpret_cast<SpreadWin<T, BY, BZ, H>*>(acc + ROWS * P);
    // exchange line of idle FFT lanes: the window is dead by then
    cplx<T>* dummy = reinterpret_cast<cplx<T>*>(&W);
    // FFT twiddles in shared memory, after the window / idle-lane line
    cplx<T>* tw = reinterpret_cast<cplx<T>*>(reinterpret_cast<unsigned char*>(&W) + spread_win_bytes<T, BY, BZ, H>());
    load_table(tw, twx, Mx);
    const int y0r = blockIdx.x * BY, z0r = (blockIdx.y + g.zs0) * BZ;
    const int cta = blockIdx.x + blockIdx.y * gridDim.x;
    // the first window stores its sums (every grid point of every row is
    // owned by one thread), later windows add; a slab without particles is
    // zeroed after the window loop
    bool fresh = true;
    // Window entries [0, count) are in W; all threads call this after a barrier.
    auto process = [&](int count) {
        // order the window by first x point, stably in entry order: a
        // counting sort (per-key counts, exclusive scan, then one warp places
        // the entries in index order, advancing a per-key cursor). After it
        // fe[v] = number of entries with key <= v, the end of key v's run.
        int* fe = W.first;
        for (int v = threadIdx.x; v < Mx; v += blockDim.x) fe[v] = 0;
        __syncthreads();
        if ((int)threadIdx.x < count) atomicAdd(&fe[W.key[threadIdx.x]], 1);
        __syncthreads();
        {
            constexpr int BPT = (Mx + 255) / 256;   // bins per thread (256 threads)
            int cnt[BPT], sum = 0;
#pragma unroll
            for (int u = 0; u < BPT; ++u) {
                const int b = (int)threadIdx.x * BPT + u;
                cnt[u] = b < Mx ? fe[b] : 0;
                sum += cnt[u];
            }
            int tot;
            int pre = block_scan(sum, W.scan, tot);
#pragma unroll
            for (int u = 0; u < BPT; ++u) {
                const int b = (int)threadIdx.x * BPT + u;
                if (b < Mx) fe[b] = pre;
                pre += cnt[u];
            }
        }
        __syncthreads();
        if (threadIdx.x < 32) {
            const unsigned lane = threadIdx.x;
            for (int c0 = 0; c0 < count; c0 += 32) {
                const int i = c0 + (int)lane;
                const bool act = i < count;
                const int key = act ? W.key[i] : -1 - (int)lane;   // inactive lanes: unique keys
                const unsigned grp = __match_any_sync(0xffffffffu, key);
                const int below = __popc(grp & ((1u << lane) - 1u));
                const int pos = act ? fe[key] + below : 0;
                __syncwarp();
                if (act && below == __popc(grp) - 1) fe[key] += __popc(grp);
                if (act) W.sk[pos] = ((unsigned)key << 7) | (unsigned)i;
                __syncwarp();
            }
        }
        __syncthreads();
        // gather: each thread owns grid points x of all slab rows
        for (int x = threadIdx.x; x < Mx; x += blockDim.x) {
            T a[3][NRP];
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int r = 0; r < NRP; ++r) a[c][r] = T(0);
            const int lo1 = x - SLAB_MG + 1;
            // entries whose stencil starts in [lo1, x] (periodic in x)
            for (int part = 0; part < 2; ++part) {
                int kb, ke;
                if (part == 0) {
                    kb = lo1 > 0 ? fe[lo1 - 1] : 0;
                    ke = fe[x];
                } else {
                    if (lo1 >= 0) break;
                    kb = fe[Mx + lo1 - 1];
                    ke = fe[Mx - 1];
                }
                for (int kk = kb; kk < ke; ++kk) {
                    const unsigned v = W.sk[kk];
                    const int i = (int)(v & 127u);
                    int e = x - (int)(v >> 7);
                    if (e < 0) e += Mx;
                    const vec4<T> fy = W.fy[i];
                    const T y0 = fy.w;
                    const unsigned m = W.msk[i];
                    const int gx0 = (int)(m >> 16) - 32768;
                    T gxe, r2xe;
                    axis_weight(p, gx0 + e, y0, gxe, r2xe);
                    // (a0 + a2 (r2x + r2yz)) gx gyz = [gx (a0 + a2 r2x)] gyz + [a2 gx] [gyz r2yz]
                    const T wa = gxe * (p.a0 + p.a2 * r2xe), wc = p.a2 * gxe;
                    const T f0 = fy.x, f1 = fy.y, f2 = fy.z;
                    T w[2 * NRP];
                    load16<T, 2 * NRP>(&W.wyz[i][0], w);
                    // rows the entry does not reach carry gyz = dyz = 0 and add nothing
#pragma unroll
                    for (int d = 0; d < BZ; ++d)
#pragma unroll
                        for (int b = 0; b < BY; ++b) {
                            const int r = d * BY + b;
                            const T wgt = wa * w[r] + wc * w[NRP + r];
                            a[0][r] += wgt * f0;
                            a[1][r] += wgt * f1;
                            a[2][r] += wgt * f2;
                        }
                }
            }
            if (fresh) {
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int r = 0; r < NRP; ++r) acc[(c * NRP + r) * P + x] = a[c][r];
            } else {
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int r = 0; r < NRP; ++r) acc[(c * NRP + r) * P + x] += a[c][r];
            }
        }
        fresh = false;
    };
    const int stored = counts[cta];
    if (stored >= 0) {
        const int* glist = lists + (int64_t)cta * g.lcap;
        for (int w0 = 0; w0 < stored; w0 += SLAB_CAP) {
            const int n = min(SLAB_CAP, stored - w0);
            if ((int)threadIdx.x < n) {
                const int s = glist[w0 + threadIdx.x];
                const vec4<T> y = Ys[s];
                int sx, sy, sz;
                unsigned m;
                slab_anchor<T, BY, BZ>(p, y, y0r, z0r, sx, sy, sz, m);
                spread_put(p, W, (int)threadIdx.x, y, Fs[s], sx, sy, sz, m, y0r, z0r);
            }
            __syncthreads();
            process(n);
            __syncthreads();
        }
    } else {
        // the list overflowed: scan the candidates in chunks of SLAB_CAP and
        // compact the touching ones into windows, in candidate order
        const SlabRows rows = slab_rows<BY, BZ>(g, y0r, z0r);
        int count = 0;
        for (int pi = 0; pi < rows.ny * rows.nz; ++pi) {
            const int c0 = slab_row_cell(g, rows, pi);
            const int sb = off[c0], se = off[c0 + g.m0];
            for (int b = sb; b < se; b += SLAB_CAP) {
                const int s = b + (int)threadIdx.x;
                unsigned m = 0;
                int sx = 0, sy = 0, sz = 0;
                vec4<T> y{};
                if ((int)threadIdx.x < SLAB_CAP && s < se) {
                    y = Ys[s];
                    slab_anchor<T, BY, BZ>(p, y, y0r, z0r, sx, sy, sz, m);
                }
                int tot;
                const int pre = block_scan(m ? 1 : 0, W.scan, tot);
                if (count + tot > SLAB_CAP) {   // block-uniform
                    process(count);
                    __syncthreads();
                    count = 0;
                }
                if (m) spread_put(p, W, count + pre, y, Fs[s], sx, sy, sz, m, y0r, z0r);
                count += tot;
                __syncthreads();
            }
        }
        if (count > 0) process(count);
        __syncthreads();
    }
    if (fresh) {   // no particle reaches the slab (block-uniform)
        for (int i = threadIdx.x; i < ROWS * P; i += blockDim.x) acc[i] = T(0);
        __syncthreads();
    }
    slab_x_r2c<T, H, BY, BZ>(acc, spec, hxp, p, tw, dummy, y0r, z0r - g.zs0 * BZ, g.mz_loc);
}

// ---- x-c2r of a slab into shared memory, then gather partial velocities ----
// Each slab adds its partial sums into Vs[3 s + c] (sorted order, zeroed
// beforehand); the correction kernel finishes V[:, perm[s]] = h^3 Vs[s] + dv.
// Bytes of a spectrum row copied into a slab row: H + 1 complex values,
// rounded up to 16 bytes (the spectrum pitch and the slab pitch hold them).
template <typename T, int H>
__host__ __device__ constexpr unsigned slab_row_copy_bytes() {
    return (unsigned)(((H + 1) * sizeof(cplx<T>) + 15) / 16 * 16);
}

template <typename T, int H, int BY, int BZ>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 3 : 2) k_interp_slab(const vec4<T>* __restrict__ Ys,
                                                     const int32_t* __restrict__ off,
                                                     const cplx<T>* __restrict__ spec, int hxp,
                                                     T* __restrict__ Vs, StencilParams<T> p,
                                                     SlabGeom g, const cplx<T>* __restrict__ twx,
                                                     const int* __restrict__ lists,
                                                     const int* __restrict__ counts, int* __restrict__ err) {
    constexpr int Mx = 2 * H, P = slab_pitch(Mx), NRP = BY * BZ, ROWS = 3 * NRP;
    constexpr unsigned RB = slab_row_copy_bytes<T, H>();
    static_assert(RB <= P * sizeof(T), "a spectrum row must fit a slab row");
    static_assert((P * sizeof(T)) % 16 == 0, "slab rows must start on 16-byte boundaries");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar[2];
    // rows of the first transform round of the 16 x L path (256 / L); when
    // they are fewer than the slab's, the rest arrive on a second barrier and
    // land while the first round runs
    constexpr bool R16 = sizeof(T) == 4 && (H == 64 || H == 128 || H == 256);
    constexpr int R1 = R16 && 256 / (H / 16) < ROWS ? 256 / (H / 16) : ROWS;
    T* acc = reinterpret_cast<T*>(smem_raw);
    cplx<T>* dummy = reinterpret_cast<cplx<T>*>(acc + ROWS * P);
    cplx<T>* tw = dummy + padded_len(H);   // FFT twiddles in shared memory
    load_table(tw, twx, Mx);
    const int y0r = blockIdx.x * BY, z0r = (blockIdx.y + g.zs0) * BZ;
    const int zl0 = z0r - g.zs0 * BZ;   // first z plane of the slab in the planes held
    const int cta = blockIdx.x + blockIdx.y * gridDim.x;
    // the slab's spectrum rows arrive by bulk copies, rows [0, R1) on bar[0]
    // and the rest on bar[1] (row starts are 16-byte aligned: the spectrum
    // pitch is a multiple of 128 bytes)
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_arrive_expect(&bar[0], R1 * RB);
        if (R1 < ROWS) mbar_arrive_expect(&bar[1], (ROWS - R1) * RB);
        for (int r = 0; r < ROWS; ++r) {
            const int c = r / NRP, bd = r % NRP;
            const cplx<T>* src = spec + (((int64_t)c * g.mz_loc + zl0 + bd / BY) * p.My + y0r + bd % BY) * hxp;
            bulk_load(acc + r * P, src, RB, r < R1 ? &bar[0] : &bar[1]);
        }
    }
    __syncthreads();
    // Block-uniform wait for barrier k: if the copies did not finish, report,
    // give all of them one more bounded chance to land in this block's shared
    // memory, and tell the caller to leave.
    auto landed = [&](int k) -> bool {
        const bool ok = mbar_wait_bounded(&bar[k], 0, 1 << 22);
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) atomicOr(err, DEVERR_COPY_TIMEOUT);
            mbar_wait_bounded(&bar[0], 0, 1 << 22);
            if (R1 < ROWS) mbar_wait_bounded(&bar[1], 0, 1 << 22);
            return false;
        }
        return true;
    };
    if (!landed(0)) return;
    if constexpr (R16) {
        // x lengths 128..512: L = H / 16 threads per row (see the spread)
        constexpr int L = H / 16;
        static_assert(ROWS % (32 / L) == 0, "a warp's rows must be all present or all absent");
        static_assert(2 * 16 * (L + 1) <= P, "the exchange scratch must fit a slab row");
        static_assert(R1 == ROWS || R1 == 256 / L, "the first round covers 256 / L rows");
        const int t = threadIdx.x & (L - 1);
        for (int r0 = 0; r0 < ROWS; r0 += R1) {
            if (r0 > 0 && !landed(1)) return;   // block-uniform
            const int r = r0 + (int)(threadIdx.x / L);
            if (r >= ROWS) continue;   // warp-uniform
            cplx<T>* rowc = reinterpret_cast<cplx<T>*>(acc + r * P);
            cplx<T> v[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int k = t + L * q;
                cplx<T> Xk = rowc[k];
                cplx<T> Xc = rowc[H - k];
                if (k == 0) {
                    Xk.y = T(0);
                    Xc.y = T(0);
                }
                const cplx<T> A = cadd(Xk, cconj(Xc));
                const cplx<T> B = cmul(csub(Xk, cconj(Xc)), cconj(tw[k]));
                v[q] = cadd(A, mul_pi(B));
            }
            fft_16xL<T, L>(v, t, rowc, tw, 2, true);
            __syncwarp();   // the exchange reads of the warp's rows are done
#pragma unroll
            for (int q = 0; q < 16; ++q) rowc[t + L * q] = v[q];   // real row, unpadded
        }
    } else {
    constexpr int TPL = H / 8, Q = H / 8;
    constexpr bool WARP = TPL <= 32;
    const int lines_per_round = blockDim.x / TPL;
    const int lr = threadIdx.x / TPL, j = threadIdx.x - lr * TPL;
    for (int r0 = 0; r0 < ROWS; r0 += lines_per_round) {
        const int r = r0 + lr;
        const bool active = r < ROWS && lr < lines_per_round;
        const cplx<T>* src = reinterpret_cast<const cplx<T>*>(acc + (active ? r : 0) * P);
        cplx<T> v[8];
#pragma unroll
        for (int qq = 0; qq < 8; ++qq) {
            const int k = j + qq * Q;
            cplx<T> Xk = active ? src[k] : cplx<T>{T(0), T(0)};
            cplx<T> Xc = active ? src[H - k] : cplx<T>{T(0), T(0)};
            if (k == 0) {
                Xk.y = T(0);
                Xc.y = T(0);
            }
            const cplx<T> A = cadd(Xk, cconj(Xc));
            const cplx<T> B = cmul(csub(Xk, cconj(Xc)), cconj(tw[k]));
            v[qq] = cadd(A, mul_pi(B));
        }
        cplx<T>* rowc = reinterpret_cast<cplx<T>*>(acc + (active ? r : 0) * P);
        Exchange<T> ex{active ? rowc : dummy, 0, 1};
        fft_line_regs<T, H, WARP>(v, j, ex, tw, 2, true);
        if (WARP) __syncwarp(); else __syncthreads();
        if (active) {
#pragma unroll
            for (int qq = 0; qq < 8; ++qq) rowc[j + qq * Q] = v[qq];   // real row, unpadded
        }
        if (WARP) __syncwarp(); else __syncthreads();
    }
    }
    __syncthreads();
    // one thread per particle: weights in registers, gather over the slab rows
    auto gather = [&](int s) {
        const vec4<T> y = Ys[s];
        int sx, sy, sz;
        unsigned m;
        slab_anchor<T, BY, BZ>(p, y, y0r, z0r, sx, sy, sz, m);
        if (!m) return;
        T gyz[NRP], r2yz[NRP], wa[SLAB_MG], wc[SLAB_MG];
        row_weights<T, BY, BZ>(p, y, sy, sz, m, y0r, z0r, gyz, r2yz);
#pragma unroll
        for (int r = 0; r < NRP; ++r) r2yz[r] *= gyz[r];   // now gy gz (r2y + r2z)
        // (a0 + a2 (r2x + r2yz)) gx gyz = [gx (a0 + a2 r2x)] gyz + [a2 gx] [gyz r2yz]
#pragma unroll
        for (int e = 0; e < SLAB_MG; ++e) {
            T gxe, r2xe;
            axis_weight(p, sx + e, y.x, gxe, r2xe);
            wa[e] = gxe * (p.a0 + p.a2 * r2xe);
            wc[e] = p.a2 * gxe;
        }
        const int x0 = wrap1(sx, Mx);
        T v0 = 0, v1 = 0, v2 = 0;
#pragma unroll
        for (int d = 0; d < BZ; ++d)
#pragma unroll
            for (int b = 0; b < BY; ++b) {
                if (!((m >> b) & (m >> (8 + d)) & 1u)) continue;
                const int r = d * BY + b;
                const T* row = acc + r * P;
#pragma unroll
                for (int e = 0; e < SLAB_MG; ++e) {
                    int x = x0 + e;
                    if (x >= Mx) x -= Mx;
                    const T wgt = wa[e] * gyz[r] + wc[e] * r2yz[r];
                    v0 += wgt * row[x];
                    v1 += wgt * row[NRP * P + x];
                    v2 += wgt * row[2 * NRP * P + x];
                }
            }
        T* vs = Vs + 3 * (int64_t)s;
        atomicAdd(vs, v0);
        atomicAdd(vs + 1, v1);
        atomicAdd(vs + 2, v2);
    };
    const int stored = counts[cta];
    if (stored >= 0) {
        const int* glist = lists + (int64_t)cta * g.lcap;
        for (int t = threadIdx.x; t < stored; t += blockDim.x) gather(glist[t]);
    } else {
        // the list overflowed: every candidate of the slab's cell rows
        const SlabRows rows = slab_rows<BY, BZ>(g, y0r, z0r);
        for (int pi = 0; pi < rows.ny * rows.nz; ++pi) {
            const int c0 = slab_row_cell(g, rows, pi);
            const int se = off[c0 + g.m0];
            for (int s = off[c0] + (int)threadIdx.x; s < se; s += blockDim.x) gather(s);
        }
    }
}

// ---- host-side dispatch over the x length ----------------------------------
template <typename T>
using SpreadSlabKernel = void (*)(const vec4<T>*, const vec4<T>*, const int32_t*, cplx<T>*, int,
                                  StencilParams<T>, SlabGeom, const cplx<T>*, const int*, const int*);
template <typename T>
using ListsKernel = void (*)(const vec4<T>*, const int32_t*, StencilParams<T>, SlabGeom, int*, int*);
template <typename T>
using InterpSlabKernel = void (*)(const vec4<T>*, const int32_t*, const cplx<T>*, int, T*,
                                  StencilParams<T>, SlabGeom, const cplx<T>*, const int*, const int*, int*);

template <typename T>
struct SlabKernels {
    SpreadSlabKernel<T> spread_fused = nullptr;
    InterpSlabKernel<T> interp = nullptr;
    ListsKernel<T> lists = nullptr;
    int BY = 0, BZ = 0;
    size_t smem = 0;          // spread
    size_t smem_interp = 0;   // interpolation
};

template <typename T, int H>
SlabKernels<T> slab_kernels_for() {
    constexpr int BY = SlabShape<T, H>::BY, BZ = SlabShape<T, H>::BZ;
    SlabKernels<T> k;
    k.spread_fused = k_spread_slab<T, H, BY, BZ>;
    k.interp = k_interp_slab<T, H, BY, BZ>;
    k.lists = k_slab_lists<T, BY, BZ>;
    k.BY = BY;
    k.BZ = BZ;
    const size_t slab_bytes = (size_t)3 * BY * BZ * slab_pitch(2 * H) * sizeof(T);
    const size_t line_bytes = (size_t)padded_len(H) * sizeof(cplx<T>);
    const size_t table_bytes = (size_t)2 * H * sizeof(cplx<T>);
    k.smem = slab_bytes + spread_win_bytes<T, BY, BZ, H>() + table_bytes;
    k.smem_interp = slab_bytes + line_bytes + table_bytes;
    return k;
}

// Kernels for x length 2H (H a power of two, 32..1024); false otherwise.
template <typename T>
bool slab_kernels(int H, SlabKernels<T>& k) {
    switch (H) {
        case 32: k = slab_kernels_for<T, 32>(); return true;
        case 64: k = slab_kernels_for<T, 64>(); return true;
        case 128: k = slab_kernels_for<T, 128>(); return true;
        case 256: k = slab_kernels_for<T, 256>(); return true;
        case 512: k = slab_kernels_for<T, 512>(); return true;
        case 1024: k = slab_kernels_for<T, 1024>(); return true;
    }
    return false;
}

}  // namespace ffcm
