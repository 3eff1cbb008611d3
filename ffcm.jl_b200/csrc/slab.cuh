// Steps 3 and 5 fused with the x-axis transforms (the fast path of the
// assembled operator): grids whose x length is a power of two (64..2048) and
// stencils of M_G = 8 points per axis.
//
// A block owns a slab: BY x BZ full x-rows of the grid, all three components,
// held in shared memory. The particles whose stencil can touch the slab are
// the particles of a few (cy, cz) rows of cells, each row one contiguous range
// of the cell-sorted order; the block scans them and keeps those that touch
// (integer anchor arithmetic, as the reference computes it), in candidate
// order, in windows of SLAB_CAP entries.
//
//  * k_spread_slab: per window, one thread per entry computes the separable
//    weights (src/stencil.jl:80-112); the entries are sorted by the first x
//    point of their stencil, and each thread then owns grid points x and
//    gathers F (a0 + a2 r^2) gx gy gz from the entries covering x into
//    registers (src/spread_forces.jl:73-130) — no atomics, deterministic.
//    Each slab row is then x-r2c transformed in shared memory and written
//    straight to the spectrum. The block also stores its particle list, so
//    the interpolation does not scan again.
//  * k_interp_slab: the slab's spectrum rows are x-c2r transformed into shared
//    memory; one thread per listed particle gathers its partial velocity over
//    the slab rows (src/interpolate.jl:322-376) and adds it, with an L2
//    reduction, to a sorted-order velocity buffer that the correction kernel
//    finishes (h^3 scale, correction, scatter to the caller's order).
#pragma once

#include "common.cuh"
#include "fft_pow2.cuh"
#include "spread_interp.cuh"

namespace ffcm {

constexpr int SLAB_MG = 8;        // stencil width of the fused path
constexpr int SLAB_CAP = 128;     // entries per list window (shared memory)
constexpr int SLAB_PAIRMAX = 512; // cell rows one slab may scan

struct SlabGeom {
    int m0, m1, m2;   // cell grid
    double cs1, cs2;  // cell sizes (y, z)
    double h;         // grid spacing
    int nty, ntz;     // slabs along y and z
    int lcap;         // capacity of a slab's stored particle list
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

// One window of listed particles and their separable weights.
template <typename T, int BY, int BZ, int H>
struct SlabWin {
    static constexpr int NRP = BY * BZ;
    int s[SLAB_CAP];          // sorted particle index
    int key[SLAB_CAP];        // first x point of the stencil, in [0, Mx)
    int sy[SLAB_CAP], sz[SLAB_CAP];
    unsigned msk[SLAB_CAP];   // y rows hit (bits 0..7) | z rows hit (bits 8..15)
    T y0[SLAB_CAP], y1[SLAB_CAP], y2[SLAB_CAP];
    T f[3][SLAB_CAP];
    // rows padded by one element: lanes reading different entries at the same
    // stencil point or slab row then fall into different banks
    T gx[SLAB_CAP][SLAB_MG + 1], r2x[SLAB_CAP][SLAB_MG + 1];
    T gyz[SLAB_CAP][NRP + 1], r2yz[SLAB_CAP][NRP + 1];
    unsigned sk[SLAB_CAP];    // sort keys (key << 7 | entry)
    int first[2 * H + 1];     // first sorted entry with key >= v
    int pair_start[SLAB_PAIRMAX + 1];
    int pair_sb[SLAB_PAIRMAX];
    int scan[32];
};

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
    sx = (int)rint_t(mul_rn(y.x, p.inv_h)) - half;
    sy = (int)rint_t(mul_rn(y.y, p.inv_h)) - half;
    sz = (int)rint_t(mul_rn(y.z, p.inv_h)) - half;
    const unsigned my = rows_hit<BY>(sy, y0r, p.My);
    const unsigned mz = rows_hit<BZ>(sz, z0r, p.Mz);
    m = (my && mz) ? (my | (mz << 8)) : 0u;
}

template <typename T, int BY, int BZ, int H>
__device__ __forceinline__ void slab_put(SlabWin<T, BY, BZ, H>& W, int i, int s, const vec4<T>& y, int sx,
                                         int sy, int sz, unsigned m) {
    W.s[i] = s;
    W.key[i] = wrap1(sx, 2 * H);
    W.sy[i] = sy;
    W.sz[i] = sz;
    W.msk[i] = m;
    W.y0[i] = y.x;
    W.y1[i] = y.y;
    W.y2[i] = y.z;
}

// Separable weights of window entry i (one thread per entry), with the
// reference's x = g h - Y for the unwrapped stencil point g. Row pairs the
// particle does not reach keep weight 0 and are skipped by the mask.
template <typename T, int BY, int BZ, int H>
__device__ __forceinline__ void slab_entry_weights(const StencilParams<T>& p, SlabWin<T, BY, BZ, H>& W,
                                                   int i, int y0r, int z0r) {
    const int gx0 = (int)rint_t(mul_rn(W.y0[i], p.inv_h)) - SLAB_MG / 2;
#pragma unroll
    for (int e = 0; e < SLAB_MG; ++e) {
        const T x = sub_rn(mul_rn((T)(gx0 + e), p.h), W.y0[i]);
        const T x2 = mul_rn(x, x);
        W.gx[i][e] = p.inv_norm * exp_t(-x2 * p.inv_2S2);
        W.r2x[i][e] = x2;
    }
    const unsigned m = W.msk[i];
    T gy[BY], r2y[BY], gz[BZ], r2z[BZ];
#pragma unroll
    for (int b = 0; b < BY; ++b) {
        gy[b] = T(0);
        r2y[b] = T(0);
        if ((m >> b) & 1u) {
            const int g = W.sy[i] + wrap1(y0r + b - W.sy[i], p.My);
            const T x = sub_rn(mul_rn((T)g, p.h), W.y1[i]);
            r2y[b] = mul_rn(x, x);
            gy[b] = p.inv_norm * exp_t(-r2y[b] * p.inv_2S2);
        }
    }
#pragma unroll
    for (int d = 0; d < BZ; ++d) {
        gz[d] = T(0);
        r2z[d] = T(0);
        if ((m >> (8 + d)) & 1u) {
            const int g = W.sz[i] + wrap1(z0r + d - W.sz[i], p.Mz);
            const T x = sub_rn(mul_rn((T)g, p.h), W.y2[i]);
            r2z[d] = mul_rn(x, x);
            gz[d] = p.inv_norm * exp_t(-r2z[d] * p.inv_2S2);
        }
    }
#pragma unroll
    for (int d = 0; d < BZ; ++d)
#pragma unroll
        for (int b = 0; b < BY; ++b) {
            W.gyz[i][d * BY + b] = gy[b] * gz[d];
            W.r2yz[i][d * BY + b] = r2y[b] + r2z[d];
        }
}

// Scan the candidates of a slab (particles of the cell rows in range, in
// sorted order) and hand the touching ones to `process(count)` in windows of
// at most SLAB_CAP entries, in candidate order. Stores the full list in
// glist (capacity g.lcap) and its length in *gcount (-1 when it did not fit).
// All threads of the block must call this.
template <typename T, int BY, int BZ, int H, bool WANT_F, typename Process>
__device__ __forceinline__ void slab_scan(const vec4<T>* __restrict__ Ys, const vec4<T>* __restrict__ Fs,
                                         const int32_t* __restrict__ off, const StencilParams<T>& p,
                                         const SlabGeom& g, int y0r, int z0r, SlabWin<T, BY, BZ, H>& W,
                                         int* __restrict__ glist, int* __restrict__ gcount,
                                         Process&& process) {
    constexpr int half = SLAB_MG / 2;
    int cy_lo, ny, cz_lo, nz;
    cell_span(y0r - SLAB_MG + 1 + half, y0r + BY - 1 + half, g.h, g.cs1, g.m1, cy_lo, ny);
    cell_span(z0r - SLAB_MG + 1 + half, z0r + BZ - 1 + half, g.h, g.cs2, g.m2, cz_lo, nz);
    const int npairs = ny * nz;   // <= SLAB_PAIRMAX (checked on the host)
    int carry = 0;
    for (int base = 0; base < npairs; base += blockDim.x) {
        const int pi = base + threadIdx.x;
        int len = 0;
        if (pi < npairs) {
            const int cy = imod(cy_lo + pi % ny, g.m1);
            const int cz = imod(cz_lo + pi / ny, g.m2);
            const int c0 = (cy + cz * g.m1) * g.m0;
            const int sb = off[c0];
            len = off[c0 + g.m0] - sb;
            W.pair_sb[pi] = sb;
        }
        int tot;
        const int pre = block_scan(len, W.scan, tot);
        if (pi < npairs) W.pair_start[pi] = carry + pre;
        carry += tot;
    }
    if (threadIdx.x == 0) W.pair_start[npairs] = carry;
    __syncthreads();
    const int ncand = carry;
    int count = 0, total = 0;
    // chunks of SLAB_CAP candidates, so one chunk always fits an emptied window
    for (int c0 = 0; c0 < ncand; c0 += SLAB_CAP) {
        const int c = c0 + threadIdx.x;
        unsigned m = 0;
        int s = 0, sx = 0, sy = 0, sz = 0;
        vec4<T> y{};
        if (threadIdx.x < SLAB_CAP && c < ncand) {
            int lo = 0, hi = npairs - 1;   // last cell row with pair_start <= c
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (W.pair_start[mid] <= c) lo = mid;
                else hi = mid - 1;
            }
            s = W.pair_sb[lo] + (c - W.pair_start[lo]);
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
        if (m) {
            const int i = count + pre;
            slab_put(W, i, s, y, sx, sy, sz, m);
            if (WANT_F) {
                const vec4<T> f = Fs[s];
                W.f[0][i] = f.x; W.f[1][i] = f.y; W.f[2][i] = f.z;
            }
            if (glist && total + pre < g.lcap) glist[total + pre] = s;
        }
        count += tot;
        total += tot;
        __syncthreads();
    }
    if (count > 0) process(count);
    if (gcount && threadIdx.x == 0) *gcount = total <= g.lcap ? total : -1;
    __syncthreads();
}

// Replay a stored slab list in windows of SLAB_CAP entries (the list holds
// only particles that touch the slab, in candidate order).
template <typename T, int BY, int BZ, int H, bool WANT_F, typename Process>
__device__ __forceinline__ void slab_replay(const vec4<T>* __restrict__ Ys, const vec4<T>* __restrict__ Fs,
                                           const StencilParams<T>& p, int y0r, int z0r,
                                           SlabWin<T, BY, BZ, H>& W, const int* __restrict__ glist, int total,
                                           Process&& process) {
    for (int w0 = 0; w0 < total; w0 += SLAB_CAP) {
        const int n = min(SLAB_CAP, total - w0);
        if ((int)threadIdx.x < n) {
            const int s = glist[w0 + threadIdx.x];
            const vec4<T> y = Ys[s];
            int sx, sy, sz;
            unsigned m;
            slab_anchor<T, BY, BZ>(p, y, y0r, z0r, sx, sy, sz, m);
            slab_put(W, (int)threadIdx.x, s, y, sx, sy, sz, m);
            if (WANT_F) {
                const vec4<T> f = Fs[s];
                W.f[0][threadIdx.x] = f.x;
                W.f[1][threadIdx.x] = f.y;
                W.f[2][threadIdx.x] = f.z;
            }
        }
        __syncthreads();
        process(n);
        __syncthreads();
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
    constexpr int half = SLAB_MG / 2;
    const int lane = threadIdx.x & 31;
    const int slab = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    if (slab >= g.nty * g.ntz) return;   // whole warps leave together
    const int ty = slab % g.nty, tz = slab / g.nty;
    const int y0r = ty * BY, z0r = tz * BZ;
    int cy_lo, ny, cz_lo, nz;
    cell_span(y0r - SLAB_MG + 1 + half, y0r + BY - 1 + half, g.h, g.cs1, g.m1, cy_lo, ny);
    cell_span(z0r - SLAB_MG + 1 + half, z0r + BZ - 1 + half, g.h, g.cs2, g.m2, cz_lo, nz);
    int* out = lists + (int64_t)slab * g.lcap;
    const unsigned lt = (1u << lane) - 1u;
    int total = 0;
    for (int pi = 0; pi < ny * nz; ++pi) {
        const int cy = imod(cy_lo + pi % ny, g.m1);
        const int cz = imod(cz_lo + pi / ny, g.m2);
        const int c0 = (cy + cz * g.m1) * g.m0;
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

// ---- spread into a slab, then x-r2c straight into the spectrum -----------
template <typename T, int H, int BY, int BZ>
__global__ void __launch_bounds__(256) k_spread_slab(const vec4<T>* __restrict__ Ys,
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
    cplx<T>* tw = reinterpret_cast<cplx<T>*>(acc + ROWS * P);
    cplx<T>* dummy = tw + Mx;   // exchange of the idle lanes of a partial FFT round
    SlabWin<T, BY, BZ, H>& W = *reinterpret_cast<SlabWin<T, BY, BZ, H>*>(dummy + padded_len(H));
    const int y0r = blockIdx.x * BY, z0r = blockIdx.y * BZ;
    const int cta = blockIdx.x + blockIdx.y * gridDim.x;
    for (int i = threadIdx.x; i < ROWS * P; i += blockDim.x) acc[i] = T(0);
    load_table(tw, twx, Mx);
    __syncthreads();
    auto process = [&](int count) {
            __syncthreads();
            // sort the window by first x point: each entry's rank is the
            // number of entries with a smaller (key, index) pair
            for (int i = threadIdx.x; i < SLAB_CAP; i += blockDim.x) {
                if (i < count) {
                    slab_entry_weights(p, W, i, y0r, z0r);
                    const unsigned me = ((unsigned)W.key[i] << 7) | (unsigned)i;
                    int rank = 0;
                    for (int k = 0; k < count; ++k) rank += (((unsigned)W.key[k] << 7) | (unsigned)k) < me;
                    W.sk[rank] = me;
                } else {
                    W.sk[i] = 0xffffffffu;
                }
            }
            __syncthreads();
            for (int v = threadIdx.x; v <= Mx; v += blockDim.x) {
                int lo = 0, hi = SLAB_CAP;   // first sorted entry with key >= v
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if ((int)(W.sk[mid] >> 7) < v) lo = mid + 1;
                    else hi = mid;
                }
                W.first[v] = lo;
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
                        kb = W.first[lo1 >= 0 ? lo1 : 0];
                        ke = W.first[x + 1];
                    } else {
                        if (lo1 >= 0) break;
                        kb = W.first[Mx + lo1];
                        ke = W.first[Mx];
                    }
                    for (int kk = kb; kk < ke; ++kk) {
                        const unsigned v = W.sk[kk];
                        const int i = (int)(v & 127u);
                        int e = x - (int)(v >> 7);
                        if (e < 0) e += Mx;
                        const T gxe = W.gx[i][e], r2xe = W.r2x[i][e];
                        const unsigned m = W.msk[i];
                        const T f0 = W.f[0][i], f1 = W.f[1][i], f2 = W.f[2][i];
#pragma unroll
                        for (int d = 0; d < BZ; ++d)
#pragma unroll
                            for (int b = 0; b < BY; ++b) {
                                if (!((m >> b) & (m >> (8 + d)) & 1u)) continue;
                                const int r = d * BY + b;
                                const T wgt = (p.a0 + p.a2 * (r2xe + W.r2yz[i][r])) * gxe * W.gyz[i][r];
                                a[0][r] += wgt * f0;
                                a[1][r] += wgt * f1;
                                a[2][r] += wgt * f2;
                            }
                    }
                }
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int r = 0; r < NRP; ++r) acc[(c * NRP + r) * P + x] += a[c][r];
            }
        };
    const int stored = counts[cta];
    if (stored >= 0) {
        slab_replay<T, BY, BZ, H, true>(Ys, Fs, p, y0r, z0r, W, lists + (int64_t)cta * g.lcap, stored, process);
    } else {
        slab_scan<T, BY, BZ, H, true>(Ys, Fs, off, p, g, y0r, z0r, W, nullptr, nullptr, process);
    }
    // x r2c of every slab row (H/8 threads per row), output straight to spec.
    // A row that fits one warp is transformed with warp-level synchronisation
    // only (rows are disjoint between warps; idle lanes exchange through a
    // scratch line whose contents are never used).
    constexpr int TPL = H / 8, Q = H / 8;
    constexpr bool WARP = TPL <= 32;
    const int lines_per_round = blockDim.x / TPL;
    const int lr = threadIdx.x / TPL, j = threadIdx.x - lr * TPL;
    __syncthreads();
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
            cplx<T>* dst = spec + (((int64_t)c * p.Mz + z0r + d) * p.My + y0r + b) * hxp;
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

// ---- x-c2r of a slab into shared memory, then gather partial velocities ----
// Each slab adds its partial sums into Vs[3 s + c] (sorted order, zeroed
// beforehand); the correction kernel finishes V[:, perm[s]] = h^3 Vs[s] + dv.
template <typename T, int H, int BY, int BZ>
__global__ void __launch_bounds__(256) k_interp_slab(const vec4<T>* __restrict__ Ys,
                                                     const int32_t* __restrict__ off,
                                                     const cplx<T>* __restrict__ spec, int hxp,
                                                     T* __restrict__ Vs, StencilParams<T> p,
                                                     SlabGeom g, const cplx<T>* __restrict__ twx,
                                                     const int* __restrict__ lists,
                                                     const int* __restrict__ counts) {
    constexpr int Mx = 2 * H, P = slab_pitch(Mx), NRP = BY * BZ, ROWS = 3 * NRP;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* acc = reinterpret_cast<T*>(smem_raw);
    cplx<T>* tw = reinterpret_cast<cplx<T>*>(acc + ROWS * P);
    cplx<T>* dummy = tw + Mx;
    SlabWin<T, BY, BZ, H>& W = *reinterpret_cast<SlabWin<T, BY, BZ, H>*>(dummy + padded_len(H));
    const int y0r = blockIdx.x * BY, z0r = blockIdx.y * BZ;
    const int cta = blockIdx.x + blockIdx.y * gridDim.x;
    load_table(tw, twx, Mx);
    __syncthreads();
    constexpr int TPL = H / 8, Q = H / 8;
    constexpr bool WARP = TPL <= 32;
    const int lines_per_round = blockDim.x / TPL;
    const int lr = threadIdx.x / TPL, j = threadIdx.x - lr * TPL;
    for (int r0 = 0; r0 < ROWS; r0 += lines_per_round) {
        const int r = r0 + lr;
        const bool active = r < ROWS && lr < lines_per_round;
        const int c = active ? r / NRP : 0, bd = active ? r % NRP : 0;
        const int b = bd % BY, d = bd / BY;
        const cplx<T>* src = spec + (((int64_t)c * p.Mz + z0r + d) * p.My + y0r + b) * hxp;
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
    __syncthreads();
    auto gather = [&](int count) {
        for (int i = threadIdx.x; i < count; i += blockDim.x) {
            slab_entry_weights(p, W, i, y0r, z0r);
            const unsigned m = W.msk[i];
            const int x0 = W.key[i];
            T v0 = 0, v1 = 0, v2 = 0;
#pragma unroll
            for (int d = 0; d < BZ; ++d)
#pragma unroll
                for (int b = 0; b < BY; ++b) {
                    if (!((m >> b) & (m >> (8 + d)) & 1u)) continue;
                    const int r = d * BY + b;
                    const T r2yz = W.r2yz[i][r], gyz = W.gyz[i][r];
                    const T* row = acc + r * P;
#pragma unroll
                    for (int e = 0; e < SLAB_MG; ++e) {
                        int x = x0 + e;
                        if (x >= Mx) x -= Mx;
                        const T wgt = (p.a0 + p.a2 * (W.r2x[i][e] + r2yz)) * W.gx[i][e] * gyz;
                        v0 += wgt * row[x];
                        v1 += wgt * row[NRP * P + x];
                        v2 += wgt * row[2 * NRP * P + x];
                    }
                }
            T* vs = Vs + 3 * (int64_t)W.s[i];
            atomicAdd(vs, v0);
            atomicAdd(vs + 1, v1);
            atomicAdd(vs + 2, v2);
        }
    };
    const int stored = counts[cta];
    if (stored >= 0) {
        slab_replay<T, BY, BZ, H, false>(Ys, nullptr, p, y0r, z0r, W, lists + (int64_t)cta * g.lcap, stored, gather);
    } else {
        slab_scan<T, BY, BZ, H, false>(Ys, nullptr, off, p, g, y0r, z0r, W, nullptr, nullptr,
                                      [&](int count) {
                                          __syncthreads();
                                          gather(count);
                                      });
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
                                  StencilParams<T>, SlabGeom, const cplx<T>*, const int*, const int*);

template <typename T>
struct SlabKernels {
    SpreadSlabKernel<T> spread_fused = nullptr;
    InterpSlabKernel<T> interp = nullptr;
    ListsKernel<T> lists = nullptr;
    int BY = 0, BZ = 0;
    size_t smem = 0;
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
    k.smem = (size_t)3 * BY * BZ * slab_pitch(2 * H) * sizeof(T) +
             (size_t)(2 * H + padded_len(H)) * sizeof(cplx<T>) + sizeof(SlabWin<T, BY, BZ, H>);
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
