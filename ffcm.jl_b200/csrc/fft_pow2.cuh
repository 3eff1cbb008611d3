// Fast path of the spectral Stokes solve for power-of-two line lengths
// (8 <= n <= 2048): register-resident Stockham FFTs.
//
// Each line of n complex values is handled by n/8 threads; thread j of a line
// holds the 8 elements j + q*n/8 (q = 0..7) in registers on entry and exit.
// Radix-8 butterflies run in registers; between stages the values are
// exchanged through shared memory (one store, one barrier, one load); a final
// radix-2 or radix-4 stage covers n = 8^a * {1, 2, 4}. The first stage reads
// straight from global memory and the last stage leaves the outputs in the
// same positions, so the passes below load and store HBM directly, coalesced.
// Twiddles W_n^t come from a shared-memory copy of the per-axis table.
//
// Same five passes and conventions as fft.cuh (x r2c, y, z + projector, y
// inverse, x c2r; c2r ignores the imaginary parts of the x DC and Nyquist
// bins).
#pragma once

#include "common.cuh"
#include "fft.cuh"

namespace ffcm {

// Padded shared-memory index: one spare slot per 8 complex values keeps the
// stride-8 stores of the early stages free of bank conflicts.
__device__ __forceinline__ int pad8(int i) { return i + (i >> 3); }
__host__ __device__ constexpr int padded_len(int n) { return n + n / 8 + 1; }

template <typename T>
__device__ __forceinline__ void dft8(cplx<T> (&v)[8], bool inv) {
    SmallDft<T, 8>::run(v, inv, nullptr, 0);
}

template <typename T>
__device__ __forceinline__ cplx<T> twid(const cplx<T>* tw, int e, int stride, bool inv) {
    cplx<T> w = tw[e * stride];
    if (inv) w.y = -w.y;
    return w;
}

__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n / 2); }

// Exchange through shared memory: line b, element i at sm[base(b) + pad8(i) * es].
template <typename T>
struct Exchange {
    cplx<T>* sm;
    int base;
    int es;
    __device__ __forceinline__ cplx<T>& at(int i) const { return sm[base + pad8(i) * es]; }
};

// Exchange through shared memory laid out densely: line b, element i at
// sm[base(b) + i * es] (no padding: the exchange is the line's own storage).
template <typename T>
struct ExchangeDense {
    cplx<T>* sm;
    int base;
    int es;
    __device__ __forceinline__ cplx<T>& at(int i) const { return sm[base + i * es]; }
};

// In-register FFT of one line: v[q] = x[j + q n/8] on entry, X[j + q n/8] on exit.
// `tw` holds W_n^t for t = e * tws (tws = table stride). All threads of the
// block must call this together (it contains __syncthreads()). With
// WARP = true every line lies inside one warp (n/8 <= 32 consecutive threads,
// lines not shared between warps) and the exchanges only synchronise the warp.
template <typename T, int n, bool WARP = false, typename EX = Exchange<T>>
__device__ __forceinline__ void fft_line_regs(cplx<T> (&v)[8], int j, const EX& ex,
                                              const cplx<T>* tw, int tws, bool inv) {
    static_assert(!WARP || n / 8 <= 32, "a warp-synchronised line must fit in one warp");
    constexpr int L2 = ilog2c(n);
    constexpr int NR8 = L2 / 3;
    constexpr int RL = 1 << (L2 % 3);
    constexpr int Q = n / 8;
#pragma unroll
    for (int s = 0; s < NR8; ++s) {
        const int Ns = 1 << (3 * s);
        if (s > 0) {
            const int k = j & (Ns - 1);
            const int step = n / (8 * Ns);
#pragma unroll
            for (int r = 1; r < 8; ++r) v[r] = cmul(v[r], twid(tw, k * r * step, tws, inv));
        }
        dft8(v, inv);
        if (s < NR8 - 1 || RL > 1) {
            const int o = (j / Ns) * 8 * Ns + (j & (Ns - 1));
            if (WARP) __syncwarp(); else __syncthreads();
#pragma unroll
            for (int r = 0; r < 8; ++r) ex.at(o + r * Ns) = v[r];
            if (WARP) __syncwarp(); else __syncthreads();
#pragma unroll
            for (int q = 0; q < 8; ++q) v[q] = ex.at(j + q * Q);
        }
    }
    if (RL == 2) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int jp = j + i * Q;
            cplx<T> a = v[i], b = cmul(v[i + 4], twid(tw, jp, tws, inv));
            v[i] = cadd(a, b);
            v[i + 4] = csub(a, b);
        }
    } else if (RL == 4) {
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int jp = j + i * Q;
            cplx<T> a0 = v[i];
            cplx<T> a1 = cmul(v[i + 2], twid(tw, jp, tws, inv));
            cplx<T> a2 = cmul(v[i + 4], twid(tw, 2 * jp, tws, inv));
            cplx<T> a3 = cmul(v[i + 6], twid(tw, 3 * jp, tws, inv));
            dft4(a0, a1, a2, a3, inv);
            v[i] = a0; v[i + 2] = a1; v[i + 4] = a2; v[i + 6] = a3;
        }
    }
}

// v *= (cr + i ci), or by its conjugate when inv
template <typename T>
__device__ __forceinline__ cplx<T> cmul_const(cplx<T> v, T cr, T ci, bool inv) {
    if (inv) ci = -ci;
    return cplx<T>{v.x * cr - v.y * ci, v.x * ci + v.y * cr};
}

// 16-point DFT in registers, 16 = 4 x 4: with q = b + 4a and k = c + 4d,
// X[c + 4d] = sum_b W4^(bd) [W16^(bc) sum_a v[b + 4a] W4^(ac)].
template <typename T>
__device__ __forceinline__ void dft16(cplx<T> (&v)[16], bool inv) {
#pragma unroll
    for (int b = 0; b < 4; ++b) dft4(v[b], v[b + 4], v[b + 8], v[b + 12], inv);   // v[b + 4c] = Y_b[c]
    // W16^e = exp(-2 pi i e / 16) for e = bc (forward)
    const T c8 = T(0.92387953251128675612818318939678828682);   // cos(pi/8)
    const T s8 = T(0.38268343236508977172845998403039886676);   // sin(pi/8)
    const T c4 = T(0.70710678118654752440084436210484903928);   // cos(pi/4)
    v[1 + 4 * 1] = cmul_const(v[1 + 4 * 1], c8, -s8, inv);     // e = 1
    v[1 + 4 * 2] = cmul_const(v[1 + 4 * 2], c4, -c4, inv);     // e = 2
    v[1 + 4 * 3] = cmul_const(v[1 + 4 * 3], s8, -c8, inv);     // e = 3
    v[2 + 4 * 1] = cmul_const(v[2 + 4 * 1], c4, -c4, inv);     // e = 2
    v[2 + 4 * 2] = inv ? mul_pi(v[2 + 4 * 2]) : mul_mi(v[2 + 4 * 2]);   // e = 4
    v[2 + 4 * 3] = cmul_const(v[2 + 4 * 3], -c4, -c4, inv);    // e = 6
    v[3 + 4 * 1] = cmul_const(v[3 + 4 * 1], s8, -c8, inv);     // e = 3
    v[3 + 4 * 2] = cmul_const(v[3 + 4 * 2], -c4, -c4, inv);    // e = 6
    v[3 + 4 * 3] = cmul_const(v[3 + 4 * 3], -c8, s8, inv);     // e = 9
    cplx<T> out[16];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        cplx<T> a0 = v[4 * c], a1 = v[4 * c + 1], a2 = v[4 * c + 2], a3 = v[4 * c + 3];
        dft4(a0, a1, a2, a3, inv);
        out[c] = a0;
        out[c + 4] = a1;
        out[c + 8] = a2;
        out[c + 12] = a3;
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = out[k];
}

// L-point DFT in registers, L = 4, 8 or 16.
template <typename T, int L>
__device__ __forceinline__ void dft_small(cplx<T> (&a)[L], bool inv) {
    if constexpr (L == 4) {
        dft4(a[0], a[1], a[2], a[3], inv);
    } else if constexpr (L == 8) {
        SmallDft<T, 8>::run(a, inv, nullptr, 0);
    } else {
        static_assert(L == 16, "L must be 4, 8 or 16");
        dft16(a, inv);
    }
}

// FFT of a line of n = 16 L points held by L consecutive lanes with 16 values
// each (the x transforms of the slab kernels at x lengths 128, 256 and 512:
// L = 4, 8, 16; 32 / L lines per warp). Decimation in time: lane t holds
// z[t + L q] (q = 0..15) on entry; a 16-point DFT over q in registers, the
// twiddle W_n^(t k1), one exchange through the line's scratch `xb`
// (16 x (L + 1) complex; may alias the line's own input, which is read
// before), then lane t takes k1 = t + L f (f < 16 / L) and runs an L-point DFT
// over the lanes' values of each. On exit lane t holds Z[t + L q], the same
// positions as on entry. `tw` holds W_n^e at e * tws (tws = 2 for the table of
// 2 n the slab kernels keep). All lanes of the warp must call it together.
template <typename T, int L>
__device__ __forceinline__ void fft_16xL(cplx<T> (&v)[16], int t, cplx<T>* xb, const cplx<T>* tw, int tws,
                                         bool inv) {
    constexpr int R = 16 / L;
    dft16(v, inv);
#pragma unroll
    for (int k1 = 1; k1 < 16; ++k1) v[k1] = cmul(v[k1], twid(tw, t * k1, tws, inv));
    __syncwarp();
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) xb[k1 * (L + 1) + t] = v[k1];
    __syncwarp();
#pragma unroll
    for (int f = 0; f < R; ++f) {
        cplx<T> u[L];
#pragma unroll
        for (int j = 0; j < L; ++j) u[j] = xb[(t + L * f) * (L + 1) + j];
        dft_small<T, L>(u, inv);
#pragma unroll
        for (int k2 = 0; k2 < L; ++k2) v[f + R * k2] = u[k2];
    }
}

// Value of lane `src` (0..L-1) of this lane's L-lane segment of the warp.
template <typename T, int L>
__device__ __forceinline__ cplx<T> shfl_seg(cplx<T> v, int src) {
    return cplx<T>{__shfl_sync(0xffffffffu, v.x, src, L), __shfl_sync(0xffffffffu, v.y, src, L)};
}

// Copy a twiddle table into shared memory.
template <typename T>
__device__ __forceinline__ void load_table(cplx<T>* dst, const cplx<T>* __restrict__ src, int count) {
    for (int i = threadIdx.x; i < count; i += blockDim.x) dst[i] = src[i];
}

// ---- pass 1: x r2c, LPB rows per block, H = Mx/2 complex points per row ---
// block = LPB * (H/8) threads; smem: table (Mx) + LPB * padded_len(H).
template <typename T, int H>
__global__ void __launch_bounds__(256) k_fftp_x_r2c(const T* __restrict__ f, cplx<T>* __restrict__ spec,
                                                    int nrows, int hxp, const cplx<T>* __restrict__ twx,
                                                    int lpb) {
    extern __shared__ unsigned char smem_raw[];
    constexpr int Mx = 2 * H, Q = H / 8, TPL = H / 8;
    cplx<T>* tw = reinterpret_cast<cplx<T>*>(smem_raw);
    cplx<T>* ex_sm = tw + Mx;
    load_table(tw, twx, Mx);
    const int b = threadIdx.x / TPL, j = threadIdx.x - b * TPL;
    const int row = blockIdx.x * lpb + b;
    const bool active = row < nrows;
    cplx<T> v[8];
    const cplx<T>* src = reinterpret_cast<const cplx<T>*>(f + (int64_t)(active ? row : 0) * Mx);
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = active ? src[j + q * Q] : cplx<T>{T(0), T(0)};
    __syncthreads();  // table ready
    // each line owns its exchange slot; a line inside one warp syncs the warp only
    constexpr bool WARP = TPL <= 32;
    Exchange<T> ex{ex_sm, b * padded_len(H), 1};
    fft_line_regs<T, H, WARP>(v, j, ex, tw, 2, false);
    if (WARP) __syncwarp(); else __syncthreads();
#pragma unroll
    for (int q = 0; q < 8; ++q) ex.at(j + q * Q) = v[q];
    if (WARP) __syncwarp(); else __syncthreads();
    if (!active) return;
    cplx<T>* dst = spec + (int64_t)row * hxp;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int k = j + q * Q;
        const cplx<T> Zk = v[q];
        const cplx<T> Zc = cconj(ex.at((H - k) & (H - 1)));
        const cplx<T> S = cadd(Zk, Zc), D = cmul(tw[k], csub(Zk, Zc));
        dst[k] = cplx<T>{T(0.5) * (S.x + D.y), T(0.5) * (S.y - D.x)};
    }
    if (j == 0) {
        const cplx<T> Z0 = ex.at(0);
        // k = H: W = -1, Zk = Z0, Zc = conj(Z0): X = Re(Z0) - Im(Z0)
        dst[H] = cplx<T>{Z0.x - Z0.y, T(0)};
    }
}

// ---- pass 5: x c2r --------------------------------------------------------
template <typename T, int H>
__global__ void __launch_bounds__(256) k_fftp_x_c2r(const cplx<T>* __restrict__ spec, T* __restrict__ u,
                                                    int nrows, int hxp, const cplx<T>* __restrict__ twx,
                                                    int lpb) {
    extern __shared__ unsigned char smem_raw[];
    constexpr int Mx = 2 * H, Q = H / 8, TPL = H / 8;
    cplx<T>* tw = reinterpret_cast<cplx<T>*>(smem_raw);
    cplx<T>* ex_sm = tw + Mx;
    load_table(tw, twx, Mx);
    const int b = threadIdx.x / TPL, j = threadIdx.x - b * TPL;
    const int row = blockIdx.x * lpb + b;
    const bool active = row < nrows;
    const cplx<T>* src = spec + (int64_t)(active ? row : 0) * hxp;
    __syncthreads();
    cplx<T> v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int k = j + q * Q;
        cplx<T> Xk = active ? src[k] : cplx<T>{T(0), T(0)};
        cplx<T> Xc = active ? src[H - k] : cplx<T>{T(0), T(0)};
        if (k == 0) {
            Xk.y = T(0);
            Xc.y = T(0);
        }
        const cplx<T> A = cadd(Xk, cconj(Xc));
        const cplx<T> B = cmul(csub(Xk, cconj(Xc)), cconj(tw[k]));
        v[q] = cadd(A, mul_pi(B));
    }
    Exchange<T> ex{ex_sm, b * padded_len(H), 1};
    fft_line_regs<T, H, (TPL <= 32)>(v, j, ex, tw, 2, true);
    if (!active) return;
    cplx<T>* dst = reinterpret_cast<cplx<T>*>(u + (int64_t)row * Mx);
#pragma unroll
    for (int q = 0; q < 8; ++q) dst[j + q * Q] = v[q];
}

// ---- passes 2 and 4: y, B consecutive kx columns of one (c, z) plane -------
// Columns kx0 <= kx < kx1 (a chunk of the spectrum; grid.x covers it).
// block = B * (n/8) threads, b fastest; smem: table (n) + B * padded_len(n).
template <typename T, int n, int B>
__global__ void __launch_bounds__(B * (n / 8)) k_fftp_y(cplx<T>* __restrict__ spec, int kx0, int kx1, int My,
                                                        int Mz, int hxp, const cplx<T>* __restrict__ twy,
                                                        int inverse) {
    extern __shared__ unsigned char smem_raw[];
    constexpr int Q = n / 8;
    cplx<T>* tw = reinterpret_cast<cplx<T>*>(smem_raw);
    cplx<T>* ex_sm = tw + n;
    load_table(tw, twy, n);
    const int b = threadIdx.x % B, j = threadIdx.x / B;
    const int kx = kx0 + blockIdx.x * B + b;
    const bool active = kx < kx1;
    cplx<T>* plane = spec + ((int64_t)blockIdx.z * Mz + blockIdx.y) * My * hxp + (active ? kx : 0);
    cplx<T> v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = active ? plane[(int64_t)(j + q * Q) * hxp] : cplx<T>{T(0), T(0)};
    __syncthreads();
    Exchange<T> ex{ex_sm, b, B};
    fft_line_regs<T, n>(v, j, ex, tw, 1, inverse != 0);
    if (!active) return;
#pragma unroll
    for (int q = 0; q < 8; ++q) plane[(int64_t)(j + q * Q) * hxp] = v[q];
}

// ---- pass 3: z forward, projector, z inverse; B kx columns of one y -------
template <typename T, int n, int B>
__global__ void __launch_bounds__(B * (n / 8)) k_fftp_z_stokes(
    cplx<T>* __restrict__ spec, int kx0, int kx1, int My, int hxp, const cplx<T>* __restrict__ twz,
    const T* __restrict__ kxv, const T* __restrict__ kyv, const T* __restrict__ kzv, T inv_mu_M) {
    extern __shared__ unsigned char smem_raw[];
    constexpr int Q = n / 8;
    cplx<T>* tw = reinterpret_cast<cplx<T>*>(smem_raw);
    cplx<T>* ex_sm = tw + n;
    load_table(tw, twz, n);
    const int b = threadIdx.x % B, j = threadIdx.x / B;
    const int kx = kx0 + blockIdx.x * B + b;
    const int y = blockIdx.y;
    const bool active = kx < kx1;
    const int64_t zs = (int64_t)My * hxp;
    const int64_t cs = (int64_t)n * zs;
    cplx<T>* col = spec + (int64_t)y * hxp + (active ? kx : 0);
    cplx<T> v0[8], v1[8], v2[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int64_t o = (int64_t)(j + q * Q) * zs;
        v0[q] = active ? col[o] : cplx<T>{T(0), T(0)};
        v1[q] = active ? col[cs + o] : cplx<T>{T(0), T(0)};
        v2[q] = active ? col[2 * cs + o] : cplx<T>{T(0), T(0)};
    }
    __syncthreads();
    Exchange<T> ex{ex_sm, b, B};
    fft_line_regs<T, n>(v0, j, ex, tw, 1, false);
    fft_line_regs<T, n>(v1, j, ex, tw, 1, false);
    fft_line_regs<T, n>(v2, j, ex, tw, 1, false);
    const T k1 = active ? kxv[kx] : T(0);
    const T k2 = kyv[y];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const T k3 = kzv[j + q * Q];
        const T ksq = k1 * k1 + k2 * k2 + k3 * k3;
        if (ksq == T(0)) {
            v0[q] = v1[q] = v2[q] = cplx<T>{T(0), T(0)};
        } else {
            const T inv_k2 = T(1) / ksq;
            const T sc = inv_mu_M * inv_k2;
            const T dre = (k1 * v0[q].x + k2 * v1[q].x + k3 * v2[q].x) * inv_k2;
            const T dim = (k1 * v0[q].y + k2 * v1[q].y + k3 * v2[q].y) * inv_k2;
            v0[q] = cplx<T>{sc * (v0[q].x - k1 * dre), sc * (v0[q].y - k1 * dim)};
            v1[q] = cplx<T>{sc * (v1[q].x - k2 * dre), sc * (v1[q].y - k2 * dim)};
            v2[q] = cplx<T>{sc * (v2[q].x - k3 * dre), sc * (v2[q].y - k3 * dim)};
        }
    }
    fft_line_regs<T, n>(v0, j, ex, tw, 1, true);
    fft_line_regs<T, n>(v1, j, ex, tw, 1, true);
    fft_line_regs<T, n>(v2, j, ex, tw, 1, true);
    if (!active) return;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int64_t o = (int64_t)(j + q * Q) * zs;
        col[o] = v0[q];
        col[cs + o] = v1[q];
        col[2 * cs + o] = v2[q];
    }
}

// ---- pass 3, low-register variant --------------------------------------
// Same result as k_fftp_z_stokes; the three components go through the
// forward transform one after the other and wait in shared memory for the
// projector, then each is inverse-transformed from there. One line of 8
// values per thread is live at a time, so more blocks fit on an SM.
// block = B * (n/8) threads, b fastest; smem: table (n) + 3 * B * padded_len(n).
template <typename T, int n, int B>
__global__ void __launch_bounds__(B * (n / 8), (768 / (B * (n / 8))) > 0 ? 768 / (B * (n / 8)) : 1)
    k_fftp_z_stokes_lr(
    cplx<T>* __restrict__ spec, int kx0, int kx1, int My, int hxp, const cplx<T>* __restrict__ twz,
    const T* __restrict__ kxv, const T* __restrict__ kyv, const T* __restrict__ kzv, T inv_mu_M) {
    extern __shared__ unsigned char smem_raw[];
    constexpr int Q = n / 8, PL = padded_len(n);
    cplx<T>* tw = reinterpret_cast<cplx<T>*>(smem_raw);
    cplx<T>* ex_sm = tw + n;
    load_table(tw, twz, n);
    const int b = threadIdx.x % B, j = threadIdx.x / B;
    const int kx = kx0 + blockIdx.x * B + b;
    const int y = blockIdx.y;
    const bool active = kx < kx1;
    const int64_t zs = (int64_t)My * hxp;
    const int64_t cs = (int64_t)n * zs;
    cplx<T>* col = spec + (int64_t)y * hxp + (active ? kx : 0);
    const Exchange<T> ex[3] = {Exchange<T>{ex_sm, b, B}, Exchange<T>{ex_sm + B * PL, b, B},
                               Exchange<T>{ex_sm + 2 * B * PL, b, B}};
    __syncthreads();  // table ready
#pragma unroll 1
    for (int c = 0; c < 3; ++c) {
        cplx<T> v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q)
            v[q] = active ? col[c * cs + (int64_t)(j + q * Q) * zs] : cplx<T>{T(0), T(0)};
        fft_line_regs<T, n>(v, j, ex[c], tw, 1, false);
        __syncthreads();   // the line's last exchange has been read
#pragma unroll
        for (int q = 0; q < 8; ++q) ex[c].at(j + q * Q) = v[q];
    }
    // projector at this thread's points (its own slots of the three lines)
    const T k1 = active ? kxv[kx] : T(0);
    const T k2 = kyv[y];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int z = j + q * Q;
        const T k3 = kzv[z];
        const T ksq = k1 * k1 + k2 * k2 + k3 * k3;
        cplx<T> a0 = ex[0].at(z), a1 = ex[1].at(z), a2 = ex[2].at(z);
        if (ksq == T(0)) {
            a0 = a1 = a2 = cplx<T>{T(0), T(0)};
        } else {
            const T inv_k2 = T(1) / ksq;
            const T sc = inv_mu_M * inv_k2;
            const T dre = (k1 * a0.x + k2 * a1.x + k3 * a2.x) * inv_k2;
            const T dim = (k1 * a0.y + k2 * a1.y + k3 * a2.y) * inv_k2;
            a0 = cplx<T>{sc * (a0.x - k1 * dre), sc * (a0.y - k1 * dim)};
            a1 = cplx<T>{sc * (a1.x - k2 * dre), sc * (a1.y - k2 * dim)};
            a2 = cplx<T>{sc * (a2.x - k3 * dre), sc * (a2.y - k3 * dim)};
        }
        ex[0].at(z) = a0;
        ex[1].at(z) = a1;
        ex[2].at(z) = a2;
    }
#pragma unroll 1
    for (int c = 0; c < 3; ++c) {
        cplx<T> v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = ex[c].at(j + q * Q);
        fft_line_regs<T, n>(v, j, ex[c], tw, 1, true);
        if (active) {
#pragma unroll
            for (int q = 0; q < 8; ++q) col[c * cs + (int64_t)(j + q * Q) * zs] = v[q];
        }
    }
}

}  // namespace ffcm
