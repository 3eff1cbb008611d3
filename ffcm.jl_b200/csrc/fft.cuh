// Step 4: the spectral Stokes solve, as a hand-written 3-D FFT in five passes
// over the half-complex spectrum, with the per-mode projector fused into the
// z pass:
//
//   x r2c  ->  y fwd  ->  [z fwd, projector, z inv]  ->  y inv  ->  x c2r
//
// Reference: src/stokes_solve.jl:21-42 (unnormalised FFTW r2c / c2r; the
// 1/M normalisation folded into the projector) and :200-240 (the projector
// f <- (inv_M/mu)(1/k^2)(f - k (k.f)/k^2), k = 0 -> 0). The c2r follows the
// FFTW / pocketfft convention for the halved x axis: complex inverse DFTs over
// y and z first, then the 1-D c2r along x, which ignores the imaginary parts
// of the x DC and Nyquist bins.
//
// Spectrum layout: spec[c][z][y][kx], kx fastest, row pitch hxp >= Mx/2+1
// complex values (rows start on aligned addresses).
//
// Transforms are mixed-radix Stockham autosort FFTs over lines held in shared
// memory (radix 8/4/2 first, then 3, 5, 7, and any prime up to 61), with
// twiddles read from a per-axis table W_M^t = exp(-2 pi i t / M) computed in
// double precision on the host.
#pragma once

#include "common.cuh"

namespace ffcm {

constexpr int FFT_MAX_STAGES = 24;
constexpr int FFT_MAX_GENERIC_RADIX = 61;

struct FftPlan {
    int n;          // complex transform length
    int tw_stride;  // W_n^e = table[e * tw_stride]
    int nstages;
    int radix[FFT_MAX_STAGES];
};

// Where line l, element i lives in shared memory:
//   (l / lpg) * gs + (l % lpg) * ls + i * es
struct LineMap {
    int lpg, gs, ls, es;
    __device__ __forceinline__ int base(int l) const {
        int g = l / lpg;
        return g * gs + (l - g * lpg) * ls;
    }
};

template <typename T>
__device__ __forceinline__ cplx<T> tw_at(const cplx<T>* __restrict__ tw, int idx, bool inv) {
    cplx<T> w = tw[idx];
    if (inv) w.y = -w.y;
    return w;
}

// Small DFTs: forward uses exp(-2 pi i q s / R), inverse the conjugate.
template <typename T, int R>
struct SmallDft {
    // generic O(R^2) with table twiddles W_R^q = table[q * step]
    __device__ __forceinline__ static void run(cplx<T>* v, bool inv, const cplx<T>* tw, int step) {
        cplx<T> out[R];
#pragma unroll
        for (int s = 0; s < R; ++s) {
            cplx<T> acc = v[0];
#pragma unroll
            for (int q = 1; q < R; ++q) acc = cadd(acc, cmul(v[q], tw_at(tw, ((q * s) % R) * step, inv)));
            out[s] = acc;
        }
#pragma unroll
        for (int s = 0; s < R; ++s) v[s] = out[s];
    }
};

template <typename T>
struct SmallDft<T, 2> {
    __device__ __forceinline__ static void run(cplx<T>* v, bool, const cplx<T>*, int) {
        cplx<T> a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <typename T>
__device__ __forceinline__ void dft4(cplx<T>& a0, cplx<T>& a1, cplx<T>& a2, cplx<T>& a3, bool inv) {
    cplx<T> s02 = cadd(a0, a2), d02 = csub(a0, a2);
    cplx<T> s13 = cadd(a1, a3), d13 = csub(a1, a3);
    cplx<T> r = inv ? mul_pi(d13) : mul_mi(d13);
    a0 = cadd(s02, s13);
    a2 = csub(s02, s13);
    a1 = cadd(d02, r);
    a3 = csub(d02, r);
}

template <typename T>
struct SmallDft<T, 4> {
    __device__ __forceinline__ static void run(cplx<T>* v, bool inv, const cplx<T>*, int) {
        dft4(v[0], v[1], v[2], v[3], inv);
    }
};

template <typename T>
struct SmallDft<T, 8> {
    __device__ __forceinline__ static void run(cplx<T>* v, bool inv, const cplx<T>*, int) {
        cplx<T> e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
        cplx<T> o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
        dft4(e0, e1, e2, e3, inv);
        dft4(o0, o1, o2, o3, inv);
        const T c = T(0.70710678118654752440084436210484903928);
        // W8^1, W8^2, W8^3 (forward: exp(-i pi k/4))
        cplx<T> t1 = inv ? cplx<T>{c * (o1.x - o1.y), c * (o1.x + o1.y)}
                         : cplx<T>{c * (o1.x + o1.y), c * (o1.y - o1.x)};
        cplx<T> t2 = inv ? mul_pi(o2) : mul_mi(o2);
        cplx<T> t3 = inv ? cplx<T>{-c * (o3.x + o3.y), c * (o3.x - o3.y)}
                         : cplx<T>{c * (o3.y - o3.x), -c * (o3.x + o3.y)};
        v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
        v[1] = cadd(e1, t1); v[5] = csub(e1, t1);
        v[2] = cadd(e2, t2); v[6] = csub(e2, t2);
        v[3] = cadd(e3, t3); v[7] = csub(e3, t3);
    }
};

// One Stockham stage of radix R over `nl` lines of length n (span Ns).
template <typename T, int R>
__device__ void fft_stage(const cplx<T>* __restrict__ A, cplx<T>* __restrict__ B, LineMap lm,
                          int nl, int n, int Ns, const cplx<T>* __restrict__ tw, int tws,
                          bool inv) {
    const int m = n / R;
    const int total = nl * m;
    const int twNR = n / (Ns * R);
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        const int l = t / m;
        const int j = t - l * m;
        const int k = j % Ns;
        const int base = lm.base(l);
        cplx<T> v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            cplx<T> a = A[base + (j + r * m) * lm.es];
            if (r > 0 && k > 0) a = cmul(a, tw_at(tw, k * r * twNR * tws, inv));
            v[r] = a;
        }
        SmallDft<T, R>::run(v, inv, tw, (n / R) * tws);
        const int o = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) B[base + (o + r * Ns) * lm.es] = v[r];
    }
}

// Runtime-radix stage for primes above 7 (values kept in local memory).
template <typename T>
__device__ void fft_stage_generic(const cplx<T>* __restrict__ A, cplx<T>* __restrict__ B,
                                  LineMap lm, int nl, int n, int Ns, int R,
                                  const cplx<T>* __restrict__ tw, int tws, bool inv) {
    const int m = n / R;
    const int total = nl * m;
    const int twNR = n / (Ns * R);
    const int step = (n / R) * tws;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        const int l = t / m;
        const int j = t - l * m;
        const int k = j % Ns;
        const int base = lm.base(l);
        cplx<T> v[FFT_MAX_GENERIC_RADIX];
        for (int r = 0; r < R; ++r) {
            cplx<T> a = A[base + (j + r * m) * lm.es];
            if (r > 0 && k > 0) a = cmul(a, tw_at(tw, k * r * twNR * tws, inv));
            v[r] = a;
        }
        const int o = (j / Ns) * Ns * R + k;
        for (int s = 0; s < R; ++s) {
            cplx<T> acc = v[0];
            for (int q = 1; q < R; ++q) acc = cadd(acc, cmul(v[q], tw_at(tw, ((q * s) % R) * step, inv)));
            B[base + (o + s * Ns) * lm.es] = acc;
        }
    }
}

// Transform `nl` lines in place (ping-pong between A and B). Returns the
// buffer that holds the result. Caller must __syncthreads() before (data in A).
template <typename T>
__device__ cplx<T>* fft_lines(cplx<T>* A, cplx<T>* B, LineMap lm, int nl, const FftPlan& p,
                              const cplx<T>* __restrict__ tw, bool inv) {
    int Ns = 1;
    for (int s = 0; s < p.nstages; ++s) {
        const int R = p.radix[s];
        switch (R) {
            case 2: fft_stage<T, 2>(A, B, lm, nl, p.n, Ns, tw, p.tw_stride, inv); break;
            case 3: fft_stage<T, 3>(A, B, lm, nl, p.n, Ns, tw, p.tw_stride, inv); break;
            case 4: fft_stage<T, 4>(A, B, lm, nl, p.n, Ns, tw, p.tw_stride, inv); break;
            case 5: fft_stage<T, 5>(A, B, lm, nl, p.n, Ns, tw, p.tw_stride, inv); break;
            case 7: fft_stage<T, 7>(A, B, lm, nl, p.n, Ns, tw, p.tw_stride, inv); break;
            case 8: fft_stage<T, 8>(A, B, lm, nl, p.n, Ns, tw, p.tw_stride, inv); break;
            default: fft_stage_generic<T>(A, B, lm, nl, p.n, Ns, R, tw, p.tw_stride, inv); break;
        }
        __syncthreads();
        cplx<T>* t = A;
        A = B;
        B = t;
        Ns *= R;
    }
    return A;
}

// ---- pass 1: x r2c, rows of the real grid -> rows of the spectrum --------
template <typename T>
__global__ void k_fft_x_r2c(const T* __restrict__ f, cplx<T>* __restrict__ spec, int Mx,
                            int nrows, int hxp, FftPlan p, const cplx<T>* __restrict__ twx,
                            int lpb) {
    extern __shared__ unsigned char smem_raw[];
    cplx<T>* A = reinterpret_cast<cplx<T>*>(smem_raw);
    cplx<T>* B = A + lpb * p.n;
    const int row0 = blockIdx.x * lpb;
    const int nl = min(lpb, nrows - row0);
    const int n = p.n;
    const bool even = (Mx % 2) == 0;
    for (int idx = threadIdx.x; idx < nl * n; idx += blockDim.x) {
        int l = idx / n, i = idx - l * n;
        const T* row = f + (int64_t)(row0 + l) * Mx;
        if (even) A[idx] = reinterpret_cast<const cplx<T>*>(row)[i];
        else A[idx] = cplx<T>{row[i], T(0)};
    }
    __syncthreads();
    LineMap lm{1 << 30, 0, n, 1};
    cplx<T>* R = fft_lines(A, B, lm, nl, p, twx, false);
    const int nk = Mx / 2 + 1;
    for (int idx = threadIdx.x; idx < nl * nk; idx += blockDim.x) {
        int l = idx / nk, k = idx - l * nk;
        cplx<T> X;
        if (even) {
            const int H = n;
            cplx<T> Zk = R[l * H + (k % H)];
            cplx<T> Zc = cconj(R[l * H + ((H - k) % H)]);
            cplx<T> W = twx[k];
            cplx<T> S = cadd(Zk, Zc), D = cmul(W, csub(Zk, Zc));
            // X = S/2 - (i/2) W D
            X = cplx<T>{T(0.5) * (S.x + D.y), T(0.5) * (S.y - D.x)};
        } else {
            X = R[l * n + k];
        }
        spec[(int64_t)(row0 + l) * hxp + k] = X;
    }
}

// ---- passes 2 and 4: y c2c on (kx tile) x My columns of one (c, z) plane --
template <typename T>
__global__ void k_fft_y(cplx<T>* __restrict__ spec, int nkx, int My, int Mz, int hxp, FftPlan p,
                        const cplx<T>* __restrict__ twy, int TX, int inverse) {
    extern __shared__ unsigned char smem_raw[];
    cplx<T>* A = reinterpret_cast<cplx<T>*>(smem_raw);
    cplx<T>* B = A + TX * My;
    const int kx0 = blockIdx.x * TX;
    cplx<T>* plane = spec + ((int64_t)blockIdx.z * Mz + blockIdx.y) * My * hxp;
    for (int idx = threadIdx.x; idx < My * TX; idx += blockDim.x) {
        int y = idx / TX, tx = idx - y * TX;
        int kx = kx0 + tx;
        A[idx] = kx < nkx ? plane[(int64_t)y * hxp + kx] : cplx<T>{T(0), T(0)};
    }
    __syncthreads();
    LineMap lm{1 << 30, 0, 1, TX};
    cplx<T>* R = fft_lines(A, B, lm, TX, p, twy, inverse != 0);
    for (int idx = threadIdx.x; idx < My * TX; idx += blockDim.x) {
        int y = idx / TX, tx = idx - y * TX;
        int kx = kx0 + tx;
        if (kx < nkx) plane[(int64_t)y * hxp + kx] = R[idx];
    }
}

// ---- pass 3: z forward, Stokes projector, z inverse (all 3 components) ----
template <typename T>
__global__ void k_fft_z_stokes(cplx<T>* __restrict__ spec, int nkx, int My, int Mz, int hxp,
                               FftPlan p, const cplx<T>* __restrict__ twz, int TX,
                               const T* __restrict__ kxv, const T* __restrict__ kyv,
                               const T* __restrict__ kzv, T inv_mu_M) {
    extern __shared__ unsigned char smem_raw[];
    cplx<T>* A = reinterpret_cast<cplx<T>*>(smem_raw);
    cplx<T>* B = A + 3 * TX * Mz;
    const int kx0 = blockIdx.x * TX;
    const int y = blockIdx.y;
    const int64_t cstride = (int64_t)Mz * My * hxp;
    const int64_t zstride = (int64_t)My * hxp;
    cplx<T>* col = spec + (int64_t)y * hxp;
    for (int idx = threadIdx.x; idx < 3 * Mz * TX; idx += blockDim.x) {
        int c = idx / (Mz * TX);
        int r = idx - c * Mz * TX;
        int z = r / TX, tx = r - z * TX;
        int kx = kx0 + tx;
        A[idx] = kx < nkx ? col[c * cstride + z * zstride + kx] : cplx<T>{T(0), T(0)};
    }
    __syncthreads();
    LineMap lm{TX, Mz * TX, 1, TX};
    cplx<T>* R = fft_lines(A, B, lm, 3 * TX, p, twz, false);
    cplx<T>* S = (R == A) ? B : A;
    const T k2v = kyv[y];
    for (int idx = threadIdx.x; idx < Mz * TX; idx += blockDim.x) {
        int z = idx / TX, tx = idx - z * TX;
        int kx = kx0 + tx;
        if (kx >= nkx) continue;
        const T k1 = kxv[kx], k3 = kzv[z];
        cplx<T> f0 = R[idx], f1 = R[Mz * TX + idx], f2 = R[2 * Mz * TX + idx];
        const T ksq = k1 * k1 + k2v * k2v + k3 * k3;
        if (ksq == T(0)) {
            f0 = f1 = f2 = cplx<T>{T(0), T(0)};
        } else {
            const T inv_k2 = T(1) / ksq;
            const T sc = inv_mu_M * inv_k2;
            const T dre = (k1 * f0.x + k2v * f1.x + k3 * f2.x) * inv_k2;
            const T dim = (k1 * f0.y + k2v * f1.y + k3 * f2.y) * inv_k2;
            f0 = cplx<T>{sc * (f0.x - k1 * dre), sc * (f0.y - k1 * dim)};
            f1 = cplx<T>{sc * (f1.x - k2v * dre), sc * (f1.y - k2v * dim)};
            f2 = cplx<T>{sc * (f2.x - k3 * dre), sc * (f2.y - k3 * dim)};
        }
        R[idx] = f0;
        R[Mz * TX + idx] = f1;
        R[2 * Mz * TX + idx] = f2;
    }
    __syncthreads();
    cplx<T>* U = fft_lines(R, S, lm, 3 * TX, p, twz, true);
    for (int idx = threadIdx.x; idx < 3 * Mz * TX; idx += blockDim.x) {
        int c = idx / (Mz * TX);
        int r = idx - c * Mz * TX;
        int z = r / TX, tx = r - z * TX;
        int kx = kx0 + tx;
        if (kx < nkx) col[c * cstride + z * zstride + kx] = U[idx];
    }
}

// ---- pass 5: x c2r, spectrum rows -> rows of the real velocity grid ------
template <typename T>
__global__ void k_fft_x_c2r(const cplx<T>* __restrict__ spec, T* __restrict__ u, int Mx,
                            int nrows, int hxp, FftPlan p, const cplx<T>* __restrict__ twx,
                            int lpb) {
    extern __shared__ unsigned char smem_raw[];
    cplx<T>* A = reinterpret_cast<cplx<T>*>(smem_raw);
    cplx<T>* B = A + lpb * p.n;
    const int row0 = blockIdx.x * lpb;
    const int nl = min(lpb, nrows - row0);
    const int n = p.n;
    const bool even = (Mx % 2) == 0;
    for (int idx = threadIdx.x; idx < nl * n; idx += blockDim.x) {
        int l = idx / n, k = idx - l * n;
        const cplx<T>* row = spec + (int64_t)(row0 + l) * hxp;
        if (even) {
            const int H = n;
            cplx<T> Xk = row[k], Xc = row[H - k];
            if (k == 0) {
                Xk.y = T(0);  // DC imaginary part ignored
                Xc.y = T(0);  // Nyquist imaginary part ignored
            }
            cplx<T> Av = cadd(Xk, cconj(Xc));
            cplx<T> Bv = cmul(csub(Xk, cconj(Xc)), cconj(twx[k]));
            A[idx] = cadd(Av, mul_pi(Bv));
        } else {
            cplx<T> X;
            if (k == 0) X = cplx<T>{row[0].x, T(0)};
            else if (k <= (Mx - 1) / 2) X = row[k];
            else X = cconj(row[Mx - k]);
            A[idx] = X;
        }
    }
    __syncthreads();
    LineMap lm{1 << 30, 0, n, 1};
    cplx<T>* R = fft_lines(A, B, lm, nl, p, twx, true);
    for (int idx = threadIdx.x; idx < nl * n; idx += blockDim.x) {
        int l = idx / n, i = idx - l * n;
        T* row = u + (int64_t)(row0 + l) * Mx;
        if (even) reinterpret_cast<cplx<T>*>(row)[i] = R[idx];
        else row[i] = R[idx].x;
    }
}

}  // namespace ffcm
