// Persistent, software-pipelined y and z passes of the spectral Stokes solve
// (power-of-two line lengths 32..1024).
//
// A block loops over tiles (B consecutive kx columns of one line bundle).
// While it transforms tile t from registers, the next tile is already on its
// way into a shared-memory staging buffer through asynchronous 16-byte copies
// (cp.async), so the HBM stream never waits for the FFT arithmetic. The z pass
// transforms its three components in lockstep: one twiddle load and one pair
// of barriers per stage serve all three lines, and the three butterflies give
// the scheduler independent work.
#pragma once

#include "common.cuh"
#include "fft_pow2.cuh"

namespace ffcm {

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// NC lines per thread in lockstep; line c exchanges through ex[c].
// v[c][q] = x_c[j + q n/8] on entry, X_c[j + q n/8] on exit.
template <typename T, int n, int NC>
__device__ __forceinline__ void fft_lines_lockstep(cplx<T> (&v)[NC][8], int j, const Exchange<T> (&ex)[NC],
                                                   const cplx<T>* tw, bool inv) {
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
            for (int r = 1; r < 8; ++r) {
                const cplx<T> w = twid(tw, k * r * step, 1, inv);
#pragma unroll
                for (int c = 0; c < NC; ++c) v[c][r] = cmul(v[c][r], w);
            }
        }
#pragma unroll
        for (int c = 0; c < NC; ++c) dft8(v[c], inv);
        if (s < NR8 - 1 || RL > 1) {
            const int o = (j / Ns) * 8 * Ns + (j & (Ns - 1));
            __syncthreads();
#pragma unroll
            for (int c = 0; c < NC; ++c)
#pragma unroll
                for (int r = 0; r < 8; ++r) ex[c].at(o + r * Ns) = v[c][r];
            __syncthreads();
#pragma unroll
            for (int c = 0; c < NC; ++c)
#pragma unroll
                for (int q = 0; q < 8; ++q) v[c][q] = ex[c].at(j + q * Q);
        }
    }
    if (RL == 2) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const cplx<T> w = twid(tw, j + i * Q, 1, inv);
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const cplx<T> a = v[c][i], b = cmul(v[c][i + 4], w);
                v[c][i] = cadd(a, b);
                v[c][i + 4] = csub(a, b);
            }
        }
    } else if (RL == 4) {
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int jp = j + i * Q;
            const cplx<T> w1 = twid(tw, jp, 1, inv), w2 = twid(tw, 2 * jp, 1, inv),
                          w3 = twid(tw, 3 * jp, 1, inv);
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                cplx<T> a0 = v[c][i], a1 = cmul(v[c][i + 2], w1), a2 = cmul(v[c][i + 4], w2),
                        a3 = cmul(v[c][i + 6], w3);
                dft4(a0, a1, a2, a3, inv);
                v[c][i] = a0; v[c][i + 2] = a1; v[c][i + 4] = a2; v[c][i + 6] = a3;
            }
        }
    }
}

// Number of 16-byte chunks in B complex values.
template <typename T, int B>
struct Chunks {
    static constexpr int PER_ROW = (B * (int)sizeof(cplx<T>)) / 16;
};

// ---- y pass: tiles of B kx columns x n rows of one (c, z) plane ------------
// Columns kx0 <= kx < kx1 (kx0 a multiple of B). block = B * n/8 threads;
// smem: table (n) | staging (n * B) | exchange (B * padded_len(n)).
template <typename T, int n, int B>
__global__ void __launch_bounds__(B * (n / 8)) k_fftq_y(cplx<T>* __restrict__ spec, int kx0, int kx1, int Mz,
                                                        int hxp, const cplx<T>* __restrict__ twy,
                                                        int inverse) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int Q = n / 8, CPR = Chunks<T, B>::PER_ROW;
    constexpr int NT = B * (n / 8);
    cplx<T>* tw = reinterpret_cast<cplx<T>*>(smem_raw);
    cplx<T>* stage = tw + n;
    cplx<T>* ex_sm = stage + n * B;
    load_table(tw, twy, n);
    const int b = threadIdx.x % B, j = threadIdx.x / B;
    const int tiles_x = (kx1 - kx0 + B - 1) / B;
    const int ntiles = tiles_x * Mz * 3;
    const int64_t plane_elems = (int64_t)n * hxp;
    auto issue = [&](int t) {
        const int tx = t % tiles_x, pz = t / tiles_x;   // pz = c * Mz + z
        const cplx<T>* src = spec + (int64_t)pz * plane_elems + kx0 + tx * B;
        for (int q = threadIdx.x; q < n * CPR; q += NT) {
            const int y = q / CPR, part = q - y * CPR;
            cp_async16(reinterpret_cast<unsigned char*>(stage + y * B) + 16 * part,
                       reinterpret_cast<const unsigned char*>(src + (int64_t)y * hxp) + 16 * part);
        }
        cp_async_commit();
    };
    int t = blockIdx.x;
    if (t < ntiles) issue(t);
    Exchange<T> ex[1] = {Exchange<T>{ex_sm, b, B}};
    for (; t < ntiles; t += gridDim.x) {
        cp_async_wait_all();
        __syncthreads();
        cplx<T> v[1][8];
#pragma unroll
        for (int q = 0; q < 8; ++q) v[0][q] = stage[(j + q * Q) * B + b];
        __syncthreads();
        if (t + (int)gridDim.x < ntiles) issue(t + gridDim.x);
        fft_lines_lockstep<T, n, 1>(v, j, ex, tw, inverse != 0);
        const int tx = t % tiles_x, pz = t / tiles_x;
        const int kx = kx0 + tx * B + b;
        if (kx < kx1) {
            cplx<T>* dst = spec + (int64_t)pz * plane_elems + kx;
#pragma unroll
            for (int q = 0; q < 8; ++q) dst[(int64_t)(j + q * Q) * hxp] = v[0][q];
        }
    }
}

// ---- z pass + projector: tiles of B kx columns x n z of one y, 3 components --
// Columns kx0 <= kx < kx1 (kx0 a multiple of B). block = B * n/8 threads;
// smem: table (n) | staging (3 n B) | exchange (3 B padded_len(n)).
template <typename T, int n, int B>
__global__ void __launch_bounds__(B * (n / 8)) k_fftq_z_stokes(
    cplx<T>* __restrict__ spec, int kx0, int kx1, int My, int hxp, const cplx<T>* __restrict__ twz,
    const T* __restrict__ kxv, const T* __restrict__ kyv, const T* __restrict__ kzv, T inv_mu_M) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int Q = n / 8, CPR = Chunks<T, B>::PER_ROW;
    constexpr int NT = B * (n / 8);
    constexpr int PL = padded_len(n);
    cplx<T>* tw = reinterpret_cast<cplx<T>*>(smem_raw);
    cplx<T>* stage = tw + n;
    cplx<T>* ex_sm = stage + 3 * n * B;
    load_table(tw, twz, n);
    const int b = threadIdx.x % B, j = threadIdx.x / B;
    const int tiles_x = (kx1 - kx0 + B - 1) / B;
    const int ntiles = tiles_x * My;
    const int64_t zs = (int64_t)My * hxp;
    const int64_t cs = (int64_t)n * zs;
    auto issue = [&](int t) {
        const int tx = t % tiles_x, y = t / tiles_x;
        const cplx<T>* src = spec + (int64_t)y * hxp + kx0 + tx * B;
        for (int q = threadIdx.x; q < 3 * n * CPR; q += NT) {
            const int row = q / CPR, part = q - row * CPR;   // row = c * n + z
            const int c = row / n, z = row - c * n;
            cp_async16(reinterpret_cast<unsigned char*>(stage + row * B) + 16 * part,
                       reinterpret_cast<const unsigned char*>(src + c * cs + z * zs) + 16 * part);
        }
        cp_async_commit();
    };
    int t = blockIdx.x;
    if (t < ntiles) issue(t);
    const Exchange<T> ex[3] = {Exchange<T>{ex_sm, b, B}, Exchange<T>{ex_sm + B * PL, b, B},
                               Exchange<T>{ex_sm + 2 * B * PL, b, B}};
    for (; t < ntiles; t += gridDim.x) {
        cp_async_wait_all();
        __syncthreads();
        cplx<T> v[3][8];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int q = 0; q < 8; ++q) v[c][q] = stage[(c * n + j + q * Q) * B + b];
        __syncthreads();
        if (t + (int)gridDim.x < ntiles) issue(t + gridDim.x);
        const int tx = t % tiles_x, y = t / tiles_x;
        const int kx = kx0 + tx * B + b;
        fft_lines_lockstep<T, n, 3>(v, j, ex, tw, false);
        const T k1 = kx < kx1 ? kxv[kx] : T(0);
        const T k2 = kyv[y];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const T k3 = kzv[j + q * Q];
            const T ksq = k1 * k1 + k2 * k2 + k3 * k3;
            if (ksq == T(0)) {
                v[0][q] = v[1][q] = v[2][q] = cplx<T>{T(0), T(0)};
            } else {
                const T inv_k2 = T(1) / ksq;
                const T sc = inv_mu_M * inv_k2;
                const T dre = (k1 * v[0][q].x + k2 * v[1][q].x + k3 * v[2][q].x) * inv_k2;
                const T dim = (k1 * v[0][q].y + k2 * v[1][q].y + k3 * v[2][q].y) * inv_k2;
                v[0][q] = cplx<T>{sc * (v[0][q].x - k1 * dre), sc * (v[0][q].y - k1 * dim)};
                v[1][q] = cplx<T>{sc * (v[1][q].x - k2 * dre), sc * (v[1][q].y - k2 * dim)};
                v[2][q] = cplx<T>{sc * (v[2][q].x - k3 * dre), sc * (v[2][q].y - k3 * dim)};
            }
        }
        fft_lines_lockstep<T, n, 3>(v, j, ex, tw, true);
        if (kx < kx1) {
            cplx<T>* col = spec + (int64_t)y * hxp + kx;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int64_t o = (int64_t)(j + q * Q) * zs;
                col[o] = v[0][q];
                col[cs + o] = v[1][q];
                col[2 * cs + o] = v[2][q];
            }
        }
    }
}

template <typename T>
using YPipeKernel = void (*)(cplx<T>*, int, int, int, int, const cplx<T>*, int);
template <typename T>
using ZPipeKernel = void (*)(cplx<T>*, int, int, int, int, const cplx<T>*, const T*, const T*, const T*, T);

template <typename T>
size_t ypipe_smem(int n, int B) {
    return (size_t)(n + n * B + B * padded_len(n)) * sizeof(cplx<T>);
}
template <typename T>
size_t zpipe_smem(int n, int B) {
    return (size_t)(n + 3 * n * B + 3 * B * padded_len(n)) * sizeof(cplx<T>);
}

// Instantiated (n, B): y with B*n/8 <= 1024 threads, z with B*n/8 <= 256.
template <typename T>
YPipeKernel<T> ypipe_kernel(int n, int B) {
#define FFCM_YP(NN, BB) if (n == NN && B == BB) return k_fftq_y<T, NN, BB>;
    FFCM_YP(32, 8) FFCM_YP(32, 16) FFCM_YP(64, 8) FFCM_YP(64, 16) FFCM_YP(128, 8) FFCM_YP(128, 16)
    FFCM_YP(256, 4) FFCM_YP(256, 8) FFCM_YP(256, 16) FFCM_YP(512, 4) FFCM_YP(512, 8)
    FFCM_YP(1024, 4) FFCM_YP(1024, 8)
#undef FFCM_YP
    return nullptr;
}

template <typename T>
ZPipeKernel<T> zpipe_kernel(int n, int B) {
#define FFCM_ZP(NN, BB) if (n == NN && B == BB) return k_fftq_z_stokes<T, NN, BB>;
    FFCM_ZP(32, 8) FFCM_ZP(32, 16) FFCM_ZP(64, 4) FFCM_ZP(64, 8) FFCM_ZP(128, 2) FFCM_ZP(128, 4)
    FFCM_ZP(256, 2) FFCM_ZP(256, 4) FFCM_ZP(512, 2) FFCM_ZP(512, 4) FFCM_ZP(1024, 2)
#undef FFCM_ZP
    return nullptr;
}

}  // namespace ffcm
