// y pass and z pass + projector with tiles brought in by the tensor memory
// accelerator.
//
// Same computation as k_fftq_z_stokes (z forward of the three components in
// lockstep, projector (I - k k^T/k^2)/(mu k^2 M), z inverse). A persistent
// block loops over tiles of B kx columns x one y x all (c, z) rows. One thread
// loads a tile with a few tiled bulk copies (cp.async.bulk.tensor) described
// by a tensor map over the spectrum, dims (kx, y, 3 Mz) -- the component and
// z axes merge because a component's stride is Mz times the z stride -- into
// a staging buffer, completing on an mbarrier; as soon as the block has moved
// the tile into registers, the next tile's copy is issued, so it lands while
// the block transforms. The transformed tile goes back the same way: the
// block writes it into its (then idle) exchange region in the staging layout
// and one thread issues tiled bulk stores through the same tensor map, waited
// for (reads of shared memory done) before the region is written again. A
// tile may extend into the padding columns of the spectrum pitch; those are
// transformed and stored like the others and never read as data. Each block
// fills and drains only its own shared memory, from and to this GPU's memory.
// The x coordinate of every copy is a multiple of B complex values (B even),
// so it starts on a 16-byte boundary.
#pragma once

#include <cuda.h>

#include "bulk_copy.cuh"
#include "common.cuh"
#include "fft_pipe.cuh"

namespace ffcm {

// Tensor-map element: 8-byte words; a complex value is 1 (float) or 2 (double).
template <typename T>
struct TmaElem {
    static constexpr int PER_CPLX = (int)(sizeof(cplx<T>) / 8);
};

// Rows of (c, z) per tiled copy (box dimensions are at most 256).
__host__ __device__ constexpr int tma_zbox(int n) { return n < 256 ? n : 256; }

__device__ __forceinline__ void tma_load_3d(void* dst_smem, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst_smem)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}

// Tiled bulk store of a box from this block's shared memory (128-byte aligned)
// to the tensor at (x, y, z), as a bulk group of the calling thread. The
// block's writes of the box must be made visible to the async proxy first
// (fence_proxy_async_smem by the writers, then a barrier).
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, int x, int y, int z, const void* src_smem) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y), "r"(z), "r"(smem_addr(src_smem))
                 : "memory");
}

// block = B * n/8 threads; smem: up to 128 bytes of alignment slack | staging
// (3 n B, 128-byte aligned) | table (n) | exchange (3 B padded_len(n)).
template <typename T, int n, int B>
__global__ void __launch_bounds__(B * (n / 8)) k_fftt_z_stokes(
    const __grid_constant__ CUtensorMap tmap, cplx<T>* __restrict__ spec, int kx0, int kx1, int My, int hxp,
    const cplx<T>* __restrict__ twz, const T* __restrict__ kxv, const T* __restrict__ kyv,
    const T* __restrict__ kzv, T inv_mu_M, int* __restrict__ err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar;
    constexpr int Q = n / 8, PL = padded_len(n), ZB = tma_zbox(n), NCOPY = 3 * n / ZB;
    constexpr unsigned TILE_BYTES = (unsigned)(3 * n * B * sizeof(cplx<T>));
    // staging starts on a 128-byte boundary (the size includes 128 bytes of slack)
    cplx<T>* stage = reinterpret_cast<cplx<T>*>(smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u));
    cplx<T>* tw = stage + 3 * n * B;
    cplx<T>* ex_sm = tw + n;
    load_table(tw, twz, n);
    const int b = threadIdx.x % B, j = threadIdx.x / B;
    const int tiles_x = (kx1 - kx0 + B - 1) / B;
    const int ntiles = tiles_x * My;
    auto issue = [&](int t) {   // one thread, after a barrier
        const int tx = t % tiles_x, y = t / tiles_x;
        fence_proxy_async_smem();   // the block's reads of the staging buffer come first
        mbar_arrive_expect(&bar, TILE_BYTES);
#pragma unroll
        for (int k = 0; k < NCOPY; ++k)
            tma_load_3d(stage + k * ZB * B, &tmap, (kx0 + tx * B) * TmaElem<T>::PER_CPLX, y, k * ZB, &bar);
    };
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        if ((int)blockIdx.x < ntiles) issue(blockIdx.x);
    }
    __syncthreads();
    const Exchange<T> ex[3] = {Exchange<T>{ex_sm, b, B}, Exchange<T>{ex_sm + B * PL, b, B},
                               Exchange<T>{ex_sm + 2 * B * PL, b, B}};
    // the result tile leaves through the exchange region, laid out like the
    // staging buffer ([c n + z][B], 128-byte aligned), by tiled bulk stores
    cplx<T>* out = ex_sm;
    static_assert(3 * n * B <= 3 * B * PL, "the result tile must fit the exchange region");
    unsigned phase = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, phase ^= 1u) {
        const bool landed = mbar_wait_bounded(&bar, phase, 1 << 22);
        if (__syncthreads_or(!landed)) {
            // the tile did not arrive: report, give the copies one more
            // bounded chance to finish, and leave
            if (threadIdx.x == 0) {
                atomicOr(err, DEVERR_COPY_TIMEOUT);
                bulk_wait_all();
            }
            mbar_wait_bounded(&bar, phase, 1 << 22);
            return;
        }
        cplx<T> v[3][8];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int q = 0; q < 8; ++q) v[c][q] = stage[(c * n + j + q * Q) * B + b];
        // the previous tile's stores have read the exchange region before
        // anyone writes it again
        if (threadIdx.x == 0) bulk_wait_read_all();
        __syncthreads();   // the staging buffer is free for the next tile
        if (threadIdx.x == 0 && t + (int)gridDim.x < ntiles) issue(t + gridDim.x);
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
        __syncthreads();   // every exchange read of the inverse transform is done
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int q = 0; q < 8; ++q) out[(c * n + j + q * Q) * B + b] = v[c][q];
        fence_proxy_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
#pragma unroll
            for (int k = 0; k < NCOPY; ++k)
                tma_store_3d(&tmap, (kx0 + tx * B) * TmaElem<T>::PER_CPLX, y, k * ZB, out + k * ZB * B);
            bulk_commit();
        }
    }
    if (threadIdx.x == 0) bulk_wait_all();
}

// z pass + projector on wide tiles transformed in place. The passes above
// keep a separate exchange region beside a staging buffer that is refilled
// while they compute, which caps a tile at 8 kx columns at z length 512 and 4
// at 1024: each z row of a tile is then a 64- or 32-byte piece of memory, and
// at 32 bytes the pass reaches 1.2 TB/s. Here a tile of B columns (B = 16 at
// 512: 128-byte pieces; B = 8 at 1024) is loaded by tiled bulk copies into
// the staging buffer, and the three components are transformed one after the
// other in that buffer (it is also their exchange space): forward, projector,
// inverse, then tiled bulk stores. Loads are not overlapped with the block's
// own compute (one tile buffer); one block per SM, other SMs interleave.
// block = B * n/8 threads; smem: up to 128 bytes of alignment slack | staging
// (3 n B, 128-byte aligned) | table (n).
template <typename T, int n, int B>
__global__ void __launch_bounds__(B * (n / 8)) k_fftr_z_stokes(
    const __grid_constant__ CUtensorMap tmap, cplx<T>* __restrict__ spec, int kx0, int kx1, int My, int hxp,
    const cplx<T>* __restrict__ twz, const T* __restrict__ kxv, const T* __restrict__ kyv,
    const T* __restrict__ kzv, T inv_mu_M, int* __restrict__ err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar;
    constexpr int Q = n / 8, ZB = tma_zbox(n), NCOPY = 3 * n / ZB;
    constexpr unsigned TILE_BYTES = (unsigned)(3 * n * B * sizeof(cplx<T>));
    cplx<T>* stage = reinterpret_cast<cplx<T>*>(smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u));
    cplx<T>* tw = stage + 3 * n * B;
    load_table(tw, twz, n);
    const int b = threadIdx.x % B, j = threadIdx.x / B;
    const int tiles_x = (kx1 - kx0 + B - 1) / B;
    const int ntiles = tiles_x * My;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    // component c of the tile: stage[(c n + z) B + b]
    auto comp = [&](int c) { return ExchangeDense<T>{stage + c * n * B, b, B}; };
    unsigned phase = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, phase ^= 1u) {
        const int tx = t % tiles_x, y = t / tiles_x;
        if (threadIdx.x == 0) {
            bulk_wait_read_all();       // the previous tile's stores have read the buffer
            fence_proxy_async_smem();   // and so have the block's own accesses
            mbar_arrive_expect(&bar, TILE_BYTES);
#pragma unroll
            for (int k = 0; k < NCOPY; ++k)
                tma_load_3d(stage + k * ZB * B, &tmap, (kx0 + tx * B) * TmaElem<T>::PER_CPLX, y, k * ZB, &bar);
        }
        const bool landed = mbar_wait_bounded(&bar, phase, 1 << 22);
        if (__syncthreads_or(!landed)) {
            if (threadIdx.x == 0) {
                atomicOr(err, DEVERR_COPY_TIMEOUT);
                bulk_wait_all();
            }
            mbar_wait_bounded(&bar, phase, 1 << 22);
            return;
        }
        // forward transforms, one component at a time, in place
#pragma unroll 1
        for (int c = 0; c < 3; ++c) {
            const ExchangeDense<T> ex = comp(c);
            cplx<T> v[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) v[q] = ex.at(j + q * Q);
            fft_line_regs<T, n, false, ExchangeDense<T>>(v, j, ex, tw, 1, false);
            __syncthreads();   // every exchange read of this component is done
#pragma unroll
            for (int q = 0; q < 8; ++q) ex.at(j + q * Q) = v[q];
        }
        __syncthreads();
        // projector (I - k k^T / k^2) / (mu k^2 M), k = 0 -> 0
        const int kx = kx0 + tx * B + b;
        const T k1 = kx < kx1 ? kxv[kx] : T(0);
        const T k2 = kyv[y];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int z = j + q * Q;
            const T k3 = kzv[z];
            const ExchangeDense<T> e0 = comp(0), e1 = comp(1), e2 = comp(2);
            cplx<T> a = e0.at(z), bb = e1.at(z), cc = e2.at(z);
            const T ksq = k1 * k1 + k2 * k2 + k3 * k3;
            if (ksq == T(0)) {
                a = bb = cc = cplx<T>{T(0), T(0)};
            } else {
                const T inv_k2 = T(1) / ksq;
                const T sc = inv_mu_M * inv_k2;
                const T dre = (k1 * a.x + k2 * bb.x + k3 * cc.x) * inv_k2;
                const T dim = (k1 * a.y + k2 * bb.y + k3 * cc.y) * inv_k2;
                a = cplx<T>{sc * (a.x - k1 * dre), sc * (a.y - k1 * dim)};
                bb = cplx<T>{sc * (bb.x - k2 * dre), sc * (bb.y - k2 * dim)};
                cc = cplx<T>{sc * (cc.x - k3 * dre), sc * (cc.y - k3 * dim)};
            }
            e0.at(z) = a;
            e1.at(z) = bb;
            e2.at(z) = cc;
        }
        __syncthreads();
        // inverse transforms
#pragma unroll 1
        for (int c = 0; c < 3; ++c) {
            const ExchangeDense<T> ex = comp(c);
            cplx<T> v[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) v[q] = ex.at(j + q * Q);
            fft_line_regs<T, n, false, ExchangeDense<T>>(v, j, ex, tw, 1, true);
            __syncthreads();
#pragma unroll
            for (int q = 0; q < 8; ++q) ex.at(j + q * Q) = v[q];
        }
        fence_proxy_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
#pragma unroll
            for (int k = 0; k < NCOPY; ++k)
                tma_store_3d(&tmap, (kx0 + tx * B) * TmaElem<T>::PER_CPLX, y, k * ZB, stage + k * ZB * B);
            bulk_commit();
        }
    }
    if (threadIdx.x == 0) bulk_wait_all();
}

// Complex values of one plane's exchange region of the TMA y pass: B lines
// of padded_len(n), rounded up to 128 bytes so that every region (the
// source of a tiled bulk store) starts on a 128-byte boundary.
template <typename T>
__host__ __device__ constexpr int ytma_exchange(int n, int B) {
    return (int)(((size_t)B * padded_len(n) * sizeof(cplx<T>) + 127) / 128 * 128 / sizeof(cplx<T>));
}

// y pass, same scheme: a tile is B kx columns x all n rows y of NP
// consecutive (c, z) planes (tensor coordinate z = c * Mz + z), each plane
// loaded with n / min(256, n) tiled copies into its staging [y][B]. With
// NP > 1 each thread transforms one line of every plane in lockstep (the
// twiddles and exchange barriers of a stage serve NP lines).
// block = B * n/8 threads; smem: slack | staging (NP n B) | table (n) |
// exchange (NP B padded_len(n)).
template <typename T, int n, int B, int NP = 1>
__global__ void __launch_bounds__(B * (n / 8)) k_fftt_y(const __grid_constant__ CUtensorMap tmap,
                                                        cplx<T>* __restrict__ spec, int kx0, int kx1, int Mz,
                                                        int hxp, const cplx<T>* __restrict__ twy, int inverse,
                                                        int* __restrict__ err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar;
    constexpr int Q = n / 8, YB = tma_zbox(n), NCOPY = n / YB;
    constexpr unsigned TILE_BYTES = (unsigned)(NP * n * B * sizeof(cplx<T>));
    constexpr int EXS = ytma_exchange<T>(n, B);   // one plane's exchange region
    cplx<T>* stage = reinterpret_cast<cplx<T>*>(smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u));
    cplx<T>* tw = stage + NP * n * B;
    cplx<T>* ex_sm = tw + n;
    load_table(tw, twy, n);
    const int b = threadIdx.x % B, j = threadIdx.x / B;
    const int tiles_x = (kx1 - kx0 + B - 1) / B;
    const int ntiles = tiles_x * (Mz * 3 / NP);
    auto issue = [&](int t) {   // one thread, after a barrier
        const int tx = t % tiles_x, pz = (t / tiles_x) * NP;
        fence_proxy_async_smem();   // the block's reads of the staging buffer come first
        mbar_arrive_expect(&bar, TILE_BYTES);
#pragma unroll
        for (int pl = 0; pl < NP; ++pl)
#pragma unroll
            for (int k = 0; k < NCOPY; ++k)
                tma_load_3d(stage + (pl * NCOPY + k) * YB * B, &tmap, (kx0 + tx * B) * TmaElem<T>::PER_CPLX,
                            k * YB, pz + pl, &bar);
    };
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        if ((int)blockIdx.x < ntiles) issue(blockIdx.x);
    }
    __syncthreads();
    Exchange<T> ex[NP];
#pragma unroll
    for (int pl = 0; pl < NP; ++pl) ex[pl] = Exchange<T>{ex_sm + pl * EXS, b, B};
    // the result tiles leave through the exchange regions ([y][B] per plane,
    // 128-byte aligned) by tiled bulk stores
    static_assert(n * B <= EXS, "a result tile must fit its exchange region");
    static_assert((EXS * sizeof(cplx<T>)) % 128 == 0, "exchange regions start on 128-byte boundaries");
    unsigned phase = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, phase ^= 1u) {
        const bool landed = mbar_wait_bounded(&bar, phase, 1 << 22);
        if (__syncthreads_or(!landed)) {
            if (threadIdx.x == 0) {
                atomicOr(err, DEVERR_COPY_TIMEOUT);
                bulk_wait_all();
            }
            mbar_wait_bounded(&bar, phase, 1 << 22);
            return;
        }
        cplx<T> v[NP][8];
#pragma unroll
        for (int pl = 0; pl < NP; ++pl)
#pragma unroll
            for (int q = 0; q < 8; ++q) v[pl][q] = stage[pl * n * B + (j + q * Q) * B + b];
        if (threadIdx.x == 0) bulk_wait_read_all();   // the previous tile's stores left the exchange regions
        __syncthreads();   // the staging buffer is free for the next tile
        if (threadIdx.x == 0 && t + (int)gridDim.x < ntiles) issue(t + gridDim.x);
        fft_lines_lockstep<T, n, NP>(v, j, ex, tw, inverse != 0);
        const int tx = t % tiles_x, pz = (t / tiles_x) * NP;
        __syncthreads();   // every exchange read of the transform is done
#pragma unroll
        for (int pl = 0; pl < NP; ++pl)
#pragma unroll
            for (int q = 0; q < 8; ++q) ex_sm[pl * EXS + (j + q * Q) * B + b] = v[pl][q];
        fence_proxy_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
#pragma unroll
            for (int pl = 0; pl < NP; ++pl)
#pragma unroll
                for (int k = 0; k < NCOPY; ++k)
                    tma_store_3d(&tmap, (kx0 + tx * B) * TmaElem<T>::PER_CPLX, k * YB, pz + pl,
                                 ex_sm + pl * EXS + k * YB * B);
            bulk_commit();
        }
    }
    if (threadIdx.x == 0) bulk_wait_all();
}

template <typename T>
using YTmaKernel = void (*)(const CUtensorMap, cplx<T>*, int, int, int, int, const cplx<T>*, int, int*);

template <typename T>
size_t ytma_smem(int n, int B, int NP = 1) {
    return 128 + (size_t)(NP * n * B + n + NP * ytma_exchange<T>(n, B)) * sizeof(cplx<T>);
}

// y pass with three planes per tile (autotuner kind 3), per (n, B).
template <typename T>
YTmaKernel<T> ytma3_kernel(int n, int B) {
#define FFCM_Y3(NN, BB) if (n == NN && B == BB) return k_fftt_y<T, NN, BB, 3>;
    // the instantiations that fit their register budget without spills
    if constexpr (sizeof(T) == 4) {
        FFCM_Y3(256, 4) FFCM_Y3(512, 4) FFCM_Y3(512, 8) FFCM_Y3(1024, 4)
    } else {
        FFCM_Y3(256, 4) FFCM_Y3(256, 8) FFCM_Y3(512, 4)
    }
#undef FFCM_Y3
    return nullptr;
}

template <typename T>
YTmaKernel<T> ytma_kernel(int n, int B) {
#define FFCM_YT(NN, BB) if (n == NN && B == BB) return k_fftt_y<T, NN, BB>;
    FFCM_YT(32, 8) FFCM_YT(32, 16) FFCM_YT(64, 8) FFCM_YT(64, 16) FFCM_YT(128, 8) FFCM_YT(128, 16)
    FFCM_YT(256, 4) FFCM_YT(256, 8) FFCM_YT(256, 16) FFCM_YT(512, 4) FFCM_YT(512, 8) FFCM_YT(512, 16)
    FFCM_YT(1024, 4) FFCM_YT(1024, 8)
#undef FFCM_YT
    return nullptr;
}

template <typename T>
using ZTmaKernel = void (*)(const CUtensorMap, cplx<T>*, int, int, int, int, const cplx<T>*, const T*,
                            const T*, const T*, T, int*);

template <typename T>
size_t ztma_smem(int n, int B) {
    return 128 + (size_t)(3 * n * B + n + 3 * B * padded_len(n)) * sizeof(cplx<T>);
}

template <typename T>
size_t zin_smem(int n, int B) {
    return 128 + (size_t)(3 * n * B + n) * sizeof(cplx<T>);
}

// In-place wide-tile z pass (k_fftr_z_stokes), per (n, B).
template <typename T>
ZTmaKernel<T> zin_kernel(int n, int B) {
#define FFCM_ZI(NN, BB) if (n == NN && B == BB) return k_fftr_z_stokes<T, NN, BB>;
    FFCM_ZI(256, 16) FFCM_ZI(512, 8) FFCM_ZI(512, 16) FFCM_ZI(1024, 8)
#undef FFCM_ZI
    return nullptr;
}

template <typename T>
ZTmaKernel<T> ztma_kernel(int n, int B) {
#define FFCM_ZT(NN, BB) if (n == NN && B == BB) return k_fftt_z_stokes<T, NN, BB>;
    FFCM_ZT(64, 8) FFCM_ZT(64, 16) FFCM_ZT(128, 4) FFCM_ZT(128, 8) FFCM_ZT(256, 2) FFCM_ZT(256, 4)
    FFCM_ZT(512, 2) FFCM_ZT(512, 4) FFCM_ZT(512, 8) FFCM_ZT(1024, 2) FFCM_ZT(1024, 4)
#undef FFCM_ZT
    return nullptr;
}

}  // namespace ffcm
