// Conjugate gradients on the mobility operator: the resistance problem
// M(Y) F = V for F, with M the FFCM mobility at fixed positions. The reference
// declares its operator symmetric positive definite for exactly this use
// (src/mobility.jl:161-162, `issymmetric`/`isposdef` on FFCMMobility), so
// that Krylov solvers such as IterativeSolvers.jl's `cg` accept it.
//
// Iteration: Hestenes & Stiefel (1952), unpreconditioned, in the order of
// IterativeSolvers.jl 0.9's CGIterable (third-party, not part of the
// reference): p = r + beta p; q = M p; alpha = |r|^2 / p.q; x += alpha p;
// r -= alpha q; beta = |r_new|^2 / |r|^2. Stopping rule also as there: stop
// once |r| <= max(reltol |r0|, abstol) (r0 the residual of the initial guess)
// or after maxiter iterations.
//
// Vectors are the caller's 3 x N column-major layout (entry 3(n-1)+i).
// Dot products accumulate in double with a fixed grid, a fixed per-thread
// stride and a fixed reduction tree, so a solve is bit-reproducible. Each
// dot product is finished by the last block to arrive (threadfence + arrival
// counter), which also updates the scalar state, so one CG iteration is the
// mobility application plus three small grid kernels, and the loop runs on
// the device as a CUDA-graph while node whose condition the update kernel
// sets.
#pragma once

#include <cuda_runtime.h>
#include "common.cuh"

namespace ffcm {

constexpr int CG_BLOCKS = 296;  // two per SM
constexpr int CG_THREADS = 256;

enum : int {
    CG_RUNNING = 0,
    CG_CONVERGED = 1,
    CG_MAXITER = 2,
    CG_BREAKDOWN = 3,     // p.q <= 0 or a non-finite scalar
    CG_DEVICE_ERROR = 4,  // a kernel of the mobility application raised its error flag
};

struct CgState {
    double rr;      // |r|^2 of the current residual
    double rr0;     // |r0|^2
    double thresh;  // stop once |r| <= thresh
    double alpha, beta;
    int iter, maxiter, status;
    unsigned int arrived;  // blocks done with the current dot product
    double part[CG_BLOCKS];
};

// Sum over the block; the result is valid in thread 0.
__device__ __forceinline__ double cg_block_sum(double v) {
    __shared__ double red[CG_THREADS / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();  // red may still be read by a previous call
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = threadIdx.x < (CG_THREADS / 32) ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    }
    return v;
}

// Posts this block's partial sum; returns the full sum (valid in thread 0 of
// the last block to arrive) and whether this block is that one. The partials
// are summed in block order, independent of the arrival order.
__device__ __forceinline__ bool cg_finish_dot(double v, CgState* st, double& total) {
    __shared__ bool last;
    v = cg_block_sum(v);
    if (threadIdx.x == 0) {
        st->part[blockIdx.x] = v;
        __threadfence();
        last = atomicAdd(&st->arrived, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double s = 0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += CG_THREADS) s += ((volatile double*)st->part)[i];
    total = cg_block_sum(s);
    if (threadIdx.x == 0) st->arrived = 0;
    return true;
}

__device__ __forceinline__ double cg_load(float v) { return (double)v; }
__device__ __forceinline__ double cg_load(double v) { return v; }

// Start: r = V - q (q = M x0, or no q for a zero initial guess), p = 0,
// |r0|^2, the threshold and the initial status.
template <typename T>
__global__ void __launch_bounds__(CG_THREADS) k_cg_start(int64_t n, const T* __restrict__ V, const T* __restrict__ q,
                                                         T* __restrict__ r, T* __restrict__ p, CgState* st,
                                                         double reltol, double abstol, int maxiter) {
    double acc = 0;
    for (int64_t i = blockIdx.x * (int64_t)CG_THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * CG_THREADS) {
        const T ri = q ? T(V[i] - q[i]) : V[i];
        r[i] = ri;
        p[i] = T(0);
        acc += cg_load(ri) * cg_load(ri);
    }
    double rr;
    if (cg_finish_dot(acc, st, rr) && threadIdx.x == 0) {
        const double res = sqrt(rr);
        const double thresh = fmax(reltol * res, abstol);
        st->rr = rr;
        st->rr0 = rr;
        st->thresh = thresh;
        st->alpha = 0;
        st->beta = 0;
        st->iter = 0;
        st->maxiter = maxiter;
        st->status = !isfinite(rr) ? CG_BREAKDOWN : res <= thresh ? CG_CONVERGED : maxiter <= 0 ? CG_MAXITER : CG_RUNNING;
    }
}

// First node of the solve graph: enter the loop only if the start left it running.
__global__ void k_cg_gate(const CgState* st, cudaGraphConditionalHandle loop) {
    if (threadIdx.x == 0 && blockIdx.x == 0) cudaGraphSetConditional(loop, st->status == CG_RUNNING ? 1u : 0u);
}

// p = r + beta p
template <typename T>
__global__ void __launch_bounds__(CG_THREADS) k_cg_direction(int64_t n, const T* __restrict__ r, T* __restrict__ p,
                                                             const CgState* __restrict__ st) {
    const double beta = st->beta;
    for (int64_t i = blockIdx.x * (int64_t)CG_THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * CG_THREADS)
        p[i] = T(cg_load(r[i]) + beta * cg_load(p[i]));
}

// alpha = |r|^2 / p.q
template <typename T>
__global__ void __launch_bounds__(CG_THREADS) k_cg_alpha(int64_t n, const T* __restrict__ p, const T* __restrict__ q,
                                                         CgState* st) {
    double acc = 0;
    for (int64_t i = blockIdx.x * (int64_t)CG_THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * CG_THREADS)
        acc += cg_load(p[i]) * cg_load(q[i]);
    double pq;
    if (cg_finish_dot(acc, st, pq) && threadIdx.x == 0) {
        if (pq > 0 && isfinite(pq)) {
            st->alpha = st->rr / pq;
        } else {
            st->alpha = 0;
            st->status = CG_BREAKDOWN;
        }
    }
}

// x += alpha p; r -= alpha q; |r|^2, beta, the iteration count, the status
// and the loop condition.
template <typename T>
__global__ void __launch_bounds__(CG_THREADS) k_cg_update(int64_t n, T* __restrict__ x, T* __restrict__ r,
                                                          const T* __restrict__ p, const T* __restrict__ q,
                                                          CgState* st, const int* __restrict__ dev_err,
                                                          cudaGraphConditionalHandle loop) {
    const double alpha = st->status == CG_RUNNING ? st->alpha : 0.0;
    double acc = 0;
    for (int64_t i = blockIdx.x * (int64_t)CG_THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * CG_THREADS) {
        const T xi = T(cg_load(x[i]) + alpha * cg_load(p[i]));
        const T ri = T(cg_load(r[i]) - alpha * cg_load(q[i]));
        x[i] = xi;
        r[i] = ri;
        acc += cg_load(ri) * cg_load(ri);
    }
    double rr;
    if (cg_finish_dot(acc, st, rr) && threadIdx.x == 0) {
        int status = st->status;
        if (status == CG_RUNNING) {
            st->beta = rr / st->rr;
            st->rr = rr;
            st->iter += 1;
            if (!isfinite(rr)) status = CG_BREAKDOWN;
            else if (sqrt(rr) <= st->thresh) status = CG_CONVERGED;
            else if (st->iter >= st->maxiter) status = CG_MAXITER;
        }
        if (*dev_err) status = CG_DEVICE_ERROR;
        st->status = status;
        cudaGraphSetConditional(loop, status == CG_RUNNING ? 1u : 0u);
    }
}

}  // namespace ffcm
