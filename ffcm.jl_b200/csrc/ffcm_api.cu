// C ABI of libffcm_b200: configuration (cold path), the six hot-path steps,
// the assembled operator, buffer access and measurement. See
// include/ffcm_b200.h for the contract of every entry point.
#include <algorithm>
#include <limits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "ffcm_b200.h"
#include "common.cuh"
#include "cell_list.cuh"
#include "correct.cuh"
#include "fft.cuh"
#include "spread_interp.cuh"

using namespace ffcm;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    int code = (e == cudaErrorMemoryAllocation) ? FFCM_ERR_OOM : FFCM_ERR_CUDA;
    return fail(code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CUDA_TRY(expr)                                          \
    do {                                                        \
        cudaError_t e_ = (expr);                                \
        if (e_ != cudaSuccess) return cuda_fail(e_, #expr);     \
    } while (0)

#define TRY(expr)                   \
    do {                            \
        int r_ = (expr);            \
        if (r_ != FFCM_OK) return r_; \
    } while (0)

std::string fmt(double v) {
    char b[64];
    snprintf(b, sizeof b, "%.9g", v);
    return b;
}

// Restores the caller's current device on scope exit.
struct DeviceGuard {
    int prev = -1;
    bool ok = false;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) == cudaSuccess && cudaSetDevice(dev) == cudaSuccess) ok = true;
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// ---------------------------------------------------------------------------
// Cold path, in the working precision T (src/config.jl:288-380)
// ---------------------------------------------------------------------------
template <typename T>
struct Derived {
    int32_t num_cells[3];
    T cell_size[3], inv_cell_size[3];
    T sigma, Sigma, h, inv_h;
};

constexpr double kPi = 3.14159265358979323846;

template <typename T>
int validate_T(const double* Ld, double R_cd, int64_t N, double ad, double ratiod,
               const int32_t* M, int32_t M_G, double mud, int32_t planning, int32_t threads) {
    const T L[3] = {T(Ld[0]), T(Ld[1]), T(Ld[2])};
    const T R_c = T(R_cd), a = T(ad), ratio = T(ratiod), mu = T(mud);
    if (!(R_c > T(0))) return fail(FFCM_ERR_ARGUMENT, "R_c must be positive");
    if (!(L[0] > T(0) && L[1] > T(0) && L[2] > T(0)))
        return fail(FFCM_ERR_ARGUMENT, "L components must be positive");
    const T minL = std::min(L[0], std::min(L[1], L[2]));
    if (!(R_c <= minL / T(2)))
        return fail(FFCM_ERR_ARGUMENT, "R_c must be at most half the smallest box length;got R_c = " +
                                           fmt(R_c) + ", min(L)/2 = " + fmt(minL / T(2)));
    if (!(N > 0)) return fail(FFCM_ERR_ARGUMENT, "N must be positive");
    if (!(a == T(1)))
        return fail(FFCM_ERR_ARGUMENT,
                    "non-unit particle radius not yet implemented; only a = 1 is supported, got a = " +
                        fmt(a));
    if (!(ratio >= T(1)))
        return fail(FFCM_ERR_ARGUMENT, "kernel widths ratio must be at least 1; got " + fmt(ratio));
    if (!(M_G >= 2)) return fail(FFCM_ERR_ARGUMENT, "M_G must be at least 2; got " + std::to_string(M_G));
    if (!(M[0] >= 1 && M[1] >= 1 && M[2] >= 1))
        return fail(FFCM_ERR_ARGUMENT, "num_grid_points components must each be >= 1");
    const int32_t minM = std::min(M[0], std::min(M[1], M[2]));
    if (!(M_G <= minM))
        return fail(FFCM_ERR_ARGUMENT, "M_G must not exceed the grid on any axis; got M_G = " +
                                           std::to_string(M_G) +
                                           ", min(num_grid_points) = " + std::to_string(minM));
    if (!(mu > T(0))) return fail(FFCM_ERR_ARGUMENT, "viscosity must be positive; got " + fmt(mu));
    if (planning < FFCM_FFT_ESTIMATE || planning > FFCM_FFT_PATIENT)
        return fail(FFCM_ERR_ARGUMENT, "fft_planning must be :estimate, :measure, or :patient; got " +
                                           std::to_string(planning));
    if (threads < 1)
        return fail(FFCM_ERR_ARGUMENT, "fft_threads must be at least 1; got " + std::to_string(threads));
    return FFCM_OK;
}

template <typename T>
int derive_T(const double* Ld, double R_cd, double ad, double ratiod, const int32_t* M,
             Derived<T>& d) {
    const T L[3] = {T(Ld[0]), T(Ld[1]), T(Ld[2])};
    const T R_c = T(R_cd), a = T(ad), ratio = T(ratiod);
    for (int i = 0; i < 3; ++i) {
        const T q = std::floor(L[i] / R_c);
        if (!(q < T(2147483647.0)))
            return fail(FFCM_ERR_UNSUPPORTED, "L/R_c exceeds the Int32 cell-index range");
        d.num_cells[i] = std::max((int32_t)q, (int32_t)3);
        d.cell_size[i] = L[i] / T(d.num_cells[i]);
        d.inv_cell_size[i] = T(1) / d.cell_size[i];
    }
    d.sigma = a / std::sqrt(T(kPi));
    d.Sigma = ratio * d.sigma;
    T hx[3];
    for (int i = 0; i < 3; ++i) hx[i] = L[i] / T(M[i]);
    const T rel_tol = std::sqrt(std::numeric_limits<T>::epsilon());
    const bool iso = std::abs(hx[1] - hx[0]) <= rel_tol * hx[0] &&
                     std::abs(hx[2] - hx[0]) <= rel_tol * hx[0];
    if (!iso)
        return fail(FFCM_ERR_ARGUMENT,
                    "anisotropic grid spacing not supported (paper §3 assumes uniform h); L_i/M_i = (" +
                        fmt(hx[0]) + ", " + fmt(hx[1]) + ", " + fmt(hx[2]) + ")");
    d.h = hx[0];
    d.inv_h = T(1) / d.h;
    return FFCM_OK;
}

// Radix plan for a complex FFT of length n (radix 8/4/2 first, then odd primes).
int make_plan(int n, int tw_stride, FftPlan& p) {
    p.n = n;
    p.tw_stride = tw_stride;
    p.nstages = 0;
    int m = n;
    auto push = [&](int r) {
        if (p.nstages >= FFT_MAX_STAGES) return false;
        p.radix[p.nstages++] = r;
        return true;
    };
    while (m % 8 == 0) { if (!push(8)) return FFCM_ERR_UNSUPPORTED; m /= 8; }
    while (m % 4 == 0) { if (!push(4)) return FFCM_ERR_UNSUPPORTED; m /= 4; }
    while (m % 2 == 0) { if (!push(2)) return FFCM_ERR_UNSUPPORTED; m /= 2; }
    for (int q = 3; m > 1; q += 2) {
        while (m % q == 0) {
            if (q > FFT_MAX_GENERIC_RADIX)
                return fail(FFCM_ERR_UNSUPPORTED,
                            "grid dimension has a prime factor above " +
                                std::to_string(FFT_MAX_GENERIC_RADIX) + " (" + std::to_string(q) + ")");
            if (!push(q)) return FFCM_ERR_UNSUPPORTED;
            m /= q;
        }
    }
    return FFCM_OK;
}

int pow2_floor(int v) {
    int p = 1;
    while (p * 2 <= v) p *= 2;
    return p;
}

// ---------------------------------------------------------------------------
// Engine: device buffers and kernels for one element type
// ---------------------------------------------------------------------------
struct EngineBase {
    virtual ~EngineBase() = default;
    virtual int wrap_hash(const void* Y, bool wrap, bool hash, cudaStream_t s) = 0;
    virtual int sort(const void* F, cudaStream_t s) = 0;
    virtual int spread(cudaStream_t s) = 0;
    virtual int stokes(cudaStream_t s) = 0;
    virtual int interp(void* V, cudaStream_t s) = 0;
    virtual int correct(void* V, cudaStream_t s) = 0;
    virtual void* Y_in() = 0;
    virtual void* F_in() = 0;
    virtual void* V_out() = 0;
};

}  // namespace

struct ffcm_handle {
    int32_t dtype = FFCM_FLOAT32;
    int32_t device = 0;
    int64_t N = 0;
    int32_t M[3] = {0, 0, 0};
    int32_t M_G = 0;
    int32_t num_cells[3] = {0, 0, 0};
    int64_t ncell = 0;
    size_t esize = 4;
    cudaStream_t stream = nullptr;
    int* d_err = nullptr;
    int* h_err = nullptr;
    int64_t launches = 0;
    // profiling
    bool profiling = false;
    std::vector<cudaEvent_t> events;
    size_t next_event = 0;
    std::vector<std::pair<int, size_t>> recorded;  // (stage, index of the start event)
    std::unique_ptr<EngineBase> eng;
    // host copies of derived data for get_buffer
    std::vector<double> kx, ky, kz;

    cudaStream_t pick(void* s) const { return s ? static_cast<cudaStream_t>(s) : stream; }
};

namespace {

// Records a CUDA event pair around one stage when profiling is on.
struct StageScope {
    ffcm_handle* h;
    int stage;
    cudaStream_t s;
    size_t idx = SIZE_MAX;
    StageScope(ffcm_handle* h_, int stage_, cudaStream_t s_) : h(h_), stage(stage_), s(s_) {
        if (h->profiling && h->next_event + 2 <= h->events.size()) {
            idx = h->next_event;
            h->next_event += 2;
            cudaEventRecord(h->events[idx], s);
        }
    }
    ~StageScope() {
        if (idx != SIZE_MAX) {
            cudaEventRecord(h->events[idx + 1], s);
            h->recorded.emplace_back(stage, idx);
        }
    }
};

template <typename K, typename... Args>
int launch(ffcm_handle* h, K kernel, dim3 grid, dim3 block, size_t smem, cudaStream_t s,
           Args... args) {
    kernel<<<grid, block, smem, s>>>(args...);
    h->launches += 1;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
    return FFCM_OK;
}

int grid_for(int64_t n, int threads, int cap = 148 * 16) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    return (int)std::min<int64_t>(b, cap);
}

template <typename T>
struct Engine final : EngineBase {
    ffcm_handle* h;
    int N;
    int Mx, My, Mz, MG;
    int m0, m1, m2, ncell;
    int nkx, hxp;
    int64_t plane;
    Derived<T> d;
    T L[3];
    StencilParams<T> sp;
    T h3, inv_mu_M;
    CorrConsts<T> cc;
    FftPlan plan_x, plan_y, plan_z;
    int lpb_x, tx_y, tx_z;
    size_t smem_x, smem_y, smem_z, smem_stencil;
    int ntiles;

    T *Yin = nullptr, *Fin = nullptr, *Vout = nullptr, *Yw = nullptr;
    int32_t *key = nullptr, *perm = nullptr, *cnt = nullptr, *off = nullptr, *tiles = nullptr;
    int32_t* scratch_i = nullptr;
    vec4<T>*Ys = nullptr, *Fs = nullptr;
    T *gf = nullptr, *gu = nullptr;
    cplx<T>* spec = nullptr;
    cplx<T>*twx = nullptr, *twy = nullptr, *twz = nullptr;
    T *kxv = nullptr, *kyv = nullptr, *kzv = nullptr;
    std::vector<void*> allocs;

    ~Engine() override {
        for (void* p : allocs) cudaFree(p);
    }

    template <typename P>
    int alloc(P*& p, size_t count) {
        void* q = nullptr;
        size_t bytes = std::max<size_t>(count * sizeof(P), 16);
        cudaError_t e = cudaMalloc(&q, bytes);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
        allocs.push_back(q);
        p = static_cast<P*>(q);
        return FFCM_OK;
    }

    int init(ffcm_handle* hh, const double* Ld, double R_c, double mu_d) {
        h = hh;
        N = (int)h->N;
        Mx = h->M[0]; My = h->M[1]; Mz = h->M[2];
        MG = h->M_G;
        m0 = d.num_cells[0]; m1 = d.num_cells[1]; m2 = d.num_cells[2];
        ncell = m0 * m1 * m2;
        for (int i = 0; i < 3; ++i) L[i] = T(Ld[i]);
        nkx = Mx / 2 + 1;
        const int align = 128 / (int)sizeof(cplx<T>);  // rows start on 128-byte boundaries
        hxp = ((nkx + align - 1) / align) * align;
        plane = (int64_t)Mx * My * Mz;
        const T mu = T(mu_d);

        // stencil scalars (src/stencil.jl:311-320)
        const T S2 = d.Sigma * d.Sigma;
        const T S4 = S2 * S2;
        const T dd = d.sigma * d.sigma - S2;
        sp.Mx = Mx; sp.My = My; sp.Mz = Mz; sp.MG = MG; sp.half = MG / 2;
        sp.h = d.h; sp.inv_h = d.inv_h;
        sp.a0 = T(1) - T(3) * dd / (T(2) * S2);
        sp.a2 = dd / (T(2) * S4);
        sp.inv_norm = T(1) / std::sqrt(T(2) * T(kPi) * S2);
        sp.inv_2S2 = T(1) / (T(2) * S2);
        h3 = d.h * d.h * d.h;
        const T inv_M = T(1) / T((double)plane);
        inv_mu_M = inv_M / mu;

        // correction constants (src/correct_velocities.jl:21-27, 71-104)
        const T pi = T(kPi);
        const T s2 = d.sigma * d.sigma;
        cc.s2 = s2; cc.s4 = s2 * s2; cc.S2 = S2; cc.S4 = S4;
        cc.d = s2 - S2;
        cc.dq = cc.d * cc.d / T(4);
        cc.fourpimu = T(4) * pi * mu;
        cc.eightpimu = T(8) * pi * mu;
        cc.mu = mu;
        cc.two_sigma = T(2) * d.sigma;
        cc.two_Sigma = T(2) * d.Sigma;
        cc.pref_s = std::pow(T(4) * pi * s2, -T(3) / T(2));
        cc.pref_S = std::pow(T(4) * pi * S2, -T(3) / T(2));
        cc.four_s2 = T(4) * s2;
        cc.four_S2 = T(4) * S2;
        {
            const T a = T(1);
            const T Ssp = d.Sigma * std::sqrt(pi);
            cc.self = T(1) / (T(6) * pi * mu * a) - T(1) / (T(6) * pi * mu * Ssp) +
                      cc.d / (T(12) * mu * (Ssp * Ssp * Ssp)) -
                      (cc.d * cc.d) / (T(32) * mu * std::pow(d.Sigma, T(5)) * std::sqrt(pi * pi * pi));
        }
        cc.L0 = L[0]; cc.L1 = L[1]; cc.L2 = L[2];
        const T R = T(R_c);
        cc.Rc2 = R * R;
        cc.ic0 = d.inv_cell_size[0]; cc.ic1 = d.inv_cell_size[1]; cc.ic2 = d.inv_cell_size[2];
        cc.m0 = m0; cc.m1 = m1; cc.m2 = m2;

        // FFT plans and launch shapes
        const bool xeven = (Mx % 2) == 0;
        TRY(make_plan(xeven ? Mx / 2 : Mx, xeven ? 2 : 1, plan_x));
        TRY(make_plan(My, 1, plan_y));
        TRY(make_plan(Mz, 1, plan_z));
        const size_t cs = sizeof(cplx<T>);
        const size_t budget = 200 * 1024;
        lpb_x = std::max(1, std::min(64, (int)(16384 / (plan_x.n * cs))));
        smem_x = 2 * (size_t)lpb_x * plan_x.n * cs;
        tx_y = pow2_floor(std::max(1, std::min(16, (int)(32768 / (My * cs)))));
        smem_y = 2 * (size_t)tx_y * My * cs;
        tx_z = pow2_floor(std::max(1, std::min(16, (int)(65536 / (3 * Mz * cs)))));
        smem_z = 2 * (size_t)3 * tx_z * Mz * cs;
        if (smem_x > budget || smem_y > budget || smem_z > budget)
            return fail(FFCM_ERR_UNSUPPORTED, "grid dimension too large for the shared-memory FFT");
        smem_stencil = 8 * 3 * (size_t)MG * (2 * sizeof(T) + sizeof(int));
        CUDA_TRY(cudaFuncSetAttribute(k_fft_x_r2c<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_x));
        CUDA_TRY(cudaFuncSetAttribute(k_fft_x_c2r<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_x));
        CUDA_TRY(cudaFuncSetAttribute(k_fft_y<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_y));
        CUDA_TRY(cudaFuncSetAttribute(k_fft_z_stokes<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_z));
        if (smem_stencil > 48 * 1024) {
            CUDA_TRY(cudaFuncSetAttribute(k_spread_atomic<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_stencil));
            CUDA_TRY(cudaFuncSetAttribute(k_interpolate_warp<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_stencil));
        }

        // buffers
        TRY(alloc(Yin, 3 * (size_t)N));
        TRY(alloc(Fin, 3 * (size_t)N));
        TRY(alloc(Vout, 3 * (size_t)N));
        TRY(alloc(Yw, 3 * (size_t)N));
        TRY(alloc(key, N));
        TRY(alloc(perm, N));
        TRY(alloc(cnt, ncell));
        TRY(alloc(off, (size_t)ncell + 1));
        ntiles = (ncell + SCAN_TILE - 1) / SCAN_TILE;
        TRY(alloc(tiles, ntiles));
        TRY(alloc(scratch_i, std::max<size_t>(N, (size_t)ncell + 1)));
        TRY(alloc(Ys, N));
        TRY(alloc(Fs, N));
        TRY(alloc(gf, 3 * (size_t)plane));
        TRY(alloc(gu, 3 * (size_t)plane));
        TRY(alloc(spec, 3 * (size_t)hxp * My * Mz));
        TRY(alloc(twx, Mx));
        TRY(alloc(twy, My));
        TRY(alloc(twz, Mz));
        TRY(alloc(kxv, nkx));
        TRY(alloc(kyv, My));
        TRY(alloc(kzv, Mz));

        // zero-initialised grids and cell list (src/config.jl:464-469)
        CUDA_TRY(cudaMemset(gf, 0, 3 * (size_t)plane * sizeof(T)));
        CUDA_TRY(cudaMemset(gu, 0, 3 * (size_t)plane * sizeof(T)));
        CUDA_TRY(cudaMemset(spec, 0, 3 * (size_t)hxp * My * Mz * sizeof(cplx<T>)));
        CUDA_TRY(cudaMemset(off, 0, ((size_t)ncell + 1) * sizeof(int32_t)));
        CUDA_TRY(cudaMemset(perm, 0, (size_t)N * sizeof(int32_t)));
        CUDA_TRY(cudaMemset(key, 0, (size_t)N * sizeof(int32_t)));
        CUDA_TRY(cudaMemset(Yw, 0, 3 * (size_t)N * sizeof(T)));
        CUDA_TRY(cudaMemset(Ys, 0, (size_t)N * sizeof(vec4<T>)));
        CUDA_TRY(cudaMemset(Fs, 0, (size_t)N * sizeof(vec4<T>)));

        // twiddle tables W_M^t = exp(-2 pi i t / M), computed in double
        auto table = [&](int M, cplx<T>* dst) -> int {
            std::vector<cplx<T>> t(M);
            for (int i = 0; i < M; ++i) {
                const double ang = -2.0 * kPi * (double)i / (double)M;
                t[i] = cplx<T>{T(std::cos(ang)), T(std::sin(ang))};
            }
            CUDA_TRY(cudaMemcpy(dst, t.data(), M * sizeof(cplx<T>), cudaMemcpyHostToDevice));
            return FFCM_OK;
        };
        TRY(table(Mx, twx));
        TRY(table(My, twy));
        TRY(table(Mz, twz));

        // wavevectors (src/config.jl:254-258, 374-377), in T
        const T twopi = T(2) * T(kPi);
        std::vector<T> kx(nkx), ky(My), kz(Mz);
        for (int i = 0; i < nkx; ++i) kx[i] = twopi * T(i) / L[0];
        auto wrapk = [&](int Mi, T Li, std::vector<T>& out) {
            const int half1 = Mi / 2 + 1;
            for (int j = 1; j <= Mi; ++j) {
                const T m = j <= half1 ? T(j - 1) : T(j - 1 - Mi);
                out[j - 1] = twopi * m / Li;
            }
        };
        wrapk(My, L[1], ky);
        wrapk(Mz, L[2], kz);
        CUDA_TRY(cudaMemcpy(kxv, kx.data(), nkx * sizeof(T), cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(kyv, ky.data(), My * sizeof(T), cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(kzv, kz.data(), Mz * sizeof(T), cudaMemcpyHostToDevice));
        h->kx.assign(kx.begin(), kx.end());
        h->ky.assign(ky.begin(), ky.end());
        h->kz.assign(kz.begin(), kz.end());
        return FFCM_OK;
    }

    void* Y_in() override { return Yin; }
    void* F_in() override { return Fin; }
    void* V_out() override { return Vout; }

    int wrap_hash(const void* Y, bool wrap, bool hash, cudaStream_t s) override {
        StageScope sc(h, FFCM_STAGE_CELL_LIST, s);
        return launch(h, k_wrap_hash<T>, grid_for(N, 256), 256, 0, s, N,
                      static_cast<const T*>(Y), Yw, key, L[0], L[1], L[2], d.inv_cell_size[0],
                      d.inv_cell_size[1], d.inv_cell_size[2], m0, m1, m2, h->d_err,
                      wrap ? 1 : 0, hash ? 1 : 0);
    }

    int sort(const void* F, cudaStream_t s) override {
        StageScope sc(h, FFCM_STAGE_CELL_LIST, s);
        CUDA_TRY(cudaMemsetAsync(cnt, 0, (size_t)ncell * sizeof(int32_t), s));
        TRY(launch(h, k_count_cells, grid_for(N, 256), 256, 0, s, N, (const int32_t*)key, cnt));
        TRY(launch(h, k_scan_tiles, ntiles, SCAN_THREADS, 0, s, (const int32_t*)cnt, ncell, tiles));
        TRY(launch(h, k_scan_tile_sums, 1, 1024, 0, s, tiles, ntiles));
        TRY(launch(h, k_scan_apply, ntiles, SCAN_THREADS, 0, s, (const int32_t*)cnt, ncell,
                   (const int32_t*)tiles, off));
        CUDA_TRY(cudaMemsetAsync(cnt, 0, (size_t)ncell * sizeof(int32_t), s));
        TRY(launch(h, k_scatter_cells, grid_for(N, 256), 256, 0, s, N, (const int32_t*)key,
                   (const int32_t*)off, cnt, perm));
        return launch(h, k_cell_order_gather<T>, grid_for(ncell, 256), 256, 0, s, ncell,
                      (const int32_t*)off, perm, (const T*)Yw, static_cast<const T*>(F), Ys, Fs);
    }

    int spread(cudaStream_t s) override {
        StageScope sc(h, FFCM_STAGE_SPREAD, s);
        CUDA_TRY(cudaMemsetAsync(gf, 0, 3 * (size_t)plane * sizeof(T), s));
        return launch(h, k_spread_atomic<T>, grid_for((int64_t)N * 32, 256, 148 * 64), 256,
                      smem_stencil, s, N, (const vec4<T>*)Ys, (const vec4<T>*)Fs, gf, sp);
    }

    int stokes(cudaStream_t s) override {
        const int nrows = 3 * My * Mz;
        {
            StageScope sc(h, FFCM_STAGE_FFT_X_FWD, s);
            TRY(launch(h, k_fft_x_r2c<T>, (nrows + lpb_x - 1) / lpb_x, 256, smem_x, s,
                       (const T*)gf, spec, Mx, nrows, hxp, plan_x, (const cplx<T>*)twx, lpb_x));
        }
        dim3 gy((nkx + tx_y - 1) / tx_y, Mz, 3);
        {
            StageScope sc(h, FFCM_STAGE_FFT_Y_FWD, s);
            TRY(launch(h, k_fft_y<T>, gy, 256, smem_y, s, spec, nkx, My, Mz, hxp, plan_y,
                       (const cplx<T>*)twy, tx_y, 0));
        }
        {
            StageScope sc(h, FFCM_STAGE_FFT_Z_STOKES, s);
            dim3 gz((nkx + tx_z - 1) / tx_z, My, 1);
            TRY(launch(h, k_fft_z_stokes<T>, gz, 256, smem_z, s, spec, nkx, My, Mz, hxp, plan_z,
                       (const cplx<T>*)twz, tx_z, (const T*)kxv, (const T*)kyv, (const T*)kzv,
                       inv_mu_M));
        }
        {
            StageScope sc(h, FFCM_STAGE_FFT_Y_INV, s);
            TRY(launch(h, k_fft_y<T>, gy, 256, smem_y, s, spec, nkx, My, Mz, hxp, plan_y,
                       (const cplx<T>*)twy, tx_y, 1));
        }
        StageScope sc(h, FFCM_STAGE_FFT_X_INV, s);
        return launch(h, k_fft_x_c2r<T>, (nrows + lpb_x - 1) / lpb_x, 256, smem_x, s,
                      (const cplx<T>*)spec, gu, Mx, nrows, hxp, plan_x, (const cplx<T>*)twx, lpb_x);
    }

    int interp(void* V, cudaStream_t s) override {
        StageScope sc(h, FFCM_STAGE_INTERPOLATE, s);
        return launch(h, k_interpolate_warp<T>, grid_for((int64_t)N * 32, 256, 148 * 64), 256,
                      smem_stencil, s, N, (const vec4<T>*)Ys, (const int32_t*)perm,
                      (const T*)gu, static_cast<T*>(V), sp, h3);
    }

    int correct(void* V, cudaStream_t s) override {
        StageScope sc(h, FFCM_STAGE_CORRECT, s);
        return launch(h, k_correct<T>, grid_for(N, 128), 128, 0, s, N, (const vec4<T>*)Ys,
                      (const vec4<T>*)Fs, (const int32_t*)off, (const int32_t*)perm,
                      static_cast<T*>(V), cc);
    }
};

__global__ void k_add_i32(int32_t* dst, const int32_t* src, int n, int delta) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        dst[i] = src[i] + delta;
}

int check_handle(const ffcm_handle* h) {
    if (!h || !h->eng) return fail(FFCM_ERR_STATE, "null or destroyed ffcm handle");
    return FFCM_OK;
}

cudaMemcpyKind kind_to_dev(int32_t memory) {
    return memory == FFCM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
}
cudaMemcpyKind kind_from_dev(int32_t memory) {
    return memory == FFCM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
}

int check_memory(int32_t memory) {
    if (memory != FFCM_HOST && memory != FFCM_DEVICE)
        return fail(FFCM_ERR_ARGUMENT, "memory must be FFCM_HOST or FFCM_DEVICE");
    return FFCM_OK;
}

// Synchronise and surface sticky device-side errors.
int finish(ffcm_handle* h, cudaStream_t s) {
    CUDA_TRY(cudaMemcpyAsync(h->h_err, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    const int e = *h->h_err;
    if (e) {
        CUDA_TRY(cudaMemsetAsync(h->d_err, 0, sizeof(int), s));
        CUDA_TRY(cudaStreamSynchronize(s));
        if (e & DEVERR_NONFINITE_POSITION)
            return fail(FFCM_ERR_ARGUMENT, "non-finite particle position (InexactError in the reference)");
        return fail(FFCM_ERR_CUDA, "device-side error flag " + std::to_string(e));
    }
    return FFCM_OK;
}

template <typename T>
int create_T(ffcm_handle* h, const double* L, double R_c, double a, double ratio, double mu) {
    auto e = std::make_unique<Engine<T>>();
    TRY(derive_T<T>(L, R_c, a, ratio, h->M, e->d));
    for (int i = 0; i < 3; ++i) h->num_cells[i] = e->d.num_cells[i];
    h->ncell = (int64_t)h->num_cells[0] * h->num_cells[1] * h->num_cells[2];
    if (h->ncell > 2147483000LL) return fail(FFCM_ERR_UNSUPPORTED, "cell count exceeds the Int32 range");
    Engine<T>* raw = e.get();
    h->eng = std::move(e);
    return raw->init(h, L, R_c, mu);
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* ffcm_last_error(void) { return g_err.c_str(); }

int ffcm_version(void) { return 100; }

int ffcm_validate_config(int32_t dtype, const double* L, double R_c, int64_t N, double a,
                         double ratio, const int32_t* M, int32_t M_G, double mu,
                         int32_t planning, int32_t threads) {
    g_err.clear();
    if (!L || !M) return fail(FFCM_ERR_ARGUMENT, "L and num_grid_points must not be NULL");
    int r;
    if (dtype == FFCM_FLOAT32) r = validate_T<float>(L, R_c, N, a, ratio, M, M_G, mu, planning, threads);
    else if (dtype == FFCM_FLOAT64) r = validate_T<double>(L, R_c, N, a, ratio, M, M_G, mu, planning, threads);
    else return fail(FFCM_ERR_ARGUMENT, "dtype must be FFCM_FLOAT32 or FFCM_FLOAT64");
    if (r != FFCM_OK) return r;
    if (N > 2147483647LL) return fail(FFCM_ERR_UNSUPPORTED, "N exceeds the Int32 particle-index range");
    if (dtype == FFCM_FLOAT32) {
        Derived<float> d;
        return derive_T<float>(L, R_c, a, ratio, M, d);
    }
    Derived<double> d;
    return derive_T<double>(L, R_c, a, ratio, M, d);
}

int ffcm_derive_scalars(int32_t dtype, const double* L, double R_c, double a, double ratio,
                        const int32_t* M, int32_t* num_cells, double* cell_size,
                        double* inv_cell_size, double* sigma, double* Sigma, double* h,
                        double* inv_h) {
    g_err.clear();
    if (!L || !M) return fail(FFCM_ERR_ARGUMENT, "L and num_grid_points must not be NULL");
    auto out = [&](auto& d) {
        for (int i = 0; i < 3; ++i) {
            if (num_cells) num_cells[i] = d.num_cells[i];
            if (cell_size) cell_size[i] = (double)d.cell_size[i];
            if (inv_cell_size) inv_cell_size[i] = (double)d.inv_cell_size[i];
        }
        if (sigma) *sigma = (double)d.sigma;
        if (Sigma) *Sigma = (double)d.Sigma;
        if (h) *h = (double)d.h;
        if (inv_h) *inv_h = (double)d.inv_h;
    };
    if (dtype == FFCM_FLOAT32) {
        Derived<float> d;
        TRY(derive_T<float>(L, R_c, a, ratio, M, d));
        out(d);
    } else if (dtype == FFCM_FLOAT64) {
        Derived<double> d;
        TRY(derive_T<double>(L, R_c, a, ratio, M, d));
        out(d);
    } else {
        return fail(FFCM_ERR_ARGUMENT, "dtype must be FFCM_FLOAT32 or FFCM_FLOAT64");
    }
    return FFCM_OK;
}

int ffcm_create(ffcm_handle** out, int32_t dtype, const double* L, double R_c, int64_t N,
                double a, double ratio, const int32_t* M, int32_t M_G, double mu,
                int32_t planning, int32_t threads, int32_t device) {
    if (!out) return fail(FFCM_ERR_ARGUMENT, "out must not be NULL");
    *out = nullptr;
    TRY(ffcm_validate_config(dtype, L, R_c, N, a, ratio, M, M_G, mu, planning, threads));
    int ndev = 0;
    CUDA_TRY(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev)
        return fail(FFCM_ERR_ARGUMENT, "device " + std::to_string(device) + " out of range");
    DeviceGuard g(device);
    if (!g.ok) return fail(FFCM_ERR_CUDA, "cudaSetDevice failed");
    auto h = std::make_unique<ffcm_handle>();
    h->dtype = dtype;
    h->device = device;
    h->N = N;
    for (int i = 0; i < 3; ++i) h->M[i] = M[i];
    h->M_G = M_G;
    h->esize = dtype == FFCM_FLOAT32 ? 4 : 8;
    CUDA_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaMalloc(&h->d_err, sizeof(int)));
    CUDA_TRY(cudaMemset(h->d_err, 0, sizeof(int)));
    CUDA_TRY(cudaHostAlloc(&h->h_err, sizeof(int), cudaHostAllocDefault));
    int r = dtype == FFCM_FLOAT32 ? create_T<float>(h.get(), L, R_c, a, ratio, mu)
                                  : create_T<double>(h.get(), L, R_c, a, ratio, mu);
    if (r != FFCM_OK) {
        std::string msg = g_err;
        ffcm_destroy(h.release());
        return fail(r, msg);
    }
    CUDA_TRY(cudaDeviceSynchronize());
    *out = h.release();
    return FFCM_OK;
}

int ffcm_destroy(ffcm_handle* h) {
    if (!h) return FFCM_OK;
    DeviceGuard g(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    h->eng.reset();
    for (cudaEvent_t e : h->events) cudaEventDestroy(e);
    if (h->d_err) cudaFree(h->d_err);
    if (h->h_err) cudaFreeHost(h->h_err);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return FFCM_OK;
}

int ffcm_get_info(const ffcm_handle* h, int64_t* N, int32_t* dtype, int64_t* ncell) {
    TRY(check_handle(h));
    if (N) *N = h->N;
    if (dtype) *dtype = h->dtype;
    if (ncell) *ncell = h->ncell;
    return FFCM_OK;
}

int ffcm_mobility(ffcm_handle* h, void* V, int64_t vr, int64_t vc, const void* Y, int64_t yr,
                  int64_t yc, const void* F, int64_t fr, int64_t fc, int32_t memory,
                  void* stream) {
    g_err.clear();
    TRY(check_handle(h));
    TRY(check_memory(memory));
    const int64_t N = h->N;
    if (!(vr == 3 && vc == N && yr == 3 && yc == N && fr == 3 && fc == N)) {
        return fail(FFCM_ERR_DIMENSION,
                    "V, Y, and F must each be 3xN for the config's N = " + std::to_string(N) +
                        "; got size(V) = (" + std::to_string(vr) + ", " + std::to_string(vc) +
                        "), size(Y) = (" + std::to_string(yr) + ", " + std::to_string(yc) +
                        "), size(F) = (" + std::to_string(fr) + ", " + std::to_string(fc) + ")");
    }
    if (!V || !Y || !F) return fail(FFCM_ERR_ARGUMENT, "V, Y and F must not be NULL");
    DeviceGuard g(h->device);
    cudaStream_t s = h->pick(stream);
    EngineBase* e = h->eng.get();
    const size_t bytes = 3 * (size_t)N * h->esize;
    const void* Yd = Y;
    const void* Fd = F;
    void* Vd = V;
    if (memory == FFCM_HOST) {
        StageScope sc(h, FFCM_STAGE_H2D, s);
        CUDA_TRY(cudaMemcpyAsync(e->Y_in(), Y, bytes, cudaMemcpyHostToDevice, s));
        CUDA_TRY(cudaMemcpyAsync(e->F_in(), F, bytes, cudaMemcpyHostToDevice, s));
        Yd = e->Y_in();
        Fd = e->F_in();
        Vd = e->V_out();
    }
    TRY(e->wrap_hash(Yd, true, true, s));
    TRY(e->sort(Fd, s));
    TRY(e->spread(s));
    TRY(e->stokes(s));
    TRY(e->interp(Vd, s));
    TRY(e->correct(Vd, s));
    if (memory == FFCM_HOST) {
        {
            StageScope sc(h, FFCM_STAGE_D2H, s);
            CUDA_TRY(cudaMemcpyAsync(V, e->V_out(), bytes, cudaMemcpyDeviceToHost, s));
        }
        return finish(h, s);
    }
    return FFCM_OK;
}

int ffcm_wrap_positions(ffcm_handle* h, const void* Y, int32_t memory, void* stream) {
    g_err.clear();
    TRY(check_handle(h));
    TRY(check_memory(memory));
    if (!Y) return fail(FFCM_ERR_ARGUMENT, "Y must not be NULL");
    DeviceGuard g(h->device);
    cudaStream_t s = h->pick(stream);
    const void* Yd = Y;
    if (memory == FFCM_HOST) {
        CUDA_TRY(cudaMemcpyAsync(h->eng->Y_in(), Y, 3 * (size_t)h->N * h->esize,
                                 cudaMemcpyHostToDevice, s));
        Yd = h->eng->Y_in();
    }
    TRY(h->eng->wrap_hash(Yd, true, false, s));
    return memory == FFCM_HOST ? finish(h, s) : FFCM_OK;
}

int ffcm_assign_cells(ffcm_handle* h, void* stream) {
    g_err.clear();
    TRY(check_handle(h));
    DeviceGuard g(h->device);
    return h->eng->wrap_hash(nullptr, false, true, h->pick(stream));
}

int ffcm_sort_particles_by_cell(ffcm_handle* h, const void* F, int32_t memory, void* stream) {
    g_err.clear();
    TRY(check_handle(h));
    TRY(check_memory(memory));
    if (!F) return fail(FFCM_ERR_ARGUMENT, "F must not be NULL");
    DeviceGuard g(h->device);
    cudaStream_t s = h->pick(stream);
    const void* Fd = F;
    if (memory == FFCM_HOST) {
        CUDA_TRY(cudaMemcpyAsync(h->eng->F_in(), F, 3 * (size_t)h->N * h->esize,
                                 cudaMemcpyHostToDevice, s));
        Fd = h->eng->F_in();
    }
    TRY(h->eng->sort(Fd, s));
    return memory == FFCM_HOST ? finish(h, s) : FFCM_OK;
}

int ffcm_spread_forces(ffcm_handle* h, void* stream) {
    g_err.clear();
    TRY(check_handle(h));
    DeviceGuard g(h->device);
    return h->eng->spread(h->pick(stream));
}

int ffcm_stokes_solve(ffcm_handle* h, void* stream) {
    g_err.clear();
    TRY(check_handle(h));
    DeviceGuard g(h->device);
    return h->eng->stokes(h->pick(stream));
}

int ffcm_interpolate_velocities(ffcm_handle* h, void* V, int32_t memory, void* stream) {
    g_err.clear();
    TRY(check_handle(h));
    TRY(check_memory(memory));
    if (!V) return fail(FFCM_ERR_ARGUMENT, "V must not be NULL");
    DeviceGuard g(h->device);
    cudaStream_t s = h->pick(stream);
    if (memory == FFCM_DEVICE) return h->eng->interp(V, s);
    TRY(h->eng->interp(h->eng->V_out(), s));
    CUDA_TRY(cudaMemcpyAsync(V, h->eng->V_out(), 3 * (size_t)h->N * h->esize,
                             cudaMemcpyDeviceToHost, s));
    return finish(h, s);
}

int ffcm_correct_velocities(ffcm_handle* h, void* V, int32_t memory, void* stream) {
    g_err.clear();
    TRY(check_handle(h));
    TRY(check_memory(memory));
    if (!V) return fail(FFCM_ERR_ARGUMENT, "V must not be NULL");
    DeviceGuard g(h->device);
    cudaStream_t s = h->pick(stream);
    if (memory == FFCM_DEVICE) return h->eng->correct(V, s);
    const size_t bytes = 3 * (size_t)h->N * h->esize;
    CUDA_TRY(cudaMemcpyAsync(h->eng->V_out(), V, bytes, cudaMemcpyHostToDevice, s));
    TRY(h->eng->correct(h->eng->V_out(), s));
    CUDA_TRY(cudaMemcpyAsync(V, h->eng->V_out(), bytes, cudaMemcpyDeviceToHost, s));
    return finish(h, s);
}

int64_t ffcm_buffer_bytes(const ffcm_handle* h, int32_t which) {
    if (!h || !h->eng) return -1;
    const int64_t N = h->N, e = (int64_t)h->esize;
    const int64_t plane = (int64_t)h->M[0] * h->M[1] * h->M[2];
    switch (which) {
        case FFCM_BUF_Y_WRAPPED:
        case FFCM_BUF_Y_SORTED:
        case FFCM_BUF_F_SORTED: return 3 * N * e;
        case FFCM_BUF_CELL_HASH:
        case FFCM_BUF_ORIGINAL_INDEX: return 4 * N;
        case FFCM_BUF_CELL_START:
        case FFCM_BUF_CELL_END: return 4 * h->ncell;
        case FFCM_BUF_FORCE_DENSITY:
        case FFCM_BUF_FLUID_VELOCITY: return 3 * plane * e;
        case FFCM_BUF_K_X: return (int64_t)(h->M[0] / 2 + 1) * e;
        case FFCM_BUF_K_Y: return (int64_t)h->M[1] * e;
        case FFCM_BUF_K_Z: return (int64_t)h->M[2] * e;
        case FFCM_BUF_NEIGHBOR_MAP: return 13 * 4 * h->ncell;
        default: return -1;
    }
}

}  // extern "C"

namespace {

template <typename T>
int buffer_io(ffcm_handle* h, Engine<T>* e, int32_t which, void* ext, int64_t nbytes, int32_t memory,
              cudaStream_t s, bool get) {
    const int64_t want = ffcm_buffer_bytes(h, which);
    if (want < 0) return fail(FFCM_ERR_ARGUMENT, "unknown buffer id " + std::to_string(which));
    if (nbytes != want)
        return fail(FFCM_ERR_DIMENSION, "buffer " + std::to_string(which) + " holds " +
                                            std::to_string(want) + " bytes, got " + std::to_string(nbytes));
    const int N = e->N;
    const cudaMemcpyKind in = kind_to_dev(memory), out = kind_from_dev(memory);
    auto copy = [&](void* dev) -> int {
        if (get) CUDA_TRY(cudaMemcpyAsync(ext, dev, nbytes, out, s));
        else CUDA_TRY(cudaMemcpyAsync(dev, ext, nbytes, in, s));
        return FFCM_OK;
    };
    switch (which) {
        case FFCM_BUF_Y_WRAPPED: TRY(copy(e->Yw)); break;
        case FFCM_BUF_CELL_HASH: TRY(copy(e->key)); break;
        case FFCM_BUF_FORCE_DENSITY: TRY(copy(e->gf)); break;
        case FFCM_BUF_FLUID_VELOCITY: TRY(copy(e->gu)); break;
        case FFCM_BUF_Y_SORTED:
        case FFCM_BUF_F_SORTED: {
            vec4<T>* dev = which == FFCM_BUF_Y_SORTED ? e->Ys : e->Fs;
            if (get)
                CUDA_TRY(cudaMemcpy2DAsync(ext, 3 * sizeof(T), dev, sizeof(vec4<T>), 3 * sizeof(T), N, out, s));
            else
                CUDA_TRY(cudaMemcpy2DAsync(dev, sizeof(vec4<T>), ext, 3 * sizeof(T), 3 * sizeof(T), N, in, s));
            break;
        }
        case FFCM_BUF_ORIGINAL_INDEX:
            if (get) {
                TRY(launch(h, k_add_i32, grid_for(N, 256), 256, 0, s, e->scratch_i, (const int32_t*)e->perm, N, 1));
                TRY(copy(e->scratch_i));
            } else {
                TRY(copy(e->scratch_i));
                TRY(launch(h, k_add_i32, grid_for(N, 256), 256, 0, s, e->perm, (const int32_t*)e->scratch_i, N, -1));
            }
            break;
        case FFCM_BUF_CELL_START:
            if (get) {
                TRY(launch(h, k_add_i32, grid_for(e->ncell, 256), 256, 0, s, e->scratch_i, (const int32_t*)e->off, e->ncell, 1));
                TRY(copy(e->scratch_i));
            } else {
                TRY(copy(e->scratch_i));
                TRY(launch(h, k_add_i32, grid_for(e->ncell, 256), 256, 0, s, e->off, (const int32_t*)e->scratch_i, e->ncell, -1));
            }
            break;
        case FFCM_BUF_CELL_END: TRY(copy(e->off + 1)); break;
        case FFCM_BUF_K_X:
        case FFCM_BUF_K_Y:
        case FFCM_BUF_K_Z: {
            T* dev = which == FFCM_BUF_K_X ? e->kxv : (which == FFCM_BUF_K_Y ? e->kyv : e->kzv);
            TRY(copy(dev));
            break;
        }
        case FFCM_BUF_NEIGHBOR_MAP: {
            if (!get) return fail(FFCM_ERR_ARGUMENT, "the neighbour map is read-only");
            // src/cell_list.jl:258-289: 13 forward half-shell neighbours per cell.
            static const int offs[13][3] = {{1, 0, 0},  {1, 1, 0},  {0, 1, 0},  {-1, 1, 0}, {1, 0, -1},
                                            {1, 1, -1}, {0, 1, -1}, {-1, 1, -1}, {1, 0, 1}, {1, 1, 1},
                                            {0, 1, 1},  {-1, 1, 1}, {0, 0, 1}};
            const int mx = e->m0, my = e->m1, mz = e->m2;
            std::vector<int32_t> nm(13 * (size_t)e->ncell);
            for (int cz = 0; cz < mz; ++cz)
                for (int cy = 0; cy < my; ++cy)
                    for (int cx = 0; cx < mx; ++cx) {
                        const size_t base = 13 * (size_t)(cx + (cy + cz * my) * mx);
                        for (int k = 0; k < 13; ++k) {
                            const int nx = ((cx + offs[k][0]) % mx + mx) % mx;
                            const int ny = ((cy + offs[k][1]) % my + my) % my;
                            const int nz = ((cz + offs[k][2]) % mz + mz) % mz;
                            nm[base + k] = nx + (ny + nz * my) * mx;
                        }
                    }
            CUDA_TRY(cudaStreamSynchronize(s));
            if (memory == FFCM_HOST) std::memcpy(ext, nm.data(), nbytes);
            else CUDA_TRY(cudaMemcpy(ext, nm.data(), nbytes, cudaMemcpyHostToDevice));
            return FFCM_OK;
        }
        default: return fail(FFCM_ERR_ARGUMENT, "unknown buffer id");
    }
    if (memory == FFCM_HOST) CUDA_TRY(cudaStreamSynchronize(s));
    return FFCM_OK;
}

int buffer_dispatch(ffcm_handle* h, int32_t which, void* ext, int64_t nbytes, int32_t memory,
                    void* stream, bool get) {
    g_err.clear();
    TRY(check_handle(h));
    TRY(check_memory(memory));
    if (!ext) return fail(FFCM_ERR_ARGUMENT, "buffer pointer must not be NULL");
    DeviceGuard g(h->device);
    cudaStream_t s = h->pick(stream);
    if (h->dtype == FFCM_FLOAT32)
        return buffer_io<float>(h, static_cast<Engine<float>*>(h->eng.get()), which, ext, nbytes, memory, s, get);
    return buffer_io<double>(h, static_cast<Engine<double>*>(h->eng.get()), which, ext, nbytes, memory, s, get);
}

}  // namespace

extern "C" {

int ffcm_get_buffer(ffcm_handle* h, int32_t which, void* dst, int64_t nbytes, int32_t memory,
                    void* stream) {
    return buffer_dispatch(h, which, dst, nbytes, memory, stream, true);
}

int ffcm_set_buffer(ffcm_handle* h, int32_t which, const void* src, int64_t nbytes,
                    int32_t memory, void* stream) {
    return buffer_dispatch(h, which, const_cast<void*>(src), nbytes, memory, stream, false);
}

int ffcm_synchronize(ffcm_handle* h, void* stream) {
    g_err.clear();
    TRY(check_handle(h));
    DeviceGuard g(h->device);
    return finish(h, h->pick(stream));
}

int ffcm_profile_begin(ffcm_handle* h) {
    g_err.clear();
    TRY(check_handle(h));
    DeviceGuard g(h->device);
    if (h->events.empty()) {
        h->events.resize(8192);
        for (auto& ev : h->events) CUDA_TRY(cudaEventCreate(&ev));
    }
    h->next_event = 0;
    h->recorded.clear();
    h->profiling = true;
    return FFCM_OK;
}

int ffcm_profile_end(ffcm_handle* h, double* stage_ms, int64_t* stage_calls) {
    g_err.clear();
    TRY(check_handle(h));
    DeviceGuard g(h->device);
    h->profiling = false;
    for (int i = 0; i < FFCM_STAGE_COUNT; ++i) {
        if (stage_ms) stage_ms[i] = 0;
        if (stage_calls) stage_calls[i] = 0;
    }
    for (auto& r : h->recorded) {
        CUDA_TRY(cudaEventSynchronize(h->events[r.second + 1]));
        float ms = 0;
        CUDA_TRY(cudaEventElapsedTime(&ms, h->events[r.second], h->events[r.second + 1]));
        if (stage_ms) stage_ms[r.first] += ms;
        if (stage_calls) stage_calls[r.first] += 1;
    }
    h->recorded.clear();
    h->next_event = 0;
    return FFCM_OK;
}

int64_t ffcm_launch_count(const ffcm_handle* h) { return h ? h->launches : -1; }

}  // extern "C"
