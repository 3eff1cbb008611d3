// C ABI of libffcm_b200: configuration (cold path), the six hot-path steps,
// the assembled operator, buffer access and measurement. See
// include/ffcm_b200.h for the contract of every entry point.
#include <algorithm>
#include <array>
#include <limits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <functional>
#include <initializer_list>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "ffcm_b200.h"
#include "common.cuh"
#include "cell_list.cuh"
#include "correct.cuh"
#include "adjoint.cuh"
#include "cg.cuh"
#include "fft.cuh"
#include "fft_dispatch.cuh"
#include "fft_pipe.cuh"
#include "fft_tma.cuh"
#include "slab.cuh"
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

// Raise a kernel's dynamic shared-memory cap to at least `bytes` on the
// current device. The cap is a property of the function in the process, not
// of a handle, so it only ever grows: several configurations of different
// sizes alive at once each keep what they need.
int raise_smem_cap(const void* func, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> cap;
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    size_t& cur = cap[{dev, func}];
    if (bytes <= cur) return FFCM_OK;
    CUDA_TRY(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    cur = bytes;
    return FFCM_OK;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library does not link the driver library itself).
using TensorMapEncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                       const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                                       CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                       CUtensorMapFloatOOBfill);

TensorMapEncodeFn tensor_map_encoder() {
    static TensorMapEncodeFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<TensorMapEncodeFn>(f);
    }();
    return fn;
}

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
// Cold path, in the working precision T (src/config.jl:267-359)
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
// Autotuner choices per (device ordinal, element size, Mx, My, Mz, SM count),
// shared by all configurations of the process (the y/z passes do not depend
// on the particles), and exported / imported as text like FFTW wisdom. The SM
// count keeps a choice made on one GPU model from being applied to another
// that happens to have the same ordinal.
struct TunedChoice {
    int ykind, By, ygrid, zkind, Bz, zgrid, kx_chunk;
};
using TuneKey = std::array<int, 6>;
std::mutex& tune_mu() {
    static std::mutex m;
    return m;
}
std::map<TuneKey, TunedChoice>& tune_store() {
    static std::map<TuneKey, TunedChoice> c;
    return c;
}

struct EngineBase {
    virtual ~EngineBase() = default;
    virtual int wrap_hash(const void* Y, bool wrap, bool hash, cudaStream_t s) = 0;
    virtual int sort(const void* F, cudaStream_t s) = 0;
    virtual int spread(cudaStream_t s) = 0;
    virtual int stokes(cudaStream_t s) = 0;
    virtual int interp(void* V, cudaStream_t s) = 0;
    virtual int correct(void* V, cudaStream_t s) = 0;
    virtual int mobility_rest(void* V, cudaStream_t s) = 0;
    // a further right-hand side on the positions of the last solve (the
    // cell list and the slab particle lists are reused)
    virtual int mobility_rest_same_positions(void* V, cudaStream_t s) = 0;
    // fixed-position operator: the forces are re-gathered into the cached
    // cell order and solved (the first solve after a new cell list also
    // builds the slab lists)
    virtual int apply_fixed(void* V, const void* F, cudaStream_t s) = 0;
    bool lists_built = false;
    virtual int gather_forces(const void* F, cudaStream_t s) = 0;
    virtual int forward_checkpoint(void* V, cudaStream_t s) = 0;
    virtual int adjoint(const void* lam, void* dY, void* dF, cudaStream_t s) = 0;
    virtual int residual(const void* V, const void* Vt, void* lam, double* J, cudaStream_t s) = 0;
    virtual int ensure_adjoint() = 0;
    virtual void* adj_buf(int which) = 0;  // 0 lambda, 1 dY, 2 dF, 3 target, 4 J (double)
    virtual int ensure_real_grids() = 0;
    virtual bool uses_slab() const = 0;
    // stencil arithmetic of every later launch (FFCM_STENCIL_*)
    virtual void set_stencil(int mode) = 0;
    // the y/z variant in use: ykind, By, ygrid, zkind, Bz, zgrid, kx_chunk
    // (-1 for an axis without the power-of-two passes)
    virtual void tuning(int32_t* out) const = 0;
    virtual void* Y_in() = 0;
    virtual void* F_in() = 0;
    virtual void* V_out() = 0;
    // conjugate gradients on apply_fixed (the resistance problem): the slab
    // particle lists (or the real grids of the generic pipeline) made ready
    // outside any graph capture; r = V - q, p = 0 and the scalar state; one
    // iteration (p update, q = M p, alpha, x/r update and the loop condition)
    virtual int ensure_lists(cudaStream_t s) = 0;
    virtual int cg_start(const void* V, const void* q, void* r, void* p, CgState* st, double reltol,
                         double abstol, int maxiter, cudaStream_t s) = 0;
    virtual int cg_iteration(void* x, void* r, void* p, void* q, CgState* st, cudaGraphConditionalHandle loop,
                             cudaStream_t s) = 0;
    // a rank of a z-slab decomposition (see ffcm_dist_*)
    virtual int dist_forward(const void* Y, const void* F, cudaStream_t s) = 0;
    virtual int dist_stokes(cudaStream_t s) = 0;
    virtual int dist_interp(cudaStream_t s) = 0;
    virtual int dist_correct(void* V, cudaStream_t s) = 0;
    virtual void dist_info(void** send, void** recv, int64_t* block_bytes, void** partial, int32_t* ranges) const = 0;
};

}  // namespace

struct ffcm_handle {
    int32_t dtype = FFCM_FLOAT32;
    int32_t device = 0;
    int64_t N = 0;
    int32_t M[3] = {0, 0, 0};
    int32_t M_G = 0;
    int32_t stencil = FFCM_STENCIL_REFERENCE;   // stencil arithmetic (FFCM_STENCIL_*)
    // a rank of a z-slab decomposition of one system (ffcm_dist_create)
    bool distributed = false;
    int32_t nranks = 1, rank = 0;
    int32_t num_cells[3] = {0, 0, 0};
    int64_t ncell = 0;
    size_t esize = 4;
    cudaStream_t stream = nullptr;
    // host-array solves: the forces' copy runs on copy_stream while the
    // positions are sorted (created on first use)
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_ready = nullptr, ev_forces = nullptr;
    // fused solves outside stream capture: the pair correction may run on
    // side_stream beside the grid stages (fork after the spread, join before
    // the last kernel; created on first use). overlap_pairs: 1 always, 0
    // never (FFCM_OVERLAP_PAIRS=1 / 0), -1 decided by the first solve's
    // timings (pair_probe: 0 not started, 1 probe events recorded, 2
    // decided; pair_overlap the decision).
    int overlap_pairs = -1;
    int pair_probe = 0;
    bool pair_overlap = false;
    cudaStream_t side_stream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaEvent_t ev_probe[4] = {nullptr, nullptr, nullptr, nullptr};   // y forward, correction
    int* d_err = nullptr;
    int* h_err = nullptr;
    int64_t launches = 0;
    // true while the state of the last ffcm_mobility_checkpoint (cell list,
    // sorted Y/F, velocity grid) is intact for ffcm_adjoint
    bool ckpt = false;
    // true while the cell list of the last ffcm_set_positions is intact for
    // ffcm_mobility_apply
    bool positions = false;
    // profiling
    bool profiling = false;
    std::vector<cudaEvent_t> events;
    size_t next_event = 0;
    std::vector<std::pair<int, size_t>> recorded;  // (stage, index of the start event)
    std::unique_ptr<EngineBase> eng;
    // conjugate-gradient solver state (allocated by the first ffcm_cg_solve):
    // solution, residual, direction and product vectors (3N each), the
    // device scalar state and its pinned host copy, and the graph of the
    // iteration loop on its own capture stream
    struct Cg {
        void* x = nullptr;
        void* r = nullptr;
        void* p = nullptr;
        void* q = nullptr;
        CgState* st = nullptr;
        CgState* host = nullptr;
        cudaStream_t cs = nullptr;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        cudaGraphConditionalHandle loop = 0;
        int64_t body_kernels = 0;  // kernels per iteration
    } cg;
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

// ---------------------------------------------------------------------------
// z-slab decomposition of one system over R ranks: rank r holds the z planes
// [zb, ze) (whole slabs of BZ planes) for the spread, the y passes and the
// interpolation, and the kx columns [kb, ke) of every plane for the z pass.
// Contiguous ranges, as even as possible.
void dist_ranges(int Mz, int BZ, int nkx, int R, int r, int& zb, int& ze, int& kb, int& ke) {
    const int nzs = Mz / BZ;
    zb = (int)((int64_t)nzs * r / R) * BZ;
    ze = (int)((int64_t)nzs * (r + 1) / R) * BZ;
    kb = (int)((int64_t)nkx * r / R);
    ke = (int)((int64_t)nkx * (r + 1) / R);
}

// dst[c dc + z dz + y dy + k] = src[c sc + z sz + y sy + k] for c < 3, z < nz,
// y < ny, k < nk: one block of a spectrum transpose (a row of k per thread
// group, coalesced on both sides).
template <typename T>
__global__ void k_copy_block(cplx<T>* __restrict__ dst, int64_t dc, int64_t dz, int64_t dy,
                             const cplx<T>* __restrict__ src, int64_t sc, int64_t sz, int64_t sy, int nz, int ny,
                             int nk) {
    const int rows = 3 * nz * ny;
    for (int row = blockIdx.x; row < rows; row += gridDim.x) {
        const int y = row % ny, t = row / ny;
        const int z = t % nz, c = t / nz;
        cplx<T>* d = dst + c * dc + z * dz + y * dy;
        const cplx<T>* s = src + c * sc + z * sz + y * sy;
        for (int k = threadIdx.x; k < nk; k += blockDim.x) d[k] = s[k];
    }
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
    // register (power-of-two) FFT path, per axis
    bool fast_x = false, fast_y = false, fast_z = false;
    int lpb_fx = 0, By = 0, Bz = 0;
    // y/z pass variant: 0 = one tile per block (k_fftp_*), 1 = persistent
    // pipelined (k_fftq_*); grid size of the persistent variant
    int ykind = 0, zkind = 0, ygrid = 0, zgrid = 0;
    // kx columns per chunk of the y/z/y passes (0: one pass over the spectrum)
    int kx_chunk = 0;
    // tensor maps of the spectrum for the TMA z pass, one per bundle width B
    // (index log2 B); valid[i] false where the map could not be made
    CUtensorMap zmap[5];
    bool zmap_ok[5] = {false, false, false, false, false};
    CUtensorMap ymap[5];   // same, boxes for the TMA y pass
    bool ymap_ok[5] = {false, false, false, false, false};
    int num_sms = 148;
    size_t smem_fx = 0, smem_fy = 0, smem_fz = 0;
    // spectrum held: planes (c, z) for z in the mzl planes of `spec` (all Mz
    // on one GPU, the rank's own z planes in a z-slab decomposition); the z
    // pass works on zbuf: nkz columns (global columns kzoff ...) of pitch
    // zpitch over all Mz planes (on one GPU zbuf = spec)
    int mzl = 0;
    cplx<T>* zbuf = nullptr;
    int zpitch = 0, nkz = 0, kzoff = 0;
    // z-slab decomposition (nranks > 1 or an explicitly distributed handle)
    struct Dist {
        bool on = false;
        int R = 1, r = 0;
        std::vector<int> zb, ze, kb, ke;   // per rank: z planes [zb, ze), kx columns [kb, ke)
        int mzl_max = 0, nk_max = 0;
        int64_t blk = 0;                   // complex values per peer block of a transpose
        cplx<T>* send = nullptr;
        cplx<T>* recv = nullptr;
    } dist;
    // slab kernels: spread/interpolation fused with the x transforms
    bool slab = false;
    SlabKernels<T> sk;
    SlabGeom sg;
    T* partial = nullptr;
    T* dvs = nullptr;            // pair terms in sorted order (side-stream correction)
    int* slab_lists = nullptr;   // per-slab particle lists kept by the spread
    int* slab_counts = nullptr;
    int ntiles;

    T *Yin = nullptr, *Fin = nullptr, *Vout = nullptr, *Yw = nullptr;
    int32_t *key = nullptr, *perm = nullptr, *cnt = nullptr, *off = nullptr, *tiles = nullptr;
    int32_t* scratch_i = nullptr;
    vec4<T>*Ys = nullptr, *Fs = nullptr;
    T *gf = nullptr, *gu = nullptr;
    // adjoint state (allocated on first use): sorted cotangent, the adjoint
    // velocity grid psi, host-staging buffers and the objective accumulator
    vec4<T>* Ls = nullptr;
    T *gpsi = nullptr, *Lin = nullptr, *dYo = nullptr, *dFo = nullptr, *Vt = nullptr;
    double* Jd = nullptr;
    CorrGradConsts<T> cgc;
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

        // stencil scalars (src/stencil.jl:22-31)
        const T S2 = d.Sigma * d.Sigma;
        const T S4 = S2 * S2;
        const T dd = d.sigma * d.sigma - S2;
        sp.Mx = Mx; sp.My = My; sp.Mz = Mz; sp.MG = MG; sp.half = MG / 2;
        sp.h = d.h; sp.inv_h = d.inv_h;
        sp.a0 = T(1) - T(3) * dd / (T(2) * S2);
        sp.a2 = dd / (T(2) * S4);
        sp.inv_norm = T(1) / std::sqrt(T(2) * T(kPi) * S2);
        sp.inv_2S2 = T(1) / (T(2) * S2);
        // the box spacing as the caller gave it (double), for Float64-geometry
        // stencils: as the Float64 reference computes h = L / M, inv_h = 1 / h
        {
            const double hd = Ld[0] / (double)Mx;
            sp.inv_hd = 1.0 / hd;
            sp.h_hi = T(hd);
            sp.h_lo = T(hd - (double)sp.h_hi);
        }
        sp.comp = h->stencil == FFCM_STENCIL_FLOAT64 ? 1 : 0;
        h3 = d.h * d.h * d.h;
        const T inv_M = T(1) / T((double)plane);
        inv_mu_M = inv_M / mu;

        // correction constants (src/correct_velocities.jl:21-27, 71-104)
        const T pi = T(kPi);
        const T s2 = d.sigma * d.sigma;
        const T s4 = s2 * s2;
        const T dd2 = s2 - S2;
        const T dq = dd2 * dd2 / T(4);
        cc.inv_two_sigma = T(1) / (T(2) * d.sigma);
        cc.inv_two_Sigma = T(1) / (T(2) * d.Sigma);
        cc.pref_s = std::pow(T(4) * pi * s2, -T(3) / T(2));
        cc.pref_S = std::pow(T(4) * pi * S2, -T(3) / T(2));
        cc.inv_four_s2 = T(1) / (T(4) * s2);
        cc.inv_four_S2 = T(1) / (T(4) * S2);
        cc.k1 = T(1) / (T(8) * pi * mu);
        cc.k2 = s2 / (T(4) * pi * mu);
        cc.k3 = T(2) * s4 / mu;
        cc.k4 = T(2) * S4 / mu;
        cc.k5 = dd2 / mu;
        cc.k6 = T(2) * S2;
        cc.k7 = dq / (T(2) * mu * S2);
        cc.k8 = T(1) / (T(2) * S2);
        cc.k9 = T(3) * s2 / (T(4) * pi * mu);
        cc.k10 = T(6) * s4 / mu;
        cc.k11 = T(6) * S4 / mu;
        cc.k12 = T(6) * S2;
        cc.k13 = dq / (T(4) * mu * S4);
        {
            const T a = T(1);
            const T Ssp = d.Sigma * std::sqrt(pi);
            cc.self = T(1) / (T(6) * pi * mu * a) - T(1) / (T(6) * pi * mu * Ssp) +
                      dd2 / (T(12) * mu * (Ssp * Ssp * Ssp)) -
                      (dd2 * dd2) / (T(32) * mu * std::pow(d.Sigma, T(5)) * std::sqrt(pi * pi * pi));
        }
        cc.L0 = L[0]; cc.L1 = L[1]; cc.L2 = L[2];
        const T R = T(R_c);
        cc.Rc2 = R * R;
        cc.ic0 = d.inv_cell_size[0]; cc.ic1 = d.inv_cell_size[1]; cc.ic2 = d.inv_cell_size[2];
        cc.m0 = m0; cc.m1 = m1; cc.m2 = m2;
        cgc.e_s = T(1) / (d.sigma * std::sqrt(pi));
        cgc.e_S = T(1) / (d.Sigma * std::sqrt(pi));
        cgc.ds_s = T(1) / (T(2) * s2);
        cgc.ds_S = T(1) / (T(2) * S2);

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
        fast_x = xeven && fast_len(Mx / 2);
        fast_y = fast_len(My);
        fast_z = fast_len(Mz);
        if (fast_x) {
            lpb_fx = FastFft<T>::x_lpb(Mx / 2);
            smem_fx = FastFft<T>::x_smem(Mx / 2);
            TRY(raise_smem_cap((const void*)xf_kernel<T>(Mx / 2), smem_fx));
            TRY(raise_smem_cap((const void*)xi_kernel<T>(Mx / 2), smem_fx));
        }
        auto max_cell_rows = [&](int B, double cs) {
            const double span = (double)(B + MG - 1 + 1) * (double)d.h + 2e-3 * (double)d.h;
            return (int)std::ceil(span / cs) + 1;
        };
        if (fast_x && slab_kernels<T>(Mx / 2, sk) && My % sk.BY == 0 && Mz % sk.BZ == 0 &&
            MG == SLAB_MG &&
            (int64_t)std::min(max_cell_rows(sk.BY, (double)d.cell_size[1]), m1) *
                    std::min(max_cell_rows(sk.BZ, (double)d.cell_size[2]), m2) <= SLAB_PAIRMAX &&
            std::getenv("FFCM_NO_SLAB") == nullptr) {
            slab = true;
            sg.m0 = m0; sg.m1 = m1; sg.m2 = m2;
            sg.cs1 = (double)d.cell_size[1];
            sg.cs2 = (double)d.cell_size[2];
            sg.h = (double)d.h;
            sg.nty = My / sk.BY;
            sg.ntz = Mz / sk.BZ;
            sg.zs0 = 0;
            sg.mz_loc = Mz;
            // expected touching particles per slab: N x (rows reached)/(rows total)
            const double expect = (double)N * (sk.BY + MG - 1) * (sk.BZ + MG - 1) / ((double)My * Mz);
            sg.lcap = (int)std::min<double>(1 << 20, std::max(256.0, 4.0 * expect + 64.0));
            sg.lcap = (sg.lcap + 31) / 32 * 32;
            TRY(raise_smem_cap((const void*)sk.spread_fused, sk.smem));
            TRY(raise_smem_cap((const void*)sk.interp, sk.smem_interp));
        }
        mzl = Mz;
        zpitch = hxp;
        nkz = nkx;
        kzoff = 0;
        if (h->distributed) {
            if (!(slab && fast_x && fast_y && fast_z))
                return fail(FFCM_ERR_UNSUPPORTED,
                            "a z-slab decomposition needs the fused slab path: power-of-two grid sides of 64..2048 "
                            "(x), 32..1024 (y, z) and M_G = 8");
            TRY(dist_setup(align));
        }
        if (fast_y) {
            int cand[4];
            const int nc = y_bundles(My, cand);
            for (int i = 0; i < nc; ++i)
                TRY(raise_smem_cap((const void*)y_kernel<T>(My, cand[i]), FastFft<T>::yz_smem(My, cand[i])));
            By = cand[nc - 1];
        }
        if (fast_z) {
            int cand[4];
            const int nc = z_bundles(Mz, cand);
            for (int i = 0; i < nc; ++i)
                TRY(raise_smem_cap((const void*)z_kernel<T>(Mz, cand[i]), FastFft<T>::yz_smem(Mz, cand[i])));
            Bz = cand[nc - 1];
        }
        {
            int dev = 0;
            CUDA_TRY(cudaGetDevice(&dev));
            CUDA_TRY(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
        }
        for (int B : {2, 4, 8, 16}) {
            if (fast_y && ypipe_kernel<T>(My, B) && hxp % B == 0 && ypipe_smem<T>(My, B) <= budget)
                TRY(raise_smem_cap((const void*)ypipe_kernel<T>(My, B), ypipe_smem<T>(My, B)));
            if (fast_y && ytma_kernel<T>(My, B) && ytma_smem<T>(My, B) <= 226 * 1024)
                TRY(raise_smem_cap((const void*)ytma_kernel<T>(My, B), ytma_smem<T>(My, B)));
            if (fast_y && ytma3_kernel<T>(My, B) && ytma_smem<T>(My, B, 3) <= 226 * 1024)
                TRY(raise_smem_cap((const void*)ytma3_kernel<T>(My, B), ytma_smem<T>(My, B, 3)));
            if (fast_z && ztma_kernel<T>(Mz, B) && ztma_smem<T>(Mz, B) <= 226 * 1024)
                TRY(raise_smem_cap((const void*)ztma_kernel<T>(Mz, B), ztma_smem<T>(Mz, B)));
            if (fast_z && zin_kernel<T>(Mz, B) && zin_smem<T>(Mz, B) <= 226 * 1024)
                TRY(raise_smem_cap((const void*)zin_kernel<T>(Mz, B), zin_smem<T>(Mz, B)));
            if (fast_z && zlr_kernel<T>(Mz, B) && FastFft<T>::zlr_smem(Mz, B) <= budget)
                TRY(raise_smem_cap((const void*)zlr_kernel<T>(Mz, B), FastFft<T>::zlr_smem(Mz, B)));
            if (fast_z && zpipe_kernel<T>(Mz, B) && zpitch % B == 0 && zpipe_smem<T>(Mz, B) <= budget)
                TRY(raise_smem_cap((const void*)zpipe_kernel<T>(Mz, B), zpipe_smem<T>(Mz, B)));
        }
        TRY(raise_smem_cap((const void*)k_fft_x_r2c<T>, smem_x));
        TRY(raise_smem_cap((const void*)k_fft_x_c2r<T>, smem_x));
        TRY(raise_smem_cap((const void*)k_fft_y<T>, smem_y));
        TRY(raise_smem_cap((const void*)k_fft_z_stokes<T>, smem_z));
        if (smem_stencil > 48 * 1024) {
            TRY(raise_smem_cap((const void*)k_spread_atomic<T>, smem_stencil));
            TRY(raise_smem_cap((const void*)k_interpolate_warp<T>, smem_stencil));
            TRY(raise_smem_cap((const void*)k_adjoint_gather<T>, smem_stencil));
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
        TRY(alloc(spec, 3 * (size_t)hxp * My * mzl));
        if (dist.on) {
            TRY(alloc(zbuf, 3 * (size_t)zpitch * My * Mz));
            TRY(alloc(dist.send, (size_t)dist.R * dist.blk));
            TRY(alloc(dist.recv, (size_t)dist.R * dist.blk));
            CUDA_TRY(cudaMemset(zbuf, 0, 3 * (size_t)zpitch * My * Mz * sizeof(cplx<T>)));
            CUDA_TRY(cudaMemset(dist.send, 0, (size_t)dist.R * dist.blk * sizeof(cplx<T>)));
            CUDA_TRY(cudaMemset(dist.recv, 0, (size_t)dist.R * dist.blk * sizeof(cplx<T>)));
        } else {
            zbuf = spec;
        }
        TRY(alloc(twx, Mx));
        TRY(alloc(twy, My));
        TRY(alloc(twz, Mz));
        TRY(alloc(kxv, nkx));
        TRY(alloc(kyv, My));
        TRY(alloc(kzv, Mz));
        if (slab) {
            TRY(alloc(partial, 3 * (size_t)N));
            TRY(alloc(slab_lists, (size_t)sg.nty * sg.ntz * sg.lcap));
            TRY(alloc(slab_counts, (size_t)sg.nty * sg.ntz));
        }

        // zero-initialised grids and cell list (src/config.jl:443-448)
        CUDA_TRY(cudaMemset(spec, 0, 3 * (size_t)hxp * My * mzl * sizeof(cplx<T>)));
        if (fast_z || fast_y) make_tma_maps();
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

        // wavevectors (src/config.jl:233-237, 353-356), in T
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
        const char* at = std::getenv("FFCM_AUTOTUNE");
        if (!(at && at[0] == '0')) TRY(autotune());
        return FFCM_OK;
    }

    // Launch-shape autotuner: times every instantiated bundle width of the y
    // and z passes on this configuration's own buffers and keeps the fastest.
    int time_launches(const std::function<int()>& f, float& ms) {
        cudaEvent_t a, b;
        CUDA_TRY(cudaEventCreate(&a));
        CUDA_TRY(cudaEventCreate(&b));
        TRY(f());
        CUDA_TRY(cudaEventRecord(a, h->stream));
        for (int i = 0; i < 3; ++i) TRY(f());
        CUDA_TRY(cudaEventRecord(b, h->stream));
        CUDA_TRY(cudaEventSynchronize(b));
        CUDA_TRY(cudaEventElapsedTime(&ms, a, b));
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        return FFCM_OK;
    }

    int persistent_grid(const void* kernel, int threads, size_t smem, int ntiles, int& grid) {
        int per_sm = 0;
        CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
        if (per_sm < 1) return fail(FFCM_ERR_UNSUPPORTED, "pipelined FFT kernel does not fit on an SM");
        grid = std::max(1, std::min(ntiles, per_sm * num_sms));
        return FFCM_OK;
    }

    // The spectrum as 3-D tensors of 8-byte words for the tiled bulk copies:
    // y pass: `spec` as (kx, y, c mzl + z), boxes of B kx columns x
    // min(256, My) rows x 1 plane; z pass: `zbuf` as (kx, y, c Mz + z), boxes
    // of B kx columns x 1 y x min(256, Mz) rows (the component and z axes merge
    // because a component's stride is the plane count times the z stride).
    void make_tma_maps() {
        TensorMapEncodeFn enc = tensor_map_encoder();
        if (!enc) return;
        constexpr int EPC = TmaElem<T>::PER_CPLX;
        const cuuint32_t estr[3] = {1, 1, 1};
        const CUtensorMapDataType dt = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_UINT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
        auto make = [&](CUtensorMap* m, void* base, int pitch, int planes, cuuint32_t bx, cuuint32_t by,
                        cuuint32_t bz) {
            const cuuint64_t dims[3] = {(cuuint64_t)pitch * EPC, (cuuint64_t)My, (cuuint64_t)planes};
            const cuuint64_t strides[2] = {(cuuint64_t)pitch * sizeof(cplx<T>),
                                           (cuuint64_t)My * pitch * sizeof(cplx<T>)};
            const cuuint32_t box[3] = {bx, by, bz};
            return enc(m, dt, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                       CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
        };
        for (int i = 1, B = 2; B <= 16; ++i, B *= 2) {
            if (fast_z && zpitch % B == 0 && (ztma_kernel<T>(Mz, B) || zin_kernel<T>(Mz, B)))
                zmap_ok[i] = make(&zmap[i], zbuf, zpitch, 3 * Mz, (cuuint32_t)(B * EPC), 1, (cuuint32_t)tma_zbox(Mz));
            if (fast_y && hxp % B == 0 && (ytma_kernel<T>(My, B) || ytma3_kernel<T>(My, B)))
                ymap_ok[i] = make(&ymap[i], spec, hxp, 3 * mzl, (cuuint32_t)(B * EPC), (cuuint32_t)tma_zbox(My), 1);
        }
    }

    static int log2i(int B) { return B == 2 ? 1 : B == 4 ? 2 : B == 8 ? 3 : B == 16 ? 4 : 0; }

    // "kind,B" from an environment variable: pins the autotuner to one
    // variant (tests use it to run every variant); -1 when unset.
    static void forced_variant(const char* name, int& kind, int& B) {
        kind = B = -1;
        const char* v = std::getenv(name);
        if (v && std::sscanf(v, "%d,%d", &kind, &B) != 2) kind = B = -1;
    }

    // True when choice t names variants this configuration can run (a
    // stored or imported choice is used only then; the autotuner runs
    // otherwise).
    bool choice_valid(const TunedChoice& t) const {
        auto in_bundles = [](int n, int B, int (*bundles)(int, int*)) {
            int cand[4];
            const int nc = bundles(n, cand);
            for (int i = 0; i < nc; ++i)
                if (cand[i] == B) return true;
            return false;
        };
        if (fast_y) {
            const int k = t.ykind, B = t.By;
            const bool ok = (k == 0 && y_kernel<T>(My, B) && in_bundles(My, B, y_bundles)) ||
                            (k == 1 && ypipe_kernel<T>(My, B) && hxp % B == 0 &&
                             ypipe_smem<T>(My, B) <= 200 * 1024 && t.ygrid >= 1) ||
                            (k == 2 && ytma_kernel<T>(My, B) && ymap_ok[log2i(B)] &&
                             ytma_smem<T>(My, B) <= 226 * 1024 && t.ygrid >= 1) ||
                            (k == 3 && ytma3_kernel<T>(My, B) && ymap_ok[log2i(B)] &&
                             ytma_smem<T>(My, B, 3) <= 226 * 1024 && t.ygrid >= 1);
            if (!ok) return false;
        }
        if (fast_z) {
            const int k = t.zkind, B = t.Bz;
            const bool ok = (k == 0 && z_kernel<T>(Mz, B) && in_bundles(Mz, B, z_bundles)) ||
                            (k == 1 && zpipe_kernel<T>(Mz, B) && zpitch % B == 0 &&
                             zpipe_smem<T>(Mz, B) <= 200 * 1024 && t.zgrid >= 1) ||
                            (k == 2 && zlr_kernel<T>(Mz, B) && FastFft<T>::zlr_smem(Mz, B) <= 200 * 1024) ||
                            (k == 3 && ztma_kernel<T>(Mz, B) && zmap_ok[log2i(B)] &&
                             ztma_smem<T>(Mz, B) <= 226 * 1024 && t.zgrid >= 1) ||
                            (k == 4 && zin_kernel<T>(Mz, B) && zmap_ok[log2i(B)] &&
                             zin_smem<T>(Mz, B) <= 226 * 1024 && t.zgrid >= 1);
            if (!ok) return false;
        }
        // persistent grids are at most (blocks per SM) x SMs; anything larger
        // came from elsewhere and would launch far too many blocks
        const int gmax = 64 * num_sms;
        if ((fast_y && t.ygrid > gmax) || (fast_z && t.zgrid > gmax)) return false;
        const int c = t.kx_chunk;
        return c == 0 || (fast_y && fast_z && c > 0 && c % t.By == 0 && c % t.Bz == 0 && c < nkx);
    }

    void tuning(int32_t* out) const override {
        out[0] = fast_y ? ykind : -1;
        out[1] = fast_y ? By : -1;
        out[2] = fast_y ? ygrid : -1;
        out[3] = fast_z ? zkind : -1;
        out[4] = fast_z ? Bz : -1;
        out[5] = fast_z ? zgrid : -1;
        out[6] = kx_chunk;
    }

    int autotune() {
        const bool verbose = std::getenv("FFCM_VERBOSE") != nullptr;
        int fyk, fyB, fzk, fzB;
        forced_variant("FFCM_FORCE_Y", fyk, fyB);
        forced_variant("FFCM_FORCE_Z", fzk, fzB);
        // a rank of a decomposition holds other shapes than its key names: it
        // neither reuses nor stores choices
        const bool forced = fyk >= 0 || fzk >= 0 || std::getenv("FFCM_FORCE_CHUNK") != nullptr || dist.on;
        int dev = 0;
        CUDA_TRY(cudaGetDevice(&dev));
        const TuneKey key{dev, (int)sizeof(T), Mx, My, Mz, num_sms};
        if (!forced) {
            std::lock_guard<std::mutex> lock(tune_mu());
            auto it = tune_store().find(key);
            if (it != tune_store().end()) {
                const TunedChoice& t = it->second;
                if (choice_valid(t)) {
                    ykind = t.ykind; By = t.By; ygrid = t.ygrid;
                    zkind = t.zkind; Bz = t.Bz; zgrid = t.zgrid;
                    kx_chunk = t.kx_chunk;
                    if (verbose) fprintf(stderr, "ffcm autotune: reusing the choice for %dx%dx%d\n", Mx, My, Mz);
                    return FFCM_OK;
                }
            }
        }
        if (fast_y) {
            float best = 1e30f;
            int bk = 0, bB = By, bg = 0;
            for (int kind = 0; kind < 4; ++kind)
                for (int B : {2, 4, 8, 16}) {
                    if (fyk >= 0 && (kind != fyk || B != fyB)) continue;
                    if (kind == 0 && !y_kernel<T>(My, B)) continue;
                    if (kind == 1 && !(ypipe_kernel<T>(My, B) && hxp % B == 0 &&
                                       ypipe_smem<T>(My, B) <= 200 * 1024)) continue;
                    if (kind == 2 && !(ytma_kernel<T>(My, B) && ymap_ok[log2i(B)] &&
                                       ytma_smem<T>(My, B) <= 226 * 1024)) continue;
                    if (kind == 3 && !(ytma3_kernel<T>(My, B) && ymap_ok[log2i(B)] &&
                                       ytma_smem<T>(My, B, 3) <= 226 * 1024)) continue;
                    if (kind == 0) {
                        int cand[4];
                        const int nc = y_bundles(My, cand);
                        bool ok = false;
                        for (int i = 0; i < nc; ++i) ok |= cand[i] == B;
                        if (!ok) continue;
                    }
                    ykind = kind;
                    By = B;
                    if (kind == 1) {
                        const int ntiles = ((nkx + B - 1) / B) * mzl * 3;
                        TRY(persistent_grid((const void*)ypipe_kernel<T>(My, B), B * (My / 8),
                                            ypipe_smem<T>(My, B), ntiles, ygrid));
                    }
                    if (kind == 2) {
                        const int ntiles = ((nkx + B - 1) / B) * mzl * 3;
                        TRY(persistent_grid((const void*)ytma_kernel<T>(My, B), B * (My / 8),
                                            ytma_smem<T>(My, B), ntiles, ygrid));
                    }
                    if (kind == 3) {
                        const int ntiles = ((nkx + B - 1) / B) * mzl;
                        TRY(persistent_grid((const void*)ytma3_kernel<T>(My, B), B * (My / 8),
                                            ytma_smem<T>(My, B, 3), ntiles, ygrid));
                    }
                    float ms = 0;
                    TRY(time_launches([&] { return launch_y(h->stream, 0); }, ms));
                    if (verbose) fprintf(stderr, "ffcm autotune: y n=%d kind=%d B=%d %.4f ms\n", My, kind, B, ms / 3);
                    if (ms < best) { best = ms; bk = kind; bB = B; bg = ygrid; }
                }
            if (fyk >= 0 && best == 1e30f) return fail(FFCM_ERR_ARGUMENT, "FFCM_FORCE_Y names no available y variant");
            ykind = bk; By = bB; ygrid = bg;
        }
        if (fast_z) {
            float best = 1e30f;
            int bk = 0, bB = Bz, bg = 0;
            for (int kind = 0; kind < 5; ++kind)
                for (int B : {2, 4, 8, 16}) {
                    if (fzk >= 0 && (kind != fzk || B != fzB)) continue;
                    if (kind == 4 && !(zin_kernel<T>(Mz, B) && zmap_ok[log2i(B)] &&
                                       zin_smem<T>(Mz, B) <= 226 * 1024)) continue;
                    if (kind == 0 && !z_kernel<T>(Mz, B)) continue;
                    if (kind == 1 && !(zpipe_kernel<T>(Mz, B) && zpitch % B == 0 &&
                                       zpipe_smem<T>(Mz, B) <= 200 * 1024)) continue;
                    if (kind == 2 && !(zlr_kernel<T>(Mz, B) && FastFft<T>::zlr_smem(Mz, B) <= 200 * 1024)) continue;
                    if (kind == 3 && !(ztma_kernel<T>(Mz, B) && zmap_ok[log2i(B)] &&
                                       ztma_smem<T>(Mz, B) <= 226 * 1024)) continue;
                    if (kind == 0) {
                        int cand[4];
                        const int nc = z_bundles(Mz, cand);
                        bool ok = false;
                        for (int i = 0; i < nc; ++i) ok |= cand[i] == B;
                        if (!ok) continue;
                    }
                    zkind = kind;
                    Bz = B;
                    if (kind == 1) {
                        const int ntiles = ((nkz + B - 1) / B) * My;
                        TRY(persistent_grid((const void*)zpipe_kernel<T>(Mz, B), B * (Mz / 8),
                                            zpipe_smem<T>(Mz, B), ntiles, zgrid));
                    }
                    if (kind == 3) {
                        const int ntiles = ((nkz + B - 1) / B) * My;
                        TRY(persistent_grid((const void*)ztma_kernel<T>(Mz, B), B * (Mz / 8),
                                            ztma_smem<T>(Mz, B), ntiles, zgrid));
                    }
                    if (kind == 4) {
                        const int ntiles = ((nkz + B - 1) / B) * My;
                        TRY(persistent_grid((const void*)zin_kernel<T>(Mz, B), B * (Mz / 8),
                                            zin_smem<T>(Mz, B), ntiles, zgrid));
                    }
                    float ms = 0;
                    TRY(time_launches([&] { return launch_z(h->stream); }, ms));
                    if (verbose) fprintf(stderr, "ffcm autotune: z n=%d kind=%d B=%d %.4f ms\n", Mz, kind, B, ms / 3);
                    if (ms < best) { best = ms; bk = kind; bB = B; bg = zgrid; }
                }
            if (fzk >= 0 && best == 1e30f) return fail(FFCM_ERR_ARGUMENT, "FFCM_FORCE_Z names no available z variant");
            zkind = bk; Bz = bB; zgrid = bg;
        }
        if (fast_y && fast_z && !dist.on) {
            // chunk widths that keep a chunk's spectrum within ~96 MB of L2
            const double col_bytes = 3.0 * My * Mz * sizeof(cplx<T>);
            float best = 1e30f;
            int bc = 0;
            const char* fc = std::getenv("FFCM_FORCE_CHUNK");
            const int force_c = fc ? std::atoi(fc) : -1;
            for (int c : {0, 64, 32, 16, 8, 4}) {
                if (force_c >= 0 && c != force_c) continue;
                if (c > 0 && (c % By != 0 || c % Bz != 0 || c >= nkx || c * col_bytes > 96e6)) continue;
                kx_chunk = c;
                float ms = 0;
                TRY(time_launches([&] { return stokes_yz(h->stream); }, ms));
                if (verbose) fprintf(stderr, "ffcm autotune: yz chunk=%d %.4f ms\n", c, ms / 3);
                if (ms < best) { best = ms; bc = c; }
            }
            if (force_c > 0 && best == 1e30f)
                return fail(FFCM_ERR_ARGUMENT, "FFCM_FORCE_CHUNK names no available chunk width");
            kx_chunk = bc;
        }
        CUDA_TRY(cudaStreamSynchronize(h->stream));
        h->launches = 0;
        if (!forced) {
            std::lock_guard<std::mutex> lock(tune_mu());
            tune_store()[key] = TunedChoice{ykind, By, ygrid, zkind, Bz, zgrid, kx_chunk};
        }
        return FFCM_OK;
    }
    int tuned_By = 0, tuned_Bz = 0;

    // The real force-density and velocity grids are needed only by the step
    // API and by the generic (non-slab) pipeline; they are allocated, zeroed,
    // on first use.
    int ensure_real_grids() override {
        if (gf) return FFCM_OK;
        TRY(alloc(gf, 3 * (size_t)plane));
        TRY(alloc(gu, 3 * (size_t)plane));
        CUDA_TRY(cudaMemset(gf, 0, 3 * (size_t)plane * sizeof(T)));
        CUDA_TRY(cudaMemset(gu, 0, 3 * (size_t)plane * sizeof(T)));
        return FFCM_OK;
    }

    bool uses_slab() const override { return slab; }
    void set_stencil(int mode) override { sp.comp = mode == FFCM_STENCIL_FLOAT64 ? 1 : 0; }

    int gather_forces(const void* F, cudaStream_t s) override {
        StageScope sc(h, FFCM_STAGE_CELL_LIST, s);
        return launch(h, k_gather_forces<T>, grid_for(N, 256), 256, 0, s, N, (const int32_t*)perm,
                      static_cast<const T*>(F), Fs);
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
                   (const int32_t*)off, cnt, scratch_i));
        return launch(h, k_rank_gather<T>, grid_for(N, 256), 256, 0, s, N, (const int32_t*)key,
                      (const int32_t*)off, (const int32_t*)scratch_i, perm, (const T*)Yw,
                      static_cast<const T*>(F), Ys, Fs);
    }

    // Hot path of the assembled operator: spread straight into the x-transformed
    // spectrum, y/z passes, then x-c2r fused with the interpolation.
    bool fused_available() const { return slab; }

    int spread_to_spectrum(cudaStream_t s, const vec4<T>* force = nullptr, bool build_lists = true) {
        StageScope sc(h, FFCM_STAGE_SPREAD, s);
        const int nslab = sg.nty * sg.ntz;
        if (build_lists)
            TRY(launch(h, sk.lists, (nslab + 7) / 8, 256, 0, s, (const vec4<T>*)Ys, (const int32_t*)off, sp, sg,
                       slab_lists, slab_counts));
        dim3 g(sg.nty, sg.ntz, 1);
        return launch(h, sk.spread_fused, g, 256, sk.smem, s, (const vec4<T>*)Ys,
                      force ? force : (const vec4<T>*)Fs,
                      (const int32_t*)off, spec, hxp, sp, sg, (const cplx<T>*)twx, (const int*)slab_lists,
                      (const int*)slab_counts);
    }

    // y forward, z + projector, y inverse. With kx chunking (kx_chunk > 0) the
    // three passes run chunk by chunk, so a chunk's intermediate spectrum
    // (3 My Mz kx_chunk values) stays in L2 between the passes and only the
    // first read and the last write of each value reach HBM.
    // probe: events recorded on s before and after the y forward pass
    // (probe[0], probe[1]; the unchunked sequence only).
    int stokes_yz(cudaStream_t s, cudaEvent_t* probe = nullptr) {
        if (kx_chunk > 0 && kx_chunk < nkx) {
            StageScope sc(h, FFCM_STAGE_FFT_Z_STOKES, s);
            for (int k0 = 0; k0 < nkx; k0 += kx_chunk) {
                const int k1 = std::min(nkx, k0 + kx_chunk);
                TRY(launch_y(s, 0, k0, k1));
                TRY(launch_z(s, k0, k1));
                TRY(launch_y(s, 1, k0, k1));
            }
            return FFCM_OK;
        }
        {
            StageScope sc(h, FFCM_STAGE_FFT_Y_FWD, s);
            if (probe) CUDA_TRY(cudaEventRecord(probe[0], s));
            TRY(launch_y(s, 0));
            if (probe) CUDA_TRY(cudaEventRecord(probe[1], s));
        }
        {
            StageScope sc(h, FFCM_STAGE_FFT_Z_STOKES, s);
            TRY(launch_z(s));
        }
        StageScope sc(h, FFCM_STAGE_FFT_Y_INV, s);
        return launch_y(s, 1);
    }

    // x-c2r + gather; leaves h^-3 V in sorted order in `partial` for correct_final.
    int interp_from_spectrum(cudaStream_t s) {
        StageScope sc(h, FFCM_STAGE_INTERPOLATE, s);
        CUDA_TRY(cudaMemsetAsync(partial, 0, 3 * (size_t)N * sizeof(T), s));
        dim3 g(sg.nty, sg.ntz, 1);
        return launch(h, sk.interp, g, 256, sk.smem_interp, s, (const vec4<T>*)Ys, (const int32_t*)off,
                      (const cplx<T>*)spec, hxp, partial, sp, sg, (const cplx<T>*)twx,
                      (const int*)slab_lists, (const int*)slab_counts, h->d_err);
    }

    int mobility_rest(void* V, cudaStream_t s) override { return solve(V, s, false); }
    int mobility_rest_same_positions(void* V, cudaStream_t s) override { return solve(V, s, false, false); }
    int apply_fixed(void* V, const void* F, cudaStream_t s) override {
        TRY(gather_forces(F, s));
        TRY(solve(V, s, false, !lists_built));
        lists_built = true;
        return FFCM_OK;
    }

    int ensure_lists(cudaStream_t s) override {
        if (lists_built) return FFCM_OK;
        if (slab) {
            StageScope sc(h, FFCM_STAGE_SPREAD, s);
            const int nslab = sg.nty * sg.ntz;
            TRY(launch(h, sk.lists, (nslab + 7) / 8, 256, 0, s, (const vec4<T>*)Ys, (const int32_t*)off, sp, sg,
                       slab_lists, slab_counts));
        } else {
            TRY(ensure_real_grids());
        }
        lists_built = true;
        return FFCM_OK;
    }

    int cg_start(const void* V, const void* q, void* r, void* p, CgState* st, double reltol, double abstol,
                 int maxiter, cudaStream_t s) override {
        return launch(h, k_cg_start<T>, CG_BLOCKS, CG_THREADS, 0, s, 3 * (int64_t)N, static_cast<const T*>(V),
                      static_cast<const T*>(q), static_cast<T*>(r), static_cast<T*>(p), st, reltol, abstol, maxiter);
    }

    int cg_iteration(void* x, void* r, void* p, void* q, CgState* st, cudaGraphConditionalHandle loop,
                     cudaStream_t s) override {
        const int64_t n = 3 * (int64_t)N;
        TRY(launch(h, k_cg_direction<T>, CG_BLOCKS, CG_THREADS, 0, s, n, static_cast<const T*>(r),
                   static_cast<T*>(p), (const CgState*)st));
        TRY(gather_forces(p, s));
        TRY(solve(q, s, false, false));
        TRY(launch(h, k_cg_alpha<T>, CG_BLOCKS, CG_THREADS, 0, s, n, static_cast<const T*>(p),
                   static_cast<const T*>(q), st));
        return launch(h, k_cg_update<T>, CG_BLOCKS, CG_THREADS, 0, s, n, static_cast<T*>(x), static_cast<T*>(r),
                      static_cast<const T*>(p), static_cast<const T*>(q), st, (const int*)h->d_err, loop);
    }

    // keep_u: also leave the velocity grid u = L^-1 S F in gu (the adjoint's
    // only checkpoint); the unfused pipeline leaves it there anyway.
    int solve(void* V, cudaStream_t s, bool keep_u, bool build_lists = true) {
        if (!slab) {
            TRY(spread(s));
            TRY(stokes(s));
            TRY(interp(V, s));
            return correct(V, s);
        }
        TRY(spread_to_spectrum(s, nullptr, build_lists));
        bool side = false, probe = false;
        TRY(fork_pairs(s, side, probe));
        TRY(stokes_yz(s, probe ? h->ev_probe : nullptr));
        if (keep_u) {
            StageScope sc(h, FFCM_STAGE_FFT_X_INV, s);
            TRY(x_inverse(gu, s));
        }
        TRY(interp_from_spectrum(s));
        if (side) {
            // (the correction stage's time is the side stream's pair kernel's)
            CUDA_TRY(cudaStreamWaitEvent(s, h->ev_join, 0));
            return launch(h, k_finish_velocity<T>, grid_for(N, 256), 256, 0, s, N, (const int32_t*)perm,
                          (const T*)partial, (const T*)dvs, h3, static_cast<T*>(V));
        }
        StageScope sc(h, FFCM_STAGE_CORRECT, s);
        if (probe) CUDA_TRY(cudaEventRecord(h->ev_probe[2], s));
        TRY(launch(h, corr_tpp(N) == 4 ? k_correct<T, 4> : k_correct<T, 1>, grid_for((int64_t)N * corr_tpp(N), 128), 128, 0, s, N, (const vec4<T>*)Ys,
                   (const vec4<T>*)Fs, (const int32_t*)off, (const int32_t*)perm,
                   static_cast<T*>(V), cc, (const T*)partial, h3));
        if (probe) CUDA_TRY(cudaEventRecord(h->ev_probe[3], s));
        return FFCM_OK;
    }

    // The pair correction depends only on the sorted particles and the cell
    // list, so outside stream capture it can run on the handle's side stream
    // while the y/z passes and the interpolation run on s: the fork follows
    // the spread (the y pass leaves a third of each SM's registers free, the
    // spread none), the join precedes k_finish_velocity. That pays while the
    // correction is short next to a y pass (it then runs in the y pass's
    // spare registers: 0.16 against 0.62 ms at 512^3, 10% by volume), and
    // costs when it is long (dense clusters: 7.7 against 6.0 ms at 1024^3,
    // where it slows the z pass by about its own time). So unless
    // FFCM_OVERLAP_PAIRS forces a mode, the first solve runs on one stream
    // with events around its y forward pass and its correction, and a later
    // solve, once those have completed, fixes the mode for the configuration:
    // overlap when the correction took under half the y pass. `side` tells
    // the caller whether it forked, `probe` whether to record the events
    // (ev_probe[0..1] around the y forward pass, [2..3] around k_correct).
    // Under capture (the batched graph, the CG loop) the solve keeps the
    // single-stream order.
    int fork_pairs(cudaStream_t s, bool& side, bool& probe) {
        side = false;
        probe = false;
        if (h->overlap_pairs == 0) return FFCM_OK;
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        CUDA_TRY(cudaStreamIsCapturing(s, &cap));
        if (cap != cudaStreamCaptureStatusNone) return FFCM_OK;
        if (h->overlap_pairs < 0) {
            if (h->pair_probe == 0) {
                if (kx_chunk > 0 && kx_chunk < nkx) {   // chunked y/z/y: no lone y pass to time
                    h->pair_probe = 2;
                    h->pair_overlap = false;
                    return FFCM_OK;
                }
                for (cudaEvent_t& e : h->ev_probe)
                    if (!e) CUDA_TRY(cudaEventCreate(&e));
                h->pair_probe = 1;
                probe = true;
                return FFCM_OK;
            }
            if (h->pair_probe == 1) {
                const cudaError_t q = cudaEventQuery(h->ev_probe[3]);
                if (q == cudaErrorNotReady) {
                    (void)cudaGetLastError();   // not an error: the probe solve is still running
                    return FFCM_OK;
                }
                CUDA_TRY(q);
                float ty = 0, tc = 0;
                CUDA_TRY(cudaEventElapsedTime(&ty, h->ev_probe[0], h->ev_probe[1]));
                CUDA_TRY(cudaEventElapsedTime(&tc, h->ev_probe[2], h->ev_probe[3]));
                h->pair_overlap = tc < 0.5f * ty;
                h->pair_probe = 2;
            }
            if (!h->pair_overlap) return FFCM_OK;
        }
        if (!dvs) TRY(alloc(dvs, 3 * (size_t)N));
        if (!h->side_stream) {
            CUDA_TRY(cudaStreamCreateWithFlags(&h->side_stream, cudaStreamNonBlocking));
            CUDA_TRY(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
            CUDA_TRY(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
        }
        CUDA_TRY(cudaEventRecord(h->ev_fork, s));
        CUDA_TRY(cudaStreamWaitEvent(h->side_stream, h->ev_fork, 0));
        {
            StageScope sc(h, FFCM_STAGE_CORRECT, h->side_stream);
            TRY(launch(h, corr_tpp(N) == 4 ? k_correct_pairs<T, 4> : k_correct_pairs<T, 1>,
                       grid_for((int64_t)N * corr_tpp(N), 128), 128, 0, h->side_stream, N, (const vec4<T>*)Ys,
                       (const vec4<T>*)Fs, (const int32_t*)off, cc, dvs));
        }
        CUDA_TRY(cudaEventRecord(h->ev_join, h->side_stream));
        side = true;
        return FFCM_OK;
    }

    // ---- z-slab decomposition --------------------------------------------
    int dist_setup(int align) {
        dist.on = true;
        dist.R = h->nranks;
        dist.r = h->rank;
        const int nzs = Mz / sk.BZ;
        if (dist.R < 1 || dist.r < 0 || dist.r >= dist.R)
            return fail(FFCM_ERR_ARGUMENT, "rank must lie in [0, nranks)");
        if (dist.R > nzs || dist.R > nkx)
            return fail(FFCM_ERR_ARGUMENT, "more ranks (" + std::to_string(dist.R) + ") than z slabs (" +
                                               std::to_string(nzs) + ") or kx columns (" + std::to_string(nkx) + ")");
        dist.zb.resize(dist.R);
        dist.ze.resize(dist.R);
        dist.kb.resize(dist.R);
        dist.ke.resize(dist.R);
        for (int q = 0; q < dist.R; ++q) {
            dist_ranges(Mz, sk.BZ, nkx, dist.R, q, dist.zb[q], dist.ze[q], dist.kb[q], dist.ke[q]);
            dist.mzl_max = std::max(dist.mzl_max, dist.ze[q] - dist.zb[q]);
            dist.nk_max = std::max(dist.nk_max, dist.ke[q] - dist.kb[q]);
        }
        const int r = dist.r;
        sg.zs0 = dist.zb[r] / sk.BZ;
        sg.ntz = (dist.ze[r] - dist.zb[r]) / sk.BZ;
        sg.mz_loc = dist.ze[r] - dist.zb[r];
        mzl = sg.mz_loc;
        kzoff = dist.kb[r];
        nkz = dist.ke[r] - dist.kb[r];
        zpitch = ((dist.nk_max + align - 1) / align) * align;
        dist.blk = 3 * (int64_t)dist.mzl_max * My * dist.nk_max;
        return FFCM_OK;
    }

    int copy_block(cplx<T>* dst, int64_t dc, int64_t dz, int64_t dy, const cplx<T>* src, int64_t sc, int64_t sz,
                   int64_t sy, int nz, int ny, int nk, cudaStream_t s) {
        if (nz <= 0 || nk <= 0) return FFCM_OK;
        const int rows = 3 * nz * ny;
        return launch(h, k_copy_block<T>, std::min(rows, num_sms * 32), 128, 0, s, dst, dc, dz, dy,
                      (const cplx<T>*)src, sc, sz, sy, nz, ny, nk);
    }

    // Peer q's block of a transpose buffer: [c][z < mzl_max][y][k < nk_max].
    int64_t bc() const { return (int64_t)dist.mzl_max * My * dist.nk_max; }
    int64_t bz() const { return (int64_t)My * dist.nk_max; }

    // Cell list (all particles), own slabs' lists, spread into the own z
    // planes, y forward; then the first transpose's send blocks: peer q gets
    // this rank's planes at q's kx columns.
    int dist_forward(const void* Y, const void* F, cudaStream_t s) override {
        TRY(wrap_hash(Y, true, true, s));
        TRY(sort(F, s));
        TRY(spread_to_spectrum(s, nullptr, true));
        {
            StageScope sc(h, FFCM_STAGE_FFT_Y_FWD, s);
            TRY(launch_y(s, 0));
        }
        StageScope sc(h, FFCM_STAGE_FFT_Z_STOKES, s);
        for (int q = 0; q < dist.R; ++q)
            TRY(copy_block(dist.send + q * dist.blk, bc(), bz(), dist.nk_max, spec + dist.kb[q],
                           (int64_t)mzl * My * hxp, (int64_t)My * hxp, hxp, mzl, My, dist.ke[q] - dist.kb[q], s));
        return FFCM_OK;
    }

    // Received blocks (every rank's planes at this rank's kx columns) into the
    // z-pass buffer, z pass and projector, and the second transpose's send
    // blocks: peer q gets its planes at this rank's columns.
    int dist_stokes(cudaStream_t s) override {
        StageScope sc(h, FFCM_STAGE_FFT_Z_STOKES, s);
        const int64_t zc = (int64_t)Mz * My * zpitch, zz = (int64_t)My * zpitch;
        for (int q = 0; q < dist.R; ++q)
            TRY(copy_block(zbuf + dist.zb[q] * zz, zc, zz, zpitch, dist.recv + q * dist.blk, bc(), bz(), dist.nk_max,
                           dist.ze[q] - dist.zb[q], My, nkz, s));
        TRY(launch_z(s));
        for (int q = 0; q < dist.R; ++q)
            TRY(copy_block(dist.send + q * dist.blk, bc(), bz(), dist.nk_max, zbuf + dist.zb[q] * zz, zc, zz, zpitch,
                           dist.ze[q] - dist.zb[q], My, nkz, s));
        return FFCM_OK;
    }

    // Received blocks (this rank's planes at every rank's columns) back into
    // the spectrum, y inverse, and the own slabs' interpolation shares in
    // `partial` (3N, zeroed first; the host sums it over ranks).
    int dist_interp(cudaStream_t s) override {
        {
            StageScope sc(h, FFCM_STAGE_FFT_Y_INV, s);
            for (int q = 0; q < dist.R; ++q)
                TRY(copy_block(spec + dist.kb[q], (int64_t)mzl * My * hxp, (int64_t)My * hxp, hxp,
                               dist.recv + q * dist.blk, bc(), bz(), dist.nk_max, mzl, My, dist.ke[q] - dist.kb[q], s));
            TRY(launch_y(s, 1));
        }
        return interp_from_spectrum(s);
    }

    // V = h^3 partial + the pair correction, with `partial` summed over ranks.
    int dist_correct(void* V, cudaStream_t s) override {
        StageScope sc(h, FFCM_STAGE_CORRECT, s);
        return launch(h, corr_tpp(N) == 4 ? k_correct<T, 4> : k_correct<T, 1>, grid_for((int64_t)N * corr_tpp(N), 128),
                      128, 0, s, N, (const vec4<T>*)Ys, (const vec4<T>*)Fs, (const int32_t*)off, (const int32_t*)perm,
                      static_cast<T*>(V), cc, (const T*)partial, h3);
    }

    void dist_info(void** send, void** recv, int64_t* block_bytes, void** partial_out,
                   int32_t* ranges) const override {
        if (send) *send = dist.send;
        if (recv) *recv = dist.recv;
        if (block_bytes) *block_bytes = dist.blk * (int64_t)sizeof(cplx<T>);
        if (partial_out) *partial_out = partial;
        if (ranges) {
            ranges[0] = dist.zb[dist.r];
            ranges[1] = dist.ze[dist.r];
            ranges[2] = dist.kb[dist.r];
            ranges[3] = dist.ke[dist.r];
        }
    }

    int spread(cudaStream_t s) override { return spread_from((const vec4<T>*)Fs, s); }

    // step API (spread_forces!): depends on Y_sorted/F_sorted only, as the
    // reference's, so it does not use the cell-list-driven slab kernel
    int spread_from(const vec4<T>* force, cudaStream_t s) {
        TRY(ensure_real_grids());
        StageScope sc(h, FFCM_STAGE_SPREAD, s);
        CUDA_TRY(cudaMemsetAsync(gf, 0, 3 * (size_t)plane * sizeof(T), s));
        return launch(h, k_spread_atomic<T>, grid_for((int64_t)N * 32, 256, 148 * 64), 256,
                      smem_stencil, s, N, (const vec4<T>*)Ys, force, gf, sp);
    }

    int forward_checkpoint(void* V, cudaStream_t s) override {
        TRY(ensure_adjoint());
        return solve(V, s, true);
    }

    int ensure_adjoint() override {
        TRY(ensure_real_grids());
        if (gpsi) return FFCM_OK;
        TRY(alloc(Ls, N));
        TRY(alloc(Lin, 3 * (size_t)N));
        TRY(alloc(dYo, 3 * (size_t)N));
        TRY(alloc(dFo, 3 * (size_t)N));
        TRY(alloc(Vt, 3 * (size_t)N));
        TRY(alloc(Jd, 1));
        TRY(alloc(gpsi, 3 * (size_t)plane));
        CUDA_TRY(cudaMemset(Ls, 0, (size_t)N * sizeof(vec4<T>)));
        CUDA_TRY(cudaMemset(gpsi, 0, 3 * (size_t)plane * sizeof(T)));
        return FFCM_OK;
    }

    void* adj_buf(int which) override {
        switch (which) {
            case 0: return Lin;
            case 1: return dYo;
            case 2: return dFo;
            case 3: return Vt;
            default: return Jd;
        }
    }

    // Pullback at cotangent lam of the last checkpointed forward (cell list,
    // sorted Y/F and the velocity grid u still in place): psi = L^-1 S lam,
    // then one stencil gather over (u, psi) and one pair pass.
    int adjoint(const void* lam, void* dY, void* dF, cudaStream_t s) override {
        TRY(ensure_adjoint());
        {
            StageScope sc(h, FFCM_STAGE_CELL_LIST, s);
            TRY(launch(h, k_gather_forces<T>, grid_for(N, 256), 256, 0, s, N, (const int32_t*)perm,
                       static_cast<const T*>(lam), Ls));
        }
        if (slab) {
            TRY(spread_to_spectrum(s, Ls, false));   // the checkpoint's lists
            TRY(stokes_yz(s));
            StageScope sc(h, FFCM_STAGE_FFT_X_INV, s);
            TRY(x_inverse(gpsi, s));
        } else {
            TRY(spread_from(Ls, s));
            TRY(stokes_to(gpsi, s));
        }
        {
            StageScope sc(h, FFCM_STAGE_INTERPOLATE, s);
            TRY(launch(h, k_adjoint_gather<T>, grid_for((int64_t)N * 32, 256, 148 * 64), 256, smem_stencil, s, N,
                       (const vec4<T>*)Ys, (const vec4<T>*)Fs, (const vec4<T>*)Ls, (const int32_t*)perm,
                       (const T*)gu, (const T*)gpsi, static_cast<T*>(dY), static_cast<T*>(dF), sp, h3));
        }
        StageScope sc(h, FFCM_STAGE_CORRECT, s);
        return launch(h, corr_tpp(N) == 4 ? k_correct_adjoint<T, 4> : k_correct_adjoint<T, 1>,
                      grid_for((int64_t)N * corr_tpp(N), 128), 128, 0, s, N, (const vec4<T>*)Ys,
                      (const vec4<T>*)Fs, (const vec4<T>*)Ls, (const int32_t*)off, (const int32_t*)perm,
                      static_cast<T*>(dY), static_cast<T*>(dF), cc, cgc);
    }

    int residual(const void* V, const void* Vtg, void* lam, double* J, cudaStream_t s) override {
        CUDA_TRY(cudaMemsetAsync(J, 0, sizeof(double), s));
        return launch(h, k_residual<T>, grid_for(3 * (int64_t)N, 256, 148 * 8), 256, 0, s, 3 * N,
                      static_cast<const T*>(V), static_cast<const T*>(Vtg), static_cast<T*>(lam), J);
    }

    // y pass over the kx columns [k0, k1) (the whole spectrum when k1 <= 0).
    int launch_y(cudaStream_t s, int inverse, int k0 = 0, int k1 = 0) {
        if (k1 <= 0) k1 = nkx;
        if (fast_y && ykind == 3) {   // three planes per tile
            const int ntiles = ((k1 - k0 + By - 1) / By) * mzl;
            return launch(h, ytma3_kernel<T>(My, By), std::min(ygrid, ntiles), By * (My / 8),
                          ytma_smem<T>(My, By, 3), s, ymap[log2i(By)], spec, k0, k1, mzl, hxp, (const cplx<T>*)twy,
                          inverse, h->d_err);
        }
        if (fast_y && ykind == 2) {
            const int ntiles = ((k1 - k0 + By - 1) / By) * mzl * 3;
            return launch(h, ytma_kernel<T>(My, By), std::min(ygrid, ntiles), By * (My / 8), ytma_smem<T>(My, By),
                          s, ymap[log2i(By)], spec, k0, k1, mzl, hxp, (const cplx<T>*)twy, inverse, h->d_err);
        }
        if (fast_y && ykind == 1) {
            const int ntiles = ((k1 - k0 + By - 1) / By) * mzl * 3;
            return launch(h, ypipe_kernel<T>(My, By), std::min(ygrid, ntiles), By * (My / 8), ypipe_smem<T>(My, By),
                          s, spec, k0, k1, mzl, hxp, (const cplx<T>*)twy, inverse);
        }
        if (fast_y) {
            dim3 g((k1 - k0 + By - 1) / By, mzl, 3);
            return launch(h, y_kernel<T>(My, By), g, By * (My / 8), FastFft<T>::yz_smem(My, By), s, spec,
                          k0, k1, My, mzl, hxp, (const cplx<T>*)twy, inverse);
        }
        dim3 gy((nkx + tx_y - 1) / tx_y, mzl, 3);
        return launch(h, k_fft_y<T>, gy, 256, smem_y, s, spec, nkx, My, mzl, hxp, plan_y,
                      (const cplx<T>*)twy, tx_y, inverse);
    }

    int launch_z(cudaStream_t s, int k0 = 0, int k1 = 0) {
        if (k1 <= 0) k1 = nkz;
        const T* kxz = kxv + kzoff;   // wavevectors of the columns zbuf holds
        if (fast_z && zkind == 4) {
            const int ntiles = ((k1 - k0 + Bz - 1) / Bz) * My;
            return launch(h, zin_kernel<T>(Mz, Bz), std::min(zgrid, ntiles), Bz * (Mz / 8), zin_smem<T>(Mz, Bz), s,
                          zmap[log2i(Bz)], zbuf, k0, k1, My, zpitch, (const cplx<T>*)twz, kxz,
                          (const T*)kyv, (const T*)kzv, inv_mu_M, h->d_err);
        }
        if (fast_z && zkind == 3) {
            const int ntiles = ((k1 - k0 + Bz - 1) / Bz) * My;
            return launch(h, ztma_kernel<T>(Mz, Bz), std::min(zgrid, ntiles), Bz * (Mz / 8), ztma_smem<T>(Mz, Bz), s,
                          zmap[log2i(Bz)], zbuf, k0, k1, My, zpitch, (const cplx<T>*)twz, kxz,
                          (const T*)kyv, (const T*)kzv, inv_mu_M, h->d_err);
        }
        if (fast_z && zkind == 2) {
            dim3 g((k1 - k0 + Bz - 1) / Bz, My, 1);
            return launch(h, zlr_kernel<T>(Mz, Bz), g, Bz * (Mz / 8), FastFft<T>::zlr_smem(Mz, Bz), s, zbuf,
                          k0, k1, My, zpitch, (const cplx<T>*)twz, kxz, (const T*)kyv,
                          (const T*)kzv, inv_mu_M);
        }
        if (fast_z && zkind == 1) {
            const int ntiles = ((k1 - k0 + Bz - 1) / Bz) * My;
            return launch(h, zpipe_kernel<T>(Mz, Bz), std::min(zgrid, ntiles), Bz * (Mz / 8), zpipe_smem<T>(Mz, Bz),
                          s, zbuf, k0, k1, My, zpitch, (const cplx<T>*)twz, kxz, (const T*)kyv,
                          (const T*)kzv, inv_mu_M);
        }
        if (fast_z) {
            dim3 g((k1 - k0 + Bz - 1) / Bz, My, 1);
            return launch(h, z_kernel<T>(Mz, Bz), g, Bz * (Mz / 8), FastFft<T>::yz_smem(Mz, Bz), s, zbuf,
                          k0, k1, My, zpitch, (const cplx<T>*)twz, kxz, (const T*)kyv,
                          (const T*)kzv, inv_mu_M);
        }
        dim3 gz((nkz + tx_z - 1) / tx_z, My, 1);
        return launch(h, k_fft_z_stokes<T>, gz, 256, smem_z, s, zbuf, nkz, My, Mz, zpitch, plan_z,
                      (const cplx<T>*)twz, tx_z, kxz, (const T*)kyv, (const T*)kzv, inv_mu_M);
    }

    int stokes(cudaStream_t s) override {
        TRY(ensure_real_grids());
        return stokes_to(gu, s);
    }

    int x_forward(const T* in, cudaStream_t s) {
        const int nrows = 3 * My * Mz;
        if (fast_x) {
            const int H = Mx / 2;
            return launch(h, xf_kernel<T>(H), (nrows + lpb_fx - 1) / lpb_fx, lpb_fx * (H / 8), smem_fx, s, in,
                          spec, nrows, hxp, (const cplx<T>*)twx, lpb_fx);
        }
        return launch(h, k_fft_x_r2c<T>, (nrows + lpb_x - 1) / lpb_x, 256, smem_x, s, in, spec, Mx, nrows, hxp,
                      plan_x, (const cplx<T>*)twx, lpb_x);
    }

    int x_inverse(T* out, cudaStream_t s) {
        const int nrows = 3 * My * Mz;
        if (fast_x) {
            const int H = Mx / 2;
            return launch(h, xi_kernel<T>(H), (nrows + lpb_fx - 1) / lpb_fx, lpb_fx * (H / 8), smem_fx, s,
                          (const cplx<T>*)spec, out, nrows, hxp, (const cplx<T>*)twx, lpb_fx);
        }
        return launch(h, k_fft_x_c2r<T>, (nrows + lpb_x - 1) / lpb_x, 256, smem_x, s, (const cplx<T>*)spec, out,
                      Mx, nrows, hxp, plan_x, (const cplx<T>*)twx, lpb_x);
    }

    // gf -> out through the full transform and the Stokes projector.
    int stokes_to(T* out, cudaStream_t s) {
        {
            StageScope sc(h, FFCM_STAGE_FFT_X_FWD, s);
            TRY(x_forward(gf, s));
        }
        TRY(stokes_yz(s));
        StageScope sc(h, FFCM_STAGE_FFT_X_INV, s);
        return x_inverse(out, s);
    }

    int interp(void* V, cudaStream_t s) override {
        TRY(ensure_real_grids());
        StageScope sc(h, FFCM_STAGE_INTERPOLATE, s);
        return launch(h, k_interpolate_warp<T>, grid_for((int64_t)N * 32, 256, 148 * 64), 256,
                      smem_stencil, s, N, (const vec4<T>*)Ys, (const int32_t*)perm,
                      (const T*)gu, static_cast<T*>(V), sp, h3);
    }

    int correct(void* V, cudaStream_t s) override {
        StageScope sc(h, FFCM_STAGE_CORRECT, s);
        return launch(h, corr_tpp(N) == 4 ? k_correct<T, 4> : k_correct<T, 1>, grid_for((int64_t)N * corr_tpp(N), 128), 128, 0, s, N, (const vec4<T>*)Ys,
                      (const vec4<T>*)Fs, (const int32_t*)off, (const int32_t*)perm,
                      static_cast<T*>(V), cc, (const T*)nullptr, T(0));
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

// The whole-system entry points: a rank of a z-slab decomposition holds only
// its own planes of the spectrum and answers to the ffcm_dist_* calls only.
int check_whole(const ffcm_handle* h) {
    TRY(check_handle(h));
    if (h->distributed)
        return fail(FFCM_ERR_STATE, "a rank of a z-slab decomposition takes the ffcm_dist_* calls only");
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

// FFCM_DEVICE arguments are read and written by kernels launched on `device`.
// Memory of another GPU, or a host pointer that CUDA does not know, would
// fault there instead of failing the call, so both are rejected up front.
// Pinned (registered) host memory and managed memory are reachable from every
// GPU and pass. NULL entries are skipped (the callers check them).
int check_device_ptrs(int device, std::initializer_list<const void*> ptrs) {
    for (const void* p : ptrs) {
        if (!p) continue;
        cudaPointerAttributes a{};
        const cudaError_t e = cudaPointerGetAttributes(&a, p);
        if (e != cudaSuccess) {
            cudaGetLastError();   // clear the non-sticky error
            return fail(FFCM_ERR_ARGUMENT, std::string("an FFCM_DEVICE pointer is not CUDA memory: ") +
                                               cudaGetErrorString(e));
        }
        if (a.type == cudaMemoryTypeUnregistered)
            return fail(FFCM_ERR_ARGUMENT, "an FFCM_DEVICE pointer is ordinary host memory; pass FFCM_HOST");
        if (a.type == cudaMemoryTypeDevice && a.device != device)
            return fail(FFCM_ERR_ARGUMENT, "an FFCM_DEVICE pointer lives on GPU " + std::to_string(a.device) +
                                               ", the configuration on GPU " + std::to_string(device));
    }
    return FFCM_OK;
}

// check_memory, then (device memory only) check_device_ptrs.
int check_args(int device, int32_t memory, std::initializer_list<const void*> ptrs) {
    TRY(check_memory(memory));
    return memory == FFCM_DEVICE ? check_device_ptrs(device, ptrs) : FFCM_OK;
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
        if (e & DEVERR_COPY_TIMEOUT)
            return fail(FFCM_ERR_TIMEOUT, "a bounded device-side wait for a bulk copy gave up");
        return fail(FFCM_ERR_CUDA, "device-side error flag " + std::to_string(e));
    }
    return FFCM_OK;
}

void cg_release(ffcm_handle* h) {
    auto& c = h->cg;
    if (c.exec) cudaGraphExecDestroy(c.exec);
    if (c.graph) cudaGraphDestroy(c.graph);
    if (c.cs) cudaStreamDestroy(c.cs);
    for (void* p : {c.x, c.r, c.p, c.q, (void*)c.st})
        if (p) cudaFree(p);
    if (c.host) cudaFreeHost(c.host);
    c = ffcm_handle::Cg{};
}

// Buffers and the graph of the iteration loop, made once per handle: a gate
// kernel that sets the loop condition from the start kernel's status, then a
// while node whose body is one iteration captured on the handle's capture
// stream. The graph holds only buffers of the handle, so it stays valid
// across ffcm_set_positions calls (the particle lists are rebuilt outside it).
int cg_build(ffcm_handle* h) {
    auto& c = h->cg;
    const size_t bytes = 3 * (size_t)h->N * h->esize;
    for (void** p : {&c.x, &c.r, &c.p, &c.q}) CUDA_TRY(cudaMalloc(p, bytes));
    CUDA_TRY(cudaMalloc(&c.st, sizeof(CgState)));
    CUDA_TRY(cudaMemset(c.st, 0, sizeof(CgState)));
    CUDA_TRY(cudaMallocHost(&c.host, sizeof(CgState)));
    CUDA_TRY(cudaStreamCreateWithFlags(&c.cs, cudaStreamNonBlocking));
    CUDA_TRY(cudaGraphCreate(&c.graph, 0));
    CUDA_TRY(cudaGraphConditionalHandleCreate(&c.loop, c.graph, 0, cudaGraphCondAssignDefault));
    cudaGraphNode_t gate = nullptr, loop = nullptr;
    {
        const CgState* st = c.st;
        cudaGraphConditionalHandle lh = c.loop;
        void* args[] = {(void*)&st, (void*)&lh};
        cudaKernelNodeParams kp = {};
        kp.func = (void*)k_cg_gate;
        kp.gridDim = dim3(1);
        kp.blockDim = dim3(32);
        kp.kernelParams = args;
        CUDA_TRY(cudaGraphAddKernelNode(&gate, c.graph, nullptr, 0, &kp));
    }
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = c.loop;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    CUDA_TRY(cudaGraphAddNode(&loop, c.graph, &gate, 1, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    // event records are not allowed in a conditional body: no stage timing
    const bool prof = h->profiling;
    h->profiling = false;
    CUDA_TRY(cudaStreamBeginCaptureToGraph(c.cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    const int64_t launches0 = h->launches;
    const int rc = h->eng->cg_iteration(c.x, c.r, c.p, c.q, c.st, c.loop, c.cs);
    c.body_kernels = h->launches - launches0;
    const std::string msg = g_err;
    const cudaError_t ce = cudaStreamEndCapture(c.cs, &body);
    h->profiling = prof;
    if (rc != FFCM_OK) return fail(rc, "capture of the conjugate-gradient iteration failed: " + msg);
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture (conjugate-gradient iteration)");
    CUDA_TRY(cudaGraphInstantiate(&c.exec, c.graph, 0));
    return FFCM_OK;
}

int cg_prepare(ffcm_handle* h) {
    if (h->cg.exec) return FFCM_OK;
    const int rc = cg_build(h);
    if (rc != FFCM_OK) {
        const std::string msg = g_err;
        cg_release(h);
        return fail(rc, msg);
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

// A configuration on `device`; with `distributed`, rank `rank` of a z-slab
// decomposition over `nranks`.
static int create_handle(ffcm_handle** out, int32_t dtype, const double* L, double R_c, int64_t N, double a,
                         double ratio, const int32_t* M, int32_t M_G, double mu, int32_t planning, int32_t threads,
                         int32_t device, bool distributed, int32_t nranks, int32_t rank) {
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
    h->distributed = distributed;
    h->nranks = nranks;
    h->rank = rank;
    {
        const char* v = std::getenv("FFCM_STENCIL");
        if (v && std::strcmp(v, "float64") == 0) h->stencil = FFCM_STENCIL_FLOAT64;
        else if (v && *v && std::strcmp(v, "reference") != 0)
            return fail(FFCM_ERR_ARGUMENT, "FFCM_STENCIL must be \"reference\" or \"float64\"");
    }
    {
        const char* v = std::getenv("FFCM_OVERLAP_PAIRS");
        if (v && std::strcmp(v, "0") == 0) h->overlap_pairs = 0;
        else if (v && std::strcmp(v, "1") == 0) h->overlap_pairs = 1;
        else if (v && *v) return fail(FFCM_ERR_ARGUMENT, "FFCM_OVERLAP_PAIRS must be \"0\" or \"1\"");
    }
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

int ffcm_create(ffcm_handle** out, int32_t dtype, const double* L, double R_c, int64_t N,
                double a, double ratio, const int32_t* M, int32_t M_G, double mu,
                int32_t planning, int32_t threads, int32_t device) {
    return create_handle(out, dtype, L, R_c, N, a, ratio, M, M_G, mu, planning, threads, device, false, 1, 0);
}

int ffcm_dist_partition(int32_t dtype, const int32_t* M, int32_t nranks, int32_t rank, int32_t* ranges) {
    g_err.clear();
    if (!M || !ranges) return fail(FFCM_ERR_ARGUMENT, "M and ranges must not be NULL");
    if (dtype != FFCM_FLOAT32 && dtype != FFCM_FLOAT64)
        return fail(FFCM_ERR_ARGUMENT, "dtype must be FFCM_FLOAT32 or FFCM_FLOAT64");
    if (nranks < 1 || rank < 0 || rank >= nranks) return fail(FFCM_ERR_ARGUMENT, "rank must lie in [0, nranks)");
    if (M[0] < 2 || (M[0] & (M[0] - 1)) || M[2] < 1)
        return fail(FFCM_ERR_UNSUPPORTED, "a z-slab decomposition needs a power-of-two x side");
    int BZ = 0;
    if (dtype == FFCM_FLOAT32) {
        SlabKernels<float> k;
        if (!slab_kernels<float>(M[0] / 2, k)) return fail(FFCM_ERR_UNSUPPORTED, "no slab kernels for this x side");
        BZ = k.BZ;
    } else {
        SlabKernels<double> k;
        if (!slab_kernels<double>(M[0] / 2, k)) return fail(FFCM_ERR_UNSUPPORTED, "no slab kernels for this x side");
        BZ = k.BZ;
    }
    const int nkx = M[0] / 2 + 1;
    if (M[2] % BZ != 0 || nranks > M[2] / BZ || nranks > nkx)
        return fail(FFCM_ERR_ARGUMENT, "more ranks than z slabs or kx columns");
    dist_ranges(M[2], BZ, nkx, nranks, rank, ranges[0], ranges[1], ranges[2], ranges[3]);
    return FFCM_OK;
}

int ffcm_dist_create(ffcm_handle** out, int32_t dtype, const double* L, double R_c, int64_t N, double a,
                     double ratio, const int32_t* M, int32_t M_G, double mu, int32_t nranks, int32_t rank,
                     int32_t device) {
    return create_handle(out, dtype, L, R_c, N, a, ratio, M, M_G, mu, FFCM_FFT_ESTIMATE, 1, device, true, nranks,
                         rank);
}

int ffcm_dist_buffers(const ffcm_handle* h, void** send, void** recv, int64_t* block_bytes, void** partial,
                      int32_t* ranges) {
    g_err.clear();
    TRY(check_handle(h));
    if (!h->distributed) return fail(FFCM_ERR_STATE, "not a rank of a z-slab decomposition (ffcm_dist_create)");
    h->eng->dist_info(send, recv, block_bytes, partial, ranges);
    return FFCM_OK;
}

int ffcm_dist_forward(ffcm_handle* h, const void* Y, const void* F, int32_t memory, void* stream) {
    g_err.clear();
    TRY(check_handle(h));
    if (!h->distributed) return fail(FFCM_ERR_STATE, "not a rank of a z-slab decomposition (ffcm_dist_create)");
    TRY(check_args(h->device, memory, {Y, F}));
    if (!Y || !F) return fail(FFCM_ERR_ARGUMENT, "Y and F must not be NULL");
    h->ckpt = false;
    h->positions = false;
    DeviceGuard g(h->device);
    cudaStream_t s = h->pick(stream);
    EngineBase* e = h->eng.get();
    const size_t bytes = 3 * (size_t)h->N * h->esize;
    const void *Yd = Y, *Fd = F;
    if (memory == FFCM_HOST) {
        StageScope sc(h, FFCM_STAGE_H2D, s);
        CUDA_TRY(cudaMemcpyAsync(e->Y_in(), Y, bytes, cudaMemcpyHostToDevice, s));
        CUDA_TRY(cudaMemcpyAsync(e->F_in(), F, bytes, cudaMemcpyHostToDevice, s));
        Yd = e->Y_in();
        Fd = e->F_in();
    }
    TRY(e->dist_forward(Yd, Fd, s));
    return memory == FFCM_HOST ? finish(h, s) : FFCM_OK;
}

int ffcm_dist_stokes(ffcm_handle* h, void* stream) {
    g_err.clear();
    TRY(check_handle(h));
    if (!h->distributed) return fail(FFCM_ERR_STATE, "not a rank of a z-slab decomposition (ffcm_dist_create)");
    DeviceGuard g(h->device);
    return h->eng->dist_stokes(h->pick(stream));
}

int ffcm_dist_interpolate(ffcm_handle* h, void* stream) {
    g_err.clear();
    TRY(check_handle(h));
    if (!h->distributed) return fail(FFCM_ERR_STATE, "not a rank of a z-slab decomposition (ffcm_dist_create)");
    DeviceGuard g(h->device);
    return h->eng->dist_interp(h->pick(stream));
}

int ffcm_dist_correct(ffcm_handle* h, void* V, int32_t memory, void* stream) {
    g_err.clear();
    TRY(check_handle(h));
    if (!h->distributed) return fail(FFCM_ERR_STATE, "not a rank of a z-slab decomposition (ffcm_dist_create)");
    TRY(check_args(h->device, memory, {V}));
    if (!V) return fail(FFCM_ERR_ARGUMENT, "V must not be NULL");
    DeviceGuard g(h->device);
    cudaStream_t s = h->pick(stream);
    EngineBase* e = h->eng.get();
    if (memory == FFCM_DEVICE) return e->dist_correct(V, s);
    TRY(e->dist_correct(e->V_out(), s));
    {
        StageScope sc(h, FFCM_STAGE_D2H, s);
        CUDA_TRY(cudaMemcpyAsync(V, e->V_out(), 3 * (size_t)h->N * h->esize, cudaMemcpyDeviceToHost, s));
    }
    return finish(h, s);
}

int ffcm_destroy(ffcm_handle* h) {
    if (!h) return FFCM_OK;
    DeviceGuard g(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->side_stream) cudaStreamSynchronize(h->side_stream);
    cg_release(h);
    h->eng.reset();
    if (h->side_stream) cudaStreamDestroy(h->side_stream);
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_join) cudaEventDestroy(h->ev_join);
    for (cudaEvent_t e : h->ev_probe)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : h->events) cudaEventDestroy(e);
    if (h->copy_stream) {
        cudaStreamSynchronize(h->copy_stream);
        cudaStreamDestroy(h->copy_stream);
    }
    if (h->ev_ready) cudaEventDestroy(h->ev_ready);
    if (h->ev_forces) cudaEventDestroy(h->ev_forces);
    if (h->d_err) cudaFree(h->d_err);
    if (h->h_err) cudaFreeHost(h->h_err);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return FFCM_OK;
}

int ffcm_get_tuning(const ffcm_handle* h, int32_t* out) {
    TRY(check_handle(h));
    if (!out) return fail(FFCM_ERR_ARGUMENT, "out must not be NULL");
    h->eng->tuning(out);
    return FFCM_OK;
}

int64_t ffcm_wisdom_export(char* buf, int64_t cap) {
    std::string text;
    {
        std::lock_guard<std::mutex> lock(tune_mu());
        for (const auto& kv : tune_store()) {
            const TuneKey& k = kv.first;
            const TunedChoice& t = kv.second;
            char line[256];
            std::snprintf(line, sizeof line, "ffcm-wisdom-2 %d %d %d %d %d %d %d %d %d %d %d %d %d\n", k[0], k[1],
                          k[2], k[3], k[4], k[5], t.ykind, t.By, t.ygrid, t.zkind, t.Bz, t.zgrid, t.kx_chunk);
            text += line;
        }
    }
    if (buf && cap > 0) {
        const size_t n = std::min<size_t>(text.size(), (size_t)cap - 1);
        std::memcpy(buf, text.data(), n);
        buf[n] = '\0';
    }
    return (int64_t)text.size();
}

int ffcm_wisdom_import(const char* text) {
    g_err.clear();
    if (!text) return fail(FFCM_ERR_ARGUMENT, "text must not be NULL");
    std::vector<std::pair<TuneKey, TunedChoice>> parsed;
    const char* p = text;
    int lineno = 0;
    while (*p) {
        const char* e = std::strchr(p, '\n');
        const std::string line(p, e ? (size_t)(e - p) : std::strlen(p));
        p = e ? e + 1 : p + line.size();
        ++lineno;
        if (line.find_first_not_of(" \t\r") == std::string::npos) continue;   // blank line
        int v[13];
        char tag[32] = {0};
        int used = 0;
        const int got = std::sscanf(line.c_str(), "%31s %d %d %d %d %d %d %d %d %d %d %d %d %d %n", tag, &v[0],
                                    &v[1], &v[2], &v[3], &v[4], &v[5], &v[6], &v[7], &v[8], &v[9], &v[10], &v[11],
                                    &v[12], &used);
        if (got != 14 || std::strcmp(tag, "ffcm-wisdom-2") != 0 || used != (int)line.size())
            return fail(FFCM_ERR_ARGUMENT, "wisdom line " + std::to_string(lineno) + " is malformed");
        // grid sizes and SM counts far beyond any GPU are rejected here;
        // choice_valid bounds the grids again against the device in use
        const bool sane = v[0] >= 0 && (v[1] == 4 || v[1] == 8) && v[2] > 0 && v[3] > 0 && v[4] > 0 && v[5] > 0 &&
                          v[5] <= 4096 && v[6] >= 0 && v[7] > 0 && v[8] >= 0 && v[8] <= (1 << 18) && v[9] >= 0 &&
                          v[10] > 0 && v[11] >= 0 && v[11] <= (1 << 18) && v[12] >= 0;
        if (!sane) return fail(FFCM_ERR_ARGUMENT, "wisdom line " + std::to_string(lineno) + " is out of range");
        parsed.push_back({TuneKey{v[0], v[1], v[2], v[3], v[4], v[5]},
                          TunedChoice{v[6], v[7], v[8], v[9], v[10], v[11], v[12]}});
    }
    std::lock_guard<std::mutex> lock(tune_mu());
    for (const auto& kv : parsed) tune_store()[kv.first] = kv.second;
    return FFCM_OK;
}

int ffcm_set_stencil(ffcm_handle* h, int32_t mode) {
    g_err.clear();
    TRY(check_handle(h));
    if (mode != FFCM_STENCIL_REFERENCE && mode != FFCM_STENCIL_FLOAT64)
        return fail(FFCM_ERR_ARGUMENT, "mode must be FFCM_STENCIL_REFERENCE or FFCM_STENCIL_FLOAT64");
    if (mode == h->stencil) return FFCM_OK;
    DeviceGuard g(h->device);
    // work already queued keeps the mode it was launched with
    if (h->stream) CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->stencil = mode;
    h->eng->set_stencil(mode);
    // a checkpoint was made with the other weights, and the conjugate-gradient
    // graph holds the old kernel parameters: neither may be reused
    h->ckpt = false;
    cg_release(h);
    return FFCM_OK;
}

int ffcm_get_stencil(const ffcm_handle* h, int32_t* mode) {
    TRY(check_handle(h));
    if (!mode) return fail(FFCM_ERR_ARGUMENT, "mode must not be NULL");
    *mode = h->stencil;
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
    TRY(check_whole(h));
    h->ckpt = false;
    h->positions = false;
    TRY(check_args(h->device, memory, {V, Y, F}));
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
    if (memory == FFCM_HOST && e->uses_slab()) {
        // The positions go first; the forces follow on the copy stream
        // (after the positions' copy and so after the work queued on s before
        // it, which may still read the staging buffer) while the positions
        // are wrapped, sorted and listed per slab, which needs no forces; they
        // are gathered into cell order once they have landed.
        if (!h->copy_stream) {
            CUDA_TRY(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
            CUDA_TRY(cudaEventCreateWithFlags(&h->ev_ready, cudaEventDisableTiming));
            CUDA_TRY(cudaEventCreateWithFlags(&h->ev_forces, cudaEventDisableTiming));
        }
        {
            StageScope sc(h, FFCM_STAGE_H2D, s);
            CUDA_TRY(cudaMemcpyAsync(e->Y_in(), Y, bytes, cudaMemcpyHostToDevice, s));
            // after the positions' copy (the two would otherwise share the
            // link and the positions would land no sooner)
            CUDA_TRY(cudaEventRecord(h->ev_ready, s));
            CUDA_TRY(cudaStreamWaitEvent(h->copy_stream, h->ev_ready, 0));
            CUDA_TRY(cudaMemcpyAsync(e->F_in(), F, bytes, cudaMemcpyHostToDevice, h->copy_stream));
            CUDA_TRY(cudaEventRecord(h->ev_forces, h->copy_stream));
        }
        TRY(e->wrap_hash(e->Y_in(), true, true, s));
        TRY(e->sort(nullptr, s));
        e->lists_built = false;
        TRY(e->ensure_lists(s));
        CUDA_TRY(cudaStreamWaitEvent(s, h->ev_forces, 0));
        TRY(e->gather_forces(e->F_in(), s));
        TRY(e->mobility_rest_same_positions(e->V_out(), s));
        {
            StageScope sc(h, FFCM_STAGE_D2H, s);
            CUDA_TRY(cudaMemcpyAsync(V, e->V_out(), bytes, cudaMemcpyDeviceToHost, s));
        }
        return finish(h, s);
    }
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
    TRY(e->mobility_rest(Vd, s));
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
    TRY(check_whole(h));
    h->ckpt = false;
    h->positions = false;
    TRY(check_args(h->device, memory, {Y}));
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
    TRY(check_whole(h));
    h->ckpt = false;
    h->positions = false;
    DeviceGuard g(h->device);
    return h->eng->wrap_hash(nullptr, false, true, h->pick(stream));
}

int ffcm_sort_particles_by_cell(ffcm_handle* h, const void* F, int32_t memory, void* stream) {
    g_err.clear();
    TRY(check_whole(h));
    h->ckpt = false;
    h->positions = false;
    TRY(check_args(h->device, memory, {F}));
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
    TRY(check_whole(h));
    h->ckpt = false;
    h->positions = false;
    DeviceGuard g(h->device);
    return h->eng->spread(h->pick(stream));
}

int ffcm_stokes_solve(ffcm_handle* h, void* stream) {
    g_err.clear();
    TRY(check_whole(h));
    h->ckpt = false;
    h->positions = false;
    DeviceGuard g(h->device);
    return h->eng->stokes(h->pick(stream));
}

int ffcm_interpolate_velocities(ffcm_handle* h, void* V, int32_t memory, void* stream) {
    g_err.clear();
    TRY(check_whole(h));
    TRY(check_args(h->device, memory, {V}));
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
    TRY(check_whole(h));
    TRY(check_args(h->device, memory, {V}));
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

int ffcm_mobility_checkpoint(ffcm_handle* h, void* V, const void* Y, const void* F, int32_t memory,
                             void* stream) {
    g_err.clear();
    TRY(check_whole(h));
    TRY(check_args(h->device, memory, {V, Y, F}));
    h->ckpt = false;
    h->positions = false;
    if (!V || !Y || !F) return fail(FFCM_ERR_ARGUMENT, "V, Y and F must not be NULL");
    DeviceGuard g(h->device);
    cudaStream_t s = h->pick(stream);
    EngineBase* e = h->eng.get();
    TRY(e->ensure_adjoint());
    const size_t bytes = 3 * (size_t)h->N * h->esize;
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
    TRY(e->forward_checkpoint(Vd, s));
    h->ckpt = true;
    if (memory == FFCM_HOST) {
        {
            StageScope sc(h, FFCM_STAGE_D2H, s);
            CUDA_TRY(cudaMemcpyAsync(V, e->V_out(), bytes, cudaMemcpyDeviceToHost, s));
        }
        const int rc = finish(h, s);
        if (rc != FFCM_OK) h->ckpt = false;
        return rc;
    }
    return FFCM_OK;
}

int ffcm_adjoint(ffcm_handle* h, void* dJdY, void* dJdF, const void* lambda, int32_t memory, void* stream) {
    g_err.clear();
    TRY(check_whole(h));
    TRY(check_args(h->device, memory, {dJdY, dJdF, lambda}));
    if (!dJdY || !dJdF || !lambda) return fail(FFCM_ERR_ARGUMENT, "dJdY, dJdF and lambda must not be NULL");
    if (!h->ckpt)
        return fail(FFCM_ERR_STATE,
                    "ffcm_adjoint needs the state of a preceding ffcm_mobility_checkpoint on this handle, "
                    "with no other solve or step call in between");
    DeviceGuard g(h->device);
    cudaStream_t s = h->pick(stream);
    EngineBase* e = h->eng.get();
    const size_t bytes = 3 * (size_t)h->N * h->esize;
    if (memory == FFCM_DEVICE) return e->adjoint(lambda, dJdY, dJdF, s);
    {
        StageScope sc(h, FFCM_STAGE_H2D, s);
        CUDA_TRY(cudaMemcpyAsync(e->adj_buf(0), lambda, bytes, cudaMemcpyHostToDevice, s));
    }
    TRY(e->adjoint(e->adj_buf(0), e->adj_buf(1), e->adj_buf(2), s));
    {
        StageScope sc(h, FFCM_STAGE_D2H, s);
        CUDA_TRY(cudaMemcpyAsync(dJdY, e->adj_buf(1), bytes, cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaMemcpyAsync(dJdF, e->adj_buf(2), bytes, cudaMemcpyDeviceToHost, s));
    }
    return finish(h, s);
}

int ffcm_objective_gradient(ffcm_handle* h, double* J, void* dJdY, void* dJdF, void* V, const void* Y,
                            const void* F, const void* V_target, int32_t memory, void* stream) {
    g_err.clear();
    TRY(check_whole(h));
    TRY(check_args(h->device, memory, {J, dJdY, dJdF, V, Y, F, V_target}));
    h->ckpt = false;
    h->positions = false;
    if (!J || !dJdY || !dJdF || !V || !Y || !F || !V_target)
        return fail(FFCM_ERR_ARGUMENT, "no argument of ffcm_objective_gradient may be NULL");
    DeviceGuard g(h->device);
    cudaStream_t s = h->pick(stream);
    EngineBase* e = h->eng.get();
    TRY(e->ensure_adjoint());
    const size_t bytes = 3 * (size_t)h->N * h->esize;
    const void *Yd = Y, *Fd = F, *Td = V_target;
    void *Vd = V, *dYd = dJdY, *dFd = dJdF;
    double* Jdev = static_cast<double*>(e->adj_buf(4));
    if (memory == FFCM_HOST) {
        StageScope sc(h, FFCM_STAGE_H2D, s);
        CUDA_TRY(cudaMemcpyAsync(e->Y_in(), Y, bytes, cudaMemcpyHostToDevice, s));
        CUDA_TRY(cudaMemcpyAsync(e->F_in(), F, bytes, cudaMemcpyHostToDevice, s));
        CUDA_TRY(cudaMemcpyAsync(e->adj_buf(3), V_target, bytes, cudaMemcpyHostToDevice, s));
        Yd = e->Y_in();
        Fd = e->F_in();
        Td = e->adj_buf(3);
        Vd = e->V_out();
        dYd = e->adj_buf(1);
        dFd = e->adj_buf(2);
    }
    TRY(e->wrap_hash(Yd, true, true, s));
    TRY(e->sort(Fd, s));
    TRY(e->forward_checkpoint(Vd, s));
    TRY(e->residual(Vd, Td, e->adj_buf(0), Jdev, s));
    TRY(e->adjoint(e->adj_buf(0), dYd, dFd, s));
    h->ckpt = true;
    if (memory == FFCM_HOST) {
        {
            StageScope sc(h, FFCM_STAGE_D2H, s);
            CUDA_TRY(cudaMemcpyAsync(V, Vd, bytes, cudaMemcpyDeviceToHost, s));
            CUDA_TRY(cudaMemcpyAsync(dJdY, dYd, bytes, cudaMemcpyDeviceToHost, s));
            CUDA_TRY(cudaMemcpyAsync(dJdF, dFd, bytes, cudaMemcpyDeviceToHost, s));
            CUDA_TRY(cudaMemcpyAsync(J, Jdev, sizeof(double), cudaMemcpyDeviceToHost, s));
        }
        const int rc = finish(h, s);
        if (rc != FFCM_OK) h->ckpt = false;
        return rc;
    }
    CUDA_TRY(cudaMemcpyAsync(J, Jdev, sizeof(double), cudaMemcpyDeviceToDevice, s));
    return FFCM_OK;
}

int ffcm_set_positions(ffcm_handle* h, const void* Y, int32_t memory, void* stream) {
    g_err.clear();
    TRY(check_whole(h));
    TRY(check_args(h->device, memory, {Y}));
    h->ckpt = false;
    h->positions = false;
    if (!Y) return fail(FFCM_ERR_ARGUMENT, "Y must not be NULL");
    DeviceGuard g(h->device);
    cudaStream_t s = h->pick(stream);
    EngineBase* e = h->eng.get();
    const size_t bytes = 3 * (size_t)h->N * h->esize;
    const void* Yd = Y;
    if (memory == FFCM_HOST) {
        StageScope sc(h, FFCM_STAGE_H2D, s);
        CUDA_TRY(cudaMemcpyAsync(e->Y_in(), Y, bytes, cudaMemcpyHostToDevice, s));
        Yd = e->Y_in();
    }
    // the sort gathers some forces along; zeros stand in until the first apply
    CUDA_TRY(cudaMemsetAsync(e->F_in(), 0, bytes, s));
    TRY(e->wrap_hash(Yd, true, true, s));
    TRY(e->sort(e->F_in(), s));
    e->lists_built = false;
    if (memory == FFCM_HOST) TRY(finish(h, s));
    h->positions = true;
    return FFCM_OK;
}

int ffcm_mobility_apply(ffcm_handle* h, void* V, const void* F, int32_t memory, void* stream) {
    g_err.clear();
    TRY(check_whole(h));
    TRY(check_args(h->device, memory, {V, F}));
    if (!V || !F) return fail(FFCM_ERR_ARGUMENT, "V and F must not be NULL");
    if (!h->positions)
        return fail(FFCM_ERR_STATE,
                    "ffcm_mobility_apply needs the cell list of a preceding ffcm_set_positions on this handle, "
                    "with no other solve or step call in between");
    h->ckpt = false;
    DeviceGuard g(h->device);
    cudaStream_t s = h->pick(stream);
    EngineBase* e = h->eng.get();
    const size_t bytes = 3 * (size_t)h->N * h->esize;
    const void* Fd = F;
    void* Vd = V;
    if (memory == FFCM_HOST) {
        StageScope sc(h, FFCM_STAGE_H2D, s);
        CUDA_TRY(cudaMemcpyAsync(e->F_in(), F, bytes, cudaMemcpyHostToDevice, s));
        Fd = e->F_in();
        Vd = e->V_out();
    }
    TRY(e->apply_fixed(Vd, Fd, s));
    if (memory == FFCM_HOST) {
        {
            StageScope sc(h, FFCM_STAGE_D2H, s);
            CUDA_TRY(cudaMemcpyAsync(V, e->V_out(), bytes, cudaMemcpyDeviceToHost, s));
        }
        return finish(h, s);
    }
    return FFCM_OK;
}

int ffcm_cg_solve(ffcm_handle* h, void* F, const void* V, int32_t memory, double reltol, double abstol,
                  int32_t maxiter, int32_t flags, int32_t* iterations, double* residual, int32_t* cg_status,
                  void* stream) {
    g_err.clear();
    TRY(check_whole(h));
    TRY(check_args(h->device, memory, {F, V}));
    if (!F || !V) return fail(FFCM_ERR_ARGUMENT, "F and V must not be NULL");
    if (flags & ~FFCM_CG_INITIAL_GUESS) return fail(FFCM_ERR_ARGUMENT, "unknown flag bits");
    if (!(abstol >= 0) || std::isnan(reltol) || std::isinf(reltol) || std::isinf(abstol))
        return fail(FFCM_ERR_ARGUMENT, "abstol must be finite and non-negative, reltol finite");
    if (!h->positions)
        return fail(FFCM_ERR_STATE,
                    "ffcm_cg_solve needs the cell list of a preceding ffcm_set_positions on this handle, "
                    "with no other solve or step call in between");
    h->ckpt = false;
    DeviceGuard g(h->device);
    cudaStream_t s = h->pick(stream);
    EngineBase* e = h->eng.get();
    if (reltol < 0) reltol = h->dtype == FFCM_FLOAT32 ? std::sqrt((double)std::numeric_limits<float>::epsilon())
                                                      : std::sqrt(std::numeric_limits<double>::epsilon());
    if (maxiter < 0) maxiter = (int32_t)std::min<int64_t>(3 * h->N, INT32_MAX);
    TRY(e->ensure_lists(s));
    TRY(cg_prepare(h));
    auto& c = h->cg;
    const size_t bytes = 3 * (size_t)h->N * h->esize;
    const cudaMemcpyKind in = memory == FFCM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    const cudaMemcpyKind out = memory == FFCM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    const void* Vd = V;
    if (memory == FFCM_HOST) {
        StageScope sc(h, FFCM_STAGE_H2D, s);
        CUDA_TRY(cudaMemcpyAsync(e->V_out(), V, bytes, in, s));
        Vd = e->V_out();
    }
    const void* q = nullptr;
    if (flags & FFCM_CG_INITIAL_GUESS) {
        {
            StageScope sc(h, FFCM_STAGE_H2D, s);
            CUDA_TRY(cudaMemcpyAsync(c.x, F, bytes, in, s));
        }
        TRY(e->apply_fixed(c.q, c.x, s));
        q = c.q;
    } else {
        CUDA_TRY(cudaMemsetAsync(c.x, 0, bytes, s));
    }
    TRY(e->cg_start(Vd, q, c.r, c.p, c.st, reltol, abstol, maxiter, s));
    CUDA_TRY(cudaGraphLaunch(c.exec, s));
    {
        StageScope sc(h, FFCM_STAGE_D2H, s);
        CUDA_TRY(cudaMemcpyAsync(F, c.x, bytes, out, s));
    }
    CUDA_TRY(cudaMemcpyAsync(c.host, c.st, sizeof(CgState), cudaMemcpyDeviceToHost, s));
    TRY(finish(h, s));
    // kernels the graph ran: the gate plus one iteration body per iteration
    h->launches += 1 + (int64_t)c.host->iter * c.body_kernels;
    if (iterations) *iterations = c.host->iter;
    if (residual) *residual = std::sqrt(c.host->rr);
    if (cg_status) *cg_status = c.host->status;
    if (c.host->status == CG_DEVICE_ERROR)
        return fail(FFCM_ERR_CUDA, "a kernel of the mobility application raised its device error flag");
    return FFCM_OK;
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
        case FFCM_BUF_FORCE_DENSITY: TRY(e->ensure_real_grids()); TRY(copy(e->gf)); break;
        case FFCM_BUF_FLUID_VELOCITY: TRY(e->ensure_real_grids()); TRY(copy(e->gu)); break;
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
    TRY(check_whole(h));
    TRY(check_args(h->device, memory, {ext}));
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
    if (h) {   // the overwritten state no longer matches a checkpoint or cached cell list
        h->ckpt = false;
        h->positions = false;
    }
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

// ===========================================================================
// Batched form: many systems x many right-hand sides, one graph launch
// ===========================================================================
struct ffcm_batch {
    int32_t dtype = FFCM_FLOAT32, device = 0, nrhs = 1;
    int64_t nsys = 0, totalN = 0;
    size_t esize = 4;
    std::vector<ffcm_handle*> sys;
    std::vector<int64_t> N, yoff, fvoff;
    void* Yb = nullptr;
    void* Fb = nullptr;
    void* Vb = nullptr;
    cudaStream_t main = nullptr;
    std::vector<cudaStream_t> ws;
    std::vector<cudaEvent_t> ev;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t kernels = 0;
};

namespace {

void batch_release(ffcm_batch* b) {
    if (!b) return;
    DeviceGuard g(b->device);
    if (b->main) cudaStreamSynchronize(b->main);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (cudaEvent_t e : b->ev) cudaEventDestroy(e);
    for (cudaStream_t s : b->ws) cudaStreamDestroy(s);
    if (b->main) cudaStreamDestroy(b->main);
    if (b->Yb) cudaFree(b->Yb);
    if (b->Fb) cudaFree(b->Fb);
    if (b->Vb) cudaFree(b->Vb);
    for (ffcm_handle* h : b->sys) ffcm_destroy(h);
    delete b;
}

// Capture every system's pipeline (cell list once, then nrhs grid solves) as
// one dependency branch per system, forked from and joined into b->main.
int batch_build_graph(ffcm_batch* b) {
    const size_t es = b->esize;
    CUDA_TRY(cudaStreamBeginCapture(b->main, cudaStreamCaptureModeThreadLocal));
    int rc = FFCM_OK;
    cudaEvent_t fork = b->ev[0];
    rc = cudaEventRecord(fork, b->main) == cudaSuccess ? FFCM_OK : FFCM_ERR_CUDA;
    int64_t launches0 = 0;
    for (ffcm_handle* h : b->sys) launches0 += h->launches;
    for (int64_t i = 0; i < b->nsys && rc == FFCM_OK; ++i) {
        cudaStream_t s = b->ws[i];
        if (cudaStreamWaitEvent(s, fork, 0) != cudaSuccess) { rc = FFCM_ERR_CUDA; break; }
        EngineBase* e = b->sys[i]->eng.get();
        const char* Y = static_cast<const char*>(b->Yb) + 3 * b->yoff[i] * es;
        auto Fr = [&](int r) { return static_cast<const char*>(b->Fb) + (b->fvoff[i] + 3 * r * b->N[i]) * es; };
        auto Vr = [&](int r) { return static_cast<char*>(b->Vb) + (b->fvoff[i] + 3 * r * b->N[i]) * es; };
        rc = e->wrap_hash(Y, true, true, s);
        if (rc == FFCM_OK) rc = e->sort(Fr(0), s);
        if (rc == FFCM_OK) rc = e->mobility_rest(Vr(0), s);
        for (int r = 1; r < b->nrhs && rc == FFCM_OK; ++r) {
            rc = e->gather_forces(Fr(r), s);
            if (rc == FFCM_OK) rc = e->mobility_rest_same_positions(Vr(r), s);
        }
        if (rc == FFCM_OK && (cudaEventRecord(b->ev[1 + i], s) != cudaSuccess ||
                              cudaStreamWaitEvent(b->main, b->ev[1 + i], 0) != cudaSuccess))
            rc = FFCM_ERR_CUDA;
    }
    std::string msg = g_err;
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(b->main, &graph);
    if (rc != FFCM_OK) {
        if (graph) cudaGraphDestroy(graph);
        return fail(rc, "graph capture failed: " + msg);
    }
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
    b->graph = graph;
    CUDA_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
    int64_t launches1 = 0;
    for (ffcm_handle* h : b->sys) launches1 += h->launches;
    b->kernels = launches1 - launches0;
    return FFCM_OK;
}

}  // namespace

extern "C" {

int ffcm_batch_create(ffcm_batch** out, int32_t dtype, int64_t nsys, const double* L,
                      const double* R_c, const int64_t* N, double a, double ratio,
                      const int32_t* M, int32_t M_G, double mu, int32_t nrhs, int32_t device) {
    g_err.clear();
    if (!out) return fail(FFCM_ERR_ARGUMENT, "out must not be NULL");
    *out = nullptr;
    if (nsys < 1) return fail(FFCM_ERR_ARGUMENT, "a batch needs at least one system");
    if (nrhs < 1) return fail(FFCM_ERR_ARGUMENT, "nrhs must be at least 1");
    if (!L || !R_c || !N || !M) return fail(FFCM_ERR_ARGUMENT, "per-system arrays must not be NULL");
    for (int64_t i = 0; i < nsys; ++i) {
        const int r = ffcm_validate_config(dtype, L + 3 * i, R_c[i], N[i], a, ratio, M + 3 * i, M_G,
                                           mu, FFCM_FFT_ESTIMATE, 1);
        if (r != FFCM_OK) return fail(r, "system " + std::to_string(i) + ": " + g_err);
    }
    DeviceGuard g(device);
    if (!g.ok) return fail(FFCM_ERR_CUDA, "cudaSetDevice failed");
    auto* b = new ffcm_batch();
    b->dtype = dtype;
    b->device = device;
    b->nrhs = nrhs;
    b->nsys = nsys;
    b->esize = dtype == FFCM_FLOAT32 ? 4 : 8;
    auto bail = [&](int code) {
        const std::string msg = g_err;
        batch_release(b);
        return fail(code, msg);
    };
    int64_t acc = 0;
    for (int64_t i = 0; i < nsys; ++i) {
        ffcm_handle* h = nullptr;
        const int r = ffcm_create(&h, dtype, L + 3 * i, R_c[i], N[i], a, ratio, M + 3 * i, M_G, mu,
                                  FFCM_FFT_ESTIMATE, 1, device);
        if (r != FFCM_OK) return bail(r);
        b->sys.push_back(h);
        if (!h->eng->uses_slab()) {
            const int rr = h->eng->ensure_real_grids();   // before any capture
            if (rr != FFCM_OK) return bail(rr);
        }
        b->N.push_back(N[i]);
        b->yoff.push_back(acc);
        b->fvoff.push_back(3 * nrhs * acc);
        acc += N[i];
    }
    b->totalN = acc;
    const size_t ybytes = 3 * (size_t)acc * b->esize, fvbytes = (size_t)nrhs * ybytes;
    if (cudaMalloc(&b->Yb, ybytes) != cudaSuccess || cudaMalloc(&b->Fb, fvbytes) != cudaSuccess ||
        cudaMalloc(&b->Vb, fvbytes) != cudaSuccess) {
        fail(FFCM_ERR_OOM, "batch staging buffers");
        return bail(FFCM_ERR_OOM);
    }
    if (cudaStreamCreateWithFlags(&b->main, cudaStreamNonBlocking) != cudaSuccess) {
        fail(FFCM_ERR_CUDA, "stream creation");
        return bail(FFCM_ERR_CUDA);
    }
    b->ws.resize(nsys, nullptr);
    b->ev.resize(nsys + 1, nullptr);
    for (auto& s : b->ws)
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
            fail(FFCM_ERR_CUDA, "stream creation");
            return bail(FFCM_ERR_CUDA);
        }
    for (auto& e : b->ev)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
            fail(FFCM_ERR_CUDA, "event creation");
            return bail(FFCM_ERR_CUDA);
        }
    const int r = batch_build_graph(b);
    if (r != FFCM_OK) return bail(r);
    *out = b;
    return FFCM_OK;
}

int ffcm_batch_destroy(ffcm_batch* b) {
    batch_release(b);
    return FFCM_OK;
}

int ffcm_batch_get_info(const ffcm_batch* b, int64_t* total, int64_t* nsys, int32_t* nrhs,
                        int64_t* kernels) {
    if (!b) return fail(FFCM_ERR_STATE, "null batch");
    if (total) *total = b->totalN;
    if (nsys) *nsys = b->nsys;
    if (nrhs) *nrhs = b->nrhs;
    if (kernels) *kernels = b->kernels;
    return FFCM_OK;
}

int ffcm_batch_mobility(ffcm_batch* b, void* V, const void* Y, const void* F, int32_t memory,
                        void* stream) {
    g_err.clear();
    if (!b || !b->exec) return fail(FFCM_ERR_STATE, "null or unbuilt batch");
    TRY(check_args(b->device, memory, {V, Y, F}));
    if (!V || !Y || !F) return fail(FFCM_ERR_ARGUMENT, "V, Y and F must not be NULL");
    DeviceGuard g(b->device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : b->main;
    const size_t ybytes = 3 * (size_t)b->totalN * b->esize, fvbytes = (size_t)b->nrhs * ybytes;
    CUDA_TRY(cudaMemcpyAsync(b->Yb, Y, ybytes, kind_to_dev(memory), s));
    CUDA_TRY(cudaMemcpyAsync(b->Fb, F, fvbytes, kind_to_dev(memory), s));
    CUDA_TRY(cudaGraphLaunch(b->exec, s));
    for (ffcm_handle* h : b->sys) h->launches += b->kernels / std::max<int64_t>(1, b->nsys);
    CUDA_TRY(cudaMemcpyAsync(V, b->Vb, fvbytes, kind_from_dev(memory), s));
    if (memory != FFCM_HOST) return FFCM_OK;
    for (ffcm_handle* h : b->sys) TRY(finish(h, s));
    return FFCM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Cell-list sort with library-owned scratch (no allocation per call).
//
// ffcm_sort_cells_noalloc computes the reference's three cell-list buffers
// (original_index, cell_start, cell_end of src/cell_list.jl:64-93) from a
// caller's cell_hash array, using only memory the caller passes in plus a
// fixed scratch array that lives in this library's own device image. It never
// calls cudaMalloc or cudaFree, nor anything that allocates on its behalf.
//
// Who needs this: an ffcm_handle allocates all of its buffers when it is
// created, and holds them, which is right for repeated solves of one system.
// A caller that builds cell lists for many differently sized systems, or that
// runs under a fixed device-memory budget (a Julia or Python host that has
// handed its memory to its own pool allocator, or an application that keeps
// other streams busy and cannot afford the device-wide synchronisation that
// cudaFree, and sometimes cudaMalloc, performs) cannot create a handle per
// system. It can call this function with its own arrays instead.
//
// Limits and rules:
//   * at most FFCM_NOALLOC_MAX_CELLS cells (the scratch holds two int32 arrays
//     of that length plus the scan's tile sums, 16 MiB in total);
//   * the scratch is one array per device: calls that overlap in time on one
//     device (different streams, different host threads) race on it and must
//     be serialised by the caller;
//   * every call looks the scratch up with cudaGetSymbolAddress on the
//     current device; the first call on a device may load this library's
//     device code there, so make that first call before any stream capture
//     begins (a reset device reloads it on the next call);
//   * nothing needs to be zero beforehand: every call clears the counters it
//     uses and its range-check flag before counting;
//   * the call runs on the calling thread's current device, on `stream`, and
//     returns after the sort is complete (it reads back the range-check flag).
// ---------------------------------------------------------------------------

namespace {

constexpr int64_t kNoallocMaxCells = FFCM_NOALLOC_MAX_CELLS;
constexpr int64_t kNoallocMaxTiles = (kNoallocMaxCells + SCAN_TILE - 1) / SCAN_TILE;
// [0, C): per-cell counts, then per-cell cursors; [C, 2C+1): 0-based cell
// offsets; then the scan's tile sums; the last word is the range-check flag.
constexpr int64_t kNoallocScratchInts = 2 * kNoallocMaxCells + 1 + kNoallocMaxTiles + 1;

}  // namespace

static __device__ __align__(256) int32_t g_noalloc_scratch[kNoallocScratchInts];

namespace {

// The device address of the scratch array on the current device. It is looked
// up on every call, not cached: cudaGetSymbolAddress of an already loaded
// module is a table lookup with no device work, and a cached address would go
// stale if the caller reset the device (cudaDeviceReset unloads the module;
// the next lookup loads it again at a possibly different address).
int noalloc_scratch(int32_t** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(cell-sort scratch)");
    *out = static_cast<int32_t*>(p);
    return FFCM_OK;
}

// Zero a[0, n) and, when flag is given, the range-check flag.
__global__ void k_noalloc_zero(int32_t* __restrict__ a, int n, int32_t* __restrict__ flag) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = 0;
    if (flag && blockIdx.x == 0 && threadIdx.x == 0) *flag = 0;
}

// Histogram of the keys; a key outside [0, ncell) raises the flag and is skipped.
__global__ void k_noalloc_count(int n_part, const int32_t* __restrict__ key, int ncell,
                                int32_t* __restrict__ count, int32_t* __restrict__ flag) {
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < n_part; n += gridDim.x * blockDim.x) {
        const int c = key[n];
        if (c < 0 || c >= ncell) {
            atomicOr(flag, 1);
            continue;
        }
        atomicAdd(&count[c], 1);
    }
}

__global__ void k_noalloc_scatter(int n_part, const int32_t* __restrict__ key, int ncell,
                                  const int32_t* __restrict__ off, int32_t* __restrict__ cursor,
                                  int32_t* __restrict__ slot_of) {
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < n_part; n += gridDim.x * blockDim.x) {
        const int c = key[n];
        if (c < 0 || c >= ncell) continue;
        slot_of[off[c] + atomicAdd(&cursor[c], 1)] = n;
    }
}

// Cells of up to this many particles are put in order by one thread each
// (insertion sort); larger ones are listed for k_noalloc_sort_large.
constexpr int kNoallocSmallCell = 32;
// Cells up to this size are sorted by one block in shared memory.
constexpr int kNoallocBlockCell = 8192;

// Per cell: ascending original order (stability), 1-based indices, and the
// reference's 1-based inclusive ranges (an empty cell has start = end + 1).
// Crowded cells are appended to `large` (count in *nlarge) and finished by
// k_noalloc_sort_large, so no thread sorts more than kNoallocSmallCell values.
__global__ void k_noalloc_finish(int ncell, const int32_t* __restrict__ off, int32_t* __restrict__ idx,
                                 int32_t* __restrict__ cell_start, int32_t* __restrict__ cell_end,
                                 int32_t* __restrict__ large, int32_t* __restrict__ nlarge) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
        const int b = off[c], e = off[c + 1];
        cell_start[c] = b + 1;
        cell_end[c] = e;
        if (e - b > kNoallocSmallCell) {
            large[atomicAdd(nlarge, 1)] = c;
            continue;
        }
        for (int i = b + 1; i < e; ++i) {
            const int v = idx[i];
            int j = i - 1;
            while (j >= b && idx[j] > v) {
                idx[j + 1] = idx[j];
                --j;
            }
            idx[j + 1] = v;
        }
        for (int i = b; i < e; ++i) idx[i] += 1;
    }
}

// One block per crowded cell (grid-stride over the list): the cell's indices
// are staged in shared memory, each one's rank (the number of smaller ones,
// all distinct) is counted there, and the block writes them back in order,
// 1-based. A cell beyond kNoallocBlockCell is sorted by a single thread in
// place (a degenerate input: every particle in a handful of cells).
__global__ void k_noalloc_sort_large(const int32_t* __restrict__ off, int32_t* __restrict__ idx,
                                     const int32_t* __restrict__ large, const int32_t* __restrict__ nlarge) {
    __shared__ int32_t vals[kNoallocBlockCell];
    const int count = *nlarge;
    for (int q = blockIdx.x; q < count; q += gridDim.x) {
        const int c = large[q];
        const int b = off[c], n = off[c + 1] - b;
        if (n > kNoallocBlockCell) {
            if (threadIdx.x == 0) {
                for (int i = b + 1; i < b + n; ++i) {
                    const int v = idx[i];
                    int j = i - 1;
                    while (j >= b && idx[j] > v) {
                        idx[j + 1] = idx[j];
                        --j;
                    }
                    idx[j + 1] = v;
                }
                for (int i = b; i < b + n; ++i) idx[i] += 1;
            }
            __syncthreads();
            continue;
        }
        for (int i = threadIdx.x; i < n; i += blockDim.x) vals[i] = idx[b + i];
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const int v = vals[i];
            int rank = 0;
            for (int j = 0; j < n; ++j) rank += vals[j] < v ? 1 : 0;
            idx[b + rank] = v + 1;
        }
        __syncthreads();   // vals is reused by the next cell
    }
}

}  // namespace

extern "C" int ffcm_sort_cells_noalloc(const int32_t* cell_hash, int64_t N, int32_t ncell, int32_t* original_index,
                            int32_t* cell_start, int32_t* cell_end, void* stream) {
    g_err.clear();
    if (N < 0 || N > (int64_t)std::numeric_limits<int32_t>::max())
        return fail(FFCM_ERR_ARGUMENT, "N must be in [0, 2^31 - 1]; got " + std::to_string(N));
    if (ncell < 1 || ncell > kNoallocMaxCells)
        return fail(FFCM_ERR_ARGUMENT, "ncell must be in [1, " + std::to_string(kNoallocMaxCells) +
                                           "] (the fixed scratch size); got " + std::to_string(ncell));
    if ((N > 0 && (!cell_hash || !original_index)) || !cell_start || !cell_end)
        return fail(FFCM_ERR_ARGUMENT, "cell_hash, original_index, cell_start and cell_end must not be NULL");
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    TRY(check_device_ptrs(dev, {cell_hash, original_index, cell_start, cell_end}));
    int32_t* scratch = nullptr;
    TRY(noalloc_scratch(&scratch));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int n = (int)N;
    int32_t* cnt = scratch;
    int32_t* off = scratch + kNoallocMaxCells;
    int32_t* tiles = off + kNoallocMaxCells + 1;
    int32_t* flag = tiles + kNoallocMaxTiles;
    const int ntiles = (ncell + SCAN_TILE - 1) / SCAN_TILE;
    auto chk = [](const char* what) -> int {
        const cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? FFCM_OK : cuda_fail(e, what);
    };
    k_noalloc_zero<<<grid_for(ncell, 256), 256, 0, s>>>(cnt, ncell, flag);
    TRY(chk("k_noalloc_zero"));
    if (n > 0) {
        k_noalloc_count<<<grid_for(n, 256), 256, 0, s>>>(n, cell_hash, ncell, cnt, flag);
        TRY(chk("k_noalloc_count"));
    }
    k_scan_tiles<<<ntiles, SCAN_THREADS, 0, s>>>(cnt, ncell, tiles);
    TRY(chk("k_scan_tiles"));
    k_scan_tile_sums<<<1, 1024, 0, s>>>(tiles, ntiles);
    TRY(chk("k_scan_tile_sums"));
    k_scan_apply<<<ntiles, SCAN_THREADS, 0, s>>>(cnt, ncell, tiles, off);
    TRY(chk("k_scan_apply"));
    k_noalloc_zero<<<grid_for(ncell, 256), 256, 0, s>>>(cnt, ncell, nullptr);  // cursors; keep the flag
    TRY(chk("k_noalloc_zero"));
    if (n > 0) {
        k_noalloc_scatter<<<grid_for(n, 256), 256, 0, s>>>(n, cell_hash, ncell, off, cnt, original_index);
        TRY(chk("k_noalloc_scatter"));
    }
    // the cursors and the scan's tile sums are consumed: the cursor space
    // holds the list of crowded cells (fewer than ncell) and the first tile
    // sum its length
    int32_t* large = cnt;
    int32_t* nlarge = tiles;
    k_noalloc_zero<<<1, 32, 0, s>>>(nlarge, 1, nullptr);
    TRY(chk("k_noalloc_zero"));
    k_noalloc_finish<<<grid_for(ncell, 256), 256, 0, s>>>(ncell, off, original_index, cell_start, cell_end,
                                                           large, nlarge);
    TRY(chk("k_noalloc_finish"));
    k_noalloc_sort_large<<<148 * 2, 256, 0, s>>>(off, original_index, large, nlarge);
    TRY(chk("k_noalloc_sort_large"));
    int32_t bad = 0;
    CUDA_TRY(cudaMemcpyAsync(&bad, flag, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    if (bad) return fail(FFCM_ERR_ARGUMENT, "a cell_hash value lies outside [0, ncell)");
    return FFCM_OK;
}
