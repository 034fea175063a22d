// solver.cu — host driver and C ABI of the B200 LLG path.
//
// Engine<R> owns a set of films (one for llg_solver, many for llg_batch) and
// runs integrator attempts as sequences of field evaluations (three kernels
// each, one launch per pass over the work items of every film) followed by a
// one-thread-per-film FP64 step controller.  Every kernel reads its dynamic
// state (dt, buffer parity, activity, relax requests) from device memory, so
// an attempt — or a run of attempts, or relax iterations — is captured once as
// a CUDA graph and replayed without host round trips; films advance with their
// own dt and acceptance.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/llg_b200.h"
#include "build_api.h"
#include "field_kernels.cuh"
#include "relax_dev.cuh"
#include "minimize_dev.cuh"

namespace llg {

static thread_local std::string g_last_error;

static int set_error(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define CUDA_TRY(x)                                                                                      \
    do {                                                                                                 \
        cudaError_t _e = (x);                                                                            \
        if (_e != cudaSuccess) {                                                                         \
            return set_error(_e == cudaErrorMemoryAllocation ? LLG_ERR_OOM : LLG_ERR_CUDA, "%s: %s (%s:%d)", \
                             #x, cudaGetErrorString(_e), __FILE__, __LINE__);                            \
        }                                                                                                \
    } while (0)

// Butcher tableaux (llg.rs:813-846, 296-309).
namespace dp5 {
constexpr double A21 = 1.0 / 5.0;
constexpr double A31 = 3.0 / 40.0, A32 = 9.0 / 40.0;
constexpr double A41 = 44.0 / 45.0, A42 = -56.0 / 15.0, A43 = 32.0 / 9.0;
constexpr double A51 = 19372.0 / 6561.0, A52 = -25360.0 / 2187.0, A53 = 64448.0 / 6561.0, A54 = -212.0 / 729.0;
constexpr double A61 = 9017.0 / 3168.0, A62 = -355.0 / 33.0, A63 = 46732.0 / 5247.0, A64 = 49.0 / 176.0,
                 A65 = -5103.0 / 18656.0;
constexpr double B1 = 35.0 / 384.0, B3 = 500.0 / 1113.0, B4 = 125.0 / 192.0, B5 = -2187.0 / 6784.0, B6 = 11.0 / 84.0;
constexpr double BH1 = 5179.0 / 57600.0, BH3 = 7571.0 / 16695.0, BH4 = 393.0 / 640.0, BH5 = -92097.0 / 339200.0,
                 BH6 = 187.0 / 2100.0, BH7 = 1.0 / 40.0;
}  // namespace dp5
namespace bs3 {
constexpr double A21 = 1.0 / 2.0, A32 = 3.0 / 4.0;
constexpr double B1 = 2.0 / 9.0, B2 = 1.0 / 3.0, B3 = 4.0 / 9.0;
constexpr double BH1 = 7.0 / 24.0, BH2 = 1.0 / 4.0, BH3 = 1.0 / 3.0, BH4 = 1.0 / 8.0;
}  // namespace bs3

enum { KIND_RK45 = 1, KIND_RK23 = 2, KIND_RELAX = 3, KIND_MINIMIZE = 4 };

// Shared controller settings; per-film dt and FSAL invalidation come as FilmCtl.
struct Control {
    double t_end, max_err, headroom, dt_min, dt_max;
    long long target_acc, attempts;
    int reset_time;
};
struct FilmCtl {
    double dt;
    int invalidate_fsal;
    int keep_dt;  // 1: leave StepState::dt as it is
};

// ---------------------------------------------------------------------------
// small kernels (one thread per film unless noted)
// ---------------------------------------------------------------------------
__global__ void k_set_control(FilmDev* films, int nfilms, Control c, const FilmCtl* __restrict__ fc) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nfilms) return;
    StepState* st = films[f].st;
    if (!fc[f].keep_dt) st->dt = fc[f].dt;
    st->t_end = c.t_end;
    st->max_err = c.max_err;
    st->headroom = c.headroom;
    st->dt_min = c.dt_min;
    st->dt_max = c.dt_max;
    st->target_acc = c.target_acc >= 0 ? st->n_acc + c.target_acc : -1;
    st->attempts_left = c.attempts;
    st->active = 1;
    st->err_code = 0;
    st->err_bits = 0ull;
    st->req = REQ_NONE;
    if (fc[f].invalidate_fsal) st->fsal_valid = 0;
    if (c.reset_time) st->t = 0.0;
    if (isfinite(c.t_end)) {
        double rem = c.t_end - st->t;
        if (st->dt > rem) st->dt = rem;
        if (!(st->t + 1e-18 < c.t_end)) st->active = 0;
    }
}

// Step-size controller (llg.rs:997-1025 for order 5, llg.rs:401-435 for order 3).
__global__ void k_controller(FilmDev* films, int nfilms, int order, int req) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nfilms) return;
    StepState* st = films[f].st;
    if (!st->active) return;
    if (req && st->req != req) return;
    const unsigned long long bits = st->err_bits;
    st->err_bits = 0ull;
    const double err = __longlong_as_double((long long)bits);
    const double dt0 = st->dt;
    const double eps = order == 5 ? err * dt0 : err;
    st->eps = eps;
    st->dt_used = dt0;
    if (!(eps == eps) || isinf(eps)) {
        st->err_code = LLG_ERR_NONFINITE;
        st->accepted = 0;
        st->fsal_valid = 0;
        st->active = 0;
        return;
    }
    double dt_next = eps > 0.0 ? dt0 * st->headroom * pow(st->max_err / eps, order == 5 ? 0.2 : 1.0 / 3.0) : dt0 * 2.0;
    dt_next = fmin(fmax(dt_next, st->dt_min), st->dt_max);
    const bool acc = (eps <= st->max_err) || (dt0 <= st->dt_min * 1.0000000001);
    if (acc) {
        st->cur ^= 1;
        st->fsal_valid = 1;
        st->n_acc += 1;
        st->t += dt0;
    } else {
        // RK45: k1 of the unchanged state stays valid (its buffer is not written by
        // the rejected attempt, and the run / step calls evaluate it before their
        // first attempt); RK23 re-evaluates it, as the relax loop expects
        st->fsal_valid = order == 5 ? 1 : 0;
        st->n_rej += 1;
    }
    st->accepted = acc ? 1 : 0;
    st->dt = dt_next;
    if (st->attempts_left > 0) st->attempts_left -= 1;
    bool stop = st->attempts_left == 0 || (st->target_acc >= 0 && st->n_acc >= st->target_acc);
    if (isfinite(st->t_end)) {
        double rem = st->t_end - st->t;
        if (!(st->t + 1e-18 < st->t_end)) stop = true;
        else if (st->dt > rem) st->dt = rem;
    }
    if (stop) st->active = 0;
}

// Sum the per-block partial reductions of each film in block order (deterministic).
// One warp per film: lane l sums blocks l, l + 32, ... in order, then a fixed
// butterfly combines the lanes (deterministic; the loads of the 32 lanes overlap).
constexpr int kFinalizeFilmsPerBlock = 4;
__global__ void k_finalize(FilmDev* films, int nfilms, int req) {
    const int f = blockIdx.x * kFinalizeFilmsPerBlock + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (f >= nfilms) return;   // uniform over the warp
    const FilmDev& F = films[f];
    if (req && (!F.st->active || F.st->req != req)) return;
    double acc[RED_NSLOT];
#pragma unroll
    for (int s = 0; s < RED_NSLOT; ++s) acc[s] = 0.0;
    for (int b = lane; b < F.nblk; b += 32) {
        const double* p = F.red_part + (size_t)b * RED_NSLOT;
#pragma unroll
        for (int s = 0; s < RED_NSLOT; ++s) acc[s] = (s == RED_TMAX) ? fmax(acc[s], p[s]) : acc[s] + p[s];
    }
#pragma unroll
    for (int s = 0; s < RED_NSLOT; ++s)
        for (int o = 16; o > 0; o >>= 1) {
            const double w = __shfl_xor_sync(0xffffffffu, acc[s], o);
            acc[s] = (s == RED_TMAX) ? fmax(acc[s], w) : acc[s] + w;
        }
    if (lane == 0)
        for (int s = 0; s < RED_NSLOT; ++s) F.st->red[s] = acc[s];
}

// <m> partial sums per row block of every film.
template <typename R>
__global__ void k_mean_m(const FilmDev* films, const WorkItem* __restrict__ items, int nitems) {
    __shared__ double sm_red[32 * RED_NSLOT];
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const WorkItem w = items[it];
        const FilmDev& F = films[w.film];
        const int nx = F.nx, ny = F.ny, n = nx * ny, T = F.rows_per_block;
        const R* m = mbuf<R>(F, MB_M0, F.st->cur);
        double red[RED_NSLOT];
        for (int s = 0; s < RED_NSLOT; ++s) red[s] = 0.0;
        for (int e = threadIdx.x; e < T * nx; e += blockDim.x) {
            int j = w.blk * T + e / nx, i = e % nx;
            if (j >= ny) continue;
            int idx = j * nx + i;
            red[RED_MX] += (double)m[idx];
            red[RED_MY] += (double)m[n + idx];
            red[RED_MZ] += (double)m[2 * n + idx];
        }
        block_reduce(red, sm_red);
        if (threadIdx.x == 0)
            for (int s = 0; s < RED_NSLOT; ++s) F.red_part[(size_t)w.blk * RED_NSLOT + s] = red[s];
        __syncthreads();
    }
}

__device__ __forceinline__ bool same_bits(float a, float b) { return __float_as_uint(a) == __float_as_uint(b); }
__device__ __forceinline__ bool same_bits(double a, double b) {
    return __double_as_longlong(a) == __double_as_longlong(b);
}

// Uploaded AoS f64 state -> resident SoA planes.  The FSAL torque of the resident
// state stays valid when the upload equals that state bit for bit (a caller that
// passes back the state it just read, as a per-step host binding does); any
// difference drops it (every thread that sees one writes the same 0).
template <typename R>
__global__ void k_aos_to_soa(const FilmDev* films, int film, const double* __restrict__ src) {
    const FilmDev& F = films[film];
    const int n = F.nx * F.ny;
    R* dst = mbuf<R>(F, MB_M0, F.st->cur);
    bool changed = false;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const R v = (R)src[idx * 3 + c];
            changed |= !same_bits(v, dst[c * n + idx]);
            dst[c * n + idx] = v;
        }
    }
    if (__syncthreads_or(changed) && threadIdx.x == 0) F.st->fsal_valid = 0;
}

// The resident m as AoS f32 (the OVF binary4 payload), rounded to nearest.
template <typename R>
__global__ void k_soa_to_aos_f32(const FilmDev* films, int film, float* __restrict__ dst) {
    const FilmDev& F = films[film];
    const int n = F.nx * F.ny;
    const R* src = mbuf<R>(F, MB_M0, F.st->cur);
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
        dst[idx * 3 + 0] = (float)src[idx];
        dst[idx * 3 + 1] = (float)src[n + idx];
        dst[idx * 3 + 2] = (float)src[2 * n + idx];
    }
}

template <typename R>
__global__ void k_soa_to_aos(const FilmDev* films, int film, int which, double* __restrict__ dst) {
    const FilmDev& F = films[film];
    const int n = F.nx * F.ny;
    const R* src = which == 0 ? mbuf<R>(F, MB_M0, F.st->cur) : reinterpret_cast<const R*>(F.bout);
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
        dst[idx * 3 + 0] = (double)src[idx];
        dst[idx * 3 + 1] = (double)src[n + idx];
        dst[idx * 3 + 2] = (double)src[2 * n + idx];
    }
}

// ---------------------------------------------------------------------------
// Engine
// ---------------------------------------------------------------------------
struct EngineBase {
    virtual ~EngineBase() {}
    virtual int nfilms() const = 0;
    virtual int64_t cells(int f) const = 0;
    virtual int set_stream(cudaStream_t s) = 0;
    virtual int sync() = 0;
    virtual int set_state(int f, const double* m) = 0;
    virtual int get_state(int f, double* m) = 0;
    virtual int write_ovf(int f, const char* path, const llg_ovf_meta* meta, int format) = 0;
    virtual int mean_m(double* out3n) = 0;
    virtual int build_h_eff(int f, const llg_params* p, int fmask, double* b) = 0;
    virtual int demag_field(int f, double* b) = 0;
    virtual int step(int kind, llg_params* p, int fmask, double max_err, double headroom, double dt_min,
                     double dt_max, double* eps, int32_t* acc, double* dtu) = 0;
    virtual int run(int kind, llg_params* p, int fmask, double max_err, double headroom, double dt_min, double dt_max,
                    int64_t n_acc, double t_end, int64_t max_attempts, int64_t* acc_out, int64_t* rej_out,
                    double* t_adv) = 0;
    virtual int relax(llg_params* p, int fmask, const llg_relax_settings* st, llg_relax_report* rep) = 0;
    virtual int minimize(const llg_params* p, int fmask, const llg_minimize_settings* st,
                         llg_minimize_report* rep) = 0;
    virtual int energy(const double* bext3n, llg_energy_breakdown* out) = 0;
    virtual int torque_metric(const llg_params* p, int fmask, int metric, double* out) = 0;
    virtual int kernel_kspace(int f, double* out) = 0;
    virtual int profile_stage(const llg_params* p, int fmask, int reps, double* ms4) = 0;
    virtual long long launch_count() = 0;
    virtual int warm_start(ws::Net* net, const double* bext3n) = 0;
    virtual int fft_plans(int* rows, int nr, int* cols, int nc) const = 0;
};

// LLG_B200_GENERIC_FFT=1 selects the generic shared-memory Stockham kernels
// even where a register-FFT kernel exists (used to cross-check the two paths).
static bool env_flag(const char* name) {
    const char* e = std::getenv(name);
    return e && e[0] == '1';
}
static bool force_generic() { return env_flag("LLG_B200_GENERIC_FFT"); }
static int env_int(const char* name, int dflt) {
    const char* e = std::getenv(name);
    if (!e || !e[0]) return dflt;
    char* end = nullptr;
    const long v = std::strtol(e, &end, 10);
    return (end && *end == 0) ? (int)v : dflt;
}

// A row radix plan is usable in a segment if it exists and keeps the rows per
// block of plan 0 (the row work items are shared by the plans).
static bool row_plan_ok(const FastCfg& fc, int v) { return fc.ok_row[v] && fc.T[v] == fc.T[0]; }

// Radix plan chosen per (precision, pass kind, length) for the process.
static std::mutex g_plan_mutex;
static std::map<std::tuple<int, int, int>, int> g_plan_cache;

// LLG_B200_FFT_PLAN=0 or 1 fixes the register-FFT radix plan where it exists
// (-1: the autotuner decides).
static int forced_plan() {
    const char* e = std::getenv("LLG_B200_FFT_PLAN");
    if (e && (e[0] == '0' || e[0] == '1') && e[1] == 0) return e[0] - '0';
    return -1;
}

template <typename R>
struct Engine final : EngineBase {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    int nf = 0;
    std::vector<llg_grid> grids;
    std::vector<llg_material> mats;
    std::vector<FilmDev> fh;           // host mirror of the device descriptors
    FilmDev* d_films = nullptr;
    StepState* d_states = nullptr;
    StepState* h_states = nullptr;     // pinned
    RelaxStateDev* d_relax = nullptr;
    RelaxStateDev* h_relax = nullptr;  // pinned
    MinimizeStateDev* d_min = nullptr;
    MinimizeStateDev* h_min = nullptr; // pinned
    FilmCtl* d_ctl = nullptr;
    FilmCtl* h_ctl = nullptr;          // pinned
    WorkItem* d_row_items = nullptr;
    WorkItem* d_col_items = nullptr;
    LaunchGeom geom{};
    double* d_stage = nullptr;         // AoS FP64 staging (largest film)
    int64_t max_cells = 0;
    bool any_demag = false;
    std::vector<double*> d_k64;        // FP64 kernel planes per film (nullptr without demag)
    std::vector<void*> allocs;
    // host-side FSAL bookkeeping: the FSAL torque belongs to the last kind / mask / b_ext stepped
    int fsal_kind = 0;
    int fsal_mask = -1;
    std::vector<double> fsal_bext;
    std::map<long long, cudaGraphExec_t> graphs;
    std::map<long long, cudaGraph_t> graph_defs;
    std::map<long long, long long> graph_kernels;  // kernel nodes per graph
    long long launches = 0;                         // kernels issued so far
    bool l2_window = false;
    cudaStreamAttrValue l2_attr{};
    RelaxSettingsDev relax_graph_settings{};
    MinimizeSettingsDev minimize_graph_settings{};
    // launch segments: films grouped by the row (rseg) / column (cseg) kernel they use,
    // with the resident blocks per SM of each segment's kernels
    std::vector<LaunchGeom> rseg, cseg;
    // each segment's geometry under radix plan 0 / 1 (where the plan exists) and
    // the resident blocks per SM of its kernels; the autotuner picks one
    // (a column segment has 4 forms: 2 * plan + lean)
    std::vector<std::array<LaunchGeom, 2>> rseg_alt;
    std::vector<std::array<LaunchGeom, 4>> cseg_alt;
    std::vector<std::array<char, 2>> rseg_has;
    std::vector<std::array<char, 4>> cseg_has;
    std::vector<std::array<std::array<int, 4>, 2>> rocc;
    std::vector<std::vector<int>> rseg_films, cseg_films;   // films of each segment
    std::vector<std::array<int, 4>> cocc;

    int nfilms() const override { return nf; }
    int64_t cells(int f) const override { return grids[f].nx * grids[f].ny; }

    ~Engine() override {
        if (stream) cudaStreamSynchronize(stream);
        for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
        for (auto& kv : graph_defs) cudaGraphDestroy(kv.second);
        for (void* p : allocs) cudaFree(p);
        if (h_states) cudaFreeHost(h_states);
        if (h_relax) cudaFreeHost(h_relax);
        if (h_min) cudaFreeHost(h_min);
        if (h_ctl) cudaFreeHost(h_ctl);
        if (own_stream) cudaStreamDestroy(own_stream);
    }

    template <typename T>
    int dalloc(T** p, size_t bytes) {
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, bytes ? bytes : 16);
        if (e != cudaSuccess) return set_error(LLG_ERR_OOM, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
        allocs.push_back(q);
        *p = reinterpret_cast<T*>(q);
        return LLG_OK;
    }

    // One evaluation: row forward, column (with demag), row inverse, one launch per segment.
    int eval(const EvalSpec& e) {
        int nk = 0;
        for (auto& sg : rseg) CUDA_TRY(launch_one<R>(0, e, sg, stream, &nk));
        if (e.demag && geom.any_demag)
            for (auto& sg : cseg) CUDA_TRY(launch_one<R>(1, e, sg, stream, &nk));
        for (auto& sg : rseg) CUDA_TRY(launch_one<R>(2, e, sg, stream, &nk));
        launches += nk;
        return LLG_OK;
    }

    // The stages of one attempt in order.  Where a segment allows it (register-FFT
    // rows, a lean stage followed by a combination that ends with its torque),
    // stage i's row inverse and stage i+1's row forward run as one fused row pass.
    int eval_chain(const std::vector<EvalSpec>& v) {
        int nk = 0;
        const int n = (int)v.size();
        std::vector<char> fwd_done(rseg.size(), 0);
        for (int i = 0; i < n; ++i) {
            const EvalSpec& e = v[i];
            for (size_t q = 0; q < rseg.size(); ++q)
                if (!fwd_done[q]) CUDA_TRY(launch_one<R>(0, e, rseg[q], stream, &nk));
            if (e.demag && geom.any_demag)
                for (auto& sg : cseg) CUDA_TRY(launch_one<R>(1, e, sg, stream, &nk));
            for (size_t q = 0; q < rseg.size(); ++q) {
                if (i + 1 < n && can_fuse(e, v[i + 1], rseg[q])) {
                    CUDA_TRY(launch_fused<R>(e, v[i + 1], rseg[q], stream, &nk));
                    fwd_done[q] = 1;
                } else {
                    CUDA_TRY(launch_one<R>(2, e, rseg[q], stream, &nk));
                    fwd_done[q] = 0;
                }
            }
        }
        launches += nk;
        return LLG_OK;
    }

    int init(int dev, int n_films, const llg_grid* g, const llg_material* m, const uint8_t* const* masks) {
        device = dev;
        nf = n_films;
        grids.assign(g, g + nf);
        mats.assign(m, m + nf);
        fh.assign(nf, FilmDev{});
        d_k64.assign(nf, nullptr);
        fsal_bext.assign(3 * (size_t)nf, 0.0);
        CUDA_TRY(cudaSetDevice(dev));
        CUDA_TRY(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking));
        stream = own_stream;
        CUDA_TRY(cudaMallocHost(&h_states, sizeof(StepState) * nf));
        CUDA_TRY(cudaMallocHost(&h_relax, sizeof(RelaxStateDev) * nf));
        CUDA_TRY(cudaMallocHost(&h_min, sizeof(MinimizeStateDev) * nf));
        CUDA_TRY(cudaMallocHost(&h_ctl, sizeof(FilmCtl) * nf));
        // kernel choice per film and pass: register-FFT row kernels where nx has one,
        // register-FFT column kernel where ny has one; the generic kernels otherwise.
        // Films are grouped into launch segments by that choice (one launch per segment
        // and pass), so a mixed batch still runs its power-of-two films on the fast path.
        for (int f = 0; f < nf; ++f) any_demag |= m[f].demag != 0;
        const bool gen = force_generic();
        std::vector<FastCfg> fcs(nf);
        std::vector<char> frow(nf), fcol(nf);
        for (int f = 0; f < nf; ++f) {
            fcs[f] = fast_config<R>((int)g[f].nx, (int)g[f].ny);
            frow[f] = !gen && fcs[f].ok_row[0];
            fcol[f] = !gen && fcs[f].ok_col[0];
        }
        size_t smem_row = 0, smem_col = 0;   // generic kernels
        for (int f = 0; f < nf; ++f) {
            if (!m[f].demag) continue;
            if (!frow[f]) smem_row = std::max(smem_row, 4 * (size_t)3 * g[f].nx * sizeof(cx<R>));
            if (!fcol[f]) smem_col = std::max(smem_col, 12 * (size_t)g[f].ny * sizeof(cx<R>));
        }
        const size_t smem_max = 227 * 1024;
        if (smem_row > smem_max || smem_col > smem_max)
            return set_error(LLG_ERR_INVALID, "a film exceeds the in-shared-memory FFT limit for this precision");
        int rc;
        if ((rc = dalloc(&d_states, sizeof(StepState) * nf))) return rc;
        CUDA_TRY(cudaMemsetAsync(d_states, 0, sizeof(StepState) * nf, stream));
        if ((rc = dalloc(&d_relax, sizeof(RelaxStateDev) * nf))) return rc;
        if ((rc = dalloc(&d_min, sizeof(MinimizeStateDev) * nf))) return rc;
        if ((rc = dalloc(&d_ctl, sizeof(FilmCtl) * nf))) return rc;
        std::map<int, std::vector<WorkItem>> rows_by, cols_by;   // segment key: L of the fast kernel, 0 generic
        for (int f = 0; f < nf; ++f) {
            const int nx = (int)g[f].nx, ny = (int)g[f].ny;
            const int T = frow[f] ? fcs[f].T[0] : 2;
            const int64_t n = (int64_t)nx * ny;
            max_cells = std::max(max_cells, n);
            const size_t plane = sizeof(R) * 3 * (size_t)n;
            FilmDev& F = fh[f];
            F.nx = nx;
            F.ny = ny;
            F.rows_per_block = T;
            F.nblk = (ny + T - 1) / T;
            F.dx = g[f].dx;
            F.dy = g[f].dy;
            F.dz = g[f].dz;
            F.ms = m[f].ms;
            F.a_ex = m[f].a_ex;
            F.k_u = m[f].k_u;
            F.dmi = m[f].has_dmi ? m[f].dmi : 0.0;
            F.exch = (m[f].a_ex != 0.0 && m[f].ms != 0.0) ? 2.0 * m[f].a_ex / m[f].ms : 0.0;
            F.has_eta = (m[f].has_dmi && m[f].dmi != 0.0) ? 1 : 0;
            F.eta = (F.has_eta && m[f].a_ex != 0.0) ? m[f].dmi / (2.0 * m[f].a_ex) : 0.0;
            F.dmi_avail = (m[f].has_dmi && m[f].dmi != 0.0 && m[f].ms != 0.0 && m[f].a_ex != 0.0) ? 1 : 0;
            F.dmi_pref = F.dmi_avail ? 2.0 * m[f].dmi / m[f].ms : 0.0;
            F.anis = (m[f].k_u != 0.0 && m[f].ms != 0.0) ? 2.0 * m[f].k_u / m[f].ms : 0.0;
            F.inv_dx2 = 1.0 / (g[f].dx * g[f].dx);
            F.inv_dy2 = 1.0 / (g[f].dy * g[f].dy);
            F.half_inv_dx = 0.5 / g[f].dx;
            F.half_inv_dy = 0.5 / g[f].dy;
            for (int c = 0; c < 3; ++c) F.u[c] = m[f].easy_axis[c];
            F.demag_mat = m[f].demag ? 1 : 0;
            F.plan_row = make_plan(nx);
            F.plan_col = make_plan(ny);
            for (int b = 0; b < 2; ++b) {
                if ((rc = dalloc(&F.m[b], plane))) return rc;
                if ((rc = dalloc(&F.ms_buf[b], plane))) return rc;
                CUDA_TRY(cudaMemsetAsync(F.m[b], 0, plane, stream));
                CUDA_TRY(cudaMemsetAsync(F.ms_buf[b], 0, plane, stream));
            }
            for (int q = 1; q <= 7; ++q) {
                if ((rc = dalloc(&F.k[q], plane))) return rc;
                CUDA_TRY(cudaMemsetAsync(F.k[q], 0, plane, stream));
            }
            if ((rc = dalloc(&F.red_part, sizeof(double) * RED_NSLOT * (size_t)F.nblk))) return rc;
            F.st = d_states + f;
            if (masks && masks[f]) {
                uint8_t* dm = nullptr;
                if ((rc = dalloc(&dm, (size_t)n))) return rc;
                std::vector<uint8_t> norm((size_t)n);
                for (int64_t i = 0; i < n; ++i) norm[i] = masks[f][i] ? 1 : 0;
                CUDA_TRY(cudaMemcpyAsync(dm, norm.data(), (size_t)n, cudaMemcpyHostToDevice, stream));
                CUDA_TRY(cudaStreamSynchronize(stream));
                F.mask = dm;
                F.has_mask = 1;
            }
            if (m[f].demag) {
                void* tw_row;
                void* tw_col;
                if ((rc = dalloc(&tw_row, sizeof(cx<R>) * 2 * (size_t)nx))) return rc;
                if ((rc = dalloc(&tw_col, sizeof(cx<R>) * 2 * (size_t)ny))) return rc;
                CUDA_TRY(launch_twiddles(tw_row, 2 * nx, sizeof(R) == 8, stream));
                CUDA_TRY(launch_twiddles(tw_col, 2 * ny, sizeof(R) == 8, stream));
                F.tw_row = tw_row;
                F.tw_col = tw_col;
                // register-FFT pass tables of every radix plan the film's lengths have
                const FastCfg& fc = fcs[f];
                for (int v = 0; v < 2; ++v) {
                    if (frow[f] && row_plan_ok(fc, v)) {
                        void* t;
                        if ((rc = dalloc(&t, sizeof(cx<R>) * (size_t)std::max(fc.twp_row_size[v], 1)))) return rc;
                        CUDA_TRY(build_pass_tables<R>(t, nx, v, stream));
                        F.twp_row[v] = t;
                    }
                    if (fcol[f] && fc.ok_col[v]) {
                        void* t;
                        if ((rc = dalloc(&t, sizeof(cx<R>) * (size_t)std::max(fc.twp_col_size[v], 1)))) return rc;
                        CUDA_TRY(build_pass_tables<R>(t, ny, v, stream));
                        F.twp_col[v] = t;
                    }
                }
                if ((rc = dalloc(&F.X, sizeof(cx<R>) * 3 * (size_t)(nx + 1) * ny))) return rc;
                if (frow[f] && (rc = dalloc(&F.bdem, plane))) return rc;
                // films sharing a grid share the kernel planes (get_demag_operator, demag_fft_uniform.rs:86)
                int same = -1;
                for (int e = 0; e < f && same < 0; ++e)
                    if (mats[e].demag && grids[e].nx == nx && grids[e].ny == ny && grids[e].dx == g[f].dx &&
                        grids[e].dy == g[f].dy && grids[e].dz == g[f].dz)
                        same = e;
                if (same >= 0) {
                    F.Khat = fh[same].Khat;
                    d_k64[f] = d_k64[same];
                } else {
                    void* kh;
                    if ((rc = dalloc(&kh, sizeof(r4<R>) * (size_t)(nx + 1) * (ny + 1)))) return rc;
                    F.Khat = kh;
                    if ((rc = dalloc(&d_k64[f], sizeof(double) * 4 * (size_t)(nx + 1) * (ny + 1)))) return rc;
                    // the register-FFT column pass reads parity-split columns
                    CUDA_TRY(build_demag_kernel(nx, ny, g[f].dx, g[f].dy, g[f].dz, sizeof(R) == 8, kh, d_k64[f],
                                                stream, fcol[f] != 0));
                }
            }
            for (int b = 0; b < F.nblk; ++b) rows_by[frow[f] ? nx : 0].push_back(WorkItem{f, b});
            // column items per radix plan (a plan fixes the columns per item)
            if (m[f].demag)
                for (int v = 0; v < 2; ++v) {
                    if (fcol[f] ? !fcs[f].ok_col[v] : v > 0) continue;
                    const int NC = fcol[f] ? fcs[f].NC[v] : 1;
                    const int ncb = (nx + 1 + NC - 1) / NC;
                    for (int b = 0; b < ncb; ++b) cols_by[fcol[f] ? 2 * ny + v : 0].push_back(WorkItem{f, b});
                }
        }
        std::vector<WorkItem> rows, cols;
        std::vector<std::pair<int, std::pair<size_t, size_t>>> rspan, cspan;   // key, [offset, count)
        for (auto& kv : rows_by) {
            rspan.push_back({kv.first, {rows.size(), kv.second.size()}});
            rows.insert(rows.end(), kv.second.begin(), kv.second.end());
        }
        for (auto& kv : cols_by) {
            cspan.push_back({kv.first, {cols.size(), kv.second.size()}});
            cols.insert(cols.end(), kv.second.begin(), kv.second.end());
        }
        if ((rc = dalloc(&d_films, sizeof(FilmDev) * nf))) return rc;
        CUDA_TRY(cudaMemcpyAsync(d_films, fh.data(), sizeof(FilmDev) * nf, cudaMemcpyHostToDevice, stream));
        if ((rc = dalloc(&d_row_items, sizeof(WorkItem) * std::max<size_t>(rows.size(), 1)))) return rc;
        if ((rc = dalloc(&d_col_items, sizeof(WorkItem) * std::max<size_t>(cols.size(), 1)))) return rc;
        CUDA_TRY(cudaMemcpyAsync(d_row_items, rows.data(), sizeof(WorkItem) * rows.size(), cudaMemcpyHostToDevice,
                                 stream));
        if (!cols.empty())
            CUDA_TRY(cudaMemcpyAsync(d_col_items, cols.data(), sizeof(WorkItem) * cols.size(), cudaMemcpyHostToDevice,
                                     stream));
        geom.films = d_films;
        geom.row_items = d_row_items;
        geom.n_row_items = (int)rows.size();
        geom.col_items = d_col_items;
        geom.n_col_items = (int)cols.size();
        geom.smem_row = smem_row;
        geom.smem_col = smem_col;
        geom.any_demag = any_demag;
        geom.fast_row = 0;
        geom.fast_col = 0;
        geom.fuse_rows = !env_flag("LLG_B200_NO_FUSE");
        geom.row_var = 0;
        geom.col_var = 0;
        CUDA_TRY(prepare_eval_kernels<R>(smem_row, smem_col));
        {
            // persistent grids: at most one wave of resident blocks looping over the work
            // items, shrunk to the fewest blocks that need the same number of rounds
            const int nsm = nsm_count();
            auto balanced = [&](int items, int per_sm) {
                items = std::max(items, 1);
                const int slots = std::max(1, nsm * per_sm);
                const int rounds = (items + slots - 1) / slots;
                return (items + rounds - 1) / rounds;
            };
            const int gen_r = std::min(8, std::max(1, (int)(200 * 1024 / std::max<size_t>(smem_row, 1))));
            const int gen_c = std::min(8, std::max(1, (int)(200 * 1024 / std::max<size_t>(smem_col, 1))));
            for (auto& sp : rspan) {
                std::array<LaunchGeom, 2> alt{};
                std::array<char, 2> has{0, 0};
                std::array<std::array<int, 4>, 2> occ{};
                for (int v = 0; v < 2; ++v) {
                    const int L = sp.first;
                    if (L ? !row_plan_ok(fast_config<R>(L, 2), v) : v > 0) continue;
                    LaunchGeom s = geom;
                    s.row_items = d_row_items + sp.second.first;
                    s.n_row_items = (int)sp.second.second;
                    s.fast_row = L;
                    s.row_var = v;
                    int fb = gen_r, ib = gen_r, ub = gen_r, zb = 1, cb = 1;
                    if (L) fast_occupancy<R>(L, 0, v, 0, &fb, &ib, &ub, &zb, &cb);
                    s.grid_row = balanced(s.n_row_items, fb);
                    s.grid_rinv = balanced(s.n_row_items, ib);
                    s.grid_rfull = balanced(s.n_row_items, ub);
                    s.grid_fused = balanced(s.n_row_items, zb);
                    alt[v] = s;
                    has[v] = 1;
                    occ[v] = {fb, ib, ub, zb};
                }
                {
                    std::vector<int> fl;
                    for (size_t q = 0; q < sp.second.second; ++q) fl.push_back(rows[sp.second.first + q].film);
                    std::sort(fl.begin(), fl.end());
                    fl.erase(std::unique(fl.begin(), fl.end()), fl.end());
                    rseg_films.push_back(fl);
                }
                rseg.push_back(alt[0]);
                rseg_alt.push_back(alt);
                rseg_has.push_back(has);
                rocc.push_back(occ);
            }
            // column segments: one per length, with the geometry of each radix plan
            std::map<int, size_t> col_index;
            for (auto& sp : cspan) {
                const int L = sp.first ? sp.first / 2 : 0, v = sp.first ? sp.first % 2 : 0;
                if (!col_index.count(L)) {
                    col_index[L] = cseg.size();
                    std::vector<int> fl;
                    for (size_t q = 0; q < sp.second.second; ++q) fl.push_back(cols[sp.second.first + q].film);
                    std::sort(fl.begin(), fl.end());
                    fl.erase(std::unique(fl.begin(), fl.end()), fl.end());
                    cseg_films.push_back(fl);
                    cseg.push_back(LaunchGeom{});
                    cseg_alt.push_back({});
                    cseg_has.push_back({0, 0, 0, 0});
                    cocc.push_back({1, 1, 1, 1});
                }
                const size_t i = col_index[L];
                for (int lean = 0; lean < (L ? 2 : 1); ++lean) {
                    const int cv = 2 * v + lean;
                    LaunchGeom s = geom;
                    s.col_items = d_col_items + sp.second.first;
                    s.n_col_items = (int)sp.second.second;
                    s.fast_col = L;
                    s.col_var = cv;
                    int fb = 1, ib = 1, ub = 1, zb = 1, cb = gen_c;
                    if (L) fast_occupancy<R>(0, L, 0, cv, &fb, &ib, &ub, &zb, &cb);
                    s.grid_col = balanced(s.n_col_items, cb);
                    cseg_alt[i][cv] = s;
                    cseg_has[i][cv] = 1;
                    cocc[i][cv] = cb;
                    if (cv == 0) cseg[i] = s;
                }
            }
        }
        if (any_demag && nf == 1) set_l2_window();
        if ((rc = autotune_grids(nsm_count()))) return rc;
        CUDA_TRY(cudaStreamSynchronize(stream));
        return LLG_OK;
    }

    int nsm_count() const {
        int nsm = 148;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
        return nsm;
    }

    // Grid autotuner of the register-FFT passes: for each pass, time the candidate
    // persistent grid sizes (for 1..occupancy resident blocks per SM: the fewest
    // blocks that need the same number of rounds over the work items, and the full
    // resident wave) on a representative RK45 stage and keep the fastest.  Runs once
    // per engine, on the engine's own buffers, before any state is set.
    // Radix plans and persistent grids of the register-FFT passes.  For each launch
    // segment and each radix plan its length has, the candidate grids of every pass
    // (the fewest blocks that need the same number of rounds over the work items for
    // 1..occupancy resident blocks per SM, and the full resident wave) are timed on a
    // representative RK45 stage on the engine's own buffers; a segment keeps the plan
    // whose passes are fastest in sum, each with its fastest grid.  The plan decides
    // the arithmetic order of the transforms, so the first decision for a (precision,
    // pass, length) is kept for the whole process and every engine computes the same
    // bits; grids do not change results.  LLG_B200_FFT_PLAN=0/1 fixes the plan,
    // LLG_B200_NO_AUTOTUNE=1 keeps plan 0 and the balanced grids.
    int autotune_grids(int nsm) {
        const int forced = forced_plan();
        const bool tuning = !env_flag("LLG_B200_NO_AUTOTUNE");
        const bool tune_log = env_flag("LLG_B200_TUNE_LOG");
        int rc;
        if ((rc = set_control(idle_control(), nullptr, nullptr, true))) return rc;
        EvalSpec stage = base_spec(LLG_FIELD_FULL);
        stage.rhs = RHS_LLG;
        combo(stage, MB_S0, {KB_K1, KB_K2, KB_K3}, {dp5::A41, dp5::A42, dp5::A43});
        stage.k_out = KB_K4;
        EvalSpec full = stage;
        full.reduce = 1;
        EvalSpec next = stage;   // the stage after `stage`, for the fused row pass
        combo(next, MB_S1, {KB_K1, KB_K2, KB_K3, KB_K4}, {dp5::A51, dp5::A52, dp5::A53, dp5::A54});
        next.k_out = KB_K5;
        cudaEvent_t e0, e1;
        CUDA_TRY(cudaEventCreate(&e0));
        CUDA_TRY(cudaEventCreate(&e1));
        auto candidates = [&](int items, int occ) {
            std::vector<int> c;
            items = std::max(items, 1);
            for (int per = 1; per <= occ; ++per) {
                const int slots = std::max(1, nsm * per), rounds = (items + slots - 1) / slots;
                c.push_back((items + rounds - 1) / rounds);
                c.push_back(std::min(items, slots));
            }
            std::sort(c.begin(), c.end());
            c.erase(std::unique(c.begin(), c.end()), c.end());
            return c;
        };
        // best grid of one pass; *best_ms receives its time (4 launches).  The
        // candidates are timed in three interleaved sweeps and each keeps its
        // fastest sweep, so a transient slowdown does not decide the choice.
        auto tune = [&](int which, const EvalSpec& spec, LaunchGeom& geom, int* grid, int items, int occ,
                        float* best_ms) -> int {
            auto one = [&]() {
                return which == 3 ? launch_fused<R>(spec, next, geom, stream) : launch_one<R>(which, spec, geom, stream);
            };
            const std::vector<int> cand = candidates(items, occ);
            std::vector<float> tmin(cand.size(), 1e30f);
            for (int sweep = 0; sweep < 3; ++sweep) {
                for (size_t ci = 0; ci < cand.size(); ++ci) {
                    *grid = cand[ci];
                    for (int w = 0; w < 2; ++w) CUDA_TRY(one());
                    CUDA_TRY(cudaEventRecord(e0, stream));
                    for (int r = 0; r < 4; ++r) CUDA_TRY(one());
                    CUDA_TRY(cudaEventRecord(e1, stream));
                    CUDA_TRY(cudaEventSynchronize(e1));
                    float ms = 0.f;
                    CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
                    tmin[ci] = std::min(tmin[ci], ms);
                }
            }
            size_t bi = 0;
            for (size_t ci = 1; ci < cand.size(); ++ci)
                if (tmin[ci] < tmin[bi]) bi = ci;
            // candidates are in increasing grid size: take the smallest grid within 2 %
            // of the fastest (equal in isolation, a pass with fewer resident blocks
            // measured faster between its neighbours in a step)
            for (size_t ci = 0; ci < bi; ++ci)
                if (tmin[ci] <= 1.02f * tmin[bi]) {
                    bi = ci;
                    break;
                }
            *grid = cand[bi];
            *best_ms = tmin[bi];
            if (tune_log) {   // LLG_B200_TUNE_LOG=1: candidate grids and their times on stderr
                std::fprintf(stderr, "llg_b200 tune pass %d items %d:", which, items);
                for (size_t ci = 0; ci < cand.size(); ++ci)
                    std::fprintf(stderr, " %d=%.4f%s", cand[ci], tmin[ci] / 4, ci == bi ? "*" : "");
                std::fprintf(stderr, "\n");
            }
            return LLG_OK;
        };
        auto tune_row = [&](size_t i, int v, float* total) -> int {
            LaunchGeom& sg = rseg_alt[i][v];
            const int nr = sg.n_row_items;
            const auto& oc = rocc[i][v];
            float t0 = 0.f, t1 = 0.f, t2 = 0.f, t3 = 0.f;
            int rc2;
            if ((rc2 = tune(0, stage, sg, &sg.grid_row, nr, oc[0], &t0))) return rc2;
            if ((rc2 = tune(2, stage, sg, &sg.grid_rinv, nr, oc[1], &t1))) return rc2;
            if ((rc2 = tune(2, full, sg, &sg.grid_rfull, nr, oc[2], &t2))) return rc2;
            if (sg.fast_row && sg.fuse_rows && (rc2 = tune(3, stage, sg, &sg.grid_fused, nr, oc[3], &t3))) return rc2;
            *total = t0 + t1 + t2 + t3;
            return LLG_OK;
        };
        auto pick = [&](int kind, int L, const auto& has, auto&& time_plan, int* chosen) -> int {
            *chosen = 0;
            if (!L) return LLG_OK;
            if (forced >= 0) {   // the register plan is fixed; a column keeps its staged form
                const int f = kind == 1 ? 2 * forced : forced;
                *chosen = has[f] ? f : 0;
                return LLG_OK;
            }
            const std::tuple<int, int, int> key{(int)sizeof(R), kind, L};
            {
                std::lock_guard<std::mutex> lock(g_plan_mutex);
                auto it = g_plan_cache.find(key);
                if (it != g_plan_cache.end()) {
                    *chosen = has[it->second] ? it->second : 0;
                    return LLG_OK;
                }
            }
            if (!tuning) return LLG_OK;
            float best = 1e30f;
            for (int v = 0; v < (int)has.size(); ++v) {
                if (!has[v]) continue;
                float t = 0.f;
                int rc2;
                if ((rc2 = time_plan(v, &t))) return rc2;
                if (t < best) {
                    best = t;
                    *chosen = v;
                }
            }
            std::lock_guard<std::mutex> lock(g_plan_mutex);
            g_plan_cache.emplace(key, *chosen);
            return LLG_OK;
        };
        for (size_t i = 0; i < rseg.size(); ++i) {
            int v = 0;
            if ((rc = pick(0, rseg[i].fast_row, rseg_has[i],
                           [&](int pv, float* t) { return tune_row(i, pv, t); }, &v)))
                return rc;
            float t = 0.f;
            if (tuning && (rc = tune_row(i, v, &t))) return rc;   // the kept plan's grids
            rseg[i] = rseg_alt[i][v];
        }
        for (size_t i = 0; i < cseg.size(); ++i) {
            auto time_col = [&](int pv, float* t) {
                LaunchGeom& sg = cseg_alt[i][pv];
                return tune(1, stage, sg, &sg.grid_col, sg.n_col_items, cocc[i][pv], t);
            };
            int v = 0;
            const int fixed = env_int("LLG_B200_COLUMN_FORM", -1);
            if (fixed >= 0 && fixed < 4 && cseg[i].fast_col && cseg_has[i][fixed]) v = fixed;
            else if ((rc = pick(1, cseg[i].fast_col, cseg_has[i], time_col, &v))) return rc;
            float t = 0.f;
            if (tuning && (rc = time_col(v, &t))) return rc;
            cseg[i] = cseg_alt[i][v];
        }
        // generic shared-memory kernels: the radix order / grouping of each length,
        // timed on the segment's passes at its current grid
        auto time_pass = [&](int kind, LaunchGeom& g, float* t) -> int {
            const int whiches[2][2] = {{0, 2}, {1, 1}};
            const int nw = kind == 0 ? 2 : 1;
            for (int w = 0; w < 2; ++w)
                for (int q = 0; q < nw; ++q) CUDA_TRY(launch_one<R>(whiches[kind][q], stage, g, stream));
            CUDA_TRY(cudaEventRecord(e0, stream));
            for (int r = 0; r < 4; ++r)
                for (int q = 0; q < nw; ++q) CUDA_TRY(launch_one<R>(whiches[kind][q], stage, g, stream));
            CUDA_TRY(cudaEventRecord(e1, stream));
            CUDA_TRY(cudaEventSynchronize(e1));
            CUDA_TRY(cudaEventElapsedTime(t, e0, e1));
            return LLG_OK;
        };
        if ((rc = tune_generic_plans(forced, tuning, time_pass))) return rc;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        invalidate_fsal_host();
        return LLG_OK;
    }

    // Radix plans of the generic shared-memory transforms: for every length that a
    // generic row or column segment transforms, the candidate orders / groupings of
    // its radices (plan_candidates) are timed on that segment's pass, one length at a
    // time with the others fixed, and the fastest is kept for every film of that
    // length.  Like the register-FFT plans, the first decision per (precision, pass,
    // length) holds for the whole process.
    template <typename TimeFn>
    int tune_generic_plans(int forced, bool tuning, TimeFn&& time_pass) {
        for (int kind = 0; kind < 2; ++kind) {
            auto& segs = kind == 0 ? rseg : cseg;
            auto& films = kind == 0 ? rseg_films : cseg_films;
            for (size_t i = 0; i < segs.size(); ++i) {
                LaunchGeom& sg = segs[i];
                if ((kind == 0 ? sg.fast_row : sg.fast_col) != 0) continue;
                std::vector<int> lengths;
                for (int f : films[i]) lengths.push_back(kind == 0 ? fh[f].nx : fh[f].ny);
                std::sort(lengths.begin(), lengths.end());
                lengths.erase(std::unique(lengths.begin(), lengths.end()), lengths.end());
                for (int L : lengths) {
                    const std::vector<FftPlan> cand = plan_candidates(L);
                    auto apply = [&](const FftPlan& pl) {
                        for (int f : films[i]) {
                            if ((kind == 0 ? fh[f].nx : fh[f].ny) != L) continue;
                            (kind == 0 ? fh[f].plan_row : fh[f].plan_col) = pl;
                        }
                        return upload_films();
                    };
                    const std::tuple<int, int, int> key{(int)sizeof(R), 2 + kind, L};
                    int chosen = -1;
                    {
                        std::lock_guard<std::mutex> lock(g_plan_mutex);
                        auto it = g_plan_cache.find(key);
                        if (it != g_plan_cache.end()) chosen = it->second;
                    }
                    if (chosen < 0 && tuning && forced < 0 && cand.size() > 1) {
                        float best = 1e30f;
                        for (size_t c = 0; c < cand.size(); ++c) {
                            int rc;
                            if ((rc = apply(cand[c]))) return rc;
                            float t = 0.f;
                            if ((rc = time_pass(kind, sg, &t))) return rc;
                            if (t < best) {
                                best = t;
                                chosen = (int)c;
                            }
                        }
                        std::lock_guard<std::mutex> lock(g_plan_mutex);
                        g_plan_cache.emplace(key, chosen);
                    }
                    if (chosen < 0 || chosen >= (int)cand.size()) chosen = 0;
                    int rc;
                    if ((rc = apply(cand[chosen]))) return rc;
                }
            }
        }
        return LLG_OK;
    }

    // The radix plan each launch segment runs (for reports): [row segments..., column segments...]
    int fft_plans(int* rows, int nr, int* cols, int nc) const override {
        for (int i = 0; i < nr && i < (int)rseg.size(); ++i) rows[i] = rseg[i].fast_row ? rseg[i].row_var : -1;
        for (int i = 0; i < nc && i < (int)cseg.size(); ++i) cols[i] = cseg[i].fast_col ? cseg[i].col_var : -1;
        return LLG_OK;
    }

    // Keep the spectrum scratch (written by the row pass, read by the column
    // pass, read again by the row-inverse pass) resident in L2 across the
    // passes of an evaluation.  The persisting carve-out belongs to this
    // process's context only.
    void set_l2_window() {
        int max_persist = 0, max_window = 0;
        cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, device);
        cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, device);
        if (max_persist <= 0 || max_window <= 0 || !fh[0].X) return;
        const size_t xbytes = sizeof(cx<R>) * 3 * (size_t)(fh[0].nx + 1) * fh[0].ny;
        size_t want = std::min<size_t>(xbytes, (size_t)max_persist);
        if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        cudaStreamAttrValue attr{};
        attr.accessPolicyWindow.base_ptr = fh[0].X;
        attr.accessPolicyWindow.num_bytes = std::min<size_t>(xbytes, (size_t)max_window);
        attr.accessPolicyWindow.hitRatio =
            (float)std::min(1.0, (double)want / (double)attr.accessPolicyWindow.num_bytes);
        attr.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
        attr.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
        l2_attr = attr;
        l2_window = true;
        if (cudaStreamSetAttribute(own_stream, cudaStreamAttributeAccessPolicyWindow, &attr) != cudaSuccess)
            cudaGetLastError();
    }

    int upload_films() {
        CUDA_TRY(cudaMemcpyAsync(d_films, fh.data(), sizeof(FilmDev) * nf, cudaMemcpyHostToDevice, stream));
        return LLG_OK;
    }

    int set_stream(cudaStream_t s) override {
        CUDA_TRY(cudaStreamSynchronize(stream));
        stream = s ? s : own_stream;
        if (l2_window && cudaStreamSetAttribute(stream, cudaStreamAttributeAccessPolicyWindow, &l2_attr) != cudaSuccess)
            cudaGetLastError();
        return LLG_OK;
    }
    int sync() override {
        CUDA_TRY(cudaStreamSynchronize(stream));
        return LLG_OK;
    }

    int ensure_stage() {
        if (!d_stage) return dalloc(&d_stage, sizeof(double) * 3 * (size_t)max_cells);
        return LLG_OK;
    }

    int read_states() {
        CUDA_TRY(cudaMemcpyAsync(h_states, d_states, sizeof(StepState) * nf, cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        return LLG_OK;
    }

    void invalidate_fsal_host() {
        fsal_kind = 0;
        fsal_mask = -1;
    }

    // Per-film control: dt from params (or kept) and FSAL invalidation flags.
    int set_control(const Control& c, const llg_params* p, const bool* invalidate, bool keep_dt) {
        for (int f = 0; f < nf; ++f) {
            h_ctl[f].dt = p ? p[f].dt : 0.0;
            h_ctl[f].keep_dt = (keep_dt || !p) ? 1 : 0;
            h_ctl[f].invalidate_fsal = invalidate ? (invalidate[f] ? 1 : 0) : 0;
        }
        CUDA_TRY(cudaMemcpyAsync(d_ctl, h_ctl, sizeof(FilmCtl) * nf, cudaMemcpyHostToDevice, stream));
        k_set_control<<<(nf + 127) / 128, 128, 0, stream>>>(d_films, nf, c, d_ctl);
        CUDA_TRY(cudaGetLastError());
        launches += 1;
        return LLG_OK;
    }

    Control idle_control() {
        Control c{};
        c.t_end = INFINITY;
        c.max_err = 1.0;
        c.headroom = 1.0;
        c.dt_min = 0.0;
        c.dt_max = 1.0;
        c.target_acc = -1;
        c.attempts = -1;
        c.reset_time = 0;
        return c;
    }

    int set_state(int f, const double* m) override {
        int rc;
        if ((rc = ensure_stage())) return rc;
        CUDA_TRY(cudaMemcpyAsync(d_stage, m, sizeof(double) * 3 * (size_t)cells(f), cudaMemcpyHostToDevice, stream));
        k_aos_to_soa<R><<<592, 256, 0, stream>>>(d_films, f, d_stage);
        CUDA_TRY(cudaGetLastError());
        launches += 1;
        // FSAL validity of film f is decided on the device by k_aos_to_soa
        if ((rc = set_control(idle_control(), nullptr, nullptr, true))) return rc;
        CUDA_TRY(cudaStreamSynchronize(stream));
        return LLG_OK;
    }

    // Replace every film's state by the warm-start network's proposal, on the device.
    int warm_start(ws::Net* net, const double* bext3n) override {
        int rc;
        if ((rc = read_states())) return rc;
        for (int f = 0; f < nf; ++f) {
            R* m = reinterpret_cast<R*>(const_cast<void*>(fh[f].m[h_states[f].cur ? 1 : 0]));
            CUDA_TRY(ws::net_apply<R>(net, m, m, fh[f].has_mask ? fh[f].mask : nullptr, bext3n + 3 * f, 1,
                                      fh[f].ny, fh[f].nx, stream));
        }
        invalidate_fsal_host();
        std::unique_ptr<bool[]> iv(new bool[nf]);
        for (int e = 0; e < nf; ++e) iv[e] = true;
        if ((rc = set_control(idle_control(), nullptr, iv.get(), true))) return rc;
        CUDA_TRY(cudaStreamSynchronize(stream));
        if (ws::net_error(net)) return set_error(LLG_ERR_TIMEOUT, "warm-start network: tensor-core wait timed out");
        return LLG_OK;
    }

    int write_ovf(int f, const char* path, const llg_ovf_meta* meta, int format) override {
        if (format == LLG_OVF_TEXT) {
            std::vector<double> m(3 * (size_t)cells(f));
            int rc = get_state(f, m.data());
            return rc ? rc : llg_ovf2_write(path, &grids[f], m.data(), meta, format);
        }
        if (format != LLG_OVF_BINARY4) return set_error(LLG_ERR_INVALID, "unknown OVF format %d", format);
        int rc;
        if ((rc = ensure_stage())) return rc;
        k_soa_to_aos_f32<R><<<592, 256, 0, stream>>>(d_films, f, reinterpret_cast<float*>(d_stage));
        CUDA_TRY(cudaGetLastError());
        std::vector<float> payload(3 * (size_t)cells(f));
        CUDA_TRY(cudaMemcpyAsync(payload.data(), d_stage, sizeof(float) * payload.size(), cudaMemcpyDeviceToHost,
                                 stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        return ovf2_write_packed(path, &grids[f], payload.data(), meta);
    }

    int get_state(int f, double* m) override {
        int rc;
        if ((rc = ensure_stage())) return rc;
        k_soa_to_aos<R><<<592, 256, 0, stream>>>(d_films, f, 0, d_stage);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(m, d_stage, sizeof(double) * 3 * (size_t)cells(f), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        return LLG_OK;
    }

    int mean_m(double* out3n) override {
        k_mean_m<R><<<std::min(geom.n_row_items, 148 * 8), 256, 0, stream>>>(d_films, d_row_items, geom.n_row_items);
        CUDA_TRY(cudaGetLastError());
        k_finalize<<<(nf + kFinalizeFilmsPerBlock - 1) / kFinalizeFilmsPerBlock, 32 * kFinalizeFilmsPerBlock, 0,
                     stream>>>(d_films, nf, 0);
        CUDA_TRY(cudaGetLastError());
        int rc;
        if ((rc = read_states())) return rc;
        for (int f = 0; f < nf; ++f)
            for (int c = 0; c < 3; ++c) out3n[3 * f + c] = h_states[f].red[RED_MX + c] / (double)cells(f);
        return LLG_OK;
    }

    // Sets gamma / alpha / b_ext of every film.
    int apply_params(const llg_params* p) {
        bool any = false;
        for (int f = 0; f < nf; ++f) {
            FilmDev& F = fh[f];
            bool ch = F.gamma != p[f].gamma || F.alpha != p[f].alpha || F.bext[0] != p[f].b_ext[0] ||
                      F.bext[1] != p[f].b_ext[1] || F.bext[2] != p[f].b_ext[2];
            if (ch) {
                F.gamma = p[f].gamma;
                F.alpha = p[f].alpha;
                for (int c = 0; c < 3; ++c) F.bext[c] = p[f].b_ext[c];
                any = true;
            }
        }
        return any ? upload_films() : LLG_OK;
    }

    EvalSpec base_spec(int fmask) {
        EvalSpec s;
        std::memset(&s, 0, sizeof(s));
        s.demag = fmask == LLG_FIELD_FULL ? 1 : 0;
        s.dmi = fmask == LLG_FIELD_EXCH_ANIS_DMI || fmask == LLG_FIELD_FULL ? 1 : 0;
        s.local = 1;
        s.m_in = MB_M0;
        s.k_out = KB_NONE;
        s.rhs = RHS_FIELD;
        return s;
    }

    static void combo(EvalSpec& s, int m_in, std::initializer_list<int> ks, std::initializer_list<double> as) {
        s.m_in = m_in;
        s.nterm = (int)ks.size();
        int q = 0;
        for (int k : ks) s.kidx[q++] = k;
        q = 0;
        for (double a : as) s.a[q++] = a;
    }

    int finalize(int req) {
        k_finalize<<<(nf + kFinalizeFilmsPerBlock - 1) / kFinalizeFilmsPerBlock, 32 * kFinalizeFilmsPerBlock, 0,
                     stream>>>(d_films, nf, req);
        CUDA_TRY(cudaGetLastError());
        launches += 1;
        return LLG_OK;
    }

    // Stage 1 of an attempt: k1 = f(m0), skipped on the device for films whose
    // first-same-as-last torque is valid.
    EvalSpec stage1_spec(int kind, int fmask, int req) {
        EvalSpec e = base_spec(fmask);
        e.req = req;
        e.rhs = kind == KIND_RK45 ? RHS_LLG : RHS_RELAX;
        e.k_out = KB_K1;
        e.skip_if_fsal = 1;
        return e;
    }

    // One integrator attempt: stages 1 (unless with_stage1 is false: RK45 graphs,
    // whose callers evaluate stage 1 once before their first attempt, since after
    // any attempt k1 of the film's state is valid) to s, then the controller; req
    // gates every kernel on StepState::req (relax).
    int launch_attempt(int kind, int fmask, int req, bool with_stage1 = true) {
        int rc;
        std::vector<EvalSpec> ch;
        EvalSpec e = stage1_spec(kind, fmask, req);
        if (with_stage1) ch.push_back(e);
        e.skip_if_fsal = 0;
        if (kind == KIND_RK45) {
            using namespace dp5;
            combo(e, MB_S0, {KB_K1}, {A21});
            e.k_out = KB_K2;
            ch.push_back(e);
            combo(e, MB_S1, {KB_K1, KB_K2}, {A31, A32});
            e.k_out = KB_K3;
            ch.push_back(e);
            combo(e, MB_S0, {KB_K1, KB_K2, KB_K3}, {A41, A42, A43});
            e.k_out = KB_K4;
            ch.push_back(e);
            combo(e, MB_S1, {KB_K1, KB_K2, KB_K3, KB_K4}, {A51, A52, A53, A54});
            e.k_out = KB_K5;
            ch.push_back(e);
            combo(e, MB_S0, {KB_K1, KB_K2, KB_K3, KB_K4, KB_K5}, {A61, A62, A63, A64, A65});
            e.k_out = KB_K6;
            ch.push_back(e);
            combo(e, MB_M7, {KB_K1, KB_K3, KB_K4, KB_K5, KB_K6}, {B1, B3, B4, B5, B6});
            e.k_out = KB_K7;
            e.err = ERR_RK45;
            const double wb[8] = {0, B1, 0, B3, B4, B5, B6, 0};
            const double wh[8] = {0, BH1, 0, BH3, BH4, BH5, BH6, BH7};
            std::memcpy(e.wb, wb, sizeof(wb));
            std::memcpy(e.wh, wh, sizeof(wh));
            ch.push_back(e);
            if ((rc = eval_chain(ch))) return rc;
            k_controller<<<(nf + 127) / 128, 128, 0, stream>>>(d_films, nf, 5, req);
            CUDA_TRY(cudaGetLastError());
            launches += 1;
        } else {
            using namespace bs3;
            combo(e, MB_S0, {KB_K1}, {A21});
            e.k_out = KB_K2;
            ch.push_back(e);
            combo(e, MB_S1, {KB_K2}, {A32});
            e.k_out = KB_K3;
            ch.push_back(e);
            combo(e, MB_M7, {KB_K1, KB_K2, KB_K3}, {B1, B2, B3});
            e.k_out = KB_K7;
            e.err = ERR_RK23;
            e.reduce = 1;
            const double wb[8] = {0, B1, B2, B3, 0, 0, 0, 0};
            const double wh[8] = {0, BH1, BH2, BH3, BH4, 0, 0, 0};
            std::memcpy(e.wb, wb, sizeof(wb));
            std::memcpy(e.wh, wh, sizeof(wh));
            ch.push_back(e);
            if ((rc = eval_chain(ch))) return rc;
            k_controller<<<(nf + 127) / 128, 128, 0, stream>>>(d_films, nf, 3, req);
            CUDA_TRY(cudaGetLastError());
            launches += 1;
            if ((rc = finalize(req))) return rc;
        }
        return LLG_OK;
    }

    // One relax iteration: the request-gated energy, torque and RK23 step, then the controller.
    int launch_relax_iteration(int fmask, const RelaxSettingsDev& S) {
        int rc;
        EvalSpec en = base_spec(LLG_FIELD_FULL);
        en.req = REQ_ENERGY;
        en.rhs = RHS_ENERGY;
        en.reduce = 1;
        en.demag = 1;  // the energy includes demag iff Material::demag (energy.rs:117-121)
        if ((rc = eval(en))) return rc;
        if ((rc = finalize(REQ_ENERGY))) return rc;
        EvalSpec tq = base_spec(fmask);
        tq.req = REQ_TORQUE;
        tq.rhs = RHS_TORQUE;
        tq.reduce = 1;
        if ((rc = eval(tq))) return rc;
        if ((rc = finalize(REQ_TORQUE))) return rc;
        if ((rc = launch_attempt(KIND_RK23, fmask, REQ_STEP))) return rc;
        k_relax_control<<<(nf + 127) / 128, 128, 0, stream>>>(d_films, d_relax, nf, S);
        CUDA_TRY(cudaGetLastError());
        launches += 1;
        return LLG_OK;
    }

    // One minimiser iteration: the RHS_MINIMIZE evaluation, the reductions, the controller.
    int launch_minimize_iteration(int fmask, const MinimizeSettingsDev& S) {
        int rc;
        EvalSpec e = base_spec(fmask);
        e.req = REQ_MINIMIZE;
        e.rhs = RHS_MINIMIZE;
        e.reduce = 1;
        if ((rc = eval(e))) return rc;
        if ((rc = finalize(REQ_MINIMIZE))) return rc;
        k_minimize_control<<<(nf + 127) / 128, 128, 0, stream>>>(d_films, d_min, nf, S);
        CUDA_TRY(cudaGetLastError());
        launches += 1;
        return LLG_OK;
    }

    int graph_launch(long long key, cudaGraphExec_t ge) {
        CUDA_TRY(cudaGraphLaunch(ge, stream));
        launches += graph_kernels[key];
        return LLG_OK;
    }

    static long long graph_key(int kind, int fmask, int reps) {
        return ((long long)kind << 40) | ((long long)fmask << 32) | (long long)reps;
    }

    // Graph of `reps` back-to-back attempts (or relax iterations).
    template <typename Body>
    int get_graph(long long key, int reps, Body body, cudaGraphExec_t* out) {
        auto it = graphs.find(key);
        if (it != graphs.end()) {
            *out = it->second;
            return LLG_OK;
        }
        cudaStream_t cap = own_stream;
        CUDA_TRY(cudaStreamSynchronize(stream));
        CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        cudaStream_t saved = stream;
        stream = cap;
        int rc = LLG_OK;
        const long long before = launches;
        for (int r = 0; r < reps && rc == LLG_OK; ++r) rc = body();
        graph_kernels[key] = launches - before;
        launches = before;
        stream = saved;
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(cap, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        CUDA_TRY(e);
        cudaGraphExec_t ge = nullptr;
        CUDA_TRY(cudaGraphInstantiate(&ge, g, 0));
        graphs[key] = ge;
        graph_defs[key] = g;
        *out = ge;
        return LLG_OK;
    }

    int attempt_graph(int kind, int fmask, int reps, cudaGraphExec_t* out) {
        return get_graph(graph_key(kind, fmask, reps), reps,
                         [&]() { return launch_attempt(kind, fmask, 0, kind != KIND_RK45); }, out);
    }

    // FSAL validity across calls (llg.rs:854-867, 317-330): same kind, mask and b_ext.
    void fsal_flags(int kind, const llg_params* p, int fmask, bool* inval) {
        for (int f = 0; f < nf; ++f) {
            bool same = fsal_kind == kind && fsal_mask == fmask && fsal_bext[3 * f] == p[f].b_ext[0] &&
                        fsal_bext[3 * f + 1] == p[f].b_ext[1] && fsal_bext[3 * f + 2] == p[f].b_ext[2];
            inval[f] = !same;
        }
    }

    void note_fsal(int kind, int fmask, const llg_params* p) {
        fsal_kind = kind;
        fsal_mask = fmask;
        for (int f = 0; f < nf; ++f)
            for (int c = 0; c < 3; ++c) fsal_bext[3 * f + c] = p[f].b_ext[c];
    }

    int step(int kind, llg_params* p, int fmask, double max_err, double headroom, double dt_min, double dt_max,
             double* eps, int32_t* acc, double* dtu) override {
        if (fmask < 0 || fmask > 2) return set_error(LLG_ERR_INVALID, "bad field mask %d", fmask);
        int rc;
        if ((rc = apply_params(p))) return rc;
        Control c = idle_control();
        c.max_err = max_err;
        c.headroom = headroom;
        c.dt_min = dt_min;
        c.dt_max = dt_max;
        c.attempts = 1;
        std::unique_ptr<bool[]> inv(new bool[nf]);
        fsal_flags(kind, p, fmask, inv.get());
        if ((rc = set_control(c, p, inv.get(), false))) return rc;
        cudaGraphExec_t ge = nullptr;
        if ((rc = attempt_graph(kind, fmask, 1, &ge))) return rc;
        if (kind == KIND_RK45 && (rc = eval(stage1_spec(kind, fmask, 0)))) return rc;
        if ((rc = graph_launch(graph_key(kind, fmask, 1), ge))) return rc;
        if ((rc = read_states())) return rc;
        for (int f = 0; f < nf; ++f) {
            const StepState& s = h_states[f];
            if (s.err_code) {
                invalidate_fsal_host();
                return set_error(s.err_code, "film %d: non-finite error norm (NaN/Inf in the state or field)", f);
            }
            eps[f] = s.eps;
            acc[f] = s.accepted;
            dtu[f] = s.dt_used;
            p[f].dt = s.dt;
        }
        // per-film FSAL validity is tracked on the device; the host tracks kind / mask / b_ext
        note_fsal(kind, fmask, p);
        return LLG_OK;
    }

    int run(int kind, llg_params* p, int fmask, double max_err, double headroom, double dt_min, double dt_max,
            int64_t n_acc, double t_end, int64_t max_attempts, int64_t* acc_out, int64_t* rej_out,
            double* t_adv) override {
        if (fmask < 0 || fmask > 2) return set_error(LLG_ERR_INVALID, "bad field mask %d", fmask);
        int rc;
        if ((rc = apply_params(p))) return rc;
        if ((rc = read_states())) return rc;
        std::vector<long long> acc0(nf), rej0(nf);
        for (int f = 0; f < nf; ++f) {
            acc0[f] = h_states[f].n_acc;
            rej0[f] = h_states[f].n_rej;
        }
        Control c = idle_control();
        c.t_end = t_end;
        c.max_err = max_err;
        c.headroom = headroom;
        c.dt_min = dt_min;
        c.dt_max = dt_max;
        c.target_acc = n_acc;
        c.attempts = max_attempts > 0 ? max_attempts : -1;
        c.reset_time = 1;
        std::unique_ptr<bool[]> inv(new bool[nf]);
        fsal_flags(kind, p, fmask, inv.get());
        if ((rc = set_control(c, p, inv.get(), false))) return rc;
        // Poll the device every 32 attempts.  With a step-count target no film can
        // finish in fewer attempts than its remaining steps, so a round launches at
        // most the smallest remaining count (graphs of 8 attempts, then single ones)
        // and no attempt is launched after every film is done.
        const int reps = 8;
        cudaGraphExec_t ge = nullptr, ge1 = nullptr;
        if ((rc = attempt_graph(kind, fmask, reps, &ge))) return rc;
        if (kind == KIND_RK45 && (rc = eval(stage1_spec(kind, fmask, 0)))) return rc;
        long long launched = 0;
        const long long limit = max_attempts > 0 ? max_attempts : (1LL << 40);
        long long round = 32;
        bool first = true;   // h_states predates set_control: every film is active in the first round
        for (;;) {
            if (n_acc > 0) {
                round = 32;
                for (int f = 0; f < nf; ++f)
                    if (first || h_states[f].active)
                        round = std::min(round, n_acc - (h_states[f].n_acc - acc0[f]));
                round = std::max(round, 1LL);
            }
            first = false;
            round = std::min(round, limit - launched);
            long long q = 0;
            for (; q + reps <= round; q += reps)
                if ((rc = graph_launch(graph_key(kind, fmask, reps), ge))) return rc;
            if (q < round && !ge1 && (rc = attempt_graph(kind, fmask, 1, &ge1))) return rc;
            for (; q < round; ++q)
                if ((rc = graph_launch(graph_key(kind, fmask, 1), ge1))) return rc;
            launched += round;
            if ((rc = read_states())) return rc;
            bool any = false;
            for (int f = 0; f < nf; ++f) any |= h_states[f].active != 0;
            if (!any || launched >= limit) break;
        }
        for (int f = 0; f < nf; ++f) {
            const StepState& s = h_states[f];
            acc_out[f] = s.n_acc - acc0[f];
            rej_out[f] = s.n_rej - rej0[f];
            t_adv[f] = s.t;
            p[f].dt = s.dt;
            if (s.err_code) {
                invalidate_fsal_host();
                return set_error(s.err_code, "film %d: non-finite error norm (NaN/Inf in the state or field)", f);
            }
        }
        note_fsal(kind, fmask, p);
        return LLG_OK;
    }

    // relax_with_report (relax.rs:334-768) for every film, on the device.
    int relax(llg_params* p, int fmask, const llg_relax_settings* st, llg_relax_report* rep) override {
        if (fmask < 0 || fmask > 2) return set_error(LLG_ERR_INVALID, "bad field mask %d", fmask);
        int rc;
        if ((rc = apply_params(p))) return rc;
        RelaxSettingsDev S;
        std::memset(&S, 0, sizeof(S));   // padding too: the graph cache compares settings bytewise
        S.max_err = st->max_err;
        S.headroom = st->headroom;
        S.dt_min = st->dt_min;
        S.dt_max = st->dt_max;
        S.rel_energy_tol = st->rel_energy_tol;
        S.thr = st->torque_threshold;
        S.plateau_rel = st->torque_plateau_rel;
        S.plateau_abs = st->torque_plateau_abs;
        S.tighten_factor = st->tighten_factor;
        S.tighten_floor = st->tighten_floor;
        S.gate = st->final_torque_gate;
        S.gate_max = st->final_torque_gate_max;
        S.energy_stride = st->energy_stride;
        S.check_stride = st->torque_check_stride;
        S.plateau_checks = st->torque_plateau_checks;
        S.plateau_min_checks = st->torque_plateau_min_checks;
        S.max_acc = st->max_accepted_steps;
        S.gate_extra = st->gate_max_extra_accepted_steps;
        S.gate_plateau_fails = st->gate_plateau_fails;
        S.phase1 = st->phase1_enabled;
        S.phase2 = st->phase2_enabled;
        S.metric = st->torque_metric;
        S.has_thr = st->has_torque_threshold;
        S.has_gate = st->has_final_torque_gate;
        S.has_gmax = st->has_final_torque_gate_max;
        for (int f = 0; f < nf; ++f) {
            std::memset(&h_relax[f], 0, sizeof(RelaxStateDev));
            h_relax[f].pc = RP_START;
            h_relax[f].last_stage = -1;
            h_relax[f].max_err = st->max_err;
            h_relax[f].n_cells = (double)cells(f);
            p[f].dt = std::min(std::max(p[f].dt, st->dt_min), st->dt_max);  // relax.rs:373
        }
        CUDA_TRY(cudaMemcpyAsync(d_relax, h_relax, sizeof(RelaxStateDev) * nf, cudaMemcpyHostToDevice, stream));
        Control c = idle_control();
        c.max_err = st->max_err;
        c.headroom = st->headroom;
        c.dt_min = st->dt_min;
        c.dt_max = st->dt_max;
        std::unique_ptr<bool[]> inv(new bool[nf]);
        for (int f = 0; f < nf; ++f) inv[f] = true;  // scratch.invalidate_last_b_eff() (relax.rs:374)
        invalidate_fsal_host();
        if ((rc = set_control(c, p, inv.get(), false))) return rc;
        // issue the first requests
        k_relax_control<<<(nf + 127) / 128, 128, 0, stream>>>(d_films, d_relax, nf, S);
        CUDA_TRY(cudaGetLastError());
        launches += 1;
        const int reps = 8;
        const long long key = graph_key(KIND_RELAX, fmask, reps);
        // the graph bakes the settings into the controller launches: rebuild when they differ
        if (graphs.count(key) && std::memcmp(&relax_graph_settings, &S, sizeof(S)) != 0) {
            cudaGraphExecDestroy(graphs[key]);
            cudaGraphDestroy(graph_defs[key]);
            graphs.erase(key);
            graph_defs.erase(key);
        }
        relax_graph_settings = S;
        cudaGraphExec_t ge = nullptr;
        if ((rc = get_graph(key, reps, [&]() { return launch_relax_iteration(fmask, S); }, &ge))) return rc;
        // Each iteration executes one request per film; accepted steps are capped by
        // max_accepted_steps and every step size reaches dt_min within a bounded number
        // of rejections, so this bound is only a safety net against a stuck film.
        const long long max_iters = 16 * std::max<long long>(st->max_accepted_steps, 1) + 1000000;
        long long iters = 0;
        for (;;) {
            for (int q = 0; q < 4; ++q)
                if ((rc = graph_launch(key, ge))) return rc;
            iters += 4 * reps;
            if (iters > max_iters)
                return set_error(LLG_ERR_TIMEOUT, "relax did not finish within %lld iterations", max_iters);
            CUDA_TRY(cudaMemcpyAsync(h_relax, d_relax, sizeof(RelaxStateDev) * nf, cudaMemcpyDeviceToHost, stream));
            if ((rc = read_states())) return rc;
            bool all = true;
            for (int f = 0; f < nf; ++f) all &= (h_relax[f].done != 0) || h_states[f].err_code != 0;
            if (all) break;
        }
        for (int f = 0; f < nf; ++f) {
            const RelaxStateDev& Q = h_relax[f];
            const StepState& s = h_states[f];
            if (s.err_code) return set_error(s.err_code, "film %d: non-finite error norm during relax", f);
            rep[f].accepted_steps = Q.accepted;
            rep[f].rejected_steps = Q.rejected;
            rep[f].torque_checks = Q.checks;
            rep[f].torque_field_rebuilds = Q.rebuilds;
            rep[f].stop_reason = Q.stop_reason;
            rep[f].last_stage_stop = Q.last_stage;
            rep[f].has_final_torque = Q.has_ft;
            rep[f].final_torque = Q.ft;
            rep[f].has_final_torque_max = Q.has_ftm;
            rep[f].final_torque_max = Q.ftm;
            rep[f].final_max_err = Q.max_err;
            rep[f].final_dt = s.dt;
            p[f].dt = s.dt;
        }
        note_fsal(KIND_RK23, fmask, p);
        return LLG_OK;
    }

    // minimize_damping_only (minimize.rs:107-369) for every film, device resident:
    // graphs of minimiser iterations replayed until every film has finished.
    int minimize(const llg_params* p, int fmask, const llg_minimize_settings* st, llg_minimize_report* rep) override {
        if (fmask < 0 || fmask > 2) return set_error(LLG_ERR_INVALID, "bad field mask %d", fmask);
        int rc;
        if ((rc = apply_params(p))) return rc;
        MinimizeSettingsDev S;
        std::memset(&S, 0, sizeof(S));   // padding too: the graph cache compares settings bytewise
        S.thr = st->torque_threshold;
        S.lambda0 = st->lambda0;
        S.lambda_min = st->lambda_min;
        S.lambda_max = st->lambda_max;
        S.grow = st->grow;
        S.shrink = st->shrink;
        S.stall_rel = st->stall_rel;
        S.dm_stop = st->dm_stop;
        S.gate = st->dm_torque_gate;
        S.gate_max = st->dm_torque_gate_max;
        S.max_iters = st->max_iters;
        S.stall_iters = st->stall_iters;
        S.min_iters_before_stall = st->min_iters_before_stall;
        S.dm_samples = st->dm_samples;
        S.dm_min_iters = st->dm_min_iters;
        S.has_dm_stop = st->has_dm_stop;
        S.has_gate = st->has_dm_torque_gate;
        S.has_gate_max = st->has_dm_torque_gate_max;
        for (int f = 0; f < nf; ++f) minimize_state_init(h_min[f], S, (double)cells(f));
        CUDA_TRY(cudaMemcpyAsync(d_min, h_min, sizeof(MinimizeStateDev) * nf, cudaMemcpyHostToDevice, stream));
        // the state changes: every FSAL torque and cached field goes stale
        std::unique_ptr<bool[]> inv(new bool[nf]);
        for (int f = 0; f < nf; ++f) inv[f] = true;
        invalidate_fsal_host();
        if ((rc = set_control(idle_control(), nullptr, inv.get(), true))) return rc;
        k_minimize_begin<<<(nf + 127) / 128, 128, 0, stream>>>(d_films, d_min, nf);
        CUDA_TRY(cudaGetLastError());
        launches += 1;
        const int reps = 8;
        const long long key = graph_key(KIND_MINIMIZE, fmask, reps);
        // the graph bakes the settings into the controller launches: rebuild when they differ
        if (graphs.count(key) && std::memcmp(&minimize_graph_settings, &S, sizeof(S)) != 0) {
            cudaGraphExecDestroy(graphs[key]);
            cudaGraphDestroy(graph_defs[key]);
            graphs.erase(key);
            graph_defs.erase(key);
        }
        minimize_graph_settings = S;
        cudaGraphExec_t ge = nullptr;
        if ((rc = get_graph(key, reps, [&]() { return launch_minimize_iteration(fmask, S); }, &ge))) return rc;
        // every film finishes within max_iters iterations; the bound is a safety net
        const long long bound = std::max<long long>(st->max_iters, 0) + 4 * reps;
        long long iters = 0;
        int per_poll = 1;
        bool all = true;
        for (int f = 0; f < nf; ++f) all &= h_min[f].done != 0;
        while (!all) {
            for (int q = 0; q < per_poll; ++q)
                if ((rc = graph_launch(key, ge))) return rc;
            iters += (long long)per_poll * reps;
            per_poll = std::min(per_poll * 2, 8);
            CUDA_TRY(cudaMemcpyAsync(h_min, d_min, sizeof(MinimizeStateDev) * nf, cudaMemcpyDeviceToHost, stream));
            CUDA_TRY(cudaStreamSynchronize(stream));
            all = true;
            for (int f = 0; f < nf; ++f) all &= h_min[f].done != 0;
            if (!all && iters > bound)
                return set_error(LLG_ERR_TIMEOUT, "minimize did not finish within %lld iterations", bound);
        }
        for (int f = 0; f < nf; ++f) {
            const MinimizeStateDev& M = h_min[f];
            rep[f].iters = M.iters;
            rep[f].converged = M.converged;
            rep[f].stalled = M.stalled;
            rep[f].dm_converged = M.dm_converged;
            rep[f].reserved = 0;
            rep[f].final_torque = M.final_torque;
            rep[f].final_max_dm = M.final_max_dm;
            rep[f].final_tmean = M.final_tmean;
            rep[f].final_lambda = M.final_lambda;
        }
        invalidate_fsal_host();
        return LLG_OK;
    }

    int ensure_bout() {
        bool any = false;
        for (int f = 0; f < nf; ++f) {
            if (!fh[f].bout) {
                int rc = dalloc(&fh[f].bout, sizeof(R) * 3 * (size_t)cells(f));
                if (rc) return rc;
                any = true;
            }
        }
        return any ? upload_films() : LLG_OK;
    }

    // Runs one evaluation of the resident states with an idle controller (dt kept).
    int eval_resident(const EvalSpec& e) {
        int rc;
        if ((rc = set_control(idle_control(), nullptr, nullptr, true))) return rc;
        if ((rc = eval(e))) return rc;
        if (e.reduce && (rc = finalize(0))) return rc;
        return LLG_OK;
    }

    int build_h_eff(int f, const llg_params* p, int fmask, double* b) override {
        if (fmask < 0 || fmask > 2) return set_error(LLG_ERR_INVALID, "bad field mask %d", fmask);
        int rc;
        if ((rc = apply_params(p))) return rc;
        if ((rc = ensure_bout())) return rc;
        if ((rc = ensure_stage())) return rc;
        EvalSpec e = base_spec(fmask);
        e.rhs = RHS_FIELD;
        if ((rc = eval_resident(e))) return rc;
        k_soa_to_aos<R><<<592, 256, 0, stream>>>(d_films, f, 1, d_stage);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(b, d_stage, sizeof(double) * 3 * (size_t)cells(f), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        return LLG_OK;
    }

    int demag_field(int f, double* b) override {
        int rc;
        if (!mats[f].demag) {
            std::memset(b, 0, sizeof(double) * 3 * (size_t)cells(f));
            return LLG_OK;
        }
        if ((rc = ensure_bout())) return rc;
        if ((rc = ensure_stage())) return rc;
        EvalSpec e = base_spec(LLG_FIELD_FULL);
        e.rhs = RHS_FIELD;
        e.local = 0;
        if ((rc = eval_resident(e))) return rc;
        k_soa_to_aos<R><<<592, 256, 0, stream>>>(d_films, f, 1, d_stage);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(b, d_stage, sizeof(double) * 3 * (size_t)cells(f), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        return LLG_OK;
    }

    int energy(const double* bext3n, llg_energy_breakdown* out) override {
        // compute_energy_geom (energy.rs:80-285): demag enters iff Material::demag
        std::vector<llg_params> p(nf);
        for (int f = 0; f < nf; ++f) {
            p[f].gamma = fh[f].gamma;
            p[f].alpha = fh[f].alpha;
            for (int c = 0; c < 3; ++c) p[f].b_ext[c] = bext3n[3 * f + c];
        }
        int rc;
        if ((rc = apply_params(p.data()))) return rc;
        EvalSpec e = base_spec(LLG_FIELD_FULL);
        e.demag = 1;
        e.rhs = RHS_ENERGY;
        e.reduce = 1;
        if ((rc = eval_resident(e))) return rc;
        if ((rc = read_states())) return rc;
        for (int f = 0; f < nf; ++f) {
            out[f].exchange = h_states[f].red[RED_E_EX];
            out[f].anisotropy = h_states[f].red[RED_E_AN];
            out[f].zeeman = h_states[f].red[RED_E_ZEE];
            out[f].dmi = h_states[f].red[RED_E_DMI];
            out[f].demag = h_states[f].red[RED_E_DEMAG];
        }
        return LLG_OK;
    }

    static double torque_from_host(int metric, double tmax, double tsum, double tsum2, double n) {
        switch (metric) {
            case LLG_TORQUE_MAX: return tmax;
            case LLG_TORQUE_MEAN: return tsum / std::max(n, 1.0);
            case LLG_TORQUE_RMS: return std::sqrt(tsum2 / std::max(n, 1.0));
            default: return tsum2 / std::max(n, 1.0);
        }
    }

    int torque_metric(const llg_params* p, int fmask, int metric, double* out) override {
        int rc;
        if ((rc = apply_params(p))) return rc;
        EvalSpec e = base_spec(fmask);
        e.rhs = RHS_TORQUE;
        e.reduce = 1;
        if ((rc = eval_resident(e))) return rc;
        if ((rc = read_states())) return rc;
        for (int f = 0; f < nf; ++f)
            out[f] = torque_from_host(metric, h_states[f].red[RED_TMAX], h_states[f].red[RED_TSUM],
                                      h_states[f].red[RED_TSUM2], (double)cells(f));
        return LLG_OK;
    }

    // Per-pass CUDA-event timing of one representative RK45 stage evaluation
    // (stage 4: three-term combination) repeated `reps` times on the stream.
    // Device time per pass of one RK45 stage (stage 4 of the tableau, CUDA events on
    // the solver stream): ms[0] row forward, ms[1] column, ms[2] row inverse (the
    // transform and the streaming torque kernel), ms[3] the fused row pass that ends
    // this stage and starts the next (0 where no segment fuses).
    int profile_stage(const llg_params* p, int fmask, int reps, double* ms4) override {
        int rc;
        if ((rc = apply_params(p))) return rc;
        if ((rc = set_control(idle_control(), nullptr, nullptr, true))) return rc;
        EvalSpec e = base_spec(fmask);
        e.rhs = RHS_LLG;
        combo(e, MB_S0, {KB_K1, KB_K2, KB_K3}, {dp5::A41, dp5::A42, dp5::A43});
        e.k_out = KB_K4;
        EvalSpec f = e;
        combo(f, MB_S1, {KB_K1, KB_K2, KB_K3, KB_K4}, {dp5::A51, dp5::A52, dp5::A53, dp5::A54});
        f.k_out = KB_K5;
        cudaEvent_t ev[5];
        for (auto& x : ev) CUDA_TRY(cudaEventCreate(&x));
        double acc[4] = {0, 0, 0, 0};
        bool any_fused = false;
        for (int r = 0; r < reps; ++r) {
            CUDA_TRY(cudaEventRecord(ev[0], stream));
            for (auto& sg : rseg) CUDA_TRY(launch_one<R>(0, e, sg, stream));
            CUDA_TRY(cudaEventRecord(ev[1], stream));
            if (e.demag && geom.any_demag)
                for (auto& sg : cseg) CUDA_TRY(launch_one<R>(1, e, sg, stream));
            CUDA_TRY(cudaEventRecord(ev[2], stream));
            for (auto& sg : rseg) CUDA_TRY(launch_one<R>(2, e, sg, stream));
            CUDA_TRY(cudaEventRecord(ev[3], stream));
            for (auto& sg : rseg)
                if (can_fuse(e, f, sg)) {
                    CUDA_TRY(launch_fused<R>(e, f, sg, stream));
                    any_fused = true;
                }
            CUDA_TRY(cudaEventRecord(ev[4], stream));
            CUDA_TRY(cudaEventSynchronize(ev[4]));
            for (int q = 0; q < 4; ++q) {
                float ms = 0.f;
                CUDA_TRY(cudaEventElapsedTime(&ms, ev[q], ev[q + 1]));
                acc[q] += ms;
            }
        }
        for (auto& x : ev) cudaEventDestroy(x);
        for (int q = 0; q < 4; ++q) ms4[q] = acc[q] / reps;
        if (!any_fused) ms4[3] = 0.0;
        return LLG_OK;
    }

    long long launch_count() override { return launches; }

    int kernel_kspace(int f, double* out) override {
        if (!mats[f].demag || !d_k64[f]) return set_error(LLG_ERR_INVALID, "material has demag disabled");
        size_t cnt = 4 * (size_t)(grids[f].nx + 1) * (grids[f].ny + 1);
        CUDA_TRY(cudaMemcpyAsync(out, d_k64[f], sizeof(double) * cnt, cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        return LLG_OK;
    }
};

}  // namespace llg

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
struct llg_ctx {
    int device;
};
namespace llg {
int ctx_device(const llg_ctx* c) { return c->device; }
}  // namespace llg
struct llg_solver {
    std::unique_ptr<llg::EngineBase> eng;
    int device;
};
struct llg_batch {
    std::unique_ptr<llg::EngineBase> eng;
    int device;
};

using llg::set_error;

// Lets other translation units report through llg_last_error().
void llg_set_error_message(const char* msg) { llg::g_last_error = msg ? msg : ""; }

struct llg_warmstart {
    llg::ws::Net* net;
    int device;
};

namespace {
int check_device(int device) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) return set_error(LLG_ERR_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(e));
    if (device < 0 || device >= count) return set_error(LLG_ERR_INVALID, "device %d out of range (%d)", device, count);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return set_error(LLG_ERR_CUDA, "cudaGetDeviceProperties");
    if (prop.major != 10) return set_error(LLG_ERR_NO_DEVICE, "device %d is sm_%d%d; the library is compiled for sm_100a", device,
                                           prop.major, prop.minor);
    return LLG_OK;
}
template <typename H>
int bind(H* s) {
    if (!s || !s->eng) return set_error(LLG_ERR_INVALID, "null handle");
    cudaError_t e = cudaSetDevice(s->device);
    if (e != cudaSuccess) return set_error(LLG_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
    return LLG_OK;
}
int check_grid(const llg_grid* g) {
    if (g->nx < 1 || g->ny < 1 || g->nx > 4096 || g->ny > 4096)
        return set_error(LLG_ERR_INVALID, "grid %lldx%lld out of range [1, 4096]", (long long)g->nx, (long long)g->ny);
    if (!(g->dx > 0) || !(g->dy > 0) || !(g->dz > 0)) return set_error(LLG_ERR_INVALID, "cell sizes must be > 0");
    return LLG_OK;
}
int make_engine(int device, int n, const llg_grid* g, const llg_material* m, int32_t precision,
                const uint8_t* const* masks, std::unique_ptr<llg::EngineBase>* out) {
    if (precision != LLG_PREC_FP32 && precision != LLG_PREC_FP64) return set_error(LLG_ERR_INVALID, "bad precision");
    for (int f = 0; f < n; ++f) {
        int rc = check_grid(&g[f]);
        if (rc) return rc;
    }
    if (precision == LLG_PREC_FP32) {
        auto* e = new llg::Engine<float>();
        out->reset(e);
        return e->init(device, n, g, m, masks);
    }
    auto* e = new llg::Engine<double>();
    out->reset(e);
    return e->init(device, n, g, m, masks);
}
}  // namespace

extern "C" {

int llg_abi_version(void) { return LLG_B200_ABI_VERSION; }

int llg_last_error(char* buf, size_t len) {
    if (!buf || len == 0) return LLG_ERR_INVALID;
    std::snprintf(buf, len, "%s", llg::g_last_error.c_str());
    return LLG_OK;
}

int llg_ctx_create(int device, llg_ctx** out) {
    if (!out) return set_error(LLG_ERR_INVALID, "null out");
    int rc = check_device(device);
    if (rc) return rc;
    *out = new llg_ctx{device};
    return LLG_OK;
}

int llg_ctx_destroy(llg_ctx* ctx) {
    delete ctx;
    return LLG_OK;
}

int llg_solver_create(llg_ctx* ctx, const llg_grid* grid, const llg_material* mat, int32_t precision,
                      const uint8_t* geom_mask, llg_solver** out) {
    if (!ctx || !grid || !mat || !out) return set_error(LLG_ERR_INVALID, "null argument");
    std::unique_ptr<llg_solver> s(new llg_solver());
    s->device = ctx->device;
    const uint8_t* masks[1] = {geom_mask};
    int rc = make_engine(ctx->device, 1, grid, mat, precision, masks, &s->eng);
    if (rc) return rc;
    *out = s.release();
    return LLG_OK;
}

int llg_solver_destroy(llg_solver* s) {
    if (!s) return LLG_OK;
    if (s->eng) cudaSetDevice(s->device);
    delete s;
    return LLG_OK;
}

int llg_solver_set_stream(llg_solver* s, void* stream) {
    int rc = bind(s);
    return rc ? rc : s->eng->set_stream(reinterpret_cast<cudaStream_t>(stream));
}
int llg_solver_sync(llg_solver* s) {
    int rc = bind(s);
    return rc ? rc : s->eng->sync();
}
int llg_set_state(llg_solver* s, const double* m) {
    int rc = bind(s);
    if (!rc && !m) rc = set_error(LLG_ERR_INVALID, "null m");
    return rc ? rc : s->eng->set_state(0, m);
}
int llg_get_state(llg_solver* s, double* m) {
    int rc = bind(s);
    if (!rc && !m) rc = set_error(LLG_ERR_INVALID, "null m");
    return rc ? rc : s->eng->get_state(0, m);
}
int llg_ovf2_write_state(llg_solver* s, const char* path, const llg_ovf_meta* meta, int32_t format) {
    int rc = bind(s);
    if (!rc && (!path || !meta)) rc = set_error(LLG_ERR_INVALID, "null argument");
    return rc ? rc : s->eng->write_ovf(0, path, meta, format);
}
int llg_mean_m(llg_solver* s, double out3[3]) {
    int rc = bind(s);
    return rc ? rc : s->eng->mean_m(out3);
}
int llg_build_h_eff(llg_solver* s, const llg_params* p, int32_t fmask, double* b) {
    int rc = bind(s);
    if (!rc && (!p || !b)) rc = set_error(LLG_ERR_INVALID, "null argument");
    return rc ? rc : s->eng->build_h_eff(0, p, fmask, b);
}
int llg_compute_demag_field(llg_solver* s, double* b) {
    int rc = bind(s);
    if (!rc && !b) rc = set_error(LLG_ERR_INVALID, "null argument");
    return rc ? rc : s->eng->demag_field(0, b);
}
int llg_step_rk45(llg_solver* s, llg_params* p, int32_t fmask, double max_err, double headroom, double dt_min,
                  double dt_max, double* eps, int32_t* acc, double* dtu) {
    int rc = bind(s);
    if (!rc && (!p || !eps || !acc || !dtu)) rc = set_error(LLG_ERR_INVALID, "null argument");
    return rc ? rc : s->eng->step(llg::KIND_RK45, p, fmask, max_err, headroom, dt_min, dt_max, eps, acc, dtu);
}
int llg_step_rk23_relax(llg_solver* s, llg_params* p, int32_t fmask, double max_err, double headroom, double dt_min,
                        double dt_max, double* eps, int32_t* acc, double* dtu) {
    int rc = bind(s);
    if (!rc && (!p || !eps || !acc || !dtu)) rc = set_error(LLG_ERR_INVALID, "null argument");
    return rc ? rc : s->eng->step(llg::KIND_RK23, p, fmask, max_err, headroom, dt_min, dt_max, eps, acc, dtu);
}
int llg_run_rk45(llg_solver* s, llg_params* p, int32_t fmask, double max_err, double headroom, double dt_min,
                 double dt_max, int64_t n_accepted, double t_end, int64_t max_attempts, int64_t* acc_out,
                 int64_t* rej_out, double* t_adv) {
    int rc = bind(s);
    if (!rc && (!p || !acc_out || !rej_out || !t_adv)) rc = set_error(LLG_ERR_INVALID, "null argument");
    return rc ? rc
              : s->eng->run(llg::KIND_RK45, p, fmask, max_err, headroom, dt_min, dt_max, n_accepted, t_end,
                            max_attempts, acc_out, rej_out, t_adv);
}
int llg_relax(llg_solver* s, llg_params* p, int32_t fmask, llg_relax_settings* st, llg_relax_report* rep) {
    int rc = bind(s);
    if (!rc && (!p || !st || !rep)) rc = set_error(LLG_ERR_INVALID, "null argument");
    if (rc) return rc;
    rc = s->eng->relax(p, fmask, st, rep);
    if (!rc) st->max_err = rep->final_max_err;  // written back as relax_with_report does
    return rc;
}
int llg_minimize(llg_solver* s, const llg_params* p, int32_t fmask, const llg_minimize_settings* st,
                 llg_minimize_report* rep) {
    int rc = bind(s);
    if (!rc && (!p || !st || !rep)) rc = set_error(LLG_ERR_INVALID, "null argument");
    return rc ? rc : s->eng->minimize(p, fmask, st, rep);
}
void llg_default_minimize_settings(llg_minimize_settings* st) {
    std::memset(st, 0, sizeof(*st));
    st->torque_threshold = 5e-4;
    st->max_iters = 20000;
    st->lambda0 = 2e-2;
    st->lambda_min = 1e-5;
    st->lambda_max = 5e-2;
    st->grow = 1.05;
    st->shrink = 0.8;
    st->stall_iters = 5000;
    st->stall_rel = 5e-4;
    st->min_iters_before_stall = 500;
    st->has_dm_stop = 1;
    st->dm_stop = 1e-6;
    st->dm_samples = 10;
    st->has_dm_torque_gate = 1;
    st->dm_torque_gate = 2e-3;
    st->has_dm_torque_gate_max = 1;
    st->dm_torque_gate_max = 5e-3;
    st->dm_min_iters = 50;
}
void llg_default_relax_settings(llg_relax_settings* st) {
    std::memset(st, 0, sizeof(*st));
    st->max_err = 1e-5;
    st->headroom = 0.8;
    st->dt_min = 1e-18;
    st->dt_max = 1e-11;
    st->phase1_enabled = 1;
    st->phase2_enabled = 1;
    st->energy_stride = 3;
    st->rel_energy_tol = 1e-12;
    st->torque_metric = LLG_TORQUE_MAX;
    st->has_torque_threshold = 1;
    st->torque_threshold = 1e-4;
    st->torque_check_stride = 1;
    st->torque_plateau_rel = 1e-3;
    st->torque_plateau_abs = 0.0;
    st->torque_plateau_checks = 0;
    st->torque_plateau_min_checks = 5;
    st->tighten_factor = 0.70710678118654752440;
    st->tighten_floor = 1e-9;
    st->max_accepted_steps = 2000000;
}
int llg_compute_energy(llg_solver* s, const double b_ext[3], llg_energy_breakdown* out) {
    int rc = bind(s);
    if (!rc && (!b_ext || !out)) rc = set_error(LLG_ERR_INVALID, "null argument");
    return rc ? rc : s->eng->energy(b_ext, out);
}
int llg_torque_metric(llg_solver* s, const llg_params* p, int32_t fmask, int32_t metric, double* out) {
    int rc = bind(s);
    if (!rc && (!p || !out)) rc = set_error(LLG_ERR_INVALID, "null argument");
    return rc ? rc : s->eng->torque_metric(p, fmask, metric, out);
}
int llg_demag_kernel_kspace(llg_solver* s, double* out) {
    int rc = bind(s);
    if (!rc && !out) rc = set_error(LLG_ERR_INVALID, "null argument");
    return rc ? rc : s->eng->kernel_kspace(0, out);
}
int llg_profile_stage(llg_solver* s, const llg_params* p, int32_t fmask, int32_t reps, double* ms4) {
    int rc = bind(s);
    if (!rc && (!p || !ms4 || reps < 1)) rc = set_error(LLG_ERR_INVALID, "bad argument");
    return rc ? rc : s->eng->profile_stage(p, fmask, reps, ms4);
}
static int fft_plans_of(llg::EngineBase* eng, int32_t* rows, int32_t nr, int32_t* cols, int32_t nc) {
    std::vector<int> r(std::max(nr, 0)), c(std::max(nc, 0));
    for (auto& x : r) x = -2;
    for (auto& x : c) x = -2;
    eng->fft_plans(r.data(), nr, c.data(), nc);
    for (int i = 0; i < nr; ++i) rows[i] = r[i];
    for (int i = 0; i < nc; ++i) cols[i] = c[i];
    return LLG_OK;
}

int llg_solver_fft_plans(llg_solver* s, int32_t* row_plan, int32_t* col_plan) {
    int rc = bind(s);
    if (!rc && (!row_plan || !col_plan)) rc = set_error(LLG_ERR_INVALID, "null argument");
    return rc ? rc : fft_plans_of(s->eng.get(), row_plan, 1, col_plan, 1);
}

int llg_solver_launch_count(llg_solver* s, int64_t* out) {
    int rc = bind(s);
    if (!rc && !out) rc = set_error(LLG_ERR_INVALID, "null argument");
    if (rc) return rc;
    *out = s->eng->launch_count();
    return LLG_OK;
}

// ---------------- batches of independent films ----------------
int llg_batch_create(llg_ctx* ctx, int32_t n, const llg_grid* grids, const llg_material* mats, int32_t precision,
                     const uint8_t* const* masks, llg_batch** out) {
    if (!ctx || !grids || !mats || !out || n < 1) return set_error(LLG_ERR_INVALID, "bad argument");
    std::unique_ptr<llg_batch> b(new llg_batch());
    b->device = ctx->device;
    int rc = make_engine(ctx->device, n, grids, mats, precision, masks, &b->eng);
    if (rc) return rc;
    *out = b.release();
    return LLG_OK;
}
int llg_batch_destroy(llg_batch* b) {
    if (!b) return LLG_OK;
    if (b->eng) cudaSetDevice(b->device);
    delete b;
    return LLG_OK;
}
int llg_batch_set_stream(llg_batch* b, void* stream) {
    int rc = bind(b);
    return rc ? rc : b->eng->set_stream(reinterpret_cast<cudaStream_t>(stream));
}
int llg_batch_set_state(llg_batch* b, int32_t film, const double* m) {
    int rc = bind(b);
    if (!rc && (!m || film < 0 || film >= b->eng->nfilms())) rc = set_error(LLG_ERR_INVALID, "bad film or null m");
    return rc ? rc : b->eng->set_state(film, m);
}
int llg_batch_get_state(llg_batch* b, int32_t film, double* m) {
    int rc = bind(b);
    if (!rc && (!m || film < 0 || film >= b->eng->nfilms())) rc = set_error(LLG_ERR_INVALID, "bad film or null m");
    return rc ? rc : b->eng->get_state(film, m);
}
int llg_batch_mean_m(llg_batch* b, double* out) {
    int rc = bind(b);
    if (!rc && !out) rc = set_error(LLG_ERR_INVALID, "null argument");
    return rc ? rc : b->eng->mean_m(out);
}
int llg_batch_step_rk45(llg_batch* b, llg_params* params, int32_t fmask, double max_err, double headroom,
                        double dt_min, double dt_max, double* eps, int32_t* accepted, double* dt_used) {
    int rc = bind(b);
    if (!rc && (!params || !eps || !accepted || !dt_used)) rc = set_error(LLG_ERR_INVALID, "null argument");
    return rc ? rc
              : b->eng->step(llg::KIND_RK45, params, fmask, max_err, headroom, dt_min, dt_max, eps, accepted, dt_used);
}
int llg_batch_run_rk45(llg_batch* b, llg_params* params, int32_t fmask, double max_err, double headroom,
                       double dt_min, double dt_max, int64_t n_accepted, double t_end, int64_t max_attempts,
                       int64_t* accepted, int64_t* rejected, double* t) {
    int rc = bind(b);
    if (!rc && (!params || !accepted || !rejected || !t)) rc = set_error(LLG_ERR_INVALID, "null argument");
    return rc ? rc
              : b->eng->run(llg::KIND_RK45, params, fmask, max_err, headroom, dt_min, dt_max, n_accepted, t_end,
                            max_attempts, accepted, rejected, t);
}
int llg_batch_relax(llg_batch* b, llg_params* params, int32_t fmask, const llg_relax_settings* settings,
                    llg_relax_report* reports) {
    int rc = bind(b);
    if (!rc && (!params || !settings || !reports)) rc = set_error(LLG_ERR_INVALID, "null argument");
    return rc ? rc : b->eng->relax(params, fmask, settings, reports);
}
int llg_batch_minimize(llg_batch* b, const llg_params* params, int32_t fmask, const llg_minimize_settings* settings,
                       llg_minimize_report* reports) {
    int rc = bind(b);
    if (!rc && (!params || !settings || !reports)) rc = set_error(LLG_ERR_INVALID, "null argument");
    return rc ? rc : b->eng->minimize(params, fmask, settings, reports);
}
int llg_batch_ovf2_write_state(llg_batch* b, int32_t film, const char* path, const llg_ovf_meta* meta,
                               int32_t format) {
    int rc = bind(b);
    if (!rc && (!path || !meta)) rc = set_error(LLG_ERR_INVALID, "null argument");
    if (!rc && (film < 0 || film >= b->eng->nfilms())) rc = set_error(LLG_ERR_INVALID, "bad film %d", film);
    return rc ? rc : b->eng->write_ovf(film, path, meta, format);
}
int llg_batch_compute_energy(llg_batch* b, const double* b_ext, llg_energy_breakdown* out) {
    int rc = bind(b);
    if (!rc && (!b_ext || !out)) rc = set_error(LLG_ERR_INVALID, "null argument");
    return rc ? rc : b->eng->energy(b_ext, out);
}
int llg_batch_fft_plans(llg_batch* b, int32_t* row_plans, int32_t n_row, int32_t* col_plans, int32_t n_col) {
    int rc = bind(b);
    if (!rc && ((n_row > 0 && !row_plans) || (n_col > 0 && !col_plans))) rc = set_error(LLG_ERR_INVALID, "null argument");
    return rc ? rc : fft_plans_of(b->eng.get(), row_plans, n_row, col_plans, n_col);
}

int llg_batch_launch_count(llg_batch* b, int64_t* out) {
    int rc = bind(b);
    if (!rc && !out) rc = set_error(LLG_ERR_INVALID, "null argument");
    if (rc) return rc;
    *out = b->eng->launch_count();
    return LLG_OK;
}

// ---------------------------------------------------------------------------
// Learned warm start (no reference counterpart)
// ---------------------------------------------------------------------------
int64_t llg_warmstart_param_count(void) { return llg::ws::net_param_count(); }

int llg_warmstart_create(llg_ctx* ctx, const float* params, int64_t n_params, llg_warmstart** out) {
    if (!ctx || !params || !out) return set_error(LLG_ERR_INVALID, "null argument");
    if (n_params != llg::ws::net_param_count())
        return set_error(LLG_ERR_INVALID, "expected %lld parameters, got %lld",
                         (long long)llg::ws::net_param_count(), (long long)n_params);
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return set_error(LLG_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
    llg::ws::Net* net = nullptr;
    e = llg::ws::net_create(params, n_params, ctx->device, &net);
    if (e != cudaSuccess) return set_error(LLG_ERR_CUDA, "warm-start network: %s", cudaGetErrorString(e));
    *out = new llg_warmstart{net, ctx->device};
    return LLG_OK;
}

int llg_warmstart_set_spin_limit(llg_warmstart* w, int64_t polls) {
    if (!w) return set_error(LLG_ERR_INVALID, "null argument");
    if (polls < 0) return set_error(LLG_ERR_INVALID, "negative spin limit");
    llg::ws::net_set_spin_limit(w->net, polls);
    return LLG_OK;
}

int llg_warmstart_destroy(llg_warmstart* w) {
    if (!w) return LLG_OK;
    cudaSetDevice(w->device);
    llg::ws::net_destroy(w->net);
    delete w;
    return LLG_OK;
}

int llg_warmstart_forward(llg_warmstart* w, int64_t nimg, int64_t ny, int64_t nx, const double* m_aos,
                          const uint8_t* mask, const double* b_ext, double* out_aos) {
    if (!w || !m_aos || !b_ext || !out_aos) return set_error(LLG_ERR_INVALID, "null argument");
    if (nimg < 1 || ny < 1 || nx < 1 || nimg * ny * nx > (1LL << 28))
        return set_error(LLG_ERR_INVALID, "bad sizes %lld x %lld x %lld", (long long)nimg, (long long)ny,
                         (long long)nx);
    cudaError_t e = cudaSetDevice(w->device);
    if (e != cudaSuccess) return set_error(LLG_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
    const long long hw = ny * nx, cells = nimg * hw;
    std::vector<float> soa((size_t)cells * 3);
    for (long long im = 0; im < nimg; ++im)
        for (long long c = 0; c < hw; ++c)
            for (int q = 0; q < 3; ++q) soa[(size_t)im * 3 * hw + q * hw + c] = (float)m_aos[3 * (im * hw + c) + q];
    float* d_m = nullptr;
    uint8_t* d_mask = nullptr;
    e = cudaMalloc(&d_m, sizeof(float) * soa.size());
    if (e == cudaSuccess && mask) e = cudaMalloc(&d_mask, (size_t)cells);
    if (e == cudaSuccess) e = cudaMemcpy(d_m, soa.data(), sizeof(float) * soa.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && mask) e = cudaMemcpy(d_mask, mask, (size_t)cells, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = llg::ws::net_apply<float>(w->net, d_m, d_m, d_mask, b_ext, (int)nimg, (int)ny, (int)nx, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(soa.data(), d_m, sizeof(float) * soa.size(), cudaMemcpyDeviceToHost);
    cudaFree(d_m);
    cudaFree(d_mask);
    if (e != cudaSuccess) return set_error(LLG_ERR_CUDA, "warm-start forward: %s", cudaGetErrorString(e));
    if (llg::ws::net_error(w->net)) return set_error(LLG_ERR_TIMEOUT, "warm-start network: tensor-core wait timed out");
    for (long long im = 0; im < nimg; ++im)
        for (long long c = 0; c < hw; ++c)
            for (int q = 0; q < 3; ++q) out_aos[3 * (im * hw + c) + q] = soa[(size_t)im * 3 * hw + q * hw + c];
    return LLG_OK;
}

int llg_batch_warm_start(llg_batch* b, llg_warmstart* w, const double* b_ext) {
    int rc = bind(b);
    if (!rc && (!w || !b_ext)) rc = set_error(LLG_ERR_INVALID, "null argument");
    if (!rc && w->device != b->device) rc = set_error(LLG_ERR_INVALID, "network and batch on different devices");
    return rc ? rc : b->eng->warm_start(w->net, b_ext);
}

// XorShift64 seeded initial states (initial_states.rs:43-68, 230-254).
static uint64_t xs_next(uint64_t* st) {
    uint64_t x = *st;
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    *st = x;
    return x;
}
static double xs_f64(uint64_t* st) { return (double)(xs_next(st) >> 11) * (1.0 / (double)(1ULL << 53)); }
static void norm3(const double* v, double* o) {
    double n2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    if (n2 == 0.0) {
        o[0] = 0.0; o[1] = 0.0; o[2] = 1.0;
        return;
    }
    double inv = 1.0 / std::sqrt(n2);
    o[0] = v[0] * inv; o[1] = v[1] * inv; o[2] = v[2] * inv;
}

void llg_init_random(int64_t n, uint64_t seed, double* m) {
    uint64_t st = seed == 0 ? 0x9E3779B97F4A7C15ULL : seed;
    for (int64_t i = 0; i < n; ++i) {
        double v[3];
        v[0] = xs_f64(&st) * 2.0 - 1.0;
        v[1] = xs_f64(&st) * 2.0 - 1.0;
        v[2] = xs_f64(&st) * 2.0 - 1.0;
        norm3(v, &m[i * 3]);
    }
}

void llg_init_uniform_with_noise(int64_t n, const double dir[3], double noise, uint64_t seed, double* m) {
    double base[3];
    norm3(dir, base);
    uint64_t st = seed == 0 ? 0x9E3779B97F4A7C15ULL : seed;
    for (int64_t i = 0; i < n; ++i) {
        double* v = &m[i * 3];
        if (v[0] == 0.0 && v[1] == 0.0 && v[2] == 0.0) continue;
        double dx = noise * (xs_f64(&st) * 2.0 - 1.0);
        double dy = noise * (xs_f64(&st) * 2.0 - 1.0);
        double dz = noise * (xs_f64(&st) * 2.0 - 1.0);
        double w[3] = {base[0] + dx, base[1] + dy, base[2] + dz};
        norm3(w, v);
    }
}

}  // extern "C"
