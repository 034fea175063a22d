// solver.cu — host driver and C ABI of the B200 LLG path.
//
// Engine<R> owns one film's device buffers and runs the integrator attempts as
// sequences of field evaluations (three kernels each) followed by a one-thread
// FP64 step controller, all reading their dynamic state (dt, buffer parity,
// activity) from device memory so that an attempt — or a run of attempts — is
// captured once as a CUDA graph and replayed without host round trips.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/llg_b200.h"
#include "build_api.h"
#include "field_kernels.cuh"

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

enum { KIND_RK45 = 1, KIND_RK23 = 2 };

struct Control {
    double dt, t_end, max_err, headroom, dt_min, dt_max;
    long long target_acc, attempts;
    int invalidate_fsal;
    int reset_time;
};

// ---------------------------------------------------------------------------
// small kernels
// ---------------------------------------------------------------------------
__global__ void k_set_control(FilmDev* films, int nfilms, Control c) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nfilms) return;
    StepState* st = films[f].st;
    st->dt = c.dt;
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
    if (c.invalidate_fsal) st->fsal_valid = 0;
    if (c.reset_time) st->t = 0.0;
    if (isfinite(c.t_end)) {
        double rem = c.t_end - st->t;
        if (st->dt > rem) st->dt = rem;
        if (!(st->t + 1e-18 < c.t_end)) st->active = 0;
    }
}

// Step-size controller (llg.rs:997-1025 for order 5, llg.rs:401-435 for order 3).
__global__ void k_controller(FilmDev* films, int nfilms, int order) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nfilms) return;
    StepState* st = films[f].st;
    if (!st->active) return;
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
        st->fsal_valid = 0;
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

// Sum the per-block partial reductions in block order (deterministic).
__global__ void k_finalize(FilmDev* films, int nfilms) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nfilms) return;
    const FilmDev& F = films[f];
    double acc[RED_NSLOT];
    for (int s = 0; s < RED_NSLOT; ++s) acc[s] = 0.0;
    for (int b = 0; b < F.nblk; ++b) {
        const double* p = F.red_part + (size_t)b * RED_NSLOT;
        for (int s = 0; s < RED_NSLOT; ++s) acc[s] = (s == RED_TMAX) ? fmax(acc[s], p[s]) : acc[s] + p[s];
    }
    for (int s = 0; s < RED_NSLOT; ++s) F.st->red[s] = acc[s];
}

template <typename R>
__global__ void k_mean_m(const FilmDev* films) {
    __shared__ double sm_red[32 * RED_NSLOT];
    const FilmDev& F = films[0];
    const int nx = F.nx, ny = F.ny, n = nx * ny, T = F.rows_per_block;
    const R* m = mbuf<R>(F, MB_M0, F.st->cur);
    for (int blk = blockIdx.x; blk < F.nblk; blk += gridDim.x) {
        double red[RED_NSLOT];
        for (int s = 0; s < RED_NSLOT; ++s) red[s] = 0.0;
        for (int e = threadIdx.x; e < T * nx; e += blockDim.x) {
            int j = blk * T + e / nx, i = e % nx;
            if (j >= ny) continue;
            int idx = j * nx + i;
            red[RED_MX] += (double)m[idx];
            red[RED_MY] += (double)m[n + idx];
            red[RED_MZ] += (double)m[2 * n + idx];
        }
        block_reduce(red, sm_red);
        if (threadIdx.x == 0)
            for (int s = 0; s < RED_NSLOT; ++s) F.red_part[(size_t)blk * RED_NSLOT + s] = red[s];
        __syncthreads();
    }
}

template <typename R>
__global__ void k_aos_to_soa(const FilmDev* films, const double* __restrict__ src) {
    const FilmDev& F = films[0];
    const int n = F.nx * F.ny;
    R* dst = mbuf<R>(F, MB_M0, F.st->cur);
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
        dst[idx] = (R)src[idx * 3 + 0];
        dst[n + idx] = (R)src[idx * 3 + 1];
        dst[2 * n + idx] = (R)src[idx * 3 + 2];
    }
}

template <typename R>
__global__ void k_soa_to_aos(const FilmDev* films, int which, double* __restrict__ dst) {
    const FilmDev& F = films[0];
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
    virtual int set_stream(cudaStream_t s) = 0;
    virtual int sync() = 0;
    virtual int set_state(const double* m) = 0;
    virtual int get_state(double* m) = 0;
    virtual int mean_m(double* out3) = 0;
    virtual int build_h_eff(const llg_params* p, int fmask, double* b) = 0;
    virtual int demag_field(double* b) = 0;
    virtual int step(int kind, llg_params* p, int fmask, double max_err, double headroom, double dt_min,
                     double dt_max, double* eps, int32_t* acc, double* dtu) = 0;
    virtual int run(int kind, llg_params* p, int fmask, double max_err, double headroom, double dt_min, double dt_max,
                    int64_t n_acc, double t_end, int64_t max_attempts, int64_t* acc_out, int64_t* rej_out,
                    double* t_adv) = 0;
    virtual int relax(llg_params* p, int fmask, llg_relax_settings* st, llg_relax_report* rep) = 0;
    virtual int energy(const double* bext, llg_energy_breakdown* out) = 0;
    virtual int torque_metric(const llg_params* p, int fmask, int metric, double* out) = 0;
    virtual int kernel_kspace(double* out) = 0;
    virtual int profile_stage(const llg_params* p, int fmask, int reps, double* ms3) = 0;
    virtual long long launch_count() = 0;
};

// LLG_B200_GENERIC_FFT=1 selects the generic shared-memory Stockham kernels
// even where a register-FFT kernel exists (used to cross-check the two paths).
static bool force_generic() {
    const char* e = std::getenv("LLG_B200_GENERIC_FFT");
    return e && e[0] == '1';
}

template <typename R>
struct Engine final : EngineBase {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    llg_grid grid{};
    llg_material mat{};
    int64_t n = 0;
    bool has_mask = false;
    FilmDev fh{};
    FilmDev* d_film = nullptr;
    StepState* d_state = nullptr;
    StepState* h_state = nullptr;  // pinned
    WorkItem* d_row_items = nullptr;
    WorkItem* d_col_items = nullptr;
    LaunchGeom geom{};
    double* d_stage = nullptr;
    double* d_k64 = nullptr;
    std::vector<void*> allocs;
    std::vector<double> k64_host;
    // host-side FSAL bookkeeping: the FSAL torque belongs to the last kind/mask/b_ext stepped
    int fsal_kind = 0;
    int fsal_mask = -1;
    double fsal_bext[3] = {0, 0, 0};
    bool last_b_eff_valid = false;  // relax: torque stats of the resident state are current
    std::map<long long, cudaGraphExec_t> graphs;
    std::map<long long, cudaGraph_t> graph_defs;
    std::map<long long, long long> graph_kernels;  // kernel nodes per graph
    long long launches = 0;                         // kernels issued on the stream so far

    int eval(const EvalSpec& e) {
        CUDA_TRY(launch_eval<R>(e, geom, stream));
        launches += (e.demag && geom.any_demag) ? 3 : 2;
        return LLG_OK;
    }

    ~Engine() override {
        if (stream) cudaStreamSynchronize(stream);
        for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
        for (auto& kv : graph_defs) cudaGraphDestroy(kv.second);
        for (void* p : allocs) cudaFree(p);
        if (h_state) cudaFreeHost(h_state);
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

    int init(int dev, const llg_grid* g, const llg_material* m, const uint8_t* mask) {
        device = dev;
        grid = *g;
        mat = *m;
        n = g->nx * g->ny;
        const int nx = (int)g->nx, ny = (int)g->ny;
        CUDA_TRY(cudaSetDevice(dev));
        CUDA_TRY(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking));
        stream = own_stream;
        CUDA_TRY(cudaMallocHost(&h_state, sizeof(StepState)));
        const bool demag = mat.demag != 0;
        // register-FFT kernels for power-of-two sizes, generic kernels otherwise
        const FastCfg fc = fast_config<R>(nx, ny);
        const bool fast = fc.ok && !force_generic();
        const int T = fast ? fc.T : 2;
        const int NC = fast ? fc.NC : 1;
        const int G = T + (T + 1) / 2;
        size_t smem_row = demag ? 4 * (size_t)G * nx * sizeof(cx<R>) : 0;
        size_t smem_col = demag ? 12 * (size_t)ny * sizeof(cx<R>) : 0;
        const size_t smem_max = 227 * 1024;
        if (!fast && (smem_row > smem_max || smem_col > smem_max))
            return set_error(LLG_ERR_INVALID, "grid %dx%d exceeds the in-shared-memory FFT limit for this precision",
                             nx, ny);
        int rc;
        const size_t plane = sizeof(R) * 3 * (size_t)n;
        FilmDev& F = fh;
        std::memset(&F, 0, sizeof(F));
        F.nx = nx;
        F.ny = ny;
        F.rows_per_block = T;
        F.nblk = (ny + T - 1) / T;
        F.dx = g->dx;
        F.dy = g->dy;
        F.dz = g->dz;
        F.ms = m->ms;
        F.a_ex = m->a_ex;
        F.k_u = m->k_u;
        F.dmi = m->has_dmi ? m->dmi : 0.0;
        F.exch = (m->a_ex != 0.0 && m->ms != 0.0) ? 2.0 * m->a_ex / m->ms : 0.0;
        F.has_eta = (m->has_dmi && m->dmi != 0.0) ? 1 : 0;
        F.eta = (F.has_eta && m->a_ex != 0.0) ? m->dmi / (2.0 * m->a_ex) : 0.0;
        F.dmi_avail = (m->has_dmi && m->dmi != 0.0 && m->ms != 0.0 && m->a_ex != 0.0) ? 1 : 0;
        F.dmi_pref = F.dmi_avail ? 2.0 * m->dmi / m->ms : 0.0;
        F.anis = (m->k_u != 0.0 && m->ms != 0.0) ? 2.0 * m->k_u / m->ms : 0.0;
        for (int c = 0; c < 3; ++c) F.u[c] = m->easy_axis[c];
        F.demag_mat = demag ? 1 : 0;
        F.plan_row = make_plan(nx);
        F.plan_col = make_plan(ny);
        for (int b = 0; b < 2; ++b) {
            if ((rc = dalloc(&F.m[b], plane))) return rc;
            if ((rc = dalloc(&F.ms_buf[b], plane))) return rc;
        }
        for (int q = 1; q <= 7; ++q)
            if ((rc = dalloc(&F.k[q], plane))) return rc;
        for (void* p : {F.m[0], F.m[1], F.ms_buf[0], F.ms_buf[1]}) CUDA_TRY(cudaMemsetAsync(p, 0, plane, stream));
        for (int q = 1; q <= 7; ++q) CUDA_TRY(cudaMemsetAsync(F.k[q], 0, plane, stream));
        if ((rc = dalloc(&F.red_part, sizeof(double) * RED_NSLOT * (size_t)F.nblk))) return rc;
        if ((rc = dalloc(&d_state, sizeof(StepState)))) return rc;
        CUDA_TRY(cudaMemsetAsync(d_state, 0, sizeof(StepState), stream));
        F.st = d_state;
        if (mask) {
            has_mask = true;
            uint8_t* dm = nullptr;
            if ((rc = dalloc(&dm, (size_t)n))) return rc;
            std::vector<uint8_t> norm((size_t)n);
            for (int64_t i = 0; i < n; ++i) norm[i] = mask[i] ? 1 : 0;
            CUDA_TRY(cudaMemcpyAsync(dm, norm.data(), (size_t)n, cudaMemcpyHostToDevice, stream));
            CUDA_TRY(cudaStreamSynchronize(stream));
            F.mask = dm;
            F.has_mask = 1;
        }
        if (demag) {
            void* tw_row;
            void* tw_col;
            if ((rc = dalloc(&tw_row, sizeof(cx<R>) * 2 * (size_t)nx))) return rc;
            if ((rc = dalloc(&tw_col, sizeof(cx<R>) * 2 * (size_t)ny))) return rc;
            CUDA_TRY(launch_twiddles(tw_row, 2 * nx, sizeof(R) == 8, stream));
            CUDA_TRY(launch_twiddles(tw_col, 2 * ny, sizeof(R) == 8, stream));
            F.tw_row = tw_row;
            F.tw_col = tw_col;
            if (fast) {
                void* twp_row;
                void* twp_col;
                if ((rc = dalloc(&twp_row, sizeof(cx<R>) * (size_t)std::max(fc.twp_row_size, 1)))) return rc;
                if ((rc = dalloc(&twp_col, sizeof(cx<R>) * (size_t)std::max(fc.twp_col_size, 1)))) return rc;
                CUDA_TRY(build_pass_tables<R>(twp_row, nx, twp_col, ny, stream));
                F.twp_row = twp_row;
                F.twp_col = twp_col;
            }
            if ((rc = dalloc(&F.X, sizeof(cx<R>) * 3 * (size_t)(nx + 1) * ny))) return rc;
            void* kh;
            if ((rc = dalloc(&kh, sizeof(r4<R>) * (size_t)(nx + 1) * (ny + 1)))) return rc;
            F.Khat = kh;
            if ((rc = dalloc(&d_k64, sizeof(double) * 4 * (size_t)(nx + 1) * (ny + 1)))) return rc;
            CUDA_TRY(build_demag_kernel(nx, ny, g->dx, g->dy, g->dz, sizeof(R) == 8, kh, d_k64, stream));
            if (fast) {
                void* kp;
                if ((rc = dalloc(&kp, sizeof(r4<R>) * (size_t)(nx + 1) * 2 * ny))) return rc;
                CUDA_TRY(build_kernel_parity(nx, ny, sizeof(R) == 8, kh, kp, stream));
                F.Kpar = kp;
            }
        }
        if ((rc = dalloc(&d_film, sizeof(FilmDev)))) return rc;
        CUDA_TRY(cudaMemcpyAsync(d_film, &F, sizeof(FilmDev), cudaMemcpyHostToDevice, stream));
        const int ncol_blk = (nx + 1 + NC - 1) / NC;
        std::vector<WorkItem> rows(F.nblk), cols(ncol_blk);
        for (int b = 0; b < F.nblk; ++b) rows[b] = WorkItem{0, b};
        for (int b = 0; b < ncol_blk; ++b) cols[b] = WorkItem{0, b};
        if ((rc = dalloc(&d_row_items, sizeof(WorkItem) * rows.size()))) return rc;
        if ((rc = dalloc(&d_col_items, sizeof(WorkItem) * cols.size()))) return rc;
        CUDA_TRY(cudaMemcpyAsync(d_row_items, rows.data(), sizeof(WorkItem) * rows.size(), cudaMemcpyHostToDevice,
                                 stream));
        CUDA_TRY(cudaMemcpyAsync(d_col_items, cols.data(), sizeof(WorkItem) * cols.size(), cudaMemcpyHostToDevice,
                                 stream));
        geom.films = d_film;
        geom.row_items = d_row_items;
        geom.n_row_items = F.nblk;
        geom.col_items = d_col_items;
        geom.n_col_items = ncol_blk;
        geom.smem_row = smem_row;
        geom.smem_col = smem_col;
        geom.grid_row = F.nblk;
        geom.grid_col = ncol_blk;
        geom.any_demag = demag;
        geom.fast_row = fast ? nx : 0;
        geom.fast_col = fast ? ny : 0;
        geom.row_threads = fast ? fc.row_threads : 256;
        geom.col_threads = fast ? fc.col_threads : 256;
        CUDA_TRY(prepare_eval_kernels<R>(fast ? 0 : smem_row, fast ? 0 : smem_col));
        if (fast) {
            // persistent grids: one wave of resident blocks looping over the work
            // items, so the twiddle tables are loaded once per block
            int nsm = 148, rb = 1, cb = 1;
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
            fast_occupancy<R>(nx, ny, &rb, &cb);
            geom.grid_row = std::min(F.nblk, nsm * rb);
            geom.grid_col = std::min(ncol_blk, nsm * cb);
        }
        if (demag) set_l2_window();
        CUDA_TRY(cudaStreamSynchronize(stream));
        return LLG_OK;
    }

    // Keep the spectrum scratch (written by the row pass, read by the column
    // pass, read again by the row-inverse pass) resident in L2 across the
    // passes of an evaluation.  The persisting carve-out is a property of this
    // process's context only.
    void set_l2_window() {
        int dev = device;
        int max_persist = 0, max_window = 0;
        cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, dev);
        cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, dev);
        if (max_persist <= 0 || max_window <= 0 || !fh.X) return;
        const size_t xbytes = sizeof(cx<R>) * 3 * (size_t)(fh.nx + 1) * fh.ny;
        size_t want = std::min<size_t>(xbytes, (size_t)max_persist);
        if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        cudaStreamAttrValue attr{};
        attr.accessPolicyWindow.base_ptr = fh.X;
        attr.accessPolicyWindow.num_bytes = std::min<size_t>(xbytes, (size_t)max_window);
        attr.accessPolicyWindow.hitRatio = (float)std::min(1.0, (double)want / (double)attr.accessPolicyWindow.num_bytes);
        attr.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
        attr.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
        l2_attr = attr;
        l2_window = true;
        if (cudaStreamSetAttribute(own_stream, cudaStreamAttributeAccessPolicyWindow, &attr) != cudaSuccess)
            cudaGetLastError();
    }
    bool l2_window = false;
    cudaStreamAttrValue l2_attr{};

    int upload_film() {
        CUDA_TRY(cudaMemcpyAsync(d_film, &fh, sizeof(FilmDev), cudaMemcpyHostToDevice, stream));
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
        if (!d_stage) return dalloc(&d_stage, sizeof(double) * 3 * (size_t)n);
        return LLG_OK;
    }

    int set_state(const double* m) override {
        int rc;
        if ((rc = ensure_stage())) return rc;
        CUDA_TRY(cudaMemcpyAsync(d_stage, m, sizeof(double) * 3 * (size_t)n, cudaMemcpyHostToDevice, stream));
        k_aos_to_soa<R><<<592, 256, 0, stream>>>(d_film, d_stage);
        CUDA_TRY(cudaGetLastError());
        invalidate_fsal_host();
        Control c = idle_control();
        c.invalidate_fsal = 1;
        k_set_control<<<1, 32, 0, stream>>>(d_film, 1, c);
        CUDA_TRY(cudaGetLastError());
        launches += 1;
        CUDA_TRY(cudaStreamSynchronize(stream));
        return LLG_OK;
    }

    int get_state(double* m) override {
        int rc;
        if ((rc = ensure_stage())) return rc;
        k_soa_to_aos<R><<<592, 256, 0, stream>>>(d_film, 0, d_stage);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(m, d_stage, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        return LLG_OK;
    }

    int read_state() {
        CUDA_TRY(cudaMemcpyAsync(h_state, d_state, sizeof(StepState), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        return LLG_OK;
    }

    int mean_m(double* out3) override {
        k_mean_m<R><<<fh.nblk, 256, 0, stream>>>(d_film);
        CUDA_TRY(cudaGetLastError());
        k_finalize<<<1, 32, 0, stream>>>(d_film, 1);
        CUDA_TRY(cudaGetLastError());
        int rc;
        if ((rc = read_state())) return rc;
        for (int c = 0; c < 3; ++c) out3[c] = h_state->red[RED_MX + c] / (double)n;
        return LLG_OK;
    }

    void invalidate_fsal_host() {
        fsal_kind = 0;
        fsal_mask = -1;
        last_b_eff_valid = false;
    }

    Control idle_control() {
        Control c{};
        c.dt = 0.0;
        c.t_end = INFINITY;
        c.max_err = 1.0;
        c.headroom = 1.0;
        c.dt_min = 0.0;
        c.dt_max = 1.0;
        c.target_acc = -1;
        c.attempts = -1;
        c.invalidate_fsal = 0;
        c.reset_time = 0;
        return c;
    }

    // Sets gamma/alpha/b_ext of the film; returns true when b_ext changed.
    int apply_params(const llg_params* p, bool* changed_bext) {
        bool ch = fh.gamma != p->gamma || fh.alpha != p->alpha;
        bool chb = fh.bext[0] != p->b_ext[0] || fh.bext[1] != p->b_ext[1] || fh.bext[2] != p->b_ext[2];
        if (ch || chb) {
            fh.gamma = p->gamma;
            fh.alpha = p->alpha;
            for (int c = 0; c < 3; ++c) fh.bext[c] = p->b_ext[c];
            int rc = upload_film();
            if (rc) return rc;
        }
        if (changed_bext) *changed_bext = chb;
        return LLG_OK;
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

    int launch_attempt(int kind, int fmask) {
        EvalSpec e = base_spec(fmask);
        const int rhs = kind == KIND_RK45 ? RHS_LLG : RHS_RELAX;
        e.rhs = rhs;
        e.k_out = KB_K1;
        e.skip_if_fsal = 1;
        { int _rc = eval(e); if (_rc) return _rc; }
        e.skip_if_fsal = 0;
        if (kind == KIND_RK45) {
            using namespace dp5;
            combo(e, MB_S0, {KB_K1}, {A21});
            e.k_out = KB_K2;
            { int _rc = eval(e); if (_rc) return _rc; }
            combo(e, MB_S1, {KB_K1, KB_K2}, {A31, A32});
            e.k_out = KB_K3;
            { int _rc = eval(e); if (_rc) return _rc; }
            combo(e, MB_S0, {KB_K1, KB_K2, KB_K3}, {A41, A42, A43});
            e.k_out = KB_K4;
            { int _rc = eval(e); if (_rc) return _rc; }
            combo(e, MB_S1, {KB_K1, KB_K2, KB_K3, KB_K4}, {A51, A52, A53, A54});
            e.k_out = KB_K5;
            { int _rc = eval(e); if (_rc) return _rc; }
            combo(e, MB_S0, {KB_K1, KB_K2, KB_K3, KB_K4, KB_K5}, {A61, A62, A63, A64, A65});
            e.k_out = KB_K6;
            { int _rc = eval(e); if (_rc) return _rc; }
            combo(e, MB_M7, {KB_K1, KB_K3, KB_K4, KB_K5, KB_K6}, {B1, B3, B4, B5, B6});
            e.k_out = KB_K7;
            e.err = ERR_RK45;
            const double wb[8] = {0, B1, 0, B3, B4, B5, B6, 0};
            const double wh[8] = {0, BH1, 0, BH3, BH4, BH5, BH6, BH7};
            std::memcpy(e.wb, wb, sizeof(wb));
            std::memcpy(e.wh, wh, sizeof(wh));
            { int _rc = eval(e); if (_rc) return _rc; }
            k_controller<<<1, 32, 0, stream>>>(d_film, 1, 5);
            CUDA_TRY(cudaGetLastError());
            launches += 1;
        } else {
            using namespace bs3;
            combo(e, MB_S0, {KB_K1}, {A21});
            e.k_out = KB_K2;
            { int _rc = eval(e); if (_rc) return _rc; }
            combo(e, MB_S1, {KB_K2}, {A32});
            e.k_out = KB_K3;
            { int _rc = eval(e); if (_rc) return _rc; }
            combo(e, MB_M7, {KB_K1, KB_K2, KB_K3}, {B1, B2, B3});
            e.k_out = KB_K7;
            e.err = ERR_RK23;
            e.reduce = 1;
            const double wb[8] = {0, B1, B2, B3, 0, 0, 0, 0};
            const double wh[8] = {0, BH1, BH2, BH3, BH4, 0, 0, 0};
            std::memcpy(e.wb, wb, sizeof(wb));
            std::memcpy(e.wh, wh, sizeof(wh));
            { int _rc = eval(e); if (_rc) return _rc; }
            k_controller<<<1, 32, 0, stream>>>(d_film, 1, 3);
            CUDA_TRY(cudaGetLastError());
            k_finalize<<<1, 32, 0, stream>>>(d_film, 1);
            CUDA_TRY(cudaGetLastError());
            launches += 2;
        }
        return LLG_OK;
    }

    int graph_launch(long long key, cudaGraphExec_t ge) {
        CUDA_TRY(cudaGraphLaunch(ge, stream));
        launches += graph_kernels[key];
        return LLG_OK;
    }

    // Graph of `reps` back-to-back attempts.
    static long long graph_key(int kind, int fmask, int reps) {
        return ((long long)kind << 40) | ((long long)fmask << 32) | (long long)reps;
    }

    int attempt_graph(int kind, int fmask, int reps, cudaGraphExec_t* out) {
        long long key = graph_key(kind, fmask, reps);
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
        for (int r = 0; r < reps && rc == LLG_OK; ++r) rc = launch_attempt(kind, fmask);
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

    int prepare_step(int kind, const llg_params* p, int fmask, Control* c) {
        bool chb = false;
        int rc = apply_params(p, &chb);
        if (rc) return rc;
        bool same = fsal_kind == kind && fsal_mask == fmask && fsal_bext[0] == p->b_ext[0] &&
                    fsal_bext[1] == p->b_ext[1] && fsal_bext[2] == p->b_ext[2];
        c->invalidate_fsal = same ? 0 : 1;
        return LLG_OK;
    }

    void note_fsal(int kind, int fmask, const llg_params* p) {
        fsal_kind = kind;
        fsal_mask = fmask;
        for (int c = 0; c < 3; ++c) fsal_bext[c] = p->b_ext[c];
    }

    int step(int kind, llg_params* p, int fmask, double max_err, double headroom, double dt_min, double dt_max,
             double* eps, int32_t* acc, double* dtu) override {
        if (fmask < 0 || fmask > 2) return set_error(LLG_ERR_INVALID, "bad field mask %d", fmask);
        Control c = idle_control();
        c.dt = p->dt;
        c.max_err = max_err;
        c.headroom = headroom;
        c.dt_min = dt_min;
        c.dt_max = dt_max;
        c.attempts = 1;
        int rc = prepare_step(kind, p, fmask, &c);
        if (rc) return rc;
        k_set_control<<<1, 32, 0, stream>>>(d_film, 1, c);
        CUDA_TRY(cudaGetLastError());
        launches += 1;
        cudaGraphExec_t ge = nullptr;
        if ((rc = attempt_graph(kind, fmask, 1, &ge))) return rc;
        if ((rc = graph_launch(graph_key(kind, fmask, 1), ge))) return rc;
        if ((rc = read_state())) return rc;
        const StepState& s = *h_state;
        if (s.err_code) {
            invalidate_fsal_host();
            return set_error(s.err_code, "non-finite error norm (NaN/Inf in the state or field)");
        }
        *eps = s.eps;
        *acc = s.accepted;
        *dtu = s.dt_used;
        p->dt = s.dt;
        if (s.accepted) note_fsal(kind, fmask, p);
        else invalidate_fsal_host();
        last_b_eff_valid = kind == KIND_RK23 && s.accepted;
        return LLG_OK;
    }

    int run(int kind, llg_params* p, int fmask, double max_err, double headroom, double dt_min, double dt_max,
            int64_t n_acc, double t_end, int64_t max_attempts, int64_t* acc_out, int64_t* rej_out,
            double* t_adv) override {
        if (fmask < 0 || fmask > 2) return set_error(LLG_ERR_INVALID, "bad field mask %d", fmask);
        int rc;
        if ((rc = read_state())) return rc;
        const long long acc0 = h_state->n_acc, rej0 = h_state->n_rej;
        Control c = idle_control();
        c.dt = p->dt;
        c.t_end = t_end;
        c.max_err = max_err;
        c.headroom = headroom;
        c.dt_min = dt_min;
        c.dt_max = dt_max;
        c.target_acc = n_acc;
        c.attempts = max_attempts > 0 ? max_attempts : -1;
        c.reset_time = 1;
        if ((rc = prepare_step(kind, p, fmask, &c))) return rc;
        k_set_control<<<1, 32, 0, stream>>>(d_film, 1, c);
        CUDA_TRY(cudaGetLastError());
        launches += 1;
        const int reps = 8;
        cudaGraphExec_t ge = nullptr;
        if ((rc = attempt_graph(kind, fmask, reps, &ge))) return rc;
        long long launched = 0;
        const long long limit = max_attempts > 0 ? max_attempts : (1LL << 40);
        for (;;) {
            // several graph launches between polls
            for (int q = 0; q < 4 && launched < limit; ++q) {
                if ((rc = graph_launch(graph_key(kind, fmask, reps), ge))) return rc;
                launched += reps;
            }
            if ((rc = read_state())) return rc;
            if (!h_state->active || launched >= limit) break;
        }
        const StepState& s = *h_state;
        *acc_out = s.n_acc - acc0;
        *rej_out = s.n_rej - rej0;
        *t_adv = s.t;
        p->dt = s.dt;
        if (s.err_code) {
            invalidate_fsal_host();
            return set_error(s.err_code, "non-finite error norm (NaN/Inf in the state or field)");
        }
        if (s.fsal_valid) note_fsal(kind, fmask, p);
        else invalidate_fsal_host();
        last_b_eff_valid = false;
        return LLG_OK;
    }

    int ensure_bout() {
        if (!fh.bout) {
            int rc = dalloc(&fh.bout, sizeof(R) * 3 * (size_t)n);
            if (rc) return rc;
            return upload_film();
        }
        return LLG_OK;
    }

    // Runs one evaluation of the resident state with an idle controller.
    int eval_resident(const EvalSpec& e) {
        Control c = idle_control();
        c.dt = 0.0;
        // keep the device dt: read it back first so that set_control preserves it
        int rc;
        if ((rc = read_state())) return rc;
        c.dt = h_state->dt;
        k_set_control<<<1, 32, 0, stream>>>(d_film, 1, c);
        CUDA_TRY(cudaGetLastError());
        launches += 1;
        { int _rc = eval(e); if (_rc) return _rc; }
        if (e.reduce) {
            k_finalize<<<1, 32, 0, stream>>>(d_film, 1);
            CUDA_TRY(cudaGetLastError());
        }
        return LLG_OK;
    }

    int build_h_eff(const llg_params* p, int fmask, double* b) override {
        if (fmask < 0 || fmask > 2) return set_error(LLG_ERR_INVALID, "bad field mask %d", fmask);
        int rc;
        if ((rc = apply_params(p, nullptr))) return rc;
        if ((rc = ensure_bout())) return rc;
        if ((rc = ensure_stage())) return rc;
        EvalSpec e = base_spec(fmask);
        e.rhs = RHS_FIELD;
        if ((rc = eval_resident(e))) return rc;
        k_soa_to_aos<R><<<592, 256, 0, stream>>>(d_film, 1, d_stage);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(b, d_stage, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        return LLG_OK;
    }

    int demag_field(double* b) override {
        int rc;
        if (!mat.demag) {
            std::memset(b, 0, sizeof(double) * 3 * (size_t)n);
            return LLG_OK;
        }
        if ((rc = ensure_bout())) return rc;
        if ((rc = ensure_stage())) return rc;
        EvalSpec e = base_spec(LLG_FIELD_FULL);
        e.rhs = RHS_FIELD;
        e.local = 0;
        if ((rc = eval_resident(e))) return rc;
        k_soa_to_aos<R><<<592, 256, 0, stream>>>(d_film, 1, d_stage);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(b, d_stage, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        return LLG_OK;
    }

    int energy(const double* bext, llg_energy_breakdown* out) override {
        // compute_energy_geom (energy.rs:80-285): demag enters iff Material::demag
        llg_params p{};
        p.gamma = fh.gamma;
        p.alpha = fh.alpha;
        for (int c = 0; c < 3; ++c) p.b_ext[c] = bext[c];
        int rc;
        if ((rc = apply_params(&p, nullptr))) return rc;
        EvalSpec e = base_spec(LLG_FIELD_FULL);
        e.demag = mat.demag ? 1 : 0;
        e.rhs = RHS_ENERGY;
        e.reduce = 1;
        if ((rc = eval_resident(e))) return rc;
        if ((rc = read_state())) return rc;
        out->exchange = h_state->red[RED_E_EX];
        out->anisotropy = h_state->red[RED_E_AN];
        out->zeeman = h_state->red[RED_E_ZEE];
        out->dmi = h_state->red[RED_E_DMI];
        out->demag = h_state->red[RED_E_DEMAG];
        return LLG_OK;
    }

    double metric_from(const StepState& s, int metric) {
        const double nf = (double)n;
        switch (metric) {
            case LLG_TORQUE_MAX: return s.red[RED_TMAX];
            case LLG_TORQUE_MEAN: return s.red[RED_TSUM] / std::max(nf, 1.0);
            case LLG_TORQUE_RMS: return std::sqrt(s.red[RED_TSUM2] / std::max(nf, 1.0));
            default: return s.red[RED_TSUM2] / std::max(nf, 1.0);
        }
    }

    int torque_metric(const llg_params* p, int fmask, int metric, double* out) override {
        int rc;
        if ((rc = apply_params(p, nullptr))) return rc;
        EvalSpec e = base_spec(fmask);
        e.rhs = RHS_TORQUE;
        e.reduce = 1;
        if ((rc = eval_resident(e))) return rc;
        if ((rc = read_state())) return rc;
        *out = metric_from(*h_state, metric);
        return LLG_OK;
    }

    // Per-kernel CUDA-event timing of one representative RK45 stage evaluation
    // (stage 4: three-term combination) repeated `reps` times on the stream.
    int profile_stage(const llg_params* p, int fmask, int reps, double* ms3) override {
        int rc;
        if ((rc = apply_params(p, nullptr))) return rc;
        Control c = idle_control();
        if ((rc = read_state())) return rc;
        c.dt = h_state->dt > 0 ? h_state->dt : p->dt;
        k_set_control<<<1, 32, 0, stream>>>(d_film, 1, c);
        CUDA_TRY(cudaGetLastError());
        EvalSpec e = base_spec(fmask);
        e.rhs = RHS_LLG;
        combo(e, MB_S0, {KB_K1, KB_K2, KB_K3}, {dp5::A41, dp5::A42, dp5::A43});
        e.k_out = KB_K4;
        cudaEvent_t ev[4];
        for (auto& x : ev) CUDA_TRY(cudaEventCreate(&x));
        double acc[3] = {0, 0, 0};
        for (int r = 0; r < reps; ++r) {
            CUDA_TRY(cudaEventRecord(ev[0], stream));
            k_row_forward_launch(e);
            CUDA_TRY(cudaEventRecord(ev[1], stream));
            if (e.demag && geom.any_demag) k_column_launch(e);
            CUDA_TRY(cudaEventRecord(ev[2], stream));
            k_row_inverse_launch(e);
            CUDA_TRY(cudaEventRecord(ev[3], stream));
            CUDA_TRY(cudaEventSynchronize(ev[3]));
            for (int q = 0; q < 3; ++q) {
                float ms = 0.f;
                CUDA_TRY(cudaEventElapsedTime(&ms, ev[q], ev[q + 1]));
                acc[q] += ms;
            }
        }
        for (auto& x : ev) cudaEventDestroy(x);
        for (int q = 0; q < 3; ++q) ms3[q] = acc[q] / reps;
        return LLG_OK;
    }
    void k_row_forward_launch(const EvalSpec& e) { launch_one<R>(0, e, geom, stream); }
    void k_column_launch(const EvalSpec& e) { launch_one<R>(1, e, geom, stream); }
    void k_row_inverse_launch(const EvalSpec& e) { launch_one<R>(2, e, geom, stream); }

    long long launch_count() override { return launches; }

    int kernel_kspace(double* out) override {
        if (!mat.demag || !d_k64) return set_error(LLG_ERR_INVALID, "material has demag disabled");
        size_t cnt = 4 * (size_t)(grid.nx + 1) * (grid.ny + 1);
        CUDA_TRY(cudaMemcpyAsync(out, d_k64, sizeof(double) * cnt, cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        return LLG_OK;
    }

    // relax_with_report (relax.rs:334-768) driving the GPU RK23 attempts.
    int relax(llg_params* p, int fmask, llg_relax_settings* st, llg_relax_report* rep) override {
        const bool phase1 = st->phase1_enabled != 0, phase2 = st->phase2_enabled != 0;
        const int64_t energy_stride = std::max<int64_t>(st->energy_stride, 1);
        const int metric = st->torque_metric;
        const bool has_thr = st->has_torque_threshold != 0;
        const double thr = st->torque_threshold;
        const int64_t check_stride = std::max<int64_t>(st->torque_check_stride, 1);
        const double plateau_rel = st->torque_plateau_rel, plateau_abs = st->torque_plateau_abs;
        const int64_t plateau_checks = st->torque_plateau_checks;
        const int64_t plateau_min_checks = std::max<int64_t>(st->torque_plateau_min_checks, 1);
        const int64_t max_acc = st->max_accepted_steps;
        double max_err = st->max_err;
        p->dt = std::min(std::max(p->dt, st->dt_min), st->dt_max);
        invalidate_fsal_host();  // scratch.invalidate_last_b_eff()
        int64_t accepted = 0, rejected = 0, checks = 0, rebuilds = 0;
        int last_stage = -1;
        bool has_ft = false, has_ftm = false;
        double ft = 0.0, ftm = 0.0;
        double torque_cache[RED_NSLOT];
        int rc = LLG_OK;
        auto finish = [&](int reason) {
            st->max_err = max_err;
            rep->accepted_steps = accepted;
            rep->rejected_steps = rejected;
            rep->torque_checks = checks;
            rep->torque_field_rebuilds = rebuilds;
            rep->stop_reason = reason;
            rep->last_stage_stop = last_stage;
            rep->has_final_torque = has_ft;
            rep->final_torque = ft;
            rep->has_final_torque_max = has_ftm;
            rep->final_torque_max = ftm;
            rep->final_max_err = max_err;
            rep->final_dt = p->dt;
            return LLG_OK;
        };
        auto advance = [&](int64_t n_accept, bool* ok) -> int {
            int64_t target = accepted + std::max<int64_t>(n_accept, 1);
            *ok = true;
            while (accepted < target) {
                if (accepted >= max_acc) {
                    *ok = false;
                    return LLG_OK;
                }
                double eps, dtu;
                int32_t acc = 0;
                int r = step(KIND_RK23, p, fmask, max_err, st->headroom, st->dt_min, st->dt_max, &eps, &acc, &dtu);
                if (r) return r;
                if (acc) {
                    ++accepted;
                    std::memcpy(torque_cache, h_state->red, sizeof(torque_cache));
                } else {
                    ++rejected;
                }
            }
            return LLG_OK;
        };
        auto torque_now = [&](int met, double* out) -> int {
            ++checks;
            if (last_b_eff_valid) {
                StepState tmp;
                std::memcpy(tmp.red, torque_cache, sizeof(torque_cache));
                *out = metric_from(tmp, met);
                return LLG_OK;
            }
            ++rebuilds;
            return torque_metric(p, fmask, met, out);
        };
        auto total_energy = [&](double* e) -> int {
            llg_energy_breakdown b;
            int r = energy(p->b_ext, &b);
            *e = b.exchange + b.anisotropy + b.zeeman + b.dmi + b.demag;
            return r;
        };
        bool ok;
        if (phase1) {
            double e0, e1;
            if ((rc = total_energy(&e0))) return rc;
            for (;;) {
                if ((rc = advance(energy_stride, &ok))) return rc;
                if (!ok) return finish(0);
                if ((rc = total_energy(&e1))) return rc;
                double tol = st->rel_energy_tol * std::max(std::fabs(e0), 1e-30);
                if (e1 < e0 - tol) {
                    e0 = e1;
                    continue;
                }
                break;
            }
        }
        if (!phase2) return finish(1);
        const bool plateau_enabled = !has_thr && plateau_checks > 0;
        const int64_t need_fails = std::max<int64_t>(plateau_checks, 1);
        for (;;) {
            double t_prev;
            if ((rc = torque_now(metric, &t_prev))) return rc;
            const bool f32mode = plateau_enabled && metric == LLG_TORQUE_MEANSQ && plateau_rel == 0.0 &&
                                 plateau_abs == 0.0 && plateau_checks == 1 && plateau_min_checks == 1;
            const double nf = (double)n;
            float t_prev_f32 = f32mode ? (float)(t_prev * nf) : (float)t_prev;
            int64_t fails = 0, comparisons = 0;
            for (;;) {
                if (has_thr && t_prev <= thr) {
                    last_stage = 0;
                    break;
                }
                if (plateau_enabled && fails >= need_fails) {
                    last_stage = 1;
                    break;
                }
                if (accepted >= max_acc) {
                    last_stage = 2;
                    has_ft = true;
                    ft = t_prev;
                    return finish(0);
                }
                if ((rc = advance(check_stride, &ok))) return rc;
                if (!ok) {
                    last_stage = 2;
                    has_ft = true;
                    ft = t_prev;
                    return finish(0);
                }
                double t_new;
                if ((rc = torque_now(metric, &t_new))) return rc;
                if (plateau_enabled) {
                    ++comparisons;
                    if (comparisons < plateau_min_checks) {
                        fails = 0;
                    } else if (f32mode) {
                        float t_new_f32 = (float)(t_new * nf);
                        bool improved = t_new_f32 < t_prev_f32;
                        t_prev_f32 = t_new_f32;
                        fails = improved ? 0 : fails + 1;
                    } else {
                        double need = std::max(plateau_rel * std::max(std::fabs(t_prev), 1e-30), plateau_abs);
                        fails = (t_prev - t_new) > need ? 0 : fails + 1;
                    }
                }
                t_prev = t_new;
            }
            has_ft = true;
            ft = t_prev;
            if (max_err <= st->tighten_floor) break;
            max_err *= st->tighten_factor;
            if (max_err < st->tighten_floor) max_err = st->tighten_floor;
        }
        if ((rc = torque_now(LLG_TORQUE_MAX, &ftm))) return rc;
        has_ftm = true;
        const bool has_gate = st->has_final_torque_gate != 0, has_gmax = st->has_final_torque_gate_max != 0;
        if ((has_gate || has_gmax) && st->gate_max_extra_accepted_steps > 0) {
            const int64_t start = accepted;
            double last_t = has_ft ? ft : INFINITY;
            int64_t gfails = 0;
            for (;;) {
                double t_metric, t_max = NAN;
                if ((rc = torque_now(metric, &t_metric))) return rc;
                if (has_gmax || metric == LLG_TORQUE_MAX) {
                    if (metric == LLG_TORQUE_MAX) t_max = t_metric;
                    else if ((rc = torque_now(LLG_TORQUE_MAX, &t_max))) return rc;
                }
                const bool okm = !has_gate || t_metric <= st->final_torque_gate;
                const bool okx = !has_gmax || t_max <= st->final_torque_gate_max;
                has_ft = true;
                ft = t_metric;
                if (std::isfinite(t_max)) {
                    has_ftm = true;
                    ftm = t_max;
                }
                if (okm && okx) break;
                if (accepted - start >= st->gate_max_extra_accepted_steps) return finish(3);
                if (st->gate_plateau_fails > 0) {
                    double need = std::max(plateau_rel * std::max(std::fabs(last_t), 1e-30), plateau_abs);
                    gfails = (last_t - t_metric) > need ? 0 : gfails + 1;
                    if (gfails >= st->gate_plateau_fails) return finish(3);
                    last_t = t_metric;
                }
                if ((rc = advance(check_stride, &ok))) return rc;
                if (!ok) {
                    last_stage = 2;
                    return finish(0);
                }
            }
        }
        return finish(2);
    }
};

}  // namespace llg

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
struct llg_ctx {
    int device;
};
struct llg_solver {
    std::unique_ptr<llg::EngineBase> eng;
    int device;
};

using llg::set_error;

namespace {
int check_device(int device) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) return set_error(LLG_ERR_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(e));
    if (device < 0 || device >= count) return set_error(LLG_ERR_INVALID, "device %d out of range (%d)", device, count);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return set_error(LLG_ERR_CUDA, "cudaGetDeviceProperties");
    if (prop.major != 10) return set_error(LLG_ERR_NO_DEVICE, "device %d is sm_%d%d; this build targets sm_100a", device,
                                           prop.major, prop.minor);
    return LLG_OK;
}
int bind(llg_solver* s) {
    if (!s || !s->eng) return set_error(LLG_ERR_INVALID, "null solver");
    cudaError_t e = cudaSetDevice(s->device);
    if (e != cudaSuccess) return set_error(LLG_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
    return LLG_OK;
}
}  // namespace

// Lets other translation units report through llg_last_error().
void llg_set_error_message(const char* msg) { llg::g_last_error = msg ? msg : ""; }

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
    if (grid->nx < 1 || grid->ny < 1 || grid->nx > 4096 || grid->ny > 4096)
        return set_error(LLG_ERR_INVALID, "grid %lldx%lld out of range [1, 4096]", (long long)grid->nx,
                         (long long)grid->ny);
    if (!(grid->dx > 0) || !(grid->dy > 0) || !(grid->dz > 0)) return set_error(LLG_ERR_INVALID, "cell sizes must be > 0");
    if (precision != LLG_PREC_FP32 && precision != LLG_PREC_FP64) return set_error(LLG_ERR_INVALID, "bad precision");
    std::unique_ptr<llg_solver> s(new llg_solver());
    s->device = ctx->device;
    int rc;
    if (precision == LLG_PREC_FP32) {
        auto* e = new llg::Engine<float>();
        s->eng.reset(e);
        rc = e->init(ctx->device, grid, mat, geom_mask);
    } else {
        auto* e = new llg::Engine<double>();
        s->eng.reset(e);
        rc = e->init(ctx->device, grid, mat, geom_mask);
    }
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
    return rc ? rc : s->eng->set_state(m);
}
int llg_get_state(llg_solver* s, double* m) {
    int rc = bind(s);
    if (!rc && !m) rc = set_error(LLG_ERR_INVALID, "null m");
    return rc ? rc : s->eng->get_state(m);
}
int llg_mean_m(llg_solver* s, double out3[3]) {
    int rc = bind(s);
    return rc ? rc : s->eng->mean_m(out3);
}
int llg_build_h_eff(llg_solver* s, const llg_params* p, int32_t fmask, double* b) {
    int rc = bind(s);
    if (!rc && (!p || !b)) rc = set_error(LLG_ERR_INVALID, "null argument");
    return rc ? rc : s->eng->build_h_eff(p, fmask, b);
}
int llg_compute_demag_field(llg_solver* s, double* b) {
    int rc = bind(s);
    if (!rc && !b) rc = set_error(LLG_ERR_INVALID, "null argument");
    return rc ? rc : s->eng->demag_field(b);
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
    return rc ? rc : s->eng->relax(p, fmask, st, rep);
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
    return rc ? rc : s->eng->kernel_kspace(out);
}

int llg_profile_stage(llg_solver* s, const llg_params* p, int32_t fmask, int32_t reps, double* ms3) {
    int rc = bind(s);
    if (!rc && (!p || !ms3 || reps < 1)) rc = set_error(LLG_ERR_INVALID, "bad argument");
    return rc ? rc : s->eng->profile_stage(p, fmask, reps, ms3);
}
int llg_solver_launch_count(llg_solver* s, int64_t* out) {
    int rc = bind(s);
    if (!rc && !out) rc = set_error(LLG_ERR_INVALID, "null argument");
    if (rc) return rc;
    *out = s->eng->launch_count();
    return LLG_OK;
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
