// amr_demag.cu — the AMR consumers of the uniform FFT demag, on the GPU.
//
// compute_coarse_fft_demag (coarse_fft_demag.rs:367-511): restrict the patches'
// fine magnetisation onto the base (L0) grid without renormalising
// (restrict_m_to_coarse, :170-240), optionally restrict L0 onto a coarser demag
// grid (restrict_l0_to_demag_grid, :256-290), run the FP64 FFT demag on that
// grid, sample it back onto L0 (interpolate_demag_to_l0, :299-318) and
// bilinear-sample the L0 field onto every patch cell including ghosts
// (sample_demag_to_patch, :327-340).
//
// The AllFft branch of AmrStepper::compute_demag (amr/stepper.rs:799-835): the
// FFT demag of the flattened fine grid, zero in vacuum, sampled at the base-grid
// cell centres.
//
// Restriction, sampling and interpolation keep the reference's FP64 operation
// order without contraction (explicit round-to-nearest products), so for the
// same input they give the same bits as the CPU restatement; the FFT demag is
// the operator of llg_demag_op_create (FP64, round-off level).
//
// Data: every field is AoS FP64 [cells][3] as VectorField2D stores it.  One
// pinned staging buffer takes the per-call inputs (L0 m, the patches' fine m,
// masks and parent flags), which go to the device in one copy; the patch
// descriptors carry offsets into it.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/llg_b200.h"
#include "build_api.h"

namespace llg {
int ctx_device(const llg_ctx* c);
}

namespace {

struct PatchDev {
    long long i0, j0, cnx, cny, ratio, ghost, pnx, pny;
    long long m_off;      // first double of the patch's fine m in the staged inputs
    long long mask_off;   // first byte of its fine mask (-1: none)
    long long pm_off;     // first byte of its parent_material flags (-1: all material)
    long long out_off;    // first cell of its samples in b_patches
};

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    llg_set_error_message(buf);
    return code;
}

#define AMR_TRY(x)                                                                                           \
    do {                                                                                                     \
        cudaError_t _e = (x);                                                                                \
        if (_e != cudaSuccess)                                                                               \
            return fail(_e == cudaErrorMemoryAllocation ? LLG_ERR_OOM : LLG_ERR_CUDA, "%s: %s", #x,          \
                        cudaGetErrorString(_e));                                                             \
    } while (0)

constexpr int kGrid = 148 * 8;

__device__ __forceinline__ long long clamp_idx(long long i, long long n) { return i < 0 ? 0 : (i >= n ? n - 1 : i); }

// sample_bilinear (amr/interp.rs:28-72), products and sums rounded separately
__device__ __forceinline__ void sample_bilinear(const double* __restrict__ f, long long nx, long long ny, double dx,
                                                double dy, double x, double y, double* o) {
    if (nx == 0 || ny == 0) {
        o[0] = o[1] = o[2] = 0.0;
        return;
    }
    const double fx = __dsub_rn(__ddiv_rn(x, dx), 0.5), fy = __dsub_rn(__ddiv_rn(y, dy), 0.5);
    const double i0f = floor(fx), j0f = floor(fy);
    const double tx = __dsub_rn(fx, i0f), ty = __dsub_rn(fy, j0f);
    const long long i0 = clamp_idx((long long)i0f, nx), j0 = clamp_idx((long long)j0f, ny);
    const long long i1 = clamp_idx((long long)i0f + 1, nx), j1 = clamp_idx((long long)j0f + 1, ny);
    const double* v00 = f + (j0 * nx + i0) * 3;
    const double* v10 = f + (j0 * nx + i1) * 3;
    const double* v01 = f + (j1 * nx + i0) * 3;
    const double* v11 = f + (j1 * nx + i1) * 3;
    const double ux = __dsub_rn(1.0, tx), uy = __dsub_rn(1.0, ty);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const double a = __dadd_rn(__dmul_rn(v00[c], ux), __dmul_rn(v10[c], tx));
        const double b = __dadd_rn(__dmul_rn(v01[c], ux), __dmul_rn(v11[c], tx));
        o[c] = __dadd_rn(__dmul_rn(a, uy), __dmul_rn(b, ty));
    }
}

// restrict_m_to_coarse (coarse_fft_demag.rs:170-240).  Patches are applied in order
// and a later one overwrites an earlier one, so each L0 cell takes the last patch
// that covers it (scanned backwards), or keeps its own value.
__global__ void k_restrict_patches(const double* __restrict__ mc, long long nx, long long ny,
                                   const PatchDev* __restrict__ pd, int np, const unsigned char* __restrict__ staged,
                                   double* __restrict__ out) {
    const double* pm = reinterpret_cast<const double*>(staged);
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nx * ny;
         e += (long long)gridDim.x * blockDim.x) {
        const long long i = e % nx, j = e / nx;
        int q = np - 1;
        for (; q >= 0; --q) {
            const PatchDev& p = pd[q];
            if (i >= p.i0 && i < p.i0 + p.cnx && j >= p.j0 && j < p.j0 + p.cny) break;
        }
        double v[3];
        if (q < 0) {
            v[0] = mc[e * 3];
            v[1] = mc[e * 3 + 1];
            v[2] = mc[e * 3 + 2];
        } else {
            const PatchDev& p = pd[q];
            const long long ic = i - p.i0, jc = j - p.j0;
            v[0] = v[1] = v[2] = 0.0;
            if (p.pm_off < 0 || staged[p.pm_off + jc * p.cnx + ic]) {
                double s0 = 0.0, s1 = 0.0, s2 = 0.0;
                long long nmat = 0;
                const double* m = pm + p.m_off;
                for (long long fj = 0; fj < p.ratio; ++fj)
                    for (long long fi = 0; fi < p.ratio; ++fi) {
                        const long long idx = (p.ghost + jc * p.ratio + fj) * p.pnx + p.ghost + ic * p.ratio + fi;
                        if (p.mask_off >= 0 && !staged[p.mask_off + idx]) continue;
                        s0 = __dadd_rn(s0, m[idx * 3]);
                        s1 = __dadd_rn(s1, m[idx * 3 + 1]);
                        s2 = __dadd_rn(s2, m[idx * 3 + 2]);
                        nmat += 1;
                    }
                if (nmat > 0) {
                    const double inv = __ddiv_rn(1.0, (double)nmat);
                    v[0] = __dmul_rn(s0, inv);
                    v[1] = __dmul_rn(s1, inv);
                    v[2] = __dmul_rn(s2, inv);
                }
            }
        }
        out[e * 3] = v[0];
        out[e * 3 + 1] = v[1];
        out[e * 3 + 2] = v[2];
    }
}

// restrict_l0_to_demag_grid (coarse_fft_demag.rs:256-290)
__global__ void k_restrict_l0(const double* __restrict__ l0, long long nx_l0, long long dnx, long long dny, long long r,
                              double* __restrict__ out) {
    const double inv_r2 = __ddiv_rn(1.0, (double)(r * r));
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < dnx * dny;
         e += (long long)gridDim.x * blockDim.x) {
        const long long id = e % dnx, jd = e / dnx;
        double s[3] = {0.0, 0.0, 0.0};
        for (long long fj = 0; fj < r; ++fj) {
            const long long row = (jd * r + fj) * nx_l0 + id * r;
            for (long long fi = 0; fi < r; ++fi)
#pragma unroll
                for (int c = 0; c < 3; ++c) s[c] = __dadd_rn(s[c], l0[(row + fi) * 3 + c]);
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) out[e * 3 + c] = __dmul_rn(s[c], inv_r2);
    }
}

// Bilinear samples of field f (fnx x fny, cell fdx x fdy) at the cell centres of an
// onx x ony grid with cells odx x ody (interpolate_demag_to_l0, coarse_fft_demag.rs:299-318;
// the coarse addend of amr/stepper.rs:826-834).
__global__ void k_sample_grid(const double* __restrict__ f, long long fnx, long long fny, double fdx, double fdy,
                              long long onx, long long ony, double odx, double ody, double* __restrict__ out) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < onx * ony;
         e += (long long)gridDim.x * blockDim.x) {
        const long long i = e % onx, j = e / onx;
        const double x = __dmul_rn(__dadd_rn((double)i, 0.5), odx);
        const double y = __dmul_rn(__dadd_rn((double)j, 0.5), ody);
        sample_bilinear(f, fnx, fny, fdx, fdy, x, y, out + e * 3);
    }
}

// sample_demag_to_patch (coarse_fft_demag.rs:327-340) for every patch cell incl.
// ghosts, at Patch2D::cell_center_xy (amr/patch.rs:377-387).
__global__ void k_sample_patches(const double* __restrict__ bc, long long nx, long long ny, double dx, double dy,
                                 const PatchDev* __restrict__ pd, int np, long long total, double* __restrict__ out) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = np - 1;   // last patch with out_off <= e
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (pd[mid].out_off <= e) lo = mid;
            else hi = mid - 1;
        }
        const PatchDev& p = pd[lo];
        const long long loc = e - p.out_off, i = loc % p.pnx, j = loc / p.pnx;
        const double fdx = __ddiv_rn(dx, (double)p.ratio), fdy = __ddiv_rn(dy, (double)p.ratio);
        const double gi0 = (double)(p.i0 * p.ratio), gj0 = (double)(p.j0 * p.ratio);
        const double li = __dsub_rn((double)i, (double)p.ghost), lj = __dsub_rn((double)j, (double)p.ghost);
        const double x = __dmul_rn(__dadd_rn(__dadd_rn(gi0, li), 0.5), fdx);
        const double y = __dmul_rn(__dadd_rn(__dadd_rn(gj0, lj), 0.5), fdy);
        sample_bilinear(bc, nx, ny, dx, dy, x, y, out + e * 3);
    }
}

__global__ void k_zero_vacuum(double* __restrict__ b, const unsigned char* __restrict__ mask, long long n) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        if (!mask[e]) b[e * 3] = b[e * 3 + 1] = b[e * 3 + 2] = 0.0;
}

bool is_pow2(long long r) { return r >= 1 && (r & (r - 1)) == 0; }

int validated_ratio(long long nx, long long ny, long long ratio) {
    // validated_ratio, coarse_fft_demag.rs:118-150
    if (ratio <= 1) return 1;
    if (nx % ratio != 0 || ny % ratio != 0) return 1;
    if (nx / ratio < 4 || ny / ratio < 4) return 1;
    return (int)ratio;
}

}  // namespace

struct llg_amr_demag {
    int device = 0;
    llg_grid base{};
    long long r = 1;
    llg_grid fft{};               // the grid the FFT runs on (base, or base / r)
    llg_demag_op* op = nullptr;
    cudaStream_t stream = nullptr;
    double* d_mc = nullptr;       // L0 m
    double* d_enh = nullptr;      // restricted L0 m
    double* d_bc = nullptr;       // L0 demag field
    double* d_dm = nullptr;       // demag-grid m (r > 1)
    double* d_db = nullptr;       // demag-grid field (r > 1)
    // per-call buffers, grown on demand
    unsigned char* d_staged = nullptr;
    size_t cap_staged = 0;
    unsigned char* h_staged = nullptr;   // pinned
    size_t cap_h_staged = 0;
    PatchDev* d_pd = nullptr;
    size_t cap_pd = 0;
    double* d_bp = nullptr;
    size_t cap_bp = 0;
};

namespace {

void amr_destroy(llg_amr_demag* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (void* p : {(void*)h->d_mc, (void*)h->d_enh, (void*)h->d_bc, (void*)h->d_dm, (void*)h->d_db,
                    (void*)h->d_staged, (void*)h->d_pd, (void*)h->d_bp})
        if (p) cudaFree(p);
    if (h->h_staged) cudaFreeHost(h->h_staged);
    if (h->op) llg_demag_op_destroy(h->op);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

template <typename T>
int grow(T** p, size_t* cap, size_t need) {
    if (need <= *cap) return LLG_OK;
    const size_t n = std::max(need, *cap * 2);
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    if (cudaMalloc(p, n * sizeof(T)) != cudaSuccess) return fail(LLG_ERR_OOM, "cudaMalloc of %zu bytes", n * sizeof(T));
    *cap = n;
    return LLG_OK;
}

int grow_host(unsigned char** p, size_t* cap, size_t need) {
    if (need <= *cap) return LLG_OK;
    if (*p) cudaFreeHost(*p);
    *p = nullptr;
    *cap = 0;
    if (cudaMallocHost(p, need) != cudaSuccess) return fail(LLG_ERR_OOM, "cudaMallocHost of %zu bytes", need);
    *cap = need;
    return LLG_OK;
}

long long patch_cells(const llg_amr_patch& p) {
    return (p.cny * p.ratio + 2 * p.ghost) * (p.cnx * p.ratio + 2 * p.ghost);
}

int check_patches(const llg_grid& base, int np, const llg_amr_patch* ps) {
    if (np < 0 || (np > 0 && !ps)) return fail(LLG_ERR_INVALID, "bad patch list");
    for (int q = 0; q < np; ++q) {
        const llg_amr_patch& p = ps[q];
        if (p.ratio < 1 || p.ghost < 0 || p.cnx < 1 || p.cny < 1 || p.i0 < 0 || p.j0 < 0 ||
            p.i0 + p.cnx > base.nx || p.j0 + p.cny > base.ny || !p.m)
            return fail(LLG_ERR_INVALID, "patch %d: rect outside the base grid, bad ratio/ghost or no m", q);
    }
    return LLG_OK;
}

// Stages the L0 m and the patches (fine m, masks, parent flags) into one pinned buffer,
// copies it and the descriptors to the device.  Returns the total patch cells.
int stage_inputs(llg_amr_demag* h, const double* m_coarse, int np, const llg_amr_patch* ps, long long* total_cells) {
    const long long n = h->base.nx * h->base.ny;
    std::vector<PatchDev> pd(np);
    size_t doubles = 0, bytes_flags = 0;
    long long cells = 0;
    for (int q = 0; q < np; ++q) {
        const long long pc = patch_cells(ps[q]);
        doubles += 3 * (size_t)pc;
        if (ps[q].geom_mask_fine) bytes_flags += (size_t)pc;
        if (ps[q].parent_material) bytes_flags += (size_t)(ps[q].cnx * ps[q].cny);
        cells += pc;
    }
    const size_t bytes = doubles * sizeof(double) + bytes_flags;
    int rc;
    if ((rc = grow_host(&h->h_staged, &h->cap_h_staged, std::max<size_t>(bytes, 64)))) return rc;
    if ((rc = grow(&h->d_staged, &h->cap_staged, std::max<size_t>(bytes, 64)))) return rc;
    if ((rc = grow(&h->d_pd, &h->cap_pd, std::max<size_t>(np, 1)))) return rc;
    double* dst = reinterpret_cast<double*>(h->h_staged);
    size_t off_d = 0, off_b = doubles * sizeof(double);
    long long out_off = 0;
    for (int q = 0; q < np; ++q) {
        const llg_amr_patch& p = ps[q];
        const long long pc = patch_cells(p);
        PatchDev& d = pd[q];
        d.i0 = p.i0;
        d.j0 = p.j0;
        d.cnx = p.cnx;
        d.cny = p.cny;
        d.ratio = p.ratio;
        d.ghost = p.ghost;
        d.pnx = p.cnx * p.ratio + 2 * p.ghost;
        d.pny = p.cny * p.ratio + 2 * p.ghost;
        d.m_off = (long long)off_d;
        std::memcpy(dst + off_d, p.m, sizeof(double) * 3 * (size_t)pc);
        off_d += 3 * (size_t)pc;
        d.mask_off = -1;
        if (p.geom_mask_fine) {
            d.mask_off = (long long)off_b;
            std::memcpy(h->h_staged + off_b, p.geom_mask_fine, (size_t)pc);
            off_b += (size_t)pc;
        }
        d.pm_off = -1;
        if (p.parent_material) {
            d.pm_off = (long long)off_b;
            std::memcpy(h->h_staged + off_b, p.parent_material, (size_t)(p.cnx * p.cny));
            off_b += (size_t)(p.cnx * p.cny);
        }
        d.out_off = out_off;
        out_off += pc;
    }
    AMR_TRY(cudaMemcpyAsync(h->d_mc, m_coarse, sizeof(double) * 3 * (size_t)n, cudaMemcpyHostToDevice, h->stream));
    if (bytes) AMR_TRY(cudaMemcpyAsync(h->d_staged, h->h_staged, bytes, cudaMemcpyHostToDevice, h->stream));
    if (np) AMR_TRY(cudaMemcpyAsync(h->d_pd, pd.data(), sizeof(PatchDev) * np, cudaMemcpyHostToDevice, h->stream));
    // the staging buffers are reused by the next call: finish the copies first
    AMR_TRY(cudaStreamSynchronize(h->stream));
    *total_cells = cells;
    return LLG_OK;
}

}  // namespace

extern "C" {

int64_t llg_amr_validated_ratio(int64_t nx, int64_t ny, int64_t ratio) { return validated_ratio(nx, ny, ratio); }

int64_t llg_amr_patch_cells(const llg_amr_patch* p) { return p ? patch_cells(*p) : 0; }

int llg_amr_demag_create(llg_ctx* ctx, const llg_grid* base, int64_t coarsen_ratio, llg_amr_demag** out) {
    if (!ctx || !base || !out) return fail(LLG_ERR_INVALID, "null argument");
    if (base->nx < 1 || base->ny < 1 || !(base->dx > 0) || !(base->dy > 0) || !(base->dz > 0))
        return fail(LLG_ERR_INVALID, "bad base grid");
    llg_amr_demag* h = new llg_amr_demag();
    h->device = llg::ctx_device(ctx);
    h->base = *base;
    // demag_coarsen_ratio (:82-111): a ratio that is not a power of two means 1
    h->r = is_pow2(coarsen_ratio) ? validated_ratio(base->nx, base->ny, coarsen_ratio) : 1;
    h->fft = *base;
    if (h->r > 1) {
        h->fft.nx = base->nx / h->r;
        h->fft.ny = base->ny / h->r;
        h->fft.dx = base->dx * (double)h->r;
        h->fft.dy = base->dy * (double)h->r;
    }
    auto bail = [&](int rc) {
        amr_destroy(h);
        return rc;
    };
    if (cudaSetDevice(h->device) != cudaSuccess) return bail(fail(LLG_ERR_CUDA, "cudaSetDevice failed"));
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(LLG_ERR_CUDA, "stream"));
    int rc = llg_demag_op_create(ctx, &h->fft, 0, 0, nullptr, nullptr, &h->op);
    if (rc) return bail(rc);
    const size_t n = (size_t)(base->nx * base->ny), nd = (size_t)(h->fft.nx * h->fft.ny);
    if (cudaMalloc(&h->d_mc, 3 * n * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&h->d_enh, 3 * n * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&h->d_bc, 3 * n * sizeof(double)) != cudaSuccess)
        return bail(fail(LLG_ERR_OOM, "cudaMalloc"));
    if (h->r > 1 && (cudaMalloc(&h->d_dm, 3 * nd * sizeof(double)) != cudaSuccess ||
                     cudaMalloc(&h->d_db, 3 * nd * sizeof(double)) != cudaSuccess))
        return bail(fail(LLG_ERR_OOM, "cudaMalloc"));
    *out = h;
    return LLG_OK;
}

int llg_amr_demag_ratio(const llg_amr_demag* h, int64_t* ratio) {
    if (!h || !ratio) return fail(LLG_ERR_INVALID, "null argument");
    *ratio = h->r;
    return LLG_OK;
}

int llg_amr_demag_destroy(llg_amr_demag* h) {
    amr_destroy(h);
    return LLG_OK;
}

int llg_amr_restrict_m(llg_amr_demag* h, const double* m_coarse, int32_t n_patches, const llg_amr_patch* patches,
                       double* out) {
    if (!h || !m_coarse || !out) return fail(LLG_ERR_INVALID, "null argument");
    int rc;
    if ((rc = check_patches(h->base, n_patches, patches))) return rc;
    AMR_TRY(cudaSetDevice(h->device));
    long long cells = 0;
    if ((rc = stage_inputs(h, m_coarse, n_patches, patches, &cells))) return rc;
    k_restrict_patches<<<kGrid, 256, 0, h->stream>>>(h->d_mc, h->base.nx, h->base.ny, h->d_pd, n_patches,
                                                      h->d_staged, h->d_enh);
    AMR_TRY(cudaGetLastError());
    const size_t n = (size_t)(h->base.nx * h->base.ny);
    AMR_TRY(cudaMemcpyAsync(out, h->d_enh, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    AMR_TRY(cudaStreamSynchronize(h->stream));
    return LLG_OK;
}

int llg_coarse_fft_demag(llg_amr_demag* h, const llg_material* mat, const double* m_coarse, int32_t n_patches,
                         const llg_amr_patch* patches, double* b_coarse, double* b_patches) {
    if (!h || !mat || !m_coarse || !b_coarse || (n_patches > 0 && !b_patches))
        return fail(LLG_ERR_INVALID, "null argument");
    int rc;
    if ((rc = check_patches(h->base, n_patches, patches))) return rc;
    AMR_TRY(cudaSetDevice(h->device));
    const long long n = h->base.nx * h->base.ny;
    if (!mat->demag) {
        // no demag: zero L0 field and no patch fields (empty vectors in the reference)
        std::memset(b_coarse, 0, sizeof(double) * 3 * (size_t)n);
        return LLG_OK;
    }
    long long cells = 0;
    if ((rc = stage_inputs(h, m_coarse, n_patches, patches, &cells))) return rc;
    k_restrict_patches<<<kGrid, 256, 0, h->stream>>>(h->d_mc, h->base.nx, h->base.ny, h->d_pd, n_patches,
                                                      h->d_staged, h->d_enh);
    AMR_TRY(cudaGetLastError());
    if (h->r <= 1) {
        if ((rc = llg::demag_op_apply_device(h->op, mat->ms, h->d_enh, h->d_bc, h->stream))) return rc;
    } else {
        k_restrict_l0<<<kGrid, 256, 0, h->stream>>>(h->d_enh, h->base.nx, h->fft.nx, h->fft.ny, h->r, h->d_dm);
        AMR_TRY(cudaGetLastError());
        if ((rc = llg::demag_op_apply_device(h->op, mat->ms, h->d_dm, h->d_db, h->stream))) return rc;
        k_sample_grid<<<kGrid, 256, 0, h->stream>>>(h->d_db, h->fft.nx, h->fft.ny, h->fft.dx, h->fft.dy, h->base.nx,
                                                     h->base.ny, h->base.dx, h->base.dy, h->d_bc);
        AMR_TRY(cudaGetLastError());
    }
    if (cells > 0) {
        if ((rc = grow(&h->d_bp, &h->cap_bp, 3 * (size_t)cells))) return rc;
        k_sample_patches<<<kGrid, 256, 0, h->stream>>>(h->d_bc, h->base.nx, h->base.ny, h->base.dx, h->base.dy,
                                                        h->d_pd, n_patches, cells, h->d_bp);
        AMR_TRY(cudaGetLastError());
        AMR_TRY(cudaMemcpyAsync(b_patches, h->d_bp, 3 * (size_t)cells * sizeof(double), cudaMemcpyDeviceToHost,
                                h->stream));
    }
    AMR_TRY(cudaMemcpyAsync(b_coarse, h->d_bc, 3 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    AMR_TRY(cudaStreamSynchronize(h->stream));
    return LLG_OK;
}

int llg_amr_allfft_demag(llg_demag_op* fine_op, const llg_material* mat, const double* m_fine,
                         const uint8_t* fine_mask, const llg_grid* base, double* b_fine, double* b_coarse) {
    if (!fine_op || !mat || !m_fine || !base || !b_fine || !b_coarse) return fail(LLG_ERR_INVALID, "null argument");
    int device = 0, pbx = 0, pby = 0;
    llg_grid fg{};
    llg::demag_op_info(fine_op, &device, &fg, &pbx, &pby);
    if (pbx || pby) return fail(LLG_ERR_INVALID, "the AllFft demag uses open boundaries (pbc 0, 0)");
    if (base->nx < 1 || base->ny < 1 || !(base->dx > 0) || !(base->dy > 0)) return fail(LLG_ERR_INVALID, "bad base grid");
    AMR_TRY(cudaSetDevice(device));
    const long long nf = fg.nx * fg.ny, nb = base->nx * base->ny;
    if (!mat->demag) {
        // compute_demag_field_pbc leaves zero without Material::demag
        std::memset(b_fine, 0, sizeof(double) * 3 * (size_t)nf);
        std::memset(b_coarse, 0, sizeof(double) * 3 * (size_t)nb);
        return LLG_OK;
    }
    cudaStream_t s = nullptr;
    AMR_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    double* d_f = nullptr;
    double* d_c = nullptr;
    unsigned char* d_mask = nullptr;
    int rc = LLG_OK;
    auto done = [&](int code) {
        cudaStreamSynchronize(s);
        if (d_f) cudaFreeAsync(d_f, s);
        if (d_c) cudaFreeAsync(d_c, s);
        if (d_mask) cudaFreeAsync(d_mask, s);
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
        return code;
    };
    if (cudaMallocAsync(&d_f, 3 * (size_t)nf * sizeof(double), s) != cudaSuccess ||
        cudaMallocAsync(&d_c, 3 * (size_t)nb * sizeof(double), s) != cudaSuccess ||
        (fine_mask && cudaMallocAsync(&d_mask, (size_t)nf, s) != cudaSuccess))
        return done(fail(LLG_ERR_OOM, "cudaMallocAsync"));
    if (cudaMemcpyAsync(d_f, m_fine, 3 * (size_t)nf * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        (fine_mask && cudaMemcpyAsync(d_mask, fine_mask, (size_t)nf, cudaMemcpyHostToDevice, s) != cudaSuccess))
        return done(fail(LLG_ERR_CUDA, "input copy"));
    if ((rc = llg::demag_op_apply_device(fine_op, mat->ms, d_f, d_f, s))) return done(rc);
    if (fine_mask) k_zero_vacuum<<<kGrid, 256, 0, s>>>(d_f, d_mask, nf);
    k_sample_grid<<<kGrid, 256, 0, s>>>(d_f, fg.nx, fg.ny, fg.dx, fg.dy, base->nx, base->ny, base->dx, base->dy, d_c);
    if (cudaGetLastError() != cudaSuccess) return done(fail(LLG_ERR_CUDA, "sampling kernels"));
    if (cudaMemcpyAsync(b_fine, d_f, 3 * (size_t)nf * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(b_coarse, d_c, 3 * (size_t)nb * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return done(fail(LLG_ERR_CUDA, "output copy"));
    if (cudaStreamSynchronize(s) != cudaSuccess) return done(fail(LLG_ERR_CUDA, "AllFft demag"));
    return done(LLG_OK);
}

// The AllFft demag on device arrays: no host transfer and no allocation (the
// operator's own buffers hold the transforms), asynchronous on `stream`.
int llg_amr_allfft_demag_device(llg_demag_op* fine_op, const llg_material* mat, const double* d_m_fine,
                                const uint8_t* d_fine_mask, const llg_grid* base, double* d_b_fine,
                                double* d_b_coarse, void* stream) {
    if (!fine_op || !mat || !d_m_fine || !base || !d_b_fine || !d_b_coarse) return fail(LLG_ERR_INVALID, "null argument");
    int device = 0, pbx = 0, pby = 0;
    llg_grid fg{};
    llg::demag_op_info(fine_op, &device, &fg, &pbx, &pby);
    if (pbx || pby) return fail(LLG_ERR_INVALID, "the AllFft demag uses open boundaries (pbc 0, 0)");
    if (base->nx < 1 || base->ny < 1 || !(base->dx > 0) || !(base->dy > 0)) return fail(LLG_ERR_INVALID, "bad base grid");
    AMR_TRY(cudaSetDevice(device));
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const long long nf = fg.nx * fg.ny, nb = base->nx * base->ny;
    if (!mat->demag) {
        AMR_TRY(cudaMemsetAsync(d_b_fine, 0, sizeof(double) * 3 * (size_t)nf, s));
        AMR_TRY(cudaMemsetAsync(d_b_coarse, 0, sizeof(double) * 3 * (size_t)nb, s));
        return LLG_OK;
    }
    int rc;
    if ((rc = llg::demag_op_apply_device(fine_op, mat->ms, d_m_fine, d_b_fine, s))) return rc;
    if (d_fine_mask) k_zero_vacuum<<<kGrid, 256, 0, s>>>(d_b_fine, d_fine_mask, nf);
    k_sample_grid<<<kGrid, 256, 0, s>>>(d_b_fine, fg.nx, fg.ny, fg.dx, fg.dy, base->nx, base->ny, base->dx, base->dy,
                                        d_b_coarse);
    if (cudaGetLastError() != cudaSuccess) return fail(LLG_ERR_CUDA, "AllFft demag kernels");
    return LLG_OK;
}

}  // extern "C"
