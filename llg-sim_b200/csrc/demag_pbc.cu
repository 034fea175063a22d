// demag_pbc.cu — demag field with periodic images, and the LLGDMAG v2 k-space
// kernel cache of the reference.
//
// Demag2D (demag_fft_uniform.rs:434-770) for pbc_x / pbc_y periodic images: no
// padding in a periodic direction (px = pbc_x ? nx : 2 nx, likewise py), the
// real-space kernel summed over the image ranges into wrapped bins
// (build_kernel_realspace_pbc, :941-1005), then the full complex px x py FFT
// convolution of add_field (:636-769).  Everything is FP64: this is the
// field-only entry compute_demag_field_pbc (demag.rs:146-156), which the
// reference's steppers do not call.  Transforms use the shared-memory FP64 FFT
// (one block per row or column), so px and py are limited to 4096.
//
// The k-space planes are stored unscaled exactly as write_kernel_kspace writes
// them (:279-319), so a cache file written here is read by the reference and
// one written by the reference is read here.
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "../../include/llg_b200.h"
#include "build_api.h"
#include "fft_smem.cuh"

namespace llg {
int ctx_device(const llg_ctx* c);
}

struct llg_demag_op {
    int device = 0;
    int nx = 0, ny = 0, pbc_x = 0, pbc_y = 0, px = 0, py = 0;
    double dx = 0, dy = 0, dz = 0;
    llg::cx<double>* K = nullptr;    // [4][py][px] unscaled kernel spectrum
    llg::cx<double>* M = nullptr;    // [3][py][px] work planes
    double* stage = nullptr;         // [nx*ny*3] AoS staging
    llg::cx<double>* twx = nullptr;
    llg::cx<double>* twy = nullptr;
};

namespace {

using llg::cx;
using llg::mkc;

constexpr double kAccuracy = 10.0;   // DEMAG_ACCURACY, demag_fft_uniform.rs:432

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    llg_set_error_message(buf);
    return code;
}

#define PBC_TRY(x)                                                                                           \
    do {                                                                                                     \
        cudaError_t _e = (x);                                                                                \
        if (_e != cudaSuccess)                                                                               \
            return fail(_e == cudaErrorMemoryAllocation ? LLG_ERR_OOM : LLG_ERR_CUDA, "%s: %s", #x,          \
                        cudaGetErrorString(_e));                                                             \
    } while (0)

__global__ void k_pbc_pack(const double* __restrict__ m, int nx, int ny, int px, int py, double ms,
                           cx<double>* __restrict__ M) {
    const long long np = (long long)px * py;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < np; e += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(e % px), iy = (int)(e / px);
        double v[3] = {0.0, 0.0, 0.0};
        if (ix < nx && iy < ny) {
            const double* mm = m + ((long long)iy * nx + ix) * 3;
            v[0] = ms * mm[0];
            v[1] = ms * mm[1];
            v[2] = ms * mm[2];
        }
        for (int c = 0; c < 3; ++c) M[c * np + e] = mkc(v[c], 0.0);
    }
}

// B = K M per bin with complex products, demag_fft_uniform.rs:700-742
__global__ void k_pbc_multiply(const cx<double>* __restrict__ K, long long np, cx<double>* __restrict__ M) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < np; e += (long long)gridDim.x * blockDim.x) {
        const cx<double> mx = M[e], my = M[np + e], mz = M[2 * np + e];
        const cx<double> kxx = K[e], kxy = K[np + e], kyy = K[2 * np + e], kzz = K[3 * np + e];
        M[e] = llg::cmul(kxx, mx) + llg::cmul(kxy, my);
        M[np + e] = llg::cmul(kxy, mx) + llg::cmul(kyy, my);
        M[2 * np + e] = llg::cmul(kzz, mz);
    }
}

__global__ void k_pbc_extract(const cx<double>* __restrict__ M, int nx, int ny, int px, int py, double scale,
                              double* __restrict__ b) {
    const long long np = (long long)px * py, n = (long long)nx * ny;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long j = e / nx, i = e % nx, src = j * px + i;
        for (int c = 0; c < 3; ++c) b[e * 3 + c] = M[c * np + src].re * scale;
    }
}

}  // namespace

namespace llg {

int demag_op_apply_device(llg_demag_op* op, double ms, const double* d_m_aos, double* d_b_aos, cudaStream_t s) {
    const long long np = (long long)op->px * op->py;
    k_pbc_pack<<<1184, 256, 0, s>>>(d_m_aos, op->nx, op->ny, op->px, op->py, ms, op->M);
    PBC_TRY(cudaGetLastError());
    PBC_TRY(llg::launch_fft_strided<double>(op->M, op->px, op->twx, 1, op->py, op->px, 3, np, false, s));
    PBC_TRY(llg::launch_fft_strided<double>(op->M, op->py, op->twy, op->px, op->px, 1, 3, np, false, s));
    k_pbc_multiply<<<1184, 256, 0, s>>>(op->K, np, op->M);
    PBC_TRY(cudaGetLastError());
    PBC_TRY(llg::launch_fft_strided<double>(op->M, op->px, op->twx, 1, op->py, op->px, 3, np, true, s));
    PBC_TRY(llg::launch_fft_strided<double>(op->M, op->py, op->twy, op->px, op->px, 1, 3, np, true, s));
    k_pbc_extract<<<1184, 256, 0, s>>>(op->M, op->nx, op->ny, op->px, op->py, 1.0 / (double)np, d_b_aos);
    PBC_TRY(cudaGetLastError());
    return LLG_OK;
}

void demag_op_info(const llg_demag_op* op, int* device, llg_grid* g, int* pbc_x, int* pbc_y) {
    *device = op->device;
    g->nx = op->nx;
    g->ny = op->ny;
    g->dx = op->dx;
    g->dy = op->dy;
    g->dz = op->dz;
    *pbc_x = op->pbc_x;
    *pbc_y = op->pbc_y;
}

}  // namespace llg

namespace {

// Rust's `{:.3e}`: mantissa with three decimals, exponent without sign padding.
std::string rust_exp3(double v) {
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%.3e", v);
    std::string s(buf);
    const size_t p = s.find('e');
    if (p == std::string::npos) return s;
    const int ex = std::atoi(s.c_str() + p + 1);
    return s.substr(0, p) + "e" + std::to_string(ex);
}

std::string cache_name(int nx, int ny, int pbc_x, int pbc_y, int px, int py, double dx, double dy, double dz) {
    // demag_cache_path, demag_fft_uniform.rs:261-277
    char acc[32];
    std::snprintf(acc, sizeof(acc), "%.2f", kAccuracy);
    return "out/demag_cache/demag_kernel_nx" + std::to_string(nx) + "_ny" + std::to_string(ny) + "_pbcx" +
           std::to_string(pbc_x) + "_pbcy" + std::to_string(pbc_y) + "_px" + std::to_string(px) + "_py" +
           std::to_string(py) + "_dx" + rust_exp3(dx) + "_dy" + rust_exp3(dy) + "_dz" + rust_exp3(dz) + "_acc" + acc +
           ".bin";
}

#pragma pack(push, 1)
struct CacheHeader {          // KernelCacheHeader, demag_fft_uniform.rs:207-221 (little endian)
    char magic[8];
    uint32_t version, nx, ny, pbc_x, pbc_y, px, py;
    double dx, dy, dz, accuracy;
};
#pragma pack(pop)
static_assert(sizeof(CacheHeader) == 68, "LLGDMAG v2 header is 68 bytes");

CacheHeader make_header(const llg_demag_op* op) {
    CacheHeader h;
    std::memcpy(h.magic, "LLGDMAG\0", 8);
    h.version = 2;
    h.nx = (uint32_t)op->nx;
    h.ny = (uint32_t)op->ny;
    h.pbc_x = (uint32_t)op->pbc_x;
    h.pbc_y = (uint32_t)op->pbc_y;
    h.px = (uint32_t)op->px;
    h.py = (uint32_t)op->py;
    h.dx = op->dx;
    h.dy = op->dy;
    h.dz = op->dz;
    h.accuracy = kAccuracy;
    return h;
}

// try_load_kernel_kspace (:322-429): false (and nothing changed) on any mismatch or short file.
bool try_load(llg_demag_op* op, const char* path) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    CacheHeader h;
    const CacheHeader want = make_header(op);
    bool ok = std::fread(&h, sizeof(h), 1, f) == 1 && std::memcmp(h.magic, want.magic, 8) == 0 && h.version == 2 &&
              h.nx == want.nx && h.ny == want.ny && h.pbc_x == want.pbc_x && h.pbc_y == want.pbc_y &&
              h.px == want.px && h.py == want.py && h.dx == want.dx && h.dy == want.dy && h.dz == want.dz &&
              h.accuracy == want.accuracy;
    const size_t np = (size_t)op->px * op->py;
    std::vector<cx<double>> host;
    if (ok) {
        host.resize(4 * np);
        ok = std::fread(host.data(), sizeof(cx<double>), host.size(), f) == host.size();
    }
    std::fclose(f);
    if (!ok) return false;
    return cudaMemcpy(op->K, host.data(), host.size() * sizeof(cx<double>), cudaMemcpyHostToDevice) == cudaSuccess;
}

// fs::create_dir_all of the file's parent directory, as write_kernel_kspace does
void make_parent_dirs(const char* path) {
    std::string p(path);
    for (size_t i = 1; i < p.size(); ++i)
        if (p[i] == '/') mkdir(p.substr(0, i).c_str(), 0777);
}

int save(const llg_demag_op* op, const char* path) {
    const size_t np = (size_t)op->px * op->py;
    make_parent_dirs(path);
    std::vector<cx<double>> host(4 * np);
    PBC_TRY(cudaMemcpy(host.data(), op->K, host.size() * sizeof(cx<double>), cudaMemcpyDeviceToHost));
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(LLG_ERR_INVALID, "cannot open %s for writing", path);
    const CacheHeader h = make_header(op);
    bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1 &&
              std::fwrite(host.data(), sizeof(cx<double>), host.size(), f) == host.size();
    ok = (std::fclose(f) == 0) && ok;
    return ok ? LLG_OK : fail(LLG_ERR_INVALID, "short write to %s", path);
}

void destroy(llg_demag_op* op) {
    if (!op) return;
    cudaSetDevice(op->device);
    cudaFree(op->K);
    cudaFree(op->M);
    cudaFree(op->stage);
    cudaFree(op->twx);
    cudaFree(op->twy);
    delete op;
}

}  // namespace

extern "C" {

int llg_demag_cache_filename(const llg_grid* g, int64_t pbc_x, int64_t pbc_y, char* buf, int64_t len) {
    if (!g || !buf || len <= 0) return fail(LLG_ERR_INVALID, "null argument");
    const int px = pbc_x > 0 ? (int)g->nx : 2 * (int)g->nx, py = pbc_y > 0 ? (int)g->ny : 2 * (int)g->ny;
    const std::string s = cache_name((int)g->nx, (int)g->ny, (int)pbc_x, (int)pbc_y, px, py, g->dx, g->dy, g->dz);
    if ((int64_t)s.size() + 1 > len) return fail(LLG_ERR_INVALID, "buffer of %lld bytes too small", (long long)len);
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return LLG_OK;
}

int llg_demag_op_create(llg_ctx* ctx, const llg_grid* g, int64_t pbc_x, int64_t pbc_y, const char* cache_path,
                        int32_t* loaded, llg_demag_op** out) {
    if (!ctx || !g || !out) return fail(LLG_ERR_INVALID, "null argument");
    if (g->nx < 1 || g->ny < 1 || pbc_x < 0 || pbc_y < 0 || pbc_x > 4096 || pbc_y > 4096 || !(g->dx > 0) ||
        !(g->dy > 0) || !(g->dz > 0))
        return fail(LLG_ERR_INVALID, "bad grid or image counts");
    const long long px = pbc_x > 0 ? g->nx : 2 * g->nx, py = pbc_y > 0 ? g->ny : 2 * g->ny;
    if (px > 4096 || py > 4096)
        return fail(LLG_ERR_INVALID, "padded size %lldx%lld exceeds 4096 (shared-memory FFT limit)", px, py);
    const long long sx = pbc_x == 0 ? g->nx - 1 : g->nx * pbc_x - 1, sy = pbc_y == 0 ? g->ny - 1 : g->ny * pbc_y - 1;
    if ((2 * sx + 1) * (2 * sy + 1) > (1LL << 26))
        return fail(LLG_ERR_INVALID, "%lld periodic-image displacements exceed 2^26",
                    (long long)((2 * sx + 1) * (2 * sy + 1)));
    llg_demag_op* op = new llg_demag_op();
    op->device = llg::ctx_device(ctx);
    op->nx = (int)g->nx;
    op->ny = (int)g->ny;
    op->pbc_x = (int)pbc_x;
    op->pbc_y = (int)pbc_y;
    op->px = (int)px;
    op->py = (int)py;
    op->dx = g->dx;
    op->dy = g->dy;
    op->dz = g->dz;
    const size_t np = (size_t)px * py;
    auto bail = [&](int rc) {
        destroy(op);
        return rc;
    };
    if (cudaSetDevice(op->device) != cudaSuccess) return bail(fail(LLG_ERR_CUDA, "cudaSetDevice failed"));
    if (cudaMalloc(&op->K, 4 * np * sizeof(cx<double>)) != cudaSuccess ||
        cudaMalloc(&op->M, 3 * np * sizeof(cx<double>)) != cudaSuccess ||
        cudaMalloc(&op->stage, 3 * (size_t)g->nx * g->ny * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&op->twx, 2 * (size_t)px * sizeof(cx<double>)) != cudaSuccess ||
        cudaMalloc(&op->twy, 2 * (size_t)py * sizeof(cx<double>)) != cudaSuccess)
        return bail(fail(LLG_ERR_OOM, "cudaMalloc failed for a %lldx%lld demag operator", px, py));
    if (llg::launch_twiddles(op->twx, 2 * op->px, true, 0) != cudaSuccess ||
        llg::launch_twiddles(op->twy, 2 * op->py, true, 0) != cudaSuccess)
        return bail(fail(LLG_ERR_CUDA, "twiddle tables"));
    bool hit = cache_path && try_load(op, cache_path);
    if (!hit) {
        cudaError_t e = llg::build_demag_kernel_pbc(op->nx, op->ny, op->dx, op->dy, op->dz, op->pbc_x, op->pbc_y,
                                                    op->K, 0);
        if (e != cudaSuccess) return bail(fail(LLG_ERR_CUDA, "kernel build: %s", cudaGetErrorString(e)));
        if (cache_path && save(op, cache_path) != LLG_OK) {
            // like the reference, a cache that cannot be written is not an error
        }
    }
    if (cudaDeviceSynchronize() != cudaSuccess) return bail(fail(LLG_ERR_CUDA, "demag operator set-up"));
    if (loaded) *loaded = hit ? 1 : 0;
    *out = op;
    return LLG_OK;
}

int llg_demag_op_destroy(llg_demag_op* op) {
    destroy(op);
    return LLG_OK;
}

int llg_demag_op_field(llg_demag_op* op, double ms, const double* m_aos, double* b_aos) {
    if (!op || !m_aos || !b_aos) return fail(LLG_ERR_INVALID, "null argument");
    PBC_TRY(cudaSetDevice(op->device));
    const long long n = (long long)op->nx * op->ny;
    PBC_TRY(cudaMemcpy(op->stage, m_aos, sizeof(double) * 3 * (size_t)n, cudaMemcpyHostToDevice));
    int rc = llg::demag_op_apply_device(op, ms, op->stage, op->stage, 0);
    if (rc) return rc;
    PBC_TRY(cudaMemcpy(b_aos, op->stage, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToHost));
    return LLG_OK;
}

int llg_demag_op_kspace(llg_demag_op* op, double* out) {
    if (!op || !out) return fail(LLG_ERR_INVALID, "null argument");
    PBC_TRY(cudaSetDevice(op->device));
    PBC_TRY(cudaMemcpy(out, op->K, 4 * (size_t)op->px * op->py * sizeof(cx<double>), cudaMemcpyDeviceToHost));
    return LLG_OK;
}

int llg_demag_op_save(llg_demag_op* op, const char* path) {
    if (!op || !path) return fail(LLG_ERR_INVALID, "null argument");
    PBC_TRY(cudaSetDevice(op->device));
    return save(op, path);
}

}  // extern "C"
