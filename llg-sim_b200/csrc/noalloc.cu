// noalloc.cu — demag field of one film without any device allocation.
//
// Some callers cannot allocate device memory when they need the field: a host
// framework that owns every device allocation through its own pool, a
// real-time loop that must not pay allocation latency, or code running where
// cudaMalloc is not permitted.  llg_demag_field_noalloc serves them: the
// caller passes device pointers for the magnetisation, the kernel planes and
// the output; the spectrum scratch and the twiddle tables live in one
// file-scope static device array of kScratchBytes (every GPU that loads this
// library holds that array until the process exits).
//
// Same algorithm as the three evaluation passes of field_kernels.cuh (zero-
// padded FFT convolution, demag_fft_uniform.rs:636-769): pruned R2C rows ->
// per-column transform, multiply by the real kernel planes, inverse -> C2R rows.
#include <cstdio>
#include <mutex>

#include "../../include/llg_b200.h"
#include "build_api.h"
#include "fft_smem.cuh"

namespace llg {
namespace noalloc {

constexpr size_t kScratchBytes = size_t(32) << 20;  // 32 MiB
constexpr int kMaxDevices = 64;
constexpr int kT = 2;          // rows per block
constexpr int kThreads = 256;

// The shared scratch.  In host code this name is only a stand-in for the
// device array; kernels receive its device address from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {nullptr};

inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

__global__ void k_na_twiddles(cx<float>* tw_row, int nx, cx<float>* tw_col, int ny) {
    const int total = 2 * nx + 2 * ny;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const bool row = e < 2 * nx;
        const int k = row ? e : e - 2 * nx;
        const int L2 = row ? 2 * nx : 2 * ny;
        double s, c;
        sincospi(2.0 * (double)k / (double)L2, &s, &c);
        (row ? tw_row : tw_col)[k] = mkc((float)c, (float)(-s));
    }
}

// Rows j0..j0+kT-1: M = Ms*m, pruned R2C along x, Hermitian bins to X[c][kx][j].
__global__ void __launch_bounds__(kThreads) k_na_rows_forward(int nx, int ny, float ms, const float* __restrict__ m,
                                                              cx<float>* __restrict__ X,
                                                              const cx<float>* __restrict__ tw, FftPlan plan) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L = nx, G = kT + (kT + 1) / 2, n = nx * ny, K1 = nx + 1, L2 = 2 * nx;
    cx<float>* A = reinterpret_cast<cx<float>*>(smem_raw);
    cx<float>* B = A + 2 * G * L;
    const int j0 = blockIdx.x * kT;
    for (int e = threadIdx.x; e < kT * nx; e += blockDim.x) {
        const int r = e / nx, i = e - r * nx, j = j0 + r;
        float v0 = 0.f, v1 = 0.f, v2 = 0.f;
        if (j < ny) {
            const int idx = j * nx + i;
            v0 = m[idx]; v1 = m[n + idx]; v2 = m[2 * n + idx];
        }
        A[(2 * r) * L + i] = mkc(ms * v0, ms * v1);
        cx<float>* zp = &A[(2 * (kT + r / 2)) * L + i];
        if ((r & 1) == 0) zp->re = ms * v2;
        else zp->im = ms * v2;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < G * L; e += blockDim.x) {
        const int g = e / L, i = e - g * L;
        A[(2 * g + 1) * L + i] = cmul(A[(2 * g) * L + i], tw[i]);
    }
    __syncthreads();
    cx<float>* res = fft_smem<float>(A, B, 2 * G, plan, tw, false);
    for (int e = threadIdx.x; e < 3 * K1 * kT; e += blockDim.x) {
        const int r = e % kT, rest = e / kT;
        const int k = rest % K1, c = rest / K1;
        const int j = j0 + r;
        if (j >= ny) continue;
        const int g = c < 2 ? r : kT + r / 2;
        const int half = c < 2 ? c : (r & 1);
        const int km = (L2 - k) % L2;
        const cx<float> zk = res[(2 * g + (k & 1)) * L + (k >> 1)];
        const cx<float> zm = res[(2 * g + (km & 1)) * L + (km >> 1)];
        X[(c * K1 + k) * ny + j] = half == 0 ? mkc(0.5f * (zk.re + zm.re), 0.5f * (zk.im - zm.im))
                                             : mkc(0.5f * (zk.im + zm.im), 0.5f * (zm.re - zk.re));
    }
}

// One kx column: pruned y transform, kernel multiply, pruned inverse.
// kp: FP64 kernel planes [4][ny+1][nx+1] (xx, xy, yy, zz), unscaled.
__global__ void __launch_bounds__(kThreads) k_na_column(int nx, int ny, const double* __restrict__ kp, double scale,
                                                        cx<float>* __restrict__ X, const cx<float>* __restrict__ tw,
                                                        FftPlan plan) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L = ny, K1 = nx + 1, kx = blockIdx.x;
    const size_t plane = (size_t)(ny + 1) * (nx + 1);
    cx<float>* A = reinterpret_cast<cx<float>*>(smem_raw);
    cx<float>* B = A + 6 * L;
    for (int e = threadIdx.x; e < 3 * L; e += blockDim.x) {
        const int c = e / L, y = e - c * L;
        const cx<float> x = X[(c * K1 + kx) * ny + y];
        A[(2 * c) * L + y] = x;
        A[(2 * c + 1) * L + y] = cmul(x, tw[y]);
    }
    __syncthreads();
    cx<float>* res = fft_smem<float>(A, B, 6, plan, tw, false);
    for (int e = threadIdx.x; e < 2 * L; e += blockDim.x) {
        const int par = e / L, kk = e - par * L;
        const int ky = 2 * kk + par;
        const int kyf = ky <= ny ? ky : 2 * ny - ky;
        const size_t o = (size_t)kyf * (nx + 1) + kx;
        const float kxx = (float)(kp[o] * scale), kyy = (float)(kp[2 * plane + o] * scale);
        const float kzz = (float)(kp[3 * plane + o] * scale);
        const float kxy = (float)(kp[plane + o] * scale) * (ky <= ny ? 1.f : -1.f);
        const cx<float> Mx = res[(0 + par) * L + kk], My = res[(2 + par) * L + kk], Mz = res[(4 + par) * L + kk];
        res[(0 + par) * L + kk] = mkc(kxx * Mx.re + kxy * My.re, kxx * Mx.im + kxy * My.im);
        res[(2 + par) * L + kk] = mkc(kxy * Mx.re + kyy * My.re, kxy * Mx.im + kyy * My.im);
        res[(4 + par) * L + kk] = mkc(kzz * Mz.re, kzz * Mz.im);
    }
    __syncthreads();
    cx<float>* other = res == A ? B : A;
    cx<float>* res2 = fft_smem<float>(res, other, 6, plan, tw, true);
    for (int e = threadIdx.x; e < 3 * L; e += blockDim.x) {
        const int c = e / L, y = e - c * L;
        X[(c * K1 + kx) * ny + y] = res2[(2 * c) * L + y] + cmulc(res2[(2 * c + 1) * L + y], tw[y]);
    }
}

// Rows: C2R along x keeping nx cells, B_demag to b (SoA FP32).
__global__ void __launch_bounds__(kThreads) k_na_rows_inverse(int nx, int ny, const cx<float>* __restrict__ X,
                                                              const cx<float>* __restrict__ tw, FftPlan plan,
                                                              float* __restrict__ b) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L = nx, K1 = nx + 1, L2 = 2 * nx, G = kT + (kT + 1) / 2, P = (kT + 1) / 2, n = nx * ny;
    cx<float>* A = reinterpret_cast<cx<float>*>(smem_raw);
    cx<float>* B = A + 2 * G * L;
    const int j0 = blockIdx.x * kT;
    auto xval = [&](int c, int k, int j) -> cx<float> {
        if (k <= nx) return X[(c * K1 + k) * ny + j];
        return conjc(X[(c * K1 + (L2 - k)) * ny + j]);
    };
    for (int e = threadIdx.x; e < L2 * kT; e += blockDim.x) {
        const int r = e % kT, k = e / kT, j = j0 + r;
        cx<float> z = mkc(0.f, 0.f);
        if (j < ny) {
            const cx<float> bx = xval(0, k, j), by = xval(1, k, j);
            z = mkc(bx.re - by.im, bx.im + by.re);
        }
        A[(2 * r + (k & 1)) * L + (k >> 1)] = z;
    }
    for (int e = threadIdx.x; e < L2 * P; e += blockDim.x) {
        const int p = e % P, k = e / P;
        const int ja = j0 + 2 * p, jb = ja + 1;
        const cx<float> za = ja < ny ? xval(2, k, ja) : mkc(0.f, 0.f);
        const cx<float> zb = (2 * p + 1 < kT && jb < ny) ? xval(2, k, jb) : mkc(0.f, 0.f);
        A[(2 * (kT + p) + (k & 1)) * L + (k >> 1)] = mkc(za.re - zb.im, za.im + zb.re);
    }
    __syncthreads();
    cx<float>* res = fft_smem<float>(A, B, 2 * G, plan, tw, true);
    for (int e = threadIdx.x; e < G * L; e += blockDim.x) {
        const int g = e / L, x = e - g * L;
        const cx<float> z = res[(2 * g) * L + x] + cmulc(res[(2 * g + 1) * L + x], tw[x]);
        if (g < kT) {
            const int j = j0 + g;
            if (j < ny) {
                b[j * nx + x] = z.re;
                b[n + j * nx + x] = z.im;
            }
        } else {
            const int ja = j0 + 2 * (g - kT), jb = ja + 1;
            if (ja < ny) b[2 * n + ja * nx + x] = z.re;
            if (2 * (g - kT) + 1 < kT && jb < ny) b[2 * n + jb * nx + x] = z.im;
        }
    }
}

// Per-device set-up: device address of the static scratch (with the device
// current) and the shared-memory opt-in of the three kernels.  It runs on the
// first call on a device, and again when the opt-in is gone (after
// cudaDeviceReset the device has a new context: the static array is reloaded,
// possibly at another address, and the kernels' attributes are back at their
// defaults), so a cached address never outlives the context it came from.
int setup(int dev, void** out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    const int smax = 227 * 1024;
    if (g_scratch_addr[dev]) {
        cudaFuncAttributes fa;
        if (cudaFuncGetAttributes(&fa, k_na_rows_forward) == cudaSuccess && fa.maxDynamicSharedSizeBytes >= smax) {
            *out = g_scratch_addr[dev];
            return LLG_OK;
        }
        cudaGetLastError();
        g_scratch_addr[dev] = nullptr;
    }
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_scratch);
    if (e != cudaSuccess || !ptr) return LLG_ERR_CUDA;
    if (cudaFuncSetAttribute(k_na_rows_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, smax) != cudaSuccess ||
        cudaFuncSetAttribute(k_na_rows_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, smax) != cudaSuccess ||
        cudaFuncSetAttribute(k_na_column, cudaFuncAttributeMaxDynamicSharedMemorySize, smax) != cudaSuccess)
        return LLG_ERR_CUDA;
    g_scratch_addr[dev] = ptr;
    *out = ptr;
    return LLG_OK;
}

}  // namespace noalloc
}  // namespace llg

extern "C" int llg_demag_field_noalloc(int64_t nx, int64_t ny, double ms, const float* m, const double* kernel_planes,
                                       float* b_out, void* stream) {
    using namespace llg;
    using namespace llg::noalloc;
    char msg[256];
    auto fail = [&](int code, const char* text) {
        std::snprintf(msg, sizeof(msg), "llg_demag_field_noalloc: %s", text);
        llg_set_error_message(msg);
        return code;
    };
    if (!m || !kernel_planes || !b_out) return fail(LLG_ERR_INVALID, "null pointer");
    if (nx < 1 || ny < 1 || nx > 2048 || ny > 2048) return fail(LLG_ERR_INVALID, "nx and ny must lie in [1, 2048]");
    const size_t xbytes = align256(sizeof(cx<float>) * 3 * (size_t)(nx + 1) * (size_t)ny);
    const size_t twr = align256(sizeof(cx<float>) * 2 * (size_t)nx);
    const size_t twc = align256(sizeof(cx<float>) * 2 * (size_t)ny);
    if (xbytes + twr + twc > kScratchBytes)
        return fail(LLG_ERR_INVALID, "film too large for the 32 MiB static scratch (24*(nx+1)*ny + 16*(nx+ny) bytes)");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return fail(LLG_ERR_CUDA, "no current CUDA device");
    void* base = nullptr;
    if (setup(dev, &base) != LLG_OK) return fail(LLG_ERR_CUDA, "static scratch set-up failed");
    unsigned char* b8 = static_cast<unsigned char*>(base);
    cx<float>* X = reinterpret_cast<cx<float>*>(b8);
    cx<float>* tw_row = reinterpret_cast<cx<float>*>(b8 + xbytes);
    cx<float>* tw_col = reinterpret_cast<cx<float>*>(b8 + xbytes + twr);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int inx = (int)nx, iny = (int)ny;
    const FftPlan prow = make_plan(inx), pcol = make_plan(iny);
    const int G = kT + (kT + 1) / 2;
    const size_t smem_row = 4 * (size_t)G * inx * sizeof(cx<float>);
    const size_t smem_col = 12 * (size_t)iny * sizeof(cx<float>);
    const int row_blocks = (iny + kT - 1) / kT;
    k_na_twiddles<<<(2 * inx + 2 * iny + 255) / 256, 256, 0, s>>>(tw_row, inx, tw_col, iny);
    k_na_rows_forward<<<row_blocks, kThreads, smem_row, s>>>(inx, iny, (float)ms, m, X, tw_row, prow);
    k_na_column<<<inx + 1, kThreads, smem_col, s>>>(inx, iny, kernel_planes, 1.0 / (4.0 * (double)nx * (double)ny),
                                                    X, tw_col, pcol);
    k_na_rows_inverse<<<row_blocks, kThreads, smem_row, s>>>(inx, iny, X, tw_row, prow, b_out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::snprintf(msg, sizeof(msg), "llg_demag_field_noalloc: launch failed: %s", cudaGetErrorString(e));
        llg_set_error_message(msg);
        return LLG_ERR_CUDA;
    }
    return LLG_OK;
}
