// conv_tc.cu — the learned warm-start network on the 5th-generation tensor cores.
//
// Network (no reference counterpart): six 3x3 convolutions with zero padding,
// 32 channels, ReLU between layers.  Input per cell: (mx, my, mz, inside, bx, by,
// bz) with b = B_ext / 0.05 T, channel-padded to 16; output: three channels,
// normalised to a unit vector inside the film and zero in holes.  Weights and
// activations are BF16, accumulation FP32, bias FP32.
//
// One CTA computes a tile of 128 cells x N output channels as an implicit GEMM
// D[128 x N] = A[128 x K] * B[N x K]^T with K = 9 * Cin:
//   * the im2col rows of the tile (A) and the layer's weights (B) are written to
//     shared memory in the no-swizzle K-major core-matrix layout (8 rows x 16 B
//     per core matrix; core matrices along K 128 B apart, along M/N K*16 B apart);
//   * one thread issues K/16 tcgen05.mma (kind::f16, BF16 x BF16 -> FP32) into a
//     32-column TMEM accumulator and commits them to an mbarrier;
//   * each warp reads its 32 TMEM lanes with tcgen05.ld and applies bias,
//     activation and the store (or the final normalisation).
// Waits are bounded; a wait that runs out records an error and the CTA frees its
// TMEM before returning.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "async_copy.cuh"

namespace llg {
namespace ws {

constexpr int kTile = 128;       // cells per CTA (MMA M)
constexpr int kCh = 32;          // hidden channels
constexpr int kCin0 = 16;        // padded input channels (7 used)
constexpr int kNout = 16;        // padded output channels of the last layer (3 used)
constexpr int kLayers = 6;
constexpr float kFieldScale = 1.0f / 0.05f;

__device__ int g_ws_error;       // set when an mbarrier wait ran out

struct Layer {
    const __nv_bfloat16* w;      // [npad][9*cin] row-major, k = tap*cin + ci, tap = ky*3 + kx
    const float* b;              // [npad]
    int cin, npad, nreal, relu;
};

__host__ __device__ constexpr size_t conv_smem_bytes(int cin, int npad) {
    return (size_t)kTile * 9 * cin * 2 + (size_t)npad * 9 * cin * 2;
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
           (1ull << 46);   // descriptor version for tcgen05; no swizzle, base offset 0
}

__device__ __forceinline__ uint32_t instr_desc_bf16(int n) {
    // D f32, A bf16, B bf16, both K-major, N >> 3 at bit 17, M >> 4 at bit 24
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTile >> 4) << 24);
}

template <int NCOL>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, float (&v)[NCOL]);

template <>
__device__ __forceinline__ void tmem_ld<16>(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

template <>
__device__ __forceinline__ void tmem_ld<32>(uint32_t taddr, float (&v)[32]) {
    float* lo = v;
    float* hi = v + 16;
    float (&a)[16] = *reinterpret_cast<float(*)[16]>(lo);
    float (&b)[16] = *reinterpret_cast<float(*)[16]>(hi);
    tmem_ld<16>(taddr, a);
    tmem_ld<16>(taddr + 16, b);
}

// One 3x3 convolution layer over nimg images of H x W cells (NHWC, C = cin).
// Hidden layers write BF16 NHWC with C = 32; the last layer (NOUT = 16) writes
// the normalised unit vector to m_out (SoA planes of `R`, one film per image,
// cell stride H*W) with zero where mask == 0.
template <int NCOL, typename R>
__global__ void __launch_bounds__(kTile) k_conv3x3_tc(const __nv_bfloat16* __restrict__ x, int nimg, int H, int W,
                                                      Layer L, __nv_bfloat16* __restrict__ y, R* __restrict__ m_out,
                                                      const uint8_t* __restrict__ mask) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t bar;
    __shared__ uint32_t tmem_base;
    const int cin = L.cin, K = 9 * cin;
    const uint32_t sbo = (uint32_t)K * 16;   // bytes between 8-row groups
    unsigned char* As = smem;
    unsigned char* Bs = smem + (size_t)kTile * K * 2;
    const int t = threadIdx.x, warp = t >> 5;
    const long long hw = (long long)H * W;
    const long long p = (long long)blockIdx.x * kTile + t;
    const bool valid = p < (long long)nimg * hw;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_addr(&tmem_base)),
                     "r"(NCOL < 32 ? 32 : NCOL)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (t == 0) {
        mbar_init(&bar, 1);
        mbar_init_fence();
    }
    // im2col row of cell p: 9 taps x cin channels, 16-byte chunks of 8 channels
    {
        const int img = valid ? (int)(p / hw) : 0;
        const int rem = valid ? (int)(p - (long long)img * hw) : 0;
        const int yy = rem / W, xx = rem - (rem / W) * W;
        const int groups = cin / 8;
        unsigned char* arow = As + (size_t)(t >> 3) * sbo + (size_t)(t & 7) * 16;
        for (int tap = 0; tap < 9; ++tap) {
            const int sy = yy + tap / 3 - 1, sx = xx + tap % 3 - 1;
            const bool in = valid && sy >= 0 && sy < H && sx >= 0 && sx < W;
            const uint4* src = reinterpret_cast<const uint4*>(x + (((long long)img * H + (in ? sy : 0)) * W +
                                                                     (in ? sx : 0)) * cin);
            for (int g = 0; g < groups; ++g) {
                const uint4 v = in ? src[g] : make_uint4(0u, 0u, 0u, 0u);
                const int k0 = tap * cin + g * 8;
                *reinterpret_cast<uint4*>(arow + (size_t)(k0 >> 3) * 128) = v;
            }
        }
    }
    // weights: npad rows of K
    {
        const int chunks = L.npad * (K / 8);
        for (int c = t; c < chunks; c += kTile) {
            const int n = c / (K / 8), kc = c - n * (K / 8);
            const uint4 v = reinterpret_cast<const uint4*>(L.w + (size_t)n * K)[kc];
            *reinterpret_cast<uint4*>(Bs + (size_t)(n >> 3) * sbo + (size_t)kc * 128 + (size_t)(n & 7) * 16) = v;
        }
    }
    fence_async_smem();   // generic-proxy tile writes -> tensor-core reads
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    if (t == 0) {
        const uint32_t a0 = smem_addr(As), b0 = smem_addr(Bs);
        const uint32_t idesc = instr_desc_bf16(L.npad);
        for (int kk = 0; kk < K / 16; ++kk) {
            const uint64_t da = smem_desc(a0 + kk * 256, 128, sbo);
            const uint64_t db = smem_desc(b0 + kk * 256, 128, sbo);
            const uint32_t acc = kk > 0 ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                "l"(da), "l"(db), "r"(idesc), "r"(acc)
                : "memory");
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_addr(&bar))
                     : "memory");
    }
    const bool done = mbar_wait(&bar, 0);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!done) {
        if (t == 0) atomicExch(&g_ws_error, 1);
        mbar_wait(&bar, 0);   // give the MMAs one more bounded wait before the TMEM is freed
    } else {
        float acc[NCOL];
        tmem_ld<NCOL>(tmem + ((uint32_t)(warp * 32) << 16), acc);
        if (valid) {
            if (m_out == nullptr) {
                alignas(16) __nv_bfloat16 o[NCOL];
#pragma unroll
                for (int c = 0; c < NCOL; ++c) {
                    float v = acc[c] + L.b[c];
                    if (L.relu) v = fmaxf(v, 0.0f);
                    o[c] = __float2bfloat16(v);
                }
                uint4* dst = reinterpret_cast<uint4*>(y + p * NCOL);
#pragma unroll
                for (int q = 0; q < NCOL / 8; ++q) dst[q] = reinterpret_cast<const uint4*>(o)[q];
            } else {
                const int img = (int)(p / hw);
                const long long cell = p - (long long)img * hw;
                float v0 = acc[0] + L.b[0], v1 = acc[1] + L.b[1], v2 = acc[2] + L.b[2];
                const bool inside = mask == nullptr || mask[p] != 0;
                const float nn = v0 * v0 + v1 * v1 + v2 * v2;
                if (!inside) {
                    v0 = v1 = v2 = 0.0f;
                } else if (nn > 0.0f) {
                    const float inv = 1.0f / sqrtf(nn);
                    v0 *= inv; v1 *= inv; v2 *= inv;
                } else {
                    v0 = 0.0f; v1 = 0.0f; v2 = 1.0f;   // normalize(0) = +z (vec3.rs:21-25)
                }
                R* mo = m_out + (size_t)img * 3 * hw;
                mo[cell] = (R)v0;
                mo[hw + cell] = (R)v1;
                mo[2 * hw + cell] = (R)v2;
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(NCOL < 32 ? 32 : NCOL)
                     : "memory");
}

// Network input of image f from SoA planes m (R), mask and the image's field.
template <typename R>
__global__ void k_ws_input(const R* __restrict__ m, const uint8_t* __restrict__ mask, const double* __restrict__ bext,
                           int nimg, long long hw, __nv_bfloat16* __restrict__ x) {
    const long long total = (long long)nimg * hw;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < total;
         p += (long long)gridDim.x * blockDim.x) {
        const int img = (int)(p / hw);
        const long long cell = p - (long long)img * hw;
        const R* mi = m + (size_t)img * 3 * hw;
        const bool inside = mask == nullptr || mask[p] != 0;
        alignas(16) __nv_bfloat16 v[kCin0];
        const float in = inside ? 1.0f : 0.0f;
        v[0] = __float2bfloat16(in * (float)mi[cell]);
        v[1] = __float2bfloat16(in * (float)mi[hw + cell]);
        v[2] = __float2bfloat16(in * (float)mi[2 * hw + cell]);
        v[3] = __float2bfloat16(in);
        v[4] = __float2bfloat16((float)bext[3 * img + 0] * kFieldScale);
        v[5] = __float2bfloat16((float)bext[3 * img + 1] * kFieldScale);
        v[6] = __float2bfloat16((float)bext[3 * img + 2] * kFieldScale);
#pragma unroll
        for (int c = 7; c < kCin0; ++c) v[c] = __float2bfloat16(0.0f);
        uint4* dst = reinterpret_cast<uint4*>(x + p * kCin0);
        dst[0] = reinterpret_cast<const uint4*>(v)[0];
        dst[1] = reinterpret_cast<const uint4*>(v)[1];
    }
}

}  // namespace ws
}  // namespace llg

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
#include "build_api.h"

namespace llg {
namespace ws {

struct Net {
    int device = 0;
    __nv_bfloat16* w[kLayers] = {};
    float* b[kLayers] = {};
    Layer L[kLayers];
    __nv_bfloat16* x0 = nullptr;   // input, 16 channels
    __nv_bfloat16* h[2] = {};       // hidden activations, 32 channels
    double* bext = nullptr;
    long long cap_cells = 0;
    int cap_img = 0;
};

static const int kCinReal[kLayers] = {7, kCh, kCh, kCh, kCh, kCh};
static const int kCoutReal[kLayers] = {kCh, kCh, kCh, kCh, kCh, 3};

long long net_param_count() {
    long long n = 0;
    for (int l = 0; l < kLayers; ++l) n += (long long)kCoutReal[l] * 9 * kCinReal[l] + kCoutReal[l];
    return n;
}

void net_destroy(Net* net) {
    if (!net) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(net->device);
    for (int l = 0; l < kLayers; ++l) {
        cudaFree(net->w[l]);
        cudaFree(net->b[l]);
    }
    cudaFree(net->x0);
    cudaFree(net->h[0]);
    cudaFree(net->h[1]);
    cudaFree(net->bext);
    cudaSetDevice(prev);
    delete net;
}

// params: per layer W[cout][3][3][cin] then b[cout], FP32, real (unpadded) sizes.
cudaError_t net_create(const float* params, long long n, int device, Net** out) {
    if (n != net_param_count()) return cudaErrorInvalidValue;
    Net* net = new Net();
    net->device = device;
    cudaError_t e = cudaSuccess;
    const float* q = params;
    for (int l = 0; l < kLayers && e == cudaSuccess; ++l) {
        const int cin = l == 0 ? kCin0 : kCh, npad = l == kLayers - 1 ? kNout : kCh;
        const int ci_r = kCinReal[l], co_r = kCoutReal[l], K = 9 * cin;
        std::vector<__nv_bfloat16> w((size_t)npad * K, __float2bfloat16(0.0f));
        std::vector<float> b(npad, 0.0f);
        for (int co = 0; co < co_r; ++co)
            for (int tap = 0; tap < 9; ++tap)
                for (int ci = 0; ci < ci_r; ++ci)
                    w[(size_t)co * K + tap * cin + ci] = __float2bfloat16(q[((size_t)co * 9 + tap) * ci_r + ci]);
        q += (size_t)co_r * 9 * ci_r;
        for (int co = 0; co < co_r; ++co) b[co] = q[co];
        q += co_r;
        e = cudaMalloc(&net->w[l], w.size() * sizeof(__nv_bfloat16));
        if (e == cudaSuccess) e = cudaMalloc(&net->b[l], b.size() * sizeof(float));
        if (e == cudaSuccess) e = cudaMemcpy(net->w[l], w.data(), w.size() * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(net->b[l], b.data(), b.size() * sizeof(float), cudaMemcpyHostToDevice);
        net->L[l] = Layer{net->w[l], net->b[l], cin, npad, co_r, l < kLayers - 1 ? 1 : 0};
    }
    if (e == cudaSuccess) {
        const size_t smax = conv_smem_bytes(kCh, kCh);
        e = cudaFuncSetAttribute(k_conv3x3_tc<kCh, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_conv3x3_tc<kNout, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_conv3x3_tc<kCh, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_conv3x3_tc<kNout, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax);
    }
    if (e != cudaSuccess) {
        net_destroy(net);
        return e;
    }
    *out = net;
    return cudaSuccess;
}

static cudaError_t ensure_scratch(Net* net, long long cells, int nimg) {
    if (cells > net->cap_cells) {
        cudaFree(net->x0);
        cudaFree(net->h[0]);
        cudaFree(net->h[1]);
        net->x0 = net->h[0] = net->h[1] = nullptr;
        net->cap_cells = 0;
        cudaError_t e = cudaMalloc(&net->x0, (size_t)cells * kCin0 * sizeof(__nv_bfloat16));
        if (e == cudaSuccess) e = cudaMalloc(&net->h[0], (size_t)cells * kCh * sizeof(__nv_bfloat16));
        if (e == cudaSuccess) e = cudaMalloc(&net->h[1], (size_t)cells * kCh * sizeof(__nv_bfloat16));
        if (e != cudaSuccess) return e;
        net->cap_cells = cells;
    }
    if (nimg > net->cap_img) {
        cudaFree(net->bext);
        net->bext = nullptr;
        net->cap_img = 0;
        cudaError_t e = cudaMalloc(&net->bext, (size_t)nimg * 3 * sizeof(double));
        if (e != cudaSuccess) return e;
        net->cap_img = nimg;
    }
    return cudaSuccess;
}

int net_error() {
    int v = 0;
    cudaMemcpyFromSymbol(&v, g_ws_error, sizeof(int));
    return v;
}

// Proposal for nimg images of ny x nx cells (SoA planes of R, image stride 3*ny*nx):
// m_out may alias m_in (the input is consumed by the first layer).
template <typename R>
cudaError_t net_apply(Net* net, const R* m_in, R* m_out, const uint8_t* mask, const double* bext_host, int nimg,
                      int ny, int nx, cudaStream_t s) {
    const long long hw = (long long)ny * nx, cells = hw * nimg;
    if (cells <= 0) return cudaSuccess;
    cudaError_t e = ensure_scratch(net, cells, nimg);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(net->bext, bext_host, (size_t)nimg * 3 * sizeof(double), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    k_ws_input<R><<<(unsigned)std::min<long long>((cells + 255) / 256, 148 * 16), 256, 0, s>>>(m_in, mask, net->bext,
                                                                                              nimg, hw, net->x0);
    const unsigned grid = (unsigned)((cells + kTile - 1) / kTile);
    const __nv_bfloat16* cur = net->x0;
    for (int l = 0; l < kLayers; ++l) {
        const Layer& L = net->L[l];
        const size_t smem = conv_smem_bytes(L.cin, L.npad);
        if (l < kLayers - 1) {
            __nv_bfloat16* nxt = net->h[l & 1];
            k_conv3x3_tc<kCh, R><<<grid, kTile, smem, s>>>(cur, nimg, ny, nx, L, nxt, nullptr, nullptr);
            cur = nxt;
        } else {
            k_conv3x3_tc<kNout, R><<<grid, kTile, smem, s>>>(cur, nimg, ny, nx, L, nullptr, m_out, mask);
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template cudaError_t net_apply<float>(Net*, const float*, float*, const uint8_t*, const double*, int, int, int,
                                      cudaStream_t);
template cudaError_t net_apply<double>(Net*, const double*, double*, const uint8_t*, const double*, int, int, int,
                                       cudaStream_t);

}  // namespace ws
}  // namespace llg
