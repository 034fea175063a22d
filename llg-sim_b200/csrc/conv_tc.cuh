// conv_tc.cuh — 3x3 convolutions of the learned warm-start network on the
// 5th-generation tensor cores (tcgen05, BF16 x BF16 -> FP32 in TMEM).
//
// Network (no reference counterpart): six 3x3 convolutions with zero padding,
// 32 channels, ReLU between layers.  Input per cell: (mx, my, mz, inside, bx, by,
// bz) with b = B_ext / 0.05 T, channel-padded to 16; output: three channels.
// Activations are BF16 NHWC ([cell][channel]); accumulation FP32, bias FP32.
//
// Forward / input-gradient kernel (k_conv3x3_tc): one CTA computes a tile of
// 128 cells x N output channels as an implicit GEMM D[128 x N] = A[128 x K] *
// B[N x K]^T, K = 9 * Cin, both operands K-major in shared memory (core matrices
// of 8 rows x 16 B; K neighbours 128 B apart, M/N neighbours K*16 B apart).
// The input gradient of a layer is the same convolution of the output gradient
// with the weights transposed in (cout, cin) and flipped in the taps, so the
// backward pass reuses this kernel with another epilogue.
//
// Weight-gradient kernel (k_wgrad_tc): D[m][n] = sum over cells p of
// X[p + off(tap)][ci] * G[p][n] with m = tap*Cin + ci: the reduction runs over
// cells, so both operands are MN-major in shared memory (the cells' channel
// vectors are the 16-byte rows of the core matrices as they sit in HBM) and
// the accumulators stay in TMEM across the CTA's cell range.
//
// Every mbarrier wait is bounded by the caller's spin limit; a wait that runs out
// sets the caller's error flag, waits once more (bounded) for the MMAs in flight,
// and the CTA frees its TMEM before returning.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstdlib>

#include "async_copy.cuh"

namespace llg {
namespace ws {

constexpr int kTile = 128;       // cells per CTA tile (MMA M)
constexpr int kCh = 32;          // hidden channels
constexpr int kCin0 = 16;        // padded input channels (7 used)
constexpr int kNout = 16;        // padded output channels of the last layer (3 used)
constexpr int kLayers = 6;
constexpr float kFieldScale = 1.0f / 0.05f;

// Epilogues of k_conv3x3_tc.
enum ConvEpi : int {
    EPI_HIDDEN = 0,      // + bias, ReLU, BF16 [p][N]
    EPI_FINAL_NORM = 1,  // + bias, normalised unit vector into SoA planes (zero in holes)
    EPI_FINAL_RAW = 2,   // + bias, FP32 [p][4] (3 channels used): the training output
    EPI_DGRAD = 3,       // no bias, times (act[p][c] > 0) (ReLU gradient), BF16 [p][N]
};

struct Layer {
    const __nv_bfloat16* w;      // [npad][9*cin] row-major, k = tap*cin + ci, tap = ky*3 + kx
    const float* b;              // [npad] (null for EPI_DGRAD)
    int cin, npad, nreal, relu;
};

__host__ __device__ constexpr size_t conv_smem_bytes(int cin, int npad) {
    return (size_t)kTile * 9 * cin * 2 + (size_t)npad * 9 * cin * 2;
}

// Shared-memory matrix descriptor (tcgen05): start address, leading / stride
// byte offsets (16-byte units), descriptor version 1 at bit 46, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
           (1ull << 46);
}

// Instruction descriptor of kind::f16: D f32 (bit 4), A and B bf16 (bits 7, 10),
// A / B MN-major flags (bits 15, 16), N >> 3 at bit 17, M >> 4 at bit 24.
__device__ __forceinline__ uint32_t instr_desc_bf16(int m, int n, bool a_mn, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
           ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
        "l"(da), "l"(db), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncol) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst_smem)),
                 "r"(ncol)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t tmem, uint32_t ncol) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncol) : "memory");
}

// Bounded wait on an mbarrier phase with a caller-given poll limit.
__device__ __forceinline__ bool mbar_wait_n(uint64_t* bar, uint32_t parity, long long limit) {
    for (long long i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
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
    float (&a)[16] = *reinterpret_cast<float(*)[16]>(v);
    float (&b)[16] = *reinterpret_cast<float(*)[16]>(v + 16);
    tmem_ld<16>(taddr, a);
    tmem_ld<16>(taddr + 16, b);
}

// One 3x3 convolution over nimg images of H x W cells (input NHWC BF16, C = cin).
//   EPI_HIDDEN:     y = BF16(ReLU?(acc + b)) [p][NCOL]
//   EPI_FINAL_NORM: m_out (SoA planes of R, image stride 3*H*W) = normalize(acc + b), 0 where mask == 0
//   EPI_FINAL_RAW:  out32[p][0..3] = acc + b (FP32)
//   EPI_DGRAD:      y = BF16(acc * (act[p][c] > 0)) [p][NCOL]
template <int NCOL, int EPI, typename R>
__global__ void __launch_bounds__(kTile) k_conv3x3_tc(const __nv_bfloat16* __restrict__ x, int nimg, int H, int W,
                                                      Layer L, __nv_bfloat16* __restrict__ y, R* __restrict__ m_out,
                                                      float* __restrict__ out32, const uint8_t* __restrict__ mask,
                                                      const __nv_bfloat16* __restrict__ act, int* err,
                                                      long long spin) {
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
    constexpr uint32_t kCols = NCOL < 32 ? 32 : NCOL;

    if (warp == 0) tmem_alloc(&tmem_base, kCols);
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
        const uint32_t idesc = instr_desc_bf16(kTile, L.npad, false, false);
        for (int kk = 0; kk < K / 16; ++kk)
            mma_bf16(tmem, smem_desc(a0 + kk * 256, 128, sbo), smem_desc(b0 + kk * 256, 128, sbo), idesc,
                     kk > 0 ? 1u : 0u);
        mma_commit(&bar);
    }
    const bool done = mbar_wait_n(&bar, 0, spin);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!done) {
        if (t == 0) atomicExch(err, 1);
        mbar_wait(&bar, 0);   // one more bounded wait for the MMAs before the TMEM is freed
    } else {
        float acc[NCOL];
        tmem_ld<NCOL>(tmem + ((uint32_t)(warp * 32) << 16), acc);
        if (valid) {
            if constexpr (EPI == EPI_HIDDEN || EPI == EPI_DGRAD) {
                alignas(16) __nv_bfloat16 o[NCOL];
                if constexpr (EPI == EPI_DGRAD) {
                    alignas(16) __nv_bfloat16 a[NCOL];
#pragma unroll
                    for (int q = 0; q < NCOL / 8; ++q)
                        reinterpret_cast<uint4*>(a)[q] = reinterpret_cast<const uint4*>(act + p * NCOL)[q];
#pragma unroll
                    for (int c = 0; c < NCOL; ++c)
                        o[c] = __float2bfloat16(__bfloat162float(a[c]) > 0.0f ? acc[c] : 0.0f);
                } else {
#pragma unroll
                    for (int c = 0; c < NCOL; ++c) {
                        float v = acc[c] + L.b[c];
                        if (L.relu) v = fmaxf(v, 0.0f);
                        o[c] = __float2bfloat16(v);
                    }
                }
                uint4* dst = reinterpret_cast<uint4*>(y + p * NCOL);
#pragma unroll
                for (int q = 0; q < NCOL / 8; ++q) dst[q] = reinterpret_cast<const uint4*>(o)[q];
            } else if constexpr (EPI == EPI_FINAL_RAW) {
                *reinterpret_cast<float4*>(out32 + p * 4) =
                    make_float4(acc[0] + L.b[0], acc[1] + L.b[1], acc[2] + L.b[2], 0.0f);
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
    if (warp == 0) tmem_dealloc(tmem, kCols);
}

// Per-cell epilogue shared by the one-shot and the pipelined convolution.
template <int NCOL, int EPI, typename R>
__device__ __forceinline__ void conv_epilogue(const float (&acc)[NCOL], long long p, long long hw, const Layer& L,
                                              __nv_bfloat16* __restrict__ y, R* __restrict__ m_out,
                                              float* __restrict__ out32, const uint8_t* __restrict__ mask,
                                              const __nv_bfloat16* __restrict__ act) {
    if constexpr (EPI == EPI_HIDDEN || EPI == EPI_DGRAD) {
        alignas(16) __nv_bfloat16 o[NCOL];
        if constexpr (EPI == EPI_DGRAD) {
            alignas(16) __nv_bfloat16 a[NCOL];
#pragma unroll
            for (int q = 0; q < NCOL / 8; ++q)
                reinterpret_cast<uint4*>(a)[q] = reinterpret_cast<const uint4*>(act + p * NCOL)[q];
#pragma unroll
            for (int c = 0; c < NCOL; ++c) o[c] = __float2bfloat16(__bfloat162float(a[c]) > 0.0f ? acc[c] : 0.0f);
        } else {
#pragma unroll
            for (int c = 0; c < NCOL; ++c) {
                float v = acc[c] + L.b[c];
                if (L.relu) v = fmaxf(v, 0.0f);
                o[c] = __float2bfloat16(v);
            }
        }
        uint4* dst = reinterpret_cast<uint4*>(y + p * NCOL);
#pragma unroll
        for (int q = 0; q < NCOL / 8; ++q) dst[q] = reinterpret_cast<const uint4*>(o)[q];
    } else if constexpr (EPI == EPI_FINAL_RAW) {
        *reinterpret_cast<float4*>(out32 + p * 4) = make_float4(acc[0] + L.b[0], acc[1] + L.b[1], acc[2] + L.b[2], 0.0f);
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

// Pipelined convolution for images up to kHaloW cells wide: a persistent CTA loads
// the layer's weights once and walks 128-cell tiles.  For each tile the cells it
// reads (the tile and one image row plus one cell on either side) are one
// contiguous NHWC range, fetched by a 1-D bulk copy (cp.async.bulk, this GPU's
// memory, no multicast) into one of two halo buffers while the previous tile is
// processed; the im2col rows are built from shared memory; the MMAs of a tile
// accumulate into one of two TMEM accumulators, so the epilogue of tile k-1 runs
// while the tensor cores work on tile k.  The MMA sequence of a tile is the one
// of k_conv3x3_tc (same operands, same order), so both kernels give the same bits.
constexpr int kHaloW = 256;
constexpr int kHaloCells = kTile + 2 * kHaloW + 2;

template <int CIN>
__host__ __device__ constexpr size_t conv_pipe_smem_bytes(int npad) {
    return (size_t)npad * 9 * CIN * 2 + (size_t)kTile * 9 * CIN * 2 + 2 * (size_t)kHaloCells * CIN * 2;
}

template <int NCOL, int EPI, typename R, int CIN>
__global__ void __launch_bounds__(kTile) k_conv3x3_pipe(const __nv_bfloat16* __restrict__ x, int nimg, int H, int W,
                                                        Layer L, __nv_bfloat16* __restrict__ y,
                                                        R* __restrict__ m_out, float* __restrict__ out32,
                                                        const uint8_t* __restrict__ mask,
                                                        const __nv_bfloat16* __restrict__ act, int* err,
                                                        long long spin) {
    constexpr int K = 9 * CIN;
    constexpr uint32_t sbo = (uint32_t)K * 16;
    constexpr uint32_t kCols = 2 * (NCOL < 32 ? 32 : NCOL);
    constexpr uint32_t kAcc = NCOL < 32 ? 32 : NCOL;   // column offset of the second accumulator
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t bar_halo[2], bar_mma;
    __shared__ uint32_t tmem_base;
    unsigned char* Bs = smem;
    unsigned char* As = Bs + (size_t)L.npad * K * 2;
    unsigned char* Hs = As + (size_t)kTile * K * 2;   // two halo buffers of kHaloCells * CIN bf16
    const int t = threadIdx.x, warp = t >> 5;
    const long long hw = (long long)H * W, total = (long long)nimg * hw;
    const long long ntiles = (total + kTile - 1) / kTile;

    if (warp == 0) tmem_alloc(&tmem_base, kCols);
    if (t == 0) {
        mbar_init(&bar_halo[0], 1);
        mbar_init(&bar_halo[1], 1);
        mbar_init(&bar_mma, 1);
        mbar_init_fence();
    }
    // weights, K-major core matrices
    for (int c = t; c < L.npad * (K / 8); c += kTile) {
        const int n = c / (K / 8), kc = c - n * (K / 8);
        const uint4 v = reinterpret_cast<const uint4*>(L.w + (size_t)n * K)[kc];
        *reinterpret_cast<uint4*>(Bs + (size_t)(n >> 3) * sbo + (size_t)kc * 128 + (size_t)(n & 7) * 16) = v;
    }
    __syncthreads();
    const uint32_t tmem = tmem_base;
    auto halo_range = [&](long long tile, long long* lo, long long* cnt) {
        const long long p0 = tile * kTile;
        const long long a = p0 - W - 1 < 0 ? 0 : p0 - W - 1;
        long long b = p0 + kTile + W + 1;
        if (b > total) b = total;
        *lo = a;
        *cnt = b - a;
    };
    auto issue_halo = [&](long long tile, int buf) {
        long long lo, cnt;
        halo_range(tile, &lo, &cnt);
        const uint32_t bytes = (uint32_t)(cnt * CIN * 2);
        mbar_arrive_expect_tx(&bar_halo[buf], bytes);
        bulk_copy_g2s(Hs + (size_t)buf * kHaloCells * CIN * 2, x + lo * CIN, bytes, &bar_halo[buf]);
    };
    // Outstanding asynchronous work, tracked identically by every thread (the tile
    // sequence is fixed): the phase parity of the last copy issued into each halo
    // buffer that has not been waited for (-1: none), and of the last MMA commit.
    int halo_pending[2] = {-1, -1};
    int mma_pending = -1;
    long long tile = blockIdx.x;
    if (tile < ntiles) {
        if (t == 0) {
            fence_async_smem();
            issue_halo(tile, 0);
        }
        halo_pending[0] = 0;
    }
    const uint32_t idesc = instr_desc_bf16(kTile, L.npad, false, false);
    bool ok = true;
    int k = 0;
    long long prev = -1;
    for (; tile < ntiles; tile += gridDim.x, ++k) {
        const int hb = k & 1;
        ok = mbar_wait_n(&bar_halo[hb], (uint32_t)((k >> 1) & 1), spin);
        if (!ok) break;
        halo_pending[hb] = -1;
        if (mma_pending >= 0) {   // the MMAs of the previous tile have read the im2col buffer
            ok = mbar_wait_n(&bar_mma, (uint32_t)mma_pending, spin);
            if (!ok) break;
            mma_pending = -1;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        }
        // the other halo buffer was read by the previous tile's im2col build (before
        // the previous barrier): refill it with the next tile's range
        if (tile + gridDim.x < ntiles) {
            if (t == 0) {
                fence_async_smem();
                issue_halo(tile + gridDim.x, hb ^ 1);
            }
            halo_pending[hb ^ 1] = ((k + 1) >> 1) & 1;
        }
        // im2col row of cell p from the halo (zero outside the image)
        {
            long long lo, cnt;
            halo_range(tile, &lo, &cnt);
            const unsigned char* hsrc = Hs + (size_t)hb * kHaloCells * CIN * 2;
            const long long p = tile * kTile + t;
            const bool valid = p < total;
            const int img = valid ? (int)(p / hw) : 0;
            const int rem = valid ? (int)(p - (long long)img * hw) : 0;
            const int yy = rem / W, xx = rem - (rem / W) * W;
            unsigned char* arow = As + (size_t)(t >> 3) * sbo + (size_t)(t & 7) * 16;
#pragma unroll
            for (int tap = 0; tap < 9; ++tap) {
                const int sy = yy + tap / 3 - 1, sx = xx + tap % 3 - 1;
                const bool in = valid && sy >= 0 && sy < H && sx >= 0 && sx < W;
                const long long q = p + (long long)(tap / 3 - 1) * W + (tap % 3 - 1);
                const uint4* src = reinterpret_cast<const uint4*>(hsrc + (in ? (q - lo) : 0) * CIN * 2);
#pragma unroll
                for (int g = 0; g < CIN / 8; ++g) {
                    const uint4 v = in ? src[g] : make_uint4(0u, 0u, 0u, 0u);
                    *reinterpret_cast<uint4*>(arow + (size_t)((tap * CIN + g * 8) >> 3) * 128) = v;
                }
            }
        }
        fence_async_smem();
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t acc_col = (uint32_t)hb * kAcc;
        if (t == 0) {
            const uint32_t a0 = smem_addr(As), b0 = smem_addr(Bs);
            for (int kk = 0; kk < K / 16; ++kk)
                mma_bf16(tmem + acc_col, smem_desc(a0 + kk * 256, 128, sbo), smem_desc(b0 + kk * 256, 128, sbo), idesc,
                         kk > 0 ? 1u : 0u);
            mma_commit(&bar_mma);
        }
        mma_pending = k & 1;
        // epilogue of the previous tile while the tensor cores work on this one
        if (prev >= 0) {
            float acc[NCOL];
            tmem_ld<NCOL>(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(hb ^ 1) * kAcc, acc);
            const long long p = prev * kTile + t;
            if (p < total) conv_epilogue<NCOL, EPI, R>(acc, p, hw, L, y, m_out, out32, mask, act);
        }
        prev = tile;
    }
    if (ok && mma_pending >= 0) {
        ok = mbar_wait_n(&bar_mma, (uint32_t)mma_pending, spin);
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (ok) {
            mma_pending = -1;
            float acc[NCOL];
            tmem_ld<NCOL>(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((k - 1) & 1) * kAcc, acc);
            const long long p = prev * kTile + t;
            if (p < total) conv_epilogue<NCOL, EPI, R>(acc, p, hw, L, y, m_out, out32, mask, act);
        }
    }
    if (!ok) {
        if (t == 0) atomicExch(err, 1);
        // one more bounded wait for the copies and MMAs still in flight, so that none
        // writes shared memory or TMEM after the CTA has released them
        if (mma_pending >= 0) mbar_wait(&bar_mma, (uint32_t)mma_pending);
        for (int b = 0; b < 2; ++b)
            if (halo_pending[b] >= 0) mbar_wait(&bar_halo[b], (uint32_t)halo_pending[b]);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, kCols);
}

// Launch of one convolution layer: the pipelined kernel for images up to kHaloW
// cells wide, the one-shot kernel otherwise (LLG_B200_CONV_ONESHOT=1 selects the
// one-shot kernel everywhere; both give the same bits).
inline bool conv_oneshot_forced() {
    const char* e = std::getenv("LLG_B200_CONV_ONESHOT");
    return e && e[0] == '1';
}

template <int NCOL, int EPI, typename R>
cudaError_t conv_launch(const __nv_bfloat16* x, int nimg, int H, int W, const Layer& L, __nv_bfloat16* y, R* m_out,
                        float* out32, const uint8_t* mask, const __nv_bfloat16* act, int* err, long long spin,
                        cudaStream_t s) {
    const long long cells = (long long)nimg * H * W;
    if (cells <= 0) return cudaSuccess;
    const long long ntiles = (cells + kTile - 1) / kTile;
    if (W <= kHaloW && (L.cin == 16 || L.cin == 32) && !conv_oneshot_forced()) {
        int dev = 0, nsm = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        const unsigned grid = (unsigned)std::min<long long>(ntiles, nsm);
        if (L.cin == 32) {
            const size_t smem = conv_pipe_smem_bytes<32>(L.npad);
            cudaError_t e = cudaFuncSetAttribute(k_conv3x3_pipe<NCOL, EPI, R, 32>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            k_conv3x3_pipe<NCOL, EPI, R, 32><<<grid, kTile, smem, s>>>(x, nimg, H, W, L, y, m_out, out32, mask, act,
                                                                        err, spin);
        } else {
            const size_t smem = conv_pipe_smem_bytes<16>(L.npad);
            cudaError_t e = cudaFuncSetAttribute(k_conv3x3_pipe<NCOL, EPI, R, 16>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            k_conv3x3_pipe<NCOL, EPI, R, 16><<<grid, kTile, smem, s>>>(x, nimg, H, W, L, y, m_out, out32, mask, act,
                                                                        err, spin);
        }
        return cudaGetLastError();
    }
    const size_t smem = conv_smem_bytes(L.cin, L.npad);
    cudaError_t e = cudaFuncSetAttribute(k_conv3x3_tc<NCOL, EPI, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    k_conv3x3_tc<NCOL, EPI, R><<<(unsigned)ntiles, kTile, smem, s>>>(x, nimg, H, W, L, y, m_out, out32, mask, act, err,
                                                                     spin);
    return cudaGetLastError();
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
