// train_tc.cu — training of the learned warm-start network on the GPU with this
// project's own tensor-core kernels (no reference counterpart).
//
// One training step over a minibatch of films (device-resident inputs):
//   forward   x0 = input(m0, inside, B_ext), h_l = ReLU(conv_l(h_{l-1})) in BF16,
//             v = conv_5(h_4) in FP32                       (k_conv3x3_tc)
//   loss      L = mean over film cells of 1 - (v/|v|) . m_relaxed, and
//             g_5 = dL/dv = -(t - (u.t) u) / |v| per cell   (k_cos_loss)
//   backward  for l = 5 .. 0: dW_l = sum_p im2col(a_l)[p] (x) g_l[p]  (k_wgrad_tc,
//             tcgen05 with the reduction over cells in TMEM), db_l = sum_p g_l[p],
//             g_{l-1} = conv(g_l, W_l flipped / transposed) * (h_{l-1} > 0)
//             (k_conv3x3_tc, EPI_DGRAD)
//   update    Adam on FP32 master weights; the BF16 forward and input-gradient
//             weight layouts are rewritten in the same kernel      (k_adam_pack)
// Activations and gradients are BF16, every accumulation FP32, all reductions
// in a fixed order (the gradients are deterministic).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "conv_tc.cuh"

namespace llg {
namespace ws {

constexpr int kWgKC = 64;            // cells per shared-memory chunk of the weight-gradient kernel
constexpr int kRedThreads = 256;

// Weight gradient of one layer, partial over this CTA's cells:
//   part[blockIdx][m][n] = sum_p A[m][p] G[n][p],  A[m = tap*cin + ci][p] = X[p + off(tap)][ci]
// (zero outside the image), G[n][p] = g[p][n].  NT M tiles of 128 rows, N = NN.
// Both operands MN-major, no swizzle: element (mn, k) of a tile sits at byte
// (k / 8) * LBO + (mn / 8) * SBO + (k % 8) * 16 + (mn % 8) * 2 with SBO = 128
// (the 8-channel groups of one cell group are adjacent) and LBO = (MN / 8) * 128.
template <int NT, int NN>
__global__ void __launch_bounds__(128) k_wgrad_tc(const __nv_bfloat16* __restrict__ x, int cin,
                                                  const __nv_bfloat16* __restrict__ g, int nimg, int H, int W,
                                                  long long cells_per_cta, float* __restrict__ part, int* err,
                                                  long long spin) {
    constexpr int A_TILE = kTile * kWgKC * 2;           // bytes per M tile and chunk
    constexpr uint32_t A_LBO = (kTile / 8) * 128, B_LBO = (NN / 8) * 128;
    constexpr uint32_t kCols = NT * NN <= 32 ? 32 : NT * NN <= 64 ? 64 : NT * NN <= 128 ? 128 : 256;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t bar;
    __shared__ uint32_t tmem_base;
    unsigned char* As = smem;
    unsigned char* Bs = smem + NT * A_TILE;
    const int t = threadIdx.x, warp = t >> 5;
    const long long hw = (long long)H * W, total = (long long)nimg * hw;
    const long long c_begin = (long long)blockIdx.x * cells_per_cta;
    const long long c_end = min(total, c_begin + cells_per_cta);
    const int M = 9 * cin, groups = cin / 8;

    if (warp == 0) tmem_alloc(&tmem_base, kCols);
    if (t == 0) {
        mbar_init(&bar, 1);
        mbar_init_fence();
    }
    // rows past 9*cin of the last tile stay zero for the whole kernel
    for (int i = t; i < NT * A_TILE / 16; i += 128) reinterpret_cast<uint4*>(As)[i] = make_uint4(0u, 0u, 0u, 0u);
    __syncthreads();
    const uint32_t tmem = tmem_base;
    const uint32_t idesc = instr_desc_bf16(kTile, NN, true, true);
    uint32_t phase = 0;
    bool ok = true, first = true;
    for (long long c0 = c_begin; c0 < c_end; c0 += kWgKC) {
        // A: (cell k, tap, 8-channel group) -> one 16-byte chunk
        for (int e = t; e < kWgKC * 9 * groups; e += 128) {
            const int k = e / (9 * groups), r = e - k * (9 * groups), tap = r / groups, cg = r - tap * groups;
            const long long p = c0 + k;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (p < c_end) {
                const int img = (int)(p / hw);
                const int rem = (int)(p - (long long)img * hw);
                const int sy = rem / W + tap / 3 - 1, sx = rem % W + tap % 3 - 1;
                if (sy >= 0 && sy < H && sx >= 0 && sx < W)
                    v = reinterpret_cast<const uint4*>(x + (((long long)img * H + sy) * W + sx) * cin)[cg];
            }
            const int m = tap * cin + cg * 8, tile = m / kTile, mm = m - tile * kTile;
            *reinterpret_cast<uint4*>(As + tile * A_TILE + (k >> 3) * A_LBO + (mm >> 3) * 128 + (k & 7) * 16) = v;
        }
        // B: (cell k, 8-channel group of the output gradient)
        for (int e = t; e < kWgKC * (NN / 8); e += 128) {
            const int k = e / (NN / 8), ng = e - k * (NN / 8);
            const long long p = c0 + k;
            const uint4 v = p < c_end ? reinterpret_cast<const uint4*>(g + p * NN)[ng] : make_uint4(0u, 0u, 0u, 0u);
            *reinterpret_cast<uint4*>(Bs + (k >> 3) * B_LBO + ng * 128 + (k & 7) * 16) = v;
        }
        fence_async_smem();
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (t == 0) {
            const uint32_t a0 = smem_addr(As), b0 = smem_addr(Bs);
            for (int tile = 0; tile < NT; ++tile)
                for (int kk = 0; kk < kWgKC / 16; ++kk) {
                    const uint64_t da = smem_desc(a0 + tile * A_TILE + kk * 2 * A_LBO, A_LBO, 128);
                    const uint64_t db = smem_desc(b0 + kk * 2 * B_LBO, B_LBO, 128);
                    mma_bf16(tmem + tile * NN, da, db, idesc, (first && kk == 0) ? 0u : 1u);
                }
            mma_commit(&bar);
        }
        first = false;
        // the chunk buffers are rewritten only after these MMAs have read them
        ok = mbar_wait_n(&bar, phase, spin);
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (!ok) break;
    }
    if (!ok) {
        if (t == 0) atomicExch(err, 1);
        mbar_wait(&bar, phase ^ 1u);   // one more bounded wait for the MMAs before the TMEM is freed
    } else if (!first) {
        for (int tile = 0; tile < NT; ++tile) {
            float acc[NN];
            tmem_ld<NN>(tmem + ((uint32_t)(warp * 32) << 16) + tile * NN, acc);
            const int m = tile * kTile + warp * 32 + (t & 31);
            if (m < M) {
                float* dst = part + ((size_t)blockIdx.x * (NT * kTile) + m) * NN;
#pragma unroll
                for (int q = 0; q < NN / 4; ++q)
                    reinterpret_cast<float4*>(dst)[q] = make_float4(acc[4 * q], acc[4 * q + 1], acc[4 * q + 2],
                                                                    acc[4 * q + 3]);
            }
        }
    } else {
        // no cells for this CTA: its partial is zero
        for (int i = t; i < NT * kTile * NN; i += 128) part[(size_t)blockIdx.x * NT * kTile * NN + i] = 0.0f;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, kCols);
}

// Cosine loss of the output against the relaxed states and its gradient.
// v = out32[p][0..2], t = target (SoA planes, image stride 3*H*W); inside cells
// only.  g[p][0..2] = -(t - (u.t) u) / |v| (not yet divided by the cell count),
// g[p][3..15] = 0.  Per-block partial sums of (1 - u.t) and of the inside count.
__global__ void __launch_bounds__(kRedThreads) k_cos_loss(const float* __restrict__ out32,
                                                          const float* __restrict__ target,
                                                          const uint8_t* __restrict__ mask, int nimg, long long hw,
                                                          __nv_bfloat16* __restrict__ g, double* __restrict__ part) {
    __shared__ double s_loss[kRedThreads], s_cnt[kRedThreads];
    const long long total = (long long)nimg * hw;
    double loss = 0.0, cnt = 0.0;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < total;
         p += (long long)gridDim.x * blockDim.x) {
        const int img = (int)(p / hw);
        const long long cell = p - (long long)img * hw;
        alignas(16) __nv_bfloat16 o[kNout];
#pragma unroll
        for (int c = 0; c < kNout; ++c) o[c] = __float2bfloat16(0.0f);
        if (mask == nullptr || mask[p] != 0) {
            const float4 v = *reinterpret_cast<const float4*>(out32 + p * 4);
            const float* tg = target + (size_t)img * 3 * hw;
            const float t0 = tg[cell], t1 = tg[hw + cell], t2 = tg[2 * hw + cell];
            const float n = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
            cnt += 1.0;
            if (n > 0.0f) {
                const float inv = 1.0f / n;
                const float u0 = v.x * inv, u1 = v.y * inv, u2 = v.z * inv;
                const float c = u0 * t0 + u1 * t1 + u2 * t2;
                loss += 1.0 - (double)c;
                o[0] = __float2bfloat16(-(t0 - c * u0) * inv);
                o[1] = __float2bfloat16(-(t1 - c * u1) * inv);
                o[2] = __float2bfloat16(-(t2 - c * u2) * inv);
            } else {
                loss += 1.0;
            }
        }
        uint4* dst = reinterpret_cast<uint4*>(g + p * kNout);
        dst[0] = reinterpret_cast<const uint4*>(o)[0];
        dst[1] = reinterpret_cast<const uint4*>(o)[1];
    }
    s_loss[threadIdx.x] = loss;
    s_cnt[threadIdx.x] = cnt;
    __syncthreads();
    for (int o = kRedThreads / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            s_loss[threadIdx.x] += s_loss[threadIdx.x + o];
            s_cnt[threadIdx.x] += s_cnt[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = s_loss[0];
        part[2 * blockIdx.x + 1] = s_cnt[0];
    }
}

// Sum of the loss partials in block order: red[0] = mean loss, red[1] = 1 / inside cells.
__global__ void k_loss_finalize(const double* __restrict__ part, int nblocks, double* __restrict__ red) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double l = 0.0, c = 0.0;
    for (int b = 0; b < nblocks; ++b) {
        l += part[2 * b];
        c += part[2 * b + 1];
    }
    red[0] = c > 0.0 ? l / c : 0.0;
    red[1] = c > 0.0 ? 1.0 / c : 0.0;
}

// Per-block column sums of g [P][NN] (bias gradient), FP32 partials [block][NN].
template <int NN>
__global__ void __launch_bounds__(kRedThreads) k_bias_part(const __nv_bfloat16* __restrict__ g, long long total,
                                                           float* __restrict__ part) {
    __shared__ float s[kRedThreads / NN][NN];
    constexpr int ROWS = kRedThreads / NN;
    const int c = threadIdx.x % NN, r = threadIdx.x / NN;
    float acc = 0.0f;
    for (long long p = (long long)blockIdx.x * ROWS + r; p < total; p += (long long)gridDim.x * ROWS)
        acc += __bfloat162float(g[p * NN + c]);
    s[r][c] = acc;
    __syncthreads();
    if (r == 0) {
        float v = 0.0f;
        for (int q = 0; q < ROWS; ++q) v += s[q][c];
        part[blockIdx.x * NN + c] = v;
    }
}

// Gradient of one layer in the flat parameter layout (W[cout][3][3][cin_real] then
// b[cout_real]) from the CTA partials, summed in CTA order.
__global__ void k_grad_reduce(const float* __restrict__ wpart, int nwb, int rows_per_cta, int nn,
                              const float* __restrict__ bpart, int nbb, int cin_pad, int cin_real, int cout_real,
                              float* __restrict__ grad) {
    const int nw = cout_real * 9 * cin_real;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nw + cout_real; i += gridDim.x * blockDim.x) {
        float s = 0.0f;
        if (i < nw) {
            const int co = i / (9 * cin_real), r = i - co * 9 * cin_real, tap = r / cin_real, ci = r - tap * cin_real;
            const int m = tap * cin_pad + ci;
            for (int b = 0; b < nwb; ++b) s += wpart[((size_t)b * rows_per_cta + m) * nn + co];
        } else {
            const int co = i - nw;
            for (int b = 0; b < nbb; ++b) s += bpart[b * nn + co];
        }
        grad[i] = s;
    }
}

// Geometry of one layer in the flat parameter vector.
struct LayerDims {
    int off, cin_real, cout_real, cin_pad, cout_pad;
};
struct NetDims {
    LayerDims l[kLayers];
    int n;
};

__device__ __forceinline__ int layer_of(const NetDims& d, int i) {
    int l = 0;
#pragma unroll
    for (int q = 1; q < kLayers; ++q)
        if (i >= d.l[q].off) l = q;
    return l;
}

// Adam step on the FP32 master parameters (gradient = raw gradient * red[1]) and
// the BF16 weight layouts: forward wf[l][co][tap*cin_pad + ci], input-gradient
// wd[l][ci][(8 - tap)*cout_pad + co], bias bf[l][co].  step_scale1/2 = 1 / (1 - beta^t).
__global__ void k_adam_pack(NetDims d, float* __restrict__ w, float* __restrict__ mom, float* __restrict__ vel,
                            const float* __restrict__ graw, const double* __restrict__ red, float lr, float beta1,
                            float beta2, float eps, float bc1, float bc2, int update,
                            __nv_bfloat16* const* __restrict__ wf, float* const* __restrict__ bf,
                            __nv_bfloat16* const* __restrict__ wd) {
    const float scale = red ? (float)red[1] : 1.0f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.n; i += gridDim.x * blockDim.x) {
        float wi = w[i];
        if (update) {
            const float gi = graw[i] * scale;
            const float m = beta1 * mom[i] + (1.0f - beta1) * gi;
            const float v = beta2 * vel[i] + (1.0f - beta2) * gi * gi;
            mom[i] = m;
            vel[i] = v;
            wi -= lr * (m * bc1) / (sqrtf(v * bc2) + eps);
            w[i] = wi;
        }
        const int l = layer_of(d, i);
        const LayerDims& L = d.l[l];
        const int r = i - L.off, nw = L.cout_real * 9 * L.cin_real;
        if (r < nw) {
            const int co = r / (9 * L.cin_real), q = r - co * 9 * L.cin_real, tap = q / L.cin_real,
                      ci = q - tap * L.cin_real;
            const __nv_bfloat16 b = __float2bfloat16(wi);
            wf[l][(size_t)co * 9 * L.cin_pad + tap * L.cin_pad + ci] = b;
            if (wd[l]) wd[l][(size_t)ci * 9 * L.cout_pad + (8 - tap) * L.cout_pad + co] = b;
        } else {
            bf[l][r - nw] = wi;
        }
    }
}

// ---------------------------------------------------------------------------
// Host side: the trainer
// ---------------------------------------------------------------------------
static const int kTrCinReal[kLayers] = {7, kCh, kCh, kCh, kCh, kCh};
static const int kTrCoutReal[kLayers] = {kCh, kCh, kCh, kCh, kCh, 3};

struct Trainer {
    int device = 0;
    cudaStream_t stream = nullptr;
    NetDims dims{};
    long long cap_cells = 0;
    int cap_img = 0;
    int n = 0;
    long long steps = 0;
    long long spin = kMbarSpinLimit;
    std::vector<void*> allocs;
    float *w = nullptr, *mom = nullptr, *vel = nullptr, *graw = nullptr;
    __nv_bfloat16* wf[kLayers] = {};
    __nv_bfloat16* wd[kLayers] = {};
    float* bf[kLayers] = {};
    __nv_bfloat16** d_wf = nullptr;
    __nv_bfloat16** d_wd = nullptr;
    float** d_bf = nullptr;
    __nv_bfloat16* x0 = nullptr;        // [cap][16]
    __nv_bfloat16* h[kLayers - 1] = {}; // [cap][32] post-ReLU activations
    float* out32 = nullptr;             // [cap][4]
    __nv_bfloat16* g[2] = {};           // [cap][32] output gradients (ping-pong)
    float* wpart = nullptr;             // [wg_ctas][384][32]
    float* bpart = nullptr;             // [bias blocks][32]
    double* lpart = nullptr;            // [loss blocks][2]
    double* red = nullptr;              // [0] mean loss, [1] 1 / inside cells
    int* err = nullptr;
    int wg_ctas = 0, bias_blocks = 0, loss_blocks = 0;
};

static cudaError_t tr_alloc(Trainer* tr, void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
    if (e == cudaSuccess) {
        tr->allocs.push_back(*p);
        e = cudaMemset(*p, 0, bytes ? bytes : 16);
    }
    return e;
}

void trainer_destroy(Trainer* tr) {
    if (!tr) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(tr->device);
    if (tr->stream) cudaStreamSynchronize(tr->stream);
    for (void* p : tr->allocs) cudaFree(p);
    if (tr->stream) cudaStreamDestroy(tr->stream);
    cudaSetDevice(prev);
    delete tr;
}

static cudaError_t trainer_set_attrs() {
    cudaError_t e = cudaSuccess;
    const int smax = (int)conv_smem_bytes(kCh, kCh);
    auto set = [&](const void* f, int bytes) {
        if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    };
    set((const void*)k_conv3x3_tc<kCh, EPI_HIDDEN, float>, smax);
    set((const void*)k_conv3x3_tc<kNout, EPI_FINAL_RAW, float>, smax);
    set((const void*)k_conv3x3_tc<kCh, EPI_DGRAD, float>, smax);
    const int wg3 = 3 * kTile * kWgKC * 2 + 32 * kWgKC * 2;
    set((const void*)k_wgrad_tc<3, 32>, wg3);
    set((const void*)k_wgrad_tc<3, 16>, wg3);
    set((const void*)k_wgrad_tc<2, 32>, wg3);
    return e;
}

// params: FP32 flat vector (per layer W[cout][3][3][cin] then b[cout]); max_cells:
// the largest minibatch (images x cells) a step will be given.
cudaError_t trainer_create(const float* params, long long n, int device, long long max_cells, Trainer** out) {
    long long count = 0;
    for (int l = 0; l < kLayers; ++l) count += (long long)kTrCoutReal[l] * 9 * kTrCinReal[l] + kTrCoutReal[l];
    if (n != count || max_cells < 1) return cudaErrorInvalidValue;
    Trainer* tr = new Trainer();
    tr->device = device;
    tr->n = (int)n;
    tr->cap_cells = max_cells;
    int off = 0;
    for (int l = 0; l < kLayers; ++l) {
        LayerDims& L = tr->dims.l[l];
        L.off = off;
        L.cin_real = kTrCinReal[l];
        L.cout_real = kTrCoutReal[l];
        L.cin_pad = l == 0 ? kCin0 : kCh;
        L.cout_pad = l == kLayers - 1 ? kNout : kCh;
        off += L.cout_real * 9 * L.cin_real + L.cout_real;
    }
    tr->dims.n = off;
    cudaError_t e = cudaStreamCreateWithFlags(&tr->stream, cudaStreamNonBlocking);
    auto A = [&](auto** p, size_t bytes) {
        if (e == cudaSuccess) e = tr_alloc(tr, reinterpret_cast<void**>(p), bytes);
    };
    A(&tr->w, sizeof(float) * n);
    A(&tr->mom, sizeof(float) * n);
    A(&tr->vel, sizeof(float) * n);
    A(&tr->graw, sizeof(float) * n);
    for (int l = 0; l < kLayers; ++l) {
        const LayerDims& L = tr->dims.l[l];
        A(&tr->wf[l], sizeof(__nv_bfloat16) * (size_t)L.cout_pad * 9 * L.cin_pad);
        A(&tr->bf[l], sizeof(float) * (size_t)L.cout_pad);
        if (l > 0) A(&tr->wd[l], sizeof(__nv_bfloat16) * (size_t)L.cin_pad * 9 * L.cout_pad);
    }
    A(&tr->d_wf, sizeof(void*) * kLayers);
    A(&tr->d_wd, sizeof(void*) * kLayers);
    A(&tr->d_bf, sizeof(void*) * kLayers);
    A(&tr->x0, sizeof(__nv_bfloat16) * (size_t)max_cells * kCin0);
    for (int l = 0; l < kLayers - 1; ++l) A(&tr->h[l], sizeof(__nv_bfloat16) * (size_t)max_cells * kCh);
    A(&tr->out32, sizeof(float) * (size_t)max_cells * 4);
    A(&tr->g[0], sizeof(__nv_bfloat16) * (size_t)max_cells * kCh);
    A(&tr->g[1], sizeof(__nv_bfloat16) * (size_t)max_cells * kCh);
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    tr->wg_ctas = nsm * 4;
    tr->bias_blocks = nsm * 4;
    tr->loss_blocks = nsm * 4;
    A(&tr->wpart, sizeof(float) * (size_t)tr->wg_ctas * 3 * kTile * kCh);
    A(&tr->bpart, sizeof(float) * (size_t)tr->bias_blocks * kCh);
    A(&tr->lpart, sizeof(double) * (size_t)tr->loss_blocks * 2);
    A(&tr->red, sizeof(double) * 2);
    A(&tr->err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(tr->w, params, sizeof(float) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(tr->d_wf, tr->wf, sizeof(void*) * kLayers, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(tr->d_wd, tr->wd, sizeof(void*) * kLayers, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(tr->d_bf, tr->bf, sizeof(void*) * kLayers, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = trainer_set_attrs();
    if (e == cudaSuccess) {
        k_adam_pack<<<64, 256, 0, tr->stream>>>(tr->dims, tr->w, tr->mom, tr->vel, tr->graw, nullptr, 0.f, 0.f, 0.f,
                                                 0.f, 1.f, 1.f, 0, tr->d_wf, tr->d_bf, tr->d_wd);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(tr->stream);
    if (e != cudaSuccess) {
        trainer_destroy(tr);
        return e;
    }
    *out = tr;
    return cudaSuccess;
}

void trainer_set_spin_limit(Trainer* tr, long long polls) { tr->spin = polls; }
int trainer_error(Trainer* tr) {
    int v = 0;
    if (cudaMemcpy(&v, tr->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return 1;
    return v;
}

static Layer fwd_layer(const Trainer* tr, int l) {
    const LayerDims& L = tr->dims.l[l];
    return Layer{tr->wf[l], tr->bf[l], L.cin_pad, L.cout_pad, L.cout_real, l < kLayers - 1 ? 1 : 0};
}

// Forward, loss and gradients of one minibatch: nimg films of ny x nx cells, device
// inputs m0 (SoA planes, image stride 3*ny*nx), mask (nullable), bext [nimg][3]
// double, target (SoA planes).  Leaves the raw gradient in tr->graw and the mean
// loss / 1 / inside count in tr->red.
cudaError_t trainer_backprop(Trainer* tr, int nimg, int ny, int nx, const float* m0, const uint8_t* mask,
                             const double* bext, const float* target) {
    const long long hw = (long long)ny * nx, P = hw * nimg;
    if (P < 1 || P > tr->cap_cells) return cudaErrorInvalidValue;
    cudaStream_t s = tr->stream;
    cudaError_t e = cudaMemsetAsync(tr->err, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    k_ws_input<float><<<(unsigned)std::min<long long>((P + 255) / 256, 148 * 16), 256, 0, s>>>(m0, mask, bext, nimg,
                                                                                             hw, tr->x0);
    // forward
    const __nv_bfloat16* cur = tr->x0;
    for (int l = 0; l < kLayers; ++l) {
        const Layer L = fwd_layer(tr, l);
        if (l < kLayers - 1) {
            e = conv_launch<kCh, EPI_HIDDEN, float>(cur, nimg, ny, nx, L, tr->h[l], nullptr, nullptr, nullptr, nullptr,
                                                    tr->err, tr->spin, s);
            cur = tr->h[l];
        } else {
            e = conv_launch<kNout, EPI_FINAL_RAW, float>(cur, nimg, ny, nx, L, nullptr, nullptr, tr->out32, nullptr,
                                                         nullptr, tr->err, tr->spin, s);
        }
        if (e != cudaSuccess) return e;
    }
    // loss and its gradient (layer 5 output gradient, 16 channels, in g[0])
    k_cos_loss<<<tr->loss_blocks, kRedThreads, 0, s>>>(tr->out32, target, mask, nimg, hw, tr->g[0], tr->lpart);
    k_loss_finalize<<<1, 1, 0, s>>>(tr->lpart, tr->loss_blocks, tr->red);
    // backward
    const long long per_cta = ((P + tr->wg_ctas - 1) / tr->wg_ctas + kWgKC - 1) / kWgKC * kWgKC;
    const int wg_grid = (int)((P + per_cta - 1) / per_cta);
    const int wg_smem = 3 * kTile * kWgKC * 2 + 32 * kWgKC * 2;
    int gi = 0;
    for (int l = kLayers - 1; l >= 0; --l) {
        const LayerDims& D = tr->dims.l[l];
        const __nv_bfloat16* a = l == 0 ? tr->x0 : tr->h[l - 1];
        const __nv_bfloat16* gl = tr->g[gi];
        const int nt = (9 * D.cin_pad + kTile - 1) / kTile;
        if (D.cout_pad == 32 && nt == 3)
            k_wgrad_tc<3, 32><<<wg_grid, 128, wg_smem, s>>>(a, D.cin_pad, gl, nimg, ny, nx, per_cta, tr->wpart,
                                                            tr->err, tr->spin);
        else if (D.cout_pad == 16 && nt == 3)
            k_wgrad_tc<3, 16><<<wg_grid, 128, wg_smem, s>>>(a, D.cin_pad, gl, nimg, ny, nx, per_cta, tr->wpart,
                                                            tr->err, tr->spin);
        else
            k_wgrad_tc<2, 32><<<wg_grid, 128, wg_smem, s>>>(a, D.cin_pad, gl, nimg, ny, nx, per_cta, tr->wpart,
                                                            tr->err, tr->spin);
        if (D.cout_pad == 32)
            k_bias_part<32><<<tr->bias_blocks, kRedThreads, 0, s>>>(gl, P, tr->bpart);
        else
            k_bias_part<16><<<tr->bias_blocks, kRedThreads, 0, s>>>(gl, P, tr->bpart);
        k_grad_reduce<<<(D.cout_real * 9 * D.cin_real + D.cout_real + 255) / 256, 256, 0, s>>>(
            tr->wpart, wg_grid, nt * kTile, D.cout_pad, tr->bpart, tr->bias_blocks, D.cin_pad, D.cin_real,
            D.cout_real, tr->graw + D.off);
        if (l > 0) {
            // g_{l-1} = conv(g_l, W_l transposed / flipped) * (h_{l-1} > 0)
            const Layer Ld{tr->wd[l], nullptr, D.cout_pad, D.cin_pad, D.cin_pad, 0};
            e = conv_launch<kCh, EPI_DGRAD, float>(gl, nimg, ny, nx, Ld, tr->g[gi ^ 1], nullptr, nullptr, nullptr,
                                                   tr->h[l - 1], tr->err, tr->spin, s);
            if (e != cudaSuccess) return e;
            gi ^= 1;
        }
    }
    return cudaGetLastError();
}

cudaError_t trainer_update(Trainer* tr, float lr, float beta1, float beta2, float eps) {
    tr->steps += 1;
    const float bc1 = 1.0f / (1.0f - powf(beta1, (float)tr->steps));
    const float bc2 = 1.0f / (1.0f - powf(beta2, (float)tr->steps));
    k_adam_pack<<<64, 256, 0, tr->stream>>>(tr->dims, tr->w, tr->mom, tr->vel, tr->graw, tr->red, lr, beta1, beta2,
                                            eps, bc1, bc2, 1, tr->d_wf, tr->d_bf, tr->d_wd);
    return cudaGetLastError();
}

// Mean loss of the last backprop and, with grad != null, the gradient of the mean
// loss (raw gradient / inside cells) on the host; synchronises the stream.
cudaError_t trainer_read(Trainer* tr, double* loss, float* grad) {
    double red[2];
    cudaError_t e = cudaMemcpyAsync(red, tr->red, sizeof(red), cudaMemcpyDeviceToHost, tr->stream);
    if (e == cudaSuccess && grad)
        e = cudaMemcpyAsync(grad, tr->graw, sizeof(float) * tr->n, cudaMemcpyDeviceToHost, tr->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(tr->stream);
    if (e != cudaSuccess) return e;
    if (loss) *loss = red[0];
    if (grad)
        for (int i = 0; i < tr->n; ++i) grad[i] = (float)((double)grad[i] * red[1]);
    return cudaSuccess;
}

cudaError_t trainer_params(Trainer* tr, float* out) {
    cudaError_t e = cudaMemcpyAsync(out, tr->w, sizeof(float) * tr->n, cudaMemcpyDeviceToHost, tr->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(tr->stream);
    return e;
}

cudaError_t trainer_set_stream_sync(Trainer* tr) { return cudaStreamSynchronize(tr->stream); }

}  // namespace ws
}  // namespace llg

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
#include <cstdarg>
#include <cstdio>

#include "build_api.h"

namespace llg {
int ctx_device(const llg_ctx* c);
}

struct llg_wstrain {
    llg::ws::Trainer* tr;
};

static int tr_fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    llg_set_error_message(buf);
    return code;
}

static int tr_bind(llg_wstrain* t) {
    if (!t || !t->tr) return tr_fail(LLG_ERR_INVALID, "null trainer");
    cudaError_t e = cudaSetDevice(t->tr->device);
    return e == cudaSuccess ? LLG_OK : tr_fail(LLG_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
}

extern "C" {

int llg_wstrain_create(llg_ctx* ctx, const float* params, int64_t n_params, int64_t max_cells, llg_wstrain** out) {
    if (!ctx || !params || !out) return tr_fail(LLG_ERR_INVALID, "null argument");
    if (n_params != llg::ws::net_param_count())
        return tr_fail(LLG_ERR_INVALID, "expected %lld parameters, got %lld", (long long)llg::ws::net_param_count(),
                       (long long)n_params);
    if (max_cells < 1 || max_cells > (1LL << 28)) return tr_fail(LLG_ERR_INVALID, "bad max_cells %lld",
                                                                 (long long)max_cells);
    const int dev = llg::ctx_device(ctx);
    cudaError_t e = cudaSetDevice(dev);
    if (e != cudaSuccess) return tr_fail(LLG_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
    llg::ws::Trainer* tr = nullptr;
    e = llg::ws::trainer_create(params, n_params, dev, max_cells, &tr);
    if (e == cudaErrorMemoryAllocation) return tr_fail(LLG_ERR_OOM, "trainer: out of device memory");
    if (e != cudaSuccess) return tr_fail(LLG_ERR_CUDA, "trainer: %s", cudaGetErrorString(e));
    *out = new llg_wstrain{tr};
    return LLG_OK;
}

int llg_wstrain_destroy(llg_wstrain* t) {
    if (!t) return LLG_OK;
    llg::ws::trainer_destroy(t->tr);
    delete t;
    return LLG_OK;
}

int llg_wstrain_set_spin_limit(llg_wstrain* t, int64_t polls) {
    int rc = tr_bind(t);
    if (rc) return rc;
    if (polls < 0) return tr_fail(LLG_ERR_INVALID, "negative spin limit");
    llg::ws::trainer_set_spin_limit(t->tr, polls);
    return LLG_OK;
}

static int tr_check_batch(int64_t nimg, int64_t ny, int64_t nx, const float* m0, const double* bext,
                          const float* target) {
    if (!m0 || !bext || !target) return tr_fail(LLG_ERR_INVALID, "null device pointer");
    if (nimg < 1 || ny < 1 || nx < 1 || nimg * ny * nx > (1LL << 28))
        return tr_fail(LLG_ERR_INVALID, "bad sizes %lld x %lld x %lld", (long long)nimg, (long long)ny,
                       (long long)nx);
    return LLG_OK;
}

int llg_wstrain_gradients(llg_wstrain* t, int64_t nimg, int64_t ny, int64_t nx, const float* m0, const uint8_t* mask,
                          const double* bext, const float* target, double* loss, float* grad) {
    int rc = tr_bind(t);
    if (!rc) rc = tr_check_batch(nimg, ny, nx, m0, bext, target);
    if (rc) return rc;
    if (nimg * ny * nx > t->tr->cap_cells)
        return tr_fail(LLG_ERR_INVALID, "minibatch of %lld cells exceeds the trainer's %lld",
                       (long long)(nimg * ny * nx), t->tr->cap_cells);
    cudaError_t e = llg::ws::trainer_backprop(t->tr, (int)nimg, (int)ny, (int)nx, m0, mask, bext, target);
    if (e == cudaSuccess) e = llg::ws::trainer_read(t->tr, loss, grad);
    if (e != cudaSuccess) return tr_fail(LLG_ERR_CUDA, "trainer gradients: %s", cudaGetErrorString(e));
    if (llg::ws::trainer_error(t->tr)) return tr_fail(LLG_ERR_TIMEOUT, "trainer: tensor-core wait timed out");
    return LLG_OK;
}

int llg_wstrain_step(llg_wstrain* t, int64_t nimg, int64_t ny, int64_t nx, const float* m0, const uint8_t* mask,
                     const double* bext, const float* target, float lr, float beta1, float beta2, float eps,
                     double* loss) {
    int rc = tr_bind(t);
    if (!rc) rc = tr_check_batch(nimg, ny, nx, m0, bext, target);
    if (rc) return rc;
    if (nimg * ny * nx > t->tr->cap_cells)
        return tr_fail(LLG_ERR_INVALID, "minibatch of %lld cells exceeds the trainer's %lld",
                       (long long)(nimg * ny * nx), t->tr->cap_cells);
    if (!(lr >= 0.0f) || !(beta1 >= 0.0f && beta1 < 1.0f) || !(beta2 >= 0.0f && beta2 < 1.0f) || !(eps > 0.0f))
        return tr_fail(LLG_ERR_INVALID, "bad Adam settings");
    cudaError_t e = llg::ws::trainer_backprop(t->tr, (int)nimg, (int)ny, (int)nx, m0, mask, bext, target);
    if (e == cudaSuccess) e = llg::ws::trainer_update(t->tr, lr, beta1, beta2, eps);
    if (e == cudaSuccess && loss) e = llg::ws::trainer_read(t->tr, loss, nullptr);
    if (e != cudaSuccess) return tr_fail(LLG_ERR_CUDA, "trainer step: %s", cudaGetErrorString(e));
    if (loss && llg::ws::trainer_error(t->tr)) return tr_fail(LLG_ERR_TIMEOUT, "trainer: tensor-core wait timed out");
    return LLG_OK;
}

int llg_wstrain_sync(llg_wstrain* t) {
    int rc = tr_bind(t);
    if (rc) return rc;
    cudaError_t e = llg::ws::trainer_set_stream_sync(t->tr);
    if (e != cudaSuccess) return tr_fail(LLG_ERR_CUDA, "trainer sync: %s", cudaGetErrorString(e));
    if (llg::ws::trainer_error(t->tr)) return tr_fail(LLG_ERR_TIMEOUT, "trainer: tensor-core wait timed out");
    return LLG_OK;
}

int llg_wstrain_get_params(llg_wstrain* t, float* out) {
    int rc = tr_bind(t);
    if (rc) return rc;
    if (!out) return tr_fail(LLG_ERR_INVALID, "null argument");
    cudaError_t e = llg::ws::trainer_params(t->tr, out);
    return e == cudaSuccess ? LLG_OK : tr_fail(LLG_ERR_CUDA, "trainer params: %s", cudaGetErrorString(e));
}

}  // extern "C"
