// conv_tc.cu — host side of the learned warm-start network's inference: weights
// packed for the tensor-core convolution (conv_tc.cuh), activation scratch, and
// the proposal of a film batch's states.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "conv_tc.cuh"

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
#include "build_api.h"

namespace llg {
namespace ws {

struct Net {
    int device = 0;
    int* err = nullptr;            // device flag: a tensor-core wait ran out during the last apply
    long long spin = kMbarSpinLimit;
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
    cudaFree(net->err);
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
    if (e == cudaSuccess) e = cudaMalloc(&net->err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(net->err, 0, sizeof(int));
    if (e == cudaSuccess) {
        const int smax = (int)conv_smem_bytes(kCh, kCh);
        e = cudaFuncSetAttribute(k_conv3x3_tc<kCh, EPI_HIDDEN, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 smax);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_conv3x3_tc<kNout, EPI_FINAL_NORM, float>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, smax);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_conv3x3_tc<kCh, EPI_HIDDEN, double>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, smax);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_conv3x3_tc<kNout, EPI_FINAL_NORM, double>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, smax);
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

// Whether a tensor-core wait of the last apply ran out (reads the flag that
// net_apply cleared at its start; call after the apply's stream is synchronised).
int net_error(Net* net) {
    int v = 0;
    if (cudaMemcpy(&v, net->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return 1;
    return v;
}

void net_set_spin_limit(Net* net, long long polls) { net->spin = polls; }

// Proposal for nimg images of ny x nx cells (SoA planes of R, image stride 3*ny*nx):
// m_out may alias m_in (the input is consumed by the first layer).
template <typename R>
cudaError_t net_apply(Net* net, const R* m_in, R* m_out, const uint8_t* mask, const double* bext_host, int nimg,
                      int ny, int nx, cudaStream_t s) {
    const long long hw = (long long)ny * nx, cells = hw * nimg;
    if (cells <= 0) return cudaSuccess;
    cudaError_t e = ensure_scratch(net, cells, nimg);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(net->err, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(net->bext, bext_host, (size_t)nimg * 3 * sizeof(double), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    k_ws_input<R><<<(unsigned)std::min<long long>((cells + 255) / 256, 148 * 16), 256, 0, s>>>(m_in, mask, net->bext,
                                                                                              nimg, hw, net->x0);
    const __nv_bfloat16* cur = net->x0;
    for (int l = 0; l < kLayers; ++l) {
        const Layer& L = net->L[l];
        if (l < kLayers - 1) {
            __nv_bfloat16* nxt = net->h[l & 1];
            e = conv_launch<kCh, EPI_HIDDEN, R>(cur, nimg, ny, nx, L, nxt, nullptr, nullptr, nullptr, nullptr, net->err,
                                                net->spin, s);
            cur = nxt;
        } else {
            e = conv_launch<kNout, EPI_FINAL_NORM, R>(cur, nimg, ny, nx, L, nullptr, m_out, nullptr, mask, nullptr,
                                                      net->err, net->spin, s);
        }
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
