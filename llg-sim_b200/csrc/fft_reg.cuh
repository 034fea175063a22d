// fft_reg.cuh — compile-time-specialised register FFTs (the fast path).
//
// A length-L transform is computed by a group of G = L/E threads, each holding
// E complex values in registers.  Pass 0 is a radix-E DFT entirely in
// registers; later passes (radix R_i dividing E) read their inputs from a
// padded shared-memory exchange buffer, apply twiddles from per-pass tables
// laid out [r][k] (so that a warp reads consecutive entries), and run E/R_i
// register DFTs.  Radix-16/32 DFTs are built by Cooley–Tukey from radix-4/8
// with compile-time internal twiddles.  L = 1024 in FP32 is two radix-32
// passes with a single shared-memory exchange.
#pragma once
#include "fft_smem.cuh"

namespace llg {

// cos(2*pi*j/64), j < 64 (multiples of pi/2 exact).
__device__ constexpr double kCos64[64] = {
    1.0, 0.9951847266721969, 0.9807852804032304, 0.9569403357322088,
    0.9238795325112867, 0.881921264348355, 0.8314696123025452, 0.773010453362737,
    0.7071067811865476, 0.6343932841636455, 0.5555702330196023, 0.4713967368259978,
    0.38268343236508984, 0.29028467725446233, 0.19509032201612833, 0.09801714032956077,
    0.0, -0.09801714032956065, -0.1950903220161282, -0.29028467725446216,
    -0.3826834323650897, -0.4713967368259977, -0.555570233019602, -0.6343932841636454,
    -0.7071067811865475, -0.773010453362737, -0.8314696123025453, -0.8819212643483549,
    -0.9238795325112867, -0.9569403357322088, -0.9807852804032304, -0.9951847266721968,
    -1.0, -0.9951847266721969, -0.9807852804032304, -0.9569403357322089,
    -0.9238795325112868, -0.881921264348355, -0.8314696123025455, -0.7730104533627371,
    -0.7071067811865477, -0.6343932841636459, -0.5555702330196022, -0.47139673682599786,
    -0.38268343236509034, -0.29028467725446244, -0.19509032201612866, -0.09801714032956045,
    0.0, 0.09801714032956009, 0.1950903220161283, 0.29028467725446205,
    0.38268343236509, 0.4713967368259976, 0.5555702330196018, 0.6343932841636456,
    0.7071067811865474, 0.7730104533627367, 0.8314696123025452, 0.8819212643483548,
    0.9238795325112865, 0.9569403357322088, 0.9807852804032303, 0.9951847266721969};

// x * W_N^k with W_N = exp(-2 pi i / N) (forward) or its conjugate (inverse);
// N divides 64 and k is a compile-time constant.
template <typename R, int N, int K, bool INV>
__device__ __forceinline__ cx<R> twc(cx<R> x) {
    constexpr int j = ((K * (64 / N)) % 64 + 64) % 64;
    if constexpr (j == 0) {
        return x;
    } else if constexpr (j == 16) {  // -i (fwd)
        return INV ? mkc(-x.im, x.re) : mkc(x.im, -x.re);
    } else if constexpr (j == 32) {
        return mkc(-x.re, -x.im);
    } else if constexpr (j == 48) {  // +i (fwd)
        return INV ? mkc(x.im, -x.re) : mkc(-x.im, x.re);
    } else {
        constexpr double c = kCos64[j];
        constexpr double s = INV ? kCos64[(j + 48) % 64] : -kCos64[(j + 48) % 64];  // +/- sin(2 pi j/64)
        return mkc((R)c * x.re - (R)s * x.im, (R)c * x.im + (R)s * x.re);
    }
}

// In-register DFT of N points stored in v[O + S*n], n < N; result in natural
// order at the same slots.
template <typename R, int N, bool INV>
struct RegDFT {
    template <int O, int S, int M>
    __device__ __forceinline__ static void run(cx<R> (&v)[M]) {
        if constexpr (N == 1) {
        } else if constexpr (N == 2) {
            cx<R> a = v[O], b = v[O + S];
            v[O] = a + b;
            v[O + S] = a - b;
        } else if constexpr (N == 4) {
            cx<R> x[4] = {v[O], v[O + S], v[O + 2 * S], v[O + 3 * S]};
            bfly4(x, INV);
            v[O] = x[0]; v[O + S] = x[1]; v[O + 2 * S] = x[2]; v[O + 3 * S] = x[3];
        } else if constexpr (N == 8) {
            cx<R> x[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) x[i] = v[O + i * S];
            bfly8(x, INV);
#pragma unroll
            for (int i = 0; i < 8; ++i) v[O + i * S] = x[i];
        } else {
            // N = N1*N2, input n = N2*n1 + n2, output k = k1 + N1*k2
            constexpr int N1 = 4;
            constexpr int N2 = N / N1;
            cx<R> y[N];
            sub1<O, S, N1, N2, 0>(v, y);
            sub2<O, S, N1, N2, 0>(v, y);
        }
    }

   private:
    template <int O, int S, int N1, int N2, int n2, int M>
    __device__ __forceinline__ static void sub1(cx<R> (&v)[M], cx<R> (&y)[N]) {
        if constexpr (n2 < N2) {
            cx<R> a[N1];
#pragma unroll
            for (int n1 = 0; n1 < N1; ++n1) a[n1] = v[O + S * (N2 * n1 + n2)];
            RegDFT<R, N1, INV>::template run<0, 1>(a);
            tw_row<n2, N1, 0>(a, y);
            sub1<O, S, N1, N2, n2 + 1>(v, y);
        }
    }
    template <int n2, int N1, int k1>
    __device__ __forceinline__ static void tw_row(cx<R> (&a)[N1], cx<R> (&y)[N]) {
        if constexpr (k1 < N1) {
            y[n2 * N1 + k1] = twc<R, N, n2 * k1, INV>(a[k1]);
            tw_row<n2, N1, k1 + 1>(a, y);
        }
    }
    template <int O, int S, int N1, int N2, int k1, int M>
    __device__ __forceinline__ static void sub2(cx<R> (&v)[M], cx<R> (&y)[N]) {
        if constexpr (k1 < N1) {
            cx<R> b[N2];
#pragma unroll
            for (int n2 = 0; n2 < N2; ++n2) b[n2] = y[n2 * N1 + k1];
            RegDFT<R, N2, INV>::template run<0, 1>(b);
#pragma unroll
            for (int k2 = 0; k2 < N2; ++k2) v[O + S * (k1 + N1 * k2)] = b[k2];
            sub2<O, S, N1, N2, k1 + 1>(v, y);
        }
    }
};

// Pass plans.  E = registers (complex) per thread = first radix; later passes
// have radices RAD1, RAD2 dividing E.  V = 0 is the default plan of a length;
// V = 1 an alternative with half the registers per thread and twice the threads
// per transform (ok = false where a length has none), chosen per launch segment by
// the engine's autotuner.
template <typename R, int L, int V = 0>
struct FPlan {
    static constexpr bool ok = false;
    static constexpr int E = 1, NP = 1, G = L, RAD1 = 1, RAD2 = 1;
};
#define LLG_PLAN(RT, LL, VV, EE, NPASS, R1, R2)                      \
    template <>                                                      \
    struct FPlan<RT, LL, VV> {                                       \
        static constexpr bool ok = true;                             \
        static constexpr int E = EE, NP = NPASS, G = LL / EE;        \
        static constexpr int RAD1 = R1, RAD2 = R2;                   \
    };
//      type    L     V  E   NP  R1  R2
LLG_PLAN(float, 16, 0, 16, 1, 1, 1)
LLG_PLAN(float, 32, 0, 8, 2, 4, 1)
LLG_PLAN(float, 64, 0, 8, 2, 8, 1)
LLG_PLAN(float, 128, 0, 16, 2, 8, 1)
LLG_PLAN(float, 256, 0, 16, 2, 16, 1)
LLG_PLAN(float, 512, 0, 32, 2, 16, 1)
LLG_PLAN(float, 1024, 0, 32, 2, 32, 1)
LLG_PLAN(float, 2048, 0, 32, 3, 32, 2)
LLG_PLAN(double, 16, 0, 16, 1, 1, 1)
LLG_PLAN(double, 32, 0, 8, 2, 4, 1)
LLG_PLAN(double, 64, 0, 8, 2, 8, 1)
LLG_PLAN(double, 128, 0, 16, 2, 8, 1)
LLG_PLAN(double, 256, 0, 16, 2, 16, 1)
LLG_PLAN(double, 512, 0, 16, 3, 16, 2)
LLG_PLAN(double, 1024, 0, 16, 3, 16, 4)
LLG_PLAN(double, 2048, 0, 16, 3, 16, 8)
// alternatives: half the registers per thread
LLG_PLAN(float, 128, 1, 8, 3, 8, 2)
LLG_PLAN(float, 256, 1, 8, 3, 8, 4)
LLG_PLAN(float, 512, 1, 16, 3, 16, 2)
LLG_PLAN(float, 1024, 1, 16, 3, 16, 4)
LLG_PLAN(float, 2048, 1, 16, 3, 16, 8)
LLG_PLAN(double, 128, 1, 8, 3, 8, 2)
LLG_PLAN(double, 256, 1, 8, 3, 8, 4)
LLG_PLAN(double, 512, 1, 8, 3, 8, 8)
#undef LLG_PLAN

template <int L>
struct FastSize {
    static constexpr bool ok = L == 16 || L == 32 || L == 64 || L == 128 || L == 256 || L == 512 || L == 1024 ||
                               L == 2048;
};

// Padded shared-memory index: one pad slot per E entries (conflict-free for
// the pass exchange patterns used here).
template <int E>
__device__ __forceinline__ int padi(int i) {
    return i + i / E;
}
template <typename R, int L, int V = 0>
struct Pad {
    static constexpr int E = FPlan<R, L, V>::E;
    static constexpr int size = L + L / E;  // complex slots per signal buffer
};

// Twiddle tables of passes 1.. in [r][k] layout: pass with radix Rr and stride
// ns holds W_{ns*Rr}^{k*r} for r < Rr, k < ns.  Total entries:
template <typename R, int L, int V = 0>
struct TwTab {
    using P = FPlan<R, L, V>;
    static constexpr int ns1 = P::E;
    static constexpr int size1 = P::NP >= 2 ? P::RAD1 * ns1 : 0;
    static constexpr int ns2 = P::E * P::RAD1;
    static constexpr int size2 = P::NP >= 3 ? P::RAD2 * ns2 : 0;
    static constexpr int size = size1 + size2;
};

template <typename R, int RADIX, bool INV, int U, int NB, int E>
__device__ __forceinline__ void run_blocks(cx<R> (&v)[E]) {
    if constexpr (U < NB) {
        RegDFT<R, RADIX, INV>::template run<U * RADIX, 1>(v);
        run_blocks<R, RADIX, INV, U + 1, NB, E>(v);
    }
}

// One pass p >= 1: read inputs of this thread's butterflies from `buf`,
// twiddle, DFT in registers.
template <typename R, int L, int V, bool INV, int RADIX, int NS>
__device__ __forceinline__ void group_pass(cx<R> (&v)[FPlan<R, L, V>::E], int t, const cx<R>* buf, const cx<R>* tw) {
    using P = FPlan<R, L, V>;
    constexpr int E = P::E, G = P::G, NB = E / RADIX, STRIDE = L / RADIX;
#pragma unroll
    for (int u = 0; u < NB; ++u) {
        const int b = t + G * u;
        const int k = b % NS;
#pragma unroll
        for (int r = 0; r < RADIX; ++r) {
            cx<R> x = buf[padi<E>(b + r * STRIDE)];
            if (r > 0) {
                cx<R> w = tw[r * NS + k];
                x = INV ? cmulc(x, w) : cmul(x, w);
            }
            v[u * RADIX + r] = x;
        }
    }
    run_blocks<R, RADIX, INV, 0, NB, E>(v);
}

// Output index of register v[i] after the pass with radix RADIX and stride NS.
template <typename R, int L, int V, int RADIX, int NS>
__device__ __forceinline__ int pass_out_index(int t, int i) {
    constexpr int G = FPlan<R, L, V>::G;
    const int u = i / RADIX, q = i % RADIX;
    const int b = t + G * u;
    return (b / NS) * NS * RADIX + (b % NS) + q * NS;
}

// Barrier over the threads of one transform group: a warp (or the part of one
// holding whole groups) for G <= 32, the block otherwise.
template <int G>
__device__ __forceinline__ void group_sync() {
    if constexpr (G <= 32) __syncwarp();
    else __syncthreads();
}

// Full transform of one signal by its group.  On entry v[r] = x[t + G*r];
// on exit v[i] = X[out_index(t, i)].  `buf` is this signal's padded exchange
// buffer (only this group touches it inside); `tw` the pass tables.  Every
// thread of the block must call this the same number of times (it contains
// group_sync<G>(), a block barrier when G > 32).
template <typename R, int L, bool INV, int V = 0>
struct GroupFFT {
    using P = FPlan<R, L, V>;
    static constexpr int E = P::E, G = P::G, NP = P::NP;

    __device__ __forceinline__ static int out_index(int t, int i) {
        if constexpr (NP == 1) return t * E + i;
        else if constexpr (NP == 2) return pass_out_index<R, L, V, P::RAD1, E>(t, i);
        else return pass_out_index<R, L, V, P::RAD2, E * P::RAD1>(t, i);
    }

    __device__ __forceinline__ static void run(cx<R> (&v)[E], int t, cx<R>* buf, const cx<R>* tw) {
        RegDFT<R, E, INV>::template run<0, 1>(v);
        if constexpr (NP >= 2) {
#pragma unroll
            for (int q = 0; q < E; ++q) buf[padi<E>(t * E + q)] = v[q];
            group_sync<G>();
            group_pass<R, L, V, INV, P::RAD1, E>(v, t, buf, tw);
            if constexpr (NP >= 3) {
                group_sync<G>();
#pragma unroll
                for (int i = 0; i < E; ++i) buf[padi<E>(pass_out_index<R, L, V, P::RAD1, E>(t, i))] = v[i];
                group_sync<G>();
                group_pass<R, L, V, INV, P::RAD2, E * P::RAD1>(v, t, buf, tw + TwTab<R, L, V>::size1);
            }
        }
    }
};

}  // namespace llg
