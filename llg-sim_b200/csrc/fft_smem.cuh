// fft_smem.cuh — the project's own shared-memory FFT for sm_100a.
//
// Batched complex FFTs of one runtime length L per call, data resident in
// shared memory, mixed-radix Stockham autosort passes (radix 8/4/2/3/5 in
// registers, any other prime factor by a direct small DFT), natural-order
// output.  Twiddles come from a table of exp(-2 pi i k / (2L)), k < 2L, so that
// the same table serves the zero-padding pre/post twiddles W_{2L}^n of the
// pruned 2L-point transforms used by the demag convolution.
#pragma once
#include "types.cuh"

namespace llg {

template <typename R>
struct __align__(2 * sizeof(R)) cx {
    R re, im;
};

template <typename R>
__device__ __forceinline__ cx<R> mkc(R a, R b) {
    cx<R> r;
    r.re = a;
    r.im = b;
    return r;
}
template <typename R>
__device__ __forceinline__ cx<R> operator+(cx<R> a, cx<R> b) { return mkc(a.re + b.re, a.im + b.im); }
template <typename R>
__device__ __forceinline__ cx<R> operator-(cx<R> a, cx<R> b) { return mkc(a.re - b.re, a.im - b.im); }
template <typename R>
__device__ __forceinline__ cx<R> cmul(cx<R> a, cx<R> b) {
    return mkc(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
// a * conj(b)
template <typename R>
__device__ __forceinline__ cx<R> cmulc(cx<R> a, cx<R> b) {
    return mkc(a.re * b.re + a.im * b.im, a.im * b.re - a.re * b.im);
}
template <typename R>
__device__ __forceinline__ cx<R> cscale(cx<R> a, R s) { return mkc(a.re * s, a.im * s); }
template <typename R>
__device__ __forceinline__ cx<R> conjc(cx<R> a) { return mkc(a.re, -a.im); }
// multiply by -i (forward) or +i (inverse)
template <typename R>
__device__ __forceinline__ cx<R> rot(cx<R> a, bool inv) { return inv ? mkc(-a.im, a.re) : mkc(a.im, -a.re); }

// twiddle W_L^idx = tw2[2*idx] (forward), conj for inverse
template <typename R>
__device__ __forceinline__ cx<R> twl(const cx<R>* tw2, int idx, bool inv) {
    cx<R> w = tw2[2 * idx];
    return inv ? conjc(w) : w;
}

template <typename R>
__device__ __forceinline__ void bfly2(cx<R>* v) {
    cx<R> a = v[0], b = v[1];
    v[0] = a + b;
    v[1] = a - b;
}
template <typename R>
__device__ __forceinline__ void bfly4(cx<R>* v, bool inv) {
    cx<R> s02 = v[0] + v[2], d02 = v[0] - v[2];
    cx<R> s13 = v[1] + v[3], d13 = v[1] - v[3];
    cx<R> r = rot(d13, inv);
    v[0] = s02 + s13;
    v[1] = d02 + r;
    v[2] = s02 - s13;
    v[3] = d02 - r;
}
template <typename R>
__device__ __forceinline__ void bfly8(cx<R>* v, bool inv) {
    const R h = (R)0.70710678118654752440;
    cx<R> e[4] = {v[0], v[2], v[4], v[6]};
    cx<R> o[4] = {v[1], v[3], v[5], v[7]};
    bfly4(e, inv);
    bfly4(o, inv);
    // o[q] *= w8^q
    cx<R> o1, o3;
    if (!inv) {
        o1 = mkc((o[1].re + o[1].im) * h, (o[1].im - o[1].re) * h);
        o3 = mkc((o[3].im - o[3].re) * h, (-o[3].re - o[3].im) * h);
    } else {
        o1 = mkc((o[1].re - o[1].im) * h, (o[1].re + o[1].im) * h);
        o3 = mkc((-o[3].re - o[3].im) * h, (o[3].re - o[3].im) * h);
    }
    cx<R> o2 = rot(o[2], inv);
    v[0] = e[0] + o[0];
    v[4] = e[0] - o[0];
    v[1] = e[1] + o1;
    v[5] = e[1] - o1;
    v[2] = e[2] + o2;
    v[6] = e[2] - o2;
    v[3] = e[3] + o3;
    v[7] = e[3] - o3;
}
template <typename R>
__device__ __forceinline__ void bfly3(cx<R>* v, bool inv) {
    const R s3 = (R)0.86602540378443864676;  // sqrt(3)/2
    cx<R> s = v[1] + v[2], d = v[1] - v[2];
    cx<R> t = mkc(v[0].re - (R)0.5 * s.re, v[0].im - (R)0.5 * s.im);
    cx<R> r = rot(cscale(d, s3), inv);
    v[0] = v[0] + s;
    v[1] = t + r;
    v[2] = t - r;
}
template <typename R>
__device__ __forceinline__ void bfly5(cx<R>* v, bool inv) {
    const R c1 = (R)0.30901699437494742410, c2 = (R)-0.80901699437494742410;
    const R s1 = (R)0.95105651629515357212, s2 = (R)0.58778525229247312917;
    cx<R> a1s = v[1] + v[4], a1d = v[1] - v[4];
    cx<R> a2s = v[2] + v[3], a2d = v[2] - v[3];
    cx<R> x0 = v[0];
    cx<R> p1 = mkc(x0.re + c1 * a1s.re + c2 * a2s.re, x0.im + c1 * a1s.im + c2 * a2s.im);
    cx<R> p2 = mkc(x0.re + c2 * a1s.re + c1 * a2s.re, x0.im + c2 * a1s.im + c1 * a2s.im);
    cx<R> q1 = mkc(s1 * a1d.re + s2 * a2d.re, s1 * a1d.im + s2 * a2d.im);
    cx<R> q2 = mkc(s2 * a1d.re - s1 * a2d.re, s2 * a1d.im - s1 * a2d.im);
    cx<R> r1 = rot(q1, inv), r2 = rot(q2, inv);  // -i*q (fwd)
    v[0] = x0 + a1s + a2s;
    v[1] = p1 + r1;
    v[4] = p1 - r1;
    v[2] = p2 + r2;
    v[3] = p2 - r2;
}

template <typename R, int P>
__device__ __forceinline__ void stockham_pass_fixed(const cx<R>* __restrict__ a, cx<R>* __restrict__ b, int nsig,
                                                    int L, int ns, const cx<R>* __restrict__ tw2, bool inv) {
    const int m = L / P;
    const int tstep = L / (ns * P);
    const int total = nsig * m;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        const int sig = t / m;
        const int j = t - sig * m;
        const int k = j % ns;
        const cx<R>* in = a + sig * L;
        cx<R> v[P];
#pragma unroll
        for (int r = 0; r < P; ++r) {
            cx<R> x = in[j + r * m];
            if (r > 0 && k > 0) x = cmul(x, twl(tw2, k * r * tstep, inv));
            v[r] = x;
        }
        if (P == 2) bfly2(v);
        if (P == 3) bfly3(v, inv);
        if (P == 4) bfly4(v, inv);
        if (P == 5) bfly5(v, inv);
        if (P == 8) bfly8(v, inv);
        cx<R>* out = b + sig * L + (j / ns) * ns * P + k;
#pragma unroll
        for (int r = 0; r < P; ++r) out[r * ns] = v[r];
    }
}

// Any prime radix p: one output per thread iteration, direct p-term sum.
template <typename R>
__device__ void stockham_pass_generic(const cx<R>* __restrict__ a, cx<R>* __restrict__ b, int nsig, int L, int p,
                                      int ns, const cx<R>* __restrict__ tw2, bool inv) {
    const int m = L / p;
    const int tstep = L / (ns * p);
    const int total = nsig * L;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        const int sig = e / L;
        const int rem = e - sig * L;
        const int q = rem / m;
        const int j = rem - q * m;
        const int k = j % ns;
        const cx<R>* in = a + sig * L;
        cx<R> acc = in[j];
        for (int r = 1; r < p; ++r) {
            cx<R> x = in[j + r * m];
            if (k > 0) x = cmul(x, twl(tw2, k * r * tstep, inv));
            int qr = (q * r) % p;
            if (qr) x = cmul(x, twl(tw2, qr * m, inv));
            acc = acc + x;
        }
        b[sig * L + (j / ns) * ns * p + k + q * ns] = acc;
    }
}

// Runs the plan on nsig contiguous signals in `a` (scratch `b`, same size).
// Returns the buffer holding the result.  Ends with __syncthreads().
template <typename R>
__device__ cx<R>* fft_smem(cx<R>* a, cx<R>* b, int nsig, const FftPlan& plan, const cx<R>* __restrict__ tw2,
                           bool inv) {
    const int L = plan.L;
    int ns = 1;
    for (int s = 0; s < plan.npass; ++s) {
        const int p = plan.radix[s];
        switch (p) {
            case 2: stockham_pass_fixed<R, 2>(a, b, nsig, L, ns, tw2, inv); break;
            case 3: stockham_pass_fixed<R, 3>(a, b, nsig, L, ns, tw2, inv); break;
            case 4: stockham_pass_fixed<R, 4>(a, b, nsig, L, ns, tw2, inv); break;
            case 5: stockham_pass_fixed<R, 5>(a, b, nsig, L, ns, tw2, inv); break;
            case 8: stockham_pass_fixed<R, 8>(a, b, nsig, L, ns, tw2, inv); break;
            default: stockham_pass_generic<R>(a, b, nsig, L, p, ns, tw2, inv); break;
        }
        __syncthreads();
        cx<R>* t = a;
        a = b;
        b = t;
        ns *= p;
    }
    return a;
}

}  // namespace llg
