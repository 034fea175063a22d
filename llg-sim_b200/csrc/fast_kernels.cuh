// fast_kernels.cuh — register-FFT versions of the three evaluation passes for
// power-of-two film sizes (16..2048).  Same data layout, same algorithm and
// same epilogue as field_kernels.cuh; the transforms use GroupFFT (fft_reg.cuh)
// with per-pass twiddle tables and the W_{2L}^n pre-twiddles resident in
// shared memory.
#pragma once
#include "field_kernels.cuh"
#include "fft_reg.cuh"

namespace llg {

// Row passes: T rows per block; signals: T packed xy rows and T/2 packed z
// row pairs, each as an even-bin and an odd-bin transform (s = 2g + parity).
template <typename R, int L>
struct RowCfg {
    using P = FPlan<R, L>;
    static constexpr int G = P::G, E = P::E;
    static constexpr int T = (64 / G) < 2 ? 2 : 64 / G;
    static constexpr int NGRP = T + T / 2;
    static constexpr int NSIG = 2 * NGRP;
    static constexpr int THREADS = NSIG * G;
    static constexpr int BUF = Pad<R, L>::size;
    static constexpr int SMEM_CX = NSIG * BUF + TwTab<R, L>::size + L;
    static constexpr size_t SMEM = sizeof(cx<R>) * (size_t)SMEM_CX;
};

// Column pass: NC columns per block, six signals per column (3 components x
// even / odd ky bins).
template <typename R, int L>
struct ColCfg {
    using P = FPlan<R, L>;
    static constexpr int G = P::G, E = P::E;
    static constexpr int NC = (32 / G) < 1 ? 1 : 32 / G;
    static constexpr int NSIG = 6 * NC;
    static constexpr int THREADS = NSIG * G;
    static constexpr int BUF = Pad<R, L>::size;
    static constexpr int SMEM_CX = NSIG * BUF + TwTab<R, L>::size + L;
    static constexpr size_t SMEM = sizeof(cx<R>) * (size_t)SMEM_CX;
};

template <typename R>
__device__ __forceinline__ void load_tables(cx<R>* twp, const cx<R>* __restrict__ gtwp, int ntwp, cx<R>* pre,
                                            const cx<R>* __restrict__ gpre, int L) {
    for (int i = threadIdx.x; i < ntwp; i += blockDim.x) twp[i] = gtwp[i];
    for (int i = threadIdx.x; i < L; i += blockDim.x) pre[i] = gpre[i];
}

// ---------------------------------------------------------------------------
template <typename R, int L>
__global__ void __launch_bounds__(RowCfg<R, L>::THREADS) k_row_forward_fast(const FilmDev* __restrict__ films,
                                                                            const WorkItem* __restrict__ items,
                                                                            int nitems, EvalSpec spec) {
    using C = RowCfg<R, L>;
    using FFT = GroupFFT<R, L, false>;
    constexpr int G = C::G, E = C::E, T = C::T, BUF = C::BUF;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<R>* buf = reinterpret_cast<cx<R>*>(smem_raw);
    cx<R>* twp = buf + C::NSIG * BUF;
    cx<R>* pre = twp + TwTab<R, L>::size;
    const int tid = threadIdx.x, s = tid / G, t = tid % G, g = s >> 1, par = s & 1;
    bool tables = false;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const WorkItem w = items[it];
        const FilmDev& F = films[w.film];
        const StepState* st = F.st;
        if (skip_item(spec, st)) continue;
        const bool do_fft = spec.demag && F.demag_mat;
        if (do_fft && !tables) {
            load_tables<R>(twp, reinterpret_cast<const cx<R>*>(F.twp_row), TwTab<R, L>::size, pre,
                           reinterpret_cast<const cx<R>*>(F.tw_row), L);
            tables = true;
        }
        const int ny = F.ny, n = L * ny;
        const int j0 = w.blk * T;
        const int cur = st->cur;
        const R* __restrict__ m0 = mbuf<R>(F, MB_M0, cur);
        R* __restrict__ ms = mbuf<R>(F, spec.m_in, cur);
        const double dt = st->dt;
        const R* kp[6];
        R cq[6];
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            kp[q] = q < spec.nterm ? kbuf<R>(F, spec.kidx[q], cur) : nullptr;
            cq[q] = q < spec.nterm ? (R)(dt * spec.a[q]) : (R)0;
        }
        const R Ms = (R)F.ms;
        for (int e = tid; e < T * L; e += C::THREADS) {
            const int r = e / L, i = e - r * L, j = j0 + r;
            R v[3] = {(R)0, (R)0, (R)0};
            if (j < ny) {
                const int idx = j * L + i;
                if (spec.nterm > 0) {
                    v[0] = m0[idx]; v[1] = m0[n + idx]; v[2] = m0[2 * n + idx];
#pragma unroll
                    for (int q = 0; q < 6; ++q) {
                        if (q < spec.nterm) {
                            const R* k = kp[q];
                            v[0] = v[0] + cq[q] * k[idx];
                            v[1] = v[1] + cq[q] * k[n + idx];
                            v[2] = v[2] + cq[q] * k[2 * n + idx];
                        }
                    }
                    if (cell_inside(F, idx)) normalize3(v);
                    else { v[0] = (R)0; v[1] = (R)0; v[2] = (R)0; }
                    ms[idx] = v[0]; ms[n + idx] = v[1]; ms[2 * n + idx] = v[2];
                } else {
                    v[0] = ms[idx]; v[1] = ms[n + idx]; v[2] = ms[2 * n + idx];
                }
            }
            if (do_fft) {
                buf[(2 * r) * BUF + padi<E>(i)] = mkc(Ms * v[0], Ms * v[1]);
                cx<R>* zp = &buf[(2 * (T + r / 2)) * BUF + padi<E>(i)];
                if ((r & 1) == 0) zp->re = Ms * v[2];
                else zp->im = Ms * v[2];
            }
        }
        if (!do_fft) continue;
        __syncthreads();
        cx<R> v[E];
        {
            const cx<R>* zb = buf + (2 * g) * BUF;
#pragma unroll
            for (int r = 0; r < E; ++r) {
                const int nn = t + G * r;
                cx<R> x = zb[padi<E>(nn)];
                v[r] = par ? cmul(x, pre[nn]) : x;
            }
        }
        __syncthreads();
        FFT::run(v, t, buf + s * BUF, twp);
        __syncthreads();
#pragma unroll
        for (int i = 0; i < E; ++i) buf[s * BUF + padi<E>(FFT::out_index(t, i))] = v[i];
        __syncthreads();
        cx<R>* __restrict__ X = reinterpret_cast<cx<R>*>(F.X);
        constexpr int K1 = L + 1, L2 = 2 * L;
        for (int e = tid; e < 3 * K1 * T; e += C::THREADS) {
            const int r = e % T, rest = e / T;
            const int k = rest % K1, c = rest / K1;
            const int j = j0 + r;
            if (j >= ny) continue;
            int gg, half;
            if (c < 2) { gg = r; half = c; }
            else { gg = T + r / 2; half = r & 1; }
            const int km = (L2 - k) % L2;
            const cx<R> zk = buf[(2 * gg + (k & 1)) * BUF + padi<E>(k >> 1)];
            const cx<R> zm = buf[(2 * gg + (km & 1)) * BUF + padi<E>(km >> 1)];
            cx<R> out;
            if (half == 0) out = mkc((R)0.5 * (zk.re + zm.re), (R)0.5 * (zk.im - zm.im));
            else out = mkc((R)0.5 * (zk.im + zm.im), (R)0.5 * (zm.re - zk.re));
            X[(c * K1 + k) * ny + j] = out;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
template <typename R, int L>
__global__ void __launch_bounds__(ColCfg<R, L>::THREADS) k_column_fast(const FilmDev* __restrict__ films,
                                                                       const WorkItem* __restrict__ items, int nitems,
                                                                       EvalSpec spec) {
    using C = ColCfg<R, L>;
    using FF = GroupFFT<R, L, false>;
    using FI = GroupFFT<R, L, true>;
    constexpr int G = C::G, E = C::E, BUF = C::BUF;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<R>* buf = reinterpret_cast<cx<R>*>(smem_raw);
    cx<R>* twp = buf + C::NSIG * BUF;
    cx<R>* pre = twp + TwTab<R, L>::size;
    const int tid = threadIdx.x, s = tid / G, t = tid % G;
    const int cl = s / 6, comp = (s % 6) >> 1, par = s & 1;
    bool tables = false;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const WorkItem w = items[it];
        const FilmDev& F = films[w.film];
        const StepState* st = F.st;
        if (skip_item(spec, st)) continue;
        if (!(spec.demag && F.demag_mat)) continue;
        if (!tables) {
            load_tables<R>(twp, reinterpret_cast<const cx<R>*>(F.twp_col), TwTab<R, L>::size, pre,
                           reinterpret_cast<const cx<R>*>(F.tw_col), L);
            tables = true;
            __syncthreads();
        }
        const int nx = F.nx, K1 = nx + 1;
        constexpr int ny = L;
        const int kx = w.blk * C::NC + cl;
        const bool valid = kx <= nx;
        cx<R>* __restrict__ X = reinterpret_cast<cx<R>*>(F.X);
        cx<R> v[E];
#pragma unroll
        for (int r = 0; r < E; ++r) {
            const int nn = t + G * r;
            cx<R> x = valid ? X[(size_t)(comp * K1 + kx) * ny + nn] : mkc((R)0, (R)0);
            v[r] = par ? cmul(x, pre[nn]) : x;
        }
        FF::run(v, t, buf + s * BUF, twp);
        __syncthreads();
#pragma unroll
        for (int i = 0; i < E; ++i) buf[s * BUF + padi<E>(FF::out_index(t, i))] = v[i];
        __syncthreads();
        {
            const r4<R>* __restrict__ Kp =
                reinterpret_cast<const r4<R>*>(F.Kpar) + ((size_t)(valid ? kx : 0) * 2 + par) * ny;
            const cx<R>* sx = buf + (6 * cl + 0 + par) * BUF;
            const cx<R>* sy = buf + (6 * cl + 2 + par) * BUF;
            const cx<R>* sz = buf + (6 * cl + 4 + par) * BUF;
#pragma unroll
            for (int r = 0; r < E; ++r) {
                const int kk = t + G * r;
                const r4<R> K = Kp[kk];
                const int pi = padi<E>(kk);
                cx<R> out;
                if (comp == 0) {
                    const cx<R> Mx = sx[pi], My = sy[pi];
                    out = mkc(K.x * Mx.re + K.y * My.re, K.x * Mx.im + K.y * My.im);
                } else if (comp == 1) {
                    const cx<R> Mx = sx[pi], My = sy[pi];
                    out = mkc(K.y * Mx.re + K.z * My.re, K.y * Mx.im + K.z * My.im);
                } else {
                    const cx<R> Mz = sz[pi];
                    out = mkc(K.w * Mz.re, K.w * Mz.im);
                }
                v[r] = out;
            }
        }
        __syncthreads();
        FI::run(v, t, buf + s * BUF, twp);
        __syncthreads();
        if (par) {
#pragma unroll
            for (int i = 0; i < E; ++i) buf[s * BUF + padi<E>(FI::out_index(t, i))] = v[i];
        }
        __syncthreads();
        if (!par && valid) {
            const cx<R>* ob = buf + (s + 1) * BUF;
#pragma unroll
            for (int i = 0; i < E; ++i) {
                const int nn = FI::out_index(t, i);
                X[(size_t)(comp * K1 + kx) * ny + nn] = v[i] + cmulc(ob[padi<E>(nn)], pre[nn]);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
template <typename R, int L, bool LEAN>
__global__ void __launch_bounds__(RowCfg<R, L>::THREADS) k_row_inverse_fast(const FilmDev* __restrict__ films,
                                                                            const WorkItem* __restrict__ items,
                                                                            int nitems, EvalSpec spec) {
    using C = RowCfg<R, L>;
    using FI = GroupFFT<R, L, true>;
    constexpr int G = C::G, E = C::E, T = C::T, BUF = C::BUF;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double sm_red[32 * RED_NSLOT];
    cx<R>* buf = reinterpret_cast<cx<R>*>(smem_raw);
    cx<R>* twp = buf + C::NSIG * BUF;
    cx<R>* pre = twp + TwTab<R, L>::size;
    const int tid = threadIdx.x, s = tid / G, t = tid % G, g = s >> 1, par = s & 1;
    bool tables = false;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const WorkItem w = items[it];
        const FilmDev& F = films[w.film];
        StepState* st = F.st;
        if (skip_item(spec, st)) continue;
        const bool do_fft = spec.demag && F.demag_mat;
        if (do_fft && !tables) {
            load_tables<R>(twp, reinterpret_cast<const cx<R>*>(F.twp_row), TwTab<R, L>::size, pre,
                           reinterpret_cast<const cx<R>*>(F.tw_row), L);
            tables = true;
            __syncthreads();
        }
        const int ny = F.ny;
        const int j0 = w.blk * T;
        if (do_fft) {
            const cx<R>* __restrict__ X = reinterpret_cast<const cx<R>*>(F.X);
            constexpr int K1 = L + 1, L2 = 2 * L;
            // stage this block's rows of the spectrum, [c][k][r], with contiguous
            // T-row chunks per (c, k) (the signal buffers are free here)
            cx<R>* stg = buf;
            for (int e = tid; e < 3 * K1 * T; e += C::THREADS) {
                const int r = e % T, ck = e / T;
                const int j = j0 + r;
                stg[e] = j < ny ? X[(size_t)ck * ny + j] : mkc((R)0, (R)0);
            }
            __syncthreads();
            auto xval = [&](int c, int k, int r) -> cx<R> {
                if (k <= L) return stg[(c * K1 + k) * T + r];
                return conjc(stg[(c * K1 + (L2 - k)) * T + r]);
            };
            cx<R> v[E];
#pragma unroll
            for (int r = 0; r < E; ++r) {
                const int k = 2 * (t + G * r) + par;
                cx<R> z;
                if (g < T) {
                    const cx<R> bx = xval(0, k, g), by = xval(1, k, g);
                    z = mkc(bx.re - by.im, bx.im + by.re);
                } else {
                    const int ra = 2 * (g - T);
                    const cx<R> za = xval(2, k, ra), zb = xval(2, k, ra + 1);
                    z = mkc(za.re - zb.im, za.im + zb.re);
                }
                v[r] = z;
            }
            __syncthreads();
            FI::run(v, t, buf + s * BUF, twp);
            __syncthreads();
            if (par) {
#pragma unroll
                for (int i = 0; i < E; ++i) buf[s * BUF + padi<E>(FI::out_index(t, i))] = v[i];
            }
            __syncthreads();
            if (!par) {
                const cx<R>* ob = buf + (s + 1) * BUF;
                cx<R>* db = buf + s * BUF;
#pragma unroll
                for (int i = 0; i < E; ++i) {
                    const int nn = FI::out_index(t, i);
                    db[padi<E>(nn)] = v[i] + cmulc(ob[padi<E>(nn)], pre[nn]);
                }
            }
            __syncthreads();
        }
        // demag field of row r, cell i: xy rows in buffer 2r, z pairs in buffer 2(T + r/2)
        auto dfield = [&](int r, int i, int c) -> R {
            if (c < 2) {
                const cx<R> z = buf[(2 * r) * BUF + padi<E>(i)];
                return c == 0 ? z.re : z.im;
            }
            const cx<R> z = buf[(2 * (T + r / 2)) * BUF + padi<E>(i)];
            return (r & 1) ? z.im : z.re;
        };
        if constexpr (LEAN) row_epilogue_lean<R>(F, spec, st, w.blk, T, do_fft, dfield);
        else row_epilogue<R>(F, spec, st, w.blk, T, do_fft, dfield, sm_red);
        __syncthreads();
    }
}

// Pass twiddle tables [r][k] for GroupFFT<R, L>.
template <typename R, int L>
__global__ void k_pass_tables(cx<R>* out) {
    using P = FPlan<R, L>;
    using TT = TwTab<R, L>;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < TT::size; e += gridDim.x * blockDim.x) {
        long long k, r, N;
        if (e < TT::size1) {
            r = e / TT::ns1;
            k = e % TT::ns1;
            N = (long long)TT::ns1 * P::RAD1;
        } else {
            const int f = e - TT::size1;
            r = f / TT::ns2;
            k = f % TT::ns2;
            N = (long long)TT::ns2 * P::RAD2;
        }
        double sn, cs;
        sincospi(2.0 * (double)((k * r) % N) / (double)N, &sn, &cs);
        out[e] = mkc((R)cs, (R)(-sn));
    }
}

}  // namespace llg
