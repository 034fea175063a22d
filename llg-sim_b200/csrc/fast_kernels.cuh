// fast_kernels.cuh — register-FFT versions of the three evaluation passes for
// power-of-two film sizes (16..2048).  Same data layout, same algorithm and
// same epilogue as field_kernels.cuh; the transforms use GroupFFT (fft_reg.cuh)
// with per-pass twiddle tables and the W_{2L}^n pre-twiddles resident in
// shared memory.
#pragma once
#include "field_kernels.cuh"
#include "fft_reg.cuh"
#include "async_copy.cuh"

namespace llg {

// Row passes: T rows per block; signals: T packed xy rows and T/2 packed z
// row pairs, each as an even-bin and an odd-bin transform (s = 2g + parity).
// Registers per thread that let `blocks` blocks of `threads` threads reside on
// one SM.  The register file is split over the SM's four sub-partitions (16384
// 32-bit registers each) and a warp takes its registers from the sub-partition it
// is scheduled on, so the sub-partition with the most warps sets the bound: 112
// registers allow two 192-thread blocks, not three (18 warps put five on one
// sub-partition; 96 registers are needed).
constexpr int regs_for_blocks(int threads, int blocks) {
    const int warps = blocks * ((threads + 31) / 32);
    const int per_partition = (warps + 3) / 4;
    const int r = (16384 / (32 * per_partition)) / 8 * 8;
    return r > 255 ? 255 : r;
}

template <typename R, int L, int V = 0>
struct RowCfg {
    using P = FPlan<R, L, V>;
    static constexpr int G = P::G, E = P::E;
    static constexpr int T = (64 / G) < 2 ? 2 : 64 / G;
    static constexpr int NGRP = T + T / 2;
    static constexpr int NSIG = 2 * NGRP;
    static constexpr int THREADS = NSIG * G;
    // register caps (regs_for_blocks): one resident block at least (REGCAP); the
    // FP32 forward and lean inverse passes of 192-thread blocks capped for three
    // resident blocks, plan 1 (half the registers per thread) for two (MAXREG);
    // the fused pass and the inverse passes with an epilogue, 192-thread FP32
    // blocks, for two (REG2: they hold a transform and a stencil at once; the
    // smaller cap only spilled without adding a block)
    static constexpr int REGCAP = regs_for_blocks(THREADS, 1);
    static constexpr int MAXREG = V == 1 ? regs_for_blocks(THREADS, 2)
                                         : (sizeof(R) == 4 && THREADS <= 192) ? regs_for_blocks(THREADS, 3) : REGCAP;
    static constexpr int REG2 = V == 1 ? regs_for_blocks(THREADS, 2)
                                       : (sizeof(R) == 4 && THREADS <= 192) ? regs_for_blocks(THREADS, 2) : REGCAP;
    static constexpr int BUF = Pad<R, L, V>::size;
    static constexpr int SMEM_CX = NSIG * BUF + TwTab<R, L, V>::size + L;
    // the staged spectrum (swizzled slots, stage_slot) lives in the signal buffers
    static constexpr int STAGE_CX = ((3 * (L + 1) * T * (int)sizeof(cx<R>) / 16 + 7) / 8 * 8) * (16 / (int)sizeof(cx<R>));
    static_assert(STAGE_CX <= NSIG * BUF, "staged spectrum does not fit the signal buffers");
    static constexpr size_t SMEM = sizeof(cx<R>) * (size_t)SMEM_CX;
};

// Column pass: NC columns per block, six signals per column (3 components x
// even / odd ky bins).  Shared memory: the signal exchange buffers, the pass
// tables and pre-twiddles, and the staging areas that the bulk copies of the
// next item's spectrum columns (Xst, [3][NC][L]) and folded kernel columns
// (Kst, [NC][L+1]) land in while the current item is transformed.  The LEAN form
// reads the tables and the kernel columns from global memory (through L1) and
// keeps only the signal buffers and Xst in shared memory, so that more blocks fit
// per SM.
template <typename R, int L, int V = 0, bool LEAN = false>
struct ColCfg {
    using P = FPlan<R, L, V>;
    static constexpr int G = P::G, E = P::E;
    static constexpr int NC = (32 / G) < 1 ? 1 : 32 / G;
    static constexpr int NSIG = 6 * NC;
    static constexpr int THREADS = NSIG * G;
    static constexpr int BUF = Pad<R, L, V>::size;
    static constexpr size_t al16(size_t b) { return (b + 15) / 16 * 16; }
    static constexpr size_t OFF_TW = al16(sizeof(cx<R>) * (size_t)NSIG * BUF);
    static constexpr size_t OFF_PRE = al16(OFF_TW + (LEAN ? 0 : sizeof(cx<R>) * (size_t)TwTab<R, L, V>::size));
    static constexpr size_t OFF_XST = al16(OFF_PRE + (LEAN ? 0 : sizeof(cx<R>) * (size_t)L));
    static constexpr size_t OFF_KST = al16(OFF_XST + sizeof(cx<R>) * 3 * (size_t)NC * L);
    static constexpr size_t SMEM = al16(OFF_KST + (LEAN ? 0 : sizeof(r4<R>) * (size_t)NC * (L + 1)));
    // register cap: plan 1 (half the registers per thread) for two resident blocks,
    // the lean FP32 form of 192-thread blocks for three (its shared memory allows
    // three), one block otherwise
    static constexpr int MAXREG = V == 1 ? regs_for_blocks(THREADS, 2)
                                         : (LEAN && sizeof(R) == 4 && THREADS <= 192) ? regs_for_blocks(THREADS, 3)
                                                                                      : regs_for_blocks(THREADS, 1);
};

// Staged spectrum of a row block, [c][k][r] in 16-byte pieces (PER complex values).
// With two rows per block a warp of the inverse transform reads every other piece,
// which put its lanes on a quarter of the shared-memory banks; the piece slot is
// XOR-swizzled within each group of eight so that the lanes spread over all of
// them.  The slots of a group stay in the group, so the staging area needs the
// piece count rounded up to a multiple of eight.
template <typename R, int T>
__host__ __device__ __forceinline__ int stage_slot(int p) {
    if constexpr (T == 2) return p ^ ((p >> 3) & (sizeof(R) == 4 ? 1 : 3));
    else return p;
}
template <typename R, int T>
__host__ __device__ __forceinline__ int stage_index(int e) {
    constexpr int PER = 16 / (int)sizeof(cx<R>);
    return stage_slot<R, T>(e / PER) * PER + e % PER;
}

template <typename R>
__device__ __forceinline__ void load_tables(cx<R>* twp, const cx<R>* __restrict__ gtwp, int ntwp, cx<R>* pre,
                                            const cx<R>* __restrict__ gpre, int L) {
    for (int i = threadIdx.x; i < ntwp; i += blockDim.x) twp[i] = gtwp[i];
    for (int i = threadIdx.x; i < L; i += blockDim.x) pre[i] = gpre[i];
}

// ---------------------------------------------------------------------------
template <typename R, int L, int V>
__global__ void __launch_bounds__(RowCfg<R, L, V>::THREADS) __maxnreg__((RowCfg<R, L, V>::MAXREG)) k_row_forward_fast(const FilmDev* __restrict__ films,
                                                                            const WorkItem* __restrict__ items,
                                                                            int nitems, EvalSpec spec) {
    using C = RowCfg<R, L, V>;
    using FFT = GroupFFT<R, L, false, V>;
    constexpr int G = C::G, E = C::E, T = C::T, BUF = C::BUF;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<R>* buf = reinterpret_cast<cx<R>*>(smem_raw);
    cx<R>* twp = buf + C::NSIG * BUF;
    cx<R>* pre = twp + TwTab<R, L, V>::size;
    const int tid = threadIdx.x, s = tid / G, t = tid % G, g = s >> 1, par = s & 1;
    bool tables = false;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const WorkItem w = items[it];
        const FilmDev& F = films[w.film];
        const StepState* st = F.st;
        if (skip_item(spec, st)) continue;
        const bool do_fft = spec.demag && F.demag_mat;
        if (do_fft && !tables) {
            load_tables<R>(twp, reinterpret_cast<const cx<R>*>(F.twp_row[V]), TwTab<R, L, V>::size, pre,
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
        // m_s = normalize(m0 + sum_q dt*a_q*k_q) in two sweeps over 16-byte vectors of
        // W cells: (1) per component, the combination (all its loads in flight
        // together) into the packed signal slots; (2) per cell, normalisation (or
        // vacuum), the m_s store and the scaling by Ms.  Signal slots: x, y of row r
        // in buffer 2r (re, im); z of rows 2p, 2p+1 in buffer 2(T+p) (re, im).
        constexpr int W = Vec16<R>::W, NV = T * L / W;
        auto slot = [&](int c, int r, int i) -> R* {
            cx<R>* z = c < 2 ? &buf[(2 * r) * BUF + padi<E>(i)] : &buf[(2 * (T + r / 2)) * BUF + padi<E>(i)];
            return (c == 0 || (c == 2 && (r & 1) == 0)) ? &z->re : &z->im;
        };
        // two vectors per thread and round: both vectors' loads are in flight before
        // either is stored (the stores go to shared memory after the loads)
        constexpr int U = 2;
        for (int e0 = tid; e0 < 3 * NV; e0 += U * C::THREADS) {
            Vec16<R> a[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int e = e0 + u * C::THREADS;
                const int c = e / NV, ev = e - c * NV;
                const int r = (ev * W) / L, j = j0 + r;
#pragma unroll
                for (int l = 0; l < W; ++l) a[u].v[l] = (R)0;
                if (e < 3 * NV && j < ny) {
                    const int idx = c * n + j * L + (ev * W - r * L);
                    if (spec.nterm > 0) {
                        a[u] = ldv(m0 + idx);
                        Vec16<R> ka[6];
#pragma unroll
                        for (int q = 0; q < 6; ++q)
                            if (q < spec.nterm) ka[q] = ldv(kp[q] + idx);
#pragma unroll
                        for (int q = 0; q < 6; ++q)
                            if (q < spec.nterm) {
#pragma unroll
                                for (int l = 0; l < W; ++l) a[u].v[l] = a[u].v[l] + cq[q] * ka[q].v[l];
                            }
                    } else {
                        a[u] = ldv(ms + idx);
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int e = e0 + u * C::THREADS;
                if (e >= 3 * NV) continue;
                const int c = e / NV, ev = e - c * NV;
                const int c0 = ev * W, r = c0 / L, i0 = c0 - r * L;
#pragma unroll
                for (int l = 0; l < W; ++l) *slot(c, r, i0 + l) = a[u].v[l];
            }
        }
        __syncthreads();
        for (int e = tid; e < NV; e += C::THREADS) {
            const int c0 = e * W, r = c0 / L, i0 = c0 - r * L, j = j0 + r;
            Vec16<R> v0, v1, v2;
#pragma unroll
            for (int l = 0; l < W; ++l) {
                R a[3] = {*slot(0, r, i0 + l), *slot(1, r, i0 + l), *slot(2, r, i0 + l)};
                if (spec.nterm > 0 && j < ny) {
                    if (cell_inside(F, j * L + i0 + l)) normalize3(a);
                    else { a[0] = (R)0; a[1] = (R)0; a[2] = (R)0; }
                }
                v0.v[l] = a[0]; v1.v[l] = a[1]; v2.v[l] = a[2];
                *slot(0, r, i0 + l) = Ms * a[0];
                *slot(1, r, i0 + l) = Ms * a[1];
                *slot(2, r, i0 + l) = Ms * a[2];
            }
            if (spec.nterm > 0 && j < ny) {
                const int idx = j * L + i0;
                stv(ms + idx, v0); stv(ms + n + idx, v1); stv(ms + 2 * n + idx, v2);
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
        // unpack the two real rows of each transform; PER consecutive rows of one
        // (component, kx) make one 16-byte store into the column-major spectrum
        constexpr int PER = 16 / (int)sizeof(cx<R>), TP = T / PER;
        for (int e = tid; e < 3 * K1 * TP; e += C::THREADS) {
            const int rp = e % TP, rest = e / TP;
            const int k = rest % K1, c = rest / K1;
            const int r0 = rp * PER;
            if (j0 + r0 >= ny) continue;
            const int km = (L2 - k) % L2;
            cx<R> out[PER];
#pragma unroll
            for (int q = 0; q < PER; ++q) {
                const int r = r0 + q;
                int gg, half;
                if (c < 2) { gg = r; half = c; }
                else { gg = T + r / 2; half = r & 1; }
                const cx<R> zk = buf[(2 * gg + (k & 1)) * BUF + padi<E>(k >> 1)];
                const cx<R> zm = buf[(2 * gg + (km & 1)) * BUF + padi<E>(km >> 1)];
                if (half == 0) out[q] = mkc((R)0.5 * (zk.re + zm.re), (R)0.5 * (zk.im - zm.im));
                else out[q] = mkc((R)0.5 * (zk.im + zm.im), (R)0.5 * (zm.re - zk.re));
            }
            Vec16<R> pk;
#pragma unroll
            for (int q = 0; q < PER; ++q) { pk.v[2 * q] = out[q].re; pk.v[2 * q + 1] = out[q].im; }
            stv(reinterpret_cast<R*>(X + ((size_t)c * K1 + k) * ny + j0 + r0), pk);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Column pass.  Item = NC consecutive kx columns of one film.  Per column: the
// pruned forward y-transforms of the three components (even and odd ky bins as
// two length-L transforms, odd ones pre-twiddled by W_{2L}^n), the product with
// the real kernel planes (Bx = Kxx Mx + Kxy My, By = Kxy Mx + Kyy My,
// Bz = Kzz Mz; demag_fft_uniform.rs:700-742), and the pruned inverse keeping
// the L physical rows.  The spectrum and kernel columns of the block's next item
// are fetched by bulk copies while this item is transformed.
template <typename R, int L>
__device__ __forceinline__ bool col_item_has(const FilmDev* __restrict__ films, const WorkItem* __restrict__ items,
                                             int nitems, const EvalSpec& spec, int it) {
    return it < nitems && spec.demag && films[items[it].film].demag_mat;
}

template <typename R, int L, int V>
__device__ __forceinline__ void col_issue_x(const FilmDev* __restrict__ films, const WorkItem* __restrict__ items,
                                            int it, cx<R>* xst, uint64_t* bar) {
    using C = ColCfg<R, L, V>;
    const WorkItem w = items[it];
    const FilmDev& F = films[w.film];
    const int K1 = F.nx + 1, kx0 = w.blk * C::NC;
    const int nv = min(C::NC, K1 - kx0);
    const uint32_t bytes = (uint32_t)(sizeof(cx<R>) * (size_t)nv * L);
    const cx<R>* X = reinterpret_cast<const cx<R>*>(F.X);
    mbar_arrive_expect_tx(bar, 3 * bytes);
#pragma unroll
    for (int c = 0; c < 3; ++c) bulk_copy_g2s(xst + (size_t)c * C::NC * L, X + ((size_t)c * K1 + kx0) * L, bytes, bar);
}

template <typename R, int L, int V>
__device__ __forceinline__ void col_issue_k(const FilmDev* __restrict__ films, const WorkItem* __restrict__ items,
                                            int it, r4<R>* kst, uint64_t* bar) {
    using C = ColCfg<R, L, V>;
    const WorkItem w = items[it];
    const FilmDev& F = films[w.film];
    const int K1 = F.nx + 1, kx0 = w.blk * C::NC;
    const int nv = min(C::NC, K1 - kx0);
    const uint32_t bytes = (uint32_t)(sizeof(r4<R>) * (size_t)nv * (L + 1));
    mbar_arrive_expect_tx(bar, bytes);
    bulk_copy_g2s(kst, reinterpret_cast<const r4<R>*>(F.Khat) + (size_t)kx0 * (L + 1), bytes, bar);
}

template <typename R, int L, int V, bool LEAN>
__global__ void __launch_bounds__(ColCfg<R, L, V, LEAN>::THREADS) __maxnreg__((ColCfg<R, L, V, LEAN>::MAXREG)) k_column_fast(
    const FilmDev* __restrict__ films, const WorkItem* __restrict__ items, int nitems, EvalSpec spec) {
    using C = ColCfg<R, L, V, LEAN>;
    using FF = GroupFFT<R, L, false, V>;
    using FI = GroupFFT<R, L, true, V>;
    constexpr int G = C::G, E = C::E, BUF = C::BUF, NC = C::NC;
    constexpr int ny = L;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint64_t bars[2];   // 0: spectrum columns, 1: kernel columns
    __shared__ int s_timeout;
    cx<R>* buf = reinterpret_cast<cx<R>*>(smem_raw);
    const cx<R>* twp = reinterpret_cast<const cx<R>*>(smem_raw + C::OFF_TW);
    const cx<R>* pre = reinterpret_cast<const cx<R>*>(smem_raw + C::OFF_PRE);
    cx<R>* xst = reinterpret_cast<cx<R>*>(smem_raw + C::OFF_XST);
    r4<R>* kst = reinterpret_cast<r4<R>*>(smem_raw + C::OFF_KST);
    const int tid = threadIdx.x, s = tid / G, t = tid % G;
    const int cl = s / 6, comp = (s % 6) >> 1, par = s & 1;
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        s_timeout = 0;
        mbar_init_fence();
    }
    __syncthreads();
    const int it0 = blockIdx.x;
    if (tid == 0 && col_item_has<R, L>(films, items, nitems, spec, it0)) {
        col_issue_x<R, L, V>(films, items, it0, xst, &bars[0]);
        if (!LEAN) col_issue_k<R, L, V>(films, items, it0, kst, &bars[1]);
    }
    uint32_t phase = 0;
    bool tables = false;
    for (int it = it0; it < nitems; it += gridDim.x) {
        const int nxt = it + gridDim.x;
        const bool has = col_item_has<R, L>(films, items, nitems, spec, it);
        const bool has_next = col_item_has<R, L>(films, items, nitems, spec, nxt);
        if (!has) {   // nothing was fetched for this item (uniform over the block)
            if (tid == 0 && has_next) {
                fence_async_smem();
                col_issue_x<R, L, V>(films, items, nxt, xst, &bars[0]);
                if (!LEAN) col_issue_k<R, L, V>(films, items, nxt, kst, &bars[1]);
            }
            continue;
        }
        const WorkItem w = items[it];
        const FilmDev& F = films[w.film];
        if constexpr (LEAN) {
            twp = reinterpret_cast<const cx<R>*>(F.twp_col[V]);
            pre = reinterpret_cast<const cx<R>*>(F.tw_col);
        } else if (!tables) {
            load_tables<R>(const_cast<cx<R>*>(twp), reinterpret_cast<const cx<R>*>(F.twp_col[V]), TwTab<R, L, V>::size,
                           const_cast<cx<R>*>(pre), reinterpret_cast<const cx<R>*>(F.tw_col), L);
            tables = true;
        }
        const bool okx = mbar_wait(&bars[0], phase);
        const bool okk = LEAN ? true : mbar_wait(&bars[1], phase);
        if (!(okx && okk)) s_timeout = 1;
        phase ^= 1u;
        __syncthreads();   // tables, staged columns, timeout flag
        if (s_timeout) {
            // a copy that never completed: report and leave without touching its buffers again
            if (tid == 0) atomicExch(const_cast<int*>(&F.st->err_code), kErrAsyncTimeout);
            return;
        }
        const bool run = !skip_item(spec, F.st);
        const int K1 = F.nx + 1;
        const int kx = w.blk * NC + cl;
        const bool valid = kx < K1;
        cx<R> v[E];
        if (run) {
#pragma unroll
            for (int r = 0; r < E; ++r) {
                const int nn = t + G * r;
                const cx<R> x = valid ? xst[((size_t)comp * NC + cl) * L + nn] : mkc((R)0, (R)0);
                v[r] = par ? cmul(x, pre[nn]) : x;
            }
        }
        __syncthreads();   // staged spectrum consumed
        if (tid == 0 && has_next) {
            fence_async_smem();
            col_issue_x<R, L, V>(films, items, nxt, xst, &bars[0]);
        }
        if (run) {
            FF::run(v, t, buf + s * BUF, twp);
            group_sync<G>();
#pragma unroll
            for (int i = 0; i < E; ++i) buf[s * BUF + padi<E>(FF::out_index(t, i))] = v[i];
            __syncthreads();   // all components of the column transformed
            const r4<R>* kc = LEAN ? reinterpret_cast<const r4<R>*>(F.Khat) + (size_t)(valid ? kx : 0) * (L + 1)
                                   : kst + (size_t)cl * (L + 1);
            const cx<R>* sx = buf + (6 * cl + 0 + par) * BUF;
            const cx<R>* sy = buf + (6 * cl + 2 + par) * BUF;
            const cx<R>* sz = buf + (6 * cl + 4 + par) * BUF;
#pragma unroll
            for (int r = 0; r < E; ++r) {
                const int kk = t + G * r;
                const int ky = 2 * kk + par;
                // the kernel spectrum is even in ky except Kxy, which is odd; the
                // column is parity-split (khat_index): ky and L2 - ky have the parity
                // of this signal, so a warp reads consecutive entries
                const bool up = ky > ny;
                const r4<R> K = kc[par ? (up ? ny / 2 + L - kk : ny / 2 + 1 + kk) : (up ? L - kk : kk)];
                const R kxy = up ? -K.y : K.y;
                const int pi = padi<E>(kk);
                cx<R> out;
                if (comp == 0) {
                    const cx<R> Mx = sx[pi], My = sy[pi];
                    out = mkc(K.x * Mx.re + kxy * My.re, K.x * Mx.im + kxy * My.im);
                } else if (comp == 1) {
                    const cx<R> Mx = sx[pi], My = sy[pi];
                    out = mkc(kxy * Mx.re + K.z * My.re, kxy * Mx.im + K.z * My.im);
                } else {
                    const cx<R> Mz = sz[pi];
                    out = mkc(K.w * Mz.re, K.w * Mz.im);
                }
                v[r] = out;
            }
        }
        __syncthreads();   // products formed: the signal buffers and staged kernel are free
        if (!LEAN && tid == 0 && has_next) {
            fence_async_smem();
            col_issue_k<R, L, V>(films, items, nxt, kst, &bars[1]);
        }
        if (run) {
            FI::run(v, t, buf + s * BUF, twp);
            group_sync<G>();
            if (par) {
#pragma unroll
                for (int i = 0; i < E; ++i) buf[s * BUF + padi<E>(FI::out_index(t, i))] = v[i];
            }
            __syncthreads();   // odd-bin results visible to the even-bin groups
            if (!par && valid) {
                cx<R>* __restrict__ X = reinterpret_cast<cx<R>*>(F.X);
                const cx<R>* ob = buf + (s + 1) * BUF;
#pragma unroll
                for (int i = 0; i < E; ++i) {
                    const int nn = FI::out_index(t, i);
                    X[((size_t)comp * K1 + kx) * ny + nn] = v[i] + cmulc(ob[padi<E>(nn)], pre[nn]);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// MODE 0: full epilogue; 1: no epilogue, the demag field is written to the film's
// bdem planes for k_stage_torque; 2: the minimiser epilogue (RHS_MINIMIZE).
template <typename R, int L, int MODE, int V>
__global__ void __launch_bounds__(RowCfg<R, L, V>::THREADS) __maxnreg__((MODE == 1 ? RowCfg<R, L, V>::MAXREG : RowCfg<R, L, V>::REG2)) k_row_inverse_fast(const FilmDev* __restrict__ films,
                                                                            const WorkItem* __restrict__ items,
                                                                            int nitems, EvalSpec spec) {
    using C = RowCfg<R, L, V>;
    using FI = GroupFFT<R, L, true, V>;
    constexpr int G = C::G, E = C::E, T = C::T, BUF = C::BUF;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double sm_red[32 * RED_NSLOT];
    cx<R>* buf = reinterpret_cast<cx<R>*>(smem_raw);
    cx<R>* twp = buf + C::NSIG * BUF;
    cx<R>* pre = twp + TwTab<R, L, V>::size;
    const int tid = threadIdx.x, s = tid / G, t = tid % G, g = s >> 1, par = s & 1;
    bool tables = false;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const WorkItem w = items[it];
        const FilmDev& F = films[w.film];
        StepState* st = F.st;
        if (skip_item(spec, st)) continue;
        const bool do_fft = spec.demag && F.demag_mat;
        if (do_fft && !tables) {
            load_tables<R>(twp, reinterpret_cast<const cx<R>*>(F.twp_row[V]), TwTab<R, L, V>::size, pre,
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
            constexpr int PER = 16 / (int)sizeof(cx<R>);
            for (int p = tid; p < 3 * K1 * T / PER; p += C::THREADS) {
                const int e = p * PER, r = e % T, ck = e / T;
                cx<R>* dst = stg + stage_slot<R, T>(p) * PER;
                if (j0 + r < ny) {
                    cp_async16(dst, X + (size_t)ck * ny + j0 + r);
                } else {
#pragma unroll
                    for (int q = 0; q < PER; ++q) dst[q] = mkc((R)0, (R)0);
                }
            }
            cp_async_wait_all();
            __syncthreads();
            static_assert(T != 2 || (2 * G * T / PER) % 32 == 0, "swizzle needs 32-piece strides");
            const int kb = 2 * t + par;
            auto xval = [&](int c, int rr, int k, int r) -> cx<R> {
                // k = kb + 2*G*rr: the swizzle of a slot depends only on the bits below
                // 2*G*T/PER pieces, so the slots of a thread are its slot at rr = 0 plus
                // a constant per rr (immediate offsets, no per-value swizzle)
                const int off = 2 * G * rr * T;
                if constexpr (T != 2) {   // identity slots
                    if (k <= L) return stg[(c * K1 + k) * T + r];
                    return conjc(stg[(c * K1 + (L2 - k)) * T + r]);
                }
                if (k <= L) return stg[stage_index<R, T>((c * K1 + kb) * T + r) + off];
                return conjc(stg[stage_index<R, T>((c * K1 + (L2 - kb)) * T + r) - off]);
            };
            cx<R> v[E];
#pragma unroll
            for (int r = 0; r < E; ++r) {
                const int k = 2 * (t + G * r) + par;
                cx<R> z;
                if (g < T) {
                    const cx<R> bx = xval(0, r, k, g), by = xval(1, r, k, g);
                    z = mkc(bx.re - by.im, bx.im + by.re);
                } else {
                    const int ra = 2 * (g - T);
                    const cx<R> za = xval(2, r, k, ra), zb = xval(2, r, k, ra + 1);
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
        if constexpr (MODE == 1) {
            // demag field only, for the streaming torque kernel
            if (do_fft) {
                constexpr int W = Vec16<R>::W;
                const int n = F.nx * ny;
                R* __restrict__ bd = reinterpret_cast<R*>(F.bdem);
                for (int e = tid; e < T * L / W; e += C::THREADS) {
                    const int c0 = e * W, r = c0 / L, i0 = c0 - r * L, j = j0 + r;
                    if (j >= ny) continue;
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        Vec16<R> o;
#pragma unroll
                        for (int l = 0; l < W; ++l) o.v[l] = dfield(r, i0 + l, c);
                        stv(bd + c * n + j * L + i0, o);
                    }
                }
            }
        } else {
            row_epilogue<R, MODE == 2>(F, spec, st, w.blk, T, do_fft, dfield, sm_red);
        }
        __syncthreads();
    }
}

// Pass twiddle tables [r][k] for GroupFFT<R, L>.
template <typename R, int L, int V>
__global__ void k_pass_tables(cx<R>* out) {
    using P = FPlan<R, L, V>;
    using TT = TwTab<R, L, V>;
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
