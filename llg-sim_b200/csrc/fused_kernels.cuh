// fused_kernels.cuh — one row pass that ends RK stage s and starts stage s+1
// (register-FFT path, power-of-two nx).
//
// Per block of T rows it does, in shared memory and registers:
//   1. the inverse x transform of the block's spectrum rows (the last third of
//      stage s's field evaluation, as k_row_inverse_fast),
//   2. per cell: the local terms (Zeeman, exchange, anisotropy, DMI in the
//      reference's order; cells away from edges and vacuum by the ghost-free
//      path with the same arithmetic) plus the demag field, the torque k_s (llg_rhs /
//      llg_rhs_relax, llg.rs:20-50), stored for the later combinations and the
//      error norm, and at once the stage s+1 state
//        m_{s+1} = normalize(m0 + sum_q dt*a_q k_q)   (llg.rs:869-942 / 296-309)
//      with k_s taken from registers (it is always the last term of the next
//      combination in both tableaux),
//   3. the zero-padded forward x transform of Ms*m_{s+1} and the store of its
//      Hermitian bins (the first third of stage s+1, as k_row_forward_fast).
// An RK45 attempt is then one row-forward pass, six column passes, five fused
// row passes and the last stage's row inverse, instead of three passes per
// evaluation.  The arithmetic of every value is the one of the unfused passes
// (same operations in the same order), so both paths give the same bits.
#pragma once
#include "fast_kernels.cuh"

namespace llg {

// si: stage s (inverse half: m_in, k_out, rhs, field terms); sf: stage s+1
// (forward half: m_in receives m_{s+1}, the combination kidx / a with
// sf.kidx[sf.nterm - 1] == si.k_out).  Both carry the same request gate.
template <typename R, int L, int V>
__global__ void __launch_bounds__(RowCfg<R, L, V>::THREADS) __maxnreg__((RowCfg<R, L, V>::REG2)) k_row_fused(
    const FilmDev* __restrict__ films, const WorkItem* __restrict__ items, int nitems, EvalSpec si, EvalSpec sf) {
    using C = RowCfg<R, L, V>;
    using FF = GroupFFT<R, L, false, V>;
    using FI = GroupFFT<R, L, true, V>;
    constexpr int G = C::G, E = C::E, T = C::T, BUF = C::BUF;
    // phase 2 takes W = 2 cells per step of its loop: the stencil (and, with EARLY,
    // m0 and the previous torques) of both cells are loaded before any arithmetic
    constexpr int W = 2, NV = T * L / W;
    using VW = VecW<R, W>;
    // the early loads of the combination's torques and the ghost-free path of
    // interior cells need the registers of the FP32 plan-0 budget; the other
    // instantiations load the torques where they are used and take the general path
    constexpr bool EARLY = sizeof(R) == 4 && V == 0;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<R>* buf = reinterpret_cast<cx<R>*>(smem_raw);
    cx<R>* twp = buf + C::NSIG * BUF;
    cx<R>* pre = twp + TwTab<R, L, V>::size;
    const int tid = threadIdx.x, s = tid / G, t = tid % G, g = s >> 1, par = s & 1;
    // signal slot of component c of row r, cell i: x, y of row r in buffer 2r
    // (re, im); z of rows 2p, 2p+1 in buffer 2(T+p) (re, im).  The inverse
    // transform leaves the demag field there and the forward one takes M there.
    auto slot = [&](int c, int r, int i) -> R* {
        cx<R>* z = c < 2 ? &buf[(2 * r) * BUF + padi<E>(i)] : &buf[(2 * (T + r / 2)) * BUF + padi<E>(i)];
        return (c == 0 || (c == 2 && (r & 1) == 0)) ? &z->re : &z->im;
    };
    bool tables = false;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const WorkItem w = items[it];
        const FilmDev& F = films[w.film];
        StepState* st = F.st;
        if (skip_item(si, st)) continue;   // uniform over the block
        const bool do_fft = si.demag && F.demag_mat;
        if (do_fft && !tables) {
            load_tables<R>(twp, reinterpret_cast<const cx<R>*>(F.twp_row[V]), TwTab<R, L, V>::size, pre,
                           reinterpret_cast<const cx<R>*>(F.tw_row), L);
            tables = true;
            __syncthreads();
        }
        const int ny = F.ny, n = L * ny;
        const int j0 = w.blk * T;
        const int cur = st->cur;
        cx<R>* __restrict__ X = reinterpret_cast<cx<R>*>(F.X);
        constexpr int K1 = L + 1, L2 = 2 * L;
        if (do_fft) {
            // ---- 1. inverse transform of stage s (k_row_inverse_fast) ----
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
        // ---- 2. torque of stage s and state of stage s+1, W cells per step ----
        {
            const R* __restrict__ msb = mbuf<R>(F, si.m_in, cur);
            const R* __restrict__ m0 = mbuf<R>(F, MB_M0, cur);
            R* __restrict__ kout = kbuf<R>(F, si.k_out, cur);
            R* __restrict__ mnext = mbuf<R>(F, sf.m_in, cur);
            const double dt = st->dt;
            const R gam = (R)F.gamma, alp = (R)F.alpha;
            const R denom = (R)1 + alp * alp;
            const R pref = si.rhs == RHS_LLG ? -gam / denom : -gam * alp / denom;
            const R c1 = si.rhs == RHS_LLG ? (R)1 : (R)0;
            const R c2 = si.rhs == RHS_LLG ? alp : (R)1;
            const int nq = sf.nterm - 1;   // terms read from HBM; the last one is k_s
            const R* kp[5];
            R cq[6];
#pragma unroll
            for (int q = 0; q < 5; ++q) kp[q] = q < nq ? kbuf<R>(F, sf.kidx[q], cur) : nullptr;
#pragma unroll
            for (int q = 0; q < 6; ++q) cq[q] = q < sf.nterm ? (R)(dt * sf.a[q]) : (R)0;
            const R cs = (R)(dt * sf.a[nq]);   // k_s coefficient
            const R Ms = (R)F.ms;
            const LocalCoef<R> cf = local_coef<R>(F, si.dmi != 0);
            for (int e = tid; e < NV; e += C::THREADS) {
                const int c0 = e * W, r = c0 / L, i0 = c0 - r * L, j = j0 + r;
                if (j >= ny) {   // rows past the film are zero in the forward transform
                    if (do_fft)
#pragma unroll
                        for (int l = 0; l < W; ++l)
#pragma unroll
                            for (int c = 0; c < 3; ++c) *slot(c, r, i0 + l) = (R)0;
                    continue;
                }
                const int base = j * L + i0;
                // stencil of m_s: centre, the rows below / above, one x halo on each side;
                // m0 and the torques of the combination
                VW cen[3], dn[3], upv[3], a[3], kq[EARLY ? 5 : 1][3];
                R hl[3], hr[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    cen[c] = ldw<R, W>(msb + c * n + base);
                    if (j > 0) dn[c] = ldw<R, W>(msb + c * n + base - L);
                    if (j + 1 < ny) upv[c] = ldw<R, W>(msb + c * n + base + L);
                    hl[c] = i0 > 0 ? msb[c * n + base - 1] : (R)0;
                    hr[c] = i0 + W < L ? msb[c * n + base + W] : (R)0;
                }
                if constexpr (EARLY) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) a[c] = ldw<R, W>(m0 + c * n + base);
#pragma unroll
                    for (int q = 0; q < 5; ++q)
                        if (q < nq)
#pragma unroll
                            for (int c = 0; c < 3; ++c) kq[q][c] = ldw<R, W>(kp[q] + c * n + base);
                }
                const bool inner = EARLY && cf.mask == nullptr && j > 0 && j + 1 < ny && i0 > 0 && i0 + W < L;
                VW ko[3];
#pragma unroll
                for (int l = 0; l < W; ++l) {
                    const int i = i0 + l;
                    const R mc[3] = {cen[0].v[l], cen[1].v[l], cen[2].v[l]};
                    auto nb = [&](int d, R* o) {
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            if (d == 0) o[c] = l > 0 ? cen[c].v[l > 0 ? l - 1 : 0] : hl[c];
                            else if (d == 1) o[c] = l < W - 1 ? cen[c].v[l < W - 1 ? l + 1 : 0] : hr[c];
                            else if (d == 2) o[c] = dn[c].v[l];
                            else o[c] = upv[c].v[l];
                        }
                    };
                    R b[3];
                    if (inner) local_field_interior<R>(cf, nb, mc, b);
                    else local_field_c<R>(cf, nb, i, j, mc, b);
                    if (do_fft) {
#pragma unroll
                        for (int c = 0; c < 3; ++c) b[c] += *slot(c, r, i);
                    }
                    R k[3];
                    torque_cell<R>(mc, b, pref, c1, c2, k);
#pragma unroll
                    for (int c = 0; c < 3; ++c) ko[c].v[l] = k[c];
                }
#pragma unroll
                for (int c = 0; c < 3; ++c) stw<R, W>(kout + c * n + base, ko[c]);
                // m_{s+1} = normalize(m0 + sum_q dt*a_q k_q), terms in the tableau's order
                if constexpr (!EARLY) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) a[c] = ldw<R, W>(m0 + c * n + base);
                }
#pragma unroll
                for (int q = 0; q < 5; ++q) {
                    if (q < nq) {
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            const VW kv = EARLY ? kq[EARLY ? q : 0][c] : ldw<R, W>(kp[q] + c * n + base);
#pragma unroll
                            for (int l = 0; l < W; ++l) a[c].v[l] = a[c].v[l] + cq[q] * kv.v[l];
                        }
                    }
                }
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int l = 0; l < W; ++l) a[c].v[l] = a[c].v[l] + cs * ko[c].v[l];
#pragma unroll
                for (int l = 0; l < W; ++l) {
                    R v3[3] = {a[0].v[l], a[1].v[l], a[2].v[l]};
                    if (coef_inside(cf, base + l)) normalize3(v3);
                    else { v3[0] = (R)0; v3[1] = (R)0; v3[2] = (R)0; }   // vacuum pinned at m = 0
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        a[c].v[l] = v3[c];
                        if (do_fft) *slot(c, r, i0 + l) = Ms * v3[c];
                    }
                }
#pragma unroll
                for (int c = 0; c < 3; ++c) stw<R, W>(mnext + c * n + base, a[c]);
            }
        }
        if (!do_fft) continue;
        __syncthreads();
        // ---- 3. forward transform of stage s+1 (k_row_forward_fast) ----
        cx<R> v[E];
        {
            const cx<R>* zb = buf + (2 * g) * BUF;
#pragma unroll
            for (int r = 0; r < E; ++r) {
                const int nn = t + G * r;
                const cx<R> x = zb[padi<E>(nn)];
                v[r] = par ? cmul(x, pre[nn]) : x;
            }
        }
        __syncthreads();
        FF::run(v, t, buf + s * BUF, twp);
        __syncthreads();
#pragma unroll
        for (int i = 0; i < E; ++i) buf[s * BUF + padi<E>(FF::out_index(t, i))] = v[i];
        __syncthreads();
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

}  // namespace llg
