// field_kernels.cuh — the per-evaluation kernels of the uniform-grid LLG path.
//
// One effective-field evaluation (build_h_eff_masked, effective_field/mod.rs:48-75,
// with the demag of Demag2D::add_field, demag_fft_uniform.rs:636-769) plus the
// torque (llg_rhs / llg_rhs_relax, llg.rs:20-50) runs as three passes:
//
//   k_row_forward  rows j of the film: RK stage combination
//                  m_s = normalize(m0 + sum dt*a_q k_q) (llg.rs:869-942), write m_s,
//                  M = Ms*m_s, zero-padded real-to-complex transform along x
//                  (length 2nx, only nx inputs nonzero -> two length-nx FFTs of the
//                  even / odd output bins; two real rows packed per complex FFT),
//                  write the nx+1 Hermitian bins of Mx, My, Mz to X[c][kx][j].
//   k_column       one kx column: zero-padded 2ny-point FFT along y (two ny-point
//                  FFTs), multiply by the real kernel planes (Bx = Kxx Mx + Kxy My,
//                  By = Kxy Mx + Kyy My, Bz = Kzz Mz, demag_fft_uniform.rs:700-723),
//                  inverse 2ny-point FFT keeping the ny physical rows.
//   k_row_inverse  rows j: complex-to-real inverse along x keeping nx cells, add the
//                  local terms (Zeeman, exchange, anisotropy, DMI in the reference's
//                  order), torque, RK error norm and FP64 block reductions.
//
// The kernel spectrum is real (the real-space kernel is even/even for xx, yy, zz
// and odd/odd for xy with zeros on the axes and Nyquist planes,
// demag_fft_uniform.rs:1007-1071), so only its real part is stored, folded in ky.
#pragma once
#include "async_copy.cuh"
#include "fft_smem.cuh"
#include "types.cuh"

namespace llg {

template <typename R>
struct __align__(4 * sizeof(R)) r4 {
    R x, y, z, w;
};

// Entry of ky (0..ny, ny even) in a parity-split kernel column: the even ky
// first (ky / 2), then the odd ones (ny / 2 + 1 + (ky - 1) / 2).  A warp of the
// register-FFT column pass reads bins of one parity at consecutive kk, which are
// then consecutive entries.
__host__ __device__ __forceinline__ int khat_index(int ky, int ny) {
    return (ky & 1) ? ny / 2 + 1 + (ky >> 1) : (ky >> 1);
}

template <typename R>
__device__ __forceinline__ R* mbuf(const FilmDev& F, int id, int cur) {
    switch (id) {
        case MB_M0: return reinterpret_cast<R*>(F.m[cur]);
        case MB_M7: return reinterpret_cast<R*>(F.m[cur ^ 1]);
        case MB_S0: return reinterpret_cast<R*>(F.ms_buf[0]);
        default: return reinterpret_cast<R*>(F.ms_buf[1]);
    }
}
template <typename R>
__device__ __forceinline__ R* kbuf(const FilmDev& F, int id, int cur) {
    if (id == KB_K1) return reinterpret_cast<R*>(F.k[cur ? 7 : 1]);
    if (id == KB_K7) return reinterpret_cast<R*>(F.k[cur ? 1 : 7]);
    return reinterpret_cast<R*>(F.k[id]);
}

template <typename R>
__device__ __forceinline__ void normalize3(R* v) {
    // vec3::normalize (vec3.rs:21-28): zero maps to +z
    R n2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    if (n2 == (R)0) {
        v[0] = (R)0; v[1] = (R)0; v[2] = (R)1;
        return;
    }
    R inv = (R)1 / sqrt(n2);
    v[0] *= inv; v[1] *= inv; v[2] *= inv;
}

// Whether this evaluation skips a film: inactive, FSAL torque still valid, or
// (request-gated evaluations) the film did not request it.
__device__ __forceinline__ bool skip_item(const EvalSpec& spec, const StepState* st) {
    if (!st->active) return true;
    if (spec.skip_if_fsal && st->fsal_valid) return true;
    if (spec.req && st->req != spec.req) return true;
    return false;
}

__device__ __forceinline__ bool cell_inside(const FilmDev& F, int idx) { return !F.has_mask || F.mask[idx] != 0; }

// Ghost neighbours (exchange.rs:8-35, dmi.rs:19-52, energy.rs:37-64).
template <typename R>
__device__ __forceinline__ void ghost_x(const R* m, R nxs, R eta, R dx, R* o) {
    o[0] = m[0] + nxs * dx * (-eta * m[2]);
    o[1] = m[1];
    o[2] = m[2] + nxs * dx * (eta * m[0]);
}
template <typename R>
__device__ __forceinline__ void ghost_y(const R* m, R nys, R eta, R dy, R* o) {
    o[0] = m[0];
    o[1] = m[1] + nys * dy * (-eta * m[2]);
    o[2] = m[2] + nys * dy * (eta * m[1]);
}
template <typename R>
__device__ __forceinline__ void ld3(const R* __restrict__ m, int n, int idx, R* o) {
    o[0] = m[idx];
    o[1] = m[n + idx];
    o[2] = m[2 * n + idx];
}
template <typename R>
__device__ __forceinline__ void cp3(const R* a, R* o) {
    o[0] = a[0]; o[1] = a[1]; o[2] = a[2];
}

// Coefficients of the local terms of one film in the solver precision, formed once
// per work item (the kernels would otherwise reload and convert the FP64 film
// descriptor for every cell).  The values are the ones the per-cell conversions
// gave, so results do not change.
template <typename R>
struct LocalCoef {
    R bx, by, bz;                  // Zeeman
    R exch, ix2, iy2;              // 2A/Ms, 1/dx^2, 1/dy^2
    R dx, dy, eta;                 // ghost rules
    R dmi_pref, hx, hy;            // 2D/Ms, 1/(2dx), 1/(2dy)
    R anis, u0, u1, u2;            // 2Ku/Ms, easy axis
    bool has_eta, ex_on, dmi_on, anis_on;
    int nx, ny;
    const uint8_t* mask;           // null without a geometry mask
};

template <typename R>
__device__ __forceinline__ LocalCoef<R> local_coef(const FilmDev& F, bool dmi_on) {
    LocalCoef<R> c;
    c.bx = (R)F.bext[0];
    c.by = (R)F.bext[1];
    c.bz = (R)F.bext[2];
    c.exch = (R)F.exch;
    c.ix2 = (R)F.inv_dx2;
    c.iy2 = (R)F.inv_dy2;
    c.dx = (R)F.dx;
    c.dy = (R)F.dy;
    c.eta = (R)F.eta;
    c.dmi_pref = (R)F.dmi_pref;
    c.hx = (R)F.half_inv_dx;
    c.hy = (R)F.half_inv_dy;
    c.anis = (R)F.anis;
    c.u0 = (R)F.u[0];
    c.u1 = (R)F.u[1];
    c.u2 = (R)F.u[2];
    c.has_eta = F.has_eta != 0;
    c.ex_on = F.exch != 0.0;
    c.dmi_on = dmi_on && F.dmi_avail;
    c.anis_on = F.anis != 0.0;
    c.nx = F.nx;
    c.ny = F.ny;
    c.mask = F.has_mask ? F.mask : nullptr;
    return c;
}

template <typename R>
__device__ __forceinline__ bool coef_inside(const LocalCoef<R>& c, int idx) {
    return c.mask == nullptr || c.mask[idx] != 0;
}

// Rounded operations that the compiler may not fuse or reorder: the cores below
// spell out every product, sum and fused multiply-add, so a cell's field has the
// same bits whichever kernel (and whichever surrounding code) evaluates it.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }

// Arithmetic of the exchange (exchange.rs:45-222), anisotropy (anisotropy.rs:10-26)
// and DMI (dmi.rs:67-209) terms of one cell from its four neighbour values (real
// neighbours or ghosts, chosen by the caller); xs / ys: the film has more than one
// cell along x / y.  Both local-field paths below call these, so a cell gets the
// same bits from either.
template <typename R>
__device__ __forceinline__ void exch_core(const LocalCoef<R>& k, bool xs, bool ys, const R* mc, const R* mim,
                                          const R* mip, const R* mjm, const R* mjp, R* b) {
    const R coeff = k.exch, ix2 = k.ix2, iy2 = k.iy2;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        // (m(i+1) - 2 m(i) + m(i-1)) / dx^2 + (...) / dy^2
        const R d2x = xs ? mul_rn(add_rn(fma_rn((R)-2, mc[c], mip[c]), mim[c]), ix2) : (R)0;
        const R d2y = ys ? mul_rn(add_rn(fma_rn((R)-2, mc[c], mjp[c]), mjm[c]), iy2) : (R)0;
        b[c] = fma_rn(coeff, add_rn(d2x, d2y), b[c]);
    }
}
template <typename R>
__device__ __forceinline__ void anis_core(const LocalCoef<R>& k, const R* mc, R* b) {
    const R mdotu = fma_rn(mc[2], k.u2, fma_rn(mc[1], k.u1, mul_rn(mc[0], k.u0)));
    const R f = mul_rn(k.anis, mdotu);
    b[0] = fma_rn(f, k.u0, b[0]);
    b[1] = fma_rn(f, k.u1, b[1]);
    b[2] = fma_rn(f, k.u2, b[2]);
}
template <typename R>
__device__ __forceinline__ void dmi_core(const LocalCoef<R>& k, bool xs, bool ys, const R* mim, const R* mip,
                                         const R* mjm, const R* mjp, R* b) {
    const R pref = k.dmi_pref, hx = k.hx, hy = k.hy;
    const R dmz_dx = xs ? mul_rn(sub_rn(mip[2], mim[2]), hx) : (R)0;
    const R dmz_dy = ys ? mul_rn(sub_rn(mjp[2], mjm[2]), hy) : (R)0;
    const R dmx_dx = xs ? mul_rn(sub_rn(mip[0], mim[0]), hx) : (R)0;
    const R dmy_dy = ys ? mul_rn(sub_rn(mjp[1], mjm[1]), hy) : (R)0;
    b[0] = fma_rn(pref, dmz_dx, b[0]);
    b[1] = fma_rn(pref, dmz_dy, b[1]);
    b[2] = fma_rn(-pref, add_rn(dmx_dx, dmy_dy), b[2]);
}

// Torque of one cell from m and B (llg.rs:20-32 with c1 = 1, c2 = alpha; the
// damping-only relax torque llg.rs:38-50 with c1 = 0, c2 = 1), with the same
// explicit rounding in every kernel that forms it.
template <typename R>
__device__ __forceinline__ void torque_cell(const R* mc, const R* b, R pref, R c1, R c2, R* k) {
    const R t0 = fma_rn(mc[1], b[2], -mul_rn(mc[2], b[1]));
    const R t1 = fma_rn(mc[2], b[0], -mul_rn(mc[0], b[2]));
    const R t2 = fma_rn(mc[0], b[1], -mul_rn(mc[1], b[0]));
    const R u0 = fma_rn(mc[1], t2, -mul_rn(mc[2], t1));
    const R u1 = fma_rn(mc[2], t0, -mul_rn(mc[0], t2));
    const R u2 = fma_rn(mc[0], t1, -mul_rn(mc[1], t0));
    k[0] = mul_rn(pref, fma_rn(c2, u0, mul_rn(c1, t0)));
    k[1] = mul_rn(pref, fma_rn(c2, u1, mul_rn(c1, t1)));
    k[2] = mul_rn(pref, fma_rn(c2, u2, mul_rn(c1, t2)));
}

// Local effective-field terms at cell (i, j): Zeeman (zeeman.rs:6-12), exchange
// (exchange.rs:45-222), anisotropy (anisotropy.rs:10-26), DMI (dmi.rs:67-209),
// accumulated in that order.  With a geometry mask this is the _geom variant
// (mod.rs:78-101).
// Neighbour values come from `nb(dir, out)`, dir 0..3 = (i-1, i+1, j-1, j+1); it
// is called only for neighbours inside the film, once each: exchange and DMI share
// the loaded values and differ only in their boundary rules (an edge or vacuum
// neighbour is a chiral ghost for exchange when D != 0, else a copy of the centre;
// for DMI an edge neighbour is a ghost and a vacuum neighbour a copy).  Divisions
// by dx^2 and 2 dx are products with reciprocals formed in FP64 on the host.
template <typename R, typename NB>
__device__ __forceinline__ void local_field_c(const LocalCoef<R>& k, NB&& nb, int i, int j, const R* mc, R* b) {
    const int nx = k.nx, ny = k.ny, idx = j * nx + i;
    b[0] = (R)0 + k.bx;
    b[1] = (R)0 + k.by;
    b[2] = (R)0 + k.bz;
    const bool in_c = coef_inside(k, idx);
    const bool want_ex = k.ex_on && in_c, want_dmi = k.dmi_on && in_c;
    R rim[3], rip[3], rjm[3], rjp[3];
    bool vim = false, vip = false, vjm = false, vjp = false;
    if (want_ex || want_dmi) {
        vim = nx > 1 && i > 0 && coef_inside(k, idx - 1);
        vip = nx > 1 && i < nx - 1 && coef_inside(k, idx + 1);
        vjm = ny > 1 && j > 0 && coef_inside(k, idx - nx);
        vjp = ny > 1 && j < ny - 1 && coef_inside(k, idx + nx);
        if (vim) nb(0, rim);
        if (vip) nb(1, rip);
        if (vjm) nb(2, rjm);
        if (vjp) nb(3, rjp);
    }
    const R dx = k.dx, dy = k.dy, eta = k.eta;
    if (want_ex) {
        // exchange ghosts: exchange.rs:8-36
        const bool he = k.has_eta;
        R mim[3], mip[3], mjm[3], mjp[3];
        if (nx == 1) { cp3(mc, mim); cp3(mc, mip); }
        else {
            if (vim) cp3(rim, mim); else if (he) ghost_x(mc, (R)-1, eta, dx, mim); else cp3(mc, mim);
            if (vip) cp3(rip, mip); else if (he) ghost_x(mc, (R)1, eta, dx, mip); else cp3(mc, mip);
        }
        if (ny == 1) { cp3(mc, mjm); cp3(mc, mjp); }
        else {
            if (vjm) cp3(rjm, mjm); else if (he) ghost_y(mc, (R)-1, eta, dy, mjm); else cp3(mc, mjm);
            if (vjp) cp3(rjp, mjp); else if (he) ghost_y(mc, (R)1, eta, dy, mjp); else cp3(mc, mjp);
        }
        exch_core<R>(k, nx > 1, ny > 1, mc, mim, mip, mjm, mjp, b);
    }
    if (k.anis_on) anis_core<R>(k, mc, b);
    if (want_dmi) {
        // DMI ghosts: dmi.rs:19-52
        R mim[3], mip[3], mjm[3], mjp[3];
        if (nx == 1) { cp3(mc, mim); cp3(mc, mip); }
        else {
            if (i == 0) ghost_x(mc, (R)-1, eta, dx, mim); else if (vim) cp3(rim, mim); else cp3(mc, mim);
            if (i == nx - 1) ghost_x(mc, (R)1, eta, dx, mip); else if (vip) cp3(rip, mip); else cp3(mc, mip);
        }
        if (ny == 1) { cp3(mc, mjm); cp3(mc, mjp); }
        else {
            if (j == 0) ghost_y(mc, (R)-1, eta, dy, mjm); else if (vjm) cp3(rjm, mjm); else cp3(mc, mjm);
            if (j == ny - 1) ghost_y(mc, (R)1, eta, dy, mjp); else if (vjp) cp3(rjp, mjp); else cp3(mc, mjp);
        }
        dmi_core<R>(k, nx > 1, ny > 1, mim, mip, mjm, mjp, b);
    }
}

// The same terms for a cell whose four neighbours are film cells (not on an edge,
// no vacuum next to it, film without a mask): no ghost can occur, exchange and DMI
// read the neighbours themselves.  Same arithmetic as local_field_c.
template <typename R, typename NB>
__device__ __forceinline__ void local_field_interior(const LocalCoef<R>& k, NB&& nb, const R* mc, R* b) {
    b[0] = (R)0 + k.bx;
    b[1] = (R)0 + k.by;
    b[2] = (R)0 + k.bz;
    R rim[3], rip[3], rjm[3], rjp[3];
    nb(0, rim);
    nb(1, rip);
    nb(2, rjm);
    nb(3, rjp);
    if (k.ex_on) exch_core<R>(k, true, true, mc, rim, rip, rjm, rjp, b);
    if (k.anis_on) anis_core<R>(k, mc, b);
    if (k.dmi_on) dmi_core<R>(k, true, true, rim, rip, rjm, rjp, b);
}

template <typename R, typename NB>
__device__ __forceinline__ void local_field_nb(const FilmDev& F, NB&& nb, int i, int j, bool dmi_on, const R* mc,
                                               R* b) {
    local_field_c<R>(local_coef<R>(F, dmi_on), nb, i, j, mc, b);
}

template <typename R>
__device__ __forceinline__ void local_field(const FilmDev& F, const R* __restrict__ m, int i, int j, bool dmi_on,
                                            const R* mc, R* b) {
    const int nx = F.nx, n = nx * F.ny, idx = j * nx + i;
    local_field_nb<R>(
        F, [&](int d, R* o) { ld3(m, n, d == 0 ? idx - 1 : d == 1 ? idx + 1 : d == 2 ? idx - nx : idx + nx, o); }, i, j,
        dmi_on, mc, b);
}

// Energy density terms of one cell, FP64 (compute_energy_geom, energy.rs:131-275).
template <typename R>
__device__ __forceinline__ void energy_terms(const FilmDev& F, const R* __restrict__ m, int i, int j,
                                             const double* bd, bool demag_on, double* e) {
    const int nx = F.nx, ny = F.ny, n = nx * ny, idx = j * nx + i;
    if (!cell_inside(F, idx)) return;
    const double dx = F.dx, dy = F.dy, v = F.dx * F.dy * F.dz;
    const double mx = (double)m[idx], my = (double)m[n + idx], mz = (double)m[2 * n + idx];
    const double aex = F.a_ex, ku = F.k_u, ms = F.ms;
    if (aex != 0.0) {
        if (i + 1 < nx && cell_inside(F, idx + 1)) {
            double d0 = (double)m[idx + 1] - mx, d1 = (double)m[n + idx + 1] - my, d2 = (double)m[2 * n + idx + 1] - mz;
            double sq = d0 * d0 + d1 * d1 + d2 * d2;
            e[RED_E_EX] += aex * (sq / (dx * dx)) * v;
        }
        if (j + 1 < ny && cell_inside(F, idx + nx)) {
            double d0 = (double)m[idx + nx] - mx, d1 = (double)m[n + idx + nx] - my,
                   d2 = (double)m[2 * n + idx + nx] - mz;
            double sq = d0 * d0 + d1 * d1 + d2 * d2;
            e[RED_E_EX] += aex * (sq / (dy * dy)) * v;
        }
    }
    if (ku != 0.0) {
        double mdotu = mx * F.u[0] + my * F.u[1] + mz * F.u[2];
        e[RED_E_AN] += ku * (1.0 - mdotu * mdotu) * v;
    }
    if (ms != 0.0) {
        double mdotb = mx * F.bext[0] + my * F.bext[1] + mz * F.bext[2];
        e[RED_E_ZEE] -= ms * mdotb * v;
    }
    const bool has_dmi = F.dmi_avail && F.dmi != 0.0 && aex != 0.0;
    if (has_dmi && ms != 0.0) {
        const double d = F.dmi, eta = d / (2.0 * aex), pref = 2.0 * d / ms;
        double mc[3] = {mx, my, mz}, mim[3], mip[3], mjm[3], mjp[3];
        auto ldd = [&](int id, double* o) {
            o[0] = (double)m[id]; o[1] = (double)m[n + id]; o[2] = (double)m[2 * n + id];
        };
        if (nx == 1) { cp3(mc, mim); cp3(mc, mip); }
        else {
            if (i > 0 && cell_inside(F, idx - 1)) ldd(idx - 1, mim); else ghost_x(mc, -1.0, eta, dx, mim);
            if (i < nx - 1 && cell_inside(F, idx + 1)) ldd(idx + 1, mip); else ghost_x(mc, 1.0, eta, dx, mip);
        }
        if (ny == 1) { cp3(mc, mjm); cp3(mc, mjp); }
        else {
            if (j > 0 && cell_inside(F, idx - nx)) ldd(idx - nx, mjm); else ghost_y(mc, -1.0, eta, dy, mjm);
            if (j < ny - 1 && cell_inside(F, idx + nx)) ldd(idx + nx, mjp); else ghost_y(mc, 1.0, eta, dy, mjp);
        }
        double dmz_dx = nx > 1 ? (mip[2] - mim[2]) / (2.0 * dx) : 0.0;
        double dmz_dy = ny > 1 ? (mjp[2] - mjm[2]) / (2.0 * dy) : 0.0;
        double dmx_dx = nx > 1 ? (mip[0] - mim[0]) / (2.0 * dx) : 0.0;
        double dmy_dy = ny > 1 ? (mjp[1] - mjm[1]) / (2.0 * dy) : 0.0;
        double bx = pref * dmz_dx, by = pref * dmz_dy, bz = -pref * (dmx_dx + dmy_dy);
        e[RED_E_DMI] += -0.5 * ms * (mx * bx + my * by + mz * bz) * v;
    }
    if (demag_on && ms != 0.0) {
        e[RED_E_DEMAG] += -0.5 * ms * (mx * bd[0] + my * bd[1] + mz * bd[2]) * v;
    }
}

// Block reduction of RED_NSLOT doubles (sum, except RED_TMAX: max); thread 0 of
// the block gets the result in red[].  Deterministic order.
__device__ __forceinline__ void block_reduce(double* red, double* sm_red /* [32][RED_NSLOT] */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int s = 0; s < RED_NSLOT; ++s) {
        double v = red[s];
        for (int o = 16; o > 0; o >>= 1) {
            double w = __shfl_down_sync(0xffffffffu, v, o);
            v = (s == RED_TMAX) ? fmax(v, w) : v + w;
        }
        if (lane == 0) sm_red[warp * RED_NSLOT + s] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int s = 0; s < RED_NSLOT; ++s) {
            double v = sm_red[s];
            for (int w = 1; w < nw; ++w) {
                double x = sm_red[w * RED_NSLOT + s];
                v = (s == RED_TMAX) ? fmax(v, x) : v + x;
            }
            red[s] = v;
        }
    }
    __syncthreads();
}

__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// ---------------------------------------------------------------------------
// Pass 1: stage combination + zero-padded R2C along x.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256) k_row_forward(const FilmDev* __restrict__ films,
                                                     const WorkItem* __restrict__ items, int nitems, EvalSpec spec) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<R>* sm = reinterpret_cast<cx<R>*>(smem_raw);
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const WorkItem w = items[it];
        const FilmDev& F = films[w.film];
        const StepState* st = F.st;
        if (skip_item(spec, st)) continue;
        const int nx = F.nx, ny = F.ny, n = nx * ny, T = F.rows_per_block;
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
        const bool do_fft = spec.demag && F.demag_mat;
        const R Ms = (R)F.ms;
        const int L = nx;
        const int G = T + (T + 1) / 2;
        cx<R>* A = sm;
        cx<R>* B = sm + 2 * G * L;
        const cx<R>* __restrict__ tw = reinterpret_cast<const cx<R>*>(F.tw_row);
        for (int e = threadIdx.x; e < T * nx; e += blockDim.x) {
            const int r = e / nx, i = e - r * nx, j = j0 + r;
            R v[3] = {(R)0, (R)0, (R)0};
            if (j < ny) {
                const int idx = j * nx + i;
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
                    else { v[0] = (R)0; v[1] = (R)0; v[2] = (R)0; }  // vacuum pinned at m = 0
                    ms[idx] = v[0]; ms[n + idx] = v[1]; ms[2 * n + idx] = v[2];
                } else {
                    v[0] = ms[idx]; v[1] = ms[n + idx]; v[2] = ms[2 * n + idx];
                }
            }
            if (do_fft) {
                A[(2 * r) * L + i] = mkc(Ms * v[0], Ms * v[1]);
                cx<R>* zp = &A[(2 * (T + r / 2)) * L + i];
                if ((r & 1) == 0) {
                    zp->re = Ms * v[2];
                    if (r + 1 >= T) zp->im = (R)0;
                } else {
                    zp->im = Ms * v[2];
                }
            }
        }
        if (!do_fft) continue;
        __syncthreads();
        for (int e = threadIdx.x; e < G * L; e += blockDim.x) {
            const int g = e / L, i = e - g * L;
            A[(2 * g + 1) * L + i] = cmul(A[(2 * g) * L + i], tw[i]);
        }
        __syncthreads();
        cx<R>* res = fft_smem<R>(A, B, 2 * G, F.plan_row, tw, false);
        cx<R>* __restrict__ X = reinterpret_cast<cx<R>*>(F.X);
        const int K1 = nx + 1;
        const int L2 = 2 * L;
        for (int e = threadIdx.x; e < 3 * K1 * T; e += blockDim.x) {
            const int r = e % T, rest = e / T;
            const int k = rest % K1, c = rest / K1;
            const int j = j0 + r;
            if (j >= ny) continue;
            int g, half;
            if (c < 2) { g = r; half = c; }
            else { g = T + r / 2; half = r & 1; }
            const int km = (L2 - k) % L2;
            cx<R> zk = (k & 1) ? res[(2 * g + 1) * L + (k >> 1)] : res[(2 * g) * L + (k >> 1)];
            cx<R> zm = (km & 1) ? res[(2 * g + 1) * L + (km >> 1)] : res[(2 * g) * L + (km >> 1)];
            cx<R> out;
            if (half == 0) out = mkc((R)0.5 * (zk.re + zm.re), (R)0.5 * (zk.im - zm.im));
            else out = mkc((R)0.5 * (zk.im + zm.im), (R)0.5 * (zm.re - zk.re));
            X[(c * K1 + k) * ny + j] = out;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Pass 2: y transform, kernel multiply, inverse y transform (one kx column).
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256) k_column(const FilmDev* __restrict__ films, const WorkItem* __restrict__ items,
                                                int nitems, EvalSpec spec) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<R>* sm = reinterpret_cast<cx<R>*>(smem_raw);
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const WorkItem w = items[it];
        const FilmDev& F = films[w.film];
        const StepState* st = F.st;
        if (skip_item(spec, st)) continue;
        if (!(spec.demag && F.demag_mat)) continue;
        const int nx = F.nx, ny = F.ny, K1 = nx + 1, L = ny;
        const int kx = w.blk;
        cx<R>* __restrict__ X = reinterpret_cast<cx<R>*>(F.X);
        const r4<R>* __restrict__ Kh = reinterpret_cast<const r4<R>*>(F.Khat) + (size_t)kx * (ny + 1);
        const cx<R>* __restrict__ tw = reinterpret_cast<const cx<R>*>(F.tw_col);
        cx<R>* A = sm;
        cx<R>* B = sm + 6 * L;
        for (int e = threadIdx.x; e < 3 * L; e += blockDim.x) {
            const int c = e / L, y = e - c * L;
            cx<R> x = X[(c * K1 + kx) * ny + y];
            A[(2 * c) * L + y] = x;
            A[(2 * c + 1) * L + y] = cmul(x, tw[y]);
        }
        __syncthreads();
        cx<R>* res = fft_smem<R>(A, B, 6, F.plan_col, tw, false);
        for (int e = threadIdx.x; e < 2 * L; e += blockDim.x) {
            const int par = e / L, kk = e - par * L;
            const int ky = 2 * kk + par;
            const int kyf = ky <= ny ? ky : 2 * ny - ky;
            const r4<R> K = Kh[kyf];
            const R kxy = ky <= ny ? K.y : -K.y;
            cx<R> Mx = res[(0 + par) * L + kk], My = res[(2 + par) * L + kk], Mz = res[(4 + par) * L + kk];
            res[(0 + par) * L + kk] = mkc(K.x * Mx.re + kxy * My.re, K.x * Mx.im + kxy * My.im);
            res[(2 + par) * L + kk] = mkc(kxy * Mx.re + K.z * My.re, kxy * Mx.im + K.z * My.im);
            res[(4 + par) * L + kk] = mkc(K.w * Mz.re, K.w * Mz.im);
        }
        __syncthreads();
        cx<R>* other = (res == A) ? B : A;
        cx<R>* res2 = fft_smem<R>(res, other, 6, F.plan_col, tw, true);
        for (int e = threadIdx.x; e < 3 * L; e += blockDim.x) {
            const int c = e / L, y = e - c * L;
            X[(c * K1 + kx) * ny + y] = res2[(2 * c) * L + y] + cmulc(res2[(2 * c + 1) * L + y], tw[y]);
        }
        __syncthreads();
    }
}

// Per-cell epilogue of the row-inverse pass (shared by the generic and the
// register-FFT kernels): local terms, demag from dfield(r, i, c), torque,
// stage torque store, RK error norm and FP64 block reductions.  MIN selects the
// minimiser update (RHS_MINIMIZE) instead; it is a separate instantiation so
// that the integrator kernels keep their register budget.
template <typename R, bool MIN, typename DF>
__device__ __forceinline__ void row_epilogue(const FilmDev& F, const EvalSpec& spec, StepState* st, int blk, int T,
                                             bool do_fft, DF dfield, double* sm_red) {
    const int nx = F.nx, ny = F.ny, n = nx * ny;
    const int j0 = blk * T;
    const int cur = st->cur;
        const R* __restrict__ msb = mbuf<R>(F, spec.m_in, cur);
        R* __restrict__ kout = spec.k_out != KB_NONE ? kbuf<R>(F, spec.k_out, cur) : nullptr;
        R* __restrict__ bout = reinterpret_cast<R*>(F.bout);
        R* __restrict__ mout = MIN ? mbuf<R>(F, MB_M7, cur) : nullptr;
        const R gam = (R)F.gamma, alp = (R)F.alpha;
        const double dt = st->dt;
        double red[RED_NSLOT];
#pragma unroll
        for (int s = 0; s < RED_NSLOT; ++s) red[s] = 0.0;
        double errmax = 0.0;
        bool errnan = false;
        for (int e = threadIdx.x; e < T * nx; e += blockDim.x) {
            const int r = e / nx, i = e - r * nx, j = j0 + r;
            if (j >= ny) continue;
            const int idx = j * nx + i;
            R mc[3];
            ld3(msb, n, idx, mc);
            R b[3];
            if (spec.rhs == RHS_ENERGY) {
                double bd[3] = {0.0, 0.0, 0.0};
                if (do_fft) {
                    bd[0] = (double)dfield(r, i, 0);
                    bd[1] = (double)dfield(r, i, 1);
                    bd[2] = (double)dfield(r, i, 2);
                }
                energy_terms<R>(F, msb, i, j, bd, do_fft, red);
                continue;
            }
            if (spec.local) {
                local_field<R>(F, msb, i, j, spec.dmi != 0, mc, b);
            } else {
                b[0] = (R)0; b[1] = (R)0; b[2] = (R)0;
            }
            if (do_fft) {
                b[0] += dfield(r, i, 0);
                b[1] += dfield(r, i, 1);
                b[2] += dfield(r, i, 2);
            }
            if (spec.rhs == RHS_FIELD) {
                bout[idx] = b[0]; bout[n + idx] = b[1]; bout[2 * n + idx] = b[2];
            }
            // torque m x B and m x (m x B) (llg.rs:20-32, 38-50)
            R k[3] = {(R)0, (R)0, (R)0};
            if (spec.rhs == RHS_LLG || spec.rhs == RHS_RELAX) {
                const R denom = (R)1 + alp * alp;
                const bool llg = spec.rhs == RHS_LLG;
                torque_cell<R>(mc, b, llg ? -gam / denom : -gam * alp / denom, llg ? (R)1 : (R)0, llg ? alp : (R)1, k);
                kout[idx] = k[0]; kout[n + idx] = k[1]; kout[2 * n + idx] = k[2];
            }
            if (spec.reduce) {
                // torque metrics in FP64 (relax.rs:144-189)
                double d0 = (double)mc[1] * (double)b[2] - (double)mc[2] * (double)b[1];
                double d1 = (double)mc[2] * (double)b[0] - (double)mc[0] * (double)b[2];
                double d2 = (double)mc[0] * (double)b[1] - (double)mc[1] * (double)b[0];
                double t2s = d0 * d0 + d1 * d1 + d2 * d2;
                double tm = sqrt(t2s);
                red[RED_TSUM] += tm;
                red[RED_TSUM2] += t2s;
                red[RED_TMAX] = fmax(red[RED_TMAX], tm);
                red[RED_MX] += (double)mc[0];
                red[RED_MY] += (double)mc[1];
                red[RED_MZ] += (double)mc[2];
            }
            if constexpr (MIN) {
                // damping-only descent update in FP64 (minimize.rs:221-254):
                // d = (m x B) x m, m' = normalize(m + lambda d), dM = |m' - m| of the stored values
                const double m0 = (double)mc[0], m1 = (double)mc[1], m2 = (double)mc[2];
                const double b0 = (double)b[0], b1 = (double)b[1], b2 = (double)b[2];
                const double q0 = m1 * b2 - m2 * b1, q1 = m2 * b0 - m0 * b2, q2 = m0 * b1 - m1 * b0;
                const double lam = st->lam;
                double x = m0 + lam * (q1 * m2 - q2 * m1);
                double y = m1 + lam * (q2 * m0 - q0 * m2);
                double z = m2 + lam * (q0 * m1 - q1 * m0);
                const double n2 = x * x + y * y + z * z;
                if (n2 > 0.0) {
                    const double inv = 1.0 / sqrt(n2);
                    x *= inv;
                    y *= inv;
                    z *= inv;
                }
                const R xs = (R)x, ys = (R)y, zs = (R)z;
                mout[idx] = xs; mout[n + idx] = ys; mout[2 * n + idx] = zs;
                const double ex = (double)xs - m0, ey = (double)ys - m1, ez = (double)zs - m2;
                // max dM through the error-norm accumulator (an order-independent max)
                errmax = fmax(errmax, sqrt(ex * ex + ey * ey + ez * ez));
            }
            if (spec.err == ERR_RK45) {
                // eps contribution: max_c |sum b_q k_q - sum bhat_q k_q| (llg.rs:948-997), FP64
                double th[3] = {0.0, 0.0, 0.0}, tl[3] = {0.0, 0.0, 0.0};
#pragma unroll
                for (int q = 1; q <= 7; ++q) {
                    const double wb = spec.wb[q], wh = spec.wh[q];
                    if (wb == 0.0 && wh == 0.0) continue;
                    double kq[3];
                    if (q == 7) {
                        kq[0] = (double)k[0]; kq[1] = (double)k[1]; kq[2] = (double)k[2];
                    } else {
                        const R* kb = kbuf<R>(F, q, cur);
                        kq[0] = (double)kb[idx]; kq[1] = (double)kb[n + idx]; kq[2] = (double)kb[2 * n + idx];
                    }
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        th[c] = th[c] + wb * kq[c];
                        tl[c] = tl[c] + wh * kq[c];
                    }
                }
                double dm = fmax(fmax(fabs(th[0] - tl[0]), fabs(th[1] - tl[1])), fabs(th[2] - tl[2]));
                if (dm != dm) errnan = true;
                else errmax = fmax(errmax, dm);
            } else if (spec.err == ERR_RK23) {
                // eps contribution: max |m_3rd - m_2nd| (llg.rs:386-401), both recomputed in FP64
                if (cell_inside(F, idx)) {
                    const R* K1p = kbuf<R>(F, KB_K1, cur);
                    const R* K2p = kbuf<R>(F, KB_K2, cur);
                    const R* K3p = kbuf<R>(F, KB_K3, cur);
                    const R* M0p = mbuf<R>(F, MB_M0, cur);
                    double m3[3], m2[3];
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const int o = c * n + idx;
                        double base = (double)M0p[o];
                        double k1 = (double)K1p[o], k2 = (double)K2p[o], k3 = (double)K3p[o], k4 = (double)k[c];
                        double x = base;
                        x = x + (dt * spec.wb[1]) * k1;
                        x = x + (dt * spec.wb[2]) * k2;
                        x = x + (dt * spec.wb[3]) * k3;
                        m3[c] = x;
                        double y = base;
                        y = y + (dt * spec.wh[1]) * k1;
                        y = y + (dt * spec.wh[2]) * k2;
                        y = y + (dt * spec.wh[3]) * k3;
                        y = y + (dt * spec.wh[4]) * k4;
                        m2[c] = y;
                    }
                    normalize3(m3);
                    normalize3(m2);
                    double dm = fmax(fmax(fabs(m3[0] - m2[0]), fabs(m3[1] - m2[1])), fabs(m3[2] - m2[2]));
                    if (dm != dm) errnan = true;
                    else errmax = fmax(errmax, dm);
                }
            }
        }
        if (MIN || spec.err != ERR_NONE) {
            // non-negative doubles order like their bit patterns; NaN is reported
            // as a quiet-NaN pattern, above every finite value and +inf
            const double v = warp_max(errmax);
            const bool anynan = __any_sync(0xffffffffu, errnan);
            if ((threadIdx.x & 31) == 0) {
                unsigned long long bits = anynan ? 0x7ff8000000000000ull : (unsigned long long)__double_as_longlong(v);
                atomicMax(&st->err_bits, bits);
            }
        }
        if (spec.reduce) {
            block_reduce(red, sm_red);
            if (threadIdx.x == 0) {
                double* dst = F.red_part + (size_t)blk * RED_NSLOT;
                for (int s = 0; s < RED_NSLOT; ++s) dst[s] = red[s];
            }
        }
}

// Warp maximum of the error norm into the film's accumulator: non-negative doubles
// order like their bit patterns; NaN is reported as a quiet-NaN pattern, above every
// finite value and +inf.  All lanes of the warp must call it for the same film.
__device__ __forceinline__ void err_to_state(StepState* st, double errmax, bool errnan) {
    const double v = warp_max(errmax);
    const bool anynan = __any_sync(0xffffffffu, errnan);
    if ((threadIdx.x & 31) == 0) {
        unsigned long long bits = anynan ? 0x7ff8000000000000ull : (unsigned long long)__double_as_longlong(v);
        atomicMax(&st->err_bits, bits);
    }
}

// ---------------------------------------------------------------------------
// Pass 3: C2R along x + local terms + torque + error norm + reductions.
// ---------------------------------------------------------------------------
template <typename R, bool MIN>
__global__ void __launch_bounds__(256) k_row_inverse(const FilmDev* __restrict__ films,
                                                     const WorkItem* __restrict__ items, int nitems, EvalSpec spec) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double sm_red[32 * RED_NSLOT];
    cx<R>* sm = reinterpret_cast<cx<R>*>(smem_raw);
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const WorkItem w = items[it];
        const FilmDev& F = films[w.film];
        StepState* st = F.st;
        if (skip_item(spec, st)) continue;
        const int nx = F.nx, ny = F.ny, T = F.rows_per_block;
        const int j0 = w.blk * T;
        const int L = nx, K1 = nx + 1, L2 = 2 * nx;
        const int G = T + (T + 1) / 2, P = (T + 1) / 2;
        const bool do_fft = spec.demag && F.demag_mat;
        const cx<R>* __restrict__ tw = reinterpret_cast<const cx<R>*>(F.tw_row);
        R* D = nullptr;
        if (do_fft) {
            const cx<R>* __restrict__ X = reinterpret_cast<const cx<R>*>(F.X);
            cx<R>* A = sm;
            cx<R>* B = sm + 2 * G * L;
            auto xval = [&](int c, int k, int j) -> cx<R> {
                if (k <= nx) return X[(c * K1 + k) * ny + j];
                return conjc(X[(c * K1 + (L2 - k)) * ny + j]);
            };
            for (int e = threadIdx.x; e < L2 * T; e += blockDim.x) {
                const int r = e % T, k = e / T, j = j0 + r;
                cx<R> z = mkc((R)0, (R)0);
                if (j < ny) {
                    cx<R> bx = xval(0, k, j), by = xval(1, k, j);
                    z = mkc(bx.re - by.im, bx.im + by.re);
                }
                A[(2 * r + (k & 1)) * L + (k >> 1)] = z;
            }
            for (int e = threadIdx.x; e < L2 * P; e += blockDim.x) {
                const int p = e % P, k = e / P;
                const int ja = j0 + 2 * p, jb = j0 + 2 * p + 1;
                cx<R> za = (ja < ny) ? xval(2, k, ja) : mkc((R)0, (R)0);
                cx<R> zb = (2 * p + 1 < T && jb < ny) ? xval(2, k, jb) : mkc((R)0, (R)0);
                A[(2 * (T + p) + (k & 1)) * L + (k >> 1)] = mkc(za.re - zb.im, za.im + zb.re);
            }
            __syncthreads();
            cx<R>* res = fft_smem<R>(A, B, 2 * G, F.plan_row, tw, true);
            D = reinterpret_cast<R*>(res == A ? B : A);
            for (int e = threadIdx.x; e < G * L; e += blockDim.x) {
                const int g = e / L, x = e - g * L;
                cx<R> z = res[(2 * g) * L + x] + cmulc(res[(2 * g + 1) * L + x], tw[x]);
                if (g < T) {
                    D[(g * 3 + 0) * L + x] = z.re;
                    D[(g * 3 + 1) * L + x] = z.im;
                } else {
                    const int p = g - T;
                    D[((2 * p) * 3 + 2) * L + x] = z.re;
                    if (2 * p + 1 < T) D[((2 * p + 1) * 3 + 2) * L + x] = z.im;
                }
            }
            __syncthreads();
        }
        auto dfield = [&](int r, int i, int c) -> R { return D[(r * 3 + c) * L + i]; };
        row_epilogue<R, MIN>(F, spec, st, w.blk, T, do_fft, dfield, sm_red);
        __syncthreads();
    }
}

}  // namespace llg
