// stage_kernels.cuh — the torque epilogue of an RK stage on the register-FFT
// path, split out of the row-inverse FFT kernel so that it runs at full
// occupancy: k_stage_torque takes the local terms and the demag field that the
// row-inverse transform left in the film's bdem planes, forms the torque, stores
// k_s and, for the last RK45 stage, the error norm.  It walks the row work items
// of one launch segment, CPI cells per item (a multiple of 512, so a warp never
// spans two items and therefore never two films).
#pragma once
#include "field_kernels.cuh"

namespace llg {

// One cell per thread, consecutive threads on consecutive cells of a row
// (coalesced loads, ~60 registers, high occupancy).
template <typename R, bool ERR45>
__global__ void __launch_bounds__(256, 4) k_stage_torque(const FilmDev* __restrict__ films,
                                                          const WorkItem* __restrict__ items, int nitems, int cpi,
                                                          EvalSpec spec) {
    const long long total = (long long)nitems * cpi;
    int coef_film = -1;
    LocalCoef<R> cf;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < total;
         v += (long long)gridDim.x * blockDim.x) {
        const WorkItem w = items[v / cpi];
        const FilmDev& F = films[w.film];
        if (w.film != coef_film) {   // coefficients of the local terms, once per film
            cf = local_coef<R>(F, spec.dmi != 0);
            coef_film = w.film;
        }
        StepState* st = F.st;
        if (skip_item(spec, st)) continue;   // uniform over the warp (one item per warp)
        const int nx = F.nx, ny = F.ny, n = nx * ny;
        const int c0 = (int)(v % cpi), r = c0 / nx, i = c0 - r * nx, j = w.blk * F.rows_per_block + r;
        double errmax = 0.0;
        bool errnan = false;
        if (j < ny) {
            const int idx = j * nx + i, cur = st->cur;
            const R* __restrict__ msb = mbuf<R>(F, spec.m_in, cur);
            R* __restrict__ kout = kbuf<R>(F, spec.k_out, cur);
            R mc[3], b[3];
            ld3(msb, n, idx, mc);
            local_field_c<R>(
                cf, [&](int d, R* o) { ld3(msb, n, d == 0 ? idx - 1 : d == 1 ? idx + 1 : d == 2 ? idx - nx : idx + nx, o); },
                i, j, mc, b);
            if (spec.demag && F.demag_mat) {
                const R* bd = reinterpret_cast<const R*>(F.bdem);
                b[0] += bd[idx];
                b[1] += bd[n + idx];
                b[2] += bd[2 * n + idx];
            }
            const R gam = (R)F.gamma, alp = (R)F.alpha;
            const R denom = (R)1 + alp * alp;
            const R pref = spec.rhs == RHS_LLG ? -gam / denom : -gam * alp / denom;
            const R c1 = spec.rhs == RHS_LLG ? (R)1 : (R)0;
            const R c2 = spec.rhs == RHS_LLG ? alp : (R)1;
            R k[3];
            torque_cell<R>(mc, b, pref, c1, c2, k);
            kout[idx] = k[0];
            kout[n + idx] = k[1];
            kout[2 * n + idx] = k[2];
            if constexpr (ERR45) {
                double th[3] = {0.0, 0.0, 0.0}, tl[3] = {0.0, 0.0, 0.0};
#pragma unroll
                for (int q = 1; q <= 7; ++q) {
                    const double wb = spec.wb[q], wh = spec.wh[q];
                    if (wb == 0.0 && wh == 0.0) continue;
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const double kq = q == 7 ? (double)k[c] : (double)kbuf<R>(F, q, cur)[c * n + idx];
                        th[c] = th[c] + wb * kq;
                        tl[c] = tl[c] + wh * kq;
                    }
                }
                const double dm = fmax(fmax(fabs(th[0] - tl[0]), fabs(th[1] - tl[1])), fabs(th[2] - tl[2]));
                if (dm != dm) errnan = true;
                else errmax = dm;
            }
        }
        if constexpr (ERR45) err_to_state(st, errmax, errnan);
    }
}

}  // namespace llg
