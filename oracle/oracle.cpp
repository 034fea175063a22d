// oracle.cpp — CPU FP64 restatement of llg-sim's uniform-grid LLG hot path.
//
// TEST INFRASTRUCTURE ONLY (see oracle.h).  Citations are to files of the
// llg-sim project (src/...).  Compiled with -ffp-contract=off so that every
// expression rounds in the order written, as the Rust reference does.
//
// Threading mirrors the reference: OpenMP only where the reference uses rayon
// (demag pack / FFT rows and columns / k-space multiply / unpack,
// demag_fft_uniform.rs:653-768, 794-838); every other loop is serial.

#include "oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const double PI = 3.14159265358979323846;
const double MU0 = 4.0 * PI * 1e-7;  // params.rs:15
const double DEMAG_ACCURACY = 10.0;  // demag_fft_uniform.rs:432

struct cplx {
    double re, im;
};
inline cplx cadd(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
inline cplx csub(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
inline cplx cmul(cplx a, cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }

typedef double v3[3];

inline void vcross(const double* a, const double* b, double* o) {
    // vec3.rs:10-16
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
inline void vnormalize(const double* v, double* o) {
    // vec3.rs:21-28: zero vector maps to +z
    double n2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    if (n2 == 0.0) {
        o[0] = 0.0; o[1] = 0.0; o[2] = 1.0;
        return;
    }
    double inv = 1.0 / std::sqrt(n2);
    o[0] = v[0] * inv; o[1] = v[1] * inv; o[2] = v[2] * inv;
}

// ---------------------------------------------------------------------------
// FFT: mixed-radix Stockham autosort (own implementation; stands in for
// rustfft's FftPlanner, demag_fft_uniform.rs:484-488).  Unnormalised.
// ---------------------------------------------------------------------------
struct Fft1D {
    int64_t n = 0;
    bool inverse = false;
    std::vector<int> radices;
    std::vector<cplx> tw;  // tw[k] = exp(sign * 2 pi i k / n)

    Fft1D() {}
    Fft1D(int64_t n_, bool inv) : n(n_), inverse(inv) {
        int64_t r = n;
        for (int p : {4, 2, 3, 5}) {
            while (r % p == 0) { radices.push_back(p); r /= p; }
        }
        for (int64_t p = 7; r > 1; p += 2) {
            while (r % p == 0) { radices.push_back((int)p); r /= p; }
        }
        tw.resize(std::max<int64_t>(n, 1));
        double sign = inverse ? 1.0 : -1.0;
        for (int64_t k = 0; k < n; ++k) {
            double a = sign * 2.0 * PI * (double)k / (double)n;
            tw[k] = {std::cos(a), std::sin(a)};
        }
    }

    // data: n complex, work: n complex scratch.  Result left in data.
    void exec(cplx* data, cplx* work) const {
        if (n <= 1) return;
        cplx* a = data;
        cplx* b = work;
        int64_t ns = 1;
        cplx v[64];
        std::vector<cplx> vbig;
        for (int p : radices) {
            cplx* vv = v;
            if (p > 64) { vbig.resize(p); vv = vbig.data(); }
            int64_t m = n / p;
            int64_t tstep = n / (ns * p);
            for (int64_t j = 0; j < m; ++j) {
                int64_t k = j % ns;
                for (int r = 0; r < p; ++r) {
                    cplx x = a[j + r * m];
                    int64_t ti = (k * r * tstep) % n;
                    vv[r] = (r == 0 || k == 0) ? x : cmul(x, tw[ti]);
                }
                int64_t base = (j / ns) * ns * p + k;
                butterfly(vv, p, b + base, ns);
            }
            std::swap(a, b);
            ns *= p;
        }
        if (a != data) std::memcpy(data, a, sizeof(cplx) * n);
    }

    void butterfly(const cplx* x, int p, cplx* out, int64_t stride) const {
        if (p == 2) {
            out[0] = cadd(x[0], x[1]);
            out[stride] = csub(x[0], x[1]);
        } else if (p == 4) {
            cplx s02 = cadd(x[0], x[2]), d02 = csub(x[0], x[2]);
            cplx s13 = cadd(x[1], x[3]), d13 = csub(x[1], x[3]);
            // multiply d13 by -i (forward) or +i (inverse)
            cplx rd = inverse ? cplx{-d13.im, d13.re} : cplx{d13.im, -d13.re};
            out[0] = cadd(s02, s13);
            out[stride] = cadd(d02, rd);
            out[2 * stride] = csub(s02, s13);
            out[3 * stride] = csub(d02, rd);
        } else {
            // generic p-point DFT with twiddles tw[(q*r*(n/p)) % n]
            int64_t unit = n / p;
            for (int q = 0; q < p; ++q) {
                cplx acc = x[0];
                for (int r = 1; r < p; ++r) {
                    int64_t ti = ((int64_t)q * r % p) * unit;
                    acc = cadd(acc, cmul(x[r], tw[ti]));
                }
                out[q * stride] = acc;
            }
        }
    }
};

int g_threads = 1;
// Variant of the CPU baseline: the reference runs its local field terms, torques and
// RK combinations serially on the caller (only the FFT demag uses rayon); with
// g_par_local set those per-cell loops run OpenMP-parallel too.  Each cell's
// arithmetic is unchanged, so results are identical in both modes.
bool g_par_local = false;

// fft2 over a px-by-py row-major array: rows then columns
// (demag_fft_uniform.rs:777-922).  inverse scales by 1/(px*py) at the end.
void fft2(std::vector<cplx>& d, int64_t px, int64_t py, const Fft1D& fx, const Fft1D& fy, bool inverse) {
#pragma omp parallel num_threads(g_threads)
    {
        std::vector<cplx> work(std::max(px, py));
        std::vector<cplx> col(py);
#pragma omp for schedule(static)
        for (int64_t y = 0; y < py; ++y) fx.exec(&d[y * px], work.data());
#pragma omp for schedule(static)
        for (int64_t x = 0; x < px; ++x) {
            for (int64_t y = 0; y < py; ++y) col[y] = d[y * px + x];
            fy.exec(col.data(), work.data());
            for (int64_t y = 0; y < py; ++y) d[y * px + x] = col[y];
        }
        if (inverse) {
            double scale = 1.0 / (double)(px * py);
#pragma omp for schedule(static)
            for (int64_t i = 0; i < px * py; ++i) {
                d[i].re *= scale;
                d[i].im *= scale;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Demag kernel: MuMax-like face-charge integration (demag_fft_uniform.rs)
// ---------------------------------------------------------------------------
inline double delta_cell(int64_t d) {
    // demag_fft_uniform.rs:1247-1253
    double a = (double)(d < 0 ? -d : d);
    if (a > 0.0) a -= 1.0;
    return a;
}
inline int64_t mumax_n(double x) {
    // demag_fft_uniform.rs:1164-1166
    return (int64_t)std::floor(std::max(x, 1.0) + 0.5);
}

void h_from_unit_m(int u, const double* r_center, const double* cell, const int64_t* disp,
                   double accuracy, double* h) {
    // demag_fft_uniform.rs:1139-1242, same loop order and rounding order
    int v = (u + 1) % 3;
    int w = (u + 2) % 3;
    double lmin = std::min(std::min(cell[0], cell[1]), cell[2]);
    double dx_min = delta_cell(disp[0]) * cell[0];
    double dy_min = delta_cell(disp[1]) * cell[1];
    double dz_min = delta_cell(disp[2]) * cell[2];
    double d = std::sqrt(dx_min * dx_min + dy_min * dy_min + dz_min * dz_min);
    if (d == 0.0) d = lmin;
    double max_size = d / accuracy;
    int64_t nx = mumax_n(cell[0] / max_size);
    int64_t ny = mumax_n(cell[1] / max_size);
    int64_t nz = mumax_n(cell[2] / max_size);
    int64_t nv = mumax_n(cell[v] / max_size);
    int64_t nw = mumax_n(cell[w] / max_size);
    nv *= 2;
    nw *= 2;
    double scale = 1.0 / (double)(nv * nw * nx * ny * nz);
    double face_area = cell[v] * cell[w];
    double charge = face_area * scale;
    double pu1 = 0.5 * cell[u];
    double pu2 = -pu1;
    double pole[3] = {0.0, 0.0, 0.0};
    h[0] = h[1] = h[2] = 0.0;
    for (int64_t i = 0; i < nv; ++i) {
        double pv = -0.5 * cell[v] + cell[v] / (2.0 * (double)nv) + (double)i * (cell[v] / (double)nv);
        pole[v] = pv;
        for (int64_t j = 0; j < nw; ++j) {
            double pw = -0.5 * cell[w] + cell[w] / (2.0 * (double)nw) + (double)j * (cell[w] / (double)nw);
            pole[w] = pw;
            for (int64_t ax = 0; ax < nx; ++ax) {
                double rx = r_center[0] - 0.5 * cell[0] + cell[0] / (2.0 * (double)nx) +
                            (double)ax * (cell[0] / (double)nx);
                for (int64_t ay = 0; ay < ny; ++ay) {
                    double ry = r_center[1] - 0.5 * cell[1] + cell[1] / (2.0 * (double)ny) +
                                (double)ay * (cell[1] / (double)ny);
                    for (int64_t az = 0; az < nz; ++az) {
                        double rz = r_center[2] - 0.5 * cell[2] + cell[2] / (2.0 * (double)nz) +
                                    (double)az * (cell[2] / (double)nz);
                        pole[u] = pu1;
                        double r1x = rx - pole[0];
                        double r1y = ry - pole[1];
                        double r1z = rz - pole[2];
                        double r1 = std::sqrt(r1x * r1x + r1y * r1y + r1z * r1z);
                        double q1 = charge / (4.0 * PI * r1 * r1 * r1);
                        double hx1 = r1x * q1;
                        double hy1 = r1y * q1;
                        double hz1 = r1z * q1;
                        pole[u] = pu2;
                        double r2x = rx - pole[0];
                        double r2y = ry - pole[1];
                        double r2z = rz - pole[2];
                        double r2 = std::sqrt(r2x * r2x + r2y * r2y + r2z * r2z);
                        double q2 = -charge / (4.0 * PI * r2 * r2 * r2);
                        h[0] += hx1 + r2x * q2;
                        h[1] += hy1 + r2y * q2;
                        h[2] += hz1 + r2z * q2;
                    }
                }
            }
        }
    }
}

void kernel_components(double dx, double dy, double dz, int64_t sx, int64_t sy, double acc, double* out) {
    // demag_fft_uniform.rs:1076-1097
    double rc[3] = {(double)sx * dx, (double)sy * dy, 0.0};
    double cell[3] = {dx, dy, dz};
    int64_t disp[3] = {sx, sy, 0};
    double hx[3], hy[3], hz[3];
    h_from_unit_m(0, rc, cell, disp, acc, hx);
    h_from_unit_m(1, rc, cell, disp, acc, hy);
    h_from_unit_m(2, rc, cell, disp, acc, hz);
    out[0] = MU0 * hx[0];  // xx
    out[1] = MU0 * hy[0];  // xy (Hx from My)
    out[2] = MU0 * hy[1];  // yy
    out[3] = MU0 * hz[2];  // zz
}

inline int64_t wrap_index(int64_t d, int64_t n) {
    // demag_fft_uniform.rs:198-205
    int64_t v = d % n;
    if (v < 0) v += n;
    return v;
}

// Real-space kernel (4 planes of px*py doubles).
void build_kernel_realspace(const orc_grid& g, int64_t px, int64_t py, int64_t pbc_x, int64_t pbc_y,
                            std::vector<double>* k4) {
    for (int c = 0; c < 4; ++c) k4[c].assign(px * py, 0.0);
    if (pbc_x == 0 && pbc_y == 0) {
        // build_kernel_realspace_mumax_2d, demag_fft_uniform.rs:1013-1072
        int64_t rx_max = g.nx - 1, ry_max = g.ny - 1;
        std::vector<double> quad((rx_max + 1) * (ry_max + 1) * 4);
#pragma omp parallel for schedule(dynamic, 1) num_threads(g_threads)
        for (int64_t q = 0; q < (rx_max + 1) * (ry_max + 1); ++q) {
            int64_t sy = q / (rx_max + 1), sx = q % (rx_max + 1);
            kernel_components(g.dx, g.dy, g.dz, sx, sy, DEMAG_ACCURACY, &quad[q * 4]);
        }
        for (int64_t sy = 0; sy <= ry_max; ++sy) {
            for (int64_t sx = 0; sx <= rx_max; ++sx) {
                const double* kc = &quad[(sy * (rx_max + 1) + sx) * 4];
                for (int64_t sxs : {1, -1}) {
                    for (int64_t sys : {1, -1}) {
                        int64_t ix = wrap_index(sxs * sx, px), iy = wrap_index(sys * sy, py);
                        int64_t idx = iy * px + ix;
                        k4[0][idx] = kc[0];
                        k4[1][idx] = (double)sxs * (double)sys * kc[1];
                        k4[2][idx] = kc[2];
                        k4[3][idx] = kc[3];
                    }
                }
            }
        }
        for (int64_t sy = -ry_max; sy <= ry_max; ++sy) k4[1][wrap_index(sy, py) * px + wrap_index(0, px)] = 0.0;
        for (int64_t sx = -rx_max; sx <= rx_max; ++sx) k4[1][wrap_index(0, py) * px + wrap_index(sx, px)] = 0.0;
    } else {
        // build_kernel_realspace_pbc, demag_fft_uniform.rs:941-1005
        int64_t sx_max = pbc_x == 0 ? g.nx - 1 : g.nx * pbc_x - 1;
        int64_t sy_max = pbc_y == 0 ? g.ny - 1 : g.ny * pbc_y - 1;
        const int64_t nsx = 2 * sx_max + 1, nsy = 2 * sy_max + 1;
        std::vector<double> comp((size_t)(nsx * nsy * 4));
        // the displacements in parallel, then the wrapped sums in the reference's order
#pragma omp parallel for schedule(dynamic, 16) num_threads(g_threads)
        for (int64_t q = 0; q < nsx * nsy; ++q)
            kernel_components(g.dx, g.dy, g.dz, q % nsx - sx_max, q / nsx - sy_max, DEMAG_ACCURACY, &comp[q * 4]);
        for (int64_t sy = -sy_max; sy <= sy_max; ++sy) {
            int64_t iy = wrap_index(sy, py);
            for (int64_t sx = -sx_max; sx <= sx_max; ++sx) {
                int64_t ix = wrap_index(sx, px);
                const double* kc = &comp[((sy + sy_max) * nsx + (sx + sx_max)) * 4];
                for (int c = 0; c < 4; ++c) k4[c][iy * px + ix] += kc[c];
            }
        }
        for (int64_t sy = -sy_max; sy <= sy_max; ++sy) k4[1][wrap_index(sy, py) * px + wrap_index(0, px)] = 0.0;
        for (int64_t sx = -sx_max; sx <= sx_max; ++sx) k4[1][wrap_index(0, py) * px + wrap_index(sx, px)] = 0.0;
    }
}

// ---------------------------------------------------------------------------
// Demag operator (Demag2D, demag_fft_uniform.rs:434-770): open boundaries, or
// pbc_x / pbc_y periodic images (no padding in a periodic direction).
// ---------------------------------------------------------------------------
struct Demag2D {
    orc_grid g;
    int64_t px, py;
    Fft1D fx_f, fx_i, fy_f, fy_i;
    std::vector<cplx> kxx, kxy, kyy, kzz;
    std::vector<cplx> mx, my, mz, bx, by, bz;

    explicit Demag2D(const orc_grid& grid, int64_t pbc_x = 0, int64_t pbc_y = 0) : g(grid) {
        px = pbc_x > 0 ? g.nx : 2 * g.nx;  // demag_fft_uniform.rs:477-478
        py = pbc_y > 0 ? g.ny : 2 * g.ny;
        fx_f = Fft1D(px, false); fx_i = Fft1D(px, true);
        fy_f = Fft1D(py, false); fy_i = Fft1D(py, true);
        std::vector<double> k4[4];
        build_kernel_realspace(g, px, py, pbc_x, pbc_y, k4);
        std::vector<cplx>* dst[4] = {&kxx, &kxy, &kyy, &kzz};
        for (int c = 0; c < 4; ++c) {
            dst[c]->resize(px * py);
            for (int64_t i = 0; i < px * py; ++i) (*dst[c])[i] = {k4[c][i], 0.0};
            fft2(*dst[c], px, py, fx_f, fy_f, false);  // :573-576
        }
        for (auto* v : {&mx, &my, &mz, &bx, &by, &bz}) v->assign(px * py, {0.0, 0.0});
    }

    // Demag2D::add_field, demag_fft_uniform.rs:636-769
    void add_field(const double* m, double* b, double ms) {
        int64_t nx = g.nx, ny = g.ny;
        std::fill(mx.begin(), mx.end(), cplx{0.0, 0.0});
        std::fill(my.begin(), my.end(), cplx{0.0, 0.0});
        std::fill(mz.begin(), mz.end(), cplx{0.0, 0.0});
#pragma omp parallel for schedule(static) num_threads(g_threads)
        for (int64_t j = 0; j < ny; ++j) {
            for (int64_t i = 0; i < nx; ++i) {
                const double* v = &m[(j * nx + i) * 3];
                mx[j * px + i].re = ms * v[0];
                my[j * px + i].re = ms * v[1];
                mz[j * px + i].re = ms * v[2];
            }
        }
        fft2(mx, px, py, fx_f, fy_f, false);
        fft2(my, px, py, fx_f, fy_f, false);
        fft2(mz, px, py, fx_f, fy_f, false);
#pragma omp parallel for schedule(static) num_threads(g_threads)
        for (int64_t idx = 0; idx < px * py; ++idx) {
            bx[idx] = cadd(cmul(kxx[idx], mx[idx]), cmul(kxy[idx], my[idx]));
            by[idx] = cadd(cmul(kxy[idx], mx[idx]), cmul(kyy[idx], my[idx]));
            bz[idx] = cmul(kzz[idx], mz[idx]);
        }
        fft2(bx, px, py, fx_i, fy_i, true);
        fft2(by, px, py, fx_i, fy_i, true);
        fft2(bz, px, py, fx_i, fy_i, true);
#pragma omp parallel for schedule(static) num_threads(g_threads)
        for (int64_t j = 0; j < ny; ++j) {
            for (int64_t i = 0; i < nx; ++i) {
                double* o = &b[(j * nx + i) * 3];
                int64_t src = j * px + i;
                o[0] += bx[src].re;
                o[1] += by[src].re;
                o[2] += bz[src].re;
            }
        }
    }
};

// ---------------------------------------------------------------------------
// Local field terms
// ---------------------------------------------------------------------------
inline void ghost_x(const double* m, double n_x, double eta, double dx, double* o) {
    // exchange.rs:8-20 / dmi.rs:19-34 / energy.rs:37-49
    double mx = m[0], my = m[1], mz = m[2];
    double dmx_dx = -eta * mz, dmy_dx = 0.0, dmz_dx = eta * mx;
    o[0] = mx + n_x * dx * dmx_dx;
    o[1] = my + n_x * dx * dmy_dx;
    o[2] = mz + n_x * dx * dmz_dx;
}
inline void ghost_y(const double* m, double n_y, double eta, double dy, double* o) {
    // exchange.rs:22-35 / dmi.rs:36-52 / energy.rs:51-64
    double mx = m[0], my = m[1], mz = m[2];
    double dmx_dy = 0.0, dmy_dy = -eta * mz, dmz_dy = eta * my;
    o[0] = mx + n_y * dy * dmx_dy;
    o[1] = my + n_y * dy * dmy_dy;
    o[2] = mz + n_y * dy * dmz_dy;
}
inline void cp3(const double* a, double* o) { o[0] = a[0]; o[1] = a[1]; o[2] = a[2]; }

void add_exchange(const orc_grid& g, const double* m, double* b, const orc_material& mat, const uint8_t* mask) {
    // exchange.rs:45-222
    int64_t nx = g.nx, ny = g.ny;
    if (nx == 0 || ny == 0) return;
    double a = mat.a_ex, ms = mat.ms;
    if (a == 0.0 || ms == 0.0) return;
    double dx2 = g.dx * g.dx, dy2 = g.dy * g.dy;
    double coeff = 2.0 * a / ms;
    bool has_eta = mat.has_dmi && mat.dmi != 0.0;
    double eta = has_eta ? mat.dmi / (2.0 * a) : 0.0;
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_par_local)
    for (int64_t j = 0; j < ny; ++j) {
        for (int64_t i = 0; i < nx; ++i) {
            int64_t ic = j * nx + i;
            if (mask && !mask[ic]) continue;
            const double* mij = &m[ic * 3];
            double mim[3], mip[3], mjm[3], mjp[3];
            // x neighbours
            if (nx == 1) cp3(mij, mim);
            else if (i == 0) { if (has_eta) ghost_x(mij, -1.0, eta, g.dx, mim); else cp3(mij, mim); }
            else {
                int64_t il = j * nx + i - 1;
                if (mask && !mask[il]) { if (has_eta) ghost_x(mij, -1.0, eta, g.dx, mim); else cp3(mij, mim); }
                else cp3(&m[il * 3], mim);
            }
            if (nx == 1) cp3(mij, mip);
            else if (i == nx - 1) { if (has_eta) ghost_x(mij, 1.0, eta, g.dx, mip); else cp3(mij, mip); }
            else {
                int64_t ir = j * nx + i + 1;
                if (mask && !mask[ir]) { if (has_eta) ghost_x(mij, 1.0, eta, g.dx, mip); else cp3(mij, mip); }
                else cp3(&m[ir * 3], mip);
            }
            // y neighbours
            if (ny == 1) cp3(mij, mjm);
            else if (j == 0) { if (has_eta) ghost_y(mij, -1.0, eta, g.dy, mjm); else cp3(mij, mjm); }
            else {
                int64_t id = (j - 1) * nx + i;
                if (mask && !mask[id]) { if (has_eta) ghost_y(mij, -1.0, eta, g.dy, mjm); else cp3(mij, mjm); }
                else cp3(&m[id * 3], mjm);
            }
            if (ny == 1) cp3(mij, mjp);
            else if (j == ny - 1) { if (has_eta) ghost_y(mij, 1.0, eta, g.dy, mjp); else cp3(mij, mjp); }
            else {
                int64_t iu = (j + 1) * nx + i;
                if (mask && !mask[iu]) { if (has_eta) ghost_y(mij, 1.0, eta, g.dy, mjp); else cp3(mij, mjp); }
                else cp3(&m[iu * 3], mjp);
            }
            for (int c = 0; c < 3; ++c) {
                double d2x = nx > 1 ? (mip[c] - 2.0 * mij[c] + mim[c]) / dx2 : 0.0;
                double d2y = ny > 1 ? (mjp[c] - 2.0 * mij[c] + mjm[c]) / dy2 : 0.0;
                b[ic * 3 + c] += coeff * (d2x + d2y);
            }
        }
    }
}

void add_anisotropy(int64_t n, const double* m, double* b, const orc_material& mat) {
    // anisotropy.rs:10-26
    if (mat.k_u == 0.0 || mat.ms == 0.0) return;
    double coeff = 2.0 * mat.k_u / mat.ms;
    const double* u = mat.easy_axis;
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_par_local)
    for (int64_t i = 0; i < n; ++i) {
        const double* mc = &m[i * 3];
        double mdotu = mc[0] * u[0] + mc[1] * u[1] + mc[2] * u[2];
        b[i * 3 + 0] += coeff * mdotu * u[0];
        b[i * 3 + 1] += coeff * mdotu * u[1];
        b[i * 3 + 2] += coeff * mdotu * u[2];
    }
}

void add_dmi(const orc_grid& g, const double* m, double* b, const orc_material& mat, const uint8_t* mask) {
    // dmi.rs:67-209
    if (!mat.has_dmi || mat.dmi == 0.0) return;
    double d = mat.dmi, ms = mat.ms, a = mat.a_ex;
    if (ms == 0.0 || a == 0.0) return;
    int64_t nx = g.nx, ny = g.ny;
    if (nx == 0 || ny == 0) return;
    double dx = g.dx, dy = g.dy;
    double pref = 2.0 * d / ms;
    double eta = d / (2.0 * a);
    auto inside = [&](int64_t idx) { return mask ? mask[idx] != 0 : true; };
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_par_local)
    for (int64_t j = 0; j < ny; ++j) {
        for (int64_t i = 0; i < nx; ++i) {
            int64_t ic = j * nx + i;
            if (!inside(ic)) continue;
            const double* mij = &m[ic * 3];
            double mim[3], mip[3], mjm[3], mjp[3];
            if (nx == 1) { cp3(mij, mim); cp3(mij, mip); }
            else {
                if (i == 0) ghost_x(mij, -1.0, eta, dx, mim);
                else { int64_t il = ic - 1; if (inside(il)) cp3(&m[il * 3], mim); else cp3(mij, mim); }
                if (i == nx - 1) ghost_x(mij, 1.0, eta, dx, mip);
                else { int64_t ir = ic + 1; if (inside(ir)) cp3(&m[ir * 3], mip); else cp3(mij, mip); }
            }
            if (ny == 1) { cp3(mij, mjm); cp3(mij, mjp); }
            else {
                if (j == 0) ghost_y(mij, -1.0, eta, dy, mjm);
                else { int64_t id = ic - nx; if (inside(id)) cp3(&m[id * 3], mjm); else cp3(mij, mjm); }
                if (j == ny - 1) ghost_y(mij, 1.0, eta, dy, mjp);
                else { int64_t iu = ic + nx; if (inside(iu)) cp3(&m[iu * 3], mjp); else cp3(mij, mjp); }
            }
            double dmz_dx = nx > 1 ? (mip[2] - mim[2]) / (2.0 * dx) : 0.0;
            double dmz_dy = ny > 1 ? (mjp[2] - mjm[2]) / (2.0 * dy) : 0.0;
            double dmx_dx = nx > 1 ? (mip[0] - mim[0]) / (2.0 * dx) : 0.0;
            double dmy_dy = ny > 1 ? (mjp[1] - mjm[1]) / (2.0 * dy) : 0.0;
            b[ic * 3 + 0] += pref * dmz_dx;
            b[ic * 3 + 1] += pref * dmz_dy;
            b[ic * 3 + 2] += -pref * (dmx_dx + dmy_dy);
        }
    }
}

// llg.rs:20-32
inline void llg_rhs(const double* m, const double* b, double gamma, double alpha, double* o) {
    double denom = 1.0 + alpha * alpha;
    double pref = -gamma / denom;
    double mxb[3], mxmxb[3];
    vcross(m, b, mxb);
    vcross(m, mxb, mxmxb);
    o[0] = pref * (mxb[0] + alpha * mxmxb[0]);
    o[1] = pref * (mxb[1] + alpha * mxmxb[1]);
    o[2] = pref * (mxb[2] + alpha * mxmxb[2]);
}
// llg.rs:38-50
inline void llg_rhs_relax(const double* m, const double* b, double gamma, double alpha, double* o) {
    double denom = 1.0 + alpha * alpha;
    double pref = -gamma * alpha / denom;
    double mxb[3], mxmxb[3];
    vcross(m, b, mxb);
    vcross(m, mxb, mxmxb);
    o[0] = pref * mxmxb[0];
    o[1] = pref * mxmxb[1];
    o[2] = pref * mxmxb[2];
}

}  // namespace

// ---------------------------------------------------------------------------
// Solver handle: grid + material + demag operator + RK scratch state.
// ---------------------------------------------------------------------------
struct orc_solver {
    orc_grid g;
    orc_material mat;
    std::vector<uint8_t> mask;  // empty = no geometry mask
    std::unique_ptr<Demag2D> demag;
    int64_t n;
    // RK45 scratch (llg.rs:126-156)
    std::vector<double> m45[8], b45[8], k45[8];
    bool fsal45 = false;
    int last_mask45 = -1;
    double last_bext45[3];
    // RK23 scratch (llg.rs:196-222)
    std::vector<double> m23[5], b23[5], k23[5];
    bool last_b_eff_valid = false;
    int last_mask23 = -1;
    double last_bext23[3];

    const uint8_t* maskp() const { return mask.empty() ? nullptr : mask.data(); }
    Demag2D& op() {
        if (!demag) demag.reset(new Demag2D(g));
        return *demag;
    }
};

namespace {

// build_h_eff_masked (mod.rs:48-75) and, with a geometry mask, the
// build_h_eff_masked_geom variant (mod.rs:78-101).
void build_h_eff(orc_solver* s, const double* m, const double* bext, int fmask, double* b) {
    int64_t n = s->n;
    const uint8_t* mask = s->maskp();
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_par_local)
    for (int64_t i = 0; i < n; ++i) {
        b[i * 3 + 0] = 0.0 + bext[0];
        b[i * 3 + 1] = 0.0 + bext[1];
        b[i * 3 + 2] = 0.0 + bext[2];
    }
    add_exchange(s->g, m, b, s->mat, mask);
    add_anisotropy(n, m, b, s->mat);
    bool include_dmi = fmask == ORC_EXCH_ANIS_DMI || fmask == ORC_FULL;
    if (include_dmi && s->mat.has_dmi) add_dmi(s->g, m, b, s->mat, mask);
    if (fmask == ORC_FULL && s->mat.demag) s->op().add_field(m, b, s->mat.ms);
}

// Stage state m_s = normalize(v).  Geometry-mask extension: vacuum cells stay
// at m = 0 (the reference would map them to +z through vec3::normalize).
inline void stage_normalize(const orc_solver* s, int64_t i, const double* v, double* o) {
    if (!s->mask.empty() && !s->mask[i]) { o[0] = o[1] = o[2] = 0.0; return; }
    vnormalize(v, o);
}

}  // namespace

extern "C" {

void orc_set_threads(int n) { g_threads = n < 1 ? 1 : n; }
int orc_get_threads(void) { return g_threads; }
void orc_set_parallel_local(int on) { g_par_local = on != 0; }
int orc_get_parallel_local(void) { return g_par_local ? 1 : 0; }

orc_solver* orc_solver_create(const orc_grid* g, const orc_material* mat, const uint8_t* geom_mask) {
    orc_solver* s = new orc_solver();
    s->g = *g;
    s->mat = *mat;
    s->n = g->nx * g->ny;
    if (geom_mask) s->mask.assign(geom_mask, geom_mask + s->n);
    for (int i = 0; i < 8; ++i) {
        s->m45[i].assign(s->n * 3, 0.0);
        s->b45[i].assign(s->n * 3, 0.0);
        s->k45[i].assign(s->n * 3, 0.0);
    }
    for (int i = 0; i < 5; ++i) {
        s->m23[i].assign(s->n * 3, 0.0);
        s->b23[i].assign(s->n * 3, 0.0);
        s->k23[i].assign(s->n * 3, 0.0);
    }
    return s;
}

void orc_solver_destroy(orc_solver* s) { delete s; }

void orc_solver_invalidate(orc_solver* s) {
    // RK23Scratch::invalidate_last_b_eff (llg.rs:264-268) plus the RK45 FSAL flag
    s->last_b_eff_valid = false;
    s->last_mask23 = -1;
    s->fsal45 = false;
    s->last_mask45 = -1;
}

void orc_build_h_eff(orc_solver* s, const double* m, const double b_ext[3], int field_mask, double* b_out) {
    build_h_eff(s, m, b_ext, field_mask, b_out);
}

void orc_demag_field(orc_solver* s, const double* m, double* b_out) {
    // compute_demag_field (demag.rs:57-64 -> demag_fft_uniform.rs:146-186)
    std::fill(b_out, b_out + s->n * 3, 0.0);
    if (!s->mat.demag) return;
    s->op().add_field(m, b_out, s->mat.ms);
}

void orc_step_rk45(orc_solver* s, double* m, orc_params* p, int fmask, double max_err, double headroom,
                   double dt_min, double dt_max, double* eps_out, int* accepted_out, double* dt_used_out) {
    // step_llg_rk45_recompute_field_masked_adaptive, llg.rs:795-1026
    const int64_t n = s->n;
    const double gamma = p->gamma, alpha = p->alpha, dt0 = p->dt;
    const double A21 = 1.0 / 5.0;
    const double A31 = 3.0 / 40.0, A32 = 9.0 / 40.0;
    const double A41 = 44.0 / 45.0, A42 = -56.0 / 15.0, A43 = 32.0 / 9.0;
    const double A51 = 19372.0 / 6561.0, A52 = -25360.0 / 2187.0, A53 = 64448.0 / 6561.0, A54 = -212.0 / 729.0;
    const double A61 = 9017.0 / 3168.0, A62 = -355.0 / 33.0, A63 = 46732.0 / 5247.0, A64 = 49.0 / 176.0,
                 A65 = -5103.0 / 18656.0;
    const double B1 = 35.0 / 384.0, B3 = 500.0 / 1113.0, B4 = 125.0 / 192.0, B5 = -2187.0 / 6784.0,
                 B6 = 11.0 / 84.0;
    const double BH1 = 5179.0 / 57600.0, BH3 = 7571.0 / 16695.0, BH4 = 393.0 / 640.0,
                 BH5 = -92097.0 / 339200.0, BH6 = 187.0 / 2100.0, BH7 = 1.0 / 40.0;
    auto& K = s->k45;
    auto& Bf = s->b45;
    auto& M = s->m45;
    bool fsal_ok = s->fsal45 && s->last_mask45 == fmask && s->last_bext45[0] == p->b_ext[0] &&
                   s->last_bext45[1] == p->b_ext[1] && s->last_bext45[2] == p->b_ext[2];
    if (fsal_ok) {
        Bf[1] = Bf[7];
        K[1] = K[7];
    } else {
        build_h_eff(s, m, p->b_ext, fmask, Bf[1].data());
    #pragma omp parallel for schedule(static) num_threads(g_threads) if (g_par_local)
        for (int64_t i = 0; i < n; ++i) llg_rhs(&m[i * 3], &Bf[1][i * 3], gamma, alpha, &K[1][i * 3]);
    }
    // stage s: m_s = normalize(m + sum_j (dt0*a_sj) k_j), then B_s and k_s
    auto stage = [&](int st, int nk, const int* ks, const double* as) {
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_par_local)
        for (int64_t i = 0; i < n; ++i) {
            double v[3] = {m[i * 3], m[i * 3 + 1], m[i * 3 + 2]};
            for (int q = 0; q < nk; ++q) {
                double sc = dt0 * as[q];
                const double* kk = &K[ks[q]][i * 3];
                v[0] = v[0] + sc * kk[0];
                v[1] = v[1] + sc * kk[1];
                v[2] = v[2] + sc * kk[2];
            }
            stage_normalize(s, i, v, &M[st][i * 3]);
        }
        build_h_eff(s, M[st].data(), p->b_ext, fmask, Bf[st].data());
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_par_local)
        for (int64_t i = 0; i < n; ++i) llg_rhs(&M[st][i * 3], &Bf[st][i * 3], gamma, alpha, &K[st][i * 3]);
    };
    {
        int ks[] = {1};
        double as[] = {A21};
        stage(2, 1, ks, as);
    }
    {
        int ks[] = {1, 2};
        double as[] = {A31, A32};
        stage(3, 2, ks, as);
    }
    {
        int ks[] = {1, 2, 3};
        double as[] = {A41, A42, A43};
        stage(4, 3, ks, as);
    }
    {
        int ks[] = {1, 2, 3, 4};
        double as[] = {A51, A52, A53, A54};
        stage(5, 4, ks, as);
    }
    {
        int ks[] = {1, 2, 3, 4, 5};
        double as[] = {A61, A62, A63, A64, A65};
        stage(6, 5, ks, as);
    }
    {
        int ks[] = {1, 3, 4, 5, 6};
        double as[] = {B1, B3, B4, B5, B6};
        stage(7, 5, ks, as);
    }
    double err_inf = 0.0;
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_par_local) reduction(max : err_inf)
    for (int64_t i = 0; i < n; ++i) {
        double d = 0.0;
        for (int c = 0; c < 3; ++c) {
            double th = B1 * K[1][i * 3 + c] + B3 * K[3][i * 3 + c] + B4 * K[4][i * 3 + c] +
                        B5 * K[5][i * 3 + c] + B6 * K[6][i * 3 + c];
            double tl = BH1 * K[1][i * 3 + c] + BH3 * K[3][i * 3 + c] + BH4 * K[4][i * 3 + c] +
                        BH5 * K[5][i * 3 + c] + BH6 * K[6][i * 3 + c] + BH7 * K[7][i * 3 + c];
            double e = std::fabs(th - tl);
            d = c == 0 ? e : std::max(d, e);
        }
        if (d > err_inf) err_inf = d;
    }
    double eps = err_inf * dt0;
    double dt_next = eps > 0.0 ? dt0 * headroom * std::pow(max_err / eps, 0.2) : dt0 * 2.0;
    dt_next = std::min(std::max(dt_next, dt_min), dt_max);
    bool accept = (eps <= max_err) || (dt0 <= dt_min * 1.0000000001);
    if (accept) {
        std::memcpy(m, M[7].data(), sizeof(double) * n * 3);
        s->fsal45 = true;
        s->last_mask45 = fmask;
        std::memcpy(s->last_bext45, p->b_ext, sizeof(double) * 3);
    } else {
        s->fsal45 = false;
        s->last_mask45 = -1;
    }
    p->dt = dt_next;
    *eps_out = eps;
    *accepted_out = accept ? 1 : 0;
    *dt_used_out = dt0;
}

void orc_step_rk23_relax(orc_solver* s, double* m, orc_params* p, int fmask, double max_err, double headroom,
                         double dt_min, double dt_max, double* eps_out, int* accepted_out, double* dt_used_out) {
    // step_llg_rk23_recompute_field_masked_relax_adaptive, llg.rs:278-436
    const int64_t n = s->n;
    const double gamma = p->gamma, alpha = p->alpha, dt0 = p->dt;
    const double A21 = 1.0 / 2.0, A32 = 3.0 / 4.0;
    const double B1 = 2.0 / 9.0, B2 = 1.0 / 3.0, B3 = 4.0 / 9.0;
    const double BH1 = 7.0 / 24.0, BH2 = 1.0 / 4.0, BH3 = 1.0 / 3.0, BH4 = 1.0 / 8.0;
    auto& K = s->k23;
    auto& Bf = s->b23;
    auto& M = s->m23;
    bool fsal_ok = s->last_b_eff_valid && s->last_mask23 == fmask && s->last_bext23[0] == p->b_ext[0] &&
                   s->last_bext23[1] == p->b_ext[1] && s->last_bext23[2] == p->b_ext[2];
    if (fsal_ok) {
        Bf[1] = Bf[4];
        K[1] = K[4];
    } else {
        build_h_eff(s, m, p->b_ext, fmask, Bf[1].data());
        for (int64_t i = 0; i < n; ++i) llg_rhs_relax(&m[i * 3], &Bf[1][i * 3], gamma, alpha, &K[1][i * 3]);
    }
    for (int64_t i = 0; i < n; ++i) {
        double sc = dt0 * A21;
        double v[3] = {m[i * 3] + sc * K[1][i * 3], m[i * 3 + 1] + sc * K[1][i * 3 + 1],
                       m[i * 3 + 2] + sc * K[1][i * 3 + 2]};
        stage_normalize(s, i, v, &M[2][i * 3]);
    }
    build_h_eff(s, M[2].data(), p->b_ext, fmask, Bf[2].data());
    for (int64_t i = 0; i < n; ++i) llg_rhs_relax(&M[2][i * 3], &Bf[2][i * 3], gamma, alpha, &K[2][i * 3]);
    for (int64_t i = 0; i < n; ++i) {
        double sc = dt0 * A32;
        double v[3] = {m[i * 3] + sc * K[2][i * 3], m[i * 3 + 1] + sc * K[2][i * 3 + 1],
                       m[i * 3 + 2] + sc * K[2][i * 3 + 2]};
        stage_normalize(s, i, v, &M[3][i * 3]);
    }
    build_h_eff(s, M[3].data(), p->b_ext, fmask, Bf[3].data());
    for (int64_t i = 0; i < n; ++i) llg_rhs_relax(&M[3][i * 3], &Bf[3][i * 3], gamma, alpha, &K[3][i * 3]);
    for (int64_t i = 0; i < n; ++i) {
        double v[3];
        for (int c = 0; c < 3; ++c) {
            double x = m[i * 3 + c];
            x = x + (dt0 * B1) * K[1][i * 3 + c];
            x = x + (dt0 * B2) * K[2][i * 3 + c];
            x = x + (dt0 * B3) * K[3][i * 3 + c];
            v[c] = x;
        }
        stage_normalize(s, i, v, &M[4][i * 3]);
    }
    build_h_eff(s, M[4].data(), p->b_ext, fmask, Bf[4].data());
    for (int64_t i = 0; i < n; ++i) llg_rhs_relax(&M[4][i * 3], &Bf[4][i * 3], gamma, alpha, &K[4][i * 3]);
    for (int64_t i = 0; i < n; ++i) {
        double v[3];
        for (int c = 0; c < 3; ++c) {
            double x = m[i * 3 + c];
            x = x + (dt0 * BH1) * K[1][i * 3 + c];
            x = x + (dt0 * BH2) * K[2][i * 3 + c];
            x = x + (dt0 * BH3) * K[3][i * 3 + c];
            x = x + (dt0 * BH4) * K[4][i * 3 + c];
            v[c] = x;
        }
        stage_normalize(s, i, v, &M[2][i * 3]);
    }
    double err_inf = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double* a = &M[4][i * 3];
        const double* b = &M[2][i * 3];
        double d = std::max(std::max(std::fabs(a[0] - b[0]), std::fabs(a[1] - b[1])), std::fabs(a[2] - b[2]));
        if (d > err_inf) err_inf = d;
    }
    double eps = err_inf;
    double dt_next = eps > 0.0 ? dt0 * headroom * std::pow(max_err / eps, 1.0 / 3.0) : dt0 * 2.0;
    dt_next = std::min(std::max(dt_next, dt_min), dt_max);
    bool accept = (eps <= max_err) || (dt0 <= dt_min * 1.0000000001);
    if (accept) {
        std::memcpy(m, M[4].data(), sizeof(double) * n * 3);
        s->last_b_eff_valid = true;
        s->last_mask23 = fmask;
        std::memcpy(s->last_bext23, p->b_ext, sizeof(double) * 3);
    } else {
        s->last_b_eff_valid = false;
        s->last_mask23 = -1;
    }
    p->dt = dt_next;
    *eps_out = eps;
    *accepted_out = accept ? 1 : 0;
    *dt_used_out = dt0;
}

double orc_torque_metric(int64_t n, const double* m, const double* b, int metric) {
    // torque_metric_from_field, relax.rs:144-189
    double nf = (double)n;
    double acc = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        double t[3];
        vcross(&m[i * 3], &b[i * 3], t);
        double mag2 = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
        if (metric == ORC_TORQUE_MAX) {
            double mag = std::sqrt(mag2);
            if (mag > acc) acc = mag;
        } else if (metric == ORC_TORQUE_MEAN) {
            acc += std::sqrt(mag2);
        } else {
            acc += mag2;
        }
    }
    if (metric == ORC_TORQUE_MAX) return acc;
    if (metric == ORC_TORQUE_MEAN) return acc / std::max(nf, 1.0);
    if (metric == ORC_TORQUE_RMS) return std::sqrt(acc / std::max(nf, 1.0));
    return acc / std::max(nf, 1.0);
}

void orc_energy_breakdown(orc_solver* s, const double* m, const double b_ext[3], orc_energy* out) {
    // compute_energy_geom, energy.rs:80-285
    const orc_grid& g = s->g;
    const orc_material& mat = s->mat;
    const uint8_t* mask = s->maskp();
    int64_t nx = g.nx, ny = g.ny;
    double dx = g.dx, dy = g.dy;
    double v = g.dx * g.dy * g.dz;
    double aex = mat.a_ex, ku = mat.k_u, ms = mat.ms;
    const double* u = mat.easy_axis;
    double bx = b_ext[0], by = b_ext[1], bz = b_ext[2];
    double e_ex = 0.0, e_an = 0.0, e_zee = 0.0, e_dmi = 0.0, e_demag = 0.0;
    bool has_dmi = mat.has_dmi && mat.dmi != 0.0 && aex != 0.0;
    double d = has_dmi ? mat.dmi : 0.0;
    double eta = has_dmi ? d / (2.0 * aex) : 0.0;
    std::vector<double> bd;
    if (mat.demag) {
        bd.assign(s->n * 3, 0.0);
        s->op().add_field(m, bd.data(), ms);
    }
    auto inside = [&](int64_t idx) { return mask ? mask[idx] != 0 : true; };
    for (int64_t j = 0; j < ny; ++j) {
        for (int64_t i = 0; i < nx; ++i) {
            int64_t idx = j * nx + i;
            if (!inside(idx)) continue;
            const double* mij = &m[idx * 3];
            double mx = mij[0], my = mij[1], mz = mij[2];
            if (aex != 0.0) {
                if (i + 1 < nx) {
                    int64_t ir = idx + 1;
                    if (inside(ir)) {
                        const double* mp = &m[ir * 3];
                        double d0 = mp[0] - mx, d1 = mp[1] - my, d2 = mp[2] - mz;
                        double sq = d0 * d0 + d1 * d1 + d2 * d2;
                        e_ex += aex * (sq / (dx * dx)) * v;
                    }
                }
                if (j + 1 < ny) {
                    int64_t iu = idx + nx;
                    if (inside(iu)) {
                        const double* mp = &m[iu * 3];
                        double d0 = mp[0] - mx, d1 = mp[1] - my, d2 = mp[2] - mz;
                        double sq = d0 * d0 + d1 * d1 + d2 * d2;
                        e_ex += aex * (sq / (dy * dy)) * v;
                    }
                }
            }
            if (ku != 0.0) {
                double mdotu = mx * u[0] + my * u[1] + mz * u[2];
                e_an += ku * (1.0 - mdotu * mdotu) * v;
            }
            if (ms != 0.0) {
                double mdotb = mx * bx + my * by + mz * bz;
                e_zee -= ms * mdotb * v;
            }
            if (has_dmi && ms != 0.0) {
                double pref = 2.0 * d / ms;
                double mim[3], mip[3], mjm[3], mjp[3];
                if (nx == 1) { cp3(mij, mim); cp3(mij, mip); }
                else {
                    if (i == 0) ghost_x(mij, -1.0, eta, dx, mim);
                    else if (inside(idx - 1)) cp3(&m[(idx - 1) * 3], mim);
                    else ghost_x(mij, -1.0, eta, dx, mim);
                    if (i == nx - 1) ghost_x(mij, 1.0, eta, dx, mip);
                    else if (inside(idx + 1)) cp3(&m[(idx + 1) * 3], mip);
                    else ghost_x(mij, 1.0, eta, dx, mip);
                }
                if (ny == 1) { cp3(mij, mjm); cp3(mij, mjp); }
                else {
                    if (j == 0) ghost_y(mij, -1.0, eta, dy, mjm);
                    else if (inside(idx - nx)) cp3(&m[(idx - nx) * 3], mjm);
                    else ghost_y(mij, -1.0, eta, dy, mjm);
                    if (j == ny - 1) ghost_y(mij, 1.0, eta, dy, mjp);
                    else if (inside(idx + nx)) cp3(&m[(idx + nx) * 3], mjp);
                    else ghost_y(mij, 1.0, eta, dy, mjp);
                }
                double dmz_dx = nx > 1 ? (mip[2] - mim[2]) / (2.0 * dx) : 0.0;
                double dmz_dy = ny > 1 ? (mjp[2] - mjm[2]) / (2.0 * dy) : 0.0;
                double dmx_dx = nx > 1 ? (mip[0] - mim[0]) / (2.0 * dx) : 0.0;
                double dmy_dy = ny > 1 ? (mjp[1] - mjm[1]) / (2.0 * dy) : 0.0;
                double bdx = pref * dmz_dx, bdy = pref * dmz_dy, bdz = -pref * (dmx_dx + dmy_dy);
                double mdotb = mx * bdx + my * bdy + mz * bdz;
                e_dmi += -0.5 * ms * mdotb * v;
            }
            if (mat.demag && ms != 0.0) {
                const double* b = &bd[idx * 3];
                double mdotb = mx * b[0] + my * b[1] + mz * b[2];
                e_demag += -0.5 * ms * mdotb * v;
            }
        }
    }
    out->exchange = e_ex;
    out->anisotropy = e_an;
    out->zeeman = e_zee;
    out->dmi = e_dmi;
    out->demag = e_demag;
}

void orc_default_relax_settings(orc_relax_settings* st) {
    // impl Default for RelaxSettings, relax.rs:107-141
    std::memset(st, 0, sizeof(*st));
    st->max_err = 1e-5;
    st->headroom = 0.8;
    st->dt_min = 1e-18;
    st->dt_max = 1e-11;
    st->phase1_enabled = 1;
    st->phase2_enabled = 1;
    st->energy_stride = 3;
    st->rel_energy_tol = 1e-12;
    st->torque_metric = ORC_TORQUE_MAX;
    st->has_torque_threshold = 1;
    st->torque_threshold = 1e-4;
    st->torque_check_stride = 1;
    st->torque_plateau_rel = 1e-3;
    st->torque_plateau_abs = 0.0;
    st->torque_plateau_checks = 0;
    st->torque_plateau_min_checks = 5;
    st->tighten_factor = 0.70710678118654752440;  // FRAC_1_SQRT_2
    st->tighten_floor = 1e-9;
    st->max_accepted_steps = 2000000;
}

void orc_relax(orc_solver* s, double* m, orc_params* p, int fmask, orc_relax_settings* st,
               orc_relax_report* rep) {
    // relax_with_report, relax.rs:334-768
    const int64_t n = s->n;
    const bool phase1 = st->phase1_enabled != 0, phase2 = st->phase2_enabled != 0;
    const int64_t energy_stride = std::max<int64_t>(st->energy_stride, 1);
    const int metric = st->torque_metric;
    const bool has_thr = st->has_torque_threshold != 0;
    const double thr = st->torque_threshold;
    const int64_t check_stride = std::max<int64_t>(st->torque_check_stride, 1);
    const double plateau_rel = st->torque_plateau_rel, plateau_abs = st->torque_plateau_abs;
    const int64_t plateau_checks = st->torque_plateau_checks;
    const int64_t plateau_min_checks = std::max<int64_t>(st->torque_plateau_min_checks, 1);
    const double tighten_factor = st->tighten_factor, tighten_floor = st->tighten_floor;
    const int64_t max_acc = st->max_accepted_steps;
    double max_err = st->max_err;
    p->dt = std::min(std::max(p->dt, st->dt_min), st->dt_max);
    orc_solver_invalidate(s);
    int64_t accepted = 0, rejected = 0, checks = 0, rebuilds = 0;
    int last_stage = -1;
    bool has_ft = false, has_ftm = false;
    double ft = 0.0, ftm = 0.0;
    std::vector<double> bscratch(n * 3);
    double eps;
    int acc;
    double dtu;

    auto finish = [&](int reason) {
        st->max_err = max_err;
        rep->accepted_steps = accepted;
        rep->rejected_steps = rejected;
        rep->torque_checks = checks;
        rep->torque_field_rebuilds = rebuilds;
        rep->stop_reason = reason;
        rep->last_stage_stop = last_stage;
        rep->has_final_torque = has_ft;
        rep->final_torque = ft;
        rep->has_final_torque_max = has_ftm;
        rep->final_torque_max = ftm;
        rep->final_max_err = max_err;
        rep->final_dt = p->dt;
    };
    // advance_accepted, relax.rs:247-272
    auto advance = [&](int64_t n_accept) -> bool {
        int64_t target = accepted + std::max<int64_t>(n_accept, 1);
        while (accepted < target) {
            if (accepted >= max_acc) return false;
            orc_step_rk23_relax(s, m, p, fmask, max_err, st->headroom, st->dt_min, st->dt_max, &eps, &acc, &dtu);
            if (acc) ++accepted; else ++rejected;
        }
        return true;
    };
    // torque_now, relax.rs:206-227
    auto torque_now = [&](int met) -> double {
        ++checks;
        if (s->last_b_eff_valid) return orc_torque_metric(n, m, s->b23[4].data(), met);
        ++rebuilds;
        build_h_eff(s, m, p->b_ext, fmask, bscratch.data());
        return orc_torque_metric(n, m, bscratch.data(), met);
    };
    auto total_energy = [&]() {
        orc_energy e;
        orc_energy_breakdown(s, m, p->b_ext, &e);
        return e.exchange + e.anisotropy + e.zeeman + e.dmi + e.demag;
    };

    if (phase1) {
        double e0 = total_energy();
        for (;;) {
            if (!advance(energy_stride)) { finish(0); return; }
            double e1 = total_energy();
            double tol = st->rel_energy_tol * std::max(std::fabs(e0), 1e-30);
            if (e1 < e0 - tol) { e0 = e1; continue; }
            break;
        }
    }
    if (!phase2) {
        has_ft = has_ftm = false;
        finish(1);
        return;
    }
    bool plateau_enabled = !has_thr && plateau_checks > 0;
    int64_t need_fails = std::max<int64_t>(plateau_checks, 1);
    for (;;) {
        double t_prev = torque_now(metric);
        bool f32mode = plateau_enabled && metric == ORC_TORQUE_MEANSQ && plateau_rel == 0.0 &&
                       plateau_abs == 0.0 && plateau_checks == 1 && plateau_min_checks == 1;
        double nf = (double)n;
        float t_prev_f32 = f32mode ? (float)(t_prev * nf) : (float)t_prev;
        int64_t fails = 0, comparisons = 0;
        for (;;) {
            if (has_thr && t_prev <= thr) { last_stage = 0; break; }
            if (plateau_enabled && fails >= need_fails) { last_stage = 1; break; }
            if (accepted >= max_acc) {
                last_stage = 2; has_ft = true; ft = t_prev;
                finish(0);
                return;
            }
            if (!advance(check_stride)) {
                last_stage = 2; has_ft = true; ft = t_prev;
                finish(0);
                return;
            }
            double t_new = torque_now(metric);
            if (plateau_enabled) {
                ++comparisons;
                if (comparisons < plateau_min_checks) fails = 0;
                else if (f32mode) {
                    float t_new_f32 = (float)(t_new * nf);
                    bool improved = t_new_f32 < t_prev_f32;
                    t_prev_f32 = t_new_f32;
                    fails = improved ? 0 : fails + 1;
                } else {
                    double need_rel = plateau_rel * std::max(std::fabs(t_prev), 1e-30);
                    double need = std::max(need_rel, plateau_abs);
                    bool improved = (t_prev - t_new) > need;
                    fails = improved ? 0 : fails + 1;
                }
            }
            t_prev = t_new;
        }
        has_ft = true;
        ft = t_prev;
        if (max_err <= tighten_floor) break;
        max_err *= tighten_factor;
        if (max_err < tighten_floor) max_err = tighten_floor;
    }
    ftm = torque_now(ORC_TORQUE_MAX);
    has_ftm = true;
    bool has_gate = st->has_final_torque_gate != 0, has_gmax = st->has_final_torque_gate_max != 0;
    bool gate_enabled = (has_gate || has_gmax) && st->gate_max_extra_accepted_steps > 0;
    if (gate_enabled) {
        int64_t start_acc = accepted;
        double last_t = has_ft ? ft : INFINITY;
        int64_t gfails = 0;
        for (;;) {
            // gates_ok, relax.rs:275-332
            double t_metric = torque_now(metric);
            bool need_max = has_gmax || metric == ORC_TORQUE_MAX;
            double t_max = NAN;
            if (need_max) t_max = metric == ORC_TORQUE_MAX ? t_metric : torque_now(ORC_TORQUE_MAX);
            bool ok_metric = !has_gate || t_metric <= st->final_torque_gate;
            bool ok_max = !has_gmax || t_max <= st->final_torque_gate_max;
            has_ft = true; ft = t_metric;
            if (std::isfinite(t_max)) { has_ftm = true; ftm = t_max; }
            if (ok_metric && ok_max) break;
            int64_t extra = accepted - start_acc;
            if (extra >= st->gate_max_extra_accepted_steps) { finish(3); return; }
            if (st->gate_plateau_fails > 0) {
                double need_rel = plateau_rel * std::max(std::fabs(last_t), 1e-30);
                double need = std::max(need_rel, plateau_abs);
                bool improved = (last_t - t_metric) > need;
                gfails = improved ? 0 : gfails + 1;
                if (gfails >= st->gate_plateau_fails) { finish(3); return; }
                last_t = t_metric;
            }
            if (!advance(check_stride)) { last_stage = 2; finish(0); return; }
        }
    }
    finish(2);
}

void orc_default_minimize_settings(orc_minimize_settings* st) {
    // impl Default for MinimizeSettings, minimize.rs:65-92
    std::memset(st, 0, sizeof(*st));
    st->torque_threshold = 5e-4;
    st->max_iters = 20000;
    st->lambda0 = 2e-2;
    st->lambda_min = 1e-5;
    st->lambda_max = 5e-2;
    st->grow = 1.05;
    st->shrink = 0.8;
    st->stall_iters = 5000;
    st->stall_rel = 5e-4;
    st->min_iters_before_stall = 500;
    st->has_dm_stop = 1;
    st->dm_stop = 1e-6;
    st->dm_samples = 10;
    st->has_dm_torque_gate = 1;
    st->dm_torque_gate = 2e-3;
    st->has_dm_torque_gate_max = 1;
    st->dm_torque_gate_max = 5e-3;
    st->dm_min_iters = 50;
}

void orc_minimize(orc_solver* s, double* m, const orc_params* p, int fmask, const orc_minimize_settings* st,
                  orc_minimize_report* rep) {
    // minimize_damping_only, minimize.rs:107-369 (the sequential per-cell pass, :216-256)
    const int64_t n = s->n;
    std::vector<double> b(n * 3);
    double lambda = st->lambda0;
    double t_prev_mean = INFINITY;
    int64_t stall_count = 0;
    std::deque<double> dm_hist;
    double last_max_dm = INFINITY, last_tmax = INFINITY, last_tmean = INFINITY;
    const size_t samples = (size_t)std::max<int64_t>(st->dm_samples, 1);
    auto report = [&](int64_t iters, double ft, bool conv, bool stalled, double mdm, bool dmc, double tm) {
        rep->iters = iters;
        rep->converged = conv ? 1 : 0;
        rep->stalled = stalled ? 1 : 0;
        rep->dm_converged = dmc ? 1 : 0;
        rep->final_torque = ft;
        rep->final_max_dm = mdm;
        rep->final_tmean = tm;
        rep->final_lambda = lambda;
    };
    for (int64_t it = 0; it < st->max_iters; ++it) {
        build_h_eff(s, m, p->b_ext, fmask, b.data());
        double tmax = 0.0, tsum = 0.0, max_dm = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            const double* m0 = &m[i * 3];
            double t[3], d[3];
            vcross(m0, &b[i * 3], t);
            const double tmag = std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
            tsum += tmag;
            if (tmag > tmax) tmax = tmag;
            vcross(t, m0, d);  // damping-only direction (m x B) x m
            double x = m0[0] + lambda * d[0];
            double y = m0[1] + lambda * d[1];
            double z = m0[2] + lambda * d[2];
            const double n2 = x * x + y * y + z * z;
            if (n2 > 0.0) {
                const double inv = 1.0 / std::sqrt(n2);
                x *= inv;
                y *= inv;
                z *= inv;
            }
            const double ddx = x - m0[0], ddy = y - m0[1], ddz = z - m0[2];
            const double dm = std::sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
            if (dm > max_dm) max_dm = dm;
            m[i * 3] = x;
            m[i * 3 + 1] = y;
            m[i * 3 + 2] = z;
        }
        const double tmean = tsum / std::max((double)n, 1.0);
        last_tmean = tmean;
        if (tmax < st->torque_threshold) {
            report(it + 1, tmax, true, false, max_dm, false, tmean);
            return;
        }
        last_max_dm = max_dm;
        last_tmax = tmax;
        if (st->has_dm_stop && it + 1 >= st->dm_min_iters) {
            dm_hist.push_back(max_dm);
            while (dm_hist.size() > samples) dm_hist.pop_front();
            bool all = dm_hist.size() == samples;
            for (double v : dm_hist) all = all && v < st->dm_stop;
            if (all) {
                const bool mean_ok = !st->has_dm_torque_gate || tmean <= st->dm_torque_gate;
                const bool max_ok = !st->has_dm_torque_gate_max || tmax <= st->dm_torque_gate_max;
                report(it + 1, tmax, mean_ok && max_ok, false, max_dm, true, tmean);
                return;
            }
        }
        if (tmean < t_prev_mean) lambda = std::fmin(lambda * st->grow, st->lambda_max);
        else lambda = std::fmax(lambda * st->shrink, st->lambda_min);
        if (it + 1 >= st->min_iters_before_stall && std::isfinite(t_prev_mean)) {
            const double good = t_prev_mean - tmean;
            const double need = st->stall_rel * std::fmax(std::fabs(t_prev_mean), 1e-30);
            if (good <= need) stall_count += 1;
            else stall_count = 0;
        }
        if (stall_count >= st->stall_iters) {
            report(it + 1, tmax, false, true, last_max_dm, false, tmean);
            return;
        }
        t_prev_mean = tmean;
    }
    report(std::max<int64_t>(st->max_iters, 0), last_tmax, false, false, last_max_dm, false, last_tmean);
}

// ---------------------------------------------------------------------------------------------
// AMR consumers of the uniform FFT demag

int64_t orc_validated_ratio(int64_t nx, int64_t ny, int64_t ratio) {
    // validated_ratio, coarse_fft_demag.rs:118-150 (warnings omitted)
    if (ratio <= 1) return 1;
    if (nx % ratio != 0 || ny % ratio != 0) return 1;
    if (nx / ratio < 4 || ny / ratio < 4) return 1;
    return ratio;
}

static inline int64_t clamp_idx(int64_t i, int64_t n) { return i < 0 ? 0 : (i >= n ? n - 1 : i); }

void orc_sample_bilinear(const orc_grid* g, const double* f, double x, double y, double out[3]) {
    // sample_bilinear, amr/interp.rs:28-72
    const int64_t nx = g->nx, ny = g->ny;
    if (nx == 0 || ny == 0) {
        out[0] = out[1] = out[2] = 0.0;
        return;
    }
    const double fx = x / g->dx - 0.5, fy = y / g->dy - 0.5;
    const double i0f = std::floor(fx), j0f = std::floor(fy);
    const double tx = fx - i0f, ty = fy - j0f;
    const int64_t i0 = clamp_idx((int64_t)i0f, nx), j0 = clamp_idx((int64_t)j0f, ny);
    const int64_t i1 = clamp_idx((int64_t)i0f + 1, nx), j1 = clamp_idx((int64_t)j0f + 1, ny);
    const double* v00 = &f[(j0 * nx + i0) * 3];
    const double* v10 = &f[(j0 * nx + i1) * 3];
    const double* v01 = &f[(j1 * nx + i0) * 3];
    const double* v11 = &f[(j1 * nx + i1) * 3];
    for (int c = 0; c < 3; ++c) {
        const double a = v00[c] * (1.0 - tx) + v10[c] * tx;
        const double b = v01[c] * (1.0 - tx) + v11[c] * tx;
        out[c] = a * (1.0 - ty) + b * ty;
    }
}

void orc_restrict_m_to_coarse(const orc_grid* base, const double* m_coarse, int32_t n_patches,
                              const orc_amr_patch* patches, double* out) {
    // restrict_m_to_coarse, coarse_fft_demag.rs:170-240: un-normalised area average of each
    // patch's material fine cells, patches in order (finer levels last overwrite)
    const int64_t n = base->nx * base->ny;
    std::memcpy(out, m_coarse, sizeof(double) * 3 * (size_t)n);
    for (int q = 0; q < n_patches; ++q) {
        const orc_amr_patch& p = patches[q];
        const int64_t r = p.ratio, gh = p.ghost, pnx = p.cnx * r + 2 * gh;
        for (int64_t jc = 0; jc < p.cny; ++jc)
            for (int64_t ic = 0; ic < p.cnx; ++ic) {
                double* dst = &out[((p.j0 + jc) * base->nx + p.i0 + ic) * 3];
                if (p.parent_material && !p.parent_material[jc * p.cnx + ic]) {
                    dst[0] = dst[1] = dst[2] = 0.0;
                    continue;
                }
                double sum[3] = {0.0, 0.0, 0.0};
                int64_t n_mat = 0;
                for (int64_t fj = 0; fj < r; ++fj)
                    for (int64_t fi = 0; fi < r; ++fi) {
                        const int64_t idx = (gh + jc * r + fj) * pnx + gh + ic * r + fi;
                        if (p.geom_mask_fine && !p.geom_mask_fine[idx]) continue;
                        sum[0] += p.m[idx * 3];
                        sum[1] += p.m[idx * 3 + 1];
                        sum[2] += p.m[idx * 3 + 2];
                        n_mat += 1;
                    }
                if (n_mat == 0) {
                    dst[0] = dst[1] = dst[2] = 0.0;
                } else {
                    const double inv = 1.0 / (double)n_mat;
                    dst[0] = sum[0] * inv;
                    dst[1] = sum[1] * inv;
                    dst[2] = sum[2] * inv;
                }
            }
    }
}

void orc_restrict_l0_to_demag_grid(int64_t nx_l0, const double* l0_m, int64_t dnx, int64_t dny, int64_t ratio,
                                   double* out) {
    // restrict_l0_to_demag_grid, coarse_fft_demag.rs:256-290
    const double inv_r2 = 1.0 / (double)(ratio * ratio);
    for (int64_t jd = 0; jd < dny; ++jd)
        for (int64_t id = 0; id < dnx; ++id) {
            double sum[3] = {0.0, 0.0, 0.0};
            for (int64_t fj = 0; fj < ratio; ++fj) {
                const int64_t row = (jd * ratio + fj) * nx_l0 + id * ratio;
                for (int64_t fi = 0; fi < ratio; ++fi)
                    for (int c = 0; c < 3; ++c) sum[c] += l0_m[(row + fi) * 3 + c];
            }
            for (int c = 0; c < 3; ++c) out[(jd * dnx + id) * 3 + c] = sum[c] * inv_r2;
        }
}

static void uniform_demag(const orc_grid* g, const orc_material* mat, const double* m, double* b) {
    // compute_demag_field (demag_fft_uniform.rs:146-186): zero, then add unless !mat.demag.
    // Operators are kept per grid as get_demag_operator's cache does (:86-108).
    static std::map<std::array<double, 5>, std::unique_ptr<orc_solver, void (*)(orc_solver*)>> cache;
    const std::array<double, 5> key = {(double)g->nx, (double)g->ny, g->dx, g->dy, g->dz};
    auto it = cache.find(key);
    if (it == cache.end())
        it = cache.emplace(key, std::unique_ptr<orc_solver, void (*)(orc_solver*)>(orc_solver_create(g, mat, nullptr),
                                                                                  orc_solver_destroy)).first;
    orc_solver* s = it->second.get();
    s->mat = *mat;
    orc_demag_field(s, m, b);
}

void orc_coarse_fft_demag(const orc_grid* base, const orc_material* mat, const double* m_coarse,
                          int32_t n_patches, const orc_amr_patch* patches, int64_t ratio, double* b_coarse,
                          double* b_patches) {
    // compute_coarse_fft_demag, coarse_fft_demag.rs:367-511
    const int64_t n = base->nx * base->ny;
    if (!mat->demag) {
        std::fill(b_coarse, b_coarse + 3 * n, 0.0);
        return;   // no patch fields (empty vectors in the reference)
    }
    // a ratio that is not a power of two falls back to 1 as demag_coarsen_ratio does (:98-106)
    const bool pow2 = ratio >= 1 && (ratio & (ratio - 1)) == 0;
    const int64_t r = pow2 ? orc_validated_ratio(base->nx, base->ny, ratio) : 1;
    std::vector<double> enhanced(3 * n);
    orc_restrict_m_to_coarse(base, m_coarse, n_patches, patches, enhanced.data());
    if (r <= 1) {
        uniform_demag(base, mat, enhanced.data(), b_coarse);
    } else {
        const orc_grid dg = {base->nx / r, base->ny / r, base->dx * (double)r, base->dy * (double)r, base->dz};
        std::vector<double> dm(3 * dg.nx * dg.ny), db(3 * dg.nx * dg.ny);
        orc_restrict_l0_to_demag_grid(base->nx, enhanced.data(), dg.nx, dg.ny, r, dm.data());
        uniform_demag(&dg, mat, dm.data(), db.data());
        // interpolate_demag_to_l0 (:299-318)
        for (int64_t j = 0; j < base->ny; ++j) {
            const double y = ((double)j + 0.5) * base->dy;
            for (int64_t i = 0; i < base->nx; ++i) {
                const double x = ((double)i + 0.5) * base->dx;
                orc_sample_bilinear(&dg, db.data(), x, y, &b_coarse[(j * base->nx + i) * 3]);
            }
        }
    }
    // sample_demag_to_patch (:327-340) for every patch, incl. ghosts
    double* dst = b_patches;
    for (int q = 0; q < n_patches; ++q) {
        const orc_amr_patch& p = patches[q];
        const int64_t pnx = p.cnx * p.ratio + 2 * p.ghost, pny = p.cny * p.ratio + 2 * p.ghost;
        const double fdx = base->dx / (double)p.ratio, fdy = base->dy / (double)p.ratio;
        const double gi0 = (double)(p.i0 * p.ratio), gj0 = (double)(p.j0 * p.ratio);
        for (int64_t j = 0; j < pny; ++j)
            for (int64_t i = 0; i < pnx; ++i) {
                // Patch2D::cell_center_xy, amr/patch.rs:377-387
                const double li = (double)i - (double)p.ghost, lj = (double)j - (double)p.ghost;
                const double x = (gi0 + li + 0.5) * fdx, y = (gj0 + lj + 0.5) * fdy;
                orc_sample_bilinear(base, b_coarse, x, y, dst);
                dst += 3;
            }
    }
}

void orc_allfft_demag(const orc_grid* fine, const orc_material* mat, const double* m_fine, const uint8_t* fine_mask,
                      const orc_grid* base, double* b_fine, double* b_coarse) {
    // AmrDemagMode::AllFft, amr/stepper.rs:799-835
    const int64_t nf = fine->nx * fine->ny;
    uniform_demag(fine, mat, m_fine, b_fine);
    if (fine_mask)
        for (int64_t i = 0; i < nf; ++i)
            if (!fine_mask[i]) b_fine[3 * i] = b_fine[3 * i + 1] = b_fine[3 * i + 2] = 0.0;
    for (int64_t j = 0; j < base->ny; ++j) {
        const double y = ((double)j + 0.5) * base->dy;
        for (int64_t i = 0; i < base->nx; ++i) {
            const double x = ((double)i + 0.5) * base->dx;
            orc_sample_bilinear(fine, b_fine, x, y, &b_coarse[(j * base->nx + i) * 3]);
        }
    }
}

void orc_kernel_components(double dx, double dy, double dz, int64_t sx, int64_t sy, double accuracy,
                           double out4[4]) {
    kernel_components(dx, dy, dz, sx, sy, accuracy, out4);
}

void orc_demag_kernel_kspace(orc_solver* s, double* out) {
    Demag2D& d = s->op();
    int64_t np = d.px * d.py;
    const std::vector<cplx>* src[4] = {&d.kxx, &d.kxy, &d.kyy, &d.kzz};
    for (int c = 0; c < 4; ++c) std::memcpy(out + c * np * 2, src[c]->data(), sizeof(cplx) * np);
}

void orc_demag_kernel_realspace(const orc_grid* g, int64_t pbc_x, int64_t pbc_y, double* out4) {
    int64_t px = pbc_x > 0 ? g->nx : 2 * g->nx;
    int64_t py = pbc_y > 0 ? g->ny : 2 * g->ny;
    std::vector<double> k4[4];
    build_kernel_realspace(*g, px, py, pbc_x, pbc_y, k4);
    for (int c = 0; c < 4; ++c) std::memcpy(out4 + c * px * py, k4[c].data(), sizeof(double) * px * py);
}

void orc_demag_field_pbc(const orc_grid* g, double ms, int64_t pbc_x, int64_t pbc_y, const double* m,
                         double* b_out) {
    // compute_demag_field_pbc (demag.rs:146-156 -> demag_fft_uniform.rs:157-186)
    Demag2D d(*g, pbc_x, pbc_y);
    std::fill(b_out, b_out + g->nx * g->ny * 3, 0.0);
    d.add_field(m, b_out, ms);
}

void orc_demag_kernel_kspace_pbc(const orc_grid* g, int64_t pbc_x, int64_t pbc_y, double* out) {
    Demag2D d(*g, pbc_x, pbc_y);
    int64_t np = d.px * d.py;
    const std::vector<cplx>* src[4] = {&d.kxx, &d.kxy, &d.kyy, &d.kzz};
    for (int c = 0; c < 4; ++c) std::memcpy(out + c * np * 2, src[c]->data(), sizeof(cplx) * np);
}

int orc_write_llgdmag(const orc_grid* g, int64_t pbc_x, int64_t pbc_y, const char* path) {
    // write_kernel_kspace, demag_fft_uniform.rs:279-319: little-endian header
    // (magic "LLGDMAG\0", version 2, nx, ny, pbc_x, pbc_y, px, py as u32; dx, dy, dz,
    // accuracy as f64) then kxx, kxy, kyy, kzz as px*py complex (re, im) f64 each.
    Demag2D d(*g, pbc_x, pbc_y);
    FILE* f = std::fopen(path, "wb");
    if (!f) return -1;
    const char magic[8] = {'L', 'L', 'G', 'D', 'M', 'A', 'G', '\0'};
    const uint32_t u[7] = {2u, (uint32_t)g->nx, (uint32_t)g->ny, (uint32_t)pbc_x, (uint32_t)pbc_y, (uint32_t)d.px,
                           (uint32_t)d.py};
    const double h[4] = {g->dx, g->dy, g->dz, DEMAG_ACCURACY};
    std::fwrite(magic, 1, 8, f);
    std::fwrite(u, 4, 7, f);
    std::fwrite(h, 8, 4, f);
    for (const std::vector<cplx>* v : {&d.kxx, &d.kxy, &d.kyy, &d.kzz})
        std::fwrite(v->data(), sizeof(cplx), v->size(), f);
    return std::fclose(f) == 0 ? 0 : -1;
}

void orc_demag_field_direct_pbc(const orc_grid* g, double ms, int64_t pbc_x, int64_t pbc_y, const double* m,
                                double* b_out) {
    // Direct circular convolution with the wrapped real-space kernel on the px x py
    // grid (no FFT): B(i,j) = sum K((i-i') mod px, (j-j') mod py) . Ms m(i',j')
    int64_t nx = g->nx, ny = g->ny;
    int64_t px = pbc_x > 0 ? nx : 2 * nx, py = pbc_y > 0 ? ny : 2 * ny;
    std::vector<double> k4[4];
    build_kernel_realspace(*g, px, py, pbc_x, pbc_y, k4);
#pragma omp parallel for schedule(static) num_threads(g_threads)
    for (int64_t j = 0; j < ny; ++j) {
        for (int64_t i = 0; i < nx; ++i) {
            double sx_ = 0, sy_ = 0, sz_ = 0;
            for (int64_t jj = 0; jj < ny; ++jj) {
                for (int64_t ii = 0; ii < nx; ++ii) {
                    int64_t idx = wrap_index(j - jj, py) * px + wrap_index(i - ii, px);
                    const double* mm = &m[(jj * nx + ii) * 3];
                    double Mx = ms * mm[0], My = ms * mm[1], Mz = ms * mm[2];
                    sx_ += k4[0][idx] * Mx + k4[1][idx] * My;
                    sy_ += k4[1][idx] * Mx + k4[2][idx] * My;
                    sz_ += k4[3][idx] * Mz;
                }
            }
            b_out[(j * nx + i) * 3 + 0] = sx_;
            b_out[(j * nx + i) * 3 + 1] = sy_;
            b_out[(j * nx + i) * 3 + 2] = sz_;
        }
    }
}

void orc_demag_field_direct(const orc_grid* g, double ms, const double* m, double* b_out) {
    // Direct linear convolution with the same real-space kernel:
    // B(i,j) = sum_{i',j'} K(i-i', j-j') . Ms m(i',j')   (no FFT involved)
    int64_t nx = g->nx, ny = g->ny, px = 2 * nx, py = 2 * ny;
    std::vector<double> k4[4];
    build_kernel_realspace(*g, px, py, 0, 0, k4);
#pragma omp parallel for schedule(static) num_threads(g_threads)
    for (int64_t j = 0; j < ny; ++j) {
        for (int64_t i = 0; i < nx; ++i) {
            double sx_ = 0, sy_ = 0, sz_ = 0;
            for (int64_t jj = 0; jj < ny; ++jj) {
                for (int64_t ii = 0; ii < nx; ++ii) {
                    int64_t idx = wrap_index(j - jj, py) * px + wrap_index(i - ii, px);
                    const double* mm = &m[(jj * nx + ii) * 3];
                    double Mx = ms * mm[0], My = ms * mm[1], Mz = ms * mm[2];
                    sx_ += k4[0][idx] * Mx + k4[1][idx] * My;
                    sy_ += k4[1][idx] * Mx + k4[2][idx] * My;
                    sz_ += k4[3][idx] * Mz;
                }
            }
            b_out[(j * nx + i) * 3 + 0] = sx_;
            b_out[(j * nx + i) * 3 + 1] = sy_;
            b_out[(j * nx + i) * 3 + 2] = sz_;
        }
    }
}

void orc_fft(int64_t n, double* data, int inverse) {
    Fft1D f(n, inverse != 0);
    std::vector<cplx> work(std::max<int64_t>(n, 1));
    f.exec(reinterpret_cast<cplx*>(data), work.data());
}

// XorShift64, initial_states.rs:230-254
static uint64_t xs_next(uint64_t* st) {
    uint64_t x = *st;
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    *st = x;
    return x;
}
static double xs_f64(uint64_t* st) { return (double)(xs_next(st) >> 11) * (1.0 / (double)(1ULL << 53)); }

void orc_xorshift_f64(uint64_t seed, int64_t count, double* out) {
    uint64_t st = seed == 0 ? 0x9E3779B97F4A7C15ULL : seed;
    for (int64_t i = 0; i < count; ++i) out[i] = xs_f64(&st);
}

void orc_init_random(int64_t n, uint64_t seed, double* m) {
    // init_random, initial_states.rs:59-68
    uint64_t st = seed == 0 ? 0x9E3779B97F4A7C15ULL : seed;
    for (int64_t i = 0; i < n; ++i) {
        double v[3];
        v[0] = xs_f64(&st) * 2.0 - 1.0;
        v[1] = xs_f64(&st) * 2.0 - 1.0;
        v[2] = xs_f64(&st) * 2.0 - 1.0;
        vnormalize(v, &m[i * 3]);
    }
}

void orc_init_uniform_with_noise(int64_t n, const double dir[3], double noise, uint64_t seed, double* m) {
    // init_uniform_with_noise, initial_states.rs:43-56 (pre-masked zero cells are skipped)
    double base[3];
    vnormalize(dir, base);
    uint64_t st = seed == 0 ? 0x9E3779B97F4A7C15ULL : seed;
    for (int64_t i = 0; i < n; ++i) {
        double* v = &m[i * 3];
        if (v[0] == 0.0 && v[1] == 0.0 && v[2] == 0.0) continue;
        double dx = noise * (xs_f64(&st) * 2.0 - 1.0);
        double dy = noise * (xs_f64(&st) * 2.0 - 1.0);
        double dz = noise * (xs_f64(&st) * 2.0 - 1.0);
        double w[3] = {base[0] + dx, base[1] + dy, base[2] + dz};
        vnormalize(w, v);
    }
}

}  // extern "C"
