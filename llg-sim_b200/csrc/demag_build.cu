// demag_build.cu — FP64 construction of the demag kernel on the GPU.
//
// Follows Demag2D::new for open boundaries (demag_fft_uniform.rs:470-634):
//   1. quadrant kernel K = mu0*N(sx, sy) for 0 <= sx < nx, 0 <= sy < ny by the
//      MuMax-like face-charge integration (kernel_2d_components_mumax_like /
//      mumax_like_h_from_unit_m, demag_fft_uniform.rs:1076-1253) — one warp per
//      displacement, the integration points split over the lanes;
//   2. reflection onto the 2nx x 2ny padded grid with exact parity, Kxy zero on
//      the axes, Nyquist planes zero (demag_fft_uniform.rs:1013-1072);
//   3. FP64 2-D FFT of the four planes (rows then columns, the project's
//      shared-memory FFT in double precision);
//   4. extraction of the real parts on kx in [0,nx], ky in [0,ny], scaled by
//      1/(px*py) and cast to the solver precision.
// Each integration sample differences two charge/(4 pi r^3) pole terms that
// cancel at large r, so all of this stays FP64.
#include <algorithm>
#include <vector>

#include "build_api.h"
#include "fft_smem.cuh"
#include "field_kernels.cuh"

namespace llg {

namespace {

constexpr double kPi = 3.14159265358979323846;

__device__ __forceinline__ double delta_cell(long long d) {
    double a = (double)(d < 0 ? -d : d);
    if (a > 0.0) a -= 1.0;
    return a;
}
__device__ __forceinline__ long long mumax_n(double x) { return (long long)floor(fmax(x, 1.0) + 0.5); }

// One warp integrates the field of unit magnetisation along `u` of the source
// cell at r_center (mumax_like_h_from_unit_m, demag_fft_uniform.rs:1139-1242).
__device__ void warp_h_from_unit_m(int u, const double* rc, const double* cell, const long long* disp, double accuracy,
                                   double* h_out) {
    const int lane = threadIdx.x & 31;
    const int v = (u + 1) % 3, w = (u + 2) % 3;
    const double lmin = fmin(fmin(cell[0], cell[1]), cell[2]);
    const double dxm = delta_cell(disp[0]) * cell[0];
    const double dym = delta_cell(disp[1]) * cell[1];
    const double dzm = delta_cell(disp[2]) * cell[2];
    double d = sqrt(dxm * dxm + dym * dym + dzm * dzm);
    if (d == 0.0) d = lmin;
    const double max_size = d / accuracy;
    const long long nx = mumax_n(cell[0] / max_size);
    const long long ny = mumax_n(cell[1] / max_size);
    const long long nz = mumax_n(cell[2] / max_size);
    const long long nv = 2 * mumax_n(cell[v] / max_size);
    const long long nw = 2 * mumax_n(cell[w] / max_size);
    const double scale = 1.0 / (double)(nv * nw * nx * ny * nz);
    const double charge = cell[v] * cell[w] * scale;
    const double pu1 = 0.5 * cell[u], pu2 = -pu1;
    const long long total = nv * nw * nx * ny * nz;
    double h0 = 0.0, h1 = 0.0, h2 = 0.0;
    for (long long t = lane; t < total; t += 32) {
        long long q = t;
        const long long az = q % nz; q /= nz;
        const long long ay = q % ny; q /= ny;
        const long long ax = q % nx; q /= nx;
        const long long jw = q % nw;
        const long long iv = q / nw;
        double pole[3];
        pole[v] = -0.5 * cell[v] + cell[v] / (2.0 * (double)nv) + (double)iv * (cell[v] / (double)nv);
        pole[w] = -0.5 * cell[w] + cell[w] / (2.0 * (double)nw) + (double)jw * (cell[w] / (double)nw);
        const double rx = rc[0] - 0.5 * cell[0] + cell[0] / (2.0 * (double)nx) + (double)ax * (cell[0] / (double)nx);
        const double ry = rc[1] - 0.5 * cell[1] + cell[1] / (2.0 * (double)ny) + (double)ay * (cell[1] / (double)ny);
        const double rz = rc[2] - 0.5 * cell[2] + cell[2] / (2.0 * (double)nz) + (double)az * (cell[2] / (double)nz);
        pole[u] = pu1;
        const double r1x = rx - pole[0], r1y = ry - pole[1], r1z = rz - pole[2];
        const double r1 = sqrt(r1x * r1x + r1y * r1y + r1z * r1z);
        const double q1 = charge / (4.0 * kPi * r1 * r1 * r1);
        pole[u] = pu2;
        const double r2x = rx - pole[0], r2y = ry - pole[1], r2z = rz - pole[2];
        const double r2 = sqrt(r2x * r2x + r2y * r2y + r2z * r2z);
        const double q2 = -charge / (4.0 * kPi * r2 * r2 * r2);
        h0 += r1x * q1 + r2x * q2;
        h1 += r1y * q1 + r2y * q2;
        h2 += r1z * q1 + r2z * q2;
    }
    for (int o = 16; o > 0; o >>= 1) {
        h0 += __shfl_xor_sync(0xffffffffu, h0, o);
        h1 += __shfl_xor_sync(0xffffffffu, h1, o);
        h2 += __shfl_xor_sync(0xffffffffu, h2, o);
    }
    h_out[0] = h0;
    h_out[1] = h1;
    h_out[2] = h2;
}

__global__ void k_kernel_quadrant(int nx, int ny, double dx, double dy, double dz, double accuracy,
                                  double* __restrict__ quad) {
    const long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (wid >= (long long)nx * ny) return;
    const int sy = (int)(wid / nx), sx = (int)(wid % nx);
    const double rc[3] = {(double)sx * dx, (double)sy * dy, 0.0};
    const double cell[3] = {dx, dy, dz};
    const long long disp[3] = {sx, sy, 0};
    double hx[3], hy[3], hz[3];
    warp_h_from_unit_m(0, rc, cell, disp, accuracy, hx);
    warp_h_from_unit_m(1, rc, cell, disp, accuracy, hy);
    warp_h_from_unit_m(2, rc, cell, disp, accuracy, hz);
    if ((threadIdx.x & 31) == 0) {
        const double mu0 = 4.0 * kPi * 1e-7;  // params.rs:15
        double* o = quad + wid * 4;
        o[0] = mu0 * hx[0];
        o[1] = mu0 * hy[0];
        o[2] = mu0 * hy[1];
        o[3] = mu0 * hz[2];
    }
}

__global__ void k_kernel_expand(int nx, int ny, const double* __restrict__ quad, cx<double>* __restrict__ planes) {
    const int px = 2 * nx, py = 2 * ny;
    const long long np = (long long)px * py;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < np; e += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(e % px), iy = (int)(e / px);
        double v[4] = {0.0, 0.0, 0.0, 0.0};
        if (ix != nx && iy != ny) {
            const int sx = ix < nx ? ix : ix - px;
            const int sy = iy < ny ? iy : iy - py;
            const int ax = sx < 0 ? -sx : sx, ay = sy < 0 ? -sy : sy;
            const double* q = quad + ((long long)ay * nx + ax) * 4;
            v[0] = q[0];
            v[2] = q[2];
            v[3] = q[3];
            v[1] = (sx == 0 || sy == 0) ? 0.0 : ((sx < 0) != (sy < 0) ? -q[1] : q[1]);
        }
        for (int c = 0; c < 4; ++c) planes[c * np + e] = mkc(v[c], 0.0);
    }
}

template <typename R>
__global__ void k_kernel_extract(int nx, int ny, const cx<double>* __restrict__ planes, double scale,
                                 r4<R>* __restrict__ khat, double* __restrict__ k64, bool split) {
    const int px = 2 * nx, py = 2 * ny;
    const long long np = (long long)px * py;
    const int total = (nx + 1) * (ny + 1);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int kx = e / (ny + 1), ky = e % (ny + 1);
        const int slot = split ? kx * (ny + 1) + khat_index(ky, ny) : e;
        double v[4];
        for (int c = 0; c < 4; ++c) v[c] = planes[c * np + (long long)ky * px + kx].re;
        r4<R> o;
        o.x = (R)(v[0] * scale);
        o.y = (R)(v[1] * scale);
        o.z = (R)(v[2] * scale);
        o.w = (R)(v[3] * scale);
        khat[slot] = o;
        // export layout [c][ky][kx]
        for (int c = 0; c < 4; ++c) k64[((long long)c * (ny + 1) + ky) * (nx + 1) + kx] = v[c];
    }
}

// Periodic images (build_kernel_realspace_pbc, demag_fft_uniform.rs:941-1005):
// one warp per displacement (sx, sy) in [-sx_max, sx_max] x [-sy_max, sy_max].
__global__ void k_kernel_displacements(int sx_max, int sy_max, double dx, double dy, double dz, double accuracy,
                                       double* __restrict__ comp) {
    const long long nsx = 2LL * sx_max + 1, nsy = 2LL * sy_max + 1;
    const long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (wid >= nsx * nsy) return;
    const long long sx = wid % nsx - sx_max, sy = wid / nsx - sy_max;
    const double rc[3] = {(double)sx * dx, (double)sy * dy, 0.0};
    const double cell[3] = {dx, dy, dz};
    const long long disp[3] = {sx, sy, 0};
    double hx[3], hy[3], hz[3];
    warp_h_from_unit_m(0, rc, cell, disp, accuracy, hx);
    warp_h_from_unit_m(1, rc, cell, disp, accuracy, hy);
    warp_h_from_unit_m(2, rc, cell, disp, accuracy, hz);
    if ((threadIdx.x & 31) == 0) {
        const double mu0 = 4.0 * kPi * 1e-7;  // params.rs:15
        double* o = comp + wid * 4;
        o[0] = mu0 * hx[0];
        o[1] = mu0 * hy[0];
        o[2] = mu0 * hy[1];
        o[3] = mu0 * hz[2];
    }
}

// Wrapped sums of the images into the px x py bins, per bin in the reference's
// accumulation order (sy ascending, then sx ascending); Kxy zero on the axes.
__global__ void k_kernel_wrap(int sx_max, int sy_max, int px, int py, const double* __restrict__ comp,
                              cx<double>* __restrict__ planes) {
    const long long nsx = 2LL * sx_max + 1;
    const long long np = (long long)px * py;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < np; e += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(e % px), iy = (int)(e / px);
        double v[4] = {0.0, 0.0, 0.0, 0.0};
        // smallest sy >= -sy_max with sy = iy (mod py)
        long long sy0 = iy - ((iy + (long long)sy_max) / py) * py;
        long long sx0 = ix - ((ix + (long long)sx_max) / px) * px;
        for (long long sy = sy0; sy <= sy_max; sy += py)
            for (long long sx = sx0; sx <= sx_max; sx += px) {
                const double* kc = comp + ((sy + sy_max) * nsx + (sx + sx_max)) * 4;
                for (int c = 0; c < 4; ++c) v[c] += kc[c];
            }
        if (ix == 0 || iy == 0) v[1] = 0.0;
        for (int c = 0; c < 4; ++c) planes[c * np + e] = mkc(v[c], 0.0);
    }
}

}  // namespace

template <typename R>
__global__ void k_twiddles(cx<R>* tw, int L2) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < L2; k += gridDim.x * blockDim.x) {
        double s, c;
        sincospi(2.0 * (double)k / (double)L2, &s, &c);
        tw[k] = mkc((R)c, (R)(-s));
    }
}

template <typename R>
__global__ void k_fft_strided(cx<R>* data, FftPlan plan, const cx<R>* tw2, long long elem_stride, int nsig_a,
                              long long stride_a, long long stride_b, int inverse) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<R>* A = reinterpret_cast<cx<R>*>(smem_raw);
    cx<R>* B = A + plan.L;
    const int sig = blockIdx.x;
    const long long base = (long long)(sig % nsig_a) * stride_a + (long long)(sig / nsig_a) * stride_b;
    for (int t = threadIdx.x; t < plan.L; t += blockDim.x) A[t] = data[base + t * elem_stride];
    __syncthreads();
    cx<R>* res = fft_smem<R>(A, B, 1, plan, tw2, inverse != 0);
    for (int t = threadIdx.x; t < plan.L; t += blockDim.x) data[base + t * elem_stride] = res[t];
}

// Column transforms of adjacent signals (stride between signals 1 element): a block
// takes NS neighbouring columns, so that one row of the tile is NS consecutive
// elements in memory (whole 32-byte sectors in FP64 instead of half ones); each
// signal's arithmetic is the one of k_fft_strided.
template <typename R>
__global__ void k_fft_strided_tiled(cx<R>* data, FftPlan plan, const cx<R>* tw2, long long elem_stride, int nsig_a,
                                    long long stride_b, int ns, int inverse) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L = plan.L;
    cx<R>* A = reinterpret_cast<cx<R>*>(smem_raw);
    cx<R>* B = A + (size_t)ns * L;
    const int tiles_a = nsig_a / ns;
    const long long base = (long long)(blockIdx.x % tiles_a) * ns + (long long)(blockIdx.x / tiles_a) * stride_b;
    for (int e = threadIdx.x; e < ns * L; e += blockDim.x) {
        const int c = e % ns, t = e / ns;
        A[(size_t)c * L + t] = data[base + c + t * elem_stride];
    }
    __syncthreads();
    cx<R>* res = fft_smem<R>(A, B, ns, plan, tw2, inverse != 0);
    for (int e = threadIdx.x; e < ns * L; e += blockDim.x) {
        const int c = e % ns, t = e / ns;
        data[base + c + t * elem_stride] = res[(size_t)c * L + t];
    }
}

template __global__ void k_twiddles<float>(cx<float>*, int);
template __global__ void k_twiddles<double>(cx<double>*, int);

FftPlan make_plan(int L) {
    FftPlan p{};
    p.L = L;
    p.npass = 0;
    int r = L;
    for (int f : {8, 4, 2, 3, 5}) {
        while (r % f == 0 && r > 1) {
            p.radix[p.npass++] = f;
            r /= f;
        }
    }
    for (int f = 7; r > 1; f += 2) {
        while (r % f == 0) {
            p.radix[p.npass++] = f;
            r /= f;
        }
    }
    return p;
}

// Candidate radix plans of the generic Stockham transform of length L (any radix
// order is a valid Stockham plan): the powers of two grouped mostly as 8s or
// mostly as 4s, each with the odd factors last (make_plan's order), first, or the
// powers of two in ascending order.  The first candidate is make_plan(L).
std::vector<FftPlan> plan_candidates(int L) {
    std::vector<FftPlan> out;
    out.push_back(make_plan(L));
    int r = L, e2 = 0;
    while (r % 2 == 0 && r > 1) {
        r /= 2;
        ++e2;
    }
    std::vector<int> odd;
    for (int f : {3, 5}) while (r % f == 0) { odd.push_back(f); r /= f; }
    for (int f = 7; r > 1; f += 2) while (r % f == 0) { odd.push_back(f); r /= f; }
    auto twos = [&](bool eights) {
        std::vector<int> v;
        int e = e2;
        if (eights) {
            while (e >= 3) { v.push_back(8); e -= 3; }
            if (e == 2) v.push_back(4);
            if (e == 1) v.push_back(2);
        } else {
            while (e >= 2) { v.push_back(4); e -= 2; }
            if (e == 1) v.push_back(2);
        }
        return v;
    };
    auto add = [&](const std::vector<int>& rad) {
        if (rad.empty() || (int)rad.size() > kMaxRadices) return;
        FftPlan p{};
        p.L = L;
        p.npass = (int)rad.size();
        for (size_t i = 0; i < rad.size(); ++i) p.radix[i] = rad[i];
        for (const FftPlan& q : out)
            if (q.npass == p.npass && std::equal(q.radix, q.radix + q.npass, p.radix)) return;
        out.push_back(p);
    };
    for (bool eights : {true, false}) {
        std::vector<int> t = twos(eights);
        std::vector<int> a = t, b = odd, c = t;
        a.insert(a.end(), odd.begin(), odd.end());           // powers of two first
        b.insert(b.end(), t.begin(), t.end());               // odd factors first
        std::reverse(c.begin(), c.end());                    // ascending powers of two, then odd
        c.insert(c.end(), odd.begin(), odd.end());
        add(a);
        add(b);
        add(c);
    }
    return out;
}

cudaError_t launch_twiddles(void* tw, int L2, bool fp64, cudaStream_t s) {
    int blocks = (L2 + 255) / 256;
    if (fp64) k_twiddles<double><<<blocks, 256, 0, s>>>(reinterpret_cast<cx<double>*>(tw), L2);
    else k_twiddles<float><<<blocks, 256, 0, s>>>(reinterpret_cast<cx<float>*>(tw), L2);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_fft_strided(void* data, int L, const void* tw2, long long elem_stride, int nsig_a, long long stride_a,
                               int nsig_b, long long stride_b, bool inverse, cudaStream_t s) {
    FftPlan plan = make_plan(L);
    if (elem_stride > 1 && stride_a == 1) {
        // adjacent columns: tile NS of them per block where shared memory allows
        int ns = 1;
        while (ns < 8 && nsig_a % (2 * ns) == 0 && 2 * (size_t)(2 * ns) * L * sizeof(cx<R>) <= 200 * 1024) ns *= 2;
        if (ns > 1) {
            const size_t smem = 2 * (size_t)ns * L * sizeof(cx<R>);
            cudaError_t e = cudaFuncSetAttribute(k_fft_strided_tiled<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)smem);
            if (e != cudaSuccess) return e;
            k_fft_strided_tiled<R><<<(nsig_a / ns) * nsig_b, 256, smem, s>>>(
                reinterpret_cast<cx<R>*>(data), plan, reinterpret_cast<const cx<R>*>(tw2), elem_stride, nsig_a,
                stride_b, ns, inverse ? 1 : 0);
            return cudaGetLastError();
        }
    }
    size_t smem = 2 * (size_t)L * sizeof(cx<R>);
    cudaError_t e = cudaFuncSetAttribute(k_fft_strided<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_fft_strided<R><<<nsig_a * nsig_b, 256, smem, s>>>(reinterpret_cast<cx<R>*>(data), plan,
                                                        reinterpret_cast<const cx<R>*>(tw2), elem_stride, nsig_a,
                                                        stride_a, stride_b, inverse ? 1 : 0);
    return cudaGetLastError();
}
template cudaError_t launch_fft_strided<float>(void*, int, const void*, long long, int, long long, int, long long,
                                               bool, cudaStream_t);
template cudaError_t launch_fft_strided<double>(void*, int, const void*, long long, int, long long, int, long long,
                                                bool, cudaStream_t);

#define CK(x)                                  \
    do {                                       \
        cudaError_t _e = (x);                  \
        if (_e != cudaSuccess) return _e;      \
    } while (0)

cudaError_t build_demag_kernel(int nx, int ny, double dx, double dy, double dz, bool fp64_out, void* khat_out,
                               double* k64_out_dev, cudaStream_t s, bool split_columns) {
    if (split_columns && (ny % 2) != 0) return cudaErrorInvalidValue;
    const int px = 2 * nx, py = 2 * ny;
    const long long np = (long long)px * py;
    double* quad = nullptr;
    cx<double>* planes = nullptr;
    cx<double>* twx = nullptr;
    cx<double>* twy = nullptr;
    cudaError_t err = cudaSuccess;
    auto cleanup = [&]() {
        if (quad) cudaFree(quad);
        if (planes) cudaFree(planes);
        if (twx) cudaFree(twx);
        if (twy) cudaFree(twy);
    };
    do {
        if ((err = cudaMalloc(&quad, sizeof(double) * 4 * (size_t)nx * ny)) != cudaSuccess) break;
        if ((err = cudaMalloc(&planes, sizeof(cx<double>) * 4 * (size_t)np)) != cudaSuccess) break;
        if ((err = cudaMalloc(&twx, sizeof(cx<double>) * 2 * (size_t)px)) != cudaSuccess) break;
        if ((err = cudaMalloc(&twy, sizeof(cx<double>) * 2 * (size_t)py)) != cudaSuccess) break;
        {
            long long warps = (long long)nx * ny;
            long long threads = warps * 32;
            int blocks = (int)((threads + 255) / 256);
            k_kernel_quadrant<<<blocks, 256, 0, s>>>(nx, ny, dx, dy, dz, 10.0 /* DEMAG_ACCURACY :432 */, quad);
            if ((err = cudaGetLastError()) != cudaSuccess) break;
        }
        k_kernel_expand<<<1184, 256, 0, s>>>(nx, ny, quad, planes);
        if ((err = cudaGetLastError()) != cudaSuccess) break;
        if ((err = launch_twiddles(twx, 2 * px, true, s)) != cudaSuccess) break;
        if ((err = launch_twiddles(twy, 2 * py, true, s)) != cudaSuccess) break;
        // rows: length px, contiguous; signals = py rows x 4 planes
        if ((err = launch_fft_strided<double>(planes, px, twx, 1, py, px, 4, np, false, s)) != cudaSuccess) break;
        // columns: length py, stride px; signals = px columns x 4 planes
        if ((err = launch_fft_strided<double>(planes, py, twy, px, px, 1, 4, np, false, s)) != cudaSuccess) break;
        const double scale = 1.0 / (double)np;
        int blocks = ((nx + 1) * (ny + 1) + 255) / 256;
        if (fp64_out)
            k_kernel_extract<double><<<blocks, 256, 0, s>>>(
                nx, ny, planes, scale, reinterpret_cast<r4<double>*>(khat_out), k64_out_dev, split_columns);
        else
            k_kernel_extract<float><<<blocks, 256, 0, s>>>(
                nx, ny, planes, scale, reinterpret_cast<r4<float>*>(khat_out), k64_out_dev, split_columns);
        if ((err = cudaGetLastError()) != cudaSuccess) break;
        err = cudaStreamSynchronize(s);
    } while (0);
    cleanup();
    return err;
}

// Unscaled k-space kernel planes (xx, xy, yy, zz; [c][iy][ix] complex) of Demag2D::new
// for pbc_x / pbc_y images (0 = open, padded to 2n), px = pbc_x ? nx : 2 nx.
cudaError_t build_demag_kernel_pbc(int nx, int ny, double dx, double dy, double dz, int pbc_x, int pbc_y,
                                   void* planes_out, cudaStream_t s) {
    const int px = pbc_x > 0 ? nx : 2 * nx, py = pbc_y > 0 ? ny : 2 * ny;
    const long long np = (long long)px * py;
    const int sx_max = pbc_x == 0 ? nx - 1 : nx * pbc_x - 1;
    const int sy_max = pbc_y == 0 ? ny - 1 : ny * pbc_y - 1;
    const long long ndisp = (2LL * sx_max + 1) * (2LL * sy_max + 1);
    cx<double>* planes = reinterpret_cast<cx<double>*>(planes_out);
    double* comp = nullptr;
    cx<double>* twx = nullptr;
    cx<double>* twy = nullptr;
    cudaError_t err = cudaSuccess;
    do {
        if ((err = cudaMalloc(&comp, sizeof(double) * 4 * (size_t)ndisp)) != cudaSuccess) break;
        if ((err = cudaMalloc(&twx, sizeof(cx<double>) * 2 * (size_t)px)) != cudaSuccess) break;
        if ((err = cudaMalloc(&twy, sizeof(cx<double>) * 2 * (size_t)py)) != cudaSuccess) break;
        const long long blocks = (ndisp * 32 + 255) / 256;
        k_kernel_displacements<<<(unsigned)blocks, 256, 0, s>>>(sx_max, sy_max, dx, dy, dz, 10.0, comp);
        if ((err = cudaGetLastError()) != cudaSuccess) break;
        k_kernel_wrap<<<1184, 256, 0, s>>>(sx_max, sy_max, px, py, comp, planes);
        if ((err = cudaGetLastError()) != cudaSuccess) break;
        if ((err = launch_twiddles(twx, 2 * px, true, s)) != cudaSuccess) break;
        if ((err = launch_twiddles(twy, 2 * py, true, s)) != cudaSuccess) break;
        if ((err = launch_fft_strided<double>(planes, px, twx, 1, py, px, 4, np, false, s)) != cudaSuccess) break;
        if ((err = launch_fft_strided<double>(planes, py, twy, px, px, 1, 4, np, false, s)) != cudaSuccess) break;
        err = cudaStreamSynchronize(s);
    } while (0);
    if (comp) cudaFree(comp);
    if (twx) cudaFree(twx);
    if (twy) cudaFree(twy);
    return err;
}

}  // namespace llg
