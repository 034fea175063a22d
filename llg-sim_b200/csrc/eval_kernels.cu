// eval_kernels.cu — instantiation and launch of the per-evaluation kernels for
// FP32 and FP64: register-FFT kernels for power-of-two sizes, generic
// shared-memory Stockham kernels otherwise.
#include "build_api.h"
#include "fast_kernels.cuh"
#include "fused_kernels.cuh"
#include "stage_kernels.cuh"

#include <algorithm>
#include <cstdlib>

namespace llg {

namespace {

template <typename R, typename F>
bool dispatch_L(int L, F&& f) {
    switch (L) {
        case 16: f(std::integral_constant<int, 16>{}); return true;
        case 32: f(std::integral_constant<int, 32>{}); return true;
        case 64: f(std::integral_constant<int, 64>{}); return true;
        case 128: f(std::integral_constant<int, 128>{}); return true;
        case 256: f(std::integral_constant<int, 256>{}); return true;
        case 512: f(std::integral_constant<int, 512>{}); return true;
        case 1024: f(std::integral_constant<int, 1024>{}); return true;
        case 2048: f(std::integral_constant<int, 2048>{}); return true;
        default: return false;
    }
}

constexpr size_t kSmemMax = 227 * 1024;
constexpr size_t kStaticSmemCol = 64;   // mbarriers and the timeout flag of k_column_fast

// Intermediate RK stages need only the torque: no reductions, error norm or
// field output.
bool lean_epilogue(const EvalSpec& e) {
    return e.err == ERR_NONE && !e.reduce && e.local && (e.rhs == RHS_LLG || e.rhs == RHS_RELAX);
}
int stage_grid(long long work) {
    return (int)std::max(1LL, std::min((work + 255) / 256, 148LL * 8));
}

// The last RK45 stage of a run (no reductions): torque plus the error norm.
bool lean_err45_epilogue(const EvalSpec& e) {
    return e.err == ERR_RK45 && !e.reduce && e.local && e.rhs == RHS_LLG && e.k_out != KB_NONE;
}

}  // namespace

template <typename R>
FastCfg fast_config(int nx, int ny) {
    FastCfg c{};
    bool okr = dispatch_L<R>(nx, [&](auto LC) {
        constexpr int L = decltype(LC)::value;
        c.T = RowCfg<R, L>::T;
        c.row_threads = RowCfg<R, L>::THREADS;
        c.smem_row = RowCfg<R, L>::SMEM;
        c.twp_row_size = TwTab<R, L>::size;
    });
    bool okc = dispatch_L<R>(ny, [&](auto LC) {
        constexpr int L = decltype(LC)::value;
        c.NC = ColCfg<R, L>::NC;
        c.col_threads = ColCfg<R, L>::THREADS;
        c.smem_col = ColCfg<R, L>::SMEM;
        c.twp_col_size = TwTab<R, L>::size;
    });
    // The register-FFT row kernels move the spectrum of consecutive rows as 16-byte
    // pieces of the column-major X[c][kx][j]: in FP32 a piece is two rows, so the
    // column stride ny must be even for every piece to start on a 16-byte boundary.
    c.ok_row = okr && c.smem_row <= kSmemMax && (sizeof(R) == 8 || ny % 2 == 0);
    c.ok_col = okc && c.smem_col + kStaticSmemCol <= kSmemMax;
    c.ok = c.ok_row && c.ok_col;
    return c;
}

template <typename R>
cudaError_t build_pass_tables(void* out_row, int nx, void* out_col, int ny, cudaStream_t s) {
    cudaError_t err = cudaSuccess;
    dispatch_L<R>(nx, [&](auto LC) {
        constexpr int L = decltype(LC)::value;
        if (TwTab<R, L>::size > 0) {
            k_pass_tables<R, L><<<(TwTab<R, L>::size + 255) / 256, 256, 0, s>>>(reinterpret_cast<cx<R>*>(out_row));
            err = cudaGetLastError();
        }
    });
    if (err != cudaSuccess) return err;
    dispatch_L<R>(ny, [&](auto LC) {
        constexpr int L = decltype(LC)::value;
        if (TwTab<R, L>::size > 0) {
            k_pass_tables<R, L><<<(TwTab<R, L>::size + 255) / 256, 256, 0, s>>>(reinterpret_cast<cx<R>*>(out_col));
            err = cudaGetLastError();
        }
    });
    return err;
}

template <typename R>
cudaError_t prepare_eval_kernels(size_t smem_row, size_t smem_col) {
    cudaError_t e;
    e = cudaFuncSetAttribute(k_row_forward<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_row_inverse<R, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_row_inverse<R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_column<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_col);
    if (e != cudaSuccess) return e;
    // fast kernels: every instantiation whose shared memory fits
    auto set_all = [&](auto LC) {
        constexpr int L = decltype(LC)::value;
        if (RowCfg<R, L>::SMEM <= kSmemMax) {
            cudaFuncSetAttribute(k_row_forward_fast<R, L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)RowCfg<R, L>::SMEM);
            cudaFuncSetAttribute(k_row_inverse_fast<R, L, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)RowCfg<R, L>::SMEM);
            cudaFuncSetAttribute(k_row_inverse_fast<R, L, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)RowCfg<R, L>::SMEM);
            cudaFuncSetAttribute(k_row_inverse_fast<R, L, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)RowCfg<R, L>::SMEM);
        }
        if (RowCfg<R, L>::SMEM <= kSmemMax) {
            cudaFuncSetAttribute(k_row_fused<R, L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)RowCfg<R, L>::SMEM);
            cudaFuncSetAttribute(k_row_fused<R, L>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        }
        if (ColCfg<R, L>::SMEM + kStaticSmemCol <= kSmemMax)
            cudaFuncSetAttribute(k_column_fast<R, L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)ColCfg<R, L>::SMEM);
        if (ColDirectCfg<R, L>::SMEM <= kSmemMax) {
            cudaFuncSetAttribute(k_column_direct<R, L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)ColDirectCfg<R, L>::SMEM);
            cudaFuncSetAttribute(k_column_direct<R, L>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        }
        // the whole unified L1/shared array as shared memory, so that occupancy is
        // bounded by registers and the blocks' own shared memory only
        cudaFuncSetAttribute(k_row_forward_fast<R, L>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        cudaFuncSetAttribute(k_row_inverse_fast<R, L, 0>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        cudaFuncSetAttribute(k_row_inverse_fast<R, L, 1>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        cudaFuncSetAttribute(k_row_inverse_fast<R, L, 2>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        cudaFuncSetAttribute(k_column_fast<R, L>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    };
    for (int L : {16, 32, 64, 128, 256, 512, 1024, 2048}) dispatch_L<R>(L, set_all);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_one(int which, const EvalSpec& spec, const LaunchGeom& g, cudaStream_t s, int* nk) {
    int count = 0;
    if (which == 0 || which == 2) {
        if (g.fast_row) {
            dispatch_L<R>(g.fast_row, [&](auto LC) {
                constexpr int L = decltype(LC)::value;
                if constexpr (RowCfg<R, L>::SMEM <= kSmemMax) {
                    using C = RowCfg<R, L>;
                    if (which == 0) {
                        k_row_forward_fast<R, L><<<g.grid_row, C::THREADS, C::SMEM, s>>>(g.films, g.row_items,
                                                                                        g.n_row_items, spec);
                        ++count;
                    } else if (lean_epilogue(spec) || lean_err45_epilogue(spec)) {
                        // transform only, then the torque epilogue as a streaming kernel
                        constexpr int CPI = C::T * L;
                        const long long cells = (long long)g.n_row_items * CPI;
                        k_row_inverse_fast<R, L, 1><<<g.grid_rinv, C::THREADS, C::SMEM, s>>>(g.films, g.row_items,
                                                                                            g.n_row_items, spec);
                        if (lean_err45_epilogue(spec))
                            k_stage_torque<R, true><<<stage_grid(cells), 256, 0, s>>>(g.films, g.row_items,
                                                                                        g.n_row_items, CPI, spec);
                        else
                            k_stage_torque<R, false><<<stage_grid(cells), 256, 0, s>>>(g.films, g.row_items,
                                                                                         g.n_row_items, CPI, spec);
                        count += 2;
                    } else if (spec.rhs == RHS_MINIMIZE) {
                        k_row_inverse_fast<R, L, 2><<<g.grid_rfull, C::THREADS, C::SMEM, s>>>(g.films, g.row_items,
                                                                                             g.n_row_items, spec);
                        ++count;
                    } else {
                        k_row_inverse_fast<R, L, 0><<<g.grid_rfull, C::THREADS, C::SMEM, s>>>(g.films, g.row_items,
                                                                                             g.n_row_items, spec);
                        ++count;
                    }
                }
            });
        } else if (which == 0) {
            k_row_forward<R><<<g.grid_row, 256, g.smem_row, s>>>(g.films, g.row_items, g.n_row_items, spec);
            ++count;
        } else {
            if (spec.rhs == RHS_MINIMIZE)
                k_row_inverse<R, true><<<g.grid_row, 256, g.smem_row, s>>>(g.films, g.row_items, g.n_row_items,
                                                                           spec);
            else
                k_row_inverse<R, false><<<g.grid_row, 256, g.smem_row, s>>>(g.films, g.row_items, g.n_row_items,
                                                                            spec);
            ++count;
        }
    } else {
        if (g.fast_col) {
            dispatch_L<R>(g.fast_col, [&](auto LC) {
                constexpr int L = decltype(LC)::value;
                if (g.col_direct) {
                    if constexpr (ColDirectCfg<R, L>::SMEM <= kSmemMax)
                        k_column_direct<R, L><<<g.grid_col, ColCfg<R, L>::THREADS, ColDirectCfg<R, L>::SMEM, s>>>(
                            g.films, g.col_items, g.n_col_items, spec);
                } else if constexpr (ColCfg<R, L>::SMEM + kStaticSmemCol <= kSmemMax) {
                    k_column_fast<R, L><<<g.grid_col, ColCfg<R, L>::THREADS, ColCfg<R, L>::SMEM, s>>>(
                        g.films, g.col_items, g.n_col_items, spec);
                }
            });
        } else {
            k_column<R><<<g.grid_col, 256, g.smem_col, s>>>(g.films, g.col_items, g.n_col_items, spec);
        }
        ++count;
    }
    if (nk) *nk += count;
    return cudaGetLastError();
}

bool can_fuse(const EvalSpec& si, const EvalSpec& sf, const LaunchGeom& g) {
    return g.fast_row != 0 && g.fuse_rows && lean_epilogue(si) && si.k_out != KB_NONE && !si.skip_if_fsal &&
           !sf.skip_if_fsal && sf.nterm >= 1 && sf.nterm <= 6 && sf.kidx[sf.nterm - 1] == si.k_out &&
           sf.req == si.req && sf.demag == si.demag && sf.m_in != si.m_in;
}

template <typename R>
cudaError_t launch_fused(const EvalSpec& si, const EvalSpec& sf, const LaunchGeom& g, cudaStream_t s, int* nk) {
    dispatch_L<R>(g.fast_row, [&](auto LC) {
        constexpr int L = decltype(LC)::value;
        if constexpr (RowCfg<R, L>::SMEM <= kSmemMax) {
            using C = RowCfg<R, L>;
            k_row_fused<R, L><<<g.grid_fused, C::THREADS, C::SMEM, s>>>(g.films, g.row_items, g.n_row_items, si, sf);
        }
    });
    if (nk) *nk += 1;
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_eval(const EvalSpec& spec, const LaunchGeom& g, cudaStream_t s) {
    cudaError_t e = launch_one<R>(0, spec, g, s, nullptr);
    if (e != cudaSuccess) return e;
    if (spec.demag && g.any_demag) {
        e = launch_one<R>(1, spec, g, s, nullptr);
        if (e != cudaSuccess) return e;
    }
    return launch_one<R>(2, spec, g, s, nullptr);
}

template <typename R>
void fast_occupancy(int nx, int ny, bool col_direct, int* fwd_blocks_per_sm, int* inv_blocks_per_sm,
                    int* full_blocks_per_sm, int* fused_blocks_per_sm, int* col_blocks_per_sm) {
    *fwd_blocks_per_sm = *inv_blocks_per_sm = *full_blocks_per_sm = *fused_blocks_per_sm = *col_blocks_per_sm = 1;
    dispatch_L<R>(nx, [&](auto LC) {
        constexpr int L = decltype(LC)::value;
        if constexpr (RowCfg<R, L>::SMEM <= kSmemMax) {
            int a = 1, b = 1, c = 1;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_row_forward_fast<R, L>, RowCfg<R, L>::THREADS,
                                                          RowCfg<R, L>::SMEM);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_row_inverse_fast<R, L, 1>, RowCfg<R, L>::THREADS,
                                                          RowCfg<R, L>::SMEM);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, k_row_inverse_fast<R, L, 0>, RowCfg<R, L>::THREADS,
                                                          RowCfg<R, L>::SMEM);
            *fwd_blocks_per_sm = std::max(1, a);
            *inv_blocks_per_sm = std::max(1, b);
            *full_blocks_per_sm = std::max(1, c);
            int d = 1;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d, k_row_fused<R, L>, RowCfg<R, L>::THREADS,
                                                          RowCfg<R, L>::SMEM);
            *fused_blocks_per_sm = std::max(1, d);
        }
    });
    dispatch_L<R>(ny, [&](auto LC) {
        constexpr int L = decltype(LC)::value;
        if constexpr (ColCfg<R, L>::SMEM + kStaticSmemCol <= kSmemMax) {
            int a = 1;
            if (col_direct)
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_column_direct<R, L>, ColCfg<R, L>::THREADS,
                                                              ColDirectCfg<R, L>::SMEM);
            else
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_column_fast<R, L>, ColCfg<R, L>::THREADS,
                                                              ColCfg<R, L>::SMEM);
            *col_blocks_per_sm = std::max(1, a);
        }
    });
}
template void fast_occupancy<float>(int, int, bool, int*, int*, int*, int*, int*);
template void fast_occupancy<double>(int, int, bool, int*, int*, int*, int*, int*);
template cudaError_t launch_fused<float>(const EvalSpec&, const EvalSpec&, const LaunchGeom&, cudaStream_t, int*);
template cudaError_t launch_fused<double>(const EvalSpec&, const EvalSpec&, const LaunchGeom&, cudaStream_t, int*);
template FastCfg fast_config<float>(int, int);
template FastCfg fast_config<double>(int, int);
template cudaError_t build_pass_tables<float>(void*, int, void*, int, cudaStream_t);
template cudaError_t build_pass_tables<double>(void*, int, void*, int, cudaStream_t);
template cudaError_t launch_one<float>(int, const EvalSpec&, const LaunchGeom&, cudaStream_t, int*);
template cudaError_t launch_one<double>(int, const EvalSpec&, const LaunchGeom&, cudaStream_t, int*);
template cudaError_t prepare_eval_kernels<float>(size_t, size_t);
template cudaError_t prepare_eval_kernels<double>(size_t, size_t);
template cudaError_t launch_eval<float>(const EvalSpec&, const LaunchGeom&, cudaStream_t);
template cudaError_t launch_eval<double>(const EvalSpec&, const LaunchGeom&, cudaStream_t);

}  // namespace llg
