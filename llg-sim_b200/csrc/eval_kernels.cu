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

// f(L, V) for a power-of-two length L and radix plan V that exist (FPlan::ok).
template <typename R, typename F>
bool dispatch_LV(int L, int V, F&& f) {
    bool done = false;
    dispatch_L<R>(L, [&](auto LC) {
        constexpr int LL = decltype(LC)::value;
        if (V == 0) {
            f(LC, std::integral_constant<int, 0>{});
            done = true;
        } else if constexpr (FPlan<R, LL, 1>::ok) {
            f(LC, std::integral_constant<int, 1>{});
            done = true;
        }
    });
    return done;
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
    for (int v = 0; v < 2; ++v) {
        bool okr = dispatch_LV<R>(nx, v, [&](auto LC, auto VC) {
            constexpr int L = decltype(LC)::value, V = decltype(VC)::value;
            c.T[v] = RowCfg<R, L, V>::T;
            c.row_threads[v] = RowCfg<R, L, V>::THREADS;
            c.smem_row[v] = RowCfg<R, L, V>::SMEM;
            c.twp_row_size[v] = TwTab<R, L, V>::size;
        });
        bool okc = dispatch_LV<R>(ny, v, [&](auto LC, auto VC) {
            constexpr int L = decltype(LC)::value, V = decltype(VC)::value;
            c.NC[v] = ColCfg<R, L, V>::NC;
            c.col_threads[v] = ColCfg<R, L, V>::THREADS;
            c.smem_col[v] = ColCfg<R, L, V>::SMEM;
            c.twp_col_size[v] = TwTab<R, L, V>::size;
        });
        // The register-FFT row kernels move the spectrum of consecutive rows as 16-byte
        // pieces of the column-major X[c][kx][j]: in FP32 a piece is two rows, so the
        // column stride ny must be even for every piece to start on a 16-byte boundary.
        c.ok_row[v] = okr && c.smem_row[v] <= kSmemMax && (sizeof(R) == 8 || ny % 2 == 0);
        c.ok_col[v] = okc && c.smem_col[v] + kStaticSmemCol <= kSmemMax;
    }
    return c;
}

template <typename R>
cudaError_t build_pass_tables(void* out, int L_, int v, cudaStream_t s) {
    cudaError_t err = cudaSuccess;
    dispatch_LV<R>(L_, v, [&](auto LC, auto VC) {
        constexpr int L = decltype(LC)::value, V = decltype(VC)::value;
        if (TwTab<R, L, V>::size > 0) {
            k_pass_tables<R, L, V><<<(TwTab<R, L, V>::size + 255) / 256, 256, 0, s>>>(reinterpret_cast<cx<R>*>(out));
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
    // fast kernels: every instantiation whose shared memory fits; the whole unified
    // L1/shared array as shared memory, so that occupancy is bounded by registers
    // and the blocks' own shared memory only
    auto set_all = [&](auto LC, auto VC) {
        constexpr int L = decltype(LC)::value, V = decltype(VC)::value;
        auto both = [](const void* f, int bytes) {
            cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
            cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        };
        if constexpr (RowCfg<R, L, V>::SMEM <= kSmemMax) {
            constexpr int sm = (int)RowCfg<R, L, V>::SMEM;
            both((const void*)k_row_forward_fast<R, L, V>, sm);
            both((const void*)k_row_inverse_fast<R, L, 0, V>, sm);
            both((const void*)k_row_inverse_fast<R, L, 1, V>, sm);
            both((const void*)k_row_inverse_fast<R, L, 2, V>, sm);
            both((const void*)k_row_fused<R, L, V>, sm);
        }
        if constexpr (ColCfg<R, L, V>::SMEM + kStaticSmemCol <= kSmemMax) {
            both((const void*)k_column_fast<R, L, V, false>, (int)ColCfg<R, L, V, false>::SMEM);
            both((const void*)k_column_fast<R, L, V, true>, (int)ColCfg<R, L, V, true>::SMEM);
        }
    };
    for (int L : {16, 32, 64, 128, 256, 512, 1024, 2048})
        for (int v = 0; v < 2; ++v) dispatch_LV<R>(L, v, set_all);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_one(int which, const EvalSpec& spec, const LaunchGeom& g, cudaStream_t s, int* nk) {
    int count = 0;
    if (which == 0 || which == 2) {
        if (g.fast_row) {
            dispatch_LV<R>(g.fast_row, g.row_var, [&](auto LC, auto VC) {
                constexpr int L = decltype(LC)::value, V = decltype(VC)::value;
                if constexpr (RowCfg<R, L, V>::SMEM <= kSmemMax) {
                    using C = RowCfg<R, L, V>;
                    if (which == 0) {
                        k_row_forward_fast<R, L, V><<<g.grid_row, C::THREADS, C::SMEM, s>>>(g.films, g.row_items,
                                                                                           g.n_row_items, spec);
                        ++count;
                    } else if (lean_epilogue(spec) || lean_err45_epilogue(spec)) {
                        // transform only, then the torque epilogue as a streaming kernel
                        constexpr int CPI = C::T * L;
                        const long long cells = (long long)g.n_row_items * CPI;
                        k_row_inverse_fast<R, L, 1, V><<<g.grid_rinv, C::THREADS, C::SMEM, s>>>(
                            g.films, g.row_items, g.n_row_items, spec);
                        if (lean_err45_epilogue(spec))
                            k_stage_torque<R, true><<<stage_grid(cells), 256, 0, s>>>(g.films, g.row_items,
                                                                                        g.n_row_items, CPI, spec);
                        else
                            k_stage_torque<R, false><<<stage_grid(cells), 256, 0, s>>>(g.films, g.row_items,
                                                                                         g.n_row_items, CPI, spec);
                        count += 2;
                    } else if (spec.rhs == RHS_MINIMIZE) {
                        k_row_inverse_fast<R, L, 2, V><<<g.grid_rfull, C::THREADS, C::SMEM, s>>>(
                            g.films, g.row_items, g.n_row_items, spec);
                        ++count;
                    } else {
                        k_row_inverse_fast<R, L, 0, V><<<g.grid_rfull, C::THREADS, C::SMEM, s>>>(
                            g.films, g.row_items, g.n_row_items, spec);
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
            // col_var = 2 * radix plan + lean form
            dispatch_LV<R>(g.fast_col, g.col_var / 2, [&](auto LC, auto VC) {
                constexpr int L = decltype(LC)::value, V = decltype(VC)::value;
                if constexpr (ColCfg<R, L, V>::SMEM + kStaticSmemCol <= kSmemMax) {
                    if (g.col_var % 2)
                        k_column_fast<R, L, V, true><<<g.grid_col, ColCfg<R, L, V, true>::THREADS,
                                                       ColCfg<R, L, V, true>::SMEM, s>>>(g.films, g.col_items,
                                                                                         g.n_col_items, spec);
                    else
                        k_column_fast<R, L, V, false><<<g.grid_col, ColCfg<R, L, V, false>::THREADS,
                                                        ColCfg<R, L, V, false>::SMEM, s>>>(g.films, g.col_items,
                                                                                           g.n_col_items, spec);
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
    dispatch_LV<R>(g.fast_row, g.row_var, [&](auto LC, auto VC) {
        constexpr int L = decltype(LC)::value, V = decltype(VC)::value;
        if constexpr (RowCfg<R, L, V>::SMEM <= kSmemMax) {
            using C = RowCfg<R, L, V>;
            k_row_fused<R, L, V><<<g.grid_fused, C::THREADS, C::SMEM, s>>>(g.films, g.row_items, g.n_row_items, si,
                                                                           sf);
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
void fast_occupancy(int nx, int ny, int row_var, int col_var, int* fwd_blocks_per_sm, int* inv_blocks_per_sm,
                    int* full_blocks_per_sm, int* fused_blocks_per_sm, int* col_blocks_per_sm) {
    *fwd_blocks_per_sm = *inv_blocks_per_sm = *full_blocks_per_sm = *fused_blocks_per_sm = *col_blocks_per_sm = 1;
    dispatch_LV<R>(nx, row_var, [&](auto LC, auto VC) {
        constexpr int L = decltype(LC)::value, V = decltype(VC)::value;
        if constexpr (RowCfg<R, L, V>::SMEM <= kSmemMax) {
            using C = RowCfg<R, L, V>;
            int a = 1, b = 1, c = 1, d = 1;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_row_forward_fast<R, L, V>, C::THREADS, C::SMEM);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_row_inverse_fast<R, L, 1, V>, C::THREADS, C::SMEM);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, k_row_inverse_fast<R, L, 0, V>, C::THREADS, C::SMEM);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d, k_row_fused<R, L, V>, C::THREADS, C::SMEM);
            *fwd_blocks_per_sm = std::max(1, a);
            *inv_blocks_per_sm = std::max(1, b);
            *full_blocks_per_sm = std::max(1, c);
            *fused_blocks_per_sm = std::max(1, d);
        }
    });
    dispatch_LV<R>(ny, col_var / 2, [&](auto LC, auto VC) {
        constexpr int L = decltype(LC)::value, V = decltype(VC)::value;
        if constexpr (ColCfg<R, L, V>::SMEM + kStaticSmemCol <= kSmemMax) {
            int a = 1;
            if (col_var % 2)
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_column_fast<R, L, V, true>,
                                                              ColCfg<R, L, V, true>::THREADS,
                                                              ColCfg<R, L, V, true>::SMEM);
            else
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_column_fast<R, L, V, false>,
                                                              ColCfg<R, L, V, false>::THREADS,
                                                              ColCfg<R, L, V, false>::SMEM);
            *col_blocks_per_sm = std::max(1, a);
        }
    });
}
template void fast_occupancy<float>(int, int, int, int, int*, int*, int*, int*, int*);
template void fast_occupancy<double>(int, int, int, int, int*, int*, int*, int*, int*);
template FastCfg fast_config<float>(int, int);
template FastCfg fast_config<double>(int, int);
template cudaError_t build_pass_tables<float>(void*, int, int, cudaStream_t);
template cudaError_t build_pass_tables<double>(void*, int, int, cudaStream_t);
template cudaError_t launch_one<float>(int, const EvalSpec&, const LaunchGeom&, cudaStream_t, int*);
template cudaError_t launch_one<double>(int, const EvalSpec&, const LaunchGeom&, cudaStream_t, int*);
template cudaError_t launch_fused<float>(const EvalSpec&, const EvalSpec&, const LaunchGeom&, cudaStream_t, int*);
template cudaError_t launch_fused<double>(const EvalSpec&, const EvalSpec&, const LaunchGeom&, cudaStream_t, int*);
template cudaError_t prepare_eval_kernels<float>(size_t, size_t);
template cudaError_t prepare_eval_kernels<double>(size_t, size_t);
template cudaError_t launch_eval<float>(const EvalSpec&, const LaunchGeom&, cudaStream_t);
template cudaError_t launch_eval<double>(const EvalSpec&, const LaunchGeom&, cudaStream_t);

}  // namespace llg
