// eval_kernels.cu — instantiation and launch of the per-evaluation kernels for
// FP32 and FP64.
#include "build_api.h"
#include "field_kernels.cuh"

namespace llg {

template <typename R>
cudaError_t prepare_eval_kernels(size_t smem_row, size_t smem_col) {
    cudaError_t e;
    e = cudaFuncSetAttribute(k_row_forward<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_row_inverse<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_column<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_col);
    return e;
}

template <typename R>
cudaError_t launch_eval(const EvalSpec& spec, const LaunchGeom& g, cudaStream_t s) {
    k_row_forward<R><<<g.grid_row, 256, g.smem_row, s>>>(g.films, g.row_items, g.n_row_items, spec);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (spec.demag && g.any_demag) {
        k_column<R><<<g.grid_col, 256, g.smem_col, s>>>(g.films, g.col_items, g.n_col_items, spec);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    k_row_inverse<R><<<g.grid_row, 256, g.smem_row, s>>>(g.films, g.row_items, g.n_row_items, spec);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_one(int which, const EvalSpec& spec, const LaunchGeom& g, cudaStream_t s) {
    if (which == 0) k_row_forward<R><<<g.grid_row, 256, g.smem_row, s>>>(g.films, g.row_items, g.n_row_items, spec);
    else if (which == 1) k_column<R><<<g.grid_col, 256, g.smem_col, s>>>(g.films, g.col_items, g.n_col_items, spec);
    else k_row_inverse<R><<<g.grid_row, 256, g.smem_row, s>>>(g.films, g.row_items, g.n_row_items, spec);
    return cudaGetLastError();
}

template cudaError_t launch_one<float>(int, const EvalSpec&, const LaunchGeom&, cudaStream_t);
template cudaError_t launch_one<double>(int, const EvalSpec&, const LaunchGeom&, cudaStream_t);
template cudaError_t prepare_eval_kernels<float>(size_t, size_t);
template cudaError_t prepare_eval_kernels<double>(size_t, size_t);
template cudaError_t launch_eval<float>(const EvalSpec&, const LaunchGeom&, cudaStream_t);
template cudaError_t launch_eval<double>(const EvalSpec&, const LaunchGeom&, cudaStream_t);

}  // namespace llg
