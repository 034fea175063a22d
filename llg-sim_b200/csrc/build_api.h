// build_api.h — host-side entry points shared between the compilation units.
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "../../include/llg_b200.h"
#include "types.cuh"

// Sets the calling thread's message returned by llg_last_error().
void llg_set_error_message(const char* msg);

namespace llg {

FftPlan make_plan(int L);
// Alternative radix plans of length L for the autotuner (the first is make_plan(L)).
std::vector<FftPlan> plan_candidates(int L);
cudaError_t launch_twiddles(void* tw, int L2, bool fp64, cudaStream_t s);
template <typename R>
cudaError_t launch_fft_strided(void* data, int L, const void* tw2, long long elem_stride, int nsig_a,
                               long long stride_a, int nsig_b, long long stride_b, bool inverse, cudaStream_t s);

// Unscaled FP64 k-space kernel planes [4][py][px] complex for pbc_x / pbc_y images.
cudaError_t build_demag_kernel_pbc(int nx, int ny, double dx, double dy, double dz, int pbc_x, int pbc_y,
                                   void* planes_out, cudaStream_t s);
// Builds the demag kernel spectrum of an open-boundary nx x ny grid in FP64 on
// the GPU.  khat_out: (nx+1)*(ny+1) real4 in the solver precision, scaled by
// 1/(4 nx ny), one column of ny+1 entries per kx; with split_columns (even ny)
// each column holds its even ky (0, 2, .., ny) and then its odd ky (1, 3, ..,
// ny-1), the order in which the register-FFT column pass reads them (khat_index).
// k64_out_dev: 4*(ny+1)*(nx+1) doubles, unscaled, layout [c][ky][kx].
// Synchronises the stream.
cudaError_t build_demag_kernel(int nx, int ny, double dx, double dy, double dz, bool fp64_out, void* khat_out,
                               double* k64_out_dev, cudaStream_t s, bool split_columns = false);


// The demag operator of llg_demag_op_create applied to a device AoS FP64 m on
// stream s (the input is read before the output is written, so they may alias).
int demag_op_apply_device(llg_demag_op* op, double ms, const double* d_m_aos, double* d_b_aos, cudaStream_t s);
void demag_op_info(const llg_demag_op* op, int* device, llg_grid* g, int* pbc_x, int* pbc_y);

// OVF 2.0 binary4 file of a packed payload (3*nx*ny f32, x, y, z per cell).
int ovf2_write_packed(const char* path, const llg_grid* g, const float* payload, const llg_ovf_meta* meta);

// Launch geometry of one film set.
struct LaunchGeom {
    const FilmDev* films;
    const WorkItem* row_items;
    int n_row_items;
    const WorkItem* col_items;
    int n_col_items;
    size_t smem_row;
    size_t smem_col;
    int grid_row;     // row-forward pass (and generic row kernels)
    int grid_rinv;    // register-FFT row-inverse pass, lean epilogue
    int grid_rfull;   // register-FFT row-inverse pass, full epilogue
    int grid_col;
    int grid_fused;   // fused row pass (k_row_fused)
    bool any_demag;
    bool fuse_rows;   // end a stage and start the next in one row pass where possible
    int row_var;      // register-FFT radix plan of the row kernels (FPlan V)
    int col_var;      // column kernel form: 2 * register-FFT radix plan (FPlan V) + lean form (0 / 1)
    int fast_row;     // register-FFT row kernels for L = nx (0: generic kernels)
    int fast_col;     // register-FFT column kernel for L = ny (0: generic kernel)
    int row_threads;
    int col_threads;
};

// Register-FFT configuration for a film size per radix plan v (0 default, 1
// alternative): rows per block T, columns per block NC, threads, shared memory,
// pass-table sizes; ok_row / ok_col = false where the size has no such kernel.
struct FastCfg {
    bool ok_row[2], ok_col[2];
    int T[2], NC[2], row_threads[2], col_threads[2];
    size_t smem_row[2], smem_col[2];
    int twp_row_size[2], twp_col_size[2];
};
template <typename R>
FastCfg fast_config(int nx, int ny);
// Resident blocks per SM of the fast kernels of the given plans (after prepare_eval_kernels).
template <typename R>
void fast_occupancy(int nx, int ny, int row_var, int col_var, int* fwd_blocks_per_sm, int* inv_blocks_per_sm,
                    int* full_blocks_per_sm, int* fused_blocks_per_sm, int* col_blocks_per_sm);
// Pass twiddle tables of the register FFT of length L, plan v.
template <typename R>
cudaError_t build_pass_tables(void* out, int L, int v, cudaStream_t s);
// Whether stage si's row inverse and stage sf's row forward can run as one fused
// row pass on segment g (register-FFT rows, lean epilogue, sf's combination ends
// with si's torque).
bool can_fuse(const EvalSpec& si, const EvalSpec& sf, const LaunchGeom& g);
template <typename R>
cudaError_t launch_fused(const EvalSpec& si, const EvalSpec& sf, const LaunchGeom& g, cudaStream_t s,
                         int* nk = nullptr);
template <typename R>
cudaError_t launch_eval(const EvalSpec& spec, const LaunchGeom& g, cudaStream_t s);
template <typename R>
cudaError_t prepare_eval_kernels(size_t smem_row, size_t smem_col);
// Launches one pass of an evaluation: 0 = row forward, 1 = column, 2 = row inverse
// (on the register-FFT path with the streaming stage kernels around them); adds the
// number of kernels launched to *nk when nk is not null.
template <typename R>
cudaError_t launch_one(int which, const EvalSpec& spec, const LaunchGeom& g, cudaStream_t s, int* nk = nullptr);

// Learned warm-start network (conv_tc.cu).
namespace ws {
struct Net;
long long net_param_count();
cudaError_t net_create(const float* params, long long n, int device, Net** out);
void net_destroy(Net* net);
int net_error(Net* net);
void net_set_spin_limit(Net* net, long long polls);
template <typename R>
cudaError_t net_apply(Net* net, const R* m_in, R* m_out, const uint8_t* mask, const double* bext_host, int nimg,
                      int ny, int nx, cudaStream_t s);
}  // namespace ws

}  // namespace llg
