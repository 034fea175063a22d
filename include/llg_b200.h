/*
 * llg_b200.h — C ABI of the B200 (sm_100a) implementation of llg-sim's
 * uniform-grid LLG hot path.
 *
 * Scope: effective field (exchange, uniaxial anisotropy, interfacial DMI,
 * Zeeman, zero-padded FFT demag), the LLG torque, the Dormand–Prince RK45
 * and Bogacki–Shampine RK23 relax steppers, the relax controller and the
 * energy bookkeeping.  Each entry point names the llg-sim (Rust) interface it
 * replaces, as file:line in that project.
 *
 * Conventions
 *  - Host arrays use the reference layout: AoS double[3] per cell, cell index
 *    j*nx + i (grid.rs:27-30, vector_field.rs:24-27).  Masks are one byte per
 *    cell, nonzero = material.
 *  - Every call returns an int status: LLG_OK (0) or a negative LLG_ERR_*.
 *    No exception or abort crosses the ABI; llg_last_error() returns the
 *    message of the calling thread's last failure.
 *  - The caller owns every host array; the library copies in and out.  Device
 *    buffers are owned by the handle that allocated them.
 *  - A handle is not thread-safe; distinct handles are.  Each solver / batch
 *    issues its work on one CUDA stream (llg_*_set_stream may replace it).
 *  - Precision: LLG_PREC_FP32 runs fields, FFTs and stages in FP32 with FP64
 *    kernel construction, error norms, step controllers and convergence
 *    reductions; LLG_PREC_FP64 runs everything in FP64.
 */
#ifndef LLG_B200_H
#define LLG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LLG_B200_ABI_VERSION 2

enum llg_status {
    LLG_OK = 0,
    LLG_ERR_INVALID = -1,   /* bad argument / unsupported size */
    LLG_ERR_CUDA = -2,      /* CUDA runtime error */
    LLG_ERR_TIMEOUT = -3,   /* a bounded device wait gave up */
    LLG_ERR_NONFINITE = -4, /* NaN/Inf in the state or the error norm; the film is retired */
    LLG_ERR_OOM = -5,       /* device allocation failed */
    LLG_ERR_NO_DEVICE = -6  /* no usable sm_100 device */
};

/* FieldMask, effective_field/mod.rs:38-45 */
enum llg_field_mask { LLG_FIELD_EXCH_ANIS = 0, LLG_FIELD_EXCH_ANIS_DMI = 1, LLG_FIELD_FULL = 2 };
/* TorqueMetric, relax.rs:32-37 */
enum llg_torque_metric { LLG_TORQUE_MAX = 0, LLG_TORQUE_MEAN = 1, LLG_TORQUE_RMS = 2, LLG_TORQUE_MEANSQ = 3 };
enum llg_precision { LLG_PREC_FP32 = 0, LLG_PREC_FP64 = 1 };

/* Grid2D, grid.rs:4-11 */
typedef struct llg_grid {
    int64_t nx, ny;
    double dx, dy, dz;
} llg_grid;

/* Material, params.rs:170-184 (demag_method: only the FFT method is on this path) */
typedef struct llg_material {
    double ms, a_ex, k_u;
    double easy_axis[3];
    double dmi;      /* J/m^2, used when has_dmi != 0 (Option<f64>) */
    int32_t has_dmi;
    int32_t demag;   /* Material::demag */
} llg_material;

/* LLGParams, params.rs:213-219 */
typedef struct llg_params {
    double gamma, alpha, dt;
    double b_ext[3];
} llg_params;

/* RelaxSettings, relax.rs:73-105 (Option<f64> fields as has_* + value) */
typedef struct llg_relax_settings {
    double max_err, headroom, dt_min, dt_max;
    int32_t phase1_enabled, phase2_enabled;
    int64_t energy_stride;
    double rel_energy_tol;
    int32_t torque_metric;
    int32_t has_torque_threshold;
    double torque_threshold;
    int64_t torque_check_stride;
    double torque_plateau_rel, torque_plateau_abs;
    int64_t torque_plateau_checks, torque_plateau_min_checks;
    double tighten_factor, tighten_floor;
    int64_t max_accepted_steps;
    int32_t has_final_torque_gate, has_final_torque_gate_max;
    double final_torque_gate, final_torque_gate_max;
    int64_t gate_max_extra_accepted_steps, gate_plateau_fails;
} llg_relax_settings;

/* RelaxReport, relax.rs:55-71; stop_reason in RelaxStopReason order
 * (relax.rs:40-45), last_stage_stop -1 = None else RelaxStageStop order (relax.rs:48-52) */
typedef struct llg_relax_report {
    int64_t accepted_steps, rejected_steps, torque_checks, torque_field_rebuilds;
    int32_t stop_reason;
    int32_t last_stage_stop;
    int32_t has_final_torque, has_final_torque_max;
    double final_torque, final_torque_max, final_max_err, final_dt;
} llg_relax_report;

/* MinimizeSettings (minimize.rs:20-63); the Option<f64> fields dm_stop,
 * dm_torque_gate and dm_torque_gate_max as has_* flags.  `parallel` and
 * `print_every` (minimize.rs:57-62) change neither the result nor the report
 * and are not carried; `reserved` must be 0. */
typedef struct llg_minimize_settings {
    double torque_threshold;
    int64_t max_iters;
    double lambda0, lambda_min, lambda_max, grow, shrink;
    int64_t stall_iters;
    double stall_rel;
    int64_t min_iters_before_stall;
    int32_t has_dm_stop, has_dm_torque_gate, has_dm_torque_gate_max, reserved;
    double dm_stop;
    int64_t dm_samples;
    double dm_torque_gate, dm_torque_gate_max;
    int64_t dm_min_iters;
} llg_minimize_settings;

/* MinimizeReport, minimize.rs:94-104 */
typedef struct llg_minimize_report {
    int64_t iters;
    int32_t converged, stalled, dm_converged, reserved;
    double final_torque, final_max_dm, final_tmean, final_lambda;
} llg_minimize_report;

/* EnergyBreakdown, energy.rs:22-28 (Joule) */
typedef struct llg_energy_breakdown {
    double exchange, anisotropy, zeeman, dmi, demag;
} llg_energy_breakdown;

typedef struct llg_ctx llg_ctx;
typedef struct llg_solver llg_solver;

/* ---------------- context ---------------- */
int llg_ctx_create(int device, llg_ctx** out);
int llg_ctx_destroy(llg_ctx* ctx);
/* Message of the calling thread's last failure (always NUL-terminated). */
int llg_last_error(char* buf, size_t len);
int llg_abi_version(void);

/* ---------------- single film ----------------
 * llg_solver_create builds the demag operator for the grid (the role of
 * get_demag_operator / Demag2D::new, demag_fft_uniform.rs:86-108, 470-634):
 * FP64 face-charge kernel integration and FP64 FFT on the GPU, stored as four
 * real Fourier planes (xx, xy, yy, zz) in the solver precision.
 * geom_mask (nullable) switches on the geometry-aware path (field per
 * build_h_eff_masked_geom, mod.rs:78-101; energy per compute_energy_geom,
 * energy.rs:80-285; vacuum cells pinned at m = 0 through the steppers). */
int llg_solver_create(llg_ctx* ctx, const llg_grid* grid, const llg_material* mat, int32_t precision,
                      const uint8_t* geom_mask, llg_solver** out);
int llg_solver_destroy(llg_solver* s);
/* Use an external CUDA stream (cudaStream_t passed as void*; NULL = own stream). */
int llg_solver_set_stream(llg_solver* s, void* stream);
int llg_solver_sync(llg_solver* s);

/* Upload / download the resident magnetisation (VectorField2D::data).
 * An upload that equals the resident state bit for bit (the state just read
 * back by llg_get_state) keeps the FSAL torque, so a binding that passes the
 * caller's `&mut m` in and out of every step (llg.rs:795) steps exactly as a
 * resident loop does; any other upload drops it. */
int llg_set_state(llg_solver* s, const double* m_aos);
int llg_get_state(llg_solver* s, double* m_aos);
/* Mean magnetisation <m> of the resident state, FP64 reduction on the GPU. */
int llg_mean_m(llg_solver* s, double out3[3]);

/* build_h_eff_masked (effective_field/mod.rs:48-75; _geom variant mod.rs:78-101)
 * evaluated at the resident state; b_out: AoS double[3] per cell (Tesla). */
int llg_build_h_eff(llg_solver* s, const llg_params* params, int32_t field_mask, double* b_out);
/* demag::compute_demag_field (demag.rs:57-64 -> demag_fft_uniform.rs:146-186) at the resident state. */
int llg_compute_demag_field(llg_solver* s, double* b_out);

/* step_llg_rk45_recompute_field_masked_adaptive (llg.rs:795-1026): one attempt
 * on the resident state.  params->dt is read as dt0 and overwritten with the
 * next step size, as the reference mutates LLGParams::dt.  FSAL reuse follows
 * llg.rs:854-867 (valid after an accepted step with the same mask and b_ext);
 * after a rejected attempt the stored k1 of the unchanged state is reused too
 * instead of being evaluated again (same values: k1 = f(m0) of the same m0). */
int llg_step_rk45(llg_solver* s, llg_params* params, int32_t field_mask, double max_err, double headroom,
                  double dt_min, double dt_max, double* eps, int32_t* accepted, double* dt_used);
/* step_llg_rk23_recompute_field_masked_relax_adaptive (llg.rs:278-436). */
int llg_step_rk23_relax(llg_solver* s, llg_params* params, int32_t field_mask, double max_err, double headroom,
                        double dt_min, double dt_max, double* eps, int32_t* accepted, double* dt_used);

/* Device-resident RK45 integration: repeats attempts on the GPU without host
 * round trips until `n_accepted` more steps are accepted or the simulated time
 * reaches t_end, measured from the start of this call (dt is clamped to land on t_end, as the reference drivers do in
 * st_problems/sp4.rs:308-314).  Pass n_accepted < 0 or t_end = +inf to disable
 * either limit.  max_attempts bounds the work. */
int llg_run_rk45(llg_solver* s, llg_params* params, int32_t field_mask, double max_err, double headroom,
                 double dt_min, double dt_max, int64_t n_accepted, double t_end, int64_t max_attempts,
                 int64_t* accepted_out, int64_t* rejected_out, double* t_advanced);

/* relax_with_report (relax.rs:334-768), run by a device-side controller that
 * restates its two phases, torque checks and MaxErr tightening per film;
 * settings->max_err is written back. */
int llg_relax(llg_solver* s, llg_params* params, int32_t field_mask, llg_relax_settings* settings,
              llg_relax_report* report);
void llg_default_relax_settings(llg_relax_settings* st); /* impl Default, relax.rs:107-141 */

/* minimize_damping_only (minimize.rs:107-369): damping-only descent
 * m <- normalize(m + lambda (m x B) x m), one effective-field build per
 * iteration, with the reference's lambda controller, torque threshold, dM stop
 * and stall test, run as a device-resident loop.  params->dt is not used or
 * changed; the resident state is updated in place. */
int llg_minimize(llg_solver* s, const llg_params* params, int32_t field_mask, const llg_minimize_settings* settings,
                 llg_minimize_report* report);
void llg_default_minimize_settings(llg_minimize_settings* st); /* impl Default, minimize.rs:65-92 */

/* compute_energy / compute_energy_geom (energy.rs:66-285) at the resident state. */
int llg_compute_energy(llg_solver* s, const double b_ext[3], llg_energy_breakdown* out);
/* torque_metric_rebuild (relax.rs:192-203): field rebuild + metric, FP64 reduction. */
int llg_torque_metric(llg_solver* s, const llg_params* params, int32_t field_mask, int32_t metric,
                      double* out);

/* Demag operator export: the four real Fourier planes (xx, xy, yy, zz) of
 * K = mu0 * N on kx in [0,nx], ky in [0,ny], as FP64, without the 1/(px*py)
 * scaling (compare with the real part of Demag2D::kxx.. at those indices). */
int llg_demag_kernel_kspace(llg_solver* s, double* out /* 4*(nx+1)*(ny+1) */);

/* ---------------- batches of independent films ----------------
 * Many films (sizes, materials, masks may differ) advance together: every
 * pass of an evaluation is one launch over the work items of all films, each
 * film with its own dt, acceptance and FSAL state (the per-film semantics of
 * the single-film calls above, llg.rs:278-436 / 795-1026).  When all films
 * share one power-of-two shape the register-FFT kernels are used, otherwise the
 * generic shared-memory ones.  Films with identical grids share the demag
 * operator (get_demag_operator keys it by grid, demag_fft_uniform.rs:86).
 * Arrays of params / results are indexed by film; masks is nullable and may
 * hold null entries. */
typedef struct llg_batch llg_batch;
int llg_batch_create(llg_ctx* ctx, int32_t nfilms, const llg_grid* grids, const llg_material* mats,
                     int32_t precision, const uint8_t* const* masks, llg_batch** out);
int llg_batch_destroy(llg_batch* b);
int llg_batch_set_stream(llg_batch* b, void* stream);
int llg_batch_set_state(llg_batch* b, int32_t film, const double* m_aos);
int llg_batch_get_state(llg_batch* b, int32_t film, double* m_aos);
int llg_batch_mean_m(llg_batch* b, double* out /* 3*nfilms */);
/* one RK45 attempt for every film (step_llg_rk45_recompute_field_masked_adaptive, llg.rs:795) */
int llg_batch_step_rk45(llg_batch* b, llg_params* params, int32_t field_mask, double max_err, double headroom,
                        double dt_min, double dt_max, double* eps, int32_t* accepted, double* dt_used);
/* device-resident RK45 for every film until n_accepted more steps or simulated time t_end each */
int llg_batch_run_rk45(llg_batch* b, llg_params* params, int32_t field_mask, double max_err, double headroom,
                       double dt_min, double dt_max, int64_t n_accepted, double t_end, int64_t max_attempts,
                       int64_t* accepted, int64_t* rejected, double* t);
/* relax_with_report (relax.rs:334-768) for every film, driven by a device-side controller */
int llg_batch_relax(llg_batch* b, llg_params* params, int32_t field_mask, const llg_relax_settings* settings,
                    llg_relax_report* reports);
/* minimize_damping_only (minimize.rs:107-369) for every film, one report per film */
int llg_batch_minimize(llg_batch* b, const llg_params* params, int32_t field_mask,
                       const llg_minimize_settings* settings, llg_minimize_report* reports);
int llg_batch_compute_energy(llg_batch* b, const double* b_ext /* 3*nfilms */, llg_energy_breakdown* out);
int llg_batch_launch_count(llg_batch* b, int64_t* out);

/* ---------------- instrumentation (no reference counterpart) ----------------
 * llg_profile_stage: CUDA-event timing of the passes of one RK45 stage
 * evaluation, averaged over `reps` launches on the solver stream; ms4 receives
 * milliseconds per pass: row forward, column, row inverse, and the fused row
 * pass that ends this stage and starts the next (0 when no film uses it).
 * llg_solver_launch_count: kernels this solver has issued so far. */
int llg_profile_stage(llg_solver* s, const llg_params* params, int32_t field_mask, int32_t reps, double* ms4);
/* Register-FFT form the autotuner chose for the row and the column pass.  Row:
 * the radix plan (0 default, 1 alternative with half the registers per thread).
 * Column: 2 * plan + lean, lean = 1 when the pass reads its twiddle tables and
 * kernel columns through L1 instead of staging them in shared memory (more
 * resident blocks).  -1 where the pass runs the generic shared-memory kernels.
 * For a batch, one entry per launch segment (films grouped by length), in
 * segment order; unused entries -2. */
int llg_solver_fft_plans(llg_solver* s, int32_t* row_plan, int32_t* col_plan);
int llg_batch_fft_plans(llg_batch* b, int32_t* row_plans, int32_t n_row, int32_t* col_plans, int32_t n_col);
int llg_solver_launch_count(llg_solver* s, int64_t* out);

/* ---------------- demag field without device allocation ----------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory at the point of use — a host framework whose pool owns every device
 * allocation, a real-time loop that cannot pay allocation latency, code where
 * cudaMalloc is not permitted.  Computes the demag field of one nx x ny film
 * (the field of llg_compute_demag_field) on the current CUDA device and calls
 * no cudaMalloc/cudaFree or allocating library routine.
 *   m             device, FP32 SoA [3][ny][nx] magnetisation (unit vectors)
 *   ms            saturation magnetisation (A/m)
 *   kernel_planes device, FP64 [4][ny+1][nx+1]: the planes llg_demag_kernel_kspace returns
 *   b_out         device, FP32 SoA [3][ny][nx], overwritten with B_demag (T)
 *   stream        cudaStream_t or NULL; the call is asynchronous on it
 * Scratch: one static 32 MiB device array per GPU that loads the library,
 * held until exit; requires 1 <= nx, ny <= 2048 and
 * 24*(nx+1)*ny + 16*(nx+ny) <= 32 MiB (e.g. 1024 x 1024), else LLG_ERR_INVALID.
 * The first call on a device looks up the array's device address and opts the
 * kernels into large shared memory; make that first call before any stream
 * capture.  After cudaDeviceReset the next call on that device repeats this
 * set-up (the reset drops the context the address belonged to), so it too
 * belongs before any capture.  Every call shares the array (no state carries over: each call
 * rewrites all of it before reading), so calls that overlap on the GPU — on
 * different streams or from different threads — race; serialise them. */
int llg_demag_field_noalloc(int64_t nx, int64_t ny, double ms, const float* m, const double* kernel_planes,
                            float* b_out, void* stream);

/* ---------------- initial states (initial_states.rs) ---------------- */
void llg_init_random(int64_t n, uint64_t seed, double* m_aos);                   /* :59-68 */
void llg_init_uniform_with_noise(int64_t n, const double dir[3], double noise,  /* :43-56 */
                                 uint64_t seed, double* m_aos);

/* ---------------------------------------------------------------------------
 * Demag with periodic images and the k-space kernel cache.
 * llg_demag_op is Demag2D (demag_fft_uniform.rs:434-770) for pbc_x / pbc_y
 * periodic images (0 = open boundary in that direction; a periodic direction is
 * not padded: px = pbc_x ? nx : 2 nx, likewise py; px, py <= 4096), FP64.
 * ------------------------------------------------------------------------- */
typedef struct llg_demag_op llg_demag_op;
/* Demag2D::new (:470-634): with a non-NULL cache_path a matching LLGDMAG v2 file is
 * loaded (try_load_kernel_kspace, :322-429), otherwise the kernel is built
 * (build_kernel_realspace_pbc, :941-1005, or the open builder) and written there
 * (write_kernel_kspace, :279-319; a failed write is ignored as in the reference).
 * *loaded (may be NULL) tells which happened. */
int llg_demag_op_create(llg_ctx* ctx, const llg_grid* grid, int64_t pbc_x, int64_t pbc_y, const char* cache_path,
                        int32_t* loaded, llg_demag_op** out);
int llg_demag_op_destroy(llg_demag_op* op);
/* compute_demag_field_pbc (demag.rs:146-156): b_aos = B_demag of Ms m (host AoS, FP64) */
int llg_demag_op_field(llg_demag_op* op, double ms, const double* m_aos, double* b_aos);
/* the four unscaled k-space planes (xx, xy, yy, zz): [4][py][px] complex (re, im) */
int llg_demag_op_kspace(llg_demag_op* op, double* out);
/* write the LLGDMAG v2 cache file (write_kernel_kspace, :279-319) */
int llg_demag_op_save(llg_demag_op* op, const char* path);
/* the reference's cache path for this grid (demag_cache_path, :261-277) */
int llg_demag_cache_filename(const llg_grid* grid, int64_t pbc_x, int64_t pbc_y, char* buf, int64_t len);

/* ---------------------------------------------------------------------------
 * Learned warm start.  No reference counterpart: a six-layer 3x3 convolutional
 * network (32 channels, BF16 weights and activations, FP32 accumulation on the
 * tensor cores) maps (m, inside, B_ext / 0.05 T) to a proposal m that a relax can
 * start from.  Parameters are FP32, per layer W[cout][3][3][cin] then b[cout],
 * with (cin, cout) = (7,32), (32,32) x4, (32,3); llg_warmstart_param_count()
 * gives the total.
 * ------------------------------------------------------------------------- */
/* ---------------- AMR consumers of the uniform FFT demag ----------------
 * Patch2D (amr/patch.rs:15-80) as the demag consumers read it: coarse_rect
 * (i0, j0, cnx, cny) in base-grid cells, refinement ratio relative to the base
 * grid, ghost width; m on the patch grid incl. ghosts, AoS FP64
 * [(cny*ratio + 2*ghost) * (cnx*ratio + 2*ghost)][3]; geom_mask_fine on the same
 * grid (NULL: none); parent_material[cny*cnx] (NULL: all material).  Patch lists
 * are in the reference's processing order (level 1, then level 2, ...), later
 * patches overwriting earlier ones. */
typedef struct llg_amr_patch {
    int64_t i0, j0, cnx, cny, ratio, ghost;
    const double* m;
    const uint8_t* geom_mask_fine;
    const uint8_t* parent_material;
} llg_amr_patch;
typedef struct llg_amr_demag llg_amr_demag;
/* validated_ratio (coarse_fft_demag.rs:118-150) */
int64_t llg_amr_validated_ratio(int64_t nx, int64_t ny, int64_t ratio);
/* cells of a patch grid including ghosts */
int64_t llg_amr_patch_cells(const llg_amr_patch* p);
/* Coarse-FFT demag context for a base (L0) grid: the FFT demag operator of the
 * base grid, or with coarsen_ratio R > 1 of the (nx/R) x (ny/R) demag grid with
 * R dx x R dy cells.  R follows LLG_DEMAG_COARSEN_RATIO's rules: not a power of
 * two, not dividing nx and ny, or leaving fewer than 4 cells -> 1 (read back with
 * llg_amr_demag_ratio). */
int llg_amr_demag_create(llg_ctx* ctx, const llg_grid* base, int64_t coarsen_ratio, llg_amr_demag** out);
int llg_amr_demag_ratio(const llg_amr_demag* h, int64_t* ratio);
int llg_amr_demag_destroy(llg_amr_demag* h);
/* restrict_m_to_coarse (coarse_fft_demag.rs:170-240): un-normalised area averages
 * of the patches over L0 (AoS FP64 base grid in and out). */
int llg_amr_restrict_m(llg_amr_demag* h, const double* m_coarse, int32_t n_patches, const llg_amr_patch* patches,
                       double* out);
/* compute_coarse_fft_demag (coarse_fft_demag.rs:367-511).  b_coarse: base grid AoS;
 * b_patches: every patch's grid incl. ghosts, concatenated in list order
 * (sum of llg_amr_patch_cells x 3 doubles).  Without Material::demag b_coarse is
 * zeroed and b_patches is not written (the reference returns no patch fields). */
int llg_coarse_fft_demag(llg_amr_demag* h, const llg_material* mat, const double* m_coarse, int32_t n_patches,
                         const llg_amr_patch* patches, double* b_coarse, double* b_patches);
/* The AllFft branch of AmrStepper::compute_demag (amr/stepper.rs:799-835): demag of
 * the flattened fine grid (fine_op: llg_demag_op_create with pbc 0, 0), zero where
 * fine_mask is 0 (NULL: no mask), bilinear samples at the base-grid cell centres. */
int llg_amr_allfft_demag(llg_demag_op* fine_op, const llg_material* mat, const double* m_fine,
                         const uint8_t* fine_mask, const llg_grid* base, double* b_fine, double* b_coarse);
/* The same on DEVICE arrays (m_fine, fine_mask or NULL, b_fine, b_coarse), for an
 * AMR code that keeps its hierarchy on the GPU: no host transfer and no
 * allocation, asynchronous on `stream` (cudaStream_t as void*, NULL = default). */
int llg_amr_allfft_demag_device(llg_demag_op* fine_op, const llg_material* mat, const double* d_m_fine,
                                const uint8_t* d_fine_mask, const llg_grid* base, double* d_b_fine,
                                double* d_b_coarse, void* stream);

/* ---------------- OVF 2.0 writers (ovf.rs:17-251) ----------------
 * OvfMeta (ovf.rs:17-45): title, "# Desc:" lines, value labels and units.
 * Formats: LLG_OVF_TEXT = write_ovf2_rectangular_text (:54-151),
 * LLG_OVF_BINARY4 = write_ovf2_rectangular_binary4 (:153-251); byte-identical to
 * the reference's files.  The parent directory is created as needed. */
enum { LLG_OVF_TEXT = 0, LLG_OVF_BINARY4 = 1 };
typedef struct llg_ovf_meta {
    const char* title;
    const char* const* desc_lines;
    int32_t n_desc;
    const char* valuelabels[3];
    const char* valueunits[3];
} llg_ovf_meta;
/* a host field (AoS FP64 [nx*ny][3]) */
int llg_ovf2_write(const char* path, const llg_grid* g, const double* m_aos, const llg_ovf_meta* meta,
                   int32_t format);
/* the solver's resident m; binary4 is packed to f32 on the GPU (12 bytes per cell cross the bus) */
int llg_ovf2_write_state(llg_solver* s, const char* path, const llg_ovf_meta* meta, int32_t format);
int llg_batch_ovf2_write_state(llg_batch* b, int32_t film, const char* path, const llg_ovf_meta* meta,
                               int32_t format);
/* Rust's `{:.<precision>e}` of v (the number format of the OVF headers and text data) */
int llg_ovf_format_exp(double v, int32_t precision, char* buf, int64_t len);

typedef struct llg_warmstart llg_warmstart;
int64_t llg_warmstart_param_count(void);
int llg_warmstart_create(llg_ctx* ctx, const float* params, int64_t n_params, llg_warmstart** out);
int llg_warmstart_destroy(llg_warmstart* w);
/* host buffers: m_aos [nimg][ny*nx][3], mask [nimg][ny*nx] or NULL, b_ext [nimg][3] -> out_aos */
int llg_warmstart_forward(llg_warmstart* w, int64_t nimg, int64_t ny, int64_t nx, const double* m_aos,
                          const uint8_t* mask, const double* b_ext, double* out_aos);
/* replace every film's state by the proposal computed from it on the device; b_ext [n][3] */
int llg_batch_warm_start(llg_batch* b, llg_warmstart* w, const double* b_ext);
/* Bound (in polls) of the network's tensor-core waits; a wait that runs out makes
 * the call return LLG_ERR_TIMEOUT and the next call starts clean. */
int llg_warmstart_set_spin_limit(llg_warmstart* w, int64_t polls);

/* Training of the network on the GPU with the same tensor-core convolutions
 * (forward, input gradient) plus a tensor-core weight-gradient kernel; FP32
 * master weights and Adam on the device.  A minibatch is nimg films of ny x nx
 * cells given by DEVICE pointers: m0 and target FP32 SoA planes with image
 * stride 3*ny*nx (the initial and the relaxed states), mask uint8 [nimg][ny*nx]
 * or NULL, bext double [nimg][3].  The loss is the mean over film cells of
 * 1 - cos(angle) between the normalised output and the target.
 *   llg_wstrain_gradients: loss and the gradient of the mean loss (host FP32,
 *     the parameter layout; grad may be NULL), parameters unchanged;
 *   llg_wstrain_step: one Adam step (lr, beta1, beta2, eps); loss may be NULL,
 *     then the call does not synchronise;
 *   llg_wstrain_get_params: the current FP32 parameters (host). */
typedef struct llg_wstrain llg_wstrain;
int llg_wstrain_create(llg_ctx* ctx, const float* params, int64_t n_params, int64_t max_cells, llg_wstrain** out);
int llg_wstrain_destroy(llg_wstrain* t);
int llg_wstrain_set_spin_limit(llg_wstrain* t, int64_t polls);
int llg_wstrain_gradients(llg_wstrain* t, int64_t nimg, int64_t ny, int64_t nx, const float* m0, const uint8_t* mask,
                          const double* bext, const float* target, double* loss, float* grad);
int llg_wstrain_step(llg_wstrain* t, int64_t nimg, int64_t ny, int64_t nx, const float* m0, const uint8_t* mask,
                     const double* bext, const float* target, float lr, float beta1, float beta2, float eps,
                     double* loss);
int llg_wstrain_sync(llg_wstrain* t);
int llg_wstrain_get_params(llg_wstrain* t, float* out);

#ifdef __cplusplus
}
#endif
#endif /* LLG_B200_H */
