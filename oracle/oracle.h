/*
 * oracle.h — CPU FP64 restatement of llg-sim's uniform-grid LLG hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path
 * (tests/, __graft_entry__.smoke(), bench.py's cpu_baseline / reference arm).
 * The product library never links, loads or calls it.
 *
 * Every routine restates a reference routine (file:line in llg-sim, cited at
 * each definition in oracle.cpp) with the same evaluation order, in FP64,
 * so that it can stand in for the Rust reference, which cannot be compiled in
 * this environment (no Rust toolchain).  The FFT that the reference takes
 * from rustfft 6.4.1 (Cargo.lock:1224) is replaced by the oracle's own FP64
 * mixed-radix FFT; a DFT is defined mathematically, so any correct FFT agrees
 * to round-off, and the tests pin this one against numpy.fft and against a
 * direct real-space convolution.
 *
 * Parity status: pinned against the reference's own known-answer tests
 * (tests/validation.rs, demag_fft_uniform.rs:1261-1293,
 * tests/test_demag_methods.rs) and against independent numerics (numpy FFT,
 * O(N^2) direct demag convolution).  The reference publishes no golden
 * output vectors, so bit-level parity with the Rust binary is unpinned.
 */
#ifndef LLG_ORACLE_H
#define LLG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_grid {
    int64_t nx, ny;
    double dx, dy, dz;
} orc_grid;

typedef struct orc_material {
    double ms, a_ex, k_u;
    double easy_axis[3];
    double dmi;        /* used only when has_dmi != 0 */
    int32_t has_dmi;   /* Option<f64>::is_some() */
    int32_t demag;     /* Material::demag */
} orc_material;

typedef struct orc_params {
    double gamma, alpha, dt;
    double b_ext[3];
} orc_params;

/* FieldMask (effective_field/mod.rs:38-45) */
enum { ORC_EXCH_ANIS = 0, ORC_EXCH_ANIS_DMI = 1, ORC_FULL = 2 };
/* TorqueMetric (relax.rs:32-37) */
enum { ORC_TORQUE_MAX = 0, ORC_TORQUE_MEAN = 1, ORC_TORQUE_RMS = 2, ORC_TORQUE_MEANSQ = 3 };

typedef struct orc_relax_settings {
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
} orc_relax_settings;

typedef struct orc_relax_report {
    int64_t accepted_steps, rejected_steps, torque_checks, torque_field_rebuilds;
    int32_t stop_reason;     /* RelaxStopReason order, relax.rs:40-45 */
    int32_t last_stage_stop; /* -1 = None, else RelaxStageStop order, relax.rs:48-52 */
    int32_t has_final_torque, has_final_torque_max;
    double final_torque, final_torque_max, final_max_err, final_dt;
} orc_relax_report;

/* MinimizeSettings (minimize.rs:20-63); Option<f64> fields as has_* flags.
 * `parallel` and `print_every` change neither the result nor the report and are
 * not carried. */
typedef struct orc_minimize_settings {
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
} orc_minimize_settings;

/* MinimizeReport (minimize.rs:94-104) */
typedef struct orc_minimize_report {
    int64_t iters;
    int32_t converged, stalled, dm_converged, reserved;
    double final_torque, final_max_dm, final_tmean, final_lambda;
} orc_minimize_report;

typedef struct orc_energy {
    double exchange, anisotropy, zeeman, dmi, demag;
} orc_energy;

typedef struct orc_solver orc_solver;

void orc_set_threads(int n);
int orc_get_threads(void);
// 1: also run the per-cell local-term, torque and RK-combination loops in parallel
// (the reference runs them serially); results are identical either way.
void orc_set_parallel_local(int on);
int orc_get_parallel_local(void);

/* geom_mask: nullable; one byte per cell, nonzero = material. */
orc_solver* orc_solver_create(const orc_grid* g, const orc_material* mat, const uint8_t* geom_mask);
void orc_solver_destroy(orc_solver* s);
void orc_solver_invalidate(orc_solver* s);

void orc_build_h_eff(orc_solver* s, const double* m, const double b_ext[3], int field_mask, double* b_out);
void orc_demag_field(orc_solver* s, const double* m, double* b_out);
void orc_step_rk45(orc_solver* s, double* m, orc_params* p, int field_mask, double max_err,
                   double headroom, double dt_min, double dt_max, double* eps, int* accepted,
                   double* dt_used);
void orc_step_rk23_relax(orc_solver* s, double* m, orc_params* p, int field_mask, double max_err,
                         double headroom, double dt_min, double dt_max, double* eps, int* accepted,
                         double* dt_used);
void orc_relax(orc_solver* s, double* m, orc_params* p, int field_mask, orc_relax_settings* st,
               orc_relax_report* rep);
void orc_default_relax_settings(orc_relax_settings* st);
void orc_default_minimize_settings(orc_minimize_settings* st);
void orc_minimize(orc_solver* s, double* m, const orc_params* p, int field_mask, const orc_minimize_settings* st,
                  orc_minimize_report* rep);
/* ---- AMR consumers of the uniform FFT demag (coarse_fft_demag.rs, amr/stepper.rs) ---- */
/* Patch2D (amr/patch.rs:15-80) as the demag consumers read it: coarse_rect in
 * base-grid cells, refinement ratio relative to the base grid, ghost width; m on
 * the patch grid incl. ghosts ((cny*ratio+2*ghost) x (cnx*ratio+2*ghost), AoS);
 * geom_mask_fine on the same grid (NULL: none); parent_material[cny*cnx]
 * (NULL: all material). */
typedef struct orc_amr_patch {
    int64_t i0, j0, cnx, cny, ratio, ghost;
    const double* m;
    const uint8_t* geom_mask_fine;
    const uint8_t* parent_material;
} orc_amr_patch;

int64_t orc_validated_ratio(int64_t nx, int64_t ny, int64_t ratio);
void orc_sample_bilinear(const orc_grid* g, const double* field, double x, double y, double out[3]);
void orc_restrict_m_to_coarse(const orc_grid* base, const double* m_coarse, int32_t n_patches,
                              const orc_amr_patch* patches, double* out);
void orc_restrict_l0_to_demag_grid(int64_t nx_l0, const double* l0_m, int64_t dnx, int64_t dny, int64_t ratio,
                                   double* out);
/* compute_coarse_fft_demag (coarse_fft_demag.rs:367-511) with an explicit
 * coarsening ratio (validated as the reference validates its environment value);
 * b_patches receives every patch's full grid, patches concatenated in order. */
void orc_coarse_fft_demag(const orc_grid* base, const orc_material* mat, const double* m_coarse,
                          int32_t n_patches, const orc_amr_patch* patches, int64_t ratio, double* b_coarse,
                          double* b_patches);
/* The AllFft branch of AmrStepper::compute_demag (amr/stepper.rs:799-835). */
void orc_allfft_demag(const orc_grid* fine, const orc_material* mat, const double* m_fine, const uint8_t* fine_mask,
                      const orc_grid* base, double* b_fine, double* b_coarse);

void orc_energy_breakdown(orc_solver* s, const double* m, const double b_ext[3], orc_energy* out);
double orc_torque_metric(int64_t n, const double* m, const double* b, int metric);

/* demag kernel (demag_fft_uniform.rs:925-1253) */
void orc_kernel_components(double dx, double dy, double dz, int64_t sx, int64_t sy,
                           double accuracy, double out4[4]);
/* k-space kernel of the solver: 4 planes (xx, xy, yy, zz) of px*py interleaved complex */
void orc_demag_kernel_kspace(orc_solver* s, double* out);
void orc_demag_kernel_realspace(const orc_grid* g, int64_t pbc_x, int64_t pbc_y, double* out4);
/* direct O(N^2) real-space convolution of the same kernel (independent of any FFT) */
void orc_demag_field_direct(const orc_grid* g, double ms, const double* m, double* b_out);

/* periodic boundaries (compute_demag_field_pbc, demag.rs:146-156; kernel demag_fft_uniform.rs:941-1005):
 * pbc_x / pbc_y image counts, 0 = open; px = pbc_x ? nx : 2 nx (likewise py) */
void orc_demag_field_pbc(const orc_grid* g, double ms, int64_t pbc_x, int64_t pbc_y, const double* m,
                         double* b_out);
/* unscaled k-space kernel, 4 planes of py*px interleaved complex */
void orc_demag_kernel_kspace_pbc(const orc_grid* g, int64_t pbc_x, int64_t pbc_y, double* out);
/* LLGDMAG v2 k-space cache file (write_kernel_kspace, demag_fft_uniform.rs:279-319); 0 on success */
int orc_write_llgdmag(const orc_grid* g, int64_t pbc_x, int64_t pbc_y, const char* path);
/* direct circular convolution with the wrapped kernel (no FFT) */
void orc_demag_field_direct_pbc(const orc_grid* g, double ms, int64_t pbc_x, int64_t pbc_y, const double* m,
                                double* b_out);

/* 1-D FFT, interleaved complex, unnormalised, forward = exp(-2 pi i k n / N) */
void orc_fft(int64_t n, double* data, int inverse);

/* initial states (initial_states.rs) */
void orc_xorshift_f64(uint64_t seed, int64_t count, double* out);
void orc_init_random(int64_t n, uint64_t seed, double* m);
void orc_init_uniform_with_noise(int64_t n, const double dir[3], double noise, uint64_t seed, double* m);

#ifdef __cplusplus
}
#endif
#endif
