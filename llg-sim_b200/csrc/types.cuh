// types.cuh — device-side data structures shared by the kernels and the host driver.
//
// Layout in HBM (per film):
//   m, stage states, torques k : SoA planes [3][ny][nx] of `real` (cell j*nx+i)
//   spectrum X                 : [3][nx+1][ny] complex, column-major per kx so that
//                                the y-pass reads whole columns contiguously
//   kernel spectrum Khat       : [nx+1][ny+1] of real4 (xx, xy, yy, zz), real
//                                Fourier planes of K = mu0*N folded by parity and
//                                pre-scaled by 1/(px*py)
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace llg {

constexpr int kMaxRadices = 24;

// Radix plan for a shared-memory FFT of length L (product of radices).
struct FftPlan {
    int L;
    int npass;
    int radix[kMaxRadices];
};

// Logical buffer ids resolved per film at run time (parity `cur` swaps the
// accepted state m0 <-> m7 and the FSAL torque k1 <-> k7 on acceptance).
enum MBuf : int { MB_M0 = 0, MB_M7 = 1, MB_S0 = 2, MB_S1 = 3 };
enum KBuf : int { KB_NONE = 0, KB_K1 = 1, KB_K2, KB_K3, KB_K4, KB_K5, KB_K6, KB_K7 = 7 };

// RHS_MINIMIZE: one damping-only descent update m' = normalize(m + lambda (m x B) x m)
// written to the other parity buffer (minimize.rs:216-256)
enum RhsMode : int { RHS_LLG = 0, RHS_RELAX = 1, RHS_FIELD = 2, RHS_ENERGY = 3, RHS_TORQUE = 4, RHS_MINIMIZE = 5 };
enum ErrMode : int { ERR_NONE = 0, ERR_RK45 = 1, ERR_RK23 = 2 };
// Requests of the device-side relax and minimiser controllers.
enum ReqKind : int { REQ_NONE = 0, REQ_ENERGY = 1, REQ_TORQUE = 2, REQ_STEP = 3, REQ_MINIMIZE = 4 };

// Slots of the per-block FP64 partial reductions.
enum RedSlot : int {
    RED_E_EX = 0, RED_E_AN, RED_E_ZEE, RED_E_DMI, RED_E_DEMAG,
    RED_TSUM, RED_TSUM2, RED_TMAX, RED_MX, RED_MY, RED_MZ,
    RED_NSLOT
};

// Per-film integrator / controller state (device resident, FP64).
struct StepState {
    double dt;          // trial step of the next attempt (LLGParams::dt)
    double t;           // simulated time advanced by accepted steps
    double t_end;       // driver target time (+inf = none)
    double max_err, headroom, dt_min, dt_max;
    double eps, dt_used;
    unsigned long long err_bits;  // running max of the per-cell error norm (FP64 bit pattern)
    long long n_acc, n_rej;
    long long target_acc;         // stop after this many accepted steps (<0 = none)
    long long attempts_left;      // bound on device-side attempts
    int cur;
    int fsal_valid;
    int accepted;
    int active;
    int err_code;
    int order;                    // 5 for RK45, 3 for RK23 (controller exponent 1/order)
    int req;                      // request of the device relax controller (ReqKind)
    double lam;                   // minimiser pseudo-step lambda of the next update
    double red[RED_NSLOT];        // finalised reductions of the last reduction pass
};

// Per-film description: geometry, material coefficients, buffers.
struct FilmDev {
    int nx, ny;
    int rows_per_block;           // T
    int nblk;                     // row blocks = ceil(ny / T)
    double dx, dy, dz;
    double ms, a_ex, k_u, dmi;
    double exch;                  // 2A/Ms   (0 = exchange off)
    double eta;                   // D/(2A)  chiral-ghost coupling
    int has_eta;                  // exchange uses chiral ghosts (Material::dmi is Some(d != 0))
    int dmi_avail;                // Material::dmi is Some and DMI field term can run
    double dmi_pref;              // 2D/Ms
    double anis;                  // 2Ku/Ms  (0 = anisotropy off)
    double inv_dx2, inv_dy2;      // 1/dx^2, 1/dy^2 (exchange Laplacian)
    double half_inv_dx, half_inv_dy;   // 1/(2dx), 1/(2dy) (DMI central differences)
    double u[3];
    double bext[3];
    double gamma, alpha;
    int demag_mat;                // Material::demag
    int has_mask;
    FftPlan plan_row;             // length nx
    FftPlan plan_col;             // length ny
    void* m[2];                   // accepted-state ping-pong
    void* ms_buf[2];              // stage-state ping-pong
    void* k[8];                   // k[1..7]; k[1]/k[7] swap with parity
    void* bout;                   // field output (RHS_FIELD)
    void* bdem;                   // demag field planes between the split row-inverse and torque kernels
    void* X;                      // spectrum scratch
    const void* Khat;             // kernel spectrum
    const uint8_t* mask;
    const void* tw_row;           // exp(-2 pi i k / (2nx)), k < 2nx
    const void* tw_col;           // exp(-2 pi i k / (2ny)), k < 2ny
    const void* twp_row[2];       // register-FFT pass tables for length nx, per radix plan (fast path)
    const void* twp_col[2];       // register-FFT pass tables for length ny, per radix plan (fast path)
    double* red_part;             // [nblk][RED_NSLOT] per-block partial reductions
    StepState* st;
};

// One field evaluation inside an integrator step.
struct EvalSpec {
    int m_in;                     // logical buffer holding / receiving the stage state
    int nterm;                    // number of torques in the combination (0: m_in is used as is)
    int kidx[6];
    double a[6];                  // m_s = normalize(m0 + sum dt*a_q k_q)
    int k_out;                    // logical torque buffer written (KB_NONE: none)
    int rhs;                      // RhsMode
    int err;                      // ErrMode
    int demag;                    // include demag in this evaluation
    int dmi;                      // include the DMI field term (FieldMask admits it)
    int local;                    // include the local terms (0: demag field only)
    int skip_if_fsal;             // skip when the film's FSAL torque is valid
    int reduce;                   // write per-block reductions (torque / energy / mean m)
    int req;                      // run only for films whose StepState::req equals this (0: always)
    // Error-norm weights over k1..k7: wb = solution weights b_q, wh = embedded
    // weights bhat_q (RK45: torques, llg.rs:948-997; RK23: states, llg.rs:356-401)
    double wb[8];
    double wh[8];
};

// Work item of a (possibly persistent) launch: film and row/column block.
struct WorkItem {
    int film;
    int blk;
};

}  // namespace llg
