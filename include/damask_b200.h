/*
 * damask_b200 — C-ABI of the B200 (sm_100a) implementation of DAMASK's grid
 * mechanical hot path: the basic spectral (FFT) fixed-point scheme with the
 * Gamma-operator convolution (and the spectral polarization scheme), driving the
 * per-voxel phenopowerlaw/Hooke constitutive update (FPI state integration, Lp
 * Newton-Raphson, dP/dF); coordinates, the grid geometry reader and the driver's
 * increment loop.
 *
 * The entry points mirror the Fortran procedures the reference selects through
 * procedure pointers in src/grid/DAMASK_grid.f90:110-119,171-206, so a Fortran
 * host can bind them with ISO_C_BINDING: one bind(C) interface per function,
 * structs as bind(C) derived types, contexts as type(C_PTR).
 *
 * Conventions
 *  - Plain C types only; all arrays are host pointers owned by the caller and
 *    used only for the duration of the call.  Device memory (per-voxel state,
 *    cuFFT plans, scratch) is owned by the context from init to destroy.
 *  - 3x3 tensors are column-major (Fortran order: T11 T21 T31 T12 ...); fields
 *    are voxel-major with x fastest, i.e. reshape(F,[3,3,cells1,cells2,cells3]).
 *    4th-order tensors are column-major 3x3x3x3 (81 doubles).
 *  - Every function returns a status: 0 on success, DMK_STATUS_* (mirroring
 *    src/constants.f90:29-44) for constitutive failures, DMK_ERR_* otherwise.
 *    Nothing is thrown across the ABI.
 *  - A context is not re-entrant; call it from one host thread.
 */
#ifndef DAMASK_B200_H
#define DAMASK_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes (constants.f90:29-44) */
#define DMK_STATUS_OK 0
#define DMK_STATUS_ITERATING 1
#define DMK_STATUS_FAIL_PHASE_MECHANICAL 2
#define DMK_STATUS_FAIL_STATE 3
#define DMK_STATUS_FAIL_DELTASTATE 4
#define DMK_STATUS_FAIL_STRESS 5
#define DMK_STATUS_FAIL_LP_MAXIT 6
#define DMK_STATUS_FAIL_LP_NAN 7
#define DMK_STATUS_FAIL_LP_DGESV 8
/* errors of this library */
#define DMK_ERR_CUDA (-1)
#define DMK_ERR_CUFFT (-2)
#define DMK_ERR_CONFIG (-3)
#define DMK_ERR_ARG (-4)
#define DMK_ERR_STATE (-5)
#define DMK_STATUS_TIMEOUT (-6)
#define DMK_ERR_NOT_CONVERGED (-7)   /* the driver's IO_error 950: no convergence after the cutbacks */

/* precision of the spectral part (FFT, Gamma, field update) */
#define DMK_PRECISION_FP64 0
#define DMK_PRECISION_MIXED 1

/* Phase: Hooke elasticity + phenopowerlaw slip (SI units).
   Keys as in material.yaml, phase_mechanical_elastic.f90:22-84 and
   phase_mechanical_plastic_phenopowerlaw.f90:76-295; per-family arrays. */
typedef struct {
  int lattice;            /* 0 = cF, 1 = cI */
  int n_families;         /* entries used in the per-family arrays */
  int N_sl[4];            /* active systems per family, 1 to 48 in total: the kernels exist for 12, 18,
                             24 and 48; other sums run on the next of these with inert systems */
  double C11, C12, C44;
  double dot_gamma_0[4], n[4], a[4], h_0[4], xi_0[4], xi_inf[4], c_1[4], c_2[4], f_sat[4];
  int n_h;                /* number of h_sl-sl interaction values */
  double h_sl_sl[64];
  int n_nonschmid;        /* cI family-1 non-Schmid coefficients a_non-Schmid (0..6) */
  double a_nonschmid[6];
  double atol_xi, atol_gamma;
} dmk_phase;

/* Numerical parameters: numerics.yaml keys (grid_mech_spectral_basic.f90:130-136,
   spectral_utilities.f90:176-224, phase_mechanical.f90:281-295). */
typedef struct {
  int N_iter_min, N_iter_max;
  double eps_abs_div, eps_rel_div, eps_abs_P, eps_rel_P;
  int update_gamma;
  int divergence_correction;   /* 0 none, 1 size, 2 grid+size */
  int derivative;              /* 0 continuous, 1 central_difference, 2 FWBW_difference (utilities_getFreqDerivative) */
  double r_cutback_min, r_cutback, r_increase, eps_rel_state;
  int N_iter_state_max;
  int N_iter_Lp_max;
  double r_linesearch_Lp, eps_rel_Lp, eps_abs_Lp;
  int f_update_jacobi_Lp;
  int N_iter_Li_max;
  double r_linesearch_Li, eps_rel_Li, eps_abs_Li;
  int f_update_jacobi_Li;
  int snes_type;               /* fixed-point iteration of the residual: 0 Richardson F <- F - r
                                  (PETSc -snes_type nrichardson), 1 Anderson-accelerated */
  int anderson_m;              /* Anderson history depth (1..32) */
  /* mechanical solver, selected by load.yaml solver: mechanical: (DAMASK_grid.f90:171-206):
     0 spectral_basic, 1 spectral_polarization (grid_mech_spectral_polarization.f90) */
  int solver;
  double alpha, beta;          /* polarization parameters: 0 < alpha <= 2, 0 <= beta <= 2 */
  double eps_abs_curl, eps_rel_curl;   /* eps_abs_curl(F), eps_rel_curl(F) (polarization) */
  int snes_max_it;             /* iteration cap of the fixed point: PETSc's -snes_max_it (default 50), which
                                  the reference's PETSc_options can set; 0 means 50 */
} dmk_numerics;

/* tBCmech (grid_utilities.f90:35-39): values/mask column-major, mask 1 = 'x' */
typedef struct {
  double values[9];
  int mask[9];
  int type;               /* 0 none, 1 L, 2 dot_F, 3 F, 4 P, 5 dot_P */
} dmk_bc;

/* tSolutionState (spectral_utilities.f90:77-83) plus diagnostics */
typedef struct {
  int iterationsNeeded;
  int converged;
  int stagConverged;
  int residualEvals;
  double err_div, err_BC;
  double P_av[9];
} dmk_solution_state;

typedef struct dmk_ctx dmk_ctx;

/* Field identifiers for dmk_get_field / dmk_set_field. */
enum {
  DMK_FIELD_F = 0,        /* phase F (3,3,N) */
  DMK_FIELD_P = 1,        /* first Piola-Kirchhoff stress (3,3,N) */
  DMK_FIELD_FE = 2,
  DMK_FIELD_FP = 3,
  DMK_FIELD_LP = 4,
  DMK_FIELD_S = 5,
  DMK_FIELD_XI_SL = 6,    /* (Ns,N) */
  DMK_FIELD_GAMMA_SL = 7, /* (Ns,N) */
  DMK_FIELD_F_LASTINC = 8,
  DMK_FIELD_FI = 9,
  DMK_FIELD_LI = 10,
  DMK_FIELD_F_SOLVER = 11, /* solution field F of the spectral solver */
  DMK_FIELD_O = 12,        /* orientation (4,N): unit quaternion w,x,y,z of the rotational part of Fe,
                              as crystallite_orientations (phase.f90:659-673); get only.  A voxel whose
                              rotation has |det - 1| > 1e-5 makes the call fail with DMK_ERR_STATE
                              (IO_error 402 of rotations.f90:221-222). */
  DMK_FIELD_F_TAU = 13,    /* polarization solver: F_tau and F_tau_lastinc (3,3,N) */
  DMK_FIELD_F_TAU_LASTINC = 14
};

/* Create a context and run grid_mechanical_spectral_basic_init
   (grid_mech_spectral_basic.f90:103-237; mechanical_init phase_mechanical.f90:184-338):
   F := I, one constitutive sweep at dt = 0, Gamma reference stiffness := C_minMaxAvg.
   With num->solver = 1 the context is grid_mech_spectral_polarization instead (init
   grid_mech_spectral_polarization.f90:115-270: also F_tau := 2 I, C_scale := C_minMaxAvg,
   S_scale := invSym3333(C_minMaxAvg)); forward, solution, updateCoords and the restart calls
   then follow that module, with F_tau as a second solution field.  The polarization scheme
   runs its spectral steps in FP64 for either precision.
   materialAt: N entries, 0-based material index; quaternions: 4 per material (w,x,y,z).
   precision: DMK_PRECISION_FP64 or DMK_PRECISION_MIXED. device: CUDA ordinal. */
int dmk_mech_init(dmk_ctx** ctx, const int cells[3], const double geomSize[3], const int* materialAt,
                  int n_materials, const double* quaternions, const dmk_phase* phase,
                  const dmk_numerics* num, int precision, int device);

/* grid_mechanical_spectral_basic_forward, grid_mech_spectral_basic.f90:284-355 */
int dmk_mech_forward(dmk_ctx* ctx, int cutBack, int guess, double dt, double dt_old, double t_remaining,
                     const dmk_bc* deformation, const dmk_bc* stress, const double q_rot[4]);

/* grid_mechanical_spectral_basic_solution, grid_mech_spectral_basic.f90:243-277.
   The residual r(F) is driven to zero by the fixed-point iteration that dmk_numerics.snes_type
   selects: Anderson-accelerated (the default, standing in for the reference's
   -snes_type ngmres) or the Richardson iteration F <- F - r(F) (-snes_type nrichardson). */
int dmk_mech_solution(dmk_ctx* ctx, dmk_solution_state* out);

/* materialpoint_forward -> mechanical_forward, phase_mechanical.f90:987-1002 */
int dmk_materialpoint_forward(dmk_ctx* ctx);

/* grid_mechanical_spectral_basic_updateCoords, grid_mech_spectral_basic.f90:361-372, which
   calls utilities_updateCoords (spectral_utilities.f90:857-968) on the solver's F field:
   cell-centre and node coordinates of the current configuration by integration of F in
   Fourier space (average part Favg times the undeformed position plus the periodic
   fluctuation).  The result replaces discretization_setIPcoords / _setNodeCoords
   (discretization.f90:102-122) and is read with dmk_get_coords. */
int dmk_mech_update_coords(dmk_ctx* ctx);

/* discretization_IPcoords and discretization_NodeCoords (discretization.f90:23-26) as set
   by the last dmk_mech_update_coords; before the first call the undeformed coordinates
   IPcoordinates0 / nodes0 (discretization_grid.f90:270-313).  ip: (3, cells1*cells2*cells3),
   nodes: (3, (cells1+1)*(cells2+1)*(cells3+1)), x fastest; either may be NULL. */
int dmk_get_coords(dmk_ctx* ctx, double* ip, double* nodes);

/* Field transfer to/from host buffers (Fortran layout). */
int dmk_get_field(dmk_ctx* ctx, int field, double* host_out);
int dmk_set_field(dmk_ctx* ctx, int field, const double* host_in);
int dmk_field_size(dmk_ctx* ctx, int field);   /* doubles per voxel, or <0 */

/* Restart data: what grid_mechanical_spectral_basic_restartWrite
   (grid_mech_spectral_basic.f90:378-416) and mechanical_restartWrite
   (phase_mechanical.f90:1248-1261) store.  Per-voxel arrays are host buffers owned by
   the caller, voxel-major: 9 per voxel (3x3 column-major) or 2 Ns per voxel (xi then
   gamma).  F_i and L_i are I and 0 on this path and are not carried. */
typedef struct {
  double* F;             /* solver F (9 N) */
  double* F_lastinc;     /* solver F of the last converged increment (9 N) */
  double* F_phase;       /* phase F ('F' of the phase group, 9 N) */
  double* F_p;           /* (9 N) */
  double* L_p;           /* (9 N) */
  double* omega_plastic; /* plastic state (2 Ns N) */
  double P_aim[9], F_aim[9], F_aim_lastinc[9], F_aimDot[9];
  double C_volAvg[81], C_volAvgLastInc[81];
  double C_minMaxAvg[81];   /* the Gamma reference stiffness in use (C_minMaxAvgRestart) */
  double* F_tau;            /* polarization solver only (else unused): F_tau, F_tau_lastinc (9 N each), */
  double* F_tau_lastinc;    /* grid_mech_spectral_polarization.f90:412-415 */
} dmk_restart;

/* Fill r (caller-allocated arrays) from the context, after a converged increment and
   dmk_materialpoint_forward, as the reference writes its restart file. */
int dmk_restart_write(dmk_ctx* ctx, dmk_restart* r);

/* Resume from r on a freshly initialised context with the same grid and phase, as
   grid_mechanical_spectral_basic_init and mechanical_restartRead do for a restart
   increment (grid_mech_spectral_basic.f90:198-235, phase_mechanical.f90:1267-1280):
   the converged phase state (F0, Fp0, Lp0, state0) and the solver fields and aims are
   loaded, one constitutive sweep at dt = 0 runs at the loaded F (S0 = 0, as the
   reference keeps it), then C_volAvg, C_volAvgLastInc and C_minMaxAvg are taken from r
   and the Gamma operator is set up with C_minMaxAvg. */
int dmk_restart_read(dmk_ctx* ctx, const dmk_restart* r);

/* Restart contract (grid_mech_spectral_basic.f90:378-416): F_aim, F_aim_lastinc,
   F_aimDot, P_aim (9 each), C_volAvg, C_volAvgLastInc, C_minMaxAvg (81 each). */
int dmk_get_aims(dmk_ctx* ctx, double F_aim[9], double F_aim_lastinc[9], double F_aimDot[9],
                 double P_aim[9], double C_volAvg[81], double C_volAvgLastInc[81], double C_minMaxAvg[81]);

/* Operator-level entry points (unit parity).  Inputs/outputs are host arrays.
   utilities_constitutiveResponse, grid_utilities.f90:133-207 */
int dmk_constitutive_response(dmk_ctx* ctx, const double* F, double dt, double* P, double P_av[9],
                              double C_volAvg[81], double C_minMaxAvg[81], int* status);
/* utilities_updateGamma, spectral_utilities.f90:356-395 */
int dmk_update_gamma(dmk_ctx* ctx, const double C[81]);
/* utilities_GammaConvolution, spectral_utilities.f90:436-501 (in place) */
int dmk_gamma_convolution(dmk_ctx* ctx, double* field, const double aim[9]);
/* utilities_divergenceRMS, spectral_utilities.f90:650-691 */
int dmk_divergence_rms(dmk_ctx* ctx, const double* P, double* out);
/* utilities_curlRMS, spectral_utilities.f90:695-757 (the polarization scheme's compatibility
   criterion); uses the solver's scratch buffers, so call it between solutions */
int dmk_curl_rms(dmk_ctx* ctx, const double* F, double* out);
/* phase_mechanical_dPdF, phase_mechanical.f90:1121-1242, for every voxel (81 per voxel) */
int dmk_dPdF(dmk_ctx* ctx, double dt, double* dPdF);

/* Per-voxel iteration counters of the last constitutive sweep: 4 ints per voxel
   (integrateStateFPI iterations, integrateStress Newton iterations, substeps, status). */
int dmk_get_iteration_counts(dmk_ctx* ctx, int* out);
/* Totals of the last dmk_mech_solution: constitutive evaluations, state iterations,
   Newton iterations, residual evaluations. */
int dmk_get_counters(dmk_ctx* ctx, int64_t out[4]);
/* Device time (ms) of the kernels of the last dmk_mech_solution, by stage:
   constitutive, spectral (FFT + Gamma), other. */
int dmk_get_timings(dmk_ctx* ctx, double out[3]);

/* Host-only phase constants (no device needed), crystal_SchmidMatrix_slip
   (crystal.f90:1348-1454) and crystal_interaction_SlipBySlip (crystal.f90:591-902):
   Schmid matrices of the active slip systems (column-major, 9 per system; sense +1/-1,
   with the non-Schmid terms of the phase) and the Ns x Ns hardening matrix (row =
   reacting system).  Return the number of systems Ns, or an error code < 0. */
int dmk_phase_schmid(const dmk_phase* phase, int sense, double* out);
int dmk_phase_interaction(const dmk_phase* phase, double* h);
/* Miller indices of the active slip systems (6 per system: direction d1 d2 d3, plane normal
   n1 n2 n3, the rows of CF_SYSTEMSLIP / CI_SYSTEMSLIP, crystal.f90:43,125) for the 'systems'
   labels of slip outputs (crystal_labels_slip, crystal.f90:1642-1676).  Returns Ns. */
int dmk_phase_slip_systems(const dmk_phase* phase, int* out);

/* Grid geometry files (.vti): the native reader that replaces the reference's C++ reader
   (src/grid/VTI.cpp:417-445: C_VTI_new, C_VTI_readGeometry, C_VTI_readDatasetInt,
   C_VTI_readDatasetReal, C_VTI_delete; descriptors there, pointers and sizes here).  Host code
   only (no device needed).  Labels are the CellData array names in file order; the datasets
   have cells1*cells2*cells3*NumberOfComponents values, x fastest. */
typedef struct dmk_vti dmk_vti;
int dmk_vti_open(const char* path, dmk_vti** out);
int dmk_vti_geometry(const dmk_vti* vti, int cells[3], double size[3], double origin[3]);
/* name (and NumberOfComponents) of label `index`; returns the label count */
int dmk_vti_label(const dmk_vti* vti, int index, char* out, int cap, int* components);
int dmk_vti_read_int(const dmk_vti* vti, const char* label, int64_t* out, int64_t n);
int dmk_vti_read_real(const dmk_vti* vti, const char* label, double* out, int64_t n);
void dmk_vti_close(dmk_vti* vti);

/* The grid driver's increment loop (DAMASK_grid.f90:288-460) for the mechanical field: time steps
   t * math_geometricFraction(r, inc, N), the global cutback (time step halved up to N_cutback_max
   times, then DMK_ERR_NOT_CONVERGED as IO_error 950), the guess flag, restart skipping
   (increments <= restart_inc only advance t), and per (sub)increment the calls forward,
   materialpoint_forward (not after a cutback), solution and, when converged, updateCoords.  The
   plugin is a table of the five procedures (DAMASK_grid.f90:110-119), so the same loop drives this
   library's context (dmk_grid_run_ctx) or any other implementation. */
typedef struct {
  dmk_bc deformation, stress;   /* tBCmech of the load step */
  double q_rot[4];              /* load-case rotation R as a quaternion */
  double t;                     /* duration */
  int N;                        /* increments */
  double r;                     /* geometric ratio of the increments (1: equal) */
  int f_out, f_restart;         /* output and restart frequency (for the callback's use) */
  int estimate_rate;            /* guess the rate of the first increment from the last one */
} dmk_loadstep;
typedef struct {
  int inc;                      /* total increment counter */
  double t;                     /* time at the end of the (sub)increment */
  int cutback_level, converged, iterations, residual_evals;
  int load_step, step_inc;      /* 0-based load step, 1-based increment within it */
  double P_av[9];
} dmk_increment_info;
/* called after every converged (sub)increment; a nonzero return stops the run (returns 0) */
typedef int (*dmk_increment_cb)(const dmk_increment_info* info, void* user);
typedef struct {
  void* ctx;
  int (*forward)(void* ctx, int cutBack, int guess, double dt, double dt_old, double t_remaining,
                 const dmk_bc* deformation, const dmk_bc* stress, const double q_rot[4]);
  int (*solution)(void* ctx, dmk_solution_state* out);
  int (*update_coords)(void* ctx);
  int (*materialpoint_forward)(void* ctx);
} dmk_grid_solver;
int dmk_grid_run(const dmk_grid_solver* solver, const dmk_loadstep* steps, int n_steps, int N_cutback_max,
                 int restart_inc, int max_increments /* <= 0: all */, dmk_increment_cb cb, void* user);
int dmk_grid_run_ctx(dmk_ctx* ctx, const dmk_loadstep* steps, int n_steps, int N_cutback_max, int restart_inc,
                     int max_increments, dmk_increment_cb cb, void* user);

/* Measured FP64 fused-multiply-add throughput of a device in TFLOP/s (8 independent register FMA
   chains per thread, 8 blocks of 256 threads per SM, best of 3 launches of about 10 ms); the
   denominator of the constitutive update's FP64 roofline. */
int dmk_fp64_peak(int device, double* tflops);

/* Autotuner (no counterpart in the reference): times the constitutive evaluation at the context's
   current state (its solver F and time step; call it after dmk_mech_forward, before the solution)
   for every stress-kernel variant (register bound for 2, 3 or 4 resident blocks per SM up to 24
   slip systems; one variant at 48) and voxel-chunk count (1, 2, 4), best of `reps` runs each, and
   keeps the fastest pair.  The fields an evaluation changes are restored after every trial, so the
   solve continues bit for bit as without tuning.  Needs free device memory for a copy of Fp, Lp, S,
   Fe and the state (fails with DMK_ERR_CUDA otherwise, leaving the settings).  report (optional, 36
   doubles): per candidate (blocks per SM, chunks, ms); *n_report candidates.  Basic scheme only. */
int dmk_autotune(dmk_ctx* ctx, int reps, double* report, int* n_report);
int dmk_get_tuning(dmk_ctx* ctx, int* stress_blocks, int* chunks);
int dmk_set_tuning(dmk_ctx* ctx, int stress_blocks, int chunks);

/* Number of kernels of this library launched by the context so far. */
int dmk_get_launches(dmk_ctx* ctx, int64_t* out);
/* Device timer on the context's stream: CUDA events recorded at start and stop;
   stop waits for the stream and returns the elapsed milliseconds. */
int dmk_timer_start(dmk_ctx* ctx);
int dmk_timer_stop(dmk_ctx* ctx, double* ms);

/* Device checkpoints of a context (basic spectral scheme).  No counterpart in the reference,
   whose restart files go through the host (dmk_restart_write): a checkpoint keeps the complete
   solver and phase state in device memory owned by the context (one buffer per slot, made on
   first use, freed by dmk_destroy), and restoring it continues bit for bit as the run from which
   it was saved.  The adjoint's recomputation of checkpointed increments uses them. */
int dmk_checkpoint_save(dmk_ctx* ctx, int slot);
int dmk_checkpoint_restore(dmk_ctx* ctx, int slot);

/* Hand-written adjoint of increments of the basic scheme (no counterpart in the reference), for
   gradients of a loss L(<P>_1, ..., <P>_n) of the volume-averaged stresses with respect to the
   phenopowerlaw parameters theta = (xi_0, xi_inf, h_0, n, a) of each slip family.
   Per increment the converged state solves, per voxel, the Lp Newton system and the fixed point
   of the state integration (phase_mechanical.f90:379-676) and, globally, equilibrium with the
   boundary conditions (grid_mech_spectral_basic.f90:464-521).  The adjoint differentiates the
   converged equations (implicit-function theorem): per voxel the total Jacobian of (P, Fp, xi)
   with respect to (F, Fp0, xi0, theta) through the coupled (Lp, xi) system, and globally the
   transposed equilibrium problem K^T Lambda - G (K = dP/dF), solved with the solver's Gamma
   operator and masked-compliance average, by restarted GMRES to a relative residual of 1e-12.
   Usage (reverse order of the increments, each recomputed from a checkpoint):
     dmk_adj_begin(ctx, n)              n slots for linearization points; state cotangent := 0
     per increment (after dmk_mech_solution converged, before the next dmk_materialpoint_forward):
       dmk_adj_record(ctx, slot)        keeps F, Fp0, xi0, Lp, xi and dt of the increment
     per recorded increment, last first:
       dmk_adj_step(ctx, slot, dL/d<P>, theta_bar, &iterations)   adds the increment's share
     dmk_adj_finish(ctx, theta_bar)     adds the share of xi_0 (the initial state)
   theta_bar[p * 4 + f]: p = 0 xi_0, 1 xi_inf, 2 h_0, 3 n, 4 a; f = slip family.  Requirements:
   load-case rotation R = I, one substep per voxel in every recorded increment (checked), no twins.
   The derivative is that of the exactly converged equations; the forward's tolerances bound how
   well the forward values obey them. */
int dmk_adj_begin(dmk_ctx* ctx, int n_slots);
int dmk_adj_record(dmk_ctx* ctx, int slot);
int dmk_adj_step(dmk_ctx* ctx, int slot, const double P_av_bar[9], double theta_bar[20], int* iterations);
int dmk_adj_finish(dmk_ctx* ctx, double theta_bar[20]);
/* Host-only (no device): the local Jacobian D = d(P, Fp, xi)/d(F, Fp0, xi0, theta) of one voxel
   at the linearization point `point` (F, Fp0, xi0, Lp, xi: 27 + 2 Ns values, 3x3 column-major),
   D row-major (18 + Ns) x (18 + Ns + 4 n_families), theta columns ordered (xi_inf, h_0, n, a) x
   family.  Ns is the compiled slip-system count (12, 18, 24 or 48). */
int dmk_adj_local_jacobian(const dmk_phase* phase, double dt, const double* point, double* D);

/* Batches of independent RVEs (no counterpart in the reference, which solves one grid per
   process).  A batch takes contexts of one phase and one set of constitutive numerics, basic scheme
   (FP64 or mixed form, per context), on one device, and solves one increment of any subset of them
   together:
   dmk_batch_solution does what dmk_mech_solution does for each listed context, with the
   iterations of all of them in shared launches (per fixed-point iteration one CUDA graph for the
   constitutive evaluation of every active context, one cuFFT plan pair per edge size, batched
   aim / Gamma / convergence / Anderson kernels, one host read of the solver scalars).  Each
   context's results equal those of its own dmk_mech_solution call.  The other calls
   (dmk_mech_forward, dmk_materialpoint_forward, ...) stay per context and may put the members of a
   batch at different increments and time steps.  A batch uses the contexts' memory: destroy it
   before them.  which[k] indexes ctxs of dmk_batch_create; out[k] is its solution state. */
typedef struct dmk_batch dmk_batch;
int dmk_batch_create(dmk_batch** out, dmk_ctx* const* ctxs, int n);
int dmk_batch_solution(dmk_batch* batch, const int* which, int n_which, dmk_solution_state* out);
/* out: device ms of the constitutive graphs and of the whole last dmk_batch_solution, graphs
   launched, constitutive passes, fixed-point iterations and dmk_batch_solution calls so far, and the
   host ms of the last call's set-up, iterations, and tangents with counters */
int dmk_batch_stats(dmk_batch* batch, double out[9]);
void dmk_batch_destroy(dmk_batch* batch);
/* The increment loops of all members of a batch, each as dmk_grid_run_ctx (no restart skipping),
   with their solutions computed together: every round, each unfinished member runs up to its next
   solution request (dmk_mech_forward, dmk_materialpoint_forward), one dmk_batch_solution solves
   all requests, and each member goes on (dmk_mech_update_coords, cb, cutback).  Members may fall
   out of step.  steps[k], n_steps[k]: the load steps of member k; max_increments <= 0: all.
   cb(member, info, user) after every converged (sub)increment of a member (nonzero stops that
   member).  status[k]: 0, or DMK_ERR_NOT_CONVERGED when member k did not converge after
   N_cutback_max cutbacks (IO_error 950; it stops, the others go on).  Returns 0, or the first
   error of the library, which stops all members. */
typedef int (*dmk_batch_increment_cb)(int member, const dmk_increment_info* info, void* user);
int dmk_batch_run(dmk_batch* batch, const dmk_loadstep* const* steps, const int* n_steps, int N_cutback_max,
                  int max_increments, dmk_batch_increment_cb cb, void* user, int* status);

/* Volume average <f> of a 9-component field that the caller already holds in device
   memory (9 planes of n_voxels doubles: component c of voxel v at field[c*n_voxels + v]),
   written to mean[9] on the host.  No counterpart in the reference: it exists for hosts
   that may not allocate device memory at the time they need the average (a solver loop
   confined to a memory arena its framework handed out, or a loop where an allocation
   and its implicit device synchronisation are not allowed).  It allocates nothing: its
   partial sums live in a fixed 1.13 MiB device array that every GPU loading the library
   holds until the process exits.  n_voxels is limited to 16,777,216 (256^3); larger
   sizes are rejected with DMK_ERR_ARG.  Every call looks up that array's device address on the
   current device (cudaGetSymbolAddress); the first lookup on a device loads the library's device
   code there, so make the first call on each device before any stream capture.  All calls share
   the array: calls that overlap on the GPU (different streams or threads) race; each call
   overwrites what it uses, so no state carries over.  stream: a cudaStream_t, or NULL for the
   default stream; the call copies the result to `mean` and synchronises `stream` before it returns. */
int dmk_field_mean_noalloc(const double* field, int64_t n_voxels, double mean[9], void* stream);

void dmk_destroy(dmk_ctx* ctx);
const char* dmk_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
