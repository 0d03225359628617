/*
 * ORACLE — test infrastructure only.
 *
 * A CPU FP64 restatement of the DAMASK grid-mechanics hot path (basic spectral
 * scheme + phenopowerlaw/Hooke constitutive update).  It exists so that tests,
 * the package smoke check and the benchmark's CPU-baseline leg have something
 * to compare the CUDA product against.  Nothing in the product links, imports
 * or calls it.
 *
 * Every function names the reference file:line it restates.  Tensors follow
 * Fortran semantics: M3 a[i][j] is M(i+1,j+1); fields are stored per voxel as
 * column-major 3x3 blocks (F11 F21 F31 F12 ...), voxels x-fastest.
 *
 * Pinning: the restatement reproduces the reference's stored regression result
 * (tests/integration/resources/plastic_detect_changes, phenopowerlaw bcc with
 * non-Schmid terms, 150 increments; xi_sl and gamma_sl of increments 75 and 150)
 * at the reference test's tolerance (tests/test_golden_17grains.py), and the
 * spectral self-test invariants of spectral_utilities.f90:974-1108.  The
 * reference's solver uses PETSc SNES NGMRES, which is third-party and absent;
 * the fixed point here is Anderson acceleration (Walker-Ni type II) or the
 * Richardson form of the same residual, so iteration counts are pinned only
 * against this restatement.
 */
#pragma once
#include <cstdint>

extern "C" {

/* Phase definition (one phase, phenopowerlaw slip + Hooke), SI units. */
typedef struct {
  int lattice;            /* 0 = cF, 1 = cI */
  int n_families;
  int N_sl[4];
  double C11, C12, C44;
  double dot_gamma_0[4], n[4], a[4], h_0[4], xi_0[4], xi_inf[4], c_1[4], c_2[4], f_sat[4];
  int n_h;
  double h_sl_sl[64];
  int n_nonschmid;        /* cI family-1 non-Schmid coefficients (0..6) */
  double a_nonschmid[6];
  double atol_xi, atol_gamma;
} orc_phase;

typedef struct {
  int N_iter_min, N_iter_max;
  double eps_abs_div, eps_rel_div, eps_abs_P, eps_rel_P;
  int update_gamma;
  int divergence_correction;   /* 0 none, 1 size, 2 grid+size */
  int derivative;              /* 0 continuous, 1 central difference, 2 FWBW difference */
  double r_cutback_min, r_cutback, r_increase, eps_rel_state;
  int N_iter_state_max;
  int N_iter_Lp_max;
  double r_linesearch_Lp, eps_rel_Lp, eps_abs_Lp;
  int f_update_jacobi_Lp;
  int N_iter_Li_max;
  double r_linesearch_Li, eps_rel_Li, eps_abs_Li;
  int f_update_jacobi_Li;
  int snes_type;               /* 0 Richardson (nrichardson), 1 Anderson-accelerated */
  int anderson_m;              /* Anderson history depth */
  int solver;                  /* 0 spectral_basic, 1 spectral_polarization */
  double alpha, beta;          /* polarization scheme parameters */
  double eps_abs_curl, eps_rel_curl;
  int snes_max_it;           /* PETSc -snes_max_it (0: PETSc's default 50) */
} orc_numerics;

typedef struct {
  double values[9];   /* column-major 3x3 */
  int mask[9];        /* 1 = component not prescribed ('x') */
  int type;           /* 0 none, 1 L, 2 dot_F, 3 F, 4 P, 5 dot_P */
} orc_bc;

typedef struct {
  int iterationsNeeded;
  int converged;
  int stagConverged;
  int residualEvals;
  double err_div, err_BC;
  double P_av[9];
} orc_solution;

typedef struct orc_ctx orc_ctx;

orc_ctx* orc_create(const int cells[3], const double geomSize[3], const int* materialAt,
                    int n_materials, const double* quaternions, const orc_phase* phase,
                    const orc_numerics* num, int n_threads);
void orc_destroy(orc_ctx*);

/* grid_mechanical_spectral_basic_* (grid_mech_spectral_basic.f90:103-355), or with
   num->solver = 1 grid_mech_spectral_polarization_* (grid_mech_spectral_polarization.f90:115-636) */
int  orc_mech_init(orc_ctx*);
int  orc_mech_forward(orc_ctx*, int cutBack, int guess, double dt, double dt_old, double t_remaining,
                      const orc_bc* deformation, const orc_bc* stress, const double q_rot[4]);
int  orc_mech_solution(orc_ctx*, orc_solution* out);
int  orc_materialpoint_forward(orc_ctx*);
/* utilities_updateCoords (spectral_utilities.f90:857-968) on the solver F; coordinates
   (3 per cell centre / per node, x fastest), undeformed before the first update */
int  orc_update_coords(orc_ctx*);
void orc_get_coords(orc_ctx*, double* ip, double* nodes);

/* operator-level entry points */
int  orc_constitutive_response(orc_ctx*, const double* F, double dt, double* P, double P_av[9],
                               double C_volAvg[81], double C_minMaxAvg[81], int* status);
void orc_update_gamma(orc_ctx*, const double C[81]);
void orc_gamma_convolution(orc_ctx*, double* field, const double aim[9]);
double orc_divergence_rms(orc_ctx*, const double* P);
double orc_curl_rms(orc_ctx*, const double* F);   /* utilities_curlRMS, spectral_utilities.f90:695-757 */
void orc_dPdF(orc_ctx*, double dt, double* dPdF /* 81 per voxel */);

/* field access: 0 F, 1 P, 2 Fe, 3 Fp, 4 Lp, 5 S, 6 xi_sl, 7 gamma_sl, 8 F_lastinc, 9 Fi, 10 Li,
   11 F of the solver, 12 O (orientation quaternion w,x,y,z per voxel; get only),
   13 F_tau and 14 F_tau_lastinc of the polarization solver */
int  orc_get_field(orc_ctx*, int field, double* out);
int  orc_set_field(orc_ctx*, int field, const double* in);
void orc_get_aims(orc_ctx*, double F_aim[9], double P_aim[9], double C_volAvg[81], double C_minMaxAvg[81]);

/* err_curl of the last polarization residual */
double orc_err_curl(orc_ctx*);

/* counters for the last call: constitutive calls, Newton iterations, state iterations */
void orc_counters(orc_ctx*, int64_t out[4]);

/* lattice constants as built by the restatement (for unit tests) */
int  orc_schmid(const orc_phase*, int sense, double* P /* 9*Ns, column-major */);
int  orc_interaction(const orc_phase*, double* h /* Ns*Ns, row = reacting */);

/* FFT used by the restatement: in-place 3D complex transform of n[0]*n[1]*n[2] points,
   x fastest; sign -1 forward, +1 backward, unnormalised. */
void orc_fft3(double* data /* interleaved re,im */, const int n[3], int sign);
}
