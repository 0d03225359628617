// Kernel launch interface shared by the kernel and host translation units.
#pragma once
#include "dmk_device.cuh"

namespace dmk {

constexpr int CONST_THREADS = 128;   // block size of the per-voxel partial sums of P
constexpr int PASS_CHUNKS = 4;       // voxel chunks whose constitutive passes run on their own streams
constexpr int SPEC_THREADS = 256;    // spectral pointwise kernels

// Solver scalars living in device memory (grid_mech_spectral_basic.f90:30-45 module state
// that the residual evaluation reads or updates).
struct SolverScalars {
  double F_aim[9];
  double P_aim[9];
  double P_av[9];
  double Scomp[81];      // masked compliance S (grid_utilities.f90:74-127)
  double q_rot[4];       // load-frame rotation
  double aim_rot[9];     // rotation_BC%rotate(deltaF_aim, active) for the DC term
  double avRate[9];      // forward: rotated F_aimDot
  double aim_fwd[9];     // forward: rotated F_aim
  int stress_mask[9];    // 1 = stress component not prescribed
  double err_div, err_BC;
  int totalIter;
  int status;
  int reason;
};

struct GammaConst {
  double Cref[81];       // C_ref = C / wgt, column-major 3x3x3x3
  double rescale[3];     // geomSize / scaledGeomSize
  int derivative;        // 0 continuous, 1 central difference, 2 FWBW difference
};

// Imaginary part a of the spectral derivative xi = i a for signed frequency k of an edge of n
// cells and length L (utilities_getFreqDerivative, spectral_utilities.f90:808-850): continuous
// 2 pi k / L, central difference sin(2 pi k / n) / (2 L / n).  first_order: the first-derivative
// frequencies xi1st, whose Nyquist component is zero on even edges for the continuous
// derivative (:322-332).
__device__ __forceinline__ double freq_derivative(int k, int n, double L, int derivative, bool first_order) {
  const double TAU = 6.283185307179586;
  if (derivative == 1) return sin(TAU * double(k) / double(n)) / (2.0 * L / double(n));
  if (first_order && n % 2 == 0 && k == n / 2) return 0.0;
  return TAU * double(k) / L;
}

// FWBW_difference (utilities_getFreqDerivative, spectral_utilities.f90:823-849): the complex
// frequencies xi_d = (e^{i t_d} - 1) prod_{e != d} (e^{i t_e} + 1) / (4 L_d / n_d), t_e = 2 pi k_e / n_e,
// for the signed indices k; the factors multiply in the order e = 1, 2, 3.  xi1st = xi2nd here.
// In real space xi_d is the forward difference along d averaged over the four edges of the
// staggered cell, so xi(-k) = conj(xi(k)) and the operators built on it keep spectra Hermitian.
__device__ __forceinline__ void freq_fwbw(const int k[3], const int n[3], const double L[3], double xr[3],
                                          double xim[3]) {
  const double TAU = 6.283185307179586;
  double c[3], s[3];
#pragma unroll
  for (int e = 0; e < 3; ++e) sincos(TAU * double(k[e]) / double(n[e]), &s[e], &c[e]);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double pr = 1.0, pi = 0.0;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      const double fr = c[e] + (e == d ? -1.0 : 1.0), fi = s[e];
      const double t = pr * fr - pi * fi;
      pi = pr * fi + pi * fr;
      pr = t;
    }
    const double h4 = 4.0 * L[d] / double(n[d]);
    xr[d] = pr / h4;
    xim[d] = pi / h4;
  }
}

struct Numerics2 {
  int N_iter_min, N_iter_max, cells0;
  double eps_abs_div, eps_rel_div, eps_abs_P, eps_rel_P;
};

// constitutive passes (constitutive.cu)
template <int NS>
cudaError_t launch_constitutive_begin(const PhaseConst<NS>& pc, const Numerics& nm, const Fields& f,
                                      const PassWork& w, double dt, int apply_update, int use_dot0, int64_t v_begin,
                                      int64_t v_end, cudaStream_t s);
// variant: the stress kernel's register bound (stress_variant_blocks: resident blocks per SM)
template <int NS>
cudaError_t launch_constitutive_pass(const PhaseConst<NS>& pc, const Numerics& nm, const Fields& f,
                                     const PassWork& w, double dt, const int* list_in, int64_t n_in, cudaStream_t s,
                                     int variant = 0);
int stress_variant_count(int ns);
int stress_variant_blocks(int ns, int variant);
// Tables of a batch of contexts of one phase (the constitutive passes of all of them in shared
// launches): items are the voxels of all contexts, context after context.
struct BatchTables {
  const Fields* f;               // per context: its fields
  const PassWork* w;             // per context: its pass work planes
  const double* dt;              // per context: the time step of its current increment
  const int64_t* off;            // per context: its first item (off[n_ctx] = n_items)
  const int* ctx_of;             // per item: its context
  const unsigned char* active;   // per context: evaluated in this launch
  const int* use_dot0;           // per context: the increment-start rates are stored already
  const int* apply;              // per context: fuse F <- F - r into the first pass
  int64_t n_items;
};
struct BatchPassBuffers {
  int* list[2];                  // item lists of the passes (n_items entries each)
  int* count;                    // their 2 entry counts
  int* status;                   // per context: worst status of the evaluation (Fields::status)
  int n_ctx;
  int* iter;                     // [0] passes run, [1] set when max_passes stopped the loop
  int max_passes;
};
template <int NS>
cudaError_t build_batch_pass_graph(const PhaseConst<NS>& pc, const Numerics& nm, const BatchTables& t,
                                   const BatchPassBuffers& b, int nsm, cudaStream_t s, cudaGraph_t* out);
cudaError_t launch_sum9(const double* X, int64_t N, double* partials, cudaStream_t s);
cudaError_t launch_aim(SolverScalars* sc, const double* partials, int nparts, double wgt, int update_aim, cudaStream_t s);
cudaError_t launch_converge(SolverScalars* sc, const double* div_partials, int nparts, double wgt, const int* status,
                            const Numerics2& nm2, int count_iteration, cudaStream_t s);
template <typename Real>
cudaError_t launch_gamma_div(Real* spec, int n0, int n1, int n2, const double L[3], const GammaConst& gc,
                             const SolverScalars* sc, double* div_partials, int do_gamma, int do_div, cudaStream_t s);
int gamma_div_blocks(int n0, int n1, int n2);
cudaError_t launch_to_planes(const double* in, double* out, int64_t N, int K, cudaStream_t s);
cudaError_t launch_from_planes(const double* in, double* out, int64_t N, int K, cudaStream_t s);
cudaError_t launch_sym6_to9(const double* in, double* out, int64_t N, cudaStream_t s);
cudaError_t launch_forward(double* Fsol, double* Flast, double* Fdot, int64_t N, int cutBack, int guess, double dt,
                           double dt_old, const double* avRate, double* partials, double* sums, double wgt,
                           const double* aim, cudaStream_t s);
cudaError_t launch_init_state(const int* material, const double* quats, const double* xi0, int NS, int64_t N, double* F,
                              double* F0, double* Fsol, double* Flast, double* Fp, double* Fp0, double* Fe, double* state,
                              double* state0, cudaStream_t s);
cudaError_t launch_copy(const double* a, double* b, int64_t n, int nsm, cudaStream_t s);
cudaError_t launch_orientations(const double* Fe, int64_t N, double* out /* 4 per voxel */, int* bad, cudaStream_t s);
cudaError_t launch_to_float(const double* a, float* b, int64_t n, int nsm, cudaStream_t s);
cudaError_t launch_to_double(const float* a, double* b, int64_t n, int nsm, cudaStream_t s);

cudaError_t launch_reduce9(const double* partials, int nparts, double* out9, cudaStream_t s);
cudaError_t launch_fp64_probe(double* sink, int blocks, int iters, cudaStream_t s);

// spectral polarization scheme (polarization.cu)
struct PolConst {
  double C[81];          // C_scale (column-major 3x3x3x3)
  double S[81];          // S_scale = invSym3333(C_scale)
  double alpha, beta;
};
cudaError_t launch_pol_pre(const double* F, const double* Ftau, int64_t N, const PolConst& pc, double* out,
                           cudaStream_t s);
cudaError_t launch_pol_tau(const double* F, const double* G, double* rtau, int64_t N, double beta, double* Feval,
                           cudaStream_t s);
cudaError_t launch_pol_rF(const double* F, const double* Ftau, const double* P, const double* dPdF, const double* rtau,
                          int64_t N, const PolConst& pc, double* rF, cudaStream_t s);
cudaError_t launch_curl(const double* spec, int n0, int n1, int n2, const double L[3], const double rg[3],
                        int derivative, double* partials, cudaStream_t s);
cudaError_t launch_pol_forward_tau(const double* F, double* Ftau, double* Flast, double* Fdot, int64_t N, int cutBack,
                                   int guess, double dt, double dt_old, const double* avRate, const PolConst& pc,
                                   cudaStream_t s);
cudaError_t launch_sub(double* X, const double* r, int64_t n, int nsm, cudaStream_t s);

// utilities_updateCoords (kernels.cu): u_hat from the spectrum of F (planes 0..2, Hermitian), then
// cell-centre and node coordinates from the C2R output u (null: undeformed coordinates)
cudaError_t launch_coords_spec(double* spec, int n0, int n1, int n2, const double L[3], double wgt, double* favg,
                               int derivative, cudaStream_t s);
cudaError_t launch_coords(const double* u, const double* favg, const int n[3], const double step[3], double wgt,
                          double* xp, double* xn, cudaStream_t s);

// Anderson acceleration of the fixed point (kernels.cu)
constexpr int AA_MAX = 32;
constexpr int AA_CHUNK = 8;    // history slots per inner-product launch
struct AASlots {
  int n;                       // slots in this chunk
  int slot[AA_CHUNK];
};
struct AAUpdate {              // X <- X - R - sum_q gamma_q (dX[slot_q] - dR[slot_q])
  int n;
  int slot[AA_MAX];
  double gamma[AA_MAX];
};
cudaError_t launch_aa_dots(const double* R, const double* Rprev, double* dR, int64_t n, int write_slot,
                           const int* slots, int nslots, double* partials, int nblocks, double* out, cudaStream_t s);
cudaError_t launch_aa_update(double* X, const double* R, double* Rprev, double* dX, const double* dR, int64_t n,
                             int new_slot, const int* slots, const double* gamma, int nslots, int nblocks, cudaStream_t s);

// ------------------------------------------------------------------ batches of contexts (kernels.cu)
// The fixed-point iteration of many contexts (RVEs) in shared launches.  Each context is one entry
// of a device table; a batched kernel takes its context from blockIdx.y (blockIdx.x for one block
// per context) and keeps the block decomposition of the single-context kernel, so every context's
// sums, spectra and updates are those of its standalone solve.
struct BatchCtx {
  const double* P;          // stress kept when the evaluation failed
  const double* Pnew;       // stress of the evaluation, committed when its status is 0
  const int* status;        // status of the evaluation
  double* r;                // residual field (9 planes)
  double* X;                // solver F (9 planes)
  double* Rprev;            // Anderson: residual of the previous evaluation
  double* dX;               // Anderson history
  double* dR;
  SolverScalars* sc;
  double* partials;         // per block of CONST_THREADS voxels: 9 sums of the committed stress
  double* divp;             // per Gamma block: divergence partial sums
  double* aa_partials;      // per Anderson block: 2 AA_CHUNK partial sums
  double* aa_out;           // per chunk: 2 AA_CHUNK sums (g then b)
  double* fft_real;         // the context's 9 planes in its edge group's real buffer
  void* fft_spec;           // the context's 9 spectra in the group's spectrum buffer
  float* fft_real_f;        // the same in FP32 (mixed form), or null
  void* fft_spec_f;
  int64_t N;
  double wgt;
  double L[3];
  int n[3];
  int nconst, nspec, aa_blocks;
  int active;               // evaluated in this fixed-point iteration (<P>, aim)
  int mode;                 // its spectral pass now: 0 none, 1 FP32, 2 FP64
  int count_iter;           // the convergence test counts an iteration (not in an FP64 correction pass)
  int write_slot;           // Anderson: slot of the new dR, -1 for none
  int nsl;                  // Anderson: history slots of the inner products (oldest -> newest)
  int slots[AA_MAX];
  Numerics2 nm2;
  GammaConst gc;
};
struct BatchAA {            // Anderson update of one context
  int active, new_slot;
  AAUpdate u;
};
struct BatchScal {          // solver scalars of one context, read back after each iteration
  double P_av[9], F_aim[9];
  double err_div, err_BC;
  int totalIter, reason, status, pad;
};
// <P> of the committed stress and the aim update (sum9 + aim)
cudaError_t launch_batch_aim(const BatchCtx* t, int n_ctx, int max_nconst, cudaStream_t s);
// committed stress -> the group's real buffers, FP32 or FP64 by each context's mode
cudaError_t launch_batch_gather(const BatchCtx* t, int n_ctx, int64_t max_n9, cudaStream_t s);
// Gamma convolution and divergence partial sums on the group spectra of the contexts in mode 1
// (Real = float) or 2 (double)
template <typename Real>
cudaError_t launch_batch_gamma(const BatchCtx* t, int n_ctx, int max_nspec, cudaStream_t s);
// the group's real buffers (after the inverse transforms) -> residual fields
cudaError_t launch_batch_scatter(const BatchCtx* t, int n_ctx, int64_t max_n9, cudaStream_t s);
// convergence test, and the scalars of every context into out
cudaError_t launch_batch_converge(const BatchCtx* t, int n_ctx, BatchScal* out, cudaStream_t s);
// Anderson inner products of one chunk of history slots (dots and their reduction)
cudaError_t launch_batch_aa_dots(const BatchCtx* t, int n_ctx, int max_blocks, int chunk, cudaStream_t s);
cudaError_t launch_batch_aa_update(const BatchCtx* t, const BatchAA* u, int n_ctx, int max_blocks, cudaStream_t s);

// hand-written adjoint of an increment (adjoint.cu)
constexpr int ADJ_KRYLOV_MAX = 30;   // restart length of the Krylov solve of the transposed equilibrium problem
int adj_ws_size(int ns, int nf);     // doubles of per-voxel workspace of the local Jacobian
int adj_blocks(int64_t N);
int adj_mdot_blocks(int nsm);
template <int NS>
cudaError_t launch_adj_jacobian(const PhaseConst<NS>& pc, double dt, const double* pts, int64_t N, int64_t v0,
                                int64_t count, double* ws, double* D, int* bad, cudaStream_t s);
template <int NS>
cudaError_t launch_adj_vjp(const double* D, int64_t N, int nx, const double ell[9], const double* lam,
                           const double* s_in, double* g_out, double* s_out, double* th_part, int mode, cudaStream_t s);
cudaError_t launch_adj_sigma(const double* D, int64_t N, int nx, const double* lam, const double* G, double* sig,
                             double* partials, cudaStream_t s);
cudaError_t launch_adj_mdot(const double* w, const double* V, int64_t n, int nv, double* partials, int nsm,
                            cudaStream_t s);
cudaError_t launch_adj_maxpy(double* y, const double* V, int64_t n, int nv, const double* c, int nsm, cudaStream_t s);
cudaError_t launch_adj_scale(double* y, const double* x, double a, int64_t n, int nsm, cudaStream_t s);
template <int NS>
int host_local_jacobian(const PhaseConst<NS>& pc, const double* h, double dt, const double* pt, double* D);

// consistent tangent (dpdf.cu)
struct TangentOut {
  double* partials;      // per block: 81 sums of dPdF
  double* nmax;          // per block: max Frobenius norm^2
  double* nmin;
  double* per_voxel;     // optional: 81 per voxel, voxel-major (Fortran layout)
  double* norms;         // per voxel Frobenius norm^2
  double* planes;        // dPdF of every voxel, 81 planes (component i + 3j + 9k + 27l)
  double* l2;            // second-level reduction buffer (tangent_reduce_doubles())
};
int tangent_reduce_doubles();
template <int NS>
cudaError_t launch_dPdF(const PhaseConst<NS>& pc, const Fields& f, double dt, const TangentOut& o, int64_t first,
                        int64_t count, cudaStream_t s, bool with_sums = true);
// column sums and norms of the dPdF planes (the second stage of launch_dPdF)
cudaError_t launch_tangent_sums(const TangentOut& o, int64_t first, int64_t count, int64_t N, cudaStream_t s);
int dPdF_blocks(int64_t count);
template <int NS>
cudaError_t launch_tangent_pick(const PhaseConst<NS>& pc, const Fields& f, double dt, const long long* idx, double* out,
                                const double* planes, cudaStream_t s);
cudaError_t launch_tangent_finalize(const TangentOut& o, int nparts, double wgt,
                                    double* out /* 81 vol, 81 max, 81 min, max/min norm */, long long* idx /* 2 */,
                                    int64_t first, int64_t count, cudaStream_t s);

}  // namespace dmk
