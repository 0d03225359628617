// Per-voxel constitutive update of the DAMASK grid hot path, FP64, one thread per
// material point, organised as passes over the voxels that still iterate.
//
// Restates, for one constituent with pass/isostrain homogenization (F_phase =
// F_cell, homogenization_mechanical.f90:94-123) and Hooke + phenopowerlaw slip:
//   phase_mechanical_constitutive   phase_mechanical.f90:1008-1090 (substep cutback)
//   mechanical_restore              phase_mechanical.f90:1096-1115
//   integrateStateFPI (+ damper)    phase_mechanical.f90:591-676
//   integrateStress (Lp Newton)     phase_mechanical.f90:379-584
//   plastic_LpAndItsTangents        phase_mechanical_plastic.f90:239-298
//   phenopowerlaw kinetics/dotState phase_mechanical_plastic_phenopowerlaw.f90:303-399,449-488
//
// Specialisation: no eigenstrain mechanism is active on this path, so the
// intermediate configuration stays Fi = I and Li = 0 (phase_mechanical_eigen.f90:133-165
// returns Li = 0; the Li loop of integrateStress then exits on its first pass).
// With Fi = I the Mandel stress is Mp = S and the Newton Jacobian
//   dR/dLp = I - dLp/dS : dS/dFe : dFe/dLp
// collapses to  J[kl][pb] = delta + dt * sum_s dgamma_s P_s(k,l) (A^T Fe Q_s)(p,b)
// with A = F Fp0^-1 and Q_s = C : P_nS_s precomputed per phase, so no 3x3x3x3
// temporaries are formed.
//
// Execution model.  The nested loops of the reference (substeps > state
// iterations > Newton iterations) are split at the state iteration: one pass
// performs, for every voxel still iterating, exactly one integrateStress (the Newton
// loop, in registers) followed by the state update and whatever substep control
// leads to the next integrateStress.  Between passes the per-voxel iteration state
// lives in HBM planes (PassWork), so the large per-system arrays of the state
// iteration are never live during the Newton loop; all indexing into register
// arrays is static, and the 9x9 Newton system, a rank-6 update of the identity, is
// solved through its 6x6 Woodbury form by Householder QR (no data-dependent row
// exchange, so the matrix stays in registers).
#pragma once
#include "dmk_device.cuh"

namespace dmk {

__device__ __forceinline__ void load_ctl(const PassWork& w, int64_t N, int64_t v, VoxelCtl& c) {
  c.phase = w.ctl[v];
  c.status = w.ctl[N + v];
  c.it = w.ctl[2 * N + v];
  c.nsub = w.ctl[3 * N + v];
  c.nstate = w.ctl[4 * N + v];
  c.newton = w.ctl[5 * N + v];
  c.stepFrac = w.sub[v];
  c.step = w.sub[N + v];
}
__device__ __forceinline__ void store_ctl(const PassWork& w, int64_t N, int64_t v, const VoxelCtl& c) {
  w.ctl[v] = c.phase;
  w.ctl[N + v] = c.status;
  w.ctl[2 * N + v] = c.it;
  w.ctl[3 * N + v] = c.nsub;
  w.ctl[4 * N + v] = c.nstate;
  w.ctl[5 * N + v] = c.newton;
  w.sub[v] = c.stepFrac;
  w.sub[N + v] = c.step;
}

// Solves A x = b for a row-major n x n A (overwritten with R) by Householder QR:
// column k is reflected onto alpha e_k with alpha = -sign(x0) |x|, v = x - alpha e_k,
// H y = y + v (v.y) / (alpha v0).  Returns true when a column of the remaining
// matrix is exactly zero (the matrix is singular; dgesv info > 0).  All indices are
// compile-time constants, so A stays in registers.
template <int n>
__device__ __forceinline__ bool qr_solve(double* A, double* b) {
#pragma unroll
  for (int k = 0; k < n - 1; ++k) {
    double s2 = 0.0;
#pragma unroll
    for (int i = k; i < n; ++i) s2 = fma(A[i * n + k], A[i * n + k], s2);
    if (s2 == 0.0) return true;
    const double sig = sqrt(s2);
    const double x0 = A[k * n + k];
    const double alpha = x0 >= 0.0 ? -sig : sig;
    const double v0 = x0 - alpha;
    const double rs = 1.0 / (alpha * v0);
#pragma unroll
    for (int c = k + 1; c < n; ++c) {
      double d = v0 * A[k * n + c];
#pragma unroll
      for (int i = k + 1; i < n; ++i) d = fma(A[i * n + k], A[i * n + c], d);
      d *= rs;
      A[k * n + c] = fma(d, v0, A[k * n + c]);
#pragma unroll
      for (int i = k + 1; i < n; ++i) A[i * n + c] = fma(d, A[i * n + k], A[i * n + c]);
    }
    {
      double d = v0 * b[k];
#pragma unroll
      for (int i = k + 1; i < n; ++i) d = fma(A[i * n + k], b[i], d);
      d *= rs;
      b[k] = fma(d, v0, b[k]);
#pragma unroll
      for (int i = k + 1; i < n; ++i) b[i] = fma(d, A[i * n + k], b[i]);
    }
    A[k * n + k] = alpha;
  }
  if (A[n * n - 1] == 0.0) return true;
#pragma unroll
  for (int i = n - 1; i >= 0; --i) {
    double s = b[i];
#pragma unroll
    for (int k = i + 1; k < n; ++k) s = fma(-A[i * n + k], b[k], s);
    b[i] = s / A[i * n + i];
  }
  return false;
}

// integrateStress, phase_mechanical.f90:379-584 (Fi = I, Li = 0).
// F and Fp0 point at voxel v's planes (stride N); they are read at the start and again
// for the final Fp / P so that no copy stays in registers through the Newton loop.
// xs: this thread's shared-memory slots (stride pass_threads<NS>()): 1/xi (NS entries), the
// Newton weights dt*dgamma (NS), then A (9).  The voxel's planes (stride N) receive |dot_gamma|
// of the last residual evaluation (adg_g; the state update after a converged integration reads
// it), the last accepted Lp guess (lo_g) and the Newton step (dl_g): they are written once per
// Newton iteration and read back rarely (line search, step), so they stay out of the shared
// memory that bounds the kernel's occupancy.  Lp (in/out) is the warm start and, on success,
// the result; S, Fp, P and Fe are written only on success.
template <int NS>
__device__ int integrate_stress(const PhaseConst<NS>& pc, const SysConst* __restrict__ sc, const Numerics& nm,
                                const double* Fg, const double* Fp0g, int64_t N, double* xs, double dt, double* Lp,
                                double* S, double* Fp, double* Pout, double* Feout, int& newton,
                                double* __restrict__ adg_g, double* __restrict__ lo_g, double* __restrict__ dl_g) {
  double* const sw = xs + NS * pass_threads<NS>();
  double* const sA = xs + 2 * NS * pass_threads<NS>();
  {
    double F[9], Fp0[9], invFp0[9], A[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) { F[k] = Fg[k * N]; Fp0[k] = Fp0g[k * N]; }
    if (inv33(Fp0, invFp0)) return 5;                     // STATUS_FAIL_PHASE_MECHANICAL_STRESS
    mm33(F, invFp0, A);
#pragma unroll
    for (int k = 0; k < 9; ++k) sA[k * pass_threads<NS>()] = A[k];
  }

  double Lg[9], B[9], s6[6];
#pragma unroll
  for (int k = 0; k < 9; ++k) { Lg[k] = Lp[k]; lo_g[k * N] = Lp[k]; dl_g[k * N] = 0.0; }
  double step = 1.0, res_old = 1.7976931348623157e308;
  int jaco = 0;
  for (int it = 1;; ++it) {
    if (it > nm.N_iter_Lp_max) return 6;                  // STATUS_FAIL_PHASE_MECHANICAL_STRESS_LP_MAXIT
    ++newton;
#pragma unroll
    for (int k = 0; k < 9; ++k) B[k] = ((k % 4 == 0) ? 1.0 : 0.0) - dt * Lg[k];
    double Fe[9];
    {
      double A[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) A[k] = sA[k * pass_threads<NS>()];
      mm33(A, B, Fe);
    }
    hooke_S<NS>(pc, Fe, s6);
    // Lp_c = sum_s dot_gamma_s P_s and the weights of its derivative
    double Lc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    static_assert(NS <= 64, "one sense bit per slip system");
    SenseMask<NS> neg = 0u;
#pragma unroll 2
    for (int s = 0; s < NS; ++s) {
      const SysConst& c = sc[s];
      double2 p[6];
#pragma unroll
      for (int t = 0; t < 6; ++t) p[t] = c.p6[t];
      const double tp = s6[0] * p[0].x + s6[1] * p[1].x + s6[2] * p[2].x + s6[3] * p[3].x + s6[4] * p[4].x + s6[5] * p[5].x;
      const double tn = s6[0] * p[0].y + s6[1] * p[1].y + s6[2] * p[2].y + s6[3] * p[3].y + s6[4] * p[4].y + s6[5] * p[5].y;
      const bool pos = tp > tn;
      const double tmax = pos ? tp : tn;
      const double ixs = xs[s * pass_threads<NS>()];
      const double r = tmax * ixs;
      const double2 kin = c.kin;
      const int ni = c.n_int;
      double g, dg;
      if (ni >= 1) {
        const double rn1 = powi_fixed<6>(r, ni - 1);
        const double sd = pos ? kin.x : -kin.x;
        g = sd * (rn1 * r);
        dg = (sd * kin.y) * rn1 * ixs;
      } else {
        g = (pos ? kin.x : -kin.x) * pow(r, kin.y);
        dg = g * kin.y / tmax;
      }
      if (!(fabs(g) > TINY10)) dg = 0.0;
      // P_nS sense of the derivative follows the sign of dot_gamma (phenopowerlaw.f90:327)
      if (!(g > 0.0)) neg |= SenseMask<NS>(1) << s;
      sw[s * pass_threads<NS>()] = dt * dg;
      adg_g[s * N] = fabs(g);
      double2 P[5];
#pragma unroll
      for (int k = 0; k < 5; ++k) P[k] = c.P[k];
      const double Ps[9] = {P[0].x, P[0].y, P[1].x, P[1].y, P[2].x, P[2].y, P[3].x, P[3].y, P[4].x};
#pragma unroll
      for (int k = 0; k < 9; ++k) Lc[k] = fma(g, Ps[k], Lc[k]);
    }
    double R[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) R[k] = Lg[k] - Lc[k];
    const double nR = norm9(R);
    const double atol = fmax(nm.eps_rel_Lp * fmax(norm9(Lg), norm9(Lc)), nm.eps_abs_Lp);
    if (isnan(nR)) return 7;                              // STATUS_FAIL_PHASE_MECHANICAL_STRESS_LP_NAN
    if (nR < atol) break;
    if (nR < res_old) {
      res_old = nR;
#pragma unroll
      for (int k = 0; k < 9; ++k) lo_g[k * N] = Lg[k];
      step = 1.0;
    } else {
      step = nm.r_linesearch_Lp * step;
#pragma unroll
      for (int k = 0; k < 9; ++k) Lg[k] = fma(dl_g[k * N], step, lo_g[k * N]);
      continue;
    }
    if (jaco % nm.f_update_jacobi_Lp == 0) {
      ++jaco;
      // Newton step J dLp = -R with J = I + K, K[kl][pb] = (M H^(kl))(p,b), M = A^T Fe,
      // H^(kl) = sum_s w_s P_s(k,l) Q_s.  Every row of K is M times a symmetric matrix,
      // so K = Hm L^T has rank 6 (Hm: 9x6 rows h^(kl); L: 9x6, L^T z = symfold(M^T Z)) and
      // by the Woodbury identity  J^-1 z = z - Hm (I6 + L^T Hm)^-1 L^T z.  With P_s = d_s (x) n_s,
      //   C6 = I6 + sum_s w_s symfold((M^T d_s) (x) n_s) (x) q_s,   y = C6^-1 symfold(M^T R),
      //   dLp = sum_s w_s (q_s . y) P_s - R,
      // the same solution as the 9x9 system without forming it.
      double M[9];
      {
        double A[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) A[k] = sA[k * pass_threads<NS>()];
        mtm33(A, Fe, M);                                  // M = A^T Fe, M[p + 3q] = M(p,q)
      }
      double C6[36];
#pragma unroll
      for (int i = 0; i < 36; ++i) C6[i] = (i % 7 == 0) ? 1.0 : 0.0;
#pragma unroll 2
      for (int s = 0; s < NS; ++s) {
        const SysConst& c = sc[s];
        const double ws = sw[s * pass_threads<NS>()];
        const bool ng = (neg >> s) & 1u;
        double q[6];
#pragma unroll
        for (int t = 0; t < 6; ++t) {
          const double2 qq = c.q6[t];
          q[t] = ng ? qq.y : qq.x;
        }
        const double2 dn0 = c.dn[0], dn1 = c.dn[1], dn2 = c.dn[2];
        const double d0 = dn0.x, d1 = dn0.y, d2 = dn1.x, n0 = dn1.y, n1 = dn2.x, n2 = dn2.y;
        // u = M^T d
        const double u0 = M[0] * d0 + M[1] * d1 + M[2] * d2;
        const double u1 = M[3] * d0 + M[4] * d1 + M[5] * d2;
        const double u2 = M[6] * d0 + M[7] * d1 + M[8] * d2;
        const double a6[6] = {ws * (u0 * n0), ws * (u1 * n1), ws * (u2 * n2), ws * (u1 * n2 + u2 * n1),
                              ws * (u0 * n2 + u2 * n0), ws * (u0 * n1 + u1 * n0)};
#pragma unroll
        for (int i = 0; i < 6; ++i)
#pragma unroll
          for (int j = 0; j < 6; ++j) C6[6 * i + j] = fma(a6[i], q[j], C6[6 * i + j]);
      }
      // y6 = symfold(M^T R)
      double y6[6];
      {
        double G[9];
        mtm33(M, R, G);                                   // G(a,b) = sum_p M(p,a) R(p,b)
        y6[0] = G[0]; y6[1] = G[4]; y6[2] = G[8];
        y6[3] = G[7] + G[5]; y6[4] = G[6] + G[2]; y6[5] = G[3] + G[1];
      }
      if (qr_solve<6>(C6, y6)) return 8;                 // singular: STATUS_FAIL_PHASE_MECHANICAL_STRESS_LP_DGESV
      double X[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) X[k] = -R[k];
#pragma unroll 2
      for (int s = 0; s < NS; ++s) {
        const SysConst& c = sc[s];
        const bool ng = (neg >> s) & 1u;
        double cq = 0.0;
#pragma unroll
        for (int t = 0; t < 6; ++t) {
          const double2 qq = c.q6[t];
          cq = fma(ng ? qq.y : qq.x, y6[t], cq);
        }
        cq *= sw[s * pass_threads<NS>()];
        double2 P[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) P[k] = c.P[k];
        const double Ps[9] = {P[0].x, P[0].y, P[1].x, P[1].y, P[2].x, P[2].y, P[3].x, P[3].y, P[4].x};
#pragma unroll
        for (int k = 0; k < 9; ++k) X[k] = fma(cq, Ps[k], X[k]);
      }
#pragma unroll
      for (int k = 0; k < 9; ++k) dl_g[k * N] = X[k];
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) Lg[k] = fma(dl_g[k * N], step, Lg[k]);
  }
  // Fp = (Fp0^-1 B)^-1 / det^(1/3); P = F Fp^-1 S Fp^-T; Fe = F Fp^-1  (:571-581)
  double F[9], invFpn[9], Fpn[9];
  {
    double Fp0[9], invFp0[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) { F[k] = Fg[k * N]; Fp0[k] = Fp0g[k * N]; }
    inv33(Fp0, invFp0);                                   // invertible: checked on entry
    mm33(invFp0, B, invFpn);
  }
  if (inv33(invFpn, Fpn)) return 5;
  const double cb = 1.0 / cbrt(det33(Fpn));
  double FiF[9];
  mm33(F, invFpn, FiF);
  const double Sm[9] = {s6[0], s6[5], s6[4], s6[5], s6[1], s6[3], s6[4], s6[3], s6[2]};
  double T1[9], T2[9];
  mmt33(Sm, invFpn, T1);          // S Fp^-T
  mm33(FiF, T1, T2);
#pragma unroll
  for (int k = 0; k < 9; ++k) { Pout[k] = T2[k]; Feout[k] = FiF[k]; Fp[k] = Fpn[k] * cb; Lp[k] = Lg[k]; }
#pragma unroll
  for (int k = 0; k < 6; ++k) S[k] = s6[k];
  return 0;
}

// Hardening matrix staged in shared memory once per block (row = reacting system),
// read with uniform addresses (broadcast) in the control kernels.
// doubles of shared memory for the hardening matrix: staged up to 24 systems; at 48 (18 KB) the
// control and begin kernels read it from device memory (uniform addresses, L1 resident), so that
// four 64-thread blocks fit per SM instead of three
template <int NS>
__host__ __device__ constexpr size_t hard_smem_doubles() { return NS <= 24 ? size_t(NS) * NS : 0; }

template <int NS>
__device__ __forceinline__ void stage_hardening(const PhaseConst<NS>& pc, double* hs) {
  for (int i = threadIdx.x; i < NS * NS; i += blockDim.x) hs[i] = pc.hmat[i];
}

// Slots of the stress kernel (stride pass_threads<NS>()): 1/xi [0, NS), Newton weights
// [NS, 2NS), A = F Fp0^-1 [2NS, 2NS + 9).
template <int NS>
__host__ __device__ constexpr int stress_slots() { return 2 * NS + 9; }

// phenopowerlaw_dotState (Fi = I => Mp = S; no twins => sumF = 0) at the stored
// stress and state of voxel v, written to this thread's slots: xi rates first, then
// |dot_gamma|.  hs: the hardening matrix (shared memory, or device memory read with uniform
// addresses).  adg_in (element s at adg_in[s * adg_stride]), when given, holds |dot_gamma| at
// this stress and state already (the kinetics of the converged integrateStress); otherwise
// the kinetics are evaluated.  Returns true if any rate is NaN.
template <int NS>
__device__ bool dot_state_slots(const PhaseConst<NS>& pc, const double* __restrict__ hs, const double s6[6],
                                const double* __restrict__ state, int64_t N, int64_t v, double* xs,
                                const double* adg_in, int64_t adg_stride) {
  double adg[NS];
  if (adg_in) {
#pragma unroll
    for (int s = 0; s < NS; ++s) adg[s] = adg_in[s * adg_stride];
  } else {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const double tp = dot6(s6, pc.p6[0][s]), tn = dot6(s6, pc.p6[1][s]);
      const double tmax = tp > tn ? tp : tn;
      adg[s] = fabs(pc.dg0[s] * powr(tmax / state[s * N + v], pc.n[s], pc.n_int[s]));
    }
  }
  bool bad = false;
  // xi of every system into the slots first, so that the loads overlap
#pragma unroll 8
  for (int l = 0; l < NS; ++l) xs[l * pass_threads<NS>()] = state[l * N + v];
#pragma unroll 2
  for (int l = 0; l < NS; ++l) {
    const double x = fma(-xs[l * pass_threads<NS>()], pc.ixiinf[l], 1.0);  // 1 - xi/xi_inf
    const double left = copysign(powr(fabs(x), pc.a[l], pc.a_int[l]), x);
    const double2* hrow = reinterpret_cast<const double2*>(hs + l * NS);
    double hg = 0.0;
#pragma unroll
    for (int k = 0; k < NS / 2; ++k) {
      const double2 hh = hrow[k];
      hg = fma(hh.x, adg[2 * k], hg);
      hg = fma(hh.y, adg[2 * k + 1], hg);
    }
    const double d = pc.h0f[l] * left * hg;
    bad |= isnan(d);
    xs[l * pass_threads<NS>()] = d;
  }
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    bad |= isnan(adg[s]);
    xs[(NS + s) * pass_threads<NS>()] = adg[s];
  }
  return bad;
}

// damper, phase_mechanical.f90:653-674
__device__ __forceinline__ double damper(double d01, double d12, double d22) {
  if (fmin(d01, d12) < 0.0 && d22 > 0.0) return 0.75 + 0.25 * tanh(2.0 + 4.0 * d12 / d22);
  return 1.0;
}

// Substep-start values (subF0, subFp0, subLp0, subState0 of phase_mechanical_constitutive).
// Until the first substep of an evaluation has advanced (stepFrac == 0) they equal the
// increment-start values F0, Fp0, Lp0, state0 and are read from there; the first advance
// writes them to the pass records, which are read from then on.
struct SubStart {
  const double *F0, *Fp0, *Lp0, *st0;
};
__device__ __forceinline__ SubStart sub_start(const Fields& f, const PassWork& w, double stepFrac) {
  const bool first = stepFrac == 0.0;
  return {first ? f.F0 : w.F0s, first ? f.Fp0 : w.Fp0s, first ? f.Lp0 : w.Lp0s, first ? f.state0 : w.st0s};
}

// dotState generations of the state iteration alternate between two 2NS-plane arrays:
// iteration it (0 = the start) stores its damped rate in array it % 2, which then holds
// dotState_last(:,1) for iteration it + 1 and dotState_last(:,2) for iteration it + 2.
__device__ __forceinline__ double* dot_gen(const PassWork& w, int it, int NST, int64_t N) {
  return w.D + int64_t(it & 1) * NST * N;
}

// Advances voxel v through the control flow of phase_mechanical_constitutive and
// integrateStateFPI until its next integrateStress (phase PH_STRESS) or its end
// (PH_DONE).  Entered in PH_CTRL (substep control after an integration attempt) or
// PH_DOT1 (state update after a successful integrateStress, whose |dot_gamma| is at
// adg[s * adg_stride]).
template <int NS>
__device__ void advance(const PhaseConst<NS>& pc, const double* __restrict__ hs, const Numerics& nm, const Fields& f,
                        const PassWork& w, int64_t v, double dt, VoxelCtl& c, double* xs, const double* adg,
                        int64_t adg_stride) {
  constexpr int NST = 2 * NS;
  const int64_t N = f.N;
  // every control step shrinks the substep or advances stepFrac; the bound only
  // guards against numerics (r_cutback >= 1) under which the reference loops forever
  for (int guard = 0; c.phase != PH_STRESS && c.phase != PH_DONE; ++guard) {
    if (guard > 4096) { c.status = 3; c.phase = PH_DONE; break; }
    if (c.phase == PH_CTRL) {
      // substep control, phase_mechanical.f90:1040-1080
      bool todo;
      if (c.status == 0) {
        c.stepFrac = c.stepFrac + c.step;
        c.step = fmin(1.0 - c.stepFrac, nm.r_increase * c.step);
        todo = c.step > 0.0;
        if (todo) {
#pragma unroll
          for (int k = 0; k < 9; ++k) {
            w.F0s[k * N + v] = w.Fs[k * N + v];
            w.Lp0s[k * N + v] = f.Lp[k * N + v];
            w.Fp0s[k * N + v] = f.Fp[k * N + v];
          }
#pragma unroll 12
          for (int i = 0; i < NST; ++i) w.st0s[i * N + v] = f.state[i * N + v];
        }
      } else {
        c.step = nm.r_cutback * c.step;
        const SubStart ss = sub_start(f, w, c.stepFrac);
#pragma unroll
        for (int k = 0; k < 9; ++k) f.Fp[k * N + v] = ss.Fp0[k * N + v];
#pragma unroll
        for (int k = 0; k < 6; ++k) f.S[k * N + v] = f.S0[k * N + v];
        if (c.step < 1.0)
#pragma unroll
          for (int k = 0; k < 9; ++k) f.Lp[k * N + v] = ss.Lp0[k * N + v];
#pragma unroll 12
        for (int i = 0; i < NST; ++i) f.state[i * N + v] = ss.st0[i * N + v];
        todo = c.step > nm.r_cutback_min;
      }
      if (!todo) { c.phase = PH_DONE; break; }
      ++c.nsub;
      const double* F0s = sub_start(f, w, c.stepFrac).F0;
#pragma unroll
      for (int k = 0; k < 9; ++k)
        w.Fs[k * N + v] = fma(c.step, f.F[k * N + v] - f.F0[k * N + v], F0s[k * N + v]);
      c.phase = PH_DOT0;
    } else {
      // dotState at the current stress and state: start (DOT0) or update (DOT1) of a state
      // iteration; after a converged integrateStress its kinetics are stored already
      double s6[6];
      const bool after_stress = c.phase == PH_DOT1;
      if (!after_stress)
#pragma unroll
        for (int k = 0; k < 6; ++k) s6[k] = f.S[k * N + v];
      const bool bad = dot_state_slots<NS>(pc, hs, s6, f.state, N, v, xs, after_stress ? adg : nullptr, adg_stride);
      const double dts = c.step * dt;
      if (c.phase == PH_DOT0) {
        // integrateStateFPI:616-620
        if (bad) { c.status = 3; c.phase = PH_CTRL; continue; }   // STATUS_FAIL_PHASE_MECHANICAL_STATE
        double* D0 = dot_gen(w, 0, NST, N) + v;
        const double* st0 = sub_start(f, w, c.stepFrac).st0;
#pragma unroll 12
        for (int i = 0; i < NST; ++i) {
          const double d = xs[i * pass_threads<NS>()];
          f.state[i * N + v] = fma(d, dts, st0[i * N + v]);
          D0[i * N] = d;
        }
        c.it = 0;
        c.phase = PH_STRESS;
      } else {
        // integrateStateFPI:631-646 (the stress integration of this iteration succeeded: status 0)
        if (bad) { c.phase = PH_CTRL; continue; }
        // generations: dotState of the last iteration (it - 1) and the one before (it - 2,
        // whose storage receives the damped rate of this iteration)
        const double* L1 = dot_gen(w, c.it + 1, NST, N) + v;
        double* L2 = dot_gen(w, c.it, NST, N) + v;
        double d01 = 0.0, d12 = 0.0, d22 = 0.0;
#pragma unroll 24
        for (int i = 0; i < NST; ++i) {
          const double d = xs[i * pass_threads<NS>()];
          const double l1 = L1[i * N];                                 // dotState_last(:,1)
          const double l2 = c.it > 1 ? L2[i * N] : 0.0;               // dotState_last(:,2)
          const double a = d - l1, b = l1 - l2;
          d12 = fma(a, b, d12);
          d22 = fma(b, b, d22);
          d01 = fma(d, l1, d01);
        }
        const double zeta = damper(d01, d12, d22);
        const double* st0 = sub_start(f, w, c.stepFrac).st0;
        bool conv = true;
#pragma unroll 12
        for (int i = 0; i < NST; ++i) {
          const double l1 = L1[i * N];
          const double d = xs[i * pass_threads<NS>()] * zeta + l1 * (1.0 - zeta);
          const double st = f.state[i * N + v];
          const double r = st - st0[i * N + v] - d * dts;
          const double stn = st - r;
          f.state[i * N + v] = stn;
          L2[i * N] = d;
          const double atol = i < NS ? pc.atol_xi : pc.atol_gamma;
          conv = conv && (fabs(r) <= fmax(atol, nm.eps_rel_state * fabs(stn)));
        }
        c.phase = (conv || c.it >= nm.N_iter_state_max) ? PH_CTRL : PH_STRESS;
      }
    }
  }
}

}  // namespace dmk
