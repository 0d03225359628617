// Per-voxel constitutive update of the DAMASK grid hot path, one thread per
// material point, FP64.
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
#pragma once
#include "dmk_device.cuh"

namespace dmk {

// kinetics_sl without derivative; returns |dot_gamma| per system
template <int NS>
__device__ __forceinline__ void kinetics_abs(const PhaseConst<NS>& pc, const double s6[6], const double* xi, double* adg) {
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const double tp = dot6(s6, pc.p6[0][s]), tn = dot6(s6, pc.p6[1][s]);
    const double tmax = tp > tn ? tp : tn;
    adg[s] = fabs(pc.dg0[s] * powr(tmax / xi[s], pc.n[s], pc.n_int[s]));
  }
}

// phenopowerlaw_dotState (Fi = I => Mp = S; no twins => sumF = 0)
template <int NS>
__device__ __forceinline__ void dot_state(const PhaseConst<NS>& pc, const double s6[6], const double* st, double* dot) {
  double adg[NS];
  kinetics_abs<NS>(pc, s6, st, adg);
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    const double x = 1.0 - st[l] / pc.xiinf[l];
    const double left = copysign(powr(fabs(x), pc.a[l], pc.a_int[l]), x);
    double hg = 0.0;
#pragma unroll
    for (int k = 0; k < NS; ++k) hg = fma(pc.h[l][k], adg[k], hg);
    dot[l] = pc.h0f[l] * left * hg;
    dot[NS + l] = adg[l];
  }
}

// 9x9 LU with partial pivoting (first maximal |a|, as dgetrf) + solve; row-major J.
// Returns true if a pivot is exactly zero (dgesv info > 0).
__device__ __forceinline__ bool lu_solve9(double* J, double* b) {
#pragma unroll
  for (int j = 0; j < 9; ++j) {
    int p = j;
    double amax = fabs(J[j * 9 + j]);
#pragma unroll
    for (int i = j + 1; i < 9; ++i) {
      const double v = fabs(J[i * 9 + j]);
      if (v > amax) { amax = v; p = i; }
    }
    if (amax == 0.0) return true;
    if (p != j) {
#pragma unroll
      for (int k = 0; k < 9; ++k) { const double t = J[j * 9 + k]; J[j * 9 + k] = J[p * 9 + k]; J[p * 9 + k] = t; }
      const double t = b[j]; b[j] = b[p]; b[p] = t;
    }
    const double rp = 1.0 / J[j * 9 + j];
#pragma unroll
    for (int i = j + 1; i < 9; ++i) {
      const double l = J[i * 9 + j] * rp;
#pragma unroll
      for (int k = j + 1; k < 9; ++k) J[i * 9 + k] = fma(-l, J[j * 9 + k], J[i * 9 + k]);
      b[i] = fma(-l, b[j], b[i]);
    }
  }
#pragma unroll
  for (int i = 8; i >= 0; --i) {
    double s = b[i];
#pragma unroll
    for (int k = i + 1; k < 9; ++k) s = fma(-J[i * 9 + k], b[k], s);
    b[i] = s / J[i * 9 + i];
  }
  return false;
}

// Outcome of one integrateStress call kept in registers by the caller.
struct StressOut {
  double S[6];
  double Lp[9];
  double Fp[9];
};

// integrateStress, phase_mechanical.f90:379-584 (Fi = I, Li = 0).
// Lp (in/out) is the warm start / result; on success P and Fe are written through.
template <int NS>
__device__ int integrate_stress(const PhaseConst<NS>& pc, const Numerics& nm, const double* F, const double* Fp0,
                                const double* xi, double dt, double* Lp, double* S, double* Fp,
                                double* Pout, double* Feout, int& newton) {
  double invFp0[9];
  if (inv33(Fp0, invFp0)) return 5;                       // STATUS_FAIL_PHASE_MECHANICAL_STRESS
  double A[9];
  mm33(F, invFp0, A);
  double inv_xi[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) inv_xi[s] = 1.0 / xi[s];

  double Lg[9], Lg_old[9], dL[9], B[9], Fe[9], s6[6];
#pragma unroll
  for (int k = 0; k < 9; ++k) { Lg[k] = Lp[k]; Lg_old[k] = Lp[k]; dL[k] = 0.0; }
  double step = 1.0, res_old = 1.7976931348623157e308;
  int jaco = 0;
  for (int it = 1;; ++it) {
    if (it > nm.N_iter_Lp_max) return 6;                  // STATUS_FAIL_PHASE_MECHANICAL_STRESS_LP_MAXIT
    ++newton;
#pragma unroll
    for (int k = 0; k < 9; ++k) B[k] = ((k % 4 == 0) ? 1.0 : 0.0) - dt * Lg[k];
    mm33(A, B, Fe);
    hooke_S<NS>(pc, Fe, s6);
    // Lp_c and its derivative weights
    double Lc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double w[NS];
    int sense[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const double tp = dot6(s6, pc.p6[0][s]), tn = dot6(s6, pc.p6[1][s]);
      const bool pos = tp > tn;
      const double tmax = pos ? tp : tn;
      const double r = tmax * inv_xi[s];
      double g, dg;
      if (pc.n_int[s] >= 1) {
        const double rn1 = powi(r, pc.n_int[s] - 1);
        const double sd = pos ? pc.dg0[s] : -pc.dg0[s];
        g = sd * (rn1 * r);
        dg = (sd * pc.n[s]) * rn1 * inv_xi[s];
      } else {
        g = (pos ? pc.dg0[s] : -pc.dg0[s]) * pow(r, pc.n[s]);
        dg = g * pc.n[s] / tmax;
      }
      if (!(fabs(g) > TINY10)) dg = 0.0;
      // P_nS sense of the derivative follows the sign of dot_gamma (phenopowerlaw.f90:327)
      sense[s] = g > 0.0 ? 0 : 1;
      w[s] = dt * dg;
#pragma unroll
      for (int k = 0; k < 9; ++k) Lc[k] = fma(g, pc.P[s][k], Lc[k]);
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
      for (int k = 0; k < 9; ++k) Lg_old[k] = Lg[k];
      step = 1.0;
    } else {
      step = nm.r_linesearch_Lp * step;
#pragma unroll
      for (int k = 0; k < 9; ++k) Lg[k] = fma(dL[k], step, Lg_old[k]);
      continue;
    }
    if (jaco % nm.f_update_jacobi_Lp == 0) {
      ++jaco;
      double M[9];
      mtm33(A, Fe, M);                                    // M = A^T Fe
      double J[81], rhs[9];
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int l = 0; l < 3; ++l) {
          const int row = 3 * k + l;
          double H[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
          for (int s = 0; s < NS; ++s) {
            const double c = w[s] * pc.P[s][k + 3 * l];
            const double* q = pc.q6[sense[s]][s];
#pragma unroll
            for (int t = 0; t < 6; ++t) H[t] = fma(c, q[t], H[t]);
          }
          // H as symmetric 3x3: (11,22,33,23,13,12)
          const double Hm[9] = {H[0], H[5], H[4], H[5], H[1], H[3], H[4], H[3], H[2]};
#pragma unroll
          for (int p = 0; p < 3; ++p)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
              const double v = M[p] * Hm[3 * b] + M[p + 3] * Hm[1 + 3 * b] + M[p + 6] * Hm[2 + 3 * b];
              J[row * 9 + 3 * p + b] = (row == 3 * p + b ? 1.0 : 0.0) + v;
            }
          rhs[row] = R[k + 3 * l];                        // math_33to9 (row-major flattening)
        }
      if (lu_solve9(J, rhs)) return 8;                   // STATUS_FAIL_PHASE_MECHANICAL_STRESS_LP_DGESV
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int l = 0; l < 3; ++l) dL[k + 3 * l] = -rhs[3 * k + l];
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) Lg[k] = fma(dL[k], step, Lg[k]);
  }
  // Fp = (Fp0^-1 B)^-1 / det^(1/3); P = F Fp^-1 S Fp^-T; Fe = F Fp^-1  (:571-581)
  double invFpn[9], Fpn[9];
  mm33(invFp0, B, invFpn);
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

// damper, phase_mechanical.f90:653-674
__device__ __forceinline__ double damper(double d01, double d12, double d22) {
  if (fmin(d01, d12) < 0.0 && d22 > 0.0) return 0.75 + 0.25 * tanh(2.0 + 4.0 * d12 / d22);
  return 1.0;
}

// integrateStateFPI, phase_mechanical.f90:591-676.
// S (in/out) is the current stress (S0 after restore), st (in/out) the current state.
template <int NS>
__device__ int integrate_state_fpi(const PhaseConst<NS>& pc, const Numerics& nm, const double* F, const double* Fp0,
                                   const double* st0, double dt, double* st, double* S, double* Lp, double* Fp,
                                   double* Pout, double* Feout, int& nstate, int& newton) {
  constexpr int NST = 2 * NS;
  double dot[NST], last1[NST], last2[NST];
  dot_state<NS>(pc, S, st, dot);
#pragma unroll
  for (int i = 0; i < NST; ++i)
    if (isnan(dot[i])) return 3;                           // STATUS_FAIL_PHASE_MECHANICAL_STATE
#pragma unroll
  for (int i = 0; i < NST; ++i) { st[i] = fma(dot[i], dt, st0[i]); last1[i] = 0.0; }
  int status = 3;
  for (int it = 1; it <= nm.N_iter_state_max; ++it) {
    ++nstate;
#pragma unroll
    for (int i = 0; i < NST; ++i) { last2[i] = it > 1 ? last1[i] : 0.0; last1[i] = dot[i]; }
    status = integrate_stress<NS>(pc, nm, F, Fp0, st, dt, Lp, S, Fp, Pout, Feout, newton);
    if (status != 0) break;
    dot_state<NS>(pc, S, st, dot);
    bool bad = false;
    double d01 = 0.0, d12 = 0.0, d22 = 0.0;
#pragma unroll
    for (int i = 0; i < NST; ++i) {
      bad |= isnan(dot[i]);
      const double a = dot[i] - last1[i], b = last1[i] - last2[i];
      d12 = fma(a, b, d12);
      d22 = fma(b, b, d22);
      d01 = fma(dot[i], last1[i], d01);
    }
    if (bad) break;
    const double zeta = damper(d01, d12, d22);
    bool conv = true;
#pragma unroll
    for (int i = 0; i < NST; ++i) {
      const double d = dot[i] * zeta + last1[i] * (1.0 - zeta);
      dot[i] = d;
      const double r = st[i] - st0[i] - d * dt;
      st[i] = st[i] - r;
      const double atol = i < NS ? pc.atol_xi : pc.atol_gamma;
      conv = conv && (fabs(r) <= fmax(atol, nm.eps_rel_state * fabs(st[i])));
    }
    if (conv) { status = 0; break; }
  }
  return status;
}

// phase_mechanical_constitutive, phase_mechanical.f90:1008-1090, after
// mechanical_restore (Fp := Fp0, S := S0, state := state0; Lp kept as warm start).
template <int NS>
__device__ int constitutive_point(const PhaseConst<NS>& pc, const Numerics& nm, const Fields& f, int64_t v,
                                  const double* Fnew, double dt, int& nstate, int& newton, int& nsub) {
  constexpr int NST = 2 * NS;
  const int64_t N = f.N;
  double F0[9], Fp0s[9], Lp0s[9], Lp[9], Fp[9], S[6], st[NST], st0s[NST], Fs[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    F0[k] = f.F0[k * N + v];
    Fp0s[k] = f.Fp0[k * N + v];
    Lp0s[k] = f.Lp0[k * N + v];
    Lp[k] = f.Lp[k * N + v];
    Fp[k] = Fp0s[k];
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) S[k] = f.S0[k * N + v];
#pragma unroll
  for (int i = 0; i < NST; ++i) { st0s[i] = f.state0[i * N + v]; st[i] = st0s[i]; }
  double Pl[9], Fel[9];
  bool wrote = false;
  double stepFrac = 0.0, step = 1.0 / nm.r_cutback;
  int status = 1;                                         // STATUS_ITERATING
  bool todo = true;
  while (todo) {
    if (status == 0) {
      stepFrac = stepFrac + step;
      step = fmin(1.0 - stepFrac, nm.r_increase * step);
      todo = step > 0.0;
      if (todo) {
#pragma unroll
        for (int k = 0; k < 9; ++k) { F0[k] = Fs[k]; Lp0s[k] = Lp[k]; Fp0s[k] = Fp[k]; }
#pragma unroll
        for (int i = 0; i < NST; ++i) st0s[i] = st[i];
      }
    } else {
      step = nm.r_cutback * step;
#pragma unroll
      for (int k = 0; k < 9; ++k) Fp[k] = Fp0s[k];
#pragma unroll
      for (int k = 0; k < 6; ++k) S[k] = f.S0[k * N + v];
      if (step < 1.0)
#pragma unroll
        for (int k = 0; k < 9; ++k) Lp[k] = Lp0s[k];
#pragma unroll
      for (int i = 0; i < NST; ++i) st[i] = st0s[i];
      todo = step > nm.r_cutback_min;
    }
    if (todo) {
      ++nsub;
#pragma unroll
      for (int k = 0; k < 9; ++k) Fs[k] = fma(step, Fnew[k] - f.F0[k * N + v], F0[k]);
      status = integrate_state_fpi<NS>(pc, nm, Fs, Fp0s, st0s, step * dt, st, S, Lp, Fp, Pl, Fel, nstate, newton);
      if (status == 0) wrote = true;
    }
  }
  // write back the phase containers (current values)
#pragma unroll
  for (int k = 0; k < 9; ++k) { f.Lp[k * N + v] = Lp[k]; f.Fp[k * N + v] = Fp[k]; }
#pragma unroll
  for (int k = 0; k < 6; ++k) f.S[k * N + v] = S[k];
#pragma unroll
  for (int i = 0; i < NST; ++i) f.state[i * N + v] = st[i];
  if (wrote) {
#pragma unroll
    for (int k = 0; k < 9; ++k) { f.P[k * N + v] = Pl[k]; f.Fe[k * N + v] = Fel[k]; }
  }
  return status;
}

}  // namespace dmk
