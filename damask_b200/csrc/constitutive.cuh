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
// arrays is static, and the 9x9 Newton system is solved by Householder QR
// (backward stable without a data-dependent row exchange).
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

// Solves J x = b for a row-major 9x9 J (overwritten with R) by Householder QR:
// column k is reflected onto alpha e_k with alpha = -sign(x0) |x|, v = x - alpha e_k,
// H y = y + v (v.y) / (alpha v0).  Returns true when a column of the remaining
// matrix is exactly zero (the matrix is singular; dgesv info > 0).
__device__ __forceinline__ bool qr_solve9(double* J, double* b) {
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    double s2 = 0.0;
#pragma unroll
    for (int i = k; i < 9; ++i) s2 = fma(J[i * 9 + k], J[i * 9 + k], s2);
    if (s2 == 0.0) return true;
    const double sig = sqrt(s2);
    const double x0 = J[k * 9 + k];
    const double alpha = x0 >= 0.0 ? -sig : sig;
    const double v0 = x0 - alpha;
    const double rs = 1.0 / (alpha * v0);
#pragma unroll
    for (int c = k + 1; c < 9; ++c) {
      double d = v0 * J[k * 9 + c];
#pragma unroll
      for (int i = k + 1; i < 9; ++i) d = fma(J[i * 9 + k], J[i * 9 + c], d);
      d *= rs;
      J[k * 9 + c] = fma(d, v0, J[k * 9 + c]);
#pragma unroll
      for (int i = k + 1; i < 9; ++i) J[i * 9 + c] = fma(d, J[i * 9 + k], J[i * 9 + c]);
    }
    {
      double d = v0 * b[k];
#pragma unroll
      for (int i = k + 1; i < 9; ++i) d = fma(J[i * 9 + k], b[i], d);
      d *= rs;
      b[k] = fma(d, v0, b[k]);
#pragma unroll
      for (int i = k + 1; i < 9; ++i) b[i] = fma(d, J[i * 9 + k], b[i]);
    }
    J[k * 9 + k] = alpha;
  }
  if (J[80] == 0.0) return true;
#pragma unroll
  for (int i = 8; i >= 0; --i) {
    double s = b[i];
#pragma unroll
    for (int k = i + 1; k < 9; ++k) s = fma(-J[i * 9 + k], b[k], s);
    b[i] = s / J[i * 9 + i];
  }
  return false;
}

// integrateStress, phase_mechanical.f90:379-584 (Fi = I, Li = 0).
// xs: this thread's shared-memory slots (stride PASS_THREADS) holding 1/xi (first NS)
// and the Newton weights dt*dgamma (next NS).  Lp (in/out) is the warm start and, on
// success, the result; S, Fp, P and Fe are written only on success.
template <int NS>
__device__ int integrate_stress(const PhaseConst<NS>& pc, const Numerics& nm, const double* F, const double* Fp0,
                                double* xs, double dt, double* Lp, double* S, double* Fp, double* Pout, double* Feout,
                                int& newton) {
  double* const sw = xs + NS * PASS_THREADS;
  double invFp0[9];
  if (inv33(Fp0, invFp0)) return 5;                       // STATUS_FAIL_PHASE_MECHANICAL_STRESS
  double A[9];
  mm33(F, invFp0, A);

  double Lg[9], Lg_old[9], dL[9], B[9], s6[6];
#pragma unroll
  for (int k = 0; k < 9; ++k) { Lg[k] = Lp[k]; Lg_old[k] = Lp[k]; dL[k] = 0.0; }
  double step = 1.0, res_old = 1.7976931348623157e308;
  int jaco = 0;
  for (int it = 1;; ++it) {
    if (it > nm.N_iter_Lp_max) return 6;                  // STATUS_FAIL_PHASE_MECHANICAL_STRESS_LP_MAXIT
    ++newton;
#pragma unroll
    for (int k = 0; k < 9; ++k) B[k] = ((k % 4 == 0) ? 1.0 : 0.0) - dt * Lg[k];
    double Fe[9];
    mm33(A, B, Fe);
    hooke_S<NS>(pc, Fe, s6);
    // Lp_c = sum_s dot_gamma_s P_s and the weights of its derivative
    double Lc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    unsigned neg = 0u;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const double tp = dot6(s6, pc.p6[0][s]), tn = dot6(s6, pc.p6[1][s]);
      const bool pos = tp > tn;
      const double tmax = pos ? tp : tn;
      const double r = tmax * xs[s * PASS_THREADS];
      double g, dg;
      if (pc.n_int[s] >= 1) {
        const double rn1 = powi(r, pc.n_int[s] - 1);
        const double sd = pos ? pc.dg0[s] : -pc.dg0[s];
        g = sd * (rn1 * r);
        dg = (sd * pc.n[s]) * rn1 * xs[s * PASS_THREADS];
      } else {
        g = (pos ? pc.dg0[s] : -pc.dg0[s]) * pow(r, pc.n[s]);
        dg = g * pc.n[s] / tmax;
      }
      if (!(fabs(g) > TINY10)) dg = 0.0;
      // P_nS sense of the derivative follows the sign of dot_gamma (phenopowerlaw.f90:327)
      if (!(g > 0.0)) neg |= 1u << s;
      sw[s * PASS_THREADS] = dt * dg;
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
      // H^(kl) = sum_s w_s P_s(k,l) Q_s (symmetric, 11 22 33 23 13 12), row kl = 3k + l
      double H[9][6];
#pragma unroll
      for (int i = 0; i < 9; ++i)
#pragma unroll
        for (int t = 0; t < 6; ++t) H[i][t] = 0.0;
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const double ws = sw[s * PASS_THREADS];
        const bool ng = (neg >> s) & 1u;
        double q[6];
#pragma unroll
        for (int t = 0; t < 6; ++t) q[t] = ng ? pc.q6[1][s][t] : pc.q6[0][s][t];
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
          for (int l = 0; l < 3; ++l) {
            const double c = ws * pc.P[s][k + 3 * l];
#pragma unroll
            for (int t = 0; t < 6; ++t) H[3 * k + l][t] = fma(c, q[t], H[3 * k + l][t]);
          }
      }
      double M[9];
      mtm33(A, Fe, M);                                    // M = A^T Fe
      double J[81], rhs[9];
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int l = 0; l < 3; ++l) {
          const int row = 3 * k + l;
          const double* h = H[row];
          const double Hm[9] = {h[0], h[5], h[4], h[5], h[1], h[3], h[4], h[3], h[2]};
#pragma unroll
          for (int p = 0; p < 3; ++p)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
              const double v = M[p] * Hm[3 * b] + M[p + 3] * Hm[1 + 3 * b] + M[p + 6] * Hm[2 + 3 * b];
              J[row * 9 + 3 * p + b] = (row == 3 * p + b ? 1.0 : 0.0) + v;
            }
          rhs[row] = R[k + 3 * l];                        // math_33to9 (row-major flattening)
        }
      if (qr_solve9(J, rhs)) return 8;                   // STATUS_FAIL_PHASE_MECHANICAL_STRESS_LP_DGESV
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

// phenopowerlaw_dotState (Fi = I => Mp = S; no twins => sumF = 0) at the stored
// stress and state of voxel v, written to this thread's slots: xi rates first, then
// |dot_gamma|.  Returns true if any rate is NaN.
template <int NS>
__device__ bool dot_state_slots(const PhaseConst<NS>& pc, const double s6[6], const double* __restrict__ state,
                                int64_t N, int64_t v, double* xs) {
  double adg[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const double tp = dot6(s6, pc.p6[0][s]), tn = dot6(s6, pc.p6[1][s]);
    const double tmax = tp > tn ? tp : tn;
    adg[s] = fabs(pc.dg0[s] * powr(tmax / state[s * N + v], pc.n[s], pc.n_int[s]));
  }
  bool bad = false;
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    const double x = 1.0 - state[l * N + v] / pc.xiinf[l];
    const double left = copysign(powr(fabs(x), pc.a[l], pc.a_int[l]), x);
    double hg = 0.0;
#pragma unroll
    for (int k = 0; k < NS; ++k) hg = fma(pc.h[l][k], adg[k], hg);
    const double d = pc.h0f[l] * left * hg;
    bad |= isnan(d) || isnan(adg[l]);
    xs[l * PASS_THREADS] = d;
    xs[(NS + l) * PASS_THREADS] = adg[l];
  }
  return bad;
}

// damper, phase_mechanical.f90:653-674
__device__ __forceinline__ double damper(double d01, double d12, double d22) {
  if (fmin(d01, d12) < 0.0 && d22 > 0.0) return 0.75 + 0.25 * tanh(2.0 + 4.0 * d12 / d22);
  return 1.0;
}

// Advances voxel v through the control flow of phase_mechanical_constitutive and
// integrateStateFPI until its next integrateStress (phase PH_STRESS) or its end
// (PH_DONE).  Entered in PH_CTRL (substep control after an integration attempt) or
// PH_DOT1 (state update after a successful integrateStress).
template <int NS>
__device__ void advance(const PhaseConst<NS>& pc, const Numerics& nm, const Fields& f, const PassWork& w, int64_t v,
                        double dt, VoxelCtl& c, double* xs) {
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
          for (int i = 0; i < NST; ++i) w.st0s[i * N + v] = f.state[i * N + v];
        }
      } else {
        c.step = nm.r_cutback * c.step;
#pragma unroll
        for (int k = 0; k < 9; ++k) f.Fp[k * N + v] = w.Fp0s[k * N + v];
#pragma unroll
        for (int k = 0; k < 6; ++k) f.S[k * N + v] = f.S0[k * N + v];
        if (c.step < 1.0)
#pragma unroll
          for (int k = 0; k < 9; ++k) f.Lp[k * N + v] = w.Lp0s[k * N + v];
        for (int i = 0; i < NST; ++i) f.state[i * N + v] = w.st0s[i * N + v];
        todo = c.step > nm.r_cutback_min;
      }
      if (!todo) { c.phase = PH_DONE; break; }
      ++c.nsub;
#pragma unroll
      for (int k = 0; k < 9; ++k)
        w.Fs[k * N + v] = fma(c.step, f.F[k * N + v] - f.F0[k * N + v], w.F0s[k * N + v]);
      c.phase = PH_DOT0;
    } else {
      // dotState at the current stress and state: start (DOT0) or update (DOT1) of a state iteration
      double s6[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) s6[k] = f.S[k * N + v];
      const bool bad = dot_state_slots<NS>(pc, s6, f.state, N, v, xs);
      const double dts = c.step * dt;
      if (c.phase == PH_DOT0) {
        // integrateStateFPI:616-620
        if (bad) { c.status = 3; c.phase = PH_CTRL; continue; }   // STATUS_FAIL_PHASE_MECHANICAL_STATE
        for (int i = 0; i < NST; ++i) {
          const double d = xs[i * PASS_THREADS];
          f.state[i * N + v] = fma(d, dts, w.st0s[i * N + v]);
          w.dot[i * N + v] = d;
        }
        c.it = 0;
        c.phase = PH_STRESS;
      } else {
        // integrateStateFPI:631-646 (the stress integration of this iteration succeeded: status 0)
        if (bad) { c.phase = PH_CTRL; continue; }
        double d01 = 0.0, d12 = 0.0, d22 = 0.0;
        for (int i = 0; i < NST; ++i) {
          const double d = xs[i * PASS_THREADS];
          const double l1 = w.dot[i * N + v];                          // dotState_last(:,1)
          const double l2 = c.it > 1 ? w.last1[i * N + v] : 0.0;      // dotState_last(:,2)
          const double a = d - l1, b = l1 - l2;
          d12 = fma(a, b, d12);
          d22 = fma(b, b, d22);
          d01 = fma(d, l1, d01);
        }
        const double zeta = damper(d01, d12, d22);
        bool conv = true;
        for (int i = 0; i < NST; ++i) {
          const double l1 = w.dot[i * N + v];
          const double d = xs[i * PASS_THREADS] * zeta + l1 * (1.0 - zeta);
          const double st = f.state[i * N + v];
          const double r = st - w.st0s[i * N + v] - d * dts;
          const double stn = st - r;
          f.state[i * N + v] = stn;
          w.last1[i * N + v] = l1;
          w.dot[i * N + v] = d;
          const double atol = i < NS ? pc.atol_xi : pc.atol_gamma;
          conv = conv && (fabs(r) <= fmax(atol, nm.eps_rel_state * fabs(stn)));
        }
        c.phase = (conv || c.it >= nm.N_iter_state_max) ? PH_CTRL : PH_STRESS;
      }
    }
  }
}

}  // namespace dmk
