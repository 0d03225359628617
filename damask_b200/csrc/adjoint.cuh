// Local model of one voxel's increment for the adjoint: the converged constitutive update as an
// implicit function, written once for plain doubles and for dual numbers, on host and device.
//
// With no eigenstrain (Fi = I, Li = 0) and one substep, the converged state of an increment
// solves (integrateStress, phase_mechanical.f90:379-584, and the fixed point of
// integrateStateFPI, :591-676, with phenopowerlaw_LpAndItsTangent / dotState,
// phase_mechanical_plastic_phenopowerlaw.f90:303-399,449-488)
//   G_L = Lp - sum_s dot_gamma_s(S(Lp), xi) P_s                          = 0   (9)
//   G_x = xi - xi0 - dt h_0 sign(1 - xi/xi_inf)|1 - xi/xi_inf|^a (h |dot_gamma|)  = 0   (Ns)
// for the unknowns y = (Lp, xi), given x = (F, Fp0, xi0, theta), theta = per family (xi_inf, h_0,
// n, a).  S = C : (Fe^T Fe - I)/2 with Fe = F Fp0^-1 (I - dt Lp) (phase_hooke_SandItsTangents,
// phase_mechanical_elastic.f90:172-205), dot_gamma_s = sign dot_gamma_0 (max(tau+, tau-)/xi_s)^n.
// The outputs z = (P, Fp, xi) are those of the increment's end (phase_mechanical.f90:571-581):
//   invFp = Fp0^-1 (I - dt Lp),  P = F invFp S invFp^T,  Fp = invFp^-1 det(invFp^-1)^(-1/3).
// The adjoint uses the total derivative dz/dx = dZ/dx - dZ/dy (dG/dy)^-1 dG/dx (implicit-function
// theorem); the partial derivatives come from evaluating G and Z in dual numbers, one seed
// direction per column.  Branch decisions (the sense of the resolved shear, the sign of
// 1 - xi/xi_inf) follow the values, as in the forward kernels.
#pragma once
#include "dmk_device.cuh"

#include <math.h>

#if defined(__CUDACC__)
#define DMK_HD __host__ __device__
#else
#define DMK_HD
#endif

namespace dmk {

// forward-mode dual number: value and one directional derivative
struct Dual {
  double v, d;
};
DMK_HD inline Dual dual(double v, double d = 0.0) { return Dual{v, d}; }
DMK_HD inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
DMK_HD inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
DMK_HD inline Dual operator-(Dual a) { return {-a.v, -a.d}; }
DMK_HD inline Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
DMK_HD inline Dual operator/(Dual a, Dual b) { return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; }
DMK_HD inline Dual operator+(Dual a, double b) { return {a.v + b, a.d}; }
DMK_HD inline Dual operator+(double a, Dual b) { return {a + b.v, b.d}; }
DMK_HD inline Dual operator-(Dual a, double b) { return {a.v - b, a.d}; }
DMK_HD inline Dual operator-(double a, Dual b) { return {a - b.v, -b.d}; }
DMK_HD inline Dual operator*(Dual a, double b) { return {a.v * b, a.d * b}; }
DMK_HD inline Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
DMK_HD inline Dual operator/(Dual a, double b) { return {a.v / b, a.d / b}; }

// a constant of type T (zero derivative)
DMK_HD inline void set_const(double& t, double v) { t = v; }
DMK_HD inline void set_const(Dual& t, double v) { t = Dual{v, 0.0}; }
template <class T>
DMK_HD inline T cst(double v) {
  T t;
  set_const(t, v);
  return t;
}

DMK_HD inline double value(double x) { return x; }
DMK_HD inline double value(Dual x) { return x.v; }
DMK_HD inline double dabs(double x) { return fabs(x); }
DMK_HD inline Dual dabs(Dual x) { return x.v < 0.0 ? -x : x; }
// x^e for x >= 0: d(x^e) = e x^(e-1) dx + x^e ln(x) de (the second term vanishes at x = 0)
DMK_HD inline double dpow(double x, double e) { return pow(x, e); }
DMK_HD inline Dual dpow(Dual x, Dual e) {
  const double p = pow(x.v, e.v);
  double d = 0.0;
  if (x.d != 0.0) d += e.v * pow(x.v, e.v - 1.0) * x.d;
  if (e.d != 0.0 && x.v > 0.0) d += p * log(x.v) * e.d;
  return {p, d};
}
DMK_HD inline Dual dpow(Dual x, double e) {
  const double p = pow(x.v, e);
  return {p, x.d != 0.0 ? e * pow(x.v, e - 1.0) * x.d : 0.0};
}

template <class T>
DMK_HD inline void mm33t(const T* A, const T* B, T* C) {   // C = A B (column-major)
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) C[i + 3 * j] = A[i] * B[3 * j] + A[i + 3] * B[1 + 3 * j] + A[i + 6] * B[2 + 3 * j];
}
template <class T>
DMK_HD inline void mmtr33t(const T* A, const T* B, T* C) {   // C = A B^T
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) C[i + 3 * j] = A[i] * B[j] + A[i + 3] * B[j + 3] + A[i + 6] * B[j + 6];
}
template <class T>
DMK_HD inline T det33t(const T* m) {
  return m[0] * (m[4] * m[8] - m[7] * m[5]) - m[3] * (m[1] * m[8] - m[7] * m[2]) + m[6] * (m[1] * m[5] - m[4] * m[2]);
}
template <class T>
DMK_HD inline void inv33t(const T* A, T* I) {   // Cramer's rule (math_invert33, math.f90:471-509)
  I[0] = A[4] * A[8] - A[7] * A[5];
  I[1] = A[7] * A[2] - A[1] * A[8];
  I[2] = A[1] * A[5] - A[4] * A[2];
  const T det = A[0] * I[0] + A[3] * I[1] + A[6] * I[2];
  I[3] = A[6] * A[5] - A[3] * A[8];
  I[4] = A[0] * A[8] - A[6] * A[2];
  I[5] = A[3] * A[2] - A[0] * A[5];
  I[6] = A[3] * A[7] - A[6] * A[4];
  I[7] = A[6] * A[1] - A[0] * A[7];
  I[8] = A[0] * A[4] - A[3] * A[1];
  for (int k = 0; k < 9; ++k) I[k] = I[k] / det;
}

// Sizes of the local problem for NS slip systems and nf families.
DMK_HD inline int adj_ny(int ns) { return 9 + ns; }                       // unknowns (Lp, xi)
DMK_HD inline int adj_nx(int ns, int nf) { return 18 + ns + 4 * nf; }     // inputs (F, Fp0, xi0, theta)
DMK_HD inline int adj_nz(int ns) { return 18 + ns; }                      // outputs (P, Fp, xi)
constexpr int ADJ_MAX_FAMILIES = 4;
constexpr int ADJ_THETA = 5 * ADJ_MAX_FAMILIES;   // gradient layout: (xi_0, xi_inf, h_0, n, a) x family

// G and Z of one voxel.  y: Lp (9), xi (NS); x: F (9), Fp0 (9), xi0 (NS), theta (4 nf:
// xi_inf[f], h_0[f], n[f], a[f] at theta[p * nf + f]).  G: 9 + NS, Z: 18 + NS.  Systems of
// family -1 (inert padding) keep their constants.  h: the NS x NS hardening matrix (row = reacting
// system), readable by the caller's processor.
template <int NS, class T>
DMK_HD void local_model(const PhaseConst<NS>& pc, const double* __restrict__ h, double dt, const T* y, const T* x,
                        T* G, T* Z) {
  const int nf = pc.nf;
  const T* Lp = y;
  const T* xi = y + 9;
  const T* F = x;
  const T* Fp0 = x + 9;
  const T* xi0 = x + 18;
  const T* th = x + 18 + NS;
  // invFp = Fp0^-1 (I - dt Lp), Fe = F invFp
  T invFp0[9], B[9], invFp[9], Fe[9];
  inv33t(Fp0, invFp0);
  for (int k = 0; k < 9; ++k) B[k] = ((k % 4 == 0) ? 1.0 : 0.0) - dt * Lp[k];
  mm33t(invFp0, B, invFp);
  mm33t(F, invFp, Fe);
  // Hooke, Mandel notation (11,22,33,23,13,12)
  const double W = 1.4142135623730951;
  T E[6], s6[6];
  E[0] = 0.5 * (Fe[0] * Fe[0] + Fe[1] * Fe[1] + Fe[2] * Fe[2] - 1.0);
  E[1] = 0.5 * (Fe[3] * Fe[3] + Fe[4] * Fe[4] + Fe[5] * Fe[5] - 1.0);
  E[2] = 0.5 * (Fe[6] * Fe[6] + Fe[7] * Fe[7] + Fe[8] * Fe[8] - 1.0);
  E[3] = 0.5 * (Fe[3] * Fe[6] + Fe[4] * Fe[7] + Fe[5] * Fe[8]) * W;
  E[4] = 0.5 * (Fe[0] * Fe[6] + Fe[1] * Fe[7] + Fe[2] * Fe[8]) * W;
  E[5] = 0.5 * (Fe[0] * Fe[3] + Fe[1] * Fe[4] + Fe[2] * Fe[5]) * W;
  for (int i = 0; i < 6; ++i) {
    T s = E[0] * pc.C66[i][0];
    for (int k = 1; k < 6; ++k) s = s + E[k] * pc.C66[i][k];
    s6[i] = i < 3 ? s : s / W;
  }
  // kinetics and Lp_c
  T Lc[9], adg[NS];
  for (int k = 0; k < 9; ++k) Lc[k] = cst<T>(0.0);
  for (int s = 0; s < NS; ++s) {
    T tp = s6[0] * pc.p6[0][s][0], tn = s6[0] * pc.p6[1][s][0];
    for (int t = 1; t < 6; ++t) {
      tp = tp + s6[t] * pc.p6[0][s][t];
      tn = tn + s6[t] * pc.p6[1][s][t];
    }
    const bool pos = value(tp) > value(tn);
    const T tmax = pos ? tp : tn;
    const int f = pc.fam[s];
    T n;
    if (f >= 0) n = th[2 * nf + f];
    else n = cst<T>(pc.n[s]);
    const T g = (pos ? pc.dg0[s] : -pc.dg0[s]) * dpow(tmax / xi[s], n);
    for (int k = 0; k < 9; ++k) Lc[k] = Lc[k] + g * pc.P[s][k];
    adg[s] = dabs(g);
  }
  for (int k = 0; k < 9; ++k) G[k] = Lp[k] - Lc[k];
  // dotState of xi, backward Euler residual
  for (int l = 0; l < NS; ++l) {
    const int f = pc.fam[l];
    T xinf, h0, a;
    if (f >= 0) {
      xinf = th[f];
      h0 = th[nf + f] * pc.hfac[l];
      a = th[3 * nf + f];
    } else {
      xinf = cst<T>(pc.xiinf[l]);
      h0 = cst<T>(pc.h0f[l]);
      a = cst<T>(pc.a[l]);
    }
    const T r = 1.0 - xi[l] / xinf;
    const T left = value(r) >= 0.0 ? dpow(dabs(r), a) : -dpow(dabs(r), a);
    T hg = adg[0] * h[l * NS];
    for (int k = 1; k < NS; ++k) hg = hg + adg[k] * h[l * NS + k];
    G[9 + l] = xi[l] - xi0[l] - dt * (h0 * left * hg);
  }
  // outputs
  T Fpn[9], Sm[9], T1[9], P[9];
  inv33t(invFp, Fpn);
  const T cb = dpow(det33t(Fpn), -1.0 / 3.0);
  Sm[0] = s6[0]; Sm[1] = s6[5]; Sm[2] = s6[4];
  Sm[3] = s6[5]; Sm[4] = s6[1]; Sm[5] = s6[3];
  Sm[6] = s6[4]; Sm[7] = s6[3]; Sm[8] = s6[2];
  mmtr33t(Sm, invFp, T1);       // S invFp^T
  mm33t(Fe, T1, P);             // F invFp S invFp^T
  for (int k = 0; k < 9; ++k) {
    Z[k] = P[k];
    Z[9 + k] = Fpn[k] * cb;
  }
  for (int s = 0; s < NS; ++s) Z[18 + s] = xi[s];
}

}  // namespace dmk
