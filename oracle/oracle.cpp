// ORACLE — test infrastructure only (see oracle.h).  CPU FP64 restatement of the
// DAMASK grid basic spectral scheme and the phenopowerlaw/Hooke constitutive
// update.  Each routine cites the reference file:line it follows.
#include "oracle.h"
#include "lattice_tables.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using cd = std::complex<double>;

// status codes: constants.f90:29-44
enum {
  ST_OK = 0, ST_ITERATING, ST_FAIL_MECH, ST_FAIL_STATE, ST_FAIL_DELTASTATE, ST_FAIL_STRESS,
  ST_FAIL_LP_MAXIT, ST_FAIL_LP_NAN, ST_FAIL_LP_DGESV
};

const double TINY = std::numeric_limits<double>::min();
const double TAU = 6.283185307179586476925286766559;

// ---------------------------------------------------------------- small tensors
struct M3 { double a[3][3]; };
struct T4 { double a[3][3][3][3]; };

inline M3 zero3() { M3 r; std::memset(&r, 0, sizeof r); return r; }
inline M3 eye3() { M3 r = zero3(); r.a[0][0] = r.a[1][1] = r.a[2][2] = 1.0; return r; }
inline M3 mm(const M3& A, const M3& B) {            // matmul
  M3 C;
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) {
    double s = 0.0;
    for (int k = 0; k < 3; ++k) s += A.a[i][k] * B.a[k][j];
    C.a[i][j] = s;
  }
  return C;
}
inline M3 tr(const M3& A) { M3 C; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) C.a[i][j] = A.a[j][i]; return C; }
inline M3 add(const M3& A, const M3& B) { M3 C; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) C.a[i][j] = A.a[i][j] + B.a[i][j]; return C; }
inline M3 sub(const M3& A, const M3& B) { M3 C; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) C.a[i][j] = A.a[i][j] - B.a[i][j]; return C; }
inline M3 scl(double s, const M3& A) { M3 C; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) C.a[i][j] = s * A.a[i][j]; return C; }
// sum(A*B) in Fortran column-major order (math_tensordot, math.f90:373)
inline double ddot33(const M3& A, const M3& B) {
  double s = 0.0;
  for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) s += A.a[i][j] * B.a[i][j];
  return s;
}
// gfortran norm2: scaled sum of squares, column-major
inline double norm2_(const double* x, int n) {
  double scale = 0.0, ssq = 1.0;
  for (int i = 0; i < n; ++i) {
    if (x[i] != 0.0) {
      double ax = std::fabs(x[i]);
      if (scale < ax) { ssq = 1.0 + ssq * (scale / ax) * (scale / ax); scale = ax; }
      else ssq += (ax / scale) * (ax / scale);
    }
  }
  return scale * std::sqrt(ssq);
}
inline double norm33(const M3& A) {
  double v[9];
  for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) v[3 * j + i] = A.a[i][j];
  return norm2_(v, 9);
}
inline bool anynan(const M3& A) {
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) if (std::isnan(A.a[i][j])) return true;
  return false;
}
// math_det33, math.f90:626
inline double det33(const M3& m) {
  const auto& a = m.a;
  return a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1])
       - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0])
       + a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
}
// math_invert33, math.f90:471-509 (Cramer; error if |det| <= 10*tiny)
inline bool invert33(M3& inv, const M3& m, double* detOut = nullptr) {
  const auto& A = m.a;
  auto& I = inv.a;
  I[0][0] = A[1][1] * A[2][2] - A[1][2] * A[2][1];
  I[1][0] = -A[1][0] * A[2][2] + A[1][2] * A[2][0];
  I[2][0] = A[1][0] * A[2][1] - A[1][1] * A[2][0];
  double det = A[0][0] * I[0][0] + A[0][1] * I[1][0] + A[0][2] * I[2][0];
  if (std::fabs(det) <= TINY * 10.0) {
    inv = zero3();
    if (detOut) *detOut = 0.0;
    return true;
  }
  I[0][1] = -A[0][1] * A[2][2] + A[0][2] * A[2][1];
  I[1][1] = A[0][0] * A[2][2] - A[0][2] * A[2][0];
  I[2][1] = -A[0][0] * A[2][1] + A[0][1] * A[2][0];
  I[0][2] = A[0][1] * A[1][2] - A[0][2] * A[1][1];
  I[1][2] = -A[0][0] * A[1][2] + A[0][2] * A[1][0];
  I[2][2] = A[0][0] * A[1][1] - A[0][1] * A[1][0];
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) I[i][j] /= det;
  if (detOut) *detOut = det;
  return false;
}
inline M3 inv33(const M3& m) { M3 r; invert33(r, m); return r; }   // math_inv33, math.f90:452

// math_mul3333xx3333, math.f90:405 (sum over a 3x3 section, column-major)
T4 mul4x4(const T4& A, const T4& B) {
  T4 C;
  for (int l = 0; l < 3; ++l) for (int k = 0; k < 3; ++k) for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) {
    double s = 0.0;
    for (int n = 0; n < 3; ++n) for (int m = 0; m < 3; ++m) s += A.a[i][j][m][n] * B.a[m][n][k][l];
    C.a[i][j][k][l] = s;
  }
  return C;
}
// math_mul3333xx33, math.f90:387
M3 mul4x2(const T4& A, const M3& B) {
  M3 C;
  for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) {
    double s = 0.0;
    for (int n = 0; n < 3; ++n) for (int m = 0; m < 3; ++m) s += A.a[i][j][m][n] * B.a[m][n];
    C.a[i][j] = s;
  }
  return C;
}
// math_3333to99 / math_99to3333 (math.f90:736,762): row 3i+j, column 3k+l
void to99(const T4& T, double* M) {
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) for (int k = 0; k < 3; ++k) for (int l = 0; l < 3; ++l)
    M[(3 * i + j) * 9 + (3 * k + l)] = T.a[i][j][k][l];
}
T4 from99(const double* M) {
  T4 T;
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) for (int k = 0; k < 3; ++k) for (int l = 0; l < 3; ++l)
    T.a[i][j][k][l] = M[(3 * i + j) * 9 + (3 * k + l)];
  return T;
}

// ---------------------------------------------------------------- LAPACK-like LU
// dgetrf (unblocked, partial pivoting, first maximal |a|): A row-major n x n.
int lu_factor(double* A, int n, int* piv) {
  int info = 0;
  for (int j = 0; j < n; ++j) {
    int p = j;
    double amax = std::fabs(A[j * n + j]);
    for (int i = j + 1; i < n; ++i) if (std::fabs(A[i * n + j]) > amax) { amax = std::fabs(A[i * n + j]); p = i; }
    piv[j] = p;
    if (A[p * n + j] != 0.0) {
      if (p != j) for (int k = 0; k < n; ++k) std::swap(A[j * n + k], A[p * n + k]);
      double r = 1.0 / A[j * n + j];
      for (int i = j + 1; i < n; ++i) A[i * n + j] *= r;
    } else if (info == 0) {
      info = j + 1;
    }
    for (int i = j + 1; i < n; ++i) {
      double l = A[i * n + j];
      for (int k = j + 1; k < n; ++k) A[i * n + k] -= l * A[j * n + k];
    }
  }
  return info;
}
void lu_solve(const double* LU, int n, const int* piv, double* b) {   // dgetrs, one right-hand side
  for (int j = 0; j < n; ++j) if (piv[j] != j) std::swap(b[j], b[piv[j]]);
  for (int i = 1; i < n; ++i) { double s = b[i]; for (int k = 0; k < i; ++k) s -= LU[i * n + k] * b[k]; b[i] = s; }
  for (int i = n - 1; i >= 0; --i) {
    double s = b[i];
    for (int k = i + 1; k < n; ++k) s -= LU[i * n + k] * b[k];
    b[i] = s / LU[i * n + i];
  }
}
// math_invert (dgetrf + dgetri), math.f90:538-556; returns true on error
bool invert_n(double* Ainv, const double* A, int n) {
  std::vector<double> LU(A, A + n * n);
  std::vector<int> piv(n);
  int info = lu_factor(LU.data(), n, piv.data());
  if (info) return true;
  std::vector<double> col(n);
  for (int c = 0; c < n; ++c) {
    for (int r = 0; r < n; ++r) col[r] = (r == c) ? 1.0 : 0.0;
    lu_solve(LU.data(), n, piv.data(), col.data());
    for (int r = 0; r < n; ++r) Ainv[r * n + c] = col[r];
  }
  return false;
}

// ---------------------------------------------------------------- rotations
// qu2om, rotations.f90:399-423 (P = -1 => transpose; renormalise by det^(1/3))
M3 qu2om(const double q[4]) {
  M3 om;
  double qq = q[0] * q[0] - (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  om.a[0][0] = qq + 2.0 * q[1] * q[1];
  om.a[1][1] = qq + 2.0 * q[2] * q[2];
  om.a[2][2] = qq + 2.0 * q[3] * q[3];
  om.a[0][1] = 2.0 * (q[1] * q[2] - q[0] * q[3]);
  om.a[1][2] = 2.0 * (q[2] * q[3] - q[0] * q[1]);
  om.a[2][0] = 2.0 * (q[3] * q[1] - q[0] * q[2]);
  om.a[1][0] = 2.0 * (q[2] * q[1] + q[0] * q[3]);
  om.a[2][1] = 2.0 * (q[3] * q[2] + q[0] * q[1]);
  om.a[0][2] = 2.0 * (q[1] * q[3] + q[0] * q[2]);
  om = tr(om);
  double d = std::pow(det33(om), 1.0 / 3.0);
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) om.a[i][j] /= d;
  return om;
}
// rotate_vector, rotations.f90:776-791 (P = -1)
void rotvec(const double v[3], const double q[4], double out[3]) {
  double A = q[0] * q[0] - (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  double B = 2.0 * (q[1] * v[0] + q[2] * v[1] + q[3] * v[2]);
  double C = 2.0 * -1.0 * q[0];
  double cx = q[2] * v[2] - q[3] * v[1], cy = q[3] * v[0] - q[1] * v[2], cz = q[1] * v[1] - q[2] * v[0];
  out[0] = A * v[0] + B * q[1] + C * cx;
  out[1] = A * v[1] + B * q[2] + C * cy;
  out[2] = A * v[2] + B * q[3] + C * cz;
}
// rotate3x3, rotations.f90:282-303; active => conjugate quaternion
M3 rot33(const double qin[4], const M3& T, bool active) {
  double q[4] = {qin[0], active ? -qin[1] : qin[1], active ? -qin[2] : qin[2], active ? -qin[3] : qin[3]};
  M3 R;
  for (int i = 0; i < 3; ++i) { double v[3] = {T.a[i][0], T.a[i][1], T.a[i][2]}, o[3]; rotvec(v, q, o); for (int j = 0; j < 3; ++j) R.a[i][j] = o[j]; }
  for (int j = 0; j < 3; ++j) { double v[3] = {R.a[0][j], R.a[1][j], R.a[2][j]}, o[3]; rotvec(v, q, o); for (int i = 0; i < 3; ++i) R.a[i][j] = o[i]; }
  return R;
}
// rotate3x3x3x3, rotations.f90:310-339 (passive)
T4 rot3333(const double q[4], const T4& T) {
  T4 R = T;
  double v[3], o[3];
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) for (int k = 0; k < 3; ++k) {
    for (int l = 0; l < 3; ++l) v[l] = R.a[i][j][k][l];
    rotvec(v, q, o); for (int l = 0; l < 3; ++l) R.a[i][j][k][l] = o[l];
  }
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) for (int l = 0; l < 3; ++l) {
    for (int k = 0; k < 3; ++k) v[k] = R.a[i][j][k][l];
    rotvec(v, q, o); for (int k = 0; k < 3; ++k) R.a[i][j][k][l] = o[k];
  }
  for (int i = 0; i < 3; ++i) for (int k = 0; k < 3; ++k) for (int l = 0; l < 3; ++l) {
    for (int j = 0; j < 3; ++j) v[j] = R.a[i][j][k][l];
    rotvec(v, q, o); for (int j = 0; j < 3; ++j) R.a[i][j][k][l] = o[j];
  }
  for (int j = 0; j < 3; ++j) for (int k = 0; k < 3; ++k) for (int l = 0; l < 3; ++l) {
    for (int i = 0; i < 3; ++i) v[i] = R.a[i][j][k][l];
    rotvec(v, q, o); for (int i = 0; i < 3; ++i) R.a[i][j][k][l] = o[i];
  }
  return R;
}

// ---------------------------------------------------------------- phase constants
struct PhaseC {
  int Ns;
  double C66[6][6];
  T4 C;
  std::vector<M3> P_sl, P_pos, P_neg;
  std::vector<double> dg0, n, a, h0, xi0, xiinf, c1, c2, fsat;
  std::vector<double> h;   // Ns x Ns, row = reacting
  double atol_xi, atol_gamma;
};

const double SQRT2 = std::sqrt(2.0);

// crystal_assembleStiffness, crystal.f90:1711-1759 (cubic)
void assemble_stiffness(double C11, double C12, double C44, double Ct[6][6]) {
  std::memset(Ct, 0, sizeof(double) * 36);
  Ct[0][0] = C11; Ct[1][1] = C11; Ct[0][1] = C12;
  Ct[3][3] = C44 * 2.0; Ct[4][4] = C44 * 2.0;
  Ct[2][2] = C11; Ct[0][2] = C12; Ct[1][2] = C12; Ct[5][5] = C44 * 2.0;
  for (int i = 0; i < 3; ++i) for (int j = i + 1; j < 3; ++j) Ct[j][i] = Ct[i][j];
}
// math_66toSym3333, math.f90:851
T4 m66toSym3333(const double m[6][6]) {
  T4 t;
  const double I1 = 1.0 / SQRT2, I2 = 1.0 / 2.0;
  auto blk = [&](int col, double wd, double ws, M3& out) {
    out.a[0][0] = m[0][col] * wd; out.a[1][0] = m[5][col] * ws; out.a[2][0] = m[4][col] * ws;
    out.a[0][1] = m[5][col] * ws; out.a[1][1] = m[1][col] * wd; out.a[2][1] = m[3][col] * ws;
    out.a[0][2] = m[4][col] * ws; out.a[1][2] = m[3][col] * ws; out.a[2][2] = m[2][col] * wd;
  };
  M3 b;
  const int kl[6][2] = {{0, 0}, {1, 1}, {2, 2}, {1, 2}, {0, 2}, {0, 1}};
  for (int c = 0; c < 6; ++c) {
    if (c < 3) blk(c, 1.0, I1, b); else blk(c, I1, I2, b);
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) {
      t.a[i][j][kl[c][0]][kl[c][1]] = b.a[i][j];
      t.a[i][j][kl[c][1]][kl[c][0]] = b.a[i][j];
    }
  }
  return t;
}
// math_sym33to6 / math_6toSym33, math.f90:792-830
void sym33to6(const M3& m, double v[6]) {
  v[0] = m.a[0][0]; v[1] = m.a[1][1]; v[2] = m.a[2][2];
  v[3] = m.a[2][1] * SQRT2; v[4] = m.a[2][0] * SQRT2; v[5] = m.a[1][0] * SQRT2;
}
M3 m6toSym33(const double v[6]) {
  const double I1 = 1.0 / SQRT2;
  M3 m;
  m.a[0][0] = v[0];      m.a[1][0] = v[5] * I1; m.a[2][0] = v[4] * I1;
  m.a[0][1] = v[5] * I1; m.a[1][1] = v[1];      m.a[2][1] = v[3] * I1;
  m.a[0][2] = v[4] * I1; m.a[1][2] = v[3] * I1; m.a[2][2] = v[2];
  return m;
}
inline M3 outer(const double a[3], const double b[3]) { M3 r; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) r.a[i][j] = a[i] * b[j]; return r; }
inline void cross(const double a[3], const double b[3], double c[3]) {
  c[0] = a[1] * b[2] - a[2] * b[1]; c[1] = a[2] * b[0] - a[0] * b[2]; c[2] = a[0] * b[1] - a[1] * b[0];
}

// buildCoordinateSystem (crystal.f90:1937-2001) + crystal_SchmidMatrix_slip (:1348-1454)
std::vector<M3> schmid(const orc_phase& p, int sense, bool nonSchmid) {
  const int nfam_max = p.lattice == 0 ? 2 : 3;
  const int* NslipMax = p.lattice == 0 ? CF_NSLIP_FAMILY : CI_NSLIP_FAMILY;
  std::vector<M3> out;
  int base = 0;
  for (int f = 0; f < p.n_families && f < nfam_max; ++f) {
    for (int s = 0; s < p.N_sl[f]; ++s) {
      const signed char* sys = p.lattice == 0 ? CF_SLIP_SYSTEMS[base + s] : CI_SLIP_SYSTEMS[base + s];
      double d[3] = {double(sys[0]), double(sys[1]), double(sys[2])};
      double nn[3] = {double(sys[3]), double(sys[4]), double(sys[5])};
      double nd = norm2_(d, 3), nnrm = norm2_(nn, 3);
      for (int i = 0; i < 3; ++i) { d[i] = d[i] / nd * double(sense); nn[i] = nn[i] / nnrm; }
      M3 P = outer(d, nn);
      if (nonSchmid && p.lattice == 1 && f == 0 && p.n_nonschmid > 0) {
        double coeff[6] = {0, 0, 0, 0, 0, 0};
        for (int c = 0; c < p.n_nonschmid; ++c) coeff[c] = p.a_nonschmid[c];
        // R%fromAxisAngle([direction,60],degrees,P=1): axis negated for P=+1 (rotations.f90:192-213)
        double ang = 60.0 * (TAU / 2.0) / 180.0;
        double c = std::cos(ang * 0.5), sn = std::sin(ang * 0.5);
        double q[4] = {c, -d[0] * sn, -d[1] * sn, -d[2] * sn};
        double np[3];
        rotvec(nn, q, np);                          // R%rotate(normal), passive
        double nxd[3], npxd[3];
        cross(nn, d, nxd); cross(np, d, npxd);
        P = add(P, scl(coeff[0], outer(d, np)));
        P = add(P, scl(coeff[1], outer(nxd, nn)));
        P = add(P, scl(coeff[2], outer(npxd, np)));
        P = add(P, scl(coeff[3], outer(nn, nn)));
        P = add(P, scl(coeff[4], outer(nxd, nxd)));
        P = add(P, scl(coeff[5], outer(d, d)));
      }
      out.push_back(P);
    }
    base += NslipMax[f];
  }
  return out;
}

// crystal_interaction_SlipBySlip + buildInteraction, crystal.f90:591-902,1893-1930
std::vector<double> interaction(const orc_phase& p, int& Ns) {
  const int nfam_max = p.lattice == 0 ? 2 : 3;
  const int* NslipMax = p.lattice == 0 ? CF_NSLIP_FAMILY : CI_NSLIP_FAMILY;
  Ns = 0;
  for (int f = 0; f < p.n_families; ++f) Ns += p.N_sl[f];
  std::vector<double> h(Ns * Ns, 0.0);
  int ai = 0;
  for (int fa = 0; fa < p.n_families && fa < nfam_max; ++fa) {
    int aoff = 0; for (int q = 0; q < fa; ++q) aoff += NslipMax[q];
    for (int sa = 0; sa < p.N_sl[fa]; ++sa, ++ai) {
      int ri = 0;
      for (int fr = 0; fr < p.n_families && fr < nfam_max; ++fr) {
        int roff = 0; for (int q = 0; q < fr; ++q) roff += NslipMax[q];
        for (int sr = 0; sr < p.N_sl[fr]; ++sr, ++ri) {
          int ga = aoff + sa, gr = roff + sr;
          int type = p.lattice == 0 ? CF_INTERACTION[gr][ga] : CI_INTERACTION[gr][ga];
          if (type > p.n_h) return {};            // IO_error 138
          h[ri * Ns + ai] = p.h_sl_sl[type - 1];
        }
      }
    }
  }
  return h;
}

bool build_phase(const orc_phase& p, PhaseC& pc) {
  int Ns;
  pc.h = interaction(p, Ns);
  if (pc.h.empty() && Ns > 0) return false;
  pc.Ns = Ns;
  assemble_stiffness(p.C11, p.C12, p.C44, pc.C66);
  pc.C = m66toSym3333(pc.C66);
  pc.P_sl = schmid(p, +1, false);
  pc.P_pos = schmid(p, +1, true);
  pc.P_neg = schmid(p, -1, true);
  auto expand = [&](const double* v) { std::vector<double> r; for (int f = 0; f < p.n_families; ++f) for (int s = 0; s < p.N_sl[f]; ++s) r.push_back(v[f]); return r; };
  pc.dg0 = expand(p.dot_gamma_0); pc.n = expand(p.n); pc.a = expand(p.a); pc.h0 = expand(p.h_0);
  pc.xi0 = expand(p.xi_0); pc.xiinf = expand(p.xi_inf); pc.c1 = expand(p.c_1); pc.c2 = expand(p.c_2); pc.fsat = expand(p.f_sat);
  pc.atol_xi = p.atol_xi; pc.atol_gamma = p.atol_gamma;
  return true;
}

// ---------------------------------------------------------------- FFT
struct FFT1 {
  int n;
  std::vector<cd> tw;    // exp(-2 pi i k / n)
  std::vector<int> fac;
  explicit FFT1(int n_) : n(n_), tw(n_) {
    for (int k = 0; k < n; ++k) { double ang = -TAU * double(k) / double(n); tw[k] = cd(std::cos(ang), std::sin(ang)); }
    int m = n;
    for (int p : {4, 2, 3, 5}) while (m % p == 0) { fac.push_back(p); m /= p; }
    for (int p = 7; m > 1; p += 2) while (m % p == 0) { fac.push_back(p); m /= p; }
  }
  // recursive decimation in time; out[k] = sum_j in[j*stride] w^(sign jk)
  void rec(const cd* in, int stride, cd* out, int len, int fi, int sign, cd* scratch) const {
    if (len == 1) { out[0] = in[0]; return; }
    int p = fac[fi], m = len / p;
    for (int r = 0; r < p; ++r) rec(in + r * stride, stride * p, out + r * m, m, fi + 1, sign, scratch);
    int step = n / len;
    cd tmp[64];
    for (int k = 0; k < m; ++k) {
      for (int r = 0; r < p; ++r) tmp[r] = out[r * m + k];
      for (int q = 0; q < p; ++q) {
        cd s = 0.0;
        for (int r = 0; r < p; ++r) {
          long e = (long(r) * (k + q * m)) % len;
          cd w = tw[e * step];
          if (sign > 0) w = std::conj(w);
          s += tmp[r] * w;
        }
        scratch[q] = s;
      }
      for (int q = 0; q < p; ++q) out[q * m + k] = scratch[q];
    }
  }
  void run(cd* x, int sign) const {
    std::vector<cd> in(x, x + n), scratch(64);
    rec(in.data(), 1, x, n, 0, sign, scratch.data());
  }
};

void fft3(cd* data, const int nn[3], int sign) {
  const int n0 = nn[0], n1 = nn[1], n2 = nn[2];
  FFT1 f0(n0), f1(n1), f2(n2);
  #pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < n2; ++z) for (int y = 0; y < n1; ++y) f0.run(data + (long(z) * n1 + y) * n0, sign);
  #pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < n2; ++z) for (int x = 0; x < n0; ++x) {
    std::vector<cd> line(n1);
    for (int y = 0; y < n1; ++y) line[y] = data[(long(z) * n1 + y) * n0 + x];
    f1.run(line.data(), sign);
    for (int y = 0; y < n1; ++y) data[(long(z) * n1 + y) * n0 + x] = line[y];
  }
  #pragma omp parallel for collapse(2) schedule(static)
  for (int y = 0; y < n1; ++y) for (int x = 0; x < n0; ++x) {
    std::vector<cd> line(n2);
    for (int z = 0; z < n2; ++z) line[z] = data[(long(z) * n1 + y) * n0 + x];
    f2.run(line.data(), sign);
    for (int z = 0; z < n2; ++z) data[(long(z) * n1 + y) * n0 + x] = line[z];
  }
}

}  // namespace

// ==================================================================== context
struct orc_ctx {
  int cells[3];
  double geomSize[3];
  long N;
  double wgt;
  int nthreads;
  orc_numerics num;
  orc_phase phase;
  PhaseC pc;
  int sizeState;
  // phase_mechanical.f90:7-23 containers (per voxel)
  std::vector<M3> F, F0, Fp, Fp0, Fi, Fi0, Li, Li0, Lp, Lp0, S, S0, Fe, P;
  std::vector<double> state, state0;
  std::vector<M3> homP;
  std::vector<T4> homdPdF;
  // spectral
  int red;                        // cells1/2+1
  double scaledGeomSize[3];
  std::vector<cd> xi;             // xi1st, 3 per Fourier point, index ((z*n1+y)*red+x)
  T4 C_ref;
  std::vector<cd> work;           // full complex workspace, 9 components
  std::vector<double> xp, xn;     // discretization_IPcoords / _NodeCoords, 3 per point
  // basic solver (grid_mech_spectral_basic.f90:30-45)
  std::vector<M3> Fsol, F_lastinc, Fdot;
  // polarization solver (grid_mech_spectral_polarization.f90:61-95)
  std::vector<M3> Ftau, Ftau_lastinc, Ftaudot;
  T4 C_scale, S_scale;
  double err_curl = 0.0;
  M3 F_aim, F_aim_lastinc, F_aimDot, P_aim, P_av;
  T4 C_volAvg, C_volAvgLastInc, C_minMaxAvg, C_minMaxAvgLastInc, C_minMaxAvgRestart, Scomp;
  bool stress_mask[3][3];
  double rot_q[4];
  double dt;
  int totalIter;
  double err_div, err_BC;
  int status;
  int64_t counters[4];
};

namespace {

// ---------------------------------------------------------------- constitutive
// phase_hooke_SandItsTangents, phase_mechanical_elastic.f90:172-205
void hooke(const orc_ctx* c, M3& S, T4* dS_dFe, T4* dS_dFi, const M3& Fe, const M3& Fi) {
  const T4& C = c->pc.C;
  M3 E = scl(0.5, sub(mm(tr(Fe), Fe), eye3()));
  double v6[6], s6[6];
  sym33to6(mm(mm(tr(Fi), E), Fi), v6);
  for (int i = 0; i < 6; ++i) { double s = 0.0; for (int k = 0; k < 6; ++k) s += c->pc.C66[i][k] * v6[k]; s6[i] = s; }
  S = m6toSym33(s6);
  if (!dS_dFe) return;
  M3 EFi2 = scl(2.0, mm(E, Fi));
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) {
    M3 Cij; for (int k = 0; k < 3; ++k) for (int l = 0; l < 3; ++l) Cij.a[k][l] = C.a[i][j][k][l];
    M3 a = mm(Fe, mm(mm(Fi, Cij), tr(Fi)));
    M3 b = mm(EFi2, Cij);
    for (int k = 0; k < 3; ++k) for (int l = 0; l < 3; ++l) { dS_dFe->a[i][j][k][l] = a.a[k][l]; dS_dFi->a[i][j][k][l] = b.a[k][l]; }
  }
}

// kinetics_sl, phase_mechanical_plastic_phenopowerlaw.f90:449-488
void kinetics_sl(const PhaseC& pc, const M3& Mp, const double* xi, double* dg, double* ddg) {
  for (int i = 0; i < pc.Ns; ++i) {
    double tp = ddot33(Mp, pc.P_pos[i]), tn = ddot33(Mp, pc.P_neg[i]);
    double tmax = std::max(tp, tn);
    dg[i] = ((tp > tn ? 1.0 : -1.0) * pc.dg0[i]) * std::pow(tmax / xi[i], pc.n[i]);
    if (ddg) ddg[i] = (std::fabs(dg[i]) > TINY * 10.0) ? dg[i] * pc.n[i] / tmax : 0.0;
  }
}

// plastic_LpAndItsTangents (phase_mechanical_plastic.f90:239-298) with
// phenopowerlaw_LpAndItsTangent (phenopowerlaw.f90:303-350)
void lp_tangents(const orc_ctx* c, M3& Lp, T4* dLp_dS, T4* dLp_dFi, const M3& S, const M3& Fi, const double* xi) {
  const PhaseC& pc = c->pc;
  M3 FtF = mm(tr(Fi), Fi);
  M3 Mp = mm(FtF, S);
  std::vector<double> dg(pc.Ns), ddg(pc.Ns);
  kinetics_sl(pc, Mp, xi, dg.data(), ddg.data());
  Lp = zero3();
  T4 dLp_dMp; std::memset(&dLp_dMp, 0, sizeof dLp_dMp);
  for (int i = 0; i < pc.Ns; ++i) {
    const M3& PnS = dg[i] > 0.0 ? pc.P_pos[i] : pc.P_neg[i];
    Lp = add(Lp, scl(dg[i], pc.P_sl[i]));
    for (int k = 0; k < 3; ++k) for (int l = 0; l < 3; ++l) for (int m = 0; m < 3; ++m) for (int n = 0; n < 3; ++n)
      dLp_dMp.a[k][l][m][n] += ddg[i] * pc.P_sl[i].a[k][l] * PnS.a[m][n];
  }
  if (!dLp_dS) return;
  M3 FiS = mm(Fi, S);
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) {
    M3 D; for (int k = 0; k < 3; ++k) for (int l = 0; l < 3; ++l) D.a[k][l] = dLp_dMp.a[i][j][k][l];
    M3 a = add(mm(FiS, tr(D)), mm(mm(Fi, D), S));
    M3 b = mm(FtF, D);
    for (int k = 0; k < 3; ++k) for (int l = 0; l < 3; ++l) { dLp_dFi->a[i][j][k][l] = a.a[k][l]; dLp_dS->a[i][j][k][l] = b.a[k][l]; }
  }
}

// phenopowerlaw_dotState (phenopowerlaw.f90:356-399) via plastic_dotState (phase_mechanical_plastic.f90:304-345)
void dot_state(const orc_ctx* c, long en, double* dot) {
  const PhaseC& pc = c->pc;
  const int Ns = pc.Ns;
  M3 Mp = mm(mm(tr(c->Fi[en]), c->Fi[en]), c->S[en]);
  const double* xi = &c->state[en * c->sizeState];
  std::vector<double> dg(Ns);
  kinetics_sl(pc, Mp, xi, dg.data(), nullptr);
  for (int i = 0; i < Ns; ++i) dg[i] = std::fabs(dg[i]);
  const double sumF = 0.0;   // no twin systems
  for (int l = 0; l < Ns; ++l) {
    double off = pc.fsat[l] * std::sqrt(sumF);
    double x = 1.0 - xi[l] / (pc.xiinf[l] + off);
    double left = std::copysign(std::pow(std::fabs(x), pc.a[l]), x);
    double hg = 0.0;
    for (int k = 0; k < Ns; ++k) hg += pc.h[l * Ns + k] * dg[k];
    dot[l] = pc.h0[l] * (1.0 + pc.c1[l] * std::pow(sumF, pc.c2[l])) * left * hg + 0.0;
    dot[Ns + l] = dg[l];
  }
}

// integrateStress, phase_mechanical.f90:379-584
int integrate_stress(orc_ctx* c, long en, const M3& F, const M3& Fp0, const M3& Fi0, double dt) {
  const orc_numerics& nm = c->num;
  int status = ST_FAIL_STRESS;
  M3 Lpguess = c->Lp[en], Liguess = c->Li[en];
  M3 invFp_current, invFi_current;
  if (invert33(invFp_current, Fp0)) return status;
  if (invert33(invFi_current, Fi0)) return status;
  M3 A = mm(F, invFp_current);
  const double* xi = &c->state[en * c->sizeState];

  int jacoCounterLi = 0;
  double steplengthLi = 1.0;
  M3 Liguess_old = Liguess, deltaLi = zero3();
  double residuumLi_old_norm = std::numeric_limits<double>::max();
  int NiterLi = 0;
  M3 B, Fe, S, invFi_new, Fi_new, Lpguess_old, deltaLp = zero3();
  T4 dS_dFe, dS_dFi, dLp_dS, dLp_dFi;
  for (;;) {   // LiLoop
    NiterLi++;
    if (NiterLi > nm.N_iter_Li_max) return status;
    invFi_new = mm(invFi_current, sub(eye3(), scl(dt, Liguess)));
    Fi_new = inv33(invFi_new);
    int jacoCounterLp = 0;
    double steplengthLp = 1.0;
    Lpguess_old = Lpguess;
    double residuumLp_old_norm = std::numeric_limits<double>::max();
    int NiterLp = 0;
    for (;;) {   // LpLoop
      NiterLp++;
      #pragma omp atomic
      c->counters[2]++;
      if (NiterLp > nm.N_iter_Lp_max) return ST_FAIL_LP_MAXIT;
      B = sub(eye3(), scl(dt, Lpguess));
      Fe = mm(mm(A, B), invFi_new);
      hooke(c, S, &dS_dFe, &dS_dFi, Fe, Fi_new);
      M3 Lp_c;
      lp_tangents(c, Lp_c, &dLp_dS, &dLp_dFi, S, Fi_new, xi);
      double atol_Lp = std::max(nm.eps_rel_Lp * std::max(norm33(Lpguess), norm33(Lp_c)), nm.eps_abs_Lp);
      M3 residuumLp = sub(Lpguess, Lp_c);
      double rn = norm33(residuumLp);
      if (anynan(residuumLp)) return ST_FAIL_LP_NAN;
      else if (rn < atol_Lp) break;
      else if (rn < residuumLp_old_norm) {
        residuumLp_old_norm = rn;
        Lpguess_old = Lpguess;
        steplengthLp = 1.0;
      } else {
        steplengthLp = nm.r_linesearch_Lp * steplengthLp;
        Lpguess = add(Lpguess_old, scl(steplengthLp, deltaLp));
        continue;
      }
      if (jacoCounterLp % nm.f_update_jacobi_Lp == 0) {
        jacoCounterLp++;
        T4 dFe_dLp;
        M3 invFiT = tr(invFi_new);
        for (int o = 0; o < 3; ++o) for (int p = 0; p < 3; ++p)
          for (int j = 0; j < 3; ++j) for (int l = 0; l < 3; ++l)
            dFe_dLp.a[o][j][p][l] = -dt * A.a[o][p] * invFiT.a[j][l];
        T4 prod = mul4x4(mul4x4(dLp_dS, dS_dFe), dFe_dLp);
        double J[81];
        to99(prod, J);
        for (int i = 0; i < 81; ++i) J[i] = ((i / 9 == i % 9) ? 1.0 : 0.0) - J[i];
        double rhs[9];
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) rhs[3 * i + j] = residuumLp.a[i][j];   // math_33to9
        int piv[9];
        if (lu_factor(J, 9, piv)) return ST_FAIL_LP_DGESV;
        lu_solve(J, 9, piv, rhs);
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) deltaLp.a[i][j] = -rhs[3 * i + j];
      }
      Lpguess = add(Lpguess, scl(steplengthLp, deltaLp));
    }
    // phase_LiAndItsTangents (phase_mechanical_eigen.f90:106-178): no eigenstrain mechanism active => Li = 0, tangents 0
    M3 Li_c = zero3();
    double atol_Li = std::max(nm.eps_rel_Li * std::max(norm33(Liguess), norm33(Li_c)), nm.eps_abs_Li);
    M3 residuumLi = sub(Liguess, Li_c);
    double rn = norm33(residuumLi);
    if (anynan(residuumLi)) return status;
    else if (rn < atol_Li) break;
    else if (rn < residuumLi_old_norm) {
      residuumLi_old_norm = rn; Liguess_old = Liguess; steplengthLi = 1.0;
    } else {
      steplengthLi = nm.r_linesearch_Li * steplengthLi;
      Liguess = add(Liguess_old, scl(steplengthLi, deltaLi));
      continue;
    }
    if (jacoCounterLi % nm.f_update_jacobi_Li == 0) {
      jacoCounterLi++;
      // dLi_dS = dLi_dFi = 0 => dRLi_dLi = I, deltaLi = -residuumLi (phase_mechanical.f90:541-559)
      deltaLi = scl(-1.0, residuumLi);
    }
    Liguess = add(Liguess, scl(steplengthLi, deltaLi));
  }
  M3 invFp_new = mm(invFp_current, B);
  M3 Fp_new;
  if (invert33(Fp_new, invFp_new)) return status;
  c->P[en] = mm(mm(F, invFp_new), mm(S, tr(invFp_new)));
  c->S[en] = S;
  c->Lp[en] = Lpguess;
  c->Li[en] = Liguess;
  const double detcube = std::pow(det33(Fp_new), 1.0 / 3.0);
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) c->Fp[en].a[i][j] = Fp_new.a[i][j] / detcube;
  c->Fi[en] = Fi_new;
  c->Fe[en] = mm(mm(F, invFp_new), invFi_new);
  return ST_OK;
}

// damper, phase_mechanical.f90:653-674
double damper(const double* w0, const double* w1, const double* w2, int n) {
  double d12 = 0.0, d22 = 0.0, d01 = 0.0;
  for (int i = 0; i < n; ++i) d12 += (w0[i] - w1[i]) * (w1[i] - w2[i]);
  for (int i = 0; i < n; ++i) d22 += (w1[i] - w2[i]) * (w1[i] - w2[i]);
  for (int i = 0; i < n; ++i) d01 += w0[i] * w1[i];
  if (std::min(d01, d12) < 0.0 && d22 > 0.0) return 0.75 + 0.25 * std::tanh(2.0 + 4.0 * d12 / d22);
  return 1.0;
}

// integrateStateFPI, phase_mechanical.f90:591-676
int integrate_state_fpi(orc_ctx* c, long en, const M3& F0, const M3& F, const M3& Fp0, const M3& Fi0,
                        const double* state0, double dt) {
  (void)F0;
  const int n = c->sizeState;
  const PhaseC& pc = c->pc;
  int status = ST_FAIL_STATE;
  std::vector<double> dot(n), last1(n, 0.0), last2(n, 0.0), r(n);
  dot_state(c, en, dot.data());
  for (int i = 0; i < n; ++i) if (std::isnan(dot[i])) return status;
  double* st = &c->state[en * n];
  for (int i = 0; i < n; ++i) st[i] = state0[i] + dot[i] * dt;
  for (int it = 1; it <= c->num.N_iter_state_max; ++it) {
    #pragma omp atomic
      c->counters[3]++;
    for (int i = 0; i < n; ++i) last2[i] = it > 1 ? last1[i] : 0.0;
    for (int i = 0; i < n; ++i) last1[i] = dot[i];
    status = integrate_stress(c, en, F, Fp0, Fi0, dt);
    if (status != ST_OK) break;
    dot_state(c, en, dot.data());
    bool nan = false;
    for (int i = 0; i < n; ++i) nan |= std::isnan(dot[i]);
    if (nan) break;
    double zeta = damper(dot.data(), last1.data(), last2.data(), n);
    for (int i = 0; i < n; ++i) dot[i] = dot[i] * zeta + last1[i] * (1.0 - zeta);
    for (int i = 0; i < n; ++i) r[i] = st[i] - state0[i] - dot[i] * dt;
    for (int i = 0; i < n; ++i) st[i] = st[i] - r[i];
    // converged, phase.f90:703-716
    bool conv = true;
    for (int i = 0; i < n; ++i) {
      double atol = i < pc.Ns ? pc.atol_xi : pc.atol_gamma;
      conv &= std::fabs(r[i]) <= std::max(atol, c->num.eps_rel_state * std::fabs(st[i]));
    }
    if (conv) { status = ST_OK; break; }   // plastic_deltaState is a no-op for phenopowerlaw
  }
  return status;
}

// phase_mechanical_constitutive, phase_mechanical.f90:1008-1090
int constitutive(orc_ctx* c, long en, double dt) {
  const orc_numerics& nm = c->num;
  const int n = c->sizeState;
  std::vector<double> state0(c->state0.begin() + en * n, c->state0.begin() + (en + 1) * n);
  M3 Li0 = c->Li0[en], Lp0 = c->Lp0[en], Fp0 = c->Fp0[en], Fi0 = c->Fi0[en], F0 = c->F0[en], F = zero3();
  double stepFrac = 0.0, step = 1.0 / nm.r_cutback;
  int status = ST_ITERATING;
  bool todo = true;
  while (todo) {
    if (status == ST_OK) {
      stepFrac = stepFrac + step;
      step = std::min(1.0 - stepFrac, nm.r_increase * step);
      todo = step > 0.0;
      if (todo) {
        F0 = F; Lp0 = c->Lp[en]; Li0 = c->Li[en]; Fp0 = c->Fp[en]; Fi0 = c->Fi[en];
        std::copy(c->state.begin() + en * n, c->state.begin() + (en + 1) * n, state0.begin());
      }
    } else {
      step = nm.r_cutback * step;
      c->Fp[en] = Fp0; c->Fi[en] = Fi0; c->S[en] = c->S0[en];
      if (step < 1.0) { c->Lp[en] = Lp0; c->Li[en] = Li0; }
      std::copy(state0.begin(), state0.end(), c->state.begin() + en * n);
      todo = step > nm.r_cutback_min;
    }
    if (todo) {
      F = add(F0, scl(step, sub(c->F[en], c->F0[en])));
      #pragma omp atomic
      c->counters[1]++;
      status = integrate_state_fpi(c, en, F0, F, Fp0, Fi0, state0.data(), step * dt);
    }
  }
  return status;
}

// mechanical_restore, phase_mechanical.f90:1096-1115
void restore(orc_ctx* c, long en) {
  c->Fp[en] = c->Fp0[en]; c->Fi[en] = c->Fi0[en]; c->S[en] = c->S0[en];
  std::copy(c->state0.begin() + en * c->sizeState, c->state0.begin() + (en + 1) * c->sizeState, c->state.begin() + en * c->sizeState);
}

// phase_mechanical_dPdF, phase_mechanical.f90:1121-1242
T4 dPdF(orc_ctx* c, long en, double dt) {
  M3 devNull;
  T4 dSdFe, dSdFi, dLidS, dLidFi, dLpdS, dLpdFi, dFidS, rhs, lhs, tmp, dSdF, dFpinvdF, out;
  hooke(c, devNull, &dSdFe, &dSdFi, c->Fe[en], c->Fi[en]);
  std::memset(&dLidS, 0, sizeof dLidS); std::memset(&dLidFi, 0, sizeof dLidFi);   // no eigenstrain mechanism
  M3 invFp = inv33(c->Fp[en]), invFi = inv33(c->Fi[en]);
  M3 invSubFp0 = inv33(c->Fp0[en]), invSubFi0 = inv33(c->Fi0[en]);
  std::memset(&dFidS, 0, sizeof dFidS);   // sum(abs(dLidS)) < tol_math_check
  lp_tangents(c, devNull, &dLpdS, &dLpdFi, c->S[en], c->Fi[en], &c->state[en * c->sizeState]);
  dLpdS = [&] { T4 a = mul4x4(dLpdFi, dFidS); for (int i = 0; i < 81; ++i) (&a.a[0][0][0][0])[i] += (&dLpdS.a[0][0][0][0])[i]; return a; }();
  M3 t1 = tr(mm(invFp, invFi));
  M3 t2 = mm(c->F[en], invSubFp0);
  M3 t3 = mm(mm(c->F[en], invFp), invSubFi0);
  for (int o = 0; o < 3; ++o) for (int p = 0; p < 3; ++p) {
    M3 D, Dl, Di;
    for (int k = 0; k < 3; ++k) for (int l = 0; l < 3; ++l) { D.a[k][l] = dSdFe.a[p][o][k][l]; Dl.a[k][l] = dLpdS.a[k][l][p][o]; Di.a[k][l] = dLidS.a[k][l][p][o]; }
    M3 r = mm(D, t1);
    M3 t = add(mm(mm(t2, Dl), invFi), mm(t3, Di));
    for (int k = 0; k < 3; ++k) for (int l = 0; l < 3; ++l) { rhs.a[p][o][k][l] = r.a[k][l]; tmp.a[k][l][p][o] = t.a[k][l]; }
  }
  {
    T4 a = mul4x4(dSdFe, tmp), b = mul4x4(dSdFi, dFidS);
    for (int i = 0; i < 81; ++i) (&lhs.a[0][0][0][0])[i] = (&a.a[0][0][0][0])[i] * dt + (&b.a[0][0][0][0])[i];
  }
  double M[81], Minv[81];
  to99(lhs, M);
  for (int i = 0; i < 9; ++i) M[i * 9 + i] += 1.0;
  if (invert_n(Minv, M, 9)) dSdF = rhs;
  else dSdF = mul4x4(from99(Minv), rhs);
  tmp = mul4x4(dLpdS, dSdF);
  for (int o = 0; o < 3; ++o) for (int p = 0; p < 3; ++p) {
    M3 T; for (int k = 0; k < 3; ++k) for (int l = 0; l < 3; ++l) T.a[k][l] = tmp.a[k][l][p][o];
    M3 X = mm(invSubFp0, mm(T, invFi));
    for (int k = 0; k < 3; ++k) for (int l = 0; l < 3; ++l) dFpinvdF.a[k][l][p][o] = -X.a[k][l] * dt;
  }
  t1 = mm(c->S[en], tr(invFp));
  t2 = mm(c->F[en], invFp);
  t3 = mm(t2, c->S[en]);
  std::memset(&out, 0, sizeof out);
  M3 d = tr(mm(invFp, t1));
  for (int p = 0; p < 3; ++p) for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) out.a[p][i][p][j] = d.a[i][j];
  for (int o = 0; o < 3; ++o) for (int p = 0; p < 3; ++p) {
    M3 Dfp, Ds;
    for (int k = 0; k < 3; ++k) for (int l = 0; l < 3; ++l) { Dfp.a[k][l] = dFpinvdF.a[k][l][p][o]; Ds.a[k][l] = dSdF.a[k][l][p][o]; }
    M3 add1 = mm(mm(c->F[en], Dfp), t1);
    M3 add2 = mm(mm(t2, Ds), tr(invFp));
    M3 add3 = mm(t3, tr(Dfp));
    for (int k = 0; k < 3; ++k) for (int l = 0; l < 3; ++l)
      out.a[k][l][p][o] = out.a[k][l][p][o] + add1.a[k][l] + add2.a[k][l] + add3.a[k][l];
  }
  return out;
}

// homogenization_mechanical_response (homogenization.f90:294-362) for one
// constituent with pass/isostrain partitioning (F_constituent = F_cell).
int hom_response(orc_ctx* c, double dt, bool with_dPdF) {
  int status = ST_OK;
  const long N = c->N;
  int64_t cnt[4] = {0, 0, 0, 0};
  #pragma omp parallel num_threads(c->nthreads)
  {
    int my = ST_OK;
    #pragma omp for schedule(dynamic, 64)
    for (long ce = 0; ce < N; ++ce) {
      restore(c, ce);
      c->F[ce] = c->Fsol[ce];
      int st = constitutive(c, ce, dt);
      if (st != ST_OK) my = ST_FAIL_MECH;
    }
    #pragma omp critical
    { if (my != ST_OK) status = my; }
  }
  (void)cnt;
  c->counters[0] += N;
  if (status != ST_OK) return status;
  #pragma omp parallel for schedule(dynamic, 64) num_threads(c->nthreads)
  for (long ce = 0; ce < N; ++ce) {
    c->homP[ce] = scl(1.0, c->P[ce]);
    if (with_dPdF) {
      T4 d = dPdF(c, ce, dt);
      for (int i = 0; i < 81; ++i) (&c->homdPdF[ce].a[0][0][0][0])[i] = (&d.a[0][0][0][0])[i] * 1.0;
    }
  }
  return status;
}

// utilities_constitutiveResponse, grid_utilities.f90:133-207
int constitutive_response(orc_ctx* c, double dt, bool rotate) {
  int status = hom_response(c, dt, true);
  const long N = c->N;
  const int n0 = c->cells[0], n1 = c->cells[1], n2 = c->cells[2];
  // P_av = sum(sum(sum(P,dim=5),dim=4),dim=3) * wgt
  M3 Pav = zero3();
  for (int x = 0; x < n0; ++x) {
    M3 sy = zero3();
    for (int y = 0; y < n1; ++y) {
      M3 sz = zero3();
      for (int z = 0; z < n2; ++z) sz = add(sz, c->homP[(long(z) * n1 + y) * n0 + x]);
      sy = add(sy, sz);
    }
    Pav = add(Pav, sy);
  }
  Pav = scl(c->wgt, Pav);
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) Pav.a[i][j] = Pav.a[i][j];
  if (rotate) Pav = rot33(c->rot_q, Pav, false);
  c->P_av = Pav;
  // dPdF_max / dPdF_min (grid_utilities.f90:171-197): the voxel of maximal / minimal
  // Frobenius norm in voxel order.  Norms that agree to 1e-12 relative count as equal
  // and the first such voxel is taken, so that the pick does not depend on rounding
  // (at F = I every grain's tangent has the same norm).
  std::vector<double> nrm(N);
  T4 vol; std::memset(&vol, 0, sizeof vol);
  double nmax = 0.0, nmin = std::numeric_limits<double>::max();
  for (long ce = 0; ce < N; ++ce) {
    const double* d = &c->homdPdF[ce].a[0][0][0][0];
    double s = 0.0;
    for (int l = 0; l < 3; ++l) for (int k = 0; k < 3; ++k) for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) {
      double v = c->homdPdF[ce].a[i][j][k][l];
      s += v * v;
    }
    nrm[ce] = s;
    nmax = std::max(nmax, s);
    nmin = std::min(nmin, s);
    for (int i = 0; i < 81; ++i) (&vol.a[0][0][0][0])[i] += d[i];
  }
  long imax = -1, imin = -1;
  for (long ce = 0; ce < N; ++ce) {
    if (imax < 0 && nrm[ce] >= nmax * (1.0 - 1.0e-12) && nrm[ce] > 0.0) imax = ce;
    if (imin < 0 && nrm[ce] <= nmin * (1.0 + 1.0e-12)) imin = ce;
  }
  T4 dmax, dmin;
  std::memset(&dmax, 0, sizeof dmax);
  for (int i = 0; i < 81; ++i) (&dmin.a[0][0][0][0])[i] = std::numeric_limits<double>::max();
  if (imax >= 0) dmax = c->homdPdF[imax];
  if (imin >= 0) dmin = c->homdPdF[imin];
  for (int i = 0; i < 81; ++i) {
    (&c->C_minMaxAvg.a[0][0][0][0])[i] = 0.5 * ((&dmax.a[0][0][0][0])[i] + (&dmin.a[0][0][0][0])[i]);
    (&c->C_volAvg.a[0][0][0][0])[i] = (&vol.a[0][0][0][0])[i] * c->wgt;
  }
  c->status = status;
  return status;
}

// ---------------------------------------------------------------- spectral
inline long fidx(const orc_ctx* c, int x, int y, int z) { return (long(z) * c->cells[1] + y) * c->red + x; }

// utilities_getFreqDerivative, spectral_utilities.f90:808-850: component d of the derivative
// frequency of the signed index triple ks.  continuous: i 2 pi k_d / L_d; central difference:
// i sin(2 pi k_d / n_d) / (2 L_d / n_d); FWBW difference: (e^{i t_d} - 1) times (e^{i t_e} + 1)
// for the other two directions e, over 4 L_d / n_d, with t = 2 pi k / n (factors in the order 1, 2, 3).
cd freq_derivative(const orc_ctx* c, const int ks[3], int d) {
  if (c->num.derivative == 1)
    return cd(0.0, std::sin(TAU * double(ks[d]) / double(c->cells[d])) / (2.0 * c->geomSize[d] / double(c->cells[d])));
  if (c->num.derivative == 2) {
    cd p(1.0, 0.0);
    for (int e = 0; e < 3; ++e) {
      const double t = TAU * double(ks[e]) / double(c->cells[e]);
      p = p * cd(std::cos(t) + (e == d ? -1.0 : 1.0), std::sin(t));
    }
    return p / (4.0 * c->geomSize[d] / double(c->cells[d]));
  }
  return cd(0.0, TAU * double(ks[d]) / c->geomSize[d]);
}

void spectral_init(orc_ctx* c) {
  const int* n = c->cells;
  c->red = n[0] / 2 + 1;
  const double* g = c->geomSize;
  // scaledGeomSize, spectral_utilities.f90:181-197
  double sp[3] = {g[0] / n[0], g[1] / n[1], g[2] / n[2]};
  auto argmin = [](const double* v) { int k = 0; for (int i = 1; i < 3; ++i) if (v[i] < v[k]) k = i; return k; };
  auto argmax = [](const double* v) { int k = 0; for (int i = 1; i < 3; ++i) if (v[i] > v[k]) k = i; return k; };
  if (c->num.divergence_correction == 2) {
    for (int j = 0; j < 3; ++j) if (j != argmin(sp) && j != argmax(sp))
      for (int i = 0; i < 3; ++i) c->scaledGeomSize[i] = g[i] / g[j] * double(n[j]);
  } else if (c->num.divergence_correction == 0) {
    for (int j = 0; j < 3; ++j) if (j != argmin(g) && j != argmax(g))
      for (int i = 0; i < 3; ++i) c->scaledGeomSize[i] = g[i] / g[j];
  } else {
    for (int i = 0; i < 3; ++i) c->scaledGeomSize[i] = g[i];
  }
  // xi1st, spectral_utilities.f90:315-333 and :808-850 (continuous: Nyquist zeroed on even
  // edges; the difference schemes: as xi2nd)
  c->xi.assign(size_t(c->red) * n[1] * n[2] * 3, cd(0.0, 0.0));
  for (int z = 0; z < n[2]; ++z) for (int y = 0; y < n[1]; ++y) for (int x = 0; x < c->red; ++x) {
    int ks[3] = {x, y > n[1] / 2 ? y - n[1] : y, z > n[2] / 2 ? z - n[2] : z};
    int idx[3] = {x, y, z};
    for (int d = 0; d < 3; ++d) {
      cd v = freq_derivative(c, ks, d);
      if (c->num.derivative == 0 && n[d] % 2 == 0 && idx[d] == n[d] / 2) v = 0.0;
      c->xi[fidx(c, x, y, z) * 3 + d] = v;
    }
  }
  c->work.assign(size_t(9) * n[0] * n[1] * n[2], cd(0.0, 0.0));
}

// forward R2C of a 9-component field into c->work (full complex spectrum per component)
void r2c(orc_ctx* c, const M3* field) {
  const long N = c->N;
  for (int comp = 0; comp < 9; ++comp) {
    int i = comp % 3, j = comp / 3;
    cd* w = c->work.data() + comp * N;
    for (long v = 0; v < N; ++v) w[v] = cd(field[v].a[i][j], 0.0);
    fft3(w, c->cells, -1);
  }
}
inline cd spec(const orc_ctx* c, int comp, int x, int y, int z) {
  return c->work[comp * c->N + (long(z) * c->cells[1] + y) * c->cells[0] + x];
}

// utilities_updateGamma, spectral_utilities.f90:356-395 (memory-efficient form)
void update_gamma(orc_ctx* c, const T4& C) {
  for (int i = 0; i < 81; ++i) (&c->C_ref.a[0][0][0][0])[i] = (&C.a[0][0][0][0])[i] / c->wgt;
}

// utilities_divergenceRMS, spectral_utilities.f90:650-691 (spectrum already in c->work)
double divergence_rms(orc_ctx* c) {
  const int n0 = c->cells[0], n1 = c->cells[1], n2 = c->cells[2];
  const double rg[3] = {c->geomSize[0] / c->scaledGeomSize[0], c->geomSize[1] / c->scaledGeomSize[1], c->geomSize[2] / c->scaledGeomSize[2]};
  auto term = [&](int x, int y, int z) {
    const cd* xv = &c->xi[fidx(c, x, y, z) * 3];
    cd w[3];
    for (int m = 0; m < 3; ++m) w[m] = std::conj(-xv[m]) * cd(rg[m], 0.0);
    double sr = 0.0, si = 0.0;
    cd v[3];
    for (int l = 0; l < 3; ++l) { cd s = 0.0; for (int m = 0; m < 3; ++m) s += spec(c, l + 3 * m, x, y, z) * w[m]; v[l] = s; }
    for (int l = 0; l < 3; ++l) sr += v[l].real() * v[l].real();
    for (int l = 0; l < 3; ++l) si += v[l].imag() * v[l].imag();
    return std::make_pair(sr, si);
  };
  double res = 0.0;
  for (int y = 0; y < n1; ++y) for (int z = 0; z < n2; ++z) {
    for (int x = 1; x < c->red - 1; ++x) { auto t = term(x, y, z); res += 2.0 * (t.first + t.second); }
    auto a = term(0, y, z), b = term(c->red - 1, y, z);
    res += a.first + a.second + b.first + b.second;
  }
  res = std::sqrt(res) * c->wgt;
  if (n0 == 1) res *= 0.5;
  return res;
}

// C2R of one component given by its stored half spectrum (kx in [0, cells1/2], index fidx):
// Hermitian extension of the stored half, complex inverse transform, real part.  The real part
// makes the planes kx = 0 and kx = cells1/2 count with their Hermitian part, as a C2R does.
// w: workspace of N complex values.
void c2r(orc_ctx* c, const cd* half, cd* w, double* out) {
  const int n0 = c->cells[0], n1 = c->cells[1], n2 = c->cells[2];
  for (int z = 0; z < n2; ++z) for (int y = 0; y < n1; ++y) for (int x = 0; x < n0; ++x) {
    cd v;
    if (x < c->red) v = half[fidx(c, x, y, z)];
    else v = std::conj(half[fidx(c, n0 - x, (n1 - y) % n1, (n2 - z) % n2)]);
    w[(long(z) * n1 + y) * n0 + x] = v;
  }
  fft3(w, c->cells, +1);
  for (long v = 0; v < c->N; ++v) out[v] = w[v].real();
}

// utilities_GammaConvolution, spectral_utilities.f90:436-501 (spectrum in c->work; result to field)
void gamma_convolution(orc_ctx* c, M3* field, const M3& aim) {
  const int n1 = c->cells[1], n2 = c->cells[2];
  const long N = c->N;
  std::vector<cd> half(size_t(9) * c->red * n1 * n2);
  #pragma omp parallel for collapse(2) schedule(static) num_threads(c->nthreads)
  for (int z = 0; z < n2; ++z) for (int y = 0; y < n1; ++y) for (int x = 0; x < c->red; ++x) {
    long f = fidx(c, x, y, z);
    cd P[3][3];
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) P[i][j] = spec(c, i + 3 * j, x, y, z);
    cd R[3][3];
    if (x == 0 && y == 0 && z == 0) {
      for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) R[i][j] = cd(aim.a[i][j], 0.0);
    } else {
      const cd* xv = &c->xi[f * 3];
      cd xd[3][3];
      for (int l = 0; l < 3; ++l) for (int m = 0; m < 3; ++m) xd[l][m] = std::conj(-xv[l]) * xv[m];
      cd t[3][3];
      for (int l = 0; l < 3; ++l) for (int m = 0; m < 3; ++m) {
        cd s = 0.0;
        for (int k = 0; k < 3; ++k) for (int j = 0; j < 3; ++j) s += cd(c->C_ref.a[l][j][m][k], 0.0) * xd[j][k];
        t[l][m] = s;
      }
      double A[36], Ainv[36];
      for (int l = 0; l < 3; ++l) for (int m = 0; m < 3; ++m) {
        A[l * 6 + m] = t[l][m].real(); A[(l + 3) * 6 + m + 3] = t[l][m].real();
        A[l * 6 + m + 3] = t[l][m].imag(); A[(l + 3) * 6 + m] = -t[l][m].imag();
      }
      M3 re; for (int l = 0; l < 3; ++l) for (int m = 0; m < 3; ++m) re.a[l][m] = A[l * 6 + m];
      if (std::fabs(det33(re)) > 1.0e-16) {
        invert_n(Ainv, A, 6);
        cd ti[3][3];
        for (int l = 0; l < 3; ++l) for (int m = 0; m < 3; ++m) ti[l][m] = cd(Ainv[l * 6 + m], Ainv[l * 6 + m + 3]);
        for (int l = 0; l < 3; ++l) for (int m = 0; m < 3; ++m) {
          cd s = 0.0;
          for (int o = 0; o < 3; ++o) for (int n = 0; n < 3; ++n) s += (ti[l][n] * xd[o][m]) * P[n][o];
          R[l][m] = s;
        }
      } else {
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) R[i][j] = 0.0;
      }
    }
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) half[(i + 3 * j) * (long(c->red) * n1 * n2) + f] = R[i][j];
  }
  const long H = long(c->red) * n1 * n2;
  std::vector<double> out(N);
  for (int comp = 0; comp < 9; ++comp) {
    c2r(c, half.data() + comp * H, c->work.data() + comp * N, out.data());
    int i = comp % 3, j = comp / 3;
    for (long v = 0; v < N; ++v) field[v].a[i][j] = out[v];
  }
}

// utilities_updateCoords, spectral_utilities.f90:857-968 (single process: the z padding of the
// cell-centre fluctuations is the periodic wrap)
void update_coords(orc_ctx* c) {
  const int n0 = c->cells[0], n1 = c->cells[1], n2 = c->cells[2];
  const long N = c->N;
  const double* g = c->geomSize;
  const double step[3] = {g[0] / n0, g[1] / n1, g[2] / n2};
  r2c(c, c->Fsol.data());
  M3 Favg;
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) Favg.a[i][j] = spec(c, i + 3 * j, 0, 0, 0).real() * c->wgt;
  // vectorField_fourier = F_hat . xi2nd / sum(conjg(-xi2nd) xi2nd), zero at k = 0 (:899-909)
  const long H = long(c->red) * n1 * n2;
  std::vector<cd> half(size_t(3) * H);
  for (int z = 0; z < n2; ++z) for (int y = 0; y < n1; ++y) for (int x = 0; x < c->red; ++x) {
    const long f = fidx(c, x, y, z);
    if (x == 0 && y == 0 && z == 0) { for (int l = 0; l < 3; ++l) half[l * H + f] = 0.0; continue; }
    int ks[3] = {x, y > n1 / 2 ? y - n1 : y, z > n2 / 2 ? z - n2 : z};
    cd xi2[3];
    for (int d = 0; d < 3; ++d) xi2[d] = freq_derivative(c, ks, d);   // no Nyquist zeroing
    cd den = 0.0;
    for (int d = 0; d < 3; ++d) den += std::conj(-xi2[d]) * xi2[d];
    for (int l = 0; l < 3; ++l) {
      cd s = 0.0;
      for (int m = 0; m < 3; ++m) s += spec(c, l + 3 * m, x, y, z) * xi2[m];
      half[l * H + f] = s / den;
    }
  }
  std::vector<double> u(size_t(3) * N);
  for (int l = 0; l < 3; ++l) {
    c2r(c, half.data() + l * H, c->work.data() + l * N, u.data() + l * N);
    for (long v = 0; v < N; ++v) u[l * N + v] *= c->wgt;
  }
  // nodal positions (:940-952): Favg (step ijk) + mean of the 8 surrounding cell fluctuations
  static const int nb[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  auto mod = [](int a, int n) { return ((a % n) + n) % n; };
  c->xn.assign(size_t(3) * (n0 + 1) * (n1 + 1) * (n2 + 1), 0.0);
  long t = 0;
  for (int k = 0; k <= n2; ++k) for (int j = 0; j <= n1; ++j) for (int i = 0; i <= n0; ++i, ++t) {
    const double p[3] = {step[0] * i, step[1] * j, step[2] * k};
    for (int l = 0; l < 3; ++l) {
      double x = 0.0;
      for (int m = 0; m < 3; ++m) x += Favg.a[l][m] * p[m];
      for (int n = 0; n < 8; ++n) {
        const long w = (long(mod(k + nb[n][2] - 1, n2)) * n1 + mod(j + nb[n][1] - 1, n1)) * n0 + mod(i + nb[n][0] - 1, n0);
        x += u[l * N + w] * 0.125;
      }
      c->xn[3 * t + l] = x;
    }
  }
  // cell centres (:955-959): fluctuation + Favg (step (ijk - 1/2))
  c->xp.assign(size_t(3) * N, 0.0);
  for (long v = 0; v < N; ++v) {
    const long idx[3] = {v % n0, (v / n0) % n1, v / (long(n0) * n1)};
    double p[3];
    for (int d = 0; d < 3; ++d) p[d] = step[d] * (double(idx[d] + 1) - 0.5);
    for (int l = 0; l < 3; ++l) {
      double x = 0.0;
      for (int m = 0; m < 3; ++m) x += Favg.a[l][m] * p[m];
      c->xp[3 * v + l] = u[l * N + v] + x;
    }
  }
}

// utilities_maskedCompliance, grid_utilities.f90:74-127
T4 masked_compliance(orc_ctx* c, const T4& C) {
  bool sv[9];
  int nred = 0;
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) { sv[3 * i + j] = !c->stress_mask[i][j]; nred += sv[3 * i + j]; }
  double t99[81] = {0};
  if (nred > 0) {
    T4 Cr = rot3333(c->rot_q, C);
    double full[81];
    to99(Cr, full);
    // pack in column-major order of the 9x9 mask
    std::vector<double> cr(nred * nred), sr(nred * nred);
    std::vector<int> idx;
    for (int i = 0; i < 9; ++i) if (sv[i]) idx.push_back(i);
    for (int a = 0; a < nred; ++a) for (int b = 0; b < nred; ++b) cr[a * nred + b] = full[idx[a] * 9 + idx[b]];
    invert_n(sr.data(), cr.data(), nred);
    for (int a = 0; a < nred; ++a) for (int b = 0; b < nred; ++b) t99[idx[a] * 9 + idx[b]] = sr[a * nred + b];
  }
  return from99(t99);
}

// form_residual, grid_mech_spectral_basic.f90:464-521; F in c->Fsol, residual into r
void form_residual(orc_ctx* c, std::vector<M3>& r) {
  c->totalIter++;
  bool rotate = true;
  int status = constitutive_response(c, c->dt, rotate);
  c->status = status;
  for (long v = 0; v < c->N; ++v) r[v] = c->homP[v];
  r2c(c, r.data());
  c->err_div = divergence_rms(c);
  M3 d = sub(c->P_av, c->P_aim);
  M3 deltaF_aim = mul4x2(c->Scomp, d);
  c->F_aim = sub(c->F_aim, deltaF_aim);
  double e = 0.0;
  for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) e = std::max(e, std::fabs(c->stress_mask[i][j] ? 0.0 : d.a[i][j]));
  c->err_BC = e;
  gamma_convolution(c, r.data(), rot33(c->rot_q, deltaF_aim, true));
}

// math_sym3333to66, math.f90:826-845: rows/columns in the Mandel order (11,22,33,23,13,12),
// weights 1 for normal and sqrt(2) for shear pairs; the (i<j) components are the ones read.
void sym3333to66(const T4& m, double out[6][6]) {
  const int p[6][2] = {{0, 0}, {1, 1}, {2, 2}, {1, 2}, {0, 2}, {0, 1}};
  for (int r = 0; r < 6; ++r) for (int q = 0; q < 6; ++q)
    out[r][q] = m.a[p[r][0]][p[r][1]][p[q][0]][p[q][1]] * (r < 3 ? 1.0 : SQRT2) * (q < 3 ? 1.0 : SQRT2);
}
// math_invSym3333, math.f90:511-532 (dgetrf + dgetri of the Mandel 6x6)
T4 inv_sym3333(const T4& A) {
  double m[6][6], inv[36], mi[6][6];
  sym3333to66(A, m);
  invert_n(inv, &m[0][0], 6);
  for (int r = 0; r < 6; ++r) for (int q = 0; q < 6; ++q) mi[r][q] = inv[r * 6 + q];
  return m66toSym3333(mi);
}

// utilities_curlRMS, spectral_utilities.f90:695-757 (spectrum of the field in c->work).  The
// planes kx = 0 and kx = cells1/2 (stored index cells1Red) assign every entry of curl_fourier
// the last of the nine expressions (l = 3, third column), as the reference does.
double curl_rms(orc_ctx* c) {
  const int n0 = c->cells[0], n1 = c->cells[1], n2 = c->cells[2];
  const double rg[3] = {c->geomSize[0] / c->scaledGeomSize[0], c->geomSize[1] / c->scaledGeomSize[1],
                        c->geomSize[2] / c->scaledGeomSize[2]};
  auto xi = [&](int x, int y, int z, int d) { return c->xi[fidx(c, x, y, z) * 3 + d] * cd(rg[d], 0.0); };
  auto T = [&](int l, int m, int x, int y, int z) { return spec(c, l + 3 * m, x, y, z); };
  double res = 0.0;
  for (int y = 0; y < n1; ++y) for (int z = 0; z < n2; ++z) {
    for (int x = 1; x < c->red - 1; ++x) {
      double s = 0.0;
      for (int l = 0; l < 3; ++l) {
        const cd c1 = T(l, 2, x, y, z) * xi(x, y, z, 1) - T(l, 1, x, y, z) * xi(x, y, z, 2);
        const cd c2 = T(l, 0, x, y, z) * xi(x, y, z, 2) - T(l, 2, x, y, z) * xi(x, y, z, 0);
        const cd c3 = T(l, 1, x, y, z) * xi(x, y, z, 0) - T(l, 0, x, y, z) * xi(x, y, z, 1);
        s += c1.real() * c1.real() + c2.real() * c2.real() + c3.real() * c3.real();
        s += c1.imag() * c1.imag() + c2.imag() * c2.imag() + c3.imag() * c3.imag();
      }
      res += 2.0 * s;
    }
    for (int x : {0, c->red - 1}) {
      const cd last = T(2, 1, x, y, z) * xi(x, y, z, 0) - T(2, 0, x, y, z) * xi(x, y, z, 1);
      res += 9.0 * (last.real() * last.real() + last.imag() * last.imag());
    }
  }
  res = std::sqrt(res) * c->wgt;
  if (n0 == 1) res *= 0.5;
  return res;
}

// volume average sum(sum(sum(field,dim=5),dim=4),dim=3) * wgt
M3 field_average(const orc_ctx* c, const std::vector<M3>& f) {
  const int n0 = c->cells[0], n1 = c->cells[1], n2 = c->cells[2];
  M3 a = zero3();
  for (int x = 0; x < n0; ++x) {
    M3 sy = zero3();
    for (int y = 0; y < n1; ++y) { M3 sz = zero3(); for (int z = 0; z < n2; ++z) sz = add(sz, f[(long(z) * n1 + y) * n0 + x]); sy = add(sy, sz); }
    a = add(a, sy);
  }
  return scl(c->wgt, a);
}

// form_residual of the polarization scheme, grid_mech_spectral_polarization.f90:562-632.
// F in c->Fsol, F_tau in c->Ftau; r = [r_F (N); r_F_tau (N)].
void form_residual_pol(orc_ctx* c, std::vector<M3>& r) {
  const long N = c->N;
  const double alpha = c->num.alpha, beta = c->num.beta;
  const M3 I = eye3();
  const M3 F_av = field_average(c, c->Fsol);
  c->totalIter++;
  std::vector<M3> t(N), rtau(N), Feval(N);
  for (long v = 0; v < N; ++v) {
    const M3& F = c->Fsol[v];
    t[v] = sub(scl(beta, mul4x2(c->C_scale, sub(F, I))),
               scl(alpha, mm(F, mul4x2(c->C_scale, sub(sub(c->Ftau[v], F), I)))));
  }
  r2c(c, t.data());
  gamma_convolution(c, t.data(), rot33(c->rot_q, scl(beta, c->F_aim), true));
  for (long v = 0; v < N; ++v) {
    rtau[v] = sub(scl(beta, c->Fsol[v]), t[v]);
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) Feval[v].a[i][j] = c->Fsol[v].a[i][j] - rtau[v].a[i][j] / beta;
  }
  r2c(c, c->Fsol.data());
  c->err_curl = curl_rms(c);
  std::swap(c->Fsol, Feval);
  c->status = constitutive_response(c, c->dt, true);
  std::swap(c->Fsol, Feval);
  r2c(c, c->homP.data());
  c->err_div = divergence_rms(c);
  #pragma omp parallel for schedule(static) num_threads(c->nthreads)
  for (long v = 0; v < N; ++v) {
    const M3& F = c->Fsol[v];
    T4 A = c->homdPdF[v];
    for (int i = 0; i < 81; ++i) (&A.a[0][0][0][0])[i] += (&c->C_scale.a[0][0][0][0])[i];
    const M3 rhs = sub(c->homP[v], mm(F, mul4x2(c->C_scale, sub(sub(c->Ftau[v], F), I))));
    r[v] = add(mul4x2(inv_sym3333(A), rhs), rtau[v]);
    r[N + v] = rtau[v];
  }
  const M3 d = sub(c->P_av, c->P_aim);
  c->F_aim = sub(c->F_aim, mul4x2(c->Scomp, d));
  const M3 e = mul4x2(c->C_scale, sub(c->F_aim, rot33(c->rot_q, F_av, false)));
  double eb = 0.0;
  for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) eb = std::max(eb, std::fabs(c->stress_mask[i][j] ? e.a[i][j] : d.a[i][j]));
  c->err_BC = eb;
}

// Least-squares coefficients of the Anderson update: solve G_S gamma = b_S on the
// slots S (oldest first) by Cholesky; while a pivot is not safely positive
// (< 1e-13 of the largest diagonal), drop the oldest slot and retry.
template <class BFn>
std::vector<double> anderson_coefficients(const std::vector<double>& G, int m, std::vector<int>& slots, BFn bfn) {
  std::vector<double> b(slots.size());
  for (size_t q = 0; q < slots.size(); ++q) b[q] = bfn(slots[q]);
  size_t first = 0;
  while (first < slots.size()) {
    const size_t n = slots.size() - first;
    std::vector<double> L(n * n, 0.0);
    double dmax = 0.0;
    for (size_t i = 0; i < n; ++i) dmax = std::max(dmax, G[size_t(slots[first + i]) * m + slots[first + i]]);
    bool ok = dmax > 0.0;
    for (size_t i = 0; ok && i < n; ++i) {
      for (size_t j = 0; j <= i; ++j) {
        double sum = G[size_t(slots[first + i]) * m + slots[first + j]];
        for (size_t k = 0; k < j; ++k) sum -= L[i * n + k] * L[j * n + k];
        if (i == j) {
          if (!(sum > 1.0e-13 * dmax)) { ok = false; break; }
          L[i * n + i] = std::sqrt(sum);
        } else {
          L[i * n + j] = sum / L[j * n + j];
        }
      }
    }
    if (!ok) { ++first; continue; }
    std::vector<double> y(n), x(n);
    for (size_t i = 0; i < n; ++i) { double sum = b[first + i]; for (size_t k = 0; k < i; ++k) sum -= L[i * n + k] * y[k]; y[i] = sum / L[i * n + i]; }
    for (size_t i = n; i-- > 0;) { double sum = y[i]; for (size_t k = i + 1; k < n; ++k) sum -= L[k * n + i] * x[k]; x[i] = sum / L[i * n + i]; }
    std::vector<double> gam(slots.size(), 0.0);
    for (size_t i = 0; i < n; ++i) gam[first + i] = x[i];
    return gam;
  }
  return std::vector<double>(slots.size(), 0.0);
}

}  // namespace

// ==================================================================== C API
extern "C" {

orc_ctx* orc_create(const int cells[3], const double geomSize[3], const int* materialAt,
                    int n_materials, const double* quaternions, const orc_phase* phase,
                    const orc_numerics* num, int n_threads) {
  orc_ctx* c = new orc_ctx();
  for (int i = 0; i < 3; ++i) { c->cells[i] = cells[i]; c->geomSize[i] = geomSize[i]; }
  c->N = long(cells[0]) * cells[1] * cells[2];
  c->wgt = 1.0 / double(c->N);
  c->nthreads = n_threads > 0 ? n_threads : 1;
#ifdef _OPENMP
  omp_set_num_threads(c->nthreads);
#endif
  c->num = *num;
  c->phase = *phase;
  if (!build_phase(*phase, c->pc)) { delete c; return nullptr; }
  c->sizeState = 2 * c->pc.Ns;
  const long N = c->N;
  for (auto* v : {&c->F, &c->F0, &c->Fp, &c->Fp0, &c->Fi, &c->Fi0, &c->Li, &c->Li0, &c->Lp, &c->Lp0, &c->S, &c->S0, &c->Fe, &c->P, &c->homP})
    v->assign(N, zero3());
  c->homdPdF.assign(N, T4{});
  c->state.assign(N * c->sizeState, 0.0);
  // mechanical_init, phase_mechanical.f90:249-266 (V_e = I)
  for (long ce = 0; ce < N; ++ce) {
    int ma = materialAt[ce];
    if (ma < 0 || ma >= n_materials) { delete c; return nullptr; }
    const double* q = quaternions + 4 * ma;
    c->F[ce] = eye3();
    c->Fp[ce] = qu2om(q);
    c->Fe[ce] = mm(eye3(), tr(c->Fp[ce]));
    c->Fi[ce] = rot33(q, inv33(eye3()), false);
    for (int i = 0; i < c->pc.Ns; ++i) c->state[ce * c->sizeState + i] = c->pc.xi0[i];
  }
  c->F0 = c->F; c->Fp0 = c->Fp; c->Fi0 = c->Fi;
  c->state0 = c->state;
  spectral_init(c);
  // discretization_init: current coordinates start as the undeformed ones
  // (IPcoordinates0 / nodes0, discretization_grid.f90:270-313)
  {
    const double step[3] = {geomSize[0] / cells[0], geomSize[1] / cells[1], geomSize[2] / cells[2]};
    c->xp.assign(size_t(3) * N, 0.0);
    for (long v = 0; v < N; ++v) {
      const long idx[3] = {v % cells[0], (v / cells[0]) % cells[1], v / (long(cells[0]) * cells[1])};
      for (int d = 0; d < 3; ++d) c->xp[3 * v + d] = step[d] * (double(idx[d] + 1) - 0.5);
    }
    c->xn.clear();
    for (int k = 0; k <= cells[2]; ++k) for (int j = 0; j <= cells[1]; ++j) for (int i = 0; i <= cells[0]; ++i) {
      c->xn.push_back(step[0] * i); c->xn.push_back(step[1] * j); c->xn.push_back(step[2] * k);
    }
  }
  c->Fsol.assign(N, eye3()); c->F_lastinc.assign(N, eye3()); c->Fdot.assign(N, zero3());
  c->F_aim = eye3(); c->F_aim_lastinc = eye3(); c->F_aimDot = zero3(); c->P_aim = zero3(); c->P_av = zero3();
  std::memset(&c->C_volAvg, 0, sizeof(T4)); c->C_volAvgLastInc = c->C_volAvg; c->C_minMaxAvg = c->C_volAvg;
  c->C_minMaxAvgLastInc = c->C_volAvg; c->C_minMaxAvgRestart = c->C_volAvg; c->Scomp = c->C_volAvg;
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) c->stress_mask[i][j] = true;
  c->rot_q[0] = 1; c->rot_q[1] = c->rot_q[2] = c->rot_q[3] = 0;
  c->dt = 0.0;
  c->totalIter = 0;
  std::memset(c->counters, 0, sizeof c->counters);
  return c;
}

void orc_destroy(orc_ctx* c) { delete c; }

// grid_mechanical_spectral_basic_init, grid_mech_spectral_basic.f90:103-237 (no restart)
// grid_mech_spectral_polarization_init, grid_mech_spectral_polarization.f90:115-270 (no restart):
// in addition F_tau = F_tau_lastinc = 2 I, C_scale = C_minMaxAvg, S_scale = its Mandel inverse
int orc_mech_init(orc_ctx* c) {
  for (long v = 0; v < c->N; ++v) { c->F_lastinc[v] = eye3(); c->Fsol[v] = eye3(); }
  if (c->num.solver == 1) {
    c->Ftau.assign(c->N, scl(2.0, eye3()));
    c->Ftau_lastinc = c->Ftau;
    c->Ftaudot.assign(c->N, zero3());
  }
  int status = constitutive_response(c, 0.0, false);
  update_gamma(c, c->C_minMaxAvg);
  c->C_minMaxAvgRestart = c->C_minMaxAvg;
  if (c->num.solver == 1) {
    c->C_scale = c->C_minMaxAvg;
    c->S_scale = inv_sym3333(c->C_minMaxAvg);
  }
  return status;
}

// grid_mechanical_spectral_basic_forward, grid_mech_spectral_basic.f90:284-355
int orc_mech_forward(orc_ctx* c, int cutBack, int guess, double dt, double dt_old, double t_remaining,
                     const orc_bc* def, const orc_bc* stress, const double q_rot[4]) {
  auto m3 = [](const double* v) { M3 m; for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) m.a[i][j] = v[3 * j + i]; return m; };
  auto msk = [](const int* v, int i, int j) { return v[3 * j + i] != 0; };
  const long N = c->N;
  if (cutBack) {
    c->C_volAvg = c->C_volAvgLastInc;
    c->C_minMaxAvg = c->C_minMaxAvgLastInc;
  } else {
    c->C_volAvgLastInc = c->C_volAvg;
    c->C_minMaxAvgLastInc = c->C_minMaxAvg;
    M3 rate = zero3();
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j)
      rate.a[i][j] = guess ? (msk(stress->mask, i, j) ? 0.0 : (c->F_aim.a[i][j] - c->F_aim_lastinc.a[i][j]) / dt_old) : 0.0;
    c->F_aimDot = rate;
    c->F_aim_lastinc = c->F_aim;
    M3 vals = m3(def->values);
    M3 masked; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) masked.a[i][j] = msk(def->mask, i, j) ? 0.0 : vals.a[i][j];
    if (def->type == 1) c->F_aimDot = add(c->F_aimDot, mm(masked, c->F_aim_lastinc));
    else if (def->type == 2) c->F_aimDot = add(c->F_aimDot, masked);
    else if (def->type == 3) {
      M3 t; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) t.a[i][j] = msk(def->mask, i, j) ? 0.0 : (vals.a[i][j] - c->F_aim_lastinc.a[i][j]) / t_remaining;
      c->F_aimDot = add(c->F_aimDot, t);
    }
    M3 avRate = rot33(q_rot, c->F_aimDot, true);
    for (long v = 0; v < N; ++v) c->Fdot[v] = avRate;
    if (guess) for (long v = 0; v < N; ++v) for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j)
      c->Fdot[v].a[i][j] = (c->Fsol[v].a[i][j] - c->F_lastinc[v].a[i][j]) / dt_old;
    if (c->num.solver == 1) {
      // F_tauDot = utilities_calculateRate(guess, F_tau_lastinc, F_tau, ...), polarization.f90:366-368
      for (long v = 0; v < N; ++v) c->Ftaudot[v] = avRate;
      if (guess) for (long v = 0; v < N; ++v) for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j)
        c->Ftaudot[v].a[i][j] = (c->Ftau[v].a[i][j] - c->Ftau_lastinc[v].a[i][j]) / dt_old;
      c->Ftau_lastinc = c->Ftau;
    }
    c->F_lastinc = c->Fsol;
  }
  c->F_aim = add(c->F_aim_lastinc, scl(dt, c->F_aimDot));
  M3 sv = m3(stress->values);
  if (stress->type == 4) for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j)
    c->P_aim.a[i][j] = c->P_aim.a[i][j] + (msk(stress->mask, i, j) ? 0.0 : (sv.a[i][j] - c->P_aim.a[i][j]) / t_remaining) * dt;
  if (stress->type == 5) for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j)
    c->P_aim.a[i][j] = c->P_aim.a[i][j] + (msk(stress->mask, i, j) ? 0.0 : sv.a[i][j]) * dt;
  // utilities_forwardTensorField, grid_utilities.f90:271-297
  M3 aim = rot33(q_rot, c->F_aim, true);
  const int n0 = c->cells[0], n1 = c->cells[1], n2 = c->cells[2];
  for (long v = 0; v < N; ++v) for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j)
    c->Fsol[v].a[i][j] = c->F_lastinc[v].a[i][j] + c->Fdot[v].a[i][j] * dt;
  M3 diff = zero3();
  for (int x = 0; x < n0; ++x) {
    M3 sy = zero3();
    for (int y = 0; y < n1; ++y) { M3 sz = zero3(); for (int z = 0; z < n2; ++z) sz = add(sz, c->Fsol[(long(z) * n1 + y) * n0 + x]); sy = add(sy, sz); }
    diff = add(diff, sy);
  }
  diff = sub(scl(c->wgt, diff), aim);
  for (long v = 0; v < N; ++v) c->Fsol[v] = sub(c->Fsol[v], diff);
  if (c->num.solver == 1) {
    // grid_mech_spectral_polarization.f90:384-396
    if (guess) {
      for (long v = 0; v < N; ++v) for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j)
        c->Ftau[v].a[i][j] = c->Ftau_lastinc[v].a[i][j] + c->Ftaudot[v].a[i][j] * dt;
    } else {
      for (long v = 0; v < N; ++v) {
        const M3 Fl = sub(c->Ftau[v], c->Fsol[v]);
        const M3 t = add(eye3(), mul4x2(c->S_scale, scl(0.5, mm(Fl, mul4x2(c->C_scale, sub(mm(tr(Fl), Fl), eye3()))))));
        c->Ftau[v] = add(t, c->Fsol[v]);
      }
    }
  }
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) c->stress_mask[i][j] = msk(stress->mask, i, j);
  for (int i = 0; i < 4; ++i) c->rot_q[i] = q_rot[i];
  c->dt = dt;
  return 0;
}

// grid_mechanical_spectral_basic_solution (grid_mech_spectral_basic.f90:243-277) with the
// residual iterated as SNES nrichardson + basic line search: F <- F - r(F).
int orc_mech_solution(orc_ctx* c, orc_solution* out) {
  std::memset(c->counters, 0, sizeof c->counters);
  const bool pol = c->num.solver == 1;
  c->Scomp = masked_compliance(c, c->C_volAvg);
  if (c->num.update_gamma) {
    update_gamma(c, c->C_minMaxAvg);
    if (pol) { c->C_scale = c->C_minMaxAvg; c->S_scale = inv_sym3333(c->C_minMaxAvg); }
  }
  const int snes_max_its = c->num.snes_max_it > 0 ? c->num.snes_max_it : 50;   // PETSc -snes_max_it (default 50)
  // iteration vector X: F (basic), or [F; F_tau] (polarization), with its residual r
  const long NX = pol ? 2 * c->N : c->N;
  std::vector<M3> X(NX), r(NX);
  auto load = [&]() {
    for (long v = 0; v < c->N; ++v) X[v] = c->Fsol[v];
    if (pol) for (long v = 0; v < c->N; ++v) X[c->N + v] = c->Ftau[v];
  };
  auto residual = [&]() {
    for (long v = 0; v < c->N; ++v) c->Fsol[v] = X[v];
    if (pol) {
      for (long v = 0; v < c->N; ++v) c->Ftau[v] = X[c->N + v];
      form_residual_pol(c, r);
    } else {
      form_residual(c, r);
    }
  };
  load();
  c->totalIter = -1;
  int evals = 0;
  int reason = 0;   // 0 iterating, 1 converged, -1 diverged
  auto converged = [&]() {
    double pmax = 0.0, fmax = 0.0;
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) {
      pmax = std::max(pmax, std::fabs(c->P_av.a[i][j]));
      fmax = std::max(fmax, std::fabs(c->F_aim.a[i][j] - (i == j ? 1.0 : 0.0)));
    }
    double divTol = std::max(pmax * c->num.eps_rel_div, c->num.eps_abs_div);
    double BCTol = std::max(pmax * c->num.eps_rel_P, c->num.eps_abs_P);
    bool ok = c->err_div / divTol < 1.0 && c->err_BC / BCTol < 1.0;
    if (pol) ok = ok && c->err_curl / std::max(fmax * c->num.eps_rel_curl, c->num.eps_abs_curl) < 1.0;   // polarization.f90:530-541
    if (c->totalIter >= c->num.N_iter_min && ok && c->status == ST_OK) return 1;
    if (c->totalIter >= c->num.N_iter_max) return -1;
    return 0;
  };
  auto finite = [&]() {
    for (long v = 0; v < NX; ++v) for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) if (!std::isfinite(r[v].a[i][j])) return false;
    return true;
  };
  residual(); evals++;
  if (!finite()) reason = -1; else reason = converged();
  if (c->num.snes_type == 0) {
    for (int it = 1; reason == 0 && it <= snes_max_its; ++it) {
      for (long v = 0; v < NX; ++v) X[v] = sub(X[v], r[v]);
      residual(); evals++;
      if (!finite()) { reason = -1; break; }
      reason = converged();
      if (reason == 0 && it == snes_max_its) reason = -1;
    }
  } else {
    // Anderson-accelerated fixed point of X <- X - r(X) (Walker & Ni 2011, type II, depth m):
    // gamma = argmin |r_k - dR gamma|, X_{k+1} = X_k - r_k - (dX - dR) gamma, where dX, dR hold
    // the last m differences of iterates and residuals.
    const int m = std::max(1, std::min(c->num.anderson_m, 32));
    const long N = NX;
    std::vector<std::vector<M3>> dX(m, std::vector<M3>(N)), dR(m, std::vector<M3>(N));
    std::vector<M3> Rprev(N);
    std::vector<double> G(size_t(m) * m, 0.0);
    int count = 0;
    auto dot = [&](const std::vector<M3>& a, const std::vector<M3>& b) {
      double s = 0.0;
      for (long v = 0; v < N; ++v) for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) s += a[v].a[i][j] * b[v].a[i][j];
      return s;
    };
    for (int it = 1; reason == 0 && it <= snes_max_its; ++it) {
      const int mk = std::min(count, m);
      std::vector<int> slots;                       // oldest -> newest
      for (int q = count - mk; q < count; ++q) slots.push_back(q % m);
      std::vector<double> gam = anderson_coefficients(G, m, slots, [&](int sl) { return dot(dR[sl], r); });
      const int slot = count % m;
      for (long v = 0; v < N; ++v) {
        M3 xn = sub(X[v], r[v]);
        for (size_t q = 0; q < slots.size(); ++q) {
          if (gam[q] == 0.0) continue;
          xn = sub(xn, scl(gam[q], sub(dX[slots[q]][v], dR[slots[q]][v])));
        }
        dX[slot][v] = sub(xn, X[v]);
        X[v] = xn;
        Rprev[v] = r[v];
      }
      residual(); evals++;
      if (!finite()) { reason = -1; break; }
      for (long v = 0; v < N; ++v) dR[slot][v] = sub(r[v], Rprev[v]);
      ++count;
      const int mk2 = std::min(count, m);
      for (int q = count - mk2; q < count; ++q) {
        const int t = q % m;
        G[size_t(slot) * m + t] = G[size_t(t) * m + slot] = dot(dR[slot], dR[t]);
      }
      reason = converged();
      if (reason == 0 && it == snes_max_its) reason = -1;
    }
  }
  out->converged = reason > 0;
  out->iterationsNeeded = c->totalIter;
  out->stagConverged = 1;
  out->residualEvals = evals;
  out->err_div = c->err_div; out->err_BC = c->err_BC;
  for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) out->P_av[3 * j + i] = c->P_av.a[i][j];
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) if (c->stress_mask[i][j]) c->P_aim.a[i][j] = c->P_av.a[i][j];
  return 0;
}

// grid_mechanical_spectral_basic_updateCoords, grid_mech_spectral_basic.f90:361-372
int orc_update_coords(orc_ctx* c) { update_coords(c); return 0; }

void orc_get_coords(orc_ctx* c, double* ip, double* nodes) {
  if (ip) std::memcpy(ip, c->xp.data(), sizeof(double) * c->xp.size());
  if (nodes) std::memcpy(nodes, c->xn.data(), sizeof(double) * c->xn.size());
}

// materialpoint_forward -> mechanical_forward, phase_mechanical.f90:987-1002
int orc_materialpoint_forward(orc_ctx* c) {
  c->Fi0 = c->Fi; c->Fp0 = c->Fp; c->F0 = c->F; c->Li0 = c->Li; c->Lp0 = c->Lp; c->S0 = c->S;
  c->state0 = c->state;
  return 0;
}

int orc_constitutive_response(orc_ctx* c, const double* F, double dt, double* P, double P_av[9],
                              double C_volAvg[81], double C_minMaxAvg[81], int* status) {
  for (long v = 0; v < c->N; ++v) for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) c->Fsol[v].a[i][j] = F[9 * v + 3 * j + i];
  std::memset(c->counters, 0, sizeof c->counters);
  *status = constitutive_response(c, dt, false);
  for (long v = 0; v < c->N; ++v) for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) P[9 * v + 3 * j + i] = c->homP[v].a[i][j];
  for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) P_av[3 * j + i] = c->P_av.a[i][j];
  for (int l = 0; l < 3; ++l) for (int k = 0; k < 3; ++k) for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) {
    C_volAvg[i + 3 * j + 9 * k + 27 * l] = c->C_volAvg.a[i][j][k][l];
    C_minMaxAvg[i + 3 * j + 9 * k + 27 * l] = c->C_minMaxAvg.a[i][j][k][l];
  }
  return 0;
}

void orc_update_gamma(orc_ctx* c, const double C[81]) {
  T4 t;
  for (int l = 0; l < 3; ++l) for (int k = 0; k < 3; ++k) for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i)
    t.a[i][j][k][l] = C[i + 3 * j + 9 * k + 27 * l];
  update_gamma(c, t);
}

void orc_gamma_convolution(orc_ctx* c, double* field, const double aim[9]) {
  std::vector<M3> f(c->N);
  for (long v = 0; v < c->N; ++v) for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) f[v].a[i][j] = field[9 * v + 3 * j + i];
  r2c(c, f.data());
  M3 a; for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) a.a[i][j] = aim[3 * j + i];
  gamma_convolution(c, f.data(), a);
  for (long v = 0; v < c->N; ++v) for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) field[9 * v + 3 * j + i] = f[v].a[i][j];
}

double orc_curl_rms(orc_ctx* c, const double* F) {
  std::vector<M3> f(c->N);
  for (long v = 0; v < c->N; ++v) for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) f[v].a[i][j] = F[9 * v + 3 * j + i];
  r2c(c, f.data());
  return curl_rms(c);
}

double orc_divergence_rms(orc_ctx* c, const double* P) {
  std::vector<M3> f(c->N);
  for (long v = 0; v < c->N; ++v) for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) f[v].a[i][j] = P[9 * v + 3 * j + i];
  r2c(c, f.data());
  return divergence_rms(c);
}

void orc_dPdF(orc_ctx* c, double dt, double* out) {
  for (long v = 0; v < c->N; ++v) {
    T4 d = dPdF(c, v, dt);
    for (int l = 0; l < 3; ++l) for (int k = 0; k < 3; ++k) for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i)
      out[81 * v + i + 3 * j + 9 * k + 27 * l] = d.a[i][j][k][l];
  }
}

static std::vector<M3>* field_ptr(orc_ctx* c, int field) {
  switch (field) {
    case 0: return &c->F; case 1: return &c->P; case 2: return &c->Fe; case 3: return &c->Fp;
    case 4: return &c->Lp; case 5: return &c->S; case 8: return &c->F_lastinc; case 9: return &c->Fi;
    case 10: return &c->Li; case 11: return &c->Fsol; case 13: return &c->Ftau;
    case 14: return &c->Ftau_lastinc;
    default: return nullptr;
  }
}

namespace {
// math_rotationalPart, math.f90:1004-1044 (closed form through the invariants of C = F^T F)
M3 rotational_part(const M3& F) {
  const M3 C = mm(tr(F), F);
  const double IC1 = C.a[0][0] + C.a[1][1] + C.a[2][2];
  const double IC2 = C.a[0][0] * C.a[1][1] + C.a[0][0] * C.a[2][2] + C.a[1][1] * C.a[2][2]
                   - (C.a[0][1] * C.a[0][1] + C.a[0][2] * C.a[0][2] + C.a[1][2] * C.a[1][2]);
  const double IC3 = -(C.a[0][0] * C.a[1][2] * C.a[1][2] + C.a[1][1] * C.a[0][2] * C.a[0][2]
                       + C.a[2][2] * C.a[0][1] * C.a[0][1])
                     + C.a[0][0] * C.a[1][1] * C.a[2][2] + 2.0 * C.a[0][1] * C.a[0][2] * C.a[1][2];   // math_detSym33
  const M3 FF = mm(F, F);
  const double IF1 = F.a[0][0] + F.a[1][1] + F.a[2][2];
  const double IF2 = 0.5 * (IF1 * IF1 - (FF.a[0][0] + FF.a[1][1] + FF.a[2][2]));
  const double x = std::pow(std::max(IC1 * IC1 - 3.0 * IC2, 0.0), 1.5);
  double lam[3];
  if (std::fabs(x) > 10.0 * TINY) {                                   // dNeq0
    const double Phi = std::acos(std::min(std::max((IC1 * IC1 * IC1 - 4.5 * IC1 * IC2 + 13.5 * IC3) / x, -1.0), 1.0));
    for (int k = 0; k < 3; ++k) {
      const double l = IC1 + (2.0 * std::sqrt(std::max(IC1 * IC1 - 3.0 * IC2, 0.0))) * std::cos((Phi - TAU * double(k + 1)) / 3.0);
      lam[k] = std::sqrt(std::max(l, 0.0) / 3.0);
    }
  } else {
    for (int k = 0; k < 3; ++k) lam[k] = std::sqrt(IC1 / 3.0);
  }
  const double IU1 = lam[0] + lam[1] + lam[2];
  const double IU2 = lam[0] * lam[1] + lam[1] * lam[2] + lam[2] * lam[0];
  const M3 FT = tr(F), FFT = tr(FF), FC = mm(F, C);
  M3 R;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      R.a[i][j] = (i == j ? IU1 * IF2 : 0.0) + (IU1 * IU1 - IU2) * F.a[i][j] - IU1 * IF1 * FT.a[i][j]
                + IU1 * FFT.a[i][j] - FC.a[i][j];
  return scl(std::pow(det33(R), -1.0 / 3.0), R);
}

// om2qu, rotations.f90:486-514 (P = -1, rotations.f90:57)
void om2qu(const M3& om, double* qu) {
  const double t = om.a[0][0] + om.a[1][1] + om.a[2][2];
  if (t > 0.0) {
    const double s = 0.5 / std::sqrt(t + 1.0);
    qu[0] = 0.25 / s; qu[1] = (om.a[2][1] - om.a[1][2]) * s; qu[2] = (om.a[0][2] - om.a[2][0]) * s; qu[3] = (om.a[1][0] - om.a[0][1]) * s;
  } else if (om.a[0][0] > om.a[1][1] && om.a[0][0] > om.a[2][2]) {
    const double s = 2.0 * std::sqrt(1.0 + om.a[0][0] - om.a[1][1] - om.a[2][2]);
    qu[0] = (om.a[2][1] - om.a[1][2]) / s; qu[1] = 0.25 * s; qu[2] = (om.a[0][1] + om.a[1][0]) / s; qu[3] = (om.a[0][2] + om.a[2][0]) / s;
  } else if (om.a[1][1] > om.a[2][2]) {
    const double s = 2.0 * std::sqrt(1.0 + om.a[1][1] - om.a[0][0] - om.a[2][2]);
    qu[0] = (om.a[0][2] - om.a[2][0]) / s; qu[1] = (om.a[0][1] + om.a[1][0]) / s; qu[2] = 0.25 * s; qu[3] = (om.a[1][2] + om.a[2][1]) / s;
  } else {
    const double s = 2.0 * std::sqrt(1.0 + om.a[2][2] - om.a[0][0] - om.a[1][1]);
    qu[0] = (om.a[1][0] - om.a[0][1]) / s; qu[1] = (om.a[0][2] + om.a[2][0]) / s; qu[2] = (om.a[1][2] + om.a[2][1]) / s; qu[3] = 0.25 * s;
  }
  if (std::signbit(qu[0])) for (int k = 0; k < 4; ++k) qu[k] = -qu[k];
  for (int k = 1; k < 4; ++k) if (!(std::fabs(qu[k]) <= 10.0 * TINY)) qu[k] = -qu[k];
  const double n = std::sqrt(qu[0] * qu[0] + qu[1] * qu[1] + qu[2] * qu[2] + qu[3] * qu[3]);
  for (int k = 0; k < 4; ++k) qu[k] /= n;
}
}  // namespace

// crystallite_orientations, phase.f90:659-673: O = fromMatrix(transpose(rotationalPart(Fe)));
// fromMatrix (rotations.f90:215-226) rejects |det - 1| > 1e-5 (IO_error 402)
static int orientations(const orc_ctx* c, double* out) {
  for (long v = 0; v < c->N; ++v) {
    const M3 om = tr(rotational_part(c->Fe[v]));
    if (!(std::fabs(det33(om) - 1.0) <= 1.0e-5)) return -2;
    om2qu(om, out + 4 * v);
  }
  return 0;
}

int orc_get_field(orc_ctx* c, int field, double* out) {
  if (field == 12) return orientations(c, out);
  if (field == 6 || field == 7) {
    const int Ns = c->pc.Ns;
    for (long v = 0; v < c->N; ++v) for (int s = 0; s < Ns; ++s) out[v * Ns + s] = c->state[v * c->sizeState + (field == 6 ? 0 : Ns) + s];
    return 0;
  }
  std::vector<M3>* f = field_ptr(c, field);
  if (!f) return -1;
  for (long v = 0; v < c->N; ++v) for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) out[9 * v + 3 * j + i] = (*f)[v].a[i][j];
  return 0;
}

int orc_set_field(orc_ctx* c, int field, const double* in) {
  std::vector<M3>* f = field_ptr(c, field);
  if (!f) return -1;
  for (long v = 0; v < c->N; ++v) for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) (*f)[v].a[i][j] = in[9 * v + 3 * j + i];
  return 0;
}

void orc_get_aims(orc_ctx* c, double F_aim[9], double P_aim[9], double C_volAvg[81], double C_minMaxAvg[81]) {
  for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) { F_aim[3 * j + i] = c->F_aim.a[i][j]; P_aim[3 * j + i] = c->P_aim.a[i][j]; }
  for (int l = 0; l < 3; ++l) for (int k = 0; k < 3; ++k) for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) {
    C_volAvg[i + 3 * j + 9 * k + 27 * l] = c->C_volAvg.a[i][j][k][l];
    C_minMaxAvg[i + 3 * j + 9 * k + 27 * l] = c->C_minMaxAvg.a[i][j][k][l];
  }
}

double orc_err_curl(orc_ctx* c) { return c->err_curl; }

void orc_counters(orc_ctx* c, int64_t out[4]) { for (int i = 0; i < 4; ++i) out[i] = c->counters[i]; }

int orc_schmid(const orc_phase* p, int sense, double* P) {
  std::vector<M3> v = schmid(*p, sense, true);
  for (size_t s = 0; s < v.size(); ++s) for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) P[9 * s + 3 * j + i] = v[s].a[i][j];
  return int(v.size());
}

int orc_interaction(const orc_phase* p, double* h) {
  int Ns;
  std::vector<double> v = interaction(*p, Ns);
  if (v.empty()) return -1;
  std::copy(v.begin(), v.end(), h);
  return Ns;
}

void orc_fft3(double* data, const int n[3], int sign) { fft3(reinterpret_cast<cd*>(data), n, sign); }

}  // extern "C"
