// Phase constants for the constitutive kernels (host).
//
//  slip systems / families        crystal.f90:43-220 (tables in lattice_tables.h)
//  Schmid + non-Schmid projection crystal_SchmidMatrix_slip, crystal.f90:1348-1454
//  coordinate system              buildCoordinateSystem, crystal.f90:1937-2001
//  slip-slip interaction          crystal_interaction_SlipBySlip / buildInteraction, crystal.f90:591-902,1893-1930
//  stiffness (Mandel)             crystal_assembleStiffness, crystal.f90:1711-1759; math_66toSym3333, math.f90:851
//  hardening prefactor            phenopowerlaw_dotState, phenopowerlaw.f90:356-399 (no twins: sumF = 0)
#include "lattice.h"
#include "lattice_tables.h"

#include <cmath>
#include <cstring>

namespace dmk {

namespace {

const double PI = 3.14159265358979323846;

void normalize(double* v) {
  const double n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  for (int i = 0; i < 3; ++i) v[i] /= n;
}
void cross(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
void add_outer(double s, const double* a, const double* b, double* M) {
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) M[i + 3 * j] += s * a[i] * b[j];
}
// passive rotation of a vector by quaternion q (P = -1)
void rotate_vector(const double* v, const double* q, double* o) {
  const double A = q[0] * q[0] - (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  const double B = 2.0 * (q[1] * v[0] + q[2] * v[1] + q[3] * v[2]);
  const double C = -2.0 * q[0];
  double c[3];
  const double qv[3] = {q[1], q[2], q[3]};
  cross(qv, v, c);
  for (int i = 0; i < 3; ++i) o[i] = A * v[i] + B * qv[i] + C * c[i];
}

// unit slip direction and plane normal of every system (the factors of the Schmid matrix)
std::vector<std::array<double, 6>> slip_dn(const dmk_phase& p) {
  const int* famMax = p.lattice == 0 ? CF_NSLIP_FAMILY : CI_NSLIP_FAMILY;
  std::vector<std::array<double, 6>> out;
  int base = 0;
  for (int f = 0; f < p.n_families; ++f) {
    for (int s = 0; s < p.N_sl[f]; ++s) {
      const signed char* row = p.lattice == 0 ? CF_SLIP_SYSTEMS[base + s] : CI_SLIP_SYSTEMS[base + s];
      double d[3] = {double(row[0]), double(row[1]), double(row[2])};
      double n[3] = {double(row[3]), double(row[4]), double(row[5])};
      normalize(d);
      normalize(n);
      out.push_back({d[0], d[1], d[2], n[0], n[1], n[2]});
    }
    base += famMax[f];
  }
  return out;
}

// Schmid matrices for one sense; non-Schmid terms for cI family 1
std::vector<std::array<double, 9>> schmid(const dmk_phase& p, int sense, bool with_nonschmid) {
  const int* famMax = p.lattice == 0 ? CF_NSLIP_FAMILY : CI_NSLIP_FAMILY;
  std::vector<std::array<double, 9>> out;
  int base = 0;
  for (int f = 0; f < p.n_families; ++f) {
    for (int s = 0; s < p.N_sl[f]; ++s) {
      const signed char* row = p.lattice == 0 ? CF_SLIP_SYSTEMS[base + s] : CI_SLIP_SYSTEMS[base + s];
      double d[3] = {double(row[0]), double(row[1]), double(row[2])};
      double n[3] = {double(row[3]), double(row[4]), double(row[5])};
      normalize(d);
      normalize(n);
      for (int i = 0; i < 3; ++i) d[i] *= double(sense);
      std::array<double, 9> M{};
      add_outer(1.0, d, n, M.data());
      if (with_nonschmid && p.lattice == 1 && f == 0 && p.n_nonschmid > 0) {
        // rotation about the slip direction by 60 degrees, constructed with P = +1
        // (axis negated), applied passively: n_p = R n
        const double half = 0.5 * 60.0 * PI / 180.0;
        const double q[4] = {std::cos(half), -d[0] * std::sin(half), -d[1] * std::sin(half), -d[2] * std::sin(half)};
        double np[3], nxd[3], npxd[3];
        rotate_vector(n, q, np);
        cross(n, d, nxd);
        cross(np, d, npxd);
        double c[6] = {0, 0, 0, 0, 0, 0};
        for (int k = 0; k < p.n_nonschmid; ++k) c[k] = p.a_nonschmid[k];
        add_outer(c[0], d, np, M.data());
        add_outer(c[1], nxd, n, M.data());
        add_outer(c[2], npxd, np, M.data());
        add_outer(c[3], n, n, M.data());
        add_outer(c[4], nxd, nxd, M.data());
        add_outer(c[5], d, d, M.data());
      }
      out.push_back(M);
    }
    base += famMax[f];
  }
  return out;
}

}  // namespace

int build_host_phase(const dmk_phase& p, HostPhase& hp, std::string& err) {
  if (p.lattice != 0 && p.lattice != 1) { err = "lattice must be cF or cI"; return -1; }
  const int nfMax = p.lattice == 0 ? 2 : 3;
  const int* famMax = p.lattice == 0 ? CF_NSLIP_FAMILY : CI_NSLIP_FAMILY;
  if (p.n_families < 1 || p.n_families > nfMax) { err = "invalid number of slip families"; return -1; }
  int Ns = 0;
  for (int f = 0; f < p.n_families; ++f) {
    if (p.N_sl[f] < 0 || p.N_sl[f] > famMax[f]) { err = "N_sl exceeds the systems of the family"; return -1; }
    if (!(p.dot_gamma_0[f] > 0.0) || !(p.n[f] > 0.0) || !(p.a[f] > 0.0) || !(p.xi_0[f] > 0.0) || !(p.xi_inf[f] > 0.0)) {
      err = "phenopowerlaw parameters out of range (dot_gamma_0_sl, n_sl, a_sl, xi_0_sl, xi_inf_sl must be > 0)";
      return -1;
    }
    Ns += p.N_sl[f];
  }
  if (p.n_nonschmid < 0 || p.n_nonschmid > 6 || (p.n_nonschmid > 0 && p.lattice != 1)) {
    err = "non-Schmid coefficients are supported for cI only (at most 6)";
    return -1;
  }
  if (!(p.atol_xi >= 0.0) || !(p.atol_gamma >= 0.0)) { err = "negative state tolerance"; return -1; }
  hp.Ns = Ns;
  // stiffness in Mandel notation (cubic)
  std::memset(hp.C66, 0, sizeof hp.C66);
  hp.C66[0][0] = hp.C66[1][1] = hp.C66[2][2] = p.C11;
  hp.C66[0][1] = hp.C66[1][0] = hp.C66[0][2] = hp.C66[2][0] = hp.C66[1][2] = hp.C66[2][1] = p.C12;
  hp.C66[3][3] = hp.C66[4][4] = hp.C66[5][5] = p.C44 * 2.0;
  // expand to 3x3x3x3 (Mandel weights: 1/sqrt(2) for normal-shear, 1/2 for shear-shear)
  const int vi[6] = {0, 1, 2, 1, 0, 0}, vj[6] = {0, 1, 2, 2, 2, 1};
  for (int a = 0; a < 6; ++a)
    for (int b = 0; b < 6; ++b) {
      // math_66toSym3333 weights: 1/sqrt(2) for one shear index, 1/2 for two
      const double w = (a >= 3 && b >= 3) ? 1.0 / 2.0 : (a >= 3 || b >= 3) ? 1.0 / std::sqrt(2.0) : 1.0;
      const double v = hp.C66[a][b] * w;
      const int ii[2] = {vi[a], vj[a]}, jj[2] = {vj[a], vi[a]};
      const int kk[2] = {vi[b], vj[b]}, ll[2] = {vj[b], vi[b]};
      for (int x = 0; x < 2; ++x)
        for (int y = 0; y < 2; ++y) hp.C[ii[x] + 3 * jj[x] + 9 * kk[y] + 27 * ll[y]] = v;
    }
  hp.P = schmid(p, +1, false);
  hp.dn = slip_dn(p);
  hp.Ppos = schmid(p, +1, true);
  hp.Pneg = schmid(p, -1, true);
  // interaction matrix
  hp.h.assign(size_t(Ns) * Ns, 0.0);
  int ka = 0;
  for (int fa = 0; fa < p.n_families; ++fa) {
    int offa = 0;
    for (int q = 0; q < fa; ++q) offa += famMax[q];
    for (int sa = 0; sa < p.N_sl[fa]; ++sa, ++ka) {
      int kr = 0;
      for (int fr = 0; fr < p.n_families; ++fr) {
        int offr = 0;
        for (int q = 0; q < fr; ++q) offr += famMax[q];
        for (int sr = 0; sr < p.N_sl[fr]; ++sr, ++kr) {
          const int type = p.lattice == 0 ? CF_INTERACTION[offr + sr][offa + sa] : CI_INTERACTION[offr + sr][offa + sa];
          if (type > p.n_h) {
            err = "h_sl-sl has too few values for the active slip families";
            return -1;
          }
          hp.h[size_t(kr) * Ns + ka] = p.h_sl_sl[type - 1];
        }
      }
    }
  }
  for (int f = 0; f < p.n_families; ++f)
    for (int s = 0; s < p.N_sl[f]; ++s) {
      hp.dg0.push_back(p.dot_gamma_0[f]);
      hp.n.push_back(p.n[f]);
      hp.a.push_back(p.a[f]);
      // h_0 * (1 + c_1 * sumF**c_2) with sumF = 0 (no twin systems)
      hp.h0f.push_back(p.h_0[f] * (1.0 + p.c_1[f] * std::pow(0.0, p.c_2[f])));
      hp.xiinf.push_back(p.xi_inf[f] + p.f_sat[f] * std::sqrt(0.0));
      hp.xi0.push_back(p.xi_0[f]);
      hp.fam.push_back(f);
      hp.hfac.push_back(1.0 + p.c_1[f] * std::pow(0.0, p.c_2[f]));
    }
  hp.nf = p.n_families;
  for (int f = 0; f < p.n_families; ++f) {
    hp.th[0][f] = p.xi_inf[f];
    hp.th[1][f] = p.h_0[f];
    hp.th[2][f] = p.n[f];
    hp.th[3][f] = p.a[f];
  }
  hp.atol_xi = p.atol_xi;
  hp.atol_gamma = p.atol_gamma;
  return 0;
}

void quaternion_to_matrix(const double* q, double* om) {
  const double qq = q[0] * q[0] - (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  double m[3][3];
  m[0][0] = qq + 2.0 * q[1] * q[1];
  m[1][1] = qq + 2.0 * q[2] * q[2];
  m[2][2] = qq + 2.0 * q[3] * q[3];
  m[0][1] = 2.0 * (q[1] * q[2] - q[0] * q[3]);
  m[1][2] = 2.0 * (q[2] * q[3] - q[0] * q[1]);
  m[2][0] = 2.0 * (q[3] * q[1] - q[0] * q[2]);
  m[1][0] = 2.0 * (q[2] * q[1] + q[0] * q[3]);
  m[2][1] = 2.0 * (q[3] * q[2] + q[0] * q[1]);
  m[0][2] = 2.0 * (q[1] * q[3] + q[0] * q[2]);
  // P = -1: transpose; then renormalise by det^(1/3)
  double t[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) t[i + 3 * j] = m[j][i];
  const double det = t[0] * (t[4] * t[8] - t[7] * t[5]) - t[3] * (t[1] * t[8] - t[7] * t[2]) + t[6] * (t[1] * t[5] - t[4] * t[2]);
  const double c = std::cbrt(det);
  for (int k = 0; k < 9; ++k) om[k] = t[k] / c;
}

bool invert_dense(const double* A, double* Ainv, int n) {
  std::vector<double> M(A, A + size_t(n) * n), I(size_t(n) * n, 0.0);
  for (int i = 0; i < n; ++i) I[size_t(i) * n + i] = 1.0;
  for (int j = 0; j < n; ++j) {
    int p = j;
    for (int i = j + 1; i < n; ++i)
      if (std::fabs(M[size_t(i) * n + j]) > std::fabs(M[size_t(p) * n + j])) p = i;
    if (M[size_t(p) * n + j] == 0.0) return true;
    if (p != j)
      for (int k = 0; k < n; ++k) {
        std::swap(M[size_t(j) * n + k], M[size_t(p) * n + k]);
        std::swap(I[size_t(j) * n + k], I[size_t(p) * n + k]);
      }
    const double r = 1.0 / M[size_t(j) * n + j];
    for (int k = 0; k < n; ++k) { M[size_t(j) * n + k] *= r; I[size_t(j) * n + k] *= r; }
    for (int i = 0; i < n; ++i) {
      if (i == j) continue;
      const double l = M[size_t(i) * n + j];
      if (l == 0.0) continue;
      for (int k = 0; k < n; ++k) {
        M[size_t(i) * n + k] -= l * M[size_t(j) * n + k];
        I[size_t(i) * n + k] -= l * I[size_t(j) * n + k];
      }
    }
  }
  std::memcpy(Ainv, I.data(), sizeof(double) * size_t(n) * n);
  return false;
}

// Miller indices (direction, plane normal) of the active systems, in system order
std::vector<std::array<int, 6>> slip_miller(const dmk_phase& p) {
  const int* famMax = p.lattice == 0 ? CF_NSLIP_FAMILY : CI_NSLIP_FAMILY;
  std::vector<std::array<int, 6>> out;
  int base = 0;
  for (int f = 0; f < p.n_families; ++f) {
    for (int s = 0; s < p.N_sl[f]; ++s) {
      const signed char* row = p.lattice == 0 ? CF_SLIP_SYSTEMS[base + s] : CI_SLIP_SYSTEMS[base + s];
      out.push_back({row[0], row[1], row[2], row[3], row[4], row[5]});
    }
    base += famMax[f];
  }
  return out;
}

}  // namespace dmk
