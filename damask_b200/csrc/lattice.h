// Host-side phase constants of the product: slip systems, Schmid and non-Schmid
// projections, slip-slip interaction matrix and the Mandel stiffness.
#pragma once
#include "../../include/damask_b200.h"

#include <array>
#include <string>
#include <vector>

namespace dmk {

struct HostPhase {
  int Ns = 0;
  double C66[6][6];
  double C[81];                                  // column-major 3x3x3x3
  std::vector<std::array<double, 9>> P, Ppos, Pneg;   // column-major 3x3 per system
  std::vector<std::array<double, 6>> dn;              // unit slip direction d and plane normal n: P = d (x) n
  std::vector<double> dg0, n, a, h0f, xiinf, xi0;
  std::vector<int> fam;                          // family of each system (-1: inert padding)
  std::vector<double> hfac;                      // h0f = h_0 of the family * hfac (twin factor, 1 here)
  int nf = 0;                                    // slip families
  double th[4][4] = {};                          // per family: xi_inf, h_0, n, a
  std::vector<double> h;                         // Ns x Ns, row = reacting system
  double atol_xi = 1.0, atol_gamma = 1.0e-6;
};

// Returns 0 on success; err describes invalid input otherwise.
int build_host_phase(const dmk_phase& p, HostPhase& hp, std::string& err);

// Miller indices (direction d1 d2 d3, plane normal n1 n2 n3) of the active slip systems
std::vector<std::array<int, 6>> slip_miller(const dmk_phase& p);

// Unit quaternion (w,x,y,z) -> orientation matrix, column-major (rotations.f90:399-423, P = -1)
void quaternion_to_matrix(const double* q, double* om);

// Dense inverse with partial pivoting (row-major n x n); true if singular.
bool invert_dense(const double* A, double* Ainv, int n);

}  // namespace dmk
