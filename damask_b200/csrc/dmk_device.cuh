// Device-side types and small-tensor helpers for the damask_b200 kernels.
//
// Layout in HBM: every per-voxel quantity is stored as structure-of-arrays
// "planes": component c of voxel v lives at base[c * N + v], so a warp reading
// one component of 32 consecutive voxels issues one coalesced 256-byte request.
// 3x3 tensors use the Fortran component order c = i + 3*j; the symmetric stress
// S uses six planes (11, 22, 33, 23, 13, 12).
#pragma once
#include <type_traits>
#include <cuda_runtime.h>
#include <stdint.h>

namespace dmk {

constexpr double TINY10 = 10.0 * 2.2250738585072014e-308;   // dEq0 threshold, prec.f90:131-143

struct SysConst;

// Per-phase constants, passed by value as a __grid_constant__ kernel parameter so
// that every uniform access is served by the constant bank.
template <int NS>
struct PhaseConst {
  double C66[6][6];        // Mandel stiffness (crystal_assembleStiffness, crystal.f90:1711-1759)
  double C[81];            // math_66toSym3333(C66), column-major 3x3x3x3
  double P[NS][9];         // Schmid matrices P_sl (column-major)
  double p6[2][NS][6];     // tau = S : P_nS  ->  symmetric weights (pos/neg sense)
  double q6[2][NS][6];     // Q = C : P_nS, symmetric (11,22,33,23,13,12)
  double PnS[2][NS][9];    // P_nS (pos/neg sense), column-major
  double dn[NS][6];        // slip direction d and plane normal n (unit): P = d (x) n
  double dg0[NS], n[NS], a[NS], h0f[NS], xiinf[NS], ixiinf[NS];
  const double* hmat;      // slip-slip hardening matrix (NS x NS, row = reacting system) in device memory
  const SysConst* sys;     // the per-system constants of the Newton loop (NS entries) in device memory
  int n_int[NS];           // stress exponent as integer if integral, else -1
  int a_int[NS];           // hardening exponent as integer if integral, else -1
  double atol_xi, atol_gamma;
  // slip families (used by the adjoint's local model)
  int fam[NS];             // family of system s, -1 for inert padding
  double hfac[NS];         // h0f[s] = h_0 of the family * hfac[s]
  int nf;                  // number of families
  double th[4][4];         // per family: xi_inf, h_0, n, a (the parameters of the gradient)
};

struct Numerics {
  double r_cutback_min, r_cutback, r_increase, eps_rel_state;
  int N_iter_state_max, N_iter_Lp_max;
  double r_linesearch_Lp, eps_rel_Lp, eps_abs_Lp;
  int f_update_jacobi_Lp;
};

// Device pointers of one RVE's fields.
struct Fields {
  int64_t N;
  double* Fsol;     // solver F (9 planes)
  const double* r;  // residual of the previous evaluation (9 planes) or null
  double* F;        // phase F (9)
  double* F0;       // phase F0 (9)
  double* Fp;       // (9)
  double* Fp0;      // (9)
  double* Lp;       // (9)
  double* Lp0;      // (9)
  double* S;        // (6)
  double* S0;       // (6)
  double* Fe;       // (9)
  double* P;        // output stress of this evaluation (9)
  double* state;    // (2 NS)
  double* state0;   // (2 NS)
  double* partials; // per block: 9 sums of P
  int* status;      // worst status (atomicMax)
  int* iter;        // optional per-voxel counters: 4 ints per voxel (planes)
  unsigned long long* counters;   // [0] evaluations [1] state iterations [2] Newton iterations
};

constexpr int PASS_THREADS = 128;   // threads per block of the pass kernels
// threads per block of the pass kernels for NS systems: 64 above 24 systems, where the per-thread
// shared-memory slots of 128-thread blocks would leave one block per SM in the begin and control kernels
template <int NS>
__host__ __device__ constexpr int pass_threads() { return NS > 24 ? 64 : PASS_THREADS; }

// Per-voxel iteration state of the pass scheme (planes of N entries each).
struct PassWork {
  double* Fs;      // 9: F of the current substep
  double* F0s;     // 9: F at the start of the current substep (subF0)
  double* Fp0s;    // 9: subFp0
  double* Lp0s;    // 9: subLp0
  double* st0s;    // 2 NS: subState0
  double* D;       // 2 x 2 NS: (damped) dotState of the last two state iterations
  double* adg;     // NS: |dot_gamma| at the stress of the last converged integrateStress
  double* dot0;    // 2 NS: dotState at the increment-start stress and state (S0, state0)
  double* sub;     // 2: stepFrac (subFrac), step (subStep)
  double* lo;      // 9: the last accepted Lp guess of the current integrateStress
  double* dl;      // 9: its Newton step
  int* ctl;        // 6: phase, status, state iteration, substeps, state iterations total, Newton total
  int* list_out;   // voxels that continue into the next pass
  int* count_out;  // number of entries appended to list_out
};

enum : int { PH_CTRL = 0, PH_DOT0 = 1, PH_STRESS = 2, PH_DOT1 = 3, PH_DONE = 4 };

struct VoxelCtl {
  int phase, status, it, nsub, nstate, newton;
  double stepFrac, step;
};

// ------------------------------------------------------------- 3x3 helpers
// Column-major: a[i + 3*j] = A(i,j)
__device__ __forceinline__ void mm33(const double* A, const double* B, double* C) {
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 3; ++i)
      C[i + 3 * j] = A[i] * B[3 * j] + A[i + 3] * B[1 + 3 * j] + A[i + 6] * B[2 + 3 * j];
}
// C = A^T B
__device__ __forceinline__ void mtm33(const double* A, const double* B, double* C) {
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 3; ++i)
      C[i + 3 * j] = A[3 * i] * B[3 * j] + A[1 + 3 * i] * B[1 + 3 * j] + A[2 + 3 * i] * B[2 + 3 * j];
}
// C = A B^T
__device__ __forceinline__ void mmt33(const double* A, const double* B, double* C) {
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 3; ++i)
      C[i + 3 * j] = A[i] * B[j] + A[i + 3] * B[j + 3] + A[i + 6] * B[j + 6];
}
__device__ __forceinline__ double det33(const double* m) {
  return m[0] * (m[4] * m[8] - m[7] * m[5]) - m[3] * (m[1] * m[8] - m[7] * m[2]) + m[6] * (m[1] * m[5] - m[4] * m[2]);
}
// math_invert33 (Cramer), math.f90:471-509; returns true on error
__device__ __forceinline__ bool inv33(const double* A, double* I) {
  I[0] = A[4] * A[8] - A[7] * A[5];
  I[1] = -A[1] * A[8] + A[7] * A[2];
  I[2] = A[1] * A[5] - A[4] * A[2];
  const double det = A[0] * I[0] + A[3] * I[1] + A[6] * I[2];
  if (fabs(det) <= TINY10) return true;
  I[3] = -A[3] * A[8] + A[6] * A[5];
  I[4] = A[0] * A[8] - A[6] * A[2];
  I[5] = -A[0] * A[5] + A[3] * A[2];
  I[6] = A[3] * A[7] - A[6] * A[4];
  I[7] = -A[0] * A[7] + A[6] * A[1];
  I[8] = A[0] * A[4] - A[3] * A[1];
  const double r = 1.0 / det;
#pragma unroll
  for (int k = 0; k < 9; ++k) I[k] *= r;
  return false;
}
__device__ __forceinline__ double norm9(const double* x) {
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 9; ++k) s = fma(x[k], x[k], s);
  return sqrt(s);
}
// x^n for a non-negative integer n by binary powering
__device__ __forceinline__ double powi(double x, int n) {
  double r = 1.0;
  while (n) {
    if (n & 1) r *= x;
    n >>= 1;
    if (n) x *= x;
  }
  return r;
}
// x^n for 0 <= n < 2^BITS: the products of powi in the same order, as a fixed
// sequence of predicated steps (no data-dependent branch)
template <int BITS>
__device__ __forceinline__ double powi_fixed(double x, int n) {
  double r = 1.0;
#pragma unroll
  for (int b = 0; b < BITS; ++b) {
    if ((n >> b) & 1) r *= x;
    x *= x;
  }
  return r;
}
// integral exponents are at most 64 (set up on the host), otherwise pow
// (exponents are per slip system, so the powering loop is uniform across a warp)
__device__ __forceinline__ double powr(double x, double e, int ei) { return ei >= 0 ? powi(x, ei) : pow(x, e); }

// Per slip system constants of the Newton loop, staged in shared memory once per
// block; pairs hold the positive and negative sense so that one 16-byte load serves both.
// one bit per slip system (the sense of its resolved shear): 32 bits up to 32 systems, else 64
template <int NS>
using SenseMask = typename std::conditional<(NS > 32), unsigned long long, unsigned>::type;

struct SysConst {
  double2 p6[6];     // (p6[0][s][t], p6[1][s][t]): tau = S : P_nS
  double2 q6[6];     // (q6[0][s][t], q6[1][s][t]): Q = C : P_nS
  double2 P[5];      // P_s in column-major order, P[4].y unused
  double2 dn[3];     // (d0, d1), (d2, n0), (n1, n2): P = d (x) n
  double2 kin;       // (dot_gamma_0, n)
  int n_int;         // stress exponent if integral (1..64), else -1
  int pad[3];
};

// Host-side assembly of the per-system constants (the device copy is staged into shared memory
// by stage_sys_const with coalesced 16-byte loads).
template <int NS>
__host__ __device__ inline SysConst make_sys_const(const PhaseConst<NS>& pc, int i) {
  SysConst c;
  for (int t = 0; t < 6; ++t) {
    c.p6[t] = make_double2(pc.p6[0][i][t], pc.p6[1][i][t]);
    c.q6[t] = make_double2(pc.q6[0][i][t], pc.q6[1][i][t]);
  }
  for (int k = 0; k < 4; ++k) c.P[k] = make_double2(pc.P[i][2 * k], pc.P[i][2 * k + 1]);
  c.P[4] = make_double2(pc.P[i][8], 0.0);
  c.dn[0] = make_double2(pc.dn[i][0], pc.dn[i][1]);
  c.dn[1] = make_double2(pc.dn[i][2], pc.dn[i][3]);
  c.dn[2] = make_double2(pc.dn[i][4], pc.dn[i][5]);
  c.kin = make_double2(pc.dg0[i], pc.n[i]);
  c.n_int = pc.n_int[i];
  c.pad[0] = c.pad[1] = c.pad[2] = 0;
  return c;
}

// Copies the NS per-system constants from device memory into shared memory: every thread of
// the block moves 16-byte words of the contiguous array (no per-thread divergent reads of the
// parameter space).
template <int NS>
__device__ __forceinline__ void stage_sys_const(const PhaseConst<NS>& pc, SysConst* sc) {
  constexpr int WORDS = NS * int(sizeof(SysConst) / sizeof(double2));
  const double2* __restrict__ src = reinterpret_cast<const double2*>(pc.sys);
  double2* dst = reinterpret_cast<double2*>(sc);
  for (int i = threadIdx.x; i < WORDS; i += blockDim.x) dst[i] = src[i];
}

// Hooke in Mandel notation with Fi = I: S = C66 : sym6(E), E = (Fe^T Fe - I)/2
// (phase_hooke_SandItsTangents, phase_mechanical_elastic.f90:172-205)
template <int NS>
__device__ __forceinline__ void hooke_S(const PhaseConst<NS>& pc, const double* Fe, double s6[6]) {
  const double W = 1.4142135623730951;        // WGT_MANDEL(1) = sqrt(2)
  const double IW = 1.0 / W;                  // 1/WGT_MANDEL(1)
  double E[6];
  // E = 0.5 (Fe^T Fe - I): (11,22,33,23,13,12)
  E[0] = 0.5 * (Fe[0] * Fe[0] + Fe[1] * Fe[1] + Fe[2] * Fe[2] - 1.0);
  E[1] = 0.5 * (Fe[3] * Fe[3] + Fe[4] * Fe[4] + Fe[5] * Fe[5] - 1.0);
  E[2] = 0.5 * (Fe[6] * Fe[6] + Fe[7] * Fe[7] + Fe[8] * Fe[8] - 1.0);
  E[3] = 0.5 * (Fe[3] * Fe[6] + Fe[4] * Fe[7] + Fe[5] * Fe[8]) * W;
  E[4] = 0.5 * (Fe[0] * Fe[6] + Fe[1] * Fe[7] + Fe[2] * Fe[8]) * W;
  E[5] = 0.5 * (Fe[0] * Fe[3] + Fe[1] * Fe[4] + Fe[2] * Fe[5]) * W;
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) s = fma(pc.C66[i][k], E[k], s);
    s6[i] = i < 3 ? s : s * IW;
  }
}

__device__ __forceinline__ double dot6(const double* a, const double* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3] + a[4] * b[4] + a[5] * b[5];
}

// warp + block reduction of a small vector; result valid in thread 0
template <int K>
__device__ __forceinline__ void block_reduce_sum(double (&v)[K], double* smem /* K * nwarps */) {
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) smem[k * nw + warp] = v[k];
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double s = 0.0;
      for (int w = 0; w < nw; ++w) s += smem[k * nw + w];
      v[k] = s;
    }
}

}  // namespace dmk
