// Consistent tangent dP/dF per voxel (phase_mechanical_dPdF, phase_mechanical.f90:1121-1242)
// with Fi = I, Li = 0 (dFi/dS = 0), and the reductions that consume it in
// utilities_constitutiveResponse (grid_utilities.f90:171-202): the volume sum (C_volAvg)
// and the voxels of maximal and minimal Frobenius norm (C_minMaxAvg).
//
// The tangent is only consumed by those two averages, which the solver reads at the start of
// the next increment (masked compliance) or for the Gamma reference stiffness; the host
// therefore evaluates it once per converged increment from the stored converged state
// instead of inside every residual evaluation.  The values equal those of the last residual
// evaluation because they depend only on the stored F, Fe, Fp, Fp0, S and state.
//
// Structure used.  The reference solves (I + lhs) : dS/dF = rhs with lhs = dt dS/dFe :
// (A dLp/dS), A = F Fp0^-1, as a 9x9 system.  dS is symmetric and dLp/dS only sees its
// symmetric part (dLp = K s with K = sum_s dgamma_s P_s (x) p_s, s = the 6 independent
// components of dS, p_s the weights of tau = S : P_nS), so the system is the 6x6
//     (I6 + L) s = r,   L = dt sym6(C : sym(Fe^T A K)),   r = sym6(C : sym(Fe^T dF Fp^-1)),
// solved by Householder QR once per voxel for the 9 unit perturbations dF = e_p (x) e_o.
// Each perturbation then gives one column of dP/dF:
//     dFp^-1 = -dt Fp0^-1 dLp,
//     dP = dF Fp^-1 S Fp^-T + F dFp^-1 S Fp^-T + F Fp^-1 dS Fp^-T + F Fp^-1 S dFp^-T.
// The 81 components go to planes (component i + 3j + 9p + 27o of voxel v at [c N + v]) and are
// summed by a separate, coalesced reduction in a fixed order.
#include "kernels.cuh"
#include "constitutive.cuh"

#include <algorithm>

namespace dmk {

constexpr int TAN_THREADS = 64;
// per-thread shared-memory slots (stride TAN_THREADS):
//   [0, 54)    K (9x6, row q = k + 3 l)
//   [54, 90)   L (6x6) while it is built, then a1, a2, a3, d (3x3 each)
//   [90, 99)   Fp0^-1
//   [99, 99 + G)      dgamma (NS entries) while K is built, then Fe and Fp^-1 (3x3 each);
//                     G = max(NS, 24)
//   [99 + G, 108 + G) F
template <int NS>
__host__ __device__ constexpr int tan_dg_slots() { return NS > 24 ? NS : 24; }
template <int NS>
__host__ __device__ constexpr int tan_slots() { return 108 + tan_dg_slots<NS>(); }

// sym6(C : sym(Y)) for a 3x3 Y (column-major), through the Mandel stiffness; (11 22 33 23 13 12)
template <int NS>
__device__ __forceinline__ void hooke_sym(const PhaseConst<NS>& pc, const double* Y, double r[6]) {
  const double W = 1.4142135623730951;
  const double E[6] = {Y[0], Y[4], Y[8], 0.5 * (Y[5] + Y[7]) * W, 0.5 * (Y[2] + Y[6]) * W, 0.5 * (Y[1] + Y[3]) * W};
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) s = fma(pc.C66[i][k], E[k], s);
    r[i] = i < 3 ? s : s * (1.0 / W);
  }
}

// dP/dF of voxel v into planes (stride N); returns its squared Frobenius norm
template <int NS>
__device__ double tangent_voxel(const PhaseConst<NS>& pc, const Fields& f, int64_t v, double dt,
                                double* __restrict__ planes, double* xs) {
  constexpr int T = TAN_THREADS;
  const int64_t N = f.N;
  double* const sK = xs;
  double* const sL = xs + 54 * T;              // later: a1, a2, a3, d
  double* const sFp0i = xs + 90 * T;
  double* const sdg = xs + 99 * T;             // later: Fe, Fp^-1
  double* const sF = xs + (99 + tan_dg_slots<NS>()) * T;
  double s6[6];
  {
    double F[9], invFp[9], Fe[9], Fp[9], Fp0[9], invFp0[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      F[k] = f.F[k * N + v]; Fe[k] = f.Fe[k * N + v]; Fp[k] = f.Fp[k * N + v]; Fp0[k] = f.Fp0[k * N + v];
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) s6[k] = f.S[k * N + v];
    inv33(Fp, invFp);
    inv33(Fp0, invFp0);
#pragma unroll
    for (int k = 0; k < 9; ++k) sFp0i[k * T] = invFp0[k];
    // kinetics (phenopowerlaw.f90:303-350): dgamma_s and the sense of each system
    static_assert(NS <= 64, "one sense bit per slip system");
    SenseMask<NS> neg = 0u;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const double tp = dot6(s6, pc.p6[0][s]), tn = dot6(s6, pc.p6[1][s]);
      const bool pos = tp > tn;
      const double tmax = pos ? tp : tn;
      const double g = (pos ? pc.dg0[s] : -pc.dg0[s]) * powr(tmax / f.state[s * N + v], pc.n[s], pc.n_int[s]);
      sdg[s * T] = fabs(g) > TINY10 ? g * pc.n[s] / tmax : 0.0;
      if (!(g > 0.0)) neg |= SenseMask<NS>(1) << s;
    }
    // K = dLp/dS on symmetric dS, column by column: K_c = sum_s dgamma_s p_s[c] P_s; and
    // L_c = e_c + dt sym6(C : sym(B K_c)) with B = Fe^T A, A = F Fp0^-1
    double A[9], B[9];
    mm33(F, invFp0, A);
    mtm33(Fe, A, B);
#pragma unroll 1
    for (int c = 0; c < 6; ++c) {
      double Y[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const double w = sdg[s * T] * pc.p6[(neg >> s) & 1u][s][c];
#pragma unroll
        for (int q = 0; q < 9; ++q) Y[q] = fma(w, pc.P[s][q], Y[q]);
      }
#pragma unroll
      for (int q = 0; q < 9; ++q) sK[(6 * q + c) * T] = Y[q];
      double BY[9], h[6];
      mm33(B, Y, BY);
      hooke_sym<NS>(pc, BY, h);
#pragma unroll
      for (int r = 0; r < 6; ++r) sL[(6 * r + c) * T] = (r == c ? 1.0 : 0.0) + dt * h[r];
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      sdg[k * T] = Fe[k];
      sdg[(9 + k) * T] = invFp[k];
      sF[k * T] = F[k];
    }
  }
  double L[36], v0[5], rs[5];
#pragma unroll
  for (int i = 0; i < 36; ++i) L[i] = sL[i * T];
  {
    double F[9], invFp[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) { F[k] = sF[k * T]; invFp[k] = sdg[(9 + k) * T]; }
    // assembly factors: a1 = S Fp^-T, a2 = F Fp^-1, a3 = F Fp^-1 S, d = Fp^-1 S Fp^-T
    const double Sm[9] = {s6[0], s6[5], s6[4], s6[5], s6[1], s6[3], s6[4], s6[3], s6[2]};
    double a1[9], a2[9], a3[9], d[9];
    mmt33(Sm, invFp, a1);
    mm33(F, invFp, a2);
    mm33(a2, Sm, a3);
    mm33(invFp, a1, d);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      sL[k * T] = a1[k]; sL[(9 + k) * T] = a2[k]; sL[(18 + k) * T] = a3[k]; sL[(27 + k) * T] = d[k];
    }
  }
  // Householder QR of I6 + L (reflectors below the diagonal, as qr_solve)
  bool singular = false;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    double s2 = 0.0;
#pragma unroll
    for (int i = k; i < 6; ++i) s2 = fma(L[6 * i + k], L[6 * i + k], s2);
    if (s2 == 0.0) singular = true;
    const double sig = sqrt(s2);
    const double x0 = L[6 * k + k];
    const double alpha = x0 >= 0.0 ? -sig : sig;
    v0[k] = x0 - alpha;
    rs[k] = s2 == 0.0 ? 0.0 : 1.0 / (alpha * v0[k]);
#pragma unroll
    for (int c = k + 1; c < 6; ++c) {
      double dd = v0[k] * L[6 * k + c];
#pragma unroll
      for (int i = k + 1; i < 6; ++i) dd = fma(L[6 * i + k], L[6 * i + c], dd);
      dd *= rs[k];
      L[6 * k + c] = fma(dd, v0[k], L[6 * k + c]);
#pragma unroll
      for (int i = k + 1; i < 6; ++i) L[6 * i + c] = fma(dd, L[6 * i + k], L[6 * i + c]);
    }
    L[6 * k + k] = alpha;
  }
  if (L[35] == 0.0) singular = true;
  double norm = 0.0;
#pragma unroll 1
  for (int po = 0; po < 9; ++po) {
    const int o = po / 3, p = po % 3;              // dF = e_p (x) e_o: component index 9 p + 27 o
    // r = sym6(C : sym(Fe^T dF Fp^-1)): (Fe^T dF Fp^-1)(m,l) = Fe(p,m) Fp^-1(o,l)
    double Y[9], s[6];
#pragma unroll
    for (int l = 0; l < 3; ++l)
#pragma unroll
      for (int m = 0; m < 3; ++m) Y[m + 3 * l] = sdg[(p + 3 * m) * T] * sdg[(9 + o + 3 * l) * T];
    hooke_sym<NS>(pc, Y, s);
    if (!singular) {
      // (I6 + L) s = r: apply the reflectors, back-substitute (phase_mechanical.f90:1205-1211)
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        double dd = v0[k] * s[k];
#pragma unroll
        for (int i = k + 1; i < 6; ++i) dd = fma(L[6 * i + k], s[i], dd);
        dd *= rs[k];
        s[k] = fma(dd, v0[k], s[k]);
#pragma unroll
        for (int i = k + 1; i < 6; ++i) s[i] = fma(dd, L[6 * i + k], s[i]);
      }
#pragma unroll
      for (int i = 5; i >= 0; --i) {
        double t = s[i];
#pragma unroll
        for (int k = i + 1; k < 6; ++k) t = fma(-L[6 * i + k], s[k], t);
        s[i] = t / L[6 * i + i];
      }
    }                                               // singular: dS/dF = rhs, as the reference
    // dP(:,:,p,o) = delta_ip d(o,:) + a2 dS Fp^-T + F dFpi a1 + a3 dFpi^T, accumulated term by term
    double acc[9], a[9], T1[9];
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int i = 0; i < 3; ++i) acc[i + 3 * j] = i == p ? sL[(27 + o + 3 * j) * T] : 0.0;
    {
      const double dS[9] = {s[0], s[5], s[4], s[5], s[1], s[3], s[4], s[3], s[2]};
#pragma unroll
      for (int k = 0; k < 9; ++k) a[k] = sL[(9 + k) * T];
      mm33(a, dS, T1);                                // a2 dS
#pragma unroll
      for (int k = 0; k < 9; ++k) a[k] = sdg[(9 + k) * T];
#pragma unroll
      for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int i = 0; i < 3; ++i)                   // + (a2 dS) Fp^-T
          acc[i + 3 * j] += T1[i] * a[j] + T1[i + 3] * a[j + 3] + T1[i + 6] * a[j + 6];
    }
    // dLp = K s, dFp^-1 = -dt Fp0^-1 dLp
    double dFpi[9];
    {
      double dLp[9];
#pragma unroll
      for (int q = 0; q < 9; ++q) {
        double t = 0.0;
#pragma unroll
        for (int c = 0; c < 6; ++c) t = fma(sK[(6 * q + c) * T], s[c], t);
        dLp[q] = t;
      }
#pragma unroll
      for (int k = 0; k < 9; ++k) a[k] = sFp0i[k * T];
      mm33(a, dLp, dFpi);
#pragma unroll
      for (int k = 0; k < 9; ++k) dFpi[k] *= -dt;
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) a[k] = sF[k * T];
    mm33(a, dFpi, T1);                                // F dFpi
#pragma unroll
    for (int k = 0; k < 9; ++k) a[k] = sL[k * T];
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int i = 0; i < 3; ++i)                     // + (F dFpi) a1
        acc[i + 3 * j] += T1[i] * a[3 * j] + T1[i + 3] * a[1 + 3 * j] + T1[i + 6] * a[2 + 3 * j];
#pragma unroll
    for (int k = 0; k < 9; ++k) a[k] = sL[(18 + k) * T];
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int i = 0; i < 3; ++i)                     // + a3 dFpi^T
        acc[i + 3 * j] += a[i] * dFpi[j] + a[i + 3] * dFpi[j + 3] + a[i + 6] * dFpi[j + 6];
    const int64_t base = int64_t(9 * p + 27 * o) * N + v;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      planes[base + int64_t(k) * N] = acc[k];
      norm = fma(acc[k], acc[k], norm);
    }
  }
  return norm;
}

template <int NS>
__global__ void __launch_bounds__(TAN_THREADS)
dPdF_kernel(const __grid_constant__ PhaseConst<NS> pc, const __grid_constant__ Fields f, double dt, TangentOut o,
            int64_t first, int64_t count) {
  extern __shared__ double slots[];
  const int64_t li = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (li >= count) return;
  const int64_t v = first + li;
  o.norms[v] = tangent_voxel<NS>(pc, f, v, dt, o.planes, slots + threadIdx.x);
}

// Per block: the sums of the 81 planes over a contiguous voxel range and the extreme norms
// of that range (fixed summation order).
constexpr int TSUM_THREADS = 256, TSUM_BLOCKS = 1184;

__global__ void __launch_bounds__(TSUM_THREADS)
tangent_sum_kernel(const double* __restrict__ planes, const double* __restrict__ norms, int64_t first, int64_t count,
                   int64_t N, TangentOut o) {
  __shared__ double red[TSUM_THREADS / 32];
  __shared__ double rmax[TSUM_THREADS / 32], rmin[TSUM_THREADS / 32];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int64_t per = (count + gridDim.x - 1) / gridDim.x;
  const int64_t b0 = first + int64_t(blockIdx.x) * per;
  const int64_t b1 = b0 + per < first + count ? b0 + per : first + count;
  for (int c = 0; c < 81; ++c) {
    double s = 0.0;
    for (int64_t v = b0 + t; v < b1; v += TSUM_THREADS) s += planes[int64_t(c) * N + v];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if (lane == 0) red[w] = s;
    __syncthreads();
    if (t == 0) {
      double tot = 0.0;
      for (int k = 0; k < TSUM_THREADS / 32; ++k) tot += red[k];
      o.partials[int64_t(blockIdx.x) * 81 + c] = tot;
    }
    __syncthreads();
  }
  double mx = 0.0, mn = 1.7976931348623157e308;
  for (int64_t v = b0 + t; v < b1; v += TSUM_THREADS) {
    mx = fmax(mx, norms[v]);
    mn = fmin(mn, norms[v]);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, off));
    mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, off));
  }
  if (lane == 0) { rmax[w] = mx; rmin[w] = mn; }
  __syncthreads();
  if (t == 0) {
    for (int k = 1; k < TSUM_THREADS / 32; ++k) { mx = fmax(mx, rmax[k]); mn = fmin(mn, rmin[k]); }
    o.nmax[blockIdx.x] = mx;
    o.nmin[blockIdx.x] = mn;
  }
}

// dPdF of the selected max/min voxels -> out[81..161], out[162..242] (column-major)
__global__ void tangent_pick_kernel(const double* __restrict__ planes, int64_t N, const long long* idx, double* out) {
  const int t = threadIdx.x;
  if (t > 1) return;
  double* dst = out + 81 * (1 + t);
  const long long v = idx[t];
  if (v < 0 || v == 0x7fffffffffffffffLL) {
    for (int k = 0; k < 81; ++k) dst[k] = t == 0 ? 0.0 : 1.7976931348623157e308;
    return;
  }
  for (int k = 0; k < 81; ++k) dst[k] = planes[int64_t(k) * N + v];
}

template <int NS>
cudaError_t launch_tangent_pick(const PhaseConst<NS>& pc, const Fields& f, double dt, const long long* idx, double* out,
                                const double* planes, cudaStream_t s) {
  tangent_pick_kernel<<<1, 32, 0, s>>>(planes, f.N, idx, out);
  return cudaGetLastError();
}
template cudaError_t launch_tangent_pick<12>(const PhaseConst<12>&, const Fields&, double, const long long*, double*,
                                             const double*, cudaStream_t);
template cudaError_t launch_tangent_pick<18>(const PhaseConst<18>&, const Fields&, double, const long long*, double*,
                                             const double*, cudaStream_t);
template cudaError_t launch_tangent_pick<24>(const PhaseConst<24>&, const Fields&, double, const long long*, double*,
                                             const double*, cudaStream_t);
template cudaError_t launch_tangent_pick<48>(const PhaseConst<48>&, const Fields&, double, const long long*, double*,
                                             const double*, cudaStream_t);

// number of per-block partials the tangent reduction produces for count voxels
int dPdF_blocks(int64_t count) { return int(std::max<int64_t>(1, std::min<int64_t>(TSUM_BLOCKS, (count + 255) / 256))); }

template <int NS>
cudaError_t launch_dPdF(const PhaseConst<NS>& pc, const Fields& f, double dt, const TangentOut& o, int64_t first,
                        int64_t count, cudaStream_t s, bool with_sums) {
  const size_t smem = size_t(tan_slots<NS>()) * TAN_THREADS * sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(dPdF_kernel<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  const int nb = int((count + TAN_THREADS - 1) / TAN_THREADS);
  dPdF_kernel<NS><<<nb, TAN_THREADS, smem, s>>>(pc, f, dt, o, first, count);
  if (with_sums) tangent_sum_kernel<<<dPdF_blocks(count), TSUM_THREADS, 0, s>>>(o.planes, o.norms, first, count, f.N, o);
  return cudaGetLastError();
}

cudaError_t launch_tangent_sums(const TangentOut& o, int64_t first, int64_t count, int64_t N, cudaStream_t s) {
  tangent_sum_kernel<<<dPdF_blocks(count), TSUM_THREADS, 0, s>>>(o.planes, o.norms, first, count, N, o);
  return cudaGetLastError();
}
template cudaError_t launch_dPdF<12>(const PhaseConst<12>&, const Fields&, double, const TangentOut&, int64_t, int64_t,
                                     cudaStream_t, bool);
template cudaError_t launch_dPdF<18>(const PhaseConst<18>&, const Fields&, double, const TangentOut&, int64_t, int64_t,
                                     cudaStream_t, bool);
template cudaError_t launch_dPdF<24>(const PhaseConst<24>&, const Fields&, double, const TangentOut&, int64_t, int64_t,
                                     cudaStream_t, bool);
template cudaError_t launch_dPdF<48>(const PhaseConst<48>&, const Fields&, double, const TangentOut&, int64_t, int64_t,
                                     cudaStream_t, bool);

// Sums the per-block partials (C_volAvg) and finds the extreme Frobenius norms.
// dPdF_max / dPdF_min (grid_utilities.f90:171-197) are the voxels of maximal /
// minimal norm in voxel order; norms that agree to 1e-12 relative count as equal
// and the first such voxel is taken, so that the pick does not depend on rounding
// (at F = I every grain's tangent has the same norm).
// Reduction of the per-block tangent partials in two stages: FIN_BLOCKS blocks each sum a
// contiguous range of parts (81 sums, max and min of the norms) into a second-level buffer;
// one block then combines those.
constexpr int FIN_BLOCKS = 592, FIN_THREADS = 243;   // 243 = 3 lanes per component

__global__ void __launch_bounds__(FIN_THREADS) tangent_reduce_kernel(TangentOut o, int nparts, double* l2) {
  __shared__ double acc[FIN_THREADS];
  __shared__ double ext[2][FIN_THREADS];
  const int t = threadIdx.x, comp = t % 81, lane = t / 81;
  const int per = (nparts + gridDim.x - 1) / gridDim.x;
  const int b0 = blockIdx.x * per, b1 = min(nparts, b0 + per);
  double s = 0.0, mx = 0.0, mn = 1.7976931348623157e308;
  for (int b = b0 + lane; b < b1; b += 3) s += o.partials[int64_t(b) * 81 + comp];
  for (int b = b0 + t; b < b1; b += FIN_THREADS) {
    mx = fmax(mx, o.nmax[b]);
    mn = fmin(mn, o.nmin[b]);
  }
  acc[t] = s;
  ext[0][t] = mx;
  ext[1][t] = mn;
  __syncthreads();
  if (t < 81) l2[int64_t(blockIdx.x) * 83 + t] = acc[t] + acc[t + 81] + acc[t + 162];
  if (t == 0) {
    for (int i = 1; i < FIN_THREADS; ++i) {
      mx = fmax(mx, ext[0][i]);
      mn = fmin(mn, ext[1][i]);
    }
    l2[int64_t(blockIdx.x) * 83 + 81] = mx;
    l2[int64_t(blockIdx.x) * 83 + 82] = mn;
  }
}

__global__ void tangent_finalize_kernel(const double* __restrict__ l2, int nblocks, double wgt, double* out,
                                        long long* idx) {
  const int t = threadIdx.x;
  if (t < 81) {
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += l2[int64_t(b) * 83 + t];
    out[t] = s * wgt;
  }
  if (t == 0) {
    double bmax = 0.0, bmin = 1.7976931348623157e308;
    for (int b = 0; b < nblocks; ++b) {
      bmax = fmax(bmax, l2[int64_t(b) * 83 + 81]);
      bmin = fmin(bmin, l2[int64_t(b) * 83 + 82]);
    }
    out[243] = bmax;
    out[244] = bmin;
    idx[0] = 0x7fffffffffffffffLL;
    idx[1] = 0x7fffffffffffffffLL;
  }
}
__global__ void tangent_first_kernel(const double* __restrict__ norms, int64_t first, int64_t count,
                                     const double* __restrict__ ext, long long* idx) {
  const double M = ext[243], m = ext[244];
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t v = first + i;
    const double s = norms[v];
    if (s >= M * (1.0 - 1.0e-12) && s > 0.0) atomicMin(&idx[0], (long long)v);
    if (s <= m * (1.0 + 1.0e-12)) atomicMin(&idx[1], (long long)v);
  }
}
int tangent_reduce_doubles() { return FIN_BLOCKS * 83; }
cudaError_t launch_tangent_finalize(const TangentOut& o, int nparts, double wgt, double* out, long long* idx,
                                    int64_t first, int64_t count, cudaStream_t s) {
  const int nr = std::max(1, std::min(FIN_BLOCKS, nparts));
  tangent_reduce_kernel<<<nr, FIN_THREADS, 0, s>>>(o, nparts, o.l2);
  tangent_finalize_kernel<<<1, 96, 0, s>>>(o.l2, nr, wgt, out, idx);
  const int nb = int(std::min<int64_t>((count + 255) / 256, 4096));
  tangent_first_kernel<<<nb, 256, 0, s>>>(o.norms, first, count, out, idx);
  return cudaGetLastError();
}

}  // namespace dmk
