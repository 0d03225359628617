// Consistent tangent dP/dF per voxel (phase_mechanical_dPdF, phase_mechanical.f90:1121-1242)
// with Fi = I, Li = 0 (dFi/dS = 0), fused with the reductions that consume it in
// utilities_constitutiveResponse (grid_utilities.f90:171-202): the volume sum
// (C_volAvg) and the voxels of maximal and minimal Frobenius norm (C_minMaxAvg).
//
// The tangent is only consumed by those two averages, which the solver reads at
// the start of the next increment (masked compliance) or for the Gamma reference
// stiffness; the host therefore evaluates it once per converged increment from the
// stored converged state instead of inside every residual evaluation.  The values
// equal those of the last residual evaluation because they depend only on the
// stored F, Fe, Fp, Fp0, S and state.
//
// 3x3x3x3 tensors are held as 9x9 matrices T[(3i+j)*9 + 3k+l] (math_3333to99 order),
// so every double contraction is a 9x9 matrix product.
#include "kernels.cuh"
#include "constitutive.cuh"

#include <algorithm>

namespace dmk {

__device__ __forceinline__ void mm99(const double* A, const double* B, double* C) {
  for (int r = 0; r < 9; ++r)
    for (int c = 0; c < 9; ++c) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 9; ++k) s = fma(A[r * 9 + k], B[k * 9 + c], s);
      C[r * 9 + c] = s;
    }
}

// in-place inverse of a 9x9 matrix by Gauss-Jordan with partial pivoting; true on error
__device__ bool inv99(double* A, double* Ai) {
  for (int i = 0; i < 81; ++i) Ai[i] = 0.0;
  for (int i = 0; i < 9; ++i) Ai[i * 9 + i] = 1.0;
  for (int j = 0; j < 9; ++j) {
    int p = j;
    double amax = fabs(A[j * 9 + j]);
    for (int i = j + 1; i < 9; ++i)
      if (fabs(A[i * 9 + j]) > amax) { amax = fabs(A[i * 9 + j]); p = i; }
    if (amax == 0.0) return true;
    if (p != j)
      for (int k = 0; k < 9; ++k) {
        double t = A[j * 9 + k]; A[j * 9 + k] = A[p * 9 + k]; A[p * 9 + k] = t;
        t = Ai[j * 9 + k]; Ai[j * 9 + k] = Ai[p * 9 + k]; Ai[p * 9 + k] = t;
      }
    const double rp = 1.0 / A[j * 9 + j];
    for (int k = 0; k < 9; ++k) { A[j * 9 + k] *= rp; Ai[j * 9 + k] *= rp; }
    for (int i = 0; i < 9; ++i) {
      if (i == j) continue;
      const double l = A[i * 9 + j];
      if (l == 0.0) continue;
      for (int k = 0; k < 9; ++k) {
        A[i * 9 + k] = fma(-l, A[j * 9 + k], A[i * 9 + k]);
        Ai[i * 9 + k] = fma(-l, Ai[j * 9 + k], Ai[i * 9 + k]);
      }
    }
  }
  return false;
}

template <int NS>
__device__ void tangent_point(const PhaseConst<NS>& pc, const Fields& f, int64_t v, double dt, double* out /* 81, 99 order */) {
  const int64_t N = f.N;
  double F[9], Fe[9], Fp[9], Fp0[9], s6[6], xi[NS];
  for (int k = 0; k < 9; ++k) {
    F[k] = f.F[k * N + v]; Fe[k] = f.Fe[k * N + v]; Fp[k] = f.Fp[k * N + v]; Fp0[k] = f.Fp0[k * N + v];
  }
  for (int k = 0; k < 6; ++k) s6[k] = f.S[k * N + v];
  for (int s = 0; s < NS; ++s) xi[s] = f.state[s * N + v];
  const double Sm[9] = {s6[0], s6[5], s6[4], s6[5], s6[1], s6[3], s6[4], s6[3], s6[2]};

  double dSdFe[81], dLpdS[81], T1[81], T2[81], T3[81];
  // dSdFe(i,j,k,l) = sum_m Fe(k,m) C(i,j,m,l)
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k)
        for (int l = 0; l < 3; ++l) {
          double s = 0.0;
          for (int m = 0; m < 3; ++m) s = fma(Fe[k + 3 * m], pc.C[i + 3 * j + 9 * m + 27 * l], s);
          dSdFe[(3 * i + j) * 9 + 3 * k + l] = s;
        }
  // dLp/dS = dLp/dMp (Fi = I) = sum_s dgamma_s P_s (x) P_nS_s
  for (int r = 0; r < 81; ++r) dLpdS[r] = 0.0;
  for (int s = 0; s < NS; ++s) {
    const double tp = dot6(s6, pc.p6[0][s]), tn = dot6(s6, pc.p6[1][s]);
    const bool pos = tp > tn;
    const double tmax = pos ? tp : tn;
    const double g = (pos ? pc.dg0[s] : -pc.dg0[s]) * powr(tmax / xi[s], pc.n[s], pc.n_int[s]);
    const double dg = fabs(g) > TINY10 ? g * pc.n[s] / tmax : 0.0;
    if (dg == 0.0) continue;
    const double* PnS = pc.PnS[g > 0.0 ? 0 : 1][s];
    for (int k = 0; k < 3; ++k)
      for (int l = 0; l < 3; ++l) {
        const double a = dg * pc.P[s][k + 3 * l];
        for (int m = 0; m < 3; ++m)
          for (int n = 0; n < 3; ++n) dLpdS[(3 * k + l) * 9 + 3 * m + n] = fma(a, PnS[m + 3 * n], dLpdS[(3 * k + l) * 9 + 3 * m + n]);
      }
  }
  double invFp[9], invFp0[9];
  inv33(Fp, invFp);
  inv33(Fp0, invFp0);
  double t2[9];
  mm33(F, invFp0, t2);                     // temp_33_2 = F invSubFp0
  // rhs(p,o,k,l) = sum_m dSdFe(p,o,k,m) invFp(l,m)          -> T1
  for (int po = 0; po < 9; ++po)
    for (int k = 0; k < 3; ++k)
      for (int l = 0; l < 3; ++l) {
        double s = 0.0;
        for (int m = 0; m < 3; ++m) s = fma(dSdFe[po * 9 + 3 * k + m], invFp[l + 3 * m], s);
        T1[po * 9 + 3 * k + l] = s;
      }
  // temp(k,l,p,o) = sum_m t2(k,m) dLpdS(m,l,p,o)              -> T2
  for (int k = 0; k < 3; ++k)
    for (int l = 0; l < 3; ++l)
      for (int po = 0; po < 9; ++po) {
        double s = 0.0;
        for (int m = 0; m < 3; ++m) s = fma(t2[k + 3 * m], dLpdS[(3 * m + l) * 9 + po], s);
        T2[(3 * k + l) * 9 + po] = s;
      }
  // lhs = dSdFe : temp * dt ;  I + lhs                           -> T3
  mm99(dSdFe, T2, T3);
  for (int r = 0; r < 81; ++r) T3[r] *= dt;
  for (int r = 0; r < 9; ++r) T3[r * 9 + r] += 1.0;
  double X[81];
  double* dSdF = T2;
  if (inv99(T3, X)) {
    for (int r = 0; r < 81; ++r) dSdF[r] = T1[r];
  } else {
    mm99(X, T1, dSdF);
  }
  // dFpinvdF(k,l,p,o) = -dt sum_m invFp0(k,m) (dLpdS : dSdF)(m,l,p,o)
  mm99(dLpdS, dSdF, X);
  double* dFpi = T3;
  for (int k = 0; k < 3; ++k)
    for (int l = 0; l < 3; ++l)
      for (int po = 0; po < 9; ++po) {
        double s = 0.0;
        for (int m = 0; m < 3; ++m) s = fma(invFp0[k + 3 * m], X[(3 * m + l) * 9 + po], s);
        dFpi[(3 * k + l) * 9 + po] = -s * dt;
      }
  // assemble dPdF
  double a1[9], a2[9], a3[9], d[9];
  mmt33(Sm, invFp, a1);                 // temp_33_1 = S invFp^T
  mm33(F, invFp, a2);                   // temp_33_2 = F invFp
  mm33(a2, Sm, a3);                     // temp_33_3 = F invFp S
  mm33(invFp, a1, d);                   // (invFp temp_33_1), transposed into dPdF(p,:,p,:)
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int p = 0; p < 3; ++p)
        for (int o = 0; o < 3; ++o) {
          const int po = 3 * p + o;
          double s = (i == p) ? d[o + 3 * j] : 0.0;
          // F dFpinvdF(:,:,p,o) temp_33_1
          for (int m = 0; m < 3; ++m)
            for (int n = 0; n < 3; ++n) s = fma(F[i + 3 * m] * dFpi[(3 * m + n) * 9 + po], a1[n + 3 * j], s);
          // temp_33_2 dSdF(:,:,p,o) invFp^T
          for (int m = 0; m < 3; ++m)
            for (int n = 0; n < 3; ++n) s = fma(a2[i + 3 * m] * dSdF[(3 * m + n) * 9 + po], invFp[j + 3 * n], s);
          // temp_33_3 dFpinvdF(:,:,p,o)^T
          for (int m = 0; m < 3; ++m) s = fma(a3[i + 3 * m], dFpi[(3 * j + m) * 9 + po], s);
          out[(3 * i + j) * 9 + po] = s;
        }
}

constexpr int TAN_THREADS = 64;

template <int NS>
__global__ void __launch_bounds__(TAN_THREADS)
dPdF_kernel(const __grid_constant__ PhaseConst<NS> pc, const __grid_constant__ Fields f, double dt, TangentOut o,
            int64_t first, int64_t count) {
  __shared__ double buf[81 * TAN_THREADS];          // deterministic in-block summation
  __shared__ double smax[TAN_THREADS], smin[TAN_THREADS];
  __shared__ long long sidx[TAN_THREADS];
  const int t = threadIdx.x;
  const int64_t li = int64_t(blockIdx.x) * blockDim.x + t;
  double nrm = 0.0;
  long long idx = -1;
  if (li < count) {
    const int64_t v = first + li;
    double T[81];
    tangent_point<NS>(pc, f, v, dt, T);
    // Frobenius norm^2 in column-major order, as sum(dPdF**2)
    double s = 0.0;
    for (int l = 0; l < 3; ++l)
      for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 3; ++j)
          for (int i = 0; i < 3; ++i) {
            const double x = T[(3 * i + j) * 9 + 3 * k + l];
            s = fma(x, x, s);
          }
    nrm = s;
    idx = v;
    o.norms[v] = s;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 3; ++k)
          for (int l = 0; l < 3; ++l) {
            const double x = T[(3 * i + j) * 9 + 3 * k + l];
            buf[(i + 3 * j + 9 * k + 27 * l) * TAN_THREADS + t] = x;
            if (o.per_voxel) o.per_voxel[v * 81 + i + 3 * j + 9 * k + 27 * l] = x;
          }
  } else {
    for (int k = 0; k < 81; ++k) buf[k * TAN_THREADS + t] = 0.0;
  }
  smax[t] = nrm;
  smin[t] = nrm;
  sidx[t] = idx;
  __syncthreads();
  for (int k = t; k < 81; k += TAN_THREADS) {
    double s = 0.0;
    for (int w = 0; w < TAN_THREADS; ++w) s += buf[k * TAN_THREADS + w];
    o.partials[int64_t(blockIdx.x) * 81 + k] = s;
  }
  if (t == 0) {
    double bmax = 0.0, bmin = 1.7976931348623157e308;
    for (int w = 0; w < TAN_THREADS; ++w) {
      if (sidx[w] < 0) continue;
      bmax = fmax(bmax, smax[w]);
      bmin = fmin(bmin, smin[w]);
    }
    o.nmax[blockIdx.x] = bmax;
    o.nmin[blockIdx.x] = bmin;
  }
}

// dPdF of the selected max/min voxels -> out[81..161], out[162..242] (column-major)
template <int NS>
__global__ void tangent_pick_kernel(const __grid_constant__ PhaseConst<NS> pc, const __grid_constant__ Fields f, double dt,
                                    const long long* idx, double* out) {
  const int t = threadIdx.x;
  if (t > 1) return;
  double* dst = out + 81 * (1 + t);
  const long long v = idx[t];
  if (v < 0 || v == 0x7fffffffffffffffLL) {
    for (int k = 0; k < 81; ++k) dst[k] = t == 0 ? 0.0 : 1.7976931348623157e308;
    return;
  }
  double T[81];
  tangent_point<NS>(pc, f, v, dt, T);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k)
        for (int l = 0; l < 3; ++l) dst[i + 3 * j + 9 * k + 27 * l] = T[(3 * i + j) * 9 + 3 * k + l];
}

template <int NS>
cudaError_t launch_tangent_pick(const PhaseConst<NS>& pc, const Fields& f, double dt, const long long* idx, double* out,
                                cudaStream_t s) {
  tangent_pick_kernel<NS><<<1, 32, 0, s>>>(pc, f, dt, idx, out);
  return cudaGetLastError();
}
template cudaError_t launch_tangent_pick<12>(const PhaseConst<12>&, const Fields&, double, const long long*, double*, cudaStream_t);
template cudaError_t launch_tangent_pick<18>(const PhaseConst<18>&, const Fields&, double, const long long*, double*, cudaStream_t);
template cudaError_t launch_tangent_pick<24>(const PhaseConst<24>&, const Fields&, double, const long long*, double*, cudaStream_t);

int dPdF_blocks(int64_t count) { return int((count + TAN_THREADS - 1) / TAN_THREADS); }

template <int NS>
cudaError_t launch_dPdF(const PhaseConst<NS>& pc, const Fields& f, double dt, const TangentOut& o, int64_t first,
                        int64_t count, cudaStream_t s) {
  dPdF_kernel<NS><<<dPdF_blocks(count), TAN_THREADS, 0, s>>>(pc, f, dt, o, first, count);
  return cudaGetLastError();
}
template cudaError_t launch_dPdF<12>(const PhaseConst<12>&, const Fields&, double, const TangentOut&, int64_t, int64_t, cudaStream_t);
template cudaError_t launch_dPdF<18>(const PhaseConst<18>&, const Fields&, double, const TangentOut&, int64_t, int64_t, cudaStream_t);
template cudaError_t launch_dPdF<24>(const PhaseConst<24>&, const Fields&, double, const TangentOut&, int64_t, int64_t, cudaStream_t);

// Sums the per-block partials (C_volAvg) and finds the extreme Frobenius norms.
// dPdF_max / dPdF_min (grid_utilities.f90:171-197) are the voxels of maximal /
// minimal norm in voxel order; norms that agree to 1e-12 relative count as equal
// and the first such voxel is taken, so that the pick does not depend on rounding
// (at F = I every grain's tangent has the same norm).
__global__ void tangent_finalize_kernel(TangentOut o, int nparts, double wgt, double* out, long long* idx) {
  const int t = threadIdx.x;
  if (t < 81) {
    double s = 0.0;
    for (int b = 0; b < nparts; ++b) s += o.partials[int64_t(b) * 81 + t];
    out[t] = s * wgt;
  }
  if (t == 0) {
    double bmax = 0.0, bmin = 1.7976931348623157e308;
    for (int b = 0; b < nparts; ++b) {
      bmax = fmax(bmax, o.nmax[b]);
      bmin = fmin(bmin, o.nmin[b]);
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
cudaError_t launch_tangent_finalize(const TangentOut& o, int nparts, double wgt, double* out, long long* idx,
                                    int64_t first, int64_t count, cudaStream_t s) {
  tangent_finalize_kernel<<<1, 96, 0, s>>>(o, nparts, wgt, out, idx);
  const int nb = int(std::min<int64_t>((count + 255) / 256, 4096));
  tangent_first_kernel<<<nb, 256, 0, s>>>(o.norms, first, count, out, idx);
  return cudaGetLastError();
}

}  // namespace dmk
