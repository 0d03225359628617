// Kernels of the spectral polarization scheme (grid_mech_spectral_polarization.f90) and its
// curl criterion (utilities_curlRMS, spectral_utilities.f90:695-757).  Fields are planes
// (component c of voxel v at c * N + v, column-major 3x3 components); fourth-order
// constants are column-major, index i + 3j + 9k + 27l.
#include "constitutive.cuh"
#include "kernels.cuh"

namespace dmk {

namespace {

// math_mul3333xx33 (math.f90:386-399): out(i,j) = sum_kl A(i,j,k,l) B(k,l)
__device__ __forceinline__ void ddot4(const double* __restrict__ A, const double B[9], double out[9]) {
#pragma unroll
  for (int ij = 0; ij < 9; ++ij) {
    double s = 0.0;
#pragma unroll
    for (int kl = 0; kl < 9; ++kl) s = fma(A[ij + 9 * kl], B[kl], s);
    out[ij] = s;
  }
}

// matmul of column-major 3x3
__device__ __forceinline__ void pol_mm33(const double A[9], const double B[9], double out[9]) {
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 3; ++i) out[i + 3 * j] = A[i] * B[3 * j] + A[i + 3] * B[1 + 3 * j] + A[i + 6] * B[2 + 3 * j];
}

__device__ __forceinline__ void load9(const double* __restrict__ p, int64_t N, int64_t v, double x[9]) {
#pragma unroll
  for (int k = 0; k < 9; ++k) x[k] = p[k * N + v];
}
__device__ __forceinline__ void store9(double* __restrict__ p, int64_t N, int64_t v, const double x[9]) {
#pragma unroll
  for (int k = 0; k < 9; ++k) p[k * N + v] = x[k];
}

// F . (C : (F_tau - F - I)), the polarization term shared by both residual parts
__device__ __forceinline__ void polarization_term(const double* __restrict__ C, const double F[9], const double Ft[9],
                                                  double out[9]) {
  double A[9], t[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) A[k] = Ft[k] - F[k] - ((k % 4 == 0) ? 1.0 : 0.0);
  ddot4(C, A, t);
  pol_mm33(F, t, out);
}

}  // namespace

// r_F_tau before the convolution (form_residual, :585-590):
// beta C:(F - I) - alpha F.(C:(F_tau - F - I))
__global__ void pol_pre_kernel(const double* __restrict__ F, const double* __restrict__ Ftau, int64_t N,
                               const __grid_constant__ PolConst pc, double* __restrict__ out) {
  const int64_t v = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= N) return;
  double f[9], ft[9], t1[9], t2[9], d[9];
  load9(F, N, v, f);
  load9(Ftau, N, v, ft);
#pragma unroll
  for (int k = 0; k < 9; ++k) d[k] = f[k] - ((k % 4 == 0) ? 1.0 : 0.0);
  ddot4(pc.C, d, t1);
  polarization_term(pc.C, f, ft, t2);
#pragma unroll
  for (int k = 0; k < 9; ++k) out[k * N + v] = pc.beta * t1[k] - pc.alpha * t2[k];
}

// r_F_tau = beta F - Gamma(...) from the convolution result G and the deformation gradient of
// the constitutive evaluation, F - r_F_tau / beta (:591, :596-604).  G may be Feval itself (each
// element is read before it is overwritten by the same thread).
__global__ void pol_tau_kernel(const double* __restrict__ F, const double* G, double* __restrict__ rtau, int64_t N,
                               double beta, double* Feval) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= 9 * N) return;
  const double f = F[i];
  const double r = beta * f - G[i];
  rtau[i] = r;
  Feval[i] = f - r / beta;
}

// r_F = invSym3333(dPdF + C) : (P - F.(C:(F_tau - F - I))) + r_F_tau (:606-617).
// invSym3333 (math.f90:511-532) inverts the Mandel 6x6 M(r,q) = A(p_r, p_q) w_r w_q
// (math_sym3333to66: pairs 11,22,33,23,13,12, w = 1 for normal and sqrt(2) for shear pairs)
// and expands it with minor symmetry (math_66toSym3333), so the contraction with a 3x3 B is
// out(p_r) = y_r / w_r with M y = z, z_q = (B(k,l) [+ B(l,k) for k != l]) / w_q; out symmetric.
// The 6x6 system is solved by Householder QR with compile-time indices (registers only); a
// singular matrix gives NaN, as the reference's inversion error would stop.  Only the 36 dPdF
// planes of the Mandel pairs are read.
__global__ void __launch_bounds__(128)
pol_rF_kernel(const double* __restrict__ F, const double* __restrict__ Ftau, const double* __restrict__ P,
              const double* __restrict__ dPdF, const double* __restrict__ rtau, int64_t N,
              const __grid_constant__ PolConst pc, double* __restrict__ rF) {
  const int64_t v = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= N) return;
  constexpr int pi[6] = {0, 1, 2, 1, 0, 0}, pj[6] = {0, 1, 2, 2, 2, 1};
  const double SQ2 = 1.4142135623730951;
  double f[9], ft[9], b[9];
  load9(F, N, v, f);
  load9(Ftau, N, v, ft);
  polarization_term(pc.C, f, ft, b);
#pragma unroll
  for (int k = 0; k < 9; ++k) b[k] = P[k * N + v] - b[k];
  double M[36], z[6];
#pragma unroll
  for (int r = 0; r < 6; ++r)
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const int c = pi[r] + 3 * pj[r] + 9 * pi[q] + 27 * pj[q];
      M[6 * r + q] = (dPdF[int64_t(c) * N + v] + pc.C[c]) * (r < 3 ? 1.0 : SQ2) * (q < 3 ? 1.0 : SQ2);
    }
#pragma unroll
  for (int q = 0; q < 6; ++q)
    z[q] = q < 3 ? b[pi[q] + 3 * pj[q]] : (b[pi[q] + 3 * pj[q]] + b[pj[q] + 3 * pi[q]]) / SQ2;
  if (qr_solve<6>(M, z))
#pragma unroll
    for (int q = 0; q < 6; ++q) z[q] = __longlong_as_double(0x7ff8000000000000LL);
  double out[9];
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    const double y = r < 3 ? z[r] : z[r] / SQ2;
    out[pi[r] + 3 * pj[r]] = y;
    out[pj[r] + 3 * pi[r]] = y;
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) rF[k * N + v] = out[k] + rtau[k * N + v];
}

// utilities_curlRMS partial sums over the stored Fourier points of F (spectrum planes c =
// i + 3j).  Interior kx count twice; the planes kx = 0 and kx = n0/2+1-1 (stored index
// cells1Red) count the last of the nine curl expressions (l = 3, third column) nine times,
// as the reference's scalar assignment to the whole array does.
__global__ void __launch_bounds__(SPEC_THREADS)
curl_kernel(const double2* __restrict__ S, int64_t plane, int n0, int n1, int n2, double L0, double L1, double L2,
            double rg0, double rg1, double rg2, int derivative, double* __restrict__ partials) {
  __shared__ double red[SPEC_THREADS / 32];
  const int red0 = n0 / 2 + 1;
  const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  double sum = 0.0;
  if (idx < plane) {
    const int kx = int(idx % red0);
    const int64_t rest = idx / red0;
    const int ky = int(rest % n1);
    const int kz = int(rest / n1);
    const int sy = ky > n1 / 2 ? ky - n1 : ky;
    const int sz = kz > n2 / 2 ? kz - n2 : kz;
    // xi1st * rescaledGeom = wr + i wi (continuous and central difference: wr = 0)
    double wr[3] = {0.0, 0.0, 0.0}, wi[3];
    if (derivative == 2) {
      const int ks[3] = {kx, sy, sz};
      const int nn[3] = {n0, n1, n2};
      const double LL[3] = {L0, L1, L2};
      freq_fwbw(ks, nn, LL, wr, wi);
      wr[0] *= rg0; wr[1] *= rg1; wr[2] *= rg2;
      wi[0] *= rg0; wi[1] *= rg1; wi[2] *= rg2;
    } else {
      wi[0] = freq_derivative(kx, n0, L0, derivative, true) * rg0;
      wi[1] = freq_derivative(sy, n1, L1, derivative, true) * rg1;
      wi[2] = freq_derivative(sz, n2, L2, derivative, true) * rg2;
    }
    // a w[d1] - b w[d2]; with wr = 0: (x + i y) (i w) = -y w + i x w
    auto term = [&](int c1, int d1, int c2, int d2, double& re, double& im) {
      const double2 a = S[c1 * plane + idx], b = S[c2 * plane + idx];
      if (derivative == 2) {
        re = (a.x * wr[d1] - a.y * wi[d1]) - (b.x * wr[d2] - b.y * wi[d2]);
        im = (a.x * wi[d1] + a.y * wr[d1]) - (b.x * wi[d2] + b.y * wr[d2]);
      } else {
        re = -a.y * wi[d1] + b.y * wi[d2];
        im = a.x * wi[d1] - b.x * wi[d2];
      }
    };
    if (kx >= 1 && kx < red0 - 1) {
      double s = 0.0;
#pragma unroll
      for (int l = 0; l < 3; ++l) {
        double re, im;
        term(l + 6, 1, l + 3, 2, re, im);   // T(l,3) xi2 - T(l,2) xi3
        s += re * re + im * im;
        term(l + 0, 2, l + 6, 0, re, im);   // T(l,1) xi3 - T(l,3) xi1
        s += re * re + im * im;
        term(l + 3, 0, l + 0, 1, re, im);   // T(l,2) xi1 - T(l,1) xi2
        s += re * re + im * im;
      }
      sum = 2.0 * s;
    } else {
      double re, im;
      term(2 + 3, 0, 2 + 0, 1, re, im);     // T(3,2) xi1 - T(3,1) xi2
      sum = 9.0 * (re * re + im * im);
      // with a single stored plane (n0 == 1) it is both the first and the last one
      if (red0 == 1) sum *= 2.0;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < SPEC_THREADS / 32; ++w) s += red[w];
    partials[blockIdx.x] = s;
  }
}

// forward of F_tau (grid_mech_spectral_polarization.f90:366-396) after F has been forwarded:
// unless cut back, F_tauDot = calculateRate(guess, F_tau_lastinc, F_tau) and F_tau_lastinc = F_tau;
// then with guess F_tau = F_tau_lastinc + F_tauDot dt (no average correction), otherwise
// F_tau = F + I + S_scale : (1/2 F_l (C_scale : (F_l^T F_l - I))) with F_l = F_tau - F.
__global__ void pol_forward_tau_kernel(const double* __restrict__ F, double* __restrict__ Ftau,
                                       double* __restrict__ Flast, double* __restrict__ Fdot, int64_t N, int cutBack,
                                       int guess, double dt, double dt_old, const double* __restrict__ avRate,
                                       const __grid_constant__ PolConst pc) {
  const int64_t v = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= N) return;
  double ft[9], fl[9], fd[9];
  load9(Ftau, N, v, ft);
  load9(Flast, N, v, fl);
  load9(Fdot, N, v, fd);
  if (!cutBack) {
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      fd[k] = guess ? (ft[k] - fl[k]) / dt_old : avRate[k];
      fl[k] = ft[k];
    }
    store9(Fdot, N, v, fd);
    store9(Flast, N, v, fl);
  }
  if (guess) {
#pragma unroll
    for (int k = 0; k < 9; ++k) ft[k] = fl[k] + fd[k] * dt;
  } else {
    double f[9], Fl[9], Ft[9], E[9], t[9], u[9], w[9];
    load9(F, N, v, f);
#pragma unroll
    for (int k = 0; k < 9; ++k) Fl[k] = ft[k] - f[k];
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int i = 0; i < 3; ++i) Ft[i + 3 * j] = Fl[j + 3 * i];
    pol_mm33(Ft, Fl, E);
#pragma unroll
    for (int k = 0; k < 9; ++k) E[k] -= (k % 4 == 0) ? 1.0 : 0.0;
    ddot4(pc.C, E, t);
    pol_mm33(Fl, t, u);
#pragma unroll
    for (int k = 0; k < 9; ++k) u[k] *= 0.5;
    ddot4(pc.S, u, w);
#pragma unroll
    for (int k = 0; k < 9; ++k) ft[k] = ((k % 4 == 0) ? 1.0 : 0.0) + w[k] + f[k];
  }
  store9(Ftau, N, v, ft);
}

__global__ void sub_kernel(double* __restrict__ X, const double* __restrict__ r, int64_t n) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    X[i] -= r[i];
}

cudaError_t launch_pol_pre(const double* F, const double* Ftau, int64_t N, const PolConst& pc, double* out,
                           cudaStream_t s) {
  pol_pre_kernel<<<unsigned((N + 127) / 128), 128, 0, s>>>(F, Ftau, N, pc, out);
  return cudaGetLastError();
}
cudaError_t launch_pol_tau(const double* F, const double* G, double* rtau, int64_t N, double beta, double* Feval,
                           cudaStream_t s) {
  pol_tau_kernel<<<unsigned((9 * N + 255) / 256), 256, 0, s>>>(F, G, rtau, N, beta, Feval);
  return cudaGetLastError();
}
cudaError_t launch_pol_rF(const double* F, const double* Ftau, const double* P, const double* dPdF, const double* rtau,
                          int64_t N, const PolConst& pc, double* rF, cudaStream_t s) {
  pol_rF_kernel<<<unsigned((N + 127) / 128), 128, 0, s>>>(F, Ftau, P, dPdF, rtau, N, pc, rF);
  return cudaGetLastError();
}
cudaError_t launch_curl(const double* spec, int n0, int n1, int n2, const double L[3], const double rg[3],
                        int derivative, double* partials, cudaStream_t s) {
  const int64_t plane = int64_t(n0 / 2 + 1) * n1 * n2;
  curl_kernel<<<unsigned(gamma_div_blocks(n0, n1, n2)), SPEC_THREADS, 0, s>>>(
      reinterpret_cast<const double2*>(spec), plane, n0, n1, n2, L[0], L[1], L[2], rg[0], rg[1], rg[2], derivative,
      partials);
  return cudaGetLastError();
}
cudaError_t launch_pol_forward_tau(const double* F, double* Ftau, double* Flast, double* Fdot, int64_t N, int cutBack,
                                   int guess, double dt, double dt_old, const double* avRate, const PolConst& pc,
                                   cudaStream_t s) {
  pol_forward_tau_kernel<<<unsigned((N + 127) / 128), 128, 0, s>>>(F, Ftau, Flast, Fdot, N, cutBack, guess, dt, dt_old,
                                                                   avRate, pc);
  return cudaGetLastError();
}
cudaError_t launch_sub(double* X, const double* r, int64_t n, int nsm, cudaStream_t s) {
  sub_kernel<<<nsm * 8, 256, 0, s>>>(X, r, n);
  return cudaGetLastError();
}

}  // namespace dmk
