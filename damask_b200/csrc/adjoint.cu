// Kernels of the hand-written adjoint of an increment (see adjoint.cuh for the local model).
//
//  adj_jacobian_kernel  per voxel: the total derivative D = dz/dx of the converged local update
//                       (outputs P, Fp, xi; inputs F, Fp0, xi0, theta) by the implicit-function
//                       theorem: dual-number columns of dG/dy, dG/dx, dZ/dy, dZ/dx, an LU solve with
//                       partial pivoting of dG/dy, then D = dZ/dx - dZ/dy (dG/dy)^-1 dG/dx
//  adj_vjp_kernel       per voxel: the cotangent of the inputs, x_bar = D^T z_bar, for a stress
//                       cotangent (the loss's, minus the adjoint field) and the state cotangent
//  adj_sigma_kernel     per voxel: sigma = K^T Lambda - G with K = dP/dF (the rows of D for P and its
//                       columns for F), the "stress" of the transposed equilibrium problem
//  adj_mdot / adj_maxpy / adj_scale: inner products and linear combinations of the Krylov basis
#include "adjoint.cuh"
#include "kernels.cuh"

#include <vector>

namespace dmk {

namespace {

// Strided view of one voxel's entries: element e at p[e * s].
struct SView {
  double* p;
  int64_t s;
  DMK_HD double& operator[](int64_t e) const { return p[e * s]; }
};
struct CView {
  const double* p;
  int64_t s;
  DMK_HD double operator[](int64_t e) const { return p[e * s]; }
};

// The local Jacobian of one voxel.  pt: the linearization point (27 + 2 NS entries: F, Fp0, xi0,
// Lp, xi); ws: workspace of adj_ws_size(NS, nf) entries; D: nz x nx entries, row-major (output
// r, input c at D[r * nx + c]).  Returns 1 if dG/dy is singular (D is then left unset).
template <int NS>
DMK_HD int local_jacobian(const PhaseConst<NS>& pc, const double* h, double dt, CView pt, SView ws, SView D) {
  const int nf = pc.nf;
  const int ny = adj_ny(NS), nx = adj_nx(NS, nf), nz = adj_nz(NS);
  const int oJ = 0, oX = ny * ny, oZy = oX + ny * nx, oZx = oZy + nz * ny;
  Dual y[9 + NS], x[18 + NS + 4 * ADJ_MAX_FAMILIES], G[9 + NS], Z[18 + NS];
  for (int j = 0; j < ny + nx; ++j) {
    for (int k = 0; k < 9; ++k) y[k] = dual(pt[18 + NS + k]);
    for (int s = 0; s < NS; ++s) y[9 + s] = dual(pt[27 + NS + s]);
    for (int k = 0; k < 18 + NS; ++k) x[k] = dual(pt[k]);
    for (int p = 0; p < 4; ++p)
      for (int f = 0; f < nf; ++f) x[18 + NS + p * nf + f] = dual(pc.th[p][f]);
    if (j < ny) y[j].d = 1.0;
    else x[j - ny].d = 1.0;
    local_model<NS, Dual>(pc, h, dt, y, x, G, Z);
    if (j < ny) {
      for (int r = 0; r < ny; ++r) ws[oJ + r * ny + j] = G[r].d;
      for (int r = 0; r < nz; ++r) ws[oZy + r * ny + j] = Z[r].d;
    } else {
      for (int r = 0; r < ny; ++r) ws[oX + r * nx + (j - ny)] = G[r].d;
      for (int r = 0; r < nz; ++r) ws[oZx + r * nx + (j - ny)] = Z[r].d;
    }
  }
  // LU with partial pivoting of J = dG/dy, applied to X = dG/dx on the way
  for (int k = 0; k < ny; ++k) {
    int p = k;
    double best = fabs(ws[oJ + k * ny + k]);
    for (int r = k + 1; r < ny; ++r) {
      const double a = fabs(ws[oJ + r * ny + k]);
      if (a > best) { best = a; p = r; }
    }
    if (!(best > 0.0)) return 1;
    if (p != k) {
      for (int c = 0; c < ny; ++c) { const double t = ws[oJ + k * ny + c]; ws[oJ + k * ny + c] = ws[oJ + p * ny + c]; ws[oJ + p * ny + c] = t; }
      for (int c = 0; c < nx; ++c) { const double t = ws[oX + k * nx + c]; ws[oX + k * nx + c] = ws[oX + p * nx + c]; ws[oX + p * nx + c] = t; }
    }
    const double piv = ws[oJ + k * ny + k];
    for (int r = k + 1; r < ny; ++r) {
      const double l = ws[oJ + r * ny + k] / piv;
      if (l == 0.0) continue;
      for (int c = k + 1; c < ny; ++c) ws[oJ + r * ny + c] -= l * ws[oJ + k * ny + c];
      for (int c = 0; c < nx; ++c) ws[oX + r * nx + c] -= l * ws[oX + k * nx + c];
    }
  }
  for (int c = 0; c < nx; ++c)
    for (int r = ny - 1; r >= 0; --r) {
      double s = ws[oX + r * nx + c];
      for (int q = r + 1; q < ny; ++q) s -= ws[oJ + r * ny + q] * ws[oX + q * nx + c];
      ws[oX + r * nx + c] = s / ws[oJ + r * ny + r];
    }
  // D = dZ/dx - dZ/dy X
  for (int r = 0; r < nz; ++r)
    for (int c = 0; c < nx; ++c) {
      double s = ws[oZx + r * nx + c];
      for (int q = 0; q < ny; ++q) s -= ws[oZy + r * ny + q] * ws[oX + q * nx + c];
      D[r * nx + c] = s;
    }
  return 0;
}

constexpr int ADJ_THREADS = 128;

template <int NS>
__global__ void __launch_bounds__(ADJ_THREADS)
adj_jacobian_kernel(const __grid_constant__ PhaseConst<NS> pc, double dt, const double* __restrict__ pts, int64_t N,
                    int64_t v0, int64_t count, double* __restrict__ ws, double* __restrict__ D, int* bad) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int64_t v = v0 + i;
  if (local_jacobian<NS>(pc, pc.hmat, dt, CView{pts + v, N}, SView{ws + i, count}, SView{D + v, N})) atomicAdd(bad, 1);
}

struct VjpArgs {
  double ell[9];          // cotangent of the volume-averaged stress (the same at every voxel)
  const double* lam;      // adjoint field Lambda (9 planes), subtracted from ell; null: none
  const double* s_in;     // state cotangent (Fp: 9 planes, xi: NS planes)
  double* g_out;          // mode 0: cotangent of F (9 planes)
  double* s_out;          // mode 1: state cotangent of the increment start (9 + NS planes)
  double* th_part;        // mode 1: per block, the theta cotangent summed over the block's voxels
  int mode;
};

template <int NS>
__global__ void __launch_bounds__(ADJ_THREADS)
adj_vjp_kernel(const double* __restrict__ D, int64_t N, int nx, const VjpArgs a) {
  constexpr int NZ = 18 + NS;
  constexpr int NTH = 4 * ADJ_MAX_FAMILIES;
  __shared__ double red[NTH][ADJ_THREADS / 32];
  const int64_t v = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const bool active = v < N;
  double zb[NZ];
  double th[NTH];
  for (int p = 0; p < NTH; ++p) th[p] = 0.0;
  if (active) {
    for (int r = 0; r < 9; ++r) zb[r] = a.ell[r] - (a.lam ? a.lam[r * N + v] : 0.0);
    for (int r = 9; r < NZ; ++r) zb[r] = a.s_in[(r - 9) * N + v];
    const int c0 = a.mode == 0 ? 0 : 9, c1 = a.mode == 0 ? 9 : nx;
    for (int c = c0; c < c1; ++c) {
      double s = 0.0;
      for (int r = 0; r < NZ; ++r) s = fma(D[(int64_t(r) * nx + c) * N + v], zb[r], s);
      if (a.mode == 0) a.g_out[c * N + v] = s;
      else if (c < 18 + NS) a.s_out[(c - 9) * N + v] = s;
      else th[c - 18 - NS] = s;
    }
  }
  if (a.mode != 1) return;
  for (int p = 0; p < NTH; ++p)
    for (int o = 16; o > 0; o >>= 1) th[p] += __shfl_down_sync(0xffffffffu, th[p], o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
    for (int p = 0; p < NTH; ++p) red[p][warp] = th[p];
  __syncthreads();
  if (threadIdx.x < NTH) {
    double s = 0.0;
    for (int w = 0; w < ADJ_THREADS / 32; ++w) s += red[threadIdx.x][w];
    a.th_part[int64_t(blockIdx.x) * NTH + threadIdx.x] = s;
  }
}

// sigma_b = sum_a D[a][b] Lambda_a - G_b  (a, b < 9: K = dP/dF); per block the 9 sums of sigma
__global__ void __launch_bounds__(ADJ_THREADS)
adj_sigma_kernel(const double* __restrict__ D, int64_t N, int nx, const double* __restrict__ lam,
                 const double* __restrict__ G, double* __restrict__ sig, double* __restrict__ partials) {
  __shared__ double red[9][ADJ_THREADS / 32];
  const int64_t v = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  double s9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (v < N) {
    double l[9];
    for (int k = 0; k < 9; ++k) l[k] = lam[k * N + v];
    for (int b = 0; b < 9; ++b) {
      double s = G ? -G[b * N + v] : 0.0;
      for (int k = 0; k < 9; ++k) s = fma(D[(int64_t(k) * nx + b) * N + v], l[k], s);
      sig[b * N + v] = s;
      s9[b] = s;
    }
  }
  for (int k = 0; k < 9; ++k)
    for (int o = 16; o > 0; o >>= 1) s9[k] += __shfl_down_sync(0xffffffffu, s9[k], o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
    for (int k = 0; k < 9; ++k) red[k][warp] = s9[k];
  __syncthreads();
  if (threadIdx.x < 9) {
    double s = 0.0;
    for (int w = 0; w < ADJ_THREADS / 32; ++w) s += red[threadIdx.x][w];
    partials[int64_t(blockIdx.x) * 9 + threadIdx.x] = s;
  }
}

constexpr int MDOT_THREADS = 256;

// per block: sum over its elements of w * V_i for i < nv (V_i = V + i n)
__global__ void __launch_bounds__(MDOT_THREADS)
adj_mdot_kernel(const double* __restrict__ w, const double* __restrict__ V, int64_t n, int nv, double* partials) {
  __shared__ double red[ADJ_KRYLOV_MAX + 1][MDOT_THREADS / 32];
  double acc[ADJ_KRYLOV_MAX + 1];
  for (int i = 0; i <= ADJ_KRYLOV_MAX; ++i) acc[i] = 0.0;
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
    const double we = w[e];
    for (int i = 0; i < nv; ++i) acc[i] = fma(we, V[int64_t(i) * n + e], acc[i]);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = 0; i < nv; ++i) {
    double s = acc[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) red[i][warp] = s;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nv; i += blockDim.x) {
    double s = 0.0;
    for (int q = 0; q < MDOT_THREADS / 32; ++q) s += red[i][q];
    partials[int64_t(blockIdx.x) * nv + i] = s;
  }
}

struct Coefs {
  double c[ADJ_KRYLOV_MAX + 1];
};

// y += sum_i c_i V_i
__global__ void adj_maxpy_kernel(double* __restrict__ y, const double* __restrict__ V, int64_t n, int nv, const Coefs c) {
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
    double s = y[e];
    for (int i = 0; i < nv; ++i) s = fma(c.c[i], V[int64_t(i) * n + e], s);
    y[e] = s;
  }
}

__global__ void adj_scale_kernel(double* __restrict__ y, const double* __restrict__ x, double a, int64_t n) {
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x)
    y[e] = a * x[e];
}

}  // namespace

int adj_ws_size(int ns, int nf) {
  const int ny = adj_ny(ns), nx = adj_nx(ns, nf), nz = adj_nz(ns);
  return ny * ny + ny * nx + nz * ny + nz * nx;
}

template <int NS>
cudaError_t launch_adj_jacobian(const PhaseConst<NS>& pc, double dt, const double* pts, int64_t N, int64_t v0,
                                int64_t count, double* ws, double* D, int* bad, cudaStream_t s) {
  const int nb = int((count + ADJ_THREADS - 1) / ADJ_THREADS);
  adj_jacobian_kernel<NS><<<nb, ADJ_THREADS, 0, s>>>(pc, dt, pts, N, v0, count, ws, D, bad);
  return cudaGetLastError();
}

template <int NS>
cudaError_t launch_adj_vjp(const double* D, int64_t N, int nx, const double ell[9], const double* lam,
                           const double* s_in, double* g_out, double* s_out, double* th_part, int mode, cudaStream_t s) {
  VjpArgs a;
  for (int k = 0; k < 9; ++k) a.ell[k] = ell[k];
  a.lam = lam;
  a.s_in = s_in;
  a.g_out = g_out;
  a.s_out = s_out;
  a.th_part = th_part;
  a.mode = mode;
  adj_vjp_kernel<NS><<<adj_blocks(N), ADJ_THREADS, 0, s>>>(D, N, nx, a);
  return cudaGetLastError();
}

int adj_blocks(int64_t N) { return int((N + ADJ_THREADS - 1) / ADJ_THREADS); }

cudaError_t launch_adj_sigma(const double* D, int64_t N, int nx, const double* lam, const double* G, double* sig,
                             double* partials, cudaStream_t s) {
  adj_sigma_kernel<<<adj_blocks(N), ADJ_THREADS, 0, s>>>(D, N, nx, lam, G, sig, partials);
  return cudaGetLastError();
}

int adj_mdot_blocks(int nsm) { return 2 * nsm; }

cudaError_t launch_adj_mdot(const double* w, const double* V, int64_t n, int nv, double* partials, int nsm,
                            cudaStream_t s) {
  if (nv < 1 || nv > ADJ_KRYLOV_MAX + 1) return cudaErrorInvalidValue;
  adj_mdot_kernel<<<adj_mdot_blocks(nsm), MDOT_THREADS, 0, s>>>(w, V, n, nv, partials);
  return cudaGetLastError();
}

cudaError_t launch_adj_maxpy(double* y, const double* V, int64_t n, int nv, const double* c, int nsm, cudaStream_t s) {
  if (nv < 1 || nv > ADJ_KRYLOV_MAX + 1) return cudaErrorInvalidValue;
  Coefs cc;
  for (int i = 0; i <= ADJ_KRYLOV_MAX; ++i) cc.c[i] = i < nv ? c[i] : 0.0;
  adj_maxpy_kernel<<<2 * nsm, 256, 0, s>>>(y, V, n, nv, cc);
  return cudaGetLastError();
}

cudaError_t launch_adj_scale(double* y, const double* x, double a, int64_t n, int nsm, cudaStream_t s) {
  adj_scale_kernel<<<2 * nsm, 256, 0, s>>>(y, x, a, n);
  return cudaGetLastError();
}

// Host evaluation of the same local Jacobian (tests and host tools): pt 27 + 2 NS entries, D nz x nx.
template <int NS>
int host_local_jacobian(const PhaseConst<NS>& pc, const double* h, double dt, const double* pt, double* D) {
  std::vector<double> ws(adj_ws_size(NS, pc.nf));
  return local_jacobian<NS>(pc, h, dt, CView{pt, 1}, SView{ws.data(), 1}, SView{D, 1});
}

#define DMK_INSTANTIATE(NS)                                                                                      \
  template cudaError_t launch_adj_jacobian<NS>(const PhaseConst<NS>&, double, const double*, int64_t, int64_t,  \
                                               int64_t, double*, double*, int*, cudaStream_t);                 \
  template cudaError_t launch_adj_vjp<NS>(const double*, int64_t, int, const double*, const double*,            \
                                          const double*, double*, double*, double*, int, cudaStream_t);         \
  template int host_local_jacobian<NS>(const PhaseConst<NS>&, const double*, double, const double*, double*);
DMK_INSTANTIATE(12)
DMK_INSTANTIATE(18)
DMK_INSTANTIATE(24)
DMK_INSTANTIATE(48)
#undef DMK_INSTANTIATE

}  // namespace dmk
