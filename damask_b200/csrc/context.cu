// Host side of the damask_b200 C-ABI: context (device-resident per-voxel state,
// cuFFT plans, solver scalars) and the grid_mechanical_spectral_basic_* entry points.
#include "../../include/damask_b200.h"
#include "kernels.cuh"
#include "adjoint.cuh"
#include "host_parallel.h"
#include "lattice.h"

#include <cufft.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

using namespace dmk;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CK(x)                                                                              \
  do {                                                                                     \
    cudaError_t e_ = (x);                                                                  \
    if (e_ != cudaSuccess) return fail(DMK_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)
#define CKL(x)                                                                             \
  do {                                                                                     \
    cudaError_t e_ = (x);                                                                  \
    if (e_ != cudaSuccess) return fail(DMK_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    ++c->launches;                                                                         \
  } while (0)
#define CKF(x)                                                                             \
  do {                                                                                     \
    cufftResult r_ = (x);                                                                  \
    if (r_ != CUFFT_SUCCESS) return fail(DMK_ERR_CUFFT, std::string(#x) + " failed: " + std::to_string(int(r_))); \
  } while (0)

template <typename T>
int dalloc(T** p, size_t n) {
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T) + 256);
  if (e != cudaSuccess) return fail(DMK_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  return 0;
}

}  // namespace

namespace dmk {
void set_last_error(const std::string& msg) { g_err = msg; }
}  // namespace dmk

struct dmk_ctx {
  int device = 0;
  int nsm = 148;
  int cells[3];
  double geom[3];
  int64_t N = 0;
  double wgt = 0.0;
  int NS = 0;                    // slip systems of the kernels (the compiled count)
  int NSact = 0;                 // active slip systems of the phase (NS minus the inert padding)
  int precision = DMK_PRECISION_FP64;
  dmk_numerics num;
  HostPhase hp;
  PhaseConst<12>* pc12 = nullptr;
  PhaseConst<18>* pc18 = nullptr;
  PhaseConst<24>* pc24 = nullptr;
  PhaseConst<48>* pc48 = nullptr;
  double* hmat = nullptr;        // slip-slip hardening matrix (NS x NS), read by the pass kernels
  SysConst* sysc = nullptr;      // per-system constants of the Newton loop (NS entries)
  Numerics nm;
  Numerics2 nm2;
  GammaConst gc;
  cudaStream_t stream = nullptr;

  // device fields (planes)
  double *Fsol = nullptr, *r = nullptr, *F = nullptr, *F0 = nullptr, *Fp = nullptr, *Fp0 = nullptr, *Lp = nullptr,
         *Lp0 = nullptr, *S = nullptr, *S0 = nullptr, *Fe = nullptr, *P = nullptr, *Pnew = nullptr, *Flast = nullptr,
         *Fdot = nullptr, *state = nullptr, *state0 = nullptr;
  double* spec = nullptr;       // FP64 spectrum (9 planes of complex)
  float* specf = nullptr;       // FP32 spectrum (mixed)
  float* Pf = nullptr;          // FP32 stress / residual planes (mixed)
  double* partials = nullptr;   // constitutive / forward partial sums
  double* sums = nullptr;
  double* div_partials = nullptr;
  int* status = nullptr;
  int* iter = nullptr;
  unsigned long long* counters = nullptr;
  SolverScalars* sc = nullptr;
  double* scratch = nullptr;    // host <-> device staging, grown on demand
  size_t scratch_len = 0;
  TangentOut tan{};
  double* tan_out = nullptr;    // 243 doubles
  double* tan_host = nullptr;   // pinned: 243 doubles of tan_out, then the 4 counters (as unsigned long long)
  long long* tan_idx = nullptr;
  int tan_blocks = 0;
  void* fft_work = nullptr;
  cufftHandle plan_fwd = 0, plan_bwd = 0, plan_fwd_f = 0, plan_bwd_f = 0;
  cufftHandle plan_vec_bwd = 0; // Z2D of a 3-component (vector) spectrum, updateCoords
  double* xp = nullptr;         // cell-centre coordinates, 3 per voxel (discretization_IPcoords)
  double* xn = nullptr;         // node coordinates, 3 per node (discretization_NodeCoords)
  double* favg = nullptr;       // average F of the last updateCoords (9)
  // spectral polarization scheme (solver 1): Fsol and r hold [F; F_tau] (18 planes)
  int solver = 0;
  double *Ftau = nullptr, *Ftau_last = nullptr, *Ftau_dot = nullptr, *Feval = nullptr, *curl_partials = nullptr;
  PolConst polc{};
  double err_curl = 0.0;
  double h_aim[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};   // host source of the DC term upload
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};

  // host copy of the solver module state (grid_mech_spectral_basic.f90:30-45)
  double F_aim[9], F_aim_lastinc[9], F_aimDot[9], P_aim[9], P_av[9];
  double C_volAvg[81], C_volAvgLastInc[81], C_minMaxAvg[81], C_minMaxAvgLastInc[81], Scomp[81];
  double C_gamma[81];            // reference stiffness of the Gamma operator in use (C_minMaxAvgRestart)
  int stress_mask[9];
  double q_rot[4];
  double dt = 0.0;
  int64_t last_counters[4] = {0, 0, 0, 0};
  double last_ms[3] = {0, 0, 0};
  bool iter_enabled = false;
  int64_t launches = 0;                  // kernels of this library launched by the context
  cudaEvent_t tev[2] = {nullptr, nullptr};
  // Anderson acceleration history (snes_type 1)
  int aa_m = 0;
  int aa_blocks = 0;
  double *aa_dX = nullptr, *aa_dR = nullptr, *aa_Rprev = nullptr, *aa_partials = nullptr, *aa_out = nullptr;
  // constitutive pass scheme: per-voxel iteration state, voxel lists, pass counts
  double* pw = nullptr;          // Fs F0s Fp0s Lp0s (9 each), st0s dot last1 (2 NS each), stepFrac, step
  int* pctl = nullptr;           // 6 planes of per-voxel control integers
  double* dot0 = nullptr;        // 2 NS planes: dotState at (S0, state0), see dot0_valid
  bool dot0_valid = false;       // dot0 holds the rates of the current increment-start values
  // The voxels are split into PASS_CHUNKS chunks whose pass loops run on their own streams,
  // so that the latency-bound control kernel of one chunk overlaps the compute-bound stress
  // kernel of another.  Per chunk: two voxel lists alternating between passes, their counts.
  cudaStream_t cstream[PASS_CHUNKS] = {};   // [0] is `stream`
  cudaEvent_t fork = nullptr, join[PASS_CHUNKS] = {};
  int* plist[PASS_CHUNKS][2] = {};
  int nchunks = PASS_CHUNKS;     // chunks in use: fewer for small RVEs (one host sync per chunk and pass)
  int stress_variant = 0;        // register bound of the stress kernel (stress_variant_blocks); dmk_autotune
  int* pcount = nullptr;         // [2 h + k]: entries appended to plist[h][k]
  int* hcount = nullptr;         // pinned host copies of the current counts of the chunks
  int64_t passes = 0;            // constitutive passes launched (all evaluations)

  // device checkpoints (dmk_checkpoint_save / _restore): per slot, the per-voxel state and the
  // device solver scalars in one device buffer, the host solver state in a host vector
  struct Checkpoint {
    double* dev = nullptr;
    std::vector<double> host;
  };
  std::vector<Checkpoint> ckpts;

  // adjoint of increments (dmk_adj_*)
  int adj_slots = 0, adj_nx = 0, adj_nz = 0;
  double* adj_pts = nullptr;       // per slot: the linearization point, 27 + 2 NS planes (F, Fp0, xi0, Lp, xi)
  std::vector<double> adj_dt;      // per slot: time step of the increment
  std::vector<std::array<int, 9>> adj_mask;   // per slot: stress mask of the load case (1 = not prescribed)
  std::vector<char> adj_rec;       // per slot: recorded
  double* adj_s = nullptr;         // 2 x (9 + NS) planes: state cotangent (Fp, xi), current and next
  int adj_cur = 0;
  double* adj_D = nullptr;         // nz x nx planes: the local Jacobians of the increment being reversed
  double* adj_ws = nullptr;        // workspace of the local Jacobian, adj_chunk voxels
  int64_t adj_chunk = 0;
  double *adj_G = nullptr, *adj_lam = nullptr, *adj_sig = nullptr, *adj_w = nullptr;   // 9 planes each
  double* adj_V = nullptr;         // Krylov basis: ADJ_KRYLOV_MAX + 1 fields of 9 planes
  double* adj_part = nullptr;      // per-block partial sums
  int* adj_bad = nullptr;          // voxels whose local Jacobian was singular
};

namespace {

int64_t node_count(const dmk_ctx* c) { return int64_t(c->cells[0] + 1) * (c->cells[1] + 1) * (c->cells[2] + 1); }

Fields make_fields(dmk_ctx* c, const double* r) {
  Fields f;
  f.N = c->N;
  f.Fsol = c->Fsol; f.r = r; f.F = c->F; f.F0 = c->F0; f.Fp = c->Fp; f.Fp0 = c->Fp0; f.Lp = c->Lp; f.Lp0 = c->Lp0;
  f.S = c->S; f.S0 = c->S0; f.Fe = c->Fe; f.P = c->Pnew; f.state = c->state; f.state0 = c->state0;
  f.partials = c->partials; f.status = c->status; f.iter = c->iter_enabled ? c->iter : nullptr;
  f.counters = c->counters;
  return f;
}

PassWork pass_work(dmk_ctx* c, int half, int out) {
  const int64_t N = c->N;
  const int NST = 2 * c->NS;
  PassWork w;
  w.Fs = c->pw;
  w.F0s = w.Fs + 9 * N;
  w.Fp0s = w.F0s + 9 * N;
  w.Lp0s = w.Fp0s + 9 * N;
  w.st0s = w.Lp0s + 9 * N;
  w.D = w.st0s + NST * N;
  w.adg = w.D + 2 * NST * N;
  w.dot0 = c->dot0;
  w.sub = w.adg + int64_t(c->NS) * N;
  w.lo = w.sub + 2 * N;
  w.dl = w.lo + 9 * N;
  w.ctl = c->pctl;
  w.list_out = c->plist[half][out];
  w.count_out = c->pcount + 2 * half + out;
  return w;
}
size_t pass_work_doubles(int64_t N, int NS) { return size_t(N) * size_t(36 + 7 * NS + 2 + 18); }

template <int NS>
int constitutive_passes(dmk_ctx* c, const PhaseConst<NS>& pc, const Fields& f, double dt, int apply) {
  const int K = c->nchunks;
  int64_t lo[PASS_CHUNKS], hi[PASS_CHUNKS];
  for (int h = 0; h < K; ++h) {
    lo[h] = c->N * h / K;
    hi[h] = c->N * (h + 1) / K;
  }
  // the other streams start after everything queued on the first
  CK(cudaEventRecord(c->fork, c->stream));
  for (int h = 1; h < K; ++h) CK(cudaStreamWaitEvent(c->cstream[h], c->fork, 0));
  int cur[PASS_CHUNKS];
  bool active[PASS_CHUNKS];
  for (int h = 0; h < K; ++h) {
    // pass 0: restore and control up to the first integrateStress of every voxel of the chunk
    cur[h] = 0;
    CK(cudaMemsetAsync(c->pcount + 2 * h, 0, 2 * sizeof(int), c->cstream[h]));
    CKL(launch_constitutive_begin<NS>(pc, c->nm, f, pass_work(c, h, 0), dt, apply, c->dot0_valid ? 1 : 0, lo[h], hi[h],
                                      c->cstream[h]));
    CK(cudaMemcpyAsync(c->hcount + h, c->pcount + 2 * h, sizeof(int), cudaMemcpyDeviceToHost, c->cstream[h]));
    ++c->passes;
    active[h] = hi[h] > lo[h];
  }
  c->dot0_valid = true;   // the begin kernels above stored (or read) the increment-start rates
  // each chunk advances as soon as its previous pass has ended, so the chunks pipeline
  for (int pass = 1;;) {
    bool any = false;
    for (int h = 0; h < K; ++h) {
      if (!active[h]) continue;
      CK(cudaStreamSynchronize(c->cstream[h]));
      const int64_t n = c->hcount[h];
      if (n == 0) { active[h] = false; continue; }
      any = true;
      // bounded by substeps x state iterations; a runaway count means corrupted control state
      if (++pass > 400000) return fail(DMK_ERR_CUDA, "constitutive passes did not terminate");
      const int nxt = 1 - cur[h];
      CK(cudaMemsetAsync(c->pcount + 2 * h + nxt, 0, sizeof(int), c->cstream[h]));
      CKL(launch_constitutive_pass<NS>(pc, c->nm, f, pass_work(c, h, nxt), dt, c->plist[h][cur[h]], n,
                                       c->cstream[h], c->stress_variant));
      ++c->launches;                                       // a pass is a stress and a control kernel
      ++c->passes;
      CK(cudaMemcpyAsync(c->hcount + h, c->pcount + 2 * h + nxt, sizeof(int), cudaMemcpyDeviceToHost, c->cstream[h]));
      cur[h] = nxt;
    }
    if (!any) break;
  }
  // join: later work on the first stream sees all chunks
  for (int h = 1; h < K; ++h) {
    CK(cudaEventRecord(c->join[h], c->cstream[h]));
    CK(cudaStreamWaitEvent(c->stream, c->join[h], 0));
  }
  return 0;
}

int run_constitutive(dmk_ctx* c, const Fields& f, double dt, int apply) {
  switch (c->NS) {
    case 12: return constitutive_passes<12>(c, *c->pc12, f, dt, apply);
    case 18: return constitutive_passes<18>(c, *c->pc18, f, dt, apply);
    case 24: return constitutive_passes<24>(c, *c->pc24, f, dt, apply);
    case 48: return constitutive_passes<48>(c, *c->pc48, f, dt, apply);
  }
  return fail(DMK_ERR_CONFIG, "unsupported number of slip systems");
}
cudaError_t run_dPdF(dmk_ctx* c, const Fields& f, double dt, const TangentOut& o, bool with_sums = true) {
  switch (c->NS) {
    case 12: return launch_dPdF<12>(*c->pc12, f, dt, o, 0, c->N, c->stream, with_sums);
    case 18: return launch_dPdF<18>(*c->pc18, f, dt, o, 0, c->N, c->stream, with_sums);
    case 24: return launch_dPdF<24>(*c->pc24, f, dt, o, 0, c->N, c->stream, with_sums);
    case 48: return launch_dPdF<48>(*c->pc48, f, dt, o, 0, c->N, c->stream, with_sums);
  }
  return cudaErrorInvalidValue;
}
cudaError_t run_pick(dmk_ctx* c, const Fields& f, double dt) {
  switch (c->NS) {
    case 12: return launch_tangent_pick<12>(*c->pc12, f, dt, c->tan_idx, c->tan_out, c->tan.planes, c->stream);
    case 18: return launch_tangent_pick<18>(*c->pc18, f, dt, c->tan_idx, c->tan_out, c->tan.planes, c->stream);
    case 24: return launch_tangent_pick<24>(*c->pc24, f, dt, c->tan_idx, c->tan_out, c->tan.planes, c->stream);
    case 48: return launch_tangent_pick<48>(*c->pc48, f, dt, c->tan_idx, c->tan_out, c->tan.planes, c->stream);
  }
  return cudaErrorInvalidValue;
}

int nblocks_const(const dmk_ctx* c) { return int((c->N + CONST_THREADS - 1) / CONST_THREADS); }

// Slip-system counts with compiled kernels are 12, 18, 24 and 48.  Any other count (the reference
// takes any N_sl up to the family sizes) runs on the next larger one with inert systems appended:
// zero Schmid matrices, dot_gamma_0 = 0, h_0 = 0 and zero interaction rows and columns, so they
// never slip or harden and each term they add to a sum over systems is an exact zero.  Their
// states (xi = 1, gamma = 0) stay on the device; field and restart accessors show the active ones.
int padded_slip_count(int ns) {
  for (int k : {12, 18, 24, 48})
    if (ns <= k) return k;
  return 0;
}
void pad_host_phase(HostPhase& hp, int np) {
  const int ns = hp.Ns;
  if (np == ns) return;
  const std::array<double, 9> z9{};
  const std::array<double, 6> z6{};
  hp.P.resize(np, z9);
  hp.Ppos.resize(np, z9);
  hp.Pneg.resize(np, z9);
  hp.dn.resize(np, z6);
  hp.dg0.resize(np, 0.0);
  hp.n.resize(np, 1.0);
  hp.a.resize(np, 1.0);
  hp.h0f.resize(np, 0.0);
  hp.xiinf.resize(np, 1.0);
  hp.xi0.resize(np, 1.0);
  hp.fam.resize(np, -1);
  hp.hfac.resize(np, 0.0);
  std::vector<double> h(size_t(np) * np, 0.0);
  for (int s = 0; s < ns; ++s)
    for (int k = 0; k < ns; ++k) h[size_t(s) * np + k] = hp.h[size_t(s) * ns + k];
  hp.h.swap(h);
  hp.Ns = np;
}

template <int NS>
void fill_phase_const(const HostPhase& hp, const double* hmat, PhaseConst<NS>& pc) {
  pc.hmat = hmat;
  std::memcpy(pc.C66, hp.C66, sizeof pc.C66);
  std::memcpy(pc.C, hp.C, sizeof pc.C);
  for (int s = 0; s < NS; ++s) {
    for (int k = 0; k < 9; ++k) {
      pc.P[s][k] = hp.P[s][k];
      pc.PnS[0][s][k] = hp.Ppos[s][k];
      pc.PnS[1][s][k] = hp.Pneg[s][k];
    }
    for (int k = 0; k < 6; ++k) pc.dn[s][k] = hp.dn[s][k];
    for (int sense = 0; sense < 2; ++sense) {
      const double* Pn = sense == 0 ? hp.Ppos[s].data() : hp.Pneg[s].data();
      // tau = S : P_nS with S symmetric -> weights on (11,22,33,23,13,12)
      double* p = pc.p6[sense][s];
      p[0] = Pn[0]; p[1] = Pn[4]; p[2] = Pn[8];
      p[3] = Pn[7] + Pn[5]; p[4] = Pn[6] + Pn[2]; p[5] = Pn[3] + Pn[1];
      // Q(t,r) = sum_mn P_nS(m,n) C(m,n,t,r)
      double Q[9];
      for (int t = 0; t < 3; ++t)
        for (int r = 0; r < 3; ++r) {
          double acc = 0.0;
          for (int n = 0; n < 3; ++n)
            for (int m = 0; m < 3; ++m) acc += Pn[m + 3 * n] * hp.C[m + 3 * n + 9 * t + 27 * r];
          Q[t + 3 * r] = acc;
        }
      double* q = pc.q6[sense][s];
      q[0] = Q[0]; q[1] = Q[4]; q[2] = Q[8]; q[3] = 0.5 * (Q[7] + Q[5]); q[4] = 0.5 * (Q[6] + Q[2]); q[5] = 0.5 * (Q[3] + Q[1]);
    }
    pc.dg0[s] = hp.dg0[s];
    pc.n[s] = hp.n[s];
    pc.a[s] = hp.a[s];
    pc.h0f[s] = hp.h0f[s];
    pc.xiinf[s] = hp.xiinf[s];
    pc.ixiinf[s] = 1.0 / hp.xiinf[s];
    pc.n_int[s] = (hp.n[s] == std::floor(hp.n[s]) && hp.n[s] >= 1.0 && hp.n[s] <= 64.0) ? int(hp.n[s]) : -1;
    pc.a_int[s] = (hp.a[s] == std::floor(hp.a[s]) && hp.a[s] >= 0.0 && hp.a[s] <= 64.0) ? int(hp.a[s]) : -1;
  }
  pc.atol_xi = hp.atol_xi;
  pc.atol_gamma = hp.atol_gamma;
  for (int s = 0; s < NS; ++s) {
    pc.fam[s] = hp.fam[s];
    pc.hfac[s] = hp.hfac[s];
  }
  pc.nf = hp.nf;
  std::memcpy(pc.th, hp.th, sizeof pc.th);
}

// host rotations (rotations.f90:282-339, P = -1)
void h_rotvec(const double* v, const double* q, double* o) {
  const double A = q[0] * q[0] - (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  const double B = 2.0 * (q[1] * v[0] + q[2] * v[1] + q[3] * v[2]);
  const double C = -2.0 * q[0];
  const double cx = q[2] * v[2] - q[3] * v[1], cy = q[3] * v[0] - q[1] * v[2], cz = q[1] * v[1] - q[2] * v[0];
  o[0] = A * v[0] + B * q[1] + C * cx;
  o[1] = A * v[1] + B * q[2] + C * cy;
  o[2] = A * v[2] + B * q[3] + C * cz;
}
void h_rot33(const double* qin, const double* T, double* R, bool active) {
  const double q[4] = {qin[0], active ? -qin[1] : qin[1], active ? -qin[2] : qin[2], active ? -qin[3] : qin[3]};
  double tmp[9];
  for (int i = 0; i < 3; ++i) {
    const double v[3] = {T[i], T[i + 3], T[i + 6]};
    double o[3];
    h_rotvec(v, q, o);
    tmp[i] = o[0]; tmp[i + 3] = o[1]; tmp[i + 6] = o[2];
  }
  for (int j = 0; j < 3; ++j) {
    const double v[3] = {tmp[3 * j], tmp[3 * j + 1], tmp[3 * j + 2]};
    double o[3];
    h_rotvec(v, q, o);
    R[3 * j] = o[0]; R[3 * j + 1] = o[1]; R[3 * j + 2] = o[2];
  }
}
void h_rot3333(const double* q, const double* T, double* R) {
  std::memcpy(R, T, 81 * sizeof(double));
  auto at = [&](int i, int j, int k, int l) -> double& { return R[i + 3 * j + 9 * k + 27 * l]; };
  double v[3], o[3];
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) for (int k = 0; k < 3; ++k) {
    for (int l = 0; l < 3; ++l) v[l] = at(i, j, k, l);
    h_rotvec(v, q, o); for (int l = 0; l < 3; ++l) at(i, j, k, l) = o[l];
  }
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) for (int l = 0; l < 3; ++l) {
    for (int k = 0; k < 3; ++k) v[k] = at(i, j, k, l);
    h_rotvec(v, q, o); for (int k = 0; k < 3; ++k) at(i, j, k, l) = o[k];
  }
  for (int i = 0; i < 3; ++i) for (int k = 0; k < 3; ++k) for (int l = 0; l < 3; ++l) {
    for (int j = 0; j < 3; ++j) v[j] = at(i, j, k, l);
    h_rotvec(v, q, o); for (int j = 0; j < 3; ++j) at(i, j, k, l) = o[j];
  }
  for (int j = 0; j < 3; ++j) for (int k = 0; k < 3; ++k) for (int l = 0; l < 3; ++l) {
    for (int i = 0; i < 3; ++i) v[i] = at(i, j, k, l);
    h_rotvec(v, q, o); for (int i = 0; i < 3; ++i) at(i, j, k, l) = o[i];
  }
}

// utilities_maskedCompliance, grid_utilities.f90:74-127
int masked_compliance(const double* q, const int* mask9 /* column-major, 1 = 'x' */, const double* C, double* S) {
  bool sv[9];
  int nred = 0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) { sv[3 * i + j] = !mask9[i + 3 * j]; nred += sv[3 * i + j]; }
  double t99[81];
  std::fill(t99, t99 + 81, 0.0);
  if (nred > 0) {
    double Cr[81], M[81];
    h_rot3333(q, C, Cr);
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) for (int k = 0; k < 3; ++k) for (int l = 0; l < 3; ++l)
      M[(3 * i + j) * 9 + 3 * k + l] = Cr[i + 3 * j + 9 * k + 27 * l];
    std::vector<int> idx;
    for (int i = 0; i < 9; ++i) if (sv[i]) idx.push_back(i);
    std::vector<double> cr(nred * nred), sr(nred * nred);
    for (int a = 0; a < nred; ++a) for (int b = 0; b < nred; ++b) cr[a * nred + b] = M[idx[a] * 9 + idx[b]];
    if (invert_dense(cr.data(), sr.data(), nred)) return fail(DMK_ERR_STATE, "masked compliance: singular reduced stiffness");
    // C * S == I check (grid_utilities.f90:106-118)
    for (int a = 0; a < nred; ++a) for (int b = 0; b < nred; ++b) {
      double s = 0.0;
      for (int k = 0; k < nred; ++k) s += cr[a * nred + k] * sr[k * nred + b];
      if (std::fabs(s - (a == b ? 1.0 : 0.0)) > 1.0e-12 || std::isnan(s))
        return fail(DMK_ERR_STATE, "masked compliance: matrix inversion error");
    }
    for (int a = 0; a < nred; ++a) for (int b = 0; b < nred; ++b) t99[idx[a] * 9 + idx[b]] = sr[a * nred + b];
  }
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) for (int k = 0; k < 3; ++k) for (int l = 0; l < 3; ++l)
    S[i + 3 * j + 9 * k + 27 * l] = t99[(3 * i + j) * 9 + 3 * k + l];
  return 0;
}

// the solver scalars of the host state, in one copy (with the forward's rotated rate and aim, when given)
int upload_scalars(dmk_ctx* c, bool reset_iter, const double* avRate = nullptr, const double* aim_fwd = nullptr) {
  SolverScalars h;
  std::memset(&h, 0, sizeof h);
  if (avRate) std::memcpy(h.avRate, avRate, sizeof h.avRate);
  if (aim_fwd) std::memcpy(h.aim_fwd, aim_fwd, sizeof h.aim_fwd);
  std::memcpy(h.F_aim, c->F_aim, sizeof h.F_aim);
  std::memcpy(h.P_aim, c->P_aim, sizeof h.P_aim);
  std::memcpy(h.P_av, c->P_av, sizeof h.P_av);
  std::memcpy(h.Scomp, c->Scomp, sizeof h.Scomp);
  std::memcpy(h.q_rot, c->q_rot, sizeof h.q_rot);
  std::memcpy(h.stress_mask, c->stress_mask, sizeof h.stress_mask);
  h.totalIter = reset_iter ? -1 : 0;
  CK(cudaMemcpyAsync(c->sc, &h, sizeof h, cudaMemcpyHostToDevice, c->stream));
  return 0;
}

// spectral_utilities_init scaledGeomSize (spectral_utilities.f90:181-197)
void scaled_geom(const int* n, const double* g, int mode, double* out) {
  const double sp[3] = {g[0] / n[0], g[1] / n[1], g[2] / n[2]};
  auto argmin = [](const double* v) { int k = 0; for (int i = 1; i < 3; ++i) if (v[i] < v[k]) k = i; return k; };
  auto argmax = [](const double* v) { int k = 0; for (int i = 1; i < 3; ++i) if (v[i] > v[k]) k = i; return k; };
  for (int i = 0; i < 3; ++i) out[i] = g[i];
  if (mode == 2) {
    for (int j = 0; j < 3; ++j) if (j != argmin(sp) && j != argmax(sp)) for (int i = 0; i < 3; ++i) out[i] = g[i] / g[j] * double(n[j]);
  } else if (mode == 0) {
    for (int j = 0; j < 3; ++j) if (j != argmin(g) && j != argmax(g)) for (int i = 0; i < 3; ++i) out[i] = g[i] / g[j];
  }
}

int make_plans(dmk_ctx* c) {
  int n[3] = {c->cells[2], c->cells[1], c->cells[0]};
  const int red0 = c->cells[0] / 2 + 1;
  int inemb[3] = {c->cells[2], c->cells[1], c->cells[0]};
  int onemb[3] = {c->cells[2], c->cells[1], red0};
  const long long plane = (long long)red0 * c->cells[1] * c->cells[2];
  size_t w1 = 0, w2 = 0, w3 = 0, w4 = 0, w5 = 0;
  CKF(cufftCreate(&c->plan_fwd));
  CKF(cufftCreate(&c->plan_bwd));
  CKF(cufftCreate(&c->plan_vec_bwd));
  CKF(cufftSetAutoAllocation(c->plan_fwd, 0));
  CKF(cufftSetAutoAllocation(c->plan_bwd, 0));
  CKF(cufftSetAutoAllocation(c->plan_vec_bwd, 0));
  CKF(cufftMakePlanMany(c->plan_fwd, 3, n, inemb, 1, int(c->N), onemb, 1, int(plane), CUFFT_D2Z, 9, &w1));
  CKF(cufftMakePlanMany(c->plan_bwd, 3, n, onemb, 1, int(plane), inemb, 1, int(c->N), CUFFT_Z2D, 9, &w2));
  CKF(cufftMakePlanMany(c->plan_vec_bwd, 3, n, onemb, 1, int(plane), inemb, 1, int(c->N), CUFFT_Z2D, 3, &w5));
  if (c->precision == DMK_PRECISION_MIXED) {
    CKF(cufftCreate(&c->plan_fwd_f));
    CKF(cufftCreate(&c->plan_bwd_f));
    CKF(cufftSetAutoAllocation(c->plan_fwd_f, 0));
    CKF(cufftSetAutoAllocation(c->plan_bwd_f, 0));
    CKF(cufftMakePlanMany(c->plan_fwd_f, 3, n, inemb, 1, int(c->N), onemb, 1, int(plane), CUFFT_R2C, 9, &w3));
    CKF(cufftMakePlanMany(c->plan_bwd_f, 3, n, onemb, 1, int(plane), inemb, 1, int(c->N), CUFFT_C2R, 9, &w4));
  }
  const size_t w = std::max(std::max(std::max(w1, w2), std::max(w3, w4)), w5);
  if (w) CK(cudaMalloc(&c->fft_work, w));
  CKF(cufftSetWorkArea(c->plan_fwd, c->fft_work));
  CKF(cufftSetWorkArea(c->plan_bwd, c->fft_work));
  CKF(cufftSetWorkArea(c->plan_vec_bwd, c->fft_work));
  CKF(cufftSetStream(c->plan_fwd, c->stream));
  CKF(cufftSetStream(c->plan_bwd, c->stream));
  CKF(cufftSetStream(c->plan_vec_bwd, c->stream));
  if (c->precision == DMK_PRECISION_MIXED) {
    CKF(cufftSetWorkArea(c->plan_fwd_f, c->fft_work));
    CKF(cufftSetWorkArea(c->plan_bwd_f, c->fft_work));
    CKF(cufftSetStream(c->plan_fwd_f, c->stream));
    CKF(cufftSetStream(c->plan_bwd_f, c->stream));
  }
  return 0;
}

// One constitutive sweep + commit of P (homogenization_mechanical_response + the P part of
// utilities_constitutiveResponse).  On a failed sweep the previous P field is kept (the
// reference skips mechanical_homogenize when any cell fails, homogenization.f90:343).
int evaluate_constitutive(dmk_ctx* c, double dt, const double* r, int apply, int* status_out,
                          const double* Fsrc = nullptr) {
  CK(cudaMemsetAsync(c->status, 0, sizeof(int), c->stream));
  Fields f = make_fields(c, r);
  if (Fsrc) f.Fsol = const_cast<double*>(Fsrc);   // read only when apply == 0
  CK(cudaEventRecord(c->ev[0], c->stream));
  if (int rc = run_constitutive(c, f, dt, apply)) return rc;
  CK(cudaEventRecord(c->ev[1], c->stream));
  int st = 0;
  CK(cudaMemcpyAsync(&st, c->status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
  c->last_ms[0] += ms;
  if (st == 0) std::swap(c->P, c->Pnew);
  CKL(launch_sum9(c->P, c->N, c->partials, c->stream));   // <P> of the committed (or kept) stress field
  *status_out = st;
  return 0;
}

// dP/dF of every voxel from the stored state: C_volAvg and C_minMaxAvg (grid_utilities.f90:171-202)
int ensure_scratch(dmk_ctx* c, int K);

// C_volAvg and C_minMaxAvg from the tangent sums copied to tan_host
void tangent_complete(dmk_ctx* c);
int tangent_enqueue(dmk_ctx* c, double dt);
void tangent_complete(dmk_ctx* c) {
  const double* h = c->tan_host;
  for (int k = 0; k < 81; ++k) {
    c->C_volAvg[k] = h[k];
    c->C_minMaxAvg[k] = 0.5 * (h[81 + k] + h[162 + k]);
  }
}

// planes_ready: the dPdF planes and norms of the current state are in place (evaluate_tangent_planes),
// only their reductions remain
int tangent_launch(dmk_ctx* c, double dt, double* per_voxel_dev, bool planes_ready) {
  Fields f = make_fields(c, nullptr);
  TangentOut o = c->tan;
  o.per_voxel = per_voxel_dev;
  if (planes_ready) {
    CKL(launch_tangent_sums(o, 0, c->N, c->N, c->stream));
  } else {
    CKL(run_dPdF(c, f, dt, o));
    ++c->launches;                                         // tangent and its column sums
  }
  if (per_voxel_dev) CKL(launch_from_planes(c->tan.planes, per_voxel_dev, c->N, 81, c->stream));
  CKL(launch_tangent_finalize(o, c->tan_blocks, c->wgt, c->tan_out, c->tan_idx, 0, c->N, c->stream));
  c->launches += 2;   // reduce, finalize and first-index kernels
  CKL(run_pick(c, f, dt));
  CK(cudaMemcpyAsync(c->tan_host, c->tan_out, sizeof(double) * 243, cudaMemcpyDeviceToHost, c->stream));
  return 0;
}
// the tangent queued on the context's stream; tangent_complete after the stream has finished
int tangent_enqueue(dmk_ctx* c, double dt) { return tangent_launch(c, dt, nullptr, false); }
int evaluate_tangent(dmk_ctx* c, double dt, double* per_voxel_dev, bool planes_ready = false) {
  if (int rc = tangent_launch(c, dt, per_voxel_dev, planes_ready)) return rc;
  CK(cudaStreamSynchronize(c->stream));
  tangent_complete(c);
  return 0;
}

// math_invSym3333 (math.f90:511-532): Mandel 6x6 of A (math_sym3333to66, :826-845), its inverse,
// expanded with minor symmetry (math_66toSym3333, :851-900).  Column-major 3x3x3x3.
bool inv_sym3333_host(const double* A, double* out) {
  const int pi[6] = {0, 1, 2, 1, 0, 0}, pj[6] = {0, 1, 2, 2, 2, 1};
  const double SQ2 = std::sqrt(2.0);
  auto w = [&](int r) { return r < 3 ? 1.0 : SQ2; };
  double M[6][12];
  for (int r = 0; r < 6; ++r)
    for (int q = 0; q < 6; ++q) {
      M[r][q] = A[pi[r] + 3 * pj[r] + 9 * pi[q] + 27 * pj[q]] * w(r) * w(q);
      M[r][6 + q] = r == q ? 1.0 : 0.0;
    }
  for (int j = 0; j < 6; ++j) {     // Gauss-Jordan with partial pivoting
    int p = j;
    for (int i = j + 1; i < 6; ++i) if (std::fabs(M[i][j]) > std::fabs(M[p][j])) p = i;
    if (M[p][j] == 0.0) return false;
    for (int k = 0; k < 12; ++k) std::swap(M[j][k], M[p][k]);
    const double d = M[j][j];
    for (int k = 0; k < 12; ++k) M[j][k] /= d;
    for (int i = 0; i < 6; ++i)
      if (i != j) {
        const double l = M[i][j];
        for (int k = 0; k < 12; ++k) M[i][k] -= l * M[j][k];
      }
  }
  for (int r = 0; r < 6; ++r)
    for (int q = 0; q < 6; ++q) {
      const double v = M[r][6 + q] / (w(r) * w(q));
      for (int a : {0, 1})
        for (int b : {0, 1}) {
          const int i = a ? pj[r] : pi[r], j = a ? pi[r] : pj[r], k = b ? pj[q] : pi[q], l = b ? pi[q] : pj[q];
          out[i + 3 * j + 9 * k + 27 * l] = v;
        }
    }
  return true;
}

// C_scale = C_minMaxAvg, S_scale = invSym3333(C_minMaxAvg) (grid_mech_spectral_polarization.f90:266-268, 292-296)
int set_polarization_scale(dmk_ctx* c) {
  std::memcpy(c->polc.C, c->C_minMaxAvg, sizeof c->polc.C);
  if (!inv_sym3333_host(c->C_minMaxAvg, c->polc.S)) return fail(DMK_ERR_STATE, "matrix inversion error (S_scale)");
  return 0;
}

// dP/dF planes (and norms) of every voxel from the stored state, without the reductions
int evaluate_tangent_planes(dmk_ctx* c, double dt) {
  Fields f = make_fields(c, nullptr);
  CKL(run_dPdF(c, f, dt, c->tan, false));
  return 0;
}

void update_gamma_host(dmk_ctx* c, const double* C) {
  for (int k = 0; k < 81; ++k) {
    c->C_gamma[k] = C[k];
    c->gc.Cref[k] = C[k] / c->wgt;
  }
}

// D2Z of the committed P, fused divergence + Gamma, Z2D into r (FP64 or FP32 spectral path)
// Gamma convolution (do_gamma, into out, DC from the device scalars' aim_rot) and divergence
// partial sums (do_div) of the 9-plane field `in` (the stress P unless given).
int spectral_pass(dmk_ctx* c, bool fp32, int do_gamma, int do_div, void* out, double* in = nullptr) {
  const double L[3] = {c->geom[0], c->geom[1], c->geom[2]};
  if (!in) in = c->P;
  if (!fp32) {
    CKF(cufftExecD2Z(c->plan_fwd, in, reinterpret_cast<cufftDoubleComplex*>(c->spec)));
    CK(launch_gamma_div<double>(c->spec, c->cells[0], c->cells[1], c->cells[2], L, c->gc, c->sc, c->div_partials, do_gamma,
                                do_div, c->stream));
    if (do_gamma) CKF(cufftExecZ2D(c->plan_bwd, reinterpret_cast<cufftDoubleComplex*>(c->spec), static_cast<double*>(out)));
  } else {
    CKL(launch_to_float(in, c->Pf, 9 * c->N, c->nsm, c->stream));
    CKF(cufftExecR2C(c->plan_fwd_f, c->Pf, reinterpret_cast<cufftComplex*>(c->specf)));
    CK(launch_gamma_div<float>(c->specf, c->cells[0], c->cells[1], c->cells[2], L, c->gc, c->sc, c->div_partials, do_gamma,
                               do_div, c->stream));
    if (do_gamma) CKF(cufftExecC2R(c->plan_bwd_f, reinterpret_cast<cufftComplex*>(c->specf), static_cast<float*>(out)));
  }
  return 0;
}

int ensure_scratch(dmk_ctx* c, int K) {
  const size_t need = size_t(K) * size_t(c->N);
  if (need <= c->scratch_len) return 0;
  if (c->scratch) { cudaStreamSynchronize(c->stream); cudaFree(c->scratch); c->scratch = nullptr; c->scratch_len = 0; }
  int rc = dalloc(&c->scratch, need);
  if (rc) return rc;
  c->scratch_len = need;
  return 0;
}

int h2d_planes(dmk_ctx* c, const double* host, double* dev_planes, int K) {
  if (int rc = ensure_scratch(c, K)) return rc;
  CK(cudaMemcpyAsync(c->scratch, host, sizeof(double) * K * c->N, cudaMemcpyHostToDevice, c->stream));
  CKL(launch_to_planes(c->scratch, dev_planes, c->N, K, c->stream));
  return 0;
}
int d2h_planes(dmk_ctx* c, const double* dev_planes, double* host, int K) {
  if (int rc = ensure_scratch(c, K)) return rc;
  CKL(launch_from_planes(dev_planes, c->scratch, c->N, K, c->stream));
  CK(cudaMemcpyAsync(host, c->scratch, sizeof(double) * K * c->N, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int response(dmk_ctx* c, double dt, int* status) {
  int st = 0;
  int rc = evaluate_constitutive(c, dt, nullptr, 0, &st);
  if (rc) return rc;
  CKL(launch_aim(c->sc, c->partials, nblocks_const(c), c->wgt, 0, c->stream));
  double pav[9];
  CK(cudaMemcpyAsync(pav, reinterpret_cast<char*>(c->sc) + offsetof(SolverScalars, P_av), sizeof pav,
                     cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  std::memcpy(c->P_av, pav, sizeof pav);
  if (st == 0) {
    rc = evaluate_tangent(c, dt, nullptr);
    if (rc) return rc;
  }
  *status = st;
  return 0;
}

constexpr int AA_CHUNK_HOST = 8;

// Least-squares coefficients of the Anderson update (Walker & Ni 2011, type II):
// gamma = argmin |r - dR gamma| from the normal equations G gamma = b on the slots
// (oldest first), solved by Cholesky; while a pivot is not safely positive
// (< 1e-13 of the largest diagonal) the oldest slot is dropped (gamma = 0 there).
std::vector<double> anderson_coefficients(const std::vector<double>& G, int m, const std::vector<int>& slots,
                                          const std::vector<double>& b) {
  std::vector<double> gam(slots.size(), 0.0);
  for (size_t first = 0; first < slots.size(); ++first) {
    const size_t n = slots.size() - first;
    std::vector<double> L(n * n, 0.0);
    double dmax = 0.0;
    for (size_t i = 0; i < n; ++i) dmax = std::max(dmax, G[size_t(slots[first + i]) * m + slots[first + i]]);
    bool ok = dmax > 0.0;
    for (size_t i = 0; ok && i < n; ++i)
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
    if (!ok) continue;
    std::vector<double> y(n), x(n);
    for (size_t i = 0; i < n; ++i) {
      double sum = b[first + i];
      for (size_t k = 0; k < i; ++k) sum -= L[i * n + k] * y[k];
      y[i] = sum / L[i * n + i];
    }
    for (size_t i = n; i-- > 0;) {
      double sum = y[i];
      for (size_t k = i + 1; k < n; ++k) sum -= L[k * n + i] * x[k];
      x[i] = sum / L[i * n + i];
    }
    for (size_t i = 0; i < n; ++i) gam[first + i] = x[i];
    return gam;
  }
  return gam;
}

// grid_mech_spectral_polarization_solution (grid_mech_spectral_polarization.f90:273-309) with its
// form_residual (:562-632) and converged (:521-556) on the solution vector [F; F_tau]; the masked
// compliance S and the Gamma stiffness are set by the caller.  Fixed point as for the basic
// scheme: Richardson X <- X - r, or Anderson acceleration over both fields.
int solution_polarization(dmk_ctx* c, dmk_solution_state* out) {
  if (c->num.update_gamma)
    if (int rc = set_polarization_scale(c)) return rc;
  const int64_t N = c->N, n18 = 18 * N;
  const int snes_max_its = c->num.snes_max_it > 0 ? c->num.snes_max_it : 50;   // PETSc -snes_max_it (default 50)
  const bool anderson = c->num.snes_type == 1;
  const int m = c->aa_m;
  const int nspec = gamma_div_blocks(c->cells[0], c->cells[1], c->cells[2]);
  const double L[3] = {c->geom[0], c->geom[1], c->geom[2]};
  const double beta = c->polc.beta;
  double* rF = c->r;
  double* rtau = c->r + 9 * N;
  auto* spec = reinterpret_cast<cufftDoubleComplex*>(c->spec);
  int evals = 0, reason = 0, totalIter = -1, status = 0;
  std::vector<double> G(size_t(m > 0 ? m : 1) * (m > 0 ? m : 1), 0.0), bvec, divp(nspec), curlp(nspec);
  std::vector<int> slots_b;
  double dots[4 * AA_MAX];
  int count = 0, new_slot = -1;
  double F_av[9], P_av[9];

  auto residual = [&]() -> int {
    ++totalIter;
    CKL(launch_sum9(c->Fsol, N, c->partials, c->stream));             // F_av
    CKL(launch_reduce9(c->partials, nblocks_const(c), c->sums, c->stream));
    CKL(launch_pol_pre(c->Fsol, c->Ftau, N, c->polc, rF, c->stream));
    double bF[9];
    for (int k = 0; k < 9; ++k) bF[k] = beta * c->F_aim[k];
    h_rot33(c->q_rot, bF, c->h_aim, true);
    CK(cudaMemcpyAsync(reinterpret_cast<char*>(c->sc) + offsetof(SolverScalars, aim_rot), c->h_aim, sizeof c->h_aim,
                       cudaMemcpyHostToDevice, c->stream));
    CK(cudaEventRecord(c->ev[2], c->stream));
    CKF(cufftExecD2Z(c->plan_fwd, rF, spec));
    CK(launch_gamma_div<double>(c->spec, c->cells[0], c->cells[1], c->cells[2], L, c->gc, c->sc, c->div_partials, 1, 0,
                                c->stream));
    ++c->launches;
    // the transform writes to Feval: rtau = r + 9N is only 8-byte aligned for odd N, which cuFFT rejects
    CKF(cufftExecZ2D(c->plan_bwd, spec, c->Feval));
    CKL(launch_pol_tau(c->Fsol, c->Feval, rtau, N, beta, c->Feval, c->stream));
    CKF(cufftExecD2Z(c->plan_fwd, c->Fsol, spec));                      // curl of F
    CKL(launch_curl(c->spec, c->cells[0], c->cells[1], c->cells[2], L, c->gc.rescale, c->gc.derivative,
                    c->curl_partials, c->stream));
    CK(cudaEventRecord(c->ev[3], c->stream));
    int st = 0;                                                          // constitutive at F - r_F_tau / beta
    if (int e = evaluate_constitutive(c, c->dt, nullptr, 0, &st, c->Feval)) return e;
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]));
    c->last_ms[1] += ms;
    CKL(launch_aim(c->sc, c->partials, nblocks_const(c), c->wgt, 0, c->stream));
    CK(cudaEventRecord(c->ev[0], c->stream));
    // the per-voxel tangent enters r_F; C_volAvg / C_minMaxAvg of the last residual are reduced
    // from its planes after the solve (nothing reads them before)
    if (int e = evaluate_tangent_planes(c, c->dt)) return e;
    CK(cudaEventRecord(c->ev[1], c->stream));
    CKF(cufftExecD2Z(c->plan_fwd, c->P, spec));                         // divergence of P
    CK(launch_gamma_div<double>(c->spec, c->cells[0], c->cells[1], c->cells[2], L, c->gc, c->sc, c->div_partials, 0, 1,
                                c->stream));
    ++c->launches;
    CKL(launch_pol_rF(c->Fsol, c->Ftau, c->P, c->tan.planes, rtau, N, c->polc, rF, c->stream));
    int nsl = 0;
    if (anderson && new_slot >= 0) {
      slots_b.clear();
      const int mk = std::min(count, m);
      for (int q = count - mk; q < count; ++q) slots_b.push_back(q % m);
      nsl = int(slots_b.size());
      CKL(launch_aa_dots(c->r, c->aa_Rprev, c->aa_dR, n18, new_slot, slots_b.data(), nsl, c->aa_partials, c->aa_blocks,
                        c->aa_out, c->stream));
      c->launches += 2 * ((nsl + AA_CHUNK_HOST - 1) / AA_CHUNK_HOST) - 1;
      CK(cudaMemcpyAsync(dots, c->aa_out, sizeof(double) * 2 * AA_CHUNK_HOST * ((nsl + AA_CHUNK_HOST - 1) / AA_CHUNK_HOST),
                         cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaMemcpyAsync(F_av, c->sums, sizeof F_av, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(P_av, reinterpret_cast<char*>(c->sc) + offsetof(SolverScalars, P_av), sizeof P_av,
                       cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(divp.data(), c->div_partials, sizeof(double) * nspec, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(curlp.data(), c->curl_partials, sizeof(double) * nspec, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
    c->last_ms[2] += ms;
    ++evals;
    status = st;
    if (nsl > 0) {
      bvec.assign(nsl, 0.0);
      for (int q = 0; q < nsl; ++q) {
        const int ch = q / AA_CHUNK_HOST, k = q % AA_CHUNK_HOST;
        const double g = dots[ch * 2 * AA_CHUNK_HOST + k], b = dots[ch * 2 * AA_CHUNK_HOST + AA_CHUNK_HOST + k];
        G[size_t(new_slot) * m + slots_b[q]] = G[size_t(slots_b[q]) * m + new_slot] = g;
        bvec[q] = b;
      }
    }
    double sdiv = 0.0, scurl = 0.0;
    for (int b = 0; b < nspec; ++b) { sdiv += divp[b]; scurl += curlp[b]; }
    c->err_curl = std::sqrt(scurl) * c->wgt * (c->cells[0] == 1 ? 0.5 : 1.0);
    const double err_div = std::sqrt(sdiv) * c->wgt * (c->cells[0] == 1 ? 0.5 : 1.0);
    for (int k = 0; k < 9; ++k) F_av[k] *= c->wgt;
    std::memcpy(c->P_av, P_av, sizeof P_av);
    // F_aim = F_aim - S : (P_av - P_aim); err_BC (:625-630)
    double d[9], e[9], t[9], Rav[9];
    for (int k = 0; k < 9; ++k) d[k] = P_av[k] - c->P_aim[k];
    for (int ij = 0; ij < 9; ++ij) {
      double s = 0.0;
      for (int kl = 0; kl < 9; ++kl) s += c->Scomp[ij + 9 * kl] * d[kl];
      c->F_aim[ij] -= s;
    }
    h_rot33(c->q_rot, F_av, Rav, false);
    for (int k = 0; k < 9; ++k) t[k] = c->F_aim[k] - Rav[k];
    for (int ij = 0; ij < 9; ++ij) {
      double s = 0.0;
      for (int kl = 0; kl < 9; ++kl) s += c->polc.C[ij + 9 * kl] * t[kl];
      e[ij] = s;
    }
    double err_BC = 0.0;
    for (int k = 0; k < 9; ++k) err_BC = std::max(err_BC, std::fabs(c->stress_mask[k] ? e[k] : d[k]));
    // converged (:521-556)
    double pmax = 0.0, fmax = 0.0;
    for (int k = 0; k < 9; ++k) {
      pmax = std::max(pmax, std::fabs(P_av[k]));
      fmax = std::max(fmax, std::fabs(c->F_aim[k] - ((k % 4 == 0) ? 1.0 : 0.0)));
    }
    const double curlTol = std::max(fmax * c->num.eps_rel_curl, c->num.eps_abs_curl);
    const double divTol = std::max(pmax * c->num.eps_rel_div, c->num.eps_abs_div);
    const double BCTol = std::max(pmax * c->num.eps_rel_P, c->num.eps_abs_P);
    reason = 0;
    if (totalIter >= c->num.N_iter_min && err_div / divTol < 1.0 && c->err_curl / curlTol < 1.0 && err_BC / BCTol < 1.0 &&
        status == 0)
      reason = 1;
    else if (totalIter >= c->num.N_iter_max)
      reason = -1;
    if (!std::isfinite(err_div) || !std::isfinite(c->err_curl)) reason = -1;
    out->err_div = err_div;
    out->err_BC = err_BC;
    return 0;
  };

  if (int rc = residual()) return rc;
  if (anderson) { bvec.clear(); slots_b.clear(); }
  for (int it = 1; reason == 0; ++it) {
    if (it > snes_max_its) { reason = -1; break; }
    if (!anderson) {
      CKL(launch_sub(c->Fsol, c->r, n18, c->nsm, c->stream));
    } else {
      std::vector<double> gam = anderson_coefficients(G, m, slots_b, bvec);
      new_slot = count % m;
      CKL(launch_aa_update(c->Fsol, c->r, c->aa_Rprev, c->aa_dX, c->aa_dR, n18, new_slot, slots_b.data(), gam.data(),
                          int(slots_b.size()), c->aa_blocks, c->stream));
      ++count;
    }
    if (int rc = residual()) return rc;
  }
  if (int rc = evaluate_tangent(c, c->dt, nullptr, true)) return rc;   // reductions of the last planes
  out->converged = reason > 0;
  out->iterationsNeeded = totalIter;
  out->stagConverged = 1;
  out->residualEvals = evals;
  std::memcpy(out->P_av, c->P_av, sizeof out->P_av);
  for (int k = 0; k < 9; ++k)
    if (c->stress_mask[k]) c->P_aim[k] = c->P_av[k];
  unsigned long long hc[4];
  CK(cudaMemcpyAsync(hc, c->counters, sizeof hc, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->last_counters[0] = int64_t(evals) * c->N;
  c->last_counters[1] = int64_t(hc[1]);
  c->last_counters[2] = int64_t(hc[2]);
  c->last_counters[3] = evals;
  return 0;
}

// grid_mechanical_spectral_basic_solution before SNESsolve (grid_mech_spectral_basic.f90:259-262):
// masked compliance, reference stiffness of Gamma, device scalars, counters
int solution_prepare(dmk_ctx* c) {
  int rc = masked_compliance(c->q_rot, c->stress_mask, c->C_volAvg, c->Scomp);
  if (rc) return rc;
  if (c->num.update_gamma) update_gamma_host(c, c->C_minMaxAvg);
  if ((rc = upload_scalars(c, true))) return rc;
  CK(cudaMemsetAsync(c->counters, 0, 4 * sizeof(unsigned long long), c->stream));
  c->last_ms[0] = c->last_ms[1] = c->last_ms[2] = 0.0;
  return 0;
}

// grid_mechanical_spectral_basic_solution after SNESsolve (grid_mech_spectral_basic.f90:266-277):
// the solution state, P_aim of the stress-controlled components, and the tangent of the converged
// state (C_volAvg, C_minMaxAvg for the next increment); counters of the solve.  In two halves, so
// that a batch queues the tangents of all its contexts before it waits for them: the first
// queues the tangent and the counters' read-back, the second waits for them.
int solution_finish_begin(dmk_ctx* c, const double F_aim[9], const double P_av[9], int totalIter, double err_div,
                          double err_BC, int reason, int evals, dmk_solution_state* out) {
  std::memcpy(c->F_aim, F_aim, sizeof c->F_aim);
  std::memcpy(c->P_av, P_av, sizeof c->P_av);
  out->converged = reason > 0;
  out->iterationsNeeded = totalIter;
  out->stagConverged = 1;
  out->residualEvals = evals;
  out->err_div = err_div;
  out->err_BC = err_BC;
  std::memcpy(out->P_av, P_av, sizeof out->P_av);
  for (int k = 0; k < 9; ++k)
    if (c->stress_mask[k]) c->P_aim[k] = c->P_av[k];
  if (out->converged) {
    CK(cudaEventRecord(c->ev[0], c->stream));
    if (int rc = tangent_enqueue(c, c->dt)) return rc;
    CK(cudaEventRecord(c->ev[1], c->stream));
  }
  CK(cudaMemcpyAsync(c->tan_host + 243, c->counters, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                     c->stream));
  c->last_counters[0] = int64_t(evals) * c->N;
  c->last_counters[3] = evals;
  return 0;
}
int solution_finish_end(dmk_ctx* c, const dmk_solution_state* out) {
  CK(cudaStreamSynchronize(c->stream));
  if (out->converged) {
    tangent_complete(c);
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
    c->last_ms[2] += ms;
  }
  unsigned long long hc[4];
  std::memcpy(hc, c->tan_host + 243, sizeof hc);
  c->last_counters[1] = int64_t(hc[1]);
  c->last_counters[2] = int64_t(hc[2]);
  return 0;
}
int solution_finish(dmk_ctx* c, const double F_aim[9], const double P_av[9], int totalIter, double err_div,
                    double err_BC, int reason, int evals, dmk_solution_state* out) {
  if (int rc = solution_finish_begin(c, F_aim, P_av, totalIter, err_div, err_BC, reason, evals, out)) return rc;
  return solution_finish_end(c, out);
}

}  // namespace

namespace dmk {
int record_error(int code, const std::string& msg) { return fail(code, msg); }
}  // namespace dmk

extern "C" {

const char* dmk_last_error(void) { return g_err.c_str(); }

int dmk_mech_init(dmk_ctx** out, const int cells[3], const double geomSize[3], const int* materialAt, int n_materials,
                  const double* quaternions, const dmk_phase* phase, const dmk_numerics* num, int precision, int device) {
  if (!out || !cells || !geomSize || !materialAt || !quaternions || !phase || !num) return fail(DMK_ERR_ARG, "null argument");
  *out = nullptr;
  for (int i = 0; i < 3; ++i)
    if (cells[i] < 1 || !(geomSize[i] > 0.0)) return fail(DMK_ERR_ARG, "cells and geomSize must be positive");
  if (precision != DMK_PRECISION_FP64 && precision != DMK_PRECISION_MIXED) return fail(DMK_ERR_ARG, "unknown precision");
  if (num->derivative < 0 || num->derivative > 2)
    return fail(DMK_ERR_CONFIG, "spectral derivative must be continuous (0), central_difference (1) or FWBW_difference (2)");
  if (num->N_iter_max < 1 || num->N_iter_min < 1 || num->N_iter_min > num->N_iter_max)
    return fail(DMK_ERR_CONFIG, "invalid N_iter_min/N_iter_max");
  if (num->N_iter_Lp_max < 1 || num->N_iter_state_max < 1 || num->f_update_jacobi_Lp < 1 || !(num->r_cutback > 0.0) ||
      !(num->r_cutback_min > 0.0) || !(num->r_increase > 0.0) || !(num->r_linesearch_Lp > 0.0))
    return fail(DMK_ERR_CONFIG, "invalid phase.mechanical numerics");
  if (num->solver != 0 && num->solver != 1) return fail(DMK_ERR_CONFIG, "solver must be 0 (spectral_basic) or 1 (spectral_polarization)");
  // grid_mech_spectral_polarization.f90:150-161
  if (num->solver == 1 && (!(num->eps_abs_curl > 0.0) || !(num->eps_rel_curl > 0.0) || !(num->alpha > 0.0) ||
                           num->alpha > 2.0 || num->beta < 0.0 || num->beta > 2.0))
    return fail(DMK_ERR_CONFIG, "invalid polarization numerics (eps_abs_curl(F), eps_rel_curl(F), alpha, beta)");
  dmk_ctx* c = new dmk_ctx();
  int rc = build_host_phase(*phase, c->hp, g_err);
  if (rc) { delete c; return DMK_ERR_CONFIG; }
  c->NSact = c->hp.Ns;
  if (c->NSact < 1 || padded_slip_count(c->NSact) == 0) {
    delete c;
    return fail(DMK_ERR_CONFIG, "between 1 and 48 active slip systems on this path");
  }
  pad_host_phase(c->hp, padded_slip_count(c->NSact));
  c->NS = c->hp.Ns;
  c->device = device;
  c->precision = precision;
  c->num = *num;
  c->solver = num->solver;
  c->polc.alpha = num->alpha;
  c->polc.beta = num->beta;
  for (int i = 0; i < 3; ++i) { c->cells[i] = cells[i]; c->geom[i] = geomSize[i]; }
  c->N = int64_t(cells[0]) * cells[1] * cells[2];
  c->wgt = 1.0 / double(c->N);
  const int64_t N = c->N;
  if (N > 2147483647LL) { delete c; return fail(DMK_ERR_ARG, "at most 2^31 - 1 cells per context"); }
  for (int64_t v = 0; v < N; ++v)
    if (materialAt[v] < 0 || materialAt[v] >= n_materials) { delete c; return fail(DMK_ERR_ARG, "material index out of range"); }

  auto bail = [&](int code) { dmk_destroy(c); return code; };
  if (cudaSetDevice(device) != cudaSuccess) { delete c; return fail(DMK_ERR_CUDA, "cudaSetDevice failed"); }
  cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device);
  bool ok = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming) == cudaSuccess;
  c->cstream[0] = c->stream;
  for (int h = 1; ok && h < PASS_CHUNKS; ++h)
    ok = cudaStreamCreateWithFlags(&c->cstream[h], cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&c->join[h], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    dmk_destroy(c);
    return fail(DMK_ERR_CUDA, "stream");
  }
  for (auto& e : c->ev) cudaEventCreate(&e);

  c->nm.r_cutback_min = num->r_cutback_min; c->nm.r_cutback = num->r_cutback; c->nm.r_increase = num->r_increase;
  c->nm.eps_rel_state = num->eps_rel_state; c->nm.N_iter_state_max = num->N_iter_state_max;
  c->nm.N_iter_Lp_max = num->N_iter_Lp_max; c->nm.r_linesearch_Lp = num->r_linesearch_Lp;
  c->nm.eps_rel_Lp = num->eps_rel_Lp; c->nm.eps_abs_Lp = num->eps_abs_Lp; c->nm.f_update_jacobi_Lp = num->f_update_jacobi_Lp;
  c->nm2.N_iter_min = num->N_iter_min; c->nm2.N_iter_max = num->N_iter_max; c->nm2.cells0 = cells[0];
  c->nm2.eps_abs_div = num->eps_abs_div; c->nm2.eps_rel_div = num->eps_rel_div;
  c->nm2.eps_abs_P = num->eps_abs_P; c->nm2.eps_rel_P = num->eps_rel_P;
  double sgs[3];
  scaled_geom(cells, geomSize, num->divergence_correction, sgs);
  for (int i = 0; i < 3; ++i) c->gc.rescale[i] = geomSize[i] / sgs[i];
  c->gc.derivative = num->derivative;

  if ((rc = dalloc(&c->hmat, size_t(c->NS) * c->NS))) return bail(rc);
  if (cudaMemcpy(c->hmat, c->hp.h.data(), sizeof(double) * c->NS * c->NS, cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(fail(DMK_ERR_CUDA, "copy of the hardening matrix failed"));
  switch (c->NS) {
    case 12: c->pc12 = new PhaseConst<12>(); fill_phase_const<12>(c->hp, c->hmat, *c->pc12); break;
    case 18: c->pc18 = new PhaseConst<18>(); fill_phase_const<18>(c->hp, c->hmat, *c->pc18); break;
    case 24: c->pc24 = new PhaseConst<24>(); fill_phase_const<24>(c->hp, c->hmat, *c->pc24); break;
    case 48: c->pc48 = new PhaseConst<48>(); fill_phase_const<48>(c->hp, c->hmat, *c->pc48); break;
  }
  {
    // per-system constants of the Newton loop, staged into shared memory by the pass kernels
    std::vector<SysConst> sys(c->NS);
    for (int i = 0; i < c->NS; ++i) {
      switch (c->NS) {
        case 12: sys[i] = make_sys_const<12>(*c->pc12, i); break;
        case 18: sys[i] = make_sys_const<18>(*c->pc18, i); break;
        case 24: sys[i] = make_sys_const<24>(*c->pc24, i); break;
        case 48: sys[i] = make_sys_const<48>(*c->pc48, i); break;
      }
    }
    if (cudaMalloc(&c->sysc, sizeof(SysConst) * c->NS) != cudaSuccess ||
        cudaMemcpy(c->sysc, sys.data(), sizeof(SysConst) * c->NS, cudaMemcpyHostToDevice) != cudaSuccess)
      return bail(fail(DMK_ERR_CUDA, "copy of the per-system constants failed"));
    switch (c->NS) {
      case 12: c->pc12->sys = c->sysc; break;
      case 18: c->pc18->sys = c->sysc; break;
      case 24: c->pc24->sys = c->sysc; break;
      case 48: c->pc48->sys = c->sysc; break;
    }
  }

  const int NST = 2 * c->NS;
  const int64_t plane = int64_t(cells[0] / 2 + 1) * cells[1] * cells[2];
  const int64_t nvec = (c->solver == 1 ? 18 : 9) * N;   // solution vector: F, or [F; F_tau]
  if ((rc = dalloc(&c->Fsol, nvec)) || (rc = dalloc(&c->r, nvec)) || (rc = dalloc(&c->F, 9 * N)) ||
      (rc = dalloc(&c->F0, 9 * N)) || (rc = dalloc(&c->Fp, 9 * N)) || (rc = dalloc(&c->Fp0, 9 * N)) ||
      (rc = dalloc(&c->Lp, 9 * N)) || (rc = dalloc(&c->Lp0, 9 * N)) || (rc = dalloc(&c->S, 6 * N)) ||
      (rc = dalloc(&c->S0, 6 * N)) || (rc = dalloc(&c->Fe, 9 * N)) || (rc = dalloc(&c->P, 9 * N)) ||
      (rc = dalloc(&c->Pnew, 9 * N)) || (rc = dalloc(&c->Flast, 9 * N)) || (rc = dalloc(&c->Fdot, 9 * N)) ||
      (rc = dalloc(&c->state, NST * N)) || (rc = dalloc(&c->state0, NST * N)) ||
      (rc = dalloc(&c->spec, 2 * 9 * plane)) ||
      (rc = dalloc(&c->partials, 9 * (size_t)nblocks_const(c))) || (rc = dalloc(&c->sums, 16)) ||
      (rc = dalloc(&c->div_partials, (size_t)gamma_div_blocks(cells[0], cells[1], cells[2]))) ||
      (rc = dalloc(&c->status, 1)) || (rc = dalloc(&c->iter, 4 * N)) || (rc = dalloc(&c->counters, 4)) ||
      (rc = dalloc(&c->sc, 1)) || (rc = dalloc(&c->tan_out, 245)) || (rc = dalloc(&c->tan_idx, 2)) ||
      (rc = dalloc(&c->pw, pass_work_doubles(N, c->NS))) || (rc = dalloc(&c->pctl, 6 * size_t(N))) ||
      (rc = dalloc(&c->dot0, size_t(NST) * N)) ||
      (rc = dalloc(&c->pcount, 2 * PASS_CHUNKS)) || (rc = dalloc(&c->xp, 3 * size_t(N))) ||
      (rc = dalloc(&c->xn, 3 * size_t(node_count(c)))) || (rc = dalloc(&c->favg, 9)))
    return bail(rc);
  // a chunk of at least 65536 voxels keeps a pass kernel wide enough to be worth its own stream
  c->nchunks = int(std::max<int64_t>(1, std::min<int64_t>(PASS_CHUNKS, N / 65536)));
  // voxel lists for every chunk count (the autotuner and dmk_set_tuning change it): chunk h of K
  // chunks holds at most ceil(N / K) voxels and exists for K > h, so its lists hold ceil(N / (h + 1))
  for (int h = 0; h < PASS_CHUNKS; ++h) {
    const size_t len = size_t((N + h) / (h + 1));
    if ((rc = dalloc(&c->plist[h][0], len)) || (rc = dalloc(&c->plist[h][1], len))) return bail(rc);
  }
  if (cudaMallocHost(reinterpret_cast<void**>(&c->hcount), PASS_CHUNKS * sizeof(int)) != cudaSuccess) {
    c->hcount = nullptr;
    return bail(fail(DMK_ERR_CUDA, "cudaMallocHost failed"));
  }
  if (cudaMallocHost(reinterpret_cast<void**>(&c->tan_host), 247 * sizeof(double)) != cudaSuccess) {
    c->tan_host = nullptr;
    return bail(fail(DMK_ERR_CUDA, "cudaMallocHost failed"));
  }
  if (precision == DMK_PRECISION_MIXED)
    if ((rc = dalloc(&c->specf, 2 * 9 * plane)) || (rc = dalloc(&c->Pf, 9 * N))) return bail(rc);
  if (c->solver == 1) {
    c->Ftau = c->Fsol + 9 * N;
    if ((rc = dalloc(&c->Ftau_last, 9 * N)) || (rc = dalloc(&c->Ftau_dot, 9 * N)) || (rc = dalloc(&c->Feval, 9 * N)) ||
        (rc = dalloc(&c->curl_partials, (size_t)gamma_div_blocks(cells[0], cells[1], cells[2]))))
      return bail(rc);
  }
  c->tan_blocks = dPdF_blocks(N);
  if ((rc = dalloc(&c->tan.partials, 81 * (size_t)c->tan_blocks)) || (rc = dalloc(&c->tan.nmax, c->tan_blocks)) ||
      (rc = dalloc(&c->tan.nmin, c->tan_blocks)) || (rc = dalloc(&c->tan.norms, N)) ||
      (rc = dalloc(&c->tan.l2, size_t(tangent_reduce_doubles()))) || (rc = dalloc(&c->tan.planes, 81 * size_t(N))))
    return bail(rc);
  if (num->snes_type == 1) {
    c->aa_m = std::max(1, std::min(num->anderson_m, AA_MAX));
    // grid-stride blocks of the Anderson kernels: 8 per SM, fewer for smaller fields (at least 8
    // elements per thread, so that a batch of small RVEs launches few idle blocks)
    c->aa_blocks = int(std::max<int64_t>(1, std::min<int64_t>(int64_t(c->nsm) * 8, (nvec + 2047) / 2048)));
    if ((rc = dalloc(&c->aa_dX, size_t(c->aa_m) * nvec)) || (rc = dalloc(&c->aa_dR, size_t(c->aa_m) * nvec)) ||
        (rc = dalloc(&c->aa_Rprev, nvec)) || (rc = dalloc(&c->aa_partials, size_t(c->aa_blocks) * 2 * AA_CHUNK_HOST)) ||
        (rc = dalloc(&c->aa_out, 4 * AA_MAX)))
      return bail(rc);
  } else if (num->snes_type != 0) {
    return bail(fail(DMK_ERR_CONFIG, "snes_type must be 0 (Richardson) or 1 (Anderson)"));
  }
  if ((rc = make_plans(c))) return bail(rc);

  // mechanical_init (phase_mechanical.f90:249-266), computed per voxel on the device
  {
    int* dmat = nullptr;
    double *dq = nullptr, *dxi = nullptr;
    if ((rc = dalloc(&dmat, N)) || (rc = dalloc(&dq, 4 * size_t(n_materials))) || (rc = dalloc(&dxi, c->NS))) {
      cudaFree(dmat); cudaFree(dq); cudaFree(dxi);
      return bail(rc);
    }
    cudaError_t e = cudaMemcpyAsync(dmat, materialAt, sizeof(int) * N, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dq, quaternions, sizeof(double) * 4 * n_materials, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dxi, c->hp.xi0.data(), sizeof(double) * c->NS, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
      e = launch_init_state(dmat, dq, dxi, c->NS, N, c->F, c->F0, c->Fsol, c->Flast, c->Fp, c->Fp0, c->Fe, c->state,
                            c->state0, c->stream);
    for (double* p : {c->Lp, c->Lp0, c->P, c->Pnew, c->Fdot, c->r})
      if (e == cudaSuccess) e = cudaMemsetAsync(p, 0, sizeof(double) * 9 * N, c->stream);
    for (double* p : {c->S, c->S0})
      if (e == cudaSuccess) e = cudaMemsetAsync(p, 0, sizeof(double) * 6 * N, c->stream);
    if (c->solver == 1 && e == cudaSuccess) e = cudaMemsetAsync(c->Ftau_dot, 0, sizeof(double) * 9 * N, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->counters, 0, 4 * sizeof(unsigned long long), c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(dmat); cudaFree(dq); cudaFree(dxi);
    if (e != cudaSuccess) return bail(fail(DMK_ERR_CUDA, std::string("init: ") + cudaGetErrorString(e)));
  }
  // solver module state (grid_mech_spectral_basic.f90:30-45)
  for (int k = 0; k < 9; ++k) {
    c->F_aim[k] = c->F_aim_lastinc[k] = (k % 4 == 0) ? 1.0 : 0.0;
    c->F_aimDot[k] = c->P_aim[k] = c->P_av[k] = 0.0;
    c->stress_mask[k] = 1;
  }
  std::fill(c->C_volAvg, c->C_volAvg + 81, 0.0);
  std::fill(c->C_volAvgLastInc, c->C_volAvgLastInc + 81, 0.0);
  std::fill(c->C_minMaxAvg, c->C_minMaxAvg + 81, 0.0);
  std::fill(c->C_minMaxAvgLastInc, c->C_minMaxAvgLastInc + 81, 0.0);
  std::fill(c->Scomp, c->Scomp + 81, 0.0);
  c->q_rot[0] = 1.0; c->q_rot[1] = c->q_rot[2] = c->q_rot[3] = 0.0;
  if ((rc = upload_scalars(c, true))) return bail(rc);

  // staging buffer of the field transfers, allocated here so that no transfer allocates
  if ((rc = ensure_scratch(c, 9))) return bail(rc);
  // discretization_init: current coordinates = undeformed coordinates (IPcoordinates0, nodes0)
  {
    const double step[3] = {geomSize[0] / cells[0], geomSize[1] / cells[1], geomSize[2] / cells[2]};
    cudaError_t e = launch_coords(nullptr, nullptr, c->cells, step, c->wgt, c->xp, c->xn, c->stream);
    if (e != cudaSuccess) return bail(fail(DMK_ERR_CUDA, std::string("init coordinates: ") + cudaGetErrorString(e)));
  }
  // grid_mechanical_spectral_basic_init: constitutive response at F = I, dt = 0, then updateGamma
  int st = 0;
  if ((rc = response(c, 0.0, &st))) return bail(rc);
  update_gamma_host(c, c->C_minMaxAvg);
  if (c->solver == 1) {
    if ((rc = set_polarization_scale(c))) return bail(rc);
    // F_tau = F_tau_lastinc = 2 F with F = I (grid_mech_spectral_polarization.f90:250-253)
    std::vector<double> two(9 * size_t(N));
    for (int64_t v = 0; v < N; ++v)
      for (int k = 0; k < 9; ++k) two[size_t(k) * N + v] = (k % 4 == 0) ? 2.0 : 0.0;
    if (cudaMemcpy(c->Ftau, two.data(), sizeof(double) * two.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->Ftau_last, two.data(), sizeof(double) * two.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return bail(fail(DMK_ERR_CUDA, "init: F_tau upload failed"));
  }
  *out = c;
  return 0;
}

int dmk_mech_forward(dmk_ctx* c, int cutBack, int guess, double dt, double dt_old, double t_remaining,
                     const dmk_bc* def, const dmk_bc* stress, const double q_rot[4]) {
  if (!c || !def || !stress || !q_rot) return fail(DMK_ERR_ARG, "null argument");
  if (cutBack) {
    std::memcpy(c->C_volAvg, c->C_volAvgLastInc, sizeof c->C_volAvg);
    std::memcpy(c->C_minMaxAvg, c->C_minMaxAvgLastInc, sizeof c->C_minMaxAvg);
  } else {
    std::memcpy(c->C_volAvgLastInc, c->C_volAvg, sizeof c->C_volAvg);
    std::memcpy(c->C_minMaxAvgLastInc, c->C_minMaxAvg, sizeof c->C_minMaxAvg);
    for (int k = 0; k < 9; ++k)
      c->F_aimDot[k] = guess ? (stress->mask[k] ? 0.0 : (c->F_aim[k] - c->F_aim_lastinc[k]) / dt_old) : 0.0;
    std::memcpy(c->F_aim_lastinc, c->F_aim, sizeof c->F_aim);
    double m[9];
    for (int k = 0; k < 9; ++k) m[k] = def->mask[k] ? 0.0 : def->values[k];
    if (def->type == 1) {                      // L: F_aimDot += L F_aim_lastinc
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          double s = 0.0;
          for (int k = 0; k < 3; ++k) s += m[i + 3 * k] * c->F_aim_lastinc[k + 3 * j];
          c->F_aimDot[i + 3 * j] += s;
        }
    } else if (def->type == 2) {               // dot_F
      for (int k = 0; k < 9; ++k) c->F_aimDot[k] += m[k];
    } else if (def->type == 3) {               // F at end of load case
      for (int k = 0; k < 9; ++k)
        c->F_aimDot[k] += def->mask[k] ? 0.0 : (def->values[k] - c->F_aim_lastinc[k]) / t_remaining;
    } else {
      return fail(DMK_ERR_ARG, "deformation BC type must be L, dot_F or F");
    }
  }
  double avRate[9], aim[9];
  h_rot33(q_rot, c->F_aimDot, avRate, true);
  for (int k = 0; k < 9; ++k) c->F_aim[k] = c->F_aim_lastinc[k] + c->F_aimDot[k] * dt;
  if (stress->type == 4)
    for (int k = 0; k < 9; ++k) c->P_aim[k] = c->P_aim[k] + (stress->mask[k] ? 0.0 : (stress->values[k] - c->P_aim[k]) / t_remaining) * dt;
  if (stress->type == 5)
    for (int k = 0; k < 9; ++k) c->P_aim[k] = c->P_aim[k] + (stress->mask[k] ? 0.0 : stress->values[k]) * dt;
  h_rot33(q_rot, c->F_aim, aim, true);
  for (int k = 0; k < 9; ++k) c->stress_mask[k] = stress->mask[k] ? 1 : 0;
  std::memcpy(c->q_rot, q_rot, sizeof c->q_rot);
  c->dt = dt;
  int rc = upload_scalars(c, true, avRate, aim);
  if (rc) return rc;
  const double* dsc = reinterpret_cast<const double*>(c->sc);
  CKL(launch_forward(c->Fsol, c->Flast, c->Fdot, c->N, cutBack, guess, dt, dt_old,
                    dsc + offsetof(SolverScalars, avRate) / sizeof(double), c->partials, c->sums, c->wgt,
                    dsc + offsetof(SolverScalars, aim_fwd) / sizeof(double), c->stream));
  c->launches += 2;   // forward, partial reduction, shift
  if (c->solver == 1) {
    CKL(launch_pol_forward_tau(c->Fsol, c->Ftau, c->Ftau_last, c->Ftau_dot, c->N, cutBack, guess, dt, dt_old,
                              dsc + offsetof(SolverScalars, avRate) / sizeof(double), c->polc, c->stream));
  }
  return 0;
}

int dmk_mech_solution(dmk_ctx* c, dmk_solution_state* out) {
  if (!c || !out) return fail(DMK_ERR_ARG, "null argument");
  int rc = solution_prepare(c);
  if (rc) return rc;
  if (c->solver == 1) return solution_polarization(c, out);
  const int snes_max_its = c->num.snes_max_it > 0 ? c->num.snes_max_it : 50;   // PETSc -snes_max_it (default 50)
  const bool mixed = c->precision == DMK_PRECISION_MIXED;
  const bool anderson = c->num.snes_type == 1;
  const int m = c->aa_m;
  const int64_t n9 = 9 * c->N;
  const int nspec = gamma_div_blocks(c->cells[0], c->cells[1], c->cells[2]);
  bool fp32 = mixed;
  int evals = 0, reason = 0;
  SolverScalars hs;
  int count = 0;                        // Anderson history pairs created so far
  std::vector<double> G(size_t(m > 0 ? m : 1) * (m > 0 ? m : 1), 0.0), bvec;
  std::vector<int> slots_b;             // slots that bvec refers to (oldest -> newest)
  double dots[4 * AA_MAX];
  int new_slot = -1;

  // One residual evaluation at the current Fsol (apply: fuse F <- F - r into the sweep).
  // Leaves r (FP64) and the convergence decision in hs; with Anderson also the inner
  // products of the new residual with the history.
  auto evaluate = [&](int apply) -> int {
    int st = 0;
    if (int e = evaluate_constitutive(c, c->dt, apply ? c->r : nullptr, apply, &st)) return e;
    ++evals;
    CKL(launch_aim(c->sc, c->partials, nblocks_const(c), c->wgt, 1, c->stream));
    for (int pass = 0; pass < 2; ++pass) {
      const bool use32 = fp32 && pass == 0;
      CK(cudaEventRecord(c->ev[2], c->stream));
      if (int e = spectral_pass(c, use32, 1, 1, use32 ? static_cast<void*>(c->Pf) : static_cast<void*>(c->r))) return e;
      if (use32) CKL(launch_to_double(c->Pf, c->r, n9, c->nsm, c->stream));
      CKL(launch_converge(c->sc, c->div_partials, nspec, c->wgt, c->status, c->nm2, pass == 0 ? 1 : 0, c->stream));
      CK(cudaEventRecord(c->ev[3], c->stream));
      int nsl = 0;
      if (anderson && new_slot >= 0) {
        slots_b.clear();
        const int mk = std::min(count, m);
        for (int q = count - mk; q < count; ++q) slots_b.push_back(q % m);
        nsl = int(slots_b.size());
        CKL(launch_aa_dots(c->r, c->aa_Rprev, c->aa_dR, n9, new_slot, slots_b.data(), nsl, c->aa_partials,
                          c->aa_blocks, c->aa_out, c->stream));
        c->launches += 2 * ((nsl + AA_CHUNK_HOST - 1) / AA_CHUNK_HOST) - 1;   // dots + reduce per chunk
        CK(cudaMemcpyAsync(dots, c->aa_out, sizeof(double) * 2 * AA_CHUNK_HOST * ((nsl + AA_CHUNK_HOST - 1) / AA_CHUNK_HOST),
                           cudaMemcpyDeviceToHost, c->stream));
      }
      CK(cudaMemcpyAsync(&hs, c->sc, sizeof hs, cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]));
      c->last_ms[1] += ms;
      if (nsl > 0) {
        bvec.assign(nsl, 0.0);
        for (int q = 0; q < nsl; ++q) {
          const int ch = q / AA_CHUNK_HOST, k = q % AA_CHUNK_HOST;
          const double g = dots[ch * 2 * AA_CHUNK_HOST + k], b = dots[ch * 2 * AA_CHUNK_HOST + AA_CHUNK_HOST + k];
          G[size_t(new_slot) * m + slots_b[q]] = G[size_t(slots_b[q]) * m + new_slot] = g;
          bvec[q] = b;
        }
      }
      // FP32 spectral iterations that meet the tolerance get a correction sweep in FP64
      // on the same stress field; its residual and decision replace the FP32 ones.
      if (use32 && hs.reason == 1) { fp32 = false; continue; }
      break;
    }
    return 0;
  };

  if ((rc = evaluate(0))) return rc;
  if (anderson) {
    // b for the first Anderson step is empty (plain Richardson step)
    bvec.clear();
    slots_b.clear();
  }
  reason = hs.reason;
  for (int it = 1; reason == 0; ++it) {
    if (it > snes_max_its) { reason = -1; break; }
    if (!anderson) {
      if ((rc = evaluate(1))) return rc;
    } else {
      std::vector<double> gam = anderson_coefficients(G, m, slots_b, bvec);
      new_slot = count % m;
      CKL(launch_aa_update(c->Fsol, c->r, c->aa_Rprev, c->aa_dX, c->aa_dR, n9, new_slot, slots_b.data(), gam.data(),
                          int(slots_b.size()), c->aa_blocks, c->stream));
      ++count;
      if ((rc = evaluate(0))) return rc;
    }
    reason = hs.reason;
  }
  return solution_finish(c, hs.F_aim, hs.P_av, hs.totalIter, hs.err_div, hs.err_BC, reason, evals, out);
}

int dmk_materialpoint_forward(dmk_ctx* c) {
  if (!c) return fail(DMK_ERR_ARG, "null argument");
  const size_t b9 = sizeof(double) * 9 * c->N, b6 = sizeof(double) * 6 * c->N, bs = sizeof(double) * 2 * c->NS * c->N;
  CK(cudaMemcpyAsync(c->F0, c->F, b9, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(c->Fp0, c->Fp, b9, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(c->Lp0, c->Lp, b9, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(c->S0, c->S, b6, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(c->state0, c->state, bs, cudaMemcpyDeviceToDevice, c->stream));
  c->dot0_valid = false;                                   // new increment-start values
  return 0;
}

// omega_plastic of the restart data: per voxel xi then gamma of the active systems (sizeState = 2 Ns)
static int state_to_host(dmk_ctx* c, const double* dev_state, double* host) {
  const int na = c->NSact;
  if (na == c->NS) return d2h_planes(c, dev_state, host, 2 * na);
  std::vector<double> xi(size_t(na) * c->N), ga(size_t(na) * c->N);
  if (int rc = d2h_planes(c, dev_state, xi.data(), na)) return rc;
  if (int rc = d2h_planes(c, dev_state + int64_t(c->NS) * c->N, ga.data(), na)) return rc;
  for (int64_t v = 0; v < c->N; ++v)
    for (int s = 0; s < na; ++s) {
      host[v * 2 * na + s] = xi[v * na + s];
      host[v * 2 * na + na + s] = ga[v * na + s];
    }
  return 0;
}
static int state_from_host(dmk_ctx* c, const double* host, double* dev_state) {
  const int na = c->NSact;
  if (na == c->NS) return h2d_planes(c, host, dev_state, 2 * na);
  std::vector<double> xi(size_t(na) * c->N), ga(size_t(na) * c->N);
  for (int64_t v = 0; v < c->N; ++v)
    for (int s = 0; s < na; ++s) {
      xi[v * na + s] = host[v * 2 * na + s];
      ga[v * na + s] = host[v * 2 * na + na + s];
    }
  // pageable sources: each copy has left the host buffer when cudaMemcpyAsync returns
  if (int rc = h2d_planes(c, xi.data(), dev_state, na)) return rc;
  return h2d_planes(c, ga.data(), dev_state + int64_t(c->NS) * c->N, na);
}

int dmk_restart_write(dmk_ctx* c, dmk_restart* r) {
  if (!c || !r || !r->F || !r->F_lastinc || !r->F_phase || !r->F_p || !r->L_p || !r->omega_plastic)
    return fail(DMK_ERR_ARG, "null argument");
  int rc;
  if ((rc = d2h_planes(c, c->Fsol, r->F, 9)) || (rc = d2h_planes(c, c->Flast, r->F_lastinc, 9)) ||
      (rc = d2h_planes(c, c->F, r->F_phase, 9)) || (rc = d2h_planes(c, c->Fp, r->F_p, 9)) ||
      (rc = d2h_planes(c, c->Lp, r->L_p, 9)) || (rc = state_to_host(c, c->state, r->omega_plastic)))
    return rc;
  std::memcpy(r->P_aim, c->P_aim, sizeof r->P_aim);
  std::memcpy(r->F_aim, c->F_aim, sizeof r->F_aim);
  std::memcpy(r->F_aim_lastinc, c->F_aim_lastinc, sizeof r->F_aim_lastinc);
  std::memcpy(r->F_aimDot, c->F_aimDot, sizeof r->F_aimDot);
  std::memcpy(r->C_volAvg, c->C_volAvg, sizeof r->C_volAvg);
  std::memcpy(r->C_volAvgLastInc, c->C_volAvgLastInc, sizeof r->C_volAvgLastInc);
  std::memcpy(r->C_minMaxAvg, c->C_gamma, sizeof r->C_minMaxAvg);
  if (c->solver == 1) {   // grid_mech_spectral_polarization_restartWrite (:412-415)
    if (!r->F_tau || !r->F_tau_lastinc) return fail(DMK_ERR_ARG, "F_tau / F_tau_lastinc buffers are required");
    if ((rc = d2h_planes(c, c->Ftau, r->F_tau, 9)) || (rc = d2h_planes(c, c->Ftau_last, r->F_tau_lastinc, 9))) return rc;
  }
  return 0;
}

int dmk_restart_read(dmk_ctx* c, const dmk_restart* r) {
  if (!c || !r || !r->F || !r->F_lastinc || !r->F_phase || !r->F_p || !r->L_p || !r->omega_plastic)
    return fail(DMK_ERR_ARG, "null argument");
  const size_t b9 = sizeof(double) * 9 * c->N, bs = sizeof(double) * 2 * c->NS * c->N;
  int rc;
  // mechanical_restartRead: the converged phase state; the current values follow at the sweep
  if ((rc = h2d_planes(c, r->F_phase, c->F0, 9)) || (rc = h2d_planes(c, r->F_p, c->Fp0, 9)) ||
      (rc = h2d_planes(c, r->L_p, c->Lp0, 9)) || (rc = state_from_host(c, r->omega_plastic, c->state0)) ||
      (rc = h2d_planes(c, r->F, c->Fsol, 9)) || (rc = h2d_planes(c, r->F_lastinc, c->Flast, 9)))
    return rc;
  if (c->solver == 1) {   // grid_mech_spectral_polarization.f90:236-245
    if (!r->F_tau || !r->F_tau_lastinc) return fail(DMK_ERR_ARG, "F_tau / F_tau_lastinc buffers are required");
    if ((rc = h2d_planes(c, r->F_tau, c->Ftau, 9)) || (rc = h2d_planes(c, r->F_tau_lastinc, c->Ftau_last, 9))) return rc;
  }
  CK(cudaMemcpyAsync(c->F, c->F0, b9, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(c->Fp, c->Fp0, b9, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(c->Lp, c->Lp0, b9, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(c->state, c->state0, bs, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemsetAsync(c->S0, 0, sizeof(double) * 6 * c->N, c->stream));
  c->dot0_valid = false;
  CK(cudaMemsetAsync(c->S, 0, sizeof(double) * 6 * c->N, c->stream));
  // solver module state (grid_mech_spectral_basic.f90:203-208)
  std::memcpy(c->P_aim, r->P_aim, sizeof c->P_aim);
  std::memcpy(c->F_aim, r->F_aim, sizeof c->F_aim);
  std::memcpy(c->F_aim_lastinc, r->F_aim_lastinc, sizeof c->F_aim_lastinc);
  std::memcpy(c->F_aimDot, r->F_aimDot, sizeof c->F_aimDot);
  if ((rc = upload_scalars(c, true))) return rc;
  // constitutive response at the loaded F, dt = 0 (:216-221), then the stored stiffnesses (:224-235)
  int st = 0;
  if ((rc = response(c, 0.0, &st))) return rc;
  std::memcpy(c->C_volAvg, r->C_volAvg, sizeof c->C_volAvg);
  std::memcpy(c->C_volAvgLastInc, r->C_volAvgLastInc, sizeof c->C_volAvgLastInc);
  std::memcpy(c->C_minMaxAvg, r->C_minMaxAvg, sizeof c->C_minMaxAvg);
  update_gamma_host(c, c->C_minMaxAvg);
  if (c->solver == 1)
    if ((rc = set_polarization_scale(c))) return rc;
  return 0;
}

// grid_mechanical_spectral_basic_updateCoords -> utilities_updateCoords
// (spectral_utilities.f90:857-968) on the solver's F field: D2Z of F, u_hat = F_hat xi / (conj(-xi) . xi),
// Z2D of u into the staging buffer, then cell-centre and node coordinates.
int dmk_mech_update_coords(dmk_ctx* c) {
  if (!c) return fail(DMK_ERR_ARG, "null argument");
  if (int rc = ensure_scratch(c, 3)) return rc;
  const double L[3] = {c->geom[0], c->geom[1], c->geom[2]};
  const double step[3] = {c->geom[0] / c->cells[0], c->geom[1] / c->cells[1], c->geom[2] / c->cells[2]};
  CKF(cufftExecD2Z(c->plan_fwd, c->Fsol, reinterpret_cast<cufftDoubleComplex*>(c->spec)));
  CKL(launch_coords_spec(c->spec, c->cells[0], c->cells[1], c->cells[2], L, c->wgt, c->favg, c->gc.derivative,
                         c->stream));
  CKF(cufftExecZ2D(c->plan_vec_bwd, reinterpret_cast<cufftDoubleComplex*>(c->spec), c->scratch));
  CKL(launch_coords(c->scratch, c->favg, c->cells, step, c->wgt, c->xp, c->xn, c->stream));
  c->launches += 2;   // each launcher above issues two kernels
  return 0;
}

int dmk_get_coords(dmk_ctx* c, double* ip, double* nodes) {
  if (!c) return fail(DMK_ERR_ARG, "null argument");
  if (ip) CK(cudaMemcpyAsync(ip, c->xp, sizeof(double) * 3 * c->N, cudaMemcpyDeviceToHost, c->stream));
  if (nodes) CK(cudaMemcpyAsync(nodes, c->xn, sizeof(double) * 3 * node_count(c), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int dmk_field_size(dmk_ctx* c, int field) {
  if (!c) return fail(DMK_ERR_ARG, "null argument");
  if (field == DMK_FIELD_XI_SL || field == DMK_FIELD_GAMMA_SL) return c->NSact;
  if (field == DMK_FIELD_O) return 4;
  if (field >= 0 && field <= DMK_FIELD_F_SOLVER) return 9;
  if ((field == DMK_FIELD_F_TAU || field == DMK_FIELD_F_TAU_LASTINC) && c->solver == 1) return 9;
  return fail(DMK_ERR_ARG, "unknown field");
}

int dmk_get_field(dmk_ctx* c, int field, double* host) {
  if (!c || !host) return fail(DMK_ERR_ARG, "null argument");
  const int64_t N = c->N;
  switch (field) {
    case DMK_FIELD_F: return d2h_planes(c, c->F, host, 9);
    case DMK_FIELD_P: return d2h_planes(c, c->P, host, 9);
    case DMK_FIELD_FE: return d2h_planes(c, c->Fe, host, 9);
    case DMK_FIELD_FP: return d2h_planes(c, c->Fp, host, 9);
    case DMK_FIELD_LP: return d2h_planes(c, c->Lp, host, 9);
    case DMK_FIELD_F_LASTINC: return d2h_planes(c, c->Flast, host, 9);
    case DMK_FIELD_F_SOLVER: return d2h_planes(c, c->Fsol, host, 9);
    case DMK_FIELD_F_TAU:
      if (c->solver != 1) break;
      return d2h_planes(c, c->Ftau, host, 9);
    case DMK_FIELD_F_TAU_LASTINC:
      if (c->solver != 1) break;
      return d2h_planes(c, c->Ftau_last, host, 9);
    case DMK_FIELD_XI_SL: return d2h_planes(c, c->state, host, c->NSact);
    case DMK_FIELD_GAMMA_SL: return d2h_planes(c, c->state + int64_t(c->NS) * N, host, c->NSact);
    case DMK_FIELD_S:
      if (int rc = ensure_scratch(c, 9)) return rc;
      CKL(launch_sym6_to9(c->S, c->scratch, N, c->stream));
      CK(cudaMemcpyAsync(host, c->scratch, sizeof(double) * 9 * N, cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      return 0;
    case DMK_FIELD_O: {
      if (int rc = ensure_scratch(c, 4)) return rc;
      CK(cudaMemsetAsync(c->status, 0, sizeof(int), c->stream));
      CKL(launch_orientations(c->Fe, N, c->scratch, c->status, c->stream));
      int bad = 0;
      CK(cudaMemcpyAsync(host, c->scratch, sizeof(double) * 4 * N, cudaMemcpyDeviceToHost, c->stream));
      CK(cudaMemcpyAsync(&bad, c->status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      if (bad) return fail(DMK_ERR_STATE, "orientation: the rotational part of Fe is not a rotation (|det - 1| > 1e-5)");
      return 0;
    }
    case DMK_FIELD_FI:
    case DMK_FIELD_LI:
      for (int64_t v = 0; v < N; ++v)
        for (int k = 0; k < 9; ++k) host[v * 9 + k] = (field == DMK_FIELD_FI && k % 4 == 0) ? 1.0 : 0.0;
      return 0;
  }
  return fail(DMK_ERR_ARG, "unknown field");
}

int dmk_set_field(dmk_ctx* c, int field, const double* host) {
  if (!c || !host) return fail(DMK_ERR_ARG, "null argument");
  int rc = 0;
  switch (field) {
    case DMK_FIELD_F_SOLVER: rc = h2d_planes(c, host, c->Fsol, 9); break;
    case DMK_FIELD_F_LASTINC: rc = h2d_planes(c, host, c->Flast, 9); break;
    case DMK_FIELD_F_TAU:
    case DMK_FIELD_F_TAU_LASTINC:
      if (c->solver != 1) return fail(DMK_ERR_ARG, "F_tau exists for the polarization solver only");
      rc = h2d_planes(c, host, field == DMK_FIELD_F_TAU ? c->Ftau : c->Ftau_last, 9);
      break;
    default: return fail(DMK_ERR_ARG, "field is not settable");
  }
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int dmk_get_aims(dmk_ctx* c, double F_aim[9], double F_aim_lastinc[9], double F_aimDot[9], double P_aim[9],
                 double C_volAvg[81], double C_volAvgLastInc[81], double C_minMaxAvg[81]) {
  if (!c) return fail(DMK_ERR_ARG, "null argument");
  if (F_aim) std::memcpy(F_aim, c->F_aim, 9 * sizeof(double));
  if (F_aim_lastinc) std::memcpy(F_aim_lastinc, c->F_aim_lastinc, 9 * sizeof(double));
  if (F_aimDot) std::memcpy(F_aimDot, c->F_aimDot, 9 * sizeof(double));
  if (P_aim) std::memcpy(P_aim, c->P_aim, 9 * sizeof(double));
  if (C_volAvg) std::memcpy(C_volAvg, c->C_volAvg, 81 * sizeof(double));
  if (C_volAvgLastInc) std::memcpy(C_volAvgLastInc, c->C_volAvgLastInc, 81 * sizeof(double));
  if (C_minMaxAvg) std::memcpy(C_minMaxAvg, c->C_minMaxAvg, 81 * sizeof(double));
  return 0;
}

int dmk_constitutive_response(dmk_ctx* c, const double* F, double dt, double* P, double P_av[9], double C_volAvg[81],
                              double C_minMaxAvg[81], int* status) {
  if (!c || !F || !P || !status) return fail(DMK_ERR_ARG, "null argument");
  int rc = h2d_planes(c, F, c->Fsol, 9);
  if (rc) return rc;
  const double q0[4] = {1.0, 0.0, 0.0, 0.0};
  std::memcpy(c->q_rot, q0, sizeof q0);
  if ((rc = upload_scalars(c, true))) return rc;
  c->iter_enabled = true;
  rc = response(c, dt, status);
  c->iter_enabled = false;
  if (rc) return rc;
  if ((rc = d2h_planes(c, c->P, P, 9))) return rc;
  if (P_av) std::memcpy(P_av, c->P_av, 9 * sizeof(double));
  if (C_volAvg) std::memcpy(C_volAvg, c->C_volAvg, 81 * sizeof(double));
  if (C_minMaxAvg) std::memcpy(C_minMaxAvg, c->C_minMaxAvg, 81 * sizeof(double));
  return 0;
}

int dmk_update_gamma(dmk_ctx* c, const double C[81]) {
  if (!c || !C) return fail(DMK_ERR_ARG, "null argument");
  update_gamma_host(c, C);
  return 0;
}

int dmk_gamma_convolution(dmk_ctx* c, double* field, const double aim[9]) {
  if (!c || !field || !aim) return fail(DMK_ERR_ARG, "null argument");
  int rc = h2d_planes(c, field, c->P, 9);
  if (rc) return rc;
  CK(cudaMemcpyAsync(reinterpret_cast<char*>(c->sc) + offsetof(SolverScalars, aim_rot), aim, 9 * sizeof(double),
                     cudaMemcpyHostToDevice, c->stream));
  if ((rc = spectral_pass(c, false, 1, 0, c->r))) return rc;
  return d2h_planes(c, c->r, field, 9);
}

// utilities_curlRMS (spectral_utilities.f90:695-757) of a host tensor field; the solver's spectrum
// and staging buffers are used as scratch.
int dmk_curl_rms(dmk_ctx* c, const double* F, double* out) {
  if (!c || !F || !out) return fail(DMK_ERR_ARG, "null argument");
  if (int rc = h2d_planes(c, F, c->r, 9)) return rc;
  CKF(cufftExecD2Z(c->plan_fwd, c->r, reinterpret_cast<cufftDoubleComplex*>(c->spec)));
  const double L[3] = {c->geom[0], c->geom[1], c->geom[2]};
  CKL(launch_curl(c->spec, c->cells[0], c->cells[1], c->cells[2], L, c->gc.rescale, c->gc.derivative,
                    c->div_partials, c->stream));
  const int nb = gamma_div_blocks(c->cells[0], c->cells[1], c->cells[2]);
  std::vector<double> h(nb);
  CK(cudaMemcpyAsync(h.data(), c->div_partials, sizeof(double) * nb, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  double s = 0.0;
  for (double x : h) s += x;
  *out = std::sqrt(s) * c->wgt * (c->cells[0] == 1 ? 0.5 : 1.0);
  return 0;
}

int dmk_divergence_rms(dmk_ctx* c, const double* P, double* out) {
  if (!c || !P || !out) return fail(DMK_ERR_ARG, "null argument");
  int rc = h2d_planes(c, P, c->P, 9);
  if (rc) return rc;
  if ((rc = spectral_pass(c, false, 0, 1, nullptr))) return rc;
  const int nb = gamma_div_blocks(c->cells[0], c->cells[1], c->cells[2]);
  std::vector<double> h(nb);
  CK(cudaMemcpyAsync(h.data(), c->div_partials, sizeof(double) * nb, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  double s = 0.0;
  for (double x : h) s += x;
  double r = std::sqrt(s) * c->wgt;
  if (c->cells[0] == 1) r *= 0.5;
  *out = r;
  return 0;
}

int dmk_dPdF(dmk_ctx* c, double dt, double* dPdF) {
  if (!c || !dPdF) return fail(DMK_ERR_ARG, "null argument");
  int rc = ensure_scratch(c, 81);
  if (rc) return rc;
  rc = evaluate_tangent(c, dt, c->scratch);
  if (rc) return rc;
  CK(cudaMemcpyAsync(dPdF, c->scratch, sizeof(double) * 81 * c->N, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int dmk_get_iteration_counts(dmk_ctx* c, int* out) {
  if (!c || !out) return fail(DMK_ERR_ARG, "null argument");
  std::vector<int> h(4 * c->N);
  CK(cudaMemcpyAsync(h.data(), c->iter, sizeof(int) * 4 * c->N, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int64_t v = 0; v < c->N; ++v)
    for (int k = 0; k < 4; ++k) out[v * 4 + k] = h[k * c->N + v];
  return 0;
}

int dmk_get_counters(dmk_ctx* c, int64_t out[4]) {
  if (!c || !out) return fail(DMK_ERR_ARG, "null argument");
  for (int k = 0; k < 4; ++k) out[k] = c->last_counters[k];
  return 0;
}

int dmk_phase_schmid(const dmk_phase* phase, int sense, double* out) {
  if (!phase || !out || (sense != 1 && sense != -1)) return fail(DMK_ERR_ARG, "invalid argument");
  HostPhase hp;
  std::string err;
  if (build_host_phase(*phase, hp, err)) return fail(DMK_ERR_CONFIG, err);
  const auto& P = sense > 0 ? hp.Ppos : hp.Pneg;
  for (int s = 0; s < hp.Ns; ++s)
    for (int k = 0; k < 9; ++k) out[9 * s + k] = P[s][k];
  return hp.Ns;
}

int dmk_phase_slip_systems(const dmk_phase* phase, int* out) {
  if (!phase || !out) return fail(DMK_ERR_ARG, "invalid argument");
  HostPhase hp;
  std::string err;
  if (build_host_phase(*phase, hp, err)) return fail(DMK_ERR_CONFIG, err);
  const auto m = slip_miller(*phase);
  for (size_t s = 0; s < m.size(); ++s)
    for (int k = 0; k < 6; ++k) out[6 * s + k] = m[s][k];
  return int(m.size());
}

int dmk_phase_interaction(const dmk_phase* phase, double* h) {
  if (!phase || !h) return fail(DMK_ERR_ARG, "invalid argument");
  HostPhase hp;
  std::string err;
  if (build_host_phase(*phase, hp, err)) return fail(DMK_ERR_CONFIG, err);
  std::copy(hp.h.begin(), hp.h.end(), h);
  return hp.Ns;
}

int dmk_get_launches(dmk_ctx* c, int64_t* out) {
  if (!c || !out) return fail(DMK_ERR_ARG, "null argument");
  *out = c->launches;
  return 0;
}

int dmk_timer_start(dmk_ctx* c) {
  if (!c) return fail(DMK_ERR_ARG, "null argument");
  if (!c->tev[0]) { CK(cudaEventCreate(&c->tev[0])); CK(cudaEventCreate(&c->tev[1])); }
  CK(cudaEventRecord(c->tev[0], c->stream));
  return 0;
}

int dmk_timer_stop(dmk_ctx* c, double* ms) {
  if (!c || !ms || !c->tev[0]) return fail(DMK_ERR_ARG, "timer not started");
  CK(cudaEventRecord(c->tev[1], c->stream));
  CK(cudaEventSynchronize(c->tev[1]));
  float f = 0.f;
  CK(cudaEventElapsedTime(&f, c->tev[0], c->tev[1]));
  *ms = f;
  return 0;
}

int dmk_fp64_peak(int device, double* tflops) {
  if (!tflops) return fail(DMK_ERR_ARG, "null argument");
  CK(cudaSetDevice(device));
  int nsm = 0;
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
  const int blocks = nsm * 8, iters = 1 << 16;
  double* sink = nullptr;
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  auto release = [&]() {
    if (sink) cudaFree(sink);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
  };
  if (cudaMalloc(&sink, sizeof(double) * blocks) != cudaSuccess || cudaStreamCreate(&s) != cudaSuccess ||
      cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    release();
    return fail(DMK_ERR_CUDA, "fp64 probe: allocation failed");
  }
  float best = 1e30f;
  cudaError_t e = launch_fp64_probe(sink, blocks, iters, s);           // warm-up
  for (int r = 0; r < 3 && e == cudaSuccess; ++r) {
    e = cudaEventRecord(e0, s);
    if (e == cudaSuccess) e = launch_fp64_probe(sink, blocks, iters, s);
    if (e == cudaSuccess) e = cudaEventRecord(e1, s);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e == cudaSuccess && ms < best) best = ms;
  }
  release();
  if (e != cudaSuccess) return fail(DMK_ERR_CUDA, std::string("fp64 probe: ") + cudaGetErrorString(e));
  *tflops = 2.0 * 8.0 * double(iters) * blocks * 256.0 / (double(best) * 1e-3) / 1e12;
  return 0;
}

int dmk_get_timings(dmk_ctx* c, double out[3]) {
  if (!c || !out) return fail(DMK_ERR_ARG, "null argument");
  for (int k = 0; k < 3; ++k) out[k] = c->last_ms[k];
  return 0;
}

void dmk_destroy(dmk_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (int h = 1; h < PASS_CHUNKS; ++h)
    if (c->cstream[h]) cudaStreamSynchronize(c->cstream[h]);
  for (cufftHandle p : {c->plan_fwd, c->plan_bwd, c->plan_fwd_f, c->plan_bwd_f, c->plan_vec_bwd})
    if (p) cufftDestroy(p);
  for (void* p : {(void*)c->Fsol, (void*)c->r, (void*)c->F, (void*)c->F0, (void*)c->Fp, (void*)c->Fp0, (void*)c->Lp,
                  (void*)c->Lp0, (void*)c->S, (void*)c->S0, (void*)c->Fe, (void*)c->P, (void*)c->Pnew, (void*)c->Flast,
                  (void*)c->Fdot, (void*)c->state, (void*)c->state0, (void*)c->spec, (void*)c->specf, (void*)c->Pf,
                  (void*)c->partials, (void*)c->sums, (void*)c->div_partials, (void*)c->status, (void*)c->iter,
                  (void*)c->counters, (void*)c->sc, (void*)c->scratch, (void*)c->tan_out, (void*)c->tan_idx,
                  (void*)c->tan.partials, (void*)c->tan.nmax, (void*)c->tan.nmin, (void*)c->tan.norms, (void*)c->tan.l2, (void*)c->tan.planes,
                  c->fft_work,
                  (void*)c->aa_dX, (void*)c->aa_dR, (void*)c->aa_Rprev, (void*)c->aa_partials, (void*)c->aa_out,
                  (void*)c->pw, (void*)c->pctl, (void*)c->pcount, (void*)c->dot0, (void*)c->xp, (void*)c->xn, (void*)c->favg,
                  (void*)c->Ftau_last, (void*)c->Ftau_dot, (void*)c->Feval, (void*)c->curl_partials})
    if (p) cudaFree(p);
  for (auto& ck : c->ckpts)
    if (ck.dev) cudaFree(ck.dev);
  for (void* p : {(void*)c->adj_pts, (void*)c->adj_s, (void*)c->adj_D, (void*)c->adj_ws, (void*)c->adj_G,
                  (void*)c->adj_lam, (void*)c->adj_sig, (void*)c->adj_w, (void*)c->adj_V, (void*)c->adj_part,
                  (void*)c->adj_bad})
    if (p) cudaFree(p);
  for (auto& l : c->plist)
    for (int* p : l)
      if (p) cudaFree(p);
  if (c->hcount) cudaFreeHost(c->hcount);
  if (c->tan_host) cudaFreeHost(c->tan_host);
  for (auto e : c->ev)
    if (e) cudaEventDestroy(e);
  for (auto e : c->tev)
    if (e) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
  for (int h = 1; h < PASS_CHUNKS; ++h) {
    if (c->cstream[h]) cudaStreamDestroy(c->cstream[h]);
    if (c->join[h]) cudaEventDestroy(c->join[h]);
  }
  if (c->fork) cudaEventDestroy(c->fork);
  delete c->pc12;
  delete c->pc18;
  delete c->pc24;
  delete c->pc48;
  if (c->hmat) cudaFree(c->hmat);
  if (c->sysc) cudaFree(c->sysc);
  delete c;
}

}  // extern "C"

// ------------------------------------------------------------------ checkpoints and the adjoint
namespace {

// The per-voxel buffers whose values carry from one increment to the next (basic scheme).
std::vector<std::pair<double*, size_t>> state_buffers(dmk_ctx* c) {
  const size_t N = size_t(c->N), NST = size_t(2 * c->NS);
  return {{c->Fsol, 9 * N}, {c->Flast, 9 * N}, {c->Fdot, 9 * N}, {c->F, 9 * N},  {c->F0, 9 * N},
          {c->Fp, 9 * N},   {c->Fp0, 9 * N},   {c->Lp, 9 * N},   {c->Lp0, 9 * N}, {c->S, 6 * N},
          {c->S0, 6 * N},   {c->Fe, 9 * N},    {c->P, 9 * N},    {c->Pnew, 9 * N}, {c->state, NST * N},
          {c->state0, NST * N}, {c->dot0, NST * N}};
}
constexpr size_t SC_DOUBLES = (sizeof(SolverScalars) + sizeof(double) - 1) / sizeof(double);

// host solver state, packed in a fixed order
template <bool SAVE>
void pack_host(dmk_ctx* c, std::vector<double>& h) {
  size_t o = 0;
  auto io = [&](double* p, size_t n) {
    if (SAVE) h.insert(h.end(), p, p + n);
    else std::copy(h.begin() + o, h.begin() + o + n, p);
    o += n;
  };
  io(c->F_aim, 9); io(c->F_aim_lastinc, 9); io(c->F_aimDot, 9); io(c->P_aim, 9); io(c->P_av, 9);
  io(c->C_volAvg, 81); io(c->C_volAvgLastInc, 81); io(c->C_minMaxAvg, 81); io(c->C_minMaxAvgLastInc, 81);
  io(c->Scomp, 81); io(c->C_gamma, 81); io(c->q_rot, 4); io(&c->dt, 1); io(c->h_aim, 9);
  double ints[10];
  for (int k = 0; k < 9; ++k) ints[k] = c->stress_mask[k];
  ints[9] = c->dot0_valid ? 1.0 : 0.0;
  io(ints, 10);
  if (!SAVE) {
    for (int k = 0; k < 9; ++k) c->stress_mask[k] = int(ints[k]);
    c->dot0_valid = ints[9] != 0.0;
  }
}

bool is_identity_rotation(const double* q) { return q[0] == 1.0 && q[1] == 0.0 && q[2] == 0.0 && q[3] == 0.0; }

int adj_jacobians(dmk_ctx* c, int slot) {
  const int64_t N = c->N;
  const double* pts = c->adj_pts + size_t(slot) * size_t(27 + 2 * c->NS) * size_t(N);
  CK(cudaMemsetAsync(c->adj_bad, 0, sizeof(int), c->stream));
  for (int64_t v0 = 0; v0 < N; v0 += c->adj_chunk) {
    const int64_t cnt = std::min<int64_t>(c->adj_chunk, N - v0);
    const double dt = c->adj_dt[slot];
    switch (c->NS) {
      case 12: CKL(launch_adj_jacobian<12>(*c->pc12, dt, pts, N, v0, cnt, c->adj_ws, c->adj_D, c->adj_bad, c->stream)); break;
      case 18: CKL(launch_adj_jacobian<18>(*c->pc18, dt, pts, N, v0, cnt, c->adj_ws, c->adj_D, c->adj_bad, c->stream)); break;
      case 24: CKL(launch_adj_jacobian<24>(*c->pc24, dt, pts, N, v0, cnt, c->adj_ws, c->adj_D, c->adj_bad, c->stream)); break;
      case 48: CKL(launch_adj_jacobian<48>(*c->pc48, dt, pts, N, v0, cnt, c->adj_ws, c->adj_D, c->adj_bad, c->stream)); break;
    }
  }
  int bad = 0;
  CK(cudaMemcpyAsync(&bad, c->adj_bad, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (bad) return fail(DMK_ERR_STATE, "adjoint: singular local Jacobian in " + std::to_string(bad) + " voxels");
  return 0;
}

int adj_vjp(dmk_ctx* c, const double ell[9], const double* lam, int mode) {
  const double* s_in = c->adj_s + size_t(c->adj_cur) * size_t(9 + c->NS) * size_t(c->N);
  double* s_out = c->adj_s + size_t(1 - c->adj_cur) * size_t(9 + c->NS) * size_t(c->N);
  switch (c->NS) {
    case 12: CKL(launch_adj_vjp<12>(c->adj_D, c->N, c->adj_nx, ell, lam, s_in, c->adj_G, s_out, c->adj_part, mode, c->stream)); break;
    case 18: CKL(launch_adj_vjp<18>(c->adj_D, c->N, c->adj_nx, ell, lam, s_in, c->adj_G, s_out, c->adj_part, mode, c->stream)); break;
    case 24: CKL(launch_adj_vjp<24>(c->adj_D, c->N, c->adj_nx, ell, lam, s_in, c->adj_G, s_out, c->adj_part, mode, c->stream)); break;
    case 48: CKL(launch_adj_vjp<48>(c->adj_D, c->N, c->adj_nx, ell, lam, s_in, c->adj_G, s_out, c->adj_part, mode, c->stream)); break;
  }
  return 0;
}

// fixed-order host sum of per-block partials: out[k] = sum_b part[b * K + k]
int sum_partials(dmk_ctx* c, const double* dev, int nblocks, int K, double* out) {
  std::vector<double> h(size_t(nblocks) * K);
  CK(cudaMemcpyAsync(h.data(), dev, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < K; ++k) out[k] = 0.0;
  for (int b = 0; b < nblocks; ++b)
    for (int k = 0; k < K; ++k) out[k] += h[size_t(b) * K + k];
  return 0;
}

// y = M x (+ the affine part for G != null): sigma = K^T x - G, then the Gamma convolution of sigma
// with the reference medium of the forward solver, whose average is replaced by S_m : <sigma>
// (S_m: the masked compliance, non-zero on the stress-controlled components only).
int adj_apply(dmk_ctx* c, const double* x, const double* G, const double* Sm, double* y) {
  const int nb = adj_blocks(c->N);
  CKL(launch_adj_sigma(c->adj_D, c->N, c->adj_nx, x, G, c->adj_sig, c->adj_part, c->stream));
  double m9[9];
  if (int rc = sum_partials(c, c->adj_part, nb, 9, m9)) return rc;
  double dc[9];
  for (int a = 0; a < 9; ++a) {
    double s = 0.0;
    for (int b = 0; b < 9; ++b) s += Sm[a + 9 * b] * m9[b] * c->wgt;
    dc[a] = s;
  }
  CK(cudaMemcpyAsync(reinterpret_cast<char*>(c->sc) + offsetof(SolverScalars, aim_rot), dc, 9 * sizeof(double),
                     cudaMemcpyHostToDevice, c->stream));
  return spectral_pass(c, false, 1, 0, y, c->adj_sig);
}

int adj_dots(dmk_ctx* c, const double* w, const double* V, int nv, double* out) {
  CKL(launch_adj_mdot(w, V, 9 * c->N, nv, c->adj_part, c->nsm, c->stream));
  return sum_partials(c, c->adj_part, adj_mdot_blocks(c->nsm), nv, out);
}

// Restarted GMRES (Saad & Schultz 1986) with classical Gram-Schmidt and one reorthogonalisation
// for M lam = b, b = -(M 0 with G); lam starts at zero.  Returns the iterations in *its.
int adj_solve(dmk_ctx* c, const double* Sm, double rtol, int* its, double* relres) {
  const int m = ADJ_KRYLOV_MAX;
  const int64_t n9 = 9 * c->N;
  double* V = c->adj_V;
  auto Vj = [&](int j) { return V + size_t(j) * size_t(n9); };
  CK(cudaMemsetAsync(c->adj_lam, 0, sizeof(double) * n9, c->stream));
  if (int rc = adj_apply(c, c->adj_lam, c->adj_G, Sm, c->adj_w)) return rc;   // w = -b
  CKL(launch_adj_scale(Vj(0), c->adj_w, -1.0, n9, c->nsm, c->stream));
  double beta2;
  if (int rc = adj_dots(c, Vj(0), Vj(0), 1, &beta2)) return rc;
  const double bnorm = std::sqrt(beta2);
  double beta = bnorm;
  *its = 0;
  *relres = 0.0;
  if (!(bnorm > 0.0)) return 0;
  for (int restart = 0; restart < 40; ++restart) {
    CKL(launch_adj_scale(Vj(0), Vj(0), 1.0 / beta, n9, c->nsm, c->stream));
    std::vector<double> H(size_t(m + 1) * m, 0.0), g(m + 1, 0.0), cs(m, 0.0), sn(m, 0.0);
    g[0] = beta;
    int jend = 0;
    double res = beta;
    for (int j = 0; j < m; ++j) {
      if (int rc = adj_apply(c, Vj(j), nullptr, Sm, c->adj_w)) return rc;
      double h[ADJ_KRYLOV_MAX + 1], h2[ADJ_KRYLOV_MAX + 1], neg[ADJ_KRYLOV_MAX + 1];
      if (int rc = adj_dots(c, c->adj_w, V, j + 1, h)) return rc;
      for (int i = 0; i <= j; ++i) neg[i] = -h[i];
      CKL(launch_adj_maxpy(c->adj_w, V, n9, j + 1, neg, c->nsm, c->stream));
      if (int rc = adj_dots(c, c->adj_w, V, j + 1, h2)) return rc;
      for (int i = 0; i <= j; ++i) { neg[i] = -h2[i]; h[i] += h2[i]; }
      CKL(launch_adj_maxpy(c->adj_w, V, n9, j + 1, neg, c->nsm, c->stream));
      double hn2;
      if (int rc = adj_dots(c, c->adj_w, c->adj_w, 1, &hn2)) return rc;
      const double hn = std::sqrt(hn2);
      for (int i = 0; i <= j; ++i) H[size_t(i) * m + j] = h[i];
      H[size_t(j + 1) * m + j] = hn;
      // Givens rotations
      for (int i = 0; i < j; ++i) {
        const double a = H[size_t(i) * m + j], b = H[size_t(i + 1) * m + j];
        H[size_t(i) * m + j] = cs[i] * a + sn[i] * b;
        H[size_t(i + 1) * m + j] = -sn[i] * a + cs[i] * b;
      }
      const double a = H[size_t(j) * m + j], b = H[size_t(j + 1) * m + j];
      const double r = std::hypot(a, b);
      cs[j] = r > 0.0 ? a / r : 1.0;
      sn[j] = r > 0.0 ? b / r : 0.0;
      H[size_t(j) * m + j] = r;
      H[size_t(j + 1) * m + j] = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      res = std::fabs(g[j + 1]);
      ++*its;
      jend = j + 1;
      if (res <= rtol * bnorm || !(hn > 0.0)) break;
      CKL(launch_adj_scale(Vj(j + 1), c->adj_w, 1.0 / hn, n9, c->nsm, c->stream));
    }
    // lam += V y, H y = g (upper triangular)
    std::vector<double> yv(jend, 0.0);
    for (int i = jend - 1; i >= 0; --i) {
      double s = g[i];
      for (int k = i + 1; k < jend; ++k) s -= H[size_t(i) * m + k] * yv[k];
      yv[i] = s / H[size_t(i) * m + i];
    }
    CKL(launch_adj_maxpy(c->adj_lam, V, n9, jend, yv.data(), c->nsm, c->stream));
    // true residual b - M lam
    if (int rc = adj_apply(c, c->adj_lam, c->adj_G, Sm, c->adj_w)) return rc;
    CKL(launch_adj_scale(Vj(0), c->adj_w, -1.0, n9, c->nsm, c->stream));
    double r2;
    if (int rc = adj_dots(c, Vj(0), Vj(0), 1, &r2)) return rc;
    beta = std::sqrt(r2);
    *relres = beta / bnorm;
    if (beta <= rtol * bnorm || !(beta > 0.0)) return 0;
  }
  return fail(DMK_ERR_NOT_CONVERGED, "adjoint: the transposed equilibrium problem did not converge (relative residual " +
                                         std::to_string(*relres) + ")");
}

}  // namespace

extern "C" {

int dmk_checkpoint_save(dmk_ctx* c, int slot) {
  if (!c || slot < 0) return fail(DMK_ERR_ARG, "checkpoint: null context or negative slot");
  if (c->solver != 0) return fail(DMK_ERR_CONFIG, "checkpoints are implemented for the basic spectral scheme");
  CK(cudaSetDevice(c->device));
  if (size_t(slot) >= c->ckpts.size()) c->ckpts.resize(slot + 1);
  auto& ck = c->ckpts[slot];
  const auto bufs = state_buffers(c);
  size_t total = SC_DOUBLES;
  for (const auto& b : bufs) total += b.second;
  if (!ck.dev)
    if (int rc = dalloc(&ck.dev, total)) return rc;
  size_t o = 0;
  for (const auto& b : bufs) {
    CK(cudaMemcpyAsync(ck.dev + o, b.first, sizeof(double) * b.second, cudaMemcpyDeviceToDevice, c->stream));
    o += b.second;
  }
  CK(cudaMemcpyAsync(ck.dev + o, c->sc, sizeof(SolverScalars), cudaMemcpyDeviceToDevice, c->stream));
  ck.host.clear();
  pack_host<true>(c, ck.host);
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int dmk_checkpoint_restore(dmk_ctx* c, int slot) {
  if (!c || slot < 0 || size_t(slot) >= c->ckpts.size() || !c->ckpts[slot].dev)
    return fail(DMK_ERR_ARG, "checkpoint: no checkpoint in this slot");
  CK(cudaSetDevice(c->device));
  auto& ck = c->ckpts[slot];
  size_t o = 0;
  for (const auto& b : state_buffers(c)) {
    CK(cudaMemcpyAsync(b.first, ck.dev + o, sizeof(double) * b.second, cudaMemcpyDeviceToDevice, c->stream));
    o += b.second;
  }
  CK(cudaMemcpyAsync(c->sc, ck.dev + o, sizeof(SolverScalars), cudaMemcpyDeviceToDevice, c->stream));
  pack_host<false>(c, ck.host);
  update_gamma_host(c, c->C_gamma);
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int dmk_adj_begin(dmk_ctx* c, int n_slots) {
  if (!c || n_slots < 1) return fail(DMK_ERR_ARG, "adjoint: null context or no slots");
  if (c->solver != 0) return fail(DMK_ERR_CONFIG, "the adjoint is implemented for the basic spectral scheme");
  CK(cudaSetDevice(c->device));
  const int64_t N = c->N;
  const int NS = c->NS;
  const int nf = c->hp.nf;
  if (nf < 1 || nf > ADJ_MAX_FAMILIES) return fail(DMK_ERR_CONFIG, "adjoint: unsupported number of slip families");
  if (n_slots != c->adj_slots) {
    if (c->adj_pts) cudaFree(c->adj_pts);
    c->adj_pts = nullptr;
    if (int rc = dalloc(&c->adj_pts, size_t(n_slots) * size_t(27 + 2 * NS) * size_t(N))) return rc;
    c->adj_slots = n_slots;
  }
  c->adj_nx = adj_nx(NS, nf);
  c->adj_nz = adj_nz(NS);
  if (!c->adj_s) {
    const int64_t per = adj_ws_size(NS, nf);
    c->adj_chunk = std::max<int64_t>(128, std::min<int64_t>(N, (int64_t(1) << 28) / (8 * per)));
    const int nbv = std::max(adj_blocks(N) * 16, adj_mdot_blocks(c->nsm) * (ADJ_KRYLOV_MAX + 1));
    if (int rc = dalloc(&c->adj_s, 2 * size_t(9 + NS) * size_t(N))) return rc;
    if (int rc = dalloc(&c->adj_D, size_t(c->adj_nz) * size_t(c->adj_nx) * size_t(N))) return rc;
    if (int rc = dalloc(&c->adj_ws, size_t(per) * size_t(c->adj_chunk))) return rc;
    if (int rc = dalloc(&c->adj_G, 9 * size_t(N))) return rc;
    if (int rc = dalloc(&c->adj_lam, 9 * size_t(N))) return rc;
    if (int rc = dalloc(&c->adj_sig, 9 * size_t(N))) return rc;
    if (int rc = dalloc(&c->adj_w, 9 * size_t(N))) return rc;
    if (int rc = dalloc(&c->adj_V, size_t(ADJ_KRYLOV_MAX + 1) * 9 * size_t(N))) return rc;
    if (int rc = dalloc(&c->adj_part, size_t(nbv))) return rc;
    if (int rc = dalloc(&c->adj_bad, 1)) return rc;
  }
  c->adj_dt.assign(n_slots, 0.0);
  c->adj_mask.assign(n_slots, std::array<int, 9>{});
  c->adj_rec.assign(n_slots, 0);
  c->adj_cur = 0;
  CK(cudaMemsetAsync(c->adj_s, 0, sizeof(double) * 2 * size_t(9 + NS) * size_t(N), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->iter_enabled = true;          // per-voxel substep counts, checked when an increment is recorded
  return 0;
}

int dmk_adj_record(dmk_ctx* c, int slot) {
  if (!c || slot < 0 || slot >= c->adj_slots) return fail(DMK_ERR_ARG, "adjoint: slot out of range (call dmk_adj_begin)");
  CK(cudaSetDevice(c->device));
  if (!is_identity_rotation(c->q_rot)) return fail(DMK_ERR_CONFIG, "adjoint: load-case rotation R must be the identity");
  const int64_t N = c->N;
  const int NS = c->NS;
  // one substep per voxel (the local model is that of a single substep) and no failed voxel
  std::vector<int> it(2 * size_t(N));
  CK(cudaMemcpyAsync(it.data(), c->iter + 2 * N, sizeof(int) * 2 * N, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int64_t v = 0; v < N; ++v) {
    if (it[size_t(N + v)] != 0) return fail(DMK_ERR_STATE, "adjoint: the increment has failed voxels");
    if (it[size_t(v)] != 1)
      return fail(DMK_ERR_STATE, "adjoint: a voxel needed substeps in this increment (the adjoint covers single substeps)");
  }
  double* p = c->adj_pts + size_t(slot) * size_t(27 + 2 * NS) * size_t(N);
  const size_t N9 = 9 * size_t(N), NN = size_t(NS) * size_t(N);
  CK(cudaMemcpyAsync(p, c->F, sizeof(double) * N9, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(p + N9, c->Fp0, sizeof(double) * N9, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(p + 2 * N9, c->state0, sizeof(double) * NN, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(p + 2 * N9 + NN, c->Lp, sizeof(double) * N9, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(p + 3 * N9 + NN, c->state, sizeof(double) * NN, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->adj_dt[slot] = c->dt;
  for (int k = 0; k < 9; ++k) c->adj_mask[slot][k] = c->stress_mask[k];
  c->adj_rec[slot] = 1;
  return 0;
}

int dmk_adj_step(dmk_ctx* c, int slot, const double P_av_bar[9], double theta_bar[20], int* iterations) {
  if (!c || !P_av_bar || !theta_bar) return fail(DMK_ERR_ARG, "null argument");
  if (slot < 0 || slot >= c->adj_slots || !c->adj_rec[slot]) return fail(DMK_ERR_ARG, "adjoint: slot not recorded");
  CK(cudaSetDevice(c->device));
  const int64_t N = c->N;
  const int NS = c->NS;
  const int nf = c->hp.nf;
  if (int rc = adj_jacobians(c, slot)) return rc;
  // masked compliance of the transposed average tangent (stress-controlled components only)
  double CT[81], Sm[81];
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) for (int k = 0; k < 3; ++k) for (int l = 0; l < 3; ++l)
    CT[k + 3 * l + 9 * i + 27 * j] = c->C_volAvg[i + 3 * j + 9 * k + 27 * l];
  const double qI[4] = {1.0, 0.0, 0.0, 0.0};
  if (int rc = masked_compliance(qI, c->adj_mask[slot].data(), CT, Sm)) return rc;
  // G = (dP/dF)^T ell + (ds/dF)^T s_hat
  if (int rc = adj_vjp(c, P_av_bar, nullptr, 0)) return rc;
  int its = 0;
  double relres = 0.0;
  if (int rc = adj_solve(c, Sm, 1.0e-12, &its, &relres)) return rc;
  if (iterations) *iterations = its;
  // state cotangent of the increment start and the parameter cotangent
  if (int rc = adj_vjp(c, P_av_bar, c->adj_lam, 1)) return rc;
  double th[4 * ADJ_MAX_FAMILIES];
  if (int rc = sum_partials(c, c->adj_part, adj_blocks(N), 4 * ADJ_MAX_FAMILIES, th)) return rc;
  for (int p = 0; p < 4; ++p)
    for (int f = 0; f < nf; ++f) theta_bar[(1 + p) * ADJ_MAX_FAMILIES + f] += th[p * nf + f] / double(N);
  c->adj_cur = 1 - c->adj_cur;
  (void)NS;
  return 0;
}

int dmk_adj_finish(dmk_ctx* c, double theta_bar[20]) {
  if (!c || !theta_bar) return fail(DMK_ERR_ARG, "null argument");
  CK(cudaSetDevice(c->device));
  const int64_t N = c->N;
  const int NS = c->NSact;
  std::vector<double> s(size_t(NS) * size_t(N));
  const double* xi_bar = c->adj_s + size_t(c->adj_cur) * size_t(9 + c->NS) * size_t(N) + 9 * size_t(N);
  CK(cudaMemcpyAsync(s.data(), xi_bar, sizeof(double) * s.size(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  // xi(t = 0) = xi_0 of the system's family in every voxel
  for (int k = 0; k < NS; ++k) {
    const int f = c->hp.fam[k];
    if (f < 0) continue;
    double t = 0.0;
    for (int64_t v = 0; v < N; ++v) t += s[size_t(k) * size_t(N) + size_t(v)];
    theta_bar[f] += t / double(N);
  }
  return 0;
}

int dmk_adj_local_jacobian(const dmk_phase* phase, double dt, const double* point, double* D) {
  if (!phase || !point || !D) return fail(DMK_ERR_ARG, "null argument");
  HostPhase hp;
  std::string err;
  if (build_host_phase(*phase, hp, err)) return fail(DMK_ERR_CONFIG, err);
  const int np = padded_slip_count(hp.Ns);
  if (!np) return fail(DMK_ERR_CONFIG, "unsupported number of slip systems");
  pad_host_phase(hp, np);
  switch (np) {
    case 12: { auto pc = std::make_unique<PhaseConst<12>>(); fill_phase_const<12>(hp, hp.h.data(), *pc);
               return host_local_jacobian<12>(*pc, hp.h.data(), dt, point, D) ? fail(DMK_ERR_STATE, "singular") : 0; }
    case 18: { auto pc = std::make_unique<PhaseConst<18>>(); fill_phase_const<18>(hp, hp.h.data(), *pc);
               return host_local_jacobian<18>(*pc, hp.h.data(), dt, point, D) ? fail(DMK_ERR_STATE, "singular") : 0; }
    case 24: { auto pc = std::make_unique<PhaseConst<24>>(); fill_phase_const<24>(hp, hp.h.data(), *pc);
               return host_local_jacobian<24>(*pc, hp.h.data(), dt, point, D) ? fail(DMK_ERR_STATE, "singular") : 0; }
    case 48: { auto pc = std::make_unique<PhaseConst<48>>(); fill_phase_const<48>(hp, hp.h.data(), *pc);
               return host_local_jacobian<48>(*pc, hp.h.data(), dt, point, D) ? fail(DMK_ERR_STATE, "singular") : 0; }
  }
  return fail(DMK_ERR_CONFIG, "unsupported number of slip systems");
}

}  // extern "C"

// ------------------------------------------------------------------ batches of contexts
// The basic scheme's fixed point of many contexts (RVEs of one phase) in shared launches: per
// iteration one CUDA graph runs the constitutive evaluation of every active context (its pass loop
// is a device-side while node, so the host reads no voxel counts), then batched kernels and one
// cuFFT plan per edge size form the residuals; the host reads the solver scalars of all contexts
// once per iteration and makes the Anderson / Richardson decisions.

struct dmk_batch {
  int n = 0, NS = 0, device = 0, nsm = 148;
  std::vector<dmk_ctx*> ctx;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  int64_t n_items = 0;
  // per-context tables of the constitutive kernels: one device block, one pinned host mirror
  char* d_tab = nullptr;
  char* h_tab = nullptr;
  size_t tab_bytes = 0, o_f = 0, o_w = 0, o_dt = 0, o_dot0 = 0, o_apply = 0, o_active = 0;
  int64_t* d_off = nullptr;
  int* d_ctx_of = nullptr;
  int* d_list[2] = {nullptr, nullptr};
  int* d_count = nullptr;
  int* d_status = nullptr;
  int* d_iter = nullptr;
  int* h_iter = nullptr;
  // tables of the batched solver kernels
  BatchCtx* d_bc = nullptr;
  BatchCtx* h_bc = nullptr;
  BatchAA* d_aa = nullptr;
  BatchAA* h_aa = nullptr;
  BatchScal* d_scal = nullptr;
  BatchScal* h_scal = nullptr;
  double* d_red = nullptr;       // partial sums of every context (sum9, divergence, Anderson)
  double* d_dots = nullptr;      // Anderson inner products, 4 chunks of 2 AA_CHUNK per context
  double* h_dots = nullptr;
  struct Group {
    int cells[3];
    std::vector<int> members;
    double* real = nullptr;
    double* spec = nullptr;
    cufftHandle fwd = 0, bwd = 0;
    float* real_f = nullptr;       // the mixed form's FP32 buffers and plans (when a member is mixed)
    float* spec_f = nullptr;
    cufftHandle fwd_f = 0, bwd_f = 0;
    bool run32 = false, run64 = false;   // transforms needed in the current spectral pass
  };
  std::vector<Group> groups;
  void* fft_work = nullptr;
  int max_nconst = 0, max_nspec = 0, max_aa_blocks = 0;
  int64_t max_n9 = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  double last_ms[2] = {0.0, 0.0};     // constitutive graphs, whole solution (device time)
  int64_t graph_launches = 0, passes = 0, iterations = 0, solutions = 0;
  double host_ms[3] = {0.0, 0.0, 0.0};  // last solution, host time: set-up, iterations, tangents and counters
  std::unique_ptr<HostPool> pool;        // host threads for the per-member calls
};

namespace {

constexpr int BATCH_DOTS = 4 * 2 * AA_CHUNK;   // Anderson inner products per context (AA_MAX slots)

void batch_free(dmk_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (auto& g : b->groups) {
    for (cufftHandle p : {g.fwd, g.bwd, g.fwd_f, g.bwd_f})
      if (p) cufftDestroy(p);
    for (void* p : {(void*)g.real, (void*)g.spec, (void*)g.real_f, (void*)g.spec_f})
      if (p) cudaFree(p);
  }
  for (void* p : {(void*)b->d_tab, (void*)b->d_off, (void*)b->d_ctx_of, (void*)b->d_list[0], (void*)b->d_list[1],
                  (void*)b->d_count, (void*)b->d_status, (void*)b->d_iter, (void*)b->d_bc, (void*)b->d_aa,
                  (void*)b->d_scal, (void*)b->d_red, (void*)b->d_dots, b->fft_work})
    if (p) cudaFree(p);
  for (void* p : {(void*)b->h_tab, (void*)b->h_iter, (void*)b->h_bc, (void*)b->h_aa, (void*)b->h_scal, (void*)b->h_dots})
    if (p) cudaFreeHost(p);
  for (auto e : b->ev)
    if (e) cudaEventDestroy(e);
  if (b->stream) cudaStreamDestroy(b->stream);
  b->pool.reset();
  delete b;
}

template <int NS>
const PhaseConst<NS>* phase_const_of(const dmk_ctx* c);
template <> const PhaseConst<12>* phase_const_of<12>(const dmk_ctx* c) { return c->pc12; }
template <> const PhaseConst<18>* phase_const_of<18>(const dmk_ctx* c) { return c->pc18; }
template <> const PhaseConst<24>* phase_const_of<24>(const dmk_ctx* c) { return c->pc24; }
template <> const PhaseConst<48>* phase_const_of<48>(const dmk_ctx* c) { return c->pc48; }

// the phase constants of two contexts agree (their device pointers aside)
template <int NS>
bool same_phase_const(const dmk_ctx* a, const dmk_ctx* b) {
  auto x = std::make_unique<PhaseConst<NS>>(*phase_const_of<NS>(a));
  auto y = std::make_unique<PhaseConst<NS>>(*phase_const_of<NS>(b));
  x->hmat = y->hmat = nullptr;
  x->sys = y->sys = nullptr;
  return std::memcmp(x.get(), y.get(), sizeof(PhaseConst<NS>)) == 0;
}
bool same_phase(const dmk_ctx* a, const dmk_ctx* b) {
  if (a->NS != b->NS || a->hp.h != b->hp.h || std::memcmp(&a->nm, &b->nm, sizeof a->nm) != 0) return false;
  switch (a->NS) {
    case 12: return same_phase_const<12>(a, b);
    case 18: return same_phase_const<18>(a, b);
    case 24: return same_phase_const<24>(a, b);
    case 48: return same_phase_const<48>(a, b);
  }
  return false;
}

template <int NS>
cudaError_t batch_graph(dmk_batch* b, const BatchTables& t, const BatchPassBuffers& pb) {
  const dmk_ctx* c0 = b->ctx[0];
  return build_batch_pass_graph<NS>(*phase_const_of<NS>(c0), c0->nm, t, pb, b->nsm, b->stream, &b->graph);
}

int batch_build(dmk_batch* b) {
  const int n = b->n;
  CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  for (auto& e : b->ev) CK(cudaEventCreate(&e));
  // items: the voxels of all contexts, context after context
  std::vector<int64_t> off(n + 1, 0);
  for (int r = 0; r < n; ++r) off[r + 1] = off[r] + b->ctx[r]->N;
  b->n_items = off[n];
  if (b->n_items > INT32_MAX) return fail(DMK_ERR_ARG, "a batch holds at most 2^31 - 1 voxels");
  std::vector<int> ctx_of(b->n_items);
  for (int r = 0; r < n; ++r)
    for (int64_t v = off[r]; v < off[r + 1]; ++v) ctx_of[v] = r;
  int rc;
  if ((rc = dalloc(&b->d_off, n + 1)) || (rc = dalloc(&b->d_ctx_of, b->n_items)) ||
      (rc = dalloc(&b->d_list[0], b->n_items)) || (rc = dalloc(&b->d_list[1], b->n_items)) ||
      (rc = dalloc(&b->d_count, 2)) || (rc = dalloc(&b->d_status, n)) || (rc = dalloc(&b->d_iter, 2)) ||
      (rc = dalloc(&b->d_bc, n)) || (rc = dalloc(&b->d_aa, n)) || (rc = dalloc(&b->d_scal, n)) ||
      (rc = dalloc(&b->d_dots, size_t(n) * BATCH_DOTS)))
    return rc;
  CK(cudaMemcpy(b->d_off, off.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b->d_ctx_of, ctx_of.data(), sizeof(int) * b->n_items, cudaMemcpyHostToDevice));
  CK(cudaMallocHost(reinterpret_cast<void**>(&b->h_iter), 2 * sizeof(int)));
  CK(cudaMallocHost(reinterpret_cast<void**>(&b->h_bc), sizeof(BatchCtx) * n));
  CK(cudaMallocHost(reinterpret_cast<void**>(&b->h_aa), sizeof(BatchAA) * n));
  CK(cudaMallocHost(reinterpret_cast<void**>(&b->h_scal), sizeof(BatchScal) * n));
  CK(cudaMallocHost(reinterpret_cast<void**>(&b->h_dots), sizeof(double) * n * BATCH_DOTS));
  std::memset(b->h_bc, 0, sizeof(BatchCtx) * n);
  std::memset(b->h_aa, 0, sizeof(BatchAA) * n);
  // the tables of the constitutive kernels, 256-byte aligned sections of one block
  auto sec = [&](size_t bytes) {
    const size_t o = b->tab_bytes;
    b->tab_bytes += (bytes + 255) / 256 * 256;
    return o;
  };
  b->o_f = sec(sizeof(Fields) * n);
  b->o_w = sec(sizeof(PassWork) * n);
  b->o_dt = sec(sizeof(double) * n);
  b->o_dot0 = sec(sizeof(int) * n);
  b->o_apply = sec(sizeof(int) * n);
  b->o_active = sec(n);
  if ((rc = dalloc(&b->d_tab, b->tab_bytes))) return rc;
  CK(cudaMallocHost(reinterpret_cast<void**>(&b->h_tab), b->tab_bytes));
  std::memset(b->h_tab, 0, b->tab_bytes);
  // per-context partial sums, and the static part of the solver kernels' table
  size_t red = 0;
  std::vector<size_t> o_part(n), o_div(n), o_aap(n);
  for (int r = 0; r < n; ++r) {
    dmk_ctx* c = b->ctx[r];
    BatchCtx& x = b->h_bc[r];
    x.N = c->N;
    x.wgt = c->wgt;
    for (int d = 0; d < 3; ++d) {
      x.L[d] = c->geom[d];
      x.n[d] = c->cells[d];
    }
    x.nconst = nblocks_const(c);
    x.nspec = gamma_div_blocks(c->cells[0], c->cells[1], c->cells[2]);
    x.aa_blocks = c->aa_blocks > 0 ? c->aa_blocks : 1;
    b->max_nconst = std::max(b->max_nconst, x.nconst);
    b->max_nspec = std::max(b->max_nspec, x.nspec);
    b->max_aa_blocks = std::max(b->max_aa_blocks, x.aa_blocks);
    b->max_n9 = std::max(b->max_n9, 9 * c->N);
    o_part[r] = red;
    red += size_t(9) * x.nconst;
    o_div[r] = red;
    red += size_t(x.nspec);
    o_aap[r] = red;
    red += size_t(x.aa_blocks) * 2 * AA_CHUNK;
  }
  if ((rc = dalloc(&b->d_red, red))) return rc;
  for (int r = 0; r < n; ++r) {
    BatchCtx& x = b->h_bc[r];
    x.partials = b->d_red + o_part[r];
    x.divp = b->d_red + o_div[r];
    x.aa_partials = b->d_red + o_aap[r];
    x.aa_out = b->d_dots + size_t(r) * BATCH_DOTS;
    x.status = b->d_status + r;
  }
  // one cuFFT plan pair per edge size over the 9 components of all its contexts
  for (int r = 0; r < n; ++r) {
    const dmk_ctx* c = b->ctx[r];
    auto it = std::find_if(b->groups.begin(), b->groups.end(), [&](const dmk_batch::Group& g) {
      return g.cells[0] == c->cells[0] && g.cells[1] == c->cells[1] && g.cells[2] == c->cells[2];
    });
    if (it == b->groups.end()) {
      b->groups.emplace_back();
      it = b->groups.end() - 1;
      for (int d = 0; d < 3; ++d) it->cells[d] = c->cells[d];
    }
    it->members.push_back(r);
  }
  size_t work = 0;
  bool any_mixed = false;
  for (int r = 0; r < n; ++r) any_mixed |= b->ctx[r]->precision == DMK_PRECISION_MIXED;
  for (auto& g : b->groups) {
    const int m = int(g.members.size());
    const int64_t N = int64_t(g.cells[0]) * g.cells[1] * g.cells[2];
    const int64_t plane = int64_t(g.cells[0] / 2 + 1) * g.cells[1] * g.cells[2];
    if (int64_t(9) * m * plane * 2 > INT32_MAX) return fail(DMK_ERR_ARG, "edge group too large for one cuFFT plan");
    if ((rc = dalloc(&g.real, size_t(9) * m * N)) || (rc = dalloc(&g.spec, size_t(18) * m * plane))) return rc;
    int nn[3] = {g.cells[2], g.cells[1], g.cells[0]};
    int inemb[3] = {g.cells[2], g.cells[1], g.cells[0]};
    int onemb[3] = {g.cells[2], g.cells[1], g.cells[0] / 2 + 1};
    size_t w1 = 0, w2 = 0;
    CKF(cufftCreate(&g.fwd));
    CKF(cufftCreate(&g.bwd));
    CKF(cufftSetAutoAllocation(g.fwd, 0));
    CKF(cufftSetAutoAllocation(g.bwd, 0));
    CKF(cufftMakePlanMany(g.fwd, 3, nn, inemb, 1, int(N), onemb, 1, int(plane), CUFFT_D2Z, 9 * m, &w1));
    CKF(cufftMakePlanMany(g.bwd, 3, nn, onemb, 1, int(plane), inemb, 1, int(N), CUFFT_Z2D, 9 * m, &w2));
    work = std::max(work, std::max(w1, w2));
    if (any_mixed) {
      if ((rc = dalloc(&g.real_f, size_t(9) * m * N)) || (rc = dalloc(&g.spec_f, size_t(18) * m * plane))) return rc;
      CKF(cufftCreate(&g.fwd_f));
      CKF(cufftCreate(&g.bwd_f));
      CKF(cufftSetAutoAllocation(g.fwd_f, 0));
      CKF(cufftSetAutoAllocation(g.bwd_f, 0));
      CKF(cufftMakePlanMany(g.fwd_f, 3, nn, inemb, 1, int(N), onemb, 1, int(plane), CUFFT_R2C, 9 * m, &w1));
      CKF(cufftMakePlanMany(g.bwd_f, 3, nn, onemb, 1, int(plane), inemb, 1, int(N), CUFFT_C2R, 9 * m, &w2));
      work = std::max(work, std::max(w1, w2));
    }
    for (int k = 0; k < m; ++k) {
      BatchCtx& x = b->h_bc[g.members[k]];
      x.fft_real = g.real + size_t(9) * k * N;
      x.fft_spec = g.spec + size_t(18) * k * plane;
      x.fft_real_f = g.real_f ? g.real_f + size_t(9) * k * N : nullptr;
      x.fft_spec_f = g.spec_f ? g.spec_f + size_t(18) * k * plane : nullptr;
    }
  }
  if (work) CK(cudaMalloc(&b->fft_work, work));
  for (auto& g : b->groups)
    for (cufftHandle p : {g.fwd, g.bwd, g.fwd_f, g.bwd_f})
      if (p) {
        CKF(cufftSetWorkArea(p, b->fft_work));
        CKF(cufftSetStream(p, b->stream));
      }
  // the constitutive evaluation of the batch as a graph over the tables
  BatchTables t;
  t.f = reinterpret_cast<const Fields*>(b->d_tab + b->o_f);
  t.w = reinterpret_cast<const PassWork*>(b->d_tab + b->o_w);
  t.dt = reinterpret_cast<const double*>(b->d_tab + b->o_dt);
  t.off = b->d_off;
  t.ctx_of = b->d_ctx_of;
  t.active = reinterpret_cast<const unsigned char*>(b->d_tab + b->o_active);
  t.use_dot0 = reinterpret_cast<const int*>(b->d_tab + b->o_dot0);
  t.apply = reinterpret_cast<const int*>(b->d_tab + b->o_apply);
  t.n_items = b->n_items;
  BatchPassBuffers pb;
  pb.list[0] = b->d_list[0];
  pb.list[1] = b->d_list[1];
  pb.count = b->d_count;
  pb.status = b->d_status;
  pb.n_ctx = n;
  pb.iter = b->d_iter;
  pb.max_passes = 400000;   // bounded by substeps x state iterations; more means corrupted control state
  cudaError_t e = cudaErrorInvalidValue;
  switch (b->NS) {
    case 12: e = batch_graph<12>(b, t, pb); break;
    case 18: e = batch_graph<18>(b, t, pb); break;
    case 24: e = batch_graph<24>(b, t, pb); break;
    case 48: e = batch_graph<48>(b, t, pb); break;
  }
  if (e != cudaSuccess) return fail(DMK_ERR_CUDA, std::string("batch graph: ") + cudaGetErrorString(e));
  CK(cudaGraphInstantiate(&b->exec, b->graph, 0));
  return 0;
}

// Fixed-point state of one context of a batched solve (the locals of dmk_mech_solution)
struct BatchSolve {
  int evals = 0, reason = 0, count = 0, new_slot = -1, it = 0, apply = 0, m = 0, snes_max_its = 50, nsl = 0;
  bool anderson = false, first = true, active = false;
  bool fp32 = false;               // mixed form: the spectral pass runs in FP32 until it first converges
  std::vector<double> G, bvec;
  std::vector<int> slots_b;
};

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

int batch_solution_impl(dmk_batch* b, const int* which, int nw, dmk_solution_state* out) {
  const int n = b->n;
  auto t0 = std::chrono::steady_clock::now();
  std::vector<BatchSolve> st(n);
  std::vector<int> pos(n, -1);
  for (int k = 0; k < nw; ++k) {
    const int r = which[k];
    if (r < 0 || r >= n) return fail(DMK_ERR_ARG, "batch member index out of range");
    if (pos[r] >= 0) return fail(DMK_ERR_ARG, "batch member listed twice");
    pos[r] = k;
  }
  b->last_ms[0] = b->last_ms[1] = 0.0;
  std::string msg;
  int rc0 = b->pool->run(nw, [&](int k) -> int {
    const int r = which[k];
    dmk_ctx* c = b->ctx[r];
    if (int rc = solution_prepare(c)) return rc;
    BatchSolve& S = st[r];
    S.active = true;
    S.snes_max_its = c->num.snes_max_it > 0 ? c->num.snes_max_it : 50;
    S.anderson = c->num.snes_type == 1;
    S.fp32 = c->precision == DMK_PRECISION_MIXED;
    S.m = c->aa_m;
    S.G.assign(size_t(S.m > 0 ? S.m : 1) * (S.m > 0 ? S.m : 1), 0.0);
    // the batch's launches follow the context's queued work (forward, solver scalars)
    CK(cudaEventRecord(c->fork, c->stream));
    CK(cudaStreamWaitEvent(b->stream, c->fork, 0));
    return 0;
  }, &msg);
  if (rc0) return fail(rc0, msg);
  CK(cudaEventRecord(b->ev[0], b->stream));
  b->host_ms[0] = ms_since(t0);
  t0 = std::chrono::steady_clock::now();
  Fields* hf = reinterpret_cast<Fields*>(b->h_tab + b->o_f);
  PassWork* hw = reinterpret_cast<PassWork*>(b->h_tab + b->o_w);
  double* hdt = reinterpret_cast<double*>(b->h_tab + b->o_dt);
  int* hdot0 = reinterpret_cast<int*>(b->h_tab + b->o_dot0);
  int* happly = reinterpret_cast<int*>(b->h_tab + b->o_apply);
  unsigned char* hact = reinterpret_cast<unsigned char*>(b->h_tab + b->o_active);
  for (;;) {
    int nact = 0, nchunks = 0;
    for (int r = 0; r < n; ++r) {
      dmk_ctx* c = b->ctx[r];
      BatchSolve& S = st[r];
      BatchCtx& x = b->h_bc[r];
      x.active = S.active ? 1 : 0;
      x.mode = S.active ? (S.fp32 ? 1 : 2) : 0;
      x.count_iter = 1;
      hact[r] = S.active ? 1 : 0;
      if (!S.active) continue;
      ++nact;
      Fields f = make_fields(c, S.apply ? c->r : nullptr);
      f.status = b->d_status + r;
      hf[r] = f;
      hw[r] = pass_work(c, 0, 0);
      hdt[r] = c->dt;
      hdot0[r] = c->dot0_valid ? 1 : 0;
      happly[r] = S.apply;
      x.P = c->P;
      x.Pnew = c->Pnew;
      x.r = c->r;
      x.X = c->Fsol;
      x.Rprev = c->aa_Rprev;
      x.dX = c->aa_dX;
      x.dR = c->aa_dR;
      x.sc = c->sc;
      x.nm2 = c->nm2;
      x.gc = c->gc;
      x.write_slot = -1;
      x.nsl = 0;
      S.nsl = 0;
      if (S.anderson && S.new_slot >= 0) {
        S.slots_b.clear();
        const int mk = std::min(S.count, S.m);
        for (int q = S.count - mk; q < S.count; ++q) S.slots_b.push_back(q % S.m);
        S.nsl = int(S.slots_b.size());
        x.write_slot = S.new_slot;
        x.nsl = S.nsl;
        for (int q = 0; q < S.nsl; ++q) x.slots[q] = S.slots_b[q];
        nchunks = std::max(nchunks, (S.nsl + AA_CHUNK - 1) / AA_CHUNK);
      }
    }
    if (nact == 0) break;
    ++b->iterations;
    CK(cudaMemcpyAsync(b->d_tab, b->h_tab, b->tab_bytes, cudaMemcpyHostToDevice, b->stream));
    CK(cudaMemcpyAsync(b->d_bc, b->h_bc, sizeof(BatchCtx) * n, cudaMemcpyHostToDevice, b->stream));
    // constitutive evaluation of every active context
    CK(cudaEventRecord(b->ev[2], b->stream));
    CK(cudaGraphLaunch(b->exec, b->stream));
    CK(cudaEventRecord(b->ev[3], b->stream));
    ++b->graph_launches;
    // residuals: <P> and aim, Gamma convolution per edge group (FP32 or FP64 by each context's
    // mode), convergence test, inner products; the scalars of all contexts read back once
    CK(launch_batch_aim(b->d_bc, n, b->max_nconst, b->stream));
    auto spectral = [&](int nch) -> int {
      for (auto& g : b->groups) {
        g.run32 = g.run64 = false;
        for (int r : g.members) {
          g.run32 |= b->h_bc[r].mode == 1;
          g.run64 |= b->h_bc[r].mode == 2;
        }
      }
      CK(launch_batch_gather(b->d_bc, n, b->max_n9, b->stream));
      for (auto& g : b->groups) {
        if (g.run32) CKF(cufftExecR2C(g.fwd_f, g.real_f, reinterpret_cast<cufftComplex*>(g.spec_f)));
        if (g.run64) CKF(cufftExecD2Z(g.fwd, g.real, reinterpret_cast<cufftDoubleComplex*>(g.spec)));
      }
      CK(launch_batch_gamma<float>(b->d_bc, n, b->max_nspec, b->stream));
      CK(launch_batch_gamma<double>(b->d_bc, n, b->max_nspec, b->stream));
      for (auto& g : b->groups) {
        if (g.run32) CKF(cufftExecC2R(g.bwd_f, reinterpret_cast<cufftComplex*>(g.spec_f), g.real_f));
        if (g.run64) CKF(cufftExecZ2D(g.bwd, reinterpret_cast<cufftDoubleComplex*>(g.spec), g.real));
      }
      CK(launch_batch_scatter(b->d_bc, n, b->max_n9, b->stream));
      CK(launch_batch_converge(b->d_bc, n, b->d_scal, b->stream));
      for (int ch = 0; ch < nch; ++ch) CK(launch_batch_aa_dots(b->d_bc, n, b->max_aa_blocks, ch, b->stream));
      CK(cudaMemcpyAsync(b->h_scal, b->d_scal, sizeof(BatchScal) * n, cudaMemcpyDeviceToHost, b->stream));
      CK(cudaMemcpyAsync(b->h_iter, b->d_iter, 2 * sizeof(int), cudaMemcpyDeviceToHost, b->stream));
      if (nch)
        CK(cudaMemcpyAsync(b->h_dots, b->d_dots, sizeof(double) * n * BATCH_DOTS, cudaMemcpyDeviceToHost, b->stream));
      CK(cudaStreamSynchronize(b->stream));
      return 0;
    };
    if (int rc = spectral(nchunks)) return rc;
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, b->ev[2], b->ev[3]));
    b->last_ms[0] += ms;
    b->passes += b->h_iter[0];
    if (b->h_iter[1]) return fail(DMK_ERR_CUDA, "constitutive passes did not terminate");
    // FP32 passes that meet the tolerance get a correction pass in FP64 on the same stress field;
    // its residual, decision and inner products replace the FP32 ones (dmk_mech_solution's)
    int ncorr = 0, nch1 = 0;
    for (int r = 0; r < n; ++r) {
      BatchCtx& x = b->h_bc[r];
      const bool corr = x.mode == 1 && b->h_scal[r].reason == 1;
      if (corr) {
        st[r].fp32 = false;
        ++ncorr;
        if (x.write_slot >= 0) nch1 = std::max(nch1, (x.nsl + AA_CHUNK - 1) / AA_CHUNK);
      }
      x.mode = corr ? 2 : 0;
      x.count_iter = 0;
    }
    if (ncorr) {
      CK(cudaMemcpyAsync(b->d_bc, b->h_bc, sizeof(BatchCtx) * n, cudaMemcpyHostToDevice, b->stream));
      if (int rc = spectral(nch1)) return rc;
    }
    // decisions and Anderson updates
    int naa = 0;
    for (int r = 0; r < n; ++r) {
      BatchSolve& S = st[r];
      b->h_aa[r].active = 0;
      if (!S.active) continue;
      dmk_ctx* c = b->ctx[r];
      const BatchScal& hs = b->h_scal[r];
      if (hs.status == 0) std::swap(c->P, c->Pnew);
      c->dot0_valid = true;
      ++S.evals;
      if (S.nsl > 0) {
        const double* dots = b->h_dots + size_t(r) * BATCH_DOTS;
        S.bvec.assign(S.nsl, 0.0);
        for (int q = 0; q < S.nsl; ++q) {
          const int ch = q / AA_CHUNK, k = q % AA_CHUNK;
          const double gq = dots[ch * 2 * AA_CHUNK + k], bq = dots[ch * 2 * AA_CHUNK + AA_CHUNK + k];
          S.G[size_t(S.new_slot) * S.m + S.slots_b[q]] = S.G[size_t(S.slots_b[q]) * S.m + S.new_slot] = gq;
          S.bvec[q] = bq;
        }
      }
      if (S.first && S.anderson) {   // b for the first Anderson step is empty (plain Richardson step)
        S.bvec.clear();
        S.slots_b.clear();
      }
      S.first = false;
      S.reason = hs.reason;
      if (S.reason == 0 && ++S.it > S.snes_max_its) S.reason = -1;
      if (S.reason != 0) {
        S.active = false;
        continue;
      }
      if (!S.anderson) {
        S.apply = 1;
        continue;
      }
      std::vector<double> gam = anderson_coefficients(S.G, S.m, S.slots_b, S.bvec);
      S.new_slot = S.count % S.m;
      BatchAA& a = b->h_aa[r];
      a.active = 1;
      a.new_slot = S.new_slot;
      a.u.n = int(S.slots_b.size());
      for (int q = 0; q < AA_MAX; ++q) {
        a.u.slot[q] = q < a.u.n ? S.slots_b[q] : 0;
        a.u.gamma[q] = q < a.u.n ? gam[q] : 0.0;
      }
      ++S.count;
      ++naa;
    }
    if (naa) {
      CK(cudaMemcpyAsync(b->d_aa, b->h_aa, sizeof(BatchAA) * n, cudaMemcpyHostToDevice, b->stream));
      CK(launch_batch_aa_update(b->d_bc, b->d_aa, n, b->max_aa_blocks, b->stream));
    }
  }
  CK(cudaEventRecord(b->ev[1], b->stream));
  CK(cudaEventSynchronize(b->ev[1]));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]));
  b->last_ms[1] = ms;
  b->host_ms[1] = ms_since(t0);
  t0 = std::chrono::steady_clock::now();
  // the contexts' own streams continue after the batch (tangent, forward of the next increment);
  // all tangents are queued before the first wait
  rc0 = b->pool->run(nw, [&](int k) -> int {
    const int r = which[k];
    dmk_ctx* c = b->ctx[r];
    CK(cudaStreamWaitEvent(c->stream, b->ev[1], 0));
    const BatchScal& hs = b->h_scal[r];
    return solution_finish_begin(c, hs.F_aim, hs.P_av, hs.totalIter, hs.err_div, hs.err_BC, st[r].reason,
                                 st[r].evals, &out[k]);
  }, &msg);
  if (rc0) return fail(rc0, msg);
  rc0 = b->pool->run(nw, [&](int k) -> int { return solution_finish_end(b->ctx[which[k]], &out[k]); }, &msg);
  if (rc0) return fail(rc0, msg);
  b->host_ms[2] = ms_since(t0);
  return 0;
}

}  // namespace

extern "C" {

int dmk_batch_create(dmk_batch** out, dmk_ctx* const* ctxs, int n) {
  if (!out || !ctxs) return fail(DMK_ERR_ARG, "null argument");
  *out = nullptr;
  if (n < 1 || n > 65535) return fail(DMK_ERR_ARG, "a batch holds 1 to 65535 contexts");
  for (int r = 0; r < n; ++r) {
    const dmk_ctx* c = ctxs[r];
    if (!c) return fail(DMK_ERR_ARG, "null context");
    if (c->solver != 0) return fail(DMK_ERR_CONFIG, "batched solves run the basic scheme");
    if (c->device != ctxs[0]->device) return fail(DMK_ERR_ARG, "contexts of a batch share one device");
    if (!same_phase(c, ctxs[0])) return fail(DMK_ERR_CONFIG, "contexts of a batch share one phase and its numerics");
    for (int q = 0; q < r; ++q)
      if (ctxs[q] == c) return fail(DMK_ERR_ARG, "context listed twice");
  }
  dmk_batch* b = new dmk_batch();
  b->n = n;
  b->ctx.assign(ctxs, ctxs + n);
  b->NS = ctxs[0]->NS;
  b->device = ctxs[0]->device;
  b->nsm = ctxs[0]->nsm;
  {
    // host threads for the per-member calls: one per 32 members, at most 7 besides the caller
    const int hw = int(std::thread::hardware_concurrency());
    const int workers = std::max(0, std::min({n / 32, 7, hw > 1 ? hw - 1 : 0}));
    b->pool = std::make_unique<HostPool>(workers, b->device);
  }
  if (cudaSetDevice(b->device) != cudaSuccess) {
    batch_free(b);
    return fail(DMK_ERR_CUDA, "cudaSetDevice failed");
  }
  if (int rc = batch_build(b)) {
    const std::string msg = g_err;
    batch_free(b);
    return fail(rc, msg);
  }
  *out = b;
  return 0;
}

int dmk_batch_solution(dmk_batch* b, const int* which, int n_which, dmk_solution_state* out) {
  if (!b || (n_which > 0 && (!which || !out))) return fail(DMK_ERR_ARG, "null argument");
  if (n_which < 0 || n_which > b->n) return fail(DMK_ERR_ARG, "n_which out of range");
  CK(cudaSetDevice(b->device));
  ++b->solutions;
  return batch_solution_impl(b, which, n_which, out);
}

int dmk_batch_stats(dmk_batch* b, double out[9]) {
  if (!b || !out) return fail(DMK_ERR_ARG, "null argument");
  out[0] = b->last_ms[0];
  out[1] = b->last_ms[1];
  out[2] = double(b->graph_launches);
  out[3] = double(b->passes);
  out[4] = double(b->iterations);
  out[5] = double(b->solutions);
  for (int k = 0; k < 3; ++k) out[6 + k] = b->host_ms[k];
  return 0;
}

void dmk_batch_destroy(dmk_batch* b) { batch_free(b); }

}  // extern "C"

namespace dmk {
HostPool* batch_pool(dmk_batch* b) { return b ? b->pool.get() : nullptr; }
int batch_size(const dmk_batch* b) { return b ? b->n : 0; }
dmk_ctx* batch_member(dmk_batch* b, int k) { return (b && k >= 0 && k < b->n) ? b->ctx[k] : nullptr; }
}  // namespace dmk

// ------------------------------------------------------------------ autotuner
// The constitutive evaluation at the context's current state (its solver F and time step), timed
// for every stress-kernel variant (register bound for 2, 3 or 4 resident blocks per SM up to 24
// slip systems) and voxel-chunk count (1, 2, 4); the fastest pair is kept.  The fields an
// evaluation changes (Fp, Lp, S, Fe, state) are copied to a scratch buffer first and restored after
// every trial, and the stress buffers are swapped back, so a solve after the tuning runs bit for bit
// as without it (the variants and chunk counts change the schedule, not the arithmetic).

namespace {

std::vector<std::pair<double*, size_t>> tuning_buffers(dmk_ctx* c) {
  const size_t N = size_t(c->N), NST = size_t(2 * c->NS);
  return {{c->Fp, 9 * N}, {c->Lp, 9 * N}, {c->S, 6 * N}, {c->Fe, 9 * N}, {c->state, NST * N}};
}

int copy_buffers(dmk_ctx* c, double* scratch, bool save) {
  size_t o = 0;
  for (const auto& b : tuning_buffers(c)) {
    CK(cudaMemcpyAsync(save ? scratch + o : b.first, save ? b.first : scratch + o, sizeof(double) * b.second,
                       cudaMemcpyDeviceToDevice, c->stream));
    o += b.second;
  }
  return 0;
}

int autotune_impl(dmk_ctx* c, int reps, double* report, int* n_report) {
  size_t total = 0;
  for (const auto& b : tuning_buffers(c)) total += b.second;
  size_t free_b = 0, total_b = 0;
  CK(cudaMemGetInfo(&free_b, &total_b));
  if (total * sizeof(double) + (size_t(1) << 30) > free_b)
    return fail(DMK_ERR_CUDA, "autotune: not enough free device memory for the state copy");
  double* scratch = nullptr;
  if (int rc = dalloc(&scratch, total)) return rc;
  std::unique_ptr<double, void (*)(double*)> guard(scratch, [](double* p) { cudaFree(p); });
  double* const P0 = c->P;
  double* const Pn0 = c->Pnew;
  const bool dot0_valid = c->dot0_valid;
  const int variant0 = c->stress_variant, chunks0 = c->nchunks;
  if (int rc = copy_buffers(c, scratch, true)) return rc;
  const double ms0 = c->last_ms[0];
  int best_v = variant0, best_k = chunks0, n = 0;
  double best = 1e300;
  const int nv = stress_variant_count(c->NS);
  for (int v = 0; v < nv; ++v)
    for (int k : {1, 2, 4}) {
      if (k > PASS_CHUNKS) continue;
      c->stress_variant = v;
      c->nchunks = k;
      double t = 1e300;
      for (int r = 0; r < std::max(1, reps); ++r) {
        const double before = c->last_ms[0];
        int st = 0;
        if (int rc = evaluate_constitutive(c, c->dt, nullptr, 0, &st)) return rc;
        t = std::min(t, c->last_ms[0] - before);
        c->P = P0;
        c->Pnew = Pn0;
        if (int rc = copy_buffers(c, scratch, false)) return rc;
      }
      if (report && n < 12) {
        report[3 * n] = stress_variant_blocks(c->NS, v);
        report[3 * n + 1] = k;
        report[3 * n + 2] = t;
      }
      ++n;
      if (t < best) {
        best = t;
        best_v = v;
        best_k = k;
      }
    }
  CK(cudaStreamSynchronize(c->stream));
  c->stress_variant = best_v;
  c->nchunks = best_k;
  c->last_ms[0] = ms0;
  (void)dot0_valid;   // the evaluation stores the increment-start rates the next one would compute
  if (n_report) *n_report = std::min(n, 12);
  return 0;
}

}  // namespace

extern "C" {

int dmk_autotune(dmk_ctx* c, int reps, double* report, int* n_report) {
  if (!c) return fail(DMK_ERR_ARG, "null argument");
  if (c->solver != 0) return fail(DMK_ERR_CONFIG, "the autotuner runs on the basic spectral scheme");
  CK(cudaSetDevice(c->device));
  return autotune_impl(c, reps, report, n_report);
}

int dmk_get_tuning(dmk_ctx* c, int* stress_blocks, int* chunks) {
  if (!c) return fail(DMK_ERR_ARG, "null argument");
  if (stress_blocks) *stress_blocks = stress_variant_blocks(c->NS, c->stress_variant);
  if (chunks) *chunks = c->nchunks;
  return 0;
}

int dmk_set_tuning(dmk_ctx* c, int stress_blocks, int chunks) {
  if (!c) return fail(DMK_ERR_ARG, "null argument");
  if (chunks < 1 || chunks > PASS_CHUNKS) return fail(DMK_ERR_ARG, "chunks must be 1 to 4");
  int v = -1;
  for (int k = 0; k < stress_variant_count(c->NS); ++k)
    if (stress_variant_blocks(c->NS, k) == stress_blocks) v = k;
  if (v < 0) return fail(DMK_ERR_ARG, "no stress-kernel variant for that block count");
  c->stress_variant = v;
  c->nchunks = chunks;
  return 0;
}

}  // extern "C"
