// Pass kernels of the constitutive update (see constitutive.cuh for the scheme).
//
//  constitutive_begin_kernel  every voxel: fused field update F <- F - r, phase restore
//                             (mechanical_restore), substep set-up, then control up to
//                             the first integrateStress.
//  constitutive_stress_kernel every voxel of the list: one integrateStress (the Newton
//                             loop; compute bound, register resident)
//  constitutive_control_kernel every voxel of the list: state update and substep control
//                             up to the next integrateStress (memory bound, high
//                             occupancy); voxels that continue are appended to the next list.
#include "kernels.cuh"
#include "constitutive.cuh"

namespace dmk {

namespace {

// voxel finished: iteration record and worst status
__device__ __forceinline__ void finish_voxel(const Fields& f, int64_t v, const VoxelCtl& c) {
  const int64_t N = f.N;
  if (f.iter) {
    f.iter[v] = c.nstate;
    f.iter[N + v] = c.newton;
    f.iter[2 * N + v] = c.nsub;
    f.iter[3 * N + v] = c.status;
  }
  if (c.status != 0) atomicMax(f.status, 2);               // STATUS_FAIL_PHASE_MECHANICAL
}

// warp-aggregated append of the continuing voxels and of the iteration counters;
// every thread of the block reaches this point
__device__ __forceinline__ void append_and_count(const Fields& f, const PassWork& w, bool keep, int64_t v, int dstate,
                                                 int dnewton) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned m = __ballot_sync(full, keep);
  if (m) {
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(w.count_out, __popc(m));
    base = __shfl_sync(full, base, leader);
    if (keep) w.list_out[base + __popc(m & ((1u << lane) - 1u))] = int(v);
  }
  unsigned long long cs = dstate, cn = dnewton;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    cs += __shfl_down_sync(full, cs, o);
    cn += __shfl_down_sync(full, cn, o);
  }
  if (lane == 0 && f.counters && (cs | cn)) {
    atomicAdd(&f.counters[1], cs);
    atomicAdd(&f.counters[2], cn);
  }
}

}  // namespace

template <int NS>
__global__ void __launch_bounds__(pass_threads<NS>(), 4)
constitutive_begin_kernel(const __grid_constant__ PhaseConst<NS> pc, const __grid_constant__ Numerics nm,
                          const __grid_constant__ Fields f, const __grid_constant__ PassWork w, double dt,
                          int apply_update, int use_dot0, int64_t v_begin, int64_t v_end) {
  extern __shared__ double slots[];
  constexpr int NST = 2 * NS;
  double* hs = slots;
  double* xs = slots + NS * NS + threadIdx.x;
  stage_hardening<NS>(pc, hs);
  __syncthreads();
  const int64_t v = v_begin + int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t N = f.N;
  bool keep = false;
  if (v < v_end) {
    // F <- F - r (the Richardson/Anderson update of the previous evaluation), phase F
    double Fn[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      double x = f.Fsol[k * N + v];
      if (apply_update) {
        x = x - f.r[k * N + v];
        f.Fsol[k * N + v] = x;
      }
      f.F[k * N + v] = x;
      Fn[k] = x;
    }
    // mechanical_restore and the first substep control step (status ITERATING: subStep =
    // r_cutback / r_cutback = 1, nothing to restore beyond the increment-start values,
    // which stay where they are while stepFrac = 0; Lp is kept as warm start)
    VoxelCtl c;
    c.status = 1;
    c.it = 0;
    c.nsub = 0;
    c.nstate = 0;
    c.newton = 0;
    c.stepFrac = 0.0;
    c.step = nm.r_cutback * (1.0 / nm.r_cutback);
    if (!(c.step > nm.r_cutback_min)) {
      c.phase = PH_DONE;
    } else {
      c.nsub = 1;
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        const double f0 = f.F0[k * N + v];
        w.Fs[k * N + v] = fma(c.step, Fn[k] - f0, f0);
      }
      // start of the state iteration (integrateStateFPI:614-620) at S0 and state0.  The rate
      // depends on the increment-start values only, so every evaluation of an increment after
      // the first reads it back (use_dot0) instead of evaluating the kinetics and hardening.
      bool bad = false;
      if (use_dot0) {
#pragma unroll 12
        for (int i = 0; i < NST; ++i) {
          const double d = w.dot0[i * N + v];
          bad |= isnan(d);
          xs[i * pass_threads<NS>()] = d;
        }
      } else {
        double s0[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) s0[k] = f.S0[k * N + v];
        bad = dot_state_slots<NS>(pc, hs, s0, f.state0, N, v, xs, nullptr, 0);
#pragma unroll 12
        for (int i = 0; i < NST; ++i) w.dot0[i * N + v] = xs[i * pass_threads<NS>()];
      }
      if (bad) {
        double s6[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) s6[k] = f.S0[k * N + v];
        // STATUS_FAIL_PHASE_MECHANICAL_STATE: restore as the cutback branch does and continue
        // with the general control flow
#pragma unroll
        for (int k = 0; k < 9; ++k) f.Fp[k * N + v] = f.Fp0[k * N + v];
#pragma unroll
        for (int k = 0; k < 6; ++k) f.S[k * N + v] = s6[k];
#pragma unroll 12
        for (int i = 0; i < NST; ++i) f.state[i * N + v] = f.state0[i * N + v];
        c.status = 3;
        c.phase = PH_CTRL;
        advance<NS>(pc, hs, nm, f, w, v, dt, c, xs, nullptr, 0);
      } else {
        const double dts = c.step * dt;
        double* D0 = w.D + v;                               // dotState generation 0
#pragma unroll 12
        for (int i = 0; i < NST; ++i) {
          const double d = xs[i * pass_threads<NS>()];
          f.state[i * N + v] = fma(d, dts, f.state0[i * N + v]);
          D0[i * N] = d;
        }
        // S is written by the first successful integrateStress (a failure restores S0)
        c.phase = PH_STRESS;
      }
    }
    store_ctl(w, N, v, c);
    keep = c.phase == PH_STRESS;
    if (!keep) finish_voxel(f, v, c);
  }
  append_and_count(f, w, keep, v, 0, 0);
}

// one state iteration of every listed voxel: integrateStress (integrateStateFPI:626-629)
template <int NS>
__global__ void __launch_bounds__(pass_threads<NS>())
constitutive_stress_kernel(const __grid_constant__ PhaseConst<NS> pc, const __grid_constant__ Numerics nm,
                           const __grid_constant__ Fields f, const __grid_constant__ PassWork w, double dt,
                           const int* __restrict__ list_in, int64_t n_in) {
  extern __shared__ double2 smem2[];
  SysConst* sc = reinterpret_cast<SysConst*>(smem2);
  double* xs = reinterpret_cast<double*>(sc + NS) + threadIdx.x;
  stage_sys_const<NS>(pc, sc);
  __syncthreads();
  const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t N = f.N;
  int dnewton = 0;
  const bool active = idx < n_in;
  if (active) {
    const int64_t v = list_in[idx];
    const double step = w.sub[N + v];
    double Lp[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) Lp[k] = f.Lp[k * N + v];
#pragma unroll
    for (int s = 0; s < NS; ++s) xs[s * pass_threads<NS>()] = 1.0 / f.state[s * N + v];
    double S[6], Fp[9], P[9], Fe[9];
    const double* Fp0s = (w.sub[v] == 0.0 ? f.Fp0 : w.Fp0s) + v;   // subFp0 (see sub_start)
    const int st = integrate_stress<NS>(pc, sc, nm, w.Fs + v, Fp0s, N, xs, step * dt, Lp, S, Fp, P, Fe,
                                        dnewton);
    if (st == 0) {
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        f.Lp[k * N + v] = Lp[k];
        f.Fp[k * N + v] = Fp[k];
        f.P[k * N + v] = P[k];
        f.Fe[k * N + v] = Fe[k];
      }
#pragma unroll
      for (int k = 0; k < 6; ++k) f.S[k * N + v] = S[k];
#pragma unroll
      for (int s = 0; s < NS; ++s) w.adg[s * N + v] = xs[(2 * NS + s) * pass_threads<NS>()];
    }
    w.ctl[v] = st == 0 ? PH_DOT1 : PH_CTRL;
    w.ctl[N + v] = st;
    w.ctl[2 * N + v] += 1;                                 // state iteration of this substep
    w.ctl[4 * N + v] += 1;                                 // state iterations, total
    w.ctl[5 * N + v] += dnewton;                           // Newton iterations, total
  }
  // iteration counters (warp aggregated)
  unsigned long long cs = active ? 1 : 0, cn = dnewton;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    cs += __shfl_down_sync(0xffffffffu, cs, o);
    cn += __shfl_down_sync(0xffffffffu, cn, o);
  }
  if ((threadIdx.x & 31) == 0 && f.counters && cs) {
    atomicAdd(&f.counters[1], cs);
    atomicAdd(&f.counters[2], cn);
  }
}

// state update and substep control of every listed voxel up to its next
// integrateStress; the voxels that continue are appended to the next list
template <int NS>
__global__ void __launch_bounds__(pass_threads<NS>(), 4)
constitutive_control_kernel(const __grid_constant__ PhaseConst<NS> pc, const __grid_constant__ Numerics nm,
                            const __grid_constant__ Fields f, const __grid_constant__ PassWork w, double dt,
                            const int* __restrict__ list_in, int64_t n_in) {
  extern __shared__ double slots[];
  double* hs = slots;
  double* xs = slots + NS * NS + threadIdx.x;
  stage_hardening<NS>(pc, hs);
  __syncthreads();
  const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t N = f.N;
  bool keep = false;
  int64_t v = 0;
  if (idx < n_in) {
    v = list_in[idx];
    VoxelCtl c;
    load_ctl(w, N, v, c);
    advance<NS>(pc, hs, nm, f, w, v, dt, c, xs, w.adg + v, N);
    store_ctl(w, N, v, c);
    keep = c.phase == PH_STRESS;
    if (!keep) finish_voxel(f, v, c);
  }
  append_and_count(f, w, keep, v, 0, 0);
}

template <int NS>
cudaError_t launch_constitutive_begin(const PhaseConst<NS>& pc, const Numerics& nm, const Fields& f,
                                      const PassWork& w, double dt, int apply_update, int use_dot0, int64_t v_begin,
                                      int64_t v_end, cudaStream_t s) {
  const size_t smem = (size_t(NS) * NS + size_t(2 * NS) * pass_threads<NS>()) * sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(constitutive_begin_kernel<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(smem));
  if (e != cudaSuccess) return e;
  if (v_end <= v_begin) return cudaSuccess;
  const int nb = int((v_end - v_begin + pass_threads<NS>() - 1) / pass_threads<NS>());
  constitutive_begin_kernel<NS><<<nb, pass_threads<NS>(), smem, s>>>(pc, nm, f, w, dt, apply_update, use_dot0, v_begin,
                                                                v_end);
  return cudaGetLastError();
}

template <int NS>
cudaError_t launch_constitutive_pass(const PhaseConst<NS>& pc, const Numerics& nm, const Fields& f,
                                     const PassWork& w, double dt, const int* list_in, int64_t n_in, cudaStream_t s) {
  const size_t smem_s = size_t(NS) * sizeof(SysConst) + size_t(stress_slots<NS>()) * pass_threads<NS>() * sizeof(double);
  const size_t smem_c = (size_t(NS) * NS + size_t(2 * NS) * pass_threads<NS>()) * sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(constitutive_stress_kernel<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(smem_s));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(constitutive_control_kernel<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem_c));
  if (e != cudaSuccess) return e;
  const int nb = int((n_in + pass_threads<NS>() - 1) / pass_threads<NS>());
  constitutive_stress_kernel<NS><<<nb, pass_threads<NS>(), smem_s, s>>>(pc, nm, f, w, dt, list_in, n_in);
  constitutive_control_kernel<NS><<<nb, pass_threads<NS>(), smem_c, s>>>(pc, nm, f, w, dt, list_in, n_in);
  return cudaGetLastError();
}

#define DMK_INSTANTIATE(NS)                                                                                         \
  template cudaError_t launch_constitutive_begin<NS>(const PhaseConst<NS>&, const Numerics&, const Fields&,          \
                                                     const PassWork&, double, int, int, int64_t, int64_t,          \
                                                     cudaStream_t);                                                 \
  template cudaError_t launch_constitutive_pass<NS>(const PhaseConst<NS>&, const Numerics&, const Fields&,           \
                                                    const PassWork&, double, const int*, int64_t, cudaStream_t);
DMK_INSTANTIATE(12)
DMK_INSTANTIATE(18)
DMK_INSTANTIATE(24)
DMK_INSTANTIATE(48)
#undef DMK_INSTANTIATE

}  // namespace dmk
