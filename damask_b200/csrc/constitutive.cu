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

#include <algorithm>
#include <cstdint>
#include <vector>

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

// warp-aggregated append of the entries that continue (voxel indices, or batch items) to a list;
// every thread of the block reaches this point
__device__ __forceinline__ void append(int* list_out, int* count_out, bool keep, int64_t entry) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned m = __ballot_sync(full, keep);
  if (m) {
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(count_out, __popc(m));
    base = __shfl_sync(full, base, leader);
    if (keep) list_out[base + __popc(m & ((1u << lane) - 1u))] = int(entry);
  }
}

// state and Newton iteration counters of one context, warp aggregated; every thread reaches this point
__device__ __forceinline__ void count_iterations(unsigned long long* counters, int dstate, int dnewton) {
  unsigned long long cs = dstate, cn = dnewton;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    cs += __shfl_down_sync(0xffffffffu, cs, o);
    cn += __shfl_down_sync(0xffffffffu, cn, o);
  }
  if ((threadIdx.x & 31) == 0 && counters && cs) {
    atomicAdd(&counters[1], cs);
    atomicAdd(&counters[2], cn);
  }
}

// the same for lanes of several contexts (r: the lane's context, -1 for none): lanes of one context
// are summed together, and one lane of each adds the sums to that context's counters
__device__ __forceinline__ void count_iterations_batch(const Fields* __restrict__ fs, int r, int dstate, int dnewton) {
  const unsigned peers = __match_any_sync(0xffffffffu, r);
  const unsigned cs = __reduce_add_sync(peers, unsigned(dstate));
  const unsigned cn = __reduce_add_sync(peers, unsigned(dnewton));
  const int lane = threadIdx.x & 31;
  if (r >= 0 && lane == __ffs(peers) - 1 && cs) {
    unsigned long long* counters = fs[r].counters;
    if (counters) {
      atomicAdd(&counters[1], (unsigned long long)cs);
      atomicAdd(&counters[2], (unsigned long long)cn);
    }
  }
}

// ------------------------------------------------------------------ per-voxel bodies of the passes
// Each takes the voxel's context (fields, pass work, time step) by reference, so that the kernels of
// one context (grid constants) and the batch kernels (tables of many contexts in device memory)
// share them.

// begin: F <- F - r, mechanical_restore, first substep control, state-iteration start; returns
// whether the voxel goes on to an integrateStress
template <int NS>
__device__ __forceinline__ bool begin_voxel(const PhaseConst<NS>& pc, const double* __restrict__ hs, double* xs,
                                            const Numerics& nm, const Fields& f, const PassWork& w, int64_t v,
                                            double dt, int apply_update, int use_dot0) {
  constexpr int NST = 2 * NS;
  const int64_t N = f.N;
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
  const bool keep = c.phase == PH_STRESS;
  if (!keep) finish_voxel(f, v, c);
  return keep;
}

// one integrateStress (integrateStateFPI:626-629); returns its Newton iterations
template <int NS>
__device__ __forceinline__ int stress_voxel(const PhaseConst<NS>& pc, const SysConst* __restrict__ sc, double* xs,
                                            const Numerics& nm, const Fields& f, const PassWork& w, int64_t v,
                                            double dt) {
  const int64_t N = f.N;
  int dnewton = 0;
  const double step = w.sub[N + v];
  double Lp[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) Lp[k] = f.Lp[k * N + v];
#pragma unroll
  for (int s = 0; s < NS; ++s) xs[s * pass_threads<NS>()] = 1.0 / f.state[s * N + v];
  double S[6], Fp[9], P[9], Fe[9];
  const double* Fp0s = (w.sub[v] == 0.0 ? f.Fp0 : w.Fp0s) + v;   // subFp0 (see sub_start)
  const int st = integrate_stress<NS>(pc, sc, nm, w.Fs + v, Fp0s, N, xs, step * dt, Lp, S, Fp, P, Fe,
                                      dnewton, w.adg + v, w.lo + v, w.dl + v);
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
  }
  w.ctl[v] = st == 0 ? PH_DOT1 : PH_CTRL;
  w.ctl[N + v] = st;
  w.ctl[2 * N + v] += 1;                                 // state iteration of this substep
  w.ctl[4 * N + v] += 1;                                 // state iterations, total
  w.ctl[5 * N + v] += dnewton;                           // Newton iterations, total
  return dnewton;
}

// state update and substep control up to the next integrateStress; returns whether the voxel
// continues
template <int NS>
__device__ __forceinline__ bool control_voxel(const PhaseConst<NS>& pc, const double* __restrict__ hs, double* xs,
                                              const Numerics& nm, const Fields& f, const PassWork& w, int64_t v,
                                              double dt) {
  const int64_t N = f.N;
  VoxelCtl c;
  load_ctl(w, N, v, c);
  advance<NS>(pc, hs, nm, f, w, v, dt, c, xs, w.adg + v, N);
  store_ctl(w, N, v, c);
  const bool keep = c.phase == PH_STRESS;
  if (!keep) finish_voxel(f, v, c);
  return keep;
}

}  // namespace

template <int NS>
__global__ void __launch_bounds__(pass_threads<NS>(), 4)
constitutive_begin_kernel(const __grid_constant__ PhaseConst<NS> pc, const __grid_constant__ Numerics nm,
                          const __grid_constant__ Fields f, const __grid_constant__ PassWork w, double dt,
                          int apply_update, int use_dot0, int64_t v_begin, int64_t v_end) {
  extern __shared__ double slots[];
  const double* hs = pc.hmat;
  double* xs = slots + hard_smem_doubles<NS>() + threadIdx.x;
  if constexpr (hard_smem_doubles<NS>() > 0) {
    stage_hardening<NS>(pc, slots);
    hs = slots;
  }
  __syncthreads();
  const int64_t v = v_begin + int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const bool keep = v < v_end && begin_voxel<NS>(pc, hs, xs, nm, f, w, v, dt, apply_update, use_dot0);
  append(w.list_out, w.count_out, keep, v);
}

// one state iteration of every listed voxel: integrateStress (integrateStateFPI:626-629).
// MINB: resident blocks per SM that the register allocation is bounded for (the variants the
// autotuner chooses from, stress_variant_blocks); three up to 24 systems by default (168 registers,
// a few spilled; 67 KB of shared memory per block at 24 systems): measured 5 % faster at 256^3 than
// two blocks without spills
template <int NS, int MINB>
__global__ void __launch_bounds__(pass_threads<NS>(), MINB)
constitutive_stress_kernel(const __grid_constant__ PhaseConst<NS> pc, const __grid_constant__ Numerics nm,
                           const __grid_constant__ Fields f, const __grid_constant__ PassWork w, double dt,
                           const int* __restrict__ list_in, int64_t n_in) {
  extern __shared__ double2 smem2[];
  SysConst* sc = reinterpret_cast<SysConst*>(smem2);
  double* xs = reinterpret_cast<double*>(sc + NS) + threadIdx.x;
  stage_sys_const<NS>(pc, sc);
  __syncthreads();
  const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const bool active = idx < n_in;
  const int dnewton = active ? stress_voxel<NS>(pc, sc, xs, nm, f, w, list_in[idx], dt) : 0;
  count_iterations(f.counters, active ? 1 : 0, dnewton);
}

// state update and substep control of every listed voxel up to its next
// integrateStress; the voxels that continue are appended to the next list
template <int NS>
__global__ void __launch_bounds__(pass_threads<NS>(), 4)
constitutive_control_kernel(const __grid_constant__ PhaseConst<NS> pc, const __grid_constant__ Numerics nm,
                            const __grid_constant__ Fields f, const __grid_constant__ PassWork w, double dt,
                            const int* __restrict__ list_in, int64_t n_in) {
  extern __shared__ double slots[];
  const double* hs = pc.hmat;
  double* xs = slots + hard_smem_doubles<NS>() + threadIdx.x;
  if constexpr (hard_smem_doubles<NS>() > 0) {
    stage_hardening<NS>(pc, slots);
    hs = slots;
  }
  __syncthreads();
  const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  int64_t v = 0;
  bool keep = false;
  if (idx < n_in) {
    v = list_in[idx];
    keep = control_voxel<NS>(pc, hs, xs, nm, f, w, v, dt);
  }
  append(w.list_out, w.count_out, keep, v);
}

// ------------------------------------------------------------------ batch kernels
// The passes of many contexts of one phase.  Items are the voxels of all contexts, numbered context
// after context (context r owns items [off[r], off[r + 1])); the lists hold item numbers.  Every
// item reads its context's fields, pass work and time step from the tables.  The stress and control
// kernels run on a fixed grid and loop over the entries that the previous kernel left in device
// memory, so that a CUDA graph repeats the passes without the host (build_batch_pass_graph).

template <int NS>
__global__ void __launch_bounds__(pass_threads<NS>(), 4)
constitutive_begin_batch_kernel(const __grid_constant__ PhaseConst<NS> pc, const __grid_constant__ Numerics nm,
                                const __grid_constant__ BatchTables t, int* list_out, int* count_out) {
  extern __shared__ double slots[];
  const double* hs = pc.hmat;
  double* xs = slots + hard_smem_doubles<NS>() + threadIdx.x;
  if constexpr (hard_smem_doubles<NS>() > 0) {
    stage_hardening<NS>(pc, slots);
    hs = slots;
  }
  __syncthreads();
  const int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  bool keep = false;
  if (g < t.n_items) {
    const int r = t.ctx_of[g];
    if (t.active[r])
      keep = begin_voxel<NS>(pc, hs, xs, nm, t.f[r], t.w[r], g - t.off[r], t.dt[r], t.apply[r], t.use_dot0[r]);
  }
  append(list_out, count_out, keep, g);
}

template <int NS>
__global__ void __launch_bounds__(pass_threads<NS>(), NS > 24 ? 1 : 3)
constitutive_stress_batch_kernel(const __grid_constant__ PhaseConst<NS> pc, const __grid_constant__ Numerics nm,
                                 const __grid_constant__ BatchTables t, const int* __restrict__ list_in,
                                 const int* __restrict__ count_in) {
  const int64_t n_in = *count_in;
  const int64_t first = int64_t(blockIdx.x) * blockDim.x;
  if (first >= n_in) return;
  extern __shared__ double2 smem2[];
  SysConst* sc = reinterpret_cast<SysConst*>(smem2);
  double* xs = reinterpret_cast<double*>(sc + NS) + threadIdx.x;
  stage_sys_const<NS>(pc, sc);
  __syncthreads();
  for (int64_t base = first; base < n_in; base += int64_t(gridDim.x) * blockDim.x) {
    const int64_t idx = base + threadIdx.x;
    int r = -1, dnewton = 0;
    if (idx < n_in) {
      const int64_t g = list_in[idx];
      r = t.ctx_of[g];
      dnewton = stress_voxel<NS>(pc, sc, xs, nm, t.f[r], t.w[r], g - t.off[r], t.dt[r]);
    }
    count_iterations_batch(t.f, r, r >= 0 ? 1 : 0, dnewton);
  }
}

template <int NS>
__global__ void __launch_bounds__(pass_threads<NS>(), 4)
constitutive_control_batch_kernel(const __grid_constant__ PhaseConst<NS> pc, const __grid_constant__ Numerics nm,
                                  const __grid_constant__ BatchTables t, const int* __restrict__ list_in,
                                  const int* __restrict__ count_in, int* list_out, int* count_out) {
  const int64_t n_in = *count_in;
  const int64_t first = int64_t(blockIdx.x) * blockDim.x;
  if (first >= n_in) return;
  extern __shared__ double slots[];
  const double* hs = pc.hmat;
  double* xs = slots + hard_smem_doubles<NS>() + threadIdx.x;
  if constexpr (hard_smem_doubles<NS>() > 0) {
    stage_hardening<NS>(pc, slots);
    hs = slots;
  }
  __syncthreads();
  for (int64_t base = first; base < n_in; base += int64_t(gridDim.x) * blockDim.x) {
    const int64_t idx = base + threadIdx.x;
    int64_t g = 0;
    bool keep = false;
    if (idx < n_in) {
      g = list_in[idx];
      const int r = t.ctx_of[g];
      keep = control_voxel<NS>(pc, hs, xs, nm, t.f[r], t.w[r], g - t.off[r], t.dt[r]);
    }
    append(list_out, count_out, keep, g);
  }
}

// statuses, entry counts and pass counter of an evaluation start at zero
__global__ void batch_prologue_kernel(int* count, int* status, int n_ctx, int* iter) {
  for (int i = threadIdx.x; i < n_ctx; i += blockDim.x) status[i] = 0;
  if (threadIdx.x == 0) {
    count[0] = count[1] = 0;
    iter[0] = iter[1] = 0;
  }
}

// after a pass: its input list is spent (count_done = 0); the loop goes on while the next list has
// entries, and stops with iter[1] = 1 once max_passes passes have run
__global__ void batch_flip_kernel(int* count_done, const int* count_next, int* iter, int max_passes,
                                  cudaGraphConditionalHandle h) {
  *count_done = 0;
  const int it = ++iter[0];
  unsigned go = *count_next > 0 ? 1u : 0u;
  if (go && it >= max_passes) {
    iter[1] = 1;
    go = 0u;
  }
  cudaGraphSetConditional(h, go);
}

template <int NS>
cudaError_t launch_constitutive_begin(const PhaseConst<NS>& pc, const Numerics& nm, const Fields& f,
                                      const PassWork& w, double dt, int apply_update, int use_dot0, int64_t v_begin,
                                      int64_t v_end, cudaStream_t s) {
  const size_t smem = (hard_smem_doubles<NS>() + size_t(2 * NS) * pass_threads<NS>()) * sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(constitutive_begin_kernel<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(smem));
  if (e != cudaSuccess) return e;
  if (v_end <= v_begin) return cudaSuccess;
  const int nb = int((v_end - v_begin + pass_threads<NS>() - 1) / pass_threads<NS>());
  constitutive_begin_kernel<NS><<<nb, pass_threads<NS>(), smem, s>>>(pc, nm, f, w, dt, apply_update, use_dot0, v_begin,
                                                                v_end);
  return cudaGetLastError();
}

// stress kernel variants: up to 24 systems bounded for 3 (default), 2 or 4 resident blocks per SM;
// 48 systems (64-thread blocks, three fit by shared memory) one variant
int stress_variant_count(int ns) { return ns > 24 ? 1 : 3; }
int stress_variant_blocks(int ns, int variant) {
  if (ns > 24) return 1;
  static const int blocks[3] = {3, 2, 4};
  return blocks[variant >= 0 && variant < 3 ? variant : 0];
}

namespace {
template <int NS, int MINB>
cudaError_t launch_stress(const PhaseConst<NS>& pc, const Numerics& nm, const Fields& f, const PassWork& w, double dt,
                          const int* list_in, int64_t n_in, int nb, size_t smem, cudaStream_t s) {
  cudaError_t e = cudaFuncSetAttribute(constitutive_stress_kernel<NS, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(smem));
  if (e != cudaSuccess) return e;
  constitutive_stress_kernel<NS, MINB><<<nb, pass_threads<NS>(), smem, s>>>(pc, nm, f, w, dt, list_in, n_in);
  return cudaGetLastError();
}
}  // namespace

template <int NS>
cudaError_t launch_constitutive_pass(const PhaseConst<NS>& pc, const Numerics& nm, const Fields& f,
                                     const PassWork& w, double dt, const int* list_in, int64_t n_in, cudaStream_t s,
                                     int variant) {
  const size_t smem_s = size_t(NS) * sizeof(SysConst) + size_t(stress_slots<NS>()) * pass_threads<NS>() * sizeof(double);
  const size_t smem_c = (hard_smem_doubles<NS>() + size_t(2 * NS) * pass_threads<NS>()) * sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(constitutive_control_kernel<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(smem_c));
  if (e != cudaSuccess) return e;
  const int nb = int((n_in + pass_threads<NS>() - 1) / pass_threads<NS>());
  if constexpr (NS > 24) {
    e = launch_stress<NS, 1>(pc, nm, f, w, dt, list_in, n_in, nb, smem_s, s);
  } else {
    switch (stress_variant_blocks(NS, variant)) {
      case 2: e = launch_stress<NS, 2>(pc, nm, f, w, dt, list_in, n_in, nb, smem_s, s); break;
      case 4: e = launch_stress<NS, 4>(pc, nm, f, w, dt, list_in, n_in, nb, smem_s, s); break;
      default: e = launch_stress<NS, 3>(pc, nm, f, w, dt, list_in, n_in, nb, smem_s, s); break;
    }
  }
  if (e != cudaSuccess) return e;
  constitutive_control_kernel<NS><<<nb, pass_threads<NS>(), smem_c, s>>>(pc, nm, f, w, dt, list_in, n_in);
  return cudaGetLastError();
}

namespace {
template <int NS>
int resident_blocks(const void* fn, size_t smem, int nsm, int64_t n_items) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, pass_threads<NS>(), smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  const int64_t need = (n_items + pass_threads<NS>() - 1) / pass_threads<NS>();
  return int(std::max<int64_t>(1, std::min<int64_t>(int64_t(per_sm) * nsm, need)));
}
}  // namespace

// One constitutive evaluation of every active context of a batch as a CUDA graph: prologue, begin
// kernel (list A), then a while node whose body runs two passes (A -> B, B -> A) and whose
// condition is set on the device after each pass from the next list's entry count.
template <int NS>
cudaError_t build_batch_pass_graph(const PhaseConst<NS>& pc, const Numerics& nm, const BatchTables& t,
                                   const BatchPassBuffers& b, int nsm, cudaStream_t s, cudaGraph_t* out) {
  const size_t smem_b = (hard_smem_doubles<NS>() + size_t(2 * NS) * pass_threads<NS>()) * sizeof(double);
  const size_t smem_s = size_t(NS) * sizeof(SysConst) + size_t(stress_slots<NS>()) * pass_threads<NS>() * sizeof(double);
  const size_t smem_c = smem_b;
  cudaError_t e = cudaFuncSetAttribute(constitutive_begin_batch_kernel<NS>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem_b));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(constitutive_stress_batch_kernel<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(smem_s));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(constitutive_control_batch_kernel<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(smem_c));
  if (e != cudaSuccess) return e;
  if (t.n_items <= 0 || t.n_items > INT32_MAX) return cudaErrorInvalidValue;
  const int nb_begin = int((t.n_items + pass_threads<NS>() - 1) / pass_threads<NS>());
  const int nb_s = resident_blocks<NS>(reinterpret_cast<const void*>(constitutive_stress_batch_kernel<NS>), smem_s, nsm,
                                       t.n_items);
  const int nb_c = resident_blocks<NS>(reinterpret_cast<const void*>(constitutive_control_batch_kernel<NS>), smem_c,
                                       nsm, t.n_items);
  cudaGraph_t g = nullptr;
  if ((e = cudaGraphCreate(&g, 0)) != cudaSuccess) return e;
  auto bail = [&](cudaError_t err) {
    cudaGraphDestroy(g);
    return err;
  };
  cudaGraphConditionalHandle h;
  if ((e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault)) != cudaSuccess) return bail(e);
  // prologue and begin
  if ((e = cudaStreamBeginCaptureToGraph(s, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
    return bail(e);
  batch_prologue_kernel<<<1, 256, 0, s>>>(b.count, b.status, b.n_ctx, b.iter);
  constitutive_begin_batch_kernel<NS><<<nb_begin, pass_threads<NS>(), smem_b, s>>>(pc, nm, t, b.list[0], b.count);
  cudaGraph_t captured = nullptr;
  e = cudaStreamEndCapture(s, &captured);
  if (e != cudaSuccess) return bail(e);
  size_t nn = 0;
  if ((e = cudaGraphGetNodes(g, nullptr, &nn)) != cudaSuccess) return bail(e);
  std::vector<cudaGraphNode_t> nodes(nn);
  if ((e = cudaGraphGetNodes(g, nodes.data(), &nn)) != cudaSuccess) return bail(e);
  cudaGraphNode_t leaf = nullptr;
  for (cudaGraphNode_t n : nodes) {
    size_t nd = 0;
    if ((e = cudaGraphNodeGetDependentNodes(n, nullptr, &nd)) != cudaSuccess) return bail(e);
    if (nd == 0) leaf = n;
  }
  if (!leaf) return bail(cudaErrorInvalidValue);
  // the loop of passes
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cond;
  if ((e = cudaGraphAddNode(&cond, g, &leaf, 1, &cp)) != cudaSuccess) return bail(e);
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  if ((e = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
      cudaSuccess)
    return bail(e);
  for (int p = 0; p < 2; ++p) {
    const int a = p, z = 1 - p;
    constitutive_stress_batch_kernel<NS><<<nb_s, pass_threads<NS>(), smem_s, s>>>(pc, nm, t, b.list[a], b.count + a);
    constitutive_control_batch_kernel<NS><<<nb_c, pass_threads<NS>(), smem_c, s>>>(pc, nm, t, b.list[a], b.count + a,
                                                                                   b.list[z], b.count + z);
    batch_flip_kernel<<<1, 1, 0, s>>>(b.count + a, b.count + z, b.iter, b.max_passes, h);
  }
  e = cudaStreamEndCapture(s, &captured);
  if (e != cudaSuccess) return bail(e);
  *out = g;
  return cudaSuccess;
}

#define DMK_INSTANTIATE(NS)                                                                                         \
  template cudaError_t launch_constitutive_begin<NS>(const PhaseConst<NS>&, const Numerics&, const Fields&,          \
                                                     const PassWork&, double, int, int, int64_t, int64_t,          \
                                                     cudaStream_t);                                                 \
  template cudaError_t launch_constitutive_pass<NS>(const PhaseConst<NS>&, const Numerics&, const Fields&,           \
                                                    const PassWork&, double, const int*, int64_t, cudaStream_t,    \
                                                    int);                                                          \
  template cudaError_t build_batch_pass_graph<NS>(const PhaseConst<NS>&, const Numerics&, const BatchTables&,    \
                                                  const BatchPassBuffers&, int, cudaStream_t, cudaGraph_t*);
DMK_INSTANTIATE(12)
DMK_INSTANTIATE(18)
DMK_INSTANTIATE(24)
DMK_INSTANTIATE(48)
#undef DMK_INSTANTIATE

}  // namespace dmk
