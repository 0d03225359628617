// The increment loop of the grid driver (src/grid/DAMASK_grid.f90:288-460) for the mechanical
// field, behind the C-ABI: time stepping with geometric fractions, the global cutback (time step
// halved up to N_cutback_max times, then IO_error 950), the guess flag, restart skipping, and the
// calls of the five plugin procedures.  The plugin is a table of function pointers, so the same loop
// drives the CUDA context (dmk_grid_run_ctx) and any other implementation of the procedures.
#include <cmath>
#include <string>
#include <vector>

#include "../../include/damask_b200.h"
#include "host_parallel.h"

namespace dmk {
int record_error(int code, const std::string& msg);
int batch_size(const dmk_batch* b);
dmk_ctx* batch_member(dmk_batch* b, int k);
HostPool* batch_pool(dmk_batch* b);
}

namespace {

// math_geometricFraction, math.f90:1222-1234
double geometric_fraction(double r, int i, int N) {
  if (std::fabs(r - 1.0) <= 1.0e-9) return 1.0 / double(N);
  return (1.0 - r) * std::pow(r, i) / (r - std::pow(r, N + 1));
}

int ctx_forward(void* c, int cutBack, int guess, double dt, double dt_old, double t_remaining, const dmk_bc* def,
                const dmk_bc* stress, const double q[4]) {
  return dmk_mech_forward(static_cast<dmk_ctx*>(c), cutBack, guess, dt, dt_old, t_remaining, def, stress, q);
}
int ctx_solution(void* c, dmk_solution_state* out) { return dmk_mech_solution(static_cast<dmk_ctx*>(c), out); }
int ctx_update_coords(void* c) { return dmk_mech_update_coords(static_cast<dmk_ctx*>(c)); }
int ctx_materialpoint_forward(void* c) { return dmk_materialpoint_forward(static_cast<dmk_ctx*>(c)); }

// One member of dmk_batch_run: the loop variables of dmk_grid_run, and where the loop stands.
struct Member {
  const dmk_loadstep* steps = nullptr;
  int n_steps = 0;
  int l = 0, inc = 0, total = 0, cutBackLevel = 0, stepFraction = 0;
  double t = 0.0, Delta_t = 1.0, Delta_t_prev = 1.0, t_0 = 0.0;
  bool cutBack = false, guess = true, in_increment = false, done = false;
};

constexpr int kSubStepFactor = 2;                      // subStepFactor (DAMASK_grid.f90:80)

int substeps(int level) { return int(std::lround(std::pow(double(kSubStepFactor), double(level)))); }

// Runs member m up to its next solution request (forward and materialpoint_forward done): 1, or 0
// when it has run all its increments, or an error code.
int advance(Member& m, dmk_ctx* c, int max_increments) {
  for (;;) {
    if (m.done) return 0;
    if (!m.in_increment) {
      if (m.l >= m.n_steps || (max_increments > 0 && m.total >= max_increments)) {
        m.done = true;
        return 0;
      }
      const dmk_loadstep& lc = m.steps[m.l];
      if (m.inc == 0) {
        m.t_0 = m.t;
        m.guess = lc.estimate_rate != 0;
      }
      ++m.inc;
      ++m.total;
      m.Delta_t_prev = m.Delta_t;
      m.Delta_t = lc.t * geometric_fraction(lc.r, m.inc, lc.N) * std::pow(double(kSubStepFactor), -double(m.cutBackLevel));
      m.stepFraction = 0;
      m.in_increment = true;
    }
    const dmk_loadstep& lc = m.steps[m.l];
    if (m.stepFraction < substeps(m.cutBackLevel)) {
      const double t_remaining = lc.t + m.t_0 - m.t;
      m.t = m.t + m.Delta_t;
      ++m.stepFraction;
      int rc = dmk_mech_forward(c, m.cutBack ? 1 : 0, m.guess ? 1 : 0, m.Delta_t, m.Delta_t_prev, t_remaining,
                                &lc.deformation, &lc.stress, lc.q_rot);
      if (rc) return rc;
      if (!m.cutBack && (rc = dmk_materialpoint_forward(c))) return rc;
      return 1;
    }
    // all substeps of the increment converged
    m.cutBackLevel = m.cutBackLevel > 0 ? m.cutBackLevel - 1 : 0;
    m.in_increment = false;
    if (m.inc >= lc.N) {
      ++m.l;
      m.inc = 0;
    }
  }
}

}  // namespace

extern "C" {

int dmk_batch_run(dmk_batch* batch, const dmk_loadstep* const* steps, const int* n_steps, int N_cutback_max,
                  int max_increments, dmk_batch_increment_cb cb, void* user, int* status) {
  if (!batch || !steps || !n_steps || !status) return dmk::record_error(DMK_ERR_ARG, "null argument");
  const int n = dmk::batch_size(batch);
  std::vector<Member> m(n);
  for (int k = 0; k < n; ++k) {
    status[k] = 0;
    if (!steps[k] || n_steps[k] < 1) return dmk::record_error(DMK_ERR_ARG, "every member needs load steps");
    for (int l = 0; l < n_steps[k]; ++l)
      if (steps[k][l].N < 1 || !(steps[k][l].t > 0.0) || !(steps[k][l].r > 0.0))
        return dmk::record_error(DMK_ERR_CONFIG, "load step needs N >= 1, t > 0 and r > 0");
    m[k].steps = steps[k];
    m[k].n_steps = n_steps[k];
  }
  // the members' own calls (forward, materialpoint_forward, coordinates) run on the batch's host
  // threads; the callbacks run on this thread, in member order
  dmk::HostPool* pool = dmk::batch_pool(batch);
  std::string msg;
  std::vector<int> waiting, next, state(n, 0);   // state: the result of advance (1: waiting)
  auto advance_all = [&](const std::vector<int>& members) -> int {
    return pool->run(int(members.size()), [&](int j) -> int {
      const int k = members[j];
      const int rc = advance(m[k], dmk::batch_member(batch, k), max_increments);
      state[k] = rc;
      return rc < 0 ? rc : 0;
    }, &msg);
  };
  std::vector<int> all(n);
  for (int k = 0; k < n; ++k) all[k] = k;
  if (int rc = advance_all(all)) return dmk::record_error(rc, msg);
  for (int k = 0; k < n; ++k)
    if (state[k] == 1) waiting.push_back(k);
  std::vector<dmk_solution_state> sol;
  while (!waiting.empty()) {
    sol.assign(waiting.size(), dmk_solution_state{});
    if (int rc = dmk_batch_solution(batch, waiting.data(), int(waiting.size()), sol.data())) return rc;
    // coordinates of the converged members
    int rc = pool->run(int(waiting.size()), [&](int j) -> int {
      return (sol[j].converged && sol[j].stagConverged) ? dmk_mech_update_coords(dmk::batch_member(batch, waiting[j]))
                                                        : 0;
    }, &msg);
    if (rc) return dmk::record_error(rc, msg);
    next.clear();
    for (size_t j = 0; j < waiting.size(); ++j) {
      const int k = waiting[j];
      Member& s = m[k];
      const dmk_solution_state& o = sol[j];
      if (o.converged && o.stagConverged) {
        s.Delta_t_prev = s.Delta_t;
        s.cutBack = false;
        s.guess = true;
        if (cb) {
          dmk_increment_info info{s.total, s.t, s.cutBackLevel, 1, o.iterationsNeeded, o.residualEvals, s.l, s.inc};
          for (int q = 0; q < 9; ++q) info.P_av[q] = o.P_av[q];
          if (cb(k, &info, user)) s.done = true;
        }
      } else if (s.cutBackLevel < N_cutback_max) {
        s.cutBack = true;
        s.stepFraction = (s.stepFraction - 1) * kSubStepFactor;
        ++s.cutBackLevel;
        s.t = s.t - s.Delta_t;
        s.Delta_t = s.Delta_t / double(kSubStepFactor);
      } else {                                         // IO_error 950 for this member; the others go on
        status[k] = DMK_ERR_NOT_CONVERGED;
        s.done = true;
      }
    }
    if ((rc = advance_all(waiting))) return dmk::record_error(rc, msg);
    for (int k : waiting)
      if (state[k] == 1) next.push_back(k);
    waiting.swap(next);
  }
  return 0;
}

int dmk_grid_run(const dmk_grid_solver* s, const dmk_loadstep* steps, int n_steps, int N_cutback_max,
                 int restart_inc, int max_increments, dmk_increment_cb cb, void* user) {
  if (!s || !steps || n_steps < 1 || !s->forward || !s->solution || !s->update_coords || !s->materialpoint_forward)
    return dmk::record_error(DMK_ERR_ARG, "null argument");
  for (int l = 0; l < n_steps; ++l)
    if (steps[l].N < 1 || !(steps[l].t > 0.0) || !(steps[l].r > 0.0))
      return dmk::record_error(DMK_ERR_CONFIG, "load step needs N >= 1, t > 0 and r > 0");
  constexpr int ssf = 2;                                   // subStepFactor (DAMASK_grid.f90:80)
  double t = 0.0, Delta_t = 1.0, Delta_t_prev, t_0 = 0.0;
  int cutBackLevel = 0, total = 0;
  bool cutBack = false, guess = steps[0].estimate_rate != 0;
  for (int l = 0; l < n_steps; ++l) {
    const dmk_loadstep& lc = steps[l];
    t_0 = t;
    guess = lc.estimate_rate != 0;
    for (int inc = 1; inc <= lc.N; ++inc) {
      if (max_increments > 0 && total >= max_increments) return 0;
      ++total;
      Delta_t_prev = Delta_t;
      Delta_t = lc.t * geometric_fraction(lc.r, inc, lc.N) * std::pow(double(ssf), -double(cutBackLevel));
      if (total <= restart_inc) {                          // DAMASK_grid.f90:301-303
        t = t + Delta_t;
        guess = true;
        continue;
      }
      int stepFraction = 0;
      while (stepFraction < int(std::lround(std::pow(double(ssf), double(cutBackLevel))))) {
        const double t_remaining = lc.t + t_0 - t;
        t = t + Delta_t;
        ++stepFraction;
        int rc = s->forward(s->ctx, cutBack ? 1 : 0, guess ? 1 : 0, Delta_t, Delta_t_prev, t_remaining,
                            &lc.deformation, &lc.stress, lc.q_rot);
        if (rc) return rc;
        if (!cutBack && (rc = s->materialpoint_forward(s->ctx))) return rc;
        dmk_solution_state sol{};
        if ((rc = s->solution(s->ctx, &sol))) return rc;
        if (sol.converged && sol.stagConverged) {
          if ((rc = s->update_coords(s->ctx))) return rc;
          Delta_t_prev = Delta_t;
          cutBack = false;
          guess = true;
          if (cb) {
            dmk_increment_info info{total, t, cutBackLevel, 1, sol.iterationsNeeded, sol.residualEvals, l, inc};
            for (int k = 0; k < 9; ++k) info.P_av[k] = sol.P_av[k];
            if (cb(&info, user)) return 0;
          }
        } else if (cutBackLevel < N_cutback_max) {
          cutBack = true;
          stepFraction = (stepFraction - 1) * ssf;
          ++cutBackLevel;
          t = t - Delta_t;
          Delta_t = Delta_t / double(ssf);
        } else {
          return dmk::record_error(DMK_ERR_NOT_CONVERGED, "increment " + std::to_string(total) +
                                                              " did not converge (IO_error 950)");
        }
      }
      cutBackLevel = cutBackLevel > 0 ? cutBackLevel - 1 : 0;
    }
  }
  return 0;
}

int dmk_grid_run_ctx(dmk_ctx* ctx, const dmk_loadstep* steps, int n_steps, int N_cutback_max, int restart_inc,
                     int max_increments, dmk_increment_cb cb, void* user) {
  if (!ctx) return dmk::record_error(DMK_ERR_ARG, "null argument");
  const dmk_grid_solver s{ctx, ctx_forward, ctx_solution, ctx_update_coords, ctx_materialpoint_forward};
  return dmk_grid_run(&s, steps, n_steps, N_cutback_max, restart_inc, max_increments, cb, user);
}

}  // extern "C"
