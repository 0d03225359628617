// The increment loop of the grid driver (src/grid/DAMASK_grid.f90:288-460) for the mechanical
// field, behind the C-ABI: time stepping with geometric fractions, the global cutback (time step
// halved up to N_cutback_max times, then IO_error 950), the guess flag, restart skipping, and the
// calls of the five plugin procedures.  The plugin is a table of function pointers, so the same loop
// drives the CUDA context (dmk_grid_run_ctx) and any other implementation of the procedures.
#include <cmath>
#include <string>

#include "../../include/damask_b200.h"

namespace dmk {
int record_error(int code, const std::string& msg);
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

}  // namespace

extern "C" {

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
