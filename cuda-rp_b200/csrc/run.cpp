// crp_run: the main loop of solve_bubbles with its saves (src/bubble_CUDA.cu:203-438:
// step while (n_step_max && step < n_step_max) || (t_step_max && t < t_step_max),
// rawdata every save interval), as one call of the C ABI.
#include "crp.h"

extern "C" crp_status crp_run(crp_sim* sim, const crp_output_plan* plan, const crp_config* cfg) {
  if (!sim || !plan) return CRP_ERR_INVALID;
  int64_t n_max = plan->n_steps;
  double t_max = plan->t_max;
  if (n_max == 0 && t_max == 0.0 && cfg) {
    n_max = cfg->sim_n_step_max;
    t_max = cfg->sim_t_step_max;
  }
  if (n_max < 0 || t_max < 0.0 || plan->save_interval < 0) return CRP_ERR_INVALID;
  crp_stats st;
  crp_status s = crp_get_stats(sim, &st);
  if (s != CRP_OK) return s;
  while ((n_max != 0 && st.steps < n_max) || (t_max != 0.0 && st.time < t_max)) {
    s = crp_step(sim, 1);
    if (s != CRP_OK) return s;
    crp_get_stats(sim, &st);
    if (plan->save_interval > 0 && st.steps % plan->save_interval == 0) {
      if (plan->dir) {
        s = plan->sph ? crp_write_sph(sim, plan->dir) : crp_write_rawdata(sim, plan->dir);
        if (s != CRP_OK) return s;
      }
      if (plan->progress) plan->progress(st.steps, st.time, plan->user);
    }
  }
  return CRP_OK;
}
