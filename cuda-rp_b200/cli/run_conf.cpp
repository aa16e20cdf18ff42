// One configuration file through the crp C ABI, as `bubbles <conf>` runs it
// (src/bubbles.cpp:190-310).  One difference, outside the simulated path: the
// output directory is created if missing and never cleared (the reference runs
// `rm -rf` on it, src/output_styles.cpp:20).
#include "run_conf.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <filesystem>
#include <fstream>
#include <string>
#include <vector>

#include "crp.h"

namespace {

// Optional overrides of the *_minmax.txt values (src/bubbles.cpp:275-294).  The
// reference registers the p_min key as "debug p_min" (a typo), so only
// debug.fg_min, debug.fg_max and debug.p_max can take effect.
bool lookup_key(const std::string& path, const std::string& full, double* out) {
  std::ifstream in(path);
  std::string line, section;
  while (std::getline(in, line)) {
    size_t h = line.find('#');
    if (h != std::string::npos) line = line.substr(0, h);
    size_t a = line.find_first_not_of(" \t\r"), b = line.find_last_not_of(" \t\r");
    if (a == std::string::npos) continue;
    line = line.substr(a, b - a + 1);
    if (line[0] == '[' && line.back() == ']') {
      section = line.substr(1, line.size() - 2);
      continue;
    }
    size_t eq = line.find('=');
    if (eq == std::string::npos) continue;
    std::string k = line.substr(0, eq), v = line.substr(eq + 1);
    k = k.substr(0, k.find_last_not_of(" \t") + 1);
    v = v.substr(v.find_first_not_of(" \t") == std::string::npos ? v.size() : v.find_first_not_of(" \t"));
    if ((section.empty() ? k : section + "." + k) == full) {
      *out = std::strtod(v.c_str(), nullptr);
      return true;
    }
  }
  return false;
}

void write_minmax(const std::string& path, double lo, double hi) {
  std::ofstream f(path.c_str());
  f << lo << std::endl << hi << std::endl;
}

}  // namespace

int run_configuration(const ConfRun& run, std::ostream& out, std::ostream& err) {
  const time_t start_time = time(nullptr);
  std::string target_dir = run.target_dir;
  if (target_dir.empty() || target_dir.back() != '/') target_dir += "/";
  crp_config cfg;
  crp_config_defaults(&cfg);
  char msg[512] = {0};
  crp_status st = crp_config_parse_file(run.in_file.c_str(), &cfg, msg, sizeof(msg));
  if (st != CRP_OK) {
    err << "error: " << (msg[0] ? msg : crp_status_string(st)) << std::endl;
    return 1;
  }
  const bool ascii = run.ascii || cfg.opt_ascii;
  const bool sph = run.sph || cfg.opt_sph;
  if (run.banner) {
    out << "Input file is " << run.in_file << std::endl;
    out << "Saving results to " << target_dir << std::endl;
    out << "Save format is " << (sph && !ascii ? "sph" : "ASCII plaintext");
    out << std::endl << std::endl;
  }
  // transducer.pid_iterate passes (src/bubbles.cpp:218-306): with -d each pass
  // writes to <dir>_I/, <dir>_II/, ...; the focus control state and the
  // running min/max carry over from pass to pass.
  const int num_iters = cfg.tr_pid_iterate > 0 ? cfg.tr_pid_iterate : 1;
  std::string base_dir = target_dir;
  if (!base_dir.empty() && base_dir.back() == '/') base_dir.pop_back();
  double fg_min = 1e10, fg_max = -1e10, p0_min = 1e10, p0_max = -1e10, T_min = 1e10, T_max = -1e10;
  crp_focus_state carry{};
  for (int pass = 0; pass < num_iters; pass++) {
    if (num_iters > 1 && run.dir_given) target_dir = base_dir + "_" + std::string(pass + 1, 'I') + "/";
    std::error_code ec;
    std::filesystem::create_directories(target_dir, ec);
    if (ec) {
      err << "error: cannot create " << target_dir << ": " << ec.message() << std::endl;
      return 1;
    }
    crp_sim* sim = nullptr;
    st = crp_create(&cfg, nullptr, nullptr, &sim);
    if (st != CRP_OK) {
      err << "error: " << crp_status_string(st) << std::endl;
      return 1;
    }
    if (pass > 0) crp_set_focus_state(sim, &carry);
    crp_output_plan plan{};
    plan.save_interval = cfg.sim_save_interval > 0 ? cfg.sim_save_interval : 0;
    // As solve_bubbles: SPH when -s is given, else text rawdata when -a is
    // (src/bubble_CUDA.cu:398-411).
    plan.dir = (sph || ascii) ? target_dir.c_str() : nullptr;
    plan.sph = sph ? 1 : 0;
    plan.user = &cfg;
    if (run.progress) {
      // Progress line as the reference prints it at each save (src/bubbles.cpp:258-268).
      plan.progress = [](int64_t step, double time, void* user) {
        const crp_config* c = (const crp_config*)user;
        if (c->sim_n_step_max != 0)
          printf("\rRunning the simulation...\t\tnstep : %5lld / %i\t", (long long)step, c->sim_n_step_max);
        else
          printf("\rRunning the simulation...\t\ttstep : %4.2E / %4.2E\t", time, c->sim_t_step_max);
        fflush(stdout);
      };
    }
    st = crp_run(sim, &plan, &cfg);
    if (st != CRP_OK) {
      crp_stats stats;
      crp_get_stats(sim, &stats);
      err << "\nerror at step " << stats.steps + 1 << ": " << crp_status_string(st) << ": " << crp_last_error(sim)
          << std::endl;
      crp_destroy(sim);
      return 1;
    }
    if (run.progress) {
      printf("\rRunning the simulation...\t\tdone\n\n");
      fflush(stdout);
    }

    // focalpoint_actual_T.txt and focalpoint_controller_T.txt (src/bubbles.cpp:258-270),
    // written when the tracker ran (debug.T or transducer.pid).
    const int64_t nf = crp_focus_history(sim, 0, nullptr, 0), nc = crp_focus_history(sim, 1, nullptr, 0);
    if (nf > 0) {
      std::vector<double> f((size_t)nf), c((size_t)nc);
      crp_focus_history(sim, 0, f.data(), nf);
      crp_focus_history(sim, 1, c.data(), nc);
      std::ofstream fa((target_dir + "focalpoint_actual_T.txt").c_str());
      for (int64_t k = 0; k < nf; k++) fa << k << "\t" << f[(size_t)k] << std::endl;
      std::ofstream fc((target_dir + "focalpoint_controller_T.txt").c_str());
      for (int64_t k = 0; k < nc; k++) fc << k + cfg.tr_pid_start_step << "\t" << c[(size_t)k] << std::endl;
    }
    crp_get_focus_state(sim, &carry);

    // *_minmax.txt (src/bubbles.cpp:273-296), running over the passes.
    double a0, a1, b0, b1;
    crp_minmax(sim, &a0, &a1, &b0, &b1);
    fg_min = std::min(fg_min, a0), fg_max = std::max(fg_max, a1), p0_min = std::min(p0_min, b0),
    p0_max = std::max(p0_max, b1);
    crp_minmax_T(sim, &a0, &a1);
    T_min = std::min(T_min, a0), T_max = std::max(T_max, a1);
    double v;
    if (cfg.dbg_T) {
      if (lookup_key(run.in_file, "debug.T_min", &v)) T_min = v;
      if (lookup_key(run.in_file, "debug.T_max", &v)) T_max = v;
      write_minmax(target_dir + "T_minmax.txt", T_min, T_max);
    }
    if (cfg.dbg_p) {
      if (lookup_key(run.in_file, "debug.p_max", &v)) p0_max = v;
      write_minmax(target_dir + "p0_minmax.txt", p0_min, p0_max);
    }
    if (cfg.dbg_fg) {
      if (lookup_key(run.in_file, "debug.fg_min", &v)) fg_min = v;
      if (lookup_key(run.in_file, "debug.fg_max", &v)) fg_max = v;
      write_minmax(target_dir + "fg_minmax.txt", fg_min, fg_max);
    }
    crp_destroy(sim);
    if (num_iters == 1)
      out << "The program took ";
    else
      out << pass << " pass took ";
    out << time(nullptr) - start_time << " seconds to run" << std::endl;
    std::ofstream runtime((target_dir + "runtime.txt").c_str());
    runtime << "Finished in " << time(nullptr) - start_time << " seconds" << std::endl;
  }
  return 0;
}
