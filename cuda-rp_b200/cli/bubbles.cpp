// `bubbles <conf>`: the reference program's command line (src/bubbles.cpp:18-310)
// on top of the crp C ABI.
//
//   bubbles [-h|--help] [--help-all] [-a|--ascii] [-s|--sph] [-d|--directory DIR] <input-file>
//
// Same options, configuration keys, defaults, output directory (./rawdata/),
// rawdata files (text or SPH, fg/p0/T/vx/vy), focal-point tracker files,
// transducer.pid_iterate passes and *_minmax.txt / runtime.txt; the run itself
// is run_configuration (run_conf.cpp).
#include <iostream>
#include <string>

#include "run_conf.h"

namespace {

const char* kHelp =
    "Options:\n\n"
    "Command line options:\n"
    "  -h [ --help ]                         Output this help message.\n"
    "  --help-all                            Output a complete list of options.\n\n"
    "Generic options:\n"
    "  -a [ --ascii ]                        Save plaintext files.\n"
    "  -s [ --sph ]                          Save sph files. This option has\n"
    "                                        precedence over --ascii.\n"
    "  -d [ --directory ] arg (=./rawdata/)  Save into a target directory.\n";

const char* kFileKeys =
    "\nConfiguration file options:\n"
    "  grid.x grid.y grid.lx grid.ly\n"
    "  pml.x0 pml.x1 pml.y0 pml.y1 pml.grid_number pml.sigma pml.order\n"
    "  simulation.cfl simulation.dt0 simulation.n_step_max simulation.t_step_max\n"
    "  simulation.save_interval simulation.order simulation.smooth_delta_band\n"
    "  transducer.amp transducer.freq transducer.focal_dist transducer.pid\n"
    "  transducer.pid_start_step transducer.init_control transducer.pid_iterate\n"
    "  transducer.box_size transducer.cylindrical transducer.on_wave transducer.off_wave\n"
    "  transducer.transducer_v transducer.transducer_p transducer.focused_wave_v\n"
    "  transducer.focused_wave_p\n"
    "  bubbles.enable bubbles.fg0 bubbles.R0 bubbles.P0 bubbles.T0 bubbles.gamma\n"
    "  bubbles.liquid_surface_tension bubbles.liquid_viscosity bubbles.liquid_density bubbles.K0\n"
    "  debug.display_dim debug.fg debug.fg_min debug.fg_max debug.T debug.T_min debug.T_max\n"
    "  debug.p debug.p_max debug.v debug.v_min debug.v_max debug.bubbles\n"
    "  ext.rho_inf ext.c_inf ext.p_inf ext.source_row ext.ramp_cycles ext.precision\n"
    "  ext.picard_cap ext.rp_step_cap ext.bubble_count ext.bubble_seed ext.r0_sigma_ln\n"
    "  ext.cloud_shape ext.cloud_r ext.cloud_h ext.n_b ext.picard_tol\n";

}  // namespace

int main(int argc, char** argv) {
  std::string in_file, target_dir = "./rawdata/";
  bool ascii = false, sph = false, dir_given = false;
  for (int k = 1; k < argc; k++) {
    std::string a = argv[k];
    if (a == "-h" || a == "--help") {
      std::cout << kHelp << std::endl;
      return 0;
    }
    if (a == "--help-all") {
      std::cout << kHelp << kFileKeys << std::endl;
      return 0;
    }
    if (a == "-a" || a == "--ascii") {
      ascii = true;
    } else if (a == "-s" || a == "--sph") {
      sph = true;
    } else if (a == "-d" || a == "--directory") {
      if (k + 1 >= argc) {
        std::cerr << "the required argument for option '--directory' is missing" << std::endl;
        return 1;
      }
      target_dir = argv[++k];
      dir_given = true;
    } else if (a.rfind("--directory=", 0) == 0) {
      target_dir = a.substr(12);
      dir_given = true;
    } else if (!a.empty() && a[0] == '-') {
      // unregistered options are ignored (allow_unregistered)
    } else if (in_file.empty()) {
      in_file = a;
    }
  }
  if (in_file.empty()) {
    std::cout << "Please specify an input configuration file" << std::endl;
    return 1;
  }
  ConfRun run;
  run.in_file = in_file;
  run.target_dir = target_dir;
  run.ascii = ascii;
  run.sph = sph;
  run.dir_given = dir_given;
  return run_configuration(run, std::cout, std::cerr);
}
