// Host-side set-up shared by the CUDA library and the `bubbles` program:
// derived scalars, PML profiles, cylindrical metrics and the bubble population.
#pragma once
#include <string>
#include <vector>

#include "crp.h"

namespace crp {

// Scalars derived once from the configuration (init_grid_size, init_transducer,
// init_mix, mix_set_time_increment, init_bub_params: src/bubble_CUDA.cu:487-518).
struct Derived {
  double elem_rap = 0.0;  // aperture radius of the source elements (ext.elements > 0), element_aperture()
  double dx, dy, rdx, rdy;
  double dt;
  double rho_inf, c_inf, P_inf, T_inf;
  double omega;
  double fpx, fpy;      // transducer focal point (seeding box centre)
  double ctl_x, ctl_y;  // focus handed to the source kernels
  double focal_dist;
  double bub_dt0;
  double pi, pi4r3;
  double dcx, dcy, dcz;  // smooth-delta coefficients
};

struct HostSetup {
  Derived d{};
  // mx, my, nx, ny, xu, rxp and the PML update factors concatenated; offsets
  // in elements.
  std::vector<double> sigma_block;
  size_t off_mx = 0, off_my = 0, off_nx = 0, off_ny = 0, off_xu = 0, off_rxp = 0;
  size_t off_vax = 0, off_vbx = 0, off_vay = 0, off_vby = 0, off_pax = 0, off_pbx = 0, off_pay = 0, off_pby = 0;
  int nb = 0;
  std::vector<double> bx, by, r0, nb_w;
};

// Largest distance from the focus axis, |x - ctl_x|, among the cells that
// carry the pressure source (row ext.source_row, or the y = 0 ghost row when
// it is 0; a focused source only within focal_dist of the focus): the radius
// that ext.elements splits into equal bands.  0 without such cells.
double element_aperture(const crp_config& c, double dx, double dy, double ctl_x, double ctl_y, double focal_dist);

// Validate the configuration and compute everything crp_create uploads.
crp_status host_setup(const crp_config& cfg, const crp_bubbles_in* bubbles, HostSetup* out, std::string* err);

// Rawdata writer (rawdata.cpp) and the accessors it uses (sim.cu).
crp_status write_rawdata(crp_sim* sim, const char* dir);
crp_status write_sph(crp_sim* sim, const char* dir);
crp_status sim_read_field(crp_sim* h, crp_field f, double* host);
crp_status sim_read_bubbles(crp_sim* h, crp_bubble_field w, double* host);
const crp_config& sim_config(const crp_sim* h);
int64_t sim_step_count(const crp_sim* h);
double sim_time(const crp_sim* h);

// Running min/max of the values written to rawdata files (the globals of
// src/bubbles.cpp:11-13 that save_ascii updates), per simulation.
struct MinMax {
  double fg_min = 1e10, fg_max = -1e10, p0_min = 1e10, p0_max = -1e10, T_min = 1e10, T_max = -1e10;
};
MinMax& sim_minmax(crp_sim* h);

// Graph-queued steps for crp_batch (sim.cu): whether the next step of a 2-D
// simulation may run as a graph, the batch's override of ext.graphs, and the
// two halves of a run of graph steps (queue on the simulation's stream; wait
// and take the device's step state).
bool sim_graph_ready(const crp_sim* h);
void sim_allow_graphs(crp_sim* h, bool on);
// Host waits inside a 2-D step: spin (default) or block on an event.
crp_status sim_blocking_waits(crp_sim* h, bool on);
crp_status sim_graphs_enqueue(crp_sim* h, int n);
crp_status sim_graphs_finish(crp_sim* h);

}  // namespace crp
