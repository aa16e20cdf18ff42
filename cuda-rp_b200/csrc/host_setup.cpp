// Host set-up: validation, derived scalars, PML profiles (init_sigma), cylindrical
// metrics (init_grid_vector) and the bubble population (init_bub_array /
// bubble_input, or an explicit or seeded [ext] population).
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "crp_host.h"

namespace crp {

namespace {

crp_status bad(std::string* err, const std::string& msg) {
  if (err) *err = msg;
  return CRP_ERR_INVALID;
}

// init_sigma, src/bubble_CUDA.cu:946-1205, for order 2 (ms=0, me=1, ns=-1, ne=0):
// mid-point profiles sigma_max((n-1/2)/N)^order on cells 1..X, node profiles
// sigma_max(n/N)^order on faces 0..X, for each face that has a PML.
void pml_profiles(const crp_config& c, const Derived& d, std::vector<double>& mx, std::vector<double>& my,
                  std::vector<double>& nx, std::vector<double>& ny) {
  const int X = c.grid_x, Y = c.grid_y, N = c.pml_grid_number;
  const double order = c.pml_order;
  const int ms = 0, me = 1, ns = -1, ne = 0;
  mx.assign(X + 2, 0.0);  // i in [0, X+1]
  my.assign(Y + 2, 0.0);
  nx.assign(X + 3, 0.0);  // i in [-1, X+1], stored at i+1
  ny.assign(Y + 3, 0.0);
  auto smax = [&](double h) { return -std::log(c.pml_sigma) * 0.5 * ((double)order + 1.0) / (h * (double)N); };
  if (c.pml_x0 && 1 <= N) {
    double s = smax(d.dx);
    for (int i = std::max(1, ms); i <= std::min(X, N); i++)
      mx[i] = s * std::pow(((double)(N - i + 1) - 0.5) / ((double)N), order);
  }
  if (c.pml_x1 && X - N + 1 <= X) {
    double s = smax(d.dx);
    for (int i = std::max(1, X - N + 1); i <= std::min(X, X + me); i++)
      mx[i] = s * std::pow(((double)(i - X + N) - 0.5) / ((double)N), order);
  }
  if (c.pml_y0 && 1 <= N) {
    double s = smax(d.dy);
    for (int j = std::max(1, ms); j <= std::min(Y, N); j++)
      my[j] = s * std::pow(((double)(N - j + 1) - 0.5) / ((double)N), order);
  }
  if (c.pml_y1 && Y - N + 1 <= Y) {
    double s = smax(d.dy);
    for (int j = std::max(1, Y - N + 1); j <= std::min(Y, Y + me); j++)
      my[j] = s * std::pow(((double)(j - Y + N) - 0.5) / ((double)N), order);
  }
  if (c.pml_x0 && 0 <= N - 1) {
    double s = smax(d.dx);
    for (int i = std::max(0, ms + ns); i <= std::min(X, N - 1); i++)
      nx[i + 1] = s * std::pow(((double)(N - i)) / ((double)N), order);
  }
  if (c.pml_x1 && X - N + 1 <= X) {
    double s = smax(d.dx);
    for (int i = std::max(0, X - N + 1); i <= std::min(X, X + me + ne + 1); i++)
      nx[i + 1] = s * std::pow(((double)(i - X + N)) / ((double)N), order);
  }
  if (c.pml_y0 && 0 <= N - 1) {
    double s = smax(d.dy);
    for (int j = std::max(0, ms + ns); j <= std::min(Y, N - 1); j++)
      ny[j + 1] = s * std::pow(((double)(N - j)) / ((double)N), order);
  }
  if (c.pml_y1 && Y - N + 1 <= Y) {
    double s = smax(d.dy);
    for (int j = std::max(0, Y - N + 1); j <= std::min(Y, Y + me + ne + 1); j++)
      ny[j + 1] = s * std::pow(((double)(j - Y + N)) / ((double)N), order);
  }
}

}  // namespace

double element_aperture(const crp_config& c, double dx, double dy, double ctl_x, double ctl_y, double focal_dist) {
  const double ym = c.ext_source_row > 0 ? ((double)c.ext_source_row - 0.5) * dy : -0.5 * dy;
  double r = 0.0;
  for (int i = 1; i <= c.grid_x; i++) {
    const double xm = ((double)i - 0.5) * dx;
    if (c.tr_focused_p) {
      const double s1 = std::sqrt((ctl_x - xm) * (ctl_x - xm) + (ctl_y - ym) * (ctl_y - ym));
      if (!(s1 <= focal_dist)) continue;
    }
    r = std::max(r, std::fabs(xm - ctl_x));
  }
  return r;
}

crp_status host_setup(const crp_config& c, const crp_bubbles_in* bin, HostSetup* out, std::string* err) {
  HostSetup& h = *out;
  if (c.grid_x < 2 || c.grid_y < 2) return bad(err, "grid.x and grid.y must be at least 2");
  if (!(c.grid_lx > 0) || !(c.grid_ly > 0)) return bad(err, "grid.lx and grid.ly must be positive");
  if (!(c.sim_cfl > 0)) return bad(err, "simulation.cfl must be positive");
  if (!(c.ext_c_inf > 0) || !(c.ext_rho_inf > 0) || !(c.ext_p_inf > 0))
    return bad(err, "ext.rho_inf, ext.c_inf and ext.p_inf must be positive");
  const bool any_pml = c.pml_x0 || c.pml_x1 || c.pml_y0 || c.pml_y1;
  if (any_pml && (c.pml_grid_number < 1 || !(c.pml_sigma > 0) || !(c.pml_sigma < 1)))
    return bad(err, "pml.grid_number must be >= 1 and 0 < pml.sigma < 1");
  const bool any_src = c.tr_plane_p || c.tr_plane_v || c.tr_focused_p || c.tr_focused_v;
  if (any_src && (!(c.tr_freq > 0) || c.tr_on_wave + c.tr_off_wave <= 0))
    return bad(err, "a source needs transducer.freq > 0 and on_wave + off_wave > 0");
  if (c.ext_source_row < 0 || c.ext_source_row > c.grid_y) return bad(err, "ext.source_row out of range");
  if (c.ext_picard_cap < 0 || c.ext_rp_step_cap <= 0) return bad(err, "ext.picard_cap/ext.rp_step_cap out of range");
  if (c.ext_elements < 0 || c.ext_elements > 65536) return bad(err, "ext.elements out of range (0..65536)");
  if (c.ext_elements > 0 && (!(c.tr_plane_p || c.tr_focused_p) || c.tr_plane_v || c.tr_focused_v))
    return bad(err, "ext.elements needs a pressure source and no velocity source");
  if (c.ext_elements > 0 && c.tr_pid) return bad(err, "ext.elements with transducer.pid is not supported");
  Derived& d = h.d;
  d.dx = (double)c.grid_lx / (double)c.grid_x;
  d.dy = (double)c.grid_ly / (double)c.grid_y;
  d.rdx = (double)1.0 / (double)d.dx;
  d.rdy = (double)1.0 / (double)d.dy;
  d.fpx = 0.0;
  d.fpy = c.tr_focal_dist ? c.tr_focal_dist * 0.5 * std::sqrt(3.0) : c.grid_ly * 0.5;
  d.omega = 2.0 * std::acos(-1.0) * c.tr_freq;
  d.T_inf = 293.15;
  d.P_inf = c.ext_p_inf;
  d.rho_inf = c.ext_rho_inf;
  d.c_inf = c.ext_c_inf;
  d.dt = c.sim_cfl * std::min(d.dx, d.dy) / d.c_inf;
  d.ctl_x = d.fpx;
  d.ctl_y = d.fpy;
  if (c.tr_pid && c.tr_init_control) d.ctl_x = 0.0, d.ctl_y = c.tr_init_control;
  d.focal_dist = d.ctl_y / 0.5 / std::sqrt(3.0);
  d.elem_rap = c.ext_elements > 0 ? element_aperture(c, d.dx, d.dy, d.ctl_x, d.ctl_y, d.focal_dist) : 0.0;
  if (c.ext_elements > 0 && !(d.elem_rap > 0.0)) return bad(err, "ext.elements: the source has no cells");
  d.bub_dt0 = 0.1 * d.dt;
  d.pi = std::acos(-1.0);
  d.pi4r3 = d.pi * 4.0 / 3.0;
  d.dcx = 1.0 / ((double)c.sim_smooth_delta_band);
  d.dcy = 2.0 * std::acos(-1.0) / ((double)c.sim_smooth_delta_band) * d.rdx;
  d.dcz = 2.0 * std::acos(-1.0) / ((double)c.sim_smooth_delta_band) * d.rdy;

  std::vector<double> mx, my, nx, ny;
  pml_profiles(c, d, mx, my, nx, ny);
  std::vector<double> xu(c.grid_x + 3), rxp(c.grid_x + 2);
  for (int i = -1; i <= c.grid_x + 1; i++) xu[i + 1] = ((double)i) * d.dx;
  for (int i = 0; i <= c.grid_x + 1; i++) rxp[i] = 1.0 / (d.dx * ((double)i - 0.5));
  h.sigma_block.clear();
  auto put = [&](const std::vector<double>& v, size_t* off) {
    *off = h.sigma_block.size();
    h.sigma_block.insert(h.sigma_block.end(), v.begin(), v.end());
  };
  put(mx, &h.off_mx);
  put(my, &h.off_my);
  put(nx, &h.off_nx);
  put(ny, &h.off_ny);
  put(xu, &h.off_xu);
  put(rxp, &h.off_rxp);
  // PML factors (1 - s) and 1 / (1 + s) of every velocity face (s3 = dt c
  // sigma / 2 of VelocityKernel, inc/bubble_CUDA_kernel.cuh:664-665, 674-675) and
  // of every pressure component (s2 of MixturePressureKernel, :853), so that
  // the grid kernels multiply where the reference divides.  Both are exactly 1
  // outside the PML.
  auto factors = [&](const std::vector<double>& sigma, double per_sigma, size_t* off_a, size_t* off_b) {
    std::vector<double> fa(sigma.size()), fb(sigma.size());
    for (size_t k = 0; k < sigma.size(); k++) {
      const double sk = per_sigma * sigma[k];
      fa[k] = 1.0 - sk;
      fb[k] = 1.0 / (1.0 + sk);
    }
    put(fa, off_a);
    put(fb, off_b);
  };
  const double v_per_sigma = (d.c_inf + d.c_inf) * 0.5 * 0.5 * d.dt;
  const double p_per_sigma = 0.5 * d.dt * d.c_inf;
  factors(nx, v_per_sigma, &h.off_vax, &h.off_vbx);
  factors(ny, v_per_sigma, &h.off_vay, &h.off_vby);
  factors(mx, p_per_sigma, &h.off_pax, &h.off_pbx);
  factors(my, p_per_sigma, &h.off_pay, &h.off_pby);

  h.bx.clear();
  h.by.clear();
  h.r0.clear();
  h.nb_w.clear();
  if (c.bub_enable) {
    if (!(c.bub_gamma > 1) || !(c.bub_T0 > 0) || !(c.bub_K0 > 0) || !(c.bub_rho > 0))
      return bad(err, "bubbles: gamma > 1, T0 > 0, K0 > 0 and liquid_density > 0 are required");
    if (bin && bin->n > 0) {
      for (int k = 0; k < bin->n; k++) {
        if (!(bin->r0[k] > 0)) return bad(err, "explicit bubble with R0 <= 0");
        h.bx.push_back(bin->x[k]);
        h.by.push_back(bin->y[k]);
        h.r0.push_back(bin->r0[k]);
        h.nb_w.push_back(bin->n_b[k]);
      }
    } else if (c.ext_bubble_count > 0) {
      int n = c.ext_bubble_count;
      h.bx.resize(n);
      h.by.resize(n);
      h.r0.resize(n);
      h.nb_w.resize(n);
      crp_status st = crp_seed_bubbles(&c, h.bx.data(), h.by.data(), h.r0.data(), h.nb_w.data());
      if (st != CRP_OK) return bad(err, "bubble seeding failed");
    } else {
      if (!(c.bub_R0 > 0)) return bad(err, "bubbles.R0 must be positive");
      // init_bub_array (src/bubble_CUDA.cu:811-839): one bubble per cell centre
      // inside the box around the focal point; weight of bubble_input (:922-931).
      const double pi = std::acos(-1.0);
      for (int i = 1; i <= c.grid_x; i++) {
        double x = ((double)i - 0.5) * d.dx;
        for (int j = 1; j <= c.grid_y; j++) {
          double y = ((double)j - 0.5) * d.dy;
          bool take = c.tr_box_size ? (std::fabs(x - d.fpx) < 0.5 * c.tr_box_size &&
                                       std::fabs(y - d.fpy) < 0.5 * c.tr_box_size)
                                    : true;
          if (!take) continue;
          double R0 = c.bub_R0;
          double w = c.tr_cylindrical ? c.bub_fg0 * (x * d.dx * d.dy) / (4.0 / 3.0 * pi * std::pow(R0, 3))
                                      : c.bub_fg0 * (d.dx * d.dy) / (4.0 / 3.0 * pi * std::pow(R0, 3));
          h.bx.push_back(x);
          h.by.push_back(y);
          h.r0.push_back(R0);
          h.nb_w.push_back(w);
        }
      }
    }
  }
  h.nb = (int)h.bx.size();
  return CRP_OK;
}

}  // namespace crp
