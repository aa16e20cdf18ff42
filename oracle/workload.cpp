// Workload inputs for the CPU oracle — TEST INFRASTRUCTURE ONLY.
//
// The oracle's own configuration defaults, configuration-file parser and
// seeded bubble population, so that a run of the oracle (the bench's
// reference arm, the CPU baseline) needs nothing from the product library.
//
// * Defaults: the values registered with Boost program_options in
//   src/bubbles.cpp:97-132, zero where the reference registers none (it
//   malloc's the structs, src/bubbles.cpp:51-56), and the constants the
//   reference hard-codes (rho 1000, c 1500, P_inf 1e5: inc/bubble_CUDA_kernel.cuh:153-169,
//   src/bubble_CUDA.cu:636-646) for the [ext] keys that replace them.
// * Parser: Boost program_options' config-file grammar as the reference uses it
//   (src/bubbles.cpp:188-195): `#` comments, `[section]` prefixes giving
//   `section.key`, `key = value`, unregistered keys ignored
//   (allow_unregistered = true), a key given twice is an error, bool values
//   1/0/true/false/yes/no/on/off.
// * Seeding: the [ext] bubble cloud (cylinder, ball or Gaussian around the
//   focus of init_transducer, src/bubble_CUDA.cu:546-555; R0 lognormal) drawn
//   from Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers:
//   as easy as 1, 2, 3", SC'11): two blocks per bubble k, counter k, stream
//   words 0 and 1, key = the 64-bit seed.
//
// tests/test_oracle_workload.py checks all three against the product's
// crp_config_parse_file / crp_seed_bubbles bit for bit.
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <set>
#include <sstream>
#include <string>

#include "crp_oracle.h"

namespace {

enum class T { I32, F64, Bool, U64, Prec, Shape, Scheme };

struct Slot {
  T type;
  size_t off;
};

const std::map<std::string, Slot>& registry() {
#define S(key, type, member) {key, Slot{type, offsetof(crp_config, member)}}
  static const std::map<std::string, Slot> m = {
      S("grid.x", T::I32, grid_x), S("grid.y", T::I32, grid_y), S("grid.lx", T::F64, grid_lx),
      S("grid.ly", T::F64, grid_ly), S("pml.x0", T::Bool, pml_x0), S("pml.x1", T::Bool, pml_x1),
      S("pml.y0", T::Bool, pml_y0), S("pml.y1", T::Bool, pml_y1), S("pml.grid_number", T::I32, pml_grid_number),
      S("pml.sigma", T::F64, pml_sigma), S("pml.order", T::I32, pml_order), S("simulation.cfl", T::F64, sim_cfl),
      S("simulation.dt0", T::F64, sim_dt0), S("simulation.n_step_max", T::I32, sim_n_step_max),
      S("simulation.t_step_max", T::F64, sim_t_step_max),
      S("simulation.save_interval", T::I32, sim_save_interval), S("simulation.order", T::I32, sim_order),
      S("simulation.smooth_delta_band", T::I32, sim_smooth_delta_band), S("transducer.amp", T::F64, tr_amp),
      S("transducer.freq", T::F64, tr_freq), S("transducer.focal_dist", T::F64, tr_focal_dist),
      S("transducer.pid", T::Bool, tr_pid), S("transducer.pid_start_step", T::I32, tr_pid_start_step),
      S("transducer.init_control", T::F64, tr_init_control),
      S("transducer.pid_iterate", T::I32, tr_pid_iterate), S("transducer.box_size", T::F64, tr_box_size),
      S("transducer.cylindrical", T::Bool, tr_cylindrical), S("transducer.on_wave", T::I32, tr_on_wave),
      S("transducer.off_wave", T::I32, tr_off_wave), S("transducer.transducer_v", T::Bool, tr_plane_v),
      S("transducer.transducer_p", T::Bool, tr_plane_p),
      S("transducer.focused_wave_v", T::Bool, tr_focused_v),
      S("transducer.focused_wave_p", T::Bool, tr_focused_p), S("bubbles.enable", T::Bool, bub_enable),
      S("bubbles.fg0", T::F64, bub_fg0), S("bubbles.R0", T::F64, bub_R0), S("bubbles.P0", T::F64, bub_P0),
      S("bubbles.T0", T::F64, bub_T0), S("bubbles.gamma", T::F64, bub_gamma),
      S("bubbles.liquid_surface_tension", T::F64, bub_sigma),
      S("bubbles.liquid_viscosity", T::F64, bub_mu), S("bubbles.liquid_density", T::F64, bub_rho),
      S("bubbles.K0", T::F64, bub_K0), S("debug.display_dim", T::I32, dbg_display),
      S("debug.fg", T::Bool, dbg_fg), S("debug.T", T::Bool, dbg_T), S("debug.p", T::Bool, dbg_p),
      S("debug.v", T::Bool, dbg_v), S("debug.bubbles", T::Bool, dbg_bubbles), S("ascii", T::Bool, opt_ascii),
      S("sph", T::Bool, opt_sph), S("ext.rho_inf", T::F64, ext_rho_inf), S("ext.c_inf", T::F64, ext_c_inf),
      S("ext.p_inf", T::F64, ext_p_inf), S("ext.source_row", T::I32, ext_source_row),
      S("ext.ramp_cycles", T::F64, ext_ramp_cycles), S("ext.precision", T::Prec, ext_precision),
      S("ext.picard_cap", T::I32, ext_picard_cap), S("ext.rp_step_cap", T::I32, ext_rp_step_cap),
      S("ext.bubble_count", T::I32, ext_bubble_count), S("ext.bubble_seed", T::U64, ext_bubble_seed),
      S("ext.r0_sigma_ln", T::F64, ext_r0_sigma_ln), S("ext.cloud_shape", T::Shape, ext_cloud_shape),
      S("ext.cloud_r", T::F64, ext_cloud_r), S("ext.cloud_h", T::F64, ext_cloud_h),
      S("ext.n_b", T::F64, ext_n_b), S("ext.picard_tol", T::F64, ext_picard_tol),
      S("ext.graphs", T::Bool, ext_graphs), S("ext.elements", T::I32, ext_elements),
      S("ext.rp_scheme", T::Scheme, ext_rp_scheme), S("ext.rp_tol", T::F64, ext_rp_tol),
      S("ext.grid_z", T::I32, ext_grid_z), S("ext.grid_lz", T::F64, ext_grid_lz),
      S("ext.pml_z0", T::Bool, ext_pml_z0), S("ext.pml_z1", T::Bool, ext_pml_z1),
      S("ext.array_elements", T::I32, ext_array_elements), S("ext.array_radius", T::F64, ext_array_radius),
      S("ext.array_focus_dx", T::F64, ext_array_focus_dx), S("ext.array_seed", T::U64, ext_array_seed),
      S("ext.array_phases", T::I32, ext_array_phases), S("ext.rp_reuse", T::Bool, ext_rp_reuse),
  };
#undef S
  return m;
}

std::string strip(const std::string& s) {
  const char* ws = " \t\r\n\f\v";
  size_t a = s.find_first_not_of(ws);
  if (a == std::string::npos) return std::string();
  size_t b = s.find_last_not_of(ws);
  return s.substr(a, b - a + 1);
}

// One word from a fixed list of spellings, case-insensitive; -1 if absent.
int pick(std::string v, std::initializer_list<std::initializer_list<const char*>> names) {
  for (auto& c : v) c = (char)std::tolower((unsigned char)c);
  int k = 0;
  for (auto& group : names) {
    for (const char* n : group)
      if (v == n) return k;
    k++;
  }
  return -1;
}

bool store(const Slot& s, const std::string& v, crp_config* cfg) {
  char* p = reinterpret_cast<char*>(cfg) + s.off;
  if (v.empty()) return false;
  char* end = nullptr;
  errno = 0;
  switch (s.type) {
    case T::I32: {
      long long x = std::strtoll(v.c_str(), &end, 10);
      if (errno || *end || x < INT32_MIN || x > INT32_MAX) return false;
      *reinterpret_cast<int32_t*>(p) = (int32_t)x;
      return true;
    }
    case T::U64: {
      unsigned long long x = std::strtoull(v.c_str(), &end, 0);
      if (errno || *end) return false;
      *reinterpret_cast<uint64_t*>(p) = (uint64_t)x;
      return true;
    }
    case T::F64: {
      double x = std::strtod(v.c_str(), &end);
      if ((errno == ERANGE && !std::isfinite(x)) || *end) return false;
      *reinterpret_cast<double*>(p) = x;
      return true;
    }
    case T::Bool: {
      int k = pick(v, {{"0", "false", "no", "off"}, {"1", "true", "yes", "on"}});
      if (k < 0) return false;
      *reinterpret_cast<int32_t*>(p) = k;
      return true;
    }
    case T::Prec: {
      int k = pick(v, {{"fp64", "0"}, {"mixed", "1"}});
      if (k < 0) return false;
      *reinterpret_cast<int32_t*>(p) = k;
      return true;
    }
    case T::Shape: {
      int k = pick(v, {{"cylinder", "0"}, {"sphere", "1"}, {"gaussian", "2"}});
      if (k < 0) return false;
      *reinterpret_cast<int32_t*>(p) = k;
      return true;
    }
    case T::Scheme: {
      int k = pick(v, {{"ref", "0"}, {"rk45", "1"}});
      if (k < 0) return false;
      *reinterpret_cast<int32_t*>(p) = k;
      return true;
    }
  }
  return false;
}

crp_status fail(char* err, size_t n, int line, const std::string& what) {
  if (err && n) std::snprintf(err, n, "line %d: %s", line, what.c_str());
  return CRP_ERR_PARSE;
}

// Philox-4x32-10: ten rounds of the 4x32 bijection with the published
// multipliers 0xD2511F53, 0xCD9E8D57 and Weyl key increments 0x9E3779B9,
// 0xBB67AE85 (SC'11, section 3).
void philox4x32(uint64_t seed, uint64_t counter, uint32_t stream, uint32_t out[4]) {
  uint32_t x0 = (uint32_t)counter, x1 = (uint32_t)(counter >> 32), x2 = stream, x3 = 0u;
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  for (int round = 0; round < 10; round++) {
    const uint64_t m0 = (uint64_t)0xD2511F53u * x0;
    const uint64_t m1 = (uint64_t)0xCD9E8D57u * x2;
    const uint32_t y0 = (uint32_t)(m1 >> 32) ^ x1 ^ k0;
    const uint32_t y1 = (uint32_t)m1;
    const uint32_t y2 = (uint32_t)(m0 >> 32) ^ x3 ^ k1;
    const uint32_t y3 = (uint32_t)m0;
    x0 = y0;
    x1 = y1;
    x2 = y2;
    x3 = y3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = x0;
  out[1] = x1;
  out[2] = x2;
  out[3] = x3;
}

// A 32-bit word as a double in (0, 1): the midpoint of its 2^-32-wide bin.
double open01(uint32_t w) { return ((double)w + 0.5) / 4294967296.0; }

}  // namespace

extern "C" {

crp_status crpo_config_defaults(crp_config* cfg) {
  if (!cfg) return CRP_ERR_INVALID;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->tr_pid_start_step = 1;
  cfg->tr_pid_iterate = 1;
  cfg->dbg_display = 4;
  cfg->dbg_fg = 1;
  cfg->dbg_T = 1;
  cfg->dbg_bubbles = 1;
  cfg->ext_rho_inf = 1000.0;
  cfg->ext_c_inf = 1500.0;
  cfg->ext_p_inf = 1.0e5;
  cfg->ext_picard_cap = 1000;
  cfg->ext_rp_reuse = 1;
  cfg->ext_rp_step_cap = 1000000;
  cfg->ext_n_b = 1.0;
  return CRP_OK;
}

crp_status crpo_config_parse_file(const char* path, crp_config* cfg, char* err, size_t err_len) {
  if (!path || !cfg) return CRP_ERR_INVALID;
  std::ifstream in(path);
  if (!in) {
    if (err && err_len) std::snprintf(err, err_len, "cannot open %s", path);
    return CRP_ERR_IO;
  }
  const auto& reg = registry();
  std::set<std::string> given;
  std::string raw, prefix;
  for (int line = 1; std::getline(in, raw); line++) {
    std::string s = strip(raw.substr(0, raw.find('#')));
    if (s.empty()) continue;
    if (s[0] == '[') {
      if (s.back() != ']') return fail(err, err_len, line, "bad section header");
      prefix = strip(s.substr(1, s.size() - 2));
      continue;
    }
    size_t eq = s.find('=');
    if (eq == std::string::npos) return fail(err, err_len, line, "expected name = value");
    std::string key = strip(s.substr(0, eq));
    if (!prefix.empty()) key = prefix + "." + key;
    auto it = reg.find(key);
    if (it == reg.end()) continue;
    if (!given.insert(key).second) return fail(err, err_len, line, "multiple occurrences of '" + key + "'");
    std::string value = strip(s.substr(eq + 1));
    if (!store(it->second, value, cfg))
      return fail(err, err_len, line, "invalid value '" + value + "' for option '" + key + "'");
  }
  return CRP_OK;
}

crp_status crpo_seed_bubbles(const crp_config* cfg, double* x, double* y, double* r0, double* n_b) {
  if (!cfg || !x || !y || !r0 || !n_b || cfg->ext_bubble_count <= 0) return CRP_ERR_INVALID;
  const double two_pi = 2.0 * std::acos(-1.0);
  const bool axisym = cfg->tr_cylindrical != 0;
  // Focal depth of init_transducer (src/bubble_CUDA.cu:549): f_dist * sqrt(3) / 2.
  const double focus = cfg->tr_focal_dist ? cfg->tr_focal_dist * 0.5 * std::sqrt(3.0) : cfg->grid_ly * 0.5;
  const double R = cfg->ext_cloud_r;
  for (int32_t k = 0; k < cfg->ext_bubble_count; k++) {
    uint32_t w[4], v[4];
    philox4x32(cfg->ext_bubble_seed, (uint64_t)k, 0u, w);
    philox4x32(cfg->ext_bubble_seed, (uint64_t)k, 1u, v);
    double r, z;
    if (cfg->ext_cloud_shape == 1) {
      // Uniform in a ball: radius R u^(1/3), polar cosine uniform in [-1, 1].
      const double rad = R * std::cbrt(open01(w[0]));
      const double cth = 2.0 * open01(w[1]) - 1.0;
      const double sth = std::sqrt(std::max(0.0, 1.0 - cth * cth));
      r = axisym ? rad * sth : std::fabs(rad * sth * std::cos(two_pi * open01(w[2])));
      z = rad * cth;
    } else if (cfg->ext_cloud_shape == 2) {
      // Gaussian, standard deviation R per axis (Box-Muller).
      const double m = std::sqrt(-2.0 * std::log(open01(w[0])));
      r = axisym ? R * m : std::fabs(R * m * std::cos(two_pi * open01(w[1])));
      z = R * std::sqrt(-2.0 * std::log(open01(v[2]))) * std::cos(two_pi * open01(v[3]));
    } else {
      // Cylinder r <= R, |z| <= h/2; area-uniform in r about the axis.
      r = axisym ? R * std::sqrt(open01(w[0])) : R * open01(w[0]);
      z = (open01(w[1]) - 0.5) * cfg->ext_cloud_h;
    }
    const double gauss = std::sqrt(-2.0 * std::log(open01(v[0]))) * std::cos(two_pi * open01(v[1]));
    x[k] = r;
    y[k] = focus + z;
    r0[k] = cfg->bub_R0 * std::exp(cfg->ext_r0_sigma_ln * gauss);
    n_b[k] = cfg->ext_n_b;
  }
  return CRP_OK;
}

// 3-D cloud about the bowl's focus (grid centre + ext_array_focus_dx along x):
// cylinder along z (area-uniform radius), ball, or Gaussian per axis; the
// same two Philox blocks per bubble as the 2-D seeding.
crp_status crpo_seed_bubbles3(const crp_config* cfg, double* x, double* y, double* z, double* r0, double* n_b) {
  if (!cfg || !x || !y || !z || !r0 || !n_b || cfg->ext_bubble_count <= 0 || cfg->ext_grid_z <= 0)
    return CRP_ERR_INVALID;
  const double two_pi = 2.0 * std::acos(-1.0);
  const double fx = 0.5 * cfg->grid_lx + cfg->ext_array_focus_dx, fy = 0.5 * cfg->grid_ly,
               fz = 0.5 * cfg->ext_grid_lz;
  const double R = cfg->ext_cloud_r;
  for (int32_t k = 0; k < cfg->ext_bubble_count; k++) {
    uint32_t w[4], v[4];
    philox4x32(cfg->ext_bubble_seed, (uint64_t)k, 0u, w);
    philox4x32(cfg->ext_bubble_seed, (uint64_t)k, 1u, v);
    double ox, oy, oz;
    if (cfg->ext_cloud_shape == 1) {
      const double rad = R * std::cbrt(open01(w[0]));
      const double cth = 2.0 * open01(w[1]) - 1.0;
      const double sth = std::sqrt(std::max(0.0, 1.0 - cth * cth));
      const double ph = two_pi * open01(w[2]);
      ox = rad * sth * std::cos(ph);
      oy = rad * sth * std::sin(ph);
      oz = rad * cth;
    } else if (cfg->ext_cloud_shape == 2) {
      const double m = std::sqrt(-2.0 * std::log(open01(w[0])));
      ox = R * m * std::cos(two_pi * open01(w[1]));
      oy = R * m * std::sin(two_pi * open01(w[1]));
      oz = R * std::sqrt(-2.0 * std::log(open01(v[2]))) * std::cos(two_pi * open01(v[3]));
    } else {
      const double rr = R * std::sqrt(open01(w[0]));
      const double ph = two_pi * open01(w[2]);
      ox = rr * std::cos(ph);
      oy = rr * std::sin(ph);
      oz = (open01(w[1]) - 0.5) * cfg->ext_cloud_h;
    }
    const double gauss = std::sqrt(-2.0 * std::log(open01(v[0]))) * std::cos(two_pi * open01(v[1]));
    x[k] = fx + ox;
    y[k] = fy + oy;
    z[k] = fz + oz;
    r0[k] = cfg->bub_R0 * std::exp(cfg->ext_r0_sigma_ln * gauss);
    n_b[k] = cfg->ext_n_b;
  }
  return CRP_OK;
}

void crpo_philox_block(uint64_t seed, uint64_t counter, uint32_t stream, uint32_t out[4]) {
  philox4x32(seed, counter, stream, out);
}

}  // extern "C"
