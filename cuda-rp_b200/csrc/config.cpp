// Configuration: reference defaults, the INI grammar of Boost program_options'
// config files as src/bubbles.cpp uses it, and the [ext] bubble seeding.
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <set>
#include <sstream>
#include <string>

#include "crp.h"

namespace {

void set_err(char* err, size_t n, const std::string& msg) {
  if (err && n) {
    std::snprintf(err, n, "%s", msg.c_str());
  }
}

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) a++;
  while (b > a && std::isspace((unsigned char)s[b - 1])) b--;
  return s.substr(a, b - a);
}

std::string lower(std::string s) {
  for (auto& c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

bool parse_int(const std::string& v, int32_t* out) {
  if (v.empty()) return false;
  char* end = nullptr;
  errno = 0;
  long long x = std::strtoll(v.c_str(), &end, 10);
  if (errno || *end != '\0' || x < INT32_MIN || x > INT32_MAX) return false;
  *out = (int32_t)x;
  return true;
}

bool parse_u64(const std::string& v, uint64_t* out) {
  if (v.empty()) return false;
  char* end = nullptr;
  errno = 0;
  unsigned long long x = std::strtoull(v.c_str(), &end, 0);
  if (errno || *end != '\0') return false;
  *out = (uint64_t)x;
  return true;
}

bool parse_double(const std::string& v, double* out) {
  if (v.empty()) return false;
  char* end = nullptr;
  errno = 0;
  double x = std::strtod(v.c_str(), &end);
  if (errno == ERANGE && !std::isfinite(x)) return false;
  if (*end != '\0') return false;
  *out = x;
  return true;
}

// Boolean spellings accepted by program_options' bool validator.
bool parse_bool(const std::string& v, int32_t* out) {
  std::string s = lower(v);
  if (s == "1" || s == "true" || s == "yes" || s == "on") {
    *out = 1;
    return true;
  }
  if (s == "0" || s == "false" || s == "no" || s == "off") {
    *out = 0;
    return true;
  }
  return false;
}

enum Kind { kInt, kDouble, kBool, kU64, kPrecision, kShape, kScheme };

struct Key {
  const char* name;
  Kind kind;
  size_t offset;
};

#define K(name, kind, field) {name, kind, offsetof(crp_config, field)}
// Registered keys of src/bubbles.cpp:70-133 (file options and the generic
// options that may appear in a file), then the [ext] section.
const Key kKeys[] = {
    K("grid.x", kInt, grid_x),
    K("grid.y", kInt, grid_y),
    K("grid.lx", kDouble, grid_lx),
    K("grid.ly", kDouble, grid_ly),
    K("pml.x0", kBool, pml_x0),
    K("pml.x1", kBool, pml_x1),
    K("pml.y0", kBool, pml_y0),
    K("pml.y1", kBool, pml_y1),
    K("pml.grid_number", kInt, pml_grid_number),
    K("pml.sigma", kDouble, pml_sigma),
    K("pml.order", kInt, pml_order),
    K("simulation.cfl", kDouble, sim_cfl),
    K("simulation.dt0", kDouble, sim_dt0),
    K("simulation.n_step_max", kInt, sim_n_step_max),
    K("simulation.t_step_max", kDouble, sim_t_step_max),
    K("simulation.save_interval", kInt, sim_save_interval),
    K("simulation.order", kInt, sim_order),
    K("simulation.smooth_delta_band", kInt, sim_smooth_delta_band),
    K("transducer.amp", kDouble, tr_amp),
    K("transducer.freq", kDouble, tr_freq),
    K("transducer.focal_dist", kDouble, tr_focal_dist),
    K("transducer.pid", kBool, tr_pid),
    K("transducer.pid_start_step", kInt, tr_pid_start_step),
    K("transducer.init_control", kDouble, tr_init_control),
    K("transducer.pid_iterate", kInt, tr_pid_iterate),
    K("transducer.box_size", kDouble, tr_box_size),
    K("transducer.cylindrical", kBool, tr_cylindrical),
    K("transducer.on_wave", kInt, tr_on_wave),
    K("transducer.off_wave", kInt, tr_off_wave),
    K("transducer.transducer_v", kBool, tr_plane_v),
    K("transducer.transducer_p", kBool, tr_plane_p),
    K("transducer.focused_wave_v", kBool, tr_focused_v),
    K("transducer.focused_wave_p", kBool, tr_focused_p),
    K("bubbles.enable", kBool, bub_enable),
    K("bubbles.fg0", kDouble, bub_fg0),
    K("bubbles.R0", kDouble, bub_R0),
    K("bubbles.P0", kDouble, bub_P0),
    K("bubbles.T0", kDouble, bub_T0),
    K("bubbles.gamma", kDouble, bub_gamma),
    K("bubbles.liquid_surface_tension", kDouble, bub_sigma),
    K("bubbles.liquid_viscosity", kDouble, bub_mu),
    K("bubbles.liquid_density", kDouble, bub_rho),
    K("bubbles.K0", kDouble, bub_K0),
    K("debug.display_dim", kInt, dbg_display),
    K("debug.fg", kBool, dbg_fg),
    K("debug.T", kBool, dbg_T),
    K("debug.p", kBool, dbg_p),
    K("debug.v", kBool, dbg_v),
    K("debug.bubbles", kBool, dbg_bubbles),
    K("ascii", kBool, opt_ascii),
    K("sph", kBool, opt_sph),
    K("ext.rho_inf", kDouble, ext_rho_inf),
    K("ext.c_inf", kDouble, ext_c_inf),
    K("ext.p_inf", kDouble, ext_p_inf),
    K("ext.source_row", kInt, ext_source_row),
    K("ext.ramp_cycles", kDouble, ext_ramp_cycles),
    K("ext.precision", kPrecision, ext_precision),
    K("ext.picard_cap", kInt, ext_picard_cap),
    K("ext.rp_step_cap", kInt, ext_rp_step_cap),
    K("ext.bubble_count", kInt, ext_bubble_count),
    K("ext.bubble_seed", kU64, ext_bubble_seed),
    K("ext.r0_sigma_ln", kDouble, ext_r0_sigma_ln),
    K("ext.cloud_shape", kShape, ext_cloud_shape),
    K("ext.cloud_r", kDouble, ext_cloud_r),
    K("ext.cloud_h", kDouble, ext_cloud_h),
    K("ext.n_b", kDouble, ext_n_b),
    K("ext.picard_tol", kDouble, ext_picard_tol),
    K("ext.graphs", kBool, ext_graphs),
    K("ext.elements", kInt, ext_elements),
    K("ext.rp_scheme", kScheme, ext_rp_scheme),
    K("ext.rp_tol", kDouble, ext_rp_tol),
    K("ext.grid_z", kInt, ext_grid_z),
    K("ext.grid_lz", kDouble, ext_grid_lz),
    K("ext.pml_z0", kBool, ext_pml_z0),
    K("ext.pml_z1", kBool, ext_pml_z1),
    K("ext.array_elements", kInt, ext_array_elements),
    K("ext.array_radius", kDouble, ext_array_radius),
    K("ext.array_focus_dx", kDouble, ext_array_focus_dx),
    K("ext.array_seed", kU64, ext_array_seed),
    K("ext.array_phases", kInt, ext_array_phases),
    K("ext.rp_reuse", kBool, ext_rp_reuse),
};
#undef K

// Keys registered in the reference with a value but not stored in a struct
// (src/bubbles.cpp:121-131); accepted and ignored.
const char* kIgnoredKeys[] = {"debug.fg_min", "debug.fg_max", "debug.T_min", "debug.T_max",
                              "debug.p_max",  "debug.v_min",  "debug.v_max", "directory"};

bool assign(const Key& k, const std::string& value, crp_config* cfg) {
  char* base = reinterpret_cast<char*>(cfg) + k.offset;
  switch (k.kind) {
    case kInt: return parse_int(value, reinterpret_cast<int32_t*>(base));
    case kDouble: return parse_double(value, reinterpret_cast<double*>(base));
    case kBool: return parse_bool(value, reinterpret_cast<int32_t*>(base));
    case kU64: return parse_u64(value, reinterpret_cast<uint64_t*>(base));
    case kPrecision: {
      std::string s = lower(value);
      int32_t* p = reinterpret_cast<int32_t*>(base);
      if (s == "fp64" || s == "0") return *p = CRP_PREC_FP64, true;
      if (s == "mixed" || s == "1") return *p = CRP_PREC_MIXED, true;
      return false;
    }
    case kShape: {
      std::string s = lower(value);
      int32_t* p = reinterpret_cast<int32_t*>(base);
      if (s == "cylinder" || s == "0") return *p = 0, true;
      if (s == "sphere" || s == "1") return *p = 1, true;
      if (s == "gaussian" || s == "2") return *p = 2, true;
      return false;
    }
    case kScheme: {
      std::string s = lower(value);
      int32_t* p = reinterpret_cast<int32_t*>(base);
      if (s == "ref" || s == "0") return *p = CRP_RP_REF, true;
      if (s == "rk45" || s == "1") return *p = CRP_RP_RK45, true;
      return false;
    }
  }
  return false;
}

crp_status parse_stream(std::istream& in, crp_config* cfg, char* err, size_t err_len) {
  std::string line, section;
  std::set<std::string> seen;
  int lineno = 0;
  while (std::getline(in, line)) {
    lineno++;
    size_t hash = line.find('#');
    if (hash != std::string::npos) line = line.substr(0, hash);
    line = trim(line);
    if (line.empty()) continue;
    if (line.front() == '[') {
      if (line.back() != ']') {
        set_err(err, err_len, "line " + std::to_string(lineno) + ": bad section header");
        return CRP_ERR_PARSE;
      }
      section = trim(line.substr(1, line.size() - 2));
      continue;
    }
    size_t eq = line.find('=');
    if (eq == std::string::npos) {
      set_err(err, err_len, "line " + std::to_string(lineno) + ": expected name = value");
      return CRP_ERR_PARSE;
    }
    std::string name = trim(line.substr(0, eq));
    std::string value = trim(line.substr(eq + 1));
    std::string full = section.empty() ? name : section + "." + name;
    const Key* key = nullptr;
    for (const Key& k : kKeys)
      if (full == k.name) key = &k;
    if (!key) continue;  // unregistered keys are ignored (allow_unregistered)
    if (!seen.insert(full).second) {
      set_err(err, err_len, "line " + std::to_string(lineno) + ": multiple occurrences of '" + full + "'");
      return CRP_ERR_PARSE;
    }
    if (!assign(*key, value, cfg)) {
      set_err(err, err_len,
              "line " + std::to_string(lineno) + ": invalid value '" + value + "' for option '" + full + "'");
      return CRP_ERR_PARSE;
    }
  }
  (void)kIgnoredKeys;
  return CRP_OK;
}

// ---------------------------------------------------------------------------
// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), counter-based.
struct Philox {
  uint32_t k0, k1;
  static void mulhilo(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
    uint64_t p = (uint64_t)a * (uint64_t)b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
  }
  void block(uint64_t counter, uint32_t stream, uint32_t out[4]) const {
    uint32_t c[4] = {(uint32_t)counter, (uint32_t)(counter >> 32), stream, 0u};
    uint32_t a = k0, b = k1;
    for (int r = 0; r < 10; r++) {
      uint32_t hi0, lo0, hi1, lo1;
      mulhilo(0xD2511F53u, c[0], hi0, lo0);
      mulhilo(0xCD9E8D57u, c[2], hi1, lo1);
      uint32_t n0 = hi1 ^ c[1] ^ a;
      uint32_t n2 = hi0 ^ c[3] ^ b;
      c[0] = n0;
      c[1] = lo1;
      c[2] = n2;
      c[3] = lo0;
      a += 0x9E3779B9u;
      b += 0xBB67AE85u;
    }
    for (int i = 0; i < 4; i++) out[i] = c[i];
  }
};

inline double unit(uint32_t u) { return ((double)u + 0.5) * (1.0 / 4294967296.0); }

}  // namespace

extern "C" {

crp_status crp_config_defaults(crp_config* cfg) {
  if (!cfg) return CRP_ERR_INVALID;
  std::memset(cfg, 0, sizeof(*cfg));
  // Defaults registered in src/bubbles.cpp:97-132.
  cfg->tr_pid = 0;
  cfg->tr_pid_start_step = 1;
  cfg->tr_init_control = 0.0;
  cfg->tr_pid_iterate = 1;
  cfg->bub_enable = 0;
  cfg->dbg_display = 4;
  cfg->dbg_fg = 1;
  cfg->dbg_T = 1;
  cfg->dbg_p = 0;
  cfg->dbg_v = 0;
  cfg->dbg_bubbles = 1;
  // Values the reference hard-codes (density_water, adiabatic_sound_speed_water,
  // init_mix: inc/bubble_CUDA_kernel.cuh:153-169, src/bubble_CUDA.cu:636-646).
  cfg->ext_rho_inf = 1000.0;
  cfg->ext_c_inf = 1500.0;
  cfg->ext_p_inf = 0.1e6;
  cfg->ext_precision = CRP_PREC_FP64;
  cfg->ext_picard_cap = 1000;
  cfg->ext_rp_reuse = 1;
  cfg->ext_graphs = 0;
  cfg->ext_elements = 0;
  cfg->ext_rp_step_cap = 1000000;
  cfg->ext_n_b = 1.0;
  return CRP_OK;
}

crp_status crp_config_parse_string(const char* text, crp_config* cfg, char* err, size_t err_len) {
  if (!text || !cfg) return CRP_ERR_INVALID;
  std::istringstream in(text);
  return parse_stream(in, cfg, err, err_len);
}

crp_status crp_config_parse_file(const char* path, crp_config* cfg, char* err, size_t err_len) {
  if (!path || !cfg) return CRP_ERR_INVALID;
  std::ifstream in(path);
  if (!in) {
    set_err(err, err_len, std::string("cannot open ") + path);
    return CRP_ERR_IO;
  }
  return parse_stream(in, cfg, err, err_len);
}

crp_status crp_seed_bubbles(const crp_config* cfg, double* x, double* y, double* r0, double* n_b) {
  if (!cfg || !x || !y || !r0 || !n_b || cfg->ext_bubble_count <= 0) return CRP_ERR_INVALID;
  const double pi = std::acos(-1.0);
  // Focus of init_transducer (src/bubble_CUDA.cu:546-555).
  double fy = cfg->tr_focal_dist ? cfg->tr_focal_dist * 0.5 * std::sqrt(3.0) : cfg->grid_ly * 0.5;
  Philox g{(uint32_t)cfg->ext_bubble_seed, (uint32_t)(cfg->ext_bubble_seed >> 32)};
  for (int32_t k = 0; k < cfg->ext_bubble_count; k++) {
    uint32_t a[4], b[4];
    g.block((uint64_t)k, 0u, a);
    g.block((uint64_t)k, 1u, b);
    double u0 = unit(a[0]), u1 = unit(a[1]), u2 = unit(a[2]);
    const bool cyl = cfg->tr_cylindrical != 0;
    double r = 0.0, z = 0.0;
    switch (cfg->ext_cloud_shape) {
      case 1: {  // uniform in a ball of radius cloud_r around the focus
        double rs = cfg->ext_cloud_r * std::cbrt(u0);
        double ct = 2.0 * u1 - 1.0;
        double st = std::sqrt(std::max(0.0, 1.0 - ct * ct));
        r = cyl ? rs * st : std::fabs(rs * st * std::cos(2.0 * pi * u2));
        z = rs * ct;
        break;
      }
      case 2: {  // gaussian cloud, standard deviation cloud_r per axis
        double s = cfg->ext_cloud_r;
        double rad = std::sqrt(-2.0 * std::log(u0));
        r = cyl ? s * rad : std::fabs(s * rad * std::cos(2.0 * pi * u1));
        z = s * std::sqrt(-2.0 * std::log(unit(b[2]))) * std::cos(2.0 * pi * unit(b[3]));
        break;
      }
      default: {  // cylinder r <= cloud_r, |z| <= cloud_h / 2 (area-uniform in r when axisymmetric)
        r = cyl ? cfg->ext_cloud_r * std::sqrt(u0) : cfg->ext_cloud_r * u0;
        z = (u1 - 0.5) * cfg->ext_cloud_h;
        break;
      }
    }
    double nrm = std::sqrt(-2.0 * std::log(unit(b[0]))) * std::cos(2.0 * pi * unit(b[1]));
    x[k] = r;
    y[k] = fy + z;
    r0[k] = cfg->bub_R0 * std::exp(cfg->ext_r0_sigma_ln * nrm);
    n_b[k] = cfg->ext_n_b;
  }
  return CRP_OK;
}

crp_status crp_seed_bubbles3(const crp_config* cfg, double* x, double* y, double* z, double* r0, double* n_b) {
  if (!cfg || !x || !y || !z || !r0 || !n_b || cfg->ext_bubble_count <= 0 || cfg->ext_grid_z <= 0)
    return CRP_ERR_INVALID;
  const double pi = std::acos(-1.0);
  // The cloud sits at the bowl's focus: the grid's centre moved by focus_dx along x.
  const double cx = 0.5 * cfg->grid_lx + cfg->ext_array_focus_dx, cy = 0.5 * cfg->grid_ly,
               cz = 0.5 * cfg->ext_grid_lz;
  const double R = cfg->ext_cloud_r;
  Philox g{(uint32_t)cfg->ext_bubble_seed, (uint32_t)(cfg->ext_bubble_seed >> 32)};
  for (int32_t k = 0; k < cfg->ext_bubble_count; k++) {
    uint32_t a[4], b[4];
    g.block((uint64_t)k, 0u, a);
    g.block((uint64_t)k, 1u, b);
    double ox, oy, oz;
    switch (cfg->ext_cloud_shape) {
      case 1: {  // ball
        const double rs = R * std::cbrt(unit(a[0]));
        const double ct = 2.0 * unit(a[1]) - 1.0;
        const double st = std::sqrt(std::max(0.0, 1.0 - ct * ct));
        const double ph = 2.0 * pi * unit(a[2]);
        ox = rs * st * std::cos(ph);
        oy = rs * st * std::sin(ph);
        oz = rs * ct;
        break;
      }
      case 2: {  // Gaussian per axis
        const double rad = std::sqrt(-2.0 * std::log(unit(a[0])));
        ox = R * rad * std::cos(2.0 * pi * unit(a[1]));
        oy = R * rad * std::sin(2.0 * pi * unit(a[1]));
        oz = R * std::sqrt(-2.0 * std::log(unit(b[2]))) * std::cos(2.0 * pi * unit(b[3]));
        break;
      }
      default: {  // cylinder along z, area-uniform in the radius
        const double rr = R * std::sqrt(unit(a[0]));
        const double ph = 2.0 * pi * unit(a[2]);
        ox = rr * std::cos(ph);
        oy = rr * std::sin(ph);
        oz = (unit(a[1]) - 0.5) * cfg->ext_cloud_h;
        break;
      }
    }
    const double nrm = std::sqrt(-2.0 * std::log(unit(b[0]))) * std::cos(2.0 * pi * unit(b[1]));
    x[k] = cx + ox;
    y[k] = cy + oy;
    z[k] = cz + oz;
    r0[k] = cfg->bub_R0 * std::exp(cfg->ext_r0_sigma_ln * nrm);
    n_b[k] = cfg->ext_n_b;
  }
  return CRP_OK;
}

const char* crp_status_string(crp_status s) {
  switch (s) {
    case CRP_OK: return "ok";
    case CRP_ERR_INVALID: return "invalid argument";
    case CRP_ERR_UNSUPPORTED: return "unsupported configuration";
    case CRP_ERR_CUDA: return "CUDA error";
    case CRP_ERR_ALLOC: return "allocation failed";
    case CRP_ERR_RP_STEPS: return "Rayleigh-Plesset sub-step cap exceeded";
    case CRP_ERR_PICARD: return "Picard iteration cap exceeded";
    case CRP_ERR_NONFINITE: return "non-finite value in state";
    case CRP_ERR_IO: return "I/O error";
    case CRP_ERR_PARSE: return "configuration parse error";
    case CRP_ERR_NO_DEVICE: return "no CUDA device";
    case CRP_ERR_TOO_LARGE: return "input larger than the library's fixed scratch buffer";
  }
  return "unknown status";
}

}  // extern "C"

namespace crp {
// One Philox-4x32-10 block of the seeding's generator (the 3-D source's seeded phases).
void philox_block(uint64_t seed, uint64_t counter, uint32_t stream, uint32_t out[4]) {
  Philox g{(uint32_t)seed, (uint32_t)(seed >> 32)};
  g.block(counter, stream, out);
}
}  // namespace crp
