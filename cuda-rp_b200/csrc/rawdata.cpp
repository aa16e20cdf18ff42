// Plain-text rawdata writer: the file names, column order, number formatting
// and row separators of save_ascii (src/output_styles.cpp:139-341).
//
//   fg_step_%05d.txt, T_step_%05d.txt, p0_step_%05d.txt, vx_step_%05d.txt, vy_step_%05d.txt:
//     one line "x<TAB>y<TAB>value" per point for j = 0..Y and i = 0..X (or
//     i = -X..X mirrored when axisymmetric), a blank line after each row j;
//   bubble_radii_%05d.txt, bubble_PG_%05d.txt: "x<TAB>y<TAB>R" / "x<TAB>y<TAB>PG".
// Numbers use the default ostream conversion (%g, 6 significant digits).
//
// SPH files (save_sph, src/output_styles.cpp:36-137, and SphData::SaveSph,
// src/SphDataType.cpp:142-192): fg/p0/T_step_%05d.sph, each a sequence of
// length-framed records (int length, bytes, int length): {svType = 1 (scalar),
// dType = 1 (float)}, dims {X+1, Y+1, 1}, origin {0, 0, 0}, pitch {dx, dy, 1}
// (float), {step (int), time (float)}, then the values as floats for
// j = 0..Y, i = 0..X (no mirroring), x fastest.
#include <sys/stat.h>

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "crp_host.h"

namespace crp {

namespace {

crp_status make_dirs(const std::string& dir) {
  std::string acc;
  for (size_t k = 0; k < dir.size(); k++) {
    acc.push_back(dir[k]);
    if (dir[k] == '/' || k + 1 == dir.size()) {
      if (acc == "/" || acc.empty()) continue;
      if (mkdir(acc.c_str(), 0755) != 0 && errno != EEXIST) return CRP_ERR_IO;
    }
  }
  return CRP_OK;
}

std::string step_name(const std::string& dir, const char* stem, int64_t step) {
  char buf[64];
  std::snprintf(buf, sizeof(buf), "%s%05lld.txt", stem, (long long)step);
  return dir + buf;
}

class Out {
 public:
  explicit Out(const std::string& path) { f_ = std::fopen(path.c_str(), "w"); }
  ~Out() {
    if (f_) std::fclose(f_);
  }
  bool ok() const { return f_ != nullptr; }
  void triple(double a, double b, double c) { std::fprintf(f_, "%g\t%g\t%g\n", a, b, c); }
  void blank() { std::fputc('\n', f_); }

 private:
  FILE* f_;
};

// One grid field: value(|i|, j) from a dense array with origin (i0, j0) and width w.
crp_status write_grid(const std::string& path, const crp_config& c, double dx, double dy,
                      const std::vector<double>& a, int i0, int j0, int w, double* vmin, double* vmax) {
  Out o(path);
  if (!o.ok()) return CRP_ERR_IO;
  const int X = c.grid_x, Y = c.grid_y;
  for (int j = 0; j <= Y; j++) {
    for (int i = (c.tr_cylindrical ? -X : 0); i <= X; i++) {
      double v = a[(size_t)(j - j0) * w + (std::abs(i) - i0)];
      o.triple((double)i * dx, (double)j * dy, v);
      if (vmin) {
        *vmax = std::max(*vmax, v);
        *vmin = std::min(*vmin, v);
      }
    }
    o.blank();
  }
  return CRP_OK;
}

// One SPH file.
crp_status write_sph_grid(const std::string& path, const crp_config& c, double dx, double dy, int64_t step,
                          double t, const std::vector<double>& a, int w, double* vmin, double* vmax) {
  const int X = c.grid_x, Y = c.grid_y;
  std::vector<float> v((size_t)(X + 1) * (Y + 1));
  for (int j = 0; j <= Y; j++)
    for (int i = 0; i <= X; i++) {
      const double x = a[(size_t)j * w + i];
      v[(size_t)j * (X + 1) + i] = (float)x;
      *vmax = std::max(*vmax, x);
      *vmin = std::min(*vmin, x);
    }
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return CRP_ERR_IO;
  auto rec = [&](const void* p, int32_t len) {
    std::fwrite(&len, 4, 1, f);
    std::fwrite(p, 1, (size_t)len, f);
    std::fwrite(&len, 4, 1, f);
  };
  const int32_t types[2] = {1, 1};
  const int32_t dims[3] = {X + 1, Y + 1, 1};
  const float origin[3] = {0.0f, 0.0f, 0.0f};
  const float pitch[3] = {(float)dx, (float)dy, 1.0f};
  struct {
    int32_t step;
    float time;
  } st{(int32_t)step, (float)t};
  rec(types, 8);
  rec(dims, 12);
  rec(origin, 12);
  rec(pitch, 12);
  rec(&st, 8);
  rec(v.data(), (int32_t)(4 * v.size()));
  const bool ok = std::ferror(f) == 0;
  std::fclose(f);
  return ok ? CRP_OK : CRP_ERR_IO;
}

std::string sph_name(const std::string& dir, const char* stem, int64_t step) {
  char buf[64];
  std::snprintf(buf, sizeof(buf), "%s%05lld.sph", stem, (long long)step);
  return dir + buf;
}

}  // namespace

crp_status write_sph(crp_sim* sim, const char* dir_c) {
  const crp_config& c = sim_config(sim);
  std::string dir(dir_c);
  if (dir.empty()) dir = "./rawdata/";
  if (dir.back() != '/') dir += "/";
  if (make_dirs(dir) != CRP_OK) return CRP_ERR_IO;
  crp_dims d;
  crp_status st = crp_get_dims(sim, &d);
  if (st != CRP_OK) return st;
  const int64_t step = sim_step_count(sim);
  // save_sph receives the time as a float (src/bubble_CUDA.cu:397).
  const double t = (double)(float)sim_time(sim);
  MinMax& mm = sim_minmax(sim);
  std::vector<double> buf;
  if (c.dbg_fg) {
    buf.resize((size_t)d.i2m * d.j2m);
    if ((st = sim_read_field(sim, CRP_FIELD_FG, buf.data())) != CRP_OK) return st;
    st = write_sph_grid(sph_name(dir, "fg_step_", step), c, d.dx, d.dy, step, t, buf, d.i2m, &mm.fg_min, &mm.fg_max);
    if (st != CRP_OK) return st;
  }
  if (c.dbg_p) {
    buf.resize((size_t)d.i1m * d.j1m);
    if ((st = sim_read_field(sim, CRP_FIELD_P0, buf.data())) != CRP_OK) return st;
    st = write_sph_grid(sph_name(dir, "p0_step_", step), c, d.dx, d.dy, step, t, buf, d.i1m, &mm.p0_min, &mm.p0_max);
    if (st != CRP_OK) return st;
  }
  if (c.dbg_T) {
    buf.resize((size_t)d.i2m * d.j2m);
    if ((st = sim_read_field(sim, CRP_FIELD_T, buf.data())) != CRP_OK) return st;
    st = write_sph_grid(sph_name(dir, "T_step_", step), c, d.dx, d.dy, step, t, buf, d.i2m, &mm.T_min, &mm.T_max);
    if (st != CRP_OK) return st;
  }
  return CRP_OK;
}

crp_status write_rawdata(crp_sim* sim, const char* dir_c) {
  const crp_config& c = sim_config(sim);
  std::string dir(dir_c);
  if (dir.empty()) dir = "./rawdata/";
  if (dir.back() != '/') dir += "/";
  if (make_dirs(dir) != CRP_OK) return CRP_ERR_IO;
  crp_dims d;
  crp_status st = crp_get_dims(sim, &d);
  if (st != CRP_OK) return st;
  const int64_t step = sim_step_count(sim);
  MinMax& mm = sim_minmax(sim);
  std::vector<double> buf;
  if (c.dbg_fg) {
    buf.resize((size_t)d.i2m * d.j2m);
    if ((st = sim_read_field(sim, CRP_FIELD_FG, buf.data())) != CRP_OK) return st;
    st = write_grid(step_name(dir, "fg_step_", step), c, d.dx, d.dy, buf, 0, 0, d.i2m, &mm.fg_min, &mm.fg_max);
    if (st != CRP_OK) return st;
  }
  if (c.dbg_T) {
    buf.resize((size_t)d.i2m * d.j2m);
    if ((st = sim_read_field(sim, CRP_FIELD_T, buf.data())) != CRP_OK) return st;
    st = write_grid(step_name(dir, "T_step_", step), c, d.dx, d.dy, buf, 0, 0, d.i2m, &mm.T_min, &mm.T_max);
    if (st != CRP_OK) return st;
  }
  if (c.dbg_p) {
    buf.resize((size_t)d.i1m * d.j1m);
    if ((st = sim_read_field(sim, CRP_FIELD_P0, buf.data())) != CRP_OK) return st;
    st = write_grid(step_name(dir, "p0_step_", step), c, d.dx, d.dy, buf, 0, 0, d.i1m, &mm.p0_min, &mm.p0_max);
    if (st != CRP_OK) return st;
  }
  if (c.dbg_v) {
    buf.resize((size_t)d.i2n * d.j2m);
    if ((st = sim_read_field(sim, CRP_FIELD_VX, buf.data())) != CRP_OK) return st;
    st = write_grid(step_name(dir, "vx_step_", step), c, d.dx, d.dy, buf, -1, 0, d.i2n, nullptr, nullptr);
    if (st != CRP_OK) return st;
    buf.resize((size_t)d.i2m * d.j2n);
    if ((st = sim_read_field(sim, CRP_FIELD_VY, buf.data())) != CRP_OK) return st;
    st = write_grid(step_name(dir, "vy_step_", step), c, d.dx, d.dy, buf, 0, -1, d.i2m, nullptr, nullptr);
    if (st != CRP_OK) return st;
  }
  if (c.dbg_bubbles && d.num_bubbles > 0) {
    std::vector<double> x(d.num_bubbles), y(d.num_bubbles), v(d.num_bubbles);
    if ((st = sim_read_bubbles(sim, CRP_BUB_X, x.data())) != CRP_OK) return st;
    if ((st = sim_read_bubbles(sim, CRP_BUB_Y, y.data())) != CRP_OK) return st;
    if ((st = sim_read_bubbles(sim, CRP_BUB_R_T, v.data())) != CRP_OK) return st;
    {
      Out o(step_name(dir, "bubble_radii_", step));
      if (!o.ok()) return CRP_ERR_IO;
      for (int k = 0; k < d.num_bubbles; k++) o.triple(x[k], y[k], v[k]);
    }
    if ((st = sim_read_bubbles(sim, CRP_BUB_PG, v.data())) != CRP_OK) return st;
    {
      Out o(step_name(dir, "bubble_PG_", step));
      if (!o.ok()) return CRP_ERR_IO;
      for (int k = 0; k < d.num_bubbles; k++) o.triple(x[k], y[k], v[k]);
    }
  }
  return CRP_OK;
}

}  // namespace crp
