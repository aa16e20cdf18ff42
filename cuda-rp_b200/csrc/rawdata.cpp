// Plain-text rawdata writer: the file names, column order, number formatting
// and row separators of save_ascii (src/output_styles.cpp:139-341).
//
//   fg_step_%05d.txt, T_step_%05d.txt, p0_step_%05d.txt, vx_step_%05d.txt, vy_step_%05d.txt:
//     one line "x<TAB>y<TAB>value" per point for j = 0..Y and i = 0..X (or
//     i = -X..X mirrored when axisymmetric), a blank line after each row j;
//   bubble_radii_%05d.txt, bubble_PG_%05d.txt: "x<TAB>y<TAB>R" / "x<TAB>y<TAB>PG".
// Numbers use the default ostream conversion (%g, 6 significant digits).
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

}  // namespace

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
