// Device-side data layout, parameters and physics of the simulation path.
//
// HBM layout.  Every grid field is one 2-D array on a common padded frame
// covering logical i in [-1, X+2] and j in [-1, Y+2]; element (i, j) sits at
// (j + 1) * pitch + (i + 1), pitch a multiple of 32 elements, base 256-byte
// aligned.  The reference's differently-sized staggered arrays (vx over
// i2n x j2m, vy over i2m x j2n, p/f_g over i1m/i2m x j1m/j2m) are windows of this
// frame, so one index expression serves every field.  The mixture pressure is
// stored only as its split components (px, py); p0 = px + py and the boundary
// values of p0 are evaluated where they are read (p0_at).  The mixture density
// is derived from the previous void fraction, rho_m = (1 - f_g^{n-1}) rho_inf,
// exactly the value MixturePropertiesKernel stores
// (inc/bubble_CUDA_kernel.cuh:1122), so neither p0 nor rho_m occupies HBM.
#pragma once
#include <cuda_pipeline.h>

#include <cstdint>

namespace crp {

struct Frame {
  int X, Y;
  int pitch;  // elements
  __host__ __device__ __forceinline__ long idx(int i, int j) const { return (long)(j + 1) * pitch + (i + 1); }
};

// Scalars of grid_t, PML_t, transducer_t, mix_params_t and the [ext] keys the
// kernels read (inc/bubble_CUDA.h:71-164).
struct GridParams {
  Frame f;
  double dx, dy, rdx, rdy;
  double dt;
  double rho_inf, c_inf, P_inf;
  int pml_x0, pml_x1, pml_y0, pml_y1;
  int cyl;
  int plane_p, focused_p, plane_v, focused_v;
  int source_row;     // 0: ghost row y=0 when pml.y0 is off (reference); >0: forced row
  double amp, pamp, freq, omega;
  double on_time, period, ramp_time;
  double ctl_x, ctl_y, focal_dist;  // focal_point_c, focal_dist_c
  double dt_rho;    // dt / rho_inf
  double s3p, s4p;  // dt rho_inf c_inf^2 and dt c_inf / 2 of MixturePressureKernel (:852-853)
  // PML profiles and cylindrical metrics, indexed by logical i or j:
  // mx[i] i in [0,X+1], my[j] j in [0,Y+1], nx[i+1] i in [-1,X+1], ny[j+1] j in [-1,Y+1],
  // xu[i+1] i in [-1,X+1], rxp[i] i in [0,X+1].
  const double* mx;
  const double* my;
  const double* nx;
  const double* ny;
  const double* xu;
  const double* rxp;
  // PML update factors, 1 - s and 1 / (1 + s) (exactly 1 and 1 outside the
  // PML): velocity faces vax/vbx[i+1], vay/vby[j+1] (s = dt c sigma / 2 of the
  // face), pressure components pax/pbx[i], pay/pby[j] (s = dt c sigma_m / 2).
  const double* vax;
  const double* vbx;
  const double* vay;
  const double* vby;
  const double* pax;
  const double* pbx;
  const double* pay;
  const double* pby;
  // Source elements (ext.elements): count, aperture radius, and per-element
  // amplitude factors and phase offsets (device arrays of elem_n values).
  int elem_n;
  double elem_rap;
  const double* elem_amp;
  const double* elem_phase;
};

// bub_params_t scalars shared by every bubble (inc/bubble_CUDA.h:135-154); the
// per-bubble R0-derived values live in the bubble arrays.
struct BubbleParams {
  double PL0, T0, gam, sig, mu, rho, K0, dt0;
  double inv_rho;  // 1 / rho
  // Smallest |a|^2 whose square root exceeds 0.1 in FP64 / FP32: the series
  // switch of Upsilon and Lp (cabs(a) > 0.1) without a square root on the
  // sub-step's critical path, deciding exactly as the square root would.
  double abs2_cut64;
  float abs2_cut32;
  float rho32, sig32, mu32, gam32, inv_rho32;  // FP32 copies for the mixed path's thermal model
  double pi, pi4r3;
  double dcx, dcy, dcz;  // delta_coef (src/bubble_CUDA.cu:1469-1471)
  long long step_cap;
  double rk_rtol;  // relative tolerance of the rk45 scheme
  int reuse;       // ext.rp_reuse: keep a bubble's last solve of the step while its gathered pressure is unchanged
};

// Default relative tolerance of the rk45 scheme (ext.rp_tol = 0).
constexpr double kRk45DefaultTol = 1.0e-6;

__host__ __device__ __forceinline__ bool src_pressure(const GridParams& g) { return g.plane_p || g.focused_p; }
__host__ __device__ __forceinline__ bool src_velocity(const GridParams& g) { return g.plane_v || g.focused_v; }

// Burst envelope of the [ext] cosine ramp (1 when ramp_time is 0).
__device__ __forceinline__ double burst_ramp(const GridParams& g, double tau) {
  if (!(g.ramp_time > 0.0)) return 1.0;
  const double pi = 3.14159265358979323846;
  double w = 1.0;
  if (tau < g.ramp_time) w = fmin(w, 0.5 * (1.0 - cos(pi * tau / g.ramp_time)));
  double rest = g.on_time - tau;
  if (rest < g.ramp_time) w = fmin(w, rest > 0.0 ? 0.5 * (1.0 - cos(pi * rest / g.ramp_time)) : 0.0);
  return w;
}

// Source element of the cell at x = xm: equal bands of |xm - ctl_x| over the
// aperture radius elem_rap.
__device__ __forceinline__ int element_of(const GridParams& g, double xm) {
  const int e = (int)(fabs(xm - g.ctl_x) * (double)g.elem_n / g.elem_rap);
  return e < g.elem_n ? e : g.elem_n - 1;
}

// Transducer value at (xm, ym), time t.  Plane source then focused source, as
// inc/bubble_CUDA_kernel.cuh:749-787 (velocity) and :889-925 (pressure).  Returns
// false when no source of that kind is configured.  With ext.elements, the
// pressure source's value at a cell of element e is a_e times the reference's,
// with phi_e added to the sine's argument.
__device__ __forceinline__ bool source_value(const GridParams& g, bool pressure, double xm, double ym, double t,
                                             double& out) {
  double amp = pressure ? g.pamp : g.amp;
  double ph = 0.0;
  if (pressure && g.elem_n > 0) {
    const int e = element_of(g, xm);
    amp = g.elem_amp[e] * amp;
    ph = g.elem_phase[e];
  }
  bool set = false;
  if (pressure ? g.plane_p : g.plane_v) {
    double tau = fmod(t, g.period);
    out = (tau <= g.on_time) ? amp * burst_ramp(g, tau) * sin(g.omega * t + ph) : 0.0;
    set = true;
  }
  if (pressure ? g.focused_p : g.focused_v) {
    double s1 = sqrt((g.ctl_x - xm) * (g.ctl_x - xm) + (g.ctl_y - ym) * (g.ctl_y - ym));
    if (s1 <= g.focal_dist) {
      s1 = fmax(t - (g.focal_dist - s1) / g.c_inf, 0.0);
      double s2 = fmod(s1, g.period);
      out = (s2 < g.on_time) ? amp * burst_ramp(g, s2) * sin(g.omega * s2 + ph) : 0.0;
    } else {
      out = 0.0;
    }
    set = true;
  }
  // At t = 0 the pressure source is 0: the reference's p0 array starts at zero
  // and is first written by the pressure evaluation of step 1, so the first
  // velocity update reads no source.  (Its own source is 0 at t = 0 anyway; an
  // element's phase offset would not be.)
  if (pressure && set && !(t > 0.0)) out = 0.0;
  return set;
}

// Derivatives of the pressure source's value at (xm, ym), time t, with respect
// to the amplitude factor (dA) and the phase offset (dP) of the cell's element
// (ext.elements > 0).  The focused source, when set, is the value the source
// takes (source_value applies it last).
__device__ __forceinline__ void source_derivatives(const GridParams& g, double xm, double ym, double t, double& dA,
                                                   double& dP) {
  dA = dP = 0.0;
  if (!(t > 0.0)) return;  // the source is 0 at t = 0 (source_value)
  const int e = element_of(g, xm);
  const double a = g.elem_amp[e], ph = g.elem_phase[e];
  double arg, env;
  if (g.focused_p) {
    double s1 = sqrt((g.ctl_x - xm) * (g.ctl_x - xm) + (g.ctl_y - ym) * (g.ctl_y - ym));
    if (!(s1 <= g.focal_dist)) return;
    s1 = fmax(t - (g.focal_dist - s1) / g.c_inf, 0.0);
    const double s2 = fmod(s1, g.period);
    if (!(s2 < g.on_time)) return;
    env = g.pamp * burst_ramp(g, s2);
    arg = g.omega * s2 + ph;
  } else if (g.plane_p) {
    const double tau = fmod(t, g.period);
    if (!(tau <= g.on_time)) return;
    env = g.pamp * burst_ramp(g, tau);
    arg = g.omega * t + ph;
  } else {
    return;
  }
  dA = env * sin(arg);
  dP = a * env * cos(arg);
}

// Field storage.  FP64 path: one double per value.  Mixed path: an FP32 value
// plus an FP32 compensation term holding its rounding error (value +
// compensation carries about 48 significant bits), stored as one float2;
// arithmetic is done in FP64 registers and each store re-splits the result,
// so no rounding error accumulates step to step.
struct F64 {
  double* p;
  template <typename K>
  __device__ __forceinline__ double get(K k) const {
    return p[k];
  }
  template <typename K>
  __device__ __forceinline__ void put(K k, double v) const {
    p[k] = v;
  }
  // The value get() returns after put(v).
  __device__ static __forceinline__ double stored(double v) { return v; }
  // Asynchronous copy of element k into an 8-byte shared-memory slot, and the
  // value of a slot once the copy has landed.
  template <typename K>
  __device__ __forceinline__ void stage(void* dst, K k) const {
    __pipeline_memcpy_async(dst, p + k, 8);
  }
  __device__ static __forceinline__ double staged(const void* src) { return *(const double*)src; }
};
struct F32c {
  float2* p;  // (value, compensation) pairs, one 8-byte access per element
  template <typename K>
  __device__ __forceinline__ double get(K k) const {
    const float2 v = p[k];
    return (double)v.x + (double)v.y;
  }
  template <typename K>
  __device__ __forceinline__ void put(K k, double v) const {
    const float h = (float)v;
    p[k] = make_float2(h, (float)(v - (double)h));
  }
  __device__ static __forceinline__ double stored(double v) {
    const float h = (float)v;
    return (double)h + (double)(float)(v - (double)h);
  }
  template <typename K>
  __device__ __forceinline__ void stage(void* dst, K k) const {
    __pipeline_memcpy_async(dst, p + k, 8);
  }
  __device__ static __forceinline__ double staged(const void* src) {
    const float2 v = *(const float2*)src;
    return (double)v.x + (double)v.y;
  }
};
// Void-fraction history of the mixed path: FP32 storage (sums are FP64).
struct F32 {
  float* p;
  template <typename K>
  __device__ __forceinline__ double get(K k) const {
    return (double)p[k];
  }
  template <typename K>
  __device__ __forceinline__ void put(K k, double v) const {
    p[k] = (float)v;
  }
  __device__ static __forceinline__ double stored(double v) { return (double)(float)v; }
  template <typename K>
  __device__ __forceinline__ void stage(void* dst, K k) const {
    __pipeline_memcpy_async(dst, p + k, 4);
  }
  __device__ static __forceinline__ double staged(const void* src) { return (double)*(const float*)src; }
};

// Mixture pressure p0 at logical (i, j), i in [0, X+1], j in [0, Y+1], from the
// split components of one pressure buffer, with the boundary values that
// MixtureBoundaryPressureKernel (inc/bubble_CUDA_kernel.cuh:870-952) leaves in
// p0: its y-face section is applied before its x-face section, PML faces keep
// p0 = 0, and the y1 mirror is p0(Y+1) = p0(Y).  t is the time of the pressure
// evaluation that produced the buffer (the source value on the forced row).
template <typename S>
__device__ __forceinline__ double p0_at(const GridParams& g, const S& px, const S& py, int i, int j, double t) {
  const int X = g.f.X, Y = g.f.Y;
  if (i == 0 || i == X + 1) {
    if (i == 0 ? g.pml_x0 : g.pml_x1) return 0.0;
    i = (i == 0) ? 1 : X;
  }
  if (j == 0) {
    if (g.pml_y0) return 0.0;
    double v;
    if (g.source_row == 0 && source_value(g, true, ((double)i - 0.5) * g.dx, -0.5 * g.dy, t, v)) return v;
    j = 1;
  } else if (j == Y + 1) {
    if (g.pml_y1) return 0.0;
    j = Y;
  }
  if (g.source_row > 0 && j == g.source_row) {
    double v;
    if (source_value(g, true, ((double)i - 0.5) * g.dx, ((double)g.source_row - 0.5) * g.dy, t, v)) return v;
  }
  const long k = g.f.idx(i, j);
  return px.get(k) + py.get(k);
}

// ---------------------------------------------------------------------------
// Bubble physics (inc/bubble_CUDA_kernel.cuh:227-340, inc/complex.cuh).  The
// thermal model (alpha_N, Upsilon, omega_N, Lp_N) is a template on the real
// type: FP64 for the FP64 path, FP32 for the mixed path.  The radius update,
// its step-size control and the gas-pressure update stay FP64 in both.
template <typename R>
struct Cx {
  R re, im;
};
// Division in the thermal model: IEEE in FP64, the fast approximate FP32
// division (max 2 ulp) in the mixed path.
__device__ __forceinline__ double xdiv(double a, double b) { return a / b; }
__device__ __forceinline__ float xdiv(float a, float b) { return __fdividef(a, b); }
template <typename R>
__device__ __forceinline__ Cx<R> cmul(Cx<R> a, Cx<R> b) {
  return {a.re * b.re - a.im * b.im, a.im * b.re + a.re * b.im};
}
// Complex quotients with one real division (the reciprocal of |b|^2).
template <typename R>
__device__ __forceinline__ Cx<R> cdiv(Cx<R> a, Cx<R> b) {
  const R ic = xdiv(R(1), b.re * b.re + b.im * b.im);
  return {(a.re * b.re + a.im * b.im) * ic, (a.im * b.re - a.re * b.im) * ic};
}
template <typename R>
__device__ __forceinline__ Cx<R> rdiv(R a, Cx<R> b) {
  const R ic = xdiv(R(1), b.re * b.re + b.im * b.im);
  return {(a * b.re) * ic, (-a * b.im) * ic};
}
template <typename R>
__device__ __forceinline__ Cx<R> cscl(Cx<R> a, R s) {
  return {a.re * s, a.im * s};
}
template <typename R>
__device__ __forceinline__ R cabsx(Cx<R> a) {
  return sqrt(a.re * a.re + a.im * a.im);
}
// cabs(a) > 0.1, decided on |a|^2 (see BubbleParams::abs2_cut64).
template <typename R>
__device__ __forceinline__ bool above_series_cut(Cx<R> a, R cut2) {
  return a.re * a.re + a.im * a.im >= cut2;
}
// coth(a) = N / D for Re a >= 0 (every argument here is (s, s), s >= 0):
// N = 1 + E, D = 1 - E with E = exp(-2a) = exp(-2 re) (cos 2 im - i sin 2 im).
// The reference evaluates coth as (1, tanh(re) tan(im)) / (tanh(re), tan(im))
// (inc/complex.cuh); this form needs one exp and one sincos instead of a tanh
// and a tan (whose range reduction and pole at pi/2 sit on the sub-step's
// critical path), and cannot overflow.  Callers fold the division into their
// own and use N and D only in ratios homogeneous in the pair, so a sub-step
// carries one complex division per Upsilon / Lp evaluation.
template <typename R>
__device__ __forceinline__ void coth_parts(Cx<R> a, Cx<R>& N, Cx<R>& D) {
  const R m = exp(R(-2) * a.re);
  R sn, cs;
  sincos(R(2) * a.im, &sn, &cs);
  const R er = m * cs, ei = -m * sn;
  N = Cx<R>{R(1) + er, ei};
  D = Cx<R>{R(1) - er, -ei};
}
using C64 = Cx<double>;

// Per-bubble constants derived from its R0 (init_bub_params, src/bubble_CUDA.cu:666-670).
struct BubbleR0 {
  double R0, PG0, R03, coeff_alpha, inv_R0, inv_PG0;
  double T0_PG0R03;                      // T0 / (PG0 R0^3) of the heat flux
  float PG0_32, ca32, inv_R0_32;  // FP32 copies for the mixed path's thermal model
};
__device__ __forceinline__ BubbleR0 bubble_r0(const BubbleParams& b, double R0) {
  BubbleR0 r;
  r.R0 = R0;
  r.inv_R0 = 1.0 / R0;
  r.R03 = R0 * R0 * R0;
  r.PG0 = b.PL0 + 2.0 * b.sig / R0;
  r.inv_PG0 = 1.0 / r.PG0;
  r.coeff_alpha = b.gam * r.PG0 * r.R03 / (2.0 * (b.gam - 1.0) * b.T0 * b.K0);
  r.T0_PG0R03 = b.T0 / (r.PG0 * r.R03);
  r.PG0_32 = (float)r.PG0;
  r.ca32 = (float)r.coeff_alpha;
  r.inv_R0_32 = (float)r.inv_R0;
  return r;
}

// Upsilon (:297-307): 3 gam / (1 + 3 (gam - 1) t), t = (a coth(a) - 1) / a^2.
// With coth(a) = N / D and M = a N - D (so a coth(a) - 1 = M / D) this is
// 3 gam D a^2 / (D a^2 + 3 (gam - 1) M): the same quantity with one division.
template <typename R>
__device__ __forceinline__ Cx<R> upsilon(Cx<R> a, R gam, R cut2) {
  Cx<R> aa = cmul(a, a);
  Cx<R> t;
  if (above_series_cut(a, cut2)) {
    Cx<R> N, D;
    coth_parts(a, N, D);
    const Cx<R> aN = cmul(a, N);
    const Cx<R> M{aN.re - D.re, aN.im - D.im};
    const Cx<R> Da = cmul(D, aa);
    const R g3 = R(3) * (gam - R(1));
    return cdiv(cscl(Da, R(3) * gam), Cx<R>{Da.re + g3 * M.re, Da.im + g3 * M.im});
  } else {
    Cx<R> q = cmul(aa, Cx<R>{R(2.0 / 945.0) - xdiv(aa.re, R(4725.0)), xdiv(-aa.im, R(4725.0))});
    Cx<R> m = cmul(aa, Cx<R>{R(-1.0 / 45.0) + q.re, q.im});
    t = Cx<R>{R(1.0 / 3.0) + m.re, m.im};
  }
  Cx<R> d = cscl(cscl(t, gam - R(1)), R(3));
  return rdiv(R(3) * gam, Cx<R>{R(1) + d.re, d.im});
}

// solveLp (:310-323).
template <typename R>
__device__ __forceinline__ Cx<R> lp_n(Cx<R> a, R Rb, R cut2) {
  Cx<R> aa = cmul(a, a);
  Cx<R> c;
  if (above_series_cut(a, cut2)) {
    // (a^2 - 3 c) / (a^2 c) with c = a coth(a) - 1 = M / D:
    // (a^2 D - 3 M) / (a^2 M), one division.
    Cx<R> N, D;
    coth_parts(a, N, D);
    const Cx<R> aN = cmul(a, N);
    const Cx<R> M{aN.re - D.re, aN.im - D.im};
    const Cx<R> Da = cmul(aa, D);
    c = cdiv(Cx<R>{Da.re - R(3) * M.re, Da.im - R(3) * M.im}, cmul(aa, M));
  } else {
    Cx<R> a37 = cscl(aa, R(37));
    Cx<R> q = cmul(aa, Cx<R>{R(2.0 / 7875.0) - xdiv(a37.re, R(3031875.0)), xdiv(-a37.im, R(3031875.0))});
    Cx<R> m = cmul(aa, Cx<R>{R(-1.0 / 175.0) + q.re, q.im});
    c = Cx<R>{R(1.0 / 5.0) + m.re, m.im};
  }
  return cscl(c, Rb);
}

template <typename R>
__device__ __forceinline__ R series_cut(const BubbleParams& b);
template <>
__device__ __forceinline__ double series_cut<double>(const BubbleParams& b) {
  return b.abs2_cut64;
}
template <>
__device__ __forceinline__ float series_cut<float>(const BubbleParams& b) {
  return b.abs2_cut32;
}

// Constants of the thermal model in its real type.
template <typename R>
struct ThermalConst {
  R rho, sig, mu, gam, ca, inv_R0, PG0, cut2, inv_rho;
};
__device__ __forceinline__ ThermalConst<double> thermal_const64(const BubbleParams& b, const BubbleR0& r) {
  return {b.rho, b.sig, b.mu, b.gam, r.coeff_alpha, r.inv_R0, r.PG0, b.abs2_cut64, b.inv_rho};
}
__device__ __forceinline__ ThermalConst<float> thermal_const32(const BubbleParams& b, const BubbleR0& r) {
  return {b.rho32, b.sig32, b.mu32, b.gam32, r.ca32, r.inv_R0_32, r.PG0_32, b.abs2_cut32, b.inv_rho32};
}

// solveOmegaN (:263-288): omega_N and alpha_N for gas pressure PG at radius Rb.
template <typename R>
__device__ __forceinline__ R omega_n(Cx<R>& alpha, R PG, R Rb, const ThermalConst<R>& c) {
  const R eps = R(2.22044604925031308e-016);
  const R rho = c.rho, sig = c.sig, mu = c.mu, gam = c.gam, ca = c.ca;
  // One division for the five quotients by the radius.
  const R inv_Rb = xdiv(R(1), Rb);
  R Rx = Rb * c.inv_R0;
  R coef1 = xdiv(c.PG0, PG * Rx * Rx * Rx);
  R coef2 = PG * rho;
  R coef3 = R(4) * inv_Rb * inv_Rb;
  R value1 = R(-2) * sig * rho * inv_Rb;
  R ups_re = R(3) * gam * coef1;
  R mu_eff = mu;
  R eta = ups_re * coef2 + value1 - mu_eff * mu_eff * coef3;
  // Loop invariants as reciprocals/quotients, so that the iteration's chain is
  // sqrt -> Upsilon (one division) -> sqrt.
  const R inv_rho_Rb = c.inv_rho * inv_Rb;
  const R ca_Rb = ca * inv_Rb;
  R omega = sqrt(fmax(eta, R(1.0e-6) * eps)) * inv_rho_Rb;
  for (int k = 0; k < 3; k++) {
    R s = sqrt(ca_Rb * omega);
    const R pg_4w = xdiv(PG, R(4) * omega);  // independent of Upsilon
    Cx<R> u = cscl(upsilon(Cx<R>{s, s}, gam, c.cut2), coef1);
    mu_eff = mu + u.im * pg_4w;
    eta = u.re * coef2 + value1 - mu_eff * mu_eff * coef3;
    omega = sqrt(fmax(eta, R(1.0e-6) * eps)) * inv_rho_Rb;
  }
  R s = sqrt(ca_Rb * omega);
  alpha = Cx<R>{s, s};
  return omega;
}

// solvePG (:326-340), with the reference's c1, c2, c3 and numerator multiplied
// by den = |Lp|^2, so that Lp = (lpr, lpi) |Lp|^2 enters without a division of
// its own and the gas pressure costs one division on the sub-step's critical
// path.  inv_wdt = 1 / (omega dt), shared with the heat flux of the sub-step.
__device__ __forceinline__ double gas_pressure(double PGn, double Rp, double Rn, double inv_wdt, double dt,
                                               double den, C64 lp, const BubbleParams& b, const BubbleR0& r) {
  double R = 0.5 * (Rp + Rn);
  double Rx = R * r.inv_R0;
  double Rpx = Rp * r.inv_R0;
  double Rnx = Rn * r.inv_R0;
  const double inv_R = 1.0 / R;
  double c0 = dt * 3.0 * (b.gam - 1.0) * b.K0 * b.T0 * inv_R * r.inv_PG0;
  const double g = 1.5 * b.gam * (Rp - Rn) * inv_R;      // c3 without its Lp term
  const double a3 = c0 * lp.re * 0.5 * Rx * Rx * Rx;     // den x (c3 - g)
  const double wn = c0 * lp.im * inv_wdt;                 // den x w
  const double c1 = den * (1.0 + g) + a3 - wn * Rpx * Rpx * Rpx;
  const double c2 = den * (1.0 - g) - a3 - wn * Rnx * Rnx * Rnx;
  return (c2 * PGn + c0 * lp.re * r.PG0) / c1;
}

// solveRayleighPlesset (:227-260): one variable sub-step of the three-level scheme.
__device__ __forceinline__ void rp_substep(double& Rt, double& Rp, double& Rn, double& d1R, double PG, double PL,
                                           double& dt, double& remain, const BubbleParams& b) {
  const double eps = 2.22044604925031308e-016;
  double Rm = Rn;
  Rn = Rp;
  const double inv_Rn = 1.0 / Rn;
  double acc = (PG - PL - 2.0 * b.sig * inv_Rn - 4.0 * b.mu * inv_Rn * d1R) * b.inv_rho - 1.5 * d1R * d1R;
  double dtm = dt;
  double dtp = fmin(1.01 * dt, b.dt0);
  // The velocity and acceleration limits, 0.01 Rn / |d1R| and 0.1 Rn / sqrt(|acc|)
  // (:238-241): each quotient is formed only where it is the smaller step, decided
  // on the products (the squares for the second), so a quiet sub-step divides
  // by neither.
  const double ad = fabs(d1R), aa = fabs(acc);
  if (ad > eps && 0.01 * Rn < dtp * ad) dtp = fmin(dtp, 0.01 * Rn / ad);
  if (aa > eps) {
    const double lim = 0.1 * Rn;
    if (lim * lim < dtp * dtp * aa) dtp = fmin(dtp, lim / sqrt(aa));
  }
  double q = dtp / dtm;
  Rt = Rp = (1.0 + q) * Rn - q * Rm + (dtp * inv_Rn) * (0.5 * (dtp + dtm) * acc);
  d1R = (dtm * dtm * Rp + (-dtm * dtm + dtp * dtp) * Rn - dtp * dtp * Rm) / (dtm * dtp * (dtm + dtp)) +
        (dtp * inv_Rn) * acc;
  dt = dtp;
  if (dtp >= remain) {
    dtp = remain;
    double qr = dtp / dtm;
    Rt = (1.0 + qr) * Rn - qr * Rm + (dtp * inv_Rn) * (0.5 * (dtp + dtm) * acc);
  }
  remain -= dtp;
}

// Smooth delta (inc/bubble_CUDA_kernel.cuh:214-222), band 2 (the only band
// this path implements): delta(pos) = dcx (1 + cos(dcy ((pos - 1/2) dx - x))).
// Adjacent points' arguments differ by dcy dx = pi, so the cosines of a
// stencil's points alternate in sign: with c0 the cosine at one point p0,
// delta(p0 + k) = dcx (1 + c0) for even k and dcx (1 - c0) for odd k.  Each
// bubble then needs one cosine per axis instead of one per point (the values
// move by a rounding at most).
__device__ __forceinline__ double delta_cos_x(const BubbleParams& b, const GridParams& g, int pos, double bx) {
  return cos(b.dcy * (((double)pos - 0.5) * g.dx - bx));
}
__device__ __forceinline__ double delta_cos_y(const BubbleParams& b, const GridParams& g, int pos, double by) {
  return cos(b.dcz * (((double)pos - 0.5) * g.dy - by));
}
// Weight of the point p0 + k, from c0 = delta_cos_* at p0 (any integer k).
__device__ __forceinline__ double delta_w(const BubbleParams& b, double c0, int k) {
  return b.dcx * (1.0 + ((k & 1) ? -c0 : c0));
}

}  // namespace crp
