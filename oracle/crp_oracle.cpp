// CPU oracle for the CUDA-RP simulation path — TEST INFRASTRUCTURE ONLY.
//
// FP64 restatement of the reference's simulated path.  Each function names the
// reference lines it follows; the arithmetic is kept in the reference's
// operation order so the host results agree bit-for-bit with the reference's
// own host-compiled functions (checked by tests/test_oracle_pin.py).  Where the
// reference has data races (the boundary kernels, the atomic void-fraction
// scatter) this restatement fixes one order and says which.
//
// Only the tests, __graft_entry__.smoke() and bench.py's CPU baseline load it.
#include "crp_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// -------------------------------------------------------------------------
// Complex arithmetic with the operation order of inc/complex.cuh:1-90.
struct Cplx {
  double re, im;
};
inline Cplx cmul(Cplx a, Cplx b) { return {a.re * b.re - a.im * b.im, a.im * b.re + a.re * b.im}; }
inline Cplx cdiv(Cplx a, Cplx b) {
  double c = (b.re * b.re + b.im * b.im);
  return {(a.re * b.re + a.im * b.im) / c, (a.im * b.re - a.re * b.im) / c};
}
inline Cplx rdivc(double a, Cplx b) {
  double c = (b.re * b.re + b.im * b.im);
  return {a * b.re / c, -a * b.im / c};
}
inline Cplx cscale(Cplx a, double b) { return {a.re * b, a.im * b}; }
inline Cplx caddr(double a, Cplx b) { return {a + b.re, b.im}; }
inline Cplx csubr(Cplx a, double b) { return {a.re - b, a.im}; }
inline Cplx rsubc(double a, Cplx b) { return {a - b.re, -b.im}; }
inline Cplx csub(Cplx a, Cplx b) { return {a.re - b.re, a.im - b.im}; }
inline Cplx cdivr(Cplx a, double b) { return {a.re / b, a.im / b}; }
inline double cabs_(Cplx a) { return std::sqrt(a.re * a.re + a.im * a.im); }
inline Cplx ccoth(Cplx a) {
  double x = std::tanh(a.re), y = std::tan(a.im);
  return cdiv(Cplx{1.0, x * y}, Cplx{x, y});
}

// epsilon() of inc/bubble_CUDA_kernel.cuh:145-149 (a constant).
constexpr double kEps = 2.22044604925031308e-016;

// Per-bubble constants: bub_params_t fields the physics reads
// (inc/bubble_CUDA.h:135-154).  R0/PG0/R03/coeff_alpha are per bubble here so a
// seeded R0 distribution can be used; with one R0 they equal the reference's.
struct BubConst {
  double R0, PG0, PL0, T0, gam, sig, mu, rho, K0, dt0, R03, coeff_alpha;
};

BubConst make_bubconst(double R0, double PL0, double T0, double gam, double sig, double mu, double rho,
                       double K0, double dt0) {
  // init_bub_params, src/bubble_CUDA.cu:666-670.
  BubConst b;
  b.R0 = R0;
  b.PL0 = PL0;
  b.T0 = T0;
  b.gam = gam;
  b.sig = sig;
  b.mu = mu;
  b.rho = rho;
  b.K0 = K0;
  b.dt0 = dt0;
  b.R03 = R0 * R0 * R0;
  b.PG0 = PL0 + 2.0 * sig / R0;
  b.coeff_alpha = gam * b.PG0 * b.R03 / (2.0 * (gam - 1.0) * T0 * K0);
  return b;
}

// solveRayleighPlesset, inc/bubble_CUDA_kernel.cuh:227-260.
void rp_substep(double& Rt, double& Rp, double& Rn, double& d1R, double PG, double PL, double& dt,
                double& remain, const BubConst& b) {
  double Rm = Rn;
  Rn = Rp;
  double acc = (PG - PL - 2.0 * b.sig / Rn - 4.0 * b.mu / Rn * d1R) / b.rho - 1.5 * d1R * d1R;
  double dtm = dt;
  double dtp = std::min(1.01 * dt, b.dt0);
  if (std::fabs(d1R) > kEps) dtp = std::min(dtp, 0.01 * Rn / std::fabs(d1R));
  if (std::fabs(acc) > kEps) dtp = std::min(dtp, 0.1 * Rn / std::sqrt(std::fabs(acc)));
  Rt = Rp = (1.0 + dtp / dtm) * Rn - dtp / dtm * Rm + (dtp / Rn) * (0.5 * (dtp + dtm) * acc);
  d1R = (dtm * dtm * Rp + (-dtm * dtm + dtp * dtp) * Rn - dtp * dtp * Rm) / (dtm * dtp * (dtm + dtp)) +
        (dtp / Rn) * acc;
  dt = dtp;
  if (dtp >= remain) {
    dtp = remain;
    Rt = (1.0 + dtp / dtm) * Rn - dtp / dtm * Rm + (dtp / Rn) * (0.5 * (dtp + dtm) * acc);
  }
  remain -= dtp;
}

// Alpha, inc/bubble_CUDA_kernel.cuh:291-294.
inline Cplx thermal_alpha(double R, double omega, double ca) {
  double s = std::sqrt(ca / R * omega);
  return Cplx{1.0 * s, 1.0 * s};
}

// Upsilon, inc/bubble_CUDA_kernel.cuh:297-307.
Cplx thermal_upsilon(Cplx a, double gam) {
  Cplx aa = cmul(a, a);
  if (cabs_(a) > 1.0e-1) {
    Cplx t = cdiv(csubr(cmul(a, ccoth(a)), 1.0), aa);
    return rdivc(3.0 * gam, caddr(1.0, cscale(cscale(t, gam - 1.0), 3.0)));
  }
  Cplx inner = rsubc(2.0 / 945.0, cdivr(aa, 4725.0));
  Cplx mid = caddr(-1.0 / 45.0, cmul(aa, inner));
  Cplx ser = caddr(1.0 / 3.0, cmul(aa, mid));
  return rdivc(3.0 * gam, caddr(1.0, cscale(cscale(ser, gam - 1.0), 3.0)));
}

// solveLp, inc/bubble_CUDA_kernel.cuh:310-323.
Cplx thermal_lp(Cplx a, double R) {
  Cplx aa = cmul(a, a);
  Cplx c;
  if (cabs_(a) > 1.0e-1) {
    c = csubr(cmul(a, ccoth(a)), 1.0);
    c = cdiv(csub(aa, cscale(c, 3.0)), cmul(aa, c));
  } else {
    Cplx inner = rsubc(2.0 / 7875.0, cdivr(cscale(aa, 37.0), 3031875.0));
    Cplx mid = caddr(-1.0 / 175.0, cmul(aa, inner));
    c = caddr(1.0 / 5.0, cmul(aa, mid));
  }
  return cscale(c, R);
}

// solveOmegaN, inc/bubble_CUDA_kernel.cuh:263-288.
double thermal_omega(Cplx& alpha, double PG, double R, const BubConst& b) {
  double Rx = R / b.R0;
  double coef1 = b.PG0 / (PG * Rx * Rx * Rx);
  double coef2 = PG * b.rho;
  double coef3 = 4.0 / (R * R);
  double value1 = -2.0 * b.sig * b.rho / R;
  Cplx ups = Cplx{3.0 * b.gam * coef1, 0.0 * coef1};
  double mu_eff = b.mu;
  double eta = ups.re * coef2 + value1 - mu_eff * mu_eff * coef3;
  double omega = std::sqrt(std::max(eta, 1.0e-6 * kEps)) / (b.rho * R);
  for (int k = 0; k < 3; k++) {
    alpha = thermal_alpha(R, omega, b.coeff_alpha);
    ups = cscale(thermal_upsilon(alpha, b.gam), coef1);
    mu_eff = b.mu + ups.im * PG / (4.0 * (omega));
    eta = ups.re * coef2 + value1 - mu_eff * mu_eff * coef3;
    omega = std::sqrt(std::max(eta, 1.0e-6 * kEps)) / (b.rho * R);
  }
  alpha = thermal_alpha(R, omega, b.coeff_alpha);
  return omega;
}

// solvePG, inc/bubble_CUDA_kernel.cuh:326-340.
double gas_pressure(double PGn, double Rp, double Rn, double omega, double dt, Cplx lp, const BubConst& b) {
  double R = 0.5 * (Rp + Rn);
  double Rx = R / b.R0;
  double Rpx = Rp / b.R0;
  double Rnx = Rn / b.R0;
  double lpr = lp.re / (lp.re * lp.re + lp.im * lp.im);
  double lpi = lp.im / (lp.re * lp.re + lp.im * lp.im);
  double c0 = dt * 3.0 * (b.gam - 1.0) * b.K0 * b.T0 / (R * b.PG0);
  double c3 = 1.5 * b.gam * (Rp - Rn) / R + c0 * lpr * 0.5 * Rx * Rx * Rx;
  double c1 = 1.0 + c3 - c0 * lpi / (omega * dt) * Rpx * Rpx * Rpx;
  double c2 = 1.0 - c3 - c0 * lpi / (omega * dt) * Rnx * Rnx * Rnx;
  return (c2 * PGn + c0 * lpr * b.PG0) / c1;
}

// The reference's sub-step with its step limits scaled down by `refine`
// (dt0 / refine, 0.01 / refine radius change, 0.1 / refine of R / sqrt|R''|):
// refine = 1 is rp_substep.  Used only to converge the reference scheme in the
// single-bubble comparison with the rk45 scheme.
void rp_substep_refined(double& Rt, double& Rp, double& Rn, double& d1R, double PG, double PL, double& dt,
                        double& remain, const BubConst& b, double refine) {
  double Rm = Rn;
  Rn = Rp;
  double acc = (PG - PL - 2.0 * b.sig / Rn - 4.0 * b.mu / Rn * d1R) / b.rho - 1.5 * d1R * d1R;
  double dtm = dt;
  double dtp = std::min(1.01 * dt, b.dt0 / refine);
  if (std::fabs(d1R) > kEps) dtp = std::min(dtp, 0.01 / refine * Rn / std::fabs(d1R));
  if (std::fabs(acc) > kEps) dtp = std::min(dtp, 0.1 / refine * Rn / std::sqrt(std::fabs(acc)));
  Rt = Rp = (1.0 + dtp / dtm) * Rn - dtp / dtm * Rm + (dtp / Rn) * (0.5 * (dtp + dtm) * acc);
  d1R = (dtm * dtm * Rp + (-dtm * dtm + dtp * dtp) * Rn - dtp * dtp * Rm) / (dtm * dtp * (dtm + dtp)) +
        (dtp / Rn) * acc;
  dt = dtp;
  if (dtp >= remain) {
    dtp = remain;
    Rt = (1.0 + dtp / dtm) * Rn - dtp / dtm * Rm + (dtp / Rn) * (0.5 * (dtp + dtm) * acc);
  }
  remain -= dtp;
}

// ext.rp_scheme = rk45: the same bubble model as a continuous system in
// (R, R', PG), integrated by the Dormand-Prince 5(4) pair (Dormand & Prince
// 1980) with embedded error control; the restatement of the CUDA path's
// scheme (its model and controller are documented in cuda-rp_b200/csrc/rk45.cuh).
// PG' is the dt -> 0 limit of solvePG (inc/bubble_CUDA_kernel.cuh:326-340),
// omega and Lp are the reference's thermal model (solveOmegaN, solveLp).
struct RkD {
  double R, V, PG, q;
};

struct RkBubble {
  const BubConst* k;
  double K;              // 3 (gam - 1) K0 T0 / PG0
  double PC0, PC1, PC2;  // liquid pressure PC2 t^2 + PC1 t + PC0, t from the step's start
  double pi;
  RkD rhs(double t, double R, double V, double PG) const {
    const BubConst& b = *k;
    const double PL = PC2 * t * t + PC1 * t + PC0;
    RkD d;
    d.R = V;
    d.V = ((PG - PL - 2.0 * b.sig / R - 4.0 * b.mu / R * V) / b.rho - 1.5 * V * V) / R;
    Cplx alpha;
    const double omega = thermal_omega(alpha, PG, R, b);
    const Cplx lp = thermal_lp(alpha, R);
    const double den = lp.re * lp.re + lp.im * lp.im;
    const double Lr = lp.re / den, Liw = lp.im / den / omega;
    const double x = R / b.R0;
    const double x3 = x * x * x;
    const double KR = K / R;
    const double num = -3.0 * b.gam * PG * V / R + KR * (Lr * (b.PG0 - x3 * PG) + Liw * 3.0 * x * x * V / b.R0 * PG);
    d.PG = num / (1.0 - KR * Liw * x3);
    const double R3 = R * R * R;
    const double dTdr = b.T0 / (b.PG0 * b.R03) * (Lr * (b.PG0 * b.R03 - PG * R3) + Liw * (R3 * d.PG + 3.0 * R * R * V * PG));
    d.q = -4.0 * pi * R * R * b.K0 * dTdr + 16.0 * pi * b.mu * R * V * V;
    return d;
  }
};

struct RkRun {
  double R, V, PG, h, t, tend, Q;
  int64_t count;
};

// Integrates over [t, tend]; false when the step cap is reached or the step
// size collapses.
bool rk45_run(const RkBubble& m, RkRun& s, double rtol, int64_t cap) {
  const double c2 = 1.0 / 5.0, c3 = 3.0 / 10.0, c4 = 4.0 / 5.0, c5 = 8.0 / 9.0;
  const double a21 = 1.0 / 5.0;
  const double a31 = 3.0 / 40.0, a32 = 9.0 / 40.0;
  const double a41 = 44.0 / 45.0, a42 = -56.0 / 15.0, a43 = 32.0 / 9.0;
  const double a51 = 19372.0 / 6561.0, a52 = -25360.0 / 2187.0, a53 = 64448.0 / 6561.0, a54 = -212.0 / 729.0;
  const double a61 = 9017.0 / 3168.0, a62 = -355.0 / 33.0, a63 = 46732.0 / 5247.0, a64 = 49.0 / 176.0,
               a65 = -5103.0 / 18656.0;
  const double b1 = 35.0 / 384.0, b3 = 500.0 / 1113.0, b4 = 125.0 / 192.0, b5 = -2187.0 / 6784.0, b6 = 11.0 / 84.0;
  const double e1 = 71.0 / 57600.0, e3 = -71.0 / 16695.0, e4 = 71.0 / 1920.0, e5 = -17253.0 / 339200.0,
               e6 = 22.0 / 525.0, e7 = -1.0 / 40.0;
  RkD k1 = m.rhs(s.t, s.R, s.V, s.PG);
  while (s.t < s.tend) {
    if (s.count >= cap) return false;
    const double rem = s.tend - s.t;
    double h = s.h;
    bool last = false;
    if (h >= rem || 1.01 * h >= rem) {
      h = rem;
      last = true;
    }
    s.count++;
    const double t = s.t;
    const RkD k2 = m.rhs(t + c2 * h, s.R + h * (a21 * k1.R), s.V + h * (a21 * k1.V), s.PG + h * (a21 * k1.PG));
    const RkD k3 = m.rhs(t + c3 * h, s.R + h * (a31 * k1.R + a32 * k2.R), s.V + h * (a31 * k1.V + a32 * k2.V),
                         s.PG + h * (a31 * k1.PG + a32 * k2.PG));
    const RkD k4 = m.rhs(t + c4 * h, s.R + h * (a41 * k1.R + a42 * k2.R + a43 * k3.R),
                         s.V + h * (a41 * k1.V + a42 * k2.V + a43 * k3.V),
                         s.PG + h * (a41 * k1.PG + a42 * k2.PG + a43 * k3.PG));
    const RkD k5 = m.rhs(t + c5 * h, s.R + h * (a51 * k1.R + a52 * k2.R + a53 * k3.R + a54 * k4.R),
                         s.V + h * (a51 * k1.V + a52 * k2.V + a53 * k3.V + a54 * k4.V),
                         s.PG + h * (a51 * k1.PG + a52 * k2.PG + a53 * k3.PG + a54 * k4.PG));
    const RkD k6 = m.rhs(t + h, s.R + h * (a61 * k1.R + a62 * k2.R + a63 * k3.R + a64 * k4.R + a65 * k5.R),
                         s.V + h * (a61 * k1.V + a62 * k2.V + a63 * k3.V + a64 * k4.V + a65 * k5.V),
                         s.PG + h * (a61 * k1.PG + a62 * k2.PG + a63 * k3.PG + a64 * k4.PG + a65 * k5.PG));
    const double Rn = s.R + h * (b1 * k1.R + b3 * k3.R + b4 * k4.R + b5 * k5.R + b6 * k6.R);
    const double Vn = s.V + h * (b1 * k1.V + b3 * k3.V + b4 * k4.V + b5 * k5.V + b6 * k6.V);
    const double PGn = s.PG + h * (b1 * k1.PG + b3 * k3.PG + b4 * k4.PG + b5 * k5.PG + b6 * k6.PG);
    const bool finite = Rn > 0.0 && PGn > 0.0 && std::isfinite(Rn) && std::isfinite(Vn) && std::isfinite(PGn);
    RkD k7{0.0, 0.0, 0.0, 0.0};
    double err = 1.0e30;
    if (finite) {
      k7 = m.rhs(t + h, Rn, Vn, PGn);
      const double eR = h * (e1 * k1.R + e3 * k3.R + e4 * k4.R + e5 * k5.R + e6 * k6.R + e7 * k7.R);
      const double eV = h * (e1 * k1.V + e3 * k3.V + e4 * k4.V + e5 * k5.V + e6 * k6.V + e7 * k7.V);
      const double eP = h * (e1 * k1.PG + e3 * k3.PG + e4 * k4.PG + e5 * k5.PG + e6 * k6.PG + e7 * k7.PG);
      const double sR = rtol * std::max(std::fabs(s.R), std::fabs(Rn));
      const double sV = rtol * (std::max(std::fabs(s.V), std::fabs(Vn)) + 1.0);
      const double sP = rtol * std::max(std::fabs(s.PG), std::fabs(PGn));
      err = std::max(std::fabs(eR) / sR, std::max(std::fabs(eV) / sV, std::fabs(eP) / sP));
      if (!std::isfinite(err)) err = 1.0e30;
    }
    double fac = err > 0.0 ? 0.9 * std::pow(err, -0.2) : 5.0;
    if (err <= 1.0) {
      s.Q += h * (b1 * k1.q + b3 * k3.q + b4 * k4.q + b5 * k5.q + b6 * k6.q);
      s.R = Rn;
      s.V = Vn;
      s.PG = PGn;
      k1 = k7;
      s.t = last ? s.tend : t + h;
      fac = std::min(5.0, std::max(0.2, fac));
      s.h = last ? std::max(s.h, h * fac) : h * fac;
    } else {
      s.h = h * std::min(1.0, std::max(0.2, fac));
    }
    if (!(s.h > 1.0e-22)) return false;
  }
  return true;
}

// -------------------------------------------------------------------------
// array_index_t and init_array, inc/bubble_CUDA.h:59-69, src/bubble_CUDA.cu:561-597.
struct Index {
  int ms, me, ns, ne;
  int istam, iendm, istan, iendn, ista1m, iend1m, ista1n, iend1n, ista2m, iend2m, ista2n, iend2n;
  int jstam, jendm, jstan, jendn, jsta1m, jend1m, jsta1n, jend1n, jsta2m, jend2m, jsta2n, jend2n;
};

Index make_index(int X, int Y, int order) {
  Index a;
  a.ms = -order / 2 + 1;
  a.me = order + a.ms - 1;
  a.ns = -order / 2;
  a.ne = order + a.ns - 1;
  a.istam = 1;
  a.iendm = X;
  a.istan = a.istam - 1;
  a.iendn = a.iendm;
  a.ista1m = a.istan + a.ms;
  a.iend1m = a.iendn + a.me;
  a.ista1n = a.istam + a.ns;
  a.iend1n = a.iendm + a.ne;
  a.ista2m = a.ista1n + a.ms;
  a.iend2m = a.iend1n + a.me;
  a.ista2n = a.ista1m + a.ns;
  a.iend2n = a.iend1m + a.ne;
  a.jstam = 1;
  a.jendm = Y;
  a.jstan = a.jstam - 1;
  a.jendn = a.jendm;
  a.jsta1m = a.jstan + a.ms;
  a.jend1m = a.jendn + a.me;
  a.jsta1n = a.jstam + a.ns;
  a.jend1n = a.jendm + a.ne;
  a.jsta2m = a.jsta1n + a.ms;
  a.jend2m = a.jend1n + a.me;
  a.jsta2n = a.jsta1m + a.ns;
  a.jend2n = a.jend1m + a.ne;
  return a;
}

// A dense 2-D array addressed by the reference's logical (i, j).
struct Field {
  int i0 = 0, j0 = 0, w = 0, h = 0;
  std::vector<double> v;
  void init(int ista, int iend, int jsta, int jend, double fill) {
    i0 = ista;
    j0 = jsta;
    w = iend - ista + 1;
    h = jend - jsta + 1;
    v.assign((size_t)w * h, fill);
  }
  double& at(int i, int j) { return v[(size_t)(j - j0) * w + (i - i0)]; }
  double at(int i, int j) const { return v[(size_t)(j - j0) * w + (i - i0)]; }
  bool in(int i, int j) const { return i >= i0 && i < i0 + w && j >= j0 && j < j0 + h; }
};

// Water properties, inc/bubble_CUDA_kernel.cuh:176-193 (float literals as written there).
double conductivity_water(double T) { return 0.76760 + ((double)7.5390e-3f * T) - (double)9.8250e-6f * (T * T); }
double heat_capacity_water(double T) {
  const double H2O = (double)18.0e-3f;
  return (917.5 - (double)10.1016f * T + (double)0.0454134f * (T * T) - 9.07517e-5 * (T * T * T) +
          (double)6.80700e-8f * (T * T * T * T)) /
         H2O;
}

struct Derived {
  double dx, dy, rdx, rdy;
  double fpx, fpy, omega, dt;
  double ctlx, ctly;        // focal_point_c, the focus the source kernels use
  double rho_inf, cs_inf, P_inf, T_inf;
  double focal_dist;
  double dc_x, dc_y, dc_z;  // delta_coef, src/bubble_CUDA.cu:1469-1471
  double pi, pi4r3;         // Pi_h, Pi4r3_h, src/bubble_CUDA.cu:13-14
  double bub_dt0;
  int mbs, mbe, nbs, nbe;   // src/bubble_CUDA.cu:672-675
};

Derived derive(const crp_config& c) {
  Derived d;
  // init_grid_size, src/bubble_CUDA.cu:524-540.
  d.dx = (double)c.grid_lx / (double)c.grid_x;
  d.dy = (double)c.grid_ly / (double)c.grid_y;
  d.rdx = (double)1.0 / (double)d.dx;
  d.rdy = (double)1.0 / (double)d.dy;
  // init_transducer, src/bubble_CUDA.cu:543-558.
  if (c.tr_focal_dist) {
    d.fpx = 0.0;
    d.fpy = c.tr_focal_dist * 0.5 * std::sqrt(3.0);
  } else {
    d.fpx = 0.0;
    d.fpy = c.grid_ly * 0.5;
  }
  d.omega = 2.0 * std::acos(-1.0) * c.tr_freq;
  // init_mix, src/bubble_CUDA.cu:636-646 (rho_inf and cs_inf from the [ext] keys).
  d.T_inf = 293.15;
  d.P_inf = c.ext_p_inf;
  d.rho_inf = c.ext_rho_inf;
  d.cs_inf = c.ext_c_inf;
  // mix_set_time_increment, src/bubble_CUDA.cu:649-658.
  d.dt = c.sim_cfl * std::min(d.dx, d.dy) / d.cs_inf;
  // Focal point handed to the kernels without a PID update, src/bubble_CUDA.cu:132-153, 214-215.
  d.ctlx = d.fpx;
  d.ctly = d.fpy;
  if (c.tr_pid && c.tr_init_control) d.ctlx = 0.0, d.ctly = c.tr_init_control;
  d.focal_dist = d.ctly / 0.5 / std::sqrt(3.0);
  d.dc_x = 1.0 / ((double)c.sim_smooth_delta_band);
  d.dc_y = 2.0 * std::acos(-1.0) / ((double)c.sim_smooth_delta_band) * d.rdx;
  d.dc_z = 2.0 * std::acos(-1.0) / ((double)c.sim_smooth_delta_band) * d.rdy;
  d.pi = std::acos(-1.0);
  d.pi4r3 = d.pi * 4.0 / 3.0;
  d.bub_dt0 = 0.1 * d.dt;
  d.mbs = -c.sim_smooth_delta_band / 2 + 1;
  d.mbe = c.sim_smooth_delta_band + d.mbs - 1;
  d.nbs = -c.sim_smooth_delta_band / 2;
  d.nbe = c.sim_smooth_delta_band + d.nbs - 1;
  return d;
}

// init_sigma, src/bubble_CUDA.cu:946-1205.
void make_sigma(const crp_config& c, const Index& a, const Derived& d, std::vector<double>& mx,
                std::vector<double>& my, std::vector<double>& nx, std::vector<double>& ny) {
  mx.assign(a.iend1m - a.ista1m + 1, 0.0);
  my.assign(a.jend1m - a.jsta1m + 1, 0.0);
  nx.assign(a.iend2n - a.ista2n + 1, 0.0);
  ny.assign(a.jend2n - a.jsta2n + 1, 0.0);
  const int npml = c.pml_grid_number;
  const double sig = c.pml_sigma;
  const double order = c.pml_order;
  const int X = c.grid_x, Y = c.grid_y;
  auto smax = [&](double h) { return -std::log(sig) * 0.5 * ((double)order + 1.0) / (h * (double)npml); };
  if (c.pml_x0 && a.istam <= npml) {
    double s = smax(d.dx);
    for (int i = std::max(a.istam, a.ms); i <= std::min(a.iendm, npml); i++)
      mx[i - a.ista1m] = s * std::pow(((double)(npml - i + 1) - 0.5) / ((double)npml), order);
  }
  if (c.pml_x1 && X - npml + 1 <= a.iendm) {
    double s = smax(d.dx);
    for (int i = std::max(a.istam, X - npml + 1); i <= std::min(a.iendm, X + a.me); i++)
      mx[i - a.ista1m] = s * std::pow(((double)(i - X + npml) - 0.5) / ((double)npml), order);
  }
  if (c.pml_y0 && a.jstam <= npml) {
    double s = smax(d.dy);
    for (int j = std::max(a.jstam, a.ms); j <= std::min(a.jendm, npml); j++)
      my[j - a.jsta1m] = s * std::pow(((double)(npml - j + 1) - 0.5) / ((double)npml), order);
  }
  if (c.pml_y1 && Y - npml + 1 <= a.jendm) {
    double s = smax(d.dy);
    for (int j = std::max(a.jstam, Y - npml + 1); j <= std::min(a.jendm, Y + a.me); j++)
      my[j - a.jsta1m] = s * std::pow(((double)(j - Y + npml) - 0.5) / ((double)npml), order);
  }
  if (c.pml_x0 && a.istan <= npml - 1) {
    double s = smax(d.dx);
    for (int i = std::max(a.istan, a.ms + a.ns); i <= std::min(a.iendn, npml - 1); i++)
      nx[i - a.ista2n] = s * std::pow(((double)(npml - i)) / ((double)npml), order);
  }
  if (c.pml_x1 && X - npml + 1 <= a.iendn) {
    double s = smax(d.dx);
    for (int i = std::max(a.istan, X - npml + 1); i <= std::min(a.iendn, X + a.me + a.ne + 1); i++)
      nx[i - a.ista2n] = s * std::pow(((double)(i - X + npml)) / ((double)npml), order);
  }
  if (c.pml_y0 && a.jstan <= npml - 1) {
    double s = smax(d.dy);
    for (int j = std::max(a.jstan, a.ms + a.ns); j <= std::min(a.jendn, npml - 1); j++)
      ny[j - a.jsta2n] = s * std::pow(((double)(npml - j)) / ((double)npml), order);
  }
  if (c.pml_y1 && Y - npml + 1 <= a.jendn) {
    double s = smax(d.dy);
    for (int j = std::max(a.jstan, Y - npml + 1); j <= std::min(a.jendn, Y + a.me + a.ne + 1); j++)
      ny[j - a.jsta2n] = s * std::pow(((double)(j - Y + npml)) / ((double)npml), order);
  }
}

// Burst envelope of the [ext] cosine ramp; 1 when ext_ramp_cycles is 0.
double ramp(const crp_config& c, double tau) {
  if (!(c.ext_ramp_cycles > 0.0)) return 1.0;
  const double pi = std::acos(-1.0);
  double tr = c.ext_ramp_cycles / c.tr_freq;
  double ton = (double)c.tr_on_wave / c.tr_freq;
  double w = 1.0;
  if (tau < tr) w = std::min(w, 0.5 * (1.0 - std::cos(pi * tau / tr)));
  double rest = ton - tau;
  if (rest < tr) w = std::min(w, rest > 0.0 ? 0.5 * (1.0 - std::cos(pi * rest / tr)) : 0.0);
  return w;
}

int g_threads = 0;

}  // namespace

// -------------------------------------------------------------------------
struct crpo_sim {
  crp_config cfg;
  Index a;
  Derived d;
  int X, Y;
  bool cyl, bubbles_on;
  std::vector<double> mx, my, nx, ny, xu, rxp;
  Field p0, px, py, pnx, pny, vx, vy, fg, fgn, fgm, rho_m, work;
  // Temperature branch (debug.T): T and k_m on the 2m window, C_pm on the 1m
  // window, the energy fluxes Ex / Ey, and the reference's Work array.
  bool temperature_on = false;
  Field T, k_m, C_pm, Ex, Ey, twork;
  // Focal tracker and PID (src/bubble_CUDA.cu:123-153, 310-352): tracked and
  // controlled focal depths, Butterworth state, PID accumulators.
  std::vector<double> focal_hist, control_hist;
  double filt_in[5] = {0, 0, 0, 0, 0}, filt_out[5] = {0, 0, 0, 0, 0};
  double pid_cum_y = 0.0, pid_der_y = 0.0;
  // Bubble state, bubble_t (inc/bubble_CUDA.h:172-189), structure of arrays.
  int nb = 0;
  std::vector<BubConst> bc;
  std::vector<double> x, y, R_t, R_p, R_pn, R_n, R_nn, d1_R_p, d1_R_n, PG_p, PG_n, PL_p, PL_n, PL_m, Q_B,
      n_B, dtb, dt_n, re, re_n, vbx, vby;
  std::vector<int> ibmx, ibmy, ibnx, ibny, nsub;
  double tstep = 0.0, tstepx = 0.0;
  int64_t nstep = 0;
  crp_stats stats{};
  int source_row;  // row carrying the source (0: reference ghost row)
  // Source elements (ext.elements, an extension without a reference
  // counterpart): count, aperture radius, amplitude factors, phase offsets.
  int elem_n = 0;
  double elem_rap = 0.0;
  std::vector<double> elem_amp, elem_phase;

  // ---- helpers ----
  double delta_x(int pos, double bx) const {
    return d.dc_x * (1.0 + std::cos(d.dc_y * (((double)pos - 0.5) * d.dx - bx)));
  }
  double delta_y(int pos, double by) const {
    return d.dc_x * (1.0 + std::cos(d.dc_z * (((double)pos - 0.5) * d.dy - by)));
  }
  bool src_pressure() const { return cfg.tr_plane_p || cfg.tr_focused_p; }
  bool src_velocity() const { return cfg.tr_plane_v || cfg.tr_focused_v; }

  // Source value at x = xm, y = ym, time t; amplitude amp_scale * amp.
  // Plane source: inc/bubble_CUDA_kernel.cuh:749-762 / 889-902; focused: :763-787 / :903-925.
  // Returns false when neither source of this kind is active (value unchanged).
  // With ext.elements, a pressure source cell of element e (equal bands of
  // |xm - ctl_x| over the aperture radius) takes a_e times the value, with
  // phi_e added to the sine's argument.
  bool source_value(bool pressure, double xm, double ym, double t, double& out) const {
    const crp_config& c = cfg;
    double period = ((double)c.tr_on_wave + (double)c.tr_off_wave) / c.tr_freq;
    double amp = pressure ? d.rho_inf * d.cs_inf * c.tr_amp : c.tr_amp;
    double ph = 0.0;
    if (pressure && elem_n > 0) {
      int e = (int)(std::fabs(xm - d.ctlx) * (double)elem_n / elem_rap);
      if (e >= elem_n) e = elem_n - 1;
      amp = elem_amp[e] * amp;
      ph = elem_phase[e];
    }
    bool set = false;
    if (pressure ? c.tr_plane_p : c.tr_plane_v) {
      double tau = std::fmod(t, period);
      if (tau <= ((double)c.tr_on_wave) / c.tr_freq)
        out = amp * ramp(c, tau) * std::sin(d.omega * t + ph);
      else
        out = 0.0;
      set = true;
    }
    if (pressure ? c.tr_focused_p : c.tr_focused_v) {
      double s1 = std::sqrt((d.ctlx - xm) * (d.ctlx - xm) + (d.ctly - ym) * (d.ctly - ym));
      if (s1 <= d.focal_dist) {
        s1 = std::max(t - (d.focal_dist - s1) / d.cs_inf, 0.0);
        double s2 = std::fmod(s1, period);
        if (s2 < (double)c.tr_on_wave / c.tr_freq)
          out = amp * ramp(c, s2) * std::sin(d.omega * s2 + ph);
        else
          out = 0.0;
      } else {
        out = 0.0;
      }
      set = true;
    }
    return set;
  }

  // ---------------------------------------------------------------------
  crp_status init(const crp_config& c, const crp_bubbles_in* bin) {
    cfg = c;
    X = c.grid_x;
    Y = c.grid_y;
    a = make_index(X, Y, c.sim_order);
    d = derive(c);
    cyl = c.tr_cylindrical != 0;
    bubbles_on = c.bub_enable != 0;
    source_row = c.ext_source_row;
    if (c.ext_elements > 0) {
      // Aperture radius: the largest |x - ctl_x| among the pressure source's
      // cells (a focused source only within focal_dist of the focus).
      if (!(c.tr_plane_p || c.tr_focused_p) || c.tr_plane_v || c.tr_focused_v || c.tr_pid) return CRP_ERR_INVALID;
      const double ym = source_row > 0 ? ((double)source_row - 0.5) * d.dy : -0.5 * d.dy;
      elem_rap = 0.0;
      for (int i = 1; i <= X; i++) {
        const double xm = ((double)i - 0.5) * d.dx;
        if (c.tr_focused_p) {
          const double s1 = std::sqrt((d.ctlx - xm) * (d.ctlx - xm) + (d.ctly - ym) * (d.ctly - ym));
          if (!(s1 <= d.focal_dist)) continue;
        }
        elem_rap = std::max(elem_rap, std::fabs(xm - d.ctlx));
      }
      if (!(elem_rap > 0.0)) return CRP_ERR_INVALID;
      elem_n = c.ext_elements;
      elem_amp.assign(elem_n, 1.0);
      elem_phase.assign(elem_n, 0.0);
    }
    make_sigma(c, a, d, mx, my, nx, ny);
    // init_grid_vector, src/bubble_CUDA.cu:690-713.
    rxp.assign(a.iend2m - a.ista2m + 1, 0.0);
    xu.assign(a.iend2n - a.ista2n + 1, 0.0);
    for (int i = a.ista2m; i <= a.iend2m; i++) rxp[i - a.ista2m] = 1.0 / (d.dx * ((double)i - 0.5));
    for (int i = a.ista2n; i <= a.iend2n; i++) xu[i - a.ista2n] = ((double)i) * d.dx;
    // init_mix_array, src/bubble_CUDA.cu:716-794.
    p0.init(a.ista1m, a.iend1m, a.jsta1m, a.jend1m, 0.0);
    px.init(a.ista1m, a.iend1m, a.jsta1m, a.jend1m, 0.0);
    py = px;
    pnx = px;
    pny = px;
    rho_m.init(a.ista1m, a.iend1m, a.jsta1m, a.jend1m, d.rho_inf);
    vx.init(a.ista2n, a.iend2n, a.jsta2m, a.jend2m, 0.0);
    vy.init(a.ista2m, a.iend2m, a.jsta2n, a.jend2n, 0.0);
    fg.init(a.ista2m, a.iend2m, a.jsta2m, a.jend2m, 0.0);
    fgn = fg;
    fgm = fg;
    work = fg;
    temperature_on = c.dbg_T != 0 || c.tr_pid != 0;
    focal_hist.assign(1, 0.0);
    control_hist.assign(1, d.ctly);
    if (temperature_on) {
      T.init(a.ista2m, a.iend2m, a.jsta2m, a.jend2m, 0.0);
      k_m = T;
      twork = T;
      C_pm.init(a.ista1m, a.iend1m, a.jsta1m, a.jend1m, heat_capacity_water(d.T_inf));
      Ex.init(a.ista1n, a.iend1n, a.jsta1m, a.jend1m, 0.0);
      Ey.init(a.ista1m, a.iend1m, a.jsta1n, a.jend1n, 0.0);
    }
    if (bubbles_on) {
      crp_status st = init_bubbles(bin);
      if (st != CRP_OK) return st;
    }
    // Init kernels, src/bubble_CUDA.cu:175-187.
    if (bubbles_on) {
      update_indices();
      void_fraction();
    }
    fgn = fg;
    fgm = fg;
    return CRP_OK;
  }

  void add_bubble(double bx, double by, double R0, double nB) {
    BubConst b = make_bubconst(R0, cfg.bub_P0, cfg.bub_T0, cfg.bub_gamma, cfg.bub_sigma, cfg.bub_mu, cfg.bub_rho,
                               cfg.bub_K0, d.bub_dt0);
    // bubble_input, src/bubble_CUDA.cu:900-943.
    bc.push_back(b);
    x.push_back(bx);
    y.push_back(by);
    R_t.push_back(R0);
    R_p.push_back(R0);
    R_pn.push_back(R0);
    R_n.push_back(R0);
    R_nn.push_back(R0);
    d1_R_p.push_back(0.0);
    d1_R_n.push_back(0.0);
    PG_p.push_back(b.PG0);
    PG_n.push_back(b.PG0);
    PL_p.push_back(0.0);
    PL_n.push_back(0.0);
    PL_m.push_back(0.0);
    Q_B.push_back(0.0);
    n_B.push_back(nB);
    dtb.push_back(b.dt0);
    dt_n.push_back(b.dt0);
    re.push_back(0.0);
    re_n.push_back(0.0);
    vbx.push_back(0.0);
    vby.push_back(0.0);
    ibmx.push_back(0);
    ibmy.push_back(0);
    ibnx.push_back(0);
    ibny.push_back(0);
    nsub.push_back(0);
  }

  crp_status init_bubbles(const crp_bubbles_in* bin) {
    if (bin && bin->n > 0) {
      for (int k = 0; k < bin->n; k++) add_bubble(bin->x[k], bin->y[k], bin->r0[k], bin->n_b[k]);
    } else if (cfg.ext_bubble_count > 0) {
      return CRP_ERR_INVALID;  // seeded populations are passed in explicitly
    } else {
      // init_bub_array cell loop, src/bubble_CUDA.cu:811-839; n_B of bubble_input :922-931.
      const double pi = std::acos(-1.0);
      for (int i = a.istam; i <= a.iendm; i++) {
        double bx = ((double)i - 0.5) * d.dx;
        for (int j = a.jstam; j <= a.jendm; j++) {
          double by = ((double)j - 0.5) * d.dy;
          bool take = cfg.tr_box_size ? (std::fabs(bx - d.fpx) < 0.5 * cfg.tr_box_size &&
                                         std::fabs(by - d.fpy) < 0.5 * cfg.tr_box_size)
                                      : true;
          if (!take) continue;
          double R0 = cfg.bub_R0;
          double nB = cyl ? cfg.bub_fg0 * (bx * d.dx * d.dy) / (4.0 / 3.0 * pi * std::pow(R0, 3))
                          : cfg.bub_fg0 * (d.dx * d.dy) / (4.0 / 3.0 * pi * std::pow(R0, 3));
          add_bubble(bx, by, R0, nB);
        }
      }
    }
    nb = (int)x.size();
    return CRP_OK;
  }

  // BubbleUpdateIndexKernel, inc/bubble_CUDA_kernel.cuh:345-358.
  void update_indices() {
    for (int b = 0; b < nb; b++) {
      ibmx[b] = (int)std::floor(x[b] * d.rdx + 1.0);
      ibmy[b] = (int)std::floor(y[b] * d.rdy + 1.0);
      ibnx[b] = (int)std::floor(x[b] * d.rdx + 0.5);
      ibny[b] = (int)std::floor(y[b] * d.rdy + 0.5);
    }
  }

  // calculate_void_fraction, inc/bubble_CUDA_kernel.cuh:1198-1218, with
  // VoidFractionReverseLookupKernel (:576-619) and VoidFractionCylinderKernel (:559-573).
  // The reference accumulates with unordered atomics; here each cell sums its
  // contributions in ascending bubble order.
  void void_fraction() {
    std::fill(fg.v.begin(), fg.v.end(), 0.0);
    for (int b = 0; b < nb; b++) {
      double r = R_t[b];
      double t = cyl ? d.pi4r3 * n_B[b] * (r * r * r) * d.rdx * d.rdy / x[b] : d.pi4r3 * n_B[b] * (r * r * r) * d.rdx * d.rdy;
      for (int i = ibnx[b] + d.mbs; i <= ibnx[b] + d.mbe; i++) {
        double dxw = delta_x(i, x[b]);
        for (int j = ibny[b] + d.mbs; j <= ibny[b] + d.mbe; j++) {
          double dyw = delta_y(j, y[b]);
          if (i >= a.ista2m && i <= a.iend2m && j >= a.jsta2m && j <= a.jend2m) fg.at(i, j) += t * dxw * dyw;
        }
      }
    }
    if (cyl) {
      for (int j = a.jsta2m; j <= a.jend2m; j++)
        for (int k = 1 + a.ns + a.ms; k <= 0; k++) {
          fg.at(k, j) += fg.at(1 - k, j);
          fg.at(1 - k, j) = fg.at(k, j);
        }
    }
  }

  // store_variables + VFPredictionKernel, inc/bubble_CUDA_kernel.cuh:1229-1262, 622-633.
  void store_variables() {
    std::fill(work.v.begin(), work.v.end(), 0.0);
    R_pn = R_p;
    R_nn = R_n;
    d1_R_n = d1_R_p;
    PG_n = PG_p;
    PL_m = PL_n;
    PL_n = PL_p;
    dt_n = dtb;
    re_n = re;
    const size_t n = fg.v.size();
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < n; k++) work.v[k] = 3.0 * fg.v[k] - 3.0 * fgn.v[k] + fgm.v[k];
    pnx.v = px.v;
    pny.v = py.v;
    fgm.v = fgn.v;
    fgn.v = fg.v;
    fg.v = work.v;
  }

  // VelocityKernel (inc/bubble_CUDA_kernel.cuh:635-677) then VelocityBoundaryKernel (:680-813).
  void velocity() {
    const double dt = d.dt;
    const double c = d.cs_inf;
#pragma omp parallel for schedule(static)
    for (int jn = a.jsta2n; jn <= std::max(a.jend2m, a.jend2n); jn++) {
      for (int in = a.ista2n; in <= std::max(a.iend2m, a.iend2n); in++) {
        bool ok1 = in >= a.istan && in <= a.iendn && jn >= a.jstam && jn <= a.jendm;
        bool ok2 = in >= a.istam && in <= a.iendm && jn >= a.jstan && jn <= a.jendn;
        if (ok1) {
          double s1 = (rho_m.at(in, jn) + rho_m.at(in + 1, jn)) * 0.5;
          double s2 = (-p0.at(in, jn) + p0.at(in + 1, jn)) * d.rdx;
          double s3 = (c + c) * 0.5;
          s3 = s3 * 0.5 * dt * nx[in - a.ista2n];
          vx.at(in, jn) = (vx.at(in, jn) * (1.0 - s3) - dt / s1 * s2) / (1.0 + s3);
        }
        if (ok2) {
          double s1 = (rho_m.at(in, jn) + rho_m.at(in, jn + 1)) * 0.5;
          double s2 = (-p0.at(in, jn) + p0.at(in, jn + 1)) * d.rdx;  // rdx, as the reference (:671)
          double s3 = (c + c) * 0.5;
          s3 = s3 * 0.5 * dt * ny[jn - a.jsta2n];
          vy.at(in, jn) = (vy.at(in, jn) * (1.0 - s3) - dt / s1 * s2) / (1.0 + s3);
        }
      }
    }
    velocity_boundary();
  }

  // VelocityBoundaryKernel, inc/bubble_CUDA_kernel.cuh:680-813.  Its four
  // sections race with each other across threads; they run here in program
  // order, each over all indices before the next.
  void velocity_boundary() {
    const int X_ = X, Y_ = Y;
    // vx along x: rows jstam..jendm (:702-721).
    for (int j = a.jstam; j <= a.jendm; j++) {
      if (!cfg.pml_x0) {
        for (int i = a.ms + a.ns; i <= -1; i++) vx.at(i, j) = vx.at(-i, j);
        vx.at(0, j) = 0.0;
      }
      if (!cfg.pml_x1) {
        for (int i = X_ + 1; i <= X_ + a.me + a.ne; i++) vx.at(i, j) = -vx.at(X_ - (i - X_), j);
        vx.at(X_, j) = 0.0;
      }
    }
    // vx along y: columns ista2n..iend2n (:722-732).
    for (int i = a.ista2n; i <= a.iend2n; i++) {
      for (int j = 1 + a.ms + a.ns; j <= 0; j++) vx.at(i, j) = vx.at(i, 1 - j);
      for (int j = Y_ + 1; j <= Y_ + a.me + a.ne; j++) vx.at(i, j) = vx.at(i, Y_ - (j - Y_ - 1));
    }
    // vy along y: columns istam..iendm (:734-798).  With an [ext] source row
    // the source is forced on that row after the y0 block and before the y1 block.
    for (int i = a.istam; i <= a.iendm; i++) {
      if (!cfg.pml_y0) {
        if (!src_pressure()) vy.at(i, 0) = 0.0;
        for (int j = a.ns + a.ms; j <= -1; j++) vy.at(i, j) = vy.at(i, -(j + 1));
        double v;
        if (source_row == 0 && source_value(false, ((double)i - 0.5) * d.dx, 0.0, tstep, v)) vy.at(i, 0) = v;
      }
      if (source_row > 0) {
        double v;
        if (source_value(false, ((double)i - 0.5) * d.dx, (double)source_row * d.dy, tstep, v))
          vy.at(i, source_row) = v;
      }
      if (!cfg.pml_y1) {
        vy.at(i, Y_) = 0.0;
        for (int j = Y_ + 1; j <= Y_ + a.ne + a.me; j++) vy.at(i, j) = vy.at(i, Y_ - (j - Y_));
      }
    }
    // vy along x: rows jsta2n..jend2n (:799-811).  The X1 mirror reads array
    // row X+1 (logical j = X+1+jsta2n), column X, for every row, as the
    // reference's index expression does (:808); where that row does not exist
    // (X > Y+1, an out-of-bounds read in the reference) it mirrors column X of
    // the same row.
    for (int j = a.jsta2n; j <= a.jend2n; j++) {
      for (int i = 1 + a.ms + a.ns; i <= 0; i++) vy.at(i, j) = vy.at(1 - i, j);
      for (int i = X_ + 1; i <= X_ + a.me + a.ne; i++) {
        int jr = i + a.jsta2n;
        vy.at(i, j) = vy.at(X_ - (i - X_ - 1), jr <= a.jend2n ? jr : j);
      }
    }
  }

  // BubbleInterpolationVelocityKernel + BubbleMotionKernel, inc/bubble_CUDA_kernel.cuh:398-468, 1282-1297.
  void bubble_motion() {
#pragma omp parallel for schedule(static)
    for (int b = 0; b < nb; b++) {
      double vlx = 0.0, vly = 0.0;
      for (int i = ibmx[b] + d.nbs; i <= ibmx[b] + d.nbe; i++) {
        double dxw = delta_x(i, x[b]);
        for (int j = ibny[b] + d.mbs; j <= ibny[b] + d.mbe; j++) {
          double dyw = delta_y(j, y[b]);
          if (i >= a.ista2n && i <= a.iend2n && j >= a.jsta2m && j <= a.jend2m) vlx += vx.at(i, j) * dxw * dyw;
        }
      }
      for (int i = ibnx[b] + d.mbs; i <= ibnx[b] + d.mbe; i++) {
        double dxw = delta_x(i, x[b]);
        for (int j = ibmy[b] + d.nbs; j <= ibmy[b] + d.nbe; j++) {
          double dyw = delta_y(j, y[b]);
          if (i >= a.ista2m && i <= a.iend2m && j >= a.jsta2n && j <= a.jend2n) vly += vy.at(i, j) * dxw * dyw;
        }
      }
      vbx[b] = vlx;
      vby[b] = vly;
      x[b] = x[b] + vbx[b] * d.dt;
      y[b] = y[b] + vby[b] * d.dt;
      ibmx[b] = (int)std::floor(x[b] * d.rdx + 1.0);
      ibmy[b] = (int)std::floor(y[b] * d.rdy + 1.0);
      ibnx[b] = (int)std::floor(x[b] * d.rdx + 0.5);
      ibny[b] = (int)std::floor(y[b] * d.rdy + 0.5);
    }
  }

  // calculate_pressure_field: MixturePressureKernel (inc/bubble_CUDA_kernel.cuh:816-867),
  // MixtureBoundaryPressureKernel (:870-952), residual max (:1317-1328).
  double pressure() {
    std::fill(work.v.begin(), work.v.end(), 0.0);
    const double dt = d.dt;
    const double c = d.cs_inf;
    const bool forced_row = source_row > 0 && src_pressure();
#pragma omp parallel for schedule(static)
    for (int j = a.jstam; j <= a.jendm; j++) {
      for (int i = a.istam; i <= a.iendm; i++) {
        double s1x;
        if (cyl)
          s1x = (-xu[(i - 1) - a.ista2n] * vx.at(i - 1, j) + xu[i - a.ista2n] * vx.at(i, j)) * d.rdx *
                rxp[i - a.ista2m];
        else
          s1x = (-vx.at(i - 1, j) + vx.at(i, j)) * d.rdx;
        double s1y = (-vy.at(i, j - 1) + vy.at(i, j)) * d.rdy;
        double s3 = dt * d.rho_inf * c * c;
        double s4 = 0.5 * dt * c;
        double f = fg.at(i, j), fn = fgn.at(i, j);
        double s5 = -(f - fn) / dt / (1.0 - 0.5 * (f + fn));
        double s2x = s4 * mx[i - a.ista1m], s2y = s4 * my[j - a.jsta1m];
        double h = 0.5 * s5;
        double qx = pnx.at(i, j) * (1.0 - s2x) - s3 * (s1x + h) / (1.0 + s2x);
        double qy = pny.at(i, j) * (1.0 - s2y) - s3 * (s1y + h) / (1.0 + s2y);
        px.at(i, j) = qx;
        py.at(i, j) = qy;
        if (forced_row && j == source_row) continue;  // residual taken after forcing
        work.at(i, j) = std::fabs(p0.at(i, j) - (qx + qy));
        p0.at(i, j) = qx + qy;
      }
    }
    pressure_boundary();
    double m = 0.0;
    for (double w : work.v)
      if (m < w) m = w;
    return m / d.P_inf;
  }

  // MixtureBoundaryPressureKernel, inc/bubble_CUDA_kernel.cuh:870-952.  The
  // y-face section runs over all columns before the x-face section (the
  // reference races them).  The y1 mirror follows the reference's intent,
  // p0(Y+1) = p0(Y); its index expression (:929-931) reads outside the array.
  // An [ext] source row is forced first, so the y0 mirror sees the forced value.
  void pressure_boundary() {
    for (int i = a.istam; i <= a.iendm; i++) {
      double xm = ((double)i - 0.5) * d.dx;
      if (source_row > 0) {
        double v;
        if (source_value(true, xm, ((double)source_row - 0.5) * d.dy, tstep, v)) {
          work.at(i, source_row) = std::fabs(p0.at(i, source_row) - v);
          p0.at(i, source_row) = v;
        }
      }
      if (!cfg.pml_y0) {
        for (int j = a.ms; j <= 0; j++) p0.at(i, j) = p0.at(i, 1 - j);
        double v;
        if (source_row == 0 && source_value(true, xm, -0.5 * d.dy, tstep, v)) p0.at(i, 0) = v;
      }
      if (!cfg.pml_y1)
        for (int j = Y + 1; j <= Y + a.me; j++) p0.at(i, j) = p0.at(i, Y - (j - Y - 1));
    }
    for (int j = a.jsta1m; j <= a.jend1m; j++) {
      if (!cfg.pml_x0)
        for (int i = a.ms; i <= 0; i++) p0.at(i, j) = p0.at(1 - i, j);
      if (!cfg.pml_x1)
        for (int i = X + 1; i <= X + a.me; i++) p0.at(i, j) = p0.at(X - (i - X - 1), j);
    }
  }

  // BubbleInterpolationScalarKernel, inc/bubble_CUDA_kernel.cuh:361-395.
  void interpolate_pressure() {
#pragma omp parallel for schedule(static)
    for (int b = 0; b < nb; b++) {
      double s = 0.0;
      for (int i = ibnx[b] + d.mbs; i <= ibnx[b] + d.mbe; i++) {
        double dxw = delta_x(i, x[b]);
        for (int j = ibny[b] + d.mbs; j <= ibny[b] + d.mbe; j++) {
          double dyw = delta_y(j, y[b]);
          if (i >= a.ista1m && i <= a.iend1m && j >= a.jsta1m && j <= a.jend1m) s += p0.at(i, j) * dxw * dyw;
        }
      }
      PL_p[b] = s;
    }
  }

  // BubbleRadiusKernel, inc/bubble_CUDA_kernel.cuh:471-554.  Returns the largest
  // sub-step count, or -1 if a bubble hit the sub-step cap.
  int64_t bubble_radii() {
    const double dt = d.dt;
    const int64_t cap = cfg.ext_rp_step_cap;
    int64_t worst = 0;
    bool capped = false;
    if (cfg.ext_rp_scheme == CRP_RP_RK45) return bubble_radii_rk45();
#pragma omp parallel for schedule(dynamic, 64) reduction(max : worst) reduction(|| : capped)
    for (int b = 0; b < nb; b++) {
      const BubConst& k = bc[b];
      double Rt = R_t[b];
      double Rp = R_pn[b], Rn = R_nn[b], d1Rp = d1_R_n[b], PGp = PG_n[b], dtL = dt_n[b];
      double remain = re_n[b] + dt;
      double time = -re_n[b];
      double PC0 = PL_n[b] + k.PL0;
      double PC1 = 0.5 * (PL_p[b] - PL_m[b]) / dt;
      double PC2 = 0.5 * (PL_p[b] + PL_m[b] - 2.0 * PL_n[b]) / (dt * dt);
      double heat = 0.0, vis = 0.0;
      int64_t count = 0;
      while (remain > 0.0) {
        if (count >= cap) {
          capped = true;
          break;
        }
        double PGn = PGp;
        double PL = PC2 * time * time + PC1 * time + PC0;
        rp_substep(Rt, Rp, Rn, d1Rp, PGn, PL, dtL, remain, k);
        time = time + dtL;
        Cplx alpha;
        double omega = thermal_omega(alpha, PGn, Rn, k);
        Cplx lp = thermal_lp(alpha, Rn);
        PGp = gas_pressure(PGn, Rp, Rn, omega, dtL, lp, k);
        double s0 = 0.5 * (Rp + Rn);
        double s1 = 1 / (lp.re * lp.re + lp.im * lp.im) * k.T0 / (k.PG0 * k.R03);
        double dTdr = lp.re * s1 * (k.PG0 * k.R03 - 0.5 * (PGp + PGn) * s0 * s0 * s0) +
                      lp.im * s1 * (PGp * Rp * Rp * Rp - PGn * Rn * Rn * Rn) / (omega * dtL);
        heat -= 4.0 * d.pi * Rp * Rp * k.K0 * dTdr * dtL;
        vis += 4.0 * d.pi * Rp * Rp * 4.0 * k.mu * d1Rp / Rp * d1Rp * dtL;
        count++;
      }
      R_t[b] = Rt;
      R_p[b] = Rp;
      R_n[b] = Rn;
      d1_R_p[b] = d1Rp;
      PG_p[b] = PGp;
      dtb[b] = dtL;
      re[b] = remain;
      Q_B[b] = (heat + vis) / (dt - remain + re_n[b]);
      nsub[b] = (int)std::min<int64_t>(count, INT32_MAX);
      worst = std::max(worst, count);
    }
    return capped ? -1 : worst;
  }

  // The radius solve with ext.rp_scheme = rk45 (rk45_run): from the state at
  // the start of the step (R_pn, d1_R_n, PG_n, last step size dt_n) to the
  // step's end exactly; results in the arrays the reference scheme fills.
  int64_t bubble_radii_rk45() {
    const double dt = d.dt;
    const int64_t cap = cfg.ext_rp_step_cap;
    const double rtol = cfg.ext_rp_tol > 0.0 ? cfg.ext_rp_tol : 1.0e-6;
    int64_t worst = 0;
    bool capped = false;
#pragma omp parallel for schedule(dynamic, 64) reduction(max : worst) reduction(|| : capped)
    for (int b = 0; b < nb; b++) {
      const BubConst& k = bc[b];
      RkBubble m;
      m.k = &k;
      m.K = 3.0 * (k.gam - 1.0) * k.K0 * k.T0 / k.PG0;
      m.PC0 = PL_n[b] + k.PL0;
      m.PC1 = 0.5 * (PL_p[b] - PL_m[b]) / dt;
      m.PC2 = 0.5 * (PL_p[b] + PL_m[b] - 2.0 * PL_n[b]) / (dt * dt);
      m.pi = d.pi;
      RkRun s{R_pn[b], d1_R_n[b], PG_n[b], dt_n[b], 0.0, dt, 0.0, 0};
      if (!rk45_run(m, s, rtol, cap)) capped = true;
      R_t[b] = R_p[b] = R_n[b] = s.R;
      d1_R_p[b] = s.V;
      PG_p[b] = s.PG;
      dtb[b] = std::min(s.h, dt);
      re[b] = 0.0;
      Q_B[b] = s.Q / dt;
      nsub[b] = (int)std::min<int64_t>(s.count, INT32_MAX);
      worst = std::max(worst, s.count);
    }
    return capped ? -1 : worst;
  }

  // MixturePropertiesKernel (inc/bubble_CUDA_kernel.cuh:1110-1125): density,
  // and the heat capacity when the temperature is computed.
  void properties() {
#pragma omp parallel for schedule(static)
    for (int j = a.jsta1m; j <= a.jend1m; j++)
      for (int i = a.ista1m; i <= a.iend1m; i++) {
        rho_m.at(i, j) = (1.0 - fg.at(i, j)) * d.rho_inf;
        if (temperature_on) C_pm.at(i, j) = heat_capacity_water(T.at(i, j) + d.T_inf);
      }
  }

  // Focal depth of the step (determine_focal_point, inc/bubble_CUDA_kernel.cuh:
  // 1132-1166, whose reduction functors are not in the reference's tree): the
  // mean of the cell-centre depths weighted by the temperature increment's
  // excess over half its maximum, over the interior cells (0 while the maximum
  // is at most 1e-30 K, rounding size); then filter_loop
  // (:117-129) and, with transducer.pid, focal_PID and the clamp
  // (src/bubble_CUDA.cu:328-347, inc/bubble_CUDA_kernel.cuh:1168-1184).
  void track_focus() {
    double mx = -1.0e300;
    for (int j = a.jstam; j <= a.jendm; j++)
      for (int i = a.istam; i <= a.iendm; i++) mx = std::max(mx, twork.at(i, j));
    double sw = 0.0, swy = 0.0;
    if (mx > 1.0e-30) {  // rounding-size increments define no focus
      const double thr = 0.5 * mx;
      for (int j = a.jstam; j <= a.jendm; j++) {
        const double y = ((double)j - 0.5) * d.dy;
        for (int i = a.istam; i <= a.iendm; i++) {
          const double v = twork.at(i, j) - thr;
          if (v > 0.0) {
            sw += v;
            swy += v * y;
          }
        }
      }
    }
    const double depth = sw > 0.0 ? swy / sw : 0.0;
    double* xv = filt_in;
    double* yv = filt_out;
    const double gain = 6.522112693e+08;
    for (int k = 0; k < 4; k++) xv[k] = xv[k + 1];
    xv[4] = depth / gain;
    for (int k = 0; k < 4; k++) yv[k] = yv[k + 1];
    yv[4] = (xv[0] + xv[4]) + 4 * (xv[1] + xv[3]) + 6 * xv[2] + (-0.9676955438 * yv[0]) + (3.9025587848 * yv[1]) +
            (-5.9020258615 * yv[2]) + (3.9671625959 * yv[3]);
    focal_hist.push_back(yv[4]);
    if (cfg.tr_pid && nstep > cfg.tr_pid_start_step) {
      const double K = 0.2 * 0.60, Pc = 1000.0, D = K * 0.125 * Pc, I = K / (0.5 * Pc);
      const double ty = d.fpy;
      const double ay = focal_hist[focal_hist.size() - 1], py = focal_hist[focal_hist.size() - 2];
      const double ey = ty - ay;
      pid_cum_y += ey;
      pid_der_y = py - ay;
      double cy = ty + (K * ey + D * pid_der_y + I * pid_cum_y);
      cy = cy < ty ? ty : (cy > cfg.grid_ly ? cfg.grid_ly : cy);
      control_hist.push_back(cy);
      d.ctlx = 0.0;
      d.ctly = cy;
      d.focal_dist = cy / 0.5 / std::sqrt(3.0);
    }
  }

  // calculate_temperature (inc/bubble_CUDA_kernel.cuh:1347-1376).
  void temperature() {
    // Work cleared, then BubbleHeatKernel (:972-1007), bubble by bubble.
    std::fill(twork.v.begin(), twork.v.end(), 0.0);
    if (bubbles_on) {
      for (int b = 0; b < nb; b++) {
        const double q = cyl ? n_B[b] * Q_B[b] * d.rdx * d.rdy / x[b] : n_B[b] * Q_B[b] * d.rdx * d.rdy;
        for (int i = ibnx[b] + d.mbs; i <= ibnx[b] + d.mbe; i++) {
          const double dxw = delta_x(i, x[b]);
          for (int j = ibny[b] + d.mbs; j <= ibny[b] + d.mbe; j++) {
            const double dyw = delta_y(j, y[b]);
            if (i >= a.ista2m && i <= a.iend2m && j >= a.jsta2m && j <= a.jend2m) twork.at(i, j) += q * dxw * dyw;
          }
        }
      }
    }
    // MixtureKMKernel (:955-969).
    for (int j = a.jsta2m; j <= a.jend2m; j++)
      for (int i = a.ista2m; i <= a.iend2m; i++)
        k_m.at(i, j) = conductivity_water(T.at(i, j) + d.T_inf) * (1.0 - 3.0 * fg.at(i, j) / (2.0 + fg.at(i, j)));
    // MixtureEnergyKernel (:1010-1035).
    for (int j = a.jsta1m; j <= a.jend1m; j++)
      for (int i = a.ista1n; i <= a.iend1n; i++) {
        const double s0 = 2.0 * k_m.at(i, j) * k_m.at(i + 1, j) / (k_m.at(i, j) + k_m.at(i + 1, j));
        const double s1 = (-T.at(i, j) + T.at(i + 1, j)) * d.rdx;
        Ex.at(i, j) = s0 * s1;
      }
    for (int j = a.jsta1n; j <= a.jend1n; j++)
      for (int i = a.ista1m; i <= a.iend1m; i++) {
        const double s0 = 2.0 * k_m.at(i, j) * k_m.at(i, j + 1) / (k_m.at(i, j) + k_m.at(i, j + 1));
        const double s1 = (-T.at(i, j) + T.at(i, j + 1)) * d.rdy;
        Ey.at(i, j) = s0 * s1;
      }
    // MixtureTemperatureKernel (:1038-1062).
    for (int j = a.jstam; j <= a.jendm; j++)
      for (int i = a.istam; i <= a.iendm; i++) {
        double s0 = (px.at(i, j) + py.at(i, j) - pnx.at(i, j) - pny.at(i, j)) / d.dt;
        s0 = 2.0 * (0.22) * 0.115129255 / (d.rho_inf * d.cs_inf * d.omega * d.omega) * s0 * s0;
        const double Q = twork.at(i, j) + s0;
        const double s1 = (Ex.at(i, j) - Ex.at(i - 1, j)) * d.rdx;
        const double s2 = (Ey.at(i, j) - Ey.at(i, j - 1)) * d.rdy;
        T.at(i, j) += twork.at(i, j) = d.dt * (s1 + s2 + Q) / (rho_m.at(i, j) * C_pm.at(i, j));
      }
    // MixtureBoundaryTemperatureKernel (:1065-1102), sections in order.
    if (!cfg.pml_x0)
      for (int j = a.jstam; j <= a.jendm; j++)
        for (int i = 1 + a.ns + a.ms; i <= 0; i++) T.at(i, j) = T.at(1 - i, j);
    if (!cfg.pml_x1)
      for (int j = a.jsta1m; j <= a.jend1m; j++)
        for (int i = X + 1; i <= X + a.ne + a.me; i++) T.at(i, j) = T.at(X - (i - X - 1), j);
    if (!cfg.pml_y0)
      for (int i = a.ista2m; i <= a.iend2m; i++)
        for (int j = 1 + a.ns + a.ms; j <= 0; j++) T.at(i, j) = T.at(i, 1 - j);
    if (!cfg.pml_y1)
      for (int i = a.ista2m; i <= a.iend2m; i++)
        for (int j = Y; j <= Y + a.ne + a.me; j++) T.at(i, j) = T.at(i, Y - (j - Y - 1));
  }

  // One pass of solve_bubbles' main loop, src/bubble_CUDA.cu:206-285.
  crp_status step() {
    nstep++;
    double s1 = tstep;
    tstep = tstep + d.dt + tstepx;
    double s2 = tstep - s1;
    tstepx = d.dt + tstepx - s2;
    store_variables();
    velocity();
    if (bubbles_on) bubble_motion();
    double resimax = pressure();
    int loop = 0;
    if (bubbles_on) {
      const double tol = cfg.ext_picard_tol > 0.0 ? cfg.ext_picard_tol : (double)1.0e-7f;
      while (resimax > tol) {
        if (loop >= cfg.ext_picard_cap) return CRP_ERR_PICARD;
        loop++;
        interpolate_pressure();
        int64_t worst = bubble_radii();
        if (worst < 0) return CRP_ERR_RP_STEPS;
        stats.rp_substeps_max = std::max(stats.rp_substeps_max, worst);
        void_fraction();
        resimax = pressure();
      }
    }
    if (temperature_on) {
      temperature();
      track_focus();
    }
    properties();
    stats.steps = nstep;
    stats.time = tstep;
    stats.picard_last = loop;
    stats.picard_total += loop;
    stats.picard_max = std::max(stats.picard_max, loop);
    stats.residual_last = resimax;
    return CRP_OK;
  }
};

// -------------------------------------------------------------------------
extern "C" {

crp_status crpo_create(const crp_config* cfg, const crp_bubbles_in* bubbles, crpo_sim** out) {
  if (!cfg || !out) return CRP_ERR_INVALID;
  if (cfg->grid_x <= 0 || cfg->grid_y <= 0 || cfg->sim_order < 2 || cfg->sim_smooth_delta_band < 1)
    return CRP_ERR_INVALID;
  crpo_sim* s = new (std::nothrow) crpo_sim();
  if (!s) return CRP_ERR_ALLOC;
  crp_status st = s->init(*cfg, bubbles);
  if (st != CRP_OK) {
    delete s;
    return st;
  }
  *out = s;
  return CRP_OK;
}

crp_status crpo_set_source_elements(crpo_sim* s, int32_t n, const double* amp, const double* phase) {
  if (!s || n != s->elem_n || n <= 0 || !amp || !phase) return CRP_ERR_INVALID;
  s->elem_amp.assign(amp, amp + n);
  s->elem_phase.assign(phase, phase + n);
  return CRP_OK;
}

crp_status crpo_step(crpo_sim* s, int32_t n) {
  if (!s) return CRP_ERR_INVALID;
#ifdef _OPENMP
  if (g_threads > 0) omp_set_num_threads(g_threads);
#endif
  for (int k = 0; k < n; k++) {
    crp_status st = s->step();
    if (st != CRP_OK) return st;
  }
  return CRP_OK;
}

crp_status crpo_get_dims(const crpo_sim* s, crp_dims* d) {
  if (!s || !d) return CRP_ERR_INVALID;
  d->i1m = s->p0.w;
  d->j1m = s->p0.h;
  d->i2m = s->fg.w;
  d->j2m = s->fg.h;
  d->i2n = s->vx.w;
  d->j2n = s->vy.h;
  d->num_bubbles = s->nb;
  d->dx = s->d.dx;
  d->dy = s->d.dy;
  d->dt = s->d.dt;
  return CRP_OK;
}

crp_status crpo_get_stats(const crpo_sim* s, crp_stats* st) {
  if (!s || !st) return CRP_ERR_INVALID;
  *st = s->stats;
  return CRP_OK;
}

int64_t crpo_focus_history(const crpo_sim* s, int32_t which, double* out, int64_t capacity) {
  if (!s || (which != 0 && which != 1)) return -1;
  if (!s->temperature_on) return 0;
  const std::vector<double>& v = which == 0 ? s->focal_hist : s->control_hist;
  for (int64_t k = 0; out && k < capacity && k < (int64_t)v.size(); k++) out[k] = v[k];
  return (int64_t)v.size();
}

crp_status crpo_read_field(crpo_sim* s, crp_field f, double* host) {
  if (!s || !host) return CRP_ERR_INVALID;
  const Field* src = nullptr;
  switch (f) {
    case CRP_FIELD_P0: src = &s->p0; break;
    case CRP_FIELD_PX: src = &s->px; break;
    case CRP_FIELD_PY: src = &s->py; break;
    case CRP_FIELD_PNX: src = &s->pnx; break;
    case CRP_FIELD_PNY: src = &s->pny; break;
    case CRP_FIELD_VX: src = &s->vx; break;
    case CRP_FIELD_VY: src = &s->vy; break;
    case CRP_FIELD_FG: src = &s->fg; break;
    case CRP_FIELD_FGN: src = &s->fgn; break;
    case CRP_FIELD_FGM: src = &s->fgm; break;
    case CRP_FIELD_RHO_M: src = &s->rho_m; break;
    case CRP_FIELD_T:
      if (!s->temperature_on) return CRP_ERR_UNSUPPORTED;
      src = &s->T;
      break;
    default: return CRP_ERR_INVALID;
  }
  std::memcpy(host, src->v.data(), sizeof(double) * src->v.size());
  return CRP_OK;
}

crp_status crpo_read_bubbles(crpo_sim* s, crp_bubble_field w, double* host) {
  if (!s || !host) return CRP_ERR_INVALID;
  const std::vector<double>* v = nullptr;
  const std::vector<int>* iv = nullptr;
  switch (w) {
    case CRP_BUB_X: v = &s->x; break;
    case CRP_BUB_Y: v = &s->y; break;
    case CRP_BUB_R_T: v = &s->R_t; break;
    case CRP_BUB_R_P: v = &s->R_p; break;
    case CRP_BUB_R_N: v = &s->R_n; break;
    case CRP_BUB_D1R: v = &s->d1_R_p; break;
    case CRP_BUB_PG: v = &s->PG_p; break;
    case CRP_BUB_PL_P: v = &s->PL_p; break;
    case CRP_BUB_PL_N: v = &s->PL_n; break;
    case CRP_BUB_PL_M: v = &s->PL_m; break;
    case CRP_BUB_DT: v = &s->dtb; break;
    case CRP_BUB_RE: v = &s->re; break;
    case CRP_BUB_Q_B: v = &s->Q_B; break;
    case CRP_BUB_N_B: v = &s->n_B; break;
    case CRP_BUB_VX: v = &s->vbx; break;
    case CRP_BUB_VY: v = &s->vby; break;
    case CRP_BUB_IBM_X: iv = &s->ibmx; break;
    case CRP_BUB_IBM_Y: iv = &s->ibmy; break;
    case CRP_BUB_IBN_X: iv = &s->ibnx; break;
    case CRP_BUB_IBN_Y: iv = &s->ibny; break;
    case CRP_BUB_SUBSTEPS: iv = &s->nsub; break;
    case CRP_BUB_R0:
      for (int b = 0; b < s->nb; b++) host[b] = s->bc[b].R0;
      return CRP_OK;
    default: return CRP_ERR_INVALID;
  }
  if (v) std::memcpy(host, v->data(), sizeof(double) * v->size());
  if (iv)
    for (size_t b = 0; b < iv->size(); b++) host[b] = (*iv)[b];
  return CRP_OK;
}

void crpo_set_threads(int32_t n) {
  g_threads = n;
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#endif
}

int32_t crpo_get_threads(void) {
#ifdef _OPENMP
  return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
  return 1;
#endif
}

void crpo_destroy(crpo_sim* s) { delete s; }

static BubConst bub_from(const double* bp) {
  BubConst b;
  b.R0 = bp[0];
  b.PG0 = bp[1];
  b.PL0 = bp[2];
  b.T0 = bp[3];
  b.gam = bp[4];
  b.sig = bp[5];
  b.mu = bp[6];
  b.rho = bp[7];
  b.K0 = bp[8];
  b.dt0 = bp[9];
  b.R03 = b.R0 * b.R0 * b.R0;
  b.coeff_alpha = b.gam * b.PG0 * b.R03 / (2.0 * (b.gam - 1.0) * b.T0 * b.K0);
  return b;
}

void crpo_rp_step(const double* bp, double* st, double PG, double PL) {
  BubConst b = bub_from(bp);
  rp_substep(st[0], st[1], st[2], st[3], PG, PL, st[4], st[5], b);
}

double crpo_omega_n(const double* bp, double PG, double R, double* alpha) {
  BubConst b = bub_from(bp);
  Cplx a;
  double w = thermal_omega(a, PG, R, b);
  alpha[0] = a.re;
  alpha[1] = a.im;
  return w;
}

void crpo_upsilon_lp(double are, double aim, double gam, double R, double* out) {
  Cplx u = thermal_upsilon(Cplx{are, aim}, gam);
  Cplx l = thermal_lp(Cplx{are, aim}, R);
  out[0] = u.re;
  out[1] = u.im;
  out[2] = l.re;
  out[3] = l.im;
}

double crpo_solve_pg(const double* bp, double PGn, double Rp, double Rn, double omega_N, double dt, double lp_re,
                     double lp_im) {
  return gas_pressure(PGn, Rp, Rn, omega_N, dt, Cplx{lp_re, lp_im}, bub_from(bp));
}

void crpo_host_scalars(const crp_config* cfg, double* out) {
  Derived d = derive(*cfg);
  BubConst b = make_bubconst(cfg->bub_R0, cfg->bub_P0, cfg->bub_T0, cfg->bub_gamma, cfg->bub_sigma, cfg->bub_mu,
                             cfg->bub_rho, cfg->bub_K0, d.bub_dt0);
  double o[21] = {d.dx, d.dy, d.rdx, d.rdy, d.fpx, d.fpy, d.omega, d.dt, d.rho_inf, d.cs_inf, d.P_inf,
                  d.T_inf, b.PG0, b.R03, b.coeff_alpha, d.bub_dt0, (double)d.mbs, (double)d.mbe,
                  (double)d.nbs, (double)d.nbe, d.focal_dist};
  std::memcpy(out, o, sizeof(o));
}

int64_t crpo_bubble_history(const double* bp, double R_init, double dt_mix, double dpl, int32_t nsteps, double* R_out,
                            double* PG_out) {
  // One bubble of BubbleRadiusKernel (inc/bubble_CUDA_kernel.cuh:485-550) advanced
  // nsteps mixture steps in a liquid held at PL0 + dpl, from rest at R_init.
  BubConst b = bub_from(bp);
  double Rt = R_init, Rp = R_init, Rn = R_init, d1R = 0.0, PGp = b.PG0 * std::pow(b.R0 / R_init, 3.0 * b.gam),
         dtL = b.dt0, re = 0.0;
  int64_t total = 0;
  for (int s = 0; s < nsteps; s++) {
    double remain = re + dt_mix, time = -re;
    double PC0 = dpl + b.PL0;
    while (remain > 0.0) {
      double PGn = PGp;
      double PL = 0.0 * time * time + 0.0 * time + PC0;
      rp_substep(Rt, Rp, Rn, d1R, PGn, PL, dtL, remain, b);
      time = time + dtL;
      Cplx alpha;
      double omega = thermal_omega(alpha, PGn, Rn, b);
      Cplx lp = thermal_lp(alpha, Rn);
      PGp = gas_pressure(PGn, Rp, Rn, omega, dtL, lp, b);
      total++;
      if (total > 100000000) return -1;
    }
    re = remain;
    R_out[s] = Rt;
    PG_out[s] = PGp;
  }
  return total;
}

int64_t crpo_bubble_drive(const double* bp, double R_init, double dt_mix, double p_amp, double omega_drive,
                          int32_t nsteps, int32_t scheme, double param, double* R_out, double* PG_out) {
  // One bubble from rest at R_init under a liquid pressure PL0 + p_amp sin(w t),
  // entering each mixture step as the quadratic through its values at the
  // step's start, end and the start of the previous step (the simulation's
  // PL_m, PL_n, PL_p).  scheme 0: the reference scheme with its limits scaled
  // down by param (rp_substep_refined, param >= 1); scheme 1: rk45 at rtol = param.
  BubConst b = bub_from(bp);
  const double pi = std::acos(-1.0);
  double Rt = R_init, Rp = R_init, Rn = R_init, d1R = 0.0, PGp = b.PG0 * std::pow(b.R0 / R_init, 3.0 * b.gam),
         dtL = b.dt0, re = 0.0;
  int64_t total = 0;
  auto pl = [&](int s) { return p_amp * std::sin(omega_drive * (double)s * dt_mix); };
  for (int s = 0; s < nsteps; s++) {
    const double PLm = pl(s - 1), PLn = pl(s), PLp = pl(s + 1);
    const double PC0 = PLn + b.PL0, PC1 = 0.5 * (PLp - PLm) / dt_mix,
                 PC2 = 0.5 * (PLp + PLm - 2.0 * PLn) / (dt_mix * dt_mix);
    if (scheme == 1) {
      RkBubble m{&b, 3.0 * (b.gam - 1.0) * b.K0 * b.T0 / b.PG0, PC0, PC1, PC2, pi};
      RkRun r{Rp, d1R, PGp, dtL, 0.0, dt_mix, 0.0, 0};
      if (!rk45_run(m, r, param, 100000000)) return -1;
      Rt = Rp = Rn = r.R;
      d1R = r.V;
      PGp = r.PG;
      dtL = std::min(r.h, dt_mix);
      total += r.count;
    } else {
      double remain = re + dt_mix, time = -re;
      while (remain > 0.0) {
        double PGn = PGp;
        double PL = PC2 * time * time + PC1 * time + PC0;
        rp_substep_refined(Rt, Rp, Rn, d1R, PGn, PL, dtL, remain, b, param);
        time = time + dtL;
        Cplx alpha;
        double omega = thermal_omega(alpha, PGn, Rn, b);
        Cplx lp = thermal_lp(alpha, Rn);
        PGp = gas_pressure(PGn, Rp, Rn, omega, dtL, lp, b);
        total++;
        if (total > 100000000) return -1;
      }
      re = remain;
    }
    R_out[s] = Rt;
    PG_out[s] = PGp;
  }
  return total;
}

crp_status crpo_host_sigma(const crp_config* cfg, double* mx, double* my, double* nx, double* ny, double* xu,
                           double* rxp) {
  Index a = make_index(cfg->grid_x, cfg->grid_y, cfg->sim_order);
  Derived d = derive(*cfg);
  std::vector<double> vmx, vmy, vnx, vny;
  make_sigma(*cfg, a, d, vmx, vmy, vnx, vny);
  std::memcpy(mx, vmx.data(), sizeof(double) * vmx.size());
  std::memcpy(my, vmy.data(), sizeof(double) * vmy.size());
  std::memcpy(nx, vnx.data(), sizeof(double) * vnx.size());
  std::memcpy(ny, vny.data(), sizeof(double) * vny.size());
  for (int i = a.ista2n; i <= a.iend2n; i++) xu[i - a.ista2n] = ((double)i) * d.dx;
  for (int i = a.ista2m; i <= a.iend2m; i++) rxp[i - a.ista2m] = 1.0 / (d.dx * ((double)i - 0.5));
  return CRP_OK;
}

}  // extern "C"

// The 3-D Cartesian extension.
namespace {
void philox_block(uint64_t seed, uint64_t counter, uint32_t stream, uint32_t out[4]) {
  crpo_philox_block(seed, counter, stream, out);
}
}  // namespace
#include "oracle3d.inc"
