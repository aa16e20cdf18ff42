// Dormand-Prince 5(4) integration of a bubble over one mixture step
// (ext.rp_scheme = rk45).
//
// The reference advances each bubble with a three-level variable-step scheme
// whose step is capped by a 1 % radius change and a 1 % growth per step
// (inc/bubble_CUDA_kernel.cuh:227-260); near a collapse that takes thousands
// of steps per mixture step.  This scheme integrates the same model with an
// embedded error estimate instead, so its steps follow the solution's own
// scales:
//
//   R'  = V
//   V'  = ((PG - PL(t) - 2 sigma / R - 4 mu V / R) / rho - 3/2 V^2) / R
//   PG' = [ -3 gam PG V / R + (K / R) (Lr (PG0 - x^3 PG) + (Li / omega) 3 x^2 (V / R0) PG) ]
//         / (1 - (K / R) (Li / omega) x^3),
//
// x = R / R0, K = 3 (gam - 1) K0 T0 / PG0, (Lr, Li) = conj-free parts of 1 / Lp
// (Re Lp / |Lp|^2, Im Lp / |Lp|^2), omega and Lp from the reference's thermal
// model at (PG, R) (solveOmegaN and solveLp, :263-323).  The PG' equation is
// the dt -> 0 limit of the reference's semi-implicit gas-pressure update
// (solvePG, :326-340): dividing its c1 PG^{n+1} = c2 PG^n + c0 Lr PG0 by dt
// gives PG' + 3 gam PG V / R + (K / R) Lr x^3 PG - (K / R)(Li / omega) (x^3 PG)' =
// (K / R) Lr PG0, solved here for PG'.  PL(t) is the reference's quadratic in
// time through the gathered liquid pressures of the last three steps
// (:497-499).  The heat and viscous power of the bubble (:521-536) in the same
// continuous form, -4 pi R^2 K0 dT/dr + 16 pi mu R V^2 with
// dT/dr = T0 / (PG0 R0^3) (Lr (PG0 R0^3 - PG R^3) + (Li / omega) (PG R^3)'),
// is integrated with the stages' weights; Q_B is its mean over the step.
//
// Steps: the Dormand-Prince pair (Dormand & Prince 1980) with its
// first-same-as-last stage, the error of each component scaled by
// rtol max(|y|, |y_new|) (plus rtol x 1 m/s for V, which passes through 0),
// the max norm, accepted when <= 1; the next step h 0.9 err^(-1/5) within
// [0.2 h, 5 h] (at most h after a rejection).  The last step of a mixture step
// ends exactly on it, so nothing carries over (the reference's remainder `re`
// is 0).  The thermal model runs in the type T; the mixed path passes FP32,
// and the thermal model runs in FP64 all the same in the stiff phase
// (R < 0.3 R0 or |V| > 0.1 c_inf) and once R leaves R0 by more than 0.1 %.
#pragma once

namespace crp {

struct RkState {
  double R, V, PG;       // state at local time t
  double fR, fV, fPG;    // its derivative (first-same-as-last)
  double qd;             // heat + viscous power at t
  double t, tend, h;     // local time from the start of the mixture step, its end, trial step
  double Q;              // integral of the power over [0, t]
  double PC0, PC1, PC2;  // liquid pressure PC2 t^2 + PC1 t + PC0
  double K;              // 3 (gam - 1) K0 T0 / PG0
  BubbleR0 r;
  long long count;       // step attempts
  bool fresh;            // the derivative at t is still to be evaluated
};

struct RkDeriv {
  double R, V, PG, q;
};

// Right-hand side at local time t and state (R, V, PG); the thermal model in T.
template <typename T>
__device__ __forceinline__ RkDeriv rk_rhs_t(const BubbleParams& bp, const RkState& s, double t, double R, double V,
                                            double PG) {
  const double PL = s.PC2 * t * t + s.PC1 * t + s.PC0;
  const double inv_R = 1.0 / R;
  RkDeriv d;
  d.R = V;
  d.V = ((PG - PL - 2.0 * bp.sig * inv_R - 4.0 * bp.mu * inv_R * V) * bp.inv_rho - 1.5 * V * V) * inv_R;
  Cx<T> alpha;
  ThermalConst<T> c;
  if constexpr (sizeof(T) == sizeof(double))
    c = thermal_const64(bp, s.r);
  else
    c = thermal_const32(bp, s.r);
  const double omega = (double)omega_n<T>(alpha, (T)PG, (T)R, c);
  const Cx<T> lpt = lp_n<T>(alpha, (T)R, c.cut2);
  const double lr = (double)lpt.re, li = (double)lpt.im;
  const double inv_den = 1.0 / (lr * lr + li * li);
  const double Lr = lr * inv_den, Liw = li * inv_den / omega;
  const double x = R * s.r.inv_R0, x2 = x * x, x3 = x2 * x;
  const double KR = s.K * inv_R;
  const double num = -3.0 * bp.gam * PG * V * inv_R + KR * (Lr * (s.r.PG0 - x3 * PG) + Liw * 3.0 * x2 * V * s.r.inv_R0 * PG);
  d.PG = num / (1.0 - KR * Liw * x3);
  const double R2 = R * R, R3 = R2 * R;
  const double dTdr = s.r.T0_PG0R03 * (Lr * (s.r.PG0 * s.r.R03 - PG * R3) + Liw * (R3 * d.PG + 3.0 * R2 * V * PG));
  d.q = -4.0 * bp.pi * R2 * bp.K0 * dTdr + 16.0 * bp.pi * bp.mu * R * V * V;
  return d;
}

// The thermal model's type: T, except FP64 whenever T is FP32 and the bubble
// is in the stiff phase (R < 0.3 R0 or |V| > 0.1 c_inf) or has left its
// equilibrium radius by more than kRkFp32Excursion.  Measured on the driven
// test cases: an FP32 thermal model outside the stiff phase alone left the gas
// pressure 1.3e-3 from the FP64 oracle (through the PG' denominator); near
// equilibrium its rounding stays below the scheme's tolerance.
constexpr double kRkFp32Excursion = 1.0e-3;

template <typename T>
__device__ __forceinline__ RkDeriv rk_rhs(const BubbleParams& bp, const RkState& s, double t, double R, double V,
                                          double PG, double c_inf) {
  if constexpr (sizeof(T) == sizeof(double)) {
    return rk_rhs_t<double>(bp, s, t, R, V, PG);
  } else {
    const bool stiff = R < 0.3 * s.r.R0 || fabs(V) > 0.1 * c_inf;
    if (stiff || fabs(R - s.r.R0) > kRkFp32Excursion * s.r.R0) return rk_rhs_t<double>(bp, s, t, R, V, PG);
    return rk_rhs_t<float>(bp, s, t, R, V, PG);
  }
}

// One step attempt; returns false when the step size has collapsed (an
// error: the caller flags it as a sub-step cap).
template <typename T>
__device__ __forceinline__ bool rk_attempt(const BubbleParams& bp, RkState& s, double rtol, double c_inf) {
  // Dormand-Prince 5(4) tableau (Dormand & Prince 1980).
  constexpr double c2 = 1.0 / 5.0, c3 = 3.0 / 10.0, c4 = 4.0 / 5.0, c5 = 8.0 / 9.0;
  constexpr double a21 = 1.0 / 5.0;
  constexpr double a31 = 3.0 / 40.0, a32 = 9.0 / 40.0;
  constexpr double a41 = 44.0 / 45.0, a42 = -56.0 / 15.0, a43 = 32.0 / 9.0;
  constexpr double a51 = 19372.0 / 6561.0, a52 = -25360.0 / 2187.0, a53 = 64448.0 / 6561.0, a54 = -212.0 / 729.0;
  constexpr double a61 = 9017.0 / 3168.0, a62 = -355.0 / 33.0, a63 = 46732.0 / 5247.0, a64 = 49.0 / 176.0,
                   a65 = -5103.0 / 18656.0;
  constexpr double b1 = 35.0 / 384.0, b3 = 500.0 / 1113.0, b4 = 125.0 / 192.0, b5 = -2187.0 / 6784.0,
                   b6 = 11.0 / 84.0;
  constexpr double e1 = 71.0 / 57600.0, e3 = -71.0 / 16695.0, e4 = 71.0 / 1920.0, e5 = -17253.0 / 339200.0,
                   e6 = 22.0 / 525.0, e7 = -1.0 / 40.0;
  if (s.fresh) {
    const RkDeriv d = rk_rhs<T>(bp, s, s.t, s.R, s.V, s.PG, c_inf);
    s.fR = d.R;
    s.fV = d.V;
    s.fPG = d.PG;
    s.qd = d.q;
    s.fresh = false;
  }
  const double rem = s.tend - s.t;
  double h = s.h;
  bool last = false;
  if (h >= rem || 1.01 * h >= rem) {
    h = rem;
    last = true;
  }
  s.count++;
  const double t = s.t;
  const RkDeriv k1{s.fR, s.fV, s.fPG, s.qd};
  const RkDeriv k2 = rk_rhs<T>(bp, s, t + c2 * h, s.R + h * (a21 * k1.R), s.V + h * (a21 * k1.V),
                               s.PG + h * (a21 * k1.PG), c_inf);
  const RkDeriv k3 = rk_rhs<T>(bp, s, t + c3 * h, s.R + h * (a31 * k1.R + a32 * k2.R),
                               s.V + h * (a31 * k1.V + a32 * k2.V), s.PG + h * (a31 * k1.PG + a32 * k2.PG), c_inf);
  const RkDeriv k4 = rk_rhs<T>(bp, s, t + c4 * h, s.R + h * (a41 * k1.R + a42 * k2.R + a43 * k3.R),
                               s.V + h * (a41 * k1.V + a42 * k2.V + a43 * k3.V),
                               s.PG + h * (a41 * k1.PG + a42 * k2.PG + a43 * k3.PG), c_inf);
  const RkDeriv k5 = rk_rhs<T>(bp, s, t + c5 * h, s.R + h * (a51 * k1.R + a52 * k2.R + a53 * k3.R + a54 * k4.R),
                               s.V + h * (a51 * k1.V + a52 * k2.V + a53 * k3.V + a54 * k4.V),
                               s.PG + h * (a51 * k1.PG + a52 * k2.PG + a53 * k3.PG + a54 * k4.PG), c_inf);
  const RkDeriv k6 =
      rk_rhs<T>(bp, s, t + h, s.R + h * (a61 * k1.R + a62 * k2.R + a63 * k3.R + a64 * k4.R + a65 * k5.R),
                s.V + h * (a61 * k1.V + a62 * k2.V + a63 * k3.V + a64 * k4.V + a65 * k5.V),
                s.PG + h * (a61 * k1.PG + a62 * k2.PG + a63 * k3.PG + a64 * k4.PG + a65 * k5.PG), c_inf);
  const double Rn = s.R + h * (b1 * k1.R + b3 * k3.R + b4 * k4.R + b5 * k5.R + b6 * k6.R);
  const double Vn = s.V + h * (b1 * k1.V + b3 * k3.V + b4 * k4.V + b5 * k5.V + b6 * k6.V);
  const double PGn = s.PG + h * (b1 * k1.PG + b3 * k3.PG + b4 * k4.PG + b5 * k5.PG + b6 * k6.PG);
  bool finite = Rn > 0.0 && PGn > 0.0 && isfinite(Rn) && isfinite(Vn) && isfinite(PGn);
  RkDeriv k7{0.0, 0.0, 0.0, 0.0};
  double err = 1.0e30;
  if (finite) {
    k7 = rk_rhs<T>(bp, s, t + h, Rn, Vn, PGn, c_inf);
    const double eR = h * (e1 * k1.R + e3 * k3.R + e4 * k4.R + e5 * k5.R + e6 * k6.R + e7 * k7.R);
    const double eV = h * (e1 * k1.V + e3 * k3.V + e4 * k4.V + e5 * k5.V + e6 * k6.V + e7 * k7.V);
    const double eP = h * (e1 * k1.PG + e3 * k3.PG + e4 * k4.PG + e5 * k5.PG + e6 * k6.PG + e7 * k7.PG);
    const double sR = rtol * fmax(fabs(s.R), fabs(Rn));
    const double sV = rtol * (fmax(fabs(s.V), fabs(Vn)) + 1.0);
    const double sP = rtol * fmax(fabs(s.PG), fabs(PGn));
    err = fmax(fabs(eR) / sR, fmax(fabs(eV) / sV, fabs(eP) / sP));
    if (!isfinite(err)) err = 1.0e30;
  }
  double fac = err > 0.0 ? 0.9 * pow(err, -0.2) : 5.0;
  if (err <= 1.0) {
    s.Q += h * (b1 * k1.q + b3 * k3.q + b4 * k4.q + b5 * k5.q + b6 * k6.q);
    s.R = Rn;
    s.V = Vn;
    s.PG = PGn;
    s.fR = k7.R;
    s.fV = k7.V;
    s.fPG = k7.PG;
    s.qd = k7.q;
    s.t = last ? s.tend : t + h;
    fac = fmin(5.0, fmax(0.2, fac));
    // A clipped last step does not shrink the step the next mixture step starts from.
    s.h = last ? fmax(s.h, h * fac) : h * fac;
  } else {
    s.h = h * fmin(1.0, fmax(0.2, fac));
  }
  return s.h > 1.0e-22;
}

}  // namespace crp
