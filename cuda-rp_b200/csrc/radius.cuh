// The per-bubble radius solve of the reference scheme shared by the 2-D and
// 3-D paths: the sub-step state of BubbleRadiusKernel and one pass of its
// sub-step loop (inc/bubble_CUDA_kernel.cuh:471-554).
#pragma once
#include "crp_device.cuh"

namespace crp {

// Per-bubble state of BubbleRadiusKernel (inc/bubble_CUDA_kernel.cuh:471-554)
// while its sub-steps run.
struct RpState {
  double Rt, Rp, Rn, d1Rp, PGp, dtL, remain, time, PC0, PC1, PC2, heat, vis, re_n;
  BubbleR0 r;
  long long count;
};

// One pass of the sub-step loop of BubbleRadiusKernel (:506-539).  T is the
// real type of the thermal model (omega_N, alpha_N, Lp_N); everything else is FP64.
template <typename T>
__device__ __forceinline__ void thermal_model(const BubbleParams& bp, const RpState& s, double PGn, double& omega,
                                              C64& lp) {
  Cx<T> alpha_t;
  ThermalConst<T> c;
  if constexpr (sizeof(T) == sizeof(double))
    c = thermal_const64(bp, s.r);
  else
    c = thermal_const32(bp, s.r);
  omega = (double)omega_n<T>(alpha_t, (T)PGn, (T)s.Rn, c);
  const Cx<T> lp_t = lp_n<T>(alpha_t, (T)s.Rn, c.cut2);
  lp = C64{(double)lp_t.re, (double)lp_t.im};
}

// Relative radius excursion |R/R0 - 1| above which the mixed path evaluates
// the thermal model in FP64: FP32 is accurate for the small oscillations of a
// quiet bubble, and its rounding is amplified once the bubble is driven.
constexpr double kThermalFp64Excursion = 1.0e-3;

template <typename T>
__device__ __forceinline__ void rp_substep_full(const BubbleParams& bp, RpState& s) {
  const double PGn = s.PGp;
  const double PL = s.PC2 * s.time * s.time + s.PC1 * s.time + s.PC0;
  rp_substep(s.Rt, s.Rp, s.Rn, s.d1Rp, PGn, PL, s.dtL, s.remain, bp);
  s.time = s.time + s.dtL;
  double omega;
  C64 lp;
  if (sizeof(T) == sizeof(double) || fabs(s.Rn - s.r.R0) > kThermalFp64Excursion * s.r.R0)
    thermal_model<double>(bp, s, PGn, omega, lp);
  else
    thermal_model<T>(bp, s, PGn, omega, lp);
  const double den = lp.re * lp.re + lp.im * lp.im;
  const double inv_wdt = 1.0 / (omega * s.dtL);
  s.PGp = gas_pressure(PGn, s.Rp, s.Rn, inv_wdt, s.dtL, den, lp, bp, s.r);
  const double inv_den = 1.0 / den;  // for the heat flux only, off the chain to the next sub-step
  const double Rp = s.Rp, Rn = s.Rn, PGp = s.PGp;
  const double s0 = 0.5 * (Rp + Rn);
  const double s1 = inv_den * s.r.T0_PG0R03;
  const double dTdr = lp.re * s1 * (s.r.PG0 * s.r.R03 - 0.5 * (PGp + PGn) * s0 * s0 * s0) +
                      lp.im * s1 * (PGp * Rp * Rp * Rp - PGn * Rn * Rn * Rn) * inv_wdt;
  s.heat -= 4.0 * bp.pi * Rp * Rp * bp.K0 * dTdr * s.dtL;
  // 4 pi Rp^2 (4 mu d1Rp / Rp) d1Rp dt, with Rp^2 / Rp cancelled.
  s.vis += 4.0 * bp.pi * Rp * 4.0 * bp.mu * s.d1Rp * s.d1Rp * s.dtL;
  s.count++;
}

}  // namespace crp
