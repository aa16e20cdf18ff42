// The 3-D Cartesian simulation (ext.grid_z > 0): the same bubbly-mixture
// model as the 2-D path on a staggered grid of X x Y x Z cells, with a PML on
// all six faces and a hemispherical phased array as its source.  The
// reference is 2-D only; each of its formulas gains its third component:
// VelocityKernel and MixturePressureKernel (inc/bubble_CUDA_kernel.cuh:635-677,
// 816-867) for vz and pz, init_sigma's profiles per axis, the smooth delta
// (:214-222) and the bubble stencils (:361-448, :576-619) over 2 x 2 x 2
// cells.  oracle/oracle3d.inc restates every step on the host.
//
// Kernels of one mixture step:
//   fdtd3        fused velocity update (three faces per cell), void-fraction
//                prediction, split-pressure update, source forcing and
//                residual; a 32 x 8 block of threads holds a 30 x 6 patch of
//                cells (and a ring of halo cells) and marches along z, the face
//                below in registers, x-neighbours by shuffle, y-neighbours
//                through shared memory: one pass over the state
//   move3        bubble state rotation, velocity gather over the staggered
//                2 x 2 x 2 stencils, motion, cell indices, bounding box
//   bin3_*       counting sort of bubbles by cell (when a bubble changed cell)
//   rp3 / rk3    pressure gather + radius solve (reference scheme or rk45) +
//                the eight void-fraction contributions of each bubble,
//                persistent with a work queue
//   couple3      per-cell gather of the void fraction from its eight bins,
//                pressure re-evaluation, source forcing, residual, over the
//                box where the void fraction can be nonzero
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "crp.h"
#include "crp_device.cuh"
#include "radius.cuh"
#include "rk45.cuh"
#include "lpt.cuh"
#include "sim3d.h"

namespace crp {

void philox_block(uint64_t seed, uint64_t counter, uint32_t stream, uint32_t out[4]);

namespace d3 {

struct Frame3 {
  int X, Y, Z, pitch;
  __host__ __device__ __forceinline__ long idx(int i, int j, int k) const {
    return ((long)(k + 1) * (Y + 4) + (j + 1)) * pitch + (i + 1);
  }
};

// Grid, PML and source parameters of the kernels.
struct Grid3 {
  Frame3 f;
  double dx, dy, dz, rdx, rdy, rdz, dt;
  double rho_inf, c_inf, P_inf;
  double dt_rho, s3p;  // dt / rho_inf, dt rho_inf c_inf^2
  // PML factors 1 - s and 1 / (1 + s): faces va?/vb?[n + 1], n in [-1, N+1];
  // cells pa?/pb?[n], n in [0, N+1].
  const double *vax, *vbx, *vay, *vby, *vaz, *vbz, *pax, *pbx, *pay, *pby, *paz, *pbz;
  const short* src;  // element + 1 of every frame cell, 0 = not a source cell
  const double* elem_amp;
  const double* elem_phase;
  double pamp, omega, period, on_time, ramp_time;
};

__device__ __forceinline__ double burst_env(const Grid3& g, double tau) {
  if (!(g.ramp_time > 0.0)) return 1.0;
  const double pi = 3.14159265358979323846;
  double w = 1.0;
  if (tau < g.ramp_time) w = fmin(w, 0.5 * (1.0 - cos(pi * tau / g.ramp_time)));
  const double rest = g.on_time - tau;
  if (rest < g.ramp_time) w = fmin(w, rest > 0.0 ? 0.5 * (1.0 - cos(pi * rest / g.ramp_time)) : 0.0);
  return w;
}

// Pressure of element e at time t (0 at t = 0 and outside the burst).
__device__ __noinline__ double element_pressure(const Grid3& g, int e, double t) {
  if (!(t > 0.0)) return 0.0;
  const double tau = fmod(t, g.period);
  if (!(tau <= g.on_time)) return 0.0;
  return g.pamp * g.elem_amp[e] * burst_env(g, tau) * sin(g.omega * t + g.elem_phase[e]);
}

__device__ __forceinline__ double face_q3(const Grid3& g, double ra, double rb) {
  return (ra == g.rho_inf && rb == g.rho_inf) ? g.dt_rho : g.dt / ((ra + rb) * 0.5);
}
// (v_old (1 - s3) - dt / mean(rho) (p0b - p0a) / h) / (1 + s3), with the face's
// PML factors fa = 1 - s3 and fb = 1 / (1 + s3).
__device__ __forceinline__ double face3(double v_old, double p0a, double p0b, double q, double rh, double fa,
                                        double fb) {
  return (v_old * fa - q * ((-p0a + p0b) * rh)) * fb;
}
__device__ __forceinline__ double void_half3(const Grid3& g, double fg, double fgn) {
  if (fg == 0.0 && fgn == 0.0) return 0.0;
  return 0.5 * (-(fg - fgn) / g.dt / (1.0 - 0.5 * (fg + fgn)));
}

template <typename P>
struct Fdtd3Args {
  typename P::V vx_old, vy_old, vz_old, vx_new, vy_new, vz_new;
  typename P::S pnx, pny, pnz, px, py, pz;
  typename P::G fgA, fgB, fgC;  // f_g, f_gn, f_gm of the previous step; fgC receives the prediction
  const double* tdev;           // {t_prev, t_cur}
  int rho_const;
  unsigned long long* residual;
};

constexpr int kTX = 32, kTY = 8;   // threads per block
constexpr int kCX = 30, kCY = 6;   // cells updated per block
constexpr int kZChunk = 32;        // planes per block
constexpr int kStages3 = 4;        // ring slots (planes) per thread
constexpr int kFields3 = 9;        // pnx, pny, pnz, fgA, vx_old, vy_old, vz_old, fgB, fgC
constexpr size_t kRing3Bytes = sizeof(double) * kStages3 * kFields3 * kTX * kTY;

// Each thread's inputs of plane k0 - 1 + r are staged in ring slot r % kStages3
// (dynamic shared memory, one 8-byte element per thread and field) by
// asynchronous copies issued kStages3 - 2 planes ahead, so the loads of the
// next planes are in flight while a plane is computed.
template <typename P>
__global__ void __launch_bounds__(kTX* kTY, 2) fdtd3(const __grid_constant__ Grid3 g, const Fdtd3Args<P> a) {
  using G = typename P::G;
  using S = typename P::S;
  using V = typename P::V;
  __shared__ double s_p0[2][kTY][kTX], s_rho[2][kTY][kTX], s_vy[2][kTY][kTX];
  extern __shared__ __align__(16) double ring3[];  // [kStages3][kFields3][kTY * kTX]
  const Frame3& f = g.f;
  const int X = f.X, Y = f.Y, Z = f.Z;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = blockIdx.x * kCX + tx, j = blockIdx.y * kCY + ty;
  const int k0 = 1 + blockIdx.z * kZChunk, k1 = min(Z, k0 + kZChunk - 1);
  const bool upd = tx >= 1 && tx <= kCX && ty >= 1 && ty <= kCY && i <= X && j <= Y;
  const int il = min(i, X + 1), jl = min(j, Y + 1);  // loads of threads past the window repeat the edge
  const double t_cur = a.tdev[1];
  const unsigned full = 0xffffffffu;
  auto rho_of = [&](double fa) { return a.rho_const ? g.rho_inf : (1.0 - fa) * g.rho_inf; };
  auto predict = [&](int ii, int jj, int kk) {
    const long q = f.idx(ii, jj, kk);
    const double v = G::stored(3.0 * a.fgA.get(q) - 3.0 * a.fgB.get(q) + a.fgC.get(q));
    a.fgC.put(q, v);
    return v;
  };
  const double vax = g.vax[il + 1], vbx = g.vbx[il + 1], vay = g.vay[jl + 1], vby = g.vby[jl + 1];
  const double pax = g.pax[il], pbx = g.pbx[il], pay = g.pay[jl], pby = g.pby[jl];

  const int tid = ty * kTX + tx;
  auto slot = [&](int r, int fld) -> double* { return &ring3[((r % kStages3) * kFields3 + fld) * (kTX * kTY) + tid]; };
  const long qb = f.idx(il, jl, k0 - 1), plane = (long)(Y + 4) * f.pitch;
  // Queue the copies of plane kk = k0 - 1 + r: pnx, pny, pnz, fgA for planes
  // k0-1..k1+1, vz_old for k0-1..k1, vx_old, vy_old, fgB, fgC for k0..k1.  One
  // commit group per plane, empty past the chunk, so that a fixed wait count
  // always means "the next plane landed".
  auto issue = [&](int r) {
    const int kk = k0 - 1 + r;
    if (kk <= k1 + 1) {
      const long q = qb + r * plane;
      a.pnx.stage(slot(r, 0), q);
      a.pny.stage(slot(r, 1), q);
      a.pnz.stage(slot(r, 2), q);
      a.fgA.stage(slot(r, 3), q);
      if (kk <= k1) {
        a.vz_old.stage(slot(r, 6), q);
        if (r >= 1) {
          a.vx_old.stage(slot(r, 4), q);
          a.vy_old.stage(slot(r, 5), q);
          a.fgB.stage(slot(r, 7), q);
          a.fgC.stage(slot(r, 8), q);
        }
      }
    }
    __pipeline_commit();
  };
#pragma unroll
  for (int r = 0; r < kStages3; r++) issue(r);
  __pipeline_wait_prior(kStages3 - 2);  // planes k0 - 1 and k0 have landed

  // The face below the first plane, vz(i, j, k0 - 1), from planes k0 - 1 and k0.
  double p0c, rhoc, fb, pxc, pyc, pzc, fac;
  {
    const double pxb = S::staged(slot(0, 0)), pyb = S::staged(slot(0, 1)), pzb = S::staged(slot(0, 2));
    const double fab = G::staged(slot(0, 3)), vz_old_b = V::staged(slot(0, 6));
    pxc = S::staged(slot(1, 0));
    pyc = S::staged(slot(1, 1));
    pzc = S::staged(slot(1, 2));
    fac = G::staged(slot(1, 3));
    const double p0b = pxb + pyb + pzb, rhob = rho_of(fab);
    p0c = pxc + pyc + pzc;
    rhoc = rho_of(fac);
    fb = face3(vz_old_b, p0b, p0c, face_q3(g, rhob, rhoc), g.rdz, g.vaz[k0], g.vbz[k0]);
    if (k0 == 1 && upd) a.vz_new.put(f.idx(i, j, 0), fb);
  }
  issue(kStages3);  // reuses the slot of plane k0 - 1
  int src_e = g.src[qb + plane];  // source element + 1 of plane k0
  unsigned long long res = 0ull;
  int buf = 0;
#pragma unroll 1
  for (int k = k0; k <= k1; k++) {
    const int r = k - k0 + 1;
    __pipeline_wait_prior(kStages3 - 2);  // plane k + 1 has landed
    // Next plane.
    const double pxn = S::staged(slot(r + 1, 0)), pyn = S::staged(slot(r + 1, 1)), pzn = S::staged(slot(r + 1, 2));
    const double fan = G::staged(slot(r + 1, 3));
    const double p0n = pxn + pyn + pzn, rhon = rho_of(fan);
    // This plane's old faces and void-fraction history.
    const double vxo = V::staged(slot(r, 4)), vyo = V::staged(slot(r, 5)), vzo = V::staged(slot(r, 6));
    const double fgB = G::staged(slot(r, 7)), fgC = G::staged(slot(r, 8));
    issue(r + kStages3);  // reuses the slot of plane k
    const int e = src_e;
    if (k < k1) src_e = g.src[qb + (long)(r + 1) * plane];
    s_p0[buf][ty][tx] = p0c;
    s_rho[buf][ty][tx] = rhoc;
    __syncthreads();
    const double p0r = __shfl_down_sync(full, p0c, 1), rhor = __shfl_down_sync(full, rhoc, 1);
    const double p0u = s_p0[buf][min(ty + 1, kTY - 1)][tx], rhou = s_rho[buf][min(ty + 1, kTY - 1)][tx];
    const double fe = face3(vxo, p0c, p0r, face_q3(g, rhoc, rhor), g.rdx, vax, vbx);
    const double fn = face3(vyo, p0c, p0u, face_q3(g, rhoc, rhou), g.rdy, vay, vby);
    const double ft = face3(vzo, p0c, p0n, face_q3(g, rhoc, rhon), g.rdz, g.vaz[k + 1], g.vbz[k + 1]);
    s_vy[buf][ty][tx] = fn;
    __syncthreads();
    const double fw = __shfl_up_sync(full, fe, 1);
    const double fs = s_vy[buf][max(ty - 1, 0)][tx];
    if (upd) {
      const long o = f.idx(i, j, k);
      a.vx_new.put(o, fe);
      a.vy_new.put(o, fn);
      a.vz_new.put(o, ft);
      const double fgp = G::stored(3.0 * fac - 3.0 * fgB + fgC);
      a.fgC.put(o, fgp);
      // Ghost cells next to the domain's faces take their prediction from
      // the cell beside them (every combination of the faces it touches).
      const int gi = i == 1 ? 0 : (i == X ? X + 1 : -2);
      const int gj = j == 1 ? 0 : (j == Y ? Y + 1 : -2);
      const int gk = k == 1 ? 0 : (k == Z ? Z + 1 : -2);
      if (gi > -2 || gj > -2 || gk > -2) {
        for (int ci = 0; ci < 2; ci++)
          for (int cj = 0; cj < 2; cj++)
            for (int ck = 0; ck < 2; ck++) {
              if (!(ci || cj || ck)) continue;
              if ((ci && gi == -2) || (cj && gj == -2) || (ck && gk == -2)) continue;
              predict(ci ? gi : i, cj ? gj : j, ck ? gk : k);
            }
      }
      const double h = void_half3(g, fgp, fac);
      const double qx = pxc * pax - g.s3p * ((-fw + fe) * g.rdx + h) * pbx;
      const double qy = pyc * pay - g.s3p * ((-fs + fn) * g.rdy + h) * pby;
      const double qz = pzc * g.paz[k] - g.s3p * ((-fb + ft) * g.rdz + h) * g.pbz[k];
      double p0new = qx + qy + qz;
      if (e > 0) {
        p0new = element_pressure(g, e - 1, t_cur);
        a.px.put(o, p0new);
        a.py.put(o, 0.0);
        a.pz.put(o, 0.0);
      } else {
        a.px.put(o, qx);
        a.py.put(o, qy);
        a.pz.put(o, qz);
      }
      res = max(res, (unsigned long long)__double_as_longlong(fabs(p0c - p0new)));
    }
    // The x0 and y0 faces of the domain belong to the threads on the ghost cells.
    if (i == 0 && ty >= 1 && ty <= kCY && j <= Y) a.vx_new.put(f.idx(0, j, k), fe);
    if (j == 0 && tx >= 1 && tx <= kCX && i <= X) a.vy_new.put(f.idx(i, 0, k), fn);
    fb = ft;
    pxc = pxn;
    pyc = pyn;
    pzc = pzn;
    fac = fan;
    p0c = p0n;
    rhoc = rhon;
    buf ^= 1;
  }
  for (int o = 16; o > 0; o >>= 1) res = max(res, __shfl_xor_sync(full, res, o));
  if (tx == 0 && res) atomicMax(a.residual, res);
}

// ---------------------------------------------------------------------------
// Bubbles.

struct Bub3 {
  int n;
  double *x, *y, *z, *R0, *n_B, *R_t, *R_p, *R_pn, *R_n, *R_nn, *d1_R_p, *d1_R_n, *PG_p, *PG_n, *PL_p, *PL_n,
      *PL_m, *Q_B, *dt, *dt_n, *re, *re_n, *vbx, *vby, *vbz, *contrib;
  int *ibmx, *ibmy, *ibmz, *ibnx, *ibny, *ibnz, *bin, *nsub, *pos;
};

struct Scalars3 {
  unsigned long long residual;
  long long substep_max;
  int err;
  int next;
  int moved;
  int box[6];  // bubbles' ibn box: min x, y, z, max x, y, z
  double t[2];
  unsigned long long reused;  // radius solves kept (ext.rp_reuse), summed over the handle's life
};

__global__ void set_time3(Scalars3* s, double t_prev, double t) {
  s->t[0] = t_prev;
  s->t[1] = t;
  s->residual = 0ull;
  s->moved = 0;
  s->box[0] = s->box[1] = s->box[2] = INT_MAX;
  s->box[3] = s->box[4] = s->box[5] = INT_MIN;
}

__device__ __forceinline__ int bin3_of(const Frame3& f, int ix, int iy, int iz) {
  if (ix < -1 || ix > f.X + 1 || iy < -1 || iy > f.Y + 1 || iz < -1 || iz > f.Z + 1) return -1;
  return ((iz + 1) * (f.Y + 3) + (iy + 1)) * (f.X + 3) + (ix + 1);
}

__device__ __forceinline__ double dcos(const BubbleParams& bp, double c, int pos, double h, double b) {
  return cos(c * (((double)pos - 0.5) * h - b));
}

__device__ __forceinline__ void index3(const Grid3& g, Bub3& b, int n) {
  const double x = b.x[n], y = b.y[n], z = b.z[n];
  b.ibmx[n] = (int)floor(x * g.rdx + 1.0);
  b.ibmy[n] = (int)floor(y * g.rdy + 1.0);
  b.ibmz[n] = (int)floor(z * g.rdz + 1.0);
  b.ibnx[n] = (int)floor(x * g.rdx + 0.5);
  b.ibny[n] = (int)floor(y * g.rdy + 0.5);
  b.ibnz[n] = (int)floor(z * g.rdz + 0.5);
}

__global__ void index3_kernel(const __grid_constant__ Grid3 g, Bub3 b, Scalars3* s) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= b.n) return;
  index3(g, b, n);
  b.bin[n] = bin3_of(g.f, b.ibnx[n], b.ibny[n], b.ibnz[n]);
  atomicMin(&s->box[0], b.ibnx[n]);
  atomicMin(&s->box[1], b.ibny[n]);
  atomicMin(&s->box[2], b.ibnz[n]);
  atomicMax(&s->box[3], b.ibnx[n]);
  atomicMax(&s->box[4], b.ibny[n]);
  atomicMax(&s->box[5], b.ibnz[n]);
}

// Velocity of a staggered component at the bubble: points i in ia + {0, 1},
// j in ja + {0, 1}, k in ka + {0, 1} of the array V whose logical window is
// [ilo, ihi] x [jlo, jhi] x [klo, khi].
template <typename V>
__device__ __forceinline__ double gather_v(const Grid3& g, const BubbleParams& bp, const V& v, int ia, int ja, int ka,
                                           double x, double y, double z, int ilo, int ihi, int jlo, int jhi, int klo,
                                           int khi) {
  const double cx = dcos(bp, bp.dcy, ia, g.dx, x), cy = dcos(bp, bp.dcz, ja, g.dy, y);
  const double cz = cos(2.0 * bp.pi / 2.0 * g.rdz * (((double)ka - 0.5) * g.dz - z));
  double s = 0.0;
  for (int ci = 0; ci < 2; ci++) {
    const int i = ia + ci;
    const double wx = delta_w(bp, cx, ci);
    for (int cj = 0; cj < 2; cj++) {
      const int j = ja + cj;
      const double wy = delta_w(bp, cy, cj);
      for (int ck = 0; ck < 2; ck++) {
        const int k = ka + ck;
        if (i >= ilo && i <= ihi && j >= jlo && j <= jhi && k >= klo && k <= khi)
          s += v.get(g.f.idx(i, j, k)) * wx * wy * delta_w(bp, cz, ck);
      }
    }
  }
  return s;
}

// store_variables' rotation of the bubble state, the velocity gather
// (BubbleInterpolationVelocityKernel, :398-448, with its z component), the
// motion (BubbleMotionKernel, :451-468) and the new cell indices.
template <typename V>
__global__ void move3(const __grid_constant__ Grid3 g, const __grid_constant__ BubbleParams bp, Bub3 b, const V vx,
                      const V vy, const V vz, Scalars3* s) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= b.n) return;
  b.R_pn[n] = b.R_p[n];
  b.R_nn[n] = b.R_n[n];
  b.d1_R_n[n] = b.d1_R_p[n];
  b.PG_n[n] = b.PG_p[n];
  b.PL_m[n] = b.PL_n[n];
  b.PL_n[n] = b.PL_p[n];
  b.dt_n[n] = b.dt[n];
  b.re_n[n] = b.re[n];
  const Frame3& f = g.f;
  const double x = b.x[n], y = b.y[n], z = b.z[n];
  const int mx = b.ibmx[n], my = b.ibmy[n], mz = b.ibmz[n], nx = b.ibnx[n], ny = b.ibny[n], nz = b.ibnz[n];
  const double ux = gather_v(g, bp, vx, mx - 1, ny, nz, x, y, z, -1, f.X + 1, 0, f.Y + 1, 0, f.Z + 1);
  const double uy = gather_v(g, bp, vy, nx, my - 1, nz, x, y, z, 0, f.X + 1, -1, f.Y + 1, 0, f.Z + 1);
  const double uz = gather_v(g, bp, vz, nx, ny, mz - 1, x, y, z, 0, f.X + 1, 0, f.Y + 1, -1, f.Z + 1);
  b.vbx[n] = ux;
  b.vby[n] = uy;
  b.vbz[n] = uz;
  b.x[n] = x + ux * g.dt;
  b.y[n] = y + uy * g.dt;
  b.z[n] = z + uz * g.dt;
  index3(g, b, n);
  const int bin = bin3_of(f, b.ibnx[n], b.ibny[n], b.ibnz[n]);
  if (bin != b.bin[n]) atomicOr(&s->moved, 1);
  b.bin[n] = bin;
  atomicMin(&s->box[0], b.ibnx[n]);
  atomicMin(&s->box[1], b.ibny[n]);
  atomicMin(&s->box[2], b.ibnz[n]);
  atomicMax(&s->box[3], b.ibnx[n]);
  atomicMax(&s->box[4], b.ibny[n]);
  atomicMax(&s->box[5], b.ibnz[n]);
}

// Counting sort of bubbles by bin (ascending bubble index within a bin).
constexpr int kScan = 1024;

__device__ __forceinline__ int block_scan(int v, int* total) {
  __shared__ int s_w[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_w[w] = x;
  __syncthreads();
  if (w == 0) {
    int t = s_w[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    s_w[lane] = t;
  }
  __syncthreads();
  const int before = (w > 0 ? s_w[w - 1] : 0) + x - v;
  if (total) *total = s_w[31];
  return before;
}

__global__ void bin3_count(const int* __restrict__ bin, int n, int* __restrict__ count) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n && bin[k] >= 0) atomicAdd(&count[bin[k]], 1);
}
__global__ void __launch_bounds__(kScan) bin3_scan(const int* __restrict__ count, int* __restrict__ start,
                                                  int* __restrict__ partial, int nbins) {
  const int k = blockIdx.x * kScan + threadIdx.x;
  int total;
  const int e = block_scan(k < nbins ? count[k] : 0, &total);
  if (k < nbins) start[k] = e;
  if (threadIdx.x == 0) partial[blockIdx.x] = total;
}
__global__ void __launch_bounds__(kScan) bin3_partials(int* __restrict__ partial, int nparts) {
  int carry = 0;
  for (int base = 0; base < nparts; base += kScan) {
    const int k = base + threadIdx.x;
    int total;
    const int e = block_scan(k < nparts ? partial[k] : 0, &total);
    __syncthreads();
    if (k < nparts) partial[k] = e + carry;
    carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[nparts] = carry;
}
__global__ void bin3_add(int* __restrict__ start, const int* __restrict__ partial, int nbins, int nparts) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nbins) start[k] += partial[k / kScan];
  if (k == nbins) start[nbins] = partial[nparts];
}
__global__ void bin3_fill(const int* __restrict__ bin, int n, const int* __restrict__ start, int* __restrict__ count,
                          int* __restrict__ idx) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n || bin[b] < 0) return;
  idx[start[bin[b]] + atomicSub(&count[bin[b]], 1) - 1] = b;
}
// One thread per bin: its bubbles in ascending index order.
__global__ void bin3_sort(const int* __restrict__ start, int* __restrict__ idx, int nbins) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nbins) return;
  const int a = start[c], e = start[c + 1];
  for (int q = a + 1; q < e; q++) {
    const int v = idx[q];
    int m = q - 1;
    while (m >= a && idx[m] > v) {
      idx[m + 1] = idx[m];
      m--;
    }
    idx[m + 1] = v;
  }
}
__global__ void bin3_pos(const int* __restrict__ idx, int total, int* __restrict__ pos) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < total) pos[idx[k]] = k;
}

// Pressure gather at the bubble (BubbleInterpolationScalarKernel, :361-395,
// over 2 x 2 x 2 cells) and its eight void-fraction contributions
// (VoidFractionReverseLookupKernel, :576-619, with the z factor), stored at
// 8 pos so that each cell reads contiguous runs.
template <typename S>
__device__ __forceinline__ double gather_pl3(const Grid3& g, const BubbleParams& bp, const Bub3& b, const S& px,
                                             const S& py, const S& pz, int n) {
  const Frame3& f = g.f;
  const double x = b.x[n], y = b.y[n], z = b.z[n];
  const int ix = b.ibnx[n], iy = b.ibny[n], iz = b.ibnz[n];
  const double cx = dcos(bp, bp.dcy, ix, g.dx, x), cy = dcos(bp, bp.dcz, iy, g.dy, y);
  const double cz = cos(2.0 * bp.pi / 2.0 * g.rdz * (((double)iz - 0.5) * g.dz - z));
  double s = 0.0;
  for (int ci = 0; ci < 2; ci++)
    for (int cj = 0; cj < 2; cj++)
      for (int ck = 0; ck < 2; ck++) {
        const int i = ix + ci, j = iy + cj, k = iz + ck;
        if (i >= 0 && i <= f.X + 1 && j >= 0 && j <= f.Y + 1 && k >= 0 && k <= f.Z + 1) {
          const long q = f.idx(i, j, k);
          s += (px.get(q) + py.get(q) + pz.get(q)) * delta_w(bp, cx, ci) * delta_w(bp, cy, cj) * delta_w(bp, cz, ck);
        }
      }
  return s;
}

__device__ __forceinline__ void contrib3(const Grid3& g, const BubbleParams& bp, const Bub3& b, int n, double Rt) {
  const int p = b.pos[n];
  if (p < 0) return;
  const double x = b.x[n], y = b.y[n], z = b.z[n];
  const int ix = b.ibnx[n], iy = b.ibny[n], iz = b.ibnz[n];
  const double cx = dcos(bp, bp.dcy, ix, g.dx, x), cy = dcos(bp, bp.dcz, iy, g.dy, y);
  const double cz = cos(2.0 * bp.pi / 2.0 * g.rdz * (((double)iz - 0.5) * g.dz - z));
  const double vol = bp.pi4r3 * b.n_B[n] * (Rt * Rt * Rt) * g.rdx * g.rdy * g.rdz;
  double* c = b.contrib + 8 * (long)p;
  for (int ci = 0; ci < 2; ci++)
    for (int cj = 0; cj < 2; cj++)
      for (int ck = 0; ck < 2; ck++)
        c[ci * 4 + cj * 2 + ck] = vol * delta_w(bp, cx, ci) * delta_w(bp, cy, cj) * delta_w(bp, cz, ck);
}

constexpr int kRpThreads3 = 128;

// The radius solves: the reference scheme's sub-steps (rp_substep_full) or
// the rk45 scheme (rk_attempt), from the state stored at the step's start,
// persistent lanes claiming bubbles from a queue.  With `reuse` (a solve of
// this step has completed), a bubble whose gathered pressure has the bit
// pattern of the last solve's keeps that solve's results: every input of its
// solve is unchanged.
template <typename P, bool RK>
__global__ void __launch_bounds__(kRpThreads3) radius3(const __grid_constant__ Grid3 g,
                                                       const __grid_constant__ BubbleParams bp, Bub3 b,
                                                       const typename P::S px, const typename P::S py,
                                                       const typename P::S pz, Scalars3* sc, int reuse,
                                                       const int* __restrict__ order) {
  const double dt = g.dt;
  RpState s;
  RkState r;
  int n = -1;
  bool drained = false;
  long long worst = 0;
  unsigned long long kept = 0;
  const int lane = threadIdx.x & 31;
  for (;;) {
    const unsigned need = __ballot_sync(0xffffffffu, n < 0 && !drained);
    if (need) {
      const int leader = __ffs(need) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(&sc->next, __popc(need));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need & (1u << lane)) {
        const int q = base + __popc(need & ((1u << lane) - 1u));
        const int bn = q < b.n ? (order ? order[q] : q) : -1;  // heaviest first once an order is built
        const double PLp = bn >= 0 ? gather_pl3(g, bp, b, px, py, pz, bn) : 0.0;
        if (bn < 0) {
          drained = true;
        } else if (reuse && __double_as_longlong(PLp) == __double_as_longlong(b.PL_p[bn])) {
          kept++;
        } else {
          n = bn;
          b.PL_p[n] = PLp;
          const double PLn = b.PL_n[n], PLm = b.PL_m[n];
          const double PC0 = PLn + bp.PL0, PC1 = 0.5 * (PLp - PLm) / dt,
                       PC2 = 0.5 * (PLp + PLm - 2.0 * PLn) / (dt * dt);
          if (RK) {
            r.r = bubble_r0(bp, b.R0[n]);
            r.R = b.R_pn[n];
            r.V = b.d1_R_n[n];
            r.PG = b.PG_n[n];
            r.h = b.dt_n[n];
            r.t = 0.0;
            r.tend = dt;
            r.Q = 0.0;
            r.count = 0;
            r.fresh = true;
            r.PC0 = PC0;
            r.PC1 = PC1;
            r.PC2 = PC2;
            r.K = 3.0 * (bp.gam - 1.0) * bp.K0 * bp.T0 * r.r.inv_PG0;
          } else {
            s.r = bubble_r0(bp, b.R0[n]);
            s.Rt = b.R_t[n];
            s.Rp = b.R_pn[n];
            s.Rn = b.R_nn[n];
            s.d1Rp = b.d1_R_n[n];
            s.PGp = b.PG_n[n];
            s.dtL = b.dt_n[n];
            s.re_n = b.re_n[n];
            s.remain = s.re_n + dt;
            s.time = -s.re_n;
            s.PC0 = PC0;
            s.PC1 = PC1;
            s.PC2 = PC2;
            s.heat = 0.0;
            s.vis = 0.0;
            s.count = 0;
          }
        }
      }
    }
    if (!__any_sync(0xffffffffu, n >= 0 || !drained)) break;
    if (n < 0) continue;
    if (RK) {
      if (r.t < r.tend && r.count < bp.step_cap) {
        if (!rk_attempt<typename P::T>(bp, r, bp.rk_rtol, g.c_inf)) r.count = bp.step_cap;
        continue;
      }
      if (r.t < r.tend) atomicOr(&sc->err, 1);
      b.R_t[n] = b.R_p[n] = b.R_n[n] = r.R;
      b.d1_R_p[n] = r.V;
      b.PG_p[n] = r.PG;
      b.dt[n] = fmin(r.h, dt);
      b.re[n] = 0.0;
      b.Q_B[n] = r.Q / dt;
      b.nsub[n] = (int)min(r.count, (long long)INT32_MAX);
      contrib3(g, bp, b, n, r.R);
      worst = max(worst, r.count);
    } else {
      if (s.remain > 0.0 && s.count < bp.step_cap) {
        rp_substep_full<typename P::T>(bp, s);
        continue;
      }
      if (s.remain > 0.0) atomicOr(&sc->err, 1);
      b.R_t[n] = s.Rt;
      b.R_p[n] = s.Rp;
      b.R_n[n] = s.Rn;
      b.d1_R_p[n] = s.d1Rp;
      b.PG_p[n] = s.PGp;
      b.dt[n] = s.dtL;
      b.re[n] = s.remain;
      b.Q_B[n] = (s.heat + s.vis) / (dt - s.remain + s.re_n);
      b.nsub[n] = (int)min(s.count, (long long)INT32_MAX);
      contrib3(g, bp, b, n, s.Rt);
      worst = max(worst, s.count);
    }
    n = -1;
  }
  for (int o = 16; o > 0; o >>= 1) worst = max(worst, __shfl_xor_sync(0xffffffffu, worst, o));
  if (lane == 0 && worst > 0) atomicMax(&sc->substep_max, worst);
  for (int o = 16; o > 0; o >>= 1) kept += __shfl_xor_sync(0xffffffffu, kept, o);
  if (lane == 0 && kept) atomicAdd(&sc->reused, kept);
}

template <typename P>
struct Couple3Args {
  typename P::V vx, vy, vz;
  typename P::S pnx, pny, pnz, px, py, pz;
  typename P::G fg, fgn;
  const int* start;
  const double* contrib;
  int box[6];  // cells [box0, box3] x [box1, box4] x [box2, box5]
  int gather;  // 1: void fraction from the bins; 0: keep fg
  int pressure;
  const double* tdev;
  unsigned long long* residual;
};

// Per cell of the box: the void fraction from the eight bins whose bubbles
// touch it (their runs in order, bins in a fixed order), then the pressure
// re-evaluation with it, the source forcing and the residual.
template <typename P>
__global__ void __launch_bounds__(256) couple3(const __grid_constant__ Grid3 g, const Couple3Args<P> a) {
  using G = typename P::G;
  const Frame3& f = g.f;
  const int i = a.box[0] + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = a.box[1] + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = a.box[2] + blockIdx.z;
  unsigned long long res = 0ull;
  if (i <= a.box[3] && j <= a.box[4] && k <= a.box[5]) {
    const long o = f.idx(i, j, k);
    double fgv;
    bool same = false;  // the FDTD pass's pressure is already this cell's final value
    if (a.gather) {
      fgv = 0.0;
      for (int ci = 0; ci < 2; ci++)
        for (int cj = 0; cj < 2; cj++)
          for (int ck = 0; ck < 2; ck++) {
            const int bx = i - ci, by = j - cj, bz = k - ck;
            if (bx < -1 || by < -1 || bz < -1) continue;
            const int c = ((bz + 1) * (f.Y + 3) + (by + 1)) * (f.X + 3) + (bx + 1);
            const int slot = ci * 4 + cj * 2 + ck;
            double run = 0.0;
            for (int q = a.start[c]; q < a.start[c + 1]; q++) run += a.contrib[8 * (long)q + slot];
            fgv += run;
          }
      fgv = G::stored(fgv);
      // No bubble touches the cell and its void fraction was zero in the
      // prediction and the step before: the gathered value is the stored 0
      // and the pressure evaluation would repeat the FDTD pass's (no
      // void-fraction rate), so the cell is left as it is.
      same = fgv == 0.0 && a.fg.get(o) == 0.0 && a.fgn.get(o) == 0.0;
      if (!same) a.fg.put(o, fgv);
    } else {
      fgv = a.fg.get(o);
    }
    if (!same && a.pressure && i >= 1 && i <= f.X && j >= 1 && j <= f.Y && k >= 1 && k <= f.Z) {
      const double t_cur = a.tdev[1];
      const double h = void_half3(g, fgv, a.fgn.get(o));
      const long ox = o - 1, oy = o - f.pitch, oz = o - (long)(f.Y + 4) * f.pitch;
      const double s1x = (-a.vx.get(ox) + a.vx.get(o)) * g.rdx;
      const double s1y = (-a.vy.get(oy) + a.vy.get(o)) * g.rdy;
      const double s1z = (-a.vz.get(oz) + a.vz.get(o)) * g.rdz;
      const double qx = a.pnx.get(o) * g.pax[i] - g.s3p * (s1x + h) * g.pbx[i];
      const double qy = a.pny.get(o) * g.pay[j] - g.s3p * (s1y + h) * g.pby[j];
      const double qz = a.pnz.get(o) * g.paz[k] - g.s3p * (s1z + h) * g.pbz[k];
      const double old = a.px.get(o) + a.py.get(o) + a.pz.get(o);
      double p0new = qx + qy + qz;
      const int e = g.src[o];
      if (e > 0) {
        p0new = element_pressure(g, e - 1, t_cur);
        a.px.put(o, p0new);
        a.py.put(o, 0.0);
        a.pz.put(o, 0.0);
      } else {
        a.px.put(o, qx);
        a.py.put(o, qy);
        a.pz.put(o, qz);
      }
      res = (unsigned long long)__double_as_longlong(fabs(old - p0new));
    }
  }
  const int lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31;
  for (int off = 16; off > 0; off >>= 1) res = max(res, __shfl_xor_sync(0xffffffffu, res, off));
  if (lane == 0 && res) atomicMax(a.residual, res);
}

// Contributions of every bubble at its current radius (set-up).
__global__ void contrib_init3(const __grid_constant__ Grid3 g, const __grid_constant__ BubbleParams bp, Bub3 b) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n < b.n) contrib3(g, bp, b, n, b.R_t[n]);
}

// Dense read-back of a window of the frame (x fastest).  kind 0: velocity or
// split-pressure storage; 1: void-fraction storage; 2: p0 = px + py + pz;
// 3: the mixture density (1 - f_g) rho_inf the next velocity update uses.
__global__ void read3(Frame3 f, int kind, int mixed, const void* buf, const void* px, const void* py, const void* pz,
                      int ilo, int jlo, int klo, int nx, int ny, int nz, double rho_inf, int rho_const,
                      double* __restrict__ out) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long)nx * ny * nz) return;
  const int i = ilo + (int)(e % nx), j = jlo + (int)((e / nx) % ny), k = klo + (int)(e / ((long)nx * ny));
  const long q = f.idx(i, j, k);
  auto sv = [&](const void* p) -> double {
    return mixed ? F32c{(float2*)p}.get(q) : F64{(double*)p}.get(q);
  };
  auto gv = [&](const void* p) -> double { return mixed ? F32{(float*)p}.get(q) : F64{(double*)p}.get(q); };
  double v;
  switch (kind) {
    case 0: v = sv(buf); break;
    case 1: v = gv(buf); break;
    case 2: v = sv(px) + sv(py) + sv(pz); break;
    default: v = rho_const ? rho_inf : (1.0 - gv(buf)) * rho_inf; break;
  }
  out[e] = v;
}

// Plain FP64 / mixed storage of the fields, as the 2-D path.
struct P64 {
  using V = F64;
  using S = F64;
  using G = F64;
  using T = double;
  static constexpr int kIndex = 0;
};
struct PMix {
  using V = F32c;
  using S = F32c;
  using G = F32;
  using T = float;
  static constexpr int kIndex = 1;
};

// ---------------------------------------------------------------------------
// Discrete adjoint of the bubble-free 3-D step (crp_adjoint).  Without bubbles
// the step is linear in the state:
//   v'_f  = (v_f va - dt_rho rd (p0_b - p0_a)) vb           every computed face f
//                                                            between cells a and b,
//   p'_c  = p_c pa_c - s3p pb_c (v'_east - v'_west) rd_c     interior cells, c = x, y, z,
//   p'_x  = s_e(t), p'_y = p'_z = 0                         source cells,
// with p0 = px + py + pz (0 in the ghost cells, which are never written).  The
// reverse of one step, given the adjoint of the state after it:
//   1. adj3_source: the source cells' share of the gradient, their adjoint zeroed;
//   2. adj3_step, one pass from one set of adjoint frames into the other:
//      the face adjoints take the pressure update's transpose; the component
//      adjoints become pa_c M_c plus the velocity update's transpose into p0
//      (the same for all three components); the face adjoints are multiplied
//      by va vb; and 2 dt w p0 of the step before is added for the focal cells
//      (adj3_force adds the last step's before the sweep).
// Each cell forms the transposed values of its six faces (its west, south and
// bottom faces by the same expression as the neighbour that owns them), so a
// step reads 6 doubles per cell (L and M; neighbours through L1/L2) and
// writes 6: 96 bytes.
struct Adj3 {
  double *LX, *LY, *LZ;  // adjoints of vx, vy, vz (frame layout)
  double *MX, *MY, *MZ;  // adjoints of px, py, pz
};
struct Box3 {
  int i0, j0, k0, nx, ny, nz;
  const double* w;  // weight of each box cell (0 outside the focal sphere)
};

template <typename S>
__global__ void adj3_record(const Frame3 f, const S px, const S py, const S pz, const Box3 b, double* out) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= (long)b.nx * b.ny * b.nz) return;
  const int i = b.i0 + (int)(t % b.nx), j = b.j0 + (int)((t / b.nx) % b.ny), k = b.k0 + (int)(t / ((long)b.nx * b.ny));
  const long q = f.idx(i, j, k);
  out[t] = px.get(q) + py.get(q) + pz.get(q);
}

__global__ void adj3_objective(const Box3 b, const double* p0, double* Jn) {
  // One block per recorded step: sum of w p0^2 in a fixed order.
  __shared__ double part[256];
  const long n = (long)b.nx * b.ny * b.nz;
  const double* p = p0 + blockIdx.x * n;
  double s = 0.0;
  for (long t = threadIdx.x; t < n; t += blockDim.x) s += b.w[t] * p[t] * p[t];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) Jn[blockIdx.x] = part[0];
}

__global__ void adj3_force(const Frame3 f, const Adj3 a, const Box3 b, const double* p0, double two_dt) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= (long)b.nx * b.ny * b.nz) return;
  const double w = b.w[t];
  if (w == 0.0) return;
  const int i = b.i0 + (int)(t % b.nx), j = b.j0 + (int)((t / b.nx) % b.ny), k = b.k0 + (int)(t / ((long)b.nx * b.ny));
  const long q = f.idx(i, j, k);
  const double d = two_dt * w * p0[t];
  a.MX[q] += d;
  a.MY[q] += d;
  a.MZ[q] += d;
}

// Source cell c (frame index cells[c], element elem[c]) at the step's time t:
// d p'_x / d amp_e and d p'_x / d phase_e times the adjoint of p'_x, summed
// over the steps per cell; the cell's adjoints then end (the forced values do
// not depend on the state).
__global__ void adj3_source(const __grid_constant__ Grid3 g, const Adj3 a, const long* cells, const int* elem, int n,
                            double t, double* gA, double* gP) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const long q = cells[c];
  const double m = a.MX[q];
  a.MX[q] = 0.0;
  a.MY[q] = 0.0;
  a.MZ[q] = 0.0;
  if (!(t > 0.0)) return;
  const double tau = fmod(t, g.period);
  if (!(tau <= g.on_time)) return;
  const int e = elem[c];
  double sn, cs;
  sincos(g.omega * t + g.elem_phase[e], &sn, &cs);
  const double env = g.pamp * burst_env(g, tau);
  gA[c] += m * env * sn;
  gP[c] += m * env * g.elem_amp[e] * cs;
}

// The pressure update's transpose at one face (computed faces: vx for i in
// [0, X] with j, k interior; vy for j in [0, Y]; vz for k in [0, Z]).
__device__ __forceinline__ double adj3_lxt(const Grid3& g, const Adj3& a, int i, int j, int k) {
  const Frame3& f = g.f;
  const long q = f.idx(i, j, k);
  return a.LX[q] + (-g.s3p) * g.rdx * (g.pbx[i] * a.MX[q] - g.pbx[i + 1] * a.MX[f.idx(i + 1, j, k)]);
}
__device__ __forceinline__ double adj3_lyt(const Grid3& g, const Adj3& a, int i, int j, int k) {
  const Frame3& f = g.f;
  const long q = f.idx(i, j, k);
  return a.LY[q] + (-g.s3p) * g.rdy * (g.pby[j] * a.MY[q] - g.pby[j + 1] * a.MY[f.idx(i, j + 1, k)]);
}
__device__ __forceinline__ double adj3_lzt(const Grid3& g, const Adj3& a, int i, int j, int k) {
  const Frame3& f = g.f;
  const long q = f.idx(i, j, k);
  return a.LZ[q] + (-g.s3p) * g.rdz * (g.pbz[k] * a.MZ[q] - g.pbz[k + 1] * a.MZ[f.idx(i, j, k + 1)]);
}

// One reverse step after adj3_source, from `in` into `out`; p0 (the focal
// pressures of the step before, or null) adds that step's objective term.
// Blocks of 32 x 8 cells of one plane (blockIdx.z); each interior cell writes
// its east, north and top faces, the first column, row and plane also the
// 0 faces.
__global__ void adj3_step(const __grid_constant__ Grid3 g, const Adj3 in, const Adj3 out, const Box3 b,
                          const double* __restrict__ p0, double two_dt) {
  const Frame3& f = g.f;
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x, j = 1 + blockIdx.y * blockDim.y + threadIdx.y,
            k = 1 + blockIdx.z;
  if (i > f.X || j > f.Y || k > f.Z) return;
  const long q = f.idx(i, j, k);
  const double xe = adj3_lxt(g, in, i, j, k), xw = adj3_lxt(g, in, i - 1, j, k);
  const double yn = adj3_lyt(g, in, i, j, k), ys = adj3_lyt(g, in, i, j - 1, k);
  const double zt = adj3_lzt(g, in, i, j, k), zb = adj3_lzt(g, in, i, j, k - 1);
  const double lp0 = g.dt_rho * (g.rdx * (g.vbx[i + 1] * xe - g.vbx[i] * xw) +
                                 g.rdy * (g.vby[j + 1] * yn - g.vby[j] * ys) +
                                 g.rdz * (g.vbz[k + 1] * zt - g.vbz[k] * zb));
  double mx = g.pax[i] * in.MX[q] + lp0;
  double my = g.pay[j] * in.MY[q] + lp0;
  double mz = g.paz[k] * in.MZ[q] + lp0;
  if (p0) {
    const int bi = i - b.i0, bj = j - b.j0, bk = k - b.k0;
    if (bi >= 0 && bi < b.nx && bj >= 0 && bj < b.ny && bk >= 0 && bk < b.nz) {
      const long t = bi + (long)b.nx * (bj + (long)b.ny * bk);
      const double w = b.w[t];
      if (w != 0.0) {
        const double d = two_dt * w * p0[t];
        mx += d;
        my += d;
        mz += d;
      }
    }
  }
  out.MX[q] = mx;
  out.MY[q] = my;
  out.MZ[q] = mz;
  out.LX[q] = xe * (g.vax[i + 1] * g.vbx[i + 1]);
  out.LY[q] = yn * (g.vay[j + 1] * g.vby[j + 1]);
  out.LZ[q] = zt * (g.vaz[k + 1] * g.vbz[k + 1]);
  if (i == 1) out.LX[f.idx(0, j, k)] = xw * (g.vax[1] * g.vbx[1]);
  if (j == 1) out.LY[f.idx(i, 0, k)] = ys * (g.vay[1] * g.vby[1]);
  if (k == 1) out.LZ[f.idx(i, j, 0)] = zb * (g.vaz[1] * g.vbz[1]);
}

}  // namespace d3

// ---------------------------------------------------------------------------
// Host side.

struct Sim3Impl {
  crp_config cfg{};
  d3::Grid3 g{};
  BubbleParams bp{};
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int device = 0;
  bool mixed = false;
  std::string err;
  char* pool = nullptr;
  size_t pool_bytes = 0;
  size_t cells = 0;
  void *vx[2]{}, *vy[2]{}, *vz[2]{}, *px[2]{}, *py[2]{}, *pz[2]{}, *fg[3]{};
  double* d_fac = nullptr;  // PML factors
  short* d_src = nullptr;
  double* d_elem = nullptr;
  double* scratch = nullptr;  // dense read-back
  d3::Bub3 bub{};
  int* bin_count = nullptr;
  int* bin_start = nullptr;
  int* bin_idx = nullptr;
  int* bin_partial = nullptr;
  int nbins = 0;
  d3::Scalars3* d_sc = nullptr;
  d3::Scalars3* h_sc = nullptr;
  int elem_n = 0;
  int src_cells = 0;
  int cur_v = 0, cur_p = 0, fg_a = 0, fg_b = 1, fg_c = 2;
  double tstep = 0.0, tstepx = 0.0, t_prev = 0.0;
  double picard_tol = 1.0e-7f;
  bool bins_stale = true;
  int* lpt_hist = nullptr;    // solve order (lpt.cuh): bucket counts, cursors, order
  int* lpt_cursor = nullptr;
  int* lpt_order = nullptr;
  bool use_order = false;     // the order was built for this step's radius solves
  int rp_grid = 1;
  int rp_grid_full = 1;  // one lane per bubble, up to 4 blocks per SM
  int rp_blocks_req = 0;  // crp_set_tuning (0: rp_grid_full)
  int supp[3][6];
  crp_stats stats{};
  int64_t launches = 0;
  // Profiling (crp_set_profiling): events around the FDTD launch of a step.
  bool prof_on = false, prof_pending = false;
  bool fdtd_smem_set[2] = {false, false};  // fdtd3's dynamic shared memory limit raised (FP64, mixed)
  cudaEvent_t ev_f0 = nullptr, ev_f1 = nullptr;
  crp_status set_profiling(bool on) {
    if (on && !ev_f0) {
      if (cudaEventCreate(&ev_f0) != cudaSuccess || cudaEventCreate(&ev_f1) != cudaSuccess)
        return CRP_ERR_CUDA;
    }
    prof_on = on;
    return CRP_OK;
  }

  crp_status fail(crp_status s, const char* what, cudaError_t e = cudaSuccess) {
    err = what;
    if (e != cudaSuccess) err += std::string(": ") + cudaGetErrorString(e);
    return s;
  }
#define C3(call)                                                   \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) return fail(CRP_ERR_CUDA, #call, e_);   \
  } while (0)

  template <typename T>
  T* carve(size_t count, size_t& off, bool dry) {
    const size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
    T* p = dry ? nullptr : reinterpret_cast<T*>(pool + off);
    off += bytes;
    return p;
  }

  size_t layout(bool dry, int n) {
    size_t off = 0;
    for (int q = 0; q < 2; q++) {
      vx[q] = carve<double>(cells, off, dry);
      vy[q] = carve<double>(cells, off, dry);
      vz[q] = carve<double>(cells, off, dry);
      px[q] = carve<double>(cells, off, dry);
      py[q] = carve<double>(cells, off, dry);
      pz[q] = carve<double>(cells, off, dry);
    }
    for (int q = 0; q < 3; q++) fg[q] = carve<double>(cells, off, dry);
    d_src = carve<short>(cells, off, dry);
    const int FX = g.f.X, FY = g.f.Y, FZ = g.f.Z;
    d_fac = carve<double>(4 * (size_t)(FX + 3 + FY + 3 + FZ + 3), off, dry);
    d_elem = carve<double>(2 * (size_t)std::max(elem_n, 1), off, dry);
    scratch = carve<double>((size_t)(FX + 3) * (FY + 3) * (FZ + 3), off, dry);
    d_sc = carve<d3::Scalars3>(1, off, dry);
    bub.n = n;
    double** dp[] = {&bub.x, &bub.y, &bub.z, &bub.R0, &bub.n_B, &bub.R_t, &bub.R_p, &bub.R_pn, &bub.R_n, &bub.R_nn,
                     &bub.d1_R_p, &bub.d1_R_n, &bub.PG_p, &bub.PG_n, &bub.PL_p, &bub.PL_n, &bub.PL_m, &bub.Q_B,
                     &bub.dt, &bub.dt_n, &bub.re, &bub.re_n, &bub.vbx, &bub.vby, &bub.vbz};
    for (double** p : dp) *p = carve<double>(std::max(n, 1), off, dry);
    bub.contrib = carve<double>(8 * (size_t)std::max(n, 1), off, dry);
    int** ip[] = {&bub.ibmx, &bub.ibmy, &bub.ibmz, &bub.ibnx, &bub.ibny, &bub.ibnz, &bub.bin, &bub.nsub, &bub.pos};
    for (int** p : ip) *p = carve<int>(std::max(n, 1), off, dry);
    if (n > 0) {
      nbins = (FX + 3) * (FY + 3) * (FZ + 3);
      bin_count = carve<int>(nbins, off, dry);
      bin_start = carve<int>(nbins + 1, off, dry);
      bin_idx = carve<int>(std::max(n, 1), off, dry);
      bin_partial = carve<int>((nbins + d3::kScan - 1) / d3::kScan + 1, off, dry);
      lpt_hist = carve<int>(kLptBuckets, off, dry);
      lpt_cursor = carve<int>(kLptBuckets, off, dry);
      lpt_order = carve<int>(n, off, dry);
    }
    return off;
  }

  template <typename P>
  typename P::V vview(void* p) const;
  template <typename A>
  A view(void* p) const;

  crp_status create(const crp_config& c, const crp_bubbles_in* bin, void* user_stream);
  crp_status step_once();
  template <typename P>
  crp_status launch_fdtd();
  template <typename P>
  crp_status launch_move();
  template <typename P>
  crp_status launch_radius(int done);
  template <typename P>
  crp_status launch_couple(bool gather, bool pressure, const int box[6]);
  crp_status build_bins();
  crp_status build_order();
  void bubble_box(int box[6]) const;
  static double as_double(unsigned long long b) {
    double d;
    std::memcpy(&d, &b, sizeof(d));
    return d;
  }
  crp_status read_field(crp_field w, double* host);
  crp_status read_bubbles(crp_bubble_field w, double* host);
  crp_status adjoint(const crp_objective* obj, double* J, double* grad_amp, double* grad_phase);
  void* adj_ws = nullptr;  // crp_adjoint's device workspace, kept between calls
  size_t adj_ws_bytes = 0;
  // Source cells (frame index, element) in frame order, and the focus the bowl's phases aim at.
  std::vector<long> src_list;
  std::vector<int> src_elem;
  double focus[3] = {0.0, 0.0, 0.0};
  crp_status set_elements(int n, const double* amp, const double* phase);
  ~Sim3Impl();
};

template <>
F64 Sim3Impl::view<F64>(void* p) const {
  return F64{(double*)p};
}
template <>
F32c Sim3Impl::view<F32c>(void* p) const {
  return F32c{(float2*)p};
}
template <>
F32 Sim3Impl::view<F32>(void* p) const {
  return F32{(float*)p};
}

Sim3Impl::~Sim3Impl() {
  if (adj_ws) cudaFree(adj_ws);
  if (ev_f0) cudaEventDestroy(ev_f0);
  if (ev_f1) cudaEventDestroy(ev_f1);
  if (pool) cudaFree(pool);
  if (h_sc) cudaFreeHost(h_sc);
  if (own_stream && stream) cudaStreamDestroy(stream);
}

// PML profile of one axis (init_sigma's closed forms, src/bubble_CUDA.cu:946-1205,
// with a PML at both ends): factors 1 - s and 1 / (1 + s) of the faces
// (index n + 1, n in [-1, N+1]) and cells (index n, n in [0, N+1]).
static void axis_factors(int N, int npml, double h, double sig, int order, double s4, std::vector<double>& va,
                         std::vector<double>& vb, std::vector<double>& pa, std::vector<double>& pb) {
  std::vector<double> m(N + 2, 0.0), fc(N + 3, 0.0);
  const double smax = -std::log(sig) * 0.5 * ((double)order + 1.0) / (h * (double)npml);
  for (int n = 1; n <= std::min(N, npml); n++)
    m[n] = smax * std::pow(((double)(npml - n + 1) - 0.5) / ((double)npml), (double)order);
  for (int n = std::max(1, N - npml + 1); n <= N; n++)
    m[n] = smax * std::pow(((double)(n - N + npml) - 0.5) / ((double)npml), (double)order);
  for (int n = 0; n <= std::min(N, npml - 1); n++)
    fc[n + 1] = smax * std::pow(((double)(npml - n)) / ((double)npml), (double)order);
  for (int n = std::max(0, N - npml + 1); n <= N; n++)
    fc[n + 1] = smax * std::pow(((double)(n - N + npml)) / ((double)npml), (double)order);
  va.resize(N + 3);
  vb.resize(N + 3);
  pa.resize(N + 3, 1.0);
  pb.resize(N + 3, 1.0);
  for (int q = 0; q < N + 3; q++) {
    const double s = s4 * fc[q];  // (c + c) / 2 * dt / 2 * sigma_n
    va[q] = 1.0 - s;
    vb[q] = 1.0 / (1.0 + s);
  }
  for (int q = 0; q < N + 2; q++) {
    const double s = s4 * m[q];
    pa[q] = 1.0 - s;
    pb[q] = 1.0 / (1.0 + s);
  }
}

crp_status Sim3Impl::create(const crp_config& c, const crp_bubbles_in* bin, void* user_stream) {
  cfg = c;
  const int X = c.grid_x, Y = c.grid_y, Z = c.ext_grid_z;
  if (X < 4 || Y < 4 || Z < 4 || !(c.grid_lx > 0) || !(c.grid_ly > 0) || !(c.ext_grid_lz > 0))
    return fail(CRP_ERR_INVALID, "3-D grid needs at least 4 cells and a positive length per axis");
  if (!(c.pml_x0 && c.pml_x1 && c.pml_y0 && c.pml_y1 && c.ext_pml_z0 && c.ext_pml_z1))
    return fail(CRP_ERR_UNSUPPORTED, "the 3-D path implements a PML on all six faces");
  if (c.tr_cylindrical) return fail(CRP_ERR_UNSUPPORTED, "3-D grids are Cartesian (transducer.cylindrical = 0)");
  if (c.sim_order != 2 || c.sim_smooth_delta_band != 2)
    return fail(CRP_ERR_UNSUPPORTED, "simulation.order = 2 and smooth_delta_band = 2 only");
  if (c.ext_precision != CRP_PREC_FP64 && c.ext_precision != CRP_PREC_MIXED)
    return fail(CRP_ERR_INVALID, "ext.precision must be fp64 or mixed");
  if (c.ext_rp_scheme != CRP_RP_REF && c.ext_rp_scheme != CRP_RP_RK45)
    return fail(CRP_ERR_INVALID, "ext.rp_scheme must be ref or rk45");
  if ((long long)(X + 4) * (Y + 4) * (Z + 4) >= (1ll << 31))
    return fail(CRP_ERR_UNSUPPORTED, "3-D frame of 2^31 cells or more");
  mixed = c.ext_precision == CRP_PREC_MIXED;
  picard_tol = c.ext_picard_tol > 0.0 ? c.ext_picard_tol : (mixed ? 1.0e-5 : (double)1.0e-7f);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(CRP_ERR_NO_DEVICE, "no CUDA device");
  C3(cudaGetDevice(&device));
  if (user_stream) {
    stream = (cudaStream_t)user_stream;
  } else {
    C3(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    own_stream = true;
  }
  const double pi = std::acos(-1.0);
  d3::Frame3 f{X, Y, Z, ((X + 4) + 31) / 32 * 32};
  g.f = f;
  g.dx = (double)c.grid_lx / (double)X;
  g.dy = (double)c.grid_ly / (double)Y;
  g.dz = (double)c.ext_grid_lz / (double)Z;
  g.rdx = 1.0 / g.dx;
  g.rdy = 1.0 / g.dy;
  g.rdz = 1.0 / g.dz;
  g.rho_inf = c.ext_rho_inf;
  g.c_inf = c.ext_c_inf;
  g.P_inf = c.ext_p_inf;
  g.dt = c.sim_cfl * std::min(g.dx, std::min(g.dy, g.dz)) / g.c_inf;
  g.dt_rho = g.dt / g.rho_inf;
  g.s3p = g.dt * g.rho_inf * g.c_inf * g.c_inf;
  g.omega = 2.0 * pi * c.tr_freq;
  g.pamp = g.rho_inf * g.c_inf * c.tr_amp;
  g.period = (double)(c.tr_on_wave + c.tr_off_wave) / c.tr_freq;
  g.on_time = (double)c.tr_on_wave / c.tr_freq;
  g.ramp_time = c.ext_ramp_cycles / c.tr_freq;
  cells = (size_t)f.pitch * (Y + 4) * (Z + 4);

  // Source: the bowl's elements (Fibonacci points on the lower hemisphere) and
  // the shell cells, each with its nearest element.
  elem_n = std::max(0, c.ext_array_elements);
  std::vector<double> ex(elem_n), ey(elem_n), ez(elem_n), eamp(elem_n, 1.0), eph(elem_n, 0.0);
  std::vector<short> src(cells, 0);
  {
    const double Ra = c.ext_array_radius;
    const double cx = 0.5 * X * g.dx, cy = 0.5 * Y * g.dy, cz = 0.5 * Z * g.dz;
    const double golden = pi * (3.0 - std::sqrt(5.0));
    const double fx = cx + c.ext_array_focus_dx;
    focus[0] = fx;
    focus[1] = cy;
    focus[2] = cz;
    if (elem_n > 32767) return fail(CRP_ERR_UNSUPPORTED, "more than 32767 array elements");
    for (int e = 0; e < elem_n; e++) {
      const double ct = -((double)e + 0.5) / (double)elem_n;
      const double st = std::sqrt(std::max(0.0, 1.0 - ct * ct));
      const double fph = golden * (double)e;
      ex[e] = cx + Ra * st * std::cos(fph);
      ey[e] = cy + Ra * st * std::sin(fph);
      ez[e] = cz + Ra * ct;
      const double d = std::sqrt((ex[e] - fx) * (ex[e] - fx) + (ey[e] - cy) * (ey[e] - cy) + (ez[e] - cz) * (ez[e] - cz));
      eph[e] = std::fmod(g.omega * d / g.c_inf, 2.0 * pi);
      if (c.ext_array_phases == 1) {
        uint32_t w[4];
        philox_block(c.ext_array_seed, (uint64_t)e, 2u, w);
        eph[e] = 2.0 * pi * (((double)w[0] + 0.5) / 4294967296.0);
      }
    }
    if (elem_n > 0) {
      const double half = 0.5 * g.dx;
      for (int k = 1; k <= Z; k++)
        for (int j = 1; j <= Y; j++)
          for (int i = 1; i <= X; i++) {
            const double xc = ((double)i - 0.5) * g.dx - cx, yc = ((double)j - 0.5) * g.dy - cy,
                         zc = ((double)k - 0.5) * g.dz - cz;
            const double r = std::sqrt(xc * xc + yc * yc + zc * zc);
            if (!(zc < 0.0) || !(std::fabs(r - Ra) <= half)) continue;
            int best = 0;
            double bd = 1e300;
            for (int e = 0; e < elem_n; e++) {
              const double dxe = ex[e] - cx - xc, dye = ey[e] - cy - yc, dze = ez[e] - cz - zc;
              const double dd = dxe * dxe + dye * dye + dze * dze;
              if (dd < bd) bd = dd, best = e;
            }
            src[f.idx(i, j, k)] = (short)(best + 1);
            src_list.push_back(f.idx(i, j, k));
            src_elem.push_back(best);
            src_cells++;
          }
    }
  }
  // Bubbles: explicit (with z), or seeded from the [ext] keys.
  std::vector<double> bx, by, bz, br0, bnb;
  if (c.bub_enable) {
    if (bin && bin->n > 0) {
      if (!bin->z) return fail(CRP_ERR_INVALID, "3-D bubbles need z coordinates");
      bx.assign(bin->x, bin->x + bin->n);
      by.assign(bin->y, bin->y + bin->n);
      bz.assign(bin->z, bin->z + bin->n);
      br0.assign(bin->r0, bin->r0 + bin->n);
      bnb.assign(bin->n_b, bin->n_b + bin->n);
    } else if (c.ext_bubble_count > 0) {
      const int n = c.ext_bubble_count;
      bx.resize(n);
      by.resize(n);
      bz.resize(n);
      br0.resize(n);
      bnb.resize(n);
      const crp_status st = crp_seed_bubbles3(&c, bx.data(), by.data(), bz.data(), br0.data(), bnb.data());
      if (st != CRP_OK) return fail(st, "bubble seeding failed");
    }
  }
  const int nb = (int)bx.size();
  pool_bytes = layout(true, nb);
  C3(cudaMalloc(&pool, pool_bytes));
  layout(false, nb);
  C3(cudaMemsetAsync(pool, 0, pool_bytes, stream));
  C3(cudaMallocHost(&h_sc, sizeof(d3::Scalars3)));
  std::memset(h_sc, 0, sizeof(d3::Scalars3));
  // PML factors: x faces, y faces, z faces (N+3 each), then x, y, z cells.
  {
    std::vector<double> va[3], vb[3], pa[3], pb[3];
    const double s4 = (g.c_inf + g.c_inf) * 0.5 * 0.5 * g.dt;
    axis_factors(X, c.pml_grid_number, g.dx, c.pml_sigma, c.pml_order, s4, va[0], vb[0], pa[0], pb[0]);
    axis_factors(Y, c.pml_grid_number, g.dy, c.pml_sigma, c.pml_order, s4, va[1], vb[1], pa[1], pb[1]);
    axis_factors(Z, c.pml_grid_number, g.dz, c.pml_sigma, c.pml_order, s4, va[2], vb[2], pa[2], pb[2]);
    std::vector<double> blk;
    size_t off[12];
    int q = 0;
    for (auto* v : {&va[0], &vb[0], &va[1], &vb[1], &va[2], &vb[2], &pa[0], &pb[0], &pa[1], &pb[1], &pa[2], &pb[2]}) {
      off[q++] = blk.size();
      blk.insert(blk.end(), v->begin(), v->end());
    }
    if (blk.size() > 4 * (size_t)(X + 3 + Y + 3 + Z + 3)) return fail(CRP_ERR_INVALID, "PML factor block");
    C3(cudaMemcpyAsync(d_fac, blk.data(), sizeof(double) * blk.size(), cudaMemcpyHostToDevice, stream));
    const double** dst[12] = {&g.vax, &g.vbx, &g.vay, &g.vby, &g.vaz, &g.vbz,
                              &g.pax, &g.pbx, &g.pay, &g.pby, &g.paz, &g.pbz};
    for (int r = 0; r < 12; r++) *dst[r] = d_fac + off[r];
    C3(cudaStreamSynchronize(stream));
  }
  C3(cudaMemcpyAsync(d_src, src.data(), sizeof(short) * cells, cudaMemcpyHostToDevice, stream));
  g.src = d_src;
  if (elem_n > 0) {
    std::vector<double> ev(eamp);
    ev.insert(ev.end(), eph.begin(), eph.end());
    C3(cudaMemcpyAsync(d_elem, ev.data(), sizeof(double) * ev.size(), cudaMemcpyHostToDevice, stream));
    C3(cudaStreamSynchronize(stream));
  }
  g.elem_amp = d_elem;
  g.elem_phase = d_elem + std::max(elem_n, 1);
  // Bubble parameters shared with the 2-D path.
  bp.PL0 = c.bub_P0;
  bp.T0 = c.bub_T0;
  bp.gam = c.bub_gamma;
  bp.sig = c.bub_sigma;
  bp.mu = c.bub_mu;
  bp.rho = c.bub_rho;
  bp.inv_rho = 1.0 / c.bub_rho;
  {
    double cc = 0.01;
    while (std::sqrt(cc) > 0.1) cc = std::nextafter(cc, 0.0);
    while (!(std::sqrt(cc) > 0.1)) cc = std::nextafter(cc, 1.0);
    bp.abs2_cut64 = cc;
    float cf = 0.01f;
    while (std::sqrt(cf) > 0.1f) cf = std::nextafter(cf, 0.0f);
    while (!(std::sqrt(cf) > 0.1f)) cf = std::nextafter(cf, 1.0f);
    bp.abs2_cut32 = cf;
    bp.rho32 = (float)bp.rho;
    bp.sig32 = (float)bp.sig;
    bp.mu32 = (float)bp.mu;
    bp.gam32 = (float)bp.gam;
    bp.inv_rho32 = (float)bp.inv_rho;
  }
  bp.K0 = c.bub_K0;
  bp.dt0 = 0.1 * g.dt;
  bp.pi = pi;
  bp.pi4r3 = pi * 4.0 / 3.0;
  bp.dcx = 1.0 / 2.0;
  bp.dcy = 2.0 * pi / 2.0 * g.rdx;
  bp.dcz = 2.0 * pi / 2.0 * g.rdy;
  bp.step_cap = c.ext_rp_step_cap;
  bp.rk_rtol = c.ext_rp_tol > 0.0 ? c.ext_rp_tol : kRk45DefaultTol;
  bp.reuse = c.ext_rp_reuse ? 1 : 0;
  for (int q = 0; q < 3; q++) supp[q][0] = supp[q][1] = supp[q][2] = 1, supp[q][3] = supp[q][4] = supp[q][5] = 0;
  if (nb > 0) {
    std::vector<double> zeros(nb, 0.0), dt0(nb, bp.dt0), pg0(nb);
    for (int k = 0; k < nb; k++) pg0[k] = c.bub_P0 + 2.0 * c.bub_sigma / br0[k];
    auto up = [&](double* d, const std::vector<double>& h) {
      return cudaMemcpyAsync(d, h.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, stream);
    };
    C3(up(bub.x, bx));
    C3(up(bub.y, by));
    C3(up(bub.z, bz));
    C3(up(bub.R0, br0));
    C3(up(bub.n_B, bnb));
    for (double* d : {bub.R_t, bub.R_p, bub.R_pn, bub.R_n, bub.R_nn}) C3(up(d, br0));
    for (double* d : {bub.PG_p, bub.PG_n}) C3(up(d, pg0));
    for (double* d : {bub.dt, bub.dt_n}) C3(up(d, dt0));
    C3(cudaStreamSynchronize(stream));
    d3::set_time3<<<1, 1, 0, stream>>>(d_sc, 0.0, 0.0);
    d3::index3_kernel<<<(nb + 255) / 256, 256, 0, stream>>>(g, bub, d_sc);
    C3(cudaGetLastError());
    {
      const crp_status bs = build_bins();
      if (bs != CRP_OK) return bs;
    }
    // Initial void fraction (calculate_void_fraction at set-up, src/bubble_CUDA.cu:180-187):
    // every bubble's contributions at R0, gathered per cell; the history
    // buffers start equal to it.
    d3::contrib_init3<<<(nb + 255) / 256, 256, 0, stream>>>(g, bp, bub);
    C3(cudaGetLastError());
    C3(cudaMemcpyAsync(h_sc, d_sc, sizeof(d3::Scalars3), cudaMemcpyDeviceToHost, stream));
    C3(cudaStreamSynchronize(stream));
    int box[6];
    bubble_box(box);
    const crp_status st = mixed ? launch_couple<d3::PMix>(true, false, box) : launch_couple<d3::P64>(true, false, box);
    if (st != CRP_OK) return st;
    const size_t bytes = sizeof(double) * cells;
    C3(cudaMemcpyAsync(fg[fg_b], fg[fg_a], bytes, cudaMemcpyDeviceToDevice, stream));
    C3(cudaMemcpyAsync(fg[fg_c], fg[fg_a], bytes, cudaMemcpyDeviceToDevice, stream));
    for (int q = 0; q < 3; q++) std::memcpy(supp[q], box, sizeof(box));
  }
  int sms = 0;
  C3(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  rp_grid_full = std::max(1, std::min(sms * 4, (nb + d3::kRpThreads3 - 1) / d3::kRpThreads3));
  rp_grid = rp_grid_full;
  C3(cudaStreamSynchronize(stream));
  return CRP_OK;
}

// Cells whose void fraction the bubbles' stencils reach: their ibn box
// widened by one (the stencil's second point) and clipped to the frame's
// cells [0, N+1].
void Sim3Impl::bubble_box(int box[6]) const {
  const d3::Scalars3& s = *h_sc;
  const int N[3] = {g.f.X, g.f.Y, g.f.Z};
  for (int a = 0; a < 3; a++) {
    box[a] = std::max(0, s.box[a]);
    box[a + 3] = std::min(N[a] + 1, s.box[a + 3] + 1);
  }
}

static void box_union(int out[6], const int a[6], const int b[6]) {
  const bool ea = a[0] > a[3] || a[1] > a[4] || a[2] > a[5];
  const bool eb = b[0] > b[3] || b[1] > b[4] || b[2] > b[5];
  if (ea) {
    std::memcpy(out, b, 6 * sizeof(int));
    return;
  }
  if (eb) {
    std::memcpy(out, a, 6 * sizeof(int));
    return;
  }
  for (int q = 0; q < 3; q++) {
    out[q] = std::min(a[q], b[q]);
    out[q + 3] = std::max(a[q + 3], b[q + 3]);
  }
}

crp_status Sim3Impl::build_bins() {
  const int n = bub.n;
  C3(cudaMemsetAsync(bin_count, 0, sizeof(int) * nbins, stream));
  d3::bin3_count<<<(n + 255) / 256, 256, 0, stream>>>(bub.bin, n, bin_count);
  const int nparts = (nbins + d3::kScan - 1) / d3::kScan;
  d3::bin3_scan<<<nparts, d3::kScan, 0, stream>>>(bin_count, bin_start, bin_partial, nbins);
  d3::bin3_partials<<<1, d3::kScan, 0, stream>>>(bin_partial, nparts);
  d3::bin3_add<<<(nbins + 1 + 255) / 256, 256, 0, stream>>>(bin_start, bin_partial, nbins, nparts);
  d3::bin3_fill<<<(n + 255) / 256, 256, 0, stream>>>(bub.bin, n, bin_start, bin_count, bin_idx);
  d3::bin3_sort<<<(nbins + 255) / 256, 256, 0, stream>>>(bin_start, bin_idx, nbins);
  C3(cudaMemsetAsync(bub.pos, 0xff, sizeof(int) * n, stream));
  // Every bubble lies in some bin (the frame holds every cell index a bubble
  // inside the grid can have); those outside give -1 and no contributions.
  C3(cudaMemcpyAsync(&h_sc->next, bin_partial + nparts, sizeof(int), cudaMemcpyDeviceToHost, stream));
  C3(cudaStreamSynchronize(stream));
  const int total = h_sc->next;
  if (total > 0) d3::bin3_pos<<<(total + 255) / 256, 256, 0, stream>>>(bin_idx, total, bub.pos);
  C3(cudaGetLastError());
  launches += 7;
  bins_stale = false;
  return CRP_OK;
}

template <typename P>
crp_status Sim3Impl::launch_fdtd() {
  using V = typename P::V;
  using S = typename P::S;
  using G = typename P::G;
  const int nv = cur_v ^ 1, np = cur_p ^ 1;
  d3::Fdtd3Args<P> a;
  a.vx_old = view<V>(vx[cur_v]);
  a.vy_old = view<V>(vy[cur_v]);
  a.vz_old = view<V>(vz[cur_v]);
  a.vx_new = view<V>(vx[nv]);
  a.vy_new = view<V>(vy[nv]);
  a.vz_new = view<V>(vz[nv]);
  a.pnx = view<S>(px[cur_p]);
  a.pny = view<S>(py[cur_p]);
  a.pnz = view<S>(pz[cur_p]);
  a.px = view<S>(px[np]);
  a.py = view<S>(py[np]);
  a.pz = view<S>(pz[np]);
  a.fgA = view<G>(fg[fg_a]);
  a.fgB = view<G>(fg[fg_b]);
  a.fgC = view<G>(fg[fg_c]);
  a.tdev = d_sc->t;
  a.rho_const = stats.steps == 0 ? 1 : 0;
  a.residual = &d_sc->residual;
  const dim3 block(d3::kTX, d3::kTY);
  const dim3 grid((g.f.X + 1 + d3::kCX - 1) / d3::kCX + 1, (g.f.Y + 1 + d3::kCY - 1) / d3::kCY + 1,
                  (g.f.Z + d3::kZChunk - 1) / d3::kZChunk);
  if (!fdtd_smem_set[P::kIndex]) {
    C3(cudaFuncSetAttribute(d3::fdtd3<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)d3::kRing3Bytes));
    fdtd_smem_set[P::kIndex] = true;
  }
  if (prof_on) C3(cudaEventRecord(ev_f0, stream));
  d3::fdtd3<P><<<grid, block, d3::kRing3Bytes, stream>>>(g, a);
  C3(cudaGetLastError());
  if (prof_on) {
    C3(cudaEventRecord(ev_f1, stream));
    prof_pending = true;
  }
  launches++;
  stats.fdtd_launches++;
  return CRP_OK;
}

template <typename P>
crp_status Sim3Impl::launch_move() {
  using V = typename P::V;
  d3::move3<V><<<(bub.n + 255) / 256, 256, 0, stream>>>(g, bp, bub, view<V>(vx[cur_v]), view<V>(vy[cur_v]),
                                                         view<V>(vz[cur_v]), d_sc);
  C3(cudaGetLastError());
  launches++;
  return CRP_OK;
}

crp_status Sim3Impl::build_order() {
  const int n = bub.n;
  lpt_count<<<(n + 255) / 256, 256, 0, stream>>>(bub.nsub, n, lpt_hist);
  lpt_scan<<<1, 32, 0, stream>>>(lpt_hist, lpt_cursor);
  lpt_scatter<<<(n + kLptScatterThreads - 1) / kLptScatterThreads, kLptScatterThreads, 0, stream>>>(
      bub.nsub, n, lpt_cursor, lpt_order);
  C3(cudaGetLastError());
  launches += 3;
  return CRP_OK;
}

template <typename P>
crp_status Sim3Impl::launch_radius(int done) {
  using S = typename P::S;
  const int reuse = bp.reuse && done > 0 ? 1 : 0;
  const int* order = use_order ? lpt_order : nullptr;
  C3(cudaMemsetAsync(&d_sc->next, 0, sizeof(int), stream));
  if (cfg.ext_rp_scheme == CRP_RP_RK45)
    d3::radius3<P, true><<<rp_grid, d3::kRpThreads3, 0, stream>>>(g, bp, bub, view<S>(px[cur_p]), view<S>(py[cur_p]),
                                                                   view<S>(pz[cur_p]), d_sc, reuse, order);
  else
    d3::radius3<P, false><<<rp_grid, d3::kRpThreads3, 0, stream>>>(g, bp, bub, view<S>(px[cur_p]),
                                                                    view<S>(py[cur_p]), view<S>(pz[cur_p]), d_sc, reuse,
                                                                    order);
  C3(cudaGetLastError());
  launches++;
  return CRP_OK;
}

template <typename P>
crp_status Sim3Impl::launch_couple(bool gather, bool pressure, const int box[6]) {
  using V = typename P::V;
  using S = typename P::S;
  using G = typename P::G;
  if (box[0] > box[3] || box[1] > box[4] || box[2] > box[5]) return CRP_OK;
  d3::Couple3Args<P> a;
  a.vx = view<V>(vx[cur_v]);
  a.vy = view<V>(vy[cur_v]);
  a.vz = view<V>(vz[cur_v]);
  a.pnx = view<S>(px[cur_p ^ 1]);
  a.pny = view<S>(py[cur_p ^ 1]);
  a.pnz = view<S>(pz[cur_p ^ 1]);
  a.px = view<S>(px[cur_p]);
  a.py = view<S>(py[cur_p]);
  a.pz = view<S>(pz[cur_p]);
  a.fg = view<G>(fg[fg_a]);
  a.fgn = view<G>(fg[fg_b]);
  a.start = bin_start;
  a.contrib = bub.contrib;
  for (int q = 0; q < 6; q++) a.box[q] = box[q];
  a.gather = gather ? 1 : 0;
  a.pressure = pressure ? 1 : 0;
  a.tdev = d_sc->t;
  a.residual = &d_sc->residual;
  const dim3 block(32, 8);
  const dim3 grid((box[3] - box[0] + 32) / 32, (box[4] - box[1] + 8) / 8, box[5] - box[2] + 1);
  d3::couple3<P><<<grid, block, 0, stream>>>(g, a);
  C3(cudaGetLastError());
  launches++;
  return CRP_OK;
}

crp_status Sim3Impl::step_once() {
  t_prev = tstep;
  const double s1 = tstep;
  tstep = tstep + g.dt + tstepx;
  const double s2 = tstep - s1;
  tstepx = g.dt + tstepx - s2;
  d3::set_time3<<<1, 1, 0, stream>>>(d_sc, t_prev, tstep);
  C3(cudaGetLastError());
  launches++;
  crp_status st = mixed ? launch_fdtd<d3::PMix>() : launch_fdtd<d3::P64>();
  if (st != CRP_OK) return st;
  cur_v ^= 1;
  cur_p ^= 1;
  {
    const int a = fg_a, b = fg_b, c = fg_c;
    fg_a = c;  // predicted f_g
    fg_b = a;
    fg_c = b;
  }
  if (bub.n > 0) {
    st = mixed ? launch_move<d3::PMix>() : launch_move<d3::P64>();
    if (st != CRP_OK) return st;
  }
  C3(cudaMemcpyAsync(h_sc, d_sc, sizeof(d3::Scalars3), cudaMemcpyDeviceToHost, stream));
  C3(cudaStreamSynchronize(stream));
  if (prof_pending) {
    float ms = 0.0f;
    C3(cudaEventElapsedTime(&ms, ev_f0, ev_f1));
    stats.ms_fdtd += ms;
    prof_pending = false;
  }
  double res = as_double(h_sc->residual) / g.P_inf;
  int loop = 0;
  int bnow[6] = {1, 1, 1, 0, 0, 0};
  if (bub.n > 0) {
    bubble_box(bnow);
    if (h_sc->moved) bins_stale = true;
  }
  int box[6], u1[6], u2[6];
  box_union(u1, bnow, supp[0]);
  box_union(u2, supp[1], supp[2]);
  box_union(box, u1, u2);
  if (bub.n > 0 && res > picard_tol && bins_stale) {
    st = build_bins();
    if (st != CRP_OK) return st;
  }
  // Heaviest-first solve order from the last solves' sub-step counts, once
  // some bubble has needed more than the quiet phase's.
  use_order = bub.n > 0 && res > picard_tol && h_sc->substep_max > kLptMinSubsteps;
  if (use_order) {
    st = build_order();
    if (st != CRP_OK) return st;
  }
  if (bub.n > 0) {
    while (res > picard_tol) {
      if (loop >= cfg.ext_picard_cap) return fail(CRP_ERR_PICARD, "Picard iteration cap reached");
      loop++;
      C3(cudaMemsetAsync(&d_sc->residual, 0, sizeof(unsigned long long), stream));
      st = mixed ? launch_radius<d3::PMix>(loop - 1) : launch_radius<d3::P64>(loop - 1);
      if (st != CRP_OK) return st;
      st = mixed ? launch_couple<d3::PMix>(true, true, box) : launch_couple<d3::P64>(true, true, box);
      if (st != CRP_OK) return st;
      C3(cudaMemcpyAsync(h_sc, d_sc, sizeof(d3::Scalars3), cudaMemcpyDeviceToHost, stream));
      C3(cudaStreamSynchronize(stream));
      if (h_sc->err) return fail(CRP_ERR_RP_STEPS, "Rayleigh-Plesset sub-step cap reached");
      res = as_double(h_sc->residual) / g.P_inf;
      if (mixed && loop >= 3 && res > picard_tol && res < CRP_MIXED_STALL_RESIDUAL) {
        stats.picard_stalls++;
        break;
      }
    }
  }
  if (std::isnan(res)) return fail(CRP_ERR_NONFINITE, "non-finite pressure");
  int snow[6];
  if (loop > 0) {
    std::memcpy(snow, bnow, sizeof(snow));
  } else {
    int v1[6];
    box_union(v1, supp[0], supp[1]);
    box_union(snow, v1, supp[2]);
  }
  std::memcpy(supp[2], supp[1], sizeof(snow));
  std::memcpy(supp[1], supp[0], sizeof(snow));
  std::memcpy(supp[0], snow, sizeof(snow));
  stats.steps++;
  stats.time = tstep;
  stats.picard_last = loop;
  stats.picard_total += loop;
  stats.picard_max = std::max(stats.picard_max, loop);
  stats.residual_last = res;
  stats.rp_substeps_max = h_sc->substep_max;
  stats.rp_reused = (int64_t)h_sc->reused;
  stats.kernel_launches = launches;
  return CRP_OK;
}

// Dense copies (x fastest) of a field's logical window: cells [0, N+1] per
// axis, staggered components one more along their axis from -1.
// crp_adjoint on the 3-D grid: the forward steps with the focal p0 recorded
// after each, the objective, then the reverse sweep of the kernels above.
crp_status Sim3Impl::adjoint(const crp_objective* obj, double* J, double* grad_amp, double* grad_phase) {
  if (!obj || obj->steps <= 0 || !(obj->focal_radius > 0.0))
    return fail(CRP_ERR_INVALID, "adjoint: steps > 0 and focal_radius > 0 are required");
  if ((grad_amp || grad_phase) && elem_n == 0)
    return fail(CRP_ERR_INVALID, "adjoint: gradients need ext.array_elements > 0");
  if (bub.n > 0) return fail(CRP_ERR_UNSUPPORTED, "adjoint: bubbles off only");
  const d3::Frame3& f = g.f;
  const int N = obj->steps;
  const double r = obj->focal_radius;
  // Focal box: cell centres within r of the focus along each axis.
  const int n3[3] = {f.X, f.Y, f.Z};
  const double h3[3] = {g.dx, g.dy, g.dz};
  int lo[3], hi[3];
  bool empty = false;
  for (int ax = 0; ax < 3; ax++) {
    lo[ax] = n3[ax] + 1;
    hi[ax] = 0;
    for (int m = 1; m <= n3[ax]; m++)
      if (std::fabs(((double)m - 0.5) * h3[ax] - focus[ax]) <= r) lo[ax] = std::min(lo[ax], m), hi[ax] = std::max(hi[ax], m);
    if (hi[ax] < lo[ax]) empty = true;
  }
  if (empty)
    for (int ax = 0; ax < 3; ax++) lo[ax] = hi[ax] = 1;  // one cell of weight 0
  const int bx = hi[0] - lo[0] + 1, by = hi[1] - lo[1] + 1, bz = hi[2] - lo[2] + 1;
  const size_t box_n = (size_t)bx * by * bz;
  std::vector<double> w(box_n, 0.0);
  if (!empty)
    for (int kk = 0; kk < bz; kk++)
      for (int jj = 0; jj < by; jj++)
        for (int ii = 0; ii < bx; ii++) {
          const int i = lo[0] + ii, j = lo[1] + jj, k = lo[2] + kk;
          const double x = ((double)i - 0.5) * g.dx - focus[0], y = ((double)j - 0.5) * g.dy - focus[1],
                       z = ((double)k - 0.5) * g.dz - focus[2];
          if (x * x + y * y + z * z > r * r) continue;
          if (std::binary_search(src_list.begin(), src_list.end(), f.idx(i, j, k))) continue;  // forced cells
          w[((size_t)kk * by + jj) * bx + ii] = g.dx * g.dy * g.dz;
        }
  const size_t hist_n = (size_t)N * box_n;
  if (hist_n * sizeof(double) > ((size_t)32 << 30))
    return fail(CRP_ERR_TOO_LARGE, "adjoint: focal history above 32 GiB (steps x focal cells)");
  const int ns = (int)src_list.size(), ns1 = std::max(ns, 1);
  // Two sets of six adjoint frames, per-source-cell gradients, weights,
  // history, objective per step; then the source cells' frame indices and
  // elements.
  const size_t n_doubles = 12 * cells + 2 * (size_t)ns1 + box_n + hist_n + (size_t)N;
  const size_t bytes = n_doubles * sizeof(double) + (size_t)ns1 * (sizeof(long) + sizeof(int));
  // The workspace is kept for the next call and released with the simulation.
  if (adj_ws_bytes < bytes) {
    if (adj_ws) {
      C3(cudaStreamSynchronize(stream));
      cudaFree(adj_ws);
      adj_ws = nullptr;
      adj_ws_bytes = 0;
    }
    if (cudaMalloc(&adj_ws, bytes) != cudaSuccess) {
      cudaGetLastError();
      adj_ws = nullptr;
      return fail(CRP_ERR_ALLOC, "adjoint: device memory");
    }
    adj_ws_bytes = bytes;
  }
  char* buf = static_cast<char*>(adj_ws);
  struct Drain {  // on every return: the queued work has finished
    cudaStream_t st;
    ~Drain() { cudaStreamSynchronize(st); }
  } guard{stream};
  double* base = reinterpret_cast<double*>(buf);
  d3::Adj3 fr[2];
  for (int s = 0; s < 2; s++) {
    double* b = base + (size_t)s * 6 * cells;
    fr[s] = d3::Adj3{b, b + cells, b + 2 * cells, b + 3 * cells, b + 4 * cells, b + 5 * cells};
  }
  double* gA = base + 12 * cells;
  double* gP = gA + ns1;
  double* d_w = gP + ns1;
  double* hist = d_w + box_n;
  double* d_Jn = hist + hist_n;
  long* d_cells = reinterpret_cast<long*>(base + n_doubles);
  int* d_el = reinterpret_cast<int*>(d_cells + ns1);
  C3(cudaMemsetAsync(buf, 0, n_doubles * sizeof(double), stream));
  C3(cudaMemcpyAsync(d_w, w.data(), sizeof(double) * box_n, cudaMemcpyHostToDevice, stream));
  if (ns > 0) {
    C3(cudaMemcpyAsync(d_cells, src_list.data(), sizeof(long) * ns, cudaMemcpyHostToDevice, stream));
    C3(cudaMemcpyAsync(d_el, src_elem.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, stream));
  }
  const d3::Box3 box{lo[0], lo[1], lo[2], bx, by, bz, d_w};
  const int rb = (int)((box_n + 255) / 256);
  // Forward, recording the focal p0 after every step.
  std::vector<double> times((size_t)N + 1);
  times[0] = tstep;
  for (int n = 1; n <= N; n++) {
    const crp_status st = step_once();
    if (st != CRP_OK) return st;
    double* out = hist + (size_t)(n - 1) * box_n;
    if (mixed)
      d3::adj3_record<F32c><<<rb, 256, 0, stream>>>(f, view<F32c>(px[cur_p]), view<F32c>(py[cur_p]),
                                                      view<F32c>(pz[cur_p]), box, out);
    else
      d3::adj3_record<F64><<<rb, 256, 0, stream>>>(f, view<F64>(px[cur_p]), view<F64>(py[cur_p]),
                                                     view<F64>(pz[cur_p]), box, out);
    C3(cudaGetLastError());
    launches++;
    times[n] = tstep;
  }
  // Objective.
  d3::adj3_objective<<<N, 256, 0, stream>>>(box, hist, d_Jn);
  C3(cudaGetLastError());
  std::vector<double> Jn(N);
  C3(cudaMemcpyAsync(Jn.data(), d_Jn, sizeof(double) * N, cudaMemcpyDeviceToHost, stream));
  C3(cudaStreamSynchronize(stream));
  double Jsum = 0.0;
  for (int n = 0; n < N; n++) Jsum += Jn[n];
  if (J) *J = g.dt * Jsum;
  // Reverse sweep: reverse step n reads frame set s and writes set s ^ 1.
  const dim3 sblk(32, 8), sgrid((f.X + 31) / 32, (f.Y + 7) / 8, f.Z);
  const int sb = (ns + 255) / 256;
  const double two_dt = 2.0 * g.dt;
  d3::adj3_force<<<rb, 256, 0, stream>>>(f, fr[0], box, hist + (size_t)(N - 1) * box_n, two_dt);
  launches++;
  int s = 0;
  for (int n = N; n >= 1; n--, s ^= 1) {
    if (ns > 0) {
      d3::adj3_source<<<sb, 256, 0, stream>>>(g, fr[s], d_cells, d_el, ns, times[n], gA, gP);
      launches++;
    }
    const double* p0 = n >= 2 ? hist + (size_t)(n - 2) * box_n : nullptr;
    d3::adj3_step<<<sgrid, sblk, 0, stream>>>(g, fr[s], fr[s ^ 1], box, p0, two_dt);
    C3(cudaGetLastError());
    launches++;
  }
  if (elem_n > 0 && ns > 0) {
    std::vector<double> ca(ns), cp(ns);
    C3(cudaMemcpyAsync(ca.data(), gA, sizeof(double) * ns, cudaMemcpyDeviceToHost, stream));
    C3(cudaMemcpyAsync(cp.data(), gP, sizeof(double) * ns, cudaMemcpyDeviceToHost, stream));
    C3(cudaStreamSynchronize(stream));
    std::vector<double> sa(elem_n, 0.0), sp(elem_n, 0.0);
    for (int c = 0; c < ns; c++) {
      sa[src_elem[c]] += ca[c];
      sp[src_elem[c]] += cp[c];
    }
    if (grad_amp) std::copy(sa.begin(), sa.end(), grad_amp);
    if (grad_phase) std::copy(sp.begin(), sp.end(), grad_phase);
  } else {
    C3(cudaStreamSynchronize(stream));
    if (grad_amp) std::fill(grad_amp, grad_amp + elem_n, 0.0);
    if (grad_phase) std::fill(grad_phase, grad_phase + elem_n, 0.0);
  }
  stats.kernel_launches = launches;
  return CRP_OK;
}

crp_status Sim3Impl::read_field(crp_field w, double* host) {
  const d3::Frame3& f = g.f;
  void* buf = nullptr;
  int ilo = 0, jlo = 0, klo = 0, ihi = f.X + 1, jhi = f.Y + 1, khi = f.Z + 1;
  int kind = 0;  // 0 velocity/pressure storage, 1 void-fraction storage, 2 p0 = px + py + pz
  switch (w) {
    case CRP_FIELD_P0: kind = 2; break;
    case CRP_FIELD_PX: buf = px[cur_p]; break;
    case CRP_FIELD_PY: buf = py[cur_p]; break;
    case CRP_FIELD_PZ: buf = pz[cur_p]; break;
    case CRP_FIELD_VX: buf = vx[cur_v], ilo = -1; break;
    case CRP_FIELD_VY: buf = vy[cur_v], jlo = -1; break;
    case CRP_FIELD_VZ: buf = vz[cur_v], klo = -1; break;
    case CRP_FIELD_FG: buf = fg[fg_a], kind = 1; break;
    case CRP_FIELD_FGN: buf = fg[fg_b], kind = 1; break;
    case CRP_FIELD_FGM: buf = fg[fg_c], kind = 1; break;
    case CRP_FIELD_RHO_M: buf = fg[fg_a], kind = 3; break;
    default: return fail(CRP_ERR_UNSUPPORTED, "field not available on 3-D grids");
  }
  const int nx = ihi - ilo + 1, ny = jhi - jlo + 1, nz = khi - klo + 1;
  d3::read3<<<(nx * ny * nz + 255) / 256, 256, 0, stream>>>(
      f, kind, mixed ? 1 : 0, buf, px[cur_p], py[cur_p], pz[cur_p], ilo, jlo, klo, nx, ny, nz, g.rho_inf,
      stats.steps == 0 ? 1 : 0, scratch);
  C3(cudaGetLastError());
  C3(cudaMemcpyAsync(host, scratch, sizeof(double) * nx * ny * nz, cudaMemcpyDeviceToHost, stream));
  C3(cudaStreamSynchronize(stream));
  return CRP_OK;
}

crp_status Sim3Impl::read_bubbles(crp_bubble_field w, double* host) {
  const int n = bub.n;
  if (n == 0) return CRP_OK;
  const double* src = nullptr;
  const int* isrc = nullptr;
  switch (w) {
    case CRP_BUB_X: src = bub.x; break;
    case CRP_BUB_Y: src = bub.y; break;
    case CRP_BUB_Z: src = bub.z; break;
    case CRP_BUB_R_T: src = bub.R_t; break;
    case CRP_BUB_R_P: src = bub.R_p; break;
    case CRP_BUB_R_N: src = bub.R_n; break;
    case CRP_BUB_D1R: src = bub.d1_R_p; break;
    case CRP_BUB_PG: src = bub.PG_p; break;
    case CRP_BUB_PL_P: src = bub.PL_p; break;
    case CRP_BUB_PL_N: src = bub.PL_n; break;
    case CRP_BUB_PL_M: src = bub.PL_m; break;
    case CRP_BUB_DT: src = bub.dt; break;
    case CRP_BUB_RE: src = bub.re; break;
    case CRP_BUB_Q_B: src = bub.Q_B; break;
    case CRP_BUB_N_B: src = bub.n_B; break;
    case CRP_BUB_R0: src = bub.R0; break;
    case CRP_BUB_VX: src = bub.vbx; break;
    case CRP_BUB_VY: src = bub.vby; break;
    case CRP_BUB_VZ: src = bub.vbz; break;
    case CRP_BUB_IBM_X: isrc = bub.ibmx; break;
    case CRP_BUB_IBM_Y: isrc = bub.ibmy; break;
    case CRP_BUB_IBM_Z: isrc = bub.ibmz; break;
    case CRP_BUB_IBN_X: isrc = bub.ibnx; break;
    case CRP_BUB_IBN_Y: isrc = bub.ibny; break;
    case CRP_BUB_IBN_Z: isrc = bub.ibnz; break;
    case CRP_BUB_SUBSTEPS: isrc = bub.nsub; break;
    default: return fail(CRP_ERR_INVALID, "unknown bubble field");
  }
  if (src) {
    C3(cudaMemcpyAsync(host, src, sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
    C3(cudaStreamSynchronize(stream));
    return CRP_OK;
  }
  std::vector<int> tmp(n);
  C3(cudaMemcpyAsync(tmp.data(), isrc, sizeof(int) * n, cudaMemcpyDeviceToHost, stream));
  C3(cudaStreamSynchronize(stream));
  for (int k = 0; k < n; k++) host[k] = (double)tmp[k];
  return CRP_OK;
}

crp_status Sim3Impl::set_elements(int n, const double* amp, const double* phase) {
  if (n != elem_n || n <= 0 || !amp || !phase) return fail(CRP_ERR_INVALID, "element count mismatch");
  std::vector<double> v(amp, amp + n);
  v.insert(v.end(), phase, phase + n);
  C3(cudaMemcpyAsync(d_elem, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice, stream));
  C3(cudaStreamSynchronize(stream));
  return CRP_OK;
}

// C-ABI glue used by sim.cu's entry points.
crp_status sim3_create(const crp_config* cfg, const crp_bubbles_in* bubbles, void* stream, Sim3Impl** out,
                       std::string* err) {
  Sim3Impl* s = new (std::nothrow) Sim3Impl();
  if (!s) return CRP_ERR_ALLOC;
  const crp_status st = s->create(*cfg, bubbles, stream);
  if (st != CRP_OK) {
    if (err) *err = s->err;
    delete s;
    return st;
  }
  *out = s;
  return CRP_OK;
}
void sim3_destroy(Sim3Impl* s) { delete s; }
crp_status sim3_step(Sim3Impl* s, int n) {
  for (int k = 0; k < n; k++) {
    const crp_status st = s->step_once();
    if (st != CRP_OK) return st;
  }
  return CRP_OK;
}
crp_status sim3_read_field(Sim3Impl* s, crp_field w, double* host) { return s->read_field(w, host); }
crp_status sim3_read_bubbles(Sim3Impl* s, crp_bubble_field w, double* host) { return s->read_bubbles(w, host); }
crp_status sim3_set_elements(Sim3Impl* s, int n, const double* amp, const double* phase) {
  return s->set_elements(n, amp, phase);
}
void sim3_dims(const Sim3Impl* s, crp_dims3* d) {
  d->nx = s->g.f.X + 2;
  d->ny = s->g.f.Y + 2;
  d->nz = s->g.f.Z + 2;
  d->num_bubbles = s->bub.n;
  d->dx = s->g.dx;
  d->dy = s->g.dy;
  d->dz = s->g.dz;
  d->dt = s->g.dt;
  d->source_cells = s->src_cells;
}
const crp_stats& sim3_stats(const Sim3Impl* s) { return s->stats; }
const char* sim3_error(const Sim3Impl* s) { return s->err.c_str(); }
crp_status sim3_set_profiling(Sim3Impl* s, int on) { return s->set_profiling(on != 0); }
void* sim3_stream(Sim3Impl* s) { return (void*)s->stream; }

// Snapshots: the device pool, and the host-side step state beside it.
struct HostState3 {
  int cur_v, cur_p, fg_a, fg_b, fg_c, bins_stale;
  double tstep, tstepx, t_prev;
  int supp[3][6];
  crp_stats stats;
  d3::Scalars3 hsc;
};
size_t sim3_state_bytes(const Sim3Impl* s) { return s->pool_bytes; }
crp_status sim3_save_state(Sim3Impl* s, void* blob, std::vector<unsigned char>& host) {
  if (cudaMemcpyAsync(blob, s->pool, s->pool_bytes, cudaMemcpyDeviceToDevice, s->stream) != cudaSuccess ||
      cudaStreamSynchronize(s->stream) != cudaSuccess)
    return s->fail(CRP_ERR_CUDA, "state: device copy");
  HostState3 h{};
  h.cur_v = s->cur_v, h.cur_p = s->cur_p, h.fg_a = s->fg_a, h.fg_b = s->fg_b, h.fg_c = s->fg_c;
  h.bins_stale = s->bins_stale ? 1 : 0;
  h.tstep = s->tstep, h.tstepx = s->tstepx, h.t_prev = s->t_prev;
  std::memcpy(h.supp, s->supp, sizeof(h.supp));
  h.stats = s->stats;
  h.hsc = *s->h_sc;
  host.resize(sizeof(HostState3));
  std::memcpy(host.data(), &h, sizeof(HostState3));
  return CRP_OK;
}
crp_status sim3_load_state(Sim3Impl* s, const void* blob, const std::vector<unsigned char>& host) {
  if (host.size() != sizeof(HostState3)) return s->fail(CRP_ERR_INVALID, "state: host part of the wrong size");
  HostState3 h;
  std::memcpy(&h, host.data(), sizeof(HostState3));
  if (cudaMemcpyAsync(s->pool, blob, s->pool_bytes, cudaMemcpyDeviceToDevice, s->stream) != cudaSuccess ||
      cudaStreamSynchronize(s->stream) != cudaSuccess)
    return s->fail(CRP_ERR_CUDA, "state: device copy");
  s->cur_v = h.cur_v, s->cur_p = h.cur_p, s->fg_a = h.fg_a, s->fg_b = h.fg_b, s->fg_c = h.fg_c;
  s->bins_stale = h.bins_stale != 0;
  s->tstep = h.tstep, s->tstepx = h.tstepx, s->t_prev = h.t_prev;
  std::memcpy(s->supp, h.supp, sizeof(h.supp));
  const crp_stats keep = s->stats;
  s->stats = h.stats;
  s->stats.kernel_launches = keep.kernel_launches;
  s->stats.fdtd_launches = keep.fdtd_launches;
  s->stats.rp_launches = keep.rp_launches;
  s->stats.couple_launches = keep.couple_launches;
  s->stats.ms_fdtd = keep.ms_fdtd, s->stats.ms_rp = keep.ms_rp, s->stats.ms_couple = keep.ms_couple;
  s->stats.ms_other = keep.ms_other;
  *s->h_sc = h.hsc;
  return CRP_OK;
}
crp_status sim3_set_tuning(Sim3Impl* s, const crp_tuning* t) {
  if (t->fdtd_rows != 4 && t->fdtd_rows != 8 && t->fdtd_rows != 16)
    return s->fail(CRP_ERR_INVALID, "tuning: fdtd_rows must be 4, 8 or 16");
  if (t->rp_blocks < 0) return s->fail(CRP_ERR_INVALID, "tuning: rp_blocks must be >= 0");
  s->rp_blocks_req = t->rp_blocks;
  s->rp_grid = t->rp_blocks > 0 ? std::min(t->rp_blocks, s->rp_grid_full) : s->rp_grid_full;
  return CRP_OK;
}
crp_status sim3_adjoint(Sim3Impl* s, const crp_objective* obj, double* J, double* grad_amp, double* grad_phase) {
  return s->adjoint(obj, J, grad_amp, grad_phase);
}
void sim3_get_tuning(const Sim3Impl* s, crp_tuning* t) {
  t->fdtd_rows = 8;
  t->rp_blocks = s->rp_blocks_req;
  t->rp_blocks_max = s->rp_grid_full;
}
int sim3_device(const Sim3Impl* s) { return s->device; }

}  // namespace crp
