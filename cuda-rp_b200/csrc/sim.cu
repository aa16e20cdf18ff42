// B200 implementation of CUDA-RP's simulation path behind the crp C ABI.
//
// One mixture time step (the main loop of solve_bubbles, src/bubble_CUDA.cu:206-285):
//   fdtd_strip     fused: void-fraction prediction, velocity update with its
//                  boundary overrides (VelocityKernel, VelocityBoundaryKernel),
//                  first pressure evaluation (MixturePressureKernel) and its
//                  residual, one HBM pass in column strips
//   vghost         velocity ghost cells (the rest of VelocityBoundaryKernel),
//                  a launch of its own only without bubbles
//   bubble_move    bubble state rotation (store_variables), velocity gather,
//                  motion, cell indices, occupied-bin box; its last blocks
//                  write the velocity ghost cells
//   bin_*          counting sort of bubbles by cell (deterministic order), only
//                  when a bubble changed cell
//   lpt_*          radius-solve order, heaviest sub-step counts first
//   Picard loop while max|dp0|/P_inf > 1e-7 (src/bubble_CUDA.cu:243):
//     bubble_rp    pressure gather + Rayleigh-Plesset sub-stepping + the void
//                  fraction contribution of each bubble to its four cells,
//                  persistent with a work queue
//     couple_press gather of the void fraction per cell (no atomics), axis fold,
//                  pressure re-evaluation and residual, over the cells whose
//                  void fraction can be nonzero
// Buffers rotate instead of being copied: velocity and pressure ping-pong, the
// void-fraction history is a three-buffer ring.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "crp.h"
#include "crp_device.cuh"
#include "radius.cuh"
#include "adjoint.cuh"
#include "crp_host.h"
#include "sim3d.h"

namespace crp {

// ---------------------------------------------------------------------------
// Storage of each field class and the real type of the bubble thermal model.
struct PrecFP64 {
  using V = F64;  // velocity
  using S = F64;  // split pressure
  using G = F64;  // void fraction
  using T = double;
};
struct PrecMixed {
  using V = F32c;
  using S = F32c;
  using G = F32;
  using T = float;
};

template <typename P>
struct FdtdArgs {
  typename P::V vx_old, vy_old, vx_new, vy_new;
  typename P::S pnx, pny;  // pressure of the previous step
  typename P::S px, py;    // pressure of this step
  typename P::G fgA;       // f_g of the previous step (becomes f_gn)
  typename P::G fgB;       // f_gn of the previous step
  typename P::G fgC;       // f_gm of the previous step; receives the predicted f_g
  const double* tdev;  // {t_prev, t_cur} of this step, in device memory
  int rho_const;           // first step: the mixture density is still rho_inf everywhere
  unsigned long long* residual;
};

__device__ __forceinline__ void block_max_to(double v, unsigned long long* out) {
  // Non-negative doubles order like their bit patterns; NaN (|NaN|) sorts above all.
  unsigned long long b = (unsigned long long)__double_as_longlong(v);
  for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
  __shared__ unsigned long long s_red[32];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int lane = tid & 31, w = tid >> 5;
  if (lane == 0) s_red[w] = b;
  __syncthreads();
  if (w == 0) {
    int nw = (blockDim.x * blockDim.y + 31) >> 5;
    b = lane < nw ? s_red[lane] : 0ull;
    for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
    if (lane == 0 && b) atomicMax(out, b);
  }
}

// q = dt / mean(rho) of a face of VelocityKernel (inc/bubble_CUDA_kernel.cuh:
// 660-662, 670-672); dt / rho_inf, without its division, where both densities
// are rho_inf.
__device__ __forceinline__ double face_q(const GridParams& g, double rhoa, double rhob) {
  return (rhoa == g.rho_inf && rhob == g.rho_inf) ? g.dt_rho : g.dt / ((rhoa + rhob) * 0.5);
}
// Velocity update of VelocityKernel (:658-676) for one face:
// (v_old (1 - s3) - q s2) / (1 + s3), with the face's PML factors fa = 1 - s3
// and fb = 1 / (1 + s3) precomputed on the host.  Outside the PML both are
// exactly 1 and the value is the reference's v_old - q s2; inside, the
// multiplication by fb in place of the division changes it by at most one
// rounding.
__device__ __forceinline__ double velocity_face_q(const GridParams& g, double v_old, double p0a, double p0b, double q,
                                                  double fa, double fb) {
  const double s2 = (-p0a + p0b) * g.rdx;  // rdx on both faces, as :661 and :671
  return (v_old * fa - q * s2) * fb;
}

// Split-pressure update of MixturePressureKernel (:856-859) for one component:
// pn (1 - s2) - s3 (s1 + s5/2) / (1 + s2), with s2 = dt c sigma / 2 and the
// component's PML factors fa = 1 - s2, fb = 1 / (1 + s2) (as velocity_face).
__device__ __forceinline__ double pressure_component(const GridParams& g, double pn, double fa, double fb, double s1,
                                                     double h) {
  return pn * fa - g.s3p * (s1 + h) * fb;
}

// s5 / 2 of :854: the void-fraction rate term; zero where f_g stays zero.
__device__ __forceinline__ double void_rate_half(const GridParams& g, double fg, double fgn) {
  if (fg == 0.0 && fgn == 0.0) return 0.0;
  return 0.5 * (-(fg - fgn) / g.dt / (1.0 - 0.5 * (fg + fgn)));
}

// The rarely taken parts of the strip update live in out-of-line functions so
// that their transcendental code does not raise the register count of the
// update loop.
//
// North face jf on the y0 face or the [ext] source row (VelocityBoundaryKernel
// :734-798): v is the face from the update; pre receives the face before the
// y0 source overwrites it (the value the reference mirrors into row -1).
__device__ __noinline__ double vy_face_special(const GridParams& g, int jf, double v, double xm, double t_cur,
                                               double* pre) {
  if (jf == 0 && !g.pml_y0) {
    if (!src_pressure(g)) v = 0.0;
    *pre = v;
    double s;
    if (g.source_row == 0 && source_value(g, false, xm, 0.0, t_cur, s)) v = s;
  }
  if (g.source_row > 0 && jf == g.source_row) {
    double s;
    if (source_value(g, false, xm, (double)g.source_row * g.dy, t_cur, s)) v = s;
  }
  return v;
}

// North face jf of a column (VelocityKernel :668-676 with the y sections of
// VelocityBoundaryKernel): y0 wall or source, [ext] source row, y1 wall.
// q: dt / mean(rho) of the face (face_q).
__device__ __forceinline__ double vy_face_value_f(const GridParams& g, int jf, double v_old, double p0a, double p0b,
                                                  double q, double fa, double fb, double xm, double t_cur,
                                                  double& pre) {
  double v = velocity_face_q(g, v_old, p0a, p0b, q, fa, fb);
  pre = v;
  if ((jf == 0 && !g.pml_y0) || (g.source_row > 0 && jf == g.source_row)) v = vy_face_special(g, jf, v, xm, t_cur, &pre);
  if (jf == g.f.Y && !g.pml_y1) v = 0.0;
  return v;
}
__device__ __forceinline__ double vy_face_value(const GridParams& g, int jf, double v_old, double p0a, double p0b,
                                                double q, double xm, double t_cur, double& pre) {
  double v = velocity_face_q(g, v_old, p0a, p0b, q, g.vay[jf + 1], g.vby[jf + 1]);
  pre = v;
  if ((jf == 0 && !g.pml_y0) || (g.source_row > 0 && jf == g.source_row)) v = vy_face_special(g, jf, v, xm, t_cur, &pre);
  if (jf == g.f.Y && !g.pml_y1) v = 0.0;
  return v;
}

template <typename S>
__device__ __noinline__ double p0_edge(const GridParams& g, const S px, const S py, int i, int j, double t) {
  return p0_at(g, px, py, i, j, t);
}

// Pressure source value on the [ext] source row.
__device__ __noinline__ double source_row_pressure(const GridParams& g, double xm, double t) {
  double sv = 0.0;
  source_value(g, true, xm, ((double)g.source_row - 0.5) * g.dy, t, sv);
  return sv;
}

// One mixture step of the grid, fused: void-fraction prediction (store_variables,
// src/bubble_CUDA.cu:1160-1162), VelocityKernel with VelocityBoundaryKernel's
// faces (inc/bubble_CUDA_kernel.cuh:658-798), MixturePressureKernel with the
// predicted void fraction (:816-867) and the residual of calculate_pressure_field.
// The work is organised as column strips.  A warp holds the
// 32 adjacent columns i = 30 s + lane of strip s and marches up a chunk of
// kStripRows rows: lanes 1..30 update their cells, lanes 0 and 31 only provide
// the values across the strip's edges.  Left/right neighbour values arrive by
// warp shuffle, the row below stays in registers, so every array element is
// read once per step (the two edge columns of a strip and the row under a
// chunk once more, from L2), with 256-byte coalesced rows per warp load.  Rows
// are staged through a per-warp ring of kStripStages rows in shared memory by
// asynchronous copies issued kStripStages - 2 rows ahead, so each warp keeps
// the next rows of all seven input arrays in flight while it computes.
//
// The kernel is bound by the latency of each row's dependent chain rather than
// by bytes, so its instruction stream is kept short: element offsets are 32-bit
// (the host rejects frames of 2^32 elements or more), one add per row; lanes
// past the window stage a copy of column X+1 instead of branching around
// their copies; only the stores are predicated.  The row loop stays rolled (an
// unrolled chunk measured slower).
constexpr int kStripCells = 30;
constexpr int kStripWarps = 4;
constexpr int kStripRows = 8;    // rows per chunk (measured best of 4-16 at 1024 x 2048)
constexpr int kStripStages = 4;  // ring slots (rows) per warp; a smaller ring leaves more L1 (measured)
constexpr int kStripFields = 7;  // pnx, pny, fgA, vx_old, vy_old, fgB, fgC

template <typename P, int STAGES = kStripStages, int ROWS = kStripRows, int MINB = 4>
__global__ void __launch_bounds__(32 * kStripWarps, MINB) fdtd_strip(const __grid_constant__ GridParams g,
                                                               const FdtdArgs<P> a) {
  using G = typename P::G;
  using S = typename P::S;
  using V = typename P::V;
  __shared__ __align__(16) double ring[kStripWarps][STAGES][kStripFields][32];
  const Frame& f = g.f;
  const int X = f.X, Y = f.Y;
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x;
  const int i = (blockIdx.x * kStripWarps + threadIdx.y) * kStripCells + lane;
  const double t_prev = a.tdev[0], t_cur = a.tdev[1];
  const bool inwin = i <= X + 1;                                 // column inside the window [0, X+1]
  const bool cell = lane >= 1 && lane <= kStripCells && i <= X;  // updates cell (i, j)
  const bool face = lane <= kStripCells && i <= X;               // east face F(i) needed
  // Owner of the f_g prediction of this column.
  const bool own = inwin && ((lane >= 1 && lane <= kStripCells) || (lane == 0 && i == 0) ||
                             (lane == 31 && i == X + 1));
  // Chunks are taken alternately from the bottom and the top of the grid, so
  // that the PML bands at both y ends (the slowest chunks: general updates
  // with divisions) start first and the cheap interior chunks fill the tail.
  const int by = blockIdx.y, cy = (by & 1) ? (int)gridDim.y - 1 - (by >> 1) : (by >> 1);
  const int j0 = 1 + cy * ROWS;
  const int j1 = min(Y, j0 + ROWS - 1);
  const double xm = ((double)i - 0.5) * g.dx;
  const bool inner_col = i >= 1 && i <= X;
  const bool src_rows = g.source_row > 0 && src_pressure(g);
  // Offset of element (min(i, X+1), j0 - 1 + rr) is kb + rr * pitch.
  const unsigned pitch = (unsigned)f.pitch;
  const unsigned kb = (unsigned)j0 * pitch + (unsigned)(min(i, X + 1) + 1);
  auto p0_of = [&](int r, double px_, double py_) -> double {
    if (inner_col && r >= 1 && r <= Y && !(src_rows && r == g.source_row)) return px_ + py_;
    if (!inwin) return 0.0;
    return p0_edge(g, a.pnx, a.pny, i, r, t_prev);
  };
  auto rho_of = [&](double fa) -> double { return a.rho_const ? g.rho_inf : (1.0 - fa) * g.rho_inf; };
  auto predict = [&](long k, double fa) -> double {
    const double v = G::stored(3.0 * fa - 3.0 * a.fgB.get(k) + a.fgC.get(k));
    a.fgC.put(k, v);
    return v;
  };
  // Ring slot of field fld of chunk row rr (row j0 - 1 + rr); each lane only
  // touches its own column.
  auto slot = [&](int rr, int fld) -> double* { return &ring[threadIdx.y][rr % STAGES][fld][lane]; };
  // Queue the copies of chunk row rr: pnx, pny, fgA for rows j0-1..j1+1,
  // vy_old for j0-1..j1, vx_old, fgB, fgC for j0..j1.  One commit group per
  // row, empty past the chunk, so that a fixed wait count always means "the
  // next row landed".
  auto issue = [&](int rr) {
    const int r = j0 - 1 + rr;
    if (rr <= ROWS + 1 && r <= j1 + 1) {
      const unsigned k = kb + (unsigned)rr * pitch;
      a.pnx.stage(slot(rr, 0), k);
      a.pny.stage(slot(rr, 1), k);
      a.fgA.stage(slot(rr, 2), k);
      if (r <= j1) {
        a.vy_old.stage(slot(rr, 4), k);
        if (rr >= 1) {
          a.vx_old.stage(slot(rr, 3), k);
          a.fgB.stage(slot(rr, 5), k);
          a.fgC.stage(slot(rr, 6), k);
        }
      }
    }
    __pipeline_commit();
  };
#pragma unroll
  for (int rr = 0; rr < STAGES; rr++) issue(rr);
  __pipeline_wait_prior(STAGES - 2);  // rows j0-1 and j0 have landed

  // Row below the chunk and the chunk's first row.
  double pxc, pyc, fac, p0b, rhob, vyob;
  {
    const double pxb = S::staged(slot(0, 0)), pyb = S::staged(slot(0, 1));
    const double fab = G::staged(slot(0, 2));
    vyob = V::staged(slot(0, 4));
    pxc = S::staged(slot(1, 0));
    pyc = S::staged(slot(1, 1));
    fac = G::staged(slot(1, 2));
    p0b = p0_of(j0 - 1, pxb, pyb);
    rhob = rho_of(fab);
    if (j0 == 1 && own) predict(f.idx(i, 0), fab);
  }
  issue(STAGES);  // reuses the slot of row j0-1
  double p0c = p0_of(j0, pxc, pyc), rhoc = rho_of(fac);
  double vyd = 0.0;
  if (cell) {
    double pre_d;
    vyd = vy_face_value(g, j0 - 1, vyob, p0b, p0c, face_q(g, rhob, rhoc), xm, t_cur, pre_d);
    if (j0 == 1) {
      a.vy_new.put(f.idx(i, 0), vyd);
      if (!g.pml_y0) a.vy_new.put(f.idx(i, -1), pre_d);
    }
  }

  // Per-column coefficients: PML factors of the east face and of the cell's x
  // component, and the cylindrical metrics.
  const double vax_e = face ? g.vax[i + 1] : 1.0, vbx_e = face ? g.vbx[i + 1] : 1.0;
  const double pax_c = cell ? g.pax[i] : 1.0, pbx_c = cell ? g.pbx[i] : 1.0;
  const double xu_w = cell && g.cyl ? g.xu[i] : 0.0, xu_e = cell && g.cyl ? g.xu[i + 1] : 0.0;
  const double rxp_c = cell && g.cyl ? g.rxp[i] : 0.0;
  const bool zero_e = (i == 0 && !g.pml_x0) || (i == X && !g.pml_x1);

  // One form of the updates serves every cell: the PML factors are exactly 1
  // outside the PML, and the divisions of the mixture density and of the
  // void-fraction rate run only in warps that hold void fraction (a branch
  // taken by the whole warp or skipped by it).  Special y faces (the y0 wall or
  // source face, the source row) are whole rows, so their branch is uniform
  // across the warp too.
  unsigned long long res = 0ull;  // max |dp0| as a bit pattern (NaN sorts above every number)
#pragma unroll 1
  for (int jj = 0; jj < ROWS; jj++) {
    const int j = j0 + jj;
    if (j > j1) break;
    const unsigned k = kb + (unsigned)(jj + 1) * pitch;  // (i, j) for every lane that stores
    __pipeline_wait_prior(STAGES - 2);              // row j+1 has landed
    const double pxn = S::staged(slot(jj + 2, 0)), pyn = S::staged(slot(jj + 2, 1));
    const double fan = G::staged(slot(jj + 2, 2));
    const double vxo = V::staged(slot(jj + 1, 3)), vyo = V::staged(slot(jj + 1, 4));
    const double fgp = G::stored(3.0 * fac - 3.0 * G::staged(slot(jj + 1, 5)) + G::staged(slot(jj + 1, 6)));
    if (own) a.fgC.put(k, fgp);
    const double p0n = p0_of(j + 1, pxn, pyn), rhon = rho_of(fan);
    const double p0r = __shfl_down_sync(full, p0c, 1), rhor = __shfl_down_sync(full, rhoc, 1);
    // dt / mean(rho) of the east and north faces and the void-fraction rate h.
    double q_e = g.dt_rho, q_n = g.dt_rho, h = 0.0;
    if (__any_sync(full, rhoc != g.rho_inf || rhor != g.rho_inf || rhon != g.rho_inf || fgp != 0.0 || fac != 0.0)) {
      q_e = face_q(g, rhoc, rhor);
      q_n = face_q(g, rhoc, rhon);
      h = void_rate_half(g, fgp, fac);
    }
    double fe = velocity_face_q(g, vxo, p0c, p0r, q_e, vax_e, vbx_e);
    if (zero_e) fe = 0.0;
    const double fw = __shfl_up_sync(full, fe, 1);
    double pre_u;
    const double vyu = vy_face_value(g, j, vyo, p0c, p0n, q_n, xm, t_cur, pre_u);
    const double s1x = g.cyl ? (-xu_w * fw + xu_e * fe) * g.rdx * rxp_c : (-fw + fe) * g.rdx;
    const double s1y = (-vyd + vyu) * g.rdy;
    const double qx = pressure_component(g, pxc, pax_c, pbx_c, s1x, h);
    const double qy = pressure_component(g, pyc, g.pay[j], g.pby[j], s1y, h);
    if (cell) {
      a.vx_new.put(k, fe);
      a.vy_new.put(k, vyu);
      a.px.put(k, qx);
      a.py.put(k, qy);
      double p0new = qx + qy;
      if (src_rows && j == g.source_row) p0new = source_row_pressure(g, xm, t_cur);
      res = max(res, (unsigned long long)__double_as_longlong(fabs(p0c - p0new)));
    } else if (lane == 0 && i == 0) {
      a.vx_new.put(k, fe);  // the x0 face, vx(0, j)
    }
    vyd = vyu;
    pxc = pxn;
    pyc = pyn;
    fac = fan;
    p0c = p0n;
    rhoc = rhon;
    issue(jj + 1 + STAGES);  // reuses the slot of row j
  }
  if (j1 == Y && own) predict(f.idx(i, Y + 1), fac);
  // Warp maximum, one atomic per warp with a nonzero residual (no block
  // barrier: the warps of a block finish their strips at different times).
  for (int o = 16; o > 0; o >>= 1) res = max(res, __shfl_xor_sync(0xffffffffu, res, o));
  if (lane == 0 && res) atomicMax(a.residual, res);
}

}  // namespace crp
#include "fdtd_tma.cuh"
namespace crp {

// Velocity ghost cells (VelocityBoundaryKernel, inc/bubble_CUDA_kernel.cuh:701-811,
// the parts outside the faces the update computes).  Each value is written in
// closed form from computed faces, in the section order of the reference;
// thread k of the launch writes the k-th cell of each ghost row and column.
template <typename V>
__device__ __forceinline__ void vghost_cells(const GridParams& g, const V& vx, const V& vy, int k) {
  const Frame& f = g.f;
  const int X = f.X, Y = f.Y;
  // vx after the x-face section (:702-721), for rows 1..Y.
  auto vxA = [&](int i, int j) -> double {
    if (i == -1) return g.pml_x0 ? 0.0 : vx.get(f.idx(1, j));
    if (i == X + 1) return g.pml_x1 ? 0.0 : -vx.get(f.idx(X - 1, j));
    return vx.get(f.idx(i, j));
  };
  // vy after the y-face section (:734-798).
  auto vyC = [&](int i, int j) -> double {
    if (j == Y + 1) return g.pml_y1 ? 0.0 : vy.get(f.idx(i, Y - 1));
    return vy.get(f.idx(i, j));
  };
  if (k >= 1 && k <= Y) {
    if (!g.pml_x0) vx.put(f.idx(-1, k), vx.get(f.idx(1, k)));
    if (!g.pml_x1) vx.put(f.idx(X + 1, k), -vx.get(f.idx(X - 1, k)));
  }
  if (k <= X + 2) {
    int i = k - 1;
    vx.put(f.idx(i, 0), vxA(i, 1));
    vx.put(f.idx(i, Y + 1), vxA(i, Y));
  }
  if (k >= 1 && k <= X && !g.pml_y1) vy.put(f.idx(k, Y + 1), vy.get(f.idx(k, Y - 1)));
  if (k <= Y + 2) {
    int j = k - 1;
    vy.put(f.idx(0, j), vyC(1, j));
    // The X1 mirror reads row X+1 of the array, logical (X, X) (:808).
    vy.put(f.idx(X + 1, j), (X <= Y + 1) ? vyC(X, X) : vyC(X, j));
  }
}

// Threads for vghost_cells: max(X, Y) + 3 cover every ghost row and column.
__host__ __device__ __forceinline__ int vghost_threads(const Frame& f) { return (f.X > f.Y ? f.X : f.Y) + 3; }

template <typename V>
__global__ void vghost(const __grid_constant__ GridParams g, const V vx, const V vy) {
  vghost_cells(g, vx, vy, blockIdx.x * blockDim.x + threadIdx.x);
}

// The values vghost_cells leaves in the ghost cells, formed from the computed
// faces (and the stored value where it writes none), so that a kernel can read
// the velocity stencil in the same launch that writes the ghost cells.  Copies
// and sign changes only: equal to what a read after vghost_cells returns.
template <typename V>
__device__ __forceinline__ double vx_final(const GridParams& g, const V& vx, int i, int j) {
  const Frame& f = g.f;
  const int X = f.X, Y = f.Y;
  if (j == 0 || j == Y + 1) j = j == 0 ? 1 : Y;  // rows 0 and Y+1: vxA(i, 1), vxA(i, Y)
  else if (!((i == -1 && !g.pml_x0) || (i == X + 1 && !g.pml_x1))) return vx.get(f.idx(i, j));
  if (i == -1) return g.pml_x0 ? 0.0 : vx.get(f.idx(1, j));
  if (i == X + 1) return g.pml_x1 ? 0.0 : -vx.get(f.idx(X - 1, j));
  return vx.get(f.idx(i, j));
}
template <typename V>
__device__ __forceinline__ double vy_final(const GridParams& g, const V& vy, int i, int j) {
  const Frame& f = g.f;
  const int X = f.X, Y = f.Y;
  if (i == 0) i = 1;  // column 0: vyC(1, j)
  else if (i == X + 1) {  // column X+1: vyC(X, X) or vyC(X, j)
    if (X <= Y + 1) j = X;
    i = X;
  } else if (j != Y + 1 || g.pml_y1) {
    return vy.get(f.idx(i, j));
  }
  if (j == Y + 1) return g.pml_y1 ? 0.0 : vy.get(f.idx(i, Y - 1));
  return vy.get(f.idx(i, j));
}

struct BubbleArrays {
  double *x, *y, *R_t, *R_p, *R_pn, *R_n, *R_nn, *d1_R_p, *d1_R_n, *PG_p, *PG_n, *PL_p, *PL_n, *PL_m, *Q_B, *n_B,
      *dt, *dt_n, *re, *re_n, *vbx, *vby, *R0, *contrib;
  int *ibmx, *ibmy, *ibnx, *ibny, *bin, *nsub;
  // Position of each bubble in the sorted bins (-1: outside every bin).  A
  // bubble's four stencil contributions are stored at 4 * pos, so that each
  // cell gathers contiguous runs.
  int* pos;
  int n;
};

struct Bins {
  int nbx, nby, nbins;
  int* count;   // nbins, zero between steps
  int* start;   // nbins + 1
  int* idx;     // n
  int* partial; // scan block sums
};

__device__ __forceinline__ int bin_of(const Frame& f, int bx, int by) {
  if (bx < -1 || bx > f.X + 1 || by < -1 || by > f.Y + 1) return -1;
  return (by + 1) * (f.X + 3) + (bx + 1);
}

// store_variables' bubble rotation (inc/bubble_CUDA_kernel.cuh:1241-1248),
// BubbleInterpolationVelocityKernel (:398-448) and BubbleMotionKernel (:451-468),
// plus the cell count for the bin sort.
constexpr int kBoxOff = 4;

constexpr int kMoveThreads = 256;
// Resident blocks per SM the register budget is set for: 7 x 148 SMs hold the
// 1024 blocks of 262,144 bubbles plus the ghost-cell blocks in one wave (at
// the unbounded 48 registers only 5 fit, and the launch took 1.4 waves).
constexpr int kMoveMinBlocks = 7;

template <typename V>
__device__ __forceinline__ void move_one(const GridParams& g, const BubbleParams& bp, const BubbleArrays& b,
                                         const V& vx, const V& vy, int* __restrict__ moved, int n, int* s_box) {
  const Frame& f = g.f;
  b.R_pn[n] = b.R_p[n];
  b.R_nn[n] = b.R_n[n];
  b.d1_R_n[n] = b.d1_R_p[n];
  b.PG_n[n] = b.PG_p[n];
  b.PL_m[n] = b.PL_n[n];
  b.PL_n[n] = b.PL_p[n];
  b.dt_n[n] = b.dt[n];
  b.re_n[n] = b.re[n];
  double x = b.x[n], y = b.y[n];
  int imx = b.ibmx[n], imy = b.ibmy[n], inx = b.ibnx[n], iny = b.ibny[n];
  double vlx = 0.0, vly = 0.0;
  // Delta weights of the two rows/columns of each stencil, from one cosine per
  // axis (delta_w).
  const double cx0 = delta_cos_x(bp, g, imx - 1, x), cy0 = delta_cos_y(bp, g, imy - 1, y);
  const double dyn[2] = {delta_w(bp, cy0, iny - (imy - 1)), delta_w(bp, cy0, iny + 1 - (imy - 1))};
  const double dym[2] = {delta_w(bp, cy0, 0), delta_w(bp, cy0, 1)};
#pragma unroll
  for (int qi = 0; qi < 2; qi++) {
    const int i = imx - 1 + qi;
    const double dxw = delta_w(bp, cx0, qi);
#pragma unroll
    for (int qj = 0; qj < 2; qj++) {
      const int j = iny + qj;
      if (i >= -1 && i <= f.X + 1 && j >= 0 && j <= f.Y + 1) vlx += vx_final(g, vx, i, j) * dxw * dyn[qj];
    }
  }
#pragma unroll
  for (int qi = 0; qi < 2; qi++) {
    const int i = inx + qi;
    const double dxw = delta_w(bp, cx0, i - (imx - 1));
#pragma unroll
    for (int qj = 0; qj < 2; qj++) {
      const int j = imy - 1 + qj;
      if (i >= 0 && i <= f.X + 1 && j >= -1 && j <= f.Y + 1) vly += vy_final(g, vy, i, j) * dxw * dym[qj];
    }
  }
  b.vbx[n] = vlx;
  b.vby[n] = vly;
  x = x + vlx * g.dt;
  y = y + vly * g.dt;
  b.x[n] = x;
  b.y[n] = y;
  b.ibmx[n] = (int)floor(x * g.rdx + 1.0);
  b.ibmy[n] = (int)floor(y * g.rdy + 1.0);
  inx = (int)floor(x * g.rdx + 0.5);
  iny = (int)floor(y * g.rdy + 0.5);
  b.ibnx[n] = inx;
  b.ibny[n] = iny;
  const int c = bin_of(f, inx, iny);
  {
    // Bounding box of the occupied bins, encoded so that every value is
    // positive and zero means "no bubble": moved[1..4] receive the maxima of
    // kBoxOff - bx, kBoxOff + bx, kBoxOff - by, kBoxOff + by (warp, then
    // block, then one atomic per block).
    const bool in = c >= 0;
    const unsigned m = __activemask();
    const int e0 = __reduce_max_sync(m, in ? kBoxOff - inx : 0), e1 = __reduce_max_sync(m, in ? kBoxOff + inx : 0);
    const int e2 = __reduce_max_sync(m, in ? kBoxOff - iny : 0), e3 = __reduce_max_sync(m, in ? kBoxOff + iny : 0);
    if ((threadIdx.x & 31) == __ffs(m) - 1 && e1 > 0) {
      atomicMax(s_box + 0, e0);
      atomicMax(s_box + 1, e1);
      atomicMax(s_box + 2, e2);
      atomicMax(s_box + 3, e3);
    }
  }
  if (c != b.bin[n]) {
    b.bin[n] = c;
    atomicOr(moved, 1);
  }
}

// Blocks [0, move_blocks) move the bubbles; the blocks after them write the
// velocity ghost cells (vghost_cells), which the bubbles' stencils read in
// closed form (vx_final, vy_final), so one launch does both.
template <typename V>
__global__ void __launch_bounds__(kMoveThreads, kMoveMinBlocks) bubble_move(const __grid_constant__ GridParams g,
                                                            const __grid_constant__ BubbleParams bp, BubbleArrays b,
                                                            const V vx, const V vy, int* __restrict__ moved,
                                                            int move_blocks) {
  if ((int)blockIdx.x >= move_blocks) {
    vghost_cells(g, vx, vy, ((int)blockIdx.x - move_blocks) * kMoveThreads + (int)threadIdx.x);
    return;
  }
  __shared__ int s_box[4];
  if (threadIdx.x < 4) s_box[threadIdx.x] = 0;
  __syncthreads();
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n < b.n) move_one(g, bp, b, vx, vy, moved, n, s_box);
  __syncthreads();
  if (threadIdx.x < 4 && s_box[threadIdx.x] > 0) atomicMax(moved + 1 + threadIdx.x, s_box[threadIdx.x]);
}

// Bin counts for a rebuild of the cell bins.
__global__ void bin_count_kernel(const int* __restrict__ bin, int n, int* __restrict__ count) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int c = bin[k];
  if (c >= 0) atomicAdd(&count[c], 1);
}

// Cell indices of the initial positions (BubbleUpdateIndexKernel, :345-358) and bin counts.
__global__ void bubble_index(const __grid_constant__ GridParams g, BubbleArrays b, int* __restrict__ bin_count) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= b.n) return;
  double x = b.x[n], y = b.y[n];
  b.ibmx[n] = (int)floor(x * g.rdx + 1.0);
  b.ibmy[n] = (int)floor(y * g.rdy + 1.0);
  int inx = (int)floor(x * g.rdx + 0.5);
  int iny = (int)floor(y * g.rdy + 0.5);
  b.ibnx[n] = inx;
  b.ibny[n] = iny;
  b.bin[n] = bin_of(g.f, inx, iny);
}

// Exclusive scan of the bin counts: per-block scan, scan of block sums, add.
constexpr int kScanThreads = 1024;

__device__ __forceinline__ int block_exclusive_scan(int v, int* total) {
  __shared__ int s_w[32];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_w[w] = x;
  __syncthreads();
  if (w == 0) {
    int s = s_w[lane];
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    s_w[lane] = s;
  }
  __syncthreads();
  int before = (w > 0 ? s_w[w - 1] : 0) + x - v;
  if (total) *total = s_w[31];
  return before;
}

__global__ void __launch_bounds__(kScanThreads) bin_scan_blocks(const int* __restrict__ count, int* __restrict__ start,
                                                                int* __restrict__ partial, int nbins) {
  int k = blockIdx.x * kScanThreads + threadIdx.x;
  int v = k < nbins ? count[k] : 0;
  int total;
  int e = block_exclusive_scan(v, &total);
  if (k < nbins) start[k] = e;
  if (threadIdx.x == 0) partial[blockIdx.x] = total;
}

// partial[nparts] receives the grand total.
__global__ void __launch_bounds__(kScanThreads) bin_scan_partials(int* __restrict__ partial, int nparts) {
  int carry = 0;
  for (int base = 0; base < nparts; base += kScanThreads) {
    int k = base + threadIdx.x;
    int v = k < nparts ? partial[k] : 0;
    int total;
    int e = block_exclusive_scan(v, &total);
    __syncthreads();
    if (k < nparts) partial[k] = e + carry;
    carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[nparts] = carry;
}

__global__ void bin_scan_add(int* __restrict__ start, const int* __restrict__ partial, int nbins, int nparts) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nbins) start[k] += partial[k / kScanThreads];
  if (k == nbins) start[nbins] = partial[nparts];
}

__global__ void bin_fill(const int* __restrict__ bin, int n, const int* __restrict__ start, int* __restrict__ count,
                         int* __restrict__ idx) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  int c = bin[b];
  if (c < 0) return;
  int slot = start[c] + atomicSub(&count[c], 1) - 1;
  idx[slot] = b;
}

// Position of every binned bubble in the sorted order (pos was set to -1 first).
__global__ void bin_pos(const int* __restrict__ idx, const int* __restrict__ total, int* __restrict__ pos, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n && k < *total) pos[idx[k]] = k;
}

// Bubbles of a cell in ascending index order, so every sum over a cell has a
// fixed order run to run.
__global__ void bin_sort(const int* __restrict__ start, int* __restrict__ idx, int nbins) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nbins) return;
  int s = start[c], e = start[c + 1];
  for (int k = s + 1; k < e; k++) {
    int v = idx[k];
    int m = k - 1;
    while (m >= s && idx[m] > v) {
      idx[m + 1] = idx[m];
      m--;
    }
    idx[m + 1] = v;
  }
}

// RpState, thermal_model and rp_substep_full live in radius.cuh (shared with the 3-D path).

// BubbleInterpolationScalarKernel (:361-395) for bubble n, then the set-up of
// BubbleRadiusKernel from the state stored at the start of the step (:488-504).
template <typename S>
__device__ __forceinline__ double gather_pl(const GridParams& g, const BubbleParams& bp, const BubbleArrays& b,
                                           const S& px, const S& py, double t_cur, int n) {
  const Frame& f = g.f;
  const double x = b.x[n], y = b.y[n];
  const int inx = b.ibnx[n], iny = b.ibny[n];
  double PLp = 0.0;
  const double cx0 = delta_cos_x(bp, g, inx, x), cy0 = delta_cos_y(bp, g, iny, y);
  for (int qi = 0; qi < 2; qi++) {
    const int i = inx + qi;
    const double dxw = delta_w(bp, cx0, qi);
    for (int qj = 0; qj < 2; qj++) {
      const int j = iny + qj;
      const double dyw = delta_w(bp, cy0, qj);
      if (i >= 0 && i <= f.X + 1 && j >= 0 && j <= f.Y + 1) PLp += p0_at(g, px, py, i, j, t_cur) * dxw * dyw;
    }
  }
  return PLp;
}

// With `reuse` (a radius solve of this step has completed with the current
// bins), a bubble whose gathered pressure has the bit pattern of the last
// solve's needs no solve: every input of its solve is unchanged, so its stored
// results are what the solve would write; returns false for it.  The set-up
// runs either way (a branch around it costs the radius kernel registers).
template <typename S>
__device__ __forceinline__ bool rp_begin(const GridParams& g, const BubbleParams& bp, const BubbleArrays& b,
                                         const S& px, const S& py, double t_cur, int n, RpState& s, bool reuse) {
  const double PLp = gather_pl(g, bp, b, px, py, t_cur, n);
  const bool same = reuse && __double_as_longlong(PLp) == __double_as_longlong(b.PL_p[n]);
  b.PL_p[n] = PLp;
  s.r = bubble_r0(bp, b.R0[n]);
  const double dt = g.dt;
  s.Rt = b.R_t[n];
  s.Rp = b.R_pn[n];
  s.Rn = b.R_nn[n];
  s.d1Rp = b.d1_R_n[n];
  s.PGp = b.PG_n[n];
  s.dtL = b.dt_n[n];
  s.re_n = b.re_n[n];
  s.remain = s.re_n + dt;
  s.time = -s.re_n;
  const double PLn = b.PL_n[n], PLm = b.PL_m[n];
  s.PC0 = PLn + bp.PL0;
  s.PC1 = 0.5 * (PLp - PLm) / dt;
  s.PC2 = 0.5 * (PLp + PLm - 2.0 * PLn) / (dt * dt);
  s.heat = 0.0;
  s.vis = 0.0;
  s.count = 0;
  return !same;
}


__device__ __forceinline__ void store_contrib(const GridParams& g, const BubbleParams& bp, const BubbleArrays& b,
                                              int n, double Rt);

// Results of BubbleRadiusKernel (:542-550), then the bubble's void-fraction
// contribution to the four cells of its stencil (VoidFractionReverseLookupKernel,
// :595-617), stored for the per-cell gather.
__device__ __forceinline__ void rp_end(const GridParams& g, const BubbleParams& bp, const BubbleArrays& b, int n,
                                       const RpState& s) {
  const double dt = g.dt;
  b.R_t[n] = s.Rt;
  b.R_p[n] = s.Rp;
  b.R_n[n] = s.Rn;
  b.d1_R_p[n] = s.d1Rp;
  b.PG_p[n] = s.PGp;
  b.dt[n] = s.dtL;
  b.re[n] = s.remain;
  b.Q_B[n] = (s.heat + s.vis) / (dt - s.remain + s.re_n);
  b.nsub[n] = (int)min(s.count, (long long)INT32_MAX);
  store_contrib(g, bp, b, n, s.Rt);
}

// The bubble's void-fraction contribution to the four cells of its stencil
// (VoidFractionReverseLookupKernel, :595-617) at radius Rt, stored at its place
// in the sorted bins for the per-cell gather.
__device__ __forceinline__ void store_contrib(const GridParams& g, const BubbleParams& bp, const BubbleArrays& b,
                                              int n, double Rt) {
  const double x = b.x[n], y = b.y[n];
  const int inx = b.ibnx[n], iny = b.ibny[n];
  const double cx0 = delta_cos_x(bp, g, inx, x), cy0 = delta_cos_y(bp, g, iny, y);
  const double dx0 = delta_w(bp, cx0, 0), dx1 = delta_w(bp, cx0, 1);
  const double dy0 = delta_w(bp, cy0, 0), dy1 = delta_w(bp, cy0, 1);
  const double vol = g.cyl ? bp.pi4r3 * b.n_B[n] * (Rt * Rt * Rt) * g.rdx * g.rdy / x
                           : bp.pi4r3 * b.n_B[n] * (Rt * Rt * Rt) * g.rdx * g.rdy;
  const int p = b.pos[n];
  if (p < 0) return;
  double* c = b.contrib + 4 * (long)p;
  c[0] = vol * dx0 * dy0;
  c[1] = vol * dx0 * dy1;
  c[2] = vol * dx1 * dy0;
  c[3] = vol * dx1 * dy1;
}

// Persistent radius solve with a work queue.  Every lane takes the next bubble
// from `order` (bubbles sorted by their previous sub-step count, heaviest
// first) as soon as its current bubble finishes, and the loop advances every
// active lane by one sub-step per pass, so a bubble that needs thousands of
// sub-steps near collapse occupies one lane, not a warp, and no lane idles
// while the queue has work.  Each bubble's arithmetic is the same as a
// thread-per-bubble solve, so results do not depend on the schedule.
constexpr int kRpThreads = 128;
// Resident blocks per SM the register budget is set for: 7 for the FP64 path
// (at most 73 registers a thread), 5 for the mixed path (102): more warps to
// hide the FP64 latency chains of the sub-step, measured faster than fewer
// warps with more registers despite the spilled values (FP64, 1024 x 2048
// quiet phase, per 100 steps: radius solve 17.2 ms at 7 blocks, 17.9 at 6,
// 17.5 at 5; the mixed path's FP32 thermal model gains nothing from a sixth).
template <typename P>
constexpr int rp_min_blocks() {
  return sizeof(typename P::T) == sizeof(double) ? 7 : 5;
}

// Lanes whose claimed bubble kept its last solve (n == -2) are counted, one
// atomic per warp, and return to claiming (n = -1).  Called by the whole warp.
__device__ __forceinline__ void count_kept(int& n, unsigned long long* reused) {
  const unsigned kept = __ballot_sync(0xffffffffu, n == -2);
  if (kept) {
    if ((threadIdx.x & 31) == 0) atomicAdd(reused, (unsigned long long)__popc(kept));
    if (n == -2) n = -1;
  }
}

template <typename P>
__global__ void __launch_bounds__(kRpThreads, rp_min_blocks<P>()) bubble_rp(const __grid_constant__ GridParams g,
                                                        const __grid_constant__ BubbleParams bp, BubbleArrays b,
                                                        const typename P::S px, const typename P::S py,
                                                        const double* __restrict__ tdev,
                                                        const int* __restrict__ order,
                                                        int* __restrict__ next, long long* __restrict__ substep_max,
                                                        int* __restrict__ err, const int* __restrict__ solved,
                                                        unsigned long long* __restrict__ reused) {
  RpState s;
  const double t_cur = tdev[1];
  const bool reuse = bp.reuse && *solved > 0;
  int n = -1;
  bool drained = false;
  long long worst = 0;
  const int lane = threadIdx.x & 31;
  for (;;) {
    // Lanes without a bubble claim the next ones from the queue together:
    // one atomic per warp instead of one per lane.
    const unsigned need = __ballot_sync(0xffffffffu, n < 0 && !drained);
    if (need) {
      const int leader = __ffs(need) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(next, __popc(need));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need & (1u << lane)) {
        const int q = base + __popc(need & ((1u << lane) - 1u));
        if (q < b.n) {
          n = order[q];
          if (!rp_begin(g, bp, b, px, py, t_cur, n, s, reuse)) n = -2;  // kept: counted below
        } else {
          drained = true;
        }
      }
      count_kept(n, reused);
    }
    if (!__any_sync(0xffffffffu, n >= 0 || !drained)) break;
    if (n >= 0) {
      if (s.remain > 0.0 && s.count < bp.step_cap) {
        rp_substep_full<typename P::T>(bp, s);
      } else {
        if (s.remain > 0.0) atomicOr(err, 1);
        rp_end(g, bp, b, n, s);
        worst = max(worst, s.count);
        n = -1;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) worst = max(worst, __shfl_xor_sync(0xffffffffu, worst, o));
  if ((threadIdx.x & 31) == 0 && worst > 0) atomicMax(substep_max, worst);
}

}  // namespace crp
#include "rk45.cuh"
namespace crp {

// Set-up of one bubble's Dormand-Prince integration over the mixture step from
// the state stored at the start of the step (as rp_begin): the pressure
// gather, the liquid-pressure polynomial, R, R', PG and the last step size.
// `reuse` as in rp_begin.
template <typename S>
__device__ __forceinline__ bool rk_begin(const GridParams& g, const BubbleParams& bp, const BubbleArrays& b,
                                         const S& px, const S& py, double t_cur, int n, RkState& s, bool reuse) {
  const double PLp = gather_pl(g, bp, b, px, py, t_cur, n);
  const bool same = reuse && __double_as_longlong(PLp) == __double_as_longlong(b.PL_p[n]);
  b.PL_p[n] = PLp;
  s.r = bubble_r0(bp, b.R0[n]);
  const double dt = g.dt;
  s.R = b.R_pn[n];
  s.V = b.d1_R_n[n];
  s.PG = b.PG_n[n];
  s.h = b.dt_n[n];
  s.t = 0.0;
  s.tend = dt;
  s.Q = 0.0;
  s.count = 0;
  s.fresh = true;
  const double PLn = b.PL_n[n], PLm = b.PL_m[n];
  s.PC0 = PLn + bp.PL0;
  s.PC1 = 0.5 * (PLp - PLm) / dt;
  s.PC2 = 0.5 * (PLp + PLm - 2.0 * PLn) / (dt * dt);
  s.K = 3.0 * (bp.gam - 1.0) * bp.K0 * bp.T0 * s.r.inv_PG0;
  return !same;
}

// Results of the integration in the arrays the reference scheme fills: the
// radius at the end of the step (R_t = R_p; R_n likewise, the scheme keeps no
// older level), R', PG, the step size to start the next mixture step with,
// no remainder, the mean heat and viscous power, the step attempts; then the
// void-fraction contributions.
__device__ __forceinline__ void rk_end(const GridParams& g, const BubbleParams& bp, const BubbleArrays& b, int n,
                                       const RkState& s) {
  b.R_t[n] = s.R;
  b.R_p[n] = s.R;
  b.R_n[n] = s.R;
  b.d1_R_p[n] = s.V;
  b.PG_p[n] = s.PG;
  b.dt[n] = fmin(s.h, g.dt);
  b.re[n] = 0.0;
  b.Q_B[n] = s.Q / g.dt;
  b.nsub[n] = (int)min(s.count, (long long)INT32_MAX);
  store_contrib(g, bp, b, n, s.R);
}

// The radius solve with ext.rp_scheme = rk45: the work queue of bubble_rp,
// each pass one step attempt of every active lane.
template <typename P>
constexpr int rk_min_blocks() {
  return 3;
}

template <typename P>
__global__ void __launch_bounds__(kRpThreads, rk_min_blocks<P>()) bubble_rk45(const __grid_constant__ GridParams g,
                                                        const __grid_constant__ BubbleParams bp, BubbleArrays b,
                                                        const typename P::S px, const typename P::S py,
                                                        const double* __restrict__ tdev,
                                                        const int* __restrict__ order,
                                                        int* __restrict__ next, long long* __restrict__ substep_max,
                                                        int* __restrict__ err, const int* __restrict__ solved,
                                                        unsigned long long* __restrict__ reused) {
  RkState s;
  const double t_cur = tdev[1];
  const bool reuse = bp.reuse && *solved > 0;
  int n = -1;
  bool drained = false;
  long long worst = 0;
  const int lane = threadIdx.x & 31;
  for (;;) {
    const unsigned need = __ballot_sync(0xffffffffu, n < 0 && !drained);
    if (need) {
      const int leader = __ffs(need) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(next, __popc(need));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need & (1u << lane)) {
        const int q = base + __popc(need & ((1u << lane) - 1u));
        if (q < b.n) {
          n = order[q];
          if (!rk_begin(g, bp, b, px, py, t_cur, n, s, reuse)) n = -2;  // kept: counted below
        } else {
          drained = true;
        }
      }
      count_kept(n, reused);
    }
    if (!__any_sync(0xffffffffu, n >= 0 || !drained)) break;
    if (n >= 0) {
      if (s.t < s.tend && s.count < bp.step_cap) {
        if (!rk_attempt<typename P::T>(bp, s, bp.rk_rtol, g.c_inf)) s.count = bp.step_cap;
      } else {
        if (s.t < s.tend) atomicOr(err, 1);
        rk_end(g, bp, b, n, s);
        worst = max(worst, s.count);
        n = -1;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) worst = max(worst, __shfl_xor_sync(0xffffffffu, worst, o));
  if ((threadIdx.x & 31) == 0 && worst > 0) atomicMax(substep_max, worst);
}

}  // namespace crp
#include "lpt.cuh"
namespace crp {

// Void fraction of one cell from the bubbles of the four bins whose stencils
// cover it (bins (i-1..i) x (j-1..j), each in ascending bubble order): their
// contributions sit contiguously at 4 * (position in the sorted bins).
// One of the four bins whose bubbles contribute to cell (i, j): bin b = 0..3 is
// (i-1, j-1), (i, j-1), (i-1, j), (i, j); the sum of its bubbles' contributions
// to (i, j): the even and the odd positions of the bin's sorted run summed
// separately (two independent chains), then added.
__device__ __forceinline__ double gather_bin(const Frame& f, const int* __restrict__ start,
                                             const double* __restrict__ contrib, int i, int j, int b) {
  const int bx = i - 1 + (b & 1), by = j - 1 + (b >> 1);
  const int c = (by + 1) * (f.X + 3) + (bx + 1);
  const int slot = (i - bx) * 2 + (j - by);
  double s = 0.0, t = 0.0;
  int k = start[c];
  const int e = start[c + 1];
  for (; k + 1 < e; k += 2) {
    s += contrib[4 * (long)k + slot];
    t += contrib[4 * (long)k + 4 + slot];
  }
  if (k < e) s += contrib[4 * (long)k + slot];
  return s + t;
}
// Sum over the four bins of cell (i, j), as (b0 + b1) + (b2 + b3); with the
// axis fold (fold: cells 0 and 1 take the sum of both) each bin's part is that
// of cell 0 plus that of cell 1.  couple_press forms the same sums in the same
// order across four lanes, so both give bit-identical void fractions.
__device__ __forceinline__ double gather_fg(const Frame& f, const int* __restrict__ start,
                                            const double* __restrict__ contrib, int i, int j, bool fold = false) {
  double sb[4];
  for (int b = 0; b < 4; b++)
    sb[b] = fold ? gather_bin(f, start, contrib, 0, j, b) + gather_bin(f, start, contrib, 1, j, b)
                 : gather_bin(f, start, contrib, i, j, b);
  return (sb[0] + sb[1]) + (sb[2] + sb[3]);
}

template <typename P>
struct CoupleArgs {
  typename P::V vx, vy;
  typename P::S pnx, pny;
  typename P::S px, py;
  typename P::G fg;   // receives the gathered void fraction
  typename P::G fgn;
  const int* start;
  const int* idx;
  const double* contrib;
  unsigned long long* residual;
  int i0, j0, i1, j1;  // cells to update (inclusive)
  const int* dbox;     // if set: the box {i0, j0, i1, j1} in device memory instead
};

// calculate_void_fraction (memset, scatter, VoidFractionCylinderKernel fold:
// :1198-1218, :559-573) as a gather, then MixturePressureKernel (:816-867) on
// the new void fraction and the residual of calculate_pressure_field.  Four
// lanes per cell, one per contributing bin, so that the per-bin runs are
// summed side by side; the cell's void fraction is (b0 + b1) + (b2 + b3), the
// same in the four lanes and the same from run to run.  A block covers
// kCoupleW x 8 cells.
constexpr int kCoupleW = 8;

// One tile of kCoupleW x 8 cells (tile (tx, ty) of the box [i0, i1] x [j0, j1]):
// returns this thread's residual |dp0| (0 where it updates nothing; NaN sorts
// above every number in the bit-pattern maximum taken by the caller).
template <typename P>
__device__ __forceinline__ double couple_tile(const GridParams& g, const CoupleArgs<P>& a, int i0, int j0, int i1,
                                              int j1, int tx, int ty) {
  const Frame& f = g.f;
  const int X = f.X, Y = f.Y;
  const int bin = threadIdx.x & 3;
  const int i = i0 + tx * kCoupleW + (threadIdx.x >> 2);
  const int j = j0 + ty * blockDim.y + threadIdx.y;
  const bool in = i <= i1 && j <= j1;
  double fgv = 0.0;
  if (in) {
    if (g.cyl && i <= 1)  // the axis fold: cells 0 and 1 both take the sum of the two
      fgv = gather_bin(f, a.start, a.contrib, 0, j, bin) + gather_bin(f, a.start, a.contrib, 1, j, bin);
    else
      fgv = gather_bin(f, a.start, a.contrib, i, j, bin);
  }
  fgv += __shfl_xor_sync(0xffffffffu, fgv, 1);
  fgv += __shfl_xor_sync(0xffffffffu, fgv, 2);
  double res = 0.0;
  if (in && bin == 0) {
    long k = f.idx(i, j);
    a.fg.put(k, fgv);
    fgv = a.fg.get(k);  // the stored value (FP32 in the mixed path) is what the step uses
    if (i >= 1 && i <= X && j >= 1 && j <= Y) {
      double vxl = a.vx.get(f.idx(i - 1, j)), vxr = a.vx.get(k);
      double s1x = g.cyl ? (-g.xu[i] * vxl + g.xu[i + 1] * vxr) * g.rdx * g.rxp[i] : (-vxl + vxr) * g.rdx;
      double s1y = (-a.vy.get(f.idx(i, j - 1)) + a.vy.get(k)) * g.rdy;
      const double h = void_rate_half(g, fgv, a.fgn.get(k));
      double qx = pressure_component(g, a.pnx.get(k), g.pax[i], g.pbx[i], s1x, h);
      double qy = pressure_component(g, a.pny.get(k), g.pay[j], g.pby[j], s1y, h);
      bool forced = g.source_row > 0 && src_pressure(g) && j == g.source_row;
      if (!forced) res = fabs((a.px.get(k) + a.py.get(k)) - (qx + qy));
      a.px.put(k, qx);
      a.py.put(k, qy);
    }
  }
  return res;
}

// Host-driven steps launch one block per tile of the box.  Graph steps, whose
// box is decided on the device (dbox), launch a fixed grid whose blocks stride
// over the box's tiles.
template <typename P>
__global__ void __launch_bounds__(256) couple_press(const __grid_constant__ GridParams g, const CoupleArgs<P> a) {
  unsigned long long rb = 0ull;  // max |dp0| as a bit pattern
  if (a.dbox) {
    const int i0 = a.dbox[0], j0 = a.dbox[1], i1 = a.dbox[2], j1 = a.dbox[3];
    if (i0 <= i1 && j0 <= j1) {
      const int tw = (i1 - i0 + kCoupleW) / kCoupleW, th = (j1 - j0 + (int)blockDim.y) / (int)blockDim.y;
      for (int t = blockIdx.x; t < tw * th; t += gridDim.x)  // the same trip count in every thread of a block
        rb = max(rb, (unsigned long long)__double_as_longlong(couple_tile(g, a, i0, j0, i1, j1, t % tw, t / tw)));
    }
  } else {
    rb = (unsigned long long)__double_as_longlong(couple_tile(g, a, a.i0, a.j0, a.i1, a.j1, blockIdx.x, blockIdx.y));
  }
  block_max_to(__longlong_as_double((long long)rb), a.residual);
}

// p0 with its boundary values into a dense (X+2) x (Y+2) array, for readback.
template <typename S>
__global__ void materialize_p0(const __grid_constant__ GridParams g, const S px, const S py, double t,
                               double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i > g.f.X + 1 || j > g.f.Y + 1) return;
  out[(long)j * (g.f.X + 2) + i] = p0_at(g, px, py, i, j, t);
}

// ---------------------------------------------------------------------------
// Host side.

#define CRP_CUDA(call)                                                      \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess) return fail(CRP_ERR_CUDA, #call, e_);            \
  } while (0)

// Kernel classes for launch counting and optional per-class device timing.
enum KernelClass { kClassFdtd = 0, kClassRp = 1, kClassCouple = 2, kClassOther = 3 };

// ---------------------------------------------------------------------------
// Temperature branch (calculate_temperature, inc/bubble_CUDA_kernel.cuh:1347-1376):
// bubble heat scattered to cells, mixture conductivity, energy fluxes, the
// temperature update with acoustic absorption, and the non-PML mirrors.  Run
// after the Picard loop when the temperature is requested (debug.T); nothing
// on the pressure/bubble path reads it.

// Water properties (:176-193); the float literals are the reference's.
__host__ __device__ __forceinline__ double conductivity_water(double T) {
  return 0.76760 + ((double)7.5390e-3f * T) - (double)9.8250e-6f * (T * T);
}
__host__ __device__ __forceinline__ double heat_capacity_water(double T) {
  const double H2O = (double)18.0e-3f;
  return (917.5 - (double)10.1016f * T + (double)0.0454134f * (T * T) - 9.07517e-5 * (T * T * T) +
          (double)6.80700e-8f * (T * T * T * T)) /
         H2O;
}

// Heat of each bubble to the four cells of its stencil (BubbleHeatKernel,
// :972-1007): n_B Q_B / (dx dy [x]) delta_x delta_y, laid out like the
// void-fraction contributions so the same bin gather sums them.
__global__ void heat_contrib(const __grid_constant__ GridParams g, const __grid_constant__ BubbleParams bp,
                             BubbleArrays b, double* __restrict__ hc) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= b.n) return;
  const double x = b.x[n], y = b.y[n];
  const int inx = b.ibnx[n], iny = b.ibny[n];
  const double q = g.cyl ? b.n_B[n] * b.Q_B[n] * g.rdx * g.rdy / x : b.n_B[n] * b.Q_B[n] * g.rdx * g.rdy;
  const double cx0 = delta_cos_x(bp, g, inx, x), cy0 = delta_cos_y(bp, g, iny, y);
  const double dx0 = delta_w(bp, cx0, 0), dx1 = delta_w(bp, cx0, 1);
  const double dy0 = delta_w(bp, cy0, 0), dy1 = delta_w(bp, cy0, 1);
  const int p = b.pos[n];
  if (p < 0) return;
  double* c = hc + 4 * (long)p;
  c[0] = q * dx0 * dy0;
  c[1] = q * dx0 * dy1;
  c[2] = q * dx1 * dy0;
  c[3] = q * dx1 * dy1;
}

struct TempArgs {
  F64 T_old, T_new;
  double* dT;           // if set: the step's temperature increment (the focal tracker's input)
  const int* start;
  const int* idx;
  const double* hc;     // heat contributions (heat_contrib)
  double coef_abs;      // 2 (0.22) 0.115129255 / (rho c omega^2) of MixtureTemperatureKernel
  double T_inf;
  int rho_const;
  int bubbles;
};

// MixtureKMKernel, MixtureEnergyKernel and MixtureTemperatureKernel
// (:955-1062) fused: each interior cell forms its conductivities, the four
// face fluxes and its new temperature from the old field.
template <typename P>
__global__ void __launch_bounds__(256) temperature_step(const __grid_constant__ GridParams g, const TempArgs t,
                                                         const typename P::G fg, const typename P::G fgn,
                                                         const typename P::S px, const typename P::S py,
                                                         const typename P::S pnx, const typename P::S pny) {
  const Frame& f = g.f;
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i > f.X || j > f.Y) return;
  auto km = [&](int a, int b) -> double {
    const long k = f.idx(a, b);
    const double fv = fg.get(k);
    return conductivity_water(t.T_old.get(k) + t.T_inf) * (1.0 - 3.0 * fv / (2.0 + fv));
  };
  const long k = f.idx(i, j);
  const double Tc = t.T_old.get(k);
  const double kc = km(i, j), kl = km(i - 1, j), kr = km(i + 1, j), kd = km(i, j - 1), ku = km(i, j + 1);
  const double exr = 2.0 * kc * kr / (kc + kr) * ((-Tc + t.T_old.get(f.idx(i + 1, j))) * g.rdx);
  const double exl = 2.0 * kl * kc / (kl + kc) * ((-t.T_old.get(f.idx(i - 1, j)) + Tc) * g.rdx);
  const double eyu = 2.0 * kc * ku / (kc + ku) * ((-Tc + t.T_old.get(f.idx(i, j + 1))) * g.rdy);
  const double eyd = 2.0 * kd * kc / (kd + kc) * ((-t.T_old.get(f.idx(i, j - 1)) + Tc) * g.rdy);
  double s0 = (px.get(k) + py.get(k) - pnx.get(k) - pny.get(k)) / g.dt;
  s0 = t.coef_abs * s0 * s0;
  const double work = t.bubbles ? gather_fg(f, t.start, t.hc, i, j) : 0.0;
  const double Q = work + s0;
  const double s1 = (exr - exl) * g.rdx;
  const double s2 = (eyu - eyd) * g.rdy;
  const double rho_m = t.rho_const ? g.rho_inf : (1.0 - fgn.get(k)) * g.rho_inf;
  const double cpm = heat_capacity_water(Tc + t.T_inf);
  const double dT = g.dt * (s1 + s2 + Q) / (rho_m * cpm);
  t.T_new.put(k, Tc + dT);
  if (t.dT) t.dT[k] = dT;
}

// MixtureBoundaryTemperatureKernel (:1065-1102) as one block: the old ghost
// ring is carried over, then the sections run in the reference's order, each
// over all its indices before the next (X0, X1, Y0, Y1; the Y1 loop starts at
// row Y, so row Y takes the ghost row's value and the ghost row keeps it).
__global__ void __launch_bounds__(1024) temperature_bc(const __grid_constant__ GridParams g, const F64 T_old,
                                                        const F64 T_new) {
  const Frame& f = g.f;
  const int X = f.X, Y = f.Y;
  for (int q = threadIdx.x; q <= X + 1; q += blockDim.x) {
    T_new.put(f.idx(q, 0), T_old.get(f.idx(q, 0)));
    T_new.put(f.idx(q, Y + 1), T_old.get(f.idx(q, Y + 1)));
  }
  for (int q = threadIdx.x; q <= Y + 1; q += blockDim.x) {
    T_new.put(f.idx(0, q), T_old.get(f.idx(0, q)));
    T_new.put(f.idx(X + 1, q), T_old.get(f.idx(X + 1, q)));
  }
  __syncthreads();
  if (!g.pml_x0)
    for (int q = 1 + threadIdx.x; q <= Y; q += blockDim.x) T_new.put(f.idx(0, q), T_new.get(f.idx(1, q)));
  __syncthreads();
  if (!g.pml_x1)
    for (int q = threadIdx.x; q <= Y + 1; q += blockDim.x) T_new.put(f.idx(X + 1, q), T_new.get(f.idx(X, q)));
  __syncthreads();
  if (!g.pml_y0)
    for (int q = threadIdx.x; q <= X + 1; q += blockDim.x) T_new.put(f.idx(q, 0), T_new.get(f.idx(q, 1)));
  __syncthreads();
  if (!g.pml_y1)
    for (int q = threadIdx.x; q <= X + 1; q += blockDim.x) {
      T_new.put(f.idx(q, Y), T_new.get(f.idx(q, Y + 1)));
      T_new.put(f.idx(q, Y + 1), T_new.get(f.idx(q, Y)));
    }
}

struct Profiler {
  bool on = false;
  std::vector<cudaEvent_t> ev;  // pairs
  std::vector<int> cls;
  size_t used = 0;
  double ms[4] = {0, 0, 0, 0};
  cudaError_t begin(cudaStream_t s, int c) {
    if (!on) return cudaSuccess;
    if (2 * used + 2 > ev.size()) {
      for (int k = 0; k < 2; k++) {
        cudaEvent_t e;
        cudaError_t r = cudaEventCreate(&e);
        if (r != cudaSuccess) return r;
        ev.push_back(e);
      }
      cls.push_back(0);
    }
    cls[used] = c;
    return cudaEventRecord(ev[2 * used], s);
  }
  cudaError_t end(cudaStream_t s) {
    if (!on) return cudaSuccess;
    cudaError_t r = cudaEventRecord(ev[2 * used + 1], s);
    used++;
    return r;
  }
  // After the stream has been synchronised.
  void resolve() {
    for (size_t k = 0; k < used; k++) {
      float t = 0.f;
      if (cudaEventElapsedTime(&t, ev[2 * k], ev[2 * k + 1]) == cudaSuccess) ms[cls[k]] += t;
    }
    used = 0;
  }
  ~Profiler() {
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
  }
};

// ---------------------------------------------------------------------------
// Focal tracker (determine_focal_point, inc/bubble_CUDA_kernel.cuh:1132-1166).
// The reference reduces the Work array (the step's temperature increment) with
// functors of a header that its source tree does not contain, so their exact
// weighting is unknown; here the focal depth is the centroid, over the
// interior cells, of the increment's excess over half of its maximum:
//   y_f = sum(w (j - 1/2) dy) / sum(w),  w = max(dT - max(dT) / 2, 0),
// a weight that goes to zero continuously at the half maximum, so rounding
// differences move y_f by rounding amounts (a hard cut would flip cells in
// and out of the region),
// and y_f = 0 while max(dT) <= kFocalFloor: increments of rounding size (the
// prediction's multiply-adds leave ~1e-40 K where nothing heats) define no focus.
// Three launches, each in a fixed order, so the result is the same run to run.
constexpr int kFocalBlocks = 148, kFocalThreads = 256;
constexpr double kFocalFloor = 1.0e-30;  // K per step

__device__ __forceinline__ double block_sum_fixed(double v, double* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kFocalThreads) focal_max(const double* __restrict__ dT, const Frame f,
                                                            double* __restrict__ part) {
  __shared__ double sh[kFocalThreads];
  double m = -1.0e300;
  for (int j = 1 + blockIdx.x; j <= f.Y; j += gridDim.x)
    for (int i = 1 + threadIdx.x; i <= f.X; i += blockDim.x) m = fmax(m, dT[f.idx(i, j)]);
  sh[threadIdx.x] = m;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void __launch_bounds__(kFocalThreads) focal_sums(const double* __restrict__ dT, const Frame f, double dy,
                                                             const double* __restrict__ pmax, int nparts,
                                                             double* __restrict__ part2) {
  __shared__ double sh[kFocalThreads];
  double mx = -1.0e300;
  for (int k = 0; k < nparts; k++) mx = fmax(mx, pmax[k]);
  const double thr = 0.5 * mx;
  double sw = 0.0, swy = 0.0;
  if (mx > kFocalFloor)
    for (int j = 1 + blockIdx.x; j <= f.Y; j += gridDim.x) {
      const double y = ((double)j - 0.5) * dy;
      for (int i = 1 + threadIdx.x; i <= f.X; i += blockDim.x) {
        const double v = dT[f.idx(i, j)] - thr;
        if (v > 0.0) {
          sw += v;
          swy += v * y;
        }
      }
    }
  sw = block_sum_fixed(sw, sh);
  swy = block_sum_fixed(swy, sh);
  if (threadIdx.x == 0) {
    part2[2 * blockIdx.x] = sw;
    part2[2 * blockIdx.x + 1] = swy;
  }
}

__global__ void focal_final(const double* __restrict__ part2, int nparts, double* __restrict__ out) {
  double sw = 0.0, swy = 0.0;
  for (int k = 0; k < nparts; k++) {
    sw += part2[2 * k];
    swy += part2[2 * k + 1];
  }
  out[0] = sw;
  out[1] = swy;
}

// ---------------------------------------------------------------------------
// Device-resident step state.  The host path reads it after each residual
// evaluation; the graph path (below) keeps the whole step's control on the
// device and reads it back once per crp_step call.
struct Scalars {
  unsigned long long residual;  // max |dp0| as the bit pattern of a non-negative double
  long long substep_max;        // largest RP sub-step count of one bubble
  int err;                      // nonzero: a bubble hit the sub-step cap
  int next;                     // work-queue head of the radius solve
  int moved;                    // nonzero: a bubble changed cell bin this step
  int bbox[4];                  // bins occupied this step, encoded (bubble_move)
  double t[3];                  // t_prev, t (the step's time) and the Fast2Sum carry
  // Graph path only: the Picard loop and the step's bookkeeping.
  double res, prev, res_last;   // residual now, at the previous iteration, at the step's end
  long long steps, picard_total, stalls;
  int picard_last, picard_max;
  int status;                   // crp_status of the first failure (0: none)
  int loop;                     // Picard iterations of this step completed (both paths; the radius
                                // solves keep unchanged bubbles' results from the second on)
  unsigned long long reused;    // radius solves kept (ext.rp_reuse), summed over the handle's life
  int stale;                    // bins need a rebuild
  int bnow[4], box[4];          // bubbles' cell box, coupling box
  int supp[3][4];               // void-fraction supports of the last three steps
  int entered, rebuilt;         // this step ran the Picard loop / rebuilt the bins
  long long launches[4];        // kernels run by completed graph steps, per class
  int pipe_err;                 // nonzero: an mbarrier wait of the FDTD pass ran out (never cleared)
};

// Fast2Sum time step (src/bubble_CUDA.cu:208-212), written by the host path.
// Start of a host-driven step: the step's times, and the residual and the
// bubble-motion flags cleared (one launch instead of a kernel and two memsets).
__global__ void set_time(Scalars* s, double t_prev, double t, double carry) {
  s->t[0] = t_prev;
  s->t[1] = t;
  s->t[2] = carry;
  s->residual = 0ull;
  s->moved = 0;
  for (int k = 0; k < 4; k++) s->bbox[k] = 0;
  s->loop = 0;
}
// Start of a Picard iteration of a host-driven step: residual and work-queue
// head cleared; `done` iterations of this step have completed.
__global__ void picard_begin(Scalars* s, int done) {
  s->residual = 0ull;
  s->next = 0;
  s->loop = done;
}
// The first Picard iteration's start, launched with the radius solve before the
// host has read the prediction's residual: the iteration runs when the host
// will run it (residual above the tolerance, computed as the host computes it,
// and no bubble changed bin, so the bins stand).  Otherwise the work queue is
// left closed (head at n) and the radius solve returns without touching a
// bubble; the host then rebuilds the bins and starts the loop itself, or skips it.
__global__ void picard_gate(Scalars* s, double P_inf, double tol, int n) {
  const double r = __longlong_as_double((long long)s->residual) / P_inf;
  s->loop = 0;
  if (r > tol && s->moved == 0) {
    s->residual = 0ull;
    s->next = 0;
  } else {
    s->next = n;
  }
}

struct CtlParams {
  double tol, P_inf, dt, stall;
  int cap, nb, mixed, X, Y, cyl;
  cudaGraphConditionalHandle h_step, h_picard, h_bins, h_loop;
};

__device__ __forceinline__ bool dbox_empty(const int* b) { return b[0] > b[2] || b[1] > b[3]; }
__device__ __forceinline__ void dbox_union(int* o, const int* a, const int* b) {
  if (dbox_empty(a)) {
    for (int q = 0; q < 4; q++) o[q] = b[q];
  } else if (dbox_empty(b)) {
    for (int q = 0; q < 4; q++) o[q] = a[q];
  } else {
    o[0] = min(a[0], b[0]);
    o[1] = min(a[1], b[1]);
    o[2] = max(a[2], b[2]);
    o[3] = max(a[3], b[3]);
  }
}
__device__ __forceinline__ double residual_of(const Scalars* s, double P_inf) {
  return __longlong_as_double((long long)s->residual) / P_inf;
}

// Start of a step: skip it after a failure; advance the time; clear the
// per-step accumulators.
__global__ void ctl_step_begin(Scalars* s, const CtlParams c) {
  if (s->status) {
    cudaGraphSetConditional(c.h_step, 0);
    return;
  }
  const double tstep = s->t[1], tstepx = s->t[2];
  const double s1 = tstep;
  const double t = tstep + c.dt + tstepx;
  const double s2 = t - s1;
  s->t[0] = tstep;
  s->t[1] = t;
  s->t[2] = c.dt + tstepx - s2;
  s->residual = 0ull;
  s->moved = 0;
  for (int q = 0; q < 4; q++) s->bbox[q] = 0;
  s->loop = 0;
  cudaGraphSetConditional(c.h_step, 1);
}

// After the FDTD pass and the bubble motion: the coupling box, the bin state,
// and whether the Picard loop runs.
__global__ void ctl_enter(Scalars* s, const CtlParams c, int box_off) {
  const double r = residual_of(s, c.P_inf);
  s->res = r;
  s->prev = r;
  s->stale |= s->moved;
  int* bn = s->bnow;
  const int* e = s->bbox;
  if (c.nb > 0 && e[1] != 0) {
    bn[0] = max(0, box_off - e[0]);
    bn[1] = max(0, box_off - e[2]);
    bn[2] = min(c.X + 1, e[1] - box_off + 1);
    bn[3] = min(c.Y + 1, e[3] - box_off + 1);
    if (!dbox_empty(bn) && c.cyl && bn[0] <= 1) {
      bn[0] = 0;
      bn[2] = max(bn[2], 1);
    }
  } else {
    bn[0] = bn[1] = 1;
    bn[2] = bn[3] = 0;
  }
  int u[4], w[4];
  dbox_union(u, bn, s->supp[0]);
  dbox_union(w, s->supp[1], s->supp[2]);
  dbox_union(s->box, u, w);
  bool enter = c.nb > 0 && r > c.tol;
  if (enter && c.cap <= 0) {
    s->status = CRP_ERR_PICARD;
    enter = false;
  }
  s->entered = enter;
  s->rebuilt = 0;
  s->residual = 0ull;
  s->next = 0;
  cudaGraphSetConditional(c.h_picard, enter ? 1u : 0u);
}

__global__ void ctl_bins(Scalars* s, const CtlParams c) {
  cudaGraphSetConditional(c.h_bins, s->stale ? 1u : 0u);
  s->rebuilt = s->stale;
  s->stale = 0;
}

// End of a Picard iteration: the loop continues while the residual is above
// the threshold, up to the cap; the mixed path's stagnation rule as in the
// host path.
__global__ void ctl_iter(Scalars* s, const CtlParams c) {
  const int loop = ++s->loop;
  unsigned go = 0;
  if (s->err) {
    s->status = CRP_ERR_RP_STEPS;
  } else {
    const double r = residual_of(s, c.P_inf);
    s->res = r;
    if (c.mixed && loop >= 3 && r > c.tol && r > 0.5 * s->prev && r < c.stall) {
      s->stalls++;
    } else if (r > c.tol) {
      if (loop >= c.cap)
        s->status = CRP_ERR_PICARD;
      else
        go = 1;
    }
    s->prev = r;
  }
  s->residual = 0ull;
  s->next = 0;
  cudaGraphSetConditional(c.h_loop, go);
}

// End of a step: non-finite check, void-fraction support history, counters.
__global__ void ctl_end(Scalars* s, const CtlParams c) {
  if (s->status) return;
  if (isnan(s->res)) {
    s->status = CRP_ERR_NONFINITE;
    return;
  }
  int snow[4];
  if (s->loop > 0) {
    for (int q = 0; q < 4; q++) snow[q] = s->bnow[q];
  } else {
    int u[4];
    dbox_union(u, s->supp[0], s->supp[1]);
    dbox_union(snow, u, s->supp[2]);
  }
  for (int q = 0; q < 4; q++) {
    s->supp[2][q] = s->supp[1][q];
    s->supp[1][q] = s->supp[0][q];
    s->supp[0][q] = snow[q];
  }
  // Kernels of the step, per class (fdtd, rp, couple, other), as the host path counts them.
  s->launches[0] += 1;
  s->launches[1] += s->loop;
  s->launches[2] += s->loop;
  s->launches[3] += 4 + (c.nb > 0) + (s->entered ? 4 + s->loop + (s->rebuilt ? 6 : 0) : 0);
  s->steps++;
  s->picard_last = s->loop;
  s->picard_total += s->loop;
  s->picard_max = max(s->picard_max, s->loop);
  s->res_last = s->res;
}

struct Sim {
  crp_config cfg{};
  Profiler prof;
  int64_t launches[4] = {0, 0, 0, 0};
  HostSetup hs;
  GridParams gp{};
  BubbleParams bp{};
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int device = 0;  // the device current at crp_create
  std::string err;

  // Device memory: one allocation carved into aligned pieces.
  char* pool = nullptr;
  size_t pool_bytes = 0;
  // Field buffers, 8 bytes per frame cell: one double (FP64 path) or an FP32
  // value array followed by its FP32 compensation array (mixed path; f_g uses
  // the first half only).
  void* vx[2]{};
  void* vy[2]{};
  void* px[2]{};
  void* py[2]{};
  void* fg[3]{};
  size_t cells = 0;  // frame cells per field
  bool mixed = false;
  double* scratch = nullptr;  // dense (X+2) x (Y+2) doubles for readback
  double* d_sigma = nullptr;
  double* d_elem = nullptr;  // source elements: amplitude factors, then phase offsets
  // Tensor maps of every field buffer for fdtd_tma: velocity [vx, vy][buffer],
  // split pressure [px, py][buffer], void-fraction ring.
  CUtensorMap tm_v[2][2]{}, tm_p[2][2]{}, tm_fg[3]{};
  bool fdtd_tma_on = std::getenv("CRP_FDTD_TILE") != nullptr;  int tile_ntx = 1, tile_n = 1, tile_grid = 1;
  BubbleArrays bub{};
  Bins bins{};
  // Device scalars written by the kernels, read back once per pressure evaluation.
  Scalars* d_scalars = nullptr;
  unsigned long long* d_residual = nullptr;
  long long* d_substep_max = nullptr;
  int* d_err = nullptr;
  int* d_next = nullptr;
  int* d_moved = nullptr;
  Scalars* h_scalars = nullptr;  // pinned
  cudaEvent_t ev_scalars = nullptr;  // the prediction's scalars have reached h_scalars
  cudaEvent_t ev_block = nullptr;    // the same, for blocking waits (set_blocking_waits)
  bool blocking_waits = false;
  double picard_tol = 1.0e-7f;
  // Cell boxes {i0, j0, i1, j1} (empty when i0 > i1).  supp[q] bounds the
  // nonzero void fraction of step n-1-q; the coupling kernel updates only the
  // union of the bubbles' box and supp[0..2]: outside it both the gathered and
  // the predicted void fraction are zero, so the pressure from the FDTD pass
  // already has its final value there.
  struct Box {
    int i0, j0, i1, j1;
  };
  Box supp[3];
  Box couple_box;
  bool bins_stale = false;  // a bubble changed cell since the bins were built
  // Graph path: one executable graph per buffer phase (velocity/pressure
  // ping-pong x f_g ring = 6), built on first use by stream capture.
  cudaStream_t cap_stream = nullptr;
  cudaGraph_t step_graph[6] = {};
  cudaGraphExec_t step_exec[6] = {};
  bool capturing = false;    // launches go into a graph (device-decided coupling box)
  // Temperature branch (debug.T): two temperature buffers and the bubbles'
  // heat contributions.
  bool temperature_on = false;
  void* Tbuf[2] = {nullptr, nullptr};
  int cur_t = 0;
  double* heat = nullptr;
  // Focal tracker and PID focus control (src/bubble_CUDA.cu:123-153, 310-352),
  // run with the temperature branch: the step's temperature increment, the
  // reduction partials, the tracked and controlled focal depths, the
  // Butterworth filter's state and the PID accumulators.
  double* dTbuf = nullptr;
  double* focal_part = nullptr;
  double* h_focal = nullptr;  // pinned {sum w, sum w y}
  std::vector<double> focal_hist, control_hist;
  crp_focus_state focus{};
  bool graphs_on = true;     // ext: off runs every step from the host
  Scalars* h_push = nullptr;  // pinned staging of the host state for the graph path
  bool debug_picard = std::getenv("CRP_DEBUG_PICARD") != nullptr;  // residual of every Picard iteration to stderr
  struct Lpt {
    int* hist;    // kLptBuckets
    int* cursor;  // kLptBuckets
    int* order;   // n
  } lpt{};
  int rp_grid = 1;
  int rp_grid_full = 1;       // the radius kernel's grid at one lane per bubble, up to the occupancy limit
  int couple_graph_grid = 1;  // blocks of the graph steps' coupling launch (striding over the box's tiles)
  // Launch tuning (crp_set_tuning): rows per FDTD strip chunk and the radius
  // kernel's block count (0: rp_grid_full).
  int strip_rows = kStripRows;
  int rp_blocks_req = 0;
  // Graph steps queued by graphs_enqueue and not yet completed by graphs_finish.
  struct Pending {
    bool on = false;
    int64_t steps0 = 0;
    int cur_v = 0, cur_p = 0, fg_a = 0, fg_b = 1, fg_c = 2;
  } pend;

  MinMax mm;       // running min/max of written rawdata values
  int cur_v = 0;   // velocity buffer holding the latest velocities
  int cur_p = 0;   // pressure buffer holding the latest pressure
  int fg_a = 0, fg_b = 1, fg_c = 2;  // ring: f_g, f_gn, f_gm
  double tstep = 0.0, tstepx = 0.0, t_prev = 0.0;
  crp_stats stats{};

  crp_status fail(crp_status s, const char* what, cudaError_t e = cudaSuccess) {
    err = std::string(what);
    if (e != cudaSuccess) err += std::string(": ") + cudaGetErrorString(e);
    return s;
  }

  template <typename T>
  T* carve(size_t count, size_t& off, bool dry) {
    size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
    T* p = dry ? nullptr : reinterpret_cast<T*>(pool + off);
    off += bytes;
    return p;
  }

  size_t layout(bool dry) {
    const Frame& f = gp.f;
    cells = (size_t)f.pitch * (f.Y + 4);
    size_t off = 0;
    for (int k = 0; k < 2; k++) {
      vx[k] = carve<double>(cells, off, dry);
      vy[k] = carve<double>(cells, off, dry);
      px[k] = carve<double>(cells, off, dry);
      py[k] = carve<double>(cells, off, dry);
    }
    for (int k = 0; k < 3; k++) fg[k] = carve<double>(cells, off, dry);
    if (temperature_on) {
      for (int k = 0; k < 2; k++) Tbuf[k] = carve<double>(cells, off, dry);
      dTbuf = carve<double>(cells, off, dry);
      focal_part = carve<double>(3 * kFocalBlocks + 2, off, dry);
    }
    scratch = carve<double>((size_t)(f.X + 2) * (f.Y + 2), off, dry);
    d_sigma = carve<double>(hs.sigma_block.size(), off, dry);
    d_elem = carve<double>(2 * (size_t)std::max(cfg.ext_elements, 1), off, dry);
    d_scalars = carve<Scalars>(1, off, dry);
    if (!dry) {
      d_residual = &d_scalars->residual;
      d_substep_max = &d_scalars->substep_max;
      d_err = &d_scalars->err;
      d_next = &d_scalars->next;
      d_moved = &d_scalars->moved;
    }
    const int n = hs.nb;
    bub.n = n;
    double** dp[] = {&bub.x, &bub.y, &bub.R_t, &bub.R_p, &bub.R_pn, &bub.R_n, &bub.R_nn, &bub.d1_R_p, &bub.d1_R_n,
                     &bub.PG_p, &bub.PG_n, &bub.PL_p, &bub.PL_n, &bub.PL_m, &bub.Q_B, &bub.n_B, &bub.dt, &bub.dt_n,
                     &bub.re, &bub.re_n, &bub.vbx, &bub.vby, &bub.R0};
    for (double** p : dp) *p = carve<double>(std::max(n, 1), off, dry);
    bub.contrib = carve<double>(4 * (size_t)std::max(n, 1), off, dry);
    heat = temperature_on ? carve<double>(4 * (size_t)std::max(n, 1), off, dry) : nullptr;
    int** ip[] = {&bub.ibmx, &bub.ibmy, &bub.ibnx, &bub.ibny, &bub.bin, &bub.nsub, &bub.pos};
    for (int** p : ip) *p = carve<int>(std::max(n, 1), off, dry);
    bins.nbx = f.X + 3;
    bins.nby = f.Y + 3;
    bins.nbins = bins.nbx * bins.nby;
    bins.count = carve<int>(bins.nbins, off, dry);
    bins.start = carve<int>(bins.nbins + 1, off, dry);
    bins.idx = carve<int>(std::max(n, 1), off, dry);
    bins.partial = carve<int>((bins.nbins + kScanThreads - 1) / kScanThreads + 1, off, dry);
    lpt.hist = carve<int>(kLptBuckets, off, dry);
    lpt.cursor = carve<int>(kLptBuckets, off, dry);
    lpt.order = carve<int>(std::max(n, 1), off, dry);
    return off;
  }

  // Typed views of the raw field buffers.
  template <typename A>
  A view(void* b) const;

  // Launch one kernel (the callable enqueues it on `stream`), counted by class
  // and bracketed by profiling events when profiling is on.
  template <typename F>
  cudaError_t launch(int cls, F&& enqueue) {
    cudaError_t e = prof.begin(stream, cls);
    if (e != cudaSuccess) return e;
    enqueue();
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    launches[cls]++;
    return prof.end(stream);
  }

  crp_status create(const crp_config& c, const crp_bubbles_in* bin, void* user_stream) {
    cfg = c;
    crp_status st = host_setup(cfg, bin, &hs, &err);
    if (st != CRP_OK) return st;
    if (cfg.sim_order != 2 || cfg.sim_smooth_delta_band != 2)
      return fail(CRP_ERR_UNSUPPORTED, "the CUDA path implements simulation.order = 2 and smooth_delta_band = 2");
    if (cfg.ext_precision != CRP_PREC_FP64 && cfg.ext_precision != CRP_PREC_MIXED)
      return fail(CRP_ERR_INVALID, "ext.precision must be fp64 or mixed");
    if (cfg.ext_rp_scheme != CRP_RP_REF && cfg.ext_rp_scheme != CRP_RP_RK45)
      return fail(CRP_ERR_INVALID, "ext.rp_scheme must be ref or rk45");
    if (cfg.ext_rp_tol < 0.0 || !(cfg.ext_rp_tol < 1.0)) return fail(CRP_ERR_INVALID, "ext.rp_tol must be in [0, 1)");
    mixed = cfg.ext_precision == CRP_PREC_MIXED;
    picard_tol = cfg.ext_picard_tol > 0.0 ? cfg.ext_picard_tol : (mixed ? 1.0e-5 : (double)1.0e-7f);
    graphs_on = cfg.ext_graphs != 0;
    // The focal tracker reads the temperature increment, so the PID controller
    // turns the temperature branch on (its output stays governed by debug.T).
    temperature_on = cfg.dbg_T != 0 || cfg.tr_pid != 0;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(CRP_ERR_NO_DEVICE, "no CUDA device");
    CRP_CUDA(cudaGetDevice(&device));
    if (user_stream) {
      stream = (cudaStream_t)user_stream;
    } else {
      CRP_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
      own_stream = true;
    }
    fill_params();
    // The grid kernels address the frame with 32-bit element offsets.
    if ((unsigned long long)gp.f.pitch * (unsigned long long)(gp.f.Y + 4) >= (1ull << 32))
      return fail(CRP_ERR_UNSUPPORTED, "grid frame of 2^32 elements or more");
    supp[0] = supp[1] = supp[2] = full_box();
    couple_box = full_box();
    pool_bytes = layout(true);
    CRP_CUDA(cudaMalloc(&pool, pool_bytes));
    layout(false);
    if (fdtd_tma_on) {
      const crp_status ts = make_tensor_maps();
      if (ts != CRP_OK) return ts;
    }
    CRP_CUDA(cudaMemsetAsync(pool, 0, pool_bytes, stream));
    CRP_CUDA(cudaMallocHost(&h_scalars, sizeof(Scalars)));
    std::memset(h_scalars, 0, sizeof(Scalars));
    CRP_CUDA(cudaEventCreateWithFlags(&ev_scalars, cudaEventDisableTiming));
    CRP_CUDA(cudaMallocHost(&h_focal, 2 * sizeof(double)));
    // Control system start (src/bubble_CUDA.cu:123-153): the first tracked
    // point is (0, 0); the first control point is the focus the source uses.
    focal_hist.assign(1, 0.0);
    control_hist.assign(1, gp.ctl_y);
    focus.control_x = gp.ctl_x;
    focus.control_y = gp.ctl_y;
    {
      int dev = 0, sms = 0, per_sm = 0;
      CRP_CUDA(cudaGetDevice(&dev));
      CRP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      const bool rk = cfg.ext_rp_scheme == CRP_RP_RK45;
      if (mixed)
        CRP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, rk ? bubble_rk45<PrecMixed> : bubble_rp<PrecMixed>, kRpThreads, 0));
      else
        CRP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, rk ? bubble_rk45<PrecFP64> : bubble_rp<PrecFP64>, kRpThreads, 0));
      rp_grid_full = std::max(1, std::min(sms * std::max(per_sm, 1), (hs.nb + kRpThreads - 1) / kRpThreads));
      rp_grid = rp_grid_full;
      couple_graph_grid = 4 * sms;
    }
    // PML profiles and metrics.
    CRP_CUDA(cudaMemcpyAsync(d_sigma, hs.sigma_block.data(), sizeof(double) * hs.sigma_block.size(),
                             cudaMemcpyHostToDevice, stream));
    set_sigma_pointers();
    if (cfg.ext_elements > 0) {
      std::vector<double> e0(2 * (size_t)cfg.ext_elements, 0.0);
      std::fill(e0.begin(), e0.begin() + cfg.ext_elements, 1.0);
      // On the simulation's stream, after the pool's clearing (a pageable
      // source is staged before the call returns).
      CRP_CUDA(cudaMemcpyAsync(d_elem, e0.data(), sizeof(double) * e0.size(), cudaMemcpyHostToDevice, stream));
    }
    gp.elem_n = cfg.ext_elements;
    gp.elem_rap = hs.d.elem_rap;
    gp.elem_amp = d_elem;
    gp.elem_phase = d_elem + std::max(cfg.ext_elements, 1);
    // Bubbles: initial state of bubble_input (src/bubble_CUDA.cu:900-943).
    if (hs.nb > 0) {
      const int n = hs.nb;
      std::vector<double> zeros(n, 0.0), dt0(n, bp.dt0), pg0(n);
      for (int k = 0; k < n; k++) pg0[k] = cfg.bub_P0 + 2.0 * cfg.bub_sigma / hs.r0[k];
      auto up = [&](double* d, const std::vector<double>& h) {
        return cudaMemcpyAsync(d, h.data(), sizeof(double) * n, cudaMemcpyHostToDevice, stream);
      };
      {
        std::vector<int> ident(n);
        for (int k = 0; k < n; k++) ident[k] = k;
        CRP_CUDA(cudaMemcpyAsync(lpt.order, ident.data(), sizeof(int) * n, cudaMemcpyHostToDevice, stream));
        CRP_CUDA(cudaStreamSynchronize(stream));
      }
      CRP_CUDA(up(bub.x, hs.bx));
      CRP_CUDA(up(bub.y, hs.by));
      CRP_CUDA(up(bub.R0, hs.r0));
      CRP_CUDA(up(bub.n_B, hs.nb_w));
      for (double* d : {bub.R_t, bub.R_p, bub.R_pn, bub.R_n, bub.R_nn}) CRP_CUDA(up(d, hs.r0));
      for (double* d : {bub.PG_p, bub.PG_n}) CRP_CUDA(up(d, pg0));
      for (double* d : {bub.dt, bub.dt_n}) CRP_CUDA(up(d, dt0));
      CRP_CUDA(cudaStreamSynchronize(stream));
      // Init kernels (src/bubble_CUDA.cu:175-187): indices, void fraction, history.
      int nb = (n + 255) / 256;
      CRP_CUDA(launch(kClassOther, [&] { bubble_index<<<nb, 256, 0, stream>>>(gp, bub, bins.count); }));
      CRP_CUDA(build_bins());
      CRP_CUDA(launch_contrib_only());
      CRP_CUDA(launch_couple(/*pressure=*/false));
      size_t bytes = sizeof(double) * cells;
      CRP_CUDA(cudaMemcpyAsync(fg[fg_b], fg[fg_a], bytes, cudaMemcpyDeviceToDevice, stream));
      CRP_CUDA(cudaMemcpyAsync(fg[fg_c], fg[fg_a], bytes, cudaMemcpyDeviceToDevice, stream));
    }
    CRP_CUDA(cudaStreamSynchronize(stream));
    return CRP_OK;
  }

  // Tensor maps (2-D, the whole frame, boxes of kBoxX x kBoxY) of
  // every field buffer, for the TMA-fed FDTD pass.  The encoder is the CUDA
  // driver API's cuTensorMapEncodeTiled, reached through the runtime's entry-point query.
  crp_status make_tensor_maps() {
    using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    CRP_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
    if (!fn || q != cudaDriverEntryPointSuccess) return fail(CRP_ERR_CUDA, "cuTensorMapEncodeTiled not available");
    const Encode enc = reinterpret_cast<Encode>(fn);
    const Frame& f = gp.f;
    auto make = [&](CUtensorMap* m, void* base, int esz) -> bool {
      const cuuint64_t dims[2] = {(cuuint64_t)f.pitch, (cuuint64_t)(f.Y + 4)};
      const cuuint64_t strides[1] = {(cuuint64_t)f.pitch * (cuuint64_t)esz};
      const cuuint32_t box[2] = {(cuuint32_t)kBoxX, (cuuint32_t)kBoxY};
      const cuuint32_t estr[2] = {1, 1};
      return enc(m, esz == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims,
                 strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    };
    const int fg_esz = mixed ? 4 : 8;
    bool ok = true;
    for (int k = 0; k < 2; k++) {
      ok = ok && make(&tm_v[0][k], vx[k], 8) && make(&tm_v[1][k], vy[k], 8);
      ok = ok && make(&tm_p[0][k], px[k], 8) && make(&tm_p[1][k], py[k], 8);
    }
    for (int k = 0; k < 3; k++) ok = ok && make(&tm_fg[k], fg[k], fg_esz);
    if (!ok) return fail(CRP_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    // Tiles of kTileX x kTileY cells; a persistent grid of two blocks per SM.
    int dev = 0, sms = 0;
    CRP_CUDA(cudaGetDevice(&dev));
    CRP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    tile_ntx = (f.X + kTileX - 1) / kTileX;
    tile_n = tile_ntx * ((f.Y + kTileY - 1) / kTileY);
    tile_grid = std::max(1, std::min(tile_n, 2 * sms));
    if (mixed)
      CRP_CUDA(cudaFuncSetAttribute(fdtd_tile<PrecMixed>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    TileLayout<PrecMixed>::smem_bytes));
    else
      CRP_CUDA(cudaFuncSetAttribute(fdtd_tile<PrecFP64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    TileLayout<PrecFP64>::smem_bytes));
    return CRP_OK;
  }

  void fill_params() {
    const Derived& d = hs.d;
    Frame f;
    f.X = cfg.grid_x;
    f.Y = cfg.grid_y;
    f.pitch = ((f.X + 4) + 31) / 32 * 32;
    gp.f = f;
    gp.dx = d.dx;
    gp.dy = d.dy;
    gp.rdx = d.rdx;
    gp.rdy = d.rdy;
    gp.dt = d.dt;
    gp.rho_inf = d.rho_inf;
    gp.c_inf = d.c_inf;
    gp.P_inf = d.P_inf;
    gp.pml_x0 = cfg.pml_x0;
    gp.pml_x1 = cfg.pml_x1;
    gp.pml_y0 = cfg.pml_y0;
    gp.pml_y1 = cfg.pml_y1;
    gp.cyl = cfg.tr_cylindrical;
    gp.plane_p = cfg.tr_plane_p;
    gp.focused_p = cfg.tr_focused_p;
    gp.plane_v = cfg.tr_plane_v;
    gp.focused_v = cfg.tr_focused_v;
    gp.source_row = cfg.ext_source_row;
    gp.amp = cfg.tr_amp;
    gp.pamp = d.rho_inf * d.c_inf * cfg.tr_amp;
    gp.freq = cfg.tr_freq;
    gp.omega = d.omega;
    gp.on_time = (double)cfg.tr_on_wave / cfg.tr_freq;
    gp.period = ((double)cfg.tr_on_wave + (double)cfg.tr_off_wave) / cfg.tr_freq;
    gp.ramp_time = cfg.ext_ramp_cycles > 0.0 ? cfg.ext_ramp_cycles / cfg.tr_freq : 0.0;
    gp.ctl_x = d.ctl_x;
    gp.ctl_y = d.ctl_y;
    gp.focal_dist = d.focal_dist;
    gp.dt_rho = d.dt / d.rho_inf;
    gp.s3p = d.dt * d.rho_inf * d.c_inf * d.c_inf;
    gp.s4p = 0.5 * d.dt * d.c_inf;
    bp.PL0 = cfg.bub_P0;
    bp.T0 = cfg.bub_T0;
    bp.gam = cfg.bub_gamma;
    bp.sig = cfg.bub_sigma;
    bp.mu = cfg.bub_mu;
    bp.rho = cfg.bub_rho;
    bp.inv_rho = 1.0 / cfg.bub_rho;
    {
      // Smallest squared modulus whose square root is above 0.1, per precision.
      double c = 0.01;
      while (std::sqrt(c) > 0.1) c = std::nextafter(c, 0.0);
      while (!(std::sqrt(c) > 0.1)) c = std::nextafter(c, 1.0);
      bp.abs2_cut64 = c;
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
    bp.K0 = cfg.bub_K0;
    bp.dt0 = d.bub_dt0;
    bp.pi = d.pi;
    bp.pi4r3 = d.pi4r3;
    bp.dcx = d.dcx;
    bp.dcy = d.dcy;
    bp.dcz = d.dcz;
    bp.step_cap = cfg.ext_rp_step_cap;
    bp.rk_rtol = cfg.ext_rp_tol > 0.0 ? cfg.ext_rp_tol : kRk45DefaultTol;
    bp.reuse = cfg.ext_rp_reuse ? 1 : 0;
  }

  void set_sigma_pointers() {
    const double* b = d_sigma;
    gp.mx = b + hs.off_mx;
    gp.my = b + hs.off_my;
    gp.nx = b + hs.off_nx;
    gp.ny = b + hs.off_ny;
    gp.xu = b + hs.off_xu;
    gp.rxp = b + hs.off_rxp;
    gp.vax = b + hs.off_vax;
    gp.vbx = b + hs.off_vbx;
    gp.vay = b + hs.off_vay;
    gp.vby = b + hs.off_vby;
    gp.pax = b + hs.off_pax;
    gp.pbx = b + hs.off_pbx;
    gp.pay = b + hs.off_pay;
    gp.pby = b + hs.off_pby;
  }

  cudaError_t build_bins() {
    const int nbins = bins.nbins;
    const int nblk = (nbins + kScanThreads - 1) / kScanThreads;
    cudaError_t e;
    if ((e = launch(kClassOther, [&] {
           bin_count_kernel<<<(bub.n + 255) / 256, 256, 0, stream>>>(bub.bin, bub.n, bins.count);
         })) != cudaSuccess)
      return e;
    if ((e = launch(kClassOther, [&] {
           bin_scan_blocks<<<nblk, kScanThreads, 0, stream>>>(bins.count, bins.start, bins.partial, nbins);
         })) != cudaSuccess)
      return e;
    if ((e = launch(kClassOther, [&] { bin_scan_partials<<<1, kScanThreads, 0, stream>>>(bins.partial, nblk); })) !=
        cudaSuccess)
      return e;
    if ((e = launch(kClassOther, [&] {
           bin_scan_add<<<(nbins + 1 + 255) / 256, 256, 0, stream>>>(bins.start, bins.partial, nbins, nblk);
         })) != cudaSuccess)
      return e;
    if ((e = launch(kClassOther, [&] {
           bin_fill<<<(bub.n + 255) / 256, 256, 0, stream>>>(bub.bin, bub.n, bins.start, bins.count, bins.idx);
         })) != cudaSuccess)
      return e;
    if ((e = launch(kClassOther, [&] {
           bin_sort<<<(nbins + 255) / 256, 256, 0, stream>>>(bins.start, bins.idx, nbins);
         })) != cudaSuccess)
      return e;
    if ((e = cudaMemsetAsync(bub.pos, 0xff, sizeof(int) * bub.n, stream)) != cudaSuccess) return e;
    return launch(kClassOther, [&] {
      bin_pos<<<(bub.n + 255) / 256, 256, 0, stream>>>(bins.idx, bins.start + nbins, bub.pos, bub.n);
    });
  }

  // Radius-solve order from the last sub-step counts (heaviest first).
  cudaError_t build_order() {
    const int n = bub.n;
    cudaError_t e;
    if ((e = launch(kClassOther, [&] { lpt_count<<<(n + 255) / 256, 256, 0, stream>>>(bub.nsub, n, lpt.hist); })) !=
        cudaSuccess)
      return e;
    if ((e = launch(kClassOther, [&] { lpt_scan<<<1, 32, 0, stream>>>(lpt.hist, lpt.cursor); })) != cudaSuccess)
      return e;
    return launch(kClassOther,
                  [&] {
                    lpt_scatter<<<(n + kLptScatterThreads - 1) / kLptScatterThreads, kLptScatterThreads, 0, stream>>>(
                        bub.nsub, n, lpt.cursor, lpt.order);
                  });
  }

  // Void-fraction contributions of the initial radii (no RP step).
  cudaError_t launch_contrib_only();

  cudaError_t launch_couple(bool pressure);

  Box full_box() const { return Box{0, 0, gp.f.X + 1, gp.f.Y + 1}; }
  static bool box_empty(const Box& b) { return b.i0 > b.i1 || b.j0 > b.j1; }
  static Box box_union(const Box& a, const Box& b) {
    if (box_empty(a)) return b;
    if (box_empty(b)) return a;
    return Box{std::min(a.i0, b.i0), std::min(a.j0, b.j0), std::max(a.i1, b.i1), std::max(a.j1, b.j1)};
  }
  // Cells reached by the stencils of the occupied bins (bin (bx, by) feeds
  // cells bx..bx+1, by..by+1; with the axis fold cells 0 and 1 go together).
  Box bubble_box() const {
    const int* e = h_scalars->bbox;
    if (e[1] == 0) return Box{1, 1, 0, 0};
    const int X = gp.f.X, Y = gp.f.Y;
    Box b{std::max(0, kBoxOff - e[0]), std::max(0, kBoxOff - e[2]), std::min(X + 1, e[1] - kBoxOff + 1),
          std::min(Y + 1, e[3] - kBoxOff + 1)};
    if (box_empty(b)) return b;
    if (gp.cyl && b.i0 <= 1) {
      b.i0 = 0;
      b.i1 = std::max(b.i1, 1);
    }
    return b;
  }

  crp_status read_scalars() {
    CRP_CUDA(cudaMemcpyAsync(h_scalars, d_scalars, sizeof(Scalars), cudaMemcpyDeviceToHost, stream));
    CRP_CUDA(wait_stream());
    prof.resolve();
    return CRP_OK;
  }

  // The host's waits inside a step: spinning (the default: the shortest
  // wake-up), or blocking on an event that yields the CPU core (crp_batch with
  // more host threads than cores).
  cudaError_t wait_stream() {
    if (!blocking_waits) return cudaStreamSynchronize(stream);
    cudaError_t e = cudaEventRecord(ev_block, stream);
    return e != cudaSuccess ? e : cudaEventSynchronize(ev_block);
  }
  crp_status set_blocking_waits(bool on) {
    if (on && !ev_block) CRP_CUDA(cudaEventCreateWithFlags(&ev_block, cudaEventDisableTiming | cudaEventBlockingSync));
    blocking_waits = on;
    return CRP_OK;
  }

  // The first part of every step: the step's times (compensated sum,
  // src/bubble_CUDA.cu:208-212), set_time and the FDTD pass, with the buffer
  // rotations.
  cudaError_t queue_fdtd_step() {
    t_prev = tstep;
    double s1 = tstep;
    tstep = tstep + gp.dt + tstepx;
    double s2 = tstep - s1;
    tstepx = gp.dt + tstepx - s2;
    cudaError_t e = launch(kClassOther, [&] { set_time<<<1, 1, 0, stream>>>(d_scalars, t_prev, tstep, tstepx); });
    if (e != cudaSuccess) return e;
    const int nv = cur_v ^ 1, np = cur_p ^ 1;
    // Ring rotation of store_variables: the predicted f_g goes to the f_gm buffer.
    const int a = fg_a, b = fg_b, c = fg_c;
    e = mixed ? launch_fdtd<PrecMixed>(nv, np, a, b, c) : launch_fdtd<PrecFP64>(nv, np, a, b, c);
    if (e != cudaSuccess) return e;
    cur_v = nv;
    cur_p = np;
    fg_a = c;  // predicted f_g
    fg_b = a;  // f_gn
    fg_c = b;  // f_gm
    return cudaSuccess;
  }

  // Steps of a simulation without bubbles (no temperature branch, profiling or
  // Picard trace): nothing the host decides depends on a step's scalars, so
  // queue_plain queues the steps back to back and finish_plain reads the
  // scalars once, after the last.  The FDTD pass's error flag is sticky and
  // a non-finite pressure stays non-finite in the linear bubble-free step, so
  // the last step's scalars carry what step_once would have found at any step.
  bool plain_ok() const { return hs.nb == 0 && !temperature_on && !prof.on && !debug_picard && stats.steps > 0; }
  crp_status queue_plain() {
    CRP_CUDA(queue_fdtd_step());
    // The support boxes as step_once leaves them without bubbles.
    const Box snow = box_union(supp[0], box_union(supp[1], supp[2]));
    couple_box = box_union(box_union(Box{1, 1, 0, 0}, supp[0]), box_union(supp[1], supp[2]));
    supp[2] = supp[1];
    supp[1] = supp[0];
    supp[0] = snow;
    stats.steps++;
    stats.time = tstep;
    stats.picard_last = 0;
    return CRP_OK;
  }
  crp_status finish_plain() {
    CRP_CUDA(cudaMemcpyAsync(h_scalars, d_scalars, sizeof(Scalars), cudaMemcpyDeviceToHost, stream));
    CRP_CUDA(wait_stream());
    if (h_scalars->pipe_err) return fail(CRP_ERR_CUDA, "an mbarrier wait of the FDTD pass timed out");
    const double resimax = __longlong_as_double_host(h_scalars->residual) / gp.P_inf;
    if (std::isnan(resimax)) return fail(CRP_ERR_NONFINITE, "non-finite pressure");
    stats.residual_last = resimax;
    stats.rp_substeps_max = h_scalars->substep_max;
    stats.rp_reused = (int64_t)h_scalars->reused;
    fill_launch_stats();
    return CRP_OK;
  }

  crp_status step_once() {
    CRP_CUDA(queue_fdtd_step());
    if (hs.nb > 0) CRP_CUDA(mixed ? launch_move<PrecMixed>() : launch_move<PrecFP64>());
    // The first radius solve is queued right behind the read-back of the
    // prediction's scalars, and picard_gate decides on the device whether it
    // runs, so that the GPU does not idle while the host decides.  Not while
    // the bins are already known to be stale: the solve stores each bubble's
    // contributions at its place in the bins.  The solve order depends only on
    // the sub-step counts of earlier solves, known before this read-back.
    // Bins change only when a bubble crosses into another cell; the order is
    // left as it is while no bubble has needed more than kLptMinSubsteps
    // sub-steps (all equal: the order cannot shorten the launch).
    const long long substep_prev = h_scalars->substep_max;
    const bool ahead = hs.nb > 0 && !bins_stale && cfg.ext_picard_cap > 0;
    CRP_CUDA(cudaMemcpyAsync(h_scalars, d_scalars, sizeof(Scalars), cudaMemcpyDeviceToHost, stream));
    if (ahead) {
      cudaEvent_t ev = blocking_waits ? ev_block : ev_scalars;
      CRP_CUDA(cudaEventRecord(ev, stream));
      if (substep_prev > kLptMinSubsteps) CRP_CUDA(build_order());
      CRP_CUDA(launch(kClassOther,
                      [&] { picard_gate<<<1, 1, 0, stream>>>(d_scalars, gp.P_inf, picard_tol, hs.nb); }));
      CRP_CUDA(mixed ? launch_rp<PrecMixed>() : launch_rp<PrecFP64>());
      CRP_CUDA(cudaEventSynchronize(ev));
    } else {
      CRP_CUDA(wait_stream());
      prof.resolve();
    }
    crp_status st = CRP_OK;
    if (h_scalars->pipe_err) return fail(CRP_ERR_CUDA, "an mbarrier wait of the FDTD pass timed out");
    double resimax = __longlong_as_double_host(h_scalars->residual) / gp.P_inf;
    int loop = 0;
    // picard_gate's decision: the first iteration's solve is already queued.
    const bool first_queued = ahead && resimax > picard_tol && h_scalars->moved == 0;
    bins_stale = bins_stale || h_scalars->moved != 0;
    const Box bnow = hs.nb > 0 ? bubble_box() : Box{1, 1, 0, 0};
    couple_box = box_union(box_union(bnow, supp[0]), box_union(supp[1], supp[2]));
    if (hs.nb > 0 && resimax > picard_tol && !first_queued) {
      if (bins_stale) CRP_CUDA(build_bins());
      bins_stale = false;
      if (!ahead && substep_prev > kLptMinSubsteps) CRP_CUDA(build_order());
    }
    if (hs.nb > 0) {
      double prev = resimax;
      while (resimax > picard_tol) {
        if (loop >= cfg.ext_picard_cap) return fail(CRP_ERR_PICARD, "Picard iteration cap reached");
        loop++;
        if (!(first_queued && loop == 1)) {
          CRP_CUDA(launch(kClassOther, [&] { picard_begin<<<1, 1, 0, stream>>>(d_scalars, loop - 1); }));
          CRP_CUDA(mixed ? launch_rp<PrecMixed>() : launch_rp<PrecFP64>());
        }
        CRP_CUDA(launch_couple(true));
        st = read_scalars();
        if (st != CRP_OK) return st;
        if (h_scalars->err) return fail(CRP_ERR_RP_STEPS, "Rayleigh-Plesset sub-step cap reached");
        resimax = __longlong_as_double_host(h_scalars->residual) / gp.P_inf;
        if (debug_picard && loop <= 40)
          fprintf(stderr, "step %lld picard %d residual %.6e\n", (long long)stats.steps + 1, loop, resimax);
        if (mixed && loop >= 3 && resimax > picard_tol && resimax > 0.5 * prev && resimax < CRP_MIXED_STALL_RESIDUAL) {
          stats.picard_stalls++;
          break;
        }
        prev = resimax;
      }
    }
    if (ahead && loop == 0 && prof.on) {
      // The gated solve and its timing events are still in flight.
      CRP_CUDA(cudaStreamSynchronize(stream));
      prof.resolve();
    }
    if (std::isnan(resimax)) return fail(CRP_ERR_NONFINITE, "non-finite pressure");
    if (temperature_on) {
      CRP_CUDA(mixed ? launch_temperature<PrecMixed>() : launch_temperature<PrecFP64>());
      const crp_status fs = track_focus(stats.steps + 1);
      if (fs != CRP_OK) return fs;
    }
    // Support of this step's void fraction: the gather's when it ran, else the
    // prediction's.
    const Box snow = loop > 0 ? bnow : box_union(supp[0], box_union(supp[1], supp[2]));
    supp[2] = supp[1];
    supp[1] = supp[0];
    supp[0] = snow;
    stats.steps++;
    stats.time = tstep;
    stats.picard_last = loop;
    stats.picard_total += loop;
    stats.picard_max = std::max(stats.picard_max, loop);
    stats.residual_last = resimax;
    stats.rp_substeps_max = h_scalars->substep_max;
    stats.rp_reused = (int64_t)h_scalars->reused;
    fill_launch_stats();
    return CRP_OK;
  }

  void fill_launch_stats() {
    stats.kernel_launches = launches[0] + launches[1] + launches[2] + launches[3];
    stats.fdtd_launches = launches[kClassFdtd];
    stats.rp_launches = launches[kClassRp];
    stats.couple_launches = launches[kClassCouple];
    stats.ms_fdtd = prof.ms[kClassFdtd];
    stats.ms_rp = prof.ms[kClassRp];
    stats.ms_couple = prof.ms[kClassCouple];
    stats.ms_other = prof.ms[kClassOther];
  }

  static double __longlong_as_double_host(unsigned long long b) {
    double d;
    std::memcpy(&d, &b, sizeof(d));
    return d;
  }

  // Copy the window [ilo, ihi] x [jlo, jhi] of a field buffer into a dense
  // double array.  kind: 0 FP64, 1 FP32 value + compensation, 2 FP32.
  crp_status copy_window(const void* buf, int kind, int ilo, int ihi, int jlo, int jhi, double* host) {
    const Frame& f = gp.f;
    const int w = ihi - ilo + 1, h = jhi - jlo + 1;
    const long off = f.idx(ilo, jlo);
    if (kind == 0) {
      CRP_CUDA(cudaMemcpy2DAsync(host, sizeof(double) * w, (const double*)buf + off, sizeof(double) * f.pitch,
                                 sizeof(double) * w, h, cudaMemcpyDeviceToHost, stream));
      CRP_CUDA(cudaStreamSynchronize(stream));
      return CRP_OK;
    }
    // kind 1: (value, compensation) float pairs; kind 2: single floats.
    const size_t per = kind == 1 ? 2 : 1;
    std::vector<float> v((size_t)w * h * per);
    const float* fb = (const float*)buf;
    CRP_CUDA(cudaMemcpy2DAsync(v.data(), sizeof(float) * per * w, fb + per * off, sizeof(float) * per * f.pitch,
                               sizeof(float) * per * w, h, cudaMemcpyDeviceToHost, stream));
    CRP_CUDA(cudaStreamSynchronize(stream));
    for (size_t q = 0; q < (size_t)w * h; q++)
      host[q] = kind == 1 ? (double)v[2 * q] + (double)v[2 * q + 1] : (double)v[q];
    return CRP_OK;
  }

  // ---- Graph path --------------------------------------------------------
  // One mixture step as a CUDA graph whose control flow runs on the device:
  //   ctl_step_begin -> IF(step ok) {
  //     fdtd_strip, bubble_move (with the ghost cells), ctl_enter -> IF(Picard needed) {
  //       ctl_bins -> IF(bins stale) { counting sort } -> solve order ->
  //       WHILE(residual > threshold) { bubble_rp, couple_press, ctl_iter } }
  //     -> ctl_end }
  // so a crp_step call of n steps is n graph launches and one read-back,
  // instead of two host round trips per step.  The arithmetic is the host
  // path's, kernel for kernel.
  int phase() const { return cur_v * 3 + fg_a; }

  void rotate_once() {
    cur_v ^= 1;
    cur_p ^= 1;
    const int a = fg_a, b = fg_b, c = fg_c;
    fg_a = c;
    fg_b = a;
    fg_c = b;
  }

  // Appends what fn enqueues on `stream` to graph g after the nodes deps and
  // returns the capture's last nodes in sinks.
  template <typename F>
  cudaError_t capture(cudaGraph_t g, const std::vector<cudaGraphNode_t>& deps, std::vector<cudaGraphNode_t>& sinks,
                      F&& fn) {
    cudaError_t e = cudaStreamBeginCaptureToGraph(cap_stream, g, deps.empty() ? nullptr : deps.data(), nullptr,
                                                  deps.size(), cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    const cudaStream_t saved = stream;
    int64_t saved_launches[4];
    std::memcpy(saved_launches, launches, sizeof(launches));
    stream = cap_stream;
    capturing = true;
    const cudaError_t fe = fn();
    capturing = false;
    stream = saved;
    std::memcpy(launches, saved_launches, sizeof(launches));
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* d = nullptr;
    size_t nd = 0;
    const cudaError_t ie = cudaStreamGetCaptureInfo(cap_stream, &cs, nullptr, nullptr, &d, &nd);
    if (ie == cudaSuccess) sinks.assign(d, d + nd);
    cudaGraph_t out = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(cap_stream, &out);
    return fe != cudaSuccess ? fe : ie != cudaSuccess ? ie : ee;
  }

  static cudaError_t add_cond(cudaGraph_t g, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type,
                              cudaGraphNode_t* node, cudaGraph_t* body) {
    cudaGraphNodeParams p{};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = type;
    p.conditional.size = 1;
    const cudaError_t e = cudaGraphAddNode(node, g, nullptr, 0, &p);
    if (e == cudaSuccess) *body = p.conditional.phGraph_out[0];
    return e;
  }

  static cudaError_t link(cudaGraph_t g, const std::vector<cudaGraphNode_t>& from, cudaGraphNode_t to) {
    for (cudaGraphNode_t f : from) {
      const cudaError_t e = cudaGraphAddDependencies(g, &f, &to, 1);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }

  cudaError_t build_step_graph(int ph) {
    if (!cap_stream) {
      cudaError_t e = cudaStreamCreateWithFlags(&cap_stream, cudaStreamNonBlocking);
      if (e != cudaSuccess) return e;
    }
    cudaGraph_t top = nullptr;
    cudaError_t e = cudaGraphCreate(&top, 0);
    if (e != cudaSuccess) return e;
    step_graph[ph] = top;
    CtlParams c{};
    c.tol = picard_tol;
    c.P_inf = gp.P_inf;
    c.dt = gp.dt;
    c.stall = CRP_MIXED_STALL_RESIDUAL;
    c.cap = cfg.ext_picard_cap;
    c.nb = hs.nb;
    c.mixed = mixed ? 1 : 0;
    c.X = gp.f.X;
    c.Y = gp.f.Y;
    c.cyl = gp.cyl;
    cudaGraphNode_t n_step, n_picard, n_bins, n_loop;
    cudaGraph_t body1, body2, body3, body4;
    std::vector<cudaGraphNode_t> sinks;
#define CRP_G(x)                       \
  do {                                 \
    cudaError_t ge_ = (x);             \
    if (ge_ != cudaSuccess) return ge_; \
  } while (0)
    CRP_G(cudaGraphConditionalHandleCreate(&c.h_step, top, 0, cudaGraphCondAssignDefault));
    CRP_G(add_cond(top, c.h_step, cudaGraphCondTypeIf, &n_step, &body1));
    CRP_G(cudaGraphConditionalHandleCreate(&c.h_picard, body1, 0, cudaGraphCondAssignDefault));
    CRP_G(add_cond(body1, c.h_picard, cudaGraphCondTypeIf, &n_picard, &body2));
    CRP_G(cudaGraphConditionalHandleCreate(&c.h_bins, body2, 0, cudaGraphCondAssignDefault));
    CRP_G(cudaGraphConditionalHandleCreate(&c.h_loop, body2, 1, cudaGraphCondAssignDefault));
    CRP_G(add_cond(body2, c.h_bins, cudaGraphCondTypeIf, &n_bins, &body3));
    CRP_G(add_cond(body2, c.h_loop, cudaGraphCondTypeWhile, &n_loop, &body4));
    Scalars* ds = d_scalars;
    // Top level.
    CRP_G(capture(top, {}, sinks, [&] {
      return launch(kClassOther, [&] { ctl_step_begin<<<1, 1, 0, stream>>>(ds, c); });
    }));
    CRP_G(link(top, sinks, n_step));
    // The step body, with the buffers of this phase.
    const int sv = cur_v, sp = cur_p, sa = fg_a, sb = fg_b, sc = fg_c;
    cudaError_t be = capture(body1, {}, sinks, [&]() -> cudaError_t {
      const int nv = cur_v ^ 1, np = cur_p ^ 1;
      cudaError_t x = mixed ? launch_fdtd<PrecMixed>(nv, np, fg_a, fg_b, fg_c)
                            : launch_fdtd<PrecFP64>(nv, np, fg_a, fg_b, fg_c);
      if (x != cudaSuccess) return x;
      rotate_once();
      if (hs.nb > 0) {
        x = mixed ? launch_move<PrecMixed>() : launch_move<PrecFP64>();
        if (x != cudaSuccess) return x;
      }
      return launch(kClassOther, [&] { ctl_enter<<<1, 1, 0, stream>>>(ds, c, kBoxOff); });
    });
    if (be == cudaSuccess) be = link(body1, sinks, n_picard);
    if (be == cudaSuccess)
      be = capture(body1, {n_picard}, sinks,
                   [&] { return launch(kClassOther, [&] { ctl_end<<<1, 1, 0, stream>>>(ds, c); }); });
    // Picard body: bins, order, loop (buffers as after the rotation).
    if (be == cudaSuccess)
      be = capture(body2, {}, sinks,
                   [&] { return launch(kClassOther, [&] { ctl_bins<<<1, 1, 0, stream>>>(ds, c); }); });
    if (be == cudaSuccess) be = link(body2, sinks, n_bins);
    if (be == cudaSuccess) be = capture(body2, {n_bins}, sinks, [&] { return build_order(); });
    if (be == cudaSuccess) be = link(body2, sinks, n_loop);
    if (be == cudaSuccess) be = capture(body3, {}, sinks, [&] { return build_bins(); });
    if (be == cudaSuccess)
      be = capture(body4, {}, sinks, [&]() -> cudaError_t {
        cudaError_t x = mixed ? launch_rp<PrecMixed>() : launch_rp<PrecFP64>();
        if (x != cudaSuccess) return x;
        x = launch_couple(true);
        if (x != cudaSuccess) return x;
        return launch(kClassOther, [&] { ctl_iter<<<1, 1, 0, stream>>>(ds, c); });
      });
    cur_v = sv;
    cur_p = sp;
    fg_a = sa;
    fg_b = sb;
    fg_c = sc;
    CRP_G(be);
    CRP_G(cudaGraphInstantiate(&step_exec[ph], top, 0));
#undef CRP_G
    return cudaSuccess;
  }

  // Host state into the device block before graph steps.
  cudaError_t push_ctl() {
    Scalars& h = *h_push;
    std::memset(&h, 0, sizeof(Scalars));
    h.substep_max = h_scalars->substep_max;
    h.t[0] = t_prev;
    h.t[1] = tstep;
    h.t[2] = tstepx;
    h.steps = stats.steps;
    h.picard_total = stats.picard_total;
    h.stalls = stats.picard_stalls;
    h.reused = (unsigned long long)stats.rp_reused;
    h.picard_last = stats.picard_last;
    h.picard_max = stats.picard_max;
    h.res_last = stats.residual_last;
    h.stale = bins_stale ? 1 : 0;
    for (int q = 0; q < 3; q++) {
      h.supp[q][0] = supp[q].i0;
      h.supp[q][1] = supp[q].j0;
      h.supp[q][2] = supp[q].i1;
      h.supp[q][3] = supp[q].j1;
    }
    return cudaMemcpyAsync(d_scalars, h_push, sizeof(Scalars), cudaMemcpyHostToDevice, stream);
  }

  // n steps through the graph path; one read-back at the end.
  crp_status step_graphs(int n) {
    const crp_status st = graphs_enqueue(n);
    if (st != CRP_OK) return st;
    return graphs_finish();
  }

  // The next step may run as a graph (crp_step runs the others from the host).
  bool graph_ready() const {
    return !(stats.steps == 0 || prof.on || !graphs_on || hs.nb == 0 || debug_picard || temperature_on);
  }

  // Queues n graph steps and the read-back of the device scalars on the
  // simulation's stream without waiting for them; graphs_finish completes them.
  crp_status graphs_enqueue(int n) {
    if (pend.on) return fail(CRP_ERR_INVALID, "graph steps already queued");
    if (!h_push) CRP_CUDA(cudaMallocHost(&h_push, sizeof(Scalars)));
    for (int k = 0; k < 6; k++)
      if (!step_exec[k]) {
        // Build all phases up front so that the launches below do not interleave with captures.
        const int sv = cur_v, sp = cur_p, sa = fg_a, sb = fg_b, sc = fg_c;
        for (int r = 0; r < 6; r++) {
          const int ph = phase();
          if (!step_exec[ph]) {
            const cudaError_t e = build_step_graph(ph);
            if (e != cudaSuccess) {
              graphs_on = false;
              cur_v = sv, cur_p = sp, fg_a = sa, fg_b = sb, fg_c = sc;
              return CRP_ERR_UNSUPPORTED;
            }
          }
          rotate_once();
        }
        cur_v = sv, cur_p = sp, fg_a = sa, fg_b = sb, fg_c = sc;
        break;
      }
    pend.steps0 = stats.steps;
    pend.cur_v = cur_v, pend.cur_p = cur_p, pend.fg_a = fg_a, pend.fg_b = fg_b, pend.fg_c = fg_c;
    CRP_CUDA(push_ctl());
    for (int k = 0; k < n; k++) {
      CRP_CUDA(cudaGraphLaunch(step_exec[phase()], stream));
      rotate_once();
    }
    CRP_CUDA(cudaMemcpyAsync(h_scalars, d_scalars, sizeof(Scalars), cudaMemcpyDeviceToHost, stream));
    pend.on = true;
    return CRP_OK;
  }

  crp_status graphs_finish() {
    if (!pend.on) return CRP_OK;
    pend.on = false;
    CRP_CUDA(cudaStreamSynchronize(stream));
    const int64_t steps0 = pend.steps0;
    const int sv = pend.cur_v, sp = pend.cur_p, sa = pend.fg_a, sb = pend.fg_b, sc = pend.fg_c;
    const Scalars& d = *h_scalars;
    t_prev = d.t[0];
    tstep = d.t[1];
    tstepx = d.t[2];
    const int64_t done = d.steps - steps0;
    stats.steps = d.steps;
    stats.time = tstep;
    stats.picard_total = d.picard_total;
    stats.picard_stalls = d.stalls;
    stats.rp_reused = (int64_t)d.reused;
    stats.picard_last = d.picard_last;
    stats.picard_max = d.picard_max;
    stats.residual_last = d.res_last;
    stats.rp_substeps_max = d.substep_max;
    bins_stale = d.stale != 0;
    for (int q = 0; q < 3; q++) supp[q] = Box{d.supp[q][0], d.supp[q][1], d.supp[q][2], d.supp[q][3]};
    for (int q = 0; q < 4; q++) launches[q] += d.launches[q];
    fill_launch_stats();
    if (d.pipe_err) return fail(CRP_ERR_CUDA, "an mbarrier wait of the FDTD pass timed out");
    if (d.status) {
      // The failed step ran up to its failure (its buffers rotated); later launches did nothing.
      cur_v = sv, cur_p = sp, fg_a = sa, fg_b = sb, fg_c = sc;
      for (int64_t r = 0; r < done + 1; r++) rotate_once();
      const crp_status st = (crp_status)d.status;
      return fail(st, st == CRP_ERR_PICARD      ? "Picard iteration cap reached"
                      : st == CRP_ERR_RP_STEPS ? "Rayleigh-Plesset sub-step cap reached"
                                               : "non-finite pressure");
    }
    return CRP_OK;
  }

  // crp_step: the first step (initial mixture density), profiled steps and
  // simulations without bubbles run from the host; the rest as graphs.
  crp_status step_n(int n) {
    const crp_status pst = graphs_finish();
    if (pst != CRP_OK) return pst;
    int k = 0;
    while (k < n && (stats.steps == 0 || prof.on || !graphs_on || hs.nb == 0 || debug_picard || temperature_on)) {
      if (plain_ok()) {
        for (; k < n; k++) {
          const crp_status st = queue_plain();
          if (st != CRP_OK) return st;
        }
        return finish_plain();
      }
      const crp_status st = step_once();
      if (st != CRP_OK) return st;
      k++;
    }
    if (k >= n) return CRP_OK;
    const crp_status st = step_graphs(n - k);
    if (st == CRP_ERR_UNSUPPORTED && !graphs_on) {
      for (; k < n; k++) {
        const crp_status s2 = step_once();
        if (s2 != CRP_OK) return s2;
      }
      return CRP_OK;
    }
    return st;
  }

  crp_status read_field(crp_field which, double* host) {
    const int X = gp.f.X, Y = gp.f.Y;
    const int kv = mixed ? 1 : 0, kg = mixed ? 2 : 0;
    switch (which) {
      case CRP_FIELD_P0: {
        CRP_CUDA(mixed ? launch_p0<PrecMixed>() : launch_p0<PrecFP64>());
        CRP_CUDA(cudaMemcpyAsync(host, scratch, sizeof(double) * (X + 2) * (Y + 2), cudaMemcpyDeviceToHost, stream));
        CRP_CUDA(cudaStreamSynchronize(stream));
        return CRP_OK;
      }
      case CRP_FIELD_PX: return copy_window(px[cur_p], kv, 0, X + 1, 0, Y + 1, host);
      case CRP_FIELD_PY: return copy_window(py[cur_p], kv, 0, X + 1, 0, Y + 1, host);
      case CRP_FIELD_PNX: return copy_window(px[cur_p ^ 1], kv, 0, X + 1, 0, Y + 1, host);
      case CRP_FIELD_PNY: return copy_window(py[cur_p ^ 1], kv, 0, X + 1, 0, Y + 1, host);
      case CRP_FIELD_VX: return copy_window(vx[cur_v], kv, -1, X + 1, 0, Y + 1, host);
      case CRP_FIELD_VY: return copy_window(vy[cur_v], kv, 0, X + 1, -1, Y + 1, host);
      case CRP_FIELD_FG: return copy_window(fg[fg_a], kg, 0, X + 1, 0, Y + 1, host);
      case CRP_FIELD_FGN: return copy_window(fg[fg_b], kg, 0, X + 1, 0, Y + 1, host);
      case CRP_FIELD_FGM: return copy_window(fg[fg_c], kg, 0, X + 1, 0, Y + 1, host);
      case CRP_FIELD_T:
        if (!temperature_on) return fail(CRP_ERR_UNSUPPORTED, "the temperature is computed only with debug.T = 1");
        return copy_window(Tbuf[cur_t], 0, 0, X + 1, 0, Y + 1, host);
      case CRP_FIELD_RHO_M: {
        crp_status st = copy_window(fg[fg_a], kg, 0, X + 1, 0, Y + 1, host);
        if (st != CRP_OK) return st;
        size_t n = (size_t)(X + 2) * (Y + 2);
        for (size_t k = 0; k < n; k++) host[k] = stats.steps == 0 ? gp.rho_inf : (1.0 - host[k]) * gp.rho_inf;
        return CRP_OK;
      }
    }
    return fail(CRP_ERR_INVALID, "unknown field");
  }

  // Per-precision launches.
  template <typename P>
  cudaError_t launch_fdtd(int nv, int np, int a, int b, int c) {
    using V = typename P::V;
    using S = typename P::S;
    using G = typename P::G;
    FdtdArgs<P> fa;
    fa.vx_old = view<V>(vx[cur_v]);
    fa.vy_old = view<V>(vy[cur_v]);
    fa.vx_new = view<V>(vx[nv]);
    fa.vy_new = view<V>(vy[nv]);
    fa.pnx = view<S>(px[cur_p]);
    fa.pny = view<S>(py[cur_p]);
    fa.px = view<S>(px[np]);
    fa.py = view<S>(py[np]);
    fa.fgA = view<G>(fg[a]);
    fa.fgB = view<G>(fg[b]);
    fa.fgC = view<G>(fg[c]);
    fa.tdev = d_scalars->t;
    fa.rho_const = stats.steps == 0 ? 1 : 0;
    fa.residual = d_residual;
    cudaError_t e;
    if (fdtd_tma_on) {
      TmaMaps m;
      m.m[0] = tm_p[0][cur_p];
      m.m[1] = tm_p[1][cur_p];
      m.m[2] = tm_fg[a];
      m.m[3] = tm_v[0][cur_v];
      m.m[4] = tm_v[1][cur_v];
      m.m[5] = tm_fg[b];
      m.m[6] = tm_fg[c];
      const dim3 block(kTileX, kTileY);
      const int smem = TileLayout<P>::smem_bytes, ntx = tile_ntx, nt = tile_n, grid = tile_grid;
      int* perr = &d_scalars->pipe_err;
      e = launch(kClassFdtd, [&] { fdtd_tile<P><<<grid, block, smem, stream>>>(gp, fa, m, ntx, nt, perr); });
    } else {
      const int strips = (gp.f.X + kStripCells - 1) / kStripCells, rows = strip_rows;
      dim3 block(32, kStripWarps);
      dim3 grid((strips + kStripWarps - 1) / kStripWarps, (gp.f.Y + rows - 1) / rows);
      if (rows == 4)
        e = launch(kClassFdtd, [&] { fdtd_strip<P, kStripStages, 4><<<grid, block, 0, stream>>>(gp, fa); });
      else if (rows == 16)
        e = launch(kClassFdtd, [&] { fdtd_strip<P, kStripStages, 16><<<grid, block, 0, stream>>>(gp, fa); });
      else
        e = launch(kClassFdtd, [&] { fdtd_strip<P><<<grid, block, 0, stream>>>(gp, fa); });
    }
    if (e != cudaSuccess) return e;
    if (hs.nb > 0) return cudaSuccess;  // bubble_move, which follows, writes the ghost cells
    const int ng = vghost_threads(gp.f);
    const V vxn = view<V>(vx[nv]), vyn = view<V>(vy[nv]);
    return launch(kClassOther, [&] { vghost<V><<<(ng + 255) / 256, 256, 0, stream>>>(gp, vxn, vyn); });
  }

  // Source elements (crp_set_source_elements).
  crp_status set_source_elements(int n, const double* amp, const double* phase) {
    if (n <= 0 || n != gp.elem_n || !amp || !phase) return fail(CRP_ERR_INVALID, "source elements: n must equal ext.elements");
    std::vector<double> e(2 * (size_t)n);
    std::copy(amp, amp + n, e.begin());
    std::copy(phase, phase + n, e.begin() + n);
    CRP_CUDA(cudaMemcpyAsync(d_elem, e.data(), sizeof(double) * e.size(), cudaMemcpyHostToDevice, stream));
    CRP_CUDA(cudaStreamSynchronize(stream));
    return CRP_OK;
  }

  // crp_adjoint (defined below, after the buffer views).
  crp_status adjoint(const crp_objective* obj, double* J, double* grad_amp, double* grad_phase);

  // Fourth-order Butterworth low-pass of the tracked depth (filter_loop,
  // inc/bubble_CUDA_kernel.cuh:117-129), with this simulation's state.
  double filter_depth(double input) {
    double* xv = focus.filter_in;
    double* yv = focus.filter_out;
    const double gain = 6.522112693e+08;
    xv[0] = xv[1];
    xv[1] = xv[2];
    xv[2] = xv[3];
    xv[3] = xv[4];
    xv[4] = input / gain;
    yv[0] = yv[1];
    yv[1] = yv[2];
    yv[2] = yv[3];
    yv[3] = yv[4];
    yv[4] = (xv[0] + xv[4]) + 4 * (xv[1] + xv[3]) + 6 * xv[2] + (-0.9676955438 * yv[0]) + (3.9025587848 * yv[1]) +
            (-5.9020258615 * yv[2]) + (3.9671625959 * yv[3]);
    return yv[4];
  }

  // After the temperature step: the focal depth, its filtered value and, with
  // transducer.pid, the next focus of the source (focal_PID and the clamp of
  // src/bubble_CUDA.cu:328-347, inc/bubble_CUDA_kernel.cuh:1168-1184).
  crp_status track_focus(int64_t nstep) {
    double* part = focal_part;
    CRP_CUDA(launch(kClassOther, [&] {
      focal_max<<<kFocalBlocks, kFocalThreads, 0, stream>>>(dTbuf, gp.f, part);
    }));
    CRP_CUDA(launch(kClassOther, [&] {
      focal_sums<<<kFocalBlocks, kFocalThreads, 0, stream>>>(dTbuf, gp.f, gp.dy, part, kFocalBlocks,
                                                              part + kFocalBlocks);
    }));
    CRP_CUDA(launch(kClassOther, [&] {
      focal_final<<<1, 1, 0, stream>>>(part + kFocalBlocks, kFocalBlocks, part + 3 * kFocalBlocks);
    }));
    CRP_CUDA(cudaMemcpyAsync(h_focal, part + 3 * kFocalBlocks, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream));
    CRP_CUDA(cudaStreamSynchronize(stream));
    const double depth = h_focal[0] > 0.0 ? h_focal[1] / h_focal[0] : 0.0;
    focal_hist.push_back(filter_depth(depth));
    if (cfg.tr_pid && nstep > cfg.tr_pid_start_step) {
      const double K = 0.2 * 0.60, Pc = 1000.0, D = K * 0.125 * Pc, I = K / (0.5 * Pc);
      const double tx = hs.d.fpx, ty = hs.d.fpy;
      const double ax = 0.0, ay = focal_hist[focal_hist.size() - 1];
      const double px_ = 0.0, py_ = focal_hist[focal_hist.size() - 2];
      const double ex = tx - ax, ey = ty - ay;
      focus.err_total_x += ex;
      focus.err_total_y += ey;
      focus.d_err_x = px_ - ax;
      focus.d_err_y = py_ - ay;
      double cy = ty + (K * ey + D * focus.d_err_y + I * focus.err_total_y);
      cy = cy < ty ? ty : (cy > cfg.grid_ly ? cfg.grid_ly : cy);
      control_hist.push_back(cy);
      set_control(0.0, cy);
    }
    return CRP_OK;
  }

  void set_control(double cx, double cy) {
    focus.control_x = cx;
    focus.control_y = cy;
    gp.ctl_x = cx;
    gp.ctl_y = cy;
    gp.focal_dist = cy / 0.5 / std::sqrt(3.0);
  }

  // calculate_temperature after the Picard loop: the bins must follow the
  // bubbles' current cells for the heat gather.
  template <typename P>
  cudaError_t launch_temperature() {
    using S = typename P::S;
    using G = typename P::G;
    cudaError_t e;
    const bool bubbles = hs.nb > 0 && cfg.bub_enable;
    if (bubbles) {
      if (bins_stale) {
        if ((e = build_bins()) != cudaSuccess) return e;
        bins_stale = false;
      }
      if ((e = launch(kClassOther, [&] {
             heat_contrib<<<(bub.n + 255) / 256, 256, 0, stream>>>(gp, bp, bub, heat);
           })) != cudaSuccess)
        return e;
    }
    TempArgs ta;
    ta.T_old = F64{(double*)Tbuf[cur_t]};
    ta.T_new = F64{(double*)Tbuf[cur_t ^ 1]};
    ta.dT = dTbuf;
    ta.start = bins.start;
    ta.idx = bins.idx;
    ta.hc = heat;
    ta.coef_abs = 2.0 * (0.22) * 0.115129255 / (gp.rho_inf * gp.c_inf * gp.omega * gp.omega);
    ta.T_inf = hs.d.T_inf;
    ta.rho_const = stats.steps == 0 ? 1 : 0;
    ta.bubbles = bubbles ? 1 : 0;
    const G fgc = view<G>(fg[fg_a]), fgp = view<G>(fg[fg_b]);
    const S pxc = view<S>(px[cur_p]), pyc = view<S>(py[cur_p]), pxn = view<S>(px[cur_p ^ 1]),
            pyn = view<S>(py[cur_p ^ 1]);
    dim3 blk(32, 8), grd((gp.f.X + 31) / 32, (gp.f.Y + 7) / 8);
    if ((e = launch(kClassOther, [&] {
           temperature_step<P><<<grd, blk, 0, stream>>>(gp, ta, fgc, fgp, pxc, pyc, pxn, pyn);
         })) != cudaSuccess)
      return e;
    if ((e = launch(kClassOther, [&] { temperature_bc<<<1, 1024, 0, stream>>>(gp, ta.T_old, ta.T_new); })) !=
        cudaSuccess)
      return e;
    cur_t ^= 1;
    return cudaSuccess;
  }

  template <typename P>
  cudaError_t launch_move() {
    using V = typename P::V;
    const V vxc = view<V>(vx[cur_v]), vyc = view<V>(vy[cur_v]);
    return launch(kClassOther, [&] {
      const int mb = (bub.n + kMoveThreads - 1) / kMoveThreads;
      const int gb = (vghost_threads(gp.f) + kMoveThreads - 1) / kMoveThreads;
      bubble_move<V><<<mb + gb, kMoveThreads, 0, stream>>>(gp, bp, bub, vxc, vyc, d_moved, mb);
    });
  }

  template <typename P>
  cudaError_t launch_rp() {
    using S = typename P::S;
    const S pxc = view<S>(px[cur_p]), pyc = view<S>(py[cur_p]);
    if (cfg.ext_rp_scheme == CRP_RP_RK45)
      return launch(kClassRp, [&] {
        bubble_rk45<P><<<rp_grid, kRpThreads, 0, stream>>>(gp, bp, bub, pxc, pyc, d_scalars->t, lpt.order, d_next,
                                                            d_substep_max, d_err, &d_scalars->loop,
                                                            &d_scalars->reused);
      });
    return launch(kClassRp, [&] {
      bubble_rp<P><<<rp_grid, kRpThreads, 0, stream>>>(gp, bp, bub, pxc, pyc, d_scalars->t, lpt.order, d_next,
                                                        d_substep_max, d_err, &d_scalars->loop, &d_scalars->reused);
    });
  }

  template <typename P>
  cudaError_t launch_p0() {
    using S = typename P::S;
    const S pxc = view<S>(px[cur_p]), pyc = view<S>(py[cur_p]);
    dim3 blk(32, 8), grd((gp.f.X + 2 + 31) / 32, (gp.f.Y + 2 + 7) / 8);
    return launch(kClassOther,
                  [&] { materialize_p0<S><<<grd, blk, 0, stream>>>(gp, pxc, pyc, tstep, scratch); });
  }

  template <typename P>
  cudaError_t launch_couple_t(bool pressure);

  crp_status read_bubbles(crp_bubble_field w, double* host) {
    const int n = bub.n;
    if (n == 0) return CRP_OK;
    const double* src = nullptr;
    const int* isrc = nullptr;
    switch (w) {
      case CRP_BUB_X: src = bub.x; break;
      case CRP_BUB_Y: src = bub.y; break;
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
      case CRP_BUB_IBM_X: isrc = bub.ibmx; break;
      case CRP_BUB_IBM_Y: isrc = bub.ibmy; break;
      case CRP_BUB_IBN_X: isrc = bub.ibnx; break;
      case CRP_BUB_IBN_Y: isrc = bub.ibny; break;
      case CRP_BUB_SUBSTEPS: isrc = bub.nsub; break;
      default: return fail(CRP_ERR_INVALID, "unknown bubble field");
    }
    if (src) {
      CRP_CUDA(cudaMemcpyAsync(host, src, sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
      CRP_CUDA(cudaStreamSynchronize(stream));
    } else {
      std::vector<int> tmp(n);
      CRP_CUDA(cudaMemcpyAsync(tmp.data(), isrc, sizeof(int) * n, cudaMemcpyDeviceToHost, stream));
      CRP_CUDA(cudaStreamSynchronize(stream));
      for (int k = 0; k < n; k++) host[k] = tmp[k];
    }
    return CRP_OK;
  }

  // Executable graphs hold the launch shapes: rebuilt on next use after a change.
  void drop_graphs() {
    for (int k = 0; k < 6; k++) {
      if (step_exec[k]) cudaGraphExecDestroy(step_exec[k]);
      if (step_graph[k]) cudaGraphDestroy(step_graph[k]);
      step_exec[k] = nullptr;
      step_graph[k] = nullptr;
    }
  }

  crp_status set_tuning(const crp_tuning& t) {
    if (t.fdtd_rows != 4 && t.fdtd_rows != 8 && t.fdtd_rows != 16)
      return fail(CRP_ERR_INVALID, "tuning: fdtd_rows must be 4, 8 or 16");
    if (t.rp_blocks < 0) return fail(CRP_ERR_INVALID, "tuning: rp_blocks must be >= 0");
    const int grid = t.rp_blocks > 0 ? std::min(t.rp_blocks, rp_grid_full) : rp_grid_full;
    if (t.fdtd_rows != strip_rows || grid != rp_grid) drop_graphs();
    strip_rows = t.fdtd_rows;
    rp_blocks_req = t.rp_blocks;
    rp_grid = grid;
    return CRP_OK;
  }
  void get_tuning(crp_tuning* t) const {
    t->fdtd_rows = strip_rows;
    t->rp_blocks = rp_blocks_req;
    t->rp_blocks_max = rp_grid_full;
  }

  // Snapshots (crp_save_state / crp_load_state): the device pool holds every
  // device array of the handle; this is the host-side step state beside it.
  struct HostState {
    int cur_v, cur_p, fg_a, fg_b, fg_c, cur_t, bins_stale;
    double tstep, tstepx, t_prev;
    crp_stats stats;
    Box supp[3], couple_box;
    Scalars hsc;
    crp_focus_state focus;
    MinMax mm;
    size_t n_focal, n_control;
  };
  size_t state_bytes() const { return pool_bytes; }

  crp_status save_state(void* blob, std::vector<unsigned char>& host) {
    CRP_CUDA(cudaMemcpyAsync(blob, pool, pool_bytes, cudaMemcpyDeviceToDevice, stream));
    CRP_CUDA(cudaStreamSynchronize(stream));
    HostState h{};
    h.cur_v = cur_v, h.cur_p = cur_p, h.fg_a = fg_a, h.fg_b = fg_b, h.fg_c = fg_c, h.cur_t = cur_t;
    h.bins_stale = bins_stale ? 1 : 0;
    h.tstep = tstep, h.tstepx = tstepx, h.t_prev = t_prev;
    h.stats = stats;
    for (int q = 0; q < 3; q++) h.supp[q] = supp[q];
    h.couple_box = couple_box;
    h.hsc = *h_scalars;
    h.focus = focus;
    h.mm = mm;
    h.n_focal = focal_hist.size();
    h.n_control = control_hist.size();
    host.resize(sizeof(HostState) + sizeof(double) * (h.n_focal + h.n_control));
    std::memcpy(host.data(), &h, sizeof(HostState));
    if (h.n_focal) std::memcpy(host.data() + sizeof(HostState), focal_hist.data(), sizeof(double) * h.n_focal);
    if (h.n_control)
      std::memcpy(host.data() + sizeof(HostState) + sizeof(double) * h.n_focal, control_hist.data(),
                  sizeof(double) * h.n_control);
    return CRP_OK;
  }

  crp_status load_state(const void* blob, const std::vector<unsigned char>& host) {
    HostState h{};
    if (host.size() < sizeof(HostState)) return fail(CRP_ERR_INVALID, "state: no host part");
    std::memcpy(&h, host.data(), sizeof(HostState));
    if (host.size() != sizeof(HostState) + sizeof(double) * (h.n_focal + h.n_control))
      return fail(CRP_ERR_INVALID, "state: host part of the wrong size");
    CRP_CUDA(cudaMemcpyAsync(pool, blob, pool_bytes, cudaMemcpyDeviceToDevice, stream));
    CRP_CUDA(cudaStreamSynchronize(stream));
    cur_v = h.cur_v, cur_p = h.cur_p, fg_a = h.fg_a, fg_b = h.fg_b, fg_c = h.fg_c, cur_t = h.cur_t;
    bins_stale = h.bins_stale != 0;
    tstep = h.tstep, tstepx = h.tstepx, t_prev = h.t_prev;
    // The simulation's state returns; the counters of work done do not.
    const crp_stats keep = stats;
    stats = h.stats;
    stats.kernel_launches = keep.kernel_launches;
    stats.fdtd_launches = keep.fdtd_launches;
    stats.rp_launches = keep.rp_launches;
    stats.couple_launches = keep.couple_launches;
    stats.ms_fdtd = keep.ms_fdtd, stats.ms_rp = keep.ms_rp, stats.ms_couple = keep.ms_couple;
    stats.ms_other = keep.ms_other;
    for (int q = 0; q < 3; q++) supp[q] = h.supp[q];
    couple_box = h.couple_box;
    *h_scalars = h.hsc;
    focus = h.focus;
    mm = h.mm;
    const double* hist = reinterpret_cast<const double*>(host.data() + sizeof(HostState));
    focal_hist.assign(hist, hist + h.n_focal);
    control_hist.assign(hist + h.n_focal, hist + h.n_focal + h.n_control);
    return CRP_OK;
  }

  // crp_adjoint's device workspace: kept for the next call (an optimisation
  // loop calls it over and over) and released with the simulation, so that a
  // call neither waits for a device-wide free nor pays for a new allocation.
  void* adj_ws = nullptr;
  size_t adj_ws_bytes = 0;
  crp_status adjoint_workspace(size_t bytes, void** out) {
    if (adj_ws_bytes < bytes) {
      if (adj_ws) {
        CRP_CUDA(cudaStreamSynchronize(stream));
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
    *out = adj_ws;
    return CRP_OK;
  }

  ~Sim() {
    drop_graphs();
    if (adj_ws) cudaFree(adj_ws);
    if (cap_stream) cudaStreamDestroy(cap_stream);
    if (h_push) cudaFreeHost(h_push);
    if (pool) cudaFree(pool);
    if (h_scalars) cudaFreeHost(h_scalars);
    if (ev_scalars) cudaEventDestroy(ev_scalars);
    if (ev_block) cudaEventDestroy(ev_block);
    if (h_focal) cudaFreeHost(h_focal);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }
};

// Contributions for the initial radii: the RP kernel's tail without the solve.
__global__ void bubble_contrib(const __grid_constant__ GridParams g, const __grid_constant__ BubbleParams bp,
                               BubbleArrays b) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= b.n) return;
  const double x = b.x[n], y = b.y[n];
  const int inx = b.ibnx[n], iny = b.ibny[n];
  double dxw[2], dyw[2];
  const double cx0 = delta_cos_x(bp, g, inx, x), cy0 = delta_cos_y(bp, g, iny, y);
  for (int q = 0; q < 2; q++) {
    dxw[q] = delta_w(bp, cx0, q);
    dyw[q] = delta_w(bp, cy0, q);
  }
  const double Rt = b.R_t[n];
  const double vol = g.cyl ? bp.pi4r3 * b.n_B[n] * (Rt * Rt * Rt) * g.rdx * g.rdy / x
                           : bp.pi4r3 * b.n_B[n] * (Rt * Rt * Rt) * g.rdx * g.rdy;
  const int p = b.pos[n];
  if (p < 0) return;
  double* c = b.contrib + 4 * (long)p;
  c[0] = vol * dxw[0] * dyw[0];
  c[1] = vol * dxw[0] * dyw[1];
  c[2] = vol * dxw[1] * dyw[0];
  c[3] = vol * dxw[1] * dyw[1];
}

// Gather-only variant of couple_press for the initial void fraction.
template <typename P>
__global__ void __launch_bounds__(256) couple_fg_only(const __grid_constant__ GridParams g, const CoupleArgs<P> a) {
  const Frame& f = g.f;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i > f.X + 1 || j > f.Y + 1) return;
  a.fg.put(f.idx(i, j), gather_fg(f, a.start, a.contrib, i, j, g.cyl && i <= 1));
}

cudaError_t Sim::launch_contrib_only() {
  return launch(kClassOther, [&] { bubble_contrib<<<(bub.n + 255) / 256, 256, 0, stream>>>(gp, bp, bub); });
}

template <>
F64 Sim::view<F64>(void* b) const {
  return F64{(double*)b};
}
template <>
F32c Sim::view<F32c>(void* b) const {
  return F32c{(float2*)b};
}
template <>
F32 Sim::view<F32>(void* b) const {
  return F32{(float*)b};
}

template <typename P>
cudaError_t Sim::launch_couple_t(bool pressure) {
  using V = typename P::V;
  using S = typename P::S;
  using G = typename P::G;
  CoupleArgs<P> ca;
  ca.vx = view<V>(vx[cur_v]);
  ca.vy = view<V>(vy[cur_v]);
  ca.pnx = view<S>(px[cur_p ^ 1]);
  ca.pny = view<S>(py[cur_p ^ 1]);
  ca.px = view<S>(px[cur_p]);
  ca.py = view<S>(py[cur_p]);
  ca.fg = view<G>(fg[fg_a]);
  ca.fgn = view<G>(fg[fg_b]);
  ca.start = bins.start;
  ca.idx = bins.idx;
  ca.contrib = bub.contrib;
  ca.dbox = nullptr;
  ca.residual = d_residual;
  dim3 blk(32, 8);
  if (pressure && capturing) {
    // Graph step: the box is decided on the device each step.
    ca.i0 = ca.j0 = 0;
    ca.i1 = gp.f.X + 1;
    ca.j1 = gp.f.Y + 1;
    ca.dbox = d_scalars->box;
    return launch(kClassCouple, [&] { couple_press<P><<<couple_graph_grid, blk, 0, stream>>>(gp, ca); });
  }
  if (pressure) {
    const Box& b = couple_box;
    if (box_empty(b)) return cudaSuccess;
    ca.i0 = b.i0;
    ca.j0 = b.j0;
    ca.i1 = b.i1;
    ca.j1 = b.j1;
    dim3 grd((b.i1 - b.i0 + 1 + kCoupleW - 1) / kCoupleW, (b.j1 - b.j0 + 1 + 7) / 8);
    return launch(kClassCouple, [&] { couple_press<P><<<grd, blk, 0, stream>>>(gp, ca); });
  }
  dim3 grd((gp.f.X + 2 + 31) / 32, (gp.f.Y + 2 + 7) / 8);
  return launch(kClassOther, [&] { couple_fg_only<P><<<grd, blk, 0, stream>>>(gp, ca); });
}

// crp_adjoint: obj->steps forward steps recording the focal p0, the
// objective, then the reverse sweep (adj_force for the last step, one adj_step
// per step, adjoint.cuh) and the per-element sums of the per-column gradients.
crp_status Sim::adjoint(const crp_objective* obj, double* J, double* grad_amp, double* grad_phase) {
  if (!obj || obj->steps <= 0 || !(obj->focal_radius > 0.0))
    return fail(CRP_ERR_INVALID, "adjoint: steps > 0 and focal_radius > 0 are required");
  if ((grad_amp || grad_phase) && gp.elem_n == 0)
    return fail(CRP_ERR_INVALID, "adjoint: gradients need ext.elements > 0");
  // The temperature branch, when on, is driven by the pressure and does not act
  // back on it: the forward steps advance it, the objective does not see it.
  if (hs.nb > 0 || src_velocity(gp) || !src_pressure(gp))
    return fail(CRP_ERR_UNSUPPORTED, "adjoint: bubbles off and a pressure source only");
  const Frame& f = gp.f;
  const int X = f.X, Y = f.Y, N = obj->steps;
  // Focal box: cell centres within focal_radius of the focus.
  const double cx = gp.ctl_x, cy = gp.ctl_y, r = obj->focal_radius;
  int bi0 = X + 1, bi1 = 0, bj0 = Y + 1, bj1 = 0;
  for (int i = 1; i <= X; i++)
    if (std::fabs(((double)i - 0.5) * gp.dx - cx) <= r) bi0 = std::min(bi0, i), bi1 = std::max(bi1, i);
  for (int j = 1; j <= Y; j++)
    if (std::fabs(((double)j - 0.5) * gp.dy - cy) <= r) bj0 = std::min(bj0, j), bj1 = std::max(bj1, j);
  const int bw = std::max(bi1 - bi0 + 1, 1), bh = std::max(bj1 - bj0 + 1, 1);
  if (bi1 < bi0 || bj1 < bj0) bi0 = bj0 = 1;  // empty: one cell of weight 0
  const size_t cells_box = (size_t)bw * bh;
  std::vector<double> w(cells_box, 0.0);
  const double pi = std::acos(-1.0);
  for (int jj = 0; jj < bh; jj++)
    for (int ii = 0; ii < bw; ii++) {
      const int i = bi0 + ii, j = bj0 + jj;
      if (i > bi1 || j > bj1 || (gp.source_row > 0 && j == gp.source_row)) continue;
      const double xm = ((double)i - 0.5) * gp.dx, ym = ((double)j - 0.5) * gp.dy;
      if ((xm - cx) * (xm - cx) + (ym - cy) * (ym - cy) > r * r) continue;
      w[(size_t)jj * bw + ii] = gp.cyl ? 2.0 * pi * xm * gp.dx * gp.dy : gp.dx * gp.dy;
    }
  // Device buffers: two sets of four adjoint frames, two per-column
  // gradients, weights, the focal history and the per-step objective.
  const size_t hist_n = (size_t)N * cells_box;
  if (hist_n * sizeof(double) > ((size_t)32 << 30))
    return fail(CRP_ERR_TOO_LARGE, "adjoint: focal history above 32 GiB (steps x focal cells)");
  const size_t n_doubles = 8 * cells + 2 * (size_t)(X + 2) + cells_box + hist_n + (size_t)N;
  double* buf = nullptr;
  {
    const crp_status ws = adjoint_workspace(n_doubles * sizeof(double), reinterpret_cast<void**>(&buf));
    if (ws != CRP_OK) return ws;
  }
  struct Drain {  // on every return: the queued work has finished
    cudaStream_t st;
    ~Drain() { cudaStreamSynchronize(st); }
  } guard{stream};
  AdjFrames fr[2];
  for (int s = 0; s < 2; s++) {
    double* base = buf + (size_t)s * 4 * cells;
    fr[s] = AdjFrames{base, base + cells, base + 2 * cells, base + 3 * cells};
  }
  AdjGrad gr;
  gr.gA = buf + 8 * cells;
  gr.gP = gr.gA + (X + 2);
  double* d_w = gr.gP + (X + 2);
  double* hist = d_w + cells_box;
  double* d_Jn = hist + hist_n;
  CRP_CUDA(cudaMemsetAsync(buf, 0, n_doubles * sizeof(double), stream));
  CRP_CUDA(cudaMemcpyAsync(d_w, w.data(), sizeof(double) * cells_box, cudaMemcpyHostToDevice, stream));
  const FocalBox box{bi0, bj0, bw, bh, d_w};
  const int rb = (int)((cells_box + 255) / 256);
  // Forward, recording the focal p0 after every step.
  std::vector<double> times((size_t)N + 1);
  times[0] = tstep;
  bool queued = false;  // steps queued by queue_plain, checked by finish_plain
  for (int n = 1; n <= N; n++) {
    const bool plain = plain_ok();
    const crp_status st = plain ? queue_plain() : step_once();
    if (st != CRP_OK) return st;
    queued = queued || plain;
    double* out = hist + (size_t)(n - 1) * cells_box;
    cudaError_t e;
    if (mixed) {
      const F32c a = view<F32c>(px[cur_p]), b = view<F32c>(py[cur_p]);
      e = launch(kClassOther, [&] { adj_record<F32c><<<rb, 256, 0, stream>>>(gp, a, b, box, out); });
    } else {
      const F64 a = view<F64>(px[cur_p]), b = view<F64>(py[cur_p]);
      e = launch(kClassOther, [&] { adj_record<F64><<<rb, 256, 0, stream>>>(gp, a, b, box, out); });
    }
    CRP_CUDA(e);
    times[n] = tstep;
  }
  if (queued) {
    const crp_status st = finish_plain();
    if (st != CRP_OK) return st;
  }
  // Objective.
  CRP_CUDA(launch(kClassOther, [&] { adj_objective<<<N, kAdjSumThreads, 0, stream>>>(box, hist, d_Jn); }));
  std::vector<double> Jn(N);
  CRP_CUDA(cudaMemcpyAsync(Jn.data(), d_Jn, sizeof(double) * N, cudaMemcpyDeviceToHost, stream));
  CRP_CUDA(cudaStreamSynchronize(stream));
  double Jsum = 0.0;
  for (int n = 0; n < N; n++) Jsum += Jn[n];
  if (J) *J = gp.dt * Jsum;
  // Reverse sweep: reverse step n reads frame set s and writes set s ^ 1.
  const dim3 blk(32, 8), gcells((X + 31) / 32, (Y + 7) / 8);
  CRP_CUDA(launch(kClassOther, [&] { adj_force<<<rb, 256, 0, stream>>>(gp, fr[0], box, hist + (size_t)(N - 1) * cells_box); }));
  int s = 0;
  for (int n = N; n >= 1; n--, s ^= 1) {
    const double t_src = times[n - 1];
    const double* p0 = n >= 2 ? hist + (size_t)(n - 2) * cells_box : nullptr;
    CRP_CUDA(launch(kClassOther,
                    [&] { adj_step<<<gcells, blk, 0, stream>>>(gp, fr[s], fr[s ^ 1], gr, t_src, box, p0); }));
  }
  if (gp.elem_n > 0) {
    std::vector<double> gA(X + 2), gPh(X + 2);
    CRP_CUDA(cudaMemcpyAsync(gA.data(), gr.gA, sizeof(double) * (X + 2), cudaMemcpyDeviceToHost, stream));
    CRP_CUDA(cudaMemcpyAsync(gPh.data(), gr.gP, sizeof(double) * (X + 2), cudaMemcpyDeviceToHost, stream));
    CRP_CUDA(cudaStreamSynchronize(stream));
    const int ne = gp.elem_n;
    std::vector<double> sa(ne, 0.0), sp(ne, 0.0);
    for (int i = 1; i <= X; i++) {
      const double xm = ((double)i - 0.5) * gp.dx;
      int e = (int)(std::fabs(xm - gp.ctl_x) * (double)ne / gp.elem_rap);
      if (e >= ne) e = ne - 1;
      sa[e] += gA[i];
      sp[e] += gPh[i];
    }
    if (grad_amp) std::copy(sa.begin(), sa.end(), grad_amp);
    if (grad_phase) std::copy(sp.begin(), sp.end(), grad_phase);
  } else {
    CRP_CUDA(cudaStreamSynchronize(stream));
  }
  return CRP_OK;
}

cudaError_t Sim::launch_couple(bool pressure) {
  return mixed ? launch_couple_t<PrecMixed>(pressure) : launch_couple_t<PrecFP64>(pressure);
}

}  // namespace crp

// ---------------------------------------------------------------------------
// A snapshot (crp_save_state): the device pool's copy and the host-side state.
struct crp_state {
  int device = 0;
  int dims = 2;
  size_t bytes = 0;
  void* blob = nullptr;
  std::vector<unsigned char> host;
};

struct crp_sim {
  crp::Sim s;
  crp::Sim3Impl* s3 = nullptr;  // a 3-D grid (ext.grid_z > 0) runs here instead of s
  std::string err3;
  ~crp_sim() {
    if (s3) crp::sim3_destroy(s3);
  }
  int device() const { return s3 ? crp::sim3_device(s3) : s.device; }
};

namespace crp {
const char* noalloc_last_error();
}

namespace {
// Makes a simulation's device current for the duration of an entry point and
// restores the caller's device afterwards: the handle may be driven from any
// host thread, whose current device need not be the one it was created on.
class DeviceScope {
 public:
  explicit DeviceScope(const crp_sim* h) {
    if (cudaGetDevice(&prev_) != cudaSuccess) prev_ = -1;
    if (h && prev_ != h->device()) {
      ok_ = cudaSetDevice(h->device()) == cudaSuccess;
      switched_ = ok_;
    }
  }
  ~DeviceScope() {
    if (switched_ && prev_ >= 0) cudaSetDevice(prev_);
  }
  bool ok() const { return ok_; }

 private:
  int prev_ = -1;
  bool ok_ = true;
  bool switched_ = false;
};
}  // namespace

extern "C" {

crp_status crp_create(const crp_config* cfg, const crp_bubbles_in* bubbles, void* stream, crp_sim** out) {
  if (!cfg || !out) return CRP_ERR_INVALID;
  *out = nullptr;
  crp_sim* h = new (std::nothrow) crp_sim();
  if (!h) return CRP_ERR_ALLOC;
  if (cfg->ext_grid_z > 0) {
    const crp_status st3 = crp::sim3_create(cfg, bubbles, stream, &h->s3, &h->err3);
    if (st3 != CRP_OK) {
      fprintf(stderr, "crp_create: %s\n", h->err3.c_str());
      delete h;
      return st3;
    }
    *out = h;
    return CRP_OK;
  }
  crp_status st = h->s.create(*cfg, bubbles, stream);
  if (st != CRP_OK) {
    fprintf(stderr, "crp_create: %s\n", h->s.err.c_str());
    delete h;
    return st;
  }
  *out = h;
  return CRP_OK;
}

crp_status crp_step(crp_sim* h, int32_t n) {
  if (!h || n < 0) return CRP_ERR_INVALID;
  DeviceScope dev(h);
  if (!dev.ok()) return CRP_ERR_CUDA;
  if (h->s3) return crp::sim3_step(h->s3, n);
  return h->s.step_n(n);
}

crp_status crp_get_dims3(const crp_sim* h, crp_dims3* d) {
  if (!h || !d || !h->s3) return CRP_ERR_INVALID;
  crp::sim3_dims(h->s3, d);
  return CRP_OK;
}

crp_status crp_get_dims(const crp_sim* h, crp_dims* d) {
  if (!h || !d) return CRP_ERR_INVALID;
  if (h->s3) {
    crp_dims3 d3;
    crp::sim3_dims(h->s3, &d3);
    *d = crp_dims{d3.nx, d3.ny, d3.nx, d3.ny, d3.nx + 1, d3.ny + 1, d3.num_bubbles, d3.dx, d3.dy, d3.dt};
    return CRP_OK;
  }
  const crp::Frame& f = h->s.gp.f;
  d->i1m = f.X + 2;
  d->j1m = f.Y + 2;
  d->i2m = f.X + 2;
  d->j2m = f.Y + 2;
  d->i2n = f.X + 3;
  d->j2n = f.Y + 3;
  d->num_bubbles = h->s.bub.n;
  d->dx = h->s.gp.dx;
  d->dy = h->s.gp.dy;
  d->dt = h->s.gp.dt;
  return CRP_OK;
}

crp_status crp_get_stats(const crp_sim* h, crp_stats* st) {
  if (!h || !st) return CRP_ERR_INVALID;
  if (h->s3) {
    *st = crp::sim3_stats(h->s3);
    return CRP_OK;
  }
  *st = h->s.stats;
  return CRP_OK;
}

crp_status crp_set_profiling(crp_sim* h, int32_t enable) {
  if (!h) return CRP_ERR_INVALID;
  if (h->s3) return crp::sim3_set_profiling(h->s3, enable);
  DeviceScope dev(h);
  if (!dev.ok()) return CRP_ERR_CUDA;
  if (cudaStreamSynchronize(h->s.stream) != cudaSuccess) return CRP_ERR_CUDA;
  h->s.prof.resolve();
  h->s.prof.on = enable != 0;
  h->s.fill_launch_stats();
  return CRP_OK;
}

crp_status crp_read_field(crp_sim* h, crp_field f, double* host) {
  if (!h || !host) return CRP_ERR_INVALID;
  DeviceScope dev(h);
  if (!dev.ok()) return CRP_ERR_CUDA;
  if (h->s3) return crp::sim3_read_field(h->s3, f, host);
  return h->s.read_field(f, host);
}

crp_status crp_read_bubbles(crp_sim* h, crp_bubble_field w, double* host) {
  if (!h || !host) return CRP_ERR_INVALID;
  DeviceScope dev(h);
  if (!dev.ok()) return CRP_ERR_CUDA;
  if (h->s3) return crp::sim3_read_bubbles(h->s3, w, host);
  return h->s.read_bubbles(w, host);
}

int64_t crp_focus_history(const crp_sim* h, int32_t which, double* out, int64_t capacity) {
  if (!h || (which != 0 && which != 1)) return -1;
  const std::vector<double>& v = which == 0 ? h->s.focal_hist : h->s.control_hist;
  if (!h->s.temperature_on) return 0;
  for (int64_t k = 0; out && k < capacity && k < (int64_t)v.size(); k++) out[k] = v[k];
  return (int64_t)v.size();
}

crp_status crp_get_focus_state(const crp_sim* h, crp_focus_state* st) {
  if (!h || !st) return CRP_ERR_INVALID;
  *st = h->s.focus;
  return CRP_OK;
}

crp_status crp_set_focus_state(crp_sim* h, const crp_focus_state* st) {
  if (!h || !st) return CRP_ERR_INVALID;
  DeviceScope dev(h);
  if (!dev.ok()) return CRP_ERR_CUDA;
  if (h->s.stats.steps != 0) return CRP_ERR_INVALID;
  h->s.focus = *st;
  if (h->s.cfg.tr_pid) {
    // A carried-over control point replaces the initial one (pid_init).
    h->s.set_control(st->control_x, st->control_y);
    h->s.control_hist.assign(1, st->control_y);
  }
  return CRP_OK;
}

crp_status crp_set_source_elements(crp_sim* h, int32_t n, const double* amp, const double* phase) {
  if (!h) return CRP_ERR_INVALID;
  DeviceScope dev(h);
  if (!dev.ok()) return CRP_ERR_CUDA;
  if (h->s3) return crp::sim3_set_elements(h->s3, n, amp, phase);
  return h->s.set_source_elements(n, amp, phase);
}

crp_status crp_adjoint(crp_sim* h, const crp_objective* obj, double* J, double* grad_amp, double* grad_phase) {
  if (!h) return CRP_ERR_INVALID;
  DeviceScope dev(h);
  if (!dev.ok()) return CRP_ERR_CUDA;
  if (h->s3) return crp::sim3_adjoint(h->s3, obj, J, grad_amp, grad_phase);
  return h->s.adjoint(obj, J, grad_amp, grad_phase);
}

crp_status crp_minmax_T(const crp_sim* h, double* T_min, double* T_max) {
  if (!h || !T_min || !T_max) return CRP_ERR_INVALID;
  *T_min = h->s.mm.T_min;
  *T_max = h->s.mm.T_max;
  return CRP_OK;
}

crp_status crp_minmax(const crp_sim* h, double* fg_min, double* fg_max, double* p0_min, double* p0_max) {
  if (!h || !fg_min || !fg_max || !p0_min || !p0_max) return CRP_ERR_INVALID;
  *fg_min = h->s.mm.fg_min;
  *fg_max = h->s.mm.fg_max;
  *p0_min = h->s.mm.p0_min;
  *p0_max = h->s.mm.p0_max;
  return CRP_OK;
}

void* crp_stream(crp_sim* h) { return h ? (h->s3 ? crp::sim3_stream(h->s3) : (void*)h->s.stream) : nullptr; }

const char* crp_last_error(const crp_sim* h) {
  if (!h) return crp::noalloc_last_error();
  return h->s3 ? crp::sim3_error(h->s3) : h->s.err.c_str();
}

void crp_destroy(crp_sim* h) {
  if (!h) return;
  DeviceScope dev(h);
  delete h;
}

crp_status crp_write_rawdata(crp_sim* h, const char* dir) {
  if (!h || !dir) return CRP_ERR_INVALID;
  if (h->s3) return CRP_ERR_UNSUPPORTED;
  DeviceScope dev(h);
  if (!dev.ok()) return CRP_ERR_CUDA;
  return crp::write_rawdata(h, dir);
}

crp_status crp_write_sph(crp_sim* h, const char* dir) {
  if (!h || !dir) return CRP_ERR_INVALID;
  if (h->s3) return CRP_ERR_UNSUPPORTED;
  DeviceScope dev(h);
  if (!dev.ok()) return CRP_ERR_CUDA;
  return crp::write_sph(h, dir);
}

size_t crp_state_bytes(const crp_sim* h) {
  if (!h) return 0;
  return h->s3 ? crp::sim3_state_bytes(h->s3) : h->s.state_bytes();
}

crp_status crp_save_state(crp_sim* h, crp_state** out) {
  if (!h || !out) return CRP_ERR_INVALID;
  DeviceScope dev(h);
  if (!dev.ok()) return CRP_ERR_CUDA;
  const size_t bytes = crp_state_bytes(h);
  const int dims = h->s3 ? 3 : 2;
  crp_state* st = *out;
  if (st && (st->bytes != bytes || st->dims != dims || st->device != h->device())) return CRP_ERR_INVALID;
  if (!st) {
    st = new (std::nothrow) crp_state();
    if (!st) return CRP_ERR_ALLOC;
    st->bytes = bytes;
    st->dims = dims;
    st->device = h->device();
    if (cudaMalloc(&st->blob, bytes) != cudaSuccess) {
      cudaGetLastError();
      delete st;
      return CRP_ERR_ALLOC;
    }
  }
  const crp_status r =
      h->s3 ? crp::sim3_save_state(h->s3, st->blob, st->host) : h->s.save_state(st->blob, st->host);
  if (r != CRP_OK) {
    if (!*out) crp_state_free(st);
    return r;
  }
  *out = st;
  return CRP_OK;
}

crp_status crp_load_state(crp_sim* h, const crp_state* st) {
  if (!h || !st) return CRP_ERR_INVALID;
  if (st->bytes != crp_state_bytes(h) || st->dims != (h->s3 ? 3 : 2) || st->device != h->device())
    return CRP_ERR_INVALID;
  DeviceScope dev(h);
  if (!dev.ok()) return CRP_ERR_CUDA;
  return h->s3 ? crp::sim3_load_state(h->s3, st->blob, st->host) : h->s.load_state(st->blob, st->host);
}

void crp_state_free(crp_state* st) {
  if (!st) return;
  int prev = 0;
  const bool have = cudaGetDevice(&prev) == cudaSuccess;
  if (cudaSetDevice(st->device) == cudaSuccess && st->blob) cudaFree(st->blob);
  if (have) cudaSetDevice(prev);
  delete st;
}

crp_status crp_get_tuning(const crp_sim* h, crp_tuning* t) {
  if (!h || !t) return CRP_ERR_INVALID;
  if (h->s3)
    crp::sim3_get_tuning(h->s3, t);
  else
    h->s.get_tuning(t);
  return CRP_OK;
}

crp_status crp_set_tuning(crp_sim* h, const crp_tuning* t) {
  if (!h || !t) return CRP_ERR_INVALID;
  DeviceScope dev(h);
  if (!dev.ok()) return CRP_ERR_CUDA;
  return h->s3 ? crp::sim3_set_tuning(h->s3, t) : h->s.set_tuning(*t);
}

}  // extern "C"

namespace crp {
// Accessors used by the rawdata writer (rawdata.cpp).
crp_status sim_read_field(crp_sim* h, crp_field f, double* host) { return h->s.read_field(f, host); }
crp_status sim_read_bubbles(crp_sim* h, crp_bubble_field w, double* host) { return h->s.read_bubbles(w, host); }
const crp_config& sim_config(const crp_sim* h) { return h->s.cfg; }
int64_t sim_step_count(const crp_sim* h) { return h->s3 ? sim3_stats(h->s3).steps : h->s.stats.steps; }

// Graph-queued steps for crp_batch (batch.cpp).
bool sim_graph_ready(const crp_sim* h) { return !h->s3 && h->s.graph_ready(); }
void sim_allow_graphs(crp_sim* h, bool on) {
  if (!h->s3) h->s.graphs_on = on;
}
crp_status sim_blocking_waits(crp_sim* h, bool on) {
  if (h->s3) return CRP_OK;
  DeviceScope dev(h);
  if (!dev.ok()) return CRP_ERR_CUDA;
  return h->s.set_blocking_waits(on);
}
crp_status sim_graphs_enqueue(crp_sim* h, int n) {
  DeviceScope dev(h);
  if (!dev.ok()) return CRP_ERR_CUDA;
  return h->s.graphs_enqueue(n);
}
crp_status sim_graphs_finish(crp_sim* h) {
  DeviceScope dev(h);
  if (!dev.ok()) return CRP_ERR_CUDA;
  return h->s.graphs_finish();
}
double sim_time(const crp_sim* h) { return h->s.tstep; }
MinMax& sim_minmax(crp_sim* h) { return h->s.mm; }
}  // namespace crp
