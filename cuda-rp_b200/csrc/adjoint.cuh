// Discrete adjoint of the FDTD/PML step without bubbles (crp_adjoint).
//
// Without bubbles the step is linear in the fields (f_g = 0, rho_m = rho_inf):
//   faces       v'(f) = (v(f) A(f) - q (p0(f+1) - p0(f)) rdx) B(f)     (zeroed walls excepted)
//   components  px'(c) = px(c) a(c) - s3p b(c) (k_e(c) vx'(c) - k_w(c) vx'(c-1)),  py' likewise
//   p0          p0 = px + py inside, 0 on PML ghost cells, the source value on
//               the source row, the mirror of row 1 on the y0 ghost row
// with the factors of velocity_face_q / pressure_component (A, a = 1 - s;
// B, b = 1 / (1 + s); q = dt / rho_inf).  One reverse step applies the
// transposes in the opposite order: the pressure update's transpose takes the
// face adjoints L to Lt, then the velocity update's and p0's transposes take
// Lt and the component adjoints M one step back, and the source's share of the
// p0 adjoint times the source's derivatives with respect to the element
// amplitudes and phases goes into per-column gradient sums.  The objective
// sum_n dt sum_focal w p0^2 adds 2 dt w p0^n to both component adjoints at
// every step, from the focal pressures the forward recorded (adj_record).
//
// adj_step does all of one reverse step in one pass: each cell forms the Lt
// of the four faces it reads (its east and north faces, and its west and south
// faces, which its neighbours form too, by the same expression) from the
// previous step's L and M, and writes the next step's L and M into the other
// of two frame sets.  Per cell and step it reads 4 doubles (L_x, L_y, M_x, M_y;
// the neighbours' values come through L1/L2) and writes 4: 64 bytes.
#pragma once
#include "crp_device.cuh"

namespace crp {

// One set of adjoint fields (two alternate over the reverse sweep).
struct AdjFrames {
  double* LX;  // adjoint of the x faces
  double* LY;  // adjoint of the y faces
  double* MX;  // adjoint of px
  double* MY;  // adjoint of py
};
// Per column: d J / d (its element's amplitude factor), d J / d (its phase offset).
struct AdjGrad {
  double* gA;
  double* gP;
};

// Faces the forward updates (the others are set to zero): the x0 axis and the
// x1 and y1 walls without a PML.  The y0 face without a PML keeps its update
// when the source is a pressure source, the only kind supported here.
__device__ __forceinline__ bool adj_xface_on(const GridParams& g, int f) {
  return !((f == 0 && !g.pml_x0) || (f == g.f.X && !g.pml_x1));
}
__device__ __forceinline__ bool adj_yface_on(const GridParams& g, int f) { return !(f == g.f.Y && !g.pml_y1); }
// d v'(f) / d p0(f) of a face (-d v'(f) / d p0(f+1)), and d v'(f) / d v(f).
__device__ __forceinline__ double adj_cx(const GridParams& g, int f) { return g.dt_rho * g.rdx * g.vbx[f + 1]; }
__device__ __forceinline__ double adj_cy(const GridParams& g, int f) { return g.dt_rho * g.rdx * g.vby[f + 1]; }
__device__ __forceinline__ double adj_ax(const GridParams& g, int f) { return g.vax[f + 1] * g.vbx[f + 1]; }
__device__ __forceinline__ double adj_ay(const GridParams& g, int f) { return g.vay[f + 1] * g.vby[f + 1]; }
// Weights of the east and west faces in the x divergence of cell c.
__device__ __forceinline__ double adj_kx_east(const GridParams& g, int c) {
  return g.cyl ? g.xu[c + 1] * g.rdx * g.rxp[c] : g.rdx;
}
__device__ __forceinline__ double adj_kx_west(const GridParams& g, int c) {
  return g.cyl ? g.xu[c] * g.rdx * g.rxp[c] : g.rdx;
}

// Transpose of the pressure update at one face: Lt = L + (d p' / d v')^T M.
// x face i (0 <= i <= X) of row j (1 <= j <= Y): east face of cell i, west
// face of cell i+1.
__device__ __forceinline__ double adj_lxt(const GridParams& g, const AdjFrames& a, int i, int j) {
  const Frame& f = g.f;
  double v = a.LX[f.idx(i, j)];
  if (i >= 1) v -= g.s3p * g.pbx[i] * adj_kx_east(g, i) * a.MX[f.idx(i, j)];
  if (i + 1 <= f.X) v += g.s3p * g.pbx[i + 1] * adj_kx_west(g, i + 1) * a.MX[f.idx(i + 1, j)];
  return v;
}
// y face j (0 <= j <= Y) of column i (1 <= i <= X): north face of row j,
// south face of row j+1.
__device__ __forceinline__ double adj_lyt(const GridParams& g, const AdjFrames& a, int i, int j) {
  const Frame& f = g.f;
  double v = a.LY[f.idx(i, j)];
  if (j >= 1) v -= g.s3p * g.pby[j] * g.rdy * a.MY[f.idx(i, j)];
  if (j + 1 <= f.Y) v += g.s3p * g.pby[j + 1] * g.rdy * a.MY[f.idx(i, j + 1)];
  return v;
}

// Gradient share of one source value: L (its adjoint) times its derivatives.
__device__ __forceinline__ void adj_source_grad(const GridParams& g, const AdjGrad& gr, int i, double ym,
                                                double t_src, double L) {
  if (g.elem_n == 0) return;  // no elements: J only
  double dA, dP;
  source_derivatives(g, ((double)i - 0.5) * g.dx, ym, t_src, dA, dP);
  gr.gA[i] += L * dA;
  gr.gP[i] += L * dP;
}

// Focal box: cells [bi0, bi0 + bw) x [bj0, bj0 + bh), weights w (0 outside
// the focal disk and on the source row).
struct FocalBox {
  int bi0, bj0, bw, bh;
  const double* w;
};

// One reverse step: the transposes of the pressure update, the velocity update
// and p0, from `in` into `out`; t_src is the time of the source values that
// step read.  p0 (the focal pressures of the step before, or null for the
// first step) adds that step's objective term.  Threads over the cells
// [1, X] x [1, Y]; the cells of column 1 and row 1 also write the x0 and y0
// face adjoints.
__global__ void adj_step(const __grid_constant__ GridParams g, const AdjFrames in, const AdjFrames out,
                         const AdjGrad gr, double t_src, const FocalBox b, const double* __restrict__ p0) {
  const Frame& f = g.f;
  const int X = f.X, Y = f.Y;
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x, j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i > X || j > Y) return;
  const long k = f.idx(i, j);
  const double xe = adj_lxt(g, in, i, j), xw = adj_lxt(g, in, i - 1, j);
  const double yn = adj_lyt(g, in, i, j), ys = adj_lyt(g, in, i, j - 1);
  // Adjoint of p0(i, j): the faces that read it.
  double L0 = 0.0;
  if (adj_xface_on(g, i)) L0 += adj_cx(g, i) * xe;
  if (adj_xface_on(g, i - 1)) L0 -= adj_cx(g, i - 1) * xw;
  if (adj_yface_on(g, j)) L0 += adj_cy(g, j) * yn;
  if (adj_yface_on(g, j - 1)) L0 -= adj_cy(g, j - 1) * ys;
  if (j == 1 && !g.pml_y0) {
    // The y0 face also reads the ghost value p0(i, 0): the source on the ghost
    // row (source_row 0), else the mirror of p0(i, 1).
    const double m = adj_cy(g, 0) * ys;
    if (g.source_row == 0)
      adj_source_grad(g, gr, i, -0.5 * g.dy, t_src, m);
    else
      L0 += m;
  }
  double mx = in.MX[k], my = in.MY[k];
  if (g.source_row > 0 && j == g.source_row) {
    adj_source_grad(g, gr, i, ((double)g.source_row - 0.5) * g.dy, t_src, L0);
  } else {
    mx = g.pax[i] * mx + L0;
    my = g.pay[j] * my + L0;
  }
  if (p0) {  // d J / d p0 of the step before: M += 2 dt w p0 on the focal box
    const int bi = i - b.bi0, bj = j - b.bj0;
    if (bi >= 0 && bi < b.bw && bj >= 0 && bj < b.bh) {
      const int q = bj * b.bw + bi;
      const double v = 2.0 * g.dt * b.w[q] * p0[q];
      mx += v;
      my += v;
    }
  }
  out.MX[k] = mx;
  out.MY[k] = my;
  // Face adjoints one step back (each cell takes its east and north faces; the
  // first column and row also the x0 and y0 faces).
  out.LX[k] = adj_xface_on(g, i) ? adj_ax(g, i) * xe : 0.0;
  if (i == 1) out.LX[f.idx(0, j)] = adj_xface_on(g, 0) ? adj_ax(g, 0) * xw : 0.0;
  out.LY[k] = adj_yface_on(g, j) ? adj_ay(g, j) * yn : 0.0;
  if (j == 1) out.LY[f.idx(i, 0)] = adj_ay(g, 0) * ys;
}

// p0 of the focal box after a forward step (interior cells: px + py).
template <typename S>
__global__ void adj_record(const __grid_constant__ GridParams g, const S px, const S py, const FocalBox b,
                           double* __restrict__ out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= b.bw * b.bh) return;
  const long k = g.f.idx(b.bi0 + q % b.bw, b.bj0 + q / b.bw);
  out[q] = px.get(k) + py.get(k);
}

// d J / d p0 of the last step: MX, MY += 2 dt w p0 (the earlier steps' terms
// are added by adj_step).
__global__ void adj_force(const __grid_constant__ GridParams g, const AdjFrames a, const FocalBox b,
                          const double* __restrict__ p0) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= b.bw * b.bh) return;
  const long k = g.f.idx(b.bi0 + q % b.bw, b.bj0 + q / b.bw);
  const double v = 2.0 * g.dt * b.w[q] * p0[q];
  a.MX[k] += v;
  a.MY[k] += v;
}

// sum_focal w p0^2 of every recorded step (one block per step, fixed order).
constexpr int kAdjSumThreads = 256;
__global__ void __launch_bounds__(kAdjSumThreads) adj_objective(const FocalBox b, const double* __restrict__ hist,
                                                                double* __restrict__ Jn) {
  __shared__ double sh[kAdjSumThreads];
  const int cells = b.bw * b.bh;
  const double* p = hist + (long)blockIdx.x * cells;
  double s = 0.0;
  for (int q = threadIdx.x; q < cells; q += kAdjSumThreads) s += b.w[q] * p[q] * p[q];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = kAdjSumThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) Jn[blockIdx.x] = sh[0];
}

}  // namespace crp
