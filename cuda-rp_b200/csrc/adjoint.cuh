// Discrete adjoint of the FDTD/PML step without bubbles (crp_adjoint).
//
// Without bubbles the step is linear in the fields (f_g = 0, rho_m = rho_inf):
//   faces       v'(f) = (v(f) A(f) - q (p0(f+1) - p0(f)) rdx) B(f)     (zeroed walls excepted)
//   components  px'(c) = px(c) a(c) - s3p b(c) (k_e(c) vx'(c) - k_w(c) vx'(c-1)),  py' likewise
//   p0          p0 = px + py inside, 0 on PML ghost cells, the source value on
//               the source row, the mirror of row 1 on the y0 ghost row
// with the factors of velocity_face_q / pressure_component (A, a = 1 - s;
// B, b = 1 / (1 + s); q = dt / rho_inf).  One reverse step applies the
// transposes in the opposite order: adj_faces takes the pressure update's
// transpose into the face adjoints, adj_cells the velocity update's and p0's
// into the component adjoints, and the source's share of the p0 adjoint times
// the source's derivatives with respect to the element amplitudes and phases
// into per-column gradient sums.  The objective sum_n dt sum_focal w p0^2 adds
// 2 dt w p0^n to both component adjoints at every step (adj_force), from the
// focal pressures the forward recorded (adj_record).
#pragma once
#include "crp_device.cuh"

namespace crp {

struct AdjBuffers {
  double* LX;   // adjoint of the x faces
  double* LY;   // adjoint of the y faces
  double* LXt;  // x faces after the pressure update's transpose
  double* LYt;
  double* MX;   // adjoint of px
  double* MY;   // adjoint of py
  double* gA;   // per column: d J / d (its element's amplitude factor)
  double* gP;   // per column: d J / d (its element's phase offset)
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

// Transpose of the pressure update: LXt = LX + (d px' / d vx')^T MX, and the
// same for the y faces.  Threads over the window [0, X+1] x [0, Y+1].
__global__ void adj_faces(const __grid_constant__ GridParams g, const AdjBuffers a) {
  const Frame& f = g.f;
  const int X = f.X, Y = f.Y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i > X + 1 || j > Y + 1) return;
  const long k = f.idx(i, j);
  if (i <= X && j >= 1 && j <= Y) {  // x face i of row j: east face of cell i, west face of cell i+1
    double v = a.LX[k];
    if (i >= 1) v -= g.s3p * g.pbx[i] * adj_kx_east(g, i) * a.MX[k];
    if (i + 1 <= X) v += g.s3p * g.pbx[i + 1] * adj_kx_west(g, i + 1) * a.MX[f.idx(i + 1, j)];
    a.LXt[k] = v;
  }
  if (i >= 1 && i <= X && j <= Y) {  // y face j of column i: north face of row j, south face of row j+1
    double v = a.LY[k];
    if (j >= 1) v -= g.s3p * g.pby[j] * g.rdy * a.MY[k];
    if (j + 1 <= Y) v += g.s3p * g.pby[j + 1] * g.rdy * a.MY[f.idx(i, j + 1)];
    a.LYt[k] = v;
  }
}

// Gradient share of one source value: L (its adjoint) times its derivatives.
__device__ __forceinline__ void adj_source_grad(const GridParams& g, const AdjBuffers& a, int i, double ym,
                                                double t_src, double L) {
  if (g.elem_n == 0) return;  // no elements: J only
  double dA, dP;
  source_derivatives(g, ((double)i - 0.5) * g.dx, ym, t_src, dA, dP);
  a.gA[i] += L * dA;
  a.gP[i] += L * dP;
}

// Transpose of the velocity update and of p0, one step back; t_src is the time
// of the source values that step read.  Threads over the cells [1, X] x [1, Y].
__global__ void adj_cells(const __grid_constant__ GridParams g, const AdjBuffers a, double t_src) {
  const Frame& f = g.f;
  const int X = f.X, Y = f.Y;
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x, j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i > X || j > Y) return;
  const long k = f.idx(i, j);
  // Adjoint of p0(i, j): the faces that read it.
  double L0 = 0.0;
  if (adj_xface_on(g, i)) L0 += adj_cx(g, i) * a.LXt[k];
  if (adj_xface_on(g, i - 1)) L0 -= adj_cx(g, i - 1) * a.LXt[f.idx(i - 1, j)];
  if (adj_yface_on(g, j)) L0 += adj_cy(g, j) * a.LYt[k];
  if (adj_yface_on(g, j - 1)) L0 -= adj_cy(g, j - 1) * a.LYt[f.idx(i, j - 1)];
  if (j == 1 && !g.pml_y0) {
    // The y0 face also reads the ghost value p0(i, 0): the source on the ghost
    // row (source_row 0), else the mirror of p0(i, 1).
    const double m = adj_cy(g, 0) * a.LYt[f.idx(i, 0)];
    if (g.source_row == 0)
      adj_source_grad(g, a, i, -0.5 * g.dy, t_src, m);
    else
      L0 += m;
  }
  if (g.source_row > 0 && j == g.source_row) {
    adj_source_grad(g, a, i, ((double)g.source_row - 0.5) * g.dy, t_src, L0);
  } else {
    a.MX[k] = g.pax[i] * a.MX[k] + L0;
    a.MY[k] = g.pay[j] * a.MY[k] + L0;
  }
  // Face adjoints one step back (each cell takes its east and north faces; the
  // first column and row also the x0 and y0 faces).
  a.LX[k] = adj_xface_on(g, i) ? adj_ax(g, i) * a.LXt[k] : 0.0;
  if (i == 1) {
    const long k0 = f.idx(0, j);
    a.LX[k0] = adj_xface_on(g, 0) ? adj_ax(g, 0) * a.LXt[k0] : 0.0;
  }
  a.LY[k] = adj_yface_on(g, j) ? adj_ay(g, j) * a.LYt[k] : 0.0;
  if (j == 1) {
    const long k0 = f.idx(i, 0);
    a.LY[k0] = adj_ay(g, 0) * a.LYt[k0];
  }
}

// Focal box: cells [bi0, bi0 + bw) x [bj0, bj0 + bh), weights w (0 outside
// the focal disk and on the source row).
struct FocalBox {
  int bi0, bj0, bw, bh;
  const double* w;
};

// p0 of the focal box after a forward step (interior cells: px + py).
template <typename S>
__global__ void adj_record(const __grid_constant__ GridParams g, const S px, const S py, const FocalBox b,
                           double* __restrict__ out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= b.bw * b.bh) return;
  const long k = g.f.idx(b.bi0 + q % b.bw, b.bj0 + q / b.bw);
  out[q] = px.get(k) + py.get(k);
}

// d J / d p0 of one step: MX, MY += 2 dt w p0.
__global__ void adj_force(const __grid_constant__ GridParams g, const AdjBuffers a, const FocalBox b,
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
