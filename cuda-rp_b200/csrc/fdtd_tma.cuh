// The fused FDTD pass fed by the tensor memory accelerator (TMA).
//
// Same arithmetic and output as the strip march of fdtd_strip (void-fraction
// prediction, VelocityKernel with VelocityBoundaryKernel's faces and
// MixturePressureKernel with its residual, inc/bubble_CUDA_kernel.cuh:622-867),
// with a different way of getting rows into shared memory.  A block owns
// kTmaWarps adjacent 30-column strips (120 updated columns) and a chunk of rows;
// one producer warp streams the seven input arrays of that column range into a
// ring of kTmaStages stages, each stage kTmaRows rows of all seven arrays,
// with one 2-D tensor copy (cp.async.bulk.tensor) per array and stage, and
// signals each stage on an mbarrier with the transaction's byte count.  The
// consumer warps march their strips up the chunk exactly as fdtd_strip does
// (row below in registers, neighbours by shuffle) and hand each stage back on
// a second mbarrier once its rows are read.  Many rows of every array are in
// flight per block without one load instruction per element and lane, which
// is what limited the strip march.
//
// Tensor boxes start at the frame column of logical i = 120 b - 1, so the
// innermost coordinate is a multiple of 4 elements (16 bytes for both 8- and
// 4-byte elements) and the box is 124 columns wide (992 or 496 bytes).  Rows
// and columns outside the frame are filled with zeros by the copy and are
// never stored.  Every mbarrier wait is bounded: a wait that runs out sets
// the step's pipeline error word and the block stops; the producer then
// waits, again bounded, for the copies it issued before it returns.
#pragma once
#include <cuda.h>

namespace crp {

constexpr int kTmaWarps = 4;         // consumer warps (30-column strips) per block
constexpr int kTmaBoxCols = 124;     // columns per tensor box: 30 kTmaWarps + 4
constexpr int kTmaRows = 4;          // rows per stage
constexpr int kTmaStages = 4;        // ring depth
constexpr int kTmaFields = 7;        // pnx, pny, fgA, vx_old, vy_old, fgB, fgC
constexpr unsigned kTmaWaitLimit = 1u << 22;  // polls of one mbarrier wait before it gives up

struct TmaMaps {
  CUtensorMap m[kTmaFields];
};

__host__ __device__ constexpr int tma_region_bytes(int esz) { return (kTmaBoxCols * kTmaRows * esz + 127) / 128 * 128; }

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long* b) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(b)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_tx(unsigned long long* b, unsigned bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
                   smem_u32(b)),
               "r"(bytes)
               : "memory");
}

// true once the phase of the given parity has completed; false if it did not
// within kTmaWaitLimit polls.
__device__ __forceinline__ bool mbar_wait(unsigned long long* b, unsigned parity) {
  const unsigned a = smem_u32(b);
  for (unsigned n = 0; n < kTmaWaitLimit; n++) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 2-D tensor copy of one box into shared memory, completing on mbarrier b.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, unsigned long long* b) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(b))
      : "memory");
}

template <typename T>
struct ElemBytes {
  static constexpr int value = 8;
};
template <>
struct ElemBytes<F32> {
  static constexpr int value = 4;
};

// Shared-memory layout of one stage: the seven arrays' boxes, each padded to
// 128 bytes, in field order.
template <typename P>
struct TmaLayout {
  // Element bytes of field fld: split pressure (0, 1) and velocity (3, 4) as
  // stored, void fraction (2, 5, 6) 8 or 4.
  __host__ __device__ static constexpr int esz(int fld) {
    return (fld == 2 || fld >= 5) ? ElemBytes<typename P::G>::value
                                  : (fld <= 1 ? ElemBytes<typename P::S>::value : ElemBytes<typename P::V>::value);
  }
  __host__ __device__ static constexpr int offset(int fld) {
    int o = 0;
    for (int q = 0; q < fld; q++) o += tma_region_bytes(esz(q));
    return o;
  }
  static constexpr int stage_bytes = offset(kTmaFields);
  // Bytes the copies of one stage deliver (the boxes without padding).
  __host__ __device__ static constexpr unsigned tx_bytes() {
    unsigned t = 0;
    for (int q = 0; q < kTmaFields; q++) t += (unsigned)(kTmaBoxCols * kTmaRows * esz(q));
    return t;
  }
  static constexpr int bar_bytes = 128;  // 2 kTmaStages mbarriers, padded
  static constexpr int smem_bytes = bar_bytes + kTmaStages * stage_bytes;
};

template <typename P>
__global__ void __launch_bounds__(32 * (kTmaWarps + 1), 2)
    fdtd_tma(const __grid_constant__ GridParams g, const FdtdArgs<P> a, const __grid_constant__ TmaMaps maps,
             int chunk_rows, int* __restrict__ pipe_err) {
  using G = typename P::G;
  using S = typename P::S;
  using V = typename P::V;
  using L = TmaLayout<P>;
  extern __shared__ __align__(128) unsigned char tma_smem[];
  unsigned long long* full = reinterpret_cast<unsigned long long*>(tma_smem);
  unsigned long long* empty = full + kTmaStages;
  unsigned char* stages = tma_smem + L::bar_bytes;

  const Frame& f = g.f;
  const int X = f.X, Y = f.Y;
  const int warp = threadIdx.y;
  const int lane = threadIdx.x;
  const int by = blockIdx.y, cy = (by & 1) ? (int)gridDim.y - 1 - (by >> 1) : (by >> 1);
  const int j0 = 1 + cy * chunk_rows;
  const int j1 = min(Y, j0 + chunk_rows - 1);
  const int nrows = j1 - j0 + 3;  // rows j0-1 .. j1+1
  const int nst = (nrows + kTmaRows - 1) / kTmaRows;

  if (warp == 0 && lane == 0) {
    for (int s = 0; s < kTmaStages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kTmaWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();

  if (warp == kTmaWarps) {
    // Producer: one lane issues the copies of every stage of the chunk.
    if (lane != 0) return;
    const int x0 = blockIdx.x * (30 * kTmaWarps);  // frame column of logical i = 120 b - 1
    int issued = 0;
    bool ok = true;
    for (int s = 0; s < nst && ok; s++) {
      const int slot = s % kTmaStages;
      if (s >= kTmaStages && !mbar_wait(&empty[slot], (unsigned)((s / kTmaStages - 1) & 1))) {
        atomicOr(pipe_err, 1);
        ok = false;
        break;
      }
      unsigned char* st = stages + slot * L::stage_bytes;
      mbar_arrive_tx(&full[slot], L::tx_bytes());
      const int y = j0 + s * kTmaRows;  // frame row of logical j0 - 1 + s kTmaRows
#pragma unroll
      for (int q = 0; q < kTmaFields; q++) tma_load_2d(st + L::offset(q), &maps.m[q], x0, y, &full[slot]);
      issued = s + 1;
    }
    // The copies of the last stages are read by the consumers; when they
    // stopped early, wait (bounded) for every copy still in flight.
    for (int s = max(0, issued - kTmaStages); s < issued; s++)
      mbar_wait(&full[s % kTmaStages], (unsigned)((s / kTmaStages) & 1));
    return;
  }

  // Consumers.
  const unsigned full_mask = 0xffffffffu;
  const int i = (blockIdx.x * kTmaWarps + warp) * 30 + lane;
  const int col = warp * 30 + lane + 1;  // column of i inside the box
  const double t_prev = a.tdev[0], t_cur = a.tdev[1];
  const bool inwin = i <= X + 1;
  const bool cell = lane >= 1 && lane <= 30 && i <= X;
  const bool face = lane <= 30 && i <= X;
  const bool own = inwin && ((lane >= 1 && lane <= 30) || (lane == 0 && i == 0) || (lane == 31 && i == X + 1));
  const double xm = ((double)i - 0.5) * g.dx;
  const bool inner_col = i >= 1 && i <= X;
  const bool src_rows = g.source_row > 0 && src_pressure(g);
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
  // Element of field fld in chunk row rr (row j0 - 1 + rr).
  auto at = [&](int rr, int fld) -> const void* {
    const int slot = (rr / kTmaRows) % kTmaStages;
    return stages + slot * L::stage_bytes + L::offset(fld) + ((rr % kTmaRows) * kTmaBoxCols + col) * L::esz(fld);
  };
  bool ok = true;
  auto wait_stage = [&](int s) {
    if (ok && !mbar_wait(&full[s % kTmaStages], (unsigned)((s / kTmaStages) & 1))) {
      atomicOr(pipe_err, 1);
      ok = false;
    }
    ok = __all_sync(full_mask, ok);
  };
  auto release_stage = [&](int s) {
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s % kTmaStages]);
  };

  wait_stage(0);
  if (!ok) return;
  double pxc, pyc, fac, p0b, rhob, vyob;
  {
    const double pxb = S::staged(at(0, 0)), pyb = S::staged(at(0, 1));
    const double fab = G::staged(at(0, 2));
    vyob = V::staged(at(0, 4));
    pxc = S::staged(at(1, 0));
    pyc = S::staged(at(1, 1));
    fac = G::staged(at(1, 2));
    p0b = p0_of(j0 - 1, pxb, pyb);
    rhob = rho_of(fab);
    if (j0 == 1 && own) predict(f.idx(i, 0), fab);
  }
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

  const double vax_e = face ? g.vax[i + 1] : 1.0, vbx_e = face ? g.vbx[i + 1] : 1.0;
  const double pax_c = cell ? g.pax[i] : 1.0, pbx_c = cell ? g.pbx[i] : 1.0;
  const double xu_w = cell && g.cyl ? g.xu[i] : 0.0, xu_e = cell && g.cyl ? g.xu[i + 1] : 0.0;
  const double rxp_c = cell && g.cyl ? g.rxp[i] : 0.0;
  const bool zero_e = (i == 0 && !g.pml_x0) || (i == X && !g.pml_x1);

  unsigned long long res = 0ull;
#pragma unroll 1
  for (int jj = 0; jj < chunk_rows; jj++) {
    const int j = j0 + jj;
    if (j > j1) break;
    const unsigned k = kb + (unsigned)(jj + 1) * pitch;
    if ((jj + 2) % kTmaRows == 0) {
      wait_stage((jj + 2) / kTmaRows);
      if (!ok) return;
    }
    const double pxn = S::staged(at(jj + 2, 0)), pyn = S::staged(at(jj + 2, 1));
    const double fan = G::staged(at(jj + 2, 2));
    const double vxo = V::staged(at(jj + 1, 3)), vyo = V::staged(at(jj + 1, 4));
    const double fgp = G::stored(3.0 * fac - 3.0 * G::staged(at(jj + 1, 5)) + G::staged(at(jj + 1, 6)));
    if ((jj + 1) % kTmaRows == kTmaRows - 1) release_stage((jj + 1) / kTmaRows);
    if (own) a.fgC.put(k, fgp);
    const double p0n = p0_of(j + 1, pxn, pyn), rhon = rho_of(fan);
    const double p0r = __shfl_down_sync(full_mask, p0c, 1), rhor = __shfl_down_sync(full_mask, rhoc, 1);
    double q_e = g.dt_rho, q_n = g.dt_rho, h = 0.0;
    if (__any_sync(full_mask,
                   rhoc != g.rho_inf || rhor != g.rho_inf || rhon != g.rho_inf || fgp != 0.0 || fac != 0.0)) {
      q_e = face_q(g, rhoc, rhor);
      q_n = face_q(g, rhoc, rhon);
      h = void_rate_half(g, fgp, fac);
    }
    double fe = velocity_face_q(g, vxo, p0c, p0r, q_e, vax_e, vbx_e);
    if (zero_e) fe = 0.0;
    const double fw = __shfl_up_sync(full_mask, fe, 1);
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
      a.vx_new.put(k, fe);
    }
    vyd = vyu;
    pxc = pxn;
    pyc = pyn;
    fac = fan;
    p0c = p0n;
    rhoc = rhon;
  }
  if (j1 == Y && own) predict(f.idx(i, Y + 1), fac);
  for (int o = 16; o > 0; o >>= 1) res = max(res, __shfl_xor_sync(full_mask, res, o));
  if (lane == 0 && res) atomicMax(a.residual, res);
}

}  // namespace crp
