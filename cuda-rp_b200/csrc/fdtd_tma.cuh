// The fused FDTD pass on tiles staged by the tensor memory accelerator (TMA).
//
// Same arithmetic and output as the strip march of fdtd_strip (void-fraction
// prediction, VelocityKernel with VelocityBoundaryKernel's faces and
// MixturePressureKernel with its residual, inc/bubble_CUDA_kernel.cuh:622-867),
// organised for latency hiding instead of a serial march: one thread per cell.
//
// A persistent block of 32 x 16 threads walks a static list of 32 x 16-cell
// tiles.  For each tile one thread issues seven 2-D tensor copies
// (cp.async.bulk.tensor) of the tile and a halo (36 x 18 elements: columns
// i0-2 .. i0+33, rows j0-1 .. j0+16) of the seven input arrays into one of two
// shared-memory buffers, completing on that buffer's mbarrier; the copies of
// the next tile are issued before the current one is computed, so one tile's
// loads are always in flight behind the arithmetic.  The tile is then done in
// three phases separated by block barriers:
//   1. p0 = px + py (with the boundary rules of MixtureBoundaryPressureKernel
//      at the domain's edges) and rho_m = (1 - f_g) rho_inf for the tile and a
//      one-cell ring, into shared memory;
//   2. every east face (velocity vx, 33 columns) and north face (vy, 17 rows)
//      of the tile, each computed once, into shared memory, and stored;
//   3. the split-pressure update, residual and void-fraction prediction of
//      every cell.
// Every thread's work in a phase is independent of the others', so a tile's
// latency is hidden by the 32 warps of two resident blocks per SM.
//
// Tensor boxes start at frame column 32 tx (logical i = 32 tx - 1), a multiple
// of 4 elements, and are 36 columns wide (288 or 144 bytes): the innermost
// coordinate and extent of every copy are multiples of 16 bytes.  Rows and
// columns outside the frame are filled with zeros by the copy and never
// stored.  Every mbarrier wait is bounded: a wait that runs out sets the
// step's pipeline error word and the block stops after waiting, again
// bounded, for the copies it issued.
#pragma once
#include <cuda.h>

namespace crp {

constexpr int kTileX = 32;            // cells per tile row (one warp)
constexpr int kTileY = 16;            // cell rows per tile (one warp each)
constexpr int kBoxX = kTileX + 4;     // box columns: logical i0-2 .. i0+33
constexpr int kBoxY = kTileY + 2;     // box rows: logical j0-1 .. j0+16
constexpr int kHaloX = kTileX + 2;    // p0 / rho columns i0-1 .. i0+32
constexpr int kTmaFields = 7;         // pnx, pny, fgA, vx_old, vy_old, fgB, fgC
constexpr unsigned kTmaWaitLimit = 1u << 22;  // polls of one mbarrier wait before it gives up

struct TmaMaps {
  CUtensorMap m[kTmaFields];
};

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
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

// Shared memory of one block: two buffers of the seven boxes (each padded to
// 128 bytes), then p0 and rho of the tile and its ring, the east and north
// faces, and two mbarriers.
template <typename P>
struct TileLayout {
  // Element bytes of field fld: split pressure (0, 1) and velocity (3, 4) as
  // stored, void fraction (2, 5, 6) 8 or 4.
  __host__ __device__ static constexpr int esz(int fld) {
    return (fld == 2 || fld >= 5) ? ElemBytes<typename P::G>::value
                                  : (fld <= 1 ? ElemBytes<typename P::S>::value : ElemBytes<typename P::V>::value);
  }
  __host__ __device__ static constexpr int region(int fld) { return (kBoxX * kBoxY * esz(fld) + 127) / 128 * 128; }
  __host__ __device__ static constexpr int offset(int fld) {
    int o = 0;
    for (int q = 0; q < fld; q++) o += region(q);
    return o;
  }
  static constexpr int buf_bytes = offset(kTmaFields);
  __host__ __device__ static constexpr unsigned tx_bytes() {
    unsigned t = 0;
    for (int q = 0; q < kTmaFields; q++) t += (unsigned)(kBoxX * kBoxY * esz(q));
    return t;
  }
  static constexpr int p0_off = 2 * buf_bytes;
  static constexpr int rho_off = p0_off + kBoxY * kHaloX * 8;
  static constexpr int fx_off = rho_off + kBoxY * kHaloX * 8;
  static constexpr int fy_off = fx_off + kTileY * (kTileX + 1) * 8;
  static constexpr int bar_off = fy_off + (kTileY + 1) * kTileX * 8;
  static constexpr int smem_bytes = bar_off + 16;
};

template <typename P>
__global__ void __launch_bounds__(kTileX* kTileY, 2)
    fdtd_tile(const __grid_constant__ GridParams g, const FdtdArgs<P> a, const __grid_constant__ TmaMaps maps,
              int ntx, int ntiles, int* __restrict__ pipe_err) {
  using G = typename P::G;
  using S = typename P::S;
  using V = typename P::V;
  using L = TileLayout<P>;
  extern __shared__ __align__(128) unsigned char tsm[];
  double* p0s = reinterpret_cast<double*>(tsm + L::p0_off);   // [kBoxY][kHaloX], rows j0-1.., cols i0-1..
  double* rhos = reinterpret_cast<double*>(tsm + L::rho_off);
  double* fx = reinterpret_cast<double*>(tsm + L::fx_off);    // [kTileY][kTileX+1], east faces of i0-1 ..
  double* fy = reinterpret_cast<double*>(tsm + L::fy_off);    // [kTileY+1][kTileX], north faces of j0-1 ..
  unsigned long long* full = reinterpret_cast<unsigned long long*>(tsm + L::bar_off);

  const Frame& f = g.f;
  const int X = f.X, Y = f.Y;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * kTileX + tx;
  const double t_prev = a.tdev[0], t_cur = a.tdev[1];
  const bool src_rows = g.source_row > 0 && src_pressure(g);

  if (tid == 0) {
    mbar_init(&full[0], 1);
    mbar_init(&full[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();

  auto issue = [&](int t, int buf) {
    const int x0 = (t % ntx) * kTileX;         // frame column of logical i0 - 2
    const int y0 = 1 + (t / ntx) * kTileY;     // frame row of logical j0 - 1
    unsigned char* dst = tsm + buf * L::buf_bytes;
    mbar_arrive_tx(&full[buf], L::tx_bytes());
#pragma unroll
    for (int q = 0; q < kTmaFields; q++) tma_load_2d(dst + L::offset(q), &maps.m[q], x0, y0, &full[buf]);
  };

  const int first = blockIdx.x;
  if (tid == 0 && first < ntiles) issue(first, 0);
  unsigned long long res = 0ull;
  int k = 0;
  bool ok = true;
  int in_flight = first < ntiles ? 1 : 0;  // tile copies issued and not yet waited for (thread 0's view)
  for (int t = first; t < ntiles; t += gridDim.x, k++) {
    const int buf = k & 1;
    // The other buffer was last read by the previous tile, finished at its
    // closing barrier: the next tile's copies may go there now.
    if (tid == 0 && t + (int)gridDim.x < ntiles) {
      issue(t + gridDim.x, buf ^ 1);
      in_flight++;
    }
    if (!mbar_wait(&full[buf], (unsigned)((k >> 1) & 1))) {
      atomicOr(pipe_err, 1);
      ok = false;
    }
    if (__syncthreads_or(!ok)) {
      ok = false;
      break;
    }
    in_flight--;
    const unsigned char* box = tsm + buf * L::buf_bytes;
    // Box element of field fld at logical (i, j).
    const int i0 = 1 + (t % ntx) * kTileX, j0 = 1 + (t / ntx) * kTileY;
    auto at = [&](int fld, int i, int j) -> const void* {
      return box + L::offset(fld) + ((j - j0 + 1) * kBoxX + (i - i0 + 2)) * L::esz(fld);
    };

    // Phase 1: p0 and rho over columns i0-1 .. i0+32, rows j0-1 .. j0+16.
    for (int e = tid; e < kBoxY * kHaloX; e += kTileX * kTileY) {
      const int r = e / kHaloX, c = e % kHaloX;
      const int i = i0 - 1 + c, j = j0 - 1 + r;
      double p0 = 0.0, rho = g.rho_inf;
      if (i <= X + 1 && j <= Y + 1) {
        if (i >= 1 && i <= X && j >= 1 && j <= Y && !(src_rows && j == g.source_row))
          p0 = S::staged(at(0, i, j)) + S::staged(at(1, i, j));
        else
          p0 = p0_edge(g, a.pnx, a.pny, i, j, t_prev);
        if (!a.rho_const) rho = (1.0 - G::staged(at(2, i, j))) * g.rho_inf;
      }
      p0s[e] = p0;
      rhos[e] = rho;
    }
    __syncthreads();

    // Phase 2a: east faces vx(i, j), i in i0-1 .. i0+31, j in j0 .. j0+15.
    for (int e = tid; e < kTileY * (kTileX + 1); e += kTileX * kTileY) {
      const int r = e / (kTileX + 1), c = e % (kTileX + 1);
      const int i = i0 - 1 + c, j = j0 + r;
      double fe = 0.0;
      if (i <= X && j <= Y) {
        const int h = (r + 1) * kHaloX + c;  // cell (i, j) in p0s
        fe = velocity_face_q(g, V::staged(at(3, i, j)), p0s[h], p0s[h + 1], face_q(g, rhos[h], rhos[h + 1]),
                             g.vax[i + 1], g.vbx[i + 1]);
        if ((i == 0 && !g.pml_x0) || (i == X && !g.pml_x1)) fe = 0.0;
        if (i >= i0 || i == 0) a.vx_new.put(f.idx(i, j), fe);
      }
      fx[e] = fe;
    }
    // Phase 2b: north faces vy(i, j), j in j0-1 .. j0+15, i in i0 .. i0+31.
    for (int e = tid; e < (kTileY + 1) * kTileX; e += kTileX * kTileY) {
      const int r = e / kTileX, c = e % kTileX;
      const int i = i0 + c, j = j0 - 1 + r;
      double vn = 0.0;
      if (i <= X && j <= Y) {
        const int h = r * kHaloX + c + 1;  // cell (i, j) in p0s
        double pre;
        vn = vy_face_value(g, j, V::staged(at(4, i, j)), p0s[h], p0s[h + kHaloX],
                           face_q(g, rhos[h], rhos[h + kHaloX]), ((double)i - 0.5) * g.dx, t_cur, pre);
        if (j >= j0) {
          a.vy_new.put(f.idx(i, j), vn);
        } else if (j == 0) {
          a.vy_new.put(f.idx(i, 0), vn);
          if (!g.pml_y0) a.vy_new.put(f.idx(i, -1), pre);
        }
      }
      fy[e] = vn;
    }
    __syncthreads();

    // Phase 3: the cell (i, j) of this thread.
    const int i = i0 + tx, j = j0 + ty;
    if (i <= X && j <= Y) {
      auto predict_at = [&](int ii, int jj) -> double {
        const double v = G::stored(3.0 * G::staged(at(2, ii, jj)) - 3.0 * G::staged(at(5, ii, jj)) +
                                   G::staged(at(6, ii, jj)));
        a.fgC.put(f.idx(ii, jj), v);
        return v;
      };
      const double fac = G::staged(at(2, i, j));
      const double fgp = predict_at(i, j);
      // Ghost columns 0 and X+1 and ghost rows 0 and Y+1 (and the corners)
      // are predicted by the cells next to them.
      const bool wl = i == 1, wr = i == X, wb = j == 1, wt = j == Y;
      if (wl) predict_at(0, j);
      if (wr) predict_at(X + 1, j);
      if (wb) predict_at(i, 0);
      if (wt) predict_at(i, Y + 1);
      if (wl && wb) predict_at(0, 0);
      if (wl && wt) predict_at(0, Y + 1);
      if (wr && wb) predict_at(X + 1, 0);
      if (wr && wt) predict_at(X + 1, Y + 1);
      const double hv = void_rate_half(g, fgp, fac);
      const double fe = fx[ty * (kTileX + 1) + tx + 1], fw = fx[ty * (kTileX + 1) + tx];
      const double vyu = fy[(ty + 1) * kTileX + tx], vyd = fy[ty * kTileX + tx];
      const double s1x = g.cyl ? (-g.xu[i] * fw + g.xu[i + 1] * fe) * g.rdx * g.rxp[i] : (-fw + fe) * g.rdx;
      const double s1y = (-vyd + vyu) * g.rdy;
      const double qx = pressure_component(g, S::staged(at(0, i, j)), g.pax[i], g.pbx[i], s1x, hv);
      const double qy = pressure_component(g, S::staged(at(1, i, j)), g.pay[j], g.pby[j], s1y, hv);
      const long kk = f.idx(i, j);
      a.px.put(kk, qx);
      a.py.put(kk, qy);
      double p0new = qx + qy;
      if (src_rows && j == g.source_row) p0new = source_row_pressure(g, ((double)i - 0.5) * g.dx, t_cur);
      const double p0c = p0s[(ty + 1) * kHaloX + tx + 1];
      res = max(res, (unsigned long long)__double_as_longlong(fabs(p0c - p0new)));
    }
    __syncthreads();
  }
  if (!ok && tid == 0) {
    // Copies issued and not waited for (at most the next tile's): wait,
    // bounded, so that none lands after the block has exited.
    for (int q = 0; q < in_flight; q++) {
      const int kk = k + q;
      mbar_wait(&full[kk & 1], (unsigned)((kk >> 1) & 1));
    }
  }
  for (int o = 16; o > 0; o >>= 1) res = max(res, __shfl_xor_sync(0xffffffffu, res, o));
  if (tx == 0 && res) atomicMax(a.residual, res);
}

}  // namespace crp
