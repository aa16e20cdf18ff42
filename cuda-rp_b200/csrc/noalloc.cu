// Void fraction of a bubble population without any device allocation.
//
// Some callers cannot allocate device memory at the moment they need this
// result: latency-critical loops, where cudaMalloc/cudaFree may synchronise the
// whole device, and applications whose own memory pool owns the GPU's memory
// (a framework allocator, a fixed budget on a shared GPU).  For them,
// crp_void_fraction_noalloc computes the same deterministic bubble-to-grid
// scatter that crp_create performs for its initial void fraction (cell binning
// by counting sort, bins in ascending bubble order, per-cell gather, axis
// fold), with every scratch buffer carved from one fixed array of this library.
//
// The scratch array is a file-scope __device__ array, so every GPU that loads
// the library holds CRP_NOALLOC_SCRATCH_BYTES of it until the process exits.
// Host code cannot pass the array's name to a kernel (on the host it is only a
// stand-in symbol), so the first call on each device looks up its device
// address with cudaGetSymbolAddress while that device is current and caches
// it; make that first call outside any stream capture.  All calls share the
// one array and leave their contents in it: each call clears what must start
// at zero, and two calls whose work overlaps on the GPU (different streams,
// or different host threads on the same device) race on the array.  The cached
// address belongs to the device's context: after cudaDeviceReset on a device,
// do not call this entry point on that device again in the same process.
#include <cuda_runtime.h>

#include <climits>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>

#include "crp.h"

namespace {

constexpr size_t kScratchBytes = CRP_NOALLOC_SCRATCH_BYTES;
__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
void* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

// Message of the calling thread's last failed call (crp_last_error(NULL)).
thread_local std::string t_last_error;

crp_status failed(crp_status st, const char* what, cudaError_t e = cudaSuccess) {
  t_last_error = what;
  if (e != cudaSuccess) t_last_error += std::string(": ") + cudaGetErrorString(e);
  return st;
}

struct Geometry {
  int X, Y;
  double dx, dy, rdx, rdy;
  double dcx, dcy, dcz;  // smooth-delta coefficients (src/bubble_CUDA.cu:1469-1471)
  double pi4r3;
  int cyl;
};

struct Scratch {
  int* count;    // nbins, cleared by every call
  int* start;    // nbins + 1
  int* partial;  // block sums + total
  int* bin;      // n
  int* idx;      // n
  int* ibnx;     // n
  int* ibny;     // n
  double* contrib;  // 4 n
};

constexpr int kScan = 1024;

inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

size_t scratch_bytes(int nbins, int n, Scratch* s, unsigned char* base) {
  size_t off = 0;
  auto take = [&](size_t bytes) {
    unsigned char* p = base ? base + off : nullptr;
    off += align256(bytes);
    return p;
  };
  const int nblk = (nbins + kScan - 1) / kScan;
  int* count = (int*)take(sizeof(int) * nbins);
  int* start = (int*)take(sizeof(int) * (nbins + 1));
  int* partial = (int*)take(sizeof(int) * (nblk + 1));
  int* bin = (int*)take(sizeof(int) * n);
  int* idx = (int*)take(sizeof(int) * n);
  int* ibnx = (int*)take(sizeof(int) * n);
  int* ibny = (int*)take(sizeof(int) * n);
  double* contrib = (double*)take(sizeof(double) * 4 * (size_t)n);
  if (s) *s = Scratch{count, start, partial, bin, idx, ibnx, ibny, contrib};
  return off;
}

__global__ void na_clear(int* __restrict__ count, int nbins) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nbins) count[k] = 0;
}

// Cell of each bubble (BubbleUpdateIndexKernel, inc/bubble_CUDA_kernel.cuh:345-358),
// its bin over [-1, X+1] x [-1, Y+1], the bin counts, and the bubble's
// contribution (4/3) pi n_B R^3 / (dx dy [x]) delta_x delta_y to the four
// cells of its stencil (VoidFractionReverseLookupKernel, :595-617).
__global__ void na_index(Geometry g, int n, const double* __restrict__ x, const double* __restrict__ y,
                         const double* __restrict__ r, const double* __restrict__ nb, Scratch s) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  const double bx = x[b], by = y[b];
  const int ix = (int)floor(bx * g.rdx + 0.5);
  const int iy = (int)floor(by * g.rdy + 0.5);
  s.ibnx[b] = ix;
  s.ibny[b] = iy;
  int c = -1;
  if (ix >= -1 && ix <= g.X + 1 && iy >= -1 && iy <= g.Y + 1) c = (iy + 1) * (g.X + 3) + (ix + 1);
  s.bin[b] = c;
  if (c >= 0) atomicAdd(&s.count[c], 1);
  double dxw[2], dyw[2];
  for (int q = 0; q < 2; q++) {
    dxw[q] = g.dcx * (1.0 + cos(g.dcy * (((double)(ix + q) - 0.5) * g.dx - bx)));
    dyw[q] = g.dcx * (1.0 + cos(g.dcz * (((double)(iy + q) - 0.5) * g.dy - by)));
  }
  const double R = r[b];
  const double vol = g.cyl ? g.pi4r3 * nb[b] * (R * R * R) * g.rdx * g.rdy / bx
                           : g.pi4r3 * nb[b] * (R * R * R) * g.rdx * g.rdy;
  double* cb = s.contrib + 4 * (long)b;
  cb[0] = vol * dxw[0] * dyw[0];
  cb[1] = vol * dxw[0] * dyw[1];
  cb[2] = vol * dxw[1] * dyw[0];
  cb[3] = vol * dxw[1] * dyw[1];
}

__device__ __forceinline__ int na_block_scan(int v, int* total) {
  __shared__ int s_w[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += t;
  }
  if (lane == 31) s_w[w] = x;
  __syncthreads();
  if (w == 0) {
    int t = s_w[lane];
    for (int o = 1; o < 32; o <<= 1) {
      int u = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += u;
    }
    s_w[lane] = t;
  }
  __syncthreads();
  const int before = (w > 0 ? s_w[w - 1] : 0) + x - v;
  if (total) *total = s_w[31];
  return before;
}

__global__ void __launch_bounds__(kScan) na_scan_blocks(Scratch s, int nbins) {
  const int k = blockIdx.x * kScan + threadIdx.x;
  int total;
  const int e = na_block_scan(k < nbins ? s.count[k] : 0, &total);
  if (k < nbins) s.start[k] = e;
  if (threadIdx.x == 0) s.partial[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScan) na_scan_partials(Scratch s, int nparts) {
  int carry = 0;
  for (int base = 0; base < nparts; base += kScan) {
    const int k = base + threadIdx.x;
    int total;
    const int e = na_block_scan(k < nparts ? s.partial[k] : 0, &total);
    __syncthreads();
    if (k < nparts) s.partial[k] = e + carry;
    carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) s.partial[nparts] = carry;
}

__global__ void na_scan_add(Scratch s, int nbins, int nparts) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nbins) s.start[k] += s.partial[k / kScan];
  if (k == nbins) s.start[nbins] = s.partial[nparts];
}

__global__ void na_fill(Scratch s, int n) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  const int c = s.bin[b];
  if (c < 0) return;
  s.idx[s.start[c] + atomicSub(&s.count[c], 1) - 1] = b;
}

// Bubbles of each bin in ascending index order: a fixed summation order.
__global__ void na_sort(Scratch s, int nbins) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nbins) return;
  const int a = s.start[c], e = s.start[c + 1];
  for (int k = a + 1; k < e; k++) {
    const int v = s.idx[k];
    int m = k - 1;
    while (m >= a && s.idx[m] > v) {
      s.idx[m + 1] = s.idx[m];
      m--;
    }
    s.idx[m + 1] = v;
  }
}

__device__ __forceinline__ double na_cell(const Geometry& g, const Scratch& s, int i, int j) {
  double acc = 0.0;
  for (int by = j - 1; by <= j; by++) {
    for (int bx = i - 1; bx <= i; bx++) {
      const int c = (by + 1) * (g.X + 3) + (bx + 1);
      const int slot = (i - bx) * 2 + (j - by);
      for (int k = s.start[c]; k < s.start[c + 1]; k++) acc += s.contrib[4 * (long)s.idx[k] + slot];
    }
  }
  return acc;
}

// Per-cell gather and axis fold (VoidFractionCylinderKernel, :559-573) into the
// caller's dense (X+2) x (Y+2) array.
__global__ void na_gather(Geometry g, Scratch s, double* __restrict__ fg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i > g.X + 1 || j > g.Y + 1) return;
  const double v = (g.cyl && i <= 1) ? na_cell(g, s, 0, j) + na_cell(g, s, 1, j) : na_cell(g, s, i, j);
  fg[(long)j * (g.X + 2) + i] = v;
}

// Device address of g_scratch on the current device, looked up once per device.
cudaError_t scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" {

size_t crp_void_fraction_noalloc_scratch(int32_t grid_x, int32_t grid_y, int32_t n) {
  if (grid_x < 2 || grid_y < 2 || n < 0) return 0;
  const long long nbins = ((long long)grid_x + 3) * ((long long)grid_y + 3);
  if (nbins > (1LL << 30)) return SIZE_MAX;
  return scratch_bytes((int)nbins, n, nullptr, nullptr);
}

crp_status crp_void_fraction_noalloc(const crp_config* cfg, int32_t n, const double* x, const double* y,
                                     const double* r, const double* n_b, double* f_g, void* stream) {
  if (!cfg || !f_g || n < 0 || (n > 0 && (!x || !y || !r || !n_b)))
    return failed(CRP_ERR_INVALID, "crp_void_fraction_noalloc: null pointer or negative count");
  if (cfg->grid_x < 2 || cfg->grid_y < 2 || !(cfg->grid_lx > 0) || !(cfg->grid_ly > 0))
    return failed(CRP_ERR_INVALID, "crp_void_fraction_noalloc: grid of fewer than 2 x 2 cells or zero length");
  if (cfg->sim_smooth_delta_band != 2)
    return failed(CRP_ERR_UNSUPPORTED, "crp_void_fraction_noalloc: smooth_delta_band 2 only");
  const int X = cfg->grid_x, Y = cfg->grid_y;
  const long long nbins_ll = ((long long)X + 3) * ((long long)Y + 3);
  if (nbins_ll > (1LL << 30)) return failed(CRP_ERR_TOO_LARGE, "crp_void_fraction_noalloc: grid too large");
  const int nbins = (int)nbins_ll;
  if (scratch_bytes(nbins, n, nullptr, nullptr) > kScratchBytes)
    return failed(CRP_ERR_TOO_LARGE, "crp_void_fraction_noalloc: grid and bubbles need more than the fixed scratch");
  // A launch error left pending by earlier work on this thread is not this
  // call's: drop it, so that the check after this call's launches reports
  // only their own errors.  (A sticky error still fails the launches below.)
  (void)cudaGetLastError();

  void* base = nullptr;
  cudaError_t e = scratch_address(&base);
  if (e != cudaSuccess) return failed(CRP_ERR_CUDA, "crp_void_fraction_noalloc: cudaGetSymbolAddress", e);
  Scratch s;
  scratch_bytes(nbins, n, &s, (unsigned char*)base);

  // Grid geometry as init_grid_size and delta_coef define it (src/bubble_CUDA.cu:524-540, 1469-1471).
  Geometry g;
  g.X = X;
  g.Y = Y;
  g.dx = (double)cfg->grid_lx / (double)X;
  g.dy = (double)cfg->grid_ly / (double)Y;
  g.rdx = (double)1.0 / (double)g.dx;
  g.rdy = (double)1.0 / (double)g.dy;
  g.dcx = 1.0 / 2.0;
  g.dcy = 2.0 * std::acos(-1.0) / 2.0 * g.rdx;
  g.dcz = 2.0 * std::acos(-1.0) / 2.0 * g.rdy;
  g.pi4r3 = std::acos(-1.0) * 4.0 / 3.0;
  g.cyl = cfg->tr_cylindrical != 0;

  cudaStream_t st = (cudaStream_t)stream;
  const int nblk = (nbins + kScan - 1) / kScan;
  na_clear<<<(nbins + 255) / 256, 256, 0, st>>>(s.count, nbins);
  if (n > 0) na_index<<<(n + 255) / 256, 256, 0, st>>>(g, n, x, y, r, n_b, s);
  na_scan_blocks<<<nblk, kScan, 0, st>>>(s, nbins);
  na_scan_partials<<<1, kScan, 0, st>>>(s, nblk);
  na_scan_add<<<(nbins + 1 + 255) / 256, 256, 0, st>>>(s, nbins, nblk);
  if (n > 0) na_fill<<<(n + 255) / 256, 256, 0, st>>>(s, n);
  na_sort<<<(nbins + 255) / 256, 256, 0, st>>>(s, nbins);
  dim3 blk(32, 8), grd((X + 2 + 31) / 32, (Y + 2 + 7) / 8);
  na_gather<<<grd, blk, 0, st>>>(g, s, f_g);
  e = cudaGetLastError();
  return e == cudaSuccess ? CRP_OK : failed(CRP_ERR_CUDA, "crp_void_fraction_noalloc: kernel launch", e);
}

}  // extern "C"

namespace crp {
const char* noalloc_last_error() { return t_last_error.c_str(); }
}  // namespace crp
