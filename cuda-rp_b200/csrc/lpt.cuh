// Solve order of the persistent radius kernels (2-D and 3-D paths): bubbles
// sorted heaviest-first by their last sub-step count, so that the bubbles
// with the longest serial chains start first.  The kernels are local to each
// translation unit that includes this header.
#pragma once

namespace crp {

// Work order for the next radius solves: bubbles bucketed by the binary
// logarithm of their last sub-step count, heaviest bucket first.
constexpr int kLptBuckets = 32;
constexpr long long kLptMinSubsteps = 12;  // the quiet phase takes 10 (dt0 = dt / 10)

__device__ __forceinline__ int lpt_bucket(int nsub) {
  return kLptBuckets - 1 - min(kLptBuckets - 1, 31 - __clz(max(nsub, 1)));
}

static __global__ void lpt_count(const int* __restrict__ nsub, int n, int* __restrict__ hist) {
  __shared__ int s_h[kLptBuckets];
  if (threadIdx.x < kLptBuckets) s_h[threadIdx.x] = 0;
  __syncthreads();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) atomicAdd(&s_h[lpt_bucket(nsub[k])], 1);
  __syncthreads();
  if (threadIdx.x < kLptBuckets && s_h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], s_h[threadIdx.x]);
}

// hist -> exclusive starts (one warp); hist is left zeroed for the next count.
static __global__ void lpt_scan(int* __restrict__ hist, int* __restrict__ cursor) {
  const int lane = threadIdx.x;
  int v = hist[lane];
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  cursor[lane] = x - v;
  hist[lane] = 0;
}

// Bubbles into their buckets' ranges.  Slots are reserved per warp (shared
// atomics) and then per block (one global atomic per bucket), because most
// bubbles usually share one bucket and per-bubble atomics on one counter
// serialise.  The order inside a bucket is not fixed; it only affects scheduling.
constexpr int kLptScatterThreads = 1024;

static __global__ void __launch_bounds__(kLptScatterThreads)
    lpt_scatter(const int* __restrict__ nsub, int n, int* __restrict__ cursor, int* __restrict__ order) {
  __shared__ int s_cnt[kLptBuckets], s_base[kLptBuckets];
  if (threadIdx.x < kLptBuckets) s_cnt[threadIdx.x] = 0;
  __syncthreads();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool on = k < n;
  const int bkt = on ? lpt_bucket(nsub[k]) : -1;
  const unsigned peers = __match_any_sync(0xffffffffu, bkt);
  const int leader = __ffs(peers) - 1;
  int wbase = 0;
  if (on && lane == leader) wbase = atomicAdd(&s_cnt[bkt], __popc(peers));
  wbase = __shfl_sync(0xffffffffu, wbase, leader);
  __syncthreads();
  if (threadIdx.x < kLptBuckets && s_cnt[threadIdx.x])
    s_base[threadIdx.x] = atomicAdd(&cursor[threadIdx.x], s_cnt[threadIdx.x]);
  __syncthreads();
  if (on) order[s_base[bkt] + wbase + __popc(peers & ((1u << lane) - 1u))] = k;
}

}  // namespace crp
