// Batched sweep: many independent simulations advanced concurrently on one GPU.
//
// The reference runs one configuration per process and sweeps parameters by
// re-running the program over a list of files (scripts/executor.sh:28-47).
// Here one crp_batch owns any number of crp_sim handles, each with its own
// CUDA stream, and crp_batch_run advances them from a pool of host threads:
// while one simulation waits on its Picard residual, the kernels of the others
// keep the GPU busy, which matters for the small grids of a sweep that cannot
// fill 148 SMs on their own.  Work is handed out largest-first (cells x steps)
// so the long simulations start early.
#include <algorithm>
#include <atomic>
#include <new>
#include <numeric>
#include <thread>
#include <vector>

#include "crp.h"

struct crp_batch {
  std::vector<crp_sim*> sims;
  std::vector<double> cells;  // interior cells per simulation
};

extern "C" {

crp_status crp_batch_create(int32_t count, const crp_config* cfgs, const crp_bubbles_in* bubbles, crp_batch** out) {
  if (!out || count <= 0 || !cfgs) return CRP_ERR_INVALID;
  *out = nullptr;
  crp_batch* b = new (std::nothrow) crp_batch();
  if (!b) return CRP_ERR_ALLOC;
  for (int32_t k = 0; k < count; k++) {
    const crp_bubbles_in* bk = (bubbles && bubbles[k].n > 0) ? &bubbles[k] : nullptr;
    crp_sim* s = nullptr;
    crp_status st = crp_create(&cfgs[k], bk, nullptr, &s);
    if (st != CRP_OK) {
      crp_batch_destroy(b);
      return st;
    }
    b->sims.push_back(s);
    b->cells.push_back((double)cfgs[k].grid_x * (double)cfgs[k].grid_y);
  }
  *out = b;
  return CRP_OK;
}

int32_t crp_batch_count(const crp_batch* b) { return b ? (int32_t)b->sims.size() : 0; }

crp_sim* crp_batch_sim(crp_batch* b, int32_t k) {
  if (!b || k < 0 || k >= (int32_t)b->sims.size()) return nullptr;
  return b->sims[k];
}

crp_status crp_batch_run(crp_batch* b, const int32_t* steps, int32_t threads, crp_status* per_sim) {
  if (!b || !steps) return CRP_ERR_INVALID;
  const int n = (int)b->sims.size();
  for (int k = 0; k < n; k++)
    if (steps[k] < 0) return CRP_ERR_INVALID;
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int p, int q) {
    return b->cells[p] * (double)steps[p] > b->cells[q] * (double)steps[q];
  });
  std::vector<crp_status> st(n, CRP_OK);
  std::atomic<int> next{0};
  auto worker = [&]() {
    for (;;) {
      const int q = next.fetch_add(1);
      if (q >= n) return;
      const int k = order[q];
      st[k] = crp_step(b->sims[k], steps[k]);
    }
  };
  int t = threads > 0 ? threads : std::min(n, 32);
  t = std::max(1, std::min(t, n));
  std::vector<std::thread> pool;
  pool.reserve(t - 1);
  for (int w = 1; w < t; w++) pool.emplace_back(worker);
  worker();
  for (auto& th : pool) th.join();
  crp_status first = CRP_OK;
  for (int k = 0; k < n; k++) {
    if (per_sim) per_sim[k] = st[k];
    if (first == CRP_OK && st[k] != CRP_OK) first = st[k];
  }
  return first;
}

void crp_batch_destroy(crp_batch* b) {
  if (!b) return;
  for (crp_sim* s : b->sims) crp_destroy(s);
  delete b;
}

}  // extern "C"
