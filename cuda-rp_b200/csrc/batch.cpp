// Batched sweep: many independent simulations advanced concurrently on one GPU.
//
// The reference runs one configuration per process and sweeps parameters by
// re-running the program over a list of files (scripts/executor.sh:28-47).
// Here one crp_batch owns any number of crp_sim handles, each with its own
// CUDA stream, so that the small grids of a sweep, which cannot fill 148 SMs
// on their own, share the GPU.  Two ways to drive them:
//   CRP_BATCH_THREADS  a pool of host threads, each running its simulations'
//                      host-driven steps: while one waits on its Picard
//                      residual, the kernels of the others keep the GPU busy;
//   CRP_BATCH_GRAPHS   one host thread queues every simulation's steps as
//                      CUDA graphs whose Picard loop is decided on the device,
//                      then waits once for all of them: no host round trip per
//                      step or iteration, and no contention between threads.
// Work is handed out largest-first (cells x steps) so the long simulations
// start early.  crp_batch_tune times the candidate settings on the batch itself
// (its state saved and restored around every trial) and keeps the fastest.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <new>
#include <numeric>
#include <thread>
#include <vector>

#include "crp.h"
#include "crp_host.h"

namespace {
constexpr int kRpLaneThreads = 128;  // threads per block of the radius kernels (sim.cu, sim3d.cu)
}

struct crp_batch {
  std::vector<crp_sim*> sims;
  std::vector<double> cells;  // interior cells per simulation
  std::vector<int> nb;        // bubbles per simulation
  crp_batch_tuning tuning{CRP_BATCH_THREADS, 0, 0, 8, 1, 0.0};
};

namespace {

// Runs steps[k] on simulation k for every k in `which` from a pool of host
// threads, largest cells x steps first.
void run_threads(crp_batch* b, const std::vector<int>& which, const int32_t* steps, int threads,
                 std::vector<crp_status>& st) {
  const int n = (int)which.size();
  if (n == 0) return;
  std::vector<int> order(which);
  std::stable_sort(order.begin(), order.end(), [&](int p, int q) {
    return b->cells[p] * (double)steps[p] > b->cells[q] * (double)steps[q];
  });
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
}

// CRP_BATCH_GRAPHS: the steps that must run from the host (a simulation's
// first step, or all of them where graphs do not apply) go to a helper thread;
// the rest are queued as graphs from this thread, largest first, and waited
// for once.
void run_graphs(crp_batch* b, const int32_t* steps, std::vector<crp_status>& st) {
  const int n = (int)b->sims.size();
  std::vector<int> host_only, graph;
  std::vector<int32_t> left(steps, steps + n);
  for (int k = 0; k < n; k++) {
    crp::sim_allow_graphs(b->sims[k], true);
    // The first step (initial mixture density) runs from the host; after it
    // the simulation is graph-ready unless graphs do not apply to it.
    while (left[k] > 0 && !crp::sim_graph_ready(b->sims[k]) && crp::sim_step_count(b->sims[k]) == 0) {
      st[k] = crp_step(b->sims[k], 1);
      left[k]--;
      if (st[k] != CRP_OK) break;
    }
    if (st[k] != CRP_OK || left[k] == 0) continue;
    (crp::sim_graph_ready(b->sims[k]) ? graph : host_only).push_back(k);
  }
  std::thread helper([&] { run_threads(b, host_only, left.data(), 1, st); });
  std::stable_sort(graph.begin(), graph.end(), [&](int p, int q) {
    return b->cells[p] * (double)left[p] > b->cells[q] * (double)left[q];
  });
  std::vector<int> queued;
  for (int k : graph) {
    st[k] = crp::sim_graphs_enqueue(b->sims[k], left[k]);
    if (st[k] == CRP_OK) queued.push_back(k);
    else if (st[k] == CRP_ERR_UNSUPPORTED) st[k] = crp_step(b->sims[k], left[k]);  // graph capture refused
  }
  for (int k : queued) st[k] = crp::sim_graphs_finish(b->sims[k]);
  helper.join();
}

crp_status apply_sim_tuning(crp_batch* b, const crp_batch_tuning& t) {
  for (size_t k = 0; k < b->sims.size(); k++) {
    crp_tuning s{};
    crp_status r = crp_get_tuning(b->sims[k], &s);
    if (r != CRP_OK) return r;
    s.fdtd_rows = t.fdtd_rows;
    const long lanes = (long)kRpLaneThreads * std::max(1, t.rp_bubbles_per_lane);
    s.rp_blocks = t.rp_bubbles_per_lane <= 1 ? 0 : (int32_t)std::max(1L, (b->nb[k] + lanes - 1) / lanes);
    r = crp_set_tuning(b->sims[k], &s);
    if (r != CRP_OK) return r;
  }
  return CRP_OK;
}

bool valid(const crp_batch_tuning& t) {
  return (t.mode == CRP_BATCH_THREADS || t.mode == CRP_BATCH_GRAPHS) && t.threads >= 0 &&
         (t.blocking == 0 || t.blocking == 1) &&
         (t.fdtd_rows == 4 || t.fdtd_rows == 8 || t.fdtd_rows == 16) && t.rp_bubbles_per_lane >= 1;
}

crp_status run_with(crp_batch* b, const int32_t* steps, const crp_batch_tuning& t, crp_status* per_sim) {
  const int n = (int)b->sims.size();
  std::vector<crp_status> st(n, CRP_OK);
  if (t.mode == CRP_BATCH_GRAPHS) {
    run_graphs(b, steps, st);
  } else {
    // Each simulation as its own configuration asks (ext.graphs).
    for (crp_sim* s : b->sims) {
      crp::sim_allow_graphs(s, crp::sim_config(s).ext_graphs != 0);
      const crp_status r = crp::sim_blocking_waits(s, t.blocking != 0);
      if (r != CRP_OK) return r;
    }
    std::vector<int> all(n);
    std::iota(all.begin(), all.end(), 0);
    run_threads(b, all, steps, t.threads, st);
  }
  crp_status first = CRP_OK;
  for (int k = 0; k < n; k++) {
    if (per_sim) per_sim[k] = st[k];
    if (first == CRP_OK && st[k] != CRP_OK) first = st[k];
  }
  return first;
}

}  // namespace

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
    double cells = (double)cfgs[k].grid_x * (double)cfgs[k].grid_y;
    if (cfgs[k].ext_grid_z > 0) cells *= (double)cfgs[k].ext_grid_z;
    b->cells.push_back(cells);
    crp_dims d{};
    crp_get_dims(s, &d);
    b->nb.push_back(d.num_bubbles);
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
  crp_batch_tuning t = b->tuning;
  if (threads > 0) {
    t.mode = CRP_BATCH_THREADS;
    t.threads = threads;
  }
  return run_with(b, steps, t, per_sim);
}

crp_status crp_batch_get_tuning(const crp_batch* b, crp_batch_tuning* t) {
  if (!b || !t) return CRP_ERR_INVALID;
  *t = b->tuning;
  return CRP_OK;
}

crp_status crp_batch_set_tuning(crp_batch* b, const crp_batch_tuning* t) {
  if (!b || !t || !valid(*t)) return CRP_ERR_INVALID;
  const crp_status r = apply_sim_tuning(b, *t);
  if (r != CRP_OK) return r;
  b->tuning = *t;
  return CRP_OK;
}

crp_status crp_batch_tune(crp_batch* b, int32_t trial_steps, crp_batch_tuning* best, crp_batch_tuning* tried,
                          int32_t capacity, int32_t* n_tried) {
  if (!b || trial_steps <= 0) return CRP_ERR_INVALID;
  const int n = (int)b->sims.size();
  std::vector<crp_state*> saved(n, nullptr);
  auto release = [&]() {
    for (crp_state* s : saved) crp_state_free(s);
  };
  for (int k = 0; k < n; k++) {
    const crp_status r = crp_save_state(b->sims[k], &saved[k]);
    if (r != CRP_OK) {
      release();
      return r;
    }
  }
  auto restore = [&]() -> crp_status {
    for (int k = 0; k < n; k++) {
      const crp_status r = crp_load_state(b->sims[k], saved[k]);
      if (r != CRP_OK) return r;
    }
    return CRP_OK;
  };
  int count = 0;
  const std::vector<int32_t> warm(n, 2), timed(n, trial_steps);
  // One trial: the setting applied, two untimed steps (graph builds, first
  // steps), then trial_steps timed on the wall clock; the state restored.
  auto trial = [&](crp_batch_tuning& t) -> crp_status {
    crp_status r = apply_sim_tuning(b, t);
    if (r == CRP_OK) r = run_with(b, warm.data(), t, nullptr);
    double ms = 0.0;
    if (r == CRP_OK) {
      const auto t0 = std::chrono::steady_clock::now();
      r = run_with(b, timed.data(), t, nullptr);
      ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    const crp_status rs = restore();
    if (rs != CRP_OK) return rs;
    // A trial whose simulations failed (e.g. a Picard cap in the trial steps) is not a candidate.
    t.ms_per_step = r == CRP_OK ? ms / trial_steps : 0.0;
    if (tried && count < capacity) tried[count] = t;
    count++;
    return CRP_OK;
  };
  crp_batch_tuning cur{CRP_BATCH_THREADS, 0, 0, 8, 1, 0.0};
  crp_status r = trial(cur);
  auto better = [](const crp_batch_tuning& a, const crp_batch_tuning& c) {
    return a.ms_per_step > 0.0 && (c.ms_per_step <= 0.0 || a.ms_per_step < c.ms_per_step);
  };
  // One parameter at a time from the defaults: mode, host threads and their
  // waits, rows, radius lanes.
  for (int m : {CRP_BATCH_GRAPHS}) {
    if (r != CRP_OK) break;
    crp_batch_tuning c = cur;
    c.mode = m;
    r = trial(c);
    if (r == CRP_OK && better(c, cur)) cur = c;
  }
  if (cur.mode == CRP_BATCH_THREADS) {
    for (int th : {n, 16}) {
      if (r != CRP_OK || th == std::min(n, 32)) continue;
      crp_batch_tuning c = cur;
      c.threads = th;
      r = trial(c);
      if (r == CRP_OK && better(c, cur)) cur = c;
    }
    if (r == CRP_OK) {
      crp_batch_tuning c = cur;
      c.blocking = 1;
      r = trial(c);
      if (r == CRP_OK && better(c, cur)) cur = c;
    }
  }
  for (int rows : {4, 16}) {
    if (r != CRP_OK) break;
    crp_batch_tuning c = cur;
    c.fdtd_rows = rows;
    r = trial(c);
    if (r == CRP_OK && better(c, cur)) cur = c;
  }
  for (int lanes : {4, 16}) {
    if (r != CRP_OK) break;
    crp_batch_tuning c = cur;
    c.rp_bubbles_per_lane = lanes;
    r = trial(c);
    if (r == CRP_OK && better(c, cur)) cur = c;
  }
  release();
  if (n_tried) *n_tried = count;
  if (r != CRP_OK) {
    apply_sim_tuning(b, b->tuning);
    return r;
  }
  r = apply_sim_tuning(b, cur);
  if (r != CRP_OK) return r;
  b->tuning = cur;
  if (best) *best = cur;
  return CRP_OK;
}

void crp_batch_destroy(crp_batch* b) {
  if (!b) return;
  for (crp_sim* s : b->sims) crp_destroy(s);
  delete b;
}

}  // extern "C"
