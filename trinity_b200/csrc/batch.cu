/*
 * batch.cu — many independent meshes at once (the batched workload).
 *
 * trinity adapts one mesh per process; a batch of meshes of uneven size is
 * adapted here concurrently on one GPU: every mesh has its own CUDA stream,
 * and a pool of host threads drives the meshes (largest first) through metric
 * recovery and the rounds, so that the launch- and synchronisation-bound
 * phases of small meshes overlap with the compute of large ones. With
 * TRN_BATCH_GRAPH each round is the mesh's captured round (one graph launch,
 * no host round trip inside). Meshes share nothing on the device; no host
 * lock is held while a mesh runs.
 */
#include "../../include/trinity_b200.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

extern "C" int trn_batch_adapt(trn_mesh* const* meshes, int count, double target_factor, int lp_norm,
                               double h_min, double h_max, int rounds, int depth, int threads,
                               double* round_ms, long long* tri_in) {
  return trn_batch_adapt_ex(meshes, count, target_factor, lp_norm, h_min, h_max, rounds, depth, threads,
                            0, round_ms, tri_in);
}

extern "C" int trn_batch_adapt_ex(trn_mesh* const* meshes, int count, double target_factor, int lp_norm,
                                  double h_min, double h_max, int rounds, int depth, int threads,
                                  int flags, double* round_ms, long long* tri_in) {
  const bool graph = (flags & TRN_BATCH_GRAPH) != 0;
  if (!meshes || count <= 0 || rounds < 0 || depth < 1) return TRN_ERR_INVALID;
  for (int i = 0; i < count; ++i)
    if (!meshes[i]) return TRN_ERR_INVALID;
  std::vector<int> size(count), order(count);
  for (int i = 0; i < count; ++i) {
    int n = 0, e = 0;
    trn_mesh_counts(meshes[i], &n, &e, nullptr, nullptr);
    size[i] = e;
  }
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return size[a] > size[b]; });
  const int nthreads = std::max(1, std::min(threads > 0 ? threads : 8, count));
  std::atomic<int> next{0};
  std::atomic<int> status{TRN_OK};

  auto worker = [&]() {
    for (;;) {
      if (status.load() != TRN_OK) return;
      const int k = next.fetch_add(1);
      if (k >= count) return;
      const int i = order[k];
      trn_mesh* m = meshes[i];
      int rc = trn_metric_run(m, target_factor, lp_norm, h_min, h_max, nullptr);
      double ms = 0.0;
      long long tin = 0;
      for (int r = 0; r < rounds && rc == TRN_OK; ++r) {
        int live = 0;
        rc = trn_mesh_counts(m, nullptr, nullptr, nullptr, &live);
        tin += live;
        if (graph) {
          if (rc == TRN_OK) rc = trn_round_graph_run(m, depth, nullptr);
          if (rc == TRN_OK) ms += trn_last_time_ms(m);
          continue;
        }
        if (rc == TRN_OK) rc = trn_refine_run(m, depth, nullptr);
        if (rc == TRN_OK) ms += trn_last_time_ms(m), rc = trn_coarsen_run(m, 8, nullptr);
        if (rc == TRN_OK) ms += trn_last_time_ms(m), rc = trn_swap_run(m, nullptr);
        if (rc == TRN_OK) ms += trn_last_time_ms(m), rc = trn_smooth_run(m, 8, depth, nullptr);
        if (rc == TRN_OK) ms += trn_last_time_ms(m);
      }
      if (round_ms) round_ms[i] = ms;
      if (tri_in) tri_in[i] = tin;
      if (rc != TRN_OK) {
        int expected = TRN_OK;
        status.compare_exchange_strong(expected, rc);
        return;
      }
    }
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < nthreads; ++t) pool.emplace_back(worker);
  for (auto& t : pool) t.join();
  return status.load();
}
