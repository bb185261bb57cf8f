/*
 * heuristics.cu — the graph heuristics of the free (non-replay) mode.
 *
 * The reference resolves conflicts with a speculative first-fit coloring
 * (partition.cpp:79-306, independent set = color 1) and a Karp-Sipser-like
 * greedy matching (matching.cpp:81-135), both sequential in spirit. On the GPU
 * these become round-synchronous algorithms with seeded hash priorities:
 *
 *   mis_jp_rounds   independent set on the collapse candidates, a fixed
 *                   number of rounds per level: a candidate joins when it has
 *                   the highest hash priority of the round among its undecided
 *                   candidate neighbours and leaves when a neighbour joined
 *                   (Jones-Plassmann / Luby); candidates still undecided after
 *                   the last round are examined again at the next level.
 *   match_handshake maximal matching on the swap dual rows: every unmatched
 *                   candidate points along its heaviest free edge; mutual
 *                   candidate pairs match, a non-candidate neighbour accepts
 *                   its heaviest proposer. Edges weigh, by default, their
 *                   slot in the row (the reference's greedy takes each
 *                   candidate's first free neighbour in row order, and
 *                   uniform random weights leave the final mesh with
 *                   measurably more edges of metric length 1.2-1.4), or, on
 *                   request, the quality their flip gains, which gives a
 *                   better mesh than the reference's; ties break by a
 *                   symmetric hash.
 *   color_jp        speculative first-fit coloring of the interior vertices
 *                   with colors 1..max_col: tentative colors, kept unless a
 *                   higher-priority neighbour wants the same one (the
 *                   reference's speculative coloring made round-synchronous
 *                   and deterministic); a vertex left without a free color
 *                   is not smoothed, as in the reference. Each class lists
 *                   its vertices grouped by stencil length.
 */
#include "trn_internal.h"

#include <algorithm>
#include <cstdio>

namespace trn {

/* ---------------- persistent rounds ----------------
 * A round-synchronous heuristic runs as one cooperative launch (all blocks
 * resident at once, which cudaLaunchCooperativeKernel guarantees) whose
 * rounds are separated by a grid barrier, instead of one launch per round.
 * The barrier is a counter and a generation word: each block's thread 0
 * notes the generation, arrives, and the last to arrive resets the counter
 * and advances the generation, which the others poll. The poll is bounded:
 * past kBarrierPolls it records a failure in the barrier and in the mesh's
 * error word and the block leaves the kernel (the host then reports
 * TRN_ERR_NO_PROGRESS), so no wait can outlive a fault elsewhere. Used for
 * calls that are not being captured into a graph; a captured round keeps the
 * per-round launches. */
struct GridBar {
  unsigned count;
  unsigned gen;
  int err;
};
constexpr long long kBarrierPolls = 1LL << 24;

__device__ __forceinline__ bool grid_sync(GridBar* b, int* mesh_err, long long max_polls = kBarrierPolls) {
  __syncthreads();
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    volatile unsigned* vgen = &b->gen;
    volatile int* verr = &b->err;
    const unsigned g = *vgen;
    __threadfence();
    int ok = 1;
    if (atomicAdd(&b->count, 1u) == gridDim.x - 1) {
      b->count = 0;
      __threadfence();
      atomicAdd(&b->gen, 1u);
    } else {
      long long polls = 0;
      while (*vgen == g) {
        if (*verr || ++polls > max_polls) {
          atomicExch(&b->err, 1);
          trn_set_error(mesh_err, TRN_DERR_NO_PROGRESS);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    s_ok = ok && !*verr;
  }
  __syncthreads();
  return s_ok != 0;
}

/* the workspace's barrier, cleared before each cooperative launch (a
 * barrier that gave up keeps its arrivals and failure mark) */
static GridBar* grid_bar(HeurWs& ws, cudaStream_t s) {
  GridBar* b = reinterpret_cast<GridBar*>(ws.cnt + 100);
  cudaMemsetAsync(b, 0, sizeof(GridBar), s);
  return b;
}

/* A cooperative launch whose first block never reaches the barrier: the
 * others wait max_polls polls, give up and mark the error word (the bounded
 * wait's failure path, for the tests). */
__global__ void k_barrier_selftest(GridBar* bar, int* err, long long max_polls) {
  if (blockIdx.x == 0) return;
  grid_sync(bar, err, max_polls);
}

/* a cooperative launch of `kernel` with as many blocks of `threads` as fit
 * on the device at once (and no more than the items need); false when it
 * could not launch (the caller then takes the per-round launches). Large
 * blocks keep the barrier's arrivals few (two 1024-thread blocks an SM: 296
 * arrivals a round on 148 SMs). */
template <class K, class... Args>
static bool coop_launch(K kernel, long long items, int threads, cudaStream_t s, Args... args) {
  int dev = 0, sms = 0, coop = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
  if (!coop || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) != cudaSuccess ||
      per_sm <= 0)
    return false;
  cudaStreamCaptureStatus cs;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return false;
  const long long need = (items + threads - 1) / threads;
  const int grid = (int) std::max(1LL, std::min<long long>((long long) per_sm * sms, need));
  void* argv[] = {static_cast<void*>(&args)...};
  if (cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kernel), grid, threads, argv, 0, s) !=
      cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  note_launch();
  return true;
}

/* ---------------- independent set ---------------- */




/* free-mode round over a device-counted candidate list; states are read
 * from the previous round's buffer only (0 out / not a candidate,
 * 1 undecided, 2 in the set), so the outcome does not depend on timing */
__device__ __forceinline__ uint8_t mis_item(const DMesh& m, const uint8_t* __restrict__ in,
                                            uint8_t* __restrict__ out, int v, uint64_t seed) {
  const uint8_t sv = in[v];
  if (sv != 1) {
    out[v] = sv;
    return sv;
  }
  const uint64_t pv = trn_prio(seed, v);
  const int* vc = m.vic + (size_t) v * m.bucket;
  const int nv = m.vdeg[v];
  bool is_max = true, leave = false;
  for (int b = 0; b < nv; ++b) {
    const int w = vc[b];
    const uint8_t sw = in[w];
    if (sw == 2) { leave = true; break; }
    if (sw == 1 && trn_prio(seed, w) > pv) is_max = false;
  }
  const uint8_t st = leave ? 0 : (is_max ? 2 : 1);
  out[v] = st;
  return st;
}

/* collect the set; candidates still undecided are re-activated so that the
 * next level examines them again; every candidate's state returns to 0 */
__device__ __forceinline__ void mis_finish_item(const DMesh& m, uint8_t* state, uint8_t* other, int v,
                                                int* indep, int* nindep) {
  const uint8_t st = state[v];
  if (st == 2) trn_append(indep, nindep, v);
  else if (st == 1) trn_activate(m, v);
  state[v] = 0;
  other[v] = 0;
}

__global__ void k_mis_round_dev(DMesh m, const uint8_t* __restrict__ in, uint8_t* __restrict__ out,
                                const int* __restrict__ cand, const int* count, Seed sd,
                                uint64_t round_mix, int min_n) {
  if (trn_failed(m)) return;
  const uint64_t seed = trn_seed(sd) + round_mix;
  const int n = *count;
  if (n < min_n) return;
  for (int q = trn_tid(); q < n; q += trn_grid_stride()) mis_item(m, in, out, cand[q], seed);
}

__global__ void k_mis_finish(DMesh m, uint8_t* state, uint8_t* other, const int* __restrict__ cand,
                             const int* count, int* indep, int* nindep, int min_n) {
  const int n = *count;
  if (n < min_n) return;
  for (int q = trn_tid(); q < n; q += trn_grid_stride())
    mis_finish_item(m, state, other, cand[q], indep, nindep);
}

/* all the rounds and the collection in one block, the rounds separated by
 * block barriers: for a level whose list the host knows to be short, where
 * one launch per round would cost more than the round */
constexpr int kFusedThreads = 1024;

__global__ void __launch_bounds__(kFusedThreads) k_mis_fused(DMesh m, uint8_t* s0, uint8_t* s1,
                                                             const int* __restrict__ cand,
                                                             const int* count, Seed sd, int rounds,
                                                             int* indep, int* nindep, int max_n) {
  if (trn_failed(m)) return;
  const int n = *count;
  if (n > max_n) return;
  if (threadIdx.x == 0) *nindep = 0;
  const uint64_t base = trn_seed(sd);
  for (int r = 0; r < rounds; ++r) {
    const uint8_t* in = (r & 1) ? s1 : s0;
    uint8_t* out = (r & 1) ? s0 : s1;
    const uint64_t seed = base + 0x9e3779b97f4a7c15ULL * r;
    for (int q = threadIdx.x; q < n; q += blockDim.x) mis_item(m, in, out, cand[q], seed);
    __syncthreads();
  }
  uint8_t* state = (rounds & 1) ? s1 : s0;
  uint8_t* other = (rounds & 1) ? s0 : s1;
  for (int q = threadIdx.x; q < n; q += blockDim.x) mis_finish_item(m, state, other, cand[q], indep, nindep);
}

/* all the rounds and the collection in one cooperative launch (stopping
 * the rounds once no candidate is undecided was measured slower: the
 * undecided flag's reduction costs more on the long levels than the rounds
 * it saves on the short ones) */
__global__ void __launch_bounds__(kFusedThreads) k_mis_persist(DMesh m, uint8_t* s0, uint8_t* s1,
                                                               const int* __restrict__ cand, const int* count,
                                                               Seed sd, int rounds, int* indep, int* nindep,
                                                               GridBar* bar) {
  if (trn_failed_block(m)) return;
  const int n = *count;
  if (trn_tid() == 0) *nindep = 0;
  const uint64_t base = trn_seed(sd);
  for (int r = 0; r < rounds; ++r) {
    const uint8_t* in = (r & 1) ? s1 : s0;
    uint8_t* out = (r & 1) ? s0 : s1;
    const uint64_t seed = base + 0x9e3779b97f4a7c15ULL * r;
    for (int q = trn_tid(); q < n; q += trn_grid_stride()) mis_item(m, in, out, cand[q], seed);
    if (!grid_sync(bar, m.err)) return;
  }
  uint8_t* state = (rounds & 1) ? s1 : s0;
  uint8_t* other = (rounds & 1) ? s0 : s1;
  for (int q = trn_tid(); q < n; q += trn_grid_stride()) mis_finish_item(m, state, other, cand[q], indep, nindep);
}

void mis_jp_rounds(const DMesh& m, const int* cand, const int* count, int rounds, Seed sd,
                   HeurWs& ws, int* indep, int* nindep, cudaStream_t s, long long bound) {
  ProfScope ps("mis_jp", s, 0.0);
  uint8_t* buf[2] = {ws.state, ws.state2};
  if (bound > kFusedThreads &&
      coop_launch(k_mis_persist, bound, kFusedThreads, s, m, buf[0], buf[1], cand, count, sd, rounds, indep,
                  nindep, grid_bar(ws, s))) {
    check_launch("mis_jp_rounds");
    return;
  }
  if (bound >= 0 && bound <= kFusedThreads) {   /* known short: the one-block form only */
    k_mis_fused<<<1, kFusedThreads, 0, s>>>(m, buf[0], buf[1], cand, count, sd, rounds, indep, nindep,
                                            kFusedThreads);
    note_launch();
    check_launch("mis_jp_rounds");
    return;
  }
  /* known long: the per-round launches only; unknown (a captured round):
   * both, each form returning at once when the device count is not its case
   * (the one-block form last, as it clears the count it fills) */
  const int g = grid_bounded(bound, m.capa_node);
  const int min_n = bound < 0 ? kFusedThreads + 1 : 0;
  for (int r = 0; r < rounds; ++r) {
    k_mis_round_dev<<<TRN_RESIDENT(k_mis_round_dev, g, TRN_THREADS), TRN_THREADS, 0, s>>>(m, buf[r & 1], buf[(r + 1) & 1], cand, count, sd,
                                               0x9e3779b97f4a7c15ULL * r, min_n);
    note_launch();
  }
  cudaMemsetAsync(nindep, 0, sizeof(int), s);
  k_mis_finish<<<g, TRN_THREADS, 0, s>>>(m, buf[rounds & 1], buf[(rounds + 1) & 1], cand, count, indep,
                                         nindep, min_n);
  note_launch();
  if (bound < 0) {
    k_mis_fused<<<1, kFusedThreads, 0, s>>>(m, buf[0], buf[1], cand, count, sd, rounds, indep, nindep,
                                            kFusedThreads);
    note_launch();
  }
  check_launch("mis_jp_rounds");
}

/* ---------------- matching ---------------- */
static constexpr int kMatchRounds = 4;

/* The rank of dual edge (row i, slot q) in the upper bits of its weight, and
 * the mask of the lower bits a hash fills. Row order (rank == nullptr): the
 * slot of the edge in the row of its lower-id candidate end, first slots
 * first, as the reference's greedy takes each candidate's first free
 * neighbour. Gain: rank[4 i + q], the quantized quality change of the flip.
 * Both ends of an edge between two candidates compute the same rank. */
__device__ __forceinline__ uint32_t edge_rank(const int* __restrict__ dual, const int* __restrict__ dual_n,
                                              const uint32_t* __restrict__ rank, const int* __restrict__ map,
                                              int ntasks, int i, int q, uint32_t* low) {
  if (rank) {
    *low = 0x3ffu;
    return rank[i * 4 + q];
  }
  const int c = dual[i * 4], n = dual[i * 4 + q];
  int pos = q;
  if (n < c) {
    const int x = map[n];
    if (x >= 0 && x < ntasks && dual[x * 4] == n)
      for (int e = 1; e < dual_n[x]; ++e)
        if (dual[x * 4 + e] == c) pos = e;
  }
  *low = 0x3fffffffu;
  return (uint32_t) (4 - pos) << 30;
}

/* the weight of dual edge (row i, slot q): its rank, then a symmetric hash of
 * the pair, so equal ranks break ties at random and the edge weighs the same
 * from both ends */
__device__ __forceinline__ uint32_t edge_weight(const int* __restrict__ dual, const int* __restrict__ dual_n,
                                                const uint32_t* __restrict__ rank, const int* __restrict__ map,
                                                int ntasks, int i, int q, uint64_t seed, int round) {
  const int a = dual[i * 4], b = dual[i * 4 + q];
  const int lo = a < b ? a : b, hi = a < b ? b : a;
  const uint64_t h = trn_hash64(seed ^ ((uint64_t) (uint32_t) lo << 32 | (uint32_t) hi) ^
                                ((uint64_t) round * 0xd1b54a32d192ed03ULL));
  uint32_t low;
  const uint32_t r = edge_rank(dual, dual_n, rank, map, ntasks, i, q, &low);
  return (r & ~low) | ((uint32_t) (h >> 32) & low) | 1u;
}

struct MatchArgs {
  const int* dual;
  const int* dual_n;
  const uint32_t* rank;   /* gain ranks, or nullptr for row order */
  const int* map;
  int* mate;
  unsigned long long* prop;
  int* choice;
};

__device__ __forceinline__ void match_reset_item(const MatchArgs& a, int i) {
  for (int q = 0; q < a.dual_n[i]; ++q) {
    const int e = a.dual[i * 4 + q];
    a.mate[e] = -1;
    a.prop[e] = 0ULL;
  }
}

__device__ __forceinline__ void match_propose_item(const MatchArgs& a, int ntasks, int i, uint64_t seed,
                                                   int round) {
  const int c = a.dual[i * 4];
  int best = -1;
  uint32_t bw = 0;
  if (a.mate[c] == -1) {
    for (int q = 1; q < a.dual_n[i]; ++q) {
      const int n = a.dual[i * 4 + q];
      if (a.mate[n] != -1) continue;
      const uint32_t w = edge_weight(a.dual, a.dual_n, a.rank, a.map, ntasks, i, q, seed, round);
      if (w > bw) { bw = w; best = n; }
    }
    if (best >= 0) atomicMax(a.prop + best, ((unsigned long long) bw << 32) | (uint32_t) c);
  }
  a.choice[i] = best;
}

/* a mutual choice between two candidates, or a non-candidate's heaviest
 * proposer, is a match */
__device__ __forceinline__ void match_accept_item(const MatchArgs& a, int ntasks, int i, uint64_t seed,
                                                  int round, int* pairs, int* npairs) {
  const int n = a.choice[i];
  if (n < 0) return;
  const int c = a.dual[i * 4];
  const int x = a.map[n];
  const bool n_cand = x >= 0 && x < ntasks && a.dual[x * 4] == n;
  bool ok;
  if (n_cand) {
    ok = (a.choice[x] == c) && (c < n);
  } else {
    int q = 1;
    while (q < a.dual_n[i] - 1 && a.dual[i * 4 + q] != n) ++q;
    const uint32_t w = edge_weight(a.dual, a.dual_n, a.rank, a.map, ntasks, i, q, seed, round);
    ok = a.prop[n] == (((unsigned long long) w << 32) | (uint32_t) c);
  }
  if (ok) {
    a.mate[c] = n;
    a.mate[n] = c;
    const int p = trn_warp_reserve(npairs);
    pairs[2 * p] = c;
    pairs[2 * p + 1] = n;
  }
}

__device__ __forceinline__ void match_clear_item(const MatchArgs& a, int i) {
  for (int q = 1; q < a.dual_n[i]; ++q) a.prop[a.dual[i * 4 + q]] = 0ULL;
}

__global__ void k_match_reset(MatchArgs a, const int* ntasks_dev, int min_n) {
  const int ntasks = *ntasks_dev;
  if (ntasks < min_n) return;
  for (int i = trn_tid(); i < ntasks; i += trn_grid_stride()) match_reset_item(a, i);
}

__global__ void k_match_propose(MatchArgs a, const int* ntasks_dev, Seed sd, int round, int min_n) {
  const int ntasks = *ntasks_dev;
  if (ntasks < min_n) return;
  const uint64_t seed = trn_seed(sd);
  for (int i = trn_tid(); i < ntasks; i += trn_grid_stride()) match_propose_item(a, ntasks, i, seed, round);
}

__global__ void k_match_accept(MatchArgs a, const int* ntasks_dev, Seed sd, int round, int* pairs,
                               int* npairs, int min_n) {
  const int ntasks = *ntasks_dev;
  if (ntasks < min_n) return;
  const uint64_t seed = trn_seed(sd);
  for (int i = trn_tid(); i < ntasks; i += trn_grid_stride())
    match_accept_item(a, ntasks, i, seed, round, pairs, npairs);
}

__global__ void k_match_prop_clear(MatchArgs a, const int* ntasks_dev, int min_n) {
  const int ntasks = *ntasks_dev;
  if (ntasks < min_n) return;
  for (int i = trn_tid(); i < ntasks; i += trn_grid_stride()) match_clear_item(a, i);
}

/* the whole handshake in one block (reset, then propose / accept / clear per
 * round, separated by block barriers), for levels the host knows to be short */
__global__ void __launch_bounds__(kFusedThreads) k_match_fused(MatchArgs a, const int* ntasks_dev, Seed sd,
                                                               int* pairs, int* npairs, int max_n) {
  const int ntasks = *ntasks_dev;
  if (ntasks > max_n) return;
  const uint64_t seed = trn_seed(sd);
  if (threadIdx.x == 0) *npairs = 0;
  for (int i = threadIdx.x; i < ntasks; i += blockDim.x) match_reset_item(a, i);
  __syncthreads();
  for (int r = 0; r < kMatchRounds; ++r) {
    for (int i = threadIdx.x; i < ntasks; i += blockDim.x) match_propose_item(a, ntasks, i, seed, r);
    __syncthreads();
    for (int i = threadIdx.x; i < ntasks; i += blockDim.x) match_accept_item(a, ntasks, i, seed, r, pairs, npairs);
    __syncthreads();
    for (int i = threadIdx.x; i < ntasks; i += blockDim.x) match_clear_item(a, i);
    __syncthreads();
  }
}

void match_handshake(const DMesh& m, int nb_elems, const int* dual, const int* dual_n,
                     const int* ntasks, const int* map, const uint32_t* rank, Seed seed, HeurWs& ws,
                     int* pairs, int* npairs, cudaStream_t s, long long bound) {
  (void) m;
  ProfScope ps("match_handshake", s, 0.0);
  const MatchArgs a{dual, dual_n, rank, map, ws.mate, ws.prop, ws.choice};
  if (bound >= 0 && bound <= kFusedThreads) {   /* known short: the one-block form only */
    k_match_fused<<<1, kFusedThreads, 0, s>>>(a, ntasks, seed, pairs, npairs, kFusedThreads);
    note_launch();
    check_launch("match_handshake");
    return;
  }
  /* as in mis_jp_rounds: both forms when the length is unknown */
  const int g = grid_bounded(bound, nb_elems);
  const int min_n = bound < 0 ? kFusedThreads + 1 : 0;
  cudaMemsetAsync(npairs, 0, sizeof(int), s);
  k_match_reset<<<g, TRN_THREADS, 0, s>>>(a, ntasks, min_n);
  note_launch();
  for (int r = 0; r < kMatchRounds; ++r) {
    k_match_propose<<<g, TRN_THREADS, 0, s>>>(a, ntasks, seed, r, min_n);
    note_launch();
    k_match_accept<<<g, TRN_THREADS, 0, s>>>(a, ntasks, seed, r, pairs, npairs, min_n);
    note_launch();
    k_match_prop_clear<<<g, TRN_THREADS, 0, s>>>(a, ntasks, min_n);
    note_launch();
  }
  if (bound < 0) {
    k_match_fused<<<1, kFusedThreads, 0, s>>>(a, ntasks, seed, pairs, npairs, kFusedThreads);
    note_launch();
  }
  check_launch("match_handshake");
}

/* ---------------- greedy matching in interleaved element order ----------------
 *
 * The reference's matching (Match::computeGreedyMatching / matchAndUpdate,
 * matching.cpp:81-135) is a loop over the dual rows in list order, i.e. in
 * increasing candidate id: a row whose candidate is still free marks it
 * taken, then takes its free neighbours in slot order, going past each
 * neighbour that is not itself a candidate (the "continue" of
 * matching.cpp:124) and stopping at the first one that is; the candidate's
 * partner is the last neighbour taken. This is that loop without the
 * degree-1 stack, over the rows in the order (id mod 4, id): four
 * interleaved sweeps of the candidate ids.
 *
 * Its result is computed exactly, in parallel, as the greedy matching of an
 * order is: in each round a row decides once it comes first, under that
 * order, among the undecided rows that list any of its elements; such rows
 * share no element with one another, so they decide independently, and what
 * each finds is what the sequential loop would have found. Rows propose
 * their key with a 64-bit atomicMin on every element of their row into the
 * round's buffer (keys of later rounds compare lower, so no buffer needs
 * clearing between rounds); a row is ready when every element holds its own
 * key. A round decides the ready rows and lets the others propose for the
 * next round into the other buffer, so one launch per round. The rounds
 * run over a compacted list of the undecided rows; once that list is short
 * one block finishes the remaining rounds with block barriers. After
 * kGreedyRounds rounds any row still undecided stays unmatched (a valid, if
 * not maximal, matching). On the 2M-triangle workload the deepest level
 * needs 48 rounds, the mean is 12.
 *
 * The four-way interleave keeps the chains of dependent rows short (a plain
 * increasing-id sweep has chains as long as a row of the grid), and the
 * final meshes' metric edge-length histograms stay within half a point per
 * bin of the reference's, where a maximal handshake matching, which flips
 * more pairs, is a point and a half off. */
constexpr int kGreedyRounds = 64;
constexpr int kGreedyTail = 2048;   /* undecided rows left to the one-block rounds */
/* rows waiting above which a round runs as its own grid launch (measured:
 * such rounds are faster launched than inside the cooperative kernel) */
constexpr int kGreedyGrid = 1 << 15;

struct GreedyArgs {
  const int* dual;
  const int* dual_n;
  const int* map;
  int* vis;                 /* per element: -1 free, else taken */
  unsigned long long* mk0;  /* per element: lowest key proposed, even rounds */
  unsigned long long* mk1;  /* odd rounds */
  int* list0;               /* undecided rows, even rounds */
  int* list1;
  int* cnt;                 /* [3] list lengths, by round mod 3 */
  int* ran;                 /* [kGreedyRounds] round r ran on the grid */
};

__device__ __forceinline__ unsigned long long greedy_key(int r, int c) {
  return ((unsigned long long) (kGreedyRounds - r) << 40) | ((unsigned long long) (c & 3) << 32) |
         (uint32_t) c;
}

/* "is a candidate" as matching.cpp:124 asks it: the element has a row in the
 * map, which keeps the rows of earlier levels of the same call (it is reset
 * once per call, swapping.cpp:161-162) */
__device__ __forceinline__ bool greedy_is_row(const GreedyArgs& a, int ntasks, int e) {
  (void) ntasks;
  return a.map[e] >= 0;
}


__device__ __forceinline__ void greedy_propose(const GreedyArgs& a, int r, int i) {
  unsigned long long* mk = (r & 1) ? a.mk1 : a.mk0;
  const unsigned long long key = greedy_key(r, a.dual[i * 4]);
  for (int q = 0; q < a.dual_n[i]; ++q) atomicMin(mk + a.dual[i * 4 + q], key);
}

/* is row i first on all its elements in round r? The loads of the row's
 * slots past its length read slot 0 again (always there), so that every
 * load can be issued before any compare */
__device__ __forceinline__ bool greedy_ready(const GreedyArgs& a, int r, int i) {
  const unsigned long long* mk = (r & 1) ? a.mk1 : a.mk0;
  const int4 row = reinterpret_cast<const int4*>(a.dual)[i];
  const int dn = a.dual_n[i];
  const unsigned long long key = greedy_key(r, row.x);
  const unsigned long long k0 = mk[row.x], k1 = mk[dn > 1 ? row.y : row.x];
  const unsigned long long k2 = mk[dn > 2 ? row.z : row.x], k3 = mk[dn > 3 ? row.w : row.x];
  return k0 == key && k1 == key && k2 == key && k3 == key;
}

/* row i in round r, its readiness known: decide it when it is first on all
 * its elements (and return false), else propose it for round r + 1 (and
 * return true) */
__device__ __forceinline__ bool greedy_act(const GreedyArgs& a, int ntasks, int r, int i, bool ready,
                                           int* pairs, int* npairs) {
  const int c = a.dual[i * 4];
  const int dn = a.dual_n[i];
  if (!ready) {
    greedy_propose(a, r + 1, i);
    return true;
  }
  if (a.vis[c] != -1) return false;
  a.vis[c] = 1;
  int partner = -1;
  for (int q = 1; q < dn; ++q) {
    const int n = a.dual[i * 4 + q];
    if (a.vis[n] != -1) continue;
    a.vis[n] = 1;
    partner = n;
    if (greedy_is_row(a, ntasks, n)) break;
  }
  if (partner >= 0) {
    const int p = trn_warp_reserve(npairs);
    pairs[2 * p] = c;
    pairs[2 * p + 1] = partner;
  }
  return false;
}

__device__ __forceinline__ bool greedy_item(const GreedyArgs& a, int ntasks, int r, int i, int* pairs,
                                            int* npairs) {
  return greedy_act(a, ntasks, r, i, greedy_ready(a, r, i), pairs, npairs);
}


/* round 0's proposals; every row starts undecided */
__global__ void k_greedy_start(GreedyArgs a, const int* ntasks_dev, int min_n) {
  const int ntasks = *ntasks_dev;
  if (ntasks < min_n) return;
  if (trn_tid() == 0) a.cnt[0] = ntasks;
  for (int i = trn_tid(); i < ntasks; i += trn_grid_stride()) {
    greedy_propose(a, 0, i);
    a.list0[i] = i;
  }
}

/* round r on the grid, while more than max(kGreedyTail, min_n - 1) rows
 * are undecided and every earlier round ran here */
__global__ void k_greedy_round(GreedyArgs a, const int* ntasks_dev, int r, int* pairs, int* npairs,
                               int min_n) {
  if (r > 0 && !a.ran[r - 1]) return;
  const int n = a.cnt[r % 3];
  if (n <= kGreedyTail || n < min_n) return;
  const int ntasks = *ntasks_dev;
  const int* in = (r & 1) ? a.list1 : a.list0;
  int* out = (r & 1) ? a.list0 : a.list1;
  if (trn_tid() == 0) {
    a.ran[r] = 1;
    a.cnt[(r + 2) % 3] = 0;   /* round r + 1's output */
  }
  for (int base = blockIdx.x * blockDim.x; base < n; base += trn_grid_stride()) {
    const int q = base + threadIdx.x;
    const int i = q < n ? in[q] : -1;
    const bool wait = q < n && greedy_item(a, ntasks, r, i, pairs, npairs);
    trn_block_append(out, a.cnt + (r + 1) % 3, i, wait);
  }
}

/* the remaining rounds in one block; with `whole`, the level's first
 * proposals too (a list the host knows to be short). The per-element state
 * starts reset: the dual filter reset it for the rows it built. */
__global__ void __launch_bounds__(kFusedThreads) k_greedy_tail(GreedyArgs a, const int* ntasks_dev,
                                                               int* pairs, int* npairs, int whole,
                                                               int lim) {
  const int ntasks = *ntasks_dev;
  if (whole ? ntasks > lim : ntasks < lim) return;
  __shared__ int s_r;
  if (whole) {
    if (threadIdx.x == 0) *npairs = 0;
    for (int i = threadIdx.x; i < ntasks; i += blockDim.x) {
      greedy_propose(a, 0, i);
      a.list0[i] = i;
    }
    if (threadIdx.x == 0) {
      a.cnt[0] = ntasks;
      a.cnt[1] = 0;
      s_r = 0;
    }
  } else if (threadIdx.x == 0) {
    int r = 0;
    while (r < kGreedyRounds && a.ran[r]) ++r;
    s_r = r;
  }
  __syncthreads();
  for (int r = s_r; r < kGreedyRounds; ++r) {
    const int n = a.cnt[r % 3];
    if (n == 0) break;
    const int* in = (r & 1) ? a.list1 : a.list0;
    int* out = (r & 1) ? a.list0 : a.list1;
    if (threadIdx.x == 0) a.cnt[(r + 2) % 3] = 0;
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
      const int i = in[q];
      if (greedy_item(a, ntasks, r, i, pairs, npairs)) {
        const int k = atomicAdd(a.cnt + (r + 1) % 3, 1);
        out[k] = i;
      }
    }
    __syncthreads();
  }
}

/* the matching of a level in one cooperative launch: with `whole`, the
 * first proposals (the dual filter reset the elements' state), then rounds
 * until no row waits (at most
 * kGreedyRounds); else the rounds from the first one the grid launches did
 * not run. Once kGreedyTail rows or fewer wait, the first block finishes the
 * rounds alone, separated by block barriers, and the others return: a grid
 * barrier costs more than such a round. */
__global__ void __launch_bounds__(kFusedThreads) k_greedy_persist(GreedyArgs a, const int* ntasks_dev,
                                                                  int* pairs, int* npairs, GridBar* bar,
                                                                  int* err, int whole) {
  const int ntasks = *ntasks_dev;
  int r0 = 0;
  if (whole) {
    if (trn_tid() == 0) {
      *npairs = 0;
      a.cnt[0] = ntasks;
      a.cnt[1] = 0;
      a.cnt[2] = 0;
    }
    for (int i = trn_tid(); i < ntasks; i += trn_grid_stride()) {
      greedy_propose(a, 0, i);
      a.list0[i] = i;
    }
    if (!grid_sync(bar, err)) return;
  } else {
    while (r0 < kGreedyRounds && a.ran[r0]) ++r0;
  }
  bool alone = false;
  for (int r = r0; r < kGreedyRounds; ++r) {
    const int n = *(volatile int*) (a.cnt + r % 3);
    if (n == 0) break;
    if (!alone && n <= kGreedyTail) {
      if (blockIdx.x != 0) return;
      alone = true;
    }
    const int* in = (r & 1) ? a.list1 : a.list0;
    int* out = (r & 1) ? a.list0 : a.list1;
    const int b0 = alone ? 0 : (int) (blockIdx.x * blockDim.x);
    const int bs = alone ? (int) blockDim.x : trn_grid_stride();
    if (b0 == 0 && threadIdx.x == 0) a.cnt[(r + 2) % 3] = 0;
    for (int base = b0; base < n; base += bs) {
      const int q = base + threadIdx.x;
      const int i = q < n ? in[q] : -1;
      const bool wait = q < n && greedy_item(a, ntasks, r, i, pairs, npairs);
      trn_block_append(out, a.cnt + (r + 1) % 3, i, wait);
    }
    if (alone) __syncthreads();
    else if (!grid_sync(bar, err)) return;
  }
}

void match_greedy(const DMesh& m, int nb_elems, const int* dual, const int* dual_n, const int* ntasks,
                  const int* map, HeurWs& ws, int* pairs, int* npairs, cudaStream_t s, long long bound) {
  (void) m;
  ProfScope ps("match_greedy", s, 0.0);
  const GreedyArgs a{dual, dual_n, map, ws.mate, ws.prop, ws.prop2, ws.choice, ws.choice2, ws.cnt,
                     ws.cnt + 8};
  if (bound >= 0 && bound <= kFusedThreads) {   /* known short: one block */
    k_greedy_tail<<<1, kFusedThreads, 0, s>>>(a, ntasks, pairs, npairs, 1, kFusedThreads);
    note_launch();
    check_launch("match_greedy");
    return;
  }
  if (bound >= 0 && bound <= kGreedyGrid &&
      coop_launch(k_greedy_persist, bound, kFusedThreads, s, a, ntasks, pairs, npairs, grid_bar(ws, s), m.err, 1)) {
    check_launch("match_greedy");
    return;
  }
  /* grid rounds, each a launch that returns at once when few rows wait:
   * about two per halving of the list bound down to kGreedyTail rows (on
   * the 2M-triangle workload the first level has more than 2,048 rows
   * waiting for 18 rounds), at most kGreedyRounds - 8 */
  int rounds = kGreedyRounds - 8;
  if (bound >= 0) {
    rounds = 4;
    for (long long n = bound; n > kGreedyTail; n /= 2) rounds += 2;
    rounds = std::min(rounds, kGreedyRounds - 8);
  }
  const int g = grid_bounded(bound, nb_elems);
  const int min_n = bound < 0 ? kFusedThreads + 1 : 0;
  cudaMemsetAsync(npairs, 0, sizeof(int), s);
  cudaMemsetAsync(ws.cnt, 0, sizeof(int) * (8 + kGreedyRounds), s);
  k_greedy_start<<<g, TRN_THREADS, 0, s>>>(a, ntasks, min_n);
  note_launch();
  /* a long list known: grid launches while more than kGreedyGrid rows wait,
   * then the cooperative rounds */
  const bool coop = bound > kGreedyGrid;
  if (coop) {
    rounds = 0;
    for (long long n = bound; n > kGreedyGrid; n /= 2) rounds += 3;
    rounds = std::min(rounds, kGreedyRounds - 8);
  }
  for (int r = 0; r < rounds; ++r) {
    k_greedy_round<<<TRN_RESIDENT(k_greedy_round, g, TRN_THREADS), TRN_THREADS, 0, s>>>(a, ntasks, r, pairs, npairs, coop ? kGreedyGrid + 1 : 0);
    note_launch();
  }
  if (coop && coop_launch(k_greedy_persist, bound, kFusedThreads, s, a, ntasks, pairs, npairs, grid_bar(ws, s),
                          m.err, 0)) {
    check_launch("match_greedy");
    return;
  }
  /* the rounds left; when the list is unknown, the whole short-list form
   * too, each returning at once when the count is not its case */
  k_greedy_tail<<<1, kFusedThreads, 0, s>>>(a, ntasks, pairs, npairs, 0, min_n);
  note_launch();
  if (bound < 0) {
    k_greedy_tail<<<1, kFusedThreads, 0, s>>>(a, ntasks, pairs, npairs, 1, kFusedThreads);
    note_launch();
  }
  check_launch("match_greedy");
}

/* ---------------- coloring ---------------- */
/* color word: 0 = uncolored, else (round + 1) << 8 | color, color 0xff =
 * none. Vertices that take no part get kNotColored: to their neighbours a
 * vertex colored in no round with a color outside the palette (bit 31 of the
 * used-color mask, never a color), so a round reads one word per neighbour */
constexpr int kNotColored = (0x7fffff << 8) | 31;

__global__ void k_color_init(DMesh m, int nb_nodes, int* list, int* n, int* color) {
  nb_nodes = trn_nodes(m, nb_nodes);
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) {
    if (m.activ[v] == 1 && m.vdeg[v] > 0) trn_append(list, n, v);
    else color[v] = kNotColored;
  }
}

/* One vertex of a round of the speculative first-fit coloring: true when it
 * must wait. Each uncolored vertex holds a tentative color, chosen in the
 * round before (tent[(round - 1) & 1], none in round 0). It keeps it when no
 * neighbour colored in an earlier round has it and no neighbour still
 * competing at the round's start (uncolored, or colored in this very round)
 * with a higher priority holds the same tentative; two neighbours never keep
 * the same color in one round, so the coloring is proper. Otherwise it
 * chooses a new tentative for the next round (tent[round & 1]): the smallest
 * color unused by the neighbours colored in earlier rounds and by the
 * tentatives of its higher-priority competitors; with none left it waits
 * without one, and when the colored neighbours alone use every color it
 * takes none (0xff, not smoothed). A round reads only the state its start
 * left (round-stamped colors, the other tentative buffer), so the result does
 * not depend on timing. Unlike Jones-Plassmann, a vertex need not outrank
 * every competing neighbour, only those that want its color: fewer rounds. */
__device__ __forceinline__ bool color_item(const DMesh& m, int v, int* color, uint8_t* tent, int capa,
                                           int max_col, uint64_t seed, int round) {
  const uint64_t pv = trn_prio(seed, v);
  const int* vc = m.vic + (size_t) v * m.bucket;
  const int nv = m.vdeg[v];
  const uint8_t* prev = tent + (size_t) ((round - 1) & 1) * capa;
  const int mine = round > 0 ? prev[v] : 0;
  bool keep = mine != 0;
  unsigned used = 0, wanted = 0;
  for (int b = 0; b < nv; ++b) {
    const int w = vc[b];
    const int cw = *(volatile int*) (color + w);
    const int rw = cw >> 8;
    if (cw == 0 || rw == round + 1) {
      if (round > 0 && trn_prio(seed, w) > pv) {
        const int tw = prev[w];
        wanted |= 1u << tw;
        if (tw == mine) keep = false;
      }
    } else {
      used |= 1u << (cw & 0xff & 31);
    }
  }
  if (keep && !(used & (1u << mine))) {
    color[v] = ((round + 1) << 8) | mine;
    return false;
  }
  int c = 1;
  while (c <= max_col && ((used | wanted) & (1u << c))) ++c;
  if (c > max_col) {
    int f = 1;
    while (f <= max_col && (used & (1u << f))) ++f;
    if (f > max_col) {
      color[v] = ((round + 1) << 8) | 0xff;
      return false;
    }
    c = 0;
  }
  tent[(size_t) (round & 1) * capa + v] = (uint8_t) c;
  return true;
}

/* a list this short goes to the one-block rounds (k_color_tail) */
constexpr int kColorTail = 4096;

/* one round over the still-uncolored vertices; those that must wait go to the
 * next list. A vertex takes the smallest color unused by neighbours colored
 * in earlier rounds once its priority beats every neighbour still competing
 * (uncolored, or colored in this very round). A list of at most kColorTail
 * vertices is left to the one-block tail: the round marks the coloring
 * frozen (1 + the list's buffer) and it and the later rounds of the batch do
 * nothing. */
__global__ void k_color_round(DMesh m, const int* __restrict__ list, const int* n_in, int* color,
                              uint8_t* tent, int max_col, Seed sd, const int* round_ctr, int* next,
                              int* n_next, int* frozen, int cur) {
  if (trn_failed(m) || *frozen) return;
  const int n = *n_in;
  if (n <= kColorTail) {
    if (trn_tid() == 0) *frozen = 1 + cur;
    return;
  }
  const uint64_t seed = trn_seed(sd);
  const int round = *round_ctr;
  for (int q = trn_tid(); q < n; q += trn_grid_stride()) {
    const int v = list[q];
    if (color_item(m, v, color, tent, m.capa_node, max_col, seed, round)) trn_append(next, n_next, v);
  }
}

/* the rounds left, in one block, from the frozen list: until no vertex
 * waits (at most kColorTailRounds rounds; a vertex still waiting then is
 * not smoothed, like one that finds no free color) */
constexpr int kColorTailRounds = 512;

__global__ void __launch_bounds__(1024) k_color_tail(DMesh m, int* list_a, int* list_b, int* counts, int* color,
                                                     uint8_t* tent, int max_col, Seed sd, int* round_ctr,
                                                     int* frozen) {
  const int f = *frozen;
  if (trn_failed(m) || f == 0) return;
  const uint64_t seed = trn_seed(sd);
  int cur = f - 1;
  int round = *round_ctr;
  for (int it = 0; it < kColorTailRounds; ++it) {
    const int n = counts[cur];
    if (n == 0) break;
    int* in = cur ? list_b : list_a;
    int* out = cur ? list_a : list_b;
    if (it > 0) ++round;
    if (threadIdx.x == 0) counts[cur ^ 1] = 0;
    __syncthreads();
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
      const int v = in[q];
      if (color_item(m, v, color, tent, m.capa_node, max_col, seed, round))
        out[atomicAdd(counts + (cur ^ 1), 1)] = v;
    }
    __syncthreads();
    cur ^= 1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    *round_ctr = round;
    counts[0] = counts[1] = 0;   /* done: the batch's end sees nothing left */
  }
}

/* Within a color class the vertices are ordered by stencil length (bins of
 * 3, 4, .., 10 and more): the smoothing of a class then runs warps of equal
 * degree, whose quality loops do not wait for one long stencil. A class is
 * an independent set, so the order inside it changes no result. Keys are
 * color * kDegBins + bin. */
constexpr int kDegBins = 8;
constexpr int kColorKeys = 32 * kDegBins;

__device__ __forceinline__ int color_key(const DMesh& m, int v, int c) {
  int b = trn_deg(m, v) - 3;
  b = b < 0 ? 0 : (b >= kDegBins ? kDegBins - 1 : b);
  return c * kDegBins + b;
}

__global__ void k_color_count(DMesh m, int nb_nodes, const int* color, int* cnt, int max_col) {
  nb_nodes = trn_nodes(m, nb_nodes);
  __shared__ int sc[kColorKeys];
  for (int k = threadIdx.x; k < kColorKeys; k += blockDim.x) sc[k] = 0;
  __syncthreads();
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) {
    int c = color[v] & 0xff;
    if (color[v] != 0 && c >= 1 && c <= max_col) atomicAdd(sc + color_key(m, v, c), 1);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < kColorKeys; k += blockDim.x)
    if (sc[k]) atomicAdd(cnt + k, sc[k]);
}

/* before a round: its number, and the list it fills starts empty (nothing
 * once the coloring is frozen for the tail) */
__global__ void k_color_step(int* round_ctr, int* n_next, const int* frozen) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || *frozen) return;
  *round_ctr += 1;
  *n_next = 0;
}

/* after 8 rounds: another batch while vertices wait and fewer than 8 batches
 * ran; in a captured round the answer drives the loop node */
__global__ void k_color_batch_end(const int* left, int* batch, int* cont,
                                  cudaGraphConditionalHandle h, int use_h) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int c = (*left > 0) && (++*batch < 8);
  *cont = c;
  if (use_h) cudaGraphSetConditional(h, c);
}

__global__ void k_color_offsets(const int* cnt, int* part_off, int* cursor, int max_col,
                                unsigned* tick) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (tick) ++*tick;
  int acc = 0;
  for (int c = 1; c <= max_col; ++c) {
    part_off[c - 1] = acc;
    for (int b = 0; b < kDegBins; ++b) {
      cursor[c * kDegBins + b] = acc;
      acc += cnt[c * kDegBins + b];
    }
  }
  part_off[max_col] = acc;
}

/* vertices into their color's part, by degree bin; per block, the slots are
 * counted in shared memory and reserved with one global atomic per key (a
 * global atomic per vertex on a few cursors serialises) */
__global__ void k_color_scatter(DMesh m, int nb_nodes, const int* nbp, int* color, int* cursor, int* parts,
                                int max_col) {
  if (nbp) nb_nodes = nbp[0];
  __shared__ int cnt[kColorKeys], base[kColorKeys];
  for (int v0 = blockIdx.x * blockDim.x; v0 < nb_nodes; v0 += gridDim.x * blockDim.x) {
    for (int k = threadIdx.x; k < kColorKeys; k += blockDim.x) cnt[k] = 0;
    __syncthreads();
    const int v = v0 + threadIdx.x;
    int key = -1, slot = 0;
    if (v < nb_nodes) {
      const int cw = color[v];
      if (cw != 0 && (cw & 0xff) >= 1 && (cw & 0xff) <= max_col) {
        key = color_key(m, v, cw & 0xff);
        slot = atomicAdd(cnt + key, 1);
      }
      color[v] = 0;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < kColorKeys; k += blockDim.x)
      if (cnt[k] > 0) base[k] = atomicAdd(cursor + k, cnt[k]);
    __syncthreads();
    if (key >= 0) parts[base[key] + slot] = v;
    __syncthreads();
  }
}

/* list counters and loop state of the coloring, in ws.cnt */
static int* color_counts(HeurWs& ws) { return ws.cnt + 80; }   /* two list counters */
static int* color_round(HeurWs& ws) { return ws.cnt + 82; }
static int* color_batch_no(HeurWs& ws) { return ws.cnt + 83; }
int* color_cont(HeurWs& ws) { return ws.cnt + 84; }
static int* color_frozen(HeurWs& ws) { return ws.cnt + 85; }

void color_begin(const DMesh& m, int hint, HeurWs& ws, cudaStream_t s) {
  ProfScope ps("color_jp", s, 0.0);
  int* counts = color_counts(ws);
  cudaMemsetAsync(counts, 0, sizeof(int) * 2, s);
  cudaMemsetAsync(color_round(ws), 0xff, sizeof(int), s);   /* -1: the first step makes it 0 */
  cudaMemsetAsync(color_batch_no(ws), 0, sizeof(int), s);
  cudaMemsetAsync(color_frozen(ws), 0, sizeof(int), s);
  k_color_init<<<grid_for(hint), TRN_THREADS, 0, s>>>(m, hint, ws.list_a, counts, ws.color);
  note_launch();
}

void color_batch(const DMesh& m, int hint, int max_col, Seed sd, HeurWs& ws, cudaStream_t s,
                 cudaGraphConditionalHandle h, bool use_h) {
  ProfScope ps("color_jp", s, 0.0);
  const int g = grid_for(hint);
  int* lists[2] = {ws.list_a, ws.list_b};
  int* counts = color_counts(ws);
  for (int r = 0; r < 8; ++r) {
    const int cur = r & 1;
    k_color_step<<<1, 32, 0, s>>>(color_round(ws), counts + (cur ^ 1), color_frozen(ws));
    note_launch();
    k_color_round<<<TRN_RESIDENT(k_color_round, g, TRN_THREADS), TRN_THREADS, 0, s>>>(m, lists[cur], counts + cur, ws.color, ws.tent, max_col, sd,
                                            color_round(ws), lists[cur ^ 1], counts + (cur ^ 1),
                                            color_frozen(ws), cur);
    note_launch();
  }
  k_color_tail<<<1, 1024, 0, s>>>(m, ws.list_a, ws.list_b, counts, ws.color, ws.tent, max_col, sd,
                                  color_round(ws), color_frozen(ws));
  note_launch();
  /* an even number of rounds: the vertices still waiting are in list_a */
  k_color_batch_end<<<1, 32, 0, s>>>(counts, color_batch_no(ws), color_cont(ws), h, use_h ? 1 : 0);
  note_launch();
}

void color_finish(const DMesh& m, int hint, int max_col, HeurWs& ws, int* parts, int* part_off,
                  unsigned* tick, cudaStream_t s) {
  ProfScope ps("color_jp", s, 0.0);
  const int g = grid_for(hint);
  int* cnt = ws.color_keys;                 /* kColorKeys slots */
  int* cursor = ws.color_keys + kColorKeys;  /* kColorKeys slots */
  cudaMemsetAsync(cnt, 0, sizeof(int) * kColorKeys, s);
  k_color_count<<<g, TRN_THREADS, 0, s>>>(m, hint, ws.color, cnt, max_col);
  note_launch();
  k_color_offsets<<<1, 32, 0, s>>>(cnt, part_off, cursor, max_col, tick);
  note_launch();
  k_color_scatter<<<g, TRN_THREADS, 0, s>>>(m, hint, m.nb, ws.color, cursor, parts, max_col);
  note_launch();
  check_launch("color_jp");
}

/* every round of the coloring in one cooperative launch, until no vertex
 * waits (at most kColorTailRounds rounds); the list counts rotate over
 * three words so that the one a round fills starts at zero. Once kColorTail
 * vertices or fewer wait, the first block colors the rest alone. */
__global__ void __launch_bounds__(kFusedThreads) k_color_persist(DMesh m, int* list_a, int* list_b,
                                                                 int* counts, int* rot, int* color,
                                                                 uint8_t* tent, int max_col, Seed sd,
                                                                 int* round_ctr, GridBar* bar) {
  if (trn_failed_block(m)) return;
  const uint64_t seed = trn_seed(sd);
  int round = *round_ctr;
  if (trn_tid() == 0) {
    rot[0] = counts[0];
    rot[1] = 0;
    rot[2] = 0;
  }
  if (!grid_sync(bar, m.err)) return;
  int it = 0;
  bool alone = false;
  for (; it < kColorTailRounds; ++it) {
    const int n = *(volatile int*) (rot + it % 3);
    if (n == 0) break;
    if (!alone && n <= kColorTail) {
      if (blockIdx.x != 0) return;
      alone = true;
    }
    ++round;
    int* in = (it & 1) ? list_b : list_a;
    int* out = (it & 1) ? list_a : list_b;
    const int b0 = alone ? 0 : (int) (blockIdx.x * blockDim.x);
    const int bs = alone ? (int) blockDim.x : trn_grid_stride();
    if (b0 == 0 && threadIdx.x == 0) rot[(it + 2) % 3] = 0;
    for (int base = b0; base < n; base += bs) {
      const int q = base + threadIdx.x;
      const int v = q < n ? in[q] : -1;
      const bool wait = q < n && color_item(m, v, color, tent, m.capa_node, max_col, seed, round);
      trn_block_append(out, rot + (it + 1) % 3, v, wait);
    }
    if (alone) __syncthreads();
    else if (!grid_sync(bar, m.err)) return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *round_ctr = round;
    counts[0] = counts[1] = 0;
  }
}

void color_jp(const DMesh& m, int hint, int max_col, Seed sd, HeurWs& ws, int* parts, int* part_off,
              unsigned* tick, cudaStream_t s) {
  color_begin(m, hint, ws, s);
  bool done;
  {
    ProfScope ps("color_jp", s, 0.0);
    done = coop_launch(k_color_persist, hint, kFusedThreads, s, m, ws.list_a, ws.list_b, color_counts(ws),
                       ws.cnt + 104, ws.color, ws.tent, max_col, sd, color_round(ws), grid_bar(ws, s));
  }
  if (done) {
    color_finish(m, hint, max_col, ws, parts, part_off, tick, s);
    return;
  }
  int cont = 1;
  while (cont) {
    color_batch(m, hint, max_col, sd, ws, s, 0, false);
    cudaMemcpyAsync(&cont, color_cont(ws), sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
  }
  color_finish(m, hint, max_col, ws, parts, part_off, tick, s);
}

/* the bounded barrier's failure path on the device: a cooperative launch of
 * k_barrier_selftest on its own barrier and error word; *gave_up: the
 * waiting blocks gave up and marked the error word. Returns the CUDA status. */
cudaError_t barrier_selftest(long long max_polls, int* gave_up) {
  *gave_up = 0;
  int dev = 0, coop = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
  if (!coop) return cudaErrorNotSupported;
  void* mem = nullptr;
  cudaError_t e = cudaMalloc(&mem, sizeof(GridBar) + sizeof(int));
  if (e != cudaSuccess) return e;
  GridBar* bar = static_cast<GridBar*>(mem);
  int* err = reinterpret_cast<int*>(static_cast<char*>(mem) + sizeof(GridBar));
  cudaMemset(mem, 0, sizeof(GridBar) + sizeof(int));
  void* argv[] = {&bar, &err, &max_polls};
  e = cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k_barrier_selftest), 4, 32, argv, 0, nullptr);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  int h = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(mem);
  *gave_up = h != 0;
  return e;
}

void heur_ws_alloc(HeurWs* ws, int capa_node, int capa_elem) {
  size_t big = (size_t) (capa_node > capa_elem ? capa_node : capa_elem);
  cudaMalloc(&ws->state, big);
  cudaMemset(ws->state, 0, big);
  cudaMalloc(&ws->state2, big);
  cudaMemset(ws->state2, 0, big);
  cudaMalloc(&ws->prop, sizeof(unsigned long long) * (size_t) capa_elem);
  cudaMalloc(&ws->choice, sizeof(int) * (size_t) capa_elem);
  cudaMalloc(&ws->choice2, sizeof(int) * (size_t) capa_elem);
  cudaMalloc(&ws->prop2, sizeof(unsigned long long) * (size_t) capa_elem);
  cudaMalloc(&ws->tent, 2 * (size_t) capa_node);
  cudaMalloc(&ws->color, sizeof(int) * (size_t) capa_node);
  cudaMemset(ws->color, 0, sizeof(int) * (size_t) capa_node);
  cudaMalloc(&ws->mate, sizeof(int) * (size_t) capa_elem);
  cudaMalloc(&ws->rank, sizeof(uint32_t) * 4 * (size_t) capa_elem);
  cudaMalloc(&ws->cnt, sizeof(int) * 128);
  cudaMemset(ws->cnt, 0, sizeof(int) * 128);   /* the grid barrier's words start at zero */
  cudaMalloc(&ws->color_keys, sizeof(int) * 2 * kColorKeys);
  cudaMalloc(&ws->list_a, sizeof(int) * big);
  cudaMalloc(&ws->list_b, sizeof(int) * big);
  cudaMalloc(&ws->fix_list, sizeof(int) * (size_t) capa_node);
}

void heur_ws_free(HeurWs* ws) {
  cudaFree(ws->state);
  cudaFree(ws->state2);
  cudaFree(ws->prop);
  cudaFree(ws->choice);
  cudaFree(ws->choice2);
  cudaFree(ws->prop2);
  cudaFree(ws->tent);
  cudaFree(ws->color);
  cudaFree(ws->mate);
  cudaFree(ws->rank);
  cudaFree(ws->cnt);
  cudaFree(ws->color_keys);
  cudaFree(ws->list_a);
  cudaFree(ws->list_b);
  cudaFree(ws->fix_list);
  *ws = HeurWs();
}

}  // namespace trn
