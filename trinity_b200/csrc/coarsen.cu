/*
 * coarsen.cu — edge collapse (Coarse::run body, coarsening.cpp:480-503).
 *
 *   k_coarse_pre     activity flags: corners -1, live vertices 1, others 0;
 *                    clear repair tags (coarsening.cpp:257-281)
 *   k_coarse_filter  per active vertex: the shortest collapse target among
 *                    neighbours closer than 1/sqrt(2) whose simulated collapse
 *                    keeps every surviving element CCW with edges <= sqrt(2)
 *                    (Coarse::identifyTarget, coarsening.cpp:47-133); ties are
 *                    broken in adjacency order, like the reference's multimap
 *   k_coarse_filter_group  the same search by 4, 8 or 16 lanes per vertex, for
 *                    levels that list few vertices (free mode)
 *   k_collapse       per independent vertex: erase the 1-2 shell elements,
 *                    move the rest of the stencil to the target, relabel,
 *                    tag repairs, re-activate the 1-ring (Coarse::collapseEdge,
 *                    coarsening.cpp:136-254 with Mesh::copyStencil mesh.cpp:497)
 * Independent sources touch disjoint elements, so the collapses of one level
 * run in parallel; appends to a shared target's stencil are atomic and the
 * repair pass sorts them.
 */
#include "trn_internal.h"
#include "trn_mixed.cuh"

#include <algorithm>

namespace trn {

/* with `act`, the active vertices also go onto the list act (free mode's
 * first level; the list is unordered by design) */
__global__ void k_coarse_pre(DMesh m, int nb_nodes, int* __restrict__ act, int* act_n) {
  nb_nodes = trn_nodes(m, nb_nodes);
  for (int base = blockIdx.x * blockDim.x; base < nb_nodes; base += trn_grid_stride()) {
    const int v = base + threadIdx.x;
    int8_t a = 0;
    if (v < nb_nodes) {
      if (m.tags[v] & TRN_TAG_CORNER) a = -1;
      else a = m.alive[v] ? 1 : 0;
      m.activ[v] = a;
      m.fixes[v] = 0;
    }
    if (act) trn_block_append(act, act_n, v, a > 0);
  }
}

template <bool F32>
__device__ int identify_target(const DMesh& m, int source) {
  const bool bound_source = (m.tags[source] & TRN_TAG_BOUND) != 0;
  double lens[TRN_MAX_DEG];
  int cands[TRN_MAX_DEG];
  int nc = 0;
  const int* vc = m.vic + (size_t) source * m.bucket;
  const int nv = m.vdeg[source];
  const double2 ps = m.pts[source];
  const TenT<F32> ts = ten_load<F32>(m, source);
  for (int b = 0; b < nv; ++b) {
    int neigh = vc[b];
    bool bound_destin = (m.tags[neigh] & TRN_TAG_BOUND) != 0;
    if (bound_source && !bound_destin) continue;
    double len;
    if (length_lt<F32>(ps, m.pts[neigh], ts, ten_load<F32>(m, neigh), TRN_L_MIN, &len)) {
      int p = nc;
      while (p > 0 && lens[p - 1] > len) {
        lens[p] = lens[p - 1];
        cands[p] = cands[p - 1];
        --p;
      }
      lens[p] = len;
      cands[p] = neigh;
      nc++;
    }
  }
  const int* st = m.stenc + (size_t) source * m.bucket;
  const int deg = trn_deg(m, source);
  int destin = -1;
  bool skip = true;
  int next = 0;
  while (skip && next < nc) {
    destin = cands[next++];
    skip = false;
    int shared = 0;
    const bool bound_destin = (m.tags[destin] & TRN_TAG_BOUND) != 0;
    for (int a = 0; !skip && a < deg; ++a) {
      int4 n = m.tri[st[a]];
      if ((source == n.x && destin == n.y) || (source == n.y && destin == n.x) ||
          (source == n.y && destin == n.z) || (source == n.z && destin == n.y) ||
          (source == n.z && destin == n.x) || (source == n.x && destin == n.z)) {
        skip = (++shared > 1 && bound_source && bound_destin);
        continue;
      }
      int f0 = (n.x == source ? destin : n.x);
      int f1 = (n.y == source ? destin : n.y);
      int f2 = (n.z == source ? destin : n.z);
      double2 p0 = m.pts[f0], p1 = m.pts[f1], p2 = m.pts[f2];
      if (trn_ccw(p0, p1, p2)) {
        const TenT<F32> t0 = ten_load<F32>(m, f0), t1 = ten_load<F32>(m, f1), t2 = ten_load<F32>(m, f2);
        skip = length_gt<F32>(p0, p1, t0, t1, TRN_L_MAX) || length_gt<F32>(p1, p2, t1, t2, TRN_L_MAX) ||
               length_gt<F32>(p2, p0, t2, t0, TRN_L_MAX);
        continue;
      }
      skip = true;
    }
  }
  return skip ? -1 : destin;
}

template <bool F32>
__global__ void k_coarse_filter(DMesh m, int nb_nodes, int* __restrict__ target,
                                uint8_t* __restrict__ flag) {
  nb_nodes = trn_nodes(m, nb_nodes);
  if (trn_failed(m)) return;
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) {
    uint8_t f = 0;
    if (m.activ[v] > 0) {
      m.activ[v] = 0;
      int t = identify_target<F32>(m, v);
      target[v] = t;
      f = t > -1 ? 1 : 0;
    }
    flag[v] = f;
  }
}

/* free mode: one pass per level rebuilds the adjacency of each active vertex,
 * finds its target and appends the candidates (in no particular order: the
 * independent set is chosen by hashed priorities, not by list position),
 * marking them undecided for the independent-set rounds */
template <bool F32>
__global__ void k_coarse_filter_append(DMesh m, const int* __restrict__ act, const int* act_n,
                                       int* __restrict__ target, int* __restrict__ cand, int* count,
                                       uint8_t* __restrict__ state, int min_n) {
  if (blockIdx.x == 0 && threadIdx.x == 0) trn_level_clear(m, nullptr);
  if (trn_failed(m)) return;
  const int n = *act_n;
  if (n < min_n) return;
  /* warp-aggregated appends: a block-wide one would make every thread wait
   * for its block's longest search at each step */
  for (int q = trn_tid(); q < n; q += trn_grid_stride()) {
    const int v = act[q];
    if (m.activ[v] <= 0) continue;
    m.activ[v] = 0;
    build_one_vicin(m, v);
    const int t = identify_target<F32>(m, v);
    target[v] = t;
    if (t > -1) {
      state[v] = 1;
      trn_append(cand, count, v);
    }
  }
}

/* the same search by a group of G lanes per vertex, for the levels that
 * list few vertices, where one lane's chain of dependent gathers (adjacency,
 * stencil, triangles, points, tensors) sets the time. The lanes compute the
 * neighbours' metric lengths, then check every (candidate, element) pair at
 * once; the per-candidate verdicts are combined as bit masks, and the pick is
 * the smallest (length, adjacency index) among the valid candidates, which is
 * the first valid one in the serial search's stable length order, so the
 * targets are the same. Vertices with more than 32 neighbours fall back to
 * the serial search on the group's first lane. */

template <bool F32, int G>
__global__ void k_coarse_filter_group(DMesh m, const int* __restrict__ act, const int* act_n,
                                      int* __restrict__ target, int* __restrict__ cand, int* count,
                                      uint8_t* __restrict__ state, int max_n) {
  if (blockIdx.x == 0 && threadIdx.x == 0) trn_level_clear(m, nullptr);
  if (trn_failed(m)) return;
  const int n = *act_n;
  if (n > max_n) return;
  const int lane = threadIdx.x & 31;
  const int gl = lane & (G - 1);
  const int gbase = lane & ~(G - 1);
  const int per_warp = 32 / G;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int base = warp * per_warp; base < n; base += nwarps * per_warp) {
    const int q = base + lane / G;
    int vv = -1;
    if (gl == 0 && q < n) {
      const int x = act[q];
      if (m.activ[x] > 0) {
        m.activ[x] = 0;
        build_one_vicin(m, x);
        vv = x;
      }
    }
    const int v = __shfl_sync(0xffffffffu, vv, gbase);
    __syncwarp();
    const int nv = v >= 0 ? m.vdeg[v] : 0;
    const bool serial = nv > 32;
    const bool grp = v >= 0 && !serial;
    const int* vc = m.vic + (size_t) (v >= 0 ? v : 0) * m.bucket;
    const int* st = m.stenc + (size_t) (v >= 0 ? v : 0) * m.bucket;
    const bool bsrc = v >= 0 && (m.tags[v] & TRN_TAG_BOUND) != 0;
    double2 ps = make_double2(0, 0);
    TenT<F32> ts{};
    if (grp) {
      ps = m.pts[v];
      ts = ten_load<F32>(m, v);
    }
    /* neighbours b = gl + G * k: candidates closer than 1/sqrt(2) */
    double lenk[32 / G];
    unsigned candm = 0, boundm = 0;
    for (int k = 0; k < 32 / G; ++k) {
      const int b = gl + G * k;
      lenk[k] = 0.0;
      if (grp && b < nv) {
        const int w = vc[b];
        const bool bd = (m.tags[w] & TRN_TAG_BOUND) != 0;
        if (bd) boundm |= 1u << b;
        if (!(bsrc && !bd)) {
          double len;
          if (length_lt<F32>(ps, m.pts[w], ts, ten_load<F32>(m, w), TRN_L_MIN, &len)) {
            candm |= 1u << b;
            lenk[k] = len;
          }
        }
      }
    }
    for (int o = G / 2; o >= 1; o >>= 1) {
      candm |= __shfl_xor_sync(0xffffffffu, candm, o);
      boundm |= __shfl_xor_sync(0xffffffffu, boundm, o);
    }
    /* every (candidate, element) pair of the simulated collapses */
    const int deg = grp ? trn_deg(m, v) : 0;
    const int np = (grp && candm) ? nv * deg : 0;
    const int iters = __reduce_max_sync(0xffffffffu, (np + G - 1) / G);
    unsigned failm = 0, once = 0, twice = 0;
    for (int k = 0; k < iters; ++k) {
      const int p = gl + G * k;
      if (p >= np) continue;
      const int b = p / deg, a = p - b * deg;
      if (!((candm >> b) & 1u)) continue;
      const unsigned bit = 1u << b;
      const int destin = vc[b];
      const int4 e = m.tri[st[a]];
      if ((v == e.x && destin == e.y) || (v == e.y && destin == e.x) || (v == e.y && destin == e.z) ||
          (v == e.z && destin == e.y) || (v == e.z && destin == e.x) || (v == e.x && destin == e.z)) {
        twice |= once & bit;
        once |= bit;
        continue;
      }
      const int f0 = (e.x == v ? destin : e.x);
      const int f1 = (e.y == v ? destin : e.y);
      const int f2 = (e.z == v ? destin : e.z);
      const double2 p0 = m.pts[f0], p1 = m.pts[f1], p2 = m.pts[f2];
      if (trn_ccw(p0, p1, p2)) {
        const TenT<F32> t0 = ten_load<F32>(m, f0), t1 = ten_load<F32>(m, f1), t2 = ten_load<F32>(m, f2);
        if (length_gt<F32>(p0, p1, t0, t1, TRN_L_MAX) || length_gt<F32>(p1, p2, t1, t2, TRN_L_MAX) ||
            length_gt<F32>(p2, p0, t2, t0, TRN_L_MAX))
          failm |= bit;
      } else {
        failm |= bit;
      }
    }
    for (int o = G / 2; o >= 1; o >>= 1) {
      const unsigned fo = __shfl_xor_sync(0xffffffffu, failm, o);
      const unsigned oo = __shfl_xor_sync(0xffffffffu, once, o);
      const unsigned to = __shfl_xor_sync(0xffffffffu, twice, o);
      twice |= to | (once & oo);
      once |= oo;
      failm |= fo;
    }
    const unsigned valid = candm & ~failm & ~(bsrc ? (twice & boundm) : 0u);
    /* the smallest (length, adjacency index) among the valid candidates */
    double best = 0.0;
    int bestb = -1;
    for (int k = 0; k < 32 / G; ++k) {
      const int b = gl + G * k;
      if (b < 32 && ((valid >> b) & 1u) && (bestb < 0 || lenk[k] < best)) {
        best = lenk[k];
        bestb = b;
      }
    }
    for (int o = G / 2; o >= 1; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int obb = __shfl_xor_sync(0xffffffffu, bestb, o);
      if (obb >= 0 && (bestb < 0 || ob < best || (ob == best && obb < bestb))) {
        best = ob;
        bestb = obb;
      }
    }
    if (gl == 0 && v >= 0) {
      const int t = serial ? identify_target<F32>(m, v) : (bestb >= 0 ? vc[bestb] : -1);
      target[v] = t;
      if (t > -1) {
        state[v] = 1;
        trn_append(cand, count, v);
      }
    }
  }
}

__global__ void k_collapse(DMesh m, const int* __restrict__ indep, const int* count,
                           const int* __restrict__ target, const uint8_t* __restrict__ cand_flag) {
  if (trn_failed(m)) return;
  const int n_indep = *count;
  for (int q = trn_tid(); q < n_indep; q += trn_grid_stride()) {
    const int source = indep[q];
    if (source < 0 || source >= m.capa_node || (cand_flag && !cand_flag[source])) {
      trn_set_error(m.err, TRN_DERR_REPLAY);
      continue;
    }
    const int destin = target[source];
    int* st = m.stenc + (size_t) source * m.bucket;
    const int deg = trn_deg(m, source);
    const int limit = (m.tags[source] & TRN_TAG_BOUND) ? 1 : 2;
    int k = 0, trash0 = -1, trash1 = -1;
    int opp[2] = {-1, -1};
    for (int a = 0; k < limit && a < deg; ++a) {
      int4 n = m.tri[st[a]];
      int o = -2;
      if ((source == n.x && destin == n.y) || (destin == n.x && source == n.y)) o = n.z;
      else if ((source == n.y && destin == n.z) || (destin == n.y && source == n.z)) o = n.x;
      else if ((source == n.z && destin == n.x) || (destin == n.z && source == n.x)) o = n.y;
      if (o != -2) {
        opp[k] = o;
        if (k == 0) trash0 = a; else trash1 = a;
        ++k;
      }
    }
    int rest[TRN_MAX_DEG];
    int nr = 0;
    for (int a = 0; a < deg; ++a) {
      int e = st[a];
      if (a == trash0 || a == trash1) {
        m.tri[e] = make_int4(-1, -1, -1, 0);
        continue;
      }
      rest[nr++] = e;
    }
    for (int j = 0; j < k; ++j)
      if (opp[j] >= 0) trn_tag_fix(m, opp[j]);
    trn_stenc_append_n(m, destin, rest, nr);
    for (int a = 0; a < nr; ++a) {
      int4 n = m.tri[rest[a]];
      if (n.x == source) n.x = destin;
      else if (n.y == source) n.y = destin;
      else if (n.z == source) n.z = destin;
      m.tri[rest[a]] = n;
    }
    trn_tag_fix(m, destin);
    const int* vc = m.vic + (size_t) source * m.bucket;
    const int nv = m.vdeg[source];
    /* re-activate the 1-ring: independent flag atomics, newly set ids listed
     * in batches of 16 with one atomic each */
    int ids[16], na = 0;
    for (int b = 0; b < nv; ++b) {
      const int t = vc[b];
      if (trn_byte_cas01(m.activ + t)) ids[na++] = t;
      if (na == 16) {
        if (m.act_next) trn_list_push_n(m.act_next, m.act_next_n, ids, na);
        na = 0;
      }
    }
    if (m.act_next) trn_list_push_n(m.act_next, m.act_next_n, ids, na);
    m.vdeg[source] = 0;
    m.alive[source] = 0;
    for (int a = 0; a < deg; ++a) st[a] = -1;
    m.deg[source] = 0;
  }
}

void coarsen_pre(const DMesh& m, int nb_nodes, cudaStream_t s, int* act, int* act_n) {
  if (act) cudaMemsetAsync(act_n, 0, sizeof(int), s);
  k_coarse_pre<<<grid_for(nb_nodes), TRN_THREADS, 0, s>>>(m, nb_nodes, act, act_n);
  note_launch();
  check_launch("coarsen_pre");
}

void coarsen_filter(const DMesh& m, int nb_nodes, int* target, uint8_t* flag, bool fp32, cudaStream_t s) {
  ProfScope ps("coarsen_filter", s, (double) nb_nodes * (1 + 1 + 4 + 1));
  if (fp32) k_coarse_filter<true><<<grid_for(nb_nodes), TRN_THREADS, 0, s>>>(m, nb_nodes, target, flag);
  else k_coarse_filter<false><<<grid_for(nb_nodes), TRN_THREADS, 0, s>>>(m, nb_nodes, target, flag);
  note_launch();
  check_launch("coarsen_filter");
}



void coarsen_filter_append(const DMesh& m, const int* act, const int* act_n, int* target, int* cand,
                           int* count, uint8_t* state, bool fp32, cudaStream_t s, long long bound) {
  ProfScope ps("coarsen_filter", s, 0.0);
  /* a level listing at most group_max vertices runs the grouped search
   * (measured on B200 with 8 lanes: faster below ~16k listed vertices, 2x
   * slower on full-mesh levels), a larger one the one-lane search. A known
   * bound (the level's list length) picks the form; with an unknown one (a
   * captured round) both are launched, and the one that is not the device
   * count's case returns at once. group_lanes = 1: the one-lane search at
   * every size (a launch shape for the tests: the same targets). */
  const Tune& t = tune();
  const bool one = t.group_lanes == 1;
  const int gm = one ? -1 : t.group_max;
  const bool small = !one && bound >= 0 && bound <= gm;
  const bool large = one || bound > gm;
  const int g = grid_bounded(bound, m.capa_node, t.filter_threads);
  const int gg = grid_bounded(bound < 0 ? -1 : bound * t.group_lanes, (long long) gm * t.group_lanes);
#define TRN_GROUP(F, G)                                                                              \
  k_coarse_filter_group<F, G><<<gg, TRN_THREADS, 0, s>>>(m, act, act_n, target, cand, count, state, gm)
  if (!large) {
    if (fp32) {
      if (t.group_lanes == 4) TRN_GROUP(true, 4);
      else if (t.group_lanes == 16) TRN_GROUP(true, 16);
      else TRN_GROUP(true, 8);
    } else {
      if (t.group_lanes == 4) TRN_GROUP(false, 4);
      else if (t.group_lanes == 16) TRN_GROUP(false, 16);
      else TRN_GROUP(false, 8);
    }
    note_launch();
  }
#undef TRN_GROUP
  if (!small) {
    /* alone (a known long list, or one lane throughout), it takes any count */
    const int min_n = large ? 0 : gm + 1;
    auto* kern = fp32 ? k_coarse_filter_append<true> : k_coarse_filter_append<false>;
    kern<<<grid_resident(reinterpret_cast<const void*>(kern), t.filter_threads, g), t.filter_threads, 0, s>>>(
        m, act, act_n, target, cand, count, state, min_n);
    note_launch();
  }
  check_launch("coarsen_filter_append");
}

void collapse(const DMesh& m, const int* indep, const int* count, const int* target,
              const uint8_t* cand_flag, cudaStream_t s, long long bound) {
  ProfScope ps("collapse", s, 0.0);
  k_collapse<<<TRN_RESIDENT(k_collapse, grid_bounded(bound, m.capa_node), TRN_THREADS), TRN_THREADS, 0, s>>>(m, indep, count, target,
                                                                      cand_flag);
  note_launch();
  check_launch("collapse");
}

}  // namespace trn
