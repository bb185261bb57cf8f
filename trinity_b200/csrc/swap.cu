/*
 * swap.cu — edge flips (Swap::run, swapping.cpp:383-428).
 *
 *   k_swap_init    repair tags off, element -> dual-index map reset, quality
 *                  cache and activity of every live element (cacheQuality,
 *                  swapping.cpp:152-178)
 *   k_swap_filter  active elements lose their flag; those with q < 0.9 become
 *                  candidates (filterElems, swapping.cpp:181-201)
 *   k_swap_dual    per candidate: itself plus its edge neighbours, the two at
 *                  its first vertex found in that vertex's stencil order, then
 *                  the one across the opposite edge (extractDualGraph,
 *                  swapping.cpp:204-248); records element -> row index
 *   k_swap_filter_dual  free mode: the filter and the rows in one pass, with
 *                  the quality change of each row's flips when the matching
 *                  ranks its edges by gain
 *   k_swap_flip2   per matched pair (two lanes): flip the shared edge when both new
 *                  elements are CCW and the smaller quality does not drop;
 *                  stencil appends, repair tags, cached qualities and
 *                  re-activation of the dual rows (Swap::swap, swapping.cpp:55-149)
 * The map keeps entries of earlier levels of the same call (it is reset once
 * per call, like the reference), so re-activation may follow an older row;
 * rows therefore persist across levels.
 */
#include "trn_internal.h"
#include "trn_mixed.cuh"

namespace trn {

__global__ void k_swap_init_nodes(DMesh m, int nb_nodes) {
  nb_nodes = trn_nodes(m, nb_nodes);
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) m.fixes[v] = 0;
}

/* with `act`, the live (active) elements also go onto the list act (free
 * mode's first level; the list is unordered by design) */
template <bool F32>
__global__ void k_swap_init_elems(DMesh m, int nb_elems, int* __restrict__ map, int* __restrict__ act,
                                  int* act_n) {
  nb_elems = trn_elems(m, nb_elems);
  if (trn_failed_block(m)) return;
  for (int base = blockIdx.x * blockDim.x; base < nb_elems; base += trn_grid_stride()) {
    const int i = base + threadIdx.x;
    bool live = false;
    if (i < nb_elems) {
      map[i] = -1;
      const int4 t = m.tri[i];
      live = t.x >= 0;
      if (live) m.qual[i] = quality_of<F32>(m, t);
      m.activ[i] = live ? 1 : 0;
    }
    if (act) trn_block_append(act, act_n, i, live);
  }
}

__global__ void k_swap_filter(DMesh m, int nb_elems, uint8_t* __restrict__ flag) {
  nb_elems = trn_elems(m, nb_elems);
  for (int i = trn_tid(); i < nb_elems; i += trn_grid_stride()) {
    uint8_t f = 0;
    if (m.activ[i]) {
      m.activ[i] = 0;
      f = (m.qual[i] < TRN_Q_MIN) ? 1 : 0;
    }
    flag[i] = f;
  }
}

/* the dual row of candidate k at row index i; returns its length */
__device__ __forceinline__ int dual_row(const DMesh& m, int k, int i, int* __restrict__ dual,
                                        int* __restrict__ dual_n, int* __restrict__ map) {
  {
    const int4 n = m.tri[k];
    int row[4] = {k, -1, -1, -1};
    int dn = 1;
    const int* s0 = m.stenc + (size_t) n.x * m.bucket;
    const int d0 = trn_deg(m, n.x);
    for (int a = 0; dn < 3 && a < d0; ++a) {
      int t = s0[a];
      if (t == k) continue;
      int4 v = m.tri[t];
      if ((v.x == n.x && v.y == n.z) || (v.x == n.y && v.y == n.x) ||
          (v.y == n.x && v.z == n.z) || (v.y == n.y && v.z == n.x) ||
          (v.z == n.x && v.x == n.z) || (v.z == n.y && v.x == n.x))
        row[dn++] = t;
    }
    const int* s2 = m.stenc + (size_t) n.z * m.bucket;
    const int d2 = trn_deg(m, n.z);
    for (int a = 0; a < d2; ++a) {
      int t = s2[a];
      if (t == k) continue;
      int4 v = m.tri[t];
      if ((v.x == n.z && v.y == n.y) || (v.y == n.z && v.z == n.y) || (v.z == n.z && v.x == n.y)) {
        row[dn++] = t;
        break;
      }
    }
    reinterpret_cast<int4*>(dual)[i] = make_int4(row[0], row[1], row[2], row[3]);
    dual_n[i] = dn;
    map[k] = i;
    return dn;
  }
}

__global__ void k_swap_dual(DMesh m, const int* __restrict__ list, int ntasks, int* __restrict__ dual,
                            int* __restrict__ dual_n, int* __restrict__ map) {
  if (trn_failed(m)) return;
  for (int i = trn_tid(); i < ntasks; i += trn_grid_stride()) dual_row(m, list[i], i, dual, dual_n, map);
}

/* the two elements that replace id1 and id2 when their shared edge flips
 * (Swap::swap, swapping.cpp:59-106): false when they share no edge or a new
 * element is not CCW; else c1, c2 and their qualities q0, q1 */
template <bool F32>
__device__ __forceinline__ bool flip_eval(const DMesh& m, int id1, int id2, int c1[3], int c2[3],
                                          double* q0, double* q1) {
  const int4 a = m.tri[id1], b = m.tri[id2];
  const int o1[3] = {a.x, a.y, a.z};
  const int o2[3] = {b.x, b.y, b.z};
  c1[0] = c1[1] = c1[2] = c2[0] = c2[1] = c2[2] = -1;
  for (int i = 0; i < 3; ++i) {
    int j = (i + 1) % 3, k = (i + 2) % 3;
    if (o1[i] == o2[1] && o1[j] == o2[0]) {
      c1[0] = o1[i]; c1[1] = o2[2]; c1[2] = o1[k];
      c2[0] = o1[k]; c2[1] = o2[2]; c2[2] = o1[j];
      break;
    }
    if (o1[i] == o2[2] && o1[j] == o2[1]) {
      c1[0] = o1[i]; c1[1] = o2[0]; c1[2] = o1[k];
      c2[0] = o1[k]; c2[1] = o2[0]; c2[2] = o1[j];
      break;
    }
    if (o1[i] == o2[0] && o1[j] == o2[2]) {
      c1[0] = o1[i]; c1[1] = o2[1]; c1[2] = o1[k];
      c2[0] = o1[k]; c2[1] = o2[1]; c2[2] = o1[j];
      break;
    }
  }
  if (c1[0] < 0) return false;
  const double2 p10 = m.pts[c1[0]], p11 = m.pts[c1[1]], p12 = m.pts[c1[2]];
  const double2 p22 = m.pts[c2[2]];
  /* c2 = (c1[2], c1[1], c2[2]) */
  if (!trn_ccw(p10, p11, p12) || !trn_ccw(p12, p11, p22)) return false;
  const LogT<F32> l10 = log_load<F32>(m, c1[0]), l11 = log_load<F32>(m, c1[1]);
  const LogT<F32> l12 = log_load<F32>(m, c1[2]), l22 = log_load<F32>(m, c2[2]);
  *q0 = quality_x(p10, p11, p12, l10, l11, l12);
  *q1 = quality_x(p12, p11, p22, l12, l11, l22);
  return true;
}

/* flip_eval by two lanes of a warp: both find the new elements and test
 * them, lane `half` 0 evaluates the first new element's quality and lane 1
 * the second's, and they trade results; the same values as flip_eval.
 * Both lanes of the pair must call it (mask: the pair's two lanes). */
template <bool F32>
__device__ __forceinline__ bool flip_eval2(const DMesh& m, int id1, int id2, int c1[3], int c2[3],
                                           double* q0, double* q1, int half, unsigned mask) {
  const int4 a = m.tri[id1], b = m.tri[id2];
  const int o1[3] = {a.x, a.y, a.z};
  const int o2[3] = {b.x, b.y, b.z};
  c1[0] = c1[1] = c1[2] = c2[0] = c2[1] = c2[2] = -1;
  for (int i = 0; i < 3; ++i) {
    int j = (i + 1) % 3, k = (i + 2) % 3;
    if (o1[i] == o2[1] && o1[j] == o2[0]) {
      c1[0] = o1[i]; c1[1] = o2[2]; c1[2] = o1[k];
      c2[0] = o1[k]; c2[1] = o2[2]; c2[2] = o1[j];
      break;
    }
    if (o1[i] == o2[2] && o1[j] == o2[1]) {
      c1[0] = o1[i]; c1[1] = o2[0]; c1[2] = o1[k];
      c2[0] = o1[k]; c2[1] = o2[0]; c2[2] = o1[j];
      break;
    }
    if (o1[i] == o2[0] && o1[j] == o2[2]) {
      c1[0] = o1[i]; c1[1] = o2[1]; c1[2] = o1[k];
      c2[0] = o1[k]; c2[1] = o2[1]; c2[2] = o1[j];
      break;
    }
  }
  bool ok = c1[0] >= 0;
  double q = 0;
  if (ok) {
    const double2 p10 = m.pts[c1[0]], p11 = m.pts[c1[1]], p12 = m.pts[c1[2]];
    const double2 p22 = m.pts[c2[2]];
    ok = trn_ccw(p10, p11, p12) && trn_ccw(p12, p11, p22);
    if (ok) {
      /* lane 0: (c1[0], c1[1], c1[2]); lane 1: (c1[2], c1[1], c2[2]) */
      const int va = half ? c1[2] : c1[0], vc = half ? c2[2] : c1[2];
      const double2 pa = half ? p12 : p10, pc = half ? p22 : p12;
      q = quality_x(pa, p11, pc, log_load<F32>(m, va), log_load<F32>(m, c1[1]), log_load<F32>(m, vc));
    }
  }
  const double other = __shfl_xor_sync(mask, q, 1);
  *q0 = half ? other : q;
  *q1 = half ? q : other;
  return ok;
}

/* the matching rank of the flip of the edge shared by elements a and b: the
 * change of the smaller quality, min(q_new) - min(q_old), in [-1, 1], or
 * -1.5 when the flip is impossible, quantized to the upper 22 bits of a
 * word. Both rows of a candidate pair evaluate the flip with the smaller id
 * first, so the two ranks agree bit for bit */
template <bool F32>
__device__ __forceinline__ uint32_t flip_rank(const DMesh& m, int a, int b) {
  const int id1 = a < b ? a : b, id2 = a < b ? b : a;
  int c1[3], c2[3];
  double q0, q1, gain = -1.5;
  if (flip_eval<F32>(m, id1, id2, c1, c2, &q0, &q1))
    gain = trn_dmin(q0, q1) - trn_dmin(m.qual[id1], m.qual[id2]);
  if (!(gain >= -1.5)) gain = -1.5;
  if (gain > 1.0) gain = 1.0;
  return ((uint32_t) ((gain + 2.0) * 1048576.0)) << 10;
}

/* free mode: filter, dual extraction and (when rank is given) the ranks of
 * each row's flips in one pass; rows are numbered in append order (no use
 * depends on it) */
template <bool F32>
__global__ void k_swap_filter_dual(DMesh m, const int* __restrict__ act, const int* act_n,
                                   int* __restrict__ dual, int* __restrict__ dual_n,
                                   int* __restrict__ map, uint32_t* __restrict__ rank, int* count,
                                   GreedyReset gr, int* flips) {
  if (blockIdx.x == 0 && threadIdx.x == 0) trn_level_clear(m, flips);
  if (trn_failed(m)) return;
  const int na = *act_n;
  for (int q = trn_tid(); q < na; q += trn_grid_stride()) {
    const int k = act[q];
    if (!m.activ[k]) continue;
    m.activ[k] = 0;
    if (!(m.qual[k] < TRN_Q_MIN)) continue;
    unsigned mask = __activemask();
    int lane = threadIdx.x & 31, leader = __ffs(mask) - 1, base = 0;
    if (lane == leader) base = atomicAdd(count, __popc(mask));
    base = __shfl_sync(mask, base, leader);
    const int r = base + __popc(mask & ((1u << lane) - 1));
    const int dn = dual_row(m, k, r, dual, dual_n, map);
    if (gr.vis)   /* the greedy matching's state of the row's elements (rows sharing one write the same) */
      for (int e = 0; e < dn; ++e) {
        const int x = dual[r * 4 + e];
        gr.vis[x] = -1;
        gr.mk0[x] = ~0ULL;
        gr.mk1[x] = ~0ULL;
      }
    if (rank) {
      uint32_t w[4] = {0u, 0u, 0u, 0u};
      for (int e = 1; e < dn; ++e) w[e] = flip_rank<F32>(m, k, dual[r * 4 + e]);
      reinterpret_cast<uint4*>(rank)[r] = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

/* Swap::swap, swapping.cpp:55-149, with the two new qualities on two lanes:
 * the pair's lanes run the tests together, then lane 0 alone commits the
 * flip (new element records, stencil appends, cached qualities), tags the
 * four vertices for repair and re-activates the dual rows. The reference
 * follows the map even when it points at a row of an earlier level (the map
 * is reset once per call, swapping.cpp:161-162); replay keeps that, the free
 * mode (rows numbered in append order) only follows rows of the current
 * level. Flag atomics are independent of one another and the newly set ones
 * go onto their lists with one atomic each, which keeps a flip's chain of
 * dependent L2 round trips short. */
template <bool F32>
__device__ int flip_pair2(const DMesh& m, int id1, int id2, int index, const int* map,
                          const int* dual, const int* dual_n, int ntasks, bool strict_map, int half,
                          unsigned mask) {
  int c1[3], c2[3];
  double q0, q1;
  if (!flip_eval2<F32>(m, id1, id2, c1, c2, &q0, &q1, half, mask)) return 0;
  const double q_old = trn_dmin(m.qual[id1], m.qual[id2]);
  const double q_new = trn_dmin(q0, q1);
  if (q_new < q_old || half) return (q_new < q_old) ? 0 : 2;
  m.tri[id1] = make_int4(c1[0], c1[1], c1[2], 0);
  m.tri[id2] = make_int4(c2[0], c2[1], c2[2], 0);
  trn_stenc_append(m, c2[0], id2);
  trn_stenc_append(m, c2[1], id1);
  m.qual[id1] = q0;
  m.qual[id2] = q1;
  const int fv[4] = {c1[0], c1[1], c1[2], c2[2]};
  int fx[4], nf = 0;
  for (int j = 0; j < 4; ++j)
    if (trn_byte_cas01(m.fixes + fv[j])) fx[nf++] = fv[j];
  if (m.fix_list) trn_list_push_n(m.fix_list, m.fix_n, fx, nf);
  int act[8], na = 0;
  for (int q = 0; q < dual_n[index]; ++q) {
    const int t = dual[index * 4 + q];
    if (trn_byte_cas01(m.activ + t)) act[na++] = t;
  }
  const int x = map[id2];
  if (x > -1 && (!strict_map || (x < ntasks && dual[x * 4] == id2)))
    for (int q = 0; q < dual_n[x]; ++q) {
      const int t = dual[x * 4 + q];
      if (trn_byte_cas01(m.activ + t)) act[na++] = t;
    }
  if (m.act_next) trn_list_push_n(m.act_next, m.act_next_n, act, na);
  return 2;
}

/* two lanes per pair; the grid-stride loop keeps the lanes of a pair
 * together (both see the same p), so every shuffle has its partner */
template <bool F32>
__global__ void k_swap_flip2(DMesh m, const int* __restrict__ pairs, const int* npairs,
                             const int* __restrict__ map, const int* __restrict__ dual,
                             const int* __restrict__ dual_n, const int* ntasks_dev, int* commit,
                             int strict_map) {
  if (trn_failed(m)) return;
  const int np = *npairs;
  const int ntasks = *ntasks_dev;
  const int half = threadIdx.x & 1;
  const unsigned mask = 3u << (threadIdx.x & 30);
  int local = 0;
  const int stride = (gridDim.x * blockDim.x) >> 1;
  for (int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 1; p < np; p += stride) {
    const int k1 = pairs[2 * p], k2 = pairs[2 * p + 1];
    bool ok = k1 >= 0 && k1 < m.capa_elem && k2 >= 0 && k2 < m.capa_elem;
    int index = -1;
    if (ok) {
      index = map[k1];
      ok = index >= 0 && index < ntasks && dual[index * 4] == k1;
      if (ok) {
        ok = false;
        for (int q = 1; q < dual_n[index]; ++q) ok |= (dual[index * 4 + q] == k2);
      }
    }
    if (!ok) {
      if (!half) trn_set_error(m.err, TRN_DERR_REPLAY);
      continue;
    }
    const int r = flip_pair2<F32>(m, k1, k2, index, map, dual, dual_n, ntasks, strict_map != 0, half, mask);
    if (!half) local += r;
  }
  trn_warp_add(commit, local);
}

void swap_init(const DMesh& m, int nb_nodes, int nb_elems, int* map, bool fp32, cudaStream_t s, int* act,
               int* act_n) {
  ProfScope ps("swap_init", s, (double) nb_nodes + (double) nb_elems * (kTri + kQ + 4 + 1) +
                                 (double) nb_elems / 2 * (kPt + kTen));
  k_swap_init_nodes<<<grid_for(nb_nodes), TRN_THREADS, 0, s>>>(m, nb_nodes);
  note_launch();
  if (act) cudaMemsetAsync(act_n, 0, sizeof(int), s);
  if (fp32) k_swap_init_elems<true><<<grid_for(nb_elems), TRN_THREADS, 0, s>>>(m, nb_elems, map, act, act_n);
  else k_swap_init_elems<false><<<grid_for(nb_elems), TRN_THREADS, 0, s>>>(m, nb_elems, map, act, act_n);
  note_launch();
  check_launch("swap_init");
}

void swap_filter(const DMesh& m, int nb_elems, uint8_t* flag, cudaStream_t s) {
  ProfScope ps("swap_filter", s, (double) nb_elems * 3);
  k_swap_filter<<<grid_for(nb_elems), TRN_THREADS, 0, s>>>(m, nb_elems, flag);
  note_launch();
  check_launch("swap_filter");
}

void swap_dual(const DMesh& m, const int* list, int ntasks, int* dual, int* dual_n, int* map,
               cudaStream_t s) {
  ProfScope ps("swap_dual", s, (double) ntasks * (4 + kTri + 2 * kAvgDeg * (kIdx + kTri) + 16 + 4 + 4));
  k_swap_dual<<<grid_for(ntasks), TRN_THREADS, 0, s>>>(m, list, ntasks, dual, dual_n, map);
  note_launch();
  check_launch("swap_dual");
}

void swap_filter_dual(const DMesh& m, const int* act, const int* act_n, int* dual, int* dual_n,
                      int* map, uint32_t* rank, int* count, bool fp32, cudaStream_t s, long long bound,
                      GreedyReset gr, int* flips) {
  ProfScope ps("swap_filter", s, 0.0);
  const int g = grid_bounded(bound, m.capa_elem);
  auto* kern = fp32 ? k_swap_filter_dual<true> : k_swap_filter_dual<false>;
  kern<<<grid_resident(reinterpret_cast<const void*>(kern), TRN_THREADS, g), TRN_THREADS, 0, s>>>(
      m, act, act_n, dual, dual_n, map, rank, count, gr, flips);
  note_launch();
  check_launch("swap_filter_dual");
}

void swap_flip(const DMesh& m, const int* pairs, const int* npairs, const int* map,
               const int* dual, const int* dual_n, const int* ntasks, int* commit, bool strict_map,
               bool fp32, cudaStream_t s, long long bound) {
  ProfScope ps("swap_flip", s, 0.0);
  const int ft = tune().flip_threads;
  /* two lanes a pair: the grid sized for twice the pairs */
  const int g = grid_bounded(bound < 0 ? bound : 2 * bound, 2LL * m.capa_elem, ft);
  auto* kern = fp32 ? k_swap_flip2<true> : k_swap_flip2<false>;
  kern<<<grid_resident(reinterpret_cast<const void*>(kern), ft, g), ft, 0, s>>>(
      m, pairs, npairs, map, dual, dual_n, ntasks, commit, strict_map ? 1 : 0);
  note_launch();
  check_launch("swap_flip");
}

}  // namespace trn
