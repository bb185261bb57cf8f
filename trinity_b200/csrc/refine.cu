/*
 * refine.cu — one refinement level (Refine::run loop body, refinement.cpp:463-483).
 *
 *   k_ref_filter  per element: metric lengths of its 3 edges, pattern = number
 *                 of edges longer than sqrt(2), the neighbour across each long
 *                 edge, and which long edges this element owns (n[j] < n[k] or
 *                 boundary) — refinement.cpp:216-264 / Mesh::getElemNeigh
 *                 mesh.cpp:437-453. Writes (owned << 32 | pattern) per element.
 *   scan          exclusive scan of those pairs in element order: new vertex
 *                 ids (nb_nodes + owned prefix) and new element ids (nb_elems +
 *                 pattern prefix) come out exactly as the 1-thread reference
 *                 numbers them (refinement.cpp:275 and 308-317).
 *   k_ref_steiner per owned edge: metric mid-point and interpolated tensor,
 *                 boundary tag, and the edge -> vertex map entry
 *                 (refinement.cpp:267-297, Hashtable::push).
 *   k_ref_cut     per element with pattern > 0: 1->2, 1->3, 1->4 split with the
 *                 shorter-diagonal rule and atomic stencil appends
 *                 (Refine::cutElem, refinement.cpp:55-184).
 *
 * The edge -> Steiner vertex map is an open-addressing table keyed by the
 * vertex pair; like the reference's table (hashtable.h) it lives across all
 * levels of one refinement call and is cleared at its start.
 */
#include "trn_internal.h"
#include "trn_mixed.cuh"

#include <climits>

namespace trn {

static constexpr unsigned long long kEmpty = ~0ULL;

__device__ __forceinline__ unsigned long long edge_key(int a, int b) {
  int v = a < b ? a : b, w = a < b ? b : a;
  return ((unsigned long long) (unsigned) v << 32) | (unsigned) w;
}

__device__ __forceinline__ unsigned long long slot_of(unsigned long long key, unsigned long long mask) {
  return trn_hash64(key) & mask;
}

__device__ void h_insert(unsigned long long* hkey, int* hval, unsigned long long cap,
                         unsigned long long key, int id, int* err) {
  unsigned long long mask = cap - 1, s = slot_of(key, mask);
  for (unsigned long long probe = 0; probe < cap; ++probe) {
    unsigned long long prev = atomicCAS(hkey + s, kEmpty, key);
    if (prev == kEmpty || prev == key) {
      atomicMin(hval + s, id);
      return;
    }
    s = (s + 1) & mask;
  }
  trn_set_error(err, TRN_DERR_HASH);
}

__device__ int h_get(const unsigned long long* hkey, const int* hval, unsigned long long cap,
                     int a, int b) {
  unsigned long long key = edge_key(a, b), mask = cap - 1, s = slot_of(key, mask);
  for (unsigned long long probe = 0; probe < cap; ++probe) {
    unsigned long long k = hkey[s];
    if (k == key) return hval[s];
    if (k == kEmpty) return -1;
    s = (s + 1) & mask;
  }
  return -1;
}

/* Mesh::getElemNeigh, mesh.cpp:437-453: element != id holding edge j -> i */
__device__ __forceinline__ int elem_neigh(const DMesh& m, int id, int i, int j) {
  const int* s = m.stenc + (size_t) i * m.bucket;
  int d = trn_deg(m, i);
  for (int a = 0; a < d; ++a) {
    int t = s[a];
    if (t < 0) break;
    if (t != id) {
      int4 n = m.tri[t];
      if ((n.x == j && n.y == i) || (n.y == j && n.z == i) || (n.z == j && n.x == i)) return t;
    }
  }
  return -1;
}

template <bool F32>
__global__ void k_ref_filter(DMesh m, int nb_elems, int4* __restrict__ info,
                             long long* __restrict__ cnt) {
  nb_elems = trn_elems(m, nb_elems);
  if (trn_failed(m)) return;
  for (int i = trn_tid(); i < nb_elems; i += trn_grid_stride()) {
    int4 t = m.tri[i];
    if (t.x < 0) {
      info[i] = make_int4(0, -1, -1, -1);
      cnt[i] = 0;
      continue;
    }
    int n[3] = {t.x, t.y, t.z};
    double2 p[3] = {m.pts[n[0]], m.pts[n[1]], m.pts[n[2]]};
    const TenT<F32> q[3] = {ten_load<F32>(m, n[0]), ten_load<F32>(m, n[1]), ten_load<F32>(m, n[2])};
    int lmask = 0, pmask = 0;
    int opp[3] = {-1, -1, -1};
    for (int j = 0; j < 3; ++j) {
      int k = (j + 1) % 3;
      if (length_gt<F32>(p[j], p[k], q[j], q[k], TRN_L_MAX)) {
        lmask |= 1 << j;
        int o = elem_neigh(m, i, n[j], n[k]);
        opp[j] = o;
        if (n[j] < n[k] || o < 0) pmask |= 1 << j;
      }
    }
    info[i] = make_int4(lmask | (pmask << 3), opp[0], opp[1], opp[2]);
    cnt[i] = ((long long) __popc(pmask) << 32) | (long long) __popc(lmask);
  }
}

template <bool F32>
__global__ void k_ref_steiner(DMesh m, int nb_elems, int nb_nodes, const int4* __restrict__ info,
                              const long long* __restrict__ off, unsigned long long* hkey,
                              int* hval, unsigned long long hcap) {
  nb_elems = trn_elems(m, nb_elems); nb_nodes = trn_nodes(m, nb_nodes);
  if (trn_failed(m)) return;
  for (int i = trn_tid(); i < nb_elems; i += trn_grid_stride()) {
    int4 inf = info[i];
    int pmask = (inf.x >> 3) & 7;
    if (!pmask) continue;
    int4 t = m.tri[i];
    int n[3] = {t.x, t.y, t.z};
    int opp[3] = {inf.y, inf.z, inf.w};
    int id = nb_nodes + (int) (off[i] >> 32);
    for (int j = 0; j < 3; ++j) {
      if (!(pmask & (1 << j))) continue;
      int v1 = n[j], v2 = n[(j + 1) % 3];
      double2 rp;
      double rt[3];
      steiner_x<F32>(m.pts[v1], m.pts[v2], ten_load<F32>(m, v1), ten_load<F32>(m, v2), log_load<F32>(m, v1),
                     log_load<F32>(m, v2), &rp, rt);
      m.pts[id] = rp;
      ten_store<F32>(m, id, make_double4(rt[0], rt[1], rt[2], 0.0));
      log_store<F32>(m, id, log_of<F32>(rt[0], rt[1], rt[2]));
      if (opp[j] < 0) m.tags[id] = TRN_TAG_BOUND;
      h_insert(hkey, hval, hcap, edge_key(v1, v2), id, m.err);
      ++id;
    }
  }
}

__device__ __forceinline__ void put_tri(const DMesh& m, int id, int a, int b, int c) {
  m.tri[id] = make_int4(a, b, c, 0);
}

template <bool F32>
__global__ void k_ref_cut(DMesh m, int nb_elems, const int4* __restrict__ info,
                          const long long* __restrict__ off, const unsigned long long* hkey,
                          const int* hval, unsigned long long hcap) {
  nb_elems = trn_elems(m, nb_elems);
  if (trn_failed(m)) return;
  for (int id = trn_tid(); id < nb_elems; id += trn_grid_stride()) {
    int4 inf = info[id];
    int pattern = __popc(inf.x & 7);
    if (!pattern) continue;
    int4 tt = m.tri[id];
    int n[3] = {tt.x, tt.y, tt.z};
    const int s[3] = {h_get(hkey, hval, hcap, n[1], n[2]), h_get(hkey, hval, hcap, n[2], n[0]),
                      h_get(hkey, hval, hcap, n[0], n[1])};
    int offset = nb_elems + (int) (off[id] & 0xffffffffLL);
    if (pattern == 1) {
      const int t[2] = {id, offset};
      for (int i = 0; i < 3; ++i) {
        if (s[i] > -1) {
          int j = (i + 1) % 3, k = (i + 2) % 3;
          trn_stenc_append_n(m, s[i], t, 2);
          trn_stenc_append(m, n[i], t[1]);
          trn_stenc_append(m, n[k], t[1]);
          put_tri(m, t[0], n[i], n[j], s[i]);
          put_tri(m, t[1], n[i], s[i], n[k]);
          break;
        }
      }
    } else if (pattern == 2) {
      const int t[3] = {id, offset, offset + 1};
      for (int i = 0; i < 3; ++i) {
        if (s[i] < 0) {
          int j = (i + 1) % 3, k = (i + 2) % 3;
          /* a split count that disagrees with the edge map (possible only when
           * the two sides of an edge measure it differently) leaves the
           * element uncut instead of reading vertex -1 */
          if (s[j] < 0 || s[k] < 0) break;
          double diag0 = length_x<F32>(m.pts[n[j]], m.pts[s[j]], ten_load<F32>(m, n[j]), ten_load<F32>(m, s[j]));
          double diag1 = length_x<F32>(m.pts[n[k]], m.pts[s[k]], ten_load<F32>(m, n[k]), ten_load<F32>(m, s[k]));
          int v = (diag0 < diag1 ? j : k);
          int w = (v == j ? k : j);
          const int a3[3] = {t[0], t[1], t[2]};
          const int a2[2] = {t[0], t[2]};
          const int b2[2] = {t[1], t[2]};
          trn_stenc_append_n(m, s[v], a3, 3);
          trn_stenc_append_n(m, s[w], a2, 2);
          trn_stenc_append_n(m, n[v], b2, 2);
          trn_stenc_append(m, n[w], t[1]);
          put_tri(m, t[0], n[i], s[k], s[j]);
          put_tri(m, t[1], n[j], n[k], s[v]);
          put_tri(m, t[2], s[j], s[k], n[v]);
          break;
        }
      }
    } else {
      if (s[0] < 0 || s[1] < 0 || s[2] < 0) continue;
      const int t[4] = {id, offset, offset + 1, offset + 2};
      const int a0[3] = {t[1], t[2], t[3]};
      const int a1[3] = {t[0], t[2], t[3]};
      const int a2[3] = {t[0], t[1], t[3]};
      trn_stenc_append_n(m, s[0], a0, 3);
      trn_stenc_append_n(m, s[1], a1, 3);
      trn_stenc_append_n(m, s[2], a2, 3);
      trn_stenc_append(m, n[1], t[1]);
      trn_stenc_append(m, n[2], t[2]);
      put_tri(m, t[0], n[0], s[2], s[1]);
      put_tri(m, t[1], n[1], s[0], s[2]);
      put_tri(m, t[2], n[2], s[1], s[0]);
      put_tri(m, t[3], s[0], s[1], s[2]);
    }
  }
}

void refine_ws_alloc(RefineWs* ws, int capa_node, int capa_elem) {
  cudaMalloc(&ws->info, sizeof(int4) * (size_t) capa_elem);
  cudaMalloc(&ws->cnt, sizeof(long long) * (size_t) capa_elem);
  cudaMalloc(&ws->off, sizeof(long long) * (size_t) capa_elem);
  unsigned long long cap = 1024;
  while (cap < 2ULL * (unsigned long long) capa_node) cap <<= 1;
  ws->hcap = cap;
  cudaMalloc(&ws->hkey, sizeof(unsigned long long) * cap);
  cudaMalloc(&ws->hval, sizeof(int) * cap);
}

void refine_ws_free(RefineWs* ws) {
  cudaFree(ws->info);
  cudaFree(ws->cnt);
  cudaFree(ws->off);
  cudaFree(ws->hkey);
  cudaFree(ws->hval);
  *ws = RefineWs();
}

/* before a level's splits: a level that would overflow the capacity raises
 * the error word, and every later kernel of the call does nothing */
__global__ void k_ref_check(DMesh m, const long long* total) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const long long tot = *total;
  const long long split = tot >> 32, adds = tot & 0xffffffffLL;
  if ((long long) m.nb[0] + split > m.capa_node || (long long) m.nb[1] + adds > m.capa_elem)
    trn_set_error(m.err, TRN_DERR_CAPACITY);
}

/* after a level's splits: the new slot counts (new vertices and elements are
 * numbered after the old ones) and the call's statistics in stats[0..2]:
 * elements examined by each level up to the first that splits nothing,
 * elements added, and that level's flag */
__global__ void k_ref_commit(DMesh m, const long long* total, int* stats) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (trn_failed(m)) return;
  const long long tot = *total;
  const int split = (int) (tot >> 32), adds = (int) (tot & 0xffffffffLL);
  if (!stats[2]) {
    stats[0] += m.nb[1];
    stats[1] += adds;
    if (adds == 0) stats[2] = 1;
  }
  m.nb[0] += split;
  m.nb[1] += adds;
}

void refine_level(const DMesh& m, int hint_nodes, int hint_elems, RefineWs& ws, ScanWs& scan,
                  int* stats, bool fp32, cudaStream_t s) {
  refine_filter(m, hint_elems, ws, fp32, s);
  scan_i64(ws.cnt, ws.off, hint_elems, scan, s, m.nb + 1);
  k_ref_check<<<1, 32, 0, s>>>(m, scan.total);
  note_launch();
  refine_apply(m, hint_nodes, hint_elems, ws, fp32, s);
  k_ref_commit<<<1, 32, 0, s>>>(m, scan.total, stats);
  note_launch();
  check_launch("refine_level");
}

void refine_reset_hash(RefineWs& ws, cudaStream_t s) {
  cudaMemsetAsync(ws.hkey, 0xff, sizeof(unsigned long long) * ws.hcap, s);
  cudaMemsetAsync(ws.hval, 0x7f, sizeof(int) * ws.hcap, s);
}

void refine_filter(const DMesh& m, int nb_elems, RefineWs& ws, bool fp32, cudaStream_t s) {
  ProfScope ps("refine_filter", s, (double) nb_elems * (kTri + 16 + 8) + (double) nb_elems / 2 * (kPt + kTen));
  if (fp32) k_ref_filter<true><<<TRN_RESIDENT(k_ref_filter<true>, grid_for(nb_elems), TRN_THREADS), TRN_THREADS, 0, s>>>(m, nb_elems, ws.info, ws.cnt);
  else k_ref_filter<false><<<TRN_RESIDENT(k_ref_filter<false>, grid_for(nb_elems), TRN_THREADS), TRN_THREADS, 0, s>>>(m, nb_elems, ws.info, ws.cnt);
  note_launch();
  check_launch("refine_filter");
}

void refine_apply(const DMesh& m, int nb_nodes, int nb_elems, RefineWs& ws, bool fp32, cudaStream_t s) {
  {
  ProfScope ps("refine_steiner", s, (double) nb_elems * (16 + 8));
  if (fp32)
    k_ref_steiner<true><<<grid_for(nb_elems), TRN_THREADS, 0, s>>>(m, nb_elems, nb_nodes, ws.info, ws.off,
                                                                  ws.hkey, ws.hval, ws.hcap);
  else
    k_ref_steiner<false><<<grid_for(nb_elems), TRN_THREADS, 0, s>>>(m, nb_elems, nb_nodes, ws.info, ws.off,
                                                                   ws.hkey, ws.hval, ws.hcap);
  note_launch();
  }
  ProfScope ps("refine_cut", s, (double) nb_elems * (16 + 8 + kTri));
  if (fp32)
    k_ref_cut<true><<<TRN_RESIDENT(k_ref_cut<true>, grid_for(nb_elems), TRN_THREADS), TRN_THREADS, 0, s>>>(m, nb_elems, ws.info, ws.off, ws.hkey,
                                                              ws.hval, ws.hcap);
  else
    k_ref_cut<false><<<TRN_RESIDENT(k_ref_cut<false>, grid_for(nb_elems), TRN_THREADS), TRN_THREADS, 0, s>>>(m, nb_elems, ws.info, ws.off, ws.hkey,
                                                               ws.hval, ws.hcap);
  note_launch();
  check_launch("refine_apply");
}

}  // namespace trn
