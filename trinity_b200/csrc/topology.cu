/*
 * topology.cu — incidence build and repair.
 *
 *   k_count_fill   : vertex -> element stencils from the triangle array
 *                    (Mesh::rebuildTopology, mesh.cpp:197-210: atomic append)
 *   k_sort_stencil : sort each stencil (mesh.cpp:244)
 *   k_build_vicin  : sorted unique vertex adjacency from the stencil
 *                    (mesh.cpp:214-243 and Mesh::extractPrimalGraph 297-330)
 *   k_fix_tagged   : the fused stencil repair of Mesh::fixTagged
 *                    (mesh.cpp:716-760): keep the entries whose element still
 *                    holds the vertex, sort, drop duplicates, in one pass over
 *                    the vertex's bucket held in registers/local memory.
 */
#include "trn_internal.h"

#include <algorithm>
#include "trn_mixed.cuh"

namespace trn {

__global__ void k_fill_stencils(DMesh m, int nb_elems) {
  for (int i = trn_tid(); i < nb_elems; i += trn_grid_stride()) {
    int4 t = m.tri[i];
    if (t.x < 0) continue;
    trn_stenc_append(m, t.x, i);
    trn_stenc_append(m, t.y, i);
    trn_stenc_append(m, t.z, i);
  }
}

__global__ void k_sort_stencils(DMesh m, int nb_nodes) {
  if (trn_failed(m)) return;
  int buf[TRN_MAX_DEG];
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) {
    int d = trn_deg(m, v);
    int* s = m.stenc + (size_t) v * m.bucket;
    for (int a = 0; a < d; ++a) buf[a] = s[a];
    trn_isort(buf, d);
    for (int a = 0; a < d; ++a) s[a] = buf[a];
  }
}

__global__ void k_build_vicin(DMesh m, int nb_nodes, int only_flagged) {
  nb_nodes = trn_nodes(m, nb_nodes);
  if (trn_failed(m)) return;
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) {
    if (only_flagged && m.activ[v] == 0) continue;
    build_one_vicin(m, v);
  }
}

/* repair of one tagged stencil (Mesh::fixTagged, mesh.cpp:716-760): keep the
 * entries whose element still holds v, sorted, without duplicates. Stencils
 * of up to 16 entries stay in registers (the element loads all in flight at
 * once, a sorting network, no local memory); longer ones take the scratch
 * array. Both give the same entries in the same order. */
constexpr int kFixRegs = 16;

__device__ __forceinline__ void fix_stencil(const DMesh& m, int v, int* buf) {
  int* s = m.stenc + (size_t) v * m.bucket;
  const int d = trn_deg(m, v);
  int k = 0;
  if (d <= kFixRegs) {
    int r[kFixRegs];
#pragma unroll
    for (int a = 0; a < kFixRegs; ++a) r[a] = (a < d) ? s[a] : -1;
#pragma unroll
    for (int a = 0; a < kFixRegs; ++a) {
      int keep = 0x7fffffff;
      if (r[a] >= 0) {
        const int4 nn = m.tri[r[a]];
        if (v == nn.x || v == nn.y || v == nn.z) keep = r[a];
      }
      r[a] = keep;
    }
#pragma unroll
    for (int p = 0; p < kFixRegs; ++p)
#pragma unroll
      for (int a = p & 1; a + 1 < kFixRegs; a += 2) {
        const int lo = min(r[a], r[a + 1]), hi = max(r[a], r[a + 1]);
        r[a] = lo;
        r[a + 1] = hi;
      }
#pragma unroll
    for (int a = 0; a < kFixRegs; ++a)
      if (r[a] != 0x7fffffff && (a == 0 || r[a] != r[a - 1])) s[k++] = r[a];
  } else {
    for (int a = 0; a < d; ++a) {
      const int t = s[a];
      if (t < 0) continue;
      const int4 nn = m.tri[t];
      if (v == nn.x || v == nn.y || v == nn.z) buf[k++] = t;
    }
    trn_isort(buf, k);
    k = trn_iunique(buf, k);
    for (int a = 0; a < k; ++a) s[a] = buf[a];
  }
  for (int a = k; a < d; ++a) s[a] = -1;
  m.deg[v] = k;
}

__global__ void k_fix_tagged(DMesh m, int nb_nodes) {
  nb_nodes = trn_nodes(m, nb_nodes);
  if (trn_failed(m)) return;
  int buf[TRN_MAX_DEG];
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) {
    if (!m.fixes[v]) continue;
    m.fixes[v] = 0;
    fix_stencil(m, v, buf);
  }
}

/* The repair of the listed vertices and the end of a free-mode coarsening
 * or swapping level, in one launch (they touch disjoint state). A level
 * reads the list of active entities in one buffer and appends the ones it
 * re-activates to another; the level's end moves the new list into the
 * first buffer (so every level runs the same kernels on the same buffers),
 * and its first thread accumulates the call's statistics, bounds the number
 * of levels, advances the seed counter and decides whether another level
 * runs (level_end_decide): for a coarsening level, while it found
 * candidates and collapsed some (the loop of Coarse::run,
 * coarsening.cpp:480-503); for a swapping level, while it flipped some
 * (Swap::run, swapping.cpp:395-425). The host-driven loop reads that
 * decision back; a captured round hands it to the loop node. The level end
 * runs even after an error (a captured loop must still read its condition,
 * which then stops it). */
__global__ void k_fix_level_end(DMesh m, const int* __restrict__ list, const int* count, int* status, int kind,
                                int cap, const int* __restrict__ next, int* __restrict__ cur,
                                cudaGraphConditionalHandle h, int use_h) {
  const int na = status[S_ACT + 1];
  for (int i = trn_tid(); i < na; i += trn_grid_stride()) cur[i] = next[i];
  if (threadIdx.x == 0 && blockIdx.x == 0) level_end_decide(status, kind, cap, h, use_h);
  if (trn_failed(m)) return;
  int buf[TRN_MAX_DEG];
  const int n = *count;
  for (int q = trn_tid(); q < n; q += trn_grid_stride()) {
    const int v = list[q];
    if (!m.fixes[v]) continue;
    m.fixes[v] = 0;
    fix_stencil(m, v, buf);
  }
}

void fix_list_level_end(const DMesh& m, const int* list, const int* count, long long bound, int* status,
                        int kind, int cap, const int* next, int* cur, int hint, cudaStream_t s,
                        cudaGraphConditionalHandle h, bool use_h) {
  ProfScope ps("fix_tagged", s, 0.0);
  const int g = std::max(grid_bounded(bound, m.capa_node), grid_for(hint));
  k_fix_level_end<<<g, TRN_THREADS, 0, s>>>(m, list, count, status, kind, cap, next, cur, h, use_h ? 1 : 0);
  note_launch();
  check_launch("fix_list_level_end");
}


__global__ void k_flag_alive(DMesh m, int nb_nodes) {
  nb_nodes = trn_nodes(m, nb_nodes);
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) m.fixes[v] = m.alive[v] ? 1 : 0;
}

/* cached quality of every live element (swapping.cpp:167-174, smoothing.cpp:145-151) */
template <bool F32>
__global__ void k_quality_all(DMesh m, int nb_elems) {
  nb_elems = trn_elems(m, nb_elems);
  if (trn_failed(m)) return;
  for (int i = trn_tid(); i < nb_elems; i += trn_grid_stride()) {
    int4 t = m.tri[i];
    if (t.x < 0) continue;
    m.qual[i] = quality_of<F32>(m, t);
  }
}

__global__ void k_count_live(DMesh m, int nb_nodes, int nb_elems, int* out) {
  int cv = 0, ce = 0;
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) cv += m.alive[v] ? 1 : 0;
  for (int i = trn_tid(); i < nb_elems; i += trn_grid_stride()) ce += m.tri[i].x >= 0 ? 1 : 0;
  for (int o = 16; o > 0; o >>= 1) {
    cv += __shfl_down_sync(0xffffffffu, cv, o);
    ce += __shfl_down_sync(0xffffffffu, ce, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (cv) atomicAdd(out, cv);
    if (ce) atomicAdd(out + 1, ce);
  }
}

/* input triangles (3 x int, 0-based) -> int4 records, checking indices */
__global__ void k_expand_tris(const int* __restrict__ raw, int nb_elems, int nb_nodes,
                              int4* __restrict__ out, int* err) {
  for (int i = trn_tid(); i < nb_elems; i += trn_grid_stride()) {
    int a = raw[3 * i], b = raw[3 * i + 1], c = raw[3 * i + 2];
    if (a < 0 || a >= nb_nodes || b < 0 || b >= nb_nodes || c < 0 || c >= nb_nodes) {
      trn_set_error(err, TRN_DERR_INVALID);
      a = b = c = -1;
    }
    out[i] = make_int4(a, b, c, 0);
  }
}

void expand_tris(const int* raw, int nb_elems, int nb_nodes, int4* out, int* err, cudaStream_t s) {
  k_expand_tris<<<grid_for(nb_elems), TRN_THREADS, 0, s>>>(raw, nb_elems, nb_nodes, out, err);
  note_launch();
}

/* Mesh::store's renumbering (io.cpp:199-233) on the device: live vertex k of
 * the ordered list gets id k; its point and tensor are packed */
__global__ void k_pack_nodes(DMesh m, const int* __restrict__ list, const int* count,
                             int* __restrict__ newid, double* __restrict__ pts, double* __restrict__ ten) {
  const int n = *count;
  for (int k = trn_tid(); k < n; k += trn_grid_stride()) {
    const int v = list[k];
    newid[v] = k;
    const double2 p = m.pts[v];
    const double4 t = m.ten[v];
    pts[2 * k] = p.x;
    pts[2 * k + 1] = p.y;
    if (ten) {
      ten[3 * k] = t.x;
      ten[3 * k + 1] = t.y;
      ten[3 * k + 2] = t.z;
    }
  }
}

__global__ void k_flag_live_tris(DMesh m, int nb_elems, uint8_t* __restrict__ flag) {
  for (int i = trn_tid(); i < nb_elems; i += trn_grid_stride()) flag[i] = m.tri[i].x >= 0 ? 1 : 0;
}

__global__ void k_pack_tris(DMesh m, const int* __restrict__ list, const int* count,
                            const int* __restrict__ newid, int* __restrict__ out) {
  const int n = *count;
  for (int k = trn_tid(); k < n; k += trn_grid_stride()) {
    const int4 t = m.tri[list[k]];
    out[3 * k] = newid[t.x];
    out[3 * k + 1] = newid[t.y];
    out[3 * k + 2] = newid[t.z];
  }
}

/* the live vertices and elements as a freshly loaded mesh: points and tags
 * of the listed vertices, elements renumbered into int4 records */
__global__ void k_pack_nodes_load(DMesh m, const int* __restrict__ list, const int* count,
                                  int* __restrict__ newid, double2* __restrict__ pts,
                                  uint8_t* __restrict__ tags) {
  const int n = *count;
  for (int k = trn_tid(); k < n; k += trn_grid_stride()) {
    const int v = list[k];
    newid[v] = k;
    pts[k] = m.pts[v];
    tags[k] = m.tags[v];
  }
}

__global__ void k_pack_tris_load(DMesh m, const int* __restrict__ list, const int* count,
                                 const int* __restrict__ newid, int4* __restrict__ out) {
  const int n = *count;
  for (int k = trn_tid(); k < n; k += trn_grid_stride()) {
    const int4 t = m.tri[list[k]];
    out[k] = make_int4(newid[t.x], newid[t.y], newid[t.z], 0);
  }
}

void pack_nodes_load(const DMesh& m, const int* list, const int* count, int* newid, double2* pts,
                     uint8_t* tags, cudaStream_t s) {
  k_pack_nodes_load<<<grid_for(m.capa_node), TRN_THREADS, 0, s>>>(m, list, count, newid, pts, tags);
  note_launch();
}

void pack_tris_load(const DMesh& m, const int* list, const int* count, const int* newid, int4* out,
                    cudaStream_t s) {
  k_pack_tris_load<<<grid_for(m.capa_elem), TRN_THREADS, 0, s>>>(m, list, count, newid, out);
  note_launch();
}

void pack_nodes(const DMesh& m, const int* list, const int* count, int* newid, double* pts, double* ten,
                cudaStream_t s) {
  k_pack_nodes<<<grid_for(m.capa_node), TRN_THREADS, 0, s>>>(m, list, count, newid, pts, ten);
  note_launch();
}

void flag_live_tris(const DMesh& m, int nb_elems, uint8_t* flag, cudaStream_t s) {
  k_flag_live_tris<<<grid_for(nb_elems), TRN_THREADS, 0, s>>>(m, nb_elems, flag);
  note_launch();
}

void pack_tris(const DMesh& m, const int* list, const int* count, const int* newid, int* out,
               cudaStream_t s) {
  k_pack_tris<<<grid_for(m.capa_elem), TRN_THREADS, 0, s>>>(m, list, count, newid, out);
  note_launch();
}

void count_live(const DMesh& m, int nb_nodes, int nb_elems, int* out, cudaStream_t s) {
  cudaMemsetAsync(out, 0, sizeof(int) * 2, s);
  k_count_live<<<grid_for(nb_elems), TRN_THREADS, 0, s>>>(m, nb_nodes, nb_elems, out);
  note_launch();
}

void build_stencils(const DMesh& m, int nb_nodes, int nb_elems, cudaStream_t s) {
  ProfScope ps("build_stencils", s, 3.0 * nb_elems * (kTri + 2 * kIdx) + 2.0 * nb_nodes * kIdx);
  cudaMemsetAsync(m.deg, 0, sizeof(int) * (size_t) m.capa_node, s);
  k_fill_stencils<<<TRN_RESIDENT(k_fill_stencils, grid_for(nb_elems), TRN_THREADS), TRN_THREADS, 0, s>>>(m, nb_elems);
  note_launch();
  k_sort_stencils<<<TRN_RESIDENT(k_sort_stencils, grid_for(nb_nodes), TRN_THREADS), TRN_THREADS, 0, s>>>(m, nb_nodes);
  note_launch();
  check_launch("build_stencils");
}

void build_vicin(const DMesh& m, int nb_nodes, bool only_flagged, cudaStream_t s) {
  ProfScope ps("build_vicin", s, (double) nb_nodes * (1 + 2 * kIdx + kAvgDeg * (kIdx + kTri + kIdx)));
  k_build_vicin<<<TRN_RESIDENT(k_build_vicin, grid_for(nb_nodes), TRN_THREADS), TRN_THREADS, 0, s>>>(m, nb_nodes, only_flagged ? 1 : 0);
  note_launch();
  check_launch("build_vicin");
}

void fix_tagged(const DMesh& m, int nb_nodes, cudaStream_t s) {
  ProfScope ps("fix_tagged", s, (double) nb_nodes);
  k_fix_tagged<<<TRN_RESIDENT(k_fix_tagged, grid_for(nb_nodes), TRN_THREADS), TRN_THREADS, 0, s>>>(m, nb_nodes);
  note_launch();
  check_launch("fix_tagged");
}

void flag_all_alive(const DMesh& m, int nb_nodes, cudaStream_t s) {
  k_flag_alive<<<grid_for(nb_nodes), TRN_THREADS, 0, s>>>(m, nb_nodes);
  note_launch();
}

/* the per-vertex logarithm cache of the FP32 form, from the stored tensors */
__global__ void k_log_cache_f32(DMesh m, int nb_nodes) {
  nb_nodes = trn_nodes(m, nb_nodes);
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) {
    const double4 t = m.ten[v];
    log_store<true>(m, v, log_of<true>(t.x, t.y, t.z));
    m.tenf[v] = tenf_of(t);
  }
}

__global__ void k_log_cache_f64(DMesh m, int nb_nodes) {
  nb_nodes = trn_nodes(m, nb_nodes);
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) {
    const double4 t = m.ten[v];
    m.lten[v] = trn_log_tensor(t.x, t.y, t.z);
  }
}

void log_cache(const DMesh& m, int nb_nodes, bool fp32, cudaStream_t s) {
  if (fp32) k_log_cache_f32<<<TRN_RESIDENT(k_log_cache_f32, grid_for(nb_nodes), TRN_THREADS), TRN_THREADS, 0, s>>>(m, nb_nodes);
  else k_log_cache_f64<<<TRN_RESIDENT(k_log_cache_f64, grid_for(nb_nodes), TRN_THREADS), TRN_THREADS, 0, s>>>(m, nb_nodes);
  note_launch();
}

void quality_all(const DMesh& m, int nb_elems, bool fp32, cudaStream_t s) {
  ProfScope ps("quality_all", s, (double) nb_elems * (kTri + kQ) + (double) nb_elems / 2 * (kPt + kTen));
  if (fp32) k_quality_all<true><<<TRN_RESIDENT(k_quality_all<true>, grid_for(nb_elems), TRN_THREADS), TRN_THREADS, 0, s>>>(m, nb_elems);
  else k_quality_all<false><<<TRN_RESIDENT(k_quality_all<false>, grid_for(nb_elems), TRN_THREADS), TRN_THREADS, 0, s>>>(m, nb_elems);
  note_launch();
  check_launch("quality_all");
}

}  // namespace trn
