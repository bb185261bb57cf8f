/*
 * smooth.cu — anisotropic smart-Laplacian smoothing (Smooth::run,
 * smoothing.cpp:274-302).
 *
 *   k_smooth_pre   live vertices: interior ones active, boundary ones not
 *                  (smoothing.cpp:129-142)
 *   k_smooth_move  one launch per color class: every listed interior vertex
 *                  moves to the mean over its neighbours b of
 *                  p_a + (p_b - p_a)/L_M(a,b), takes the log-Euclidean mean of
 *                  the neighbours' tensors, and keeps the move only if every
 *                  incident element stays CCW with quality above the old
 *                  stencil minimum, backing off the step 1, 1/2, .., 1/16
 *                  (Smooth::moveSmartLaplacian, smoothing.cpp:40-126).
 *   k_smooth_move_grp  the same with 2, 4 or 8 lanes per vertex (launch shape
 *                  smooth_lanes; the same results)
 * Vertices of one color share no element, so a class moves in parallel; the
 * classes run in order, as in the reference.
 */
#include "trn_internal.h"
#include "trn_mixed.cuh"

#include <algorithm>

namespace trn {

__global__ void k_smooth_pre(DMesh m, int nb_nodes) {
  nb_nodes = trn_nodes(m, nb_nodes);
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride())
    if (m.alive[v]) m.activ[v] = (m.tags[v] & TRN_TAG_BOUND) ? 0 : 1;
}

/* Element metrics of the back-off: the log-Euclidean mean of an element's
 * three tensors (and the square root of its determinant) does not depend on
 * where the moved vertex sits, only on its new tensor, so it is computed once
 * per stencil element before the tries and kept in shared memory (kj slots a
 * thread, stride blockDim.x so that a warp's slots are contiguous); the
 * tries only redo the geometry. Elements past the kj-th (rare: long
 * stencils) take the metric inline. Same operations, same bits as
 * evaluating the whole quality in every try. */
template <bool F32>
using JmT = LogT<F32>;

template <bool F32>
__device__ int move_laplacian(const DMesh& m, int i, JmT<F32>* jc, int kj) {
  const int* vc = m.vic + (size_t) i * m.bucket;
  const int* st = m.stenc + (size_t) i * m.bucket;
  const int deg = trn_deg(m, i);
  const int nb_neigh = m.vdeg[i];
  double q_min = 1.7976931348623157e308;
  for (int a = 0; a < deg; ++a) q_min = trn_dmin(q_min, m.qual[st[a]]);
  const double2 pini = m.pts[i];
  const double4 tini = m.ten[i];
  const TenT<F32> tinf = ten_load<F32>(m, i);
  const LogT<F32> lini = log_load<F32>(m, i);
  double ox = 0, oy = 0;
  LogSum<F32> lsum;
  if constexpr (F32) {
    /* the mean displacement in single precision, added to the FP64 point */
    float dx = 0.f, dy = 0.f;
    for (int k = 0; k < nb_neigh; ++k) {
      const int nb = vc[k];
      const double2 pb = m.pts[nb];
      const float il = __frcp_rn(trnf_dist2(pini, pb, tenf_of(tinf), tenf_of(ten_load<F32>(m, nb))));
      dx += (float) (pb.x - pini.x) * il;
      dy += (float) (pb.y - pini.y) * il;
      lsum.add(log_load<F32>(m, nb));
    }
    const float inv = __frcp_rn((float) nb_neigh);
    ox = pini.x + (double) (dx * inv);
    oy = pini.y + (double) (dy * inv);
  } else {
    for (int k = 0; k < nb_neigh; ++k) {
      const int nb = vc[k];
      const double2 pb = m.pts[nb];
      const double4 tb = m.ten[nb];
      const double len = length_x<F32>(pini, pb, tini, tb);
      ox += pini.x + ((pb.x - pini.x) / len);
      oy += pini.y + ((pb.y - pini.y) / len);
      lsum.add(log_load<F32>(m, nb));
    }
    ox /= nb_neigh;
    oy /= nb_neigh;
  }
  double tn[3];
  lsum.finish(nb_neigh, tn);
  const double4 tnew = make_double4(tn[0], tn[1], tn[2], 0.0);
  const LogT<F32> lnew = log_of<F32>(tn[0], tn[1], tn[2]);
  ten_store<F32>(m, i, tnew);
  log_store<F32>(m, i, lnew);
  const int nj = deg < kj ? deg : kj;
  for (int a = 0; a < nj; ++a) {
    const int4 n = m.tri[st[a]];
    const LogT<F32> l0 = (n.x == i) ? lnew : log_load<F32>(m, n.x);
    const LogT<F32> l1 = (n.y == i) ? lnew : log_load<F32>(m, n.y);
    const LogT<F32> l2 = (n.z == i) ? lnew : log_load<F32>(m, n.z);
    jc[(size_t) a * blockDim.x] = qmetric_x(l0, l1, l2);
  }
  double qual[TRN_MAX_DEG];
  bool valid;
  int retry = 0;
  double weight = 1;
  do {
    valid = true;
    double2 pa;
    pa.x = (1 - weight) * pini.x + weight * ox;
    pa.y = (1 - weight) * pini.y + weight * oy;
    m.pts[i] = pa;
    for (int a = 0; valid && a < deg; ++a) {
      const int4 n = m.tri[st[a]];
      const double2 p0 = (n.x == i) ? pa : m.pts[n.x];
      const double2 p1 = (n.y == i) ? pa : m.pts[n.y];
      const double2 p2 = (n.z == i) ? pa : m.pts[n.z];
      valid = false;
      if (trn_ccw(p0, p1, p2)) {
        JmT<F32> jm;
        if (a < nj) {
          jm = jc[(size_t) a * blockDim.x];
        } else {
          const LogT<F32> l0 = (n.x == i) ? lnew : log_load<F32>(m, n.x);
          const LogT<F32> l1 = (n.y == i) ? lnew : log_load<F32>(m, n.y);
          const LogT<F32> l2 = (n.z == i) ? lnew : log_load<F32>(m, n.z);
          jm = qmetric_x(l0, l1, l2);
        }
        qual[a] = qgeom_x(p0, p1, p2, jm);
        valid = (qual[a] > q_min);
      }
    }
    weight *= 0.5;
  } while (!valid && ++retry < 5);
  if (valid) {
    for (int a = 0; a < deg; ++a) m.qual[st[a]] = qual[a];
  } else {
    m.pts[i] = pini;
    ten_store<F32>(m, i, tini);
    log_store<F32>(m, i, lini);
  }
  return valid ? 1 : 0;
}

/* the algorithmic bytes of one listed vertex (profiled runs only): its list
 * entry and flags; when it moves, its own point, tensor and logarithm read
 * and written, its stencil and adjacency rows, its elements' records and
 * qualities (read and written), and the point, tensor and logarithm of each
 * neighbour that no other vertex of the launch has counted yet (a bitmap
 * over the vertices keeps them distinct) */
template <bool F32>
__device__ unsigned long long smooth_bytes(const DMesh& m, int v, bool moved, unsigned* seen) {
  constexpr unsigned long long kTenB = F32 ? 16 + 32 : 32;   /* FP32 reads its copy, writes both */
  constexpr unsigned long long kLogB = F32 ? 16 : 32;
  unsigned long long b = 4 + 1 + 4;
  if (!moved) return b;
  const int deg = trn_deg(m, v), nv = m.vdeg[v];
  b += 4 + 2 * (16 + kTenB + kLogB);
  b += (unsigned long long) deg * (4 + 16 + 8 + 8) + (unsigned long long) nv * 4;
  const int* vc = m.vic + (size_t) v * m.bucket;
  for (int k = 0; k < nv; ++k) {
    const int w = vc[k];
    const unsigned bit = 1u << (w & 31);
    if (!(atomicOr(seen + (w >> 5), bit) & bit)) b += 16 + (F32 ? 16 : 32) + kLogB;
  }
  return b;
}

/* MinB: 256-thread blocks an SM the registers are capped for (2: up to 128,
 * 3: 80, 4: 64); more warps hide more of the gathers' latency, at the cost of
 * spills */
template <bool F32, int MinB>
__global__ void __launch_bounds__(256, MinB) k_smooth_move(DMesh m, const int* __restrict__ list,
                                                                   int n, const int* off, int c, int* counters,
                                                                   int kj, ByteCount bc) {
  extern __shared__ __align__(16) unsigned char smooth_smem[];
  JmT<F32>* jc = reinterpret_cast<JmT<F32>*>(smooth_smem) + threadIdx.x;
  if (trn_failed(m)) return;
  if (off) {   /* color class c of a device-side partition */
    list += off[c];
    n = off[c + 1] - off[c];
  }
  int tasks = 0, commit = 0;
  unsigned long long bytes = 0;
  for (int q = trn_tid(); q < n; q += trn_grid_stride()) {
    const int v = list[q];
    if (v < 0 || v >= m.capa_node) {
      trn_set_error(m.err, TRN_DERR_REPLAY);
      continue;
    }
    const bool moved = m.activ[v] && m.vdeg[v] != 0;
    if (bc.bytes) bytes += smooth_bytes<F32>(m, v, moved, bc.seen);
    if (!moved) continue;
    tasks++;
    commit += move_laplacian<F32>(m, v, jc, kj);
  }
  trn_warp_add(counters, tasks);
  trn_warp_add(counters + 1, commit);
  if (bytes) atomicAdd(bc.bytes, bytes);
}

/* The same move with G lanes per vertex: lane j gathers the neighbours
 * j, j+G, ... and evaluates the elements j, j+G, ... of the stencil. The
 * displacement and the tensor-logarithm sums are accumulated in neighbour
 * order by every lane from the lanes' terms (shuffles), the stencil minimum
 * is a min-reduction and validity an all-vote, so the results are the bits
 * of move_laplacian. More loads in flight per vertex and no per-thread
 * quality array: the one-lane form is bound by gather latency, divergence
 * and registers. */
template <class T>
__device__ __forceinline__ T grp_shfl(unsigned mask, T v, int src, int width);
template <>
__device__ __forceinline__ double grp_shfl(unsigned mask, double v, int src, int width) {
  return __shfl_sync(mask, v, src, width);
}
template <>
__device__ __forceinline__ float grp_shfl(unsigned mask, float v, int src, int width) {
  return __shfl_sync(mask, v, src, width);
}
template <>
__device__ __forceinline__ double4 grp_shfl(unsigned mask, double4 v, int src, int width) {
  return make_double4(__shfl_sync(mask, v.x, src, width), __shfl_sync(mask, v.y, src, width),
                      __shfl_sync(mask, v.z, src, width), __shfl_sync(mask, v.w, src, width));
}
template <>
__device__ __forceinline__ float4 grp_shfl(unsigned mask, float4 v, int src, int width) {
  return make_float4(__shfl_sync(mask, v.x, src, width), __shfl_sync(mask, v.y, src, width),
                     __shfl_sync(mask, v.z, src, width), __shfl_sync(mask, v.w, src, width));
}

/* quality of stencil element t of vertex i with i at pa (log lnew); false
 * when it is not CCW */
template <bool F32>
__device__ __forceinline__ bool elem_quality_at(const DMesh& m, int i, int4 n, double2 pa, LogT<F32> lnew,
                                                double* q) {
  const double2 p0 = (n.x == i) ? pa : m.pts[n.x];
  const double2 p1 = (n.y == i) ? pa : m.pts[n.y];
  const double2 p2 = (n.z == i) ? pa : m.pts[n.z];
  if (!trn_ccw(p0, p1, p2)) return false;
  const LogT<F32> l0 = (n.x == i) ? lnew : log_load<F32>(m, n.x);
  const LogT<F32> l1 = (n.y == i) ? lnew : log_load<F32>(m, n.y);
  const LogT<F32> l2 = (n.z == i) ? lnew : log_load<F32>(m, n.z);
  *q = quality_x(p0, p1, p2, l0, l1, l2);
  return true;
}

/* a[j] of a small register array, j known only at run time: predicated
 * selects, so the array stays in registers */
template <int K, class T>
__device__ __forceinline__ T reg_pick(const T (&a)[K], int j) {
  T r = a[0];
#pragma unroll
  for (int k = 1; k < K; ++k)
    if (j == k) r = a[k];
  return r;
}

template <int K, class T>
__device__ __forceinline__ void reg_put(T (&a)[K], int j, T v) {
#pragma unroll
  for (int k = 0; k < K; ++k)
    if (j == k) a[k] = v;
}

/* The moved vertex's new tensor (the exponentiated mean of its neighbours'
 * logarithms) and its logarithm, computed by every lane of a group: the two
 * eigenvalues' exp (log) go to the two lanes of a pair, one each, and are
 * swapped by a shuffle, so the group issues one transcendental chain where
 * it issued two. Same functions on the same inputs, composed as
 * trn_interp_finish / trn_log_tensor do: the same bits. FP64 form. */
template <int G>
__device__ __forceinline__ void finish_pair(double* lm, int nb, double* res, int lane, unsigned gmask) {
  double val[2], vec[4], cache[4];
  for (int i = 0; i < 4; ++i) lm[i] /= nb;
  trn_eigen(lm, val, vec);
  const bool h = lane & 1;
  const double mine = trn_exp(h ? val[1] : val[0]);
  const double other = __shfl_xor_sync(gmask, mine, 1, G);
  val[0] = h ? other : mine;
  val[1] = h ? mine : other;
  trn_eigen_compose(val, vec, cache);
  res[0] = cache[0];
  res[1] = cache[1];
  res[2] = cache[3];
}

template <int G>
__device__ __forceinline__ double4 log_pair(double t0, double t1, double t2, int lane, unsigned gmask) {
  double copy[4] = {t0, t1, t1, t2}, val[2], vec[4], cache[4];
  trn_eigen(copy, val, vec);
  const bool h = lane & 1;
  const double mine = trn_log(h ? val[1] : val[0]);
  const double other = __shfl_xor_sync(gmask, mine, 1, G);
  val[0] = h ? other : mine;
  val[1] = h ? mine : other;
  trn_eigen_compose(val, vec, cache);
  return make_double4(cache[0], cache[1], cache[2], cache[3]);
}

/* V selects how the back-off runs:
 *   0  the tries in turn, element metrics in registers;
 *   1  the same with the element metrics in shared memory (KQ slots a
 *      thread, stride blockDim.x) and the lane's element records prefetched
 *      into L1 while the stencil minimum is read;
 *   2  one sweep over the lane's elements evaluates all five tries (the
 *      element's points loaded once, five independent geometry chains), the
 *      group ANDs the lanes' five-bit pass masks and keeps the first try that
 *      passes; the qualities wait in shared memory (5 x KQ a thread). A
 *      warp of 8 groups almost always runs all five tries in turn anyway
 *      (half the moves fail every try), so this costs no extra issue and
 *      turns a serial chain into parallel ones. Same tries, same arithmetic,
 *      same first passing try: the same bits;
 *   3  the sweep of 2 with the element metrics in shared memory too (before
 *      the qualities), which frees the registers the five chains need. */
template <bool F32, int G, int V>
__device__ int move_laplacian_grp(const DMesh& m, int i, int lane, unsigned gmask, unsigned char* smem) {
  static_assert(G >= 2, "lane groups of two or more");
  constexpr bool JS = V == 1 || V == 3;
  constexpr bool SW = V >= 2;
  constexpr int KQ = G >= 4 ? 2 : 3;
  JmT<F32>* js = reinterpret_cast<JmT<F32>*>(smem) + threadIdx.x;
  double* qs = reinterpret_cast<double*>(smem + (JS ? (size_t) KQ * blockDim.x * sizeof(JmT<F32>) : 0)) +
               threadIdx.x;
  const int* vc = m.vic + (size_t) i * m.bucket;
  const int* st = m.stenc + (size_t) i * m.bucket;
  const int deg = trn_deg(m, i);
  const int nb_neigh = m.vdeg[i];
  double q_min = 1.7976931348623157e308;
  for (int a = lane; a < deg; a += G) {
    const int e = st[a];
    if constexpr (JS) asm volatile("prefetch.global.L1 [%0];" ::"l"(m.tri + e));
    q_min = trn_dmin(q_min, m.qual[e]);
  }
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) q_min = trn_dmin(q_min, __shfl_xor_sync(gmask, q_min, o, G));
  const double2 pini = m.pts[i];
  const double4 tini = m.ten[i];
  const TenT<F32> tinf = ten_load<F32>(m, i);
  using R = typename std::conditional<F32, float, double>::type;
  R sx = 0, sy = 0;
  LogSum<F32> lsum;
  for (int b = 0; b < nb_neigh; b += G) {
    const int k = b + lane;
    R tx = 0, ty = 0;
    LogT<F32> l{};
    if (k < nb_neigh) {
      const int nb = vc[k];
      const double2 pb = m.pts[nb];
      if constexpr (F32) {
        const float il = __frcp_rn(trnf_dist2(pini, pb, tenf_of(tinf), tenf_of(ten_load<F32>(m, nb))));
        tx = (float) (pb.x - pini.x) * il;
        ty = (float) (pb.y - pini.y) * il;
      } else {
        const double len = length_x<F32>(pini, pb, tini, m.ten[nb]);
        tx = pini.x + ((pb.x - pini.x) / len);
        ty = pini.y + ((pb.y - pini.y) / len);
      }
      l = log_load<F32>(m, nb);
    }
    const int cnt = min(G, nb_neigh - b);
    for (int j = 0; j < cnt; ++j) {
      sx += grp_shfl(gmask, tx, j, G);
      sy += grp_shfl(gmask, ty, j, G);
      lsum.add(grp_shfl(gmask, l, j, G));
    }
  }
  double ox, oy;
  if constexpr (F32) {
    const float inv = __frcp_rn((float) nb_neigh);
    ox = pini.x + (double) (sx * inv);
    oy = pini.y + (double) (sy * inv);
  } else {
    ox = sx / nb_neigh;
    oy = sy / nb_neigh;
  }
  double tn[3];
  LogT<F32> lnew;
  if constexpr (!F32) {
    finish_pair<G>(lsum.lm, nb_neigh, tn, lane, gmask);
    lnew = log_pair<G>(tn[0], tn[1], tn[2], lane, gmask);
  } else {
    lsum.finish(nb_neigh, tn);
    lnew = log_of<F32>(tn[0], tn[1], tn[2]);
  }
  const double4 tnew = make_double4(tn[0], tn[1], tn[2], 0.0);
  /* qualities and element metrics kept per lane (a stencil of 6 elements
   * fits: 2 a lane with 4 lanes, 3 with 2); later ones are recomputed */
  double qv[KQ];
  /* the element metrics of this lane's first KQ elements: they do not depend
   * on where the vertex sits, so the tries below only redo the geometry */
  JmT<F32> jv[JS ? 1 : KQ];
#pragma unroll
  for (int j = 0; j < KQ; ++j) {
    const int a = lane + j * G;
    if (a < deg) {
      const int4 n = m.tri[st[a]];
      const JmT<F32> q = qmetric_x((n.x == i) ? lnew : log_load<F32>(m, n.x),
                                   (n.y == i) ? lnew : log_load<F32>(m, n.y),
                                   (n.z == i) ? lnew : log_load<F32>(m, n.z));
      if constexpr (JS) js[(size_t) j * blockDim.x] = q;
      else jv[j] = q;
    }
  }
  if constexpr (SW) {
    unsigned okm = 0x1fu;   /* bit w: every element of this lane passes try w */
    int j = 0;
    for (int a = lane; a < deg; a += G, ++j) {
      if (j < KQ) {
        const int4 n = m.tri[st[a]];
        const double2 b0 = (n.x == i) ? pini : m.pts[n.x];
        const double2 b1 = (n.y == i) ? pini : m.pts[n.y];
        const double2 b2 = (n.z == i) ? pini : m.pts[n.z];
        JmT<F32> jm;
        if constexpr (JS) jm = js[(size_t) j * blockDim.x];
        else jm = reg_pick(jv, j);
        double weight = 1;
#pragma unroll
        for (int w = 0; w < 5; ++w) {
          double2 pw;
          pw.x = (1 - weight) * pini.x + weight * ox;
          pw.y = (1 - weight) * pini.y + weight * oy;
          const double2 p0 = (n.x == i) ? pw : b0;
          const double2 p1 = (n.y == i) ? pw : b1;
          const double2 p2 = (n.z == i) ? pw : b2;
          const bool ccw = trn_ccw(p0, p1, p2);
          const double q = qgeom_x(p0, p1, p2, jm);
          qs[(size_t) (w * KQ + j) * blockDim.x] = q;
          if (!(ccw && q > q_min)) okm &= ~(1u << w);
          weight *= 0.5;
        }
      } else {
        double weight = 1;
        for (int w = 0; w < 5; ++w) {
          double2 pw;
          pw.x = (1 - weight) * pini.x + weight * ox;
          pw.y = (1 - weight) * pini.y + weight * oy;
          double q = 0;
          if (!(elem_quality_at<F32>(m, i, m.tri[st[a]], pw, lnew, &q) && q > q_min)) okm &= ~(1u << w);
          weight *= 0.5;
        }
      }
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) okm &= __shfl_xor_sync(gmask, okm, o, G);
    if (!okm) return 0;
    const int wsel = __ffs(okm) - 1;
    double weight = 1;
    for (int w = 0; w < wsel; ++w) weight *= 0.5;
    double2 pa;
    pa.x = (1 - weight) * pini.x + weight * ox;
    pa.y = (1 - weight) * pini.y + weight * oy;
    j = 0;
    for (int a = lane; a < deg; a += G, ++j) {
      double q = 0;
      if (j < KQ) q = qs[(size_t) (wsel * KQ + j) * blockDim.x];
      else elem_quality_at<F32>(m, i, m.tri[st[a]], pa, lnew, &q);
      m.qual[st[a]] = q;
    }
    if (lane == 0) {
      m.pts[i] = pa;
      ten_store<F32>(m, i, tnew);
      log_store<F32>(m, i, lnew);
    }
    return 1;
  }
  bool valid;
  int retry = 0;
  double weight = 1;
  double2 pa;
  do {
    pa.x = (1 - weight) * pini.x + weight * ox;
    pa.y = (1 - weight) * pini.y + weight * oy;
    bool ok = true;
    int j = 0;
    for (int a = lane; ok && a < deg; a += G, ++j) {
      double q = 0;
      if (j < KQ) {
        const int4 n = m.tri[st[a]];
        const double2 p0 = (n.x == i) ? pa : m.pts[n.x];
        const double2 p1 = (n.y == i) ? pa : m.pts[n.y];
        const double2 p2 = (n.z == i) ? pa : m.pts[n.z];
        ok = trn_ccw(p0, p1, p2);
        if (ok) {
          if constexpr (JS) q = qgeom_x(p0, p1, p2, js[(size_t) j * blockDim.x]);
          else q = qgeom_x(p0, p1, p2, reg_pick(jv, j));
          ok = q > q_min;
        }
        reg_put(qv, j, q);
      } else {
        ok = elem_quality_at<F32>(m, i, m.tri[st[a]], pa, lnew, &q) && (q > q_min);
      }
    }
    valid = __all_sync(gmask, ok);
    weight *= 0.5;
  } while (!valid && ++retry < 5);
  if (valid) {
    int j = 0;
    for (int a = lane; a < deg; a += G, ++j) {
      double q = 0;
      if (j < KQ) q = reg_pick(qv, j);
      else elem_quality_at<F32>(m, i, m.tri[st[a]], pa, lnew, &q);
      m.qual[st[a]] = q;
    }
    if (lane == 0) {
      m.pts[i] = pa;
      ten_store<F32>(m, i, tnew);
      log_store<F32>(m, i, lnew);
    }
  }
  return valid ? 1 : 0;
}

template <bool F32, int G, int MinB, int V>
__global__ void __launch_bounds__(256, MinB) k_smooth_move_grp(DMesh m, const int* __restrict__ list,
                                                                       int n, const int* off, int c,
                                                                       int* counters, ByteCount bc) {
  extern __shared__ __align__(16) unsigned char smooth_smem[];
  if (trn_failed(m)) return;
  if (off) {
    list += off[c];
    n = off[c + 1] - off[c];
  }
  const int lane = threadIdx.x % G;
  const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) - lane));
  const long long g0 = ((long long) blockIdx.x * blockDim.x + threadIdx.x) / G;
  const long long gs = ((long long) gridDim.x * blockDim.x) / G;
  int tasks = 0, commit = 0;
  unsigned long long bytes = 0;
  for (long long q = g0; q < n; q += gs) {
    const int v = list[q];
    if (v < 0 || v >= m.capa_node) {
      if (lane == 0) trn_set_error(m.err, TRN_DERR_REPLAY);
      continue;
    }
    const bool moved = m.activ[v] && m.vdeg[v] != 0;
    if (bc.bytes && lane == 0) bytes += smooth_bytes<F32>(m, v, moved, bc.seen);
    if (!moved) continue;
    tasks++;
    commit += move_laplacian_grp<F32, G, V>(m, v, lane, gmask, smooth_smem);
  }
  /* the group's tallies sit on its first lane (0 on the others) */
  trn_warp_add(counters, tasks * (lane == 0));
  trn_warp_add(counters + 1, commit * (lane == 0));
  if (lane == 0 && bytes) atomicAdd(bc.bytes, bytes);
}

void smooth_pre(const DMesh& m, int nb_nodes, cudaStream_t s) {
  k_smooth_pre<<<grid_for(nb_nodes), TRN_THREADS, 0, s>>>(m, nb_nodes);
  note_launch();
  check_launch("smooth_pre");
}

static void smooth_launch(const DMesh& m, const int* list, int n, const int* off, int c, int hint,
                          int* counters, bool fp32, cudaStream_t s) {
  /* per moved vertex: list id, flag, counts, own point/tensor read+write,
   * stencil and adjacency rows, its elements and their cached qualities
   * (read+write); neighbours' points/tensors once each (at most 6 per vertex,
   * at most every vertex) */
  const double own = 4 + 1 + 8 + 2 * (kPt + kTen) + kAvgDeg * (2 * kIdx + kTri + 2 * kQ);
  const double nbr = (double) std::min<long long>((long long) m.capa_node, 6LL * n) * (kPt + kTen);
  ByteCount bc;
  ProfScope ps("smooth_move", s, n * own + nbr, &bc);
  const int t = tune().smooth_threads;
  const int lanes = tune().smooth_lanes;
  const int g = grid_for((long long) hint * lanes, t);
  const int regs = tune().smooth_regs;
  if (lanes == 8 || lanes == 4 || lanes == 2) {
    /* smooth_regs 3: the 64-register cap with the element metrics in shared
     * memory (KQ = 2 slots a thread for 4 or 8 lanes, 3 for 2); 4, 5, 6: all
     * five tries in one sweep, registers capped at 64, 80, 128, with 5 x KQ
     * qualities a thread in shared memory; 7, 8: the sweep with the element
     * metrics in shared memory too, capped at 128, 80 */
    const int kq = lanes >= 4 ? 2 : 3;
    const size_t js_smem = (size_t) kq * t * (fp32 ? sizeof(float4) : sizeof(double4));
    const size_t sw_smem = (size_t) 5 * kq * t * sizeof(double);
#define TRN_GRP(F, G, B, V)                                                                   \
  do {                                                                                        \
    auto* kern = k_smooth_move_grp<F, G, B, V>;                                               \
    const size_t sm = V == 1 ? js_smem : V == 2 ? sw_smem : V == 3 ? js_smem + sw_smem : 0;   \
    if (sm > (48u << 10))                                                                     \
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sm);      \
    kern<<<grid_resident(reinterpret_cast<const void*>(kern), t, g, sm), t, sm, s>>>(m, list, n, off, c, \
                                                                                     counters, bc); \
  } while (0)
#define TRN_GRP_B(F, G)                                                                       \
  do {                                                                                        \
    if (regs == 0) TRN_GRP(F, G, 2, 0);                                                       \
    else if (regs == 1) TRN_GRP(F, G, 3, 0);                                                  \
    else if (regs == 2) TRN_GRP(F, G, 4, 0);                                                  \
    else if (regs == 3) TRN_GRP(F, G, 4, 1);                                                  \
    else if (regs == 4) TRN_GRP(F, G, 4, 2);                                                  \
    else if (regs == 5) TRN_GRP(F, G, 3, 2);                                                  \
    else if (regs == 6) TRN_GRP(F, G, 2, 2);                                                  \
    else if (regs == 7) TRN_GRP(F, G, 2, 3);                                                  \
    else TRN_GRP(F, G, 3, 3);                                                                 \
  } while (0)
    if (lanes == 8) {
      if (fp32) TRN_GRP_B(true, 8);
      else TRN_GRP_B(false, 8);
    } else if (lanes == 4) {
      if (fp32) TRN_GRP_B(true, 4);
      else TRN_GRP_B(false, 4);
    } else {
      if (fp32) TRN_GRP_B(true, 2);
      else TRN_GRP_B(false, 2);
    }
#undef TRN_GRP_B
#undef TRN_GRP
  } else {
    /* element-metric slots a thread: what 40 KB of shared memory a block
     * holds, at most 8 (FP64) or 12 (FP32) */
    const int slot = fp32 ? (int) sizeof(float4) : (int) sizeof(double4);
    const int kj = std::min(fp32 ? 12 : 8, (40 << 10) / (t * slot));
    const size_t smem = (size_t) kj * t * slot;
#define TRN_ONE(F, B)                                                                           \
  do {                                                                                          \
    auto* kern = k_smooth_move<F, B>;                                                           \
    kern<<<grid_resident(reinterpret_cast<const void*>(kern), t, g, smem), t, smem, s>>>(m, list, n, off, \
                                                                                        c, counters, kj, bc); \
  } while (0)
#define TRN_ONE_B(F) \
  do { if (regs == 0) TRN_ONE(F, 2); else if (regs == 1) TRN_ONE(F, 3); else TRN_ONE(F, 4); } while (0)
    if (fp32) TRN_ONE_B(true);
    else TRN_ONE_B(false);
#undef TRN_ONE_B
#undef TRN_ONE
  }
  note_launch();
  check_launch("smooth_move");
}

void smooth_color(const DMesh& m, const int* list, int n, int* counters, bool fp32, cudaStream_t s) {
  if (n <= 0) return;
  smooth_launch(m, list, n, nullptr, 0, n, counters, fp32, s);
}

void smooth_class(const DMesh& m, const int* parts, const int* part_off, int c, int hint, int* counters,
                  bool fp32, cudaStream_t s) {
  smooth_launch(m, parts, hint, part_off, c, hint, counters, fp32, s);
}

}  // namespace trn
