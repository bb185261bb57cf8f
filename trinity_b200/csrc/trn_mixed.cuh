/*
 * trn_mixed.cuh — the mixed-precision form of the metric arithmetic.
 *
 * Same formulas as trn_numeric.cuh (trinity's numeric.cpp), evaluated in
 * FP32: the log-Euclidean tensor mean and its per-vertex logarithm cache,
 * metric edge lengths, the Steiner weight and the element quality. What stays
 * FP64: vertex coordinates and every coordinate difference (orientation and
 * signed areas are computed and tested in FP64, then converted), the stored
 * tensors, the Hessian recovery, and all topology decisions' inputs other than
 * the metric values. The log cache holds a float4 per vertex in the same
 * buffer as the FP64 form's double4.
 *
 * Divisions become reciprocal multiplications here (FP32 results within a
 * few ulp of the divided forms; the FP64 form keeps the reference's
 * divisions for its bit-exactness).
 *
 * Templates at the end (LogT<F32>, log_of<F32>, quality_x, length_x, ...)
 * let one kernel source serve both forms; the FP64 instantiation calls the
 * bit-exact functions unchanged.
 */
#ifndef TRN_MIXED_CUH
#define TRN_MIXED_CUH

#include <type_traits>

#include "trn_common.cuh"
#include "trn_numeric.cuh"

__device__ __forceinline__ float trnf_min(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float trnf_max(float a, float b) { return (a < b) ? b : a; }

__device__ __forceinline__ bool trnf_isnormal(float x) {
  unsigned e = (__float_as_uint(x) >> 23) & 0xff;
  return e != 0 && e != 0xff;
}

/* numeric::eigenDecompose in FP32. The discriminant is taken as
 * ((m0-m3)/2)^2 + m1 m2 (clamped at 0) instead of trace^2/4 - det: the same
 * value without the cancellation that makes it negative for near-isotropic
 * tensors in single precision (the reference uses this form for its
 * eigenvectors, numeric.cpp:69-71). */
__device__ __forceinline__ void trnf_eigen(const float* mat, float* val, float* vec) {
  if (mat[1] * mat[2] < 1.e-9f) {
    val[0] = mat[3];
    val[1] = mat[0];
    vec[0] = 0.f; vec[2] = 1.f;
    vec[1] = 1.f; vec[3] = 0.f;
    return;
  }
  const float term = (mat[0] + mat[3]) * 0.5f;
  const float dm = mat[0] - mat[3];
  const float root = sqrtf(trnf_max(0.25f * (dm * dm) + mat[1] * mat[2], 0.f));
  val[0] = term - root;
  val[1] = term + root;
  if (!trnf_isnormal(val[0]) || !trnf_isnormal(val[1])) val[0] = val[1];
  if (dm >= 0.f) {
    vec[0] = 0.5f * dm - root;
    vec[1] = mat[1];
    vec[2] = mat[2];
    vec[3] = -0.5f * dm + root;
  } else {
    vec[0] = mat[2];
    vec[1] = 0.5f * dm + root;
    vec[2] = -0.5f * dm - root;
    vec[3] = mat[1];
  }
  /* the reference divides by the norms; single precision multiplies by
   * reciprocal square roots (within a few ulp) */
  const float r0 = rsqrtf(vec[0] * vec[0] + vec[1] * vec[1]);
  const float r1 = rsqrtf(vec[2] * vec[2] + vec[3] * vec[3]);
  vec[0] *= r0;
  vec[2] *= r1;
  vec[1] *= r0;
  vec[3] *= r1;
}

/* P log(D) P^T of one tensor, FP32 */
__device__ __forceinline__ float4 trnf_log_tensor(float t0, float t1, float t2) {
  float copy[4] = {t0, t1, t1, t2}, val[2], vec[4];
  trnf_eigen(copy, val, vec);
  val[0] = logf(val[0]);
  val[1] = logf(val[1]);
  float c0 = val[0] * vec[0], c1 = val[0] * vec[2], c2 = val[1] * vec[1], c3 = val[1] * vec[3];
  return make_float4(vec[0] * c0 + vec[1] * c2, vec[0] * c1 + vec[1] * c3,
                     vec[2] * c0 + vec[3] * c2, vec[2] * c1 + vec[3] * c3);
}

/* exp of the mean logarithm; *det receives e^l0 e^l1 = det of the result
 * (exact in exact arithmetic, free of the cancellation of m11 m22 - m12^2) */
__device__ __forceinline__ void trnf_interp_finish(float* lm, int nb, float* res, float* det = nullptr) {
  float val[2], vec[4];
  const float inv = nb == 3 ? 0.333333343f : __frcp_rn((float) nb);
  for (int i = 0; i < 4; ++i) lm[i] *= inv;
  trnf_eigen(lm, val, vec);
  val[0] = expf(val[0]);
  val[1] = expf(val[1]);
  if (det) *det = val[0] * val[1];
  float c0 = val[0] * vec[0], c1 = val[0] * vec[2], c2 = val[1] * vec[1], c3 = val[1] * vec[3];
  res[0] = vec[0] * c0 + vec[1] * c2;
  res[1] = vec[0] * c1 + vec[1] * c3;
  res[2] = vec[2] * c1 + vec[3] * c3;
}

/* quality from cached FP32 logarithms; coordinate differences and the area
 * in FP64. In two halves like trn_quality_l: the tensor mean and the square
 * root of its determinant (j0, j1, j2, sqrt det), then the geometry. */
__device__ __forceinline__ float4 trnf_quality_metric(float4 la, float4 lb, float4 lc) {
  float lm[4] = {la.x + lb.x + lc.x, la.y + lb.y + lc.y, la.z + lb.z + lc.z, la.w + lb.w + lc.w};
  float j[3], det;
  trnf_interp_finish(lm, 3, j, &det);
  return make_float4(j[0], j[1], j[2], sqrtf(det));
}

__device__ __forceinline__ double trnf_quality_geom(double2 pa, double2 pb, double2 pc, float4 jm) {
  const float j[3] = {jm.x, jm.y, jm.z};
  const float e[6] = {(float) (pb.x - pa.x), (float) (pb.y - pa.y), (float) (pc.x - pb.x),
                      (float) (pc.y - pb.y), (float) (pa.x - pc.x), (float) (pa.y - pc.y)};
  float perim = 0.f;
  for (int k = 0; k < 3; ++k) {
    const float u = e[2 * k], v = e[2 * k + 1];
    perim += sqrtf(u * (j[0] * u + j[1] * v) + v * (j[1] * u + j[2] * v));
  }
  const double area = 0.5 * fabs((pb.x - pa.x) * (pc.y - pa.y) - (pc.x - pa.x) * (pb.y - pa.y));
  const float ip = __frcp_rn(perim);
  const float mean = trnf_min(perim * 0.333333343f, 3.f * ip);
  const float mm = mean * (2.f - mean);
  const float norm = 20.78460969082653f * (mm * mm * mm);  /* 12 sqrt(3) */
  return (double) ((float) area * norm * jm.w * (ip * ip));
}

__device__ __forceinline__ double trnf_quality_l(double2 pa, double2 pb, double2 pc, float4 la,
                                                 float4 lb, float4 lc) {
  return trnf_quality_geom(pa, pb, pc, trnf_quality_metric(la, lb, lc));
}

__device__ __forceinline__ float4 tenf_of(double4 t) {
  return make_float4((float) t.x, (float) t.y, (float) t.z, 0.f);
}
__device__ __forceinline__ float4 tenf_of(float4 t) { return t; }

/* metric edge length (numeric.cpp:469-497) in FP32, in the same two halves */
__device__ __forceinline__ void trnf_dist2_ends(double2 pa, double2 pb, float4 ta, float4 tb,
                                                float* l0, float* l1) {
  const float w0 = (float) (pb.x - pa.x), w1 = (float) (pb.y - pa.y);
  const float a0 = ta.x, a1 = ta.y, a2 = ta.z;
  const float b0 = tb.x, b1 = tb.y, b2 = tb.z;
  *l0 = sqrtf(w0 * (a0 * w0 + a1 * w1) + w1 * (a1 * w0 + a2 * w1));
  *l1 = sqrtf(w0 * (b0 * w0 + b1 * w1) + w1 * (b1 * w0 + b2 * w1));
}

__device__ __forceinline__ float trnf_dist2_finish(float l0, float l1) {
  if (fabsf(l0 - l1) < 1.e-9f) return l0;
  const float lmin = trnf_min(l0, l1), lmax = trnf_max(l0, l1);
  const float ratio = lmax * __frcp_rn(lmin);
  return lmax * (ratio - 1.f) * __frcp_rn(ratio * logf(ratio));
}

__device__ __forceinline__ float trnf_dist2(double2 pa, double2 pb, float4 ta, float4 tb) {
  float l0, l1;
  trnf_dist2_ends(pa, pb, ta, tb, &l0, &l1);
  return trnf_dist2_finish(l0, l1);
}

__device__ __forceinline__ float trnf_dist1(double2 pa, double2 pb, float4 t) {
  const float u0 = (float) (pb.x - pa.x), u1 = (float) (pb.y - pa.y);
  return sqrtf(u0 * (t.x * u0 + t.y * u1) + u1 * (t.y * u0 + t.z * u1));
}

/* ---------------- dispatch between the two forms ---------------- */
template <bool F32>
using LogT = typename std::conditional<F32, float4, double4>::type;

template <bool F32>
__device__ __forceinline__ LogT<F32> log_load(const DMesh& m, int v) {
  if constexpr (F32) return reinterpret_cast<const float4*>(m.lten)[v];
  else return m.lten[v];
}

template <bool F32>
__device__ __forceinline__ void log_store(const DMesh& m, int v, LogT<F32> l) {
  if constexpr (F32) reinterpret_cast<float4*>(m.lten)[v] = l;
  else m.lten[v] = l;
}

template <bool F32>
__device__ __forceinline__ LogT<F32> log_of(double t0, double t1, double t2) {
  if constexpr (F32) return trnf_log_tensor((float) t0, (float) t1, (float) t2);
  else return trn_log_tensor(t0, t1, t2);
}

__device__ __forceinline__ double quality_x(double2 a, double2 b, double2 c, double4 la, double4 lb,
                                           double4 lc) {
  return trn_quality_l(a, b, c, la, lb, lc);
}
__device__ __forceinline__ double quality_x(double2 a, double2 b, double2 c, float4 la, float4 lb,
                                           float4 lc) {
  return trnf_quality_l(a, b, c, la, lb, lc);
}

/* the two halves of quality_x (a position-independent element metric, then
 * the geometry), same bits as quality_x */
__device__ __forceinline__ double4 qmetric_x(double4 la, double4 lb, double4 lc) {
  return trn_quality_metric(la, lb, lc);
}
__device__ __forceinline__ float4 qmetric_x(float4 la, float4 lb, float4 lc) {
  return trnf_quality_metric(la, lb, lc);
}
__device__ __forceinline__ double qgeom_x(double2 a, double2 b, double2 c, double4 jm) {
  return trn_quality_geom(a, b, c, jm);
}
__device__ __forceinline__ double qgeom_x(double2 a, double2 b, double2 c, float4 jm) {
  return trnf_quality_geom(a, b, c, jm);
}

/* quality of element (v0, v1, v2) from the cached logarithms */
template <bool F32>
__device__ __forceinline__ double quality_of(const DMesh& m, int4 t) {
  return quality_x(m.pts[t.x], m.pts[t.y], m.pts[t.z], log_load<F32>(m, t.x), log_load<F32>(m, t.y),
                   log_load<F32>(m, t.z));
}

/* the stored tensors as each form reads them: FP64, or the FP32 copy */
template <bool F32>
using TenT = typename std::conditional<F32, float4, double4>::type;

template <bool F32>
__device__ __forceinline__ TenT<F32> ten_load(const DMesh& m, int v) {
  if constexpr (F32) return m.tenf[v];
  else return m.ten[v];
}

/* a new stored tensor (and its FP32 copy in the mixed form) */
template <bool F32>
__device__ __forceinline__ void ten_store(const DMesh& m, int v, double4 t) {
  m.ten[v] = t;
  if constexpr (F32) m.tenf[v] = tenf_of(t);
}

template <bool F32, class T>
__device__ __forceinline__ double length_x(double2 pa, double2 pb, T ta, T tb) {
  if constexpr (F32) return (double) trnf_dist2(pa, pb, tenf_of(ta), tenf_of(tb));
  else return trn_dist2(pa, pb, ta, tb);
}

/* Comparisons of a metric edge length with a threshold, with the answer of
 * comparing length_x itself. That length interpolates the edge's lengths
 * under its two endpoint tensors geometrically, so it lies between them: up
 * to a few units in the last place as computed, far inside the margins below
 * (1e-12 relative in FP64, 1e-5 in FP32). When the threshold lies outside
 * that range, with the margin, the answer is known without the logarithm. */
template <bool F32, class T>
__device__ __forceinline__ bool length_gt(double2 pa, double2 pb, T ta, T tb, double thresh) {
  if constexpr (F32) {
    float l0, l1;
    trnf_dist2_ends(pa, pb, tenf_of(ta), tenf_of(tb), &l0, &l1);
    const float t = (float) thresh;
    if (l0 == l0 && l1 == l1) {
      if (trnf_max(l0, l1) < t * (1.f - 1.e-5f)) return false;
      if (trnf_min(l0, l1) > t * (1.f + 1.e-5f)) return true;
    }
    return (double) trnf_dist2_finish(l0, l1) > thresh;
  } else {
    double l0, l1;
    trn_dist2_ends(pa, pb, ta, tb, &l0, &l1);
    if (l0 == l0 && l1 == l1) {
      if (trn_dmax(l0, l1) < thresh * (1 - 1.e-12)) return false;
      if (trn_dmin(l0, l1) > thresh * (1 + 1.e-12)) return true;
    }
    return trn_dist2_finish(l0, l1) > thresh;
  }
}

/* length_x < thresh; *len receives length_x whenever the answer is true */
template <bool F32, class T>
__device__ __forceinline__ bool length_lt(double2 pa, double2 pb, T ta, T tb, double thresh,
                                          double* len) {
  if constexpr (F32) {
    float l0, l1;
    trnf_dist2_ends(pa, pb, tenf_of(ta), tenf_of(tb), &l0, &l1);
    if (l0 == l0 && l1 == l1 && trnf_min(l0, l1) > (float) thresh * (1.f + 1.e-5f)) return false;
    *len = (double) trnf_dist2_finish(l0, l1);
  } else {
    double l0, l1;
    trn_dist2_ends(pa, pb, ta, tb, &l0, &l1);
    if (l0 == l0 && l1 == l1 && trn_dmin(l0, l1) > thresh * (1 + 1.e-12)) return false;
    *len = trn_dist2_finish(l0, l1);
  }
  return *len < thresh;
}

/* mean of a run of cached logarithms, then exponentiated: the new tensor */
template <bool F32>
struct LogSum {
  using R = typename std::conditional<F32, float, double>::type;
  R lm[4] = {0, 0, 0, 0};
  __device__ __forceinline__ void add(LogT<F32> l) {
    lm[0] += l.x;
    lm[1] += l.y;
    lm[2] += l.z;
    lm[3] += l.w;
  }
  __device__ __forceinline__ void finish(int nb, double* res) {
    if constexpr (F32) {
      float r[3];
      trnf_interp_finish(lm, nb, r);
      res[0] = r[0];
      res[1] = r[1];
      res[2] = r[2];
    } else {
      trn_interp_finish(lm, nb, res);
    }
  }
};

/* numeric::computeSteinerPoint in either form (point in FP64) */
template <bool F32, class T>
__device__ __forceinline__ void steiner_x(double2 pa, double2 pb, T ta, T tb,
                                          LogT<F32> la, LogT<F32> lb, double2* rp, double* rt) {
  if constexpr (F32) {
    const float l0 = trnf_dist1(pa, pb, tenf_of(ta)), l1 = trnf_dist1(pa, pb, tenf_of(tb));
    const float w = (fabsf(l0 - l1) < 1.e-9f) ? 0.5f : (sqrtf(l0 * l1) - l1) / (l0 - l1);
    const double wd = (double) w;
    rp->x = (1 - wd) * pa.x + (wd * pb.x);
    rp->y = (1 - wd) * pa.y + (wd * pb.y);
    LogSum<true> s;
    s.add(la);
    s.add(lb);
    s.finish(2, rt);
  } else {
    trn_steiner(pa, pb, ta, tb, la, lb, rp, rt);
  }
}

#endif
