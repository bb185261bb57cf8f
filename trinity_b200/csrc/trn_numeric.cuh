/*
 * trn_numeric.cuh — FP64 metric geometry on the device.
 *
 * Each function evaluates the same expressions, in the same operand order, as
 * trinity's numeric.cpp; compiled with --fmad=false and with the project's
 * log/exp/pow (trn_libm.h), results are bit-identical to the reference built
 * with -ffp-contract=off and the same log/exp/pow.
 */
#ifndef TRN_NUMERIC_CUH
#define TRN_NUMERIC_CUH

#include "trn_libm.h"

#define TRN_EPS 1.e-9
#define TRN_L_MIN 0.707106781186547   /* header.h:66 */
#define TRN_L_MAX 1.414213562373095   /* header.h:67 */
#define TRN_Q_MIN 0.9                 /* header.h:69 */

__device__ __forceinline__ double trn_dmin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double trn_dmax(double a, double b) { return (a < b) ? b : a; }

__device__ __forceinline__ bool trn_isnormal(double x) {
  unsigned long long e = ((unsigned long long) __double_as_longlong(x) >> 52) & 0x7ff;
  return e != 0 && e != 0x7ff;
}

/* numeric::eigenDecompose, numeric.cpp:25-95; vec = (v1x, v1y, v2x, v2y) */
__device__ __forceinline__ void trn_eigen(const double* mat, double* val, double* vec) {
  if (mat[1] * mat[2] < TRN_EPS) {
    val[0] = mat[3];
    val[1] = mat[0];
    vec[0] = 0; vec[2] = 1;
    vec[1] = 1; vec[3] = 0;
    return;
  }
  double trace = mat[0] + mat[3];
  double det = mat[0] * mat[3] - mat[1] * mat[2];
  double term = trace * 0.5;
  double sqrt_delta = sqrt(term * term - det);
  val[0] = term - sqrt_delta;
  val[1] = term + sqrt_delta;
  if (!trn_isnormal(val[0]) || !trn_isnormal(val[1])) val[0] = val[1];
  double dm = mat[0] - mat[3];
  term = sqrt(trn_dmax(0.25 * trn_pow(dm, 2) + mat[1] * mat[2], 0.));
  if (dm >= 0) {
    vec[0] = +0.5 * dm - term;
    vec[1] = mat[1];
    vec[2] = mat[2];
    vec[3] = -0.5 * dm + term;
  } else {
    vec[0] = mat[2];
    vec[1] = +0.5 * dm + term;
    vec[2] = -0.5 * dm - term;
    vec[3] = mat[1];
  }
  double n0 = sqrt(vec[0] * vec[0] + vec[1] * vec[1]);
  double n1 = sqrt(vec[2] * vec[2] + vec[3] * vec[3]);
  vec[0] /= n0;
  vec[2] /= n1;
  vec[1] /= n0;
  vec[3] /= n1;
}

/* P diag(val) P^T from an eigen pair (vec = the columns of P), the last
 * step of numeric::interpolateTensor's logarithm and exponentiation
 * (numeric.cpp:131-154, 196-216), all four entries */
__device__ __forceinline__ void trn_eigen_compose(const double* val, const double* vec, double* cache) {
  double copy[4];
  copy[0] = val[0] * vec[0];
  copy[1] = val[0] * vec[2];
  copy[2] = val[1] * vec[1];
  copy[3] = val[1] * vec[3];
  cache[0] = vec[0] * copy[0] + vec[1] * copy[2];
  cache[1] = vec[0] * copy[1] + vec[1] * copy[3];
  cache[2] = vec[2] * copy[0] + vec[3] * copy[2];
  cache[3] = vec[2] * copy[1] + vec[3] * copy[3];
}

/* the logarithm P log(D) P^T of one tensor as numeric::interpolateTensor
 * forms it (numeric.cpp:115-154), all four entries (not exactly symmetric).
 * It depends on the tensor alone, so a cached copy summed in the same order
 * gives the same bits as recomputing it inside every mean. */
__device__ __forceinline__ double4 trn_log_tensor(double t0, double t1, double t2) {
  double copy[4], cache[4], val[2], vec[4];
  copy[0] = t0;
  copy[1] = t1;
  copy[2] = t1;
  copy[3] = t2;
  trn_eigen(copy, val, vec);
  val[0] = trn_log(val[0]);
  val[1] = trn_log(val[1]);
  trn_eigen_compose(val, vec, cache);
  return make_double4(cache[0], cache[1], cache[2], cache[3]);
}

/* log_mat += a cached tensor logarithm (numeric.cpp:169-171) */
__device__ __forceinline__ void trn_interp_addl(double* log_mat, double4 l) {
  log_mat[0] += l.x;
  log_mat[1] += l.y;
  log_mat[2] += l.z;
  log_mat[3] += l.w;
}

/* one term of the log-Euclidean sum of numeric::interpolateTensor */
__device__ __forceinline__ void trn_interp_add(double* log_mat, double t0, double t1, double t2) {
  trn_interp_addl(log_mat, trn_log_tensor(t0, t1, t2));
}

/* the exponentiation half of numeric::interpolateTensor (numeric.cpp:189-216) */
__device__ __forceinline__ void trn_interp_finish(double* log_mat, int nb, double* res) {
  double cache[4], val[2], vec[4];
  for (int i = 0; i < 4; ++i) log_mat[i] /= nb;
  trn_eigen(log_mat, val, vec);
  val[0] = trn_exp(val[0]);
  val[1] = trn_exp(val[1]);
  trn_eigen_compose(val, vec, cache);
  res[0] = cache[0];
  res[1] = cache[1];
  res[2] = cache[3];
}

/* numeric::computeQuality, numeric.cpp:251-306, in two halves. The first
 * depends only on the three vertex tensors: their log-Euclidean mean
 * (jacob) and the square root of its determinant, returned as
 * (j0, j1, j2, sqrt det). The second takes the three points. A caller that
 * evaluates one element at several positions of a vertex whose tensor does
 * not change (the smoothing back-off) computes the first half once; the
 * operations and their order are those of the whole function, so the bits
 * are the same. */
__device__ __forceinline__ double4 trn_quality_metric(double4 la, double4 lb, double4 lc) {
  double lm[4] = {0, 0, 0, 0};
  double jacob[3];
  trn_interp_addl(lm, la);
  trn_interp_addl(lm, lb);
  trn_interp_addl(lm, lc);
  trn_interp_finish(lm, 3, jacob);
  double det = jacob[0] * jacob[2] - jacob[1] * jacob[1];
  return make_double4(jacob[0], jacob[1], jacob[2], sqrt(det));
}

__device__ __forceinline__ double trn_quality_geom(double2 pa, double2 pb, double2 pc, double4 jm) {
  const double jacob[3] = {jm.x, jm.y, jm.z};
  double coef[6];
  coef[0] = pb.x - pa.x;
  coef[1] = pb.y - pa.y;
  coef[2] = pc.x - pb.x;
  coef[3] = pc.y - pb.y;
  coef[4] = pa.x - pc.x;
  coef[5] = pa.y - pc.y;
  double perim = 0;
  for (int k = 0; k < 3; ++k) {
    int i = k * 2, j = i + 1;
    double vi = jacob[0] * coef[i] + jacob[1] * coef[j];
    double vj = jacob[1] * coef[i] + jacob[2] * coef[j];
    perim += sqrt(coef[i] * vi + coef[j] * vj);
  }
  double c0 = pb.x - pa.x;
  double c1 = pc.x - pa.x;
  double c2 = pb.y - pa.y;
  double c3 = pc.y - pa.y;
  double area = 0.5 * fabs(c0 * c3 - c1 * c2);
  double mean = trn_dmin(perim / 3, 3 / perim);
  double norm = 12 * sqrt(3.0) * trn_pow(mean * (2. - mean), 3);
  return area * norm * jm.w / trn_pow(perim, 2);
}

/* numeric::computeQuality from the vertices' cached tensor logarithms */
__device__ __forceinline__ double trn_quality_l(double2 pa, double2 pb, double2 pc,
                                                double4 la, double4 lb, double4 lc) {
  return trn_quality_geom(pa, pb, pc, trn_quality_metric(la, lb, lc));
}

/* numeric::computeQuality from the tensors themselves */
__device__ __forceinline__ double trn_quality(double2 pa, double2 pb, double2 pc,
                                              double4 ta, double4 tb, double4 tc) {
  return trn_quality_l(pa, pb, pc, trn_log_tensor(ta.x, ta.y, ta.z),
                       trn_log_tensor(tb.x, tb.y, tb.z), trn_log_tensor(tc.x, tc.y, tc.z));
}

/* numeric::approxRiemannDist(a, b, M), numeric.cpp:450-461 */
__device__ __forceinline__ double trn_dist1(double2 pa, double2 pb, double4 t) {
  double u0 = pb.x - pa.x;
  double u1 = pb.y - pa.y;
  double v0 = t.x * u0 + t.y * u1;
  double v1 = t.y * u0 + t.z * u1;
  return sqrt(u0 * v0 + u1 * v1);
}

/* numeric::approxRiemannDist(a, b, Ma, Mb), numeric.cpp:469-497, in two
 * halves: the edge's length under each endpoint tensor, then their
 * geometric interpolation */
__device__ __forceinline__ void trn_dist2_ends(double2 pa, double2 pb, double4 ta, double4 tb,
                                               double* l0, double* l1) {
  double w0 = pb.x - pa.x;
  double w1 = pb.y - pa.y;
  double m0 = ta.x * w0 + ta.y * w1;
  double m1 = ta.y * w0 + ta.z * w1;
  double m2 = tb.x * w0 + tb.y * w1;
  double m3 = tb.y * w0 + tb.z * w1;
  *l0 = sqrt(w0 * m0 + w1 * m1);
  *l1 = sqrt(w0 * m2 + w1 * m3);
}

__device__ __forceinline__ double trn_dist2_finish(double l0, double l1) {
  if (fabs(l0 - l1) < TRN_EPS) return l0;
  double lmin = trn_dmin(l0, l1);
  double lmax = trn_dmax(l0, l1);
  double ratio = lmax / lmin;
  return lmax * (ratio - 1) / (ratio * trn_log(ratio));
}

__device__ __forceinline__ double trn_dist2(double2 pa, double2 pb, double4 ta, double4 tb) {
  double l0, l1;
  trn_dist2_ends(pa, pb, ta, tb, &l0, &l1);
  return trn_dist2_finish(l0, l1);
}

/* numeric::computeSteinerPoint, numeric.cpp:387-445 (la, lb: cached
 * logarithms of ta, tb) */
__device__ __forceinline__ void trn_steiner(double2 pa, double2 pb, double4 ta, double4 tb,
                                            double4 la, double4 lb, double2* rp, double* rt) {
  double coef = 1;
  double l0 = trn_dist1(pa, pb, ta);
  double l1 = trn_dist1(pa, pb, tb);
  double weight = (fabs(l0 - l1) < TRN_EPS
    ? 0.5
    : (sqrt(coef) * sqrt(l0 * l1) - l1) / (coef * l0 - l1));
  rp->x = (1 - weight) * pa.x + (weight * pb.x);
  rp->y = (1 - weight) * pa.y + (weight * pb.y);
  double lm[4] = {0, 0, 0, 0};
  trn_interp_addl(lm, la);
  trn_interp_addl(lm, lb);
  trn_interp_finish(lm, 2, rt);
}

/* Mesh::isCounterclockwise, mesh.cpp:700-713 */
__device__ __forceinline__ bool trn_ccw(double2 a, double2 b, double2 c) {
  double c0 = b.x - a.x;
  double c1 = c.x - a.x;
  double c2 = b.y - a.y;
  double c3 = c.y - a.y;
  return 0.5 * (c0 * c3 - c1 * c2) > TRN_EPS;
}

/* tensor from eigen pairs, metric.cpp:134-148 / 222-236 */
__device__ __forceinline__ double4 trn_recompose(const double* val, const double* vec) {
  double mm0 = val[0] * vec[0];
  double mm1 = val[0] * vec[2];
  double mm2 = val[1] * vec[1];
  double mm3 = val[1] * vec[3];
  double4 r;
  r.x = vec[0] * mm0 + vec[1] * mm2;
  r.y = vec[0] * mm1 + vec[1] * mm3;
  r.z = vec[2] * mm1 + vec[3] * mm3;
  r.w = 0.0;
  return r;
}

#endif
