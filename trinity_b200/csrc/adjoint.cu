/*
 * adjoint.cu — the element-quality functional and its adjoint.
 *
 *   J(x, u) = sum over live elements T of q_T(x, M(u))
 *
 * q_T is numeric::computeQuality (numeric.cpp:251-306): the element at the
 * coordinates x, under the log-Euclidean mean of its vertices' tensors. M(u)
 * is the metric Metrics::run recovers from the nodal solution u
 * (metric.cpp:59-70): P1 gradient and Hessian recovery over the 2-ring
 * element patch (hessian.cpp:24-153), |H| eigen-clamp with the local L^p
 * scale (metric.cpp:100-150), the complexity (153-185) and the global scale
 * with the eigenvalue clamp (188-238). The recovery runs on the mesh's own
 * coordinates; x only moves the elements that the quality sees, so
 * dJ/dx is taken at a fixed nodal metric and dJ/du through the recovery.
 *
 * Every kernel gathers (no atomics), so the adjoint is deterministic:
 *   k_adj_elem        per element: q, dq/d(its 3 points), dq/d(log M_v)
 *   k_adj_vertex      per vertex over its stencil: dJ/dx_v, and the
 *                     logarithm's adjoint at M_v -> dJ/dM_v
 *   k_adj_global      per vertex: adjoint of the global scale and clamp, and
 *                     its share of dJ/d(scale)
 *   k_adj_local       per vertex: complexity term, adjoint of the local L^p
 *                     normalisation -> dJ/dH_v / (patch area)
 *   k_adj_elem_patch  per element: area x sum over the vertices whose patch
 *                     holds the element (the transpose of the patch mean)
 *   k_adj_vertex_hess per vertex: -> dJ/d(recovered gradient) / (patch area)
 *   k_adj_vertex_u    per vertex: -> dJ/du
 *
 * Matrix functions Y = Q f(L) Q^T of a symmetric 2x2 X = Q L Q^T are
 * differentiated with the Daleckii-Krein formula: in the eigenbasis the
 * diagonal of the gradient maps through df/dlambda and the off-diagonal
 * through the divided difference (f(l0) - f(l1)) / (l0 - l1). Where the
 * forward eigen solver takes its diagonal shortcut (numeric.cpp:30-38, the
 * off-diagonal entry ignored) the off-diagonal gradient is zero, as it is in
 * the forward. Symmetric gradients are held as (G00, G01, G11) with
 * dJ = G00 dX00 + 2 G01 dX01 + G11 dX11, so the gradient with respect to the
 * stored tensor (m11, m12, m22) is (G00, 2 G01, G11).
 *
 * The FP64 form evaluates q with the same bits as the adaptation kernels; the
 * FP32 form evaluates q and the whole adjoint in single precision (the
 * coordinates, their differences and the signed areas stay FP64, as in the
 * mixed form); the metric recovery itself is FP64 in both.
 */
#include "trn_internal.h"
#include "trn_mixed.cuh"

#include <algorithm>

namespace trn {

template <bool F32>
using AReal = typename std::conditional<F32, float, double>::type;

__device__ __forceinline__ void eig_x(const double* mat, double* val, double* vec) {
  trn_eigen(mat, val, vec);
}
__device__ __forceinline__ void eig_x(const float* mat, float* val, float* vec) {
  trnf_eigen(mat, val, vec);
}
__device__ __forceinline__ double exp_x(double x) { return trn_exp(x); }
__device__ __forceinline__ float exp_x(float x) { return expf(x); }
__device__ __forceinline__ double expm1_x(double x) { return expm1(x); }
__device__ __forceinline__ float expm1_x(float x) { return expm1f(x); }
__device__ __forceinline__ double log1p_x(double x) { return log1p(x); }
__device__ __forceinline__ float log1p_x(float x) { return log1pf(x); }

/* (e^a - e^b) / (a - b), ea = e^a, eb = e^b */
template <class R>
__device__ __forceinline__ R divdiff_exp(R a, R b, R ea, R eb) {
  const R d = a - b;
  if (d == R(0)) return ea;
  return eb * expm1_x(d) / d;
}

/* (log a - log b) / (a - b), a, b > 0 */
template <class R>
__device__ __forceinline__ R divdiff_log(R a, R b) {
  const R d = a - b;
  if (d == R(0)) return R(1) / a;
  return log1p_x(d / b) / d;
}

/* Adjoint of Y = Q diag(F(lambda)) Q^T at X = Q diag(lambda) Q^T; the columns
 * of Q are (vec0, vec2) and (vec1, vec3) (numeric::eigenDecompose's layout).
 * g: the symmetric gradient with respect to Y on entry, with respect to X on
 * return. jac[k][l] = dF_k/dlambda_l; gam = (F0 - F1)/(lambda0 - lambda1), or
 * 0 where the forward ignored the off-diagonal entry. diag, if set, receives
 * the gradient's diagonal in the eigenbasis (before jac). */
template <class R>
__device__ __forceinline__ void spectral_adjoint(const R* vec, const R jac[2][2], R gam, R* g,
                                                 R* diag = nullptr) {
  const R ax = vec[0], ay = vec[2], bx = vec[1], by = vec[3];
  const R h00 = g[0] * ax * ax + R(2) * g[1] * ax * ay + g[2] * ay * ay;
  const R h11 = g[0] * bx * bx + R(2) * g[1] * bx * by + g[2] * by * by;
  const R h01 = g[0] * ax * bx + g[1] * (ax * by + ay * bx) + g[2] * ay * by;
  if (diag) {
    diag[0] = h00;
    diag[1] = h11;
  }
  const R d0 = jac[0][0] * h00 + jac[1][0] * h11;
  const R d1 = jac[0][1] * h00 + jac[1][1] * h11;
  const R o = gam * h01;
  g[0] = ax * ax * d0 + R(2) * ax * bx * o + bx * bx * d1;
  g[2] = ay * ay * d0 + R(2) * ay * by * o + by * by * d1;
  g[1] = ax * ay * d0 + (ax * by + bx * ay) * o + bx * by * d1;
}

template <bool F32>
struct ElemAdj {
  double q;
  AReal<F32> gp[6];   /* dq/d(pa.x, pa.y, pb.x, pb.y, pc.x, pc.y) */
  AReal<F32> gl[3];   /* dq/d(log M_v), the same for the three vertices */
};

/* numeric::computeQuality and its adjoint, from the vertices' cached tensor
 * logarithms. The value is the adaptation kernels' own (quality_x). */
template <bool F32>
__device__ void quality_adjoint(double2 pa, double2 pb, double2 pc, LogT<F32> la, LogT<F32> lb,
                                LogT<F32> lc, bool want_log, ElemAdj<F32>& o) {
  using R = AReal<F32>;
  o.q = quality_x(pa, pb, pc, la, lb, lc);
  R lm[4] = {R(la.x) + R(lb.x) + R(lc.x), R(la.y) + R(lb.y) + R(lc.y),
             R(la.z) + R(lb.z) + R(lc.z), R(la.w) + R(lb.w) + R(lc.w)};
  for (int i = 0; i < 4; ++i) lm[i] /= R(3);
  R val[2], vec[4];
  eig_x(lm, val, vec);
  const bool shortcut = lm[1] * lm[2] < R(1.e-9);
  const R e0 = exp_x(val[0]), e1 = exp_x(val[1]);
  const R c0 = e0 * vec[0], c1 = e0 * vec[2], c2 = e1 * vec[1], c3 = e1 * vec[3];
  const R j0 = vec[0] * c0 + vec[1] * c2;
  const R j1 = vec[0] * c1 + vec[1] * c3;
  const R j2 = vec[2] * c1 + vec[3] * c3;
  const R sd = sqrt(e0 * e1);
  const R u[3] = {R(pb.x - pa.x), R(pc.x - pb.x), R(pa.x - pc.x)};
  const R v[3] = {R(pb.y - pa.y), R(pc.y - pb.y), R(pa.y - pc.y)};
  R pk[3], perim = 0;
  for (int k = 0; k < 3; ++k) {
    pk[k] = sqrt(u[k] * (j0 * u[k] + j1 * v[k]) + v[k] * (j1 * u[k] + j2 * v[k]));
    perim += pk[k];
  }
  const double cross = (pb.x - pa.x) * (pc.y - pa.y) - (pc.x - pa.x) * (pb.y - pa.y);
  const R area = R(0.5 * fabs(cross));
  const R sg = cross >= 0 ? R(1) : R(-1);
  const R p3 = perim / R(3), ip = R(3) / perim;
  const bool first = !(ip < p3);           /* min(P/3, 3/P) picks P/3 */
  const R mean = first ? p3 : ip;
  const R dmean = first ? R(1) / R(3) : -ip / perim;
  const R mm = mean * (R(2) - mean);
  const R f = mm * mm * mm;
  const R fp = R(3) * mm * mm * (R(2) - R(2) * mean);
  const R K = R(20.784609690826528);       /* 12 sqrt(3) */
  const R ip2 = R(1) / (perim * perim);
  const R dq_dp = area * K * sd * (fp * dmean * ip2 - R(2) * f * ip2 / perim);
  const R dq_da = K * f * sd * ip2;
  const R dq_dsd = area * K * f * ip2;
  R ge[6];
  for (int k = 0; k < 3; ++k) {
    const R s = pk[k] > R(0) ? dq_dp / pk[k] : R(0);
    ge[2 * k] = s * (j0 * u[k] + j1 * v[k]);
    ge[2 * k + 1] = s * (j1 * u[k] + j2 * v[k]);
  }
  const R ha = R(0.5) * sg * dq_da;
  o.gp[0] = -ge[0] + ge[4] + ha * R(pb.y - pc.y);
  o.gp[1] = -ge[1] + ge[5] + ha * R(pc.x - pb.x);
  o.gp[2] = ge[0] - ge[2] + ha * R(pc.y - pa.y);
  o.gp[3] = ge[1] - ge[3] + ha * R(pa.x - pc.x);
  o.gp[4] = ge[2] - ge[4] + ha * R(pa.y - pb.y);
  o.gp[5] = ge[3] - ge[5] + ha * R(pb.x - pa.x);
  if (!want_log) return;
  /* gradient with respect to the mean tensor: sqrt(det) and the perimeter */
  const R hs = sd > R(0) ? dq_dsd / (R(2) * sd) : R(0);
  R g[3] = {hs * j2, -hs * j1, hs * j0};
  for (int k = 0; k < 3; ++k) {
    if (!(pk[k] > R(0))) continue;
    const R w = dq_dp / (R(2) * pk[k]);
    g[0] += w * u[k] * u[k];
    g[1] += w * u[k] * v[k];
    g[2] += w * v[k] * v[k];
  }
  /* through the exponential of the mean logarithm */
  const R jac[2][2] = {{e0, R(0)}, {R(0), e1}};
  const R gam = shortcut ? R(0) : divdiff_exp(val[0], val[1], e0, e1);
  spectral_adjoint(vec, jac, gam, g);
  o.gl[0] = g[0] / R(3);
  o.gl[1] = g[1] / R(3);
  o.gl[2] = g[2] / R(3);
}

template <bool F32>
__global__ void k_adj_elem(DMesh f, int nb_elems, const double2* __restrict__ xy,
                           double* __restrict__ q, AReal<F32>* __restrict__ egp,
                           AReal<F32>* __restrict__ egl) {
  using R = AReal<F32>;
  if (trn_failed(f)) return;
  for (int t = trn_tid(); t < nb_elems; t += trn_grid_stride()) {
    const int4 n = f.tri[t];
    if (n.x < 0) {
      q[t] = 0.0;
      for (int k = 0; k < 6; ++k) egp[6 * (size_t) t + k] = R(0);
      if (egl)
        for (int k = 0; k < 3; ++k) egl[3 * (size_t) t + k] = R(0);
      continue;
    }
    ElemAdj<F32> o;
    quality_adjoint<F32>(xy[n.x], xy[n.y], xy[n.z], log_load<F32>(f, n.x), log_load<F32>(f, n.y),
                         log_load<F32>(f, n.z), egl != nullptr, o);
    q[t] = o.q;
    for (int k = 0; k < 6; ++k) egp[6 * (size_t) t + k] = o.gp[k];
    if (egl)
      for (int k = 0; k < 3; ++k) egl[3 * (size_t) t + k] = o.gl[k];
  }
}

__device__ __forceinline__ int local_index(int4 n, int v) { return n.x == v ? 0 : (n.y == v ? 1 : 2); }

/* dJ/dx_v and dJ/dM_v (the latter through the logarithm at M_v) */
template <bool F32>
__global__ void k_adj_vertex(DMesh f, int nb_nodes, const AReal<F32>* __restrict__ egp,
                             const AReal<F32>* __restrict__ egl, double* __restrict__ gxy,
                             AReal<F32>* __restrict__ gm) {
  using R = AReal<F32>;
  if (trn_failed(f)) return;
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) {
    const int* st = f.stenc + (size_t) v * f.bucket;
    const int deg = f.alive[v] ? trn_deg(f, v) : 0;
    R gx = 0, gy = 0, g[3] = {0, 0, 0};
    for (int a = 0; a < deg; ++a) {
      const int t = st[a];
      const int j = local_index(f.tri[t], v);
      gx += egp[6 * (size_t) t + 2 * j];
      gy += egp[6 * (size_t) t + 2 * j + 1];
      if (gm) {
        g[0] += egl[3 * (size_t) t];
        g[1] += egl[3 * (size_t) t + 1];
        g[2] += egl[3 * (size_t) t + 2];
      }
    }
    if (gxy) {
      gxy[2 * (size_t) v] = (double) gx;
      gxy[2 * (size_t) v + 1] = (double) gy;
    }
    if (!gm) continue;
    if (deg > 0) {
      const double4 t = f.ten[v];
      const R mat[4] = {R(t.x), R(t.y), R(t.y), R(t.z)};
      R val[2], vec[4];
      eig_x(mat, val, vec);
      const bool shortcut = mat[1] * mat[2] < R(1.e-9);
      const R jac[2][2] = {{R(1) / val[0], R(0)}, {R(0), R(1) / val[1]}};
      const R gam = shortcut ? R(0) : divdiff_log(val[0], val[1]);
      spectral_adjoint(vec, jac, gam, g);
    }
    gm[3 * (size_t) v] = g[0];
    gm[3 * (size_t) v + 1] = g[1];
    gm[3 * (size_t) v + 2] = g[2];
  }
}

/* adjoint of the global scale and clamp (metric.cpp:188-238) at the locally
 * normalised tensor; vfact[v] = this vertex's share of dJ/d(scale) */
template <bool F32>
__global__ void k_adj_global(DMesh f, int nb_nodes, const double4* __restrict__ mloc,
                             const double* complexity, double target, double eig_min,
                             double eig_max, AReal<F32>* __restrict__ gm,
                             double* __restrict__ vfact) {
  using R = AReal<F32>;
  if (trn_failed(f)) return;
  const double fact = target / *complexity;
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) {
    if (!f.alive[v] || trn_deg(f, v) == 0) {
      vfact[v] = 0.0;
      continue;
    }
    const double4 t = mloc[v];
    double mat[4] = {t.x, t.y, t.y, t.z};
    double val[2], vecd[4];
    trn_eigen(mat, val, vecd);
    const bool shortcut = mat[1] * mat[2] < TRN_EPS;
    double fv[2];
    bool in[2];
    for (int k = 0; k < 2; ++k) {
      const double x = val[k] * fact;
      in[k] = x < eig_min && x > eig_max;
      fv[k] = trn_dmax(trn_dmin(x, eig_min), eig_max);
    }
    R gam = 0;
    if (!shortcut) {
      if (in[0] && in[1]) gam = R(fact);
      else if (val[0] != val[1]) gam = R((fv[0] - fv[1]) / (val[0] - val[1]));
    }
    const R jac[2][2] = {{in[0] ? R(fact) : R(0), R(0)}, {R(0), in[1] ? R(fact) : R(0)}};
    const R vec[4] = {R(vecd[0]), R(vecd[1]), R(vecd[2]), R(vecd[3])};
    R g[3] = {gm[3 * (size_t) v], gm[3 * (size_t) v + 1], gm[3 * (size_t) v + 2]};
    R dg[2];
    spectral_adjoint(vec, jac, gam, g, dg);
    gm[3 * (size_t) v] = g[0];
    gm[3 * (size_t) v + 1] = g[1];
    gm[3 * (size_t) v + 2] = g[2];
    vfact[v] = (in[0] ? (double) dg[0] * val[0] : 0.0) + (in[1] ? (double) dg[1] * val[1] : 0.0);
  }
}

/* the complexity's share (metric.cpp:153-185) and the adjoint of the local
 * L^p normalisation (metric.cpp:100-150); graw[v] = dJ/dH_v / patch area,
 * H_v the unsymmetrised Hessian (h11, h12, h21, h22) */
template <bool F32>
__global__ void k_adj_local(DMesh f, int nb_nodes, const double4* __restrict__ hsym,
                            const double4* __restrict__ mloc, const double* __restrict__ astar,
                            const double* __restrict__ atot, const double* complexity,
                            const double* dfact, double target, double scale_exp,
                            const AReal<F32>* __restrict__ gm, AReal<F32>* __restrict__ graw) {
  using R = AReal<F32>;
  if (trn_failed(f)) return;
  const double C = *complexity;
  const double fact = target / C;
  const double dj_dc = -(*dfact) * fact / C;
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) {
    R* out = graw + 4 * (size_t) v;
    if (!f.alive[v] || trn_deg(f, v) == 0) {
      out[0] = out[1] = out[2] = out[3] = R(0);
      continue;
    }
    R g[3] = {gm[3 * (size_t) v], gm[3 * (size_t) v + 1], gm[3 * (size_t) v + 2]};
    const double4 t = mloc[v];
    const double det = t.x * t.z - t.y * t.y;
    if (det > 0) {
      const double w = dj_dc * (astar[v] / 3) / (2 * sqrt(det));
      g[0] += R(w * t.z);
      g[1] -= R(w * t.y);
      g[2] += R(w * t.x);
    }
    const double4 h = hsym[v];
    double mat[4] = {h.x, h.y, h.y, h.z};
    double val[2], vecd[4];
    trn_eigen(mat, val, vecd);
    const bool shortcut = mat[1] * mat[2] < TRN_EPS;
    double lp[2], gp[2];
    for (int k = 0; k < 2; ++k) {
      lp[k] = trn_dmax(fabs(val[k]), TRN_EPS);
      gp[k] = fabs(val[k]) < TRN_EPS ? 0.0 : (val[k] < 0 ? -1.0 : 1.0);
    }
    const double s = pow(lp[0] * lp[1], scale_exp);
    double jd[2][2];
    for (int k = 0; k < 2; ++k)
      for (int l = 0; l < 2; ++l)
        jd[k][l] = gp[l] * (s * (k == l ? 1.0 : 0.0) + scale_exp * s * lp[k] / lp[l]);
    R gam = 0;
    if (!shortcut) {
      if (val[0] != val[1]) gam = R(s * (lp[0] - lp[1]) / (val[0] - val[1]));
      else gam = R(jd[0][0] - jd[0][1]);
    }
    const R jac[2][2] = {{R(jd[0][0]), R(jd[0][1])}, {R(jd[1][0]), R(jd[1][1])}};
    const R vec[4] = {R(vecd[0]), R(vecd[1]), R(vecd[2]), R(vecd[3])};
    spectral_adjoint(vec, jac, gam, g);
    const R ia = R(1.0 / atot[v]);
    out[0] = g[0] * ia;
    out[1] = g[1] * ia;
    out[2] = g[1] * ia;
    out[3] = g[2] * ia;
  }
}

/* the vertices whose 2-ring patch holds element t: its vertices and their
 * neighbours (the patch of v is the stencils of v and of v's neighbours,
 * mesh.cpp:390-434), ascending, deduplicated */
__device__ __forceinline__ int patch_owners(const DMesh& m, int4 n, int* ids) {
  int k = 0;
  const int c[3] = {n.x, n.y, n.z};
  for (int j = 0; j < 3; ++j) {
    const int* vc = m.vic + (size_t) c[j] * m.bucket;
    const int nv = min(m.vdeg[c[j]], m.bucket);
    if (k + 1 + nv > TRN_MAX_PATCH) {
      trn_set_error(m.err, TRN_DERR_BUCKET);
      break;
    }
    ids[k++] = c[j];
    for (int b = 0; b < nv; ++b) ids[k++] = vc[b];
  }
  trn_isort(ids, k);
  return trn_iunique(ids, k);
}

/* ge[t] = area_t * sum over the patch owners i of gv[i] (NC components) */
template <bool F32, int NC>
__global__ void k_adj_elem_patch(DMesh m, int nb_elems, const AReal<F32>* __restrict__ gv,
                                 AReal<F32>* __restrict__ ge) {
  using R = AReal<F32>;
  if (trn_failed(m)) return;
  int ids[TRN_MAX_PATCH];
  for (int t = trn_tid(); t < nb_elems; t += trn_grid_stride()) {
    const int4 n = m.tri[t];
    R acc[NC];
    for (int c = 0; c < NC; ++c) acc[c] = R(0);
    if (n.x >= 0) {
      const int k = patch_owners(m, n, ids);
      for (int a = 0; a < k; ++a)
        for (int c = 0; c < NC; ++c) acc[c] += gv[NC * (size_t) ids[a] + c];
      const double2 p0 = m.pts[n.x], p1 = m.pts[n.y], p2 = m.pts[n.z];
      const R area = R(0.5 * ((p1.x - p0.x) * (p2.y - p0.y) - (p2.x - p0.x) * (p1.y - p0.y)));
      for (int c = 0; c < NC; ++c) acc[c] *= area;
    }
    for (int c = 0; c < NC; ++c) ge[NC * (size_t) t + c] = acc[c];
  }
}

/* dJ/d(recovered gradient)_v / patch area, from the per-element Hessian adjoints */
template <bool F32>
__global__ void k_adj_vertex_hess(DMesh m, int nb_nodes, const AReal<F32>* __restrict__ ge4,
                                  const double* __restrict__ atot, AReal<F32>* __restrict__ gg) {
  using R = AReal<F32>;
  if (trn_failed(m)) return;
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) {
    const int* st = m.stenc + (size_t) v * m.bucket;
    const int deg = m.alive[v] ? trn_deg(m, v) : 0;
    R gx = 0, gy = 0;
    for (int a = 0; a < deg; ++a) {
      const int t = st[a];
      const ElemGrad e = elem_grad(m, t);
      const int j = local_index(e.v, v);
      const R px = R(e.d[2 * j]), py = R(e.d[2 * j + 1]);
      const R* r = ge4 + 4 * (size_t) t;
      gx += r[0] * px + r[1] * py;
      gy += r[2] * px + r[3] * py;
    }
    const R ia = deg > 0 ? R(1.0 / atot[v]) : R(0);
    gg[2 * (size_t) v] = gx * ia;
    gg[2 * (size_t) v + 1] = gy * ia;
  }
}

template <bool F32>
__global__ void k_adj_vertex_u(DMesh m, int nb_nodes, const AReal<F32>* __restrict__ ge2,
                               double* __restrict__ gu) {
  using R = AReal<F32>;
  if (trn_failed(m)) return;
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) {
    const int* st = m.stenc + (size_t) v * m.bucket;
    const int deg = m.alive[v] ? trn_deg(m, v) : 0;
    R g = 0;
    for (int a = 0; a < deg; ++a) {
      const int t = st[a];
      const ElemGrad e = elem_grad(m, t);
      const int j = local_index(e.v, v);
      const R* r = ge2 + 2 * (size_t) t;
      g += r[0] * R(e.d[2 * j]) + r[1] * R(e.d[2 * j + 1]);
    }
    gu[v] = (double) g;
  }
}

/* stencil areas: sum of the signed areas of the elements around v */
__global__ void k_adj_star_area(DMesh m, int nb_nodes, double* __restrict__ astar) {
  if (trn_failed(m)) return;
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) {
    const int* st = m.stenc + (size_t) v * m.bucket;
    const int deg = m.alive[v] ? trn_deg(m, v) : 0;
    double a = 0;
    for (int k = 0; k < deg; ++k) a += elem_grad(m, st[k]).area;
    astar[v] = a;
  }
}

/* ------------------------------------------------------------------------ */

void adj_ws_free(AdjWs* ws) {
  for (void* p : {(void*) ws->ten, (void*) ws->lten, (void*) ws->mloc, (void*) ws->hsym,
                  (void*) ws->atot, (void*) ws->astar, (void*) ws->q, (void*) ws->egp,
                  (void*) ws->egl, (void*) ws->vbuf, (void*) ws->ebuf, (void*) ws->vfact,
                  (void*) ws->scal})
    if (p) cudaFree(p);
  *ws = AdjWs{};
}

int adj_ws_ensure(AdjWs* ws, int nv, int ne) {
  if (nv <= ws->cap_v && ne <= ws->cap_e && ws->scal) return 0;
  adj_ws_free(ws);
  const size_t V = (size_t) std::max(nv, 1), E = (size_t) std::max(ne, 1);
  bool ok = cudaMalloc(&ws->ten, V * sizeof(double4)) == cudaSuccess &&
            cudaMalloc(&ws->lten, V * sizeof(double4)) == cudaSuccess &&
            cudaMalloc(&ws->mloc, V * sizeof(double4)) == cudaSuccess &&
            cudaMalloc(&ws->hsym, V * sizeof(double4)) == cudaSuccess &&
            cudaMalloc(&ws->atot, V * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&ws->astar, V * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&ws->q, (E + 8192) * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&ws->egp, 6 * E * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&ws->egl, 4 * E * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&ws->vbuf, 8 * V * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&ws->ebuf, 4 * E * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&ws->vfact, (V + 8192) * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&ws->scal, 8 * sizeof(double)) == cudaSuccess;
  if (!ok) {
    adj_ws_free(ws);
    return 1;
  }
  ws->cap_v = (int) V;
  ws->cap_e = (int) E;
  return 0;
}

template <bool F32>
static void adjoint_impl(const DMesh& m, int nb_nodes, int nb_elems, const double2* xy,
                         const AdjMetric* um, AdjWs& ws, double* gxy, double* gu, cudaStream_t s) {
  using R = AReal<F32>;
  const double V = nb_nodes, E = nb_elems, r = sizeof(R);
  DMesh f = m;
  f.lten = ws.lten;
  if (um) {
    f.ten = ws.ten;
    MetricSaves keep;
    keep.atot = ws.atot;
    keep.hsym = ws.hsym;
    keep.mloc = ws.mloc;
    DMesh g = f;
    g.lten = nullptr;
    metric_run(g, nb_nodes, nb_elems, um->solut, um->grad, um->terms, ws.scal + 0, um->exact_sum,
               um->p, s, &keep);
  }
  log_cache(f, nb_nodes, F32, s);
  /* the solution's adjoint only when its output is asked for */
  const bool back_u = um != nullptr && gu != nullptr;
  R* egp = reinterpret_cast<R*>(ws.egp);
  R* egl = back_u ? reinterpret_cast<R*>(ws.egl) : nullptr;
  {
    ProfScope ps("adjoint_elem", s, E * (kTri + 8 + 6 * r + (egl ? 3 * r : 0)) + V * (kPt + 4 * r));
    k_adj_elem<F32><<<grid_for(nb_elems, 128), 128, 0, s>>>(f, nb_elems, xy ? xy : m.pts, ws.q,
                                                          egp, egl);
    note_launch();
  }
  sum_tree(ws.q, nb_elems, ws.q + nb_elems, ws.scal + 1, s);
  R* gm = reinterpret_cast<R*>(ws.vbuf);
  if (gxy || back_u) {
    ProfScope ps("adjoint_vertex", s,
                 V * (kIdx + 1 + (gxy ? 16 : 0) + (back_u ? kTen + 3 * r : 0)) +
                     E * (6 * r + (back_u ? 3 * r : 0) + kTri));
    k_adj_vertex<F32><<<grid_for(nb_nodes), TRN_THREADS, 0, s>>>(f, nb_nodes, egp, egl, gxy,
                                                                 back_u ? gm : nullptr);
    note_launch();
  }
  if (!back_u) {
    check_launch("quality_adjoint");
    return;
  }
  k_adj_global<F32><<<grid_for(nb_nodes), TRN_THREADS, 0, s>>>(
      f, nb_nodes, ws.mloc, ws.scal + 0, um->p.target, um->p.eig_min, um->p.eig_max, gm, ws.vfact);
  note_launch();
  sum_tree(ws.vfact, nb_nodes, ws.vfact + nb_nodes, ws.scal + 2, s);
  k_adj_star_area<<<grid_for(nb_nodes), TRN_THREADS, 0, s>>>(f, nb_nodes, ws.astar);
  note_launch();
  R* graw = reinterpret_cast<R*>(ws.vbuf) + 3 * (size_t) nb_nodes;
  k_adj_local<F32><<<grid_for(nb_nodes), TRN_THREADS, 0, s>>>(
      f, nb_nodes, ws.hsym, ws.mloc, ws.astar, ws.atot, ws.scal + 0, ws.scal + 2, um->p.target,
      um->p.scale_exp, gm, graw);
  note_launch();
  R* ebuf = reinterpret_cast<R*>(ws.ebuf);
  {
    ProfScope ps("adjoint_patch", s, E * (kTri + 4 * r) + V * (kPt + 4 * r + kIdx * kAvgDeg));
    k_adj_elem_patch<F32, 4><<<grid_for(nb_elems, 128), 128, 0, s>>>(f, nb_elems, graw, ebuf);
    note_launch();
  }
  R* ggrad = gm;   /* dJ/dM is consumed: reuse its space */
  k_adj_vertex_hess<F32><<<grid_for(nb_nodes), TRN_THREADS, 0, s>>>(f, nb_nodes, ebuf, ws.atot,
                                                                    ggrad);
  note_launch();
  {
    ProfScope ps("adjoint_patch", s, E * (kTri + 2 * r) + V * (kPt + 2 * r + kIdx * kAvgDeg));
    k_adj_elem_patch<F32, 2><<<grid_for(nb_elems, 128), 128, 0, s>>>(f, nb_elems, ggrad, ebuf);
    note_launch();
  }
  k_adj_vertex_u<F32><<<grid_for(nb_nodes), TRN_THREADS, 0, s>>>(f, nb_nodes, ebuf, gu);
  note_launch();
  check_launch("quality_adjoint");
}

void quality_adjoint(const DMesh& m, int nb_nodes, int nb_elems, const double2* xy,
                     const AdjMetric* um, bool fp32, AdjWs& ws, double* gxy, double* gu,
                     cudaStream_t s) {
  if (fp32) adjoint_impl<true>(m, nb_nodes, nb_elems, xy, um, ws, gxy, um ? gu : nullptr, s);
  else adjoint_impl<false>(m, nb_nodes, nb_elems, xy, um, ws, gxy, um ? gu : nullptr, s);
}

/* ------------------------------------------------------------------------ */
/* gradient-based smoothing: one color class of interior vertices. Each
 * vertex v moves along M_v^-1 g, g the gradient at v of its elements' summed
 * quality (mode bit 0 clear) or summed log-quality (bit 0 set: each element's
 * adjoint weighted by 1/q, so the worst elements lead). With mode bit 1 the
 * vertex's tensor becomes the log-Euclidean mean of its neighbours' tensors
 * when it moves, as Smooth::moveSmartLaplacian does (smoothing.cpp:64-81),
 * and the gradient is taken under that tensor; otherwise the tensor stays.
 * The step's metric length is max_len times the mean metric length of v's
 * edges, and it backs off 1, 1/2, .., 1/16 until every element stays CCW
 * with quality above the old stencil minimum and the objective grows. */
template <bool F32>
__device__ int move_gradient(const DMesh& m, int i, double max_len, int mode) {
  const bool use_log = (mode & 1) != 0, follow = (mode & 2) != 0;
  const int* st = m.stenc + (size_t) i * m.bucket;
  const int deg = trn_deg(m, i);
  double q_min = 1.7976931348623157e308, obj = 0;
  for (int a = 0; a < deg; ++a) {
    const double q = m.qual[st[a]];
    q_min = trn_dmin(q_min, q);
    obj += use_log ? log(q) : q;
  }
  const double2 pini = m.pts[i];
  const double4 tini = m.ten[i];
  const LogT<F32> lini = log_load<F32>(m, i);
  double4 tnew = tini;
  LogT<F32> lnew = lini;
  if (follow) {
    const int* vc = m.vic + (size_t) i * m.bucket;
    const int nb_neigh = min(m.vdeg[i], m.bucket);
    if (nb_neigh == 0) return 0;
    LogSum<F32> lsum;
    for (int k = 0; k < nb_neigh; ++k) lsum.add(log_load<F32>(m, vc[k]));
    double tn[3];
    lsum.finish(nb_neigh, tn);
    tnew = make_double4(tn[0], tn[1], tn[2], 0.0);
    lnew = log_of<F32>(tn[0], tn[1], tn[2]);
  }
  double gx = 0, gy = 0;
  for (int a = 0; a < deg; ++a) {
    const int4 n = m.tri[st[a]];
    ElemAdj<F32> o;
    quality_adjoint<F32>(m.pts[n.x], m.pts[n.y], m.pts[n.z],
                         n.x == i ? lnew : log_load<F32>(m, n.x),
                         n.y == i ? lnew : log_load<F32>(m, n.y),
                         n.z == i ? lnew : log_load<F32>(m, n.z), false, o);
    const int j = local_index(n, i);
    const double w = use_log ? 1.0 / trn_dmax(o.q, 1e-300) : 1.0;
    gx += w * (double) o.gp[2 * j];
    gy += w * (double) o.gp[2 * j + 1];
  }
  const double4 t = tnew;
  const double det = t.x * t.z - t.y * t.y;
  if (!(det > 0)) return 0;
  const double dx = (t.z * gx - t.y * gy) / det;
  const double dy = (t.x * gy - t.y * gx) / det;
  const double gn = sqrt(gx * dx + gy * dy);   /* metric length of (dx, dy) */
  if (!(gn > 0) || !isfinite(gn)) return 0;
  /* the step: max_len times the mean metric length (under M_v) of v's edges */
  double lsum = 0;
  int lcnt = 0;
  for (int a = 0; a < deg; ++a) {
    const int4 n = m.tri[st[a]];
    const int j = local_index(n, i);
    const int w = j == 0 ? n.y : (j == 1 ? n.z : n.x);   /* next vertex: each edge once */
    const double ex = m.pts[w].x - pini.x, ey = m.pts[w].y - pini.y;
    lsum += sqrt(ex * (t.x * ex + t.y * ey) + ey * (t.y * ex + t.z * ey));
    ++lcnt;
  }
  double eta = max_len * (lsum / lcnt) / gn;
  double qual[TRN_MAX_DEG];
  bool valid = false;
  for (int retry = 0; retry < 5 && !valid; ++retry, eta *= 0.5) {
    const double2 pa = make_double2(pini.x + eta * dx, pini.y + eta * dy);
    double sum = 0;
    valid = true;
    for (int a = 0; valid && a < deg; ++a) {
      const int4 n = m.tri[st[a]];
      const double2 p0 = (n.x == i) ? pa : m.pts[n.x];
      const double2 p1 = (n.y == i) ? pa : m.pts[n.y];
      const double2 p2 = (n.z == i) ? pa : m.pts[n.z];
      valid = false;
      if (trn_ccw(p0, p1, p2)) {
        const LogT<F32> l0 = (n.x == i) ? lnew : log_load<F32>(m, n.x);
        const LogT<F32> l1 = (n.y == i) ? lnew : log_load<F32>(m, n.y);
        const LogT<F32> l2 = (n.z == i) ? lnew : log_load<F32>(m, n.z);
        qual[a] = quality_x(p0, p1, p2, l0, l1, l2);
        valid = qual[a] > q_min;
        sum += use_log ? log(qual[a]) : qual[a];
      }
    }
    if (valid && !(sum > obj)) valid = false;
    if (valid) {
      m.pts[i] = pa;
      if (follow) {
        ten_store<F32>(m, i, tnew);
        log_store<F32>(m, i, lnew);
      }
      for (int a = 0; a < deg; ++a) m.qual[st[a]] = qual[a];
    }
  }
  return valid ? 1 : 0;
}

template <bool F32>
__global__ void k_smooth_gradient(DMesh m, const int* __restrict__ list, int n, double max_len,
                                  int mode, int* counters) {
  if (trn_failed(m)) return;
  int tasks = 0, commit = 0;
  for (int q = trn_tid(); q < n; q += trn_grid_stride()) {
    const int v = list[q];
    if (v < 0 || v >= m.capa_node) {
      trn_set_error(m.err, TRN_DERR_INVALID);
      continue;
    }
    if (!m.activ[v] || trn_deg(m, v) == 0) continue;
    tasks++;
    commit += move_gradient<F32>(m, v, max_len, mode);
  }
  trn_warp_add(counters, tasks);
  trn_warp_add(counters + 1, commit);
}

void smooth_gradient_color(const DMesh& m, const int* list, int n, double max_len, int mode,
                           int* counters, bool fp32, cudaStream_t s) {
  if (n <= 0) return;
  const double own = 4 + 1 + 4 + 2 * kPt + kTen + kAvgDeg * (kIdx + kTri + 2 * kQ);
  const double nbr = (double) std::min<long long>((long long) m.capa_node, 6LL * n) * (kPt + kTen);
  ProfScope ps("smooth_gradient", s, n * own + nbr);
  if (fp32)
    k_smooth_gradient<true><<<grid_for(n, 128), 128, 0, s>>>(m, list, n, max_len, mode, counters);
  else
    k_smooth_gradient<false><<<grid_for(n, 128), 128, 0, s>>>(m, list, n, max_len, mode, counters);
  note_launch();
  check_launch("smooth_gradient");
}

}  // namespace trn
