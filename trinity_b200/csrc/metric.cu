/*
 * metric.cu — Hessian-based metric recovery (Metrics::run, metric.cpp:59-70).
 *
 *   k_gradient        per vertex: area-weighted mean of the P1 gradients over
 *                     the 2-ring element patch (hessian.cpp:24-83)
 *   k_hessian_local   per vertex: the same on the gradient field, symmetrised
 *                     (hessian.cpp:86-153), then |H| eigen-clamp and local L^p
 *                     scale det^(-1/(2p+2)) (metric.cpp:100-150), fused
 *   k_complexity_term per element: area * mean_k sqrt(det M_k) (metric.cpp:159-181)
 *   k_sum_*           the complexity sum: either one thread in element order
 *                     (bit-identical to the reference's 1-thread sum) or a
 *                     deterministic two-level tree
 *   k_normalize       global scale target/complexity and eigenvalue clamp to
 *                     [1/h_max^2, 1/h_min^2] (metric.cpp:188-238)
 *   k_*_f32           the same recovery in FP32 for the mixed-precision form
 *
 * Patch order matters: the reference sums over the patch in ascending element
 * id (std::set order, mesh.cpp:396-432), so each thread gathers the stencils
 * of the vertex and of its neighbours, sorts and deduplicates them first.
 */
#include "trn_internal.h"
#include "trn_mixed.cuh"

namespace trn {

__device__ __forceinline__ int gather_patch(const DMesh& m, int v, int* patch) {
  int k = 0;
  const int* s = m.stenc + (size_t) v * m.bucket;
  int d = trn_deg(m, v);
  for (int a = 0; a < d && k < TRN_MAX_PATCH; ++a) patch[k++] = s[a];
  const int* vc = m.vic + (size_t) v * m.bucket;
  int nv = m.vdeg[v];
  for (int b = 0; b < nv; ++b) {
    int w = vc[b];
    const int* sw = m.stenc + (size_t) w * m.bucket;
    int dw = trn_deg(m, w);
    for (int a = 0; a < dw; ++a) {
      if (k == TRN_MAX_PATCH) {
        trn_set_error(m.err, TRN_DERR_BUCKET);
        break;
      }
      patch[k++] = sw[a];
    }
  }
  trn_isort(patch, k);
  return trn_iunique(patch, k);
}

__global__ void k_gradient(DMesh m, int nb_nodes, const double* __restrict__ solut,
                           double2* __restrict__ grad, double* __restrict__ atot) {
  if (trn_failed(m)) return;
  int patch[TRN_MAX_PATCH];
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) {
    int n = gather_patch(m, v, patch);
    double total_area = 0.;
    double gx = 0., gy = 0.;
    /* the reference stores per-element (area, grad) and sums afterwards in the
     * same element order; interleaving the two loops keeps every sum's order */
    for (int i = 0; i < n; ++i) {
      ElemGrad g = elem_grad(m, patch[i]);
      total_area += g.area;
      double s0 = solut[g.v.x], s1 = solut[g.v.y], s2 = solut[g.v.z];
      double ex = 0, ey = 0;
      ex += s0 * g.d[0];
      ey += s0 * g.d[1];
      ex += s1 * g.d[2];
      ey += s1 * g.d[3];
      ex += s2 * g.d[4];
      ey += s2 * g.d[5];
      gx += (g.area * ex);
      gy += (g.area * ey);
    }
    gx /= total_area;
    gy /= total_area;
    grad[v] = make_double2(gx, gy);
    if (atot) atot[v] = total_area;
  }
}

__global__ void k_hessian_local(DMesh m, int nb_nodes, const double2* __restrict__ grad,
                                double scale_exp, double4* __restrict__ hsym,
                                double4* __restrict__ mloc) {
  if (trn_failed(m)) return;
  int patch[TRN_MAX_PATCH];
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) {
    int n = gather_patch(m, v, patch);
    double total_area = 0;
    double h[4] = {0, 0, 0, 0};
    for (int i = 0; i < n; ++i) {
      ElemGrad g = elem_grad(m, patch[i]);
      total_area += g.area;
      double2 g0 = grad[g.v.x], g1 = grad[g.v.y], g2 = grad[g.v.z];
      double dl[4] = {0, 0, 0, 0};
      dl[0] += (g0.x * g.d[0]);
      dl[1] += (g0.x * g.d[1]);
      dl[2] += (g0.y * g.d[0]);
      dl[3] += (g0.y * g.d[1]);
      dl[0] += (g1.x * g.d[2]);
      dl[1] += (g1.x * g.d[3]);
      dl[2] += (g1.y * g.d[2]);
      dl[3] += (g1.y * g.d[3]);
      dl[0] += (g2.x * g.d[4]);
      dl[1] += (g2.x * g.d[5]);
      dl[2] += (g2.y * g.d[4]);
      dl[3] += (g2.y * g.d[5]);
      for (int j = 0; j < 4; ++j) h[j] += g.area * dl[j];
    }
    for (int j = 0; j < 4; ++j) h[j] /= total_area;
    /* symmetrise (hessian.cpp:149-152) */
    double t0 = h[0];
    double t1 = 0.5 * (h[1] + h[2]);
    double t2 = h[3];
    if (hsym) hsym[v] = make_double4(t0, t1, t2, 0.0);
    /* normalizeLocally (metric.cpp:107-149) */
    double mm[4] = {t0, t1, t1, t2};
    double val[2] = {0, 0}, vec[4] = {0, 0, 0, 0};
    trn_eigen(mm, val, vec);
    val[0] = trn_dmax(fabs(val[0]), TRN_EPS);
    val[1] = trn_dmax(fabs(val[1]), TRN_EPS);
    double det = val[0] * val[1];
    double scale_loc = trn_pow(det, scale_exp);
    val[0] *= scale_loc;
    val[1] *= scale_loc;
    const double4 r = trn_recompose(val, vec);
    m.ten[v] = r;
    if (mloc) mloc[v] = r;
  }
}

/* ---- the mixed-precision form of the recovery ----
 * The same patch means in FP32. Every coordinate difference is taken in
 * FP64 and then rounded; each nodal value enters as its difference to the
 * patch centre's value (the element's three P1 basis gradients sum to zero,
 * so this changes nothing in exact arithmetic and removes the cancellation
 * of summing values of nearly equal size, which single precision could not
 * afford); area x basis gradient is formed directly from the rotated edges
 * (area x 2/area x edge), so no division per element. The eigen-clamp, the
 * local L^p scale and the global scaling are FP32 too; the complexity sum
 * stays FP64. */
__device__ __forceinline__ void elem_edges_f32(const DMesh& m, int4 t, float* area, float* ey, float* ex) {
  const double2 p0 = m.pts[t.x], p1 = m.pts[t.y], p2 = m.pts[t.z];
  /* rotated edges: area x d[2j] = 2 ey[j], area x d[2j+1] = 2 ex[j] */
  ey[0] = (float) (p1.y - p2.y);
  ex[0] = (float) (p2.x - p1.x);
  ey[1] = (float) (p2.y - p0.y);
  ex[1] = (float) (p0.x - p2.x);
  ey[2] = (float) (p0.y - p1.y);
  ex[2] = (float) (p1.x - p0.x);
  const float c0 = (float) (p1.x - p0.x), c1 = (float) (p2.x - p0.x);
  const float c2 = (float) (p1.y - p0.y), c3 = (float) (p2.y - p0.y);
  *area = 0.5f * (c0 * c3 - c1 * c2);
}

__global__ void k_gradient_f32(DMesh m, int nb_nodes, const double* __restrict__ solut,
                               double2* __restrict__ grad) {
  if (trn_failed(m)) return;
  int patch[TRN_MAX_PATCH];
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) {
    const int n = gather_patch(m, v, patch);
    const double uv = solut[v];
    float tot = 0.f, gx = 0.f, gy = 0.f;
    for (int i = 0; i < n; ++i) {
      const int4 t = m.tri[patch[i]];
      float area, ey[3], ex[3];
      elem_edges_f32(m, t, &area, ey, ex);
      const float s[3] = {(float) (solut[t.x] - uv), (float) (solut[t.y] - uv), (float) (solut[t.z] - uv)};
      tot += area;
      gx += 2.f * (s[0] * ey[0] + s[1] * ey[1] + s[2] * ey[2]);
      gy += 2.f * (s[0] * ex[0] + s[1] * ex[1] + s[2] * ex[2]);
    }
    const float it = __frcp_rn(tot);
    grad[v] = make_double2((double) (gx * it), (double) (gy * it));
  }
}

__global__ void k_hessian_local_f32(DMesh m, int nb_nodes, const double2* __restrict__ grad, float scale_exp) {
  if (trn_failed(m)) return;
  int patch[TRN_MAX_PATCH];
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) {
    const int n = gather_patch(m, v, patch);
    const double2 gv = grad[v];
    float tot = 0.f, h[4] = {0.f, 0.f, 0.f, 0.f};
    for (int i = 0; i < n; ++i) {
      const int4 t = m.tri[patch[i]];
      float area, ey[3], ex[3];
      elem_edges_f32(m, t, &area, ey, ex);
      const int id[3] = {t.x, t.y, t.z};
      tot += area;
      for (int j = 0; j < 3; ++j) {
        const double2 g = grad[id[j]];
        const float dx = (float) (g.x - gv.x), dy = (float) (g.y - gv.y);
        h[0] += 2.f * (dx * ey[j]);
        h[1] += 2.f * (dx * ex[j]);
        h[2] += 2.f * (dy * ey[j]);
        h[3] += 2.f * (dy * ex[j]);
      }
    }
    const float it = __frcp_rn(tot);
    const float t0 = h[0] * it, t1 = 0.5f * (h[1] + h[2]) * it, t2 = h[3] * it;
    float mm[4] = {t0, t1, t1, t2}, val[2], vec[4];
    trnf_eigen(mm, val, vec);
    val[0] = trnf_max(fabsf(val[0]), 1.e-9f);
    val[1] = trnf_max(fabsf(val[1]), 1.e-9f);
    const float scale_loc = powf(val[0] * val[1], scale_exp);
    val[0] *= scale_loc;
    val[1] *= scale_loc;
    const float c0 = val[0] * vec[0], c1 = val[0] * vec[2], c2 = val[1] * vec[1], c3 = val[1] * vec[3];
    m.ten[v] = make_double4((double) (vec[0] * c0 + vec[1] * c2), (double) (vec[0] * c1 + vec[1] * c3),
                            (double) (vec[2] * c1 + vec[3] * c3), 0.0);
  }
}

__global__ void k_complexity_term(DMesh m, int nb_elems, double* __restrict__ terms) {
  if (trn_failed(m)) return;
  for (int i = trn_tid(); i < nb_elems; i += trn_grid_stride()) {
    int4 v = m.tri[i];
    if (v.x < 0) {
      terms[i] = 0.0;
      continue;
    }
    double2 p0 = m.pts[v.x], p1 = m.pts[v.y], p2 = m.pts[v.z];
    double s0 = p1.x - p0.x;
    double s1 = p2.x - p0.x;
    double s2 = p1.y - p0.y;
    double s3 = p2.y - p0.y;
    double area = 0.5 * (s0 * s3 - s1 * s2);
    double rho = 0.;
    int ids[3] = {v.x, v.y, v.z};
    for (int j = 0; j < 3; ++j) {
      double4 t = m.ten[ids[j]];
      double det = t.x * t.z - trn_pow(t.y, 2);
      rho += sqrt(det);
    }
    rho /= 3;
    terms[i] = rho * area;
  }
}

/* one thread, element order: the 1-thread reference's summation */
__global__ void k_sum_sequential(const double* __restrict__ terms, int n, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double phi = 0.;
  int i = 0;
  for (; i + 8 <= n; i += 8) {
    double a0 = terms[i], a1 = terms[i + 1], a2 = terms[i + 2], a3 = terms[i + 3];
    double a4 = terms[i + 4], a5 = terms[i + 5], a6 = terms[i + 6], a7 = terms[i + 7];
    phi += a0; phi += a1; phi += a2; phi += a3;
    phi += a4; phi += a5; phi += a6; phi += a7;
  }
  for (; i < n; ++i) phi += terms[i];
  *out = 0 + phi;
}

/* deterministic tree: fixed per-block partials, then one block in order */
__global__ void k_sum_partial(const double* __restrict__ terms, int n, double* partial) {
  __shared__ double sm[TRN_THREADS];
  double s = 0;
  for (int i = trn_tid(); i < n; i += trn_grid_stride()) s += terms[i];
  sm[threadIdx.x] = s;
  __syncthreads();
  for (int o = TRN_THREADS / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sm[0];
}

__global__ void k_sum_final(const double* __restrict__ partial, int nb, double* out) {
  __shared__ double sm[TRN_THREADS];
  double s = 0;
  for (int i = threadIdx.x; i < nb; i += TRN_THREADS) s += partial[i];
  sm[threadIdx.x] = s;
  __syncthreads();
  for (int o = TRN_THREADS / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sm[0];
}

__global__ void k_normalize(DMesh m, int nb_nodes, const double* complexity, double target,
                            double eig_min, double eig_max) {
  if (trn_failed(m)) return;
  double fact = target / *complexity;
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) {
    double4 t = m.ten[v];
    double mm[4] = {t.x, t.y, t.y, t.z};
    double val[2], vec[4];
    trn_eigen(mm, val, vec);
    val[0] *= fact;
    val[1] *= fact;
    for (int j = 0; j < 2; ++j) {
      val[j] = trn_dmin(val[j], eig_min);
      val[j] = trn_dmax(val[j], eig_max);
    }
    double4 t4 = trn_recompose(val, vec);
    m.ten[v] = t4;
    if (m.lten) m.lten[v] = trn_log_tensor(t4.x, t4.y, t4.z);
  }
}

__global__ void k_normalize_f32(DMesh m, int nb_nodes, const double* complexity, double target,
                                double eig_min, double eig_max) {
  if (trn_failed(m)) return;
  const float fact = (float) (target / *complexity);
  const float lo = (float) eig_max, hi = (float) eig_min;
  for (int v = trn_tid(); v < nb_nodes; v += trn_grid_stride()) {
    const double4 t = m.ten[v];
    float mm[4] = {(float) t.x, (float) t.y, (float) t.y, (float) t.z}, val[2], vec[4];
    trnf_eigen(mm, val, vec);
    for (int j = 0; j < 2; ++j) val[j] = trnf_max(trnf_min(val[j] * fact, hi), lo);
    const float c0 = val[0] * vec[0], c1 = val[0] * vec[2], c2 = val[1] * vec[1], c3 = val[1] * vec[3];
    const float r0 = vec[0] * c0 + vec[1] * c2, r1 = vec[0] * c1 + vec[1] * c3, r2 = vec[2] * c1 + vec[3] * c3;
    m.ten[v] = make_double4((double) r0, (double) r1, (double) r2, 0.0);
    if (m.tenf) m.tenf[v] = make_float4(r0, r1, r2, 0.f);
    if (m.lten) reinterpret_cast<float4*>(m.lten)[v] = trnf_log_tensor(r0, r1, r2);
  }
}

void sum_tree(const double* in, int n, double* partial, double* out, cudaStream_t s) {
  const int nb = grid_for(n);
  k_sum_partial<<<nb, TRN_THREADS, 0, s>>>(in, n, partial);
  note_launch();
  k_sum_final<<<1, TRN_THREADS, 0, s>>>(partial, nb, out);
  note_launch();
}

void metric_run(const DMesh& m, int nb_nodes, int nb_elems, const double* solut, double2* grad,
                double* terms, double* complexity, bool exact_sum, const MetricParams& p,
                cudaStream_t s, const MetricSaves* keep, bool fp32) {
  if (fp32) {
    const double V = nb_nodes, E = nb_elems;
    {
    ProfScope ps("metric_gradient", s, V * (2 * kIdx + kAvgDeg * kIdx * 2 + 8 + kPt + 16) + E * kTri);
    k_gradient_f32<<<grid_for(nb_nodes), TRN_THREADS, 0, s>>>(m, nb_nodes, solut, grad);
    note_launch();
    }
    {
    ProfScope ps("metric_hessian", s, V * (2 * kIdx + kAvgDeg * kIdx * 2 + 16 + kPt + kTen) + E * kTri);
    k_hessian_local_f32<<<grid_for(nb_nodes), TRN_THREADS, 0, s>>>(m, nb_nodes, grad, (float) p.scale_exp);
    note_launch();
    }
    ProfScope ps("metric_complexity", s, E * (kTri + 8) + V * (kPt + kTen));
    k_complexity_term<<<grid_for(nb_elems), TRN_THREADS, 0, s>>>(m, nb_elems, terms);
    note_launch();
    if (exact_sum) {
      k_sum_sequential<<<1, 32, 0, s>>>(terms, nb_elems, complexity);
      note_launch();
    } else {
      sum_tree(terms, nb_elems, terms + m.capa_elem, complexity, s);
    }
    ProfScope ps2("metric_normalize", s, V * 2 * kTen);
    k_normalize_f32<<<grid_for(nb_nodes), TRN_THREADS, 0, s>>>(m, nb_nodes, complexity, p.target,
                                                                p.eig_min, p.eig_max);
    note_launch();
    check_launch("metric_run");
    return;
  }
  double* atot = keep ? keep->atot : nullptr;
  double4* hsym = keep ? keep->hsym : nullptr;
  double4* mloc = keep ? keep->mloc : nullptr;
  const double V = nb_nodes, E = nb_elems;
  {
  ProfScope ps("metric_gradient", s, V * (2 * kIdx + kAvgDeg * kIdx * 2 + 8 + kPt + 16) + E * kTri);
  k_gradient<<<grid_for(nb_nodes), TRN_THREADS, 0, s>>>(m, nb_nodes, solut, grad, atot);
  note_launch();
  }
  {
  ProfScope ps("metric_hessian", s, V * (2 * kIdx + kAvgDeg * kIdx * 2 + 16 + kPt + kTen) + E * kTri);
  k_hessian_local<<<grid_for(nb_nodes), TRN_THREADS, 0, s>>>(m, nb_nodes, grad, p.scale_exp,
                                                                hsym, mloc);
  note_launch();
  }
  ProfScope ps("metric_complexity", s, E * (kTri + 8) + V * (kPt + kTen));
  k_complexity_term<<<grid_for(nb_elems), TRN_THREADS, 0, s>>>(m, nb_elems, terms);
  note_launch();
  if (exact_sum) {
    k_sum_sequential<<<1, 32, 0, s>>>(terms, nb_elems, complexity);
    note_launch();
  } else {
    /* partials live after the terms (terms has capa_elem + grid slots) */
    sum_tree(terms, nb_elems, terms + m.capa_elem, complexity, s);
  }
  ProfScope ps2("metric_normalize", s, V * 2 * kTen);
  k_normalize<<<grid_for(nb_nodes), TRN_THREADS, 0, s>>>(m, nb_nodes, complexity, p.target,
                                                          p.eig_min, p.eig_max);
  note_launch();
  check_launch("metric_run");
}

}  // namespace trn
