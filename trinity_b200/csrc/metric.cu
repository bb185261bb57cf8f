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
 *
 * Patch order matters: the reference sums over the patch in ascending element
 * id (std::set order, mesh.cpp:396-432), so each thread gathers the stencils
 * of the vertex and of its neighbours, sorts and deduplicates them first.
 */
#include "trn_internal.h"
#include "trn_numeric.cuh"

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

void sum_tree(const double* in, int n, double* partial, double* out, cudaStream_t s) {
  const int nb = grid_for(n);
  k_sum_partial<<<nb, TRN_THREADS, 0, s>>>(in, n, partial);
  note_launch();
  k_sum_final<<<1, TRN_THREADS, 0, s>>>(partial, nb, out);
  note_launch();
}

void metric_run(const DMesh& m, int nb_nodes, int nb_elems, const double* solut, double2* grad,
                double* terms, double* complexity, bool exact_sum, const MetricParams& p,
                cudaStream_t s, const MetricSaves* keep) {
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
