/*
 * trn_oracle.c — TEST INFRASTRUCTURE ONLY: the CPU oracle for the adaptation
 * round. Single-threaded C restatement of trinity's algorithm in the order its
 * 1-thread OpenMP execution takes; every function names the reference
 * function (file:line, paths inside the trinity project) it restates.
 *
 * Floating point: every expression keeps the reference's operand order; the
 * file is compiled with -ffp-contract=off and calls the project's log/exp/pow
 * (trinity_b200/csrc/trn_libm.h), like the pinned reference build.
 *
 * State quirks reproduced on purpose (they change results):
 *   - one activity byte array shared by vertices and elements (mesh.h:146);
 *   - vertex adjacency ("vicin") rebuilt only for flagged vertices, so
 *     boundary vertices keep a stale one during smoothing (smoothing.cpp:134-140);
 *   - the element -> dual-index mapping of swapping is reset once per run,
 *     so stale entries point at older dual lists (swapping.cpp:161-162, 246);
 *   - the first-fit coloring keeps one "forbidden" array for the whole call
 *     (partition.cpp:84-87).
 */
#include "trn_oracle.h"

#include "../trinity_b200/csrc/trn_libm.h"

#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define EPS 1.e-9
static const double L_MIN = 0.707106781186547;  /* header.h:66 */
static const double L_MAX = 1.414213562373095;  /* header.h:67 */
static const double Q_MIN = 0.9;                /* header.h:69 */
#define TAG_BOUND 4                             /* header.h:58 */
#define TAG_CORNER 8                            /* header.h:59 */
#define MAX_PART 8                              /* main.cpp:42: Partit(&mesh, 8) */
#define MATCHED (-2)                            /* matching.h:27 */
#define LOOP_CAP 100000

typedef struct { int* a; int n, cap; } ivec;

static void iv_push(ivec* v, int x) {
  if (v->n == v->cap) {
    v->cap = v->cap ? v->cap * 2 : 64;
    v->a = (int*) realloc(v->a, sizeof(int) * (size_t) v->cap);
  }
  v->a[v->n++] = x;
}

struct orc_mesh {
  int nb_nodes, nb_elems, capa_node, capa_elem, bucket, vstride;
  double *points, *tensor, *solut, *qualit, *gradient;
  int *elems, *stenc, *deg, *vicin, *vdeg;
  uint8_t *alive, *tags;
  signed char* activ;
  char* fixes;
  /* Partit state (partition.h:56-76) */
  int* subset[MAX_PART];
  int cardin[MAX_PART];
  int nb_parts;
  /* Swap / Match state (swapping.h, matching.h) */
  int *map, *dual, *dual_n, *matched;
  signed char *visited, *degree;
  int swap_rule;      /* ORC_SWAP_*: the reference's matching, or an emulation */
  int swap_strict_map; /* flips re-activate only rows of the current level */
  int swap_nt;        /* rows of the current level */
  int *hs_mate, *hs_choice;
  uint64_t* hs_prop;
  /* Refine hashtable (hashtable.h) as an open-addressing map (min,max)->id */
  int64_t* hkey;
  int* hval;
  size_t hcap, hcount;
  double complexity;
  int counters[4];
  int err;
  ivec log;
};

/* ------------------------------------------------------------------------ */
/* numerics: numeric.cpp                                                     */
/* ------------------------------------------------------------------------ */
static double dmin(double a, double b) { return (b < a) ? b : a; } /* std::min */
static double dmax(double a, double b) { return (a < b) ? b : a; } /* std::max */

/* numeric::eigenDecompose, numeric.cpp:25-95 */
static void eigen(const double* mat, double* val, double* vec1, double* vec2) {
  if (mat[1] * mat[2] < EPS) {
    val[0] = mat[3];
    val[1] = mat[0];
    vec1[0] = 0; vec2[0] = 1;
    vec1[1] = 1; vec2[1] = 0;
    return;
  }
  double trace = mat[0] + mat[3];
  double det = mat[0] * mat[3] - mat[1] * mat[2];
  double term = trace * 0.5;
  double sqrt_delta = sqrt(term * term - det);
  val[0] = term - sqrt_delta;
  val[1] = term + sqrt_delta;
  if (!isnormal(val[0]) || !isnormal(val[1])) val[0] = val[1];
  term = sqrt(dmax(0.25 * trn_pow(mat[0] - mat[3], 2) + mat[1] * mat[2], 0.));
  if (mat[0] - mat[3] >= 0) {
    vec1[0] = +0.5 * (mat[0] - mat[3]) - term;
    vec1[1] = mat[1];
    vec2[0] = mat[2];
    vec2[1] = -0.5 * (mat[0] - mat[3]) + term;
  } else {
    vec1[0] = mat[2];
    vec1[1] = +0.5 * (mat[0] - mat[3]) + term;
    vec2[0] = -0.5 * (mat[0] - mat[3]) - term;
    vec2[1] = mat[1];
  }
  double n0 = sqrt(vec1[0] * vec1[0] + vec1[1] * vec1[1]);
  double n1 = sqrt(vec2[0] * vec2[0] + vec2[1] * vec2[1]);
  for (int i = 0; i < 2; ++i) {
    vec1[i] /= n0;
    vec2[i] /= n1;
  }
}

/* numeric::interpolateTensor, numeric.cpp:98-248 (log-Euclidean mean) */
static void interpolate(const double* matrix, double* result, int nb) {
  double copy[4], cache[4], val[2], vec[4];
  double log_mat[4] = {0, 0, 0, 0};
  for (int i = 0; i < nb; ++i) {
    int j = 3 * i;
    copy[0] = matrix[j];
    copy[1] = matrix[j + 1];
    copy[2] = matrix[j + 1];
    copy[3] = matrix[j + 2];
    eigen(copy, val, vec, vec + 2);
    val[0] = trn_log(val[0]);
    val[1] = trn_log(val[1]);
    copy[0] = val[0] * vec[0];
    copy[1] = val[0] * vec[2];
    copy[2] = val[1] * vec[1];
    copy[3] = val[1] * vec[3];
    cache[0] = vec[0] * copy[0] + vec[1] * copy[2];
    cache[1] = vec[0] * copy[1] + vec[1] * copy[3];
    cache[2] = vec[2] * copy[0] + vec[3] * copy[2];
    cache[3] = vec[2] * copy[1] + vec[3] * copy[3];
    for (int k = 0; k < 4; ++k) log_mat[k] += cache[k];
  }
  for (int i = 0; i < 4; ++i) log_mat[i] /= nb;
  eigen(log_mat, val, vec, vec + 2);
  val[0] = trn_exp(val[0]);
  val[1] = trn_exp(val[1]);
  copy[0] = val[0] * vec[0];
  copy[1] = val[0] * vec[2];
  copy[2] = val[1] * vec[1];
  copy[3] = val[1] * vec[3];
  cache[0] = vec[0] * copy[0] + vec[1] * copy[2];
  cache[1] = vec[0] * copy[1] + vec[1] * copy[3];
  cache[3] = vec[2] * copy[1] + vec[3] * copy[3];
  result[0] = cache[0];
  result[1] = cache[1];
  result[2] = cache[3];
}

/* numeric::computeQuality, numeric.cpp:251-306 */
static double quality(const double* pa, const double* pb, const double* pc,
                      const double* ta, const double* tb, const double* tc) {
  double coef[6], vec[6], jacob[3], matrix[9];
  double perim = 0;
  memcpy(matrix, ta, sizeof(double) * 3);
  memcpy(matrix + 3, tb, sizeof(double) * 3);
  memcpy(matrix + 6, tc, sizeof(double) * 3);
  interpolate(matrix, jacob, 3);
  double det = jacob[0] * jacob[2] - jacob[1] * jacob[1];
  coef[0] = pb[0] - pa[0];
  coef[1] = pb[1] - pa[1];
  coef[2] = pc[0] - pb[0];
  coef[3] = pc[1] - pb[1];
  coef[4] = pa[0] - pc[0];
  coef[5] = pa[1] - pc[1];
  for (int k = 0; k < 3; ++k) {
    int i = k * 2, j = i + 1;
    vec[i] = jacob[0] * coef[i] + jacob[1] * coef[j];
    vec[j] = jacob[1] * coef[i] + jacob[2] * coef[j];
    perim += sqrt(coef[i] * vec[i] + coef[j] * vec[j]);
  }
  coef[0] = pb[0] - pa[0];
  coef[1] = pc[0] - pa[0];
  coef[2] = pb[1] - pa[1];
  coef[3] = pc[1] - pa[1];
  double area = 0.5 * fabs(coef[0] * coef[3] - coef[1] * coef[2]);
  double mean = dmin(perim / 3, 3 / perim);
  double norm = 12 * sqrt(3.0) * trn_pow(mean * (2. - mean), 3);
  return area * norm * sqrt(det) / trn_pow(perim, 2);
}

/* numeric::approxRiemannDist (one tensor), numeric.cpp:450-461 */
static double dist1(const double* pa, const double* pb, const double* t) {
  double u[2], v[2];
  u[0] = pb[0] - pa[0];
  u[1] = pb[1] - pa[1];
  v[0] = t[0] * u[0] + t[1] * u[1];
  v[1] = t[1] * u[0] + t[2] * u[1];
  return sqrt(u[0] * v[0] + u[1] * v[1]);
}

/* numeric::approxRiemannDist (two tensors), numeric.cpp:469-497 */
static double dist2(const double* pa, const double* pb, const double* ta,
                    const double* tb) {
  double length[2], vector[2], matrix[4];
  vector[0] = pb[0] - pa[0];
  vector[1] = pb[1] - pa[1];
  matrix[0] = ta[0] * vector[0] + ta[1] * vector[1];
  matrix[1] = ta[1] * vector[0] + ta[2] * vector[1];
  matrix[2] = tb[0] * vector[0] + tb[1] * vector[1];
  matrix[3] = tb[1] * vector[0] + tb[2] * vector[1];
  length[0] = sqrt(vector[0] * matrix[0] + vector[1] * matrix[1]);
  length[1] = sqrt(vector[0] * matrix[2] + vector[1] * matrix[3]);
  if (fabs(length[0] - length[1]) < EPS) return length[0];
  double lmin = dmin(length[0], length[1]);
  double lmax = dmax(length[0], length[1]);
  double ratio = lmax / lmin;
  return lmax * (ratio - 1) / (ratio * trn_log(ratio));
}

/* numeric::computeSteinerPoint, numeric.cpp:387-445 */
static void steiner(const double* pa, const double* pb, const double* ta,
                    const double* tb, double* rp, double* rt) {
  double length[2], metric[6];
  double coef = 1;
  length[0] = dist1(pa, pb, ta);
  length[1] = dist1(pa, pb, tb);
  double weight = (fabs(length[0] - length[1]) < EPS
    ? 0.5
    : (sqrt(coef) * sqrt(length[0] * length[1]) - length[1]) / (coef * length[0] - length[1]));
  rp[0] = (1 - weight) * pa[0] + (weight * pb[0]);
  rp[1] = (1 - weight) * pa[1] + (weight * pb[1]);
  memcpy(metric, ta, sizeof(double) * 3);
  memcpy(metric + 3, tb, sizeof(double) * 3);
  interpolate(metric, rt, 2);
}

/* ------------------------------------------------------------------------ */
/* mesh: mesh.cpp                                                            */
/* ------------------------------------------------------------------------ */
static const int* E(const orc_mesh* m, int t) { return m->elems + (size_t) t * 3; }
static const double* P(const orc_mesh* m, int v) { return m->points + (size_t) v * 2; }
static double* Pw(orc_mesh* m, int v) { return m->points + (size_t) v * 2; }
static double* T(orc_mesh* m, int v) { return m->tensor + (size_t) v * 3; }
static int* S(orc_mesh* m, int v) { return m->stenc + (size_t) v * m->bucket; }
static int* VC(orc_mesh* m, int v) { return m->vicin + (size_t) v * m->vstride; }

/* Mesh::computeLength, mesh.cpp:615-623 */
static double length(orc_mesh* m, int i, int j) {
  return dist2(P(m, i), P(m, j), T(m, i), T(m, j));
}

/* Mesh::computeQuality(const int*), mesh.cpp:626-639 */
static double quality_of(orc_mesh* m, const int* t) {
  return quality(P(m, t[0]), P(m, t[1]), P(m, t[2]), T(m, t[0]), T(m, t[1]), T(m, t[2]));
}

/* Mesh::isCounterclockwise, mesh.cpp:700-713 */
static int ccw(orc_mesh* m, const int* e) {
  const double *a = P(m, e[0]), *b = P(m, e[1]), *c = P(m, e[2]);
  double coef[4];
  coef[0] = b[0] - a[0];
  coef[1] = c[0] - a[0];
  coef[2] = b[1] - a[1];
  coef[3] = c[1] - a[1];
  return 0.5 * (coef[0] * coef[3] - coef[1] * coef[2]) > EPS;
}

static void isort(int* a, int n) {
  for (int i = 1; i < n; ++i) {
    int x = a[i], j = i - 1;
    while (j >= 0 && a[j] > x) { a[j + 1] = a[j]; --j; }
    a[j + 1] = x;
  }
}

static int iunique(int* a, int n) {
  if (n == 0) return 0;
  int k = 1;
  for (int i = 1; i < n; ++i)
    if (a[i] != a[k - 1]) a[k++] = a[i];
  return k;
}

/* Mesh::updateStencil, mesh.cpp:468-494 (append at the fetch-add slot) */
static void stenc_append(orc_mesh* m, int v, int t) {
  int k = m->deg[v]++;
  if (k >= m->bucket) { m->err = ORC_ERR_CAPACITY; m->deg[v]--; return; }
  S(m, v)[k] = t;
}

/* Mesh::fixTagged body for one vertex, mesh.cpp:728-757 */
static void fix_vertex(orc_mesh* m, int i) {
  int* s = S(m, i);
  int tmp[1024];
  int k = 0;
  for (int a = 0; a < m->deg[i]; ++a) {
    const int* n = E(m, s[a]);
    if (i == n[0] || i == n[1] || i == n[2]) tmp[k++] = s[a];
  }
  isort(tmp, k);
  k = iunique(tmp, k);
  for (int a = 0; a < k; ++a) s[a] = tmp[a];
  for (int a = k; a < m->bucket; ++a) s[a] = -1;
  m->deg[i] = k;
}

/* Mesh::fixTagged, mesh.cpp:716-760 */
static void fix_tagged(orc_mesh* m) {
  for (int i = 0; i < m->nb_nodes; ++i)
    if (m->fixes[i]) {
      m->fixes[i] = 0;
      fix_vertex(m, i);
    }
}

/* Mesh::fixAll, mesh.cpp:763-770 */
static void fix_all(orc_mesh* m) {
  for (int i = 0; i < m->nb_nodes; ++i) m->fixes[i] = (char) (m->alive[i] ? 1 : 0);
  fix_tagged(m);
}

/* vertex adjacency of i from its stencil (mesh.cpp:306-327) */
static void build_vicin(orc_mesh* m, int i) {
  int tmp[2048];
  int k = 0;
  const int* s = S(m, i);
  if (m->alive[i]) {
    for (int a = 0; a < m->deg[i]; ++a) {
      const int* n = E(m, s[a]);
      if (i == n[0]) { tmp[k++] = n[1]; tmp[k++] = n[2]; }
      else if (i == n[1]) { tmp[k++] = n[2]; tmp[k++] = n[0]; }
      else if (i == n[2]) { tmp[k++] = n[0]; tmp[k++] = n[1]; }
    }
  }
  /* a collapsed vertex: its cleared stencil names no element that still
   * holds it, so the rebuilt adjacency is empty */
  isort(tmp, k);
  k = iunique(tmp, k);
  if (k > m->vstride) { m->err = ORC_ERR_CAPACITY; k = m->vstride; }
  memcpy(VC(m, i), tmp, sizeof(int) * (size_t) k);
  m->vdeg[i] = k;
}

/* Mesh::extractPrimalGraph, mesh.cpp:297-330 */
static void extract_primal(orc_mesh* m) {
  for (int i = 0; i < m->nb_nodes; ++i)
    if (m->activ[i]) build_vicin(m, i);
}

/* Mesh::getElemNeigh, mesh.cpp:437-453 */
static int elem_neigh(orc_mesh* m, int id, int i, int j) {
  const int* s = S(m, i);
  for (int a = 0; a < m->deg[i]; ++a) {
    int t = s[a];
    if (t < 0) break;
    if (t != id) {
      const int* n = E(m, t);
      if ((n[0] == j && n[1] == i) || (n[1] == j && n[2] == i) || (n[2] == j && n[0] == i))
        return t;
    }
  }
  return -1;
}

/* ------------------------------------------------------------------------ */
orc_mesh* orc_create(int capa_node, int capa_elem, int bucket) {
  orc_mesh* m = (orc_mesh*) calloc(1, sizeof(orc_mesh));
  m->capa_node = capa_node;
  m->capa_elem = capa_elem;
  m->bucket = bucket;
  m->vstride = bucket;
  size_t cn = (size_t) capa_node, ce = (size_t) capa_elem;
  m->points = (double*) calloc(cn * 2, sizeof(double));
  m->tensor = (double*) calloc(cn * 3, sizeof(double));
  m->solut = (double*) calloc(cn, sizeof(double));
  m->gradient = (double*) calloc(cn * 2, sizeof(double));
  m->qualit = (double*) calloc(ce, sizeof(double));
  m->elems = (int*) malloc(ce * 3 * sizeof(int));
  m->stenc = (int*) malloc(cn * (size_t) bucket * sizeof(int));
  m->deg = (int*) calloc(cn, sizeof(int));
  m->vicin = (int*) malloc(cn * (size_t) m->vstride * sizeof(int));
  m->vdeg = (int*) calloc(cn, sizeof(int));
  m->alive = (uint8_t*) calloc(cn, 1);
  m->tags = (uint8_t*) calloc(cn, 1);
  m->activ = (signed char*) calloc(ce > cn ? ce : cn, 1);
  m->fixes = (char*) calloc(cn, 1);
  for (int i = 0; i < MAX_PART; ++i) m->subset[i] = (int*) calloc(cn, sizeof(int));
  m->map = (int*) malloc(ce * sizeof(int));
  m->dual = (int*) malloc(ce * 4 * sizeof(int));
  m->dual_n = (int*) calloc(ce, sizeof(int));
  m->matched = (int*) malloc(ce * sizeof(int));
  m->visited = (signed char*) calloc(ce, 1);
  m->degree = (signed char*) calloc(ce, 1);
  m->hs_mate = (int*) malloc(ce * sizeof(int));
  m->hs_choice = (int*) malloc(ce * sizeof(int));
  m->hs_prop = (uint64_t*) calloc(ce, sizeof(uint64_t));
  if (!m->points || !m->tensor || !m->elems || !m->stenc || !m->vicin || !m->dual) {
    orc_destroy(m);
    return NULL;
  }
  for (size_t i = 0; i < ce * 3; ++i) m->elems[i] = -1;
  for (size_t i = 0; i < cn * (size_t) bucket; ++i) m->stenc[i] = -1;
  for (size_t i = 0; i < ce; ++i) m->map[i] = -1;
  for (size_t i = 0; i < cn; ++i) m->alive[i] = 1;  /* stencil vectors start non-empty */
  return m;
}

void orc_destroy(orc_mesh* m) {
  if (!m) return;
  free(m->points); free(m->tensor); free(m->solut); free(m->gradient); free(m->qualit);
  free(m->elems); free(m->stenc); free(m->deg); free(m->vicin); free(m->vdeg);
  free(m->alive); free(m->tags); free(m->activ); free(m->fixes);
  for (int i = 0; i < MAX_PART; ++i) free(m->subset[i]);
  free(m->map); free(m->dual); free(m->dual_n); free(m->matched);
  free(m->visited); free(m->degree); free(m->hs_mate); free(m->hs_choice); free(m->hs_prop);
  free(m->hkey); free(m->hval); free(m->log.a);
  free(m);
}

/* Mesh::load (io.cpp:53-161) from arrays, then Mesh::rebuildTopology (mesh.cpp:191-249) */
int orc_load(orc_mesh* m, int nb_nodes, int nb_elems, const double* points,
             const int* tris, const uint8_t* tags, const double* solut) {
  if (nb_nodes > m->capa_node || nb_elems > m->capa_elem) return ORC_ERR_CAPACITY;
  m->nb_nodes = nb_nodes;
  m->nb_elems = nb_elems;
  memcpy(m->points, points, sizeof(double) * 2 * (size_t) nb_nodes);
  memcpy(m->elems, tris, sizeof(int) * 3 * (size_t) nb_elems);
  memcpy(m->tags, tags, (size_t) nb_nodes);
  memcpy(m->solut, solut, sizeof(double) * (size_t) nb_nodes);
  for (int i = 0; i < m->capa_node; ++i) m->deg[i] = 0;
  m->err = 0;
  for (int i = 0; i < nb_elems; ++i) {
    const int* n = E(m, i);
    if (n[0] < 0) continue;
    stenc_append(m, n[0], i);
    stenc_append(m, n[1], i);
    stenc_append(m, n[2], i);
  }
  for (int i = 0; i < nb_nodes; ++i) {
    build_vicin(m, i);
    isort(S(m, i), m->deg[i]);
  }
  return m->err;
}

/* ------------------------------------------------------------------------ */
/* metric: metric.cpp, hessian.cpp                                           */
/* ------------------------------------------------------------------------ */
/* Mesh::getVicinity(i, 2), mesh.cpp:390-434: elements incident to i or to a
 * 1-ring neighbour, ascending */
static int patch_elems(orc_mesh* m, int i, int* out) {
  int k = 0;
  for (int a = 0; a < m->deg[i]; ++a) out[k++] = S(m, i)[a];
  for (int b = 0; b < m->vdeg[i]; ++b) {
    int v = VC(m, i)[b];
    for (int a = 0; a < m->deg[v]; ++a) out[k++] = S(m, v)[a];
  }
  isort(out, k);
  return iunique(out, k);
}

/* Metrics::computeGradient, hessian.cpp:24-83 */
static void gradient(orc_mesh* m, int index, const int* patch, int size) {
  double total_area = 0., point[6], coef[4], deriv[6];
  double area[1024], grad[2048];
  for (int i = 0; i < size * 2; ++i) grad[i] = 0;
  for (int i = 0; i < size; ++i) {
    const int* v = E(m, patch[i]);
    for (int q = 0; q < 3; ++q) {
      point[2 * q] = P(m, v[q])[0];
      point[2 * q + 1] = P(m, v[q])[1];
    }
    coef[0] = point[2] - point[0];
    coef[1] = point[4] - point[0];
    coef[2] = point[3] - point[1];
    coef[3] = point[5] - point[1];
    area[i] = 0.5 * (coef[0] * coef[3] - coef[1] * coef[2]);
    double norm = 2 / area[i];
    total_area += area[i];
    deriv[0] = norm * (point[3] - point[5]);
    deriv[1] = norm * (point[4] - point[2]);
    deriv[2] = norm * (point[5] - point[1]);
    deriv[3] = norm * (point[0] - point[4]);
    deriv[4] = norm * (point[1] - point[3]);
    deriv[5] = norm * (point[2] - point[0]);
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 2; ++k)
        grad[i * 2 + k] += m->solut[v[j]] * deriv[j * 2 + k];
  }
  int k = index * 2;
  m->gradient[k] = m->gradient[k + 1] = 0.;
  for (int i = 0; i < size; ++i)
    for (int j = 0; j < 2; ++j)
      m->gradient[k + j] += (area[i] * grad[i * 2 + j]);
  m->gradient[k] /= total_area;
  m->gradient[k + 1] /= total_area;
}

/* Metrics::computeHessian, hessian.cpp:86-153 */
static void hessian(orc_mesh* m, int index, const int* patch, int size) {
  double total_area = 0, point[6], coef[4], deriv[6];
  double hess[4] = {0, 0, 0, 0};
  double area[1024], delta[4096];
  for (int i = 0; i < size * 4; ++i) delta[i] = 0;
  const double* g = m->gradient;
  for (int i = 0; i < size; ++i) {
    const int* v = E(m, patch[i]);
    for (int q = 0; q < 3; ++q) {
      point[2 * q] = P(m, v[q])[0];
      point[2 * q + 1] = P(m, v[q])[1];
    }
    coef[0] = point[2] - point[0];
    coef[1] = point[4] - point[0];
    coef[2] = point[3] - point[1];
    coef[3] = point[5] - point[1];
    area[i] = 0.5 * (coef[0] * coef[3] - coef[1] * coef[2]);
    double norm = 2 / area[i];
    total_area += area[i];
    deriv[0] = norm * (point[3] - point[5]);
    deriv[1] = norm * (point[4] - point[2]);
    deriv[2] = norm * (point[5] - point[1]);
    deriv[3] = norm * (point[0] - point[4]);
    deriv[4] = norm * (point[1] - point[3]);
    deriv[5] = norm * (point[2] - point[0]);
    for (int j = 0; j < 3; ++j) {
      delta[i * 4] += (g[v[j] * 2] * deriv[j * 2]);
      delta[i * 4 + 1] += (g[v[j] * 2] * deriv[j * 2 + 1]);
      delta[i * 4 + 2] += (g[v[j] * 2 + 1] * deriv[j * 2]);
      delta[i * 4 + 3] += (g[v[j] * 2 + 1] * deriv[j * 2 + 1]);
    }
  }
  for (int i = 0; i < size; ++i)
    for (int j = 0; j < 4; ++j) hess[j] += area[i] * delta[i * 4 + j];
  for (int j = 0; j < 4; ++j) hess[j] /= total_area;
  double* t = T(m, index);
  t[0] = hess[0];
  t[1] = 0.5 * (hess[1] + hess[2]);
  t[2] = hess[3];
}

/* rebuild a tensor from eigen pairs: metric.cpp:134-148 / 222-236 */
static void recompose(double* t, const double* val, const double* vec) {
  double mm[4], h[4];
  mm[0] = val[0] * vec[0];
  mm[1] = val[0] * vec[2];
  mm[2] = val[1] * vec[1];
  mm[3] = val[1] * vec[3];
  h[0] = vec[0] * mm[0] + vec[1] * mm[2];
  h[1] = vec[0] * mm[1] + vec[1] * mm[3];
  h[3] = vec[2] * mm[1] + vec[3] * mm[3];
  t[0] = h[0];
  t[1] = h[1];
  t[2] = h[3];
}

/* Metrics::run, metric.cpp:59-70 (+ ctor 24-53) */
int orc_metric(orc_mesh* m, double target_factor, int norm, double h_min, double h_max) {
  int target = (int) floor(m->nb_nodes * target_factor);
  double scale_exp = norm ? -1. / (2 * norm + 2) : 0.5;
  double eig_min = 1 / trn_pow(h_min, 2);
  double eig_max = 1 / trn_pow(h_max, 2);
  int patch[4096];
  /* recoverHessianField, metric.cpp:80-97 */
  for (int i = 0; i < m->nb_nodes; ++i) {
    int n = patch_elems(m, i, patch);
    gradient(m, i, patch, n);
  }
  for (int i = 0; i < m->nb_nodes; ++i) {
    int n = patch_elems(m, i, patch);
    hessian(m, i, patch, n);
  }
  /* normalizeLocally, metric.cpp:100-150 */
  for (int i = 0; i < m->nb_nodes; ++i) {
    double* t = T(m, i);
    double mm[4], val[2] = {0, 0}, vec[4] = {0, 0, 0, 0};
    mm[0] = t[0]; mm[1] = t[1]; mm[2] = mm[1]; mm[3] = t[2];
    eigen(mm, val, vec, vec + 2);
    val[0] = dmax(fabs(val[0]), EPS);
    val[1] = dmax(fabs(val[1]), EPS);
    double det = val[0] * val[1];
    double scale_loc = trn_pow(det, scale_exp);
    val[0] *= scale_loc;
    val[1] *= scale_loc;
    recompose(t, val, vec);
  }
  /* computeComplexity, metric.cpp:153-185: sequential sum in element order */
  double phi = 0.;
  for (int i = 0; i < m->nb_elems; ++i) {
    const int* v = E(m, i);
    const double *p0 = P(m, v[0]), *p1 = P(m, v[1]), *p2 = P(m, v[2]);
    double s[4];
    s[0] = p1[0] - p0[0];
    s[1] = p2[0] - p0[0];
    s[2] = p1[1] - p0[1];
    s[3] = p2[1] - p0[1];
    double area = 0.5 * (s[0] * s[3] - s[1] * s[2]);
    double rho = 0.;
    for (int j = 0; j < 3; ++j) {
      const double* t = T(m, v[j]);
      double det = t[0] * t[2] - trn_pow(t[1], 2);
      rho += sqrt(det);
    }
    rho /= 3;
    phi += rho * area;
  }
  m->complexity = 0 + phi;
  /* normalizeGlobally, metric.cpp:188-238 */
  double fact = target / m->complexity;
  for (int i = 0; i < m->nb_nodes; ++i) {
    double* t = T(m, i);
    double mm[4], val[2], vec[4];
    mm[0] = t[0]; mm[1] = t[1]; mm[2] = mm[1]; mm[3] = t[2];
    eigen(mm, val, vec, vec + 2);
    val[0] *= fact;
    val[1] *= fact;
    for (int j = 0; j < 2; ++j) {
      val[j] = dmin(val[j], eig_min);
      val[j] = dmax(val[j], eig_max);
    }
    recompose(t, val, vec);
  }
  m->counters[0] = m->counters[1] = m->nb_nodes;
  m->counters[2] = m->counters[3] = 0;
  return m->err;
}

/* ------------------------------------------------------------------------ */
/* refinement: refinement.cpp (+ hashtable.h)                               */
/* ------------------------------------------------------------------------ */
static uint64_t hmix(int64_t k) {
  uint64_t x = (uint64_t) k * 0x9e3779b97f4a7c15ULL;
  return x ^ (x >> 29);
}

static void h_reset(orc_mesh* m) {
  if (m->hcap < 1024) {
    free(m->hkey); free(m->hval);
    m->hcap = 1024;
    m->hkey = (int64_t*) malloc(sizeof(int64_t) * m->hcap);
    m->hval = (int*) malloc(sizeof(int) * m->hcap);
  }
  for (size_t i = 0; i < m->hcap; ++i) m->hkey[i] = -1;
  m->hcount = 0;
}

static void h_insert(orc_mesh* m, int v, int w, int id);

static void h_grow(orc_mesh* m) {
  size_t oc = m->hcap;
  int64_t* ok = m->hkey;
  int* ov = m->hval;
  m->hcap = oc * 2;
  m->hkey = (int64_t*) malloc(sizeof(int64_t) * m->hcap);
  m->hval = (int*) malloc(sizeof(int) * m->hcap);
  for (size_t i = 0; i < m->hcap; ++i) m->hkey[i] = -1;
  m->hcount = 0;
  for (size_t i = 0; i < oc; ++i)
    if (ok[i] >= 0) h_insert(m, (int) (ok[i] >> 32), (int) (ok[i] & 0xffffffff), ov[i]);
  free(ok);
  free(ov);
}

/* Hashtable::push(min, {max, id}), hashtable.impl.h:73-81; the first entry
 * for a pair is the one getValue finds (hashtable.impl.h:85-97) */
static void h_insert(orc_mesh* m, int v, int w, int id) {
  if ((m->hcount + 1) * 2 > m->hcap) h_grow(m);
  int64_t key = ((int64_t) v << 32) | (uint32_t) w;
  size_t i = hmix(key) & (m->hcap - 1);
  while (m->hkey[i] >= 0) {
    if (m->hkey[i] == key) return;
    i = (i + 1) & (m->hcap - 1);
  }
  m->hkey[i] = key;
  m->hval[i] = id;
  m->hcount++;
}

/* Hashtable::getValue, hashtable.impl.h:85-97 */
static int h_get(const orc_mesh* m, int v1, int v2) {
  int v = v1 < v2 ? v1 : v2, w = v1 < v2 ? v2 : v1;
  int64_t key = ((int64_t) v << 32) | (uint32_t) w;
  size_t i = hmix(key) & (m->hcap - 1);
  while (m->hkey[i] >= 0) {
    if (m->hkey[i] == key) return m->hval[i];
    i = (i + 1) & (m->hcap - 1);
  }
  return -1;
}

static void set_elem(orc_mesh* m, int id, int a, int b, int c) {
  int* e = m->elems + (size_t) id * 3;
  e[0] = a; e[1] = b; e[2] = c;
}

/* Refine::cutElem, refinement.cpp:55-184 */
static void cut_elem(orc_mesh* m, int id, int* offset, const char* pattern) {
  const int* n0 = E(m, id);
  int n[3] = {n0[0], n0[1], n0[2]};
  const int s[3] = {h_get(m, n[1], n[2]), h_get(m, n[2], n[0]), h_get(m, n[0], n[1])};
  if (pattern[id] == 1) {
    const int t[2] = {id, *offset};
    for (int i = 0; i < 3; ++i) {
      if (s[i] > -1) {
        int j = (i + 1) % 3, k = (i + 2) % 3;
        stenc_append(m, s[i], t[0]);
        stenc_append(m, s[i], t[1]);
        stenc_append(m, n[i], t[1]);
        stenc_append(m, n[k], t[1]);
        set_elem(m, t[0], n[i], n[j], s[i]);
        set_elem(m, t[1], n[i], s[i], n[k]);
        m->activ[t[0]] = m->activ[t[1]] = 1;
        break;
      }
    }
  } else if (pattern[id] == 2) {
    const int t[3] = {id, *offset, *offset + 1};
    for (int i = 0; i < 3; ++i) {
      if (s[i] < 0) {
        int j = (i + 1) % 3, k = (i + 2) % 3;
        double diag[2];
        diag[0] = length(m, n[j], s[j]);
        diag[1] = length(m, n[k], s[k]);
        int v = (diag[0] < diag[1] ? j : k);
        int w = (v == j ? k : j);
        stenc_append(m, s[v], t[0]);
        stenc_append(m, s[v], t[1]);
        stenc_append(m, s[v], t[2]);
        stenc_append(m, s[w], t[0]);
        stenc_append(m, s[w], t[2]);
        stenc_append(m, n[v], t[1]);
        stenc_append(m, n[v], t[2]);
        stenc_append(m, n[w], t[1]);
        set_elem(m, t[0], n[i], s[k], s[j]);
        set_elem(m, t[1], n[j], n[k], s[v]);
        set_elem(m, t[2], s[j], s[k], n[v]);
        m->activ[t[0]] = m->activ[t[1]] = m->activ[t[2]] = 1;
        break;
      }
    }
  } else {
    const int t[4] = {id, *offset, *offset + 1, *offset + 2};
    stenc_append(m, s[0], t[1]); stenc_append(m, s[0], t[2]); stenc_append(m, s[0], t[3]);
    stenc_append(m, s[1], t[0]); stenc_append(m, s[1], t[2]); stenc_append(m, s[1], t[3]);
    stenc_append(m, s[2], t[0]); stenc_append(m, s[2], t[1]); stenc_append(m, s[2], t[3]);
    stenc_append(m, n[1], t[1]);
    stenc_append(m, n[2], t[2]);
    set_elem(m, t[0], n[0], s[2], s[1]);
    set_elem(m, t[1], n[1], s[0], s[2]);
    set_elem(m, t[2], n[2], s[1], s[0]);
    set_elem(m, t[3], s[0], s[1], s[2]);
    m->activ[t[0]] = m->activ[t[1]] = m->activ[t[2]] = m->activ[t[3]] = 1;
  }
  *offset += pattern[id];
}

/* Refine::run, refinement.cpp:445-493 */
int orc_refine(orc_mesh* m, int depth) {
  m->err = 0;
  int eval_total = 0, task_total = 0, levels = 0;
  /* preProcess, refinement.cpp:187-213 */
  for (int i = 0; i < m->nb_elems; ++i) m->activ[i] = (signed char) (E(m, i)[0] > -1 ? 1 : 0);
  h_reset(m);
  char* pattern = (char*) calloc((size_t) m->capa_elem, 1);
  ivec edges = {0}, tasks = {0};
  int level = 0;
  do {
    /* filterElems, refinement.cpp:216-264 */
    edges.n = tasks.n = 0;
    int eval = 0, adds = 0;
    for (int i = 0; i < m->nb_elems; ++i) {
      pattern[i] = 0;
      if (m->activ[i]) {
        const int* n = E(m, i);
        double len[3];
        len[0] = length(m, n[0], n[1]);
        len[1] = length(m, n[1], n[2]);
        len[2] = length(m, n[2], n[0]);
        for (int j = 0; j < 3; ++j) {
          int k = (j + 1) % 3;
          if (len[j] > L_MAX) {
            ++pattern[i];
            int opp = elem_neigh(m, i, n[j], n[k]);
            if (n[j] < n[k] || opp < 0) {
              iv_push(&edges, n[j]);
              iv_push(&edges, n[k]);
              iv_push(&edges, opp);
            }
          }
        }
        if (pattern[i]) {
          adds += pattern[i];
          iv_push(&tasks, i);
        }
        eval++;
      }
    }
    eval_total += eval;
    task_total += tasks.n;
    int nb_split = edges.n / 3;
    if (!tasks.n) break;
    levels++;
    if (m->nb_nodes + nb_split > m->capa_node || m->nb_elems + adds > m->capa_elem) {
      m->err = ORC_ERR_CAPACITY;
      break;
    }
    /* computeSteinerPoints, refinement.cpp:267-297 */
    for (int i = 0; i < nb_split; ++i) {
      int id = m->nb_nodes + i;
      int v1 = edges.a[i * 3], v2 = edges.a[i * 3 + 1], opp = edges.a[i * 3 + 2];
      steiner(P(m, v1), P(m, v2), T(m, v1), T(m, v2), Pw(m, id), T(m, id));
      h_insert(m, v1 < v2 ? v1 : v2, v1 < v2 ? v2 : v1, id);
      if (opp < 0) m->tags[id] = TAG_BOUND;
    }
    /* processElems, refinement.cpp:300-318 */
    int offset = m->nb_elems;
    m->nb_nodes += nb_split;
    m->nb_elems += adds;
    for (int i = 0; i < tasks.n; ++i) cut_elem(m, tasks.a[i], &offset, pattern);
  } while (++level < depth);
  fix_all(m);
  free(pattern);
  free(edges.a);
  free(tasks.a);
  m->counters[0] = eval_total;
  m->counters[1] = task_total;
  m->counters[2] = 0;
  m->counters[3] = levels;
  return m->err;
}

/* ------------------------------------------------------------------------ */
/* graph heuristics: partition.cpp                                           */
/* ------------------------------------------------------------------------ */
/* Partit::reset, partition.cpp:62-75 */
static void partit_reset(orc_mesh* m) {
  m->nb_parts = 0;
  memset(m->cardin, 0, sizeof m->cardin);
  for (int i = 0; i < 3; ++i) memset(m->subset[i], 0, sizeof(int) * (size_t) m->capa_node);
}

static void log_begin(orc_mesh* m, int tag, int count) {
  iv_push(&m->log, tag);
  iv_push(&m->log, count);
}

/* Partit::extractIndepSet, partition.cpp:200-306; graph row i = [cand[i], vicin(cand[i])] */
static int indep_set(orc_mesh* m, const int* cand, int nb) {
  if (nb == 1) {
    m->subset[0][0] = cand[0];
    m->cardin[0] = 1;
    log_begin(m, ORC_LOG_MIS, 1);
    iv_push(&m->log, cand[0]);
    return 1;
  }
  partit_reset(m);
  int* color = m->subset[2];
  int forbidden[MAX_PART];
  for (int c = 0; c < MAX_PART; ++c) forbidden[c] = INT_MAX;
  for (int i = 0; i < nb; ++i) {
    int v = cand[i];
    for (int b = 0; b < m->vdeg[v]; ++b) forbidden[color[VC(m, v)[b]]] = v;
    for (int c = 1; c < MAX_PART; ++c)
      if (forbidden[c] != v) { color[v] = c; break; }
  }
  ivec lists[2] = {{0}, {0}};
  for (int i = 0; i < nb; ++i) {
    int v = cand[i];
    if (color[v] == 1)
      for (int b = 0; b < m->vdeg[v]; ++b) {
        int w = VC(m, v)[b];
        if (v < w && color[w] == 1) { iv_push(&lists[0], i); break; }
      }
  }
  int k = 0, guard = 0;
  while (lists[k].n && guard++ < LOOP_CAP) {
    for (int a = 0; a < lists[k].n; ++a) {
      int v = cand[lists[k].a[a]];
      for (int b = 0; b < m->vdeg[v]; ++b) forbidden[color[VC(m, v)[b]]] = v;
      for (int c = 1; c < MAX_PART; ++c)
        if (forbidden[c] != v) { color[v] = c; break; }
    }
    lists[k ^ 1].n = 0;
    for (int a = 0; a < lists[k].n; ++a) {
      int j = lists[k].a[a], v = cand[j];
      if (color[v] == 1)
        for (int b = 0; b < m->vdeg[v]; ++b) {
          int w = VC(m, v)[b];
          if (v < w && color[w] == 1) { iv_push(&lists[k ^ 1], j); break; }
        }
    }
    k ^= 1;
  }
  if (guard >= LOOP_CAP) m->err = ORC_ERR_NO_PROGRESS;
  int count = 0;
  for (int i = 0; i < nb; ++i)
    if (color[cand[i]] == 1) m->subset[0][count++] = cand[i];
  m->cardin[0] = count;
  log_begin(m, ORC_LOG_MIS, count);
  for (int i = 0; i < count; ++i) iv_push(&m->log, m->subset[0][i]);
  free(lists[0].a);
  free(lists[1].a);
  return count;
}

/* Partit::extractColoring, partition.cpp:79-197, graph = vicin of every vertex */
static void coloring(orc_mesh* m) {
  partit_reset(m);
  int forbidden[MAX_PART];
  for (int c = 0; c < MAX_PART; ++c) forbidden[c] = INT_MAX;
  int* color = m->subset[2];
  ivec conflicts = {0}, lists[2] = {{0}, {0}};
  for (int i = 0; i < m->nb_nodes; ++i) {
    if (!m->vdeg[i]) continue;
    for (int b = 0; b < m->vdeg[i]; ++b) forbidden[color[VC(m, i)[b]]] = i;
    for (int c = 1; c < MAX_PART; ++c)
      if (forbidden[c] != i) { color[i] = c; break; }
  }
  for (int i = 0; i < m->nb_nodes; ++i)
    for (int b = 0; b < m->vdeg[i]; ++b) {
      int j = VC(m, i)[b];
      if (i < j && color[i] == color[j]) { iv_push(&lists[0], i); break; }
    }
  int k = 0, guard = 0;
  while (lists[k].n && guard++ < LOOP_CAP) {
    for (int a = 0; a < lists[k].n; ++a) {
      int v = lists[k].a[a];
      if (!m->vdeg[v]) continue;
      for (int b = 0; b < m->vdeg[v]; ++b) forbidden[color[VC(m, v)[b]]] = v;
      for (int c = 1; c < MAX_PART; ++c)
        if (forbidden[c] != v) { color[v] = c; break; }
    }
    lists[k ^ 1].n = 0;
    for (int a = 0; a < lists[k].n; ++a) {
      int v = lists[k].a[a];
      for (int b = 0; b < m->vdeg[v]; ++b) {
        int w = VC(m, v)[b];
        if (v < w && color[v] == color[w]) { iv_push(&lists[k ^ 1], v); break; }
      }
    }
    k ^= 1;
  }
  if (guard >= LOOP_CAP) m->err = ORC_ERR_NO_PROGRESS;
  /* post-process: per-color vertex lists in ascending id */
  ivec parts[MAX_PART];
  memset(parts, 0, sizeof parts);
  int nb_col = 0;
  for (int i = 0; i < m->nb_nodes; ++i) {
    int j = color[i];
    if (j) {
      iv_push(&parts[j - 1], i);
      if (j > nb_col) nb_col = j;
    }
  }
  m->nb_parts = nb_col;
  for (int j = 0; j < nb_col; ++j) {
    memcpy(m->subset[j], parts[j].a, sizeof(int) * (size_t) parts[j].n);
    m->cardin[j] = parts[j].n;
  }
  log_begin(m, ORC_LOG_COLORING, nb_col);
  for (int j = 0; j < nb_col; ++j) {
    iv_push(&m->log, parts[j].n);
    for (int a = 0; a < parts[j].n; ++a) iv_push(&m->log, parts[j].a[a]);
  }
  for (int j = 0; j < MAX_PART; ++j) free(parts[j].a);
  free(conflicts.a);
  free(lists[0].a);
  free(lists[1].a);
}

/* ------------------------------------------------------------------------ */
/* coarsening: coarsening.cpp                                                */
/* ------------------------------------------------------------------------ */
/* Coarse::identifyTarget, coarsening.cpp:47-133; returns the target or -1 */
static int identify_target(orc_mesh* m, int source) {
  int bound_source = (m->tags[source] & TAG_BOUND) != 0;
  double lens[1024];
  int cands[1024];
  int nc = 0;
  /* std::multimap<double,int>: ascending length, ties in insertion order */
  for (int b = 0; b < m->vdeg[source]; ++b) {
    int neigh = VC(m, source)[b];
    int bound_destin = (m->tags[neigh] & TAG_BOUND) != 0;
    if (bound_source && !bound_destin) continue;
    double len = length(m, source, neigh);
    if (len < L_MIN) {
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
  int destin = -1, skip = 1, next = 0;
  const int* st = S(m, source);
  int deg = m->deg[source];
  while (skip && next < nc) {
    destin = cands[next++];
    skip = 0;
    int shared = 0;
    int bound_destin = (m->tags[destin] & TAG_BOUND) != 0;
    for (int a = 0; !skip && a < deg; ++a) {
      const int* n = E(m, st[a]);
      if ((source == n[0] && destin == n[1]) || (source == n[1] && destin == n[0]) ||
          (source == n[1] && destin == n[2]) || (source == n[2] && destin == n[1]) ||
          (source == n[2] && destin == n[0]) || (source == n[0] && destin == n[2])) {
        skip = (++shared > 1 && bound_source && bound_destin);
        continue;
      }
      int face[3];
      face[0] = (n[0] == source ? destin : n[0]);
      face[1] = (n[1] == source ? destin : n[1]);
      face[2] = (n[2] == source ? destin : n[2]);
      if (ccw(m, face)) {
        double l0 = length(m, face[0], face[1]);
        double l1 = length(m, face[1], face[2]);
        double l2 = length(m, face[2], face[0]);
        skip = (l0 > L_MAX || l1 > L_MAX || l2 > L_MAX);
        continue;
      }
      skip = 1;
    }
  }
  return skip ? -1 : destin;
}

/* Coarse::collapseEdge, coarsening.cpp:136-254 */
static void collapse_edge(orc_mesh* m, int source, int destin) {
  int* st = S(m, source);
  int deg = m->deg[source];
  int k = 0;
  int trash[2] = {-1, -1}, opp[2] = {-1, -1};
  int limit = (m->tags[source] & TAG_BOUND) ? 1 : 2;
  for (int a = 0; k < limit && a < deg; ++a) {
    const int* n = E(m, st[a]);
    if ((source == n[0] && destin == n[1]) || (destin == n[0] && source == n[1])) {
      opp[k] = n[2]; trash[k++] = a; continue;
    }
    if ((source == n[1] && destin == n[2]) || (destin == n[1] && source == n[2])) {
      opp[k] = n[0]; trash[k++] = a; continue;
    }
    if ((source == n[2] && destin == n[0]) || (destin == n[2] && source == n[0])) {
      opp[k] = n[1]; trash[k++] = a; continue;
    }
  }
  /* erase the shell element(s) and drop them from the source stencil */
  int rest[1024], nr = 0;
  for (int a = 0; a < deg; ++a) {
    if (a == trash[0] || a == trash[1]) {
      set_elem(m, st[a], -1, -1, -1);
      continue;
    }
    rest[nr++] = st[a];
  }
  for (int q = 0; q < k; ++q)
    if (opp[q] >= 0) m->fixes[opp[q]] = 1;
  /* Mesh::copyStencil(source, destin, k), mesh.cpp:497-506 */
  for (int a = 0; a < nr; ++a) stenc_append(m, destin, rest[a]);
  /* relabel source -> destin */
  for (int a = 0; a < nr; ++a) {
    int* n = m->elems + (size_t) rest[a] * 3;
    if (n[0] == source) n[0] = destin;
    else if (n[1] == source) n[1] = destin;
    else if (n[2] == source) n[2] = destin;
  }
  m->fixes[destin] = 1;
  for (int b = 0; b < m->vdeg[source]; ++b) {
    int v = VC(m, source)[b];
    if (m->activ[v] == 0) m->activ[v] = 1;
  }
  m->vdeg[source] = 0;
  m->alive[source] = 0;
  for (int a = 0; a < m->bucket; ++a) st[a] = -1;
}

/* Coarse::run, coarsening.cpp:463-508 */
int orc_coarsen(orc_mesh* m) {
  m->err = 0;
  int tasks_total = 0, indep_total = 0, levels = 0;
  /* preProcess, coarsening.cpp:257-281 */
  for (int i = 0; i < m->nb_nodes; ++i) {
    if (m->tags[i] & TAG_CORNER) m->activ[i] = -1;
    else m->activ[i] = (signed char) (m->alive[i] ? 1 : 0);
    m->fixes[i] = 0;
  }
  ivec filt = {0};
  int nb_indep = 0, guard = 0;
  do {
    extract_primal(m);
    /* filterPoints, coarsening.cpp:284-304 */
    filt.n = 0;
    nb_indep = 0;
    for (int i = 0; i < m->nb_nodes; ++i) {
      if (m->activ[i] > 0) {
        m->activ[i] = 0;
        int t = identify_target(m, i);
        m->subset[3][i] = t;
        if (t > -1) iv_push(&filt, i);
      }
    }
    if (!filt.n) break;
    tasks_total += filt.n;
    levels++;
    nb_indep = indep_set(m, filt.a, filt.n);
    indep_total += nb_indep;
    /* processPoints, coarsening.cpp:322-329 (independent: order-free) */
    for (int i = 0; i < nb_indep; ++i) {
      int v = m->subset[0][i];
      collapse_edge(m, v, m->subset[3][v]);
    }
    fix_tagged(m);
  } while (nb_indep && guard++ < LOOP_CAP);
  if (guard >= LOOP_CAP) m->err = ORC_ERR_NO_PROGRESS;
  free(filt.a);
  m->counters[0] = tasks_total;
  m->counters[1] = indep_total;
  m->counters[2] = indep_total;
  m->counters[3] = levels;
  return m->err;
}

/* ------------------------------------------------------------------------ */
/* swapping: swapping.cpp, matching.cpp                                     */
/* ------------------------------------------------------------------------ */
static int* D(orc_mesh* m, int i) { return m->dual + (size_t) i * 4; }

/* Match::matchAndUpdate, matching.cpp:103-135 */
static void match_and_update(orc_mesh* m, int vertex, ivec* stack) {
  iv_push(stack, vertex);
  do {
    int cur = stack->a[--stack->n];
    int current = D(m, cur)[0];
    if (m->visited[current]) continue;
    m->visited[current] = 1;
    for (int a = 1; a < m->dual_n[cur]; ++a) {
      int neigh = D(m, cur)[a];
      if (!m->visited[neigh]) {
        m->visited[neigh] = 1;
        m->matched[current] = neigh;
        m->matched[neigh] = MATCHED;
        int nxt = m->map[neigh];
        if (nxt < 0) continue;
        for (int b = 1; b < m->dual_n[nxt]; ++b) {
          int far = D(m, nxt)[b];
          int next = m->map[far];
          if (next > -1) {
            signed char old = m->degree[far];
            m->degree[far] = (signed char) (old - 1);
            if (old == 2) iv_push(stack, next);
          }
        }
        break;
      }
    }
  } while (stack->n);
}

/* ---- emulated matching rules (analysis only; ORC_SWAP_REFERENCE is the
 * reference) ---------------------------------------------------------- */

/* the reference's loop without the degree-1 stack: each row in order takes
 * free neighbours, stopping at the first one ever listed as a candidate in
 * this call (matching.cpp:115-132 without lines 124-129) */
static void match_sequential_rows(orc_mesh* m, int nt) {
  for (int i = 0; i < nt; ++i) {
    const int c = D(m, i)[0];
    if (m->visited[c]) continue;
    m->visited[c] = 1;
    for (int a = 1; a < m->dual_n[i]; ++a) {
      const int n = D(m, i)[a];
      if (m->visited[n]) continue;
      m->visited[n] = 1;
      m->matched[c] = n;
      m->matched[n] = MATCHED;
      if (m->map[n] < 0) continue;
      break;
    }
  }
}

/* the GPU free mode's default rule: the same loop (without the degree-1
 * stack), over the rows in the order (candidate id mod 4, candidate id) */
static int interleaved_before(const orc_mesh* m, int i, int j) {
  const int a = m->dual[(size_t) i * 4], b = m->dual[(size_t) j * 4];
  if ((a & 3) != (b & 3)) return (a & 3) < (b & 3);
  return a < b;
}

static void match_interleaved_rows(orc_mesh* m, int nt) {
  int* order = (int*) malloc(sizeof(int) * (size_t) (nt > 0 ? nt : 1));
  int k = 0;
  for (int cls = 0; cls < 4; ++cls)
    for (int i = 0; i < nt; ++i)
      if ((D(m, i)[0] & 3) == cls) order[k++] = i;
  /* within a class the rows are in list order, i.e. increasing candidate id;
   * check it rather than assume it */
  for (int a = 1; a < k; ++a)
    if (!interleaved_before(m, order[a - 1], order[a])) m->err = ORC_ERR_INVALID;
  for (int a = 0; a < k; ++a) {
    const int i = order[a];
    const int c = D(m, i)[0];
    if (m->visited[c]) continue;
    m->visited[c] = 1;
    for (int q = 1; q < m->dual_n[i]; ++q) {
      const int n = D(m, i)[q];
      if (m->visited[n]) continue;
      m->visited[n] = 1;
      m->matched[c] = n;
      m->matched[n] = MATCHED;
      if (m->map[n] < 0) continue;
      break;
    }
  }
  free(order);
}

static uint64_t hs_mix(uint64_t x) {
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ULL;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}

static int hs_row_of(orc_mesh* m, int e, int nt) {
  const int x = m->map[e];
  return (x >= 0 && x < nt && D(m, x)[0] == e) ? x : -1;
}

/* weight of dual edge (row i, slot q) in the round-synchronous handshake:
 * a symmetric hash (random rule) or the edge's slot in the row of its
 * lower-id candidate end, then the hash (row-slot rule) */
static uint32_t hs_weight(orc_mesh* m, int nt, int i, int q, int round, int level) {
  const int c = D(m, i)[0], n = D(m, i)[q];
  const int lo = c < n ? c : n, hi = c < n ? n : c;
  const uint64_t h = hs_mix(((uint64_t) (uint32_t) lo << 32 | (uint32_t) hi) ^
                            ((uint64_t) (round + 16 * level) * 0xd1b54a32d192ed03ULL));
  if (m->swap_rule == ORC_SWAP_HANDSHAKE_RANDOM) return (uint32_t) (h >> 32) | 1u;
  int pos = q;
  const int xn = hs_row_of(m, n, nt);
  if (xn >= 0 && n < c)
    for (int a = 1; a < m->dual_n[xn]; ++a)
      if (D(m, xn)[a] == c) pos = a;
  return ((uint32_t) (4 - pos) << 30) | ((uint32_t) (h >> 34)) | 1u;
}

/* the GPU free mode's rule: rounds of proposals along each unmatched
 * candidate's heaviest free edge; mutual candidate pairs match, a
 * non-candidate accepts its heaviest proposer */
static void match_handshake_emul(orc_mesh* m, int nt, int level) {
  int* mate = m->hs_mate;
  int* choice = m->hs_choice;
  uint64_t* prop = m->hs_prop;
  for (int i = 0; i < nt; ++i)
    for (int a = 0; a < m->dual_n[i]; ++a) {
      mate[D(m, i)[a]] = -1;
      prop[D(m, i)[a]] = 0;
    }
  for (int r = 0; r < 4; ++r) {
    for (int i = 0; i < nt; ++i) {
      const int c = D(m, i)[0];
      int best = -1;
      uint32_t bw = 0;
      if (mate[c] == -1)
        for (int q = 1; q < m->dual_n[i]; ++q) {
          if (mate[D(m, i)[q]] != -1) continue;
          const uint32_t w = hs_weight(m, nt, i, q, r, level);
          if (w > bw) { bw = w; best = q; }
        }
      choice[i] = best < 0 ? -1 : D(m, i)[best];
      if (best >= 0) {
        const uint64_t key = ((uint64_t) bw << 32) | (uint32_t) c;
        if (key > prop[D(m, i)[best]]) prop[D(m, i)[best]] = key;
      }
    }
    /* decisions read this round's proposals only, then apply */
    ivec acc = {0};
    for (int i = 0; i < nt; ++i) {
      const int n = choice[i];
      if (n < 0) continue;
      const int c = D(m, i)[0];
      const int x = hs_row_of(m, n, nt);
      int ok;
      if (x >= 0) {
        ok = choice[x] == c && c < n;
      } else {
        int q = 1;
        while (D(m, i)[q] != n) ++q;
        ok = prop[n] == (((uint64_t) hs_weight(m, nt, i, q, r, level) << 32) | (uint32_t) c);
      }
      if (ok) { iv_push(&acc, c); iv_push(&acc, n); }
    }
    for (int p = 0; p < acc.n; p += 2) {
      mate[acc.a[p]] = acc.a[p + 1];
      mate[acc.a[p + 1]] = acc.a[p];
      m->matched[acc.a[p]] = acc.a[p + 1];
    }
    free(acc.a);
    for (int i = 0; i < nt; ++i)
      for (int a = 1; a < m->dual_n[i]; ++a) prop[D(m, i)[a]] = 0;
  }
}

int orc_set_swap_strict_map(orc_mesh* m, int on) {
  m->swap_strict_map = on != 0;
  return ORC_OK;
}

int orc_set_swap_rule(orc_mesh* m, int rule) {
  if (rule < ORC_SWAP_REFERENCE || rule > ORC_SWAP_GREEDY_INTERLEAVED) return ORC_ERR_INVALID;
  m->swap_rule = rule;
  return ORC_OK;
}

/* Swap::swap, swapping.cpp:55-149; returns 2 on a committed flip */
static int swap_pair(orc_mesh* m, int id1, int id2, int index) {
  int cur1[3] = {-1, -1, -1}, cur2[3] = {-1, -1, -1};
  const int* o1 = E(m, id1);
  const int* o2 = E(m, id2);
  for (int i = 0; i < 3; ++i) {
    int j = (i + 1) % 3, k = (i + 2) % 3;
    if (o1[i] == o2[1] && o1[j] == o2[0]) {
      cur1[0] = o1[i]; cur1[1] = o2[2]; cur1[2] = o1[k];
      cur2[0] = o1[k]; cur2[1] = o2[2]; cur2[2] = o1[j];
      break;
    }
    if (o1[i] == o2[2] && o1[j] == o2[1]) {
      cur1[0] = o1[i]; cur1[1] = o2[0]; cur1[2] = o1[k];
      cur2[0] = o1[k]; cur2[1] = o2[0]; cur2[2] = o1[j];
      break;
    }
    if (o1[i] == o2[0] && o1[j] == o2[2]) {
      cur1[0] = o1[i]; cur1[1] = o2[1]; cur1[2] = o1[k];
      cur2[0] = o1[k]; cur2[1] = o2[1]; cur2[2] = o1[j];
      break;
    }
  }
  if (cur1[0] < 0) return 0;  /* no shared edge (reference would read index -1) */
  if (!ccw(m, cur1) || !ccw(m, cur2)) return 0;
  double q[2] = {quality_of(m, cur1), quality_of(m, cur2)};
  double q_old = dmin(m->qualit[id1], m->qualit[id2]);
  double q_new = dmin(q[0], q[1]);
  if (q_new < q_old) return 0;
  set_elem(m, id1, cur1[0], cur1[1], cur1[2]);
  set_elem(m, id2, cur2[0], cur2[1], cur2[2]);
  stenc_append(m, cur2[0], id2);
  stenc_append(m, cur2[1], id1);
  m->fixes[cur1[0]] = 1;
  m->fixes[cur1[1]] = 1;
  m->fixes[cur1[2]] = 1;
  m->fixes[cur2[2]] = 1;
  m->qualit[id1] = q[0];
  m->qualit[id2] = q[1];
  for (int a = 0; a < m->dual_n[index]; ++a) {
    int t = D(m, index)[a];
    if (m->activ[t] == 0) m->activ[t] = 1;
  }
  /* the reference follows the map even to a row of an earlier level of the
   * call; with swap_strict_map (the GPU free mode's rule) only to a row of
   * the current level */
  if (m->map[id2] > -1 &&
      (!m->swap_strict_map || (m->map[id2] < m->swap_nt && D(m, m->map[id2])[0] == id2))) {
    int x = m->map[id2];
    for (int a = 0; a < m->dual_n[x]; ++a) {
      int t = D(m, x)[a];
      if (m->activ[t] == 0) m->activ[t] = 1;
    }
  }
  return 2;
}

/* Swap::run, swapping.cpp:383-428 */
int orc_swap(orc_mesh* m) {
  m->err = 0;
  int activ_total = 0, tasks_total = 0, commit_total = 0, levels = 0;
  /* cacheQuality, swapping.cpp:152-178 */
  for (int i = 0; i < m->nb_nodes; ++i) m->fixes[i] = 0;
  for (int i = 0; i < m->nb_elems; ++i) {
    m->map[i] = -1;
    m->activ[i] = 0;
  }
  for (int i = 0; i < m->nb_elems; ++i)
    if (E(m, i)[0] > -1) {
      m->qualit[i] = quality_of(m, E(m, i));
      m->activ[i] = 1;
    }
  ivec list = {0}, stack = {0};
  int commit = 0, guard = 0;
  do {
    /* filterElems, swapping.cpp:181-201 */
    list.n = 0;
    int activ = 0;
    for (int i = 0; i < m->nb_elems; ++i)
      if (m->activ[i]) {
        m->activ[i] = 0;
        activ++;
        if (m->qualit[i] < Q_MIN) iv_push(&list, i);
      }
    activ_total += activ;
    if (!list.n) break;
    tasks_total += list.n;
    levels++;
    /* extractDualGraph, swapping.cpp:204-248 */
    for (int i = 0; i < list.n; ++i) {
      int k = list.a[i];
      const int* n = E(m, k);
      int* d = D(m, i);
      int dn = 0;
      d[dn++] = k;
      const int* s0 = S(m, n[0]);
      for (int a = 0; dn < 3 && a < m->deg[n[0]]; ++a) {
        int t = s0[a];
        if (t == k) continue;
        const int* v = E(m, t);
        if ((v[0] == n[0] && v[1] == n[2]) || (v[0] == n[1] && v[1] == n[0]) ||
            (v[1] == n[0] && v[2] == n[2]) || (v[1] == n[1] && v[2] == n[0]) ||
            (v[2] == n[0] && v[0] == n[2]) || (v[2] == n[1] && v[0] == n[0]))
          d[dn++] = t;
      }
      const int* s2 = S(m, n[2]);
      for (int a = 0; a < m->deg[n[2]]; ++a) {
        int t = s2[a];
        if (t == k) continue;
        const int* v = E(m, t);
        if ((v[0] == n[2] && v[1] == n[1]) || (v[1] == n[2] && v[2] == n[1]) ||
            (v[2] == n[2] && v[0] == n[1])) {
          d[dn++] = t;
          break;
        }
      }
      m->dual_n[i] = dn;
      m->map[k] = i;
    }
    /* Match::computeGreedyMatching, matching.cpp:81-100 */
    memset(m->visited, 0, (size_t) m->capa_elem);
    memset(m->degree, 0, (size_t) m->capa_elem);
    for (int i = 0; i < m->capa_elem; ++i) m->matched[i] = -1;
    for (int i = 0; i < list.n; ++i)
      m->degree[D(m, i)[0]] = (signed char) (m->dual_n[i] - 1);
    if (m->swap_rule == ORC_SWAP_REFERENCE)
      for (int i = 0; i < list.n; ++i) match_and_update(m, i, &stack);
    else if (m->swap_rule == ORC_SWAP_SEQUENTIAL_ROWS)
      match_sequential_rows(m, list.n);
    else if (m->swap_rule == ORC_SWAP_GREEDY_INTERLEAVED)
      match_interleaved_rows(m, list.n);
    else
      match_handshake_emul(m, list.n, levels);
    /* processFlips, swapping.cpp:251-269 (pairs are disjoint: order-free) */
    int npairs = 0;
    for (int index = 0; index < list.n; ++index) {
      int k1 = D(m, index)[0];
      if (m->matched[k1] > -1) npairs++;
    }
    log_begin(m, ORC_LOG_MATCH, npairs);
    for (int index = 0; index < list.n; ++index) {
      int k1 = D(m, index)[0];
      int k2 = m->matched[k1];
      if (k2 > -1) {
        iv_push(&m->log, k1);
        iv_push(&m->log, k2);
      }
    }
    commit = 0;
    for (int index = 0; index < list.n; ++index) {
      int k1 = D(m, index)[0];
      int k2 = m->matched[k1];
      if (k2 > -1) {
        m->swap_nt = list.n;
        commit += swap_pair(m, k1, k2, index);
      }
    }
    commit_total += commit;
    fix_tagged(m);
  } while (commit && guard++ < LOOP_CAP);
  if (guard >= LOOP_CAP) m->err = ORC_ERR_NO_PROGRESS;
  free(list.a);
  free(stack.a);
  m->counters[0] = activ_total;
  m->counters[1] = tasks_total;
  m->counters[2] = commit_total;
  m->counters[3] = levels;
  return m->err;
}

/* ------------------------------------------------------------------------ */
/* smoothing: smoothing.cpp                                                  */
/* ------------------------------------------------------------------------ */
/* Smooth::moveSmartLaplacian, smoothing.cpp:40-126 */
static int move_laplacian(orc_mesh* m, int i) {
  const int* vic = VC(m, i);
  const int* st = S(m, i);
  int deg = m->deg[i];
  int nb_neigh = m->vdeg[i];
  double q_min = 1.7976931348623157e308;
  for (int a = 0; a < deg; ++a) q_min = dmin(q_min, m->qualit[st[a]]);
  double metric[3 * 1024], qualit[1024];
  double* pa = Pw(m, i);
  double* ta = T(m, i);
  double opt[2] = {0, 0};
  for (int k = 0; k < nb_neigh; ++k) {
    int neigh = vic[k];
    const double* pb = P(m, neigh);
    double len = length(m, i, neigh);
    opt[0] += pa[0] + ((pb[0] - pa[0]) / len);
    opt[1] += pa[1] + ((pb[1] - pa[1]) / len);
    memcpy(metric + k * 3, T(m, neigh), sizeof(double) * 3);
  }
  opt[0] /= nb_neigh;
  opt[1] /= nb_neigh;
  const double pini[2] = {pa[0], pa[1]};
  const double tini[3] = {ta[0], ta[1], ta[2]};
  interpolate(metric, ta, nb_neigh);
  int valid, retry = 0;
  double weight = 1;
  do {
    valid = 1;
    pa[0] = (1 - weight) * pini[0] + weight * opt[0];
    pa[1] = (1 - weight) * pini[1] + weight * opt[1];
    for (int a = 0; valid && a < deg; ++a) {
      const int* n = E(m, st[a]);
      valid = 0;
      if (ccw(m, n)) {
        qualit[a] = quality_of(m, n);
        valid = (qualit[a] > q_min);
      }
    }
    weight *= 0.5;
  } while (!valid && ++retry < 5);
  if (valid) {
    for (int a = 0; a < deg; ++a) m->qualit[st[a]] = qualit[a];
  } else {
    pa[0] = pini[0]; pa[1] = pini[1];
    ta[0] = tini[0]; ta[1] = tini[1]; ta[2] = tini[2];
  }
  return valid;
}

/* Smooth::run, smoothing.cpp:274-302 */
int orc_smooth(orc_mesh* m, int depth) {
  m->err = 0;
  /* preProcess, smoothing.cpp:129-142 */
  for (int i = 0; i < m->nb_nodes; ++i)
    if (m->alive[i]) m->activ[i] = (signed char) ((m->tags[i] & TAG_BOUND) ? 0 : 1);
  extract_primal(m);
  coloring(m);
  /* cacheQuality, smoothing.cpp:145-155 */
  for (int i = 0; i < m->nb_elems; ++i)
    if (E(m, i)[0] > -1) m->qualit[i] = quality_of(m, E(m, i));
  int tasks = 0, commit = 0;
  for (int level = 0; level < depth; ++level)
    for (int c = 0; c < m->nb_parts; ++c)
      for (int j = 0; j < m->cardin[c]; ++j) {
        int k = m->subset[c][j];
        if (m->activ[k]) {
          commit += move_laplacian(m, k);
          tasks++;
        }
      }
  m->counters[0] = tasks;
  m->counters[1] = commit;
  m->counters[2] = commit;
  m->counters[3] = depth;
  return m->err;
}

/* ------------------------------------------------------------------------ */
int orc_nb_nodes(const orc_mesh* m) { return m->nb_nodes; }
int orc_nb_elems(const orc_mesh* m) { return m->nb_elems; }
double orc_complexity(const orc_mesh* m) { return m->complexity; }
void orc_counters(const orc_mesh* m, int out[4]) { memcpy(out, m->counters, sizeof m->counters); }

void orc_export(const orc_mesh* m, double* points, double* tensor, int* elems,
                uint8_t* alive, uint8_t* tags) {
  if (points) memcpy(points, m->points, sizeof(double) * 2 * (size_t) m->nb_nodes);
  if (tensor) memcpy(tensor, m->tensor, sizeof(double) * 3 * (size_t) m->nb_nodes);
  if (elems) memcpy(elems, m->elems, sizeof(int) * 3 * (size_t) m->nb_elems);
  if (alive) memcpy(alive, m->alive, (size_t) m->nb_nodes);
  if (tags) memcpy(tags, m->tags, (size_t) m->nb_nodes);
}

const int32_t* orc_log(const orc_mesh* m, size_t* n) {
  *n = (size_t) m->log.n;
  return m->log.a;
}

void orc_log_clear(orc_mesh* m) { m->log.n = 0; }

void orc_eigen(const double mat[4], double val[2], double v1[2], double v2[2]) {
  eigen(mat, val, v1, v2);
}
void orc_interpolate(const double* tensors, double result[3], int nb) {
  interpolate(tensors, result, nb);
}
double orc_quality(const double pa[2], const double pb[2], const double pc[2],
                   const double ta[3], const double tb[3], const double tc[3]) {
  return quality(pa, pb, pc, ta, tb, tc);
}
double orc_length(const double pa[2], const double pb[2], const double ta[3], const double tb[3]) {
  return dist2(pa, pb, ta, tb);
}
void orc_steiner(const double pa[2], const double pb[2], const double ta[3],
                 const double tb[3], double point[2], double tensor[3]) {
  steiner(pa, pb, ta, tb, point, tensor);
}
double orc_log_fn(double x) { return trn_log(x); }
double orc_exp_fn(double x) { return trn_exp(x); }
double orc_pow_fn(double x, double y) { return trn_pow(x, y); }
