/*
 * trn_oracle.h — TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * A plain-C, single-threaded restatement of trinity's adaptation round
 * (metric recovery, refinement, edge collapse, edge flips, smoothing and
 * their graph heuristics), following the reference's 1-thread execution
 * order so that its results are bit-identical to the reference built with
 * -ffp-contract=off and the project's log/exp/pow (oracle/Makefile "ref").
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load it.
 *
 * Besides the mesh state it records a decision log — the independent sets,
 * matchings and colorings the reference's heuristics produced — which the GPU
 * replays to prove its topology kernels bit-exact. Log layout (int32 stream):
 *   ORC_LOG_MIS      n  v_0 .. v_{n-1}                 (coarsening, per level)
 *   ORC_LOG_MATCH    n  k1_0 k2_0 .. k1_{n-1} k2_{n-1} (swapping, per level:
 *                                                      k2 = matched[k1] > -1)
 *   ORC_LOG_COLORING p  c_0 ids.. c_1 ids.. ...         (smoothing, per run:
 *                                                      p parts, c_j members)
 */
#ifndef TRN_ORACLE_H
#define TRN_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_LOG_MIS = 1, ORC_LOG_MATCH = 2, ORC_LOG_COLORING = 3 };

enum {
  ORC_OK = 0,
  ORC_ERR_CAPACITY = 1,
  ORC_ERR_IO = 2,
  ORC_ERR_INVALID = 3,
  ORC_ERR_NO_PROGRESS = 4,
};

typedef struct orc_mesh orc_mesh;

/* capacity: nodes/elems slots; bucket: stencil slots per vertex */
orc_mesh* orc_create(int capa_node, int capa_elem, int bucket);
void orc_destroy(orc_mesh* m);

/* tris: 0-based CCW triples; tags: 0 / 4 (boundary) / 12 (boundary|corner) */
int orc_load(orc_mesh* m, int nb_nodes, int nb_elems, const double* points,
             const int* tris, const uint8_t* tags, const double* solut);

int orc_metric(orc_mesh* m, double target, int norm, double h_min, double h_max);
int orc_refine(orc_mesh* m, int depth);
int orc_coarsen(orc_mesh* m);
int orc_swap(orc_mesh* m);
int orc_smooth(orc_mesh* m, int depth);

int orc_nb_nodes(const orc_mesh* m);
int orc_nb_elems(const orc_mesh* m);
/* copy out nb_nodes / nb_elems sized state (any pointer may be NULL) */
void orc_export(const orc_mesh* m, double* points, double* tensor, int* elems,
                uint8_t* alive, uint8_t* tags);
/* complexity of the last metric run (for diagnostics) */
double orc_complexity(const orc_mesh* m);
/* per-kernel counters of the last run: [0]=evaluated [1]=tasks [2]=committed [3]=levels */
void orc_counters(const orc_mesh* m, int out[4]);

/* Swap matching rule, for the analysis of the GPU free mode only:
 * ORC_SWAP_REFERENCE (default) is the reference's greedy with its degree-1
 * stack (matching.cpp:81-135); the others are emulations: the same loop
 * without the stack, the GPU's round-synchronous handshake with random
 * or row-slot edge weights, and the GPU free mode's default, the loop
 * without the stack over the rows in the order (id mod 4, id). */
enum {
  ORC_SWAP_REFERENCE = 0,
  ORC_SWAP_SEQUENTIAL_ROWS = 1,
  ORC_SWAP_HANDSHAKE_RANDOM = 2,
  ORC_SWAP_HANDSHAKE_ROWSLOT = 3,
  ORC_SWAP_GREEDY_INTERLEAVED = 4,
};
int orc_set_swap_rule(orc_mesh* m, int rule);
/* flips re-activate the elements of their partner's row only when that row
 * belongs to the current level (the GPU free mode's rule: its rows are
 * numbered in append order, so a row index of an earlier level names an
 * unrelated row); the reference follows any row the map names */
int orc_set_swap_strict_map(orc_mesh* m, int on);

const int32_t* orc_log(const orc_mesh* m, size_t* n);
void orc_log_clear(orc_mesh* m);

/* numerics, exported for unit tests against the reference's numeric.cpp */
void orc_eigen(const double m[4], double val[2], double v1[2], double v2[2]);
void orc_interpolate(const double* tensors, double result[3], int nb);
double orc_quality(const double pa[2], const double pb[2], const double pc[2],
                   const double ta[3], const double tb[3], const double tc[3]);
double orc_length(const double pa[2], const double pb[2], const double ta[3],
                  const double tb[3]);
void orc_steiner(const double pa[2], const double pb[2], const double ta[3],
                 const double tb[3], double point[2], double tensor[3]);
double orc_log_fn(double x);
double orc_exp_fn(double x);
double orc_pow_fn(double x, double y);

#ifdef __cplusplus
}
#endif
#endif
