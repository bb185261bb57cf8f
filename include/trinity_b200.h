/*
 * trinity_b200.h — C ABI of the B200 implementation of trinity's adaptation
 * round (metric recovery, refinement, edge collapse, edge flips, smoothing).
 *
 * Every entry point replaces one call of trinity's C++ API (include/trinity.h
 * of the reference, which pulls in include/trinity/<kernel>.h); the reference
 * interface is named beside each declaration. Plain pointers and sizes only.
 * All functions return TRN_OK (0) or a TRN_ERR_* code; trn_last_error() gives
 * the message. One CUDA stream per mesh; every call is blocking, like the
 * reference's run() methods, and not thread-safe on the same mesh.
 */
#ifndef TRINITY_B200_H
#define TRINITY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  TRN_OK = 0,
  TRN_ERR_CAPACITY = 1,    /* a capacity (nodes, elements, stencil bucket) is too small */
  TRN_ERR_IO = 2,          /* file missing or malformed */
  TRN_ERR_INVALID = 3,     /* bad argument */
  TRN_ERR_NO_PROGRESS = 4, /* an iterative loop hit its iteration cap */
  TRN_ERR_CUDA = 5,        /* CUDA runtime error */
  TRN_ERR_REPLAY = 6,      /* the replay log does not fit this run */
};

/* Per-kernel statistics: same layout as trinity::Stats (header.h:72-77). */
typedef struct trn_stats {
  int eval;     /* entities examined */
  int task;     /* entities changed */
  int elap;     /* milliseconds (device time of the call) */
  int step[5];  /* per-step milliseconds, kernel specific */
} trn_stats;

typedef struct trn_mesh trn_mesh;

/* replaces Mesh::Mesh(int size[2], int bucket, int depth, int verbosity, int rounds)
 * (include/trinity/mesh.h:46). size = {vertices, triangles} of the input mesh.
 * Capacity = scale x size with scale = max(3*(depth-1), 4). */
int trn_mesh_create(const int size[2], int bucket, int depth, int verbosity, int rounds,
                    trn_mesh** out);
/* as above with an explicit capacity scale (>= 1) */
int trn_mesh_create_ex(const int size[2], int bucket, int depth, int verbosity, int rounds,
                       int capa_scale, trn_mesh** out);
/* replaces Mesh::~Mesh (mesh.cpp:47-54) */
int trn_mesh_destroy(trn_mesh* mesh);

/* replaces Mesh::load(path, solu) (mesh.h:65, io.cpp:53-161): medit .mesh and
 * .bb solution field, then Mesh::rebuildTopology (mesh.cpp:191-249) */
int trn_mesh_load(trn_mesh* mesh, const char* mesh_path, const char* solut_path);
/* the same from arrays: points[2V], tris[3T] 0-based CCW, tags[V] (0, 4 =
 * boundary, 12 = boundary|corner, header.h:55-60), solut[V] */
int trn_mesh_load_arrays(trn_mesh* mesh, int nb_nodes, int nb_elems, const double* points,
                         const int* tris, const uint8_t* tags, const double* solut);
/* restore the state right after the last load, from device-resident copies
 * of its input (no host transfer); for repeated runs on one input */
int trn_mesh_reload(trn_mesh* mesh);
/* replaces Mesh::store(path) (mesh.h:66, io.cpp:164-255) */
int trn_mesh_store(trn_mesh* mesh, const char* path);
/* the binary form of the mesh (points, tags, triangles; renumbered like
 * trn_mesh_store), which trn_mesh_load reads in place of the .mesh text: a
 * sidecar that skips the text parse. No counterpart in the reference (its
 * loader reads the text, io.cpp:53-161). */
int trn_mesh_store_binary(trn_mesh* mesh, const char* path);
/* the files as trn_mesh_load reads them (text with one thread per chunk of
 * each section, or the binary form), into host arrays: 0-based triangles,
 * tags 0 / 4 (boundary) / 12 (corner), the .bb values (solut_path may be
 * NULL). Needs no mesh and no GPU. Always sets the counts; fills the arrays
 * (any may be NULL) when they hold cap_nodes / cap_elems entries. */
int trn_read_mesh_files(const char* mesh_path, const char* solut_path, int* nb_nodes, int* nb_elems,
                        double* points, int* tris, uint8_t* tags, double* solut, int cap_nodes,
                        int cap_elems);
/* metric field in medit .sol format (the reference writes none; an addition) */
int trn_mesh_store_sol(trn_mesh* mesh, const char* path);
/* copy out the raw state: nb_nodes / nb_elems entries (any pointer may be NULL) */
int trn_mesh_export(trn_mesh* mesh, double* points, double* tensor, int* tris, uint8_t* alive,
                    uint8_t* tags);
/* The adapted mesh without deleted entities, renumbered in id order as
 * Mesh::store numbers its output (io.cpp:199-233): points[2V'], tris[3T']
 * (0-based), tensor[3V'] (may be NULL). Size the arrays with the live counts
 * of trn_mesh_counts; V' and T' are returned. */
int trn_mesh_export_compact(trn_mesh* mesh, double* points, int* tris, double* tensor,
                            int* nb_nodes, int* nb_elems);
/* per-element quality in the current arithmetic form (nb_elems entries, 0
 * for deleted elements) */
int trn_mesh_qualities(trn_mesh* mesh, double* q);
/* replaces Mesh::computeQuality(double quality[3]) (mesh.cpp:647-681):
 * quality[0] = min(quality[0], q_min), quality[1] = max(quality[1], q_max),
 * quality[2] = mean over live elements */
int trn_mesh_quality_stats(trn_mesh* mesh, double quality[3]);
/* the vertex and element slots the mesh was created with (Mesh::capa,
 * mesh.h:98-103) */
int trn_mesh_capacity(trn_mesh* mesh, int* capa_nodes, int* capa_elems);
/* slot counts (deleted entities included) and live counts */
int trn_mesh_counts(trn_mesh* mesh, int* nb_nodes, int* nb_elems, int* live_nodes,
                    int* live_elems);

/* replaces Metrics(Mesh*, target_factor, Lp_norm, h_min, h_max) + Metrics::run
 * (include/trinity/metric.h:38-44, metric.cpp:24-70) */
int trn_metric_run(trn_mesh* mesh, double target_factor, int lp_norm, double h_min, double h_max,
                   trn_stats* stats);
/* replaces Refine(Mesh*, level) + Refine::run (refinement.h:39-42, refinement.cpp:445-493) */
int trn_refine_run(trn_mesh* mesh, int depth, trn_stats* stats);
/* replaces Coarse(Mesh*, Partit*) + Coarse::run (coarsening.h:40-42, coarsening.cpp:463-508);
 * max_colors mirrors Partit(mesh, max_part_size) (partition.h:46) */
int trn_coarsen_run(trn_mesh* mesh, int max_colors, trn_stats* stats);
/* replaces Swap(Mesh*) + Swap::run (swapping.h:39-42, swapping.cpp:383-428) */
int trn_swap_run(trn_mesh* mesh, trn_stats* stats);
/* replaces Smooth(Mesh*, Partit*, level) + Smooth::run (smoothing.h:39-42, smoothing.cpp:274-302) */
int trn_smooth_run(trn_mesh* mesh, int max_colors, int depth, trn_stats* stats);
/* one full round: refine, coarsen, swap, smooth (main.cpp:52-57) */
int trn_round_run(trn_mesh* mesh, int depth, trn_stats stats[4]);
/* The same round, free mode only, as one CUDA graph: captured on the mesh's
 * first call (and again when depth, precision or seed change), replayed by
 * later calls with no host round trip inside the round (the coarsening,
 * swapping and coloring loops are device-decided loop nodes). Ends where
 * trn_round_run ends. stats[k].eval / task per stage as trn_round_run;
 * stats[0].elap holds the whole round's device time. TRN_ERR_INVALID in
 * replay mode. No counterpart in the reference. */
int trn_round_graph_run(trn_mesh* mesh, int depth, trn_stats stats[4]);

/* Adapt a batch of independent meshes concurrently on the current GPU: each
 * mesh (already loaded) gets metric recovery and `rounds` rounds on its own
 * stream, driven by `threads` host threads, largest meshes first. Per mesh,
 * round_ms[i] (may be NULL) receives the device time of its rounds and
 * tri_in[i] (may be NULL) the sum of its live triangles at round starts.
 * No counterpart in the reference (one mesh per process there). Streams
 * beyond the device's hardware queues share them: set the environment
 * variable CUDA_DEVICE_MAX_CONNECTIONS=32 before the process initialises CUDA
 * (default 8; measured on B200 with 256 meshes: 61 -> 87 M triangles/s).
 * Returns the first error met. */
int trn_batch_adapt(trn_mesh* const* meshes, int count, double target_factor, int lp_norm,
                    double h_min, double h_max, int rounds, int depth, int threads,
                    double* round_ms, long long* tri_in);
/* as trn_batch_adapt; flags TRN_BATCH_GRAPH runs each round as the mesh's
 * captured round (trn_round_graph_run; free mode) */
#define TRN_BATCH_GRAPH 1
int trn_batch_adapt_ex(trn_mesh* const* meshes, int count, double target_factor, int lp_norm,
                       double h_min, double h_max, int rounds, int depth, int threads, int flags,
                       double* round_ms, long long* tri_in);

/* Element-quality functional and its adjoint. No counterpart in the
 * reference; it differentiates the reference's own arithmetic:
 *   J = sum over live elements T of q_T, q_T = numeric::computeQuality
 *       (numeric.cpp:251-306) of T at the coordinates `xy` under the nodal
 *       metric M.
 * M is the mesh's current tensors when `solut` is NULL; otherwise it is the
 * metric that trn_metric_run would recover from the nodal solution `solut`
 * with (target_factor, lp_norm, h_min, h_max) on the mesh's own coordinates
 * (hessian.cpp:24-153, metric.cpp:59-238), which the mesh keeps unchanged.
 * Outputs: *value = J (host pointer, may be NULL); grad_xy[2V] = dJ/dxy at
 * that fixed nodal metric; grad_solut[V] = dJ/dsolut through the gradient
 * and Hessian recovery, the local L^p normalisation and the global scale
 * with its clamp. xy (2V, NULL = the mesh's coordinates), solut, grad_xy and
 * grad_solut are DEVICE pointers in the mesh's vertex numbering; either
 * gradient may be NULL (grad_solut needs solut). precision: TRN_PRECISION_FP64
 * (q bit-identical to the adaptation kernels) or TRN_PRECISION_MIXED (q and
 * the whole adjoint in FP32; coordinates and areas FP64; the metric recovery
 * FP64). Deterministic: every sum is a gather in a fixed order. */
int trn_quality_adjoint(trn_mesh* mesh, const double* xy, const double* solut,
                        double target_factor, int lp_norm, double h_min, double h_max,
                        int precision, double* value, double* grad_xy, double* grad_solut);
/* Gradient-based smoothing, beside Smooth::run's smart Laplacian
 * (smoothing.cpp:40-126, 274-302): `steps` passes over the color classes of
 * the interior vertices; each vertex v steps along M_v^-1 g_v, g_v the
 * gradient at v of its elements' summed quality, or summed log-quality with
 * TRN_SMOOTH_LOG_Q in `mode` (the worst elements weigh most). With
 * TRN_SMOOTH_TENSOR_FOLLOWS a moved vertex takes the log-Euclidean mean of
 * its neighbours' tensors, as the smart Laplacian's does (smoothing.cpp:64-81),
 * and g_v is taken under it; otherwise M_v stays. The step's metric length is
 * `max_len` times the mean metric length of v's edges (under M_v), and it
 * backs off 1, 1/2, .., 1/16 until the elements stay CCW, each above the old
 * stencil minimum, with a larger objective. Free mode only (TRN_ERR_INVALID
 * in replay mode). stats->eval / task: vertices tried / moved. */
#define TRN_SMOOTH_LOG_Q 1
#define TRN_SMOOTH_TENSOR_FOLLOWS 2
int trn_smooth_gradient_run(trn_mesh* mesh, int max_colors, int steps, double max_len, int mode,
                            trn_stats* stats);

/* Launch shapes (none changes a result): cfg[0] smoothing block (32..256),
 * cfg[1] collapse-target search block, cfg[2] lanes per vertex of the
 * grouped search (4, 8, 16; 1: the one-lane search at every level), cfg[3]
 * longest level list the grouped search takes (longer ones run the one-lane
 * search), cfg[4] flip block, cfg[5] lanes per smoothed vertex (1, 2, 4,
 * 8), cfg[6] variant of the smoothing kernel with 2 or more lanes (0: the
 * back-off tries in turn, up to 128 registers, two 256-thread blocks per SM;
 * 1: capped for three; 2: for four; 3: as 2, element metrics in shared
 * memory; 4, 5, 6: the five tries in one sweep, capped for four, three,
 * two blocks; 7, 8: the sweep with the element metrics in shared memory,
 * two or three blocks; one lane a vertex reads 0-2 only and treats 3-8 as
 * 2). Defaults: 2 lanes, variant 7, 256-thread blocks. Per mesh; a
 * captured round is recaptured when they change. trn_autotune chooses them
 * on the loaded mesh, timing metric + `rounds` rounds from the input (the
 * best of three runs; a candidate replaces the value kept only when at
 * least 1 % faster): first the smoothing's lanes and variant jointly, then
 * coordinate descent over all seven; then it reloads the mesh; meshes of
 * similar size can share the result through trn_set_tune. No counterpart in
 * the reference. */
#define TRN_TUNE_N 7
int trn_get_tune(trn_mesh* mesh, int cfg[TRN_TUNE_N]);
int trn_set_tune(trn_mesh* mesh, const int cfg[TRN_TUNE_N]);
int trn_autotune(trn_mesh* mesh, double target_factor, int lp_norm, double h_min, double h_max,
                 int depth, int rounds, int cfg[TRN_TUNE_N]);

/* Replay mode: the independent sets, matchings and colorings are read from a
 * decision log (int32 stream: 1 = set [n, ids], 2 = matching [n, (k1,k2)*n],
 * 3 = coloring [parts, (n, ids)*parts]) instead of being computed; the
 * complexity sum is then taken in element order. Passing n = 0 leaves
 * replay mode. No counterpart in the reference: it makes the GPU's topology
 * checkable bit for bit against the reference's 1-thread run. */
int trn_set_replay(trn_mesh* mesh, const int32_t* log, size_t n);
/* Arithmetic form of the metric computations during the rounds.
 * TRN_PRECISION_FP64 (default): the drop-in, bit-compatible with the
 * reference. TRN_PRECISION_MIXED: log-Euclidean means, metric edge lengths,
 * Steiner weights and element qualities in FP32; coordinates, orientation and
 * area tests, stored tensors and the Hessian recovery stay FP64. Not
 * available together with replay. */
#define TRN_PRECISION_FP64 0
#define TRN_PRECISION_MIXED 1
int trn_set_precision(trn_mesh* mesh, int mode);
/* free-mode options: seed of the hash priorities; exact_sum = 1 takes the
 * metric complexity sum in element order (bit-compatible with the reference) */
int trn_set_options(trn_mesh* mesh, uint64_t seed, int exact_sum);
/* free-mode swap matching (swapping.cpp:404, Match::computeGreedyMatching,
 * matching.cpp:81-135).
 * TRN_SWAP_GREEDY (default): the reference's greedy loop itself (each
 * candidate takes its free neighbours in row order up to the first one that
 * is a candidate), over the candidates in the order (id mod 4, id) instead
 * of increasing id, computed exactly in parallel; the final metric
 * edge-length histogram stays within half a point per bin of the
 * reference's.
 * TRN_SWAP_ROW_ORDER: a round-synchronous handshake whose edges weigh their
 * slot in the dual row; maximal, so it flips more pairs than the reference.
 * TRN_SWAP_GAIN: the handshake with edges ranked by the quality their flip
 * gains, which makes better meshes than the reference. */
#define TRN_SWAP_ROW_ORDER 0
#define TRN_SWAP_GAIN 1
#define TRN_SWAP_GREEDY 2
int trn_set_swap_match(trn_mesh* mesh, int policy);
/* most coarsening or swapping levels one call runs while they still change
 * the mesh (default 100000); past it the call stops with
 * TRN_ERR_NO_PROGRESS. The reference loops without a bound
 * (coarsening.cpp:480-503, swapping.cpp:395-425). */
int trn_set_level_cap(trn_mesh* mesh, int cap);
/* Self-test of the bounded grid barrier that separates the rounds of the
 * cooperative heuristics (independent set, coloring, greedy matching): a
 * cooperative launch in which one block never arrives; the others give up
 * after max_polls polls and mark the failure, which a real call reports as
 * TRN_ERR_NO_PROGRESS. Returns TRN_ERR_NO_PROGRESS when the wait ran out
 * and was reported (the expected outcome), TRN_OK if it did not, and
 * TRN_ERR_CUDA when the device has no cooperative launch. No counterpart in
 * the reference. */
int trn_selftest_barrier(long long max_polls);

/* The solver-coupled loop: after some rounds, renumber the adapted mesh as
 * Mesh::store + Mesh::load would (io.cpp:164-255, io.cpp:53-161; live
 * vertices and elements in slot order), on the device and without the
 * 8-decimal rounding of the stored file, keeping boundary and corner tags;
 * then give the field evaluated on it (one value per vertex of
 * trn_mesh_export, in that order) and run trn_metric_run again. The
 * reference recomputes nothing between rounds (main.cpp:50); its adaptive
 * loop goes through files (README.md:8, scripts/bench_run.py:77-110).
 * trn_mesh_compact clears the field (set it before the next metric run) and
 * makes the compacted state the one trn_mesh_reload returns to. */
int trn_mesh_compact(trn_mesh* mesh);
int trn_mesh_set_solution(trn_mesh* mesh, const double* solut, int n);

/* last metric complexity (Metrics::field.complexity) */
double trn_last_complexity(trn_mesh* mesh);
/* device time of the last run call, milliseconds */
double trn_last_time_ms(trn_mesh* mesh);
/* the cudaStream_t every kernel of this mesh runs on */
void* trn_mesh_stream(trn_mesh* mesh);
/* message of the last error on this mesh ("" if none) */
const char* trn_last_error(trn_mesh* mesh);
/* Per-kernel device timing, process-wide: enable (resets the totals) or
 * disable; read back per-kernel launches, milliseconds and algorithmic bytes.
 * No counterpart in the reference (its timers are per-step wall clocks,
 * timer.h:42-48). */
int trn_profile_enable(int on);
/* time only the launches of the named kernel (NULL or "" = all): each timed
 * launch adds two events to its stream, which costs throughput */
int trn_profile_only(const char* name);
/* kernels that can count their algorithmic bytes on the device (distinct
 * entries touched, each once per launch) report those instead of the
 * launcher's figure: for profiled runs, the counting adds atomics; max_nodes
 * sizes the bitmap of distinct vertices. trn_profile_counted(i): how many of
 * entry i's launches were counted. */
int trn_profile_count_bytes(int on, int max_nodes);
int trn_profile_counted(int i);
int trn_profile_count(void);
/* kernels launched by this library since the process started */
unsigned long long trn_launch_count(void);
int trn_profile_entry(int i, char* name, int name_len, long long* launches, double* ms,
                      double* bytes);

/* Allocation-free metric recovery for one small mesh. No counterpart in the
 * reference. For callers that own all device memory themselves (a fixed
 * memory budget, or their own pool allocator) and so cannot let a library
 * call cudaMalloc/cudaFree: inputs and output are the caller's device
 * buffers (d_points[2V], d_tris[3T] 0-based CCW, d_solut[V] -> d_tensor[3V],
 * m11 m12 m22 per vertex), and the working memory is one fixed __device__
 * array of about 6 MB that every GPU loading this library holds until exit.
 * Limits: V <= TRN_NOALLOC_MAX_NODES, T <= TRN_NOALLOC_MAX_ELEMS, at most
 * TRN_NOALLOC_BUCKET triangles around a vertex; larger inputs return
 * TRN_ERR_CAPACITY. The tensors are those of trn_metric_run on the same mesh
 * with the complexity summed by its fixed-shape tree (the default; a mesh
 * set to exact_sum or replay sums in element order instead, which can differ
 * in the last bits). The first call on a device looks up the array's device
 * address and keeps it. Calls share the array:
 * calls that overlap on the GPU (other streams or host threads) race;
 * serialise them. Runs on `stream` (a cudaStream_t of the current device,
 * NULL = default stream) and returns when done. */
#define TRN_NOALLOC_MAX_NODES 16384
#define TRN_NOALLOC_MAX_ELEMS 32768
#define TRN_NOALLOC_BUCKET 32
int trn_metric_noalloc(int nb_nodes, int nb_elems, const double* d_points, const int* d_tris,
                       const double* d_solut, double target_factor, int lp_norm, double h_min,
                       double h_max, double* d_tensor, void* stream);

/* library version string */
const char* trn_version(void);

#ifdef __cplusplus
}
#endif
#endif
