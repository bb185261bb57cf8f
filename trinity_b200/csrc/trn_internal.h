/*
 * trn_internal.h — host-side launchers shared between the kernel files and the
 * C-ABI implementation. Not installed; the public interface is
 * include/trinity_b200.h.
 */
#ifndef TRN_INTERNAL_H
#define TRN_INTERNAL_H

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>
#include <string>
#include <vector>

#include "trn_common.cuh"

namespace trn {

/* the per-mesh status block: device words the kernels count into, mirrored
 * to pinned host memory at each synchronisation */
enum StatusSlot {
  S_ERR = 0,
  S_COMMIT = 1,
  S_SMOOTH_TASKS = 2,
  S_SMOOTH_COMMIT = 3,
  S_NPAIRS = 4,
  S_NINDEP = 5,
  S_COUNT = 6,     /* copy of a compaction count */
  S_PARTS = 8,     /* part offsets, 9 slots */
  S_LIVE = 18,     /* live vertices, live elements */
  S_NTASK = 20,    /* device-counted candidates of a level (free mode) */
  S_LEVEL = 21,    /* levels run by the current call */
  S_ACT = 22,      /* two activity-list counters (free mode) */
  S_FIX = 24,      /* repair-list counter (free mode) */
  S_CONT = 25,     /* 1 while another level should run */
  S_NB = 26,       /* slot counts: vertices, elements */
  S_TICK = 28,     /* seed counter */
  S_EVAL = 29,     /* statistics of the current call: examined, changed, */
  S_TASK = 30,
  S_RDONE = 31,    /* and refinement's "a level split nothing" */
  S_SIZE = 32,
};
constexpr int kLevelCoarsen = 0, kLevelSwap = 1;
constexpr int kLevelCap = 100000;

/* the decision at the end of a coarsening / swapping level, by one thread:
 * the call's statistics, the level cap, the seed counter, and whether
 * another level runs (S_CONT; also the captured loop's condition); it also
 * clears the candidate count the next level's filter appends to (no other
 * thread of the level's end reads it) */
__device__ __forceinline__ void level_end_decide(int* status, int kind, int cap,
                                                 cudaGraphConditionalHandle h, int use_h) {
  const int ntask = status[S_NTASK];
  int go;
  if (kind == kLevelCoarsen) {
    const int nindep = status[S_NINDEP];
    status[S_EVAL] += ntask;
    status[S_TASK] += nindep;
    go = ntask > 0 && nindep > 0;
  } else {
    const int commit = status[S_COMMIT];
    status[S_EVAL] += ntask;
    status[S_TASK] += commit / 2;
    go = commit > 0;
  }
  const int level = ++status[S_LEVEL];
  if (go && level > cap) {
    atomicCAS(status + S_ERR, 0, TRN_DERR_NO_PROGRESS);
    go = 0;
  }
  status[S_ACT] = status[S_ACT + 1];
  status[S_CONT] = go;
  status[S_NTASK] = 0;   /* the next level's candidate count starts empty */
  ++*reinterpret_cast<unsigned*>(status + S_TICK);
  if (use_h) cudaGraphSetConditional(h, go);
}

/* the stencil repair of the listed vertices fused with the level's end (the
 * two touch disjoint state): one launch instead of two per level */
void fix_list_level_end(const DMesh& m, const int* list, const int* count, long long bound, int* status,
                        int kind, int cap, const int* next, int* cur, int hint, cudaStream_t s,
                        cudaGraphConditionalHandle h, bool use_h);



/* launch shapes the autotuner (trn_autotune) chooses; none of them changes
 * a result. The defaults are the tuner's choice on the 2M-triangle workload
 * in FP64 (the smoothing by 2 lanes a vertex in 256-thread blocks, the five
 * back-off tries in one sweep). Each mesh keeps
 * its own table; the C-ABI entry that drives a mesh makes it the calling
 * thread's table for the launchers. */
struct Tune {
  int smooth_threads = 256;   /* k_smooth_move block: 64, 128, 256 */
  int filter_threads = 128;   /* one-lane collapse-target search block: 128, 256, 512 */
  int group_lanes = 16;       /* lanes per vertex of the grouped search: 1 (one-lane search), 4, 8, 16 */
  int group_max = 16384;      /* longest level list the grouped search takes */
  int flip_threads = 256;     /* k_swap_flip block: 128, 256, 512 */
  int smooth_lanes = 2;       /* lanes per smoothed vertex: 1, 2, 4, 8 */
  int smooth_regs = 7;        /* smoothing registers: 0 up to 128, 1 capped at 80 (three 256-thread
                                 blocks an SM), 2 at 64 (four), 3 at 64 with the grouped form's
                                 element metrics in shared memory; 4, 5, 6: the grouped form's
                                 five tries in one sweep, capped at 64, 80, 128; 7, 8: the sweep
                                 with the element metrics in shared memory, capped at 128, 80 */
  bool operator==(const Tune& o) const {
    return smooth_threads == o.smooth_threads && filter_threads == o.filter_threads &&
           group_lanes == o.group_lanes && group_max == o.group_max && flip_threads == o.flip_threads &&
           smooth_lanes == o.smooth_lanes && smooth_regs == o.smooth_regs;
  }
};
const Tune& tune();
void set_thread_tune(const Tune* t);

/* grid for a grid-stride kernel over n items: a multiple of the SM count */
int grid_for(long long n, int threads = TRN_THREADS);
/* grid for a kernel over a device-counted list: sized for `bound` items (an
 * upper bound the host knows, < 0 = unknown) and at most `cap`; the kernels
 * stride over the true count, so the bound only sizes the launch */
int grid_bounded(long long bound, long long cap, int threads = TRN_THREADS);
/* grid capped at the blocks of `kernel` resident at once (one wave) */
int grid_resident(const void* kernel, int threads, int grid, size_t smem = 0);
#define TRN_RESIDENT(kern, grid, threads) grid_resident(reinterpret_cast<const void*>(kern), (threads), (grid))

/* scratch used by the scans: tile sums of up to max_n items */
struct ScanWs {
  long long* tile = nullptr;   /* per-tile sums / offsets */
  int* count = nullptr;        /* device total (compaction) */
  long long* total = nullptr;  /* device total (scan) */
  int max_tiles = 0;
};
void scan_ws_alloc(ScanWs* ws, long long max_n);
void scan_ws_free(ScanWs* ws);

/* exclusive scan of n int64 values; *ws.total receives the sum. With dn,
 * the count is *dn (read on the device, at most n) */
void scan_i64(const long long* in, long long* out, int n, ScanWs& ws, cudaStream_t s,
              const int* dn = nullptr);
/* ordered compaction: list[k] = i for the k-th i < n with flags[i] != 0;
 * *ws.count receives the number kept */
void compact_u8(const uint8_t* flags, int n, int* list, ScanWs& ws, cudaStream_t s);

/* mesh files (mesh_io.cu): an input mesh as loaded (0-based triangles,
 * boundary / corner tags) */
struct MeshInput {
  long nv = 0, nt = 0;
  std::vector<double> pts;
  std::vector<int> tris;
  std::vector<uint8_t> tags;
};
bool read_file(const char* path, std::vector<char>* buf);
/* 0: parsed; 1: malformed (*err says why); -1: not one record per line,
 * read it token by token instead */
int parse_mesh_text(const std::vector<char>& buf, MeshInput* out, std::string* err);
int parse_bb_text(const std::vector<char>& buf, long nv, std::vector<double>* u, std::string* err);
bool is_binary_mesh(const std::vector<char>& buf);
int parse_mesh_binary(const std::vector<char>& buf, MeshInput* out, std::string* err);
int write_mesh_binary(const char* path, long nv, long nt, const double* pts, const uint8_t* tags,
                      const int* tris);

/* topology (topology.cu) */
void build_stencils(const DMesh& m, int nb_nodes, int nb_elems, cudaStream_t s);
void build_vicin(const DMesh& m, int nb_nodes, bool only_flagged, cudaStream_t s);
void fix_tagged(const DMesh& m, int nb_nodes, cudaStream_t s);
void flag_all_alive(const DMesh& m, int nb_nodes, cudaStream_t s);
void quality_all(const DMesh& m, int nb_elems, bool fp32, cudaStream_t s);
/* recompute the per-vertex tensor-logarithm cache of the FP64 or FP32 form */
void log_cache(const DMesh& m, int nb_nodes, bool fp32, cudaStream_t s);
void count_live(const DMesh& m, int nb_nodes, int nb_elems, int* out, cudaStream_t s);
void expand_tris(const int* raw, int nb_elems, int nb_nodes, int4* out, int* err, cudaStream_t s);
void pack_nodes(const DMesh& m, const int* list, const int* count, int* newid, double* pts, double* ten,
                cudaStream_t s);
void flag_live_tris(const DMesh& m, int nb_elems, uint8_t* flag, cudaStream_t s);
/* the listed live vertices (points, tags) and elements (renumbered through
 * newid) packed as a load would place them */
void pack_nodes_load(const DMesh& m, const int* list, const int* count, int* newid, double2* pts,
                     uint8_t* tags, cudaStream_t s);
void pack_tris_load(const DMesh& m, const int* list, const int* count, const int* newid, int4* out,
                    cudaStream_t s);
void pack_tris(const DMesh& m, const int* list, const int* count, const int* newid, int* out,
               cudaStream_t s);

/* metric (metric.cu) */
struct MetricParams {
  double target;      /* floor(V * target_factor) */
  double scale_exp;   /* -1/(2p+2) or 0.5 */
  double eig_min;     /* 1/h_min^2 */
  double eig_max;     /* 1/h_max^2 */
};
/* optional copies of the recovery's intermediates (any may be null): the
 * patch areas, the symmetrised Hessians and the locally normalised tensors */
struct MetricSaves {
  double* atot = nullptr;
  double4* hsym = nullptr;
  double4* mloc = nullptr;
};
/* fp32: the mixed-precision form's recovery (FP32 patch means with FP64
 * coordinate and value differences, FP32 normalisations, FP64 complexity
 * sum; writes the FP32 tensor copy and logarithm cache too) */
void metric_run(const DMesh& m, int nb_nodes, int nb_elems, const double* solut,
                double2* grad, double* terms, double* complexity, bool exact_sum,
                const MetricParams& p, cudaStream_t s, const MetricSaves* keep = nullptr,
                bool fp32 = false);
/* deterministic two-level sum of n doubles; partial holds grid_for(n) slots */
void sum_tree(const double* in, int n, double* partial, double* out, cudaStream_t s);

/* refinement (refine.cu) */
struct RefineWs {
  int4* info = nullptr;            /* per element: masks, opp[3] */
  long long* cnt = nullptr;        /* per element: pushes << 32 | pattern */
  long long* off = nullptr;        /* exclusive scan of cnt */
  unsigned long long* hkey = nullptr; /* (min,max) -> steiner id */
  int* hval = nullptr;
  unsigned long long hcap = 0;     /* power of two */
};
void refine_ws_alloc(RefineWs* ws, int capa_node, int capa_elem);
void refine_ws_free(RefineWs* ws);
void refine_reset_hash(RefineWs& ws, cudaStream_t s);
void refine_filter(const DMesh& m, int nb_elems, RefineWs& ws, bool fp32, cudaStream_t s);
void refine_apply(const DMesh& m, int nb_nodes, int nb_elems, RefineWs& ws, bool fp32, cudaStream_t s);
/* one refinement level driven by the device counts (m.nb): filter, scan,
 * capacity check, splits, new counts; hints size the grids (at least the
 * counts); stats: examined, added, done */
void refine_level(const DMesh& m, int hint_nodes, int hint_elems, RefineWs& ws, ScanWs& scan,
                  int* stats, bool fp32, cudaStream_t s);

/* coarsening (coarsen.cu) */
/* with act: the active vertices onto the list act too (*act_n their count) */
void coarsen_pre(const DMesh& m, int nb_nodes, cudaStream_t s, int* act = nullptr, int* act_n = nullptr);
void coarsen_filter(const DMesh& m, int nb_nodes, int* target, uint8_t* flag, bool fp32, cudaStream_t s);
void collapse(const DMesh& m, const int* indep, const int* count, const int* target,
              const uint8_t* cand_flag, cudaStream_t s, long long bound = -1);
/* free mode, per level, over the list of active vertices (coarsen_pre lists
 * them first): adjacency + target + unordered candidate append in one pass */
void coarsen_filter_append(const DMesh& m, const int* act, const int* act_n, int* target, int* cand,
                           int* count, uint8_t* state, bool fp32, cudaStream_t s,
                           long long bound = -1);

/* swapping (swap.cu) */
/* with act: the live elements onto the list act too (*act_n their count) */
void swap_init(const DMesh& m, int nb_nodes, int nb_elems, int* map, bool fp32, cudaStream_t s,
               int* act = nullptr, int* act_n = nullptr);
void swap_filter(const DMesh& m, int nb_elems, uint8_t* flag, cudaStream_t s);
void swap_dual(const DMesh& m, const int* list, int ntasks, int* dual, int* dual_n, int* map,
               cudaStream_t s);
void swap_flip(const DMesh& m, const int* pairs, const int* npairs, const int* map,
               const int* dual, const int* dual_n, const int* ntasks, int* commit, bool strict_map,
               bool fp32, cudaStream_t s, long long bound = -1);
/* free mode, per level: filter and dual rows in one pass over the list of
 * active elements (swap_init lists them first), *count rows; when rank is
 * given, rank[4 r + e]: the gain rank of the flip between row r's candidate
 * and its neighbour e */
/* the greedy swap matching's per-element state, reset by the dual filter for
 * the elements of the rows it builds (vis -1, both key buffers ~0), so the
 * matching needs no reset pass; all null when another matching runs */
struct GreedyReset {
  int* vis = nullptr;
  unsigned long long* mk0 = nullptr;
  unsigned long long* mk1 = nullptr;
};
void swap_filter_dual(const DMesh& m, const int* act, const int* act_n, int* dual, int* dual_n,
                      int* map, uint32_t* rank, int* count, bool fp32, cudaStream_t s,
                      long long bound = -1, GreedyReset gr = GreedyReset(), int* flips = nullptr);

/* smoothing (smooth.cu) */
void smooth_pre(const DMesh& m, int nb_nodes, cudaStream_t s);
void smooth_color(const DMesh& m, const int* list, int n, int* counters, bool fp32, cudaStream_t s);
/* the same over color class c of a device-side partition (parts, part_off);
 * hint: grid size, at least the class size */
void smooth_class(const DMesh& m, const int* parts, const int* part_off, int c, int hint, int* counters,
                  bool fp32, cudaStream_t s);

/* graph heuristics, free mode (heuristics.cu) */
struct HeurWs {
  uint8_t* state = nullptr;      /* per vertex / element */
  uint8_t* state2 = nullptr;     /* second buffer of the independent-set rounds */
  unsigned long long* prop = nullptr;
  unsigned long long* prop2 = nullptr;   /* second key buffer of the greedy matching */
  int* choice = nullptr;
  int* choice2 = nullptr;                /* second row list of the greedy matching */
  int* color = nullptr;
  uint8_t* tent = nullptr;       /* the coloring's tentative colors, two buffers of capa_node */
  int* mate = nullptr;
  uint32_t* rank = nullptr;      /* four flip ranks per swap dual row */
  int* cnt = nullptr;            /* small device counters */
  int* color_keys = nullptr;     /* counts and cursors of the coloring's (color, degree) keys */
  int* list_a = nullptr;         /* two worklists (activity, coloring) */
  int* list_b = nullptr;
  int* fix_list = nullptr;       /* vertices tagged for repair */
};
void heur_ws_alloc(HeurWs* ws, int capa_node, int capa_elem);
/* the cooperative kernels' bounded grid barrier made to give up (one block
 * never arrives): *gave_up when the waiting blocks marked the failure */
cudaError_t barrier_selftest(long long max_polls, int* gave_up);
void heur_ws_free(HeurWs* ws);
/* handshake matching on the dual rows (*ntasks of them), edges ranked by
 * their slot in the row (rank == nullptr) or by rank[4 i + slot] (the flip
 * gains of swap_filter_dual); pairs[2k], pairs[2k+1]; *npairs */
void match_handshake(const DMesh& m, int nb_elems, const int* dual, const int* dual_n,
                     const int* ntasks, const int* map, const uint32_t* rank, Seed seed, HeurWs& ws,
                     int* pairs, int* npairs, cudaStream_t s, long long bound = -1);
/* the reference's greedy matching loop over the dual rows, in the order
 * (candidate id mod 4, candidate id), computed exactly by rounds of rows that
 * come first on all their elements; pairs as match_handshake */
void match_greedy(const DMesh& m, int nb_elems, const int* dual, const int* dual_n, const int* ntasks,
                  const int* map, HeurWs& ws, int* pairs, int* npairs, cudaStream_t s,
                  long long bound = -1);
/* a fixed number of independent-set rounds over a device-counted candidate
 * list; undecided candidates are re-activated (next level) */
void mis_jp_rounds(const DMesh& m, const int* cand, const int* count, int rounds, Seed seed,
                   HeurWs& ws, int* indep, int* nindep, cudaStream_t s, long long bound = -1);
/* speculative first-fit coloring of interior vertices (tentative colors,
 * priority conflicts resolved round by round), colors 1..max_col;
 * parts: vertex ids grouped by color, part_off[c] offsets (c = 0..max_col).
 * hint: grid size (at least the vertex count). color_jp runs batches of 8
 * rounds while vertices wait (at most 8 batches), reading the decision back
 * after each; a captured round runs color_batch inside a loop node instead.
 * color_finish advances *tick (the seeds' counter). */
void color_jp(const DMesh& m, int hint, int max_col, Seed seed, HeurWs& ws, int* parts,
              int* part_off, unsigned* tick, cudaStream_t s);
void color_begin(const DMesh& m, int hint, HeurWs& ws, cudaStream_t s);
void color_batch(const DMesh& m, int hint, int max_col, Seed seed, HeurWs& ws, cudaStream_t s,
                 cudaGraphConditionalHandle h, bool use_h);
void color_finish(const DMesh& m, int hint, int max_col, HeurWs& ws, int* parts, int* part_off,
                  unsigned* tick, cudaStream_t s);
int* color_cont(HeurWs& ws);

/* element-quality functional and its adjoint (adjoint.cu) */
struct AdjWs {
  int cap_v = 0, cap_e = 0;
  double4* ten = nullptr;    /* metric recovered from the solution */
  double4* lten = nullptr;   /* its logarithms (double4, or float4 in the FP32 form) */
  double4* mloc = nullptr;   /* locally normalised tensors */
  double4* hsym = nullptr;   /* symmetrised Hessians */
  double* atot = nullptr;    /* 2-ring patch areas */
  double* astar = nullptr;   /* stencil areas */
  double* q = nullptr;       /* per element quality (+ sum partials) */
  double* egp = nullptr;     /* per element point partials (6) */
  double* egl = nullptr;     /* per element log-tensor partials (3) */
  double* vbuf = nullptr;    /* per vertex scratch (8 doubles) */
  double* ebuf = nullptr;    /* per element scratch (4 doubles) */
  double* vfact = nullptr;   /* per vertex share of dJ/d(global scale) (+ partials) */
  double* scal = nullptr;    /* [0] complexity, [1] J, [2] dJ/d(global scale) */
};
int adj_ws_ensure(AdjWs* ws, int nv, int ne);
void adj_ws_free(AdjWs* ws);
/* the metric of the functional recovered from a nodal solution */
struct AdjMetric {
  const double* solut;
  double2* grad;       /* recovered-gradient scratch (per vertex) */
  double* terms;       /* complexity terms (capa_elem + partial slots) */
  bool exact_sum;
  MetricParams p;
};
/* J -> ws.scal[1]; gxy (2 per vertex) and gu (per vertex) may be null; um
 * null: the metric is the mesh's own tensors */
void quality_adjoint(const DMesh& m, int nb_nodes, int nb_elems, const double2* xy,
                     const AdjMetric* um, bool fp32, AdjWs& ws, double* gxy, double* gu,
                     cudaStream_t s);
void smooth_gradient_color(const DMesh& m, const int* list, int n, double max_len, int mode,
                           int* counters, bool fp32, cudaStream_t s);

void check_launch(const char* what);

/* per-launch device timing (prof.cu): brackets the launches issued during its
 * lifetime with events on stream s when profiling is enabled; bytes is the
 * launcher's algorithmic byte count for them */
/* where a counting kernel adds its algorithmic bytes (bytes == nullptr: not
 * counting) and the zeroed bitmap it marks distinct vertices in */
struct ByteCount {
  unsigned long long* bytes = nullptr;
  unsigned* seen = nullptr;
};

class ProfScope {
 public:
  /* count: filled when the profiler counts bytes (trn_profile_count_bytes);
   * the launcher hands it to its kernel */
  ProfScope(const char* name, cudaStream_t s, double bytes = 0.0, ByteCount* count = nullptr);
  ~ProfScope();
  ProfScope(const ProfScope&) = delete;
  ProfScope& operator=(const ProfScope&) = delete;

 private:
  cudaStream_t stream_;
  cudaEvent_t a_ = nullptr;
  int id_ = -1;
  int slot_ = -1;
  double bytes_ = 0.0;
};
void prof_flush();
/* count of kernel launches issued by this library (process-wide) */
void note_launch();
void note_launches(unsigned long long n);
/* launches issued by the calling host thread */
unsigned long long thread_launches();

/* algorithmic sizes (bytes per entity) used by the launchers' byte counts:
 * point 2 x f64, tensor 3 x f64, triangle 3 x i32, quality f64, stencil and
 * adjacency entries i32; planar triangulations average 6 elements and 6
 * neighbours per vertex */
constexpr double kPt = 16, kTen = 24, kTri = 12, kQ = 8, kIdx = 4, kAvgDeg = 6;

}  // namespace trn

#endif
