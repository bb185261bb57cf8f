/*
 * trn_api.cu — host orchestration and the C ABI (include/trinity_b200.h).
 *
 * The control flow of each run() mirrors the reference's kernel drivers
 * (Refine::run refinement.cpp:445-493, Coarse::run coarsening.cpp:463-508,
 * Swap::run swapping.cpp:383-428, Smooth::run smoothing.cpp:274-302); the
 * loops whose trip count depends on the data read one small status block back
 * from the device per level (pinned memory, one stream synchronisation).
 */
#include "trn_internal.h"
#include "trn_libm.h"
#include "../../include/trinity_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

using namespace trn;

namespace {

/* host-only part of the pinned status mirror (after the device block) */
enum {
  H_WIDE = 40,     /* host-only pinned slot for one 8-byte value */
  H_STATS = 48,    /* a captured round's statistics, 8 slots */
  H_SIZE = 64,
};

constexpr int kLoopCap = kLevelCap;
constexpr int kMisRounds = 8;   /* independent-set rounds per coarsening level (free mode) */

}  // namespace

struct trn_mesh {
  int nb_nodes = 0, nb_elems = 0;
  int size0[2] = {0, 0};
  int capa_node = 0, capa_elem = 0, bucket = 64, depth = 1, verb = 0, rounds = 1;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  DMesh d{};
  double* solut = nullptr;
  double2* grad = nullptr;
  double* terms = nullptr;
  double* complexity = nullptr;
  int* target = nullptr;
  uint8_t* flag = nullptr;
  int* list = nullptr;
  int* indep = nullptr;
  int* map = nullptr;
  int* dual = nullptr;
  int* dual_n = nullptr;
  int* pairs = nullptr;
  int* parts = nullptr;
  unsigned char* stage = nullptr;   /* transfer staging: max(24 B/vertex, 12 B/element) */
  int* status = nullptr;
  int* h_status = nullptr;
  /* the last loaded input, kept on the device for trn_mesh_reload */
  double2* pts0 = nullptr;
  int4* tri0 = nullptr;
  uint8_t* tags0 = nullptr;
  int n0_nodes = 0, n0_elems = 0;
  ScanWs scan;
  RefineWs rws;
  HeurWs hws;
  AdjWs adj;
  /* a captured free-mode round (trn_round_graph_run) and what it was captured for */
  cudaGraphExec_t round_exec = nullptr;
  cudaStream_t body_stream = nullptr;   /* captures the loop bodies */
  int* rstats = nullptr;                /* device: examined / changed per stage */
  int round_depth = 0;
  Tune tune;                /* launch shapes (trn_autotune) */
  Tune round_tune;
  bool round_fp32 = false;
  /* the cached element qualities equal a recomputation of every live
   * element: set by a swap or smoothing call that ended without error,
   * cleared by every other call that can change points, tensors, elements
   * or the arithmetic form (all stage calls clear it as they begin) */
  bool qual_fresh = false;
  uint64_t round_seed = 0;
  int round_swap_match = 0;
  int round_level_cap = 0;
  unsigned long long round_launches = 0;
  /* replay */
  bool replay = false;
  std::vector<int32_t> log;
  int32_t* d_log = nullptr;
  size_t cursor = 0;
  /* options */
  uint64_t seed = 0x7472696e697479ULL;
  bool exact_sum = false;
  int swap_match = TRN_SWAP_GREEDY;
  int level_cap = kLoopCap;   /* coarsening / swapping levels per call */
  bool fp32 = false;   /* mixed-precision form of the metric arithmetic */
  double last_complexity = 0.0;
  double last_ms = 0.0;
  std::string err;
};

namespace {

int fail(trn_mesh* m, int code, const std::string& msg) {
  if (m) m->err = msg;
  return code;
}

#define CK(call)                                                                 \
  do {                                                                           \
    cudaError_t e_ = (call);                                                     \
    if (e_ != cudaSuccess)                                                       \
      return fail(m, TRN_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

/* copy the status block (and optionally one compaction count) back and sync */
int sync_status(trn_mesh* m, const int* count = nullptr) {
  CK(cudaMemcpyAsync(m->h_status, m->status, sizeof(int) * S_SIZE, cudaMemcpyDeviceToHost, m->stream));
  if (count)
    CK(cudaMemcpyAsync(m->h_status + S_COUNT, count, sizeof(int), cudaMemcpyDeviceToHost, m->stream));
  CK(cudaStreamSynchronize(m->stream));
  CK(cudaGetLastError());
  prof_flush();
  int e = m->h_status[S_ERR];
  if (e) {
    const char* what = e == TRN_DERR_CAPACITY      ? "vertex or element capacity exceeded"
                       : e == TRN_DERR_BUCKET      ? "a vertex has more triangles than the stencil bucket"
                       : e == TRN_DERR_HASH        ? "refinement edge table full"
                       : e == TRN_DERR_REPLAY      ? "replay log does not match the mesh"
                       : e == TRN_DERR_NO_PROGRESS ? "level cap reached"
                                                   : "invalid state";
    return fail(m, (e == TRN_DERR_CAPACITY || e == TRN_DERR_BUCKET || e == TRN_DERR_HASH) ? TRN_ERR_CAPACITY
                   : e == TRN_DERR_REPLAY      ? TRN_ERR_REPLAY
                   : e == TRN_DERR_NO_PROGRESS ? TRN_ERR_NO_PROGRESS : TRN_ERR_INVALID,
                std::string("device: ") + what);
  }
  return TRN_OK;
}

void begin_timing(trn_mesh* m) {
  m->qual_fresh = false;
  set_thread_tune(&m->tune);
  cudaEventRecord(m->ev0, m->stream);
}

int end_timing(trn_mesh* m, trn_stats* st, int eval, int task) {
  cudaEventRecord(m->ev1, m->stream);
  CK(cudaEventSynchronize(m->ev1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, m->ev0, m->ev1);
  m->last_ms = ms;
  if (st) {
    st->eval += eval;
    st->task += task;
    st->elap += (int) ms;
  }
  return TRN_OK;
}

/* next replay entry: checks the tag, returns the payload offset and count */
int replay_take(trn_mesh* m, int tag, size_t* payload, int* n) {
  if (m->cursor + 2 > m->log.size() || m->log[m->cursor] != tag)
    return fail(m, TRN_ERR_REPLAY, "replay log: expected entry " + std::to_string(tag) +
                                       " at " + std::to_string(m->cursor));
  *n = m->log[m->cursor + 1];
  *payload = m->cursor + 2;
  size_t len = 0;
  if (tag == 1) len = (size_t) *n;
  else if (tag == 2) len = 2 * (size_t) *n;
  else {
    size_t p = *payload;
    for (int c = 0; c < *n; ++c) {
      if (p >= m->log.size()) return fail(m, TRN_ERR_REPLAY, "replay log truncated");
      p += 1 + (size_t) m->log[p];
    }
    len = p - *payload;
  }
  if (*payload + len > m->log.size()) return fail(m, TRN_ERR_REPLAY, "replay log truncated");
  m->cursor = *payload + len;
  return TRN_OK;
}

template <typename T>
int dmalloc(trn_mesh* m, T** p, size_t count) {
  CK(cudaMalloc((void**) p, sizeof(T) * (count ? count : 1)));
  return TRN_OK;
}

void release(trn_mesh* m) {
  if (!m) return;
  if (m->stream) cudaStreamSynchronize(m->stream);
  void* bufs[] = {m->d.pts, m->d.ten, m->d.lten, m->d.tenf, m->d.tri, m->d.stenc, m->d.deg, m->d.vic, m->d.vdeg,
                  m->d.tags, m->d.alive, m->d.fixes, m->d.activ, m->d.qual, m->solut, m->grad,
                  m->terms, m->complexity, m->target, m->flag, m->list, m->indep, m->map,
                  m->dual, m->dual_n, m->pairs, m->parts, m->stage, m->status, m->d_log, m->pts0,
                  m->tri0, m->tags0};
  for (void* b : bufs) if (b) cudaFree(b);
  if (m->h_status) cudaFreeHost(m->h_status);
  scan_ws_free(&m->scan);
  refine_ws_free(&m->rws);
  heur_ws_free(&m->hws);
  adj_ws_free(&m->adj);
  if (m->round_exec) cudaGraphExecDestroy(m->round_exec);
  if (m->body_stream) cudaStreamDestroy(m->body_stream);
  if (m->rstats) cudaFree(m->rstats);
  if (m->ev0) cudaEventDestroy(m->ev0);
  if (m->ev1) cudaEventDestroy(m->ev1);
  if (m->stream) cudaStreamDestroy(m->stream);
}

/* ---------------- file parsing (io.cpp:25-161) ---------------- */
struct Reader {
  std::vector<char> buf;
  size_t pos = 0;
  void skip_ws() {
    while (pos < buf.size() && (buf[pos] == ' ' || buf[pos] == '\t' || buf[pos] == '\n' || buf[pos] == '\r'))
      ++pos;
  }
  /* io::find: next line whose first token is key; returns the count after it */
  long find(const char* key) {
    size_t klen = std::strlen(key);
    while (pos < buf.size() - 1) {
      size_t eol = pos;
      while (eol < buf.size() - 1 && buf[eol] != '\n') ++eol;
      size_t s = pos;
      while (s < eol && (buf[s] == ' ' || buf[s] == '\t' || buf[s] == '\r')) ++s;
      bool hit = (buf[s] != '#' && buf[s] != '%') && eol - s >= klen &&
                 std::strncmp(&buf[s], key, klen) == 0 &&
                 (s + klen == eol || buf[s + klen] == ' ' || buf[s + klen] == '\t' || buf[s + klen] == '\r');
      pos = eol < buf.size() - 1 ? eol + 1 : eol;
      if (hit) {
        long c = -1;
        if (next_long(&c)) return c;
        return -1;
      }
    }
    return -1;
  }
  bool next_long(long* v) {
    skip_ws();
    if (pos >= buf.size() - 1) return false;
    char* end = nullptr;
    long x = std::strtol(&buf[pos], &end, 10);
    if (end == &buf[pos]) return false;
    pos = (size_t) (end - buf.data());
    *v = x;
    return true;
  }
  bool next_double(double* v) {
    skip_ws();
    if (pos >= buf.size() - 1) return false;
    char* end = nullptr;
    double x = std::strtod(&buf[pos], &end);
    if (end == &buf[pos]) return false;
    pos = (size_t) (end - buf.data());
    *v = x;
    return true;
  }
  void skip_line() {
    while (pos < buf.size() - 1 && buf[pos] != '\n') ++pos;
    if (pos < buf.size() - 1) ++pos;
  }
};

}  // namespace

/* ======================================================================== */
extern "C" {

const char* trn_version(void) { return "trinity_b200 0.1 (sm_100a)"; }

int trn_mesh_create_ex(const int size[2], int bucket, int depth, int verbosity, int rounds,
                       int capa_scale, trn_mesh** out) {
  if (!out || !size || size[0] <= 0 || size[1] <= 0 || bucket < 8 || bucket > TRN_MAX_DEG ||
      depth < 1 || capa_scale < 1)
    return TRN_ERR_INVALID;
  *out = nullptr;
  trn_mesh* m = new trn_mesh();
  m->size0[0] = size[0];
  m->size0[1] = size[1];
  m->bucket = bucket;
  m->depth = depth;
  m->verb = verbosity;
  m->rounds = rounds;
  m->capa_node = (int) std::min<long long>((long long) size[0] * capa_scale, 1LL << 30);
  m->capa_elem = (int) std::min<long long>((long long) size[1] * capa_scale, 1LL << 30);
  const size_t cn = (size_t) m->capa_node, ce = (size_t) m->capa_elem;
  int rc = TRN_OK;
  auto bail = [&](int code) {
    release(m);
    delete m;
    return code;
  };
  if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(TRN_ERR_CUDA);
  cudaEventCreate(&m->ev0);
  cudaEventCreate(&m->ev1);
  DMesh& d = m->d;
  d.bucket = bucket;
  d.capa_node = m->capa_node;
  d.capa_elem = m->capa_elem;
  if ((rc = dmalloc(m, &d.pts, cn)) || (rc = dmalloc(m, &d.ten, cn)) || (rc = dmalloc(m, &d.lten, cn)) ||
      (rc = dmalloc(m, &d.tenf, cn)) ||
      (rc = dmalloc(m, &d.tri, ce)) ||
      (rc = dmalloc(m, &d.stenc, cn * bucket)) || (rc = dmalloc(m, &d.deg, cn)) ||
      (rc = dmalloc(m, &d.vic, cn * bucket)) || (rc = dmalloc(m, &d.vdeg, cn)) ||
      (rc = dmalloc(m, &d.tags, cn)) || (rc = dmalloc(m, &d.alive, cn)) ||
      (rc = dmalloc(m, &d.fixes, cn + 16)) || (rc = dmalloc(m, &d.activ, std::max(cn, ce) + 16)) ||
      (rc = dmalloc(m, &d.qual, ce)) || (rc = dmalloc(m, &m->solut, cn)) ||
      (rc = dmalloc(m, &m->grad, cn)) || (rc = dmalloc(m, &m->terms, ce + 8192)) ||
      (rc = dmalloc(m, &m->complexity, 2)) || (rc = dmalloc(m, &m->target, cn)) ||
      (rc = dmalloc(m, &m->flag, std::max(cn, ce))) || (rc = dmalloc(m, &m->list, std::max(cn, ce))) ||
      (rc = dmalloc(m, &m->indep, cn)) || (rc = dmalloc(m, &m->map, ce)) ||
      (rc = dmalloc(m, &m->dual, ce * 4)) || (rc = dmalloc(m, &m->dual_n, ce)) ||
      (rc = dmalloc(m, &m->pairs, ce * 2)) || (rc = dmalloc(m, &m->parts, cn)) ||
      (rc = dmalloc(m, &m->stage, std::max(24 * cn, 12 * ce))) ||
      (rc = dmalloc(m, &m->status, S_SIZE)))
    return bail(rc);
  d.err = m->status + S_ERR;
  d.nb = m->status + S_NB;
  if (cudaMallocHost(&m->h_status, sizeof(int) * H_SIZE) != cudaSuccess) return bail(TRN_ERR_CUDA);
  scan_ws_alloc(&m->scan, (long long) std::max(cn, ce));
  refine_ws_alloc(&m->rws, m->capa_node, m->capa_elem);
  heur_ws_alloc(&m->hws, m->capa_node, m->capa_elem);
  if (cudaGetLastError() != cudaSuccess) return bail(TRN_ERR_CUDA);
  *out = m;
  return TRN_OK;
}

int trn_mesh_create(const int size[2], int bucket, int depth, int verbosity, int rounds,
                    trn_mesh** out) {
  int scale = std::max(3 * (depth - 1), 4);
  return trn_mesh_create_ex(size, bucket, depth, verbosity, rounds, scale, out);
}

int trn_mesh_destroy(trn_mesh* m) {
  if (!m) return TRN_ERR_INVALID;
  release(m);
  delete m;
  return TRN_OK;
}

/* state of a freshly loaded mesh from the device copies pts0/tri0/tags0 */
static int init_from_device(trn_mesh* m) {
  DMesh& d = m->d;
  const size_t cn = (size_t) m->capa_node, ce = (size_t) m->capa_elem, b = (size_t) m->bucket;
  const int nb_nodes = m->n0_nodes, nb_elems = m->n0_elems;
  cudaStream_t s = m->stream;
  CK(cudaMemsetAsync(d.ten, 0, sizeof(double4) * cn, s));
  CK(cudaMemsetAsync(d.lten, 0, sizeof(double4) * cn, s));
  CK(cudaMemsetAsync(d.pts, 0, sizeof(double2) * cn, s));
  CK(cudaMemsetAsync(d.tri, 0xff, sizeof(int4) * ce, s));
  CK(cudaMemsetAsync(d.stenc, 0xff, sizeof(int) * cn * b, s));
  CK(cudaMemsetAsync(d.vic, 0xff, sizeof(int) * cn * b, s));
  CK(cudaMemsetAsync(d.vdeg, 0, sizeof(int) * cn, s));
  CK(cudaMemsetAsync(d.tags, 0, cn, s));
  CK(cudaMemsetAsync(d.alive, 1, cn, s));
  CK(cudaMemsetAsync(d.fixes, 0, cn, s));
  CK(cudaMemsetAsync(d.activ, 0, std::max(cn, ce), s));
  CK(cudaMemsetAsync(d.qual, 0, sizeof(double) * ce, s));
  CK(cudaMemsetAsync(m->status, 0, sizeof(int) * S_SIZE, s));
  const int counts[2] = {nb_nodes, nb_elems};
  CK(cudaMemcpyAsync(m->status + S_NB, counts, sizeof(counts), cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(m->map, 0xff, sizeof(int) * ce, s));
  CK(cudaMemcpyAsync(d.pts, m->pts0, sizeof(double2) * (size_t) nb_nodes, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(d.tri, m->tri0, sizeof(int4) * (size_t) nb_elems, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(d.tags, m->tags0, (size_t) nb_nodes, cudaMemcpyDeviceToDevice, s));
  m->nb_nodes = nb_nodes;
  m->nb_elems = nb_elems;
  m->cursor = 0;
  build_stencils(d, nb_nodes, nb_elems, s);
  build_vicin(d, nb_nodes, false, s);
  return sync_status(m);
}

int trn_mesh_load_arrays(trn_mesh* m, int nb_nodes, int nb_elems, const double* points,
                         const int* tris, const uint8_t* tags, const double* solut) {
  if (m) m->qual_fresh = false;
  if (!m || !points || !tris || nb_nodes <= 0 || nb_elems <= 0) return fail(m, TRN_ERR_INVALID, "load: bad arguments");
  if (nb_nodes > m->capa_node || nb_elems > m->capa_elem)
    return fail(m, TRN_ERR_CAPACITY, "load: mesh larger than the capacity");
  cudaStream_t s = m->stream;
  if (nb_nodes > m->n0_nodes || nb_elems > m->n0_elems || !m->pts0) {
    cudaFree(m->pts0);
    cudaFree(m->tri0);
    cudaFree(m->tags0);
    m->pts0 = nullptr;
    m->tri0 = nullptr;
    m->tags0 = nullptr;
    int rc;
    if ((rc = dmalloc(m, &m->pts0, (size_t) nb_nodes)) || (rc = dmalloc(m, &m->tri0, (size_t) nb_elems)) ||
        (rc = dmalloc(m, &m->tags0, (size_t) nb_nodes)))
      return rc;
  }
  /* the triangles travel as given (3 ints each) and are checked and widened
   * to int4 records on the device; points are already x,y interleaved */
  CK(cudaMemsetAsync(m->status, 0, sizeof(int) * S_SIZE, s));
  CK(cudaMemcpyAsync(m->stage, tris, sizeof(int) * 3 * (size_t) nb_elems, cudaMemcpyHostToDevice, s));
  expand_tris(reinterpret_cast<const int*>(m->stage), nb_elems, nb_nodes, m->tri0, m->status + S_ERR, s);
  CK(cudaMemcpyAsync(m->pts0, points, sizeof(double) * 2 * (size_t) nb_nodes, cudaMemcpyHostToDevice, s));
  if (tags) CK(cudaMemcpyAsync(m->tags0, tags, (size_t) nb_nodes, cudaMemcpyHostToDevice, s));
  else CK(cudaMemsetAsync(m->tags0, 0, (size_t) nb_nodes, s));
  if (solut) CK(cudaMemcpyAsync(m->solut, solut, sizeof(double) * (size_t) nb_nodes, cudaMemcpyHostToDevice, s));
  else CK(cudaMemsetAsync(m->solut, 0, sizeof(double) * (size_t) nb_nodes, s));
  int rc = sync_status(m);
  if (rc) {
    m->n0_nodes = m->n0_elems = 0;
    return fail(m, TRN_ERR_INVALID, "load: vertex index out of range");
  }
  m->n0_nodes = nb_nodes;
  m->n0_elems = nb_elems;
  return init_from_device(m);
}

int trn_mesh_reload(trn_mesh* m) {
  if (m) m->qual_fresh = false;
  if (!m || !m->pts0) return fail(m, TRN_ERR_INVALID, "reload: nothing loaded");
  m->err.clear();
  return init_from_device(m);
}

/* the token-by-token reader (any whitespace between numbers), for text that
 * is not laid out one record per line */
static int load_tokens(trn_mesh* m, Reader& r, MeshInput* in) {
  long nv = r.find("Vertices");
  if (nv <= 0) return fail(m, TRN_ERR_IO, "mesh: no Vertices section");
  std::vector<double>& pts = in->pts;
  std::vector<uint8_t>& tags = in->tags;
  pts.assign((size_t) nv * 2, 0.0);
  tags.assign((size_t) nv, 0);
  for (long i = 0; i < nv; ++i) {
    long tag;
    if (!r.next_double(&pts[2 * i]) || !r.next_double(&pts[2 * i + 1]) || !r.next_long(&tag))
      return fail(m, TRN_ERR_IO, "mesh: truncated Vertices");
  }
  size_t after_v = r.pos;
  long ne = r.find("Edges");
  if (ne > 0) {
    for (long i = 0; i < ne; ++i) {
      long a, b, tag;
      if (!r.next_long(&a) || !r.next_long(&b) || !r.next_long(&tag))
        return fail(m, TRN_ERR_IO, "mesh: truncated Edges");
      if (a < 1 || a > nv || b < 1 || b > nv) return fail(m, TRN_ERR_IO, "mesh: edge index out of range");
      tags[a - 1] = TRN_TAG_BOUND;
      tags[b - 1] = TRN_TAG_BOUND;
    }
  } else {
    r.pos = after_v;
  }
  long nt = r.find("Triangles");
  if (nt <= 0) return fail(m, TRN_ERR_IO, "mesh: no Triangles section");
  std::vector<int>& tris = in->tris;
  tris.assign((size_t) nt * 3, 0);
  for (long i = 0; i < nt; ++i) {
    long a, b, c, tag;
    if (!r.next_long(&a) || !r.next_long(&b) || !r.next_long(&c) || !r.next_long(&tag))
      return fail(m, TRN_ERR_IO, "mesh: truncated Triangles");
    tris[3 * i] = (int) a - 1;
    tris[3 * i + 1] = (int) b - 1;
    tris[3 * i + 2] = (int) c - 1;
  }
  size_t after_t = r.pos;
  long nc = r.find("Corners");
  if (nc > 0) {
    for (long i = 0; i < nc; ++i) {
      long v;
      if (!r.next_long(&v)) return fail(m, TRN_ERR_IO, "mesh: truncated Corners");
      if (v < 1 || v > nv) return fail(m, TRN_ERR_IO, "mesh: corner index out of range");
      tags[v - 1] = TRN_TAG_BOUND | TRN_TAG_CORNER;
    }
  } else {
    r.pos = after_t;
  }
  in->nv = nv;
  in->nt = nt;
  return TRN_OK;
}

/* Mesh::load, io.cpp:53-161: a medit .mesh (or the binary form written by
 * trn_mesh_store_binary) and an optional .bb nodal solution */
int trn_mesh_load(trn_mesh* m, const char* mesh_path, const char* solut_path) {
  if (m) m->qual_fresh = false;
  if (!m || !mesh_path) return fail(m, TRN_ERR_INVALID, "load: null path");
  MeshInput in;
  {
    Reader r;
    if (!read_file(mesh_path, &r.buf)) return fail(m, TRN_ERR_IO, std::string("cannot open ") + mesh_path);
    std::string err;
    const int prc = is_binary_mesh(r.buf) ? parse_mesh_binary(r.buf, &in, &err) : parse_mesh_text(r.buf, &in, &err);
    if (prc > 0) return fail(m, TRN_ERR_IO, err);
    if (prc < 0) {
      in = MeshInput();
      const int rc = load_tokens(m, r, &in);
      if (rc) return rc;
    }
  }
  const long nv = in.nv, nt = in.nt;
  if (nv != m->size0[0] || nt != m->size0[1])
    return fail(m, TRN_ERR_IO, "mesh: sizes differ from the ones the mesh was created with");
  std::vector<double> u;
  if (solut_path) {
    Reader rb;
    if (!read_file(solut_path, &rb.buf)) return fail(m, TRN_ERR_IO, std::string("cannot open ") + solut_path);
    std::string err;
    const int prc = parse_bb_text(rb.buf, nv, &u, &err);
    if (prc > 0) return fail(m, TRN_ERR_IO, err);
    if (prc < 0) {
      u.assign((size_t) nv, 0.0);
      rb.pos = 0;
      rb.skip_line();
      for (long i = 0; i < nv; ++i)
        if (!rb.next_double(&u[i])) return fail(m, TRN_ERR_IO, "bb: truncated values");
    }
  } else {
    u.assign((size_t) nv, 0.0);
  }
  return trn_mesh_load_arrays(m, (int) nv, (int) nt, in.pts.data(), in.tris.data(), in.tags.data(), u.data());
}

/* the .mesh (text or binary) and .bb files as trn_mesh_load reads them, into
 * host arrays, without a mesh or a GPU: the counts always, the arrays when
 * their capacities (vertices, triangles) suffice */
int trn_read_mesh_files(const char* mesh_path, const char* solut_path, int* nb_nodes, int* nb_elems,
                        double* points, int* tris, uint8_t* tags, double* solut, int cap_nodes,
                        int cap_elems) {
  if (!mesh_path || !nb_nodes || !nb_elems) return TRN_ERR_INVALID;
  MeshInput in;
  Reader r;
  if (!read_file(mesh_path, &r.buf)) return TRN_ERR_IO;
  std::string err;
  int prc = is_binary_mesh(r.buf) ? parse_mesh_binary(r.buf, &in, &err) : parse_mesh_text(r.buf, &in, &err);
  if (prc > 0) return TRN_ERR_IO;
  if (prc < 0) {
    in = MeshInput();
    if (load_tokens(nullptr, r, &in)) return TRN_ERR_IO;
  }
  *nb_nodes = (int) in.nv;
  *nb_elems = (int) in.nt;
  if (in.nv > cap_nodes || in.nt > cap_elems) return TRN_OK;
  if (points) std::memcpy(points, in.pts.data(), sizeof(double) * 2 * (size_t) in.nv);
  if (tris) std::memcpy(tris, in.tris.data(), sizeof(int) * 3 * (size_t) in.nt);
  if (tags) std::memcpy(tags, in.tags.data(), (size_t) in.nv);
  if (solut_path && solut) {
    Reader rb;
    if (!read_file(solut_path, &rb.buf)) return TRN_ERR_IO;
    std::vector<double> u;
    prc = parse_bb_text(rb.buf, in.nv, &u, &err);
    if (prc > 0) return TRN_ERR_IO;
    if (prc < 0) {
      u.assign((size_t) in.nv, 0.0);
      rb.pos = 0;
      rb.skip_line();
      for (long i = 0; i < in.nv; ++i)
        if (!rb.next_double(&u[i])) return TRN_ERR_IO;
    }
    std::memcpy(solut, u.data(), sizeof(double) * (size_t) in.nv);
  }
  return TRN_OK;
}

/* the mesh as trn_mesh_compact would renumber it (points, tags, 0-based
 * triangles), in the binary form trn_mesh_load reads */
int trn_mesh_store_binary(trn_mesh* m, const char* path) {
  if (!m || !path || m->nb_nodes <= 0) return fail(m, TRN_ERR_INVALID, "store_binary: no mesh or path");
  const size_t nn = (size_t) m->nb_nodes, ne = (size_t) m->nb_elems;
  std::vector<double> pts(2 * nn);
  std::vector<int> tri(3 * ne);
  std::vector<uint8_t> alive(nn), tags(nn);
  int rc = trn_mesh_export(m, pts.data(), nullptr, tri.data(), alive.data(), tags.data());
  if (rc) return rc;
  std::vector<int> newid(nn, -1);
  std::vector<double> cp;
  std::vector<uint8_t> ct;
  for (size_t i = 0; i < nn; ++i)
    if (alive[i]) {
      newid[i] = (int) ct.size();
      cp.push_back(pts[2 * i]);
      cp.push_back(pts[2 * i + 1]);
      ct.push_back(tags[i]);
    }
  std::vector<int> cti;
  for (size_t e = 0; e < ne; ++e)
    if (tri[3 * e] >= 0)
      for (int k = 0; k < 3; ++k) cti.push_back(newid[(size_t) tri[3 * e + k]]);
  if (write_mesh_binary(path, (long) ct.size(), (long) cti.size() / 3, cp.data(), ct.data(), cti.data()))
    return fail(m, TRN_ERR_IO, std::string("cannot write ") + path);
  return TRN_OK;
}

int trn_mesh_export(trn_mesh* m, double* points, double* tensor, int* tris, uint8_t* alive,
                    uint8_t* tags) {
  if (!m) return TRN_ERR_INVALID;
  const size_t nn = (size_t) m->nb_nodes, ne = (size_t) m->nb_elems;
  cudaStream_t s = m->stream;
  if (points) CK(cudaMemcpyAsync(points, m->d.pts, sizeof(double2) * nn, cudaMemcpyDeviceToHost, s));
  std::vector<double4> t4;
  std::vector<int4> e4;
  if (tensor) {
    t4.resize(nn);
    CK(cudaMemcpyAsync(t4.data(), m->d.ten, sizeof(double4) * nn, cudaMemcpyDeviceToHost, s));
  }
  if (tris) {
    e4.resize(ne);
    CK(cudaMemcpyAsync(e4.data(), m->d.tri, sizeof(int4) * ne, cudaMemcpyDeviceToHost, s));
  }
  if (alive) CK(cudaMemcpyAsync(alive, m->d.alive, nn, cudaMemcpyDeviceToHost, s));
  if (tags) CK(cudaMemcpyAsync(tags, m->d.tags, nn, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  for (size_t i = 0; i < t4.size(); ++i) {
    tensor[3 * i] = t4[i].x;
    tensor[3 * i + 1] = t4[i].y;
    tensor[3 * i + 2] = t4[i].z;
  }
  for (size_t i = 0; i < e4.size(); ++i) {
    tris[3 * i] = e4[i].x;
    tris[3 * i + 1] = e4[i].y;
    tris[3 * i + 2] = e4[i].z;
  }
  return TRN_OK;
}

int trn_mesh_capacity(trn_mesh* m, int* capa_nodes, int* capa_elems) {
  if (!m) return TRN_ERR_INVALID;
  if (capa_nodes) *capa_nodes = m->capa_node;
  if (capa_elems) *capa_elems = m->capa_elem;
  return TRN_OK;
}

int trn_mesh_counts(trn_mesh* m, int* nb_nodes, int* nb_elems, int* live_nodes, int* live_elems) {
  if (!m) return TRN_ERR_INVALID;
  if (nb_nodes) *nb_nodes = m->nb_nodes;
  if (nb_elems) *nb_elems = m->nb_elems;
  if (live_nodes || live_elems) {
    count_live(m->d, m->nb_nodes, m->nb_elems, m->status + S_LIVE, m->stream);
    int rc = sync_status(m);
    if (rc) return rc;
    if (live_nodes) *live_nodes = m->h_status[S_LIVE];
    if (live_elems) *live_elems = m->h_status[S_LIVE + 1];
  }
  return TRN_OK;
}

/* the adapted mesh in memory, renumbered like Mesh::store (io.cpp:199-233) */
int trn_mesh_export_compact(trn_mesh* m, double* points, int* tris, double* tensor, int* nb_nodes,
                            int* nb_elems) {
  if (!m || !nb_nodes || !nb_elems) return fail(m, TRN_ERR_INVALID, "export_compact: null argument");
  cudaStream_t s = m->stream;
  DMesh& d = m->d;
  compact_u8(d.alive, m->nb_nodes, m->list, m->scan, s);
  int rc = sync_status(m, m->scan.count);
  if (rc) return rc;
  const int nv = m->h_status[S_COUNT];
  double* st_pts = reinterpret_cast<double*>(m->stage);
  double* st_ten = reinterpret_cast<double*>(m->stage) + 2 * (size_t) nv;
  pack_nodes(d, m->list, m->scan.count, m->target, st_pts, tensor ? st_ten : nullptr, s);
  if (points) CK(cudaMemcpyAsync(points, st_pts, sizeof(double) * 2 * (size_t) nv, cudaMemcpyDeviceToHost, s));
  if (tensor) CK(cudaMemcpyAsync(tensor, st_ten, sizeof(double) * 3 * (size_t) nv, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  flag_live_tris(d, m->nb_elems, m->flag, s);
  compact_u8(m->flag, m->nb_elems, m->list, m->scan, s);
  if ((rc = sync_status(m, m->scan.count))) return rc;
  const int ne = m->h_status[S_COUNT];
  int* st_tri = reinterpret_cast<int*>(m->stage);
  pack_tris(d, m->list, m->scan.count, m->target, st_tri, s);
  if (tris) CK(cudaMemcpyAsync(tris, st_tri, sizeof(int) * 3 * (size_t) ne, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  *nb_nodes = nv;
  *nb_elems = ne;
  return TRN_OK;
}

/* The solver-coupled loop (the adaptive loop the reference is written for,
 * README.md:8, scripts/bench_run.py:77-110: evaluate the field on the
 * adapted mesh, recover the metric, adapt again). The reference closes the
 * loop through files: Mesh::store (io.cpp:164-255, coordinates printed with
 * 8 decimals, boundary only as RequiredVertices) and a fresh Mesh::load.
 * trn_mesh_compact does the same renumbering on the device, without the
 * rounding and keeping the boundary and corner tags: live vertices in slot
 * order, live elements in slot order, every structure rebuilt as a load
 * builds it. The state becomes the one trn_mesh_reload returns to. */
int trn_mesh_compact(trn_mesh* m) {
  if (m) m->qual_fresh = false;
  if (!m || m->nb_nodes <= 0) return fail(m, TRN_ERR_INVALID, "compact: no mesh loaded");
  m->err.clear();
  cudaStream_t s = m->stream;
  DMesh& d = m->d;
  compact_u8(d.alive, m->nb_nodes, m->list, m->scan, s);
  int rc = sync_status(m, m->scan.count);
  if (rc) return rc;
  const int nv = m->h_status[S_COUNT];
  flag_live_tris(d, m->nb_elems, m->flag, s);
  /* the element list goes to the stage buffer: m->list still holds the vertices */
  int* elist = reinterpret_cast<int*>(m->stage);
  compact_u8(m->flag, m->nb_elems, elist, m->scan, s);
  if ((rc = sync_status(m, m->scan.count))) return rc;
  const int ne = m->h_status[S_COUNT];
  if (nv <= 0 || ne <= 0) return fail(m, TRN_ERR_INVALID, "compact: empty mesh");
  if (nv > m->n0_nodes || ne > m->n0_elems) {
    double2* p0 = nullptr;
    int4* t0 = nullptr;
    uint8_t* g0 = nullptr;
    if ((rc = dmalloc(m, &p0, (size_t) nv)) || (rc = dmalloc(m, &t0, (size_t) ne)) ||
        (rc = dmalloc(m, &g0, (size_t) nv))) {
      cudaFree(p0);
      cudaFree(t0);
      cudaFree(g0);
      return rc;
    }
    CK(cudaStreamSynchronize(s));
    cudaFree(m->pts0);
    cudaFree(m->tri0);
    cudaFree(m->tags0);
    m->pts0 = p0;
    m->tri0 = t0;
    m->tags0 = g0;
  }
  /* the vertex list's length on the device again (the element compaction
   * reused the scan's counter, which now holds ne) */
  int nv_host = nv;
  CK(cudaMemcpyAsync(m->status + S_COUNT, &nv_host, sizeof(int), cudaMemcpyHostToDevice, s));
  pack_nodes_load(d, m->list, m->status + S_COUNT, m->target, m->pts0, m->tags0, s);
  pack_tris_load(d, elist, m->scan.count, m->target, m->tri0, s);
  CK(cudaStreamSynchronize(s));
  CK(cudaMemsetAsync(m->solut, 0, sizeof(double) * (size_t) m->capa_node, s));
  m->n0_nodes = nv;
  m->n0_elems = ne;
  return init_from_device(m);
}

/* a new nodal field for the vertex slots in use (after trn_mesh_compact:
 * the live vertices in their new order), for the next trn_metric_run */
int trn_mesh_set_solution(trn_mesh* m, const double* solut, int n) {
  if (!m || !solut) return fail(m, TRN_ERR_INVALID, "set_solution: null argument");
  if (n != m->nb_nodes) return fail(m, TRN_ERR_INVALID, "set_solution: one value per vertex slot in use");
  CK(cudaMemcpyAsync(m->solut, solut, sizeof(double) * (size_t) n, cudaMemcpyHostToDevice, m->stream));
  CK(cudaStreamSynchronize(m->stream));
  return TRN_OK;
}

/* element qualities in the current arithmetic form (dead elements: 0) */
int trn_mesh_qualities(trn_mesh* m, double* q) {
  if (!m || !q) return fail(m, TRN_ERR_INVALID, "qualities: null argument");
  CK(cudaMemsetAsync(m->d.qual, 0, sizeof(double) * (size_t) m->nb_elems, m->stream));
  quality_all(m->d, m->nb_elems, m->fp32, m->stream);
  CK(cudaMemcpyAsync(q, m->d.qual, sizeof(double) * (size_t) m->nb_elems, cudaMemcpyDeviceToHost, m->stream));
  return sync_status(m);
}

/* Mesh::computeQuality(double quality[3]), mesh.cpp:647-681: min, max and
 * mean element quality (the min and max are folded into quality[0..1]) */
int trn_mesh_quality_stats(trn_mesh* m, double quality[3]) {
  if (!m || !quality) return fail(m, TRN_ERR_INVALID, "quality_stats: null argument");
  std::vector<double> q((size_t) m->nb_elems);
  std::vector<int> tri((size_t) m->nb_elems * 3);
  int rc = trn_mesh_qualities(m, q.data());
  if (rc) return rc;
  if ((rc = trn_mesh_export(m, nullptr, nullptr, tri.data(), nullptr, nullptr))) return rc;
  double qmin = 3., qmax = 0., qtot = 0.;
  int count = 0;
  for (int i = 0; i < m->nb_elems; ++i) {
    if (tri[3 * i] < 0) continue;
    qmin = std::min(qmin, q[i]);
    qmax = std::max(qmax, q[i]);
    qtot += q[i];
    ++count;
  }
  quality[0] = std::min(quality[0], qmin);
  quality[1] = std::max(quality[1], qmax);
  quality[2] = count ? qtot / count : 0.0;
  return TRN_OK;
}

/* Mesh::store, io.cpp:164-255 */
int trn_mesh_store(trn_mesh* m, const char* path) {
  if (!m || !path) return fail(m, TRN_ERR_INVALID, "store: null path");
  const int nn = m->nb_nodes, ne = m->nb_elems;
  std::vector<double> pts((size_t) nn * 2);
  std::vector<int> tri((size_t) ne * 3);
  std::vector<uint8_t> alive((size_t) nn), tags((size_t) nn);
  int rc = trn_mesh_export(m, pts.data(), nullptr, tri.data(), alive.data(), tags.data());
  if (rc) return rc;
  FILE* f = std::fopen(path, "w");
  if (!f) return fail(m, TRN_ERR_IO, std::string("cannot write ") + path);
  int real_nodes = 0, real_elems = 0;
  for (int i = 0; i < nn; ++i) real_nodes += alive[i] ? 1 : 0;
  for (int i = 0; i < ne; ++i) real_elems += tri[3 * i] > -1 ? 1 : 0;
  std::fprintf(f, "MeshVersionFormatted 1\nDimension 2\nVertices\n%d\n", real_nodes);
  std::vector<int> index((size_t) nn, -1), required;
  int k = 0;
  for (int i = 0; i < nn; ++i) {
    if (!alive[i]) continue;
    std::fprintf(f, "%.8f\t%.8f\t0\n", pts[2 * i], pts[2 * i + 1]);
    index[i] = ++k;
    if (tags[i] & TRN_TAG_BOUND) required.push_back(k);
  }
  std::fprintf(f, "\nTriangles\n%d\n", real_elems);
  for (int i = 0; i < ne; ++i) {
    const int* n = &tri[3 * i];
    if (n[0] > -1) std::fprintf(f, "%d\t%d\t%d\t0\n", index[n[0]], index[n[1]], index[n[2]]);
  }
  std::fprintf(f, "\nRequiredVertices\n%zu\n", required.size());
  for (int v : required) std::fprintf(f, "%d\n", v);
  std::fprintf(f, "\nEnd\n");
  std::fclose(f);
  return TRN_OK;
}

int trn_mesh_store_sol(trn_mesh* m, const char* path) {
  if (!m || !path) return fail(m, TRN_ERR_INVALID, "store_sol: null path");
  const int nn = m->nb_nodes;
  std::vector<double> ten((size_t) nn * 3);
  std::vector<uint8_t> alive((size_t) nn);
  int rc = trn_mesh_export(m, nullptr, ten.data(), nullptr, alive.data(), nullptr);
  if (rc) return rc;
  FILE* f = std::fopen(path, "w");
  if (!f) return fail(m, TRN_ERR_IO, std::string("cannot write ") + path);
  int real = 0;
  for (int i = 0; i < nn; ++i) real += alive[i] ? 1 : 0;
  std::fprintf(f, "MeshVersionFormatted 1\nDimension 2\nSolAtVertices\n%d\n1 3\n", real);
  for (int i = 0; i < nn; ++i)
    if (alive[i]) std::fprintf(f, "%.17g %.17g %.17g\n", ten[3 * i], ten[3 * i + 1], ten[3 * i + 2]);
  std::fprintf(f, "\nEnd\n");
  std::fclose(f);
  return TRN_OK;
}

int trn_set_replay(trn_mesh* m, const int32_t* log, size_t n) {
  if (m) m->qual_fresh = false;
  if (!m) return TRN_ERR_INVALID;
  if (m->d_log) {
    cudaFree(m->d_log);
    m->d_log = nullptr;
  }
  m->log.clear();
  m->cursor = 0;
  m->replay = false;
  if (!log || n == 0) return TRN_OK;
  if (m->fp32) return fail(m, TRN_ERR_INVALID, "set_replay: replay needs the FP64 form");
  m->log.assign(log, log + n);
  CK(cudaMalloc(&m->d_log, sizeof(int32_t) * n));
  CK(cudaMemcpy(m->d_log, log, sizeof(int32_t) * n, cudaMemcpyHostToDevice));
  m->replay = true;
  return TRN_OK;
}

int trn_set_precision(trn_mesh* m, int mode) {
  if (m) m->qual_fresh = false;
  if (!m || (mode != TRN_PRECISION_FP64 && mode != TRN_PRECISION_MIXED))
    return fail(m, TRN_ERR_INVALID, "set_precision: unknown mode");
  const bool f = mode == TRN_PRECISION_MIXED;
  if (f && m->replay) return fail(m, TRN_ERR_INVALID, "set_precision: replay needs the FP64 form");
  if (f != m->fp32 && m->nb_nodes > 0) {
    log_cache(m->d, m->nb_nodes, f, m->stream);
    int rc = sync_status(m);
    if (rc) return rc;
  }
  m->fp32 = f;
  return TRN_OK;
}

int trn_set_options(trn_mesh* m, uint64_t seed, int exact_sum) {
  if (!m) return TRN_ERR_INVALID;
  m->seed = seed;
  m->exact_sum = exact_sum != 0;
  return TRN_OK;
}

int trn_selftest_barrier(long long max_polls) {
  if (max_polls < 1) return TRN_ERR_INVALID;
  int gave_up = 0;
  if (barrier_selftest(max_polls, &gave_up) != cudaSuccess) {
    cudaGetLastError();
    return TRN_ERR_CUDA;
  }
  return gave_up ? TRN_ERR_NO_PROGRESS : TRN_OK;
}

int trn_set_level_cap(trn_mesh* m, int cap) {
  if (!m) return TRN_ERR_INVALID;
  if (cap < 1) return fail(m, TRN_ERR_INVALID, "level cap: must be at least 1");
  m->level_cap = cap;
  return TRN_OK;
}

int trn_set_swap_match(trn_mesh* m, int policy) {
  if (!m) return TRN_ERR_INVALID;
  if (policy != TRN_SWAP_ROW_ORDER && policy != TRN_SWAP_GAIN && policy != TRN_SWAP_GREEDY)
    return fail(m, TRN_ERR_INVALID, "swap matching: unknown policy");
  m->swap_match = policy;
  return TRN_OK;
}

double trn_last_complexity(trn_mesh* m) { return m ? m->last_complexity : 0.0; }
double trn_last_time_ms(trn_mesh* m) { return m ? m->last_ms : 0.0; }
void* trn_mesh_stream(trn_mesh* m) { return m ? (void*) m->stream : nullptr; }
const char* trn_last_error(trn_mesh* m) { return m ? m->err.c_str() : "null mesh"; }

/* Metrics::run, metric.cpp:59-70 */
int trn_metric_run(trn_mesh* m, double target_factor, int norm, double h_min, double h_max,
                   trn_stats* st) {
  if (!m || m->nb_nodes <= 0) return fail(m, TRN_ERR_INVALID, "metric: no mesh loaded");
  if (norm < 0 || h_min <= 0 || h_max <= 0) return fail(m, TRN_ERR_INVALID, "metric: bad parameters");
  m->err.clear();
  MetricParams p;
  p.target = (double) (int) std::floor(m->nb_nodes * target_factor);
  p.scale_exp = norm ? -1. / (2 * norm + 2) : 0.5;
  p.eig_min = 1 / trn_pow(h_min, 2);
  p.eig_max = 1 / trn_pow(h_max, 2);
  begin_timing(m);
  metric_run(m->d, m->nb_nodes, m->nb_elems, m->solut, m->grad, m->terms, m->complexity,
             m->exact_sum || m->replay, p, m->stream, nullptr, m->fp32);
  CK(cudaMemcpyAsync(m->h_status + H_WIDE, m->complexity, sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  int rc = sync_status(m);
  if (rc) return rc;
  std::memcpy(&m->last_complexity, m->h_status + H_WIDE, sizeof(double));
  return end_timing(m, st, m->nb_nodes, m->nb_nodes);
}

/* ---------------- stage enqueuers ----------------
 * The same kernels serve the per-stage calls below (the host reads the status
 * block back once per coarsening / swapping level, or per coloring batch) and
 * a captured round (trn_round_capture: loop nodes decide on the device).
 * Every count a kernel needs is on the device (S_NB, list counters); the host
 * only sizes grids: by its own copy of a count, or, in a captured round, by
 * the capacity. */
namespace {

int hint_nodes(const trn_mesh* m, bool capture) { return capture ? m->capa_node : m->nb_nodes; }
int hint_elems(const trn_mesh* m, bool capture) { return capture ? m->capa_elem : m->nb_elems; }

Seed seed_of(trn_mesh* m, uint64_t mix) {
  return Seed{m->seed, reinterpret_cast<const unsigned*>(m->status + S_TICK), mix};
}

void stats_reset(trn_mesh* m, cudaStream_t s) {
  cudaMemsetAsync(m->status + S_EVAL, 0, sizeof(int) * 3, s);
  cudaMemsetAsync(m->status + S_NTASK, 0, sizeof(int) * 2, s);   /* S_NTASK, S_LEVEL */
}

int* act_list(trn_mesh* m, int k) { return k ? m->hws.list_b : m->hws.list_a; }

DMesh level_mesh(trn_mesh* m) {
  DMesh dl = m->d;
  dl.act_next = act_list(m, 1);
  dl.act_next_n = m->status + S_ACT + 1;
  dl.fix_list = m->hws.fix_list;
  dl.fix_n = m->status + S_FIX;
  return dl;
}

/* Refine::run: depth levels, every count on the device (refine.cu) */
void enq_refine(trn_mesh* m, int depth, cudaStream_t s) {
  stats_reset(m, s);
  refine_reset_hash(m->rws, s);
  for (int level = 0; level < depth; ++level)
    refine_level(m->d, m->capa_node, m->capa_elem, m->rws, m->scan, m->status + S_EVAL, m->fp32, s);
  flag_all_alive(m->d, m->capa_node, s);
  fix_tagged(m->d, m->capa_node, s);
}

void enq_coarsen_begin(trn_mesh* m, cudaStream_t s, bool capture) {
  stats_reset(m, s);
  coarsen_pre(m->d, hint_nodes(m, capture), s, act_list(m, 0), m->status + S_ACT);
}

/* one free-mode coarsening level over list 0 (bound: its length, < 0 unknown) */
void enq_coarsen_level(trn_mesh* m, cudaStream_t s, long long bound, cudaGraphConditionalHandle h,
                       bool use_h) {
  DMesh dl = level_mesh(m);
  /* no memsets before the filter: the previous level's end cleared the
   * candidate count and the filter clears the activity and repair list
   * counters, so after the host's read back the device starts at once */
  coarsen_filter_append(dl, act_list(m, 0), m->status + S_ACT, m->target, m->list, m->status + S_NTASK,
                        m->hws.state, m->fp32, s, bound);
  mis_jp_rounds(dl, m->list, m->status + S_NTASK, kMisRounds, seed_of(m, 0x9e37ULL), m->hws, m->indep,
                m->status + S_NINDEP, s, bound);
  collapse(dl, m->indep, m->status + S_NINDEP, m->target, nullptr, s, bound);
  fix_list_level_end(dl, dl.fix_list, dl.fix_n, bound < 0 ? -1 : 16 * bound, m->status, kLevelCoarsen,
                     m->level_cap, act_list(m, 1), act_list(m, 0),
                     bound < 0 ? m->capa_node : (int) std::max(bound, 1LL), s, h, use_h);
}

void enq_swap_begin(trn_mesh* m, cudaStream_t s, bool capture) {
  stats_reset(m, s);
  swap_init(m->d, hint_nodes(m, capture), hint_elems(m, capture), m->map, m->fp32, s, act_list(m, 0),
            m->status + S_ACT);
}

void enq_swap_level(trn_mesh* m, cudaStream_t s, long long bound, cudaGraphConditionalHandle h,
                    bool use_h) {
  DMesh dl = level_mesh(m);
  /* as for coarsening; the dual filter also clears the flip count */
  uint32_t* rank = m->swap_match == TRN_SWAP_GAIN ? m->hws.rank : nullptr;
  GreedyReset gr;
  if (m->swap_match == TRN_SWAP_GREEDY) gr = GreedyReset{m->hws.mate, m->hws.prop, m->hws.prop2};
  swap_filter_dual(dl, act_list(m, 0), m->status + S_ACT, m->dual, m->dual_n, m->map, rank,
                   m->status + S_NTASK, m->fp32, s, bound, gr, m->status + S_COMMIT);
  /* a captured round knows no list length, but the capacity bounds it and
   * sizes the matching's rounds for the mesh at hand */
  if (m->swap_match == TRN_SWAP_GREEDY)
    match_greedy(dl, m->capa_elem, m->dual, m->dual_n, m->status + S_NTASK, m->map, m->hws, m->pairs,
                 m->status + S_NPAIRS, s, bound < 0 ? (long long) m->capa_elem : bound);
  else
    match_handshake(dl, m->capa_elem, m->dual, m->dual_n, m->status + S_NTASK, m->map, rank,
                    seed_of(m, 0x51edULL), m->hws, m->pairs, m->status + S_NPAIRS, s, bound);
  swap_flip(dl, m->pairs, m->status + S_NPAIRS, m->map, m->dual, m->dual_n, m->status + S_NTASK,
            m->status + S_COMMIT, true, m->fp32, s, bound);
  fix_list_level_end(dl, dl.fix_list, dl.fix_n, bound < 0 ? -1 : 4 * bound, m->status, kLevelSwap,
                     m->level_cap, act_list(m, 1), act_list(m, 0),
                     bound < 0 ? m->capa_elem : (int) std::max(bound, 1LL), s, h, use_h);
}

int max_colors_of(int max_colors) {
  int max_col = std::max(6, max_colors) - 1;  /* Partit: max.part = max(6, n), colors 1..max.part-1 */
  return std::min(max_col, 30);
}

}  // namespace

/* Refine::run, refinement.cpp:445-493 */
int trn_refine_run(trn_mesh* m, int depth, trn_stats* st) {
  if (!m || m->nb_nodes <= 0) return fail(m, TRN_ERR_INVALID, "refine: no mesh loaded");
  if (depth < 1) return fail(m, TRN_ERR_INVALID, "refine: depth < 1");
  m->err.clear();
  begin_timing(m);
  enq_refine(m, depth, m->stream);
  int rc = sync_status(m);
  if (rc) return rc;
  m->nb_nodes = m->h_status[S_NB];
  m->nb_elems = m->h_status[S_NB + 1];
  return end_timing(m, st, m->h_status[S_EVAL], m->h_status[S_TASK]);
}

/* Coarse::run, coarsening.cpp:463-508 */
int trn_coarsen_run(trn_mesh* m, int max_colors, trn_stats* st) {
  if (!m || m->nb_nodes <= 0) return fail(m, TRN_ERR_INVALID, "coarsen: no mesh loaded");
  (void) max_colors;
  m->err.clear();
  begin_timing(m);
  cudaStream_t s = m->stream;
  if (!m->replay) {
    /* free mode: one read back per level; each level works on the list of
     * vertices the previous one activated and repairs the listed ones */
    enq_coarsen_begin(m, s, false);
    long long bound = m->nb_nodes;
    do {
      enq_coarsen_level(m, s, bound, 0, false);
      int rc = sync_status(m);
      if (rc) return rc;
      bound = m->h_status[S_ACT];
    } while (m->h_status[S_CONT]);
    return end_timing(m, st, m->h_status[S_EVAL], m->h_status[S_TASK]);
  }
  coarsen_pre(m->d, m->nb_nodes, s);
  int eval = 0, task = 0, nb_indep = 0, level = 0;
  do {
    build_vicin(m->d, m->nb_nodes, true, s);
    coarsen_filter(m->d, m->nb_nodes, m->target, m->flag, m->fp32, s);
    compact_u8(m->flag, m->nb_nodes, m->list, m->scan, s);
    int rc = sync_status(m, m->scan.count);
    if (rc) return rc;
    const int ntasks = m->h_status[S_COUNT];
    if (!ntasks) break;
    eval += ntasks;
    size_t off;
    int n;
    if ((rc = replay_take(m, 1, &off, &n))) return rc;
    nb_indep = n;
    collapse(m->d, m->d_log + off, m->d_log + off - 1, m->target, m->flag, s);
    fix_tagged(m->d, m->nb_nodes, s);
    task += nb_indep;
    if (++level > m->level_cap) return fail(m, TRN_ERR_NO_PROGRESS, "coarsen: level cap reached");
  } while (nb_indep);
  int rc = sync_status(m);
  if (rc) return rc;
  return end_timing(m, st, eval, task);
}

/* Swap::run, swapping.cpp:383-428 */
int trn_swap_run(trn_mesh* m, trn_stats* st) {
  if (!m || m->nb_nodes <= 0) return fail(m, TRN_ERR_INVALID, "swap: no mesh loaded");
  m->err.clear();
  begin_timing(m);
  cudaStream_t s = m->stream;
  if (!m->replay) {
    enq_swap_begin(m, s, false);
    long long bound = m->nb_elems;
    do {
      enq_swap_level(m, s, bound, 0, false);
      int rc = sync_status(m);
      if (rc) return rc;
      bound = m->h_status[S_ACT];
    } while (m->h_status[S_CONT]);
    const int rc = end_timing(m, st, m->h_status[S_EVAL], m->h_status[S_TASK]);
    m->qual_fresh = rc == TRN_OK;
    return rc;
  }
  swap_init(m->d, m->nb_nodes, m->nb_elems, m->map, m->fp32, s);
  int eval = 0, task = 0, commit = 0, level = 0;
  do {
    swap_filter(m->d, m->nb_elems, m->flag, s);
    compact_u8(m->flag, m->nb_elems, m->list, m->scan, s);
    int rc = sync_status(m, m->scan.count);
    if (rc) return rc;
    const int ntasks = m->h_status[S_COUNT];
    if (!ntasks) break;
    swap_dual(m->d, m->list, ntasks, m->dual, m->dual_n, m->map, s);
    size_t off;
    int n;
    if ((rc = replay_take(m, 2, &off, &n))) return rc;
    CK(cudaMemsetAsync(m->status + S_COMMIT, 0, sizeof(int), s));
    swap_flip(m->d, m->d_log + off, m->d_log + off - 1, m->map, m->dual, m->dual_n, m->scan.count,
              m->status + S_COMMIT, false, m->fp32, s);
    fix_tagged(m->d, m->nb_nodes, s);
    if ((rc = sync_status(m))) return rc;
    commit = m->h_status[S_COMMIT];
    eval += ntasks;
    task += commit / 2;
    if (++level > m->level_cap) return fail(m, TRN_ERR_NO_PROGRESS, "swap: level cap reached");
  } while (commit);
  const int rc = end_timing(m, st, eval, task);
  m->qual_fresh = rc == TRN_OK;
  return rc;
}

/* Smooth::run, smoothing.cpp:274-302 */
int trn_smooth_run(trn_mesh* m, int max_colors, int depth, trn_stats* st) {
  if (!m || m->nb_nodes <= 0) return fail(m, TRN_ERR_INVALID, "smooth: no mesh loaded");
  const int max_col = max_colors_of(max_colors);
  m->err.clear();
  const bool fresh = m->qual_fresh;
  begin_timing(m);
  cudaStream_t s = m->stream;
  smooth_pre(m->d, m->nb_nodes, s);
  build_vicin(m->d, m->nb_nodes, true, s);
  std::vector<std::pair<const int*, int>> classes;
  if (m->replay) {
    size_t off;
    int parts;
    int rc = replay_take(m, 3, &off, &parts);
    if (rc) return rc;
    size_t p = off;
    for (int c = 0; c < parts; ++c) {
      int n = m->log[p];
      classes.emplace_back(m->d_log + p + 1, n);
      p += 1 + (size_t) n;
    }
  } else {
    color_jp(m->d, m->nb_nodes, max_col, seed_of(m, 0xc01dULL), m->hws, m->parts, m->status + S_PARTS,
             reinterpret_cast<unsigned*>(m->status + S_TICK), s);
    int rc = sync_status(m);
    if (rc) return rc;
    for (int c = 0; c < max_col && c < 8; ++c) {
      int a = m->h_status[S_PARTS + c], b = m->h_status[S_PARTS + c + 1];
      classes.emplace_back(m->parts + a, b - a);
    }
  }
  /* the cached qualities (smoothing.cpp:145-151); a swap or smoothing call
   * just before left them equal to this recomputation, bit for bit (the
   * flips and moves store the qualities of the elements they change, from
   * the same arithmetic) */
  if (!fresh) quality_all(m->d, m->nb_elems, m->fp32, s);
  CK(cudaMemsetAsync(m->status + S_SMOOTH_TASKS, 0, sizeof(int) * 2, s));
  for (int level = 0; level < depth; ++level)
    for (auto& c : classes) smooth_color(m->d, c.first, c.second, m->status + S_SMOOTH_TASKS, m->fp32, s);
  int rc = sync_status(m);
  if (rc) return rc;
  rc = end_timing(m, st, m->h_status[S_SMOOTH_TASKS], m->h_status[S_SMOOTH_COMMIT]);
  m->qual_fresh = rc == TRN_OK;
  return rc;
}

/* the element-quality functional J = sum_T q_T and its adjoint */
int trn_quality_adjoint(trn_mesh* m, const double* xy, const double* solut, double target_factor,
                        int norm, double h_min, double h_max, int precision, double* value,
                        double* grad_xy, double* grad_solut) {
  if (!m || m->nb_nodes <= 0) return fail(m, TRN_ERR_INVALID, "quality_adjoint: no mesh loaded");
  if (precision != TRN_PRECISION_FP64 && precision != TRN_PRECISION_MIXED)
    return fail(m, TRN_ERR_INVALID, "quality_adjoint: unknown precision");
  if (grad_solut && !solut)
    return fail(m, TRN_ERR_INVALID, "quality_adjoint: grad_solut needs a solution");
  if (solut && (norm < 0 || h_min <= 0 || h_max <= 0))
    return fail(m, TRN_ERR_INVALID, "quality_adjoint: bad metric parameters");
  m->err.clear();
  if (adj_ws_ensure(&m->adj, m->nb_nodes, m->nb_elems))
    return fail(m, TRN_ERR_CUDA, "quality_adjoint: device allocation failed");
  AdjMetric um;
  if (solut) {
    um.solut = solut;
    um.grad = m->grad;
    um.terms = m->terms;
    um.exact_sum = m->exact_sum || m->replay;
    um.p.target = (double) (int) std::floor(m->nb_nodes * target_factor);
    um.p.scale_exp = norm ? -1. / (2 * norm + 2) : 0.5;
    um.p.eig_min = 1 / trn_pow(h_min, 2);
    um.p.eig_max = 1 / trn_pow(h_max, 2);
  }
  begin_timing(m);
  quality_adjoint(m->d, m->nb_nodes, m->nb_elems, reinterpret_cast<const double2*>(xy),
                  solut ? &um : nullptr, precision == TRN_PRECISION_MIXED, m->adj, grad_xy,
                  grad_solut, m->stream);
  CK(cudaMemcpyAsync(m->h_status + H_WIDE, m->adj.scal + 1, sizeof(double), cudaMemcpyDeviceToHost,
                     m->stream));
  int rc = sync_status(m);
  if (rc) return rc;
  if (value) std::memcpy(value, m->h_status + H_WIDE, sizeof(double));
  return end_timing(m, nullptr, m->nb_elems, m->nb_nodes);
}

/* gradient-based smoothing: steps passes over the color classes of the
 * interior vertices, each vertex moving up the gradient of its elements'
 * summed quality or log-quality (free mode only: the reference has no such
 * pass) */
int trn_smooth_gradient_run(trn_mesh* m, int max_colors, int steps, double max_len, int mode,
                            trn_stats* st) {
  if (!m || m->nb_nodes <= 0) return fail(m, TRN_ERR_INVALID, "smooth_gradient: no mesh loaded");
  if (m->replay) return fail(m, TRN_ERR_INVALID, "smooth_gradient: not available in replay mode");
  if (steps < 0 || !(max_len > 0) || (mode & ~(TRN_SMOOTH_LOG_Q | TRN_SMOOTH_TENSOR_FOLLOWS)))
    return fail(m, TRN_ERR_INVALID, "smooth_gradient: bad parameters");
  int max_col = std::max(6, max_colors) - 1;
  if (max_col > 30) max_col = 30;
  m->err.clear();
  begin_timing(m);
  cudaStream_t s = m->stream;
  smooth_pre(m->d, m->nb_nodes, s);
  build_vicin(m->d, m->nb_nodes, true, s);
  color_jp(m->d, m->nb_nodes, max_col, seed_of(m, 0xc01dULL), m->hws, m->parts, m->status + S_PARTS,
           reinterpret_cast<unsigned*>(m->status + S_TICK), s);
  int rc = sync_status(m);
  if (rc) return rc;
  std::vector<std::pair<const int*, int>> classes;
  for (int c = 0; c < max_col && c < 8; ++c) {
    int a = m->h_status[S_PARTS + c], b = m->h_status[S_PARTS + c + 1];
    classes.emplace_back(m->parts + a, b - a);
  }
  quality_all(m->d, m->nb_elems, m->fp32, s);
  CK(cudaMemsetAsync(m->status + S_SMOOTH_TASKS, 0, sizeof(int) * 2, s));
  for (int step = 0; step < steps; ++step)
    for (auto& c : classes)
      smooth_gradient_color(m->d, c.first, c.second, max_len, mode, m->status + S_SMOOTH_TASKS,
                            m->fp32, s);
  if ((rc = sync_status(m))) return rc;
  return end_timing(m, st, m->h_status[S_SMOOTH_TASKS], m->h_status[S_SMOOTH_COMMIT]);
}

/* ---------------- a captured round ----------------
 * The whole free-mode round as one CUDA graph: the refinement levels, then
 * coarsening, swapping and the coloring's batches as loop nodes whose body
 * is one level (the device decides, in k_fix_level_end / k_color_batch_end,
 * whether it runs again), then the smoothing passes over the device-side
 * color classes. Grids are sized by the capacities; every count is read on
 * the device. The kernels and seeds are those of the per-stage calls, so a
 * captured round ends where trn_round_run ends. */
}  /* extern "C" */

namespace {

template <class F>
cudaError_t capture_loop(cudaStream_t s, cudaStream_t bs, F&& body) {
  cudaStreamCaptureStatus st;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  cudaError_t e = cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd);
  if (e != cudaSuccess) return e;
  if (st != cudaStreamCaptureStatusActive) return cudaErrorStreamCaptureInvalidated;
  cudaGraphConditionalHandle h;
  if ((e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault)) != cudaSuccess) return e;
  cudaGraphNodeParams p = {};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  if ((e = cudaGraphAddNode(&node, g, deps, nd, &p)) != cudaSuccess) return e;
  cudaGraph_t bodyg = p.conditional.phGraph_out[0];
  if ((e = cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies)) != cudaSuccess)
    return e;
  if ((e = cudaStreamBeginCaptureToGraph(bs, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
      cudaSuccess)
    return e;
  body(bs, h);
  return cudaStreamEndCapture(bs, &bodyg);
}

int capture_round(trn_mesh* m, int depth) {
  if (m->round_exec) {
    cudaGraphExecDestroy(m->round_exec);
    m->round_exec = nullptr;
  }
  if (!m->body_stream) CK(cudaStreamCreateWithFlags(&m->body_stream, cudaStreamNonBlocking));
  if (!m->rstats) CK(cudaMalloc(&m->rstats, sizeof(int) * 8));
  cudaStream_t s = m->stream, bs = m->body_stream;
  const int max_col = max_colors_of(8);
  unsigned* tick = reinterpret_cast<unsigned*>(m->status + S_TICK);
  set_thread_tune(&m->tune);
  const unsigned long long l0 = thread_launches();
  CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  auto stage_stats = [&](int k) {
    cudaMemcpyAsync(m->rstats + 2 * k, m->status + S_EVAL, sizeof(int) * 2, cudaMemcpyDeviceToDevice, s);
  };
  cudaError_t e = cudaSuccess;
  enq_refine(m, depth, s);
  stage_stats(0);
  enq_coarsen_begin(m, s, true);
  if (e == cudaSuccess)
    e = capture_loop(s, bs, [&](cudaStream_t b, cudaGraphConditionalHandle h) {
      enq_coarsen_level(m, b, -1, h, true);
    });
  stage_stats(1);
  enq_swap_begin(m, s, true);
  if (e == cudaSuccess)
    e = capture_loop(s, bs, [&](cudaStream_t b, cudaGraphConditionalHandle h) {
      enq_swap_level(m, b, -1, h, true);
    });
  stage_stats(2);
  smooth_pre(m->d, m->capa_node, s);
  build_vicin(m->d, m->capa_node, true, s);
  color_begin(m->d, m->capa_node, m->hws, s);
  if (e == cudaSuccess)
    e = capture_loop(s, bs, [&](cudaStream_t b, cudaGraphConditionalHandle h) {
      color_batch(m->d, m->capa_node, max_col, seed_of(m, 0xc01dULL), m->hws, b, h, true);
    });
  color_finish(m->d, m->capa_node, max_col, m->hws, m->parts, m->status + S_PARTS, tick, s);
  quality_all(m->d, m->capa_elem, m->fp32, s);
  cudaMemsetAsync(m->status + S_SMOOTH_TASKS, 0, sizeof(int) * 2, s);
  for (int level = 0; level < depth; ++level)
    for (int c = 0; c < max_col && c < 8; ++c)
      smooth_class(m->d, m->parts, m->status + S_PARTS, c, m->capa_node, m->status + S_SMOOTH_TASKS,
                   m->fp32, s);
  cudaMemcpyAsync(m->rstats + 6, m->status + S_SMOOTH_TASKS, sizeof(int) * 2, cudaMemcpyDeviceToDevice, s);
  cudaGraph_t g = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(s, &g);
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&m->round_exec, g, 0);
  if (g) cudaGraphDestroy(g);
  cudaGetLastError();
  if (e != cudaSuccess) {
    m->round_exec = nullptr;
    return fail(m, TRN_ERR_CUDA, std::string("round capture: ") + cudaGetErrorString(e));
  }
  m->round_depth = depth;
  m->round_tune = m->tune;
  m->round_fp32 = m->fp32;
  m->round_seed = m->seed;
  m->round_swap_match = m->swap_match;
  m->round_level_cap = m->level_cap;
  m->round_launches = thread_launches() - l0;
  return TRN_OK;
}

}  // namespace

extern "C" {

int trn_round_graph_run(trn_mesh* m, int depth, trn_stats stats[4]) {
  if (!m || m->nb_nodes <= 0) return fail(m, TRN_ERR_INVALID, "round: no mesh loaded");
  if (depth < 1) return fail(m, TRN_ERR_INVALID, "round: depth < 1");
  if (m->replay) return fail(m, TRN_ERR_INVALID, "round: a captured round runs the free mode only");
  m->err.clear();
  if (!m->round_exec || m->round_depth != depth || m->round_fp32 != m->fp32 || m->round_seed != m->seed ||
      m->round_swap_match != m->swap_match || m->round_level_cap != m->level_cap ||
      !(m->round_tune == m->tune)) {
    int rc = capture_round(m, depth);
    if (rc) return rc;
  }
  begin_timing(m);
  CK(cudaGraphLaunch(m->round_exec, m->stream));
  note_launches(m->round_launches);
  CK(cudaMemcpyAsync(m->h_status + H_STATS, m->rstats, sizeof(int) * 8, cudaMemcpyDeviceToHost, m->stream));
  int rc = sync_status(m);
  if (rc) return rc;
  m->nb_nodes = m->h_status[S_NB];
  m->nb_elems = m->h_status[S_NB + 1];
  rc = end_timing(m, nullptr, 0, 0);
  if (stats)
    for (int k = 0; k < 4; ++k) {
      stats[k].eval += m->h_status[H_STATS + 2 * k];
      stats[k].task += m->h_status[H_STATS + 2 * k + 1];
      if (k == 0) stats[k].elap += (int) m->last_ms;
    }
  return rc;
}

/* ---------------- launch-shape autotuner ---------------- */
int trn_get_tune(trn_mesh* m, int cfg[TRN_TUNE_N]) {
  if (!m || !cfg) return TRN_ERR_INVALID;
  const Tune& t = m->tune;
  cfg[0] = t.smooth_threads;
  cfg[1] = t.filter_threads;
  cfg[2] = t.group_lanes;
  cfg[3] = t.group_max;
  cfg[4] = t.flip_threads;
  cfg[5] = t.smooth_lanes;
  cfg[6] = t.smooth_regs;
  return TRN_OK;
}

int trn_set_tune(trn_mesh* m, const int cfg[TRN_TUNE_N]) {
  if (!m || !cfg) return TRN_ERR_INVALID;
  auto pow2_in = [](int v, int lo, int hi) { return v >= lo && v <= hi && (v & (v - 1)) == 0; };
  if (!pow2_in(cfg[0], 32, 256) || !pow2_in(cfg[1], 32, 1024) || (cfg[2] != 1 && cfg[2] != 4 && cfg[2] != 8 && cfg[2] != 16) ||
      cfg[3] < 0 || !pow2_in(cfg[4], 32, 1024) || (cfg[5] != 1 && cfg[5] != 2 && cfg[5] != 4 && cfg[5] != 8) ||
      cfg[6] < 0 || cfg[6] > 8)
    return fail(m, TRN_ERR_INVALID, "set_tune: value out of range");
  m->tune.smooth_threads = cfg[0];
  m->tune.filter_threads = cfg[1];
  m->tune.group_lanes = cfg[2];
  m->tune.group_max = cfg[3];
  m->tune.flip_threads = cfg[4];
  m->tune.smooth_lanes = cfg[5];
  m->tune.smooth_regs = cfg[6];
  return TRN_OK;
}

/* Launch shapes timed on this mesh (the best of three runs of metric +
 * rounds from the loaded input, device time of the rounds). First the
 * smoothing's lanes a vertex and register / back-off variant jointly (they
 * interact: two lanes a vertex pay off only with the one-sweep tries), then
 * coordinate descent over every parameter: the current value and then every
 * other candidate with the others at their best so far. A candidate replaces
 * the value kept only when it is at least 1 % faster (run-to-run noise is
 * about that). The shapes change no result, only the time. The mesh is
 * reloaded at the end. */
int trn_autotune(trn_mesh* m, double target_factor, int norm, double h_min, double h_max, int depth,
                 int rounds, int cfg[TRN_TUNE_N]) {
  if (!m || !m->pts0) return fail(m, TRN_ERR_INVALID, "autotune: nothing loaded");
  if (m->replay) return fail(m, TRN_ERR_INVALID, "autotune: free mode only");
  if (depth < 1 || rounds < 1) return fail(m, TRN_ERR_INVALID, "autotune: bad depth or rounds");
  int rc = TRN_OK;
  auto measure = [&](double* out) -> int {
    double best = 1e300;
    for (int rep = 0; rep < 3; ++rep) {
      int r;
      if ((r = trn_mesh_reload(m)) || (r = trn_metric_run(m, target_factor, norm, h_min, h_max, nullptr)))
        return r;
      double ms = 0;
      for (int k = 0; k < rounds; ++k) {
        if ((r = trn_refine_run(m, depth, nullptr))) return r;
        ms += m->last_ms;
        if ((r = trn_coarsen_run(m, 8, nullptr))) return r;
        ms += m->last_ms;
        if ((r = trn_swap_run(m, nullptr))) return r;
        ms += m->last_ms;
        if ((r = trn_smooth_run(m, 8, depth, nullptr))) return r;
        ms += m->last_ms;
      }
      best = std::min(best, ms);
    }
    *out = best;
    return TRN_OK;
  };
  int* fields[TRN_TUNE_N] = {&m->tune.smooth_lanes, &m->tune.smooth_threads, &m->tune.smooth_regs,
                             &m->tune.filter_threads, &m->tune.group_lanes, &m->tune.group_max,
                             &m->tune.flip_threads};
  const std::vector<std::vector<int>> cands = {
      {1, 2, 4, 8}, {64, 128, 256}, {0, 1, 2, 3, 4, 5, 6, 7, 8}, {128, 256, 512}, {4, 8, 16}, {4096, 16384, 65536}, {128, 256, 512}};
  {
    int best_l = m->tune.smooth_lanes, best_r = m->tune.smooth_regs;
    double best_ms;
    rc = measure(&best_ms);
    for (int l : cands[0]) {
      for (int r : cands[2]) {
        if (rc != TRN_OK) break;
        if ((l == best_l && r == best_r) || (l == 1 && r > 2)) continue;  /* one lane: 0-2 only */
        m->tune.smooth_lanes = l;
        m->tune.smooth_regs = r;
        double ms;
        if ((rc = measure(&ms))) break;
        if (ms < 0.99 * best_ms) {
          best_ms = ms;
          best_l = l;
          best_r = r;
        }
      }
    }
    m->tune.smooth_lanes = best_l;
    m->tune.smooth_regs = best_r;
  }
  for (int f = 0; f < TRN_TUNE_N && rc == TRN_OK; ++f) {
    int best_v = *fields[f];
    double best_ms;
    if ((rc = measure(&best_ms))) break;
    for (int v : cands[f]) {
      if (v == best_v) continue;
      *fields[f] = v;
      double ms;
      if ((rc = measure(&ms))) break;
      if (ms < 0.99 * best_ms) {
        best_ms = ms;
        best_v = v;
      }
    }
    *fields[f] = best_v;
  }
  if (rc == TRN_OK) rc = trn_mesh_reload(m);
  if (rc == TRN_OK && cfg) trn_get_tune(m, cfg);
  return rc;
}

int trn_round_run(trn_mesh* m, int depth, trn_stats stats[4]) {
  int rc;
  if ((rc = trn_refine_run(m, depth, stats ? stats + 0 : nullptr))) return rc;
  if ((rc = trn_coarsen_run(m, 8, stats ? stats + 1 : nullptr))) return rc;
  if ((rc = trn_swap_run(m, stats ? stats + 2 : nullptr))) return rc;
  return trn_smooth_run(m, 8, depth, stats ? stats + 3 : nullptr);
}

}  /* extern "C" */
