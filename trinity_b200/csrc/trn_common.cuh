/*
 * trn_common.cuh — device-side mesh layout and helpers shared by all kernels.
 *
 * HBM layout of one mesh (capacities fixed at creation; ids are never reused,
 * deleted entities keep their slot):
 *   pts   double2[capa_node]        vertex coordinates
 *   ten   double4[capa_node]        metric tensor (m11, m12, m22, unused):
 *                                   32-byte records, one sector per gather
 *   tri   int4[capa_elem]           vertex ids (x,y,z), x = -1 when erased
 *   stenc int[capa_node * bucket]   vertex -> incident elements (the
 *                                   reference's "stencil", mesh.h:112), first
 *                                   deg[v] slots used, appended atomically
 *   vic   int[capa_node * bucket]   vertex -> adjacent vertices, sorted
 *                                   (the reference's "vicin", mesh.h:113)
 *   tags/alive/fixes  uint8 per vertex; activ int8 shared by vertices and
 *                                   elements exactly like mesh.h:146
 *   qual  double[capa_elem]         cached element quality
 */
#ifndef TRN_COMMON_CUH
#define TRN_COMMON_CUH

#include <cstdint>
#include <cuda_runtime.h>

#define TRN_TAG_BOUND 4   /* header.h:58 */
#define TRN_TAG_CORNER 8  /* header.h:59 */
#define TRN_MAX_PART 8    /* main.cpp:42, Partit(&mesh, 8) */
#define TRN_MATCHED (-2)  /* matching.h:27 */

/* device error word values (mirror the C-ABI codes) */
#define TRN_DERR_CAPACITY 1    /* vertex or element slots */
#define TRN_DERR_BUCKET 2      /* a stencil, adjacency row or patch longer than its bucket */
#define TRN_DERR_HASH 5        /* the refinement's edge table is full */
#define TRN_DERR_INVALID 3
#define TRN_DERR_NO_PROGRESS 4
#define TRN_DERR_REPLAY 6

/* per-thread scratch limits (local memory) */
#define TRN_MAX_PATCH 512   /* 2-ring element patch of the metric */
#define TRN_MAX_DEG 256     /* stencil entries of one vertex (bucket <= 256) */

#define TRN_THREADS 256

struct DMesh {
  double2* pts;
  double4* ten;
  double4* lten;   /* per-vertex tensor logarithm P log(D) P^T (4 entries) */
  float4* tenf;    /* single-precision copy of ten, kept in the mixed form */
  int4* tri;
  int* stenc;
  int* deg;
  int* vic;
  int* vdeg;
  uint8_t* tags;
  uint8_t* alive;
  uint8_t* fixes;
  int8_t* activ;
  double* qual;
  int* err;        /* device error word: first error wins */
  int* nb;         /* device slot counts {vertices, elements}, NULL = the
                      launch arguments are the counts */
  /* free-mode worklists (NULL in replay): ids whose activity flag turns
   * 0 -> 1 are appended to act_next, vertices tagged for repair to fix_list */
  int* act_next;
  int* act_next_n;
  int* fix_list;
  int* fix_n;
  int bucket;
  int capa_node;
  int capa_elem;
};

__device__ __forceinline__ void trn_set_error(int* err, int code) {
  atomicCAS(err, 0, code);
}

/* compare-and-swap 0 -> 1 on one byte (sync.h:33-38 compareAndSwap);
 * true for the one caller that made the change. The flags hold 0, 1 or -1
 * (corners), so one atomic OR of bit 0 does it: a byte at 1 or -1 keeps its
 * value, and only the caller that saw 0 returns true */
__device__ __forceinline__ bool trn_byte_cas01(void* p) {
  unsigned int* word = (unsigned int*) ((uintptr_t) p & ~(uintptr_t) 3);
  const unsigned int shift = ((uintptr_t) p & 3) * 8;
  const unsigned int old = atomicOr(word, 1u << shift);
  return ((old >> shift) & 0xffu) == 0u;
}

/* append id to list[*n]; the lanes of a warp that push to the same counter
 * at once share one atomic (a flip pushes up to a dozen ids onto two
 * counters, which one-atomic-per-push serializes in L2) */
__device__ __forceinline__ void trn_list_push(int* list, int* n, int id) {
  const unsigned mask = __activemask();
  const unsigned peers = __match_any_sync(mask, (unsigned long long) (uintptr_t) n);
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(peers) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(n, __popc(peers));
  base = __shfl_sync(peers, base, leader);
  list[base + __popc(peers & ((1u << lane) - 1))] = id;
}

/* tag vertex v for stencil repair (CAS 0 -> 1), listing it once */
__device__ __forceinline__ void trn_tag_fix(const DMesh& m, int v) {
  if (trn_byte_cas01(m.fixes + v) && m.fix_list) trn_list_push(m.fix_list, m.fix_n, v);
}

/* activate vertex or element id (CAS 0 -> 1: corners hold -1 and keep it),
 * listing it once for the next level */
__device__ __forceinline__ void trn_activate(const DMesh& m, int id) {
  if (trn_byte_cas01(m.activ + id) && m.act_next) trn_list_push(m.act_next, m.act_next_n, id);
}

/* *dst += the sum of v over the lanes of the warp that run this together,
 * with one atomic (per-thread tallies at a kernel's end otherwise add up to
 * tens of thousands of atomics on one word) */
__device__ __forceinline__ void trn_warp_add(int* dst, int v) {
  const unsigned mask = __activemask();
  const int s = (int) __reduce_add_sync(mask, (unsigned) v);
  if ((int) (threadIdx.x & 31) == __ffs(mask) - 1 && s) atomicAdd(dst, s);
}

/* a slot of *counter for each lane of the warp that calls this together,
 * reserved with one atomic; every such lane must pass the same counter */
__device__ __forceinline__ int trn_warp_reserve(int* counter) {
  const unsigned mask = __activemask();
  const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(counter, __popc(mask));
  base = __shfl_sync(mask, base, leader);
  return base + __popc(mask & ((1u << lane) - 1));
}

/* append ids[0..k) to list[*n]; the lanes of a warp that push to the same
 * counter at once share one atomic: their ids are laid out slot by slot
 * (every lane's first id, then every lane's second, ...; lists are
 * unordered). A flip or a collapse pushes a few ids onto the shared repair
 * and activity lists, and one atomic per push serialises on those two
 * counters in L2 (a few ns each, for every flip of a level). */
__device__ __forceinline__ void trn_list_push_n(int* list, int* n, const int* ids, int k) {
  const unsigned mask = __activemask();
  const unsigned peers = __match_any_sync(mask, (unsigned long long) (uintptr_t) n);
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const int kmax = (int) __reduce_max_sync(peers, (unsigned) (k > 0 ? k : 0));
  if (kmax == 0) return;
  int total = 0;
  for (int j = 0; j < kmax; ++j) total += __popc(__ballot_sync(peers, j < k));
  const int leader = __ffs(peers) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(n, total);
  base = __shfl_sync(peers, base, leader);
  int off = 0;
  for (int j = 0; j < kmax; ++j) {
    const unsigned b = __ballot_sync(peers, j < k);
    if (j < k) list[base + off + __popc(b & lt)] = ids[j];
    off += __popc(b);
  }
}

/* once any kernel raised the error word, later kernels of the call do no
 * work: a failed append may have left unwritten stencil slots behind */
__device__ __forceinline__ bool trn_failed(const DMesh& m) {
  return *(volatile int*) m.err != 0;
}

/* slot counts: the device copy when the mesh keeps one (it changes on the
 * device during a round), else the count the launch was given */
__device__ __forceinline__ int trn_nodes(const DMesh& m, int given) { return m.nb ? m.nb[0] : given; }
__device__ __forceinline__ int trn_elems(const DMesh& m, int given) { return m.nb ? m.nb[1] : given; }

/* used stencil length of v, never beyond its bucket (an overflowing append
 * only raises the error word, so the counter itself may exceed it) */
__device__ __forceinline__ int trn_deg(const DMesh& m, int v) {
  int d = m.deg[v];
  return d < m.bucket ? d : m.bucket;
}

/* append element t to the stencil of v (mesh.cpp:468-494 updateStencil) */
__device__ __forceinline__ void trn_stenc_append(const DMesh& m, int v, int t) {
  int k = atomicAdd(m.deg + v, 1);
  if (k >= m.bucket) {
    trn_set_error(m.err, TRN_DERR_BUCKET);
    return;
  }
  m.stenc[(size_t) v * m.bucket + k] = t;
}

__device__ __forceinline__ void trn_stenc_append_n(const DMesh& m, int v, const int* t, int n) {
  int k = atomicAdd(m.deg + v, n);
  if (k + n > m.bucket) {
    trn_set_error(m.err, TRN_DERR_BUCKET);
    return;
  }
  int* s = m.stenc + (size_t) v * m.bucket + k;
  for (int i = 0; i < n; ++i) s[i] = t[i];
}

__device__ __forceinline__ void trn_isort(int* a, int n) {
  for (int i = 1; i < n; ++i) {
    int x = a[i], j = i - 1;
    while (j >= 0 && a[j] > x) {
      a[j + 1] = a[j];
      --j;
    }
    a[j + 1] = x;
  }
}

__device__ __forceinline__ int trn_iunique(int* a, int n) {
  if (n == 0) return 0;
  int k = 1;
  for (int i = 1; i < n; ++i)
    if (a[i] != a[k - 1]) a[k++] = a[i];
  return k;
}

/* adjacency of v from its (canonical) stencil: the other two vertices of
 * each element, sorted, without duplicates. A stencil of up to 12 elements
 * stays in registers (its element loads all in flight, an odd-even
 * transposition network over the 24 ids, no local memory); longer ones sort
 * in a local array. Both give the same rows. */
constexpr int kVicRegs = 24;

__device__ __forceinline__ void build_one_vicin(const DMesh& m, int v) {
  if (m.alive[v] && trn_deg(m, v) <= kVicRegs / 2) {
    const int* s = m.stenc + (size_t) v * m.bucket;
    const int d = trn_deg(m, v);
    int r[kVicRegs];
#pragma unroll
    for (int a = 0; a < kVicRegs / 2; ++a) {
      int x = 0x7fffffff, y = 0x7fffffff;
      if (a < d) {
        const int4 n = m.tri[s[a]];
        if (v == n.x) { x = n.y; y = n.z; }
        else if (v == n.y) { x = n.z; y = n.x; }
        else if (v == n.z) { x = n.x; y = n.y; }
      }
      r[2 * a] = x;
      r[2 * a + 1] = y;
    }
#pragma unroll
    for (int p = 0; p < kVicRegs; ++p)
#pragma unroll
      for (int a = p & 1; a + 1 < kVicRegs; a += 2) {
        const int lo = min(r[a], r[a + 1]), hi = max(r[a], r[a + 1]);
        r[a] = lo;
        r[a + 1] = hi;
      }
    int* out = m.vic + (size_t) v * m.bucket;
    int k = 0;
#pragma unroll
    for (int a = 0; a < kVicRegs; ++a)
      if (r[a] != 0x7fffffff && (a == 0 || r[a] != r[a - 1])) {
        if (k < m.bucket) out[k] = r[a];
        ++k;
      }
    if (k > m.bucket) {
      trn_set_error(m.err, TRN_DERR_BUCKET);
      k = m.bucket;
    }
    m.vdeg[v] = k;
    return;
  }
  int buf[2 * TRN_MAX_DEG];
  int k = 0;
  if (m.alive[v]) {
    const int* s = m.stenc + (size_t) v * m.bucket;
    int d = trn_deg(m, v);
    for (int a = 0; a < d; ++a) {
      int4 n = m.tri[s[a]];
      if (v == n.x) { buf[k++] = n.y; buf[k++] = n.z; }
      else if (v == n.y) { buf[k++] = n.z; buf[k++] = n.x; }
      else if (v == n.z) { buf[k++] = n.x; buf[k++] = n.y; }
    }
  }
  trn_isort(buf, k);
  k = trn_iunique(buf, k);
  if (k > m.bucket) {
    trn_set_error(m.err, TRN_DERR_BUCKET);
    k = m.bucket;
  }
  int* out = m.vic + (size_t) v * m.bucket;
  for (int a = 0; a < k; ++a) out[a] = buf[a];
  m.vdeg[v] = k;
}

/* P1 basis gradients of one element, times the 4x factor of hessian.cpp:52
 * (the gradient and Hessian recovery, hessian.cpp:24-153) */
struct ElemGrad {
  double area;
  double d[6];
  int4 v;
};

__device__ __forceinline__ ElemGrad elem_grad(const DMesh& m, int e) {
  ElemGrad g;
  g.v = m.tri[e];
  double2 p0 = m.pts[g.v.x], p1 = m.pts[g.v.y], p2 = m.pts[g.v.z];
  double point[6] = {p0.x, p0.y, p1.x, p1.y, p2.x, p2.y};
  double c0 = point[2] - point[0];
  double c1 = point[4] - point[0];
  double c2 = point[3] - point[1];
  double c3 = point[5] - point[1];
  g.area = 0.5 * (c0 * c3 - c1 * c2);
  double norm = 2 / g.area;
  g.d[0] = norm * (point[3] - point[5]);
  g.d[1] = norm * (point[4] - point[2]);
  g.d[2] = norm * (point[5] - point[1]);
  g.d[3] = norm * (point[0] - point[4]);
  g.d[4] = norm * (point[1] - point[3]);
  g.d[5] = norm * (point[2] - point[0]);
  return g;
}

/* warp-aggregated append of id to list[*count] */
__device__ __forceinline__ void trn_append(int* list, int* count, int id) {
  unsigned mask = __activemask();
  int lane = threadIdx.x & 31;
  int leader = __ffs(mask) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(count, __popc(mask));
  base = __shfl_sync(mask, base, leader);
  list[base + __popc(mask & ((1u << lane) - 1))] = id;
}

/* a free-mode level's first kernel, one thread: the activity and repair
 * list counters (and the flip count, when given) start the level empty; the
 * level's later kernels fill them (its candidate count was cleared by the
 * previous level's end) */
__device__ __forceinline__ void trn_level_clear(const DMesh& m, int* flips) {
  if (m.act_next_n) *m.act_next_n = 0;
  if (m.fix_n) *m.fix_n = 0;
  if (flips) *flips = 0;
}

/* trn_failed read once for the whole block, so that every thread of a block
 * that goes on to trn_block_append takes the same branch */
__device__ __forceinline__ bool trn_failed_block(const DMesh& m) {
  __shared__ int s_failed;
  if (threadIdx.x == 0) s_failed = *(volatile int*) m.err;
  __syncthreads();
  return s_failed != 0;
}

/* append id to list[*count] when `want`. Every thread of the block calls it
 * together (from a block-uniform loop): the warps count their appends in
 * shared memory and the block reserves its slots with one global atomic.
 * Appends of many warps onto one counter otherwise serialize in L2 (a few
 * ns each: 62k warp atomics took 170 us when every live element of the 2M
 * workload was listed). */
__device__ __forceinline__ void trn_block_append(int* list, int* count, int id, bool want) {
  __shared__ int s_n, s_base;
  const int lane = threadIdx.x & 31;
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  const unsigned mask = __ballot_sync(0xffffffffu, want);
  int wbase = 0;
  if (lane == 0 && mask) wbase = atomicAdd(&s_n, __popc(mask));
  wbase = __shfl_sync(0xffffffffu, wbase, 0);
  __syncthreads();
  if (threadIdx.x == 0) s_base = s_n ? atomicAdd(count, s_n) : 0;
  __syncthreads();
  if (want) list[s_base + wbase + __popc(mask & ((1u << lane) - 1))] = id;
}

/* seed of a level's hashed priorities: base ^ (tick * mix), tick a device
 * counter that each coarsening / swapping level and each coloring advances,
 * so the seed sequence lives on the device (a captured round replays it) */
struct Seed {
  uint64_t base;
  const unsigned* tick;
  uint64_t mix;
};
__device__ __forceinline__ uint64_t trn_seed(const Seed& s) {
  return s.base ^ ((uint64_t) (s.tick ? *s.tick : 0u) * s.mix);
}

/* 64-bit mix for seeded hash priorities (splitmix64 finaliser) */
__device__ __forceinline__ uint64_t trn_hash64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}

/* priority of id under seed: unique for distinct ids (id in the low bits) */
__device__ __forceinline__ uint64_t trn_prio(uint64_t seed, int id) {
  return (trn_hash64(seed ^ ((uint64_t) (uint32_t) id * 0x632be59bd9b4e019ULL)) & ~0xffffffffULL) |
         (uint32_t) id;
}

__device__ __forceinline__ int trn_grid_stride() { return gridDim.x * blockDim.x; }
__device__ __forceinline__ int trn_tid() { return blockIdx.x * blockDim.x + threadIdx.x; }

#endif
