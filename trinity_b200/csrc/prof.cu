/*
 * prof.cu — optional per-launch device timing.
 *
 * When enabled, every kernel launcher brackets its launch(es) with a pair of
 * CUDA events on the launching stream; after the next stream synchronisation
 * the elapsed times are folded into per-kernel totals together with the
 * launcher's algorithmic byte count (distinct entries the launch must touch,
 * each counted once, no cache credit). Disabled, a scope costs one branch.
 * Each timed scope records two events on the stream (about 1 us of device
 * time each between launches), so a throughput measurement can restrict the
 * timing to one kernel's scopes (trn_profile_only).
 */
#include "trn_internal.h"

#include <atomic>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

namespace trn {

namespace {

struct Pending {
  int id;
  cudaEvent_t a, b;
  double bytes;
  int slot;   /* device byte counter of the scope, -1: the launcher's figure */
};

struct Total {
  std::string name;
  long long launches = 0;
  double ms = 0.0;
  double bytes = 0.0;
  long long counted = 0;   /* launches whose bytes the kernel counted */
};

struct Profiler {
  std::mutex mu;   /* meshes may run on several host threads */
  std::atomic<bool> on{false};
  std::string only;   /* time only the scopes of this name ("" = all) */
  std::vector<cudaEvent_t> pool;
  std::vector<Pending> pending;
  std::vector<Total> totals;
  /* counted bytes: one device counter per scope, and a vertex bitmap the
   * counting kernels mark distinct entries in */
  bool counting = false;
  unsigned long long* d_bytes = nullptr;
  std::vector<unsigned long long> h_bytes;
  int next_slot = 0;
  unsigned* d_seen = nullptr;
  size_t seen_words = 0;

  cudaEvent_t get() {
    if (pool.empty()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      return e;
    }
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
  }

  int id_of(const char* name) {
    for (size_t i = 0; i < totals.size(); ++i)
      if (totals[i].name == name) return (int) i;
    totals.push_back(Total());
    totals.back().name = name;
    return (int) totals.size() - 1;
  }
};

Profiler& prof() {
  static Profiler p;
  return p;
}

}  // namespace

constexpr int kByteSlots = 16384;

ProfScope::ProfScope(const char* name, cudaStream_t s, double bytes, ByteCount* count) : stream_(s) {
  Profiler& p = prof();
  if (count) *count = ByteCount();
  if (!p.on) return;
  cudaStreamCaptureStatus cs;
  if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) return;
  std::lock_guard<std::mutex> lock(p.mu);
  if (!p.only.empty() && p.only != name) return;
  id_ = p.id_of(name);
  bytes_ = bytes;
  if (count && p.counting && p.d_bytes && p.next_slot < kByteSlots) {
    slot_ = p.next_slot++;
    count->bytes = p.d_bytes + slot_;
    count->seen = p.d_seen;
    cudaMemsetAsync(count->bytes, 0, sizeof(unsigned long long), s);
    cudaMemsetAsync(p.d_seen, 0, sizeof(unsigned) * p.seen_words, s);
  }
  a_ = p.get();
  cudaEventRecord(a_, s);
}

ProfScope::~ProfScope() {
  Profiler& p = prof();
  if (!p.on || id_ < 0) return;
  std::lock_guard<std::mutex> lock(p.mu);
  cudaEvent_t b = p.get();
  cudaEventRecord(b, stream_);
  p.pending.push_back({id_, a_, b, bytes_, slot_});
}

static std::atomic<unsigned long long> g_launches{0};
constexpr size_t kEventPool = 65536;

/* per host thread as well: a round captured on one thread counts only its own launches */
static thread_local unsigned long long t_launches = 0;

void note_launch() {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  ++t_launches;
}
void note_launches(unsigned long long n) {
  g_launches.fetch_add(n, std::memory_order_relaxed);
  t_launches += n;
}
unsigned long long thread_launches() { return t_launches; }

void prof_flush() {
  Profiler& p = prof();
  std::lock_guard<std::mutex> lock(p.mu);
  if (p.next_slot > 0) {
    if (!p.pending.empty()) cudaEventSynchronize(p.pending.back().b);
    p.h_bytes.resize((size_t) p.next_slot);
    cudaMemcpy(p.h_bytes.data(), p.d_bytes, sizeof(unsigned long long) * (size_t) p.next_slot,
               cudaMemcpyDeviceToHost);
  }
  for (auto& q : p.pending) {
    cudaEventSynchronize(q.b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, q.a, q.b);
    Total& t = p.totals[q.id];
    t.launches += 1;
    t.ms += ms;
    t.bytes += q.slot >= 0 ? (double) p.h_bytes[(size_t) q.slot] : q.bytes;
    if (q.slot >= 0) t.counted += 1;
    p.pool.push_back(q.a);
    p.pool.push_back(q.b);
  }
  p.pending.clear();
  p.next_slot = 0;
}

}  // namespace trn

extern "C" {

int trn_profile_enable(int on) {
  trn::Profiler& p = trn::prof();
  trn::prof_flush();
  std::lock_guard<std::mutex> lock(p.mu);
  p.on = on != 0;
  if (on) {
    p.totals.clear();
    /* events are created here, not inside the timed launches: a few
     * thousand scopes per adaptation step, two events each */
    while (p.pool.size() < trn::kEventPool) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) break;
      p.pool.push_back(e);
    }
  }
  return 0;
}

int trn_profile_only(const char* name) {
  trn::Profiler& p = trn::prof();
  trn::prof_flush();
  std::lock_guard<std::mutex> lock(p.mu);
  p.only = name ? name : "";
  return 0;
}

/* algorithmic bytes counted by the kernels that can count them (distinct
 * entries each launch touches, marked on the device) instead of the
 * launchers' figures; for profiled, untimed runs: the counting costs atomics.
 * max_nodes sizes the bitmap of distinct vertices. */
int trn_profile_count_bytes(int on, int max_nodes) {
  trn::Profiler& p = trn::prof();
  trn::prof_flush();
  std::lock_guard<std::mutex> lock(p.mu);
  p.counting = on != 0;
  if (on) {
    if (!p.d_bytes && cudaMalloc(&p.d_bytes, sizeof(unsigned long long) * trn::kByteSlots) != cudaSuccess) {
      p.d_bytes = nullptr;
      p.counting = false;
      return 5;
    }
    const size_t words = ((size_t) (max_nodes > 0 ? max_nodes : 1) + 31) / 32;
    if (words > p.seen_words) {
      cudaFree(p.d_seen);
      if (cudaMalloc(&p.d_seen, sizeof(unsigned) * words) != cudaSuccess) {
        p.d_seen = nullptr;
        p.seen_words = 0;
        p.counting = false;
        return 5;
      }
      p.seen_words = words;
    }
  }
  return 0;
}

unsigned long long trn_launch_count(void) { return trn::g_launches.load(); }

int trn_profile_count(void) {
  trn::prof_flush();
  return (int) trn::prof().totals.size();
}

int trn_profile_counted(int i) {
  trn::Profiler& p = trn::prof();
  if (i < 0 || i >= (int) p.totals.size()) return -1;
  return (int) p.totals[i].counted;
}

int trn_profile_entry(int i, char* name, int name_len, long long* launches, double* ms,
                      double* bytes) {
  trn::Profiler& p = trn::prof();
  if (i < 0 || i >= (int) p.totals.size()) return 3;
  const trn::Total& t = p.totals[i];
  if (name && name_len > 0) {
    std::strncpy(name, t.name.c_str(), (size_t) name_len - 1);
    name[name_len - 1] = 0;
  }
  if (launches) *launches = t.launches;
  if (ms) *ms = t.ms;
  if (bytes) *bytes = t.bytes;
  return 0;
}

}  // extern "C"
