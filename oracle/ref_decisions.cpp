/*
 * ref_decisions.cpp — test infrastructure, not product code.
 *
 * Records the decisions of the UNMODIFIED reference's graph heuristics as it
 * runs: linked into oracle/_ref/trinity_ref_decide with the linker's --wrap
 * on three methods, so that every call the reference's kernels make from
 * their own translation units passes through the functions below, which call
 * the reference's own method and then append its result to one int32 stream:
 *
 *   Partit::extractIndepSet (called at coarsening.cpp:493; partition.cpp:200-306)
 *     1  n  v_0 .. v_{n-1}                 task.subset[0], task.cardin[0]
 *   Match::computeGreedyMatching (called at swapping.cpp:410; matching.cpp:81-100)
 *     2  n  k1_0 k2_0 .. k1_{n-1} k2_{n-1}  over the graph rows in order,
 *                                           k1 = graph[row][0], k2 = matched[k1] > -1
 *   Partit::extractColoring (called at smoothing.cpp:287; partition.cpp:79-197)
 *     3  p  c_0 ids.. c_1 ids.. ...          nb.parts parts, task.subset[j]
 *
 * This is the layout of the oracle's decision log (oracle/trn_oracle.h), so
 * a test compares the two streams word for word. The stream is written at
 * exit to the file named by TRN_DECISIONS_OUT (nothing is written when it is
 * unset). The class internals are reached through ref_preinclude.h's
 * widened access specifiers; no reference source is edited.
 */
#include "trinity.h"

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

using trinity::Graph;
using trinity::Match;
using trinity::Mesh;
using trinity::Partit;

namespace {

/* never destroyed: the exit handler below runs after static destructors
 * registered later than it would have */
std::vector<int32_t>& stream() {
  static std::vector<int32_t>* s = new std::vector<int32_t>;
  return *s;
}

void write_stream() {
  const char* path = std::getenv("TRN_DECISIONS_OUT");
  if (!path || !*path) return;
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    std::perror(path);
    return;
  }
  const std::vector<int32_t>& s = stream();
  if (!s.empty()) std::fwrite(s.data(), sizeof(int32_t), s.size(), f);
  std::fclose(f);
}

struct Registrar {
  Registrar() { std::atexit(write_stream); }
} registrar;

}  // namespace

/* the reference's own methods (Itanium ABI: `this` is the first argument) */
extern "C" void __real__ZN7trinity6Partit15extractIndepSetERKSt6vectorIS1_IiSaIiEESaIS3_EEi(
    Partit* self, const Graph& graph, int nb);
extern "C" void __real__ZN7trinity6Partit15extractColoringEPKNS_4MeshE(Partit* self, const Mesh* mesh);
extern "C" int* __real__ZN7trinity5Match21computeGreedyMatchingERKSt6vectorIS1_IiSaIiEESaIS3_EEi(
    Match* self, const Graph& graph, int nb);

extern "C" void __wrap__ZN7trinity6Partit15extractIndepSetERKSt6vectorIS1_IiSaIiEESaIS3_EEi(
    Partit* self, const Graph& graph, int nb) {
  __real__ZN7trinity6Partit15extractIndepSetERKSt6vectorIS1_IiSaIiEESaIS3_EEi(self, graph, nb);
  std::vector<int32_t>& s = stream();
  const int n = self->task.cardin[0];
  s.push_back(1);
  s.push_back(n);
  for (int i = 0; i < n; ++i) s.push_back(self->task.subset[0][i]);
}

extern "C" void __wrap__ZN7trinity6Partit15extractColoringEPKNS_4MeshE(Partit* self, const Mesh* mesh) {
  __real__ZN7trinity6Partit15extractColoringEPKNS_4MeshE(self, mesh);
  std::vector<int32_t>& s = stream();
  const int parts = self->nb.parts;
  s.push_back(3);
  s.push_back(parts);
  for (int j = 0; j < parts; ++j) {
    s.push_back(self->task.cardin[j]);
    for (int a = 0; a < self->task.cardin[j]; ++a) s.push_back(self->task.subset[j][a]);
  }
}

extern "C" int* __wrap__ZN7trinity5Match21computeGreedyMatchingERKSt6vectorIS1_IiSaIiEESaIS3_EEi(
    Match* self, const Graph& graph, int nb) {
  int* matched = __real__ZN7trinity5Match21computeGreedyMatchingERKSt6vectorIS1_IiSaIiEESaIS3_EEi(self, graph, nb);
  std::vector<int32_t>& s = stream();
  int pairs = 0;
  for (int row = 0; row < nb; ++row)
    if (matched[graph[row][0]] > -1) ++pairs;
  s.push_back(2);
  s.push_back(pairs);
  for (int row = 0; row < nb; ++row) {
    const int k1 = graph[row][0];
    const int k2 = matched[k1];
    if (k2 > -1) {
      s.push_back(k1);
      s.push_back(k2);
    }
  }
  return matched;
}
