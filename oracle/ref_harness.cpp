/*
 * ref_harness.cpp — test infrastructure, not product code.
 *
 * Drives the UNMODIFIED reference library (trinity's own sources, compiled by
 * oracle/Makefile into oracle/_ref/) through its public API, in the order of
 * trinity's src/main.cpp:40-57:
 *   Mesh(size, bucket, depth, verb, rounds); Metrics; Partit(&mesh, 8);
 *   Refine(&mesh, depth); Swap; Coarse(&mesh, &heuris); Smooth(&mesh, &heuris, depth);
 *   load; metric.run(); for r < rounds { refine; coarse; swap; smooth }.
 *
 * One deliberate difference from main.cpp: the Mesh constructor is given a
 * "capacity depth" instead of the refinement depth. The reference derives only
 * its storage capacity from that argument (capa.scale = (depth-1)*3,
 * src/mesh.cpp:30; param.depth is read nowhere else), and depth 1 gives a zero
 * capacity (crash) while depth 2 overflows on small meshes. Refine and Smooth
 * still receive the real depth, so the algorithm is untouched.
 *
 * Outputs:
 *   --dump PREFIX : after the metric and after every kernel, a binary snapshot
 *                   PREFIX.<stage>.bin of the full-precision mesh state (the
 *                   class internals are reached by compiling with
 *                   -Dprivate=public; no reference source is edited).
 *   --final PATH  : the same snapshot, after the last round only.
 *   --time        : one JSON line with the wall time of Mesh::load and
 *                   per-kernel wall times (std::chrono),
 *                   the active triangle count at the start of every round,
 *                   the final counts and each kernel's statistics summed over
 *                   the rounds ([eval, task] for refine, coarse, swap, smooth).
 */
#include "trinity.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

using namespace trinity;
using Clock = std::chrono::steady_clock;

static double ms_since(Clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

static int count_active_elems(const Mesh& m) {
  int c = 0;
  for (int i = 0; i < m.nb.elems; ++i)
    if (m.topo.elems[i * 3] > -1) ++c;
  return c;
}

/* snapshot layout (little endian):
 *   int32 magic 0x54524e31, int32 nb_nodes, int32 nb_elems
 *   f64 points[2*nb_nodes], f64 tensor[3*nb_nodes], i32 elems[3*nb_elems]
 *   u8 alive[nb_nodes] (stencil non-empty), u8 tags[nb_nodes]            */
static void dump(const Mesh& m, const std::string& path) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) { std::perror(path.c_str()); std::exit(2); }
  int hdr[3] = {0x54524e31, m.nb.nodes, m.nb.elems};
  std::fwrite(hdr, sizeof(int), 3, f);
  std::fwrite(m.geom.points.data(), sizeof(double), (size_t) 2 * m.nb.nodes, f);
  std::fwrite(m.geom.tensor.data(), sizeof(double), (size_t) 3 * m.nb.nodes, f);
  std::fwrite(m.topo.elems.data(), sizeof(int), (size_t) 3 * m.nb.elems, f);
  std::vector<unsigned char> alive((size_t) m.nb.nodes), tags((size_t) m.nb.nodes);
  for (int i = 0; i < m.nb.nodes; ++i) {
    alive[i] = m.topo.stenc[i].empty() ? 0 : 1;
    tags[i] = m.sync.tags[i];
  }
  std::fwrite(alive.data(), 1, alive.size(), f);
  std::fwrite(tags.data(), 1, tags.size(), f);
  std::fclose(f);
}

int main(int argc, char* argv[]) {
  if (argc < 8) {
    std::fprintf(stderr,
      "usage: %s mesh bb rounds depth bucket target norm "
      "[--capa-depth D] [--dump PREFIX] [--final PATH] [--time] [--out result.mesh]\n", argv[0]);
    return 1;
  }
  std::string input = argv[1], solut = argv[2];
  int rounds = std::atoi(argv[3]);
  int depth = std::atoi(argv[4]);
  int bucket = std::atoi(argv[5]);
  double target = std::atof(argv[6]);
  int norm = std::atoi(argv[7]);
  int capa_depth = 4;
  std::string prefix, out, final_path;
  bool timing = false;
  for (int i = 8; i < argc; ++i) {
    if (!std::strcmp(argv[i], "--capa-depth") && i + 1 < argc) capa_depth = std::atoi(argv[++i]);
    else if (!std::strcmp(argv[i], "--dump") && i + 1 < argc) prefix = argv[++i];
    else if (!std::strcmp(argv[i], "--out") && i + 1 < argc) out = argv[++i];
    else if (!std::strcmp(argv[i], "--final") && i + 1 < argc) final_path = argv[++i];
    else if (!std::strcmp(argv[i], "--time")) timing = true;
  }

  std::ifstream file(input, std::ios::in);
  if (!file.good()) { std::fprintf(stderr, "cannot open %s\n", input.c_str()); return 2; }
  int size[] = {io::find("Vertices", file), io::find("Triangles", file)};
  file.close();

  double const h_min = EPSILON, h_max = 0.4;  // src/parser.cpp:95-96
  Mesh mesh(size, bucket, capa_depth, 0, rounds);
  Metrics metric(&mesh, target, norm, h_min, h_max);
  Partit heuris(&mesh, 8);
  Refine refine(&mesh, depth);
  Swap swap(&mesh);
  Coarse coarse(&mesh, &heuris);
  Smooth smooth(&mesh, &heuris, depth);
  Stats stat[5];

  auto tl = Clock::now();
  mesh.load(input, solut);
  const double t_load = ms_since(tl);
  if (!prefix.empty()) dump(mesh, prefix + ".load.bin");

  std::vector<int> t_in;
  double t_metric, t_k[4] = {0, 0, 0, 0};
  auto t0 = Clock::now();
  metric.run(stat);
  t_metric = ms_since(t0);
  if (!prefix.empty()) dump(mesh, prefix + ".metric.bin");

  for (int r = 0; r < rounds; ++r) {
    t_in.push_back(count_active_elems(mesh));
    auto t = Clock::now();
    refine.run(stat + 1);
    t_k[0] += ms_since(t);
    if (!prefix.empty()) dump(mesh, prefix + ".r" + std::to_string(r) + ".refine.bin");
    t = Clock::now();
    coarse.run(stat + 2);
    t_k[1] += ms_since(t);
    if (!prefix.empty()) dump(mesh, prefix + ".r" + std::to_string(r) + ".coarse.bin");
    t = Clock::now();
    swap.run(stat + 3);
    t_k[2] += ms_since(t);
    if (!prefix.empty()) dump(mesh, prefix + ".r" + std::to_string(r) + ".swap.bin");
    t = Clock::now();
    smooth.run(stat + 4);
    t_k[3] += ms_since(t);
    if (!prefix.empty()) dump(mesh, prefix + ".r" + std::to_string(r) + ".smooth.bin");
  }
  if (!final_path.empty()) dump(mesh, final_path);
  if (!out.empty()) mesh.store(out);

  if (timing) {
    int nodes = 0;
    for (int i = 0; i < mesh.nb.nodes; ++i) nodes += mesh.topo.stenc[i].empty() ? 0 : 1;
    std::printf("\n{\"threads\": %d, \"load_ms\": %.3f, \"metric_ms\": %.3f, \"refine_ms\": %.3f, "
                "\"coarse_ms\": %.3f, \"swap_ms\": %.3f, \"smooth_ms\": %.3f, "
                "\"rounds_ms\": %.3f, \"tri_in\": [",
                omp_get_max_threads(), t_load, t_metric, t_k[0], t_k[1], t_k[2], t_k[3],
                t_k[0] + t_k[1] + t_k[2] + t_k[3]);
    for (size_t i = 0; i < t_in.size(); ++i)
      std::printf("%s%d", i ? ", " : "", t_in[i]);
    std::printf("], \"nodes_out\": %d, \"elems_out\": %d, \"stats\": [", nodes,
                count_active_elems(mesh));
    for (int k = 1; k < 5; ++k)
      std::printf("%s[%d, %d]", k > 1 ? ", " : "", stat[k].eval, stat[k].task);
    std::printf("]}\n");
  }
  return 0;
}
