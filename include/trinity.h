/*
 * trinity.h — C++ class layer over the B200 C ABI (include/trinity_b200.h),
 * with the names, constructor arguments and run() calls of trinity's public
 * API, so that code written against the reference (its src/main.cpp,
 * examples/adapt.cpp) compiles unchanged and runs on the GPU:
 *
 *   Mesh(int size[2], int bucket, int depth, int verbosity, int rounds)   mesh.h:46
 *   Mesh::load(path, solu), Mesh::store(path)                             mesh.h:65-66
 *   Metrics(Mesh*, double target_factor, int Lp_norm, double h_min, double h_max)
 *                                                                         metric.h:38-44
 *   Partit(Mesh const*, int max_part_size)                                partition.h:46
 *   Refine(Mesh*, int level), Coarse(Mesh*, Partit*), Swap(Mesh*),
 *   Smooth(Mesh*, Partit*, int level); each has run(Stats* total = nullptr)
 *   Stats {eval, task, elap, step[5]}                                     header.h:72-77
 *   io::find(key, ifstream&)                                              io.h:27
 *   Parser(argc, argv): the CLI flags and clamps of parser.cpp:37-96,
 *   recap(Stats*) and dump(Stats*)
 *
 * As in the reference the classes are neither copyable nor movable, the mesh
 * must outlive the kernel objects, and calls block. Failures throw
 * std::runtime_error carrying the library's message (the reference asserts).
 */
#pragma once

#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "trinity_b200.h"

#ifndef EPSILON
#define EPSILON 1.e-9
#endif

namespace trinity {

struct Stats : trn_stats {
  Stats() : trn_stats{} {}
};

class Mesh {
 public:
  Mesh() = delete;
  Mesh(const Mesh&) = delete;
  Mesh& operator=(Mesh) = delete;
  Mesh(int size[2], int bucket, int depth, int verbosity, int rounds) : verb_(verbosity) {
    int rc = trn_mesh_create(size, bucket, depth, verbosity, rounds, &h_);
    if (rc) throw std::runtime_error("trinity: mesh creation failed (code " + std::to_string(rc) + ")");
  }
  ~Mesh() { trn_mesh_destroy(h_); }

  void load(const std::string& path, const std::string& solu) {
    check(trn_mesh_load(h_, path.c_str(), solu.empty() ? nullptr : solu.c_str()));
  }
  void store(const std::string& path) const { check(trn_mesh_store(h_, path.c_str())); }
  void storeMetric(const std::string& path) const { check(trn_mesh_store_sol(h_, path.c_str())); }

  int getCapaNode() const { return counts()[0]; }
  int getCapaElem() const { return counts()[1]; }

  trn_mesh* handle() const { return h_; }
  int verbosity() const { return verb_; }
  void check(int rc) const {
    if (rc) throw std::runtime_error(std::string("trinity: ") + trn_last_error(h_));
  }

 private:
  std::vector<int> counts() const {
    int n = 0, e = 0;
    check(trn_mesh_counts(h_, &n, &e, nullptr, nullptr));
    return {n, e};
  }
  trn_mesh* h_ = nullptr;
  int verb_ = 0;
};

class Metrics {
 public:
  Metrics(Mesh* mesh, double target_factor, int Lp_norm, double h_min, double h_max)
      : m_(mesh), target_(target_factor), norm_(Lp_norm), hmin_(h_min), hmax_(h_max) {}
  Metrics(const Metrics&) = delete;
  Metrics& operator=(Metrics) = delete;
  void run(Stats* total = nullptr) {
    m_->check(trn_metric_run(m_->handle(), target_, norm_, hmin_, hmax_, total));
    if (m_->verbosity())
      std::printf("%-18s%s %.2f ms\n", "= metric field", "...", trn_last_time_ms(m_->handle()));
  }

 private:
  Mesh* m_;
  double target_;
  int norm_;
  double hmin_, hmax_;
};

class Partit {
 public:
  Partit(Mesh const* mesh, int max_part_size) : max_part_(std::max(6, max_part_size)) { (void) mesh; }
  Partit(int max_graph_size, int max_part_size) : max_part_(std::max(6, max_part_size)) {
    (void) max_graph_size;
  }
  Partit(const Partit&) = delete;
  Partit& operator=(Partit) = delete;
  int maxPart() const { return max_part_; }

 private:
  int max_part_;
};

namespace detail {
inline void report(const Mesh* m, const char* what) {
  if (m->verbosity()) std::printf("%-18s%s %.2f ms\n", what, "...", trn_last_time_ms(m->handle()));
}
}  // namespace detail

class Refine {
 public:
  Refine(Mesh* input, int level) : m_(input), level_(level) {}
  Refine(const Refine&) = delete;
  Refine& operator=(Refine) = delete;
  void run(Stats* total = nullptr) {
    m_->check(trn_refine_run(m_->handle(), level_, total));
    detail::report(m_, "= refinement");
  }

 private:
  Mesh* m_;
  int level_;
};

class Coarse {
 public:
  Coarse(Mesh* input, Partit* algo) : m_(input), algo_(algo) {}
  Coarse(const Coarse&) = delete;
  Coarse& operator=(Coarse) = delete;
  void run(Stats* total = nullptr) {
    m_->check(trn_coarsen_run(m_->handle(), algo_->maxPart(), total));
    detail::report(m_, "= coarsening");
  }

 private:
  Mesh* m_;
  Partit* algo_;
};

class Swap {
 public:
  explicit Swap(Mesh* input) : m_(input) {}
  Swap(const Swap&) = delete;
  Swap& operator=(Swap) = delete;
  void run(Stats* total = nullptr) {
    m_->check(trn_swap_run(m_->handle(), total));
    detail::report(m_, "= swapping");
  }

 private:
  Mesh* m_;
};

class Smooth {
 public:
  Smooth(Mesh* input, Partit* algo, int level) : m_(input), algo_(algo), level_(level) {}
  Smooth(const Smooth&) = delete;
  Smooth& operator=(Smooth) = delete;
  void run(Stats* total = nullptr) {
    m_->check(trn_smooth_run(m_->handle(), algo_->maxPart(), level_, total));
    detail::report(m_, "= smoothing");
  }

 private:
  Mesh* m_;
  Partit* algo_;
  int level_;
};

namespace io {
/* io::find (io.cpp:25-49): count following the first line whose first token is key */
inline int find(const std::string key, std::ifstream& file) {
  std::string line, token;
  while (std::getline(file, line)) {
    size_t off = line.find_first_not_of(" \t\r\n");
    if (off == std::string::npos) continue;
    if (line[off] == '#' || line[off] == '%') continue;
    std::stringstream buffer(line.substr(off));
    if (buffer >> token && token == key) break;
  }
  int count = -1;
  file >> count;
  return count;
}
}  // namespace io

namespace tools {
inline bool exists(const std::string& path) {
  std::ifstream f(path);
  return f.good();
}
}  // namespace tools

/* The command line of trinity (parser.cpp:30-145): same flags, same clamps. */
class Parser {
 public:
  struct {
    int size[2] = {0, 0};
    int bucket = 64, rounds = 8, depth = 3, norm = 2, verb = 1, threads = 1, cores = 1, hw_cores = 1;
    double target = 1.0, h_min = EPSILON, h_max = 0.4;
    int makespan = 0;
    std::string input, result, solut, name, arch = "b200";
  } param;

  Parser(int argc, char* argv[]) {
    std::string in, out, sol;
    int bucket = 64, rounds = 8, depth = 3, norm = 2, verb = 1, cores = 1;
    double targ = 1.0;
    for (int i = 1; i < argc; ++i) {
      std::string a = argv[i];
      auto val = [&](void) -> std::string {
        if (a.size() > 2) return a.substr(2);
        if (i + 1 >= argc) usage(argv[0], ("missing value for " + a).c_str());
        return argv[++i];
      };
      if (a == "-h" || a == "--help") usage(argv[0], nullptr);
      else if (a.rfind("-i", 0) == 0) in = val();
      else if (a.rfind("-o", 0) == 0) out = val();
      else if (a.rfind("-s", 0) == 0) sol = val();
      else if (a.rfind("-c", 0) == 0) cores = std::atoi(val().c_str());
      else if (a.rfind("-b", 0) == 0) bucket = std::atoi(val().c_str());
      else if (a.rfind("-t", 0) == 0) targ = std::atof(val().c_str());
      else if (a.rfind("-p", 0) == 0) norm = std::atoi(val().c_str());
      else if (a.rfind("-r", 0) == 0) rounds = std::atoi(val().c_str());
      else if (a.rfind("-d", 0) == 0) depth = std::atoi(val().c_str());
      else if (a.rfind("-v", 0) == 0) verb = std::atoi(val().c_str());
      else if (a.rfind("-m", 0) == 0 || a.rfind("-a", 0) == 0 || a.rfind("-P", 0) == 0) (void) val();
      else usage(argv[0], ("unknown option " + a).c_str());
    }
    param.threads = std::max(cores, 1);
    param.bucket = std::max(std::min(bucket, 256), 64);   /* parser.cpp:86 */
    param.rounds = std::max(std::min(rounds, 5), 1);      /* parser.cpp:87 */
    param.depth = std::max(std::min(depth, 3), 1);        /* parser.cpp:88 */
    param.target = std::max(std::min(targ, 1.), 0.5);     /* parser.cpp:89 */
    param.norm = std::max(std::min(norm, 4), 0);          /* parser.cpp:90 */
    param.verb = std::max(std::min(verb, 2), 0);          /* parser.cpp:91 */
    param.input = in;
    param.result = out.empty() ? std::string("adapted.mesh") : out;
    param.solut = sol;
    param.name = sol.substr(sol.find_last_of('/') + 1);
    param.name = param.name.substr(0, param.name.find_last_of('.'));
    if (in.empty() || !tools::exists(in)) usage(argv[0], "option -i: invalid mesh file");
    std::ifstream f(in);
    param.size[0] = io::find("Vertices", f);
    param.size[1] = io::find("Triangles", f);
    if (param.size[0] <= 0 || param.size[1] <= 0) usage(argv[0], "option -i: invalid mesh file");
    if (sol.empty() || !tools::exists(sol)) usage(argv[0], "option -s: invalid solut. file");
    std::ifstream fs(sol);
    int col[4] = {0, 0, 0, 0};
    fs >> col[0] >> col[1] >> col[2] >> col[3];
    if (col[2] != param.size[0]) usage(argv[0], "option -s: wrong number of vertices in solut. file");
  }

  /* makespan table (parser.cpp:148-260, condensed) */
  void recap(Stats* stat) {
    if (!stat) return;
    const char* name[] = {"metric", "refine", "coarse", "swap", "smooth"};
    const char* unit[] = {"calc", "split", "merge", "flip", "move"};
    param.makespan = 0;
    for (int i = 0; i < 5; ++i) param.makespan += stat[i].elap;
    std::printf("\n= recap: %d rounds on the GPU (%.3f s)\n", param.rounds, param.makespan / 1e3);
    for (int i = 0; i < 5; ++i) {
      int ms = std::max(stat[i].elap, 1);
      std::printf("=  %-7s %8d ms  %12.0f %s/sec (%d done)\n", name[i], stat[i].elap,
                  stat[i].task / (ms * 1e-3), unit[i], stat[i].task);
    }
  }

  /* one TSV line per kernel, appended like parser.cpp:263-312 */
  void dump(Stats* stat) {
    if (!stat) return;
    const char* kern[] = {"refine", "coarse", "swap", "smooth"};
    std::string dir = param.result.substr(0, param.result.find_last_of('/') + 1);
    for (int i = 1; i < 5; ++i) {
      std::string path = dir + param.name + "_" + param.arch + "_" + kern[i - 1] + ".dat";
      FILE* f = std::fopen(path.c_str(), "a");
      if (!f) continue;
      std::fprintf(f, "%2d \t%d \t%d \t%d \t%3.2f \t%8d \t%8d \t%.3f \t%.3f\n", param.threads,
                   param.rounds, param.size[0], param.size[1], param.target, stat[i].task,
                   stat[i].eval, param.makespan / 1e3, stat[i].elap / 1e3);
      std::fclose(f);
    }
  }

 private:
  [[noreturn]] static void usage(const char* prog, const char* err) {
    if (err) std::printf("\nError: option %s\n", err);
    std::printf(
        "usage: %s -i mesh -s solut [-o result] [-b bucket 64-256] [-t target 0.5-1.0]\n"
        "       [-p norm 0-4] [-r rounds 1-5] [-d depth 1-3] [-v verbosity 0-2] [-c threads]\n",
        prog);
    std::exit(err ? EXIT_FAILURE : EXIT_SUCCESS);
  }
};

}  // namespace trinity
