/*
 * trinity_main.cpp — the `trinity` command line on the GPU: same flags and
 * call sequence as trinity's CLI (src/main.cpp:23-62, flags parser.cpp:37-96):
 *
 *   trinity -i in.mesh -s field.bb [-o out.mesh] [-b bucket] [-t target]
 *           [-p norm] [-r rounds] [-d depth] [-v verbosity]
 *
 * metric recovery once, then `rounds` x (refine, coarsen, swap, smooth),
 * makespan table, per-kernel TSV dump, adapted mesh (and its metric as .sol).
 */
#include "trinity.h"

int main(int argc, char* argv[]) {
  try {
    trinity::Parser parser(argc, argv);
    auto& p = parser.param;
    trinity::Mesh mesh(p.size, p.bucket, p.depth, p.verb, p.rounds);
    trinity::Metrics metric(&mesh, p.target, p.norm, p.h_min, p.h_max);
    trinity::Partit heuris(&mesh, 8);
    trinity::Refine refine(&mesh, p.depth);
    trinity::Swap swap(&mesh);
    trinity::Coarse coarse(&mesh, &heuris);
    trinity::Smooth smooth(&mesh, &heuris, p.depth);
    trinity::Stats stat[5];

    mesh.load(p.input, p.solut);
    metric.run(stat);
    for (int iter = 0; iter < p.rounds; ++iter) {
      refine.run(stat + 1);
      coarse.run(stat + 2);
      swap.run(stat + 3);
      smooth.run(stat + 4);
    }
    parser.recap(stat);
    parser.dump(stat);
    mesh.store(p.result);
    std::string sol = p.result.substr(0, p.result.find_last_of('.')) + ".sol";
    mesh.storeMetric(sol);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
