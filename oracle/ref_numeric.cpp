/*
 * ref_numeric.cpp — test infrastructure, not product code.
 *
 * Calls the reference's own numeric functions (src/numeric.cpp, linked from
 * trinity's unmodified sources by oracle/Makefile "ref") on seeded
 * pseudo-random symmetric positive definite tensors and points, and prints
 * inputs and outputs as hexadecimal doubles (one JSON object per line), to be
 * frozen as golden vectors under tests/golden/.
 */
#include "trinity.h"

#include <cstdint>
#include <cstdio>

using namespace trinity;

static uint64_t state = 0x9e3779b97f4a7c15ULL;
static double unif() {  /* splitmix64 -> [0, 1) */
  uint64_t z = (state += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  z ^= z >> 31;
  return (double) (z >> 11) * (1.0 / 9007199254740992.0);
}

static void spd(double t[3]) {
  double l1 = 6.25 + unif() * 1e4, l2 = 6.25 + unif() * 1e4, th = unif() * 3.141592653589793;
  double c = std::cos(th), s = std::sin(th);
  if (unif() < 0.2) s = 0.0, c = 1.0;  /* exercise the diagonal shortcut */
  t[0] = c * c * l1 + s * s * l2;
  t[1] = c * s * (l1 - l2);
  t[2] = s * s * l1 + c * c * l2;
}

static void hx(const char* key, const double* v, int n, bool last = false) {
  std::printf("\"%s\": [", key);
  for (int i = 0; i < n; ++i) std::printf("%s\"%a\"", i ? ", " : "", v[i]);
  std::printf("]%s", last ? "" : ", ");
}

int main(int argc, char** argv) {
  int count = argc > 1 ? std::atoi(argv[1]) : 64;
  for (int k = 0; k < count; ++k) {
    double ta[3], tb[3], tc[3], pa[2], pb[2], pc[2];
    spd(ta); spd(tb); spd(tc);
    pa[0] = unif(); pa[1] = unif();
    pb[0] = pa[0] + 0.01 + 0.05 * unif(); pb[1] = pa[1] + 0.05 * (unif() - 0.5);
    pc[0] = pa[0] + 0.05 * (unif() - 0.5); pc[1] = pa[1] + 0.01 + 0.05 * unif();
    double mat[4] = {ta[0], ta[1], ta[1], ta[2]}, val[2], v1[2], v2[2];
    numeric::eigenDecompose(mat, val, v1, v2);
    double three[9] = {ta[0], ta[1], ta[2], tb[0], tb[1], tb[2], tc[0], tc[1], tc[2]}, mean[3];
    numeric::interpolateTensor(three, mean, 3);
    double q = numeric::computeQuality(pa, pb, pc, ta, tb, tc);
    double len = numeric::approxRiemannDist(pa, pb, ta, tb);
    double sp[2], st[3];
    numeric::computeSteinerPoint(pa, pb, ta, tb, sp, st);
    std::printf("{");
    hx("ta", ta, 3); hx("tb", tb, 3); hx("tc", tc, 3);
    hx("pa", pa, 2); hx("pb", pb, 2); hx("pc", pc, 2);
    hx("eig_val", val, 2); hx("eig_v1", v1, 2); hx("eig_v2", v2, 2);
    hx("mean", mean, 3); hx("quality", &q, 1); hx("length", &len, 1);
    hx("steiner_p", sp, 2); hx("steiner_t", st, 3, true);
    std::printf("}\n");
  }
  return 0;
}
