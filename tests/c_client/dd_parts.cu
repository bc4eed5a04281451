// Checks on the host that the interior (part 1) and boundary (part 2) launches
// of a slab pass cover every site of the slab exactly once, and that the
// interior reads no ghost: dd_part_sites / dd_part_site and dd_tneighbour of
// csrc/decomp.cuh, for the slab shapes given on the command line as pairs
// "Lx,Ly,Lz,Lt_loc".  Prints "ok" or the first failure; exit status 0 / 1.
#include <cstdio>
#include <vector>

#include "../../bqcd-r399-quda_b200/csrc/decomp.cuh"

using namespace bqcdg;

static int check(const int L[4]) {
  Geom g{};
  for (int d = 0; d < 4; d++) g.L[d] = L[d];
  const int V3h = L[0] * L[1] * L[2] / 2, Lt = L[3], volh = V3h * Lt;
  DdGeom d{};
  d.V3h = V3h;
  if (dd_part_sites(0, Lt, V3h) != volh) return printf("part 0 has %d sites, not %d\n", dd_part_sites(0, Lt, V3h), volh), 1;
  if (dd_part_sites(1, Lt, V3h) + dd_part_sites(2, Lt, V3h) != volh) return printf("parts 1 + 2 != volh\n"), 1;
  std::vector<int> seen(volh, 0);
  for (int part = 1; part <= 2; part++)
    for (int j = 0; j < dd_part_sites(part, Lt, V3h); j++) {
      const int i = dd_part_site(part, Lt, V3h, j);
      if (i < 0 || i >= volh) return printf("part %d thread %d -> site %d outside the slab\n", part, j, i), 1;
      seen[i]++;
      const int t = i / V3h;
      const bool ghost = dd_tneighbour(g, d, i, t, true) < 0 || dd_tneighbour(g, d, i, t, false) < 0;
      if (part == 1 && ghost) return printf("interior site %d (t %d) reads a ghost\n", i, t), 1;
      if (part == 2 && !ghost) return printf("boundary site %d (t %d) reads no ghost\n", i, t), 1;
    }
  for (int i = 0; i < volh; i++)
    if (seen[i] != 1) return printf("site %d covered %d times\n", i, seen[i]), 1;
  return 0;
}

int main(int argc, char** argv) {
  for (int a = 1; a < argc; a++) {
    int L[4];
    if (sscanf(argv[a], "%d,%d,%d,%d", &L[0], &L[1], &L[2], &L[3]) != 4) return printf("bad shape %s\n", argv[a]), 1;
    if (check(L)) return 1;
  }
  printf("ok\n");
  return 0;
}
