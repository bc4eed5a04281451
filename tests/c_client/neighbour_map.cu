// Host-side check program for the stencil kernels' index arithmetic: for a
// lattice given on the command line, it evaluates the same site_coords(),
// neighbour() and hop_sign() that the kernels run (bqcdg_internal.cuh, here
// compiled for the host) for every site, both parities, all four directions
// and both hop directions, and writes the table in the layout of BQCD's
// nn(volh, 0:1, 4, 0:1) (init_common.F90:164) followed by the hop signs.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../../bqcd-r399-quda_b200/csrc/bqcdg_internal.cuh"

int main(int argc, char** argv) {
  if (argc != 7) {
    std::fprintf(stderr, "usage: %s Lx Ly Lz Lt bc_t out.bin\n", argv[0]);
    return 2;
  }
  bqcdg::Geom g{};
  long vol = 1;
  for (int d = 0; d < 4; d++) {
    g.L[d] = std::atoi(argv[1 + d]);
    g.bcsign[d] = 1;
    vol *= g.L[d];
  }
  g.bcsign[3] = std::atoi(argv[5]);
  g.Lxh = g.L[0] / 2;
  g.volh = (int)(vol / 2);
  g.stride = g.volh;
  bqcdg::geom_finish(g);
  // nn[fb][mu][eo][i] (fb 0 forward, 1 backward), then sign[fb][mu][eo][i]
  std::vector<int> nn(2 * 4 * 2 * (size_t)g.volh), sg(nn.size());
  for (int fb = 0; fb < 2; fb++)
    for (int mu = 0; mu < 4; mu++)
      for (int eo = 0; eo < 2; eo++)
        for (int i = 0; i < g.volh; i++) {
          const bqcdg::Site s = bqcdg::site_coords(g, i, eo);
          const size_t k = (((size_t)fb * 4 + mu) * 2 + eo) * g.volh + i;
          nn[k] = bqcdg::neighbour(g, s, i, mu, fb == 0);
          sg[k] = bqcdg::hop_sign(g, s, mu, fb == 0);
        }
  FILE* f = std::fopen(argv[6], "wb");
  if (!f) return 1;
  std::fwrite(nn.data(), sizeof(int), nn.size(), f);
  std::fwrite(sg.data(), sizeof(int), sg.size(), f);
  std::fclose(f);
  return 0;
}
