// Host-side check program for the time-slab decomposition (decomp.cuh): for
// one rank of a decomposed lattice it evaluates the index maps that the slab
// kernels use -- which sites and spinor components the face packing sends to
// rank-1 and rank+1, and, for every even output site and hop, where the
// kernel reads its neighbour (a local index, or an entry of a ghost face) and
// the boundary sign it applies -- and writes them for the gloo test, which
// runs the decomposed hopping term on the host with these maps.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../../bqcd-r399-quda_b200/csrc/decomp.cuh"

int main(int argc, char** argv) {
  if (argc != 10) {
    std::fprintf(stderr, "usage: %s Lx Ly Lz Lt bc_t nranks rank dag out.bin\n", argv[0]);
    return 2;
  }
  int L[4];
  for (int d = 0; d < 4; d++) L[d] = std::atoi(argv[1 + d]);
  const int bct = std::atoi(argv[5]), nranks = std::atoi(argv[6]), rank = std::atoi(argv[7]);
  const bool dag = std::atoi(argv[8]) != 0;
  bqcdg::Geom g{};  // the slab: L[3] / nranks time slices
  for (int d = 0; d < 4; d++) {
    g.L[d] = L[d];
    g.bcsign[d] = 1;
  }
  g.L[3] = L[3] / nranks;
  g.Lxh = L[0] / 2;
  g.volh = L[0] * L[1] * L[2] / 2 * g.L[3];
  g.stride = g.volh;
  bqcdg::geom_finish(g);
  bqcdg::DdGeom d{};
  d.nranks = nranks;
  d.rank = rank;
  d.Lt_glob = L[3];
  d.t0 = rank * g.L[3];
  d.V3h = L[0] * L[1] * L[2] / 2;
  d.bct = bct;
  // faces: site[side][j], comp[side][k] (side 0: to rank-1, 1: to rank+1)
  std::vector<int> site(2 * (size_t)d.V3h), comp(12);
  for (int side = 0; side < 2; side++) {
    const int s0 = side == 0 ? bqcdg::dd_spin_fwd(dag) : bqcdg::dd_spin_bwd(dag);
    for (int k = 0; k < 6; k++) comp[side * 6 + k] = bqcdg::dd_face_comp(k, s0);
    for (int j = 0; j < d.V3h; j++) site[(size_t)side * d.V3h + j] = bqcdg::dd_face_site(g, d.V3h, side, j);
  }
  // hops of the even output sites: nb[mu][fb][i], sign[mu][fb][i]
  std::vector<int> nb(8 * (size_t)g.volh), sg(nb.size());
  for (int mu = 0; mu < 4; mu++)
    for (int fb = 0; fb < 2; fb++)
      for (int i = 0; i < g.volh; i++) {
        const bqcdg::Site st = bqcdg::site_coords(g, i, 0);
        const size_t k = ((size_t)mu * 2 + fb) * g.volh + i;
        if (mu == 3) {
          nb[k] = bqcdg::dd_tneighbour(g, d, i, st.x[3], fb == 0);
          sg[k] = bqcdg::dd_tsign(d, st.x[3], fb == 0);
        } else {
          nb[k] = bqcdg::neighbour(g, st, i, mu, fb == 0);
          sg[k] = bqcdg::hop_sign(g, st, mu, fb == 0);
        }
      }
  FILE* f = std::fopen(argv[9], "wb");
  if (!f) return 1;
  std::fwrite(site.data(), sizeof(int), site.size(), f);
  std::fwrite(comp.data(), sizeof(int), comp.size(), f);
  std::fwrite(nb.data(), sizeof(int), nb.size(), f);
  std::fwrite(sg.data(), sizeof(int), sg.size(), f);
  std::fclose(f);
  return 0;
}
