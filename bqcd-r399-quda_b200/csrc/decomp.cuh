// decomp.cuh -- the time-slab domain decomposition of the even/odd operator:
// index maps shared by the device kernels (decomp.cu) and the host programs
// that check them.
//
// The global lattice L[0..3] is cut along t into nranks slabs of
// Lt_loc = L[3] / nranks slices (Lt_loc even, so a slab's local parity is the
// global one).  In BQCD's even/odd index i = ilex/2 (index.F90:58-76) the
// sites of one time slice of one parity are the contiguous range
// [t V3h, (t+1) V3h), V3h = L[0] L[1] L[2] / 2, so a slab is the contiguous
// range [t0 V3h, (t0 + Lt_loc) V3h) of the global index and its local index
// is the global one minus t0 V3h.
//
// A stencil pass needs, besides the slab's own sites, the t-neighbours of its
// first and last slice.  The t hop only uses the half spinor that the
// projection (1 -+ gamma_4) keeps (gamma_4 = diag(1,1,-1,-1) in BQCD's basis,
// d/D21xyzt.F90:32-44): two spins, 6 complex numbers per site, the 12 reals
// that BQCD's xbound exchanges (comm/xbound_mpi.F90:418-461).  Before a pass
// each slab therefore sends
//   to rank-1: spins (s_f, s_f+1) of its first slice, s_f = 2 for d, 0 for d_dag
//              (rank-1's forward t hop from its last slice);
//   to rank+1: spins (s_b, s_b+1) of its last slice,  s_b = 0 for d, 2 for d_dag
//              (rank+1's backward t hop from its first slice);
// each a face of [6][V3h] complex numbers, component c*2 + s' for colour c and
// spin s_f/s_b + s'.  They arrive in the receiver's ghost buffers ghost_fwd
// and ghost_bwd.  The backward hop from the first slice also needs
// U_t(x - t) of rank-1's last slice: those links ([2 parities][9][V3h]) are
// exchanged once per gauge field.
//
// The fermion boundary sign of flip_bc.F90:97-121 goes with the global time
// coordinate t0 + t: the link of a forward hop from global t = L[3]-1 and of a
// backward hop from global t = 0 carries bc_t.
#pragma once

#include "bqcdg_internal.cuh"

namespace bqcdg {

struct DdGeom {
  int nranks, rank;
  int Lt_glob;   // global L[3]
  int t0;        // global t of the slab's first slice
  int V3h;       // sites of one parity in one time slice
  int bct;       // fermion boundary sign in t (+1 / -1)
  const double2* ghost_fwd;   // [6][V3h]: the t-forward neighbours of the last slice
  const double2* ghost_bwd;   // [6][V3h]: the t-backward neighbours of the first slice
  const double2* ghost_link;  // [2][9][V3h]: U_t of rank-1's last slice, by parity
};

// spins of the half spinor that the forward / backward t hop reads
__host__ __device__ __forceinline__ int dd_spin_fwd(bool dag) { return dag ? 0 : 2; }
__host__ __device__ __forceinline__ int dd_spin_bwd(bool dag) { return dag ? 2 : 0; }

// face component k (0..5) of a send buffer: colour k / 2, spin s0 + k % 2;
// its component in the spinor layout [colour*4 + spin][stride]
__host__ __device__ __forceinline__ int dd_face_comp(int k, int s0) { return (k >> 1) * 4 + s0 + (k & 1); }

// the local site of face entry j (0 <= j < V3h): first (side 0) or last
// (side 1) slice of the slab
__host__ __device__ __forceinline__ int dd_face_site(const Geom& g, int V3h, int side, int j) {
  return side ? (g.L[3] - 1) * V3h + j : j;
}

// sign of the link used by the t hop of a site at local slice t
__host__ __device__ __forceinline__ int dd_tsign(const DdGeom& d, int t, bool fwd) {
  const int tg = d.t0 + t;
  return (fwd ? tg == d.Lt_glob - 1 : tg == 0) ? d.bct : 1;
}

// where the t hop of local site i (slice t) reads its half spinor: a local
// index (>= 0), or -1 - j for entry j of the ghost face
__host__ __device__ __forceinline__ int dd_tneighbour(const Geom& g, const DdGeom& d, int i, int t, bool fwd) {
  if (fwd) return t == g.L[3] - 1 ? -1 - (i - t * d.V3h) : i + d.V3h;
  return t == 0 ? -1 - i : i - d.V3h;
}

// the block partials of one reduction on each slab of this process, summed
// in slab order by the mixed-precision solver's reduction kernel
constexpr int kMaxDdSlabs = 16;
struct DdPartials {
  const double* p[kMaxDdSlabs];
};

// Overlap of the exchange with the slab's interior: a pass runs as two
// launches, the interior slices 1 .. Lt_loc-2 (no ghost read) while the faces
// travel, then the boundary slices 0 and Lt_loc-1.  dd_part_sites: sites of
// part (0 all, 1 interior, 2 boundary); dd_part_site: the local site of
// thread j (0 <= j < dd_part_sites) of that part.
__host__ __device__ __forceinline__ int dd_part_sites(int part, int Lt_loc, int V3h) {
  return part == 0 ? Lt_loc * V3h : (part == 1 ? (Lt_loc - 2) * V3h : 2 * V3h);
}
__host__ __device__ __forceinline__ int dd_part_site(int part, int Lt_loc, int V3h, int j) {
  if (part == 1) return V3h + j;
  if (part == 2) return j < V3h ? j : (Lt_loc - 1) * V3h + (j - V3h);
  return j;
}

}  // namespace bqcdg
