// decomp.cu -- stencil kernels of one time slab of a decomposed lattice
// (decomp.cuh): the FP64 hopping term with ghost faces for the t hops across
// slab boundaries, the two halves of mtil / mtil_dag built on it, and the
// kernels that pack the faces and the boundary links for the exchange.
//
// Away from the slab boundaries the arithmetic is that of the single-domain
// kernels (wilson_hop, k_pass1, pass2_core in dslash.cu), hop by hop in the
// same order, so a decomposed operator equals the single-domain one bit for
// bit.
#include "decomp.cuh"
#include "kernels.cuh"
#include "views.cuh"

namespace bqcdg {

// b += hscale * D_{e,o} in at local site i, reading the t neighbours across the
// slab boundaries from the ghost faces (d/D21.F90:29-77; the t hop keeps two
// spins, d/D21xyzt.F90:32-44)
template <bool DAG>
__device__ __forceinline__ void dd_hop(const Geom& g, const DdGeom& d, int e, int i, const Site& st,
                                       const SpinorView<Prec::F64>& in, const GaugeView<Prec::F64>& U,
                                       Spinor<double>& b, double hscale) {
  const int o = 1 - e;
#pragma unroll
  for (int mu = 3; mu >= 0; mu--) {
#pragma unroll
    for (int fb = 0; fb < 2; fb++) {
      const bool fwd = fb == 0;
      cx<double> h[2][3], f[2][3];
      Link<double> u;
      double k;
      if (mu == 3) {
        const int s0 = fwd ? dd_spin_fwd(DAG) : dd_spin_bwd(DAG);
        const int j = dd_tneighbour(g, d, i, st.x[3], fwd);
        if (j >= 0) {
          in.load_pair(j, s0, h);
          if (fwd) U.load(3, e, i, u);
          else U.load(3, o, j, u);
        } else {
          const int jj = -1 - j;
          const double2* gh = fwd ? d.ghost_fwd : d.ghost_bwd;
#pragma unroll
          for (int c = 0; c < 3; c++)
#pragma unroll
            for (int s = 0; s < 2; s++) {
              const double2 t = gh[(size_t)(c * 2 + s) * d.V3h + jj];
              h[s][c] = mkc(t.x, t.y);
            }
          if (fwd) {
            U.load(3, e, i, u);
          } else {
            const double2* gl = d.ghost_link + (size_t)o * 9 * d.V3h + jj;
#pragma unroll
            for (int c = 0; c < 3; c++)
#pragma unroll
              for (int r = 0; r < 3; r++) {
                const double2 t = gl[(size_t)(c * 3 + r) * d.V3h];
                u.m[r][c] = mkc(t.x, t.y);
              }
          }
        }
        k = (double)dd_tsign(d, st.x[3], fwd) * hscale;
      } else {
        const int j = neighbour(g, st, i, mu, fwd);
        Spinor<double> p;
        in.load(j, p);
        project<double, DAG>(p, mu, fwd, h);
        if (fwd) U.load(mu, e, i, u);
        else U.load(mu, o, j, u);
        k = (double)hop_sign(g, st, mu, fwd) * hscale;
      }
      if (fwd) {
        mul_u(u, h, f);
        recon_fwd<double, DAG>(b, mu, f, k);
      } else {
        mul_ud(u, h, f);
        recon_bwd<double, DAG>(b, mu, f, k);
      }
    }
  }
}

template <bool DAG>
__global__ void __launch_bounds__(kBlock) k_dd_dslash(Geom g, DdGeom d, int e, double2* out, const double2* in,
                                                      const double2* gauge) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.volh) return;
  SpinorView<Prec::F64> IN{(double2*)in, g.stride}, OUT{out, g.stride};
  GaugeView<Prec::F64> U{(double2*)gauge, g.stride, 0};
  const Site st = site_coords(g, i, e);
  Spinor<double> b;
  zero(b);
  dd_hop<DAG>(g, d, e, i, st, IN, U, b, 1.0);
  OUT.store(i, b);
}

// t_o = [(1 -+ i h g5)] A_oo^-1 D_oe in_e (m_tilde.F90:55-58, 92-95)
template <bool DAG>
__global__ void __launch_bounds__(kBlock) k_dd_pass1(Geom g, DdGeom d, int part, double2* out, const double2* in,
                                                     const double2* gauge, const double2* ainv, double hval) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= dd_part_sites(part, g.L[3], d.V3h)) return;
  const int i = dd_part_site(part, g.L[3], d.V3h, j);
  SpinorView<Prec::F64> IN{(double2*)in, g.stride}, OUT{out, g.stride};
  GaugeView<Prec::F64> U{(double2*)gauge, g.stride, 0};
  const Site st = site_coords(g, i, 1);
  Spinor<double> b;
  zero(b);
  dd_hop<DAG>(g, d, 1, i, st, IN, U, b, 1.0);
  if (ainv) {
    Spinor<double> y;
    clover_apply(CloverView<Prec::F64>{(double2*)ainv, g.stride}, i, b, y);
    b = y;
  }
  if (hval != 0.0) h_mult_b(b, hval);
  OUT.store(i, b);
}

// out_e = A_ee x + b D_eo t_o (clover) or x + b D_eo t_o + i h' g5 x (Wilson),
// + rho x (m_tilde.F90:63-73, w_mult.F90:39): the site-local terms first,
// as in pass2_core
template <bool DAG>
__global__ void __launch_bounds__(kBlock) k_dd_pass2(Geom g, DdGeom d, int part, double2* out, const double2* tin,
                                                     const double2* xin, const double2* gauge, const double2* aee,
                                                     double bcoef, double hval, double rho) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= dd_part_sites(part, g.L[3], d.V3h)) return;
  const int i = dd_part_site(part, g.L[3], d.V3h, j);
  SpinorView<Prec::F64> T{(double2*)tin, g.stride}, X{(double2*)xin, g.stride}, OUT{out, g.stride};
  GaugeView<Prec::F64> U{(double2*)gauge, g.stride, 0};
  Spinor<double> x, o;
  double xsc;
  X.load_raw(i, x, xsc);
  const double rr = rho * xsc;
  if (aee) {
    double csc;
    clover_apply_raw(CloverView<Prec::F64>{(double2*)aee, g.stride}, i, x, o, csc);
    const double k = csc * xsc;
#pragma unroll
    for (int s = 0; s < 4; s++)
#pragma unroll
      for (int c = 0; c < 3; c++) o.c[s][c] = rho != 0.0 ? k * o.c[s][c] + rr * x.c[s][c] : k * o.c[s][c];
  } else {
    const double k = xsc + rr;
#pragma unroll
    for (int s = 0; s < 4; s++)
#pragma unroll
      for (int c = 0; c < 3; c++) o.c[s][c] = k * x.c[s][c];
    if (hval != 0.0) {
      const double hh = hval * xsc;
#pragma unroll
      for (int c = 0; c < 3; c++) {
        o.c[0][c] = o.c[0][c] + hh * itimes(x.c[2][c]);
        o.c[1][c] = o.c[1][c] + hh * itimes(x.c[3][c]);
        o.c[2][c] = o.c[2][c] + hh * itimes(x.c[0][c]);
        o.c[3][c] = o.c[3][c] + hh * itimes(x.c[1][c]);
      }
    }
  }
  const Site st = site_coords(g, i, 0);
  dd_hop<DAG>(g, d, 0, i, st, T, U, o, bcoef);
  OUT.store(i, o);
}

// the two faces a pass over `in` needs from this slab: spins s_f of the first
// slice for rank-1, spins s_b of the last slice for rank+1
__global__ void __launch_bounds__(kBlock) k_dd_pack(Geom g, int V3h, int sf, int sb, const double2* in,
                                                    double2* to_prev, double2* to_next) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= V3h) return;
  const int i0 = dd_face_site(g, V3h, 0, j), i1 = dd_face_site(g, V3h, 1, j);
#pragma unroll
  for (int k = 0; k < 6; k++) {
    to_prev[(size_t)k * V3h + j] = in[(size_t)dd_face_comp(k, sf) * g.stride + i0];
    to_next[(size_t)k * V3h + j] = in[(size_t)dd_face_comp(k, sb) * g.stride + i1];
  }
}

// U_t of the last slice, both parities, 9 complex each, for rank+1
__global__ void __launch_bounds__(kBlock) k_dd_pack_links(Geom g, int V3h, const double2* gauge, double2* to_next) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= V3h) return;
  const int i1 = dd_face_site(g, V3h, 1, j);
#pragma unroll
  for (int eo = 0; eo < 2; eo++)
#pragma unroll
    for (int k = 0; k < 9; k++)
      to_next[(size_t)(eo * 9 + k) * V3h + j] = gauge[(size_t)((3 * 2 + eo) * 9 + k) * g.stride + i1];
}

void launch_dd_pack(const Geom& g, const DdGeom& d, bool dag, const double2* in, double2* to_prev, double2* to_next,
                    cudaStream_t s) {
  k_dd_pack<<<nblocks(d.V3h), kBlock, 0, s>>>(g, d.V3h, dd_spin_fwd(dag), dd_spin_bwd(dag), in, to_prev, to_next);
}
void launch_dd_pack_links(const Geom& g, const DdGeom& d, const double2* gauge, double2* to_next, cudaStream_t s) {
  k_dd_pack_links<<<nblocks(d.V3h), kBlock, 0, s>>>(g, d.V3h, gauge, to_next);
}
void launch_dd_dslash(const Geom& g, const DdGeom& d, int e, bool dag, double2* out, const double2* in,
                      const double2* gauge, cudaStream_t s) {
  if (dag) k_dd_dslash<true><<<nblocks(g.volh), kBlock, 0, s>>>(g, d, e, out, in, gauge);
  else k_dd_dslash<false><<<nblocks(g.volh), kBlock, 0, s>>>(g, d, e, out, in, gauge);
}
void launch_dd_pass1(const Geom& g, const DdGeom& d, bool dag, double2* out, const double2* in, const double2* gauge,
                     const double2* ainv, const OpParams& op, cudaStream_t s, int part) {
  const int n = dd_part_sites(part, g.L[3], d.V3h);
  if (n <= 0) return;  // no interior in a slab of two slices
  const double hv = dag ? op.h : -op.h;
  const double2* ai = op.csw_kappa != 0.0 ? ainv : nullptr;
  if (dag) k_dd_pass1<true><<<nblocks(n), kBlock, 0, s>>>(g, d, part, out, in, gauge, ai, hv);
  else k_dd_pass1<false><<<nblocks(n), kBlock, 0, s>>>(g, d, part, out, in, gauge, ai, hv);
}
void launch_dd_pass2(const Geom& g, const DdGeom& d, bool dag, double2* out, const double2* t, const double2* in,
                     const double2* gauge, const double2* aee, const OpParams& op, cudaStream_t s, int part) {
  const int n = dd_part_sites(part, g.L[3], d.V3h);
  if (n <= 0) return;
  const double bcoef = -op.kappa * op.kappa / (1.0 + op.h * op.h);
  const double hv = dag ? -op.h : op.h;
  const double2* a = op.csw_kappa != 0.0 ? aee : nullptr;
  if (dag) k_dd_pass2<true><<<nblocks(n), kBlock, 0, s>>>(g, d, part, out, t, in, gauge, a, bcoef, hv, op.rho);
  else k_dd_pass2<false><<<nblocks(n), kBlock, 0, s>>>(g, d, part, out, t, in, gauge, a, bcoef, hv, op.rho);
}

}  // namespace bqcdg
