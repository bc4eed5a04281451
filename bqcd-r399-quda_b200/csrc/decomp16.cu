// decomp16.cu -- the int16 stencil passes of one time slab (decomp.cuh), for
// the mixed-precision CG over a decomposed lattice (bqcdg_dd_solve): the
// sloppy iterations of the single-domain solver (k_pass1, k_pass2 with its
// |q|^2 block partials, k_cg_pass4 in dslash.cu) with the t hops across the
// slab boundaries read from ghost faces, and the kernels that pack those
// faces and sum the CG's block partials over the slabs.
//
// A ghost face holds the two-spin half spinor that the t hop keeps (d/D21.F90:
// 53, comm/xbound_mpi.F90:418-461) in FP32, decoded from the int16 field with
// its site norm: 48 bytes per face site.  The boundary link U_t(x - t) of the
// first slice comes from the FP64 ghost links that the FP64 passes use.
// Everything else is the arithmetic of the single-domain int16 passes: the
// links of a site are loaded before the first gather (wilson_hop_lf), the
// int16 scales are folded into one factor per hop, and the clover term and
// the output norm are those of k_pass1 / pass2_core.
#include "decomp.cuh"
#include "kernels.cuh"
#include "views.cuh"

namespace bqcdg {

// b += hscale * D_{e,o} in at local site i of the slab, int16 fields, the t
// neighbours across the slab boundaries from the FP32 ghost faces
template <bool DAG>
__device__ __forceinline__ void dd_hop16(const Geom& g, const DdGeom& d, int e, int i, const Site& st,
                                         const SpinorView<Prec::F16>& in, const GaugeView<Prec::F16>& U,
                                         Spinor<float>& b, float hscale) {
  const int o = 1 - e;
  const uint2* ub = reinterpret_cast<const uint2*>(U.v);
  const int S = U.stride;
  uint2 W[4][2][3];
  int J[4][2];
#pragma unroll
  for (int mu = 3; mu >= 0; mu--) {
    if (mu == 3) {
      J[3][0] = dd_tneighbour(g, d, i, st.x[3], true);
      J[3][1] = dd_tneighbour(g, d, i, st.x[3], false);
    } else {
      J[mu][0] = neighbour(g, st, i, mu, true);
      J[mu][1] = neighbour(g, st, i, mu, false);
    }
#pragma unroll
    for (int w = 0; w < 3; w++) {
      W[mu][0][w] = ld_once(ub + (size_t)((mu * 2 + e) * 3 + w) * S + i);
      // the backward t link of the first slice is a ghost link (below)
      W[mu][1][w] = J[mu][1] >= 0 ? ld_once(ub + (size_t)((mu * 2 + o) * 3 + w) * S + J[mu][1]) : make_uint2(0u, 0u);
    }
  }
#pragma unroll
  for (int mu = 3; mu >= 0; mu--) {
#pragma unroll
    for (int fb = 0; fb < 2; fb++) {
      const bool fwd = fb == 0;
      cx<float> h[2][3], f[2][3];
      float sc, lsc;
      Link<float> u;
      float sgn;
      if (mu == 3) {
        const int j = J[3][fb];
        if (j >= 0) {
          in.load_pair_raw(j, fwd ? dd_spin_fwd(DAG) : dd_spin_bwd(DAG), h, sc);
        } else {
          const float2* gh = reinterpret_cast<const float2*>(fwd ? d.ghost_fwd : d.ghost_bwd);
          const int jj = -1 - j;
#pragma unroll
          for (int c = 0; c < 3; c++)
#pragma unroll
            for (int s = 0; s < 2; s++) {
              const float2 t = gh[(size_t)(c * 2 + s) * d.V3h + jj];
              h[s][c] = mkc(t.x, t.y);
            }
          sc = 1.f;  // the face holds the decoded values
        }
        if (fwd || j >= 0) {
          links16_decode(W[3][fb][0], W[3][fb][1], W[3][fb][2], u, lsc);
        } else {
          const double2* gl = d.ghost_link + (size_t)o * 9 * d.V3h + (-1 - j);
#pragma unroll
          for (int c = 0; c < 3; c++)
#pragma unroll
            for (int r = 0; r < 3; r++) {
              const double2 t = gl[(size_t)(c * 3 + r) * d.V3h];
              u.m[r][c] = mkc((float)t.x, (float)t.y);
            }
          lsc = 1.f;
        }
        sgn = (float)dd_tsign(d, st.x[3], fwd);
      } else {
        float2 F[4][3];
        in.load_biased(J[mu][fb], F, sc);
        project_biased<DAG>(F, mu, fwd, h);
        links16_decode(W[mu][fb][0], W[mu][fb][1], W[mu][fb][2], u, lsc);
        sgn = (float)hop_sign(g, st, mu, fwd);
      }
      const float k = sgn * sc * lsc * hscale;
      if (fwd) {
        mul_u(u, h, f);
        recon_fwd<float, DAG>(b, mu, f, k);
      } else {
        mul_ud(u, h, f);
        recon_bwd<float, DAG>(b, mu, f, k);
      }
    }
  }
}

// t_o = [(1 -+ i h g5)] A_oo^-1 D_oe in_e on the sites of one part of the slab
template <bool DAG>
__global__ void __launch_bounds__(kBlock, 4) k_dd16_pass1(Geom g, DdGeom d, int part, SpinorPtr outp, SpinorPtr inp,
                                                          const void* gauge, CloverPtr ainv, int has_clover,
                                                          double hval, const CgScalars* cg) {
  if (cg && cg->done) return;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= dd_part_sites(part, g.L[3], d.V3h)) return;
  const int i = dd_part_site(part, g.L[3], d.V3h, j);
  const auto in = sview<Prec::F16>(inp, g.stride);
  const auto out = sview<Prec::F16>(outp, g.stride);
  const auto U = gview<Prec::F16>(gauge, g);
  const Site st = site_coords(g, i, 1);
  Spinor<float> b;
  zero(b);
  dd_hop16<DAG>(g, d, 1, i, st, in, U, b, 1.f);
  float osc = 1.f;
  if (has_clover) {
    Spinor<float> y;
    clover_apply_raw(cview<Prec::F16>(ainv, g.stride), i, b, y, osc);
    b = y;
  }
  if (hval != 0.0) h_mult_b(b, (float)hval);
  out.store_scaled(i, b, osc);
}

// out = A_ee x + b D_eo t (+ rho x; Wilson: x + b D_eo t + i h' g5 x), the
// site-local terms first as in pass2_core
template <bool DAG>
__device__ __forceinline__ void dd16_pass2_core(const Geom& g, const DdGeom& d, int i, const SpinorView<Prec::F16>& t,
                                                const SpinorView<Prec::F16>& xin, const GaugeView<Prec::F16>& U,
                                                CloverPtr aee, int has_clover, double bcoef, double hval, double rho,
                                                Spinor<float>& out) {
  Spinor<float> x;
  float xsc;
  xin.load_raw(i, x, xsc);
  const float rr = (float)rho * xsc;
  if (has_clover) {
    float csc = 1.f;
    clover_apply_raw(cview<Prec::F16>(aee, g.stride), i, x, out, csc);
    const float k = csc * xsc;
#pragma unroll
    for (int s = 0; s < 4; s++)
#pragma unroll
      for (int c = 0; c < 3; c++) out.c[s][c] = rho != 0.0 ? k * out.c[s][c] + rr * x.c[s][c] : k * out.c[s][c];
  } else {
    const float k = xsc + rr;
#pragma unroll
    for (int s = 0; s < 4; s++)
#pragma unroll
      for (int c = 0; c < 3; c++) out.c[s][c] = k * x.c[s][c];
    if (hval != 0.0) {
      const float hh = (float)hval * xsc;
#pragma unroll
      for (int c = 0; c < 3; c++) {
        out.c[0][c] = out.c[0][c] + hh * itimes(x.c[2][c]);
        out.c[1][c] = out.c[1][c] + hh * itimes(x.c[3][c]);
        out.c[2][c] = out.c[2][c] + hh * itimes(x.c[0][c]);
        out.c[3][c] = out.c[3][c] + hh * itimes(x.c[1][c]);
      }
    }
  }
  const Site st = site_coords(g, i, 0);
  dd_hop16<DAG>(g, d, 0, i, st, t, U, out, (float)bcoef);
}

// second half of mtil (q = M~ p): the output and, with REDUCE, the block
// partial of |q|^2 in part[slot0 + block]
template <bool DAG, bool REDUCE>
__global__ void __launch_bounds__(kBlock, 4) k_dd16_pass2(Geom g, DdGeom d, int part, SpinorPtr outp, SpinorPtr tp,
                                                          SpinorPtr xp, const void* gauge, CloverPtr aee,
                                                          int has_clover, double bcoef, double hval, double rho,
                                                          double* partial, int slot0, const CgScalars* cg) {
  if (cg && cg->done) return;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[1] = {0.0};
  if (j < dd_part_sites(part, g.L[3], d.V3h)) {
    const int i = dd_part_site(part, g.L[3], d.V3h, j);
    Spinor<float> o;
    dd16_pass2_core<DAG>(g, d, i, sview<Prec::F16>(tp, g.stride), sview<Prec::F16>(xp, g.stride),
                         gview<Prec::F16>(gauge, g), aee, has_clover, bcoef, hval, rho, o);
    sview<Prec::F16>(outp, g.stride).store(i, o);
    if (REDUCE) {
#pragma unroll
      for (int s = 0; s < 4; s++)
#pragma unroll
        for (int c = 0; c < 3; c++) acc[0] += (double)norm2(o.c[s][c]);
    }
  }
  if (REDUCE) block_reduce_store<1>(acc, partial, 0, slot0 + (int)blockIdx.x);
}

// the CG-fused second half of mtil_dag (k_cg_pass4 with x updated by the p
// update): A p in registers, r -= alpha A p (FP32), |r|^2 block partials
__global__ void __launch_bounds__(kBlock, 4) k_dd16_pass4(Geom g, DdGeom d, int part, SpinorPtr tp, SpinorPtr qp,
                                                          const void* gauge, CloverPtr aee, int has_clover,
                                                          double bcoef, double hval, double rho, SpinorPtr rp,
                                                          double* partial, int slot0, const CgScalars* cg) {
  if (cg->done) return;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[1] = {0.0};
  if (j < dd_part_sites(part, g.L[3], d.V3h)) {
    const int i = dd_part_site(part, g.L[3], d.V3h, j);
    Spinor<float> ap;
    dd16_pass2_core<true>(g, d, i, sview<Prec::F16>(tp, g.stride), sview<Prec::F16>(qp, g.stride),
                          gview<Prec::F16>(gauge, g), aee, has_clover, bcoef, hval, rho, ap);
    const auto rv = sview<Prec::F32>(rp, g.stride);
    const float a = (float)cg->alpha;
    Spinor<float> rl;
    rv.load(i, rl);
#pragma unroll
    for (int s = 0; s < 4; s++)
#pragma unroll
      for (int c = 0; c < 3; c++) {
        rl.c[s][c] = rl.c[s][c] - a * ap.c[s][c];
        acc[0] += (double)norm2(rl.c[s][c]);
      }
    rv.store(i, rl);
  }
  block_reduce_store<1>(acc, partial, 0, slot0 + (int)blockIdx.x);
}

// the two FP32 faces of an int16 field: spins s_f of the first slice for
// rank-1, spins s_b of the last slice for rank+1
__global__ void __launch_bounds__(kBlock) k_dd16_pack(Geom g, int V3h, int sf, int sb, SpinorPtr inp, float2* to_prev,
                                                      float2* to_next) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= V3h) return;
  const auto in = sview<Prec::F16>(inp, g.stride);
  cx<float> h[2][3];
  float sc;
  in.load_pair_raw(dd_face_site(g, V3h, 0, j), sf, h, sc);
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int s = 0; s < 2; s++) to_prev[(size_t)(c * 2 + s) * V3h + j] = make_float2(sc * h[s][c].x, sc * h[s][c].y);
  in.load_pair_raw(dd_face_site(g, V3h, 1, j), sb, h, sc);
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int s = 0; s < 2; s++) to_next[(size_t)(c * 2 + s) * V3h + j] = make_float2(sc * h[s][c].x, sc * h[s][c].y);
}

// the sum over the slabs, in slab order, of each slab's block partials (in
// block order, final_sum), then by mode: 0 the total into *tot (to be summed
// over the ranks), 1 alpha = rtr / total, 2 the CG scalar step; skipped when
// the solve has stopped (the passes did not run)
__device__ __forceinline__ void dd_apply_total(CgScalars* cg, double tot, double* out, int mode) {
  if (mode == 0) *out = tot;
  else if (mode == 1) {
    cg->paap = tot;
    cg->alpha = cg->rtr / tot;
  } else {
    cg_scalar_step(cg, tot);
  }
}
constexpr int kDdSumBlock = 1024;
__global__ void __launch_bounds__(kDdSumBlock) k_dd_total(DdPartials parts, int nslabs, int nsb, CgScalars* cg,
                                                          double* out, int mode) {
  if (cg->done) return;
  double tot = 0.0;
  for (int s = 0; s < nslabs; s++) {
    double t[1];
    final_sum<1>(parts.p[s], 0, nsb, t);
    tot += t[0];
  }
  if (threadIdx.x == 0) dd_apply_total(cg, tot, out, mode);
}
__global__ void k_dd_apply(const double* tot, CgScalars* cg, int mode) {
  if (!cg->done) dd_apply_total(cg, *tot, nullptr, mode);
}

void launch_dd16_pack(const Geom& g, const DdGeom& d, bool dag, SpinorPtr in, float2* to_prev, float2* to_next,
                      cudaStream_t s) {
  k_dd16_pack<<<nblocks(d.V3h), kBlock, 0, s>>>(g, d.V3h, dd_spin_fwd(dag), dd_spin_bwd(dag), in, to_prev, to_next);
}
void launch_dd16_pass1(const Geom& g, const DdGeom& d, bool dag, int part, SpinorPtr out, SpinorPtr in,
                       const void* gauge, CloverPtr ainv, const OpParams& op, const CgScalars* cg, cudaStream_t s) {
  const int n = dd_part_sites(part, g.L[3], d.V3h);
  if (n <= 0) return;
  const int hc = op.csw_kappa != 0.0;
  const double hv = dag ? op.h : -op.h;
  if (dag) k_dd16_pass1<true><<<nblocks(n), kBlock, 0, s>>>(g, d, part, out, in, gauge, ainv, hc, hv, cg);
  else k_dd16_pass1<false><<<nblocks(n), kBlock, 0, s>>>(g, d, part, out, in, gauge, ainv, hc, hv, cg);
}
int launch_dd16_pass2(const Geom& g, const DdGeom& d, bool dag, int part, SpinorPtr out, SpinorPtr t, SpinorPtr x,
                      const void* gauge, CloverPtr aee, const OpParams& op, double* partial, int slot0,
                      const CgScalars* cg, cudaStream_t s) {
  const int n = dd_part_sites(part, g.L[3], d.V3h);
  if (n <= 0) return 0;
  const int hc = op.csw_kappa != 0.0;
  const double bcoef = -op.kappa * op.kappa / (1.0 + op.h * op.h);
  const double hv = dag ? -op.h : op.h;
  const dim3 grid(nblocks(n));
  if (partial) {
    if (dag) k_dd16_pass2<true, true><<<grid, kBlock, 0, s>>>(g, d, part, out, t, x, gauge, aee, hc, bcoef, hv,
                                                              op.rho, partial, slot0, cg);
    else k_dd16_pass2<false, true><<<grid, kBlock, 0, s>>>(g, d, part, out, t, x, gauge, aee, hc, bcoef, hv, op.rho,
                                                           partial, slot0, cg);
  } else {
    if (dag) k_dd16_pass2<true, false><<<grid, kBlock, 0, s>>>(g, d, part, out, t, x, gauge, aee, hc, bcoef, hv,
                                                               op.rho, nullptr, 0, cg);
    else k_dd16_pass2<false, false><<<grid, kBlock, 0, s>>>(g, d, part, out, t, x, gauge, aee, hc, bcoef, hv, op.rho,
                                                            nullptr, 0, cg);
  }
  return (int)grid.x;
}
int launch_dd16_pass4(const Geom& g, const DdGeom& d, int part, SpinorPtr t, SpinorPtr q, const void* gauge,
                      CloverPtr aee, const OpParams& op, SpinorPtr r, double* partial, int slot0, const CgScalars* cg,
                      cudaStream_t s) {
  const int n = dd_part_sites(part, g.L[3], d.V3h);
  if (n <= 0) return 0;
  const int hc = op.csw_kappa != 0.0;
  const double bcoef = -op.kappa * op.kappa / (1.0 + op.h * op.h);
  const double hv = -op.h;  // mtil_dag
  const dim3 grid(nblocks(n));
  k_dd16_pass4<<<grid, kBlock, 0, s>>>(g, d, part, t, q, gauge, aee, hc, bcoef, hv, op.rho, r, partial, slot0, cg);
  return (int)grid.x;
}
void launch_dd_total(const DdPartials& parts, int nslabs, int nsb, CgScalars* cg, double* out, int mode,
                     cudaStream_t s) {
  k_dd_total<<<1, kDdSumBlock, 0, s>>>(parts, nslabs, nsb, cg, out, mode);
}
void launch_dd_apply(const double* tot, CgScalars* cg, int mode, cudaStream_t s) {
  k_dd_apply<<<1, 1, 0, s>>>(tot, cg, mode);
}

}  // namespace bqcdg
