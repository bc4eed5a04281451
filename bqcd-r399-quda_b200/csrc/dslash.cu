// dslash.cu -- even/odd clover-Wilson stencil kernels for sm_100a.
//
// One thread per output site; every field is component-major so each load of
// one component by a warp is one contiguous transaction.  The kernels are
// HBM-bound (about 0.9 flop/byte in FP64), so the design goal is to touch each
// byte once: links and clover blocks are read once per output site, the
// neighbour spinors are re-read through L1/L2 (t-neighbours of a 32^3 slab are
// a few MB apart, well inside the 126 MB L2), and every BLAS step of CG that
// can be is fused into the stencil epilogue.
#include "kernels.cuh"
#include "views.cuh"

namespace bqcdg {

// Resident CTAs per SM requested from the register allocator.  The reduced-
// precision stencils move few bytes per thread, so latency hiding needs more
// warps in flight than the FP64 ones (whose per-thread loads are 2-4x larger).
// The second pass carries the clover block, the input spinor and (fused into
// CG) x, r and p besides the hop, so it gets a larger register budget.
#ifndef BQCDG_SLOPPY_MIN_BLOCKS
#define BQCDG_SLOPPY_MIN_BLOCKS 6
#endif
#ifndef BQCDG_SLOPPY_MIN_BLOCKS2
#define BQCDG_SLOPPY_MIN_BLOCKS2 5
#endif
// The int16 passes load all eight links of their site up front
// (wilson_hop_lf), which takes about 120 registers: 4 CTAs per SM.
#ifndef BQCDG_HALF_MIN_BLOCKS
#define BQCDG_HALF_MIN_BLOCKS 4
#endif
template <Prec P>
struct Occ {
  static constexpr int min_blocks =
      P == Prec::F64 ? 1 : (P == Prec::F16 ? BQCDG_HALF_MIN_BLOCKS : BQCDG_SLOPPY_MIN_BLOCKS);
  static constexpr int min_blocks2 =
      P == Prec::F64 ? 1 : (P == Prec::F16 ? BQCDG_HALF_MIN_BLOCKS : BQCDG_SLOPPY_MIN_BLOCKS2);
};

// ---------------------------------------------------------------------------
// plain hopping term: out(e) = D_{e,o} in(o)   (d / d_dag, d/D21.F90:29-77)
// ---------------------------------------------------------------------------
template <Prec P, bool DAG>
__global__ void __launch_bounds__(kBlock) k_dslash(Geom g, int e, SpinorPtr outp, SpinorPtr inp, const void* gauge) {
  using R = typename SpinorView<P>::R;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.volh) return;
  auto in = sview<P>(inp, g.stride);
  auto out = sview<P>(outp, g.stride);
  auto U = gview<P>(gauge, g);
  Site st = site_coords(g, i, e);
  Spinor<R> b;
  zero(b);
  wilson_hop<P, DAG>(g, e, i, st, in, U, b);
  out.store(i, b);
}

void launch_dslash(Prec p, const Geom& g, int e, bool dag, SpinorPtr out, SpinorPtr in, const void* gauge,
                   cudaStream_t s) {
  dim3 grid(nblocks(g.volh));
#define DS(PP, D) k_dslash<PP, D><<<grid, kBlock, 0, s>>>(g, e, out, in, gauge)
  if (p == Prec::F64) { if (dag) DS(Prec::F64, true); else DS(Prec::F64, false); }
  else if (p == Prec::F32) { if (dag) DS(Prec::F32, true); else DS(Prec::F32, false); }
  else { if (dag) DS(Prec::F16, true); else DS(Prec::F16, false); }
#undef DS
}

// ---------------------------------------------------------------------------
// clover multiply: out = A in  (clover_mult_a / clover_mult_ao)
// ---------------------------------------------------------------------------
template <Prec P>
__global__ void __launch_bounds__(kBlock) k_clover_mult(Geom g, SpinorPtr outp, SpinorPtr inp, CloverPtr ap) {
  using R = typename SpinorView<P>::R;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.volh) return;
  auto in = sview<P>(inp, g.stride);
  auto out = sview<P>(outp, g.stride);
  auto A = cview<P>(ap, g.stride);
  Spinor<R> x, y;
  in.load(i, x);
  clover_apply(A, i, x, y);
  out.store(i, y);
}

void launch_clover_mult(Prec p, const Geom& g, SpinorPtr out, SpinorPtr in, CloverPtr a, cudaStream_t s) {
  dim3 grid(nblocks(g.volh));
  if (p == Prec::F64) k_clover_mult<Prec::F64><<<grid, kBlock, 0, s>>>(g, out, in, a);
  else if (p == Prec::F32) k_clover_mult<Prec::F32><<<grid, kBlock, 0, s>>>(g, out, in, a);
  else k_clover_mult<Prec::F16><<<grid, kBlock, 0, s>>>(g, out, in, a);
}

// ---------------------------------------------------------------------------
// clover_mult_b (clover_mult_b.F90 + clover_mult_b.h90): x = B^-1 x by
// forward (L), diagonal (1/D, halved) and backward (L^+) substitution.
// B slots: L(r,c) r>c at r(r-1)/2+c (15 complex), 1/D pairs at 15,16,17.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void ldl_solve(const double2* b, int i, int stride, int chi, cx<double> y[6],
                                          cx<double> x[6]) {
  cx<double> L[15];
#pragma unroll
  for (int k = 0; k < 15; k++) {
    double2 t = __ldg(b + (chi * 18 + k) * stride + i);
    L[k] = mkc(t.x, t.y);
  }
  double dinv[6];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    double2 t = __ldg(b + (chi * 18 + 15 + k) * stride + i);
    dinv[2 * k] = t.x;
    dinv[2 * k + 1] = t.y;
  }
#pragma unroll
  for (int r = 1; r < 6; r++) {
    cx<double> s = y[r];
#pragma unroll
    for (int c = 0; c < r; c++) s = s - L[r * (r - 1) / 2 + c] * y[c];
    y[r] = s;
  }
#pragma unroll
  for (int r = 5; r >= 0; r--) {
    cx<double> s = dinv[r] * y[r];
#pragma unroll
    for (int c = r + 1; c < 6; c++) s = s - conjg(L[c * (c - 1) / 2 + r]) * x[c];
    x[r] = s;
  }
}

__global__ void __launch_bounds__(kBlock) k_clover_mult_b(Geom g, double2* xf, const double2* b) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.volh) return;
  SpinorView<Prec::F64> X{xf, g.stride};
  Spinor<double> s;
  X.load(i, s);
  cx<double> y[6], xs[6];
  Spinor<double> o;
#pragma unroll
  for (int k = 0; k < 6; k++) y[k] = s.c[k / 3][k % 3] + s.c[k / 3 + 2][k % 3];
  ldl_solve(b, i, g.stride, 0, y, xs);
#pragma unroll
  for (int k = 0; k < 6; k++) {
    o.c[k / 3][k % 3] = xs[k];
    o.c[k / 3 + 2][k % 3] = xs[k];
  }
#pragma unroll
  for (int k = 0; k < 6; k++) y[k] = s.c[k / 3][k % 3] - s.c[k / 3 + 2][k % 3];
  ldl_solve(b, i, g.stride, 1, y, xs);
#pragma unroll
  for (int k = 0; k < 6; k++) {
    o.c[k / 3][k % 3] = o.c[k / 3][k % 3] + xs[k];
    o.c[k / 3 + 2][k % 3] = o.c[k / 3 + 2][k % 3] - xs[k];
  }
  X.store(i, o);
}

void launch_clover_mult_b(const Geom& g, double2* x, const double2* b, cudaStream_t s) {
  k_clover_mult_b<<<nblocks(g.volh), kBlock, 0, s>>>(g, x, b);
}

// ---------------------------------------------------------------------------
// mtil / mtil_dag, first half (m_tilde.F90:55-58, 92-95):
//   t_o = Ainv_oo D_oe in_e, then (1 - i h g5) t_o for mtil, (1 + i h g5) for mtil_dag
// ---------------------------------------------------------------------------
// KT: the clover field holds T (clover_apply_kt), A(kappa)^-1 is formed per
// site at kappa, or at kappa_rhs[rhs] (one hopping parameter per right-hand
// side) when that is given
template <Prec P, bool DAG, bool KT>
__global__ void __launch_bounds__(kBlock, Occ<P>::min_blocks) k_pass1(Geom g, SpinorPtr outp, SpinorPtr inp, const void* gauge,
                                                  CloverPtr ainv, int has_clover, double hval, const CgScalars* cg,
                                                  int nr, double kappa, const double* kappa_rhs, AlphaFin fin) {
  using R = typename SpinorView<P>::R;
  const Tile tl = tile(nr);
  if (cg && cg[tl.rhs].done) return;  // retired right-hand side
  if (fin.partial && tl.sb == 0) {
    // alpha of the k_pass2 before (launched with defer_alpha); the first
    // CTAs of a launch run this while the others start on their sites
    double tot[1];
    final_sum<1>(fin.partial + (size_t)tl.rhs * kRedVals * fin.stride, fin.stride, tl.nsb, tot);
    if (threadIdx.x == 0) {
      CgScalars* c = fin.cg + tl.rhs;
      c->paap = tot[0];
      c->alpha = c->rtr / tot[0];
    }
  }
  const int i = tl.i;
  if (i >= g.volh) return;
  auto in = sview<P>(rhs_of(inp, tl.rhs), g.stride);
  auto out = sview<P>(rhs_of(outp, tl.rhs), g.stride);
  auto U = gview<P>(gauge, g);
  Site st = site_coords(g, i, 1);
  Spinor<R> b;
  zero(b);
  if constexpr (P == Prec::F16) wilson_hop_lf<DAG>(g, 1, i, st, in, U, b);
  else wilson_hop<P, DAG>(g, 1, i, st, in, U, b);
  R osc = 1;  // a common factor of the output, folded into its storage scale
  if (has_clover) {
    Spinor<R> y;
    if constexpr (KT) clover_inv_apply_kt(cview<P>(ainv, g.stride), i, b, y, (R)(kappa_rhs ? kappa_rhs[tl.rhs] : kappa));
    else clover_apply_raw(cview<P>(ainv, g.stride), i, b, y, osc);
    b = y;
  }
  if (hval != 0.0) h_mult_b(b, (R)hval);
  out.store_scaled(i, b, osc);
}

void launch_mtil_pass1(Prec p, const Geom& g, bool dag, SpinorPtr out_o, SpinorPtr in_e, const void* gauge,
                       CloverPtr ainv_oo, const OpParams& op, const CgScalars* cg, cudaStream_t s, int nr,
                       const double* kappa_rhs, AlphaFin fin) {
  dim3 grid(nblocks(g.volh) * nr);
  int hc = op.csw_kappa != 0.0;
  double hv = dag ? op.h : -op.h;
#define P1(PP, D, K) \
  k_pass1<PP, D, K><<<grid, kBlock, 0, s>>>(g, out_o, in_e, gauge, ainv_oo, hc, hv, cg, nr, op.kappa, kappa_rhs, fin)
#define P1K(PP, D) if (g.clover_t) P1(PP, D, true); else P1(PP, D, false);
  if (p == Prec::F64) { if (dag) { P1K(Prec::F64, true) } else { P1K(Prec::F64, false) } }
  else if (p == Prec::F32) { if (dag) { P1K(Prec::F32, true) } else { P1K(Prec::F32, false) } }
  else { if (dag) { P1K(Prec::F16, true) } else { P1K(Prec::F16, false) } }
#undef P1K
#undef P1
}

// core of the second half: out = A_ee x + b D_eo t (clover) or x + b D_eo t
// (+ i h' g5 x for Wilson, h_mult.F90:27-49), + rho x  (m_tilde.F90:63-73,
// w_mult.F90:39).  The site-local terms come first and the hop sum is added
// onto them, so the clover block and x are dead before the neighbour gathers
// start; b is applied inside the hop sum and the storage scales of x and A_ee
// as one factor, so no field is rescaled component by component.
template <Prec P, bool DAG, bool KT>
__device__ __forceinline__ void pass2_core(const Geom& g, int i, const SpinorView<P>& t, const SpinorView<P>& xin,
                                           const GaugeView<P>& U, const CloverPtr& aee, int has_clover, double bcoef,
                                           double hval, double rho, Spinor<typename SpinorView<P>::R>& out,
                                           double kappa) {
  using R = typename SpinorView<P>::R;
  Spinor<R> x;
  R xsc;
  xin.load_raw(i, x, xsc);
  const R rr = (R)rho * xsc;
  if (has_clover) {
    R csc = 1;
    if constexpr (KT) clover_apply_kt(cview<P>(aee, g.stride), i, x, out, (R)kappa);
    else clover_apply_raw(cview<P>(aee, g.stride), i, x, out, csc);
    const R k = csc * xsc;
#pragma unroll
    for (int s = 0; s < 4; s++)
#pragma unroll
      for (int c = 0; c < 3; c++) out.c[s][c] = rho != 0.0 ? k * out.c[s][c] + rr * x.c[s][c] : k * out.c[s][c];
  } else {
    const R k = xsc + rr;
#pragma unroll
    for (int s = 0; s < 4; s++)
#pragma unroll
      for (int c = 0; c < 3; c++) out.c[s][c] = k * x.c[s][c];
    if (hval != 0.0) {
      const R hh = (R)hval * xsc;
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
  if constexpr (P == Prec::F16) wilson_hop_lf<DAG>(g, 0, i, st, t, U, out, (R)bcoef);
  else wilson_hop<P, DAG>(g, 0, i, st, t, U, out, (R)bcoef);
}

template <Prec P, bool DAG, bool REDUCE, bool KT>
__global__ void __launch_bounds__(kBlock, Occ<P>::min_blocks2) k_pass2(Geom g, SpinorPtr outp, SpinorPtr tp, SpinorPtr xp,
                                                  const void* gauge, CloverPtr aee, int has_clover, double bcoef,
                                                  double hval, double rho, RedScratch red, double* norm_out,
                                                  CgScalars* cg, int nr, const double* rho_rhs, double kappa,
                                                  const double* kappa_rhs, bool defer_alpha) {
  using R = typename SpinorView<P>::R;
  const Tile tl = tile(nr);
  if (cg && cg[tl.rhs].done) return;  // retired right-hand side
  if (rho_rhs) rho = rho_rhs[tl.rhs];   // a shift per right-hand side
  if (kappa_rhs) {                       // a hopping parameter per right-hand side
    kappa = kappa_rhs[tl.rhs];
    bcoef = -kappa * kappa / (1.0 + hval * hval);
  }
  const int i = tl.i;
  double acc[1] = {0.0};
  if (i < g.volh) {
    auto t = sview<P>(rhs_of(tp, tl.rhs), g.stride);
    auto xin = sview<P>(rhs_of(xp, tl.rhs), g.stride);
    auto out = sview<P>(rhs_of(outp, tl.rhs), g.stride);
    auto U = gview<P>(gauge, g);
    Spinor<R> o;
    pass2_core<P, DAG, KT>(g, i, t, xin, U, aee, has_clover, bcoef, hval, rho, o, kappa);
    out.store(i, o);
    if (REDUCE) {
#pragma unroll
      for (int s = 0; s < 4; s++)
#pragma unroll
        for (int c = 0; c < 3; c++) acc[0] += (double)norm2(o.c[s][c]);
    }
  }
  if (REDUCE) {
    double* part = red.partial + (size_t)tl.rhs * kRedVals * red.maxblocks;
    block_reduce_store<1>(acc, part, red.maxblocks, tl.sb);
    // defer_alpha: the partials stay for the next k_pass1 (AlphaFin).  The
    // arrival counter of the last-block sum costs a k_pass2<int16> at 32^3x64
    // 8 % of its time (137 against 127 us), its partial stores alone nothing.
    if (!defer_alpha && last_block(red.counter + tl.rhs, tl.nsb)) {
      double tot[1];
      final_sum<1>(part, red.maxblocks, tl.nsb, tot);
      if (threadIdx.x == 0) {
        if (norm_out) norm_out[tl.rhs] = tot[0];
        if (cg) {
          CgScalars* c = cg + tl.rhs;
          c->paap = tot[0];
          c->alpha = c->rtr / tot[0];
        }
        red.counter[tl.rhs] = 0;
      }
    }
  }
}

void launch_mtil_pass2(Prec p, const Geom& g, bool dag, SpinorPtr out_e, SpinorPtr t_o, SpinorPtr in_e,
                       const void* gauge, CloverPtr a_ee, const OpParams& op, RedScratch red, double* norm_out,
                       CgScalars* cg, cudaStream_t s, int nr, const double* rho_rhs, const double* kappa_rhs,
                       bool defer_alpha) {
  dim3 grid(nblocks(g.volh) * nr);
  int hc = op.csw_kappa != 0.0;
  double bcoef = -op.kappa * op.kappa / (1.0 + op.h * op.h);
  double hv = dag ? -op.h : op.h;
  bool reduce = norm_out != nullptr || cg != nullptr;
  defer_alpha = defer_alpha && cg && !norm_out;  // only alpha can wait for the next pass
#define P2(PP, D, RR, K)                                                                                        \
  k_pass2<PP, D, RR, K><<<grid, kBlock, 0, s>>>(g, out_e, t_o, in_e, gauge, a_ee, hc, bcoef, hv, op.rho, red, \
                                                norm_out, cg, nr, rho_rhs, op.kappa, kappa_rhs, defer_alpha)
#define P2R(PP, D)                                         \
  if (g.clover_t) {                                        \
    if (reduce) P2(PP, D, true, true); else P2(PP, D, false, true);   \
  } else {                                                 \
    if (reduce) P2(PP, D, true, false); else P2(PP, D, false, false); \
  }
  if (p == Prec::F64) { if (dag) { P2R(Prec::F64, true) } else { P2R(Prec::F64, false) } }
  else if (p == Prec::F32) { if (dag) { P2R(Prec::F32, true) } else { P2R(Prec::F32, false) } }
  else { if (dag) { P2R(Prec::F16, true) } else { P2R(Prec::F16, false) } }
#undef P2R
#undef P2
}

// ---------------------------------------------------------------------------
// CG-fused last pass of M^+M (cg.F90:93-107 folded into mtil_dag's second half)
// ---------------------------------------------------------------------------
template <Prec XP>
struct XR;
template <>
struct XR<Prec::F64> {
  using View = SpinorView<Prec::F64>;
};
template <>
struct XR<Prec::F32> {
  using View = SpinorView<Prec::F32>;
};

template <Prec P, Prec XP, bool XUPD, bool KT>
__global__ void __launch_bounds__(kBlock, Occ<P>::min_blocks2) k_cg_pass4(Geom g, SpinorPtr tp, SpinorPtr qp, const void* gauge,
                                                     CloverPtr aee, int has_clover, double bcoef, double hval,
                                                     double rho, SpinorPtr pp, SpinorPtr xp, SpinorPtr rp,
                                                     RedScratch red, CgScalars* cgs, int nr, const double* rho_rhs,
                                                     double kappa, const double* kappa_rhs, bool defer_step) {
  using R = typename SpinorView<P>::R;
  using RX = typename SpinorView<XP>::R;
  const Tile tl = tile(nr);
  CgScalars* cg = cgs + tl.rhs;
  if (cg->done) return;  // retired right-hand side
  if (rho_rhs) rho = rho_rhs[tl.rhs];  // a shift per right-hand side
  if (kappa_rhs) {                      // a hopping parameter per right-hand side
    kappa = kappa_rhs[tl.rhs];
    bcoef = -kappa * kappa / (1.0 + hval * hval);
  }
  const int i = tl.i;
  double acc[1] = {0.0};
  if (i < g.volh) {
    auto t = sview<P>(rhs_of(tp, tl.rhs), g.stride);
    auto q = sview<P>(rhs_of(qp, tl.rhs), g.stride);
    auto U = gview<P>(gauge, g);
    auto pv = sview<P>(rhs_of(pp, tl.rhs), g.stride);
    auto xv = sview<XP>(rhs_of(xp, tl.rhs), g.stride);
    auto rv = sview<XP>(rhs_of(rp, tl.rhs), g.stride);
    const RX a = (RX)cg->alpha;
    if (XUPD) {
      // x += alpha p first: alpha is known before the stencil, and x and p are
      // then dead while the stencil runs (otherwise k_cg_pupdate does it)
      Spinor<R> pl;
      R psc;
      pv.load_raw(i, pl, psc);
      Spinor<RX> xl;
      xv.load(i, xl);
      const RX ap_sc = a * (RX)psc;  // alpha and the storage scale of p
#pragma unroll
      for (int s = 0; s < 4; s++)
#pragma unroll
        for (int c = 0; c < 3; c++)
          xl.c[s][c] = xl.c[s][c] + ap_sc * mkc((RX)pl.c[s][c].x, (RX)pl.c[s][c].y);
      xv.store(i, xl);
    }
    Spinor<R> ap;
    pass2_core<P, true, KT>(g, i, t, q, U, aee, has_clover, bcoef, hval, rho, ap, kappa);
    Spinor<RX> rl;
    rv.load(i, rl);
#pragma unroll
    for (int s = 0; s < 4; s++)
#pragma unroll
      for (int c = 0; c < 3; c++) {
        rl.c[s][c] = rl.c[s][c] - a * mkc((RX)ap.c[s][c].x, (RX)ap.c[s][c].y);
        acc[0] += (double)norm2(rl.c[s][c]);
      }
    rv.store(i, rl);
  }
  double* part = red.partial + (size_t)tl.rhs * kRedVals * red.maxblocks;
  block_reduce_store<1>(acc, part, red.maxblocks, tl.sb);
  if (!defer_step && last_block(red.counter + tl.rhs, tl.nsb)) {
    double tot[1];
    final_sum<1>(part, red.maxblocks, tl.nsb, tot);
    if (threadIdx.x == 0) {
      cg_scalar_step(cg, tot[0]);
      red.counter[tl.rhs] = 0;
    }
  }
}

// the deferred step of k_cg_pass4 (defer_step): CTA r sums RHS r's partials
// with all its threads in flight at once and steps its scalars
constexpr int kStepBlock = 1024;
__global__ void __launch_bounds__(kStepBlock) k_cg_step(RedScratch red, CgScalars* cgs, int nsb) {
  CgScalars* cg = cgs + blockIdx.x;
  if (cg->done) return;  // k_cg_pass4 did not run for this right-hand side
  double tot[1];
  final_sum<1>(red.partial + (size_t)blockIdx.x * kRedVals * red.maxblocks, red.maxblocks, nsb, tot);
  if (threadIdx.x == 0) cg_scalar_step(cg, tot[0]);
}

void launch_cg_step(RedScratch red, CgScalars* cg, int nr, int nsb, cudaStream_t s) {
  k_cg_step<<<nr, kStepBlock, 0, s>>>(red, cg, nsb);
}

void launch_cg_pass4(Prec p, const Geom& g, SpinorPtr t_o, SpinorPtr q_e, const void* gauge, CloverPtr a_ee,
                     const OpParams& op, SpinorPtr pvec, SpinorPtr x, SpinorPtr r, RedScratch red, CgScalars* cg,
                     cudaStream_t s, int nr, bool xupd, const double* rho_rhs, const double* kappa_rhs,
                     bool defer_step) {
  dim3 grid(nblocks(g.volh) * nr);
  int hc = op.csw_kappa != 0.0;
  double bcoef = -op.kappa * op.kappa / (1.0 + op.h * op.h);
  double hv = -op.h;  // mtil_dag
#define P4(PP, XX, XU, K)                                                                                   \
  k_cg_pass4<PP, XX, XU, K><<<grid, kBlock, 0, s>>>(g, t_o, q_e, gauge, a_ee, hc, bcoef, hv, op.rho, pvec, x, r, \
                                                    red, cg, nr, rho_rhs, op.kappa, kappa_rhs, defer_step)
#define P4K(PP, XX, XU) if (g.clover_t) P4(PP, XX, XU, true); else P4(PP, XX, XU, false);
  if (p == Prec::F64) { if (xupd) { P4K(Prec::F64, Prec::F64, true) } else { P4K(Prec::F64, Prec::F64, false) } }
  else if (p == Prec::F32) { if (xupd) { P4K(Prec::F32, Prec::F32, true) } else { P4K(Prec::F32, Prec::F32, false) } }
  else { if (xupd) { P4K(Prec::F16, Prec::F32, true) } else { P4K(Prec::F16, Prec::F32, false) } }
#undef P4K
#undef P4
}

// p = r + beta p   (sc_xpby, cg.F90:116), and, when x is given, the x += alpha p
// of the same iteration (cg.F90:101), which then runs here instead of in the
// stencil pass: this kernel reads p anyway.  The launch belongs to iteration
// `expect`: x is updated iff that iteration ran (its k_cg_pass4 counted it),
// p iff the solve goes on; so the update of the last iteration is not lost
// when the solver stops, and no x update is applied twice.
template <Prec P, Prec RP, bool XUPD>
__global__ void __launch_bounds__(kBlock) k_cg_pupdate(Geom g, SpinorPtr pp, SpinorPtr rp, SpinorPtr xp,
                                                       const CgScalars* cgs, int nr, int expect) {
  using R = typename SpinorView<P>::R;
  using RR = typename SpinorView<RP>::R;
  const Tile tl = tile(nr);
  const CgScalars* cg = cgs + tl.rhs;
  const bool upd_p = !cg->done;
  const bool upd_x = XUPD && cg->iter == expect;
  if (!upd_p && !upd_x) return;
  const int i = tl.i;
  if (i >= g.volh) return;
  auto pv = sview<P>(rhs_of(pp, tl.rhs), g.stride);
  Spinor<R> pl;
  R psc;
  pv.load_raw(i, pl, psc);
  if (XUPD && upd_x) {
    auto xv = sview<RP>(rhs_of(xp, tl.rhs), g.stride);
    Spinor<RR> xl;
    xv.load(i, xl);
    const RR a = (RR)cg->alpha * (RR)psc;
#pragma unroll
    for (int s = 0; s < 4; s++)
#pragma unroll
      for (int c = 0; c < 3; c++) xl.c[s][c] = xl.c[s][c] + a * mkc((RR)pl.c[s][c].x, (RR)pl.c[s][c].y);
    xv.store(i, xl);
  }
  if (!upd_p) return;
  auto rv = sview<RP>(rhs_of(rp, tl.rhs), g.stride);
  Spinor<RR> rl;
  rv.load(i, rl);
  const R b = (R)cg->beta * psc;
#pragma unroll
  for (int s = 0; s < 4; s++)
#pragma unroll
    for (int c = 0; c < 3; c++) pl.c[s][c] = mkc((R)rl.c[s][c].x, (R)rl.c[s][c].y) + b * pl.c[s][c];
  pv.store(i, pl);
}

void launch_cg_pupdate(Prec p, const Geom& g, SpinorPtr pvec, SpinorPtr r, CgScalars* cg, cudaStream_t s, int nr,
                       SpinorPtr x, int expect) {
  dim3 grid(nblocks(g.volh) * nr);
  const bool xu = x.v != nullptr;
#define PU(PP, RR, XU) k_cg_pupdate<PP, RR, XU><<<grid, kBlock, 0, s>>>(g, pvec, r, x, cg, nr, expect)
  if (p == Prec::F64) { if (xu) PU(Prec::F64, Prec::F64, true); else PU(Prec::F64, Prec::F64, false); }
  else if (p == Prec::F32) { if (xu) PU(Prec::F32, Prec::F32, true); else PU(Prec::F32, Prec::F32, false); }
  else { if (xu) PU(Prec::F16, Prec::F32, true); else PU(Prec::F16, Prec::F32, false); }
#undef PU
}

}  // namespace bqcdg
