// dslash_multi.cu -- register-blocked batched stencil passes for sm_100a.
//
// The batched kernels of dslash.cu give each CTA one right-hand side, so the
// nr CTAs of one site block share links and clover blocks only through L2:
// every RHS still loads, decodes and reconstructs each link and clover block
// itself.  Here one thread serves one site for NB right-hand sides (NB = 2 or
// 4): per hop the link is loaded, decoded and its third column rebuilt once
// and applied to the NB half spinors; each chiral clover block is loaded once
// and applied to NB spinors; the site coordinates and neighbour indices are
// computed once.  Per RHS and pass this leaves 2 spinors of HBM traffic plus
// (8 links + 1 clover block) / NB, the per-site figure (8G + C)/N + 2S.
//
// The arithmetic of every RHS is that of the single-RHS passes (m_tilde.F90:
// 43-114 through wilson_hop and the clover apply); only the loop nest differs.
// Retired right-hand sides are skipped per RHS (the flag is uniform across a
// CTA), and reductions go to the same per-RHS partial slots as in dslash.cu.
#include "kernels.cuh"
#include "views.cuh"

namespace bqcdg {

// CTA b serves RHS group b % ng (RHS grp*NB .. grp*NB+NB-1, those below nr)
// and site block b / ng: the ng CTAs of one site block are adjacent
struct GTile {
  int grp;
  int sb;
  int nsb;
  int i;
};
__device__ __forceinline__ GTile gtile(int ng) {
  GTile t;
  t.grp = blockIdx.x % ng;
  t.sb = blockIdx.x / ng;
  t.nsb = gridDim.x / ng;
  t.i = t.sb * blockDim.x + threadIdx.x;
  return t;
}

// which RHS of group rhs0.. are live (below nr and not retired); false if none
template <int NB>
__device__ __forceinline__ bool group_live(const CgScalars* cg, int rhs0, int nr, bool (&act)[NB]) {
  bool any = false;
#pragma unroll
  for (int r = 0; r < NB; r++) {
    act[r] = rhs0 + r < nr && !(cg && cg[rhs0 + r].done);
    any = any || act[r];
  }
  return any;
}

// the projected half spinor of one hop from the neighbour j (as in wilson_hop)
template <Prec PS, bool DAG>
__device__ __forceinline__ void load_project(const SpinorView<PS>& in, int j, int mu, bool fwd,
                                             cx<typename SpinorView<PS>::R> h[2][3],
                                             typename SpinorView<PS>::R& sc) {
  using R = typename SpinorView<PS>::R;
  if (mu == 3) {
    // (1 -+ gamma_4) keeps two spins: (3,4) / (1,2) by direction and dagger
    in.load_pair_raw(j, fwd ? (DAG ? 0 : 2) : (DAG ? 2 : 0), h, sc);
  } else if constexpr (PS == Prec::F16) {
    float2 F[4][3];
    in.load_biased(j, F, sc);
    project_biased<DAG>(F, mu, fwd, h);
  } else {
    Spinor<R> p;
    in.load_raw(j, p, sc);
    project<R, DAG>(p, mu, fwd, h);
  }
}

// b[r] += hscale * (hopping term of in[r]) for the live r: wilson_hop with
// the link of each hop loaded and decoded once for all NB right-hand sides
template <Prec PS, bool DAG, int NB, typename UV>
__device__ __forceinline__ void wilson_hop_n(const Geom& g, int e, int i, const Site& st,
                                             const SpinorView<PS> (&in)[NB], const bool (&act)[NB], const UV& U,
                                             Spinor<typename SpinorView<PS>::R> (&b)[NB],
                                             typename SpinorView<PS>::R hscale) {
  using R = typename SpinorView<PS>::R;
  const int o = 1 - e;
#pragma unroll
  for (int mu = 3; mu >= 0; mu--) {
    {
      const int j = neighbour(g, st, i, mu, true);
      const R sgn = (R)hop_sign(g, st, mu, true);
      Link<R> u;
      R lsc;
      U.hop_link(mu, true, e, i, u, lsc);
#pragma unroll
      for (int r = 0; r < NB; r++) {
        if (!act[r]) continue;
        cx<R> h[2][3], f[2][3];
        R sc;
        load_project<PS, DAG>(in[r], j, mu, true, h, sc);
        mul_u(u, h, f);
        recon_fwd<R, DAG>(b[r], mu, f, sgn * sc * lsc * hscale);
      }
    }
    {
      const int j = neighbour(g, st, i, mu, false);
      const R sgn = (R)hop_sign(g, st, mu, false);
      Link<R> u;
      R lsc;
      U.hop_link(mu, false, o, j, u, lsc);
#pragma unroll
      for (int r = 0; r < NB; r++) {
        if (!act[r]) continue;
        cx<R> h[2][3], f[2][3];
        R sc;
        load_project<PS, DAG>(in[r], j, mu, false, h, sc);
        mul_ud(u, h, f);
        recon_bwd<R, DAG>(b[r], mu, f, sgn * sc * lsc * hscale);
      }
    }
  }
}

// clover_block_mv with sh added to the real diagonal: y = (A + sh) x
template <typename R>
__device__ __forceinline__ void clover_block_mv_shift(const cx<R>* a, const cx<R> x[6], cx<R> y[6], R sh) {
  cx<R> b[18];
#pragma unroll
  for (int k = 0; k < 18; k++) b[k] = a[k];
  b[0] = mkc(a[0].x + sh, a[0].y + sh);
  b[10] = mkc(a[10].x + sh, a[10].y + sh);
  b[16] = mkc(a[16].x + sh, a[16].y + sh);
  clover_block_mv(b, x, y);
}

// s[r] <- (A / sc) s[r] in place for the live r (clover_apply_raw), each
// chiral block loaded once for all of them.  With SHIFT, (A / sc + 2 sh[r])
// s[r]: the halved blocks act on x+- = up +- dn, so sh on their diagonal adds
// 2 sh to the operator.  The spinors go to the chiral basis (up + dn, up - dn)
// and back in place, so besides them only one block and one 6-vector are live.
template <bool SHIFT, typename CV, typename R, int NB>
__device__ __forceinline__ void clover_apply_n(const CV& A, int i, Spinor<R> (&s)[NB], const bool (&act)[NB],
                                               const R (&sh)[NB], R& sc) {
#pragma unroll
  for (int r = 0; r < NB; r++) {
    if (!act[r]) continue;
#pragma unroll
    for (int k = 0; k < 6; k++) {
      const cx<R> up = s[r].c[k / 3][k % 3], dn = s[r].c[k / 3 + 2][k % 3];
      s[r].c[k / 3][k % 3] = up + dn;
      s[r].c[k / 3 + 2][k % 3] = up - dn;
    }
  }
#pragma unroll
  for (int chi = 0; chi < 2; chi++) {
    cx<R> a[18];
    A.load_block_raw(i, chi, a, sc);  // both blocks of a site share one scale
#pragma unroll
    for (int r = 0; r < NB; r++) {
      if (!act[r]) continue;
      cx<R> x[6], y[6];
#pragma unroll
      for (int k = 0; k < 6; k++) x[k] = s[r].c[k / 3 + 2 * chi][k % 3];
      if (SHIFT) clover_block_mv_shift(a, x, y, sh[r]);
      else clover_block_mv(a, x, y);
#pragma unroll
      for (int k = 0; k < 6; k++) s[r].c[k / 3 + 2 * chi][k % 3] = y[k];
    }
  }
#pragma unroll
  for (int r = 0; r < NB; r++) {
    if (!act[r]) continue;
#pragma unroll
    for (int k = 0; k < 6; k++) {
      const cx<R> p = s[r].c[k / 3][k % 3], m = s[r].c[k / 3 + 2][k % 3];
      s[r].c[k / 3][k % 3] = p + m;
      s[r].c[k / 3 + 2][k % 3] = p - m;
    }
  }
}

// the storage scale of a site's clover blocks (1 except for int16)
template <Prec P>
__device__ __forceinline__ float clover_scale(const CloverView<P>& A, int i) {
  if constexpr (P == Prec::F16) return __ldg(A.norm + i) * (1.0f / 32767.0f);
  else return 1.0f;
}

// register budget: NB = 2 keeps 4 CTAs of 128 threads per SM (128 registers),
// NB = 4 keeps 3 (168 registers)
template <int NB>
struct OccN {
  static constexpr int min_blocks = NB == 2 ? 4 : 3;
};

// ---------------------------------------------------------------------------
// first half of mtil / mtil_dag for NB right-hand sides per thread
// (k_pass1 of dslash.cu): t_r = Ainv_oo D_oe in_r, then (1 -+ i h g5) t_r
// ---------------------------------------------------------------------------
template <Prec P, bool DAG, int NB>
__global__ void __launch_bounds__(kBlock, OccN<NB>::min_blocks)
    k_pass1_n(Geom g, SpinorPtr outp, SpinorPtr inp, const void* gauge, CloverPtr ainv, int has_clover, double hval,
              const CgScalars* cg, int nr, int ng, AlphaFin fin) {
  using R = typename SpinorView<P>::R;
  const GTile tl = gtile(ng);
  const int rhs0 = tl.grp * NB;
  bool act[NB];
  if (!group_live<NB>(cg, rhs0, nr, act)) return;
  if (fin.partial && tl.sb == 0) {
    // alpha of the k_pass2_n before (defer_alpha), as in k_pass1
    double tot[NB];
    final_sum<NB>(fin.partial + (size_t)rhs0 * kRedVals * fin.stride, kRedVals * fin.stride, tl.nsb, tot);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int r = 0; r < NB; r++) {
        if (!act[r]) continue;
        CgScalars* c = fin.cg + rhs0 + r;
        c->paap = tot[r];
        c->alpha = c->rtr / tot[r];
      }
    }
  }
  const int i = tl.i;
  if (i >= g.volh) return;
  SpinorView<P> in[NB];
#pragma unroll
  for (int r = 0; r < NB; r++) in[r] = sview<P>(rhs_of(inp, rhs0 + r), g.stride);
  auto U = gview<P>(gauge, g);
  const Site st = site_coords(g, i, 1);
  Spinor<R> b[NB];
#pragma unroll
  for (int r = 0; r < NB; r++) zero(b[r]);
  wilson_hop_n<P, DAG, NB>(g, 1, i, st, in, act, U, b, (R)1);
  R osc = 1;  // a common factor of the outputs, folded into their storage scale
  if (has_clover) {
    const R none[NB] = {};
    clover_apply_n<false>(cview<P>(ainv, g.stride), i, b, act, none, osc);
  }
#pragma unroll
  for (int r = 0; r < NB; r++) {
    if (!act[r]) continue;
    if (hval != 0.0) h_mult_b(b[r], (R)hval);
    sview<P>(rhs_of(outp, rhs0 + r), g.stride).store_scaled(i, b[r], osc);
  }
}

void launch_mtil_pass1_n(Prec p, const Geom& g, bool dag, SpinorPtr out_o, SpinorPtr in_e, const void* gauge,
                         CloverPtr ainv_oo, const OpParams& op, const CgScalars* cg, cudaStream_t s, int nr,
                         int nbt, AlphaFin fin) {
  const int ng = (nr + nbt - 1) / nbt;
  dim3 grid(nblocks(g.volh) * ng);
  int hc = op.csw_kappa != 0.0;
  double hv = dag ? op.h : -op.h;
#define P1N(PP, D, N) \
  k_pass1_n<PP, D, N><<<grid, kBlock, 0, s>>>(g, out_o, in_e, gauge, ainv_oo, hc, hv, cg, nr, ng, fin)
#define P1NB(PP, N) \
  if (dag) P1N(PP, true, N); else P1N(PP, false, N)
  if (p == Prec::F32) { if (nbt == 2) { P1NB(Prec::F32, 2); } else { P1NB(Prec::F32, 4); } }
  else { if (nbt == 2) { P1NB(Prec::F16, 2); } else { P1NB(Prec::F16, 4); } }
#undef P1NB
#undef P1N
}

// ---------------------------------------------------------------------------
// second half for NB right-hand sides (pass2_core of dslash.cu):
// out_r = A_ee x_r + b D_eo t_r + rho_r x_r (Wilson: (1 + rho_r) x_r + b D t_r);
// h = 0.  The site-local terms come first, as in pass2_core, so the clover
// blocks and x are dead before the neighbour gathers start.
// ---------------------------------------------------------------------------
template <Prec P, bool DAG, int NB>
__device__ __forceinline__ void pass2_core_n(const Geom& g, int i, const SpinorView<P> (&t)[NB],
                                             const SpinorView<P> (&xin)[NB], const bool (&act)[NB],
                                             const GaugeView<P>& U, const CloverPtr& aee, int has_clover,
                                             double bcoef, const double (&rho)[NB],
                                             Spinor<typename SpinorView<P>::R> (&out)[NB]) {
  using R = typename SpinorView<P>::R;
  R xsc[NB];
#pragma unroll
  for (int r = 0; r < NB; r++)
    if (act[r]) xin[r].load_raw(i, out[r], xsc[r]);
  if (has_clover) {
    const auto A = cview<P>(aee, g.stride);
    // rho x = k (2 sh) x_raw with k = csc xsc: sh = rho / (2 csc)
    const R csc = (R)clover_scale<P>(A, i);
    R sh[NB];
#pragma unroll
    for (int r = 0; r < NB; r++) sh[r] = (R)rho[r] * ((R)0.5 / csc);
    R sc;
    clover_apply_n<true>(A, i, out, act, sh, sc);
#pragma unroll
    for (int r = 0; r < NB; r++) {
      if (!act[r]) continue;
      const R k = csc * xsc[r];
#pragma unroll
      for (int s = 0; s < 4; s++)
#pragma unroll
        for (int c = 0; c < 3; c++) out[r].c[s][c] = k * out[r].c[s][c];
    }
  } else {
#pragma unroll
    for (int r = 0; r < NB; r++) {
      if (!act[r]) continue;
      const R k = xsc[r] + (R)rho[r] * xsc[r];
#pragma unroll
      for (int s = 0; s < 4; s++)
#pragma unroll
        for (int c = 0; c < 3; c++) out[r].c[s][c] = k * out[r].c[s][c];
    }
  }
  const Site st = site_coords(g, i, 0);
  wilson_hop_n<P, DAG, NB>(g, 0, i, st, t, act, U, out, (R)bcoef);
}

// the shifts of the group's right-hand sides
template <int NB>
__device__ __forceinline__ void group_rho(double rho, const double* rho_rhs, int rhs0, const bool (&act)[NB],
                                          double (&out)[NB]) {
#pragma unroll
  for (int r = 0; r < NB; r++) out[r] = rho_rhs && act[r] ? rho_rhs[rhs0 + r] : rho;
}

// q_r = M~ p_r (second half, dag = false) with the CG alpha_r = rtr_r /
// |q_r|^2 of every live RHS (k_pass2 of dslash.cu with its reduction)
template <Prec P, int NB>
__global__ void __launch_bounds__(kBlock, OccN<NB>::min_blocks)
    k_pass2_n(Geom g, SpinorPtr outp, SpinorPtr tp, SpinorPtr xp, const void* gauge, CloverPtr aee, int has_clover,
              double bcoef, double rho, RedScratch red, CgScalars* cg, int nr, int ng, const double* rho_rhs,
              bool defer_alpha) {
  using R = typename SpinorView<P>::R;
  const GTile tl = gtile(ng);
  const int rhs0 = tl.grp * NB;
  bool act[NB];
  if (!group_live<NB>(cg, rhs0, nr, act)) return;
  double rh[NB];
  group_rho<NB>(rho, rho_rhs, rhs0, act, rh);
  const int i = tl.i;
  double acc[NB];
#pragma unroll
  for (int r = 0; r < NB; r++) acc[r] = 0.0;
  if (i < g.volh) {
    SpinorView<P> t[NB], x[NB];
#pragma unroll
    for (int r = 0; r < NB; r++) {
      t[r] = sview<P>(rhs_of(tp, rhs0 + r), g.stride);
      x[r] = sview<P>(rhs_of(xp, rhs0 + r), g.stride);
    }
    Spinor<R> o[NB];
    pass2_core_n<P, false, NB>(g, i, t, x, act, gview<P>(gauge, g), aee, has_clover, bcoef, rh, o);
#pragma unroll
    for (int r = 0; r < NB; r++) {
      if (!act[r]) continue;
      sview<P>(rhs_of(outp, rhs0 + r), g.stride).store(i, o[r]);
#pragma unroll
      for (int s = 0; s < 4; s++)
#pragma unroll
        for (int c = 0; c < 3; c++) acc[r] += (double)norm2(o[r].c[s][c]);
    }
  }
  // value r of the group goes to the partial slot of RHS rhs0 + r
  double* part = red.partial + (size_t)rhs0 * kRedVals * red.maxblocks;
  block_reduce_store<NB>(acc, part, kRedVals * red.maxblocks, tl.sb);
  if (!defer_alpha && last_block(red.counter + rhs0, tl.nsb)) {
    double tot[NB];
    final_sum<NB>(part, kRedVals * red.maxblocks, tl.nsb, tot);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int r = 0; r < NB; r++) {
        if (!act[r]) continue;
        CgScalars* c = cg + rhs0 + r;
        c->paap = tot[r];
        c->alpha = c->rtr / tot[r];
      }
      red.counter[rhs0] = 0;
    }
  }
}

void launch_mtil_pass2_n(Prec p, const Geom& g, SpinorPtr out_e, SpinorPtr t_o, SpinorPtr in_e, const void* gauge,
                         CloverPtr a_ee, const OpParams& op, RedScratch red, CgScalars* cg, cudaStream_t s, int nr,
                         const double* rho_rhs, int nbt, bool defer_alpha) {
  const int ng = (nr + nbt - 1) / nbt;
  dim3 grid(nblocks(g.volh) * ng);
  int hc = op.csw_kappa != 0.0;
  double bcoef = -op.kappa * op.kappa;  // h = 0
#define P2N(PP, N)                                                                                          \
  k_pass2_n<PP, N><<<grid, kBlock, 0, s>>>(g, out_e, t_o, in_e, gauge, a_ee, hc, bcoef, op.rho, red, cg, nr, ng, \
                                           rho_rhs, defer_alpha)
  if (p == Prec::F32) { if (nbt == 2) P2N(Prec::F32, 2); else P2N(Prec::F32, 4); }
  else { if (nbt == 2) P2N(Prec::F16, 2); else P2N(Prec::F16, 4); }
#undef P2N
}

// CG-fused second half of mtil_dag for NB right-hand sides (k_cg_pass4 of
// dslash.cu, x updated here): x_r += alpha_r p_r, Ap_r = A_ee q_r + b D_eo t_r
// + rho_r q_r, r_r -= alpha_r Ap_r, and the CG scalars from |r_r|^2
template <Prec P, int NB>
__global__ void __launch_bounds__(kBlock, OccN<NB>::min_blocks)
    k_cg_pass4_n(Geom g, SpinorPtr tp, SpinorPtr qp, const void* gauge, CloverPtr aee, int has_clover, double bcoef,
                 double rho, SpinorPtr pp, SpinorPtr xp, SpinorPtr rp, RedScratch red, CgScalars* cgs, int nr, int ng,
                 const double* rho_rhs, bool defer_step) {
  using R = typename SpinorView<P>::R;
  const GTile tl = gtile(ng);
  const int rhs0 = tl.grp * NB;
  bool act[NB];
  if (!group_live<NB>(cgs, rhs0, nr, act)) return;
  double rh[NB];
  group_rho<NB>(rho, rho_rhs, rhs0, act, rh);
  const int i = tl.i;
  double acc[NB];
#pragma unroll
  for (int r = 0; r < NB; r++) acc[r] = 0.0;
  if (i < g.volh) {
    // x += alpha p first: alpha is known before the stencil, and x and p are
    // then dead while the stencil runs
#pragma unroll
    for (int r = 0; r < NB; r++) {
      if (!act[r]) continue;
      const auto pv = sview<P>(rhs_of(pp, rhs0 + r), g.stride);
      const auto xv = sview<Prec::F32>(rhs_of(xp, rhs0 + r), g.stride);
      Spinor<R> pl;
      R psc;
      pv.load_raw(i, pl, psc);
      Spinor<float> xl;
      xv.load(i, xl);
      const float ap_sc = (float)cgs[rhs0 + r].alpha * (float)psc;
#pragma unroll
      for (int s = 0; s < 4; s++)
#pragma unroll
        for (int c = 0; c < 3; c++) xl.c[s][c] = xl.c[s][c] + ap_sc * mkc((float)pl.c[s][c].x, (float)pl.c[s][c].y);
      xv.store(i, xl);
    }
    SpinorView<P> t[NB], q[NB];
#pragma unroll
    for (int r = 0; r < NB; r++) {
      t[r] = sview<P>(rhs_of(tp, rhs0 + r), g.stride);
      q[r] = sview<P>(rhs_of(qp, rhs0 + r), g.stride);
    }
    Spinor<R> ap[NB];
    pass2_core_n<P, true, NB>(g, i, t, q, act, gview<P>(gauge, g), aee, has_clover, bcoef, rh, ap);
#pragma unroll
    for (int r = 0; r < NB; r++) {
      if (!act[r]) continue;
      const auto rv = sview<Prec::F32>(rhs_of(rp, rhs0 + r), g.stride);
      const float a = (float)cgs[rhs0 + r].alpha;
      Spinor<float> rl;
      rv.load(i, rl);
#pragma unroll
      for (int s = 0; s < 4; s++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
          rl.c[s][c] = rl.c[s][c] - a * mkc((float)ap[r].c[s][c].x, (float)ap[r].c[s][c].y);
          acc[r] += (double)norm2(rl.c[s][c]);
        }
      rv.store(i, rl);
    }
  }
  double* part = red.partial + (size_t)rhs0 * kRedVals * red.maxblocks;
  block_reduce_store<NB>(acc, part, kRedVals * red.maxblocks, tl.sb);
  if (!defer_step && last_block(red.counter + rhs0, tl.nsb)) {
    double tot[NB];
    final_sum<NB>(part, kRedVals * red.maxblocks, tl.nsb, tot);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int r = 0; r < NB; r++) {
        if (!act[r]) continue;
        cg_scalar_step(cgs + rhs0 + r, tot[r]);
      }
      red.counter[rhs0] = 0;
    }
  }
}

void launch_cg_pass4_n(Prec p, const Geom& g, SpinorPtr t_o, SpinorPtr q_e, const void* gauge, CloverPtr a_ee,
                       const OpParams& op, SpinorPtr pvec, SpinorPtr x, SpinorPtr r, RedScratch red, CgScalars* cg,
                       cudaStream_t s, int nr, const double* rho_rhs, int nbt, bool defer_step) {
  const int ng = (nr + nbt - 1) / nbt;
  dim3 grid(nblocks(g.volh) * ng);
  int hc = op.csw_kappa != 0.0;
  double bcoef = -op.kappa * op.kappa;  // h = 0
#define P4N(PP, N)                                                                                              \
  k_cg_pass4_n<PP, N><<<grid, kBlock, 0, s>>>(g, t_o, q_e, gauge, a_ee, hc, bcoef, op.rho, pvec, x, r, red, cg, nr, \
                                              ng, rho_rhs, defer_step)
  if (p == Prec::F32) { if (nbt == 2) P4N(Prec::F32, 2); else P4N(Prec::F32, 4); }
  else { if (nbt == 2) P4N(Prec::F16, 2); else P4N(Prec::F16, 4); }
#undef P4N
}

}  // namespace bqcdg
