// force.cu -- pseudofermion force kernels for sm_100a (FP64 accumulation).
//
//   hopping part   dsf.F90:75-100 with d/DSFxyzt.F90:77-117, one thread per
//                  link, forward and backward terms of that link fused;
//   clover part    clover_bsa.F90 / clover_ts.F90 build the six sigma_mu_nu
//                  planes w per site, then clover_d.F90:110-264 contracts them
//                  with the clover-leaf staples: one thread per link gathers
//                  the contributions of the three planes through its direction
//                  (one of the 24 loops of clover_d_mu_nu touches each link per
//                  plane), so p is read and written once per call.
#include "kernels.cuh"
#include "su3.cuh"

namespace bqcdg {

// ---------------------------------------------------------------------------
// hopping force
// ---------------------------------------------------------------------------
// gamma projections of DSFxyzt.F90:28-60; sg = +1 (forward) / -1 (backward)
__device__ __forceinline__ void dsf_gamma(const Spinor<double>& a, int ca, int mu, bool fwd, C64 g[4]) {
  const double sg = fwd ? 1.0 : -1.0;
  C64 a1 = a.c[0][ca], a2 = a.c[1][ca], a3 = a.c[2][ca], a4 = a.c[3][ca];
  if (mu == 0) {
    g[0] = a1 - sg * itimes(a4);
    g[1] = a2 - sg * itimes(a3);
    g[2] = sg * itimes(g[1]);
    g[3] = sg * itimes(g[0]);
  } else if (mu == 1) {
    g[0] = a1 - sg * a4;
    g[1] = a2 + sg * a3;
    g[2] = sg * g[1];
    g[3] = -sg * g[0];
  } else if (mu == 2) {
    g[0] = a1 - sg * itimes(a3);
    g[1] = a2 + sg * itimes(a4);
    g[2] = sg * itimes(g[0]);
    g[3] = -sg * itimes(g[1]);
  } else if (fwd) {
    g[0] = mkc(0.0, 0.0);
    g[1] = mkc(0.0, 0.0);
    g[2] = 2.0 * a3;
    g[3] = 2.0 * a4;
  } else {
    g[0] = 2.0 * a1;
    g[1] = 2.0 * a2;
    g[2] = mkc(0.0, 0.0);
    g[3] = mkc(0.0, 0.0);
  }
}

// w(ca,cb) = sum_s G_s(ca) conj(b(s,cb))
__device__ __forceinline__ void dsf_w(const Spinor<double>& a, const Spinor<double>& b, int mu, bool fwd, L64& w) {
#pragma unroll
  for (int ca = 0; ca < 3; ca++) {
    C64 gm[4];
    dsf_gamma(a, ca, mu, fwd, gm);
#pragma unroll
    for (int cb = 0; cb < 3; cb++) {
      C64 t = mulc(gm[0], b.c[0][cb]);
      t = t + mulc(gm[1], b.c[1][cb]);
      t = t + mulc(gm[2], b.c[2][cb]);
      t = t + mulc(gm[3], b.c[3][cb]);
      w.m[ca][cb] = t;
    }
  }
}

// p(eo,mu,i): link parity eo.  Even links: forward term from (b at i, at at
// x+mu), backward from (a at i, bt at x+mu); odd links swap (a,b)<->(at,bt)
// (dsf.F90:80-98).
__global__ void __launch_bounds__(kBlock) k_dsf_hop(Geom g, double* p, const double2* gauge, const double2* a,
                                                    const double2* b, const double2* at, const double2* bt,
                                                    double s) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int me = blockIdx.y;
  if (i >= g.volh) return;
  int mu = me >> 1, eo = me & 1;
  Site st = site_coords(g, i, eo);
  int j = neighbour(g, st, i, mu, true);
  const double2* bh = eo == 0 ? b : bt;   // b-type field here
  const double2* af = eo == 0 ? at : a;   // a-type field at x+mu
  const double2* ah = eo == 0 ? a : at;   // a-type field here
  const double2* bf = eo == 0 ? bt : b;   // b-type field at x+mu
  SpinorView<Prec::F64> BH{(double2*)bh, g.stride}, AF{(double2*)af, g.stride}, AH{(double2*)ah, g.stride},
      BF{(double2*)bf, g.stride};
  L64 u;
  GaugeView<Prec::F64>{(double2*)gauge, g.stride}.load(mu, eo, i, u);
  const double sgn = (double)hop_sign(g, st, mu, true);
  double q[8];
  double* pp = p + ((size_t)me * g.volh + i) * 8;
#pragma unroll
  for (int k = 0; k < 8; k++) q[k] = pp[k];
  {
    Spinor<double> sa, sb;
    AF.load(j, sa);
    BH.load(i, sb);
    L64 w, v;
    dsf_w(sa, sb, mu, true, w);
    mul2(v, u, false, w, false);
    im_tr_j(q, v, -s * sgn);
  }
  {
    Spinor<double> sa, sb;
    AH.load(i, sa);
    BF.load(j, sb);
    L64 w, v;
    dsf_w(sa, sb, mu, false, w);
    mul2(v, w, false, u, true);
    im_tr_j(q, v, s * sgn);
  }
#pragma unroll
  for (int k = 0; k < 8; k++) pp[k] = q[k];
}

void launch_dsf_hop(const Geom& g, double* p, const double2* gauge, const double2* a, const double2* b,
                    const double2* at, const double2* bt, double s, cudaStream_t st) {
  k_dsf_hop<<<dim3(nblocks(g.volh), 8), kBlock, 0, st>>>(g, p, gauge, a, b, at, bt, s);
}

// ---------------------------------------------------------------------------
// sigma_mu_nu planes.  w buffer: [6 planes][9 = cb*3+ca][stride] double2,
// plane order 12,13,14,23,24,34 (clover_d.F90:64-71)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_clover_bsa(Geom g, double2* w, const double2* bf, const double2* af) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.volh) return;
  SpinorView<Prec::F64> A{(double2*)af, g.stride}, B{(double2*)bf, g.stride};
  Spinor<double> a, b;
  A.load(i, a);
  B.load(i, b);
#pragma unroll
  for (int pl = 0; pl < 6; pl++) {
#pragma unroll
    for (int ca = 0; ca < 3; ca++) {
      C64 q1 = a.c[0][ca], q2 = a.c[1][ca], q3 = a.c[2][ca], q4 = a.c[3][ca];
      C64 g1, g2, g3, g4;
      switch (pl) {  // clover_bsa.F90:40-176
        case 0: g1 = -q1; g2 = q2; g3 = -q3; g4 = q4; break;
        case 1: g1 = -itimes(q2); g2 = itimes(q1); g3 = -itimes(q4); g4 = itimes(q3); break;
        case 2: g1 = q4; g2 = q3; g3 = q2; g4 = q1; break;
        case 3: g1 = -q2; g2 = -q1; g3 = -q4; g4 = -q3; break;
        case 4: g1 = -itimes(q4); g2 = itimes(q3); g3 = -itimes(q2); g4 = itimes(q1); break;
        default: g1 = q3; g2 = -q4; g3 = q1; g4 = -q2;
      }
#pragma unroll
      for (int cb = 0; cb < 3; cb++) {
        C64 t = mulc(g1, b.c[0][cb]) + mulc(g2, b.c[1][cb]) + mulc(g3, b.c[2][cb]) + mulc(g4, b.c[3][cb]);
        w[(pl * 9 + cb * 3 + ca) * g.stride + i] = make_double2(t.x, t.y);
      }
    }
  }
}

void launch_clover_bsa(const Geom& g, double2* w, const double2* b, const double2* a, cudaStream_t st) {
  k_clover_bsa<<<nblocks(g.volh), kBlock, 0, st>>>(g, w, b, a);
}

// element (k1,k2) of the full Hermitian 6x6 block from the packed slots
__device__ __forceinline__ C64 block_el(const C64 a[18], int r, int c) {
  const int slot_up[6][6] = {{-1, 1, 2, 3, 4, 5},    {-1, -1, 6, 7, 8, 9},    {-1, -1, -1, 11, 12, 13},
                             {-1, -1, -1, -1, 14, 15}, {-1, -1, -1, -1, -1, 17}, {-1, -1, -1, -1, -1, -1}};
  if (r == c) {
    const int ds[6] = {0, 0, 10, 10, 16, 16};
    return mkc((r & 1) ? a[ds[r]].y : a[ds[r]].x, 0.0);
  }
  if (r < c) return a[slot_up[r][c]];
  return conjg(a[slot_up[c][r]]);
}

// clover_t_init.F90 + clover_ts.F90: T = (halved) A^-1 in the Dirac basis,
// w planes = Tr_spin(T sigma_mu_nu).  T(s1,c1,s2,c2) = I1 +- I2 with the sign
// + when s1, s2 are both upper or both lower spins.
__global__ void __launch_bounds__(kBlock) k_clover_ts(Geom g, double2* w, const double2* ainv) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.volh) return;
  C64 I1[18], I2[18];
  CloverView<Prec::F64> A{(double2*)ainv, g.stride};
  A.load_block(i, 0, I1);
  A.load_block(i, 1, I2);
  for (int c1 = 0; c1 < 3; c1++)
    for (int c2 = 0; c2 < 3; c2++) {
      // T(s1,s2) for this colour pair
      C64 T[4][4];
#pragma unroll
      for (int s1 = 0; s1 < 4; s1++)
#pragma unroll
        for (int s2 = 0; s2 < 4; s2++) {
          int k1 = (s1 & 1) * 3 + c1, k2 = (s2 & 1) * 3 + c2;
          C64 e1 = block_el(I1, k1, k2), e2 = block_el(I2, k1, k2);
          T[s1][s2] = ((s1 < 2) == (s2 < 2)) ? e1 + e2 : e1 - e2;
        }
      C64 r[6];
      r[0] = -T[0][0] + T[1][1] - T[2][2] + T[3][3];
      r[1] = itimes(T[0][1]) - itimes(T[1][0]) + itimes(T[2][3]) - itimes(T[3][2]);
      r[2] = T[0][3] + T[1][2] + T[2][1] + T[3][0];
      r[3] = -T[0][1] - T[1][0] - T[2][3] - T[3][2];
      r[4] = itimes(T[0][3]) - itimes(T[1][2]) + itimes(T[2][1]) - itimes(T[3][0]);
      r[5] = T[0][2] - T[1][3] + T[2][0] - T[3][1];
#pragma unroll
      for (int pl = 0; pl < 6; pl++) w[(pl * 9 + c2 * 3 + c1) * g.stride + i] = make_double2(r[pl].x, r[pl].y);
    }
}

void launch_clover_ts(const Geom& g, double2* w, const double2* ainv, cudaStream_t st) {
  k_clover_ts<<<nblocks(g.volh), kBlock, 0, st>>>(g, w, ainv);
}

// ---------------------------------------------------------------------------
// clover_d (clover_d.F90:110-264)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void load_w(const Geom& g, const double2* w, int pl, int site, L64& m) {
#pragma unroll
  for (int cb = 0; cb < 3; cb++)
#pragma unroll
    for (int ca = 0; ca < 3; ca++) {
      double2 t = __ldg(w + (pl * 9 + cb * 3 + ca) * g.stride + site);
      m.m[ca][cb] = mkc(t.x, t.y);
    }
}

// clover_d_same_eo (clover_d.F90:203-231)
__device__ void d_same_eo(double q[8], double s, const L64& u0, const L64& u1, const L64& u2, const L64& u3,
                          const L64& u4, const L64& u5, const L64& u6, const L64& wa, const L64& wb,
                          const L64& wc) {
  L64 u, v, r;
  mul2(u, u0, false, u1, false);
  mul2(v, u3, false, u2, false);
  mul3(r, u, false, v, true, wa, false); re_tr_j(q, r, s);
  mul3(r, wa, false, v, false, u, true); re_tr_j(q, r, s);
  mul3(r, u, false, wb, false, v, true); re_tr_j(q, r, s);
  mul3(r, v, false, wb, false, u, true); re_tr_j(q, r, s);
  mul2(u, u0, false, u6, true);
  mul2(v, u4, true, u5, false);
  mul3(r, wa, false, v, false, u, true); re_tr_j(q, r, -s);
  mul3(r, u, false, v, true, wa, false); re_tr_j(q, r, -s);
  mul3(r, v, false, wc, false, u, true); re_tr_j(q, r, -s);
  mul3(r, u, false, wc, false, v, true); re_tr_j(q, r, -s);
}

// clover_d_diff_eo (clover_d.F90:233-264); uuu_fwd(a,b,c) = a b^+ c^+,
// uuu_bwd(a,b,c) = a^+ b^+ c (uuu.F90)
__device__ void d_diff_eo(double q[8], double s, const L64& u0, const L64& u1, const L64& u2, const L64& u3,
                          const L64& u4, const L64& u5, const L64& u6, const L64& wd, const L64& we,
                          const L64& wf) {
  L64 u, v, r;
  mul3(u, u1, false, u2, true, u3, true);
  mul3(v, u2, false, u1, true, u0, true);
  mul3(r, u0, false, wd, false, u, false); re_tr_j(q, r, s);
  mul3(r, u, true, wd, false, u0, true); re_tr_j(q, r, s);
  mul3(r, v, true, we, false, u3, true); re_tr_j(q, r, s);
  mul3(r, u3, false, we, false, v, false); re_tr_j(q, r, s);
  mul3(u, u6, true, u5, true, u4, false);
  mul3(v, u0, false, u6, true, u5, true);
  mul3(r, u, true, wd, false, u0, true); re_tr_j(q, r, -s);
  mul3(r, u0, false, wd, false, u, false); re_tr_j(q, r, -s);
  mul3(r, u4, true, wf, false, v, true); re_tr_j(q, r, -s);
  mul3(r, v, false, wf, false, u4, false); re_tr_j(q, r, -s);
}

__global__ void __launch_bounds__(kBlock) k_clover_d(Geom g, double* p, const double2* gauge, const double2* w,
                                                     int eo_w, double s) {
  const int PMU[6] = {0, 0, 0, 1, 1, 2}, PNU[6] = {1, 2, 3, 2, 3, 3};
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int me = blockIdx.y;
  if (i >= g.volh) return;
  int mu = me >> 1, e = me & 1;
  Site st = site_coords(g, i, e);
  double* pp = p + ((size_t)me * g.volh + i) * 8;
  double acc[8];
#pragma unroll
  for (int k = 0; k < 8; k++) acc[k] = pp[k];
  const bool same = (e == eo_w);
  for (int pl = 0; pl < 6; pl++) {
    int nu;
    double sl;
    if (PMU[pl] == mu) { nu = PNU[pl]; sl = s; }
    else if (PNU[pl] == mu) { nu = PMU[pl]; sl = -s; }
    else continue;
    // sites of clover_d_loop (clover_d.F90:175-181)
    int xa[4], xd[4], xe[4], xf[4], xb[4], xc[4];
#pragma unroll
    for (int k = 0; k < 4; k++) xa[k] = st.x[k];
    shift(g, xa, mu, 1, xd);
    shift(g, xa, nu, 1, xe);
    shift(g, xa, nu, -1, xf);
    shift(g, xd, nu, 1, xb);
    shift(g, xd, nu, -1, xc);
    L64 u0, u1, u2, u3, u4, u5, u6;
    load_link(g, gauge, mu, xa, u0);
    load_link(g, gauge, nu, xd, u1);
    load_link(g, gauge, mu, xe, u2);
    load_link(g, gauge, nu, xa, u3);
    load_link(g, gauge, nu, xf, u4);
    load_link(g, gauge, mu, xf, u5);
    load_link(g, gauge, nu, xc, u6);
    double q[8];
#pragma unroll
    for (int k = 0; k < 8; k++) q[k] = 0.0;
    L64 w1, w2, w3;
    if (same) {
      load_w(g, w, pl, i, w1);
      load_w(g, w, pl, site_index(g, xb), w2);
      load_w(g, w, pl, site_index(g, xc), w3);
      d_same_eo(q, sl, u0, u1, u2, u3, u4, u5, u6, w1, w2, w3);
    } else {
      load_w(g, w, pl, site_index(g, xd), w1);
      load_w(g, w, pl, site_index(g, xe), w2);
      load_w(g, w, pl, site_index(g, xf), w3);
      d_diff_eo(q, sl, u0, u1, u2, u3, u4, u5, u6, w1, w2, w3);
    }
#pragma unroll
    for (int k = 0; k < 8; k++) acc[k] += q[k];
  }
#pragma unroll
  for (int k = 0; k < 8; k++) pp[k] = acc[k];
}

void launch_clover_d(const Geom& g, double* p, const double2* gauge, const double2* w, int eo_w, double s,
                     cudaStream_t st) {
  k_clover_d<<<dim3(nblocks(g.volh), 8), kBlock, 0, st>>>(g, p, gauge, w, eo_w, s);
}

}  // namespace bqcdg
