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

// element (r, c) of chiral block chi of the packed A^-1 of site i, read from
// memory: with r, c known at compile time the slot is too, so nothing is
// indexed at run time (a block held in an array and indexed by a loop
// counter went to local memory)
__device__ __forceinline__ C64 ainv_el(const double2* ainv, int stride, int i, int chi, int r, int c) {
  const int slot_up[6][6] = {{-1, 1, 2, 3, 4, 5},    {-1, -1, 6, 7, 8, 9},    {-1, -1, -1, 11, 12, 13},
                             {-1, -1, -1, -1, 14, 15}, {-1, -1, -1, -1, -1, 17}, {-1, -1, -1, -1, -1, -1}};
  if (r == c) {
    const int ds[6] = {0, 0, 10, 10, 16, 16};
    const double2 t = __ldg(ainv + (size_t)(chi * 18 + ds[r]) * stride + i);
    return mkc((r & 1) ? t.y : t.x, 0.0);
  }
  const int slot = r < c ? slot_up[r][c] : slot_up[c][r];
  const double2 t = __ldg(ainv + (size_t)(chi * 18 + slot) * stride + i);
  return r < c ? mkc(t.x, t.y) : conjg(mkc(t.x, t.y));
}

// clover_t_init.F90 + clover_ts.F90: T = (halved) A^-1 in the Dirac basis,
// w planes = Tr_spin(T sigma_mu_nu).  T(s1,c1,s2,c2) = I1 +- I2 with the sign
// + when s1, s2 are both upper or both lower spins.
__global__ void __launch_bounds__(kBlock) k_clover_ts(Geom g, double2* w, const double2* ainv) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.volh) return;
#pragma unroll
  for (int c1 = 0; c1 < 3; c1++)
#pragma unroll
    for (int c2 = 0; c2 < 3; c2++) {
      // T(s1,s2) for this colour pair
      C64 T[4][4];
#pragma unroll
      for (int s1 = 0; s1 < 4; s1++)
#pragma unroll
        for (int s2 = 0; s2 < 4; s2++) {
          int k1 = (s1 & 1) * 3 + c1, k2 = (s2 & 1) * 3 + c2;
          C64 e1 = ainv_el(ainv, g.stride, i, 0, k1, k2), e2 = ainv_el(ainv, g.stride, i, 1, k1, k2);
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

// The two loops of clover_d_loop for one link and one plane.  Every link and
// w matrix is loaded where it is used (the matrices are 36 registers each in
// FP64; loaded together they spilled), so at most the two partial products,
// two operands and the result are live.  The products and their order are
// those of clover_d_same_eo / clover_d_diff_eo.

// clover_d_same_eo (clover_d.F90:203-231): u0 = U_mu(a), u1 = U_nu(d),
// u2 = U_mu(e), u3 = U_nu(a), u4 = U_nu(f), u5 = U_mu(f), u6 = U_nu(c);
// wa = w(a), wb = w(b), wc = w(c)
template <typename LINK, typename WLD>
__device__ __forceinline__ void d_same_eo(double q[8], double s, const LINK& link, const WLD& wl) {
  L64 u, v, r, x, y;
  link(0, x); link(1, y); mul2(u, x, false, y, false);  // u0 u1
  link(3, x); link(2, y); mul2(v, x, false, y, false);  // u3 u2
  wl(0, x);                                               // wa
  mul3_rows(r, u, false, v, true, x, false); re_tr_j(q, r, s);
  mul3_rows(r, x, false, v, false, u, true); re_tr_j(q, r, s);
  wl(1, x);                                               // wb
  mul3_rows(r, u, false, x, false, v, true); re_tr_j(q, r, s);
  mul3_rows(r, v, false, x, false, u, true); re_tr_j(q, r, s);
  link(0, x); link(6, y); mul2(u, x, false, y, true);   // u0 u6^+
  link(4, x); link(5, y); mul2(v, x, true, y, false);   // u4^+ u5
  wl(0, x);                                               // wa
  mul3_rows(r, x, false, v, false, u, true); re_tr_j(q, r, -s);
  mul3_rows(r, u, false, v, true, x, false); re_tr_j(q, r, -s);
  wl(2, x);                                               // wc
  mul3_rows(r, v, false, x, false, u, true); re_tr_j(q, r, -s);
  mul3_rows(r, u, false, x, false, v, true); re_tr_j(q, r, -s);
}

// clover_d_diff_eo (clover_d.F90:233-264); uuu_fwd(a,b,c) = a b^+ c^+,
// uuu_bwd(a,b,c) = a^+ b^+ c (uuu.F90); wd = w(d), we = w(e), wf = w(f)
template <typename LINK, typename WLD>
__device__ __forceinline__ void d_diff_eo(double q[8], double s, const LINK& link, const WLD& wl) {
  L64 u, v, r, x, y;
  link(1, x); link(2, y); link(3, r); mul3_rows(u, x, false, y, true, r, true);  // u1 u2^+ u3^+
  link(0, r); mul3_rows(v, y, false, x, true, r, true);                          // u2 u1^+ u0^+
  link(0, x); wl(0, y);                                                          // u0, wd
  mul3_rows(r, x, false, y, false, u, false); re_tr_j(q, r, s);
  mul3_rows(r, u, true, y, false, x, true); re_tr_j(q, r, s);
  link(3, x); wl(1, y);                                                          // u3, we
  mul3_rows(r, v, true, y, false, x, true); re_tr_j(q, r, s);
  mul3_rows(r, x, false, y, false, v, false); re_tr_j(q, r, s);
  link(6, x); link(5, y); link(4, r); mul3_rows(u, x, true, y, true, r, false);  // u6^+ u5^+ u4
  link(0, r); mul3_rows(v, r, false, x, true, y, true);                          // u0 u6^+ u5^+
  link(0, x); wl(0, y);                                                          // u0, wd
  mul3_rows(r, u, true, y, false, x, true); re_tr_j(q, r, -s);
  mul3_rows(r, x, false, y, false, u, false); re_tr_j(q, r, -s);
  link(4, x); wl(2, y);                                                          // u4, wf
  mul3_rows(r, x, true, y, false, v, true); re_tr_j(q, r, -s);
  mul3_rows(r, v, false, y, false, x, false); re_tr_j(q, r, -s);
}

__global__ void __launch_bounds__(kBlock) k_clover_d(Geom g, double* p, const double2* gauge, const double2* w,
                                                     int eo_w, double s) {
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
  // the three planes (mu, nu) of the link, in the order of clover_d.F90:
  // planes 0..5 are (0,1) (0,2) (0,3) (1,2) (1,3) (2,3); s for mu < nu
#pragma unroll 1
  for (int nu = 0; nu < 4; nu++) {
    if (nu == mu) continue;
    const int lo = mu < nu ? mu : nu, hi = mu < nu ? nu : mu;
    const int pl = lo == 0 ? hi - 1 : lo == 1 ? hi + 1 : 5;
    const double sl = mu < nu ? s : -s;
    // the corners of clover_d_loop (clover_d.F90:175-181), as shifts of
    // a = x: d = a + mu, e = a + nu, f = a - nu, b = d + nu, c = d - nu
    auto corner = [&](int k, int y[4]) {  // k: 0 a, 1 d, 2 e, 3 f, 4 b, 5 c
#pragma unroll
      for (int j = 0; j < 4; j++) y[j] = st.x[j];
      if (k == 1 || k == 4 || k == 5) y[mu] = y[mu] + 1 == g.L[mu] ? 0 : y[mu] + 1;
      if (k == 2 || k == 4) y[nu] = y[nu] + 1 == g.L[nu] ? 0 : y[nu] + 1;
      if (k == 3 || k == 5) y[nu] = y[nu] == 0 ? g.L[nu] - 1 : y[nu] - 1;
    };
    // link k of the loop: u0 = U_mu(a), u1 = U_nu(d), u2 = U_mu(e), u3 = U_nu(a),
    // u4 = U_nu(f), u5 = U_mu(f), u6 = U_nu(c)
    auto link = [&](int k, L64& m) {
      int y[4];
      corner(k == 0 || k == 3 ? 0 : k == 1 ? 1 : k == 2 ? 2 : k == 6 ? 5 : 3, y);
      load_link(g, gauge, (k == 0 || k == 2 || k == 5) ? mu : nu, y, m);
    };
    // w at the loop's corners: same parity (a, b, c), other parity (d, e, f)
    auto wl = [&](int k, L64& m) {
      int y[4];
      corner(same ? (k == 0 ? 0 : k == 1 ? 4 : 5) : (k == 0 ? 1 : k == 1 ? 2 : 3), y);
      load_w(g, w, pl, site_index(g, y), m);
    };
    double q[8];
#pragma unroll
    for (int k = 0; k < 8; k++) q[k] = 0.0;
    if (same) d_same_eo(q, sl, link, wl);
    else d_diff_eo(q, sl, link, wl);
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
