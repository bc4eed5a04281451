// clover_init.cu -- clover term construction on the device (FP64):
//   clover_f_mu_nu.F90:37-103  four-leaf field strength per plane
//   clover_init.F90:28-190     A = 1 - (c_sw kappa / 8) sigma.F in two chiral 6x6 blocks
//   clover_inv.F90:29-220      LDL^+ factors B, explicit inverse, and the halving
//                              of A, A^-1 and 1/D
// plus clover_action.F90:29-60 (2 sum log prod 1/D).
#include "kernels.cuh"
#include "su3.cuh"

namespace bqcdg {

struct Blk {
  C64 m[6][6];
};

// clover_init1 (clover_init.F90:99-120)
__device__ __forceinline__ void init1(Blk& a, const L64& f) {
#pragma unroll
  for (int r = 0; r < 3; r++) {
    a.m[r][r] = mkc(f.m[r][r].x, 0.0);
    a.m[r + 3][r + 3] = mkc(-f.m[r][r].x, 0.0);
  }
  a.m[0][1] = f.m[0][1]; a.m[0][2] = f.m[0][2]; a.m[1][2] = f.m[1][2];
  a.m[3][4] = -a.m[0][1]; a.m[3][5] = -a.m[0][2]; a.m[4][5] = -a.m[1][2];
}
// clover_init2 (clover_init.F90:122-145)
__device__ __forceinline__ void init2(Blk& a, const L64& f, const L64& gg) {
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) a.m[r][c + 3] = f.m[r][c] + itimes(gg.m[r][c]);
}

__device__ __forceinline__ C64 hel(const Blk& a, int r, int c) { return r <= c ? a.m[r][c] : conjg(a.m[c][r]); }

__device__ __forceinline__ void store_packed(double2* dst, int stride, int i, int chi, const Blk& a, double scale) {
  const int slot_up[6][6] = {{-1, 1, 2, 3, 4, 5},    {-1, -1, 6, 7, 8, 9},    {-1, -1, -1, 11, 12, 13},
                             {-1, -1, -1, -1, 14, 15}, {-1, -1, -1, -1, -1, 17}, {-1, -1, -1, -1, -1, -1}};
  double2* b = dst + chi * 18 * stride + i;
  b[0] = make_double2(scale * a.m[0][0].x, scale * a.m[1][1].x);
  b[10 * stride] = make_double2(scale * a.m[2][2].x, scale * a.m[3][3].x);
  b[16 * stride] = make_double2(scale * a.m[4][4].x, scale * a.m[5][5].x);
  for (int r = 0; r < 6; r++)
    for (int c = r + 1; c < 6; c++)
      b[slot_up[r][c] * stride] = make_double2(scale * a.m[r][c].x, scale * a.m[r][c].y);
}

// clover_inv (clover_inv.F90:29-220) on an unhalved block a; writes the
// halved A, the halved inverse and the B factors (L, halved 1/D), each only
// when its destination is given
__device__ void block_inv(const Blk& a, double2* A, double2* Ainv, double2* B, int stride, int i, int chi) {
  if (A) store_packed(A, stride, i, chi, a, 0.5);
  if (!Ainv && !B) return;
  C64 L[6][6];
  double d[6], dinv[6];
  for (int r = 0; r < 6; r++) {
    C64 tmp[6];
    for (int c = 0; c < r; c++) {
      C64 t = hel(a, r, c);
      for (int k = 0; k < c; k++) t = t - tmp[k] * conjg(L[c][k]);
      tmp[c] = t;
    }
    for (int c = 0; c < r; c++) L[r][c] = dinv[c] * tmp[c];
    double dr = a.m[r][r].x;
    for (int k = 0; k < r; k++) dr = dr - d[k] * norm2(L[r][k]);
    d[r] = dr;
    dinv[r] = 1.0 / dr;
  }
  // B = (L, 1/D / 2)
  if (B) {
    double2* bb = B + chi * 18 * stride + i;
    for (int r = 1; r < 6; r++)
      for (int c = 0; c < r; c++) bb[(r * (r - 1) / 2 + c) * stride] = make_double2(L[r][c].x, L[r][c].y);
    bb[15 * stride] = make_double2(0.5 * dinv[0], 0.5 * dinv[1]);
    bb[16 * stride] = make_double2(0.5 * dinv[2], 0.5 * dinv[3]);
    bb[17 * stride] = make_double2(0.5 * dinv[4], 0.5 * dinv[5]);
  }
  if (!Ainv) return;
  // clover_inv2: columns of A^-1 by unit solves, stored halved (upper part)
  Blk inv;
  for (int col = 0; col < 6; col++) {
    C64 y[6], x[6];
    for (int k = 0; k < 6; k++) y[k] = mkc(k == col ? 1.0 : 0.0, 0.0);
    for (int r = 1; r < 6; r++) {
      C64 s = y[r];
      for (int c = 0; c < r; c++) s = s - L[r][c] * y[c];
      y[r] = s;
    }
    for (int r = 5; r >= 0; r--) {
      C64 s = dinv[r] * y[r];
      for (int c = r + 1; c < 6; c++) s = s - conjg(L[c][r]) * x[c];
      x[r] = s;
    }
    // x = column col of A^-1; row col of the Hermitian inverse is conj(x)
    inv.m[col][col] = mkc(x[col].x, 0.0);
    for (int k = col + 1; k < 6; k++) inv.m[col][k] = conjg(x[k]);
  }
  store_packed(Ainv, stride, i, chi, inv, 0.5);
}

// The clover term in two passes over chunks of sites of one parity, so that
// no thread holds both the six field strengths and a 6x6 block inversion:
// k_clover_fields computes f(mu,nu) of one plane per thread (links loaded
// where they are used, triple products by rows), k_clover_blocks builds one
// chiral block per thread from the six planes and inverts it.  The
// arithmetic of every entry is that of clover_f_mu_nu, init1/init2 and
// block_inv above.

// clover_f_mu_nu for the plane (MU, NU) with the loads of each leaf placed at
// their use; the same products and sums as clover_f_mu_nu
template <int MU, int NU>
__device__ __forceinline__ void clover_f_plane(const Geom& g, const double2* gauge, L64& f, const int xs[4]) {
  L64 t, r, c, d;
  lzero(f);
  {  // uuuu1: u1 u2 u3^+ u4^+
    int xp_[4], x_p[4];
    shift(g, xs, MU, 1, xp_);
    shift(g, xs, NU, 1, x_p);
    load_link(g, gauge, MU, xs, c); load_link(g, gauge, NU, xp_, d); mul2(t, c, false, d, false);
    load_link(g, gauge, MU, x_p, c); load_link(g, gauge, NU, xs, d); mul3_rows(r, t, false, c, true, d, true);
#pragma unroll
    for (int p = 0; p < 3; p++)
#pragma unroll
      for (int q = 0; q < 3; q++) f.m[p][q] = f.m[p][q] + r.m[p][q];
  }
  {  // uuuu2: u1 u2^+ u3^+ u4
    int xm_[4], xmp[4];
    shift(g, xs, MU, -1, xm_);
    shift(g, xm_, NU, 1, xmp);
    load_link(g, gauge, NU, xs, c); load_link(g, gauge, MU, xmp, d); mul2(t, c, false, d, true);
    load_link(g, gauge, NU, xm_, c); load_link(g, gauge, MU, xm_, d); mul3_rows(r, t, false, c, true, d, false);
#pragma unroll
    for (int p = 0; p < 3; p++)
#pragma unroll
      for (int q = 0; q < 3; q++) f.m[p][q] = f.m[p][q] + r.m[p][q];
  }
  {  // uuuu3: u1^+ u2^+ u3 u4
    int xm_[4], xmm[4], x_m[4];
    shift(g, xs, MU, -1, xm_);
    shift(g, xm_, NU, -1, xmm);
    shift(g, xs, NU, -1, x_m);
    load_link(g, gauge, MU, xm_, c); load_link(g, gauge, NU, xmm, d); mul2(t, c, true, d, true);
    load_link(g, gauge, MU, xmm, c); load_link(g, gauge, NU, x_m, d); mul3_rows(r, t, false, c, false, d, false);
#pragma unroll
    for (int p = 0; p < 3; p++)
#pragma unroll
      for (int q = 0; q < 3; q++) f.m[p][q] = f.m[p][q] + r.m[p][q];
  }
  {  // uuuu4: u1^+ u2 u3 u4^+
    int x_m[4], xp_[4], xpm[4];
    shift(g, xs, NU, -1, x_m);
    shift(g, xs, MU, 1, xp_);
    shift(g, xp_, NU, -1, xpm);
    load_link(g, gauge, NU, x_m, c); load_link(g, gauge, MU, x_m, d); mul2(t, c, true, d, false);
    load_link(g, gauge, NU, xpm, c); load_link(g, gauge, MU, xs, d); mul3_rows(r, t, false, c, false, d, true);
#pragma unroll
    for (int p = 0; p < 3; p++)
#pragma unroll
      for (int q = 0; q < 3; q++) f.m[p][q] = f.m[p][q] + r.m[p][q];
  }
  // clover_f_mu_nu.F90:92-102
  C64 f10 = f.m[1][0], f20 = f.m[2][0], f21 = f.m[2][1];
  f.m[0][0] = mkc(2.0 * f.m[0][0].y, 0.0);
  f.m[1][1] = mkc(2.0 * f.m[1][1].y, 0.0);
  f.m[2][2] = mkc(2.0 * f.m[2][2].y, 0.0);
  f.m[0][1] = itimes(conjg(f10) - f.m[0][1]);
  f.m[0][2] = itimes(conjg(f20) - f.m[0][2]);
  f.m[1][2] = itimes(conjg(f21) - f.m[1][2]);
  f.m[1][0] = conjg(f.m[0][1]);
  f.m[2][0] = conjg(f.m[0][2]);
  f.m[2][1] = conjg(f.m[1][2]);
}

// the planes of clover_init.F90:52-77 in the order used below:
// 0 (1,0) and 1 (2,1), 2 (2,0) build p; 3 (2,3) and 4 (0,3), 5 (3,1) build q
__global__ void __launch_bounds__(64) k_clover_fields(Geom g, const double2* gauge, int eo, int i0, int n,
                                                      double2* tmp) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int pl = blockIdx.y;
  if (k >= n) return;
  const Site st = site_coords(g, i0 + k, eo);
  L64 f;
  switch (pl) {
    case 0: clover_f_plane<1, 0>(g, gauge, f, st.x); break;
    case 1: clover_f_plane<2, 1>(g, gauge, f, st.x); break;
    case 2: clover_f_plane<2, 0>(g, gauge, f, st.x); break;
    case 3: clover_f_plane<2, 3>(g, gauge, f, st.x); break;
    case 4: clover_f_plane<0, 3>(g, gauge, f, st.x); break;
    default: clover_f_plane<3, 1>(g, gauge, f, st.x); break;
  }
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) tmp[(size_t)(pl * 9 + r * 3 + c) * n + k] = make_double2(f.m[r][c].x, f.m[r][c].y);
}

__device__ __forceinline__ void load_plane(const double2* tmp, int n, int k, int pl, L64& f) {
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const double2 v = tmp[(size_t)(pl * 9 + r * 3 + c) * n + k];
      f.m[r][c] = mkc(v.x, v.y);
    }
}

// clover_init3 (a1 = s(p+q)+1, a2 = s(p-q)+1, upper triangle) and
// clover_inv for chiral block chi = blockIdx.y of each site
// tmode: store T = factor (p +- q) itself (no identity, not halved, no inverse)
__global__ void __launch_bounds__(64) k_clover_blocks(Geom g, const double2* tmp, int i0, int n, double factor,
                                                      double2* A, double2* AI, double2* B, int tmode) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int chi = blockIdx.y;
  if (k >= n) return;
  Blk p, q, bl;
  L64 f, f2;
  load_plane(tmp, n, k, 0, f);
  init1(p, f);
  load_plane(tmp, n, k, 1, f);
  load_plane(tmp, n, k, 2, f2);
  init2(p, f, f2);
  load_plane(tmp, n, k, 3, f);
  init1(q, f);
  load_plane(tmp, n, k, 4, f);
  load_plane(tmp, n, k, 5, f2);
  init2(q, f, f2);
  const double sg = chi == 0 ? 1.0 : -1.0;
  for (int r = 0; r < 6; r++)
    for (int c = r; c < 6; c++) bl.m[r][c] = factor * (p.m[r][c] + sg * q.m[r][c]);
  if (tmode) {
    store_packed(A, g.stride, i0 + k, chi, bl, 1.0);
    return;
  }
  for (int r = 0; r < 6; r++) bl.m[r][r] = mkc(bl.m[r][r].x + 1.0, 0.0);
  block_inv(bl, A, AI, B, g.stride, i0 + k, chi);
}

int clover_init_chunk(const Geom& g) { return g.volh < (1 << 20) ? g.volh : (1 << 20); }

void launch_clover_init(const Geom& g, const double2* gauge, double csw_kappa, double2* a[2], double2* ainv[2],
                        double2* b[2], double2* tmp, cudaStream_t s) {
  const int chunk = clover_init_chunk(g);
  for (int eo = 0; eo < 2; eo++) {
    if (!a[eo] && !ainv[eo] && !b[eo]) continue;  // nothing wanted of this parity
    for (int i0 = 0; i0 < g.volh; i0 += chunk) {
      const int n = g.volh - i0 < chunk ? g.volh - i0 : chunk;
      k_clover_fields<<<dim3((n + 63) / 64, 6), 64, 0, s>>>(g, gauge, eo, i0, n, tmp);
      k_clover_blocks<<<dim3((n + 63) / 64, 2), 64, 0, s>>>(g, tmp, i0, n, -csw_kappa / 8.0, a[eo], ainv[eo],
                                                            b[eo], 0);
    }
  }
}

void launch_clover_t(const Geom& g, const double2* gauge, double csw, double2* t[2], double2* tmp, cudaStream_t s) {
  const int chunk = clover_init_chunk(g);
  for (int eo = 0; eo < 2; eo++) {
    if (!t[eo]) continue;
    for (int i0 = 0; i0 < g.volh; i0 += chunk) {
      const int n = g.volh - i0 < chunk ? g.volh - i0 : chunk;
      k_clover_fields<<<dim3((n + 63) / 64, 6), 64, 0, s>>>(g, gauge, eo, i0, n, tmp);
      k_clover_blocks<<<dim3((n + 63) / 64, 2), 64, 0, s>>>(g, tmp, i0, n, -csw / 8.0, t[eo], nullptr, nullptr, 1);
    }
  }
}

__global__ void __launch_bounds__(kBlock) k_clover_action(Geom g, const double2* b, RedScratch red, double* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[1] = {0.0};
  if (i < g.volh) {
    double d1 = 1.0, d2 = 1.0;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      double2 t1 = b[(15 + k) * g.stride + i], t2 = b[(18 + 15 + k) * g.stride + i];
      d1 *= t1.x * t1.y;
      d2 *= t2.x * t2.y;
    }
    acc[0] = log(d1 * d2);
  }
  block_reduce_store<1>(acc, red.partial, red.maxblocks, blockIdx.x);
  if (last_block(red.counter, gridDim.x)) {
    double tot[1];
    final_sum<1>(red.partial, red.maxblocks, gridDim.x, tot);
    if (threadIdx.x == 0) {
      *out = 2.0 * tot[0];
      *red.counter = 0;
    }
  }
}

void launch_clover_action(const Geom& g, const double2* b, RedScratch red, double* out, cudaStream_t s) {
  k_clover_action<<<nblocks(g.volh), kBlock, 0, s>>>(g, b, red, out);
}

}  // namespace bqcdg
