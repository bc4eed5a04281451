// su3.cuh -- SU(3) helpers shared by the force and clover-construction kernels
// (su3.F90, uuu.F90, clover/clover_uuu.F90).
#pragma once
#include "bqcdg_internal.cuh"

namespace bqcdg {

using L64 = Link<double>;
using C64 = cx<double>;

__device__ __forceinline__ void lzero(L64& r) {
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) r.m[a][b] = mkc(0.0, 0.0);
}
// element of u, u^+
__device__ __forceinline__ C64 el(const L64& u, int r, int c, bool dag) {
  return dag ? conjg(u.m[c][r]) : u.m[r][c];
}
// r = op(a) op(b)
__device__ __forceinline__ void mul2(L64& r, const L64& a, bool da, const L64& b, bool db) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      C64 t = el(a, i, 0, da) * el(b, 0, j, db);
      t = t + el(a, i, 1, da) * el(b, 1, j, db);
      t = t + el(a, i, 2, da) * el(b, 2, j, db);
      r.m[i][j] = t;
    }
}
// r = op(a) op(b) op(c)
__device__ __forceinline__ void mul3(L64& r, const L64& a, bool da, const L64& b, bool db, const L64& c, bool dc) {
  L64 t;
  mul2(t, a, da, b, db);
  mul2(r, t, false, c, dc);
}
// r = op(a) op(b) op(c), one row of op(a) op(b) at a time: the same
// products and sums as mul3, with a 3-element temporary instead of a matrix
__device__ __forceinline__ void mul3_rows(L64& r, const L64& a, bool da, const L64& b, bool db, const L64& c,
                                          bool dc) {
#pragma unroll
  for (int i = 0; i < 3; i++) {
    C64 t[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      C64 x = el(a, i, 0, da) * el(b, 0, k, db);
      x = x + el(a, i, 1, da) * el(b, 1, k, db);
      t[k] = x + el(a, i, 2, da) * el(b, 2, k, db);
    }
#pragma unroll
    for (int j = 0; j < 3; j++) {
      C64 x = t[0] * el(c, 0, j, dc);
      x = x + t[1] * el(c, 1, j, dc);
      r.m[i][j] = x + t[2] * el(c, 2, j, dc);
    }
  }
}
// su3.F90:196-214: p_j += s Im Tr(lambda_j v)
__device__ __forceinline__ void im_tr_j(double p[8], const L64& v, double s) {
  p[0] += s * (v.m[0][1].y + v.m[1][0].y);
  p[1] += s * (v.m[0][1].x - v.m[1][0].x);
  p[2] += s * (v.m[0][0].y - v.m[1][1].y);
  p[3] += s * (v.m[0][2].y + v.m[2][0].y);
  p[4] += s * (v.m[0][2].x - v.m[2][0].x);
  p[5] += s * (v.m[1][2].y + v.m[2][1].y);
  p[6] += s * (v.m[1][2].x - v.m[2][1].x);
  p[7] += s * (v.m[0][0].y + v.m[1][1].y - 2.0 * v.m[2][2].y) * 0.57735026918962573;
}
// su3.F90:216-233: p_j += s Re Tr(lambda_j v)
__device__ __forceinline__ void re_tr_j(double p[8], const L64& v, double s) {
  p[0] += s * (v.m[0][1].x + v.m[1][0].x);
  p[1] += s * (v.m[1][0].y - v.m[0][1].y);
  p[2] += s * (v.m[0][0].x - v.m[1][1].x);
  p[3] += s * (v.m[0][2].x + v.m[2][0].x);
  p[4] += s * (v.m[2][0].y - v.m[0][2].y);
  p[5] += s * (v.m[1][2].x + v.m[2][1].x);
  p[6] += s * (v.m[2][1].y - v.m[1][2].y);
  p[7] += s * (v.m[0][0].x + v.m[1][1].x - 2.0 * v.m[2][2].x) * 0.57735026918962573;
}

__device__ __forceinline__ int site_index(const Geom& g, const int x[4]) {
  return (x[0] >> 1) + g.Lxh * (x[1] + g.L[1] * (x[2] + g.L[2] * x[3]));
}
// coordinates of x shifted by d (+-1) in direction mu, periodic
__device__ __forceinline__ void shift(const Geom& g, const int x[4], int mu, int d, int y[4]) {
#pragma unroll
  for (int k = 0; k < 4; k++) y[k] = x[k];
  y[mu] += d;
  if (y[mu] < 0) y[mu] += g.L[mu];
  if (y[mu] >= g.L[mu]) y[mu] -= g.L[mu];
}
__device__ __forceinline__ int parity_of(const int x[4]) { return (x[0] + x[1] + x[2] + x[3]) & 1; }

__device__ __forceinline__ void load_link(const Geom& g, const double2* gauge, int mu, const int x[4], L64& u) {
  GaugeView<Prec::F64> U{(double2*)gauge, g.stride};
  U.load(mu, parity_of(x), site_index(g, x), u);
}

// staple.F90:28-63: sum over nu != mu of the forward and backward staples.
// With mu a template parameter every shifted coordinate is a register (a
// run-time mu indexes the coordinate arrays, which puts them in local
// memory); staple() dispatches on a run-time mu, uniform across a launch.
template <int MU>
__device__ __forceinline__ void staple_t(const Geom& g, const double2* gauge, const int x[4], L64& st) {
  lzero(st);
#pragma unroll
  for (int nu = 0; nu < 4; nu++) {
    if (nu == MU) continue;
    int x1[4], x2[4], x3[4], x4[4];
    shift(g, x, MU, 1, x1);
    shift(g, x, nu, 1, x2);
    shift(g, x, nu, -1, x3);
    shift(g, x3, MU, 1, x4);
    L64 a, b, c, t, r;
    // uuu_fwd: U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+
    load_link(g, gauge, nu, x1, a);
    load_link(g, gauge, MU, x2, b);
    load_link(g, gauge, nu, x, c);
    mul2(t, a, false, b, true);
    mul2(r, t, false, c, true);
    for (int p = 0; p < 3; p++)
      for (int q = 0; q < 3; q++) st.m[p][q] = st.m[p][q] + r.m[p][q];
    // uuu_bwd: U_nu(x-nu+mu)^+ U_mu(x-nu)^+ U_nu(x-nu)
    load_link(g, gauge, nu, x4, a);
    load_link(g, gauge, MU, x3, b);
    load_link(g, gauge, nu, x3, c);
    mul2(t, a, true, b, true);
    mul2(r, t, false, c, false);
    for (int p = 0; p < 3; p++)
      for (int q = 0; q < 3; q++) st.m[p][q] = st.m[p][q] + r.m[p][q];
  }
}
__device__ __forceinline__ void staple(const Geom& g, const double2* gauge, const int x[4], int mu, L64& st) {
  switch (mu) {
    case 0: staple_t<0>(g, gauge, x, st); break;
    case 1: staple_t<1>(g, gauge, x, st); break;
    case 2: staple_t<2>(g, gauge, x, st); break;
    default: staple_t<3>(g, gauge, x, st); break;
  }
}

}  // namespace bqcdg
