// hmc.cu -- the device pieces of the HMC around the fermion path, so that the
// links U and the momenta p stay in HBM for a whole trajectory:
//   * the gauge update U <- exp(i step p) U (hmc_u.F90:28-69, gen2u of
//     su3.F90:28-193, u_normalize of su3.F90:313-365);
//   * the gauge force (dsg.F90:28-53 with the staples of staple.F90:28-63);
//   * momentum bookkeeping: the Gaussian draw of hmc_init_p.F90:28-45, the
//     kinetic term of action.F90 (sp) and the force monitor of
//     hmc_forces.F90:65-104 (|p_old - p|^2);
//   * the complex BLAS of the MRE initial guess (mre.F90:68-213) on resident
//     spinor fields: <a,b>, y += a x, x *= s.
// Momenta use BQCD's GENERATOR_FIELD layout, real(8, volh, 0:1, 4): entry
// ((mu*2 + eo)*volh + i)*8 + j.
#include "kernels.cuh"
#include "su3.cuh"

namespace bqcdg {

// ---------------------------------------------------------------------------
// u = exp(i sum_j h_j lambda_j) (su3.F90:28-193).  The closed form of the
// reference: the eigenvalues l1, l2, l3 of the Hermitian H = h.lambda from
// the invariants q = Tr H^2 and p = Tr H^3 (trigonometric solution of the
// cubic); H = hs + hk with hk a multiple of the unit matrix plus the part
// along the eigenvalue l3, and exp(iH) = exp(i hs) exp(i hk), each from a
// second-order polynomial in its argument.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void h2_of(const double h[8], double h2[8]) {
  const double sqrt33 = 0.57735026918962576451;  // sqrt(3)/3
  const double a8 = h[7] * sqrt33;
  const double a12 = h[0] * h[0] + h[1] * h[1];
  const double a45 = h[3] * h[3] + h[4] * h[4];
  const double a67 = h[5] * h[5] + h[6] * h[6];
  h2[0] = 2 * h[0] * a8 + h[3] * h[5] + h[4] * h[6];
  h2[1] = 2 * h[1] * a8 + h[4] * h[5] - h[3] * h[6];
  h2[2] = 2 * h[2] * a8 + 0.5 * (a45 - a67);
  h2[3] = h[3] * (h[2] - a8) + h[0] * h[5] - h[1] * h[6];
  h2[4] = h[4] * (h[2] - a8) + h[0] * h[6] + h[1] * h[5];
  h2[5] = h[5] * (-h[2] - a8) + h[0] * h[3] + h[1] * h[4];
  h2[6] = h[6] * (-h[2] - a8) + h[0] * h[4] - h[1] * h[3];
  h2[7] = (h[2] * h[2] - h[7] * h[7] + a12 - 0.5 * (a45 + a67)) * sqrt33;
}

__device__ __forceinline__ C64 cdiv(C64 a, C64 b) {
  const double d = b.x * b.x + b.y * b.y;
  return mkc((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}

__device__ void gen2u_dev(const double h[8], L64& u) {
  const double eps = 1e-8;
  const double pi = 3.14159265358979323846;
  const double sqrt33 = 0.57735026918962576451;
  const double twosqrt33 = 2.0 * sqrt33;
  double h2[8], hs[8], hk[8], hs2[8];
  h2_of(h, h2);
  double q = 0.0, p = 0.0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    q += h[i] * h[i];
    p += h[i] * h2[i];
  }
  q = 2.0 * q;
  p = 2.0 * p / 3.0;
  const double a = sqrt(2.0 * q / 3.0);
  const double alpha = acos(4.0 * p / (a * a * a)) / 3.0;
  double l1, l2;
  if (alpha <= pi / 6) {
    l1 = a * cos(alpha);
    l2 = a * cos(alpha + 2 * pi / 3);
  } else {
    l2 = a * cos(alpha);
    l1 = a * cos(alpha + 2 * pi / 3);
  }
  const double l3 = -l1 - l2;
  const double l12 = l1 * l2;
  const double s = -l1 - 2 * l2;
  const double aux0 = (2.0 * l3 * l3 + l12) * (l1 - l2);
  const double c = s * (l3 * l3 + 2.0 * l12) / aux0;
  const double d = -3.0 * s * l3 / aux0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    hs[i] = c * h[i] + d * h2[i];
    hk[i] = h[i] - hs[i];
  }
  h2_of(hs, hs2);
  double cs1, cs2;
  if (fabs(s) > eps) {
    cs1 = sin(s) / s;
    cs2 = (cos(s) - 1) / (s * s);
  } else {
    cs1 = 1;
    cs2 = -0.5;
  }
  const C64 ck1 = mkc(cos(l3), sin(l3));
  const C64 ck2 = cdiv(mkc(1.0, 0.0), ck1 * ck1);
  const C64 ck3 = (1.0 / 3.0) * (ck2 + 2.0 * ck1);
  const C64 ck4 = fabs(l3) > eps ? cdiv(ck1 - ck2, mkc(3 * l3, 0.0)) : mkc(0.0, 3.0);
  double aux = 0.0;
#pragma unroll
  for (int i = 0; i < 8; i++) aux += hs[i] * hs[i];
  aux = 2.0 * aux;
  L64 ms, mk;
  const double dg = 1.0 + cs2 * aux / 3.0;
  ms.m[0][0] = mkc(dg + cs2 * (hs2[2] + sqrt33 * hs2[7]), cs1 * (hs[2] + sqrt33 * hs[7]));
  ms.m[1][1] = mkc(dg + cs2 * (-hs2[2] + sqrt33 * hs2[7]), cs1 * (-hs[2] + sqrt33 * hs[7]));
  ms.m[2][2] = mkc(dg - cs2 * twosqrt33 * hs2[7], -cs1 * twosqrt33 * hs[7]);
  ms.m[0][1] = mkc(cs2 * hs2[0] + cs1 * hs[1], cs1 * hs[0] - cs2 * hs2[1]);
  ms.m[1][0] = mkc(cs2 * hs2[0] - cs1 * hs[1], cs1 * hs[0] + cs2 * hs2[1]);
  ms.m[0][2] = mkc(cs2 * hs2[3] + cs1 * hs[4], cs1 * hs[3] - cs2 * hs2[4]);
  ms.m[2][0] = mkc(cs2 * hs2[3] - cs1 * hs[4], cs1 * hs[3] + cs2 * hs2[4]);
  ms.m[1][2] = mkc(cs2 * hs2[5] + cs1 * hs[6], cs1 * hs[5] - cs2 * hs2[6]);
  ms.m[2][1] = mkc(cs2 * hs2[5] - cs1 * hs[6], cs1 * hs[5] + cs2 * hs2[6]);
  mk.m[0][0] = ck3 + (hk[2] + sqrt33 * hk[7]) * ck4;
  mk.m[1][1] = ck3 + (-hk[2] + sqrt33 * hk[7]) * ck4;
  mk.m[2][2] = ck3 - (twosqrt33 * hk[7]) * ck4;
  mk.m[0][1] = ck4 * mkc(hk[0], -hk[1]);
  mk.m[1][0] = ck4 * mkc(hk[0], hk[1]);
  mk.m[0][2] = ck4 * mkc(hk[3], -hk[4]);
  mk.m[2][0] = ck4 * mkc(hk[3], hk[4]);
  mk.m[1][2] = ck4 * mkc(hk[5], -hk[6]);
  mk.m[2][1] = ck4 * mkc(hk[5], hk[6]);
  mul2(u, ms, false, mk, false);
}

// su3.F90:313-365: Gram-Schmidt on the first two columns, third rebuilt
__device__ __forceinline__ void u_normalize_dev(L64& m) {
  double len = sqrt(norm2(m.m[0][0]) + norm2(m.m[1][0]) + norm2(m.m[2][0]));
#pragma unroll
  for (int r = 0; r < 3; r++) m.m[r][0] = mkc(m.m[r][0].x / len, m.m[r][0].y / len);
  const C64 f = mulc(m.m[0][1], m.m[0][0]) + mulc(m.m[1][1], m.m[1][0]) + mulc(m.m[2][1], m.m[2][0]);
#pragma unroll
  for (int r = 0; r < 3; r++) m.m[r][1] = m.m[r][1] - f * m.m[r][0];
  len = sqrt(norm2(m.m[0][1]) + norm2(m.m[1][1]) + norm2(m.m[2][1]));
#pragma unroll
  for (int r = 0; r < 3; r++) m.m[r][1] = mkc(m.m[r][1].x / len, m.m[r][1].y / len);
  m.m[0][2] = conjg(m.m[1][0] * m.m[2][1] - m.m[2][0] * m.m[1][1]);
  m.m[1][2] = conjg(m.m[2][0] * m.m[0][1] - m.m[0][0] * m.m[2][1]);
  m.m[2][2] = conjg(m.m[0][0] * m.m[1][1] - m.m[1][0] * m.m[0][1]);
}

// momenta of link (mu, eo, i): 8 consecutive doubles
__device__ __forceinline__ double* mom_of(double* p, const Geom& g, int me, int i) {
  return p + ((size_t)me * g.volh + i) * 8;
}

// hmc_u.F90:53-67 on every link: U <- gen2u(step p) U, then u_normalize
__global__ void __launch_bounds__(kBlock) k_hmc_u(Geom g, double2* gauge, const double* p, double step) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int me = blockIdx.y;  // mu * 2 + eo
  if (i >= g.volh) return;
  const double* pp = mom_of((double*)p, g, me, i);
  double q[8];
#pragma unroll
  for (int j = 0; j < 8; j++) q[j] = pp[j] * step;
  L64 v, u, w;
  gen2u_dev(q, v);
  GaugeView<Prec::F64>{gauge, g.stride}.load(me >> 1, me & 1, i, u);
  mul2(w, v, false, u, false);
  u_normalize_dev(w);
  double2* b = gauge + (size_t)(me * 9) * g.stride + i;
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int r = 0; r < 3; r++) b[(c * 3 + r) * g.stride] = make_double2(w.m[r][c].x, w.m[r][c].y);
}

void launch_hmc_u(const Geom& g, double2* gauge, const double* p, double step, cudaStream_t s) {
  k_hmc_u<<<dim3(nblocks(g.volh), 8), kBlock, 0, s>>>(g, gauge, p, step);
}

// dsg.F90:28-53: p(link) += s Im Tr(lambda_j U S), S the sum of the six
// staples of the link, s = -step beta / 3 (the staple sum reads links only,
// so every link is independent)
__global__ void __launch_bounds__(kBlock) k_dsg(Geom g, const double2* gauge, double* p, double s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int me = blockIdx.y;
  if (i >= g.volh) return;
  const int mu = me >> 1, eo = me & 1;
  const Site st = site_coords(g, i, eo);
  L64 uuu, u, w;
  staple(g, gauge, st.x, mu, uuu);
  GaugeView<Prec::F64>{(double2*)gauge, g.stride}.load(mu, eo, i, u);
  mul2(w, u, false, uuu, false);
  double* pp = mom_of(p, g, me, i);
  double q[8];
#pragma unroll
  for (int j = 0; j < 8; j++) q[j] = pp[j];
  im_tr_j(q, w, s);
#pragma unroll
  for (int j = 0; j < 8; j++) pp[j] = q[j];
}

void launch_dsg(const Geom& g, const double2* gauge, double* p, double s, cudaStream_t st) {
  k_dsg<<<dim3(nblocks(g.volh), 8), kBlock, 0, st>>>(g, gauge, p, s);
}

// sum over all 64 volh momentum entries of (a - b)^2 (b = nullptr: a^2);
// one block covers kBlock sites of one (mu, eo), partials in block order
__global__ void __launch_bounds__(kBlock) k_mom_sumsq(Geom g, const double* a, const double* b, RedScratch red,
                                                      double* out) {
  const int nb = gridDim.x / 8;
  const int me = blockIdx.x / nb, sb = blockIdx.x % nb;
  const int i = sb * blockDim.x + threadIdx.x;
  double acc[1] = {0.0};
  if (i < g.volh) {
    const size_t o = ((size_t)me * g.volh + i) * 8;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const double d = b ? a[o + j] - b[o + j] : a[o + j];
      acc[0] += d * d;
    }
  }
  block_reduce_store<1>(acc, red.partial, red.maxblocks, blockIdx.x);
  if (last_block(red.counter, gridDim.x)) {
    double tot[1];
    final_sum<1>(red.partial, red.maxblocks, gridDim.x, tot);
    if (threadIdx.x == 0) {
      *out = tot[0];
      *red.counter = 0;
    }
  }
}

void launch_mom_sumsq(const Geom& g, const double* a, const double* b, RedScratch red, double* out, cudaStream_t s) {
  k_mom_sumsq<<<8 * nblocks(g.volh), kBlock, 0, s>>>(g, a, b, red, out);
}

// ---------------------------------------------------------------------------
// complex BLAS on F64 spinor fields (12 complex per site)
// ---------------------------------------------------------------------------
// out[0] + i out[1] = <a, b> = sum conj(a) b
__global__ void __launch_bounds__(kBlock) k_cdot(Geom g, const double2* a, const double2* b, RedScratch red,
                                                 double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[2] = {0.0, 0.0};
  if (i < g.volh) {
#pragma unroll
    for (int k = 0; k < 12; k++) {
      const double2 x = a[k * g.stride + i], y = b[k * g.stride + i];
      acc[0] += x.x * y.x + x.y * y.y;
      acc[1] += x.x * y.y - x.y * y.x;
    }
  }
  block_reduce_store<2>(acc, red.partial, red.maxblocks, blockIdx.x);
  if (last_block(red.counter, gridDim.x)) {
    double tot[2];
    final_sum<2>(red.partial, red.maxblocks, gridDim.x, tot);
    if (threadIdx.x == 0) {
      out[0] = tot[0];
      out[1] = tot[1];
      *red.counter = 0;
    }
  }
}

void launch_cdot(const Geom& g, const double2* a, const double2* b, RedScratch red, double* out, cudaStream_t s) {
  k_cdot<<<nblocks(g.volh), kBlock, 0, s>>>(g, a, b, red, out);
}

// out[2j] + i out[2j+1] = <a_j, b_j> for j < NB, in one pass: each product
// and each sum is k_cdot's, in k_cdot's order (the per-value block
// reduction does not depend on NB), so every result equals k_cdot's bit for
// bit.  MRE (mre.F90:68-213) needs up to nvec(nvec+1)/2 of them at a time.
template <int NB>
__global__ void __launch_bounds__(kBlock) k_cdot_pairs(Geom g, FieldPairs fp, RedScratch red, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[2 * NB];
#pragma unroll
  for (int j = 0; j < 2 * NB; j++) acc[j] = 0.0;
  if (i < g.volh) {
#pragma unroll
    for (int k = 0; k < 12; k++) {
#pragma unroll
      for (int j = 0; j < NB; j++) {
        const double2 x = fp.a[j][k * g.stride + i], y = fp.b[j][k * g.stride + i];
        acc[2 * j] += x.x * y.x + x.y * y.y;
        acc[2 * j + 1] += x.x * y.y - x.y * y.x;
      }
    }
  }
  block_reduce_store<2 * NB>(acc, red.partial, red.maxblocks, blockIdx.x);
  if (last_block(red.counter, gridDim.x)) {
    double tot[2 * NB];
    final_sum<2 * NB>(red.partial, red.maxblocks, gridDim.x, tot);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int j = 0; j < 2 * NB; j++) out[j] = tot[j];
      *red.counter = 0;
    }
  }
}

void launch_cdot_pairs(const Geom& g, const FieldPairs& fp, int n, RedScratch red, double* out, cudaStream_t s) {
  const int nb = nblocks(g.volh);
  switch (n) {
    case 1: k_cdot_pairs<1><<<nb, kBlock, 0, s>>>(g, fp, red, out); break;
    case 2: k_cdot_pairs<2><<<nb, kBlock, 0, s>>>(g, fp, red, out); break;
    case 3: k_cdot_pairs<3><<<nb, kBlock, 0, s>>>(g, fp, red, out); break;
    case 4: k_cdot_pairs<4><<<nb, kBlock, 0, s>>>(g, fp, red, out); break;
    case 5: k_cdot_pairs<5><<<nb, kBlock, 0, s>>>(g, fp, red, out); break;
    case 6: k_cdot_pairs<6><<<nb, kBlock, 0, s>>>(g, fp, red, out); break;
    case 7: k_cdot_pairs<7><<<nb, kBlock, 0, s>>>(g, fp, red, out); break;
    default: k_cdot_pairs<8><<<nb, kBlock, 0, s>>>(g, fp, red, out); break;
  }
}

// y = ay y + a x with complex a (ay real: 1 for an axpy, 0 to overwrite y)
__global__ void __launch_bounds__(kBlock) k_caxpby(Geom g, double are, double aim, const double2* x, double ay,
                                                   double2* y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.volh) return;
#pragma unroll
  for (int k = 0; k < 12; k++) {
    const double2 xv = x[k * g.stride + i];
    double2 yv = ay != 0.0 ? y[k * g.stride + i] : make_double2(0.0, 0.0);
    yv.x = ay * yv.x + (are * xv.x - aim * xv.y);
    yv.y = ay * yv.y + (are * xv.y + aim * xv.x);
    y[k * g.stride + i] = yv;
  }
}

void launch_caxpby(const Geom& g, double are, double aim, const double2* x, double ay, double2* y, cudaStream_t s) {
  k_caxpby<<<nblocks(g.volh), kBlock, 0, s>>>(g, are, aim, x, ay, y);
}

}  // namespace bqcdg
