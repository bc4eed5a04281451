// gauge_gen.cu -- seeded synthetic inputs built on the device, with BQCD's own
// generators:
//   ranf.F90:25-121      48-bit LCG; each thread jumps straight to its draw
//                        with the O(log n) skip-ahead of ranset
//   ran.F90:28-110       ran_gauss_volh: Box-Muller, draws in site order
//   conf.F90:201-217     conf_hot = Gaussian 3x3 + u_normalize (su3.F90:313-365)
//   cooling.F90:131-193  conf_relax: Cabibbo-Marinari cooling, 3 SU(2) subgroups
//   action.F90:70-123    sg = 6V - sum Re Tr(plaquette)/3
// Draw number n (1-based) of a stream at state s is (s * m^n mod 2^48) / 2^48,
// so the device values equal the reference's sequential ones (up to the last
// bit of log/cos/sin).
#include "kernels.cuh"
#include "su3.cuh"

namespace bqcdg {

__constant__ unsigned long long c_mpow[48];  // m^(2^k) mod 2^48

__host__ __device__ __forceinline__ unsigned long long mul48(unsigned long long a, unsigned long long b) {
  const unsigned long long M24 = 16777215ull, M48 = 281474976710655ull;
  unsigned long long ah = (a >> 24) & M24, al = a & M24, bh = (b >> 24) & M24, bl = b & M24;
  return (al * bl + ((al * bh + ah * bl) << 24)) & M48;
}

void ranf_powers(unsigned long long* pw) {
  unsigned long long m = 2651554ull * 16777216ull + 15184245ull;  // mH * 2^24 + mL
  for (int k = 0; k < 48; k++) {
    pw[k] = m;
    m = mul48(m, m);
  }
}

unsigned long long ranf_skip(unsigned long long seed, unsigned long long n) {
  unsigned long long pw[48];
  ranf_powers(pw);
  n &= 281474976710655ull;
  for (int k = 0; k < 48 && n; k++, n >>= 1)
    if (n & 1ull) seed = mul48(seed, pw[k]);
  return seed;
}

__device__ __forceinline__ unsigned long long dev_skip(unsigned long long seed, unsigned long long n) {
#pragma unroll 1
  for (int k = 0; k < 48 && n; k++, n >>= 1)
    if (n & 1ull) seed = mul48(seed, c_mpow[k]);
  return seed;
}

// out[(i*m + j)] complex, i < volh, j < m  (ran(j, i) of ran_gauss_volh)
__global__ void k_ran_gauss(double2* out, int volh, int m, double var, unsigned long long s0) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)volh * m) return;
  unsigned long long n1 = 2ull * (unsigned long long)e + 1ull;
  unsigned long long s1 = dev_skip(s0, n1);
  unsigned long long s2 = mul48(s1, c_mpow[0]);
  double u1 = ldexp((double)s1, -48), u2 = ldexp((double)s2, -48);
  double r = sqrt(-2.0 * var * log(u1));
  double phi = 6.2831853071795862 * u2;
  double sn, cs;
  sincos(phi, &sn, &cs);
  out[e] = make_double2(r * cs, r * sn);
}

void launch_ran_gauss(double2* out, int volh, int m, double var, unsigned long long s0, cudaStream_t s) {
  static bool init = false;
  if (!init) {
    unsigned long long pw[48];
    ranf_powers(pw);
    cudaMemcpyToSymbol(c_mpow, pw, sizeof(pw));
    init = true;
  }
  long long n = (long long)volh * m;
  k_ran_gauss<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(out, volh, m, var, s0);
}

// u_normalize (su3.F90:313-365) on Fortran-layout links (9 complex each)
__global__ void k_u_normalize(double2* u, long long nlinks) {
  long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= nlinks) return;
  double2* p = u + l * 9;
  C64 m[3][3];
  for (int c = 0; c < 3; c++)
    for (int r = 0; r < 3; r++) m[r][c] = mkc(p[c * 3 + r].x, p[c * 3 + r].y);
  double len = norm2(m[0][0]) + norm2(m[1][0]) + norm2(m[2][0]);
  len = sqrt(len);
  for (int r = 0; r < 3; r++) m[r][0] = mkc(m[r][0].x / len, m[r][0].y / len);
  C64 f = mulc(m[0][1], m[0][0]) + mulc(m[1][1], m[1][0]) + mulc(m[2][1], m[2][0]);
  for (int r = 0; r < 3; r++) m[r][1] = m[r][1] - f * m[r][0];
  len = sqrt(norm2(m[0][1]) + norm2(m[1][1]) + norm2(m[2][1]));
  for (int r = 0; r < 3; r++) m[r][1] = mkc(m[r][1].x / len, m[r][1].y / len);
  m[0][2] = conjg(m[1][0] * m[2][1] - m[2][0] * m[1][1]);
  m[1][2] = conjg(m[2][0] * m[0][1] - m[0][0] * m[2][1]);
  m[2][2] = conjg(m[0][0] * m[1][1] - m[1][0] * m[0][1]);
  for (int c = 0; c < 3; c++)
    for (int r = 0; r < 3; r++) p[c * 3 + r] = make_double2(m[r][c].x, m[r][c].y);
}

void launch_u_normalize(double2* u, long long nlinks, cudaStream_t s) {
  k_u_normalize<<<(unsigned)((nlinks + 127) / 128), 128, 0, s>>>(u, nlinks);
}

// ---------------------------------------------------------------------------
// staples and cooling
// ---------------------------------------------------------------------------
__device__ __forceinline__ void store_link(const Geom& g, double2* gauge, int mu, int eo, int i, const L64& u) {
  double2* b = gauge + (size_t)((mu * 2 + eo) * 9) * g.stride + i;
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int r = 0; r < 3; r++) b[(c * 3 + r) * g.stride] = make_double2(u.m[r][c].x, u.m[r][c].y);
}

__global__ void __launch_bounds__(128) k_conf_relax(Geom g, double2* gauge, int mu, int eo) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.volh) return;
  Site st = site_coords(g, i, eo);
  L64 uuu, u, w;
  staple(g, gauge, st.x, mu, uuu);
  GaugeView<Prec::F64>{gauge, g.stride}.load(mu, eo, i, u);
  for (int k = 0; k < 3; k++) {
    int c1 = k == 2 ? 1 : 0, c2 = k == 0 ? 1 : 2;
    mul2(w, u, false, uuu, false);
    double p0 = w.m[c1][c1].x + w.m[c2][c2].x;
    double p1 = -(w.m[c1][c2].y + w.m[c2][c1].y);
    double p2 = -(w.m[c1][c2].x - w.m[c2][c1].x);
    double p3 = -(w.m[c1][c1].y - w.m[c2][c2].y);
    double fac = 1.0 / sqrt(p0 * p0 + p1 * p1 + p2 * p2 + p3 * p3);
    double a0 = fac * p0, a1 = fac * p1, a2 = fac * p2, a3 = fac * p3;
    L64 a, t;
    lzero(a);
    a.m[0][0] = mkc(1.0, 0.0);
    a.m[1][1] = mkc(1.0, 0.0);
    a.m[2][2] = mkc(1.0, 0.0);
    a.m[c1][c1] = mkc(a0, a3);
    a.m[c1][c2] = mkc(a2, a1);
    a.m[c2][c1] = mkc(-a2, a1);
    a.m[c2][c2] = mkc(a0, -a3);
    mul2(t, a, false, u, false);
    u = t;
  }
  store_link(g, gauge, mu, eo, i, u);
}

void launch_conf_relax(const Geom& g, double2* gauge, cudaStream_t s) {
  for (int mu = 0; mu < 4; mu++)
    for (int eo = 0; eo < 2; eo++) k_conf_relax<<<nblocks(g.volh), 128, 0, s>>>(g, gauge, mu, eo);
}

// sum over mu<nu and both parities of Re Tr(U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+)
__global__ void __launch_bounds__(kBlock) k_plaquette(Geom g, const double2* gauge, RedScratch red, double* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int eo = blockIdx.y;
  double acc[1] = {0.0};
  if (i < g.volh) {
    Site st = site_coords(g, i, eo);
    for (int mu = 0; mu < 4; mu++)
      for (int nu = mu + 1; nu < 4; nu++) {
        int x1[4], x2[4];
        shift(g, st.x, mu, 1, x1);
        shift(g, st.x, nu, 1, x2);
        L64 a, b, c, d, t, r;
        load_link(g, gauge, nu, x1, a);
        load_link(g, gauge, mu, x2, b);
        load_link(g, gauge, nu, st.x, c);
        load_link(g, gauge, mu, st.x, d);
        mul2(t, a, false, b, true);
        mul2(r, t, false, c, true);
        for (int p = 0; p < 3; p++)
          for (int q = 0; q < 3; q++) acc[0] += r.m[p][q].x * d.m[q][p].x - r.m[p][q].y * d.m[q][p].y;
      }
  }
  // the grid is 2D: partials indexed by the flattened block id
  __shared__ double red_s[32];
  double v = acc[0];
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  if ((threadIdx.x & 31) == 0) red_s[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red_s[w];
    atomicAdd(out, s);
  }
}

void launch_plaquette(const Geom& g, const double2* gauge, RedScratch red, double* out, cudaStream_t s) {
  cudaMemsetAsync(out, 0, sizeof(double), s);
  k_plaquette<<<dim3(nblocks(g.volh), 2), kBlock, 0, s>>>(g, gauge, red, out);
}

}  // namespace bqcdg

namespace bqcdg {

__global__ void k_cold(double2* u, long long nlinks) {
  long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= nlinks) return;
  for (int k = 0; k < 9; k++) u[l * 9 + k] = make_double2((k % 4 == 0) ? 1.0 : 0.0, 0.0);
}

void launch_cold(double2* u, long long nlinks, cudaStream_t s) {
  k_cold<<<(unsigned)((nlinks + 127) / 128), 128, 0, s>>>(u, nlinks);
}

}  // namespace bqcdg
