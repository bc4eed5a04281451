/*
 * bqcd_oracle.c -- CPU restatement (C99 + OpenMP) of the fermion hot path of
 * BQCD benchmark2 svn r399, for TESTS ONLY: parity checker of the CUDA path,
 * reproducer of the reference's golden runs, and timed CPU baseline.
 *
 * Every routine cites the reference file:line it restates.  Loop orders and
 * the order of floating-point accumulation follow the Fortran so that the
 * reference's golden outputs (ranf_test.reference, work/out.quick-test.reference)
 * are reproduced; the only deliberate change is that the libd21 half-spinor
 * projection (d/D21.F90:79-182) is evaluated on the fly at the neighbour
 * instead of through the SC2 buffer -- the arithmetic per element is the same.
 * Reductions use a fixed chunking so results do not depend on thread count.
 *
 * Compile with -fcx-fortran-rules -ffp-contract=off (Fortran complex rules,
 * no FMA contraction), as oracle/build.py does.
 */
#include "bqcd_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PI_R8 3.1415926535897931
#define TWOPI_R8 6.2831853071795862
#define SQRT3_R8 1.7320508075688772

typedef oq_cplx cplx;

static inline cplx mk(double re, double im) { return CMPLX(re, im); }
/* i_times(c) = cmplx(-aimag(c), real(c)) (e.g. d/D21.F90:91) */
static inline cplx itimes(cplx c) { return CMPLX(-cimag(c), creal(c)); }
static inline double sqc(cplx z) { return creal(z) * creal(z) + cimag(z) * cimag(z); }

/* 3x3 matrix element (row r, column c), Fortran column-major SU3 */
#define M3(u, r, c) ((u)[(c) * 3 + (r)])
/* spinor element (spin s, colour c) of site i */
#define SP(f, s, c, i) ((f)[((size_t)(i) * 3 + (c)) * 4 + (s)])
/* gauge link u(:,:,i,eo,mu) */
#define ULINK(g, u, i, eo, mu) ((u) + ((((size_t)(mu) * 2 + (eo)) * (g)->volh + (i)) * 9))
/* generator p(:,i,eo,mu) */
#define PGEN(g, p, i, eo, mu) ((p) + ((((size_t)(mu) * 2 + (eo)) * (g)->volh + (i)) * 8))

static void *xmalloc(size_t n) {
  void *p = malloc(n ? n : 1);
  if (!p) { fprintf(stderr, "oracle: out of memory (%zu bytes)\n", n); abort(); }
  return p;
}
static void *xcalloc(size_t n) {
  void *p = calloc(1, n ? n : 1);
  if (!p) { fprintf(stderr, "oracle: out of memory (%zu bytes)\n", n); abort(); }
  return p;
}

int oq_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

long oq_sc_size(const oq_geom *g) { return 12L * g->volh; }
long oq_gauge_size(const oq_geom *g) { return 72L * g->volh; }
long oq_clover_size(const oq_geom *g) { return 72L * g->volh; }
long oq_gen_size(const oq_geom *g) { return 64L * g->volh; }

/* ------------------------------------------------------------------------ */
/* RNG: 48-bit LCG (ranf.F90:25-121)                                         */
/* ------------------------------------------------------------------------ */
static const uint64_t RANF_MH = 2651554u, RANF_ML = 15184245u;
static const uint64_t RANF_MASK24 = 16777215u, RANF_MASK48 = 281474976710655ull;
static const uint64_t RANF_DEFAULT = 48131768981101ull;
static uint64_t ranf_seed = 48131768981101ull;

/* ranf.F90:44-61: seed = mod(m*seed, 2^48); result = seed * 2^-48 */
double oq_ranf(void) {
  uint64_t sh = (ranf_seed >> 24) & RANF_MASK24;
  uint64_t sl = ranf_seed & RANF_MASK24;
  ranf_seed = (sl * RANF_ML + ((sl * RANF_MH + sh * RANF_ML) << 24)) & RANF_MASK48;
  return ldexp((double)ranf_seed, -48);
}

void oq_ranget(int64_t *seed) { *seed = (int64_t)ranf_seed; }

/* ranf.F90:87-121: set seed (forced odd) and skip n_skip numbers */
void oq_ranset(int64_t seed_in, int64_t n_skip) {
  if (seed_in == 0) ranf_seed = RANF_DEFAULT;
  else ranf_seed = ((uint64_t)seed_in | 1u) & RANF_MASK48;
  uint64_t n = (uint64_t)n_skip & RANF_MASK48;
  uint64_t mmh = RANF_MH, mml = RANF_ML;
  while (n > 0) {
    if (n & 1u) {
      uint64_t sh = (ranf_seed >> 24) & RANF_MASK24;
      uint64_t sl = ranf_seed & RANF_MASK24;
      ranf_seed = (sl * mml + ((sl * mmh + sh * mml) << 24)) & RANF_MASK48;
    }
    uint64_t mm = (mml * mml + ((mmh * mml) << 25)) & RANF_MASK48;
    mmh = (mm >> 24) & RANF_MASK24;
    mml = mm & RANF_MASK24;
    n >>= 1;
  }
}

/* ran.F90:28-110 on a single process: the skips collapse to no-ops and the
 * site order (t, z, y, x/2) is the even/odd index order. */
void oq_ran_gauss_volh(const oq_geom *g, int m, cplx *ran, double var, int eo) {
  (void)eo;
  double twovar = 2.0 * var;
  for (int i = 0; i < g->volh; i++) {
    for (int j = 0; j < m; j++) {
      double r = sqrt(-twovar * log(oq_ranf()));
      double phi = TWOPI_R8 * oq_ranf();
      ran[(size_t)i * m + j] = mk(r * cos(phi), r * sin(phi));
    }
  }
}

/* ------------------------------------------------------------------------ */
/* geometry (index.F90:26-102, init_common.F90:110-205, flip_bc.F90:37-94)   */
/* ------------------------------------------------------------------------ */
int oq_parity(const int x[4]) { return (x[0] + x[1] + x[2] + x[3]) % 2; }

int oq_ieo(const oq_geom *g, const int x[4]) {
  int ilex = x[3];
  for (int d = 2; d >= 0; d--) ilex = ilex * g->L[d] + x[d];
  return ilex / 2;
}

int oq_geom_init(oq_geom *g, const int L[4], const int bc[4]) {
  memset(g, 0, sizeof(*g));
  for (int d = 0; d < 4; d++) {
    if (L[d] <= 0 || L[d] % 2) return -1;   /* init_common.F90:67-72 */
    g->L[d] = L[d];
    g->bc[d] = bc[d];
  }
  g->volume = L[0] * L[1] * L[2] * L[3];
  g->volh = g->volume / 2;
  int volh = g->volh;
  g->nn = xmalloc(sizeof(int) * 16 * (size_t)volh);
  g->coord = xmalloc(sizeof(int) * 8 * (size_t)volh);
  g->flip_list = xmalloc(sizeof(int) * 8 * (size_t)volh);
  int x[4];
  for (x[3] = 0; x[3] < L[3]; x[3]++)
    for (x[2] = 0; x[2] < L[2]; x[2]++)
      for (x[1] = 0; x[1] < L[1]; x[1]++)
        for (x[0] = 0; x[0] < L[0]; x[0]++) {
          int i = oq_ieo(g, x), eo = oq_parity(x);
          for (int d = 0; d < 4; d++) g->coord[((size_t)eo * volh + i) * 4 + d] = x[d];
          for (int fb = 0; fb < 2; fb++)
            for (int mu = 0; mu < 4; mu++) {
              int j[4] = {x[0], x[1], x[2], x[3]};
              j[mu] += fb == OQ_FWD ? 1 : -1;
              if (j[mu] < 0) j[mu] += L[mu];
              if (j[mu] >= L[mu]) j[mu] -= L[mu];
              OQ_NN(g, i, eo, mu, fb) = oq_ieo(g, j);
            }
        }
  /* flip_bc list: the last slice in each direction with bc < 0 */
  for (int mu = 0; mu < 4; mu++) {
    int cnt[2] = {0, 0};
    if (bc[mu] < 0) {
      for (int eo = 0; eo < 2; eo++)
        for (int i = 0; i < volh; i++)
          if (g->coord[((size_t)eo * volh + i) * 4 + mu] == L[mu] - 1)
            g->flip_list[((size_t)mu * 2 + eo) * volh + cnt[eo]++] = i;
      if (cnt[0] != cnt[1]) return -2;
    }
    g->flip_len[mu] = cnt[0];
  }
  return 0;
}

void oq_geom_free(oq_geom *g) {
  free(g->nn);
  free(g->coord);
  free(g->flip_list);
  memset(g, 0, sizeof(*g));
}

/* flip_bc.F90:97-121 */
void oq_flip_bc(const oq_geom *g, cplx *u) {
  for (int mu = 0; mu < 4; mu++)
    for (int eo = 0; eo < 2; eo++)
      for (int k = 0; k < g->flip_len[mu]; k++) {
        int i = g->flip_list[((size_t)mu * 2 + eo) * g->volh + k];
        cplx *l = ULINK(g, u, i, eo, mu);
        for (int e = 0; e < 9; e++) l[e] = -l[e];
      }
}

/* ------------------------------------------------------------------------ */
/* SU(3) algebra (su3.F90, uuu.F90, clover/clover_uuu.F90)                    */
/* ------------------------------------------------------------------------ */
/* su3.F90:419-433 r = a*b */
static void uu(cplx *r, const cplx *a, const cplx *b) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      M3(r, i, j) = M3(a, i, 0) * M3(b, 0, j) + M3(a, i, 1) * M3(b, 1, j) + M3(a, i, 2) * M3(b, 2, j);
}
/* su3.F90:435-449 r = a*b^+ */
static void uud(cplx *r, const cplx *a, const cplx *b) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      M3(r, i, j) = M3(a, i, 0) * conj(M3(b, j, 0)) + M3(a, i, 1) * conj(M3(b, j, 1)) +
                    M3(a, i, 2) * conj(M3(b, j, 2));
}
/* su3.F90:451-465 r = a^+*b */
static void udu(cplx *r, const cplx *a, const cplx *b) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      M3(r, i, j) = conj(M3(a, 0, i)) * M3(b, 0, j) + conj(M3(a, 1, i)) * M3(b, 1, j) +
                    conj(M3(a, 2, i)) * M3(b, 2, j);
}
/* uuu.F90:60-79 r += a b^+ c^+ */
static void uuu_fwd(cplx *r, const cplx *a, const cplx *b, const cplx *c) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      for (int k = 0; k < 3; k++)
        for (int m = 0; m < 3; m++)
          M3(r, i, j) = M3(r, i, j) + M3(a, i, k) * conj(M3(b, m, k)) * conj(M3(c, j, m));
}
/* uuu.F90:28-42 r += a^+ b^+ c */
static void uuu_bwd(cplx *r, const cplx *a, const cplx *b, const cplx *c) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      for (int k = 0; k < 3; k++)
        for (int m = 0; m < 3; m++)
          M3(r, i, j) = M3(r, i, j) + conj(M3(a, k, i)) * conj(M3(b, m, k)) * M3(c, m, j);
}
/* clover_uuu.F90:28-127: three-factor products with optional daggers */
enum { T_N = 0, T_D = 1 };
static inline cplx melt(const cplx *u, int r, int c, int dag) {
  return dag ? conj(M3(u, c, r)) : M3(u, r, c);
}
static void uuu3(cplx *r, const cplx *u, int du, const cplx *v, int dv, const cplx *w, int dw) {
  for (int i = 0; i < 3; i++)
    for (int l = 0; l < 3; l++) {
      cplx s = 0;
      for (int j = 0; j < 3; j++)
        for (int k = 0; k < 3; k++) s = s + melt(u, i, j, du) * melt(v, j, k, dv) * melt(w, k, l, dw);
      M3(r, i, l) = s;
    }
}

/* su3.F90:196-214 p(j) += s Im Tr(lambda_j U) */
void oq_im_tr_j(double *p, const cplx *u, double s) {
  p[0] = p[0] + s * (cimag(M3(u, 0, 1)) + cimag(M3(u, 1, 0)));
  p[1] = p[1] + s * (creal(M3(u, 0, 1)) - creal(M3(u, 1, 0)));
  p[2] = p[2] + s * (cimag(M3(u, 0, 0)) - cimag(M3(u, 1, 1)));
  p[3] = p[3] + s * (cimag(M3(u, 0, 2)) + cimag(M3(u, 2, 0)));
  p[4] = p[4] + s * (creal(M3(u, 0, 2)) - creal(M3(u, 2, 0)));
  p[5] = p[5] + s * (cimag(M3(u, 1, 2)) + cimag(M3(u, 2, 1)));
  p[6] = p[6] + s * (creal(M3(u, 1, 2)) - creal(M3(u, 2, 1)));
  p[7] = p[7] + s * (cimag(M3(u, 0, 0)) + cimag(M3(u, 1, 1)) - 2.0 * cimag(M3(u, 2, 2))) / SQRT3_R8;
}

/* su3.F90:216-233 p(j) += s Re Tr(lambda_j U) */
void oq_re_tr_j(double *p, const cplx *u, double s) {
  p[0] = p[0] + s * (creal(M3(u, 0, 1)) + creal(M3(u, 1, 0)));
  p[1] = p[1] + s * (cimag(M3(u, 1, 0)) - cimag(M3(u, 0, 1)));
  p[2] = p[2] + s * (creal(M3(u, 0, 0)) - creal(M3(u, 1, 1)));
  p[3] = p[3] + s * (creal(M3(u, 0, 2)) + creal(M3(u, 2, 0)));
  p[4] = p[4] + s * (cimag(M3(u, 2, 0)) - cimag(M3(u, 0, 2)));
  p[5] = p[5] + s * (creal(M3(u, 1, 2)) + creal(M3(u, 2, 1)));
  p[6] = p[6] + s * (cimag(M3(u, 2, 1)) - cimag(M3(u, 1, 2)));
  p[7] = p[7] + s * (creal(M3(u, 0, 0)) + creal(M3(u, 1, 1)) - 2.0 * creal(M3(u, 2, 2))) / SQRT3_R8;
}

/* su3.F90:300-310 third column from the first two */
static void u_complete(cplx *u) {
  M3(u, 0, 2) = conj(M3(u, 1, 0) * M3(u, 2, 1) - M3(u, 2, 0) * M3(u, 1, 1));
  M3(u, 1, 2) = conj(M3(u, 2, 0) * M3(u, 0, 1) - M3(u, 0, 0) * M3(u, 2, 1));
  M3(u, 2, 2) = conj(M3(u, 0, 0) * M3(u, 1, 1) - M3(u, 1, 0) * M3(u, 0, 1));
}

/* su3.F90:313-365 Gram-Schmidt of columns 1, 2 and completion */
void oq_u_normalize(cplx *u) {
  double len = creal(M3(u, 0, 0)) * creal(M3(u, 0, 0)) + cimag(M3(u, 0, 0)) * cimag(M3(u, 0, 0)) +
               creal(M3(u, 1, 0)) * creal(M3(u, 1, 0)) + cimag(M3(u, 1, 0)) * cimag(M3(u, 1, 0)) +
               creal(M3(u, 2, 0)) * creal(M3(u, 2, 0)) + cimag(M3(u, 2, 0)) * cimag(M3(u, 2, 0));
  len = sqrt(len);
  for (int i = 0; i < 3; i++) M3(u, i, 0) = M3(u, i, 0) / len;
  cplx f = M3(u, 0, 1) * conj(M3(u, 0, 0)) + M3(u, 1, 1) * conj(M3(u, 1, 0)) +
           M3(u, 2, 1) * conj(M3(u, 2, 0));
  for (int i = 0; i < 3; i++) M3(u, i, 1) = M3(u, i, 1) - f * M3(u, i, 0);
  len = creal(M3(u, 0, 1)) * creal(M3(u, 0, 1)) + cimag(M3(u, 0, 1)) * cimag(M3(u, 0, 1)) +
        creal(M3(u, 1, 1)) * creal(M3(u, 1, 1)) + cimag(M3(u, 1, 1)) * cimag(M3(u, 1, 1)) +
        creal(M3(u, 2, 1)) * creal(M3(u, 2, 1)) + cimag(M3(u, 2, 1)) * cimag(M3(u, 2, 1));
  len = sqrt(len);
  for (int i = 0; i < 3; i++) M3(u, i, 1) = M3(u, i, 1) / len;
  u_complete(u);
}

/* su3.F90:28-193: u = exp(i lambda_j h_j), closed form via the eigenvalues */
void oq_gen2u(cplx *u, const double *h) {
  const double eps = 0.00000001;
  const double sqrt33 = SQRT3_R8 / 3.0;
  const double twosqrt33 = 2.0 * sqrt33;
  double h2[8], hs[8], hk[8], hs2[8];
  double a8 = h[7] * sqrt33;
  double a12 = h[0] * h[0] + h[1] * h[1];
  double a45 = h[3] * h[3] + h[4] * h[4];
  double a67 = h[5] * h[5] + h[6] * h[6];
  h2[0] = 2 * h[0] * a8 + h[3] * h[5] + h[4] * h[6];
  h2[1] = 2 * h[1] * a8 + h[4] * h[5] - h[3] * h[6];
  h2[2] = 2 * h[2] * a8 + 0.5 * (a45 - a67);
  h2[3] = h[3] * (h[2] - a8) + h[0] * h[5] - h[1] * h[6];
  h2[4] = h[4] * (h[2] - a8) + h[0] * h[6] + h[1] * h[5];
  h2[5] = h[5] * (-h[2] - a8) + h[0] * h[3] + h[1] * h[4];
  h2[6] = h[6] * (-h[2] - a8) + h[0] * h[4] - h[1] * h[3];
  h2[7] = (h[2] * h[2] - h[7] * h[7] + a12 - 0.5 * (a45 + a67)) * sqrt33;

  double q = h[0] * h[0];
  for (int i = 1; i < 8; i++) q = q + h[i] * h[i];
  q = 2.0 * q;
  double p = h[0] * h2[0];
  for (int i = 1; i < 8; i++) p = p + h[i] * h2[i];
  p = 2.0 * p / 3.0;

  double a = sqrt(2.0 * q / 3.0);
  double alpha = acos(4.0 * p / (a * a * a)) / 3.0;
  double l1, l2;
  if (alpha <= PI_R8 / 6) {
    l1 = a * cos(alpha);
    l2 = a * cos(alpha + 2 * PI_R8 / 3);
  } else {
    l2 = a * cos(alpha);
    l1 = a * cos(alpha + 2 * PI_R8 / 3);
  }
  double l3 = -l1 - l2;
  double l12 = l1 * l2;
  double s = -l1 - 2 * l2;
  double aux = (2.0 * l3 * l3 + l12) * (l1 - l2);
  double c = s * (l3 * l3 + 2.0 * l12) / aux;
  double d = -3.0 * s * l3 / aux;
  for (int i = 0; i < 8; i++) {
    hs[i] = c * h[i] + d * h2[i];
    hk[i] = h[i] - hs[i];
  }
  a8 = hs[7] * sqrt33;
  a12 = hs[0] * hs[0] + hs[1] * hs[1];
  a45 = hs[3] * hs[3] + hs[4] * hs[4];
  a67 = hs[5] * hs[5] + hs[6] * hs[6];
  hs2[0] = 2 * hs[0] * a8 + hs[3] * hs[5] + hs[4] * hs[6];
  hs2[1] = 2 * hs[1] * a8 + hs[4] * hs[5] - hs[3] * hs[6];
  hs2[2] = 2 * hs[2] * a8 + 0.5 * (a45 - a67);
  hs2[3] = hs[3] * (hs[2] - a8) + hs[0] * hs[5] - hs[1] * hs[6];
  hs2[4] = hs[4] * (hs[2] - a8) + hs[0] * hs[6] + hs[1] * hs[5];
  hs2[5] = hs[5] * (-hs[2] - a8) + hs[0] * hs[3] + hs[1] * hs[4];
  hs2[6] = hs[6] * (-hs[2] - a8) + hs[0] * hs[4] - hs[1] * hs[3];
  hs2[7] = (hs[2] * hs[2] - hs[7] * hs[7] + a12 - 0.5 * (a45 + a67)) * sqrt33;

  double cs1, cs2;
  if (fabs(s) > eps) {
    cs1 = sin(s) / s;
    cs2 = (cos(s) - 1) / (s * s);
  } else {
    cs1 = 1;
    cs2 = -0.5;
  }
  cplx ck1 = mk(cos(l3), sin(l3));
  cplx ck2 = 1.0 / (ck1 * ck1);
  cplx ck3 = (ck2 + 2.0 * ck1) / 3.0;
  cplx ck4;
  if (fabs(l3) > eps) ck4 = (ck1 - ck2) / (3 * l3);
  else ck4 = mk(0.0, 3.0);

  aux = hs[0] * hs[0];
  for (int i = 1; i < 8; i++) aux = aux + hs[i] * hs[i];
  aux = 2.0 * aux;

  cplx ms[9], mkk[9];
  double dg = 1.0 + cs2 * aux / 3.0;
  M3(ms, 0, 0) = dg + mk(cs2 * (hs2[2] + sqrt33 * hs2[7]), cs1 * (hs[2] + sqrt33 * hs[7]));
  M3(ms, 1, 1) = dg + mk(cs2 * (-hs2[2] + sqrt33 * hs2[7]), cs1 * (-hs[2] + sqrt33 * hs[7]));
  M3(ms, 2, 2) = dg + mk(-cs2 * twosqrt33 * hs2[7], -cs1 * twosqrt33 * hs[7]);
  M3(ms, 0, 1) = mk(cs2 * hs2[0] + cs1 * hs[1], cs1 * hs[0] - cs2 * hs2[1]);
  M3(ms, 1, 0) = mk(cs2 * hs2[0] - cs1 * hs[1], cs1 * hs[0] + cs2 * hs2[1]);
  M3(ms, 0, 2) = mk(cs2 * hs2[3] + cs1 * hs[4], cs1 * hs[3] - cs2 * hs2[4]);
  M3(ms, 2, 0) = mk(cs2 * hs2[3] - cs1 * hs[4], cs1 * hs[3] + cs2 * hs2[4]);
  M3(ms, 1, 2) = mk(cs2 * hs2[5] + cs1 * hs[6], cs1 * hs[5] - cs2 * hs2[6]);
  M3(ms, 2, 1) = mk(cs2 * hs2[5] - cs1 * hs[6], cs1 * hs[5] + cs2 * hs2[6]);

  M3(mkk, 0, 0) = ck3 + ck4 * (hk[2] + sqrt33 * hk[7]);
  M3(mkk, 1, 1) = ck3 + ck4 * (-hk[2] + sqrt33 * hk[7]);
  M3(mkk, 2, 2) = ck3 - ck4 * twosqrt33 * hk[7];
  M3(mkk, 0, 1) = ck4 * mk(hk[0], -hk[1]);
  M3(mkk, 1, 0) = ck4 * mk(hk[0], hk[1]);
  M3(mkk, 0, 2) = ck4 * mk(hk[3], -hk[4]);
  M3(mkk, 2, 0) = ck4 * mk(hk[3], hk[4]);
  M3(mkk, 1, 2) = ck4 * mk(hk[5], -hk[6]);
  M3(mkk, 2, 1) = ck4 * mk(hk[5], hk[6]);

  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      cplx t = M3(ms, i, 0) * M3(mkk, 0, j);
      for (int k = 1; k < 3; k++) t = t + M3(ms, i, k) * M3(mkk, k, j);
      M3(u, i, j) = t;
    }
}

/* ------------------------------------------------------------------------ */
/* gauge configurations                                                      */
/* ------------------------------------------------------------------------ */
/* conf.F90:181-199 */
void oq_conf_cold(const oq_geom *g, cplx *u) {
  for (int mu = 0; mu < 4; mu++)
    for (int eo = 0; eo < 2; eo++)
      for (int i = 0; i < g->volh; i++) {
        cplx *l = ULINK(g, u, i, eo, mu);
        for (int e = 0; e < 9; e++) l[e] = 0;
        M3(l, 0, 0) = 1;
        M3(l, 1, 1) = 1;
        M3(l, 2, 2) = 1;
      }
}

/* conf.F90:201-217 */
void oq_conf_hot(const oq_geom *g, cplx *u) {
  for (int mu = 0; mu < 4; mu++)
    for (int eo = 0; eo < 2; eo++) {
      oq_ran_gauss_volh(g, 9, ULINK(g, u, 0, eo, mu), 1.0, eo);
      for (int i = 0; i < g->volh; i++) oq_u_normalize(ULINK(g, u, i, eo, mu));
    }
}

/* staple.F90:28-63 */
static void staple(const oq_geom *g, cplx *uuu, const cplx *u, int i, int e, int mu) {
  int o = 1 - e;
  for (int k = 0; k < 9; k++) uuu[k] = 0;
  for (int nu = 0; nu < 4; nu++) {
    if (nu == mu) continue;
    int j1 = OQ_NN(g, i, e, mu, OQ_FWD);
    int j2 = OQ_NN(g, i, e, nu, OQ_FWD);
    int j3 = OQ_NN(g, i, e, nu, OQ_BWD);
    int j4 = OQ_NN(g, j3, o, mu, OQ_FWD);
    uuu_fwd(uuu, ULINK(g, u, j1, o, nu), ULINK(g, u, j2, o, mu), ULINK(g, u, i, e, nu));
    uuu_bwd(uuu, ULINK(g, u, j4, e, nu), ULINK(g, u, j3, o, mu), ULINK(g, u, j3, o, nu));
  }
}

/* cooling.F90:131-193: Cabibbo-Marinari cooling over 3 SU(2) subgroups */
void oq_conf_relax(const oq_geom *g, cplx *u) {
  for (int mu = 0; mu < 4; mu++)
    for (int eo = 0; eo < 2; eo++) {
#pragma omp parallel for schedule(static)
      for (int i = 0; i < g->volh; i++) {
        cplx uuu[9], w[9], a[9], t[9];
        staple(g, uuu, u, i, eo, mu);
        for (int k = 0; k < 3; k++) {
          int c1 = k == 2 ? 1 : 0;
          int c2 = k == 0 ? 1 : 2;
          cplx *l = ULINK(g, u, i, eo, mu);
          uu(w, l, uuu);
          double p0 = creal(M3(w, c1, c1)) + creal(M3(w, c2, c2));
          double p1 = -(cimag(M3(w, c1, c2)) + cimag(M3(w, c2, c1)));
          double p2 = -(creal(M3(w, c1, c2)) - creal(M3(w, c2, c1)));
          double p3 = -(cimag(M3(w, c1, c1)) - cimag(M3(w, c2, c2)));
          double fac = 1.0 / sqrt(p0 * p0 + p1 * p1 + p2 * p2 + p3 * p3);
          double a0 = fac * p0, a1 = fac * p1, a2 = fac * p2, a3 = fac * p3;
          for (int e = 0; e < 9; e++) a[e] = 0;
          M3(a, 0, 0) = 1; M3(a, 1, 1) = 1; M3(a, 2, 2) = 1;
          M3(a, c1, c1) = mk(a0, a3);
          M3(a, c1, c2) = mk(a2, a1);
          M3(a, c2, c1) = mk(-a2, a1);
          M3(a, c2, c2) = mk(a0, -a3);
          memcpy(t, l, sizeof(t));
          uu(l, a, t);
        }
      }
    }
}

/* ------------------------------------------------------------------------ */
/* deterministic reductions over real-overindexed fields (sc.F90:224-286)    */
/* ------------------------------------------------------------------------ */
#define OQ_NCHUNK 256

double oq_dot(const double *x, const double *y, long n) {
  double part[OQ_NCHUNK];
  long chunk = (n + OQ_NCHUNK - 1) / OQ_NCHUNK;
#pragma omp parallel for schedule(static)
  for (int c = 0; c < OQ_NCHUNK; c++) {
    long lo = c * chunk, hi = lo + chunk < n ? lo + chunk : n;
    double s = 0;
    for (long k = lo; k < hi; k++) s = s + x[k] * y[k];
    part[c] = s;
  }
  double s = 0;
  for (int c = 0; c < OQ_NCHUNK; c++) s += part[c];
  return s;
}

static cplx oq_cdotc(const cplx *x, const cplx *y, long n) {
  cplx part[OQ_NCHUNK];
  long chunk = (n + OQ_NCHUNK - 1) / OQ_NCHUNK;
#pragma omp parallel for schedule(static)
  for (int c = 0; c < OQ_NCHUNK; c++) {
    long lo = c * chunk, hi = lo + chunk < n ? lo + chunk : n;
    cplx s = 0;
    for (long k = lo; k < hi; k++) s = s + conj(x[k]) * y[k];
    part[c] = s;
  }
  cplx s = 0;
  for (int c = 0; c < OQ_NCHUNK; c++) s += part[c];
  return s;
}

/* sc.F90:124-142 inout += a*in */
static void sc_axpy(double *io, const double *in, double a, long n) {
#pragma omp parallel for schedule(static)
  for (long k = 0; k < n; k++) io[k] = io[k] + a * in[k];
}
/* sc.F90:184-201 inout = b*inout + in */
static void sc_xpby(double *io, const double *in, double b, long n) {
#pragma omp parallel for schedule(static)
  for (long k = 0; k < n; k++) io[k] = b * io[k] + in[k];
}
static void sc_copy(double *out, const double *in, long n) {
#pragma omp parallel for schedule(static)
  for (long k = 0; k < n; k++) out[k] = in[k];
}
static void sc_scale(double *io, double f, long n) {
#pragma omp parallel for schedule(static)
  for (long k = 0; k < n; k++) io[k] = io[k] * f;
}

/* ------------------------------------------------------------------------ */
/* D-slash, libd21 (d/D21.F90:29-182, d/D21xyzt.F90:81-198)                   */
/* ------------------------------------------------------------------------ */
/* Half-spinor projection of ``in`` at site j for direction mu; fb selects the
 * forward (1 - gamma_mu) or backward (1 + gamma_mu) projector; dag flips the
 * signs as d_dag does (d/D21.F90:98-178). */
static inline void project(const cplx *in, int j, int mu, int fb, int dag, int c, cplx *h1, cplx *h2) {
  double s = dag ? -1.0 : 1.0;
  double sg = fb == OQ_FWD ? -s : s;  /* MINUS for forward, PLUS for backward */
  cplx p1 = SP(in, 0, c, j), p2 = SP(in, 1, c, j), p3 = SP(in, 2, c, j), p4 = SP(in, 3, c, j);
  switch (mu) {
    case 0: *h1 = p1 + sg * itimes(p4); *h2 = p2 + sg * itimes(p3); break;
    case 1: *h1 = p1 + sg * p4; *h2 = p2 - sg * p3; break;
    case 2: *h1 = p1 + sg * itimes(p3); *h2 = p2 - sg * itimes(p4); break;
    default:
      if ((fb == OQ_FWD) != (dag != 0)) { *h1 = p3; *h2 = p4; }
      else { *h1 = p1; *h2 = p2; }
  }
}

static void d21(const oq_geom *g, int e, int o, cplx *out, const cplx *in, const cplx *u, int dag) {
  const double s = dag ? -1.0 : 1.0;
  const int volh = g->volh;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < volh; i++) {
    cplx b[4][3];
    static const int order[4] = {3, 2, 1, 0};  /* t, z, y, x (d/D21.F90:58-72) */
    for (int od = 0; od < 4; od++) {
      int mu = order[od];
      int jb = OQ_NN(g, i, e, mu, OQ_BWD);
      int jf = OQ_NN(g, i, e, mu, OQ_FWD);
      const cplx *ue = ULINK(g, u, i, e, mu);
      const cplx *uo = ULINK(g, u, jb, o, mu);
      cplx bb1[3] = {0, 0, 0}, bb2[3] = {0, 0, 0}, bf1[3] = {0, 0, 0}, bf2[3] = {0, 0, 0};
      for (int k = 0; k < 3; k++) {
        cplx ab1, ab2, af1, af2;
        project(in, jb, mu, OQ_BWD, dag, k, &ab1, &ab2);
        project(in, jf, mu, OQ_FWD, dag, k, &af1, &af2);
        for (int c = 0; c < 3; c++) {
          cplx ubc = conj(M3(uo, k, c));
          bb1[c] = k ? bb1[c] + ab1 * ubc : ab1 * ubc;
          bb2[c] = k ? bb2[c] + ab2 * ubc : ab2 * ubc;
        }
        for (int c = 0; c < 3; c++) {
          cplx ufc = M3(ue, c, k);
          bf1[c] = k ? bf1[c] + af1 * ufc : af1 * ufc;
          bf2[c] = k ? bf2[c] + af2 * ufc : af2 * ufc;
        }
      }
      for (int c = 0; c < 3; c++) {
        switch (mu) {
          case 3:
            if (!dag) { b[0][c] = 2.0 * bb1[c]; b[1][c] = 2.0 * bb2[c]; b[2][c] = 2.0 * bf1[c]; b[3][c] = 2.0 * bf2[c]; }
            else { b[0][c] = 2.0 * bf1[c]; b[1][c] = 2.0 * bf2[c]; b[2][c] = 2.0 * bb1[c]; b[3][c] = 2.0 * bb2[c]; }
            break;
          case 2:
            b[0][c] = b[0][c] + bb1[c] + bf1[c];
            b[1][c] = b[1][c] + bb2[c] + bf2[c];
            b[2][c] = b[2][c] - s * itimes(bb1[c]) + s * itimes(bf1[c]);
            b[3][c] = b[3][c] + s * itimes(bb2[c]) - s * itimes(bf2[c]);
            break;
          case 1:
            b[0][c] = b[0][c] + bb1[c] + bf1[c];
            b[1][c] = b[1][c] + bb2[c] + bf2[c];
            b[2][c] = b[2][c] - s * bb2[c] + s * bf2[c];
            b[3][c] = b[3][c] + s * bb1[c] - s * bf1[c];
            break;
          default:
            b[0][c] = b[0][c] + bb1[c] + bf1[c];
            b[1][c] = b[1][c] + bb2[c] + bf2[c];
            b[2][c] = b[2][c] - s * itimes(bb2[c]) + s * itimes(bf2[c]);
            b[3][c] = b[3][c] - s * itimes(bb1[c]) + s * itimes(bf1[c]);
        }
      }
    }
    for (int c = 0; c < 3; c++)
      for (int sp = 0; sp < 4; sp++) SP(out, sp, c, i) = b[sp][c];
  }
}

void oq_d(const oq_geom *g, int e, int o, cplx *out, const cplx *in, const cplx *u) {
  d21(g, e, o, out, in, u, 0);
}
void oq_d_dag(const oq_geom *g, int e, int o, cplx *out, const cplx *in, const cplx *u) {
  d21(g, e, o, out, in, u, 1);
}

/* ------------------------------------------------------------------------ */
/* clover blocks (clover/clover.h:28-193, typedef_clover.F90)                */
/* ------------------------------------------------------------------------ */
/* packed slot of the upper triangle A(r,c), r<c, in the 18-complex layout */
static const int A_SLOT[6][6] = {
    {-1, 1, 2, 3, 4, 5}, {-1, -1, 6, 7, 8, 9}, {-1, -1, -1, 11, 12, 13},
    {-1, -1, -1, -1, 14, 15}, {-1, -1, -1, -1, -1, 17}, {-1, -1, -1, -1, -1, -1}};

static inline double a_diag(const cplx *a, int r) {
  static const int slot[6] = {0, 0, 10, 10, 16, 16};
  return (r & 1) ? cimag(a[slot[r]]) : creal(a[slot[r]]);
}
static inline cplx a_el(const cplx *a, int r, int c) {
  if (r == c) return a_diag(a, r);
  if (r < c) return a[A_SLOT[r][c]];
  return conj(a[A_SLOT[c][r]]);
}
/* B: strictly-lower L entries at slot r(r-1)/2+c, diagonal 1/D at 15..17 */
static inline double b_diag(const cplx *b, int r) {
  static const int slot[6] = {15, 15, 16, 16, 17, 17};
  return (r & 1) ? cimag(b[slot[r]]) : creal(b[slot[r]]);
}
static inline cplx b_el(const cplx *b, int r, int c) {
  if (r > c) return b[r * (r - 1) / 2 + c];
  return conj(b[c * (c - 1) / 2 + r]);
}

/* clover_mult_a.h90: y = A x (Hermitian 6x6 in packed form) */
static inline void mult_a6(const cplx *a, const cplx *x, cplx *y) {
  for (int r = 0; r < 6; r++) {
    cplx s = 0;
    for (int c = 0; c < 6; c++) {
      cplx t = r == c ? a_diag(a, r) * x[c] : a_el(a, r, c) * x[c];
      s = c ? s + t : t;
    }
    y[r] = s;
  }
}
/* clover_mult_b.h90: x = B^-1 y with B = L D L^+ (forward/back substitution) */
static inline void mult_b6(const cplx *b, cplx *y, cplx *x) {
  for (int r = 1; r < 6; r++) {
    cplx s = y[r];
    for (int c = 0; c < r; c++) s = s - b_el(b, r, c) * y[c];
    y[r] = s;
  }
  for (int r = 5; r >= 0; r--) {
    cplx s = y[r] * b_diag(b, r);
    for (int c = r + 1; c < 6; c++) s = s - b_el(b, r, c) * x[c];
    x[r] = s;
  }
}

/* spin-colour index of SC_k, k=0..11 (clover.h:182-193) */
#define SCK(k) ((((k) % 3) * 4) + ((k) / 3))

/* clover/clover_mult_a.F90:30-98 */
void oq_clover_mult_a(cplx *out, const cplx *a, const cplx *in, int volh) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < volh; i++) {
    const cplx *ps = in + (size_t)i * 12;
    cplx *po = out + (size_t)i * 12;
    const cplx *a1 = a + (size_t)i * 36, *a2 = a1 + 18;
    cplx x[6], y[6];
    for (int k = 0; k < 6; k++) x[k] = ps[SCK(k)] + ps[SCK(k + 6)];
    mult_a6(a1, x, y);
    for (int k = 0; k < 6; k++) { po[SCK(k)] = y[k]; po[SCK(k + 6)] = y[k]; }
    for (int k = 0; k < 6; k++) x[k] = ps[SCK(k)] - ps[SCK(k + 6)];
    mult_a6(a2, x, y);
    for (int k = 0; k < 6; k++) { po[SCK(k)] = po[SCK(k)] + y[k]; po[SCK(k + 6)] = po[SCK(k + 6)] - y[k]; }
  }
}

/* clover/clover_mult_ao.F90:30-98 (in place) */
void oq_clover_mult_ao(const cplx *a, cplx *xf, int volh) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < volh; i++) {
    cplx *px = xf + (size_t)i * 12;
    const cplx *a1 = a + (size_t)i * 36, *a2 = a1 + 18;
    cplx xp[6], xm[6], y[6];
    for (int k = 0; k < 6; k++) xp[k] = px[SCK(k)] + px[SCK(k + 6)];
    mult_a6(a1, xp, y);
    for (int k = 0; k < 6; k++) xm[k] = px[SCK(k)] - px[SCK(k + 6)];
    for (int k = 0; k < 6; k++) { px[SCK(k)] = y[k]; px[SCK(k + 6)] = y[k]; }
    mult_a6(a2, xm, y);
    for (int k = 0; k < 6; k++) { px[SCK(k)] = px[SCK(k)] + y[k]; px[SCK(k + 6)] = px[SCK(k + 6)] - y[k]; }
  }
}

/* clover/clover_mult_b.F90:30-99 (in place) */
void oq_clover_mult_b(const cplx *b, cplx *xf, int volh) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < volh; i++) {
    cplx *px = xf + (size_t)i * 12;
    const cplx *b1 = b + (size_t)i * 36, *b2 = b1 + 18;
    cplx y[6], x[6];
    for (int k = 0; k < 6; k++) y[k] = px[SCK(k)] + px[SCK(k + 6)];
    mult_b6(b1, y, x);
    for (int k = 0; k < 6; k++) y[k] = px[SCK(k)] - px[SCK(k + 6)];
    for (int k = 0; k < 6; k++) { px[SCK(k)] = x[k]; px[SCK(k + 6)] = x[k]; }
    mult_b6(b2, y, x);
    for (int k = 0; k < 6; k++) { px[SCK(k)] = px[SCK(k)] + x[k]; px[SCK(k + 6)] = px[SCK(k + 6)] - x[k]; }
  }
}

/* clover/clover_f_mu_nu.F90:37-103: clover-leaf field strength (mu,nu 0-based) */
static void clover_f_mu_nu(const oq_geom *g, cplx *f, int mu, int nu, int x, int e, const cplx *u) {
  int o = 1 - e;
  int xp_ = OQ_NN(g, x, e, mu, OQ_FWD), xm_ = OQ_NN(g, x, e, mu, OQ_BWD);
  int x_p = OQ_NN(g, x, e, nu, OQ_FWD), x_m = OQ_NN(g, x, e, nu, OQ_BWD);
  int xmp = OQ_NN(g, xm_, o, nu, OQ_FWD), xmm = OQ_NN(g, xm_, o, nu, OQ_BWD);
  int xpm = OQ_NN(g, xp_, o, nu, OQ_BWD);
  for (int k = 0; k < 9; k++) f[k] = 0;
  const cplx *l1, *l2, *l3, *l4;
  /* clover_uuuu1: u1 u2 u3^+ u4^+ */
  l1 = ULINK(g, u, x, e, mu); l2 = ULINK(g, u, xp_, o, nu); l3 = ULINK(g, u, x_p, o, mu); l4 = ULINK(g, u, x, e, nu);
  for (int i = 0; i < 3; i++) for (int m = 0; m < 3; m++) for (int j = 0; j < 3; j++) for (int k = 0; k < 3; k++) for (int l = 0; l < 3; l++)
    M3(f, i, m) = M3(f, i, m) + M3(l1, i, j) * M3(l2, j, k) * conj(M3(l3, l, k)) * conj(M3(l4, m, l));
  /* clover_uuuu2: u1 u2^+ u3^+ u4 */
  l1 = ULINK(g, u, x, e, nu); l2 = ULINK(g, u, xmp, e, mu); l3 = ULINK(g, u, xm_, o, nu); l4 = ULINK(g, u, xm_, o, mu);
  for (int i = 0; i < 3; i++) for (int m = 0; m < 3; m++) for (int j = 0; j < 3; j++) for (int k = 0; k < 3; k++) for (int l = 0; l < 3; l++)
    M3(f, i, m) = M3(f, i, m) + M3(l1, i, j) * conj(M3(l2, k, j)) * conj(M3(l3, l, k)) * M3(l4, l, m);
  /* clover_uuuu3: u1^+ u2^+ u3 u4 */
  l1 = ULINK(g, u, xm_, o, mu); l2 = ULINK(g, u, xmm, e, nu); l3 = ULINK(g, u, xmm, e, mu); l4 = ULINK(g, u, x_m, o, nu);
  for (int i = 0; i < 3; i++) for (int m = 0; m < 3; m++) for (int j = 0; j < 3; j++) for (int k = 0; k < 3; k++) for (int l = 0; l < 3; l++)
    M3(f, i, m) = M3(f, i, m) + conj(M3(l1, j, i)) * conj(M3(l2, k, j)) * M3(l3, k, l) * M3(l4, l, m);
  /* clover_uuuu4: u1^+ u2 u3 u4^+ */
  l1 = ULINK(g, u, x_m, o, nu); l2 = ULINK(g, u, x_m, o, mu); l3 = ULINK(g, u, xpm, e, nu); l4 = ULINK(g, u, x, e, mu);
  for (int i = 0; i < 3; i++) for (int m = 0; m < 3; m++) for (int j = 0; j < 3; j++) for (int k = 0; k < 3; k++) for (int l = 0; l < 3; l++)
    M3(f, i, m) = M3(f, i, m) + conj(M3(l1, j, i)) * M3(l2, j, k) * M3(l3, k, l) * conj(M3(l4, m, l));

  M3(f, 0, 0) = mk(2.0 * cimag(M3(f, 0, 0)), 0.0);
  M3(f, 1, 1) = mk(2.0 * cimag(M3(f, 1, 1)), 0.0);
  M3(f, 2, 2) = mk(2.0 * cimag(M3(f, 2, 2)), 0.0);
  M3(f, 0, 1) = itimes(conj(M3(f, 1, 0)) - M3(f, 0, 1));
  M3(f, 0, 2) = itimes(conj(M3(f, 2, 0)) - M3(f, 0, 2));
  M3(f, 1, 2) = itimes(conj(M3(f, 2, 1)) - M3(f, 1, 2));
  M3(f, 1, 0) = conj(M3(f, 0, 1));
  M3(f, 2, 0) = conj(M3(f, 0, 2));
  M3(f, 2, 1) = conj(M3(f, 1, 2));
}

/* full Hermitian 6x6 used while building a block */
typedef struct { cplx m[6][6]; } blk6;

/* clover_init.F90:99-120 */
static void clover_init1(blk6 *a, const cplx *f) {
  for (int r = 0; r < 3; r++) {
    a->m[r][r] = creal(M3(f, r, r));
    a->m[r + 3][r + 3] = -creal(M3(f, r, r));
  }
  a->m[0][1] = M3(f, 0, 1); a->m[0][2] = M3(f, 0, 2); a->m[1][2] = M3(f, 1, 2);
  a->m[3][4] = -a->m[0][1]; a->m[3][5] = -a->m[0][2]; a->m[4][5] = -a->m[1][2];
}
/* clover_init.F90:122-145 */
static void clover_init2(blk6 *a, const cplx *f, const cplx *gg) {
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) a->m[r][c + 3] = M3(f, r, c) + itimes(M3(gg, r, c));
}
/* clover_init.F90:147-190 */
static void clover_init3(blk6 *a1, blk6 *a2, const blk6 *p, const blk6 *q, double s) {
  for (int r = 0; r < 6; r++)
    for (int c = r; c < 6; c++) {
      a1->m[r][c] = s * (p->m[r][c] + q->m[r][c]);
      a2->m[r][c] = s * (p->m[r][c] - q->m[r][c]);
    }
  for (int r = 0; r < 6; r++) {
    a1->m[r][r] = creal(a1->m[r][r]) + 1.0;
    a2->m[r][r] = creal(a2->m[r][r]) + 1.0;
  }
}
static inline cplx blk_el(const blk6 *a, int r, int c) { return r <= c ? a->m[r][c] : conj(a->m[c][r]); }

static void pack_a(cplx *dst, const blk6 *a) {
  dst[0] = mk(creal(a->m[0][0]), creal(a->m[1][1]));
  dst[10] = mk(creal(a->m[2][2]), creal(a->m[3][3]));
  dst[16] = mk(creal(a->m[4][4]), creal(a->m[5][5]));
  for (int r = 0; r < 6; r++)
    for (int c = r + 1; c < 6; c++) dst[A_SLOT[r][c]] = a->m[r][c];
}

/* clover_inv.F90:29-220: LDL^+ factors (B), explicit inverse, then halving
 * of A, A^-1 and 1/D */
static void clover_inv(cplx *bdst, cplx *ainvdst, blk6 *a) {
  cplx L[6][6];
  double dinv[6], d[6];
  for (int r = 0; r < 6; r++) {
    cplx tmp[6];
    for (int c = 0; c < r; c++) {
      cplx t = blk_el(a, r, c);
      for (int k = 0; k < c; k++) t = t - tmp[k] * conj(L[c][k]);
      tmp[c] = t;
    }
    for (int c = 0; c < r; c++) L[r][c] = tmp[c] * dinv[c];
    double dr = creal(a->m[r][r]);
    for (int k = 0; k < r; k++) dr = dr - d[k] * sqc(L[r][k]);
    d[r] = dr;
    dinv[r] = 1.0 / dr;
  }
  /* pack B (unhalved) to run the unit solves of clover_inv2 */
  cplx b[18];
  for (int r = 1; r < 6; r++)
    for (int c = 0; c < r; c++) b[r * (r - 1) / 2 + c] = L[r][c];
  b[15] = mk(dinv[0], dinv[1]);
  b[16] = mk(dinv[2], dinv[3]);
  b[17] = mk(dinv[4], dinv[5]);
  blk6 ainv;
  for (int col = 0; col < 6; col++) {
    cplx y[6], x[6];
    for (int k = 0; k < 6; k++) y[k] = k == col ? 1.0 : 0.0;
    mult_b6(b, y, x);
    for (int k = 0; k < 6; k++) x[k] = 0.5 * conj(x[k]);
    ainv.m[col][col] = creal(x[col]);
    for (int k = col + 1; k < 6; k++) ainv.m[col][k] = x[k];
  }
  pack_a(ainvdst, &ainv);
  for (int k = 0; k < 15; k++) bdst[k] = b[k];
  bdst[15] = mk(0.5 * dinv[0], 0.5 * dinv[1]);
  bdst[16] = mk(0.5 * dinv[2], 0.5 * dinv[3]);
  bdst[17] = mk(0.5 * dinv[4], 0.5 * dinv[5]);
  for (int r = 0; r < 6; r++)
    for (int c = r; c < 6; c++) a->m[r][c] = 0.5 * a->m[r][c];
}

/* clover/clover_init.F90:28-97 */
void oq_clover_init(const oq_geom *g, cplx *a, cplx *ainv, cplx *b, const cplx *u, double csw_kappa) {
  double factor = -csw_kappa / 8.0;
  for (int eo = 0; eo < 2; eo++) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < g->volh; i++) {
      cplx f[9], gg[9];
      blk6 p, q, a1, a2;
      memset(&p, 0, sizeof p);
      memset(&q, 0, sizeof q);
      clover_f_mu_nu(g, f, 1, 0, i, eo, u);
      clover_init1(&p, f);
      clover_f_mu_nu(g, f, 2, 1, i, eo, u);
      clover_f_mu_nu(g, gg, 2, 0, i, eo, u);
      clover_init2(&p, f, gg);
      clover_f_mu_nu(g, f, 2, 3, i, eo, u);
      clover_init1(&q, f);
      clover_f_mu_nu(g, f, 0, 3, i, eo, u);
      clover_f_mu_nu(g, gg, 3, 1, i, eo, u);
      clover_init2(&q, f, gg);
      clover_init3(&a1, &a2, &p, &q, factor);
      size_t off = ((size_t)eo * g->volh + i) * 36;
      clover_inv(b + off, ainv + off, &a1);
      clover_inv(b + off + 18, ainv + off + 18, &a2);
      pack_a(a + off, &a1);
      pack_a(a + off + 18, &a2);
    }
  }
}

/* clover/clover_action.F90:29-60: 2 sum log(det(b1) det(b2)) with the halved 1/D */
double oq_clover_action(const cplx *b, int volh) {
  double part[OQ_NCHUNK];
  int chunk = (volh + OQ_NCHUNK - 1) / OQ_NCHUNK;
#pragma omp parallel for schedule(static)
  for (int c = 0; c < OQ_NCHUNK; c++) {
    double s = 0;
    for (int i = c * chunk; i < volh && i < (c + 1) * chunk; i++) {
      const cplx *b1 = b + (size_t)i * 36, *b2 = b1 + 18;
      double d1 = b_diag(b1, 0) * b_diag(b1, 1) * b_diag(b1, 2) * b_diag(b1, 3) * b_diag(b1, 4) * b_diag(b1, 5);
      double d2 = b_diag(b2, 0) * b_diag(b2, 1) * b_diag(b2, 2) * b_diag(b2, 3) * b_diag(b2, 4) * b_diag(b2, 5);
      s = s + log(d1 * d2);
    }
    part[c] = s;
  }
  double s = 0;
  for (int c = 0; c < OQ_NCHUNK; c++) s += part[c];
  return 2.0 * s;
}

/* h_mult.F90:27-49 out += i h gamma_5 in */
void oq_h_mult_a(cplx *out, double h, const cplx *in, int volh) {
  for (long k = 0; k < 3L * volh; k++) {
    cplx *o = out + 4 * k;
    const cplx *p = in + 4 * k;
    o[0] = o[0] + h * itimes(p[2]);
    o[1] = o[1] + h * itimes(p[3]);
    o[2] = o[2] + h * itimes(p[0]);
    o[3] = o[3] + h * itimes(p[1]);
  }
}
/* h_mult.F90:51-82 x = (1 + i h gamma_5) x */
void oq_h_mult_b(double h, cplx *x, int volh) {
  for (long k = 0; k < 3L * volh; k++) {
    cplx *o = x + 4 * k;
    cplx x1 = o[0], x2 = o[1], x3 = o[2], x4 = o[3];
    o[0] = o[0] + h * itimes(x3);
    o[1] = o[1] + h * itimes(x4);
    o[2] = o[2] + h * itimes(x1);
    o[3] = o[3] + h * itimes(x2);
  }
}

/* ------------------------------------------------------------------------ */
/* even-odd operators (m_tilde.F90:43-114, mtdagmt.F90, w_mult.F90)           */
/* ------------------------------------------------------------------------ */
static void mtil_impl(const oq_geom *g, cplx *out, const cplx *in, const oq_hmc_para *p,
                      const oq_conf *c, int dag) {
  long n = oq_sc_size(g);
  cplx *tmp = xmalloc(sizeof(cplx) * n);
  int volh = g->volh;
  const cplx *ioo = c->i ? c->i + (size_t)OQ_ODD * volh * 36 : NULL;
  const cplx *aee = c->a ? c->a + (size_t)OQ_EVEN * volh * 36 : NULL;
  if (p->kappa != 0) {
    d21(g, OQ_ODD, OQ_EVEN, tmp, in, c->u, dag);
    if (p->csw_kappa != 0) oq_clover_mult_ao(ioo, tmp, volh);
    if (p->h != 0) oq_h_mult_b(dag ? p->h : -p->h, tmp, volh);
    d21(g, OQ_EVEN, OQ_ODD, out, tmp, c->u, dag);
  }
  double b = -p->kappa * p->kappa / (1.0 + p->h * p->h);
  if (p->csw_kappa != 0) {
    oq_clover_mult_a(tmp, aee, in, volh);
    sc_xpby((double *)out, (const double *)tmp, b, 2 * n);
  } else {
    sc_xpby((double *)out, (const double *)in, b, 2 * n);
    if (p->h != 0) oq_h_mult_a(out, dag ? -p->h : p->h, in, volh);
  }
  free(tmp);
}

void oq_mtil(const oq_geom *g, cplx *out, const cplx *in, const oq_hmc_para *p, const oq_conf *c) {
  mtil_impl(g, out, in, p, c, 0);
}
void oq_mtil_dag(const oq_geom *g, cplx *out, const cplx *in, const oq_hmc_para *p, const oq_conf *c) {
  mtil_impl(g, out, in, p, c, 1);
}
void oq_mtdagmt(const oq_geom *g, cplx *out, const cplx *in, const oq_hmc_para *p, const oq_conf *c) {
  cplx *tmp = xmalloc(sizeof(cplx) * oq_sc_size(g));
  oq_mtil(g, tmp, in, p, c);
  oq_mtil_dag(g, out, tmp, p, c);
  free(tmp);
}
void oq_w_mult(const oq_geom *g, cplx *out, const cplx *in, const oq_hmc_para *p, const oq_conf *c) {
  oq_mtil(g, out, in, p, c);
  sc_axpy((double *)out, (const double *)in, p->rho, 2 * oq_sc_size(g));
}
void oq_w_mult_dag(const oq_geom *g, cplx *out, const cplx *in, const oq_hmc_para *p, const oq_conf *c) {
  oq_mtil_dag(g, out, in, p, c);
  sc_axpy((double *)out, (const double *)in, p->rho, 2 * oq_sc_size(g));
}
void oq_w_dagger_w(const oq_geom *g, cplx *out, const cplx *in, const oq_hmc_para *p, const oq_conf *c) {
  cplx *tmp = xmalloc(sizeof(cplx) * oq_sc_size(g));
  oq_w_mult(g, tmp, in, p, c);
  oq_w_mult_dag(g, out, tmp, p, c);
  free(tmp);
}

/* ------------------------------------------------------------------------ */
/* CG (cg.F90:51-137)                                                        */
/* ------------------------------------------------------------------------ */
int oq_cg(const oq_geom *g, oq_matrix_mult mm, cplx *xc, const cplx *bc, const oq_hmc_para *p,
          const oq_conf *c, const oq_cg_para *cp, oq_cg_stat *st, int *iterations, double *rtr_out) {
  long n = 2 * oq_sc_size(g);
  double *x = (double *)xc;
  const double *b = (const double *)bc;
  double *r = xmalloc(sizeof(double) * n), *pp = xmalloc(sizeof(double) * n), *aap = xmalloc(sizeof(double) * n);
  mm(g, (cplx *)r, xc, p, c);
  double part[OQ_NCHUNK];
  long chunk = (n + OQ_NCHUNK - 1) / OQ_NCHUNK;
#pragma omp parallel for schedule(static)
  for (int ch = 0; ch < OQ_NCHUNK; ch++) {
    double s = 0;
    for (long k = ch * chunk; k < n && k < (ch + 1) * chunk; k++) {
      r[k] = b[k] - r[k];
      pp[k] = r[k];
      s = s + r[k] * r[k];
    }
    part[ch] = s;
  }
  double rtrold = 0;
  for (int ch = 0; ch < OQ_NCHUNK; ch++) rtrold += part[ch];
  double rtr = rtrold;
  int niter, conv = 0;
  for (niter = 1; niter <= cp->maxiter; niter++) {
    mm(g, (cplx *)aap, (const cplx *)pp, p, c);
    double paap = oq_dot(pp, aap, n);
    double ak = rtrold / paap;
#pragma omp parallel for schedule(static)
    for (int ch = 0; ch < OQ_NCHUNK; ch++) {
      double s = 0;
      for (long k = ch * chunk; k < n && k < (ch + 1) * chunk; k++) {
        x[k] = x[k] + ak * pp[k];
        r[k] = r[k] - ak * aap[k];
        s = s + r[k] * r[k];
      }
      part[ch] = s;
    }
    rtr = 0;
    for (int ch = 0; ch < OQ_NCHUNK; ch++) rtr += part[ch];
    if (rtr <= (double)cp->rest) { conv = 1; break; }
    double bk = rtr / rtrold;
    rtrold = rtr;
    sc_xpby(pp, r, bk, n);
  }
  if (!conv) niter = niter - 1;
  free(r); free(pp); free(aap);
  if (st) {
    st->ncall = st->ncall + 1;
    st->niter = niter;
    st->niter_max = st->niter_max > niter ? st->niter_max : niter;
    st->niter_tot = st->niter_tot + niter;
  }
  if (iterations) *iterations = niter;
  if (rtr_out) *rtr_out = rtr;
  if (!conv && cp->log != 2) return 1;   /* cg.F90:121-124 dies here */
  return 0;
}

/* ------------------------------------------------------------------------ */
/* fermion force: hopping part (dsf.F90:28-110, d/DSFxyzt.F90:77-117)        */
/* ------------------------------------------------------------------------ */
static void dsf_dir(const oq_geom *g, double *pfield, const cplx *bf, const cplx *af, double s,
                    const cplx *ufield, const int *nn, int mu, int fwd) {
  const double sg = fwd ? 1.0 : -1.0;   /* "plus" */
  const int volh = g->volh;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < volh; i++) {
    int j = nn[i];
    int ia = fwd ? j : i, ib = fwd ? i : j;
    cplx w[9], v[9];
    for (int ca = 0; ca < 3; ca++) {
      cplx p1 = SP(af, 0, ca, ia), p2 = SP(af, 1, ca, ia), p3 = SP(af, 2, ca, ia), p4 = SP(af, 3, ca, ia);
      cplx a1, a2, a3, a4;
      switch (mu) {
        case 0: a1 = p1 - sg * itimes(p4); a2 = p2 - sg * itimes(p3); a3 = sg * itimes(a2); a4 = sg * itimes(a1); break;
        case 1: a1 = p1 - sg * p4; a2 = p2 + sg * p3; a3 = sg * a2; a4 = -sg * a1; break;
        case 2: a1 = p1 - sg * itimes(p3); a2 = p2 + sg * itimes(p4); a3 = sg * itimes(a1); a4 = -sg * itimes(a2); break;
        default:
          if (fwd) { a1 = 0; a2 = 0; a3 = 2.0 * p3; a4 = 2.0 * p4; }
          else { a1 = 2.0 * p1; a2 = 2.0 * p2; a3 = 0; a4 = 0; }
      }
      for (int cb = 0; cb < 3; cb++)
        M3(w, ca, cb) = a1 * conj(SP(bf, 0, cb, ib)) + a2 * conj(SP(bf, 1, cb, ib)) +
                        a3 * conj(SP(bf, 2, cb, ib)) + a4 * conj(SP(bf, 3, cb, ib));
    }
    const cplx *ul = ufield + (size_t)i * 9;
    if (fwd) uu(v, ul, w);
    else uud(v, w, ul);
    oq_im_tr_j(pfield + (size_t)i * 8, v, fwd ? -s : s);
  }
}

/* ------------------------------------------------------------------------ */
/* clover force (clover/clover_d.F90, clover_bsa.F90, clover_ts.F90)          */
/* ------------------------------------------------------------------------ */
static void re_tr_acc(double *p, const cplx *r, double s) { oq_re_tr_j(p, r, s); }

/* clover_d.F90:203-231 */
static void clover_d_same_eo(double *p, double s, const cplx *u0, const cplx *u1, const cplx *u2,
                             const cplx *u3, const cplx *u4, const cplx *u5, const cplx *u6,
                             const cplx *wa, const cplx *wb, const cplx *wc) {
  cplx r[9], u[9], v[9];
  for (int k = 0; k < 8; k++) p[k] = 0;
  uu(u, u0, u1);
  uu(v, u3, u2);
  uuu3(r, u, T_N, v, T_D, wa, T_N); re_tr_acc(p, r, s);
  uuu3(r, wa, T_N, v, T_N, u, T_D); re_tr_acc(p, r, s);
  uuu3(r, u, T_N, wb, T_N, v, T_D); re_tr_acc(p, r, s);
  uuu3(r, v, T_N, wb, T_N, u, T_D); re_tr_acc(p, r, s);
  uud(u, u0, u6);
  udu(v, u4, u5);
  uuu3(r, wa, T_N, v, T_N, u, T_D); re_tr_acc(p, r, -s);
  uuu3(r, u, T_N, v, T_D, wa, T_N); re_tr_acc(p, r, -s);
  uuu3(r, v, T_N, wc, T_N, u, T_D); re_tr_acc(p, r, -s);
  uuu3(r, u, T_N, wc, T_N, v, T_D); re_tr_acc(p, r, -s);
}

/* clover_d.F90:233-264 */
static void clover_d_diff_eo(double *p, double s, const cplx *u0, const cplx *u1, const cplx *u2,
                             const cplx *u3, const cplx *u4, const cplx *u5, const cplx *u6,
                             const cplx *wd, const cplx *we, const cplx *wf) {
  cplx r[9], u[9], v[9];
  for (int k = 0; k < 8; k++) p[k] = 0;
  for (int k = 0; k < 9; k++) { u[k] = 0; v[k] = 0; }
  uuu_fwd(u, u1, u2, u3);
  uuu_fwd(v, u2, u1, u0);
  uuu3(r, u0, T_N, wd, T_N, u, T_N); re_tr_acc(p, r, s);
  uuu3(r, u, T_D, wd, T_N, u0, T_D); re_tr_acc(p, r, s);
  uuu3(r, v, T_D, we, T_N, u3, T_D); re_tr_acc(p, r, s);
  uuu3(r, u3, T_N, we, T_N, v, T_N); re_tr_acc(p, r, s);
  for (int k = 0; k < 9; k++) { u[k] = 0; v[k] = 0; }
  uuu_bwd(u, u6, u5, u4);
  uuu_fwd(v, u0, u6, u5);
  uuu3(r, u, T_D, wd, T_N, u0, T_D); re_tr_acc(p, r, -s);
  uuu3(r, u0, T_N, wd, T_N, u, T_N); re_tr_acc(p, r, -s);
  uuu3(r, u4, T_D, wf, T_N, v, T_D); re_tr_acc(p, r, -s);
  uuu3(r, v, T_N, wf, T_N, u4, T_N); re_tr_acc(p, r, -s);
}

/* clover_d.F90:153-201 */
static void clover_d_loop(const oq_geom *g, int e, int mu, int nu, double *pfield, double s,
                          const cplx *u, const cplx *w, int same) {
  int o = 1 - e;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < g->volh; i++) {
    int id = OQ_NN(g, i, e, mu, OQ_FWD), ie = OQ_NN(g, i, e, nu, OQ_FWD), if_ = OQ_NN(g, i, e, nu, OQ_BWD);
    int ia = i, ib = OQ_NN(g, id, o, nu, OQ_FWD), ic = OQ_NN(g, id, o, nu, OQ_BWD);
    double q[8];
    const cplx *u0 = ULINK(g, u, ia, e, mu), *u1 = ULINK(g, u, id, o, nu), *u2 = ULINK(g, u, ie, o, mu),
               *u3 = ULINK(g, u, ia, e, nu), *u4 = ULINK(g, u, if_, o, nu), *u5 = ULINK(g, u, if_, o, mu),
               *u6 = ULINK(g, u, ic, e, nu);
    if (same)
      clover_d_same_eo(q, s, u0, u1, u2, u3, u4, u5, u6, w + (size_t)ia * 9, w + (size_t)ib * 9, w + (size_t)ic * 9);
    else
      clover_d_diff_eo(q, s, u0, u1, u2, u3, u4, u5, u6, w + (size_t)id * 9, w + (size_t)ie * 9, w + (size_t)if_ * 9);
    double *pp = PGEN(g, pfield, i, e, mu);
    for (int j = 0; j < 8; j++) pp[j] = pp[j] + q[j];
  }
}

/* the six planes in the order clover_d.F90:64-71 uses them */
static const int PLANE_MU[6] = {0, 0, 0, 1, 1, 2};
static const int PLANE_NU[6] = {1, 2, 3, 2, 3, 3};

/* clover_d.F90:110-151 */
static void clover_d(const oq_geom *g, int eo, double *p, double s, const cplx *u, const cplx *w6) {
  for (int pl = 0; pl < 6; pl++) {
    const cplx *w = w6 + (size_t)pl * g->volh * 9;
    int mu = PLANE_MU[pl], nu = PLANE_NU[pl], o = 1 - eo;
    clover_d_loop(g, eo, mu, nu, p, s, u, w, 1);
    clover_d_loop(g, eo, nu, mu, p, -s, u, w, 1);
    clover_d_loop(g, o, mu, nu, p, s, u, w, 0);
    clover_d_loop(g, o, nu, mu, p, -s, u, w, 0);
  }
}

/* clover_bsa.F90:28-176 w = (b^+ sigma_mu_nu a)^T for the six planes */
static void clover_bsa(const oq_geom *g, int pl, cplx *w, const cplx *b, const cplx *a) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < g->volh; i++) {
    for (int ca = 0; ca < 3; ca++) {
      cplx q1 = SP(a, 0, ca, i), q2 = SP(a, 1, ca, i), q3 = SP(a, 2, ca, i), q4 = SP(a, 3, ca, i);
      cplx a1, a2, a3, a4;
      switch (pl) {
        case 0: a1 = -q1; a2 = q2; a3 = -q3; a4 = q4; break;                                  /* 12 */
        case 1: a1 = -itimes(q2); a2 = itimes(q1); a3 = -itimes(q4); a4 = itimes(q3); break;  /* 13 */
        case 2: a1 = q4; a2 = q3; a3 = q2; a4 = q1; break;                                    /* 14 */
        case 3: a1 = -q2; a2 = -q1; a3 = -q4; a4 = -q3; break;                                /* 23 */
        case 4: a1 = -itimes(q4); a2 = itimes(q3); a3 = -itimes(q2); a4 = itimes(q1); break;  /* 24 */
        default: a1 = q3; a2 = -q4; a3 = q1; a4 = -q2;                                        /* 34 */
      }
      for (int cb = 0; cb < 3; cb++)
        M3(w + (size_t)i * 9, ca, cb) = a1 * conj(SP(b, 0, cb, i)) + a2 * conj(SP(b, 1, cb, i)) +
                                        a3 * conj(SP(b, 2, cb, i)) + a4 * conj(SP(b, 3, cb, i));
    }
  }
}

/* clover_d.F90:78-107 */
void oq_clover_dsf(const oq_geom *g, int eo, double *p, const cplx *b, const cplx *a, double s, const cplx *u) {
  cplx *w = xmalloc(sizeof(cplx) * 6 * 9 * (size_t)g->volh);
  for (int pl = 0; pl < 6; pl++) clover_bsa(g, pl, w + (size_t)pl * 9 * g->volh, b, a);
  clover_d(g, eo, p, s, u, w);
  free(w);
}

/* T(s1,c1,s2,c2,i) offset in CLOVER_FIELD_C (defs.h:76) */
#define TIDX(s1, c1, s2, c2, i) (((((size_t)(i) * 3 + (c2)) * 4 + (s2)) * 3 + (c1)) * 4 + (s1))

/* clover_d.F90:40-75 + clover_t_init.F90:28-65 + clover_ts.F90:28-176 */
void oq_clover_dsd(const oq_geom *g, int eo, double *p, const cplx *bfield, double s, const cplx *u) {
  int volh = g->volh;
  const cplx *b = bfield + (size_t)eo * volh * 36;
  cplx *t = xmalloc(sizeof(cplx) * 144 * (size_t)volh);
  cplx *x = xmalloc(sizeof(cplx) * 12 * (size_t)volh);
  for (int c2 = 0; c2 < 3; c2++)
    for (int s2 = 0; s2 < 4; s2++) {
      memset(x, 0, sizeof(cplx) * 12 * (size_t)volh);
      for (int i = 0; i < volh; i++) SP(x, s2, c2, i) = 1.0;
      oq_clover_mult_b(b, x, volh);
      for (int i = 0; i < volh; i++)
        for (int c1 = 0; c1 < 3; c1++)
          for (int s1 = 0; s1 < 4; s1++) t[TIDX(s1, c1, s2, c2, i)] = SP(x, s1, c1, i);
    }
  free(x);
  cplx *w = xmalloc(sizeof(cplx) * 6 * 9 * (size_t)volh);
  for (int pl = 0; pl < 6; pl++) {
    cplx *wp = w + (size_t)pl * 9 * volh;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < volh; i++)
      for (int c2 = 0; c2 < 3; c2++)
        for (int c1 = 0; c1 < 3; c1++) {
#define T(a_, b_) t[TIDX((a_) - 1, c1, (b_) - 1, c2, i)]
          cplx r;
          switch (pl) {
            case 0: r = -T(1, 1) + T(2, 2) - T(3, 3) + T(4, 4); break;
            case 1: r = itimes(T(1, 2)) - itimes(T(2, 1)) + itimes(T(3, 4)) - itimes(T(4, 3)); break;
            case 2: r = T(1, 4) + T(2, 3) + T(3, 2) + T(4, 1); break;
            case 3: r = -T(1, 2) - T(2, 1) - T(3, 4) - T(4, 3); break;
            case 4: r = itimes(T(1, 4)) - itimes(T(2, 3)) + itimes(T(3, 2)) - itimes(T(4, 1)); break;
            default: r = T(1, 3) - T(2, 4) + T(3, 1) - T(4, 2);
          }
#undef T
          M3(wp + (size_t)i * 9, c1, c2) = r;
        }
  }
  free(t);
  clover_d(g, eo, p, s, u, w);
  free(w);
}

/* dsf.F90:28-110 */
void oq_dsf(const oq_geom *g, double *p, const oq_conf *c, double step, const oq_hmc_para *para,
            const cplx *a, const cplx *b) {
  int volh = g->volh;
  long n = oq_sc_size(g);
  cplx *at = xmalloc(sizeof(cplx) * n), *bt = xmalloc(sizeof(cplx) * n);
  cplx *u = c->u;
  if (para->kappa != 0) {
    oq_d(g, OQ_ODD, OQ_EVEN, at, a, u);
    oq_d_dag(g, OQ_ODD, OQ_EVEN, bt, b, u);
    if (para->csw_kappa != 0) {
      oq_clover_mult_b(c->b + (size_t)OQ_ODD * volh * 36, at, volh);
      oq_clover_mult_b(c->b + (size_t)OQ_ODD * volh * 36, bt, volh);
    }
    if (para->h != 0) {
      oq_h_mult_b(-para->h, at, volh);
      oq_h_mult_b(para->h, bt, volh);
    }
  }
  double s = -step * 2.0 * para->kappa * para->kappa / (1.0 + para->h * para->h);
  if (s != 0) {
    for (int mu = 0; mu < 4; mu++) {
      const int *nne = &OQ_NN(g, 0, OQ_EVEN, mu, OQ_FWD), *nno = &OQ_NN(g, 0, OQ_ODD, mu, OQ_FWD);
      double *pe = PGEN(g, p, 0, OQ_EVEN, mu), *po = PGEN(g, p, 0, OQ_ODD, mu);
      const cplx *ue = ULINK(g, u, 0, OQ_EVEN, mu), *uo = ULINK(g, u, 0, OQ_ODD, mu);
      dsf_dir(g, pe, b, at, s, ue, nne, mu, 1);
      dsf_dir(g, po, bt, a, s, uo, nno, mu, 1);
      dsf_dir(g, pe, bt, a, s, ue, nne, mu, 0);
      dsf_dir(g, po, b, at, s, uo, nno, mu, 0);
    }
  }
  oq_flip_bc(g, u);
  double s1 = -step * 2.0 * (para->csw_kappa / 8.0);
  double s2 = -step * 2.0 * (para->csw_kappa / 8.0) * para->kappa * para->kappa;
  if (s1 != 0) oq_clover_dsf(g, OQ_EVEN, p, b, a, s1, u);
  if (s2 != 0) oq_clover_dsf(g, OQ_ODD, p, bt, at, s2, u);
  free(at);
  free(bt);
}

/* dsg.F90:28-53 */
void oq_dsg(const oq_geom *g, double *p, const cplx *u, double step, double beta) {
  if (beta == 0) return;
  double s = -step * beta / 3.0;
  for (int mu = 0; mu < 4; mu++)
    for (int eo = 0; eo < 2; eo++) {
#pragma omp parallel for schedule(static)
      for (int i = 0; i < g->volh; i++) {
        cplx uuu[9], w[9];
        staple(g, uuu, u, i, eo, mu);
        uu(w, ULINK(g, u, i, eo, mu), uuu);
        oq_im_tr_j(PGEN(g, p, i, eo, mu), w, s);
      }
    }
}

/* su3.F90:467-485 */
static double re_tr_uu(const cplx *u, const cplx *v) {
  double p = 0;
  for (int c2 = 0; c2 < 3; c2++)
    for (int c1 = 0; c1 < 3; c1++)
      p = p + creal(M3(u, c2, c1)) * creal(M3(v, c1, c2)) - cimag(M3(u, c2, c1)) * cimag(M3(v, c1, c2));
  return p;
}

/* action.F90:70-123 */
double oq_sg(const oq_geom *g, const cplx *u) {
  double plaq = 0;
  for (int mu = 0; mu < 4; mu++)
    for (int e = 0; e < 2; e++) {
      int o = 1 - e;
      for (int nu = mu + 1; nu < 4; nu++) {
        double part[OQ_NCHUNK];
        int chunk = (g->volh + OQ_NCHUNK - 1) / OQ_NCHUNK;
#pragma omp parallel for schedule(static)
        for (int ch = 0; ch < OQ_NCHUNK; ch++) {
          double pp = 0;
          for (int i = ch * chunk; i < g->volh && i < (ch + 1) * chunk; i++) {
            int j1 = OQ_NN(g, i, e, mu, OQ_FWD), j2 = OQ_NN(g, i, e, nu, OQ_FWD);
            cplx uuu[9];
            for (int k = 0; k < 9; k++) uuu[k] = 0;
            uuu_fwd(uuu, ULINK(g, u, j1, o, nu), ULINK(g, u, j2, o, mu), ULINK(g, u, i, e, nu));
            pp = pp + re_tr_uu(uuu, ULINK(g, u, i, e, mu));
          }
          part[ch] = pp;
        }
        double pp = 0;
        for (int ch = 0; ch < OQ_NCHUNK; ch++) pp += part[ch];
        plaq = plaq + pp;
      }
    }
  return (6.0 * g->volume) - plaq / 3.0;
}

/* action.F90:125-143 */
double oq_sp(const oq_geom *g, const double *p) {
  double s = 0;
  for (int mu = 0; mu < 4; mu++)
    for (int eo = 0; eo < 2; eo++) {
      const double *q = PGEN(g, p, 0, eo, mu);
      s = s + oq_dot(q, q, 8L * g->volh);
    }
  return s * 0.5;
}

/* ------------------------------------------------------------------------ */
/* MRE chronological guess (mre.F90:29-279)                                  */
/* ------------------------------------------------------------------------ */
typedef struct { int rank, nvec; cplx **vec; cplx **mv; } oq_mre;

static void mre_allocate(const oq_geom *g, oq_mre *m) {
  if (m->vec) return;
  m->vec = xcalloc(sizeof(cplx *) * m->nvec);
  m->mv = xcalloc(sizeof(cplx *) * m->nvec);
  for (int i = 0; i < m->nvec; i++) {
    m->vec[i] = xcalloc(sizeof(cplx) * oq_sc_size(g));
    m->mv[i] = xcalloc(sizeof(cplx) * oq_sc_size(g));
  }
  m->rank = 0;
}
static void mre_free(oq_mre *m) {
  if (!m->vec) return;
  for (int i = 0; i < m->nvec; i++) { free(m->vec[i]); free(m->mv[i]); }
  free(m->vec); free(m->mv);
  m->vec = m->mv = NULL;
}

/* mre.F90:29-66 */
static void mre_put(const oq_geom *g, oq_mre *m, const cplx *sc, int reset) {
  if (m->nvec == 0) return;
  mre_allocate(g, m);
  if (reset) { m->rank = 0; return; }
  cplx *tmp = m->vec[m->nvec - 1];
  for (int i = m->nvec - 1; i >= 1; i--) m->vec[i] = m->vec[i - 1];
  m->vec[0] = tmp;
  sc_copy((double *)m->vec[0], (const double *)sc, 2 * oq_sc_size(g));
  if (m->rank < m->nvec) m->rank++;
}

/* mre.F90:189-213 */
static void mre_gram_schmidt(const oq_geom *g, oq_mre *m) {
  long n = 2 * oq_sc_size(g);
  for (int k = 0; k < m->rank; k++) {
    double *vk = (double *)m->vec[k];
    double rkk = oq_dot(vk, vk, n);
    rkk = 1.0 / sqrt(rkk);
    sc_scale(vk, rkk, n);
    for (int j = k + 1; j < m->rank; j++) {
      double rkj = oq_dot(vk, (double *)m->vec[j], n);
      sc_axpy((double *)m->vec[j], vk, -rkj, n);
    }
  }
}

/* mre.F90:215-279 (Gauss-Jordan with full pivoting, NR style) */
static int mre_gauss_jordan(cplx *a, cplx *b, int n, int np) {
#define GA(j, k) a[(size_t)(k) * np + (j)]
  int ipiv[64] = {0};
  int irow = 0, icol = 0;
  for (int i = 0; i < n; i++) {
    double big = 0;
    for (int j = 0; j < n; j++)
      if (ipiv[j] != 1)
        for (int k = 0; k < n; k++) {
          if (ipiv[k] == 0) {
            double tmp = cabs(GA(j, k));
            if (tmp >= big) { big = tmp; irow = j; icol = k; }
          } else if (ipiv[k] > 1) return -1;
        }
    ipiv[icol]++;
    if (irow != icol) {
      for (int l = 0; l < n; l++) { cplx d = GA(irow, l); GA(irow, l) = GA(icol, l); GA(icol, l) = d; }
      cplx d = b[irow]; b[irow] = b[icol]; b[icol] = d;
    }
    if (GA(icol, icol) == 0) return -2;
    cplx pivinv = 1.0 / GA(icol, icol);
    for (int l = 0; l < n; l++) GA(icol, l) = GA(icol, l) * pivinv;
    b[icol] = b[icol] * pivinv;
    for (int ll = 0; ll < n; ll++)
      if (ll != icol) {
        cplx dum = GA(ll, icol);
        GA(ll, icol) = 0;
        for (int l = 0; l < n; l++) GA(ll, l) = GA(ll, l) - GA(icol, l) * dum;
        b[ll] = b[ll] - b[icol] * dum;
      }
  }
#undef GA
  return 0;
}

/* mre.F90:68-146 */
static void mre_get(const oq_geom *g, oq_mre *m, oq_matrix_mult mm, cplx *trial, const cplx *phi,
                    const oq_hmc_para *p, const oq_conf *c) {
  long nc = oq_sc_size(g);
  if (m->nvec == 0 || !m->vec || m->rank == 0) { sc_copy((double *)trial, (const double *)phi, 2 * nc); return; }
  if (m->rank == 1) { sc_copy((double *)trial, (const double *)m->vec[0], 2 * nc); return; }
  int np = m->nvec;
  cplx *ga = xcalloc(sizeof(cplx) * (size_t)np * (np + 1));
  cplx *bb = ga + (size_t)np * np;
  mre_gram_schmidt(g, m);
  for (int i = 0; i < m->rank; i++) {
    bb[i] = oq_cdotc(m->vec[i], phi, nc);
    mm(g, m->mv[i], m->vec[i], p, c);
  }
  for (int i = 0; i < m->rank; i++) {
    ga[(size_t)i * np + i] = oq_dot((double *)m->mv[i], (double *)m->mv[i], 2 * nc);
    for (int j = i + 1; j < m->rank; j++) {
      ga[(size_t)j * np + i] = oq_cdotc(m->mv[i], m->mv[j], nc);
      ga[(size_t)i * np + j] = conj(ga[(size_t)j * np + i]);
    }
  }
  if (mre_gauss_jordan(ga, bb, m->rank, np) != 0) {
    fprintf(stderr, "oracle: mre_gauss_jordan(): singular matrix\n");
    abort();
  }
  cplx a1 = bb[0], a2 = bb[1];
  const cplx *v1 = m->vec[0], *v2 = m->vec[1];
#pragma omp parallel for schedule(static)
  for (long k = 0; k < nc; k++) trial[k] = a1 * v1[k] + a2 * v2[k];
  int rest = m->rank % 2;
  for (int j = 3; j <= m->rank - rest; j += 2) {
    cplx b1 = bb[j - 1], b2 = bb[j];
    const cplx *w1 = m->vec[j - 1], *w2 = m->vec[j];
#pragma omp parallel for schedule(static)
    for (long k = 0; k < nc; k++) trial[k] = trial[k] + b1 * w1[k] + b2 * w2[k];
  }
  if (rest == 1) {
    int j = m->rank - 1;
    cplx b1 = bb[j];
    const cplx *w1 = m->vec[j];
#pragma omp parallel for schedule(static)
    for (long k = 0; k < nc; k++) trial[k] = trial[k] + b1 * w1[k];
  }
  free(ga);
}

/* ------------------------------------------------------------------------ */
/* HMC (hmc.F90, hmc_leap_frog.F90, hmc_integrator.F90, dsf1/dsf2, ...)       */
/* ------------------------------------------------------------------------ */
enum { I_SG = 0, I_SD = 1, I_SF1 = 2, I_SF2 = 3 };

typedef struct {
  oq_run *r;
  double *p, *p_old;
  oq_cg_stat st;
  oq_mre mre1, mre2;
  int it_f1, it_f2;
  double f_count[4], f_avg[4], f_max[4];
  int hasenbusch;
} hmc_state;

static hmc_state *g_state;  /* the MRE bases persist across trajectories like Fortran save variables */

static void forces_old(hmc_state *s) {
  if (!s->hasenbusch) return;
  memcpy(s->p_old, s->p, sizeof(double) * oq_gen_size(&s->r->geom));
}

/* hmc_forces.F90:65-104 */
static void forces_new(hmc_state *s, double step, int which) {
  if (!s->hasenbusch) return;
  const oq_geom *g = &s->r->geom;
  long n = oq_gen_size(g);
  double f = 0;
  for (long k = 0; k < n; k++) {
    double d = s->p_old[k] - s->p[k];
    f = f + d * d;
  }
  f = f / (8.0 * g->volume * 4.0);
  f = sqrt(f) / fabs(step);
  s->f_count[which] += 1.0;
  s->f_avg[which] += f;
  if (f > s->f_max[which]) s->f_max[which] = f;
}

static int solve_or_die(hmc_state *s, oq_matrix_mult mm, cplx *x, const cplx *b, int *iters) {
  oq_run *r = s->r;
  int rc = oq_cg(&r->geom, mm, x, b, &r->para, &r->conf, &r->cg, &s->st, iters, NULL);
  if (rc) { fprintf(stderr, "oracle: cg(): no convergence\n"); abort(); }
  return rc;
}

/* dsf1.F90:28-82 */
static void dsf1(hmc_state *s, double step, int calc_sf, double *sf) {
  oq_run *r = s->r;
  const oq_geom *g = &r->geom;
  long n = oq_sc_size(g);
  *sf = 0;
  cplx *a = xmalloc(sizeof(cplx) * n), *b = xmalloc(sizeof(cplx) * n);
  oq_flip_bc(g, r->conf.u);
  mre_get(g, &s->mre1, oq_w_mult, a, r->conf.phi, &r->para, &r->conf);
  int iters;
  solve_or_die(s, oq_w_dagger_w, a, r->conf.phi, &iters);
  mre_put(g, &s->mre1, a, calc_sf);
  oq_w_mult(g, b, a, &r->para, &r->conf);
  if (calc_sf) *sf = oq_dot((double *)b, (double *)b, 2 * n);
  forces_old(s);
  oq_dsf(g, s->p, &r->conf, step, &r->para, a, b);
  forces_new(s, step, I_SF1);
  s->it_f1 += iters;
  free(a);
  free(b);
}

/* dsf2.F90:28-80 */
static void dsf2(hmc_state *s, double step, int calc_sf, double *sf) {
  oq_run *r = s->r;
  const oq_geom *g = &r->geom;
  long n = oq_sc_size(g);
  *sf = 0;
  if (!s->hasenbusch) return;
  cplx *a = xmalloc(sizeof(cplx) * n), *b = xmalloc(sizeof(cplx) * n);
  oq_flip_bc(g, r->conf.u);
  oq_w_mult_dag(g, b, r->conf.phi2, &r->para, &r->conf);
  mre_get(g, &s->mre2, oq_mtil, a, b, &r->para, &r->conf);
  int iters;
  solve_or_die(s, oq_mtdagmt, a, b, &iters);
  mre_put(g, &s->mre2, a, calc_sf);
  oq_mtil(g, b, a, &r->para, &r->conf);
  if (calc_sf) *sf = oq_dot((double *)b, (double *)b, 2 * n);
  sc_axpy((double *)b, (const double *)r->conf.phi2, -1.0, 2 * n);
  forces_old(s);
  oq_dsf(g, s->p, &r->conf, step, &r->para, a, b);
  forces_new(s, step, I_SF2);
  s->it_f2 += iters;
  free(a);
  free(b);
}

/* dsd.F90:28-49 */
static void dsd(hmc_state *s, double step) {
  oq_run *r = s->r;
  double sd = -step * 2.0 * (r->para.csw_kappa / 8.0);
  if (sd != 0) {
    forces_old(s);
    oq_clover_dsd(&r->geom, OQ_ODD, s->p, r->conf.b, sd, r->conf.u);
    forces_new(s, step, I_SD);
  }
}

static void dsg_mon(hmc_state *s, double step) {
  oq_run *r = s->r;
  if (r->para.beta == 0) return;
  forces_old(s);
  oq_dsg(&r->geom, s->p, r->conf.u, step, r->para.beta);
  forces_new(s, step, I_SG);
}

/* hmc_u.F90:28-69 */
static void hmc_u(hmc_state *s, double step) {
  oq_run *r = s->r;
  const oq_geom *g = &r->geom;
  for (int mu = 0; mu < 4; mu++)
    for (int eo = 0; eo < 2; eo++) {
#pragma omp parallel for schedule(static)
      for (int i = 0; i < g->volh; i++) {
        double q[8];
        cplx v[9], w[9];
        const double *pp = PGEN(g, s->p, i, eo, mu);
        for (int j = 0; j < 8; j++) q[j] = pp[j] * step;
        oq_gen2u(v, q);
        cplx *l = ULINK(g, r->conf.u, i, eo, mu);
        memcpy(w, l, sizeof w);
        uu(l, v, w);
        oq_u_normalize(l);
      }
    }
  if (r->conf.a)
    oq_clover_init(g, r->conf.a, r->conf.i, r->conf.b, r->conf.u, r->para.csw_kappa);
}

/* hmc_integrator.F90:28-85 */
static void p_ir(hmc_state *s, double step, int calc_sf, double *sf1, double *sf2) {
  switch (s->r->para.model) {
    case 'A': dsf1(s, step, calc_sf, sf1); dsd(s, step); break;
    case 'B': dsf1(s, step, calc_sf, sf1); dsf2(s, step, calc_sf, sf2); dsd(s, step); break;
    default: dsf2(s, step, calc_sf, sf2);
  }
}
static void p_uv(hmc_state *s, double step, int calc_sf, double *sf1, double *sf2) {
  (void)sf2;
  switch (s->r->para.model) {
    case 'A':
    case 'B': dsg_mon(s, step); break;
    default: dsg_mon(s, step); dsf1(s, step, calc_sf, sf1); dsd(s, step);
  }
}

/* hmc_leap_frog.F90:28-79 */
static void leap_frog(hmc_state *s, double *sf1, double *sf2) {
  const oq_hmc_para *pa = &s->r->para;
  int calc_sf = 0;
  double step_ir = 0.5 * pa->tau, step_uv = 0.5 * pa->tau / pa->m_scale;
  p_ir(s, step_ir, calc_sf, sf1, sf2);
  p_uv(s, step_uv, calc_sf, sf1, sf2);
  step_ir = pa->tau;
  step_uv = pa->tau / pa->m_scale;
  for (int itau = 1; itau <= pa->ntau; itau++) {
    for (int is = 1; is <= pa->m_scale; is++) {
      hmc_u(s, step_uv);
      if (itau == pa->ntau && is == pa->m_scale) {
        step_ir = step_ir * 0.5;
        step_uv = step_uv * 0.5;
        calc_sf = 1;
      }
      p_uv(s, step_uv, calc_sf, sf1, sf2);
    }
    p_ir(s, step_ir, calc_sf, sf1, sf2);
  }
}

/* hmc_init_phi.F90:28-79 */
static void init_phi(hmc_state *s, double *sf1, double *sf2) {
  oq_run *r = s->r;
  const oq_geom *g = &r->geom;
  long n = oq_sc_size(g);
  *sf1 = 0;
  *sf2 = 0;
  cplx *tmp = xmalloc(sizeof(cplx) * n);
  oq_flip_bc(g, r->conf.u);
  oq_ran_gauss_volh(g, 12, tmp, 0.5, OQ_EVEN);
  *sf1 = oq_dot((double *)tmp, (double *)tmp, 2 * n);
  oq_w_mult_dag(g, r->conf.phi, tmp, &r->para, &r->conf);
  if (s->hasenbusch) {
    oq_ran_gauss_volh(g, 12, tmp, 0.5, OQ_EVEN);
    *sf2 = oq_dot((double *)tmp, (double *)tmp, 2 * n);
    oq_mtil_dag(g, r->conf.phi2, tmp, &r->para, &r->conf);
    int iters;
    solve_or_die(s, oq_w_dagger_w, tmp, r->conf.phi2, &iters);
    oq_w_mult(g, r->conf.phi2, tmp, &r->para, &r->conf);
  }
  oq_flip_bc(g, r->conf.u);
  free(tmp);
}

int oq_run_init(oq_run *r, const int L[4], const int bc[4], const oq_hmc_para *p, int cold, int64_t seed,
                float rest, int maxiter, int log, int mre_n_vec) {
  memset(r, 0, sizeof(*r));
  if (oq_geom_init(&r->geom, L, bc)) return -1;
  r->para = *p;
  r->cg.rest = rest;
  r->cg.maxiter = maxiter;
  r->cg.log = log;
  r->mre_n_vec = mre_n_vec;
  oq_ranset(seed, 0);
  const oq_geom *g = &r->geom;
  r->conf.u = xmalloc(sizeof(cplx) * oq_gauge_size(g));
  r->conf.phi = xcalloc(sizeof(cplx) * oq_sc_size(g));
  r->conf.phi2 = xcalloc(sizeof(cplx) * oq_sc_size(g));
  if (cold) oq_conf_cold(g, r->conf.u);
  else oq_conf_hot(g, r->conf.u);
  if (p->csw_kappa != 0) {
    r->conf.a = xmalloc(sizeof(cplx) * oq_clover_size(g));
    r->conf.i = xmalloc(sizeof(cplx) * oq_clover_size(g));
    r->conf.b = xmalloc(sizeof(cplx) * oq_clover_size(g));
    oq_clover_init(g, r->conf.a, r->conf.i, r->conf.b, r->conf.u, p->csw_kappa);
  }
  return 0;
}

void oq_run_free(oq_run *r) {
  if (g_state && g_state->r == r) {
    mre_free(&g_state->mre1);
    mre_free(&g_state->mre2);
    free(g_state->p);
    free(g_state->p_old);
    free(g_state);
    g_state = NULL;
  }
  free(r->conf.u); free(r->conf.phi); free(r->conf.phi2);
  free(r->conf.a); free(r->conf.i); free(r->conf.b);
  oq_geom_free(&r->geom);
  memset(r, 0, sizeof(*r));
}

/* hmc.F90:69-216 (test = HMC_TEST_NONE) */
void oq_hmc(oq_run *r, oq_hmc_out *out, int force_accept) {
  const oq_geom *g = &r->geom;
  if (!g_state || g_state->r != r) {
    g_state = xcalloc(sizeof(hmc_state));
    g_state->r = r;
    g_state->p = xcalloc(sizeof(double) * oq_gen_size(g));
    g_state->p_old = xcalloc(sizeof(double) * oq_gen_size(g));
    g_state->mre1.nvec = r->mre_n_vec;
    g_state->mre2.nvec = r->mre_n_vec;
  }
  hmc_state *s = g_state;
  s->hasenbusch = r->para.model != 'A';
  memset(&s->st, 0, sizeof(s->st));
  long nsc = oq_sc_size(g), ng = oq_gauge_size(g), ncl = oq_clover_size(g);
  cplx *u_bck = xmalloc(sizeof(cplx) * ng), *phi_bck = xmalloc(sizeof(cplx) * nsc);
  cplx *a_bck = NULL, *i_bck = NULL, *b_bck = NULL;
  memcpy(u_bck, r->conf.u, sizeof(cplx) * ng);
  memcpy(phi_bck, r->conf.phi, sizeof(cplx) * nsc);
  if (r->conf.a) {
    a_bck = xmalloc(sizeof(cplx) * ncl); i_bck = xmalloc(sizeof(cplx) * ncl); b_bck = xmalloc(sizeof(cplx) * ncl);
    memcpy(a_bck, r->conf.a, sizeof(cplx) * ncl);
    memcpy(i_bck, r->conf.i, sizeof(cplx) * ncl);
    memcpy(b_bck, r->conf.b, sizeof(cplx) * ncl);
  }
  /* hmc_init_p.F90:28-45 */
  for (int mu = 0; mu < 4; mu++)
    for (int eo = 0; eo < 2; eo++) oq_ran_gauss_volh(g, 4, (cplx *)PGEN(g, s->p, 0, eo, mu), 1.0, eo);
  double sf1_old, sf2_old;
  init_phi(s, &sf1_old, &sf2_old);
  double sd_old = r->conf.b ? oq_clover_action(r->conf.b + (size_t)OQ_ODD * g->volh * 36, g->volh) : 0;
  double sg_old = oq_sg(g, r->conf.u);
  double sp_old = oq_sp(g, s->p);
  double hg_old = sg_old * r->para.beta;
  double h_old = sd_old + sp_old + hg_old + sf1_old + sf2_old;

  double sf1 = 0, sf2 = 0;
  leap_frog(s, &sf1, &sf2);

  double sd_new = r->conf.b ? oq_clover_action(r->conf.b + (size_t)OQ_ODD * g->volh * 36, g->volh) : 0;
  double sg_new = oq_sg(g, r->conf.u);
  double sp_new = oq_sp(g, s->p);
  double hg_new = sg_new * r->para.beta;
  double h_new = sd_new + sp_new + hg_new + sf1 + sf2;
  out->exp_dh = exp(h_old - h_new);
  if (force_accept) out->accepted = 1;
  else out->accepted = oq_ranf() < out->exp_dh ? 1 : 0;
  if (out->accepted) {
    out->sg = sg_new;
    out->sf = sf1;
  } else {
    memcpy(r->conf.u, u_bck, sizeof(cplx) * ng);
    memcpy(r->conf.phi, phi_bck, sizeof(cplx) * nsc);
    if (r->conf.a) {
      memcpy(r->conf.a, a_bck, sizeof(cplx) * ncl);
      memcpy(r->conf.i, i_bck, sizeof(cplx) * ncl);
      memcpy(r->conf.b, b_bck, sizeof(cplx) * ncl);
    }
  }
  out->cg_ncall = s->st.ncall;
  out->cg_niter_max = s->st.niter_max;
  out->cg_niter_tot = s->st.niter_tot;
  out->it_f1 = s->it_f1;
  out->it_f2 = s->it_f2;
  for (int k = 0; k < 4; k++) {
    out->f_avg[k] = s->f_count[k] != 0 ? s->f_avg[k] / s->f_count[k] : s->f_avg[k];
    out->f_max[k] = s->f_max[k];
  }
  /* iteration_count_write / hmc_forces_write reset the monitors */
  s->it_f1 = s->it_f2 = 0;
  for (int k = 0; k < 4; k++) s->f_count[k] = s->f_avg[k] = s->f_max[k] = 0;
  free(u_bck); free(phi_bck); free(a_bck); free(i_bck); free(b_bck);
}
