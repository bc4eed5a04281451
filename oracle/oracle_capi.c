/*
 * oracle_capi.c -- flat entry points over the CPU oracle for the Python test
 * harness (ctypes).  Test infrastructure only: the product library never links
 * this.  Arrays use the reference's Fortran layouts (see bqcd_oracle.h).
 */
#include <stdlib.h>
#include <string.h>

#include "bqcd_oracle.h"

oq_geom *oqc_geom_new(const int L[4], const int bc[4]) {
  oq_geom *g = malloc(sizeof(oq_geom));
  if (!g) return NULL;
  if (oq_geom_init(g, L, bc)) {
    free(g);
    return NULL;
  }
  return g;
}
void oqc_geom_delete(oq_geom *g) {
  if (!g) return;
  oq_geom_free(g);
  free(g);
}
int oqc_volh(const oq_geom *g) { return g->volh; }
const int *oqc_nn(const oq_geom *g) { return g->nn; }
int oqc_threads(void) { return oq_num_threads(); }

void oqc_ranset(long long seed, long long skip) { oq_ranset(seed, skip); }
long long oqc_ranget(void) {
  int64_t s;
  oq_ranget(&s);
  return (long long)s;
}
double oqc_ranf(void) { return oq_ranf(); }
void oqc_ran_gauss_volh(const oq_geom *g, int m, double *ran, double var, int eo) {
  oq_ran_gauss_volh(g, m, (oq_cplx *)ran, var, eo);
}
void oqc_conf_hot(const oq_geom *g, double *u) { oq_conf_hot(g, (oq_cplx *)u); }
void oqc_conf_cold(const oq_geom *g, double *u) { oq_conf_cold(g, (oq_cplx *)u); }
void oqc_conf_relax(const oq_geom *g, double *u) { oq_conf_relax(g, (oq_cplx *)u); }
void oqc_flip_bc(const oq_geom *g, double *u) { oq_flip_bc(g, (oq_cplx *)u); }
double oqc_sg(const oq_geom *g, const double *u) { return oq_sg(g, (const oq_cplx *)u); }
void oqc_gen2u(double *u, const double *h) { oq_gen2u((oq_cplx *)u, h); }

void oqc_d(const oq_geom *g, int e, int o, double *out, const double *in, const double *u, int dag) {
  if (dag) oq_d_dag(g, e, o, (oq_cplx *)out, (const oq_cplx *)in, (const oq_cplx *)u);
  else oq_d(g, e, o, (oq_cplx *)out, (const oq_cplx *)in, (const oq_cplx *)u);
}

void oqc_clover_init(const oq_geom *g, double *a, double *ainv, double *b, const double *u, double csw_kappa) {
  oq_clover_init(g, (oq_cplx *)a, (oq_cplx *)ainv, (oq_cplx *)b, (const oq_cplx *)u, csw_kappa);
}
/* which: 0 mult_a (out = A in), 1 mult_ao (in place), 2 mult_b (in place) */
void oqc_clover_mult(const oq_geom *g, int which, const double *blk, double *out, const double *in) {
  if (which == 0) oq_clover_mult_a((oq_cplx *)out, (const oq_cplx *)blk, (const oq_cplx *)in, g->volh);
  else {
    memcpy(out, in, sizeof(double) * 24 * (size_t)g->volh);
    if (which == 1) oq_clover_mult_ao((const oq_cplx *)blk, (oq_cplx *)out, g->volh);
    else oq_clover_mult_b((const oq_cplx *)blk, (oq_cplx *)out, g->volh);
  }
}
double oqc_clover_action(const oq_geom *g, const double *b) { return oq_clover_action((const oq_cplx *)b, g->volh); }

static void mkpara(oq_hmc_para *p, double kappa, double csw_kappa, double h, double rho) {
  memset(p, 0, sizeof *p);
  p->kappa = kappa;
  p->csw_kappa = csw_kappa;
  p->h = h;
  p->rho = rho;
}
static void mkconf(oq_conf *c, const double *u, const double *a, const double *ainv, const double *b) {
  memset(c, 0, sizeof *c);
  c->u = (oq_cplx *)u;
  c->a = (oq_cplx *)a;
  c->i = (oq_cplx *)ainv;
  c->b = (oq_cplx *)b;
}
static oq_matrix_mult op_of(int which) {
  switch (which) {
    case 0: return oq_mtil;
    case 1: return oq_mtil_dag;
    case 2: return oq_mtdagmt;
    case 3: return oq_w_mult;
    case 4: return oq_w_mult_dag;
    default: return oq_w_dagger_w;
  }
}

/* which: 0 mtil 1 mtil_dag 2 mtdagmt 3 w_mult 4 w_mult_dag 5 w_dagger_w */
void oqc_op(const oq_geom *g, int which, double *out, const double *in, const double *u, const double *a,
            const double *ainv, const double *b, double kappa, double csw_kappa, double h, double rho) {
  oq_hmc_para p;
  oq_conf c;
  mkpara(&p, kappa, csw_kappa, h, rho);
  mkconf(&c, u, a, ainv, b);
  op_of(which)(g, (oq_cplx *)out, (const oq_cplx *)in, &p, &c);
}

/* cg(matrix_mult = mtdagmt (which 2) or w_dagger_w (which 5), x, b) */
int oqc_cg(const oq_geom *g, int which, double *x, const double *bvec, const double *u, const double *a,
           const double *ainv, const double *b, double kappa, double csw_kappa, double h, double rho, float rest,
           int maxiter, int log, int *iters, double *rtr) {
  oq_hmc_para p;
  oq_conf c;
  oq_cg_para cp = {rest, maxiter, log};
  mkpara(&p, kappa, csw_kappa, h, rho);
  mkconf(&c, u, a, ainv, b);
  return oq_cg(g, op_of(which), (oq_cplx *)x, (const oq_cplx *)bvec, &p, &c, &cp, NULL, iters, rtr);
}

/* dsf(p, conf, step, para, a, b): u is modified by flip_bc inside, as in the
 * reference (the caller passes flipped links and gets them back unflipped) */
void oqc_dsf(const oq_geom *g, double *pgen, double *u, const double *a, const double *ainv, const double *b,
             double step, double kappa, double csw_kappa, double h, const double *af, const double *bf) {
  oq_hmc_para p;
  oq_conf c;
  mkpara(&p, kappa, csw_kappa, h, 0.0);
  mkconf(&c, u, a, ainv, b);
  oq_dsf(g, pgen, &c, step, &p, (const oq_cplx *)af, (const oq_cplx *)bf);
}
void oqc_clover_dsf(const oq_geom *g, int eo, double *pgen, const double *bf, const double *af, double s,
                    const double *u) {
  oq_clover_dsf(g, eo, pgen, (const oq_cplx *)bf, (const oq_cplx *)af, s, (const oq_cplx *)u);
}
void oqc_clover_dsd(const oq_geom *g, int eo, double *pgen, const double *bfield, double s, const double *u) {
  oq_clover_dsd(g, eo, pgen, (const oq_cplx *)bfield, s, (const oq_cplx *)u);
}
void oqc_dsg(const oq_geom *g, double *pgen, const double *u, double step, double beta) {
  oq_dsg(g, pgen, (const oq_cplx *)u, step, beta);
}

/* ---- configuration files: the check sum of cksum.c ---------------------
 * POSIX.2 cksum (cksum.c:60-165): CRC with the generator polynomial
 * 0x04C11DB7, most significant bit first, register starting at 0; after
 * the data the byte count is fed in, least significant byte first, until
 * it is exhausted; the result is the complement of the low 32 bits.  The
 * byte table is generated here from the polynomial. */
static unsigned int oqc_crc_tab[256];
static int oqc_crc_ready = 0;

static void oqc_crc_init(void) {
  for (unsigned int b = 0; b < 256; b++) {
    unsigned int r = b << 24;
    for (int k = 0; k < 8; k++) r = (r & 0x80000000u) ? (r << 1) ^ 0x04C11DB7u : (r << 1);
    oqc_crc_tab[b] = r;
  }
  oqc_crc_ready = 1;
}

/* raw register after n bytes, continuing from crc */
unsigned int oqc_crc_update(unsigned int crc, const unsigned char* p, long long n) {
  if (!oqc_crc_ready) oqc_crc_init();
  for (long long k = 0; k < n; k++) crc = (crc << 8) ^ oqc_crc_tab[((crc >> 24) ^ p[k]) & 0xFFu];
  return crc;
}

/* the cksum value of n bytes */
unsigned int oqc_cksum(const unsigned char* p, long long n) {
  unsigned int crc = oqc_crc_update(0u, p, n);
  for (long long len = n; len > 0; len >>= 8) {
    unsigned char b = (unsigned char)(len & 0xFF);
    crc = oqc_crc_update(crc, &b, 1);
  }
  return ~crc;
}
