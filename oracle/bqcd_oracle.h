/*
 * bqcd_oracle.h -- CPU restatement of BQCD's (benchmark2, svn r399) fermion
 * hot path, used ONLY as test infrastructure: the parity checker for the CUDA
 * path, the golden-run reproducer and the timed CPU baseline.  Nothing in the
 * product library links or calls this code.
 *
 * Memory layouts are the reference's Fortran (column-major) layouts, 0-based:
 *   spinor   SPINCOL_FIELD  complex(4,3,volh)        -> cplx[volh][3][4]
 *   gauge    GAUGE_FIELD    complex(3,3,volh,0:1,4)  -> cplx[4][2][volh][3(col)][3(row)]
 *   clover   CLOVER_FIELD_A/B type(...)(2,volh,0:1)  -> cplx[2(eo)][volh][2(chi)][18]
 *   momenta  GENERATOR_FIELD real(8,volh,0:1,4)      -> double[4][2][volh][8]
 *   nn       nn(volh,0:1,4,0:1)                      -> int[2(fb)][4(mu)][2(eo)][volh]
 * (defs.h:64-78, modules/typedef_clover.F90:30-93, clover/clover.h:28-82).
 *
 * Pinned against the reference's own golden outputs: ranf_test.reference
 * (bit-exact RNG) and work/out.quick-test.reference (a full 4^4 HMC trajectory:
 * CG iteration counts, force norms, plaquette and exp(-dH)).
 */
#ifndef BQCD_ORACLE_H
#define BQCD_ORACLE_H

#include <complex.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double _Complex oq_cplx;

enum { OQ_EVEN = 0, OQ_ODD = 1, OQ_FWD = 0, OQ_BWD = 1 };

/* lattice geometry, single process (init_common.F90:43-205, index.F90) */
typedef struct {
  int L[4];       /* extents x,y,z,t */
  int bc[4];      /* fermion boundary conditions (+1 / -1) */
  int volume;
  int volh;
  int *nn;        /* nn[((fb*4+mu)*2+eo)*volh + i] */
  int *coord;     /* coord[(eo*volh+i)*4 + mu] */
  int flip_len[4];
  int *flip_list; /* flip_list[(mu*2+eo)*volh + k] */
} oq_geom;

/* type(hmc_para) (modules/typedef_hmc.F90:32-44) */
typedef struct {
  double beta, kappa, csw, csw_kappa, h, traj_length, tau, rho;
  int ntau, m_scale;
  char model;
} oq_hmc_para;

/* type(hmc_conf) (modules/typedef_hmc.F90:69-77) */
typedef struct {
  oq_cplx *u, *phi, *phi2, *a, *i, *b;
} oq_conf;

/* CG parameters and statistics (cg.F90:28-48) */
typedef struct { float rest; int maxiter; int log; } oq_cg_para;
typedef struct { int niter, niter_max, niter_tot, ncall; } oq_cg_stat;

/* geometry */
int  oq_geom_init(oq_geom *g, const int L[4], const int bc[4]);
void oq_geom_free(oq_geom *g);
int  oq_ieo(const oq_geom *g, const int x[4]);   /* ilex/2 (index.F90:58-76) */
int  oq_parity(const int x[4]);                  /* (x+y+z+t) mod 2 */
#define OQ_NN(g, i, eo, mu, fb) ((g)->nn[((((fb) * 4 + (mu)) * 2 + (eo)) * (g)->volh) + (i)])

/* sizes in complex numbers */
long oq_sc_size(const oq_geom *g);      /* 12*volh */
long oq_gauge_size(const oq_geom *g);   /* 72*volh */
long oq_clover_size(const oq_geom *g);  /* 72*volh (2 eo * 2 chi * 18) */
long oq_gen_size(const oq_geom *g);     /* 64*volh doubles */

/* RNG (ranf.F90, ran.F90) */
double oq_ranf(void);
void   oq_ranget(int64_t *seed);
void   oq_ranset(int64_t seed, int64_t n_skip);
void   oq_ran_gauss_volh(const oq_geom *g, int m, oq_cplx *ran, double var, int eo);

/* SU(3) helpers (su3.F90) */
void oq_u_normalize(oq_cplx *u);
void oq_gen2u(oq_cplx *u, const double *h);
void oq_im_tr_j(double *p, const oq_cplx *u, double s);
void oq_re_tr_j(double *p, const oq_cplx *u, double s);

/* gauge configurations (conf.F90:172-217, cooling.F90:131-193, flip_bc.F90) */
void oq_conf_cold(const oq_geom *g, oq_cplx *u);
void oq_conf_hot(const oq_geom *g, oq_cplx *u);
void oq_conf_relax(const oq_geom *g, oq_cplx *u);
void oq_flip_bc(const oq_geom *g, oq_cplx *u);

/* D-slash, libd21 (d/D21.F90, d/D21xyzt.F90): out(e) = D_eo in(o) */
void oq_d(const oq_geom *g, int e, int o, oq_cplx *out, const oq_cplx *in, const oq_cplx *u);
void oq_d_dag(const oq_geom *g, int e, int o, oq_cplx *out, const oq_cplx *in, const oq_cplx *u);

/* clover (clover/ *.F90).  a, ainv, b: full fields [2 eo][volh][2][18] */
void oq_clover_init(const oq_geom *g, oq_cplx *a, oq_cplx *ainv, oq_cplx *b,
                    const oq_cplx *u, double csw_kappa);
void oq_clover_mult_a(oq_cplx *out, const oq_cplx *a, const oq_cplx *in, int volh);
void oq_clover_mult_ao(const oq_cplx *a, oq_cplx *x, int volh);
void oq_clover_mult_b(const oq_cplx *b, oq_cplx *x, int volh);
double oq_clover_action(const oq_cplx *b, int volh);

/* h_mult (h_mult.F90) */
void oq_h_mult_a(oq_cplx *out, double h, const oq_cplx *in, int volh);
void oq_h_mult_b(double h, oq_cplx *x, int volh);

/* even-odd operators (m_tilde.F90, mtdagmt.F90, w_mult.F90) */
typedef void (*oq_matrix_mult)(const oq_geom *, oq_cplx *out, const oq_cplx *in,
                               const oq_hmc_para *, const oq_conf *);
void oq_mtil(const oq_geom *g, oq_cplx *out, const oq_cplx *in, const oq_hmc_para *p, const oq_conf *c);
void oq_mtil_dag(const oq_geom *g, oq_cplx *out, const oq_cplx *in, const oq_hmc_para *p, const oq_conf *c);
void oq_mtdagmt(const oq_geom *g, oq_cplx *out, const oq_cplx *in, const oq_hmc_para *p, const oq_conf *c);
void oq_w_mult(const oq_geom *g, oq_cplx *out, const oq_cplx *in, const oq_hmc_para *p, const oq_conf *c);
void oq_w_mult_dag(const oq_geom *g, oq_cplx *out, const oq_cplx *in, const oq_hmc_para *p, const oq_conf *c);
void oq_w_dagger_w(const oq_geom *g, oq_cplx *out, const oq_cplx *in, const oq_hmc_para *p, const oq_conf *c);

/* BLAS-1 on real-overindexed spinor fields (sc.F90); n = number of doubles */
double oq_dot(const double *x, const double *y, long n);

/* CG (cg.F90:51-137).  Returns 0 on convergence, 1 on no convergence. */
int oq_cg(const oq_geom *g, oq_matrix_mult mm, oq_cplx *x, const oq_cplx *b,
          const oq_hmc_para *p, const oq_conf *c, const oq_cg_para *cp,
          oq_cg_stat *st, int *iterations, double *rtr_out);

/* fermion forces (dsf.F90, d/DSFxyzt.F90, clover/clover_d.F90) */
void oq_dsf(const oq_geom *g, double *p, const oq_conf *c, double step,
            const oq_hmc_para *para, const oq_cplx *a, const oq_cplx *b);
void oq_clover_dsf(const oq_geom *g, int eo, double *p, const oq_cplx *b,
                   const oq_cplx *a, double s, const oq_cplx *u);
void oq_clover_dsd(const oq_geom *g, int eo, double *p, const oq_cplx *bfield,
                   double s, const oq_cplx *u);
void oq_dsg(const oq_geom *g, double *p, const oq_cplx *u, double step, double beta);

/* actions (action.F90) */
double oq_sg(const oq_geom *g, const oq_cplx *u);
double oq_sp(const oq_geom *g, const double *p);

/* HMC (hmc.F90) for the golden quick-test; prints the reference's
 * %it / %Favg / %Fmax / %fa records to stdout */
typedef struct {
  double exp_dh, sg, sf;
  int accepted, cg_ncall, cg_niter_max, cg_niter_tot;
  int it_f1, it_f2;
  double f_avg[4], f_max[4];
} oq_hmc_out;

typedef struct {
  oq_geom geom;
  oq_hmc_para para;
  oq_conf conf;
  oq_cg_para cg;
  int mre_n_vec;
} oq_run;

int  oq_run_init(oq_run *r, const int L[4], const int bc[4], const oq_hmc_para *p,
                 int cold, int64_t seed, float rest, int maxiter, int log, int mre_n_vec);
void oq_run_free(oq_run *r);
void oq_hmc(oq_run *r, oq_hmc_out *out, int force_accept);

/* threads used by the OpenMP loops (for the CPU baseline) */
int oq_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
