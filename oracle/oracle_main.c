/*
 * oracle_main.c -- command-line drivers of the CPU oracle (test infrastructure).
 *
 *   oracle ranf_test       reproduces ranf_test.F90:26-93 (same records)
 *   oracle quick_test      one 4^4 model-C HMC trajectory with the parameters of
 *                          work/input.quick-test; prints the %it, %Favg, %Fmax
 *                          and %fa records of work/out.quick-test.reference and
 *                          the final RNG seed
 *   oracle hmc L0 L1 L2 L3 hot|cold model rho kappa csw beta tau_len steps m_scale
 *                          a general single trajectory (same records)
 */
#include "bqcd_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static void ranf_test(void) {
  int64_t seed;
  double x;
  printf("\n\n default seed:\n\n\n");
  for (int i = 1; i <= 10; i++) {
    oq_ranget(&seed);
    x = oq_ranf();
    printf("%6d%24lld%24.16f\n", i, (long long)seed, x);
  }
  printf("\n\n seed = 4711:\n\n\n");
  oq_ranset(4711, 0);
  for (int i = 1; i <= 10; i++) {
    oq_ranget(&seed);
    x = oq_ranf();
    printf("%6d%24lld%24.16f\n", i, (long long)seed, x);
  }
  printf("\n\n seed varies, no skip:\n\n\n");
  for (int i = -10; i <= 20; i++) {
    oq_ranset(i, 0);
    oq_ranget(&seed);
    x = oq_ranf();
    printf("%6d%24lld%24.16f\n", i, (long long)seed, x);
  }
  printf("\n\n default seed, skip varies:\n\n\n");
  for (int i = -10; i <= 20; i++) {
    oq_ranset(0, i);
    oq_ranget(&seed);
    x = oq_ranf();
    printf("%6d%24lld%24.16f\n", i, (long long)seed, x);
  }
  printf("\n\n large seeds, no skip:\n\n\n");
  for (int i = 0; i <= 47; i++) {
    oq_ranset((int64_t)1 << i, 0);
    oq_ranget(&seed);
    x = oq_ranf();
    printf("%6d%24lld%24.16f\n", i, (long long)seed, x);
  }
  printf("\n\n default seeds, big skips:\n\n\n");
  for (int i = 0; i <= 47; i++) {
    oq_ranset(0, (int64_t)1 << i);
    oq_ranget(&seed);
    x = oq_ranf();
    printf("%6d%24lld%24.16f\n", i, (long long)seed, x);
  }
}

static int run_hmc(const int L[4], int cold, char model, double rho, double kappa, double csw,
                   double beta, double traj_length, int ntau, int m_scale) {
  const int bc[4] = {1, 1, 1, -1};
  oq_hmc_para p;
  memset(&p, 0, sizeof p);
  p.beta = beta;
  p.kappa = kappa;
  p.csw = csw;
  p.csw_kappa = csw * kappa;   /* bqcd.F90:170 */
  p.h = 0;
  p.traj_length = traj_length;
  p.ntau = ntau;
  p.tau = traj_length / ntau;  /* bqcd.F90:175 */
  p.rho = rho;
  p.m_scale = m_scale;
  p.model = model;
  oq_run r;
  if (oq_run_init(&r, L, bc, &p, cold, 0, 1e-5f, 1000, 0, 7)) {
    fprintf(stderr, "bad lattice\n");
    return 1;
  }
  oq_hmc_out out;
  memset(&out, 0, sizeof out);
  oq_hmc(&r, &out, 1);
  int64_t seed;
  oq_ranget(&seed);
  printf("%%it %d %d %d\n", -9, out.it_f1, out.it_f2);
  printf("%%Favg %d %.12e %.12e %.12e %.12e\n", -9, out.f_avg[0], out.f_avg[1], out.f_avg[2], out.f_avg[3]);
  printf("%%Fmax %d %.12e %.12e %.12e %.12e\n", -9, out.f_max[0], out.f_max[1], out.f_max[2], out.f_max[3]);
  printf("%%fa %d %d %.12f %.12f %d %d %d\n", -9, 1, out.sg / (6.0 * r.geom.volume), out.exp_dh,
         out.cg_ncall, out.cg_niter_tot, out.cg_niter_max);
  printf("Seed %lld\n", (long long)seed);
  oq_run_free(&r);
  return 0;
}

/* work/input.test: 20 trajectories of the quick-test system, the first 10
 * force-accepted (hmc_accept_first 10, numbered -9..0), then 10 with the
 * Metropolis test (1..10); the %it, %fa and %mc records of mc.F90 */
static int test20(void) {
  const int L[4] = {4, 4, 4, 4}, bc[4] = {1, 1, 1, -1};
  oq_hmc_para p;
  memset(&p, 0, sizeof p);
  p.beta = 5.0;
  p.kappa = 0.13;
  p.csw = 2.3327;
  p.csw_kappa = p.csw * p.kappa;
  p.traj_length = 0.2;
  p.ntau = 10;
  p.tau = p.traj_length / p.ntau;
  p.rho = 0.1;
  p.m_scale = 3;
  p.model = 'C';
  oq_run r;
  if (oq_run_init(&r, L, bc, &p, 1, 0, 1e-5f, 1000, 0, 7)) return 1;
  for (int k = -9; k <= 10; k++) {
    oq_hmc_out out;
    memset(&out, 0, sizeof out);
    oq_hmc(&r, &out, k <= 0);
    /* a rejected trajectory keeps the old links, whose plaquette is printed */
    const double sg = out.accepted ? out.sg : oq_sg(&r.geom, r.conf.u);
    printf("%%it %d %d %d\n", k, out.it_f1, out.it_f2);
    if (k <= 0)
      printf("%%fa %d %d %.12f %.12f %d %d %d\n", k, 1, sg / (6.0 * r.geom.volume), out.exp_dh, out.cg_ncall,
             out.cg_niter_tot, out.cg_niter_max);
    else
      printf("%%mc %d %d %d %.12f %.12f %d %d %d %d\n", k, 1, 1, sg / (6.0 * r.geom.volume), out.exp_dh,
             out.accepted, out.cg_ncall, out.cg_niter_tot, out.cg_niter_max);
  }
  int64_t seed;
  oq_ranget(&seed);
  printf("Seed %lld\n", (long long)seed);
  oq_run_free(&r);
  return 0;
}

/* work/input.smp: the reference's SMP benchmark, 24^3x48, model A (one
 * pseudofermion), c_sw 1.923076923076923, one force-accepted trajectory of
 * 10 steps with CG capped at 100 iterations (solver_rest 1e-99, which is 0
 * in the FP32 rest; solver_ignore_no_convergence 2) and no MRE vectors */
static int smp(void) {
  const int L[4] = {24, 24, 24, 48}, bc[4] = {1, 1, 1, -1};
  oq_hmc_para p;
  memset(&p, 0, sizeof p);
  p.beta = 5.0;
  p.kappa = 0.13;
  p.csw = 1.923076923076923;
  p.csw_kappa = p.csw * p.kappa;
  p.traj_length = 0.2;
  p.ntau = 10;
  p.tau = p.traj_length / p.ntau;
  p.rho = 0.0;
  p.m_scale = 1;
  p.model = 'A';
  oq_run r;
  if (oq_run_init(&r, L, bc, &p, 1, 0, (float)1e-99, 100, 2, 0)) return 1;
  oq_hmc_out out;
  memset(&out, 0, sizeof out);
  oq_hmc(&r, &out, 1);
  int64_t seed;
  oq_ranget(&seed);
  printf("%%fa %d %d %.12f %.12f %d %d %d\n", 0, 1, out.sg / (6.0 * r.geom.volume), out.exp_dh, out.cg_ncall,
         out.cg_niter_tot, out.cg_niter_max);
  printf("Seed %lld\n", (long long)seed);
  oq_run_free(&r);
  return 0;
}

int main(int argc, char **argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: %s ranf_test | quick_test | hmc ...\n", argv[0]);
    return 2;
  }
  if (!strcmp(argv[1], "ranf_test")) {
    ranf_test();
    return 0;
  }
  if (!strcmp(argv[1], "quick_test")) {
    /* work/input.quick-test */
    const int L[4] = {4, 4, 4, 4};
    return run_hmc(L, 1, 'C', 0.1, 0.13, 2.3327, 5.0, 0.2, 10, 3);
  }
  if (!strcmp(argv[1], "test20")) return test20();
  if (!strcmp(argv[1], "smp")) return smp();
  if (!strcmp(argv[1], "hmc") && argc == 15) {
    int L[4] = {atoi(argv[2]), atoi(argv[3]), atoi(argv[4]), atoi(argv[5])};
    return run_hmc(L, !strcmp(argv[6], "cold"), argv[7][0], atof(argv[8]), atof(argv[9]), atof(argv[10]),
                   atof(argv[11]), atof(argv[12]), atoi(argv[13]), atoi(argv[14]));
  }
  fprintf(stderr, "unknown command\n");
  return 2;
}
