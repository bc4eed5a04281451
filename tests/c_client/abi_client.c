/* A plain C99 client of the library's C ABI, built and run by
 * tests/test_c_client.py: include/bqcdg.h must compile as C, every entry
 * point must link, and without a device the calls must fail with their
 * documented status codes instead of aborting.  With a device it creates a
 * 4^4 context, builds a cold configuration and its clover term, applies the
 * operator to a point source and solves, as a Fortran or C caller would. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "bqcdg.h"

#define CHECK(cond, what)                      \
  do {                                         \
    if (!(cond)) {                             \
      fprintf(stderr, "FAILED: %s\n", what);   \
      return 1;                                \
    }                                          \
  } while (0)

static int without_device(void) {
  bqcdg_params p = {0.13, 0.13 * 1.9192, 0.0, 0.0};
  bqcdg_solver_opts o;
  bqcdg_solve_info info;
  bqcdg_conf_meta meta;
  int h = 1;
  double rho = 0.1;
  bqcdg_solver_opts_default(&o);
  CHECK(o.precision == BQCDG_PREC_HALF || o.precision == BQCDG_PREC_SINGLE || o.precision == BQCDG_PREC_DOUBLE,
        "default options");
  CHECK(bqcdg_d(NULL, 0, 1, NULL, NULL) == BQCDG_EINVAL, "d without a context");
  CHECK(bqcdg_solve_batch_shifted(NULL, 1, &h, &h, &p, &rho, NULL, &o, 1, &info) == BQCDG_EINVAL,
        "shifted batch without a context");
  CHECK(bqcdg_conf_read(NULL, "x.info", &meta) == BQCDG_EINVAL, "conf_read without a context");
  CHECK(bqcdg_conf_write(NULL, "x", &meta) == BQCDG_EINVAL, "conf_write without a context");
  CHECK(bqcdg_release_scratch(NULL, BQCDG_SCRATCH_SOLVER) == BQCDG_EINVAL, "release without a context");
  CHECK(strcmp(bqcdg_error_string(BQCDG_ECHECKSUM), "configuration check sum error") == 0, "error string");
  return 0;
}

static int with_device(bqcdg_ctx* ctx) {
  const int volh = bqcdg_volh(ctx);
  const size_t n = (size_t)volh * 24;
  double* b = calloc(n, sizeof(double));
  double* x = calloc(n, sizeof(double));
  double* y = calloc(n, sizeof(double));
  bqcdg_params p = {0.13, 0.13 * 1.9192, 0.0, 0.0};
  bqcdg_solver_opts o;
  bqcdg_solve_info info;
  CHECK(b && x && y, "host memory");
  CHECK(bqcdg_conf_cold(ctx) == BQCDG_OK, "conf_cold");
  CHECK(bqcdg_clover_init(ctx, p.csw_kappa) == BQCDG_OK, "clover_init");
  b[0] = 1.0;  /* real part of spin 1, colour 1, site 0 */
  bqcdg_solver_opts_default(&o);
  o.precision = BQCDG_PREC_DOUBLE;
  o.tol = 1e-12;
  CHECK(bqcdg_solve(ctx, x, b, &p, &o, &info) == BQCDG_OK, "solve");
  CHECK(info.converged == 1, "converged");
  CHECK(bqcdg_mtdagmt(ctx, y, x, &p) == BQCDG_OK, "mtdagmt");
  double r2 = 0.0;
  for (size_t k = 0; k < n; k++) r2 += (y[k] - b[k]) * (y[k] - b[k]);
  CHECK(sqrt(r2) < 1e-10, "M^+M x = b");
  free(b);
  free(x);
  free(y);
  return 0;
}

int main(void) {
  if (without_device()) return 1;
  const int L[4] = {4, 4, 4, 4}, bc[4] = {1, 1, 1, -1};
  bqcdg_ctx* ctx = NULL;
  const int st = bqcdg_create(&ctx, L, bc, 0);
  if (st == BQCDG_ENODEVICE) {
    printf("ok (no device)\n");
    return 0;
  }
  CHECK(st == BQCDG_OK, "create");
  const int rc = with_device(ctx);
  bqcdg_destroy(ctx);
  if (rc == 0) printf("ok (device)\n");
  return rc;
}
