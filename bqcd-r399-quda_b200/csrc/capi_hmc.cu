// capi_hmc.cu -- C ABI of the resident HMC pieces (include/bqcdg.h): the
// links, the momenta and the spinor fields stay on the device for a whole
// trajectory (hmc.F90 and the routines it calls).
#include "ctx.cuh"

using namespace bqcdg;
using namespace bqcdg_host;

extern "C" {

static int ensure_mom(bqcdg_ctx* c) {
  const size_t pn = (size_t)64 * c->g.volh * sizeof(double);
  if (!c->mom) {
    CK(c->alloc((void**)&c->mom, pn));
    CK(cudaMemsetAsync(c->mom, 0, pn, c->stream));
  }
  if (!c->mom_old) {
    CK(c->alloc((void**)&c->mom_old, pn));
    CK(cudaMemsetAsync(c->mom_old, 0, pn, c->stream));
  }
  return BQCDG_OK;
}

// one reduction over the momentum field, returned to the host
static int mom_sumsq(bqcdg_ctx* c, const double* a, const double* b, double* out) {
  RedScratch r = c->red;
  r.maxblocks = 8 * nblocks(c->g.volh);  // one partial per block, within the 64-per-block scratch
  launch_mom_sumsq(c->g, a, b, r, c->dres, c->stream);
  CKL();
  CK(cudaMemcpyAsync(c->hres, c->dres, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *out = c->hres[0];
  return BQCDG_OK;
}

// links changed on the device: cached copies are stale, the clover follows
static int gauge_changed(bqcdg_ctx* c, double csw_kappa) {
  for (int k = 0; k < 3; k++) c->gauge_s_ok[k] = false;
  c->gauge64r_ok = false;
  if (csw_kappa != 0.0) return bqcdg_clover_init(c, csw_kappa);
  CK(cudaStreamSynchronize(c->stream));
  return BQCDG_OK;
}

int bqcdg_mom_gauss(bqcdg_ctx* c) {
  if (!c) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  int st = ensure_mom(c);
  if (st) return st;
  // hmc_init_p.F90:28-45: do mu; do eo: ran_gauss_volh(4, p(1,1,eo,mu), 1.0, eo)
  const unsigned long long per = 2ull * 4ull * (unsigned long long)c->g.volh;
  for (int me = 0; me < 8; me++) {
    launch_ran_gauss((double2*)(c->mom + (size_t)me * c->g.volh * 8), c->g.volh, 4, 1.0, c->seed, c->stream);
    c->seed = ranf_skip(c->seed, per);
  }
  CKL();
  CK(cudaStreamSynchronize(c->stream));
  return BQCDG_OK;
}

int bqcdg_mom_set(bqcdg_ctx* c, const double* p) {
  if (!c || !p) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  int st = ensure_mom(c);
  if (st) return st;
  CK(cudaMemcpyAsync(c->mom, p, (size_t)64 * c->g.volh * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return BQCDG_OK;
}

int bqcdg_mom_get(bqcdg_ctx* c, double* p) {
  if (!c || !p) return BQCDG_EINVAL;
  if (!c->mom) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  CK(cudaMemcpyAsync(p, c->mom, (size_t)64 * c->g.volh * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return BQCDG_OK;
}

int bqcdg_mom_action(bqcdg_ctx* c, double* sp) {
  if (!c || !sp || !c->mom) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  double s2 = 0.0;
  int st = mom_sumsq(c, c->mom, nullptr, &s2);
  if (st) return st;
  *sp = 0.5 * s2;  // action.F90 (sp)
  return BQCDG_OK;
}

int bqcdg_mom_mark(bqcdg_ctx* c) {
  if (!c || !c->mom) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  CK(cudaMemcpyAsync(c->mom_old, c->mom, (size_t)64 * c->g.volh * sizeof(double), cudaMemcpyDeviceToDevice,
                     c->stream));
  return BQCDG_OK;
}

int bqcdg_mom_change(bqcdg_ctx* c, double* d2) {
  if (!c || !d2 || !c->mom) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  return mom_sumsq(c, c->mom_old, c->mom, d2);
}

int bqcdg_dsg_dev(bqcdg_ctx* c, double step, double beta) {
  if (!c || !c->mom) return BQCDG_EINVAL;
  if (!c->have_gauge) return BQCDG_ENOGAUGE;
  if (beta == 0.0) return BQCDG_OK;
  CK(cudaSetDevice(c->device));
  launch_dsg(c->g, c->gauge64, c->mom, -step * beta / 3.0, c->stream);
  CKL();
  return BQCDG_OK;
}

int bqcdg_hmc_u_dev(bqcdg_ctx* c, double step, double csw_kappa) {
  if (!c || !c->mom) return BQCDG_EINVAL;
  if (!c->have_gauge) return BQCDG_ENOGAUGE;
  CK(cudaSetDevice(c->device));
  launch_hmc_u(c->g, c->gauge64, c->mom, step, c->stream);
  CKL();
  return gauge_changed(c, csw_kappa);  // hmc_u.F90:68: clover_init of the new links
}

int bqcdg_dsf_dev(bqcdg_ctx* c, double step, const bqcdg_params* par, int ha, int hb) {
  if (!c || !par || !c->mom || !field(c, ha) || !field(c, hb)) return BQCDG_EINVAL;
  if (!c->have_gauge) return BQCDG_ENOGAUGE;
  CK(cudaSetDevice(c->device));
  return dsf_core(c, c->mom, step, par, field(c, ha), field(c, hb));
}

int bqcdg_dsd_dev(bqcdg_ctx* c, double step, const bqcdg_params* par) {
  if (!c || !par || !c->mom) return BQCDG_EINVAL;
  if (!c->have_gauge) return BQCDG_ENOGAUGE;
  const double sd = -step * 2.0 * (par->csw_kappa / 8.0);  // dsd.F90:40
  if (sd == 0.0) return BQCDG_OK;
  if (!c->have_Ainv[1]) return BQCDG_ENOCLOVER;
  CK(cudaSetDevice(c->device));
  int st = ensure_force_bufs(c);
  if (st) return st;
  return dsd_core(c, c->mom, 1, sd);
}

int bqcdg_gauge_save(bqcdg_ctx* c) {
  if (!c) return BQCDG_EINVAL;
  if (!c->have_gauge) return BQCDG_ENOGAUGE;
  CK(cudaSetDevice(c->device));
  const size_t n = (size_t)8 * 9 * c->g.stride * sizeof(double2);
  if (!c->gauge_bck) CK(c->alloc((void**)&c->gauge_bck, n));
  CK(cudaMemcpyAsync(c->gauge_bck, c->gauge64, n, cudaMemcpyDeviceToDevice, c->stream));
  return BQCDG_OK;
}

int bqcdg_gauge_restore(bqcdg_ctx* c, double csw_kappa) {
  if (!c || !c->gauge_bck) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  const size_t n = (size_t)8 * 9 * c->g.stride * sizeof(double2);
  CK(cudaMemcpyAsync(c->gauge64, c->gauge_bck, n, cudaMemcpyDeviceToDevice, c->stream));
  return gauge_changed(c, csw_kappa);
}

int bqcdg_ranf(bqcdg_ctx* c, double* r) {
  if (!c || !r) return BQCDG_EINVAL;
  c->seed = ranf_skip(c->seed, 1);  // ranf.F90: step the 48-bit generator, then scale
  *r = std::ldexp((double)c->seed, -48);
  return BQCDG_OK;
}

int bqcdg_op_dev(bqcdg_ctx* c, int which, int hout, int hin, const bqcdg_params* p) {
  int st = check_op(c, p);
  if (st) return st;
  if (which < 0 || which > 5 || !field(c, hout) || !field(c, hin)) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  double2 *t = c->sp64(2), *q = c->sp64(3);
  if (!t || !q) return BQCDG_ENOMEM;
  OpParams op = op_of(p, which >= 3);
  SpinorPtr so = S(field(c, hout)), si = S(field(c, hin));
  switch (which) {
    case 0: case 3: apply_mtil(c, Prec::F64, false, so, si, S(t), op, nullptr, nullptr); break;
    case 1: case 4: apply_mtil(c, Prec::F64, true, so, si, S(t), op, nullptr, nullptr); break;
    default: apply_mdagm(c, Prec::F64, so, si, S(t), S(q), op);
  }
  CKL();
  return BQCDG_OK;
}

int bqcdg_cg_dev(bqcdg_ctx* c, int hx, int hb, const bqcdg_params* p, const bqcdg_cg_para* cgp, int* iterations,
                 bqcdg_solve_info* info) {
  int st = check_op(c, p);
  if (st) return st;
  if (!cgp || !field(c, hx) || !field(c, hb)) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  bqcdg_solve_info tmp;
  if (!info) info = &tmp;
  std::memset(info, 0, sizeof(*info));
  OpParams op = op_of(p, true);
  st = cg_core(c, field(c, hx), field(c, hb), op, Prec::F64, cgp->maxiter, (double)cgp->rest, 0.0, true, false,
               info);
  if (st) return st;
  if (iterations) *iterations = info->niter;
  if (!info->converged && cgp->log != 2) return BQCDG_ENOCONV;
  return BQCDG_OK;
}

int bqcdg_field_cdot(bqcdg_ctx* c, int ha, int hb, double* re, double* im) {
  if (!c || !re || !im || !field(c, ha) || !field(c, hb)) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  launch_cdot(c->g, field(c, ha), field(c, hb), c->red, c->dres, c->stream);
  CKL();
  CK(cudaMemcpyAsync(c->hres, c->dres, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *re = c->hres[0];
  *im = c->hres[1];
  return BQCDG_OK;
}

int bqcdg_field_cdot_pairs(bqcdg_ctx* c, int n, const int* ha, const int* hb, double* re, double* im) {
  if (!c || n < 1 || n > BQCDG_MAX_DOT_PAIRS || !ha || !hb || !re || !im) return BQCDG_EINVAL;
  static_assert(BQCDG_MAX_DOT_PAIRS == kMaxDotPairs, "one limit for the header and the kernel");
  FieldPairs fp{};
  for (int j = 0; j < n; j++) {
    fp.a[j] = field(c, ha[j]);
    fp.b[j] = field(c, hb[j]);
    if (!fp.a[j] || !fp.b[j]) return BQCDG_EINVAL;
  }
  CK(cudaSetDevice(c->device));
  launch_cdot_pairs(c->g, fp, n, c->red, c->dres, c->stream);
  CKL();
  CK(cudaMemcpyAsync(c->hres, c->dres, 2 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int j = 0; j < n; j++) {
    re[j] = c->hres[2 * j];
    im[j] = c->hres[2 * j + 1];
  }
  return BQCDG_OK;
}

int bqcdg_field_caxpby(bqcdg_ctx* c, int hy, double ay, double are, double aim, int hx) {
  if (!c || !field(c, hy) || !field(c, hx)) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  launch_caxpby(c->g, are, aim, field(c, hx), ay, field(c, hy), c->stream);
  CKL();
  return BQCDG_OK;
}

}  // extern "C"
