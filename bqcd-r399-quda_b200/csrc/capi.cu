// capi.cu -- host runtime and C ABI (include/bqcdg.h).
//
// A context owns one CUDA stream, the resident FP64 gauge and clover fields
// (plus their reduced-precision copies, rebuilt lazily after each reload),
// scratch spinors and the reduction buffers.  Host arrays in BQCD's Fortran
// layouts are staged with one contiguous copy and converted on the device.
#include "ctx.cuh"

namespace bqcdg_host {

int upload_spinor(bqcdg_ctx* c, const double* host, double2* dev) {
  size_t n = (size_t)c->g.volh * 12 * sizeof(double2);
  CK(c->stage(n));
  CK(cudaMemcpyAsync(c->staging, host, n, cudaMemcpyHostToDevice, c->stream));
  launch_spinor_from_fortran(c->g, dev, c->staging, c->stream);
  CKL();
  return BQCDG_OK;
}

int download_spinor(bqcdg_ctx* c, const double2* dev, double* host) {
  size_t n = (size_t)c->g.volh * 12 * sizeof(double2);
  CK(c->stage(n));
  launch_spinor_to_fortran(c->g, c->staging, dev, c->stream);
  CKL();
  CK(cudaMemcpyAsync(host, c->staging, n, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return BQCDG_OK;
}

OpParams op_of(const bqcdg_params* p, bool with_rho) {
  OpParams o;
  o.kappa = p->kappa;
  o.csw_kappa = p->csw_kappa;
  o.h = p->h;
  o.rho = with_rho ? p->rho : 0.0;
  return o;
}

// sloppy copies of the links / clover blocks used by M~
int ensure_sloppy(bqcdg_ctx* c, Prec p, bool need_clover) {
  int k = (int)p;
  if (!c->gauge_s_ok[k]) {
    if (!c->gauge_su3) return BQCDG_ENOTSU3;
    if (!c->gauge_s[k]) {
      size_t n = (size_t)8 * 3 * c->g.stride * (p == Prec::F32 ? 16 : 8);
      CK(c->alloc(&c->gauge_s[k], n));
    }
    launch_gauge_demote(c->g, p, c->gauge_s[k], c->gauge64, c->stream);
    CKL();
    c->gauge_s_ok[k] = true;
  }
  if (need_clover && !c->clover_s_ok[k]) {
    if (!c->have_A[0] || !c->have_Ainv[1]) return BQCDG_ENOCLOVER;
    for (int w = 0; w < 2; w++) {
      CloverPtr& cp = w == 0 ? c->aee_s[k] : c->ainv_oo_s[k];
      if (!cp.v) {
        size_t n = (size_t)c->g.stride * (p == Prec::F32 ? 18 * 16 : 9 * 16);
        CK(c->alloc(&cp.v, n));
        if (p == Prec::F16) CK(c->alloc((void**)&cp.norm, sizeof(float) * c->g.stride));
      }
      launch_clover_demote(c->g, p, cp, w == 0 ? c->A[0] : c->Ainv[1], c->stream);
      CKL();
    }
    c->clover_s_ok[k] = true;
  }
  return BQCDG_OK;
}

// FP64 operator links in 12-real form when the links are SU(3)
int ensure_f64rec(bqcdg_ctx* c) {
  if (c->gauge64r_ok || !c->gauge_su3) return BQCDG_OK;
  if (!c->gauge64r) CK(c->alloc((void**)&c->gauge64r, (size_t)8 * 6 * c->g.stride * sizeof(double2)));
  launch_gauge_demote(c->g, Prec::F64, c->gauge64r, c->gauge64, c->stream);
  CKL();
  c->gauge64r_ok = true;
  return BQCDG_OK;
}
bool use_rec(bqcdg_ctx* c, Prec p) {
  return p == Prec::F64 && c->gauge_su3 && ensure_f64rec(c) == BQCDG_OK && c->gauge64r_ok;
}
const Geom& geom_of(bqcdg_ctx* c, Prec p) { return use_rec(c, p) ? c->g12 : c->g; }
const void* gauge_of(bqcdg_ctx* c, Prec p) {
  if (p == Prec::F64) return use_rec(c, p) ? (const void*)c->gauge64r : (const void*)c->gauge64;
  return c->gauge_s[(int)p];
}
CloverPtr aee_of(bqcdg_ctx* c, Prec p) { return p == Prec::F64 ? C(c->A[0]) : c->aee_s[(int)p]; }
CloverPtr ainv_of(bqcdg_ctx* c, Prec p) { return p == Prec::F64 ? C(c->Ainv[1]) : c->ainv_oo_s[(int)p]; }

int check_op(bqcdg_ctx* c, const bqcdg_params* p) {
  if (!c || !p) return BQCDG_EINVAL;
  if (!c->have_gauge) return BQCDG_ENOGAUGE;
  if (p->csw_kappa != 0.0 && (!c->have_A[0] || !c->have_Ainv[1])) return BQCDG_ENOCLOVER;
  return BQCDG_OK;
}

// out_e = M~ in_e  (dag: M~^+), with rho for W; t_o scratch (odd)
void apply_mtil(bqcdg_ctx* c, Prec p, bool dag, SpinorPtr out, SpinorPtr in, SpinorPtr t, const OpParams& op,
                double* norm_out, CgScalars* cg) {
  const Geom& g = geom_of(c, p);
  launch_mtil_pass1(p, g, dag, t, in, gauge_of(c, p), ainv_of(c, p), op, cg, c->stream);
  launch_mtil_pass2(p, g, dag, out, t, in, gauge_of(c, p), aee_of(c, p), op, c->red, norm_out, cg, c->stream);
}

// out = (W^+ W) in in precision p; scratch t (odd), q (even)
void apply_mdagm(bqcdg_ctx* c, Prec p, SpinorPtr out, SpinorPtr in, SpinorPtr t, SpinorPtr q, const OpParams& op) {
  apply_mtil(c, p, false, q, in, t, op, nullptr, nullptr);
  apply_mtil(c, p, true, out, q, t, op, nullptr, nullptr);
}

int read_cg(bqcdg_ctx* c) {
  CK(cudaMemcpyAsync(c->hcg, c->dcg, sizeof(CgScalars), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return BQCDG_OK;
}
int write_cg(bqcdg_ctx* c) {
  CK(cudaMemcpyAsync(c->dcg, c->hcg, sizeof(CgScalars), cudaMemcpyHostToDevice, c->stream));
  return BQCDG_OK;
}

struct KernelTimer {
  bqcdg_ctx* c;
  bool on;
  std::vector<cudaEvent_t> pending;
  double ms = 0.0;
  int launches = 0;
  ~KernelTimer() {  // events left when a solve returns early
    for (auto e : pending) cudaEventDestroy(e);
  }
  void begin() {
    if (!on) return;
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, c->stream);
    pending.push_back(e);
  }
  void end() { begin(); }
  // nuse: how many of the recorded launches (in order) did work; launches
  // queued after the solver stopped return at once and are left out
  void collect(int nuse = 1 << 30) {
    if (!on) return;
    cudaStreamSynchronize(c->stream);
    for (size_t k = 0; k + 1 < pending.size() && (int)(k / 2) < nuse; k += 2) {
      float t = 0.f;
      cudaEventElapsedTime(&t, pending[k], pending[k + 1]);
      ms += t;
      launches++;
    }
    for (auto e : pending) cudaEventDestroy(e);
    pending.clear();
  }
};

constexpr int kStalled = 100;  // internal: the sloppy precision stopped converging
// a reliable update at least every kRuEvery sloppy iterations, so that a
// stagnating true residual is seen even when the iterated one keeps falling
constexpr int kRuEvery = 1000;
// int16 iterations get the shorter period: two periodic updates in a row
// (the iterated residual could not fall by delta within it) show that int16
// has run out of accuracy for the system, and the solve moves to FP32
constexpr int kRuEvery16 = 500;

// Core CG on device-resident x, b (F64, device layout).  Solves (W^+W) x = b.
//   sloppy == F64: plain FP64 CG (cg.F90)
//   otherwise:     sloppy iterations in precision `sloppy` with FP64 reliable
//                  updates (x += x_s; r = b - A x in FP64) whenever |r| has
//                  dropped by `delta` since the previous one, and at the end.
int cg_core(bqcdg_ctx* c, double2* x, double2* b, const OpParams& op, Prec sloppy, int maxiter, double stop_rtr,
            double delta, bool min_one_iter, bool time_kernels, bqcdg_solve_info* info) {
  const Geom& g = c->g;
  const bool clover = op.csw_kappa != 0.0;
  if (sloppy != Prec::F64) {
    int st = ensure_sloppy(c, sloppy, clover);
    if (st) return st;
  }
  double2* r = c->sp64(0);
  double2* ax = c->sp64(1);
  double2* t64 = c->sp64(2);
  double2* q64 = c->sp64(3);
  if (!r || !ax || !t64 || !q64) return BQCDG_ENOMEM;
  SpinorPtr p, t, q, rs, xs;
  if (sloppy == Prec::F64) {
    p = S(c->sp64(4));
    t = S(t64);
    q = S(q64);
    rs = S(r);
    xs = S(x);
    if (!p.v) return BQCDG_ENOMEM;
  } else {
    p = c->sp(sloppy, 0);
    t = c->sp(sloppy, 1);
    q = c->sp(sloppy, 2);
    rs = c->sp(Prec::F32, sloppy == Prec::F32 ? 3 : 0);
    xs = c->sp(Prec::F32, sloppy == Prec::F32 ? 4 : 1);
    if (!p.v || !t.v || !q.v || !rs.v || !xs.v) return BQCDG_ENOMEM;
  }
  KernelTimer kt{c, time_kernels};
  CK(cudaEventRecord(c->ev0, c->stream));

  // r = b - A x
  apply_mdagm(c, Prec::F64, S(ax), S(x), S(t64), S(q64), op);
  if (sloppy == Prec::F64) launch_residual(g, r, b, ax, Prec::F64, p, c->red, c->dres, c->stream);
  else launch_residual(g, r, b, ax, Prec::F32, rs, c->red, c->dres, c->stream);
  CKL();
  CK(cudaMemcpyAsync(c->hres, c->dres, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  double rtr = c->hres[0];
  info->b2 = c->hres[1];
  if (sloppy != Prec::F64) {
    launch_spinor_convert(g, sloppy, p, Prec::F32, rs, c->stream);
    launch_zero(g, Prec::F32, xs, c->stream);
    CKL();
  }
  CgScalars& h = *c->hcg;
  std::memset(&h, 0, sizeof(h));
  h.rtr = rtr;
  h.rtr_old = rtr;
  h.stop_rtr = stop_rtr;
  h.maxiter = maxiter;
  h.delta2 = sloppy == Prec::F64 ? 0.0 : delta * delta;
  h.maxr2 = rtr;
  h.ru_every = sloppy == Prec::F64 ? 0 : (sloppy == Prec::F16 ? kRuEvery16 : kRuEvery);
  h.last_ru = 0;
  double best = rtr;  // smallest true |r|^2 so far
  int stall = 0;      // reliable updates in a row without progress
  int forced = 0;     // periodic (not delta-triggered) reliable updates in a row
  bool stalled = false;
  int ru = 0;
  int nl = 5 + (sloppy != Prec::F64 ? 2 : 0);  // kernels launched so far
  bool converged = false;
  if (!(rtr == rtr)) h.done = 4;
  else if (rtr == 0.0 || (!min_one_iter && rtr <= stop_rtr)) { h.done = 1; converged = true; }
  if (maxiter <= 0 && !h.done) h.done = 3;
  { int st_ = write_cg(c); if (st_) return st_; }

  int batch = 4;
  const Geom& gs = geom_of(c, sloppy);  // stencil geometry (12-real FP64 links when SU(3))
  while (!h.done) {
    nl += 6 * batch;
    const int iter0 = h.iter;
    for (int k = 0; k < batch; k++) {
      // pass 1, pass 2 (+|M~p|^2 partials), pass 3 (+ their sum -> alpha), pass 4 (+x,r update, |r|^2
      // partials), the CG step, p update.  With time_kernels, passes 1 and 3 of the second iteration of
      // each batch are bracketed by events: a sample of every batch in the steady state (the first
      // iteration follows the host's read of the scalars, or a reliable update whose FP64 fields have
      // displaced the int16 ones from L2), and events between all launches would lengthen the solve
      // they time.
      const bool timed = k == 1;
      if (timed) kt.begin();
      launch_mtil_pass1(sloppy, gs, false, t, p, gauge_of(c, sloppy), ainv_of(c, sloppy), op, c->dcg, c->stream);
      if (timed) kt.end();
      launch_mtil_pass2(sloppy, gs, false, q, t, p, gauge_of(c, sloppy), aee_of(c, sloppy), op, c->red, nullptr,
                        c->dcg, c->stream, 1, nullptr, nullptr, true);
      if (timed) kt.begin();
      launch_mtil_pass1(sloppy, gs, true, t, q, gauge_of(c, sloppy), ainv_of(c, sloppy), op, c->dcg, c->stream, 1,
                        nullptr, AlphaFin{c->red.partial, c->red.maxblocks, c->dcg});
      if (timed) kt.end();
      launch_cg_pass4(sloppy, gs, t, q, gauge_of(c, sloppy), aee_of(c, sloppy), op, p, xs, rs, c->red, c->dcg,
                      c->stream, 1, false, nullptr, nullptr, true);
      launch_cg_step(c->red, c->dcg, 1, nblocks(gs.volh), c->stream);
      launch_cg_pupdate(sloppy, g, p, rs, c->dcg, c->stream, 1, xs, iter0 + k + 1);
    }
    CKL();
    int st = read_cg(c);
    if (st) return st;
    kt.collect(h.iter > iter0 + 1 ? 2 : 0);  // the two timed passes ran if the batch's second iteration did
    if (batch < 16) batch *= 2;
    if (h.done == 4) break;
    if (h.done == 0) continue;
    if (sloppy == Prec::F64) {
      converged = h.done == 1;
      break;
    }
    // reliable update: x += x_s, r = b - A x in FP64
    const bool periodic = !(h.rtr < h.delta2 * h.maxr2);
    nl += 7;
    launch_accum_x(g, x, (float4*)xs.v, c->stream);
    apply_mdagm(c, Prec::F64, S(ax), S(x), S(t64), S(q64), op);
    launch_residual(g, r, b, ax, Prec::F32, rs, c->red, c->dres, c->stream);
    CKL();
    CK(cudaMemcpyAsync(c->hres, c->dres, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    ru++;
    double rtrue = c->hres[0];
    if (!(rtrue == rtrue)) { h.done = 4; break; }
    if (rtrue <= stop_rtr) { h.rtr = rtrue; converged = true; h.done = 1; break; }
    if (h.done == 3) { h.rtr = rtrue; break; }
    // progress check: the sloppy precision has run out when the true residual
    // stops falling (or grows) over several reliable updates
    if (rtrue < 0.5 * best) { best = rtrue; stall = 0; }
    else if (++stall >= 5 || rtrue > 1e4 * best) { h.rtr = rtrue; stalled = true; break; }
    forced = periodic ? forced + 1 : 0;
    if (sloppy == Prec::F16 && forced >= 2) { h.rtr = rtrue; stalled = true; break; }
    // continue from the true residual with p re-orthogonalised against it:
    // p = r + beta (p - (<r,p>/|r|^2) r), beta = |r|^2 / |r_old|^2
    launch_rdot(g, rs, sloppy, p, c->red, c->dres, c->stream);
    CKL();
    CK(cudaMemcpyAsync(c->hres, c->dres, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    double rpc = c->hres[0] / rtrue;
    h.beta = rtrue / h.rtr_old;
    h.rtr = rtrue;
    h.maxr2 = rtrue;
    h.last_ru = h.iter;
    h.done = 0;
    { int st_ = write_cg(c); if (st_) return st_; }
    launch_p_reorth(g, sloppy, p, rs, rpc, h.beta, c->stream);
    nl += 2;
    CKL();
  }
  CK(cudaEventRecord(c->ev1, c->stream));
  CK(cudaEventSynchronize(c->ev1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  info->seconds = ms * 1e-3;
  info->niter = h.iter;
  info->reliable_updates = ru;
  info->kernel_launches = nl;
  info->rtr = h.rtr;
  info->converged = converged ? 1 : 0;
  info->stencil_ms = kt.ms;
  info->stencil_launches = kt.launches;
  if (h.done == 4) return BQCDG_ENAN;
  if (stalled) return kStalled;
  return BQCDG_OK;
}

// cg_core with precision escalation: when the sloppy iterations stop making
// progress on the true residual (ill-conditioned systems can exhaust int16
// accuracy), continue from the current x with FP32, and then FP64, sloppy
// fields.  Statistics add up over the stages.
int cg_robust(bqcdg_ctx* c, double2* x, double2* b, const OpParams& op, Prec sloppy, int maxiter, double stop_rtr,
              double delta, bool min_one_iter, bool time_kernels, bqcdg_solve_info* info) {
  bqcdg_solve_info sum;
  std::memset(&sum, 0, sizeof(sum));
  Prec cur = sloppy;
  for (;;) {
    bqcdg_solve_info one;
    std::memset(&one, 0, sizeof(one));
    int st = cg_core(c, x, b, op, cur, maxiter - sum.niter, stop_rtr, delta, min_one_iter && sum.niter == 0,
                     time_kernels, &one);
    if (sum.niter == 0) sum.b2 = one.b2;
    sum.niter += one.niter;
    sum.reliable_updates += one.reliable_updates;
    sum.kernel_launches += one.kernel_launches;
    sum.seconds += one.seconds;
    sum.stencil_ms += one.stencil_ms;
    sum.stencil_launches += one.stencil_launches;
    sum.rtr = one.rtr;
    sum.converged = one.converged;
    if (st != kStalled || cur == Prec::F64) {
      *info = sum;
      return st == kStalled ? BQCDG_OK : st;
    }
    cur = cur == Prec::F16 ? Prec::F32 : Prec::F64;
  }
}

int true_residual(bqcdg_ctx* c, double2* x, double2* b, const OpParams& op, double* rtr) {
  double2* r = c->sp64(0);
  double2* ax = c->sp64(1);
  apply_mdagm(c, Prec::F64, S(ax), S(x), S(c->sp64(2)), S(c->sp64(3)), op);
  launch_residual(c->g, r, b, ax, Prec::F64, SpinorPtr{}, c->red, c->dres, c->stream);
  CKL();
  CK(cudaMemcpyAsync(c->hres, c->dres, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *rtr = c->hres[0];
  return BQCDG_OK;
}

Prec prec_of(int p) { return p == BQCDG_PREC_DOUBLE ? Prec::F64 : (p == BQCDG_PREC_SINGLE ? Prec::F32 : Prec::F16); }

// one buffer of nb fields of precision p, rsb bytes apart
int alloc_batched(bqcdg_ctx* c, Prec p, int nb, SpinorPtr& out) {
  out = SpinorPtr{};
  out.rsb = (long long)c->spin_bytes(p);
  CK(c->alloc(&out.v, (size_t)out.rsb * nb));
  CK(cudaMemsetAsync(out.v, 0, (size_t)out.rsb * nb, c->stream));
  if (p == Prec::F16) {
    out.rsnb = (long long)sizeof(float) * c->g.stride;
    CK(c->alloc((void**)&out.norm, (size_t)out.rsnb * nb));
    CK(cudaMemsetAsync(out.norm, 0, (size_t)out.rsnb * nb, c->stream));
  }
  return BQCDG_OK;
}

int ensure_batch(bqcdg_ctx* c, Prec p, int nb) {
  auto& B = c->batch;
  if (B.cap >= nb && B.prec == p) return BQCDG_OK;
  for (SpinorPtr* s : {&B.p, &B.t, &B.q, &B.rs, &B.xs}) {
    c->release(s->v);
    c->release(s->norm);
    *s = SpinorPtr{};
  }
  B.cap = 0;
  int st;
  if ((st = alloc_batched(c, p, nb, B.p)) || (st = alloc_batched(c, p, nb, B.t)) ||
      (st = alloc_batched(c, p, nb, B.q)) || (st = alloc_batched(c, Prec::F32, nb, B.rs)) ||
      (st = alloc_batched(c, Prec::F32, nb, B.xs)))
    return st;
  B.cap = nb;
  B.prec = p;
  return BQCDG_OK;
}

// r = b - A x in FP64 for one right-hand side, r copied into rs (F32);
// returns |r|^2 and |b|^2
int fp64_residual(bqcdg_ctx* c, double2* x, double2* b, const OpParams& op, SpinorPtr rs, double* r2, double* b2) {
  double2 *r = c->sp64(0), *ax = c->sp64(1);
  apply_mdagm(c, Prec::F64, S(ax), S(x), S(c->sp64(2)), S(c->sp64(3)), op);
  launch_residual(c->g, r, b, ax, Prec::F32, rs, c->red, c->dres, c->stream);
  CKL();
  CK(cudaMemcpyAsync(c->hres, c->dres, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *r2 = c->hres[0];
  if (b2) *b2 = c->hres[1];
  return BQCDG_OK;
}

int tune_nbt(bqcdg_ctx* c, Prec p, const OpParams& op, int nb, int* nbt, float* ms = nullptr);

// Batched mixed-precision CG over nb right-hand sides: the five kernels of a
// sloppy iteration each serve all nb (CTAs rhs-fastest), every right-hand
// side has its own scalars, stops and FP64 reliable updates, and a converged
// or paused one costs its CTAs an early return only.  nbt: right-hand sides
// per stencil thread (2, 4: the register-blocked passes of dslash_multi.cu;
// 0: timed choice).
int cg_batch(bqcdg_ctx* c, double2** x, double2** b, int nb, const OpParams& op, Prec sloppy, int maxiter,
             const double* stop, double delta, bqcdg_solve_info* info, const double* rho, int nbt,
             const double* kappa) {
  const Geom& g = c->g;
  int st = ensure_sloppy(c, sloppy, op.csw_kappa != 0.0);
  if (st) return st;
  if ((st = ensure_batch(c, sloppy, nb))) return st;
  auto& B = c->batch;
  // the register-blocked passes take h = 0, one kappa and the stored clover
  // blocks only
  const bool blocked_ok = op.h == 0.0 && !kappa && !g.clover_t;
  if (nbt == 0 && blocked_ok && (st = tune_nbt(c, sloppy, op, nb, &nbt))) return st;
  if (nbt > nb || !blocked_ok) nbt = 1;
  // the operator of right-hand side k: op, with its own shift when rho is
  // given and its own hopping parameter when kappa is
  std::vector<OpParams> ops(nb, op);
  const double* drho = nullptr;
  const double* dkap = nullptr;
  if (rho) {
    for (int k = 0; k < nb; k++) ops[k].rho = rho[k];
    std::memcpy(c->hres, rho, sizeof(double) * nb);
    CK(cudaMemcpyAsync(c->drho, c->hres, sizeof(double) * nb, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));  // hres is reused below
    drho = c->drho;
  }
  if (kappa) {
    for (int k = 0; k < nb; k++) ops[k].kappa = kappa[k];
    std::memcpy(c->hres, kappa, sizeof(double) * nb);
    CK(cudaMemcpyAsync(c->dkappa, c->hres, sizeof(double) * nb, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    dkap = c->dkappa;
  }
  CK(cudaEventRecord(c->ev0, c->stream));
  std::vector<int> ru(nb, 0), fin(nb, 0), conv(nb, 0), nl(nb, 0), stall(nb, 0), stalled(nb, 0);
  std::vector<double> best(nb, 0.0);
  for (int k = 0; k < nb; k++) {
    double r2, b2;
    if ((st = fp64_residual(c, x[k], b[k], ops[k], rhs_of(B.rs, k), &r2, &b2))) return st;
    launch_spinor_convert(g, sloppy, rhs_of(B.p, k), Prec::F32, rhs_of(B.rs, k), c->stream);
    launch_zero(g, Prec::F32, rhs_of(B.xs, k), c->stream);
    CKL();
    CgScalars& h = c->hcg[k];
    std::memset(&h, 0, sizeof(h));
    h.rtr = h.rtr_old = r2;
    h.stop_rtr = stop[k];
    h.maxiter = maxiter;
    h.delta2 = delta * delta;
    h.maxr2 = r2;
    h.ru_every = kRuEvery;
    h.last_ru = 0;
    best[k] = r2;
    info[k].b2 = b2;
    if (!(r2 == r2)) { h.done = 4; fin[k] = 1; }
    else if (r2 <= stop[k]) { h.done = 1; fin[k] = 1; conv[k] = 1; }
    else if (maxiter <= 0) { h.done = 3; fin[k] = 1; }
  }
  CK(cudaMemcpyAsync(c->dcg, c->hcg, sizeof(CgScalars) * nb, cudaMemcpyHostToDevice, c->stream));
  int batch = 4, launches = 0;
  auto running = [&]() {
    for (int k = 0; k < nb; k++)
      if (!fin[k]) return true;
    return false;
  };
  while (running()) {
    for (int it = 0; it < batch; it++) {
      if (nbt > 1) {
        launch_mtil_pass1_n(sloppy, g, false, B.t, B.p, gauge_of(c, sloppy), ainv_of(c, sloppy), op, c->dcg,
                            c->stream, nb, nbt);
        launch_mtil_pass2_n(sloppy, g, B.q, B.t, B.p, gauge_of(c, sloppy), aee_of(c, sloppy), op, c->red, c->dcg,
                            c->stream, nb, drho, nbt, true);
        launch_mtil_pass1_n(sloppy, g, true, B.t, B.q, gauge_of(c, sloppy), ainv_of(c, sloppy), op, c->dcg,
                            c->stream, nb, nbt, AlphaFin{c->red.partial, c->red.maxblocks, c->dcg});
        launch_cg_pass4_n(sloppy, g, B.t, B.q, gauge_of(c, sloppy), aee_of(c, sloppy), op, B.p, B.xs, B.rs, c->red,
                          c->dcg, c->stream, nb, drho, nbt, true);
        launch_cg_step(c->red, c->dcg, nb, nblocks(g.volh), c->stream);
      } else {
        launch_mtil_pass1(sloppy, g, false, B.t, B.p, gauge_of(c, sloppy), ainv_of(c, sloppy), op, c->dcg,
                          c->stream, nb, dkap);
        launch_mtil_pass2(sloppy, g, false, B.q, B.t, B.p, gauge_of(c, sloppy), aee_of(c, sloppy), op, c->red,
                          nullptr, c->dcg, c->stream, nb, drho, dkap, true);
        launch_mtil_pass1(sloppy, g, true, B.t, B.q, gauge_of(c, sloppy), ainv_of(c, sloppy), op, c->dcg,
                          c->stream, nb, dkap, AlphaFin{c->red.partial, c->red.maxblocks, c->dcg});
        launch_cg_pass4(sloppy, g, B.t, B.q, gauge_of(c, sloppy), aee_of(c, sloppy), op, B.p, B.xs, B.rs, c->red,
                        c->dcg, c->stream, nb, true, drho, dkap, true);
        launch_cg_step(c->red, c->dcg, nb, nblocks(g.volh), c->stream);
      }
      launch_cg_pupdate(sloppy, g, B.p, B.rs, c->dcg, c->stream, nb);
    }
    launches += 6 * batch;
    CKL();
    CK(cudaMemcpyAsync(c->hcg, c->dcg, sizeof(CgScalars) * nb, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (batch < 16) batch *= 2;
    std::vector<int> resume;
    for (int k = 0; k < nb; k++) {
      CgScalars& h = c->hcg[k];
      if (fin[k] || h.done == 0) continue;
      if (h.done == 4) { fin[k] = 1; continue; }
      // reliable update of right-hand side k: x += x_s, r = b - A x in FP64
      launch_accum_x(g, x[k], (float4*)rhs_of(B.xs, k).v, c->stream);
      double rt;
      if ((st = fp64_residual(c, x[k], b[k], ops[k], rhs_of(B.rs, k), &rt, nullptr))) return st;
      ru[k]++;
      launches += 7;
      if (!(rt == rt)) { h.done = 4; fin[k] = 1; continue; }
      if (rt <= stop[k]) { h.rtr = rt; h.done = 1; fin[k] = 1; conv[k] = 1; continue; }
      if (h.done == 3) { h.rtr = rt; fin[k] = 1; continue; }
      if (rt < 0.5 * best[k]) { best[k] = rt; stall[k] = 0; }
      else if (++stall[k] >= 5 || rt > 1e4 * best[k]) {
        // retire it here; it is finished below at a higher sloppy precision
        h.rtr = rt;
        h.done = 1;
        fin[k] = 1;
        stalled[k] = 1;
        continue;
      }
      h.beta = rt / h.rtr_old;
      h.rtr = rt;
      h.maxr2 = rt;
      h.last_ru = h.iter;
      h.done = 0;
      resume.push_back(k);
    }
    CK(cudaMemcpyAsync(c->dcg, c->hcg, sizeof(CgScalars) * nb, cudaMemcpyHostToDevice, c->stream));
    for (int k : resume) {
      // p = r + beta (p - (<r,p>/|r|^2) r)
      launch_rdot(g, rhs_of(B.rs, k), sloppy, rhs_of(B.p, k), c->red, c->dres, c->stream);
      CKL();
      CK(cudaMemcpyAsync(c->hres, c->dres, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      launch_p_reorth(g, sloppy, rhs_of(B.p, k), rhs_of(B.rs, k), c->hres[0] / c->hcg[k].rtr, c->hcg[k].beta,
                      c->stream);
      launches += 2;
    }
    CKL();
  }
  CK(cudaEventRecord(c->ev1, c->stream));
  CK(cudaEventSynchronize(c->ev1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  bool nan = false;
  std::vector<CgScalars> hs(c->hcg, c->hcg + nb);
  for (int k = 0; k < nb; k++) {
    info[k].seconds = ms * 1e-3;
    info[k].niter = hs[k].iter;
    info[k].reliable_updates = ru[k];
    info[k].rtr = hs[k].rtr;
    info[k].converged = conv[k];
    info[k].kernel_launches = launches;
    nan = nan || hs[k].done == 4;
  }
  // right-hand sides whose int16 iterations stalled: finish alone from the
  // current x with FP32 (then FP64) sloppy fields
  for (int k = 0; k < nb; k++) {
    if (!stalled[k]) continue;
    bqcdg_solve_info more;
    std::memset(&more, 0, sizeof(more));
    int st2 = cg_robust(c, x[k], b[k], ops[k], sloppy == Prec::F16 ? Prec::F32 : Prec::F64,
                        maxiter - info[k].niter, stop[k], delta, false, false, &more);
    if (st2) return st2;
    info[k].niter += more.niter;
    info[k].reliable_updates += more.reliable_updates;
    info[k].seconds += more.seconds;
    info[k].rtr = more.rtr;
    info[k].converged = more.converged;
  }
  return nan ? BQCDG_ENAN : BQCDG_OK;
}

// device time of one batched first pass over the batch buffers: nb
// right-hand sides, nbt of them per thread (1: one per CTA, dslash.cu)
int time_pass1(bqcdg_ctx* c, Prec p, const OpParams& op, int nb, int nbt, int reps, float* ms) {
  auto launch = [&]() {
    if (nbt > 1)
      launch_mtil_pass1_n(p, c->g, false, c->batch.t, c->batch.p, gauge_of(c, p), ainv_of(c, p), op, nullptr,
                          c->stream, nb, nbt);
    else
      launch_mtil_pass1(p, c->g, false, c->batch.t, c->batch.p, gauge_of(c, p), ainv_of(c, p), op, nullptr,
                        c->stream, nb);
  };
  for (int w = 0; w < 2; w++) launch();
  CK(cudaEventRecord(c->ev0, c->stream));
  for (int r = 0; r < reps; r++) launch();
  CK(cudaEventRecord(c->ev1, c->stream));
  CKL();
  CK(cudaEventSynchronize(c->ev1));
  float t = 0.f;
  cudaEventElapsedTime(&t, c->ev0, c->ev1);
  *ms = t / reps;
  return BQCDG_OK;
}

// device time of one batched M~^+M~ over the batch buffers (the four stencil
// passes of a CG iteration, the second halves with their reductions but no
// CG scalars), nbt right-hand sides per thread.  The buffers hold no solve
// while the tuner runs.
int time_mdagm_batch(bqcdg_ctx* c, Prec p, const OpParams& op, int nb, int nbt, int reps, float* ms) {
  auto& B = c->batch;
  const void* U = gauge_of(c, p);
  auto launch = [&]() {
    if (nbt > 1) {
      launch_mtil_pass1_n(p, c->g, false, B.t, B.p, U, ainv_of(c, p), op, nullptr, c->stream, nb, nbt);
      launch_mtil_pass2_n(p, c->g, B.q, B.t, B.p, U, aee_of(c, p), op, c->red, nullptr, c->stream, nb, nullptr, nbt,
                          true);
      launch_mtil_pass1_n(p, c->g, true, B.t, B.q, U, ainv_of(c, p), op, nullptr, c->stream, nb, nbt);
      launch_mtil_pass2_n(p, c->g, B.p, B.t, B.q, U, aee_of(c, p), op, c->red, nullptr, c->stream, nb, nullptr, nbt,
                          true);
    } else {
      launch_mtil_pass1(p, c->g, false, B.t, B.p, U, ainv_of(c, p), op, nullptr, c->stream, nb);
      launch_mtil_pass2(p, c->g, false, B.q, B.t, B.p, U, aee_of(c, p), op, c->red, nullptr, nullptr, c->stream, nb);
      launch_mtil_pass1(p, c->g, true, B.t, B.q, U, ainv_of(c, p), op, nullptr, c->stream, nb);
      launch_mtil_pass2(p, c->g, true, B.p, B.t, B.q, U, aee_of(c, p), op, c->red, nullptr, nullptr, c->stream, nb);
    }
  };
  launch();
  CK(cudaEventRecord(c->ev0, c->stream));
  for (int r = 0; r < reps; r++) launch();
  CK(cudaEventRecord(c->ev1, c->stream));
  CKL();
  CK(cudaEventSynchronize(c->ev1));
  float t = 0.f;
  cudaEventElapsedTime(&t, c->ev0, c->ev1);
  *ms = t / reps;
  return BQCDG_OK;
}

// right-hand sides per stencil thread for launches of nb at precision p:
// the fastest batched M~^+M~ of 1, 2 and 4 (timed once, then cached).  The
// register-blocked passes need h = 0.  ms: the chosen time, when timed.
int tune_nbt(bqcdg_ctx* c, Prec p, const OpParams& op, int nb, int* nbt, float* ms) {
  int& cached = c->tuned_nbt[(int)p][nb];
  if (cached && !ms) {
    *nbt = cached;
    return BQCDG_OK;
  }
  float best = 0.f;
  int choice = 1;
  for (int k : {1, 2, 4}) {
    if (k > 1 && (k > nb || op.h != 0.0 || p == Prec::F64 || c->g.clover_t)) break;
    float t;
    int st = time_mdagm_batch(c, p, op, nb, k, 2, &t);
    if (st) return st;
    if (k == 1 || t < 0.98f * best) {
      best = t;
      choice = k;
    }
  }
  cached = choice;
  *nbt = choice;
  if (ms) *ms = best;
  return BQCDG_OK;
}

// RHS per launch for a batch: the per-RHS time of a batched M~^+M~ (at its
// best RHS per thread), timed for 1, 4, 8 and 16 right-hand sides on the
// resident fields
int tune_block(bqcdg_ctx* c, Prec p, const OpParams& op, int nmax, int* best) {
  const int cand[4] = {1, 4, 8, 16};
  int cap = 1;
  for (int k = 0; k < 4; k++)
    if (cand[k] <= nmax) cap = cand[k];
  int st = ensure_sloppy(c, p, op.csw_kappa != 0.0);
  if (st) return st;
  if ((st = ensure_batch(c, p, cap))) return st;
  double bestt = 1e300;
  *best = 1;
  for (int k = 0; k < 4 && cand[k] <= cap; k++) {
    int nb = cand[k], nbt;
    float ms;
    if ((st = tune_nbt(c, p, op, nb, &nbt, &ms))) return st;
    double per_rhs = ms / nb;
    if (per_rhs < bestt * 0.98) {
      bestt = per_rhs;
      *best = nb;
    }
  }
  return BQCDG_OK;
}

}  // namespace bqcdg_host

using namespace bqcdg_host;

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* bqcdg_error_string(int s) {
  switch (s) {
    case BQCDG_OK: return "ok";
    case BQCDG_EINVAL: return "invalid argument";
    case BQCDG_ECUDA: return "CUDA error";
    case BQCDG_ENOCONV: return "no convergence";
    case BQCDG_ENAN: return "residual is NaN";
    case BQCDG_ENOGAUGE: return "no gauge field loaded";
    case BQCDG_ENOCLOVER: return "clover term not loaded";
    case BQCDG_ENOMEM: return "device out of memory";
    case BQCDG_EUNSUPPORTED: return "unsupported parameters";
    case BQCDG_ENOTSU3: return "links are not SU(3)";
    case BQCDG_ENODEVICE: return "no CUDA device";
    case BQCDG_ECHECKSUM: return "configuration check sum error";
    case BQCDG_EIO: return "file error";
    default: return "unknown status";
  }
}

int bqcdg_create(bqcdg_ctx** out, const int L[4], const int bc[4], int device) {
  if (!out || !L || !bc) return BQCDG_EINVAL;
  *out = nullptr;
  for (int d = 0; d < 4; d++)
    if (L[d] <= 0 || L[d] % 2 || (bc[d] != 1 && bc[d] != -1)) return BQCDG_EINVAL;  // init_common.F90:67-72
  long long vol = (long long)L[0] * L[1] * L[2] * L[3];
  if (vol / 2 > (1LL << 30)) return BQCDG_EINVAL;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return BQCDG_ENODEVICE;
  if (device < 0 || device >= ndev) return BQCDG_EINVAL;
  CK(cudaSetDevice(device));
  bqcdg_ctx* c = new bqcdg_ctx();
  c->device = device;
  for (int d = 0; d < 4; d++) {
    c->g.L[d] = L[d];
    c->g.bcsign[d] = bc[d];
  }
  c->g.Lxh = L[0] / 2;
  c->g.volh = (int)(vol / 2);
  c->g.stride = (c->g.volh + 63) / 64 * 64;
  c->g.rec12 = 0;
  geom_finish(c->g);
  c->g12 = c->g;
  c->g12.rec12 = 1;
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
  c->red.maxblocks = nblocks(c->g.volh);
  if (e == cudaSuccess)
    e = c->alloc((void**)&c->red.partial, sizeof(double) * kRedVals * kMaxRhs * c->red.maxblocks);
  if (e == cudaSuccess) e = c->alloc((void**)&c->red.counter, sizeof(unsigned int) * kMaxRhs);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->red.counter, 0, sizeof(unsigned int) * kMaxRhs, c->stream);
  if (e == cudaSuccess) e = c->alloc((void**)&c->dres, sizeof(double) * 16);
  if (e == cudaSuccess) e = c->alloc((void**)&c->drho, sizeof(double) * kMaxRhs);
  if (e == cudaSuccess) e = c->alloc((void**)&c->dkappa, sizeof(double) * kMaxRhs);
  if (e == cudaSuccess) e = c->alloc((void**)&c->dcg, sizeof(CgScalars) * kMaxRhs);
  if (e == cudaSuccess) e = cudaMallocHost((void**)&c->hres, sizeof(double) * 16);
  if (e == cudaSuccess) e = cudaMallocHost((void**)&c->hcg, sizeof(CgScalars) * kMaxRhs);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    bqcdg_destroy(c);
    return status_from_cuda(e);
  }
  *out = c;
  return BQCDG_OK;
}

int bqcdg_destroy(bqcdg_ctx* c) {
  if (!c) return BQCDG_EINVAL;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (void* p : c->allocations) cudaFree(p);
  if (c->hres) cudaFreeHost(c->hres);
  if (c->hcg) cudaFreeHost(c->hcg);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return BQCDG_OK;
}

int bqcdg_volh(const bqcdg_ctx* c) { return c ? c->g.volh : -1; }
long long bqcdg_device_bytes(const bqcdg_ctx* c) { return c ? c->bytes : -1; }

int bqcdg_release_scratch(bqcdg_ctx* c, int what) {
  if (!c || what < 0 || what > (BQCDG_SCRATCH_SOLVER | BQCDG_SCRATCH_HMC)) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->stream));
  if (what & BQCDG_SCRATCH_SOLVER) {
    c->release(c->staging);
    c->staging = nullptr;
    c->staging_bytes = 0;
    c->release(c->clov_tmp);
    c->clov_tmp = nullptr;
    for (double2* p : c->s64) c->release(p);
    c->s64.clear();
    for (std::vector<SpinorPtr>* pool : {&c->s32, &c->s16}) {
      for (SpinorPtr& sp : *pool) {
        c->release(sp.v);
        c->release(sp.norm);
      }
      pool->clear();
    }
    auto& B = c->batch;
    auto& K = c->blk;
    for (SpinorPtr* sp : {&K.P, &K.Q, &K.Z, &K.M, &K.Xs, &K.T, &K.Qe}) {
      c->release(sp->v);
      *sp = SpinorPtr{};
    }
    c->release(K.partial);
    c->release(K.gram);
    c->release(K.mats);
    K = bqcdg_ctx::BlockCg{};
    for (SpinorPtr* sp : {&B.p, &B.t, &B.q, &B.rs, &B.xs}) {
      c->release(sp->v);
      c->release(sp->norm);
      *sp = SpinorPtr{};
    }
    B.cap = 0;
  }
  if (what & BQCDG_SCRATCH_HMC) {
    for (double** p : {&c->pgen, &c->mom, &c->mom_old}) {
      c->release(*p);
      *p = nullptr;
    }
    for (double2** p : {&c->wbuf, &c->gauge_bck}) {
      c->release(*p);
      *p = nullptr;
    }
  }
  return BQCDG_OK;
}

int bqcdg_load_gauge(bqcdg_ctx* c, const double* u, int flipped) {
  if (!c || !u) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  if (!c->gauge64) CK(c->alloc((void**)&c->gauge64, (size_t)8 * 9 * c->g.stride * sizeof(double2)));
  size_t n = (size_t)c->g.volh * 72 * sizeof(double2);
  CK(c->stage(n));
  CK(cudaMemcpyAsync(c->staging, u, n, cudaMemcpyHostToDevice, c->stream));
  launch_gauge_from_fortran(c->g, c->gauge64, c->staging, flipped, c->stream);
  CKL();
  launch_gauge_check(c->g, c->gauge64, c->red, c->dres, c->stream);
  CKL();
  CK(cudaMemcpyAsync(c->hres, c->dres, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->gauge_su3 = c->hres[0] < 1e-10 && c->hres[1] < 1e-10;
  c->have_gauge = true;
  for (int k = 0; k < 3; k++) c->gauge_s_ok[k] = false;
  c->gauge64r_ok = false;
  return BQCDG_OK;
}

int bqcdg_get_gauge(bqcdg_ctx* c, double* u, int flipped) {
  if (!c || !u) return BQCDG_EINVAL;
  if (!c->have_gauge) return BQCDG_ENOGAUGE;
  CK(cudaSetDevice(c->device));
  CK(c->stage((size_t)c->g.volh * 72 * sizeof(double2)));
  launch_gauge_to_fortran(c->g, c->staging, c->gauge64, flipped, c->stream);
  CKL();
  CK(cudaMemcpyAsync(u, c->staging, (size_t)c->g.volh * 72 * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return BQCDG_OK;
}

// the clover term at any kappa: T = (-c_sw / 8)(p +- q) of the even sites in
// A[0] and of the odd sites in Ainv[1], the two fields the even-odd
// operator reads; the kernels form A(kappa) = 1 + kappa T and its inverse per
// site (g.clover_t)
static int clover_init_t(bqcdg_ctx* c, double csw) {
  if (!c->have_gauge) return BQCDG_ENOGAUGE;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->stream));
  double2** unused[4] = {&c->A[1], &c->Ainv[0], &c->B[0], &c->B[1]};
  for (double2** f : unused) {
    c->release(*f);
    *f = nullptr;
  }
  const size_t n = (size_t)36 * c->g.stride * sizeof(double2);
  if (!c->A[0]) CK(c->alloc((void**)&c->A[0], n));
  if (!c->Ainv[1]) CK(c->alloc((void**)&c->Ainv[1], n));
  if (!c->clov_tmp) CK(c->alloc((void**)&c->clov_tmp, (size_t)54 * clover_init_chunk(c->g) * sizeof(double2)));
  double2* t[2] = {c->A[0], c->Ainv[1]};
  launch_clover_t(c->g, c->gauge64, csw, t, c->clov_tmp, c->stream);
  CKL();
  CK(cudaStreamSynchronize(c->stream));
  for (int eo = 0; eo < 2; eo++) c->have_A[eo] = c->have_Ainv[eo] = c->have_B[eo] = false;
  c->have_A[0] = c->have_Ainv[1] = true;
  for (int k = 0; k < 3; k++) c->clover_s_ok[k] = false;
  c->g.clover_t = c->g12.clover_t = 1;
  return BQCDG_OK;
}

// the parities eo0..eo1 of one clover field from its Fortran array
static int load_clover_field(bqcdg_ctx* c, double2** dst, bool* have, const double* src, int eo0 = 0,
                             int eo1 = 1) {
  for (int eo = eo0; eo <= eo1; eo++) {
    if (!dst[eo]) CK(c->alloc((void**)&dst[eo], (size_t)36 * c->g.stride * sizeof(double2)));
    size_t n = (size_t)c->g.volh * 36 * sizeof(double2);
    CK(c->stage(n));
    CK(cudaMemcpyAsync(c->staging, src + (size_t)eo * c->g.volh * 72, n, cudaMemcpyHostToDevice, c->stream));
    launch_clover_from_fortran(c->g, dst[eo], c->staging, c->stream);
    CKL();
    have[eo] = true;
  }
  return BQCDG_OK;
}

int bqcdg_load_clover(bqcdg_ctx* c, const double* a, const double* ainv, const double* b) {
  if (!c) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  int st;
  if (a && (st = load_clover_field(c, c->A, c->have_A, a))) return st;
  if (ainv && (st = load_clover_field(c, c->Ainv, c->have_Ainv, ainv))) return st;
  if (b && (st = load_clover_field(c, c->B, c->have_B, b))) return st;
  // an inverse is needed by M~; derive it from B when only B was given
  if (!ainv && b) {
    for (int eo = 0; eo < 2; eo++) {
      if (!c->Ainv[eo]) CK(c->alloc((void**)&c->Ainv[eo], (size_t)36 * c->g.stride * sizeof(double2)));
      launch_ainv_from_b(c->g, c->Ainv[eo], c->B[eo], c->stream);
      CKL();
      c->have_Ainv[eo] = true;
    }
  }
  for (int k = 0; k < 3; k++) c->clover_s_ok[k] = false;
  c->g.clover_t = c->g12.clover_t = 0;
  CK(cudaStreamSynchronize(c->stream));
  return BQCDG_OK;
}

int bqcdg_load_clover_solver(bqcdg_ctx* c, const double* a, const double* ainv) {
  if (!c || !a || !ainv) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->stream));
  // only A of the even sites and A^-1 of the odd ones; the parts the even-odd
  // operator does not read are released
  double2** unused[4] = {&c->A[1], &c->Ainv[0], &c->B[0], &c->B[1]};
  for (double2** f : unused) {
    c->release(*f);
    *f = nullptr;
  }
  c->have_A[1] = c->have_Ainv[0] = c->have_B[0] = c->have_B[1] = false;
  int st;
  if ((st = load_clover_field(c, c->A, c->have_A, a, 0, 0))) return st;
  if ((st = load_clover_field(c, c->Ainv, c->have_Ainv, ainv, 1, 1))) return st;
  for (int k = 0; k < 3; k++) c->clover_s_ok[k] = false;
  c->g.clover_t = c->g12.clover_t = 0;
  CK(cudaStreamSynchronize(c->stream));
  return BQCDG_OK;
}

static int get_clover_field(bqcdg_ctx* c, double2** srcs, const bool* have, double* dst) {
  for (int eo = 0; eo < 2; eo++) {
    if (!have[eo]) return BQCDG_ENOCLOVER;
    CK(c->stage((size_t)c->g.volh * 36 * sizeof(double2)));
    launch_clover_to_fortran(c->g, c->staging, srcs[eo], c->stream);
    CKL();
    CK(cudaMemcpyAsync(dst + (size_t)eo * c->g.volh * 72, c->staging, (size_t)c->g.volh * 36 * sizeof(double2),
                       cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  return BQCDG_OK;
}

int bqcdg_get_clover(bqcdg_ctx* c, double* a, double* ainv, double* b) {
  // the fields hold T (bqcdg_clover_init_t), not BQCD's blocks
  if (c && c->g.clover_t) return BQCDG_EUNSUPPORTED;
  if (!c) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  int st;
  if (a && (st = get_clover_field(c, c->A, c->have_A, a))) return st;
  if (ainv && (st = get_clover_field(c, c->Ainv, c->have_Ainv, ainv))) return st;
  if (b && (st = get_clover_field(c, c->B, c->have_B, b))) return st;
  return BQCDG_OK;
}

int bqcdg_clover_init(bqcdg_ctx* c, double csw_kappa) {
  if (!c) return BQCDG_EINVAL;
  if (!c->have_gauge) return BQCDG_ENOGAUGE;
  CK(cudaSetDevice(c->device));
  size_t n = (size_t)36 * c->g.stride * sizeof(double2);
  for (int eo = 0; eo < 2; eo++) {
    if (!c->A[eo]) CK(c->alloc((void**)&c->A[eo], n));
    if (!c->Ainv[eo]) CK(c->alloc((void**)&c->Ainv[eo], n));
    if (!c->B[eo]) CK(c->alloc((void**)&c->B[eo], n));
  }
  if (!c->clov_tmp) CK(c->alloc((void**)&c->clov_tmp, (size_t)54 * clover_init_chunk(c->g) * sizeof(double2)));
  launch_clover_init(c->g, c->gauge64, csw_kappa, c->A, c->Ainv, c->B, c->clov_tmp, c->stream);
  CKL();
  CK(cudaStreamSynchronize(c->stream));
  for (int eo = 0; eo < 2; eo++) c->have_A[eo] = c->have_Ainv[eo] = c->have_B[eo] = true;
  for (int k = 0; k < 3; k++) c->clover_s_ok[k] = false;
  c->g.clover_t = c->g12.clover_t = 0;
  return BQCDG_OK;
}

int bqcdg_clover_init_solver(bqcdg_ctx* c, double csw_kappa) {
  if (!c) return BQCDG_EINVAL;
  if (!c->have_gauge) return BQCDG_ENOGAUGE;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->stream));
  // only A_ee and A_oo^-1; the other four fields are released if present
  double2** unused[4] = {&c->A[1], &c->Ainv[0], &c->B[0], &c->B[1]};
  for (double2** f : unused) {
    c->release(*f);
    *f = nullptr;
  }
  const size_t n = (size_t)36 * c->g.stride * sizeof(double2);
  if (!c->A[0]) CK(c->alloc((void**)&c->A[0], n));
  if (!c->Ainv[1]) CK(c->alloc((void**)&c->Ainv[1], n));
  double2* a[2] = {c->A[0], nullptr};
  double2* ai[2] = {nullptr, c->Ainv[1]};
  double2* b[2] = {nullptr, nullptr};
  if (!c->clov_tmp) CK(c->alloc((void**)&c->clov_tmp, (size_t)54 * clover_init_chunk(c->g) * sizeof(double2)));
  launch_clover_init(c->g, c->gauge64, csw_kappa, a, ai, b, c->clov_tmp, c->stream);
  CKL();
  CK(cudaStreamSynchronize(c->stream));
  c->have_A[0] = c->have_Ainv[1] = true;
  c->have_A[1] = c->have_Ainv[0] = c->have_B[0] = c->have_B[1] = false;
  for (int k = 0; k < 3; k++) c->clover_s_ok[k] = false;
  c->g.clover_t = c->g12.clover_t = 0;
  return BQCDG_OK;
}

int bqcdg_clover_action(bqcdg_ctx* c, int eo, double* action) {
  if (!c || !action || eo < 0 || eo > 1) return BQCDG_EINVAL;
  if (!c->have_B[eo]) return BQCDG_ENOCLOVER;
  CK(cudaSetDevice(c->device));
  launch_clover_action(c->g, c->B[eo], c->red, c->dres, c->stream);
  CKL();
  CK(cudaMemcpyAsync(c->hres, c->dres, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *action = c->hres[0];
  return BQCDG_OK;
}

static int dslash_host(bqcdg_ctx* c, int e, int o, double* out, const double* in, bool dag) {
  if (!c || !out || !in || e < 0 || e > 1 || o != 1 - e) return BQCDG_EINVAL;
  if (!c->have_gauge) return BQCDG_ENOGAUGE;
  CK(cudaSetDevice(c->device));
  double2* si = c->sp64(0);
  double2* so = c->sp64(1);
  if (!si || !so) return BQCDG_ENOMEM;
  int st = upload_spinor(c, in, si);
  if (st) return st;
  launch_dslash(Prec::F64, c->g, e, dag, S(so), S(si), c->gauge64, c->stream);
  CKL();
  return download_spinor(c, so, out);
}

int bqcdg_d(bqcdg_ctx* c, int e, int o, double* out, const double* in) { return dslash_host(c, e, o, out, in, false); }
int bqcdg_d_dag(bqcdg_ctx* c, int e, int o, double* out, const double* in) {
  return dslash_host(c, e, o, out, in, true);
}

static int clover_host(bqcdg_ctx* c, int eo, double* out, const double* in, int which) {
  // the fields hold T (bqcdg_clover_init_t), not BQCD's blocks
  if (c && c->g.clover_t) return BQCDG_EUNSUPPORTED;
  if (!c || !out || !in || eo < 0 || eo > 1) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  double2* si = c->sp64(0);
  if (!si) return BQCDG_ENOMEM;
  double2* blk = which == 0 ? c->A[eo] : (which == 1 ? c->Ainv[eo] : c->B[eo]);
  bool have = which == 0 ? c->have_A[eo] : (which == 1 ? c->have_Ainv[eo] : c->have_B[eo]);
  if (!have) return BQCDG_ENOCLOVER;
  int st = upload_spinor(c, in, si);
  if (st) return st;
  if (which == 2) launch_clover_mult_b(c->g, si, blk, c->stream);
  else launch_clover_mult(Prec::F64, c->g, S(si), S(si), C(blk), c->stream);
  CKL();
  return download_spinor(c, si, out);
}

int bqcdg_clover_mult_a(bqcdg_ctx* c, int eo, double* out, const double* in) { return clover_host(c, eo, out, in, 0); }
int bqcdg_clover_mult_ao(bqcdg_ctx* c, int eo, double* x) { return clover_host(c, eo, x, x, 1); }
int bqcdg_clover_mult_b(bqcdg_ctx* c, int eo, double* x) { return clover_host(c, eo, x, x, 2); }

// which: 0 mtil, 1 mtil_dag, 2 mtdagmt, 3 w_mult, 4 w_mult_dag, 5 w_dagger_w
static int op_host(bqcdg_ctx* c, double* out, const double* in, const bqcdg_params* p, int which) {
  int st = check_op(c, p);
  if (st) return st;
  if (!out || !in) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  double2 *si = c->sp64(0), *so = c->sp64(1), *t = c->sp64(2), *q = c->sp64(3);
  if (!si || !so || !t || !q) return BQCDG_ENOMEM;
  if ((st = upload_spinor(c, in, si))) return st;
  OpParams op = op_of(p, which >= 3);
  switch (which) {
    case 0: case 3: apply_mtil(c, Prec::F64, false, S(so), S(si), S(t), op, nullptr, nullptr); break;
    case 1: case 4: apply_mtil(c, Prec::F64, true, S(so), S(si), S(t), op, nullptr, nullptr); break;
    default: apply_mdagm(c, Prec::F64, S(so), S(si), S(t), S(q), op);
  }
  CKL();
  return download_spinor(c, so, out);
}

int bqcdg_mtil(bqcdg_ctx* c, double* o, const double* i, const bqcdg_params* p) { return op_host(c, o, i, p, 0); }
int bqcdg_mtil_dag(bqcdg_ctx* c, double* o, const double* i, const bqcdg_params* p) { return op_host(c, o, i, p, 1); }
int bqcdg_mtdagmt(bqcdg_ctx* c, double* o, const double* i, const bqcdg_params* p) { return op_host(c, o, i, p, 2); }
int bqcdg_w_mult(bqcdg_ctx* c, double* o, const double* i, const bqcdg_params* p) { return op_host(c, o, i, p, 3); }
int bqcdg_w_mult_dag(bqcdg_ctx* c, double* o, const double* i, const bqcdg_params* p) {
  return op_host(c, o, i, p, 4);
}
int bqcdg_w_dagger_w(bqcdg_ctx* c, double* o, const double* i, const bqcdg_params* p) {
  return op_host(c, o, i, p, 5);
}

void bqcdg_solver_opts_default(bqcdg_solver_opts* o) {
  if (!o) return;
  o->precision = BQCDG_PREC_HALF;
  o->maxiter = 100000;
  o->relative = 1;
  o->tol = 1e-10;
  o->delta = 0.1;
  o->check_true_residual = 1;
  o->time_kernels = 0;
  o->rhs_per_thread = 0;
}

// x, b device-resident; solver core + optional true-residual check
static int solve_resident(bqcdg_ctx* c, double2* x, double2* b, const bqcdg_params* p, const bqcdg_solver_opts* o,
                          bqcdg_solve_info* info) {
  bqcdg_solve_info tmp;
  if (!info) info = &tmp;
  std::memset(info, 0, sizeof(*info));
  OpParams op = op_of(p, true);
  Prec sl = prec_of(o->precision);
  double stop;
  if (o->relative) {
    // needs |b|^2 first: computed by the residual kernel inside cg_core; use a
    // pre-pass so the stop is known before the first iteration
    launch_norm2(c->g, b, c->red, c->dres, c->stream);
    CKL();
    CK(cudaMemcpyAsync(c->hres, c->dres, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    stop = o->tol * o->tol * c->hres[0];
  } else {
    stop = o->tol;
  }
  int st = cg_robust(c, x, b, op, sl, o->maxiter, stop, o->delta, false, o->time_kernels != 0, info);
  if (st) return st;
  info->kernel_launches += o->relative ? 1 : 0;
  if (o->check_true_residual) {
    info->kernel_launches += 5;
    st = true_residual(c, x, b, op, &info->true_rtr);
    if (st) return st;
    info->converged = info->true_rtr <= stop ? 1 : 0;
  }
  return info->converged ? BQCDG_OK : BQCDG_ENOCONV;
}

int bqcdg_solve(bqcdg_ctx* c, double* x, const double* b, const bqcdg_params* p, const bqcdg_solver_opts* o,
                bqcdg_solve_info* info) {
  int st = check_op(c, p);
  if (st) return st;
  if (!x || !b || !o) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  double2* dx = c->sp64(5);
  double2* db = c->sp64(6);
  if (!dx || !db) return BQCDG_ENOMEM;
  if ((st = upload_spinor(c, x, dx))) return st;
  if ((st = upload_spinor(c, b, db))) return st;
  int rs = solve_resident(c, dx, db, p, o, info);
  if (rs != BQCDG_OK && rs != BQCDG_ENOCONV) return rs;
  if ((st = download_spinor(c, dx, x))) return st;
  return rs;
}

int bqcdg_cg(bqcdg_ctx* c, double* x, const double* b, const bqcdg_params* p, const bqcdg_cg_para* cgp,
             int* iterations, bqcdg_solve_info* info) {
  int st = check_op(c, p);
  if (st) return st;
  if (!x || !b || !cgp) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  bqcdg_solve_info tmp;
  if (!info) info = &tmp;
  std::memset(info, 0, sizeof(*info));
  double2* dx = c->sp64(5);
  double2* db = c->sp64(6);
  if (!dx || !db) return BQCDG_ENOMEM;
  if ((st = upload_spinor(c, x, dx))) return st;
  if ((st = upload_spinor(c, b, db))) return st;
  OpParams op = op_of(p, true);
  st = cg_core(c, dx, db, op, Prec::F64, cgp->maxiter, (double)cgp->rest, 0.0, true, false, info);
  if (st) return st;
  if (iterations) *iterations = info->niter;
  if ((st = download_spinor(c, dx, x))) return st;
  if (!info->converged && cgp->log != 2) return BQCDG_ENOCONV;
  return BQCDG_OK;
}

int bqcdg_quda_solver(bqcdg_ctx* c, double* x, const double* b, const bqcdg_params* p, const bqcdg_cg_para* cgp,
                      int* iterations, bqcdg_solve_info* info) {
  int st = check_op(c, p);
  if (st) return st;
  if (!x || !b || !cgp) return BQCDG_EINVAL;
  if (p->h != 0.0) return BQCDG_EUNSUPPORTED;  // invert_quda.F90:298-301
  CK(cudaSetDevice(c->device));
  bqcdg_solve_info tmp;
  if (!info) info = &tmp;
  std::memset(info, 0, sizeof(*info));
  double2* dx = c->sp64(5);
  double2* db = c->sp64(6);
  if (!dx || !db) return BQCDG_ENOMEM;
  if ((st = upload_spinor(c, x, dx))) return st;
  if ((st = upload_spinor(c, b, db))) return st;
  OpParams op = op_of(p, true);
  // QUDA stops on |r| < sqrt(rest) (L2 absolute, invert_quda.F90:143,342)
  Prec sl = c->gauge_su3 ? Prec::F16 : Prec::F64;
  st = cg_robust(c, dx, db, op, sl, cgp->maxiter, (double)cgp->rest, 0.1, false, false, info);
  if (st) return st;
  // host-side check of invert_quda.F90:155-168, done in FP64 on the device
  if ((st = true_residual(c, dx, db, op, &info->true_rtr))) return st;
  info->converged = info->true_rtr <= (double)cgp->rest ? 1 : 0;
  if (iterations) *iterations = info->niter;
  if ((st = download_spinor(c, dx, x))) return st;
  if (!info->converged && cgp->log != 2) return BQCDG_ENOCONV;
  return BQCDG_OK;
}

// ---------------------------------------------------------------------------
// forces
// ---------------------------------------------------------------------------
}  // extern "C"

namespace bqcdg_host {
int ensure_force_bufs(bqcdg_ctx* c) {
  if (!c->pgen) CK(c->alloc((void**)&c->pgen, (size_t)64 * c->g.volh * sizeof(double)));
  if (!c->wbuf) CK(c->alloc((void**)&c->wbuf, (size_t)54 * c->g.stride * sizeof(double2)));
  return BQCDG_OK;
}
}  // namespace bqcdg_host

extern "C" {

}  // extern "C"

namespace bqcdg_host {
int apply_odd_clover_inverse(bqcdg_ctx* c, double2* x) {
  // clover_mult_b(conf%b(ODD), x) (dsf.F90:69-70); the explicit inverse when
  // only conf%i is resident
  if (c->have_B[1]) launch_clover_mult_b(c->g, x, c->B[1], c->stream);
  else if (c->have_Ainv[1]) launch_clover_mult(Prec::F64, c->g, S(x), S(x), C(c->Ainv[1]), c->stream);
  else return BQCDG_ENOCLOVER;
  CKL();
  return BQCDG_OK;
}
}  // namespace bqcdg_host

extern "C" {

// dsf.F90:28-110 on device momenta p (GENERATOR_FIELD layout) from the
// device spinors a, b: the hopping force of every link, then the clover
// parts of both parities.  Uses scratch spinors 2 and 3.
}  // extern "C"

namespace bqcdg_host {
int dsf_core(bqcdg_ctx* c, double* p, double step, const bqcdg_params* par, double2* da, double2* db) {
  // the fields hold T (bqcdg_clover_init_t), not BQCD's blocks
  if (c && c->g.clover_t) return BQCDG_EUNSUPPORTED;
  int st = ensure_force_bufs(c);
  if (st) return st;
  double2 *dat = c->sp64(2), *dbt = c->sp64(3);
  if (!dat || !dbt) return BQCDG_ENOMEM;
  if (par->kappa != 0.0) {
    launch_dslash(Prec::F64, c->g, 1, false, S(dat), S(da), c->gauge64, c->stream);  // A~ = D_oe A
    launch_dslash(Prec::F64, c->g, 1, true, S(dbt), S(db), c->gauge64, c->stream);   // B~ = D_eo^+ B
    CKL();
    if (par->csw_kappa != 0.0) {
      if ((st = apply_odd_clover_inverse(c, dat))) return st;
      if ((st = apply_odd_clover_inverse(c, dbt))) return st;
    }
    if (par->h != 0.0) {
      launch_h_mult_b(c->g, dat, -par->h, c->stream);
      launch_h_mult_b(c->g, dbt, par->h, c->stream);
      CKL();
    }
  }
  double s = -step * 2.0 * par->kappa * par->kappa / (1.0 + par->h * par->h);
  if (s != 0.0) {
    launch_dsf_hop(c->g, p, c->gauge64, da, db, dat, dbt, s, c->stream);
    CKL();
  }
  double s1 = -step * 2.0 * (par->csw_kappa / 8.0);
  double s2 = -step * 2.0 * (par->csw_kappa / 8.0) * par->kappa * par->kappa;
  if (s1 != 0.0) {
    launch_clover_bsa(c->g, c->wbuf, db, da, c->stream);
    launch_clover_d(c->g, p, c->gauge64, c->wbuf, 0, s1, c->stream);
    CKL();
  }
  if (s2 != 0.0) {
    launch_clover_bsa(c->g, c->wbuf, dbt, dat, c->stream);
    launch_clover_d(c->g, p, c->gauge64, c->wbuf, 1, s2, c->stream);
    CKL();
  }
  return BQCDG_OK;
}
}  // namespace bqcdg_host

extern "C" {

int bqcdg_dsf(bqcdg_ctx* c, double* p, double step, const bqcdg_params* par, const double* a, const double* b) {
  if (!c || !p || !par || !a || !b) return BQCDG_EINVAL;
  if (!c->have_gauge) return BQCDG_ENOGAUGE;
  CK(cudaSetDevice(c->device));
  int st = ensure_force_bufs(c);
  if (st) return st;
  double2 *da = c->sp64(0), *db = c->sp64(1);
  if (!da || !db) return BQCDG_ENOMEM;
  size_t pn = (size_t)64 * c->g.volh * sizeof(double);
  CK(cudaMemcpyAsync(c->pgen, p, pn, cudaMemcpyHostToDevice, c->stream));
  if ((st = upload_spinor(c, a, da))) return st;
  if ((st = upload_spinor(c, b, db))) return st;
  if ((st = dsf_core(c, c->pgen, step, par, da, db))) return st;
  CK(cudaMemcpyAsync(p, c->pgen, pn, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return BQCDG_OK;
}

int bqcdg_clover_dsf(bqcdg_ctx* c, int eo, double* p, const double* b, const double* a, double s) {
  if (!c || !p || !b || !a || eo < 0 || eo > 1) return BQCDG_EINVAL;
  if (!c->have_gauge) return BQCDG_ENOGAUGE;
  CK(cudaSetDevice(c->device));
  int st = ensure_force_bufs(c);
  if (st) return st;
  double2 *da = c->sp64(0), *db = c->sp64(1);
  if (!da || !db) return BQCDG_ENOMEM;
  size_t pn = (size_t)64 * c->g.volh * sizeof(double);
  CK(cudaMemcpyAsync(c->pgen, p, pn, cudaMemcpyHostToDevice, c->stream));
  if ((st = upload_spinor(c, a, da))) return st;
  if ((st = upload_spinor(c, b, db))) return st;
  launch_clover_bsa(c->g, c->wbuf, db, da, c->stream);
  launch_clover_d(c->g, c->pgen, c->gauge64, c->wbuf, eo, s, c->stream);
  CKL();
  CK(cudaMemcpyAsync(p, c->pgen, pn, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return BQCDG_OK;
}

// clover_d.F90:40-75 on device momenta: the det-term force of parity eo
}  // extern "C"

namespace bqcdg_host {
int dsd_core(bqcdg_ctx* c, double* p, int eo, double s) {
  // the fields hold T (bqcdg_clover_init_t), not BQCD's blocks
  if (c && c->g.clover_t) return BQCDG_EUNSUPPORTED;
  launch_clover_ts(c->g, c->wbuf, c->Ainv[eo], c->stream);
  launch_clover_d(c->g, p, c->gauge64, c->wbuf, eo, s, c->stream);
  CKL();
  return BQCDG_OK;
}
}  // namespace bqcdg_host

extern "C" {

int bqcdg_clover_dsd(bqcdg_ctx* c, int eo, double* p, double s) {
  if (!c || !p || eo < 0 || eo > 1) return BQCDG_EINVAL;
  if (!c->have_gauge) return BQCDG_ENOGAUGE;
  if (!c->have_Ainv[eo]) return BQCDG_ENOCLOVER;
  CK(cudaSetDevice(c->device));
  int st = ensure_force_bufs(c);
  if (st) return st;
  size_t pn = (size_t)64 * c->g.volh * sizeof(double);
  CK(cudaMemcpyAsync(c->pgen, p, pn, cudaMemcpyHostToDevice, c->stream));
  if ((st = dsd_core(c, c->pgen, eo, s))) return st;
  CK(cudaMemcpyAsync(p, c->pgen, pn, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return BQCDG_OK;
}

// ---------------------------------------------------------------------------
// device-resident fields
// ---------------------------------------------------------------------------
int bqcdg_field_create(bqcdg_ctx* c, int* handle) {
  if (!c || !handle) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  void* p = nullptr;
  CK(c->alloc(&p, c->spin_bytes(Prec::F64)));
  CK(cudaMemsetAsync(p, 0, c->spin_bytes(Prec::F64), c->stream));
  *handle = c->next_handle++;
  c->fields[*handle] = (double2*)p;
  return BQCDG_OK;
}

}  // extern "C"

namespace bqcdg_host {
double2* field(bqcdg_ctx* c, int h) {
  auto it = c->fields.find(h);
  return it == c->fields.end() ? nullptr : it->second;
}
}  // namespace bqcdg_host

extern "C" {

int bqcdg_field_upload(bqcdg_ctx* c, int h, const double* host) {
  if (!c || !host || !field(c, h)) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  int st = upload_spinor(c, host, field(c, h));
  if (st) return st;
  CK(cudaStreamSynchronize(c->stream));
  return BQCDG_OK;
}

int bqcdg_field_download(bqcdg_ctx* c, int h, double* host) {
  if (!c || !host || !field(c, h)) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  return download_spinor(c, field(c, h), host);
}

int bqcdg_field_destroy(bqcdg_ctx* c, int h) {
  if (!c || !field(c, h)) return BQCDG_EINVAL;
  // memory stays in the context pool until bqcdg_destroy
  c->fields.erase(h);
  return BQCDG_OK;
}

int bqcdg_field_gauss(bqcdg_ctx* c, int h, double var) {
  if (!c || !field(c, h)) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  CK(c->stage((size_t)c->g.volh * 12 * sizeof(double2)));
  launch_ran_gauss(c->staging, c->g.volh, 12, var, c->seed, c->stream);
  c->seed = ranf_skip(c->seed, 2ull * 12ull * (unsigned long long)c->g.volh);
  launch_spinor_from_fortran(c->g, field(c, h), c->staging, c->stream);
  CKL();
  CK(cudaStreamSynchronize(c->stream));
  return BQCDG_OK;
}

// ---------------------------------------------------------------------------
// seeded gauge fields
// ---------------------------------------------------------------------------
int bqcdg_ranset(bqcdg_ctx* c, long long seed, long long skip) {
  if (!c) return BQCDG_EINVAL;
  const unsigned long long M48 = 281474976710655ull;
  c->seed = seed == 0 ? 48131768981101ull : (((unsigned long long)seed | 1ull) & M48);
  c->seed = ranf_skip(c->seed, (unsigned long long)skip & M48);
  return BQCDG_OK;
}

int bqcdg_ranget(bqcdg_ctx* c, long long* seed) {
  if (!c || !seed) return BQCDG_EINVAL;
  *seed = (long long)c->seed;
  return BQCDG_OK;
}

static int gauge_finish(bqcdg_ctx* c) {
  launch_gauge_from_fortran(c->g, c->gauge64, c->staging, 0, c->stream);
  CKL();
  launch_gauge_check(c->g, c->gauge64, c->red, c->dres, c->stream);
  CKL();
  CK(cudaMemcpyAsync(c->hres, c->dres, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->gauge_su3 = c->hres[0] < 1e-10 && c->hres[1] < 1e-10;
  c->have_gauge = true;
  for (int k = 0; k < 3; k++) c->gauge_s_ok[k] = false;
  c->gauge64r_ok = false;
  return BQCDG_OK;
}

int bqcdg_conf_hot(bqcdg_ctx* c) {
  if (!c) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  if (!c->gauge64) CK(c->alloc((void**)&c->gauge64, (size_t)8 * 9 * c->g.stride * sizeof(double2)));
  CK(c->stage((size_t)c->g.volh * 72 * sizeof(double2)));
  const unsigned long long per = 2ull * 9ull * (unsigned long long)c->g.volh;
  for (int me = 0; me < 8; me++) {  // do mu; do eo (conf.F90:208-214)
    launch_ran_gauss(c->staging + (size_t)me * c->g.volh * 9, c->g.volh, 9, 1.0, c->seed, c->stream);
    c->seed = ranf_skip(c->seed, per);
  }
  launch_u_normalize(c->staging, 8LL * c->g.volh, c->stream);
  CKL();
  return gauge_finish(c);
}

int bqcdg_conf_cold(bqcdg_ctx* c) {
  if (!c) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  if (!c->gauge64) CK(c->alloc((void**)&c->gauge64, (size_t)8 * 9 * c->g.stride * sizeof(double2)));
  CK(c->stage((size_t)c->g.volh * 72 * sizeof(double2)));
  launch_cold(c->staging, 8LL * c->g.volh, c->stream);
  CKL();
  return gauge_finish(c);
}

int bqcdg_conf_relax(bqcdg_ctx* c, int n) {
  if (!c || n < 0) return BQCDG_EINVAL;
  if (!c->have_gauge) return BQCDG_ENOGAUGE;
  CK(cudaSetDevice(c->device));
  for (int k = 0; k < n; k++) launch_conf_relax(c->g, c->gauge64, c->stream);
  CKL();
  CK(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < 3; k++) c->gauge_s_ok[k] = false;
  c->gauge64r_ok = false;
  return BQCDG_OK;
}

int bqcdg_sg(bqcdg_ctx* c, double* sg) {
  if (!c || !sg) return BQCDG_EINVAL;
  if (!c->have_gauge) return BQCDG_ENOGAUGE;
  CK(cudaSetDevice(c->device));
  launch_plaquette(c->g, c->gauge64, c->red, c->dres, c->stream);
  CKL();
  CK(cudaMemcpyAsync(c->hres, c->dres, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *sg = 6.0 * 2.0 * c->g.volh - c->hres[0] / 3.0;
  return BQCDG_OK;
}

int bqcdg_solve_dev(bqcdg_ctx* c, int hx, int hb, const bqcdg_params* p, const bqcdg_solver_opts* o,
                    bqcdg_solve_info* info) {
  int st = check_op(c, p);
  if (st) return st;
  if (!o || !field(c, hx) || !field(c, hb)) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  return solve_resident(c, field(c, hx), field(c, hb), p, o, info);
}

// rho: one shift per right-hand side (null: p->rho for all); tol: one
// tolerance per right-hand side (null: o->tol for all)
static int solve_batch(bqcdg_ctx* c, int nrhs, const int* hx, const int* hb, const bqcdg_params* p,
                       const double* rho, const double* tol, const bqcdg_solver_opts* o, int block,
                       bqcdg_solve_info* infos, const double* kappa = nullptr) {
  int st = check_op(c, p);
  if (st) return st;
  if (!o || !hx || !hb || !infos || nrhs <= 0 || block < 0 || block > kMaxRhs) return BQCDG_EINVAL;
  if (o->rhs_per_thread != 0 && o->rhs_per_thread != 1 && o->rhs_per_thread != 2 && o->rhs_per_thread != 4)
    return BQCDG_EINVAL;
  if (rho)
    for (int k = 0; k < nrhs; k++)
      if (!(rho[k] == rho[k])) return BQCDG_EINVAL;
  if (tol)
    for (int k = 0; k < nrhs; k++)
      if (!(tol[k] >= 0.0)) return BQCDG_EINVAL;
  if (kappa)
    for (int k = 0; k < nrhs; k++)
      if (!(kappa[k] > 0.0)) return BQCDG_EINVAL;
  // kappa per right-hand side with the clover term needs T (bqcdg_clover_init_t)
  if (kappa && p->csw_kappa != 0.0 && !c->g.clover_t) return BQCDG_ENOCLOVER;
  for (int k = 0; k < nrhs; k++)
    if (!field(c, hx[k]) || !field(c, hb[k])) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  OpParams op = op_of(p, true);
  Prec sl = prec_of(o->precision);
  if (sl == Prec::F64) return BQCDG_EUNSUPPORTED;  // the batched path is the mixed-precision one
  std::memset(infos, 0, sizeof(bqcdg_solve_info) * nrhs);
  if (block == 0) {
    int k = (int)sl;
    if (!c->tuned_block[k] && (st = tune_block(c, sl, op, kMaxRhs, &c->tuned_block[k]))) return st;
    block = c->tuned_block[k];
  }
  std::vector<double> stop(nrhs);
  for (int k = 0; k < nrhs; k++) {
    const double t = tol ? tol[k] : o->tol;
    if (o->relative) {
      launch_norm2(c->g, field(c, hb[k]), c->red, c->dres, c->stream);
      CKL();
      CK(cudaMemcpyAsync(c->hres, c->dres, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      stop[k] = t * t * c->hres[0];
    } else {
      stop[k] = t;
    }
  }
  bool all_conv = true;
  for (int k0 = 0; k0 < nrhs; k0 += block) {
    int nb = nrhs - k0 < block ? nrhs - k0 : block;
    std::vector<double2*> xs(nb), bs(nb);
    for (int k = 0; k < nb; k++) {
      xs[k] = field(c, hx[k0 + k]);
      bs[k] = field(c, hb[k0 + k]);
    }
    st = cg_batch(c, xs.data(), bs.data(), nb, op, sl, o->maxiter, stop.data() + k0, o->delta, infos + k0,
                  rho ? rho + k0 : nullptr, o->rhs_per_thread, kappa ? kappa + k0 : nullptr);
    if (st) return st;
    for (int k = 0; k < nb; k++) {
      bqcdg_solve_info& in = infos[k0 + k];
      if (o->check_true_residual) {
        OpParams opk = op;
        if (rho) opk.rho = rho[k0 + k];
        if (kappa) opk.kappa = kappa[k0 + k];
        if ((st = true_residual(c, xs[k], bs[k], opk, &in.true_rtr))) return st;
        in.converged = in.true_rtr <= stop[k0 + k] ? 1 : 0;
      }
      all_conv = all_conv && in.converged;
    }
  }
  return all_conv ? BQCDG_OK : BQCDG_ENOCONV;
}

int bqcdg_solve_batch(bqcdg_ctx* c, int nrhs, const int* hx, const int* hb, const bqcdg_params* p,
                      const bqcdg_solver_opts* o, int block, bqcdg_solve_info* infos) {
  return solve_batch(c, nrhs, hx, hb, p, nullptr, nullptr, o, block, infos);
}

int bqcdg_solve_batch_shifted(bqcdg_ctx* c, int nrhs, const int* hx, const int* hb, const bqcdg_params* p,
                              const double* rho, const double* tol, const bqcdg_solver_opts* o, int block,
                              bqcdg_solve_info* infos) {
  if (!rho) return BQCDG_EINVAL;
  return solve_batch(c, nrhs, hx, hb, p, rho, tol, o, block, infos);
}

int bqcdg_solve_batch_kappa(bqcdg_ctx* c, int nrhs, const int* hx, const int* hb, const bqcdg_params* p,
                            const double* kappa, const double* rho, const double* tol, const bqcdg_solver_opts* o,
                            int block, bqcdg_solve_info* infos) {
  if (!kappa) return BQCDG_EINVAL;
  return solve_batch(c, nrhs, hx, hb, p, rho, tol, o, block, infos, kappa);
}

int bqcdg_clover_init_t(bqcdg_ctx* c, double csw) {
  if (!c) return BQCDG_EINVAL;
  return clover_init_t(c, csw);
}

int bqcdg_mdagm_dev(bqcdg_ctx* c, int hout, int hin, const bqcdg_params* p, int precision, int n, double* ms) {
  int st = check_op(c, p);
  if (st) return st;
  if (!field(c, hout) || !field(c, hin) || n <= 0) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  Prec pr = prec_of(precision);
  OpParams op = op_of(p, true);
  SpinorPtr in, out, t, q;
  if (pr == Prec::F64) {
    in = S(field(c, hin));
    out = S(field(c, hout));
    t = S(c->sp64(2));
    q = S(c->sp64(3));
  } else {
    if ((st = ensure_sloppy(c, pr, p->csw_kappa != 0.0))) return st;
    in = c->sp(pr, 5);
    out = c->sp(pr, 6);
    t = c->sp(pr, 7);
    q = c->sp(pr, 8);
    launch_spinor_convert(c->g, pr, in, Prec::F64, S(field(c, hin)), c->stream);
  }
  CK(cudaEventRecord(c->ev0, c->stream));
  for (int k = 0; k < n; k++) apply_mdagm(c, pr, out, in, t, q, op);
  CK(cudaEventRecord(c->ev1, c->stream));
  CKL();
  if (pr != Prec::F64) launch_spinor_convert(c->g, Prec::F64, S(field(c, hout)), pr, out, c->stream);
  CK(cudaStreamSynchronize(c->stream));
  float t_ms = 0.f;
  cudaEventElapsedTime(&t_ms, c->ev0, c->ev1);
  if (ms) *ms = t_ms / n;
  return BQCDG_OK;
}

int bqcdg_time_pass(bqcdg_ctx* c, int hin, const bqcdg_params* p, int precision, int n, double* ms) {
  int st = check_op(c, p);
  if (st) return st;
  if (!field(c, hin) || n <= 0) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  Prec pr = prec_of(precision);
  OpParams op = op_of(p, true);
  SpinorPtr in, t;
  if (pr == Prec::F64) {
    in = S(field(c, hin));
    t = S(c->sp64(2));
  } else {
    if ((st = ensure_sloppy(c, pr, p->csw_kappa != 0.0))) return st;
    in = c->sp(pr, 5);
    t = c->sp(pr, 7);
    launch_spinor_convert(c->g, pr, in, Prec::F64, S(field(c, hin)), c->stream);
  }
  CK(cudaEventRecord(c->ev0, c->stream));
  for (int k = 0; k < n; k++)
    launch_mtil_pass1(pr, geom_of(c, pr), false, t, in, gauge_of(c, pr), ainv_of(c, pr), op, nullptr, c->stream);
  CK(cudaEventRecord(c->ev1, c->stream));
  CKL();
  CK(cudaStreamSynchronize(c->stream));
  float t_ms = 0.f;
  cudaEventElapsedTime(&t_ms, c->ev0, c->ev1);
  if (ms) *ms = t_ms / n;
  return BQCDG_OK;
}

int bqcdg_time_pass_batch(bqcdg_ctx* c, int nrhs, const int* hin, const bqcdg_params* p, int precision,
                          int rhs_per_thread, int n, double* ms) {
  int st = check_op(c, p);
  if (st) return st;
  if (!hin || nrhs <= 0 || nrhs > kMaxRhs || n <= 0) return BQCDG_EINVAL;
  if (rhs_per_thread != 0 && rhs_per_thread != 1 && rhs_per_thread != 2 && rhs_per_thread != 4) return BQCDG_EINVAL;
  if (rhs_per_thread > 1 && (p->h != 0.0 || c->g.clover_t)) return BQCDG_EUNSUPPORTED;
  for (int k = 0; k < nrhs; k++)
    if (!field(c, hin[k])) return BQCDG_EINVAL;
  Prec pr = prec_of(precision);
  if (pr == Prec::F64) return BQCDG_EUNSUPPORTED;  // batches are sloppy-precision
  CK(cudaSetDevice(c->device));
  OpParams op = op_of(p, true);
  if ((st = ensure_sloppy(c, pr, p->csw_kappa != 0.0))) return st;
  if ((st = ensure_batch(c, pr, nrhs))) return st;
  auto& B = c->batch;
  for (int k = 0; k < nrhs; k++) launch_spinor_convert(c->g, pr, rhs_of(B.p, k), Prec::F64, S(field(c, hin[k])), c->stream);
  CKL();
  int nbt = rhs_per_thread;
  if (nbt == 0 && (st = tune_nbt(c, pr, op, nrhs, &nbt))) return st;
  if (nbt > nrhs) nbt = 1;
  float t_ms = 0.f;
  if ((st = time_pass1(c, pr, op, nrhs, nbt, n, &t_ms))) return st;
  if (ms) *ms = t_ms;
  return BQCDG_OK;
}

}  // extern "C"
