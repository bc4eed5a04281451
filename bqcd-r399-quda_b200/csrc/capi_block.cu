// capi_block.cu -- block conjugate gradients over up to 16 right-hand sides
// that share one operator (bqcdg_solve_block): one Krylov space for all of
// them, so each iteration searches along s directions at once and the
// iteration count drops below that of s separate solves.
//
// The recurrence is O'Leary's block CG in Dubrulle's "residual QR" form
// (BCGrQ, 2001), which keeps the search block well conditioned: with
// R = Q C (Q orthonormal, C upper triangular s x s)
//   Z = A P,  Psi = (P^H Z)^-1,  X += P Psi C,
//   Q Xi = qr(Q - Z Psi),  P = Q + P Xi^H,  C = Xi C,
// and |r_j| = |C e_j|.  The blocks are FP32 fields; each solution gathers
// in FP32 between restarts and in FP64 at them.  A restart recomputes every
// residual in FP64 (the reliable update of the single-vector solver, here for
// the whole block), retires the systems that have reached their tolerance,
// and starts the recurrence again from the QR of the remaining residuals.
// It comes when the largest residual of the block has dropped by delta since
// the last restart, when every iterated residual is below its tolerance, or
// when the QR breaks down.  Gram matrices are FP64 sums; the s x s algebra
// (Cholesky QR, done twice for orthogonality, and the inverse of P^H Z) runs
// on the host.
#include <complex>

#include "ctx.cuh"

using namespace bqcdg_host;

namespace {

using zc = std::complex<double>;

struct Dense {
  int n;
  std::vector<zc> a;  // row-major n x n
  explicit Dense(int n_ = 0) : n(n_), a((size_t)n_ * n_) {}
  zc& operator()(int i, int j) { return a[(size_t)i * n + j]; }
  zc operator()(int i, int j) const { return a[(size_t)i * n + j]; }
  static Dense eye(int n) {
    Dense d(n);
    for (int i = 0; i < n; i++) d(i, i) = 1.0;
    return d;
  }
};

Dense mul(const Dense& x, const Dense& y) {
  Dense z(x.n);
  for (int i = 0; i < x.n; i++)
    for (int k = 0; k < x.n; k++)
      for (int j = 0; j < x.n; j++) z(i, j) += x(i, k) * y(k, j);
  return z;
}
Dense herm(const Dense& x) {
  Dense z(x.n);
  for (int i = 0; i < x.n; i++)
    for (int j = 0; j < x.n; j++) z(i, j) = std::conj(x(j, i));
  return z;
}
// W = L L^H (L lower); false if W is not numerically positive definite
bool cholesky(const Dense& w, Dense& l) {
  const int n = w.n;
  l = Dense(n);
  double dmax = 0.0;
  for (int i = 0; i < n; i++) dmax = std::max(dmax, w(i, i).real());
  for (int j = 0; j < n; j++) {
    double d = w(j, j).real();
    for (int k = 0; k < j; k++) d -= std::norm(l(j, k));
    if (!(d > 1e-24 * dmax)) return false;
    l(j, j) = std::sqrt(d);
    for (int i = j + 1; i < n; i++) {
      zc s = w(i, j);
      for (int k = 0; k < j; k++) s -= l(i, k) * std::conj(l(j, k));
      l(i, j) = s / l(j, j).real();
    }
  }
  return true;
}
// inverse of an upper triangular matrix
Dense inv_upper(const Dense& r) {
  const int n = r.n;
  Dense x(n);
  for (int j = 0; j < n; j++) {
    x(j, j) = 1.0 / r(j, j);
    for (int i = j - 1; i >= 0; i--) {
      zc s = 0.0;
      for (int k = i + 1; k <= j; k++) s += r(i, k) * x(k, j);
      x(i, j) = -s / r(i, i);
    }
  }
  return x;
}

using BlockState = bqcdg_ctx::BlockCg;

int ensure_block(bqcdg_ctx* c, BlockState& bs, int s) {
  if (bs.cap >= s) return BQCDG_OK;
  for (SpinorPtr* p : {&bs.P, &bs.Q, &bs.Z, &bs.M, &bs.Xs, &bs.T, &bs.Qe}) {
    c->release(p->v);
    *p = SpinorPtr{};
  }
  for (SpinorPtr* p : {&bs.P, &bs.Q, &bs.Z, &bs.M, &bs.Xs, &bs.T, &bs.Qe}) {
    p->rsb = (long long)c->spin_bytes(Prec::F32);
    CK(c->alloc(&p->v, (size_t)p->rsb * s));
    CK(cudaMemsetAsync(p->v, 0, (size_t)p->rsb * s, c->stream));
  }
  if (!bs.partial) CK(c->alloc((void**)&bs.partial, sizeof(double2) * block_gram_scratch_pairs()));
  if (!bs.gram) CK(c->alloc((void**)&bs.gram, sizeof(double2) * 256));
  if (!bs.mats) CK(c->alloc((void**)&bs.mats, sizeof(float2) * 512));
  bs.cap = s;
  return BQCDG_OK;
}

// host Gram matrix <a_i, b_j> of two blocks of s fields
int gram(bqcdg_ctx* c, BlockState& bs, int s, SpinorPtr a, SpinorPtr b, Dense& out) {
  launch_block_gram(c->g, s, a, b, bs.partial, bs.gram, c->stream);
  CKL();
  std::vector<double2> h((size_t)s * s);
  CK(cudaMemcpyAsync(h.data(), bs.gram, sizeof(double2) * s * s, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  out = Dense(s);
  for (int i = 0; i < s; i++)
    for (int j = 0; j < s; j++) out(i, j) = zc(h[(size_t)i * s + j].x, h[(size_t)i * s + j].y);
  return BQCDG_OK;
}

// out = in1 m1 (+ in2 m2)
int combine(bqcdg_ctx* c, BlockState& bs, int s, SpinorPtr out, SpinorPtr in1, const Dense& m1, SpinorPtr in2,
            const Dense* m2) {
  std::vector<float2> h(512);
  for (int i = 0; i < s * s; i++) h[i] = make_float2((float)m1.a[i].real(), (float)m1.a[i].imag());
  if (m2)
    for (int i = 0; i < s * s; i++) h[256 + i] = make_float2((float)m2->a[i].real(), (float)m2->a[i].imag());
  CK(cudaMemcpyAsync(bs.mats, h.data(), sizeof(float2) * 512, cudaMemcpyHostToDevice, c->stream));
  launch_block_combine(c->g, s, out, in1, bs.mats, m2 ? in2 : SpinorPtr{}, bs.mats + 256, c->stream);
  CKL();
  // the staging array is reused by the next combination: wait for this one
  CK(cudaStreamSynchronize(c->stream));
  return BQCDG_OK;
}

// Q R = M with Q orthonormal (Cholesky QR twice); false: M is rank deficient
int qr2(bqcdg_ctx* c, BlockState& bs, int s, SpinorPtr m, SpinorPtr q, Dense& r, bool& ok) {
  ok = false;
  Dense w, l;
  int st = gram(c, bs, s, m, m, w);
  if (st) return st;
  if (!cholesky(w, l)) return BQCDG_OK;
  Dense r1 = herm(l);
  if ((st = combine(c, bs, s, q, m, inv_upper(r1), SpinorPtr{}, nullptr))) return st;
  if ((st = gram(c, bs, s, q, q, w))) return st;
  if (!cholesky(w, l)) return BQCDG_OK;
  Dense r2 = herm(l);
  if ((st = combine(c, bs, s, q, q, inv_upper(r2), SpinorPtr{}, nullptr))) return st;
  r = mul(r2, r1);
  ok = true;
  return BQCDG_OK;
}

}  // namespace

extern "C" int bqcdg_solve_block(bqcdg_ctx* c, int nrhs, const int* hx, const int* hb, const bqcdg_params* p,
                                 const bqcdg_solver_opts* o, bqcdg_solve_info* infos) {
  int st = check_op(c, p);
  if (st) return st;
  if (!o || !hx || !hb || !infos || nrhs <= 0 || nrhs > kMaxRhs) return BQCDG_EINVAL;
  if (o->precision != BQCDG_PREC_SINGLE) return BQCDG_EUNSUPPORTED;  // FP32 blocks, FP64 restarts
  for (int k = 0; k < nrhs; k++)
    if (!field(c, hx[k]) || !field(c, hb[k])) return BQCDG_EINVAL;
  CK(cudaSetDevice(c->device));
  const Geom& g = c->g;
  const OpParams op = op_of(p, true);
  if ((st = ensure_sloppy(c, Prec::F32, op.csw_kappa != 0.0))) return st;
  BlockState& bs = c->blk;
  if ((st = ensure_block(c, bs, nrhs))) return st;
  std::memset(infos, 0, sizeof(bqcdg_solve_info) * nrhs);
  double2* r64 = c->sp64(0);
  double2* ax = c->sp64(1);
  if (!r64 || !ax || !c->sp64(2) || !c->sp64(3)) return BQCDG_ENOMEM;
  std::vector<double> stop(nrhs), b2(nrhs);
  std::vector<int> active;  // systems still in the block, by block column
  for (int k = 0; k < nrhs; k++) active.push_back(k);
  CK(cudaEventRecord(c->ev0, c->stream));
  int iter = 0, restarts = 0, launches = 0;
  const double delta2 = o->delta * o->delta;
  bool first = true;
  int idle = 0;  // restarts in a row after which the recurrence made no step
  int prev_s = 0;
  bool keep_dirs = false;  // the search block of the last recurrence is valid
  while (!active.empty()) {
    // ---- restart: x += x_s, r = b - A x in FP64 for every system in the block
    std::vector<int> keep;
    for (size_t j = 0; j < active.size(); j++) {
      const int k = active[j];
      double2* x = field(c, hx[k]);
      double2* b = field(c, hb[k]);
      if (!first) launch_accum_x(g, x, (float4*)rhs_of(bs.Xs, (int)j).v, c->stream);
      apply_mdagm(c, Prec::F64, S(ax), S(x), S(c->sp64(2)), S(c->sp64(3)), op);
      launch_residual(g, r64, b, ax, Prec::F32, rhs_of(bs.M, (int)keep.size()), c->red, c->dres, c->stream);
      CKL();
      launches += 7;
      CK(cudaMemcpyAsync(c->hres, c->dres, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      if (first) {
        b2[k] = c->hres[1];
        stop[k] = o->relative ? o->tol * o->tol * b2[k] : o->tol;
        infos[k].b2 = b2[k];
      }
      const double r2 = c->hres[0];
      infos[k].true_rtr = r2;
      infos[k].rtr = r2;
      infos[k].niter = iter;
      infos[k].reliable_updates = restarts;
      if (!(r2 == r2)) return BQCDG_ENAN;
      if (r2 <= stop[k]) {
        infos[k].converged = 1;  // retired: its residual column is overwritten
      } else {
        keep.push_back(k);
      }
    }
    first = false;
    active = keep;
    const int s = (int)active.size();
    if (s == 0 || iter >= o->maxiter || idle > 2) break;
    const int iter_at_restart = iter;
    // Q' C = R (the FP64 residuals), x_s = 0.  The search block goes on from
    // the last one when the block kept its systems: with D = P - Q the part
    // of P beyond the old residual basis, P' = Q' + (1 - Q'Q'^H) D (Q^H Q'),
    // which keeps P'^H Q' = 1 and equals the uninterrupted recurrence when
    // the FP64 residuals equal the iterated ones (the block form of the
    // single solver's p = r + beta (p - <r,p>/|r|^2 r)); else P' = Q'.
    const bool carry = restarts > 0 && s == prev_s && keep_dirs;
    Dense C;
    bool ok;
    if (carry)  // the old residual basis, kept in Z (free until the next product)
      CK(cudaMemcpyAsync(bs.Z.v, bs.Q.v, (size_t)bs.Q.rsb * s, cudaMemcpyDeviceToDevice, c->stream));
    if ((st = qr2(c, bs, s, bs.M, bs.Q, C, ok))) return st;
    if (!ok) return BQCDG_ENAN;  // the FP64 residuals of the remaining systems are dependent
    restarts++;
    prev_s = s;
    if (carry) {
      const Dense I = Dense::eye(s), mI = [&] { Dense m(s); for (int i = 0; i < s; i++) m(i, i) = -1.0; return m; }();
      Dense U, W;
      if ((st = gram(c, bs, s, bs.Z, bs.Q, U))) return st;                   // Q^H Q'
      if ((st = combine(c, bs, s, bs.P, bs.P, I, bs.Z, &mI))) return st;     // D = P - Q
      if ((st = combine(c, bs, s, bs.P, bs.P, U, SpinorPtr{}, nullptr))) return st;  // D U
      if ((st = gram(c, bs, s, bs.Q, bs.P, W))) return st;                   // Q'^H D U
      Dense mW(s);
      for (size_t e = 0; e < W.a.size(); e++) mW.a[e] = -W.a[e];
      if ((st = combine(c, bs, s, bs.P, bs.P, I, bs.Q, &mW))) return st;     // (1 - Q'Q'^H) D U
      if ((st = combine(c, bs, s, bs.P, bs.Q, I, bs.P, &I))) return st;      // + Q'
    } else {
      CK(cudaMemcpyAsync(bs.P.v, bs.Q.v, (size_t)bs.Q.rsb * s, cudaMemcpyDeviceToDevice, c->stream));
    }
    keep_dirs = true;
    CK(cudaMemsetAsync(bs.Xs.v, 0, (size_t)bs.Xs.rsb * s, c->stream));
    double rmax0 = 0.0;
    for (int j = 0; j < s; j++) {
      double cn = 0.0;
      for (int i = 0; i < s; i++) cn += std::norm(C(i, j));
      rmax0 = std::max(rmax0, cn / stop[active[j]]);
    }
    // ---- the block recurrence until the next restart
    while (iter < o->maxiter) {
      // Z = A P over the s columns: the batched passes of the sloppy solver
      launch_mtil_pass1(Prec::F32, g, false, bs.T, bs.P, gauge_of(c, Prec::F32), ainv_of(c, Prec::F32), op,
                        nullptr, c->stream, s);
      launch_mtil_pass2(Prec::F32, g, false, bs.Qe, bs.T, bs.P, gauge_of(c, Prec::F32), aee_of(c, Prec::F32), op,
                        c->red, nullptr, nullptr, c->stream, s);
      launch_mtil_pass1(Prec::F32, g, true, bs.T, bs.Qe, gauge_of(c, Prec::F32), ainv_of(c, Prec::F32), op,
                        nullptr, c->stream, s);
      launch_mtil_pass2(Prec::F32, g, true, bs.Z, bs.T, bs.Qe, gauge_of(c, Prec::F32), aee_of(c, Prec::F32), op,
                        c->red, nullptr, nullptr, c->stream, s);
      CKL();
      Dense G, L;
      if ((st = gram(c, bs, s, bs.P, bs.Z, G))) return st;
      if (!cholesky(G, L)) {  // P^H A P lost definiteness in FP32: restart afresh
        keep_dirs = false;
        break;
      }
      const Dense Li = inv_upper(herm(L));            // (L^H)^-1
      const Dense Psi = mul(Li, herm(Li));             // (L L^H)^-1
      // x_s += P (Psi C); M = Q - Z Psi
      const Dense PsiC = mul(Psi, C);
      const Dense I = Dense::eye(s);
      if ((st = combine(c, bs, s, bs.Xs, bs.Xs, I, bs.P, &PsiC))) return st;
      Dense mPsi(s);
      for (size_t e = 0; e < Psi.a.size(); e++) mPsi.a[e] = -Psi.a[e];
      if ((st = combine(c, bs, s, bs.M, bs.Q, I, bs.Z, &mPsi))) return st;
      Dense Xi;
      if ((st = qr2(c, bs, s, bs.M, bs.Q, Xi, ok))) return st;
      launches += 4 + 6 + 10;
      iter++;
      if (!ok) {  // the new residual block is rank deficient: restart afresh
        keep_dirs = false;
        break;
      }
      // P = Q + P Xi^H; C = Xi C
      const Dense XiH = herm(Xi);
      if ((st = combine(c, bs, s, bs.P, bs.Q, I, bs.P, &XiH))) return st;
      C = mul(Xi, C);
      bool all_below = true;
      double rmax = 0.0;
      for (int j = 0; j < s; j++) {
        double cn = 0.0;
        for (int i = 0; i < s; i++) cn += std::norm(C(i, j));
        infos[active[j]].rtr = cn;
        all_below = all_below && cn <= stop[active[j]];
        rmax = std::max(rmax, cn / stop[active[j]]);
      }
      if (all_below || rmax < delta2 * rmax0 || !(rmax == rmax)) break;
    }
    idle = iter == iter_at_restart ? idle + 1 : 0;
  }
  CK(cudaEventRecord(c->ev1, c->stream));
  CK(cudaEventSynchronize(c->ev1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  bool all = true;
  for (int k = 0; k < nrhs; k++) {
    infos[k].seconds = ms * 1e-3;
    infos[k].kernel_launches = launches;
    if (!infos[k].converged) infos[k].niter = iter;
    all = all && infos[k].converged;
  }
  return all ? BQCDG_OK : BQCDG_ENOCONV;
}
