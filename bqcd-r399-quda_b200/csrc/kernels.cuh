// kernels.cuh -- host-side declarations of the sm_100a kernels (launchers).
#pragma once

#include <cuda_runtime.h>
#include "bqcdg_internal.cuh"

namespace bqcdg {

// type-erased device pointers handed from the runtime to the launchers
struct SpinorPtr {
  void* v = nullptr;
  float* norm = nullptr;  // F16 only
  long long rsb = 0;      // bytes from one RHS's field to the next (batched launches)
  long long rsnb = 0;     // same for the norms
};

// the field of right-hand side r in a batched SpinorPtr
__host__ __device__ __forceinline__ SpinorPtr rhs_of(SpinorPtr p, int r) {
  SpinorPtr q = p;
  if (r) {
    q.v = (char*)p.v + r * p.rsb;
    if (p.norm) q.norm = (float*)((char*)p.norm + r * p.rsnb);
  }
  return q;
}
struct CloverPtr {
  void* v = nullptr;
  float* norm = nullptr;  // F16 only
};

// reduction scratch: per-block partials + arrival counter
struct RedScratch {
  double* partial = nullptr;  // [nval][maxblocks]
  unsigned int* counter = nullptr;
  int maxblocks = 0;
};

// scalars of a CG kept in device memory (no host round trip per iteration)
struct CgScalars {
  double rtr;       // |r|^2 after the latest update
  double rtr_old;   // |r|^2 of the previous iteration
  double paap;      // p.(A p) = |M p|^2
  double alpha;
  double beta;
  double stop_rtr;  // converged when rtr <= stop_rtr
  double ru_rtr;    // unused (kept for layout); see delta2/maxr2
  int iter;         // iterations completed
  int maxiter;
  int done;         // 0 running, 1 converged, 2 reliable update requested, 3 maxiter, 4 NaN
  int pad;
  double delta2;    // sloppy solver: reliable update when rtr < delta2 * maxr2 (0: never)
  double maxr2;     // largest |r|^2 since the last reliable update
  int last_ru;      // iteration of the last reliable update
  int ru_every;     // also update after this many iterations without one (0: never)
};

struct OpParams {
  double kappa;
  double csw_kappa;
  double h;
  double rho;
};

constexpr int kBlock = 128;
inline int nblocks(int n) { return (n + kBlock - 1) / kBlock; }

// ---- stencil and clover operators (dslash.cu) ----
void launch_dslash(Prec p, const Geom& g, int e, bool dag, SpinorPtr out, SpinorPtr in, const void* gauge,
                   cudaStream_t s);
// out = A in (mult_a); in-place allowed (mult_ao)
void launch_clover_mult(Prec p, const Geom& g, SpinorPtr out, SpinorPtr in, CloverPtr a, cudaStream_t s);
// in-place LDL solve with the B factors (F64 only)
void launch_clover_mult_b(const Geom& g, double2* x, const double2* b, cudaStream_t s);

// first half of mtil / mtil_dag: out_o = [(1 -+ i h g5)] Ainv_oo D_oe in_e
// (nr > 1: nr right-hand sides in one launch, fields at SpinorPtr::rsb strides,
//  cg / norm_out arrays of nr entries; retired RHS return at once)
// (g.clover_t: the clover fields hold T and each pass forms A(kappa) and
//  A(kappa)^-1 per site, at op.kappa or at kappa_rhs[k] for right-hand side k;
//  kappa_rhs also sets each right-hand side's hopping coefficient)
// The |M~ p|^2 block partials that a k_pass2 launched with defer_alpha left
// in red.partial (slot 0 of each RHS).  The k_pass1 launch after it, given
// this, sums them in its first site block of each RHS, before its own sites,
// and sets that RHS's paap and alpha = rtr / paap: the same fixed-order sum
// (final_sum) that k_pass2's last block would run, so alpha is bit for bit
// the same, but no k_pass2 block waits for an arrival counter.
struct AlphaFin {
  const double* partial = nullptr;
  int stride = 0;  // RedScratch::maxblocks
  CgScalars* cg = nullptr;
};
void launch_mtil_pass1(Prec p, const Geom& g, bool dag, SpinorPtr out_o, SpinorPtr in_e, const void* gauge,
                       CloverPtr ainv_oo, const OpParams& op, const CgScalars* cg, cudaStream_t s, int nr = 1,
                       const double* kappa_rhs = nullptr, AlphaFin fin = AlphaFin{});
// second half: out_e = A_ee in_e + b D_eo t_o (+ h term for Wilson) + rho in_e;
// optional |out|^2 reduction into *norm_out (device), and CG alpha update
void launch_mtil_pass2(Prec p, const Geom& g, bool dag, SpinorPtr out_e, SpinorPtr t_o, SpinorPtr in_e,
                       const void* gauge, CloverPtr a_ee, const OpParams& op, RedScratch red, double* norm_out,
                       CgScalars* cg, cudaStream_t s, int nr = 1, const double* rho_rhs = nullptr,
                       const double* kappa_rhs = nullptr, bool defer_alpha = false);
// CG-fused second half of mtil_dag: Ap = A_ee q + b D_eo t_o + rho q computed in
// registers; x += alpha p, r -= alpha Ap, rtr = |r|^2.  Precision P for the
// stencil fields, x/r in XP (F64 for the FP64 solver, F32 for the sloppy one)
void launch_cg_pass4(Prec p, const Geom& g, SpinorPtr t_o, SpinorPtr q_e, const void* gauge, CloverPtr a_ee,
                     const OpParams& op, SpinorPtr pvec, SpinorPtr x, SpinorPtr r, RedScratch red, CgScalars* cg,
                     cudaStream_t s, int nr = 1, bool xupd = true, const double* rho_rhs = nullptr,
                     const double* kappa_rhs = nullptr, bool defer_step = false);
// With defer_step, k_cg_pass4 leaves its |r|^2 block partials in red.partial
// and launch_cg_step, queued after it, sums them (one CTA per right-hand
// side, the fixed-order final_sum) and takes the CG scalar step
// (cg_scalar_step: beta, the stop tests), which the last k_cg_pass4 block
// would otherwise take after an arrival counter.  nsb: site blocks per RHS
// of that k_cg_pass4 launch.
void launch_cg_step(RedScratch red, CgScalars* cg, int nr, int nsb, cudaStream_t s);
// (rho_rhs: device array of one shift rho per right-hand side, replacing
//  op.rho, in the second passes; null: op.rho for all)
// register-blocked batched passes (dslash_multi.cu): one thread serves one
// site of nbt (2 or 4) right-hand sides, so each link and clover block is
// loaded and decoded once for all of them.  Sloppy precisions (F32, F16)
// and h = 0 only; pass 2 is the non-dagger one with the CG alpha update, and
// pass 4 updates x (cg required for both).
void launch_mtil_pass1_n(Prec p, const Geom& g, bool dag, SpinorPtr out_o, SpinorPtr in_e, const void* gauge,
                         CloverPtr ainv_oo, const OpParams& op, const CgScalars* cg, cudaStream_t s, int nr,
                         int nbt, AlphaFin fin = AlphaFin{});
void launch_mtil_pass2_n(Prec p, const Geom& g, SpinorPtr out_e, SpinorPtr t_o, SpinorPtr in_e, const void* gauge,
                         CloverPtr a_ee, const OpParams& op, RedScratch red, CgScalars* cg, cudaStream_t s, int nr,
                         const double* rho_rhs, int nbt, bool defer_alpha = false);
void launch_cg_pass4_n(Prec p, const Geom& g, SpinorPtr t_o, SpinorPtr q_e, const void* gauge, CloverPtr a_ee,
                       const OpParams& op, SpinorPtr pvec, SpinorPtr x, SpinorPtr r, RedScratch red, CgScalars* cg,
                       cudaStream_t s, int nr, const double* rho_rhs, int nbt, bool defer_step = false);
// p = r + beta p; with x given (xupd = false above, single RHS), also the
// x += alpha p of iteration `expect` if that iteration ran
void launch_cg_pupdate(Prec p, const Geom& g, SpinorPtr pvec, SpinorPtr r, CgScalars* cg, cudaStream_t s,
                       int nr = 1, SpinorPtr x = SpinorPtr{}, int expect = -1);

// ---- block solver (blockcg.cu) ----
// out[i * s + j] = <a_i, b_j> (FP64) for two blocks of s <= 16 FP32 fields
// (batched layout); partial: block_gram_scratch_pairs() complex doubles
int block_gram_scratch_pairs();
void launch_block_gram(const Geom& g, int s, SpinorPtr a, SpinorPtr b, double2* partial, double2* out,
                       cudaStream_t st);
// out_j = sum_k in1_k m1[k * s + j] (+ sum_k in2_k m2[k * s + j] when in2.v):
// right multiplication of FP32 blocks by s x s complex matrices; out may be
// in1 or in2
void launch_block_combine(const Geom& g, int s, SpinorPtr out, SpinorPtr in1, const float2* m1, SpinorPtr in2,
                          const float2* m2, cudaStream_t st);

// ---- configuration files (confio.cu) ----
// time slice t of the resident FP64 links in the order and byte order of
// BQCD's slice files (24 big-endian complex per site, 384 bytes), and back
// with the third column rebuilt; *acc ^= the raw CRC register of the slice
// (zero it first; cksum's length and complement are applied on the host)
cudaError_t launch_links_to_file(const Geom& g, const double2* gauge, int t, void* out, unsigned* acc,
                                 cudaStream_t s);
cudaError_t launch_links_from_file(const Geom& g, const void* in, int t, double2* gauge, unsigned* acc,
                                   cudaStream_t s);

// ---- BLAS / conversions (blas.cu) ----
// r = b - Ax (F64), copy r into p (precision pp); res2[0] = |r|^2, res2[1] = |b|^2
void launch_residual(const Geom& g, double2* r, const double2* b, const double2* ax, Prec pp, SpinorPtr p,
                     RedScratch red, double* res2, cudaStream_t s);
// reliable-update helpers: *out = <r32, p> (real), then p = r + beta (p - rpc r)
void launch_rdot(const Geom& g, SpinorPtr r32, Prec pp, SpinorPtr p, RedScratch red, double* out, cudaStream_t s);
void launch_p_reorth(const Geom& g, Prec pp, SpinorPtr p, SpinorPtr r32, double rpc, double beta, cudaStream_t s);
// x = (1 + i h gamma_5) x (h_mult_b, h_mult.F90:51-82), F64
void launch_h_mult_b(const Geom& g, double2* x, double h, cudaStream_t s);
// halved inverse blocks from the LDL factors B (6 unit solves per block)
void launch_ainv_from_b(const Geom& g, double2* ainv, const double2* b, cudaStream_t s);
// generic copy/convert between spinor precisions
void launch_spinor_convert(const Geom& g, Prec pout, SpinorPtr out, Prec pin, SpinorPtr in, cudaStream_t s);
// x64 += xs (F32), xs = 0
void launch_accum_x(const Geom& g, double2* x, float4* xs, cudaStream_t s);
// |v|^2 of an F64 spinor -> *out (device)
void launch_norm2(const Geom& g, const double2* v, RedScratch red, double* out, cudaStream_t s);
// dot <a,b> real part of F64 spinors -> *out
void launch_dot(const Geom& g, const double2* a, const double2* b, RedScratch red, double* out, cudaStream_t s);
// y = a*x + y (F64)
void launch_axpy(const Geom& g, double a, const double2* x, double2* y, cudaStream_t s);
void launch_zero(const Geom& g, Prec p, SpinorPtr v, cudaStream_t s);

// ---- layout conversions (convert.cu) ----
// Fortran SPINCOL_FIELD complex(4,3,volh) <-> device F64 spinor
void launch_spinor_from_fortran(const Geom& g, double2* dev, const double2* host_layout, cudaStream_t s);
void launch_spinor_to_fortran(const Geom& g, double2* host_layout, const double2* dev, cudaStream_t s);
// Fortran GAUGE_FIELD complex(3,3,volh,0:1,4) -> device F64 links (periodic);
// flipped != 0: the input carries flip_bc's boundary sign, which is removed
void launch_gauge_from_fortran(const Geom& g, double2* dev, const double2* host_layout, int flipped, cudaStream_t s);
void launch_gauge_to_fortran(const Geom& g, double2* host_layout, const double2* dev, int flipped, cudaStream_t s);
// Fortran CLOVER_FIELD_A/B (18,2,volh) for one parity -> device F64 [36][stride]
void launch_clover_from_fortran(const Geom& g, double2* dev, const double2* host_layout, cudaStream_t s);
void launch_clover_to_fortran(const Geom& g, double2* host_layout, const double2* dev, cudaStream_t s);
// sloppy copies
void launch_gauge_demote(const Geom& g, Prec p, void* out, const double2* in, cudaStream_t s);
void launch_clover_demote(const Geom& g, Prec p, CloverPtr out, const double2* in, cudaStream_t s);
// gauge-field SU(3) check: max |U U^+ - 1| and max |det U - 1| -> out[2]
void launch_gauge_check(const Geom& g, const double2* gauge, RedScratch red, double* out, cudaStream_t s);

// ---- forces (force.cu) ----
// hopping force (dsf.F90:75-100): p(eo,mu) from a,b (even) and at,bt (odd)
void launch_dsf_hop(const Geom& g, double* p, const double2* gauge, const double2* a, const double2* b,
                    const double2* at, const double2* bt, double s, cudaStream_t st);
// w planes of clover_bsa (6 planes x 9 complex per site) -> wbuf [6][9][stride]
void launch_clover_bsa(const Geom& g, double2* w, const double2* b, const double2* a, cudaStream_t st);
// w planes of clover_ts from the halved inverse blocks (clover_t_init + ts)
void launch_clover_ts(const Geom& g, double2* w, const double2* ainv, cudaStream_t st);
// clover_d: p(link) += contributions of the w planes of parity eo_w
void launch_clover_d(const Geom& g, double* p, const double2* gauge, const double2* w, int eo_w, double s,
                     cudaStream_t st);

// ---- clover construction (clover_init.cu) ----
// clover_init.F90 + clover_inv.F90 on device: A, Ainv, B of each parity whose
// pointers are given (null: not computed), in chunks of clover_init_chunk(g)
// sites through tmp (54 complex per chunk site: the six field strengths)
int clover_init_chunk(const Geom& g);
void launch_clover_init(const Geom& g, const double2* gauge, double csw_kappa, double2* a[2], double2* ainv[2],
                        double2* b[2], double2* tmp, cudaStream_t s);
// T = (-c_sw / 8)(p +- q) of each chiral block, packed like A, for the
// parities whose pointer is given: the kappa-independent part of the clover
// term, A(kappa) = 1 + kappa T (clover_init.F90:46-77, clover_init3)
void launch_clover_t(const Geom& g, const double2* gauge, double csw, double2* t[2], double2* tmp, cudaStream_t s);
// 2 sum log det over the halved 1/D of B (clover_action.F90)
void launch_clover_action(const Geom& g, const double2* b, RedScratch red, double* out, cudaStream_t s);

// ---- seeded synthetic inputs (gauge_gen.cu) ----
void ranf_powers(unsigned long long* pw);
unsigned long long ranf_skip(unsigned long long seed, unsigned long long n);
// ran_gauss_volh on the device: out[i*m + j] for draws 2(i m + j)+1, +2 from state s0
void launch_ran_gauss(double2* out, int volh, int m, double var, unsigned long long s0, cudaStream_t s);
void launch_u_normalize(double2* u_fortran, long long nlinks, cudaStream_t s);
void launch_cold(double2* u_fortran, long long nlinks, cudaStream_t s);
void launch_conf_relax(const Geom& g, double2* gauge, cudaStream_t s);
void launch_plaquette(const Geom& g, const double2* gauge, RedScratch red, double* out, cudaStream_t s);

// ---- resident HMC pieces (hmc.cu) ----
// U <- exp(i step p) U on every link, re-unitarised (hmc_u.F90:53-67)
void launch_hmc_u(const Geom& g, double2* gauge, const double* p, double step, cudaStream_t s);
// p += s Im Tr(lambda_j U staples) (dsg.F90:28-53), s = -step beta / 3
void launch_dsg(const Geom& g, const double2* gauge, double* p, double s, cudaStream_t st);
// sum over the momentum field of (a - b)^2, or a^2 when b is null
void launch_mom_sumsq(const Geom& g, const double* a, const double* b, RedScratch red, double* out, cudaStream_t s);
// out[0] + i out[1] = <a, b> of F64 spinors
void launch_cdot(const Geom& g, const double2* a, const double2* b, RedScratch red, double* out, cudaStream_t s);
// up to kMaxDotPairs field pairs (a_j, b_j) whose <a_j, b_j> one launch computes
constexpr int kMaxDotPairs = 8;
struct FieldPairs {
  const double2* a[kMaxDotPairs];
  const double2* b[kMaxDotPairs];
};
void launch_cdot_pairs(const Geom& g, const FieldPairs& fp, int n, RedScratch red, double* out, cudaStream_t s);
// y = ay y + (are + i aim) x
void launch_caxpby(const Geom& g, double are, double aim, const double2* x, double ay, double2* y, cudaStream_t s);

}  // namespace bqcdg
