// ctx.cuh -- the context behind the C ABI (include/bqcdg.h) and the host
// helpers its parts share: capi.cu (context, fields, operators, solvers),
// capi_hmc.cu (resident HMC pieces) and capi_conf.cu (configuration files).
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <map>
#include <string>
#include <unistd.h>
#include <vector>

#include "../../include/bqcdg.h"
#include "kernels.cuh"

using namespace bqcdg;

inline int status_from_cuda(cudaError_t e) {
  if (e == cudaSuccess) return BQCDG_OK;
  if (e == cudaErrorMemoryAllocation) return BQCDG_ENOMEM;
  return BQCDG_ECUDA;
}

struct bqcdg_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  Geom g{};
  long long bytes = 0;
  std::vector<void*> allocations;
  std::vector<size_t> alloc_sizes;  // bytes of allocations[k]

  double2* staging = nullptr;  // Fortran-layout staging, grown on demand (stage)
  size_t staging_bytes = 0;

  double2* gauge64 = nullptr;
  bool have_gauge = false;
  bool gauge_su3 = false;
  void* gauge_s[3] = {nullptr, nullptr, nullptr};  // by Prec
  bool gauge_s_ok[3] = {false, false, false};
  // FP64 links of the even-odd operator stored as 12 reals (SU(3) links only)
  double2* gauge64r = nullptr;
  bool gauge64r_ok = false;
  Geom g12{};  // g with rec12 set

  double2* A[2] = {nullptr, nullptr};
  double2* Ainv[2] = {nullptr, nullptr};
  double2* B[2] = {nullptr, nullptr};
  bool have_A[2] = {false, false}, have_Ainv[2] = {false, false}, have_B[2] = {false, false};
  CloverPtr aee_s[3], ainv_oo_s[3];
  bool clover_s_ok[3] = {false, false, false};

  std::vector<double2*> s64;
  std::vector<SpinorPtr> s32, s16;

  RedScratch red{};
  double* dres = nullptr;        // device result scalars [16]
  double* hres = nullptr;        // pinned mirror
  double* drho = nullptr;        // per right-hand-side shifts of a batch [kMaxRhs]
  double* dkappa = nullptr;      // per right-hand-side hopping parameters of a batch [kMaxRhs]
  CgScalars* dcg = nullptr;
  CgScalars* hcg = nullptr;      // pinned

  double* pgen = nullptr;        // device momenta (GENERATOR_FIELD layout)
  double* mom = nullptr;         // resident momenta of the device HMC pieces
  double* mom_old = nullptr;     // their snapshot for the force monitor
  double2* gauge_bck = nullptr;  // saved links (restored on a rejected trajectory)
  double2* wbuf = nullptr;       // 6 planes x 9 complex per site
  double2* clov_tmp = nullptr;   // field strengths of one chunk of clover_init

  std::map<int, double2*> fields;
  int next_handle = 1;

  unsigned long long seed = 48131768981101ull;  // ranf.F90:36 default seed

  // batched sloppy vectors: nb right-hand sides per buffer, rsb bytes apart
  struct Batch {
    int cap = 0;
    Prec prec = Prec::F64;
    SpinorPtr p, t, q, rs, xs;
  } batch;
  // FP32 blocks of the block CG (capi_block.cu): search, residual basis,
  // A times search, scratch, solution increments, and the two intermediate
  // fields of the operator, cap fields each; Gram sums and s x s matrices
  struct BlockCg {
    int cap = 0;
    SpinorPtr P, Q, Z, M, Xs, T, Qe;
    double2* partial = nullptr;
    double2* gram = nullptr;
    float2* mats = nullptr;
  } blk;
  int tuned_block[3] = {0, 0, 0};  // chosen RHS per launch, by precision
  int tuned_nbt[3][17] = {};       // chosen RHS per stencil thread, by precision and RHS per launch

  void release(void* p) {
    if (!p) return;
    for (size_t k = 0; k < allocations.size(); k++)
      if (allocations[k] == p) {
        bytes -= (long long)alloc_sizes[k];
        allocations.erase(allocations.begin() + k);
        alloc_sizes.erase(alloc_sizes.begin() + k);
        break;
      }
    cudaFree(p);
  }

  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<cudaEvent_t> kev;  // kernel-timing event pairs

  size_t spin_bytes(Prec p) const {
    size_t st = (size_t)g.stride;
    if (p == Prec::F64) return 12 * 16 * st;
    if (p == Prec::F32) return 6 * 16 * st;
    return 3 * 16 * st;
  }

  cudaError_t alloc(void** p, size_t n) {
    cudaError_t e = cudaMalloc(p, n);
    if (e == cudaSuccess) {
      allocations.push_back(*p);
      alloc_sizes.push_back(n);
      bytes += (long long)n;
    }
    return e;
  }
  // the staging buffer holds at least n bytes afterwards (a spinor needs
  // 192 B per even site, a clover parity 576 B, the links 1152 B)
  cudaError_t stage(size_t n) {
    if (staging_bytes >= n) return cudaSuccess;
    release(staging);
    staging = nullptr;
    staging_bytes = 0;
    cudaError_t e = alloc((void**)&staging, n);
    if (e == cudaSuccess) staging_bytes = n;
    return e;
  }
  double2* sp64(size_t k) {
    while (s64.size() <= k) {
      void* p = nullptr;
      if (alloc(&p, spin_bytes(Prec::F64)) != cudaSuccess) return nullptr;
      cudaMemsetAsync(p, 0, spin_bytes(Prec::F64), stream);
      s64.push_back((double2*)p);
    }
    return s64[k];
  }
  SpinorPtr sp(Prec p, size_t k) {
    if (p == Prec::F64) {
      SpinorPtr r;
      r.v = sp64(k);
      return r;
    }
    auto& pool = p == Prec::F32 ? s32 : s16;
    while (pool.size() <= k) {
      SpinorPtr r;
      if (alloc(&r.v, spin_bytes(p)) != cudaSuccess) return SpinorPtr{};
      cudaMemsetAsync(r.v, 0, spin_bytes(p), stream);
      if (p == Prec::F16) {
        if (alloc((void**)&r.norm, sizeof(float) * g.stride) != cudaSuccess) return SpinorPtr{};
        cudaMemsetAsync(r.norm, 0, sizeof(float) * g.stride, stream);
      }
      pool.push_back(r);
    }
    return pool[k];
  }
};

namespace bqcdg_host {


inline SpinorPtr S(double2* p) {
  SpinorPtr r;
  r.v = p;
  return r;
}
inline CloverPtr C(double2* p) {
  CloverPtr r;
  r.v = p;
  return r;
}

#define CK(x)                                      \
  do {                                             \
    cudaError_t e_ = (x);                          \
    if (e_ != cudaSuccess) return status_from_cuda(e_); \
  } while (0)
#define CKL() CK(cudaGetLastError())

// ---- shared helpers (capi.cu) ----
int upload_spinor(bqcdg_ctx* c, const double* host, double2* dev);
int download_spinor(bqcdg_ctx* c, const double2* dev, double* host);
OpParams op_of(const bqcdg_params* p, bool with_rho);
int ensure_sloppy(bqcdg_ctx* c, Prec p, bool need_clover);
int ensure_f64rec(bqcdg_ctx* c);
bool use_rec(bqcdg_ctx* c, Prec p);
const Geom& geom_of(bqcdg_ctx* c, Prec p);
const void* gauge_of(bqcdg_ctx* c, Prec p);
CloverPtr aee_of(bqcdg_ctx* c, Prec p);
CloverPtr ainv_of(bqcdg_ctx* c, Prec p);
int check_op(bqcdg_ctx* c, const bqcdg_params* p);
void apply_mtil(bqcdg_ctx* c, Prec p, bool dag, SpinorPtr out, SpinorPtr in, SpinorPtr t, const OpParams& op,
                double* norm_out, CgScalars* cg);
void apply_mdagm(bqcdg_ctx* c, Prec p, SpinorPtr out, SpinorPtr in, SpinorPtr t, SpinorPtr q, const OpParams& op);
int cg_core(bqcdg_ctx* c, double2* x, double2* b, const OpParams& op, Prec sloppy, int maxiter, double stop_rtr,
            double delta, bool min_one_iter, bool time_kernels, bqcdg_solve_info* info);
// a resident field by handle (nullptr: no such handle)
double2* field(bqcdg_ctx* c, int h);
// the force work buffers (generator field, six sigma_mu_nu planes)
int ensure_force_bufs(bqcdg_ctx* c);
// the hopping and clover parts of dsf (dsf.F90) and the det-term force of
// parity eo (clover_d.F90:40-75) into device momenta
int dsf_core(bqcdg_ctx* c, double* p, double step, const bqcdg_params* par, double2* da, double2* db);
int dsd_core(bqcdg_ctx* c, double* p, int eo, double s);

}  // namespace bqcdg_host
