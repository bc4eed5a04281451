// noalloc.cu -- (W^+W) in = out on caller-owned device fields without any
// device allocation: the two intermediate fields (the odd-site half-step and
// M~ in) live in a file-scope __device__ array of fixed size.
//
// For callers whose device memory is owned by their own framework (a pool or
// arena allocator that every buffer must come from) or that must not allocate
// inside a latency-critical region: cudaMalloc may synchronise the device, and
// a context (bqcdg_create) allocates its own buffers.
#include <cuda_runtime.h>

#include "../../include/bqcdg.h"
#include "kernels.cuh"

using namespace bqcdg;

namespace {

// largest even/odd half volume served: 16384 sites (e.g. 16^3 x 8, 8^3 x 64)
constexpr int kMaxVolh = BQCDG_NOALLOC_MAX_VOLH;
// one spinor field of 12 complex numbers per site, two fields
__device__ __align__(256) double2 g_scratch[2 * 12 * kMaxVolh];

constexpr int kMaxDevices = 64;
void* g_scratch_addr[kMaxDevices] = {};

}  // namespace

extern "C" int bqcdg_mdagm_noalloc(const int L[4], const int bc[4], const double* gauge, const double* a_even,
                                   const double* ainv_odd, const bqcdg_params* p, const double* in, double* out,
                                   void* stream) {
  if (!L || !bc || !gauge || !p || !in || !out) return BQCDG_EINVAL;
  if (p->csw_kappa != 0.0 && (!a_even || !ainv_odd)) return BQCDG_ENOCLOVER;
  Geom g{};
  long long vol = 1;
  for (int d = 0; d < 4; d++) {
    if (L[d] <= 0 || L[d] % 2 || (bc[d] != 1 && bc[d] != -1)) return BQCDG_EINVAL;
    g.L[d] = L[d];
    g.bcsign[d] = bc[d];
    vol *= L[d];
  }
  if (vol / 2 > kMaxVolh) return BQCDG_EINVAL;  // larger than the static scratch
  g.Lxh = L[0] / 2;
  g.volh = (int)(vol / 2);
  g.stride = (g.volh + 63) / 64 * 64;
  g.rec12 = 0;
  geom_finish(g);
  if (g.stride > kMaxVolh) return BQCDG_EINVAL;

  // set-up, once per device and with that device current: the host-side
  // symbol is only a stand-in, the kernels need the device address
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return BQCDG_ENODEVICE;
  if (dev < 0 || dev >= kMaxDevices) return BQCDG_EINVAL;
  if (!g_scratch_addr[dev]) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_scratch);
    if (e != cudaSuccess || !ptr) return BQCDG_ECUDA;
    g_scratch_addr[dev] = ptr;
  }
  double2* scratch = (double2*)g_scratch_addr[dev];
  SpinorPtr t, q, si, so;
  t.v = scratch;                             // odd-site half step
  q.v = scratch + (size_t)12 * g.stride;     // M~ in on the even sites
  si.v = (void*)in;
  so.v = out;
  CloverPtr aee, aio;
  aee.v = (void*)a_even;
  aio.v = (void*)ainv_odd;
  OpParams op;
  op.kappa = p->kappa;
  op.csw_kappa = p->csw_kappa;
  op.h = p->h;
  op.rho = p->rho;
  cudaStream_t s = (cudaStream_t)stream;
  RedScratch none{};
  // every site these passes read is written first, so nothing in the scratch
  // has to start at zero
  launch_mtil_pass1(Prec::F64, g, false, t, si, gauge, aio, op, nullptr, s);
  launch_mtil_pass2(Prec::F64, g, false, q, t, si, gauge, aee, op, none, nullptr, nullptr, s);
  launch_mtil_pass1(Prec::F64, g, true, t, q, gauge, aio, op, nullptr, s);
  launch_mtil_pass2(Prec::F64, g, true, so, t, q, gauge, aee, op, none, nullptr, nullptr, s);
  return cudaGetLastError() == cudaSuccess ? BQCDG_OK : BQCDG_ECUDA;
}
