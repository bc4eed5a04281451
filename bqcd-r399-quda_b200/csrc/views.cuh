// views.cuh -- device pieces shared by the stencil kernel files: typed views
// of the type-erased field pointers (SpinorPtr, gauge void*, CloverPtr) by
// precision, and the CG scalar step that closes an iteration.
#pragma once
#include "kernels.cuh"

namespace bqcdg {

template <Prec P>
__device__ __forceinline__ SpinorView<P> sview(SpinorPtr p, int stride);
template <>
__device__ __forceinline__ SpinorView<Prec::F64> sview<Prec::F64>(SpinorPtr p, int stride) {
  return SpinorView<Prec::F64>{(double2*)p.v, stride};
}
template <>
__device__ __forceinline__ SpinorView<Prec::F32> sview<Prec::F32>(SpinorPtr p, int stride) {
  return SpinorView<Prec::F32>{(float4*)p.v, stride};
}
template <>
__device__ __forceinline__ SpinorView<Prec::F16> sview<Prec::F16>(SpinorPtr p, int stride) {
  return SpinorView<Prec::F16>{(int4*)p.v, p.norm, stride};
}

template <Prec P>
__device__ __forceinline__ GaugeView<P> gview(const void* p, const Geom& g);
template <>
__device__ __forceinline__ GaugeView<Prec::F64> gview<Prec::F64>(const void* p, const Geom& g) {
  return GaugeView<Prec::F64>{(double2*)p, g.stride, g.rec12};
}
template <>
__device__ __forceinline__ GaugeView<Prec::F32> gview<Prec::F32>(const void* p, const Geom& g) {
  return GaugeView<Prec::F32>{(float4*)p, g.stride};
}
template <>
__device__ __forceinline__ GaugeView<Prec::F16> gview<Prec::F16>(const void* p, const Geom& g) {
  return GaugeView<Prec::F16>{(short4*)p, g.stride};
}

template <Prec P>
__device__ __forceinline__ CloverView<P> cview(CloverPtr p, int stride);
template <>
__device__ __forceinline__ CloverView<Prec::F64> cview<Prec::F64>(CloverPtr p, int stride) {
  return CloverView<Prec::F64>{(double2*)p.v, stride};
}
template <>
__device__ __forceinline__ CloverView<Prec::F32> cview<Prec::F32>(CloverPtr p, int stride) {
  return CloverView<Prec::F32>{(float4*)p.v, stride};
}
template <>
__device__ __forceinline__ CloverView<Prec::F16> cview<Prec::F16>(CloverPtr p, int stride) {
  return CloverView<Prec::F16>{(int4*)p.v, p.norm, stride};
}

// the scalar part of one CG iteration once |r|^2 of the new residual is
// known (cg.F90:107-116), with the stop and reliable-update decisions of the
// mixed-precision solver; run by one thread: of k_cg_step in the CG loop, of
// the last block to arrive where a fused pass takes the step itself
__device__ __forceinline__ void cg_scalar_step(CgScalars* cg, double rtr) {
  cg->iter += 1;
  cg->rtr_old = cg->rtr;
  cg->rtr = rtr;
  cg->beta = rtr / cg->rtr_old;
  if (rtr > cg->maxr2) cg->maxr2 = rtr;
  if (!(rtr == rtr)) cg->done = 4;  // NaN: stop, reported as an error
  else if (rtr <= cg->stop_rtr) cg->done = 1;
  else if (cg->iter >= cg->maxiter) cg->done = 3;
  else if (rtr < cg->delta2 * cg->maxr2) cg->done = 2;  // reliable update (|r| < delta max|r|)
  else if (cg->ru_every > 0 && cg->iter - cg->last_ru >= cg->ru_every) cg->done = 2;  // periodic check
}

}  // namespace bqcdg
