// convert.cu -- conversions between BQCD's Fortran field layouts (as staged in
// device memory after one contiguous host-to-device copy) and the
// component-major device layouts, plus the reduced-precision copies used by
// the mixed-precision solver.
#include "kernels.cuh"

namespace bqcdg {

// SPINCOL_FIELD complex(4,3,volh): site-major, 12 complex per site in the
// order spin-fastest, which is the device component index k = colour*4+spin.
__global__ void __launch_bounds__(kBlock) k_spinor_from_fortran(Geom g, double2* dev, const double2* hl) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.volh) return;
#pragma unroll
  for (int k = 0; k < 12; k++) dev[k * g.stride + i] = hl[(size_t)i * 12 + k];
}
__global__ void __launch_bounds__(kBlock) k_spinor_to_fortran(Geom g, double2* hl, const double2* dev) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.volh) return;
#pragma unroll
  for (int k = 0; k < 12; k++) hl[(size_t)i * 12 + k] = dev[k * g.stride + i];
}
void launch_spinor_from_fortran(const Geom& g, double2* dev, const double2* hl, cudaStream_t s) {
  k_spinor_from_fortran<<<nblocks(g.volh), kBlock, 0, s>>>(g, dev, hl);
}
void launch_spinor_to_fortran(const Geom& g, double2* hl, const double2* dev, cudaStream_t s) {
  k_spinor_to_fortran<<<nblocks(g.volh), kBlock, 0, s>>>(g, hl, dev);
}

// GAUGE_FIELD complex(3,3,volh,0:1,4): u(row,col,i,eo,mu), column-major 3x3.
// The device copy is periodic: a flipped input (flip_bc.F90:97-121 applied)
// gets the boundary sign removed on the slice x_mu = L_mu - 1.
__global__ void __launch_bounds__(kBlock) k_gauge_from_fortran(Geom g, double2* dev, const double2* hl, int flipped) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int me = blockIdx.y;  // mu*2 + eo
  if (i >= g.volh) return;
  int mu = me >> 1, eo = me & 1;
  double sgn = 1.0;
  if (flipped && g.bcsign[mu] < 0) {
    Site st = site_coords(g, i, eo);
    if (st.x[mu] == g.L[mu] - 1) sgn = -1.0;
  }
  const double2* src = hl + ((size_t)me * g.volh + i) * 9;
  double2* dst = dev + (size_t)me * 9 * g.stride + i;
#pragma unroll
  for (int k = 0; k < 9; k++) {
    double2 t = src[k];
    dst[k * g.stride] = make_double2(sgn * t.x, sgn * t.y);
  }
}
__global__ void __launch_bounds__(kBlock) k_gauge_to_fortran(Geom g, double2* hl, const double2* dev, int flipped) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int me = blockIdx.y;
  if (i >= g.volh) return;
  int mu = me >> 1, eo = me & 1;
  double sgn = 1.0;
  if (flipped && g.bcsign[mu] < 0) {
    Site st = site_coords(g, i, eo);
    if (st.x[mu] == g.L[mu] - 1) sgn = -1.0;
  }
  double2* dst = hl + ((size_t)me * g.volh + i) * 9;
  const double2* src = dev + (size_t)me * 9 * g.stride + i;
#pragma unroll
  for (int k = 0; k < 9; k++) {
    double2 t = src[k * g.stride];
    dst[k] = make_double2(sgn * t.x, sgn * t.y);
  }
}
void launch_gauge_from_fortran(const Geom& g, double2* dev, const double2* hl, int flipped, cudaStream_t s) {
  k_gauge_from_fortran<<<dim3(nblocks(g.volh), 8), kBlock, 0, s>>>(g, dev, hl, flipped);
}
void launch_gauge_to_fortran(const Geom& g, double2* hl, const double2* dev, int flipped, cudaStream_t s) {
  k_gauge_to_fortran<<<dim3(nblocks(g.volh), 8), kBlock, 0, s>>>(g, hl, dev, flipped);
}

// CLOVER_FIELD_A/B type(...)(2,volh) of one parity: 2 x 18 complex per site
__global__ void __launch_bounds__(kBlock) k_clover_from_fortran(Geom g, double2* dev, const double2* hl) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.volh) return;
#pragma unroll 4
  for (int k = 0; k < 36; k++) dev[k * g.stride + i] = hl[(size_t)i * 36 + k];
}
__global__ void __launch_bounds__(kBlock) k_clover_to_fortran(Geom g, double2* hl, const double2* dev) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.volh) return;
#pragma unroll 4
  for (int k = 0; k < 36; k++) hl[(size_t)i * 36 + k] = dev[k * g.stride + i];
}
void launch_clover_from_fortran(const Geom& g, double2* dev, const double2* hl, cudaStream_t s) {
  k_clover_from_fortran<<<nblocks(g.volh), kBlock, 0, s>>>(g, dev, hl);
}
void launch_clover_to_fortran(const Geom& g, double2* hl, const double2* dev, cudaStream_t s) {
  k_clover_to_fortran<<<nblocks(g.volh), kBlock, 0, s>>>(g, hl, dev);
}

// ---------------------------------------------------------------------------
// reduced-precision copies: links keep columns 1 and 2 (12 reals)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_gauge_demote32(Geom g, float4* out, const double2* in) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int me = blockIdx.y;
  if (i >= g.volh) return;
  const double2* src = in + (size_t)me * 9 * g.stride + i;
  float4* dst = out + (size_t)me * 3 * g.stride + i;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    double2 a = src[(2 * k) * g.stride], b = src[(2 * k + 1) * g.stride];
    dst[k * g.stride] = make_float4((float)a.x, (float)a.y, (float)b.x, (float)b.y);
  }
}
// v in [-1, 1] -> offset-binary int16 q + 32768, q = round(32767 v)
__device__ __forceinline__ short q16(double v) {
  double t = rint(v * 32767.0);
  t = fmin(32767.0, fmax(-32767.0, t));
  return (short)(unsigned short)((int)t + 32768);
}
__global__ void __launch_bounds__(kBlock) k_gauge_demote16(Geom g, short4* out, const double2* in) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int me = blockIdx.y;
  if (i >= g.volh) return;
  const double2* src = in + (size_t)me * 9 * g.stride + i;
  short4* dst = out + (size_t)me * 3 * g.stride + i;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    double2 a = src[(2 * k) * g.stride], b = src[(2 * k + 1) * g.stride];
    dst[k * g.stride] = make_short4(q16(a.x), q16(a.y), q16(b.x), q16(b.y));
  }
}
// FP64 12-real copy: the first six entries (columns 1, 2) of every link
__global__ void __launch_bounds__(kBlock) k_gauge_compress64(Geom g, double2* out, const double2* in) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int me = blockIdx.y;
  if (i >= g.volh) return;
#pragma unroll
  for (int k = 0; k < 6; k++)
    out[((size_t)me * 6 + k) * g.stride + i] = in[((size_t)me * 9 + k) * g.stride + i];
}

void launch_gauge_demote(const Geom& g, Prec p, void* out, const double2* in, cudaStream_t s) {
  dim3 grid(nblocks(g.volh), 8);
  if (p == Prec::F64) k_gauge_compress64<<<grid, kBlock, 0, s>>>(g, (double2*)out, in);
  else if (p == Prec::F32) k_gauge_demote32<<<grid, kBlock, 0, s>>>(g, (float4*)out, in);
  else k_gauge_demote16<<<grid, kBlock, 0, s>>>(g, (short4*)out, in);
}

__global__ void __launch_bounds__(kBlock) k_clover_demote32(Geom g, float4* out, const double2* in) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.volh) return;
#pragma unroll 3
  for (int k = 0; k < 18; k++) {
    double2 a = in[(2 * k) * g.stride + i], b = in[(2 * k + 1) * g.stride + i];
    out[k * g.stride + i] = make_float4((float)a.x, (float)a.y, (float)b.x, (float)b.y);
  }
}
__global__ void __launch_bounds__(kBlock) k_clover_demote16(Geom g, int4* out, float* norm, const double2* in) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.volh) return;
  double m = 0.0;
  for (int k = 0; k < 36; k++) {
    double2 a = in[k * g.stride + i];
    m = fmax(m, fmax(fabs(a.x), fabs(a.y)));
  }
  float mf = (float)m;
  double inv = mf > 0.f ? 1.0 / (double)mf : 0.0;
  norm[i] = mf;
  for (int w = 0; w < 9; w++) {
    short q[8];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      double2 a = in[(4 * w + j) * g.stride + i];
      q[2 * j] = q16(a.x * inv);
      q[2 * j + 1] = q16(a.y * inv);
    }
    out[w * g.stride + i] = *reinterpret_cast<int4*>(q);
  }
}
void launch_clover_demote(const Geom& g, Prec p, CloverPtr out, const double2* in, cudaStream_t s) {
  if (p == Prec::F32) k_clover_demote32<<<nblocks(g.volh), kBlock, 0, s>>>(g, (float4*)out.v, in);
  else k_clover_demote16<<<nblocks(g.volh), kBlock, 0, s>>>(g, (int4*)out.v, out.norm, in);
}

// ---------------------------------------------------------------------------
// SU(3) check of the periodic device links: max_ij |(U U^+ - 1)_ij| and
// max |det U - 1| (the 12-real reconstruction is exact only for SU(3))
// ---------------------------------------------------------------------------
__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

__global__ void __launch_bounds__(kBlock) k_gauge_check(Geom g, const double2* gauge, double* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int me = blockIdx.y;
  double dev_u = 0.0, dev_d = 0.0;
  if (i < g.volh) {
    GaugeView<Prec::F64> U{(double2*)gauge, g.stride};
    Link<double> u;
    U.load(me >> 1, me & 1, i, u);
    for (int r = 0; r < 3; r++)
      for (int c = 0; c < 3; c++) {
        cx<double> t = mkc(0.0, 0.0);
        for (int k = 0; k < 3; k++) t = t + mulc(u.m[r][k], u.m[c][k]);
        if (r == c) t.x -= 1.0;
        dev_u = fmax(dev_u, fabs(t.x) + fabs(t.y));
      }
    cx<double> det = u.m[0][0] * (u.m[1][1] * u.m[2][2] - u.m[1][2] * u.m[2][1]) -
                     u.m[0][1] * (u.m[1][0] * u.m[2][2] - u.m[1][2] * u.m[2][0]) +
                     u.m[0][2] * (u.m[1][0] * u.m[2][1] - u.m[1][1] * u.m[2][0]);
    dev_d = fabs(det.x - 1.0) + fabs(det.y);
    if (!(dev_u == dev_u) || !(dev_d == dev_d)) dev_u = dev_d = 1e300;
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    dev_u = fmax(dev_u, __shfl_down_sync(0xffffffffu, dev_u, off));
    dev_d = fmax(dev_d, __shfl_down_sync(0xffffffffu, dev_d, off));
  }
  if ((threadIdx.x & 31) == 0) {
    atomic_max_nonneg(out, dev_u);
    atomic_max_nonneg(out + 1, dev_d);
  }
}

void launch_gauge_check(const Geom& g, const double2* gauge, RedScratch red, double* out, cudaStream_t s) {
  (void)red;
  cudaMemsetAsync(out, 0, 2 * sizeof(double), s);
  k_gauge_check<<<dim3(nblocks(g.volh), 8), kBlock, 0, s>>>(g, gauge, out);
}

}  // namespace bqcdg
