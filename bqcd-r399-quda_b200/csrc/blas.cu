// blas.cu -- BLAS-1 kernels on device spinor fields (sc.F90, cg.F90:81-89)
// with deterministic two-level reductions.
#include "kernels.cuh"

namespace bqcdg {

template <Prec P>
__device__ __forceinline__ SpinorView<P> bview(SpinorPtr p, int stride);
template <>
__device__ __forceinline__ SpinorView<Prec::F64> bview<Prec::F64>(SpinorPtr p, int stride) {
  return SpinorView<Prec::F64>{(double2*)p.v, stride};
}
template <>
__device__ __forceinline__ SpinorView<Prec::F32> bview<Prec::F32>(SpinorPtr p, int stride) {
  return SpinorView<Prec::F32>{(float4*)p.v, stride};
}
template <>
__device__ __forceinline__ SpinorView<Prec::F16> bview<Prec::F16>(SpinorPtr p, int stride) {
  return SpinorView<Prec::F16>{(int4*)p.v, p.norm, stride};
}

// r = b - Ax; p = r (any precision); res2 = {|r|^2, |b|^2}  (cg.F90:81-91)
template <Prec PP>
__global__ void __launch_bounds__(kBlock) k_residual(Geom g, double2* r, const double2* b, const double2* ax,
                                                     SpinorPtr pp, RedScratch red, double* res2) {
  using RP = typename SpinorView<PP>::R;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[2] = {0.0, 0.0};
  if (i < g.volh) {
    SpinorView<Prec::F64> B{(double2*)b, g.stride}, AX{(double2*)ax, g.stride}, Rv{r, g.stride};
    Spinor<double> bl, al, rl;
    B.load(i, bl);
    AX.load(i, al);
    Spinor<RP> pl;
#pragma unroll
    for (int s = 0; s < 4; s++)
#pragma unroll
      for (int c = 0; c < 3; c++) {
        rl.c[s][c] = bl.c[s][c] - al.c[s][c];
        acc[0] += norm2(rl.c[s][c]);
        acc[1] += norm2(bl.c[s][c]);
        pl.c[s][c] = mkc((RP)rl.c[s][c].x, (RP)rl.c[s][c].y);
      }
    Rv.store(i, rl);
    if (pp.v) bview<PP>(pp, g.stride).store(i, pl);
  }
  block_reduce_store<2>(acc, red.partial, red.maxblocks, blockIdx.x);
  if (last_block(red.counter, gridDim.x)) {
    double tot[2];
    final_sum<2>(red.partial, red.maxblocks, gridDim.x, tot);
    if (threadIdx.x == 0) {
      res2[0] = tot[0];
      res2[1] = tot[1];
      *red.counter = 0;
    }
  }
}

void launch_residual(const Geom& g, double2* r, const double2* b, const double2* ax, Prec pp, SpinorPtr p,
                     RedScratch red, double* res2, cudaStream_t s) {
  dim3 grid(nblocks(g.volh));
  if (pp == Prec::F64) k_residual<Prec::F64><<<grid, kBlock, 0, s>>>(g, r, b, ax, p, red, res2);
  else if (pp == Prec::F32) k_residual<Prec::F32><<<grid, kBlock, 0, s>>>(g, r, b, ax, p, red, res2);
  else k_residual<Prec::F16><<<grid, kBlock, 0, s>>>(g, r, b, ax, p, red, res2);
}

__global__ void __launch_bounds__(kBlock) k_h_mult_b(Geom g, double2* x, double h) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.volh) return;
  SpinorView<Prec::F64> X{x, g.stride};
  Spinor<double> s;
  X.load(i, s);
  h_mult_b(s, h);
  X.store(i, s);
}

void launch_h_mult_b(const Geom& g, double2* x, double h, cudaStream_t s) {
  k_h_mult_b<<<nblocks(g.volh), kBlock, 0, s>>>(g, x, h);
}

// real dot <r, p> of an F32 residual and a sloppy search direction
template <Prec PP>
__global__ void __launch_bounds__(kBlock) k_rdot(Geom g, SpinorPtr rp, SpinorPtr pp, RedScratch red, double* out) {
  using RP = typename SpinorView<PP>::R;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[1] = {0.0};
  if (i < g.volh) {
    Spinor<float> r;
    Spinor<RP> p;
    bview<Prec::F32>(rp, g.stride).load(i, r);
    bview<PP>(pp, g.stride).load(i, p);
#pragma unroll
    for (int s = 0; s < 4; s++)
#pragma unroll
      for (int c = 0; c < 3; c++)
        acc[0] += (double)r.c[s][c].x * (double)p.c[s][c].x + (double)r.c[s][c].y * (double)p.c[s][c].y;
  }
  block_reduce_store<1>(acc, red.partial, red.maxblocks, blockIdx.x);
  if (last_block(red.counter, gridDim.x)) {
    double tot[1];
    final_sum<1>(red.partial, red.maxblocks, gridDim.x, tot);
    if (threadIdx.x == 0) {
      *out = tot[0];
      *red.counter = 0;
    }
  }
}

// p = r + beta (p - rp r): the direction re-orthogonalised against the new
// residual after a reliable update, then the CG step
template <Prec PP>
__global__ void __launch_bounds__(kBlock) k_p_reorth(Geom g, SpinorPtr pp, SpinorPtr rp, double rpc, double beta) {
  using RP = typename SpinorView<PP>::R;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.volh) return;
  Spinor<float> r;
  Spinor<RP> p;
  bview<Prec::F32>(rp, g.stride).load(i, r);
  bview<PP>(pp, g.stride).load(i, p);
  const RP a = (RP)(1.0 - beta * rpc), b = (RP)beta;
#pragma unroll
  for (int s = 0; s < 4; s++)
#pragma unroll
    for (int c = 0; c < 3; c++) p.c[s][c] = a * mkc((RP)r.c[s][c].x, (RP)r.c[s][c].y) + b * p.c[s][c];
  bview<PP>(pp, g.stride).store(i, p);
}

void launch_rdot(const Geom& g, SpinorPtr r32, Prec pp, SpinorPtr p, RedScratch red, double* out, cudaStream_t s) {
  dim3 grid(nblocks(g.volh));
  if (pp == Prec::F64) k_rdot<Prec::F64><<<grid, kBlock, 0, s>>>(g, r32, p, red, out);
  else if (pp == Prec::F32) k_rdot<Prec::F32><<<grid, kBlock, 0, s>>>(g, r32, p, red, out);
  else k_rdot<Prec::F16><<<grid, kBlock, 0, s>>>(g, r32, p, red, out);
}

void launch_p_reorth(const Geom& g, Prec pp, SpinorPtr p, SpinorPtr r32, double rpc, double beta, cudaStream_t s) {
  dim3 grid(nblocks(g.volh));
  if (pp == Prec::F64) k_p_reorth<Prec::F64><<<grid, kBlock, 0, s>>>(g, p, r32, rpc, beta);
  else if (pp == Prec::F32) k_p_reorth<Prec::F32><<<grid, kBlock, 0, s>>>(g, p, r32, rpc, beta);
  else k_p_reorth<Prec::F16><<<grid, kBlock, 0, s>>>(g, p, r32, rpc, beta);
}

// halved A^-1 blocks (packed like conf%i) from the B factors, whose 1/D are
// already halved: the unit solves of clover_inv2 (clover_inv.F90:142-220)
__global__ void __launch_bounds__(kBlock) k_ainv_from_b(Geom g, double2* ainv, const double2* b) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.volh) return;
  const int slot_up[6][6] = {{-1, 1, 2, 3, 4, 5},    {-1, -1, 6, 7, 8, 9},    {-1, -1, -1, 11, 12, 13},
                             {-1, -1, -1, -1, 14, 15}, {-1, -1, -1, -1, -1, 17}, {-1, -1, -1, -1, -1, -1}};
  for (int chi = 0; chi < 2; chi++) {
    cx<double> L[15];
    double dinv[6];
    for (int k = 0; k < 15; k++) {
      double2 t = b[(chi * 18 + k) * g.stride + i];
      L[k] = mkc(t.x, t.y);
    }
    for (int k = 0; k < 3; k++) {
      double2 t = b[(chi * 18 + 15 + k) * g.stride + i];
      dinv[2 * k] = t.x;
      dinv[2 * k + 1] = t.y;
    }
    double2* dst = ainv + chi * 18 * g.stride + i;
    double diag[6];
    for (int col = 0; col < 6; col++) {
      cx<double> y[6], x[6];
      for (int k = 0; k < 6; k++) y[k] = mkc(k == col ? 1.0 : 0.0, 0.0);
      for (int r = 1; r < 6; r++) {
        cx<double> sacc = y[r];
        for (int c = 0; c < r; c++) sacc = sacc - L[r * (r - 1) / 2 + c] * y[c];
        y[r] = sacc;
      }
      for (int r = 5; r >= 0; r--) {
        cx<double> sacc = dinv[r] * y[r];
        for (int c = r + 1; c < 6; c++) sacc = sacc - conjg(L[c * (c - 1) / 2 + r]) * x[c];
        x[r] = sacc;
      }
      diag[col] = x[col].x;
      for (int k = col + 1; k < 6; k++) dst[slot_up[col][k] * g.stride] = make_double2(x[k].x, -x[k].y);
    }
    dst[0] = make_double2(diag[0], diag[1]);
    dst[10 * g.stride] = make_double2(diag[2], diag[3]);
    dst[16 * g.stride] = make_double2(diag[4], diag[5]);
  }
}

void launch_ainv_from_b(const Geom& g, double2* ainv, const double2* b, cudaStream_t s) {
  k_ainv_from_b<<<nblocks(g.volh), kBlock, 0, s>>>(g, ainv, b);
}

template <Prec PO, Prec PI>
__global__ void __launch_bounds__(kBlock) k_convert(Geom g, SpinorPtr out, SpinorPtr in) {
  using RO = typename SpinorView<PO>::R;
  using RI = typename SpinorView<PI>::R;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.volh) return;
  Spinor<RI> a;
  bview<PI>(in, g.stride).load(i, a);
  Spinor<RO> b;
#pragma unroll
  for (int s = 0; s < 4; s++)
#pragma unroll
    for (int c = 0; c < 3; c++) b.c[s][c] = mkc((RO)a.c[s][c].x, (RO)a.c[s][c].y);
  bview<PO>(out, g.stride).store(i, b);
}

void launch_spinor_convert(const Geom& g, Prec pout, SpinorPtr out, Prec pin, SpinorPtr in, cudaStream_t s) {
  dim3 grid(nblocks(g.volh));
#define CV(A, B) k_convert<A, B><<<grid, kBlock, 0, s>>>(g, out, in)
  if (pout == Prec::F64) {
    if (pin == Prec::F64) CV(Prec::F64, Prec::F64);
    else if (pin == Prec::F32) CV(Prec::F64, Prec::F32);
    else CV(Prec::F64, Prec::F16);
  } else if (pout == Prec::F32) {
    if (pin == Prec::F64) CV(Prec::F32, Prec::F64);
    else if (pin == Prec::F32) CV(Prec::F32, Prec::F32);
    else CV(Prec::F32, Prec::F16);
  } else {
    if (pin == Prec::F64) CV(Prec::F16, Prec::F64);
    else if (pin == Prec::F32) CV(Prec::F16, Prec::F32);
    else CV(Prec::F16, Prec::F16);
  }
#undef CV
}

// x += xs (F32 -> F64), xs = 0
__global__ void __launch_bounds__(kBlock) k_accum_x(Geom g, double2* x, float4* xs) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.volh) return;
#pragma unroll
  for (int k = 0; k < 6; k++) {
    float4 t = xs[k * g.stride + i];
    double2 a = x[(2 * k) * g.stride + i], b = x[(2 * k + 1) * g.stride + i];
    a.x += t.x; a.y += t.y; b.x += t.z; b.y += t.w;
    x[(2 * k) * g.stride + i] = a;
    x[(2 * k + 1) * g.stride + i] = b;
    xs[k * g.stride + i] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

void launch_accum_x(const Geom& g, double2* x, float4* xs, cudaStream_t s) {
  k_accum_x<<<nblocks(g.volh), kBlock, 0, s>>>(g, x, xs);
}

__global__ void __launch_bounds__(kBlock) k_dot(Geom g, const double2* a, const double2* b, RedScratch red,
                                                double* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[1] = {0.0};
  if (i < g.volh) {
#pragma unroll
    for (int k = 0; k < 12; k++) {
      double2 x = a[k * g.stride + i], y = b[k * g.stride + i];
      acc[0] += x.x * y.x + x.y * y.y;
    }
  }
  block_reduce_store<1>(acc, red.partial, red.maxblocks, blockIdx.x);
  if (last_block(red.counter, gridDim.x)) {
    double tot[1];
    final_sum<1>(red.partial, red.maxblocks, gridDim.x, tot);
    if (threadIdx.x == 0) {
      *out = tot[0];
      *red.counter = 0;
    }
  }
}

void launch_norm2(const Geom& g, const double2* v, RedScratch red, double* out, cudaStream_t s) {
  k_dot<<<nblocks(g.volh), kBlock, 0, s>>>(g, v, v, red, out);
}
void launch_dot(const Geom& g, const double2* a, const double2* b, RedScratch red, double* out, cudaStream_t s) {
  k_dot<<<nblocks(g.volh), kBlock, 0, s>>>(g, a, b, red, out);
}

__global__ void __launch_bounds__(kBlock) k_axpy(Geom g, double a, const double2* x, double2* y) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.volh) return;
#pragma unroll
  for (int k = 0; k < 12; k++) {
    double2 xv = x[k * g.stride + i], yv = y[k * g.stride + i];
    yv.x += a * xv.x;
    yv.y += a * xv.y;
    y[k * g.stride + i] = yv;
  }
}

void launch_axpy(const Geom& g, double a, const double2* x, double2* y, cudaStream_t s) {
  k_axpy<<<nblocks(g.volh), kBlock, 0, s>>>(g, a, x, y);
}

template <Prec P>
__global__ void __launch_bounds__(kBlock) k_zero(Geom g, SpinorPtr v) {
  using R = typename SpinorView<P>::R;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.volh) return;
  Spinor<R> z;
  zero(z);
  bview<P>(v, g.stride).store(i, z);
}

void launch_zero(const Geom& g, Prec p, SpinorPtr v, cudaStream_t s) {
  dim3 grid(nblocks(g.volh));
  if (p == Prec::F64) k_zero<Prec::F64><<<grid, kBlock, 0, s>>>(g, v);
  else if (p == Prec::F32) k_zero<Prec::F32><<<grid, kBlock, 0, s>>>(g, v);
  else k_zero<Prec::F16><<<grid, kBlock, 0, s>>>(g, v);
}

}  // namespace bqcdg
