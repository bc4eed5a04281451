// bqcdg_internal.cuh -- device data layouts and the shared Wilson-clover
// arithmetic of the B200 (sm_100a) implementation of BQCD's fermion hot path.
//
// Host-facing arrays use BQCD's Fortran layouts (defs.h:64-78); on the device
// every field is component-major ("structure of arrays") so that one warp
// reading one component of 32 consecutive sites issues one contiguous 512-byte
// (FP64) transaction:
//
//   spinor  F64 : double2 [12][stride]      component k = colour*4 + spin
//           F32 : float4  [6][stride]       two components per float4
//           F16 : int4    [3][stride]       eight int16 components per int4,
//                 + float norm[stride]      value = q * norm / 32767
//   link    F64 : double2 [9][stride]       18-real, k = col*3 + row
//           F32 : float4  [3][stride]       12-real: columns 1,2 (third column
//           F16 : short4  [3][stride]       rebuilt as in su3.F90:300-310)
//   clover  F64 : double2 [36][stride]      per parity: chiral block chi*18 +
//           F32 : float4  [18][stride]      the 18-slot packing of clover.h:28-82
//           F16 : int4    [9][stride] + float norm[stride]
//
// Device links are always stored periodic (unflipped); the fermion boundary
// sign of flip_bc.F90:97-121 is applied inside the stencil kernels, so the
// operators act exactly like BQCD's on links bracketed by flip_bc().
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace bqcdg {

enum class Prec : int { F64 = 0, F32 = 1, F16 = 2 };

// ---------------------------------------------------------------------------
// complex arithmetic
// ---------------------------------------------------------------------------
template <typename R>
struct cx {
  R x, y;
};
template <typename R>
__device__ __forceinline__ cx<R> mkc(R a, R b) { return cx<R>{a, b}; }
template <typename R>
__device__ __forceinline__ cx<R> operator+(cx<R> a, cx<R> b) { return {a.x + b.x, a.y + b.y}; }
template <typename R>
__device__ __forceinline__ cx<R> operator-(cx<R> a, cx<R> b) { return {a.x - b.x, a.y - b.y}; }
template <typename R>
__device__ __forceinline__ cx<R> operator-(cx<R> a) { return {-a.x, -a.y}; }
template <typename R>
__device__ __forceinline__ cx<R> operator*(cx<R> a, cx<R> b) {
  return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename R>
__device__ __forceinline__ cx<R> operator*(R s, cx<R> a) { return {s * a.x, s * a.y}; }
template <typename R>
__device__ __forceinline__ cx<R> conjg(cx<R> a) { return {a.x, -a.y}; }
// i * a
template <typename R>
__device__ __forceinline__ cx<R> itimes(cx<R> a) { return {-a.y, a.x}; }
// a * conj(b)
template <typename R>
__device__ __forceinline__ cx<R> mulc(cx<R> a, cx<R> b) {
  return {a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
}
// acc + a*b
template <typename R>
__device__ __forceinline__ cx<R> fma_c(cx<R> acc, cx<R> a, cx<R> b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
  return acc;
}
// acc + conj(a)*b
template <typename R>
__device__ __forceinline__ cx<R> fma_cc(cx<R> acc, cx<R> a, cx<R> b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(-a.y, b.x, acc.y);
  return acc;
}
template <typename R>
__device__ __forceinline__ R norm2(cx<R> a) { return a.x * a.x + a.y * a.y; }

template <typename R>
struct Spinor {
  cx<R> c[4][3];  // [spin][colour]
};
template <typename R>
struct Half {
  cx<R> c[2][3];
};
template <typename R>
struct Link {
  cx<R> m[3][3];  // [row][col]
};

template <typename R>
__device__ __forceinline__ void zero(Spinor<R>& s) {
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) s.c[a][b] = mkc<R>(0, 0);
}

// ---------------------------------------------------------------------------
// geometry: even/odd index i = ilex/2 (index.F90:58-76), parity (x+y+z+t)%2
// ---------------------------------------------------------------------------
// n / d for 0 <= n < 2^31 as (umulhi(n, m) + n) >> l, with l = ceil(log2 d)
// and m = floor(2^32 (2^l - d) / d) + 1 (the round-up method of Granlund and
// Montgomery, "Division by invariant integers using multiplication", 1994)
struct FastDiv {
  unsigned d, m;
  int l;
};
inline FastDiv make_fastdiv(unsigned d) {
  int l = 0;
  while ((1ull << l) < d) l++;
  const unsigned long long m = ((1ull << 32) * ((1ull << l) - d)) / d + 1;
  return FastDiv{d, (unsigned)m, l};
}
__host__ __device__ __forceinline__ unsigned fdiv(unsigned n, const FastDiv& f) {
#ifdef __CUDA_ARCH__
  return (__umulhi(n, f.m) + n) >> f.l;
#else
  return ((unsigned)(((unsigned long long)n * f.m) >> 32) + n) >> f.l;
#endif
}

struct Geom {
  int L[4];
  int Lxh;
  int volh;
  int stride;      // padded per-component stride of every field
  int bcsign[4];   // fermion boundary sign per direction (+1 / -1)
  int rec12;       // FP64 stencil links stored as 12 reals (columns 1,2)
  FastDiv dxh, d1, d2;  // division by Lxh, L[1], L[2] (geom_finish)
  int clover_t;    // the clover fields hold T, with A(kappa) = 1 + kappa T (clover_apply_kt)
};
// fills the derived members once L and Lxh are set
inline void geom_finish(Geom& g) {
  g.dxh = make_fastdiv((unsigned)g.Lxh);
  g.d1 = make_fastdiv((unsigned)g.L[1]);
  g.d2 = make_fastdiv((unsigned)g.L[2]);
}

struct Site {
  int x[4];
  int base;  // i - x/2 : index offset of the (y,z,t) row
};

__host__ __device__ __forceinline__ Site site_coords(const Geom& g, int i, int parity) {
  Site s;
  const int r = (int)fdiv((unsigned)i, g.dxh);
  const int xh = i - r * g.Lxh;
  const int r2 = (int)fdiv((unsigned)r, g.d1);
  s.x[1] = r - r2 * g.L[1];
  s.x[3] = (int)fdiv((unsigned)r2, g.d2);
  s.x[2] = r2 - s.x[3] * g.L[2];
  s.x[0] = 2 * xh + ((s.x[1] + s.x[2] + s.x[3] + parity) & 1);
  s.base = i - xh;
  return s;
}

// index of the neighbour of site s in direction mu (fwd: +1, bwd: -1)
__host__ __device__ __forceinline__ int neighbour(const Geom& g, const Site& s, int i, int mu, bool fwd) {
  if (mu == 0) {
    int x = s.x[0] + (fwd ? 1 : -1);
    if (x < 0) x += g.L[0];
    if (x >= g.L[0]) x -= g.L[0];
    return s.base + (x >> 1);
  }
  int step = g.Lxh;
  if (mu >= 2) step *= g.L[1];
  if (mu == 3) step *= g.L[2];
  if (fwd) return s.x[mu] == g.L[mu] - 1 ? i - (g.L[mu] - 1) * step : i + step;
  return s.x[mu] == 0 ? i + (g.L[mu] - 1) * step : i - step;
}

// boundary sign of the link used by a hop: the forward hop uses U_mu(x), the
// backward hop U_mu(x-mu); flip_bc negates links on the slice x_mu = L_mu-1.
__host__ __device__ __forceinline__ int hop_sign(const Geom& g, const Site& s, int mu, bool fwd) {
  if (g.bcsign[mu] > 0) return 1;
  return (fwd ? s.x[mu] == g.L[mu] - 1 : s.x[mu] == 0) ? g.bcsign[mu] : 1;
}

// ---------------------------------------------------------------------------
// field views
// ---------------------------------------------------------------------------
template <Prec P>
struct SpinorView;

template <>
struct SpinorView<Prec::F64> {
  using R = double;
  double2* v;
  int stride;
  __device__ __forceinline__ void load(int i, Spinor<double>& s) const {
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int sp = 0; sp < 4; sp++) {
        double2 t = __ldg(v + (c * 4 + sp) * stride + i);
        s.c[sp][c] = mkc(t.x, t.y);
      }
  }
  // spins (s0, s0+1) only
  __device__ __forceinline__ void load_pair(int i, int s0, cx<double> h[2][3]) const {
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int k = 0; k < 2; k++) {
        double2 t = __ldg(v + (c * 4 + s0 + k) * stride + i);
        h[k][c] = mkc(t.x, t.y);
      }
  }
  __device__ __forceinline__ void store(int i, const Spinor<double>& s) const {
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int sp = 0; sp < 4; sp++) v[(c * 4 + sp) * stride + i] = make_double2(s.c[sp][c].x, s.c[sp][c].y);
  }
  // values up to a common factor (1 here); the int16 view defers its scale
  __device__ __forceinline__ void load_raw(int i, Spinor<double>& s, double& sc) const {
    load(i, s);
    sc = 1.0;
  }
  __device__ __forceinline__ void load_pair_raw(int i, int s0, cx<double> h[2][3], double& sc) const {
    load_pair(i, s0, h);
    sc = 1.0;
  }
  __device__ __forceinline__ void store_scaled(int i, Spinor<double> s, double extra) const {
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) s.c[a][b] = extra * s.c[a][b];
    store(i, s);
  }
};

template <>
struct SpinorView<Prec::F32> {
  using R = float;
  float4* v;
  int stride;
  __device__ __forceinline__ void load(int i, Spinor<float>& s) const {
#pragma unroll
    for (int k = 0; k < 6; k++) {
      float4 t = __ldg(v + k * stride + i);
      int k0 = 2 * k, k1 = 2 * k + 1;
      s.c[k0 & 3][k0 >> 2] = mkc(t.x, t.y);
      s.c[k1 & 3][k1 >> 2] = mkc(t.z, t.w);
    }
  }
  __device__ __forceinline__ void load_pair(int i, int s0, cx<float> h[2][3]) const {
    // components (c*4+s0, c*4+s0+1) sit in float4 number c*2 + s0/2
#pragma unroll
    for (int c = 0; c < 3; c++) {
      float4 t = __ldg(v + (c * 2 + (s0 >> 1)) * stride + i);
      h[0][c] = mkc(t.x, t.y);
      h[1][c] = mkc(t.z, t.w);
    }
  }
  __device__ __forceinline__ void store(int i, const Spinor<float>& s) const {
#pragma unroll
    for (int k = 0; k < 6; k++) {
      int k0 = 2 * k, k1 = 2 * k + 1;
      v[k * stride + i] = make_float4(s.c[k0 & 3][k0 >> 2].x, s.c[k0 & 3][k0 >> 2].y, s.c[k1 & 3][k1 >> 2].x,
                                      s.c[k1 & 3][k1 >> 2].y);
    }
  }
  __device__ __forceinline__ void load_raw(int i, Spinor<float>& s, float& sc) const {
    load(i, s);
    sc = 1.0f;
  }
  __device__ __forceinline__ void load_pair_raw(int i, int s0, cx<float> h[2][3], float& sc) const {
    load_pair(i, s0, h);
    sc = 1.0f;
  }
  __device__ __forceinline__ void store_scaled(int i, Spinor<float> s, float extra) const {
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) s.c[a][b] = extra * s.c[a][b];
    store(i, s);
  }
};


// int16 fields are stored offset-binary: u = q + 32768 for q in [-32767, 32767].
// Conversions avoid the quarter-rate I2F/F2I instructions.  Load: splice u into
// the mantissa of 2^23 with a byte permute, giving the float 2^23 + u exactly
// ("biased" value q + kQBias); subtracting kQBias leaves q.  Store:
// a + kQStore rounds a (|a| <= 32767.5) to the nearest integer and leaves
// q + 32768 in the low 16 bits of the mantissa.
constexpr float kQBias = 8421376.0f;    // 2^23 + 2^15
constexpr float kQStore = 12615680.0f;  // 1.5 * 2^23 + 2^15
__device__ __forceinline__ float2 u16x2_biased(unsigned w) {
  return make_float2(__uint_as_float(__byte_perm(w, 0x4B000000u, 0x7610)),
                     __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7632)));
}
__device__ __forceinline__ float2 u16x2_to_f2(unsigned w) {
  const float2 b = u16x2_biased(w);
  return make_float2(b.x - kQBias, b.y - kQBias);
}
__device__ __forceinline__ unsigned f2_to_u16x2(float a, float b, float scale) {
  const unsigned ia = __float_as_uint(fmaf(a, scale, kQStore));
  const unsigned ib = __float_as_uint(fmaf(b, scale, kQStore));
  return __byte_perm(ia, ib, 0x5410);
}

template <>
struct SpinorView<Prec::F16> {
  using R = float;
  int4* v;      // [3][stride], each int4 = 8 int16 = 4 complex
  float* norm;  // [stride]
  int stride;
  __device__ __forceinline__ void load(int i, Spinor<float>& s) const {
    float sc;
    load_raw(i, s, sc);
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) s.c[a][b] = sc * s.c[a][b];
  }
  __device__ __forceinline__ void load_pair(int i, int s0, cx<float> h[2][3]) const {
    float sc;
    load_pair_raw(i, s0, h, sc);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      h[0][c] = sc * h[0][c];
      h[1][c] = sc * h[1][c];
    }
  }
  // raw int16 values as floats; the true value is raw * sc (the stencil
  // applies sc once, after the linear projection and transport).  int4
  // number k holds colour k, spins 0..3, one complex per 32-bit word.
  __device__ __forceinline__ void load_raw(int i, Spinor<float>& s, float& sc) const {
    sc = __ldg(norm + i) * (1.0f / 32767.0f);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const int4 t = __ldg(v + k * stride + i);
      const float2 a = u16x2_to_f2(t.x), b = u16x2_to_f2(t.y), c = u16x2_to_f2(t.z), d = u16x2_to_f2(t.w);
      s.c[0][k] = mkc(a.x, a.y);
      s.c[1][k] = mkc(b.x, b.y);
      s.c[2][k] = mkc(c.x, c.y);
      s.c[3][k] = mkc(d.x, d.y);
    }
  }
  // spins s0, s0+1 (s0 even) of every colour: one half of each int4
  __device__ __forceinline__ void load_pair_raw(int i, int s0, cx<float> h[2][3], float& sc) const {
    sc = __ldg(norm + i) * (1.0f / 32767.0f);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const int2* p = reinterpret_cast<const int2*>(v + c * stride + i);
      const int2 t = __ldg(p + (s0 >> 1));
      const float2 a = u16x2_to_f2(t.x), b = u16x2_to_f2(t.y);
      h[0][c] = mkc(a.x, a.y);
      h[1][c] = mkc(b.x, b.y);
    }
  }
  // biased values (q + kQBias, see u16x2_biased) of all 12 components,
  // F[spin][colour] = (re, im); the true value is (F - kQBias) * sc
  __device__ __forceinline__ void load_biased(int i, float2 F[4][3], float& sc) const {
    sc = __ldg(norm + i) * (1.0f / 32767.0f);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const int4 t = __ldg(v + k * stride + i);
      F[0][k] = u16x2_biased(t.x);
      F[1][k] = u16x2_biased(t.y);
      F[2][k] = u16x2_biased(t.z);
      F[3][k] = u16x2_biased(t.w);
    }
  }
  // stores s * extra: a common factor of the site (extra > 0) goes into the
  // norm instead of being multiplied into the 24 components
  __device__ __forceinline__ void store_scaled(int i, const Spinor<float>& s, float extra) const {
    float m = 0.f;
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) m = fmaxf(m, fmaxf(fabsf(s.c[a][b].x), fabsf(s.c[a][b].y)));
    // below 1e-30 the quotient could overflow: such a site is stored as zero
    const float inv = m > 1e-30f ? __fdividef(32767.0f, m) : 0.f;
    norm[i] = m * extra;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      int4 t;
      t.x = (int)f2_to_u16x2(s.c[0][k].x, s.c[0][k].y, inv);
      t.y = (int)f2_to_u16x2(s.c[1][k].x, s.c[1][k].y, inv);
      t.z = (int)f2_to_u16x2(s.c[2][k].x, s.c[2][k].y, inv);
      t.w = (int)f2_to_u16x2(s.c[3][k].x, s.c[3][k].y, inv);
      v[k * stride + i] = t;
    }
  }
  __device__ __forceinline__ void store(int i, const Spinor<float>& s) const { store_scaled(i, s, 1.0f); }
};

// Loads of data that a pass reads once (links, clover blocks): read-only
// path without L1 allocation, so these streamed fields leave L1 to the
// neighbour spinors, which each site reads eight times.  (Measured at
// 32^3x64: FP32 solves 2 % faster; int16 and FP64 unchanged.  Evict-first
// loads, ld.global.cs, changed nothing.)
__device__ __forceinline__ uint2 ld_once(const uint2* p) {
  uint2 r;
  asm("ld.global.nc.L1::no_allocate.v2.u32 {%0, %1}, [%2];" : "=r"(r.x), "=r"(r.y) : "l"(p));
  return r;
}
__device__ __forceinline__ int4 ld_once(const int4* p) {
  int4 r;
  asm("ld.global.nc.L1::no_allocate.v4.s32 {%0, %1, %2, %3}, [%4];"
      : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w) : "l"(p));
  return r;
}
__device__ __forceinline__ float4 ld_once(const float4* p) {
  float4 r;
  asm("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
      : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w) : "l"(p));
  return r;
}
__device__ __forceinline__ double2 ld_once(const double2* p) {
  double2 r;
  asm("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(r.x), "=d"(r.y) : "l"(p));
  return r;
}
__device__ __forceinline__ float ld_once(const float* p) {
  float r;
  asm("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(r) : "l"(p));
  return r;
}

// links --------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void reconstruct_col3(Link<R>& u) {
  // su3.F90:300-310: third column from the first two
  u.m[0][2] = conjg(u.m[1][0] * u.m[2][1] - u.m[2][0] * u.m[1][1]);
  u.m[1][2] = conjg(u.m[2][0] * u.m[0][1] - u.m[0][0] * u.m[2][1]);
  u.m[2][2] = conjg(u.m[0][0] * u.m[1][1] - u.m[1][0] * u.m[0][1]);
}

// the three words of an int16 link (columns 1, 2; offset-binary) -> the link
// times 32767 (U = u * lsc): the third column is rebuilt from the first two
// and brought to the same scale, so one factor per hop replaces a multiply of
// every entry
__device__ __forceinline__ void links16_decode(uint2 t0, uint2 t1, uint2 t2, Link<float>& u, float& lsc) {
  float2 e;
  e = u16x2_to_f2(t0.x); u.m[0][0] = mkc(e.x, e.y);
  e = u16x2_to_f2(t0.y); u.m[1][0] = mkc(e.x, e.y);
  e = u16x2_to_f2(t1.x); u.m[2][0] = mkc(e.x, e.y);
  e = u16x2_to_f2(t1.y); u.m[0][1] = mkc(e.x, e.y);
  e = u16x2_to_f2(t2.x); u.m[1][1] = mkc(e.x, e.y);
  e = u16x2_to_f2(t2.y); u.m[2][1] = mkc(e.x, e.y);
  reconstruct_col3(u);  // 32767^2 times the true column
  lsc = 1.0f / 32767.0f;
#pragma unroll
  for (int r = 0; r < 3; r++) u.m[r][2] = lsc * u.m[r][2];
}

template <Prec P>
struct GaugeView;

template <>
struct GaugeView<Prec::F64> {
  using R = double;
  double2* v;  // [4][2][9][stride], or [4][2][6][stride] with rec12
  int stride;
  int rec12 = 0;
  __device__ __forceinline__ void load(int mu, int eo, int i, Link<double>& u) const {
    if (rec12) {
      const double2* b = v + (size_t)((mu * 2 + eo) * 6) * stride + i;
#pragma unroll
      for (int c = 0; c < 2; c++)
#pragma unroll
        for (int r = 0; r < 3; r++) {
          double2 t = ld_once(b + (c * 3 + r) * stride);
          u.m[r][c] = mkc(t.x, t.y);
        }
      reconstruct_col3(u);
      return;
    }
    const double2* b = v + (size_t)((mu * 2 + eo) * 9) * stride + i;
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int r = 0; r < 3; r++) {
        double2 t = ld_once(b + (c * 3 + r) * stride);
        u.m[r][c] = mkc(t.x, t.y);
      }
  }
  __device__ __forceinline__ void load_raw(int mu, int eo, int i, Link<double>& u, double& lsc) const {
    load(mu, eo, i, u);
    lsc = 1.0;
  }
  // the link of one hop: U_mu(idx) of parity eo (idx = the site for a
  // forward hop, its backward neighbour for a backward one)
  __device__ __forceinline__ void hop_link(int mu, bool, int eo, int idx, Link<double>& u, double& lsc) const {
    load_raw(mu, eo, idx, u, lsc);
  }
};

template <>
struct GaugeView<Prec::F32> {
  using R = float;
  float4* v;  // [4][2][3][stride]
  int stride;
  __device__ __forceinline__ void load(int mu, int eo, int i, Link<float>& u) const {
    const float4* b = v + (size_t)((mu * 2 + eo) * 3) * stride + i;
    float4 t0 = ld_once(b), t1 = ld_once(b + stride), t2 = ld_once(b + 2 * stride);
    u.m[0][0] = mkc(t0.x, t0.y);
    u.m[1][0] = mkc(t0.z, t0.w);
    u.m[2][0] = mkc(t1.x, t1.y);
    u.m[0][1] = mkc(t1.z, t1.w);
    u.m[1][1] = mkc(t2.x, t2.y);
    u.m[2][1] = mkc(t2.z, t2.w);
    reconstruct_col3(u);
  }
  __device__ __forceinline__ void load_raw(int mu, int eo, int i, Link<float>& u, float& lsc) const {
    load(mu, eo, i, u);
    lsc = 1.0f;
  }
  // the link of one hop: U_mu(idx) of parity eo (idx = the site for a
  // forward hop, its backward neighbour for a backward one)
  __device__ __forceinline__ void hop_link(int mu, bool, int eo, int idx, Link<float>& u, float& lsc) const {
    load_raw(mu, eo, idx, u, lsc);
  }
};

template <>
struct GaugeView<Prec::F16> {
  using R = float;
  short4* v;  // [4][2][3][stride], offset-binary entries of 32767 u
  int stride;
  // the link times 32767 (U = u * lsc): columns 1, 2 as stored, the third
  // rebuilt from them and brought to the same scale, so that one factor per
  // hop replaces a multiply of every entry
  __device__ __forceinline__ void load_raw(int mu, int eo, int i, Link<float>& u, float& lsc) const {
    // one short4 = two complex entries = two 32-bit words
    const uint2* b = reinterpret_cast<const uint2*>(v) + (size_t)((mu * 2 + eo) * 3) * stride + i;
    links16_decode(ld_once(b), ld_once(b + stride), ld_once(b + 2 * stride), u, lsc);
  }
  __device__ __forceinline__ void hop_link(int mu, bool, int eo, int idx, Link<float>& u, float& lsc) const {
    load_raw(mu, eo, idx, u, lsc);
  }
  __device__ __forceinline__ void load(int mu, int eo, int i, Link<float>& u) const {
    float lsc;
    load_raw(mu, eo, i, u, lsc);
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
      for (int c = 0; c < 3; c++) u.m[r][c] = lsc * u.m[r][c];
  }
};

// clover blocks ------------------------------------------------------------
// Packed 18-slot chiral block (clover.h:28-55): slot 0 = (A11,A22), 10 =
// (A33,A44), 16 = (A55,A66) real diagonals; upper entries in slots 1-9,11-15,17.

// word k (0..4) of chiral block chi of an int16 clover site (int4 number
// chi*4 + k, 4 slots each) -> the slots of that block it holds, raw values
__device__ __forceinline__ void clover16_decode(int chi, int k, int4 t, cx<float> a[18]) {
  const unsigned w[4] = {(unsigned)t.x, (unsigned)t.y, (unsigned)t.z, (unsigned)t.w};
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const int slot = 4 * (chi * 4 + k) + j - chi * 18;
    if (slot >= 0 && slot < 18) {
      const float2 e = u16x2_to_f2(w[j]);
      a[slot] = mkc(e.x, e.y);
    }
  }
}

template <Prec P>
struct CloverView;

template <>
struct CloverView<Prec::F64> {
  using R = double;
  double2* v;  // [36][stride] for one parity
  int stride;
  __device__ __forceinline__ void load_block(int i, int chi, cx<double> a[18]) const {
#pragma unroll
    for (int k = 0; k < 18; k++) {
      double2 t = ld_once(v + (chi * 18 + k) * stride + i);
      a[k] = mkc(t.x, t.y);
    }
  }
  __device__ __forceinline__ void load_block_raw(int i, int chi, cx<double> a[18], double& sc) const {
    load_block(i, chi, a);
    sc = 1.0;
  }
};

template <>
struct CloverView<Prec::F32> {
  using R = float;
  float4* v;  // [18][stride]
  int stride;
  __device__ __forceinline__ void load_block(int i, int chi, cx<float> a[18]) const {
#pragma unroll
    for (int k = 0; k < 9; k++) {
      float4 t = ld_once(v + (chi * 9 + k) * stride + i);
      a[2 * k] = mkc(t.x, t.y);
      a[2 * k + 1] = mkc(t.z, t.w);
    }
  }
  __device__ __forceinline__ void load_block_raw(int i, int chi, cx<float> a[18], float& sc) const {
    load_block(i, chi, a);
    sc = 1.0f;
  }
};

template <>
struct CloverView<Prec::F16> {
  using R = float;
  int4* v;  // [9][stride], 8 int16 = 4 slots each
  float* norm;
  int stride;
  // slots chi*18 .. chi*18+17 live in int4 numbers (chi*18)/4 .. (chi*18+17)/4:
  // block 0 in words 0-4, block 1 in words 4-8
  __device__ __forceinline__ void load_block(int i, int chi, cx<float> a[18]) const {
    float sc;
    load_block_raw(i, chi, a, sc);
#pragma unroll
    for (int k = 0; k < 18; k++) a[k] = sc * a[k];
  }
  // raw int16 values; the block is raw * sc (applied to the block's output)
  __device__ __forceinline__ void load_block_raw(int i, int chi, cx<float> a[18], float& sc) const {
    sc = ld_once(norm + i) * (1.0f / 32767.0f);
#pragma unroll
    for (int k = 0; k < 5; k++) clover16_decode(chi, k, ld_once(v + (chi * 4 + k) * stride + i), a);
  }
};

// y = A x for one packed Hermitian 6x6 block (clover_mult_a.h90)
template <typename R>
__device__ __forceinline__ void clover_block_mv(const cx<R>* a, const cx<R> x[6], cx<R> y[6]) {
  const R d0 = a[0].x, d1 = a[0].y, d2 = a[10].x, d3 = a[10].y, d4 = a[16].x, d5 = a[16].y;
  // upper-triangle slots
  const cx<R> a01 = a[1], a02 = a[2], a03 = a[3], a04 = a[4], a05 = a[5];
  const cx<R> a12 = a[6], a13 = a[7], a14 = a[8], a15 = a[9];
  const cx<R> a23 = a[11], a24 = a[12], a25 = a[13];
  const cx<R> a34 = a[14], a35 = a[15];
  const cx<R> a45 = a[17];
  cx<R> t;
  t = d0 * x[0];
  t = fma_c(t, a01, x[1]); t = fma_c(t, a02, x[2]); t = fma_c(t, a03, x[3]); t = fma_c(t, a04, x[4]); t = fma_c(t, a05, x[5]);
  y[0] = t;
  t = d1 * x[1];
  t = fma_cc(t, a01, x[0]); t = fma_c(t, a12, x[2]); t = fma_c(t, a13, x[3]); t = fma_c(t, a14, x[4]); t = fma_c(t, a15, x[5]);
  y[1] = t;
  t = d2 * x[2];
  t = fma_cc(t, a02, x[0]); t = fma_cc(t, a12, x[1]); t = fma_c(t, a23, x[3]); t = fma_c(t, a24, x[4]); t = fma_c(t, a25, x[5]);
  y[2] = t;
  t = d3 * x[3];
  t = fma_cc(t, a03, x[0]); t = fma_cc(t, a13, x[1]); t = fma_cc(t, a23, x[2]); t = fma_c(t, a34, x[4]); t = fma_c(t, a35, x[5]);
  y[3] = t;
  t = d4 * x[4];
  t = fma_cc(t, a04, x[0]); t = fma_cc(t, a14, x[1]); t = fma_cc(t, a24, x[2]); t = fma_cc(t, a34, x[3]); t = fma_c(t, a45, x[5]);
  y[4] = t;
  t = d5 * x[5];
  t = fma_cc(t, a05, x[0]); t = fma_cc(t, a15, x[1]); t = fma_cc(t, a25, x[2]); t = fma_cc(t, a35, x[3]); t = fma_cc(t, a45, x[4]);
  y[5] = t;
}

// out = A in on one site, both chiral blocks (clover_mult_a.F90:45-95): the
// blocks act on x+- = psi(spin 1,2) +- psi(spin 3,4).  The _raw form leaves
// out = (A / sc) in, sc the storage scale of the site's blocks (1 except for
// int16), for callers that fold sc into a later factor.
template <typename CV, typename R>
__device__ __forceinline__ void clover_apply_raw(const CV& A, int i, const Spinor<R>& in, Spinor<R>& out, R& sc) {
  cx<R> x[6], y[6], a[18];
#pragma unroll
  for (int k = 0; k < 6; k++) x[k] = in.c[k / 3][k % 3] + in.c[k / 3 + 2][k % 3];
  A.load_block_raw(i, 0, a, sc);
  clover_block_mv(a, x, y);
#pragma unroll
  for (int k = 0; k < 6; k++) {
    out.c[k / 3][k % 3] = y[k];
    out.c[k / 3 + 2][k % 3] = y[k];
  }
#pragma unroll
  for (int k = 0; k < 6; k++) x[k] = in.c[k / 3][k % 3] - in.c[k / 3 + 2][k % 3];
  A.load_block_raw(i, 1, a, sc);  // both blocks of a site share one scale
  clover_block_mv(a, x, y);
#pragma unroll
  for (int k = 0; k < 6; k++) {
    out.c[k / 3][k % 3] = out.c[k / 3][k % 3] + y[k];
    out.c[k / 3 + 2][k % 3] = out.c[k / 3 + 2][k % 3] - y[k];
  }
}
template <Prec P, typename R>
__device__ __forceinline__ void clover_apply(const CloverView<P>& A, int i, const Spinor<R>& in, Spinor<R>& out) {
  R sc;
  clover_apply_raw(A, i, in, out, sc);
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) out.c[a][b] = sc * out.c[a][b];
}

// ---------------------------------------------------------------------------
// clover blocks at any hopping parameter.  clover_init.F90:46-77 builds each
// chiral block as 1 + (-c_sw kappa / 8)(p +- q), from field strengths that
// do not depend on kappa; with T = (-c_sw / 8)(p +- q) stored in the packed
// slots in place of the block, A(kappa) = 1 + kappa T gives every kappa its
// own clover term from one field.  The stored blocks of BQCD are halved
// (clover_inv.F90:105-137, 211-216): a = A/2, ainv = A^-1 / 2.
// ---------------------------------------------------------------------------
// out = (A(kappa) / 2) in on one site, in the chiral layout of clover_apply_raw
template <typename CV, typename R>
__device__ __forceinline__ void clover_apply_kt(const CV& T, int i, const Spinor<R>& in, Spinor<R>& out, R kappa) {
  cx<R> x[6], y[6], a[18];
  R sc;
#pragma unroll
  for (int chi = 0; chi < 2; chi++) {
#pragma unroll
    for (int k = 0; k < 6; k++)
      x[k] = chi == 0 ? in.c[k / 3][k % 3] + in.c[k / 3 + 2][k % 3] : in.c[k / 3][k % 3] - in.c[k / 3 + 2][k % 3];
    T.load_block_raw(i, chi, a, sc);
    clover_block_mv(a, x, y);
    const R hk = R(0.5) * kappa * sc;
#pragma unroll
    for (int k = 0; k < 6; k++) {
      const cx<R> z = mkc(fma(hk, y[k].x, R(0.5) * x[k].x), fma(hk, y[k].y, R(0.5) * x[k].y));
      if (chi == 0) {
        out.c[k / 3][k % 3] = z;
        out.c[k / 3 + 2][k % 3] = z;
      } else {
        out.c[k / 3][k % 3] = out.c[k / 3][k % 3] + z;
        out.c[k / 3 + 2][k % 3] = out.c[k / 3 + 2][k % 3] - z;
      }
    }
  }
}

// y = (A(kappa)^-1 / 2) x for one packed block a (raw values times sc): the
// LDL^+ factorisation of clover_inv.F90:45-101 in registers, then the
// substitutions of clover_mult_b.h90
template <typename R>
__device__ __forceinline__ void block_inv_apply_kt(const cx<R> a[18], R sc, R kappa, const cx<R> x[6], cx<R> y[6]) {
  // packed upper-triangle slot of (r, c), r < c (clover.h:28-55)
  constexpr int up[6][6] = {{-1, 1, 2, 3, 4, 5},    {-1, -1, 6, 7, 8, 9},    {-1, -1, -1, 11, 12, 13},
                            {-1, -1, -1, -1, 14, 15}, {-1, -1, -1, -1, -1, 17}, {-1, -1, -1, -1, -1, -1}};
  const R ks = kappa * sc;
  R dg[6];
  dg[0] = a[0].x; dg[1] = a[0].y; dg[2] = a[10].x; dg[3] = a[10].y; dg[4] = a[16].x; dg[5] = a[16].y;
  cx<R> L[6][6];
  R d[6], dinv[6];
#pragma unroll
  for (int r = 0; r < 6; r++) {
    cx<R> tmp[6];
#pragma unroll
    for (int c = 0; c < r; c++) {
      cx<R> t = ks * conjg(a[up[c][r]]);  // A(r, c) = conj(A(c, r))
#pragma unroll
      for (int k = 0; k < c; k++) t = t - tmp[k] * conjg(L[c][k]);
      tmp[c] = t;
    }
#pragma unroll
    for (int c = 0; c < r; c++) L[r][c] = dinv[c] * tmp[c];
    R dr = R(1) + ks * dg[r];
#pragma unroll
    for (int k = 0; k < r; k++) dr = dr - d[k] * norm2(L[r][k]);
    d[r] = dr;
    dinv[r] = R(1) / dr;
  }
  cx<R> w[6];
#pragma unroll
  for (int r = 0; r < 6; r++) {
    cx<R> t = x[r];
#pragma unroll
    for (int c = 0; c < r; c++) t = t - L[r][c] * w[c];
    w[r] = t;
  }
#pragma unroll
  for (int r = 5; r >= 0; r--) {
    cx<R> t = dinv[r] * w[r];
#pragma unroll
    for (int c = r + 1; c < 6; c++) t = t - conjg(L[c][r]) * y[c];
    y[r] = t;
  }
#pragma unroll
  for (int r = 0; r < 6; r++) y[r] = R(0.5) * y[r];
}

// out = (A(kappa)^-1 / 2) in on one site
template <typename CV, typename R>
__device__ __forceinline__ void clover_inv_apply_kt(const CV& T, int i, const Spinor<R>& in, Spinor<R>& out,
                                                    R kappa) {
  cx<R> x[6], y[6], a[18];
  R sc;
#pragma unroll
  for (int chi = 0; chi < 2; chi++) {
#pragma unroll
    for (int k = 0; k < 6; k++)
      x[k] = chi == 0 ? in.c[k / 3][k % 3] + in.c[k / 3 + 2][k % 3] : in.c[k / 3][k % 3] - in.c[k / 3 + 2][k % 3];
    T.load_block_raw(i, chi, a, sc);
    block_inv_apply_kt(a, sc, kappa, x, y);
#pragma unroll
    for (int k = 0; k < 6; k++) {
      if (chi == 0) {
        out.c[k / 3][k % 3] = y[k];
        out.c[k / 3 + 2][k % 3] = y[k];
      } else {
        out.c[k / 3][k % 3] = out.c[k / 3][k % 3] + y[k];
        out.c[k / 3 + 2][k % 3] = out.c[k / 3 + 2][k % 3] - y[k];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Wilson hop (d/D21.F90, d/D21xyzt.F90).  Forward hop: (1 - s gamma_mu)
// projection of psi(x+mu), times U_mu(x); backward hop: (1 + s gamma_mu)
// projection of psi(x-mu) times U_mu(x-mu)^+; s = +1 for d, -1 for d_dag.
// gamma basis of BQCD (UKQCD / Dirac): gamma_4 = diag(1,1,-1,-1).
// ---------------------------------------------------------------------------
template <typename R, bool DAG>
__device__ __forceinline__ void project(const Spinor<R>& p, int mu, bool fwd, cx<R> h[2][3]) {
  const R s = DAG ? R(-1) : R(1);
  const R sg = fwd ? -s : s;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    if (mu == 0) {
      h[0][c] = p.c[0][c] + sg * itimes(p.c[3][c]);
      h[1][c] = p.c[1][c] + sg * itimes(p.c[2][c]);
    } else if (mu == 1) {
      h[0][c] = p.c[0][c] + sg * p.c[3][c];
      h[1][c] = p.c[1][c] - sg * p.c[2][c];
    } else {
      h[0][c] = p.c[0][c] + sg * itimes(p.c[2][c]);
      h[1][c] = p.c[1][c] - sg * itimes(p.c[3][c]);
    }
  }
}

// sa*(A - kQBias) + sb*(B - kQBias) for biased int16 values A, B; the signs
// are constants once the hop loop is unrolled.  A difference of biased values
// is exact in one add, a sum takes two (every intermediate is an integer
// below 2^24).
__device__ __forceinline__ float comb_biased(float A, float B, float sa, float sb) {
  if (sa == -sb) return sa > 0.f ? A - B : B - A;
  const float t = (A - 2.0f * kQBias) + B;
  return sa > 0.f ? t : -t;
}
// project() on biased int16 components (SpinorView<F16>::load_biased): the
// same half spinor, up to the site's storage scale, without first removing
// the bias from every component
template <bool DAG>
__device__ __forceinline__ void project_biased(const float2 F[4][3], int mu, bool fwd, cx<float> h[2][3]) {
  const float s = DAG ? -1.f : 1.f;
  const float sg = fwd ? -s : s;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    if (mu == 0) {  // h0 = p0 + sg i p3, h1 = p1 + sg i p2
      h[0][c] = mkc(comb_biased(F[0][c].x, F[3][c].y, 1.f, -sg), comb_biased(F[0][c].y, F[3][c].x, 1.f, sg));
      h[1][c] = mkc(comb_biased(F[1][c].x, F[2][c].y, 1.f, -sg), comb_biased(F[1][c].y, F[2][c].x, 1.f, sg));
    } else if (mu == 1) {  // h0 = p0 + sg p3, h1 = p1 - sg p2
      h[0][c] = mkc(comb_biased(F[0][c].x, F[3][c].x, 1.f, sg), comb_biased(F[0][c].y, F[3][c].y, 1.f, sg));
      h[1][c] = mkc(comb_biased(F[1][c].x, F[2][c].x, 1.f, -sg), comb_biased(F[1][c].y, F[2][c].y, 1.f, -sg));
    } else {  // h0 = p0 + sg i p2, h1 = p1 - sg i p3
      h[0][c] = mkc(comb_biased(F[0][c].x, F[2][c].y, 1.f, -sg), comb_biased(F[0][c].y, F[2][c].x, 1.f, sg));
      h[1][c] = mkc(comb_biased(F[1][c].x, F[3][c].y, 1.f, sg), comb_biased(F[1][c].y, F[3][c].x, 1.f, -sg));
    }
  }
}

// acc + a*f and acc + a*(i f): two FMAs each
template <typename R>
__device__ __forceinline__ cx<R> axpy_c(cx<R> acc, R a, cx<R> f) {
  return mkc(fma(a, f.x, acc.x), fma(a, f.y, acc.y));
}
template <typename R>
__device__ __forceinline__ cx<R> axpy_ic(cx<R> acc, R a, cx<R> f) {
  return mkc(fma(-a, f.y, acc.x), fma(a, f.x, acc.y));
}

// b += k * (reconstruction of the transported forward half spinor f); k
// carries the hop's boundary sign and storage scales, so applying it here
// costs no instruction beyond the accumulation itself
template <typename R, bool DAG>
__device__ __forceinline__ void recon_fwd(Spinor<R>& b, int mu, const cx<R> f[2][3], R k) {
  const R sk = DAG ? -k : k;
  const R k2 = R(2) * k;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    if (mu == 3) {
      if (!DAG) {
        b.c[2][c] = axpy_c(b.c[2][c], k2, f[0][c]);
        b.c[3][c] = axpy_c(b.c[3][c], k2, f[1][c]);
      } else {
        b.c[0][c] = axpy_c(b.c[0][c], k2, f[0][c]);
        b.c[1][c] = axpy_c(b.c[1][c], k2, f[1][c]);
      }
    } else {
      b.c[0][c] = axpy_c(b.c[0][c], k, f[0][c]);
      b.c[1][c] = axpy_c(b.c[1][c], k, f[1][c]);
      if (mu == 0) {
        b.c[2][c] = axpy_ic(b.c[2][c], sk, f[1][c]);
        b.c[3][c] = axpy_ic(b.c[3][c], sk, f[0][c]);
      } else if (mu == 1) {
        b.c[2][c] = axpy_c(b.c[2][c], sk, f[1][c]);
        b.c[3][c] = axpy_c(b.c[3][c], -sk, f[0][c]);
      } else {
        b.c[2][c] = axpy_ic(b.c[2][c], sk, f[0][c]);
        b.c[3][c] = axpy_ic(b.c[3][c], -sk, f[1][c]);
      }
    }
  }
}

// b += k * (reconstruction of the transported backward half spinor f)
template <typename R, bool DAG>
__device__ __forceinline__ void recon_bwd(Spinor<R>& b, int mu, const cx<R> f[2][3], R k) {
  const R sk = DAG ? -k : k;
  const R k2 = R(2) * k;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    if (mu == 3) {
      if (!DAG) {
        b.c[0][c] = axpy_c(b.c[0][c], k2, f[0][c]);
        b.c[1][c] = axpy_c(b.c[1][c], k2, f[1][c]);
      } else {
        b.c[2][c] = axpy_c(b.c[2][c], k2, f[0][c]);
        b.c[3][c] = axpy_c(b.c[3][c], k2, f[1][c]);
      }
    } else {
      b.c[0][c] = axpy_c(b.c[0][c], k, f[0][c]);
      b.c[1][c] = axpy_c(b.c[1][c], k, f[1][c]);
      if (mu == 0) {
        b.c[2][c] = axpy_ic(b.c[2][c], -sk, f[1][c]);
        b.c[3][c] = axpy_ic(b.c[3][c], -sk, f[0][c]);
      } else if (mu == 1) {
        b.c[2][c] = axpy_c(b.c[2][c], -sk, f[1][c]);
        b.c[3][c] = axpy_c(b.c[3][c], sk, f[0][c]);
      } else {
        b.c[2][c] = axpy_ic(b.c[2][c], -sk, f[0][c]);
        b.c[3][c] = axpy_ic(b.c[3][c], sk, f[1][c]);
      }
    }
  }
}

// f = U h   (colour vectors h[0], h[1])
template <typename R>
__device__ __forceinline__ void mul_u(const Link<R>& u, const cx<R> h[2][3], cx<R> f[2][3]) {
#pragma unroll
  for (int k = 0; k < 2; k++)
#pragma unroll
    for (int r = 0; r < 3; r++) {
      cx<R> t = u.m[r][0] * h[k][0];
      t = fma_c(t, u.m[r][1], h[k][1]);
      f[k][r] = fma_c(t, u.m[r][2], h[k][2]);
    }
}
// f = U^+ h
template <typename R>
__device__ __forceinline__ void mul_ud(const Link<R>& u, const cx<R> h[2][3], cx<R> f[2][3]) {
#pragma unroll
  for (int k = 0; k < 2; k++)
#pragma unroll
    for (int r = 0; r < 3; r++) {
      cx<R> t = mulc(h[k][0], u.m[0][r]);
      t = fma_cc(t, u.m[1][r], h[k][1]);
      f[k][r] = fma_cc(t, u.m[2][r], h[k][2]);
    }
}

// b += hscale * (sum over the 8 hops of the even/odd hopping term): out(parity
// e, site i) from the field ``in`` of the opposite parity (d/D21.F90:29-77).
// b is accumulated into, so a caller either zeroes it or starts it with the
// site-local terms of its operator.
// Every storage scale (int16 spinors and links), the boundary sign and hscale
// are applied as one factor per hop, to the transported half spinor.
template <Prec PS, bool DAG, typename UV>
__device__ __forceinline__ void wilson_hop(const Geom& g, int e, int i, const Site& st,
                                           const SpinorView<PS>& in, const UV& U,
                                           Spinor<typename SpinorView<PS>::R>& b,
                                           typename SpinorView<PS>::R hscale = 1) {
  using R = typename SpinorView<PS>::R;
  const int o = 1 - e;
#pragma unroll
  for (int mu = 3; mu >= 0; mu--) {
    // forward hop
    {
      int j = neighbour(g, st, i, mu, true);
      cx<R> h[2][3], f[2][3];
      R sc, lsc;
      if (mu == 3) {
        // (1 -+ gamma_4) keeps two spins: (3,4) for d, (1,2) for d_dag
        in.load_pair_raw(j, DAG ? 0 : 2, h, sc);
      } else if constexpr (PS == Prec::F16) {
        float2 F[4][3];
        in.load_biased(j, F, sc);
        project_biased<DAG>(F, mu, true, h);
      } else {
        Spinor<R> p;
        in.load_raw(j, p, sc);
        project<R, DAG>(p, mu, true, h);
      }
      Link<R> u;
      U.hop_link(mu, true, e, i, u, lsc);
      mul_u(u, h, f);
      recon_fwd<R, DAG>(b, mu, f, (R)hop_sign(g, st, mu, true) * sc * lsc * hscale);
    }
    // backward hop
    {
      int j = neighbour(g, st, i, mu, false);
      cx<R> h[2][3], f[2][3];
      R sc, lsc;
      if (mu == 3) {
        in.load_pair_raw(j, DAG ? 2 : 0, h, sc);
      } else if constexpr (PS == Prec::F16) {
        float2 F[4][3];
        in.load_biased(j, F, sc);
        project_biased<DAG>(F, mu, false, h);
      } else {
        Spinor<R> p;
        in.load_raw(j, p, sc);
        project<R, DAG>(p, mu, false, h);
      }
      Link<R> u;
      U.hop_link(mu, false, o, j, u, lsc);
      mul_ud(u, h, f);
      recon_bwd<R, DAG>(b, mu, f, (R)hop_sign(g, st, mu, false) * sc * lsc * hscale);
    }
  }
}

// wilson_hop for int16 fields with every link of the site loaded first: the
// 24 link words (8 hops x 3) are requested before any neighbour spinor, so
// they stream from HBM while the gathers, which mostly hit L2, proceed hop by
// hop.  Same products in the same order as wilson_hop, so the result is
// bit-identical; it needs about 40 more registers.
template <bool DAG>
__device__ __forceinline__ void wilson_hop_lf(const Geom& g, int e, int i, const Site& st,
                                              const SpinorView<Prec::F16>& in, const GaugeView<Prec::F16>& U,
                                              Spinor<float>& b, float hscale = 1.f) {
  const int o = 1 - e;
  const uint2* ub = reinterpret_cast<const uint2*>(U.v);
  const int S = U.stride;
  uint2 W[4][2][3];
  int J[4][2];
#pragma unroll
  for (int mu = 3; mu >= 0; mu--) {
    J[mu][0] = neighbour(g, st, i, mu, true);
    J[mu][1] = neighbour(g, st, i, mu, false);
#pragma unroll
    for (int w = 0; w < 3; w++) {
      W[mu][0][w] = ld_once(ub + (size_t)((mu * 2 + e) * 3 + w) * S + i);
      W[mu][1][w] = ld_once(ub + (size_t)((mu * 2 + o) * 3 + w) * S + J[mu][1]);
    }
  }
#pragma unroll
  for (int mu = 3; mu >= 0; mu--) {
#pragma unroll
    for (int fb = 0; fb < 2; fb++) {
      const bool fwd = fb == 0;
      cx<float> h[2][3], f[2][3];
      float sc, lsc;
      if (mu == 3) {
        in.load_pair_raw(J[mu][fb], fwd ? (DAG ? 0 : 2) : (DAG ? 2 : 0), h, sc);
      } else {
        float2 F[4][3];
        in.load_biased(J[mu][fb], F, sc);
        project_biased<DAG>(F, mu, fwd, h);
      }
      Link<float> u;
      links16_decode(W[mu][fb][0], W[mu][fb][1], W[mu][fb][2], u, lsc);
      const float k = (float)hop_sign(g, st, mu, fwd) * sc * lsc * hscale;
      if (fwd) {
        mul_u(u, h, f);
        recon_fwd<float, DAG>(b, mu, f, k);
      } else {
        mul_ud(u, h, f);
        recon_bwd<float, DAG>(b, mu, f, k);
      }
    }
  }
}

// (1 + i h gamma_5) x, gamma_5 swapping spins 1<->3, 2<->4 (h_mult.F90:51-82)
template <typename R>
__device__ __forceinline__ void h_mult_b(Spinor<R>& x, R h) {
#pragma unroll
  for (int c = 0; c < 3; c++) {
    cx<R> x1 = x.c[0][c], x2 = x.c[1][c], x3 = x.c[2][c], x4 = x.c[3][c];
    x.c[0][c] = x1 + h * itimes(x3);
    x.c[1][c] = x2 + h * itimes(x4);
    x.c[2][c] = x3 + h * itimes(x1);
    x.c[3][c] = x4 + h * itimes(x2);
  }
}

// ---------------------------------------------------------------------------
// launch tiling: several right-hand sides share one launch.  CTA b serves RHS
// b % nr and site block b / nr, so the nr CTAs reading the same links and
// clover blocks are adjacent in the launch order: those fields come from HBM
// once and from L2 for the other nr-1.  nr = 1 is the single-RHS launch.
// ---------------------------------------------------------------------------
constexpr int kMaxRhs = 16;
constexpr int kRedVals = 4;  // reduction slots per RHS

struct Tile {
  int rhs;  // right-hand side of this CTA
  int sb;   // site block
  int nsb;  // site blocks per RHS
  int i;    // site of this thread
};
__device__ __forceinline__ Tile tile(int nr) {
  Tile t;
  t.rhs = blockIdx.x % nr;
  t.sb = blockIdx.x / nr;
  t.nsb = gridDim.x / nr;
  t.i = t.sb * blockDim.x + threadIdx.x;
  return t;
}

// ---------------------------------------------------------------------------
// deterministic block reductions: partial[k * stride + sb] per value k, the
// last of the nsb site blocks of one RHS to arrive sums them in block order
// ---------------------------------------------------------------------------
template <int N>
__device__ __forceinline__ void block_reduce_store(double (&v)[N], double* partial, int nblocks_stride, int sb) {
  __shared__ double red[N][32];
#pragma unroll
  for (int k = 0; k < N; k++) {
    double x = v[k];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    v[k] = x;
  }
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < N; k++) red[k][warp] = v[k];
  }
  __syncthreads();
  if (warp == 0) {
    int nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < N; k++) {
      double x = lane < nw ? red[k][lane] : 0.0;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
      if (lane == 0) partial[k * nblocks_stride + sb] = x;
    }
  }
}

// Called by every block after block_reduce_store; returns true in all threads
// of the last of the nsb blocks to arrive, which then sums the partials.
__device__ __forceinline__ bool last_block(unsigned int* counter, int nsb) {
  __shared__ bool is_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned int t = atomicAdd(counter, 1u);
    is_last = (t == (unsigned)nsb - 1u);
  }
  __syncthreads();
  return is_last;
}

template <int N>
__device__ __forceinline__ void final_sum(const double* partial, int nblocks_stride, int nsb, double (&out)[N]) {
  // executed by a whole block (the last to arrive, or the block that sums
  // another launch's partials): warp-parallel fixed-order sum.  Each
  // thread keeps 8 loads in flight (8 running sums, combined in a fixed
  // order), so the tail that the rest of the GPU waits for costs a few L2
  // latencies rather than one per partial.
  __shared__ double red[N][32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < N; k++) {
    const double* p = partial + k * nblocks_stride;
    double s[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    int b = threadIdx.x;
    for (; b + 7 * (int)blockDim.x < nsb; b += 8 * blockDim.x) {
      double t[8];
#pragma unroll
      for (int j = 0; j < 8; j++) t[j] = __ldcg(p + b + j * blockDim.x);
#pragma unroll
      for (int j = 0; j < 8; j++) s[j] += t[j];
    }
#pragma unroll
    for (int j = 0; j < 7; j++)
      if (b + j * (int)blockDim.x < nsb) s[j] += __ldcg(p + b + j * blockDim.x);
    double x = ((s[0] + s[1]) + (s[2] + s[3])) + ((s[4] + s[5]) + (s[6] + s[7]));
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    if (lane == 0) red[k][warp] = x;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < N; k++) {
    double x = 0.0;
    for (int w = 0; w < nw; w++) x += red[k][w];
    out[k] = x;
  }
  __syncthreads();
}

}  // namespace bqcdg
