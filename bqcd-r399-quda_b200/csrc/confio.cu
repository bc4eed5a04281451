// confio.cu -- BQCD configuration files on the device: the reordering of
// conf_seq (conf.F90:219-259) between the resident links and the file order
// of one time slice, the big-endian REAL(8) of field_io (swap_endian8,
// misc.F90:197-240), the third column rebuilt on reading (u_complete,
// su3.F90:301-310), and the POSIX cksum of each slice file (cksum.c).
//
// File order of slice t: records by z, then y, then x; per site the 24
// complex numbers u(c1, c2, mu), rows c1 fastest, columns c2 = 1, 2, then mu.
// One thread serves one site: it moves its 384 bytes and computes their CRC
// in registers.  A CRC is linear over GF(2): with the register starting at
// 0, the CRC of the whole slice is the XOR over sites of each site's CRC
// times x^(8 * 384 * (number of sites after it)) mod P.  The powers
// x^(8 * 384 * 2^j) come precomputed from the host; each thread multiplies
// by those of the set bits of its count, and the XOR over the slice goes
// through warp shuffles and one atomicXor per warp.  The byte count and the
// final complement of cksum are applied on the host.
#include "kernels.cuh"

namespace bqcdg {

namespace {

constexpr unsigned kCrcPoly = 0x04C11DB7u;  // the POSIX.2 cksum generator
constexpr int kSiteBytes = 24 * 16;          // one site of one slice file

__constant__ unsigned c_site_pow[32];        // x^(8 * 384 * 2^j) mod P

// a(x) b(x) mod P, most significant bit = coefficient of x^31
__device__ __forceinline__ unsigned gf_mul(unsigned a, unsigned b) {
  unsigned r = 0;
#pragma unroll 4
  for (int k = 0; k < 32; k++) {
    if (b & 1u) r ^= a;
    b >>= 1;
    a = (a & 0x80000000u) ? (a << 1) ^ kCrcPoly : (a << 1);
  }
  return r;
}

// the 8 bytes of a double, most significant first (big-endian), as two
// words: hi holds bytes 0-3 of the file, lo bytes 4-7, each word in
// little-endian memory order
__device__ __forceinline__ uint2 be_words(double v) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  const unsigned h = (unsigned)(b >> 32), l = (unsigned)b;
  return make_uint2(__byte_perm(h, 0, 0x0123), __byte_perm(l, 0, 0x0123));
}
__device__ __forceinline__ double be_double(uint2 w) {
  const unsigned h = __byte_perm(w.x, 0, 0x0123), l = __byte_perm(w.y, 0, 0x0123);
  return __longlong_as_double((long long)(((unsigned long long)h << 32) | l));
}

// CRC register after the 4 bytes of word w (file order = memory order)
__device__ __forceinline__ unsigned crc_word(unsigned crc, unsigned w, const unsigned* tab) {
#pragma unroll
  for (int k = 0; k < 4; k++) crc = (crc << 8) ^ tab[((crc >> 24) ^ (w >> (8 * k))) & 0xFFu];
  return crc;
}

__device__ __forceinline__ void load_tab(unsigned* tab) {
  for (int b = threadIdx.x; b < 256; b += blockDim.x) {
    unsigned r = (unsigned)b << 24;
    for (int k = 0; k < 8; k++) r = (r & 0x80000000u) ? (r << 1) ^ kCrcPoly : (r << 1);
    tab[b] = r;
  }
  __syncthreads();
}

// the site's CRC shifted past the sites after it, XOR-reduced into *acc
__device__ __forceinline__ void crc_combine(unsigned crc, int s, int nsites, bool live, unsigned* acc) {
  unsigned v = 0;
  if (live) {
    unsigned m = (unsigned)(nsites - 1 - s);
    v = crc;
    for (int j = 0; m; j++, m >>= 1)
      if (m & 1u) v = gf_mul(v, c_site_pow[j]);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v ^= __shfl_xor_sync(0xffffffffu, v, off);
  if ((threadIdx.x & 31) == 0 && v) atomicXor(acc, v);
}

struct SliceSite {
  int i, eo;
};
__device__ __forceinline__ SliceSite slice_site(const Geom& g, int s, int t) {
  const int nx = g.L[0], ny = g.L[1], nz = g.L[2];
  const int x = s % nx, r = s / nx, y = r % ny, z = r / ny;
  const long long ilex = x + (long long)nx * (y + (long long)ny * (z + (long long)nz * t));
  return SliceSite{(int)(ilex >> 1), (x + y + z + t) & 1};
}

__global__ void __launch_bounds__(kBlock) k_links_to_file(Geom g, const double2* gauge, int t, uint4* out,
                                                          unsigned* acc) {
  __shared__ unsigned tab[256];
  load_tab(tab);
  const int nsites = g.L[0] * g.L[1] * g.L[2];
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = s < nsites;
  unsigned crc = 0;
  if (live) {
    const SliceSite q = slice_site(g, s, t);
    uint4* o = out + (size_t)s * (kSiteBytes / 16);
#pragma unroll 1
    for (int mu = 0; mu < 4; mu++) {
      const double2* b = gauge + (size_t)((mu * 2 + q.eo) * 9) * g.stride + q.i;
#pragma unroll
      for (int k = 0; k < 6; k++) {  // column k / 3, row k % 3: device slot col*3 + row
        const double2 z = b[(size_t)k * g.stride];
        const uint2 re = be_words(z.x), im = be_words(z.y);
        o[mu * 6 + k] = make_uint4(re.x, re.y, im.x, im.y);
        crc = crc_word(crc, re.x, tab);
        crc = crc_word(crc, re.y, tab);
        crc = crc_word(crc, im.x, tab);
        crc = crc_word(crc, im.y, tab);
      }
    }
  }
  crc_combine(crc, s, nsites, live, acc);
}

__global__ void __launch_bounds__(kBlock) k_links_from_file(Geom g, const uint4* in, int t, double2* gauge,
                                                            unsigned* acc) {
  __shared__ unsigned tab[256];
  load_tab(tab);
  const int nsites = g.L[0] * g.L[1] * g.L[2];
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = s < nsites;
  unsigned crc = 0;
  if (live) {
    const SliceSite q = slice_site(g, s, t);
    const uint4* p = in + (size_t)s * (kSiteBytes / 16);
#pragma unroll 1
    for (int mu = 0; mu < 4; mu++) {
      cx<double> u[3][3];  // [row][col]
#pragma unroll
      for (int k = 0; k < 6; k++) {
        const uint4 w = p[mu * 6 + k];
        crc = crc_word(crc, w.x, tab);
        crc = crc_word(crc, w.y, tab);
        crc = crc_word(crc, w.z, tab);
        crc = crc_word(crc, w.w, tab);
        u[k % 3][k / 3] = mkc(be_double(make_uint2(w.x, w.y)), be_double(make_uint2(w.z, w.w)));
      }
      // u_complete (su3.F90:301-310): the third column from the first two
      u[0][2] = conjg(u[1][0] * u[2][1] - u[2][0] * u[1][1]);
      u[1][2] = conjg(u[2][0] * u[0][1] - u[0][0] * u[2][1]);
      u[2][2] = conjg(u[0][0] * u[1][1] - u[1][0] * u[0][1]);
      double2* b = gauge + (size_t)((mu * 2 + q.eo) * 9) * g.stride + q.i;
#pragma unroll
      for (int c = 0; c < 3; c++)
#pragma unroll
        for (int r = 0; r < 3; r++) b[(size_t)(c * 3 + r) * g.stride] = make_double2(u[r][c].x, u[r][c].y);
    }
  }
  crc_combine(crc, s, nsites, live, acc);
}

// host: x^n mod P for n = 8 * 384 * 2^j, j = 0..31
unsigned host_gf_mul(unsigned a, unsigned b) {
  unsigned r = 0;
  for (int k = 0; k < 32; k++) {
    if (b & 1u) r ^= a;
    b >>= 1;
    a = (a & 0x80000000u) ? (a << 1) ^ kCrcPoly : (a << 1);
  }
  return r;
}

// constant memory is per device: the devices whose table is set
unsigned long long g_pow_ready = 0;

cudaError_t ensure_pow() {
  int dev = 0;
  cudaError_t e0 = cudaGetDevice(&dev);
  if (e0 != cudaSuccess) return e0;
  const unsigned long long bit = 1ull << (dev & 63);
  if (g_pow_ready & bit) return cudaSuccess;
  // x^(8*384) mod P by 3072 multiplications by x (the polynomial 2), then
  // repeated squaring for the powers 2^j of it
  unsigned base = 1u;
  for (int k = 0; k < 8 * kSiteBytes; k++) base = host_gf_mul(base, 2u);
  unsigned pw[32];
  pw[0] = base;
  for (int j = 1; j < 32; j++) pw[j] = host_gf_mul(pw[j - 1], pw[j - 1]);
  cudaError_t e = cudaMemcpyToSymbol(c_site_pow, pw, sizeof(pw));
  if (e == cudaSuccess) g_pow_ready |= bit;
  return e;
}

}  // namespace

cudaError_t launch_links_to_file(const Geom& g, const double2* gauge, int t, void* out, unsigned* acc,
                                 cudaStream_t s) {
  cudaError_t e = ensure_pow();
  if (e != cudaSuccess) return e;
  const int nsites = g.L[0] * g.L[1] * g.L[2];
  k_links_to_file<<<nblocks(nsites), kBlock, 0, s>>>(g, gauge, t, (uint4*)out, acc);
  return cudaGetLastError();
}

cudaError_t launch_links_from_file(const Geom& g, const void* in, int t, double2* gauge, unsigned* acc,
                                   cudaStream_t s) {
  cudaError_t e = ensure_pow();
  if (e != cudaSuccess) return e;
  const int nsites = g.L[0] * g.L[1] * g.L[2];
  k_links_from_file<<<nblocks(nsites), kBlock, 0, s>>>(g, (const uint4*)in, t, gauge, acc);
  return cudaGetLastError();
}

}  // namespace bqcdg
