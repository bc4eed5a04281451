// blockcg.cu -- the block kernels of the block conjugate-gradient solver
// (capi_block.cu): Gram matrices A^H B of two blocks of s FP32 spinor fields
// and linear combinations of blocks, out = in1 M1 + in2 M2 with small s x s
// complex matrices.  A block is s fields of the batched layout (field j at
// j * rsb bytes), each float4 [6][stride] (two complex numbers per float4).
#include "kernels.cuh"

namespace bqcdg {

constexpr int kGramThreads = 256;  // 16 x 16 pairs (i, j)
constexpr int kGramSites = 8;      // sites per shared-memory tile (2 x 12 KB at S = 16)
constexpr int kGramBlocks = 592;   // 4 per SM of a B200

// partial[cta][i * S + j] = sum over the CTA's sites of <A_i, B_j> (FP64);
// the tiles keep the 12 complex components of 8 sites of every column in
// shared memory ([site][component][column], so a warp's 16 j read 16
// consecutive words), and thread (i, j) sums its pair over the tile in FP32
// before adding the tile to its FP64 total
template <int S>
__global__ void __launch_bounds__(kGramThreads) k_block_gram(Geom g, const float4* A, long long ars, const float4* B,
                                                             long long brs, double2* partial) {
  __shared__ float2 ta[kGramSites][12][S];
  __shared__ float2 tb[kGramSites][12][S];
  const int t = threadIdx.x;
  const int pi = t / 16, pj = t % 16;
  const bool mine = pi < S && pj < S;
  double sre = 0.0, sim = 0.0;
  const int ntiles = (g.volh + kGramSites - 1) / kGramSites;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int i0 = tile * kGramSites;
    // load: (column, float4 w, site) triples, 6 float4 per site and column
    for (int e = t; e < S * 6 * kGramSites; e += kGramThreads) {
      const int s = e % kGramSites, w = (e / kGramSites) % 6, col = e / (kGramSites * 6);
      const int i = i0 + s;
      float4 va = make_float4(0.f, 0.f, 0.f, 0.f), vb = va;
      if (i < g.volh) {
        va = A[col * ars + (long long)w * g.stride + i];
        vb = B[col * brs + (long long)w * g.stride + i];
      }
      ta[s][2 * w][col] = make_float2(va.x, va.y);
      ta[s][2 * w + 1][col] = make_float2(va.z, va.w);
      tb[s][2 * w][col] = make_float2(vb.x, vb.y);
      tb[s][2 * w + 1][col] = make_float2(vb.z, vb.w);
    }
    __syncthreads();
    if (mine) {
      float re = 0.f, im = 0.f;
#pragma unroll 4
      for (int s = 0; s < kGramSites; s++)
#pragma unroll
        for (int c = 0; c < 12; c++) {
          const float2 a = ta[s][c][pi], b = tb[s][c][pj];
          re = fmaf(a.x, b.x, fmaf(a.y, b.y, re));    // conj(a) b
          im = fmaf(a.x, b.y, fmaf(-a.y, b.x, im));
        }
      sre += re;
      sim += im;
    }
    __syncthreads();
  }
  if (mine) partial[(size_t)blockIdx.x * S * S + pi * S + pj] = make_double2(sre, sim);
}

// out[p] = sum over the CTAs in order of partial[cta][p]
__global__ void k_block_gram_sum(const double2* partial, int ncta, int npair, double2* out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npair) return;
  double re = 0.0, im = 0.0;
  for (int b = 0; b < ncta; b++) {
    const double2 v = partial[(size_t)b * npair + p];
    re += v.x;
    im += v.y;
  }
  out[p] = make_double2(re, im);
}

// out_j = sum_k in1_k M1[k][j] (+ sum_k in2_k M2[k][j]); one thread per
// (site, float4 w), all S columns of it, so out may be in1 or in2
template <int S, bool TWO>
__global__ void __launch_bounds__(128) k_block_combine(Geom g, float4* out, long long ors, const float4* in1,
                                                       long long rs1, const float2* M1, const float4* in2,
                                                       long long rs2, const float2* M2) {
  __shared__ float2 m1[S * S], m2[TWO ? S * S : 1];
  for (int e = threadIdx.x; e < S * S; e += blockDim.x) {
    m1[e] = M1[e];
    if (TWO) m2[e] = M2[e];
  }
  __syncthreads();
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = idx % g.volh, w = idx / g.volh;
  if (w >= 6) return;
  float2 acc0[S], acc1[S];
#pragma unroll
  for (int j = 0; j < S; j++) acc0[j] = acc1[j] = make_float2(0.f, 0.f);
#pragma unroll
  for (int src = 0; src < (TWO ? 2 : 1); src++) {
    const float4* in = src == 0 ? in1 : in2;
    const long long rs = src == 0 ? rs1 : rs2;
    const float2* m = src == 0 ? m1 : m2;
#pragma unroll
    for (int k = 0; k < S; k++) {
      const float4 v = in[k * rs + (long long)w * g.stride + i];
#pragma unroll
      for (int j = 0; j < S; j++) {
        const float2 c = m[k * S + j];
        acc0[j].x = fmaf(v.x, c.x, fmaf(-v.y, c.y, acc0[j].x));
        acc0[j].y = fmaf(v.x, c.y, fmaf(v.y, c.x, acc0[j].y));
        acc1[j].x = fmaf(v.z, c.x, fmaf(-v.w, c.y, acc1[j].x));
        acc1[j].y = fmaf(v.z, c.y, fmaf(v.w, c.x, acc1[j].y));
      }
    }
  }
#pragma unroll
  for (int j = 0; j < S; j++) out[j * ors + (long long)w * g.stride + i] = make_float4(acc0[j].x, acc0[j].y, acc1[j].x, acc1[j].y);
}

// float4 element strides of a batched field pointer
static long long f4rs(const SpinorPtr& p) { return p.rsb / (long long)sizeof(float4); }

template <int S>
static void gram_s(const Geom& g, SpinorPtr a, SpinorPtr b, double2* partial, double2* out, cudaStream_t st) {
  k_block_gram<S><<<kGramBlocks, kGramThreads, 0, st>>>(g, (const float4*)a.v, f4rs(a), (const float4*)b.v, f4rs(b),
                                                       partial);
  k_block_gram_sum<<<(S * S + 127) / 128, 128, 0, st>>>(partial, kGramBlocks, S * S, out);
}
template <int S>
static void combine_s(const Geom& g, SpinorPtr out, SpinorPtr in1, const float2* m1, SpinorPtr in2, const float2* m2,
                      cudaStream_t st) {
  const long long n = 6LL * g.volh;
  const int nb = (int)((n + 127) / 128);
  if (in2.v)
    k_block_combine<S, true><<<nb, 128, 0, st>>>(g, (float4*)out.v, f4rs(out), (const float4*)in1.v, f4rs(in1), m1,
                                                 (const float4*)in2.v, f4rs(in2), m2);
  else
    k_block_combine<S, false><<<nb, 128, 0, st>>>(g, (float4*)out.v, f4rs(out), (const float4*)in1.v, f4rs(in1), m1,
                                                  nullptr, 0, nullptr);
}

int block_gram_scratch_pairs() { return kGramBlocks * 16 * 16; }

#define BQCDG_BLOCK_SWITCH(S, CALL) \
  switch (S) {                      \
    case 1: CALL(1); break;         \
    case 2: CALL(2); break;         \
    case 3: CALL(3); break;         \
    case 4: CALL(4); break;         \
    case 5: CALL(5); break;         \
    case 6: CALL(6); break;         \
    case 7: CALL(7); break;         \
    case 8: CALL(8); break;         \
    case 9: CALL(9); break;         \
    case 10: CALL(10); break;       \
    case 11: CALL(11); break;       \
    case 12: CALL(12); break;       \
    case 13: CALL(13); break;       \
    case 14: CALL(14); break;       \
    case 15: CALL(15); break;       \
    default: CALL(16); break;       \
  }

void launch_block_gram(const Geom& g, int s, SpinorPtr a, SpinorPtr b, double2* partial, double2* out,
                       cudaStream_t st) {
#define GRAM(N) gram_s<N>(g, a, b, partial, out, st)
  BQCDG_BLOCK_SWITCH(s, GRAM)
#undef GRAM
}

void launch_block_combine(const Geom& g, int s, SpinorPtr out, SpinorPtr in1, const float2* m1, SpinorPtr in2,
                          const float2* m2, cudaStream_t st) {
#define COMB(N) combine_s<N>(g, out, in1, m1, in2, m2, st)
  BQCDG_BLOCK_SWITCH(s, COMB)
#undef COMB
}

}  // namespace bqcdg
