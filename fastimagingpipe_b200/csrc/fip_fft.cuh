// Shared-memory FFT for lengths G = 3 * M, M = 2^k >= 8 (the grid sides of
// power-of-two images: G = 1.5 N), exponent +i (the reference's
// CUFFT_INVERSE, unnormalised), producing only the N outputs an image needs.
//
// One CTA computes one length-G transform as three interleaved length-M
// transforms Z_s (inputs z[3n + s], s = 0, 1, 2) followed by the radix-3
// recombination X[p] = sum_s e^{+2 pi i s p / G} Z_s[p mod M], evaluated only
// for the requested outputs.  Each length-M transform runs on M / E threads
// that keep E (8 or 16) complex values in registers: radix-E (or smaller for
// the last factor) Stockham passes with table twiddles, exchanging values through
// shared memory padded by one element every 16 (conflict-free 64-bit
// accesses).  The first pass reads its inputs through a caller functor,
// straight from global memory; the recombination writes the outputs through
// another, in natural order.
#pragma once

#include <cuda_runtime.h>

namespace fipfft {

constexpr int kMaxPass = 8;

struct Plan {
  int g;              // transform length G = 3 M
  int m;              // sub-transform length M
  int e;              // complex values per thread (8 or 16)
  int ts;             // threads per sub-transform = M / e
  int nt;             // threads = 3 * ts
  int np;             // passes of the sub-transform
  int r[kMaxPass];    // radices, r[0] first
};

// Padded shared-memory index.
__device__ __forceinline__ int sidx(int i) { return i + (i >> 4); }
// Shared-memory elements for length g.
__host__ __device__ __forceinline__ int smem_elems(int g) { return g + g / 16 + 16; }

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 mul_i(float2 a) { return make_float2(-a.y, a.x); }  // i * a

// In-place DFT of length R with exponent +i: y_m = sum_k x_k e^{+2 pi i k m / R}.
template <int R>
__device__ __forceinline__ void dft(float2* x);

template <>
__device__ __forceinline__ void dft<2>(float2* x) {
  const float2 a = x[0], b = x[1];
  x[0] = cadd(a, b);
  x[1] = csub(a, b);
}

template <>
__device__ __forceinline__ void dft<4>(float2* x) {
  const float2 a = cadd(x[0], x[2]), b = csub(x[0], x[2]);
  const float2 c = cadd(x[1], x[3]), d = mul_i(csub(x[1], x[3]));
  x[0] = cadd(a, c);
  x[2] = csub(a, c);
  x[1] = cadd(b, d);
  x[3] = csub(b, d);
}

template <>
__device__ __forceinline__ void dft<8>(float2* x) {
  float2 e[4] = {x[0], x[2], x[4], x[6]};
  float2 o[4] = {x[1], x[3], x[5], x[7]};
  dft<4>(e);
  dft<4>(o);
  const float h = 0.70710678118654752440f;
  // o_m *= e^{+2 pi i m / 8}
  o[1] = make_float2(h * (o[1].x - o[1].y), h * (o[1].x + o[1].y));
  o[2] = mul_i(o[2]);
  o[3] = make_float2(-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y));
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    x[m] = cadd(e[m], o[m]);
    x[m + 4] = csub(e[m], o[m]);
  }
}

// 16 = 4 x 4: n = n1 + 4 n2, m = 4 m1 + m2.
template <>
__device__ __forceinline__ void dft<16>(float2* x) {
  float2 a[4][4];
#pragma unroll
  for (int n1 = 0; n1 < 4; ++n1) {
    float2 t[4] = {x[n1], x[n1 + 4], x[n1 + 8], x[n1 + 12]};
    dft<4>(t);
#pragma unroll
    for (int m2 = 0; m2 < 4; ++m2) a[n1][m2] = t[m2];
  }
  const float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f;
  const float h = 0.70710678118654752440f;
  // a[n1][m2] *= e^{+2 pi i n1 m2 / 16}
  a[1][1] = cmul(a[1][1], make_float2(c1, s1));
  a[1][2] = cmul(a[1][2], make_float2(h, h));
  a[1][3] = cmul(a[1][3], make_float2(s1, c1));
  a[2][1] = cmul(a[2][1], make_float2(h, h));
  a[2][2] = mul_i(a[2][2]);
  a[2][3] = cmul(a[2][3], make_float2(-h, h));
  a[3][1] = cmul(a[3][1], make_float2(s1, c1));
  a[3][2] = cmul(a[3][2], make_float2(-h, h));
  a[3][3] = cmul(a[3][3], make_float2(-c1, -s1));
#pragma unroll
  for (int m2 = 0; m2 < 4; ++m2) {
    float2 t[4] = {a[0][m2], a[1][m2], a[2][m2], a[3][m2]};
    dft<4>(t);
#pragma unroll
    for (int m1 = 0; m1 < 4; ++m1) x[4 * m1 + m2] = t[m1];
  }
}

template <int R>
__host__ __device__ constexpr int log2c() { return R == 2 ? 1 : R == 4 ? 2 : R == 8 ? 3 : 4; }

// w[k] = W^k for k < R, W = tw[step]: the power-of-two powers come from the
// table (exact to rounding), the rest as products of at most three of them
// (a few ulps), so one butterfly reads log2(R) table entries instead of R - 1.
template <int R>
__device__ __forceinline__ void twiddle_powers(float2 (&w)[R], const float2* __restrict__ tw,
                                               int step) {
  w[1] = __ldg(&tw[step]);
  if (R > 2) w[2] = __ldg(&tw[2 * step]);
  if (R > 4) w[4] = __ldg(&tw[4 * step]);
  if (R > 8) w[8] = __ldg(&tw[8 * step]);
  if (R > 2) w[3] = cmul(w[1], w[2]);
  if (R > 4) {
    w[5] = cmul(w[1], w[4]);
    w[6] = cmul(w[2], w[4]);
    w[7] = cmul(w[3], w[4]);
  }
  if (R > 8) {
#pragma unroll
    for (int k = 9; k < R; ++k) w[k] = cmul(w[k - 8], w[8]);
  }
}

// Radix-R pass on a length-M sub-transform: butterfly j = lt + b * ts,
// inputs at j + k M/R, twiddle e^{+2 pi i (j mod ns) k / (ns R)} read from
// the length-G table (index 3 * ...), outputs at (j/ns) ns R + (j mod ns) +
// m ns (Stockham, self-sorting).  ns and M are powers of two:
// lns = log2 ns, lm = log2 M.
template <int R, int E>
__device__ __forceinline__ void butterflies(float2 (&v)[E], const float2* __restrict__ tw, int lm,
                                            int lns, int lt, int ts) {
#pragma unroll
  for (int b = 0; b < E / R; ++b) {
    float2* x = &v[b * R];
    if (lns > 0) {
      const int j = lt + b * ts;
      const int step = 3 * ((j & ((1 << lns) - 1)) << (lm - lns - log2c<R>()));
      float2 w[R];
      twiddle_powers<R>(w, tw, step);
#pragma unroll
      for (int k = 1; k < R; ++k) x[k] = cmul(x[k], w[k]);
    }
    dft<R>(x);
  }
}

template <int R, int E>
__device__ __forceinline__ void store_smem(const float2 (&v)[E], float2* sm, int lns, int lt,
                                           int ts) {
  const int ns = 1 << lns;
#pragma unroll
  for (int b = 0; b < E / R; ++b) {
    const int j = lt + b * ts;
    const int d = ((j >> lns) << (lns + log2c<R>())) + (j & (ns - 1));
#pragma unroll
    for (int q = 0; q < R; ++q) sm[sidx(d + q * ns)] = v[b * R + q];
  }
}

template <int R, int E>
__device__ __forceinline__ void load_smem(float2 (&v)[E], const float2* sm, int m, int lt,
                                          int ts) {
#pragma unroll
  for (int b = 0; b < E / R; ++b) {
    const int j = lt + b * ts;
#pragma unroll
    for (int k = 0; k < R; ++k) v[b * R + k] = sm[sidx(j + k * (m / R))];
  }
}

// First pass inputs: sub-transform s element i is z[3 i + s].
template <int R, int E, class Load>
__device__ __forceinline__ void first_load(float2 (&v)[E], int m, int s, int lt, int ts,
                                           Load& load) {
#pragma unroll
  for (int b = 0; b < E / R; ++b) {
    const int j = lt + b * ts;
#pragma unroll
    for (int k = 0; k < R; ++k) v[b * R + k] = load(3 * (j + k * (m / R)) + s);
  }
}

// Radix dispatch; radices larger than E never occur (the plan keeps them <= E).
#define FIPFFT_DISPATCH(RADIX, CALL)                              \
  switch (RADIX) {                                                \
    case 2: { constexpr int R_ = 2; CALL; } break;                \
    case 4: { constexpr int R_ = 4; CALL; } break;                \
    case 8: { constexpr int R_ = 8; CALL; } break;                \
    default: { constexpr int R_ = (E >= 16 ? 16 : 8); CALL; } break; \
  }

// Runs one transform.  load(n) returns input element n (0 <= n < G);
// store(o, X) receives output p = (o - nout/2) mod G for o in [0, nout).
// All threads of the CTA must call it; sm holds smem_elems(g) float2.
template <int E, class Load, class Store>
__device__ __forceinline__ void run(const Plan& p, float2* sm, const float2* __restrict__ tw,
                                    int nout, Load& load, Store& store) {
  const int tid = threadIdx.x;
  const int s = tid >= 2 * p.ts ? 2 : (tid >= p.ts ? 1 : 0);
  const int lt = tid - s * p.ts, m = p.m, ts = p.ts;
  float2* sub = sm + s * (m + m / 16);  // sidx(s * m) == s * (m + m / 16) for 16 | m
  int lm = 0;
  while ((1 << lm) < m) ++lm;
  float2 v[E];
  FIPFFT_DISPATCH(p.r[0], (first_load<R_, E>(v, m, s, lt, ts, load)));
  // The loader may read a staging copy in sm; the first pass overwrites it.
  __syncthreads();
  int lns = 0;
  for (int q = 0; q < p.np; ++q) {
    const int r = p.r[q];
    FIPFFT_DISPATCH(r, (butterflies<R_, E>(v, tw, lm, lns, lt, ts)));
    FIPFFT_DISPATCH(r, (store_smem<R_, E>(v, sub, lns, lt, ts)));
    __syncthreads();
    if (q + 1 < p.np) {
      FIPFFT_DISPATCH(p.r[q + 1], (load_smem<R_, E>(v, sub, m, lt, ts)));
      __syncthreads();
    }
    lns += (r == 2 ? 1 : r == 4 ? 2 : r == 8 ? 3 : 4);
  }
  // Radix-3 recombination for the requested outputs.
  const int g = p.g, sub_stride = m + m / 16;
  for (int o = tid; o < nout; o += p.nt) {
    int pp = o - nout / 2;
    if (pp < 0) pp += g;
    const int qq = pp & (m - 1);
    const float2 z0 = sm[sidx(qq)];
    const float2 z1 = sm[sub_stride + sidx(qq)];
    const float2 z2 = sm[2 * sub_stride + sidx(qq)];
    const int p2 = (2 * pp) >= g ? 2 * pp - g : 2 * pp;
    const float2 x = cadd(z0, cadd(cmul(z1, __ldg(&tw[pp])), cmul(z2, __ldg(&tw[p2]))));
    store(o, x);
  }
}

}  // namespace fipfft
