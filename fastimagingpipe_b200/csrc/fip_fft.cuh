// Shared-memory FFT for lengths G = 3 * M, M = 2^k >= 8 (the grid sides of
// power-of-two images: G = 1.5 N), exponent +i (the reference's
// CUFFT_INVERSE, unnormalised), for inputs z[c] supported on a band
// lo <= c <= hi around 0 and the N = 2 M outputs X[p], -M <= p < M, that an
// image keeps.
//
// One CTA computes one length-G transform by decimation in frequency by 3:
// X[3 q + s] = sum_n y_s[n] e^{+2 pi i n q / M} with
// y_s[n] = sum_{c = n mod M} z[c] w^{c s}, w = e^{+2 pi i / G}, so the three
// length-M transforms Y_s need no recombination and the band folds into
// them (a band narrower than M puts at most one input on each n).  Each
// length-M transform runs on M / E threads that keep E (8 or 16) complex
// values in registers: radix-E (or smaller for the last factor) Stockham
// passes with table twiddles, exchanging values through shared memory padded
// by one element every 16 (conflict-free 64-bit accesses).  Twiddle tables:
// tw[k] = w^k for k < G, followed by the half table tw[G + m] = W^m,
// W = e^{+2 pi i / M}, m < M / 2, which is all the passes read.  A thread's
// pass twiddles depend on its lane only, so with 16 values per thread they
// are loaded into registers once per transform (PassTw), beside the band's
// staging loads, so their latency leaves the passes.  The first pass
// reads the band through a caller functor and applies w^{c s}; the last pass
// leaves Y_s in shared memory in natural order, read back per output by
// fetch().
#pragma once

#include <cuda_runtime.h>

namespace fipfft {

// Transform shape chosen on the host; the kernels are instantiated per
// (lm, le), so the passes, radices and index arithmetic are compile-time.
struct Plan {
  int g;   // transform length G = 3 M
  int m;   // sub-transform length M = 2^lm
  int lm;  // log2 M
  int le;  // log2 of the complex values per thread (3 or 4)
  int e;   // values per thread
  int nt;  // threads = 3 M / e
  int split;  // 1: one CTA per sub-transform (grid.y = s), 0: one CTA per transform
  int direct;  // 1: the first pass reads the band from global memory (no staging);
               // 2 (row pass): from a shared-memory band copy, brought in by bulk
               // tensor copies one row pair ahead
};

// Padded shared-memory index.
__device__ __forceinline__ int sidx(int i) { return i + (i >> 4); }
// Distance between the three sub-transform buffers: the padded length plus 6
// elements, so that outputs read across the buffers (fetch) start on
// different banks.
__host__ __device__ constexpr int sub_stride(int m) { return m + m / 16 + 6; }
// Shared memory: two buffers of three sub-transforms (passes alternate
// between them, so a pass's stores never wait for the previous pass's loads);
// the input band is staged in the second (stage_offset), which the first
// pass does not write.
__host__ __device__ constexpr int stage_offset(int g) { return 3 * sub_stride(g / 3); }
__host__ __device__ constexpr int smem_elems(int g) { return 6 * sub_stride(g / 3) + 16; }
// The direct form (no staging) keeps one buffer.
__host__ __device__ constexpr int direct_smem_elems(int g) { return 3 * sub_stride(g / 3) + 16; }
// Entries of the passes' half table (M / 2), stored after the G entries.
__host__ __device__ constexpr int half_table_elems(int g) { return g / 6; }

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

// w[k] = W^k for k < R from the power-of-two powers p[l] = W^{2^l}
// (table entries, exact to rounding): the rest as products of at most three
// of them (a few ulps), so one butterfly reads log2(R) table entries instead
// of R - 1.
template <int R>
__device__ __forceinline__ void twiddle_powers(float2 (&w)[R], const float2* p) {
  w[1] = p[0];
  if (R > 2) w[2] = p[1];
  if (R > 4) w[4] = p[2];
  if (R > 8) w[8] = p[3];
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

// Pass-twiddle step of butterfly j in a pass of radix 2^lr after ns = 2^lns
// outputs: its twiddles are W^{step 2^l}, l < lr, with (R / 2) step < M / 2.
__device__ __forceinline__ int pass_step(int j, int lm, int lns, int lr) {
  return (j & ((1 << lns) - 1)) << (lm - lns - lr);
}

// Radix-R pass on a length-M sub-transform: butterfly j = lt + b * ts,
// inputs at j + k M/R, twiddle e^{+2 pi i (j mod ns) k / (ns R)} = W^{step k}
// (pass_step; p[b * log2 R + l] = W^{step 2^l}; none in the first pass,
// ns = 1), outputs at (j/ns) ns R + (j mod ns) + m ns (Stockham,
// self-sorting).
template <int R, int E, bool TWIDDLED>
__device__ __forceinline__ void butterflies(float2 (&v)[E], const float2* p) {
#pragma unroll
  for (int b = 0; b < E / R; ++b) {
    float2* x = &v[b * R];
    if constexpr (TWIDDLED) {
      float2 w[R];
      twiddle_powers<R>(w, p + b * log2c<R>());
#pragma unroll
      for (int k = 1; k < R; ++k) x[k] = cmul(x[k], w[k]);
    }
    dft<R>(x);
  }
}

// Stockham store of pass outputs: butterfly j's output q goes to
// d + q ns, d = (j / ns) ns R + (j mod ns).  When ns is a multiple of 16 the
// padded index of d + q ns is sidx(d) + q ns 17/16 (no per-element shift).
template <int R, int E, int LNS>
__device__ __forceinline__ void store_smem(const float2 (&v)[E], float2* sm, int lt, int ts) {
  constexpr int ns = 1 << LNS;
#pragma unroll
  for (int b = 0; b < E / R; ++b) {
    const int j = lt + b * ts;
    const int d = ((j >> LNS) << (LNS + log2c<R>())) + (j & (ns - 1));
    if constexpr (ns % 16 == 0) {
      float2* base = sm + sidx(d);
#pragma unroll
      for (int q = 0; q < R; ++q) base[q * (ns + ns / 16)] = v[b * R + q];
    } else {
#pragma unroll
      for (int q = 0; q < R; ++q) sm[sidx(d + q * ns)] = v[b * R + q];
    }
  }
}

// Loads of the next pass: butterfly j reads j + k M/R (M/R >= 16, so the
// padded index is sidx(j) + k (M/R) 17/16).
template <int R, int E, int M>
__device__ __forceinline__ void load_smem(float2 (&v)[E], const float2* sm, int lt, int ts) {
  constexpr int step = M / R;
#pragma unroll
  for (int b = 0; b < E / R; ++b) {
    const int j = lt + b * ts;
    if constexpr (step % 16 == 0) {
      const float2* base = sm + sidx(j);
#pragma unroll
      for (int k = 0; k < R; ++k) v[b * R + k] = base[k * (step + step / 16)];
    } else {
#pragma unroll
      for (int k = 0; k < R; ++k) v[b * R + k] = sm[sidx(j + k * step)];
    }
  }
}

// First-pass inputs of sub-transform s: element n is
// y_s[n] = sum_{c = n + t M, lo <= c <= hi} z[c] w^{c s}.  WIDE: the band may
// reach past +-M (t in -2..1); otherwise only t = -1, 0 can hit.  The thread's
// elements are n = j + k M/R, so w^{c s} = w^{j s} w^{k s M/R} w^{t M s}: one
// table read per butterfly (w^{j s}), R reads shared by every lane
// (w^{k s M/R}) and the cube roots of unity w^{t M s} = e^{2 pi i t s / 3};
// the first pass touches a few hundred table entries instead of the band's
// thousands.
template <int R, int E, int M, bool WIDE, class Load>
__device__ __forceinline__ void first_load(float2 (&v)[E], int s, int lt, int lo, int hi,
                                           const float2* __restrict__ tw, Load& load) {
  constexpr int TS = M / E;
  const float h3 = 0.86602540378443864676f;  // sqrt(3) / 2
#pragma unroll
  for (int b = 0; b < E / R; ++b) {
    const int j = lt + b * TS;
    const float2 wj = s ? __ldg(&tw[j * s]) : make_float2(1.f, 0.f);
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const int n = j + k * (M / R);
      float2 wn = wj;
      if (s != 0 && k != 0) wn = cmul(wj, __ldg(&tw[k * s * (M / R)]));
      float2 acc = make_float2(0.f, 0.f);
#pragma unroll
      for (int t = (WIDE ? -2 : -1); t <= (WIDE ? 1 : 0); ++t) {
        const int c = n + t * M;
        if (c >= lo && c <= hi) {
          float2 z = load(c);
          if (s != 0) {
            float2 w = wn;
            const int m = ((t * s) % 3 + 3) % 3;  // w^{t M s} = e^{2 pi i m / 3}
            if (m == 1) w = cmul(wn, make_float2(-0.5f, h3));
            if (m == 2) w = cmul(wn, make_float2(-0.5f, -h3));
            z = cmul(z, w);
          }
          acc = cadd(acc, z);
        }
      }
      v[b * R + k] = acc;
    }
  }
}

// log2 of the radix of pass q: LE for the full passes, the remainder last.
template <int LM, int LE>
__host__ __device__ constexpr int pass_lr(int q) {
  return q < LM / LE ? LE : LM % LE;
}
template <int LM, int LE>
__host__ __device__ constexpr int pass_count() {
  return (LM + LE - 1) / LE;
}
// Table entries a thread reads in passes 1 .. Q - 1 ((E / R) butterflies of
// log2 R entries each; pass 0 has no twiddles).
template <int LM, int LE>
__host__ __device__ constexpr int pass_tw_offset(int Q) {
  int n = 0;
  for (int q = 1; q < Q; ++q) n += ((1 << LE) >> pass_lr<LM, LE>(q)) * pass_lr<LM, LE>(q);
  return n;
}

// A thread's pass twiddles.  With 16 values per thread they are loaded up
// front (load()) into registers; with 8 (launches of up to 768 threads,
// tighter register budgets) each pass loads its own from the table.
template <int LM, int LE>
struct PassTw {
  static constexpr bool kAhead = LE == 4;
  static constexpr int kCount = pass_tw_offset<LM, LE>(pass_count<LM, LE>());
  float2 w[kAhead && kCount > 0 ? kCount : 1];
  const float2* half;  // the half table (global memory)
  int lt;              // thread index within its sub-transform

  __device__ __forceinline__ void load(const float2* __restrict__ tw_half, int lane) {
    half = tw_half;
    lt = lane;
    if constexpr (kAhead) fill<1>();
  }
  template <int Q>
  __device__ __forceinline__ void fill() {
    if constexpr (Q < pass_count<LM, LE>()) {
      constexpr int L = pass_lr<LM, LE>(Q), E = 1 << LE, TS = (1 << LM) / E;
#pragma unroll
      for (int b = 0; b < (E >> L); ++b) {
        const int step = pass_step(lt + b * TS, LM, Q * LE, L);
#pragma unroll
        for (int l = 0; l < L; ++l)
          w[pass_tw_offset<LM, LE>(Q) + b * L + l] = __ldg(&half[step << l]);
      }
      fill<Q + 1>();
    }
  }
  // Pass Q's entries (log2 R per butterfly) into p.
  template <int Q, int N>
  __device__ __forceinline__ void get(float2 (&p)[N]) const {
    constexpr int L = pass_lr<LM, LE>(Q), E = 1 << LE, TS = (1 << LM) / E;
    static_assert(N == (E >> L) * L, "one pass's entries");
    if constexpr (kAhead) {
#pragma unroll
      for (int k = 0; k < N; ++k) p[k] = w[pass_tw_offset<LM, LE>(Q) + k];
    } else {
#pragma unroll
      for (int b = 0; b < (E >> L); ++b) {
        const int step = pass_step(lt + b * TS, LM, Q * LE, L);
#pragma unroll
        for (int l = 0; l < L; ++l) p[b * L + l] = __ldg(&half[step << l]);
      }
    }
  }
};

// Thread index within its sub-transform of the joint forms (3 M / E threads).
template <int LM, int LE>
__device__ __forceinline__ int sub_lane(int tid) {
  constexpr int TS = (1 << LM) >> LE;
  return tid >= 2 * TS ? tid - 2 * TS : (tid >= TS ? tid - TS : tid);
}

// Pass Q of the Stockham transform: butterflies, stores into buffer Q & 1
// (base + (Q & 1) * BUF), and the loads of pass Q + 1 from it.
// GROUP: the barriers between passes hold only the sub-transform's own
// threads (named barrier 1 + s; the group is a whole number of warps), the
// last pass ends with a CTA barrier.  Only valid when nothing else lives in
// the buffers (no staged band).
template <int LM, int LE, int Q, int BUF, bool GROUP = false>
__device__ __forceinline__ void passes(float2 (&v)[1 << LE], float2* base,
                                       const PassTw<LM, LE>& pt, int lt, int s = 0) {
  constexpr int E = 1 << LE, M = 1 << LM, TS = M / E, NP = pass_count<LM, LE>();
  if constexpr (Q < NP) {
    constexpr int LNS = Q * LE, R = 1 << pass_lr<LM, LE>(Q);
    float2* sub = base + (Q & 1) * BUF;
    if constexpr (Q > 0) {
      float2 p[(E / R) * log2c<R>()];
      pt.template get<Q>(p);
      butterflies<R, E, true>(v, p);
    } else {
      butterflies<R, E, false>(v, nullptr);
    }
    store_smem<R, E, LNS>(v, sub, lt, TS);
    if constexpr (GROUP && Q + 1 < NP && TS % 32 == 0) {
      if (s == 0)
        asm volatile("bar.sync 1, %0;" ::"n"(TS) : "memory");
      else if (s == 1)
        asm volatile("bar.sync 2, %0;" ::"n"(TS) : "memory");
      else
        asm volatile("bar.sync 3, %0;" ::"n"(TS) : "memory");
    } else {
      __syncthreads();
    }
    if constexpr (Q + 1 < NP) {
      load_smem<(1 << pass_lr<LM, LE>(Q + 1)), E, M>(v, sub, lt, TS);
      if constexpr (BUF == 0) {  // one buffer: the next stores wait for these loads
        if constexpr (GROUP && TS % 32 == 0) {
          if (s == 0)
            asm volatile("bar.sync 1, %0;" ::"n"(TS) : "memory");
          else if (s == 1)
            asm volatile("bar.sync 2, %0;" ::"n"(TS) : "memory");
          else
            asm volatile("bar.sync 3, %0;" ::"n"(TS) : "memory");
        } else {
          __syncthreads();
        }
      }
      passes<LM, LE, Q + 1, BUF, GROUP>(v, base, pt, lt, s);
    }
  }
}

// Computes Y_s for s = 0, 1, 2 into sm (natural order; see fetch), M = 2^LM,
// E = 2^LE values per thread, 3 M / E threads.  load(c) returns z[c] for
// lo <= c <= hi (-G/2 < lo <= 0 <= hi <= G/2); it may read a staging copy at
// sm + stage_offset(G) (written before a barrier).  All threads of the CTA
// must call it; sm holds smem_elems(G) float2.  Ends with a barrier: sm is
// then ready for fetch().
// DIRECT: load() reads global memory (no staged band), so the passes may
// use group barriers, and one buffer (sm holds direct_smem_elems(G)) serves
// all passes.  pt: the thread's pass twiddles (loaded for lane
// sub_lane(threadIdx.x)).
// loaded(): called by every thread once its band values are in registers
// (before the first pass's stores), e.g. to release a staging buffer.
struct NoHook {
  __device__ void operator()() const {}
};
template <int LM, int LE, bool DIRECT = false, class Load, class Loaded = NoHook>
__device__ __forceinline__ void run(float2* sm, const float2* __restrict__ tw,
                                    const PassTw<LM, LE>& pt, int lo, int hi, Load& load,
                                    const Loaded& loaded = Loaded{}) {
  constexpr int E = 1 << LE, M = 1 << LM, TS = M / E;
  constexpr int R0 = 1 << pass_lr<LM, LE>(0);
  const int tid = threadIdx.x;
  const int s = tid >= 2 * TS ? 2 : (tid >= TS ? 1 : 0);
  const int lt = tid - s * TS;
  float2 v[E];
  if (hi >= M || lo < -M)
    first_load<R0, E, M, true>(v, s, lt, lo, hi, tw, load);
  else
    first_load<R0, E, M, false>(v, s, lt, lo, hi, tw, load);
  loaded();
  passes<LM, LE, 0, DIRECT ? 0 : stage_offset(3 * M), DIRECT>(v, sm + s * sub_stride(M), pt,
                                                                 lt, s);
}

// Pre-twiddled staging, for bands no wider than M (each n then receives one
// c at most): the staging loop writes y_s[n] = z[c] w^{c s} (n = c mod M) for
// s = 0, 1, 2 at pre + s * sub_stride(M) + sidx(n), pre = sm + stage_offset(G),
// and zeros where no c lands (zero_pre); the first pass is then a plain
// shared-memory read.
template <int M>
__device__ __forceinline__ void stage_pre(float2* pre, int c, float2 z, float2 w1, float2 w2) {
  const int nn = c < 0 ? c + M : c;
  pre[sidx(nn)] = z;
  pre[sub_stride(M) + sidx(nn)] = cmul(z, w1);
  pre[2 * sub_stride(M) + sidx(nn)] = cmul(z, w2);
}

// w^c and w^{2 c} for c = c0, c0 + d, c0 + 2 d, ... (a staging loop's
// sequence): two table reads at the start, then one product per step with
// w^d and w^{2 d} (the error grows by about an ulp per step; a staging loop
// takes at most G / (2 d) steps).
struct StageTw {
  float2 w1, w2, d1, d2;
  __device__ __forceinline__ StageTw(const float2* __restrict__ tw, int g, int c0, int d) {
    const int a = c0 < 0 ? c0 + g : c0;
    int b = 2 * c0;
    b = b < 0 ? b + g : (b >= g ? b - g : b);
    w1 = __ldg(&tw[a]);
    w2 = __ldg(&tw[b]);
    d1 = __ldg(&tw[d]);
    d2 = __ldg(&tw[2 * d]);
  }
  __device__ __forceinline__ void next() {
    w1 = cmul(w1, d1);
    w2 = cmul(w2, d2);
  }
};
template <int M>
__device__ __forceinline__ void zero_pre(float2* pre, int lo, int hi, int tid, int nt) {
  for (int nn = hi + 1 + tid; nn < M + lo; nn += nt) {
    pre[sidx(nn)] = make_float2(0.f, 0.f);
    pre[sub_stride(M) + sidx(nn)] = make_float2(0.f, 0.f);
    pre[2 * sub_stride(M) + sidx(nn)] = make_float2(0.f, 0.f);
  }
}

template <int LM, int LE>
__device__ __forceinline__ void run_pre(float2* sm, const PassTw<LM, LE>& pt) {
  constexpr int E = 1 << LE, M = 1 << LM, TS = M / E;
  constexpr int R0 = 1 << pass_lr<LM, LE>(0);
  const int tid = threadIdx.x;
  const int s = tid >= 2 * TS ? 2 : (tid >= TS ? 1 : 0);
  const int lt = tid - s * TS;
  const float2* pre = sm + stage_offset(3 * M) + s * sub_stride(M);
  float2 v[E];
#pragma unroll
  for (int b = 0; b < E / R0; ++b) {
    const int j = lt + b * TS;
#pragma unroll
    for (int k = 0; k < R0; ++k) v[b * R0 + k] = pre[sidx(j + k * (M / R0))];
  }
  passes<LM, LE, 0, stage_offset(3 * M), false>(v, sm + s * sub_stride(M), pt, lt, s);
}

// Output o in [0, 2M) after run(): X[p] with p = o - M, i.e. Y_s[q] for
// (p mod G) = 3 q + s, in the buffer of the last pass.
template <int LM, int LE, bool DIRECT = false>
__device__ __forceinline__ float2 fetch(const float2* sm, int o) {
  constexpr int M = 1 << LM;
  constexpr int last = DIRECT ? 0 : (pass_count<LM, LE>() - 1) & 1;
  int pp = o - M;
  if (pp < 0) pp += 3 * M;
  const int q = pp / 3, s = pp - 3 * q;
  return sm[last * stage_offset(3 * M) + s * sub_stride(M) + sidx(q)];
}

// Outputs o, o + 1, ..., o + K - 1 (o a multiple of K, K | M) after run():
// one division by 3 for the group, then (q, s) steps through the
// interleaved sub-transforms.
template <int LM, int LE, int K, bool DIRECT = false>
__device__ __forceinline__ void fetch_run(const float2* sm, int o, float2 (&out)[K]) {
  constexpr int M = 1 << LM;
  constexpr int last = DIRECT ? 0 : (pass_count<LM, LE>() - 1) & 1;
  const float2* buf = sm + last * stage_offset(3 * M);
  int pp = o - M;
  if (pp < 0) pp += 3 * M;  // the K outputs do not straddle o = M (K | M)
  int q = pp / 3, s = pp - 3 * q;
#pragma unroll
  for (int e = 0; e < K; ++e) {
    out[e] = buf[s * sub_stride(M) + sidx(q)];
    if (++s == 3) {
      s = 0;
      ++q;
    }
  }
}

// Split form: one CTA of M / E threads computes the single sub-transform
// Y_s (s given) into two buffers of sub_stride(M) elements at sm (staging, if
// any, is read by load() before the first barrier and may sit in the second
// buffer).  Ends with a barrier; Y_s[q] is then at single_out<LM, LE>(sm, q).
template <int LM, int LE, class Load>
__device__ __forceinline__ void run_single(float2* sm, int s, const float2* __restrict__ tw,
                                           const PassTw<LM, LE>& pt, int lo, int hi, Load& load) {
  constexpr int E = 1 << LE, M = 1 << LM;
  constexpr int R0 = 1 << pass_lr<LM, LE>(0);
  float2 v[E];
  if (hi >= M || lo < -M)
    first_load<R0, E, M, true>(v, s, threadIdx.x, lo, hi, tw, load);
  else
    first_load<R0, E, M, false>(v, s, threadIdx.x, lo, hi, tw, load);
  // The first pass writes buffer 0 while the staging in buffer 1 is still
  // being read by other threads: passes' barriers come after each store, so
  // buffer 1 is only written (pass 1) after every thread passed barrier 0.
  passes<LM, LE, 0, sub_stride(M)>(v, sm, pt, threadIdx.x);
}

template <int LM, int LE>
__device__ __forceinline__ float2 single_out(const float2* sm, int q) {
  constexpr int M = 1 << LM;
  constexpr int last = (pass_count<LM, LE>() - 1) & 1;
  return sm[last * sub_stride(M) + sidx(q)];
}

}  // namespace fipfft
