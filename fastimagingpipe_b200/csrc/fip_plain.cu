// Device stages of the snapshot imaging + tLISI trigger path.
//
// This translation unit is compiled with --use_fast_math, the flags of the
// reference's CUDA build (reference Makefile:13), because the plain FP32 form
// reproduces the reference's FP32 arithmetic (fip_refmath.cuh).  Data
// movement is B200-native:
//   * gridding bins every visibility by 64x64 tile of the Hermitian half-plane
//     uv grid; a thread per visibility of a work item takes its footprint
//     and kernel values into registers and adds its in-tile taps into the
//     tile in shared memory (int32 fixed point), which is committed once
//     (plain stores for tiles owned by one work item, vector reductions for
//     the few dense tiles split over several); only tiles inside the
//     occupied uv band are written;
//   * the 2-D inverse FFT is band-pruned: column transforms run only over the
//     occupied half-plane columns and keep only the N needed outputs; row
//     transforms pack two real image rows into one complex transform and
//     apply the grid correction in their epilogue (fip_fft.cuh);
//   * the reference's pixel mapping (compute-bound) runs on a side stream
//     while gridding and the FFT run, and reprojection is destination-tile
//     major: each 64x64 output tile gathers its candidate source pixels,
//     splats them in shared memory, stores the tile once and reports its
//     maximum -- no global atomics, no memsets;
//   * the trigger reads the three images once, in 128-bit loads, with
//     warp-shuffle tile reductions; a batch's sliding window streams each
//     tile's slices through registers, every image read once for all the
//     triples it is in.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>

#include "fip_common.cuh"
#include "fip_fft.cuh"
#include "fip_kernels.h"
#include "fip_refmath.cuh"

namespace {

constexpr int kThreads = 256;

// Grid row of signed row index v in [-G, G): v mod G without a division.
__device__ __forceinline__ int wrap_row(int v, int g) { return v < 0 ? v + g : (v >= g ? v - g : v); }

// ---------------------------------------------------------------------------
// Taper (FIPkernels.cu:173-186)
// ---------------------------------------------------------------------------
// taper[t] for t <= N/2, then the reciprocal correction
// taper[N/2 + 1 + t] = 1 / (taper[t] norm) that the row transform applies.
__global__ void k_taper(float* taper, size_t n, size_t g) {
  size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t < n / 2 + 1) {
    const float c = fipref::taper(t, g);
    taper[t] = c;
    taper[n / 2 + 1 + t] = (float)(1.0 / ((double)c * (double)FIP_CONV_NORM));
  }
}

// ---------------------------------------------------------------------------
// Visibility footprint (FIPkernels.cu:211-219): taps [a0,a1] x [b0,b1],
// clamped to the grid.  Returns false when empty.
// ---------------------------------------------------------------------------
struct Footprint {
  float p1, p2;
  int a0, a1, b0, b1;
};

__device__ __forceinline__ bool footprint(const float* B, int v, float scale, int g, Footprint& f) {
  const int hs = FIP_SUPPORT / 2;
  const long gmin = -(long)g / 2, gmax = ((long)g - 1) / 2;
  f.p1 = B[2 * v + 0] * scale;
  f.p2 = B[2 * v + 1] * scale;
  long a0 = max(fipref::ceil_l(f.p1 - hs), gmin), a1 = min(fipref::floor_l(f.p1 + hs), gmax);
  long b0 = max(fipref::ceil_l(f.p2 - hs), gmin), b1 = min(fipref::floor_l(f.p2 + hs), gmax);
  f.a0 = (int)a0; f.a1 = (int)a1; f.b0 = (int)b0; f.b1 = (int)b1;
  return !(a0 > a1 || b0 > b1);
}

// Half-plane image of a virtual visibility.  The grid holds the Hermitian
// part h(r) = (g(r) + conj g(-r)) / 2 of the reference's grid g, whose real
// transform is the real part the reference keeps (FIPkernels.cu:266): the
// direct copy keeps taps with r2 >= 0 at (r1 mod G, r2), the mirrored copy
// (conjugated) keeps taps with r2 <= 0 at (-r1 mod G, -r2).  Columns are
// taken modulo G, so for even G a tap at r2 = -G/2 (the reference's first
// grid column, FIPkernels.cu:202) lies on the Nyquist column G/2 of the
// direct copy as well as of the mirrored one; a footprint spans 9 columns at
// most, so for G > 18 that column is then the direct copy's only one.
__device__ __forceinline__ bool half_cols(const Footprint& f, int mir, int g, int& c0, int& c1) {
  if (!mir) {
    if (f.b1 < 0) {
      if ((g & 1) == 0 && f.b0 == -(g / 2)) {
        c0 = c1 = g / 2;
        return true;
      }
      return false;
    }
    c0 = max(f.b0, 0); c1 = f.b1;
  } else {
    if (f.b0 > 0) return false;
    c0 = max(-f.b1, 0); c1 = -f.b0;
  }
  return true;
}

// Distinct tile rows touched by rows r1 in [a0,a1] (direct) or -r1
// (mirrored), modulo G.  At most 3.
__device__ __forceinline__ int tile_rows(const Footprint& f, int mir, int g, int* out) {
  // Signed row range [lo, hi] (<= 9 rows) wraps into at most two segments.
  const int lo = mir ? -f.a1 : f.a0, hi = mir ? -f.a0 : f.a1;
  int n = 0;
  auto add_segment = [&](int a, int b) {  // rows a..b within [0, g)
    for (int tr = a / FIP_GTILE; tr <= b / FIP_GTILE && n < 3; ++tr) {
      bool seen = false;
      for (int k = 0; k < n; ++k) seen |= (out[k] == tr);
      if (!seen) out[n++] = tr;
    }
  };
  if (lo < 0 && hi >= 0) {
    add_segment(lo + g, g - 1);
    add_segment(0, hi);
  } else if (hi >= g) {
    add_segment(lo, g - 1);
    add_segment(0, hi - g);
  } else {
    add_segment(wrap_row(lo, g), wrap_row(hi, g));
  }
  return n;
}

// Warp-aggregated increment of cnt[key]; returns this lane's slot.
__device__ __forceinline__ unsigned agg_inc(unsigned* cnt, unsigned key, unsigned active) {
  unsigned peers = __match_any_sync(active, key);
  int leader = __ffs(peers) - 1;
  unsigned rank = __popc(peers & ((1u << (threadIdx.x & 31)) - 1));
  unsigned base = 0;
  if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(&cnt[key], (unsigned)__popc(peers));
  base = __shfl_sync(peers, base, leader);
  return base + rank;
}

// pass 0: count entries per tile and record the occupied band
// (bbox[0] = max |r1|, bbox[1] = max half-plane column); pass 1: scatter.
template <int PASS>
__global__ void k_bin(const float* __restrict__ B, int nb, float scale, int g, int tiles_c,
                      unsigned* cnt, const unsigned* __restrict__ offset, unsigned* entries,
                      unsigned* bbox) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  Footprint f;
  bool ok = v < nb && footprint(B, v, scale, g, f);
  unsigned k1 = 0, k2 = 0;
  if (ok) k1 = (unsigned)max(abs(f.a0), abs(f.a1));
  for (int mir = 0; mir < 2; ++mir) {
    int c0 = 0, c1 = -1, trs[3], ntr = 0;
    bool on = ok && half_cols(f, mir, g, c0, c1);
    if (on) {
      ntr = tile_rows(f, mir, g, trs);
      k2 = max(k2, (unsigned)c1);
    }
    int tc0 = on ? c0 / FIP_GTILE : 0, tc1 = on ? c1 / FIP_GTILE : -1;
    // Up to 3 x 2 (tile-row, tile-col) pairs; every lane walks the same
    // 6 slots so the warp-aggregated atomics stay converged.
    for (int s = 0; s < 6; ++s) {
      int kr = s >> 1, kc = s & 1;
      bool act = on && kr < ntr && tc0 + kc <= tc1;
      unsigned mask = __ballot_sync(0xffffffffu, act);
      if (act) {
        unsigned tile = (unsigned)(trs[kr] * tiles_c + tc0 + kc);
        unsigned slot = agg_inc(cnt, tile, mask);
        if (PASS == 1) entries[offset[tile] + slot] = ((unsigned)v << 1) | (unsigned)mir;
      }
    }
  }
  if (PASS == 0) {
    for (int o = 16; o > 0; o >>= 1) {
      k1 = max(k1, __shfl_xor_sync(0xffffffffu, k1, o));
      k2 = max(k2, __shfl_xor_sync(0xffffffffu, k2, o));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMax(&bbox[0], k1);
      atomicMax(&bbox[1], k2);
    }
  }
}

// Is grid tile t inside the band that the transform reads?
__device__ __forceinline__ bool in_band(int t, int tiles_c, int g, int layout,
                                        const unsigned* bbox) {
  if (layout == 0) return true;
  const int tr = t / tiles_c, tc = t % tiles_c;
  const int k1 = (int)bbox[0], k2 = (int)bbox[1];
  if (tc * FIP_GTILE > k2) return false;
  const int r0 = tr * FIP_GTILE, r1 = min(r0 + FIP_GTILE, g) - 1;
  return r0 <= k1 || r1 >= g - k1;
}

// Exclusive scans of tile counts, construction of the work list (every band
// tile gets >= 1 item, so the band is fully written), and the list of tiles
// split over several items (zeroed before their reductions).  One CTA of
// kScanThreads walks the tiles in coalesced chunks.
constexpr int kScanThreads = 1024;

__device__ __forceinline__ uint3 block_exclusive_scan(uint3 v, uint3& total) {
  __shared__ uint3 s_w[kScanThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint3 inc = v;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned a = __shfl_up_sync(0xffffffffu, inc.x, o);
    const unsigned b = __shfl_up_sync(0xffffffffu, inc.y, o);
    const unsigned c = __shfl_up_sync(0xffffffffu, inc.z, o);
    if (lane >= o) {
      inc.x += a;
      inc.y += b;
      inc.z += c;
    }
  }
  if (lane == 31) s_w[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint3 w = lane < kScanThreads / 32 ? s_w[lane] : make_uint3(0, 0, 0);
    uint3 wi = w;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned a = __shfl_up_sync(0xffffffffu, wi.x, o);
      const unsigned b = __shfl_up_sync(0xffffffffu, wi.y, o);
      const unsigned c = __shfl_up_sync(0xffffffffu, wi.z, o);
      if (lane >= o) {
        wi.x += a;
        wi.y += b;
        wi.z += c;
      }
    }
    if (lane < kScanThreads / 32) s_w[lane] = make_uint3(wi.x - w.x, wi.y - w.y, wi.z - w.z);
  }
  __syncthreads();
  const uint3 base = s_w[warp];
  uint3 ex = make_uint3(base.x + inc.x - v.x, base.y + inc.y - v.y, base.z + inc.z - v.z);
  __shared__ uint3 s_total;
  if (threadIdx.x == kScanThreads - 1) s_total = make_uint3(ex.x + v.x, ex.y + v.y, ex.z + v.z);
  __syncthreads();
  total = s_total;
  __syncthreads();
  return ex;
}

__global__ void __launch_bounds__(kScanThreads) k_bin_scan(
    const unsigned* __restrict__ cnt, const unsigned* __restrict__ bbox, int ntiles, int tiles_c,
    int g, int layout, unsigned* offset, unsigned* cursor, int4* work, unsigned* nwork, int wcap,
    unsigned* multi, unsigned* nmulti) {
  uint3 carry = make_uint3(0, 0, 0);
  for (int base = 0; base < ntiles; base += kScanThreads) {
    const int t = base + threadIdx.x;
    unsigned c = 0, nch = 0;
    if (t < ntiles) {
      c = cnt[t];
      nch = in_band(t, tiles_c, g, layout, bbox) ? max(1u, (c + FIP_GCHUNK - 1) / FIP_GCHUNK)
                                                 : 0u;
    }
    uint3 total;
    const uint3 ex = block_exclusive_scan(make_uint3(c, nch, nch > 1 ? 1u : 0u), total);
    if (t < ntiles) {
      const unsigned run = carry.x + ex.x, wrun = carry.y + ex.y;
      offset[t] = run;
      cursor[t] = 0;
      for (unsigned k = 0; k < nch; ++k)
        if ((int)(wrun + k) < wcap)
          work[wrun + k] = make_int4(t, (int)(run + min(k * FIP_GCHUNK, c)),
                                     (int)(run + min((k + 1) * FIP_GCHUNK, c)), nch == 1);
      if (nch > 1) multi[carry.z + ex.z] = (unsigned)t;
    }
    carry.x += total.x;
    carry.y += total.y;
    carry.z += total.z;
  }
  if (threadIdx.x == 0) {
    offset[ntiles] = carry.x;
    *nwork = min(carry.y, (unsigned)wcap);
    *nmulti = carry.z;
  }
}

// ---------------------------------------------------------------------------
// Binning with per-CTA shared-memory histograms (grids of up to
// kMaxSmemTiles tiles).  Each CTA takes a contiguous range of visibilities,
// counts their tile entries in shared memory (native integer atomics, one
// per entry: the hardware serialises lanes that hit one counter, cheaper
// than matching the lanes first), and adds its non-zero counts to the global
// ones; one CTA then scans the tiles.  The scatter pass recounts its range,
// reserves one slice of each tile's list with one global atomic per
// (CTA, tile), and fills it through shared-memory cursors.
// ---------------------------------------------------------------------------
constexpr int kBinThreads = 256;
constexpr int kMaxSmemTiles = 12288;  // 48 KB of counters

// Visits every tile entry (tile, code) of visibility v (ok = v is valid).
template <class F>
__device__ __forceinline__ void for_each_entry(const float* B, int v, bool ok, float scale, int g,
                                               int tiles_c, unsigned& k1, unsigned& k2, F&& f) {
  Footprint fp;
  ok = ok && footprint(B, v, scale, g, fp);
  if (ok) k1 = max(k1, (unsigned)max(abs(fp.a0), abs(fp.a1)));
  for (int mir = 0; mir < 2; ++mir) {
    int c0 = 0, c1 = -1, trs[3], ntr = 0;
    const bool on = ok && half_cols(fp, mir, g, c0, c1);
    if (on) {
      ntr = tile_rows(fp, mir, g, trs);
      k2 = max(k2, (unsigned)c1);
    }
    const int tc0 = on ? c0 / FIP_GTILE : 0, tc1 = on ? c1 / FIP_GTILE : -1;
    for (int kr = 0; kr < ntr; ++kr)
      for (int tc = tc0; tc <= tc1; ++tc)
        f((unsigned)(trs[kr] * tiles_c + tc), ((unsigned)v << 1) | (unsigned)mir);
  }
}

template <int NT>
__device__ __forceinline__ uint3 block_scan3(uint3 v, uint3& total) {
  __shared__ uint3 s_w[NT / 32];
  __shared__ uint3 s_total;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint3 inc = v;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned a = __shfl_up_sync(0xffffffffu, inc.x, o);
    const unsigned b = __shfl_up_sync(0xffffffffu, inc.y, o);
    const unsigned c = __shfl_up_sync(0xffffffffu, inc.z, o);
    if (lane >= o) {
      inc.x += a;
      inc.y += b;
      inc.z += c;
    }
  }
  if (lane == 31) s_w[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const uint3 w = lane < NT / 32 ? s_w[lane] : make_uint3(0, 0, 0);
    uint3 wi = w;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned a = __shfl_up_sync(0xffffffffu, wi.x, o);
      const unsigned b = __shfl_up_sync(0xffffffffu, wi.y, o);
      const unsigned c = __shfl_up_sync(0xffffffffu, wi.z, o);
      if (lane >= o) {
        wi.x += a;
        wi.y += b;
        wi.z += c;
      }
    }
    if (lane < NT / 32) s_w[lane] = make_uint3(wi.x - w.x, wi.y - w.y, wi.z - w.z);
    if (lane == NT / 32 - 1) s_total = wi;
  }
  __syncthreads();
  const uint3 base = s_w[warp];
  total = s_total;
  __syncthreads();
  return make_uint3(base.x + inc.x - v.x, base.y + inc.y - v.y, base.z + inc.z - v.z);
}

// Tile scan run by one CTA of NT threads: offsets, cursors, the work list
// (every band tile gets >= 1 item) and the list of tiles split over several
// items.  cnt_s: the tile counts; wp_s: [ntiles + 1] scratch for the work
// prefix (both shared memory).  The work items are written in a second,
// parallel sweep (one thread per item, its tile found by bisection), so a
// tile with thousands of entries does not serialise on one thread.
template <int NT>
__device__ __forceinline__ void scan_tiles(const unsigned* cnt_s, unsigned* wp_s,
                                           const unsigned* bbox, int ntiles, int tiles_c, int g,
                                           int layout, unsigned* offset, unsigned* cursor,
                                           int4* work, unsigned* nwork, int wcap,
                                           unsigned* multi, unsigned* nmulti) {
  constexpr int PER = 8;
  uint3 carry = make_uint3(0, 0, 0);
  for (int base = 0; base < ntiles; base += NT * PER) {
    const int t0 = base + threadIdx.x * PER;
    unsigned c[PER], nch[PER];
    uint3 sum = make_uint3(0, 0, 0);
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int t = t0 + k;
      c[k] = 0;
      nch[k] = 0;
      if (t < ntiles) {
        c[k] = cnt_s[t];
        nch[k] = in_band(t, tiles_c, g, layout, bbox) ? max(1u, (c[k] + FIP_GCHUNK - 1) / FIP_GCHUNK)
                                                      : 0u;
      }
      sum.x += c[k];
      sum.y += nch[k];
      sum.z += nch[k] > 1 ? 1u : 0u;
    }
    uint3 total;
    const uint3 ex = block_scan3<NT>(sum, total);
    unsigned run = carry.x + ex.x, wrun = carry.y + ex.y, mrun = carry.z + ex.z;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int t = t0 + k;
      if (t < ntiles) {
        offset[t] = run;
        cursor[t] = 0;
        wp_s[t] = wrun;
        if (nch[k] > 1) multi[mrun++] = (unsigned)t;
        run += c[k];
        wrun += nch[k];
      }
    }
    carry.x += total.x;
    carry.y += total.y;
    carry.z += total.z;
  }
  if (threadIdx.x == 0) {
    offset[ntiles] = carry.x;
    wp_s[ntiles] = carry.y;
    *nwork = min(carry.y, (unsigned)wcap);
    *nmulti = carry.z;
  }
  __syncthreads();
  const unsigned nw = min(carry.y, (unsigned)wcap);
  for (unsigned w = threadIdx.x; w < nw; w += NT) {
    int lo = 0, hi = ntiles - 1;  // last tile with wp_s[t] <= w
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (wp_s[mid] <= w) lo = mid; else hi = mid - 1;
    }
    const int t = lo;
    const unsigned q = w - wp_s[t], nch = wp_s[t + 1] - wp_s[t], c = cnt_s[t];
    const unsigned run = offset[t];
    work[w] = make_int4(t, (int)(run + min(q * FIP_GCHUNK, c)),
                        (int)(run + min((q + 1) * FIP_GCHUNK, c)), nch == 1);
  }
}

// Count pass: per-CTA shared-memory counts added to count[], and the
// occupied band (bbox[0], bbox[1]).  count and bbox are zero on entry.
__global__ void __launch_bounds__(kBinThreads) k_bin_count(
    const float* __restrict__ B, int nb, int per_cta, float scale, int g, int tiles_c, int ntiles,
    unsigned* count, unsigned* bbox) {
  extern __shared__ unsigned s_hist[];
  __shared__ unsigned s_k[2];
  for (int t = threadIdx.x; t < ntiles; t += kBinThreads) s_hist[t] = 0;
  if (threadIdx.x < 2) s_k[threadIdx.x] = 0;
  __syncthreads();
  const int v0 = blockIdx.x * per_cta, v1 = min(nb, v0 + per_cta);
  unsigned k1 = 0, k2 = 0;
  for (int base = v0; base < v1; base += kBinThreads) {
    const int v = base + threadIdx.x;
    for_each_entry(B, v, v < v1, scale, g, tiles_c, k1, k2,
                   [&](unsigned tile, unsigned) { atomicAdd(&s_hist[tile], 1u); });
  }
  for (int o = 16; o > 0; o >>= 1) {
    k1 = max(k1, __shfl_xor_sync(0xffffffffu, k1, o));
    k2 = max(k2, __shfl_xor_sync(0xffffffffu, k2, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&s_k[0], k1);
    atomicMax(&s_k[1], k2);
  }
  __syncthreads();
  for (int t = threadIdx.x; t < ntiles; t += kBinThreads)
    if (s_hist[t]) atomicAdd(&count[t], s_hist[t]);
  if (threadIdx.x == 0) {
    atomicMax(&bbox[0], s_k[0]);
    atomicMax(&bbox[1], s_k[1]);
  }
}

// Tile scan over the final counts, one CTA of kScanThreads.
__global__ void __launch_bounds__(kScanThreads) k_bin_scan_tiles(
    const unsigned* __restrict__ count, const unsigned* __restrict__ bbox, int ntiles,
    int tiles_c, int g, int layout, unsigned* offset, unsigned* cursor, int4* work,
    unsigned* nwork, int wcap, unsigned* multi, unsigned* nmulti) {
  extern __shared__ unsigned s_cnt[];  // [ntiles] counts, then [ntiles + 1] work prefix
  __shared__ unsigned s_k[2];
  for (int t = threadIdx.x; t < ntiles; t += kScanThreads) s_cnt[t] = count[t];
  if (threadIdx.x < 2) s_k[threadIdx.x] = bbox[threadIdx.x];
  __syncthreads();
  scan_tiles<kScanThreads>(s_cnt, s_cnt + ntiles, s_k, ntiles, tiles_c, g, layout, offset,
                           cursor, work, nwork, wcap, multi, nmulti);
}

// Scatter pass: entries of the CTA's visibility range into the tile lists.
__global__ void __launch_bounds__(kBinThreads) k_bin_scatter(
    const float* __restrict__ B, int nb, int per_cta, float scale, int g, int tiles_c, int ntiles,
    const unsigned* __restrict__ offset, unsigned* cursor, unsigned* entries) {
  extern __shared__ unsigned s_hist[];
  for (int t = threadIdx.x; t < ntiles; t += kBinThreads) s_hist[t] = 0;
  __syncthreads();
  const int v0 = blockIdx.x * per_cta, v1 = min(nb, v0 + per_cta);
  unsigned k1 = 0, k2 = 0;
  for (int base = v0; base < v1; base += kBinThreads) {
    const int v = base + threadIdx.x;
    for_each_entry(B, v, v < v1, scale, g, tiles_c, k1, k2,
                   [&](unsigned tile, unsigned) { atomicAdd(&s_hist[tile], 1u); });
  }
  __syncthreads();
  for (int t = threadIdx.x; t < ntiles; t += kBinThreads) {
    const unsigned c = s_hist[t];
    if (c) s_hist[t] = offset[t] + atomicAdd(&cursor[t], c);
  }
  __syncthreads();
  for (int base = v0; base < v1; base += kBinThreads) {
    const int v = base + threadIdx.x;
    for_each_entry(B, v, v < v1, scale, g, tiles_c, k1, k2,
                   [&](unsigned tile, unsigned code) {
                     entries[atomicAdd(&s_hist[tile], 1u)] = code;
                   });
  }
}

__device__ __forceinline__ size_t cell_index(int row, int col, int g, int hp, int layout) {
  return layout ? (size_t)col * g + row : (size_t)row * hp + col;
}

// Zeroes the tiles that several work items reduce into.
// Batched launches: snapshot blockIdx.y, its lists at multi + y * multi_stride,
// nmulti[y], its grid at grid + y * grid_stride.
__global__ void k_zero_tiles(const unsigned* __restrict__ multi, const unsigned* __restrict__ nmulti,
                             int tiles_c, int g, int hp, int layout, float2* __restrict__ grid,
                             size_t multi_stride, size_t grid_stride) {
  multi += blockIdx.y * multi_stride;
  grid += blockIdx.y * grid_stride;
  const unsigned nm = nmulti[blockIdx.y];
  for (unsigned w = blockIdx.x; w < nm; w += gridDim.x) {
    const int t = (int)multi[w];
    const int row0 = (t / tiles_c) * FIP_GTILE, col0 = (t % tiles_c) * FIP_GTILE;
    for (int k = threadIdx.x; k < FIP_GTILE * FIP_GTILE; k += kThreads) {
      const int lr = layout ? k % FIP_GTILE : k / FIP_GTILE;
      const int lc = layout ? k / FIP_GTILE : k % FIP_GTILE;
      const int row = row0 + lr, col = col0 + lc;
      if (row < g && col < hp) grid[cell_index(row, col, g, hp, layout)] = make_float2(0.f, 0.f);
    }
  }
}

template <int VT>
__device__ __forceinline__ float load_vis(const void* p, int v) {
  if (VT == FIP_VIS_F32) return reinterpret_cast<const float*>(p)[v];
  if (VT == FIP_VIS_F16) return __half2float(reinterpret_cast<const __half*>(p)[v]);
  return __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(p)[v]);
}

// Shared-memory layout of one gridding work item: the tile (int32 fixed
// point) and the bound reduction; the precision form adds the tile's low
// limbs.
constexpr int kTS = FIP_GTILE + 8;  // padded row stride: 4 tap rows x 8 columns hit 32 banks
struct GridSmem {
  float re[FIP_GTILE * kTS], im[FIP_GTILE * kTS];
  float bound[kThreads / 32];
};
// Dynamic shared memory of a gridding CTA.
__host__ __device__ constexpr size_t grid_smem_bytes(bool comp) {
  return sizeof(GridSmem) + (comp ? 2 * FIP_GTILE * kTS * sizeof(float) : 0);
}

// One entry's taps inside a tile: its weights (halved for the Hermitian
// split, conjugated for the mirrored copy), its in-tile rows ia in [ia_lo,
// ia_hi) and columns ib in [ib_lo, ib_hi) of the footprint, the tile cell
// cell0 of tap (ia_lo, ib_lo), the row direction and the separable kernel
// values of the in-tile rows and columns.
struct EntryTaps {
  float wr, wi;
  int ia_lo, ia_hi, ib_lo, ib_hi, cell0, r1, mir;
  float k1[9], k2[9];
  __device__ bool empty() const { return ia_lo >= ia_hi || ib_lo >= ib_hi; }
};

template <int VT>
__device__ __forceinline__ void entry_taps(const float* __restrict__ B, const void* vr,
                                           const void* vi, const float* vis_scale, float inten,
                                           float scale, int g, unsigned ent, int trow0,
                                           int tcol0, const FipRawVis& raw, EntryTaps& e) {
  const int v = (int)(ent >> 1), mir = (int)(ent & 1);
  Footprint f;
  footprint(B, v, scale, g, f);
  int c0, c1;
  half_cols(f, mir, g, c0, c1);
  // Visibility weighting (FIPkernels.cu:188-195).
  float wr, wi;
  if constexpr (VT == FIP_VIS_RAW) {
    // Stokes-I collapse fused into the load: no collapsed copy in memory.
    float cr, ci;
    fip_collapse_sample(raw, (size_t)v, cr, ci);
    wr = cr / inten;
    wi = ci / inten;
  } else if constexpr (VT == FIP_VIS_F32) {
    wr = load_vis<VT>(vr, v) / inten;
    wi = load_vis<VT>(vi, v) / inten;
  } else {
    // Reduced storage: the value over its block's power-of-two scale.
    const float sc = vis_scale[v >> FIP_QBLOCK_SHIFT];
    wr = (load_vis<VT>(vr, v) * sc) / inten;
    wi = (load_vis<VT>(vi, v) * sc) / inten;
  }
  e.wr = 0.5f * wr;
  e.wi = mir ? -0.5f * wi : 0.5f * wi;
  e.mir = mir;
  const int nr = f.a1 - f.a0 + 1, nc = c1 - c0 + 1;
  // Tap row ia is grid row wrap(r1), r1 = a0 + ia (mirrored: -(a0 + ia)).
  // Unless the grid is one tile high, no tile holds the wrap point inside
  // it (it falls on a tile edge), so a tile's rows of the footprint are one
  // run of ia along which the tile row moves by +1 (mirrored: -1).
  int ia_lo = 9, ia_hi = 0, lr_first = 0;
#pragma unroll
  for (int a = 0; a < 9; ++a)
    if (a < nr) {
      const int lr = wrap_row(mir ? -(f.a0 + a) : f.a0 + a, g) - trow0;
      if ((unsigned)lr < (unsigned)FIP_GTILE) {
        if (a < ia_lo) {
          ia_lo = a;
          lr_first = lr;
        }
        ia_hi = a + 1;
      }
    }
  e.ia_lo = ia_lo;
  e.ia_hi = ia_hi;
  e.ib_lo = max(0, tcol0 - c0);
  e.ib_hi = min(nc, tcol0 + FIP_GTILE - c0);
  e.cell0 = lr_first * kTS + (c0 + e.ib_lo - tcol0);
  e.r1 = mir ? -(f.a0 + ia_lo) : f.a0 + ia_lo;
  const float ihs = 1 / static_cast<float>(FIP_SUPPORT / 2);
#pragma unroll
  for (int a = 0; a < 9; ++a)
    e.k1[a] = (a >= ia_lo && a < ia_hi)
                  ? fipref::es((static_cast<float>(f.a0 + a) - f.p1) * ihs)
                  : 0.f;
  // Column taps in half-plane order c0..c1: original r2 = c (direct) or -c
  // (mirrored); on the Nyquist column a direct tap is r2 = -G/2 (r2 never
  // reaches +G/2, FIPkernels.cu:203).
#pragma unroll
  for (int b = 0; b < 9; ++b) {
    const int c = c0 + b;
    const int r2 = mir ? -c : (2 * c == g ? -c : c);
    e.k2[b] = (b >= e.ib_lo && b < e.ib_hi)
                  ? fipref::es((static_cast<float>(r2) - f.p2) * ihs)
                  : 0.f;
  }
}

// One gridding work item (tile, entry range) of one snapshot, a thread per
// entry (at most one per thread: FIP_GCHUNK <= kThreads).  Phase 1 takes the
// thread's entry footprint and kernel values into registers and reduces the
// item's bound, phase 2 walks the entry's in-tile taps into the shared
// tile, phase 3 commits.  The tile sums are fixed point, so the shared-memory
// sums are native integer atomics: exact and independent of their order.
// Plain form: q = round(tap * 2^30 / bound) in one int32, `bound` (the
// item's summed weights) bounding every cell sum.
// Precision form with FP32 visibilities (COMP; with FP16/BF16 storage the
// precision form sums as the plain form does): t = tap * 2^e, 2^e = the power of two with
// bound * 2^e < 2^45, is exact in FP32 and is split exactly into
// hi * 2^23 + lo (hi < 2^22 in magnitude, 0 <= lo <= 2^23), two int32 limbs
// summed separately (at most 256 taps per cell per item: no overflow), so a
// cell holds the exact sum of its FP32 taps to 2^-45 of the bound and is
// rounded once at the commit.
template <int VT, bool COMP>
__device__ __forceinline__ void grid_item(GridSmem& S, float* s_cre, float* s_cim,
                                          const float* __restrict__ B,
                                          const void* vr, const void* vi,
                                          const float* vis_scale, float inten, float scale,
                                          int g, int hp, int tiles_c,
                                          int layout, const unsigned* __restrict__ entries,
                                          int4 item, float2* __restrict__ grid,
                                          const FipRawVis& raw = FipRawVis{}) {
  static_assert(FIP_GCHUNK <= kThreads, "one entry per thread at most");
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int tile = item.x, cnt = item.z - item.y;
  const int trow0 = (tile / tiles_c) * FIP_GTILE, tcol0 = (tile % tiles_c) * FIP_GTILE;
  for (int k = threadIdx.x; k < FIP_GTILE * kTS; k += kThreads) {
    S.re[k] = 0.f;
    S.im[k] = 0.f;
    if (COMP) {
      s_cre[k] = 0.f;
      s_cim[k] = 0.f;
    }
  }
  // Phase 1: this thread's entry.
  const int q = threadIdx.x;
  const bool have = q < cnt;
  EntryTaps et;
  float bound = 0.f;  // sum over the item of max(|wr|, |wi|): bounds every cell sum
  if (have) {
    entry_taps<VT>(B, vr, vi, vis_scale, inten, scale, g, entries[item.y + q], trow0, tcol0,
                   raw, et);
    bound = fmaxf(fabsf(et.wr), fabsf(et.wi));
  }
  for (int o = 16; o > 0; o >>= 1) bound += __shfl_xor_sync(0xffffffffu, bound, o);
  if (lane == 0) S.bound[warp] = bound;
  __syncthreads();
  float tot = 0.f;
#pragma unroll
  for (int w = 0; w < kThreads / 32; ++w) tot += S.bound[w];
  tot *= 1.0001f;  // margin for the rounding of the weights and their sum
  float fx = 0.f, fx_inv = 0.f;
  if (!COMP) {
    fx = tot > 0.f ? 1073741824.0f / tot : 0.f;
    fx_inv = tot * (1.0f / 1073741824.0f);
  } else if (tot > 0.f) {
    int ex = 0;
    frexpf(tot, &ex);  // tot < 2^ex
    fx = ldexpf(1.0f, 45 - ex);
    fx_inv = ldexpf(1.0f, ex - 45);
  }
  int* s_qre = reinterpret_cast<int*>(S.re);
  int* s_qim = reinterpret_cast<int*>(S.im);
  unsigned* s_lre = reinterpret_cast<unsigned*>(s_cre);
  unsigned* s_lim = reinterpret_cast<unsigned*>(s_cim);
  // Exact limbs of t = x * 2^e (precision form, see above).
  auto limbs = [&](float x, int& hi, unsigned& lo) {
    const float t = x * fx;
    const float hf = floorf(t * (1.0f / 8388608.0f));
    const float lf = fmaf(hf, -8388608.0f, t);  // exact: t - hi 2^23 in [0, 2^23]
    hi = __float_as_int(hf + 12582912.0f) - 0x4B400000;  // |hf| < 2^22: exact
    lo = __float_as_uint(lf + 8388608.0f) - 0x4B000000u;  // round to integer
  };
  // Phase 2: the thread walks its entry's in-tile taps.
  if (have && !et.empty()) {
    const float wrf = COMP ? et.wr : et.wr * fx, wif = COMP ? et.wi : et.wi * fx;
    const int dstep = et.mir ? -kTS : kTS;
    const int lc0 = et.cell0 - (wrap_row(et.r1, g) - trow0) * kTS;
#pragma unroll
    for (int a = 0; a < 9; ++a) {
      if (a < et.ia_lo || a >= et.ia_hi) continue;
      // One tile row holding the whole grid may hold the wrap point: each
      // tap row is then wrapped on its own.
      const int rc = g > FIP_GTILE
                         ? et.cell0 + (a - et.ia_lo) * dstep
                         : (wrap_row(et.r1 + (et.mir ? et.ia_lo - a : a - et.ia_lo), g) - trow0) *
                                   kTS + lc0;
      const float ra = wrf * et.k1[a], rb = wif * et.k1[a];
#pragma unroll
      for (int b = 0; b < 9; ++b) {
        if (b < et.ib_lo || b >= et.ib_hi) continue;
        const int c = rc + (b - et.ib_lo);
        if (!COMP) {
          atomicAdd(&s_qre[c], __float2int_rn(ra * et.k2[b]));
          atomicAdd(&s_qim[c], __float2int_rn(rb * et.k2[b]));
        } else {
          int hr, hi;
          unsigned lr2, li2;
          limbs(ra * et.k2[b], hr, lr2);
          limbs(rb * et.k2[b], hi, li2);
          atomicAdd(&s_qre[c], hr);
          atomicAdd(&s_lre[c], lr2);
          atomicAdd(&s_qim[c], hi);
          atomicAdd(&s_lim[c], li2);
        }
      }
    }
  }
  __syncthreads();
  // Phase 3: commit in the layout's contiguous direction.
  const bool single = item.w != 0;
  for (int k = threadIdx.x; k < FIP_GTILE * FIP_GTILE; k += kThreads) {
    const int lr = layout ? k % FIP_GTILE : k / FIP_GTILE;
    const int lc = layout ? k / FIP_GTILE : k % FIP_GTILE;
    const int row = trow0 + lr, col = tcol0 + lc;
    if (row < g && col < hp) {
      float2 val;
      if (COMP) {
        const int at = lr * kTS + lc;
        const unsigned* s_lre = reinterpret_cast<const unsigned*>(s_cre);
        const unsigned* s_lim = reinterpret_cast<const unsigned*>(s_cim);
        val = make_float2((float)(((double)s_qre[at] * 8388608.0 + (double)s_lre[at]) * fx_inv),
                          (float)(((double)s_qim[at] * 8388608.0 + (double)s_lim[at]) * fx_inv));
      } else {
        val = make_float2((float)s_qre[lr * kTS + lc] * fx_inv,
                          (float)s_qim[lr * kTS + lc] * fx_inv);
      }
      float2* dst = &grid[cell_index(row, col, g, hp, layout)];
      if (single) {
        *dst = val;
      } else if (val.x != 0.f || val.y != 0.f) {
        atomicAdd(dst, val);
      }
    }
  }
  __syncthreads();
}

__device__ __forceinline__ float plane_intensity(const float* V) {
  return fabs(V[0 * 3 + 0] * V[1 * 3 + 1] - V[0 * 3 + 1] * V[1 * 3 + 0]);
}

// Persistent gridder over the work items of one snapshot.
template <int VT, bool COMP>
__global__ void __launch_bounds__(kThreads) k_grid(const float* __restrict__ B, const void* vr,
                                                   const void* vi,
                                                   const float* __restrict__ vis_scale_p,
                                                   const float* __restrict__ V, float scale,
                                                   int g, int hp, int tiles_c, int layout,
                                                   const unsigned* __restrict__ entries,
                                                   const int4* __restrict__ work,
                                                   const unsigned* __restrict__ nwork,
                                                   float2* __restrict__ grid,
                                                   const FipRawVis raw) {
  extern __shared__ float4 s_raw[];
  GridSmem& S = *reinterpret_cast<GridSmem*>(s_raw);
  float* s_cre = reinterpret_cast<float*>(reinterpret_cast<char*>(s_raw) + sizeof(GridSmem));
  float* s_cim = s_cre + FIP_GTILE * kTS;
  const float inten = plane_intensity(V);
  const unsigned nw = *nwork;
  __syncthreads();
  for (unsigned w = blockIdx.x; w < nw; w += gridDim.x)
    grid_item<VT, COMP>(S, s_cre, s_cim, B, vr, vi, vis_scale_p, inten, scale, g, hp, tiles_c,
                        layout, entries, work[w], grid, raw);
}

// Persistent gridder over the work items of a batch of snapshots (one launch
// for the batch, whatever their image sizes): snapshot k's inputs, bins,
// grid and geometry are in.s[k].
template <int VT, bool COMP>
__global__ void __launch_bounds__(kThreads) k_grid_batch(const __grid_constant__ FipGridBatch in) {
  extern __shared__ float4 s_raw[];
  __shared__ unsigned s_first[FIP_MAX_BATCH + 1];  // prefix of the snapshots' item counts
  GridSmem& S = *reinterpret_cast<GridSmem*>(s_raw);
  float* s_cre = reinterpret_cast<float*>(reinterpret_cast<char*>(s_raw) + sizeof(GridSmem));
  float* s_cim = s_cre + FIP_GTILE * kTS;
  if (threadIdx.x == 0) {
    unsigned acc = 0;
    for (int k = 0; k < in.count; ++k) {
      s_first[k] = acc;
      acc += *in.s[k].nwork;
    }
    s_first[in.count] = acc;
  }
  __syncthreads();
  const unsigned total = s_first[in.count];
  int k = 0;
  for (unsigned w = blockIdx.x; w < total; w += gridDim.x) {
    while (s_first[k + 1] <= w) ++k;  // items are visited in increasing order
    const FipGridSnap& sn = in.s[k];
    const float inten = plane_intensity(sn.V);
    grid_item<VT, COMP>(S, s_cre, s_cim, sn.B, sn.vr, sn.vi, sn.vis_scale, inten, sn.scale, sn.g,
                        sn.hp, sn.tiles_c, sn.layout, sn.entries, sn.work[w - s_first[k]],
                        sn.grid);
  }
}

// Block-wide maximum of non-negative v, folded into *out (float bits) with
// one atomic per CTA.  All threads of the CTA must call it.
__device__ __forceinline__ void block_max_to(float v, unsigned* out) {
  __shared__ float s_m[32];
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) s_m[warp] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    float m = 0.f;
    for (int w = 0; w < (int)((blockDim.x + 31) >> 5); ++w) m = fmaxf(m, s_m[w]);
    atomicMax(out, __float_as_uint(m));
  }
}

// ---------------------------------------------------------------------------
// Band-pruned inverse FFT (power-of-two images), instantiated per
// M = 2^LM = G / 3 and E = 2^LE values per thread (3 M / E threads).
// Column pass: P[c][yy] = sum_r1 H[c][r1 mod G] e^{+2 pi i y r1 / G},
// y = yy - N/2, for the occupied half-plane columns c <= bbox[1] and rows
// |r1| <= bbox[0].
// ---------------------------------------------------------------------------
template <int LM, int LE>
__host__ __device__ constexpr int fft_threads() { return 3 << (LM - LE); }
// CTAs per SM the register budget allows: the staged forms hold two
// buffers of shared memory (two CTAs of 768 or 384 threads); the direct form
// holds one, so three CTAs of 384 threads fit.
template <int LM, int LE, bool DIRECT>
__host__ __device__ constexpr int fft_min_blocks() {
  return fft_threads<LM, LE>() >= 768 && LE == 4 ? 1 : (DIRECT && LE == 4 ? 3 : 2);
}

template <int LM, int LE, bool DIRECT>
__global__ void __launch_bounds__(fft_threads<LM, LE>(), (fft_min_blocks<LM, LE, DIRECT>()))
    k_fft_cols(const float2* __restrict__ H, const unsigned* __restrict__ bbox,
               float2* __restrict__ P, const float2* __restrict__ tw, size_t grid_stride,
               size_t col_stride) {
  constexpr int M = 1 << LM, g = 3 * M, half = g / 2, n = 2 * M, NT = fft_threads<LM, LE>();
  extern __shared__ float2 s_fft[];
  // Batched launches: snapshot blockIdx.y.
  H += blockIdx.y * grid_stride;
  P += blockIdx.y * col_stride;
  bbox += 4 * blockIdx.y;
  const int k2 = (int)bbox[1];
  const int k1 = min((int)bbox[0], half);
  // Row band [lo, hi]; row -G/2 is row +G/2 (counted once).
  const int lo = (k1 == half) ? 1 - k1 : -k1, hi = k1;
  // Stage the band densely (coalesced): st[r - lo] = H[c][r mod G]; or
  // (DIRECT) read it from global memory in the first pass.
  // A band no wider than M is staged pre-twiddled for the three
  // sub-transforms (fipfft::stage_pre).
  float2* st = s_fft + fipfft::stage_offset(g);
  const bool fold = !DIRECT && hi - lo + 1 <= M;
  auto band = [&](int c, int r) -> float2 { return H[(size_t)c * g + (r < 0 ? r + g : r)]; };
  // The staged form is persistent over columns (blockIdx.x + k gridDim.x):
  // a thread's first staged element of the next column is loaded while the
  // current column is transformed.
  const int r0 = lo + (int)threadIdx.x;
  float2 pf = make_float2(0.f, 0.f);
  if (!DIRECT && (int)blockIdx.x <= k2 && r0 <= hi) pf = band(blockIdx.x, r0);
  for (int c = blockIdx.x; c <= k2; c += gridDim.x) {
    // Pass twiddles (registers): loaded after the staging loop, so their
    // latency overlaps the staging barrier without holding registers through
    // the loop (measured faster here than loading them up front).
    fipfft::PassTw<LM, LE> pt;
    if (DIRECT) pt.load(tw + g, fipfft::sub_lane<LM, LE>(threadIdx.x));
    if (fold) {
      fipfft::StageTw w(tw, g, r0, NT);
      if (r0 <= hi) fipfft::stage_pre<M>(st, r0, pf, w.w1, w.w2);
      w.next();
      for (int i = threadIdx.x + NT; i <= hi - lo; i += NT, w.next()) {
        const int r = i + lo;
        fipfft::stage_pre<M>(st, r, band(c, r), w.w1, w.w2);
      }
    } else if (!DIRECT) {
      if (r0 <= hi) st[threadIdx.x] = pf;
      for (int i = threadIdx.x + NT; i <= hi - lo; i += NT) st[i] = band(c, i + lo);
    }
    if (!DIRECT) {
      pt.load(tw + g, fipfft::sub_lane<LM, LE>(threadIdx.x));
      if (fold) fipfft::zero_pre<M>(st, lo, hi, threadIdx.x, NT);
      __syncthreads();
      // The next column's first element, in flight during this transform.
      const int nx = c + gridDim.x;
      if (nx <= k2 && r0 <= hi) pf = band(nx, r0);
    }
    if (fold) {
      fipfft::run_pre<LM, LE>(s_fft, pt);
    } else {
      auto load = [&](int r) -> float2 { return DIRECT ? band(c, r) : st[r - lo]; };
      fipfft::run<LM, LE, DIRECT>(s_fft, tw, pt, lo, hi, load);
    }
    float4* out = reinterpret_cast<float4*>(P + (size_t)c * n);
    for (int o2 = threadIdx.x; o2 < n / 2; o2 += NT) {
      float2 ab[2];
      fipfft::fetch_run<LM, LE, 2, DIRECT>(s_fft, 2 * o2, ab);
      out[o2] = make_float4(ab[0].x, ab[0].y, ab[1].x, ab[1].y);
    }
    // The next staging writes the second buffer: when the last pass left
    // its outputs there, every thread must be done reading them.
    if constexpr (!DIRECT && ((fipfft::pass_count<LM, LE>() - 1) & 1)) __syncthreads();
  }
}

// Bulk tensor copies (TMA) with an mbarrier, for the row pass's band copy.
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// Bounded wait for phase `parity` of *bar: false if it did not complete
// within kMbarSpin polls.
constexpr unsigned kMbarSpin = 1u << 20;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  const unsigned a = smem_u32(bar);
  for (unsigned it = 0; it < kMbarSpin; ++it) {
    unsigned done = 0;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y,
                                            int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
// The row pass's band copy: columns 0 .. K2 (at most kBandCap; wider bands
// read global memory) of a row pair, kBandBox columns per bulk copy, 16
// bytes (rows yy1, yy1 + 1 of one column) each.
constexpr int kBandCap = 1024;
constexpr int kBandBox = 256;
// The copy's buffer follows the direct form's pass buffer; a bulk tensor
// copy's shared-memory destination must be 128-byte aligned, and dynamic
// shared memory starts after the kernel's static shared memory (not on a
// 128-byte boundary), so the buffer is aligned at run time within 128 bytes
// of slack.
template <int LM>
__host__ __device__ constexpr size_t band_offset() {  // bytes
  return (size_t)fipfft::direct_smem_elems(3 << LM) * sizeof(float2);
}
template <int LM>
__host__ __device__ constexpr size_t band_smem_bytes() {
  return band_offset<LM>() + 128 + (size_t)kBandCap * 16;
}

// Row pass for image rows yy1 = 2b, yy2 = 2b+1: their Hermitian spectra
// X1, X2 (the column-pass output, extended by X(-c) = conj X(c)) are packed as
// Z = X1 + i X2 so one complex transform yields both real rows.  The epilogue
// is the reference's crop/correction (FIPkernels.cu:256-287): the image pixel
// is |out| / (taper|x| taper|y| norm^2) (the checkerboard signs cancel
// against the centred grid origin), applied as a product of the reciprocal
// table rck[t] = 1 / (taper[t] norm).
// BAND (with DIRECT, persistent over row pairs): the first pass reads the
// row pair's band from a shared-memory copy that bulk tensor copies bring in
// one row pair ahead (band_map: the column-pass output as floats [batch][G/2
// + 1][2 N]); a copy that does not arrive within the wait limit switches the
// CTA to global reads (same results).
template <int LM, int LE, bool DIRECT, bool BAND = false>
__global__ void __launch_bounds__(fft_threads<LM, LE>(), (fft_min_blocks<LM, LE, DIRECT>()))
    k_fft_rows(const float2* __restrict__ P, unsigned* bbox,
               const float* __restrict__ rck, float* __restrict__ pre,
               const float2* __restrict__ tw, size_t col_stride, size_t pre_stride,
               const __grid_constant__ CUtensorMap band_map) {
  static_assert(!BAND || DIRECT, "the band copy replaces the direct form's global reads");
  constexpr int M = 1 << LM, g = 3 * M, half = g / 2, n = 2 * M, h = M, NT = fft_threads<LM, LE>();
  extern __shared__ float2 s_fft[];
  // Batched launches: snapshot blockIdx.y.
  P += blockIdx.y * col_stride;
  pre += blockIdx.y * pre_stride;
  bbox += 4 * blockIdx.y;
  const int k2 = min((int)bbox[1], half);
  // Column band [lo, hi]; column -G/2 is column +G/2 (counted once).
  const int lo = (k2 == half) ? 1 - k2 : -k2, hi = k2;
  // Stage Z[c] = X1[c] + i X2[c] at st[c - lo], with X(-c) = conj X(c):
  // one 16-byte load per occupied column c (the column pass stores
  // P[c][yy]), written at c and -c.
  float2* st = s_fft + fipfft::stage_offset(g);
  // Pass twiddles first: their loads overlap the staging loads.
  fipfft::PassTw<LM, LE> pt;
  pt.load(tw + g, fipfft::sub_lane<LM, LE>(threadIdx.x));
  // A band no wider than M is staged pre-twiddled (fipfft::stage_pre).
  const bool fold = !DIRECT && hi - lo + 1 <= M;
  // The staged form is persistent over row pairs (blockIdx.x + k gridDim.x):
  // a thread's first staged column of the next row pair is loaded into
  // registers while the current pair is transformed, so its latency leaves
  // the staging step (two columns measured slower: more spills).
  constexpr int kPf = 1;
  float4 pf[kPf];
  auto col_load = [&](int c, int yy) -> float4 {
    return *reinterpret_cast<const float4*>(P + (size_t)c * n + yy);
  };
#pragma unroll
  for (int m = 0; m < kPf; ++m) {
    const int c = threadIdx.x + m * NT;
    if (!DIRECT && c <= k2) pf[m] = col_load(c, 2 * blockIdx.x);
  }
  // BAND: the copy's buffer, its mbarrier, and the parity of a copy issued
  // but not yet consumed (-1: none).
  char* band_raw = reinterpret_cast<char*>(s_fft) + band_offset<LM>();
  float4* sband =
      reinterpret_cast<float4*>(band_raw + ((128u - (smem_u32(band_raw) & 127u)) & 127u));
  __shared__ uint64_t s_bandbar;
  // Uniform over the CTA; a misaligned buffer (not expected) reads global
  // memory instead.
  bool band = BAND && k2 + 1 <= kBandCap && (smem_u32(sband) & 127u) == 0;
  int pend = -1;
  const int nbox = (k2 + kBandBox) / kBandBox;  // boxes covering columns 0 .. k2
  auto issue = [&](int rpair) {  // one thread
    mbar_expect_tx(&s_bandbar, (unsigned)(nbox * kBandBox * 16));
    for (int b = 0; b < nbox; ++b)
      tma_load_3d(sband + b * kBandBox, &band_map, 4 * rpair, b * kBandBox, (int)blockIdx.y,
                  &s_bandbar);
  };
  if (BAND && band) {
    if (threadIdx.x == 0) {
      mbar_init(&s_bandbar, 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (blockIdx.x < n / 2) {
      if (threadIdx.x == 0) issue(blockIdx.x);
      pend = 0;
    }
  }
  float vmax = 0.f;
  int it = 0;
  for (int rp = blockIdx.x; rp < n / 2; rp += gridDim.x, ++it) {
    const int yy1 = 2 * rp;
    if (BAND && band) {
      const bool got = mbar_wait(&s_bandbar, (unsigned)(it & 1));
      band = __syncthreads_and(got) != 0;
      if (band) pend = -1;  // else the copy stays pending: drained at the end
    }
    if (!DIRECT) {
      fipfft::StageTw w(tw, g, threadIdx.x, NT);
      auto stage = [&](int c, const float4& ab) {
        float ay = ab.y, by = ab.w;
        if (c == 0 || c == half) {  // self-conjugate bins are real
          ay = 0.f;
          by = 0.f;
        }
        const float2 zp = make_float2(ab.x - by, ay + ab.z);
        const float2 zm = make_float2(ab.x + by, ab.z - ay);  // conj X1 + i conj X2
        if (fold) {
          // w^{-c} = conj w^c
          fipfft::stage_pre<M>(st, c, zp, w.w1, w.w2);
          if (c > 0 && -c >= lo)
            fipfft::stage_pre<M>(st, -c, zm, make_float2(w.w1.x, -w.w1.y),
                                 make_float2(w.w2.x, -w.w2.y));
        } else {
          st[c - lo] = zp;
          if (c > 0 && -c >= lo) st[-c - lo] = zm;
        }
      };
#pragma unroll
      for (int m = 0; m < kPf; ++m, w.next()) {
        const int c = threadIdx.x + m * NT;
        if (c <= k2) stage(c, pf[m]);
      }
      for (int c = threadIdx.x + kPf * NT; c <= k2; c += NT, w.next()) stage(c, col_load(c, yy1));
      if (fold) fipfft::zero_pre<M>(st, lo, hi, threadIdx.x, NT);
      __syncthreads();
      // The next row pair's first columns, in flight during this transform.
      const int nx = rp + gridDim.x;
#pragma unroll
      for (int m = 0; m < kPf; ++m) {
        const int c = threadIdx.x + m * NT;
        if (nx < n / 2 && c <= k2) pf[m] = col_load(c, 2 * nx);
      }
    }
    // DIRECT: Z[c] straight from the column-pass output (L2-resident).
    auto zval = [&](int c) -> float2 {
      const int a = c < 0 ? -c : c;
      const float4 ab = (BAND && band) ? sband[a] : col_load(a, yy1);
      float ay = ab.y, by = ab.w;
      if (a == 0 || a == half) {
        ay = 0.f;
        by = 0.f;
      }
      return c >= 0 ? make_float2(ab.x - by, ay + ab.z) : make_float2(ab.x + by, ab.z - ay);
    };
    auto load = [&](int c) -> float2 { return DIRECT ? zval(c) : st[c - lo]; };
    if (fold) {
      fipfft::run_pre<LM, LE>(s_fft, pt);
    } else if constexpr (BAND) {
      // Once every thread holds its band values, the next row pair's copy
      // goes into the buffer (it lands during this pair's passes).
      auto loaded = [&]() {
        if (!band) return;
        __syncthreads();
        const int nx = rp + (int)gridDim.x;
        if (nx < n / 2) {
          if (threadIdx.x == 0) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue(nx);
          }
          pend = (it + 1) & 1;
        }
      };
      fipfft::run<LM, LE, DIRECT>(s_fft, tw, pt, lo, hi, load, loaded);
    } else {
      fipfft::run<LM, LE, DIRECT>(s_fft, tw, pt, lo, hi, load);
    }
    const float ry1 = rck[abs(yy1 - h)], ry2 = rck[abs(yy1 + 1 - h)];
    float4* row1 = reinterpret_cast<float4*>(pre + (size_t)yy1 * n);
    float4* row2 = reinterpret_cast<float4*>(pre + (size_t)(yy1 + 1) * n);
    // The epilogue's correction factors, all loads issued before the first
    // output is formed.
    constexpr int KQ = (n / 4 + NT - 1) / NT;
    float rxs[KQ][4];
#pragma unroll
    for (int q = 0; q < KQ; ++q) {
      const int o4 = threadIdx.x + q * NT;
#pragma unroll
      for (int e = 0; e < 4; ++e)
        rxs[q][e] = o4 < n / 4 ? __ldg(&rck[abs(4 * o4 + e - h)]) : 0.f;
    }
#pragma unroll
    for (int q = 0; q < KQ; ++q) {
      const int o4 = threadIdx.x + q * NT;
      if (o4 < n / 4) {
        float a[4], b[4];
        float2 v[4];
        fipfft::fetch_run<LM, LE, 4, DIRECT>(s_fft, 4 * o4, v);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float rx = rxs[q][e];
          a[e] = fabsf(v[e].x * (rx * ry1));
          b[e] = fabsf(v[e].y * (rx * ry2));
          vmax = fmaxf(vmax, fmaxf(a[e], b[e]));
        }
        row1[o4] = make_float4(a[0], a[1], a[2], a[3]);
        row2[o4] = make_float4(b[0], b[1], b[2], b[3]);
      }
    }
    // The next staging writes the second buffer: when the last pass left
    // its outputs there, every thread must be done reading them.
    if constexpr (!DIRECT && ((fipfft::pass_count<LM, LE>() - 1) & 1)) __syncthreads();
  }
  // A copy still pending (its wait ran out) lands before the CTA's shared
  // memory goes away (bounded, like every wait here).
  if (BAND && pend >= 0 && threadIdx.x == 0) mbar_wait(&s_bandbar, (unsigned)pend);
  // Image maximum (bbox[3], float bits; zeroed by the binning), which
  // scales the reprojection's fixed-point sums.
  block_max_to(vmax, &bbox[3]);
}

// Split forms of the two passes: one CTA of M / E threads per (column or row
// pair, sub-transform s), grid.y = s, grid.z = snapshot of a batch.  Three
// times the CTAs of a quarter of the size: each CTA's barriers hold four
// warps instead of twelve, and CTAs at different phases share an SM.  Each
// CTA stages the band itself (in its second buffer when it fits, else reads
// it from global memory) and writes its outputs X[3 q + s] directly.
template <int LM, int LE>
__host__ __device__ constexpr int split_threads() { return 1 << (LM - LE); }

template <int LM, int LE>
__global__ void __launch_bounds__(split_threads<LM, LE>(), (LE == 4 ? 6 : 4))
    k_fft_cols_split(const float2* __restrict__ H, const unsigned* __restrict__ bbox,
                     float2* __restrict__ P, const float2* __restrict__ tw, size_t grid_stride,
                     size_t col_stride) {
  constexpr int M = 1 << LM, g = 3 * M, half = g / 2, n = 2 * M, NT = split_threads<LM, LE>();
  constexpr int kCap = fipfft::sub_stride(M);  // staging capacity (the second buffer)
  extern __shared__ float2 s_fft[];
  H += blockIdx.z * grid_stride;
  P += blockIdx.z * col_stride;
  bbox += 4 * blockIdx.z;
  const int c = blockIdx.x, s = blockIdx.y;
  const int k2 = (int)bbox[1];
  if (c > k2) return;
  const int k1 = min((int)bbox[0], half);
  const int lo = (k1 == half) ? 1 - k1 : -k1, hi = k1;
  const float2* col = H + (size_t)c * g;
  float2* st = s_fft + kCap;
  const bool staged = hi - lo + 1 <= kCap;
  if (staged)
    for (int i = threadIdx.x; i <= hi - lo; i += NT) {
      const int r = i + lo;
      st[i] = col[r < 0 ? r + g : r];
    }
  __syncthreads();
  auto load = [&](int r) -> float2 { return staged ? st[r - lo] : col[r < 0 ? r + g : r]; };
  fipfft::PassTw<LM, LE> pt;
  pt.load(tw + g, threadIdx.x);
  fipfft::run_single<LM, LE>(s_fft, s, tw, pt, lo, hi, load);
  float2* out = P + (size_t)c * n;
  for (int q = threadIdx.x; q < M; q += NT) {
    const int pp = 3 * q + s;  // output p = pp (mod G), kept when |p| <= M
    const int o = pp < M ? pp + M : (pp >= 2 * M ? pp - 2 * M : -1);
    if (o >= 0) out[o] = fipfft::single_out<LM, LE>(s_fft, q);
  }
}

template <int LM, int LE>
__global__ void __launch_bounds__(split_threads<LM, LE>(), (LE == 4 ? 6 : 4))
    k_fft_rows_split(const float2* __restrict__ P, unsigned* bbox, const float* __restrict__ rck,
                     float* __restrict__ pre, const float2* __restrict__ tw, size_t col_stride,
                     size_t pre_stride) {
  constexpr int M = 1 << LM, g = 3 * M, half = g / 2, n = 2 * M, h = M;
  constexpr int NT = split_threads<LM, LE>(), kCap = fipfft::sub_stride(M);
  extern __shared__ float2 s_fft[];
  P += blockIdx.z * col_stride;
  pre += blockIdx.z * pre_stride;
  bbox += 4 * blockIdx.z;
  const int yy1 = 2 * blockIdx.x, s = blockIdx.y;
  const int k2 = min((int)bbox[1], half);
  const int lo = (k2 == half) ? 1 - k2 : -k2, hi = k2;
  // Z[c] = X1[c] + i X2[c], X(-c) = conj X(c), from the column-pass output.
  auto zval = [&](int c) -> float2 {
    const int a = c < 0 ? -c : c;
    const float4 ab = *reinterpret_cast<const float4*>(P + (size_t)a * n + yy1);
    float ay = ab.y, by = ab.w;
    if (a == 0 || a == half) {  // self-conjugate bins are real
      ay = 0.f;
      by = 0.f;
    }
    return c >= 0 ? make_float2(ab.x - by, ay + ab.z) : make_float2(ab.x + by, ab.z - ay);
  };
  float2* st = s_fft + kCap;
  const bool staged = hi - lo + 1 <= kCap;
  if (staged)
    for (int c = threadIdx.x; c <= k2; c += NT) {
      const float4 ab = *reinterpret_cast<const float4*>(P + (size_t)c * n + yy1);
      float ay = ab.y, by = ab.w;
      if (c == 0 || c == half) {
        ay = 0.f;
        by = 0.f;
      }
      st[c - lo] = make_float2(ab.x - by, ay + ab.z);
      if (c > 0 && -c >= lo) st[-c - lo] = make_float2(ab.x + by, ab.z - ay);
    }
  __syncthreads();
  auto load = [&](int c) -> float2 { return staged ? st[c - lo] : zval(c); };
  fipfft::PassTw<LM, LE> pt;
  pt.load(tw + g, threadIdx.x);
  fipfft::run_single<LM, LE>(s_fft, s, tw, pt, lo, hi, load);
  const float ry1 = rck[abs(yy1 - h)], ry2 = rck[abs(yy1 + 1 - h)];
  float* row1 = pre + (size_t)yy1 * n;
  float* row2 = row1 + n;
  float vmax = 0.f;
  for (int q = threadIdx.x; q < M; q += NT) {
    const int pp = 3 * q + s;
    const int o = pp < M ? pp + M : (pp >= 2 * M ? pp - 2 * M : -1);
    if (o >= 0) {
      const float2 v = fipfft::single_out<LM, LE>(s_fft, q);
      const float rx = rck[abs(o - h)];
      const float a = fabsf(v.x * (rx * ry1)), b = fabsf(v.y * (rx * ry2));
      row1[o] = a;
      row2[o] = b;
      vmax = fmaxf(vmax, fmaxf(a, b));
    }
  }
  block_max_to(vmax, &bbox[3]);
}

// Crop + correction of the cuFFT C2R output (images whose grid side is not
// 3 * 2^k): row (y mod G), column (x mod G), row stride G + 2 floats.
__global__ void k_correct_c2r(const float* __restrict__ fft_out, const float* __restrict__ ck,
                              int n, int g, float* __restrict__ pre, unsigned* pre_max) {
  const int xx = blockIdx.x * blockDim.x + threadIdx.x, yy = blockIdx.y;
  float v = 0.f;
  if (xx < n) {
    const int h = n / 2;
    const long x = (long)xx - h, y = (long)yy - h;
    const int row = (int)(y < 0 ? y + g : y), col = (int)(x < 0 ? x + g : x);
    float px = fft_out[(size_t)row * (size_t)(g + 2) + col];
    const float norm = FIP_CONV_NORM;
    px *= 1 / (ck[labs(x)] * ck[labs(y)] * norm * norm);
    v = fabs(px);
    pre[(size_t)yy * n + xx] = v;
  }
  block_max_to(v, pre_max);
}

// ---------------------------------------------------------------------------
// Reprojection (FIPkernels.cu:289-413).
// ---------------------------------------------------------------------------

// The reference's pixel mapping for every source pixel: targets[j*N + i] =
// (LL, MM) of source column i, row j.  Compute-bound; overlapped with the
// gridding and the FFT on a side stream.
constexpr int kTargetsPerThread = 4;
// ttab: the theta-terms table (fipref::kThetaTabSize entries) or null.
__global__ void k_targets(const float* __restrict__ V, int n, float dc,
                          const float2* __restrict__ ttab, float2* __restrict__ tg) {
  const int j = blockIdx.y;
  const fipref::Frame fr{V[0], V[1], V[3], V[4], V[8], V[6], V[7], dc};
#pragma unroll
  for (int q = 0; q < kTargetsPerThread; ++q) {
    const int i = (blockIdx.x * kTargetsPerThread + q) * blockDim.x + threadIdx.x;
    if (i < n) {
      float LL, MM;
      fipref::pixel_target(fr, i, j, n, LL, MM, ttab);
      tg[(size_t)j * n + i] = make_float2(LL, MM);
    }
  }
}

__global__ void k_theta_table(float2* __restrict__ tab) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= fipref::kThetaTabSize) return;
  float r, zr0;
  fipref::theta_terms(__uint_as_float(fipref::kThetaTabLo + (unsigned)k), r, zr0);
  tab[k] = make_float2(r, zr0);
}

// Source-major reprojection, the reference's own scheme (FIPkernels.cu:378-413):
// one thread per source pixel, four atomics into a zeroed destination.
__global__ void k_reproject_scatter(const float* __restrict__ pre, const float* __restrict__ V,
                                    int n, int nb, float dc, float* __restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= n || j >= n) return;
  fipref::Frame fr{V[0], V[1], V[3], V[4], V[8], V[6], V[7], dc};
  const float inv_nb = 1.0f / static_cast<float>(nb);
  const float value = pre[(size_t)j * n + i] * inv_nb;
  float LL, MM;
  fipref::pixel_target(fr, i, j, n, LL, MM);
  const size_t half = n / 2;
  const long c = (long)(half * n + half);
  if (fabs(LL) < half - 1 && fabs(MM) < half - 1) {
    const long fl = fipref::floor_l(LL), cl = fipref::ceil_l(LL);
    const long fm = fipref::floor_l(MM), cm = fipref::ceil_l(MM);
    atomicAdd(&dst[c + fm * (long)n + fl], (1 - LL + fl) * (1 - MM + fm) * value);
    atomicAdd(&dst[c + cm * (long)n + fl], (1 - LL + fl) * (MM - fm) * value);
    atomicAdd(&dst[c + fm * (long)n + cl], (LL - fl) * (1 - MM + fm) * value);
    atomicAdd(&dst[c + cm * (long)n + cl], (LL - fl) * (MM - fm) * value);
  }
}

struct Acc {
  float s, sc, r, rc, m;
};

template <bool PRECISE>
__device__ __forceinline__ void acc_add(Acc& a, float d, float q) {
  if (!PRECISE) {
    a.s += d;
    a.r += q;
  } else {
    float t = a.s + d;
    a.sc += (fabsf(a.s) >= fabsf(d)) ? (a.s - t) + d : (d - t) + a.s;
    a.s = t;
    t = a.r + q;
    a.rc += (fabsf(a.r) >= fabsf(q)) ? (a.r - t) + q : (q - t) + a.r;
    a.r = t;
  }
  a.m = fmaxf(a.m, d);
}

template <bool PRECISE>
__device__ __forceinline__ void acc_pixel(Acc& a, float i1, float i2, float i3) {
  const float d = fabs(fabs(i1 - i2) - fabs(i2 - i3));
  const float s2 = (i2 <= 0) ? FIP_TRIGGER_FLOOR : i2;
  const float q = d / s2;
  acc_add<PRECISE>(a, d, fminf(q, 1.0f));  // NaN counts 1, as (q < 1) ? q : 1
}

// The warp's reduction of its lanes' tile statistics (valid in lane 0).
template <bool PRECISE>
__device__ __forceinline__ void warp_stats(Acc a, double& S, double& R, float& M) {
  if (!PRECISE) {
    for (int o = 16; o > 0; o >>= 1) {
      a.s += __shfl_xor_sync(0xffffffffu, a.s, o);
      a.r += __shfl_xor_sync(0xffffffffu, a.r, o);
      a.m = fmaxf(a.m, __shfl_xor_sync(0xffffffffu, a.m, o));
    }
    S = (double)a.s;
    R = (double)a.r;
  } else {
    double s = (double)a.s + (double)a.sc, r = (double)a.r + (double)a.rc;
    for (int o = 16; o > 0; o >>= 1) {
      s += __shfl_xor_sync(0xffffffffu, s, o);
      r += __shfl_xor_sync(0xffffffffu, r, o);
      a.m = fmaxf(a.m, __shfl_xor_sync(0xffffffffu, a.m, o));
    }
    S = s;
    R = r;
  }
  M = a.m;
}

// Statistics of one trigger tile (FIPkernels.cu:499-552 before the combine),
// one warp per T x T tile at base: S = sum d, R = sum min(d / I2', 1) (NaN
// counts as 1), M = max(0, max d), in the lanes' and shuffles' order (valid
// in lane 0).  Plain form: FP32 sums; precise form: Neumaier-compensated FP32
// sums combined in FP64.  L2: load through L2 only (data other SMs wrote in
// the same kernel).
template <bool PRECISE, bool L2>
__device__ __forceinline__ void tile_stats(const float* __restrict__ I1,
                                           const float* __restrict__ I2,
                                           const float* __restrict__ I3, size_t base, int n,
                                           int t, int vec, int lane, double& S, double& R,
                                           float& M) {
  auto ld4 = [](const float* p) {
    return L2 ? __ldcg(reinterpret_cast<const float4*>(p)) : *reinterpret_cast<const float4*>(p);
  };
  auto ld1 = [](const float* p) { return L2 ? __ldcg(p) : *p; };
  Acc a{0.f, 0.f, 0.f, 0.f, 0.f};
  if (vec) {
    const int q = t / 4;  // float4 per tile row
    for (int k = lane; k < t * q; k += 32) {
      const int r = k / q, c = (k % q) * 4;
      const size_t o = base + (size_t)r * n + c;
      const float4 x1 = ld4(I1 + o);
      const float4 x2 = ld4(I2 + o);
      const float4 x3 = ld4(I3 + o);
      acc_pixel<PRECISE>(a, x1.x, x2.x, x3.x);
      acc_pixel<PRECISE>(a, x1.y, x2.y, x3.y);
      acc_pixel<PRECISE>(a, x1.z, x2.z, x3.z);
      acc_pixel<PRECISE>(a, x1.w, x2.w, x3.w);
    }
  } else {
    for (int k = lane; k < t * t; k += 32) {
      const size_t o = base + (size_t)(k / t) * n + (k % t);
      acc_pixel<PRECISE>(a, ld1(I1 + o), ld1(I2 + o), ld1(I3 + o));
    }
  }
  warp_stats<PRECISE>(a, S, R, M);
}

// The tLISI of one tile from its statistics and the three image maxima
// (FIPkernels.cu:550): the plain form's FP32 expression, the precise form's
// FP64 one.
template <bool PRECISE>
__device__ __forceinline__ float tlisi_of(double S, double R, float M, const float max3[3], int t) {
  if (!PRECISE) {
    const float maxallval = max(max3[0], max(max3[1], max3[2]));
    const size_t us = (size_t)t;
    return 1 - ((float)S / us / us) * M * ((float)R / us / us) / maxallval / maxallval;
  }
  const double mx = fmax(fmax((double)max3[0], (double)max3[1]), (double)max3[2]);
  const double tt = (double)t;
  return (float)(1.0 - (S / tt / tt) * (double)M * (R / tt / tt) / mx / mx);
}

// The trigger fused into the reprojections of a three-snapshot call: the
// gather CTA that writes the last of the three images of its 64 x 64 region
// (a per-region count) computes the region's trigger-tile statistics, and a
// final one-pass kernel applies the maxima.
struct FipTriggerFuse {
  const float* img[3];  // I1, I2, I3
  unsigned* count;      // [gather tiles], zero at the call's start
  double* stats;        // [U*U][3]: S, R, M
  int t, u;
};

constexpr int kDT = 64;          // destination tile side
constexpr int kMaxRows = 256;    // candidate source rows per tile (one per thread)
static_assert(kMaxRows == kThreads, "the gather numbers rows one per thread");

// Exact map: LL = P1 - xi z / cell, MM = P2 + eta z / cell with
// z = 1 - sqrt(1 - rho), rho = cell^2 ((P1 - 1)^2 + (P2 - 1)^2),
// P = M (a, b) / |V22| -- the closed form of coordschange + p2p.
template <typename T>
struct ExactMap {
  T m00, m01, m10, m11;  // M / |V22|
  T i00, i01, i10, i11;  // its inverse
  T xi, eta, cell;
};

template <typename T>
__device__ __forceinline__ ExactMap<T> make_map(const float* V, float cell) {
  ExactMap<T> m;
  const double a22 = fabs((double)V[8]);
  const double m00 = -(double)V[0] / a22, m01 = (double)V[3] / a22;
  const double m10 = -(double)V[1] / a22, m11 = (double)V[4] / a22;
  const double det = m00 * m11 - m01 * m10;
  m.m00 = (T)m00; m.m01 = (T)m01; m.m10 = (T)m10; m.m11 = (T)m11;
  m.i00 = (T)(m11 / det); m.i01 = (T)(-m01 / det);
  m.i10 = (T)(-m10 / det); m.i11 = (T)(m00 / det);
  m.xi = (T)((double)V[6] / (double)V[8]);
  m.eta = (T)((double)V[7] / (double)V[8]);
  m.cell = (T)cell;
  return m;
}

// The same map in FP32 arithmetic throughout (three reciprocals): for the
// gather's candidate bounds, whose margins (a quarter pixel at least) dwarf
// its rounding (~1e-4 pixel at 4096^2).
__device__ __forceinline__ ExactMap<float> make_map_f32(const float* V, float cell) {
  ExactMap<float> m;
  const float ia = 1.0f / fabsf(V[8]), iv = 1.0f / V[8];
  m.m00 = -V[0] * ia;
  m.m01 = V[3] * ia;
  m.m10 = -V[1] * ia;
  m.m11 = V[4] * ia;
  const float idet = 1.0f / (m.m00 * m.m11 - m.m01 * m.m10);
  m.i00 = m.m11 * idet;
  m.i01 = -m.m01 * idet;
  m.i10 = -m.m10 * idet;
  m.i11 = m.m00 * idet;
  m.xi = V[6] * iv;
  m.eta = V[7] * iv;
  m.cell = cell;
  return m;
}

template <typename T>
__device__ __forceinline__ T slant_over_cell(const ExactMap<T>& m, T P1, T P2) {
  const T rho = m.cell * m.cell * ((P1 - 1) * (P1 - 1) + (P2 - 1) * (P2 - 1));
  return rho <= 1 ? (rho / (1 + sqrt(1 - rho))) / m.cell : (T)0;
}

// FP32, for the gather's candidate bounds only: rsqrtf and __fdividef (a few
// ulp), whose rounding the bounds' margins dwarf.
__device__ __forceinline__ float slant_over_cell(const ExactMap<float>& m, float P1, float P2) {
  const float rho = m.cell * m.cell * ((P1 - 1) * (P1 - 1) + (P2 - 1) * (P2 - 1));
  if (!(rho <= 1.f)) return 0.f;
  const float u = 1.f - rho;
  const float s = u > 0.f ? u * rsqrtf(u) : 0.f;
  return __fdividef(rho, m.cell * (1.f + s));
}

template <typename T>
__device__ __forceinline__ void exact_forward(const ExactMap<T>& m, T a, T b, T& LL, T& MM) {
  const T P1 = m.m00 * a + m.m01 * b, P2 = m.m10 * a + m.m11 * b;
  const T zc = slant_over_cell(m, P1, P2);
  LL = P1 - m.xi * zc;
  MM = P2 + m.eta * zc;
}

// Source (a, b), relative to the centre, of an exact target (LL, MM):
// fixed-point iteration on the slant term, a contraction wherever the map
// does not fold (the slant part's Jacobian determinant stays positive); it
// runs until the step is below 1e-3 pixel (or 128 steps).  Returns how far
// the forward map of the result lands from (LL, MM), in pixels.
template <typename T>
__device__ __forceinline__ T exact_inverse(const ExactMap<T>& m, T LL, T MM, T& a, T& b) {
  T P1 = LL, P2 = MM;
  for (int it = 0; it < 128; ++it) {
    const T zc = slant_over_cell(m, P1, P2);
    const T q1 = LL + m.xi * zc, q2 = MM - m.eta * zc;
    const T step = fmax(fabs(q1 - P1), fabs(q2 - P2));
    P1 = q1;
    P2 = q2;
    if (step <= (T)1e-3) break;
  }
  a = m.i00 * P1 + m.i01 * P2;
  b = m.i10 * P1 + m.i11 * P2;
  T L2, M2;
  exact_forward(m, a, b, L2, M2);
  return fmax(fabs(L2 - LL), fabs(M2 - MM));
}

// The exact map around a per-tile origin (a0, b0) of source offsets, for the
// precision form's splats.  With Q = P - 1 the vector whose squared length,
// times cell^2, is rho, and Q0 its value at the origin, a source d = M (a -
// a0, b - b0) away has
//   rho - rho0 = cell^2 g,   g = 2 Q0.d + d.d,
//   z(rho) - z(rho0) = cell g / (sqrt(1 - rho0) + sqrt(1 - rho))
// (z = slant over cell), so its target relative to the destination tile is
//   L = l0 + d1 - xi dz,  M = m0 + d2 + eta dz,
// with l0, m0 the origin's target in tile coordinates (FP64).  Every FP32
// quantity is then a tile-sized offset or a relative correction: rsqrtf and
// __fdividef (a few ulp) move a target by ~1e-5 pixel, well inside the
// FP64 tolerance, where the slant term in absolute form rounds at its own
// magnitude (hundreds of pixels on wide fields).  Beyond the horizon
// (rho > 1) the slant term is 0, as in the closed form; the relative form
// needs the origin inside it, which every tile in the gather's domain has.
struct TileMap {
  float m00, m01, m10, m11;  // M / |V22|
  float xi, eta, cell, c2;   // c2 = cell^2
  float q1, q2;              // 2 Q0
  float u0, s0, z0;          // 1 - rho0, its square root, the slant term at the origin
  float l0, m0;              // the origin's target relative to the tile's corner
  int a0, b0;
};

__device__ __forceinline__ TileMap tile_map(const ExactMap<double>& md, const float (*q)[2],
                                            int seg, int cl, int rl) {
  TileMap t;
  // Origin: the rounded mean of the preimage polygon's four corners.
  t.a0 = (int)rintf(0.25f * (q[0][0] + q[seg][0] + q[2 * seg][0] + q[3 * seg][0]));
  t.b0 = (int)rintf(0.25f * (q[0][1] + q[seg][1] + q[2 * seg][1] + q[3 * seg][1]));
  const double P1 = md.m00 * t.a0 + md.m01 * t.b0, P2 = md.m10 * t.a0 + md.m11 * t.b0;
  const double Q1 = P1 - 1.0, Q2 = P2 - 1.0;
  const double rho = md.cell * md.cell * (Q1 * Q1 + Q2 * Q2);
  const double u0 = 1.0 - rho;
  const double s0 = u0 > 0.0 ? sqrt(u0) : 0.0;
  const double z0 = rho <= 1.0 ? (rho / (1.0 + s0)) / md.cell : 0.0;
  t.m00 = (float)md.m00; t.m01 = (float)md.m01; t.m10 = (float)md.m10; t.m11 = (float)md.m11;
  t.xi = (float)md.xi; t.eta = (float)md.eta;
  t.cell = (float)md.cell; t.c2 = (float)(md.cell * md.cell);
  t.q1 = (float)(2.0 * Q1); t.q2 = (float)(2.0 * Q2);
  t.u0 = (float)u0; t.s0 = (float)s0; t.z0 = (float)z0;
  t.l0 = (float)(P1 - md.xi * z0 - (double)cl);
  t.m0 = (float)(P2 + md.eta * z0 - (double)rl);
  return t;
}

// Target (L, M), relative to the tile's corner, of the source at offsets
// (a, b) from the image centre.
__device__ __forceinline__ void tile_target(const TileMap& t, int a, int b, float& L, float& M) {
  const float da = (float)(a - t.a0), db = (float)(b - t.b0);
  const float d1 = t.m00 * da + t.m01 * db, d2 = t.m10 * da + t.m11 * db;
  const float g = d1 * (t.q1 + d1) + d2 * (t.q2 + d2);
  const float u = t.u0 - t.c2 * g;
  float dz = -t.z0;
  if (u >= 0.f) {
    const float s = u > 0.f ? u * rsqrtf(u) : 0.f;
    dz = __fdividef(t.cell * g, t.s0 + s);
  }
  L = t.l0 + d1 - t.xi * dz;
  M = t.m0 + d2 + t.eta * dz;
}

// Destination-tile-major reprojection.  The candidate source pixels of a
// 64x64 destination tile are the integer points of the preimage of the tile
// widened by the splat reach (1 pixel) and delta (the FP32 chain's deviation
// from the exact map): per source row, one column interval.  Each candidate
// is splatted (bilinear weights of FIPkernels.cu:394-410) into shared memory;
// the tile is stored once and its maximum folded into *img_max.
// EXACT: targets from the closed form (precision form), in FP32 relative to
// a per-tile origin whose terms are FP64 (TileMap), instead of the
// precomputed reference-chain targets.
// The shared tile carries an apron of kAp pixels on every side, so the four
// pixels of any candidate's splat land inside it without per-pixel checks
// (apron pixels belong to the neighbouring tiles, which splat them
// themselves, and are dropped at the commit).  Its row stride is odd, so the
// lanes of a warp (neighbouring sources, mapped along an arbitrary
// direction) fall on distinct banks down a column as well as along a row.
constexpr int kAp = 4;
constexpr int kTW = kDT + 2 * kAp;  // tile side with the apron
constexpr int kTR = kTW + 1;        // row stride
// The preimage of a tile's boundary is sampled at kSeg points per edge: a
// polygon of kPoly vertices, whose chords stay within a small curvature
// margin of the true preimage even for strongly tilted wide fields.
constexpr int kSeg = 2;
constexpr int kPoly = 4 * kSeg;
static_assert(kPoly <= 32 && (kPoly & (kPoly - 1)) == 0, "one warp's lanes, a power of two");

template <bool EXACT>
__global__ void __launch_bounds__(kThreads, EXACT ? 5 : 8) k_reproject_gather(
    const float* __restrict__ pre, const float2* __restrict__ tg, const float* __restrict__ V,
    int n, int nb, float cell, float delta, const unsigned* __restrict__ pre_max,
    float* __restrict__ dst, unsigned* img_max, unsigned* err, const FipTriggerFuse fuse) {
  __shared__ __align__(16) unsigned s_tile[kTW * kTR];
  __shared__ int s_base[kMaxRows];  // pixel index of row r's first candidate minus its number
  __shared__ int s_off[kMaxRows + 1];
  __shared__ int s_wsum[kThreads / 32];
  __shared__ float s_q[kPoly][2];
  __shared__ float s_wmax[kThreads / 32];

  const int tiles = (n + kDT - 1) / kDT;
  const int tr = blockIdx.x / tiles, tc = blockIdx.x % tiles;
  const int r0 = tr * kDT, c0 = tc * kDT;
  const int h = n / 2;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  static_assert((kTW * kTR) % 4 == 0, "the tile is zeroed in 16-byte stores");
  for (int k = threadIdx.x; k < kTW * kTR / 4; k += kThreads)
    reinterpret_cast<uint4*>(s_tile)[k] = make_uint4(0u, 0u, 0u, 0u);
  // Precision form: the FP64 map, formed once per CTA by a lane of warp 1
  // while warp 0 traces the preimage, and turned into the tile's FP32
  // constants (TileMap) by one thread after the barrier.
  __shared__ ExactMap<double> s_md;
  __shared__ TileMap s_tm;
  if (EXACT && threadIdx.x == 32) s_md = make_map<double>(V, cell);
  // Preimage of the tile's boundary, widened by the splat reach and delta:
  // kPoly points, kSeg per edge, in order around it (lanes of warp 0), the
  // tile's domain check and its curvature margin.
  __shared__ float s_sag, s_bmin, s_bmax, s_parea;
  if (warp == 0) {
    const ExactMap<float> mf = make_map_f32(V, cell);
    const float Llo = (float)(c0 - h) - 1.0f - delta, Lhi = (float)(c0 + kDT - h) + delta;
    const float Mlo = (float)(r0 - h) - 1.0f - delta, Mhi = (float)(r0 + kDT - h) + delta;
    float a = 0.f, b = 0.f, res = 0.f, r2 = 0.f, det = 1.f;
    if (lane < kPoly) {
      // Corners (Llo, Mlo), (Lhi, Mlo), (Lhi, Mhi), (Llo, Mhi); point s of
      // edge e lies s / kSeg of the way from corner e to corner e + 1.
      const int e = lane / kSeg, sg = lane % kSeg;
      const float Le = (e == 0 || e == 3) ? Llo : Lhi, Me = (e < 2) ? Mlo : Mhi;
      const int e1 = (e + 1) & 3;
      const float Ln = (e1 == 0 || e1 == 3) ? Llo : Lhi, Mn = (e1 < 2) ? Mlo : Mhi;
      const float w = (float)sg * (1.0f / (float)kSeg);
      const float L = Le + (Ln - Le) * w, M = Me + (Mn - Me) * w;
      res = exact_inverse(mf, L, M, a, b);
      s_q[lane][0] = a;
      s_q[lane][1] = b;
      // Sky offset (X, Y) in radians of the source point, held inside the
      // source image (the candidates are, too), and the slant part's Jacobian
      // determinant there: 1 - xi X / n + eta Y / n, n = sqrt(1 - r2).
      const float lim = (float)h + 2.0f;
      const float ac = fminf(fmaxf(a, -lim), lim), bc = fminf(fmaxf(b, -lim), lim);
      const float X = cell * (mf.m00 * ac + mf.m01 * bc - 1.0f);
      const float Y = cell * (mf.m10 * ac + mf.m11 * bc - 1.0f);
      r2 = X * X + Y * Y;
      const float nn = sqrtf(fmaxf(1.0f - r2, 1e-6f));
      det = 1.0f - mf.xi * X / nn + mf.eta * Y / nn;
    }
    // Row range and shoelace area of the polygon, reduced over its lanes.
    float bmn = lane < kPoly ? b : 3e38f, bmx = lane < kPoly ? b : -3e38f;
    const int nxt = (lane + 1) % kPoly;
    const float an = __shfl_sync(0xffffffffu, a, nxt), bn = __shfl_sync(0xffffffffu, b, nxt);
    float area = lane < kPoly ? a * bn - an * b : 0.f;
#pragma unroll
    for (int o = 1; o < kPoly; o <<= 1) {
      res = fmaxf(res, __shfl_xor_sync(0xffffffffu, res, o));
      r2 = fmaxf(r2, __shfl_xor_sync(0xffffffffu, r2, o));
      det = fminf(det, __shfl_xor_sync(0xffffffffu, det, o));
      bmn = fminf(bmn, __shfl_xor_sync(0xffffffffu, bmn, o));
      bmx = fmaxf(bmx, __shfl_xor_sync(0xffffffffu, bmx, o));
      area += __shfl_xor_sync(0xffffffffu, area, o);
    }
    if (lane == 0) {
      // The candidate bounds hold while the inverse converged, the tile lies
      // well inside the horizon (r2 < 0.98) and the map does not fold
      // (det > 1/4); a tile outside that domain is reported, not skipped.
      if (err && !(res < 0.05f && r2 < 0.98f && det > 0.25f)) atomicOr(err, 1u);
      // The preimage's edges bow away from the chords between its points
      // by at most ell^2 / 8 times the slant term's second derivative
      // (|(xi, eta)| cell / n^3, divided by det for the inverse), ell the
      // length of one segment: widen the candidate intervals by that (with a
      // 20 % allowance).
      const float nn = sqrtf(fmaxf(1.0f - r2, 0.02f));
      const float ell = ((float)kDT + 2.0f + 2.0f * delta) * (1.0f / (float)kSeg);
      s_sag = 0.15f * hypotf(mf.xi, mf.eta) * cell * ell * ell /
              (nn * nn * nn * fmaxf(det, 0.25f));
      s_bmin = bmn;
      s_bmax = bmx;
      s_parea = fabsf(0.5f * area);
    }
  }
  __syncthreads();
  const float bmin = s_bmin, bmax = s_bmax;
  const float sag = s_sag + 1e-3f;
  const int jlo = (int)fmaxf(0.f, ceilf(fmaxf(bmin + h - sag, -1.f)));
  const int jhi = (int)fminf((float)(n - 1), floorf(fminf(bmax + h + sag, (float)n)));
  const float inv_nb = 1.0f / static_cast<float>(nb);
  const size_t half = n / 2;
  const float lim = half - 1;  // the reference compares |LL| with size_t (N/2 - 1)
  // A candidate that reaches the tile has LL in [c0 - h - 1, c0 - h + kDT)
  // (MM likewise): for tiles at least two pixels inside that range check on
  // both axes, every such candidate passes it, and a candidate that would fail
  // it lands beyond the tile, so the check is left out there.
  const bool inner = c0 >= 4 && c0 + kDT + 4 <= 2 * h && r0 >= 4 && r0 + kDT + 4 <= 2 * h;
  // Fixed-point tile sums: a source's splat value v / nb is carried as
  // v * 2^(28 - sh) / max(pre).  Every contribution is <= 2^(28 - sh), and
  // the bilinear weights landing on one pixel sum to about the density of
  // sources per destination pixel (four times it at most), so the sums stay
  // below 2^32 while that density is <= 2^(2 + sh): the shared-memory sums
  // are native integer atomics, exact and independent of their order, and
  // the tile is converted back once.  sh is 0 (resolution 2^-28 of the image
  // maximum) unless the preimage of the tile, with its margins, covers more
  // than twice the tile's area -- a map that contracts, which only very wide
  // fields with a tilted plane reach -- and then grows by one per doubling.
  const float parea = s_parea;  // preimage polygon's area (shoelace)
  int sh = 0;
  while (sh < 12 && parea > (float)(2 * kDT * kDT) * (float)(1 << sh)) ++sh;
  const float pmax = __uint_as_float(*pre_max);
  const float qk = pmax > 0.f ? 268435456.0f / (pmax * (float)(1 << sh)) : 0.f;
  const float deq = pmax * inv_nb * ((float)(1 << sh) / 268435456.0f);
  // Precision form: the tile's constants, from FP64 by a thread of the last
  // warp (idle in the row-interval step unless a chunk has 256 rows); every
  // thread reads them after the chunk's barriers, before its first splat.
  if (EXACT && threadIdx.x == kThreads - 1) s_tm = tile_map(s_md, s_q, kSeg, c0 - h, r0 - h);
  TileMap tm;
  auto splat = [&](int i, int j, float vq, float2 t) {
    int fl, fm;
    float wl1, wm1, wl0, wm0;
    if (!EXACT) {
      const float LL = t.x, MM = t.y;
      if (!inner && !(fabsf(LL) < lim && fabsf(MM) < lim)) return;
      const float flf = floorf(LL), fmf = floorf(MM);
      // The reference's weight expressions (FIPkernels.cu:397-409).  Its far
      // pixel is ceil(LL), equal to floor(LL) + 1 except on exact integers,
      // where the far weight LL - floor(LL) is 0: splatting the far weight at
      // floor + 1 adds the same sums.
      wl0 = 1 - LL + flf; wl1 = LL - flf;
      wm0 = 1 - MM + fmf; wm1 = MM - fmf;
      fl = (int)flf + (h - c0);
      fm = (int)fmf + (h - r0);
    } else {
      float Lr, Mr;
      tile_target(tm, i - h, j - h, Lr, Mr);
      if (!inner && !(fabsf(Lr + (float)(c0 - h)) < lim && fabsf(Mr + (float)(r0 - h)) < lim))
        return;
      const float flr = floorf(Lr), fmr = floorf(Mr);
      fl = (int)flr;
      fm = (int)fmr;
      wl1 = Lr - flr; wm1 = Mr - fmr;
      wl0 = 1.0f - wl1; wm0 = 1.0f - wm1;
    }
    // Pixels (fm|fm+1, fl|fl+1), local to the tile with its apron.  A splat
    // that reaches the tile lies inside the apron (fl, fm >= -1); one that
    // does not touches no pixel of the tile and is skipped.
    fl += kAp;
    fm += kAp;
    if ((unsigned)fl > (unsigned)(kTW - 2) || (unsigned)fm > (unsigned)(kTW - 2)) return;
    const float a = wl0 * vq, b = wl1 * vq;
    unsigned* px = &s_tile[fm * kTR + fl];
    atomicAdd(px, __float2uint_rn(a * wm0));
    atomicAdd(px + 1, __float2uint_rn(b * wm0));
    atomicAdd(px + kTR, __float2uint_rn(a * wm1));
    atomicAdd(px + kTR + 1, __float2uint_rn(b * wm1));
  };
  // Candidate rows in chunks of kMaxRows (one row per thread): a single
  // chunk unless the preimage spans more than kMaxRows source rows.
  for (int cj = jlo; cj <= jhi; cj += kMaxRows) {
    const int nrows = min(kMaxRows, jhi - cj + 1);
    // Column interval of every candidate row (the preimage quadrilateral
    // intersected with the row), one row per thread, and the exclusive prefix
    // of the interval lengths: candidates are then numbered 0 .. total-1 row by
    // row, so every warp step splats 32 candidates whatever the row lengths.
    int cnt = 0, ilo = 0;
    {
      const int r = threadIdx.x;
      if (r < nrows) {
        // Rows in the margin beyond the quadrilateral's extreme corners take
        // the interval at that corner (then widened like every interval).
        const float b = fminf(fmaxf((float)(cj + r - h), bmin), bmax);
        float alo = 3e38f, ahi = -3e38f;
#pragma unroll
        for (int k = 0; k < kPoly; ++k) {
          const float ax = s_q[k][0], bx = s_q[k][1];
          const float ay = s_q[(k + 1) % kPoly][0], by = s_q[(k + 1) % kPoly][1];
          if ((bx <= b && b <= by) || (by <= b && b <= bx)) {
            if (by == bx) {
              alo = fminf(alo, fminf(ax, ay));
              ahi = fmaxf(ahi, fmaxf(ax, ay));
            } else {
              const float a = ax + (ay - ax) * ((b - bx) / (by - bx));
              alo = fminf(alo, a);
              ahi = fmaxf(ahi, a);
            }
          }
        }
        int ihi = -1;
        if (alo <= ahi) {
          ilo = (int)fmaxf(0.f, ceilf(fmaxf(alo + h - sag, -1.f)));
          ihi = (int)fminf((float)(n - 1), floorf(fminf(ahi + h + sag, (float)n)));
        }
        cnt = ihi >= ilo ? ihi - ilo + 1 : 0;
      }
      int inc = cnt;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
      }
      if (lane == 31) s_wsum[warp] = inc;
      __syncthreads();
      int wbase = 0;
      for (int w = 0; w < warp; ++w) wbase += s_wsum[w];
      if (r < kMaxRows) {
        s_off[r] = wbase + inc - cnt;
        // Candidate f of row r is pixel (cj + r) n + ilo + (f - off): s_base + f
        // (< N^2 <= 2^30 for image_size <= 32768).
        s_base[r] = (cj + r) * n + ilo - (wbase + inc - cnt);
      }
      if (r == kThreads - 1) s_off[kMaxRows] = wbase + inc;
    }
    __syncthreads();
    const int total = s_off[kMaxRows];
    if (EXACT) tm = s_tm;
    // Rows past nrows have no candidates: their offsets equal total.
    // Each warp takes a contiguous eighth of the candidates, so a lane's row
    // cursor moves about half a row per candidate; its start is found by
    // bisection of the row offsets.  Warp step: candidates f0 + lane + 32 e,
    // e < 4, all loads issued first; the cursor only moves forward.
    constexpr int kPer = 4, kWarps = kThreads / 32;
    const int per = (total + kWarps - 1) / kWarps;
    const int wb = min(total, warp * per), we = min(total, wb + per);
    int row = 0;
    for (int step = kMaxRows / 2; step > 0; step >>= 1)
      if (s_off[row + step] <= wb) row += step;  // last row whose offset is <= wb
    for (int f0 = wb; f0 < we; f0 += 32 * kPer) {
      int at[kPer], rw[kPer];
      float p[kPer];
      float2 tt[kPer];
#pragma unroll
      for (int e = 0; e < kPer; ++e) {
        const int f = f0 + lane + 32 * e;
        rw[e] = -1;
        if (f < we) {
          while (s_off[row + 1] <= f) ++row;
          rw[e] = row;
          at[e] = s_base[row] + f;
          p[e] = pre[at[e]];
          if (!EXACT) tt[e] = tg[at[e]];
        }
      }
#pragma unroll
      for (int e = 0; e < kPer; ++e) {
        if (rw[e] < 0) continue;
        const int j = cj + rw[e];
        splat(at[e] - j * n, j, p[e] * qk, EXACT ? make_float2(0.f, 0.f) : tt[e]);
      }
    }
    __syncthreads();  // the next chunk rewrites the row offsets
  }
  float vmax = 0.f;
  for (int k = threadIdx.x; k < kDT * kDT / 4; k += kThreads) {
    const int lr = (4 * k) / kDT, g4 = ((4 * k) % kDT) >> 2;
    const int rr = r0 + lr, cc = c0 + 4 * g4;
    const unsigned* src = &s_tile[(lr + kAp) * kTR + kAp + 4 * g4];
    const uint4 q = make_uint4(src[0], src[1], src[2], src[3]);
    const float4 val = make_float4((float)q.x * deq, (float)q.y * deq, (float)q.z * deq,
                                   (float)q.w * deq);
    if (rr < n) {
      if (cc + 3 < n && (n & 3) == 0) {
        *reinterpret_cast<float4*>(&dst[(size_t)rr * n + cc]) = val;
        vmax = fmaxf(vmax, fmaxf(fmaxf(val.x, val.y), fmaxf(val.z, val.w)));
      } else {
        const float vv[4] = {val.x, val.y, val.z, val.w};
        for (int e = 0; e < 4; ++e)
          if (cc + e < n) {
            dst[(size_t)rr * n + cc + e] = vv[e];
            vmax = fmaxf(vmax, vv[e]);
          }
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
  if (lane == 0) s_wmax[warp] = vmax;
  __syncthreads();
  if (threadIdx.x == 0 && img_max) {
    float b = 0.f;
    for (int w = 0; w < kThreads / 32; ++w) b = fmaxf(b, s_wmax[w]);
    atomicMax(img_max, __float_as_uint(b));
  }
  if (fuse.count) {
    // Fused trigger: every thread's stores made visible device-wide, then one
    // count per region; the CTA that completes the region's third image
    // reads all three through L2 and reduces each trigger tile in it.
    __shared__ unsigned s_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
      const unsigned old = atomicAdd(&fuse.count[blockIdx.x], 1u);
      s_last = old == 2u;
      __threadfence();
    }
    __syncthreads();
    if (s_last) {
      const int per = kDT / fuse.t;
      const int vec = (fuse.t % 4 == 0) && (n % 4 == 0);
      for (int k = warp; k < per * per; k += kThreads / 32) {
        const int ti = r0 / fuse.t + k / per, tj = c0 / fuse.t + k % per;
        const size_t base = (size_t)ti * fuse.t * n + (size_t)tj * fuse.t;
        double S, R;
        float M;
        tile_stats<EXACT, true>(fuse.img[0], fuse.img[1], fuse.img[2], base, n, fuse.t, vec,
                                lane, S, R, M);
        if (lane == 0) {
          double* o = fuse.stats + 3 * ((size_t)ti * fuse.u + tj);
          o[0] = S;
          o[1] = R;
          o[2] = (double)M;
        }
      }
    }
  }
}

// mode 0: the FP32 chain with the theta table (null: evaluated), 2: the
// chain evaluated, 1: the exact closed form.
__global__ void k_pixel_targets(const float* __restrict__ V, int n, float dc, float cell,
                                int mode, const float2* __restrict__ ttab,
                                float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= n) return;
  float LL, MM;
  if (mode != 1) {
    fipref::Frame fr{V[0], V[1], V[3], V[4], V[8], V[6], V[7], dc};
    fipref::pixel_target(fr, i, j, n, LL, MM, mode == 0 ? ttab : nullptr);
  } else {
    const ExactMap<double> m = make_map<double>(V, cell);
    double Ld, Md;
    exact_forward(m, (double)(i - n / 2), (double)(j - n / 2), Ld, Md);
    LL = (float)Ld;
    MM = (float)Md;
  }
  out[2 * ((size_t)j * n + i)] = LL;
  out[2 * ((size_t)j * n + i) + 1] = MM;
}

// Maximum of non-negative floats (bit-pattern order), NaN ignored.
__global__ void k_image_max(const float* __restrict__ img, size_t count, unsigned* out) {
  float m = 0.f;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < count;
       k += (size_t)gridDim.x * blockDim.x)
    m = fmaxf(m, img[k]);
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

// ---------------------------------------------------------------------------
// Trigger (FIPkernels.cu:415-552, 831-840).  One warp per T x T tile:
// D = | |I1-I2| - |I2-I3| |, I2 clamped to C after D, S = sum D,
// M = max(0, max D), R = sum min(D/I2c, 1) (NaN counts 1).
// PRECISE: Neumaier-compensated S and R, FP64 combine.
// ---------------------------------------------------------------------------
template <bool PRECISE>
__global__ void __launch_bounds__(kThreads) k_trigger(const float* __restrict__ I1,
                                                      const float* __restrict__ I2,
                                                      const float* __restrict__ I3,
                                                      const float* __restrict__ m1,
                                                      const float* __restrict__ m2,
                                                      const float* __restrict__ m3, int n,
                                                      int t, int u, int vec,
                                                      float* __restrict__ result,
                                                      size_t img_stride, size_t res_stride) {
  // Batched launches: triple blockIdx.y is images y, y+1, y+2 of a linear ring
  // (stride img_stride) with maxima m1[y], m2[y], m3[y].
  I1 += blockIdx.y * img_stride;
  I2 += blockIdx.y * img_stride;
  I3 += blockIdx.y * img_stride;
  const float max3[3] = {m1[blockIdx.y], m2[blockIdx.y], m3[blockIdx.y]};
  result += blockIdx.y * res_stride;
  const int lane = threadIdx.x & 31;
  const int b = blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5);
  if (b >= u * u) return;
  const int ti = b / u, tj = b % u;
  const size_t base = (size_t)ti * t * n + (size_t)tj * t;
  double S, R;
  float M;
  tile_stats<PRECISE, false>(I1, I2, I3, base, n, t, vec, lane, S, R, M);
  if (lane == 0) result[b] = tlisi_of<PRECISE>(S, R, M, max3, t);
}

// ---------------------------------------------------------------------------
// Sliding-window trigger streamed through registers: tLISI of triples
// (k, k+1, k+2) over a linear ring of images.  A warp owns one trigger tile
// and a chunk of consecutive triples; each lane keeps its float4s of the
// last three slices in registers and loads the next slice's while it
// reduces the current triple, so every image of the chunk is read from HBM
// once instead of once per triple it is in.  Lane k's float4s and the
// accumulation and shuffle order are k_trigger's (bit-identical results).
// NV: float4s per lane, >= T*T/128.
// ---------------------------------------------------------------------------
constexpr int kStreamThreads = 128;

template <bool PRECISE, int NV>
__global__ void __launch_bounds__(kStreamThreads) k_trigger_stream(
    const float* __restrict__ images, size_t img_stride, int count, int chunk,
    const float* __restrict__ maxima, int n, int t, int u, float* __restrict__ result) {
  const int lane = threadIdx.x & 31;
  const int b = blockIdx.x * (kStreamThreads / 32) + (threadIdx.x >> 5);
  if (b >= u * u) return;
  const int y0 = blockIdx.y * chunk, y1 = min(count, y0 + chunk);
  const int q = t / 4, nv = t * q;  // float4s per tile row, per tile
  const float* base = images + (size_t)(b / u) * t * n + (size_t)(b % u) * t;
  unsigned off[NV];
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    const int k = lane + 32 * i;
    off[i] = (unsigned)((k / q) * n + (k % q) * 4);
  }
  auto load = [&](float4(&v)[NV], int sl) {
    const float* img = base + (size_t)sl * img_stride;
#pragma unroll
    for (int i = 0; i < NV; ++i)
      if (lane + 32 * i < nv) v[i] = __ldcs(reinterpret_cast<const float4*>(img + off[i]));
  };
  // Triple y from slices (P0, P1, P2); slice y + 3 is loaded into NX first
  // so that its latency hides behind the reduction.
  auto step = [&](float4(&P0)[NV], float4(&P1)[NV], float4(&P2)[NV], float4(&NX)[NV], int y) {
    if (y + 1 < y1) load(NX, y + 3);
    Acc a{0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int i = 0; i < NV; ++i)
      if (lane + 32 * i < nv) {
        acc_pixel<PRECISE>(a, P0[i].x, P1[i].x, P2[i].x);
        acc_pixel<PRECISE>(a, P0[i].y, P1[i].y, P2[i].y);
        acc_pixel<PRECISE>(a, P0[i].z, P1[i].z, P2[i].z);
        acc_pixel<PRECISE>(a, P0[i].w, P1[i].w, P2[i].w);
      }
    double S, R;
    float M;
    warp_stats<PRECISE>(a, S, R, M);
    if (lane == 0) {
      const float max3[3] = {maxima[y], maxima[y + 1], maxima[y + 2]};
      result[(size_t)y * u * u + b] = tlisi_of<PRECISE>(S, R, M, max3, t);
    }
  };
  // Four slice buffers whose roles rotate with the triple (no copies).
  float4 s0[NV], s1[NV], s2[NV], s3[NV];
  load(s0, y0);
  load(s1, y0 + 1);
  load(s2, y0 + 2);
  for (int y = y0; y < y1; y += 4) {
    step(s0, s1, s2, s3, y);
    if (y + 1 >= y1) break;
    step(s1, s2, s3, s0, y + 1);
    if (y + 2 >= y1) break;
    step(s2, s3, s0, s1, y + 2);
    if (y + 3 >= y1) break;
    step(s3, s0, s1, s2, y + 3);
  }
}

// Final pass of the fused trigger: tLISI from the statistics and the maxima.
template <bool PRECISE>
__global__ void k_trigger_combine(const double* __restrict__ stats, const float* __restrict__ max3p,
                                  int u, int t, float* __restrict__ result) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= u * u) return;
  const float max3[3] = {max3p[0], max3p[1], max3p[2]};
  result[b] = tlisi_of<PRECISE>(stats[3 * b], stats[3 * b + 1], (float)stats[3 * b + 2], max3, t);
}

inline float cell_degrees(float cell) { return (float)((double)cell / FIP_M_PI * 180); }

inline int sm_count() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

}  // namespace

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------

bool fip_fft_plan(int g, fipfft::Plan& p, int values_per_thread) {
  if (g < 48 || g % 3 != 0) return false;
  const int m = g / 3;
  if (m & (m - 1)) return false;
  int lm = 0;
  while ((1 << lm) < m) ++lm;
  // Instantiated: 8 values per thread for M = 2^4..2^11, 16 for 2^5..2^12
  // (<= 768 threads).  Default: 8 up to M = 1024 (N = 2048), 16 beyond -- at
  // M = 2048 the 16-value row pass takes about two thirds of the 8-value one's
  // time on B200, and the autotuner picks it there.
  int le = (lm <= 10) ? 3 : 4;
  if (values_per_thread == 8) le = 3;
  if (values_per_thread == 16) le = 4;
  if (le == 3 && (lm < 4 || lm > 11)) return false;
  if (le == 4 && (lm < 5 || lm > 12)) return false;
  p.g = g;
  p.m = m;
  p.lm = lm;
  p.le = le;
  p.e = 1 << le;
  p.nt = 3 * (m >> le);
  p.split = 0;
  p.direct = 0;
  return true;
}

cudaError_t fip_launch_taper(float* taper, const FipGeom& geo, cudaStream_t s) {
  const int cnt = geo.n / 2 + 1;
  k_taper<<<(cnt + kThreads - 1) / kThreads, kThreads, 0, s>>>(taper, (size_t)geo.n,
                                                                (size_t)geo.g);
  return cudaGetLastError();
}

int fip_bin_launches(const FipGeom&) { return 3; }

cudaError_t fip_launch_bin(const FipGeom& geo, const float* B, int nb, FipBins& bins,
                           cudaStream_t s) {
  const int ntiles = geo.tiles_r * geo.tiles_c;
  const float scale = geo.cell * (float)(size_t)geo.g;  // r1r2_scale (FIPkernels.cu:584)
  cudaError_t e = cudaMemsetAsync(bins.count, 0, ntiles * sizeof(unsigned), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(bins.bbox, 0, 4 * sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  if (ntiles <= kMaxSmemTiles) {
    const int cta = max(1, min(8 * sm_count(), (nb + kBinThreads - 1) / kBinThreads));
    const int per_cta = (nb + cta - 1) / cta;
    const size_t smem = (size_t)ntiles * sizeof(unsigned);
    if (nb > 0)
      k_bin_count<<<cta, kBinThreads, smem, s>>>(B, nb, per_cta, scale, geo.g, geo.tiles_c,
                                                  ntiles, bins.count, bins.bbox);
    const size_t scan_smem = (2 * (size_t)ntiles + 1) * sizeof(unsigned);
    cudaError_t ea = cudaFuncSetAttribute(k_bin_scan_tiles,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)((2 * (size_t)kMaxSmemTiles + 1) * sizeof(unsigned)));
    if (ea != cudaSuccess) return ea;
    k_bin_scan_tiles<<<1, kScanThreads, scan_smem, s>>>(bins.count, bins.bbox, ntiles, geo.tiles_c,
                                                    geo.g, geo.layout, bins.offset, bins.cursor,
                                                    bins.work, bins.nwork, (int)bins.wcap,
                                                    bins.multi, bins.nmulti);
    if (nb > 0)
      k_bin_scatter<<<cta, kBinThreads, smem, s>>>(B, nb, per_cta, scale, geo.g, geo.tiles_c,
                                                    ntiles, bins.offset, bins.cursor,
                                                    bins.entries);
    return cudaGetLastError();
  }
  const int blocks = (nb + kThreads - 1) / kThreads;
  if (nb > 0)
    k_bin<0><<<blocks, kThreads, 0, s>>>(B, nb, scale, geo.g, geo.tiles_c, bins.count, nullptr,
                                         nullptr, bins.bbox);
  k_bin_scan<<<1, kScanThreads, 0, s>>>(bins.count, bins.bbox, ntiles, geo.tiles_c, geo.g,
                                    geo.layout, bins.offset, bins.cursor, bins.work, bins.nwork,
                                    (int)bins.wcap, bins.multi, bins.nmulti);
  if (nb > 0)
    k_bin<1><<<blocks, kThreads, 0, s>>>(B, nb, scale, geo.g, geo.tiles_c, bins.cursor,
                                         bins.offset, bins.entries, nullptr);
  return cudaGetLastError();
}

// CTAs per SM that fit: the precision form's shared memory (the tile and its
// low limbs) allows three, the plain form's registers four.
int fip_grid_max_ctas_per_sm(int compensated) { return compensated ? 3 : 4; }

cudaError_t fip_launch_grid(const FipGeom& geo, const float* B, const void* vr, const void* vi,
                            int vis_type, const float* vis_scale, const float* V, int nb,
                            const FipBins& bins, float2* grid, int compensated, cudaStream_t s,
                            int ctas_per_sm, const FipRawVis* raw) {
  if (vis_type == FIP_VIS_RAW && !raw) return cudaErrorInvalidValue;
  const FipRawVis rv = raw ? *raw : FipRawVis{};
  const float scale = geo.cell * (float)(size_t)geo.g;
  const int sms = sm_count();
  k_zero_tiles<<<sms, kThreads, 0, s>>>(bins.multi, bins.nmulti, geo.tiles_c, geo.g, geo.hp,
                                        geo.layout, grid, 0, 0);
  const size_t smem = grid_smem_bytes(compensated != 0);
  const int most = fip_grid_max_ctas_per_sm(compensated);
  const int blocks = sms * (ctas_per_sm > 0 ? min(ctas_per_sm, most) : most);
#define FIP_GRID_CASE(VT, C)                                                                    \
  do {                                                                                          \
    auto kern = k_grid<VT, C>;                                                                  \
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);         \
    kern<<<blocks, kThreads, smem, s>>>(B, vr, vi, vis_scale, V, scale, geo.g, geo.hp,          \
                                        geo.tiles_c, geo.layout, bins.entries, bins.work,       \
                                        bins.nwork, grid, rv);                                  \
  } while (0)
  if (vis_type == FIP_VIS_RAW) {
    if (compensated) FIP_GRID_CASE(FIP_VIS_RAW, true); else FIP_GRID_CASE(FIP_VIS_RAW, false);
  } else if (vis_type == FIP_VIS_F32) {
    if (compensated) FIP_GRID_CASE(FIP_VIS_F32, true); else FIP_GRID_CASE(FIP_VIS_F32, false);
  } else if (vis_type == FIP_VIS_F16) {
    if (compensated) FIP_GRID_CASE(FIP_VIS_F16, true); else FIP_GRID_CASE(FIP_VIS_F16, false);
  } else {
    if (compensated) FIP_GRID_CASE(FIP_VIS_BF16, true); else FIP_GRID_CASE(FIP_VIS_BF16, false);
  }
#undef FIP_GRID_CASE
  (void)nb;
  return cudaGetLastError();
}

cudaError_t fip_launch_zero_batch(const FipGeom& geo, const unsigned* multi, size_t multi_stride,
                                  const unsigned* nmulti, float2* grid, size_t grid_stride,
                                  int count, cudaStream_t s) {
  if (count < 1 || count > 65535) return cudaErrorInvalidValue;
  k_zero_tiles<<<dim3(sm_count(), count), kThreads, 0, s>>>(multi, nmulti, geo.tiles_c, geo.g,
                                                            geo.hp, geo.layout, grid,
                                                            multi_stride, grid_stride);
  return cudaGetLastError();
}

cudaError_t fip_launch_grid_batch(const FipGridBatch& in, int vis_type, int compensated,
                                  cudaStream_t s, int ctas_per_sm) {
  if (in.count < 1 || in.count > FIP_MAX_BATCH) return cudaErrorInvalidValue;
  const int sms = sm_count();
  const size_t smem = grid_smem_bytes(compensated != 0);
  const int most = fip_grid_max_ctas_per_sm(compensated);
  const int blocks = sms * (ctas_per_sm > 0 ? min(ctas_per_sm, most) : most);
#define FIP_GRID_CASE(VT, C)                                                                   \
  do {                                                                                         \
    auto kern = k_grid_batch<VT, C>;                                                           \
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);        \
    kern<<<blocks, kThreads, smem, s>>>(in);                                                   \
  } while (0)
  if (vis_type == FIP_VIS_F32) {
    if (compensated) FIP_GRID_CASE(FIP_VIS_F32, true); else FIP_GRID_CASE(FIP_VIS_F32, false);
  } else if (vis_type == FIP_VIS_F16) {
    if (compensated) FIP_GRID_CASE(FIP_VIS_F16, true); else FIP_GRID_CASE(FIP_VIS_F16, false);
  } else {
    if (compensated) FIP_GRID_CASE(FIP_VIS_BF16, true); else FIP_GRID_CASE(FIP_VIS_BF16, false);
  }
#undef FIP_GRID_CASE
  return cudaGetLastError();
}

// The transforms' dynamic shared memory depends on the grid side.  Their
// limit is raised to the most the device allows next to the kernel's static
// shared memory, the same value for every caller, so imagers of different
// sizes launching from concurrent host threads never lower it under one
// another's launch.
static cudaError_t fft_smem_attr(const void* fn, size_t smem) {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess)
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  cudaFuncAttributes fa{};
  e = cudaFuncGetAttributes(&fa, fn);
  if (e != cudaSuccess) return e;
  const int most = optin - (int)fa.sharedSizeBytes;  // static + dynamic <= opt-in maximum
  if (smem > (size_t)most) return cudaErrorInvalidConfiguration;
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
}

template <int LM, int LE>
static cudaError_t launch_cols(const FipGeom& geo, const float2* grid, const unsigned* bbox,
                               float2* colbuf, const float2* tw, cudaStream_t s, int batch,
                               size_t grid_stride, size_t col_stride, int split, int direct) {
  size_t smem;
  cudaError_t e;
  if (split) {
    smem = 2 * (size_t)fipfft::sub_stride(1 << LM) * sizeof(float2);
    if ((e = fft_smem_attr((const void*)k_fft_cols_split<LM, LE>, smem)) != cudaSuccess)
      return e;
    k_fft_cols_split<LM, LE><<<dim3(geo.hp, 3, batch), split_threads<LM, LE>(), smem, s>>>(
        grid, bbox, colbuf, tw, grid_stride, col_stride);
    return cudaGetLastError();
  }
  if (direct == 1) {  // (2: the row pass's band copy; the column pass stays staged)
    smem = (size_t)fipfft::direct_smem_elems(geo.g) * sizeof(float2);
    e = fft_smem_attr((const void*)k_fft_cols<LM, LE, true>, smem);
    if (e != cudaSuccess) return e;
    k_fft_cols<LM, LE, true><<<dim3(geo.hp, batch), fft_threads<LM, LE>(), smem, s>>>(
        grid, bbox, colbuf, tw, grid_stride, col_stride);
    return cudaGetLastError();
  }
  smem = (size_t)fipfft::smem_elems(geo.g) * sizeof(float2);
  e = fft_smem_attr((const void*)k_fft_cols<LM, LE, false>, smem);
  if (e != cudaSuccess) return e;
  // Persistent over columns: the CTAs that fit at once.
  // (Queried once per instantiation: the shape and shared memory are fixed by it.)
  static const int per_sm = [&] {
    int v = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_fft_cols<LM, LE, false>,
                                                      fft_threads<LM, LE>(), smem) != cudaSuccess)
      v = 1;
    return std::max(v, 1);
  }();
  const int ctas = std::max(1, std::min(geo.hp, per_sm * sm_count()));
  k_fft_cols<LM, LE, false><<<dim3(ctas, batch), fft_threads<LM, LE>(), smem, s>>>(
      grid, bbox, colbuf, tw, grid_stride, col_stride);
  return cudaGetLastError();
}

// The driver's tensor-map encoder (cuTensorMapEncodeTiled), or null.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault,
                                         &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      p = nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// The column-pass output of a batch as floats [batch][G/2 + 1][2 N], in boxes
// of 4 floats (rows yy1, yy1 + 1 of a column) x kBandBox columns.
static bool encode_band_map(CUtensorMap* m, const float2* colbuf, const FipGeom& geo, int batch,
                            size_t col_stride) {
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc || ((uintptr_t)colbuf & 15) != 0 || batch < 1) return false;
  const cuuint64_t dims[3] = {2 * (cuuint64_t)geo.n, (cuuint64_t)geo.hp, (cuuint64_t)batch};
  const cuuint64_t strides[2] = {2 * (cuuint64_t)geo.n * 4,
                                 (cuuint64_t)(batch > 1 ? col_stride : (size_t)geo.hp * geo.n) * 8};
  const cuuint32_t box[3] = {4, (cuuint32_t)kBandBox, 1};
  const cuuint32_t es[3] = {1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float2*>(colbuf), dims, strides,
             box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

template <int LM, int LE>
static cudaError_t launch_rows(const FipGeom& geo, const float2* colbuf, unsigned* bbox,
                               const float* taper, const float2* tw, float* pre,
                               cudaStream_t s, int batch, size_t col_stride,
                               size_t pre_stride, int split, int direct) {
  size_t smem;
  cudaError_t e;
  const CUtensorMap no_map{};
  if (split) {
    smem = 2 * (size_t)fipfft::sub_stride(1 << LM) * sizeof(float2);
    if ((e = fft_smem_attr((const void*)k_fft_rows_split<LM, LE>, smem)) != cudaSuccess)
      return e;
    k_fft_rows_split<LM, LE><<<dim3(geo.n / 2, 3, batch), split_threads<LM, LE>(), smem, s>>>(
        colbuf, bbox, taper + geo.n / 2 + 1, pre, tw, col_stride, pre_stride);
    return cudaGetLastError();
  }
  CUtensorMap band_map{};
  if (direct == 2 && encode_band_map(&band_map, colbuf, geo, batch, col_stride)) {
    // Persistent over row pairs (the CTAs that fit at once), the band copy
    // one row pair ahead.
    smem = band_smem_bytes<LM>();
    e = fft_smem_attr((const void*)k_fft_rows<LM, LE, true, true>, smem);
    if (e != cudaSuccess) return e;
    static const int per_sm = [&] {
      int v = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_fft_rows<LM, LE, true, true>,
                                                        fft_threads<LM, LE>(), smem) !=
          cudaSuccess)
        v = 1;
      return std::max(v, 1);
    }();
    const int ctas = std::max(1, std::min(geo.n / 2, per_sm * sm_count()));
    k_fft_rows<LM, LE, true, true><<<dim3(ctas, batch), fft_threads<LM, LE>(), smem, s>>>(
        colbuf, bbox, taper + geo.n / 2 + 1, pre, tw, col_stride, pre_stride, band_map);
    return cudaGetLastError();
  }
  if (direct) {
    smem = (size_t)fipfft::direct_smem_elems(geo.g) * sizeof(float2);
    e = fft_smem_attr((const void*)k_fft_rows<LM, LE, true>, smem);
    if (e != cudaSuccess) return e;
    k_fft_rows<LM, LE, true><<<dim3(geo.n / 2, batch), fft_threads<LM, LE>(), smem, s>>>(
        colbuf, bbox, taper + geo.n / 2 + 1, pre, tw, col_stride, pre_stride, no_map);
    return cudaGetLastError();
  }
  smem = (size_t)fipfft::smem_elems(geo.g) * sizeof(float2);
  e = fft_smem_attr((const void*)k_fft_rows<LM, LE, false>, smem);
  if (e != cudaSuccess) return e;
  // Persistent over row pairs: the CTAs that fit at once.
  // (Queried once per instantiation: the shape and shared memory are fixed by it.)
  static const int per_sm = [&] {
    int v = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_fft_rows<LM, LE, false>,
                                                      fft_threads<LM, LE>(), smem) != cudaSuccess)
      v = 1;
    return std::max(v, 1);
  }();
  const int ctas = std::max(1, std::min(geo.n / 2, per_sm * sm_count()));
  k_fft_rows<LM, LE, false><<<dim3(ctas, batch), fft_threads<LM, LE>(), smem, s>>>(
      colbuf, bbox, taper + geo.n / 2 + 1, pre, tw, col_stride, pre_stride, no_map);
  return cudaGetLastError();
}

// Calls F<LM, LE> for the plan's instantiation.
#define FIP_FFT_SWITCH(PLAN, CALL)                                      \
  do {                                                                  \
    const int key_ = (PLAN).lm * 8 + (PLAN).le;                         \
    switch (key_) {                                                     \
      case 4 * 8 + 3: { constexpr int LM_ = 4, LE_ = 3; return CALL; }  \
      case 5 * 8 + 3: { constexpr int LM_ = 5, LE_ = 3; return CALL; }  \
      case 6 * 8 + 3: { constexpr int LM_ = 6, LE_ = 3; return CALL; }  \
      case 7 * 8 + 3: { constexpr int LM_ = 7, LE_ = 3; return CALL; }  \
      case 8 * 8 + 3: { constexpr int LM_ = 8, LE_ = 3; return CALL; }  \
      case 9 * 8 + 3: { constexpr int LM_ = 9, LE_ = 3; return CALL; }  \
      case 10 * 8 + 3: { constexpr int LM_ = 10, LE_ = 3; return CALL; } \
      case 11 * 8 + 3: { constexpr int LM_ = 11, LE_ = 3; return CALL; } \
      case 5 * 8 + 4: { constexpr int LM_ = 5, LE_ = 4; return CALL; }  \
      case 6 * 8 + 4: { constexpr int LM_ = 6, LE_ = 4; return CALL; }  \
      case 7 * 8 + 4: { constexpr int LM_ = 7, LE_ = 4; return CALL; }  \
      case 8 * 8 + 4: { constexpr int LM_ = 8, LE_ = 4; return CALL; }  \
      case 9 * 8 + 4: { constexpr int LM_ = 9, LE_ = 4; return CALL; }  \
      case 10 * 8 + 4: { constexpr int LM_ = 10, LE_ = 4; return CALL; } \
      case 11 * 8 + 4: { constexpr int LM_ = 11, LE_ = 4; return CALL; } \
      case 12 * 8 + 4: { constexpr int LM_ = 12, LE_ = 4; return CALL; } \
      default: return cudaErrorInvalidValue;                             \
    }                                                                   \
  } while (0)

cudaError_t fip_launch_fft_cols(const FipGeom& geo, const float2* grid, const unsigned* bbox,
                                float2* colbuf, const float2* twiddles, const fipfft::Plan& plan,
                                cudaStream_t s, int batch, size_t grid_stride,
                                size_t col_stride) {
  if (plan.g != geo.g || batch < 1 || batch > 65535) return cudaErrorInvalidValue;
  FIP_FFT_SWITCH(plan, (launch_cols<LM_, LE_>(geo, grid, bbox, colbuf, twiddles, s, batch,
                                              grid_stride, col_stride, plan.split,
                                              plan.direct)));
}

cudaError_t fip_launch_fft_rows(const FipGeom& geo, const float2* colbuf, unsigned* bbox,
                                const float* taper, const float2* twiddles,
                                const fipfft::Plan& plan, float* pre, cudaStream_t s, int batch,
                                size_t col_stride, size_t pre_stride) {
  if (plan.g != geo.g || batch < 1 || batch > 65535) return cudaErrorInvalidValue;
  FIP_FFT_SWITCH(plan, (launch_rows<LM_, LE_>(geo, colbuf, bbox, taper, twiddles, pre, s, batch,
                                              col_stride, pre_stride, plan.split,
                                              plan.direct)));
}

cudaError_t fip_launch_correct_c2r(const FipGeom& geo, const float* fft_out, const float* taper,
                                   float* pre, unsigned* pre_max, cudaStream_t s) {
  dim3 bl((geo.n + kThreads - 1) / kThreads, geo.n);
  k_correct_c2r<<<bl, kThreads, 0, s>>>(fft_out, taper, geo.n, geo.g, pre, pre_max);
  return cudaGetLastError();
}

const void* fip_targets_kernel() { return reinterpret_cast<const void*>(&k_targets); }

cudaError_t fip_launch_targets(const FipGeom& geo, const float* V, const float2* theta_tab,
                               float2* targets, cudaStream_t s) {
  const int per = kThreads * kTargetsPerThread;
  dim3 bl((geo.n + per - 1) / per, geo.n);
  k_targets<<<bl, kThreads, 0, s>>>(V, geo.n, cell_degrees(geo.cell), theta_tab, targets);
  return cudaGetLastError();
}

cudaError_t fip_launch_reproject_scatter(const FipGeom& geo, const float* pre, const float* V,
                                         int nb, float* dst, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(dst, 0, (size_t)geo.n * geo.n * sizeof(float), s);
  if (e != cudaSuccess) return e;
  dim3 th(32, 8), bl((geo.n + 31) / 32, (geo.n + 7) / 8);
  k_reproject_scatter<<<bl, th, 0, s>>>(pre, V, geo.n, nb, cell_degrees(geo.cell), dst);
  return cudaGetLastError();
}

// Target deviation allowance of the FP32 chain from the exact map, in
// destination pixels: half a pixel plus eight ulps of a unit-scale cosine
// expressed in pixels (the chain evaluates cos(theta) ~ R in degrees).
static float chain_delta(float cell) { return 0.5f + 8.0f * 4.76837158e-7f / cell; }

bool fip_gather_supported(const FipGeom& geo, int exact_targets) {
  return exact_targets || chain_delta(geo.cell) <= 40.f;
}

bool fip_trigger_fusable(const FipGeom& geo) {
  return geo.t > 0 && kDT % geo.t == 0 && geo.n % kDT == 0;
}

size_t fip_trigger_fuse_counts(const FipGeom& geo) {
  const size_t tiles = (geo.n + kDT - 1) / kDT;
  return tiles * tiles;
}

cudaError_t fip_launch_reproject_gather(const FipGeom& geo, const float* pre,
                                        const float2* targets, const float* V, int nb,
                                        const unsigned* pre_max, float* dst, unsigned* img_max,
                                        int exact_targets, cudaStream_t s, unsigned* err,
                                        const FipFuse* fuse) {
  const int tiles = (geo.n + kDT - 1) / kDT;
  const float delta = exact_targets ? 0.25f : chain_delta(geo.cell);
  if (!fip_gather_supported(geo, exact_targets)) return cudaErrorInvalidValue;
  FipTriggerFuse tf{};
  if (fuse) {
    if (!fip_trigger_fusable(geo)) return cudaErrorInvalidValue;
    for (int k = 0; k < 3; ++k) tf.img[k] = fuse->img[k];
    tf.count = fuse->count;
    tf.stats = fuse->stats;
    tf.t = geo.t;
    tf.u = geo.u;
  }
  if (exact_targets)
    k_reproject_gather<true><<<tiles * tiles, kThreads, 0, s>>>(
        pre, nullptr, V, geo.n, nb, geo.cell, delta, pre_max, dst, img_max, err, tf);
  else
    k_reproject_gather<false><<<tiles * tiles, kThreads, 0, s>>>(
        pre, targets, V, geo.n, nb, geo.cell, delta, pre_max, dst, img_max, err, tf);
  return cudaGetLastError();
}

cudaError_t fip_launch_trigger_combine(const FipGeom& geo, const double* stats,
                                       const float* max3, float* result, int precise,
                                       cudaStream_t s) {
  const int tiles = geo.u * geo.u;
  if (tiles == 0) return cudaSuccess;
  const int blocks = (tiles + kThreads - 1) / kThreads;
  if (precise)
    k_trigger_combine<true><<<blocks, kThreads, 0, s>>>(stats, max3, geo.u, geo.t, result);
  else
    k_trigger_combine<false><<<blocks, kThreads, 0, s>>>(stats, max3, geo.u, geo.t, result);
  return cudaGetLastError();
}

bool fip_gather_domain_ok(const float* V, int n, float cell) {
  // The exact map on a 65 x 65 lattice over the source image (and one pixel
  // beyond): inside the horizon with room (r2 < 0.98) and no fold of the
  // slant part (its Jacobian determinant above 1/4), the conditions the
  // gather checks per tile.  V is row-major 3 x 3 on the host.
  const double a22 = fabs((double)V[8]);
  if (!(a22 > 0.0)) return false;
  const double m00 = -(double)V[0] / a22, m01 = (double)V[3] / a22;
  const double m10 = -(double)V[1] / a22, m11 = (double)V[4] / a22;
  const double xi = (double)V[6] / (double)V[8], eta = (double)V[7] / (double)V[8];
  const double h = n / 2, lo = -h - 2.0, span = (double)n + 4.0;
  for (int q = 0; q <= 64; ++q)
    for (int p = 0; p <= 64; ++p) {
      const double a = lo + span * p / 64.0, b = lo + span * q / 64.0;
      const double X = cell * (m00 * a + m01 * b - 1.0), Y = cell * (m10 * a + m11 * b - 1.0);
      const double r2 = X * X + Y * Y;
      if (!(r2 < 0.98)) return false;
      const double nn = sqrt(1.0 - r2);
      if (!(1.0 - xi * X / nn + eta * Y / nn > 0.25)) return false;
    }
  return true;
}

cudaError_t fip_launch_image_max(const float* img, size_t count, unsigned* out, cudaStream_t s) {
  k_image_max<<<1184, kThreads, 0, s>>>(img, count, out);
  return cudaGetLastError();
}

// ---- The streamed sliding-window trigger ----------------------------------
static std::atomic<int> g_trigger_stream{1};

void fip_trigger_stream_enable(int on) { g_trigger_stream.store(on ? 1 : 0); }
int fip_trigger_stream_enabled() { return g_trigger_stream.load(); }

template <bool PRECISE>
static cudaError_t launch_stream_window(const FipGeom& geo, const float* images, int count,
                                        const float* maxima, float* results, cudaStream_t s) {
  const int tiles = geo.u * geo.u;
  const int bx = (tiles + kStreamThreads / 32 - 1) / (kStreamThreads / 32);
  // Chunks of triples: enough warps to fill the device (about eight waves
  // of 12 warps per SM), each chunk re-reading only its first two slices.
  const int want = 8 * 12 * sm_count();
  int chunks = std::max(1, std::min(count, want / std::max(1, tiles)));
  const int chunk = (count + chunks - 1) / chunks;
  chunks = (count + chunk - 1) / chunk;
  if (chunks > 65535) return cudaErrorInvalidValue;
  const dim3 grid(bx, chunks);
  const size_t n2 = (size_t)geo.n * geo.n;
  const int nv = (geo.t * geo.t / 4 + 31) / 32;
#define FIP_STREAM(NV)                                                                         \
  k_trigger_stream<PRECISE, NV><<<grid, kStreamThreads, 0, s>>>(                               \
      images, n2, count, chunk, maxima, geo.n, geo.t, geo.u, results)
  if (nv <= 1)
    FIP_STREAM(1);
  else if (nv <= 2)
    FIP_STREAM(2);
  else if (nv <= 4)
    FIP_STREAM(4);
  else
    FIP_STREAM(8);
#undef FIP_STREAM
  return cudaGetLastError();
}

cudaError_t fip_launch_trigger(const FipGeom& geo, const float* I1, const float* I2,
                               const float* I3, const float* max3, float* stats, float* result,
                               int precise, cudaStream_t s) {
  (void)stats;
  return fip_launch_trigger3(geo, I1, I2, I3, max3, max3 + 1, max3 + 2, result, precise, s);
}

cudaError_t fip_launch_trigger3(const FipGeom& geo, const float* I1, const float* I2,
                                const float* I3, const float* m1, const float* m2,
                                const float* m3, float* result, int precise, cudaStream_t s) {
  const int tiles = geo.u * geo.u;
  const int blocks = (tiles + kThreads / 32 - 1) / (kThreads / 32);
  if (tiles == 0) return cudaSuccess;
  const int vec = (geo.t % 4 == 0) && (geo.n % 4 == 0) &&
                  ((((uintptr_t)I1) | ((uintptr_t)I2) | ((uintptr_t)I3)) & 15) == 0;
  if (precise)
    k_trigger<true><<<blocks, kThreads, 0, s>>>(I1, I2, I3, m1, m2, m3, geo.n, geo.t, geo.u, vec,
                                                result, 0, 0);
  else
    k_trigger<false><<<blocks, kThreads, 0, s>>>(I1, I2, I3, m1, m2, m3, geo.n, geo.t, geo.u,
                                                 vec, result, 0, 0);
  return cudaGetLastError();
}

cudaError_t fip_launch_trigger_batch(const FipGeom& geo, const float* images, const float* maxima,
                                     int count, float* results, int precise, cudaStream_t s) {
  const int tiles = geo.u * geo.u;
  if (tiles == 0 || count <= 0) return cudaSuccess;
  if (count > 65535) return cudaErrorInvalidValue;
  // Plain form, three or more triples: the register stream (each image read
  // once).  The precision form's compensated sums make it issue-bound; its
  // triples keep the plain loads, which hide latency with more warps.
  if (g_trigger_stream.load() && !precise && count >= 3 && geo.t % 4 == 0 && geo.t <= 32 &&
      geo.n % 4 == 0 && ((uintptr_t)images & 15) == 0)
    return launch_stream_window<false>(geo, images, count, maxima, results, s);
  const size_t n2 = (size_t)geo.n * geo.n;
  const dim3 blocks((tiles + kThreads / 32 - 1) / (kThreads / 32), count);
  const int vec = (geo.t % 4 == 0) && (geo.n % 4 == 0) && ((uintptr_t)images & 15) == 0;
  if (precise)
    k_trigger<true><<<blocks, kThreads, 0, s>>>(images, images + n2, images + 2 * n2, maxima,
                                                maxima + 1, maxima + 2, geo.n, geo.t, geo.u, vec,
                                                results, n2, (size_t)tiles);
  else
    k_trigger<false><<<blocks, kThreads, 0, s>>>(images, images + n2, images + 2 * n2, maxima,
                                                 maxima + 1, maxima + 2, geo.n, geo.t, geo.u,
                                                 vec, results, n2, (size_t)tiles);
  return cudaGetLastError();
}

cudaError_t fip_launch_pixel_targets(const FipGeom& geo, const float* V, float* out,
                                     int mode, const float2* theta_tab, cudaStream_t s) {
  if (mode < 0 || mode > 2) return cudaErrorInvalidValue;
  dim3 bl((geo.n + kThreads - 1) / kThreads, geo.n);
  k_pixel_targets<<<bl, kThreads, 0, s>>>(V, geo.n, cell_degrees(geo.cell), geo.cell, mode,
                                          theta_tab, out);
  return cudaGetLastError();
}

size_t fip_theta_table_elems() { return (size_t)fipref::kThetaTabSize; }

cudaError_t fip_launch_theta_table(float2* tab, cudaStream_t s) {
  k_theta_table<<<(fipref::kThetaTabSize + kThreads - 1) / kThreads, kThreads, 0, s>>>(tab);
  return cudaGetLastError();
}
