// Device stages of the snapshot imaging + tLISI trigger path.
//
// This translation unit is compiled with --use_fast_math, the flags of the
// reference's CUDA build (reference Makefile:13), because the plain FP32 form
// reproduces the reference's FP32 arithmetic (see fip_refmath.cuh).  Data
// movement is B200-native:
//   * gridding bins every visibility by 64x64 tile of the Hermitian half-plane
//     grid, accumulates each tile in shared memory and commits it once (plain
//     128-bit stores for tiles owned by one work item, vector reductions only
//     for the few dense tiles split over several);
//   * the FFT is one in-place C2R transform (half the data of the reference's
//     C2C) and the crop/checkerboard/correction pass is fused into the
//     reprojection's source loads;
//   * reprojection is destination-tile-major: each 32x32 output tile gathers
//     its candidate source pixels, splats them in shared memory, stores the
//     tile once and reports its maximum -- no global atomics, no memsets;
//   * the trigger reads the three images once, in 128-bit loads, with
//     warp-shuffle tile reductions.
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "fip_common.cuh"
#include "fip_kernels.h"
#include "fip_refmath.cuh"

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ int wrap_mod(long v, int m) {
  long r = v % m;
  return (int)(r < 0 ? r + m : r);
}

// ---------------------------------------------------------------------------
// Taper (FIPkernels.cu:173-186)
// ---------------------------------------------------------------------------
__global__ void k_taper(float* taper, size_t n, size_t g) {
  size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t < n / 2 + 1) taper[t] = fipref::taper(t, g);
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

// Half-plane image of a virtual visibility: the direct one keeps taps with
// r2 >= 0 at (r1 mod G, r2); the mirrored one (conjugate) keeps taps with
// r2 <= 0 at (-r1 mod G, -r2).  Column range in half-plane columns.
__device__ __forceinline__ bool half_cols(const Footprint& f, int mir, int& c0, int& c1) {
  if (!mir) {
    if (f.b1 < 0) return false;
    c0 = max(f.b0, 0); c1 = f.b1;
  } else {
    if (f.b0 > 0) return false;
    c0 = max(-f.b1, 0); c1 = -f.b0;
  }
  return true;
}

// Enumerate distinct tile rows touched by rows r1 in [a0,a1] (direct) or
// -r1 (mirrored), modulo G.  At most 3.
__device__ __forceinline__ int tile_rows(const Footprint& f, int mir, int g, int* out) {
  int n = 0;
  for (int r1 = f.a0; r1 <= f.a1; ++r1) {
    int row = wrap_mod(mir ? -(long)r1 : (long)r1, g);
    int tr = row / FIP_GTILE;
    bool seen = false;
    for (int k = 0; k < n; ++k) seen |= (out[k] == tr);
    if (!seen && n < 3) out[n++] = tr;
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

// pass 0: count entries per tile; pass 1: scatter entries.
template <int PASS>
__global__ void k_bin(const float* __restrict__ B, int nb, float scale, int g, int tiles_c,
                      unsigned* cnt, const unsigned* __restrict__ offset, unsigned* entries) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  Footprint f;
  bool ok = v < nb && footprint(B, v, scale, g, f);
  for (int mir = 0; mir < 2; ++mir) {
    int c0 = 0, c1 = -1, trs[3], ntr = 0;
    bool on = ok && half_cols(f, mir, c0, c1);
    if (on) ntr = tile_rows(f, mir, g, trs);
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
}

// Exclusive scan of tile counts and construction of the work list.  One CTA.
__global__ void k_bin_scan(const unsigned* __restrict__ cnt, int ntiles, unsigned* offset,
                           unsigned* cursor, int4* work, unsigned* nwork, int wcap) {
  __shared__ unsigned s_sum[kThreads];
  __shared__ unsigned s_wsum[kThreads];
  const int per = (ntiles + kThreads - 1) / kThreads;
  const int beg = threadIdx.x * per, end = min(beg + per, ntiles);
  unsigned local = 0, wlocal = 0;
  for (int t = beg; t < end; ++t) {
    local += cnt[t];
    wlocal += (cnt[t] + FIP_GCHUNK - 1) / FIP_GCHUNK;
  }
  s_sum[threadIdx.x] = local;
  s_wsum[threadIdx.x] = wlocal;
  __syncthreads();
  for (int d = 1; d < kThreads; d <<= 1) {
    unsigned a = threadIdx.x >= d ? s_sum[threadIdx.x - d] : 0;
    unsigned b = threadIdx.x >= d ? s_wsum[threadIdx.x - d] : 0;
    __syncthreads();
    s_sum[threadIdx.x] += a;
    s_wsum[threadIdx.x] += b;
    __syncthreads();
  }
  unsigned run = s_sum[threadIdx.x] - local, wrun = s_wsum[threadIdx.x] - wlocal;
  for (int t = beg; t < end; ++t) {
    offset[t] = run;
    cursor[t] = 0;
    unsigned c = cnt[t];
    unsigned nchunk = (c + FIP_GCHUNK - 1) / FIP_GCHUNK;
    for (unsigned k = 0; k < nchunk; ++k) {
      if ((int)(wrun + k) < wcap)
        work[wrun + k] = make_int4(t, (int)(run + k * FIP_GCHUNK),
                                   (int)min(run + (k + 1) * FIP_GCHUNK, run + c), nchunk == 1);
    }
    run += c;
    wrun += nchunk;
  }
  if (threadIdx.x == kThreads - 1) {
    offset[ntiles] = run;
    *nwork = min(wrun, (unsigned)wcap);
  }
}

template <int VT>
__device__ __forceinline__ float load_vis(const void* p, int v) {
  if (VT == FIP_VIS_F32) return reinterpret_cast<const float*>(p)[v];
  if (VT == FIP_VIS_F16) return __half2float(reinterpret_cast<const __half*>(p)[v]);
  return __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(p)[v]);
}

// Persistent gridder: each work item is (tile, entry range).  Warps take one
// virtual visibility at a time; lanes own taps.  COMP: Kahan-compensated
// accumulation in shared memory (precision form).
template <int VT, bool COMP>
__global__ void __launch_bounds__(kThreads) k_grid(const float* __restrict__ B, const void* vr,
                                                   const void* vi,
                                                   const float* __restrict__ vis_scale_p,
                                                   const float* __restrict__ V, float scale,
                                                   int g, int hp, int tiles_c,
                                                   const unsigned* __restrict__ entries,
                                                   const int4* __restrict__ work,
                                                   const unsigned* __restrict__ nwork,
                                                   float2* __restrict__ grid) {
  extern __shared__ float4 s_raw[];
  float2* s_tile = reinterpret_cast<float2*>(s_raw);                // [64*64]
  float2* s_comp = s_tile + FIP_GTILE * FIP_GTILE;                  // [64*64] if COMP
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const float inten = fabs(V[0 * 3 + 0] * V[1 * 3 + 1] - V[0 * 3 + 1] * V[1 * 3 + 0]);
  const float vis_scale = vis_scale_p ? *vis_scale_p : 1.0f;
  const unsigned nw = *nwork;
  for (unsigned w = blockIdx.x; w < nw; w += gridDim.x) {
    const int4 item = work[w];
    const int tile = item.x;
    const int row0 = (tile / tiles_c) * FIP_GTILE, col0 = (tile % tiles_c) * FIP_GTILE;
    for (int k = threadIdx.x; k < FIP_GTILE * FIP_GTILE; k += kThreads) {
      s_tile[k] = make_float2(0.f, 0.f);
      if (COMP) s_comp[k] = make_float2(0.f, 0.f);
    }
    __syncthreads();
    for (int e = item.y + warp; e < item.z; e += kThreads / 32) {
      const unsigned ent = entries[e];
      const int v = (int)(ent >> 1), mir = (int)(ent & 1);
      Footprint f;
      footprint(B, v, scale, g, f);
      int c0, c1;
      half_cols(f, mir, c0, c1);
      // Visibility weighting (FIPkernels.cu:188-195), halved for the
      // Hermitian split, conjugated for the mirrored image.
      float wr, wi;
      if (VT == FIP_VIS_F32) {
        wr = load_vis<VT>(vr, v) / inten;
        wi = load_vis<VT>(vi, v) / inten;
      } else {
        wr = (load_vis<VT>(vr, v) * vis_scale) / inten;
        wi = (load_vis<VT>(vi, v) * vis_scale) / inten;
      }
      wr *= 0.5f;
      wi = mir ? -0.5f * wi : 0.5f * wi;
      // 1-D kernel values: lanes 0..15 rows, lanes 16..31 columns.
      float kv = 0.f;
      {
        const float ihs = 1 / static_cast<float>(FIP_SUPPORT / 2);
        if (lane < 16) {
          int r = f.a0 + lane;
          if (r <= f.a1) kv = fipref::es((static_cast<float>(r) - f.p1) * ihs);
        } else {
          int r = f.b0 + (lane - 16);
          if (r <= f.b1) kv = fipref::es((static_cast<float>(r) - f.p2) * ihs);
        }
      }
      const int nr = f.a1 - f.a0 + 1;
      const int r2lo = mir ? -c1 : c0;  // original r2 range of the kept taps
      const int nc = c1 - c0 + 1;
      const int ntap = nr * nc;
      for (int t0 = 0; t0 < ntap; t0 += 32) {
        const int t = t0 + lane;
        const int ia = t / nc, ib = t % nc;
        const int r1 = f.a0 + min(ia, nr - 1);
        const int r2 = r2lo + ib;
        float k1 = __shfl_sync(0xffffffffu, kv, min(ia, nr - 1));
        float k2 = __shfl_sync(0xffffffffu, kv, 16 + (r2 - f.b0));
        if (t < ntap) {
          const int row = wrap_mod(mir ? -(long)r1 : (long)r1, g);
          const int col = mir ? -r2 : r2;
          const int lr = row - row0, lc = col - col0;
          if (lr >= 0 && lr < FIP_GTILE && lc >= 0 && lc < FIP_GTILE) {
            const float kval = k1 * k2;
            const float cr = wr * kval, ci = wi * kval;
            float2* cell = &s_tile[lr * FIP_GTILE + lc];
            if (!COMP) {
              atomicAdd(&cell->x, cr);
              atomicAdd(&cell->y, ci);
            } else {
              // Compensated add: old + c; the rounding error goes to s_comp.
              float o = atomicAdd(&cell->x, cr);
              float s = o + cr;
              float err = (fabsf(o) >= fabsf(cr)) ? (o - s) + cr : (cr - s) + o;
              atomicAdd(&s_comp[lr * FIP_GTILE + lc].x, err);
              o = atomicAdd(&cell->y, ci);
              s = o + ci;
              err = (fabsf(o) >= fabsf(ci)) ? (o - s) + ci : (ci - s) + o;
              atomicAdd(&s_comp[lr * FIP_GTILE + lc].y, err);
            }
          }
        }
      }
    }
    __syncthreads();
    // Commit the tile: plain stores when this item owns the tile, vector
    // reductions otherwise (grid pre-zeroed).
    const bool single = item.w != 0;
    for (int k = threadIdx.x; k < FIP_GTILE * FIP_GTILE; k += kThreads) {
      const int lr = k / FIP_GTILE, lc = k % FIP_GTILE;
      const int row = row0 + lr, col = col0 + lc;
      if (row < g && col < hp) {
        float2 val = s_tile[k];
        if (COMP) {
          val.x += s_comp[k].x;
          val.y += s_comp[k].y;
        }
        float2* dst = &grid[(size_t)row * hp + col];
        if (single) {
          *dst = val;
        } else if (val.x != 0.f || val.y != 0.f) {
          atomicAdd(dst, val);
        }
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Corrected source pixel (FIPkernels.cu:256-287 and :391-392), read from the
// in-place C2R output: row (j - N/2) mod G, column (i - N/2) mod G, row stride
// G + 2 floats.  The reference's checkerboard signs cancel against its
// centred grid origin, so none is applied here.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float source_value(const float* __restrict__ fft_out,
                                              const float* __restrict__ ck, int n, int g,
                                              int i, int j, float inv_nb) {
  const int h = n / 2;
  const long x = (long)i - h, y = (long)j - h;
  const int row = (int)(y < 0 ? y + g : y), col = (int)(x < 0 ? x + g : x);
  float px = fft_out[(size_t)row * (size_t)(g + 2) + col];
  const float norm = FIP_CONV_NORM;
  px *= 1 / (ck[labs(x)] * ck[labs(y)] * norm * norm);
  px = fabs(px);
  return px * inv_nb;
}

// Source-major reprojection, the reference's scheme (FIPkernels.cu:378-413)
// with the crop/correction fused: one thread per source pixel, four atomics.
__global__ void k_reproject_scatter(const float* __restrict__ fft_out, const float* __restrict__ ck,
                                    const float* __restrict__ V, int n, int g, int nb, float dc,
                                    float* __restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= n || j >= n) return;
  fipref::Frame fr{V[0], V[1], V[3], V[4], V[8], V[6], V[7], dc};
  const float inv_nb = 1.0f / static_cast<float>(nb);
  const float value = source_value(fft_out, ck, n, g, i, j, inv_nb);
  float LL, MM;
  fipref::pixel_target(fr, (size_t)i, (size_t)j, (size_t)n, LL, MM);
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

// ---------------------------------------------------------------------------
// Destination-tile-major reprojection.
// ---------------------------------------------------------------------------
constexpr int kDT = 32;          // destination tile side
constexpr int kMaxRows = 192;    // candidate source rows per tile

struct ExactMap {
  // LL = P1 - xi z / cell, MM = P2 + eta z / cell, z = 1 - sqrt(1 - rho),
  // rho = cell^2 ((P1 - 1)^2 + (P2 - 1)^2), P = M (a, b) / |V22|.
  double m00, m01, m10, m11;  // M / |V22|
  double i00, i01, i10, i11;  // inverse of M / |V22|
  double xi, eta, cell;
};

__device__ __forceinline__ void exact_forward(const ExactMap& m, double a, double b, double& LL,
                                              double& MM) {
  double P1 = m.m00 * a + m.m01 * b, P2 = m.m10 * a + m.m11 * b;
  double rho = m.cell * m.cell * ((P1 - 1) * (P1 - 1) + (P2 - 1) * (P2 - 1));
  double zc = rho <= 1 ? (rho / (1 + sqrt(1 - rho))) / m.cell : 0.0;
  LL = P1 - m.xi * zc;
  MM = P2 + m.eta * zc;
}

// Source coordinates (a, b) relative to the centre whose exact target is
// (LL, MM): fixed-point iteration on the slant term (a contraction for any
// field smaller than a radian).
__device__ __forceinline__ void exact_inverse(const ExactMap& m, double LL, double MM, double& a,
                                              double& b) {
  double P1 = LL, P2 = MM;
  for (int it = 0; it < 12; ++it) {
    double rho = m.cell * m.cell * ((P1 - 1) * (P1 - 1) + (P2 - 1) * (P2 - 1));
    double zc = rho <= 1 ? (rho / (1 + sqrt(1 - rho))) / m.cell : 0.0;
    P1 = LL + m.xi * zc;
    P2 = MM - m.eta * zc;
  }
  a = m.i00 * P1 + m.i01 * P2;
  b = m.i10 * P1 + m.i11 * P2;
}

__device__ __forceinline__ ExactMap make_map(const float* V, float cell) {
  ExactMap m;
  const double a22 = fabs((double)V[8]);
  m.m00 = -(double)V[0] / a22; m.m01 = (double)V[3] / a22;
  m.m10 = -(double)V[1] / a22; m.m11 = (double)V[4] / a22;
  const double det = m.m00 * m.m11 - m.m01 * m.m10;
  m.i00 = m.m11 / det; m.i01 = -m.m01 / det;
  m.i10 = -m.m10 / det; m.i11 = m.m00 / det;
  m.xi = (double)V[6] / (double)V[8];
  m.eta = (double)V[7] / (double)V[8];
  m.cell = (double)cell;
  return m;
}

// Precision-form target: the closed form in FP32 relative to a local origin
// (a0, b0) whose exact target (L0, M0) is given in double.
struct LocalMap {
  float m00, m01, m10, m11;  // M / |V22| in float
  float P10, P20;            // P at the local origin (absolute)
  float L0f, M0f;            // P at the origin minus the destination origin
  float xi, eta, cell;
};

template <bool EXACT>
__global__ void __launch_bounds__(kThreads) k_reproject_gather(
    const float* __restrict__ fft_out, const float* __restrict__ ck, const float* __restrict__ V,
    int n, int g, int nb, float dc, float cell, float delta, float* __restrict__ dst,
    unsigned* img_max) {
  __shared__ float s_tile[kDT * kDT];
  __shared__ int s_ilo[kMaxRows];
  __shared__ int s_scan[kMaxRows + 1];
  __shared__ double s_q[4][2];
  __shared__ int s_rows[2];
  __shared__ float s_wmax[kThreads / 32];

  const int tiles = (n + kDT - 1) / kDT;
  const int tr = blockIdx.x / tiles, tc = blockIdx.x % tiles;
  const int r0 = tr * kDT, c0 = tc * kDT;
  const int h = n / 2;
  const ExactMap m = make_map(V, cell);

  for (int k = threadIdx.x; k < kDT * kDT; k += kThreads) s_tile[k] = 0.f;
  // Preimage corners of the destination window widened by the splat reach
  // (one pixel) and delta (the FP32 chain's deviation from exact).
  if (threadIdx.x < 4) {
    const double Llo = (double)(c0 - h) - 1.0 - delta, Lhi = (double)(c0 + kDT - h) + delta;
    const double Mlo = (double)(r0 - h) - 1.0 - delta, Mhi = (double)(r0 + kDT - h) + delta;
    const double L = (threadIdx.x == 0 || threadIdx.x == 3) ? Llo : Lhi;
    const double M = (threadIdx.x < 2) ? Mlo : Mhi;
    double a, b;
    exact_inverse(m, L, M, a, b);
    s_q[threadIdx.x][0] = a;
    s_q[threadIdx.x][1] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double bmin = s_q[0][1], bmax = s_q[0][1];
    for (int k = 1; k < 4; ++k) {
      bmin = fmin(bmin, s_q[k][1]);
      bmax = fmax(bmax, s_q[k][1]);
    }
    int jlo = (int)fmax(0.0, ceil(fmax(bmin + h - 1e-9, -1.0)));
    int jhi = (int)fmin((double)(n - 1), floor(fmin(bmax + h + 1e-9, (double)n)));
    if (jhi - jlo + 1 > kMaxRows) jhi = jlo + kMaxRows - 1;  // unreachable for delta < 40
    s_rows[0] = jlo;
    s_rows[1] = jhi;
  }
  __syncthreads();
  const int jlo = s_rows[0], jhi = s_rows[1];
  const int nrows = max(0, jhi - jlo + 1);
  for (int r = threadIdx.x; r < nrows; r += kThreads) {
    const double b = (double)(jlo + r - h);
    double alo = 1e300, ahi = -1e300;
    for (int k = 0; k < 4; ++k) {
      const double ax = s_q[k][0], bx = s_q[k][1];
      const double ay = s_q[(k + 1) & 3][0], by = s_q[(k + 1) & 3][1];
      if ((bx <= b && b <= by) || (by <= b && b <= bx)) {
        double a;
        if (by == bx) {
          alo = fmin(alo, fmin(ax, ay));
          ahi = fmax(ahi, fmax(ax, ay));
          continue;
        }
        a = ax + (ay - ax) * (b - bx) / (by - bx);
        alo = fmin(alo, a);
        ahi = fmax(ahi, a);
      }
    }
    int ilo = 0, ihi = -1;
    if (alo <= ahi) {
      ilo = (int)fmax(0.0, ceil(fmax(alo + h - 1e-9, -1.0)));
      ihi = (int)fmin((double)(n - 1), floor(fmin(ahi + h + 1e-9, (double)n)));
    }
    s_ilo[r] = ilo;
    s_scan[r + 1] = ihi >= ilo ? ihi - ilo + 1 : 0;
  }
  if (threadIdx.x == 0) s_scan[0] = 0;
  __syncthreads();
  if (threadIdx.x == 0)
    for (int r = 0; r < nrows; ++r) s_scan[r + 1] += s_scan[r];
  __syncthreads();
  const int total = s_scan[nrows];

  const float inv_nb = 1.0f / static_cast<float>(nb);
  fipref::Frame fr{V[0], V[1], V[3], V[4], V[8], V[6], V[7], dc};
  const size_t half = n / 2;
  for (int k = threadIdx.x; k < total; k += kThreads) {
    int lo = 0, hi = nrows - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (s_scan[mid] <= k) lo = mid; else hi = mid - 1;
    }
    const int j = jlo + lo;
    const int i = s_ilo[lo] + (k - s_scan[lo]);
    const float value = source_value(fft_out, ck, n, g, i, j, inv_nb);
    float LL, MM;
    long fl, cl, fm, cm;
    float wl1, wm1, wl0, wm0;
    if (!EXACT) {
      fipref::pixel_target(fr, (size_t)i, (size_t)j, (size_t)n, LL, MM);
      if (!(fabs(LL) < half - 1 && fabs(MM) < half - 1)) continue;
      fl = fipref::floor_l(LL); cl = fipref::ceil_l(LL);
      fm = fipref::floor_l(MM); cm = fipref::ceil_l(MM);
      wl0 = 1 - LL + fl; wl1 = LL - fl;
      wm0 = 1 - MM + fm; wm1 = MM - fm;
    } else {
      double Ld, Md;
      exact_forward(m, (double)(i - h), (double)(j - h), Ld, Md);
      if (!(fabs(Ld) < (double)(half - 1) && fabs(Md) < (double)(half - 1))) continue;
      double fld = floor(Ld), fmd = floor(Md);
      fl = (long)fld; fm = (long)fmd;
      cl = (long)ceil(Ld); cm = (long)ceil(Md);
      wl1 = (float)(Ld - fld); wm1 = (float)(Md - fmd);
      wl0 = 1.0f - wl1; wm0 = 1.0f - wm1;
    }
    // Destination pixel (row h + m, column h + l), local to this tile.
    const int lf = (int)(h + fl) - c0, lc = (int)(h + cl) - c0;
    const int mf = (int)(h + fm) - r0, mc = (int)(h + cm) - r0;
    if ((unsigned)mf < (unsigned)kDT) {
      if ((unsigned)lf < (unsigned)kDT) atomicAdd(&s_tile[mf * kDT + lf], wl0 * wm0 * value);
      if ((unsigned)lc < (unsigned)kDT) atomicAdd(&s_tile[mf * kDT + lc], wl1 * wm0 * value);
    }
    if ((unsigned)mc < (unsigned)kDT) {
      if ((unsigned)lf < (unsigned)kDT) atomicAdd(&s_tile[mc * kDT + lf], wl0 * wm1 * value);
      if ((unsigned)lc < (unsigned)kDT) atomicAdd(&s_tile[mc * kDT + lc], wl1 * wm1 * value);
    }
  }
  __syncthreads();
  float vmax = 0.f;
  for (int k = threadIdx.x; k < kDT * kDT; k += kThreads) {
    const int rr = r0 + k / kDT, cc = c0 + k % kDT;
    if (rr < n && cc < n) {
      const float val = s_tile[k];
      dst[(size_t)rr * n + cc] = val;
      vmax = fmaxf(vmax, val);
    }
  }
  for (int o = 16; o > 0; o >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
  if ((threadIdx.x & 31) == 0) s_wmax[threadIdx.x >> 5] = vmax;
  __syncthreads();
  if (threadIdx.x == 0 && img_max) {
    float b = 0.f;
    for (int w = 0; w < kThreads / 32; ++w) b = fmaxf(b, s_wmax[w]);
    atomicMax(img_max, __float_as_uint(b));
  }
}

__global__ void k_pixel_targets(const float* __restrict__ V, int n, float dc, float cell,
                                int exact, float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= n) return;
  float LL, MM;
  if (!exact) {
    fipref::Frame fr{V[0], V[1], V[3], V[4], V[8], V[6], V[7], dc};
    fipref::pixel_target(fr, (size_t)i, (size_t)j, (size_t)n, LL, MM);
  } else {
    const ExactMap m = make_map(V, cell);
    double Ld, Md;
    exact_forward(m, (double)(i - n / 2), (double)(j - n / 2), Ld, Md);
    LL = (float)Ld;
    MM = (float)Md;
  }
  out[2 * ((size_t)j * n + i)] = LL;
  out[2 * ((size_t)j * n + i) + 1] = MM;
}

// Maximum of non-negative floats (bit pattern order), NaN ignored.
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
  acc_add<PRECISE>(a, d, (q < 1) ? q : 1.0f);
}

template <bool PRECISE>
__global__ void __launch_bounds__(kThreads) k_trigger(const float* __restrict__ I1,
                                                      const float* __restrict__ I2,
                                                      const float* __restrict__ I3,
                                                      const float* __restrict__ max3, int n,
                                                      int t, int u, int vec,
                                                      float* __restrict__ result) {
  const int lane = threadIdx.x & 31;
  const int b = blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5);
  if (b >= u * u) return;
  const int ti = b / u, tj = b % u;
  Acc a{0.f, 0.f, 0.f, 0.f, 0.f};
  const size_t base = (size_t)ti * t * n + (size_t)tj * t;
  if (vec) {
    const int q = t / 4;  // float4 per tile row
    for (int k = lane; k < t * q; k += 32) {
      const int r = k / q, c = (k % q) * 4;
      const size_t o = base + (size_t)r * n + c;
      const float4 x1 = *reinterpret_cast<const float4*>(I1 + o);
      const float4 x2 = *reinterpret_cast<const float4*>(I2 + o);
      const float4 x3 = *reinterpret_cast<const float4*>(I3 + o);
      acc_pixel<PRECISE>(a, x1.x, x2.x, x3.x);
      acc_pixel<PRECISE>(a, x1.y, x2.y, x3.y);
      acc_pixel<PRECISE>(a, x1.z, x2.z, x3.z);
      acc_pixel<PRECISE>(a, x1.w, x2.w, x3.w);
    }
  } else {
    for (int k = lane; k < t * t; k += 32) {
      const size_t o = base + (size_t)(k / t) * n + (k % t);
      acc_pixel<PRECISE>(a, I1[o], I2[o], I3[o]);
    }
  }
  if (!PRECISE) {
    for (int o = 16; o > 0; o >>= 1) {
      a.s += __shfl_xor_sync(0xffffffffu, a.s, o);
      a.r += __shfl_xor_sync(0xffffffffu, a.r, o);
      a.m = fmaxf(a.m, __shfl_xor_sync(0xffffffffu, a.m, o));
    }
  } else {
    double s = (double)a.s + (double)a.sc, r = (double)a.r + (double)a.rc;
    for (int o = 16; o > 0; o >>= 1) {
      s += __shfl_xor_sync(0xffffffffu, s, o);
      r += __shfl_xor_sync(0xffffffffu, r, o);
      a.m = fmaxf(a.m, __shfl_xor_sync(0xffffffffu, a.m, o));
    }
    a.s = (float)s;
    a.r = (float)r;
    if (lane == 0) {
      double mx = fmax(fmax((double)max3[0], (double)max3[1]), (double)max3[2]);
      double tt = (double)t;
      result[b] = (float)(1.0 - (s / tt / tt) * (double)a.m * (r / tt / tt) / mx / mx);
    }
    return;
  }
  if (lane == 0) {
    const float maxallval = max(max3[0], max(max3[1], max3[2]));
    const size_t us = (size_t)t;
    result[b] = 1 - (a.s / us / us) * a.m * (a.r / us / us) / maxallval / maxallval;
  }
}

inline float cell_degrees(float cell) { return (float)((double)cell / FIP_M_PI * 180); }

}  // namespace

cudaError_t fip_launch_taper(float* taper, const FipGeom& geo, cudaStream_t s) {
  const int cnt = geo.n / 2 + 1;
  k_taper<<<(cnt + kThreads - 1) / kThreads, kThreads, 0, s>>>(taper, (size_t)geo.n,
                                                                (size_t)geo.g);
  return cudaGetLastError();
}

cudaError_t fip_launch_bin(const FipGeom& geo, const float* B, int nb, FipBins& bins,
                           cudaStream_t s) {
  const int ntiles = geo.tiles_r * geo.tiles_c;
  const float scale = geo.cell * (float)(size_t)geo.g;  // r1r2_scale (FIPkernels.cu:584)
  cudaError_t e = cudaMemsetAsync(bins.count, 0, ntiles * sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  const int blocks = (nb + kThreads - 1) / kThreads;
  if (nb > 0)
    k_bin<0><<<blocks, kThreads, 0, s>>>(B, nb, scale, geo.g, geo.tiles_c, bins.count, nullptr,
                                         nullptr);
  k_bin_scan<<<1, kThreads, 0, s>>>(bins.count, ntiles, bins.offset, bins.cursor, bins.work,
                                    bins.nwork, (int)bins.wcap);
  if (nb > 0)
    k_bin<1><<<blocks, kThreads, 0, s>>>(B, nb, scale, geo.g, geo.tiles_c, bins.cursor,
                                         bins.offset, bins.entries);
  return cudaGetLastError();
}

cudaError_t fip_launch_grid(const FipGeom& geo, const float* B, const void* vr, const void* vi,
                            int vis_type, const float* vis_scale, const float* V, int nb,
                            const FipBins& bins, float2* grid, int compensated, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(grid, 0, (size_t)geo.g * geo.hp * sizeof(float2), s);
  if (e != cudaSuccess) return e;
  if (nb <= 0) return cudaSuccess;
  const float scale = geo.cell * (float)(size_t)geo.g;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t smem = (compensated ? 2 : 1) * FIP_GTILE * FIP_GTILE * sizeof(float2);
  const int blocks = sms * (compensated ? 3 : 6);
#define FIP_GRID_CASE(VT, C)                                                                    \
  do {                                                                                          \
    auto kern = k_grid<VT, C>;                                                                  \
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);         \
    kern<<<blocks, kThreads, smem, s>>>(B, vr, vi, vis_scale, V, scale, geo.g, geo.hp,          \
                                        geo.tiles_c, bins.entries, bins.work, bins.nwork, grid); \
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

cudaError_t fip_launch_reproject_scatter(const FipGeom& geo, const float* fft_out,
                                         const float* taper, const float* V, int nb, float* dst,
                                         cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(dst, 0, (size_t)geo.n * geo.n * sizeof(float), s);
  if (e != cudaSuccess) return e;
  dim3 th(32, 8), bl((geo.n + 31) / 32, (geo.n + 7) / 8);
  k_reproject_scatter<<<bl, th, 0, s>>>(fft_out, taper, V, geo.n, geo.g, nb,
                                        cell_degrees(geo.cell), dst);
  return cudaGetLastError();
}

// Target deviation allowance of the FP32 chain from the exact map, in
// destination pixels: half a pixel plus eight ulps of a unit-scale cosine
// expressed in pixels (the chain evaluates cos(theta) ~ R in degrees).
static float chain_delta(float cell) { return 0.5f + 8.0f * 4.76837158e-7f / cell; }

cudaError_t fip_launch_reproject_gather(const FipGeom& geo, const float* fft_out,
                                        const float* taper, const float* V, int nb, float* dst,
                                        unsigned* img_max, int exact_targets, cudaStream_t s) {
  const int tiles = (geo.n + kDT - 1) / kDT;
  const float delta = exact_targets ? 0.25f : chain_delta(geo.cell);
  if (delta > 40.f) return cudaErrorInvalidValue;
  if (exact_targets)
    k_reproject_gather<true><<<tiles * tiles, kThreads, 0, s>>>(
        fft_out, taper, V, geo.n, geo.g, nb, cell_degrees(geo.cell), geo.cell, delta, dst,
        img_max);
  else
    k_reproject_gather<false><<<tiles * tiles, kThreads, 0, s>>>(
        fft_out, taper, V, geo.n, geo.g, nb, cell_degrees(geo.cell), geo.cell, delta, dst,
        img_max);
  return cudaGetLastError();
}

cudaError_t fip_launch_image_max(const float* img, size_t count, unsigned* out, cudaStream_t s) {
  k_image_max<<<1184, kThreads, 0, s>>>(img, count, out);
  return cudaGetLastError();
}

cudaError_t fip_launch_trigger(const FipGeom& geo, const float* I1, const float* I2,
                               const float* I3, const float* max3, float* stats, float* result,
                               int precise, cudaStream_t s) {
  (void)stats;
  const int tiles = geo.u * geo.u;
  const int blocks = (tiles + kThreads / 32 - 1) / (kThreads / 32);
  if (tiles == 0) return cudaSuccess;
  const int vec = (geo.t % 4 == 0) && (geo.n % 4 == 0) &&
                  ((((uintptr_t)I1) | ((uintptr_t)I2) | ((uintptr_t)I3)) & 15) == 0;
  if (precise)
    k_trigger<true><<<blocks, kThreads, 0, s>>>(I1, I2, I3, max3, geo.n, geo.t, geo.u, vec,
                                                result);
  else
    k_trigger<false><<<blocks, kThreads, 0, s>>>(I1, I2, I3, max3, geo.n, geo.t, geo.u, vec,
                                                 result);
  return cudaGetLastError();
}

cudaError_t fip_launch_pixel_targets(const FipGeom& geo, const float* V, float* out,
                                     int exact_targets, cudaStream_t s) {
  dim3 bl((geo.n + kThreads - 1) / kThreads, geo.n);
  k_pixel_targets<<<bl, kThreads, 0, s>>>(V, geo.n, cell_degrees(geo.cell), geo.cell,
                                          exact_targets, out);
  return cudaGetLastError();
}
