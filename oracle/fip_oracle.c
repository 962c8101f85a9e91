/*
 * CPU oracle for the FastImagingPipe snapshot-imaging + tLISI trigger path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA product is
 * compared against (and the CPU baseline that bench.py times on a bounded
 * sample).  The product library never links, loads or calls it.
 *
 * It restates, in plain C with OpenMP, the arithmetic of the reference
 * implementation (egbdfX/FastImagingPipe), each function citing the reference
 * file:line it follows.  The same source is compiled twice:
 *   ORACLE_REAL=double -> *_f64 symbols: the FP64 oracle (exact arithmetic of
 *                         the reference formulas; this is the accuracy target);
 *   ORACLE_REAL=float  -> *_f32 symbols: the same formulas evaluated in FP32 in
 *                         the reference's operation order with IEEE libm
 *                         functions (an estimate of what plain FP32 gives).
 * Where the reference mixes float and double (its M_PI constant is a double
 * literal), the FP32 build keeps those double steps as double.
 *
 * Everything here is single-beam and single-call; it allocates freely.
 */
#include <tgmath.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef ORACLE_REAL
#define ORACLE_REAL double
#endif
typedef ORACLE_REAL real;

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#ifdef ORACLE_F32
#define SFX(name) CAT(name, _f32)
#else
#define SFX(name) CAT(name, _f64)
#endif

#define ORACLE_PI 3.14159265358979323846

/* 14-node quadrature of the ES kernel's Fourier transform used for the grid
 * correction (FIPkernels.cu:14-29).  The values must be identical to the
 * reference's for the correction taper to agree. */
static const float k_nodes[14] = {
    0.9964425f, 0.98130317f, 0.95425928f, 0.91563303f, 0.86589252f,
    0.80564137f, 0.73561088f, 0.65665109f, 0.56972047f, 0.47587422f,
    0.37625152f, 0.27206163f, 0.16456928f, 0.05507929f};
static const float k_weights[14] = {
    0.00912428f, 0.02113211f, 0.03290143f, 0.04427293f, 0.05510735f,
    0.06527292f, 0.07464621f, 0.08311342f, 0.09057174f, 0.09693066f,
    0.10211297f, 0.10605577f, 0.10871119f, 0.11004701f};
static const float k_kernel[14] = {
    7.71381676e-07f, 4.06901586e-06f, 2.09164257e-05f, 1.01923695e-04f,
    4.61199576e-04f, 1.90183990e-03f, 7.02391280e-03f, 2.28652529e-02f,
    6.46725327e-02f, 1.56933676e-01f, 3.23208771e-01f, 5.60024174e-01f,
    8.10934691e-01f, 9.76937533e-01f};

/* FIPkernels.cu:585 */
static const double k_norm = 2.4937047051153827;
/* FIPkernels.cu:205 */
static const double k_beta = 15.3704324328;

typedef struct {
  real re, im;
} cpx;

/* ------------------------------------------------------------------------ */
/* Grid geometry (FIPkernels.cu:583-584)                                    */
/* ------------------------------------------------------------------------ */

/* grid_size = ceil(1.5 * N) evaluated in float, as computeCeil does. */
size_t SFX(oracle_grid_size)(size_t image_size) {
  float g = 1.5f * (float)image_size;
  return (size_t)ceilf(g);
}

/* ------------------------------------------------------------------------ */
/* Mixed-radix FFT (own implementation; any length, fastest for 2^a 3^b)    */
/* ------------------------------------------------------------------------ */

static size_t smallest_factor(size_t n) {
  if (n % 4 == 0) return 4;
  if (n % 2 == 0) return 2;
  for (size_t p = 3; p * p <= n; p += 2)
    if (n % p == 0) return p;
  return n;
}

/* y[0..n) = sum_q x[q*xs] * W^(q k), W = tw[j * twstep] where tw is the
 * root table of the top-level length n0 = n * twstep. */
static void fft_rec(const cpx *x, cpx *y, size_t n, size_t xs, const cpx *tw,
                    size_t twstep, size_t n0) {
  if (n == 1) {
    y[0] = x[0];
    return;
  }
  size_t p = smallest_factor(n), m = n / p;
  for (size_t q = 0; q < p; q++) fft_rec(x + q * xs, y + q * m, m, xs * p, tw, twstep * p, n0);
  cpx tloc[64];
  cpx *t = p <= 64 ? tloc : (cpx *)malloc(p * sizeof(cpx));
  for (size_t k = 0; k < m; k++) {
    for (size_t q = 0; q < p; q++) {
      cpx a = y[q * m + k];
      cpx w = tw[(q * k * twstep) % n0];
      t[q].re = a.re * w.re - a.im * w.im;
      t[q].im = a.re * w.im + a.im * w.re;
    }
    for (size_t r = 0; r < p; r++) {
      real sr = 0, si = 0;
      for (size_t q = 0; q < p; q++) {
        cpx w = tw[((q * r) % p) * m * twstep % n0];
        sr += t[q].re * w.re - t[q].im * w.im;
        si += t[q].re * w.im + t[q].im * w.re;
      }
      y[k + r * m].re = sr;
      y[k + r * m].im = si;
    }
  }
  if (t != tloc) free(t);
}

static cpx *make_roots(size_t n, int sign) {
  cpx *tw = (cpx *)malloc(n * sizeof(cpx));
  for (size_t j = 0; j < n; j++) {
    double a = sign * 2.0 * ORACLE_PI * (double)j / (double)n;
    tw[j].re = (real)cos(a);
    tw[j].im = (real)sin(a);
  }
  return tw;
}

/* In-place unnormalised 2-D inverse DFT (exponent +i) of a row-major g x g
 * complex array: what cufftExecC2C(..., CUFFT_INVERSE) computes
 * (FIPkernels.cu:635-638, 679, 741). */
static void ifft2_inplace(cpx *a, size_t g) {
  cpx *tw = make_roots(g, +1);
#pragma omp parallel
  {
    cpx *in = (cpx *)malloc(g * sizeof(cpx));
    cpx *out = (cpx *)malloc(g * sizeof(cpx));
#pragma omp for schedule(static)
    for (long r = 0; r < (long)g; r++) {
      memcpy(in, a + (size_t)r * g, g * sizeof(cpx));
      fft_rec(in, out, g, 1, tw, 1, g);
      memcpy(a + (size_t)r * g, out, g * sizeof(cpx));
    }
#pragma omp for schedule(static)
    for (long c = 0; c < (long)g; c++) {
      for (size_t r = 0; r < g; r++) in[r] = a[r * g + (size_t)c];
      fft_rec(in, out, g, 1, tw, 1, g);
      for (size_t r = 0; r < g; r++) a[r * g + (size_t)c] = out[r];
    }
    free(in);
    free(out);
  }
  free(tw);
}

/* 1-D transform, exported for the oracle's own known-answer tests. */
void SFX(oracle_fft1d)(const real *in_ri, real *out_ri, size_t n, int sign) {
  cpx *tw = make_roots(n, sign);
  fft_rec((const cpx *)in_ri, (cpx *)out_ri, n, 1, tw, 1, n);
  free(tw);
}

/* ------------------------------------------------------------------------ */
/* Stage: grid-correction taper (FIPkernels.cu:173-186)                     */
/* ------------------------------------------------------------------------ */

/* taper[t], t = 0..N/2:  8/norm * sum_i kernel_i * weight_i *
 * cos(pi * (t/G) * 8 * node_i).  The angle is formed in double as in the
 * reference (M_PI is a double literal there). */
void SFX(oracle_taper)(real *taper, size_t image_size, size_t grid_size) {
  for (size_t t = 0; t < image_size / 2 + 1; t++) {
    real tn = (real)t / (real)grid_size;
    real corr = 0;
    for (int i = 0; i < 14; i++) {
      real angle = (real)(ORACLE_PI * (double)tn * 8.0 * (double)k_nodes[i]);
      corr += (real)k_kernel[i] * (real)k_weights[i] * (real)cos(angle);
    }
    taper[t] = corr * (real)8 / (real)k_norm;
  }
}

/* ------------------------------------------------------------------------ */
/* Stage: convolutional gridding (FIPkernels.cu:67-71, 188-245)            */
/* ------------------------------------------------------------------------ */

static real es_kernel(real beta, real x) {
  real xx = x * x;
  return xx > (real)1 ? (real)0 : (real)exp(beta * (sqrt((real)1 - xx) - (real)1));
}

/* Grids one snapshot onto the row-major g x g complex grid (zeroed here).
 * Visibilities are first divided by |V00*V11 - V01*V10|
 * (computeVisWeighted, FIPkernels.cu:188-195).  Row r1 comes from B[:,0],
 * column r2 from B[:,1]; each tap carries the checkerboard sign
 * (-1)^(r1+r2) (FIPkernels.cu:235-237). */
static void grid_snapshot(cpx *grid, const float *B, const float *vr, const float *vi,
                          const float *V, size_t nb, size_t g, float cell) {
  memset(grid, 0, g * g * sizeof(cpx));
  const long gmin = -(long)g / 2, gmax = ((long)g - 1) / 2, orig = (long)g / 2;
  const real scale = (real)cell * (real)g; /* r1r2_scale (FIPkernels.cu:584) */
  const real inten = (real)fabs((real)V[0] * (real)V[4] - (real)V[1] * (real)V[3]);
  for (size_t v = 0; v < nb; v++) {
    real p1 = (real)B[2 * v] * scale, p2 = (real)B[2 * v + 1] * scale;
    long a0 = (long)ceil(p1 - 4), a1 = (long)floor(p1 + 4);
    long b0 = (long)ceil(p2 - 4), b1 = (long)floor(p2 + 4);
    if (a0 < gmin) a0 = gmin;
    if (a1 > gmax) a1 = gmax;
    if (b0 < gmin) b0 = gmin;
    if (b1 > gmax) b1 = gmax;
    if (a0 > a1 || b0 > b1) continue;
    real wr = (real)vr[v] / inten, wi = (real)vi[v] / inten;
    real k1[16], k2[16];
    for (long r = a0; r <= a1; r++) k1[r - a0] = es_kernel((real)k_beta, ((real)r - p1) * (real)0.25);
    for (long r = b0; r <= b1; r++) k2[r - b0] = es_kernel((real)k_beta, ((real)r - p2) * (real)0.25);
    for (long r1 = a0; r1 <= a1; r1++)
      for (long r2 = b0; r2 <= b1; r2++) {
        real kv = k1[r1 - a0] * k2[r2 - b0];
        if ((r1 + r2) & 1) kv = -kv;
        size_t off = (size_t)((r1 + orig) * (long)g + (r2 + orig));
        grid[off].re += wr * kv;
        grid[off].im += wi * kv;
      }
  }
}

/* Exported: the checkerboarded grid of one snapshot (interleaved re/im). */
void SFX(oracle_grid)(real *grid_ri, const float *B, const float *vr, const float *vi,
                      const float *V, size_t nb, size_t g, float cell) {
  grid_snapshot((cpx *)grid_ri, B, vr, vi, V, nb, g, cell);
}

/* ------------------------------------------------------------------------ */
/* Stage: crop, checkerboard, correction, abs (FIPkernels.cu:256-287)       */
/* ------------------------------------------------------------------------ */

static void crop_correct(real *dirty_pre, const cpx *grid, const real *taper, size_t n, size_t g) {
  const long h = (long)n / 2;
  const size_t gc = g * g / 2 + g / 2;
#pragma omp parallel for schedule(static)
  for (long yy = 0; yy < (long)n; yy++) {
    long y = yy - h;
    for (long xx = 0; xx < (long)n; xx++) {
      long x = xx - h;
      real px = grid[(long)gc + y * (long)g + x].re;
      if ((labs(x) + labs(y)) & 1) px = -px;
      real den = taper[labs(x)] * taper[labs(y)] * (real)k_norm * (real)k_norm;
      px *= (real)1 / den;
      dirty_pre[(size_t)yy * n + (size_t)xx] = (real)fabs(px);
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Stage: plane -> sky reprojection (FIPkernels.cu:73-171, 289-413)         */
/* ------------------------------------------------------------------------ */

#define WCS_TOL 1e-10

static real sind_(real a) {
  if (fmod(a, (real)90) == 0) {
    int i = (int)fabs(floor(a / (real)90 - (real)0.5)) % 4;
    switch (i) {
      case 0: return 1;
      case 1: return 0;
      case 2: return -1;
      default: return 0;
    }
  }
  return (real)sin((real)((double)a * ORACLE_PI / 180.0));
}

static real cosd_(real a) {
  if (fmod(a, (real)90) == 0) {
    int i = (int)fabs(floor(a / (real)90 + (real)0.5)) % 4;
    switch (i) {
      case 0: return 1;
      case 1: return 0;
      case 2: return -1;
      default: return 0;
    }
  }
  return (real)cos((real)((double)a * ORACLE_PI / 180.0));
}

static void sincosd_(real a, real *s, real *c) {
  if (fmod(a, (real)90) == 0) {
    int i = (int)fabs(floor(a / (real)90 + (real)0.5)) % 4;
    switch (i) {
      case 0: *s = 0; *c = 1; break;
      case 1: *s = a > 0 ? 1 : -1; *c = 0; break;
      case 2: *s = 0; *c = -1; break;
      default: *s = a > 0 ? -1 : 1; *c = 0; break;
    }
    return;
  }
  *s = (real)sin((real)((double)a * ORACLE_PI / 180.0));
  *c = (real)cos((real)((double)a * ORACLE_PI / 180.0));
}

static real atan2d_(real y, real x) {
  if (y == 0) return x >= 0 ? 0 : 180;
  if (x == 0) return y > 0 ? 90 : -90;
  return (real)((double)(real)(atan2(y, x) * (real)180) / ORACLE_PI);
}

static real acosd_(real v) {
  if (v >= 1 && v - 1 < WCS_TOL) return 0;
  if (v == 0) return 90;
  if (v <= -1 && v + 1 > -WCS_TOL) return 180;
  return (real)((double)(real)(acos(v) * (real)180) / ORACLE_PI);
}

static real asind_(real v) {
  if (v <= -1 && v + 1 > -WCS_TOL) return -90;
  if (v == 0) return 0;
  if (v >= 1 && v - 1 < WCS_TOL) return 90;
  return (real)((double)(real)(asin(v) * (real)180) / ORACLE_PI);
}

/* Maps source pixel (column i, row j) to its target position (LL, MM)
 * relative to the image centre: coordschange (FIPkernels.cu:289-299)
 * followed by the SIN/slant-SIN p2p step (FIPkernels.cu:301-376). */
static void pixel_target(size_t i, size_t j, const float *V, size_t n, float cell,
                         real *LL, real *MM) {
  const real h = (real)(n / 2);
  const real a22 = (real)fabs((real)V[8]);
  real p1 = (-(real)V[0] * ((real)i - h) + (real)V[3] * ((real)j - h)) / a22 + h;
  real p2 = (-(real)V[1] * ((real)i - h) + (real)V[4] * ((real)j - h)) / a22 + h;

  const real xi = (real)V[6] / (real)V[8];
  const real eta = (real)V[7] / (real)V[8];
  const real dc = (real)((double)cell / ORACLE_PI * 180.0);
  const real half1 = (real)n / (real)2 + (real)1;
  real x = -dc * (p1 - half1);
  real y = dc * (p2 - half1);
  real r0 = (real)(180.0 / ORACLE_PI);
  real x0 = x / r0, y0 = y / r0;
  real r2 = x0 * x0 + y0 * y0;
  real phi = r2 != 0 ? atan2d_(x0, -y0) : 0;
  real theta;
  int mapped = 1;
  if (r2 < (real)0.5)
    theta = acosd_((real)sqrt(r2));
  else if (r2 <= 1)
    theta = asind_((real)sqrt((real)1 - r2));
  else {
    mapped = 0;
    theta = 0;
  }
  if (mapped) {
    real sphi, cphi;
    sincosd_(phi, &sphi, &cphi);
    x = sphi;
    y = cphi;
    real t = (real)((double)(((real)90 - (real)fabs(theta)) / (real)180) * ORACLE_PI);
    real z, costhe;
    if (t < (real)1.0e-5) {
      z = theta > 0 ? t * t / 2 : (real)2 - t * t / 2;
      costhe = t;
    } else {
      z = (real)1 - sind_(theta);
      costhe = cosd_(theta);
    }
    real r = r0 * costhe;
    real w = xi * xi + eta * eta;
    if (w == 0) {
      x = r * x;
      y = -r * y;
    } else {
      z = z * r0;
      x = r * x + xi * z;
      y = -r * y + eta * z;
    }
    p1 = (real)-1 / dc * x + (real)n / (real)2 + (real)1;
    p2 = (real)1 / dc * y + (real)n / (real)2 + (real)1;
  }
  *LL = p1 - h;
  *MM = p2 - h;
}

/* Exported: target positions of every source pixel, [N*N][2] indexed
 * (row j, column i) -> (j*N + i). */
void SFX(oracle_pixel_targets)(real *out, const float *V, size_t n, float cell) {
#pragma omp parallel for schedule(static)
  for (long j = 0; j < (long)n; j++)
    for (size_t i = 0; i < n; i++) {
      real L, M;
      pixel_target(i, (size_t)j, V, n, cell, &L, &M);
      out[2 * ((size_t)j * n + i)] = L;
      out[2 * ((size_t)j * n + i) + 1] = M;
    }
}

/* Forward bilinear splat of dirty_pre / nb into dirty (FIPkernels.cu:378-413).
 * Serial in the destination to keep the oracle deterministic. */
static void reproject(real *dirty, const real *dirty_pre, const float *V, size_t n, float cell,
                      size_t nb) {
  memset(dirty, 0, n * n * sizeof(real));
  const real inv_nb = (real)1 / (real)nb;
  const real lim = (real)(n / 2 - 1);
  const long h = (long)(n / 2);
  real *tgt = (real *)malloc(n * n * 2 * sizeof(real));
  SFX(oracle_pixel_targets)(tgt, V, n, cell);
  for (size_t j = 0; j < n; j++)
    for (size_t i = 0; i < n; i++) {
      real LL = tgt[2 * (j * n + i)], MM = tgt[2 * (j * n + i) + 1];
      real val = dirty_pre[j * n + i] * inv_nb;
      if (fabs(LL) < lim && fabs(MM) < lim) {
        long fl = (long)floor(LL), cl = (long)ceil(LL);
        long fm = (long)floor(MM), cm = (long)ceil(MM);
        real wl0 = (real)1 - LL + (real)fl, wl1 = LL - (real)fl;
        real wm0 = (real)1 - MM + (real)fm, wm1 = MM - (real)fm;
        dirty[(size_t)((h + fm) * (long)n + h + fl)] += wl0 * wm0 * val;
        dirty[(size_t)((h + cm) * (long)n + h + fl)] += wl0 * wm1 * val;
        dirty[(size_t)((h + fm) * (long)n + h + cl)] += wl1 * wm0 * val;
        dirty[(size_t)((h + cm) * (long)n + h + cl)] += wl1 * wm1 * val;
      }
    }
  free(tgt);
}

/* ------------------------------------------------------------------------ */
/* One snapshot end to end                                                  */
/* ------------------------------------------------------------------------ */

/* Images one snapshot: dirty (N*N, row-major) and, if dirty_pre_out is not
 * NULL, the corrected pre-reprojection image.  Returns max(0, max(dirty))
 * (max_large/max_small, FIPkernels.cu:431-497). */
real SFX(oracle_image_snapshot)(real *dirty, real *dirty_pre_out, const float *B,
                                const float *vr, const float *vi, const float *V, size_t nb,
                                size_t n, float cell) {
  size_t g = SFX(oracle_grid_size)(n);
  cpx *grid = (cpx *)malloc(g * g * sizeof(cpx));
  real *taper = (real *)malloc((n / 2 + 1) * sizeof(real));
  real *pre = dirty_pre_out ? dirty_pre_out : (real *)malloc(n * n * sizeof(real));
  SFX(oracle_taper)(taper, n, g);
  grid_snapshot(grid, B, vr, vi, V, nb, g, cell);
  ifft2_inplace(grid, g);
  crop_correct(pre, grid, taper, n, g);
  reproject(dirty, pre, V, n, cell, nb);
  real mx = 0;
  for (size_t k = 0; k < n * n; k++) mx = dirty[k] > mx ? dirty[k] : mx;
  free(grid);
  free(taper);
  if (!dirty_pre_out) free(pre);
  return mx;
}

/* ------------------------------------------------------------------------ */
/* Stage: FI trigger, tLISI (FIPkernels.cu:415-552, 806-840)                */
/* ------------------------------------------------------------------------ */

/* D = | |I1-I2| - |I2-I3| |; I2 clamped to C=1e-6 where <= 0 (after D);
 * per T x T tile (row-major tile index, U = N/T per side):
 * S = sum D, M = max(0, max D), R = sum min(D/I2c, 1) (NaN -> 1);
 * out = 1 - (S/T/T) * M * (R/T/T) / mx / mx with mx = max(maxall[0..2]). */
void SFX(oracle_tlisi)(real *out, const real *I1, const real *I2, const real *I3,
                       const real *maxall, size_t n, size_t t) {
  const size_t u = n / t;
  real mx = maxall[0];
  if (maxall[1] > mx) mx = maxall[1];
  if (maxall[2] > mx) mx = maxall[2];
  const real C = (real)1e-6f;
#pragma omp parallel for schedule(static)
  for (long b = 0; b < (long)(u * u); b++) {
    size_t ti = (size_t)b / u, tj = (size_t)b % u;
    real S = 0, M = 0, R = 0;
    for (size_t r = 0; r < t; r++)
      for (size_t c = 0; c < t; c++) {
        size_t k = (ti * t + r) * n + tj * t + c;
        real d = (real)fabs((real)fabs(I1[k] - I2[k]) - (real)fabs(I2[k] - I3[k]));
        real s2 = I2[k] <= 0 ? C : I2[k];
        S += d;
        M = d > M ? d : M;
        real q = d / s2;
        R += q < 1 ? q : 1;
      }
    out[b] = (real)1 - (S / (real)t / (real)t) * M * (R / (real)t / (real)t) / mx / mx;
  }
}

/* The reference entry point's computation (FIPkernels.cu:554-862): images the
 * first three snapshots and returns their tLISI matrix.  images (3*N*N) and
 * maxall (3) are optional outputs. */
void SFX(oracle_fipipe)(real *result, real *images, real *maxall_out, const float *vr,
                        const float *vi, const float *B, const float *V, size_t nb, size_t n,
                        float cell, size_t t) {
  real *img = images ? images : (real *)malloc(3 * n * n * sizeof(real));
  real mx[3];
  for (int k = 0; k < 3; k++)
    mx[k] = SFX(oracle_image_snapshot)(img + (size_t)k * n * n, NULL, B + (size_t)k * nb * 2,
                                       vr + (size_t)k * nb, vi + (size_t)k * nb,
                                       V + (size_t)k * 9, nb, n, cell);
  SFX(oracle_tlisi)(result, img, img + n * n, img + 2 * n * n, mx, n, t);
  if (maxall_out) memcpy(maxall_out, mx, sizeof(mx));
  if (!images) free(img);
}

/* ------------------------------------------------------------------------ */
/* Plane projection (SVDPreprocessKernels.cu:41-206; SVD_MFS.py:38-110)     */
/* ------------------------------------------------------------------------ */

/* Cyclic Jacobi eigen-decomposition of a symmetric 3x3 (double).  Returns
 * eigenvalues ascending in w and the matching eigenvectors as columns of Q. */
static void jacobi3(const double A_in[9], double w[3], double Q[9]) {
  double A[9];
  memcpy(A, A_in, sizeof(A));
  for (int i = 0; i < 9; i++) Q[i] = (i % 4 == 0) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 64; sweep++) {
    double off = A[1] * A[1] + A[2] * A[2] + A[5] * A[5];
    if (off < 1e-300) break;
    for (int p = 0; p < 2; p++)
      for (int q = p + 1; q < 3; q++) {
        double apq = A[p * 3 + q];
        if (fabs(apq) < 1e-300) continue;
        double app = A[p * 3 + p], aqq = A[q * 3 + q];
        double tau = (aqq - app) / (2.0 * apq);
        double tt = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
        double c = 1.0 / sqrt(1.0 + tt * tt), s = tt * c;
        for (int k = 0; k < 3; k++) {
          double akp = A[k * 3 + p], akq = A[k * 3 + q];
          A[k * 3 + p] = c * akp - s * akq;
          A[k * 3 + q] = s * akp + c * akq;
        }
        for (int k = 0; k < 3; k++) {
          double apk = A[p * 3 + k], aqk = A[q * 3 + k];
          A[p * 3 + k] = c * apk - s * aqk;
          A[q * 3 + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 3; k++) {
          double qkp = Q[k * 3 + p], qkq = Q[k * 3 + q];
          Q[k * 3 + p] = c * qkp - s * qkq;
          Q[k * 3 + q] = s * qkp + c * qkq;
        }
      }
  }
  double d[3] = {A[0], A[4], A[8]};
  int idx[3] = {0, 1, 2};
  for (int a = 0; a < 3; a++)
    for (int b = a + 1; b < 3; b++)
      if (d[idx[b]] < d[idx[a]]) {
        int tmp = idx[a];
        idx[a] = idx[b];
        idx[b] = tmp;
      }
  double Qs[9];
  for (int c = 0; c < 3; c++) {
    w[c] = d[idx[c]];
    for (int r = 0; r < 3; r++) Qs[r * 3 + c] = Q[r * 3 + idx[c]];
  }
  memcpy(Q, Qs, sizeof(Qs));
}

/* uvw: [rows][3] metres; freqs: [chans] Hz; sample s = row + chan * rows
 * (SVDPreprocessMain.cpp:36-38).  Outputs B [samples][2] (uncentred
 * projection onto the two principal axes) and V [3][3] (rows: principal
 * axes, third row their cross product), with each principal axis signed so
 * that its largest-magnitude component is positive
 * (SVDPreprocessKernels.cu:167-206).  FP64 throughout. */
void SFX(oracle_plane_fit)(double *B, double *V, const float *uvw, const float *freqs, size_t rows,
                           size_t chans) {
  const size_t ns = rows * chans;
  const double c_light = 299792458.0;
  double mean[3] = {0, 0, 0};
  for (size_t s = 0; s < ns; s++) {
    size_t r = s % rows, ch = s / rows;
    double sc = (double)freqs[ch] / c_light;
    for (int a = 0; a < 3; a++) mean[a] += (double)uvw[r * 3 + a] * sc;
  }
  for (int a = 0; a < 3; a++) mean[a] /= (double)ns;
  double C[9] = {0};
  for (size_t s = 0; s < ns; s++) {
    size_t r = s % rows, ch = s / rows;
    double sc = (double)freqs[ch] / c_light;
    double x[3];
    for (int a = 0; a < 3; a++) x[a] = (double)uvw[r * 3 + a] * sc - mean[a];
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) C[a * 3 + b] += x[a] * x[b];
  }
  double w[3], Q[9];
  jacobi3(C, w, Q);
  double basis[6];
  for (int a = 0; a < 3; a++) {
    basis[0 * 3 + a] = Q[a * 3 + 2];
    basis[1 * 3 + a] = Q[a * 3 + 1];
  }
  for (int comp = 0; comp < 2; comp++) {
    int ma = 0;
    double mv = fabs(basis[comp * 3]);
    for (int a = 1; a < 3; a++)
      if (fabs(basis[comp * 3 + a]) > mv) {
        mv = fabs(basis[comp * 3 + a]);
        ma = a;
      }
    if (basis[comp * 3 + ma] < 0)
      for (int a = 0; a < 3; a++) basis[comp * 3 + a] = -basis[comp * 3 + a];
  }
  for (int a = 0; a < 6; a++) V[a] = basis[a];
  V[6] = V[1] * V[5] - V[2] * V[4];
  V[7] = V[2] * V[3] - V[0] * V[5];
  V[8] = V[0] * V[4] - V[1] * V[3];
  for (size_t s = 0; s < ns; s++) {
    size_t r = s % rows, ch = s / rows;
    double sc = (double)freqs[ch] / c_light;
    double x[3];
    for (int a = 0; a < 3; a++) x[a] = (double)uvw[r * 3 + a] * sc;
    B[2 * s] = x[0] * basis[0] + x[1] * basis[1] + x[2] * basis[2];
    B[2 * s + 1] = x[0] * basis[3] + x[1] * basis[4] + x[2] * basis[5];
  }
}

/* Flag/weight Stokes-I collapse (SVDPreprocessKernels.cu:208-237;
 * SVD_MFS.py:77-95): weighted mean of polarisations 0 and 3, 0 when both
 * are flagged or weightless. */
void SFX(oracle_collapse)(float *out_re, float *out_im, const float *v0r, const float *v0i,
                          const float *v3r, const float *v3i, const uint8_t *f0,
                          const uint8_t *f3, const float *w0, const float *w3, size_t ns) {
  for (size_t s = 0; s < ns; s++) {
    double a = f0[s] ? 0.0 : (double)w0[s];
    double b = f3[s] ? 0.0 : (double)w3[s];
    double ws = a + b;
    if (ws > 0) {
      out_re[s] = (float)(((double)v0r[s] * a + (double)v3r[s] * b) / ws);
      out_im[s] = (float)(((double)v0i[s] * a + (double)v3i[s] * b) / ws);
    } else {
      out_re[s] = 0.0f;
      out_im[s] = 0.0f;
    }
  }
}

int SFX(oracle_num_threads)(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
