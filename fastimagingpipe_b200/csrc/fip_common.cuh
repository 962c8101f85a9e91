// Shared definitions of the B200 imaging + trigger path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#define FIP_M_PI 3.14159265358979323846

// FIPkernels.cu:585 and :205
#define FIP_CONV_NORM 2.4937047051153827
#define FIP_ES_BETA 15.3704324328
#define FIP_SUPPORT 8
#define FIP_TRIGGER_FLOOR 1e-6f  // setNonPositiveToC's C (FIPkernels.cu:811)

// Grid tiles used by the binned gridder (cells of the half-plane grid).
#define FIP_GTILE 64
#define FIP_GCHUNK 256  // virtual visibilities per gridding work item

// Geometry of one image size.  The uv grid is the Hermitian half plane
// G x (G/2+1) complex (row stride hp = G/2+1 complex = G+2 floats), which is
// also the in-place C2R output (G x G real, row stride G+2 floats).
struct FipGeom {
  int n;       // image side N
  int g;       // grid side G = ceil(1.5 N)
  int hp;      // G/2 + 1 (complex columns of the half plane)
  int t;       // trigger tile side T
  int u;       // N / T tiles per side
  int tiles_r; // grid tiles along rows
  int tiles_c; // grid tiles along half-plane columns
  float cell;  // cell size (rad)
  int layout;  // grid layout: 1 = band, column-major [col][row] (pruned FFT);
               // 0 = full half plane, row-major (cuFFT C2R fallback)
};

// Raw two-polarisation visibilities of one snapshot (device arrays of nb
// samples in the preprocessing's sample order): polarisations 0 and 3 (XX,
// YY), their flags (nonzero = flagged) and weights.
struct FipRawVis {
  const float* v0r;
  const float* v0i;
  const float* v3r;
  const float* v3i;
  const unsigned char* f0;
  const unsigned char* f3;
  const float* w0;
  const float* w3;
};

// Stokes-I collapse of sample s (SVDPreprocessKernels.cu:208-237, SVD_MFS.py
// :77-95): the weighted mean of polarisations 0 and 3 over their unflagged
// weights, 0 when both vanish.  The roundings are spelled out so that every
// translation unit (fast-math or not) gives the same bits.
__device__ __forceinline__ void fip_collapse_sample(const FipRawVis& r, size_t s, float& re,
                                                    float& im) {
  const float a = r.f0[s] ? 0.0f : r.w0[s];
  const float b = r.f3[s] ? 0.0f : r.w3[s];
  const float ws = __fadd_rn(a, b);
  if (ws > 0.0f) {
    re = __fdiv_rn(__fmaf_rn(r.v0r[s], a, __fmul_rn(r.v3r[s], b)), ws);
    im = __fdiv_rn(__fmaf_rn(r.v0i[s], a, __fmul_rn(r.v3i[s], b)), ws);
  } else {
    re = 0.0f;
    im = 0.0f;
  }
}

// Reduced (FP16/BF16) visibility storage keeps v / scale with one
// power-of-two scale per block of 2^FIP_QBLOCK_SHIFT samples, which puts the
// block's max-abs in [2^14, 2^15): a power of two leaves the FP16/BF16
// rounding of every normal value as it would be unscaled, and a block scale
// needs no pass over the whole snapshot before the conversion.
#define FIP_QBLOCK_SHIFT 10
#define FIP_QBLOCK (1 << FIP_QBLOCK_SHIFT)
__host__ __device__ constexpr size_t fip_qblocks(size_t nb) {
  return (nb + FIP_QBLOCK - 1) / FIP_QBLOCK;
}

// Batched launches: at most FIP_MAX_BATCH snapshots, of one or several
// image sizes.
#define FIP_MAX_BATCH 64

// One snapshot of a batched gridding launch: its inputs, bins and grid, and
// its grid geometry (snapshots of a launch may differ in image size).
struct FipGridSnap {
  const float* B;           // [nb][2]
  const void* vr;           // float, or half/bf16 for reduced storage
  const void* vi;
  const float* V;           // [9]
  const float* vis_scale;   // reduced storage: the block scales (fip_qblocks), or null
  const unsigned* entries;  // the snapshot's bins (FipBins)
  const int4* work;
  const unsigned* nwork;
  float2* grid;             // its half-plane grid
  float scale;              // cell * G
  int g, hp, tiles_c;
  int layout;               // grid layout (FipGeom::layout)
};

// The snapshots of one batched gridding launch (a kernel parameter of
// about 5.6 KB).
struct FipGridBatch {
  int count;
  FipGridSnap s[FIP_MAX_BATCH];
};
