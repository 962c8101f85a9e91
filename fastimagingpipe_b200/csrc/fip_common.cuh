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

// Snapshot descriptor for batched launches (device-resident arrays).
struct FipSnapDesc {
  const void* vis_re;   // float or half/bf16 depending on storage
  const void* vis_im;
  const float* B;       // [nb][2]
  const float* V;       // [9]
  int nb;               // visibilities of this snapshot
  float vis_scale;      // multiplier for reduced-precision storage (1 for FP32)
};
