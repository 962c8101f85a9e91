// Launchers of the device stages, shared by the host orchestration.
// All launchers are asynchronous on `s` and return the launch status.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>

#include <string>

#include "fip_common.cuh"
#include "fip_fft.cuh"

// Records the calling thread's last error message and returns `code`.
int fip_set_error(int code, const std::string& msg);

// Scratch of the tile-binned gridder for one image size.
struct FipBins {
  unsigned* count;    // [ntiles] entries per grid tile
  unsigned* offset;   // [ntiles + 1] exclusive scan of count
  unsigned* cursor;   // [ntiles] scatter cursors
  unsigned* entries;  // [cap] (vis << 1 | mirrored), grouped by tile
  int4* work;         // [wcap] (tile, begin, end, single-chunk flag)
  unsigned* nwork;    // [1] number of work items
  unsigned* bbox;     // [4] max |r1|, max half-plane column, (unused),
                      // image maximum (float bits, set by the transform)
  unsigned* multi;    // [ntiles] tiles split over several work items
  unsigned* nmulti;   // [1]
  size_t cap;         // capacity of entries
  size_t wcap;        // capacity of work
};

// FIP_VIS_RAW: FP32 two-polarisation samples (FipRawVis), collapsed to
// Stokes I as the gridder loads them.
enum FipVisType { FIP_VIS_F32 = 0, FIP_VIS_F16 = 1, FIP_VIS_BF16 = 2, FIP_VIS_RAW = 3 };

// ---- plain FP32 form (reference-faithful arithmetic, fip_plain.cu) ----
cudaError_t fip_launch_taper(float* taper, const FipGeom& geo, cudaStream_t s);
cudaError_t fip_launch_bin(const FipGeom& geo, const float* B, int nb, FipBins& bins,
                           cudaStream_t s);
// Kernels fip_launch_bin launches for nb > 0.
int fip_bin_launches(const FipGeom& geo);
// ctas_per_sm: persistent gridder CTAs per SM (0 = the most that fit,
// fip_grid_max_ctas_per_sm).
// vis_type FIP_VIS_RAW: vr, vi unused, the samples are *raw.
cudaError_t fip_launch_grid(const FipGeom& geo, const float* B, const void* vr, const void* vi,
                            int vis_type, const float* vis_scale, const float* V, int nb,
                            const FipBins& bins, float2* grid, int compensated, cudaStream_t s,
                            int ctas_per_sm = 0, const FipRawVis* raw = nullptr);
int fip_grid_max_ctas_per_sm(int compensated);
// Zeroes the split tiles of `count` snapshots of one geometry (their grids
// and split-tile lists at base + k * stride) before a batched gridding launch.
cudaError_t fip_launch_zero_batch(const FipGeom& geo, const unsigned* multi, size_t multi_stride,
                                  const unsigned* nmulti, float2* grid, size_t grid_stride,
                                  int count, cudaStream_t s);
// One persistent gridding launch over the work items of all the batch's
// snapshots (in.s[k]: inputs, bins, grid and geometry of snapshot k).
cudaError_t fip_launch_grid_batch(const FipGridBatch& in, int vis_type, int compensated,
                                  cudaStream_t s, int ctas_per_sm = 0);
// values_per_thread: 8 or 16 (0 = the default for the length).
bool fip_fft_plan(int g, fipfft::Plan& p, int values_per_thread = 0);
// Band-pruned inverse FFT: column pass (band grid -> colbuf [G/2+1][N]) and
// row pass with the crop + correction epilogue (colbuf -> pre [N*N]).
// Batched (batch > 1): snapshot k's grid, bbox (4 words) and colbuf at
// base + k * stride.
cudaError_t fip_launch_fft_cols(const FipGeom& geo, const float2* grid, const unsigned* bbox,
                                float2* colbuf, const float2* twiddles, const fipfft::Plan& plan,
                                cudaStream_t s, int batch = 1, size_t grid_stride = 0,
                                size_t col_stride = 0);
// Also folds the image maximum into bbox[3] (float bits, zeroed by the
// binning), which the gather reprojection reads.
cudaError_t fip_launch_fft_rows(const FipGeom& geo, const float2* colbuf, unsigned* bbox,
                                const float* taper, const float2* twiddles,
                                const fipfft::Plan& plan, float* pre, cudaStream_t s,
                                int batch = 1, size_t col_stride = 0, size_t pre_stride = 0);
// Crop + correction of an in-place cuFFT C2R output -> pre [N*N].
cudaError_t fip_launch_correct_c2r(const FipGeom& geo, const float* fft_out, const float* taper,
                                   float* pre, unsigned* pre_max, cudaStream_t s);
// The reference's pixel mapping of every source pixel -> targets [N*N].
// theta_tab: the table fip_launch_theta_table fills (bit-identical results,
// fewer instructions), or null.
cudaError_t fip_launch_targets(const FipGeom& geo, const float* V, const float2* theta_tab,
                               float2* targets, cudaStream_t s);
// The pixel-mapping kernel's entry (to tell its graph nodes apart).
const void* fip_targets_kernel();
// Entries of the theta-terms table of the pixel mapping, and its fill.
size_t fip_theta_table_elems();
cudaError_t fip_launch_theta_table(float2* tab, cudaStream_t s);
// Source-major reprojection: one thread per source pixel, atomics into a
// zeroed destination (the reference's scheme).
cudaError_t fip_launch_reproject_scatter(const FipGeom& geo, const float* pre, const float* V,
                                         int nb, float* dst, cudaStream_t s);
// Destination-tile-major reprojection: every destination tile gathers its
// candidate source pixels, splats in shared memory and is stored once.  Also
// records the image maximum into *img_max (atomic max, caller zeroes it).
bool fip_gather_supported(const FipGeom& geo, int exact_targets);
// The trigger of a three-snapshot call fused into its three reprojections:
// the images I1, I2, I3 (dst is one of them), a count per 64 x 64 region
// (fip_trigger_fuse_counts of them, zeroed before the first of the three
// launches) and the per-tile statistics [U*U][3], which
// fip_launch_trigger_combine turns into tLISI once the three are done.  The
// statistics are reduced in k_trigger's order, so the results are the
// separate trigger's bit for bit.  Needs fip_trigger_fusable(geo).
struct FipFuse {
  const float* img[3];
  unsigned* count;
  double* stats;
};
bool fip_trigger_fusable(const FipGeom& geo);
size_t fip_trigger_fuse_counts(const FipGeom& geo);
cudaError_t fip_launch_trigger_combine(const FipGeom& geo, const double* stats,
                                       const float* max3, float* result, int precise,
                                       cudaStream_t s);
// pre_max: maximum of pre (float bits), from the transform's epilogue.
// err (or null): set to nonzero when a tile lies outside the gather's domain
// (fip_gather_domain_ok); its image is then not to be trusted.
// fuse (or null): fuse the call's trigger into this reprojection.
cudaError_t fip_launch_reproject_gather(const FipGeom& geo, const float* pre,
                                        const float2* targets, const float* V, int nb,
                                        const unsigned* pre_max, float* dst, unsigned* img_max,
                                        int exact_targets, cudaStream_t s, unsigned* err,
                                        const FipFuse* fuse = nullptr);
// Whether the plane-to-sky map of basis V (host, row-major 3 x 3) stays in
// the tile gather's domain over an N x N image: well inside the horizon and
// without folds.  Outside it only the source scatter reprojects correctly.
bool fip_gather_domain_ok(const float* V, int n, float cell);
cudaError_t fip_launch_image_max(const float* img, size_t count, unsigned* out, cudaStream_t s);
// Trigger: per-tile statistics of (I1, I2, I3) and the tLISI combine.
cudaError_t fip_launch_trigger(const FipGeom& geo, const float* I1, const float* I2,
                               const float* I3, const float* max3, float* stats,
                               float* result, int precise, cudaStream_t s);
// Same, the three maxima at separate addresses.
cudaError_t fip_launch_trigger3(const FipGeom& geo, const float* I1, const float* I2,
                                const float* I3, const float* m1, const float* m2,
                                const float* m3, float* result, int precise, cudaStream_t s);
// Batched trigger over a linear ring of images (stride N*N): triple k is
// images k, k+1, k+2 with maxima[k .. k+2], result k at results + k * U*U.
// The plain form with count >= 3 and T <= 32 (T % 4 == 0) streams each tile's
// slices through registers, each image of the ring read once, bit-identical
// to the per-triple loads.
cudaError_t fip_launch_trigger_batch(const FipGeom& geo, const float* images, const float* maxima,
                                     int count, float* results, int precise, cudaStream_t s);
// Process-wide: the streamed window on (default) or off.
void fip_trigger_stream_enable(int on);
int fip_trigger_stream_enabled();
// mode 0: the FP32 chain (theta_tab as in fip_launch_targets), 1: the exact
// closed form, 2: the FP32 chain evaluated without the table.
cudaError_t fip_launch_pixel_targets(const FipGeom& geo, const float* V, float* out,
                                     int mode, const float2* theta_tab, cudaStream_t s);

// ---- plane projection (fip_precise.cu) ----
cudaError_t fip_launch_plane_project(const float* uvw, const float* freqs, size_t rows,
                                     size_t chans, double* work, float* B, float* V,
                                     cudaStream_t s);
cudaError_t fip_launch_collapse(const float* v0r, const float* v0i, const float* v3r,
                                const float* v3i, const unsigned char* f0,
                                const unsigned char* f3, const float* w0, const float* w3,
                                float* out_re, float* out_im, size_t ns, cudaStream_t s);
// FP16/BF16 storage of a snapshot's visibilities (one launch): scales
// receives one power-of-two scale per block of FIP_QBLOCK samples
// ([fip_qblocks(nb)]), out_re/out_im the values divided by their block's.
cudaError_t fip_launch_quantize(const float* vr, const float* vi, size_t nb, int vis_type,
                                void* out_re, void* out_im, float* scales, cudaStream_t s);
// The same from raw two-polarisation samples, collapsed to Stokes I on load.
cudaError_t fip_launch_quantize_raw(const FipRawVis& raw, size_t nb, int vis_type, void* out_re,
                                    void* out_im, float* scales, cudaStream_t s);
