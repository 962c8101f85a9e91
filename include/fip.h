/*
 * fip.h -- C ABI of the B200-native snapshot imaging + tLISI trigger library
 * (libfip_b200.so), a drop-in for FastImagingPipe's imaging/trigger path.
 *
 * All functions return 0 (FIP_OK) on success or a fip_status code; the
 * message of the last failure on the calling thread is fip_last_error().
 * Device pointers are plain CUDA device addresses; `stream` is a cudaStream_t
 * (NULL = the legacy default stream).  No torch types cross this boundary.
 */
#ifndef FIP_B200_H
#define FIP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
/*
 * Drop-in replacement of the reference entry point, same C++ signature and
 * therefore the same linker symbol (_Z6FIpipePfS_S_S_S_mmmfm on x86-64).
 * Replaces: int FIpipe(...) declared at pipe_interface.cpp:8, defined at
 * FIPkernels.cu:554-557.
 * Inputs are caller-owned host arrays, snapshot-concatenated:
 *   Visreal, Visimag [num_snapshots * num_baselines]
 *   Bin              [num_snapshots * num_baselines * 2]  (row-major pairs)
 *   Vin              [num_snapshots * 9]                  (row-major 3x3)
 * result_array       [(image_size / unit_size)^2], row-major tLISI matrix.
 * As in the reference, the first three snapshots are imaged and their tLISI
 * computed (FIPkernels.cu:647, 806-851).  Returns 0 on success; unlike the
 * reference (which always returns 0, FIPkernels.cu:861) a failure returns a
 * fip_status code.  Inputs are never written (the reference copies them too).
 */
int FIpipe(float* Visreal, float* Visimag, float* Bin, float* Vin, float* result_array,
           size_t num_baselines, size_t image_size, size_t num_snapshots, float cell_size,
           size_t unit_size);
extern "C" {
#endif

typedef enum {
  FIP_OK = 0,
  FIP_ERR_ARG = 1,         /* invalid argument or unsupported size */
  FIP_ERR_CUDA = 2,        /* CUDA runtime error */
  FIP_ERR_CUFFT = 3,       /* cuFFT error */
  FIP_ERR_NOMEM = 4,       /* device or pinned allocation failed */
  FIP_ERR_BUDGET = 5,      /* request exceeds the configured HBM budget */
  FIP_ERR_NOT_READY = 6,   /* no result available yet */
  FIP_ERR_STATE = 7        /* call out of order / object in an error state */
} fip_status;

/* Numerical form of an imager. */
typedef enum {
  /* Reference-faithful FP32: the reference's arithmetic (fast-math FP32
   * pixel mapping, FP32 sums), B200 data movement. */
  FIP_FORM_PLAIN = 0,
  /* Precision form: exact closed-form reprojection, compensated FP32 grid
   * sums (FP32 storage; one int32 fixed-point limb with FP16/BF16 storage,
   * whose rounding dominates) and tLISI sums, FP64 tLISI combine;
   * visibility storage per vis_storage. */
  FIP_FORM_PRECISE = 1
} fip_form;

/* Device storage of a snapshot's visibilities in the precision form: FP32,
 * or FP16/BF16 with one power-of-two scale per 1,024 visibilities (the
 * block's max-abs lands in [2^14, 2^15)), converted in one pass per call;
 * the gridder multiplies each value by its block's scale. */
typedef enum { FIP_STORE_F32 = 0, FIP_STORE_F16 = 1, FIP_STORE_BF16 = 2 } fip_vis_storage;

const char* fip_last_error(void);
const char* fip_status_string(int status);
/* Library version "major.minor.patch". */
const char* fip_version(void);

/*
 * Status-returning variant of FIpipe with the same arguments (const inputs).
 * Replaces FIPkernels.cu:554-862 for callers that check errors.
 */
int fip_pipe(const float* vis_re, const float* vis_im, const float* B, const float* V,
             float* result, size_t num_baselines, size_t image_size, size_t num_snapshots,
             float cell_size, size_t unit_size);

/* ------------------------------------------------------------------------ */
/* Imager: persistent device state for one image size (no per-call allocs). */
/* ------------------------------------------------------------------------ */
typedef struct fip_imager fip_imager;

typedef struct {
  size_t image_size;     /* N: image side; multiple of 4 */
  size_t max_baselines;  /* capacity: visibilities per snapshot */
  size_t unit_size;      /* T: trigger tile side (0 = no trigger) */
  float cell_size;       /* radians per pixel */
  int form;              /* fip_form */
  int vis_storage;       /* fip_vis_storage (precision form only) */
  int device;            /* CUDA device ordinal */
  int reproject;         /* 0 = tile gather (default), 1 = source scatter */
} fip_imager_config;

int fip_imager_create(fip_imager** out, const fip_imager_config* cfg);
int fip_imager_destroy(fip_imager* im);
/* Bytes of device memory the imager holds. */
size_t fip_imager_device_bytes(const fip_imager* im);

/*
 * Images one snapshot (device inputs): vis_re/vis_im [nb] FP32, B [nb*2],
 * V [9] -> image [N*N] (device, row-major) and, if image_max is not NULL,
 * max(0, max(image)) as a device float.  Stages: per-snapshot uv binning,
 * binned gridding, in-place C2R FFT, fused correction + reprojection.
 * Replaces the per-snapshot body of FIPkernels.cu:665-711.
 */
int fip_image_snapshot(fip_imager* im, const float* vis_re, const float* vis_im, const float* B,
                       const float* V, size_t nb, float* image, float* image_max, void* stream);

/*
 * Raw two-polarisation samples of one snapshot (device arrays of nb values,
 * in the preprocessing's sample order, sample = row + channel * rows, the
 * order fip_plane_project writes B in): polarisations 0 and 3 (XX, YY),
 * their flags (nonzero = flagged) and weights.
 */
typedef struct {
  const float* v0_re;
  const float* v0_im;
  const float* v3_re;
  const float* v3_im;
  const uint8_t* flag0;
  const uint8_t* flag3;
  const float* weight0;
  const float* weight3;
} fip_raw_vis;

/*
 * fip_image_snapshot from raw polarisations: the flag/weight Stokes-I
 * collapse (collapse_visibility_kernel, SVDPreprocessKernels.cu:208-237;
 * SVD_MFS.py:77-95) runs inside the gridder's visibility load, so no
 * collapsed copy is written or read.  Same image as fip_collapse_visibilities
 * followed by fip_image_snapshot.
 */
int fip_image_snapshot_raw(fip_imager* im, const fip_raw_vis* raw, const float* B,
                           const float* V, size_t nb, float* image, float* image_max,
                           void* stream);

/*
 * The gridding stage alone (device): the visibilities of one snapshot,
 * weighted by 1/|V00 V11 - V01 V10| and spread with the ES kernel, as the
 * Hermitian half of the uv grid the reference builds (gridding +
 * combineToComplex, FIPkernels.cu:188-254): grid [G][G/2+1] complex
 * (interleaved float pairs, row-major, G = ceil(1.5 N)), holding
 * h(r1, r2) = (g(r1, r2) + conj g(-r1, -r2)) / 2 at row r1 mod G, column
 * r2 >= 0, where g is the reference's grid without its (-1)^(r1+r2)
 * checkerboard.  This is the input layout of a C2R transform.
 */
int fip_grid_snapshot(fip_imager* im, const float* vis_re, const float* vis_im, const float* B,
                      const float* V, size_t nb, float* grid, void* stream);

/*
 * fip_grid_snapshot without any allocation, for callers that cannot
 * allocate device memory (fixed memory pools or arenas, plugins whose host
 * application owns every device allocation, real-time loops that must not
 * call the allocator).  No counterpart in the reference.  Same inputs and
 * output grid as fip_grid_snapshot (FP32 visibilities, plain FP32 sums); the
 * binning scratch is a fixed ~6.5 MB device array inside the library, held
 * on every GPU that loads it until the process exits.  Limits: nb <= 131072
 * and image_size <= 4096 (multiple of 4); larger requests return
 * FIP_ERR_ARG.  Every call made outside stream capture looks up the array's
 * device address (cudaGetSymbolAddress, with the device current), so a
 * device reset between calls is followed; a call on a capturing stream uses
 * the address of the last call outside capture, so make the first call on a
 * device before any stream capture (FIP_ERR_STATE otherwise).  All calls
 * share the array: calls whose work overlaps on the GPU race, so serialise
 * them (one stream, or events).
 */
int fip_grid_snapshot_noalloc(const float* vis_re, const float* vis_im, const float* B,
                              const float* V, size_t nb, size_t image_size, float cell_size,
                              float* grid, void* stream);

/*
 * tLISI of three consecutive images (device): maxima max3 [3] as produced by
 * fip_image_snapshot, result [U*U].  The inputs are not modified (the
 * reference clamps I2 in place, FIPkernels.cu:836; the clamp here is local).
 * Replaces FIPkernels.cu:806-851.
 */
int fip_trigger(fip_imager* im, const float* I1, const float* I2, const float* I3,
                const float* max3, float* result, void* stream);

/*
 * How sliding-window triggers (fip_trigger_window, batches) read their tiles
 * (no counterpart in the reference): enable = 1 (the default) streams every
 * tile's slices through registers in the plain form, each image read once
 * for the (up to three) triples it is in; 0 reads each triple's three images.
 * Both give bit-identical tLISI.  Windows of fewer than three triples, unit
 * sizes above 32 and the precision form (whose compensated sums are
 * issue-bound) always read per triple.  Process-wide; returns the previous
 * setting.
 */
int fip_set_trigger_streaming(int enable);

/*
 * Sliding-window tLISI over `count` consecutive device images (no
 * counterpart in the reference, which triggers on one triple per call):
 * images [count][N*N] contiguous, maxima [count] as produced by
 * fip_image_snapshot; triple k (images k, k+1, k+2) -> results + k*U*U for
 * k < count - 2.  The imager's form and unit size; in the plain form each
 * image is read once (fip_set_trigger_streaming).  count >= 3.
 */
int fip_trigger_window(fip_imager* im, const float* images, const float* maxima, size_t count,
                       float* results, void* stream);

/*
 * FIpipe on device buffers with the imager's persistent state: snapshots
 * 0..2 of the concatenated device inputs -> result [U*U] (device).  The
 * three images and their maxima stay in the imager (fip_imager_image).
 */
int fip_pipe_device(fip_imager* im, const float* vis_re, const float* vis_im, const float* B,
                    const float* V, size_t nb, float* result, void* stream);
/* Device pointer to image k (0..2) of the last fip_pipe_device call. */
const float* fip_imager_image(const fip_imager* im, int k);

/*
 * Reprojection domain check (no counterpart in the reference, whose scatter
 * has no domain limit).  The tile gather reprojection is exact while the
 * plane-to-sky map is invertible tile by tile: well inside the horizon and
 * without folds, which every field up to tens of degrees satisfies unless
 * its plane is strongly tilted.  Each gather tile checks this for itself and
 * flags a tile outside it.  fip_imager_check waits (on `stream`, after the
 * imager's earlier calls) and returns FIP_ERR_STATE if any gather since the
 * last check flagged a tile -- those images are not reliable; image such
 * snapshots with reproject = 1 -- then clears the flag.  fip_pipe_host (and
 * so FIpipe), whose bases V are host arrays, checks each snapshot's geometry
 * before imaging and reprojects an out-of-domain snapshot with the scatter.
 */
int fip_imager_check(fip_imager* im, void* stream);

/*
 * FIpipe through an imager with host buffers (pinned staging owned by the
 * imager, copies overlapped with compute): the public e2e call.
 */
int fip_pipe_host(fip_imager* im, const float* vis_re, const float* vis_im, const float* B,
                  const float* V, size_t nb, size_t num_snapshots, float* result);

/*
 * Stage timing (the reference's cudaEvent "Time elapsed" prints,
 * FIPkernels.cu:570-581, 766-770, 825-846, as data): when enabled, every
 * stage launch is bracketed by CUDA events on its stream and the device time
 * is accumulated per stage (fip_stage_name(k), k < fip_stage_count()).
 * Enabling resets the totals.  Collection synchronises the recorded events.
 */
int fip_imager_set_profiling(fip_imager* im, int enable);
int fip_imager_stage_times(fip_imager* im, double* total_ms, long* launches, int nstages);
const char* fip_stage_name(int stage);
int fip_stage_count(void);
/* Number of kernels this imager has launched (library-owned kernels only). */
unsigned long long fip_imager_kernel_launches(const fip_imager* im);
/* Occupied uv band of the last gridded snapshot: max |r1| (grid rows) and
 * max half-plane column, in grid cells (synchronous). */
int fip_imager_band(fip_imager* im, unsigned* max_row, unsigned* max_col);
/* Grid side G = ceil(1.5 N) (FIPkernels.cu:583). */
int fip_imager_grid_side(const fip_imager* im);

/* Autotuner (no counterpart in the reference).  Images the given snapshot
 * once (device buffers, as fip_image_snapshot), then times the launch shapes
 * that do not change the arithmetic beyond rounding -- the transform's complex
 * values per thread (8 or 16), one CTA per transform or one per sub-transform
 * (fft_split), the first pass reading a staged band, global memory, or (row
 * pass) a band copy brought in by bulk tensor copies one row pair ahead
 * (fft_direct 0, 1, 2), and the persistent gridder's CTAs per SM -- on
 * that snapshot's band and bins, and keeps the fastest for later calls.
 * Synchronous; overwrites the imager's trigger ring, so call it before a run
 * of snapshots, not inside one.  fip_imager_tuning reports the choice. */
int fip_imager_autotune(fip_imager* im, const float* vis_re, const float* vis_im,
                        const float* B, const float* V, size_t nb, void* stream);
int fip_imager_tuning(const fip_imager* im, int* fft_values_per_thread, int* fft_split,
                      int* fft_direct, int* grid_ctas_per_sm);
/* Pins the launch shapes instead (values per thread 8 or 16, or 0 for the
 * default; split 0 or 1; direct first pass 0, 1 or 2 (joint form only);
 * gridder CTAs per SM, 0 for the most that fit). */
int fip_imager_set_tuning(fip_imager* im, int fft_values_per_thread, int fft_split,
                          int fft_direct, int grid_ctas_per_sm);

/* ---- Batching form (no counterpart in the reference) ----------------------
 * Many snapshots of one image size per call: one persistent gridding launch
 * and one batched band-pruned transform for the whole batch, the
 * per-snapshot stages (binning, pixel mapping, reprojection) on parallel
 * branches, and the sliding-window trigger batched over the sequence, all
 * captured as one CUDA graph per call and re-launched with updated arguments.
 * Snapshot k of a call: device buffers vis_re[k], vis_im[k] ([nb[k]]),
 * B[k] ([nb[k]][2]), V[k] ([9]); nb may differ between snapshots (flagged
 * visibilities dropped).  The batch keeps the sequence's last two images, so
 * every snapshot with two predecessors (in this call or the previous ones)
 * yields a tLISI matrix (U*U floats, in order, at results); *nresults gets
 * their number.  Asynchronous on `stream`.  Power-of-two images use the
 * band-pruned transform; other sizes one batched cuFFT C2R plan per call
 * size (made before the call's capture, kept for later calls).
 * cfg->reproject must be 0. */
typedef struct fip_batch fip_batch;
int fip_batch_create(fip_batch** out, const fip_imager_config* cfg, size_t max_snapshots);
int fip_batch_destroy(fip_batch* b);
size_t fip_batch_device_bytes(const fip_batch* b);
unsigned long long fip_batch_kernel_launches(const fip_batch* b);
/* Starts a new sequence (forgets the carried images). */
int fip_batch_reset(fip_batch* b);
int fip_batch_image(fip_batch* b, const float* const* vis_re, const float* const* vis_im,
                    const float* const* B, const float* const* V, const size_t* nb, size_t count,
                    float* results, size_t* nresults, void* stream);
/*
 * One batched call whose snapshots may belong to different sequences (the
 * serving form's merged launches): snapshot k's image and maximum go to
 * slots[k].image ([N*N]) and slots[k].image_max ([1]) instead of the batch's
 * ring, and when slots[k].prev_image[0] is not null its tLISI against the two
 * given predecessors (oldest first, with their maxima; they may be images of
 * earlier slots of the same call) is written to slots[k].tlisi ([U*U]).  The
 * batch's own sequence is left untouched.  Asynchronous on `stream`.
 */
typedef struct {
  float* image;
  float* image_max;
  const float* prev_image[2];
  const float* prev_max[2];
  float* tlisi;
} fip_batch_slot;
int fip_batch_image_slots(fip_batch* b, const float* const* vis_re, const float* const* vis_im,
                          const float* const* B, const float* const* V, const size_t* nb,
                          size_t count, const fip_batch_slot* slots, void* stream);
/* Autotuner of the batch's launch shapes (transform values per thread,
 * gridder CTAs per SM) on a representative call; synchronous; resets the
 * sequence. */
int fip_batch_autotune(fip_batch* b, const float* const* vis_re, const float* const* vis_im,
                       const float* const* B, const float* const* V, const size_t* nb,
                       size_t count, void* stream);
int fip_batch_tuning(const fip_batch* b, int* fft_values_per_thread, int* fft_split,
                     int* fft_direct, int* grid_ctas_per_sm);

/* ---- Batches of several sequences (mixed image sizes) -------------------
 * A batch of nseq (1..8) sequences, sequence c with configuration cfgs[c]
 * (its own image size, cell, unit size and max_baselines; form, storage and
 * device shared): each call images up to 64 snapshots, at most max_snapshots
 * of any one sequence, with one persistent gridding launch for all of them
 * and one batched transform per sequence, in one CUDA graph.  Snapshot k
 * belongs to sequence sequence[k] (its snapshots in call order); each
 * sequence keeps its own last two images, and its tLISI matrices (U_c * U_c
 * floats each, in order) go to results[c], their number to nresults[c].
 * fip_batch_image on such a batch images everything into sequence 0;
 * fip_batch_create is the one-sequence case.  Asynchronous on `stream`. */
int fip_batch_create_sequences(fip_batch** out, const fip_imager_config* cfgs, size_t nseq,
                               size_t max_snapshots);
int fip_batch_image_sequences(fip_batch* b, const int* sequence, const float* const* vis_re,
                              const float* const* vis_im, const float* const* B,
                              const float* const* V, const size_t* nb, size_t count,
                              float* const* results, size_t* nresults, void* stream);
/* Autotuner over a representative mixed call: each sequence's transform
 * shape on its own snapshots, the gridder's CTAs per SM on the whole launch;
 * synchronous; resets every sequence. */
int fip_batch_autotune_sequences(fip_batch* b, const int* sequence, const float* const* vis_re,
                                 const float* const* vis_im, const float* const* B,
                                 const float* const* V, const size_t* nb, size_t count,
                                 void* stream);
/* The launch shapes of sequence `sequence` (fip_batch_tuning: sequence 0). */
int fip_batch_sequence_tuning(const fip_batch* b, int sequence, int* fft_values_per_thread,
                              int* fft_split, int* fft_direct, int* grid_ctas_per_sm);
/* Phase timing of batched calls (no counterpart in the reference): when
 * enabled, each call's graph carries timing events at its phase boundaries
 * and the device time of every phase is summed: 0 per-snapshot preparation
 * (storage conversion, binning; the plain form's pixel mappings run beside
 * phases 0-3 and a wait for them counts in phase 4), 1 the persistent gridding
 * launch, 2 the batched column transform, 3 the batched row transform, 4 the
 * reprojections, 5 the triggers.  Enabling resets the totals; reading them
 * waits for the last profiled call. */
int fip_batch_set_profiling(fip_batch* b, int enable);
int fip_batch_phase_times(fip_batch* b, double* total_ms, int nphases, long* calls);
/* The batch's reprojection domain check, as fip_imager_check: waits for the
 * work enqueued on `stream`, returns FIP_ERR_STATE if a gather tile lay
 * outside the gather's domain since the last check, and clears the flag. */
int fip_batch_check(fip_batch* b, void* stream);

/* Per-pixel targets (LL, MM) of the reprojection, [N*N][2] (device), for
 * tests: exact = 0 the plain form's FP32 chain as the imager evaluates it
 * (its theta-terms table where the field allows), 1 the exact closed form,
 * 2 the FP32 chain evaluated step by step (no table; the same bits as 0). */
int fip_pixel_targets(fip_imager* im, const float* V, float* out, int exact, void* stream);

/* ------------------------------------------------------------------------ */
/* Trigger post-processing                                                   */
/* ------------------------------------------------------------------------ */

/* One transient location. */
typedef struct {
  int32_t tile_row, tile_col; /* tile of the tLISI minimum (row-major matrix) */
  float tlisi;                /* its tLISI */
  float row, col;             /* refined position in image pixels (0-based) */
  float x, y;                 /* SIN projection-plane offsets of that position
                                 from the phase centre, radians, in the
                                 reference's convention (its p2p x0, y0 for a
                                 destination pixel, FIPkernels.cu:317-322):
                                 x = -cell (col - N/2 - 1),
                                 y = cell (row - N/2 - 1) */
} fip_location;

/*
 * Transient locations from a tLISI matrix (device, U*U floats row-major, U =
 * image_size / unit_size), the step the reference's output name
 * locations.fits promises (README.md:41) but its code leaves to the user: a
 * tile qualifies when its tLISI is below `threshold` and is the strict
 * minimum of its 3 x 3 neighbourhood (ties to the lower tile index; NaN tiles
 * never qualify).  Its position is refined to the centroid of the
 * neighbourhood's drops max(0, 1 - tLISI).  Up to max_out locations are
 * written to `out` (host), deepest first; *found gets the number found.  No
 * counterpart in the reference.  Synchronous on `stream`; uses stream-ordered
 * scratch (cudaMallocAsync) of 28 bytes per tile.
 */
int fip_locate_transients(const float* tlisi, size_t image_size, size_t unit_size,
                          float cell_size, float threshold, fip_location* out, size_t max_out,
                          size_t* found, void* stream);

/* ------------------------------------------------------------------------ */
/* Plane projection and visibility preparation                               */
/* ------------------------------------------------------------------------ */

/*
 * Plane fit of one snapshot on the device: uvw [rows*3] metres, freqs
 * [chans] Hz -> B [rows*chans*2] (sample s = row + chan*rows), V [9].
 * FP64 mean/covariance/3x3 eigensolve, FP32 outputs.  Replaces
 * preprocess_measurement_set_gpu's projection (SVDPreprocessKernels.cu:
 * 304-425, SVDPreprocessGpu.h:46-49).  Synchronous on `stream`'s work only.
 */
int fip_plane_project(const float* uvw, const float* freqs, size_t rows, size_t chans, float* B,
                      float* V, void* stream);

/*
 * Flag/weight Stokes-I collapse (device): weighted mean of polarisations 0
 * and 3, 0 when both weights vanish.  Replaces collapse_visibility_kernel
 * (SVDPreprocessKernels.cu:208-237).
 */
int fip_collapse_visibilities(const float* v0r, const float* v0i, const float* v3r,
                              const float* v3i, const uint8_t* f0, const uint8_t* f3,
                              const float* w0, const float* w3, float* out_re, float* out_im,
                              size_t ns, void* stream);

/* ------------------------------------------------------------------------ */
/* Batched stream of snapshots of one beam (precision/batching form).        */
/* ------------------------------------------------------------------------ */

/*
 * Images S consecutive snapshots of one beam in one call and returns the
 * S-2 sliding-window tLISI matrices (triples k, k+1, k+2).  vis_re/vis_im
 * [S*nb_stride], B [S*nb_stride*2], V [S*9], nb [S] (host array: per-snapshot
 * visibility counts <= nb_stride) -> results [(S-2)*U*U] (device).
 */
int fip_image_sequence(fip_imager* im, const float* vis_re, const float* vis_im, const float* B,
                       const float* V, const size_t* nb, size_t nb_stride, size_t num_snapshots,
                       float* results, void* stream);

/* ------------------------------------------------------------------------ */
/* Multi-beam streaming server (serving form).                              */
/* ------------------------------------------------------------------------ */
/*
 * Continuous batching of snapshot requests from several beams.  Beams of one
 * imager configuration form a group sharing a batch engine: a worker takes up
 * to the group's step size of its queued snapshots (any of its beams, each in
 * order) and images them in one merged launch (fip_batch_image_slots), while
 * requests that arrive meanwhile queue for the next step and other groups'
 * steps overlap on the device.  Each beam keeps its last two images on the
 * device, so every snapshot from the third on yields the tLISI of the triple
 * ending with it (the reference's trigger, FIPkernels.cu:806-851, applied as
 * a sliding window).  HBM admission: a beam is admitted when its resident
 * images fit in `hbm_budget_bytes` (FIP_ERR_BUDGET otherwise); a group's step
 * size -- the snapshots it may hold on the device at once -- is the largest
 * that fits in what the budget leaves, and a request enters the device only
 * when its group's next step takes it.  Submit copies the host inputs and
 * returns FIP_ERR_NOT_READY while the host queue (max_queue requests) is
 * full.  Beams whose size is not a power of two, or that reproject by
 * scatter, are served one snapshot at a time by an imager of their own.  No
 * counterpart in the reference, which images one FIpipe call at a time.
 */
typedef struct fip_server fip_server;
int fip_server_create(fip_server** out, int device, size_t hbm_budget_bytes, int slots,
                      size_t max_queue);
int fip_server_destroy(fip_server* sv);
/* cfg->device is ignored (the server's device is used). */
int fip_server_add_beam(fip_server* sv, const fip_imager_config* cfg, int* beam_id);
size_t fip_server_reserved_bytes(fip_server* sv);
/* Batched step size limit (snapshots per merged launch, 1..64, default 8);
 * set before adding beams.  A group's actual step is the largest up to the
 * limit that fits in the budget. */
int fip_server_set_max_step(fip_server* sv, int snapshots);
/* Merged launches run so far and the snapshots they imaged. */
int fip_server_stats(fip_server* sv, long* steps, long* snapshots);
int fip_server_submit(fip_server* sv, int beam, const float* vis_re, const float* vis_im,
                      const float* B, const float* V, size_t nb, long* request_id);
/*
 * Waits for a request (timeout_ms < 0: no limit) and returns its beam, its
 * snapshot index within the beam, whether a tLISI matrix was produced (from
 * the third snapshot on; copied to tlisi, tlisi_len floats) and the latency
 * from submit to completion.
 */
int fip_server_wait(fip_server* sv, long request_id, double timeout_ms, int* beam, long* seq,
                    int* has_tlisi, float* tlisi, size_t tlisi_len, double* latency_ms);

#ifdef __cplusplus
}
#endif
#endif /* FIP_B200_H */
