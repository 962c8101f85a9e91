// Host orchestration and C ABI of libfip_b200.so.
//
// One fip_imager owns every device buffer of one image size (grid, bins,
// images, staging), one cuFFT C2R plan and its streams, so repeated calls
// allocate nothing.  The reference's FIpipe re-allocates ~19 buffers, creates
// a cuFFT plan and three streams per call and returns 0 whatever happens
// (FIPkernels.cu:583-861); FIpipe here keeps a small cache of imagers and
// returns a status.
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/fip.h"
#include "fip_common.cuh"
#include "fip_kernels.h"
#include <cmath>

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define FIP_CUDA(call)                                                                     \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return fail(e_ == cudaErrorMemoryAllocation ? FIP_ERR_NOMEM : FIP_ERR_CUDA,          \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                     \
  } while (0)

#define FIP_CUFFT(call)                                                                    \
  do {                                                                                     \
    cufftResult r_ = (call);                                                               \
    if (r_ != CUFFT_SUCCESS)                                                               \
      return fail(r_ == CUFFT_ALLOC_FAILED ? FIP_ERR_NOMEM : FIP_ERR_CUFFT,                \
                  std::string(#call) + ": cufftResult " + std::to_string((int)r_));        \
  } while (0)

#define FIP_TRY(call)                  \
  do {                                 \
    int st_ = (call);                  \
    if (st_ != FIP_OK) return st_;     \
  } while (0)

// Sets the device for the lifetime of a call and restores the caller's.
struct DeviceGuard {
  int prev = -1;
  bool ok = true;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) ok = cudaSetDevice(dev) == cudaSuccess;
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

template <typename T>
cudaError_t dalloc(T** p, size_t count, size_t& total) {
  total += count * sizeof(T);
  return cudaMalloc((void**)p, std::max<size_t>(count, 1) * sizeof(T));
}

// Device-side stage timing (optional): an event pair per stage launch,
// folded into per-stage totals when a call finishes.
enum Stage {
  ST_BIN, ST_GRID, ST_FFT_COLS, ST_FFT_ROWS, ST_TARGETS, ST_REPROJECT, ST_TRIGGER, ST_COUNT
};
const char* kStageNames[ST_COUNT] = {"bin",     "grid",      "fft_cols", "fft_rows",
                                     "targets", "reproject", "trigger"};
constexpr int kMaxPending = 64;

struct StageTimer {
  bool on = false;
  cudaEvent_t ev[kMaxPending][2] = {};
  int stage[kMaxPending] = {};
  int pending = 0;
  double total_ms[ST_COUNT] = {};
  long count[ST_COUNT] = {};
};

}  // namespace

int fip_set_error(int code, const std::string& msg) { return fail(code, msg); }

namespace {
// Host copies into the pinned staging of the host-buffer path.  One thread
// copies a few GB/s from pageable memory, so a 2 MB snapshot would keep the
// first snapshot's upload (which the GPU waits for) on the critical path; a
// small pool of persistent workers shares each copy job.  A job is a list of
// segments cut into chunks that the workers and the caller claim from one
// atomic word (job epoch << 32 | next chunk, claimed by compare-and-swap, so a
// worker still finishing an earlier job never takes a chunk of the next).
// Between jobs the workers poll for a while (a call issues one job per
// snapshot, and calls often follow one another) before they block.
class CopyPool {
 public:
  struct Seg {
    void* dst;
    const void* src;
    size_t bytes;
  };
  static CopyPool& get() {
    static CopyPool pool;
    return pool;
  }
  void copy(const Seg* segs, int nseg) {
    size_t total = 0;
    for (int k = 0; k < nseg; ++k) total += segs[k].bytes;
    if (workers_.empty() || total < 2 * kChunk) {
      for (int k = 0; k < nseg; ++k) std::memcpy(segs[k].dst, segs[k].src, segs[k].bytes);
      return;
    }
    std::lock_guard<std::mutex> call(call_mu_);  // one job at a time
    uint32_t n = 0;
    for (int k = 0; k < nseg; ++k)
      for (size_t off = 0; off < segs[k].bytes; off += kChunk) {
        if (n == kMaxChunks) {  // too many chunks for one job: the rest inline
          std::memcpy(static_cast<char*>(segs[k].dst) + off,
                      static_cast<const char*>(segs[k].src) + off, segs[k].bytes - off);
          break;
        }
        chunks_[n++] = Chunk{static_cast<char*>(segs[k].dst) + off,
                             static_cast<const char*>(segs[k].src) + off,
                             std::min(kChunk, segs[k].bytes - off)};
      }
    count_.store(n, std::memory_order_relaxed);
    remaining_.store(n, std::memory_order_relaxed);
    const uint64_t epoch = (word_.load(std::memory_order_relaxed) >> 32) + 1;
    {
      std::lock_guard<std::mutex> lk(mu_);
      word_.store(epoch << 32, std::memory_order_release);  // publishes chunks_, count_
    }
    cv_.notify_all();
    work(epoch);
    while (remaining_.load(std::memory_order_acquire) != 0) std::this_thread::yield();
  }

 private:
  struct Chunk {
    char* dst;
    const char* src;
    size_t bytes;
  };
  static constexpr size_t kWorkers = 3;
  static constexpr size_t kChunk = 256 * 1024;
  static constexpr uint32_t kMaxChunks = 256;
  // Poll window between jobs: longer than one call, so back-to-back calls
  // find the workers awake.  Each worker spins (yielding) for this long after
  // every job, about 3 x 2 ms of CPU per call at the default; the
  // FIP_COPY_POLL_US environment variable sets it (0: block at once).
  static int poll_us() {
    static const int us = [] {
      const char* e = std::getenv("FIP_COPY_POLL_US");
      if (!e || !*e) return 2000;
      const long v = std::strtol(e, nullptr, 10);
      return (int)std::max(0L, std::min(v, 1000000L));
    }();
    return us;
  }

  CopyPool() {
    for (size_t k = 0; k < kWorkers; ++k) {
      try {
        workers_.emplace_back([this] { run(); });
      } catch (...) {
        break;  // fewer workers (or none: plain copies)
      }
    }
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_.store(true);
    }
    cv_.notify_all();
    for (std::thread& t : workers_) t.join();
  }
  // Claims and copies chunks of job `epoch` until none is left.
  void work(uint64_t epoch) {
    uint64_t w = word_.load(std::memory_order_acquire);
    for (;;) {
      if ((w >> 32) != epoch || (uint32_t)w >= count_.load(std::memory_order_relaxed)) return;
      if (!word_.compare_exchange_weak(w, w + 1, std::memory_order_acq_rel)) continue;
      const Chunk& c = chunks_[(uint32_t)w];
      std::memcpy(c.dst, c.src, c.bytes);
      remaining_.fetch_sub(1, std::memory_order_release);
      w = word_.load(std::memory_order_acquire);
    }
  }
  void run() {
    uint64_t seen = 0;
    for (;;) {
      const auto t0 = std::chrono::steady_clock::now();
      uint64_t e;
      while ((e = word_.load(std::memory_order_acquire) >> 32) == seen && !stop_.load()) {
        if (std::chrono::steady_clock::now() - t0 > std::chrono::microseconds(poll_us())) {
          std::unique_lock<std::mutex> lk(mu_);
          cv_.wait(lk, [&] { return stop_.load() || (word_.load() >> 32) != seen; });
        } else {
          std::this_thread::yield();
        }
      }
      if (stop_.load()) return;
      seen = e;
      work(e);
    }
  }

  std::vector<std::thread> workers_;
  std::mutex call_mu_, mu_;
  std::condition_variable cv_;
  Chunk chunks_[kMaxChunks];
  std::atomic<uint32_t> count_{0};
  std::atomic<uint64_t> word_{0};
  std::atomic<uint32_t> remaining_{0};
  std::atomic<bool> stop_{false};
};
}  // namespace

// Twiddle tables of the band-pruned transform of length g = 3 M: w^k,
// w = e^{+2 pi i / g}, for k < g, then the passes' half table W^m = w^{3 m},
// W = e^{+2 pi i / M}, for m < M / 2 (fipfft).
static std::vector<float2> fft_twiddles(int g) {
  std::vector<float2> tw((size_t)g + fipfft::half_table_elems(g));
  for (int k = 0; k < g; ++k) {
    const double a = 2.0 * FIP_M_PI * (double)k / (double)g;
    tw[k] = make_float2((float)cos(a), (float)sin(a));
  }
  for (int m = 0; m < fipfft::half_table_elems(g); ++m) tw[(size_t)g + m] = tw[(size_t)3 * m];
  return tw;
}

// Scratch of one snapshot in flight.  With the band-pruned transform an
// imager has kLanes of them, so the snapshots of one call (or of a sequence)
// image concurrently, each on its lane's stream.
struct Lane {
  float2* grid = nullptr;            // uv grid (band layout, or C2R in place)
  FipBins bins{};
  float2* colbuf = nullptr;          // column-pass output [G/2+1][N]
  float* pre = nullptr;              // corrected pre-reprojection image [N*N]
  float2* targets = nullptr;         // reference pixel mapping [N*N]
  void* q_re = nullptr;              // reduced-precision visibility storage
  void* q_im = nullptr;
  float* q_scale = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_done = nullptr;
  cudaEvent_t ev_targets = nullptr;  // pixel mapping of the lane's snapshot written
  cufftHandle plan = 0;              // cuFFT C2R fallback: the lane's own plan and work area
  bool plan_ok = false;
};
constexpr int kLanes = 3;

struct fip_imager {
  fip_imager_config cfg{};
  FipGeom geo{};
  size_t device_bytes = 0;
  cudaStream_t stream = nullptr;     // compute stream of the host-buffer path
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_copied[3] = {nullptr, nullptr, nullptr};  // host path: snapshot k's B
  cudaEvent_t ev_vis[3] = {nullptr, nullptr, nullptr};     // host path: its visibilities
  cudaEvent_t ev_used[3] = {nullptr, nullptr, nullptr};
  // Pixel-mapping stream (overlaps gridding + FFT), at the lowest priority:
  // the lanes' latency-bound stages take SM slots first and the
  // issue-bound mapping fills what they leave.
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  bool custom_fft = false;           // band-pruned FFT (fip_fft.cuh)
  fipfft::Plan fft{};
  int grid_ctas_per_sm = 0;          // persistent gridder CTAs per SM (0 = most that fit)
  float2* twiddles = nullptr;        // e^{+2 pi i k / G}, k < G
  float2* theta_tab = nullptr;       // theta terms of the pixel mapping (plain form)
  float* taper = nullptr;            // N/2 + 1 taper values, N/2 + 1 reciprocals
  Lane lane[kLanes];
  int lanes = 1;                     // lanes in use (kLanes with the pruned transform)
  int last_lane = 0;                 // lane of the last gridded snapshot
  cudaEvent_t ev_start = nullptr;    // start of a multi-snapshot call (lanes wait on it)
  cudaEvent_t ev_free[6] = {};       // sequence ring slot released by its last trigger
  float* images[6] = {};             // 0..2: one call's snapshots; all: the sequence ring
  int ring = 3;                      // images allocated (6 with lanes)
  float* maxima = nullptr;           // [6] device floats (written as max bits)
  float* result = nullptr;           // U*U
  float* stats = nullptr;
  // Set by a gather launch whose tile lay outside the gather's domain
  // (fip_gather_domain_ok), read and cleared by fip_imager_check and the
  // host-buffer path; h_err is its pinned copy.
  unsigned* gather_err = nullptr;
  unsigned* h_err = nullptr;
  // Trigger fused into a three-snapshot call's reprojections (concurrent
  // lanes, tile gather): a count per 64 x 64 region and the statistics of
  // every trigger tile.
  unsigned* fuse_count = nullptr;
  double* fuse_stats = nullptr;
  // Device and pinned staging of the host-buffer path, 3 snapshot slots.
  // Per snapshot k, one block of 4 nb floats at k * 4 nb: B [2 nb], vis
  // real [nb], vis imaginary [nb], so each snapshot crosses PCIe in one copy.
  float* d_snap = nullptr;
  float* d_V = nullptr;
  float* h_snap = nullptr;
  float* h_V = nullptr;
  float* h_result = nullptr;
  StageTimer timer;
  unsigned long long launches = 0;   // kernels launched by this imager
  // Calls may come on different streams; each call's stream first waits for
  // the previous call's work (the imager's buffers are shared).
  cudaEvent_t ev_done = nullptr;
  bool done_recorded = false;
};

namespace {
// Orders a call on stream s after every earlier call of the imager.
int call_enter(fip_imager* im, cudaStream_t s) {
  if (im->done_recorded) FIP_CUDA(cudaStreamWaitEvent(s, im->ev_done, 0));
  return FIP_OK;
}
int call_leave(fip_imager* im, cudaStream_t s) {
  FIP_CUDA(cudaEventRecord(im->ev_done, s));
  im->done_recorded = true;
  return FIP_OK;
}

// Opens a timed stage on stream s (no-op unless profiling is on).
int stage_begin(fip_imager* im, int st, cudaStream_t s) {
  StageTimer& t = im->timer;
  if (!t.on || t.pending >= kMaxPending) return -1;
  const int k = t.pending++;
  t.stage[k] = st;
  cudaEventRecord(t.ev[k][0], s);
  return k;
}
void stage_end(fip_imager* im, int k, cudaStream_t s) {
  if (k >= 0) cudaEventRecord(im->timer.ev[k][1], s);
}
// Folds finished stage timings into the totals (synchronises their events).
void stage_collect(fip_imager* im) {
  StageTimer& t = im->timer;
  for (int k = 0; k < t.pending; ++k) {
    float ms = 0.f;
    cudaEventSynchronize(t.ev[k][1]);
    if (cudaEventElapsedTime(&ms, t.ev[k][0], t.ev[k][1]) == cudaSuccess) {
      t.total_ms[t.stage[k]] += ms;
      t.count[t.stage[k]] += 1;
    }
  }
  t.pending = 0;
}
}  // namespace

static void imager_free(fip_imager* im) {
  if (!im) return;
  DeviceGuard g(im->cfg.device);
  if (im->stream) cudaStreamSynchronize(im->stream);
  if (im->copy_stream) cudaStreamSynchronize(im->copy_stream);
  if (im->side) cudaStreamSynchronize(im->side);
  for (Lane& L : im->lane) {
    if (L.stream) cudaStreamSynchronize(L.stream);
    if (L.plan_ok) cufftDestroy(L.plan);
    void* lp[] = {L.grid, L.bins.count, L.bins.offset, L.bins.cursor, L.bins.entries,
                  L.bins.work, L.bins.nwork, L.bins.bbox, L.bins.multi, L.bins.nmulti,
                  L.colbuf, L.pre, L.targets, L.q_re, L.q_im, L.q_scale};
    for (void* p : lp)
      if (p) cudaFree(p);
    if (L.ev_done) cudaEventDestroy(L.ev_done);
    if (L.ev_targets) cudaEventDestroy(L.ev_targets);
    if (L.stream) cudaStreamDestroy(L.stream);
  }
  for (float* p : im->images)
    if (p) cudaFree(p);
  void* dptrs[] = {im->taper, im->twiddles, im->theta_tab, im->maxima, im->result, im->stats,
                   im->d_snap, im->d_V, im->gather_err, im->fuse_count, im->fuse_stats};
  for (void* p : dptrs)
    if (p) cudaFree(p);
  void* hptrs[] = {im->h_snap, im->h_V, im->h_result, im->h_err};
  for (void* p : hptrs)
    if (p) cudaFreeHost(p);
  for (int k = 0; k < 3; ++k) {
    if (im->ev_copied[k]) cudaEventDestroy(im->ev_copied[k]);
    if (im->ev_vis[k]) cudaEventDestroy(im->ev_vis[k]);
    if (im->ev_used[k]) cudaEventDestroy(im->ev_used[k]);
  }
  for (int k = 0; k < kMaxPending; ++k)
    for (int e = 0; e < 2; ++e)
      if (im->timer.ev[k][e]) cudaEventDestroy(im->timer.ev[k][e]);
  if (im->ev_done) cudaEventDestroy(im->ev_done);
  if (im->ev_fork) cudaEventDestroy(im->ev_fork);
  if (im->ev_join) cudaEventDestroy(im->ev_join);
  if (im->ev_start) cudaEventDestroy(im->ev_start);
  for (cudaEvent_t e : im->ev_free)
    if (e) cudaEventDestroy(e);
  if (im->stream) cudaStreamDestroy(im->stream);
  if (im->copy_stream) cudaStreamDestroy(im->copy_stream);
  if (im->side) cudaStreamDestroy(im->side);
  delete im;
}

// The gridder's sums: the precision form's two-limb compensated sums for
// FP32 (or raw) visibilities; one int32 limb (2^-30 of a work item's summed
// weights, 2^19 below the rounding of the stored values) for FP16/BF16
// storage, whose own rounding the compensation could not recover.
static int grid_compensated(bool precise, int vt) {
  return precise && vt != FIP_VIS_F16 && vt != FIP_VIS_BF16 ? 1 : 0;
}
static int grid_compensated(const fip_imager_config& c) {
  return c.form == FIP_FORM_PRECISE && c.vis_storage == FIP_STORE_F32 ? 1 : 0;
}

static int validate_sizes(size_t n, size_t t, float cell) {
  if (n < 16 || n % 4 != 0)
    return fail(FIP_ERR_ARG, "image_size must be a multiple of 4 and >= 16 (the reference's "
                             "grid crop is misaligned when ceil(1.5 N) is odd; the half-plane "
                             "grid needs G > 18)");
  if (n > 32768) return fail(FIP_ERR_ARG, "image_size above 32768 is not supported");
  if (t > n) return fail(FIP_ERR_ARG, "unit_size larger than image_size");
  if (!(cell > 0.f) || !(cell < 1.f)) return fail(FIP_ERR_ARG, "cell_size must be in (0, 1) rad");
  return FIP_OK;
}

extern "C" {

const char* fip_last_error(void) { return g_last_error.c_str(); }

const char* fip_version(void) { return "0.1.0"; }

const char* fip_status_string(int s) {
  switch (s) {
    case FIP_OK: return "ok";
    case FIP_ERR_ARG: return "invalid argument";
    case FIP_ERR_CUDA: return "CUDA error";
    case FIP_ERR_CUFFT: return "cuFFT error";
    case FIP_ERR_NOMEM: return "out of memory";
    case FIP_ERR_BUDGET: return "over the HBM budget";
    case FIP_ERR_NOT_READY: return "not ready";
    case FIP_ERR_STATE: return "invalid state";
    default: return "unknown status";
  }
}

int fip_imager_create(fip_imager** out, const fip_imager_config* cfg) {
  if (!out || !cfg) return fail(FIP_ERR_ARG, "null argument");
  *out = nullptr;
  FIP_TRY(validate_sizes(cfg->image_size, cfg->unit_size, cfg->cell_size));
  if (cfg->max_baselines == 0 || cfg->max_baselines > (1u << 28))
    return fail(FIP_ERR_ARG, "max_baselines must be in [1, 2^28]");
  if (cfg->form != FIP_FORM_PLAIN && cfg->form != FIP_FORM_PRECISE)
    return fail(FIP_ERR_ARG, "unknown form");
  if (cfg->vis_storage < 0 || cfg->vis_storage > 2) return fail(FIP_ERR_ARG, "unknown storage");
  int ndev = 0;
  FIP_CUDA(cudaGetDeviceCount(&ndev));
  if (cfg->device < 0 || cfg->device >= ndev) return fail(FIP_ERR_ARG, "no such device");
  DeviceGuard guard(cfg->device);
  if (!guard.ok) return fail(FIP_ERR_CUDA, "cudaSetDevice failed");

  fip_imager* im = new fip_imager();
  im->cfg = *cfg;
  FipGeom& geo = im->geo;
  geo.n = (int)cfg->image_size;
  geo.g = (int)ceilf(1.5f * (float)cfg->image_size);  // computeCeil(1.5 N) (FIPkernels.cu:583)
  geo.hp = geo.g / 2 + 1;
  geo.t = (int)cfg->unit_size;
  geo.u = geo.t > 0 ? geo.n / geo.t : 0;
  geo.tiles_r = (geo.g + FIP_GTILE - 1) / FIP_GTILE;
  geo.tiles_c = (geo.hp + FIP_GTILE - 1) / FIP_GTILE;
  geo.cell = cfg->cell_size;
  im->custom_fft = fip_fft_plan(geo.g, im->fft);
  geo.layout = im->custom_fft ? 1 : 0;
  const size_t n2 = (size_t)geo.n * geo.n;
  const size_t nb = cfg->max_baselines;
  const size_t ntiles = (size_t)geo.tiles_r * geo.tiles_c;
  size_t& tot = im->device_bytes;

  auto cleanup = [&](int code) {
    std::string msg = g_last_error;
    imager_free(im);
    g_last_error = msg;
    return code;
  };
#define FIP_ALLOC(call)                                                                      \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return cleanup(fail(e_ == cudaErrorMemoryAllocation ? FIP_ERR_NOMEM : FIP_ERR_CUDA,    \
                          std::string(#call) + ": " + cudaGetErrorString(e_)));              \
  } while (0)

  FIP_ALLOC(cudaStreamCreateWithFlags(&im->stream, cudaStreamNonBlocking));
  FIP_ALLOC(cudaStreamCreateWithFlags(&im->copy_stream, cudaStreamNonBlocking));
  int prio_least = 0, prio_greatest = 0;
  FIP_ALLOC(cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest));
  FIP_ALLOC(cudaStreamCreateWithPriority(&im->side, cudaStreamNonBlocking, prio_least));
  FIP_ALLOC(cudaEventCreateWithFlags(&im->ev_fork, cudaEventDisableTiming));
  FIP_ALLOC(cudaEventCreateWithFlags(&im->ev_join, cudaEventDisableTiming));
  FIP_ALLOC(cudaEventCreateWithFlags(&im->ev_start, cudaEventDisableTiming));
  for (cudaEvent_t& e : im->ev_free) FIP_ALLOC(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  FIP_ALLOC(cudaEventCreateWithFlags(&im->ev_done, cudaEventDisableTiming));
  for (int k = 0; k < kMaxPending; ++k)
    for (int e = 0; e < 2; ++e) FIP_ALLOC(cudaEventCreate(&im->timer.ev[k][e]));
  for (int k = 0; k < 3; ++k) {
    FIP_ALLOC(cudaEventCreateWithFlags(&im->ev_copied[k], cudaEventDisableTiming));
    FIP_ALLOC(cudaEventCreateWithFlags(&im->ev_vis[k], cudaEventDisableTiming));
    FIP_ALLOC(cudaEventCreateWithFlags(&im->ev_used[k], cudaEventDisableTiming));
  }
  if (cfg->reproject != 0 && cfg->reproject != 1) return cleanup(fail(FIP_ERR_ARG, "unknown reproject mode"));
  if (cfg->reproject == 0 && !fip_gather_supported(geo, cfg->form == FIP_FORM_PRECISE))
    return cleanup(fail(FIP_ERR_ARG, "cell_size too small for the tile-gather reprojection; "
                                     "use reproject = 1"));
  FIP_ALLOC(dalloc(&im->taper, 2 * ((size_t)geo.n / 2 + 1), tot));
  if (cfg->form == FIP_FORM_PLAIN) {
    FIP_ALLOC(dalloc(&im->theta_tab, fip_theta_table_elems(), tot));
    FIP_ALLOC(fip_launch_theta_table(im->theta_tab, im->stream));
  }
  // Three lanes; with the cuFFT fallback each lane has its own plan and work
  // area (a plan's work area serves one stream at a time).
  im->lanes = kLanes;
  for (int l = 0; l < im->lanes; ++l) {
    Lane& L = im->lane[l];
    FIP_ALLOC(cudaStreamCreateWithPriority(&L.stream, cudaStreamNonBlocking, prio_greatest));
    FIP_ALLOC(cudaEventCreateWithFlags(&L.ev_done, cudaEventDisableTiming));
    FIP_ALLOC(cudaEventCreateWithFlags(&L.ev_targets, cudaEventDisableTiming));
    FIP_ALLOC(dalloc(&L.grid, (size_t)geo.g * geo.hp, tot));
    L.bins.cap = 12 * nb;
    L.bins.wcap = ntiles + L.bins.cap / FIP_GCHUNK + 1;
    FIP_ALLOC(dalloc(&L.bins.count, ntiles, tot));
    FIP_ALLOC(dalloc(&L.bins.offset, ntiles + 1, tot));
    FIP_ALLOC(dalloc(&L.bins.cursor, ntiles, tot));
    FIP_ALLOC(dalloc(&L.bins.entries, L.bins.cap, tot));
    FIP_ALLOC(dalloc(&L.bins.work, L.bins.wcap, tot));
    FIP_ALLOC(dalloc(&L.bins.nwork, 1, tot));
    FIP_ALLOC(dalloc(&L.bins.bbox, 4, tot));
    FIP_ALLOC(dalloc(&L.bins.multi, ntiles, tot));
    FIP_ALLOC(dalloc(&L.bins.nmulti, 1, tot));
    FIP_ALLOC(dalloc(&L.pre, n2, tot));
    if (cfg->form == FIP_FORM_PLAIN && cfg->reproject == 0) FIP_ALLOC(dalloc(&L.targets, n2, tot));
    if (im->custom_fft) FIP_ALLOC(dalloc(&L.colbuf, (size_t)geo.hp * geo.n, tot));
    if (cfg->form == FIP_FORM_PRECISE && cfg->vis_storage != FIP_STORE_F32) {
      FIP_ALLOC(dalloc((uint16_t**)&L.q_re, nb, tot));
      FIP_ALLOC(dalloc((uint16_t**)&L.q_im, nb, tot));
      FIP_ALLOC(dalloc(&L.q_scale, fip_qblocks(nb), tot));
    }
  }
  if (im->custom_fft) {
    const std::vector<float2> tw = fft_twiddles(geo.g);
    FIP_ALLOC(dalloc(&im->twiddles, tw.size(), tot));
    FIP_ALLOC(cudaMemcpy(im->twiddles, tw.data(), tw.size() * sizeof(float2),
                         cudaMemcpyHostToDevice));
  }
  // With concurrent lanes a sequence keeps six images, so a lane can start a
  // snapshot while the triggers of the previous ones still read theirs.
  im->ring = im->lanes > 1 ? 6 : 3;
  for (int k = 0; k < im->ring; ++k) FIP_ALLOC(dalloc(&im->images[k], n2, tot));
  FIP_ALLOC(dalloc(&im->maxima, 6, tot));
  FIP_ALLOC(dalloc(&im->result, std::max<size_t>((size_t)geo.u * geo.u, 1), tot));
  FIP_ALLOC(dalloc(&im->d_snap, 3 * 4 * nb, tot));
  FIP_ALLOC(dalloc(&im->d_V, 27, tot));
  FIP_ALLOC(cudaMallocHost((void**)&im->h_snap, 3 * 4 * nb * sizeof(float)));
  FIP_ALLOC(cudaMallocHost((void**)&im->h_V, 27 * sizeof(float)));
  FIP_ALLOC(cudaMallocHost((void**)&im->h_result,
                           std::max<size_t>((size_t)geo.u * geo.u, 1) * sizeof(float)));
  FIP_ALLOC(dalloc(&im->gather_err, 1, tot));
  FIP_ALLOC(cudaMemset(im->gather_err, 0, sizeof(unsigned)));
  // Plain form only: the precision form's compensated statistics cost the
  // last reprojection more than the separate pass (measured 3 % slower).
  if (im->lanes > 1 && cfg->reproject == 0 && cfg->form == FIP_FORM_PLAIN &&
      fip_trigger_fusable(geo)) {
    FIP_ALLOC(dalloc(&im->fuse_count, fip_trigger_fuse_counts(geo), tot));
    FIP_ALLOC(dalloc(&im->fuse_stats, 3 * (size_t)geo.u * geo.u, tot));
  }
  FIP_ALLOC(cudaMallocHost((void**)&im->h_err, sizeof(unsigned)));
  *im->h_err = 0;

  for (int l = 0; l < im->lanes && !im->custom_fft; ++l) {
    Lane& L = im->lane[l];
    cufftResult r = cufftCreate(&L.plan);
    if (r != CUFFT_SUCCESS) return cleanup(fail(FIP_ERR_CUFFT, "cufftCreate failed"));
    L.plan_ok = true;
    size_t work = 0;
    r = cufftMakePlan2d(L.plan, geo.g, geo.g, CUFFT_C2R, &work);
    if (r != CUFFT_SUCCESS)
      return cleanup(fail(r == CUFFT_ALLOC_FAILED ? FIP_ERR_NOMEM : FIP_ERR_CUFFT,
                          "cufftMakePlan2d(C2R) failed: " + std::to_string((int)r)));
    tot += work;
  }
  cudaError_t e = fip_launch_taper(im->taper, geo, im->stream);
  if (e != cudaSuccess) return cleanup(fail(FIP_ERR_CUDA, cudaGetErrorString(e)));
  e = cudaStreamSynchronize(im->stream);
  if (e != cudaSuccess) return cleanup(fail(FIP_ERR_CUDA, cudaGetErrorString(e)));
#undef FIP_ALLOC
  *out = im;
  return FIP_OK;
}

int fip_imager_destroy(fip_imager* im) {
  imager_free(im);
  return FIP_OK;
}

size_t fip_imager_device_bytes(const fip_imager* im) { return im ? im->device_bytes : 0; }

// Images one snapshot with lane L's scratch on stream s.  fork_targets: run
// the pixel mapping on the side stream beside gridding + FFT (single-snapshot
// calls; calls that image several snapshots run them on concurrent lanes
// instead).
static int image_snapshot_impl(fip_imager* im, Lane& L, const float* vr, const float* vi,
                               const float* B, const float* V, size_t nb, float* image,
                               float* image_max, cudaStream_t s, bool fork_targets,
                               bool targets_ready = false, cudaEvent_t targets_ev = nullptr,
                               bool force_scatter = false, const FipRawVis* raw = nullptr,
                               const FipFuse* fuse = nullptr,
                               const std::function<int(cudaEvent_t*)>* before_grid = nullptr) {
  const FipGeom& geo = im->geo;
  if (nb > im->cfg.max_baselines) return fail(FIP_ERR_ARG, "nb exceeds the imager's capacity");
  if (nb == 0) return fail(FIP_ERR_ARG, "nb must be positive");
  if ((!raw && (!vr || !vi)) || !B || !V || !image)
    return fail(FIP_ERR_ARG, "null device pointer");
  const bool precise = im->cfg.form == FIP_FORM_PRECISE;
  const void* gvr = vr;
  const void* gvi = vi;
  // raw: two-polarisation samples, collapsed to Stokes I inside the gridder's
  // load (or inside the reduced-storage conversion).
  int vt = raw ? FIP_VIS_RAW : FIP_VIS_F32;
  int k;
  // force_scatter: the snapshot's geometry lies outside the gather's domain
  // (checked on the host where V is a host array): the reference's scheme.
  const bool gather = im->cfg.reproject == 0 && !force_scatter;
  const bool chain_targets = gather && !precise;
  // The pixel mapping depends on V only: it may run beside gridding + FFT on
  // the side stream (serialised on s when profiling, so every stage's time
  // is its own).
  const bool fork = chain_targets && fork_targets && !im->timer.on;
  if (chain_targets && !targets_ready) {
    cudaStream_t ts = fork ? im->side : s;
    if (fork) {
      FIP_CUDA(cudaEventRecord(im->ev_fork, s));
      FIP_CUDA(cudaStreamWaitEvent(im->side, im->ev_fork, 0));
    }
    k = stage_begin(im, ST_TARGETS, ts);
    FIP_CUDA(fip_launch_targets(geo, V, im->theta_tab, L.targets, ts));
    stage_end(im, k, ts);
    im->launches += 1;
    if (fork) FIP_CUDA(cudaEventRecord(im->ev_join, im->side));
  }
  k = stage_begin(im, ST_BIN, s);
  FIP_CUDA(fip_launch_bin(geo, B, (int)nb, L.bins, s));
  stage_end(im, k, s);
  // The host path stages the visibilities while the binning runs: the
  // gridding (and the reduced-storage conversion) wait for them.
  if (before_grid && *before_grid) {
    cudaEvent_t ready = nullptr;
    FIP_TRY((*before_grid)(&ready));
    if (ready) FIP_CUDA(cudaStreamWaitEvent(s, ready, 0));
  }
  if (precise && im->cfg.vis_storage != FIP_STORE_F32) {
    vt = im->cfg.vis_storage == FIP_STORE_F16 ? FIP_VIS_F16 : FIP_VIS_BF16;
    k = stage_begin(im, ST_GRID, s);
    if (raw)
      FIP_CUDA(fip_launch_quantize_raw(*raw, nb, vt, L.q_re, L.q_im, L.q_scale, s));
    else
      FIP_CUDA(fip_launch_quantize(vr, vi, nb, vt, L.q_re, L.q_im, L.q_scale, s));
    stage_end(im, k, s);
    im->launches += 1;
    gvr = L.q_re;
    gvi = L.q_im;
  }
  k = stage_begin(im, ST_GRID, s);
  FIP_CUDA(fip_launch_grid(geo, B, gvr, gvi, vt, L.q_scale, V, (int)nb, L.bins, L.grid,
                           grid_compensated(precise, vt), s, im->grid_ctas_per_sm, raw));
  stage_end(im, k, s);
  im->launches += fip_bin_launches(geo) + 2;  // binning, zero tiles, grid
  if (im->custom_fft) {
    k = stage_begin(im, ST_FFT_COLS, s);
    FIP_CUDA(fip_launch_fft_cols(geo, L.grid, L.bins.bbox, L.colbuf, im->twiddles, im->fft, s));
    stage_end(im, k, s);
    k = stage_begin(im, ST_FFT_ROWS, s);
    FIP_CUDA(fip_launch_fft_rows(geo, L.colbuf, L.bins.bbox, im->taper, im->twiddles, im->fft,
                                 L.pre, s));
    im->launches += 2;
  } else {
    k = stage_begin(im, ST_FFT_ROWS, s);
    FIP_CUFFT(cufftSetStream(L.plan, s));
    FIP_CUFFT(cufftExecC2R(L.plan, reinterpret_cast<cufftComplex*>(L.grid),
                           reinterpret_cast<cufftReal*>(L.grid)));
    FIP_CUDA(fip_launch_correct_c2r(geo, reinterpret_cast<const float*>(L.grid), im->taper,
                                    L.pre, L.bins.bbox + 3, s));
    im->launches += 1;
  }
  stage_end(im, k, s);
  if (image_max) FIP_CUDA(cudaMemsetAsync(image_max, 0, sizeof(float), s));
  if (!gather) {
    k = stage_begin(im, ST_REPROJECT, s);
    FIP_CUDA(fip_launch_reproject_scatter(geo, L.pre, V, (int)nb, image, s));
    if (image_max)
      FIP_CUDA(fip_launch_image_max(image, (size_t)geo.n * geo.n,
                                    reinterpret_cast<unsigned*>(image_max), s));
    stage_end(im, k, s);
    im->launches += image_max ? 2 : 1;
  } else {
    if (fork) FIP_CUDA(cudaStreamWaitEvent(s, im->ev_join, 0));
    if (targets_ready && targets_ev) FIP_CUDA(cudaStreamWaitEvent(s, targets_ev, 0));
    k = stage_begin(im, ST_REPROJECT, s);
    FIP_CUDA(fip_launch_reproject_gather(geo, L.pre, L.targets, V, (int)nb, L.bins.bbox + 3,
                                         image, reinterpret_cast<unsigned*>(image_max),
                                         precise ? 1 : 0, s, im->gather_err, fuse));
    stage_end(im, k, s);
    im->launches += 1;
  }
  return FIP_OK;
}

// Images snapshot k of a multi-snapshot call on lane k % lanes: the lane's
// stream waits for `after`, images, and records the lane's ev_done, which
// the caller's stream waits for (wait_lane).  When profiling, or with one
// lane, everything runs on s in order.
static int image_on_lane(fip_imager* im, int k, const float* vr, const float* vi,
                         const float* B, const float* V, size_t nb, float* image,
                         float* image_max, cudaStream_t s, cudaEvent_t after,
                         bool targets_ready = false, bool force_scatter = false,
                         const FipFuse* fuse = nullptr,
                         const std::function<int(cudaEvent_t*)>* before_grid = nullptr) {
  if (im->lanes == 1 || im->timer.on) {
    FIP_CUDA(cudaStreamWaitEvent(s, after, 0));
    return image_snapshot_impl(im, im->lane[k % im->lanes], vr, vi, B, V, nb, image, image_max,
                               s, true, false, nullptr, force_scatter, nullptr, fuse,
                               before_grid);
  }
  Lane& L = im->lane[k % im->lanes];
  FIP_CUDA(cudaStreamWaitEvent(L.stream, after, 0));
  FIP_TRY(image_snapshot_impl(im, L, vr, vi, B, V, nb, image, image_max, L.stream, false,
                              targets_ready, targets_ready ? L.ev_targets : nullptr,
                              force_scatter, nullptr, fuse, before_grid));
  FIP_CUDA(cudaEventRecord(L.ev_done, L.stream));
  return FIP_OK;
}

// Whether a three-snapshot call fuses its trigger into the reprojections:
// the plain form on concurrent lanes (not serialised for profiling, whose
// stage times keep the trigger apart), the tile gather, a tile side dividing
// the gather's 64.
static bool fuse_ok(const fip_imager* im) {
  return im->fuse_count && !im->timer.on && im->lanes > 1;
}

static FipFuse fuse_of(const fip_imager* im) {
  FipFuse f{};
  for (int k = 0; k < 3; ++k) f.img[k] = im->images[k];
  f.count = im->fuse_count;
  f.stats = im->fuse_stats;
  return f;
}

// Whether a three-snapshot call maps its pixels ahead on the side stream:
// concurrent lanes, the gather reprojection of the plain form (the precision
// form evaluates the exact map inside the gather).
static bool targets_ahead(const fip_imager* im) {
  return im->lanes > 1 && !im->timer.on && im->cfg.reproject == 0 &&
         im->cfg.form == FIP_FORM_PLAIN;
}

// The pixel mappings of a call's three snapshots (bases V + 9 k), on the
// low-priority side stream after `after`; lane k's gather waits on its
// ev_targets.
static int launch_targets_ahead(fip_imager* im, const float* V, cudaEvent_t after) {
  FIP_CUDA(cudaStreamWaitEvent(im->side, after, 0));
  for (int k = 0; k < 3; ++k) {
    Lane& L = im->lane[k % im->lanes];
    FIP_CUDA(fip_launch_targets(im->geo, V + (size_t)k * 9, im->theta_tab, L.targets, im->side));
    FIP_CUDA(cudaEventRecord(L.ev_targets, im->side));
    im->launches += 1;
  }
  return FIP_OK;
}

static int wait_lane(fip_imager* im, int k, cudaStream_t s) {
  if (im->lanes == 1 || im->timer.on) return FIP_OK;
  FIP_CUDA(cudaStreamWaitEvent(s, im->lane[k % im->lanes].ev_done, 0));
  return FIP_OK;
}

int fip_image_snapshot(fip_imager* im, const float* vis_re, const float* vis_im, const float* B,
                       const float* V, size_t nb, float* image, float* image_max, void* stream) {
  if (!im) return fail(FIP_ERR_ARG, "null imager");
  DeviceGuard g(im->cfg.device);
  cudaStream_t s = (cudaStream_t)stream;
  FIP_TRY(call_enter(im, s));
  FIP_TRY(image_snapshot_impl(im, im->lane[0], vis_re, vis_im, B, V, nb, image, image_max, s,
                              true));
  im->last_lane = 0;
  return call_leave(im, s);
}

int fip_image_snapshot_raw(fip_imager* im, const fip_raw_vis* raw, const float* B,
                           const float* V, size_t nb, float* image, float* image_max,
                           void* stream) {
  if (!im) return fail(FIP_ERR_ARG, "null imager");
  if (!raw || !raw->v0_re || !raw->v0_im || !raw->v3_re || !raw->v3_im || !raw->flag0 ||
      !raw->flag3 || !raw->weight0 || !raw->weight3)
    return fail(FIP_ERR_ARG, "null raw visibility array");
  const FipRawVis rv{raw->v0_re, raw->v0_im, raw->v3_re, raw->v3_im,
                     raw->flag0, raw->flag3, raw->weight0, raw->weight3};
  DeviceGuard g(im->cfg.device);
  cudaStream_t s = (cudaStream_t)stream;
  FIP_TRY(call_enter(im, s));
  FIP_TRY(image_snapshot_impl(im, im->lane[0], nullptr, nullptr, B, V, nb, image, image_max, s,
                              true, false, nullptr, false, &rv));
  im->last_lane = 0;
  return call_leave(im, s);
}

int fip_grid_snapshot(fip_imager* im, const float* vis_re, const float* vis_im, const float* B,
                      const float* V, size_t nb, float* grid, void* stream) {
  if (!im) return fail(FIP_ERR_ARG, "null imager");
  if (!vis_re || !vis_im || !B || !V || !grid) return fail(FIP_ERR_ARG, "null device pointer");
  if (nb == 0 || nb > im->cfg.max_baselines)
    return fail(FIP_ERR_ARG, "nb must be in [1, the imager's max_baselines]");
  DeviceGuard g(im->cfg.device);
  cudaStream_t s = (cudaStream_t)stream;
  FIP_TRY(call_enter(im, s));
  // Full half plane, row-major: every tile is written (zero where empty).
  FipGeom geo = im->geo;
  geo.layout = 0;
  const bool precise = im->cfg.form == FIP_FORM_PRECISE;
  const void* gvr = vis_re;
  const void* gvi = vis_im;
  int vt = FIP_VIS_F32;
  Lane& L = im->lane[0];
  if (precise && im->cfg.vis_storage != FIP_STORE_F32) {
    vt = im->cfg.vis_storage == FIP_STORE_F16 ? FIP_VIS_F16 : FIP_VIS_BF16;
    FIP_CUDA(fip_launch_quantize(vis_re, vis_im, nb, vt, L.q_re, L.q_im, L.q_scale, s));
    im->launches += 1;
    gvr = L.q_re;
    gvi = L.q_im;
  }
  FIP_CUDA(fip_launch_bin(geo, B, (int)nb, L.bins, s));
  FIP_CUDA(fip_launch_grid(geo, B, gvr, gvi, vt, L.q_scale, V, (int)nb, L.bins,
                           reinterpret_cast<float2*>(grid), grid_compensated(precise, vt), s,
                           im->grid_ctas_per_sm));
  im->last_lane = 0;
  im->launches += fip_bin_launches(geo) + 2;
  return call_leave(im, s);
}

int fip_trigger(fip_imager* im, const float* I1, const float* I2, const float* I3,
                const float* max3, float* result, void* stream) {
  if (!im) return fail(FIP_ERR_ARG, "null imager");
  if (im->geo.t <= 0) return fail(FIP_ERR_ARG, "imager has no trigger tile (unit_size 0)");
  if (!I1 || !I2 || !I3 || !max3 || !result) return fail(FIP_ERR_ARG, "null device pointer");
  DeviceGuard g(im->cfg.device);
  FIP_TRY(call_enter(im, (cudaStream_t)stream));
  const int k = stage_begin(im, ST_TRIGGER, (cudaStream_t)stream);
  FIP_CUDA(fip_launch_trigger(im->geo, I1, I2, I3, max3, im->stats, result,
                              im->cfg.form == FIP_FORM_PRECISE ? 1 : 0, (cudaStream_t)stream));
  stage_end(im, k, (cudaStream_t)stream);
  im->launches += 1;
  FIP_TRY(call_leave(im, (cudaStream_t)stream));
  if (im->timer.on) stage_collect(im);
  return FIP_OK;
}

int fip_trigger_window(fip_imager* im, const float* images, const float* maxima, size_t count,
                       float* results, void* stream) {
  if (!im) return fail(FIP_ERR_ARG, "null imager");
  if (im->geo.t <= 0) return fail(FIP_ERR_ARG, "imager has no trigger tile (unit_size 0)");
  if (!images || !maxima || !results) return fail(FIP_ERR_ARG, "null device pointer");
  if (count < 3 || count - 2 > 65535) return fail(FIP_ERR_ARG, "count must be in [3, 65537]");
  DeviceGuard g(im->cfg.device);
  FIP_TRY(call_enter(im, (cudaStream_t)stream));
  const int k = stage_begin(im, ST_TRIGGER, (cudaStream_t)stream);
  FIP_CUDA(fip_launch_trigger_batch(im->geo, images, maxima, (int)(count - 2), results,
                                    im->cfg.form == FIP_FORM_PRECISE ? 1 : 0,
                                    (cudaStream_t)stream));
  stage_end(im, k, (cudaStream_t)stream);
  im->launches += 1;
  FIP_TRY(call_leave(im, (cudaStream_t)stream));
  if (im->timer.on) stage_collect(im);
  return FIP_OK;
}

int fip_set_trigger_streaming(int enable) {
  const int prev = fip_trigger_stream_enabled();
  fip_trigger_stream_enable(enable);
  return prev;
}

int fip_pipe_device(fip_imager* im, const float* vr, const float* vi, const float* B,
                    const float* V, size_t nb, float* result, void* stream) {
  if (!im) return fail(FIP_ERR_ARG, "null imager");
  DeviceGuard g(im->cfg.device);
  cudaStream_t s = (cudaStream_t)stream;
  FIP_TRY(call_enter(im, s));
  // The three snapshots image concurrently on the lanes; the trigger joins them
  // (fused into their reprojections when it can be).
  const FipFuse fz = fuse_of(im);
  const bool fused = fuse_ok(im) && result;
  if (fused) FIP_CUDA(cudaMemsetAsync(im->fuse_count, 0,
                                      fip_trigger_fuse_counts(im->geo) * sizeof(unsigned), s));
  FIP_CUDA(cudaEventRecord(im->ev_start, s));
  const bool ahead = targets_ahead(im);
  if (ahead) FIP_TRY(launch_targets_ahead(im, V, im->ev_start));
  for (int k = 0; k < 3; ++k)
    FIP_TRY(image_on_lane(im, k, vr + (size_t)k * nb, vi + (size_t)k * nb,
                          B + (size_t)k * nb * 2, V + (size_t)k * 9, nb, im->images[k],
                          im->maxima + k, s, im->ev_start, ahead, false,
                          fused ? &fz : nullptr));
  for (int k = 0; k < 3; ++k) FIP_TRY(wait_lane(im, k, s));
  im->last_lane = 2 % im->lanes;
  if (fused) {
    FIP_CUDA(fip_launch_trigger_combine(im->geo, im->fuse_stats, im->maxima, result,
                                        im->cfg.form == FIP_FORM_PRECISE ? 1 : 0, s));
    im->launches += 1;
  } else if (im->geo.t > 0 && result) {
    const int k = stage_begin(im, ST_TRIGGER, s);
    FIP_CUDA(fip_launch_trigger(im->geo, im->images[0], im->images[1], im->images[2],
                                im->maxima, im->stats, result,
                                im->cfg.form == FIP_FORM_PRECISE ? 1 : 0, s));
    stage_end(im, k, s);
    im->launches += 1;
  }
  FIP_TRY(call_leave(im, s));
  if (im->timer.on) stage_collect(im);
  return FIP_OK;
}

const float* fip_imager_image(const fip_imager* im, int k) {
  if (!im || k < 0 || k > 2) return nullptr;
  return im->images[k];
}

static const char* gather_domain_message() {
  return "a reprojection tile lay outside the tile gather's domain (the plane-to-sky map "
         "folds or nears the horizon there: a very wide field with a strongly tilted "
         "plane); its image is not reliable; image such snapshots with reproject = 1 "
         "(the reference's scatter)";
}

int fip_imager_check(fip_imager* im, void* stream) {
  if (!im) return fail(FIP_ERR_ARG, "null imager");
  DeviceGuard g(im->cfg.device);
  cudaStream_t s = (cudaStream_t)stream;
  FIP_TRY(call_enter(im, s));
  FIP_CUDA(cudaMemcpyAsync(im->h_err, im->gather_err, sizeof(unsigned), cudaMemcpyDeviceToHost,
                           s));
  FIP_CUDA(cudaMemsetAsync(im->gather_err, 0, sizeof(unsigned), s));
  FIP_TRY(call_leave(im, s));
  FIP_CUDA(cudaStreamSynchronize(s));
  if (*im->h_err) return fail(FIP_ERR_STATE, gather_domain_message());
  return FIP_OK;
}

int fip_pipe_host(fip_imager* im, const float* vr, const float* vi, const float* B,
                  const float* V, size_t nb, size_t nsnap, float* result) {
  if (!im) return fail(FIP_ERR_ARG, "null imager");
  if (!vr || !vi || !B || !V || !result) return fail(FIP_ERR_ARG, "null host pointer");
  if (nsnap < 3)
    return fail(FIP_ERR_ARG, "num_snapshots must be >= 3 (the pipeline images three snapshots)");
  // The pinned staging block and the device upload buffer hold three
  // snapshots of max_baselines each: check before any copy into them.
  if (nb == 0 || nb > im->cfg.max_baselines)
    return fail(FIP_ERR_ARG, "nb must be in [1, the imager's max_baselines]");
  if (im->geo.t <= 0) return fail(FIP_ERR_ARG, "imager has no trigger tile (unit_size 0)");
  DeviceGuard g(im->cfg.device);
  cudaStream_t s = im->stream, cs = im->copy_stream;
  FIP_TRY(call_enter(im, s));
  FIP_TRY(call_enter(im, cs));
  // The three bases V first: the pixel mapping (the longest kernel) needs
  // only V, so with concurrent lanes it starts on every lane while the host
  // still stages the visibilities.
  std::memcpy(im->h_V, V, 27 * sizeof(float));
  FIP_CUDA(cudaMemcpyAsync(im->d_V, im->h_V, 27 * sizeof(float), cudaMemcpyHostToDevice, cs));
  const bool early = targets_ahead(im);
  if (early) {
    FIP_CUDA(cudaEventRecord(im->ev_start, cs));
    FIP_TRY(launch_targets_ahead(im, im->d_V, im->ev_start));
  }
  // Snapshots whose plane-to-sky map leaves the gather's domain (very wide,
  // strongly tilted fields) reproject with the reference's scatter instead.
  // Checked on the host while the GPU already runs the pixel mappings.
  bool scatter[3] = {false, false, false};
  if (im->cfg.reproject == 0)
    for (int k = 0; k < 3; ++k)
      scatter[k] = !fip_gather_domain_ok(V + 9 * k, im->geo.n, im->cfg.cell_size);
  // The trigger fuses into the three reprojections when all three gather;
  // the counts are cleared on the copy stream, ahead of every lane.
  const FipFuse fz = fuse_of(im);
  const bool fused = fuse_ok(im) && !scatter[0] && !scatter[1] && !scatter[2];
  if (fused) FIP_CUDA(cudaMemsetAsync(im->fuse_count, 0,
                                      fip_trigger_fuse_counts(im->geo) * sizeof(unsigned), cs));
  // Per snapshot: host copy of its B into pinned slot k (CPU), async H2D on
  // the copy stream, the snapshot's lane enqueued up to its binning; then
  // the same for its visibilities, which only the gridding waits for.  The
  // lanes thus start binning while the CPU still stages.
  for (int k = 0; k < 3; ++k) {
    float* hs = im->h_snap + (size_t)k * 4 * nb;
    float* ds = im->d_snap + (size_t)k * 4 * nb;
    const CopyPool::Seg seg_b = {hs, B + (size_t)k * nb * 2, nb * 2 * sizeof(float)};
    CopyPool::get().copy(&seg_b, 1);
    FIP_CUDA(cudaMemcpyAsync(ds, hs, 2 * nb * sizeof(float), cudaMemcpyHostToDevice, cs));
    FIP_CUDA(cudaEventRecord(im->ev_copied[k], cs));
    const std::function<int(cudaEvent_t*)> stage_vis = [&, k, hs, ds](cudaEvent_t* ready) -> int {
      const CopyPool::Seg segs[2] = {{hs + 2 * nb, vr + (size_t)k * nb, nb * sizeof(float)},
                                     {hs + 3 * nb, vi + (size_t)k * nb, nb * sizeof(float)}};
      CopyPool::get().copy(segs, 2);
      FIP_CUDA(cudaMemcpyAsync(ds + 2 * nb, hs + 2 * nb, 2 * nb * sizeof(float),
                               cudaMemcpyHostToDevice, cs));
      FIP_CUDA(cudaEventRecord(im->ev_vis[k], cs));
      *ready = im->ev_vis[k];
      return FIP_OK;
    };
    FIP_TRY(image_on_lane(im, k, ds + 2 * nb, ds + 3 * nb, ds, im->d_V + (size_t)k * 9, nb,
                          im->images[k], im->maxima + k, s, im->ev_copied[k], early, scatter[k],
                          fused ? &fz : nullptr, &stage_vis));
  }
  for (int k = 0; k < 3; ++k) FIP_TRY(wait_lane(im, k, s));
  im->last_lane = 2 % im->lanes;
  if (fused) {
    FIP_CUDA(fip_launch_trigger_combine(im->geo, im->fuse_stats, im->maxima, im->result,
                                        im->cfg.form == FIP_FORM_PRECISE ? 1 : 0, s));
    im->launches += 1;
  } else {
    const int k = stage_begin(im, ST_TRIGGER, s);
    FIP_CUDA(fip_launch_trigger(im->geo, im->images[0], im->images[1], im->images[2],
                                im->maxima, im->stats, im->result,
                                im->cfg.form == FIP_FORM_PRECISE ? 1 : 0, s));
    stage_end(im, k, s);
    im->launches += 1;
  }
  const size_t uu = (size_t)im->geo.u * im->geo.u;
  FIP_CUDA(cudaMemcpyAsync(im->h_result, im->result, uu * sizeof(float), cudaMemcpyDeviceToHost,
                           s));
  FIP_CUDA(cudaMemcpyAsync(im->h_err, im->gather_err, sizeof(unsigned), cudaMemcpyDeviceToHost,
                           s));
  FIP_CUDA(cudaMemsetAsync(im->gather_err, 0, sizeof(unsigned), s));
  FIP_TRY(call_leave(im, s));
  FIP_CUDA(cudaStreamSynchronize(s));
  std::memcpy(result, im->h_result, uu * sizeof(float));
  if (*im->h_err) return fail(FIP_ERR_STATE, gather_domain_message());
  if (im->timer.on) stage_collect(im);
  return FIP_OK;
}

int fip_imager_set_profiling(fip_imager* im, int enable) {
  if (!im) return fail(FIP_ERR_ARG, "null imager");
  DeviceGuard g(im->cfg.device);
  stage_collect(im);
  im->timer.on = enable != 0;
  for (int k = 0; k < ST_COUNT; ++k) {
    im->timer.total_ms[k] = 0.0;
    im->timer.count[k] = 0;
  }
  return FIP_OK;
}

int fip_imager_stage_times(fip_imager* im, double* total_ms, long* launches, int nstages) {
  if (!im || !total_ms || !launches) return fail(FIP_ERR_ARG, "null argument");
  DeviceGuard g(im->cfg.device);
  stage_collect(im);
  for (int k = 0; k < nstages && k < ST_COUNT; ++k) {
    total_ms[k] = im->timer.total_ms[k];
    launches[k] = im->timer.count[k];
  }
  return FIP_OK;
}

const char* fip_stage_name(int stage) {
  return (stage >= 0 && stage < ST_COUNT) ? kStageNames[stage] : "";
}

int fip_stage_count(void) { return ST_COUNT; }

unsigned long long fip_imager_kernel_launches(const fip_imager* im) {
  return im ? im->launches : 0ull;
}

int fip_imager_band(fip_imager* im, unsigned* max_row, unsigned* max_col) {
  if (!im || !max_row || !max_col) return fail(FIP_ERR_ARG, "null argument");
  DeviceGuard g(im->cfg.device);
  unsigned b[4] = {0, 0, 0, 0};
  FIP_CUDA(cudaMemcpy(b, im->lane[im->last_lane].bins.bbox, sizeof(b), cudaMemcpyDeviceToHost));
  *max_row = b[0];
  *max_col = b[1];
  return FIP_OK;
}

int fip_imager_grid_side(const fip_imager* im) { return im ? im->geo.g : 0; }

int fip_pixel_targets(fip_imager* im, const float* V, float* out, int exact, void* stream) {
  if (!im || !V || !out) return fail(FIP_ERR_ARG, "null argument");
  DeviceGuard g(im->cfg.device);
  if (exact < 0 || exact > 2) return fail(FIP_ERR_ARG, "exact must be 0, 1 or 2");
  FIP_CUDA(fip_launch_pixel_targets(im->geo, V, out, exact, im->theta_tab, (cudaStream_t)stream));
  im->launches += 1;
  return FIP_OK;
}

namespace {
struct EventPair {
  cudaEvent_t a = nullptr, b = nullptr;
  ~EventPair() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};
}  // namespace

int fip_imager_autotune(fip_imager* im, const float* vr, const float* vi, const float* B,
                        const float* V, size_t nb, void* stream) {
  if (!im) return fail(FIP_ERR_ARG, "null imager");
  DeviceGuard g(im->cfg.device);
  if (!g.ok) return fail(FIP_ERR_CUDA, "cudaSetDevice failed");
  cudaStream_t s = (cudaStream_t)stream;
  FIP_TRY(call_enter(im, s));
  // One full snapshot leaves this snapshot's bins, band and grid in place.
  Lane& L = im->lane[0];
  FIP_TRY(image_snapshot_impl(im, L, vr, vi, B, V, nb, im->images[0], im->maxima, s, true));
  im->last_lane = 0;
  const FipGeom& geo = im->geo;
  const bool precise = im->cfg.form == FIP_FORM_PRECISE;
  const void* gvr = vr;
  const void* gvi = vi;
  int vt = FIP_VIS_F32;
  if (precise && im->cfg.vis_storage != FIP_STORE_F32) {
    vt = im->cfg.vis_storage == FIP_STORE_F16 ? FIP_VIS_F16 : FIP_VIS_BF16;
    gvr = L.q_re;
    gvi = L.q_im;
  }
  EventPair ev;
  FIP_CUDA(cudaEventCreate(&ev.a));
  FIP_CUDA(cudaEventCreate(&ev.b));
  // Best of three timed repetitions after one untimed.
  auto timed = [&](auto&& launch, float& ms) -> int {
    ms = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
      FIP_CUDA(cudaEventRecord(ev.a, s));
      FIP_CUDA(launch());
      FIP_CUDA(cudaEventRecord(ev.b, s));
      FIP_CUDA(cudaEventSynchronize(ev.b));
      float t = 0.f;
      FIP_CUDA(cudaEventElapsedTime(&t, ev.a, ev.b));
      if (rep > 0) ms = std::min(ms, t);
    }
    return FIP_OK;
  };
  if (im->custom_fft) {
    float best = 1e30f;
    fipfft::Plan chosen = im->fft;
    // Values per thread 8 or 16 x {joint, split, joint with a direct first
    // pass, joint with the row pass's band copied by bulk tensor copies}.
    for (int shape = 0; shape < 8; ++shape) {
      fipfft::Plan p{};
      if (!fip_fft_plan(geo.g, p, shape & 1 ? 16 : 8)) continue;
      p.split = (shape >> 1) == 1;
      p.direct = (shape >> 1) == 2 ? 1 : ((shape >> 1) == 3 ? 2 : 0);
      float ms = 0.f;
      FIP_TRY(timed(
          [&]() -> cudaError_t {
            cudaError_t e = fip_launch_fft_cols(geo, L.grid, L.bins.bbox, L.colbuf,
                                                im->twiddles, p, s);
            if (e != cudaSuccess) return e;
            return fip_launch_fft_rows(geo, L.colbuf, L.bins.bbox, im->taper, im->twiddles,
                                       p, L.pre, s);
          },
          ms));
      if (ms < best) {
        best = ms;
        chosen = p;
      }
    }
    im->fft = chosen;
  }
  {
    float best = 1e30f;
    int chosen = 0;
    for (int c = 1; c <= fip_grid_max_ctas_per_sm(grid_compensated(precise, vt)); ++c) {
      float ms = 0.f;
      FIP_TRY(timed(
          [&]() -> cudaError_t {
            return fip_launch_grid(geo, B, gvr, gvi, vt, L.q_scale, V, (int)nb, L.bins,
                                   L.grid, grid_compensated(precise, vt), s, c);
          },
          ms));
      if (ms < best) {
        best = ms;
        chosen = c;
      }
    }
    im->grid_ctas_per_sm = chosen;
  }
  FIP_TRY(call_leave(im, s));
  FIP_CUDA(cudaStreamSynchronize(s));
  return FIP_OK;
}

int fip_imager_set_tuning(fip_imager* im, int fft_values_per_thread, int fft_split,
                          int fft_direct, int grid_ctas_per_sm) {
  if (!im) return fail(FIP_ERR_ARG, "null imager");
  if (grid_ctas_per_sm < 0 || grid_ctas_per_sm > 8)
    return fail(FIP_ERR_ARG, "grid_ctas_per_sm must be in [0, 8]");
  if (im->custom_fft) {
    fipfft::Plan p{};
    if (!fip_fft_plan(im->geo.g, p, fft_values_per_thread))
      return fail(FIP_ERR_ARG, "no transform with these values per thread for this size");
    p.split = fft_split ? 1 : 0;
    p.direct = fft_split ? 0 : std::max(0, std::min(fft_direct, 2));
    im->fft = p;
  }
  im->grid_ctas_per_sm = grid_ctas_per_sm;
  return FIP_OK;
}

int fip_imager_tuning(const fip_imager* im, int* fft_values_per_thread, int* fft_split,
                      int* fft_direct, int* grid_ctas_per_sm) {
  if (!im) return fail(FIP_ERR_ARG, "null imager");
  if (fft_values_per_thread) *fft_values_per_thread = im->custom_fft ? im->fft.e : 0;
  if (fft_split) *fft_split = im->custom_fft ? im->fft.split : 0;
  if (fft_direct) *fft_direct = im->custom_fft ? im->fft.direct : 0;
  if (grid_ctas_per_sm)
    *grid_ctas_per_sm = im->grid_ctas_per_sm > 0
                            ? im->grid_ctas_per_sm
                            : fip_grid_max_ctas_per_sm(grid_compensated(im->cfg));
  return FIP_OK;
}

int fip_image_sequence(fip_imager* im, const float* vr, const float* vi, const float* B,
                       const float* V, const size_t* nb, size_t nb_stride, size_t nsnap,
                       float* results, void* stream) {
  if (!im || !nb) return fail(FIP_ERR_ARG, "null argument");
  if (nsnap < 3) return fail(FIP_ERR_ARG, "num_snapshots must be >= 3");
  if (im->geo.t <= 0) return fail(FIP_ERR_ARG, "imager has no trigger tile (unit_size 0)");
  DeviceGuard g(im->cfg.device);
  cudaStream_t s = (cudaStream_t)stream;
  const size_t uu = (size_t)im->geo.u * im->geo.u;
  FIP_TRY(call_enter(im, s));
  // Snapshot k goes to ring slot k % R on lane k % lanes; trigger k (on s)
  // waits for the lanes of snapshots k-2 .. k.  Slot k % R last held
  // snapshot k - R, whose last reader is trigger k - R + 2: ev_free[slot],
  // recorded on s after that trigger, releases it, so the lanes run up to
  // R - 3 snapshots ahead of the triggers.
  const int R = im->ring;
  FIP_CUDA(cudaEventRecord(im->ev_start, s));
  for (size_t k = 0; k < nsnap; ++k) {
    const int slot = (int)(k % R);
    FIP_TRY(image_on_lane(im, (int)k, vr + k * nb_stride, vi + k * nb_stride,
                          B + k * nb_stride * 2, V + k * 9, nb[k], im->images[slot],
                          im->maxima + slot, s, k < (size_t)R ? im->ev_start : im->ev_free[slot]));
    if (k >= 2) {
      for (int j = 0; j < 3; ++j) FIP_TRY(wait_lane(im, (int)(k - j), s));
      const int a = (int)((k - 2) % R), b = (int)((k - 1) % R), c = slot;
      const int st = stage_begin(im, ST_TRIGGER, s);
      FIP_CUDA(fip_launch_trigger3(im->geo, im->images[a], im->images[b], im->images[c],
                                   im->maxima + a, im->maxima + b, im->maxima + c,
                                   results + (k - 2) * uu,
                                   im->cfg.form == FIP_FORM_PRECISE ? 1 : 0, s));
      stage_end(im, st, s);
      im->launches += 1;
      FIP_CUDA(cudaEventRecord(im->ev_free[a], s));  // last reader of slot a
    }
  }
  im->last_lane = (int)((nsnap - 1) % im->lanes);
  FIP_TRY(call_leave(im, s));
  if (im->timer.on) stage_collect(im);
  return FIP_OK;
}

int fip_plane_project(const float* uvw, const float* freqs, size_t rows, size_t chans, float* B,
                      float* V, void* stream) {
  if (!uvw || !freqs || !B || !V) return fail(FIP_ERR_ARG, "null device pointer");
  if (rows == 0 || chans == 0) return fail(FIP_ERR_ARG, "empty measurement set");
  FIP_CUDA(fip_launch_plane_project(uvw, freqs, rows, chans, nullptr, B, V,
                                    (cudaStream_t)stream));
  return FIP_OK;
}

int fip_collapse_visibilities(const float* v0r, const float* v0i, const float* v3r,
                              const float* v3i, const uint8_t* f0, const uint8_t* f3,
                              const float* w0, const float* w3, float* out_re, float* out_im,
                              size_t ns, void* stream) {
  if (!v0r || !v0i || !v3r || !v3i || !f0 || !f3 || !w0 || !w3 || !out_re || !out_im)
    return fail(FIP_ERR_ARG, "null device pointer");
  FIP_CUDA(fip_launch_collapse(v0r, v0i, v3r, v3i, f0, f3, w0, w3, out_re, out_im, ns,
                               (cudaStream_t)stream));
  return FIP_OK;
}

// ---------------------------------------------------------------------------
// FIpipe-compatible entry points with a small cache of imagers.
// ---------------------------------------------------------------------------

namespace {
// One cached imager.  Its mutex is held for the whole call that uses it, so
// concurrent callers serialise only when they share an imager; the cache's
// own mutex covers the lookup.  An entry evicted while a call still uses it
// is freed when that call drops its reference.
struct CachedImager {
  fip_imager* im = nullptr;
  std::mutex mu;
  ~CachedImager() { imager_free(im); }
};
struct CacheEntry {
  int device;
  size_t n, nb, t;
  float cell;
  std::shared_ptr<CachedImager> box;
  unsigned long long last_use;
};
std::mutex g_cache_mu;
// Never destroyed: imagers still cached at exit are left to the driver's
// teardown rather than freed after the CUDA runtime has unloaded.
std::vector<CacheEntry>& g_cache = *new std::vector<CacheEntry>;
unsigned long long g_tick = 0;
constexpr size_t kCacheMax = 2;
}  // namespace

int fip_pipe(const float* vis_re, const float* vis_im, const float* B, const float* V,
             float* result, size_t num_baselines, size_t image_size, size_t num_snapshots,
             float cell_size, size_t unit_size) {
  if (!vis_re || !vis_im || !B || !V || !result) return fail(FIP_ERR_ARG, "null host pointer");
  if (num_baselines == 0) return fail(FIP_ERR_ARG, "num_baselines must be positive");
  if (unit_size == 0) return fail(FIP_ERR_ARG, "unit_size must be positive");
  FIP_TRY(validate_sizes(image_size, unit_size, cell_size));
  if (num_snapshots < 3)
    return fail(FIP_ERR_ARG, "num_snapshots must be >= 3 (three snapshots are imaged)");
  int dev = 0;
  FIP_CUDA(cudaGetDevice(&dev));
  std::shared_ptr<CachedImager> box;
  {
    std::lock_guard<std::mutex> lock(g_cache_mu);
    // Any imager of this geometry with room for num_baselines serves the call
    // (nb is a per-call argument below its capacity), the smallest first, so
    // a change in the flagged count does not re-create an imager.
    CacheEntry* best = nullptr;
    for (auto& e : g_cache)
      if (e.device == dev && e.n == image_size && e.nb >= num_baselines && e.t == unit_size &&
          e.cell == cell_size && (!best || e.nb < best->nb))
        best = &e;
    if (best) {
      best->last_use = ++g_tick;
      box = best->box;
    } else {
      if (g_cache.size() >= kCacheMax) {
        auto it = std::min_element(g_cache.begin(), g_cache.end(),
                                   [](const CacheEntry& a, const CacheEntry& b) {
                                     return a.last_use < b.last_use;
                                   });
        g_cache.erase(it);
      }
      fip_imager_config cfg{};
      cfg.image_size = image_size;
      cfg.max_baselines = num_baselines;
      cfg.unit_size = unit_size;
      cfg.cell_size = cell_size;
      cfg.form = FIP_FORM_PLAIN;
      cfg.vis_storage = FIP_STORE_F32;
      cfg.device = dev;
      cfg.reproject = 0;
      box = std::make_shared<CachedImager>();
      FIP_TRY(fip_imager_create(&box->im, &cfg));
      g_cache.push_back(CacheEntry{dev, image_size, num_baselines, unit_size, cell_size, box,
                                   ++g_tick});
    }
  }
  std::lock_guard<std::mutex> lock(box->mu);
  return fip_pipe_host(box->im, vis_re, vis_im, B, V, num_baselines, num_snapshots, result);
}

}  // extern "C"


// ---------------------------------------------------------------------------
// Batching form: many snapshots per call, of one or several sequences (each
// with its own image size, cell and tile), imaged with one persistent
// gridding launch for the whole call and one batched transform per image
// size, the per-snapshot stages (binning, pixel mapping, reprojection) on
// parallel branches, each sequence's trigger batched over its sliding window,
// all captured as one CUDA graph per call shape.
// ---------------------------------------------------------------------------
namespace {
constexpr int kBranches = 4;
constexpr int kMaxSequences = 8;
}  // namespace

// One sequence of a batch: its configuration, transform plan and tables, the
// scratch of up to smax snapshots per call (the call's j-th snapshot of the
// sequence at base + j * stride) and its image ring.
struct BatchSeq {
  fip_imager_config cfg{};
  FipGeom geo{};
  bool custom_fft = true;  // band-pruned transform; else batched cuFFT C2R plans
  fipfft::Plan fft{};
  // cuFFT C2R plans by number of snapshots per call (grid sides not 3 * 2^k),
  // created before the call's capture.
  std::vector<std::pair<int, cufftHandle>> plans;
  float2* twiddles = nullptr;
  float* taper = nullptr;
  size_t ntiles = 0, cap = 0, wcap = 0, n2 = 0, grid_elems = 0, col_elems = 0;
  unsigned* count = nullptr;          // [smax][ntiles]
  unsigned* offset = nullptr;         // [smax][ntiles + 1]
  unsigned* cursor = nullptr;         // [smax][ntiles]
  unsigned* entries = nullptr;        // [smax][cap]
  int4* work = nullptr;               // [smax][wcap]
  unsigned* nwork = nullptr;          // [smax]
  unsigned* bbox = nullptr;           // [smax][4]
  unsigned* multi = nullptr;          // [smax][ntiles]
  unsigned* nmulti = nullptr;         // [smax]
  float2* grid = nullptr;             // [smax][G (G/2+1)]
  float2* colbuf = nullptr;           // [smax][(G/2+1) N]
  float* pre = nullptr;               // [smax][N N]
  float2* targets = nullptr;          // [smax][N N] (plain form)
  void* q_re = nullptr;               // [smax][max_baselines] (reduced storage)
  void* q_im = nullptr;
  float* q_scale = nullptr;           // [smax][fip_qblocks(max_baselines)]
  // Linear ring: slots 0, 1 carry the sequence's last two images, the call's
  // snapshots go to slots 2 .. count + 1.
  float* images = nullptr;            // [smax + 2][N N]
  float* maxima = nullptr;            // [smax + 2]
  int carried = 0;

  FipBins bins(int k) const {
    FipBins b{};
    b.count = count + k * ntiles;
    b.offset = offset + k * (ntiles + 1);
    b.cursor = cursor + k * ntiles;
    b.entries = entries + k * cap;
    b.work = work + k * wcap;
    b.nwork = nwork + k;
    b.bbox = bbox + 4 * k;
    b.multi = multi + k * ntiles;
    b.nmulti = nmulti + k;
    b.cap = cap;
    b.wcap = wcap;
    return b;
  }
  cufftHandle plan_for(int count) const {
    for (const auto& p : plans)
      if (p.first == count) return p.second;
    return 0;
  }
  void free_all() {
    for (auto& p : plans) cufftDestroy(p.second);
    plans.clear();
    void* ptrs[] = {twiddles, taper, count, offset, cursor, entries, work, nwork, bbox, multi,
                    nmulti, grid, colbuf, pre, targets, q_re, q_im, q_scale, images, maxima};
    for (void* p : ptrs)
      if (p) cudaFree(p);
  }
};

struct fip_batch {
  fip_imager_config cfg{};  // sequence 0's; form, storage and device are every sequence's
  int smax = 0;             // snapshots of one sequence per call at most
  size_t device_bytes = 0;
  int grid_ctas_per_sm = 0;
  float2* theta_tab = nullptr;  // theta terms of the pixel mapping (plain form)
  std::vector<BatchSeq> seq;
  unsigned* gather_err = nullptr;     // [1] set by a gather tile outside its domain
  cudaStream_t branch[kBranches] = {};
  cudaStream_t capture = nullptr;  // capture and launch stream (highest priority)
  // Pixel-mapping branches at the lowest priority: the mappings need only V,
  // so they run beside the gridding and the transforms and join the call
  // only before its reprojections.
  static constexpr int kMapBranches = 2;
  cudaStream_t map_branch[kMapBranches] = {};
  cudaEvent_t map_join[kMapBranches] = {};
  cudaEvent_t fork = nullptr;
  cudaEvent_t join[kBranches] = {};
  // Phase timing (fip_batch_set_profiling): timing events captured into the
  // call's graph at the phase boundaries, read after the call.
  static constexpr int kPhases = 6;
  bool profiling = false;
  cudaEvent_t phase_ev[kPhases + 1] = {};
  double phase_ms[kPhases] = {};
  long phase_calls = 0;
  bool phase_pending = false;
  cudaGraphExec_t exec = nullptr;
  unsigned long long launches = 0;
};

namespace {
void batch_free(fip_batch* b) {
  if (!b) return;
  DeviceGuard g(b->cfg.device);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  for (BatchSeq& q : b->seq) q.free_all();
  if (b->theta_tab) cudaFree(b->theta_tab);
  if (b->gather_err) cudaFree(b->gather_err);
  for (int k = 0; k < kBranches; ++k) {
    if (b->branch[k]) cudaStreamDestroy(b->branch[k]);
    if (b->join[k]) cudaEventDestroy(b->join[k]);
  }
  for (int k = 0; k < fip_batch::kMapBranches; ++k) {
    if (b->map_branch[k]) cudaStreamDestroy(b->map_branch[k]);
    if (b->map_join[k]) cudaEventDestroy(b->map_join[k]);
  }
  if (b->capture) cudaStreamDestroy(b->capture);
  if (b->fork) cudaEventDestroy(b->fork);
  for (cudaEvent_t e : b->phase_ev)
    if (e) cudaEventDestroy(e);
  delete b;
}

// Folds the last profiled call's phase times into the totals (waits for it).
int batch_collect(fip_batch* b) {
  if (!b->phase_pending) return FIP_OK;
  b->phase_pending = false;
  FIP_CUDA(cudaEventSynchronize(b->phase_ev[fip_batch::kPhases]));
  for (int k = 0; k < fip_batch::kPhases; ++k) {
    float ms = 0.f;
    FIP_CUDA(cudaEventElapsedTime(&ms, b->phase_ev[k], b->phase_ev[k + 1]));
    b->phase_ms[k] += ms;
  }
  b->phase_calls += 1;
  return FIP_OK;
}

int batch_vis_type(const fip_batch* b) {
  const bool reduced = b->cfg.form == FIP_FORM_PRECISE && b->cfg.vis_storage != FIP_STORE_F32;
  return !reduced ? FIP_VIS_F32
                  : (b->cfg.vis_storage == FIP_STORE_F16 ? FIP_VIS_F16 : FIP_VIS_BF16);
}

// The snapshots of a call by sequence: snapshot k is the loc[k]-th of
// sequence sq[k] in this call, which holds per[c] snapshots of sequence c.
struct CallLayout {
  int sq[FIP_MAX_BATCH];
  int loc[FIP_MAX_BATCH];
  int per[kMaxSequences];
};

CallLayout call_layout(const int* seq_of, int count) {
  CallLayout l{};
  for (int k = 0; k < count; ++k) {
    l.sq[k] = seq_of ? seq_of[k] : 0;
    l.loc[k] = l.per[l.sq[k]]++;
  }
  return l;
}

// Snapshot k's entry of the batched gridding launch (its bins in place).
FipGridSnap grid_snap(const fip_batch* b, const CallLayout& l, int k, const float* B,
                      const float* V, const void* vr, const void* vi) {
  const BatchSeq& q = b->seq[l.sq[k]];
  const int j = l.loc[k];
  const bool reduced = batch_vis_type(b) != FIP_VIS_F32;
  FipGridSnap g{};
  g.B = B;
  g.V = V;
  g.vr = reduced ? static_cast<const void*>(static_cast<char*>(q.q_re) +
                                            j * q.cfg.max_baselines * 2)
                 : vr;
  g.vi = reduced ? static_cast<const void*>(static_cast<char*>(q.q_im) +
                                            j * q.cfg.max_baselines * 2)
                 : vi;
  g.vis_scale = reduced ? q.q_scale + j * fip_qblocks(q.cfg.max_baselines) : nullptr;
  const FipBins bins = q.bins(j);
  g.entries = bins.entries;
  g.work = bins.work;
  g.nwork = bins.nwork;
  g.grid = q.grid + j * q.grid_elems;
  g.scale = q.geo.cell * (float)(size_t)q.geo.g;
  g.g = q.geo.g;
  g.hp = q.geo.hp;
  g.tiles_c = q.geo.tiles_c;
  g.layout = q.geo.layout;
  return g;
}

// Captures the work of one call into a graph (stream s in capture mode).
// seq_of (or null: all sequence 0): each snapshot's sequence; first[c] and
// results[c]: sequence c's first snapshot with two predecessors and where
// its tLISI matrices go.  slots (or null): per-snapshot image destinations
// and trigger predecessors (fip_batch_image_slots) instead of the sequences'
// rings.
int batch_record(fip_batch* b, const int* seq_of, const float* const* vr,
                 const float* const* vi, const float* const* B, const float* const* V,
                 const size_t* nb, int count, const int* first, float* const* results,
                 cudaStream_t s, const fip_batch_slot* slots = nullptr) {
  const bool precise = b->cfg.form == FIP_FORM_PRECISE;
  const int vt = batch_vis_type(b);
  const bool reduced = vt != FIP_VIS_F32;
  const int nseq = (int)b->seq.size();
  const CallLayout l = call_layout(seq_of, count);
  unsigned long long launches = 0;
  auto phase = [&](int k) -> cudaError_t {
    // Inside stream capture only an external record becomes a record node.
    return b->profiling ? cudaEventRecordWithFlags(b->phase_ev[k], s, cudaEventRecordExternal)
                        : cudaSuccess;
  };
  FIP_CUDA(phase(0));
  // Per snapshot, on the branches: storage conversion and binning; the pixel
  // mappings (plain form) on the low-priority mapping branches, joined only
  // before the reprojections.
  FIP_CUDA(cudaEventRecord(b->fork, s));
  for (int i = 0; i < kBranches; ++i) FIP_CUDA(cudaStreamWaitEvent(b->branch[i], b->fork, 0));
  if (!precise) {
    for (int i = 0; i < fip_batch::kMapBranches; ++i)
      FIP_CUDA(cudaStreamWaitEvent(b->map_branch[i], b->fork, 0));
    for (int k = 0; k < count; ++k) {
      const BatchSeq& q = b->seq[l.sq[k]];
      FIP_CUDA(fip_launch_targets(q.geo, V[k], b->theta_tab, q.targets + l.loc[k] * q.n2,
                                  b->map_branch[k % fip_batch::kMapBranches]));
      launches += 1;
    }
    for (int i = 0; i < fip_batch::kMapBranches; ++i)
      FIP_CUDA(cudaEventRecord(b->map_join[i], b->map_branch[i]));
  }
  FipGridBatch in{};
  in.count = count;
  for (int k = 0; k < count; ++k) {
    const BatchSeq& q = b->seq[l.sq[k]];
    const int j = l.loc[k];
    cudaStream_t bs = b->branch[k % kBranches];
    if (reduced) {
      void* qr = static_cast<char*>(q.q_re) + j * q.cfg.max_baselines * 2;
      void* qi = static_cast<char*>(q.q_im) + j * q.cfg.max_baselines * 2;
      FIP_CUDA(fip_launch_quantize(vr[k], vi[k], nb[k], vt, qr, qi,
                                   q.q_scale + j * fip_qblocks(q.cfg.max_baselines), bs));
      launches += 1;
    }
    FipBins bins = q.bins(j);
    FIP_CUDA(fip_launch_bin(q.geo, B[k], (int)nb[k], bins, bs));
    launches += fip_bin_launches(q.geo);
    in.s[k] = grid_snap(b, l, k, B[k], V[k], vr[k], vi[k]);
  }
  for (int i = 0; i < kBranches; ++i) {
    FIP_CUDA(cudaEventRecord(b->join[i], b->branch[i]));
    FIP_CUDA(cudaStreamWaitEvent(s, b->join[i], 0));
  }
  FIP_CUDA(phase(1));
  // One persistent gridding launch for the whole call (after each sequence's
  // split tiles are zeroed), one batched transform per sequence.
  for (int c = 0; c < nseq; ++c) {
    const BatchSeq& q = b->seq[c];
    if (l.per[c] == 0) continue;
    FIP_CUDA(fip_launch_zero_batch(q.geo, q.multi, q.ntiles, q.nmulti, q.grid, q.grid_elems,
                                   l.per[c], s));
    launches += 1;
  }
  FIP_CUDA(fip_launch_grid_batch(in, vt, grid_compensated(precise, vt), s, b->grid_ctas_per_sm));
  launches += 1;
  FIP_CUDA(phase(2));
  // Grid sides not 3 * 2^k: one batched cuFFT C2R (in place, phase 2) and the
  // crop + correction per snapshot (phase 3).
  for (int c = 0; c < nseq; ++c) {
    const BatchSeq& q = b->seq[c];
    if (l.per[c] == 0) continue;
    if (q.custom_fft) {
      FIP_CUDA(fip_launch_fft_cols(q.geo, q.grid, q.bbox, q.colbuf, q.twiddles, q.fft, s,
                                   l.per[c], q.grid_elems, q.col_elems));
    } else {
      const cufftHandle plan = q.plan_for(l.per[c]);
      if (!plan) return fail(FIP_ERR_STATE, "no cuFFT plan for this call size");
      FIP_CUFFT(cufftSetStream(plan, s));
      FIP_CUFFT(cufftExecC2R(plan, reinterpret_cast<cufftComplex*>(q.grid),
                             reinterpret_cast<cufftReal*>(q.grid)));
    }
    launches += 1;
  }
  FIP_CUDA(phase(3));
  for (int c = 0; c < nseq; ++c) {
    const BatchSeq& q = b->seq[c];
    if (l.per[c] == 0) continue;
    if (q.custom_fft) {
      FIP_CUDA(fip_launch_fft_rows(q.geo, q.colbuf, q.bbox, q.taper, q.twiddles, q.fft, q.pre, s,
                                   l.per[c], q.col_elems, q.n2));
      launches += 1;
    } else {
      for (int j = 0; j < l.per[c]; ++j)
        FIP_CUDA(fip_launch_correct_c2r(q.geo, reinterpret_cast<const float*>(
                                                   q.grid + (size_t)j * q.grid_elems),
                                        q.taper, q.pre + (size_t)j * q.n2, q.bbox + 4 * j + 3, s));
      launches += l.per[c];
    }
  }
  FIP_CUDA(phase(4));
  if (!precise)
    for (int i = 0; i < fip_batch::kMapBranches; ++i)
      FIP_CUDA(cudaStreamWaitEvent(s, b->map_join[i], 0));
  // Reprojection per snapshot on the branches, into ring slots 2 .. count+1
  // of its sequence (or the caller's slots).
  if (slots) {
    for (int k = 0; k < count; ++k)
      FIP_CUDA(cudaMemsetAsync(slots[k].image_max, 0, sizeof(float), s));
  } else {
    for (int c = 0; c < nseq; ++c)
      if (l.per[c] > 0)
        FIP_CUDA(cudaMemsetAsync(b->seq[c].maxima + 2, 0, l.per[c] * sizeof(float), s));
  }
  FIP_CUDA(cudaEventRecord(b->fork, s));
  for (int i = 0; i < kBranches; ++i) FIP_CUDA(cudaStreamWaitEvent(b->branch[i], b->fork, 0));
  for (int k = 0; k < count; ++k) {
    const BatchSeq& q = b->seq[l.sq[k]];
    const int j = l.loc[k];
    cudaStream_t bs = b->branch[k % kBranches];
    float* img = slots ? slots[k].image : q.images + (j + 2) * q.n2;
    float* mx = slots ? slots[k].image_max : q.maxima + j + 2;
    FIP_CUDA(fip_launch_reproject_gather(
        q.geo, q.pre + j * q.n2, precise ? nullptr : q.targets + j * q.n2, V[k], (int)nb[k],
        q.bbox + 4 * j + 3, img, reinterpret_cast<unsigned*>(mx), precise ? 1 : 0, bs,
        b->gather_err));
    launches += 1;
  }
  for (int i = 0; i < kBranches; ++i) {
    FIP_CUDA(cudaEventRecord(b->join[i], b->branch[i]));
    FIP_CUDA(cudaStreamWaitEvent(s, b->join[i], 0));
  }
  FIP_CUDA(phase(5));
  if (slots) {
    // Each snapshot with predecessors: the tLISI of (prev 0, prev 1, itself);
    // predecessors may be images of this call (written above).
    for (int k = 0; k < count; ++k) {
      const fip_batch_slot& sl = slots[k];
      const FipGeom& geo = b->seq[l.sq[k]].geo;
      if (!sl.prev_image[0] || geo.t <= 0) continue;
      FIP_CUDA(fip_launch_trigger3(geo, sl.prev_image[0], sl.prev_image[1], sl.image,
                                   sl.prev_max[0], sl.prev_max[1], sl.image_max, sl.tlisi,
                                   precise ? 1 : 0, s));
      launches += 1;
    }
    FIP_CUDA(phase(6));
    b->launches += launches;
    return FIP_OK;
  }
  // Each sequence's sliding-window trigger: its snapshot j (slot j + 2) with
  // two predecessors.
  for (int c = 0; c < nseq; ++c) {
    const BatchSeq& q = b->seq[c];
    const int ntrig = l.per[c] - first[c];
    if (ntrig > 0 && q.geo.t > 0) {
      FIP_CUDA(fip_launch_trigger_batch(q.geo, q.images + first[c] * q.n2, q.maxima + first[c],
                                        ntrig, results[c], precise ? 1 : 0, s));
      launches += 1;
    }
  }
  FIP_CUDA(phase(6));
  // Carry each sequence's last two images (and maxima) to its slots 0, 1.
  for (int c = 0; c < nseq; ++c) {
    const BatchSeq& q = b->seq[c];
    if (l.per[c] == 0) continue;
    for (int slot = 0; slot < 2; ++slot) {
      const int from = l.per[c] + slot;  // slots per, per + 1 (per >= 1)
      if (from == slot) continue;
      FIP_CUDA(cudaMemcpyAsync(q.images + slot * q.n2, q.images + from * q.n2,
                               q.n2 * sizeof(float), cudaMemcpyDeviceToDevice, s));
      FIP_CUDA(cudaMemcpyAsync(q.maxima + slot, q.maxima + from, sizeof(float),
                               cudaMemcpyDeviceToDevice, s));
    }
  }
  b->launches += launches;
  return FIP_OK;
}

// Allocates sequence q's scratch for smax snapshots per call.
int seq_alloc(BatchSeq& q, size_t smax, size_t& tot) {
  const fip_imager_config& cfg = q.cfg;
  FipGeom& geo = q.geo;
  geo.n = (int)cfg.image_size;
  geo.g = (int)ceilf(1.5f * (float)cfg.image_size);  // FIPkernels.cu:583
  geo.hp = geo.g / 2 + 1;
  geo.t = (int)cfg.unit_size;
  geo.u = geo.t > 0 ? geo.n / geo.t : 0;
  geo.tiles_r = (geo.g + FIP_GTILE - 1) / FIP_GTILE;
  geo.tiles_c = (geo.hp + FIP_GTILE - 1) / FIP_GTILE;
  geo.cell = cfg.cell_size;
  // The band-pruned transform (grid side 3 * 2^k, power-of-two images) works
  // on the band layout; other sides on the full grid with cuFFT.
  q.custom_fft = fip_fft_plan(geo.g, q.fft);
  geo.layout = q.custom_fft ? 1 : 0;
  if (!fip_gather_supported(geo, cfg.form == FIP_FORM_PRECISE))
    return fail(FIP_ERR_ARG, "cell_size too small for the tile-gather reprojection");
#define FIP_SALLOC(call)                                                                     \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return fail(e_ == cudaErrorMemoryAllocation ? FIP_ERR_NOMEM : FIP_ERR_CUDA,            \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                       \
  } while (0)
  const size_t S = smax, nb = cfg.max_baselines;
  q.ntiles = (size_t)geo.tiles_r * geo.tiles_c;
  q.cap = 12 * nb;
  q.wcap = q.ntiles + q.cap / FIP_GCHUNK + 1;
  q.n2 = (size_t)geo.n * geo.n;
  q.grid_elems = (size_t)geo.g * geo.hp;
  q.col_elems = (size_t)geo.hp * geo.n;
  FIP_SALLOC(dalloc(&q.count, S * q.ntiles, tot));
  FIP_SALLOC(dalloc(&q.offset, S * (q.ntiles + 1), tot));
  FIP_SALLOC(dalloc(&q.cursor, S * q.ntiles, tot));
  FIP_SALLOC(dalloc(&q.entries, S * q.cap, tot));
  FIP_SALLOC(dalloc(&q.work, S * q.wcap, tot));
  FIP_SALLOC(dalloc(&q.nwork, S, tot));
  FIP_SALLOC(dalloc(&q.bbox, 4 * S, tot));
  FIP_SALLOC(dalloc(&q.multi, S * q.ntiles, tot));
  FIP_SALLOC(dalloc(&q.nmulti, S, tot));
  FIP_SALLOC(dalloc(&q.grid, S * q.grid_elems, tot));
  if (q.custom_fft) FIP_SALLOC(dalloc(&q.colbuf, S * q.col_elems, tot));
  FIP_SALLOC(dalloc(&q.pre, S * q.n2, tot));
  if (cfg.form == FIP_FORM_PLAIN) FIP_SALLOC(dalloc(&q.targets, S * q.n2, tot));
  if (cfg.form == FIP_FORM_PRECISE && cfg.vis_storage != FIP_STORE_F32) {
    FIP_SALLOC(dalloc((uint16_t**)&q.q_re, S * nb, tot));
    FIP_SALLOC(dalloc((uint16_t**)&q.q_im, S * nb, tot));
    FIP_SALLOC(dalloc(&q.q_scale, S * fip_qblocks(q.cfg.max_baselines), tot));
  }
  FIP_SALLOC(dalloc(&q.images, (S + 2) * q.n2, tot));
  FIP_SALLOC(dalloc(&q.maxima, S + 2, tot));
  FIP_SALLOC(dalloc(&q.taper, 2 * ((size_t)geo.n / 2 + 1), tot));
  if (q.custom_fft) {
    const std::vector<float2> tw = fft_twiddles(geo.g);
    FIP_SALLOC(dalloc(&q.twiddles, tw.size(), tot));
    FIP_SALLOC(cudaMemcpy(q.twiddles, tw.data(), tw.size() * sizeof(float2),
                          cudaMemcpyHostToDevice));
  }
#undef FIP_SALLOC
  return FIP_OK;
}
}  // namespace

extern "C" {

int fip_batch_create_sequences(fip_batch** out, const fip_imager_config* cfgs, size_t nseq,
                               size_t max_snapshots) {
  if (!out || !cfgs) return fail(FIP_ERR_ARG, "null argument");
  *out = nullptr;
  if (nseq < 1 || nseq > (size_t)kMaxSequences)
    return fail(FIP_ERR_ARG, "the number of sequences must be in [1, 8]");
  if (max_snapshots < 1 || max_snapshots > FIP_MAX_BATCH)
    return fail(FIP_ERR_ARG, "max_snapshots must be in [1, 64]");
  for (size_t c = 0; c < nseq; ++c) {
    const fip_imager_config* cfg = cfgs + c;
    FIP_TRY(validate_sizes(cfg->image_size, cfg->unit_size, cfg->cell_size));
    if (cfg->max_baselines == 0 || cfg->max_baselines > (1u << 24))
      return fail(FIP_ERR_ARG, "max_baselines must be in [1, 2^24]");
    if (cfg->form != FIP_FORM_PLAIN && cfg->form != FIP_FORM_PRECISE)
      return fail(FIP_ERR_ARG, "unknown form");
    if (cfg->vis_storage < 0 || cfg->vis_storage > 2) return fail(FIP_ERR_ARG, "unknown storage");
    if (cfg->reproject != 0) return fail(FIP_ERR_ARG, "the batching form reprojects by tile gather");
    if (cfg->form != cfgs[0].form || cfg->vis_storage != cfgs[0].vis_storage ||
        cfg->device != cfgs[0].device)
      return fail(FIP_ERR_ARG, "the sequences of a batch share form, storage and device");
  }
  int ndev = 0;
  FIP_CUDA(cudaGetDeviceCount(&ndev));
  if (cfgs[0].device < 0 || cfgs[0].device >= ndev) return fail(FIP_ERR_ARG, "no such device");
  DeviceGuard guard(cfgs[0].device);
  if (!guard.ok) return fail(FIP_ERR_CUDA, "cudaSetDevice failed");

  fip_batch* b = new fip_batch();
  b->cfg = cfgs[0];
  b->smax = (int)max_snapshots;
  b->seq.resize(nseq);
  auto cleanup = [&](int code) {
    std::string msg = g_last_error;
    batch_free(b);
    g_last_error = msg;
    return code;
  };
#define FIP_BALLOC(call)                                                                     \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return cleanup(fail(e_ == cudaErrorMemoryAllocation ? FIP_ERR_NOMEM : FIP_ERR_CUDA,    \
                          std::string(#call) + ": " + cudaGetErrorString(e_)));              \
  } while (0)
  size_t& tot = b->device_bytes;
  for (size_t c = 0; c < nseq; ++c) {
    b->seq[c].cfg = cfgs[c];
    const int st = seq_alloc(b->seq[c], max_snapshots, tot);
    if (st != FIP_OK) return cleanup(st);
  }
  if (b->cfg.form == FIP_FORM_PLAIN)
    FIP_BALLOC(dalloc(&b->theta_tab, fip_theta_table_elems(), tot));
  FIP_BALLOC(dalloc(&b->gather_err, 1, tot));
  FIP_BALLOC(cudaMemset(b->gather_err, 0, sizeof(unsigned)));
  {
    int least = 0, greatest = 0;
    FIP_BALLOC(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    FIP_BALLOC(cudaStreamCreateWithPriority(&b->capture, cudaStreamNonBlocking, greatest));
    for (int k = 0; k < kBranches; ++k) {
      FIP_BALLOC(cudaStreamCreateWithPriority(&b->branch[k], cudaStreamNonBlocking, greatest));
      FIP_BALLOC(cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming));
    }
    for (int k = 0; k < fip_batch::kMapBranches; ++k) {
      FIP_BALLOC(cudaStreamCreateWithPriority(&b->map_branch[k], cudaStreamNonBlocking, least));
      FIP_BALLOC(cudaEventCreateWithFlags(&b->map_join[k], cudaEventDisableTiming));
    }
  }
  FIP_BALLOC(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
  for (BatchSeq& q : b->seq) FIP_BALLOC(fip_launch_taper(q.taper, q.geo, b->branch[0]));
  if (b->theta_tab) FIP_BALLOC(fip_launch_theta_table(b->theta_tab, b->branch[0]));
  FIP_BALLOC(cudaStreamSynchronize(b->branch[0]));
#undef FIP_BALLOC
  *out = b;
  return FIP_OK;
}

int fip_batch_create(fip_batch** out, const fip_imager_config* cfg, size_t max_snapshots) {
  if (!out || !cfg) return fail(FIP_ERR_ARG, "null argument");
  return fip_batch_create_sequences(out, cfg, 1, max_snapshots);
}

int fip_batch_destroy(fip_batch* b) {
  batch_free(b);
  return FIP_OK;
}

size_t fip_batch_device_bytes(const fip_batch* b) { return b ? b->device_bytes : 0; }

unsigned long long fip_batch_kernel_launches(const fip_batch* b) { return b ? b->launches : 0; }

int fip_batch_reset(fip_batch* b) {
  if (!b) return fail(FIP_ERR_ARG, "null batch");
  for (BatchSeq& q : b->seq) q.carried = 0;
  return FIP_OK;
}

int fip_batch_set_profiling(fip_batch* b, int enable) {
  if (!b) return fail(FIP_ERR_ARG, "null batch");
  DeviceGuard g(b->cfg.device);
  FIP_TRY(batch_collect(b));
  if (enable && !b->phase_ev[0])
    for (cudaEvent_t& e : b->phase_ev) FIP_CUDA(cudaEventCreate(&e));
  if ((enable != 0) != b->profiling && b->exec) {
    cudaGraphExecDestroy(b->exec);  // the graph gains or loses its event nodes
    b->exec = nullptr;
  }
  b->profiling = enable != 0;
  for (double& v : b->phase_ms) v = 0.0;
  b->phase_calls = 0;
  return FIP_OK;
}

int fip_batch_phase_times(fip_batch* b, double* total_ms, int nphases, long* calls) {
  if (!b || !total_ms) return fail(FIP_ERR_ARG, "null argument");
  DeviceGuard g(b->cfg.device);
  FIP_TRY(batch_collect(b));
  for (int k = 0; k < nphases && k < fip_batch::kPhases; ++k) total_ms[k] = b->phase_ms[k];
  if (calls) *calls = b->phase_calls;
  return FIP_OK;
}

int fip_batch_check(fip_batch* b, void* stream) {
  if (!b) return fail(FIP_ERR_ARG, "null batch");
  DeviceGuard g(b->cfg.device);
  cudaStream_t s = (cudaStream_t)stream;
  unsigned flag = 0;
  FIP_CUDA(cudaMemcpyAsync(&flag, b->gather_err, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  FIP_CUDA(cudaMemsetAsync(b->gather_err, 0, sizeof(unsigned), s));
  FIP_CUDA(cudaStreamSynchronize(s));
  if (flag) return fail(FIP_ERR_STATE, gather_domain_message());
  return FIP_OK;
}

static int batch_run(fip_batch* b, const int* seq_of, const float* const* vis_re,
                     const float* const* vis_im, const float* const* B, const float* const* V,
                     const size_t* nb, size_t count, float* const* results, size_t* nresults,
                     void* stream, const fip_batch_slot* slots);

int fip_batch_image(fip_batch* b, const float* const* vis_re, const float* const* vis_im,
                    const float* const* B, const float* const* V, const size_t* nb, size_t count,
                    float* results, size_t* nresults, void* stream) {
  return batch_run(b, nullptr, vis_re, vis_im, B, V, nb, count, &results, nresults, stream,
                   nullptr);
}

int fip_batch_image_sequences(fip_batch* b, const int* sequence, const float* const* vis_re,
                              const float* const* vis_im, const float* const* B,
                              const float* const* V, const size_t* nb, size_t count,
                              float* const* results, size_t* nresults, void* stream) {
  if (!sequence || !results) return fail(FIP_ERR_ARG, "null argument");
  return batch_run(b, sequence, vis_re, vis_im, B, V, nb, count, results, nresults, stream,
                   nullptr);
}

int fip_batch_image_slots(fip_batch* b, const float* const* vis_re, const float* const* vis_im,
                          const float* const* B, const float* const* V, const size_t* nb,
                          size_t count, const fip_batch_slot* slots, void* stream) {
  if (!slots) return fail(FIP_ERR_ARG, "null slots");
  for (size_t k = 0; k < count; ++k) {
    const fip_batch_slot& s = slots[k];
    if (!s.image || !s.image_max) return fail(FIP_ERR_ARG, "null slot image");
    if (s.prev_image[0] && (!s.prev_image[1] || !s.prev_max[0] || !s.prev_max[1] || !s.tlisi))
      return fail(FIP_ERR_ARG, "a slot with predecessors needs both, their maxima and tlisi");
  }
  return batch_run(b, nullptr, vis_re, vis_im, B, V, nb, count, nullptr, nullptr, stream, slots);
}

static int batch_run(fip_batch* b, const int* seq_of, const float* const* vis_re,
                     const float* const* vis_im, const float* const* B, const float* const* V,
                     const size_t* nb, size_t count, float* const* results, size_t* nresults,
                     void* stream, const fip_batch_slot* slots) {
  if (!b || !vis_re || !vis_im || !B || !V || !nb) return fail(FIP_ERR_ARG, "null argument");
  const int nseq = (int)b->seq.size();
  if (count < 1 || count > (size_t)FIP_MAX_BATCH)
    return fail(FIP_ERR_ARG, "count must be in [1, 64]");
  int per[kMaxSequences] = {};
  for (size_t k = 0; k < count; ++k) {
    const int c = seq_of ? seq_of[k] : 0;
    if (c < 0 || c >= nseq) return fail(FIP_ERR_ARG, "no such sequence");
    if (++per[c] > b->smax)
      return fail(FIP_ERR_ARG, "more snapshots of one sequence than max_snapshots");
    if (!vis_re[k] || !vis_im[k] || !B[k] || !V[k]) return fail(FIP_ERR_ARG, "null device pointer");
    if (nb[k] == 0 || nb[k] > b->seq[c].cfg.max_baselines)
      return fail(FIP_ERR_ARG, "nb must be in [1, max_baselines]");
  }
  int first[kMaxSequences] = {}, ntrig[kMaxSequences] = {};
  for (int c = 0; c < nseq; ++c) {
    first[c] = std::max(0, 2 - b->seq[c].carried);
    ntrig[c] = std::max(0, per[c] - first[c]);
    if (!slots && ntrig[c] > 0 && b->seq[c].geo.t > 0 && !results[c])
      return fail(FIP_ERR_ARG, "null results");
  }
  DeviceGuard g(b->cfg.device);
  if (!g.ok) return fail(FIP_ERR_CUDA, "cudaSetDevice failed");
  cudaStream_t s = (cudaStream_t)stream;
  // The call is captured (and launched) on the batch's own highest-priority
  // stream, ordered after the caller's stream and joined back to it: its
  // latency-bound stages then take SM slots ahead of the low-priority pixel
  // mappings (and the legacy default stream, which cannot be captured, is
  // never the capture stream).
  cudaStream_t cs = b->capture;
  // cuFFT sequences: the batched C2R plan of this call's size, made before
  // the capture (making a plan allocates its work area).
  for (int c = 0; c < nseq; ++c) {
    BatchSeq& q = b->seq[c];
    if (q.custom_fft || per[c] == 0 || q.plan_for(per[c])) continue;
    cufftHandle plan = 0;
    if (cufftCreate(&plan) != CUFFT_SUCCESS) return fail(FIP_ERR_CUFFT, "cufftCreate failed");
    int nn[2] = {q.geo.g, q.geo.g}, inembed[2] = {q.geo.g, q.geo.hp},
        onembed[2] = {q.geo.g, 2 * q.geo.hp};
    size_t work = 0;
    const cufftResult r = cufftMakePlanMany(plan, 2, nn, inembed, 1, q.geo.g * q.geo.hp,
                                            onembed, 1, 2 * q.geo.g * q.geo.hp, CUFFT_C2R,
                                            per[c], &work);
    if (r != CUFFT_SUCCESS) {
      cufftDestroy(plan);
      return fail(r == CUFFT_ALLOC_FAILED ? FIP_ERR_NOMEM : FIP_ERR_CUFFT,
                  "cufftMakePlanMany(C2R) failed: " + std::to_string((int)r));
    }
    q.plans.emplace_back(per[c], plan);
    b->device_bytes += work;
  }
  FIP_CUDA(cudaEventRecord(b->fork, s));
  FIP_CUDA(cudaStreamWaitEvent(cs, b->fork, 0));
  FIP_TRY(batch_collect(b));  // the previous call's phase times, before its events are reused
  cudaGraph_t graph = nullptr;
  FIP_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  const int st = batch_record(b, seq_of, vis_re, vis_im, B, V, nb, (int)count, first, results, cs,
                              slots);
  cudaError_t e = cudaStreamEndCapture(cs, &graph);
  if (st != FIP_OK) {
    if (graph) cudaGraphDestroy(graph);
    return st;
  }
  if (e != cudaSuccess) return fail(FIP_ERR_CUDA, std::string("stream capture: ") + cudaGetErrorString(e));
  {
    // Kernel nodes run at the default (lowest) priority unless told: give
    // the call's latency-bound chain the highest and leave the pixel
    // mappings at the lowest, so they fill what the chain leaves (as the
    // lanes' stream priorities do outside graphs).
    int least = 0, greatest = 0;
    FIP_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    size_t nn = 0;
    FIP_CUDA(cudaGraphGetNodes(graph, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    if (nn) FIP_CUDA(cudaGraphGetNodes(graph, nodes.data(), &nn));
    const void* mapk = fip_targets_kernel();
    for (cudaGraphNode_t nd : nodes) {
      cudaGraphNodeType ty;
      FIP_CUDA(cudaGraphNodeGetType(nd, &ty));
      if (ty != cudaGraphNodeTypeKernel) continue;
      // Library kernels (cuFFT's) are not the runtime's to describe: such
      // nodes keep their default priority.
      cudaKernelNodeParams kp{};
      if (cudaGraphKernelNodeGetParams(nd, &kp) != cudaSuccess) {
        cudaGetLastError();
        continue;
      }
      cudaLaunchAttributeValue v{};
      v.priority = kp.func == mapk ? least : greatest;
      FIP_CUDA(cudaGraphKernelNodeSetAttribute(nd, cudaLaunchAttributePriority, &v));
    }
  }
  // Re-use the executable graph when the call's shape is unchanged (only
  // pointers, sizes and launch extents differ); instantiate otherwise.
  bool updated = false;
  if (b->exec) {
    cudaGraphExecUpdateResultInfo info{};
    updated = cudaGraphExecUpdate(b->exec, graph, &info) == cudaSuccess;
    if (!updated) {
      cudaGetLastError();
      cudaGraphExecDestroy(b->exec);
      b->exec = nullptr;
    }
  }
  if (!updated) {
    // Per-node priorities (set above) apply only with this flag.
    e = cudaGraphInstantiate(&b->exec, graph, cudaGraphInstantiateFlagUseNodePriority);
    if (e != cudaSuccess) {
      cudaGraphDestroy(graph);
      b->exec = nullptr;
      return fail(FIP_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    }
  }
  cudaGraphDestroy(graph);
  FIP_CUDA(cudaGraphLaunch(b->exec, cs));
  b->phase_pending = b->profiling;
  if (cs != s) {
    FIP_CUDA(cudaEventRecord(b->fork, cs));
    FIP_CUDA(cudaStreamWaitEvent(s, b->fork, 0));
  }
  if (!slots) {
    for (int c = 0; c < nseq; ++c) {
      BatchSeq& q = b->seq[c];
      q.carried = std::min(2, q.carried + per[c]);
      if (nresults) nresults[seq_of ? c : 0] = q.geo.t > 0 ? (size_t)ntrig[c] : 0;
      if (!seq_of) break;  // fip_batch_image: sequence 0 only
    }
  }
  return FIP_OK;
}

static int batch_autotune(fip_batch* b, const int* seq_of, const float* const* vis_re,
                          const float* const* vis_im, const float* const* B,
                          const float* const* V, const size_t* nb, size_t count, void* stream) {
  if (!b) return fail(FIP_ERR_ARG, "null batch");
  if (!vis_re || !vis_im || !B || !V || !nb) return fail(FIP_ERR_ARG, "null argument");
  const int nseq = (int)b->seq.size();
  std::vector<float*> res(nseq, nullptr);
  for (int c = 0; c < nseq; ++c) {
    const BatchSeq& q = b->seq[c];
    int per = 0;
    for (size_t k = 0; k < count; ++k) per += (seq_of ? seq_of[k] : 0) == c;
    const int ntrig = std::max(0, per - std::max(0, 2 - q.carried));
    if (ntrig > 0 && q.geo.t > 0) {
      cudaError_t e = cudaMalloc(&res[c], (size_t)ntrig * q.geo.u * q.geo.u * sizeof(float));
      if (e != cudaSuccess) {
        for (float* p : res)
          if (p) cudaFree(p);
        return fail(FIP_ERR_NOMEM, "autotune results");
      }
    }
  }
  std::vector<size_t> nr(nseq, 0);
  int st = batch_run(b, seq_of, vis_re, vis_im, B, V, nb, count, res.data(), nr.data(), stream,
                     nullptr);
  DeviceGuard g(b->cfg.device);
  cudaStream_t s = (cudaStream_t)stream;
  if (st == FIP_OK) st = cudaStreamSynchronize(s) == cudaSuccess ? FIP_OK : fail(FIP_ERR_CUDA, "sync");
  for (float* p : res)
    if (p) cudaFree(p);
  if (st != FIP_OK) return st;
  // The bins, bands and grids of these snapshots are now in place: time the
  // launch shapes on them.
  const bool precise = b->cfg.form == FIP_FORM_PRECISE;
  const int vt = batch_vis_type(b);
  const CallLayout l = call_layout(seq_of, (int)count);
  FipGridBatch in{};
  in.count = (int)count;
  for (size_t k = 0; k < count; ++k)
    in.s[k] = grid_snap(b, l, (int)k, B[k], V[k], vis_re[k], vis_im[k]);
  EventPair ev;
  FIP_CUDA(cudaEventCreate(&ev.a));
  FIP_CUDA(cudaEventCreate(&ev.b));
  auto timed = [&](auto&& launch, float& ms) -> int {
    ms = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
      FIP_CUDA(cudaEventRecord(ev.a, s));
      FIP_CUDA(launch());
      FIP_CUDA(cudaEventRecord(ev.b, s));
      FIP_CUDA(cudaEventSynchronize(ev.b));
      float t = 0.f;
      FIP_CUDA(cudaEventElapsedTime(&t, ev.a, ev.b));
      if (rep > 0) ms = std::min(ms, t);
    }
    return FIP_OK;
  };
  for (int c = 0; c < nseq; ++c) {
    BatchSeq& q = b->seq[c];
    if (l.per[c] == 0 || !q.custom_fft) continue;
    float best = 1e30f;
    fipfft::Plan chosen = q.fft;
    // Values per thread 8 or 16 x {joint, split, joint with a direct first
    // pass, joint with the row pass's band copied by bulk tensor copies}.
    for (int shape = 0; shape < 8; ++shape) {
      fipfft::Plan p{};
      if (!fip_fft_plan(q.geo.g, p, shape & 1 ? 16 : 8)) continue;
      p.split = (shape >> 1) == 1;
      p.direct = (shape >> 1) == 2 ? 1 : ((shape >> 1) == 3 ? 2 : 0);
      float ms = 0.f;
      FIP_TRY(timed(
          [&]() -> cudaError_t {
            cudaError_t e = fip_launch_fft_cols(q.geo, q.grid, q.bbox, q.colbuf, q.twiddles, p, s,
                                                l.per[c], q.grid_elems, q.col_elems);
            if (e != cudaSuccess) return e;
            return fip_launch_fft_rows(q.geo, q.colbuf, q.bbox, q.taper, q.twiddles, p, q.pre, s,
                                       l.per[c], q.col_elems, q.n2);
          },
          ms));
      if (ms < best) {
        best = ms;
        chosen = p;
      }
    }
    q.fft = chosen;
  }
  {
    float best = 1e30f;
    int chosen = 0;
    const int comp = grid_compensated(precise, vt);
    for (int c = 1; c <= fip_grid_max_ctas_per_sm(comp); ++c) {
      float ms = 0.f;
      FIP_TRY(timed([&]() -> cudaError_t { return fip_launch_grid_batch(in, vt, comp, s, c); },
                    ms));
      if (ms < best) {
        best = ms;
        chosen = c;
      }
    }
    b->grid_ctas_per_sm = chosen;
  }
  // The shapes changed: the next call instantiates a new graph.
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  for (BatchSeq& q : b->seq) q.carried = 0;
  return FIP_OK;
}

int fip_batch_autotune(fip_batch* b, const float* const* vis_re, const float* const* vis_im,
                       const float* const* B, const float* const* V, const size_t* nb,
                       size_t count, void* stream) {
  return batch_autotune(b, nullptr, vis_re, vis_im, B, V, nb, count, stream);
}

int fip_batch_autotune_sequences(fip_batch* b, const int* sequence, const float* const* vis_re,
                                 const float* const* vis_im, const float* const* B,
                                 const float* const* V, const size_t* nb, size_t count,
                                 void* stream) {
  if (!sequence) return fail(FIP_ERR_ARG, "null argument");
  return batch_autotune(b, sequence, vis_re, vis_im, B, V, nb, count, stream);
}

int fip_batch_sequence_tuning(const fip_batch* b, int sequence, int* fft_values_per_thread,
                              int* fft_split, int* fft_direct, int* grid_ctas_per_sm) {
  if (!b) return fail(FIP_ERR_ARG, "null batch");
  if (sequence < 0 || sequence >= (int)b->seq.size()) return fail(FIP_ERR_ARG, "no such sequence");
  const BatchSeq& q = b->seq[sequence];
  if (fft_values_per_thread) *fft_values_per_thread = q.fft.e;
  if (fft_split) *fft_split = q.fft.split;
  if (fft_direct) *fft_direct = q.fft.direct;
  if (grid_ctas_per_sm)
    *grid_ctas_per_sm = b->grid_ctas_per_sm > 0
                            ? b->grid_ctas_per_sm
                            : fip_grid_max_ctas_per_sm(grid_compensated(b->cfg));
  return FIP_OK;
}

int fip_batch_tuning(const fip_batch* b, int* fft_values_per_thread, int* fft_split,
                     int* fft_direct, int* grid_ctas_per_sm) {
  return fip_batch_sequence_tuning(b, 0, fft_values_per_thread, fft_split, fft_direct,
                                   grid_ctas_per_sm);
}

}  // extern "C"


int FIpipe(float* Visreal, float* Visimag, float* Bin, float* Vin, float* result_array,
           size_t num_baselines, size_t image_size, size_t num_snapshots, float cell_size,
           size_t unit_size) {
  return fip_pipe(Visreal, Visimag, Bin, Vin, result_array, num_baselines, image_size,
                  num_snapshots, cell_size, unit_size);
}
