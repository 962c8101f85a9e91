// Gridding for callers that cannot allocate device memory.
//
// Some callers of this library run where cudaMalloc is not available to them:
// code inside a pre-sized memory pool or arena that must not grow, plugins
// loaded into a host application that owns every device allocation, and
// real-time loops that may not call into the allocator (cudaMalloc can
// synchronise the device and take milliseconds).  fip_grid_snapshot needs an
// imager, whose creation allocates the binning scratch; the entry point below
// grids one snapshot with that scratch held instead in a fixed-size device
// array that is part of the library image, so the call itself allocates
// nothing.  The caller still provides the inputs and the output grid.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "../../include/fip.h"
#include "fip_common.cuh"
#include "fip_kernels.h"

namespace {

// Limits of the fixed scratch: up to 2^17 visibilities per snapshot and
// images up to 4096 x 4096 (grid side 6144, 96 x 49 tiles of 64 x 64 cells).
constexpr size_t kMaxBaselines = 131072;
constexpr size_t kMaxImage = 4096;
constexpr int kMaxTiles = 96 * 49;
constexpr size_t kMaxEntries = 12 * kMaxBaselines;  // <= 12 tile entries per visibility
constexpr size_t kMaxWork = kMaxTiles + kMaxEntries / FIP_GCHUNK + 1;

// Layout of the scratch: the per-tile bins of one snapshot.
struct Scratch {
  int4 work[kMaxWork];
  unsigned count[kMaxTiles];
  unsigned offset[kMaxTiles + 1];
  unsigned cursor[kMaxTiles];
  unsigned multi[kMaxTiles];
  unsigned nwork;
  unsigned nmulti;
  unsigned bbox[4];
  unsigned entries[kMaxEntries];
};

}  // namespace

// About 6.5 MB, present on every GPU that loads the library until the
// process exits.  Shared by all calls: every call rewrites what it reads
// (counts and the band record are cleared by the binning pass), and calls
// whose work overlaps on the GPU race on it.
static __device__ __align__(256) unsigned char g_grid_scratch[sizeof(Scratch)];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
void* g_addr[kMaxDevices] = {};

// Device address of g_grid_scratch on the current device.  Host code only
// sees a host-side stand-in for the symbol, so the address is looked up with
// the device current.  Outside stream capture the lookup runs on every call
// (it allocates nothing), so a caller that reset the device and got a new
// context gets the array's new address; while `stream` is capturing, the
// address recorded by the last call outside capture is used, so that the
// first call on a device has to come before any capture.
int scratch_address(cudaStream_t stream, Scratch** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fip_set_error(FIP_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fip_set_error(FIP_ERR_ARG, "device ordinal too large");
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(stream, &cap);
  if (e != cudaSuccess) return fip_set_error(FIP_ERR_CUDA, cudaGetErrorString(e));
  std::lock_guard<std::mutex> lock(g_addr_mu);
  if (cap == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_grid_scratch);
    if (e != cudaSuccess || p == nullptr)
      return fip_set_error(FIP_ERR_CUDA,
                           std::string("cudaGetSymbolAddress(grid scratch): ") +
                               cudaGetErrorString(e));
    g_addr[dev] = p;
  } else if (!g_addr[dev]) {
    return fip_set_error(FIP_ERR_STATE,
                         "fip_grid_snapshot_noalloc: the first call on a device must come "
                         "before any stream capture");
  }
  *out = static_cast<Scratch*>(g_addr[dev]);
  return FIP_OK;
}

}  // namespace

extern "C" int fip_grid_snapshot_noalloc(const float* vis_re, const float* vis_im,
                                         const float* B, const float* V, size_t nb,
                                         size_t image_size, float cell_size, float* grid,
                                         void* stream) {
  if (!vis_re || !vis_im || !B || !V || !grid) return fip_set_error(FIP_ERR_ARG, "null device pointer");
  if (nb == 0 || nb > kMaxBaselines)
    return fip_set_error(FIP_ERR_ARG,
                         "fip_grid_snapshot_noalloc: nb must be in [1, 131072] (fixed scratch "
                         "size); use fip_grid_snapshot for larger snapshots");
  if (image_size < 16 || image_size % 4 != 0 || image_size > kMaxImage)
    return fip_set_error(FIP_ERR_ARG,
                         "fip_grid_snapshot_noalloc: image_size must be a multiple of 4 in "
                         "[16, 4096] (fixed scratch size)");
  if (!(cell_size > 0.f) || !(cell_size < 1.f))
    return fip_set_error(FIP_ERR_ARG, "cell_size must be in (0, 1) rad");
  cudaStream_t s = (cudaStream_t)stream;
  Scratch* sc = nullptr;
  const int st = scratch_address(s, &sc);
  if (st != FIP_OK) return st;

  FipGeom geo{};
  geo.n = (int)image_size;
  geo.g = (int)ceilf(1.5f * (float)image_size);  // FIPkernels.cu:583
  geo.hp = geo.g / 2 + 1;
  geo.tiles_r = (geo.g + FIP_GTILE - 1) / FIP_GTILE;
  geo.tiles_c = (geo.hp + FIP_GTILE - 1) / FIP_GTILE;
  geo.cell = cell_size;
  geo.layout = 0;  // full half plane, row-major: every tile is written

  FipBins bins{};
  bins.count = sc->count;
  bins.offset = sc->offset;
  bins.cursor = sc->cursor;
  bins.entries = sc->entries;
  bins.work = sc->work;
  bins.nwork = &sc->nwork;
  bins.bbox = sc->bbox;
  bins.multi = sc->multi;
  bins.nmulti = &sc->nmulti;
  bins.cap = kMaxEntries;
  bins.wcap = kMaxWork;

  cudaError_t e = fip_launch_bin(geo, B, (int)nb, bins, s);
  if (e == cudaSuccess)
    e = fip_launch_grid(geo, B, vis_re, vis_im, FIP_VIS_F32, nullptr, V, (int)nb, bins,
                        reinterpret_cast<float2*>(grid), 0, s);
  if (e != cudaSuccess) return fip_set_error(FIP_ERR_CUDA, cudaGetErrorString(e));
  return FIP_OK;
}
