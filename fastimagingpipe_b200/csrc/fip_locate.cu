// Trigger post-processing: transient locations from a tLISI matrix.
//
// The reference's command line writes the raw tLISI matrix and names the
// file locations.fits (README.md:41); reducing the matrix to locations is the
// step that name promises.  A location is a tile whose tLISI is below a
// threshold and is the strict minimum of its 3 x 3 neighbourhood (ties go to
// the lower tile index), refined to the centroid of the neighbourhood's
// drops 1 - tLISI and mapped to image pixels and to the reference's SIN
// projection-plane offsets (p2p's x0, y0 at FIPkernels.cu:317-322 for a
// destination pixel: x = -cell (col - N/2 - 1), y = cell (row - N/2 - 1)).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/fip.h"
#include "fip_common.cuh"
#include "fip_kernels.h"

static_assert(sizeof(fip_location) == 28, "fip_location is seven 4-byte fields");

namespace {

constexpr int kThreads = 256;

// One thread per tile.  out holds room for `cap` records; *count receives the
// number of locations found (records past cap are dropped, the count is not).
__global__ void k_locate(const float* __restrict__ t, int u, int tile, int n, float cell,
                         float threshold, fip_location* __restrict__ out, unsigned* count,
                         unsigned cap) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= u * u) return;
  const float v = t[b];
  if (!(v < threshold)) return;  // NaN tiles never qualify
  const int r = b / u, c = b % u;
  float ws = 0.f, wr = 0.f, wc = 0.f;
  for (int dr = -1; dr <= 1; ++dr)
    for (int dc = -1; dc <= 1; ++dc) {
      const int rr = r + dr, cc = c + dc;
      if (rr < 0 || rr >= u || cc < 0 || cc >= u) continue;
      const int nb = rr * u + cc;
      const float w = t[nb];
      if (nb != b && (w < v || (w == v && nb < b))) return;  // not the minimum
      const float drop = w == w ? fmaxf(0.f, 1.0f - w) : 0.f;
      ws += drop;
      wr += drop * (float)dr;
      wc += drop * (float)dc;
    }
  const float fr = (float)r + (ws > 0.f ? wr / ws : 0.f);
  const float fc = (float)c + (ws > 0.f ? wc / ws : 0.f);
  // Tile k covers pixels k T .. k T + T - 1: its centre is k T + (T - 1) / 2.
  const float row = fr * (float)tile + 0.5f * (float)(tile - 1);
  const float col = fc * (float)tile + 0.5f * (float)(tile - 1);
  const float h1 = (float)(n / 2 + 1);
  const unsigned k = atomicAdd(count, 1u);
  if (k < cap) {
    fip_location L;
    L.tile_row = r;
    L.tile_col = c;
    L.tlisi = v;
    L.row = row;
    L.col = col;
    L.x = -cell * (col - h1);
    L.y = cell * (row - h1);
    out[k] = L;
  }
}

}  // namespace

extern "C" int fip_locate_transients(const float* tlisi, size_t image_size, size_t unit_size,
                                     float cell_size, float threshold, fip_location* out,
                                     size_t max_out, size_t* found, void* stream) {
  if (!tlisi || !found || (max_out > 0 && !out))
    return fip_set_error(FIP_ERR_ARG, "null argument");
  if (unit_size == 0 || image_size < unit_size)
    return fip_set_error(FIP_ERR_ARG, "unit_size must be in [1, image_size]");
  if (!(cell_size > 0.f)) return fip_set_error(FIP_ERR_ARG, "cell_size must be positive");
  const size_t u = image_size / unit_size;
  if (u * u > (1u << 26)) return fip_set_error(FIP_ERR_ARG, "tLISI matrix too large");
  cudaStream_t s = (cudaStream_t)stream;
  const size_t cap = u * u;  // every tile could qualify
  // Stream-ordered scratch (post-processing, not the imaging hot path): the
  // records and the count in one block.
  char* scratch = nullptr;
  const size_t rec_bytes = cap * sizeof(fip_location);
  cudaError_t e = cudaMallocAsync((void**)&scratch, rec_bytes + 16, s);
  if (e != cudaSuccess) return fip_set_error(FIP_ERR_NOMEM, cudaGetErrorString(e));
  fip_location* d_rec = reinterpret_cast<fip_location*>(scratch);
  unsigned* d_count = reinterpret_cast<unsigned*>(scratch + rec_bytes);
  unsigned count = 0;
  std::vector<fip_location> rec;
  e = cudaMemsetAsync(d_count, 0, sizeof(unsigned), s);
  if (e == cudaSuccess) {
    k_locate<<<(unsigned)((cap + kThreads - 1) / kThreads), kThreads, 0, s>>>(
        tlisi, (int)u, (int)unit_size, (int)image_size, cell_size, threshold, d_rec, d_count,
        (unsigned)cap);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&count, d_count, sizeof(unsigned),
                                            cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess && count > 0) {
    rec.resize(std::min<size_t>(count, cap));
    e = cudaMemcpyAsync(rec.data(), d_rec, rec.size() * sizeof(fip_location),
                        cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  }
  const cudaError_t ef = cudaFreeAsync(scratch, s);
  if (e == cudaSuccess) e = ef;
  if (e != cudaSuccess) return fip_set_error(FIP_ERR_CUDA, cudaGetErrorString(e));
  // Deepest drop first; equal values in tile order (the kernel's record order
  // depends on scheduling, the returned order does not).
  std::sort(rec.begin(), rec.end(), [u](const fip_location& a, const fip_location& b) {
    if (a.tlisi != b.tlisi) return a.tlisi < b.tlisi;
    return (size_t)a.tile_row * u + a.tile_col < (size_t)b.tile_row * u + b.tile_col;
  });
  for (size_t k = 0; k < rec.size() && k < max_out; ++k) out[k] = rec[k];
  *found = count;
  return FIP_OK;
}
