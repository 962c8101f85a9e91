// Multi-beam streaming server: continuous batching of snapshot requests.
//
// Each beam owns an imager (its grid, bins, FFT buffers and a ring of its last
// three images, so every new snapshot yields the tLISI of the triple ending
// with it) and one CUDA stream.  Requests from all beams enter one FIFO; a
// pool of worker threads ("slots") takes the oldest request whose beam is not
// already being served, so work of different beams overlaps on the device
// while each beam's snapshots stay in order.  A request is admitted into the
// queue only when its beam was admitted under the server's HBM budget (beam
// creation reserves the imager's device memory) and the queue has room;
// otherwise submit returns FIP_ERR_BUDGET / FIP_ERR_NOT_READY and the caller
// retries.  Latency is measured per request from submit to result.
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/fip.h"
#include "fip_kernels.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Beam {
  int id = 0;
  fip_imager_config cfg{};
  fip_imager* im = nullptr;
  cudaStream_t stream = nullptr;
  size_t bytes = 0;
  long seen = 0;       // snapshots imaged so far
  bool busy = false;   // a worker is serving it
  // Device inputs of the request in service and the three image maxima.
  float *d_vr = nullptr, *d_vi = nullptr, *d_B = nullptr, *d_V = nullptr;
  float *h_vr = nullptr, *h_vi = nullptr, *h_B = nullptr, *h_V = nullptr;  // pinned
  float* d_img[3] = {nullptr, nullptr, nullptr};
  float* d_max = nullptr;
  float* d_res = nullptr;
  float* h_res = nullptr;
};

struct Request {
  long id;
  int beam;
  size_t nb;
  std::vector<float> vr, vi, B, V;
  Clock::time_point t_submit;
};

struct Result {
  int status = FIP_OK;
  int beam = 0;
  long seq = 0;          // snapshot index within the beam
  bool has_tlisi = false;
  std::vector<float> tlisi;
  double latency_ms = 0.0;
  std::string error;
};

}  // namespace

struct fip_server {
  int device = 0;
  size_t budget = 0, reserved = 0, max_queue = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::vector<std::unique_ptr<Beam>> beams;
  std::deque<Request> queue;
  std::map<long, Result> done;
  long next_id = 1;
  long in_service = 0;
  bool stopping = false;
  std::vector<std::thread> workers;
};

namespace {

void free_beam(Beam* b) {
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->im) fip_imager_destroy(b->im);
  void* d[] = {b->d_vr, b->d_vi, b->d_B, b->d_V, b->d_img[0], b->d_img[1], b->d_img[2],
               b->d_max, b->d_res};
  for (void* p : d)
    if (p) cudaFree(p);
  void* h[] = {b->h_vr, b->h_vi, b->h_B, b->h_V, b->h_res};
  for (void* p : h)
    if (p) cudaFreeHost(p);
  if (b->stream) cudaStreamDestroy(b->stream);
}

// Images one request of beam b and, from the third snapshot on, its tLISI.
int serve(Beam* b, Request& r, Result& out) {
  const size_t nb = r.nb;
  cudaStream_t s = b->stream;
  std::memcpy(b->h_vr, r.vr.data(), nb * sizeof(float));
  std::memcpy(b->h_vi, r.vi.data(), nb * sizeof(float));
  std::memcpy(b->h_B, r.B.data(), 2 * nb * sizeof(float));
  std::memcpy(b->h_V, r.V.data(), 9 * sizeof(float));
  cudaError_t e = cudaMemcpyAsync(b->d_vr, b->h_vr, nb * sizeof(float), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_vi, b->h_vi, nb * sizeof(float), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_B, b->h_B, 2 * nb * sizeof(float), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_V, b->h_V, 9 * sizeof(float), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return fip_set_error(FIP_ERR_CUDA, cudaGetErrorString(e));
  const int slot = (int)(b->seen % 3);
  int st = fip_image_snapshot(b->im, b->d_vr, b->d_vi, b->d_B, b->d_V, nb, b->d_img[slot],
                              b->d_max + slot, s);
  if (st != FIP_OK) return st;
  out.seq = b->seen;
  if (b->seen >= 2) {
    const int a = (int)((b->seen - 2) % 3), c = (int)((b->seen - 1) % 3);
    st = fip_trigger(b->im, b->d_img[a], b->d_img[c], b->d_img[slot], b->d_max, b->d_res, s);
    if (st != FIP_OK) return st;
    const size_t uu = (b->cfg.image_size / b->cfg.unit_size) * (b->cfg.image_size / b->cfg.unit_size);
    e = cudaMemcpyAsync(b->h_res, b->d_res, uu * sizeof(float), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return fip_set_error(FIP_ERR_CUDA, cudaGetErrorString(e));
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fip_set_error(FIP_ERR_CUDA, cudaGetErrorString(e));
    out.has_tlisi = true;
    out.tlisi.assign(b->h_res, b->h_res + uu);
  } else {
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fip_set_error(FIP_ERR_CUDA, cudaGetErrorString(e));
  }
  b->seen += 1;
  return FIP_OK;
}

void worker_loop(fip_server* sv) {
  cudaSetDevice(sv->device);
  for (;;) {
    Request req;
    Beam* b = nullptr;
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      for (;;) {
        if (sv->stopping) return;
        auto it = sv->queue.begin();
        for (; it != sv->queue.end(); ++it)
          if (!sv->beams[it->beam]->busy) break;
        if (it != sv->queue.end()) {
          req = std::move(*it);
          sv->queue.erase(it);
          b = sv->beams[req.beam].get();
          b->busy = true;
          sv->in_service += 1;
          break;
        }
        sv->cv_work.wait(lk);
      }
    }
    Result res;
    res.beam = req.beam;
    res.status = serve(b, req, res);
    if (res.status != FIP_OK) res.error = fip_last_error();
    res.latency_ms =
        std::chrono::duration<double, std::milli>(Clock::now() - req.t_submit).count();
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      b->busy = false;
      sv->in_service -= 1;
      sv->done[req.id] = std::move(res);
    }
    sv->cv_work.notify_all();
    sv->cv_done.notify_all();
  }
}

}  // namespace

extern "C" {

int fip_server_create(fip_server** out, int device, size_t hbm_budget_bytes, int slots,
                      size_t max_queue) {
  if (!out) return fip_set_error(FIP_ERR_ARG, "null argument");
  *out = nullptr;
  if (slots < 1 || slots > 64) return fip_set_error(FIP_ERR_ARG, "slots must be in [1, 64]");
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess) return fip_set_error(FIP_ERR_CUDA, cudaGetErrorString(e));
  if (device < 0 || device >= ndev) return fip_set_error(FIP_ERR_ARG, "no such device");
  fip_server* sv = new fip_server();
  sv->device = device;
  sv->budget = hbm_budget_bytes;
  sv->max_queue = max_queue ? max_queue : 1024;
  for (int k = 0; k < slots; ++k) sv->workers.emplace_back(worker_loop, sv);
  *out = sv;
  return FIP_OK;
}

int fip_server_destroy(fip_server* sv) {
  if (!sv) return FIP_OK;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stopping = true;
  }
  sv->cv_work.notify_all();
  for (auto& t : sv->workers) t.join();
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(sv->device);
  for (auto& b : sv->beams) free_beam(b.get());
  cudaSetDevice(prev);
  delete sv;
  return FIP_OK;
}

int fip_server_add_beam(fip_server* sv, const fip_imager_config* cfg, int* beam_id) {
  if (!sv || !cfg || !beam_id) return fip_set_error(FIP_ERR_ARG, "null argument");
  if (cfg->unit_size == 0) return fip_set_error(FIP_ERR_ARG, "a beam needs a trigger tile");
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(sv->device);
  auto b = std::make_unique<Beam>();
  b->cfg = *cfg;
  b->cfg.device = sv->device;
  const size_t n2 = cfg->image_size * cfg->image_size, nb = cfg->max_baselines;
  const size_t uu = (cfg->image_size / cfg->unit_size) * (cfg->image_size / cfg->unit_size);
  int st = fip_imager_create(&b->im, &b->cfg);
  if (st == FIP_OK) {
    b->bytes = fip_imager_device_bytes(b->im) + (3 * n2 + uu + 3 + 4 * nb + 9) * sizeof(float);
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->reserved + b->bytes > sv->budget) {
      st = fip_set_error(FIP_ERR_BUDGET, "beam does not fit in the server's HBM budget (" +
                                             std::to_string(sv->reserved + b->bytes) + " > " +
                                             std::to_string(sv->budget) + " bytes)");
    } else {
      sv->reserved += b->bytes;  // reserve before allocating the rest
    }
  }
  cudaError_t e = cudaSuccess;
  if (st == FIP_OK) {
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_vr, nb * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_vi, nb * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_B, 2 * nb * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_V, 9 * sizeof(float));
    for (int k = 0; k < 3 && e == cudaSuccess; ++k) e = cudaMalloc(&b->d_img[k], n2 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_max, 3 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_res, uu * sizeof(float));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_vr, nb * sizeof(float));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_vi, nb * sizeof(float));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_B, 2 * nb * sizeof(float));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_V, 9 * sizeof(float));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_res, uu * sizeof(float));
    if (e != cudaSuccess) {
      st = fip_set_error(e == cudaErrorMemoryAllocation ? FIP_ERR_NOMEM : FIP_ERR_CUDA,
                         cudaGetErrorString(e));
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->reserved -= b->bytes;
    }
  }
  if (st != FIP_OK) {
    free_beam(b.get());
    cudaSetDevice(prev);
    return st;
  }
  std::lock_guard<std::mutex> lk(sv->mu);
  b->id = (int)sv->beams.size();
  *beam_id = b->id;
  sv->beams.push_back(std::move(b));
  cudaSetDevice(prev);
  return FIP_OK;
}

size_t fip_server_reserved_bytes(fip_server* sv) {
  if (!sv) return 0;
  std::lock_guard<std::mutex> lk(sv->mu);
  return sv->reserved;
}

int fip_server_submit(fip_server* sv, int beam, const float* vis_re, const float* vis_im,
                      const float* B, const float* V, size_t nb, long* request_id) {
  if (!sv || !vis_re || !vis_im || !B || !V || !request_id)
    return fip_set_error(FIP_ERR_ARG, "null argument");
  Request r;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (beam < 0 || beam >= (int)sv->beams.size()) return fip_set_error(FIP_ERR_ARG, "no such beam");
    if (nb == 0 || nb > sv->beams[beam]->cfg.max_baselines)
      return fip_set_error(FIP_ERR_ARG, "nb must be in [1, the beam's max_baselines]");
    if (sv->queue.size() >= sv->max_queue) return fip_set_error(FIP_ERR_NOT_READY, "queue full");
    r.id = sv->next_id++;
  }
  r.beam = beam;
  r.nb = nb;
  r.vr.assign(vis_re, vis_re + nb);
  r.vi.assign(vis_im, vis_im + nb);
  r.B.assign(B, B + 2 * nb);
  r.V.assign(V, V + 9);
  r.t_submit = Clock::now();
  *request_id = r.id;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->queue.push_back(std::move(r));
  }
  sv->cv_work.notify_one();
  return FIP_OK;
}

int fip_server_wait(fip_server* sv, long request_id, double timeout_ms, int* beam, long* seq,
                    int* has_tlisi, float* tlisi, size_t tlisi_len, double* latency_ms) {
  if (!sv) return fip_set_error(FIP_ERR_ARG, "null server");
  std::unique_lock<std::mutex> lk(sv->mu);
  const auto deadline = Clock::now() + std::chrono::microseconds((long)(timeout_ms * 1000.0));
  while (sv->done.find(request_id) == sv->done.end()) {
    if (timeout_ms >= 0 && sv->cv_done.wait_until(lk, deadline) == std::cv_status::timeout &&
        sv->done.find(request_id) == sv->done.end())
      return fip_set_error(FIP_ERR_NOT_READY, "request not finished");
    if (timeout_ms < 0) sv->cv_done.wait(lk);
  }
  Result r = std::move(sv->done[request_id]);
  sv->done.erase(request_id);
  lk.unlock();
  if (beam) *beam = r.beam;
  if (seq) *seq = r.seq;
  if (has_tlisi) *has_tlisi = r.has_tlisi ? 1 : 0;
  if (latency_ms) *latency_ms = r.latency_ms;
  if (r.has_tlisi && tlisi) {
    if (tlisi_len < r.tlisi.size()) return fip_set_error(FIP_ERR_ARG, "tlisi buffer too small");
    std::memcpy(tlisi, r.tlisi.data(), r.tlisi.size() * sizeof(float));
  }
  if (r.status != FIP_OK) return fip_set_error(r.status, r.error);
  return FIP_OK;
}

}  // extern "C"
