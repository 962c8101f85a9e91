// Multi-beam streaming server: continuous batching of snapshot requests.
//
// Beams whose imager configuration is the same (image size, baselines,
// cell, tile, form, storage) form a group that shares one batch engine
// (fip_batch): a worker thread ("slot") takes up to the group's step size of
// the queued snapshots of that group -- any of its beams, each beam's in
// order -- and images them in ONE batched call (one persistent gridding
// launch, one batched transform, the per-snapshot gathers and triggers in one
// CUDA graph, fip_batch_image_slots).  Each beam keeps its last two images on
// the device (in buffers of the group's image pool), so every snapshot from
// a beam's third on yields the tLISI of the triple ending with it (the
// reference's trigger, FIPkernels.cu:806-851, as a sliding window); a beam's
// snapshots later in the same step use the earlier ones' fresh images.
// Requests that arrive while a step runs wait in the queue and join the
// group's next step, so the engine never idles while work is queued, and
// steps of different groups overlap on the device.
//
// HBM admission: a beam is admitted when its two resident images fit in the
// budget, and a group's step size -- how many snapshots it may have on the
// device at once, each with its own gridding, transform and reprojection
// scratch, input staging and output image -- is the largest (up to the
// server's batch limit) whose memory fits in what the budget has left when
// the group is created.  A request enters the device only when its group's
// engine takes it into a step; until then it waits in the host queue, which
// holds max_queue requests (FIP_ERR_NOT_READY beyond that).
//
// Beams of image sizes that are not powers of two, or with the scatter
// reprojection, get an imager of their own and are served one snapshot at a
// time: the batch engine transforms such sizes with cuFFT, whose plan and
// work area per step size are made on first use, outside the memory that the
// group's HBM admission sizes.  Latency is measured per request from submit to
// result.
#include <cuda_runtime.h>

#include <algorithm>
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
constexpr int kDefaultStep = 8;  // snapshots per batched step at most

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
  long seq = 0;  // snapshot index within the beam
  bool has_tlisi = false;
  std::vector<float> tlisi;
  double latency_ms = 0.0;
  std::string error;
};

// An image buffer of a group's pool: N*N floats, then the image maximum.
struct ImageBuf {
  float* p = nullptr;
  int refs = 0;  // beams' rings holding it
};

struct Group {
  fip_imager_config cfg{};
  fip_batch* batch = nullptr;
  int step = 0;  // snapshots per batched step (budget-sized)
  bool busy = false;
  cudaStream_t stream = nullptr;
  size_t n2 = 0, uu = 0, nb = 0, bytes = 0;
  // Input staging of one step: per snapshot B [2 nb], vis real [nb], vis
  // imaginary [nb], V [9], pinned and on the device.
  float *h_in = nullptr, *d_in = nullptr;
  float *h_res = nullptr, *d_res = nullptr;  // [step][U*U]
  std::vector<ImageBuf> pool;
  size_t stride() const { return 4 * nb + 16; }
};

struct Beam {
  int id = 0;
  fip_imager_config cfg{};
  int group = -1;  // batched group, or -1: own imager
  long seen = 0;   // snapshots imaged so far
  bool busy = false;
  int ring[2] = {-1, -1};  // pool indices of the last two images (oldest first)
  // Own-imager beams: device inputs, three images and maxima.
  fip_imager* im = nullptr;
  cudaStream_t stream = nullptr;
  size_t bytes = 0;
  float *d_vr = nullptr, *d_vi = nullptr, *d_B = nullptr, *d_V = nullptr;
  float *h_vr = nullptr, *h_vi = nullptr, *h_B = nullptr, *h_V = nullptr;  // pinned
  float* d_img[3] = {nullptr, nullptr, nullptr};
  float* d_max = nullptr;
  float* d_res = nullptr;
  float* h_res = nullptr;
};

}  // namespace

struct fip_server {
  int device = 0;
  size_t budget = 0, reserved = 0, max_queue = 0;
  int max_step = kDefaultStep;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::vector<std::unique_ptr<Beam>> beams;
  std::vector<std::unique_ptr<Group>> groups;
  std::deque<Request> queue;
  std::map<long, Result> done;
  long next_id = 1;
  long steps = 0, stepped = 0;  // batched steps run and snapshots they imaged
  bool stopping = false;
  std::vector<std::thread> workers;
};

namespace {

bool same_cfg(const fip_imager_config& a, const fip_imager_config& b) {
  return a.image_size == b.image_size && a.max_baselines == b.max_baselines &&
         a.unit_size == b.unit_size && a.cell_size == b.cell_size && a.form == b.form &&
         a.vis_storage == b.vis_storage && a.reproject == b.reproject;
}

bool batchable(const fip_imager_config& c) {
  const size_t n = c.image_size;
  return c.reproject == 0 && n >= 8 && (n & (n - 1)) == 0 && c.max_baselines <= (1u << 24);
}

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

void free_group(Group* g) {
  if (!g) return;
  if (g->stream) cudaStreamSynchronize(g->stream);
  if (g->batch) fip_batch_destroy(g->batch);
  for (ImageBuf& ib : g->pool)
    if (ib.p) cudaFree(ib.p);
  if (g->d_in) cudaFree(g->d_in);
  if (g->d_res) cudaFree(g->d_res);
  if (g->h_in) cudaFreeHost(g->h_in);
  if (g->h_res) cudaFreeHost(g->h_res);
  if (g->stream) cudaStreamDestroy(g->stream);
}

int cuda_fail(cudaError_t e) {
  return fip_set_error(e == cudaErrorMemoryAllocation ? FIP_ERR_NOMEM : FIP_ERR_CUDA,
                       cudaGetErrorString(e));
}

// Adds `count` image buffers to a group's pool.
cudaError_t grow_pool(Group* g, int count) {
  for (int k = 0; k < count; ++k) {
    ImageBuf ib;
    cudaError_t e = cudaMalloc(&ib.p, (g->n2 + 64) * sizeof(float));
    if (e != cudaSuccess) return e;
    g->pool.push_back(ib);
  }
  return cudaSuccess;
}

int free_buf(Group* g) {
  for (int k = 0; k < (int)g->pool.size(); ++k)
    if (g->pool[k].refs == 0) return k;
  return -1;
}

// Images one request of an own-imager beam and, from its third snapshot on,
// its tLISI.
int serve_one(Beam* b, Request& r, Result& out) {
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
  if (e != cudaSuccess) return cuda_fail(e);
  const int slot = (int)(b->seen % 3);
  int st = fip_image_snapshot(b->im, b->d_vr, b->d_vi, b->d_B, b->d_V, nb, b->d_img[slot],
                              b->d_max + slot, s);
  if (st != FIP_OK) return st;
  out.seq = b->seen;
  if (b->seen >= 2) {
    const int a = (int)((b->seen - 2) % 3), c = (int)((b->seen - 1) % 3);
    // The trigger uses the maximum of the three maxima only, so their slot
    // order is the triple's as far as it is concerned.
    st = fip_trigger(b->im, b->d_img[a], b->d_img[c], b->d_img[slot], b->d_max, b->d_res, s);
    if (st != FIP_OK) return st;
    const size_t uu = (b->cfg.image_size / b->cfg.unit_size) * (b->cfg.image_size / b->cfg.unit_size);
    e = cudaMemcpyAsync(b->h_res, b->d_res, uu * sizeof(float), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return cuda_fail(e);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e);
    out.has_tlisi = true;
    out.tlisi.assign(b->h_res, b->h_res + uu);
  } else {
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e);
  }
  return fip_imager_check(b->im, s);
}

// One batched step of a group: the requests (in queue order; a beam's may
// repeat) imaged in one fip_batch_image_slots call.  Takes the server lock
// only to read and update the beams' rings and the pool.
void serve_step(fip_server* sv, Group* g, std::vector<Request>& reqs,
                std::vector<Result>& out) {
  const int count = (int)reqs.size();
  const size_t st = g->stride(), nb = g->nb;
  out.assign(count, Result());
  // Stage every snapshot's inputs into its slot of the pinned block.
  for (int k = 0; k < count; ++k) {
    float* h = g->h_in + k * st;
    const Request& r = reqs[k];
    std::memcpy(h, r.B.data(), 2 * r.nb * sizeof(float));
    std::memcpy(h + 2 * nb, r.vr.data(), r.nb * sizeof(float));
    std::memcpy(h + 3 * nb, r.vi.data(), r.nb * sizeof(float));
    std::memcpy(h + 4 * nb, r.V.data(), 9 * sizeof(float));
  }
  cudaStream_t s = g->stream;
  cudaError_t e =
      cudaMemcpyAsync(g->d_in, g->h_in, count * st * sizeof(float), cudaMemcpyHostToDevice, s);
  std::vector<const float*> vr(count), vi(count), B(count), V(count);
  std::vector<size_t> nbs(count);
  std::vector<fip_batch_slot> slots(count);
  // Buffers this step writes or reads, held until it ends: a buffer that
  // leaves a beam's ring during the step may still be read by the step's
  // triggers, so it is not handed to a later snapshot of the same step.
  std::vector<int> held;
  int status = e == cudaSuccess ? FIP_OK : cuda_fail(e);
  if (status == FIP_OK) {
    std::lock_guard<std::mutex> lk(sv->mu);
    for (int k = 0; k < count && status == FIP_OK; ++k) {
      Beam* b = sv->beams[reqs[k].beam].get();
      const float* d = g->d_in + k * st;
      B[k] = d;
      vr[k] = d + 2 * nb;
      vi[k] = d + 3 * nb;
      V[k] = d + 4 * nb;
      nbs[k] = reqs[k].nb;
      // The pool holds two buffers per beam (their rings) and one per step
      // snapshot: with the rings' dropped buffers held, never short.
      const int buf = free_buf(g);
      if (buf < 0) {
        status = fip_set_error(FIP_ERR_STATE, "image pool exhausted");
        break;
      }
      g->pool[buf].refs += 1;
      held.push_back(buf);
      fip_batch_slot& sl = slots[k];
      sl.image = g->pool[buf].p;
      sl.image_max = g->pool[buf].p + g->n2;
      out[k].beam = b->id;
      out[k].seq = b->seen;
      if (b->seen >= 2) {
        for (int q = 0; q < 2; ++q) {
          sl.prev_image[q] = g->pool[b->ring[q]].p;
          sl.prev_max[q] = g->pool[b->ring[q]].p + g->n2;
          g->pool[b->ring[q]].refs += 1;
          held.push_back(b->ring[q]);
        }
        sl.tlisi = g->d_res + k * g->uu;
        out[k].has_tlisi = true;
      }
      // The beam's ring moves on: its next snapshot (in this step or later)
      // sees this one as its latest image.
      if (b->ring[0] >= 0) g->pool[b->ring[0]].refs -= 1;
      b->ring[0] = b->ring[1];
      b->ring[1] = buf;
      g->pool[buf].refs += 1;
      b->seen += 1;
    }
  }
  if (status == FIP_OK)
    status = fip_batch_image_slots(g->batch, vr.data(), vi.data(), B.data(), V.data(),
                                   nbs.data(), count, slots.data(), s);
  if (status == FIP_OK) {
    e = cudaMemcpyAsync(g->h_res, g->d_res, count * g->uu * sizeof(float),
                        cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) status = cuda_fail(e);
  }
  if (status == FIP_OK) status = fip_batch_check(g->batch, s);
  std::string err = status == FIP_OK ? std::string() : std::string(fip_last_error());
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    for (int k : held) g->pool[k].refs -= 1;  // the step's holds
  }
  for (int k = 0; k < count; ++k) {
    out[k].status = status;
    out[k].error = err;
    if (status == FIP_OK && out[k].has_tlisi)
      out[k].tlisi.assign(g->h_res + k * g->uu, g->h_res + (k + 1) * g->uu);
    else
      out[k].has_tlisi = out[k].has_tlisi && status == FIP_OK;
  }
}

void worker_loop(fip_server* sv) {
  cudaSetDevice(sv->device);
  for (;;) {
    std::vector<Request> reqs;
    Group* g = nullptr;
    Beam* solo = nullptr;
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      for (;;) {
        if (sv->stopping) return;
        // The oldest request whose group (or own-imager beam) is idle opens
        // the work item; a group's step then takes every queued request of
        // that group, oldest first, up to its step size.
        auto it = sv->queue.begin();
        for (; it != sv->queue.end(); ++it) {
          Beam* b = sv->beams[it->beam].get();
          if (b->group >= 0 ? !sv->groups[b->group]->busy : !b->busy) break;
        }
        if (it != sv->queue.end()) {
          Beam* b = sv->beams[it->beam].get();
          if (b->group < 0) {
            reqs.push_back(std::move(*it));
            sv->queue.erase(it);
            solo = b;
            b->busy = true;
          } else {
            g = sv->groups[b->group].get();
            g->busy = true;
            for (auto q = sv->queue.begin(); q != sv->queue.end() && (int)reqs.size() < g->step;) {
              if (sv->beams[q->beam]->group == b->group) {
                reqs.push_back(std::move(*q));
                q = sv->queue.erase(q);
              } else {
                ++q;
              }
            }
          }
          break;
        }
        sv->cv_work.wait(lk);
      }
    }
    std::vector<Result> res;
    if (solo) {
      res.resize(1);
      res[0].beam = solo->id;
      res[0].status = serve_one(solo, reqs[0], res[0]);
      if (res[0].status != FIP_OK) res[0].error = fip_last_error();
      solo->seen += 1;
    } else {
      serve_step(sv, g, reqs, res);
    }
    const auto now = Clock::now();
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      if (solo) solo->busy = false;
      if (g) {
        g->busy = false;
        sv->steps += 1;
        sv->stepped += (long)reqs.size();
      }
      for (size_t k = 0; k < reqs.size(); ++k) {
        res[k].latency_ms =
            std::chrono::duration<double, std::milli>(now - reqs[k].t_submit).count();
        sv->done[reqs[k].id] = std::move(res[k]);
      }
    }
    sv->cv_work.notify_all();
    sv->cv_done.notify_all();
  }
}

// Creates the group of configuration cfg with the largest step (<= the
// server's limit) whose memory fits in `room` bytes.  The caller holds no
// lock; the budget is re-checked by the caller.
int make_group(fip_server* sv, const fip_imager_config& cfg, size_t room,
               std::unique_ptr<Group>& out) {
  auto g = std::make_unique<Group>();
  g->cfg = cfg;
  g->n2 = cfg.image_size * cfg.image_size;
  g->uu = (cfg.image_size / cfg.unit_size) * (cfg.image_size / cfg.unit_size);
  g->nb = cfg.max_baselines;
  int st = FIP_ERR_BUDGET;
  for (int step = sv->max_step; step >= 1; step /= 2) {
    fip_batch* b = nullptr;
    const int cs = fip_batch_create(&b, &cfg, (size_t)step);
    if (cs == FIP_ERR_NOMEM) continue;
    if (cs != FIP_OK) return cs;
    const size_t per_img = (g->n2 + 64) * sizeof(float);
    const size_t bytes = fip_batch_device_bytes(b) + (size_t)step * per_img +
                         (size_t)step * (g->stride() + g->uu) * sizeof(float);
    if (bytes <= room) {
      g->batch = b;
      g->step = step;
      g->bytes = bytes;
      st = FIP_OK;
      break;
    }
    fip_batch_destroy(b);
  }
  if (st != FIP_OK)
    return fip_set_error(FIP_ERR_BUDGET, "a batch engine for this beam's configuration does "
                                         "not fit in the server's HBM budget");
  cudaError_t e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&g->d_in, g->step * g->stride() * sizeof(float));
  if (e == cudaSuccess) e = cudaMallocHost(&g->h_in, g->step * g->stride() * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&g->d_res, g->step * g->uu * sizeof(float));
  if (e == cudaSuccess) e = cudaMallocHost(&g->h_res, g->step * g->uu * sizeof(float));
  if (e == cudaSuccess) e = grow_pool(g.get(), g->step);
  if (e != cudaSuccess) {
    free_group(g.get());
    return cuda_fail(e);
  }
  out = std::move(g);
  return FIP_OK;
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

int fip_server_set_max_step(fip_server* sv, int snapshots) {
  if (!sv) return fip_set_error(FIP_ERR_ARG, "null server");
  if (snapshots < 1 || snapshots > FIP_MAX_BATCH)
    return fip_set_error(FIP_ERR_ARG, "the step size must be in [1, 64]");
  std::lock_guard<std::mutex> lk(sv->mu);
  if (!sv->beams.empty())
    return fip_set_error(FIP_ERR_STATE, "set the step size before adding beams");
  sv->max_step = snapshots;
  return FIP_OK;
}

int fip_server_stats(fip_server* sv, long* steps, long* snapshots) {
  if (!sv) return fip_set_error(FIP_ERR_ARG, "null server");
  std::lock_guard<std::mutex> lk(sv->mu);
  if (steps) *steps = sv->steps;
  if (snapshots) *snapshots = sv->stepped;
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
  for (auto& g : sv->groups) free_group(g.get());
  cudaSetDevice(prev);
  delete sv;
  return FIP_OK;
}

int fip_server_add_beam(fip_server* sv, const fip_imager_config* cfg, int* beam_id) {
  if (!sv || !cfg || !beam_id) return fip_set_error(FIP_ERR_ARG, "null argument");
  if (cfg->unit_size == 0) return fip_set_error(FIP_ERR_ARG, "a beam needs a trigger tile");
  if (cfg->unit_size > cfg->image_size)
    return fip_set_error(FIP_ERR_ARG, "unit_size larger than image_size");
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(sv->device);
  struct Restore {
    int d;
    ~Restore() { cudaSetDevice(d); }
  } restore{prev};
  auto b = std::make_unique<Beam>();
  b->cfg = *cfg;
  b->cfg.device = sv->device;
  const size_t n2 = cfg->image_size * cfg->image_size, nb = cfg->max_baselines;
  const size_t uu = (cfg->image_size / cfg->unit_size) * (cfg->image_size / cfg->unit_size);
  if (batchable(b->cfg)) {
    // Join (or create) the group of this configuration; the beam's own share
    // is its two resident images.
    std::unique_lock<std::mutex> lk(sv->mu);
    int gi = -1;
    for (size_t k = 0; k < sv->groups.size(); ++k)
      if (same_cfg(sv->groups[k]->cfg, b->cfg)) gi = (int)k;
    const size_t ring_bytes = 2 * (n2 + 64) * sizeof(float);
    if (gi < 0) {
      if (sv->reserved + ring_bytes > sv->budget) {
        return fip_set_error(FIP_ERR_BUDGET, "beam does not fit in the server's HBM budget");
      }
      const size_t room = sv->budget - sv->reserved - ring_bytes;
      sv->reserved += ring_bytes;  // held while the group is built
      lk.unlock();
      std::unique_ptr<Group> g;
      const int st = make_group(sv, b->cfg, room, g);
      lk.lock();
      if (st != FIP_OK || sv->reserved + g->bytes > sv->budget) {
        sv->reserved -= ring_bytes;
        if (st == FIP_OK) {
          free_group(g.get());
          return fip_set_error(FIP_ERR_BUDGET, "beam does not fit in the server's HBM budget");
        }
        return st;
      }
      sv->reserved += g->bytes;
      gi = (int)sv->groups.size();
      sv->groups.push_back(std::move(g));
    } else {
      if (sv->reserved + ring_bytes > sv->budget)
        return fip_set_error(FIP_ERR_BUDGET, "beam does not fit in the server's HBM budget (" +
                                                 std::to_string(sv->reserved + ring_bytes) +
                                                 " > " + std::to_string(sv->budget) + " bytes)");
      sv->reserved += ring_bytes;
    }
    Group* g = sv->groups[gi].get();
    const cudaError_t e = grow_pool(g, 2);
    if (e != cudaSuccess) {
      sv->reserved -= ring_bytes;
      return cuda_fail(e);
    }
    b->group = gi;
    b->bytes = ring_bytes;
    b->id = (int)sv->beams.size();
    *beam_id = b->id;
    sv->beams.push_back(std::move(b));
    return FIP_OK;
  }
  int st = fip_imager_create(&b->im, &b->cfg);
  if (st == FIP_OK) {
    b->bytes = fip_imager_device_bytes(b->im) + (3 * n2 + uu + 6 + 4 * nb + 9) * sizeof(float);
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
    if (e == cudaSuccess) e = cudaMalloc(&b->d_max, 6 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_res, uu * sizeof(float));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_vr, nb * sizeof(float));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_vi, nb * sizeof(float));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_B, 2 * nb * sizeof(float));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_V, 9 * sizeof(float));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_res, uu * sizeof(float));
    if (e != cudaSuccess) {
      st = cuda_fail(e);
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->reserved -= b->bytes;
    }
  }
  if (st != FIP_OK) {
    free_beam(b.get());
    return st;
  }
  std::lock_guard<std::mutex> lk(sv->mu);
  b->id = (int)sv->beams.size();
  *beam_id = b->id;
  sv->beams.push_back(std::move(b));
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
