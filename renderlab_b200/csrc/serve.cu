// The serving loop (rt_server_*): ray-batch requests of any size, for several device-resident
// scenes, arriving at any time from any thread; results written back to the caller's host
// buffers; per-request latency recorded.
//
// * Admission by HBM budget: a scene is admitted only while the resident scenes plus the
//   launch slots fit the budget; requests are admitted to the device chunk by chunk, as launch
//   slots (fixed device ray / hit buffers) free up.
// * Continuous batching: a worker thread fills every free slot with chunks taken in arrival
//   order from the pending requests of one scene -- several requests share a slot, a large
//   request spreads over several slots -- and traces the slot with one many-batch launch
//   (rt_trace_batches: mixed closest / any hit). Each slot has its own stream, so one slot's
//   copies overlap another's traversal, and requests that arrive while slots are busy join the
//   next free one.
// * A ray's result does not depend on which slot, launch or neighbours it gets: the traversal
//   kernels compute every ray alone. So each request's results equal those of the same rays
//   traced alone with the same kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "ctx.hpp"

using namespace rtc;

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t ticket = 0;
  uint32_t scene = 0;
  rt_mode mode = RT_CLOSEST;
  const rt_ray* h_rays = nullptr;
  uint8_t* h_hits = nullptr;
  uint32_t n = 0;
  uint32_t handed = 0;  // rays given to slots
  uint32_t done = 0;    // rays whose results are back
  size_t hit_bytes = 0;
  rt_status status = RT_OK;
  bool finished = false;
  Clock::time_point submitted;
};

struct Chunk {
  Request* req;
  uint32_t first, n;
  size_t ray_off, hit_off;  // in the slot's buffers (elements, bytes)
};

struct SceneEntry {
  rt_scene* scene = nullptr;
  size_t bytes = 0;
  uint32_t layout = 0;
  uint32_t live = 0;  // requests not yet finished
};

}  // namespace

struct rt_server;

namespace {
struct Slot {
  rt_server* srv = nullptr;
  uint32_t id = 0;
  cudaStream_t stream = nullptr;
  rt_ray* d_rays = nullptr;
  uint8_t* d_hits = nullptr;
  uint32_t scene = 0;
  std::vector<Chunk> chunks;
  rt_status status = RT_OK;
};
}  // namespace

struct rt_server {
  rt_ctx* ctx = nullptr;
  rt_server_desc desc{};
  size_t slot_bytes = 0;
  std::vector<SceneEntry> scenes;
  std::deque<Request*> pending;  // arrival order; requests with rays not yet handed out
  std::unordered_map<uint64_t, Request*> requests;
  std::vector<Slot> slots;
  std::vector<uint32_t> free_slots;
  std::deque<uint32_t> completed;  // slots whose launch finished (host callbacks)
  std::mutex mu;
  std::condition_variable wake, finished;
  std::thread worker;
  bool stop = false;
  uint64_t next_ticket = 1;
  // rt_server_fail_next: slot launches still to fail on the host, and the status they fail with
  uint32_t fail_launches = 0;
  rt_status fail_status = RT_OK;
  // statistics since the last reset
  std::vector<double> latency_ms;
  uint64_t rays = 0, launches = 0, requests_done = 0;
  Clock::time_point since = Clock::now();
};

namespace {

void CUDART_CB slot_done(void* p) {
  Slot* s = static_cast<Slot*>(p);
  rt_server* srv = s->srv;
  {
    std::lock_guard<std::mutex> lock(srv->mu);
    srv->completed.push_back(s->id);
  }
  srv->wake.notify_one();
}

void finish(rt_server* srv, Request* r, rt_status st) {
  if (r->finished) return;
  if (st != RT_OK) r->status = st;
  r->finished = true;
  srv->scenes[r->scene].live -= 1;
  const double ms = std::chrono::duration<double, std::milli>(Clock::now() - r->submitted).count();
  srv->latency_ms.push_back(ms);
  srv->requests_done += 1;
  srv->finished.notify_all();
}

// Retires a finished slot (lock held): its chunks' rays are done.
void retire(rt_server* srv, Slot& s) {
  for (Chunk& c : s.chunks) {
    Request* r = c.req;
    if (s.status != RT_OK) r->status = s.status;
    r->done += c.n;
    if (r->done == r->n) finish(srv, r, RT_OK);
  }
  s.chunks.clear();
  s.status = RT_OK;
  srv->free_slots.push_back(s.id);
}

// Fills slot s with chunks of the oldest pending request's scene (lock held).
void fill(rt_server* srv, Slot& s) {
  const uint32_t scene = srv->pending.front()->scene;
  const uint32_t cap = srv->desc.launch_rays;
  uint32_t used = 0;
  size_t hit_off = 0;
  s.scene = scene;
  for (auto it = srv->pending.begin(); it != srv->pending.end() && used < cap && s.chunks.size() < RT_MAX_BATCHES;) {
    Request* r = *it;
    if (r->scene != scene) {
      ++it;
      continue;
    }
    const uint32_t take = std::min(r->n - r->handed, cap - used);
    s.chunks.push_back(Chunk{r, r->handed, take, used, hit_off});
    r->handed += take;
    used += take;
    hit_off += ((size_t)take * r->hit_bytes + 15) & ~(size_t)15;
    if (r->handed == r->n) it = srv->pending.erase(it);
    else ++it;
  }
}

// Enqueues a filled slot: rays in, one many-batch launch, hits out, completion callback.
rt_status launch(rt_server* srv, Slot& s) {
  rt_ctx* ctx = srv->ctx;
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  std::vector<rt_batch> batches;
  batches.reserve(s.chunks.size());
  for (const Chunk& c : s.chunks) {
    RT_CUDA(ctx, cudaMemcpyAsync(s.d_rays + c.ray_off, c.req->h_rays + c.first, (size_t)c.n * sizeof(rt_ray),
                                 cudaMemcpyHostToDevice, s.stream));
    batches.push_back(rt_batch{s.d_rays + c.ray_off, s.d_hits + c.hit_off, c.n, c.req->mode});
  }
  rt_status st = rt_trace_batches(ctx, srv->scenes[s.scene].scene, srv->desc.kernel, batches.data(),
                                  (uint32_t)batches.size(), s.stream);
  if (st != RT_OK) return st;
  for (const Chunk& c : s.chunks)
    RT_CUDA(ctx, cudaMemcpyAsync(c.req->h_hits + (size_t)c.first * c.req->hit_bytes, s.d_hits + c.hit_off,
                                 (size_t)c.n * c.req->hit_bytes, cudaMemcpyDeviceToHost, s.stream));
  RT_CUDA(ctx, cudaLaunchHostFunc(s.stream, slot_done, &s));
  return RT_OK;
}

void work(rt_server* srv) {
  std::unique_lock<std::mutex> lock(srv->mu);
  for (;;) {
    while (!srv->completed.empty()) {
      const uint32_t id = srv->completed.front();
      srv->completed.pop_front();
      retire(srv, srv->slots[id]);
    }
    while (!srv->free_slots.empty() && !srv->pending.empty()) {
      Slot& s = srv->slots[srv->free_slots.back()];
      srv->free_slots.pop_back();
      fill(srv, s);
      uint32_t rays = 0;
      for (const Chunk& c : s.chunks) rays += c.n;
      rt_status injected = RT_OK;
      if (srv->fail_launches) {  // a fake of a failing enqueue: nothing of this slot is enqueued
        srv->fail_launches -= 1;
        injected = srv->fail_status;
      }
      lock.unlock();  // copies from pageable memory block; new requests may arrive meanwhile
      const rt_status st = injected != RT_OK ? injected : launch(srv, s);
      lock.lock();
      if (st != RT_OK) {  // nothing of this slot is in flight after a failed enqueue
        cudaStreamSynchronize(s.stream);
        s.status = st;
        retire(srv, s);
        continue;
      }
      srv->rays += rays;
      srv->launches += 1;
    }
    const bool idle = srv->free_slots.size() == srv->slots.size();
    if (srv->stop && srv->pending.empty() && idle) break;
    srv->wake.wait(lock, [&] {
      return !srv->completed.empty() || (!srv->pending.empty() && !srv->free_slots.empty()) ||
             (srv->stop && srv->pending.empty() && srv->free_slots.size() == srv->slots.size());
    });
  }
}

void free_slots(rt_server* srv) {
  for (Slot& s : srv->slots) {
    if (s.stream) cudaStreamDestroy(s.stream);
    cudaFree(s.d_rays);
    cudaFree(s.d_hits);
  }
  srv->slots.clear();
}

size_t resident_bytes(const rt_server* srv) {
  size_t b = srv->slot_bytes * srv->slots.size();
  for (const SceneEntry& e : srv->scenes) b += e.scene ? e.bytes : 0;
  return b;
}

}  // namespace

rt_status rt_server_create(rt_ctx* ctx, const rt_server_desc* desc, rt_server** out) {
  if (!ctx || !desc || !out) return fail(ctx, RT_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  if ((unsigned)desc->kernel > (unsigned)RT_KERNEL_WIDE8_PACKET)
    return fail(ctx, RT_ERR_INVALID_ARG, "unknown kernel %d", (int)desc->kernel);
  if (desc->slots == 0 || desc->slots > 64) return fail(ctx, RT_ERR_INVALID_ARG, "slots must be 1-64");
  if (desc->launch_rays == 0 || desc->launch_rays > (1u << 26))
    return fail(ctx, RT_ERR_INVALID_ARG, "launch_rays must be 1-2^26");
  rt_server* srv = new rt_server;
  srv->ctx = ctx;
  srv->desc = *desc;
  // hits of every mode fit 40 bytes a ray; each chunk's hit region is 16-byte aligned
  srv->slot_bytes = (size_t)desc->launch_rays * (sizeof(rt_ray) + GI_HIT_BYTES) + 16 * RT_MAX_BATCHES;
  if (srv->slot_bytes * desc->slots > desc->hbm_budget) {
    delete srv;
    return fail(ctx, RT_ERR_OOM, "the launch slots alone (%zu bytes) exceed the HBM budget", srv->slot_bytes * desc->slots);
  }
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  srv->slots.resize(desc->slots);
  for (uint32_t i = 0; i < desc->slots; ++i) {
    Slot& s = srv->slots[i];
    s.srv = srv;
    s.id = i;
    const size_t hit_bytes = srv->slot_bytes - (size_t)desc->launch_rays * sizeof(rt_ray);
    if (cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&s.d_rays, (size_t)desc->launch_rays * sizeof(rt_ray)) != cudaSuccess ||
        cudaMalloc(&s.d_hits, hit_bytes) != cudaSuccess) {
      cudaGetLastError();
      free_slots(srv);
      delete srv;
      return fail(ctx, RT_ERR_OOM, "launch slot %u", i);
    }
    srv->free_slots.push_back(desc->slots - 1 - i);
  }
  srv->worker = std::thread(work, srv);
  *out = srv;
  return RT_OK;
}

rt_status rt_server_add_scene(rt_server* srv, rt_layout layout, const uint32_t* words, size_t n_words, uint32_t* id) {
  if (!srv || !id) return RT_ERR_INVALID_ARG;
  rt_ctx* ctx = srv->ctx;
  if (layout == RT_LAYOUT_REFLECTION_BVH2 && srv->desc.kernel != RT_KERNEL_PLAIN)
    return fail(ctx, RT_ERR_UNSUPPORTED, "the legacy BVH2 layout is served by a PLAIN-kernel server");
  rt_scene* scene = nullptr;
  rt_status st = rt_scene_upload(ctx, layout, words, n_words, &scene);
  if (st != RT_OK) return st;
  // WIDE8: the derived layout, and the top level's entries per instance measured for this scene
  if (srv->desc.kernel >= RT_KERNEL_WIDE8 &&
      ((st = rt_scene_prepare(ctx, scene, RT_KERNEL_WIDE8)) != RT_OK ||
       (st = rt_scene_tune_top(ctx, scene, nullptr, 0, 0, nullptr)) != RT_OK)) {
    rt_scene_release(ctx, scene);
    return st;
  }
  std::lock_guard<std::mutex> lock(srv->mu);
  const size_t bytes = rt_scene_device_bytes(scene);
  if (resident_bytes(srv) + bytes > srv->desc.hbm_budget) {
    const size_t have = resident_bytes(srv);
    rt_scene_release(ctx, scene);
    return fail(ctx, RT_ERR_OOM, "scene of %zu device bytes refused: %zu of the %llu-byte HBM budget in use", bytes,
                have, (unsigned long long)srv->desc.hbm_budget);
  }
  srv->scenes.push_back(SceneEntry{scene, bytes, (uint32_t)layout, 0});
  *id = (uint32_t)srv->scenes.size() - 1;
  return RT_OK;
}

rt_status rt_server_remove_scene(rt_server* srv, uint32_t id) {
  if (!srv) return RT_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lock(srv->mu);
  if (id >= srv->scenes.size() || !srv->scenes[id].scene) return fail(srv->ctx, RT_ERR_INVALID_ARG, "no scene %u", id);
  if (srv->scenes[id].live) return fail(srv->ctx, RT_ERR_BUSY, "scene %u has unfinished requests", id);
  rt_scene_release(srv->ctx, srv->scenes[id].scene);
  srv->scenes[id].scene = nullptr;
  return RT_OK;
}

rt_status rt_server_submit(rt_server* srv, uint32_t scene, rt_mode mode, const rt_ray* h_rays, uint32_t n, void* h_hits,
                           uint64_t* ticket) {
  if (!srv || !ticket) return RT_ERR_INVALID_ARG;
  if ((unsigned)mode > 2u) return fail(srv->ctx, RT_ERR_INVALID_ARG, "unknown mode %d", (int)mode);
  if (n && (!h_rays || !h_hits)) return fail(srv->ctx, RT_ERR_INVALID_ARG, "null ray or hit buffer");
  Request* r = new Request;
  r->mode = mode;
  r->h_rays = h_rays;
  r->h_hits = static_cast<uint8_t*>(h_hits);
  r->n = n;
  r->submitted = Clock::now();
  {
    std::lock_guard<std::mutex> lock(srv->mu);
    if (scene >= srv->scenes.size() || !srv->scenes[scene].scene) {
      delete r;
      return fail(srv->ctx, RT_ERR_INVALID_ARG, "no scene %u", scene);
    }
    if (srv->stop) {
      delete r;
      return fail(srv->ctx, RT_ERR_BUSY, "the server is shutting down");
    }
    r->scene = scene;
    r->hit_bytes = hit_bytes(srv->scenes[scene].layout, (uint32_t)mode);
    r->ticket = srv->next_ticket++;
    srv->requests[r->ticket] = r;
    srv->scenes[scene].live += 1;
    if (n == 0) finish(srv, r, RT_OK);
    else srv->pending.push_back(r);
    *ticket = r->ticket;
  }
  srv->wake.notify_one();
  return RT_OK;
}

rt_status rt_server_wait(rt_server* srv, uint64_t ticket, int32_t timeout_ms) {
  if (!srv) return RT_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> lock(srv->mu);
  auto it = srv->requests.find(ticket);
  if (it == srv->requests.end()) return fail(srv->ctx, RT_ERR_INVALID_ARG, "unknown ticket %llu", (unsigned long long)ticket);
  Request* r = it->second;
  auto done = [&] { return r->finished; };
  if (timeout_ms < 0) {
    srv->finished.wait(lock, done);
  } else if (!srv->finished.wait_for(lock, std::chrono::milliseconds(timeout_ms), done)) {
    return RT_ERR_TIMEOUT;  // still running: wait again later
  }
  const rt_status st = r->status;
  srv->requests.erase(it);
  delete r;
  return st;
}

rt_status rt_server_fail_next(rt_server* srv, uint32_t launches, rt_status status) {
  if (!srv || (launches && status == RT_OK)) return RT_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lock(srv->mu);
  srv->fail_launches = launches;
  srv->fail_status = status;
  return RT_OK;
}

rt_status rt_server_get_stats(rt_server* srv, rt_server_stats* out, int reset) {
  if (!srv || !out) return RT_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lock(srv->mu);
  std::vector<double> l = srv->latency_ms;
  std::sort(l.begin(), l.end());
  auto pct = [&](double q) { return l.empty() ? 0.0 : l[std::min(l.size() - 1, (size_t)(q * (double)(l.size() - 1) + 0.5))]; };
  out->requests = srv->requests_done;
  out->rays = srv->rays;
  out->launches = srv->launches;
  out->p50_ms = pct(0.50);
  out->p99_ms = pct(0.99);
  out->max_ms = l.empty() ? 0.0 : l.back();
  out->wall_s = std::chrono::duration<double>(Clock::now() - srv->since).count();
  out->device_bytes = resident_bytes(srv);
  out->pending = srv->pending.size();
  if (reset) {
    srv->latency_ms.clear();
    srv->rays = srv->launches = srv->requests_done = 0;
    srv->since = Clock::now();
  }
  return RT_OK;
}

rt_status rt_server_destroy(rt_server* srv) {
  if (!srv) return RT_OK;
  {
    std::lock_guard<std::mutex> lock(srv->mu);
    srv->stop = true;
  }
  srv->wake.notify_one();
  srv->worker.join();  // every admitted request finishes first
  cudaSetDevice(srv->ctx->device);
  free_slots(srv);
  for (SceneEntry& e : srv->scenes)
    if (e.scene) rt_scene_release(srv->ctx, e.scene);
  for (auto& kv : srv->requests) delete kv.second;
  delete srv;
  return RT_OK;
}
