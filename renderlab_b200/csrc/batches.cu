// Many-batch launches (rt_trace_batches) and prepared plans (rt_plan_*): uneven ray batches of
// one scene, mixed closest / any hit, traced by one persistent launch whose lanes take rays from
// the concatenation of the batches.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "ctx.hpp"

using namespace rtc;

namespace {

constexpr uint64_t MAX_LAUNCH_RAYS = 1ull << 31;  // the ray counter's headroom stays below 2^32

// Checks the batches and fills the device-format table; total receives the launch's rays and
// uniform the shared mode of its non-empty batches (0 closest, 1 any hit, -1 mixed).
rt_status make_table(rt_ctx* ctx, const rt_scene* scene, rt_kernel kernel, const rt_batch* b, uint32_t n,
                     rtk::BatchEntry* table, uint64_t& total, int& uniform) {
  if (!scene) return fail(ctx, RT_ERR_INVALID_ARG, "null scene");
  const bool wide = kernel == RT_KERNEL_WIDE8 || kernel == RT_KERNEL_WIDE8_PACKET;
  if (kernel != RT_KERNEL_PLAIN && kernel != RT_KERNEL_FAST && !wide)
    return fail(ctx, RT_ERR_UNSUPPORTED, "kernel %d is not available", (int)kernel);
  if (scene->layout == RT_LAYOUT_REFLECTION_BVH2 && kernel != RT_KERNEL_PLAIN)
    return fail(ctx, RT_ERR_UNSUPPORTED, "the legacy BVH2 layout is traced by the PLAIN kernel");
  if (wide && !scene->d_wide8)
    return fail(ctx, RT_ERR_UNSUPPORTED, "the WIDE8 kernel needs rt_scene_prepare(scene, RT_KERNEL_WIDE8) first");
  if (n && !b) return fail(ctx, RT_ERR_INVALID_ARG, "null batch array");
  if (n > RT_MAX_BATCHES) return fail(ctx, RT_ERR_INVALID_ARG, "%u batches (at most %u)", n, RT_MAX_BATCHES);
  total = 0;
  uniform = -2;  // no non-empty batch yet
  for (uint32_t i = 0; i < n; ++i) {
    if ((unsigned)b[i].mode > 2u) return fail(ctx, RT_ERR_INVALID_ARG, "batch %u: unknown mode %d", i, (int)b[i].mode);
    if (b[i].n) {
      if (!b[i].d_rays || !b[i].d_hits) return fail(ctx, RT_ERR_INVALID_ARG, "batch %u: null ray or hit buffer", i);
      if (reinterpret_cast<uintptr_t>(b[i].d_rays) % 16 != 0)
        return fail(ctx, RT_ERR_INVALID_ARG, "batch %u: rays must be 16-byte aligned", i);
      if (reinterpret_cast<uintptr_t>(b[i].d_hits) % 4 != 0)
        return fail(ctx, RT_ERR_INVALID_ARG, "batch %u: hits must be 4-byte aligned", i);
    }
    table[i].rays = reinterpret_cast<const float4*>(b[i].d_rays);
    table[i].hits = b[i].d_hits;
    table[i].first = static_cast<uint32_t>(total);
    table[i].n = b[i].n;
    table[i].mode = static_cast<uint32_t>(b[i].mode);
    table[i].pad = 0;
    total += b[i].n;
    if (total > MAX_LAUNCH_RAYS) return fail(ctx, RT_ERR_INVALID_ARG, "more than 2^31 rays in one launch");
    if (b[i].n) {
      const int m = b[i].mode != RT_CLOSEST ? 1 : 0;
      uniform = uniform == -2 ? m : (uniform == m ? m : -1);
    }
  }
  if (uniform == -2) uniform = 0;
  return RT_OK;
}

// The PLAIN kernel has no ray queue: one launch per non-empty batch, from the host table.
cudaError_t enqueue_plain(const rt_scene* scene, const rtk::BatchEntry* h_table, uint32_t entries, rtk::DevStatus* st,
                          cudaStream_t s) {
  const rtl::SceneView v = view_of(scene);
  for (uint32_t i = 0; i < entries; ++i) {
    if (!h_table[i].n) continue;
    cudaError_t e = rtl::launch_plain(v, h_table[i].mode, h_table[i].rays, h_table[i].hits, h_table[i].n, st, s);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t enqueue(const rt_scene* scene, rt_kernel kernel, const rtk::BatchEntry* d_table, uint32_t entries,
                    uint32_t total, const uint32_t* order, unsigned int* counter, rtk::DevStatus* st, cudaStream_t s,
                    uint32_t refill, int uniform, uint32_t stack) {
  const rtl::SceneView v = view_of(scene);
  if (kernel == RT_KERNEL_WIDE8)
    return rtl::launch_wide8_batches(v, d_table, entries, total, order, counter, st, s, refill, uniform,
                                     stack == RT_STACK_SHARED ? 1u : 0u);
  if (kernel == RT_KERNEL_WIDE8_PACKET)
    return rtl::launch_wide8_packet_batches(v, d_table, entries, total, order, counter, st, s, uniform);
  return rtl::launch_fast_batches(v, d_table, entries, total, order, counter, st, s, refill, uniform);
}

void world_box(const rt_scene* scene, float lo[3], float hi[3]) {
  const rtb::Aabb& wb = scene->info.world;
  for (int a = 0; a < 3; ++a) {
    lo[a] = std::isfinite(wb.lo[a]) ? wb.lo[a] : -1.0f;
    hi[a] = std::isfinite(wb.hi[a]) ? wb.hi[a] : 1.0f;
  }
}

}  // namespace

rt_status rt_trace_batches(rt_ctx* ctx, const rt_scene* scene, rt_kernel kernel, const rt_batch* h_batches,
                           uint32_t n_batches, void* stream) {
  if (!ctx) return RT_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lock(ctx->mu);
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  if (!ctx->h_tables) {
    const size_t bytes = sizeof(rtk::BatchEntry) * RT_MAX_BATCHES * rt_ctx::TABLE_SLOTS;
    if (cudaMallocHost(&ctx->h_tables, bytes) != cudaSuccess || cudaMalloc(&ctx->d_tables, bytes) != cudaSuccess) {
      cudaGetLastError();
      cudaFreeHost(ctx->h_tables);
      ctx->h_tables = nullptr;
      return fail(ctx, RT_ERR_OOM, "batch table staging (%zu bytes)", bytes);
    }
    for (cudaEvent_t& e : ctx->table_done) RT_CUDA(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  const uint32_t slot = ctx->table_seq++ % rt_ctx::TABLE_SLOTS;
  RT_CUDA(ctx, cudaEventSynchronize(ctx->table_done[slot]));  // the slot's last copy has been read
  rtk::BatchEntry* h = ctx->h_tables + (size_t)slot * RT_MAX_BATCHES;
  rtk::BatchEntry* d = ctx->d_tables + (size_t)slot * RT_MAX_BATCHES;
  uint64_t total = 0;
  int uniform = -1;
  rt_status st = make_table(ctx, scene, kernel, h_batches, n_batches, h, total, uniform);
  if (st != RT_OK || total == 0) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (kernel == RT_KERNEL_PLAIN) {
    cudaError_t e = enqueue_plain(scene, h, n_batches, ctx->d_status, s);
    if (e != cudaSuccess) return fail(ctx, RT_ERR_CUDA, "plain batch launch: %s", cudaGetErrorString(e));
    ctx->rays += total;
    ctx->launches += n_batches;
    return RT_OK;
  }
  RT_CUDA(ctx, cudaMemcpyAsync(d, h, sizeof(rtk::BatchEntry) * n_batches, cudaMemcpyHostToDevice, s));
  RT_CUDA(ctx, cudaEventRecord(ctx->table_done[slot], s));
  const uint32_t refill = kernel == RT_KERNEL_FAST ? ctx->tuning.fast_refill : ctx->tuning.wide8_refill;
  if (kernel == RT_KERNEL_WIDE8 && ctx->tuning.wide8_stack == RT_STACK_SHARED && !rtl::shared_stack_fits(view_of(scene)))
    return fail(ctx, RT_ERR_UNSUPPORTED, "the shared group stack holds 16 levels; this scene's 8-wide trees have %u",
                scene->w8_depth);
  cudaError_t e = enqueue(scene, kernel, d, n_batches, (uint32_t)total, nullptr,
                          ctx->d_counters + (ctx->counter_seq++ % COUNTER_SLOTS), ctx->d_status, s, refill, uniform,
                          ctx->tuning.wide8_stack);
  if (e != cudaSuccess) return fail(ctx, RT_ERR_CUDA, "many-batch launch: %s", cudaGetErrorString(e));
  ctx->rays += total;
  ctx->launches += 1;
  return RT_OK;
}

struct rt_plan {
  rt_ctx* ctx = nullptr;
  const rt_scene* scene = nullptr;
  rt_plan_desc desc{};
  uint32_t entries = 0, total = 0, refill = 8, stack = RT_STACK_LOCAL;
  int uniform = -1;
  rtk::BatchEntry* d_table = nullptr;
  unsigned int* d_counter = nullptr;
  uint32_t* d_order = nullptr;
  void* d_sort = nullptr;
  size_t sort_bytes = 0;
  size_t device_bytes = 0;
  float lo[3] = {}, hi[3] = {};
  std::vector<rtk::BatchEntry> h_table;  // the PLAIN kernel's launches read it
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

cudaError_t plan_enqueue(const rt_plan* p, cudaStream_t s) {
  if (p->total == 0) return cudaSuccess;
  if (p->desc.kernel == RT_KERNEL_PLAIN) return enqueue_plain(p->scene, p->h_table.data(), p->entries, p->ctx->d_status, s);
  if (p->d_order) {
    cudaError_t e = rtl::launch_order_batches(p->d_table, p->entries, p->total, p->lo, p->hi, (uint32_t)p->desc.order,
                                              p->d_order, p->d_sort, p->sort_bytes, s);
    if (e != cudaSuccess) return e;
  }
  return enqueue(p->scene, p->desc.kernel, p->d_table, p->entries, p->total, p->d_order, p->d_counter,
                 p->ctx->d_status, s, p->refill, p->uniform, p->stack);
}

void plan_free(rt_plan* p) {
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  cudaFree(p->d_table);
  cudaFree(p->d_counter);
  cudaFree(p->d_order);
  cudaFree(p->d_sort);
  delete p;
}

}  // namespace

rt_status rt_plan_create(rt_ctx* ctx, const rt_scene* scene, const rt_batch* h_batches, uint32_t n_batches,
                         const rt_plan_desc* desc, rt_plan** out) {
  if (!ctx || !desc || !out) return fail(ctx, RT_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  if ((unsigned)desc->order > 3u) return fail(ctx, RT_ERR_INVALID_ARG, "unknown ray order %d", (int)desc->order);
  if (desc->refill > 32) return fail(ctx, RT_ERR_INVALID_ARG, "refill thresholds are 1-32 lanes");
  if (desc->kernel == RT_KERNEL_PLAIN && desc->order != RT_ORDER_NONE)
    return fail(ctx, RT_ERR_UNSUPPORTED, "the PLAIN kernel takes no ray order");
  if (desc->stack > RT_STACK_SHARED) return fail(ctx, RT_ERR_INVALID_ARG, "unknown stack placement %u", desc->stack);
  std::vector<rtk::BatchEntry> table(n_batches ? n_batches : 1);
  uint64_t total = 0;
  int uniform = -1;
  rt_status st = make_table(ctx, scene, desc->kernel, h_batches, n_batches, table.data(), total, uniform);
  if (st != RT_OK) return st;
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  rt_plan* p = new rt_plan;
  p->ctx = ctx;
  p->scene = scene;
  p->desc = *desc;
  p->entries = n_batches;
  p->total = (uint32_t)total;
  p->uniform = uniform;
  p->h_table = table;
  p->refill = desc->refill ? desc->refill
                           : (desc->kernel == RT_KERNEL_FAST ? ctx->tuning.fast_refill : ctx->tuning.wide8_refill);
  p->stack = desc->stack ? desc->stack : ctx->tuning.wide8_stack;
  if (desc->kernel == RT_KERNEL_WIDE8 && p->stack == RT_STACK_SHARED && !rtl::shared_stack_fits(view_of(scene))) {
    const uint32_t depth = scene->w8_depth;
    delete p;
    return fail(ctx, RT_ERR_UNSUPPORTED, "the shared group stack holds 16 levels; this scene's 8-wide trees have %u",
                depth);
  }
  world_box(scene, p->lo, p->hi);
  auto oom = [&](const char* what, size_t bytes) {
    cudaGetLastError();
    plan_free(p);
    return fail(ctx, RT_ERR_OOM, "plan %s (%zu bytes)", what, bytes);
  };
  const size_t table_bytes = sizeof(rtk::BatchEntry) * table.size();
  if (cudaMalloc(&p->d_table, table_bytes) != cudaSuccess) return oom("batch table", table_bytes);
  if (cudaMalloc(&p->d_counter, 256) != cudaSuccess) return oom("ray counter", 256);
  p->device_bytes = table_bytes + 256;
  if (desc->order != RT_ORDER_NONE && total > 0) {
    p->sort_bytes = rtl::order_scratch_bytes(p->total);
    if (cudaMalloc(&p->d_order, sizeof(uint32_t) * total) != cudaSuccess) return oom("ray order", 4 * total);
    if (cudaMalloc(&p->d_sort, p->sort_bytes) != cudaSuccess) return oom("sort scratch", p->sort_bytes);
    p->device_bytes += sizeof(uint32_t) * total + p->sort_bytes;
  }
  cudaError_t e = cudaMemcpy(p->d_table, table.data(), table_bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && desc->graph) {
    cudaStream_t cs = nullptr;
    e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
      e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        cudaError_t le = plan_enqueue(p, cs);
        e = cudaStreamEndCapture(cs, &p->graph);
        if (le != cudaSuccess) e = le;
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&p->exec, p->graph, 0);
      cudaStreamDestroy(cs);
    }
  }
  if (e != cudaSuccess) {
    plan_free(p);
    return fail(ctx, RT_ERR_CUDA, "plan: %s", cudaGetErrorString(e));
  }
  *out = p;
  return RT_OK;
}

rt_status rt_plan_launch(rt_plan* p, void* stream) {
  if (!p) return RT_ERR_INVALID_ARG;
  rt_ctx* ctx = p->ctx;
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (p->exec) {
    RT_CUDA(ctx, cudaGraphLaunch(p->exec, s));
  } else {
    cudaError_t e = plan_enqueue(p, s);
    if (e != cudaSuccess) return fail(ctx, RT_ERR_CUDA, "plan launch: %s", cudaGetErrorString(e));
  }
  ctx->rays += p->total;
  ctx->launches += 1;
  return RT_OK;
}

rt_status rt_plan_info(const rt_plan* p, uint64_t* rays, uint64_t* device_bytes) {
  if (!p) return RT_ERR_INVALID_ARG;
  if (rays) *rays = p->total;
  if (device_bytes) *device_bytes = p->device_bytes;
  return RT_OK;
}

rt_status rt_plan_destroy(rt_plan* p) {
  if (!p) return RT_OK;
  cudaSetDevice(p->ctx->device);
  plan_free(p);
  return RT_OK;
}
