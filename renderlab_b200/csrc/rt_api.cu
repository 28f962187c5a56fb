// The C ABI (include/rt_trace.h): contexts, scene upload, traversal dispatch, host builders.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/rt_trace.h"
#include "ctx.hpp"
#include "host/host.hpp"
#include "host/wide8.hpp"
#include "launch.hpp"

using namespace rtc;

namespace {

rt_status dispatch(rt_ctx* ctx, const rt_scene* scene, rt_mode mode, rt_kernel kernel, const rt_ray* rays,
                   const uint32_t* order, void* hits, uint32_t n, cudaStream_t stream) {
  const rtl::SceneView v = view_of(scene);
  const float4* r = reinterpret_cast<const float4*>(rays);
  cudaError_t e;
  switch (kernel) {
    case RT_KERNEL_PLAIN:
      if (order) return fail(ctx, RT_ERR_UNSUPPORTED, "the PLAIN kernel takes no ray order");
      e = rtl::launch_plain(v, (uint32_t)mode, r, hits, n, ctx->d_status, stream);
      break;
    case RT_KERNEL_FAST:
      e = rtl::launch_fast(v, (uint32_t)mode, r, order, hits, n,
                           ctx->d_counters + (ctx->counter_seq++ % COUNTER_SLOTS), ctx->d_status, stream,
                           ctx->tuning.fast_refill);
      break;
    case RT_KERNEL_WIDE8:
      if (!scene->d_wide8)
        return fail(ctx, RT_ERR_UNSUPPORTED, "the WIDE8 kernel needs rt_scene_prepare(scene, RT_KERNEL_WIDE8) first");
      if (ctx->tuning.wide8_stack == RT_STACK_SHARED && !rtl::shared_stack_fits(v))
        return fail(ctx, RT_ERR_UNSUPPORTED, "the shared group stack holds 16 levels; this scene's 8-wide trees have %u",
                    v.w8_depth);
      e = rtl::launch_wide8(v, (uint32_t)mode, r, order, hits, n,
                            ctx->d_counters + (ctx->counter_seq++ % COUNTER_SLOTS), ctx->d_status, stream,
                            ctx->tuning.wide8_refill, ctx->tuning.wide8_stack == RT_STACK_SHARED ? 1u : 0u);
      break;
    case RT_KERNEL_WIDE8_PACKET:
      if (!scene->d_wide8)
        return fail(ctx, RT_ERR_UNSUPPORTED, "the WIDE8 kernel needs rt_scene_prepare(scene, RT_KERNEL_WIDE8) first");
      e = rtl::launch_wide8_packet(v, (uint32_t)mode, r, order, hits, n,
                                   ctx->d_counters + (ctx->counter_seq++ % COUNTER_SLOTS), ctx->d_status, stream);
      break;
    default:
      return fail(ctx, RT_ERR_UNSUPPORTED, "kernel %d is not available", (int)kernel);
  }
  if (e != cudaSuccess) return fail(ctx, RT_ERR_CUDA, "traversal launch: %s", cudaGetErrorString(e));
  ctx->rays += n;
  ctx->launches += 1;
  return RT_OK;
}

rt_status check_trace_args(rt_ctx* ctx, const rt_scene* scene, rt_mode mode, rt_kernel kernel) {
  if (!ctx || !scene) return fail(ctx, RT_ERR_INVALID_ARG, "null context or scene");
  if ((unsigned)mode > 2u) return fail(ctx, RT_ERR_INVALID_ARG, "unknown mode %d", (int)mode);
  if (scene->layout == RT_LAYOUT_REFLECTION_BVH2 && kernel != RT_KERNEL_PLAIN)
    return fail(ctx, RT_ERR_UNSUPPORTED, "the legacy BVH2 layout is traced by the PLAIN kernel");
  if ((unsigned)kernel > 3u) return fail(ctx, RT_ERR_INVALID_ARG, "unknown kernel %d", (int)kernel);
  return RT_OK;
}

}  // namespace

namespace {

// Replaces the scene's 8-wide top level with these nodes and items (none: the walk uses the
// packed top level).
rt_status upload_top(rt_ctx* ctx, rt_scene* scene, const std::vector<uint32_t>& nodes, const std::vector<uint32_t>& items) {
  if (scene->d_w8_top) {
    cudaFree(scene->d_w8_top);
    scene->device_bytes -= scene->w8_top_bytes;
    ctx->scene_bytes -= scene->w8_top_bytes;
    scene->d_w8_top = nullptr, scene->w8_top_bytes = 0, scene->w8_top_nodes = 0;
  }
  scene->w8_top_valid = false;
  if (nodes.empty()) return RT_OK;
  const size_t items_at = nodes.size(), total = items_at + std::max<size_t>(items.size(), 1);
  void* d = nullptr;
  if (cudaMalloc(&d, total * 4) != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, RT_ERR_OOM, "device allocation of %zu bytes for the 8-wide top level failed", total * 4);
  }
  cudaError_t e = cudaMemcpy(d, nodes.data(), nodes.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !items.empty())
    e = cudaMemcpy(static_cast<uint32_t*>(d) + items_at, items.data(), items.size() * 4, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(d);
    return fail(ctx, RT_ERR_CUDA, "8-wide top-level upload: %s", cudaGetErrorString(e));
  }
  scene->d_w8_top = d;
  scene->w8_top_bytes = total * 4;
  scene->w8_top_items_at = items_at;
  scene->w8_top_nodes = (uint32_t)(nodes.size() / rtb::W8_NODE_WORDS);
  scene->w8_top_valid = true;
  scene->device_bytes += scene->w8_top_bytes;
  ctx->scene_bytes += scene->w8_top_bytes;
  return RT_OK;
}

// The top level's entries per instance for this scene: its tuned budget, else the context's.
uint32_t entries_of(const rt_ctx* ctx, const rt_scene* scene) {
  return scene->w8_entries ? scene->w8_entries : ctx->tuning.wide8_entries;
}

// Host copies of the scene's built 8-wide BLAS nodes and instance table (read back from the device).
rt_status read_wide8_blas(rt_ctx* ctx, const rt_scene* scene, uint32_t instances, rtb::Wide8Scene& top) {
  top.nodes.resize(scene->w8_tris_at - scene->w8_nodes_at);
  top.inst.resize(2 * (size_t)instances);
  const uint32_t* d = static_cast<const uint32_t*>(scene->d_wide8);
  RT_CUDA(ctx, cudaMemcpy(top.nodes.data(), d + scene->w8_nodes_at, top.nodes.size() * 4, cudaMemcpyDeviceToHost));
  if (!top.inst.empty())
    RT_CUDA(ctx, cudaMemcpy(top.inst.data(), d + scene->w8_inst_at, top.inst.size() * 4, cudaMemcpyDeviceToHost));
  return RT_OK;
}

// Builds and uploads the 8-wide top level with `entries` leaves per instance over `top`'s BLAS
// nodes and instance table (the packed top level when the build or its check fails).
rt_status rebuild_top(rt_ctx* ctx, rt_scene* scene, const std::vector<uint32_t>& words, rtb::Wide8Scene& top,
                      uint32_t entries) {
  std::string err;
  rtb::build_wide8_top_of(scene->layout, words.data(), top.nodes, top.inst, top.top_nodes, top.top_items, &top.top_depth,
                          entries);
  if (!rtb::check_wide8_top(scene->layout, words.data(), top, err)) top.top_nodes.clear();  // the packed top level
  return upload_top(ctx, scene, top.top_nodes, top.top_items);
}

// Rebuilds only the 8-wide top level, from the scene's current records and its built 8-wide
// BLAS nodes and instance table.
rt_status prepare_top(rt_ctx* ctx, rt_scene* scene, const std::vector<uint32_t>& words) {
  rtb::Wide8Scene top;
  rt_status s = read_wide8_blas(ctx, scene, words[0], top);
  if (s != RT_OK) return s;
  return rebuild_top(ctx, scene, words, top, entries_of(ctx, scene));
}

// Frees the scene's derived 8-wide layout (its BLASes, instance table and top level): WIDE8 then
// needs rt_scene_prepare again.
void drop_wide8(rt_ctx* ctx, rt_scene* scene) {
  if (!scene->d_wide8) return;
  cudaFree(scene->d_wide8);
  scene->d_wide8 = nullptr;
  scene->device_bytes -= scene->wide8_bytes;
  ctx->scene_bytes -= scene->wide8_bytes;
  scene->wide8_bytes = 0;
  upload_top(ctx, scene, {}, {});
}

// Whether two versions of a scene's leading words give the 8-wide layout the same instance
// table: the same instance count and, per record, the same BLAS words.
bool same_instances(uint32_t layout, const uint32_t* a, const uint32_t* b) {
  if (a[0] != b[0]) return false;
  const size_t header = layout == 0 ? 16 : 8, stride = layout == 0 ? 32 : 24;
  for (uint32_t i = 0; i < a[0]; ++i) {
    const uint32_t *ra = a + header + stride * (size_t)i, *rb = b + header + stride * (size_t)i;
    const bool same = layout == 0 ? std::equal(ra + 18, ra + 23, rb + 18)
                                  : ((ra[18] ^ rb[18]) & ~3u) == 0 && ((ra[19] ^ rb[19]) & ~3u) == 0 && ra[20] == rb[20];
    if (!same) return false;
  }
  return true;
}

}  // namespace

extern "C" {

uint32_t rt_abi_version(void) { return RT_ABI_VERSION; }

rt_status rt_ctx_create(int device, rt_ctx** out) {
  if (!out) return RT_ERR_INVALID_ARG;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) return RT_ERR_CUDA;
  auto ctx = std::make_unique<rt_ctx>();
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess) return RT_ERR_CUDA;
  if (cudaMalloc(&ctx->d_status, sizeof(rtk::DevStatus)) != cudaSuccess) return RT_ERR_OOM;
  if (cudaMemset(ctx->d_status, 0, sizeof(rtk::DevStatus)) != cudaSuccess) return RT_ERR_CUDA;
  if (cudaMalloc(&ctx->d_scratch, 64) != cudaSuccess) return RT_ERR_OOM;
  if (cudaMalloc(&ctx->d_counters, COUNTER_SLOTS * sizeof(unsigned int)) != cudaSuccess) return RT_ERR_OOM;
  for (auto& s : ctx->streams)
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return RT_ERR_CUDA;
  *out = ctx.release();
  return RT_OK;
}

void rt_ctx_destroy(rt_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  for (auto s : ctx->streams)
    if (s) cudaStreamSynchronize(s), cudaStreamDestroy(s);
  cudaFree(ctx->d_status);
  cudaFree(ctx->d_scratch);
  cudaFree(ctx->d_counters);
  cudaFree(ctx->d_rays);
  cudaFree(ctx->d_hits);
  cudaFree(ctx->d_order_scratch);
  cudaFree(ctx->d_tables);
  cudaFreeHost(ctx->h_tables);
  for (cudaEvent_t e : ctx->table_done)
    if (e) cudaEventDestroy(e);
  delete ctx;
}

const char* rt_get_last_error(const rt_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

rt_status rt_get_stats(rt_ctx* ctx, rt_stats* out) {
  if (!ctx || !out) return fail(ctx, RT_ERR_INVALID_ARG, "null argument");
  rtk::DevStatus st;
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  RT_CUDA(ctx, cudaMemcpy(&st, ctx->d_status, sizeof st, cudaMemcpyDeviceToHost));
  out->rays_traced = ctx->rays;
  out->stack_overflows = st.stack_drops;
  out->launches = ctx->launches;
  out->scene_bytes = ctx->scene_bytes;
  return RT_OK;
}

rt_status rt_ctx_set_tuning(rt_ctx* ctx, const rt_tuning* t) {
  if (!ctx || !t) return fail(ctx, RT_ERR_INVALID_ARG, "null argument");
  rt_tuning next = ctx->tuning;
  for (uint32_t v : {t->fast_refill, t->wide8_refill})
    if (v > 32) return fail(ctx, RT_ERR_INVALID_ARG, "refill thresholds are 1-32 lanes");
  if (t->wide8_stack > RT_STACK_SHARED) return fail(ctx, RT_ERR_INVALID_ARG, "unknown stack placement %u", t->wide8_stack);
  if (t->wide8_entries > 1024) return fail(ctx, RT_ERR_INVALID_ARG, "top-level entries per instance are 1-1024");
  if (t->fast_refill) next.fast_refill = t->fast_refill;
  if (t->wide8_refill) next.wide8_refill = t->wide8_refill;
  if (t->wide8_stack) next.wide8_stack = t->wide8_stack;
  if (t->wide8_entries) next.wide8_entries = t->wide8_entries;
  ctx->tuning = next;
  return RT_OK;
}

rt_status rt_ctx_get_tuning(const rt_ctx* ctx, rt_tuning* out) {
  if (!ctx || !out) return RT_ERR_INVALID_ARG;
  *out = ctx->tuning;
  return RT_OK;
}

rt_status rt_selftest(rt_ctx* ctx, uint32_t out[16]) {
  if (!ctx || !out) return fail(ctx, RT_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> lock(ctx->mu);
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  RT_CUDA(ctx, rtl::launch_selftest(ctx->d_scratch, nullptr));
  RT_CUDA(ctx, cudaMemcpy(out, ctx->d_scratch, 64, cudaMemcpyDeviceToHost));
  return RT_OK;
}

rt_status rt_scene_upload(rt_ctx* ctx, rt_layout layout, const uint32_t* words, size_t n_words, rt_scene** out) {
  if (!ctx || !words || !out) return fail(ctx, RT_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  if ((unsigned)layout > 2u) return fail(ctx, RT_ERR_INVALID_ARG, "unknown layout %d", (int)layout);
  auto s = std::make_unique<rt_scene>();
  s->layout = (uint32_t)layout;
  std::string err;
  if (!rtb::validate_scene(s->layout, words, n_words, s->info, err))
    return fail(ctx, RT_ERR_LAYOUT, "scene rejected: %s", err.c_str());
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t bytes = std::max<size_t>(n_words, 4) * 4;
  if (cudaMalloc(&s->d_words, bytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, RT_ERR_OOM, "device allocation of %zu bytes failed", bytes);
  }
  s->n_words = n_words;
  s->device_bytes = bytes;
  cudaError_t e = cudaMemcpy(s->d_words, words, n_words * 4, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(s->d_words);
    return fail(ctx, RT_ERR_CUDA, "scene copy: %s", cudaGetErrorString(e));
  }
  ctx->scene_bytes += s->device_bytes;
  *out = s.release();
  return RT_OK;
}

rt_status rt_scene_validate(rt_layout layout, const uint32_t* words, size_t n_words, uint32_t info[8], char* err,
                            size_t err_len) {
  if (!words || (unsigned)layout > 2u) return RT_ERR_INVALID_ARG;
  rtb::SceneInfo si;
  std::string e;
  bool ok = rtb::validate_scene((uint32_t)layout, words, n_words, si, e);
  if (info) {
    info[0] = si.instances, info[1] = si.top, info[2] = si.root;
    info[3] = (uint32_t)std::min<size_t>(si.triangles, UINT32_MAX), info[4] = (uint32_t)std::min<size_t>(si.nodes, UINT32_MAX);
    info[5] = si.max_blas_depth, info[6] = si.max_top_depth, info[7] = 0;
  }
  if (!ok && err && err_len) std::snprintf(err, err_len, "%s", e.c_str());
  return ok ? RT_OK : RT_ERR_LAYOUT;
}

rt_status rt_scene_update_records(rt_ctx* ctx, rt_scene* scene, const uint32_t* words, size_t n_words) {
  if (!ctx || !scene || !words) return fail(ctx, RT_ERR_INVALID_ARG, "null argument");
  if (n_words > scene->n_words) return fail(ctx, RT_ERR_INVALID_ARG, "record words exceed the scene");
  // Validate the whole buffer as it will be: the new leading words over the old mesh words.
  std::vector<uint32_t> all(scene->n_words);
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  RT_CUDA(ctx, cudaMemcpy(all.data(), scene->d_words, scene->n_words * 4, cudaMemcpyDeviceToHost));
  // the old records, to tell whether the 8-wide instance table still holds
  const size_t header = scene->layout == 0 ? 16 : 8, stride = scene->layout == 0 ? 32 : 24;
  const uint32_t most = std::max(all.empty() ? 0u : all[0], n_words ? words[0] : 0u);
  const std::vector<uint32_t> before(all.begin(), all.begin() + std::min(all.size(), header + stride * (size_t)most));
  std::copy(words, words + n_words, all.begin());
  rtb::SceneInfo info;
  std::string err;
  if (!rtb::validate_scene(scene->layout, all.data(), all.size(), info, err))
    return fail(ctx, RT_ERR_LAYOUT, "records rejected: %s", err.c_str());
  // records that name other BLASes, or another instance count, void the 8-wide instance table
  if (scene->d_wide8 && !same_instances(scene->layout, before.data(), all.data())) drop_wide8(ctx, scene);
  RT_CUDA(ctx, cudaMemcpy(scene->d_words, words, n_words * 4, cudaMemcpyHostToDevice));
  scene->info = info;
  scene->w8_top_valid = false;  // the instances' boxes may have moved: the packed top level until re-prepared
  return RT_OK;
}

rt_status rt_scene_prepare(rt_ctx* ctx, rt_scene* scene, rt_kernel kernel) {
  if (!ctx || !scene) return fail(ctx, RT_ERR_INVALID_ARG, "null argument");
  if (kernel != RT_KERNEL_WIDE8 && kernel != RT_KERNEL_WIDE8_PACKET) return RT_OK;  // PLAIN, FAST: the packed words
  if (scene->layout == RT_LAYOUT_REFLECTION_BVH2)
    return fail(ctx, RT_ERR_UNSUPPORTED, "the legacy BVH2 layout is traced by the PLAIN kernel");
  if (scene->d_wide8 && (scene->w8_top_valid || scene->info.top == 0)) return RT_OK;
  std::vector<uint32_t> words(scene->n_words);
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  RT_CUDA(ctx, cudaMemcpy(words.data(), scene->d_words, scene->n_words * 4, cudaMemcpyDeviceToHost));
  if (scene->d_wide8) return prepare_top(ctx, scene, words);  // the BLASes stand; the instances moved
  rtb::Wide8Scene w8;
  std::string err;
  const int threads = (int)std::max(1u, std::thread::hardware_concurrency());
  if (!rtb::build_wide8_scene(scene->layout, words.data(), words.size(), w8, err, threads, entries_of(ctx, scene)))
    return fail(ctx, RT_ERR_LAYOUT, "8-wide build: %s", err.c_str());
  // one allocation: nodes | triangles | instance table, each 16-byte aligned
  auto up4 = [](size_t x) { return (x + 3) & ~(size_t)3; };
  const size_t nodes_at = 0, tris_at = up4(w8.nodes.size()), inst_at = tris_at + up4(w8.tris.size());
  const size_t total = inst_at + up4(std::max<size_t>(w8.inst.size(), 1));
  void* d = nullptr;
  if (cudaMalloc(&d, total * 4) != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, RT_ERR_OOM, "device allocation of %zu bytes for the 8-wide layout failed", total * 4);
  }
  cudaError_t e = cudaMemcpy(static_cast<uint32_t*>(d) + nodes_at, w8.nodes.data(), w8.nodes.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(static_cast<uint32_t*>(d) + tris_at, w8.tris.data(), w8.tris.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !w8.inst.empty())
    e = cudaMemcpy(static_cast<uint32_t*>(d) + inst_at, w8.inst.data(), w8.inst.size() * 4, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(d);
    return fail(ctx, RT_ERR_CUDA, "8-wide upload: %s", cudaGetErrorString(e));
  }
  scene->d_wide8 = d;
  scene->wide8_bytes = total * 4;
  scene->w8_nodes_at = nodes_at, scene->w8_tris_at = tris_at, scene->w8_inst_at = inst_at;
  scene->w8_depth = w8.depth;
  scene->device_bytes += scene->wide8_bytes;
  ctx->scene_bytes += scene->wide8_bytes;
  if (!rtb::check_wide8_top(scene->layout, words.data(), w8, err)) w8.top_nodes.clear();  // the packed top level
  return upload_top(ctx, scene, w8.top_nodes, w8.top_items);
}

rt_status rt_wide8_check(rt_layout layout, const uint32_t* words, size_t n_words, uint32_t info[4], char* err,
                         size_t err_len) {
  if (!words || !info || (unsigned)layout > 1u) return RT_ERR_INVALID_ARG;
  std::string why;
  rtb::SceneInfo si;
  rtb::Wide8Scene w8;
  const int threads = (int)std::max(1u, std::thread::hardware_concurrency());
  bool ok = rtb::validate_scene((uint32_t)layout, words, n_words, si, why) &&
            rtb::build_wide8_scene((uint32_t)layout, words, n_words, w8, why, threads) &&
            rtb::check_wide8_scene(w8, info, why) && rtb::check_wide8_top((uint32_t)layout, words, w8, why);
  if (!ok && err && err_len) std::snprintf(err, err_len, "%s", why.c_str());
  return ok ? RT_OK : RT_ERR_LAYOUT;
}

rt_status rt_scene_wide8_depth(const rt_scene* scene, uint32_t* depth) {
  if (!scene || !depth) return RT_ERR_INVALID_ARG;
  if (!scene->d_wide8) return RT_ERR_UNSUPPORTED;
  *depth = scene->w8_depth;
  return RT_OK;
}

namespace {
// Seeded uniform floats for the top-level probe (splitmix64, top 24 bits).
struct ProbeRng {
  uint64_t s;
  float next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return (float)((z ^ (z >> 31)) >> 40) * (1.0f / 16777216.0f);
  }
};

// The probe of rt_scene_tune_top: n incoherent rays over the scene's world box, the first half
// closest-hit queries (origins uniform in the box, directions uniform on the sphere), the rest
// any-hit queries toward a uniform point of the box, stopping short of it.
std::vector<float> probe_rays(const rtb::Aabb& box, uint32_t n) {
  std::vector<float> r(8 * (size_t)n);
  ProbeRng g{0x70B5EEDull};
  auto point = [&](float* p) {
    for (int a = 0; a < 3; ++a) p[a] = box.lo[a] + (box.hi[a] - box.lo[a]) * g.next();
  };
  for (uint32_t i = 0; i < n; ++i) {
    float* x = r.data() + 8 * (size_t)i;
    point(x);
    x[3] = 0.0f;
    float d[3], len = 0.0f;
    if (i < n / 2) {
      const float z = 2.0f * g.next() - 1.0f, phi = 6.2831853f * g.next(), s = std::sqrt(std::max(0.0f, 1.0f - z * z));
      d[0] = s * std::cos(phi), d[1] = s * std::sin(phi), d[2] = z;
      x[7] = 1e30f;
    } else {
      float q[3];
      point(q);
      for (int a = 0; a < 3; ++a) d[a] = q[a] - x[a];
      len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      if (!(len > 1e-3f)) d[0] = 1.0f, d[1] = d[2] = 0.0f, len = 1e-3f;
      else for (int a = 0; a < 3; ++a) d[a] /= len;
      x[7] = len * (1.0f - 1e-4f);
    }
    x[4] = d[0], x[5] = d[1], x[6] = d[2];
  }
  return r;
}
}  // namespace

rt_status rt_scene_tune_top(rt_ctx* ctx, rt_scene* scene, const uint32_t* budgets, uint32_t n_budgets,
                            uint32_t probe, uint32_t* chosen) {
  if (!ctx || !scene) return fail(ctx, RT_ERR_INVALID_ARG, "null argument");
  if (n_budgets > 16 || (n_budgets && !budgets)) return fail(ctx, RT_ERR_INVALID_ARG, "0-16 budgets");
  for (uint32_t k = 0; k < n_budgets; ++k)
    if (budgets[k] == 0 || budgets[k] > 1024) return fail(ctx, RT_ERR_INVALID_ARG, "entries per instance are 1-1024");
  if (!scene->d_wide8) return fail(ctx, RT_ERR_UNSUPPORTED, "rt_scene_tune_top needs rt_scene_prepare(scene, RT_KERNEL_WIDE8)");
  if (chosen) *chosen = 0;
  if (scene->info.top == 0 || scene->info.instances < 2) return RT_OK;  // no top level to tune
  static const uint32_t kDefault[] = {1, 4, 16, 64, 256};
  if (n_budgets == 0) budgets = kDefault, n_budgets = 5;
  const uint32_t n = std::max<uint32_t>(64, std::min<uint32_t>(probe ? probe : 1u << 16, 1u << 22));
  rtb::Aabb box = scene->info.world;
  for (int a = 0; a < 3; ++a)
    if (!std::isfinite(box.lo[a]) || !std::isfinite(box.hi[a]) || !(box.hi[a] >= box.lo[a]))
      return fail(ctx, RT_ERR_LAYOUT, "the scene has no finite world box to probe");
  std::vector<uint32_t> words(scene->n_words);
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  RT_CUDA(ctx, cudaMemcpy(words.data(), scene->d_words, scene->n_words * 4, cudaMemcpyDeviceToHost));
  rtb::Wide8Scene top;
  rt_status s = read_wide8_blas(ctx, scene, words[0], top);
  if (s != RT_OK) return s;
  const std::vector<float> rays = probe_rays(box, n);
  const size_t hit_words = scene->layout == 0 ? 10 : 5;
  void *d_rays = nullptr, *d_hits = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  auto cleanup = [&]() {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (stream) cudaStreamDestroy(stream);
    cudaFree(d_rays);
    cudaFree(d_hits);
  };
  if (cudaMalloc(&d_rays, rays.size() * 4) != cudaSuccess || cudaMalloc(&d_hits, hit_words * 4 * (size_t)n) != cudaSuccess ||
      cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
      cudaEventCreate(&e1) != cudaSuccess || cudaMemcpy(d_rays, rays.data(), rays.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaGetLastError();
    cleanup();
    return fail(ctx, RT_ERR_OOM, "top-level probe buffers for %u rays", n);
  }
  const rt_ray* pr = static_cast<const rt_ray*>(d_rays);
  const uint32_t half = n / 2;
  // one pass of the probe: the closest-hit half, then the any-hit half, WIDE8 on the probe's stream
  auto pass = [&]() -> rt_status {
    rt_status t = dispatch(ctx, scene, RT_CLOSEST, RT_KERNEL_WIDE8, pr, nullptr, d_hits, half, stream);
    if (t == RT_OK) t = dispatch(ctx, scene, RT_ANY_CASTERS, RT_KERNEL_WIDE8, pr + half, nullptr, d_hits, n - half, stream);
    return t;
  };
  uint32_t best = 0;
  float best_ms = 0.0f;
  for (uint32_t k = 0; k < n_budgets && s == RT_OK; ++k) {
    s = rebuild_top(ctx, scene, words, top, budgets[k]);
    if (s != RT_OK) break;
    float ms = 0.0f;
    for (int rep = 0; rep < 3 && s == RT_OK; ++rep) {  // a warm-up pass, then the faster of two timed ones
      cudaEventRecord(e0, stream);
      s = pass();
      cudaEventRecord(e1, stream);
      if (s != RT_OK) break;
      if (cudaEventSynchronize(e1) != cudaSuccess) s = fail(ctx, RT_ERR_CUDA, "top-level probe: %s", cudaGetErrorString(cudaGetLastError()));
      float t = 0.0f;
      cudaEventElapsedTime(&t, e0, e1);
      if (rep == 1 || (rep == 2 && t < ms)) ms = t;
    }
    if (s == RT_OK && (best == 0 || ms < best_ms)) best = budgets[k], best_ms = ms;
  }
  cleanup();
  if (s != RT_OK) return s;
  scene->w8_entries = best;
  if (best != budgets[n_budgets - 1]) s = rebuild_top(ctx, scene, words, top, best);
  if (s == RT_OK && chosen) *chosen = best;
  return s;
}

rt_status rt_scene_release(rt_ctx* ctx, rt_scene* scene) {
  if (!ctx || !scene) return fail(ctx, RT_ERR_INVALID_ARG, "null argument");
  cudaSetDevice(ctx->device);
  cudaFree(scene->d_words);
  cudaFree(scene->d_wide8);
  cudaFree(scene->d_w8_top);
  cudaFree(scene->d_move);
  cudaFree(scene->d_top_order);
  for (auto& kv : scene->refit) cudaFree(kv.second.d_order);
  ctx->scene_bytes -= scene->device_bytes;
  delete scene;
  return RT_OK;
}

size_t rt_scene_device_bytes(const rt_scene* scene) { return scene ? scene->device_bytes : 0; }

rt_status rt_trace(rt_ctx* ctx, const rt_scene* scene, rt_mode mode, const rt_ray* d_rays, void* d_hits, uint32_t n,
                   void* stream) {
  return rt_trace_ex(ctx, scene, mode, RT_KERNEL_PLAIN, d_rays, nullptr, d_hits, n, stream);
}

rt_status rt_trace_ex(rt_ctx* ctx, const rt_scene* scene, rt_mode mode, rt_kernel kernel, const rt_ray* d_rays,
                      const uint32_t* d_order, void* d_hits, uint32_t n, void* stream) {
  rt_status s = check_trace_args(ctx, scene, mode, kernel);
  if (s != RT_OK) return s;
  if (n == 0) return RT_OK;
  if (!d_rays || !d_hits) return fail(ctx, RT_ERR_INVALID_ARG, "null ray or hit buffer");
  if (reinterpret_cast<uintptr_t>(d_rays) % 16 != 0) return fail(ctx, RT_ERR_INVALID_ARG, "rays must be 16-byte aligned");
  if (reinterpret_cast<uintptr_t>(d_hits) % 4 != 0) return fail(ctx, RT_ERR_INVALID_ARG, "hits must be 4-byte aligned");
  return dispatch(ctx, scene, mode, kernel, d_rays, d_order, d_hits, n, static_cast<cudaStream_t>(stream));
}

rt_status rt_trace_counted(rt_ctx* ctx, const rt_scene* scene, rt_mode mode, rt_kernel kernel, const rt_ray* d_rays,
                           void* d_hits, uint32_t n, uint64_t counts[8]) {
  rt_status s = check_trace_args(ctx, scene, mode, kernel);
  if (s != RT_OK) return s;
  if (!d_rays || !d_hits || !counts) return fail(ctx, RT_ERR_INVALID_ARG, "null argument");
  if (kernel != RT_KERNEL_WIDE8) return fail(ctx, RT_ERR_UNSUPPORTED, "counted traversal is provided for RT_KERNEL_WIDE8");
  if (!scene->d_wide8) return fail(ctx, RT_ERR_UNSUPPORTED, "the WIDE8 kernel needs rt_scene_prepare first");
  std::lock_guard<std::mutex> lock(ctx->mu);
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  unsigned long long* d_cnt = nullptr;
  RT_CUDA(ctx, cudaMalloc(&d_cnt, 8 * sizeof(unsigned long long)));
  cudaError_t e = cudaMemset(d_cnt, 0, 8 * sizeof(unsigned long long));
  if (e == cudaSuccess)
    e = rtl::count_wide8(view_of(scene), (uint32_t)mode, reinterpret_cast<const float4*>(d_rays), d_hits, n,
                         ctx->d_counters + (ctx->counter_seq++ % COUNTER_SLOTS), ctx->d_status, d_cnt, nullptr);
  if (e == cudaSuccess) e = cudaMemcpy(counts, d_cnt, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
  cudaFree(d_cnt);
  if (e != cudaSuccess) return fail(ctx, RT_ERR_CUDA, "counted traversal: %s", cudaGetErrorString(e));
  return RT_OK;
}

namespace {
// Grows the ordering scratch to cover n rays (caller holds ctx->mu).
rt_status ensure_order_scratch(rt_ctx* ctx, uint32_t n) {
  const size_t need = rtl::order_scratch_bytes(n);
  if (need <= ctx->order_scratch_bytes) return RT_OK;
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  RT_CUDA(ctx, cudaDeviceSynchronize());
  cudaFree(ctx->d_order_scratch);
  ctx->d_order_scratch = nullptr;
  ctx->order_scratch_bytes = 0;
  if (cudaMalloc(&ctx->d_order_scratch, need) != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, RT_ERR_OOM, "ordering scratch of %zu bytes", need);
  }
  ctx->order_scratch_bytes = need;
  return RT_OK;
}
}  // namespace

rt_status rt_order_rays(rt_ctx* ctx, const rt_scene* scene, const rt_ray* d_rays, uint32_t n, rt_ray_order key,
                        uint32_t* d_order, void* stream) {
  if (!ctx || !scene || (n && (!d_rays || !d_order))) return fail(ctx, RT_ERR_INVALID_ARG, "null argument");
  if ((unsigned)key > 3u) return fail(ctx, RT_ERR_INVALID_ARG, "unknown ray order %d", (int)key);
  if (n == 0) return RT_OK;
  std::lock_guard<std::mutex> lock(ctx->mu);
  rt_status s = ensure_order_scratch(ctx, n);
  if (s != RT_OK) return s;
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  const rtb::Aabb& wb = scene->info.world;
  float lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = std::isfinite(wb.lo[a]) ? wb.lo[a] : -1.0f;
    hi[a] = std::isfinite(wb.hi[a]) ? wb.hi[a] : 1.0f;
  }
  if (key == RT_ORDER_NONE) key = RT_ORDER_ORIGIN;
  RT_CUDA(ctx, rtl::launch_order(reinterpret_cast<const float4*>(d_rays), n, lo, hi, (uint32_t)key, d_order,
                                 ctx->d_order_scratch, ctx->order_scratch_bytes, static_cast<cudaStream_t>(stream)));
  return RT_OK;
}

rt_status rt_ctx_reserve(rt_ctx* ctx, uint32_t max_rays) {
  if (!ctx) return RT_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lock(ctx->mu);
  {
    rt_status so = ensure_order_scratch(ctx, max_rays);
    if (so != RT_OK) return so;
  }
  const size_t want = std::min<size_t>(max_rays, HOST_CHUNK);
  if (want <= ctx->stage_rays) return RT_OK;
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  for (auto s : ctx->streams) RT_CUDA(ctx, cudaStreamSynchronize(s));
  cudaFree(ctx->d_rays);
  cudaFree(ctx->d_hits);
  ctx->d_rays = ctx->d_hits = nullptr;
  ctx->stage_rays = 0;
  if (cudaMalloc(&ctx->d_rays, RT_HOST_STAGES * want * RAY_BYTES) != cudaSuccess ||
      cudaMalloc(&ctx->d_hits, RT_HOST_STAGES * want * GI_HIT_BYTES) != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, RT_ERR_OOM, "staging allocation for %zu rays failed", want);
  }
  ctx->stage_rays = want;
  return RT_OK;
}

rt_status rt_trace_host_batches(rt_ctx* ctx, const rt_scene* scene, const rt_host_batch* batches,
                                uint32_t n_batches) {
  if (!ctx || (n_batches && !batches)) return fail(ctx, RT_ERR_INVALID_ARG, "null argument");
  uint32_t most = 0;
  for (uint32_t k = 0; k < n_batches; ++k) {
    const rt_host_batch& hb = batches[k];
    rt_status s = check_trace_args(ctx, scene, hb.mode, hb.kernel);
    if (s != RT_OK) return s;
    if (hb.n && (!hb.h_rays || !hb.h_hits)) return fail(ctx, RT_ERR_INVALID_ARG, "null ray or hit buffer");
    most = std::max(most, hb.n);
  }
  if (most == 0) return RT_OK;
  rt_status s = rt_ctx_reserve(ctx, most);
  if (s != RT_OK) return s;
  std::lock_guard<std::mutex> lock(ctx->mu);
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  const uint32_t chunk = (uint32_t)ctx->stage_rays;
  uint32_t c = 0;  // chunks take the streams and staging slots in turn, across batches
  for (uint32_t k = 0; k < n_batches; ++k) {
    const rt_host_batch& hb = batches[k];
    const size_t bytes = hit_bytes(scene->layout, (uint32_t)hb.mode);
    for (uint32_t off = 0; off < hb.n; off += chunk, ++c) {
      const uint32_t m = std::min(chunk, hb.n - off);
      const uint32_t b = c % RT_HOST_STAGES;
      cudaStream_t st = ctx->streams[b];
      char* dr = static_cast<char*>(ctx->d_rays) + (size_t)b * chunk * RAY_BYTES;
      char* dh = static_cast<char*>(ctx->d_hits) + (size_t)b * chunk * GI_HIT_BYTES;
      RT_CUDA(ctx, cudaMemcpyAsync(dr, hb.h_rays + off, (size_t)m * RAY_BYTES, cudaMemcpyHostToDevice, st));
      rt_status d = dispatch(ctx, scene, hb.mode, hb.kernel, reinterpret_cast<const rt_ray*>(dr), nullptr, dh, m, st);
      if (d != RT_OK) {
        for (auto t : ctx->streams) cudaStreamSynchronize(t);
        return d;
      }
      RT_CUDA(ctx, cudaMemcpyAsync(static_cast<char*>(hb.h_hits) + (size_t)off * bytes, dh, (size_t)m * bytes,
                                   cudaMemcpyDeviceToHost, st));
    }
  }
  for (auto st : ctx->streams) RT_CUDA(ctx, cudaStreamSynchronize(st));
  return RT_OK;
}

rt_status rt_trace_host(rt_ctx* ctx, const rt_scene* scene, rt_mode mode, rt_kernel kernel, const rt_ray* h_rays,
                        void* h_hits, uint32_t n) {
  const rt_host_batch one{h_rays, h_hits, n, mode, kernel};
  return rt_trace_host_batches(ctx, scene, &one, 1);
}

// ---------------------------------------------------------------- host builders

rt_status rt_blas_build(const float* positions, uint32_t n_positions, const uint32_t* indices, uint32_t n_indices,
                        uint32_t build_flags, rt_blas** out) {
  if (!positions || !indices || !out) return RT_ERR_INVALID_ARG;
  *out = nullptr;
  auto b = std::make_unique<rt_blas>();
  std::string err;
  bool ok = (build_flags & RT_BUILD_MEDIAN)
                ? rtb::build_blas(positions, n_positions, indices, n_indices, false, b->b, err)
                : rtb::build_blas_sah(positions, n_positions, indices, n_indices, b->b, err);
  if (!ok) return RT_ERR_INVALID_ARG;
  *out = b.release();
  return RT_OK;
}

rt_status rt_blas_info(const rt_blas* blas, uint32_t info[6]) {
  if (!blas || !info) return RT_ERR_INVALID_ARG;
  const rtb::Blas& b = blas->b;
  info[0] = (uint32_t)b.node_count();
  info[1] = (uint32_t)b.leaf_count();
  info[2] = (uint32_t)(b.positions.size() / 3);
  info[3] = (uint32_t)b.indices.size();
  info[4] = b.root;
  info[5] = (uint32_t)rtb::blas_depth(b, b.root);
  return RT_OK;
}

rt_status rt_blas_nodes(const rt_blas* blas, uint32_t* out) {
  if (!blas || !out) return RT_ERR_INVALID_ARG;
  std::copy(blas->b.nodes.begin(), blas->b.nodes.end(), out);
  return RT_OK;
}

rt_status rt_blas_indices(const rt_blas* blas, uint32_t* out) {
  if (!blas || !out) return RT_ERR_INVALID_ARG;
  std::copy(blas->b.indices.begin(), blas->b.indices.end(), out);
  return RT_OK;
}

rt_status rt_blas_refit(rt_blas* blas, const float* positions, uint32_t n_positions) {
  if (!blas || !positions) return RT_ERR_INVALID_ARG;
  std::string err;
  return rtb::refit_blas(blas->b, positions, n_positions, err) ? RT_OK : RT_ERR_INVALID_ARG;
}

void rt_blas_free(rt_blas* blas) { delete blas; }

rt_status rt_pack_scene(rt_layout layout, const rt_blas* const* meshes, uint32_t n_meshes,
                        const float* const* mesh_positions, const uint32_t* const* mesh_indices,
                        const uint32_t* mesh_n_indices, const uint32_t* mesh_primitives, const rt_instance* instances,
                        uint32_t n_instances, int tlas_mode, uint32_t* out_words, size_t* n_words) {
  if (!n_words || (n_meshes && (!meshes || !mesh_positions || !mesh_indices || !mesh_n_indices)) ||
      (n_instances && !instances))
    return RT_ERR_INVALID_ARG;
  std::vector<rtb::MeshRef> refs(n_meshes);
  for (uint32_t m = 0; m < n_meshes; ++m) {
    if (!meshes[m]) return RT_ERR_INVALID_ARG;
    refs[m] = rtb::MeshRef{&meshes[m]->b, mesh_positions[m], mesh_indices[m], mesh_n_indices[m],
                           mesh_primitives ? mesh_primitives[m] != 0 : false};
  }
  std::vector<rtb::Placement> inst(n_instances);
  for (uint32_t i = 0; i < n_instances; ++i) {
    const rt_instance& s = instances[i];
    rtb::Placement& p = inst[i];
    std::copy(s.model, s.model + 12, p.model);
    std::copy(s.rows, s.rows + 12, p.rows);
    p.mesh = s.mesh, p.slot = s.slot, p.casts_shadow = s.casts_shadow, p.near_base = s.near_base;
    std::copy(s.extra, s.extra + 8, p.extra);
  }
  std::vector<uint32_t> words;
  std::string err;
  bool ok = layout == RT_LAYOUT_GI ? rtb::pack_gi(refs, inst, tlas_mode, words, err)
                                   : rtb::pack_reflection(refs, inst, tlas_mode, words, err);
  if (!ok) return RT_ERR_LAYOUT;
  if (!out_words) {
    *n_words = words.size();
    return RT_OK;
  }
  if (*n_words < words.size()) {
    *n_words = words.size();
    return RT_ERR_INVALID_ARG;
  }
  std::copy(words.begin(), words.end(), out_words);
  *n_words = words.size();
  return RT_OK;
}

rt_status rt_object_box(rt_layout layout, const rt_blas* blas, const float* positions, const uint32_t* indices,
                        uint32_t n_indices, float box[6]) {
  if (!blas || !box || (unsigned)layout > 1u) return RT_ERR_INVALID_ARG;
  rtb::Aabb b = rtb::Aabb::empty();
  if (layout == RT_LAYOUT_GI) {
    b = blas->b.bounds;
  } else {
    if (n_indices && (!positions || !indices)) return RT_ERR_INVALID_ARG;
    for (uint32_t k = 0; k < n_indices; ++k) b.grow(positions + 3 * (size_t)indices[k]);
  }
  for (int a = 0; a < 3; ++a) box[a] = b.lo[a], box[3 + a] = b.hi[a];
  return RT_OK;
}

namespace {
bool placements_of(const rt_instance* instances, uint32_t n, std::vector<rtb::Placement>& out) {
  if (n && !instances) return false;
  out.resize(n);
  for (uint32_t i = 0; i < n; ++i) {
    const rt_instance& s = instances[i];
    rtb::Placement& p = out[i];
    std::copy(s.model, s.model + 12, p.model);
    std::copy(s.rows, s.rows + 12, p.rows);
    p.mesh = s.mesh, p.slot = s.slot, p.casts_shadow = s.casts_shadow, p.near_base = s.near_base;
    std::copy(s.extra, s.extra + 8, p.extra);
  }
  return true;
}
}  // namespace

rt_status rt_move_instances_host(rt_layout layout, uint32_t* words, size_t n_words, const rt_instance* instances,
                                 uint32_t n, const float* mesh_boxes, uint32_t n_meshes) {
  if (!words || n_words < 8 || (unsigned)layout > 1u || (n_meshes && !mesh_boxes)) return RT_ERR_INVALID_ARG;
  std::vector<rtb::Placement> inst;
  if (!placements_of(instances, n, inst)) return RT_ERR_INVALID_ARG;
  std::vector<rtb::Aabb> boxes(n_meshes);
  for (uint32_t m = 0; m < n_meshes; ++m)
    for (int a = 0; a < 3; ++a) boxes[m].lo[a] = mesh_boxes[6 * m + a], boxes[m].hi[a] = mesh_boxes[6 * m + 3 + a];
  std::string err;
  return rtb::move_instances((uint32_t)layout, words, n_words, inst, boxes, err) ? RT_OK : RT_ERR_LAYOUT;
}

rt_status rt_tlas_build(const float* boxes, uint32_t n, int sah, uint32_t* out, size_t* n_words) {
  if (!boxes || !n_words || n < 2) return RT_ERR_INVALID_ARG;
  std::vector<rtb::Aabb> b(n);
  for (uint32_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) b[i].lo[a] = boxes[6 * i + a], b[i].hi[a] = boxes[6 * i + 3 + a];
  std::vector<uint32_t> nodes = rtb::tlas_build(b, sah != 0);
  if (!out) {
    *n_words = nodes.size();
    return RT_OK;
  }
  if (*n_words < nodes.size()) {
    *n_words = nodes.size();
    return RT_ERR_INVALID_ARG;
  }
  std::copy(nodes.begin(), nodes.end(), out);
  *n_words = nodes.size();
  return RT_OK;
}

rt_status rt_tlas_refit(uint32_t* nodes, size_t n_words, const float* boxes, uint32_t n) {
  if (!nodes || !boxes || n < 2 || n_words < 32) return RT_ERR_INVALID_ARG;
  std::vector<rtb::Aabb> b(n);
  for (uint32_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) b[i].lo[a] = boxes[6 * i + a], b[i].hi[a] = boxes[6 * i + 3 + a];
  rtb::tlas_refit(nodes, b);
  return RT_OK;
}

}  // extern "C"

rt_status rt_gi_cell_rays(rt_ctx* ctx, const rt_gi_cell* d_cells, uint32_t n_cells, uint32_t flags, rt_ray* d_rays,
                          void* stream) {
  if (!ctx || (n_cells && (!d_cells || !d_rays))) return fail(ctx, RT_ERR_INVALID_ARG, "null argument");
  if (n_cells > (1u << 25)) return fail(ctx, RT_ERR_INVALID_ARG, "at most 2^25 cells a call");
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  RT_CUDA(ctx, rtl::launch_cell_rays(d_cells, n_cells, (flags & RT_GI_ROTATE) ? 1u : 0u, reinterpret_cast<float4*>(d_rays),
                                     static_cast<cudaStream_t>(stream)));
  return RT_OK;
}

rt_status rt_trace_gi_cells(rt_ctx* ctx, const rt_scene* scene, rt_mode mode, const rt_gi_cell* d_cells,
                            uint32_t n_cells, uint32_t flags, void* d_hits, void* stream) {
  rt_status s = check_trace_args(ctx, scene, mode, RT_KERNEL_FAST);
  if (s != RT_OK) return s;
  if (scene->layout != RT_LAYOUT_GI) return fail(ctx, RT_ERR_INVALID_ARG, "the cell producers trace GI-layout scenes");
  if (n_cells && (!d_cells || !d_hits)) return fail(ctx, RT_ERR_INVALID_ARG, "null argument");
  if (n_cells > (1u << 25)) return fail(ctx, RT_ERR_INVALID_ARG, "at most 2^25 cells a call");
  if (reinterpret_cast<uintptr_t>(d_hits) % 4 != 0) return fail(ctx, RT_ERR_INVALID_ARG, "hits must be 4-byte aligned");
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaError_t e = rtl::launch_fast_cells(view_of(scene), (uint32_t)mode, d_cells, n_cells, (flags & RT_GI_ROTATE) ? 1u : 0u,
                                         d_hits, ctx->d_counters + (ctx->counter_seq++ % COUNTER_SLOTS), ctx->d_status,
                                         static_cast<cudaStream_t>(stream), ctx->tuning.fast_refill);
  if (e != cudaSuccess) return fail(ctx, RT_ERR_CUDA, "cell traversal: %s", cudaGetErrorString(e));
  ctx->rays += (uint64_t)n_cells * RT_GI_DIRECTIONS;
  ctx->launches += 1;
  return RT_OK;
}

rt_status rt_trace_gi_lights(rt_ctx* ctx, const rt_scene* scene, rt_kernel kernel, const rt_gi_cell* d_cells,
                             uint32_t n_cells, const rt_gi_light* d_lights, uint32_t n_lights, uint32_t* d_words,
                             void* stream) {
  rt_status s = check_trace_args(ctx, scene, RT_ANY_CASTERS, kernel);
  if (s != RT_OK) return s;
  if (scene->layout != RT_LAYOUT_GI) return fail(ctx, RT_ERR_INVALID_ARG, "the light producer traces GI-layout scenes");
  if (kernel != RT_KERNEL_FAST && kernel != RT_KERNEL_WIDE8)
    return fail(ctx, RT_ERR_UNSUPPORTED, "light visibility is traced by RT_KERNEL_FAST or RT_KERNEL_WIDE8");
  if (kernel == RT_KERNEL_WIDE8 && !scene->d_wide8)
    return fail(ctx, RT_ERR_UNSUPPORTED, "the WIDE8 kernel needs rt_scene_prepare first");
  if (n_cells == 0 || n_lights == 0) return RT_OK;
  if (!d_cells || !d_lights || !d_words) return fail(ctx, RT_ERR_INVALID_ARG, "null argument");
  if ((uint64_t)n_cells * n_lights > (1ull << 31))
    return fail(ctx, RT_ERR_INVALID_ARG, "at most 2^31 (cell, light) pairs a call");
  if (reinterpret_cast<uintptr_t>(d_cells) % 16 != 0 || reinterpret_cast<uintptr_t>(d_lights) % 16 != 0 ||
      reinterpret_cast<uintptr_t>(d_words) % 4 != 0)
    return fail(ctx, RT_ERR_INVALID_ARG, "cells and lights must be 16-byte aligned, words 4-byte aligned");
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  const rtl::SceneView v = view_of(scene);
  unsigned int* counter = ctx->d_counters + (ctx->counter_seq++ % COUNTER_SLOTS);
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e;
  if (kernel == RT_KERNEL_FAST) {
    e = rtl::launch_fast_lights(v, d_cells, n_cells, d_lights, n_lights, d_words, counter, ctx->d_status, st,
                                ctx->tuning.fast_refill);
  } else {
    const uint32_t stack = ctx->tuning.wide8_stack == RT_STACK_SHARED && rtl::shared_stack_fits(v) ? 1u : 0u;
    e = rtl::launch_wide8_lights(v, d_cells, n_cells, d_lights, n_lights, d_words, counter, ctx->d_status, st,
                                 ctx->tuning.wide8_refill, stack);
  }
  if (e != cudaSuccess) return fail(ctx, RT_ERR_CUDA, "light visibility traversal: %s", cudaGetErrorString(e));
  ctx->rays += (uint64_t)n_cells * n_lights;
  ctx->launches += 1;
  return RT_OK;
}

// ---------------------------------------------------------------- cooked files

namespace {

rt_status cooked_error(const std::string& what, char* err, size_t err_len) {
  if (err && err_len) {
    const size_t k = std::min(what.size(), err_len - 1);
    std::memcpy(err, what.data(), k);
    err[k] = 0;
  }
  return RT_ERR_LAYOUT;
}

rt_status copy_out(const std::vector<uint8_t>& bytes, uint8_t* out, size_t* n_bytes) {
  if (!out) {
    *n_bytes = bytes.size();
    return RT_OK;
  }
  const bool fits = *n_bytes >= bytes.size();
  *n_bytes = bytes.size();
  if (!fits) return RT_ERR_INVALID_ARG;
  std::copy(bytes.begin(), bytes.end(), out);
  return RT_OK;
}

}  // namespace

rt_status rt_blas_positions(const rt_blas* blas, float* out) {
  if (!blas || !out) return RT_ERR_INVALID_ARG;
  std::copy(blas->b.positions.begin(), blas->b.positions.end(), out);
  return RT_OK;
}

rt_status rt_blas_encode_rlb(const rt_blas* blas, uint64_t max_bytes, uint8_t* out, size_t* n_bytes, char* err,
                             size_t err_len) {
  if (!blas || !n_bytes) return RT_ERR_INVALID_ARG;
  std::vector<uint8_t> bytes;
  std::string why;
  if (!rtb::encode_rlb(blas->b, max_bytes, bytes, why)) return cooked_error(why, err, err_len);
  return copy_out(bytes, out, n_bytes);
}

rt_status rt_rlb_decode(const uint8_t* bytes, size_t n_bytes, uint64_t max_bytes, uint32_t level, rt_blas** out,
                        char* err, size_t err_len) {
  if ((!bytes && n_bytes) || !out) return RT_ERR_INVALID_ARG;
  *out = nullptr;
  auto b = std::make_unique<rt_blas>();
  std::string why;
  if (!rtb::decode_rlb(bytes, n_bytes, max_bytes, level, b->b, why)) return cooked_error(why, err, err_len);
  *out = b.release();
  return RT_OK;
}

rt_status rt_rnf_decode(const uint8_t* bytes, size_t n_bytes, uint64_t max_bytes, rt_rnf** out, char* err,
                        size_t err_len) {
  if ((!bytes && n_bytes) || !out) return RT_ERR_INVALID_ARG;
  *out = nullptr;
  auto f = std::make_unique<rt_rnf>();
  std::string why;
  static const uint8_t none[1] = {0};
  if (!rtb::decode_rnf(bytes ? bytes : none, n_bytes, max_bytes, f->f, why)) return cooked_error(why, err, err_len);
  *out = f.release();
  return RT_OK;
}

rt_status rt_rnf_info(const rt_rnf* field, rt_rnf_settings* settings, uint8_t source[32], uint32_t* n_meshes,
                      uint32_t* n_placements) {
  if (!field) return RT_ERR_INVALID_ARG;
  const rtb::Rnf& f = field->f;
  if (settings) *settings = rt_rnf_settings{f.settings.lod_error, f.settings.reach, f.settings.skip, f.settings.bins};
  if (source) std::memcpy(source, f.source, 32);
  if (n_meshes) *n_meshes = (uint32_t)f.meshes.size();
  if (n_placements) *n_placements = (uint32_t)f.placements.size();
  return RT_OK;
}

rt_status rt_rnf_mesh(const rt_rnf* field, uint32_t mesh, rt_blas** out) {
  if (!field || !out || mesh >= field->f.meshes.size()) return RT_ERR_INVALID_ARG;
  auto b = std::make_unique<rt_blas>();
  b->b = field->f.meshes[mesh];
  *out = b.release();
  return RT_OK;
}

rt_status rt_rnf_placement_get(const rt_rnf* field, uint32_t k, rt_rnf_placement* out) {
  if (!field || !out || k >= field->f.placements.size()) return RT_ERR_INVALID_ARG;
  const rtb::RnfPlacement& p = field->f.placements[k];
  out->mesh = p.mesh;
  std::copy(p.transform, p.transform + 16, out->transform);
  out->masks = p.masks.data();
  out->n_masks = p.masks.size();
  return RT_OK;
}

rt_status rt_rnf_encode(const rt_rnf_settings* settings, const uint8_t source[32], const rt_blas* const* meshes,
                        uint32_t n_meshes, const rt_rnf_placement* placements, uint32_t n_placements,
                        uint64_t max_bytes, uint8_t* out, size_t* n_bytes, char* err, size_t err_len) {
  if (!settings || !source || !n_bytes || (n_meshes && !meshes) || (n_placements && !placements))
    return RT_ERR_INVALID_ARG;
  rtb::Rnf f;
  f.settings = rtb::RnfSettings{settings->lod_error, settings->reach, settings->skip, settings->bins};
  std::memcpy(f.source, source, 32);
  for (uint32_t m = 0; m < n_meshes; ++m) {
    if (!meshes[m]) return RT_ERR_INVALID_ARG;
    f.meshes.push_back(meshes[m]->b);
  }
  for (uint32_t k = 0; k < n_placements; ++k) {
    const rt_rnf_placement& s = placements[k];
    if (s.n_masks && !s.masks) return RT_ERR_INVALID_ARG;
    rtb::RnfPlacement p;
    p.mesh = s.mesh;
    std::copy(s.transform, s.transform + 16, p.transform);
    p.masks.assign(s.masks, s.masks + s.n_masks);
    f.placements.push_back(std::move(p));
  }
  std::vector<uint8_t> bytes;
  std::string why;
  if (!rtb::encode_rnf(f, max_bytes, bytes, why)) return cooked_error(why, err, err_len);
  return copy_out(bytes, out, n_bytes);
}

rt_status rt_rnf_pack_gi(const rt_rnf* field, const rt_instance* instances, uint32_t n_instances, int tlas_mode,
                         uint32_t* out_words, size_t* n_words) {
  if (!field || !n_words || (n_instances && !instances)) return RT_ERR_INVALID_ARG;
  const rtb::Rnf& f = field->f;
  std::vector<rtb::MeshRef> refs(f.meshes.size());
  for (size_t m = 0; m < f.meshes.size(); ++m) {
    const rtb::Blas& b = f.meshes[m];
    refs[m] = rtb::MeshRef{&b, b.positions.data(), b.indices.data(), b.indices.size(), false};
  }
  // set_indirect_near_field (gi_cache.rs:3240-3248): per mesh, its placements that have masks.
  for (const rtb::RnfPlacement& p : f.placements) {
    if (p.masks.empty()) continue;
    rtb::NearMasks q;
    std::copy(p.transform, p.transform + 16, q.transform);
    q.masks = p.masks.data(), q.n_masks = p.masks.size();
    refs[p.mesh].near.push_back(q);
  }
  std::vector<rtb::Placement> inst(n_instances);
  for (uint32_t i = 0; i < n_instances; ++i) {
    const rt_instance& s = instances[i];
    rtb::Placement& p = inst[i];
    std::copy(s.model, s.model + 12, p.model);
    std::copy(s.rows, s.rows + 12, p.rows);
    p.mesh = s.mesh, p.slot = s.slot, p.casts_shadow = s.casts_shadow, p.near_base = 0;
    std::copy(s.extra, s.extra + 8, p.extra);
  }
  std::vector<uint32_t> words;
  std::string err;
  if (!rtb::pack_gi(refs, inst, tlas_mode, words, err)) return RT_ERR_LAYOUT;
  if (!out_words) {
    *n_words = words.size();
    return RT_OK;
  }
  if (*n_words < words.size()) {
    *n_words = words.size();
    return RT_ERR_INVALID_ARG;
  }
  std::copy(words.begin(), words.end(), out_words);
  *n_words = words.size();
  return RT_OK;
}

rt_status rt_rnf_world(const rt_rnf* field, rt_blas** out, uint32_t* bases) {
  if (!field || !out) return RT_ERR_INVALID_ARG;
  *out = nullptr;
  auto b = std::make_unique<rt_blas>();
  std::vector<uint32_t> at;
  std::string err;
  if (!rtb::rnf_world(field->f, b->b, at, err)) return RT_ERR_INVALID_ARG;
  if (bases) std::copy(at.begin(), at.end(), bases);
  *out = b.release();
  return RT_OK;
}

void rt_rnf_free(rt_rnf* field) { delete field; }
