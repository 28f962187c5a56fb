// Internal state behind the C ABI's opaque handles, shared by the translation units that
// implement it (rt_api.cu, batches.cu).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdarg>
#include <map>
#include <vector>
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/rt_trace.h"
#include "host/host.hpp"
#include "host/wide8.hpp"
#include "launch.hpp"

// Per BLAS of a scene, what rt_scene_refit needs about its (fixed) topology: its nodes ordered
// by height above the leaves, and where each height starts.
struct RefitLevels {
  uint32_t node_count = 0;
  uint32_t tri_count = 0;           // reflection layout: packed triangles of the BLAS
  uint32_t position_count = 0;      // GI layout: position records of the BLAS
  std::vector<uint32_t> level_start;  // level h: d_order[level_start[h], level_start[h + 1])
  uint32_t* d_order = nullptr;
};

struct rt_scene {
  uint32_t layout = 0;
  uint32_t* d_words = nullptr;
  size_t n_words = 0;
  rtb::SceneInfo info;
  size_t device_bytes = 0;
  void* d_wide8 = nullptr;
  size_t wide8_bytes = 0;
  size_t w8_nodes_at = 0, w8_tris_at = 0, w8_inst_at = 0;
  uint32_t w8_depth = 0;  // levels of the deepest 8-wide BLAS
  // The WIDE8 walk's 8-wide top level over the instance world boxes (its own allocation: nodes,
  // then instance items). Built by rt_scene_prepare when the packed scene has a top level; a
  // rewrite of the records or the top level makes it stale, and the walk then uses the packed
  // BVH4 top level until rt_scene_prepare builds it again.
  void* d_w8_top = nullptr;
  size_t w8_top_bytes = 0, w8_top_items_at = 0;
  uint32_t w8_top_nodes = 0;
  bool w8_top_valid = false;
  uint32_t w8_entries = 0;  // the top level's entries per instance (rt_scene_tune_top); 0: the context's

  std::map<uint32_t, RefitLevels> refit;  // by the BLAS's node base word
  // rt_scene_move_instances: staging for the moved instances and mesh boxes, and the top level's
  // nodes grouped by height (deepest last), kept until a rebuild changes the tree.
  void* d_move = nullptr;
  size_t move_bytes = 0;
  std::vector<uint32_t> top_order, top_level_start;
  uint32_t* d_top_order = nullptr;
};

struct rt_blas {
  rtb::Blas b;
};

struct rt_rnf {
  rtb::Rnf f;
};

// Chunks a host-buffer call keeps in flight, each with its own stream and staging slot. A
// stream runs its chunk's copy in, trace and copy out in order, so with two slots the next copy
// in waits for the copy out two chunks back; four leave the copies off the critical path.
#ifndef RT_HOST_STAGES
#define RT_HOST_STAGES 4
#endif

struct rt_ctx {
  int device = 0;
  rtk::DevStatus* d_status = nullptr;
  uint32_t* d_scratch = nullptr;  // 16 words for the self-test
  // Ray counters of persistent launches: launch k uses slot k mod COUNTER_SLOTS, so up to that
  // many launches may be in flight at once across streams.
  unsigned int* d_counters = nullptr;
  std::atomic<uint64_t> counter_seq{0};
  rt_tuning tuning = {8, 8, RT_STACK_LOCAL, rtb::W8_BRAID_PER_INSTANCE, {0, 0, 0, 0}};
  std::mutex mu;
  std::string last_error;
  std::atomic<uint64_t> rays{0}, launches{0}, scene_bytes{0};
  // rt_trace_host staging: HOST_STAGES chunks in flight, one stream and staging slot each.
  cudaStream_t streams[RT_HOST_STAGES] = {};
  void* d_rays = nullptr;
  void* d_hits = nullptr;
  size_t stage_rays = 0;  // rays per chunk buffer
  // rt_order_rays scratch
  void* d_order_scratch = nullptr;
  size_t order_scratch_bytes = 0;
  // rt_trace_batches: batch tables staged through a ring of pinned / device slots, each reused
  // once the copy that last read it has completed.
  static constexpr uint32_t TABLE_SLOTS = 8;
  rtk::BatchEntry* h_tables = nullptr;
  rtk::BatchEntry* d_tables = nullptr;
  cudaEvent_t table_done[TABLE_SLOTS] = {};
  uint32_t table_seq = 0;
};

namespace rtc {

// The instance top level built on the device (tlas_build.cu), word for word rtb::tlas_build's:
// instance i's box is lo xyz at d_box_words[i * stride], hi xyz right after (float bits). The
// nodes go to d_out (cap_words available, the rest zeroed); with d_order, the node ids grouped
// by level, deepest first (a bottom-up refit order), level starts in *level_start. Synchronous
// on `st`; the caller holds the context's lock.
rt_status tlas_build_device(rt_ctx* ctx, const uint32_t* d_box_words, size_t stride, uint32_t n, bool sah, uint32_t* d_out,
                            size_t cap_words, uint32_t* d_order, std::vector<uint32_t>* level_start, uint32_t* n_nodes,
                            cudaStream_t st);

constexpr size_t GI_HIT_BYTES = 40, RS_HIT_BYTES = 20, ANY_HIT_BYTES = 4, RAY_BYTES = 32;
#ifndef RT_HOST_CHUNK_LOG2
#define RT_HOST_CHUNK_LOG2 20
#endif
// Rays a host-buffer call stages per chunk (copies of one chunk overlap the next chunk's kernel).
// 2^20: measured end to end on the precision-4M step (16.8M rays, four stages) at 771 Mrays/s,
// against 752 for 2^19 (more launches, each with its tail of idle lanes and its final pass) and
// 773 for 2^21 (eight stages of 2^20: 776).
constexpr uint32_t HOST_CHUNK = 1u << RT_HOST_CHUNK_LOG2;
constexpr uint32_t COUNTER_SLOTS = 4096;

inline rt_status fail(rt_ctx* ctx, rt_status s, const char* fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    ctx->last_error = buf;
  }
  return s;
}

#define RT_CUDA(ctx, call)                                                                     \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) return fail(ctx, RT_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

inline size_t hit_bytes(uint32_t layout, uint32_t mode) {
  if (mode != 0) return ANY_HIT_BYTES;
  return layout == 0 ? GI_HIT_BYTES : RS_HIT_BYTES;
}

inline rtl::SceneView view_of(const rt_scene* s) {
  rtl::SceneView v;
  v.layout = s->layout;
  v.words = s->d_words;
  v.n_words = s->n_words;
  v.instances = s->info.instances;
  v.top = s->info.top;
  v.wide8 = s->d_wide8;
  v.wide8_bytes = s->wide8_bytes;
  v.w8_nodes_at = s->w8_nodes_at, v.w8_tris_at = s->w8_tris_at, v.w8_inst_at = s->w8_inst_at;
  v.w8_depth = s->w8_depth;
  v.w8_top = s->w8_top_valid ? s->d_w8_top : nullptr;
  v.w8_top_nodes = s->w8_top_valid ? s->w8_top_nodes : 0;
  v.w8_top_items_at = s->w8_top_items_at;
  return v;
}

}  // namespace rtc
