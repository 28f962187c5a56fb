// Launchers for the WIDE8 kernels.
#include <map>
#include <mutex>

#include "kernels/cells.cuh"
#include "kernels/wide8.cuh"
#include "launch.hpp"

namespace rtl {

namespace {
constexpr int W8_BLOCK = 128;
}

// Resident blocks of `kernel` on the current device: one cache per kernel, since instances of one
// signature (the same function-pointer type) can differ in registers and shared memory.
template <class K>
cudaError_t resident(K kernel, uint32_t& out) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, uint32_t> cached;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const auto key = std::make_pair(reinterpret_cast<const void*>(kernel), dev);
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = cached.find(key);
    if (it != cached.end()) {
      out = it->second;
      return cudaSuccess;
    }
  }
  int sms = 0, per_sm = 0;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, W8_BLOCK, 0);
  if (e != cudaSuccess) return e;
  out = (uint32_t)sms * (uint32_t)(per_sm > 0 ? per_sm : 1);
  std::lock_guard<std::mutex> lock(mu);
  cached[key] = out;
  return cudaSuccess;
}

template <class K, class Src>
cudaError_t run(K kernel, const uint32_t* words, const rtk::W8View& v, const Src& src, unsigned int* counter, uint32_t n,
                rtk::DevStatus* st, cudaStream_t stream, unsigned long long* cnt, uint32_t refill) {
  uint32_t full = 0;
  cudaError_t e = resident(kernel, full);
  if (e != cudaSuccess) return e;
  const uint32_t need = (n + W8_BLOCK - 1) / W8_BLOCK;
  if ((e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), stream)) != cudaSuccess) return e;
  kernel<<<need < full ? need : full, W8_BLOCK, 0, stream>>>(words, v, src, counter, n, st, cnt, refill);
  return cudaGetLastError();
}

// The f64 final pass of a closest-hit launch (rtk::k_wide8_final), on the walk's stream.
template <class Src>
cudaError_t final_pass(const SceneView& s, const rtk::W8View& v, const Src& src, uint32_t n, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  const uint32_t blocks = (n + 255) / 256;
  if (s.layout == 0) rtk::k_wide8_final<0><<<blocks, 256, 0, stream>>>(s.words, v, src, n);
  else rtk::k_wide8_final<1><<<blocks, 256, 0, stream>>>(s.words, v, src, n);
  return cudaGetLastError();
}

// A launch's walk followed, where it answers closest-hit queries, by the final pass.
template <class Src>
cudaError_t then_final(cudaError_t walk, bool closest, const SceneView& s, const rtk::W8View& v, const Src& src,
                       uint32_t n, cudaStream_t stream) {
  if (walk != cudaSuccess || !closest) return walk;
  return final_pass(s, v, src, n, stream);
}

bool view_of(const SceneView& s, rtk::W8View& v) {
  if (!s.wide8) return false;
  const uint32_t* base = static_cast<const uint32_t*>(s.wide8);
  v.nodes = reinterpret_cast<const uint4*>(base + s.w8_nodes_at);
  v.tris = reinterpret_cast<const uint4*>(base + s.w8_tris_at);
  v.inst = base + s.w8_inst_at;
  if (s.w8_top) {
    v.top = static_cast<const uint4*>(s.w8_top);
    v.top_items = static_cast<const uint32_t*>(s.w8_top) + s.w8_top_items_at;
    v.top_count = s.w8_top_nodes;
  }
  return true;
}

// Scenes with a top level set up each entered instance's triangle test lazily (at its first
// triangle: most entries of an instance-heavy scene end at the BLAS root's boxes); flat scenes,
// whose rays enter one or a few instances, set it up on entry.
template <bool COUNT, int SS, bool LAZY>
cudaError_t launch_one(const SceneView& s, const rtk::W8View& v, uint32_t mode, const rtk::OneBatch& src, uint32_t n,
                       unsigned int* counter, rtk::DevStatus* st, cudaStream_t stream, unsigned long long* cnt,
                       uint32_t refill) {
  using rtk::OneBatch;
  if (s.layout == 0) {
    return mode == 0 ? run(rtk::k_wide8<0, 0, W8_BLOCK, COUNT, OneBatch, SS, LAZY>, s.words, v, src, counter, n, st, stream, cnt, refill)
                     : run(rtk::k_wide8<0, 1, W8_BLOCK, COUNT, OneBatch, SS, LAZY>, s.words, v, src, counter, n, st, stream, cnt, refill);
  }
  return mode == 0 ? run(rtk::k_wide8<1, 0, W8_BLOCK, COUNT, OneBatch, SS, LAZY>, s.words, v, src, counter, n, st, stream, cnt, refill)
                   : run(rtk::k_wide8<1, 1, W8_BLOCK, COUNT, OneBatch, SS, LAZY>, s.words, v, src, counter, n, st, stream, cnt, refill);
}

template <bool COUNT, int SS>
cudaError_t launch_any(const SceneView& s, uint32_t mode, const float4* rays, const uint32_t* order, void* hits,
                       uint32_t n, unsigned int* counter, rtk::DevStatus* st, cudaStream_t stream,
                       unsigned long long* cnt, uint32_t refill) {
  if (n == 0) return cudaSuccess;
  rtk::W8View v;
  if (!view_of(s, v)) return cudaErrorInvalidValue;
  const rtk::OneBatch src{rays, order, hits};
  const cudaError_t e = s.top ? launch_one<COUNT, SS, true>(s, v, mode, src, n, counter, st, stream, cnt, refill)
                              : launch_one<COUNT, SS, false>(s, v, mode, src, n, counter, st, stream, cnt, refill);
  return then_final(e, mode == 0, s, v, src, n, stream);
}

bool shared_stack_fits(const SceneView& s) { return s.w8_depth <= rtk::W8_SSTACK; }

cudaError_t launch_wide8(const SceneView& s, uint32_t mode, const float4* rays, const uint32_t* order, void* hits,
                         uint32_t n, unsigned int* counter, rtk::DevStatus* st, cudaStream_t stream, uint32_t refill,
                         uint32_t stack) {
  if (stack == 0) return launch_any<false, 0>(s, mode, rays, order, hits, n, counter, st, stream, nullptr, refill);
  if (!shared_stack_fits(s)) return cudaErrorInvalidValue;
  return launch_any<false, (int)rtk::W8_SSTACK>(s, mode, rays, order, hits, n, counter, st, stream, nullptr, refill);
}

cudaError_t count_wide8(const SceneView& s, uint32_t mode, const float4* rays, void* hits, uint32_t n,
                        unsigned int* counter, rtk::DevStatus* st, unsigned long long* cnt, cudaStream_t stream) {
  return launch_any<true, 0>(s, mode, rays, nullptr, hits, n, counter, st, stream, cnt, 1);
}

cudaError_t launch_wide8_batches(const SceneView& s, const rtk::BatchEntry* table, uint32_t entries, uint32_t total,
                                 const uint32_t* order, unsigned int* counter, rtk::DevStatus* st, cudaStream_t stream,
                                 uint32_t refill, int uniform_mode, uint32_t stack) {
  if (total == 0) return cudaSuccess;
  rtk::W8View v;
  if (!view_of(s, v)) return cudaErrorInvalidValue;
  using rtk::ManyBatches;
  const ManyBatches src{table, entries, order};
#define RT_W8B(L, AM, SS)                                                                                         \
  (s.top ? run(rtk::k_wide8<L, AM, W8_BLOCK, false, ManyBatches, SS, true>, s.words, v, src, counter, total, st, stream, \
               nullptr, refill)                                                                                       \
         : run(rtk::k_wide8<L, AM, W8_BLOCK, false, ManyBatches, SS, false>, s.words, v, src, counter, total, st,       \
               stream, nullptr, refill))
  cudaError_t e;
  if (stack == 0) {
    if (s.layout == 0) e = uniform_mode == 0 ? RT_W8B(0, 0, 0) : (uniform_mode == 1 ? RT_W8B(0, 1, 0) : RT_W8B(0, 2, 0));
    else e = uniform_mode == 0 ? RT_W8B(1, 0, 0) : (uniform_mode == 1 ? RT_W8B(1, 1, 0) : RT_W8B(1, 2, 0));
  } else {
    if (!shared_stack_fits(s)) return cudaErrorInvalidValue;
    constexpr int SS = (int)rtk::W8_SSTACK;
    if (s.layout == 0) e = uniform_mode == 0 ? RT_W8B(0, 0, SS) : (uniform_mode == 1 ? RT_W8B(0, 1, SS) : RT_W8B(0, 2, SS));
    else e = uniform_mode == 0 ? RT_W8B(1, 0, SS) : (uniform_mode == 1 ? RT_W8B(1, 1, SS) : RT_W8B(1, 2, SS));
  }
#undef RT_W8B
  // an all any-hit launch has no closest hits to finish; a mixed one skips its any-hit entries
  return then_final(e, uniform_mode != 1, s, v, src, total, stream);
}

cudaError_t launch_wide8_lights(const SceneView& s, const void* cells, uint32_t n_cells, const void* lights,
                                uint32_t n_lights, uint32_t* words, unsigned int* counter, rtk::DevStatus* st,
                                cudaStream_t stream, uint32_t refill, uint32_t stack) {
  rtk::W8View v;
  if (s.layout != 0 || !view_of(s, v)) return cudaErrorInvalidValue;
  const uint32_t per_cell = (n_lights + 31) / 32, items = n_cells * n_lights;
  if (n_cells == 0 || n_lights == 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(words, 0, (size_t)n_cells * per_cell * sizeof(uint32_t), stream);
  if (e != cudaSuccess) return e;
  using rtk::LightRays;
  const LightRays src{static_cast<const rtk::GiCell*>(cells), static_cast<const rtk::GiLight*>(lights), n_lights, per_cell,
                      words};
  if (stack != 0 && !shared_stack_fits(s)) return cudaErrorInvalidValue;
  constexpr int SS = (int)rtk::W8_SSTACK;
  if (s.top) {
    return stack == 0 ? run(rtk::k_wide8<0, 1, W8_BLOCK, false, LightRays, 0, true>, s.words, v, src, counter, items, st, stream, nullptr, refill)
                      : run(rtk::k_wide8<0, 1, W8_BLOCK, false, LightRays, SS, true>, s.words, v, src, counter, items, st, stream, nullptr, refill);
  }
  return stack == 0 ? run(rtk::k_wide8<0, 1, W8_BLOCK, false, LightRays, 0, false>, s.words, v, src, counter, items, st, stream, nullptr, refill)
                    : run(rtk::k_wide8<0, 1, W8_BLOCK, false, LightRays, SS, false>, s.words, v, src, counter, items, st, stream, nullptr, refill);
}

namespace {
template <class K, class Src>
cudaError_t run_packet(K kernel, const uint32_t* words, const rtk::W8View& v, const Src& src, unsigned int* counter,
                       uint32_t n, rtk::DevStatus* st, cudaStream_t stream) {
  uint32_t full = 0;
  cudaError_t e = resident(kernel, full);
  if (e != cudaSuccess) return e;
  const uint32_t need = (n + W8_BLOCK - 1) / W8_BLOCK;
  if ((e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), stream)) != cudaSuccess) return e;
  kernel<<<need < full ? need : full, W8_BLOCK, 0, stream>>>(words, v, src, counter, n, st);
  return cudaGetLastError();
}
}  // namespace

cudaError_t launch_wide8_packet(const SceneView& s, uint32_t mode, const float4* rays, const uint32_t* order, void* hits,
                                uint32_t n, unsigned int* counter, rtk::DevStatus* st, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  rtk::W8View v;
  if (!view_of(s, v)) return cudaErrorInvalidValue;
  using rtk::OneBatch;
  const OneBatch src{rays, order, hits};
  cudaError_t e;
  if (s.layout == 0) {
    e = mode == 0 ? run_packet(rtk::k_wide8_packet<0, 0, W8_BLOCK, OneBatch>, s.words, v, src, counter, n, st, stream)
                  : run_packet(rtk::k_wide8_packet<0, 1, W8_BLOCK, OneBatch>, s.words, v, src, counter, n, st, stream);
  } else {
    e = mode == 0 ? run_packet(rtk::k_wide8_packet<1, 0, W8_BLOCK, OneBatch>, s.words, v, src, counter, n, st, stream)
                  : run_packet(rtk::k_wide8_packet<1, 1, W8_BLOCK, OneBatch>, s.words, v, src, counter, n, st, stream);
  }
  return e;  // the packet walk makes its closest hits' final values itself
}

cudaError_t launch_wide8_packet_batches(const SceneView& s, const rtk::BatchEntry* table, uint32_t entries,
                                        uint32_t total, const uint32_t* order, unsigned int* counter,
                                        rtk::DevStatus* st, cudaStream_t stream, int uniform_mode) {
  if (total == 0) return cudaSuccess;
  rtk::W8View v;
  if (!view_of(s, v)) return cudaErrorInvalidValue;
  using rtk::ManyBatches;
  const ManyBatches src{table, entries, order};
#define RT_W8P(L, AM) run_packet(rtk::k_wide8_packet<L, AM, W8_BLOCK, ManyBatches>, s.words, v, src, counter, total, st, stream)
  cudaError_t e;
  if (s.layout == 0) e = uniform_mode == 0 ? RT_W8P(0, 0) : (uniform_mode == 1 ? RT_W8P(0, 1) : RT_W8P(0, 2));
  else e = uniform_mode == 0 ? RT_W8P(1, 0) : (uniform_mode == 1 ? RT_W8P(1, 1) : RT_W8P(1, 2));
#undef RT_W8P
  return e;  // the packet walk makes its closest hits' final values itself
}

}  // namespace rtl
