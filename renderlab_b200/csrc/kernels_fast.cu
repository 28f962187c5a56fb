// Launchers for the FAST kernels: persistent grids sized to fill every SM once.
#include <cuda_runtime.h>

#include <map>
#include <mutex>

#include "kernels/cells.cuh"
#include "kernels/fast.cuh"
#include "launch.hpp"

namespace rtl {

namespace {
constexpr int FAST_BLOCK = 128;

// Resident blocks of `kernel` on the current device, cached per (kernel, device) under a lock:
// kernels of one signature share this template instance but can differ in registers, and
// rt_trace_static calls arrive from any thread without a context lock.
template <class K>
cudaError_t resident_blocks(K kernel, uint32_t& out) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, uint32_t> cached;
  int dev = 0, sms = 0, per_sm = 0;
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
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, FAST_BLOCK, 0)) != cudaSuccess) return e;
  out = (uint32_t)sms * (uint32_t)(per_sm > 0 ? per_sm : 1);
  std::lock_guard<std::mutex> lock(mu);
  cached[key] = out;
  return cudaSuccess;
}

template <class K>
cudaError_t grid_for(K kernel, uint32_t n, dim3& grid) {
  uint32_t full = 0;
  cudaError_t e = resident_blocks(kernel, full);
  if (e != cudaSuccess) return e;
  const uint32_t need = (n + FAST_BLOCK - 1) / FAST_BLOCK;
  grid = dim3(need < full ? need : full);
  return cudaSuccess;
}

template <class K, class Src>
cudaError_t run(K kernel, const SceneView& s, const Src& src, uint32_t n, unsigned int* counter, rtk::DevStatus* st,
                cudaStream_t stream, uint32_t refill) {
  dim3 grid;
  cudaError_t e = grid_for(kernel, n, grid);
  if (e != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), stream)) != cudaSuccess) return e;
  kernel<<<grid, FAST_BLOCK, 0, stream>>>(s.words, src, rtk::RayQueue{counter, n, refill}, st);
  return cudaGetLastError();
}
}  // namespace

cudaError_t launch_fast(const SceneView& s, uint32_t mode, const float4* rays, const uint32_t* order, void* hits,
                        uint32_t n, unsigned int* counter, rtk::DevStatus* st, cudaStream_t stream, uint32_t refill) {
  if (n == 0) return cudaSuccess;
  using rtk::OneBatch;
  const OneBatch src{rays, order, hits};
  if (s.layout == 0) {
    if (mode == 0) return run(rtk::k_gi_fast<0, FAST_BLOCK, OneBatch>, s, src, n, counter, st, stream, refill);
    return run(rtk::k_gi_fast<1, FAST_BLOCK, OneBatch>, s, src, n, counter, st, stream, refill);
  }
  if (mode == 0) return run(rtk::k_rs_fast<0, FAST_BLOCK, OneBatch>, s, src, n, counter, st, stream, refill);
  return run(rtk::k_rs_fast<1, FAST_BLOCK, OneBatch>, s, src, n, counter, st, stream, refill);
}

cudaError_t launch_fast_batches(const SceneView& s, const rtk::BatchEntry* table, uint32_t entries, uint32_t total,
                                const uint32_t* order, unsigned int* counter, rtk::DevStatus* st, cudaStream_t stream,
                                uint32_t refill, int uniform_mode) {
  if (total == 0) return cudaSuccess;
  using rtk::ManyBatches;
  const ManyBatches src{table, entries, order};
  if (s.layout == 0) {
    if (uniform_mode == 0) return run(rtk::k_gi_fast<0, FAST_BLOCK, ManyBatches>, s, src, total, counter, st, stream, refill);
    if (uniform_mode == 1) return run(rtk::k_gi_fast<1, FAST_BLOCK, ManyBatches>, s, src, total, counter, st, stream, refill);
    return run(rtk::k_gi_fast<2, FAST_BLOCK, ManyBatches>, s, src, total, counter, st, stream, refill);
  }
  if (uniform_mode == 0) return run(rtk::k_rs_fast<0, FAST_BLOCK, ManyBatches>, s, src, total, counter, st, stream, refill);
  if (uniform_mode == 1) return run(rtk::k_rs_fast<1, FAST_BLOCK, ManyBatches>, s, src, total, counter, st, stream, refill);
  return run(rtk::k_rs_fast<2, FAST_BLOCK, ManyBatches>, s, src, total, counter, st, stream, refill);
}

cudaError_t launch_fast_cells(const SceneView& s, uint32_t mode, const void* cells, uint32_t n_cells, uint32_t rotate,
                              void* hits, unsigned int* counter, rtk::DevStatus* st, cudaStream_t stream, uint32_t refill) {
  const uint32_t items = n_cells * rtk::GI_DIRECTIONS;
  if (items == 0) return cudaSuccess;
  if (s.layout != 0) return cudaErrorInvalidValue;
  using rtk::CellRays;
  const CellRays src{static_cast<const rtk::GiCell*>(cells), rotate, hits};
  if (mode == 0) return run(rtk::k_gi_fast<0, FAST_BLOCK, CellRays>, s, src, items, counter, st, stream, refill);
  return run(rtk::k_gi_fast<1, FAST_BLOCK, CellRays>, s, src, items, counter, st, stream, refill);
}

cudaError_t launch_fast_lights(const SceneView& s, const void* cells, uint32_t n_cells, const void* lights,
                               uint32_t n_lights, uint32_t* words, unsigned int* counter, rtk::DevStatus* st,
                               cudaStream_t stream, uint32_t refill) {
  if (s.layout != 0) return cudaErrorInvalidValue;
  const uint32_t per_cell = (n_lights + 31) / 32, items = n_cells * n_lights;
  if (n_cells == 0 || n_lights == 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(words, 0, (size_t)n_cells * per_cell * sizeof(uint32_t), stream);
  if (e != cudaSuccess) return e;
  using rtk::LightRays;
  const LightRays src{static_cast<const rtk::GiCell*>(cells), static_cast<const rtk::GiLight*>(lights), n_lights, per_cell,
                      words};
  return run(rtk::k_gi_fast<1, FAST_BLOCK, LightRays>, s, src, items, counter, st, stream, refill);
}

}  // namespace rtl
