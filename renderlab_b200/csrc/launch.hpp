// Internal launcher interface between the C ABI (rt_api.cu) and the kernel translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels/common.cuh"

namespace rtl {

struct SceneView {
  uint32_t layout;        // 0 GI, 1 reflection
  const uint32_t* words;  // device words
  size_t n_words;
  uint32_t instances;
  uint32_t top;
  // Derived 8-wide layout for the WIDE8 kernel (null until rt_scene_prepare): one device
  // allocation holding nodes, triangles and the per-instance table at these word offsets.
  const void* wide8;
  size_t wide8_bytes;
  size_t w8_nodes_at, w8_tris_at, w8_inst_at;
  uint32_t w8_depth;  // levels of the deepest 8-wide BLAS
  // The 8-wide top level (null: walk the packed top level): w8_top_nodes 80-byte nodes, breadth
  // first from the root, then the leaves' entries (instance, BLAS node below the instance's root)
  // at word w8_top_items_at.
  const void* w8_top = nullptr;
  uint32_t w8_top_nodes = 0;
  size_t w8_top_items_at = 0;
};

// PLAIN: mode 0 closest, 1/2 any-hit. Hits as documented in rt_trace.h.
cudaError_t launch_plain(const SceneView& s, uint32_t mode, const float4* rays, void* hits, uint32_t n,
                         rtk::DevStatus* st, cudaStream_t stream);
// FAST: bit-exact with PLAIN; `order` (optional) permutes which ray each thread traces.
// `counter` is a device word the launch owns until it completes (zeroed on `stream`).
cudaError_t launch_fast(const SceneView& s, uint32_t mode, const float4* rays, const uint32_t* order, void* hits,
                        uint32_t n, unsigned int* counter, rtk::DevStatus* st, cudaStream_t stream, uint32_t refill);
// WIDE8: the precision variant over the scene's derived 8-wide layout.
// `refill`: idle lanes (1-32) a warp waits for before it takes more rays. `stack`: 0 keeps each
// lane's node-group stack in local memory (32 entries), 1 in shared memory (16 entries: only for
// scenes whose 8-wide trees are at most 16 levels deep, else cudaErrorInvalidValue).
cudaError_t launch_wide8(const SceneView& s, uint32_t mode, const float4* rays, const uint32_t* order, void* hits,
                         uint32_t n, unsigned int* counter, rtk::DevStatus* st, cudaStream_t stream, uint32_t refill,
                         uint32_t stack);
bool shared_stack_fits(const SceneView& s);
// Many batches in one persistent launch: `table` (device, `entries` records sorted by `first`)
// covers `total` rays; `order` (optional) permutes the launch's ray space. Mode per entry;
// `uniform_mode` 0 / 1 when every non-empty entry is closest / any hit (a kernel with the mode
// fixed), -1 for a mix.
cudaError_t launch_fast_batches(const SceneView& s, const rtk::BatchEntry* table, uint32_t entries, uint32_t total,
                                const uint32_t* order, unsigned int* counter, rtk::DevStatus* st, cudaStream_t stream,
                                uint32_t refill, int uniform_mode);
cudaError_t launch_wide8_batches(const SceneView& s, const rtk::BatchEntry* table, uint32_t entries, uint32_t total,
                                 const uint32_t* order, unsigned int* counter, rtk::DevStatus* st, cudaStream_t stream,
                                 uint32_t refill, int uniform_mode, uint32_t stack);
// WIDE8 with per-event device counters (rtk::W8Count order) accumulated into cnt[8].
cudaError_t count_wide8(const SceneView& s, uint32_t mode, const float4* rays, void* hits, uint32_t n,
                        unsigned int* counter, rtk::DevStatus* st, unsigned long long* cnt, cudaStream_t stream);
// WIDE8 walked by warp-wide packets of 32 consecutive rays (top level or flat instance list); the
// same results as launch_wide8.
cudaError_t launch_wide8_packet(const SceneView& s, uint32_t mode, const float4* rays, const uint32_t* order, void* hits,
                                uint32_t n, unsigned int* counter, rtk::DevStatus* st, cudaStream_t stream);
cudaError_t launch_wide8_packet_batches(const SceneView& s, const rtk::BatchEntry* table, uint32_t entries,
                                        uint32_t total, const uint32_t* order, unsigned int* counter,
                                        rtk::DevStatus* st, cudaStream_t stream, int uniform_mode);
// The GI cache's cell ray producers (kernels/cells.cuh): 64 rays a cell written to `rays`
// (kernels_cells.cu), or generated inside the FAST GI kernel and traced (mode 0 closest, else sky
// any hit), results at the item index (kernels_fast.cu).
cudaError_t launch_cell_rays(const void* cells, uint32_t n_cells, uint32_t rotate, float4* rays, cudaStream_t stream);
cudaError_t launch_fast_cells(const SceneView& s, uint32_t mode, const void* cells, uint32_t n_cells, uint32_t rotate,
                              void* hits, unsigned int* counter, rtk::DevStatus* st, cudaStream_t stream, uint32_t refill);
// The GI cache's per-light visibility (gi_light): item c * n_lights + l is cell c's ray toward
// light l, traced any-hit (FAST or WIDE8, generated in the ray refill), results packed into
// ceil(n_lights / 32) words a cell at `words` (zeroed on `stream` first).
cudaError_t launch_fast_lights(const SceneView& s, const void* cells, uint32_t n_cells, const void* lights,
                               uint32_t n_lights, uint32_t* words, unsigned int* counter, rtk::DevStatus* st,
                               cudaStream_t stream, uint32_t refill);
cudaError_t launch_wide8_lights(const SceneView& s, const void* cells, uint32_t n_cells, const void* lights,
                                uint32_t n_lights, uint32_t* words, unsigned int* counter, rtk::DevStatus* st,
                                cudaStream_t stream, uint32_t refill, uint32_t stack);
// Ray ordering (kernels_order.cu): scratch holds the keys, the unsorted indices and the radix
// sort's temporary storage.
size_t order_scratch_bytes(uint32_t n);
cudaError_t launch_order(const float4* rays, uint32_t n, const float lo[3], const float hi[3], uint32_t kind,
                         uint32_t* order, void* scratch, size_t scratch_bytes, cudaStream_t stream);
// The same over a many-batch launch's ray space (its batch table).
cudaError_t launch_order_batches(const rtk::BatchEntry* table, uint32_t entries, uint32_t total, const float lo[3],
                                 const float hi[3], uint32_t kind, uint32_t* order, void* scratch, size_t scratch_bytes,
                                 cudaStream_t stream);
cudaError_t launch_selftest(uint32_t* out16, cudaStream_t stream);

}  // namespace rtl
