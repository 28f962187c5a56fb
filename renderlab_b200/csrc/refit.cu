// GPU refit of one BLAS of an uploaded scene (near_field::refit_bvh, near_field.rs:445-478, on the
// device): new positions for the same vertices, the BVH4-Q8 node boxes recomputed bottom-up and
// quantised with the host quantiser's exact arithmetic (quantize_node, near_field.rs:481-525), so
// the words equal those of rt_blas_refit followed by packing, bit for bit. Nodes of one height
// above the leaves are independent: one launch per height.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <vector>

#include "ctx.hpp"
#include "kernels/bvh4_quant.cuh"
#include "kernels/common.cuh"

using namespace rtc;

namespace {

using namespace rtq;

__global__ void k_refit_nodes(View v, const uint32_t* __restrict__ order, uint32_t count) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  uint32_t* w = v.w + v.nodes + 16 * (size_t)order[i];
  uint32_t kids[4];
  Box boxes[4];
  int m = 0;
  for (int s = 0; s < 4; ++s) {
    const uint32_t c = w[6 + s];
    if (c == EMPTY) continue;
    kids[m] = c;
    boxes[m] = child_box(v, c);
    ++m;
  }
  quantize(w, kids, boxes, m);
}

// GI: the new positions into the BLAS's position words.
__global__ void k_refit_positions(uint32_t* __restrict__ dst, const float* __restrict__ pos, uint32_t n_floats) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_floats) dst[i] = __float_as_uint(pos[i]);
}

// Reflection: each packed triangle's a, b - a, c - a from its primitive's vertices (the packer's
// arithmetic: one f32 subtraction a component).
__global__ void k_refit_triangles(View v, uint32_t n_tris) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_tris) return;
  uint32_t* x = v.w + v.tris + 12 * (size_t)t;
  const uint32_t prim = x[9];
  const float* a = v.pos + 3 * (size_t)v.src[3 * (size_t)prim];
  const float* b = v.pos + 3 * (size_t)v.src[3 * (size_t)prim + 1];
  const float* c = v.pos + 3 * (size_t)v.src[3 * (size_t)prim + 2];
  for (int j = 0; j < 3; ++j) {
    x[j] = __float_as_uint(a[j]);
    x[3 + j] = __float_as_uint(__fsub_rn(b[j], a[j]));
    x[6 + j] = __float_as_uint(__fsub_rn(c[j], a[j]));
  }
}

// The BLAS's topology (once per BLAS): node heights, triangle / position counts.
rt_status levels_of(rt_ctx* ctx, rt_scene* scene, const uint32_t* rec, RefitLevels& out) {
  const bool gi = scene->layout == 0;
  const size_t nodes = gi ? rec[18] : (rec[18] & ~3u);
  const uint32_t root = gi ? rec[22] : rec[20];
  if (root & LEAF) return RT_OK;  // a single leaf: nothing to refit
  const uint32_t n = root + 1;    // postorder: the root is the last node
  std::vector<uint32_t> w(16 * (size_t)n);
  RT_CUDA(ctx, cudaMemcpy(w.data(), scene->d_words + nodes, w.size() * 4, cudaMemcpyDeviceToHost));
  std::vector<uint32_t> height(n, 0);
  uint32_t top = 0, tris = 0, leaves_max = 0;
  for (uint32_t k = 0; k < n; ++k) {
    uint32_t h = 0;
    for (int s = 0; s < 4; ++s) {
      const uint32_t c = w[16 * (size_t)k + 6 + s];
      if (c == EMPTY) continue;
      if (c & LEAF) {
        if (gi) leaves_max = std::max(leaves_max, (c & ~LEAF) + 1);
        else tris = std::max(tris, ((c & ~LEAF) >> 4) + (c & 15u));
      } else if (c < k) {
        h = std::max(h, height[c]);
      } else {
        return fail(ctx, RT_ERR_LAYOUT, "refit: BLAS children must precede their parent");
      }
    }
    height[k] = h + 1;
    top = std::max(top, h + 1);
  }
  std::vector<uint32_t> order;
  order.reserve(n);
  out.level_start.assign(top + 1, 0);
  for (uint32_t h = 1; h <= top; ++h) {
    out.level_start[h - 1] = (uint32_t)order.size();
    for (uint32_t k = 0; k < n; ++k)
      if (height[k] == h) order.push_back(k);
  }
  out.level_start[top] = (uint32_t)order.size();
  out.node_count = n;
  out.tri_count = tris;
  (void)leaves_max;
  if (gi) {  // the packer lays a mesh's positions (3 words each) right before its indices
    if (rec[21] < rec[20] || (rec[21] - rec[20]) % 3 != 0) return fail(ctx, RT_ERR_LAYOUT, "refit: GI position words");
    out.position_count = (rec[21] - rec[20]) / 3;
  }
  if (cudaMalloc(&out.d_order, std::max<size_t>(order.size(), 1) * 4) != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, RT_ERR_OOM, "refit node order");
  }
  RT_CUDA(ctx, cudaMemcpy(out.d_order, order.data(), order.size() * 4, cudaMemcpyHostToDevice));
  return RT_OK;
}

}  // namespace

rt_status rt_scene_refit(rt_ctx* ctx, rt_scene* scene, uint32_t instance, const float* d_positions,
                         uint32_t n_positions, const uint32_t* d_indices, uint32_t n_indices, void* stream) {
  if (!ctx || !scene || !d_positions) return fail(ctx, RT_ERR_INVALID_ARG, "null argument");
  if (instance >= scene->info.instances) return fail(ctx, RT_ERR_INVALID_ARG, "no instance %u", instance);
  if (scene->layout == RT_LAYOUT_REFLECTION_BVH2)
    return fail(ctx, RT_ERR_UNSUPPORTED, "refit covers the BVH4 layouts (the legacy BVH2 one is rebuilt on the host)");
  const bool gi = scene->layout == 0;
  if (!gi && !d_indices) return fail(ctx, RT_ERR_INVALID_ARG, "the reflection layout refits from the triangle list");
  std::lock_guard<std::mutex> lock(ctx->mu);
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  uint32_t rec[24];
  const size_t r = gi ? 16 + 32 * (size_t)instance : 8 + 24 * (size_t)instance;
  RT_CUDA(ctx, cudaMemcpy(rec, scene->d_words + r, 24 * 4, cudaMemcpyDeviceToHost));
  const uint32_t base = gi ? rec[18] : (rec[18] & ~3u);
  auto it = scene->refit.find(base);
  if (it == scene->refit.end()) {
    RefitLevels lv;
    rt_status st = levels_of(ctx, scene, rec, lv);
    if (st != RT_OK) return st;
    it = scene->refit.emplace(base, std::move(lv)).first;
  }
  const RefitLevels& lv = it->second;
  if (gi && n_positions != lv.position_count)
    return fail(ctx, RT_ERR_INVALID_ARG, "the BLAS has %u positions, not %u", lv.position_count, n_positions);
  if (!gi && (size_t)n_indices < 3 * (size_t)lv.tri_count)
    return fail(ctx, RT_ERR_INVALID_ARG, "the triangle list is shorter than the BLAS's triangles");
  if (scene->d_wide8) {  // the derived 8-wide layout no longer matches: rt_scene_prepare again
    RT_CUDA(ctx, cudaFree(scene->d_wide8));
    scene->d_wide8 = nullptr;
    scene->device_bytes -= scene->wide8_bytes;
    ctx->scene_bytes -= scene->wide8_bytes;
    scene->wide8_bytes = 0;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  View v{};
  v.w = scene->d_words;
  v.layout = scene->layout;
  v.nodes = base;
  if (gi) {
    v.leaves = rec[19], v.positions = rec[20], v.indices = rec[21];
    const uint32_t nf = 3 * n_positions;
    if (nf) k_refit_positions<<<(nf + 255) / 256, 256, 0, s>>>(scene->d_words + v.positions, d_positions, nf);
  } else {
    v.tris = rec[19] & ~3u, v.pos = d_positions, v.src = d_indices;
    if (lv.tri_count) k_refit_triangles<<<(lv.tri_count + 255) / 256, 256, 0, s>>>(v, lv.tri_count);
  }
  RT_CUDA(ctx, cudaGetLastError());
  for (size_t h = 0; h + 1 < lv.level_start.size(); ++h) {
    const uint32_t a = lv.level_start[h], n = lv.level_start[h + 1] - a;
    if (n) k_refit_nodes<<<(n + 127) / 128, 128, 0, s>>>(v, lv.d_order + a, n);
  }
  RT_CUDA(ctx, cudaGetLastError());
  return RT_OK;
}

rt_status rt_scene_read_words(rt_ctx* ctx, const rt_scene* scene, size_t first, size_t n, uint32_t* out) {
  if (!ctx || !scene || (n && !out)) return fail(ctx, RT_ERR_INVALID_ARG, "null argument");
  if (first > scene->n_words || n > scene->n_words - first) return fail(ctx, RT_ERR_INVALID_ARG, "words out of range");
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  if (n) RT_CUDA(ctx, cudaMemcpy(out, scene->d_words + first, n * 4, cudaMemcpyDeviceToHost));
  return RT_OK;
}
