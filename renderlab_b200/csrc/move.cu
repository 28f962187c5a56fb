// Moving the instances of an uploaded scene on the device: the records' rows and world boxes
// (the packers' arithmetic: gi_bvh.rs:230-274, reflection_software.rs:347-388), the top level
// refit over the new boxes as instance_bvh::place does for a moved set (instance_bvh.rs:162-275:
// refit, word 3 counting refits, a rebuild after 64, made on the device by tlas_build.cu), and
// the reflection layout's scene bounds
// (reflection_software.rs:295-313). Every float operation is an explicit round-to-nearest step in
// the host code's order, so the words equal rt_move_instances_host's, bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "ctx.hpp"
#include "kernels/common.cuh"

using namespace rtc;

namespace {

using rtk::EMPTY;
using rtk::LEAF;

constexpr size_t TOP_WORDS = 32;  // a top-level node: 24 box words, 4 child ids, 4 unused

struct Moved {  // one instance's new placement, as staged on the device
  float model[12], rows[12];
  uint32_t mesh, pad[3];
};

struct Box {
  float lo[3], hi[3];
};

__device__ __forceinline__ float lo_of(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float hi_of(float a, float b) { return b > a ? b : a; }
__device__ __forceinline__ Box empty_box() { return Box{{INFINITY, INFINITY, INFINITY}, {-INFINITY, -INFINITY, -INFINITY}}; }
__device__ __forceinline__ void grow(Box& b, const float* l, const float* h) {
  for (int a = 0; a < 3; ++a) b.lo[a] = lo_of(b.lo[a], l[a]), b.hi[a] = hi_of(b.hi[a], h[a]);
}

// pack.cpp's instance_box: the eight corners of the object box through the model (x, + y, + z,
// + w, rounded in turn), then the layout's margin.
__device__ Box instance_box(uint32_t layout, const float* m, const float* obj) {
  Box wb = empty_box();
  for (int c = 0; c < 8; ++c) {
    float p[3], w[3];
    for (int a = 0; a < 3; ++a) p[a] = (c >> a) & 1 ? obj[3 + a] : obj[a];
    for (int r = 0; r < 3; ++r) {
      float acc = __fmul_rn(m[4 * r], p[0]);
      acc = __fadd_rn(__fmul_rn(m[4 * r + 1], p[1]), acc);
      acc = __fadd_rn(__fmul_rn(m[4 * r + 2], p[2]), acc);
      w[r] = __fadd_rn(m[4 * r + 3], acc);
    }
    grow(wb, w, w);
  }
  Box out;
  if (layout == 0) {
    for (int a = 0; a < 3; ++a) {
      const float pad = __fmul_rn(1e-5f, __fadd_rn(1.0f, hi_of(fabsf(wb.lo[a]), fabsf(wb.hi[a]))));
      out.lo[a] = __fsub_rn(wb.lo[a], pad), out.hi[a] = __fadd_rn(wb.hi[a], pad);
    }
    return out;
  }
  float margin = 0.0f;
  for (int a = 0; a < 3; ++a)
    margin = hi_of(margin, hi_of(hi_of(fabsf(wb.hi[a]), fabsf(wb.lo[a])), __fsub_rn(wb.hi[a], wb.lo[a])));
  margin = __fmul_rn(margin, 1e-5f);
  for (int a = 0; a < 3; ++a) out.lo[a] = __fsub_rn(wb.lo[a], margin), out.hi[a] = __fadd_rn(wb.hi[a], margin);
  return out;
}

__global__ void k_move_records(uint32_t* __restrict__ w, uint32_t layout, const Moved* __restrict__ moved, uint32_t n,
                               const float* __restrict__ mesh_boxes) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Moved& g = moved[i];
  uint32_t* r = w + (layout == 0 ? 16 + 32 * (size_t)i : 8 + 24 * (size_t)i);
  for (int k = 0; k < 12; ++k) r[k] = __float_as_uint(g.rows[k]);
  const Box b = instance_box(layout, g.model, mesh_boxes + 6 * (size_t)g.mesh);
  for (int a = 0; a < 3; ++a) r[12 + a] = __float_as_uint(b.lo[a]), r[15 + a] = __float_as_uint(b.hi[a]);
}

// One height of the top level: each node's child boxes from its instances' records or from its
// inner children's (already refit) boxes, grown in slot order as instance_bvh::refit_wide does.
__global__ void k_refit_top(uint32_t* __restrict__ w, uint32_t layout, size_t base, const uint32_t* __restrict__ order,
                            uint32_t first, uint32_t count) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  uint32_t* node = w + base + TOP_WORDS * (size_t)order[first + k];
  for (int c = 0; c < 4; ++c) {
    const uint32_t id = node[24 + c];
    if (id == EMPTY) continue;
    Box b;
    if (id & LEAF) {
      const uint32_t* r = w + (layout == 0 ? 16 + 32 * (size_t)(id & ~LEAF) : 8 + 24 * (size_t)(id & ~LEAF));
      for (int a = 0; a < 3; ++a) b.lo[a] = __uint_as_float(r[12 + a]), b.hi[a] = __uint_as_float(r[15 + a]);
    } else {
      const uint32_t* child = w + base + TOP_WORDS * (size_t)id;
      b = empty_box();
      for (int cc = 0; cc < 4; ++cc) {
        if (child[24 + cc] == EMPTY) continue;
        float l[3], h[3];
        for (int a = 0; a < 3; ++a) l[a] = __uint_as_float(child[4 * a + cc]), h[a] = __uint_as_float(child[12 + 4 * a + cc]);
        grow(b, l, h);
      }
    }
    for (int a = 0; a < 3; ++a) node[4 * a + c] = __float_as_uint(b.lo[a]), node[12 + 4 * a + c] = __float_as_uint(b.hi[a]);
  }
}

// The reflection scene bounds: the instances' boxes grown in record order. Each thread grows a
// contiguous run, then thread 0 grows the runs in order; a strict comparison keeps the earlier of
// two equal values (+0 and -0), as one sequential pass does.
constexpr int BOUNDS_THREADS = 256;
__global__ void k_scene_bounds(uint32_t* __restrict__ w, uint32_t n) {
  __shared__ Box part[BOUNDS_THREADS];
  const uint32_t t = threadIdx.x, per = (n + BOUNDS_THREADS - 1) / BOUNDS_THREADS;
  Box b = empty_box();
  for (uint32_t i = t * per; i < n && i < (t + 1) * per; ++i) {
    const uint32_t* r = w + 8 + 24 * (size_t)i;
    float l[3], h[3];
    for (int a = 0; a < 3; ++a) l[a] = __uint_as_float(r[12 + a]), h[a] = __uint_as_float(r[15 + a]);
    grow(b, l, h);
  }
  part[t] = b;
  __syncthreads();
  if (t != 0) return;
  Box all = empty_box();
  for (int k = 0; k < BOUNDS_THREADS; ++k) grow(all, part[k].lo, part[k].hi);
  const size_t at = w[4];
  for (int a = 0; a < 3; ++a) w[at + a] = __float_as_uint(all.lo[a]), w[at + 4 + a] = __float_as_uint(all.hi[a]);
}

// The top level's nodes grouped by height above the instances (height 1 first).
void top_levels(const std::vector<uint32_t>& nodes, std::vector<uint32_t>& order, std::vector<uint32_t>& start) {
  const size_t nn = nodes.size() / TOP_WORDS;
  std::vector<uint32_t> height(nn, 0);
  for (size_t i = nn; i-- > 0;) {  // children follow their parents
    uint32_t h = 1;
    for (int c = 0; c < 4; ++c) {
      const uint32_t id = nodes[i * TOP_WORDS + 24 + c];
      if (id != EMPTY && !(id & LEAF) && id < nn) h = std::max(h, height[id] + 1);
    }
    height[i] = h;
  }
  // only the nodes reachable from the root (the reserve may hold unused space)
  std::vector<uint8_t> live(nn, 0);
  std::vector<uint32_t> stack{0};
  while (!stack.empty()) {
    const uint32_t i = stack.back();
    stack.pop_back();
    if (i >= nn || live[i]) continue;
    live[i] = 1;
    for (int c = 0; c < 4; ++c) {
      const uint32_t id = nodes[(size_t)i * TOP_WORDS + 24 + c];
      if (id != EMPTY && !(id & LEAF)) stack.push_back(id);
    }
  }
  const uint32_t top = nn ? height[0] : 0;
  order.clear();
  start.assign(1, 0);
  for (uint32_t h = 1; h <= top; ++h) {
    for (size_t i = 0; i < nn; ++i)
      if (live[i] && height[i] == h) order.push_back((uint32_t)i);
    start.push_back((uint32_t)order.size());
  }
}

}  // namespace

extern "C" rt_status rt_scene_move_instances(rt_ctx* ctx, rt_scene* scene, const rt_instance* instances, uint32_t n,
                                             const float* mesh_boxes, uint32_t n_meshes, void* stream) {
  if (!ctx || !scene || (n && !instances) || (n_meshes && !mesh_boxes)) return fail(ctx, RT_ERR_INVALID_ARG, "null argument");
  if (scene->layout > 1) return fail(ctx, RT_ERR_UNSUPPORTED, "instances move in the BVH4 layouts");
  const uint32_t layout = scene->layout;
  std::lock_guard<std::mutex> lock(ctx->mu);
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  uint32_t head[8];
  RT_CUDA(ctx, cudaMemcpy(head, scene->d_words, sizeof head, cudaMemcpyDeviceToHost));
  const uint32_t count = head[0];
  if (n != count || (layout == 0 && head[4] > count))  // GI word 4: a see-through tail
    return fail(ctx, RT_ERR_INVALID_ARG, "moved instances must be the scene's %u instances, in record order", count);
  std::vector<Moved> moved(n);
  std::vector<rtb::Placement> placed(n);
  for (uint32_t i = 0; i < n; ++i) {
    const rt_instance& s = instances[i];
    std::copy(s.model, s.model + 12, moved[i].model);
    std::copy(s.rows, s.rows + 12, moved[i].rows);
    moved[i].mesh = s.mesh;
    std::copy(s.model, s.model + 12, placed[i].model);
    std::copy(s.rows, s.rows + 12, placed[i].rows);
    placed[i].mesh = s.mesh;
    if (s.mesh >= n_meshes) return fail(ctx, RT_ERR_INVALID_ARG, "instance %u: mesh %u of %u", i, s.mesh, n_meshes);
    if (rtb::is_singular(placed[i])) return fail(ctx, RT_ERR_LAYOUT, "instance %u: singular placement", i);
  }
  if (n == 0) return RT_OK;
  scene->w8_top_valid = false;  // the instances move: the packed top level until re-prepared
  const size_t need = sizeof(Moved) * n + 24 * (size_t)n_meshes;
  if (need > scene->move_bytes) {
    RT_CUDA(ctx, cudaFree(scene->d_move));
    scene->d_move = nullptr;
    scene->device_bytes -= scene->move_bytes;
    ctx->scene_bytes -= scene->move_bytes;
    scene->move_bytes = 0;
    if (cudaMalloc(&scene->d_move, need) != cudaSuccess) {
      cudaGetLastError();
      return fail(ctx, RT_ERR_OOM, "move staging (%zu bytes)", need);
    }
    scene->move_bytes = need;
    scene->device_bytes += need;
    ctx->scene_bytes += need;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Moved* d_moved = static_cast<Moved*>(scene->d_move);
  float* d_boxes = reinterpret_cast<float*>(d_moved + n);
  RT_CUDA(ctx, cudaMemcpyAsync(d_moved, moved.data(), sizeof(Moved) * n, cudaMemcpyHostToDevice, s));
  RT_CUDA(ctx, cudaMemcpyAsync(d_boxes, mesh_boxes, 24 * (size_t)n_meshes, cudaMemcpyHostToDevice, s));
  k_move_records<<<(n + 127) / 128, 128, 0, s>>>(scene->d_words, layout, d_moved, n, d_boxes);
  RT_CUDA(ctx, cudaGetLastError());
  const size_t base = layout == 0 ? head[1] : (head[1] & ~3u);
  if (head[1] != 0 && count >= 2) {
    const size_t span = rtb::tlas_reserve(count);
    if (base + span > scene->n_words) return fail(ctx, RT_ERR_LAYOUT, "top level exceeds the scene's words");
    uint32_t refits = head[3];
    std::vector<uint32_t> nodes;
    if (refits >= rtb::TLAS_REFITS) {
      // Rebuilt on the device from the records' new boxes (instance_bvh::place for a moved set),
      // with the new tree's refit order.
      RT_CUDA(ctx, cudaFree(scene->d_top_order));
      scene->d_top_order = nullptr;
      scene->top_order.clear();
      if (cudaMalloc(&scene->d_top_order, 4 * (size_t)n) != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, RT_ERR_OOM, "top-level order");
      }
      const size_t header = layout == 0 ? 16 : 8, stride = layout == 0 ? 32 : 24;
      uint32_t n_nodes = 0;
      std::vector<uint32_t> starts;
      const rt_status st = tlas_build_device(ctx, scene->d_words + header + 12, stride, n, true, scene->d_words + base, span,
                                             scene->d_top_order, &starts, &n_nodes, s);
      if (st != RT_OK) return st;
      scene->top_order.resize(n_nodes);
      RT_CUDA(ctx, cudaMemcpy(scene->top_order.data(), scene->d_top_order, 4 * (size_t)n_nodes, cudaMemcpyDeviceToHost));
      scene->top_level_start = starts;
      refits = 0;
    } else {
      if (scene->top_order.empty()) {  // the tree's topology, once (and after every rebuild)
        nodes.resize(span);
        RT_CUDA(ctx, cudaMemcpyAsync(nodes.data(), scene->d_words + base, 4 * span, cudaMemcpyDeviceToHost, s));
        RT_CUDA(ctx, cudaStreamSynchronize(s));
        top_levels(nodes, scene->top_order, scene->top_level_start);
        RT_CUDA(ctx, cudaFree(scene->d_top_order));
        scene->d_top_order = nullptr;
        if (cudaMalloc(&scene->d_top_order, 4 * std::max<size_t>(1, scene->top_order.size())) != cudaSuccess) {
          cudaGetLastError();
          scene->top_order.clear();
          return fail(ctx, RT_ERR_OOM, "top-level order");
        }
        RT_CUDA(ctx, cudaMemcpy(scene->d_top_order, scene->top_order.data(), 4 * scene->top_order.size(),
                                cudaMemcpyHostToDevice));
      }
      const std::vector<uint32_t>& st = scene->top_level_start;
      for (size_t h = 0; h + 1 < st.size(); ++h) {
        const uint32_t first = st[h], cnt = st[h + 1] - st[h];
        if (!cnt) continue;
        k_refit_top<<<(cnt + 127) / 128, 128, 0, s>>>(scene->d_words, layout, base, scene->d_top_order, first, cnt);
        RT_CUDA(ctx, cudaGetLastError());
      }
      refits += 1;
    }
    RT_CUDA(ctx, cudaMemcpyAsync(scene->d_words + 3, &refits, 4, cudaMemcpyHostToDevice, s));
    RT_CUDA(ctx, cudaStreamSynchronize(s));  // `refits` is a local
  }
  if (layout == 1) {
    if ((size_t)head[4] + 8 > scene->n_words) return fail(ctx, RT_ERR_LAYOUT, "scene bounds exceed the words");
    k_scene_bounds<<<1, BOUNDS_THREADS, 0, s>>>(scene->d_words, n);
    RT_CUDA(ctx, cudaGetLastError());
  }
  return RT_OK;
}
