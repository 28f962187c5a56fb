// The BVH4-Q8 node quantiser on the device, shared by the GPU refit and the GPU build: child boxes
// formed as the host builder forms them (a leaf's vertices in index order; an inner child's
// decoded planes, unfused and fused, over its children in slot order) and quantize_node's exact
// arithmetic (near_field.rs:402-430, 481-525), every step an explicit round-to-nearest operation,
// so the node words equal the host's bit for bit.
#pragma once
#include <cuda_runtime.h>

#include <cfloat>
#include <cstddef>
#include <cstdint>

#include "common.cuh"

namespace rtq {

using rtk::EMPTY;
using rtk::LEAF;

struct Box {
  float lo[3], hi[3];
};

// f32::min / f32::max as the host builders write them (the first operand wins a tie).
__device__ __forceinline__ float lo_of(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float hi_of(float a, float b) { return b > a ? b : a; }
__device__ __forceinline__ void grow(Box& b, float x, float y, float z) {
  b.lo[0] = lo_of(b.lo[0], x), b.lo[1] = lo_of(b.lo[1], y), b.lo[2] = lo_of(b.lo[2], z);
  b.hi[0] = hi_of(b.hi[0], x), b.hi[1] = hi_of(b.hi[1], y), b.hi[2] = hi_of(b.hi[2], z);
}
__device__ __forceinline__ Box empty_box() { return Box{{INFINITY, INFINITY, INFINITY}, {-INFINITY, -INFINITY, -INFINITY}}; }
// A decoded plane, unfused (origin + step * q) or fused (fma).
__device__ __forceinline__ float plane(float o, float s, uint32_t q, bool fused) {
  return fused ? __fmaf_rn(s, (float)q, o) : __fadd_rn(o, __fmul_rn(s, (float)q));
}
__device__ __forceinline__ uint32_t to_u8(float f) {  // `f.clamp(0.0, 255.0) as u8`
  if (!(f > 0.0f)) return 0;
  if (f >= 255.0f) return 255;
  return (uint32_t)f;
}

struct View {
  uint32_t* w;
  uint32_t layout;
  size_t nodes, leaves, positions, indices;  // GI word offsets of the BLAS
  size_t tris;                               // reflection: its triangles
  const float* pos;                          // reflection: the new positions
  const uint32_t* src;                       // reflection: the source triangle list
};

__device__ __forceinline__ void grow_vertex(const View& v, Box& b, uint32_t vi, bool from_words) {
  if (from_words) {
    const uint32_t* p = v.w + v.positions + 3 * (size_t)vi;
    grow(b, __uint_as_float(p[0]), __uint_as_float(p[1]), __uint_as_float(p[2]));
  } else {
    const float* p = v.pos + 3 * (size_t)vi;
    grow(b, p[0], p[1], p[2]);
  }
}

// The box of one child, as the host refit forms it: a leaf's vertices in index order; an inner
// child's decoded planes, unfused and fused, over its children in slot order.
inline __device__ Box child_box(const View& v, uint32_t c) {
  Box b = empty_box();
  if (c & LEAF) {
    if (v.layout == 0) {
      const size_t l = v.leaves + 2 * (size_t)(c & ~LEAF);
      const uint32_t first = v.w[l], count = v.w[l + 1];
      for (uint32_t k = first; k < first + count; ++k) grow_vertex(v, b, v.w[v.indices + k], true);
    } else {
      const uint32_t first = (c & ~LEAF) >> 4, count = c & 15u;
      for (uint32_t t = first; t < first + count; ++t) {
        const uint32_t prim = v.w[v.tris + 12 * (size_t)t + 9];
        for (int j = 0; j < 3; ++j) grow_vertex(v, b, v.src[3 * (size_t)prim + j], false);
      }
    }
    return b;
  }
  const uint32_t* n = v.w + v.nodes + 16 * (size_t)c;
  for (int t = 0; t < 4; ++t) {
    if (n[6 + t] == EMPTY) continue;
    for (int fused = 0; fused < 2; ++fused)
      for (int a = 0; a < 3; ++a) {
        const float o = __uint_as_float(n[a]), s = __uint_as_float(n[3 + a]);
        b.lo[a] = lo_of(b.lo[a], plane(o, s, (n[10 + a] >> (8 * t)) & 255u, fused));
        b.hi[a] = hi_of(b.hi[a], plane(o, s, (n[13 + a] >> (8 * t)) & 255u, fused));
      }
  }
  return b;
}

// quantize_node: the node's origin and step per axis, then the outward 8-bit planes of each child.
inline __device__ void quantize(uint32_t* w, const uint32_t* kids, const Box* boxes, int n) {
  Box all = empty_box();
  for (int k = 0; k < n; ++k)
    for (int a = 0; a < 3; ++a) all.lo[a] = lo_of(all.lo[a], boxes[k].lo[a]), all.hi[a] = hi_of(all.hi[a], boxes[k].hi[a]);
  float step[3];
  for (int a = 0; a < 3; ++a) {
    const float lo = all.lo[a], hi = all.hi[a];
    float s = hi_of(__fdiv_rn(__fsub_rn(hi, lo), 255.0f), hi_of(FLT_MIN, __fmul_rn(fabsf(lo), 1e-7f)));
    while (__fadd_rn(lo, __fmul_rn(s, 255.0f)) < hi || __fmaf_rn(s, 255.0f, lo) < hi) s = __fmul_rn(s, 1.0f + 1.0f / 1048576.0f);
    step[a] = s;
  }
  uint32_t lower[3] = {0, 0, 0}, upper[3] = {0, 0, 0};
  for (int k = 0; k < n; ++k)
    for (int a = 0; a < 3; ++a) {
      const float o = all.lo[a], s = step[a], x = boxes[k].lo[a], y = boxes[k].hi[a];
      uint32_t ql = to_u8(floorf(__fdiv_rn(__fsub_rn(x, o), s)));
      while (ql > 0 && (plane(o, s, ql, false) > x || plane(o, s, ql, true) > x)) --ql;
      uint32_t qh = to_u8(ceilf(__fdiv_rn(__fsub_rn(y, o), s)));
      while (qh < 255 && (plane(o, s, qh, false) < y || plane(o, s, qh, true) < y)) ++qh;
      lower[a] |= ql << (8 * k);
      upper[a] |= qh << (8 * k);
    }
  for (int a = 0; a < 3; ++a) w[a] = __float_as_uint(all.lo[a]), w[3 + a] = __float_as_uint(step[a]);
  for (int s = 0; s < 4; ++s) w[6 + s] = s < n ? kids[s] : EMPTY;
  for (int a = 0; a < 3; ++a) w[10 + a] = lower[a], w[13 + a] = upper[a];
}

}  // namespace rtq
