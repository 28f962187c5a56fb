// The legacy reflection traversal over the median BVH2 layout (shaders/reflections_software.wgsl:
// 22-149), the reference's rollback path and the layout its geometry dumps carry
// (src/reflection_geometry_dump.rs, format "reflection-bvh2-u32-le"). One thread per ray, the
// WGSL statement for statement with the PLAIN kernels' arithmetic convention (every operation an
// explicit round-to-nearest step), 32-entry stacks whose overflowing pushes are dropped and
// counted.
//
// Layout: the reflection header and 24-word instance records; a BVH2 top level of 16-word nodes
// (two boxes lo/hi, children at words 12 and 13) at header word 1 (0: a flat instance list);
// BLAS nodes of the same 16-word form; leaves LEAF | first << 3 | count (count <= 7) over 12-word
// pre-edged triangles (a, e1, e2, primitive).
#pragma once
#include "plain.cuh"

namespace rtk {

constexpr uint32_t RS2_STACK = 32;

// legacy rs_limit (reflections_software.wgsl:38-40): only strictly lower instances win a tie
RT_DEV float rs2_limit(const RsBest& b, uint32_t i) { return (b.rec[0] != 0 && i < b.inst) ? next_up(b.t) : b.t; }

// legacy rs_instance (reflections_software.wgsl:43-110); true when an any-hit ray is blocked.
template <bool ANY>
RT_DEV bool rs2_instance(const uint32_t* __restrict__ w, uint32_t i, const Ray& ray, F3 world_inv, RsBest& best,
                         uint32_t* stack, DevStatus* st) {
  const size_t R = 8 + (size_t)i * 24;
  const uint32_t root = ld(w, R + 20), slot = ld(w, R + 21), noshadow = ld(w, R + 22);
  if (ANY && noshadow != 0) return false;
  const float bound = rs2_limit(best, i);
  if (slab_near(ray.o, world_inv, ld3(w, R + 12), ld3(w, R + 15), ray.tmin, bound) > bound) return false;
  const float r00 = ldf(w, R), r01 = ldf(w, R + 1), r02 = ldf(w, R + 2), r03 = ldf(w, R + 3);
  const float r10 = ldf(w, R + 4), r11 = ldf(w, R + 5), r12 = ldf(w, R + 6), r13 = ldf(w, R + 7);
  const float r20 = ldf(w, R + 8), r21 = ldf(w, R + 9), r22 = ldf(w, R + 10), r23 = ldf(w, R + 11);
  const F3 o = {dot4p(r00, r01, r02, r03, ray.o), dot4p(r10, r11, r12, r13, ray.o), dot4p(r20, r21, r22, r23, ray.o)};
  const F3 d = {dot3({r00, r01, r02}, ray.d), dot3({r10, r11, r12}, ray.d), dot3({r20, r21, r22}, ray.d)};
  const F3 inv = safe_inverse(d);
  const size_t nodes = ld(w, R + 18) & ~3u, tris = ld(w, R + 19) & ~3u;
  stack[0] = root;
  uint32_t sp = 1;
  while (sp > 0) {
    uint32_t child = stack[--sp];
    for (;;) {
      if (child & LEAF) {
        const uint32_t start = (child & ~LEAF) >> 3;
        for (uint32_t k = 0; k < (child & 7u); ++k) {
          const size_t X = tris + (size_t)(start + k) * 12;
          const F3 a = ld3(w, X), e1 = ld3(w, X + 3), e2 = ld3(w, X + 6);
          const F3 p = cross3(d, e2);
          const float det = dot3(e1, p);
          if (fabsf(det) < 1e-30f) continue;
          const float inv_det = __frcp_rn(det);
          const F3 s = sub3(o, a);
          const float u = mul(dot3(s, p), inv_det);
          if (u < -RS_EDGE || u > 1.0f + RS_EDGE) continue;
          const F3 q = cross3(s, e1);
          const float v = mul(dot3(d, q), inv_det);
          if (v < -RS_EDGE || add(u, v) > 1.0f + RS_EDGE) continue;
          const float t = mul(dot3(e2, q), inv_det);
          if (t > ray.tmin && t < rs2_limit(best, i)) {
            best.t = t;
            best.rec[0] = slot + 1, best.rec[1] = ld(w, X + 9), best.rec[2] = __float_as_uint(u);
            best.rec[3] = __float_as_uint(v);
            best.inst = i;
            if (ANY) return true;
          }
        }
        break;
      }
      const size_t N = nodes + (size_t)child * 16;
      const float lim = rs2_limit(best, i);
      const float t0 = slab_near(o, inv, ld3(w, N), ld3(w, N + 3), ray.tmin, lim);
      const float t1 = slab_near(o, inv, ld3(w, N + 6), ld3(w, N + 9), ray.tmin, lim);
      const uint32_t c0 = ld(w, N + 12), c1 = ld(w, N + 13);
      const bool h0 = t0 <= lim, h1 = t1 <= lim;
      if (h0 && h1) {
        const bool near_first = t0 <= t1;
        if (sp < RS2_STACK) stack[sp++] = near_first ? c1 : c0;
        else atomicAdd(&st->stack_drops, 1ull);
        child = near_first ? c0 : c1;
      } else if (h0) {
        child = c0;
      } else if (h1) {
        child = c1;
      } else {
        break;
      }
    }
  }
  return false;
}

// legacy rs_trace (reflections_software.wgsl:115-149)
template <bool ANY>
RT_DEV RsBest rs2_trace(const uint32_t* __restrict__ w, const Ray& ray, DevStatus* st) {
  RsBest best;
  best.t = ray.tmax, best.rec[0] = best.rec[1] = best.rec[2] = best.rec[3] = 0, best.inst = EMPTY;
  uint32_t stack[RS2_STACK];
  const F3 world_inv = safe_inverse(ray.d);
  const uint32_t count = ld(w, 0), top = ld(w, 1);
  if (top == 0) {
    for (uint32_t i = 0; i < count; ++i)
      if (rs2_instance<ANY>(w, i, ray, world_inv, best, stack, st)) return best;
    return best;
  }
  uint32_t nodes[RS2_STACK];
  nodes[0] = ld(w, 2);
  uint32_t sp = 1;
  while (sp > 0) {
    const uint32_t item = nodes[--sp];
    if (item & LEAF) {
      if (rs2_instance<ANY>(w, item & ~LEAF, ray, world_inv, best, stack, st)) return best;
      continue;
    }
    const size_t n = (top & ~3u) + (size_t)item * 16;
    const float bound = best.rec[0] != 0 ? next_up(best.t) : best.t;
    const float t0 = slab_near(ray.o, world_inv, ld3(w, n), ld3(w, n + 3), ray.tmin, bound);
    const float t1 = slab_near(ray.o, world_inv, ld3(w, n + 6), ld3(w, n + 9), ray.tmin, bound);
    const bool near = t0 <= t1;
    const float tf = near ? t1 : t0, tn = near ? t0 : t1;
    const uint32_t cf = near ? ld(w, n + 13) : ld(w, n + 12), cn = near ? ld(w, n + 12) : ld(w, n + 13);
    if (tf <= bound) {
      if (sp < RS2_STACK) nodes[sp++] = cf;
      else atomicAdd(&st->stack_drops, 1ull);
    }
    if (tn <= bound) {
      if (sp < RS2_STACK) nodes[sp++] = cn;
      else atomicAdd(&st->stack_drops, 1ull);
    }
  }
  return best;
}

template <bool ANY>
__global__ void __launch_bounds__(128) k_rs2_plain(const uint32_t* __restrict__ w, const float4* __restrict__ rays,
                                                   void* __restrict__ out, uint32_t n, DevStatus* st) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Ray ray = load_ray(rays, i);
  const RsBest b = rs2_trace<ANY>(w, ray, st);
  if (ANY) {
    reinterpret_cast<uint32_t*>(out)[i] = b.rec[0] != 0 ? 1u : 0u;
    return;
  }
  uint32_t* o = reinterpret_cast<uint32_t*>(out) + 5 * (size_t)i;
  o[0] = __float_as_uint(b.t), o[1] = b.rec[0], o[2] = b.rec[1], o[3] = b.rec[2], o[4] = b.rec[3];
}

}  // namespace rtk
