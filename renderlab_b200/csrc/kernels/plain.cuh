// PLAIN traversal kernels: one thread per ray, a 48-entry stack per thread, the WGSL loops
// statement for statement:
//   gi_traverse  -> shaders/gi_rays_software.wgsl:98-279 (opaque instances, BVH4 top level)
//   rs_trace     -> shaders/reflections_software_bvh4.wgsl:50-204
// Same arithmetic, same child order, same tie rules, so hits are bit-identical to the WGSL
// restatement. Two safety rules the WGSL leaves to robust buffer access: a child id EMPTY is
// never pushed, and a push onto a full stack is dropped and counted (DevStatus::stack_drops).
#pragma once
#include "common.cuh"

namespace rtk {

// ---------------------------------------------------------------- GI layout

struct GiBest {
  bool hit;
  float t;
  F3 n;
  uint32_t inst;
  uint32_t tri[3];
  float u, v;
};

// gi_limit (gi_rays_software.wgsl:68-70)
RT_DEV float gi_limit(const GiBest& b, uint32_t i) { return (b.hit && i < b.inst) ? next_up(b.t) : b.t; }

// gi_triangle (gi_rays_software.wgsl:42-58): true with (t, u, v) inside (tmin, tmax)
RT_DEV bool gi_triangle(F3 o, F3 d, F3 a, F3 b, F3 c, float tmin, float tmax, float& t, float& u, float& v) {
  F3 e1 = sub3(b, a), e2 = sub3(c, a);
  F3 p = cross3(d, e2);
  float det = dot3(e1, p);
  if (fabsf(det) < 1e-30f) return false;
  float inv = __frcp_rn(det);
  F3 s = sub3(o, a);
  u = mul(dot3(s, p), inv);
  if (u < 0.0f || u > 1.0f) return false;
  F3 q = cross3(s, e1);
  v = mul(dot3(d, q), inv);
  if (v < 0.0f || add(u, v) > 1.0f) return false;
  t = mul(dot3(e2, q), inv);
  return t > tmin && t < tmax;
}

// unit_normal (shaders/scene.wgsl:86-90) with inverseSqrt as a correctly rounded 1/sqrt.
RT_DEV F3 unit_normal(F3 n) {
  float m = fmaxf(fmaxf(fmaxf(fabsf(n.x), fabsf(n.y)), fabsf(n.z)), 1e-30f);
  F3 s = {__fdiv_rn(n.x, m), __fdiv_rn(n.y, m), __fdiv_rn(n.z, m)};
  float k = __frcp_rn(__fsqrt_rn(fmaxf(dot3(s, s), 1e-30f)));
  return {mul(s.x, k), mul(s.y, k), mul(s.z, k)};
}

// gi_instance (gi_rays_software.wgsl:98-207), opaque mode.
template <bool ANY>
RT_DEV bool gi_instance(const uint32_t* __restrict__ w, uint32_t i, const Ray& ray, F3 world_inv, GiBest& best,
                        uint32_t* stack, DevStatus* st) {
  const size_t r = 16 + (size_t)i * 32;
  if (ANY && (ld(w, r + 27) & 1u) != 0) return false;
  {
    float lim = gi_limit(best, i);
    if (!(slab_near(ray.o, world_inv, ld3(w, r + 12), ld3(w, r + 15), ray.tmin, lim) <= lim)) return false;
  }
  const float r00 = ldf(w, r), r01 = ldf(w, r + 1), r02 = ldf(w, r + 2), r03 = ldf(w, r + 3);
  const float r10 = ldf(w, r + 4), r11 = ldf(w, r + 5), r12 = ldf(w, r + 6), r13 = ldf(w, r + 7);
  const float r20 = ldf(w, r + 8), r21 = ldf(w, r + 9), r22 = ldf(w, r + 10), r23 = ldf(w, r + 11);
  const F3 o = {dot4p(r00, r01, r02, r03, ray.o), dot4p(r10, r11, r12, r13, ray.o), dot4p(r20, r21, r22, r23, ray.o)};
  const F3 d = {dot3({r00, r01, r02}, ray.d), dot3({r10, r11, r12}, ray.d), dot3({r20, r21, r22}, ray.d)};
  const F3 inv = safe_inverse(d);
  const uint32_t nodes = ld(w, r + 18), leaves = ld(w, r + 19), positions = ld(w, r + 20), indices = ld(w, r + 21);
  const uint32_t prim_base = ld(w, r + 28);
  auto normal_of = [&](F3 a, F3 b, F3 c) {
    F3 cr = cross3(sub3(b, a), sub3(c, a));
    F3 n = {add(add(mul(r00, cr.x), mul(r10, cr.y)), mul(r20, cr.z)),
            add(add(mul(r01, cr.x), mul(r11, cr.y)), mul(r21, cr.z)),
            add(add(mul(r02, cr.x), mul(r12, cr.y)), mul(r22, cr.z))};
    return unit_normal(n);
  };
  stack[0] = ld(w, r + 22);
  uint32_t sp = 1;
  while (sp > 0) {
    sp -= 1;
    const uint32_t child = stack[sp];
    if (child & LEAF) {
      const size_t l = leaves + (size_t)(child & ~LEAF) * 2;
      const uint32_t first = ld(w, l), count = ld(w, l + 1);
      for (uint32_t k = 0; k < count; k += 6) {
        const size_t x = (size_t)indices + first + k;
        const bool two = k + 3 < count;
        const size_t y = two ? x + 3 : x;
        const uint32_t ia = ld(w, x), ib = ld(w, x + 1), ic = ld(w, x + 2);
        const uint32_t ja = ld(w, y), jb = ld(w, y + 1), jc = ld(w, y + 2);
        const F3 a = ld3(w, positions + (size_t)ia * 3), b = ld3(w, positions + (size_t)ib * 3),
                 c = ld3(w, positions + (size_t)ic * 3);
        const F3 a2 = ld3(w, positions + (size_t)ja * 3), b2 = ld3(w, positions + (size_t)jb * 3),
                 c2 = ld3(w, positions + (size_t)jc * 3);
        float t, u, v;
        if (gi_triangle(o, d, a, b, c, ray.tmin, gi_limit(best, i), t, u, v)) {
          best.hit = true, best.t = t, best.inst = i, best.u = u, best.v = v;
          if (ANY) return true;
          best.n = normal_of(a, b, c);
          if (prim_base != 0) best.tri[0] = ld(w, prim_base + (first + k) / 3), best.tri[1] = 0, best.tri[2] = 0;
          else best.tri[0] = ia, best.tri[1] = ib, best.tri[2] = ic;
        }
        if (two && gi_triangle(o, d, a2, b2, c2, ray.tmin, gi_limit(best, i), t, u, v)) {
          best.hit = true, best.t = t, best.inst = i, best.u = u, best.v = v;
          if (ANY) return true;
          best.n = normal_of(a2, b2, c2);
          if (prim_base != 0) best.tri[0] = ld(w, prim_base + (first + k) / 3 + 1), best.tri[1] = 0, best.tri[2] = 0;
          else best.tri[0] = ja, best.tri[1] = jb, best.tri[2] = jc;
        }
      }
      continue;
    }
    const size_t n = nodes + (size_t)child * 16;
    const F3 oq = ld3(w, n), step = ld3(w, n + 3);
    uint32_t c[4] = {ld(w, n + 6), ld(w, n + 7), ld(w, n + 8), ld(w, n + 9)};
    const uint32_t lx = ld(w, n + 10), ly = ld(w, n + 11), lz = ld(w, n + 12);
    const uint32_t hx = ld(w, n + 13), hy = ld(w, n + 14), hz = ld(w, n + 15);
    uint32_t tb[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      tb[s] = __float_as_uint(BIG);
      if (c[s] == EMPTY) continue;
      const uint32_t sh = 8 * s;
      const F3 lo = {add(oq.x, mul(step.x, (float)((lx >> sh) & 0xffu))), add(oq.y, mul(step.y, (float)((ly >> sh) & 0xffu))),
                     add(oq.z, mul(step.z, (float)((lz >> sh) & 0xffu)))};
      const F3 hi = {add(oq.x, mul(step.x, (float)((hx >> sh) & 0xffu))), add(oq.y, mul(step.y, (float)((hy >> sh) & 0xffu))),
                     add(oq.z, mul(step.z, (float)((hz >> sh) & 0xffu)))};
      tb[s] = __float_as_uint(slab_near(o, inv, lo, hi, ray.tmin, gi_limit(best, i)));
    }
    // (distance bits, child), descending: gi_rays_software.wgsl:191-197
#define RT_SW(a, b)                          \
  if (tb[a] < tb[b]) {                       \
    uint32_t x = tb[a]; tb[a] = tb[b]; tb[b] = x; \
    x = c[a]; c[a] = c[b]; c[b] = x;         \
  }
    RT_SW(0, 1) RT_SW(2, 3) RT_SW(0, 2) RT_SW(1, 3) RT_SW(1, 2)
#undef RT_SW
    const float lim = gi_limit(best, i);
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      if (__uint_as_float(tb[s]) <= lim && c[s] != EMPTY) {
        if (sp < STACK) stack[sp++] = c[s];
        else atomicAdd(&st->stack_drops, 1ull);
      }
    }
  }
  return false;
}

// The BVH4 top-level node step (gi_rays_software.wgsl:241-261, reflections_software_bvh4.wgsl
// :173-193): four slabs, the ascending five-exchange network, pushes far to near.
RT_DEV void top_step(const uint32_t* __restrict__ w, size_t n, const Ray& ray, F3 world_inv, float bound,
                     uint32_t* stack, uint32_t& sp, DevStatus* st) {
  float dist[4];
  uint32_t ids[4];
  // the node's seven 16-byte rows: lo x, lo y, lo z, hi x, hi y, hi z (four children each), ids
  const uint4 lx = ld4u(w, n), ly = ld4u(w, n + 4), lz = ld4u(w, n + 8);
  const uint4 hx = ld4u(w, n + 12), hy = ld4u(w, n + 16), hz = ld4u(w, n + 20), id4 = ld4u(w, n + 24);
  auto at = [](const uint4& q, int c) { return c == 0 ? q.x : (c == 1 ? q.y : (c == 2 ? q.z : q.w)); };
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const float ax = mul(sub(__uint_as_float(at(lx, c)), ray.o.x), world_inv.x),
                bx = mul(sub(__uint_as_float(at(hx, c)), ray.o.x), world_inv.x);
    const float ay = mul(sub(__uint_as_float(at(ly, c)), ray.o.y), world_inv.y),
                by = mul(sub(__uint_as_float(at(hy, c)), ray.o.y), world_inv.y);
    const float az = mul(sub(__uint_as_float(at(lz, c)), ray.o.z), world_inv.z),
                bz = mul(sub(__uint_as_float(at(hz, c)), ray.o.z), world_inv.z);
    const float near = fmaxf(fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fminf(az, bz)), ray.tmin);
    const float far = fminf(fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fmaxf(az, bz)), bound);
    ids[c] = at(id4, c);
    dist[c] = (near <= far && ids[c] != EMPTY) ? near : BIG;
  }
#define RT_SW(a, b)                                      \
  if (dist[b] < dist[a]) {                               \
    float x = dist[a]; dist[a] = dist[b]; dist[b] = x;   \
    uint32_t y = ids[a]; ids[a] = ids[b]; ids[b] = y;    \
  }
  RT_SW(0, 1) RT_SW(2, 3) RT_SW(0, 2) RT_SW(1, 3) RT_SW(1, 2)
#undef RT_SW
#pragma unroll
  for (int c = 3; c >= 0; --c) {
    if (dist[c] <= bound && ids[c] != EMPTY) {
      if (sp < STACK) stack[sp++] = ids[c];
      else atomicAdd(&st->stack_drops, 1ull);
    }
  }
}

// gi_traverse (gi_rays_software.wgsl:217-279)
template <bool ANY>
RT_DEV GiBest gi_traverse(const uint32_t* __restrict__ w, const Ray& ray, DevStatus* st) {
  GiBest best;
  best.hit = false, best.t = ray.tmax, best.n = {0.0f, 0.0f, 0.0f}, best.inst = EMPTY;
  best.tri[0] = best.tri[1] = best.tri[2] = 0, best.u = best.v = 0.0f;
  uint32_t stack[STACK];
  const F3 world_inv = safe_inverse(ray.d);
  const uint32_t instances = ld(w, 0), top = ld(w, 1);
  if (top == 0) {
    for (uint32_t i = 0; i < instances; ++i)
      if (gi_instance<ANY>(w, i, ray, world_inv, best, stack, st)) return best;
    return best;
  }
  uint32_t nodes[STACK];
  nodes[0] = ld(w, 2);
  uint32_t sp = 1;
  while (sp > 0) {
    sp -= 1;
    const uint32_t item = nodes[sp];
    if (item & LEAF) {
      if (gi_instance<ANY>(w, item & ~LEAF, ray, world_inv, best, stack, st)) return best;
      continue;
    }
    const float bound = best.hit ? next_up(best.t) : best.t;
    top_step(w, top + (size_t)item * 32, ray, world_inv, bound, nodes, sp, st);
  }
  return best;
}

template <uint32_t MODE>
__global__ void __launch_bounds__(128) k_gi_plain(const uint32_t* __restrict__ w, const float4* __restrict__ rays,
                                                  void* __restrict__ out, uint32_t n, DevStatus* st) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Ray ray = load_ray(rays, i);
  const GiBest b = gi_traverse<MODE != 0>(w, ray, st);
  if (MODE != 0) {
    reinterpret_cast<uint32_t*>(out)[i] = b.hit ? 1u : 0u;
    return;
  }
  uint32_t* o = reinterpret_cast<uint32_t*>(out) + 10 * (size_t)i;
  o[0] = __float_as_uint(b.t), o[1] = b.inst, o[2] = b.tri[0], o[3] = b.tri[1], o[4] = b.tri[2];
  o[5] = __float_as_uint(b.u), o[6] = __float_as_uint(b.v);
  o[7] = __float_as_uint(b.n.x), o[8] = __float_as_uint(b.n.y), o[9] = __float_as_uint(b.n.z);
}

// ---------------------------------------------------------------- reflection layout

constexpr float RS_EDGE = 4e-6f;

struct RsBest {
  float t;
  uint32_t rec[4];
  uint32_t inst;
};

// rs_limit (reflections_software_bvh4.wgsl:45-47)
RT_DEV float rs_limit(const RsBest& b, uint32_t i) { return (b.rec[0] != 0 && i <= b.inst) ? next_up(b.t) : b.t; }

// rs_instance (reflections_software_bvh4.wgsl:50-130)
template <bool ANY>
RT_DEV bool rs_instance(const uint32_t* __restrict__ w, uint32_t i, const Ray& ray, F3 world_inv, RsBest& best,
                        uint32_t* stack, DevStatus* st) {
  const size_t R = 8 + (size_t)i * 24;
  const uint4 tail = ld4(w, R + 20);  // root, slot, casts no shadow, 0
  if (ANY && tail.z != 0) return false;
  const uint4 b0 = ld4(w, R + 12), b1 = ld4(w, R + 16);
  {
    const float bound = rs_limit(best, i);
    const F3 lo = {__uint_as_float(b0.x), __uint_as_float(b0.y), __uint_as_float(b0.z)};
    const F3 hi = {__uint_as_float(b0.w), __uint_as_float(b1.x), __uint_as_float(b1.y)};
    if (slab_near(ray.o, world_inv, lo, hi, ray.tmin, bound) > bound) return false;
  }
  const uint4 q0 = ld4(w, R), q1 = ld4(w, R + 4), q2 = ld4(w, R + 8);
  const float r00 = __uint_as_float(q0.x), r01 = __uint_as_float(q0.y), r02 = __uint_as_float(q0.z), r03 = __uint_as_float(q0.w);
  const float r10 = __uint_as_float(q1.x), r11 = __uint_as_float(q1.y), r12 = __uint_as_float(q1.z), r13 = __uint_as_float(q1.w);
  const float r20 = __uint_as_float(q2.x), r21 = __uint_as_float(q2.y), r22 = __uint_as_float(q2.z), r23 = __uint_as_float(q2.w);
  const F3 o = {dot4p(r00, r01, r02, r03, ray.o), dot4p(r10, r11, r12, r13, ray.o), dot4p(r20, r21, r22, r23, ray.o)};
  const F3 d = {dot3({r00, r01, r02}, ray.d), dot3({r10, r11, r12}, ray.d), dot3({r20, r21, r22}, ray.d)};
  const F3 inv = safe_inverse(d);
  const size_t nodes = b1.z & ~3u, tris = b1.w & ~3u;
  const uint32_t slot = tail.y;
  stack[0] = tail.x;
  uint32_t sp = 1;
  while (sp > 0) {
    sp -= 1;
    uint32_t child = stack[sp];
    for (;;) {
      if (child & LEAF) {
        const uint32_t start = (child & ~LEAF) >> 4;
        for (uint32_t k = 0; k < (child & 15u); ++k) {
          const size_t X = tris + (size_t)(start + k) * 12;
          const uint4 w0 = ld4u(w, X), w1 = ld4u(w, X + 4), w2 = ld4u(w, X + 8);
          const F3 a = {__uint_as_float(w0.x), __uint_as_float(w0.y), __uint_as_float(w0.z)};
          const F3 e1 = {__uint_as_float(w0.w), __uint_as_float(w1.x), __uint_as_float(w1.y)};
          const F3 e2 = {__uint_as_float(w1.z), __uint_as_float(w1.w), __uint_as_float(w2.x)};
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
          const bool tied = best.rec[0] != 0 && t == best.t && (i < best.inst || (i == best.inst && w2.y < best.rec[1]));
          if (t > ray.tmin && (t < best.t || tied)) {
            best.t = t;
            best.rec[0] = slot + 1, best.rec[1] = w2.y, best.rec[2] = __float_as_uint(u), best.rec[3] = __float_as_uint(v);
            best.inst = i;
            if (ANY) return true;
          }
        }
        break;
      }
      const size_t N = nodes + (size_t)child * 16;
      const uint4 n0 = ld4u(w, N), n1 = ld4u(w, N + 4), n2 = ld4u(w, N + 8), n3 = ld4u(w, N + 12);
      const float lim = rs_limit(best, i);
      const F3 base = {__uint_as_float(n0.x), __uint_as_float(n0.y), __uint_as_float(n0.z)};
      const F3 step = {__uint_as_float(n0.w), __uint_as_float(n1.x), __uint_as_float(n1.y)};
      uint32_t ids[4] = {n1.z, n1.w, n2.x, n2.y};
      const uint32_t lower[3] = {n2.z, n2.w, n3.x}, upper[3] = {n3.y, n3.z, n3.w};
      float dist[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        dist[c] = BIG;
        if (ids[c] == EMPTY) continue;
        const uint32_t sh = 8 * c;
        // rs_child: q * step + base (reflections_software_bvh4.wgsl:38-39)
        const F3 lo = {add(mul((float)((lower[0] >> sh) & 255u), step.x), base.x),
                       add(mul((float)((lower[1] >> sh) & 255u), step.y), base.y),
                       add(mul((float)((lower[2] >> sh) & 255u), step.z), base.z)};
        const F3 hi = {add(mul((float)((upper[0] >> sh) & 255u), step.x), base.x),
                       add(mul((float)((upper[1] >> sh) & 255u), step.y), base.y),
                       add(mul((float)((upper[2] >> sh) & 255u), step.z), base.z)};
        dist[c] = slab_near(o, inv, lo, hi, ray.tmin, lim);
      }
#define RT_SW(a, b)                                      \
  if (dist[b] < dist[a]) {                               \
    float x = dist[a]; dist[a] = dist[b]; dist[b] = x;   \
    uint32_t y = ids[a]; ids[a] = ids[b]; ids[b] = y;    \
  }
      RT_SW(0, 1) RT_SW(2, 3) RT_SW(0, 2) RT_SW(1, 3) RT_SW(1, 2)
#undef RT_SW
#pragma unroll
      for (int c = 3; c >= 1; --c) {
        if (dist[c] <= lim && ids[c] != EMPTY) {
          if (sp < STACK) stack[sp++] = ids[c];
          else atomicAdd(&st->stack_drops, 1ull);
        }
      }
      if (dist[0] <= lim && ids[0] != EMPTY) {
        child = ids[0];
        continue;
      }
      break;
    }
  }
  return false;
}

// rs_trace (reflections_software_bvh4.wgsl:140-204)
template <bool ANY>
RT_DEV RsBest rs_trace(const uint32_t* __restrict__ w, const Ray& ray, DevStatus* st) {
  RsBest best;
  best.t = ray.tmax, best.rec[0] = best.rec[1] = best.rec[2] = best.rec[3] = 0, best.inst = EMPTY;
  const F3 world_inv = safe_inverse(ray.d);
  const uint4 head = ld4(w, 0);
  if (head.x == 0) return best;
  const size_t bounds = ld(w, 4) & ~3u;
  const F3 lo = ld3(w, bounds), hi = ld3(w, bounds + 4);
  const float ax = mul(sub(lo.x, ray.o.x), world_inv.x), ay = mul(sub(lo.y, ray.o.y), world_inv.y), az = mul(sub(lo.z, ray.o.z), world_inv.z);
  const float bx = mul(sub(hi.x, ray.o.x), world_inv.x), by = mul(sub(hi.y, ray.o.y), world_inv.y), bz = mul(sub(hi.z, ray.o.z), world_inv.z);
  const float near = fmaxf(fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fminf(az, bz)), ray.tmin);
  const float far = fminf(fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fmaxf(az, bz)), ray.tmax);
  if (near > far) return best;
  best.t = fminf(ray.tmax, __uint_as_float(__float_as_uint(far) + 2u));
  uint32_t stack[STACK];
  if (head.y == 0) {
    for (uint32_t i = 0; i < head.x; ++i)
      if (rs_instance<ANY>(w, i, ray, world_inv, best, stack, st)) return best;
    return best;
  }
  uint32_t nodes[STACK];
  nodes[0] = head.z;
  uint32_t sp = 1;
  while (sp > 0) {
    sp -= 1;
    const uint32_t item = nodes[sp];
    if (item & LEAF) {
      if (rs_instance<ANY>(w, item & ~LEAF, ray, world_inv, best, stack, st)) return best;
      continue;
    }
    const float bound = best.rec[0] != 0 ? next_up(best.t) : best.t;
    top_step(w, (head.y & ~3u) + (size_t)item * 32, ray, world_inv, bound, nodes, sp, st);
  }
  return best;
}

template <bool ANY>
__global__ void __launch_bounds__(128) k_rs_plain(const uint32_t* __restrict__ w, const float4* __restrict__ rays,
                                                  void* __restrict__ out, uint32_t n, DevStatus* st) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Ray ray = load_ray(rays, i);
  const RsBest b = rs_trace<ANY>(w, ray, st);
  if (ANY) {
    reinterpret_cast<uint32_t*>(out)[i] = b.rec[0] != 0 ? 1u : 0u;
    return;
  }
  uint32_t* o = reinterpret_cast<uint32_t*>(out) + 5 * (size_t)i;
  o[0] = __float_as_uint(b.t), o[1] = b.rec[0], o[2] = b.rec[1], o[3] = b.rec[2], o[4] = b.rec[3];
}

}  // namespace rtk
