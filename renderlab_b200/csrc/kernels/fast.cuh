// FAST traversal kernels: the PLAIN per-ray arithmetic and visit order, rescheduled.
//
// Each ray performs exactly the operations of rs_trace / gi_traverse in the same order (so its
// hit is bit-identical), but the loop is flattened into a per-lane state machine -- one node,
// one leaf or one top-level step per iteration -- inside persistent warps that refill a lane
// with the next ray as soon as its ray ends (warp-aggregated atomics on a global ray counter).
// Lanes therefore stop idling behind the longest ray of their warp, and the divergent nested
// loops of the direct transcription become one reconverging loop.
//
// Quantised planes are decoded without integer-to-float conversions: for a byte q,
// as_float(0x4B000000 | q) - 2^23 is q exactly, an integer OR and one FP32 subtract.
#pragma once
#include "plain.cuh"

namespace rtk {

// q as float, exactly (q <= 255 < 2^23).
RT_DEV float byte_f(uint32_t word, uint32_t shift) {
  return __fsub_rn(__uint_as_float(0x4B000000u | ((word >> shift) & 0xffu)), 8388608.0f);
}

// Persistent-kernel ray distribution: every lane that needs a ray takes the next index of the
// launch; one atomic per warp per refill round.
struct RayQueue {
  unsigned int* next;  // global counter, zeroed before the launch
  uint32_t n;
  uint32_t refill;     // idle lanes a warp waits for before taking more rays (1-32)
};

// Called by all 32 lanes together. `drained` (warp-uniform) stops the requests once the
// counter has passed the end, so finished warps add no atomic traffic.
RT_DEV uint32_t take_ray(const RayQueue& q, bool need, bool& drained) {
  const unsigned idle = __ballot_sync(0xffffffffu, need);
  const unsigned want = (!drained && (uint32_t)__popc(idle) >= q.refill) ? idle : 0u;
  if (!want) return EMPTY;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(want) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(q.next, (unsigned)__popc(want));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (base + (uint32_t)__popc(want) >= q.n) drained = true;
  const uint32_t idx = base + __popc(want & ((1u << lane) - 1u));
  return (need && (want >> lane & 1u) && idx < q.n) ? idx : EMPTY;
}

// ---------------------------------------------------------------- reflection layout

enum : uint32_t { PH_IDLE = 0, PH_TOP = 1, PH_BLAS = 2 };

template <int AM>
struct RsLane {
  Ray ray;
  F3 world_inv;
  RsBest best;
  uint32_t ray_id;
  uint32_t entry;  // batch entry (many-batch launches)
  bool any;        // any-hit ray (AM 2)
  uint32_t phase;
  // top level (or flat list position)
  uint32_t tsp;
  uint32_t flat_i;
  // current instance
  uint32_t inst, slot;
  F3 o, d, inv;
  uint32_t nodes, tris;
  uint32_t cur;  // child to process next, EMPTY: pop
  uint32_t sp;
};

template <int AM, class Src>
RT_DEV void rs_finish(RsLane<AM>& L, const Src& src) {
  if (any_of<AM>(L)) {
    put_flag(src, L.entry, L.ray_id, L.ray, L.best.rec[0] != 0);
  } else {
    uint32_t* o = reinterpret_cast<uint32_t*>(out_of(src, L.entry)) + 5 * (size_t)L.ray_id;
    o[0] = __float_as_uint(L.best.t), o[1] = L.best.rec[0], o[2] = L.best.rec[1], o[3] = L.best.rec[2];
    o[4] = L.best.rec[3];
  }
  L.phase = PH_IDLE;
}

// rs_instance's entry (reflections_software_bvh4.wgsl:50-67): true when the lane now walks the
// instance's BLAS.
template <int AM>
RT_DEV bool rs_enter(const uint32_t* __restrict__ w, RsLane<AM>& L, uint32_t i) {
  const size_t R = 8 + (size_t)i * 24;
  const uint4 tail = ld4(w, R + 20);
  if (any_of<AM>(L) && tail.z != 0) return false;
  const uint4 b0 = ld4(w, R + 12), b1 = ld4(w, R + 16);
  const float bound = rs_limit(L.best, i);
  const F3 lo = {__uint_as_float(b0.x), __uint_as_float(b0.y), __uint_as_float(b0.z)};
  const F3 hi = {__uint_as_float(b0.w), __uint_as_float(b1.x), __uint_as_float(b1.y)};
  if (slab_near(L.ray.o, L.world_inv, lo, hi, L.ray.tmin, bound) > bound) return false;
  const uint4 q0 = ld4(w, R), q1 = ld4(w, R + 4), q2 = ld4(w, R + 8);
  const F3 ro = L.ray.o, rd = L.ray.d;
  L.o = {dot4p(__uint_as_float(q0.x), __uint_as_float(q0.y), __uint_as_float(q0.z), __uint_as_float(q0.w), ro),
         dot4p(__uint_as_float(q1.x), __uint_as_float(q1.y), __uint_as_float(q1.z), __uint_as_float(q1.w), ro),
         dot4p(__uint_as_float(q2.x), __uint_as_float(q2.y), __uint_as_float(q2.z), __uint_as_float(q2.w), ro)};
  L.d = {dot3({__uint_as_float(q0.x), __uint_as_float(q0.y), __uint_as_float(q0.z)}, rd),
         dot3({__uint_as_float(q1.x), __uint_as_float(q1.y), __uint_as_float(q1.z)}, rd),
         dot3({__uint_as_float(q2.x), __uint_as_float(q2.y), __uint_as_float(q2.z)}, rd)};
  L.inv = safe_inverse(L.d);
  L.nodes = b1.z & ~3u;
  L.tris = b1.w & ~3u;
  L.inst = i;
  L.slot = tail.y;
  L.cur = tail.x;
  L.sp = 0;
  L.phase = PH_BLAS;
  return true;
}

// One leaf (reflections_software_bvh4.wgsl:72-95). True when an any-hit ray is blocked.
template <int AM>
RT_DEV bool rs_leaf(const uint32_t* __restrict__ w, RsLane<AM>& L, uint32_t child) {
  const uint32_t start = (child & ~LEAF) >> 4, count = child & 15u;
  const F3 o = L.o, d = L.d;
  for (uint32_t k = 0; k < count; ++k) {
    const size_t X = L.tris + (size_t)(start + k) * 12;
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
    const bool tied = L.best.rec[0] != 0 && t == L.best.t &&
                      (L.inst < L.best.inst || (L.inst == L.best.inst && w2.y < L.best.rec[1]));
    if (t > L.ray.tmin && (t < L.best.t || tied)) {
      L.best.t = t;
      L.best.rec[0] = L.slot + 1, L.best.rec[1] = w2.y, L.best.rec[2] = __float_as_uint(u);
      L.best.rec[3] = __float_as_uint(v);
      L.best.inst = L.inst;
      if (any_of<AM>(L)) return true;
    }
  }
  return false;
}

// One BLAS node (reflections_software_bvh4.wgsl:99-125): children sorted, the nearest kept.
template <int AM>
RT_DEV void rs_node(const uint32_t* __restrict__ w, RsLane<AM>& L, uint32_t child, uint32_t* stack, DevStatus* st) {
  const size_t N = L.nodes + (size_t)child * 16;
  const uint4 n0 = ld4u(w, N), n1 = ld4u(w, N + 4), n2 = ld4u(w, N + 8), n3 = ld4u(w, N + 12);
  const float lim = rs_limit(L.best, L.inst);
  const F3 base = {__uint_as_float(n0.x), __uint_as_float(n0.y), __uint_as_float(n0.z)};
  const F3 step = {__uint_as_float(n0.w), __uint_as_float(n1.x), __uint_as_float(n1.y)};
  uint32_t ids[4] = {n1.z, n1.w, n2.x, n2.y};
  float dist[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    dist[c] = BIG;
    if (ids[c] == EMPTY) continue;
    const uint32_t sh = 8 * c;
    const F3 lo = {add(mul(byte_f(n2.z, sh), step.x), base.x), add(mul(byte_f(n2.w, sh), step.y), base.y),
                   add(mul(byte_f(n3.x, sh), step.z), base.z)};
    const F3 hi = {add(mul(byte_f(n3.y, sh), step.x), base.x), add(mul(byte_f(n3.z, sh), step.y), base.y),
                   add(mul(byte_f(n3.w, sh), step.z), base.z)};
    dist[c] = slab_near(L.o, L.inv, lo, hi, L.ray.tmin, lim);
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
      if (L.sp < STACK) stack[L.sp++] = ids[c];
      else atomicAdd(&st->stack_drops, 1ull);
    }
  }
  L.cur = (dist[0] <= lim && ids[0] != EMPTY) ? ids[0] : EMPTY;
}

template <int AM, int BLOCK, class Src>
__global__ void __launch_bounds__(BLOCK) k_rs_fast(const uint32_t* __restrict__ w, const Src src, RayQueue queue,
                                                   DevStatus* st) {
  uint32_t stack[STACK];
  uint32_t top_stack[STACK];
  RsLane<AM> L;
  L.phase = PH_IDLE;
  const uint4 head = ld4(w, 0);
  const size_t bounds = ld(w, 4) & ~3u;
  bool drained = false;
  for (;;) {
    // Refill idle lanes; a warp leaves when none of its lanes holds a ray.
    __syncwarp();
    const uint32_t id = take_ray(queue, L.phase == PH_IDLE, drained);
    if (L.phase == PH_IDLE && id != EMPTY) {
      L.ray = fetch(src, id, L);
      L.world_inv = safe_inverse(L.ray.d);
      L.best.t = L.ray.tmax, L.best.rec[0] = L.best.rec[1] = L.best.rec[2] = L.best.rec[3] = 0, L.best.inst = EMPTY;
      // rs_trace prologue (reflections_software_bvh4.wgsl:141-155)
      bool live = head.x != 0;
      if (live) {
        const F3 lo = ld3(w, bounds), hi = ld3(w, bounds + 4);
        const F3 o = L.ray.o, wi = L.world_inv;
        const float ax = mul(sub(lo.x, o.x), wi.x), ay = mul(sub(lo.y, o.y), wi.y), az = mul(sub(lo.z, o.z), wi.z);
        const float bx = mul(sub(hi.x, o.x), wi.x), by = mul(sub(hi.y, o.y), wi.y), bz = mul(sub(hi.z, o.z), wi.z);
        const float near = fmaxf(fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fminf(az, bz)), L.ray.tmin);
        const float far = fminf(fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fmaxf(az, bz)), L.ray.tmax);
        live = !(near > far);
        if (live) L.best.t = fminf(L.ray.tmax, __uint_as_float(__float_as_uint(far) + 2u));
      }
      if (live) {
        L.phase = PH_TOP;
        L.flat_i = 0;
        L.tsp = 1;
        top_stack[0] = head.z;
      } else {
        rs_finish<AM>(L, src);  // misses the scene box: done, refilled next iteration
      }
    }
    // Every lane reaches this vote once per iteration (no exit above it); the warp leaves only
    // when no lane holds a ray and the queue is drained.
    if (!__any_sync(0xffffffffu, L.phase != PH_IDLE)) {
      if (drained) break;
      continue;
    }
    if (L.phase == PH_BLAS) {
      if (L.cur == EMPTY) {
        if (L.sp == 0) {
          L.phase = PH_TOP;  // instance done
        } else {
          L.cur = stack[--L.sp];
        }
      }
      if (L.phase == PH_BLAS) {
        const uint32_t child = L.cur;
        if (child & LEAF) {
          if (rs_leaf<AM>(w, L, child)) {
            rs_finish<AM>(L, src);
            continue;
          }
          L.cur = EMPTY;
        } else {
          rs_node<AM>(w, L, child, stack, st);
        }
        continue;
      }
    }
    if (L.phase == PH_TOP) {
      if (head.y == 0) {  // flat instance list
        if (L.flat_i >= head.x) {
          rs_finish<AM>(L, src);
          continue;
        }
        rs_enter<AM>(w, L, L.flat_i++);
        continue;
      }
      if (L.tsp == 0) {
        rs_finish<AM>(L, src);
        continue;
      }
      const uint32_t item = top_stack[--L.tsp];
      if (item & LEAF) {
        rs_enter<AM>(w, L, item & ~LEAF);
        continue;
      }
      const float bound = L.best.rec[0] != 0 ? next_up(L.best.t) : L.best.t;
      top_step(w, (head.y & ~3u) + (size_t)item * 32, L.ray, L.world_inv, bound, top_stack, L.tsp, st);
    }
  }
}

// ---------------------------------------------------------------- GI layout

template <int AM>
struct GiLane {
  Ray ray;
  F3 world_inv;
  GiBest best;
  uint32_t ray_id;
  uint32_t entry;
  bool any;
  uint32_t phase;
  uint32_t tsp, flat_i;
  uint32_t inst;
  float r[12];
  F3 o, d, inv;
  uint32_t nodes, leaves, positions, indices, prim_base;
  uint32_t cur, sp;
};

template <int AM, class Src>
RT_DEV void gi_finish(GiLane<AM>& L, const Src& src) {
  const GiBest& b = L.best;
  if (any_of<AM>(L)) {
    put_flag(src, L.entry, L.ray_id, L.ray, b.hit);
  } else {
    uint32_t* o = reinterpret_cast<uint32_t*>(out_of(src, L.entry)) + 10 * (size_t)L.ray_id;
    o[0] = __float_as_uint(b.t), o[1] = b.inst, o[2] = b.tri[0], o[3] = b.tri[1], o[4] = b.tri[2];
    o[5] = __float_as_uint(b.u), o[6] = __float_as_uint(b.v);
    o[7] = __float_as_uint(b.n.x), o[8] = __float_as_uint(b.n.y), o[9] = __float_as_uint(b.n.z);
  }
  L.phase = PH_IDLE;
}

// gi_instance's entry (gi_rays_software.wgsl:100-113)
template <int AM>
RT_DEV void gi_enter(const uint32_t* __restrict__ w, GiLane<AM>& L, uint32_t i) {
  const size_t r = 16 + (size_t)i * 32;
  if (any_of<AM>(L) && (ld(w, r + 27) & 1u) != 0) return;
  const float lim = gi_limit(L.best, i);
  if (!(slab_near(L.ray.o, L.world_inv, ld3(w, r + 12), ld3(w, r + 15), L.ray.tmin, lim) <= lim)) return;
  for (int k = 0; k < 12; ++k) L.r[k] = ldf(w, r + k);
  const F3 ro = L.ray.o, rd = L.ray.d;
  L.o = {dot4p(L.r[0], L.r[1], L.r[2], L.r[3], ro), dot4p(L.r[4], L.r[5], L.r[6], L.r[7], ro),
         dot4p(L.r[8], L.r[9], L.r[10], L.r[11], ro)};
  L.d = {dot3({L.r[0], L.r[1], L.r[2]}, rd), dot3({L.r[4], L.r[5], L.r[6]}, rd), dot3({L.r[8], L.r[9], L.r[10]}, rd)};
  L.inv = safe_inverse(L.d);
  L.nodes = ld(w, r + 18), L.leaves = ld(w, r + 19), L.positions = ld(w, r + 20), L.indices = ld(w, r + 21);
  L.prim_base = ld(w, r + 28);
  L.inst = i;
  L.cur = ld(w, r + 22);
  L.sp = 0;
  L.phase = PH_BLAS;
}

// One GI leaf (gi_rays_software.wgsl:117-169). True when an any-hit ray is blocked.
template <int AM>
RT_DEV bool gi_leaf(const uint32_t* __restrict__ w, GiLane<AM>& L, uint32_t child) {
  const size_t l = L.leaves + (size_t)(child & ~LEAF) * 2;
  const uint32_t first = ld(w, l), count = ld(w, l + 1);
  const uint32_t i = L.inst;
  auto normal_of = [&](F3 a, F3 b, F3 c) {
    F3 cr = cross3(sub3(b, a), sub3(c, a));
    F3 n = {add(add(mul(L.r[0], cr.x), mul(L.r[4], cr.y)), mul(L.r[8], cr.z)),
            add(add(mul(L.r[1], cr.x), mul(L.r[5], cr.y)), mul(L.r[9], cr.z)),
            add(add(mul(L.r[2], cr.x), mul(L.r[6], cr.y)), mul(L.r[10], cr.z))};
    return unit_normal(n);
  };
  for (uint32_t k = 0; k < count; k += 6) {
    const size_t x = (size_t)L.indices + first + k;
    const bool two = k + 3 < count;
    const size_t y = two ? x + 3 : x;
    const uint32_t ia = ld(w, x), ib = ld(w, x + 1), ic = ld(w, x + 2);
    const uint32_t ja = ld(w, y), jb = ld(w, y + 1), jc = ld(w, y + 2);
    const F3 a = ld3(w, L.positions + (size_t)ia * 3), b = ld3(w, L.positions + (size_t)ib * 3),
             c = ld3(w, L.positions + (size_t)ic * 3);
    const F3 a2 = ld3(w, L.positions + (size_t)ja * 3), b2 = ld3(w, L.positions + (size_t)jb * 3),
             c2 = ld3(w, L.positions + (size_t)jc * 3);
    float t, u, v;
    if (gi_triangle(L.o, L.d, a, b, c, L.ray.tmin, gi_limit(L.best, i), t, u, v)) {
      L.best.hit = true, L.best.t = t, L.best.inst = i, L.best.u = u, L.best.v = v;
      if (any_of<AM>(L)) return true;
      L.best.n = normal_of(a, b, c);
      if (L.prim_base != 0) L.best.tri[0] = ld(w, L.prim_base + (first + k) / 3), L.best.tri[1] = 0, L.best.tri[2] = 0;
      else L.best.tri[0] = ia, L.best.tri[1] = ib, L.best.tri[2] = ic;
    }
    if (two && gi_triangle(L.o, L.d, a2, b2, c2, L.ray.tmin, gi_limit(L.best, i), t, u, v)) {
      L.best.hit = true, L.best.t = t, L.best.inst = i, L.best.u = u, L.best.v = v;
      if (any_of<AM>(L)) return true;
      L.best.n = normal_of(a2, b2, c2);
      if (L.prim_base != 0) L.best.tri[0] = ld(w, L.prim_base + (first + k) / 3 + 1), L.best.tri[1] = 0, L.best.tri[2] = 0;
      else L.best.tri[0] = ja, L.best.tri[1] = jb, L.best.tri[2] = jc;
    }
  }
  return false;
}

// One GI BLAS node (gi_rays_software.wgsl:171-204): every surviving child pushed far to near.
template <int AM>
RT_DEV void gi_node(const uint32_t* __restrict__ w, GiLane<AM>& L, uint32_t child, uint32_t* stack, DevStatus* st) {
  const size_t n = L.nodes + (size_t)child * 16;
  const uint4 n0 = ld4u(w, n), n1 = ld4u(w, n + 4), n2 = ld4u(w, n + 8), n3 = ld4u(w, n + 12);
  const F3 oq = {__uint_as_float(n0.x), __uint_as_float(n0.y), __uint_as_float(n0.z)};
  const F3 step = {__uint_as_float(n0.w), __uint_as_float(n1.x), __uint_as_float(n1.y)};
  uint32_t c[4] = {n1.z, n1.w, n2.x, n2.y};
  const float lim = gi_limit(L.best, L.inst);
  uint32_t tb[4];
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    tb[s] = __float_as_uint(BIG);
    if (c[s] == EMPTY) continue;
    const uint32_t sh = 8 * s;
    const F3 lo = {add(oq.x, mul(step.x, byte_f(n2.z, sh))), add(oq.y, mul(step.y, byte_f(n2.w, sh))),
                   add(oq.z, mul(step.z, byte_f(n3.x, sh)))};
    const F3 hi = {add(oq.x, mul(step.x, byte_f(n3.y, sh))), add(oq.y, mul(step.y, byte_f(n3.z, sh))),
                   add(oq.z, mul(step.z, byte_f(n3.w, sh)))};
    tb[s] = __float_as_uint(slab_near(L.o, L.inv, lo, hi, L.ray.tmin, lim));
  }
#define RT_SW(a, b)                          \
  if (tb[a] < tb[b]) {                       \
    uint32_t x = tb[a]; tb[a] = tb[b]; tb[b] = x; \
    x = c[a]; c[a] = c[b]; c[b] = x;         \
  }
  RT_SW(0, 1) RT_SW(2, 3) RT_SW(0, 2) RT_SW(1, 3) RT_SW(1, 2)
#undef RT_SW
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    if (__uint_as_float(tb[s]) <= lim && c[s] != EMPTY) {
      if (L.sp < STACK) stack[L.sp++] = c[s];
      else atomicAdd(&st->stack_drops, 1ull);
    }
  }
  L.cur = EMPTY;
}

template <int AM, int BLOCK, class Src>
__global__ void __launch_bounds__(BLOCK) k_gi_fast(const uint32_t* __restrict__ w, const Src src, RayQueue queue,
                                                   DevStatus* st) {
  uint32_t stack[STACK];
  uint32_t top_stack[STACK];
  GiLane<AM> L;
  L.phase = PH_IDLE;
  const uint32_t instances = ld(w, 0), top = ld(w, 1), root = ld(w, 2);
  bool drained = false;
  for (;;) {
    __syncwarp();
    const uint32_t id = take_ray(queue, L.phase == PH_IDLE, drained);
    if (L.phase == PH_IDLE && id != EMPTY) {
      L.ray = fetch(src, id, L);
      L.world_inv = safe_inverse(L.ray.d);
      L.best.hit = false, L.best.t = L.ray.tmax, L.best.n = {0.0f, 0.0f, 0.0f}, L.best.inst = EMPTY;
      L.best.tri[0] = L.best.tri[1] = L.best.tri[2] = 0, L.best.u = L.best.v = 0.0f;
      L.phase = PH_TOP;
      L.flat_i = 0;
      L.tsp = 1;
      top_stack[0] = root;
    }
    if (!__any_sync(0xffffffffu, L.phase != PH_IDLE)) {
      if (drained) break;
      continue;
    }
    if (L.phase == PH_BLAS) {
      if (L.cur == EMPTY) {
        if (L.sp == 0) L.phase = PH_TOP;
        else L.cur = stack[--L.sp];
      }
      if (L.phase == PH_BLAS) {
        const uint32_t child = L.cur;
        if (child & LEAF) {
          if (gi_leaf<AM>(w, L, child)) {
            gi_finish<AM>(L, src);
            continue;
          }
          L.cur = EMPTY;
        } else {
          gi_node<AM>(w, L, child, stack, st);
        }
        continue;
      }
    }
    if (L.phase == PH_TOP) {
      if (top == 0) {
        if (L.flat_i >= instances) {
          gi_finish<AM>(L, src);
          continue;
        }
        gi_enter<AM>(w, L, L.flat_i++);
        continue;
      }
      if (L.tsp == 0) {
        gi_finish<AM>(L, src);
        continue;
      }
      const uint32_t item = top_stack[--L.tsp];
      if (item & LEAF) {
        gi_enter<AM>(w, L, item & ~LEAF);
        continue;
      }
      const float bound = L.best.hit ? next_up(L.best.t) : L.best.t;
      top_step(w, top + (size_t)item * 32, L.ray, L.world_inv, bound, top_stack, L.tsp, st);
    }
  }
}

}  // namespace rtk
