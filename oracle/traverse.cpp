// CPU ORACLE — test infrastructure only. Scalar f32 restatement, loop for loop, of
//   shaders/gi_rays_software.wgsl:25-291        (gi_traverse, modes 0/1/2, BVH4 top level)
//   shaders/reflections_software_bvh4.wgsl:23-207 (rs_trace, closest / any-hit)
//   shaders/reflections_software.wgsl:22-149    (legacy BVH2 rs_trace, pinned by replay vectors)
// Compiled with -ffp-contract=off: each WGSL multiply and add rounds separately. Vector dot
// products sum left to right; cross products use the textbook component order.
//
// Three deliberate differences from the WGSL text, none of which changes a result the WGSL
// defines: (1) a child id EMPTY is never pushed (the WGSL pushes it only when the bound reaches
// FLT_MAX, and then reads out of bounds); (2) pushes past the 48-entry stack are dropped and
// counted (C_STACK_DROPS) in every loop, including the reflection BLAS loop that has no guard;
// (3) min/max follow IEEE 754-2019 minimum/maximum (-0 < +0), the convention the CUDA kernels
// use.
#include <algorithm>
#include <cfloat>

#include "oracle.hpp"

namespace orc {

namespace {

inline float kmin(float a, float b) {
  if (std::isnan(a)) return b;
  if (std::isnan(b)) return a;
  if (a < b) return a;
  if (b < a) return b;
  return std::signbit(a) ? a : b;
}
inline float kmax(float a, float b) {
  if (std::isnan(a)) return b;
  if (std::isnan(b)) return a;
  if (a > b) return a;
  if (b > a) return b;
  return std::signbit(a) ? b : a;
}
struct F3 { float x, y, z; };
inline F3 sub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F3 cross(F3 a, F3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float dot4(const float r[4], F3 p) { return r[0] * p.x + r[1] * p.y + r[2] * p.z + r[3] * 1.0f; }
inline float next_up_bits(float t) { return bitsf(fbits(t) + 1u); }

// gi_safe_inverse / rs_inverse (gi_rays_software.wgsl:27-30)
inline float safe_inv1(float d) {
  float tiny = d >= 0.0f ? 1e-30f : -1e-30f;
  return 1.0f / (std::fabs(d) < 1e-30f ? tiny : d);
}
inline F3 safe_inverse(F3 d) { return {safe_inv1(d.x), safe_inv1(d.y), safe_inv1(d.z)}; }

// gi_slab_near / rs_box (gi_rays_software.wgsl:35-40)
inline float slab_near(F3 o, F3 inv, F3 lo, F3 hi, float tmin, float tmax) {
  float ax = (lo.x - o.x) * inv.x, ay = (lo.y - o.y) * inv.y, az = (lo.z - o.z) * inv.z;
  float bx = (hi.x - o.x) * inv.x, by = (hi.y - o.y) * inv.y, bz = (hi.z - o.z) * inv.z;
  float near = kmax(kmax(kmax(kmin(ax, bx), kmin(ay, by)), kmin(az, bz)), tmin);
  float far = kmin(kmin(kmin(kmax(ax, bx), kmax(ay, by)), kmax(az, bz)), tmax);
  return near <= far ? near : FLT_BIG;
}

inline float wf(const uint32_t* w, size_t i) { return bitsf(w[i]); }
inline F3 wv(const uint32_t* w, size_t i) { return {wf(w, i), wf(w, i + 1), wf(w, i + 2)}; }

// gi_triangle (gi_rays_software.wgsl:42-58): (t,u,v) or t = -1
inline F3 gi_triangle(F3 o, F3 d, F3 a, F3 b, F3 c, float tmin, float tmax) {
  const F3 none = {-1.0f, 0.0f, 0.0f};
  F3 e1 = sub(b, a), e2 = sub(c, a);
  F3 p = cross(d, e2);
  float det = dot(e1, p);
  if (std::fabs(det) < 1e-30f) return none;
  float inv = 1.0f / det;
  F3 s = sub(o, a);
  float u = dot(s, p) * inv;
  if (u < 0.0f || u > 1.0f) return none;
  F3 q = cross(s, e1);
  float v = dot(d, q) * inv;
  if (v < 0.0f || u + v > 1.0f) return none;
  float t = dot(e2, q) * inv;
  if (t > tmin && t < tmax) return {t, u, v};
  return none;
}

// unit_normal (shaders/scene.wgsl:86-90); inverseSqrt as 1/sqrt, both correctly rounded.
inline F3 unit_normal(F3 n) {
  float scale = kmax(kmax(std::fabs(n.x), std::fabs(n.y)), std::fabs(n.z));
  float m = kmax(scale, 1e-30f);
  F3 s = {n.x / m, n.y / m, n.z / m};
  float k = 1.0f / std::sqrt(kmax(dot(s, s), 1e-30f));
  return {s.x * k, s.y * k, s.z * k};
}

constexpr uint32_t GI_STACK = 48;
constexpr uint32_t GI_INSTANCE_WORDS = 32;

// gi_limit (gi_rays_software.wgsl:68-70)
inline float gi_limit(const GiHit& b, uint32_t i) {
  return (b.hit && i < b.inst) ? next_up_bits(b.t) : b.t;
}

void bump(uint64_t* c, int k, uint64_t n = 1) {
  if (c) c[k] += n;
}

// gi_instance (gi_rays_software.wgsl:98-207), opaque mode (GI_SW_SEE_THROUGH=false).
bool gi_instance(const uint32_t* w, uint32_t i, F3 origin, F3 direction, F3 world_inv, float tmin,
                 bool any_hit, GiHit& best, uint32_t* stack, uint64_t* cnt) {
  size_t r = 16 + (size_t)i * GI_INSTANCE_WORDS;
  bump(cnt, C_TLAS_INSTANCE_ENTRIES);
  if (any_hit && (w[r + 27] & 1u) != 0) return false;
  bump(cnt, C_INSTANCE_BOX_TESTS);
  float lim0 = gi_limit(best, i);
  if (!(slab_near(origin, world_inv, wv(w, r + 12), wv(w, r + 15), tmin, lim0) <= lim0)) return false;
  bump(cnt, C_INSTANCE_BOX_ENTRIES);
  bump(cnt, C_BLAS_VISITS);
  float r0[4] = {wf(w, r), wf(w, r + 1), wf(w, r + 2), wf(w, r + 3)};
  float r1[4] = {wf(w, r + 4), wf(w, r + 5), wf(w, r + 6), wf(w, r + 7)};
  float r2[4] = {wf(w, r + 8), wf(w, r + 9), wf(w, r + 10), wf(w, r + 11)};
  F3 o = {dot4(r0, origin), dot4(r1, origin), dot4(r2, origin)};
  F3 d = {dot({r0[0], r0[1], r0[2]}, direction), dot({r1[0], r1[1], r1[2]}, direction),
          dot({r2[0], r2[1], r2[2]}, direction)};
  F3 inv = safe_inverse(d);
  uint32_t nodes = w[r + 18], leaves = w[r + 19], positions = w[r + 20], indices = w[r + 21];
  uint32_t prim_base = w[r + 28];
  auto normal_of = [&](F3 a, F3 b, F3 c) {
    F3 cr = cross(sub(b, a), sub(c, a));
    F3 n = {r0[0] * cr.x + r1[0] * cr.y + r2[0] * cr.z, r0[1] * cr.x + r1[1] * cr.y + r2[1] * cr.z,
            r0[2] * cr.x + r1[2] * cr.y + r2[2] * cr.z};
    return unit_normal(n);
  };
  stack[0] = w[r + 22];
  uint32_t sp = 1;
  while (sp > 0) {
    sp -= 1;
    uint32_t child = stack[sp];
    if (child & LEAF_BIT) {
      bump(cnt, C_LEAVES);
      size_t l = leaves + (size_t)(child & ~LEAF_BIT) * 2;
      uint32_t first = w[l], count = w[l + 1];
      for (uint32_t k = 0; k < count; k += 6) {
        size_t x = (size_t)indices + first + k;
        bool two = k + 3 < count;
        size_t y = two ? x + 3 : x;
        uint32_t ia = w[x], ib = w[x + 1], ic = w[x + 2];
        uint32_t ja = w[y], jb = w[y + 1], jc = w[y + 2];
        F3 a = wv(w, positions + (size_t)ia * 3), b = wv(w, positions + (size_t)ib * 3),
           c = wv(w, positions + (size_t)ic * 3);
        F3 a2 = wv(w, positions + (size_t)ja * 3), b2 = wv(w, positions + (size_t)jb * 3),
           c2 = wv(w, positions + (size_t)jc * 3);
        bump(cnt, C_TRIANGLE_TESTS);
        F3 h = gi_triangle(o, d, a, b, c, tmin, gi_limit(best, i));
        if (h.x >= 0.0f) {
          F3 n = normal_of(a, b, c);
          GiHit nb{true, h.x, {n.x, n.y, n.z}, i, {ia, ib, ic}, {h.y, h.z}};
          if (!any_hit && prim_base != 0) nb.tri[0] = w[prim_base + (first + k) / 3], nb.tri[1] = 0, nb.tri[2] = 0;
          best = nb;
          if (any_hit) return true;
        }
        if (two) {
          bump(cnt, C_TRIANGLE_TESTS);
          F3 h2 = gi_triangle(o, d, a2, b2, c2, tmin, gi_limit(best, i));
          if (h2.x >= 0.0f) {
            F3 n = normal_of(a2, b2, c2);
            GiHit nb{true, h2.x, {n.x, n.y, n.z}, i, {ja, jb, jc}, {h2.y, h2.z}};
            if (!any_hit && prim_base != 0) nb.tri[0] = w[prim_base + (first + k) / 3 + 1], nb.tri[1] = 0, nb.tri[2] = 0;
            best = nb;
            if (any_hit) return true;
          }
        }
      }
      continue;
    }
    bump(cnt, C_BLAS_NODES);
    size_t n = nodes + (size_t)child * 16;
    F3 oq = wv(w, n), step = wv(w, n + 3);
    float t[4] = {FLT_BIG, FLT_BIG, FLT_BIG, FLT_BIG};
    uint32_t c[4] = {w[n + 6], w[n + 7], w[n + 8], w[n + 9]};
    uint32_t lx = w[n + 10], ly = w[n + 11], lz = w[n + 12];
    uint32_t hx = w[n + 13], hy = w[n + 14], hz = w[n + 15];
    for (uint32_t s = 0; s < 4; ++s) {
      if (c[s] == EMPTY) continue;
      bump(cnt, C_BLAS_BOX_TESTS);
      uint32_t sh = 8 * s;
      F3 lq = {(float)((lx >> sh) & 0xffu), (float)((ly >> sh) & 0xffu), (float)((lz >> sh) & 0xffu)};
      F3 hq = {(float)((hx >> sh) & 0xffu), (float)((hy >> sh) & 0xffu), (float)((hz >> sh) & 0xffu)};
      F3 lo = {oq.x + step.x * lq.x, oq.y + step.y * lq.y, oq.z + step.z * lq.z};
      F3 hi = {oq.x + step.x * hq.x, oq.y + step.y * hq.y, oq.z + step.z * hq.z};
      t[s] = slab_near(o, inv, lo, hi, tmin, gi_limit(best, i));
    }
    // Four-element network on (distance bits, child), descending (gi_rays_software.wgsl:191-197).
    uint32_t a0x = fbits(t[0]), a0y = c[0], a1x = fbits(t[1]), a1y = c[1];
    uint32_t a2x = fbits(t[2]), a2y = c[2], a3x = fbits(t[3]), a3y = c[3];
    auto sw = [](uint32_t& ax, uint32_t& ay, uint32_t& bx, uint32_t& by) {
      if (ax < bx) std::swap(ax, bx), std::swap(ay, by);
    };
    sw(a0x, a0y, a1x, a1y);
    sw(a2x, a2y, a3x, a3y);
    sw(a0x, a0y, a2x, a2y);
    sw(a1x, a1y, a3x, a3y);
    sw(a1x, a1y, a2x, a2y);
    uint32_t ex[4] = {a0x, a1x, a2x, a3x}, ey[4] = {a0y, a1y, a2y, a3y};
    for (int s = 0; s < 4; ++s) {
      if (bitsf(ex[s]) <= gi_limit(best, i) && ey[s] != EMPTY) {
        if (sp < GI_STACK) stack[sp++] = ey[s];
        else bump(cnt, C_STACK_DROPS);
      }
    }
  }
  return false;
}

// The BVH4 top-level step shared by both traversals (gi_rays_software.wgsl:241-261,
// reflections_software_bvh4.wgsl:173-193): four slabs, the ascending network, far-to-near push.
void top_wide_step(const uint32_t* w, size_t n, F3 origin, F3 world_inv, float tmin, float bound,
                   uint32_t* stack, uint32_t& sp, uint64_t* cnt) {
  float dist[4];
  uint32_t ids[4];
  for (int c = 0; c < 4; ++c) {
    float ax = (wf(w, n + 0 + c) - origin.x) * world_inv.x, bx = (wf(w, n + 12 + c) - origin.x) * world_inv.x;
    float ay = (wf(w, n + 4 + c) - origin.y) * world_inv.y, by = (wf(w, n + 16 + c) - origin.y) * world_inv.y;
    float az = (wf(w, n + 8 + c) - origin.z) * world_inv.z, bz = (wf(w, n + 20 + c) - origin.z) * world_inv.z;
    float near = kmax(kmax(kmax(kmin(ax, bx), kmin(ay, by)), kmin(az, bz)), tmin);
    float far = kmin(kmin(kmin(kmax(ax, bx), kmax(ay, by)), kmax(az, bz)), bound);
    ids[c] = w[n + 24 + c];
    dist[c] = (near <= far && ids[c] != EMPTY) ? near : FLT_BIG;
  }
  bump(cnt, C_TLAS_BOX_TESTS, 4);
  auto sw = [&](int a, int b) {
    if (dist[b] < dist[a]) std::swap(dist[a], dist[b]), std::swap(ids[a], ids[b]);
  };
  sw(0, 1);
  sw(2, 3);
  sw(0, 2);
  sw(1, 3);
  sw(1, 2);
  for (int c = 3; c >= 0; --c) {
    if (dist[c] <= bound && ids[c] != EMPTY) {
      if (sp < TOP_STACK) stack[sp++] = ids[c];
      else bump(cnt, C_STACK_DROPS);
    }
  }
}

}  // namespace

// gi_traverse (gi_rays_software.wgsl:217-279)
GiHit gi_traverse(const uint32_t* w, const Ray& ray, uint32_t mode, bool top_wide, uint64_t* cnt) {
  bool any_hit = mode != 0;
  GiHit best{false, ray.tmax, {0, 0, 0}, 0xffffffffu, {0, 0, 0}, {0, 0}};
  uint32_t stack[GI_STACK];
  F3 origin = {ray.o[0], ray.o[1], ray.o[2]}, direction = {ray.d[0], ray.d[1], ray.d[2]};
  F3 world_inv = safe_inverse(direction);
  uint32_t instances = w[0], top = w[1];
  if (top == 0) {
    for (uint32_t i = 0; i < instances; ++i)
      if (gi_instance(w, i, origin, direction, world_inv, ray.tmin, any_hit, best, stack, cnt)) return best;
    return best;
  }
  uint32_t nodes[TOP_STACK];
  nodes[0] = w[2];
  uint32_t sp = 1;
  while (sp > 0) {
    sp -= 1;
    uint32_t item = nodes[sp];
    if (item & LEAF_BIT) {
      if (gi_instance(w, item & ~LEAF_BIT, origin, direction, world_inv, ray.tmin, any_hit, best, stack, cnt))
        return best;
      continue;
    }
    bump(cnt, C_TLAS_NODES);
    float bound = best.hit ? next_up_bits(best.t) : best.t;
    if (top_wide) {
      top_wide_step(w, top + (size_t)item * 32, origin, world_inv, ray.tmin, bound, nodes, sp, cnt);
      continue;
    }
    size_t n = top + (size_t)item * 16;
    float t0 = slab_near(origin, world_inv, wv(w, n), wv(w, n + 3), ray.tmin, bound);
    float t1 = slab_near(origin, world_inv, wv(w, n + 6), wv(w, n + 9), ray.tmin, bound);
    bump(cnt, C_TLAS_BOX_TESTS, 2);
    uint32_t c0 = w[n + 12], c1 = w[n + 13];
    bool near = t0 <= t1;
    float tf = near ? t1 : t0, tn = near ? t0 : t1;
    uint32_t cf = near ? c1 : c0, cn = near ? c0 : c1;
    if (tf <= bound && sp < TOP_STACK) nodes[sp++] = cf;
    if (tn <= bound && sp < TOP_STACK) nodes[sp++] = cn;
  }
  return best;
}

namespace {

constexpr uint32_t RS_STACK = 48;
constexpr float RS_EDGE = 4e-6f;

// rs_limit (reflections_software_bvh4.wgsl:45-47)
inline float rs_limit(const RsHit& b, uint32_t best_i, uint32_t i) {
  return (b.rec[0] != 0 && i <= best_i) ? next_up_bits(b.t) : b.t;
}

// rs_instance (reflections_software_bvh4.wgsl:50-130)
bool rs_instance(const uint32_t* w, uint32_t i, F3 origin, F3 direction, F3 world_inv, float tmin,
                 bool any_hit, RsHit& best, uint32_t& best_i, uint32_t* stack, uint64_t* cnt) {
  size_t R = 8 + (size_t)i * 24;
  bump(cnt, C_TLAS_INSTANCE_ENTRIES);
  uint32_t root = w[R + 20], slot = w[R + 21], noshadow = w[R + 22];
  if (any_hit && noshadow != 0) return false;
  bump(cnt, C_INSTANCE_BOX_TESTS);
  float bound = rs_limit(best, best_i, i);
  if (slab_near(origin, world_inv, wv(w, R + 12), wv(w, R + 15), tmin, bound) > bound) return false;
  bump(cnt, C_INSTANCE_BOX_ENTRIES);
  bump(cnt, C_BLAS_VISITS);
  float r0[4] = {wf(w, R), wf(w, R + 1), wf(w, R + 2), wf(w, R + 3)};
  float r1[4] = {wf(w, R + 4), wf(w, R + 5), wf(w, R + 6), wf(w, R + 7)};
  float r2[4] = {wf(w, R + 8), wf(w, R + 9), wf(w, R + 10), wf(w, R + 11)};
  F3 o = {dot4(r0, origin), dot4(r1, origin), dot4(r2, origin)};
  F3 d = {dot({r0[0], r0[1], r0[2]}, direction), dot({r1[0], r1[1], r1[2]}, direction),
          dot({r2[0], r2[1], r2[2]}, direction)};
  F3 inv = safe_inverse(d);
  size_t nodes = w[R + 18] & ~3u, triangles = w[R + 19] & ~3u;
  stack[0] = root;
  uint32_t sp = 1;
  while (sp > 0) {
    sp -= 1;
    uint32_t child = stack[sp];
    for (;;) {
      if (child & LEAF_BIT) {
        bump(cnt, C_LEAVES);
        uint32_t start = (child & ~LEAF_BIT) >> 4;
        for (uint32_t k = 0; k < (child & 15u); ++k) {
          bump(cnt, C_TRIANGLE_TESTS);
          size_t X = triangles + (size_t)(start + k) * 12;
          F3 a = wv(w, X), e1 = wv(w, X + 3), e2 = wv(w, X + 6);
          uint32_t prim = w[X + 9];
          F3 p = cross(d, e2);
          float det = dot(e1, p);
          if (std::fabs(det) < 1e-30f) continue;
          float inv_det = 1.0f / det;
          F3 s = sub(o, a);
          float u = dot(s, p) * inv_det;
          if (u < -RS_EDGE || u > 1.0f + RS_EDGE) continue;
          F3 q = cross(s, e1);
          float v = dot(d, q) * inv_det;
          if (v < -RS_EDGE || u + v > 1.0f + RS_EDGE) continue;
          float t = dot(e2, q) * inv_det;
          bool tied = best.rec[0] != 0 && t == best.t && (i < best_i || (i == best_i && prim < best.rec[1]));
          if (t > tmin && (t < best.t || tied)) {
            best = RsHit{t, {slot + 1, prim, fbits(u), fbits(v)}};
            best_i = i;
            if (any_hit) return true;
          }
        }
        break;
      }
      bump(cnt, C_BLAS_NODES);
      size_t N = nodes + (size_t)child * 16;
      F3 base = wv(w, N), step = wv(w, N + 3);
      uint32_t ids[4] = {w[N + 6], w[N + 7], w[N + 8], w[N + 9]};
      uint32_t lower[3] = {w[N + 10], w[N + 11], w[N + 12]}, upper[3] = {w[N + 13], w[N + 14], w[N + 15]};
      float lim = rs_limit(best, best_i, i);
      float dist[4];
      for (int c = 0; c < 4; ++c) {
        if (ids[c] == EMPTY) {
          dist[c] = FLT_BIG;
          continue;
        }
        bump(cnt, C_BLAS_BOX_TESTS);
        uint32_t sh = 8 * c;
        // rs_child: q * step + base (reflections_software_bvh4.wgsl:38-39)
        F3 lo = {(float)((lower[0] >> sh) & 255u) * step.x + base.x, (float)((lower[1] >> sh) & 255u) * step.y + base.y,
                 (float)((lower[2] >> sh) & 255u) * step.z + base.z};
        F3 hi = {(float)((upper[0] >> sh) & 255u) * step.x + base.x, (float)((upper[1] >> sh) & 255u) * step.y + base.y,
                 (float)((upper[2] >> sh) & 255u) * step.z + base.z};
        dist[c] = slab_near(o, inv, lo, hi, tmin, lim);
      }
      auto sw = [&](int a, int b) {
        if (dist[b] < dist[a]) std::swap(dist[a], dist[b]), std::swap(ids[a], ids[b]);
      };
      sw(0, 1);
      sw(2, 3);
      sw(0, 2);
      sw(1, 3);
      sw(1, 2);
      for (int c = 3; c >= 1; --c) {
        if (dist[c] <= lim && ids[c] != EMPTY) {
          if (sp < RS_STACK) stack[sp++] = ids[c];
          else bump(cnt, C_STACK_DROPS);
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

}  // namespace

// rs_trace (reflections_software_bvh4.wgsl:140-204)
RsHit rs_trace(const uint32_t* w, const Ray& ray, bool any_hit, uint64_t* cnt) {
  RsHit best{ray.tmax, {0, 0, 0, 0}};
  uint32_t best_i = 0xffffffffu;
  uint32_t stack[RS_STACK];
  F3 origin = {ray.o[0], ray.o[1], ray.o[2]}, direction = {ray.d[0], ray.d[1], ray.d[2]};
  F3 world_inv = safe_inverse(direction);
  uint32_t count = w[0], top = w[1], root = w[2];
  if (count == 0) return best;
  size_t bounds = w[4] & ~3u;
  F3 lo = wv(w, bounds), hi = wv(w, bounds + 4);
  float ax = (lo.x - origin.x) * world_inv.x, ay = (lo.y - origin.y) * world_inv.y, az = (lo.z - origin.z) * world_inv.z;
  float bx = (hi.x - origin.x) * world_inv.x, by = (hi.y - origin.y) * world_inv.y, bz = (hi.z - origin.z) * world_inv.z;
  float near = kmax(kmax(kmax(kmin(ax, bx), kmin(ay, by)), kmin(az, bz)), ray.tmin);
  float far = kmin(kmin(kmin(kmax(ax, bx), kmax(ay, by)), kmax(az, bz)), ray.tmax);
  if (near > far) return best;
  best.t = kmin(ray.tmax, bitsf(fbits(far) + 2u));
  if (top == 0) {
    for (uint32_t i = 0; i < count; ++i)
      if (rs_instance(w, i, origin, direction, world_inv, ray.tmin, any_hit, best, best_i, stack, cnt)) return best;
    return best;
  }
  uint32_t nodes[TOP_STACK];
  nodes[0] = root;
  uint32_t sp = 1;
  while (sp > 0) {
    sp -= 1;
    uint32_t item = nodes[sp];
    if (item & LEAF_BIT) {
      if (rs_instance(w, item & ~LEAF_BIT, origin, direction, world_inv, ray.tmin, any_hit, best, best_i, stack, cnt))
        return best;
      continue;
    }
    bump(cnt, C_TLAS_NODES);
    float bound = best.rec[0] != 0 ? next_up_bits(best.t) : best.t;
    top_wide_step(w, (top & ~3u) + (size_t)item * 32, origin, world_inv, ray.tmin, bound, nodes, sp, cnt);
  }
  return best;
}

namespace {

constexpr uint32_t RS2_STACK = 32;

// legacy rs_limit (reflections_software.wgsl:38-40): strictly lower instances only
inline float rs2_limit(const RsHit& b, uint32_t best_i, uint32_t i) {
  return (b.rec[0] != 0 && i < best_i) ? next_up_bits(b.t) : b.t;
}

// legacy rs_instance (reflections_software.wgsl:43-110)
bool rs2_instance(const uint32_t* w, uint32_t i, F3 origin, F3 direction, F3 world_inv, float tmin,
                  bool any_hit, RsHit& best, uint32_t& best_i, uint32_t* stack, uint64_t* cnt) {
  size_t R = 8 + (size_t)i * 24;
  bump(cnt, C_TLAS_INSTANCE_ENTRIES);
  uint32_t root = w[R + 20], slot = w[R + 21], noshadow = w[R + 22];
  if (any_hit && noshadow != 0) return false;
  bump(cnt, C_INSTANCE_BOX_TESTS);
  float bound = rs2_limit(best, best_i, i);
  if (slab_near(origin, world_inv, wv(w, R + 12), wv(w, R + 15), tmin, bound) > bound) return false;
  bump(cnt, C_INSTANCE_BOX_ENTRIES);
  bump(cnt, C_BLAS_VISITS);
  float r0[4] = {wf(w, R), wf(w, R + 1), wf(w, R + 2), wf(w, R + 3)};
  float r1[4] = {wf(w, R + 4), wf(w, R + 5), wf(w, R + 6), wf(w, R + 7)};
  float r2[4] = {wf(w, R + 8), wf(w, R + 9), wf(w, R + 10), wf(w, R + 11)};
  F3 o = {dot4(r0, origin), dot4(r1, origin), dot4(r2, origin)};
  F3 d = {dot({r0[0], r0[1], r0[2]}, direction), dot({r1[0], r1[1], r1[2]}, direction),
          dot({r2[0], r2[1], r2[2]}, direction)};
  F3 inv = safe_inverse(d);
  size_t nodes = w[R + 18] & ~3u, triangles = w[R + 19] & ~3u;
  stack[0] = root;
  uint32_t sp = 1;
  while (sp > 0) {
    sp -= 1;
    uint32_t child = stack[sp];
    for (;;) {
      if (child & LEAF_BIT) {
        bump(cnt, C_LEAVES);
        uint32_t start = (child & ~LEAF_BIT) >> 3;
        for (uint32_t k = 0; k < (child & 7u); ++k) {
          bump(cnt, C_TRIANGLE_TESTS);
          size_t X = triangles + (size_t)(start + k) * 12;
          F3 a = wv(w, X), e1 = wv(w, X + 3), e2 = wv(w, X + 6);
          F3 p = cross(d, e2);
          float det = dot(e1, p);
          if (std::fabs(det) < 1e-30f) continue;
          float inv_det = 1.0f / det;
          F3 s = sub(o, a);
          float u = dot(s, p) * inv_det;
          if (u < -RS_EDGE || u > 1.0f + RS_EDGE) continue;
          F3 q = cross(s, e1);
          float v = dot(d, q) * inv_det;
          if (v < -RS_EDGE || u + v > 1.0f + RS_EDGE) continue;
          float t = dot(e2, q) * inv_det;
          if (t > tmin && t < rs2_limit(best, best_i, i)) {
            best = RsHit{t, {slot + 1, w[X + 9], fbits(u), fbits(v)}};
            best_i = i;
            if (any_hit) return true;
          }
        }
        break;
      }
      bump(cnt, C_BLAS_NODES);
      size_t N = nodes + (size_t)child * 16;
      float lim = rs2_limit(best, best_i, i);
      float t0 = slab_near(o, inv, wv(w, N), wv(w, N + 3), tmin, lim);
      float t1 = slab_near(o, inv, wv(w, N + 6), wv(w, N + 9), tmin, lim);
      bump(cnt, C_BLAS_BOX_TESTS, 2);
      uint32_t c0 = w[N + 12], c1 = w[N + 13];
      bool h0 = t0 <= lim, h1 = t1 <= lim;
      if (h0 && h1) {
        bool near_first = t0 <= t1;
        if (sp < RS2_STACK) stack[sp++] = near_first ? c1 : c0;
        else bump(cnt, C_STACK_DROPS);
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

}  // namespace

// legacy rs_trace (reflections_software.wgsl:115-149)
RsHit rs_trace_bvh2(const uint32_t* w, const Ray& ray, bool any_hit, uint64_t* cnt) {
  RsHit best{ray.tmax, {0, 0, 0, 0}};
  uint32_t best_i = 0xffffffffu;
  uint32_t stack[RS2_STACK];
  F3 origin = {ray.o[0], ray.o[1], ray.o[2]}, direction = {ray.d[0], ray.d[1], ray.d[2]};
  F3 world_inv = safe_inverse(direction);
  uint32_t count = w[0], top = w[1];
  if (top == 0) {
    for (uint32_t i = 0; i < count; ++i)
      if (rs2_instance(w, i, origin, direction, world_inv, ray.tmin, any_hit, best, best_i, stack, cnt)) return best;
    return best;
  }
  uint32_t nodes[RS2_STACK];
  nodes[0] = w[2];
  uint32_t sp = 1;
  while (sp > 0) {
    sp -= 1;
    uint32_t item = nodes[sp];
    if (item & LEAF_BIT) {
      if (rs2_instance(w, item & ~LEAF_BIT, origin, direction, world_inv, ray.tmin, any_hit, best, best_i, stack, cnt))
        return best;
      continue;
    }
    bump(cnt, C_TLAS_NODES);
    size_t n = (top & ~3u) + (size_t)item * 16;
    float bound = best.rec[0] != 0 ? next_up_bits(best.t) : best.t;
    float t0 = slab_near(origin, world_inv, wv(w, n), wv(w, n + 3), ray.tmin, bound);
    float t1 = slab_near(origin, world_inv, wv(w, n + 6), wv(w, n + 9), ray.tmin, bound);
    bump(cnt, C_TLAS_BOX_TESTS, 2);
    bool near = t0 <= t1;
    float tf = near ? t1 : t0, tn = near ? t0 : t1;
    uint32_t cf = near ? w[n + 13] : w[n + 12], cn = near ? w[n + 12] : w[n + 13];
    if (tf <= bound) {
      if (sp < RS2_STACK) nodes[sp++] = cf;
      else bump(cnt, C_STACK_DROPS);
    }
    if (tn <= bound) {
      if (sp < RS2_STACK) nodes[sp++] = cn;
      else bump(cnt, C_STACK_DROPS);
    }
  }
  return best;
}

}  // namespace orc
