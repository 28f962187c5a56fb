// Shared device helpers for the traversal kernels.
//
// Arithmetic convention of the bit-exact kernels (PLAIN, FAST): every multiply, add, subtract
// and reciprocal is an explicit round-to-nearest intrinsic (__fmul_rn, __fadd_rn, __fsub_rn,
// __frcp_rn), which nvcc never contracts into an FMA, so each WGSL operation rounds on its own.
// Sums run left to right; cross products use the textbook component order. min/max are
// fminf/fmaxf.
#pragma once
#include <cstdint>

#define RT_DEV __device__ __forceinline__

namespace rtk {

constexpr uint32_t LEAF = 0x80000000u;
constexpr uint32_t EMPTY = 0xffffffffu;
constexpr float BIG = 3.4028235e38f;
constexpr uint32_t STACK = 48;

struct F3 {
  float x, y, z;
};

RT_DEV float mul(float a, float b) { return __fmul_rn(a, b); }
RT_DEV float add(float a, float b) { return __fadd_rn(a, b); }
RT_DEV float sub(float a, float b) { return __fsub_rn(a, b); }
RT_DEV F3 sub3(F3 a, F3 b) { return {sub(a.x, b.x), sub(a.y, b.y), sub(a.z, b.z)}; }
RT_DEV float dot3(F3 a, F3 b) { return add(add(mul(a.x, b.x), mul(a.y, b.y)), mul(a.z, b.z)); }
RT_DEV F3 cross3(F3 a, F3 b) {
  return {sub(mul(a.y, b.z), mul(a.z, b.y)), sub(mul(a.z, b.x), mul(a.x, b.z)), sub(mul(a.x, b.y), mul(a.y, b.x))};
}
// dot(r, vec4(p, 1.0))
RT_DEV float dot4p(float r0, float r1, float r2, float r3, F3 p) {
  return add(add(add(mul(r0, p.x), mul(r1, p.y)), mul(r2, p.z)), mul(r3, 1.0f));
}
RT_DEV float next_up(float t) { return __uint_as_float(__float_as_uint(t) + 1u); }

// gi_safe_inverse / rs_inverse: 1/d with |d| < 1e-30 replaced by +-1e-30 (sign of d >= 0).
RT_DEV float safe_rcp(float d) {
  float tiny = d >= 0.0f ? 1e-30f : -1e-30f;
  return __frcp_rn(fabsf(d) < 1e-30f ? tiny : d);
}
RT_DEV F3 safe_inverse(F3 d) { return {safe_rcp(d.x), safe_rcp(d.y), safe_rcp(d.z)}; }

// gi_slab_near / rs_box: entry distance clamped to tmin, or BIG when the slabs miss.
RT_DEV float slab_near(F3 o, F3 inv, F3 lo, F3 hi, float tmin, float tmax) {
  float ax = mul(sub(lo.x, o.x), inv.x), ay = mul(sub(lo.y, o.y), inv.y), az = mul(sub(lo.z, o.z), inv.z);
  float bx = mul(sub(hi.x, o.x), inv.x), by = mul(sub(hi.y, o.y), inv.y), bz = mul(sub(hi.z, o.z), inv.z);
  float near = fmaxf(fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fminf(az, bz)), tmin);
  float far = fminf(fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fmaxf(az, bz)), tmax);
  return near <= far ? near : BIG;
}

RT_DEV uint32_t ld(const uint32_t* __restrict__ w, size_t i) { return __ldg(w + i); }
RT_DEV float ldf(const uint32_t* __restrict__ w, size_t i) { return __uint_as_float(__ldg(w + i)); }
RT_DEV F3 ld3(const uint32_t* __restrict__ w, size_t i) { return {ldf(w, i), ldf(w, i + 1), ldf(w, i + 2)}; }
RT_DEV uint4 ld4(const uint32_t* __restrict__ w, size_t i) {
  return __ldg(reinterpret_cast<const uint4*>(w + i));
}
// Four words at any word offset: one 16-byte load when the offset is a multiple of 4, else four
// word loads. The reference's packers align only some records: GI meshes follow one another
// with no padding, so a mesh's node records start wherever the previous mesh ended. The offset's
// alignment is the same for every node of a mesh, so lanes of one mesh take the same path.
RT_DEV uint4 ld4u(const uint32_t* __restrict__ w, size_t i) {
  if ((i & 3) == 0) return __ldg(reinterpret_cast<const uint4*>(w + i));
  return make_uint4(__ldg(w + i), __ldg(w + i + 1), __ldg(w + i + 2), __ldg(w + i + 3));
}

struct Ray {
  F3 o;
  float tmin;
  F3 d;
  float tmax;
};
RT_DEV Ray load_ray(const float4* __restrict__ rays, uint32_t i) {
  float4 a = __ldg(rays + 2 * (size_t)i), b = __ldg(rays + 2 * (size_t)i + 1);
  return Ray{{a.x, a.y, a.z}, a.w, {b.x, b.y, b.z}, b.w};
}
// The streaming form (ld.global.cs: evict first from L1 and L2): a walk reads each ray once, and
// a launch's ray stream (32 bytes a ray, hundreds of MB) should not push the scene out of L2.
RT_DEV Ray load_ray_cs(const float4* __restrict__ rays, uint32_t i) {
  float4 a = __ldcs(rays + 2 * (size_t)i), b = __ldcs(rays + 2 * (size_t)i + 1);
  return Ray{{a.x, a.y, a.z}, a.w, {b.x, b.y, b.z}, b.w};
}
template <bool CS>
RT_DEV Ray load_ray_as(const float4* __restrict__ rays, uint32_t i) {
  return CS ? load_ray_cs(rays, i) : load_ray(rays, i);
}

// One ray batch of a many-batch launch, as the device reads it (32 bytes).
struct BatchEntry {
  const float4* rays;
  void* hits;
  uint32_t first;  // the entry's first ray in the launch
  uint32_t n;
  uint32_t mode;   // 0 closest hit, else any hit
  uint32_t pad;
};

// Where a persistent launch's rays come from and where their results go.
// One batch: ray i of the launch is rays[order ? order[i] : i]; every ray has the launch's mode.
struct OneBatch {
  const float4* rays;
  const uint32_t* order;
  void* out;
};
// Many batches (rt_trace_batches): the launch's ray space is the concatenation of the entries
// (BatchEntry); a ray's entry is found by binary search over `first`, and each entry has its own
// rays, results and mode.
struct ManyBatches {
  const BatchEntry* table;
  uint32_t entries;
  const uint32_t* order;  // optional permutation of the launch's whole ray space
};

// Mode of a lane: AM 0 closest, 1 any hit, 2 per ray (from its batch entry).
template <int AM, class Lane>
RT_DEV bool any_of(const Lane& L) {
  return AM == 2 ? L.any : AM == 1;
}

// CS: the ray is read in the streaming form (load_ray_cs).
template <bool CS = false, class Lane>
RT_DEV Ray fetch(const OneBatch& s, uint32_t id, Lane& L) {
  L.ray_id = s.order ? __ldg(s.order + id) : id;
  L.entry = 0;
  return load_ray_as<CS>(s.rays, L.ray_id);
}
template <bool CS = false, class Lane>
RT_DEV Ray fetch(const ManyBatches& s, uint32_t id, Lane& L) {
  const uint32_t g = s.order ? __ldg(s.order + id) : id;
  uint32_t lo = 0, hi = s.entries;  // the last entry whose first ray is at or before g
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (s.table[mid].first <= g) lo = mid;
    else hi = mid;
  }
  const BatchEntry& e = s.table[lo];
  L.entry = lo;
  L.ray_id = g - e.first;
  L.any = e.mode != 0;
  return load_ray_as<CS>(e.rays, L.ray_id);
}
RT_DEV void* out_of(const OneBatch& s, uint32_t) { return s.out; }
RT_DEV void* out_of(const ManyBatches& s, uint32_t entry) { return s.table[entry].hits; }

// Stores an any-hit result: one word a ray, 1 when something blocks it. A ray source that packs
// its results otherwise (the GI cache's light words) overloads this for its own type.
template <class Src>
RT_DEV void put_flag(const Src& s, uint32_t entry, uint32_t id, const Ray&, bool blocked) {
  reinterpret_cast<uint32_t*>(out_of(s, entry))[id] = blocked ? 1u : 0u;
}

// Device-side counters every traversal kernel may bump (rare events only).
struct DevStatus {
  unsigned long long stack_drops;
  unsigned long long reserved[7];
};

}  // namespace rtk
