// The GI cache's ray producers, restated: the fixed gather / visibility directions of a cache cell
// (gi_cache.wgsl:1046-1054 gi_direction, gi_cells.wgsl:463-468 gi_basis, gi_cache.wgsl:1064-1068
// gi_origin_offset, gi_cells.wgsl:481-487 gi_unpack_normal), generated on the fly as a ray source
// of the persistent traversal: ray k of cell c is item c * 64 + k, as gi_gather traces them
// (gi_gather_software.wgsl:89-94) and gi_ray tests them (gi_cache.wgsl:1562-1575).
//
// Arithmetic: every operation is an explicit round-to-nearest f32 step in the WGSL's order; the
// square roots and the division are correctly rounded; cos and sin are evaluated in double and
// rounded once to f32 (so that the CPU restatement gives the same bits).
#pragma once
#include "common.cuh"

namespace rtk {

constexpr uint32_t GI_DIRECTIONS = 64;  // gi_cells.wgsl:35
constexpr uint32_t GI_F_ROTATE = 4;     // gi_cells.wgsl:148

// One cache cell as the producers read it (32 bytes): its query point, cell edge, octahedral
// normal (pack2x16snorm), and the key word whose high 24 bits turn its directions.
struct GiCell {
  float q[3];
  float edge;
  uint32_t normal;
  uint32_t key_b;
  uint32_t pad[2];
};

RT_DEV float snorm16(uint32_t v) {  // unpack2x16snorm, one half
  const float f = __fdiv_rn((float)(int16_t)(v & 0xffffu), 32767.0f);
  return fminf(fmaxf(f, -1.0f), 1.0f);
}

RT_DEV F3 gi_unpack_normal(uint32_t w) {
  F3 n = {snorm16(w), snorm16(w >> 16), 0.0f};
  n.z = sub(sub(1.0f, fabsf(n.x)), fabsf(n.y));
  const float t = fmaxf(-n.z, 0.0f);
  n.x = add(n.x, n.x >= 0.0f ? -t : t);
  n.y = add(n.y, n.y >= 0.0f ? -t : t);
  const float len = __fsqrt_rn(dot3(n, n));
  return {__fdiv_rn(n.x, len), __fdiv_rn(n.y, len), __fdiv_rn(n.z, len)};
}

// gi_basis (Duff et al. 2017): columns c0, c1 and n.
RT_DEV void gi_basis(F3 n, F3& c0, F3& c1) {
  const float s = n.z >= 0.0f ? 1.0f : -1.0f;
  const float a = __fdiv_rn(-1.0f, add(s, n.z));
  const float b = mul(mul(n.x, n.y), a);
  c0 = {add(1.0f, mul(mul(mul(s, n.x), n.x), a)), mul(s, b), -mul(s, n.x)};
  c1 = {b, add(s, mul(mul(n.y, n.y), a)), -n.y};
}

RT_DEV F3 gi_direction(F3 c0, F3 c1, F3 n, uint32_t key_b, uint32_t k, bool rotate) {
  const float z = sub(1.0f, __fdiv_rn(add((float)k, 0.5f), (float)GI_DIRECTIONS));
  const float r = __fsqrt_rn(fmaxf(sub(1.0f, mul(z, z)), 0.0f));
  const float rotation = rotate ? mul((float)(key_b >> 8), (float)(6.283185307179586 / 16777216.0)) : 0.0f;
  const float phi = add(mul((float)k, 2.399963229728653f), rotation);
  const float x = mul(r, (float)cos((double)phi)), y = mul(r, (float)sin((double)phi));
  return {add(add(mul(c0.x, x), mul(c1.x, y)), mul(n.x, z)), add(add(mul(c0.y, x), mul(c1.y, y)), mul(n.y, z)),
          add(add(mul(c0.z, x), mul(c1.z, y)), mul(n.z, z))};
}

RT_DEV float gi_origin_offset(F3 q, float edge) {
  const float m = fmaxf(fmaxf(fabsf(q.x), fabsf(q.y)), fabsf(q.z));
  const float mm = fmaxf(m, 1e-30f);
  const float ulp = sub(__uint_as_float(__float_as_uint(mm) + 1u), mm);
  return fmaxf(add(fmaxf(1e-5f, mul(32.0f, ulp)), mul(1e-4f, edge)), add(1e-4f, mul(4e-7f, m)));
}

// The ray of item `i`: cell i / 64, direction i % 64; tmin 0, tmax 1e20 (gi_closest / gi_visible).
RT_DEV Ray gi_cell_ray(const GiCell* __restrict__ cells, uint32_t i, bool rotate) {
  const GiCell& c = cells[i / GI_DIRECTIONS];
  const F3 q = {c.q[0], c.q[1], c.q[2]};
  const F3 n = gi_unpack_normal(c.normal);
  F3 c0, c1;
  gi_basis(n, c0, c1);
  const float off = gi_origin_offset(q, c.edge);
  const F3 o = {add(q.x, mul(n.x, off)), add(q.y, mul(n.y, off)), add(q.z, mul(n.z, off))};
  return Ray{o, 0.0f, gi_direction(c0, c1, n, c.key_b, i % GI_DIRECTIONS, rotate), 1e20f};
}

// Ray source of the persistent kernels: the cells' directions, results at the item index.
struct CellRays {
  const GiCell* cells;
  uint32_t rotate;
  void* out;
};
template <bool CS = false, class Lane>  // CS: no ray is read (the ray is made here)
RT_DEV Ray fetch(const CellRays& s, uint32_t id, Lane& L) {
  L.ray_id = id;
  L.entry = 0;
  return gi_cell_ray(s.cells, id, s.rotate != 0);
}
RT_DEV void* out_of(const CellRays& s, uint32_t) { return s.out; }

// ---- per-light visibility (gi_light, gi_cache.wgsl:2040-2077) ----

// A light as the GI cache reads it (light_cluster.wgsl:10, 80 bytes): position and range,
// travel direction and spot cosine, colour and inner cosine, kind (x: 0 directional, 1 point,
// 2 spot), source.
struct GiLight {
  float position_range[4];
  float travel_outer[4];
  float rgb_inner[4];
  uint32_t kind[4];
  float source[4];
};

// gi_light_direction (gi_cache.wgsl:1977-1983): the unit direction from q toward the light and
// its distance (1e20 for a directional light).
RT_DEV void gi_light_direction(const GiLight& l, F3 q, F3& d, float& dist) {
  if (l.kind[0] == 0u) {
    d = {-l.travel_outer[0], -l.travel_outer[1], -l.travel_outer[2]};
    dist = 1e20f;
    return;
  }
  const F3 e = {sub(l.position_range[0], q.x), sub(l.position_range[1], q.y), sub(l.position_range[2], q.z)};
  dist = __fsqrt_rn(dot3(e, e));
  const float den = fmaxf(dist, 1e-30f);
  d = {__fdiv_rn(e.x, den), __fdiv_rn(e.y, den), __fdiv_rn(e.z, den)};
}

// gi_light_affects (gi_cache.wgsl:2028-2036): a lit light whose direction leaves the cell's
// surface, within range, and inside a spot light's cone.
RT_DEV bool gi_light_affects(const GiLight& l, F3 n, F3 d, float dist) {
  if (l.rgb_inner[0] == 0.0f && l.rgb_inner[1] == 0.0f && l.rgb_inner[2] == 0.0f) return false;
  if (dot3(n, d) <= 0.0f) return false;
  if (l.kind[0] == 0u) return true;
  if (l.position_range[3] > 0.0f && dist >= l.position_range[3]) return false;
  return l.kind[0] != 2u || dot3({-d.x, -d.y, -d.z}, {l.travel_outer[0], l.travel_outer[1], l.travel_outer[2]}) > l.travel_outer[3];
}

// Ray source: item i is (cell i / n_lights, light i % n_lights), the ray gi_light traces with
// gi_visible_within from the cell's offset origin toward the light (tmin 0, tmax the light's
// distance from the query point). A light that does not reach the cell is not traced: its ray
// gets tmax -1, which nothing meets, and no bit. Results are the cells' light words: bit l % 32
// of word l / 32 of cell c (words_per_cell words a cell, zeroed before the launch) is set when
// the light reaches the cell and nothing blocks its ray.
struct LightRays {
  const GiCell* cells;
  const GiLight* lights;
  uint32_t n_lights;
  uint32_t words_per_cell;
  uint32_t* words;
};
RT_DEV Ray gi_light_ray(const LightRays& s, uint32_t i) {
  const uint32_t c = i / s.n_lights, l = i - c * s.n_lights;
  const GiCell& cell = s.cells[c];
  const F3 q = {cell.q[0], cell.q[1], cell.q[2]};
  const F3 n = gi_unpack_normal(cell.normal);
  const float off = gi_origin_offset(q, cell.edge);
  const F3 o = {add(q.x, mul(n.x, off)), add(q.y, mul(n.y, off)), add(q.z, mul(n.z, off))};
  const GiLight& light = s.lights[l];
  F3 d;
  float dist;
  gi_light_direction(light, q, d, dist);
  return Ray{o, 0.0f, d, gi_light_affects(light, n, d, dist) ? dist : -1.0f};
}
template <bool CS = false, class Lane>  // CS: no ray is read (the ray is made here)
RT_DEV Ray fetch(const LightRays& s, uint32_t id, Lane& L) {
  L.ray_id = id;
  L.entry = 0;
  return gi_light_ray(s, id);
}
RT_DEV void* out_of(const LightRays& s, uint32_t) { return s.words; }
RT_DEV void put_flag(const LightRays& s, uint32_t, uint32_t id, const Ray& ray, bool blocked) {
  if (blocked || !(ray.tmax > 0.0f)) return;
  const uint32_t c = id / s.n_lights, l = id - c * s.n_lights;
  atomicOr(s.words + (size_t)c * s.words_per_cell + (l >> 5), 1u << (l & 31u));
}

}  // namespace rtk
