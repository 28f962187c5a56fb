// Oracle (test infrastructure): the GI cache's cell ray producers restated on the CPU -- the
// fixed directions of a cache cell about its normal. Follows gi_cells.wgsl:481-487
// (gi_unpack_normal), gi_cells.wgsl:463-468 (gi_basis), gi_cache.wgsl:1046-1054 (gi_direction)
// and gi_cache.wgsl:1064-1068 (gi_origin_offset), each f32 operation rounded on its own
// (-ffp-contract=off); square roots and the division correctly rounded (IEEE); cos and sin in
// double, rounded once to f32.
#include <cmath>
#include <cstdint>
#include <cstring>

namespace {

constexpr uint32_t DIRECTIONS = 64;  // gi_cells.wgsl:35

float fbits(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
uint32_t ubits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }

float snorm16(uint32_t v) {  // unpack2x16snorm
  float f = (float)(int16_t)(uint16_t)(v & 0xffffu) / 32767.0f;
  return std::fmin(std::fmax(f, -1.0f), 1.0f);
}

struct V3 { float x, y, z; };

V3 unpack_normal(uint32_t w) {
  V3 n{snorm16(w), snorm16(w >> 16), 0.0f};
  n.z = (1.0f - std::fabs(n.x)) - std::fabs(n.y);
  const float t = std::fmax(-n.z, 0.0f);
  n.x = n.x + (n.x >= 0.0f ? -t : t);
  n.y = n.y + (n.y >= 0.0f ? -t : t);
  const float len = std::sqrt((n.x * n.x + n.y * n.y) + n.z * n.z);
  return {n.x / len, n.y / len, n.z / len};
}

}  // namespace

namespace {

float origin_offset(V3 q, float edge) {  // gi_origin_offset, gi_cache.wgsl:1064-1068
  const float m = std::fmax(std::fmax(std::fabs(q.x), std::fabs(q.y)), std::fabs(q.z));
  const float mm = std::fmax(m, 1e-30f);
  const float ulp = fbits(ubits(mm) + 1u) - mm;
  return std::fmax(std::fmax(1e-5f, 32.0f * ulp) + 1e-4f * edge, 1e-4f + 4e-7f * m);
}

}  // namespace

// The GI cache's per-light visibility rays (gi_light, gi_cache.wgsl:2054-2077): for every cell
// and light, whether the light reaches the cell (gi_light_affects, gi_cache.wgsl:2028-2036) and
// the ray that gi_visible_within traces toward it (gi_light_direction, gi_cache.wgsl:1977-1983):
// from the cell's offset origin, tmin 0, tmax the light's distance (1e20 for a directional
// light). A light is the renderer's 80-byte record (light_cluster.wgsl:10): position_range,
// travel_outer, rgb_inner (f32 xyzw each), kind (u32 x: 0 directional, 1 point, 2 spot), source.
// Ray (c, l) is rays[8 * (c * n_lights + l)]; affects has the same index.
extern "C" void orc_gi_light_rays(const uint32_t* cells, uint32_t n_cells, const uint32_t* lights, uint32_t n_lights,
                                  float* rays, uint8_t* affects) {
  for (uint32_t c = 0; c < n_cells; ++c) {
    const uint32_t* cell = cells + 8 * (size_t)c;
    const V3 q{fbits(cell[0]), fbits(cell[1]), fbits(cell[2])};
    const V3 n = unpack_normal(cell[4]);
    const float off = origin_offset(q, fbits(cell[3]));
    const V3 o{q.x + n.x * off, q.y + n.y * off, q.z + n.z * off};
    for (uint32_t l = 0; l < n_lights; ++l) {
      const uint32_t* L = lights + 20 * (size_t)l;
      const float px = fbits(L[0]), py = fbits(L[1]), pz = fbits(L[2]), range = fbits(L[3]);
      const float tx = fbits(L[4]), ty = fbits(L[5]), tz = fbits(L[6]), outer = fbits(L[7]);
      const uint32_t kind = L[12];
      float dx, dy, dz, dist;
      if (kind == 0) {
        dx = -tx, dy = -ty, dz = -tz, dist = 1e20f;
      } else {
        const float ex = px - q.x, ey = py - q.y, ez = pz - q.z;
        dist = std::sqrt((ex * ex + ey * ey) + ez * ez);
        const float den = std::fmax(dist, 1e-30f);
        dx = ex / den, dy = ey / den, dz = ez / den;
      }
      bool reach = !(fbits(L[8]) == 0.0f && fbits(L[9]) == 0.0f && fbits(L[10]) == 0.0f);
      if (reach && (n.x * dx + n.y * dy) + n.z * dz <= 0.0f) reach = false;
      if (reach && kind != 0) {
        if (range > 0.0f && dist >= range) reach = false;
        else if (kind == 2 && !(((-dx) * tx + (-dy) * ty) + (-dz) * tz > outer)) reach = false;
      }
      const size_t k = (size_t)c * n_lights + l;
      float* ray = rays + 8 * k;
      ray[0] = o.x, ray[1] = o.y, ray[2] = o.z, ray[3] = 0.0f;
      ray[4] = dx, ray[5] = dy, ray[6] = dz, ray[7] = dist;
      affects[k] = reach ? 1 : 0;
    }
  }
}

extern "C" void orc_gi_cell_rays(const uint32_t* cells, uint32_t n_cells, int rotate, float* rays) {
  for (uint32_t c = 0; c < n_cells; ++c) {
    const uint32_t* cell = cells + 8 * (size_t)c;
    const V3 q{fbits(cell[0]), fbits(cell[1]), fbits(cell[2])};
    const float edge = fbits(cell[3]);
    const V3 n = unpack_normal(cell[4]);
    const uint32_t key_b = cell[5];
    // gi_basis
    const float s = n.z >= 0.0f ? 1.0f : -1.0f;
    const float a = -1.0f / (s + n.z);
    const float b = (n.x * n.y) * a;
    const V3 c0{1.0f + ((s * n.x) * n.x) * a, s * b, -(s * n.x)};
    const V3 c1{b, s + (n.y * n.y) * a, -n.y};
    // gi_origin_offset
    const float m = std::fmax(std::fmax(std::fabs(q.x), std::fabs(q.y)), std::fabs(q.z));
    const float mm = std::fmax(m, 1e-30f);
    const float ulp = fbits(ubits(mm) + 1u) - mm;
    const float off = std::fmax(std::fmax(1e-5f, 32.0f * ulp) + 1e-4f * edge, 1e-4f + 4e-7f * m);
    const V3 o{q.x + n.x * off, q.y + n.y * off, q.z + n.z * off};
    for (uint32_t k = 0; k < DIRECTIONS; ++k) {
      const float z = 1.0f - ((float)k + 0.5f) / (float)DIRECTIONS;
      const float r = std::sqrt(std::fmax(1.0f - z * z, 0.0f));
      const float rotation = rotate ? (float)(key_b >> 8) * (float)(6.283185307179586 / 16777216.0) : 0.0f;
      const float phi = (float)k * 2.399963229728653f + rotation;
      const float x = r * (float)std::cos((double)phi), y = r * (float)std::sin((double)phi);
      float* ray = rays + 8 * ((size_t)c * DIRECTIONS + k);
      ray[0] = o.x, ray[1] = o.y, ray[2] = o.z, ray[3] = 0.0f;
      ray[4] = (c0.x * x + c1.x * y) + n.x * z;
      ray[5] = (c0.y * x + c1.y * y) + n.y * z;
      ray[6] = (c0.z * x + c1.z * y) + n.z * z;
      ray[7] = 1e20f;
    }
  }
}
