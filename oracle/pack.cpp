// CPU ORACLE — test infrastructure only. Restates the packed-buffer writers:
// src/gi_bvh.rs:108-274 (GI layout), gi_cache.rs:4388-4488 (instance words 24-31, place),
// src/reflection_software.rs:108-368 (reflection layout, incl. the legacy median BVH2).
#include <algorithm>
#include <limits>
#include <map>

#include "oracle.hpp"

namespace orc {

namespace {

constexpr size_t GI_HEADER = 16, GI_INSTANCE = 32;  // gi_bvh.rs:19,25
constexpr size_t RS_HEADER = 8, RS_INSTANCE = 24;   // reflection_software.rs:38,42
constexpr uint32_t RS_LEAF = 0x80000000u;            // reflection_software.rs:35
constexpr size_t RS_TRIANGLE_WORDS = 12;            // reflection_software.rs:33

Box empty_box() {
  const float inf = std::numeric_limits<float>::infinity();
  return Box{{inf, inf, inf}, {-inf, -inf, -inf}};
}
void add_point(Box& b, const float* p) {
  for (int i = 0; i < 3; ++i) b.lo[i] = rmin(b.lo[i], p[i]), b.hi[i] = rmax(b.hi[i], p[i]);
}

// glam Mat4::transform_point3 for an affine model (3 rows of 4): x*px + y*py + z*pz + w, summed
// in that order, one rounding each.
void transform_point(const float* m, const float* p, float* out) {
  for (int r = 0; r < 3; ++r) {
    float acc = m[r * 4 + 0] * p[0];
    acc = m[r * 4 + 1] * p[1] + acc;
    acc = m[r * 4 + 2] * p[2] + acc;
    out[r] = m[r * 4 + 3] + acc;
  }
}

bool singular(const float* model, const float* rows) {
  double a[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) a[r * 3 + c] = model[r * 4 + c];
  double det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
               a[2] * (a[3] * a[7] - a[4] * a[6]);
  if (det == 0.0) return true;
  for (int k = 0; k < 12; ++k)
    if (!std::isfinite(rows[k])) return true;
  return false;
}

}  // namespace

// gi_bvh.rs:108-136
std::vector<uint32_t> map_primitives(const std::vector<uint32_t>& bvh_indices, const uint32_t* src,
                                     size_t nsrc) {
  size_t tri_count = nsrc / 3, bvh_tris = bvh_indices.size() / 3;
  if (tri_count == 0 || bvh_tris == 0) return {};
  std::map<std::array<uint32_t, 3>, uint32_t> head;
  std::vector<uint32_t> next(tri_count, 0xffffffffu);
  for (size_t id = tri_count; id-- > 0;) {
    std::array<uint32_t, 3> key = {src[3 * id], src[3 * id + 1], src[3 * id + 2]};
    auto it = head.find(key);
    if (it != head.end()) {
      next[id] = it->second;
      it->second = (uint32_t)id;
    } else {
      head[key] = (uint32_t)id;
    }
  }
  std::vector<uint32_t> prims;
  prims.reserve(bvh_tris);
  for (size_t t = 0; t < bvh_tris; ++t) {
    std::array<uint32_t, 3> key = {bvh_indices[3 * t], bvh_indices[3 * t + 1], bvh_indices[3 * t + 2]};
    auto it = head.find(key);
    if (it == head.end()) return {};
    uint32_t id = it->second;
    if (id == 0xffffffffu) return {};
    it->second = next[id];
    prims.push_back(id);
  }
  return prims;
}

// gi_bvh.rs:151-274 and gi_cache.rs:4476-4487: layout, mesh words, instance words, extra words,
// then the top level.
bool gi_pack(const std::vector<GiMesh>& meshes, const std::vector<GiInstance>& inst, int tlas_mode,
             std::vector<uint32_t>& words, std::string& err) {
  size_t n = inst.size();
  size_t at = GI_HEADER + n * GI_INSTANCE + tlas_reserve(n);
  std::vector<std::array<uint32_t, 4>> offsets;
  for (const GiMesh& m : meshes) {
    uint32_t nodes = (uint32_t)at;
    uint32_t leaves = nodes + (uint32_t)m.bvh.nodes.size() * 16;
    uint32_t positions = leaves + (uint32_t)m.bvh.leaves.size() * 2;
    uint32_t indices = positions + (uint32_t)m.bvh.positions.size() * 3;
    at += m.bvh.nodes.size() * 16 + m.bvh.leaves.size() * 2 + m.bvh.positions.size() * 3 +
          m.bvh.indices.size() + m.primitives.size();
    offsets.push_back({nodes, leaves, positions, indices});
  }
  size_t total = at;
  // instance_words (gi_bvh.rs:230-274)
  std::vector<uint32_t> head(GI_HEADER + n * GI_INSTANCE, 0);
  head[0] = (uint32_t)n;
  for (size_t i = 0; i < n; ++i) {
    const GiInstance& g = inst[i];
    if (g.mesh >= meshes.size()) {
      err = "instance mesh index";
      return false;
    }
    if (singular(g.model, g.rows)) {
      err = "indirect geometry transform is singular";
      return false;
    }
    const GiMesh& m = meshes[g.mesh];
    size_t r = GI_HEADER + i * GI_INSTANCE;
    for (int k = 0; k < 12; ++k) head[r + k] = fbits(g.rows[k]);
    float lo[3], hi[3];
    for (int a = 0; a < 3; ++a) lo[a] = INFINITY, hi[a] = -INFINITY;
    for (int c = 0; c < 8; ++c) {
      float p[3], w[3];
      for (int a = 0; a < 3; ++a) p[a] = (c & (1 << a)) == 0 ? m.lo[a] : m.hi[a];
      transform_point(g.model, p, w);
      for (int a = 0; a < 3; ++a) lo[a] = rmin(lo[a], w[a]), hi[a] = rmax(hi[a], w[a]);
    }
    for (int a = 0; a < 3; ++a) {
      float pad = 1e-5f * (1.0f + rmax(std::fabs(lo[a]), std::fabs(hi[a])));
      head[r + 12 + a] = fbits(lo[a] - pad);
      head[r + 15 + a] = fbits(hi[a] + pad);
    }
    for (int k = 0; k < 4; ++k) head[r + 18 + k] = offsets[g.mesh][k];
    head[r + 22] = m.bvh.root;
    head[r + 23] = g.near_base;
    for (int k = 0; k < 8; ++k) head[r + 24 + k] = g.extra[k];
    // gi_cache.rs:4409-4413: the primitive table follows the mesh's indices, when it has one.
    head[r + 28] = m.primitives.empty() ? 0u : offsets[g.mesh][3] + (uint32_t)m.bvh.indices.size();
  }
  tlas_place(head, GI_HEADER, GI_INSTANCE, n, {}, tlas_mode, true, true);
  words.assign(total, 0);
  std::copy(head.begin(), head.end(), words.begin());
  // mesh_words (gi_bvh.rs:182-226)
  for (size_t mi = 0; mi < meshes.size(); ++mi) {
    const GiMesh& m = meshes[mi];
    size_t w = offsets[mi][0];
    for (const Node& nd : m.bvh.nodes) {
      for (int a = 0; a < 3; ++a) words[w++] = fbits(nd.origin[a]);
      for (int a = 0; a < 3; ++a) words[w++] = fbits(nd.step[a]);
      for (int s = 0; s < 4; ++s) words[w++] = nd.children[s];
      for (int a = 0; a < 3; ++a)
        words[w++] = nd.lower[a][0] | nd.lower[a][1] << 8 | nd.lower[a][2] << 16 | (uint32_t)nd.lower[a][3] << 24;
      for (int a = 0; a < 3; ++a)
        words[w++] = nd.upper[a][0] | nd.upper[a][1] << 8 | nd.upper[a][2] << 16 | (uint32_t)nd.upper[a][3] << 24;
    }
    for (const Leaf& l : m.bvh.leaves) words[w++] = l.offset, words[w++] = l.count;
    for (const auto& p : m.bvh.positions)
      for (int a = 0; a < 3; ++a) words[w++] = fbits(p[a]);
    for (uint32_t x : m.bvh.indices) words[w++] = x;
    for (uint32_t x : m.primitives) words[w++] = x;
  }
  return true;
}

// reflection_software.rs:108-168
bool rs_from_bvh(const float* pos, const uint32_t* idx, size_t nidx, const Bvh& bvh, RsMesh& out) {
  auto tag = [&](uint32_t child) -> uint32_t {
    if (child == EMPTY) return EMPTY;
    if (!(child & LEAF_BIT)) return child;
    const Leaf& l = bvh.leaves[child & ~LEAF_BIT];
    return RS_LEAF | ((l.offset / 3) << 4) | (l.count / 3);
  };
  out.nodes.clear();
  out.triangles.clear();
  for (const Node& nd : bvh.nodes) {
    for (int a = 0; a < 3; ++a) out.nodes.push_back(fbits(nd.origin[a]));
    for (int a = 0; a < 3; ++a) out.nodes.push_back(fbits(nd.step[a]));
    for (int s = 0; s < 4; ++s) out.nodes.push_back(tag(nd.children[s]));
    for (int a = 0; a < 3; ++a)
      out.nodes.push_back(nd.lower[a][0] | nd.lower[a][1] << 8 | nd.lower[a][2] << 16 | (uint32_t)nd.lower[a][3] << 24);
    for (int a = 0; a < 3; ++a)
      out.nodes.push_back(nd.upper[a][0] | nd.upper[a][1] << 8 | nd.upper[a][2] << 16 | (uint32_t)nd.upper[a][3] << 24);
  }
  std::vector<uint32_t> prims = map_primitives(bvh.indices, idx, nidx);
  if (prims.size() != bvh.indices.size() / 3) return false;
  for (size_t t = 0; t < prims.size(); ++t) {
    const float* a = pos + 3 * (size_t)bvh.indices[3 * t];
    const float* b = pos + 3 * (size_t)bvh.indices[3 * t + 1];
    const float* c = pos + 3 * (size_t)bvh.indices[3 * t + 2];
    for (int k = 0; k < 3; ++k) out.triangles.push_back(fbits(a[k]));
    for (int k = 0; k < 3; ++k) out.triangles.push_back(fbits(b[k] - a[k]));
    for (int k = 0; k < 3; ++k) out.triangles.push_back(fbits(c[k] - a[k]));
    out.triangles.push_back(prims[t]);
    out.triangles.push_back(0);
    out.triangles.push_back(0);
  }
  Box bb = empty_box();
  for (size_t k = 0; k < nidx; ++k) add_point(bb, pos + 3 * (size_t)idx[k]);
  out.lo = bb.lo;
  out.hi = bb.hi;
  out.root = tag(bvh.root);
  out.wide = true;
  return true;
}

namespace {
// reflection_software.rs:209-264 (legacy median BVH2, four triangles a leaf)
struct MedianBuilder {
  const float* pos;
  const uint32_t* idx;
  std::vector<V3> centroids;
  std::vector<uint32_t> nodes, triangles;
  struct R { uint32_t id; V3 lo, hi; };
  R subtree(uint32_t* order, size_t n) {
    if (n <= 4) return leaf(order, n);
    Box cb = empty_box();
    for (size_t k = 0; k < n; ++k) add_point(cb, centroids[order[k]].data());
    int axis = 0;
    for (int k = 1; k < 3; ++k)
      if (total_key(cb.hi[k] - cb.lo[k]) >= total_key(cb.hi[axis] - cb.lo[axis])) axis = k;
    size_t mid = n / 2;
    std::sort(order, order + n, [&](uint32_t a, uint32_t b) {
      int32_t ka = total_key(centroids[a][axis]), kb = total_key(centroids[b][axis]);
      return ka != kb ? ka < kb : a < b;
    });
    size_t node = nodes.size() / 16;
    nodes.resize(nodes.size() + 16, 0);
    R a = subtree(order, mid);
    R b = subtree(order + mid, n - mid);
    uint32_t* w = &nodes[node * 16];
    for (int k = 0; k < 3; ++k) w[k] = fbits(a.lo[k]), w[3 + k] = fbits(a.hi[k]);
    for (int k = 0; k < 3; ++k) w[6 + k] = fbits(b.lo[k]), w[9 + k] = fbits(b.hi[k]);
    w[12] = a.id;
    w[13] = b.id;
    R r;
    r.id = (uint32_t)node;
    for (int k = 0; k < 3; ++k) r.lo[k] = rmin(a.lo[k], b.lo[k]), r.hi[k] = rmax(a.hi[k], b.hi[k]);
    return r;
  }
  R leaf(const uint32_t* order, size_t n) {
    uint32_t first = (uint32_t)(triangles.size() / RS_TRIANGLE_WORDS);
    Box bb = empty_box();
    for (size_t k = 0; k < n; ++k) {
      uint32_t t = order[k];
      const float* a = pos + 3 * (size_t)idx[3 * t];
      const float* b = pos + 3 * (size_t)idx[3 * t + 1];
      const float* c = pos + 3 * (size_t)idx[3 * t + 2];
      for (int i = 0; i < 3; ++i) triangles.push_back(fbits(a[i]));
      for (int i = 0; i < 3; ++i) triangles.push_back(fbits(b[i] - a[i]));
      for (int i = 0; i < 3; ++i) triangles.push_back(fbits(c[i] - a[i]));
      triangles.push_back(t);
      triangles.push_back(0);
      triangles.push_back(0);
      add_point(bb, a);
      add_point(bb, b);
      add_point(bb, c);
    }
    return R{RS_LEAF | first << 3 | (uint32_t)n, bb.lo, bb.hi};
  }
};
}  // namespace

// reflection_software.rs:170-198. The order of triangles inside a leaf follows a full sort by
// (centroid, index); Rust's select_nth_unstable leaves it unspecified.
bool rs_build_median(const float* pos, const uint32_t* idx, size_t nidx, RsMesh& out) {
  size_t count = nidx / 3;
  if (count == 0 || count >= (1u << 28)) return false;
  MedianBuilder b;
  b.pos = pos;
  b.idx = idx;
  b.centroids.resize(count);
  for (size_t t = 0; t < count; ++t)
    for (int a = 0; a < 3; ++a)
      b.centroids[t][a] = (pos[3 * (size_t)idx[3 * t] + a] + pos[3 * (size_t)idx[3 * t + 1] + a] +
                           pos[3 * (size_t)idx[3 * t + 2] + a]) / 3.0f;
  std::vector<uint32_t> order(count);
  for (size_t t = 0; t < count; ++t) order[t] = (uint32_t)t;
  MedianBuilder::R r = b.subtree(order.data(), count);
  out.nodes = std::move(b.nodes);
  out.triangles = std::move(b.triangles);
  out.root = r.id;
  out.lo = r.lo;
  out.hi = r.hi;
  out.wide = false;
  return true;
}

// reflection_software.rs:285-388 and the caller's sequence (primary_ray_gpu.rs:3640-3662):
// pack, instance_words, pad to the traced count, place, finish_scene_bounds.
bool rs_pack(const std::vector<RsMesh>& meshes, const std::vector<RsInstance>& inst, int tlas_mode,
             bool bvh4, std::vector<uint32_t>& words, std::string& err) {
  size_t n = inst.size();
  size_t records = RS_HEADER + n * RS_INSTANCE + tlas_reserve(n) + (bvh4 ? 8 : 0);
  size_t at = records;
  std::vector<std::array<uint32_t, 2>> bases;
  size_t total = records;
  for (const RsMesh& m : meshes) total += m.nodes.size() + m.triangles.size();
  words.assign(std::max(total, RS_HEADER), 0);
  for (const RsMesh& m : meshes) {
    uint32_t nb = (uint32_t)at;
    std::copy(m.nodes.begin(), m.nodes.end(), words.begin() + at);
    at += m.nodes.size();
    uint32_t tb = (uint32_t)at;
    std::copy(m.triangles.begin(), m.triangles.end(), words.begin() + at);
    at += m.triangles.size();
    bases.push_back({nb, tb});
  }
  // instance_words (reflection_software.rs:347-368)
  std::vector<uint32_t> out(RS_HEADER, 0);
  if (bvh4) out[4] = (uint32_t)(records - 8);
  uint32_t count = 0;
  for (const RsInstance& g : inst) {
    if (g.mesh >= meshes.size()) {
      err = "instance mesh index";
      return false;
    }
    if (singular(g.model, g.rows)) continue;
    const RsMesh& m = meshes[g.mesh];
    for (int k = 0; k < 12; ++k) out.push_back(fbits(g.rows[k]));
    // world_bounds (reflection_software.rs:373-388)
    Box bb = empty_box();
    for (int c = 0; c < 8; ++c) {
      float p[3] = {(c & 1) ? m.hi[0] : m.lo[0], (c & 2) ? m.hi[1] : m.lo[1], (c & 4) ? m.hi[2] : m.lo[2]};
      float w[3];
      transform_point(g.model, p, w);
      add_point(bb, w);
    }
    float margin = 0.0f;
    for (int a = 0; a < 3; ++a)
      margin = rmax(margin, rmax(rmax(std::fabs(bb.hi[a]), std::fabs(bb.lo[a])), bb.hi[a] - bb.lo[a]));
    margin = margin * 1e-5f;
    for (int a = 0; a < 3; ++a) out.push_back(fbits(bb.lo[a] - margin));
    for (int a = 0; a < 3; ++a) out.push_back(fbits(bb.hi[a] + margin));
    out.push_back(bases[g.mesh][0]);
    out.push_back(bases[g.mesh][1]);
    out.push_back(m.root);
    out.push_back(g.slot);
    out.push_back(g.casts ? 0u : 1u);
    out.push_back(0);
    count += 1;
  }
  out[0] = count;
  out.resize(RS_HEADER + n * RS_INSTANCE, 0);
  tlas_place(out, RS_HEADER, RS_INSTANCE, n, {}, tlas_mode, bvh4, true);
  if (bvh4) {
    // finish_scene_bounds (reflection_software.rs:295-313)
    Box bb = empty_box();
    for (size_t i = 0; i < out[0]; ++i) {
      size_t r = RS_HEADER + i * RS_INSTANCE;
      for (int a = 0; a < 3; ++a) {
        bb.lo[a] = rmin(bb.lo[a], bitsf(out[r + 12 + a]));
        bb.hi[a] = rmax(bb.hi[a], bitsf(out[r + 15 + a]));
      }
    }
    out[4] = (uint32_t)out.size();
    for (int a = 0; a < 3; ++a) out.push_back(fbits(bb.lo[a]));
    out.push_back(0);
    for (int a = 0; a < 3; ++a) out.push_back(fbits(bb.hi[a]));
    out.push_back(0);
  }
  std::copy(out.begin(), out.end(), words.begin());
  return true;
}

}  // namespace orc
