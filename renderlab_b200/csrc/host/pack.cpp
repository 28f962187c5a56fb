// Packed-buffer writers for the two layouts the traversal reads.
//
// GI (`gi_geometry`, src/gi_bvh.rs:151-274 with the extra words of gi_cache.rs:4388-4488):
//   [16-word header][32-word instance records][top-level reserve][per mesh: 16-word nodes,
//   2-word leaves, 3-word positions, indices, optional primitive table]
// Reflection (`rl_geometry`, src/reflection_software.rs:285-388, primary_ray_gpu.rs:3640-3662):
//   [8-word header][24-word records][top-level reserve][8 scene-bounds words]
//   [per mesh: 16-word nodes with leaf tags LEAF | first << 4 | count, 12-word triangles]
// Word-level formats are the reference's; instance rows are taken from the caller (the
// reference derives them with glam's Mat4::inverse, which is not restated here).
#include <algorithm>
#include <unordered_map>

#include "host.hpp"

namespace rtb {

namespace {

// glam Mat4::transform_point3 for an affine model: x*px, + y*py, + z*pz, + w, rounded in turn.
void to_world(const float* m, const float* p, float* out) {
  for (int r = 0; r < 3; ++r) {
    float acc = m[4 * r] * p[0];
    acc = m[4 * r + 1] * p[1] + acc;
    acc = m[4 * r + 2] * p[2] + acc;
    out[r] = m[4 * r + 3] + acc;
  }
}

}  // namespace

bool is_singular(const Placement& g) {
  const float* m = g.model;
  double det = (double)m[0] * ((double)m[5] * m[10] - (double)m[6] * m[9]) -
               (double)m[1] * ((double)m[4] * m[10] - (double)m[6] * m[8]) +
               (double)m[2] * ((double)m[4] * m[9] - (double)m[5] * m[8]);
  if (det == 0.0) return true;
  for (float r : g.rows)
    if (!std::isfinite(r)) return true;
  return false;
}

namespace {

struct TriKey {
  uint32_t a, b, c;
  bool operator==(const TriKey& o) const { return a == o.a && b == o.b && c == o.c; }
};
struct TriHash {
  size_t operator()(const TriKey& k) const {
    uint64_t h = k.a * 0x9E3779B97F4A7C15ull ^ (k.b + 0x632BE59BD9B4E019ull) * 0xC2B2AE3D27D4EB4Full;
    return (size_t)(h ^ (k.c * 0x165667B19E3779F9ull));
  }
};

// gi_bvh.rs:108-136 / reflection_software.rs:132-158: the source primitive of each reordered
// triangle; duplicates of one index triple take ascending source ids. Empty when unmatched.
std::vector<uint32_t> source_primitives(const std::vector<uint32_t>& bvh_idx, const uint32_t* src, size_t nsrc) {
  const size_t n = nsrc / 3, m = bvh_idx.size() / 3;
  if (n == 0 || m == 0) return {};
  std::unordered_map<TriKey, uint32_t, TriHash> head;
  head.reserve(n * 2);
  std::vector<uint32_t> next(n, EMPTY);
  for (size_t id = n; id-- > 0;) {
    TriKey k{src[3 * id], src[3 * id + 1], src[3 * id + 2]};
    auto [it, fresh] = head.try_emplace(k, (uint32_t)id);
    if (!fresh) {
      next[id] = it->second;
      it->second = (uint32_t)id;
    }
  }
  std::vector<uint32_t> out(m);
  for (size_t t = 0; t < m; ++t) {
    auto it = head.find(TriKey{bvh_idx[3 * t], bvh_idx[3 * t + 1], bvh_idx[3 * t + 2]});
    if (it == head.end() || it->second == EMPTY) return {};
    out[t] = it->second;
    it->second = next[it->second];
  }
  return out;
}

void world_box(const float* model, const Aabb& obj, Aabb& out) {
  out = Aabb::empty();
  for (int c = 0; c < 8; ++c) {
    float p[3], w[3];
    for (int a = 0; a < 3; ++a) p[a] = (c & (1 << a)) ? obj.hi[a] : obj.lo[a];
    to_world(model, p, w);
    out.grow(w);
  }
}

// Blas::near_base (gi_bvh.rs:95-104): the base of the first masks cooked under exactly this
// model's bits (an affine model: the column-major transform's last row is 0, 0, 0, 1), else 0.
uint32_t near_base(const float* model, const std::vector<NearMasks>& near, const std::vector<size_t>& bases) {
  for (size_t k = 0; k < near.size(); ++k) {
    const float* t = near[k].transform;
    bool same = as_bits(t[3]) == 0 && as_bits(t[7]) == 0 && as_bits(t[11]) == 0 && as_bits(t[15]) == as_bits(1.0f);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 4; ++c) same = same && as_bits(model[4 * r + c]) == as_bits(t[4 * c + r]);
    if (same) return (uint32_t)bases[k];
  }
  return 0;
}

}  // namespace

void instance_box(uint32_t layout, const float* model, const Aabb& obj, float lo[3], float hi[3]) {
  Aabb wb;
  world_box(model, obj, wb);
  if (layout == 0) {  // gi_bvh.rs:236-262: a pad per axis
    for (int a = 0; a < 3; ++a) {
      const float pad = 1e-5f * (1.0f + hi_of(std::fabs(wb.lo[a]), std::fabs(wb.hi[a])));
      lo[a] = wb.lo[a] - pad, hi[a] = wb.hi[a] + pad;
    }
    return;
  }
  // world_bounds (reflection_software.rs:373-388): one margin from the largest coordinate or
  // extent over the three axes.
  float margin = 0.0f;
  for (int a = 0; a < 3; ++a)
    margin = hi_of(margin, hi_of(hi_of(std::fabs(wb.hi[a]), std::fabs(wb.lo[a])), wb.hi[a] - wb.lo[a]));
  margin = margin * 1e-5f;
  for (int a = 0; a < 3; ++a) lo[a] = wb.lo[a] - margin, hi[a] = wb.hi[a] + margin;
}

bool move_instances(uint32_t layout, uint32_t* w, size_t n_words, const std::vector<Placement>& inst,
                    const std::vector<Aabb>& mesh_boxes, std::string& err) {
  const size_t header = layout == 0 ? 16 : 8, stride = layout == 0 ? 32 : 24;
  const uint32_t count = w[0];
  if (inst.size() != count || (layout == 0 && w[4] > count))  // GI word 4: a see-through tail
    return err = "moved instances must be the scene's instances, in record order", false;
  if (header + stride * (size_t)count > n_words) return err = "instance records exceed the words", false;
  std::vector<Aabb> boxes(count);
  for (uint32_t i = 0; i < count; ++i) {
    const Placement& g = inst[i];
    if (g.mesh >= mesh_boxes.size()) return err = "instance mesh index out of range", false;
    if (is_singular(g)) return err = "a moved instance is singular", false;
    uint32_t* r = w + header + stride * (size_t)i;
    for (int k = 0; k < 12; ++k) r[k] = as_bits(g.rows[k]);
    instance_box(layout, g.model, mesh_boxes[g.mesh], boxes[i].lo, boxes[i].hi);
    for (int a = 0; a < 3; ++a) r[12 + a] = as_bits(boxes[i].lo[a]), r[15 + a] = as_bits(boxes[i].hi[a]);
  }
  const size_t base = layout == 0 ? w[1] : (w[1] & ~3u);
  if (w[1] != 0 && count >= 2) {  // instance_bvh::place, a moved set (the same records, new boxes)
    if (base + tlas_reserve(count) > n_words) return err = "top level exceeds the words", false;
    if (w[3] < TLAS_REFITS) {
      w[3] += 1;
      tlas_refit(w + base, boxes);
    } else {
      std::vector<uint32_t> nodes = tlas_build(boxes, true);
      std::fill(w + base, w + base + tlas_reserve(count), 0u);
      std::copy(nodes.begin(), nodes.end(), w + base);
      w[3] = 0;
    }
  }
  if (layout == 1) {  // finish_scene_bounds (reflection_software.rs:295-313)
    Aabb scene = Aabb::empty();
    for (const Aabb& b : boxes) scene.grow(b);
    const size_t at = w[4];
    if (at + 8 > n_words) return err = "scene bounds exceed the words", false;
    for (int a = 0; a < 3; ++a) w[at + a] = as_bits(scene.lo[a]), w[at + 4 + a] = as_bits(scene.hi[a]);
  }
  return true;
}

bool pack_gi(const std::vector<MeshRef>& meshes, const std::vector<Placement>& inst, int tlas_mode,
             std::vector<uint32_t>& out, std::string& err) {
  const size_t n = inst.size();
  size_t at = 16 + 32 * n + tlas_reserve(n);
  std::vector<std::array<uint32_t, 4>> base(meshes.size());
  std::vector<std::vector<uint32_t>> prims(meshes.size());
  for (size_t m = 0; m < meshes.size(); ++m) {
    const Blas& b = *meshes[m].blas;
    if (meshes[m].primitives) prims[m] = source_primitives(b.indices, meshes[m].indices, meshes[m].n_indices);
    base[m][0] = (uint32_t)at;
    base[m][1] = base[m][0] + (uint32_t)b.nodes.size();
    base[m][2] = base[m][1] + (uint32_t)b.leaves.size();
    base[m][3] = base[m][2] + (uint32_t)b.positions.size();
    at = base[m][3] + b.indices.size() + prims[m].size();
  }
  // gi_bvh.rs:165-177: every mesh's near-field masks after all the records, mesh by mesh.
  std::vector<std::vector<size_t>> near(meshes.size());
  for (size_t m = 0; m < meshes.size(); ++m)
    for (const NearMasks& q : meshes[m].near) {
      near[m].push_back(at);
      at += q.n_masks;
    }
  if (at >= (size_t)UINT32_MAX) {
    err = "packed GI geometry exceeds 2^32 words";
    return false;
  }
  std::vector<uint32_t> head(16 + 32 * n, 0);
  head[0] = (uint32_t)n;
  for (size_t i = 0; i < n; ++i) {
    const Placement& g = inst[i];
    if (g.mesh >= meshes.size()) {
      err = "instance mesh index out of range";
      return false;
    }
    if (is_singular(g)) {
      err = "indirect geometry transform is singular";  // gi_bvh.rs:236-241
      return false;
    }
    const Blas& b = *meshes[g.mesh].blas;
    uint32_t* r = &head[16 + 32 * i];
    for (int k = 0; k < 12; ++k) r[k] = as_bits(g.rows[k]);
    float lo[3], hi[3];
    instance_box(0, g.model, b.bounds, lo, hi);
    for (int a = 0; a < 3; ++a) r[12 + a] = as_bits(lo[a]), r[15 + a] = as_bits(hi[a]);
    for (int k = 0; k < 4; ++k) r[18 + k] = base[g.mesh][k];
    r[22] = b.root;
    r[23] = meshes[g.mesh].near.empty() ? g.near_base : near_base(g.model, meshes[g.mesh].near, near[g.mesh]);
    for (int k = 0; k < 8; ++k) r[24 + k] = g.extra[k];
    r[28] = prims[g.mesh].empty() ? 0u : base[g.mesh][3] + (uint32_t)b.indices.size();
  }
  tlas_place(head, 16, 32, n, tlas_mode);
  out.assign(at, 0);
  std::copy(head.begin(), head.end(), out.begin());
  for (size_t m = 0; m < meshes.size(); ++m) {
    const Blas& b = *meshes[m].blas;
    uint32_t* w = out.data() + base[m][0];
    std::copy(b.nodes.begin(), b.nodes.end(), w);
    std::copy(b.leaves.begin(), b.leaves.end(), out.data() + base[m][1]);
    uint32_t* p = out.data() + base[m][2];
    for (size_t k = 0; k < b.positions.size(); ++k) p[k] = as_bits(b.positions[k]);
    std::copy(b.indices.begin(), b.indices.end(), out.data() + base[m][3]);
    std::copy(prims[m].begin(), prims[m].end(), out.data() + base[m][3] + b.indices.size());
    for (size_t k = 0; k < meshes[m].near.size(); ++k)
      std::copy(meshes[m].near[k].masks, meshes[m].near[k].masks + meshes[m].near[k].n_masks, out.data() + near[m][k]);
  }
  return true;
}

bool pack_reflection(const std::vector<MeshRef>& meshes, const std::vector<Placement>& inst,
                     int tlas_mode, std::vector<uint32_t>& out, std::string& err) {
  const size_t n = inst.size();
  const size_t records = 8 + 24 * n + tlas_reserve(n) + 8;
  // reflection_software.rs:108-168: tagged nodes and pre-edged triangles per mesh.
  std::vector<std::array<uint32_t, 2>> base(meshes.size());
  std::vector<Aabb> obj(meshes.size());
  std::vector<uint32_t> roots(meshes.size());
  size_t at = records;
  std::vector<std::vector<uint32_t>> prims(meshes.size());
  for (size_t m = 0; m < meshes.size(); ++m) {
    const Blas& b = *meshes[m].blas;
    if (b.indices.size() / 3 >= (1u << 27)) {
      err = "mesh too large for a reflection leaf tag";
      return false;
    }
    prims[m] = source_primitives(b.indices, meshes[m].indices, meshes[m].n_indices);
    if (prims[m].size() != b.indices.size() / 3) {
      err = "reflection triangles do not map to source primitives";
      return false;
    }
    base[m][0] = (uint32_t)at;
    base[m][1] = (uint32_t)(at + b.nodes.size());
    at += b.nodes.size() + 12 * (b.indices.size() / 3);
    Aabb ob = Aabb::empty();
    for (size_t k = 0; k < meshes[m].n_indices; ++k) ob.grow(meshes[m].positions + 3 * (size_t)meshes[m].indices[k]);
    obj[m] = ob;
  }
  if (at >= (size_t)UINT32_MAX) {
    err = "packed reflection geometry exceeds 2^32 words";
    return false;
  }
  out.assign(at, 0);
  for (size_t m = 0; m < meshes.size(); ++m) {
    const Blas& b = *meshes[m].blas;
    auto tag = [&](uint32_t c) -> uint32_t {
      if (c == EMPTY || !(c & LEAF)) return c;
      uint32_t l = c & ~LEAF;
      return LEAF | ((b.leaves[2 * l] / 3) << 4) | (b.leaves[2 * l + 1] / 3);
    };
    uint32_t* w = out.data() + base[m][0];
    for (size_t k = 0; k < b.node_count(); ++k) {
      std::copy(&b.nodes[16 * k], &b.nodes[16 * k] + 16, w + 16 * k);
      for (int s = 0; s < 4; ++s) w[16 * k + 6 + s] = tag(b.nodes[16 * k + 6 + s]);
    }
    roots[m] = tag(b.root);
    uint32_t* t = out.data() + base[m][1];
    const float* P = meshes[m].positions;
    for (size_t k = 0; k < b.indices.size() / 3; ++k, t += 12) {
      const float* a = P + 3 * (size_t)b.indices[3 * k];
      const float* bb = P + 3 * (size_t)b.indices[3 * k + 1];
      const float* cc = P + 3 * (size_t)b.indices[3 * k + 2];
      for (int j = 0; j < 3; ++j) {
        t[j] = as_bits(a[j]);
        t[3 + j] = as_bits(bb[j] - a[j]);
        t[6 + j] = as_bits(cc[j] - a[j]);
      }
      t[9] = prims[m][k];
    }
  }
  // reflection_software.rs:347-368: singular placements are skipped, their records stay zero.
  std::vector<uint32_t> head(8, 0);
  head[4] = (uint32_t)(records - 8);
  uint32_t count = 0;
  for (const Placement& g : inst) {
    if (g.mesh >= meshes.size()) {
      err = "instance mesh index out of range";
      return false;
    }
    if (is_singular(g)) continue;
    for (int k = 0; k < 12; ++k) head.push_back(as_bits(g.rows[k]));
    float lo[3], hi[3];
    instance_box(1, g.model, obj[g.mesh], lo, hi);
    for (int a = 0; a < 3; ++a) head.push_back(as_bits(lo[a]));
    for (int a = 0; a < 3; ++a) head.push_back(as_bits(hi[a]));
    head.push_back(base[g.mesh][0]);
    head.push_back(base[g.mesh][1]);
    head.push_back(roots[g.mesh]);
    head.push_back(g.slot);
    head.push_back(g.casts_shadow ? 0u : 1u);
    head.push_back(0);
    ++count;
  }
  head[0] = count;
  head.resize(8 + 24 * n, 0);
  tlas_place(head, 8, 24, n, tlas_mode);
  // finish_scene_bounds (reflection_software.rs:295-313)
  Aabb scene = Aabb::empty();
  for (uint32_t i = 0; i < count; ++i) {
    const uint32_t* r = &head[8 + 24 * (size_t)i];
    for (int a = 0; a < 3; ++a) {
      scene.lo[a] = lo_of(scene.lo[a], as_float(r[12 + a]));
      scene.hi[a] = hi_of(scene.hi[a], as_float(r[15 + a]));
    }
  }
  head[4] = (uint32_t)head.size();
  for (int a = 0; a < 3; ++a) head.push_back(as_bits(scene.lo[a]));
  head.push_back(0);
  for (int a = 0; a < 3; ++a) head.push_back(as_bits(scene.hi[a]));
  head.push_back(0);
  std::copy(head.begin(), head.end(), out.begin());
  return true;
}

}  // namespace rtb
