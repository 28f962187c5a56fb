// CPU ORACLE — test infrastructure only. Restates crates/asset/src/near_field.rs:172-537 (the
// BVH4-Q8 builder, quantiser and refit) and the enclosure checks of
// crates/asset/src/cluster_bvh.rs:170-264.
#include <algorithm>
#include <cfloat>
#include <limits>

#include "oracle.hpp"

namespace orc {

namespace {

Box empty_box() {
  const float inf = std::numeric_limits<float>::infinity();
  return Box{{inf, inf, inf}, {-inf, -inf, -inf}};
}
// near_field.rs:278-283 `merge` and :527-537 `bounds`
Box merge(const Box& a, const Box& b) {
  Box r;
  for (int i = 0; i < 3; ++i) {
    r.lo[i] = rmin(a.lo[i], b.lo[i]);
    r.hi[i] = rmax(a.hi[i], b.hi[i]);
  }
  return r;
}
Box add_point(const Box& a, const float* p) {
  Box r;
  for (int i = 0; i < 3; ++i) {
    r.lo[i] = rmin(a.lo[i], p[i]);
    r.hi[i] = rmax(a.hi[i], p[i]);
  }
  return r;
}
// Rust `f as usize`: NaN and negatives give 0, values past the range saturate.
size_t sat_usize(float f) {
  if (!(f > 0.0f)) return 0;
  if (f >= 1.8e19f) return SIZE_MAX;
  return (size_t)f;
}
// Rust `f.clamp(0.0, 255.0) as u8` (NaN gives 0).
uint8_t sat_u8(float f) {
  if (!(f > 0.0f)) return 0;
  if (f >= 255.0f) return 255;
  return (uint8_t)f;
}
// near_field.rs:274-277
float half_area(const V3& lo, const V3& hi) {
  float e[3];
  for (int a = 0; a < 3; ++a) e[a] = rmax(hi[a] - lo[a], 0.0f);
  return e[0] * e[1] + e[1] * e[2] + e[2] * e[0];
}

struct Builder {
  const float* pos;  // xyz per vertex
  const uint32_t* idx;
  std::vector<V3> centroids;
  std::vector<Box> boxes;  // empty for the median build
  Bvh bvh;

  const float* P(uint32_t i) const { return pos + 3 * (size_t)i; }

  // near_field.rs:286-306
  uint32_t subtree(std::vector<uint32_t> tris) {
    if (tris.size() <= LEAF_TRIANGLES) return leaf(tris);
    std::vector<std::vector<uint32_t>> groups;
    groups.push_back(std::move(tris));
    for (int round = 0; round < 2; ++round) {
      std::vector<std::vector<uint32_t>> next;
      for (auto& g : groups) {
        if (g.size() <= LEAF_TRIANGLES) {
          next.push_back(std::move(g));
          continue;
        }
        std::vector<uint32_t> a, b;
        split(g, a, b);
        next.push_back(std::move(a));
        next.push_back(std::move(b));
      }
      groups = std::move(next);
    }
    std::vector<uint32_t> children;
    for (auto& g : groups) children.push_back(subtree(std::move(g)));
    return node(children);
  }
  // near_field.rs:307-314
  void split(const std::vector<uint32_t>& g, std::vector<uint32_t>& a, std::vector<uint32_t>& b) {
    if (!boxes.empty() && split_sah(g, a, b)) return;
    split_median(g, a, b);
  }
  Box centroid_bounds(const std::vector<uint32_t>& g) const {
    Box r = empty_box();
    for (uint32_t t : g) r = add_point(r, centroids[t].data());
    return r;
  }
  // near_field.rs:317-366
  bool split_sah(const std::vector<uint32_t>& g, std::vector<uint32_t>& a,
                 std::vector<uint32_t>& b) const {
    Box cb = centroid_bounds(g);
    bool have = false;
    float best_cost = 0;
    int best_axis = 0;
    size_t best_plane = 0;
    for (int axis = 0; axis < 3; ++axis) {
      float extent = cb.hi[axis] - cb.lo[axis];
      if (std::isnan(extent) || extent <= 0.0f) continue;
      auto bin = [&](uint32_t t) {
        float f = (centroids[t][axis] - cb.lo[axis]) / extent * (float)SAH_BINS;
        return std::min(sat_usize(f), SAH_BINS - 1);
      };
      size_t count[SAH_BINS] = {};
      Box bb[SAH_BINS];
      for (auto& x : bb) x = empty_box();
      for (uint32_t t : g) {
        size_t k = bin(t);
        count[k] += 1;
        bb[k] = merge(bb[k], boxes[t]);
      }
      float right[SAH_BINS] = {};
      Box acc = empty_box();
      size_t n = 0;
      for (size_t k = SAH_BINS - 1; k >= 1; --k) {
        acc = merge(acc, bb[k]);
        n += count[k];
        right[k] = half_area(acc.lo, acc.hi) * (float)n;
      }
      acc = empty_box();
      n = 0;
      for (size_t k = 0; k + 1 < SAH_BINS; ++k) {
        acc = merge(acc, bb[k]);
        n += count[k];
        if (n == 0 || n == g.size()) continue;
        float cost = half_area(acc.lo, acc.hi) * (float)n + right[k + 1];
        if (!have || cost < best_cost) {
          have = true;
          best_cost = cost;
          best_axis = axis;
          best_plane = k;
        }
      }
    }
    if (!have) return false;
    float extent = cb.hi[best_axis] - cb.lo[best_axis];
    for (uint32_t t : g) {
      float f = (centroids[t][best_axis] - cb.lo[best_axis]) / extent * (float)SAH_BINS;
      if (std::min(sat_usize(f), SAH_BINS - 1) <= best_plane) a.push_back(t); else b.push_back(t);
    }
    return true;
  }
  // near_field.rs:367-379. Iterator::max_by keeps the last of equal maxima.
  void split_median(std::vector<uint32_t> g, std::vector<uint32_t>& a,
                    std::vector<uint32_t>& b) const {
    Box cb = centroid_bounds(g);
    int axis = 0;
    for (int k = 1; k < 3; ++k)
      if (total_key(cb.hi[k] - cb.lo[k]) >= total_key(cb.hi[axis] - cb.lo[axis])) axis = k;
    std::sort(g.begin(), g.end(), [&](uint32_t x, uint32_t y) {
      int32_t kx = total_key(centroids[x][axis]), ky = total_key(centroids[y][axis]);
      return kx != ky ? kx < ky : x < y;
    });
    size_t half = g.size() / 2;
    a.assign(g.begin(), g.begin() + half);
    b.assign(g.begin() + half, g.end());
  }
  // near_field.rs:380-401
  uint32_t leaf(const std::vector<uint32_t>& tris) {
    uint32_t offset = (uint32_t)bvh.indices.size();
    for (uint32_t t : tris)
      for (int k = 0; k < 3; ++k) bvh.indices.push_back(idx[3 * (size_t)t + k]);
    uint32_t id = (uint32_t)bvh.leaves.size();
    bvh.leaves.push_back(Leaf{offset, (uint32_t)(tris.size() * 3), tris[0] * 3});
    return id | LEAF_BIT;
  }
  // near_field.rs:402-430
  Box child_bounds(uint32_t child) const {
    if (child & LEAF_BIT) {
      const Leaf& l = bvh.leaves[child & ~LEAF_BIT];
      Box r = empty_box();
      for (uint32_t k = l.offset; k < l.offset + l.count; ++k) r = add_point(r, P(bvh.indices[k]));
      return r;
    }
    const Node& n = bvh.nodes[child];
    Box r = empty_box();
    for (int slot = 0; slot < 4; ++slot) {
      if (n.children[slot] == EMPTY) continue;
      for (int fused = 0; fused < 2; ++fused)
        for (int axis = 0; axis < 3; ++axis) {
          r.lo[axis] = rmin(r.lo[axis], decode_plane(n, axis, n.lower[axis][slot], fused));
          r.hi[axis] = rmax(r.hi[axis], decode_plane(n, axis, n.upper[axis][slot], fused));
        }
    }
    return r;
  }
  // near_field.rs:431-437
  uint32_t node(const std::vector<uint32_t>& children) {
    std::vector<Box> bs;
    for (uint32_t c : children) bs.push_back(child_bounds(c));
    Node nd = quantized_node(children.data(), bs.data(), children.size());
    uint32_t id = (uint32_t)bvh.nodes.size();
    bvh.nodes.push_back(nd);
    return id;
  }
};

}  // namespace

// near_field.rs:481-525
Node quantized_node(const uint32_t* children, const Box* boxes, size_t n) {
  Box all = empty_box();
  for (size_t i = 0; i < n; ++i) all = merge(all, boxes[i]);
  Node node;
  std::memset(&node, 0, sizeof node);
  for (int a = 0; a < 3; ++a) node.origin[a] = all.lo[a];
  for (int s = 0; s < 4; ++s) node.children[s] = EMPTY;
  for (int axis = 0; axis < 3; ++axis) {
    float lo = all.lo[axis], hi = all.hi[axis];
    float extent = hi - lo;
    float step = rmax(extent / 255.0f, rmax(FLT_MIN, std::fabs(lo) * 1e-7f));
    while (lo + step * 255.0f < hi || std::fma(step, 255.0f, lo) < hi)
      step *= 1.0f + 1.0f / 1048576.0f;
    node.step[axis] = step;
  }
  for (size_t slot = 0; slot < n; ++slot) {
    node.children[slot] = children[slot];
    for (int axis = 0; axis < 3; ++axis) {
      float o = node.origin[axis], s = node.step[axis];
      auto dec_u = [&](uint8_t q) { return o + s * (float)q; };
      auto dec_f = [&](uint8_t q) { return std::fma(s, (float)q, o); };
      float a = boxes[slot].lo[axis], b = boxes[slot].hi[axis];
      uint8_t low = sat_u8(std::floor((a - o) / s));
      while (low > 0 && (dec_u(low) > a || dec_f(low) > a)) low -= 1;
      uint8_t high = sat_u8(std::ceil((b - o) / s));
      while (high < 255 && (dec_u(high) < b || dec_f(high) < b)) high += 1;
      node.lower[axis][slot] = low;
      node.upper[axis][slot] = high;
    }
  }
  return node;
}

// near_field.rs:206-262
bool build_bvh(const float* pos, size_t npos, const uint32_t* idx, size_t nidx, bool sah,
               Bvh& out, std::string& err) {
  if (nidx == 0 || nidx % 3 != 0) {
    err = "BVH geometry needs a nonempty triangle list";
    return false;
  }
  for (size_t i = 0; i < nidx; ++i)
    if (idx[i] >= npos) {
      err = "BVH geometry has an invalid index or position";
      return false;
    }
  for (size_t i = 0; i < npos * 3; ++i)
    if (!std::isfinite(pos[i])) {
      err = "BVH geometry has an invalid index or position";
      return false;
    }
  size_t nt = nidx / 3;
  Builder bld;
  bld.pos = pos;
  bld.idx = idx;
  bld.centroids.resize(nt);
  for (size_t t = 0; t < nt; ++t)
    for (int a = 0; a < 3; ++a) {
      // `Sum for f32` starts from -0.0, which leaves the first term unchanged.
      float s = pos[3 * (size_t)idx[3 * t] + a];
      s = s + pos[3 * (size_t)idx[3 * t + 1] + a];
      s = s + pos[3 * (size_t)idx[3 * t + 2] + a];
      bld.centroids[t][a] = s / 3.0f;
    }
  if (sah) {
    bld.boxes.resize(nt);
    for (size_t t = 0; t < nt; ++t) {
      Box b = empty_box();
      for (int k = 0; k < 3; ++k) b = add_point(b, pos + 3 * (size_t)idx[3 * t + k]);
      bld.boxes[t] = b;
    }
  }
  bld.bvh.positions.resize(npos);
  for (size_t i = 0; i < npos; ++i)
    bld.bvh.positions[i] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], 0.0f};
  std::vector<uint32_t> all(nt);
  for (size_t t = 0; t < nt; ++t) all[t] = (uint32_t)t;
  uint32_t root = bld.subtree(std::move(all));
  out = std::move(bld.bvh);
  out.root = root;
  if (!validate_bvh(out, err)) return false;
  return true;
}

// near_field.rs:192-204
size_t bvh_depth(const Bvh& b, uint32_t child) {
  if (child & LEAF_BIT) return 0;
  const Node& n = b.nodes[child];
  size_t m = 0;
  for (uint32_t c : n.children)
    if (c != EMPTY) m = std::max(m, bvh_depth(b, c));
  return 1 + m;
}

// near_field.rs:184-190
bool build_bvh_sah(const float* pos, size_t npos, const uint32_t* idx, size_t nidx, Bvh& out,
                   std::string& err) {
  if (!build_bvh(pos, npos, idx, nidx, true, out, err)) return false;
  if (bvh_depth(out, out.root) > MAX_SAH_DEPTH) return build_bvh(pos, npos, idx, nidx, false, out, err);
  return true;
}

// near_field.rs:445-478
bool refit_bvh(Bvh& b, const float* pos, size_t npos, std::string& err) {
  if (npos != b.positions.size()) {
    err = "BVH refit needs finite positions of the same vertices";
    return false;
  }
  for (size_t i = 0; i < npos * 3; ++i)
    if (!std::isfinite(pos[i])) {
      err = "BVH refit needs finite positions of the same vertices";
      return false;
    }
  for (size_t i = 0; i < npos; ++i) b.positions[i] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], 0.0f};
  for (size_t n = 0; n < b.nodes.size(); ++n) {
    std::vector<uint32_t> ch;
    for (uint32_t c : b.nodes[n].children)
      if (c != EMPTY) ch.push_back(c);
    std::vector<Box> bs;
    for (uint32_t c : ch) {
      Box r = empty_box();
      if (c & LEAF_BIT) {
        const Leaf& l = b.leaves[c & ~LEAF_BIT];
        for (uint32_t k = l.offset; k < l.offset + l.count; ++k) r = add_point(r, pos + 3 * (size_t)b.indices[k]);
      } else {
        const Node& m = b.nodes[c];
        for (int slot = 0; slot < 4; ++slot) {
          if (m.children[slot] == EMPTY) continue;
          for (int fused = 0; fused < 2; ++fused)
            for (int axis = 0; axis < 3; ++axis) {
              r.lo[axis] = rmin(r.lo[axis], decode_plane(m, axis, m.lower[axis][slot], fused));
              r.hi[axis] = rmax(r.hi[axis], decode_plane(m, axis, m.upper[axis][slot], fused));
            }
        }
      }
      bs.push_back(r);
    }
    b.nodes[n] = quantized_node(ch.data(), bs.data(), ch.size());
  }
  return true;
}

// cluster_bvh.rs:170-264, the checks a one-level build can fail: ranges, postorder, and
// enclosure of every child under both decodes (in f64).
bool validate_bvh(const Bvh& b, std::string& err) {
  size_t end = 0;
  for (const Leaf& l : b.leaves) {
    if (l.offset != end || l.count == 0 || l.count % 3 != 0) {
      err = "invalid cluster BVH leaf";
      return false;
    }
    end = l.offset + l.count;
  }
  if (end != b.indices.size()) {
    err = "unowned cluster BVH indices";
    return false;
  }
  for (uint32_t i : b.indices)
    if (i >= b.positions.size()) {
      err = "cluster BVH vertex index";
      return false;
    }
  std::vector<std::array<double, 6>> boxes;
  for (size_t i = 0; i < b.nodes.size(); ++i) {
    const Node& n = b.nodes[i];
    bool any = false;
    for (int a = 0; a < 3; ++a)
      if (!std::isfinite(n.origin[a]) || !std::isfinite(n.step[a]) || n.step[a] <= 0) {
        err = "invalid cluster BVH node frame";
        return false;
      }
    std::array<double, 6> all = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
    for (int slot = 0; slot < 4; ++slot) {
      uint32_t c = n.children[slot];
      if (c == EMPTY) continue;
      any = true;
      double clo[3], chi[3];
      if (c & LEAF_BIT) {
        uint32_t li = c & ~LEAF_BIT;
        if (li >= b.leaves.size()) {
          err = "BVH leaf reference";
          return false;
        }
        const Leaf& l = b.leaves[li];
        for (int a = 0; a < 3; ++a) clo[a] = INFINITY, chi[a] = -INFINITY;
        for (uint32_t k = l.offset; k < l.offset + l.count; ++k)
          for (int a = 0; a < 3; ++a) {
            clo[a] = std::min(clo[a], (double)b.positions[b.indices[k]][a]);
            chi[a] = std::max(chi[a], (double)b.positions[b.indices[k]][a]);
          }
      } else {
        if (c >= i) {
          err = "BVH unordered/cyclic node";
          return false;
        }
        for (int a = 0; a < 3; ++a) clo[a] = boxes[c][a], chi[a] = boxes[c][3 + a];
      }
      for (int fused = 0; fused < 2; ++fused)
        for (int a = 0; a < 3; ++a) {
          double lo = decode_plane(n, a, n.lower[a][slot], fused);
          double hi = decode_plane(n, a, n.upper[a][slot], fused);
          if (!std::isfinite(lo) || !std::isfinite(hi) || lo > clo[a] || hi < chi[a]) {
            err = "BVH child bounds/error do not enclose geometry";
            return false;
          }
          all[a] = std::min(all[a], lo);
          all[3 + a] = std::max(all[3 + a], hi);
        }
    }
    if (!any) {
      err = "invalid cluster BVH node frame";
      return false;
    }
    boxes.push_back(all);
  }
  return true;
}

}  // namespace orc
