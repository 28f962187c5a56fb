// A host-side check of the engine's derived 8-wide layout (wide8.hpp): the properties the WIDE8
// kernels rely on, verified node by node in exact arithmetic, so that the builder's output can be
// tested without a GPU. The box rule is the one traversal needs: a ray that meets a triangle meets
// every child box on the path to its leaf.
#include <algorithm>
#include <cmath>
#include <set>

#include "host.hpp"
#include "wide8.hpp"

namespace rtb {

namespace {

struct Extent {
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  void grow(const double* l, const double* h) {
    for (int a = 0; a < 3; ++a) lo[a] = std::min(lo[a], l[a]), hi[a] = std::max(hi[a], h[a]);
  }
  bool within(const double* l, const double* h) const {
    for (int a = 0; a < 3; ++a)
      if (lo[a] < l[a] || hi[a] > h[a]) return false;
    return true;
  }
};

uint32_t byte_of(const uint32_t* w, int plane, int s) { return (w[8 + 2 * plane + (s >> 2)] >> (8 * (s & 3))) & 255u; }

// Checks the subtree at `node`; returns the box of its triangles' vertices through `ext`. A child
// box must enclose its child's triangles (what a ray must not miss), not the child's own, larger,
// outward-rounded child boxes.
bool check_node(const Wide8Scene& s, uint32_t node, uint32_t level, std::vector<uint8_t>& seen_node,
                std::vector<uint8_t>& seen_tri, uint32_t& depth, Extent& ext, std::string& err) {
  const size_t nn = s.nodes.size() / W8_NODE_WORDS, nt = s.tris.size() / W8_TRI_WORDS;
  if (node >= nn) return err = "node index out of range", false;
  if (seen_node[node]) return err = "a node is reached twice", false;
  seen_node[node] = 1;
  depth = std::max(depth, level);
  const uint32_t* w = &s.nodes[(size_t)node * W8_NODE_WORDS];
  double p[3], scale[3];
  for (int a = 0; a < 3; ++a) {
    const int e = (int)((w[3] >> (8 * a)) & 255u) - 127;
    if (e > W8_MAX_EXPONENT || e < -126) return err = "node scale exponent out of range", false;
    p[a] = as_float(w[a]);
    scale[a] = std::ldexp(1.0, e);
    if (!std::isfinite(p[a])) return err = "non-finite node origin", false;
  }
  const uint32_t imask = w[3] >> 24, child_base = w[4], tri_base = w[5];
  uint32_t next_offset = 0;
  for (int slot = 0; slot < 8; ++slot) {
    const uint32_t meta = ((slot < 4 ? w[6] : w[7]) >> (8 * (slot & 3))) & 255u;
    const bool inner = (imask >> slot) & 1u;
    double lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {  // exact: a float plus an integer times a power of two
      lo[a] = p[a] + byte_of(w, a, slot) * scale[a];
      hi[a] = p[a] + byte_of(w, 3 + a, slot) * scale[a];
    }
    if (!inner && meta == 0) {  // empty: an inverted box no ray meets
      for (int a = 0; a < 3; ++a)
        if (byte_of(w, a, slot) != 255 || byte_of(w, 3 + a, slot) != 0) return err = "empty slot is not inverted", false;
      continue;
    }
    if (inner && meta != 0) return err = "a slot is both inner and a leaf", false;
    for (int a = 0; a < 3; ++a)
      if (lo[a] > hi[a]) return err = "child box lower plane above its upper plane", false;
    Extent child;
    if (inner) {
      const uint32_t c = child_base + (uint32_t)__builtin_popcount(imask & ((1u << slot) - 1u));
      if (c <= node) return err = "inner child not after its parent", false;
      if (!check_node(s, c, level + 1, seen_node, seen_tri, depth, child, err)) return false;
    } else {
      const uint32_t count = meta >> 5, offset = meta & 31u;
      if (count > W8_MAX_LEAF) return err = "leaf holds more triangles than the builder allows", false;
      if (offset != next_offset) return err = "leaf triangles not contiguous in slot order", false;
      next_offset = offset + count;
      for (uint32_t k = 0; k < count; ++k) {
        const size_t t = (size_t)tri_base + offset + k;
        if (t >= nt) return err = "triangle index out of range", false;
        if (seen_tri[t]++) return err = "a triangle is referenced by two leaves", false;
        const uint32_t* tw = &s.tris[t * W8_TRI_WORDS];
        for (int v = 0; v < 3; ++v) {
          double x[3];
          for (int a = 0; a < 3; ++a) x[a] = as_float(tw[3 * v + a]);
          child.grow(x, x);
        }
      }
    }
    if (!child.within(lo, hi)) return err = "a child box does not enclose its child's triangles", false;
    ext.grow(child.lo, child.hi);
  }
  return true;
}

// The box a top-level leaf must enclose for entry (instance i, BLAS node `rel` below its root):
// the node's box under the instance's object-to-world map, or the record world box when the
// record's rows cannot be inverted.
bool entry_box(const Wide8Scene& s, const uint32_t* r, uint32_t i, uint32_t rel, double* lo, double* hi,
               std::string& err) {
  const size_t nn = s.nodes.size() / W8_NODE_WORDS;
  if (s.inst[2 * i] >= nn || rel >= nn - s.inst[2 * i]) return err = "a top-level entry names no node of its BLAS", false;
  double m[12];
  if (!instance_model(r, m)) {
    for (int a = 0; a < 3; ++a) lo[a] = as_float(r[12 + a]), hi[a] = as_float(r[15 + a]);
    return true;
  }
  double olo[3], ohi[3];
  if (!entry_object_box(&s.nodes[(size_t)(s.inst[2 * i] + rel) * W8_NODE_WORDS], olo, ohi))
    return err = "a top-level entry's node has no children", false;
  entry_world_box(m, olo, ohi, lo, hi);
  return true;
}

// The same for a node of the 8-wide top level: its leaves hold entries (instance, BLAS node), and
// a child box must enclose the world boxes of the entries below it. Collects each instance's
// entries.
bool check_top_node(const Wide8Scene& s, const uint32_t* words, size_t header, size_t stride, uint32_t count,
                    uint32_t node, uint32_t level, std::vector<uint8_t>& seen_node,
                    std::vector<std::vector<uint32_t>>& entries, uint32_t& depth, Extent& ext, std::string& err) {
  const size_t nn = s.top_nodes.size() / W8_NODE_WORDS;
  if (node >= nn) return err = "top-level node index out of range", false;
  if (seen_node[node]) return err = "a top-level node is reached twice", false;
  seen_node[node] = 1;
  depth = std::max(depth, level);
  const uint32_t* w = &s.top_nodes[(size_t)node * W8_NODE_WORDS];
  double p[3], scale[3];
  for (int a = 0; a < 3; ++a) {
    const int e = (int)((w[3] >> (8 * a)) & 255u) - 127;
    if (e > W8_MAX_EXPONENT || e < -126) return err = "top-level node scale exponent out of range", false;
    p[a] = as_float(w[a]);
    scale[a] = std::ldexp(1.0, e);
  }
  const uint32_t imask = w[3] >> 24, child_base = w[4], item_base = w[5];
  for (int slot = 0; slot < 8; ++slot) {
    const uint32_t meta = ((slot < 4 ? w[6] : w[7]) >> (8 * (slot & 3))) & 255u;
    const bool inner = (imask >> slot) & 1u;
    double lo[3], hi[3];
    for (int a = 0; a < 3; ++a) lo[a] = p[a] + byte_of(w, a, slot) * scale[a], hi[a] = p[a] + byte_of(w, 3 + a, slot) * scale[a];
    if (!inner && meta == 0) continue;
    Extent child;
    if (inner) {
      const uint32_t c = child_base + (uint32_t)__builtin_popcount(imask & ((1u << slot) - 1u));
      if (c <= node) return err = "top-level child not after its parent", false;
      if (!check_top_node(s, words, header, stride, count, c, level + 1, seen_node, entries, depth, child, err)) return false;
    } else {
      for (uint32_t k = 0; k < (meta >> 5); ++k) {
        const size_t at = (size_t)item_base + (meta & 31u) + k;
        if (2 * at + 1 >= s.top_items.size()) return err = "top-level item out of range", false;
        const uint32_t i = s.top_items[2 * at], rel = s.top_items[2 * at + 1];
        if (i >= count) return err = "top-level leaf names no instance", false;
        double l[3], h[3];
        if (!entry_box(s, words + header + stride * (size_t)i, i, rel, l, h, err)) return false;
        entries[i].push_back(rel);
        child.grow(l, h);
      }
    }
    if (!child.within(lo, hi)) return err = "a top-level child box does not enclose its entries' world boxes", false;
    ext.grow(child.lo, child.hi);
  }
  return true;
}

// Whether the entries `cut` (sorted node indices below the BLAS root `base`) cut the BLAS at
// `node` exactly: `node` is an entry, or has no leaf slots and each of its inner children is cut.
bool cuts(const Wide8Scene& s, uint32_t base, uint32_t node, const std::vector<uint32_t>& cut, size_t& used) {
  if (std::binary_search(cut.begin(), cut.end(), node - base)) return ++used, true;
  const uint32_t* w = &s.nodes[(size_t)node * W8_NODE_WORDS];
  if (w[6] != 0 || w[7] != 0) return false;  // leaf triangles above every entry: no entry holds them
  const uint32_t imask = w[3] >> 24;
  for (int k = 0; k < __builtin_popcount(imask); ++k)
    if (!cuts(s, base, w[4] + (uint32_t)k, cut, used)) return false;
  return true;
}

}  // namespace

bool check_wide8_top(uint32_t layout, const uint32_t* words, const Wide8Scene& s, std::string& err) {
  if (s.top_nodes.empty()) return true;  // no 8-wide top level: the walk uses the packed one
  const uint32_t count = words[0];
  const size_t header = layout == 0 ? 16 : 8, stride = layout == 0 ? 32 : 24;
  if (s.inst.size() < 2 * (size_t)count) return err = "instance table shorter than the records", false;
  std::vector<uint8_t> seen_node(s.top_nodes.size() / W8_NODE_WORDS, 0);
  std::vector<std::vector<uint32_t>> entries(count);
  uint32_t depth = 0;
  Extent ext;
  if (!check_top_node(s, words, header, stride, count, 0, 1, seen_node, entries, depth, ext, err)) return false;
  if (std::find(seen_node.begin(), seen_node.end(), 0) != seen_node.end()) return err = "an unreachable top-level node", false;
  for (uint32_t i = 0; i < count; ++i) {
    const uint32_t* r = words + header + stride * (size_t)i;
    bool valid = s.inst[2 * i] != EMPTY;
    for (int a = 0; a < 3; ++a) {
      const float l = as_float(r[12 + a]), h = as_float(r[15 + a]);
      valid = valid && std::isfinite(l) && std::isfinite(h) && l <= h;
    }
    std::vector<uint32_t>& cut = entries[i];
    if (!valid) {
      if (!cut.empty()) return err = "a top-level entry for an instance the walk must not enter", false;
      continue;
    }
    if (cut.empty()) return err = "an instance no top-level leaf holds", false;
    std::sort(cut.begin(), cut.end());
    if (std::adjacent_find(cut.begin(), cut.end()) != cut.end()) return err = "an entry is in two top-level leaves", false;
    size_t used = 0;
    if (!cuts(s, s.inst[2 * i], s.inst[2 * i], cut, used) || used != cut.size())
      return err = "an instance's entries do not cut its BLAS exactly", false;
  }
  if (depth != s.top_depth || depth + 9 > W8_TOP_STACK) return err = "top-level depth differs from the record or the walk's stack", false;
  return true;
}

bool check_wide8_scene(const Wide8Scene& s, uint32_t info[4], std::string& err) {
  const size_t nn = s.nodes.size() / W8_NODE_WORDS, nt = s.tris.size() / W8_TRI_WORDS;
  std::vector<uint8_t> seen_node(nn, 0), seen_tri(nt, 0);
  std::set<uint32_t> roots;
  for (size_t i = 0; i + 1 < s.inst.size(); i += 2)
    if (s.inst[i] != EMPTY) roots.insert(s.inst[i]);
  uint32_t depth = 0;
  for (uint32_t r : roots) {
    Extent ext;
    uint32_t d = 0;
    if (!check_node(s, r, 1, seen_node, seen_tri, d, ext, err)) return false;
    depth = std::max(depth, d);
  }
  if (std::find(seen_node.begin(), seen_node.end(), 0) != seen_node.end()) return err = "an unreachable node", false;
  if (std::find(seen_tri.begin(), seen_tri.end(), 0) != seen_tri.end()) return err = "a triangle no leaf holds", false;
  if (depth != s.depth) return err = "recorded depth differs from the tree's", false;
  info[0] = (uint32_t)nn, info[1] = (uint32_t)nt, info[2] = depth, info[3] = (uint32_t)s.blas_count;
  return true;
}

}  // namespace rtb
