// Instance top level (src/instance_bvh.rs:36-460): a binary tree over the instances' world
// boxes, split by 16-bin SAH over the box centres (doubled: lo + hi) or at the centre median,
// then collapsed into 32-word BVH4 nodes (four float boxes axis-major, four tagged children,
// four pad words). The binary tree lives in a node array here rather than in words; the split
// choices, the preorder numbering and the collapse rule are the reference's, so the words match.
#include <algorithm>
#include <numeric>

#include "host.hpp"

namespace rtb {

namespace {

constexpr int BINS = 16;
constexpr size_t WIDE = 32;

inline size_t to_usize(float f) {
  if (!(f > 0.0f)) return 0;
  if (f >= 1.8e19f) return SIZE_MAX;
  return (size_t)f;
}
inline float area(const Aabb& b) {  // instance_bvh.rs:290-293
  float e0 = hi_of(b.hi[0] - b.lo[0], 0.0f), e1 = hi_of(b.hi[1] - b.lo[1], 0.0f),
        e2 = hi_of(b.hi[2] - b.lo[2], 0.0f);
  return e0 * e1 + e1 * e2 + e2 * e0;
}

struct BinNode {
  uint32_t child[2];  // binary node index or LEAF | instance
  Aabb box[2];
};

class TopBuilder {
 public:
  TopBuilder(const std::vector<Aabb>& boxes, bool sah) : boxes_(boxes), sah_(sah) {
    centre_.resize(3 * boxes.size());
    for (size_t i = 0; i < boxes.size(); ++i)
      for (int a = 0; a < 3; ++a) centre_[3 * i + a] = boxes[i].lo[a] + boxes[i].hi[a];
    ids_.resize(boxes.size());
    std::iota(ids_.begin(), ids_.end(), 0u);
  }
  void build() { binary(0, ids_.size()); }
  const std::vector<BinNode>& nodes() const { return bin_; }

 private:
  const std::vector<Aabb>& boxes_;
  bool sah_;
  std::vector<float> centre_;
  std::vector<uint32_t> ids_;
  std::vector<BinNode> bin_;

  float cen(uint32_t i, int a) const { return centre_[3 * (size_t)i + a]; }

  // instance_bvh.rs:414-460; returns (tagged id, box)
  std::pair<uint32_t, Aabb> binary(size_t lo, size_t hi) {
    if (hi - lo == 1) return {LEAF | ids_[lo], boxes_[ids_[lo]]};
    Aabb cb = Aabb::empty();
    for (size_t k = lo; k < hi; ++k) cb.grow(&centre_[3 * (size_t)ids_[k]]);
    size_t mid = 0;
    if (!(sah_ && sah_cut(lo, hi, cb, mid))) {
      int axis = 0;
      for (int a = 1; a < 3; ++a)
        if (order_key(cb.hi[a] - cb.lo[a]) >= order_key(cb.hi[axis] - cb.lo[axis])) axis = a;
      mid = lo + (hi - lo) / 2;
      std::nth_element(ids_.begin() + lo, ids_.begin() + mid, ids_.begin() + hi, [&](uint32_t x, uint32_t y) {
        int32_t kx = order_key(cen(x, axis)), ky = order_key(cen(y, axis));
        return kx != ky ? kx < ky : x < y;
      });
    }
    uint32_t me = (uint32_t)bin_.size();
    bin_.emplace_back();
    auto a = binary(lo, mid);
    auto b = binary(mid, hi);
    BinNode& n = bin_[me];
    n.child[0] = a.first, n.child[1] = b.first;
    n.box[0] = a.second, n.box[1] = b.second;
    Aabb u = a.second;
    u.grow(b.second);
    Aabb all = Aabb::empty();
    all.grow(a.second);
    all.grow(b.second);
    (void)u;
    return {me, all};
  }

  // instance_bvh.rs:298-342 and the partition at :427-437
  bool sah_cut(size_t lo, size_t hi, const Aabb& cb, size_t& mid) {
    bool found = false;
    float best = 0.0f;
    int best_axis = 0, best_bin = 0;
    for (int axis = 0; axis < 3; ++axis) {
      const float extent = cb.hi[axis] - cb.lo[axis];
      if (!(extent > 0.0f)) continue;
      const float scale = (float)BINS / extent;
      size_t count[BINS] = {};
      Aabb bins[BINS];
      for (auto& b : bins) b = Aabb::empty();
      for (size_t k = lo; k < hi; ++k) {
        uint32_t i = ids_[k];
        size_t bin = std::min(to_usize((cen(i, axis) - cb.lo[axis]) * scale), (size_t)BINS - 1);
        count[bin] += 1;
        bins[bin].grow(boxes_[i]);
      }
      float r_area[BINS];
      size_t r_n[BINS];
      Aabb acc = Aabb::empty();
      size_t n = 0;
      for (int b = BINS - 1; b >= 1; --b) {
        acc.grow(bins[b]);
        n += count[b];
        r_area[b - 1] = area(acc);
        r_n[b - 1] = n;
      }
      acc = Aabb::empty();
      n = 0;
      for (int b = 0; b < BINS - 1; ++b) {
        acc.grow(bins[b]);
        n += count[b];
        if (n == 0 || r_n[b] == 0) continue;
        float cost = area(acc) * (float)n + r_area[b] * (float)r_n[b];
        if (!found || cost < best) found = true, best = cost, best_axis = axis, best_bin = b;
      }
    }
    if (!found) return false;
    const float base = cb.lo[best_axis], scale = (float)BINS / (cb.hi[best_axis] - cb.lo[best_axis]);
    auto it = std::partition(ids_.begin() + lo, ids_.begin() + hi, [&](uint32_t i) {
      return (int)std::min(to_usize((cen(i, best_axis) - base) * scale), (size_t)BINS - 1) <= best_bin;
    });
    mid = (size_t)(it - ids_.begin());
    return true;
  }
};

void put_box(uint32_t* node, int c, const Aabb& b) {  // instance_bvh.rs:270-275
  for (int a = 0; a < 3; ++a) node[4 * a + c] = as_bits(b.lo[a]), node[12 + 4 * a + c] = as_bits(b.hi[a]);
}

struct Kid { uint32_t id; Aabb box; };

// instance_bvh.rs:370-401: a binary node's two children, then repeatedly the largest-area inner
// child (ties: the earlier slot) replaced by its own two, up to four; children follow parents.
uint32_t collapse(const std::vector<BinNode>& bin, uint32_t node, std::vector<uint32_t>& out) {
  uint32_t me = (uint32_t)(out.size() / WIDE);
  out.resize(out.size() + WIDE, 0);
  Kid kids[4];
  int n = 2;
  kids[0] = {bin[node].child[0], bin[node].box[0]};
  kids[1] = {bin[node].child[1], bin[node].box[1]};
  while (n < 4) {
    int pick = -1;
    for (int k = 0; k < n; ++k)
      if (!(kids[k].id & LEAF) && (pick < 0 || order_key(area(kids[k].box)) > order_key(area(kids[pick].box)))) pick = k;
    if (pick < 0) break;
    uint32_t id = kids[pick].id;
    for (int k = n; k > pick + 1; --k) kids[k] = kids[k - 1];
    kids[pick] = {bin[id].child[0], bin[id].box[0]};
    kids[pick + 1] = {bin[id].child[1], bin[id].box[1]};
    ++n;
  }
  for (int c = 0; c < 4; ++c) {
    size_t at = (size_t)me * WIDE;
    if (c >= n) {
      out[at + 24 + c] = EMPTY;
      continue;
    }
    uint32_t id = (kids[c].id & LEAF) ? kids[c].id : collapse(bin, kids[c].id, out);
    put_box(&out[at], c, kids[c].box);
    out[at + 24 + c] = id;
  }
  return me;
}

size_t wide_depth(const std::vector<uint32_t>& w, uint32_t node) {
  size_t d = 0;
  for (int c = 0; c < 4; ++c) {
    uint32_t id = w[(size_t)node * WIDE + 24 + c];
    if (id != EMPTY && !(id & LEAF)) d = std::max(d, wide_depth(w, id));
  }
  return 1 + d;
}

Aabb refit_node(uint32_t* nodes, uint32_t node, const std::vector<Aabb>& boxes) {
  Aabb all = Aabb::empty();
  uint32_t* w = nodes + (size_t)node * WIDE;
  for (int c = 0; c < 4; ++c) {
    uint32_t id = w[24 + c];
    if (id == EMPTY) continue;
    Aabb b = (id & LEAF) ? boxes[id & ~LEAF] : refit_node(nodes, id, boxes);
    put_box(w, c, b);
    all.grow(b);
  }
  return all;
}

}  // namespace

size_t tlas_reserve(size_t instances) {  // instance_bvh.rs:36-38
  return std::max<size_t>(instances > 0 ? instances - 1 : 0, 1) * WIDE;
}

// instance_bvh.rs:346-366: SAH, collapsed; a tree too deep for the 48-entry stack falls back to
// median splits.
std::vector<uint32_t> tlas_build(const std::vector<Aabb>& boxes, bool sah) {
  TopBuilder b(boxes, sah);
  b.build();
  std::vector<uint32_t> out;
  out.reserve(boxes.size() * WIDE);
  collapse(b.nodes(), 0, out);
  if (sah && 1 + 3 * wide_depth(out, 0) > STACK_DEPTH) return tlas_build(boxes, false);
  return out;
}

void tlas_refit(uint32_t* nodes, const std::vector<Aabb>& boxes) { refit_node(nodes, 0, boxes); }

// instance_bvh.rs:162-220 for a fresh buffer (no previous words): header words 1-3, the reserve,
// and a build when the top level is enabled.
void tlas_place(std::vector<uint32_t>& words, size_t header, size_t stride, size_t slots, int mode) {
  const size_t base = words.size();
  const size_t count = words[0];
  const bool enabled = (mode < 0 ? count >= 40 : mode != 0) && count > 0;  // MIN_INSTANCES = 40
  if (enabled) {
    words[1] = (uint32_t)base;
    words[2] = count == 1 ? LEAF : 0;
  }
  words.resize(base + tlas_reserve(slots), 0);
  if (!enabled || count < 2) return;
  std::vector<Aabb> boxes(count);
  for (size_t i = 0; i < count; ++i) {
    const uint32_t* r = &words[header + i * stride];
    for (int a = 0; a < 3; ++a) boxes[i].lo[a] = as_float(r[12 + a]), boxes[i].hi[a] = as_float(r[15 + a]);
  }
  words[3] = 0;
  std::vector<uint32_t> nodes = tlas_build(boxes, true);
  std::copy(nodes.begin(), nodes.end(), words.begin() + base);
}

}  // namespace rtb
