// CPU ORACLE — test infrastructure only. Restates src/instance_bvh.rs:36-472: the instance top
// level (binned-SAH or median BVH2, collapsed to 32-word BVH4 nodes), its refit and `place`.
#include <algorithm>
#include <limits>

#include "oracle.hpp"

namespace orc {

namespace {

constexpr size_t BINS = 16;  // instance_bvh.rs:287

Box empty_box() {
  const float inf = std::numeric_limits<float>::infinity();
  return Box{{inf, inf, inf}, {-inf, -inf, -inf}};
}
Box unite(const Box& a, const Box& b) {  // instance_bvh.rs:462-472
  Box r;
  for (int i = 0; i < 3; ++i) {
    r.lo[i] = rmin(a.lo[i], b.lo[i]);
    r.hi[i] = rmax(a.hi[i], b.hi[i]);
  }
  return r;
}
float area(const Box& b) {  // instance_bvh.rs:290-293
  float e[3];
  for (int a = 0; a < 3; ++a) e[a] = rmax(b.hi[a] - b.lo[a], 0.0f);
  return e[0] * e[1] + e[1] * e[2] + e[2] * e[0];
}
size_t sat_usize(float f) {
  if (!(f > 0.0f)) return 0;
  if (f >= 1.8e19f) return SIZE_MAX;
  return (size_t)f;
}
V3 centre(const std::vector<Box>& boxes, uint32_t i) {  // instance_bvh.rs:418-421
  const Box& b = boxes[i];
  return V3{b.lo[0] + b.hi[0], b.lo[1] + b.hi[1], b.lo[2] + b.hi[2]};
}

struct Split { int axis; size_t last; float base, scale; };

// instance_bvh.rs:298-342
bool sah_split(const std::vector<Box>& boxes, const uint32_t* order, size_t n, const Box& cb,
               Split& out) {
  bool have = false;
  float best_cost = 0;
  int best_axis = 0;
  size_t best_b = 0;
  for (int axis = 0; axis < 3; ++axis) {
    float extent = cb.hi[axis] - cb.lo[axis];
    if (!(extent > 0.0f)) continue;
    float scale = (float)BINS / extent;
    size_t count[BINS] = {};
    Box bounds[BINS];
    for (auto& x : bounds) x = empty_box();
    for (size_t k = 0; k < n; ++k) {
      uint32_t i = order[k];
      size_t b = std::min(sat_usize((centre(boxes, i)[axis] - cb.lo[axis]) * scale), BINS - 1);
      count[b] += 1;
      bounds[b] = unite(bounds[b], boxes[i]);
    }
    float right_area[BINS] = {};
    size_t right_n[BINS] = {};
    Box acc = empty_box();
    size_t m = 0;
    for (size_t b = BINS - 1; b >= 1; --b) {
      acc = unite(acc, bounds[b]);
      m += count[b];
      right_area[b - 1] = area(acc);
      right_n[b - 1] = m;
    }
    acc = empty_box();
    m = 0;
    for (size_t b = 0; b + 1 < BINS; ++b) {
      acc = unite(acc, bounds[b]);
      m += count[b];
      if (m == 0 || right_n[b] == 0) continue;
      float cost = area(acc) * (float)m + right_area[b] * (float)right_n[b];
      if (!have || cost < best_cost) {
        have = true;
        best_cost = cost;
        best_axis = axis;
        best_b = b;
      }
    }
  }
  if (!have) return false;
  out = Split{best_axis, best_b, cb.lo[best_axis], (float)BINS / (cb.hi[best_axis] - cb.lo[best_axis])};
  return true;
}

struct Sub { uint32_t id; Box box; };

void write_box(uint32_t* w, const Box& b) {
  for (int k = 0; k < 3; ++k) w[k] = fbits(b.lo[k]);
  for (int k = 0; k < 3; ++k) w[3 + k] = fbits(b.hi[k]);
}

// instance_bvh.rs:414-460
Sub subtree(const std::vector<Box>& boxes, uint32_t* order, size_t n, std::vector<uint32_t>& nodes,
            bool sah) {
  if (n == 1) return Sub{TOP_LEAF | order[0], boxes[order[0]]};
  Box cb = empty_box();
  for (size_t k = 0; k < n; ++k) {
    V3 c = centre(boxes, order[k]);
    cb = unite(cb, Box{c, c});
  }
  Split sp;
  size_t mid;
  if (sah && sah_split(boxes, order, n, cb, sp)) {
    size_t left = 0;
    for (size_t k = 0; k < n; ++k) {
      size_t b = std::min(sat_usize((centre(boxes, order[k])[sp.axis] - sp.base) * sp.scale), BINS - 1);
      if (b <= sp.last) {
        std::swap(order[left], order[k]);
        left += 1;
      }
    }
    mid = left;
  } else {
    int axis = 0;  // Iterator::max_by: the last of equal maxima
    for (int k = 1; k < 3; ++k)
      if (total_key(cb.hi[k] - cb.lo[k]) >= total_key(cb.hi[axis] - cb.lo[axis])) axis = k;
    mid = n / 2;
    // select_nth_unstable_by: the sets on either side of `mid` are fixed by the total order
    // (position, index); a full sort gives the same sets.
    std::sort(order, order + n, [&](uint32_t a, uint32_t b) {
      int32_t ka = total_key(centre(boxes, a)[axis]), kb = total_key(centre(boxes, b)[axis]);
      return ka != kb ? ka < kb : a < b;
    });
  }
  size_t node = nodes.size() / TOP_NODE_WORDS;
  nodes.resize(nodes.size() + TOP_NODE_WORDS, 0);
  Sub a = subtree(boxes, order, mid, nodes, sah);
  Sub b = subtree(boxes, order + mid, n - mid, nodes, sah);
  uint32_t* w = &nodes[node * TOP_NODE_WORDS];
  write_box(w, a.box);
  write_box(w + 6, b.box);
  w[12] = a.id;
  w[13] = b.id;
  return Sub{(uint32_t)node, unite(a.box, b.box)};
}

// instance_bvh.rs:270-275
void write_child(uint32_t* node, int c, const Box& b) {
  for (int a = 0; a < 3; ++a) {
    node[a * 4 + c] = fbits(b.lo[a]);
    node[12 + a * 4 + c] = fbits(b.hi[a]);
  }
}

struct Kid { uint32_t id; Box box; };

Kid binary_child(const std::vector<uint32_t>& bin, uint32_t node, int c) {
  const uint32_t* w = &bin[node * TOP_NODE_WORDS];
  Box b;
  for (int k = 0; k < 3; ++k) b.lo[k] = bitsf(w[c * 6 + k]), b.hi[k] = bitsf(w[c * 6 + 3 + k]);
  return Kid{w[12 + c], b};
}

// instance_bvh.rs:370-401
uint32_t collapse(const std::vector<uint32_t>& bin, uint32_t node, std::vector<uint32_t>& out) {
  size_t index = out.size() / TOP_WIDE_WORDS;
  out.resize(out.size() + TOP_WIDE_WORDS, 0);
  std::vector<Kid> kids = {binary_child(bin, node, 0), binary_child(bin, node, 1)};
  while (kids.size() < 4) {
    int pick = -1;
    for (size_t i = 0; i < kids.size(); ++i) {
      if (kids[i].id & TOP_LEAF) continue;
      // max_by(area total_cmp, then b.cmp(&a)): the largest area, ties to the lower index.
      if (pick < 0 || total_key(area(kids[i].box)) > total_key(area(kids[pick].box))) pick = (int)i;
    }
    if (pick < 0) break;
    uint32_t id = kids[pick].id;
    kids.erase(kids.begin() + pick);
    kids.insert(kids.begin() + pick, binary_child(bin, id, 1));
    kids.insert(kids.begin() + pick, binary_child(bin, id, 0));
  }
  for (int c = 0; c < 4; ++c) {
    size_t at = index * TOP_WIDE_WORDS;
    if ((size_t)c >= kids.size()) {
      out[at + 24 + c] = EMPTY;
      continue;
    }
    Kid k = kids[c];
    uint32_t id = (k.id & TOP_LEAF) ? k.id : collapse(bin, k.id, out);
    write_child(&out[at], c, k.box);
    out[at + 24 + c] = id;
  }
  return (uint32_t)index;
}

// instance_bvh.rs:403-411
size_t wide_depth(const std::vector<uint32_t>& nodes, uint32_t node) {
  size_t at = node * TOP_WIDE_WORDS, m = 0;
  for (int c = 0; c < 4; ++c) {
    uint32_t id = nodes[at + 24 + c];
    if (id != EMPTY && !(id & TOP_LEAF)) m = std::max(m, wide_depth(nodes, id));
  }
  return 1 + m;
}

// instance_bvh.rs:255-268
Box refit_wide(uint32_t* nodes, uint32_t node, const std::vector<Box>& boxes) {
  size_t at = node * TOP_WIDE_WORDS;
  Box all = empty_box();
  for (int c = 0; c < 4; ++c) {
    uint32_t id = nodes[at + 24 + c];
    if (id == EMPTY) continue;
    Box b = (id & TOP_LEAF) ? boxes[id & ~TOP_LEAF] : refit_wide(nodes, id, boxes);
    write_child(nodes + at, c, b);
    all = unite(all, b);
  }
  return all;
}

}  // namespace

// instance_bvh.rs:36-38
size_t tlas_reserve(size_t instances) {
  size_t n = instances > 0 ? instances - 1 : 0;
  return std::max<size_t>(n, 1) * TOP_WIDE_WORDS;
}

// instance_bvh.rs:353-366
std::vector<uint32_t> tlas_build_with(const std::vector<Box>& boxes, bool sah, bool wide) {
  std::vector<uint32_t> nodes;
  std::vector<uint32_t> order(boxes.size());
  for (size_t i = 0; i < boxes.size(); ++i) order[i] = (uint32_t)i;
  subtree(boxes, order.data(), order.size(), nodes, sah);
  if (!wide) return nodes;
  std::vector<uint32_t> out;
  collapse(nodes, 0, out);
  if (sah && 1 + 3 * wide_depth(out, 0) > TOP_STACK) return tlas_build_with(boxes, false, wide);
  return out;
}

// instance_bvh.rs:224-253
void tlas_refit(uint32_t* nodes, size_t n_words, const std::vector<Box>& boxes, bool wide) {
  (void)n_words;
  if (wide) {
    refit_wide(nodes, 0, boxes);
    return;
  }
  for (size_t node = boxes.size() >= 1 ? boxes.size() - 1 : 0; node-- > 0;) {
    for (int c = 0; c < 2; ++c) {
      uint32_t id = nodes[node * TOP_NODE_WORDS + 12 + c];
      Box b;
      if (id & TOP_LEAF) {
        b = boxes[id & ~TOP_LEAF];
      } else {
        const uint32_t* w = nodes + (size_t)id * TOP_NODE_WORDS;
        Box x, y;
        for (int k = 0; k < 3; ++k) {
          x.lo[k] = bitsf(w[k]), x.hi[k] = bitsf(w[3 + k]);
          y.lo[k] = bitsf(w[6 + k]), y.hi[k] = bitsf(w[9 + k]);
        }
        b = unite(unite(empty_box(), x), y);
      }
      write_box(nodes + node * TOP_NODE_WORDS + c * 6, b);
    }
  }
}

// instance_bvh.rs:162-220 with the worker build off (RENDERLAB_INSTANCE_BVH_ASYNC=0).
void tlas_place(std::vector<uint32_t>& words, size_t header, size_t stride, size_t slots,
                const std::vector<uint32_t>& previous, int mode, bool wide, bool sah) {
  size_t base = words.size();
  size_t count = words[0];
  bool enabled = (mode < 0 ? count >= MIN_INSTANCES : mode != 0) && count > 0;
  if (enabled) {
    words[1] = (uint32_t)base;
    words[2] = count == 1 ? TOP_LEAF : 0;
  }
  size_t reserve = tlas_reserve(slots);
  bool same_layout = previous.size() == base + reserve && previous[0] == words[0] &&
                     previous[1] == words[1] && previous[2] == words[2];
  if (same_layout && std::equal(previous.begin() + 4, previous.begin() + base, words.begin() + 4)) {
    words[3] = previous[3];
    words.insert(words.end(), previous.begin() + base, previous.end());
    return;
  }
  words.resize(base + reserve, 0);
  if (!enabled || count < 2) return;
  std::vector<Box> boxes(count);
  for (size_t i = 0; i < count; ++i) {
    size_t r = header + i * stride;
    for (int k = 0; k < 3; ++k) boxes[i].lo[k] = bitsf(words[r + 12 + k]), boxes[i].hi[k] = bitsf(words[r + 15 + k]);
  }
  if (same_layout && previous[3] < REFITS) {
    words[3] = std::min(previous[3] + 1, REFITS);
    std::copy(previous.begin() + base, previous.end(), words.begin() + base);
    tlas_refit(&words[base], reserve, boxes, wide);
    return;
  }
  words[3] = 0;
  std::vector<uint32_t> nodes = tlas_build_with(boxes, sah, wide);
  std::copy(nodes.begin(), nodes.end(), words.begin() + base);
}

}  // namespace orc
