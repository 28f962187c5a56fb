// Builder of the compressed 8-wide BLAS (layout in wide8.hpp): a binned-SAH binary tree with
// leaves of at most W8_MAX_LEAF triangles, collapsed into 8-wide nodes by the SAH-optimal forest
// of each node, child slots assigned by octant, child boxes quantised outward to 8 bits against
// a power-of-two scale.
#include "wide8.hpp"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <deque>
#include <map>
#include <mutex>
#include <numeric>
#include <thread>
#include <array>

#include "host.hpp"

namespace rtb {

namespace {

constexpr int BINS = 32;
constexpr float COST_NODE = 1.0f, COST_TRI = 1.0f;

double area(const Aabb& b) {
  double e0 = std::max(0.0, (double)b.hi[0] - b.lo[0]), e1 = std::max(0.0, (double)b.hi[1] - b.lo[1]),
         e2 = std::max(0.0, (double)b.hi[2] - b.lo[2]);
  return e0 * e1 + e1 * e2 + e2 * e0;
}

struct BNode {
  Aabb box;
  int kid[2];
  uint32_t first, count;  // count > 0: leaf over refs[first, first + count)
};

// Binned-SAH binary tree over primitive boxes: triangles for a BLAS, instance world boxes for a
// top level.
class Binary {
 public:
  explicit Binary(const std::vector<SrcTri>& t) {
    std::vector<Aabb> boxes(t.size());
    for (size_t i = 0; i < t.size(); ++i) {
      Aabb b = Aabb::empty();
      for (int k = 0; k < 3; ++k) b.grow(&t[i].v[3 * k]);
      boxes[i] = b;
    }
    init(std::move(boxes));
  }
  explicit Binary(std::vector<Aabb> boxes) { init(std::move(boxes)); }
  int build() { return node(0, (uint32_t)ref_.size()); }
  const std::vector<BNode>& nodes() const { return nodes_; }
  const std::vector<uint32_t>& refs() const { return ref_; }

 private:
  void init(std::vector<Aabb> boxes) {
    box_ = std::move(boxes);
    const size_t n = box_.size();
    cen_.resize(3 * n);
    for (size_t i = 0; i < n; ++i)
      for (int a = 0; a < 3; ++a) cen_[3 * i + a] = 0.5f * (box_[i].lo[a] + box_[i].hi[a]);
    ref_.resize(n);
    std::iota(ref_.begin(), ref_.end(), 0u);
  }
  std::vector<Aabb> box_;
  std::vector<float> cen_;
  std::vector<uint32_t> ref_;
  std::vector<BNode> nodes_;

  int leaf(uint32_t first, uint32_t n, const Aabb& b) {
    nodes_.push_back(BNode{b, {-1, -1}, first, n});
    return (int)nodes_.size() - 1;
  }

  int node(uint32_t first, uint32_t n) {
    Aabb b = Aabb::empty(), cb = Aabb::empty();
    for (uint32_t k = first; k < first + n; ++k) {
      b.grow(box_[ref_[k]]);
      cb.grow(&cen_[3 * (size_t)ref_[k]]);
    }
    if (n == 1) return leaf(first, n, b);
    // binned SAH over the centroid bounds, all three axes
    double best = INFINITY;
    int best_axis = -1, best_bin = 0;
    const double parent = std::max(area(b), 1e-30);
    for (int a = 0; a < 3; ++a) {
      const float ext = cb.hi[a] - cb.lo[a];
      if (!(ext > 0.0f)) continue;
      const float scale = (float)BINS / ext;
      uint32_t cnt[BINS] = {};
      Aabb bb[BINS];
      for (auto& x : bb) x = Aabb::empty();
      for (uint32_t k = first; k < first + n; ++k) {
        uint32_t r = ref_[k];
        int bin = std::min(BINS - 1, (int)((cen_[3 * (size_t)r + a] - cb.lo[a]) * scale));
        cnt[bin]++;
        bb[bin].grow(box_[r]);
      }
      double ra[BINS];
      uint32_t rn[BINS];
      Aabb acc = Aabb::empty();
      uint32_t m = 0;
      for (int k = BINS - 1; k > 0; --k) {
        acc.grow(bb[k]);
        m += cnt[k];
        ra[k] = area(acc);
        rn[k] = m;
      }
      acc = Aabb::empty();
      m = 0;
      for (int k = 0; k < BINS - 1; ++k) {
        acc.grow(bb[k]);
        m += cnt[k];
        if (m == 0 || rn[k + 1] == 0) continue;
        double c = COST_NODE + COST_TRI * (area(acc) * m + ra[k + 1] * rn[k + 1]) / parent;
        if (c < best) best = c, best_axis = a, best_bin = k;
      }
    }
    if (n <= W8_MAX_LEAF && (best_axis < 0 || COST_TRI * n <= best)) return leaf(first, n, b);
    uint32_t mid;
    if (best_axis >= 0) {
      const float ext = cb.hi[best_axis] - cb.lo[best_axis], scale = (float)BINS / ext, lo = cb.lo[best_axis];
      auto it = std::partition(ref_.begin() + first, ref_.begin() + first + n, [&](uint32_t r) {
        return std::min(BINS - 1, (int)((cen_[3 * (size_t)r + best_axis] - lo) * scale)) <= best_bin;
      });
      mid = (uint32_t)(it - ref_.begin());
    } else {
      mid = first + n / 2;  // coincident centroids: split the list
    }
    const int me = (int)nodes_.size();
    nodes_.push_back(BNode{b, {-1, -1}, 0, 0});
    const int l = node(first, mid - first);
    const int r = node(mid, first + n - mid);
    nodes_[me].kid[0] = l;
    nodes_[me].kid[1] = r;
    return me;
  }
};

// Smallest power-of-two exponent e with 255 * 2^e >= ext (a normal float scale).
int scale_exponent(double ext) {
  if (!(ext > 0.0)) return -126;
  int e;
  std::frexp(ext / 255.0, &e);  // ext/255 = f * 2^e, f in [0.5, 1)
  while (std::ldexp(255.0, e - 1) >= ext && e - 1 >= -126) --e;
  while (std::ldexp(255.0, e) < ext) ++e;
  return std::max(-126, std::min(127, e));
}

// SAH-optimal collapse of the binary tree into 8-wide nodes (Ylitie, Karras and Laine 2017,
// section 3.1). cost[n][j] is the least SAH cost of the subtree at n as a forest of at most j
// roots; each root becomes a leaf slot (at most W8_MAX_LEAF triangles) or an 8-wide node of its
// own. Measured in a visit-count model of the kernel on 1M-triangle cluster soup, against
// opening the largest child greedily: 3 % fewer node visits a ray, 20 % fewer nodes.
class Collapse {
 public:
  explicit Collapse(std::vector<BNode>& bn) : bn_(bn), cost_(bn.size()), split_(bn.size()), count_(bn.size()) {
    // the binary builder appends a node before its children: children have larger indices
    for (size_t i = bn.size(); i-- > 0;) visit((int)i);
  }
  // The roots of the 8-wide node made from binary node n (an inner node).
  std::vector<int> children(int n) const {
    std::vector<int> out;
    const int k = split_[n][0];
    expand(bn_[n].kid[0], k, out);
    expand(bn_[n].kid[1], 8 - k, out);
    return out;
  }

 private:
  std::vector<BNode>& bn_;
  std::vector<std::array<double, 9>> cost_;
  std::vector<std::array<int8_t, 9>> split_;  // [j]: 0 keeps j - 1 roots, k splits k | j - k; [0] the node's own
  std::vector<uint32_t> count_;

  void visit(int n) {
    BNode& b = bn_[n];
    const double a = area(b.box);
    if (b.count > 0) {
      count_[n] = b.count;
      for (int j = 1; j <= 8; ++j) cost_[n][j] = COST_TRI * a * b.count, split_[n][j] = 0;
      return;
    }
    const int l = b.kid[0], r = b.kid[1];
    count_[n] = count_[l] + count_[r];
    double inner = INFINITY;
    for (int k = 1; k < 8; ++k) {
      const double c = cost_[l][k] + cost_[r][8 - k];
      if (c < inner) inner = c, split_[n][0] = (int8_t)k;
    }
    inner += COST_NODE * a;
    const double as_leaf = count_[n] <= W8_MAX_LEAF ? COST_TRI * a * count_[n] : INFINITY;
    cost_[n][1] = std::min(inner, as_leaf);
    split_[n][1] = 0;
    if (as_leaf <= inner) {  // the whole subtree as one leaf slot, kept whole in every forest
      b.first = first_of(l), b.count = count_[n];
      for (int j = 2; j <= 8; ++j) cost_[n][j] = cost_[n][1], split_[n][j] = 0;
      return;
    }
    for (int j = 2; j <= 8; ++j) {
      double best = cost_[n][j - 1];
      split_[n][j] = 0;
      for (int k = 1; k < j; ++k) {
        const double c = cost_[l][k] + cost_[r][j - k];
        if (c < best) best = c, split_[n][j] = (int8_t)k;
      }
      cost_[n][j] = best;
    }
  }
  // A subtree's first triangle reference (its references are contiguous: the builder partitions
  // them in place, left before right).
  uint32_t first_of(int n) const {
    while (bn_[n].count == 0) n = bn_[n].kid[0];
    return bn_[n].first;
  }
  void expand(int n, int j, std::vector<int>& out) const {
    while (j > 1 && split_[n][j] == 0) --j;
    if (j == 1 || bn_[n].count > 0) {
      out.push_back(n);
      return;
    }
    const int k = split_[n][j];
    expand(bn_[n].kid[0], k, out);
    expand(bn_[n].kid[1], j - k, out);
  }
};

// The 8-wide nodes of a binary tree (root `broot`), breadth first from node 0 (the upper levels
// get the lowest indices; a node's inner children are one contiguous block): the SAH-optimal
// collapse, octant slots, child boxes quantised outward. A leaf slot's primitives are appended by
// `leaf(ref)` (its first one at index `leaf.base()` when the node is written), so the same
// emission serves triangle BLASes and instance top levels. (Writing each child's subtree before
// the next child's instead was measured: the same speed on clusters-1M and -4M.)
template <class Leaf>
void emit_wide8(std::vector<BNode>& bn, int broot, const std::vector<uint32_t>& refs, std::vector<uint32_t>& nodes,
                int& max_exponent, uint32_t& depth, Leaf& leaf) {
  const Collapse plan(bn);
  struct Task { uint32_t wide; int b; uint32_t level; };
  std::deque<Task> queue;
  nodes.resize(W8_NODE_WORDS, 0);
  queue.push_back({0, broot, 1});
  while (!queue.empty()) {
    const Task task = queue.front();
    queue.pop_front();
    depth = std::max(depth, task.level);
    std::vector<int> kids;
    if (bn[task.b].count > 0) kids.push_back(task.b);  // a tree of one leaf
    else kids = plan.children(task.b);
    // octant slots: greedy on the children's centre offsets from the node centre
    Aabb nb = Aabb::empty();
    for (int k : kids) nb.grow(bn[k].box);
    double c0[3];
    for (int a = 0; a < 3; ++a) c0[a] = 0.5 * ((double)nb.lo[a] + nb.hi[a]);
    int slot_of[8];
    std::fill(slot_of, slot_of + 8, -1);
    {
      double score[8][8];
      for (size_t k = 0; k < kids.size(); ++k)
        for (int s = 0; s < 8; ++s) {
          double v = 0;
          for (int a = 0; a < 3; ++a) {
            double c = 0.5 * ((double)bn[kids[k]].box.lo[a] + bn[kids[k]].box.hi[a]) - c0[a];
            v += (s >> a & 1) ? c : -c;
          }
          score[k][s] = v;
        }
      bool kid_done[8] = {}, slot_done[8] = {};
      for (size_t round = 0; round < kids.size(); ++round) {
        double bs = -INFINITY;
        int bk = -1, bsl = -1;
        for (size_t k = 0; k < kids.size(); ++k)
          if (!kid_done[k])
            for (int s = 0; s < 8; ++s)
              if (!slot_done[s] && score[k][s] > bs) bs = score[k][s], bk = (int)k, bsl = s;
        kid_done[bk] = slot_done[bsl] = true;
        slot_of[bsl] = bk;
      }
    }
    // scale
    float p[3];
    int ex[3];
    for (int a = 0; a < 3; ++a) {
      p[a] = nb.lo[a];
      ex[a] = scale_exponent((double)nb.hi[a] - (double)p[a]);
      max_exponent = std::max(max_exponent, ex[a]);
    }
    uint32_t imask = 0, child_base = (uint32_t)(nodes.size() / W8_NODE_WORDS), leaf_base = leaf.base();
    uint8_t meta[8] = {}, q[6][8] = {};
    uint32_t inner = 0, offset = 0;
    for (int s = 0; s < 8; ++s) {
      if (slot_of[s] < 0) {  // empty: an inverted box (lower 255, upper 0) that no ray meets
        for (int a = 0; a < 3; ++a) q[a][s] = 255, q[3 + a][s] = 0;
        continue;
      }
      const BNode& k = bn[kids[slot_of[s]]];
      for (int a = 0; a < 3; ++a) {
        const double sc = std::ldexp(1.0, ex[a]);
        double lo = std::floor(((double)k.box.lo[a] - p[a]) / sc), hi = std::ceil(((double)k.box.hi[a] - p[a]) / sc);
        q[a][s] = (uint8_t)std::max(0.0, std::min(255.0, lo));
        q[3 + a][s] = (uint8_t)std::max(0.0, std::min(255.0, hi));
      }
      if (k.count == 0) {
        imask |= 1u << s;
        ++inner;
      } else {
        meta[s] = (uint8_t)(k.count << 5 | offset);
        for (uint32_t t = 0; t < k.count; ++t) leaf(refs[k.first + t]);
        offset += k.count;
      }
    }
    nodes.resize(nodes.size() + (size_t)inner * W8_NODE_WORDS, 0);
    uint32_t* w = &nodes[(size_t)task.wide * W8_NODE_WORDS];
    for (int a = 0; a < 3; ++a) w[a] = as_bits(p[a]);
    w[3] = (uint32_t)(ex[0] + 127) | (uint32_t)(ex[1] + 127) << 8 | (uint32_t)(ex[2] + 127) << 16 | imask << 24;
    w[4] = child_base;
    w[5] = leaf_base;
    w[6] = meta[0] | meta[1] << 8 | meta[2] << 16 | (uint32_t)meta[3] << 24;
    w[7] = meta[4] | meta[5] << 8 | meta[6] << 16 | (uint32_t)meta[7] << 24;
    for (int plane = 0; plane < 6; ++plane) {
      w[8 + 2 * plane] = q[plane][0] | q[plane][1] << 8 | q[plane][2] << 16 | (uint32_t)q[plane][3] << 24;
      w[9 + 2 * plane] = q[plane][4] | q[plane][5] << 8 | q[plane][6] << 16 | (uint32_t)q[plane][7] << 24;
    }
    uint32_t next = child_base;
    for (int s = 0; s < 8; ++s)
      if (slot_of[s] >= 0 && bn[kids[slot_of[s]]].count == 0) queue.push_back({next++, kids[slot_of[s]], task.level + 1});
  }
}

}  // namespace

void build_wide8(const std::vector<SrcTri>& tris, Wide8Blas& out) {
  out = Wide8Blas{};
  if (tris.empty()) return;
  Binary bin(tris);
  const int broot = bin.build();
  std::vector<BNode> bn = bin.nodes();
  struct TriLeaf {
    const std::vector<SrcTri>& tris;
    std::vector<uint32_t>& words;
    uint32_t base() const { return (uint32_t)(words.size() / W8_TRI_WORDS); }
    void operator()(uint32_t ref) {
      const SrcTri& src = tris[ref];
      for (int j = 0; j < 9; ++j) words.push_back(as_bits(src.v[j]));
      words.push_back(src.ident);
      words.push_back(src.ref);
      words.push_back(0);
    }
  } leaf{tris, out.tris};
  emit_wide8(bn, broot, bin.refs(), out.nodes, out.max_exponent, out.depth, leaf);
}

void build_wide8_top(const std::vector<Aabb>& boxes, Wide8Top& out) {
  out = Wide8Top{};
  if (boxes.empty()) return;
  Binary bin(boxes);
  const int broot = bin.build();
  std::vector<BNode> bn = bin.nodes();
  struct InstanceLeaf {
    std::vector<uint32_t>& items;
    uint32_t base() const { return (uint32_t)items.size(); }
    void operator()(uint32_t ref) { items.push_back(ref); }
  } leaf{out.items};
  emit_wide8(bn, broot, bin.refs(), out.nodes, out.max_exponent, out.depth, leaf);
}

namespace {

// Triangles of one BLAS of the packed words, in the BVH4-Q8's leaf order.
void gather(uint32_t layout, const uint32_t* w, const uint32_t* rec, std::vector<SrcTri>& out) {
  std::vector<uint32_t> stack;
  if (layout == 1) {
    const size_t nodes = rec[18] & ~3u, tris = rec[19] & ~3u;
    stack.push_back(rec[20]);
    while (!stack.empty()) {
      uint32_t c = stack.back();
      stack.pop_back();
      if (c & LEAF) {
        const uint32_t start = (c & ~LEAF) >> 4, cnt = c & 15u;
        for (uint32_t k = 0; k < cnt; ++k) {
          const size_t X = tris + 12 * (size_t)(start + k);
          SrcTri t;
          for (int a = 0; a < 3; ++a) {
            const double va = as_float(w[X + a]);
            t.v[a] = (float)va;
            t.v[3 + a] = (float)(va + (double)as_float(w[X + 3 + a]));
            t.v[6 + a] = (float)(va + (double)as_float(w[X + 6 + a]));
          }
          t.ident = w[X + 9];
          t.ref = (uint32_t)X;
          out.push_back(t);
        }
        continue;
      }
      const uint32_t* n = w + nodes + 16 * (size_t)c;
      for (int s = 3; s >= 0; --s)
        if (n[6 + s] != EMPTY) stack.push_back(n[6 + s]);
    }
    return;
  }
  const size_t nodes = rec[18], leaves = rec[19], positions = rec[20], indices = rec[21];
  stack.push_back(rec[22]);
  while (!stack.empty()) {
    uint32_t c = stack.back();
    stack.pop_back();
    if (c & LEAF) {
      const size_t l = leaves + 2 * (size_t)(c & ~LEAF);
      const uint32_t first = w[l], cnt = w[l + 1];
      for (uint32_t k = 0; k < cnt; k += 3) {
        const size_t x = indices + first + k;
        SrcTri t;
        for (int j = 0; j < 3; ++j)
          for (int a = 0; a < 3; ++a) t.v[3 * j + a] = as_float(w[positions + 3 * (size_t)w[x + j] + a]);
        t.ident = (first + k) / 3;
        t.ref = (uint32_t)x;
        out.push_back(t);
      }
      continue;
    }
    const uint32_t* n = w + nodes + 16 * (size_t)c;
    for (int s = 3; s >= 0; --s)
      if (n[6 + s] != EMPTY) stack.push_back(n[6 + s]);
  }
}

}  // namespace

bool build_wide8_scene(uint32_t layout, const uint32_t* w, size_t n_words, Wide8Scene& out, std::string& err,
                       int threads) {
  (void)n_words;
  out = Wide8Scene{};
  const uint32_t count = w[0];
  const size_t header = layout == 0 ? 16 : 8, stride = layout == 0 ? 32 : 24;
  std::map<std::vector<uint32_t>, uint32_t> key_to_blas;
  std::vector<const uint32_t*> first_rec;
  std::vector<uint32_t> blas_of(count);
  for (uint32_t i = 0; i < count; ++i) {
    const uint32_t* r = w + header + stride * (size_t)i;
    std::vector<uint32_t> key = layout == 0 ? std::vector<uint32_t>{r[18], r[19], r[20], r[21], r[22]}
                                            : std::vector<uint32_t>{r[18] & ~3u, r[19] & ~3u, r[20]};
    auto it = key_to_blas.find(key);
    if (it == key_to_blas.end()) {
      it = key_to_blas.emplace(key, (uint32_t)first_rec.size()).first;
      first_rec.push_back(r);
    }
    blas_of[i] = it->second;
  }
  const size_t nb = first_rec.size();
  std::vector<Wide8Blas> built(nb);
  std::atomic<size_t> next{0};
  auto work = [&] {
    for (;;) {
      size_t b = next.fetch_add(1);
      if (b >= nb) break;
      std::vector<SrcTri> tris;
      gather(layout, w, first_rec[b], tris);
      build_wide8(tris, built[b]);
    }
  };
  const int nt = std::max(1, std::min<int>(threads, (int)nb));
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t) pool.emplace_back(work);
  work();
  for (auto& t : pool) t.join();
  std::vector<uint32_t> node_base(nb), tri_base(nb);
  size_t nn = 0, ntri = 0;
  for (size_t b = 0; b < nb; ++b) {
    out.depth = std::max(out.depth, built[b].depth);
    if (built[b].max_exponent > W8_MAX_EXPONENT) {
      err = "a BLAS extends beyond 255 * 2^13 units on an axis: its 8-wide nodes cannot be decoded exactly";
      return false;
    }
    node_base[b] = (uint32_t)nn;
    tri_base[b] = (uint32_t)ntri;
    nn += built[b].nodes.size() / W8_NODE_WORDS;
    ntri += built[b].tris.size() / W8_TRI_WORDS;
  }
  if (nn >= (1u << 31) || ntri >= (1u << 31)) {
    err = "8-wide layout too large";
    return false;
  }
  out.nodes.reserve(nn * W8_NODE_WORDS);
  out.tris.reserve(ntri * W8_TRI_WORDS);
  for (size_t b = 0; b < nb; ++b) {
    const size_t at = out.nodes.size();
    out.nodes.insert(out.nodes.end(), built[b].nodes.begin(), built[b].nodes.end());
    for (size_t k = at; k < out.nodes.size(); k += W8_NODE_WORDS) {
      out.nodes[k + 4] += node_base[b];
      out.nodes[k + 5] += tri_base[b];
    }
    out.tris.insert(out.tris.end(), built[b].tris.begin(), built[b].tris.end());
  }
  out.inst.resize(2 * (size_t)count);
  for (uint32_t i = 0; i < count; ++i) {
    out.inst[2 * i] = built[blas_of[i]].nodes.empty() ? EMPTY : node_base[blas_of[i]];
    out.inst[2 * i + 1] = tri_base[blas_of[i]];
  }
  out.blas_count = nb;
  build_wide8_top_of(layout, w, out.top_nodes, out.top_items, &out.top_depth);
  return true;
}

bool build_wide8_top_of(uint32_t layout, const uint32_t* w, std::vector<uint32_t>& nodes, std::vector<uint32_t>& items,
                        uint32_t* depth) {
  nodes.clear(), items.clear();
  const uint32_t count = w[0];
  if (w[1] == 0 || count < 2) return false;  // a flat instance list: the walk loops over it
  const size_t header = layout == 0 ? 16 : 8, stride = layout == 0 ? 32 : 24;
  std::vector<Aabb> boxes;
  std::vector<uint32_t> which;
  for (uint32_t i = 0; i < count; ++i) {
    const uint32_t* r = w + header + stride * (size_t)i;
    Aabb b;
    bool ok = true;
    for (int a = 0; a < 3; ++a) {
      b.lo[a] = as_float(r[12 + a]), b.hi[a] = as_float(r[15 + a]);
      ok = ok && std::isfinite(b.lo[a]) && std::isfinite(b.hi[a]) && b.lo[a] <= b.hi[a];
    }
    if (ok) boxes.push_back(b), which.push_back(i);
  }
  if (boxes.empty()) return false;
  Wide8Top top;
  build_wide8_top(boxes, top);
  // the walk's top stack holds a group entry a level plus one node's eight leaves
  if (top.max_exponent > W8_MAX_EXPONENT || top.depth + 9 > W8_TOP_STACK) return false;
  for (uint32_t& it : top.items) it = which[it];
  nodes = std::move(top.nodes);
  items = std::move(top.items);
  if (depth) *depth = top.depth;
  return true;
}

}  // namespace rtb
