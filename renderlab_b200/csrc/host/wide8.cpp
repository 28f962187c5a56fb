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
#include <queue>
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
  // `fork_levels`: the top levels whose right subtrees are built by threads of their own (subtrees
  // of at least FORK_MIN primitives). The tree is the same as a serial build's, node for node.
  int build(int fork_levels = 0) { return node(0, (uint32_t)ref_.size(), nodes_, fork_levels); }
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

  static constexpr uint32_t FORK_MIN = 1u << 15;

  static int leaf(std::vector<BNode>& out, uint32_t first, uint32_t n, const Aabb& b) {
    out.push_back(BNode{b, {-1, -1}, first, n});
    return (int)out.size() - 1;
  }

  // Builds the subtree over refs [first, first + n) into `out`, in preorder (a node before its
  // left subtree, the left subtree before the right). Threads touch disjoint ref ranges.
  int node(uint32_t first, uint32_t n, std::vector<BNode>& out, int fork) {
    Aabb b = Aabb::empty(), cb = Aabb::empty();
    for (uint32_t k = first; k < first + n; ++k) {
      b.grow(box_[ref_[k]]);
      cb.grow(&cen_[3 * (size_t)ref_[k]]);
    }
    if (n == 1) return leaf(out, first, n, b);
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
    if (n <= W8_MAX_LEAF && (best_axis < 0 || COST_TRI * n <= best)) return leaf(out, first, n, b);
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
    const int me = (int)out.size();
    out.push_back(BNode{b, {-1, -1}, 0, 0});
    int l, r;
    if (fork > 0 && first + n - mid >= FORK_MIN && mid - first >= FORK_MIN) {
      std::vector<BNode> right;
      int rr = 0;
      std::thread t([&] { rr = node(mid, first + n - mid, right, fork - 1); });
      l = node(first, mid - first, out, fork - 1);
      t.join();
      const int base = (int)out.size();
      for (BNode x : right) {
        if (x.kid[0] >= 0) x.kid[0] += base, x.kid[1] += base;
        out.push_back(x);
      }
      r = rr + base;
    } else {
      l = node(first, mid - first, out, fork);
      r = node(mid, first + n - mid, out, fork);
    }
    out[me].kid[0] = l;
    out[me].kid[1] = r;
    return me;
  }
};

// Levels of a binary build that fork their right subtrees, for about `threads` threads at once.
int fork_levels(int threads) {
  int levels = 0;
  while (levels < 6 && (2 << levels) <= threads) ++levels;
  return levels;
}

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

void build_wide8(const std::vector<SrcTri>& tris, Wide8Blas& out, int threads) {
  out = Wide8Blas{};
  if (tris.empty()) return;
  Binary bin(tris);
  const int broot = bin.build(fork_levels(threads));
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

void build_wide8_top(const std::vector<Aabb>& boxes, Wide8Top& out, int threads) {
  out = Wide8Top{};
  if (boxes.empty()) return;
  Binary bin(boxes);
  const int broot = bin.build(fork_levels(threads));
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
                       int threads, uint32_t per_instance) {
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
      build_wide8(tris, built[b], std::max(1, threads / (int)nb));
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
  build_wide8_top_of(layout, w, out.nodes, out.inst, out.top_nodes, out.top_items, &out.top_depth, per_instance);
  return true;
}

namespace {

// Object-space box of an 8-wide node: the union of its non-empty children's boxes, exact.
bool node_box(const uint32_t* n, double lo[3], double hi[3]) {
  bool any = false;
  for (int a = 0; a < 3; ++a) lo[a] = INFINITY, hi[a] = -INFINITY;
  for (int s = 0; s < 8; ++s) {
    const uint32_t meta = ((s < 4 ? n[6] : n[7]) >> (8 * (s & 3))) & 255u;
    if (!((n[3] >> (24 + s)) & 1u) && meta == 0) continue;  // empty
    any = true;
    for (int a = 0; a < 3; ++a) {
      const int e = (int)((n[3] >> (8 * a)) & 255u) - 127;
      const uint32_t ql = (n[8 + 2 * a + (s >> 2)] >> (8 * (s & 3))) & 255u;
      const uint32_t qh = (n[8 + 2 * (3 + a) + (s >> 2)] >> (8 * (s & 3))) & 255u;
      lo[a] = std::min(lo[a], (double)as_float(n[a]) + std::ldexp((double)ql, e));
      hi[a] = std::max(hi[a], (double)as_float(n[a]) + std::ldexp((double)qh, e));
    }
  }
  return any;
}

// The inverse of the affine map whose rows are a[0..11] (an instance's world-to-object rows):
// the object-to-world map, in double. False when it is singular or not finite.
bool affine_inverse(const double* a, double* m) {
  const double c00 = a[5] * a[10] - a[6] * a[9], c01 = a[2] * a[9] - a[1] * a[10], c02 = a[1] * a[6] - a[2] * a[5];
  const double c10 = a[6] * a[8] - a[4] * a[10], c11 = a[0] * a[10] - a[2] * a[8], c12 = a[2] * a[4] - a[0] * a[6];
  const double c20 = a[4] * a[9] - a[5] * a[8], c21 = a[1] * a[8] - a[0] * a[9], c22 = a[0] * a[5] - a[1] * a[4];
  const double det = a[0] * c00 + a[1] * c10 + a[2] * c20;
  if (!std::isfinite(det) || det == 0.0) return false;
  const double r[9] = {c00 / det, c01 / det, c02 / det, c10 / det, c11 / det, c12 / det, c20 / det, c21 / det, c22 / det};
  bool ok = true;
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) m[4 * i + j] = r[3 * i + j];
    m[4 * i + 3] = -(r[3 * i] * a[3] + r[3 * i + 1] * a[7] + r[3 * i + 2] * a[11]);
    for (int j = 0; j < 4; ++j) ok = ok && std::isfinite(m[4 * i + j]);
  }
  return ok;
}

double inf_norm(const double* m) {
  double n = 0.0;
  for (int i = 0; i < 3; ++i) n = std::max(n, std::fabs(m[4 * i]) + std::fabs(m[4 * i + 1]) + std::fabs(m[4 * i + 2]));
  return n;
}

// One leaf of the re-braided top level: instance `inst` entered at its BLAS node `node` (global
// index), with the world box of that node's subtree.
struct Entry {
  uint32_t inst, node;
  double lo[3], hi[3];
  double area() const {
    const double x = hi[0] - lo[0], y = hi[1] - lo[1], z = hi[2] - lo[2];
    return x * y + y * z + z * x;
  }
};

}  // namespace

bool instance_model(const uint32_t* rows, double* m) {
  double a[12];
  for (int k = 0; k < 12; ++k) a[k] = as_float(rows[k]);
  return affine_inverse(a, m);
}

bool entry_object_box(const uint32_t* node, double* lo, double* hi) { return node_box(node, lo, hi); }

void entry_world_box(const double* m, const double* olo, const double* ohi, double* lo, double* hi) {
  for (int a = 0; a < 3; ++a) lo[a] = INFINITY, hi[a] = -INFINITY;
  for (int c = 0; c < 8; ++c) {
    const double p[3] = {c & 1 ? ohi[0] : olo[0], c & 2 ? ohi[1] : olo[1], c & 4 ? ohi[2] : olo[2]};
    for (int a = 0; a < 3; ++a) {
      const double x = m[4 * a] * p[0] + m[4 * a + 1] * p[1] + m[4 * a + 2] * p[2] + m[4 * a + 3];
      lo[a] = std::min(lo[a], x), hi[a] = std::max(hi[a], x);
    }
  }
}

bool build_wide8_top_of(uint32_t layout, const uint32_t* w, const std::vector<uint32_t>& blas_nodes,
                        const std::vector<uint32_t>& inst, std::vector<uint32_t>& nodes, std::vector<uint32_t>& items,
                        uint32_t* depth, uint32_t per_instance) {
  nodes.clear(), items.clear();
  const uint32_t count = w[0];
  if (w[1] == 0 || count < 2) return false;  // a flat instance list: the walk loops over it
  const size_t header = layout == 0 ? 16 : 8, stride = layout == 0 ? 32 : 24;
  const size_t n_blas_nodes = blas_nodes.size() / W8_NODE_WORDS;
  // the instances the walk may enter: a usable record world box (the reference's top level culls
  // every other one) and a non-empty BLAS
  std::vector<uint32_t> live;
  double scene_abs = 0.0;
  for (uint32_t i = 0; i < count; ++i) {
    const uint32_t* r = w + header + stride * (size_t)i;
    bool ok = 2 * (size_t)i + 1 < inst.size() && inst[2 * i] < n_blas_nodes;
    for (int a = 0; a < 3; ++a) {
      const float l = as_float(r[12 + a]), h = as_float(r[15 + a]);
      ok = ok && std::isfinite(l) && std::isfinite(h) && l <= h;
    }
    if (!ok) continue;
    live.push_back(i);
    for (int a = 0; a < 3; ++a)
      scene_abs = std::max({scene_abs, std::fabs((double)as_float(r[12 + a])), std::fabs((double)as_float(r[15 + a]))});
  }
  if (live.empty()) return false;
  // Per instance its object-to-world map and the map's condition (|M| |M^-1|, infinity norms).
  std::vector<std::array<double, 12>> model(count);
  std::vector<double> cond(count, 0.0);
  std::vector<uint8_t> mapped(count, 0);
  std::vector<Entry> entries;
  entries.reserve(std::min<size_t>((size_t)per_instance * live.size(), W8_BRAID_MAX) + 8);
  auto world_of = [&](uint32_t i, uint32_t node, Entry& e) {
    double olo[3], ohi[3];
    if (!node_box(&blas_nodes[(size_t)node * W8_NODE_WORDS], olo, ohi)) return false;
    entry_world_box(model[i].data(), olo, ohi, e.lo, e.hi);
    // Margin for the rounding of the walk's f32 object-space ray: the world ray passes within
    // about 12 u |M| |M^-1| (|o| + |hit|) of M p when the f32 object ray meets object point p
    // (u = 2^-24); 2^-16 of the scene's extent covers rays starting within about 20 extents.
    const double pad = W8_BRAID_PAD * cond[i] * (scene_abs + std::max({e.hi[0] - e.lo[0], e.hi[1] - e.lo[1], e.hi[2] - e.lo[2]}));
    for (int a = 0; a < 3; ++a) e.lo[a] -= pad, e.hi[a] += pad;
    e.inst = i, e.node = node;
    return std::isfinite(e.lo[0] + e.lo[1] + e.lo[2] + e.hi[0] + e.hi[1] + e.hi[2]);
  };
  struct Open {
    double area;
    size_t at;
    bool operator<(const Open& o) const { return area < o.area; }
  };
  std::priority_queue<Open> open;
  for (uint32_t i : live) {
    const uint32_t* r = w + header + stride * (size_t)i;
    double rows[12];
    for (int k = 0; k < 12; ++k) rows[k] = as_float(r[k]);
    Entry e;
    if (affine_inverse(rows, model[i].data())) {
      mapped[i] = 1;
      cond[i] = inf_norm(model[i].data()) * inf_norm(rows);
      if (world_of(i, inst[2 * i], e)) {
        entries.push_back(e);
        open.push({e.area(), entries.size() - 1});
        continue;
      }
      mapped[i] = 0;
    }
    // no usable object-to-world map: the instance whole, under its record world box
    e.inst = i, e.node = inst[2 * i];
    for (int a = 0; a < 3; ++a) e.lo[a] = as_float(r[12 + a]), e.hi[a] = as_float(r[15 + a]);
    entries.push_back(e);
  }
  // Re-braiding (Benthin, Woop, Wald and Afra 2017, "Improved Two-Level BVHs using Partial
  // Re-Braiding"): the entry with the largest world box is replaced by its node's children while
  // the budget lasts. Only nodes whose children are all inner nodes open, so the entries of an
  // instance stay an exact cut of its BLAS: every triangle under exactly one entry.
  const size_t budget = std::min<size_t>((size_t)per_instance * live.size(), std::max<size_t>(live.size(), W8_BRAID_MAX));
  while (!open.empty() && entries.size() < budget) {
    const Open top = open.top();
    open.pop();
    const Entry e = entries[top.at];
    const uint32_t* n = &blas_nodes[(size_t)e.node * W8_NODE_WORDS];
    const uint32_t imask = n[3] >> 24;
    if (n[6] != 0 || n[7] != 0 || __builtin_popcount(imask) < 2) continue;  // has leaves, or one child
    Entry kids[8];
    int nk = 0;
    bool ok = true;
    for (int s = 0; s < 8 && ok; ++s)
      if ((imask >> s) & 1u) ok = world_of(e.inst, n[4] + (uint32_t)__builtin_popcount(imask & ((1u << s) - 1u)), kids[nk++]);
    if (!ok) continue;
    entries[top.at] = kids[0];
    open.push({kids[0].area(), top.at});
    for (int k = 1; k < nk; ++k) {
      entries.push_back(kids[k]);
      open.push({kids[k].area(), entries.size() - 1});
    }
  }
  std::vector<Aabb> boxes(entries.size());
  for (size_t k = 0; k < entries.size(); ++k)
    for (int a = 0; a < 3; ++a) {  // rounded outward to f32
      float l = (float)entries[k].lo[a], h = (float)entries[k].hi[a];
      if ((double)l > entries[k].lo[a]) l = std::nextafter(l, -INFINITY);
      if ((double)h < entries[k].hi[a]) h = std::nextafter(h, INFINITY);
      boxes[k].lo[a] = l, boxes[k].hi[a] = h;
    }
  Wide8Top top;
  build_wide8_top(boxes, top, (int)std::max(1u, std::thread::hardware_concurrency()));
  // the walk's top stack holds a group entry a level plus one node's eight leaves
  if (top.max_exponent > W8_MAX_EXPONENT || top.depth + 9 > W8_TOP_STACK) return false;
  items.resize(2 * top.items.size());
  for (size_t k = 0; k < top.items.size(); ++k) {
    const Entry& e = entries[top.items[k]];
    items[2 * k] = e.inst, items[2 * k + 1] = e.node - inst[2 * e.inst];
  }
  nodes = std::move(top.nodes);
  if (depth) *depth = top.depth;
  return true;
}

}  // namespace rtb
