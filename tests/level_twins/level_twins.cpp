// CPU models of the device builders' level-synchronous decompositions (renderlab_b200/csrc/
// blas_build.cu, tlas_build.cu), checked against the host builders they must reproduce word for
// word (host/blas.cpp, host/tlas.cpp). Each model:
//  * splits every pending range of one binary depth at once;
//  * takes each range's min/max reductions over its elements in a shuffled order, through
//    order-preserving integer keys, as the device's atomics do in whatever order they land;
//  * derives the record ids and child slots from the ranges alone: BLAS nodes in postorder by
//    (range end, range length), leaves by range start, children by range start; top-level nodes
//    in preorder from subtree sizes after the largest-area-first collapse.
// main() runs both over seeded inputs: ties, signed zeros, shared vertices, identical and
// zero-area boxes, and trees deep enough for each builder's median fallback. It prints one line
// per mismatch and exits non-zero if there is any.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <random>
#include <string>

#include "host/host.hpp"

using namespace rtb;

namespace {

uint32_t okey(float f) {  // f32::total_cmp as an unsigned comparison
  const uint32_t b = as_bits(f);
  return b ^ ((b >> 31) ? 0xffffffffu : 0x80000000u);
}
float unkey(uint32_t k) { return as_float(k ^ ((k >> 31) ? 0x80000000u : 0xffffffffu)); }
size_t to_usize(float f) {  // `f as usize`
  if (!(f > 0.0f)) return 0;
  if (f >= 1.8e19f) return SIZE_MAX;
  return (size_t)f;
}
float area(const float* lo, const float* hi) {  // near_field.rs:274-277, instance_bvh.rs:290-293
  const float e0 = hi_of(hi[0] - lo[0], 0.0f), e1 = hi_of(hi[1] - lo[1], 0.0f), e2 = hi_of(hi[2] - lo[2], 0.0f);
  return e0 * e1 + e1 * e2 + e2 * e0;
}

// Bin boxes kept as keys; an empty bin adds nothing to a sweep.
struct KeyBins {
  uint32_t cnt[16] = {};
  uint32_t lo[16][3], hi[16][3];
  KeyBins() {
    for (int b = 0; b < 16; ++b)
      for (int a = 0; a < 3; ++a) lo[b][a] = ~0u, hi[b][a] = 0;
  }
  void add(int b, const float* l, const float* h) {
    ++cnt[b];
    for (int a = 0; a < 3; ++a) lo[b][a] = std::min(lo[b][a], okey(l[a])), hi[b][a] = std::max(hi[b][a], okey(h[a]));
  }
  void grow(int b, float* al, float* ah) const {
    if (!cnt[b]) return;
    for (int a = 0; a < 3; ++a) al[a] = lo_of(al[a], unkey(lo[b][a])), ah[a] = hi_of(ah[a], unkey(hi[b][a]));
  }
};

void key_box(const std::vector<uint32_t>& order, const float* pts, float* lo, float* hi) {
  uint32_t l[3] = {~0u, ~0u, ~0u}, h[3] = {0, 0, 0};
  for (uint32_t i : order)
    for (int a = 0; a < 3; ++a) l[a] = std::min(l[a], okey(pts[3 * (size_t)i + a])), h[a] = std::max(h[a], okey(pts[3 * (size_t)i + a]));
  for (int a = 0; a < 3; ++a) lo[a] = unkey(l[a]), hi[a] = unkey(h[a]);
}

int median_axis(const float* lo, const float* hi) {  // the last of equal extents (Iterator::max_by)
  int axis = 0;
  for (int a = 1; a < 3; ++a)
    if (order_key(hi[a] - lo[a]) >= order_key(hi[axis] - lo[axis])) axis = a;
  return axis;
}

void median_sort(std::vector<uint32_t>& perm, uint32_t b, uint32_t e, const float* pts, int axis) {
  std::sort(perm.begin() + b, perm.begin() + e, [&](uint32_t x, uint32_t y) {
    const uint64_t kx = (uint64_t)okey(pts[3 * (size_t)x + axis]) << 32 | x, ky = (uint64_t)okey(pts[3 * (size_t)y + axis]) << 32 | y;
    return kx < ky;
  });
}

// ---- BLAS (near_field.rs:172-436) ----

struct Range {
  uint32_t b, e, depth, owner;
};

bool model_blas(const float* P, size_t npos, const uint32_t* I, size_t nidx, bool sah, Blas& out, bool& too_deep,
                std::mt19937& rng) {
  const size_t nt = nidx / 3;
  std::vector<float> cen(3 * nt), tb(6 * nt);
  for (size_t t = 0; t < nt; ++t) {
    for (int a = 0; a < 3; ++a) {
      float s = P[3 * (size_t)I[3 * t] + a];
      s = s + P[3 * (size_t)I[3 * t + 1] + a];
      s = s + P[3 * (size_t)I[3 * t + 2] + a];
      cen[3 * t + a] = s / 3.0f;
    }
    Aabb b = Aabb::empty();
    for (int k = 0; k < 3; ++k) b.grow(P + 3 * (size_t)I[3 * t + k]);
    for (int a = 0; a < 3; ++a) tb[6 * t + a] = b.lo[a], tb[6 * t + 3 + a] = b.hi[a];
  }
  std::vector<uint32_t> perm(nt);
  for (size_t i = 0; i < nt; ++i) perm[i] = (uint32_t)i;
  std::vector<Range> ranges{{0, (uint32_t)nt, 0, EMPTY}};
  std::vector<std::pair<size_t, size_t>> levels;
  size_t lv0 = 0, lv1 = 1;
  too_deep = false;
  for (;;) {
    levels.push_back({lv0, lv1});
    std::vector<Range> next;
    for (size_t s = lv0; s < lv1; ++s) {
      const Range g = ranges[s];
      const uint32_t len = g.e - g.b;
      if (len <= LEAF_TRIANGLES) continue;
      if (sah && g.depth >= 2 * MAX_SAH_DEPTH) return too_deep = true, false;
      std::vector<uint32_t> shuffled(perm.begin() + g.b, perm.begin() + g.e);
      std::shuffle(shuffled.begin(), shuffled.end(), rng);
      float lo[3], hi[3];
      key_box(shuffled, cen.data(), lo, hi);
      bool found = false;
      float best = 0.0f;
      int bax = 0, bplane = 0;
      for (int axis = 0; sah && axis < 3; ++axis) {
        const float ext = hi[axis] - lo[axis];
        if (!(ext > 0.0f)) continue;
        KeyBins bins;
        for (uint32_t t : shuffled)
          bins.add((int)std::min(to_usize((cen[3 * (size_t)t + axis] - lo[axis]) / ext * 16.0f), (size_t)15), &tb[6 * (size_t)t],
                   &tb[6 * (size_t)t + 3]);
        float right[16], al[3] = {INFINITY, INFINITY, INFINITY}, ah[3] = {-INFINITY, -INFINITY, -INFINITY};
        size_t seen = 0;
        for (int b = 15; b >= 1; --b) {
          bins.grow(b, al, ah);
          seen += bins.cnt[b];
          right[b] = area(al, ah) * (float)seen;
        }
        for (int a = 0; a < 3; ++a) al[a] = INFINITY, ah[a] = -INFINITY;
        seen = 0;
        for (int b = 0; b < 15; ++b) {
          bins.grow(b, al, ah);
          seen += bins.cnt[b];
          if (seen == 0 || seen == len) continue;
          const float cost = area(al, ah) * (float)seen + right[b + 1];
          if (!found || cost < best) found = true, best = cost, bax = axis, bplane = b;
        }
      }
      uint32_t mid;
      if (found) {
        const float ext = hi[bax] - lo[bax];
        auto left = [&](uint32_t t) { return (int)std::min(to_usize((cen[3 * (size_t)t + bax] - lo[bax]) / ext * 16.0f), (size_t)15) <= bplane; };
        mid = (uint32_t)(std::stable_partition(perm.begin() + g.b, perm.begin() + g.e, left) - perm.begin());
      } else {
        median_sort(perm, g.b, g.e, cen.data(), median_axis(lo, hi));
        mid = g.b + len / 2;
      }
      const uint32_t own = (g.depth % 2 == 0) ? (uint32_t)s : g.owner;
      next.push_back({g.b, mid, g.depth + 1, own});
      next.push_back({mid, g.e, g.depth + 1, own});
    }
    if (next.empty()) break;
    lv0 = ranges.size();
    ranges.insert(ranges.end(), next.begin(), next.end());
    lv1 = ranges.size();
  }
  out = Blas{};
  out.positions.assign(P, P + 3 * npos);
  std::vector<uint32_t> leaf_at(nt, EMPTY);
  std::vector<std::pair<uint64_t, uint32_t>> nodes;
  for (uint32_t s = 0; s < ranges.size(); ++s) {
    const Range& g = ranges[s];
    const uint32_t len = g.e - g.b;
    if (len <= LEAF_TRIANGLES) leaf_at[g.b] = s;
    else if (g.depth % 2 == 0) nodes.push_back({(uint64_t)g.e << 32 | len, s});
  }
  std::vector<uint32_t> id(ranges.size(), EMPTY);
  uint32_t n_leaves = 0;
  for (size_t p = 0; p < nt; ++p)
    if (leaf_at[p] != EMPTY) id[leaf_at[p]] = (n_leaves++) | LEAF;
  std::sort(nodes.begin(), nodes.end());
  for (uint32_t r = 0; r < nodes.size(); ++r) id[nodes[r].second] = r;
  out.leaves.resize(2 * (size_t)n_leaves);
  out.leaf_source.resize(n_leaves);
  out.indices.resize(3 * nt);
  for (size_t k = 0; k < nt; ++k)
    for (int j = 0; j < 3; ++j) out.indices[3 * k + j] = I[3 * (size_t)perm[k] + j];
  for (uint32_t s = 0; s < ranges.size(); ++s)
    if (id[s] != EMPTY && (id[s] & LEAF)) {
      const uint32_t l = id[s] & ~LEAF;
      out.leaves[2 * l] = 3 * ranges[s].b, out.leaves[2 * l + 1] = 3 * (ranges[s].e - ranges[s].b);
      out.leaf_source[l] = 3 * perm[ranges[s].b];
    }
  out.nodes.assign(16 * nodes.size(), 0);
  std::vector<std::vector<std::pair<uint32_t, uint32_t>>> kids(nodes.size());
  for (uint32_t s = 1; s < ranges.size(); ++s)
    if (id[s] != EMPTY) kids[id[ranges[s].owner]].push_back({ranges[s].b, id[s]});
  for (size_t li = levels.size(); li-- > 0;)
    for (size_t s = levels[li].first; s < levels[li].second; ++s) {
      if (id[s] == EMPTY || (id[s] & LEAF)) continue;
      auto& c = kids[id[s]];
      std::sort(c.begin(), c.end());
      uint32_t ch[4];
      Aabb boxes[4];
      const int n = (int)c.size();
      for (int k = 0; k < n; ++k) {
        ch[k] = c[k].second;
        Aabb b = Aabb::empty();
        if (ch[k] & LEAF) {
          const uint32_t l = ch[k] & ~LEAF;
          for (uint32_t q = out.leaves[2 * l]; q < out.leaves[2 * l] + out.leaves[2 * l + 1]; ++q) b.grow(P + 3 * (size_t)out.indices[q]);
        } else {
          const uint32_t* w = &out.nodes[16 * (size_t)ch[k]];
          for (int t = 0; t < 4; ++t) {
            if (w[6 + t] == EMPTY) continue;
            for (int fused = 0; fused < 2; ++fused)
              for (int a = 0; a < 3; ++a) {
                const float o = as_float(w[a]), st = as_float(w[3 + a]);
                const float ql = (float)((w[10 + a] >> (8 * t)) & 255u), qh = (float)((w[13 + a] >> (8 * t)) & 255u);
                b.lo[a] = lo_of(b.lo[a], fused ? std::fma(st, ql, o) : o + st * ql);
                b.hi[a] = hi_of(b.hi[a], fused ? std::fma(st, qh, o) : o + st * qh);
              }
          }
        }
        boxes[k] = b;
      }
      quantize_node(ch, boxes, n, &out.nodes[16 * (size_t)id[s]]);
    }
  out.root = id[0];
  return true;
}

// ---- instance top level (instance_bvh.rs:346-460) ----

std::vector<uint32_t> model_tlas(const std::vector<Aabb>& boxes, bool sah, size_t& levels4, std::mt19937& rng) {
  const uint32_t n = (uint32_t)boxes.size();
  std::vector<float> cen(3 * (size_t)n);
  for (uint32_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) cen[3 * (size_t)i + a] = boxes[i].lo[a] + boxes[i].hi[a];
  std::vector<uint32_t> ids(n);
  for (uint32_t i = 0; i < n; ++i) ids[i] = i;
  struct Node {
    uint32_t b, e, child;
  };
  std::vector<Node> ranges{{0, n, EMPTY}};
  std::vector<std::pair<uint32_t, uint32_t>> levels;
  uint32_t lv0 = 0, width = 1;
  for (;;) {
    levels.push_back({lv0, width});
    std::vector<Node> next;
    for (uint32_t s = lv0; s < lv0 + width; ++s) {
      Node& g = ranges[s];
      const uint32_t len = g.e - g.b;
      if (len < 2) continue;
      std::vector<uint32_t> shuffled(ids.begin() + g.b, ids.begin() + g.e);
      std::shuffle(shuffled.begin(), shuffled.end(), rng);
      float lo[3], hi[3];
      key_box(shuffled, cen.data(), lo, hi);
      bool found = false;
      float best = 0.0f;
      int bax = 0, bbin = 0;
      for (int axis = 0; sah && axis < 3; ++axis) {
        const float ext = hi[axis] - lo[axis];
        if (!(ext > 0.0f)) continue;
        const float scale = 16.0f / ext;
        KeyBins bins;
        for (uint32_t i : shuffled)
          bins.add((int)std::min(to_usize((cen[3 * (size_t)i + axis] - lo[axis]) * scale), (size_t)15), boxes[i].lo, boxes[i].hi);
        float ra[16], al[3] = {INFINITY, INFINITY, INFINITY}, ah[3] = {-INFINITY, -INFINITY, -INFINITY};
        uint32_t rn[16], m = 0;
        for (int b = 15; b >= 1; --b) {
          bins.grow(b, al, ah);
          m += bins.cnt[b];
          ra[b - 1] = area(al, ah), rn[b - 1] = m;
        }
        for (int a = 0; a < 3; ++a) al[a] = INFINITY, ah[a] = -INFINITY;
        m = 0;
        for (int b = 0; b < 15; ++b) {
          bins.grow(b, al, ah);
          m += bins.cnt[b];
          if (m == 0 || rn[b] == 0) continue;
          const float cost = area(al, ah) * (float)m + ra[b] * (float)rn[b];
          if (!found || cost < best) found = true, best = cost, bax = axis, bbin = b;
        }
      }
      uint32_t mid;
      if (found) {
        const float scale = 16.0f / (hi[bax] - lo[bax]);
        auto left = [&](uint32_t i) { return (int)std::min(to_usize((cen[3 * (size_t)i + bax] - lo[bax]) * scale), (size_t)15) <= bbin; };
        mid = (uint32_t)(std::stable_partition(ids.begin() + g.b, ids.begin() + g.e, left) - ids.begin());
      } else {
        median_sort(ids, g.b, g.e, cen.data(), median_axis(lo, hi));
        mid = g.b + len / 2;
      }
      g.child = lv0 + width + (uint32_t)next.size();
      next.push_back({g.b, mid, EMPTY});
      next.push_back({mid, g.e, EMPTY});
    }
    if (next.empty()) break;
    lv0 += width;
    width = (uint32_t)next.size();
    ranges.insert(ranges.end(), next.begin(), next.end());
  }
  auto single = [&](uint32_t s) { return ranges[s].e - ranges[s].b == 1; };
  std::vector<Aabb> box(ranges.size());
  for (size_t li = levels.size(); li-- > 0;)
    for (uint32_t s = levels[li].first; s < levels[li].first + levels[li].second; ++s) {
      if (single(s)) {
        box[s] = boxes[ids[ranges[s].b]];
        continue;
      }
      Aabb all = Aabb::empty();
      all.grow(box[ranges[s].child]);
      all.grow(box[ranges[s].child + 1]);
      box[s] = all;
    }
  std::vector<std::array<uint32_t, 4>> kids(ranges.size());
  std::vector<int> nk(ranges.size(), 0);
  std::vector<std::vector<uint32_t>> wide{{0}};
  for (;;) {
    std::vector<uint32_t> next;
    for (uint32_t x : wide.back()) {
      uint32_t k[4] = {ranges[x].child, ranges[x].child + 1, EMPTY, EMPTY};
      int m = 2;
      while (m < 4) {
        int pick = -1;
        for (int j = 0; j < m; ++j)
          if (!single(k[j]) &&
              (pick < 0 || order_key(area(box[k[j]].lo, box[k[j]].hi)) > order_key(area(box[k[pick]].lo, box[k[pick]].hi))))
            pick = j;
        if (pick < 0) break;
        const uint32_t id = k[pick];
        for (int j = m; j > pick + 1; --j) k[j] = k[j - 1];
        k[pick] = ranges[id].child, k[pick + 1] = ranges[id].child + 1;
        ++m;
      }
      for (int j = 0; j < m; ++j) {
        kids[x][j] = k[j];
        if (!single(k[j])) next.push_back(k[j]);
      }
      nk[x] = m;
    }
    if (next.empty()) break;
    wide.push_back(next);
  }
  levels4 = wide.size();
  std::vector<uint32_t> size(ranges.size(), 0), id(ranges.size(), 0);
  for (size_t li = wide.size(); li-- > 0;)
    for (uint32_t x : wide[li]) {
      size[x] = 1;
      for (int j = 0; j < nk[x]; ++j)
        if (!single(kids[x][j])) size[x] += size[kids[x][j]];
    }
  for (auto& lv : wide)
    for (uint32_t x : lv) {
      uint32_t r = id[x] + 1;
      for (int j = 0; j < nk[x]; ++j)
        if (!single(kids[x][j])) id[kids[x][j]] = r, r += size[kids[x][j]];
    }
  std::vector<uint32_t> out(32 * (size_t)size[0], 0);
  for (auto& lv : wide)
    for (uint32_t x : lv) {
      uint32_t* w = &out[32 * (size_t)id[x]];
      for (int c = 0; c < 4; ++c) {
        if (c >= nk[x]) {
          w[24 + c] = EMPTY;
          continue;
        }
        const uint32_t k = kids[x][c];
        for (int a = 0; a < 3; ++a) w[4 * a + c] = as_bits(box[k].lo[a]), w[12 + 4 * a + c] = as_bits(box[k].hi[a]);
        w[24 + c] = single(k) ? (LEAF | ids[ranges[k].b]) : id[k];
      }
    }
  return out;
}

}  // namespace

int main() {
  int fails = 0;
  std::mt19937 shuffle_rng(7);
  // BLAS: soups, rounded coordinates, signed zeros on one axis, shared vertices; SAH and median.
  for (int trial = 0; trial < 40; ++trial) {
    std::mt19937 r(trial);
    const size_t nt = trial < 5 ? 1 + trial * 3 : 50 + r() % 20000;
    const int mode = trial % 4;
    std::uniform_real_distribution<float> U(-10, 10);
    const size_t nv = mode == 3 ? 40 : 3 * nt;
    std::vector<float> P;
    std::vector<uint32_t> I;
    for (size_t v = 0; v < nv; ++v)
      for (int a = 0; a < 3; ++a) {
        float x = U(r);
        if (mode == 1) x = std::round(x);
        if (mode == 2 && a == 1) x = (r() & 1) ? 0.0f : -0.0f;
        P.push_back(x);
      }
    for (size_t t = 0; t < nt; ++t)
      for (int k = 0; k < 3; ++k) I.push_back(mode == 3 ? (uint32_t)(r() % nv) : (uint32_t)(3 * t + k));
    for (int sah = 0; sah < 2; ++sah) {
      Blas want, got;
      std::string err;
      bool deep = false;
      if (sah) build_blas_sah(P.data(), nv, I.data(), I.size(), want, err);
      else build_blas(P.data(), nv, I.data(), I.size(), false, want, err);
      bool ok = model_blas(P.data(), nv, I.data(), I.size(), sah, got, deep, shuffle_rng);
      if (!ok && deep) ok = model_blas(P.data(), nv, I.data(), I.size(), false, got, deep, shuffle_rng);
      if (!ok || want.nodes != got.nodes || want.leaves != got.leaves || want.indices != got.indices ||
          want.leaf_source != got.leaf_source || want.root != got.root) {
        ++fails;
        std::printf("blas trial %d (%zu triangles, mode %d, sah %d) differs\n", trial, nt, mode, sah);
      }
    }
  }
  // BLAS: exponentially spaced triangles, on both sides of the 15-level SAH limit.
  for (int n : {350, 390}) {
    std::vector<float> P;
    std::vector<uint32_t> I;
    for (int i = 0; i < n; ++i) {
      const float x = std::pow(1.25f, (float)i * 0.999f);
      const float v[9] = {x, 0, 0, x, 1, 0, x, 0, 1};
      P.insert(P.end(), v, v + 9);
      for (int k = 0; k < 3; ++k) I.push_back((uint32_t)(3 * i + k));
    }
    Blas want, got;
    std::string err;
    bool deep = false;
    build_blas_sah(P.data(), P.size() / 3, I.data(), I.size(), want, err);
    bool ok = model_blas(P.data(), P.size() / 3, I.data(), I.size(), true, got, deep, shuffle_rng);
    if (!ok && deep) ok = model_blas(P.data(), P.size() / 3, I.data(), I.size(), false, got, deep, shuffle_rng);
    if (!ok || want.nodes != got.nodes || want.indices != got.indices || want.root != got.root) {
      ++fails;
      std::printf("blas deep %d differs\n", n);
    }
  }
  // Top level: random placements, equal centres, identical boxes, zero-area boxes, signed zeros.
  for (int trial = 0; trial < 60; ++trial) {
    std::mt19937 r(1000 + trial);
    const int mode = trial % 5;
    const uint32_t n = trial < 6 ? 2 + trial : 10 + r() % 30000;
    std::vector<Aabb> b(n);
    std::uniform_real_distribution<float> U(-500, 500), H(0.5f, 4.0f);
    for (uint32_t i = 0; i < n; ++i)
      for (int a = 0; a < 3; ++a) {
        float c = U(r), h = H(r);
        if (mode == 1) c = std::round(c / 100.0f) * 100.0f;
        if (mode == 2) c = 0.0f, h = 1.0f;
        if (mode == 3 && a > 0) h = 0.0f;
        if (mode == 4 && a == 1) c = (r() & 1) ? 0.0f : -0.0f, h = 0.0f;
        b[i].lo[a] = c - h, b[i].hi[a] = c + h;
      }
    for (int sah = 0; sah < 2; ++sah) {
      size_t levels4 = 0;
      std::vector<uint32_t> got = model_tlas(b, sah, levels4, shuffle_rng);
      if (sah && 1 + 3 * levels4 > STACK_DEPTH) got = model_tlas(b, false, levels4, shuffle_rng);
      if (got != tlas_build(b, sah)) {
        ++fails;
        std::printf("top level trial %d (%u boxes, mode %d, sah %d) differs\n", trial, n, mode, sah);
      }
    }
  }
  // Top level: exponentially spaced boxes, with and without the median rebuild.
  for (int n : {200, 400}) {
    std::vector<Aabb> b(n);
    for (int i = 0; i < n; ++i)
      for (int a = 0; a < 3; ++a) {
        const float c = a == 0 ? std::pow(1.25f, (float)i * 0.5f) : 0.0f;
        b[i].lo[a] = c - 0.5f, b[i].hi[a] = c + 0.5f;
      }
    size_t levels4 = 0;
    std::vector<uint32_t> got = model_tlas(b, true, levels4, shuffle_rng);
    if (1 + 3 * levels4 > STACK_DEPTH) got = model_tlas(b, false, levels4, shuffle_rng);
    if (got != tlas_build(b, true)) {
      ++fails;
      std::printf("top level deep %d differs\n", n);
    }
  }
  std::printf("mismatches %d\n", fails);
  return fails != 0;
}
