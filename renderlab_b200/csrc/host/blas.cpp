// BVH4-Q8 builder for one mesh: the reference's binned-SAH / median BVH4 with outward-rounded
// 8-bit child boxes (crates/asset/src/near_field.rs:172-537), reorganised around one triangle
// permutation that every split partitions in place. The arithmetic (centroids, bins, costs,
// quantisation) is the reference's, term for term, so the records come out word-identical:
//  * a split's halves keep their input order (`Iterator::partition`, near_field.rs:361-364),
//    which a stable partition of the permutation's range reproduces;
//  * a median split sorts its range by (centroid, triangle) and cuts it in half (:367-379);
//  * leaves, then nodes, are emitted in depth-first postorder (:286-306), so a child's records
//    precede its parent's and the root node is the last one.
// Independent meshes build on separate threads (rt_pack_scene); one mesh builds on one.
#include <algorithm>
#include <cfloat>
#include <numeric>

#include "host.hpp"

namespace rtb {

namespace {

constexpr int BINS = 16;  // near_field.rs:273

inline size_t to_usize(float f) {  // `f as usize`
  if (!(f > 0.0f)) return 0;
  if (f >= 1.8e19f) return SIZE_MAX;
  return (size_t)f;
}
inline uint8_t to_u8(float f) {  // `f.clamp(0.0, 255.0) as u8`
  if (!(f > 0.0f)) return 0;
  if (f >= 255.0f) return 255;
  return (uint8_t)f;
}
inline float half_area(const Aabb& b) {  // near_field.rs:274-277
  float e0 = hi_of(b.hi[0] - b.lo[0], 0.0f), e1 = hi_of(b.hi[1] - b.lo[1], 0.0f),
        e2 = hi_of(b.hi[2] - b.lo[2], 0.0f);
  return e0 * e1 + e1 * e2 + e2 * e0;
}
inline float plane_value(float origin, float step, uint8_t q, bool fused) {
  return fused ? std::fma(step, (float)q, origin) : origin + step * (float)q;
}

class Builder {
 public:
  Builder(const float* pos, const uint32_t* idx, size_t nt, bool sah) : P_(pos), I_(idx), sah_(sah) {
    cen_.resize(3 * nt);
    for (size_t t = 0; t < nt; ++t)
      for (int a = 0; a < 3; ++a) {
        // near_field.rs:216-226: the three corners summed in order, then / 3.
        float s = P_[3 * (size_t)I_[3 * t] + a];
        s = s + P_[3 * (size_t)I_[3 * t + 1] + a];
        s = s + P_[3 * (size_t)I_[3 * t + 2] + a];
        cen_[3 * t + a] = s / 3.0f;
      }
    if (sah_) {
      box_.resize(nt);
      for (size_t t = 0; t < nt; ++t) {
        Aabb b = Aabb::empty();
        for (int k = 0; k < 3; ++k) b.grow(P_ + 3 * (size_t)I_[3 * t + k]);
        box_[t] = b;
      }
    }
    perm_.resize(nt);
    std::iota(perm_.begin(), perm_.end(), 0u);
  }

  uint32_t build(Blas& out) {
    out_ = &out;
    return range(0, perm_.size());
  }

 private:
  const float* P_;
  const uint32_t* I_;
  bool sah_;
  std::vector<float> cen_;
  std::vector<Aabb> box_;
  std::vector<uint32_t> perm_;
  Blas* out_ = nullptr;

  float c(uint32_t t, int a) const { return cen_[3 * (size_t)t + a]; }

  Aabb centroid_box(size_t lo, size_t hi) const {
    Aabb b = Aabb::empty();
    for (size_t k = lo; k < hi; ++k) b.grow(&cen_[3 * (size_t)perm_[k]]);
    return b;
  }

  // Child id of the subtree over perm_[lo, hi) (near_field.rs:286-306).
  uint32_t range(size_t lo, size_t hi) {
    if (hi - lo <= LEAF_TRIANGLES) return leaf(lo, hi);
    size_t cut[5] = {lo, hi, 0, 0, 0};
    int n = 1;  // groups [cut[g], cut[g+1])
    for (int round = 0; round < 2; ++round) {
      size_t next[5];
      int m = 0;
      next[0] = cut[0];
      for (int g = 0; g < n; ++g) {
        size_t a = cut[g], b = cut[g + 1];
        if (b - a > LEAF_TRIANGLES) next[++m] = split(a, b);
        next[++m] = b;
      }
      std::copy(next, next + m + 1, cut);
      n = m;
    }
    uint32_t kids[4];
    for (int g = 0; g < n; ++g) kids[g] = range(cut[g], cut[g + 1]);
    return node(kids, n);
  }

  size_t split(size_t lo, size_t hi) {
    size_t mid;
    if (sah_ && split_sah(lo, hi, mid)) return mid;
    return split_median(lo, hi);
  }

  // near_field.rs:317-366
  bool split_sah(size_t lo, size_t hi, size_t& mid) {
    const Aabb cb = centroid_box(lo, hi);
    const size_t len = hi - lo;
    bool found = false;
    float best = 0.0f;
    int best_axis = 0;
    int best_plane = 0;
    for (int axis = 0; axis < 3; ++axis) {
      const float extent = cb.hi[axis] - cb.lo[axis];
      if (std::isnan(extent) || extent <= 0.0f) continue;
      size_t count[BINS] = {};
      Aabb bins[BINS];
      for (auto& b : bins) b = Aabb::empty();
      for (size_t k = lo; k < hi; ++k) {
        uint32_t t = perm_[k];
        size_t bin = std::min(to_usize((c(t, axis) - cb.lo[axis]) / extent * (float)BINS), (size_t)BINS - 1);
        count[bin] += 1;
        bins[bin].grow(box_[t]);
      }
      float right[BINS];
      Aabb acc = Aabb::empty();
      size_t seen = 0;
      for (int b = BINS - 1; b >= 1; --b) {
        acc.grow(bins[b]);
        seen += count[b];
        right[b] = half_area(acc) * (float)seen;
      }
      acc = Aabb::empty();
      seen = 0;
      for (int b = 0; b < BINS - 1; ++b) {
        acc.grow(bins[b]);
        seen += count[b];
        if (seen == 0 || seen == len) continue;
        const float cost = half_area(acc) * (float)seen + right[b + 1];
        if (!found || cost < best) found = true, best = cost, best_axis = axis, best_plane = b;
      }
    }
    if (!found) return false;
    const float extent = cb.hi[best_axis] - cb.lo[best_axis];
    const float base = cb.lo[best_axis];
    auto left = std::stable_partition(perm_.begin() + lo, perm_.begin() + hi, [&](uint32_t t) {
      size_t bin = std::min(to_usize((c(t, best_axis) - base) / extent * (float)BINS), (size_t)BINS - 1);
      return (int)bin <= best_plane;
    });
    mid = (size_t)(left - perm_.begin());
    return true;
  }

  // near_field.rs:367-379; the last of equal extents wins (Iterator::max_by).
  size_t split_median(size_t lo, size_t hi) {
    const Aabb cb = centroid_box(lo, hi);
    int axis = 0;
    for (int a = 1; a < 3; ++a)
      if (order_key(cb.hi[a] - cb.lo[a]) >= order_key(cb.hi[axis] - cb.lo[axis])) axis = a;
    std::sort(perm_.begin() + lo, perm_.begin() + hi, [&](uint32_t x, uint32_t y) {
      int32_t kx = order_key(c(x, axis)), ky = order_key(c(y, axis));
      return kx != ky ? kx < ky : x < y;
    });
    return lo + (hi - lo) / 2;
  }

  // near_field.rs:380-401
  uint32_t leaf(size_t lo, size_t hi) {
    uint32_t offset = (uint32_t)out_->indices.size();
    for (size_t k = lo; k < hi; ++k) {
      const uint32_t* t = I_ + 3 * (size_t)perm_[k];
      out_->indices.insert(out_->indices.end(), t, t + 3);
    }
    uint32_t id = (uint32_t)out_->leaf_count();
    out_->leaves.push_back(offset);
    out_->leaves.push_back((uint32_t)(3 * (hi - lo)));
    out_->leaf_source.push_back((uint32_t)(3 * (size_t)perm_[lo]));  // Leaf::source_index_offset
    return id | LEAF;
  }

  // near_field.rs:402-430: a leaf's vertex bounds, or the union of a node's children under both
  // decodes.
  Aabb bounds_of(uint32_t child) const {
    Aabb b = Aabb::empty();
    if (child & LEAF) {
      uint32_t l = child & ~LEAF;
      uint32_t off = out_->leaves[2 * l], cnt = out_->leaves[2 * l + 1];
      for (uint32_t k = off; k < off + cnt; ++k) b.grow(P_ + 3 * (size_t)out_->indices[k]);
      return b;
    }
    const uint32_t* w = &out_->nodes[16 * (size_t)child];
    for (int s = 0; s < 4; ++s) {
      if (w[6 + s] == EMPTY) continue;
      for (int fused = 0; fused < 2; ++fused)
        for (int a = 0; a < 3; ++a) {
          float o = as_float(w[a]), st = as_float(w[3 + a]);
          uint8_t ql = (w[10 + a] >> (8 * s)) & 255u, qh = (w[13 + a] >> (8 * s)) & 255u;
          b.lo[a] = lo_of(b.lo[a], plane_value(o, st, ql, fused));
          b.hi[a] = hi_of(b.hi[a], plane_value(o, st, qh, fused));
        }
    }
    return b;
  }

  uint32_t node(const uint32_t* kids, int n) {
    Aabb boxes[4];
    for (int k = 0; k < n; ++k) boxes[k] = bounds_of(kids[k]);
    uint32_t id = (uint32_t)out_->node_count();
    out_->nodes.resize(out_->nodes.size() + 16);
    quantize_node(kids, boxes, n, &out_->nodes[16 * (size_t)id]);
    return id;
  }
};

}  // namespace

// near_field.rs:481-525: origin = the children's union low corner; per axis the smallest step
// (grown by 2^-20 steps) whose code 255 reaches the top under both decodes; codes rounded
// outward until both decodes enclose the child.
void quantize_node(const uint32_t* children, const Aabb* boxes, int n, uint32_t* w) {
  Aabb all = Aabb::empty();
  for (int k = 0; k < n; ++k) all.grow(boxes[k]);
  float step[3];
  for (int a = 0; a < 3; ++a) {
    const float lo = all.lo[a], hi = all.hi[a];
    float s = hi_of((hi - lo) / 255.0f, hi_of(FLT_MIN, std::fabs(lo) * 1e-7f));
    while (lo + s * 255.0f < hi || std::fma(s, 255.0f, lo) < hi) s *= 1.0f + 1.0f / 1048576.0f;
    step[a] = s;
  }
  uint8_t lower[3][4] = {}, upper[3][4] = {};
  for (int k = 0; k < n; ++k)
    for (int a = 0; a < 3; ++a) {
      const float o = all.lo[a], s = step[a], x = boxes[k].lo[a], y = boxes[k].hi[a];
      uint8_t ql = to_u8(std::floor((x - o) / s));
      while (ql > 0 && (plane_value(o, s, ql, false) > x || plane_value(o, s, ql, true) > x)) --ql;
      uint8_t qh = to_u8(std::ceil((y - o) / s));
      while (qh < 255 && (plane_value(o, s, qh, false) < y || plane_value(o, s, qh, true) < y)) ++qh;
      lower[a][k] = ql;
      upper[a][k] = qh;
    }
  for (int a = 0; a < 3; ++a) w[a] = as_bits(all.lo[a]), w[3 + a] = as_bits(step[a]);
  for (int s = 0; s < 4; ++s) w[6 + s] = s < n ? children[s] : EMPTY;
  for (int a = 0; a < 3; ++a) {
    w[10 + a] = lower[a][0] | lower[a][1] << 8 | lower[a][2] << 16 | (uint32_t)lower[a][3] << 24;
    w[13 + a] = upper[a][0] | upper[a][1] << 8 | upper[a][2] << 16 | (uint32_t)upper[a][3] << 24;
  }
}

bool build_blas(const float* pos, size_t npos, const uint32_t* idx, size_t nidx, bool sah, Blas& out,
                std::string& err) {
  if (nidx == 0 || nidx % 3 != 0) {
    err = "BVH geometry needs a nonempty triangle list";
    return false;
  }
  for (size_t k = 0; k < nidx; ++k)
    if (idx[k] >= npos) {
      err = "BVH geometry has an invalid index or position";
      return false;
    }
  for (size_t k = 0; k < 3 * npos; ++k)
    if (!std::isfinite(pos[k])) {
      err = "BVH geometry has an invalid index or position";
      return false;
    }
  out = Blas{};
  out.positions.assign(pos, pos + 3 * npos);
  out.indices.reserve(nidx);
  out.bounds = Aabb::empty();
  for (size_t v = 0; v < npos; ++v) out.bounds.grow(pos + 3 * v);
  Builder b(pos, idx, nidx / 3, sah);
  out.root = b.build(out);
  return true;
}

size_t blas_depth(const Blas& b, uint32_t child) {
  if (child & LEAF) return 0;
  size_t deepest = 0;
  const uint32_t* w = &b.nodes[16 * (size_t)child];
  for (int s = 0; s < 4; ++s)
    if (w[6 + s] != EMPTY) deepest = std::max(deepest, blas_depth(b, w[6 + s]));
  return 1 + deepest;
}

bool build_blas_sah(const float* pos, size_t npos, const uint32_t* idx, size_t nidx, Blas& out,
                    std::string& err) {
  if (!build_blas(pos, npos, idx, nidx, true, out, err)) return false;
  if (blas_depth(out, out.root) > MAX_SAH_DEPTH) return build_blas(pos, npos, idx, nidx, false, out, err);
  return true;
}

// near_field.rs:445-478: nodes are in postorder, so one forward pass sees children first.
bool refit_blas(Blas& b, const float* pos, size_t npos, std::string& err) {
  if (npos * 3 != b.positions.size()) {
    err = "BVH refit needs finite positions of the same vertices";
    return false;
  }
  for (size_t k = 0; k < 3 * npos; ++k)
    if (!std::isfinite(pos[k])) {
      err = "BVH refit needs finite positions of the same vertices";
      return false;
    }
  b.positions.assign(pos, pos + 3 * npos);
  for (size_t n = 0; n < b.node_count(); ++n) {
    uint32_t* w = &b.nodes[16 * n];
    uint32_t kids[4];
    Aabb boxes[4];
    int m = 0;
    for (int s = 0; s < 4; ++s) {
      uint32_t ch = w[6 + s];
      if (ch == EMPTY) continue;
      Aabb bb = Aabb::empty();
      if (ch & LEAF) {
        uint32_t l = ch & ~LEAF;
        for (uint32_t k = b.leaves[2 * l]; k < b.leaves[2 * l] + b.leaves[2 * l + 1]; ++k) bb.grow(pos + 3 * (size_t)b.indices[k]);
      } else {
        const uint32_t* c = &b.nodes[16 * (size_t)ch];
        for (int t = 0; t < 4; ++t) {
          if (c[6 + t] == EMPTY) continue;
          for (int fused = 0; fused < 2; ++fused)
            for (int a = 0; a < 3; ++a) {
              float o = as_float(c[a]), st = as_float(c[3 + a]);
              bb.lo[a] = lo_of(bb.lo[a], plane_value(o, st, (c[10 + a] >> (8 * t)) & 255u, fused));
              bb.hi[a] = hi_of(bb.hi[a], plane_value(o, st, (c[13 + a] >> (8 * t)) & 255u, fused));
            }
        }
      }
      kids[m] = ch;
      boxes[m] = bb;
      ++m;
    }
    quantize_node(kids, boxes, m, w);
  }
  b.bounds = Aabb::empty();
  for (size_t v = 0; v < npos; ++v) b.bounds.grow(pos + 3 * v);
  return true;
}

}  // namespace rtb
