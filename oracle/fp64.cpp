// CPU ORACLE — test infrastructure only. The f64 reference traversal of
// crates/asset/src/cluster_bvh/reference.rs:47-194 (Möller–Trumbore, slab test, closest hit with
// a lexicographic tie rule), restated for one Bvh (`fp64_trace_bvh`) and wrapped over the packed
// GI and reflection buffers: each instance's f32 world-to-object rows are widened to f64 and the
// object-space ray keeps the world ray's parameter t. Ties resolve on (t, instance, triangle).
// Rays are accepted on the open interval (tmin, tmax), the contract of the f32 traversal.
#include <algorithm>
#include <vector>

#include "oracle.hpp"

namespace orc {

namespace {

struct D3 { double x, y, z; };
inline D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
// reference.rs:50-52: `Sum for f64` starts from -0.0, which leaves the first product unchanged.
inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline D3 cross(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double comp(D3 v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

// reference.rs:60-79
bool box_hit(D3 o, D3 d, double tmin, const double lo[3], const double hi[3], double max) {
  double near = tmin, far = max;
  for (int a = 0; a < 3; ++a) {
    double oa = comp(o, a), da = comp(d, a);
    if (da == 0.0) {
      if (oa < lo[a] || oa > hi[a]) return false;
    } else {
      double x = (lo[a] - oa) / da, y = (hi[a] - oa) / da;
      near = std::max(near, std::min(x, y));
      far = std::min(far, std::max(x, y));
      if (near > far) return false;
    }
  }
  return true;
}

// reference.rs:121-158, one triangle given corner a and edges ab, ac. Returns t (or NAN).
bool mt64(D3 o, D3 d, D3 a, D3 ab, D3 ac, double& t, double& u, double& v) {
  D3 p = cross(d, ac);
  double det = dot(ab, p);
  if (det == 0.0) return false;
  D3 s = sub(o, a);
  u = dot(s, p) / det;
  if (!(u >= 0.0 && u <= 1.0)) return false;
  D3 q = cross(s, ab);
  v = dot(d, q) / det;
  if (v < 0.0 || u + v > 1.0) return false;
  t = dot(ac, q) / det;
  return true;
}

struct Cand { double t; uint32_t inst, ord; };
inline bool better(const Cand& c, const Hit64& b) {
  if (!b.hit) return true;
  if (c.t != b.t) return c.t < b.t;
  if (c.inst != b.inst) return c.inst < b.inst;
  return c.ord < b.prim;
}

// One instance's BVH4-Q8 walk in f64. `tri` gives (a, ab, ac, ident) for a leaf-relative triangle.
template <class LeafFn>
void blas64(const uint32_t* w, size_t nodes, uint32_t root, D3 o, D3 d, double tmin, double tmax,
            Hit64& best, bool rs_tags, LeafFn&& leaf) {
  std::vector<uint32_t> stack = {root};
  while (!stack.empty()) {
    uint32_t id = stack.back();
    stack.pop_back();
    if (id & LEAF_BIT) {
      leaf(id);
      continue;
    }
    size_t n = nodes + (size_t)id * 16;
    float org[3] = {bitsf(w[n]), bitsf(w[n + 1]), bitsf(w[n + 2])};
    float stp[3] = {bitsf(w[n + 3]), bitsf(w[n + 4]), bitsf(w[n + 5])};
    for (int s = 3; s >= 0; --s) {
      uint32_t c = w[n + 6 + s];
      if (c == EMPTY) continue;
      double lo[3], hi[3];
      for (int a = 0; a < 3; ++a) {
        uint8_t ql = (w[n + 10 + a] >> (8 * s)) & 255u, qh = (w[n + 13 + a] >> (8 * s)) & 255u;
        lo[a] = (double)(org[a] + stp[a] * (float)ql);  // cluster_bvh.rs:45 unfused decode
        hi[a] = (double)(org[a] + stp[a] * (float)qh);
        // Widened by 1e-9 relative: the f64 slab test then never culls a hit the f64 triangle
        // test accepts (a ray grazing a box face), so the walk equals a brute force.
        lo[a] -= 1e-9 * (std::fabs(lo[a]) + 1.0);
        hi[a] += 1e-9 * (std::fabs(hi[a]) + 1.0);
      }
      double lim = best.hit ? best.t : tmax;
      if (box_hit(o, d, tmin, lo, hi, lim)) stack.push_back(c);
    }
  }
  (void)rs_tags;
}

inline void rows64(const uint32_t* w, size_t r, const Ray& ray, D3& o, D3& d) {
  double m[12];
  for (int k = 0; k < 12; ++k) m[k] = (double)bitsf(w[r + k]);
  D3 wo = {ray.o[0], ray.o[1], ray.o[2]}, wd = {ray.d[0], ray.d[1], ray.d[2]};
  o = {m[0] * wo.x + m[1] * wo.y + m[2] * wo.z + m[3], m[4] * wo.x + m[5] * wo.y + m[6] * wo.z + m[7],
       m[8] * wo.x + m[9] * wo.y + m[10] * wo.z + m[11]};
  d = {m[0] * wd.x + m[1] * wd.y + m[2] * wd.z, m[4] * wd.x + m[5] * wd.y + m[6] * wd.z,
       m[8] * wd.x + m[9] * wd.y + m[10] * wd.z};
}

inline bool world_box(const uint32_t* w, size_t r, const Ray& ray, double tmin, double lim) {
  double lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = bitsf(w[r + 12 + a]), hi[a] = bitsf(w[r + 15 + a]);
    lo[a] -= 1e-9 * (std::fabs(lo[a]) + 1.0);
    hi[a] += 1e-9 * (std::fabs(hi[a]) + 1.0);
  }
  D3 o = {ray.o[0], ray.o[1], ray.o[2]}, d = {ray.d[0], ray.d[1], ray.d[2]};
  return box_hit(o, d, tmin, lo, hi, lim);
}

}  // namespace

Hit64 fp64_trace_rs(const uint32_t* w, const Ray& ray, bool any_hit) {
  Hit64 best{};
  best.hit = false;
  double tmin = ray.tmin, tmax = ray.tmax;
  for (uint32_t i = 0; i < w[0]; ++i) {
    size_t R = 8 + (size_t)i * 24;
    if (any_hit && w[R + 22] != 0) continue;
    if (!world_box(w, R, ray, tmin, best.hit ? best.t : tmax)) continue;
    D3 o, d;
    rows64(w, R, ray, o, d);
    size_t nodes = w[R + 18] & ~3u, tris = w[R + 19] & ~3u;
    uint32_t slot = w[R + 21];
    blas64(w, nodes, w[R + 20], o, d, tmin, tmax, best, true, [&](uint32_t id) {
      uint32_t start = (id & ~LEAF_BIT) >> 4, count = id & 15u;
      for (uint32_t k = 0; k < count; ++k) {
        size_t X = tris + (size_t)(start + k) * 12;
        D3 a = {bitsf(w[X]), bitsf(w[X + 1]), bitsf(w[X + 2])};
        D3 e1 = {bitsf(w[X + 3]), bitsf(w[X + 4]), bitsf(w[X + 5])};
        D3 e2 = {bitsf(w[X + 6]), bitsf(w[X + 7]), bitsf(w[X + 8])};
        double t, u, v;
        if (!mt64(o, d, a, e1, e2, t, u, v)) continue;
        if (!(t > tmin && t < tmax)) continue;
        uint32_t prim = w[X + 9];
        Cand c{t, i, prim};
        if (better(c, best)) {
          best.hit = true;
          best.t = t;
          best.inst = i;
          best.prim = prim;
          best.u = u;
          best.v = v;
          best.ident[0] = slot + 1;
          best.ident[1] = prim;
          best.ident[2] = best.ident[3] = 0;
        }
      }
    });
    (void)any_hit;
  }
  return best;
}

Hit64 fp64_trace_gi(const uint32_t* w, const Ray& ray, bool any_hit) {
  Hit64 best{};
  best.hit = false;
  double tmin = ray.tmin, tmax = ray.tmax;
  for (uint32_t i = 0; i < w[0]; ++i) {
    size_t r = 16 + (size_t)i * 32;
    if (any_hit && (w[r + 27] & 1u) != 0) continue;
    if (!world_box(w, r, ray, tmin, best.hit ? best.t : tmax)) continue;
    D3 o, d;
    rows64(w, r, ray, o, d);
    size_t nodes = w[r + 18], leaves = w[r + 19], positions = w[r + 20], indices = w[r + 21];
    uint32_t prim_base = w[r + 28];
    auto P = [&](uint32_t vi) {
      size_t at = positions + (size_t)vi * 3;
      return D3{bitsf(w[at]), bitsf(w[at + 1]), bitsf(w[at + 2])};
    };
    blas64(w, nodes, w[r + 22], o, d, tmin, tmax, best, false, [&](uint32_t id) {
      size_t l = leaves + (size_t)(id & ~LEAF_BIT) * 2;
      uint32_t first = w[l], count = w[l + 1];
      for (uint32_t k = 0; k < count; k += 3) {
        size_t x = indices + first + k;
        uint32_t ia = w[x], ib = w[x + 1], ic = w[x + 2];
        D3 a = P(ia), b = P(ib), c = P(ic);
        double t, u, v;
        if (!mt64(o, d, a, sub(b, a), sub(c, a), t, u, v)) continue;
        if (!(t > tmin && t < tmax)) continue;
        uint32_t ord = (first + k) / 3;
        Cand cd{t, i, ord};
        if (better(cd, best)) {
          best.hit = true;
          best.t = t;
          best.inst = i;
          best.prim = ord;
          best.u = u;
          best.v = v;
          best.ident[0] = i;
          if (!any_hit && prim_base != 0) {
            best.ident[1] = w[prim_base + ord];
            best.ident[2] = best.ident[3] = 0;
          } else {
            best.ident[1] = ia, best.ident[2] = ib, best.ident[3] = ic;
          }
        }
      }
    });
  }
  return best;
}

// reference.rs:160-194 over one Bvh in object space: `trace` walks the tree (children pushed
// 3 -> 0), `trace_brute` every leaf. inst = leaf id, prim = triangle within the leaf.
bool fp64_trace_bvh(const Bvh& b, const double o[3], const double d[3], double tmin, double tmax,
                    bool brute, Hit64& out) {
  out = Hit64{};
  out.hit = false;
  // Ray::valid (reference.rs:26-36)
  for (int a = 0; a < 3; ++a)
    if (!std::isfinite(o[a]) || !std::isfinite(d[a])) return false;
  if (d[0] == 0 && d[1] == 0 && d[2] == 0) return false;
  if (!std::isfinite(tmin) || std::isnan(tmax) || tmin < 0 || tmax < tmin) return false;
  D3 O = {o[0], o[1], o[2]}, Dd = {d[0], d[1], d[2]};
  auto leaf = [&](uint32_t li) {
    const Leaf& l = b.leaves[li];
    for (uint32_t tri = 0; tri < l.count / 3; ++tri) {
      D3 v[3];
      for (int k = 0; k < 3; ++k) {
        const auto& p = b.positions[b.indices[l.offset + tri * 3 + k]];
        v[k] = {p[0], p[1], p[2]};
      }
      double t, u, vv;
      if (!mt64(O, Dd, v[0], sub(v[1], v[0]), sub(v[2], v[0]), t, u, vv)) continue;
      bool ok = t >= tmin && t <= tmax &&
                (!out.hit || t < out.t || (t == out.t && (li < out.inst || (li == out.inst && tri < out.prim))));
      if (ok) {
        out.hit = true;
        out.t = t;
        out.inst = li;
        out.prim = tri;
        out.u = u;
        out.v = vv;
      }
    }
  };
  if (brute) {
    for (uint32_t li = 0; li < b.leaves.size(); ++li) leaf(li);
    return true;
  }
  std::vector<uint32_t> stack = {b.root};
  while (!stack.empty()) {
    uint32_t id = stack.back();
    stack.pop_back();
    if (id & LEAF_BIT) {
      leaf(id & ~LEAF_BIT);
      continue;
    }
    const Node& n = b.nodes[id];
    for (int slot = 3; slot >= 0; --slot) {
      if (n.children[slot] == EMPTY) continue;
      double lo[3], hi[3];
      for (int a = 0; a < 3; ++a) {
        lo[a] = decode_plane(n, a, n.lower[a][slot], false);
        hi[a] = decode_plane(n, a, n.upper[a][slot], false);
      }
      if (box_hit(O, Dd, tmin, lo, hi, out.hit ? out.t : tmax)) stack.push_back(n.children[slot]);
    }
  }
  return true;
}

}  // namespace orc
