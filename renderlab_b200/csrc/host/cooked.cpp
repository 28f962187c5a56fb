// Cooked files, restated: the RLB cluster-BVH codec (crates/asset/src/cluster_bvh/codec.rs:4-188,
// its checks Bvh::validate, crates/asset/src/cluster_bvh.rs:170-333) and the RNF near-field
// codec (crates/asset/src/near_field.rs:540-660, NearField::validate :106-133). Explicit
// little-endian fields, never a struct image; the checks run in the reference's order and fail
// with its messages.
//
// A BLAS is written as the near-field builder writes its cluster BVH (near_field.rs:206-262,
// :380-400): the 80-byte nodes are the 16-word runtime nodes plus four zero child errors, each
// leaf is mesh 0, cluster = its index, page 0, its first triangle's source offset, its index
// span, error 0, material 0; one zero-error level over every leaf; positions with w = 0.
// Decoding one level of an RLB gives a BLAS whose root is that level's root (gi_bvh.rs:62-78).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "host.hpp"

namespace rtb {

namespace {

constexpr uint32_t RLB_VERSION = 1, RNF_VERSION = 1;
constexpr uint64_t NODE_BYTES = 80, LEAF_BYTES = 32, LEVEL_BYTES = 24;
constexpr size_t RNF_HEADER_BYTES = 64;

struct Fail {
  const char* what;
};
inline void need(bool ok, const char* what) {
  if (!ok) throw Fail{what};
}

void put32(std::vector<uint8_t>& o, uint32_t v) {
  for (int k = 0; k < 4; ++k) o.push_back((uint8_t)(v >> (8 * k)));
}
void put64(std::vector<uint8_t>& o, uint64_t v) {
  for (int k = 0; k < 8; ++k) o.push_back((uint8_t)(v >> (8 * k)));
}

struct Reader {
  const uint8_t* p;
  size_t n, at;
  const char* short_read;
  const uint8_t* take(uint64_t k) {
    need(k <= n - at, short_read);
    const uint8_t* r = p + at;
    at += (size_t)k;
    return r;
  }
  uint32_t u32() {
    const uint8_t* b = take(4);
    return (uint32_t)b[0] | (uint32_t)b[1] << 8 | (uint32_t)b[2] << 16 | (uint32_t)b[3] << 24;
  }
  uint64_t u64() {
    const uint64_t lo = u32(), hi = u32();
    return lo | hi << 32;
  }
};

// A cluster BVH as the file holds it: every level, error and leaf identity.
struct Rlb {
  std::vector<uint32_t> nodes;   // 16 runtime words a node
  std::vector<float> errors;     // 4 a node
  std::vector<uint32_t> leaves;  // 8 words: mesh, cluster, page, source offset, offset, count, error, material
  std::vector<uint32_t> levels;  // 6 words: mesh, root, requested error, max error, leaves offset, count
  std::vector<uint32_t> level_leaves;
  std::vector<float> positions;  // 4 a position
  std::vector<uint32_t> indices;
  size_t node_count() const { return nodes.size() / 16; }
  size_t leaf_count() const { return leaves.size() / 8; }
  size_t level_count() const { return levels.size() / 6; }
  size_t position_count() const { return positions.size() / 4; }
  uint64_t gpu_bytes() const {  // Bvh::gpu_bytes (cluster_bvh.rs:134-141)
    return node_count() * NODE_BYTES + leaf_count() * LEAF_BYTES + level_count() * LEVEL_BYTES +
           4 * (uint64_t)level_leaves.size() + 16 * (uint64_t)position_count() + 4 * (uint64_t)indices.size();
  }
};

// Span::range (virtual_mesh.rs:75-82): [offset, offset + count) within `length`.
void span(uint32_t offset, uint32_t count, size_t length, size_t& lo, size_t& hi) {
  need((uint64_t)offset + count <= UINT32_MAX, "virtual span overflow");
  need((size_t)offset + count <= length, "virtual span out of range");
  lo = offset, hi = (size_t)offset + count;
}

// Node::decode_bounds (cluster_bvh.rs:40-53): origin + step * q in f32, or fused, widened to f64.
double plane(const uint32_t* n, int a, uint32_t q, bool fused) {
  const float o = as_float(n[a]), s = as_float(n[3 + a]);
  return fused ? (double)std::fma(s, (float)q, o) : (double)(o + s * (float)q);
}
uint32_t lane(uint32_t word, int s) { return (word >> (8 * s)) & 255u; }

// Bvh::validate (cluster_bvh.rs:170-333).
void validate(const Rlb& b, uint64_t max_bytes) {
  const size_t nn = b.node_count(), nl = b.leaf_count(), nt = b.level_count(), np = b.position_count();
  need(b.gpu_bytes() <= max_bytes && nn < LEAF && nl < LEAF - 1 && nt > 0,
       "cluster BVH byte/count limit or empty levels");
  for (size_t v = 0; v < np; ++v) {
    bool ok = b.positions[4 * v + 3] == 0.0f;
    for (int a = 0; a < 4; ++a) ok = ok && std::isfinite(b.positions[4 * v + a]);
    need(ok, "invalid cluster BVH position");
  }
  for (uint32_t i : b.indices) need(i < np, "cluster BVH vertex index");
  size_t end = 0;
  for (size_t l = 0; l < nl; ++l) {
    const uint32_t* L = &b.leaves[8 * l];
    size_t lo, hi;
    span(L[4], L[5], b.indices.size(), lo, hi);
    const float err = as_float(L[6]);
    need(lo == end && hi > lo && (hi - lo) % 3 == 0 && std::isfinite(err) && err >= 0.0f, "invalid cluster BVH leaf");
    end = hi;
  }
  need(end == b.indices.size(), "unowned cluster BVH indices");
  struct Box {
    double lo[3], hi[3];
    float error;
  };
  std::vector<Box> boxes(nn);
  for (size_t i = 0; i < nn; ++i) {
    const uint32_t* n = &b.nodes[16 * i];
    bool frame = n[6] != EMPTY || n[7] != EMPTY || n[8] != EMPTY || n[9] != EMPTY;
    for (int a = 0; a < 3; ++a)
      frame = frame && std::isfinite(as_float(n[a])) && std::isfinite(as_float(n[3 + a])) && as_float(n[3 + a]) > 0.0f;
    need(frame, "invalid cluster BVH node frame");
    Box box{{INFINITY, INFINITY, INFINITY}, {-INFINITY, -INFINITY, -INFINITY}, 0.0f};
    for (int s = 0; s < 4; ++s) {
      const uint32_t c = n[6 + s];
      const float e = b.errors[4 * i + s];
      if (c == EMPTY) {
        bool zero = e == 0.0f;
        for (int a = 0; a < 3; ++a) zero = zero && lane(n[10 + a], s) == 0 && lane(n[13 + a], s) == 0;
        need(zero, "noncanonical empty BVH child");
        continue;
      }
      double clo[3], chi[3];
      float ce;
      if (c & LEAF) {
        const size_t l = c & ~LEAF;
        need(l < nl, "BVH leaf reference");
        for (int a = 0; a < 3; ++a) clo[a] = INFINITY, chi[a] = -INFINITY;
        for (uint32_t k = b.leaves[8 * l + 4]; k < b.leaves[8 * l + 4] + b.leaves[8 * l + 5]; ++k)
          for (int a = 0; a < 3; ++a) {
            const double v = b.positions[4 * (size_t)b.indices[k] + a];
            clo[a] = std::min(clo[a], v), chi[a] = std::max(chi[a], v);
          }
        ce = as_float(b.leaves[8 * l + 6]);
      } else {
        need(c < i, "BVH unordered/cyclic node");
        for (int a = 0; a < 3; ++a) clo[a] = boxes[c].lo[a], chi[a] = boxes[c].hi[a];
        ce = boxes[c].error;
      }
      bool ok = std::isfinite(e) && e == ce;
      double lo[3], hi[3], flo[3], fhi[3];
      for (int a = 0; a < 3; ++a) {
        lo[a] = plane(n, a, lane(n[10 + a], s), false), hi[a] = plane(n, a, lane(n[13 + a], s), false);
        flo[a] = plane(n, a, lane(n[10 + a], s), true), fhi[a] = plane(n, a, lane(n[13 + a], s), true);
        ok = ok && std::isfinite(lo[a]) && std::isfinite(hi[a]) && std::isfinite(flo[a]) && std::isfinite(fhi[a]) &&
             lo[a] <= clo[a] && hi[a] >= chi[a] && flo[a] <= clo[a] && fhi[a] >= chi[a];
      }
      need(ok, "BVH child bounds/error do not enclose geometry");
      for (int a = 0; a < 3; ++a) {
        box.lo[a] = std::min(std::min(box.lo[a], lo[a]), flo[a]);
        box.hi[a] = std::max(std::max(box.hi[a], hi[a]), fhi[a]);
      }
      box.error = std::max(box.error, ce);
    }
    boxes[i] = box;
  }
  std::vector<uint8_t> used_nodes(nn, 0), used_leaves(nl, 0);
  size_t cut_end = 0;
  bool have_previous = false;
  uint32_t prev_mesh = 0;
  float prev_error = 0.0f;
  for (size_t t = 0; t < nt; ++t) {
    const uint32_t* V = &b.levels[6 * t];
    const float req = as_float(V[2]), mx = as_float(V[3]);
    need(std::isfinite(req) && req >= 0.0f && std::isfinite(mx) && mx >= 0.0f && mx <= req &&
             !(have_previous && (V[0] < prev_mesh || (V[0] == prev_mesh && req <= prev_error))),
         "invalid BVH level/error order");
    have_previous = true, prev_mesh = V[0], prev_error = req;
    size_t lo, hi;
    span(V[4], V[5], b.level_leaves.size(), lo, hi);
    need(lo == cut_end && hi > lo, "invalid BVH cut span");
    cut_end = hi;
    for (size_t k = lo + 1; k < hi; ++k) need(b.level_leaves[k - 1] < b.level_leaves[k], "BVH duplicate/unordered cut leaf");
    std::vector<uint32_t> found, stack{V[1]};
    size_t visits = 0;
    float error = 0.0f;
    while (!stack.empty()) {
      const uint32_t c = stack.back();
      stack.pop_back();
      need(++visits <= nn + nl, "BVH repeated subtree");
      need(c != EMPTY, "BVH empty root");
      if (c & LEAF) {
        const uint32_t id = c & ~LEAF;
        need(id < nl, "BVH cut leaf reference");
        need(b.leaves[8 * (size_t)id] == V[0], "BVH cross-mesh cut");
        used_leaves[id] = 1;
        error = std::max(error, as_float(b.leaves[8 * (size_t)id + 6]));
        found.push_back(id);
      } else {
        need(c < nn, "BVH root reference");
        used_nodes[c] = 1;
        for (int s = 0; s < 4; ++s)
          if (b.nodes[16 * (size_t)c + 6 + s] != EMPTY) stack.push_back(b.nodes[16 * (size_t)c + 6 + s]);
      }
    }
    std::sort(found.begin(), found.end());
    need(std::equal(found.begin(), found.end(), b.level_leaves.begin() + lo, b.level_leaves.begin() + hi) &&
             error == mx,
         "BVH cut/root disagreement");
  }
  bool all_used = cut_end == b.level_leaves.size();
  for (uint8_t u : used_nodes) all_used = all_used && u;
  for (uint8_t u : used_leaves) all_used = all_used && u;
  need(all_used, "unreachable cluster BVH records");
}

Rlb from_blas(const Blas& b) {
  Rlb r;
  r.nodes = b.nodes;
  r.errors.assign(4 * b.node_count(), 0.0f);
  const size_t nl = b.leaf_count();
  need(b.leaf_source.size() == nl, "BLAS has no source offsets for its leaves");
  for (size_t l = 0; l < nl; ++l) {
    const uint32_t rec[8] = {0, (uint32_t)l, 0, b.leaf_source[l], b.leaves[2 * l], b.leaves[2 * l + 1], as_bits(0.0f), 0};
    r.leaves.insert(r.leaves.end(), rec, rec + 8);
    r.level_leaves.push_back((uint32_t)l);
  }
  const uint32_t level[6] = {0, b.root, as_bits(0.0f), as_bits(0.0f), 0, (uint32_t)nl};
  r.levels.assign(level, level + 6);
  for (size_t v = 0; v < b.positions.size() / 3; ++v) {
    for (int a = 0; a < 3; ++a) r.positions.push_back(b.positions[3 * v + a]);
    r.positions.push_back(0.0f);
  }
  r.indices = b.indices;
  return r;
}

// cluster_bvh::encode (codec.rs:4-76).
std::vector<uint8_t> encode(const Rlb& r, uint64_t max_bytes) {
  validate(r, max_bytes);
  std::vector<uint8_t> out;
  out.reserve(32 + r.gpu_bytes());
  for (char c : {'R', 'L', 'B', '\0'}) out.push_back((uint8_t)c);
  put32(out, RLB_VERSION);
  for (size_t n : {r.node_count(), r.leaf_count(), r.level_count(), r.level_leaves.size(), r.position_count(),
                   r.indices.size()}) {
    need(n <= UINT32_MAX, "BVH encoded count overflow");
    put32(out, (uint32_t)n);
  }
  for (size_t i = 0; i < r.node_count(); ++i) {
    for (int k = 0; k < 16; ++k) put32(out, r.nodes[16 * i + k]);  // origin, step, children, lower, upper
    for (int s = 0; s < 4; ++s) put32(out, as_bits(r.errors[4 * i + s]));
  }
  for (uint32_t v : r.leaves) put32(out, v);
  for (uint32_t v : r.levels) put32(out, v);
  for (uint32_t v : r.level_leaves) put32(out, v);
  for (float v : r.positions) put32(out, as_bits(v));
  for (uint32_t v : r.indices) put32(out, v);
  need(out.size() <= max_bytes, "BVH encoded byte limit");
  return out;
}

// cluster_bvh::decode (codec.rs:108-188).
Rlb decode(const uint8_t* bytes, size_t n, uint64_t max_bytes) {
  need(n <= max_bytes, "BVH file byte limit");
  Reader rd{bytes, n, 0, "truncated cluster BVH"};
  const uint8_t* magic = rd.take(4);
  need(std::memcmp(magic, "RLB\0", 4) == 0 && rd.u32() == RLB_VERSION, "unknown cluster BVH schema");
  uint64_t counts[6], length = 32;
  const uint64_t stride[6] = {NODE_BYTES, LEAF_BYTES, LEVEL_BYTES, 4, 16, 4};
  for (int k = 0; k < 6; ++k) {
    counts[k] = rd.u32();
    length += counts[k] * stride[k];  // at most 6 * 80 * 2^32: no overflow in 64 bits
  }
  need(length == n && length <= max_bytes, "BVH extent/count limit");
  Rlb r;
  r.nodes.resize(16 * counts[0]);
  r.errors.resize(4 * counts[0]);
  for (size_t i = 0; i < counts[0]; ++i) {
    for (int k = 0; k < 16; ++k) r.nodes[16 * i + k] = rd.u32();
    for (int s = 0; s < 4; ++s) r.errors[4 * i + s] = as_float(rd.u32());
  }
  auto words = [&](std::vector<uint32_t>& v, size_t m) {
    v.resize(m);
    for (auto& x : v) x = rd.u32();
  };
  words(r.leaves, 8 * counts[1]);
  words(r.levels, 6 * counts[2]);
  words(r.level_leaves, counts[3]);
  r.positions.resize(4 * counts[4]);
  for (auto& x : r.positions) x = as_float(rd.u32());
  words(r.indices, counts[5]);
  validate(r, max_bytes);
  return r;
}

// Blas::new (gi_bvh.rs:62-78): the level's root over the whole record arrays.
Blas to_blas(const Rlb& r, uint32_t level) {
  need(level < r.level_count(), "indirect geometry level");
  Blas b;
  b.nodes = r.nodes;
  for (size_t l = 0; l < r.leaf_count(); ++l) {
    b.leaves.push_back(r.leaves[8 * l + 4]);
    b.leaves.push_back(r.leaves[8 * l + 5]);
    b.leaf_source.push_back(r.leaves[8 * l + 3]);
  }
  b.bounds = Aabb::empty();
  for (size_t v = 0; v < r.position_count(); ++v) {
    for (int a = 0; a < 3; ++a) b.positions.push_back(r.positions[4 * v + a]);
    b.bounds.grow(&r.positions[4 * v]);
  }
  b.indices = r.indices;
  b.root = r.levels[6 * (size_t)level + 1];
  return b;
}

// Settings::validate (near_field.rs:39-52).
void validate_settings(const RnfSettings& s) {
  need(std::isfinite(s.lod_error) && s.lod_error >= 0.0f && std::isfinite(s.reach) && s.reach > 0.0f &&
           std::isfinite(s.skip) && s.skip >= 0.0f && s.skip < s.reach &&
           (s.bins == 0 || s.bins == 8 || s.bins == 16 || s.bins == 32),
       "invalid near-field settings");
}

// NearField::validate (near_field.rs:106-133) over the meshes' records as cluster BVHs.
void validate_field(const RnfSettings& s, const std::vector<Rlb>& meshes, const std::vector<RnfPlacement>& placements,
                    uint64_t max_bytes) {
  validate_settings(s);
  uint64_t bytes = 0;
  for (const Rlb& m : meshes) bytes += m.gpu_bytes();
  for (const RnfPlacement& p : placements) bytes += 4 * (uint64_t)p.masks.size();
  need(bytes <= max_bytes && !meshes.empty(), "near field byte limit or no meshes");
  for (const Rlb& m : meshes) {
    validate(m, max_bytes);
    need(m.level_count() == 1, "near-field mesh must have one level");
  }
  const size_t words = (size_t)s.bins * s.bins / 32;
  for (const RnfPlacement& p : placements) {
    need(p.mesh < meshes.size(), "near-field placement mesh");
    bool finite = true;
    for (float v : p.transform) finite = finite && std::isfinite(v);
    need(p.masks.size() == meshes[p.mesh].position_count() * 2 * words && finite,
         "near-field placement masks or transform");
  }
}

}  // namespace

bool encode_rlb(const Blas& b, uint64_t max_bytes, std::vector<uint8_t>& out, std::string& err) {
  try {
    out = encode(from_blas(b), max_bytes);
  } catch (const Fail& f) {
    err = f.what;
    return false;
  }
  return true;
}

bool decode_rlb(const uint8_t* bytes, size_t n, uint64_t max_bytes, uint32_t level, Blas& out, std::string& err) {
  try {
    out = to_blas(decode(bytes, n, max_bytes), level);
  } catch (const Fail& f) {
    err = f.what;
    return false;
  }
  return true;
}

// near_field::encode (near_field.rs:546-584).
bool encode_rnf(const Rnf& f, uint64_t max_bytes, std::vector<uint8_t>& out, std::string& err) {
  try {
    std::vector<Rlb> meshes;
    for (const Blas& b : f.meshes) meshes.push_back(from_blas(b));
    validate_field(f.settings, meshes, f.placements, max_bytes);
    need(meshes.size() <= UINT32_MAX, "near-field mesh count");
    need(f.placements.size() <= UINT32_MAX, "near-field placement count");
    out.clear();
    for (char c : {'R', 'N', 'F', '\0'}) out.push_back((uint8_t)c);
    for (uint32_t v : {RNF_VERSION, (uint32_t)meshes.size(), (uint32_t)f.placements.size(), f.settings.bins,
                       as_bits(f.settings.lod_error), as_bits(f.settings.reach), as_bits(f.settings.skip)})
      put32(out, v);
    out.insert(out.end(), f.source, f.source + 32);
    for (const Rlb& m : meshes) {
      const std::vector<uint8_t> blob = encode(m, max_bytes);
      put64(out, blob.size());
      out.insert(out.end(), blob.begin(), blob.end());
    }
    for (const RnfPlacement& p : f.placements) {
      put32(out, p.mesh);
      for (float v : p.transform) put32(out, as_bits(v));
      put64(out, p.masks.size());
      for (uint32_t m : p.masks) put32(out, m);
    }
    const size_t slack = RNF_HEADER_BYTES + 4096;
    need(out.size() <= slack || out.size() - slack <= max_bytes, "near-field encoded size");
  } catch (const Fail& e) {
    err = e.what;
    return false;
  }
  return true;
}

// near_field::decode (near_field.rs:586-660).
bool decode_rnf(const uint8_t* bytes, size_t n, uint64_t max_bytes, Rnf& out, std::string& err) {
  try {
    need(n >= RNF_HEADER_BYTES && std::memcmp(bytes, "RNF\0", 4) == 0 && (n <= (1u << 24) || n - (1u << 24) <= max_bytes),
         "near-field header or size");
    Reader rd{bytes, n, 4, "near-field truncated"};
    need(rd.u32() == RNF_VERSION, "unsupported near-field version");
    const size_t n_meshes = rd.u32(), n_placements = rd.u32();
    RnfSettings s;
    s.bins = rd.u32();
    s.lod_error = as_float(rd.u32());
    s.reach = as_float(rd.u32());
    s.skip = as_float(rd.u32());
    validate_settings(s);
    uint8_t source[32];
    std::memcpy(source, rd.take(32), 32);
    need(n_meshes <= n / 8 && n_placements <= n / 76, "near-field counts exceed the file");
    std::vector<Rlb> meshes;
    for (size_t m = 0; m < n_meshes; ++m) {
      const uint64_t len = rd.u64();
      const uint8_t* blob = rd.take(len);
      meshes.push_back(decode(blob, (size_t)len, max_bytes));
    }
    std::vector<RnfPlacement> placements(n_placements);
    for (RnfPlacement& p : placements) {
      p.mesh = rd.u32();
      for (float& v : p.transform) v = as_float(rd.u32());
      const uint64_t words = rd.u64();
      need(words <= UINT64_MAX / 4, "near-field mask length");
      const uint8_t* raw = rd.take(4 * words);
      p.masks.resize((size_t)words);
      for (size_t k = 0; k < p.masks.size(); ++k)
        p.masks[k] = (uint32_t)raw[4 * k] | (uint32_t)raw[4 * k + 1] << 8 | (uint32_t)raw[4 * k + 2] << 16 |
                     (uint32_t)raw[4 * k + 3] << 24;
    }
    need(rd.at == n, "near-field trailing bytes");
    validate_field(s, meshes, placements, max_bytes);
    out = Rnf{};
    out.settings = s;
    std::memcpy(out.source, source, 32);
    for (const Rlb& m : meshes) out.meshes.push_back(to_blas(m, 0));
    out.placements = std::move(placements);
  } catch (const Fail& e) {
    err = e.what;
    return false;
  }
  return true;
}

bool rnf_world(const Rnf& f, Blas& out, std::vector<uint32_t>& bases, std::string& err) {
  std::vector<float> positions;
  std::vector<uint32_t> indices;
  bases.clear();
  for (const RnfPlacement& p : f.placements) {
    if (p.mesh >= f.meshes.size()) {
      err = "near-field placement mesh";
      return false;
    }
    const Blas& m = f.meshes[p.mesh];
    const float* t = p.transform;
    const size_t base = positions.size() / 3;
    if (base + m.positions.size() / 3 > UINT32_MAX) {
      err = "near-field world exceeds 2^32 positions";
      return false;
    }
    bases.push_back((uint32_t)base);
    // glam Mat4::transform_point3: x * c0 + y * c1 + z * c2 + c3, rounded in turn.
    for (size_t v = 0; v < m.positions.size() / 3; ++v) {
      const float* q = &m.positions[3 * v];
      for (int r = 0; r < 3; ++r) {
        float acc = t[r] * q[0];
        acc = t[4 + r] * q[1] + acc;
        acc = t[8 + r] * q[2] + acc;
        positions.push_back(t[12 + r] + acc);
      }
    }
    // The sign of Mat4::determinant, taken in double (a mirroring transform is far from 0).
    double d[16];
    for (int k = 0; k < 16; ++k) d[k] = t[k];
    auto minor = [&](int c0, int c1, int c2, int r0, int r1, int r2) {
      auto e = [&](int c, int r) { return d[4 * c + r]; };
      return e(c0, r0) * (e(c1, r1) * e(c2, r2) - e(c2, r1) * e(c1, r2)) -
             e(c1, r0) * (e(c0, r1) * e(c2, r2) - e(c2, r1) * e(c0, r2)) +
             e(c2, r0) * (e(c0, r1) * e(c1, r2) - e(c1, r1) * e(c0, r2));
    };
    const double det = d[3] * -minor(1, 2, 3, 0, 1, 2) + d[7] * minor(0, 2, 3, 0, 1, 2) -
                       d[11] * minor(0, 1, 3, 0, 1, 2) + d[15] * minor(0, 1, 2, 0, 1, 2);
    const bool flip = det < 0.0;
    for (size_t k = 0; k + 2 < m.indices.size(); k += 3) {
      const uint32_t a = m.indices[k], b = m.indices[k + 1], c = m.indices[k + 2];
      indices.push_back((uint32_t)base + a);
      indices.push_back((uint32_t)base + (flip ? c : b));
      indices.push_back((uint32_t)base + (flip ? b : c));
    }
  }
  return build_blas_sah(positions.data(), positions.size() / 3, indices.data(), indices.size(), out, err);
}

}  // namespace rtb
