// Host side of the engine: the CPU builders and packers that produce the packed words the
// traversal kernels read, and the validator that admits a buffer to the device.
#pragma once
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace rtb {

constexpr uint32_t LEAF = 0x80000000u;
constexpr uint32_t EMPTY = 0xffffffffu;
constexpr uint32_t LEAF_TRIANGLES = 8;  // near_field.rs:23
constexpr uint32_t MAX_SAH_DEPTH = 15;  // near_field.rs:178
constexpr uint32_t STACK_DEPTH = 48;    // gi_rays_software.wgsl:22, reflections_software_bvh4.wgsl:12

inline uint32_t as_bits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float as_float(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
// f32::min / f32::max over non-NaN operands (the first operand wins a tie).
inline float lo_of(float a, float b) { return b < a ? b : a; }
inline float hi_of(float a, float b) { return b > a ? b : a; }
inline int32_t order_key(float f) {  // f32::total_cmp
  int32_t x; std::memcpy(&x, &f, 4);
  return x ^ (int32_t)(((uint32_t)(x >> 31)) >> 1);
}

struct Aabb {
  float lo[3], hi[3];
  static Aabb empty() { return {{INFINITY, INFINITY, INFINITY}, {-INFINITY, -INFINITY, -INFINITY}}; }
  void grow(const float* p) {
    for (int a = 0; a < 3; ++a) lo[a] = lo_of(lo[a], p[a]), hi[a] = hi_of(hi[a], p[a]);
  }
  void grow(const Aabb& b) {
    for (int a = 0; a < 3; ++a) lo[a] = lo_of(lo[a], b.lo[a]), hi[a] = hi_of(hi[a], b.hi[a]);
  }
};

// A one-level BVH4 with 8-bit child boxes in its 16-word runtime form: origin[3], step[3],
// children[4], lower byte planes[3], upper byte planes[3] (gi_bvh.rs:191-203).
struct Blas {
  std::vector<uint32_t> nodes;    // 16 words a node, postorder (root last)
  std::vector<uint32_t> leaves;   // (index offset, index count) a leaf
  std::vector<float> positions;   // xyz a vertex (the input positions, unchanged)
  std::vector<uint32_t> indices;  // reordered triangle list
  std::vector<uint32_t> leaf_source;  // per leaf: 3 * its first triangle's index in the source list
  uint32_t root = EMPTY;
  Aabb bounds;                    // every position (gi_bvh.rs:70)
  size_t node_count() const { return nodes.size() / 16; }
  size_t leaf_count() const { return leaves.size() / 2; }
};

bool build_blas(const float* pos, size_t npos, const uint32_t* idx, size_t nidx, bool sah, Blas& out,
                std::string& err);
bool build_blas_sah(const float* pos, size_t npos, const uint32_t* idx, size_t nidx, Blas& out,
                    std::string& err);
size_t blas_depth(const Blas& b, uint32_t child);
bool refit_blas(Blas& b, const float* pos, size_t npos, std::string& err);
void quantize_node(const uint32_t* children, const Aabb* boxes, int n, uint32_t* w16);

// Instance top level (instance_bvh.rs)
size_t tlas_reserve(size_t instances);
std::vector<uint32_t> tlas_build(const std::vector<Aabb>& boxes, bool sah);
void tlas_refit(uint32_t* nodes, const std::vector<Aabb>& boxes);
void tlas_place(std::vector<uint32_t>& words, size_t header, size_t stride, size_t slots, int mode);

struct Placement {
  float model[12];
  float rows[12];
  uint32_t mesh, slot, casts_shadow, near_base;
  uint32_t extra[8];
};
// One cooked placement's near-field masks (gi_bvh.rs:38-43): the column-major transform they
// were cooked under and two sides of bins^2/32 words per BLAS position.
struct NearMasks {
  float transform[16];
  const uint32_t* masks;
  size_t n_masks;
};
struct MeshRef {
  const Blas* blas;
  const float* positions;  // source positions (reflection triangles are written from them)
  const uint32_t* indices; // source triangle list (primitive ids)
  size_t n_indices;
  bool primitives;         // GI: append the primitive table
  // GI: masks appended after every mesh's records (gi_bvh.rs:150-178); an instance of this mesh
  // whose model has exactly one entry's transform bits gets that entry's base in word 23.
  std::vector<NearMasks> near = {};
};
bool pack_gi(const std::vector<MeshRef>& meshes, const std::vector<Placement>& inst, int tlas_mode,
             std::vector<uint32_t>& out, std::string& err);
bool pack_reflection(const std::vector<MeshRef>& meshes, const std::vector<Placement>& inst,
                     int tlas_mode, std::vector<uint32_t>& out, std::string& err);
// Instances moved in packed words (pack.cpp): each record's rows and world box rewritten with
// the packer's arithmetic (mesh_boxes: the object box the packer used for each mesh), then the
// top level as instance_bvh::place treats a moved set: refit (word 3 counting refits) until
// TLAS_REFITS refits, then rebuilt; reflection scene bounds recomputed. Every instance must be
// non-singular and the count unchanged.
constexpr uint32_t TLAS_REFITS = 64;  // instance_bvh.rs:94
bool move_instances(uint32_t layout, uint32_t* words, size_t n_words, const std::vector<Placement>& inst,
                    const std::vector<Aabb>& mesh_boxes, std::string& err);
// A placement the packers skip or refuse: a zero determinant or a non-finite row (pack.cpp).
bool is_singular(const Placement& g);
// The world box (with the layout's margin) of a placement of an object box (pack.cpp), as the
// packers write instance words 12-17.
void instance_box(uint32_t layout, const float* model, const Aabb& obj, float lo[3], float hi[3]);

// Cooked files (cooked.cpp). RLB: crates/asset/src/cluster_bvh/codec.rs; RNF:
// crates/asset/src/near_field.rs:540-660. A BLAS is written as the near-field builder's cluster
// BVH (one zero-error level over every leaf); decoding one level gives a BLAS. max_bytes is the
// reference's Limits::max_bytes (160,000,000 by default, near_field.rs:86-92).
struct RnfSettings {
  float lod_error = 0.0f, reach = 0.0f, skip = 0.0f;
  uint32_t bins = 0;
};
struct RnfPlacement {
  uint32_t mesh = 0;
  float transform[16] = {};  // four columns of four
  std::vector<uint32_t> masks;
};
struct Rnf {
  RnfSettings settings;
  uint8_t source[32] = {};
  std::vector<Blas> meshes;
  std::vector<RnfPlacement> placements;
};
bool encode_rlb(const Blas& b, uint64_t max_bytes, std::vector<uint8_t>& out, std::string& err);
bool decode_rlb(const uint8_t* bytes, size_t n, uint64_t max_bytes, uint32_t level, Blas& out, std::string& err);
bool encode_rnf(const Rnf& f, uint64_t max_bytes, std::vector<uint8_t>& out, std::string& err);
bool decode_rnf(const uint8_t* bytes, size_t n, uint64_t max_bytes, Rnf& out, std::string& err);
// World::new (src/gi_cache.rs:1234-1268): every placement's cut moved to world space (winding
// reversed under a mirroring transform) and built as one SAH BLAS; bases[k] is placement k's
// first position in it.
bool rnf_world(const Rnf& f, Blas& out, std::vector<uint32_t>& bases, std::string& err);

// What a validated buffer holds, for the launchers and the derived layouts.
struct SceneInfo {
  uint32_t layout = 0;
  uint32_t instances = 0;
  uint32_t top = 0;           // top-level base word (0: flat list)
  uint32_t root = 0;
  size_t triangles = 0;       // distinct mesh triangles
  size_t nodes = 0;           // distinct BLAS nodes
  uint32_t max_blas_depth = 0;
  uint32_t max_top_depth = 0;
  Aabb world = Aabb::empty();  // union of the instance world boxes
};
bool validate_scene(uint32_t layout, const uint32_t* w, size_t n, SceneInfo& info, std::string& err);

}  // namespace rtb
