// CPU ORACLE — test infrastructure only. Nothing in the product links this code.
//
// A scalar C++17 restatement of renderlab's software-ray path (Ara-Engine/renderlab 0.1.3):
// the BVH4-Q8 builder and quantiser, the instance top level, the two packed-buffer layouts and
// the two WGSL traversal loops, plus the f64 reference traversal. Every function cites the
// reference line it restates. Built with -ffp-contract=off so every f32 multiply and add rounds
// on its own, as the WGSL source writes them; `std::fma` appears only where the reference calls
// `mul_add`.
//
// Parity pins: tests/golden holds vectors produced by the reference's own Python replay
// (tools/sunrt/replay_geometry.py) over dyadic scenes, plus the reference's known-answer tests
// restated in tests/. The glam 4x4 inverse (instance rows) is not restated: callers pass the
// world-to-object rows explicitly, so traversal parity does not depend on it.
#pragma once
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace orc {

constexpr uint32_t LEAF_BIT = 0x80000000u;  // crates/asset/src/cluster_bvh.rs:12
constexpr uint32_t EMPTY = 0xffffffffu;     // crates/asset/src/cluster_bvh.rs:13
constexpr size_t LEAF_TRIANGLES = 8;        // crates/asset/src/near_field.rs:23
constexpr size_t MAX_SAH_DEPTH = 15;        // crates/asset/src/near_field.rs:178
constexpr size_t SAH_BINS = 16;             // crates/asset/src/near_field.rs:273
constexpr float FLT_BIG = 3.4028235e38f;    // the WGSL miss distance

using V3 = std::array<float, 3>;
struct Box { V3 lo, hi; };

inline uint32_t fbits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float bitsf(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

// Rust f32::min / f32::max over non-NaN operands. For +0/-0 the reference's choice is
// unspecified (LLVM minnum); this restatement returns the first operand when they compare equal.
inline float rmin(float a, float b) { return b < a ? b : a; }
inline float rmax(float a, float b) { return b > a ? b : a; }

// Rust f32::total_cmp key: orders -0 < +0 and every finite value.
inline int32_t total_key(float f) {
  int32_t x; std::memcpy(&x, &f, 4);
  x ^= (int32_t)(((uint32_t)(x >> 31)) >> 1);
  return x;
}

// crates/asset/src/cluster_bvh.rs:21-30 (errors kept for the on-disk record; always 0 here).
struct Node {
  float origin[3];
  float step[3];
  uint32_t children[4];
  uint8_t lower[3][4];
  uint8_t upper[3][4];
  float errors[4];
};
// crates/asset/src/cluster_bvh.rs:60-68, the fields the builder fills.
struct Leaf { uint32_t offset, count, source_index_offset; };
struct Bvh {
  std::vector<Node> nodes;
  std::vector<Leaf> leaves;
  std::vector<std::array<float, 4>> positions;
  std::vector<uint32_t> indices;
  uint32_t root = EMPTY;
};

// ---- builder: crates/asset/src/near_field.rs:172-537 ----
bool build_bvh(const float* pos, size_t npos, const uint32_t* idx, size_t nidx, bool sah,
               Bvh& out, std::string& err);
bool build_bvh_sah(const float* pos, size_t npos, const uint32_t* idx, size_t nidx, Bvh& out,
                   std::string& err);
size_t bvh_depth(const Bvh& b, uint32_t child);
bool refit_bvh(Bvh& b, const float* pos, size_t npos, std::string& err);
Node quantized_node(const uint32_t* children, const Box* boxes, size_t n);
// Decode of slot `slot` on `axis` of the lower/upper plane: unfused o + s*q, or fused fma(s,q,o).
inline float decode_plane(const Node& n, int axis, uint8_t q, bool fused) {
  float s = n.step[axis], o = n.origin[axis], fq = (float)q;
  return fused ? std::fma(s, fq, o) : o + s * fq;
}
bool validate_bvh(const Bvh& b, std::string& err);

// ---- instance top level: src/instance_bvh.rs ----
constexpr uint32_t TOP_LEAF = 0x80000000u;
constexpr size_t TOP_NODE_WORDS = 16;  // BVH2
constexpr size_t TOP_WIDE_WORDS = 32;  // BVH4
constexpr size_t TOP_STACK = 48;
constexpr size_t MIN_INSTANCES = 40;
constexpr uint32_t REFITS = 64;
size_t tlas_reserve(size_t instances);
std::vector<uint32_t> tlas_build_with(const std::vector<Box>& boxes, bool sah, bool wide);
void tlas_refit(uint32_t* nodes, size_t n_words, const std::vector<Box>& boxes, bool wide);
// place(): synchronous form (RENDERLAB_INSTANCE_BVH_ASYNC=0). mode: -1 unset, 0 off, 1 on.
void tlas_place(std::vector<uint32_t>& words, size_t header, size_t stride, size_t slots,
                const std::vector<uint32_t>& previous, int mode, bool wide, bool sah);

// ---- packers: src/gi_bvh.rs and src/reflection_software.rs ----
struct GiMesh {
  Bvh bvh;
  V3 lo, hi;                      // bounds of every position (gi_bvh.rs:70)
  std::vector<uint32_t> primitives;
};
struct GiInstance {
  float model[12];  // object-to-world, 3 rows of 4 (row-major affine)
  float rows[12];   // world-to-object rows written to words 0-11
  uint32_t mesh;
  uint32_t near_base;
  uint32_t extra[8];  // words 24-31 (identity, map, map length, flags, prim base, placement)
};
std::vector<uint32_t> map_primitives(const std::vector<uint32_t>& bvh_indices,
                                     const uint32_t* src, size_t nsrc);
bool gi_pack(const std::vector<GiMesh>& meshes, const std::vector<GiInstance>& inst,
             int tlas_mode, std::vector<uint32_t>& words, std::string& err);

struct RsMesh {
  std::vector<uint32_t> nodes, triangles;
  uint32_t root;
  V3 lo, hi;
  bool wide;
};
bool rs_from_bvh(const float* pos, const uint32_t* idx, size_t nidx, const Bvh& bvh, RsMesh& out);
bool rs_build_median(const float* pos, const uint32_t* idx, size_t nidx, RsMesh& out);
struct RsInstance {
  float model[12];
  float rows[12];
  uint32_t mesh;
  uint32_t slot;
  bool casts;
};
bool rs_pack(const std::vector<RsMesh>& meshes, const std::vector<RsInstance>& inst, int tlas_mode,
             bool bvh4, std::vector<uint32_t>& words, std::string& err);

// ---- traversal: shaders/gi_rays_software.wgsl, shaders/reflections_software_bvh4.wgsl ----
struct Ray { float o[3]; float tmin; float d[3]; float tmax; };
enum Counter {
  C_TLAS_NODES, C_TLAS_BOX_TESTS, C_TLAS_INSTANCE_ENTRIES, C_INSTANCE_BOX_TESTS,
  C_INSTANCE_BOX_ENTRIES, C_BLAS_VISITS, C_BLAS_NODES, C_BLAS_BOX_TESTS, C_TRIANGLE_TESTS,
  C_LEAVES, C_STACK_DROPS, C_COUNT
};
struct GiHit { bool hit; float t; float normal[3]; uint32_t inst; uint32_t tri[3]; float bary[2]; };
struct RsHit { float t; uint32_t rec[4]; };
GiHit gi_traverse(const uint32_t* w, const Ray& r, uint32_t mode, bool top_wide, uint64_t* cnt);
RsHit rs_trace(const uint32_t* w, const Ray& r, bool any_hit, uint64_t* cnt);
RsHit rs_trace_bvh2(const uint32_t* w, const Ray& r, bool any_hit, uint64_t* cnt);

// ---- f64 reference: crates/asset/src/cluster_bvh/reference.rs ----
// ident: reflection (slot + 1, primitive, 0, 0); GI (instance, the three position indices, or
// the primitive id then 0, 0, as the f32 traversal reports them).
struct Hit64 { bool hit; double t; uint32_t inst; uint32_t prim; uint32_t ident[4]; double u, v; };
Hit64 fp64_trace_gi(const uint32_t* w, const Ray& r, bool any_hit);
Hit64 fp64_trace_rs(const uint32_t* w, const Ray& r, bool any_hit);
bool fp64_trace_bvh(const Bvh& b, const double o[3], const double d[3], double tmin, double tmax,
                    bool brute, Hit64& out);

}  // namespace orc
