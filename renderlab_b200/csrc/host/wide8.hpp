// The engine's compressed 8-wide BLAS (the WIDE8 kernel's layout), derived from an uploaded
// scene's packed words.
//
// Node, 80 bytes (20 words, five 16-byte loads):
//   0-2   p: float origin of the child boxes
//   3     exponent bytes ex | ey << 8 | ez << 16 (scale 2^(e-127), e - 127 <= 13), inner-child mask << 24
//   4     index of the first inner child node (inner children are contiguous, in slot order)
//   5     index of the first triangle (leaf children's triangles are contiguous, in slot order)
//   6-7   meta byte per slot: leaf (count << 5 | offset), 0 for an inner or empty slot; an empty
//         slot's box is inverted (lower planes 255, upper 0), so no ray meets it
//   8-19  child boxes: lo x, lo y, lo z, hi x, hi y, hi z, one byte per slot (two words each)
// A child box is the real interval [p + q_lo * 2^e, p + q_hi * 2^e] per axis; the builder
// rounds q outward in exact arithmetic, so it encloses the child's triangles exactly.
// Slots are assigned by octant: slot bit a set means the child lies toward +a, so a ray with
// direction-sign bits o meets slot k ^ o roughly k-th (Ylitie, Karras, Laine 2017, "Efficient
// Incoherent Ray Traversal on GPUs Through Compressed Wide BVHs").
//
// Triangle, 48 bytes (12 words): v0 xyz, v1 xyz, v2 xyz (f32, as the watertight test reads
// them), ident (reflection: primitive id; GI: triangle ordinal in the mesh's index array), ref
// (the word offset of the source triangle in the packed buffer: reflection a/e1/e2, GI its three
// indices), 0.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace rtb {

constexpr uint32_t W8_NODE_WORDS = 20;
constexpr uint32_t W8_TRI_WORDS = 12;
// Triangles a leaf may hold. One: measured on 1M-triangle cluster soup against three, it tests
// 15 % fewer triangles a ray for 1 % more nodes, and traces GI rays 9 % faster.
#ifndef RT_W8_MAX_LEAF
#define RT_W8_MAX_LEAF 1
#endif
constexpr uint32_t W8_MAX_LEAF = RT_W8_MAX_LEAF;
// Largest node scale exponent: the kernel multiplies 2^(e+15) by 1/d, which reaches 1e30, so
// e <= 13 keeps the product finite (a BLAS at most 255 * 2^13 = 2,088,960 units wide).
constexpr int W8_MAX_EXPONENT = 13;

struct Wide8Blas {
  std::vector<uint32_t> nodes;  // root is node 0
  std::vector<uint32_t> tris;
  int max_exponent = -126;      // the largest scale exponent of its nodes
  uint32_t depth = 0;           // levels of 8-wide nodes (a walk stacks at most depth - 1 groups)
};

// The whole derived scene: per distinct BLAS of the packed words, its nodes and triangles, and
// per instance the (node base, triangle base) of its BLAS in the concatenated arrays.
struct Wide8Scene {
  std::vector<uint32_t> nodes;
  std::vector<uint32_t> tris;
  std::vector<uint32_t> inst;  // 2 words per instance: node base, triangle base
  size_t blas_count = 0;
  uint32_t depth = 0;  // the deepest BLAS's levels
  // the 8-wide top level (empty: the scene is a flat instance list, or keeps its BVH4 top level)
  // and its leaves' entries, two words each: instance, node of the instance's BLAS to enter at
  // (relative to the BLAS's root)
  std::vector<uint32_t> top_nodes, top_items;
  uint32_t top_depth = 0;
};

// An 8-wide top level in the BLAS node format: a leaf slot's `count` items (one: W8_MAX_LEAF) are
// at items[node word 5 + offset]; node 0 is the root and nodes are numbered breadth first, so the
// upper levels are the lowest node indices.
struct Wide8Top {
  std::vector<uint32_t> nodes;
  std::vector<uint32_t> items;
  int max_exponent = -126;
  uint32_t depth = 0;
};

// Source triangle for the builder: f32 vertices plus identity words.
struct SrcTri {
  float v[9];
  uint32_t ident, ref;
};

// `threads`: about how many threads the build may use (large subtrees are built concurrently;
// the tree does not depend on it).
void build_wide8(const std::vector<SrcTri>& tris, Wide8Blas& out, int threads = 1);
struct Aabb;
void build_wide8_top(const std::vector<Aabb>& boxes, Wide8Top& out, int threads = 1);
// Entries of the WIDE8 walk's top-level stack (pairs of words): a level's group, plus one node's
// eight leaves.
constexpr uint32_t W8_TOP_STACK = 32;
// The re-braided top level's size: at most this many leaves per instance, and in all (at least one
// per instance), and the relative margin of its world boxes.
#ifndef RT_W8_BRAID
#define RT_W8_BRAID 256
#endif
constexpr uint32_t W8_BRAID_PER_INSTANCE = RT_W8_BRAID;
constexpr size_t W8_BRAID_MAX = size_t(1) << 22;
constexpr double W8_BRAID_PAD = 1.0 / 65536.0;
// The 8-wide top level of a packed scene with a top level, over its built 8-wide BLAS nodes and
// instance table (Wide8Scene::nodes, ::inst). Its leaves are entries (instance, BLAS node): each
// instance starts as one entry at its BLAS root, and the entry with the largest world box is
// replaced by its node's children -- nodes whose children are all inner nodes only, so an
// instance's entries always cover each of its triangles exactly once -- until there are
// `per_instance` entries per instance (Benthin, Woop, Wald and Afra 2017, partial re-braiding).
// An entry's world box bounds its node's box under the instance's object-to-world map (the
// inverse of the record's rows, in double), with a margin for the walk's f32 object-space ray.
// Instances without a usable record world box are left out (the reference's top level never
// enters them); one whose rows cannot be inverted is one entry under its record world box.
// False (nothing built) for a flat instance list, or when the entries span more than the node
// scale allows or the tree is too deep for the walk's stack: the walk then uses the packed BVH4
// top level.
bool build_wide8_top_of(uint32_t layout, const uint32_t* words, const std::vector<uint32_t>& blas_nodes,
                        const std::vector<uint32_t>& inst, std::vector<uint32_t>& nodes, std::vector<uint32_t>& items,
                        uint32_t* depth = nullptr, uint32_t per_instance = W8_BRAID_PER_INSTANCE);
// An instance's object-to-world map (3 rows of 4): the inverse of its record's world-to-object rows
// (12 f32 words), in double; false when they cannot be inverted.
bool instance_model(const uint32_t* rows, double* m);
// The box of a BLAS node's subtree: the union of its children's boxes, exact; false when it has none.
bool entry_object_box(const uint32_t* node, double* lo, double* hi);
// The box of the eight corners of the object box [olo, ohi] under the affine map m (3 rows of 4).
void entry_world_box(const double* m, const double* olo, const double* ohi, double* lo, double* hi);
// `per_instance`: the top level's entries per instance (build_wide8_top_of).
bool build_wide8_scene(uint32_t layout, const uint32_t* words, size_t n_words, Wide8Scene& out, std::string& err,
                       int threads, uint32_t per_instance = W8_BRAID_PER_INSTANCE);
// Checks a built layout (wide8_check.cpp): ranges, one leaf per triangle, every child box
// enclosing its child in exact arithmetic, inverted empty slots, the recorded depth. info: nodes,
// triangles, depth, distinct BLAS.
bool check_wide8_scene(const Wide8Scene& s, uint32_t info[4], std::string& err);
// Checks the 8-wide top level of a scene built from `words`: each instance with a usable world
// box and a non-empty BLAS has entries that cut its BLAS exactly (every triangle under exactly one
// entry), every leaf box encloses its entry's node box under the instance's object-to-world map
// (or the record world box, for rows that cannot be inverted), every inner child box the boxes
// below it, nodes after their parents, the recorded depth within the walk's stack.
bool check_wide8_top(uint32_t layout, const uint32_t* words, const Wide8Scene& s, std::string& err);

}  // namespace rtb
