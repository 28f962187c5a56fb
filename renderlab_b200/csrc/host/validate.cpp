// Admission check for a packed buffer. The traversal kernels index the words without bounds
// checks, so a buffer reaches the device only when every record a ray can reach lies inside it:
// every top-level and BLAS node, leaf, index, position, triangle and primitive word. Trees must
// be trees: BLAS children precede their parent (postorder, near_field.rs:286-306), top-level
// children follow it (preorder, instance_bvh.rs:370-401), and no node is reachable twice, so
// every traversal ends. The reference's own `Bvh::validate` (cluster_bvh.rs:170-333) checks the
// same ordering on its records.
#include <algorithm>
#include <map>
#include <tuple>
#include <vector>

#include "host.hpp"

namespace rtb {

namespace {

struct Fail {
  std::string what;
};

inline void need(bool ok, const char* what) {
  if (!ok) throw Fail{what};
}

// Walks one tree from `root` with an explicit stack. visit(node) returns its children; the
// ordering rule (child < parent for a BLAS, child > parent for a top level) makes the walk
// finite; `seen` rejects a node reachable twice.
// order: +1 children below their parent, -1 above it, 0 any order (reachable-once alone keeps
// the walk finite).
template <class Children>
uint32_t walk(uint32_t root, int order, size_t max_nodes, Children&& children) {
  std::vector<uint8_t> seen;
  std::vector<std::pair<uint32_t, uint32_t>> stack;  // (id, depth)
  stack.push_back({root, 0});
  uint32_t deepest = 0;
  while (!stack.empty()) {
    auto [id, depth] = stack.back();
    stack.pop_back();
    if (id & LEAF) {
      children(id, nullptr);
      continue;
    }
    need(id < max_nodes, "node index out of range");
    if (seen.size() <= id) seen.resize((size_t)id + 1, 0);
    need(!seen[id], "node reachable twice");
    seen[id] = 1;
    deepest = std::max(deepest, depth + 1);
    uint32_t kids[4];
    int n = children(id, kids);
    for (int k = 0; k < n; ++k) {
      uint32_t c = kids[k];
      if (c == EMPTY) continue;
      if (!(c & LEAF) && order != 0) need(order > 0 ? c < id : c > id, "tree children out of order");
      stack.push_back({c, depth + 1});
    }
  }
  return deepest;
}

void check_top(const uint32_t* w, size_t n, size_t base, uint32_t root, uint32_t count, SceneInfo& info) {
  need(base < n, "top level base out of range");
  size_t max_nodes = (n - base) / 32;
  info.max_top_depth = walk(root, -1, max_nodes, [&](uint32_t id, uint32_t* kids) -> int {
    if (id & LEAF) {
      need((id & ~LEAF) < count, "top level leaf names a missing instance");
      return 0;
    }
    const uint32_t* node = w + base + 32 * (size_t)id;
    for (int c = 0; c < 4; ++c) kids[c] = node[24 + c];
    return 4;
  });
}

}  // namespace

bool validate_scene(uint32_t layout, const uint32_t* w, size_t n, SceneInfo& info, std::string& err) {
  info = SceneInfo{};
  info.layout = layout;
  try {
    if (layout == 0) {
      need(n >= 16, "GI buffer shorter than its header");
      const uint32_t count = w[0];
      need(16 + 32 * (size_t)count <= n, "GI instance records past the buffer");
      info.instances = count;
      info.top = w[1];
      info.root = w[2];
      if (info.top != 0 && count > 0) check_top(w, n, info.top, info.root, count, info);
      std::map<std::array<uint32_t, 6>, bool> done;
      for (uint32_t i = 0; i < count; ++i) {
        const uint32_t* r = w + 16 + 32 * (size_t)i;
        for (int a = 0; a < 3; ++a) {
          info.world.lo[a] = lo_of(info.world.lo[a], as_float(r[12 + a]));
          info.world.hi[a] = hi_of(info.world.hi[a], as_float(r[15 + a]));
        }
        std::array<uint32_t, 6> key = {r[18], r[19], r[20], r[21], r[22], r[28]};
        if (done.count(key)) continue;
        done[key] = true;
        const size_t nodes = r[18], leaves = r[19], positions = r[20], indices = r[21], prim = r[28];
        need(nodes <= n, "GI node base out of range");
        size_t max_nodes = (n - nodes) / 16;
        uint32_t depth = walk(r[22], 1, max_nodes, [&](uint32_t id, uint32_t* kids) -> int {
          if (id & LEAF) {
            size_t l = leaves + 2 * (size_t)(id & ~LEAF);
            need(l + 2 <= n, "GI leaf record out of range");
            size_t first = w[l], cnt = w[l + 1];
            need(cnt > 0 && cnt % 3 == 0, "GI leaf count not a positive multiple of 3");
            need(indices + first + cnt <= n, "GI leaf indices out of range");
            for (size_t k = 0; k < cnt; ++k)
              need(positions + 3 * (size_t)w[indices + first + k] + 3 <= n, "GI position index out of range");
            if (prim != 0) need(prim + (first + cnt) / 3 <= n, "GI primitive table out of range");
            info.triangles += cnt / 3;
            return 0;
          }
          const uint32_t* node = w + nodes + 16 * (size_t)id;
          for (int c = 0; c < 4; ++c) kids[c] = node[6 + c];
          info.nodes += 1;
          return 4;
        });
        info.max_blas_depth = std::max(info.max_blas_depth, depth);
      }
    } else if (layout == 1) {
      need(n >= 8, "reflection buffer shorter than its header");
      const uint32_t count = w[0];
      need(8 + 24 * (size_t)count <= n, "reflection instance records past the buffer");
      info.instances = count;
      info.top = w[1];
      info.root = w[2];
      if (count > 0) need((size_t)(w[4] & ~3u) + 8 <= n, "scene bounds out of range");
      if (info.top != 0 && count > 0) check_top(w, n, info.top & ~3u, info.root, count, info);
      std::map<std::array<uint32_t, 6>, bool> done;
      for (uint32_t i = 0; i < count; ++i) {
        const uint32_t* r = w + 8 + 24 * (size_t)i;
        for (int a = 0; a < 3; ++a) {
          info.world.lo[a] = lo_of(info.world.lo[a], as_float(r[12 + a]));
          info.world.hi[a] = hi_of(info.world.hi[a], as_float(r[15 + a]));
        }
        std::array<uint32_t, 6> key = {r[18] & ~3u, r[19] & ~3u, r[20], 0, 0, 0};
        if (done.count(key)) continue;
        done[key] = true;
        const size_t nodes = r[18] & ~3u, tris = r[19] & ~3u;
        need(nodes <= n, "reflection node base out of range");
        size_t max_nodes = (n - nodes) / 16;
        uint32_t depth = walk(r[20], 1, max_nodes, [&](uint32_t id, uint32_t* kids) -> int {
          if (id & LEAF) {
            size_t start = (id & ~LEAF) >> 4, cnt = id & 15u;
            need(tris + 12 * (start + cnt) <= n, "reflection triangles out of range");
            info.triangles += cnt;
            return 0;
          }
          const uint32_t* node = w + nodes + 16 * (size_t)id;
          for (int c = 0; c < 4; ++c) kids[c] = node[6 + c];
          info.nodes += 1;
          return 4;
        });
        info.max_blas_depth = std::max(info.max_blas_depth, depth);
      }
    } else if (layout == 2) {
      // The legacy median BVH2 reflection layout (reflection_software.rs:170-264): 16-word nodes
      // with two boxes and children at words 12-13, leaves LEAF | first << 3 | count.
      need(n >= 8, "reflection buffer shorter than its header");
      const uint32_t count = w[0];
      need(8 + 24 * (size_t)count <= n, "reflection instance records past the buffer");
      info.instances = count;
      info.top = w[1];
      info.root = w[2];
      auto bvh2 = [&](size_t base, uint32_t root, bool top, size_t tris) -> uint32_t {
        need(base <= n, "BVH2 node base out of range");
        return walk(root, 0, (n - base) / 16, [&](uint32_t id, uint32_t* kids) -> int {
          if (id & LEAF) {
            if (top) {
              need((id & ~LEAF) < count, "top level leaf names a missing instance");
            } else {
              const size_t start = (id & ~LEAF) >> 3, cnt = id & 7u;
              need(tris + 12 * (start + cnt) <= n, "reflection triangles out of range");
              info.triangles += cnt;
            }
            return 0;
          }
          const uint32_t* node = w + base + 16 * (size_t)id;
          kids[0] = node[12], kids[1] = node[13], kids[2] = kids[3] = EMPTY;
          if (!top) info.nodes += 1;
          return 4;
        });
      };
      if (info.top != 0 && count > 0) info.max_top_depth = bvh2(info.top & ~3u, info.root, true, 0);
      std::map<std::array<uint32_t, 6>, bool> done;
      for (uint32_t i = 0; i < count; ++i) {
        const uint32_t* r = w + 8 + 24 * (size_t)i;
        for (int a = 0; a < 3; ++a) {
          info.world.lo[a] = lo_of(info.world.lo[a], as_float(r[12 + a]));
          info.world.hi[a] = hi_of(info.world.hi[a], as_float(r[15 + a]));
        }
        std::array<uint32_t, 6> key = {r[18] & ~3u, r[19] & ~3u, r[20], 0, 0, 0};
        if (done.count(key)) continue;
        done[key] = true;
        info.max_blas_depth = std::max(info.max_blas_depth, bvh2(r[18] & ~3u, r[20], false, r[19] & ~3u));
      }
    } else {
      need(false, "unknown layout");
    }
  } catch (const Fail& f) {
    err = f.what;
    return false;
  }
  return true;
}

}  // namespace rtb
