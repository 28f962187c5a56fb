// CPU ORACLE — test infrastructure only: the C entry points tests/ (and bench.py's CPU-baseline
// leg) reach through ctypes. Every compute call here runs the scalar restatement in this folder.
#include <algorithm>
#include <atomic>
#include <thread>

#include "oracle.hpp"

using namespace orc;

namespace {

void set_err(char* err, int len, const std::string& s) {
  if (err && len > 0) {
    std::snprintf(err, (size_t)len, "%s", s.c_str());
  }
}

// Runs fn(i) for i in [0, n) on `threads` workers pulling chunks of 256.
template <class F>
void parallel_for(uint32_t n, int threads, F&& fn) {
  if (threads <= 1 || n < 1024) {
    for (uint32_t i = 0; i < n; ++i) fn(i);
    return;
  }
  std::atomic<uint32_t> next{0};
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([&] {
      for (;;) {
        uint32_t s = next.fetch_add(256);
        if (s >= n) break;
        uint32_t e = std::min(n, s + 256);
        for (uint32_t i = s; i < e; ++i) fn(i);
      }
    });
  for (auto& th : pool) th.join();
}

struct Words { std::vector<uint32_t> w; };

void node16(const Node& nd, uint32_t* w) {
  for (int a = 0; a < 3; ++a) w[a] = fbits(nd.origin[a]);
  for (int a = 0; a < 3; ++a) w[3 + a] = fbits(nd.step[a]);
  for (int s = 0; s < 4; ++s) w[6 + s] = nd.children[s];
  for (int a = 0; a < 3; ++a)
    w[10 + a] = nd.lower[a][0] | nd.lower[a][1] << 8 | nd.lower[a][2] << 16 | (uint32_t)nd.lower[a][3] << 24;
  for (int a = 0; a < 3; ++a)
    w[13 + a] = nd.upper[a][0] | nd.upper[a][1] << 8 | nd.upper[a][2] << 16 | (uint32_t)nd.upper[a][3] << 24;
}

Ray ray_at(const float* rays, uint32_t i) {
  Ray r;
  std::memcpy(&r, rays + 8 * (size_t)i, sizeof r);
  return r;
}

}  // namespace

extern "C" {

// ---- BLAS ----
// mode 0: build_bvh (median), 1: build_bvh_sah (with its depth fallback), 2: SAH only.
void* orc_bvh_build(const float* pos, uint32_t npos, const uint32_t* idx, uint32_t nidx, int mode,
                    char* err, int errlen) {
  Bvh* b = new Bvh;
  std::string e;
  bool ok = mode == 1 ? build_bvh_sah(pos, npos, idx, nidx, *b, e) : build_bvh(pos, npos, idx, nidx, mode == 2, *b, e);
  if (!ok) {
    set_err(err, errlen, e);
    delete b;
    return nullptr;
  }
  return b;
}
void orc_bvh_free(void* h) { delete (Bvh*)h; }
// info: nodes, leaves, positions, indices, root, depth
void orc_bvh_info(void* h, uint32_t* info) {
  const Bvh& b = *(Bvh*)h;
  info[0] = (uint32_t)b.nodes.size();
  info[1] = (uint32_t)b.leaves.size();
  info[2] = (uint32_t)b.positions.size();
  info[3] = (uint32_t)b.indices.size();
  info[4] = b.root;
  info[5] = (uint32_t)bvh_depth(b, b.root);
}
// 16-word runtime records (gi_bvh.rs:191-203)
void orc_bvh_nodes(void* h, uint32_t* out) {
  const Bvh& b = *(Bvh*)h;
  for (size_t i = 0; i < b.nodes.size(); ++i) node16(b.nodes[i], out + 16 * i);
}
void orc_bvh_leaves(void* h, uint32_t* out) {
  const Bvh& b = *(Bvh*)h;
  for (size_t i = 0; i < b.leaves.size(); ++i)
    out[3 * i] = b.leaves[i].offset, out[3 * i + 1] = b.leaves[i].count, out[3 * i + 2] = b.leaves[i].source_index_offset;
}
void orc_bvh_indices(void* h, uint32_t* out) {
  const Bvh& b = *(Bvh*)h;
  std::copy(b.indices.begin(), b.indices.end(), out);
}
int orc_bvh_refit(void* h, const float* pos, uint32_t npos, char* err, int errlen) {
  std::string e;
  if (!refit_bvh(*(Bvh*)h, pos, npos, e)) {
    set_err(err, errlen, e);
    return 0;
  }
  return 1;
}
int orc_bvh_validate(void* h, char* err, int errlen) {
  std::string e;
  if (!validate_bvh(*(Bvh*)h, e)) {
    set_err(err, errlen, e);
    return 0;
  }
  return 1;
}
// rays: 8 doubles (o3, tmin, d3, tmax); out: 6 doubles (hit, t, leaf, triangle, u, v)
int orc_bvh_trace64(void* h, const double* rays, uint32_t n, int brute, double* out) {
  const Bvh& b = *(Bvh*)h;
  for (uint32_t i = 0; i < n; ++i) {
    const double* r = rays + 8 * (size_t)i;
    Hit64 hit;
    bool valid = fp64_trace_bvh(b, r, r + 4, r[3], r[7], brute != 0, hit);
    double* o = out + 6 * (size_t)i;
    o[0] = valid && hit.hit ? 1.0 : 0.0;
    o[1] = hit.t, o[2] = hit.inst, o[3] = hit.prim, o[4] = hit.u, o[5] = hit.v;
  }
  return 1;
}
// children (n <= 4), boxes 6 floats each (lo xyz, hi xyz) -> 16-word runtime node
void orc_quantized_node(const uint32_t* children, const float* boxes, uint32_t n, uint32_t* out16) {
  std::vector<Box> bs(n);
  for (uint32_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) bs[i].lo[a] = boxes[6 * i + a], bs[i].hi[a] = boxes[6 * i + 3 + a];
  node16(quantized_node(children, bs.data(), n), out16);
}

// ---- TLAS ----
uint32_t orc_tlas_reserve(uint32_t n) { return (uint32_t)tlas_reserve(n); }
uint32_t orc_tlas_build(const float* boxes, uint32_t n, int sah, int wide, uint32_t* out, uint32_t cap) {
  std::vector<Box> bs(n);
  for (uint32_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) bs[i].lo[a] = boxes[6 * i + a], bs[i].hi[a] = boxes[6 * i + 3 + a];
  std::vector<uint32_t> nodes = tlas_build_with(bs, sah != 0, wide != 0);
  if (nodes.size() <= cap) std::copy(nodes.begin(), nodes.end(), out);
  return (uint32_t)nodes.size();
}
void orc_tlas_refit(uint32_t* nodes, uint32_t nwords, const float* boxes, uint32_t n, int wide) {
  std::vector<Box> bs(n);
  for (uint32_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) bs[i].lo[a] = boxes[6 * i + a], bs[i].hi[a] = boxes[6 * i + 3 + a];
  tlas_refit(nodes, nwords, bs, wide != 0);
}
// words: the records (length nwords); out must hold cap words. Returns the new length.
uint32_t orc_tlas_place(const uint32_t* words, uint32_t nwords, uint32_t header, uint32_t stride,
                        uint32_t slots, const uint32_t* prev, uint32_t nprev, int mode, int wide,
                        uint32_t* out, uint32_t cap) {
  std::vector<uint32_t> w(words, words + nwords), p(prev, prev + nprev);
  tlas_place(w, header, stride, slots, p, mode, wide != 0, true);
  if (w.size() <= cap) std::copy(w.begin(), w.end(), out);
  return (uint32_t)w.size();
}

// ---- scenes ----
// Meshes: pos_off[m..m+1] vertex range, idx_off[m..m+1] index range into pos / idx.
// mesh_flags bit 0: GI primitive table (gi_bvh.rs:82-87).
// Instances: models / rows 12 floats each (3 rows of 4), mesh ids, aux:
//   GI: 9 words (near base, extra words 24-31);  reflection: 2 words (slot, casts shadows).
// kind 0: GI; 1: reflection BVH4; 2: reflection legacy BVH2 (median).
void* orc_scene(int kind, uint32_t n_meshes, const float* pos, const uint32_t* pos_off,
                const uint32_t* idx, const uint32_t* idx_off, const uint32_t* mesh_flags,
                uint32_t n_inst, const float* models, const float* rows, const uint32_t* mesh,
                const uint32_t* aux, int tlas_mode, char* err, int errlen) {
  Words* out = new Words;
  std::string e;
  bool ok = true;
  if (kind == 0) {
    std::vector<GiMesh> meshes(n_meshes);
    for (uint32_t m = 0; m < n_meshes && ok; ++m) {
      const float* p = pos + 3 * (size_t)pos_off[m];
      uint32_t np = pos_off[m + 1] - pos_off[m];
      const uint32_t* ix = idx + idx_off[m];
      uint32_t ni = idx_off[m + 1] - idx_off[m];
      ok = build_bvh_sah(p, np, ix, ni, meshes[m].bvh, e);
      if (!ok) break;
      Box bb{{INFINITY, INFINITY, INFINITY}, {-INFINITY, -INFINITY, -INFINITY}};
      for (uint32_t v = 0; v < np; ++v)
        for (int a = 0; a < 3; ++a) bb.lo[a] = rmin(bb.lo[a], p[3 * v + a]), bb.hi[a] = rmax(bb.hi[a], p[3 * v + a]);
      meshes[m].lo = bb.lo;
      meshes[m].hi = bb.hi;
      if (mesh_flags && (mesh_flags[m] & 1)) meshes[m].primitives = map_primitives(meshes[m].bvh.indices, ix, ni);
    }
    std::vector<GiInstance> inst(n_inst);
    for (uint32_t i = 0; i < n_inst; ++i) {
      std::memcpy(inst[i].model, models + 12 * (size_t)i, 48);
      std::memcpy(inst[i].rows, rows + 12 * (size_t)i, 48);
      inst[i].mesh = mesh[i];
      inst[i].near_base = aux[9 * (size_t)i];
      for (int k = 0; k < 8; ++k) inst[i].extra[k] = aux[9 * (size_t)i + 1 + k];
    }
    if (ok) ok = gi_pack(meshes, inst, tlas_mode, out->w, e);
  } else {
    std::vector<RsMesh> meshes(n_meshes);
    for (uint32_t m = 0; m < n_meshes && ok; ++m) {
      const float* p = pos + 3 * (size_t)pos_off[m];
      uint32_t np = pos_off[m + 1] - pos_off[m];
      const uint32_t* ix = idx + idx_off[m];
      uint32_t ni = idx_off[m + 1] - idx_off[m];
      if (kind == 2) {
        ok = rs_build_median(p, ix, ni, meshes[m]);
        if (!ok) e = "legacy BVH2 build";
      } else {
        Bvh b;
        ok = build_bvh_sah(p, np, ix, ni, b, e) && rs_from_bvh(p, ix, ni, b, meshes[m]);
        if (!ok && e.empty()) e = "reflection primitive mapping";
      }
    }
    std::vector<RsInstance> inst(n_inst);
    for (uint32_t i = 0; i < n_inst; ++i) {
      std::memcpy(inst[i].model, models + 12 * (size_t)i, 48);
      std::memcpy(inst[i].rows, rows + 12 * (size_t)i, 48);
      inst[i].mesh = mesh[i];
      inst[i].slot = aux[2 * (size_t)i];
      inst[i].casts = aux[2 * (size_t)i + 1] != 0;
    }
    if (ok) ok = rs_pack(meshes, inst, tlas_mode, kind == 1, out->w, e);
  }
  if (!ok) {
    set_err(err, errlen, e);
    delete out;
    return nullptr;
  }
  return out;
}
uint64_t orc_words_len(void* h) { return ((Words*)h)->w.size(); }
void orc_words_copy(void* h, uint32_t* out) {
  auto& w = ((Words*)h)->w;
  std::copy(w.begin(), w.end(), out);
}
void orc_words_free(void* h) { delete (Words*)h; }

// ---- traversal ----
// rays: 8 floats (o3, tmin, d3, tmax). GI hits: 10 words (t, inst, tri3, u, v, normal3);
// reflection hits: 5 words (t, record4). counters: C_COUNT sums (may be null).
int orc_gi_trace(const uint32_t* w, const float* rays, uint32_t n, uint32_t mode, int top_wide,
                 uint32_t* hits, uint64_t* counters, int threads) {
  std::vector<uint64_t> cnt((size_t)std::max(threads, 1) * C_COUNT, 0);
  std::atomic<int> slot{0};
  thread_local int my = -1;
  (void)my;
  auto run = [&](uint32_t i, uint64_t* c) {
    GiHit h = gi_traverse(w, ray_at(rays, i), mode, top_wide != 0, c);
    uint32_t* o = hits + 10 * (size_t)i;
    o[0] = fbits(h.t), o[1] = h.inst, o[2] = h.tri[0], o[3] = h.tri[1], o[4] = h.tri[2];
    o[5] = fbits(h.bary[0]), o[6] = fbits(h.bary[1]);
    o[7] = fbits(h.normal[0]), o[8] = fbits(h.normal[1]), o[9] = fbits(h.normal[2]);
  };
  if (!counters) {
    parallel_for(n, threads, [&](uint32_t i) { run(i, nullptr); });
    return 1;
  }
  // Counters: per-ray locals summed under a lock-free add.
  std::vector<std::atomic<uint64_t>> total(C_COUNT);
  for (auto& t : total) t = 0;
  parallel_for(n, threads, [&](uint32_t i) {
    uint64_t c[C_COUNT] = {};
    run(i, c);
    for (int k = 0; k < C_COUNT; ++k)
      if (c[k]) total[k].fetch_add(c[k], std::memory_order_relaxed);
  });
  for (int k = 0; k < C_COUNT; ++k) counters[k] = total[k];
  (void)slot;
  return 1;
}
int orc_rs_trace(const uint32_t* w, const float* rays, uint32_t n, int any_hit, int bvh2,
                 uint32_t* hits, uint64_t* counters, int threads) {
  auto run = [&](uint32_t i, uint64_t* c) {
    RsHit h = bvh2 ? rs_trace_bvh2(w, ray_at(rays, i), any_hit != 0, c) : rs_trace(w, ray_at(rays, i), any_hit != 0, c);
    uint32_t* o = hits + 5 * (size_t)i;
    o[0] = fbits(h.t);
    for (int k = 0; k < 4; ++k) o[1 + k] = h.rec[k];
  };
  if (!counters) {
    parallel_for(n, threads, [&](uint32_t i) { run(i, nullptr); });
    return 1;
  }
  std::vector<std::atomic<uint64_t>> total(C_COUNT);
  for (auto& t : total) t = 0;
  parallel_for(n, threads, [&](uint32_t i) {
    uint64_t c[C_COUNT] = {};
    run(i, c);
    for (int k = 0; k < C_COUNT; ++k)
      if (c[k]) total[k].fetch_add(c[k], std::memory_order_relaxed);
  });
  for (int k = 0; k < C_COUNT; ++k) counters[k] = total[k];
  return 1;
}
// Per-ray counters (C_COUNT each), for tests that compare ray by ray.
int orc_rs_trace_counts(const uint32_t* w, const float* rays, uint32_t n, int any_hit, int bvh2,
                        uint32_t* hits, uint64_t* per_ray) {
  for (uint32_t i = 0; i < n; ++i) {
    uint64_t* c = per_ray + (size_t)C_COUNT * i;
    std::fill(c, c + C_COUNT, 0);
    RsHit h = bvh2 ? rs_trace_bvh2(w, ray_at(rays, i), any_hit != 0, c) : rs_trace(w, ray_at(rays, i), any_hit != 0, c);
    uint32_t* o = hits + 5 * (size_t)i;
    o[0] = fbits(h.t);
    for (int k = 0; k < 4; ++k) o[1 + k] = h.rec[k];
  }
  return 1;
}
// layout 0: GI, 1: reflection. out: 4 doubles (hit, t, u, v); ident: 6 words (inst, prim, ident4)
int orc_fp64_trace(const uint32_t* w, int layout, const float* rays, uint32_t n, int any_hit,
                   double* out, uint32_t* ident, int threads) {
  parallel_for(n, threads, [&](uint32_t i) {
    Ray r = ray_at(rays, i);
    Hit64 h = layout == 0 ? fp64_trace_gi(w, r, any_hit != 0) : fp64_trace_rs(w, r, any_hit != 0);
    double* o = out + 4 * (size_t)i;
    o[0] = h.hit ? 1.0 : 0.0, o[1] = h.t, o[2] = h.u, o[3] = h.v;
    uint32_t* d = ident + 6 * (size_t)i;
    d[0] = h.inst, d[1] = h.prim;
    for (int k = 0; k < 4; ++k) d[2 + k] = h.ident[k];
  });
  return 1;
}
int orc_counter_count() { return C_COUNT; }

}  // extern "C"
