// WIDE8 traversal: the precision variant over the compressed 8-wide BLAS of host/wide8.hpp.
//
// * Top level and instance records: the packed words, walked as the reference does.
// * BLAS: 80-byte nodes; a ray's direction-sign octant o orders the children (slot k ^ o is
//   visited k-th); inner hits form a node group (first child, pending bits, inner mask) that is
//   pushed whole, so the stack holds one entry per level.
// * Child boxes: t = fma(1 + q 2^-15, 2^(e+15) / d, (p - o) / d - 2^(e+15) / d) per plane (one
//   byte permute and one fma), widened by a per-node bound on its rounding error so that no box a
//   ray meets is ever culled (the boxes themselves enclose their triangles exactly).
// * Triangles: the watertight test of Woop, Benthin and Wald (2013) through a per-instance
//   shear matrix; an edge function that rounds to zero is recomputed in double. Shared vertices
//   transform identically, so a ray never slips between two triangles.
// * FP64: candidates whose f32 result is uncertain -- within 8e-6 relative of the current best
//   (a near tie), of tmin or tmax, or within the f32 edge functions' error bound of an edge -- are
//   re-intersected with the f64 Möller-Trumbore test over the source triangle in the packed
//   words, in the exact arithmetic of the f64 reference (crates/asset/src/cluster_bvh/reference.rs:121-158), and ties resolve
//   on (t, instance, triangle) as it does.
// * Final values: a closest-hit walk records only the winner (t estimate, instance, 8-wide
//   triangle); k_wide8_final then recomputes t, u, v of every hit in f64 over the source triangle
//   (the same arithmetic), and the GI record's primitive words and normal, one thread per ray.
//   f32 barycentrics of a ray whose origin lies hundreds of units from a sub-unit triangle carry
//   errors near 1e-5 from the rounding of the coordinates alone; f64 leaves only the final
//   rounding to f32. The pass is fully converged and coalesced, so it costs far less than the
//   same work done by single lanes inside the divergent walk.
#pragma once
#include "plain.cuh"

namespace rtk {

constexpr float W8_U = 5.9604645e-8f;  // 2^-24
constexpr float W8_TIE = 8e-6f;
constexpr float W8_EDGE = 1e-5f;
constexpr uint32_t W8_STACK = 32;
// Entries of the shared-memory group stack (a scene whose 8-wide trees are at most this many
// levels deep stacks at most W8_SSTACK - 1 groups).
constexpr uint32_t W8_SSTACK = 16;
// Resident 128-thread blocks per SM the register allocation is sized for: the per-ray walk
// (RT_W8_MIN_BLOCKS: 7, 72 registers) and the packet walk (RT_W8P_MIN_BLOCKS: 7, 72 registers).
// The f64 resolution of uncertain candidates is out of line, so the per-ray loop fits its budget
// with a few bytes of spills (the packet walk with about 150). Measured on clusters-1M and
// clusters-4M rays against 4 to 8 blocks, with neither walk holding shared memory: 7 is the
// fastest for both.
#ifndef RT_W8_MIN_BLOCKS
#define RT_W8_MIN_BLOCKS 7
#endif
#ifndef RT_W8P_MIN_BLOCKS
#define RT_W8P_MIN_BLOCKS 7
#endif

// Opt-in device counters of the WIDE8 walk (diagnostics and the bytes-per-ray roofline).
enum W8Count { W8C_RAYS, W8C_TOP_NODES, W8C_INSTANCE_TESTS, W8C_NODES, W8C_LEAVES, W8C_TRIS, W8C_RETESTS, W8C_FINAL64, W8C_N };
template <bool COUNT>
RT_DEV void w8_count(unsigned long long* cnt, int k, unsigned long long n = 1) {
  if (COUNT) atomicAdd(cnt + k, n);
}

struct W8View {
  const uint4* nodes;     // 5 uint4 a node
  const uint4* tris;      // 3 uint4 a triangle
  const uint32_t* inst;   // 2 words an instance: node base, triangle base
  // the 8-wide top level (null: walk the packed BVH4 top level), breadth first from its root, and
  // its leaves' entries, two words each: instance, node of the instance's BLAS to enter at
  // (relative to the BLAS's root)
  const uint4* top = nullptr;
  const uint32_t* top_items = nullptr;
  uint32_t top_count = 0;
};

// Top-level nodes staged in shared memory by every block of the per-ray walk over a scene with a
// top level (the first levels, which every ray reads): 16 nodes, 1.25 KB. Measured on the
// 10,000-instance batching scene: 0, 16, 64, 128 and 256 nodes give 16.9, 17.3, 16.6, 16.3 and
// 16.0 Mrays/s (more shared memory leaves L1 less room).
#ifndef RT_W8_TOP_CACHE
#define RT_W8_TOP_CACHE 16
#endif
constexpr uint32_t W8_TOP_CACHE = RT_W8_TOP_CACHE;
// Pairs of words in the per-ray walk's 8-wide top-level stack: a group entry (first child node,
// pending bits | inner mask << 8) a level, and one node's leaf entries (instance, BLAS node |
// W8_ENTRY).
constexpr uint32_t W8_TOP_STACK = 32;
constexpr uint32_t W8_ENTRY = 0x80000000u;

struct W8Best {
  float t;          // f32 t of the best candidate (f32(t64) once re-tested)
  float band;       // bound on |t - t64| while !has64
  double t64;       // valid when has64
  bool has64;
  bool hit;
  uint32_t inst;    // instance index
  uint32_t tri;     // 8-wide triangle index
  uint32_t ident;   // primitive id (reflection) or triangle ordinal (GI)
};

// f64 reference arithmetic, never contracted (reference.rs:47-59).
struct D3 {
  double x, y, z;
};
RT_DEV D3 dsub3(D3 a, D3 b) { return {__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y), __dsub_rn(a.z, b.z)}; }
RT_DEV double ddot(D3 a, D3 b) { return __dadd_rn(__dadd_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)), __dmul_rn(a.z, b.z)); }
RT_DEV D3 dcross(D3 a, D3 b) {
  return {__dsub_rn(__dmul_rn(a.y, b.z), __dmul_rn(a.z, b.y)), __dsub_rn(__dmul_rn(a.z, b.x), __dmul_rn(a.x, b.z)),
          __dsub_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x))};
}

// The ray in object space in f64, from the instance's f32 rows (the f64 reference's TLAS
// wrapper: left-to-right sums of f64 products).
template <uint32_t LAYOUT>
RT_DEV void ray64(const uint32_t* __restrict__ w, uint32_t inst, const Ray& ray, D3& o, D3& d) {
  const size_t r = LAYOUT == 0 ? 16 + (size_t)inst * 32 : 8 + (size_t)inst * 24;
  double m[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) m[k] = (double)ldf(w, r + k);
  const D3 wo = {ray.o.x, ray.o.y, ray.o.z}, wd = {ray.d.x, ray.d.y, ray.d.z};
  o = {__dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(m[0], wo.x), __dmul_rn(m[1], wo.y)), __dmul_rn(m[2], wo.z)), m[3]),
       __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(m[4], wo.x), __dmul_rn(m[5], wo.y)), __dmul_rn(m[6], wo.z)), m[7]),
       __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(m[8], wo.x), __dmul_rn(m[9], wo.y)), __dmul_rn(m[10], wo.z)), m[11])};
  d = {__dadd_rn(__dadd_rn(__dmul_rn(m[0], wd.x), __dmul_rn(m[1], wd.y)), __dmul_rn(m[2], wd.z)),
       __dadd_rn(__dadd_rn(__dmul_rn(m[4], wd.x), __dmul_rn(m[5], wd.y)), __dmul_rn(m[6], wd.z)),
       __dadd_rn(__dadd_rn(__dmul_rn(m[8], wd.x), __dmul_rn(m[9], wd.y)), __dmul_rn(m[10], wd.z))};
}

// f64 Möller-Trumbore over the source triangle at word `ref` (reference.rs:121-158). The
// reflection layout's triangle is a, a + e1, a + e2 with e1/e2 as stored; the GI layout's is
// three indexed positions. Accepts t in (tmin, tmax).
template <uint32_t LAYOUT>
__device__ __noinline__ bool mt64(const uint32_t* __restrict__ w, uint32_t inst, uint32_t ref, const Ray& ray, double& t, double& u,
                 double& v) {
  D3 o, d;
  ray64<LAYOUT>(w, inst, ray, o, d);
  D3 a, ab, ac;
  if (LAYOUT == 1) {
    a = {ldf(w, ref), ldf(w, ref + 1), ldf(w, ref + 2)};
    ab = {ldf(w, ref + 3), ldf(w, ref + 4), ldf(w, ref + 5)};
    ac = {ldf(w, ref + 6), ldf(w, ref + 7), ldf(w, ref + 8)};
  } else {
    const size_t positions = ld(w, 16 + (size_t)inst * 32 + 20);
    const uint32_t ia = ld(w, ref), ib = ld(w, ref + 1), ic = ld(w, ref + 2);
    a = {ldf(w, positions + 3 * (size_t)ia), ldf(w, positions + 3 * (size_t)ia + 1), ldf(w, positions + 3 * (size_t)ia + 2)};
    const D3 b = {ldf(w, positions + 3 * (size_t)ib), ldf(w, positions + 3 * (size_t)ib + 1), ldf(w, positions + 3 * (size_t)ib + 2)};
    const D3 c = {ldf(w, positions + 3 * (size_t)ic), ldf(w, positions + 3 * (size_t)ic + 1), ldf(w, positions + 3 * (size_t)ic + 2)};
    ab = dsub3(b, a);
    ac = dsub3(c, a);
  }
  const D3 p = dcross(d, ac);
  const double det = ddot(ab, p);
  if (det == 0.0) return false;
  const D3 s = dsub3(o, a);
  u = __ddiv_rn(ddot(s, p), det);
  if (!(u >= 0.0 && u <= 1.0)) return false;
  const D3 q = dcross(s, ab);
  v = __ddiv_rn(ddot(d, q), det);
  if (v < 0.0 || __dadd_rn(u, v) > 1.0) return false;
  t = __ddiv_rn(ddot(ac, q), det);
  return t > (double)ray.tmin && t < (double)ray.tmax;
}

// Per-instance object-space ray state for the 8-wide walk. The walk's part (o, d, inv, oct) is
// set when the instance is entered; the triangle test's part (the shear, oerr, tscale) when the
// instance's first leaf triangle is tested (w8_shear): in scenes of many overlapping instances
// most entered instances end at their root node's boxes, and never need it.
struct W8Ray {
  F3 o, d, inv;
  uint32_t oct;
  // watertight shear rows: (Ax, Ay, Az) = M (v - o)
  F3 mx, my, mz;
  float oerr;   // |o - o64|_inf: the f32 object-space origin against the f64 reference's
  float tscale; // 8 u |1 / d_kz|: absolute error of t per unit of |v - o|
  bool valid;
  bool sheared; // the triangle test's part is set
};

// The walk's part: reciprocal direction, octant, and whether the direction is usable at all.
RT_DEV void w8_setup(W8Ray& R) {
  R.inv = safe_inverse(R.d);
  R.oct = (R.d.x < 0.0f ? 1u : 0u) | (R.d.y < 0.0f ? 2u : 0u) | (R.d.z < 0.0f ? 4u : 0u);
  R.valid = R.d.x != 0.0f || R.d.y != 0.0f || R.d.z != 0.0f;
  R.sheared = false;
}

// The triangle test's part for instance `inst` of the packed words (record rows at `r`): the
// shear of Woop, Benthin and Wald (2013) for the object-space direction, and the error of the
// f32 object-space origin against the f64 reference's (ray64's arithmetic over the same rows).
__device__ __forceinline__ void w8_shear(const uint32_t* __restrict__ w, size_t r, const F3& world_o, W8Ray& R) {
  const float ax = fabsf(R.d.x), ay = fabsf(R.d.y), az = fabsf(R.d.z);
  const int kz = (ax >= ay && ax >= az) ? 0 : (ay >= az ? 1 : 2);
  int kx = kz == 2 ? 0 : kz + 1, ky = kx == 2 ? 0 : kx + 1;
  auto comp = [&](int k) { return k == 0 ? R.d.x : (k == 1 ? R.d.y : R.d.z); };
  const float dz = comp(kz);
  if (dz < 0.0f) {
    const int t = kx;
    kx = ky;
    ky = t;
  }
  const float sz = __frcp_rn(dz);  // dz != 0: the instance was entered with a valid direction
  const float sx = __fmul_rn(comp(kx), sz), sy = __fmul_rn(comp(ky), sz);
  // rows of the shear: M_x = e_kx - sx e_kz, M_y = e_ky - sy e_kz, M_z = sz e_kz
  auto row = [&](int one, float at_z) {
    return F3{one == 0 ? 1.0f : (kz == 0 ? at_z : 0.0f), one == 1 ? 1.0f : (kz == 1 ? at_z : 0.0f),
              one == 2 ? 1.0f : (kz == 2 ? at_z : 0.0f)};
  };
  R.mx = row(kx, -sx);
  R.my = row(ky, -sy);
  R.mz = {kz == 0 ? sz : 0.0f, kz == 1 ? sz : 0.0f, kz == 2 ? sz : 0.0f};
  R.tscale = 8.0f * W8_U * fabsf(sz);
  // the origin of the f64 reference (ray64's arithmetic), to bound the f32 origin's error
  const double ox = world_o.x, oy = world_o.y, oz = world_o.z;
  auto o64 = [&](size_t k) {
    return __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn((double)ldf(w, k), ox), __dmul_rn((double)ldf(w, k + 1), oy)),
                               __dmul_rn((double)ldf(w, k + 2), oz)),
                     (double)ldf(w, k + 3));
  };
  const double e = fmax(fmax(fabs(o64(r) - (double)R.o.x), fabs(o64(r + 4) - (double)R.o.y)),
                        fabs(o64(r + 8) - (double)R.o.z));
  R.oerr = e > 0.0 ? __double2float_ru(e) : 0.0f;
  R.sheared = true;
}
// The same, out of line: a lazy setup at an instance's first triangle (see W8Ray), which most
// entries of an instance-heavy scene never reach, so its code stays out of the walk's registers.
__device__ __noinline__ void w8_shear_late(const uint32_t* __restrict__ w, size_t r, const F3& world_o, W8Ray& R) {
  w8_shear(w, r, world_o, R);
}

// Projected vertex (Ax, Ay, Az): one fixed chain of operations per vertex. `m` keeps the
// largest |v - o| component seen; each component is one rounding of the exact difference, so
// its error is relative to itself, not to |v| or |o|.
RT_DEV F3 w8_project(const W8Ray& R, F3 v, float& m) {
  const F3 a = {__fsub_rn(v.x, R.o.x), __fsub_rn(v.y, R.o.y), __fsub_rn(v.z, R.o.z)};
  m = fmaxf(m, fmaxf(fabsf(a.x), fmaxf(fabsf(a.y), fabsf(a.z))));
  return {__fmaf_rn(a.z, R.mx.z, __fmaf_rn(a.y, R.mx.y, __fmul_rn(a.x, R.mx.x))),
          __fmaf_rn(a.z, R.my.z, __fmaf_rn(a.y, R.my.y, __fmul_rn(a.x, R.my.x))),
          __fmaf_rn(a.z, R.mz.z, __fmaf_rn(a.y, R.mz.y, __fmul_rn(a.x, R.mz.x)))};
}

// An edge function, antisymmetric in its two vertices; exact zero recomputed in double.
RT_DEV float w8_edge(float px, float py, float qx, float qy) {
  float e = __fsub_rn(__fmul_rn(px, qy), __fmul_rn(py, qx));
  if (e == 0.0f) e = (float)__dsub_rn((double)px * (double)qy, (double)py * (double)qx);
  return e;
}

// Watertight test. Returns 0 miss, 1 hit, 2 uncertain (near an edge: the caller re-tests in
// f64). On hit / uncertain, t holds the f32 estimate (it may be outside the range); the
// barycentrics of the final hit come from the f64 final pass.
RT_DEV int w8_triangle(const W8Ray& R, F3 v0, F3 v1, F3 v2, float& t, float& dmax) {
  dmax = 0.0f;
  const F3 A = w8_project(R, v0, dmax), B = w8_project(R, v1, dmax), C = w8_project(R, v2, dmax);
  const float U = w8_edge(C.x, C.y, B.x, B.y);  // opposite v0
  const float V = w8_edge(A.x, A.y, C.x, C.y);  // opposite v1
  const float W = w8_edge(B.x, B.y, A.x, A.y);  // opposite v2
  const float sum = __fadd_rn(__fadd_rn(fabsf(U), fabsf(V)), fabsf(W));
  // How far an f32 edge function may be from the exact one. A projected coordinate is off by at
  // most eA = 8 u |v - o| (the rounding of v - o, of the shear factor and of the fma; |shear| <= 1)
  // plus twice the origin's own error; an edge function of coordinates up to pm is then off by at
  // most 4 pm eA + 2 eA^2 + 4 u pm^2 (taken here with margin). For a small triangle far from the
  // origin this dominates the relative part, W8_EDGE * sum: such hits near an edge are re-tested.
  const float pm = fmaxf(fmaxf(fmaxf(fabsf(A.x), fabsf(A.y)), fmaxf(fabsf(B.x), fabsf(B.y))),
                         fmaxf(fabsf(C.x), fabsf(C.y)));
  const float eA = fmaf(8.0f * W8_U, dmax, 2.0f * R.oerr);
  const float lim = fmaf(W8_EDGE, sum, fmaf(fmaf(3.0f, eA, 5.0f * pm), eA, 5.0f * W8_U * pm * pm));
  const bool neg = U < 0.0f || V < 0.0f || W < 0.0f, pos = U > 0.0f || V > 0.0f || W > 0.0f;
  int kind = 1;
  if (neg && pos) {
    // outside, unless every edge function of the wrong sign is tiny
    const float s = (U + V + W) >= 0.0f ? 1.0f : -1.0f;
    const bool near_edge = (s * U >= -lim) && (s * V >= -lim) && (s * W >= -lim);
    if (!near_edge) return 0;
    kind = 2;
  }
  const float det = __fadd_rn(__fadd_rn(U, V), W);
  if (det == 0.0f) return sum > 0.0f ? 2 : 0;
  if (fabsf(U) <= lim || fabsf(V) <= lim || fabsf(W) <= lim) kind = 2;
  const float T = __fadd_rn(__fadd_rn(__fmul_rn(U, A.z), __fmul_rn(V, B.z)), __fmul_rn(W, C.z));
  t = __fmul_rn(T, __frcp_rn(det));
  return kind;
}

// An uncertain candidate, decided in f64 (out of line: it is rare, and its doubles would
// otherwise take registers from the walk). The candidate and, if the incumbent is still an f32
// estimate, the incumbent are re-intersected with the f64 reference's arithmetic; the lower
// (t, instance, triangle) wins. Returns true when the candidate is the new best.
template <uint32_t LAYOUT>
__device__ __noinline__ bool w8_resolve64(const uint32_t* __restrict__ w, const W8View& V, const Ray& ray, uint32_t inst,
                                          uint32_t tri, uint32_t ident, uint32_t ref, W8Best& best) {
  double t64 = 0.0, u64 = 0.0, v64 = 0.0;
  if (!mt64<LAYOUT>(w, inst, ref, ray, t64, u64, v64)) return false;
  if (best.hit && !best.has64) {
    // the incumbent needs its f64 result too
    const uint4 b2 = __ldg(V.tris + 3 * (size_t)best.tri + 2);
    double bt, bu, bv;
    if (mt64<LAYOUT>(w, best.inst, b2.z, ray, bt, bu, bv)) {
      best.t64 = bt, best.t = (float)bt, best.has64 = true, best.band = 0.0f;
    } else {
      best.hit = false;  // the f32 estimate was a false hit: drop it
    }
  }
  if (best.hit) {
    const bool better = t64 < best.t64 || (t64 == best.t64 && (inst < best.inst || (inst == best.inst && ident < best.ident)));
    if (!better) return false;
  }
  best.hit = true, best.has64 = true, best.t64 = t64, best.t = (float)t64, best.band = 0.0f;
  best.inst = inst, best.tri = tri, best.ident = ident;
  return true;
}

// Considers one candidate triangle; returns true when an any-hit query is satisfied.
template <uint32_t LAYOUT, int AM, bool COUNT, bool LAZY = false>
RT_DEV bool w8_candidate(const uint32_t* __restrict__ w, const W8View& V, W8Ray& R, const Ray& ray, uint32_t inst,
                         uint32_t tri, W8Best& best, unsigned long long* cnt, bool lane_any) {
  w8_count<COUNT>(cnt, W8C_TRIS);
  if (LAZY && !R.sheared) w8_shear_late(w, (LAYOUT == 0 ? 16 : 8) + (size_t)(LAYOUT == 0 ? 32 : 24) * inst, ray.o, R);
  const uint4 q0 = __ldg(V.tris + 3 * (size_t)tri), q1 = __ldg(V.tris + 3 * (size_t)tri + 1),
              q2 = __ldg(V.tris + 3 * (size_t)tri + 2);
  const F3 v0 = {__uint_as_float(q0.x), __uint_as_float(q0.y), __uint_as_float(q0.z)};
  const F3 v1 = {__uint_as_float(q0.w), __uint_as_float(q1.x), __uint_as_float(q1.y)};
  const F3 v2 = {__uint_as_float(q1.z), __uint_as_float(q1.w), __uint_as_float(q2.x)};
  float t, dmax;
  const int kind = w8_triangle(R, v0, v1, v2, t, dmax);
  if (kind == 0) return false;
  const uint32_t ident = q2.y, ref = q2.z;
  const float tmin = ray.tmin, tmax = ray.tmax;
  // How far the f32 t may be from the f64 one: relative W8_TIE, or the absolute part from the
  // rounding of v - o (relative to |v - o|) and from the f32 origin's own error (oerr).
  const float abs_err = R.tscale * (dmax + R.oerr);
  const float band = fmaxf(W8_TIE * fabsf(t), abs_err);
  // Clearly outside the range or clearly behind the current best: nothing to decide.
  if (kind == 1) {
    if (!(t > tmin - band) || !(t < tmax + band)) return false;
    if (best.hit && t > best.t + band + best.band) return false;
  }
  const bool uncertain = kind == 2 || !(t > tmin + band) || !(t < tmax - band) ||
                         (best.hit && t >= best.t - band - best.band);
  if (uncertain) {
    w8_count<COUNT>(cnt, W8C_RETESTS);
    if (!w8_resolve64<LAYOUT>(w, V, ray, inst, tri, ident, ref, best)) return false;
  } else {
    best.hit = true, best.has64 = false, best.t = t, best.band = band;
    best.inst = inst, best.tri = tri, best.ident = ident;
  }
  return AM == 2 ? lane_any : AM == 1;
}

// XOR-permute an 8-bit slot mask: bit k of the result is bit (k ^ o) of m.
RT_DEV uint32_t oct_permute(uint32_t m, uint32_t o) {
  if (o & 1u) m = ((m & 0x55u) << 1) | ((m & 0xAAu) >> 1);
  if (o & 2u) m = ((m & 0x33u) << 2) | ((m & 0xCCu) >> 2);
  if (o & 4u) m = ((m & 0x0Fu) << 4) | ((m & 0xF0u) >> 4);
  return m;
}

// Byte `byte` of `word` as 1 + q * 2^-15, exactly: the byte lands in mantissa bits 8-15 of 1.0f.
RT_DEV float q15(uint32_t word, uint32_t byte) {
  return __uint_as_float(__byte_perm(word, 0x3F800000u, 0x7604u | (byte << 4)));
}

// The per-lane traversal state of the persistent WIDE8 kernel.
struct W8Lane {
  Ray ray;
  F3 world_inv;
  W8Best best;
  uint32_t ray_id, entry, phase;
  bool any;
  uint32_t tsp, flat;
  uint32_t inst;
  W8Ray R;
  uint32_t node;                     // next node to process, EMPTY: take one from the group
  uint32_t g_base, g_bits, g_imask;  // current node group
  uint32_t sp;
};

// The eight child-box tests of one node for one ray: bit s is set when slot s's box meets
// [tmin, lim] (conservatively: no box the ray meets is missed).
RT_DEV uint32_t w8_box_hits(const W8Ray& R, const uint4& a0, const uint4& a2, const uint4& a3, const uint4& a4, float tmin,
                            float lim) {
  const float px = __uint_as_float(a0.x), py = __uint_as_float(a0.y), pz = __uint_as_float(a0.z);
  // A' = 2^(e+15) / d and C = (p - o) / d - A' per axis, so that a plane's t = q 2^e / d + (p - o) / d
  // is one fma of the decoded 1 + q 2^-15: fma(Q, A', C). The same rounded A' enters both terms,
  // so its rounding cancels; exponents stay <= 13 (the builder's bound), so A' never overflows.
  const float Ax = __fmul_rn(__uint_as_float(((a0.w & 0xffu) + 15u) << 23), R.inv.x);
  const float Ay = __fmul_rn(__uint_as_float((((a0.w >> 8) & 0xffu) + 15u) << 23), R.inv.y);
  const float Az = __fmul_rn(__uint_as_float((((a0.w >> 16) & 0xffu) + 15u) << 23), R.inv.z);
  const float Bx = __fmul_rn(__fsub_rn(px, R.o.x), R.inv.x), By = __fmul_rn(__fsub_rn(py, R.o.y), R.inv.y),
              Bz = __fmul_rn(__fsub_rn(pz, R.o.z), R.inv.z);
  // Per axis, |error of a plane's t| <= u (2 * 255 * 2^-15 |A'| + 3 |B|) (the rounding of 1/d,
  // of 2^e / d, of p - o and of (p - o) / d) + 2 u (|B| + |A'|) (the rounding of B - A' and of
  // C -/+ E) + u |t| (the fma), and |t| <= (1 + 255 * 2^-15) |A'| + |C| + |E| <= 2.01 |A'| + 1.01 |B|.
  // So each plane is within u (4.02 |A'| + 6.01 |B|) of exact; doubled (8.4 |A'| + 14.2 |B| with
  // margin for E's own rounding) it moves the near planes down and the far planes up. The max /
  // min of the planes adds no rounding, so the entry and exit need no further widening.
  const float Ex = 2.0f * W8_U * fmaf(4.2f, fabsf(Ax), 7.1f * fabsf(Bx));
  const float Ey = 2.0f * W8_U * fmaf(4.2f, fabsf(Ay), 7.1f * fabsf(By));
  const float Ez = 2.0f * W8_U * fmaf(4.2f, fabsf(Az), 7.1f * fabsf(Bz));
  const float Cx = __fsub_rn(Bx, Ax), Cy = __fsub_rn(By, Ay), Cz = __fsub_rn(Bz, Az);
  const float Bnx = Cx - Ex, Bfx = Cx + Ex, Bny = Cy - Ey, Bfy = Cy + Ey, Bnz = Cz - Ez, Bfz = Cz + Ez;
  // near / far planes per axis by the direction's sign
  const uint32_t nx0 = R.oct & 1u ? a3.z : a2.x, nx1 = R.oct & 1u ? a3.w : a2.y;
  const uint32_t fx0 = R.oct & 1u ? a2.x : a3.z, fx1 = R.oct & 1u ? a2.y : a3.w;
  const uint32_t ny0 = R.oct & 2u ? a4.x : a2.z, ny1 = R.oct & 2u ? a4.y : a2.w;
  const uint32_t fy0 = R.oct & 2u ? a2.z : a4.x, fy1 = R.oct & 2u ? a2.w : a4.y;
  const uint32_t nz0 = R.oct & 4u ? a4.z : a3.x, nz1 = R.oct & 4u ? a4.w : a3.y;
  const uint32_t fz0 = R.oct & 4u ? a3.x : a4.z, fz1 = R.oct & 4u ? a3.y : a4.w;
  uint32_t hits = 0;
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    const uint32_t b = s & 3;
    const float tnx = fmaf(q15(s < 4 ? nx0 : nx1, b), Ax, Bnx), tfx = fmaf(q15(s < 4 ? fx0 : fx1, b), Ax, Bfx);
    const float tny = fmaf(q15(s < 4 ? ny0 : ny1, b), Ay, Bny), tfy = fmaf(q15(s < 4 ? fy0 : fy1, b), Ay, Bfy);
    const float tnz = fmaf(q15(s < 4 ? nz0 : nz1, b), Az, Bnz), tfz = fmaf(q15(s < 4 ? fz0 : fz1, b), Az, Bfz);
    const float tn = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, tmin)), tf = fminf(fminf(tfx, tfy), fminf(tfz, lim));
    if (tn <= tf) hits |= 1u << s;
  }
  return hits;
}

// One 8-wide node: its leaf triangles are tested now, its inner hits become the group.
// Returns true when an any-hit query is satisfied.
// A lane's node-group stack: W8_STACK entries in local memory (cached by L1), or SS entries in a
// shared-memory column of the block (entry i of thread t at i * BLOCK + t: the lanes of a warp
// touch 32 consecutive words, so no bank conflict).
template <int SS, int BLOCK>
struct W8GroupStack {
  uint2* col;
  static constexpr uint32_t cap = SS;
  RT_DEV void push(uint32_t& sp, uint2 v) { col[sp++ * BLOCK] = v; }
  RT_DEV uint2 pop(uint32_t& sp) { return col[--sp * BLOCK]; }
};
template <int BLOCK>
struct W8GroupStack<0, BLOCK> {
  uint2 e[W8_STACK];
  static constexpr uint32_t cap = W8_STACK;
  RT_DEV void push(uint32_t& sp, uint2 v) { e[sp++] = v; }
  RT_DEV uint2 pop(uint32_t& sp) { return e[--sp]; }
};

template <uint32_t LAYOUT, int AM, bool COUNT, bool LAZY, class Stack>
RT_DEV bool w8_node(const uint32_t* __restrict__ w, const W8View& V, W8Lane& L, Stack& stack, DevStatus* st,
                    unsigned long long* cnt) {
  w8_count<COUNT>(cnt, W8C_NODES);
  W8Ray& R = L.R;
  const uint4* np = V.nodes + 5 * (size_t)L.node;
  const uint4 a0 = __ldg(np), a1 = __ldg(np + 1), a2 = __ldg(np + 2), a3 = __ldg(np + 3), a4 = __ldg(np + 4);
  const uint32_t imask = a0.w >> 24;
  const uint32_t child_base = a1.x, tri_base = a1.y, meta_lo = a1.z, meta_hi = a1.w;
  const W8Best& best = L.best;
  const float lim = best.hit ? best.t + 2.0f * best.band + W8_TIE * best.t : L.ray.tmax;
  const uint32_t hits = w8_box_hits(R, a0, a2, a3, a4, L.ray.tmin, lim);
  // Empty slots hold inverted boxes, which no ray meets; one that is met all the same (a node
  // tiny beside its distance, where the widening exceeds 255 steps) has a zero count.
  uint32_t leaf_hits = hits & ~imask;
  while (leaf_hits) {
    const uint32_t s = __ffs(leaf_hits) - 1;
    leaf_hits &= leaf_hits - 1;
    const uint32_t m = ((s < 4 ? meta_lo : meta_hi) >> (8 * (s & 3))) & 0xffu;
    const uint32_t first = tri_base + (m & 31u), count = m >> 5;
    w8_count<COUNT>(cnt, W8C_LEAVES);
    for (uint32_t k = 0; k < count; ++k)
      if (w8_candidate<LAYOUT, AM, COUNT, LAZY>(w, V, R, L.ray, L.inst, first + k, L.best, cnt, L.any)) return true;
  }
  const uint32_t inner = oct_permute(hits & imask, R.oct);
  if (inner) {
    if (L.g_bits) {
      if (L.sp < Stack::cap) stack.push(L.sp, make_uint2(L.g_base, L.g_bits | L.g_imask << 8));
      else atomicAdd(&st->stack_drops, 1ull);
    }
    L.g_base = child_base, L.g_bits = inner, L.g_imask = imask;
  }
  L.node = EMPTY;
  return false;
}

// The next node of the current group (or of a popped one); false when the BLAS is done.
template <class Stack>
RT_DEV bool w8_next(W8Lane& L, Stack& stack) {
  while (L.g_bits == 0) {
    if (L.sp == 0) return false;
    const uint2 e = stack.pop(L.sp);
    L.g_base = e.x, L.g_bits = e.y & 0xffu, L.g_imask = e.y >> 8;
  }
  const uint32_t k = __ffs(L.g_bits) - 1;
  L.g_bits &= L.g_bits - 1;
  const uint32_t slot = k ^ L.R.oct;
  L.node = L.g_base + __popc(L.g_imask & ((1u << slot) - 1u));
  return true;
}

// Enters instance i when its world box survives; sets up the object-space ray.
template <uint32_t LAYOUT, int AM, bool COUNT, bool LAZY = false>
// `from_top`: the instance comes from a leaf of the 8-wide top level, whose box the walk has just
// tested: a box around the world positions of the subtree of BLAS node `at` (relative to the root),
// where this entry starts the walk. The instance's world box would not cull anything more that
// the walk would find (WIDE8's results do not depend on which extra instances it enters, only its
// work does), so it is not tested. A flat instance list has no top-level test, so there the world
// box is tested here.
RT_DEV void w8_enter(const uint32_t* __restrict__ w, const W8View& V, W8Lane& L, uint32_t i, unsigned long long* cnt,
                     bool from_top, uint32_t at = 0) {
  const size_t r = (LAYOUT == 0 ? 16 : 8) + (size_t)(LAYOUT == 0 ? 32 : 24) * i;  // 16-byte aligned records
  if (any_of<AM>(L) && (LAYOUT == 0 ? (ld(w, r + 27) & 1u) != 0 : ld(w, r + 22) != 0)) return;
  w8_count<COUNT>(cnt, W8C_INSTANCE_TESTS);
  if (!from_top) {
    const W8Best& best = L.best;
    const float bound = best.hit ? best.t + 2.0f * best.band + 2.0f * W8_TIE * best.t : L.ray.tmax;
    if (!(slab_near(L.ray.o, L.world_inv, ld3(w, r + 12), ld3(w, r + 15), L.ray.tmin, bound) <= bound)) return;
  }
  const uint32_t root = __ldg(V.inst + 2 * (size_t)i);
  if (root == EMPTY) return;
  const uint4 q0 = ld4(w, r), q1 = ld4(w, r + 4), q2 = ld4(w, r + 8);
  const float r00 = __uint_as_float(q0.x), r01 = __uint_as_float(q0.y), r02 = __uint_as_float(q0.z), r03 = __uint_as_float(q0.w);
  const float r10 = __uint_as_float(q1.x), r11 = __uint_as_float(q1.y), r12 = __uint_as_float(q1.z), r13 = __uint_as_float(q1.w);
  const float r20 = __uint_as_float(q2.x), r21 = __uint_as_float(q2.y), r22 = __uint_as_float(q2.z), r23 = __uint_as_float(q2.w);
  L.R.o = {dot4p(r00, r01, r02, r03, L.ray.o), dot4p(r10, r11, r12, r13, L.ray.o), dot4p(r20, r21, r22, r23, L.ray.o)};
  L.R.d = {dot3({r00, r01, r02}, L.ray.d), dot3({r10, r11, r12}, L.ray.d), dot3({r20, r21, r22}, L.ray.d)};
  w8_setup(L.R);
  if (!L.R.valid) return;
  if (!LAZY) w8_shear(w, r, L.ray.o, L.R);
  L.inst = i;
  L.node = root + at;
  L.g_bits = 0;
  L.sp = 0;
  L.phase = 2;
}

// Ends a lane's ray. Any hit: the flag. Closest hit: the winner as the walk knows it -- the f32 t
// estimate, the record's identity words and, in the words k_wide8_final overwrites, the instance
// and 8-wide triangle that pass needs (reflection: u <- instance, v <- triangle; GI: word 2 <-
// triangle). A miss is written in full here.
template <uint32_t LAYOUT, int AM, bool COUNT, class Src>
RT_DEV void w8_finish(const uint32_t* __restrict__ w, const W8View& V, W8Lane& L, const Src& src,
                      unsigned long long* cnt) {
  w8_count<COUNT>(cnt, W8C_RAYS);
  W8Best& b = L.best;
  const uint32_t id = L.ray_id;
  L.phase = 0;
  if (any_of<AM>(L)) {
    put_flag(src, L.entry, id, L.ray, b.hit);
    return;
  }
  void* __restrict__ out = out_of(src, L.entry);
  if (b.hit) w8_count<COUNT>(cnt, W8C_FINAL64);
  // streaming stores (st.global.cs): the record is written once here and read once by the final pass
  if (LAYOUT == 1) {
    uint32_t* o = reinterpret_cast<uint32_t*>(out) + 5 * (size_t)id;
    __stcs(o, __float_as_uint(b.t));
    __stcs(o + 1, b.hit ? ld(w, 8 + 24 * (size_t)b.inst + 21) + 1 : 0u);
    __stcs(o + 2, b.hit ? b.ident : 0u);
    __stcs(o + 3, b.hit ? b.inst : 0u);
    __stcs(o + 4, b.hit ? b.tri : 0u);
    return;
  }
  uint32_t* o = reinterpret_cast<uint32_t*>(out) + 10 * (size_t)id;
  if (!b.hit) {
    __stcs(o, __float_as_uint(L.ray.tmax)), __stcs(o + 1, EMPTY);
    for (int k = 2; k < 10; ++k) __stcs(o + k, 0u);
    return;
  }
  __stcs(o, __float_as_uint(b.t)), __stcs(o + 1, b.inst), __stcs(o + 2, b.tri);
}

// t, u, v of the f64 reference's Möller-Trumbore (reference.rs:121-158) over the source triangle
// at word `ref`, without its range checks: the walk has already chosen this triangle. False only
// when the f64 determinant is zero.
template <uint32_t LAYOUT>
__device__ __noinline__ bool mt64_values(const uint32_t* __restrict__ w, uint32_t inst, uint32_t ref, const Ray& ray,
                                         double& t, double& u, double& v) {
  D3 o, d;
  ray64<LAYOUT>(w, inst, ray, o, d);
  D3 a, ab, ac;
  if (LAYOUT == 1) {
    a = {ldf(w, ref), ldf(w, ref + 1), ldf(w, ref + 2)};
    ab = {ldf(w, ref + 3), ldf(w, ref + 4), ldf(w, ref + 5)};
    ac = {ldf(w, ref + 6), ldf(w, ref + 7), ldf(w, ref + 8)};
  } else {
    const size_t positions = ld(w, 16 + (size_t)inst * 32 + 20);
    const uint32_t ia = ld(w, ref), ib = ld(w, ref + 1), ic = ld(w, ref + 2);
    a = {ldf(w, positions + 3 * (size_t)ia), ldf(w, positions + 3 * (size_t)ia + 1), ldf(w, positions + 3 * (size_t)ia + 2)};
    const D3 b = {ldf(w, positions + 3 * (size_t)ib), ldf(w, positions + 3 * (size_t)ib + 1), ldf(w, positions + 3 * (size_t)ib + 2)};
    const D3 c = {ldf(w, positions + 3 * (size_t)ic), ldf(w, positions + 3 * (size_t)ic + 1), ldf(w, positions + 3 * (size_t)ic + 2)};
    ab = dsub3(b, a);
    ac = dsub3(c, a);
  }
  const D3 p = dcross(d, ac);
  const double det = ddot(ab, p);
  if (det == 0.0) return false;
  const D3 s = dsub3(o, a);
  const D3 q = dcross(s, ab);
  u = __ddiv_rn(ddot(s, p), det);
  v = __ddiv_rn(ddot(d, q), det);
  t = __ddiv_rn(ddot(ac, q), det);
  return true;
}

// The final values of one closest hit (see the header): f64 t, u, v; for the GI layout also the
// primitive words and the world-space normal (unit_normal of the source winding, as gi_triangle's
// caller forms it). The hit is on 8-wide triangle `tri` of instance `inst`; the walk has written
// its record `o` (the identity words), and t_walk is the walk's t estimate.
template <uint32_t LAYOUT>
RT_DEV void w8_final_values(const uint32_t* __restrict__ w, const W8View& V, const Ray& ray, uint32_t inst, uint32_t tri,
                            float t_walk, uint32_t* __restrict__ o) {
  const uint4 q2 = __ldg(V.tris + 3 * (size_t)tri + 2);
  const uint32_t ident = q2.y, ref = q2.z;
  double t64, u64, v64;
  float t = t_walk, u = 0.0f, v = 0.0f;
  if (mt64_values<LAYOUT>(w, inst, ref, ray, t64, u64, v64)) t = (float)t64, u = (float)u64, v = (float)v64;
  if (LAYOUT == 1) {
    o[0] = __float_as_uint(t), o[3] = __float_as_uint(u), o[4] = __float_as_uint(v);
    return;
  }
  const size_t r = 16 + 32 * (size_t)inst;
  const uint32_t prim_base = ld(w, r + 28), positions = ld(w, r + 20);
  const uint32_t ia = ld(w, ref), ib = ld(w, ref + 1), ic = ld(w, ref + 2);
  const F3 a = ld3(w, positions + 3 * (size_t)ia), bb = ld3(w, positions + 3 * (size_t)ib), c = ld3(w, positions + 3 * (size_t)ic);
  const F3 cr = cross3(sub3(bb, a), sub3(c, a));
  const float m0 = ldf(w, r), m1 = ldf(w, r + 1), m2 = ldf(w, r + 2), m4 = ldf(w, r + 4), m5 = ldf(w, r + 5),
              m6 = ldf(w, r + 6), m8 = ldf(w, r + 8), m9 = ldf(w, r + 9), m10 = ldf(w, r + 10);
  const F3 nrm = unit_normal({add(add(mul(m0, cr.x), mul(m4, cr.y)), mul(m8, cr.z)),
                              add(add(mul(m1, cr.x), mul(m5, cr.y)), mul(m9, cr.z)),
                              add(add(mul(m2, cr.x), mul(m6, cr.y)), mul(m10, cr.z))});
  o[0] = __float_as_uint(t);
  if (prim_base != 0) o[2] = ld(w, prim_base + ident), o[3] = 0, o[4] = 0;
  else o[2] = ia, o[3] = ib, o[4] = ic;
  o[5] = __float_as_uint(u), o[6] = __float_as_uint(v);
  o[7] = __float_as_uint(nrm.x), o[8] = __float_as_uint(nrm.y), o[9] = __float_as_uint(nrm.z);
}

// The packet walk's form, out of line: called once a packet ends, it keeps the f64 work's
// registers out of the walk's own allocation.
template <uint32_t LAYOUT>
__device__ __noinline__ void w8_final_values_call(const uint32_t* __restrict__ w, const W8View& V, const Ray& ray,
                                                  uint32_t inst, uint32_t tri, float t_walk, uint32_t* __restrict__ o) {
  w8_final_values<LAYOUT>(w, V, ray, inst, tri, t_walk, o);
}

// The final pass's form: the record at `o`, its ray read only for a hit.
template <uint32_t LAYOUT>
RT_DEV void w8_final_hit(const uint32_t* __restrict__ w, const W8View& V, const float4* __restrict__ rays, uint32_t i,
                         uint32_t* __restrict__ o) {
  if (LAYOUT == 1 ? o[1] == 0u : o[1] == EMPTY) return;  // a miss (its ray is not read)
  const Ray ray = load_ray_cs(rays, i);
  w8_final_values<LAYOUT>(w, V, ray, LAYOUT == 1 ? o[3] : o[1], LAYOUT == 1 ? o[4] : o[2], __uint_as_float(o[0]), o);
}

// The final pass after a closest-hit WIDE8 launch: one thread per ray of the launch's ray space
// (hits sit at the ray's index, whatever order the walk took the rays in); entries of a
// many-batch launch that are any-hit queries are skipped.
template <uint32_t LAYOUT>
__global__ void __launch_bounds__(256) k_wide8_final(const uint32_t* __restrict__ w, W8View V, OneBatch src, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t* o = reinterpret_cast<uint32_t*>(src.out) + (LAYOUT == 1 ? 5 : 10) * (size_t)i;
  w8_final_hit<LAYOUT>(w, V, src.rays, i, o);
}
template <uint32_t LAYOUT>
__global__ void __launch_bounds__(256) k_wide8_final(const uint32_t* __restrict__ w, W8View V, ManyBatches src, uint32_t n) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  uint32_t lo = 0, hi = src.entries;  // the last entry whose first ray is at or before g
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (src.table[mid].first <= g) lo = mid;
    else hi = mid;
  }
  const BatchEntry& e = src.table[lo];
  if (e.mode != 0) return;
  const uint32_t i = g - e.first;
  uint32_t* o = reinterpret_cast<uint32_t*>(e.hits) + (LAYOUT == 1 ? 5 : 10) * (size_t)i;
  w8_final_hit<LAYOUT>(w, V, e.rays, i, o);
}

RT_DEV uint32_t octant_of(const F3& d) {
  return (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
}

// One node of the 8-wide top level (world space): its children's quantised boxes against the
// world ray and the lane's bound. The inner children met become one group entry; each leaf met
// pushes its entry (instance, BLAS node) above it, the first in visiting order on top, so a node's
// entries are entered before the walk goes deeper.
template <bool COUNT>
RT_DEV void w8_top_node(const W8View& V, const uint4* cache, uint32_t cached, uint32_t node, const W8Lane& L,
                        uint32_t* tstack, uint32_t& tsp, DevStatus* st, unsigned long long* cnt) {
  w8_count<COUNT>(cnt, W8C_TOP_NODES);
  uint4 a0, a1, a2, a3, a4;
  if (node < cached) {
    const uint4* np = cache + 5 * node;
    a0 = np[0], a1 = np[1], a2 = np[2], a3 = np[3], a4 = np[4];
  } else {
    const uint4* np = V.top + 5 * (size_t)node;
    a0 = __ldg(np), a1 = __ldg(np + 1), a2 = __ldg(np + 2), a3 = __ldg(np + 3), a4 = __ldg(np + 4);
  }
  W8Ray TW;
  TW.o = L.ray.o;
  TW.inv = L.world_inv;
  TW.oct = octant_of(L.ray.d);
  const W8Best& b = L.best;
  const float lim = b.hit ? b.t + 2.0f * b.band + 2.0f * W8_TIE * b.t : L.ray.tmax;
  const uint32_t hits = w8_box_hits(TW, a0, a2, a3, a4, L.ray.tmin, lim);
  const uint32_t imask = a0.w >> 24;
  const uint32_t inner = oct_permute(hits & imask, TW.oct);
  if (inner) {
    if (tsp + 2 <= 2 * W8_TOP_STACK) tstack[tsp] = a1.x, tstack[tsp + 1] = inner | imask << 8, tsp += 2;
    else atomicAdd(&st->stack_drops, 1ull);
  }
  for (uint32_t leaves = oct_permute(hits & ~imask, TW.oct); leaves;) {
    const uint32_t k = 31 - __clz(leaves);
    leaves &= ~(1u << k);
    const uint32_t s = k ^ TW.oct;
    const uint32_t m = ((s < 4 ? a1.z : a1.w) >> (8 * (s & 3))) & 0xffu;
    for (uint32_t j = m >> 5; j-- > 0;) {  // an empty slot met all the same has no items
      if (tsp + 2 <= 2 * W8_TOP_STACK) {
        const uint2 e = __ldg(reinterpret_cast<const uint2*>(V.top_items) + a1.y + (m & 31u) + j);
        tstack[tsp] = e.x, tstack[tsp + 1] = e.y | W8_ENTRY, tsp += 2;
      } else {
        atomicAdd(&st->stack_drops, 1ull);
      }
    }
  }
}

// Persistent warps, one ray per lane, refilled as rays end; every iteration a lane takes one
// step (a top-level node, an instance entry, or one 8-wide node with its leaves) and the warp
// re-converges at the top of the loop.
template <uint32_t LAYOUT, int AM, int BLOCK, bool COUNT, class Src, int SS = 0, bool LAZY = false>
__global__ void __launch_bounds__(BLOCK, RT_W8_MIN_BLOCKS) k_wide8(const uint32_t* __restrict__ w, W8View V, const Src src,
                                                 unsigned int* __restrict__ counter, uint32_t n, DevStatus* st,
                                                 unsigned long long* cnt, uint32_t refill) {
  W8GroupStack<SS, BLOCK> stack;
  if constexpr (SS > 0) {
    __shared__ uint2 columns[SS * BLOCK];
    stack.col = columns + threadIdx.x;
  }
  // the packed BVH4 top level's stack (STACK items), or the 8-wide top level's (word pairs)
  uint32_t tstack[STACK > 2 * W8_TOP_STACK ? STACK : 2 * W8_TOP_STACK];
  W8Lane L;
  L.phase = 0;
  const uint32_t count = ld(w, 0), top = ld(w, 1), root = ld(w, 2);
  const size_t top_base = LAYOUT == 0 ? top : (top & ~3u);
  // the 8-wide top level's first nodes, staged once per block (LAZY: the launches over scenes
  // with a top level; a flat scene's launch keeps no shared memory, which leaves L1 more room)
  const bool top8 = top != 0 && V.top != nullptr;
  const uint4* top_cache = nullptr;
  uint32_t cached = 0;
  if constexpr (LAZY && W8_TOP_CACHE > 0) {
    __shared__ uint4 staged[5 * (W8_TOP_CACHE > 0 ? W8_TOP_CACHE : 1)];
    cached = top8 ? min(V.top_count, W8_TOP_CACHE) : 0u;
    for (uint32_t i = threadIdx.x; i < 5 * cached; i += BLOCK) staged[i] = __ldg(V.top + i);
    __syncthreads();
    top_cache = staged;
  }
  bool drained = false;
  for (;;) {
    __syncwarp();
    // ray refill (warp-aggregated) once `refill` lanes are idle: 1 keeps every lane busy,
    // 32 hands out whole runs of 32 consecutive rays (keeps a coherent batch's tiles together)
    const unsigned idle = __ballot_sync(0xffffffffu, L.phase == 0);
    const unsigned want = (!drained && (uint32_t)__popc(idle) >= refill) ? idle : 0u;
    uint32_t id = EMPTY;
    if (want) {
      const int lane = threadIdx.x & 31, leader = __ffs(want) - 1;
      uint32_t base = 0;
      if (lane == leader) base = atomicAdd(counter, (unsigned)__popc(want));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (base + (uint32_t)__popc(want) >= n) drained = true;
      const uint32_t idx = base + __popc(want & ((1u << lane) - 1u));
      if ((want >> lane & 1u) && idx < n) id = idx;
    }
    if (id != EMPTY) {
      L.ray = fetch<true>(src, id, L);
      L.world_inv = safe_inverse(L.ray.d);
      W8Best& b = L.best;
      b.hit = false, b.has64 = false, b.t = L.ray.tmax, b.band = 0.0f, b.t64 = 0.0;
      b.inst = EMPTY, b.tri = 0, b.ident = 0;
      L.phase = 1;
      L.flat = 0;
      L.tsp = 0;
      if (top8) {  // the root as a group of one: slot 0 of an all-inner group at node 0
        tstack[0] = 0, tstack[1] = (1u << octant_of(L.ray.d)) | 0xffu << 8, L.tsp = 2;
      } else if (top != 0 && count != 0) {
        tstack[L.tsp++] = root;
      }
    }
    if (!__any_sync(0xffffffffu, L.phase != 0)) {
      if (drained) break;
      continue;
    }
    if (L.phase == 2) {
      if (L.node == EMPTY && !w8_next(L, stack)) {
        L.phase = 1;
      } else {
        if (w8_node<LAYOUT, AM, COUNT, LAZY>(w, V, L, stack, st, cnt)) w8_finish<LAYOUT, AM, COUNT>(w, V, L, src, cnt);
        continue;
      }
    }
    if (L.phase == 1) {
      if (top == 0) {
        if (L.flat >= count) {
          w8_finish<LAYOUT, AM, COUNT>(w, V, L, src, cnt);
          continue;
        }
        w8_enter<LAYOUT, AM, COUNT, LAZY>(w, V, L, L.flat++, cnt, false);
        continue;
      }
      if (L.tsp == 0) {
        w8_finish<LAYOUT, AM, COUNT>(w, V, L, src, cnt);
        continue;
      }
      if (top8) {
        L.tsp -= 2;
        const uint32_t ex = tstack[L.tsp], ey = tstack[L.tsp + 1];
        if (ey & W8_ENTRY) {  // a leaf's entry: an instance, at a node of its BLAS
          w8_enter<LAYOUT, AM, COUNT, LAZY>(w, V, L, ex, cnt, true, ey & ~W8_ENTRY);
          continue;
        }
        uint32_t bits = ey & 0xffu;  // a group: its first pending child now, the rest back on the stack
        const uint32_t imask = ey >> 8, k = __ffs(bits) - 1;
        bits &= bits - 1;
        if (bits) tstack[L.tsp] = ex, tstack[L.tsp + 1] = bits | imask << 8, L.tsp += 2;
        const uint32_t slot = k ^ octant_of(L.ray.d);
        w8_top_node<COUNT>(V, top_cache, cached, ex + __popc(imask & ((1u << slot) - 1u)), L, tstack, L.tsp, st, cnt);
        continue;
      }
      const uint32_t item = tstack[--L.tsp];
      if (item & LEAF) {
        w8_enter<LAYOUT, AM, COUNT, LAZY>(w, V, L, item & ~LEAF, cnt, true);
        continue;
      }
      const W8Best& b = L.best;
      const float bound = b.hit ? b.t + 2.0f * b.band + 2.0f * W8_TIE * b.t : b.t;
      w8_count<COUNT>(cnt, W8C_TOP_NODES);
      top_step(w, top_base + (size_t)item * 32, L.ray, L.world_inv, bound, tstack, L.tsp, st);
    }
  }
}

// The packet walk's stacks, held in registers across the warp: entry i lives in lane i % 32, in
// register i / 32 of that lane. The walk pushes and pops warp-uniform entries at a warp-uniform
// depth, so a push is one predicated move and a pop one shuffle per register (no shared memory,
// which leaves L1 its full size).
template <int N>
struct WarpStack {
  uint32_t r[(N + 31) / 32];
  RT_DEV void put(uint32_t at, uint32_t v) {
#pragma unroll
    for (int k = 0; k < (N + 31) / 32; ++k)
      if (at == (uint32_t)(threadIdx.x & 31) + 32u * k) r[k] = v;
  }
  RT_DEV uint32_t get(uint32_t at) const {
    uint32_t v = 0;
#pragma unroll
    for (int k = 0; k < (N + 31) / 32; ++k) {
      const uint32_t x = __shfl_sync(0xffffffffu, r[k], at & 31u);
      if ((at >> 5) == (uint32_t)k) v = x;
    }
    return v;
  }
};
struct WarpGroupStack {  // W8_STACK (32) node-group entries: (first child, pending bits | inner mask << 8)
  uint32_t base, bits;
  RT_DEV void put(uint32_t at, uint2 e) {
    if (at == (threadIdx.x & 31)) base = e.x, bits = e.y;
  }
  RT_DEV uint2 get(uint32_t at) const {
    return make_uint2(__shfl_sync(0xffffffffu, base, at), __shfl_sync(0xffffffffu, bits, at));
  }
};
static_assert(W8_STACK == 32, "WarpGroupStack holds one entry a lane");

// One top-level node of the packet walk: each live lane computes its four slab entries against its
// own bound (the per-ray walk's, from its best hit); a child is visited when any lane meets it,
// nearest (over the lanes' entries) first, pushed onto the warp's top stack. Every lane returns
// the stack's new depth.
RT_DEV uint32_t w8_packet_top(const uint32_t* __restrict__ w, size_t n, const W8Lane& L, bool live,
                              WarpStack<STACK>& tstack, uint32_t sp, DevStatus* st) {
  uint32_t key[4], ids[4];
  const W8Best& b = L.best;
  const float bound = b.hit ? b.t + 2.0f * b.band + 2.0f * W8_TIE * b.t : b.t;
  const uint4 lx = ld4u(w, n), ly = ld4u(w, n + 4), lz = ld4u(w, n + 8);
  const uint4 hx = ld4u(w, n + 12), hy = ld4u(w, n + 16), hz = ld4u(w, n + 20), id4 = ld4u(w, n + 24);
  auto at = [](const uint4& q, int c) { return c == 0 ? q.x : (c == 1 ? q.y : (c == 2 ? q.z : q.w)); };
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    ids[c] = at(id4, c);
    uint32_t k = 0xffffffffu;  // no lane meets the child
    if (live && ids[c] != EMPTY) {
      const F3& o = L.ray.o;
      const F3& inv = L.world_inv;
      const float ax = mul(sub(__uint_as_float(at(lx, c)), o.x), inv.x), bx = mul(sub(__uint_as_float(at(hx, c)), o.x), inv.x);
      const float ay = mul(sub(__uint_as_float(at(ly, c)), o.y), inv.y), by = mul(sub(__uint_as_float(at(hy, c)), o.y), inv.y);
      const float az = mul(sub(__uint_as_float(at(lz, c)), o.z), inv.z), bz = mul(sub(__uint_as_float(at(hz, c)), o.z), inv.z);
      const float near = fmaxf(fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fminf(az, bz)), L.ray.tmin);
      const float far = fminf(fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fmaxf(az, bz)), bound);
      if (near <= far) {  // an order-preserving key of the entry distance
        const uint32_t u = __float_as_uint(near);
        k = (u >> 31) ? ~u : (u | 0x80000000u);
        k = k == 0xffffffffu ? 0xfffffffeu : k;
      }
    }
    key[c] = __reduce_min_sync(0xffffffffu, k);
  }
#define RT_SW(a, b)                                                     \
  if (key[b] < key[a]) {                                                \
    uint32_t x = key[a]; key[a] = key[b]; key[b] = x;                   \
    x = ids[a]; ids[a] = ids[b]; ids[b] = x;                            \
  }
  RT_SW(0, 1) RT_SW(2, 3) RT_SW(0, 2) RT_SW(1, 3) RT_SW(1, 2)
#undef RT_SW
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int c = 3; c >= 0; --c) {  // far to near: the nearest is popped first
    if (key[c] == 0xffffffffu) continue;
    if (sp < STACK) {
      tstack.put(sp, ids[c]);
      ++sp;
    } else if (lane == 0) {
      atomicAdd(&st->stack_drops, 1ull);
    }
  }
  return sp;
}

// Packet walk, for coherent batches: a warp takes 32 consecutive rays and walks ONE traversal for
// all of them -- the top level's BVH4 (or the flat instance list) and each entered instance's
// 8-wide BLAS. A node's child is visited when any lane's ray meets its box, in the first entering
// lane's octant order (top-level nodes: nearest entry over the lanes first), so every lane reads
// the same node (one broadcast load) and no lane diverges on the walk; the traversal stacks are
// the warp's, in registers (WarpStack). Each lane still tests its own ray against every visited
// node's boxes (its own hits and closest-hit bound), enters only the instances whose world box its
// ray meets, and tests the triangles of the leaves its ray meets. WIDE8's results do not depend on
// the visit order (conservative boxes, ties resolved in f64 on (t, instance, triangle)), so each
// ray gets the hit the per-ray walk finds.
template <uint32_t LAYOUT, int AM, int BLOCK, class Src>
__global__ void __launch_bounds__(BLOCK, RT_W8P_MIN_BLOCKS) k_wide8_packet(const uint32_t* __restrict__ w, W8View V, const Src src,
                                                           unsigned int* __restrict__ counter, uint32_t n, DevStatus* st) {
  WarpGroupStack stack;
  WarpStack<STACK> tstack;
  const int lane = threadIdx.x & 31;
  const uint32_t count = ld(w, 0), top = ld(w, 1), root = ld(w, 2);
  const size_t top_base = LAYOUT == 0 ? top : (top & ~3u);
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(counter, 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= n) break;
    const uint32_t id = base + lane;
    W8Lane L;
    L.phase = 0;
    bool live = id < n;  // the lane's ray still wants hits
    if (live) {
      L.ray = fetch<true>(src, id, L);
      L.world_inv = safe_inverse(L.ray.d);
      W8Best& b = L.best;
      b.hit = false, b.has64 = false, b.t = L.ray.tmax, b.band = 0.0f, b.t64 = 0.0;
      b.inst = EMPTY, b.tri = 0, b.ident = 0;
    }
    uint32_t flat = 0, tsp = 0;
    if (top != 0 && count != 0) {
      tstack.put(0, root);
      tsp = 1;
    }
    while (__any_sync(0xffffffffu, live)) {
      uint32_t i;  // the next instance the warp tries (uniform)
      if (top == 0) {
        if (flat >= count) break;
        i = flat++;
      } else {
        if (tsp == 0) break;
        const uint32_t item = tstack.get(--tsp);
        if (!(item & LEAF)) {
          tsp = w8_packet_top(w, top_base + (size_t)item * 32, L, live, tstack, tsp, st);
          continue;
        }
        i = item & ~LEAF;
      }
      L.phase = 0;
      if (live) w8_enter<LAYOUT, AM, false>(w, V, L, i, nullptr, false);
      bool in = L.phase == 2;
      const unsigned entering = __ballot_sync(0xffffffffu, in);
      if (!entering) continue;
      const uint32_t oct = __shfl_sync(0xffffffffu, L.R.oct, __ffs(entering) - 1);
      uint32_t node = __ldg(V.inst + 2 * (size_t)i), g_base = 0, g_bits = 0, g_imask = 0, sp = 0;
      for (;;) {
        if (node == EMPTY) {  // the warp's next node (uniform)
          while (g_bits == 0 && sp > 0) {
            const uint2 e = stack.get(--sp);
            g_base = e.x, g_bits = e.y & 0xffu, g_imask = e.y >> 8;
          }
          if (g_bits == 0) break;
          const uint32_t slot = (__ffs(g_bits) - 1) ^ oct;
          g_bits &= g_bits - 1;
          node = g_base + __popc(g_imask & ((1u << slot) - 1u));
        }
        const uint4* np = V.nodes + 5 * (size_t)node;
        const uint4 a0 = __ldg(np), a1 = __ldg(np + 1), a2 = __ldg(np + 2), a3 = __ldg(np + 3), a4 = __ldg(np + 4);
        const uint32_t imask = a0.w >> 24, child_base = a1.x, tri_base = a1.y, meta_lo = a1.z, meta_hi = a1.w;
        uint32_t hits = 0;
        if (in) {
          const W8Best& best = L.best;
          const float lim = best.hit ? best.t + 2.0f * best.band + W8_TIE * best.t : L.ray.tmax;
          hits = w8_box_hits(L.R, a0, a2, a3, a4, L.ray.tmin, lim);
        }
        // leaves: every lane whose ray meets one tests its triangles
        for (uint32_t lh = __reduce_or_sync(0xffffffffu, hits & ~imask); lh; lh &= lh - 1) {
          const uint32_t s = __ffs(lh) - 1;
          if (!in || !(hits >> s & 1u)) continue;
          const uint32_t m = ((s < 4 ? meta_lo : meta_hi) >> (8 * (s & 3))) & 0xffu;
          const uint32_t first = tri_base + (m & 31u), cnt = m >> 5;
          for (uint32_t k = 0; k < cnt; ++k)
            if (w8_candidate<LAYOUT, AM, false>(w, V, L.R, L.ray, L.inst, first + k, L.best, nullptr, L.any)) {
              in = false, live = false;  // an any-hit ray is blocked
              break;
            }
        }
        const uint32_t inner = oct_permute(__reduce_or_sync(0xffffffffu, hits & imask), oct);
        node = EMPTY;
        if (!__any_sync(0xffffffffu, in)) break;
        if (inner) {
          if (g_bits) {
            if (sp < W8_STACK) {
              stack.put(sp, make_uint2(g_base, g_bits | g_imask << 8));
              ++sp;
            } else if (lane == 0) {
              atomicAdd(&st->stack_drops, 1ull);
            }
          }
          g_base = child_base, g_bits = inner, g_imask = imask;
        }
      }
    }
    if (id < n) {
      w8_finish<LAYOUT, AM, false>(w, V, L, src, nullptr);
      // The lanes of a warp end their packet together, so a closest hit's final values are made
      // here, converged, rather than by a separate final pass (the same arithmetic on the same
      // instance, triangle, ray and t estimate, hence the same words).
      if (!any_of<AM>(L) && L.best.hit)
        w8_final_values_call<LAYOUT>(w, V, L.ray, L.best.inst, L.best.tri, L.best.t,
                                     reinterpret_cast<uint32_t*>(out_of(src, L.entry)) + (LAYOUT == 1 ? 5 : 10) * (size_t)L.ray_id);
    }
  }
}

}  // namespace rtk
