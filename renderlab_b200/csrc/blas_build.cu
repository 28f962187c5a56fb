// GPU build of one mesh's BVH4-Q8 (near_field::build_bvh_sah / build_bvh, near_field.rs:172-436)
// whose records equal the host builder's (host/blas.cpp), word for word.
//
// The host builder recurses depth first; this one splits level by level. Both give the same
// tree, for four reasons:
//  * a split depends only on its own range of the triangle permutation, and its halves keep
//    their input order (near_field.rs:361-364), so every range of one level splits in parallel
//    and the permutation ends up as the host's, leaves in depth-first order;
//  * the centroid and bin boxes are min/max reductions, taken here in any order through
//    order-preserving integer keys. They can differ from the host's only in the sign of a zero
//    bound, and that changes no bin, extent test, cost comparison or split;
//  * the cost sweep runs on one thread per split, with the host's operations in the host's order;
//  * a median split sorts by (centroid, triangle), a key with no ties.
// A split of a range is a node group when its binary depth is even: its halves, and the halves of
// those halves, are the node's children (near_field.rs:286-306). The node ids follow postorder,
// which is the order of (range end, range length). A child's slot is its order by range start.
// Nodes are quantised bottom-up, one launch per node level, with the refit's device quantiser.
// An SAH tree deeper than 15 node levels is built again by median splits (near_field.rs:184-190).
// The deepest node group then sits at binary depth 30 or more, which the level loop sees as it
// gets there.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_segmented_sort.cuh>

#include <algorithm>
#include <memory>
#include <thread>
#include <vector>

#include "ctx.hpp"
#include "kernels/bvh4_quant.cuh"
#include "kernels/order_keys.cuh"

using namespace rtc;

namespace {

using namespace rtq;

constexpr uint32_t LEAF_TRIS = rtb::LEAF_TRIANGLES;     // near_field.rs:23
constexpr uint32_t BINS = 16;                           // near_field.rs:273
constexpr uint32_t TOO_DEEP = 2 * rtb::MAX_SAH_DEPTH;   // binary depth of node level 16
constexpr uint32_t SMALL = 2048;          // a range of at most this many triangles splits in one block
constexpr uint32_t SMALL_THREADS = 128;
constexpr uint32_t CHUNK = 4096;          // triangles one block takes of a larger range
constexpr uint32_t CHUNK_THREADS = 256;
constexpr uint32_t MAX_TRIANGLES = 1u << 29;
constexpr int KIND_MEDIAN = 0, KIND_SAH = 1;

struct Seg {  // a range [b, e) of the permutation at binary depth `depth`
  uint32_t b, e, depth, owner;  // owner: the node group whose child the range is (or EMPTY)
};

struct LargeSeg {  // a range split by several blocks
  uint32_t i, b, e, first, n;  // level index, range, its chunks
};

struct Chunk {
  uint32_t j, b, e;  // large range, part of it
};

struct LWork {  // a large range's reductions and decision
  uint32_t cb[6];
  uint32_t cnt[3 * BINS];
  uint32_t bl[3 * BINS * 3], bh[3 * BINS * 3];
  int kind, axis, plane;
  uint32_t mid;
};

// The SAH bin of a centroid coordinate (near_field.rs:327-330): ((c - lo) / extent * 16) as
// usize, at most 15.
__device__ __forceinline__ uint32_t bin_of(float c, float lo, float extent) {
  const float f = __fmul_rn(__fdiv_rn(__fsub_rn(c, lo), extent), (float)BINS);
  if (!(f > 0.0f)) return 0;
  return f >= (float)(BINS - 1) ? BINS - 1 : (uint32_t)f;
}

__device__ __forceinline__ float half_area(const float* lo, const float* hi) {  // near_field.rs:274-277
  const float e0 = hi_of(__fsub_rn(hi[0], lo[0]), 0.0f), e1 = hi_of(__fsub_rn(hi[1], lo[1]), 0.0f),
              e2 = hi_of(__fsub_rn(hi[2], lo[2]), 0.0f);
  return __fadd_rn(__fadd_rn(__fmul_rn(e0, e1), __fmul_rn(e1, e2)), __fmul_rn(e2, e0));
}

struct Choice {
  int kind, axis, plane;
};

// The split of one range from its centroid box and bins (near_field.rs:317-379): the cheapest
// SAH plane, ties to the lower axis and bin, else the median on the axis of largest extent (the
// last of equal extents). Bin boxes are order keys; an empty bin adds nothing.
__device__ Choice choose(const float* lo, const float* hi, const uint32_t* cnt, const uint32_t* bl,
                         const uint32_t* bh, uint32_t len, bool sah) {
  bool found = false;
  float best = 0.0f;
  Choice c{KIND_SAH, 0, 0};
  for (int axis = 0; sah && axis < 3; ++axis) {
    const float extent = __fsub_rn(hi[axis], lo[axis]);
    if (!(extent > 0.0f)) continue;
    const uint32_t* n = cnt + axis * BINS;
    const uint32_t* l = bl + axis * BINS * 3;
    const uint32_t* h = bh + axis * BINS * 3;
    float right[BINS];
    float al[3] = {INFINITY, INFINITY, INFINITY}, ah[3] = {-INFINITY, -INFINITY, -INFINITY};
    uint32_t seen = 0;
    for (int b = BINS - 1; b >= 1; --b) {
      if (n[b])
        for (int a = 0; a < 3; ++a) al[a] = lo_of(al[a], unkey(l[3 * b + a])), ah[a] = hi_of(ah[a], unkey(h[3 * b + a]));
      seen += n[b];
      right[b] = __fmul_rn(half_area(al, ah), (float)seen);
    }
    for (int a = 0; a < 3; ++a) al[a] = INFINITY, ah[a] = -INFINITY;
    seen = 0;
    for (int b = 0; b < (int)BINS - 1; ++b) {
      if (n[b])
        for (int a = 0; a < 3; ++a) al[a] = lo_of(al[a], unkey(l[3 * b + a])), ah[a] = hi_of(ah[a], unkey(h[3 * b + a]));
      seen += n[b];
      if (seen == 0 || seen == len) continue;
      const float cost = __fadd_rn(__fmul_rn(half_area(al, ah), (float)seen), right[b + 1]);
      if (!found || cost < best) found = true, best = cost, c.axis = axis, c.plane = b;
    }
  }
  if (found) return c;
  c.kind = KIND_MEDIAN;
  c.axis = 0;
  for (int a = 1; a < 3; ++a)
    if (order_key(__fsub_rn(hi[a], lo[a])) >= order_key(__fsub_rn(hi[c.axis], lo[c.axis]))) c.axis = a;
  c.plane = 0;
  return c;
}

__device__ __forceinline__ unsigned long long median_key(const float* cen, uint32_t t, int axis) {
  return (unsigned long long)okey(cen[3 * (size_t)t + axis]) << 32 | t;
}

// build_blas's geometry checks (near_field.rs:208-214) on the device: bit 0 an index past the
// positions, bit 1 a position that is not finite.
__global__ void k_validate(const float* __restrict__ pos, uint32_t n_floats, const uint32_t* __restrict__ idx,
                           uint32_t n_idx, uint32_t n_pos, uint32_t* __restrict__ bad) {
  uint32_t found = 0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < (size_t)n_floats + n_idx; k += (size_t)gridDim.x * blockDim.x) {
    if (k < n_floats) found |= isfinite(pos[k]) ? 0u : 2u;
    else found |= idx[k - n_floats] >= n_pos ? 1u : 0u;
  }
  if (found) atomicOr(bad, found);
}

// Centroids (near_field.rs:216-226: the corners summed in order, then / 3), the triangles' boxes
// as order keys, and the identity permutation.
__global__ void k_prepare(const float* __restrict__ pos, const uint32_t* __restrict__ idx, uint32_t nt,
                          float* __restrict__ cen, uint32_t* __restrict__ tbk, uint32_t* __restrict__ perm) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const float* p0 = pos + 3 * (size_t)idx[3 * (size_t)t];
  const float* p1 = pos + 3 * (size_t)idx[3 * (size_t)t + 1];
  const float* p2 = pos + 3 * (size_t)idx[3 * (size_t)t + 2];
  for (int a = 0; a < 3; ++a) {
    cen[3 * (size_t)t + a] = __fdiv_rn(__fadd_rn(__fadd_rn(p0[a], p1[a]), p2[a]), 3.0f);
    tbk[6 * (size_t)t + a] = okey(lo_of(lo_of(p0[a], p1[a]), p2[a]));
    tbk[6 * (size_t)t + 3 + a] = okey(hi_of(hi_of(p0[a], p1[a]), p2[a]));
  }
  perm[t] = t;
}

// Per range of the level: pending (more than a leaf's triangles) in the low word, split by
// several blocks in the high word; one extra zero entry so the exclusive sum ends in the totals.
__global__ void k_level_flags(const Seg* __restrict__ segs, uint32_t width, unsigned long long* __restrict__ flags) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > width) return;
  if (i == width) {
    flags[i] = 0;
    return;
  }
  const uint32_t len = segs[i].e - segs[i].b;
  flags[i] = (unsigned long long)(len > LEAF_TRIS) | (unsigned long long)(len > SMALL) << 32;
}

__device__ __forceinline__ void write_children(Seg* segs, uint32_t lv0, uint32_t i, const Seg& g, uint32_t mid,
                                               uint32_t next, const unsigned long long* rank) {
  const uint32_t r = (uint32_t)rank[i];
  const uint32_t own = (g.depth & 1u) ? g.owner : lv0 + i;
  segs[next + 2 * r] = Seg{g.b, mid, g.depth + 1, own};
  segs[next + 2 * r + 1] = Seg{mid, g.e, g.depth + 1, own};
}

struct LevelArgs {
  Seg* segs;
  uint32_t lv0, width, next;  // this level's ranges: segs[lv0, lv0 + width); the next level from `next`
  const unsigned long long* rank;
  const float* cen;
  const uint32_t* tbk;
  uint32_t* perm;
  int sah;
};

// One block splits one range of at most SMALL triangles, all in shared memory.
__global__ void __launch_bounds__(SMALL_THREADS) k_split_small(LevelArgs a) {
  const uint32_t i = blockIdx.x;
  const Seg g = a.segs[a.lv0 + i];
  const uint32_t len = g.e - g.b;
  if (len <= LEAF_TRIS || len > SMALL) return;
  __shared__ uint32_t sp[SMALL];
  __shared__ unsigned long long skey[SMALL];
  __shared__ uint32_t cb[6], cnt[3 * BINS], bl[3 * BINS * 3], bh[3 * BINS * 3], runs[SMALL_THREADS];
  __shared__ Choice choice;
  __shared__ uint32_t total;
  const uint32_t tid = threadIdx.x, nth = blockDim.x;
  if (tid < 3) cb[tid] = 0xffffffffu, cb[3 + tid] = 0u;
  for (uint32_t k = tid; k < 3 * BINS; k += nth) cnt[k] = 0;
  for (uint32_t k = tid; k < 3 * BINS * 3; k += nth) bl[k] = 0xffffffffu, bh[k] = 0u;
  __syncthreads();
  uint32_t l[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, h[3] = {0u, 0u, 0u};
  for (uint32_t k = tid; k < len; k += nth) {
    const uint32_t t = a.perm[g.b + k];
    sp[k] = t;
    for (int x = 0; x < 3; ++x) {
      const uint32_t v = okey(a.cen[3 * (size_t)t + x]);
      l[x] = min(l[x], v), h[x] = max(h[x], v);
    }
  }
  for (int x = 0; x < 3; ++x) atomicMin(&cb[x], l[x]), atomicMax(&cb[3 + x], h[x]);
  __syncthreads();
  float lo[3], hi[3];
  for (int x = 0; x < 3; ++x) lo[x] = unkey(cb[x]), hi[x] = unkey(cb[3 + x]);
  if (a.sah) {
    for (uint32_t k = tid; k < len; k += nth) {
      const uint32_t t = sp[k];
      for (int axis = 0; axis < 3; ++axis) {
        const float extent = __fsub_rn(hi[axis], lo[axis]);
        if (!(extent > 0.0f)) continue;
        const uint32_t b = axis * BINS + bin_of(a.cen[3 * (size_t)t + axis], lo[axis], extent);
        atomicAdd(&cnt[b], 1u);
        for (int x = 0; x < 3; ++x)
          atomicMin(&bl[3 * b + x], a.tbk[6 * (size_t)t + x]), atomicMax(&bh[3 * b + x], a.tbk[6 * (size_t)t + 3 + x]);
      }
    }
    __syncthreads();
  }
  if (tid == 0) choice = choose(lo, hi, cnt, bl, bh, len, a.sah != 0);
  __syncthreads();
  const Choice c = choice;
  uint32_t mid;
  if (c.kind == KIND_SAH) {  // stable partition: thread tid moves the run [r0, r1) of the range
    const float extent = __fsub_rn(hi[c.axis], lo[c.axis]);
    const uint32_t per = (len + nth - 1) / nth, r0 = min(len, tid * per), r1 = min(len, r0 + per);
    uint32_t nl = 0;
    for (uint32_t k = r0; k < r1; ++k) nl += bin_of(a.cen[3 * (size_t)sp[k] + c.axis], lo[c.axis], extent) <= (uint32_t)c.plane;
    runs[tid] = nl;
    __syncthreads();
    if (tid == 0) {
      uint32_t s = 0;
      for (uint32_t j = 0; j < nth; ++j) {
        const uint32_t v = runs[j];
        runs[j] = s;
        s += v;
      }
      total = s;
    }
    __syncthreads();
    uint32_t left = runs[tid], right = r0 - runs[tid];
    const uint32_t n_left = total;
    for (uint32_t k = r0; k < r1; ++k) {
      const uint32_t t = sp[k];
      if (bin_of(a.cen[3 * (size_t)t + c.axis], lo[c.axis], extent) <= (uint32_t)c.plane)
        a.perm[g.b + left++] = t;
      else
        a.perm[g.b + n_left + right++] = t;
    }
    mid = g.b + n_left;
  } else {  // bitonic sort of (centroid key, triangle), padded to a power of two
    uint32_t n2 = 1;
    while (n2 < len) n2 <<= 1;
    for (uint32_t k = tid; k < n2; k += nth) skey[k] = k < len ? median_key(a.cen, sp[k], c.axis) : ~0ull;
    __syncthreads();
    for (uint32_t size = 2; size <= n2; size <<= 1)
      for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
        for (uint32_t k = tid; k < n2; k += nth) {
          const uint32_t p = k ^ stride;
          if (p > k) {
            const unsigned long long x = skey[k], y = skey[p];
            if ((x > y) == ((k & size) == 0)) skey[k] = y, skey[p] = x;
          }
        }
        __syncthreads();
      }
    for (uint32_t k = tid; k < len; k += nth) a.perm[g.b + k] = (uint32_t)skey[k];
    mid = g.b + len / 2;
  }
  if (tid == 0) write_children(a.segs, a.lv0, i, g, mid, a.next, a.rank);
}

// ---- ranges larger than SMALL: several blocks each, reductions merged through global atomics ----

__global__ void k_large_list(const Seg* __restrict__ segs, uint32_t width, const unsigned long long* __restrict__ rank,
                             LargeSeg* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= width) return;
  const Seg g = segs[i];
  if (g.e - g.b > SMALL) out[rank[i] >> 32] = LargeSeg{i, g.b, g.e, 0, 0};
}

__global__ void k_large_init(LWork* __restrict__ w, uint32_t n) {
  const uint32_t j = blockIdx.x;
  if (j >= n) return;
  LWork& x = w[j];
  for (uint32_t k = threadIdx.x; k < 3 * BINS * 3; k += blockDim.x) {
    x.bl[k] = 0xffffffffu, x.bh[k] = 0u;
    if (k < 3 * BINS) x.cnt[k] = 0u;
    if (k < 6) x.cb[k] = k < 3 ? 0xffffffffu : 0u;
  }
}

__device__ __forceinline__ void bounds_of(const LWork& w, float* lo, float* hi) {
  for (int x = 0; x < 3; ++x) lo[x] = unkey(w.cb[x]), hi[x] = unkey(w.cb[3 + x]);
}

__global__ void __launch_bounds__(CHUNK_THREADS) k_large_cbox(const Chunk* __restrict__ chunks, const uint32_t* __restrict__ perm,
                                                              const float* __restrict__ cen, LWork* __restrict__ work) {
  const Chunk ch = chunks[blockIdx.x];
  __shared__ uint32_t cb[6];
  if (threadIdx.x < 6) cb[threadIdx.x] = threadIdx.x < 3 ? 0xffffffffu : 0u;
  __syncthreads();
  uint32_t l[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, h[3] = {0u, 0u, 0u};
  for (uint32_t k = ch.b + threadIdx.x; k < ch.e; k += blockDim.x) {
    const uint32_t t = perm[k];
    for (int x = 0; x < 3; ++x) {
      const uint32_t v = okey(cen[3 * (size_t)t + x]);
      l[x] = min(l[x], v), h[x] = max(h[x], v);
    }
  }
  for (int x = 0; x < 3; ++x) atomicMin(&cb[x], l[x]), atomicMax(&cb[3 + x], h[x]);
  __syncthreads();
  if (threadIdx.x < 3) atomicMin(&work[ch.j].cb[threadIdx.x], cb[threadIdx.x]);
  else if (threadIdx.x < 6) atomicMax(&work[ch.j].cb[threadIdx.x], cb[threadIdx.x]);
}

__global__ void __launch_bounds__(CHUNK_THREADS) k_large_bins(const Chunk* __restrict__ chunks, const uint32_t* __restrict__ perm,
                                                              const float* __restrict__ cen, const uint32_t* __restrict__ tbk,
                                                              LWork* __restrict__ work) {
  const Chunk ch = chunks[blockIdx.x];
  __shared__ uint32_t cnt[3 * BINS], bl[3 * BINS * 3], bh[3 * BINS * 3];
  for (uint32_t k = threadIdx.x; k < 3 * BINS * 3; k += blockDim.x) {
    bl[k] = 0xffffffffu, bh[k] = 0u;
    if (k < 3 * BINS) cnt[k] = 0u;
  }
  __syncthreads();
  LWork& w = work[ch.j];
  float lo[3], hi[3];
  bounds_of(w, lo, hi);
  for (uint32_t k = ch.b + threadIdx.x; k < ch.e; k += blockDim.x) {
    const uint32_t t = perm[k];
    for (int axis = 0; axis < 3; ++axis) {
      const float extent = __fsub_rn(hi[axis], lo[axis]);
      if (!(extent > 0.0f)) continue;
      const uint32_t b = axis * BINS + bin_of(cen[3 * (size_t)t + axis], lo[axis], extent);
      atomicAdd(&cnt[b], 1u);
      for (int x = 0; x < 3; ++x)
        atomicMin(&bl[3 * b + x], tbk[6 * (size_t)t + x]), atomicMax(&bh[3 * b + x], tbk[6 * (size_t)t + 3 + x]);
    }
  }
  __syncthreads();
  for (uint32_t b = threadIdx.x; b < 3 * BINS; b += blockDim.x) {
    if (!cnt[b]) continue;
    atomicAdd(&w.cnt[b], cnt[b]);
    for (int x = 0; x < 3; ++x) atomicMin(&w.bl[3 * b + x], bl[3 * b + x]), atomicMax(&w.bh[3 * b + x], bh[3 * b + x]);
  }
}

__global__ void k_large_choose(const LargeSeg* __restrict__ large, uint32_t n, LWork* __restrict__ work, int sah) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  LWork& w = work[j];
  float lo[3], hi[3];
  bounds_of(w, lo, hi);
  const Choice c = choose(lo, hi, w.cnt, w.bl, w.bh, large[j].e - large[j].b, sah != 0);
  w.kind = c.kind, w.axis = c.axis, w.plane = c.plane;
}

__device__ __forceinline__ bool goes_left(const LWork& w, const float* cen, uint32_t t) {
  const float lo = unkey(w.cb[w.axis]), extent = __fsub_rn(unkey(w.cb[3 + w.axis]), lo);
  return bin_of(cen[3 * (size_t)t + w.axis], lo, extent) <= (uint32_t)w.plane;
}

// Left-going triangles of each chunk of an SAH range.
__global__ void __launch_bounds__(CHUNK_THREADS) k_large_count(const Chunk* __restrict__ chunks, const uint32_t* __restrict__ perm,
                                                               const float* __restrict__ cen, const LWork* __restrict__ work,
                                                               uint32_t* __restrict__ chunk_left) {
  const Chunk ch = chunks[blockIdx.x];
  const LWork& w = work[ch.j];
  if (w.kind != KIND_SAH) return;
  __shared__ uint32_t n;
  if (threadIdx.x == 0) n = 0;
  __syncthreads();
  uint32_t m = 0;
  for (uint32_t k = ch.b + threadIdx.x; k < ch.e; k += blockDim.x) m += goes_left(w, cen, perm[k]);
  atomicAdd(&n, m);
  __syncthreads();
  if (threadIdx.x == 0) chunk_left[blockIdx.x] = n;
}

// Per large range: where each chunk's left- and right-going triangles start, the cut, the sort
// range of a median split (empty for an SAH one), and the two children.
__global__ void k_large_scan(const LargeSeg* __restrict__ large, uint32_t n, LWork* __restrict__ work,
                             const uint32_t* __restrict__ chunk_left, uint32_t* __restrict__ chunk_base,
                             uint32_t* __restrict__ sort_begin, uint32_t* __restrict__ sort_end, Seg* segs, uint32_t lv0,
                             uint32_t next, const unsigned long long* __restrict__ rank) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const LargeSeg L = large[j];
  LWork& w = work[j];
  uint32_t mid;
  if (w.kind == KIND_SAH) {
    uint32_t s = 0;
    for (uint32_t k = L.first; k < L.first + L.n; ++k) chunk_base[k] = s, s += chunk_left[k];
    mid = L.b + s;
    sort_begin[j] = sort_end[j] = L.b;
  } else {
    mid = L.b + (L.e - L.b) / 2;
    sort_begin[j] = L.b, sort_end[j] = L.e;
  }
  w.mid = mid;
  write_children(segs, lv0, L.i, segs[lv0 + L.i], mid, next, rank);
}

// The stable partition of each SAH range's chunk into `tmp`: thread t moves a run of the chunk.
__global__ void __launch_bounds__(CHUNK_THREADS) k_large_scatter(const Chunk* __restrict__ chunks, const LargeSeg* __restrict__ large,
                                                                 const uint32_t* __restrict__ perm, const float* __restrict__ cen,
                                                                 const LWork* __restrict__ work, const uint32_t* __restrict__ chunk_base,
                                                                 uint32_t* __restrict__ tmp) {
  const Chunk ch = chunks[blockIdx.x];
  const LWork& w = work[ch.j];
  if (w.kind != KIND_SAH) return;
  __shared__ uint32_t runs[CHUNK_THREADS];
  const uint32_t len = ch.e - ch.b, tid = threadIdx.x, nth = blockDim.x;
  const uint32_t per = (len + nth - 1) / nth, r0 = min(len, tid * per), r1 = min(len, r0 + per);
  uint32_t nl = 0;
  for (uint32_t k = r0; k < r1; ++k) nl += goes_left(w, cen, perm[ch.b + k]);
  runs[tid] = nl;
  __syncthreads();
  if (tid == 0) {
    uint32_t s = 0;
    for (uint32_t q = 0; q < nth; ++q) {
      const uint32_t v = runs[q];
      runs[q] = s;
      s += v;
    }
  }
  __syncthreads();
  const uint32_t seg_b = large[ch.j].b, lefts_before = chunk_base[blockIdx.x];
  const uint32_t rights_before = (ch.b - seg_b) - lefts_before;
  uint32_t left = seg_b + lefts_before + runs[tid];
  uint32_t right = w.mid + rights_before + (r0 - runs[tid]);
  for (uint32_t k = r0; k < r1; ++k) {
    const uint32_t t = perm[ch.b + k];
    if (goes_left(w, cen, t)) tmp[left++] = t;
    else tmp[right++] = t;
  }
}

__global__ void k_large_copy(const Chunk* __restrict__ chunks, const LWork* __restrict__ work, const uint32_t* __restrict__ tmp,
                             uint32_t* __restrict__ perm) {
  const Chunk ch = chunks[blockIdx.x];
  if (work[ch.j].kind != KIND_SAH) return;
  for (uint32_t k = ch.b + threadIdx.x; k < ch.e; k += blockDim.x) perm[k] = tmp[k];
}

__global__ void k_large_keys(const Chunk* __restrict__ chunks, const LWork* __restrict__ work, const uint32_t* __restrict__ perm,
                             const float* __restrict__ cen, unsigned long long* __restrict__ keys) {
  const Chunk ch = chunks[blockIdx.x];
  const LWork& w = work[ch.j];
  if (w.kind != KIND_MEDIAN) return;
  for (uint32_t k = ch.b + threadIdx.x; k < ch.e; k += blockDim.x) keys[k] = median_key(cen, perm[k], w.axis);
}

__global__ void k_large_unkey(const Chunk* __restrict__ chunks, const LWork* __restrict__ work,
                              const unsigned long long* __restrict__ keys, uint32_t* __restrict__ perm) {
  const Chunk ch = chunks[blockIdx.x];
  if (work[ch.j].kind != KIND_MEDIAN) return;
  for (uint32_t k = ch.b + threadIdx.x; k < ch.e; k += blockDim.x) perm[k] = (uint32_t)keys[k];
}

// ---- the records ----

// Leaves mark their first position; node groups are counted.
__global__ void k_classify(const Seg* __restrict__ segs, uint32_t n, uint32_t* __restrict__ mark, uint32_t* __restrict__ node_n) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const Seg g = segs[s];
  const uint32_t len = g.e - g.b;
  if (len <= LEAF_TRIS) mark[g.b] = 1;
  else if ((g.depth & 1u) == 0) atomicAdd(node_n, 1u);
}

// Node groups list (range end, range length), their postorder key; `slot` counts up to the
// number k_classify counted.
__global__ void k_node_list(const Seg* __restrict__ segs, uint32_t n, unsigned long long* __restrict__ node_key,
                            uint32_t* __restrict__ node_seg, uint32_t* __restrict__ slot) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const Seg g = segs[s];
  const uint32_t len = g.e - g.b;
  if (len <= LEAF_TRIS || (g.depth & 1u)) return;
  const uint32_t q = atomicAdd(slot, 1u);
  node_key[q] = (unsigned long long)g.e << 32 | len;
  node_seg[q] = s;
}

__global__ void k_node_ids(const uint32_t* __restrict__ sorted_seg, uint32_t n, uint32_t* __restrict__ id) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n) id[sorted_seg[r]] = r;
}

// near_field.rs:380-401: a leaf's index span and source offset.
__global__ void k_leaves(const Seg* __restrict__ segs, uint32_t n, const uint32_t* __restrict__ leaf_rank,
                         const uint32_t* __restrict__ perm, uint32_t* __restrict__ id, uint32_t* __restrict__ leaves,
                         uint32_t* __restrict__ leaf_source) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const Seg g = segs[s];
  if (g.e - g.b > LEAF_TRIS) return;
  const uint32_t l = leaf_rank[g.b];
  id[s] = l | LEAF;
  leaves[2 * (size_t)l] = 3 * g.b;
  leaves[2 * (size_t)l + 1] = 3 * (g.e - g.b);
  leaf_source[l] = 3 * perm[g.b];
}

__global__ void k_indices(const uint32_t* __restrict__ perm, const uint32_t* __restrict__ idx, uint32_t nt,
                          uint32_t* __restrict__ out) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nt) return;
  const uint32_t t = perm[k];
  for (int j = 0; j < 3; ++j) out[3 * (size_t)k + j] = idx[3 * (size_t)t + j];
}

// Each leaf and node group joins its owner's children.
__global__ void k_link(const Seg* __restrict__ segs, uint32_t n, const uint32_t* __restrict__ id, uint32_t* __restrict__ kid_n,
                       uint32_t* __restrict__ kid_b, uint32_t* __restrict__ kid_id) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s == 0 || s >= n || id[s] == EMPTY) return;
  const uint32_t o = id[segs[s].owner];
  const uint32_t q = atomicAdd(&kid_n[o], 1u);
  if (q >= 4) return;  // a node group has two to four children; never more
  kid_b[4 * (size_t)o + q] = segs[s].b;
  kid_id[4 * (size_t)o + q] = id[s];
}

// A node's child slots in range order.
__global__ void k_node_children(uint32_t n, const uint32_t* __restrict__ kid_n, const uint32_t* __restrict__ kid_b,
                                const uint32_t* __restrict__ kid_id, uint32_t* __restrict__ nodes) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const uint32_t m = min(kid_n[r], 4u);
  uint32_t b[4], c[4];
  for (uint32_t q = 0; q < m; ++q) b[q] = kid_b[4 * (size_t)r + q], c[q] = kid_id[4 * (size_t)r + q];
  for (uint32_t q = 1; q < m; ++q)
    for (uint32_t p = q; p > 0 && b[p - 1] > b[p]; --p) {
      const uint32_t tb = b[p], tc = c[p];
      b[p] = b[p - 1], c[p] = c[p - 1];
      b[p - 1] = tb, c[p - 1] = tc;
    }
  for (uint32_t q = 0; q < 4; ++q) nodes[16 * (size_t)r + 6 + q] = q < m ? c[q] : EMPTY;
}

// Quantises the node groups of one level (their node children are a level pair deeper, done).
__global__ void k_quantize_level(const Seg* __restrict__ segs, uint32_t lv0, uint32_t width, const uint32_t* __restrict__ id,
                                 View v) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= width) return;
  const Seg g = segs[lv0 + i];
  if (g.e - g.b <= LEAF_TRIS || (g.depth & 1u)) return;
  uint32_t* w = v.w + v.nodes + 16 * (size_t)id[lv0 + i];
  uint32_t kids[4];
  Box boxes[4];
  int m = 0;
  for (int s = 0; s < 4; ++s) {
    const uint32_t c = w[6 + s];
    if (c == EMPTY) continue;
    kids[m] = c;
    boxes[m] = child_box(v, c);
    ++m;
  }
  quantize(w, kids, boxes, m);
}

// Device memory for one build, carved out of one allocation; freed once the build's stream has
// drained (an early error return may leave work in flight).
class Arena {
 public:
  explicit Arena(cudaStream_t s) : stream_(s) {}
  ~Arena() {
    if (base_) {
      cudaStreamSynchronize(stream_);
      cudaFree(base_);
    }
  }
  template <class T>
  T* take(size_t n) {
    const size_t at = used_;
    used_ += (n * sizeof(T) + 255) & ~(size_t)255;
    return reinterpret_cast<T*>(static_cast<char*>(base_) + at);
  }
  template <class T>
  void plan(size_t n) { size_ += (n * sizeof(T) + 255) & ~(size_t)255; }
  cudaError_t allocate() { return cudaMalloc(&base_, size_); }

 private:
  cudaStream_t stream_;
  void* base_ = nullptr;
  size_t size_ = 0, used_ = 0;
};

struct Joiner {  // joins its thread on every return path
  std::thread t;
  explicit Joiner(std::thread&& x) : t(std::move(x)) {}
  ~Joiner() { join(); }
  void join() {
    if (t.joinable()) t.join();
  }
};

struct StreamGuard {
  cudaStream_t s = nullptr;
  ~StreamGuard() {
    if (s) cudaStreamDestroy(s);
  }
};

inline uint32_t blocks(size_t n, uint32_t t) { return (uint32_t)((n + t - 1) / t); }

}  // namespace

rt_status rt_blas_build_device(rt_ctx* ctx, const float* positions, uint32_t n_positions, const uint32_t* indices,
                               uint32_t n_indices, uint32_t build_flags, rt_blas** out) {
  if (!ctx || !positions || !indices || !out) return fail(ctx, RT_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  // build_blas's checks (near_field.rs:208-214)
  if (n_indices == 0 || n_indices % 3 != 0) return fail(ctx, RT_ERR_INVALID_ARG, "BVH geometry needs a nonempty triangle list");
  const uint32_t nt = n_indices / 3;
  if (nt > MAX_TRIANGLES) return fail(ctx, RT_ERR_INVALID_ARG, "the device build takes at most 2^29 triangles");
  if ((size_t)n_positions * 3 > 0xffffffffu) return fail(ctx, RT_ERR_INVALID_ARG, "the device build takes at most 2^32 / 3 positions");
  bool sah = !(build_flags & RT_BUILD_MEDIAN);

  std::lock_guard<std::mutex> lock(ctx->mu);
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  // The host BLAS's own copy of the positions and their bounds (every position, gi_bvh.rs:70),
  // formed on a second host thread while the device builds.
  auto blas = std::make_unique<rt_blas>();
  rtb::Blas& B = blas->b;
  Joiner host_part(std::thread([&B, positions, n_positions] {
    B.positions.assign(positions, positions + 3 * (size_t)n_positions);
    B.bounds = rtb::Aabb::empty();
    for (uint32_t p = 0; p < n_positions; ++p) B.bounds.grow(positions + 3 * (size_t)p);
  }));
  StreamGuard sg;
  RT_CUDA(ctx, cudaStreamCreateWithFlags(&sg.s, cudaStreamNonBlocking));
  cudaStream_t st = sg.s;

  const size_t seg_cap = 2 * (size_t)nt + 2;
  const size_t large_cap = nt / SMALL + 2, chunk_cap = nt / CHUNK + large_cap + 2;
  // CUB scratch: the largest of the scans and sorts below.
  size_t cub_bytes = 0, b = 0;
  {
    unsigned long long* u64 = nullptr;
    uint32_t* u32 = nullptr;
    RT_CUDA(ctx, cub::DeviceScan::ExclusiveSum(nullptr, b, u64, u64, (int)(seg_cap + 1), st));
    cub_bytes = std::max(cub_bytes, b);
    RT_CUDA(ctx, cub::DeviceScan::ExclusiveSum(nullptr, b, u32, u32, (int)nt + 1, st));
    cub_bytes = std::max(cub_bytes, b);
    RT_CUDA(ctx, cub::DeviceSegmentedSort::SortKeys(nullptr, b, u64, u64, (int)nt, (int)large_cap, u32, u32, st));
    cub_bytes = std::max(cub_bytes, b);
  }
  Arena ar(st);
  ar.plan<float>(3 * (size_t)n_positions);  // positions
  ar.plan<uint32_t>(n_indices);             // indices
  ar.plan<float>(3 * (size_t)nt);           // centroids
  ar.plan<uint32_t>(6 * (size_t)nt);        // triangle box keys
  ar.plan<uint32_t>(nt);                    // permutation
  ar.plan<uint32_t>(nt);                    // partition scratch
  ar.plan<Seg>(seg_cap);
  ar.plan<unsigned long long>(seg_cap + 1);  // level flags
  ar.plan<unsigned long long>(seg_cap + 1);  // their exclusive sums
  ar.plan<LargeSeg>(large_cap);
  ar.plan<Chunk>(chunk_cap);
  ar.plan<LWork>(large_cap);
  ar.plan<uint32_t>(chunk_cap);  // left-going per chunk
  ar.plan<uint32_t>(chunk_cap);  // their starts
  ar.plan<uint32_t>(large_cap);  // median sort ranges
  ar.plan<uint32_t>(large_cap);
  ar.plan<unsigned long long>(nt);  // median keys in / out
  ar.plan<unsigned long long>(nt);
  ar.plan<uint32_t>((size_t)nt + 1);  // leaf marks
  ar.plan<uint32_t>((size_t)nt + 1);  // leaf ranks
  ar.plan<uint32_t>(seg_cap);  // record id of each range
  ar.plan<uint32_t>(4);        // counters and the validation flag
  ar.plan<char>(cub_bytes);
  if (ar.allocate() != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, RT_ERR_OOM, "device build scratch for %u triangles", nt);
  }
  float* d_pos = ar.take<float>(3 * (size_t)n_positions);
  uint32_t* d_idx = ar.take<uint32_t>(n_indices);
  float* d_cen = ar.take<float>(3 * (size_t)nt);
  uint32_t* d_tbk = ar.take<uint32_t>(6 * (size_t)nt);
  uint32_t* d_perm = ar.take<uint32_t>(nt);
  uint32_t* d_tmp = ar.take<uint32_t>(nt);
  Seg* d_segs = ar.take<Seg>(seg_cap);
  unsigned long long* d_flags = ar.take<unsigned long long>(seg_cap + 1);
  unsigned long long* d_rank = ar.take<unsigned long long>(seg_cap + 1);
  LargeSeg* d_large = ar.take<LargeSeg>(large_cap);
  Chunk* d_chunks = ar.take<Chunk>(chunk_cap);
  LWork* d_work = ar.take<LWork>(large_cap);
  uint32_t* d_chunk_left = ar.take<uint32_t>(chunk_cap);
  uint32_t* d_chunk_base = ar.take<uint32_t>(chunk_cap);
  uint32_t* d_sort_begin = ar.take<uint32_t>(large_cap);
  uint32_t* d_sort_end = ar.take<uint32_t>(large_cap);
  unsigned long long* d_keys = ar.take<unsigned long long>(nt);
  unsigned long long* d_keys_out = ar.take<unsigned long long>(nt);
  uint32_t* d_mark = ar.take<uint32_t>((size_t)nt + 1);
  uint32_t* d_leaf_rank = ar.take<uint32_t>((size_t)nt + 1);
  uint32_t* d_id = ar.take<uint32_t>(seg_cap);
  uint32_t* d_count = ar.take<uint32_t>(4);
  void* d_cub = ar.take<char>(cub_bytes);

  RT_CUDA(ctx, cudaMemcpyAsync(d_pos, positions, 12 * (size_t)n_positions, cudaMemcpyHostToDevice, st));
  RT_CUDA(ctx, cudaMemcpyAsync(d_idx, indices, 4 * (size_t)n_indices, cudaMemcpyHostToDevice, st));
  RT_CUDA(ctx, cudaMemsetAsync(d_count, 0, 16, st));
  k_validate<<<4 * 148, 256, 0, st>>>(d_pos, 3 * n_positions, d_idx, n_indices, n_positions, d_count);
  uint32_t bad = 0;
  RT_CUDA(ctx, cudaMemcpyAsync(&bad, d_count, 4, cudaMemcpyDeviceToHost, st));
  RT_CUDA(ctx, cudaStreamSynchronize(st));
  if (bad) return fail(ctx, RT_ERR_INVALID_ARG, "BVH geometry has an invalid index or position");
  k_prepare<<<blocks(nt, 256), 256, 0, st>>>(d_pos, d_idx, nt, d_cen, d_tbk, d_perm);
  RT_CUDA(ctx, cudaGetLastError());

  // The level loop; an SAH tree past 15 node levels starts over with median splits.
  std::vector<std::pair<uint32_t, uint32_t>> levels;  // (first range, ranges) of each binary depth
  std::vector<LargeSeg> large;
  std::vector<Chunk> chunks;
  uint32_t total = 0;
  for (;;) {
    levels.clear();
    const Seg root{0, nt, 0, EMPTY};
    RT_CUDA(ctx, cudaMemcpyAsync(d_segs, &root, sizeof root, cudaMemcpyHostToDevice, st));
    uint32_t lv0 = 0, width = 1, depth = 0;
    bool too_deep = false;
    for (;;) {
      levels.emplace_back(lv0, width);
      k_level_flags<<<blocks(width + 1, 256), 256, 0, st>>>(d_segs + lv0, width, d_flags);
      size_t nb = 0;
      RT_CUDA(ctx, cub::DeviceScan::ExclusiveSum(nullptr, nb, d_flags, d_rank, (int)width + 1, st));
      if (nb > cub_bytes) return fail(ctx, RT_ERR_OOM, "device build: scan scratch");
      RT_CUDA(ctx, cub::DeviceScan::ExclusiveSum(d_cub, nb, d_flags, d_rank, (int)width + 1, st));
      unsigned long long totals = 0;
      RT_CUDA(ctx, cudaMemcpyAsync(&totals, d_rank + width, 8, cudaMemcpyDeviceToHost, st));
      RT_CUDA(ctx, cudaStreamSynchronize(st));
      const uint32_t pending = (uint32_t)totals, n_large = (uint32_t)(totals >> 32);
      if (pending == 0) break;
      if (sah && depth >= TOO_DEEP) {
        too_deep = true;
        break;
      }
      const uint32_t next = lv0 + width;
      if ((size_t)next + 2 * (size_t)pending > seg_cap || n_large > large_cap)
        return fail(ctx, RT_ERR_OOM, "device build: range table overflow");
      if (n_large) {
        k_large_list<<<blocks(width, 256), 256, 0, st>>>(d_segs + lv0, width, d_rank, d_large);
        large.resize(n_large);
        RT_CUDA(ctx, cudaMemcpyAsync(large.data(), d_large, n_large * sizeof(LargeSeg), cudaMemcpyDeviceToHost, st));
        RT_CUDA(ctx, cudaStreamSynchronize(st));
        chunks.clear();
        for (uint32_t j = 0; j < n_large; ++j) {
          large[j].first = (uint32_t)chunks.size();
          for (uint32_t s = large[j].b; s < large[j].e; s += std::min(CHUNK, large[j].e - s))
            chunks.push_back(Chunk{j, s, s + std::min(CHUNK, large[j].e - s)});
          large[j].n = (uint32_t)chunks.size() - large[j].first;
        }
        const uint32_t nc = (uint32_t)chunks.size();
        if (nc > chunk_cap) return fail(ctx, RT_ERR_OOM, "device build: chunk table overflow");
        RT_CUDA(ctx, cudaMemcpyAsync(d_large, large.data(), n_large * sizeof(LargeSeg), cudaMemcpyHostToDevice, st));
        RT_CUDA(ctx, cudaMemcpyAsync(d_chunks, chunks.data(), nc * sizeof(Chunk), cudaMemcpyHostToDevice, st));
        k_large_init<<<n_large, 128, 0, st>>>(d_work, n_large);
        k_large_cbox<<<nc, CHUNK_THREADS, 0, st>>>(d_chunks, d_perm, d_cen, d_work);
        if (sah) k_large_bins<<<nc, CHUNK_THREADS, 0, st>>>(d_chunks, d_perm, d_cen, d_tbk, d_work);
        k_large_choose<<<blocks(n_large, 64), 64, 0, st>>>(d_large, n_large, d_work, sah);
        k_large_count<<<nc, CHUNK_THREADS, 0, st>>>(d_chunks, d_perm, d_cen, d_work, d_chunk_left);
        k_large_scan<<<blocks(n_large, 64), 64, 0, st>>>(d_large, n_large, d_work, d_chunk_left, d_chunk_base, d_sort_begin,
                                                           d_sort_end, d_segs, lv0, next, d_rank);
        k_large_scatter<<<nc, CHUNK_THREADS, 0, st>>>(d_chunks, d_large, d_perm, d_cen, d_work, d_chunk_base, d_tmp);
        k_large_copy<<<nc, CHUNK_THREADS, 0, st>>>(d_chunks, d_work, d_tmp, d_perm);
        k_large_keys<<<nc, CHUNK_THREADS, 0, st>>>(d_chunks, d_work, d_perm, d_cen, d_keys);
        nb = 0;
        RT_CUDA(ctx, cub::DeviceSegmentedSort::SortKeys(nullptr, nb, d_keys, d_keys_out, (int)nt, (int)n_large, d_sort_begin,
                                                        d_sort_end, st));
        if (nb > cub_bytes) return fail(ctx, RT_ERR_OOM, "device build: sort scratch");
        RT_CUDA(ctx, cub::DeviceSegmentedSort::SortKeys(d_cub, nb, d_keys, d_keys_out, (int)nt, (int)n_large, d_sort_begin,
                                                        d_sort_end, st));
        k_large_unkey<<<nc, CHUNK_THREADS, 0, st>>>(d_chunks, d_work, d_keys_out, d_perm);
        RT_CUDA(ctx, cudaGetLastError());
      }
      LevelArgs a{d_segs, lv0, width, next, d_rank, d_cen, d_tbk, d_perm, sah ? 1 : 0};
      k_split_small<<<width, SMALL_THREADS, 0, st>>>(a);
      RT_CUDA(ctx, cudaGetLastError());
      lv0 = next, width = 2 * pending, ++depth;
    }
    if (!too_deep) {
      total = lv0 + width;
      break;
    }
    sah = false;  // near_field.rs:186-188
    k_prepare<<<blocks(nt, 256), 256, 0, st>>>(d_pos, d_idx, nt, d_cen, d_tbk, d_perm);
  }

  // Records: leaf ids by range start, node ids by (range end, range length), children by range
  // start, then the node boxes from the deepest node level up.
  RT_CUDA(ctx, cudaMemsetAsync(d_mark, 0, 4 * ((size_t)nt + 1), st));
  RT_CUDA(ctx, cudaMemsetAsync(d_count, 0, 16, st));
  RT_CUDA(ctx, cudaMemsetAsync(d_id, 0xff, 4 * (size_t)total, st));
  k_classify<<<blocks(total, 256), 256, 0, st>>>(d_segs, total, d_mark, d_count);
  size_t nb = 0;
  RT_CUDA(ctx, cub::DeviceScan::ExclusiveSum(nullptr, nb, d_mark, d_leaf_rank, (int)nt + 1, st));
  if (nb > cub_bytes) return fail(ctx, RT_ERR_OOM, "device build: scan scratch");
  RT_CUDA(ctx, cub::DeviceScan::ExclusiveSum(d_cub, nb, d_mark, d_leaf_rank, (int)nt + 1, st));
  uint32_t counts[2] = {0, 0};
  RT_CUDA(ctx, cudaMemcpyAsync(&counts[0], d_leaf_rank + nt, 4, cudaMemcpyDeviceToHost, st));
  RT_CUDA(ctx, cudaMemcpyAsync(&counts[1], d_count, 4, cudaMemcpyDeviceToHost, st));
  RT_CUDA(ctx, cudaStreamSynchronize(st));
  const uint32_t n_leaves = counts[0], n_nodes = counts[1];
  if (n_leaves > nt || (n_leaves && n_nodes >= n_leaves) || (!n_leaves))
    return fail(ctx, RT_ERR_OOM, "device build: record counts out of range");
  // The records, sized now that the counts are known: nodes, leaves, indices and positions in
  // one word buffer (the quantiser reads them there), then the node lists.
  const size_t out_nodes = 0, out_leaves = 16 * (size_t)n_nodes, out_indices = out_leaves + 2 * (size_t)n_leaves,
               out_positions = out_indices + 3 * (size_t)nt, out_words = out_positions + 3 * (size_t)n_positions;
  size_t sort_bytes = 0;
  {
    unsigned long long* u64 = nullptr;
    uint32_t* u32 = nullptr;
    RT_CUDA(ctx, cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, u64, u64, u32, u32, (int)std::max(n_nodes, 1u), 0, 64, st));
  }
  const size_t nn = std::max(n_nodes, 1u);
  Arena rec(st);
  rec.plan<uint32_t>(out_words);
  rec.plan<uint32_t>(n_leaves);  // leaf sources
  rec.plan<unsigned long long>(nn);  // node keys, sorted
  rec.plan<unsigned long long>(nn);
  rec.plan<uint32_t>(nn);  // node ranges, sorted
  rec.plan<uint32_t>(nn);
  rec.plan<uint32_t>(nn);  // children per node
  rec.plan<uint32_t>(4 * nn);
  rec.plan<uint32_t>(4 * nn);
  rec.plan<char>(sort_bytes);
  if (rec.allocate() != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, RT_ERR_OOM, "device build records for %u triangles", nt);
  }
  uint32_t* d_out = rec.take<uint32_t>(out_words);
  uint32_t* d_leaf_source = rec.take<uint32_t>(n_leaves);
  unsigned long long* d_node_key = rec.take<unsigned long long>(nn);
  unsigned long long* d_node_key_sorted = rec.take<unsigned long long>(nn);
  uint32_t* d_node_seg = rec.take<uint32_t>(nn);
  uint32_t* d_node_seg_sorted = rec.take<uint32_t>(nn);
  uint32_t* d_kid_n = rec.take<uint32_t>(nn);
  uint32_t* d_kid_b = rec.take<uint32_t>(4 * nn);
  uint32_t* d_kid_id = rec.take<uint32_t>(4 * nn);
  void* d_sort = rec.take<char>(sort_bytes);
  uint32_t* d_nodes = d_out + out_nodes;
  uint32_t* d_leaves = d_out + out_leaves;
  if (n_nodes) {
    k_node_list<<<blocks(total, 256), 256, 0, st>>>(d_segs, total, d_node_key, d_node_seg, d_count + 1);
    nb = sort_bytes;
    RT_CUDA(ctx, cub::DeviceRadixSort::SortPairs(d_sort, nb, d_node_key, d_node_key_sorted, d_node_seg, d_node_seg_sorted,
                                                 (int)n_nodes, 0, 64, st));
    k_node_ids<<<blocks(n_nodes, 256), 256, 0, st>>>(d_node_seg_sorted, n_nodes, d_id);
  }
  k_leaves<<<blocks(total, 256), 256, 0, st>>>(d_segs, total, d_leaf_rank, d_perm, d_id, d_leaves, d_leaf_source);
  k_indices<<<blocks(nt, 256), 256, 0, st>>>(d_perm, d_idx, nt, d_out + out_indices);
  RT_CUDA(ctx, cudaMemcpyAsync(d_out + out_positions, d_pos, 12 * (size_t)n_positions, cudaMemcpyDeviceToDevice, st));
  if (n_nodes) {
    RT_CUDA(ctx, cudaMemsetAsync(d_kid_n, 0, 4 * (size_t)n_nodes, st));
    k_link<<<blocks(total, 256), 256, 0, st>>>(d_segs, total, d_id, d_kid_n, d_kid_b, d_kid_id);
    k_node_children<<<blocks(n_nodes, 256), 256, 0, st>>>(n_nodes, d_kid_n, d_kid_b, d_kid_id, d_nodes);
    View v{};
    v.w = d_out, v.layout = 0, v.nodes = out_nodes, v.leaves = out_leaves, v.indices = out_indices,
    v.positions = out_positions;
    for (size_t d = levels.size(); d-- > 0;) {
      if (d & 1) continue;
      const uint32_t lv0 = levels[d].first, width = levels[d].second;
      k_quantize_level<<<blocks(width, 128), 128, 0, st>>>(d_segs, lv0, width, d_id, v);
    }
  }
  RT_CUDA(ctx, cudaGetLastError());

  B.nodes.resize(16 * (size_t)n_nodes);
  B.leaves.resize(2 * (size_t)n_leaves);
  B.indices.resize(n_indices);
  B.leaf_source.resize(n_leaves);
  if (n_nodes) RT_CUDA(ctx, cudaMemcpyAsync(B.nodes.data(), d_nodes, 64 * (size_t)n_nodes, cudaMemcpyDeviceToHost, st));
  RT_CUDA(ctx, cudaMemcpyAsync(B.leaves.data(), d_leaves, 8 * (size_t)n_leaves, cudaMemcpyDeviceToHost, st));
  RT_CUDA(ctx, cudaMemcpyAsync(B.indices.data(), d_out + out_indices, 4 * (size_t)n_indices, cudaMemcpyDeviceToHost, st));
  RT_CUDA(ctx, cudaMemcpyAsync(B.leaf_source.data(), d_leaf_source, 4 * (size_t)n_leaves, cudaMemcpyDeviceToHost, st));
  RT_CUDA(ctx, cudaStreamSynchronize(st));
  B.root = n_nodes ? n_nodes - 1 : LEAF;  // postorder puts the root last; a one-leaf mesh is leaf 0
  host_part.join();
  *out = blas.release();
  return RT_OK;
}
