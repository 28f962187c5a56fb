// GPU build of the instance top level (instance_bvh::build, src/instance_bvh.rs:346-460) whose
// node words equal the host builder's (host/tlas.cpp), word for word.
//
// The reference splits a set of instances by 16-bin SAH over the box centres (lo + hi), or at the
// median of (centre, index), down to single instances. Its halves are sets: a split's outcome
// depends on which instances a range holds, not on their order (leaves hold one instance each).
// So all ranges of one binary depth split at once here, in any order, with min/max reductions
// through order-preserving keys (which can differ from the host's only in the sign of a zero bound,
// and that changes no bin or cost comparison). The binary boxes are then grown bottom-up in the
// host's child order, the binary tree is collapsed into BVH4 nodes top-down with the reference's
// largest-area-first rule (instance_bvh.rs:370-401), and each node gets its preorder id from the
// subtree sizes below it. An SAH tree too deep for the 48-entry stack (1 + 3 * levels > 48) is
// built again by median splits (instance_bvh.rs:346-366). A BVH4 level descends at most three
// binary levels, so a range still splitting at binary depth 48 already implies that.
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>
#include <cub/device/device_segmented_sort.cuh>

#include <algorithm>
#include <vector>

#include "ctx.hpp"
#include "kernels/bvh4_quant.cuh"
#include "kernels/order_keys.cuh"

using namespace rtc;

namespace {

using rtk::EMPTY;
using rtk::LEAF;
using rtq::hi_of;
using rtq::lo_of;
using rtq::okey;
using rtq::order_key;
using rtq::unkey;

constexpr uint32_t BINS = 16;         // instance_bvh.rs: BINS
constexpr uint32_t NODE_WORDS = 32;
constexpr uint32_t THREADS = 256;
constexpr uint32_t PER = 8;           // elements a thread takes of one partition tile
constexpr uint32_t SORT_SMALL = 4096; // a median range up to this size sorts in shared memory
constexpr uint32_t DEEP_BINARY = 48;  // a range splitting at this binary depth means > 15 BVH4 levels
constexpr int KIND_MEDIAN = 0, KIND_SAH = 1;

struct Seg {          // a range [b, e) of the instance permutation
  uint32_t b, e;
  uint32_t child;     // its first child range (the second follows), or EMPTY for one instance
  uint32_t pad;
};

__device__ __forceinline__ float area(const float* lo, const float* hi) {  // instance_bvh.rs:290-293
  const float e0 = hi_of(__fsub_rn(hi[0], lo[0]), 0.0f), e1 = hi_of(__fsub_rn(hi[1], lo[1]), 0.0f),
              e2 = hi_of(__fsub_rn(hi[2], lo[2]), 0.0f);
  return __fadd_rn(__fadd_rn(__fmul_rn(e0, e1), __fmul_rn(e1, e2)), __fmul_rn(e2, e0));
}
// ((centre - base) * scale) as usize, at most 15 (instance_bvh.rs:310-312, 427-430)
__device__ __forceinline__ uint32_t bin_of(float c, float base, float scale) {
  const float f = __fmul_rn(__fsub_rn(c, base), scale);
  if (!(f > 0.0f)) return 0;
  return f >= (float)(BINS - 1) ? BINS - 1 : (uint32_t)f;
}

struct BoxWords {  // instance i's box: lo xyz at w[i * stride], hi xyz right after
  const uint32_t* w;
  size_t stride;
  __device__ float lo(uint32_t i, int a) const { return __uint_as_float(w[i * stride + a]); }
  __device__ float hi(uint32_t i, int a) const { return __uint_as_float(w[i * stride + 3 + a]); }
  __device__ float centre(uint32_t i, int a) const { return __fadd_rn(lo(i, a), hi(i, a)); }
};

struct Choice {
  int kind, axis, bin;
};

// instance_bvh.rs:298-342: the cheapest plane over 16 bins a axis (ties: lower axis, lower bin),
// cost area(L) n(L) + area(R) n(R); else the median on the axis of largest centre extent.
__device__ Choice choose(const float* lo, const float* hi, const uint32_t* cnt, const uint32_t* bl, const uint32_t* bh,
                         bool sah) {
  bool found = false;
  float best = 0.0f;
  Choice c{KIND_SAH, 0, 0};
  for (int axis = 0; sah && axis < 3; ++axis) {
    if (!(__fsub_rn(hi[axis], lo[axis]) > 0.0f)) continue;
    const uint32_t* n = cnt + axis * BINS;
    const uint32_t* l = bl + axis * BINS * 3;
    const uint32_t* h = bh + axis * BINS * 3;
    float ra[BINS];
    uint32_t rn[BINS];
    float al[3] = {INFINITY, INFINITY, INFINITY}, ah[3] = {-INFINITY, -INFINITY, -INFINITY};
    uint32_t m = 0;
    for (int b = BINS - 1; b >= 1; --b) {
      if (n[b])
        for (int a = 0; a < 3; ++a) al[a] = lo_of(al[a], unkey(l[3 * b + a])), ah[a] = hi_of(ah[a], unkey(h[3 * b + a]));
      m += n[b];
      ra[b - 1] = area(al, ah);
      rn[b - 1] = m;
    }
    for (int a = 0; a < 3; ++a) al[a] = INFINITY, ah[a] = -INFINITY;
    m = 0;
    for (int b = 0; b < (int)BINS - 1; ++b) {
      if (n[b])
        for (int a = 0; a < 3; ++a) al[a] = lo_of(al[a], unkey(l[3 * b + a])), ah[a] = hi_of(ah[a], unkey(h[3 * b + a]));
      m += n[b];
      if (m == 0 || rn[b] == 0) continue;
      const float cost = __fadd_rn(__fmul_rn(area(al, ah), (float)m), __fmul_rn(ra[b], (float)rn[b]));
      if (!found || cost < best) found = true, best = cost, c.axis = axis, c.bin = b;
    }
  }
  if (found) return c;
  c.kind = KIND_MEDIAN;
  c.axis = 0;
  for (int a = 1; a < 3; ++a)
    if (order_key(__fsub_rn(hi[a], lo[a])) >= order_key(__fsub_rn(hi[c.axis], lo[c.axis]))) c.axis = a;
  return c;
}

__global__ void k_identity(uint32_t* __restrict__ ids, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) ids[i] = i;
}

__global__ void k_flags(const Seg* __restrict__ segs, uint32_t width, uint32_t* __restrict__ flags) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < width) flags[i] = segs[i].e - segs[i].b >= 2 ? 1u : 0u;
  else if (i == width) flags[i] = 0;
}

struct SplitArgs {
  Seg* segs;
  uint32_t lv0, next;
  const uint32_t* rank;
  BoxWords box;
  uint32_t* ids;
  uint32_t* tmp;
  unsigned long long* keys;
  uint32_t* sort_begin;  // per range of the level: the median range to sort after the launch
  uint32_t* sort_end;
  uint32_t* n_sorts;     // ranges that set one
  int sah;
};

// One block splits one range of any size: its centre box, SAH bins, the choice, then a stable
// partition by tiles, or a median sort (in shared memory up to SORT_SMALL, else after the launch).
__global__ void __launch_bounds__(THREADS) k_split(SplitArgs a) {
  const uint32_t i = blockIdx.x, tid = threadIdx.x, nth = blockDim.x;
  Seg* g = a.segs + a.lv0 + i;
  const uint32_t b = g->b, e = g->e, len = e - b;
  if (tid == 0) a.sort_begin[i] = a.sort_end[i] = 0;
  if (len < 2) return;
  __shared__ unsigned long long skey[SORT_SMALL];
  __shared__ uint32_t cb[6], cnt[3 * BINS], bl[3 * BINS * 3], bh[3 * BINS * 3], runs[THREADS];
  __shared__ uint32_t total_left, tile_left;
  __shared__ Choice choice;
  if (tid < 3) cb[tid] = 0xffffffffu, cb[3 + tid] = 0u;
  if (tid == 0) total_left = 0;
  for (uint32_t k = tid; k < 3 * BINS * 3; k += nth) {
    bl[k] = 0xffffffffu, bh[k] = 0u;
    if (k < 3 * BINS) cnt[k] = 0;
  }
  __syncthreads();
  uint32_t l[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, h[3] = {0u, 0u, 0u};
  for (uint32_t k = tid; k < len; k += nth) {
    const uint32_t id = a.ids[b + k];
    for (int x = 0; x < 3; ++x) {
      const uint32_t v = okey(a.box.centre(id, x));
      l[x] = min(l[x], v), h[x] = max(h[x], v);
    }
  }
  for (int x = 0; x < 3; ++x) atomicMin(&cb[x], l[x]), atomicMax(&cb[3 + x], h[x]);
  __syncthreads();
  float lo[3], hi[3], scale[3];
  for (int x = 0; x < 3; ++x) {
    lo[x] = unkey(cb[x]), hi[x] = unkey(cb[3 + x]);
    scale[x] = __fdiv_rn((float)BINS, __fsub_rn(hi[x], lo[x]));
  }
  if (a.sah) {
    for (uint32_t k = tid; k < len; k += nth) {
      const uint32_t id = a.ids[b + k];
      for (int axis = 0; axis < 3; ++axis) {
        if (!(__fsub_rn(hi[axis], lo[axis]) > 0.0f)) continue;
        const uint32_t q = axis * BINS + bin_of(a.box.centre(id, axis), lo[axis], scale[axis]);
        atomicAdd(&cnt[q], 1u);
        for (int x = 0; x < 3; ++x) atomicMin(&bl[3 * q + x], okey(a.box.lo(id, x))), atomicMax(&bh[3 * q + x], okey(a.box.hi(id, x)));
      }
    }
    __syncthreads();
  }
  if (tid == 0) choice = choose(lo, hi, cnt, bl, bh, a.sah != 0);
  __syncthreads();
  const Choice c = choice;
  uint32_t mid;
  if (c.kind == KIND_SAH) {
    const float base = lo[c.axis], sc = scale[c.axis];
    uint32_t m = 0;
    for (uint32_t k = tid; k < len; k += nth) m += bin_of(a.box.centre(a.ids[b + k], c.axis), base, sc) <= (uint32_t)c.bin;
    atomicAdd(&total_left, m);
    __syncthreads();
    const uint32_t L = total_left;
    uint32_t before = 0;  // left-going instances of the earlier tiles
    for (uint32_t t0 = 0; t0 < len; t0 += nth * PER) {
      const uint32_t r0 = min(len, t0 + tid * PER), r1 = min(len, r0 + PER);
      uint32_t cl = 0;
      for (uint32_t k = r0; k < r1; ++k) cl += bin_of(a.box.centre(a.ids[b + k], c.axis), base, sc) <= (uint32_t)c.bin;
      runs[tid] = cl;
      __syncthreads();
      if (tid == 0) {
        uint32_t s = 0;
        for (uint32_t j = 0; j < nth; ++j) {
          const uint32_t v = runs[j];
          runs[j] = s;
          s += v;
        }
        tile_left = s;
      }
      __syncthreads();
      uint32_t lp = b + before + runs[tid];
      uint32_t rp = b + L + (t0 - before) + ((r0 - t0) - runs[tid]);
      for (uint32_t k = r0; k < r1; ++k) {
        const uint32_t id = a.ids[b + k];
        if (bin_of(a.box.centre(id, c.axis), base, sc) <= (uint32_t)c.bin) a.tmp[lp++] = id;
        else a.tmp[rp++] = id;
      }
      before += tile_left;
      __syncthreads();
    }
    for (uint32_t k = tid; k < len; k += nth) a.ids[b + k] = a.tmp[b + k];
    mid = b + L;
  } else if (len <= SORT_SMALL) {  // bitonic sort of (centre key, index), padded to a power of two
    uint32_t n2 = 1;
    while (n2 < len) n2 <<= 1;
    for (uint32_t k = tid; k < n2; k += nth) {
      if (k < len) {
        const uint32_t id = a.ids[b + k];
        skey[k] = (unsigned long long)okey(a.box.centre(id, c.axis)) << 32 | id;
      } else {
        skey[k] = ~0ull;
      }
    }
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
    for (uint32_t k = tid; k < len; k += nth) a.ids[b + k] = (uint32_t)skey[k];
    mid = b + len / 2;
  } else {  // keys now, sorted by the segmented sort after this launch
    for (uint32_t k = tid; k < len; k += nth) {
      const uint32_t id = a.ids[b + k];
      a.keys[b + k] = (unsigned long long)okey(a.box.centre(id, c.axis)) << 32 | id;
    }
    if (tid == 0) a.sort_begin[i] = b, a.sort_end[i] = e, atomicAdd(a.n_sorts, 1u);
    mid = b + len / 2;
  }
  if (tid == 0) {
    const uint32_t r = a.next + 2 * a.rank[i];
    g->child = r;
    a.segs[r] = Seg{b, mid, EMPTY, 0};
    a.segs[r + 1] = Seg{mid, e, EMPTY, 0};
  }
}

__global__ void k_unkey(const uint32_t* __restrict__ sort_begin, const uint32_t* __restrict__ sort_end,
                        const unsigned long long* __restrict__ keys, uint32_t* __restrict__ ids) {
  const uint32_t i = blockIdx.x;
  for (uint32_t k = sort_begin[i] + threadIdx.x; k < sort_end[i]; k += blockDim.x) ids[k] = (uint32_t)keys[k];
}

// A binary level's boxes: one instance's own box, else the union of the two children's, grown
// first then second from the empty box (instance_bvh.rs:450-458).
__global__ void k_boxes(const Seg* __restrict__ segs, uint32_t lv0, uint32_t width, const uint32_t* __restrict__ ids,
                        BoxWords box, float* __restrict__ sbox) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= width) return;
  const uint32_t s = lv0 + i;
  const Seg g = segs[s];
  float* o = sbox + 6 * (size_t)s;
  if (g.e - g.b == 1) {
    const uint32_t id = ids[g.b];
    for (int a = 0; a < 3; ++a) o[a] = box.lo(id, a), o[3 + a] = box.hi(id, a);
    return;
  }
  const float* p = sbox + 6 * (size_t)g.child;
  const float* q = sbox + 6 * (size_t)(g.child + 1);
  for (int a = 0; a < 3; ++a) {
    o[a] = lo_of(lo_of(INFINITY, p[a]), q[a]);
    o[3 + a] = hi_of(hi_of(-INFINITY, p[3 + a]), q[3 + a]);
  }
}

__device__ __forceinline__ bool inner(const Seg* segs, uint32_t s) { return segs[s].e - segs[s].b >= 2; }
__device__ __forceinline__ int32_t area_key(const float* sbox, uint32_t s) {
  return order_key(area(sbox + 6 * (size_t)s, sbox + 6 * (size_t)s + 3));
}

// instance_bvh.rs:370-401: a node's kids start as its binary children; the largest-area inner
// kid (ties: the earlier slot) is replaced by its own two until there are four. Inner kids make
// the next level.
__global__ void k_collapse(const Seg* __restrict__ segs, const float* __restrict__ sbox, uint32_t* __restrict__ list,
                           uint32_t first, uint32_t count, uint32_t* __restrict__ next_n, uint32_t* __restrict__ kids) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const uint32_t x = list[first + i];
  uint32_t k[4] = {segs[x].child, segs[x].child + 1, EMPTY, EMPTY};
  int m = 2;
  while (m < 4) {
    int pick = -1;
    for (int j = 0; j < m; ++j)
      if (inner(segs, k[j]) && (pick < 0 || area_key(sbox, k[j]) > area_key(sbox, k[pick]))) pick = j;
    if (pick < 0) break;
    const uint32_t id = k[pick];
    for (int j = m; j > pick + 1; --j) k[j] = k[j - 1];
    k[pick] = segs[id].child;
    k[pick + 1] = segs[id].child + 1;
    ++m;
  }
  for (int j = 0; j < 4; ++j) {
    kids[4 * (size_t)x + j] = j < m ? k[j] : EMPTY;
    if (j < m && inner(segs, k[j])) list[first + count + atomicAdd(next_n, 1u)] = k[j];
  }
}

// Subtree sizes in BVH4 nodes, one level, deepest first.
__global__ void k_sizes(const Seg* __restrict__ segs, const uint32_t* __restrict__ list, uint32_t first, uint32_t count,
                        const uint32_t* __restrict__ kids, uint32_t* __restrict__ size) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const uint32_t x = list[first + i];
  uint32_t s = 1;
  for (int j = 0; j < 4; ++j) {
    const uint32_t c = kids[4 * (size_t)x + j];
    if (c != EMPTY && inner(segs, c)) s += size[c];
  }
  size[x] = s;
}

// Preorder ids, one level, root first: a node's inner kids follow it in slot order, each after
// the subtrees of the kids before it.
__global__ void k_ids(const Seg* __restrict__ segs, const uint32_t* __restrict__ list, uint32_t first, uint32_t count,
                      const uint32_t* __restrict__ kids, const uint32_t* __restrict__ size, uint32_t* __restrict__ id) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const uint32_t x = list[first + i];
  uint32_t r = id[x] + 1;
  for (int j = 0; j < 4; ++j) {
    const uint32_t c = kids[4 * (size_t)x + j];
    if (c != EMPTY && inner(segs, c)) id[c] = r, r += size[c];
  }
}

// The node words (instance_bvh.rs:270-275): child boxes axis-major, child ids (LEAF | instance
// or a node id), EMPTY for an unused slot, whose box words stay 0.
__global__ void k_words(const Seg* __restrict__ segs, const uint32_t* __restrict__ list, uint32_t first, uint32_t count,
                        const uint32_t* __restrict__ kids, const uint32_t* __restrict__ id, const uint32_t* __restrict__ ids,
                        const float* __restrict__ sbox, uint32_t* __restrict__ out, uint32_t* __restrict__ order_at) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const uint32_t x = list[first + i];
  uint32_t* w = out + NODE_WORDS * (size_t)id[x];
  for (int c = 0; c < 4; ++c) {
    const uint32_t k = kids[4 * (size_t)x + c];
    if (k == EMPTY) {
      w[24 + c] = EMPTY;
      continue;
    }
    const float* bx = sbox + 6 * (size_t)k;
    for (int a = 0; a < 3; ++a) w[4 * a + c] = __float_as_uint(bx[a]), w[12 + 4 * a + c] = __float_as_uint(bx[3 + a]);
    w[24 + c] = inner(segs, k) ? id[k] : (LEAF | ids[segs[k].b]);
  }
  if (order_at) order_at[i] = id[x];
}

class Scratch {
 public:
  explicit Scratch(cudaStream_t s) : s_(s) {}
  ~Scratch() {
    if (base_) {
      cudaStreamSynchronize(s_);
      cudaFree(base_);
    }
  }
  template <class T>
  void plan(size_t n) { size_ += (n * sizeof(T) + 255) & ~(size_t)255; }
  template <class T>
  T* take(size_t n) {
    T* p = reinterpret_cast<T*>(static_cast<char*>(base_) + used_);
    used_ += (n * sizeof(T) + 255) & ~(size_t)255;
    return p;
  }
  cudaError_t allocate() { return cudaMalloc(&base_, size_); }

 private:
  cudaStream_t s_;
  void* base_ = nullptr;
  size_t size_ = 0, used_ = 0;
};

inline uint32_t grid(size_t n, uint32_t t) { return (uint32_t)((n + t - 1) / t); }

}  // namespace

namespace rtc {

rt_status tlas_build_device(rt_ctx* ctx, const uint32_t* d_box_words, size_t stride, uint32_t n, bool sah, uint32_t* d_out,
                            size_t cap_words, uint32_t* d_order, std::vector<uint32_t>* level_start, uint32_t* n_nodes,
                            cudaStream_t st) {
  if (n < 2) return fail(ctx, RT_ERR_INVALID_ARG, "a top level needs two instances");
  if ((size_t)n - 1 > cap_words / NODE_WORDS) return fail(ctx, RT_ERR_INVALID_ARG, "top-level words too small");
  if (n > (1u << 29)) return fail(ctx, RT_ERR_INVALID_ARG, "the device top-level build takes at most 2^29 instances");
  const BoxWords box{d_box_words, stride};
  const size_t seg_cap = 2 * (size_t)n;  // a full binary tree over n leaves has 2n - 1 ranges
  size_t scan_bytes = 0, sort_bytes = 0;
  {
    uint32_t* u32 = nullptr;
    unsigned long long* u64 = nullptr;
    RT_CUDA(ctx, cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, u32, u32, (int)(seg_cap + 1), st));
    RT_CUDA(ctx, cub::DeviceSegmentedSort::SortKeys(nullptr, sort_bytes, u64, u64, (int)n, (int)seg_cap, u32, u32, st));
  }
  Scratch sc(st);
  sc.plan<uint32_t>(n);                  // instance permutation
  sc.plan<uint32_t>(n);                  // partition scratch
  sc.plan<Seg>(seg_cap);
  sc.plan<uint32_t>(seg_cap + 1);        // level flags
  sc.plan<uint32_t>(seg_cap + 1);        // their exclusive sums
  sc.plan<uint32_t>(seg_cap);            // median sort ranges
  sc.plan<uint32_t>(seg_cap);
  sc.plan<unsigned long long>(n);        // median keys in / out
  sc.plan<unsigned long long>(n);
  sc.plan<float>(6 * seg_cap);           // range boxes
  sc.plan<uint32_t>(n);                  // BVH4 nodes by level (ranges)
  sc.plan<uint32_t>(4 * seg_cap);        // their kids
  sc.plan<uint32_t>(seg_cap);            // subtree sizes
  sc.plan<uint32_t>(seg_cap);            // node ids
  sc.plan<uint32_t>(4);                  // counter
  sc.plan<char>(std::max(scan_bytes, sort_bytes));
  if (sc.allocate() != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, RT_ERR_OOM, "top-level build scratch for %u instances", n);
  }
  uint32_t* d_ids = sc.take<uint32_t>(n);
  uint32_t* d_tmp = sc.take<uint32_t>(n);
  Seg* d_segs = sc.take<Seg>(seg_cap);
  uint32_t* d_flags = sc.take<uint32_t>(seg_cap + 1);
  uint32_t* d_rank = sc.take<uint32_t>(seg_cap + 1);
  uint32_t* d_sort_begin = sc.take<uint32_t>(seg_cap);
  uint32_t* d_sort_end = sc.take<uint32_t>(seg_cap);
  unsigned long long* d_keys = sc.take<unsigned long long>(n);
  unsigned long long* d_keys_out = sc.take<unsigned long long>(n);
  float* d_sbox = sc.take<float>(6 * seg_cap);
  uint32_t* d_list = sc.take<uint32_t>(n);
  uint32_t* d_kids = sc.take<uint32_t>(4 * seg_cap);
  uint32_t* d_size = sc.take<uint32_t>(seg_cap);
  uint32_t* d_id = sc.take<uint32_t>(seg_cap);
  uint32_t* d_count = sc.take<uint32_t>(4);
  void* d_tmp_bytes = sc.take<char>(std::max(scan_bytes, sort_bytes));

  std::vector<std::pair<uint32_t, uint32_t>> levels;  // binary levels: (first range, ranges)
  std::vector<uint32_t> wide;                         // BVH4 levels: starts in d_list
  for (;;) {
    // Binary splits, level by level. A level's median sorts past SORT_SMALL run after the next
    // level's flags are counted (they need only the ranges), before its splits.
    levels.clear();
    k_identity<<<grid(n, 256), 256, 0, st>>>(d_ids, n);
    const Seg root{0, n, EMPTY, 0};
    RT_CUDA(ctx, cudaMemcpyAsync(d_segs, &root, sizeof root, cudaMemcpyHostToDevice, st));
    uint32_t lv0 = 0, width = 1, depth = 0, pending_sort = 0;
    RT_CUDA(ctx, cudaMemsetAsync(d_count, 0, 16, st));
    bool too_deep = false;
    for (;;) {
      levels.emplace_back(lv0, width);
      k_flags<<<grid(width + 1, 256), 256, 0, st>>>(d_segs + lv0, width, d_flags);
      size_t nb = 0;
      RT_CUDA(ctx, cub::DeviceScan::ExclusiveSum(nullptr, nb, d_flags, d_rank, (int)width + 1, st));
      if (nb > scan_bytes) return fail(ctx, RT_ERR_OOM, "top-level build: scan scratch");
      RT_CUDA(ctx, cub::DeviceScan::ExclusiveSum(d_tmp_bytes, nb, d_flags, d_rank, (int)width + 1, st));
      uint32_t pending = 0, sorts = 0;
      RT_CUDA(ctx, cudaMemcpyAsync(&pending, d_rank + width, 4, cudaMemcpyDeviceToHost, st));
      RT_CUDA(ctx, cudaMemcpyAsync(&sorts, d_count + 1, 4, cudaMemcpyDeviceToHost, st));
      RT_CUDA(ctx, cudaStreamSynchronize(st));
      if (pending_sort && sorts) {  // the previous level's large median ranges
        nb = 0;
        RT_CUDA(ctx, cub::DeviceSegmentedSort::SortKeys(nullptr, nb, d_keys, d_keys_out, (int)n, (int)pending_sort,
                                                        d_sort_begin, d_sort_end, st));
        if (nb > sort_bytes) return fail(ctx, RT_ERR_OOM, "top-level build: sort scratch");
        RT_CUDA(ctx, cub::DeviceSegmentedSort::SortKeys(d_tmp_bytes, nb, d_keys, d_keys_out, (int)n, (int)pending_sort,
                                                        d_sort_begin, d_sort_end, st));
        k_unkey<<<pending_sort, 256, 0, st>>>(d_sort_begin, d_sort_end, d_keys_out, d_ids);
      }
      pending_sort = 0;
      if (pending == 0) break;
      if (sah && depth >= DEEP_BINARY) {
        too_deep = true;
        break;
      }
      const uint32_t next = lv0 + width;
      if ((size_t)next + 2 * (size_t)pending > seg_cap) return fail(ctx, RT_ERR_OOM, "top-level build: range table overflow");
      RT_CUDA(ctx, cudaMemsetAsync(d_count + 1, 0, 4, st));
      SplitArgs a{d_segs, lv0, next, d_rank, box, d_ids, d_tmp, d_keys, d_sort_begin, d_sort_end, d_count + 1, sah ? 1 : 0};
      k_split<<<width, THREADS, 0, st>>>(a);
      RT_CUDA(ctx, cudaGetLastError());
      pending_sort = width;  // the sort ranges of this level, empty unless a large median split set one
      lv0 = next, width = 2 * pending, ++depth;
    }
    if (too_deep) {
      sah = false;
      continue;
    }
    // Boxes bottom-up, then the BVH4 levels top-down.
    for (size_t d = levels.size(); d-- > 0;)
      k_boxes<<<grid(levels[d].second, 256), 256, 0, st>>>(d_segs, levels[d].first, levels[d].second, d_ids, box, d_sbox);
    const uint32_t zero = 0;
    RT_CUDA(ctx, cudaMemcpyAsync(d_list, &zero, 4, cudaMemcpyHostToDevice, st));
    wide.assign({0u, 1u});
    for (;;) {
      const uint32_t first = wide[wide.size() - 2], count = wide.back() - first;
      RT_CUDA(ctx, cudaMemsetAsync(d_count, 0, 4, st));
      k_collapse<<<grid(count, 128), 128, 0, st>>>(d_segs, d_sbox, d_list, first, count, d_count, d_kids);
      uint32_t more = 0;
      RT_CUDA(ctx, cudaMemcpyAsync(&more, d_count, 4, cudaMemcpyDeviceToHost, st));
      RT_CUDA(ctx, cudaStreamSynchronize(st));
      if (!more) break;
      if ((size_t)wide.back() + more > n) return fail(ctx, RT_ERR_OOM, "top-level build: node list overflow");
      wide.push_back(wide.back() + more);
    }
    const size_t levels4 = wide.size() - 1;
    if (sah && 1 + 3 * levels4 > rtb::STACK_DEPTH) {  // instance_bvh.rs:360-364
      sah = false;
      continue;
    }
    break;
  }
  const size_t levels4 = wide.size() - 1;
  const uint32_t nodes = wide.back();
  if (nodes > cap_words / NODE_WORDS) return fail(ctx, RT_ERR_OOM, "top-level build: %u nodes past the reserve", nodes);
  for (size_t l = levels4; l-- > 0;)
    k_sizes<<<grid(wide[l + 1] - wide[l], 128), 128, 0, st>>>(d_segs, d_list, wide[l], wide[l + 1] - wide[l], d_kids, d_size);
  const uint32_t zero = 0;
  RT_CUDA(ctx, cudaMemcpyAsync(d_id, &zero, 4, cudaMemcpyHostToDevice, st));  // the root range is range 0
  for (size_t l = 0; l < levels4; ++l)
    k_ids<<<grid(wide[l + 1] - wide[l], 128), 128, 0, st>>>(d_segs, d_list, wide[l], wide[l + 1] - wide[l], d_kids, d_size, d_id);
  RT_CUDA(ctx, cudaMemsetAsync(d_out, 0, 4 * cap_words, st));
  // The node ids a level, deepest level first in `d_order` (a bottom-up refit order).
  std::vector<uint32_t> starts(1, 0);
  for (size_t l = levels4; l-- > 0;) starts.push_back(starts.back() + (wide[l + 1] - wide[l]));
  for (size_t l = 0; l < levels4; ++l) {
    const uint32_t first = wide[l], count = wide[l + 1] - wide[l];
    const size_t at = starts[levels4 - 1 - l];
    k_words<<<grid(count, 128), 128, 0, st>>>(d_segs, d_list, first, count, d_kids, d_id, d_ids, d_sbox, d_out,
                                               d_order ? d_order + at : nullptr);
  }
  RT_CUDA(ctx, cudaGetLastError());
  RT_CUDA(ctx, cudaStreamSynchronize(st));
  if (level_start) *level_start = starts;
  if (n_nodes) *n_nodes = nodes;
  return RT_OK;
}

}  // namespace rtc

rt_status rt_tlas_build_device(rt_ctx* ctx, const float* boxes, uint32_t n, int sah, uint32_t* out, size_t* n_words) {
  if (!ctx || !boxes || !n_words || n < 2) return fail(ctx, RT_ERR_INVALID_ARG, "null argument or fewer than two boxes");
  std::lock_guard<std::mutex> lock(ctx->mu);
  RT_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = nullptr;
  RT_CUDA(ctx, cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  struct StreamEnd {
    cudaStream_t s;
    ~StreamEnd() { cudaStreamDestroy(s); }
  } end{st};
  const size_t cap = (size_t)(n - 1) * NODE_WORDS;
  uint32_t* d = nullptr;
  if (cudaMalloc(&d, 24 * (size_t)n + 4 * cap) != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, RT_ERR_OOM, "top-level build buffers for %u instances", n);
  }
  struct Free {
    void* p;
    cudaStream_t s;
    ~Free() {
      cudaStreamSynchronize(s);
      cudaFree(p);
    }
  } free_d{d, st};
  uint32_t* d_boxes = d;
  uint32_t* d_out = d + 6 * (size_t)n;
  RT_CUDA(ctx, cudaMemcpyAsync(d_boxes, boxes, 24 * (size_t)n, cudaMemcpyHostToDevice, st));
  uint32_t nodes = 0;
  rt_status s = rtc::tlas_build_device(ctx, d_boxes, 6, n, sah != 0, d_out, cap, nullptr, nullptr, &nodes, st);
  if (s != RT_OK) return s;
  const size_t words = (size_t)nodes * NODE_WORDS;
  if (!out) {
    *n_words = words;
    return RT_OK;
  }
  if (*n_words < words) {
    *n_words = words;
    return fail(ctx, RT_ERR_INVALID_ARG, "the output holds %zu words, the top level %zu", *n_words, words);
  }
  RT_CUDA(ctx, cudaMemcpyAsync(out, d_out, 4 * words, cudaMemcpyDeviceToHost, st));
  RT_CUDA(ctx, cudaStreamSynchronize(st));
  *n_words = words;
  return RT_OK;
}
