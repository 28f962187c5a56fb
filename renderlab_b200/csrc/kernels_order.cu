// Ray ordering: a sort key per ray, then a radix sort of (key, ray index) pairs. The sorted
// indices are the `order` permutation the FAST and WIDE8 kernels read, so that a warp takes rays
// that start close together and travel the same way.
#include <cub/device/device_radix_sort.cuh>

#include "launch.hpp"

namespace rtl {

namespace {

__device__ __forceinline__ uint32_t spread3(uint32_t x) {  // 10 bits -> every third bit
  x &= 0x3ffu;
  x = (x | (x << 16)) & 0x030000FFu;
  x = (x | (x << 8)) & 0x0300F00Fu;
  x = (x | (x << 4)) & 0x030C30C3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}

__device__ __forceinline__ uint32_t cell(float v, float lo, float scale, uint32_t top) {
  const float c = (v - lo) * scale;
  return c <= 0.0f ? 0u : (c >= (float)top ? top : (uint32_t)c);
}

// kind 1: 30-bit Morton code of the origin; kind 2: direction octant (3 bits) above a 27-bit
// Morton code of the origin; kind 3: a 12-bit octahedral direction cell above an 18-bit origin code.
struct KeyLane {
  uint32_t ray_id, entry;
  bool any;
};

template <class Src>
__global__ void k_keys(const Src src, uint32_t n, float3 lo, float3 inv_ext, uint32_t kind, uint32_t* __restrict__ keys,
                       uint32_t* __restrict__ vals) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  KeyLane lane;
  const rtk::Ray r = rtk::fetch(src, i, lane);
  const float3 a = make_float3(r.o.x, r.o.y, r.o.z), b = make_float3(r.d.x, r.d.y, r.d.z);
  uint32_t key;
  if (kind == 1) {
    key = spread3(cell(a.x, lo.x, 1024.0f * inv_ext.x, 1023)) | spread3(cell(a.y, lo.y, 1024.0f * inv_ext.y, 1023)) << 1 |
          spread3(cell(a.z, lo.z, 1024.0f * inv_ext.z, 1023)) << 2;
  } else if (kind == 2) {
    const uint32_t oct = (b.x < 0.0f ? 1u : 0u) | (b.y < 0.0f ? 2u : 0u) | (b.z < 0.0f ? 4u : 0u);
    key = oct << 27 | spread3(cell(a.x, lo.x, 512.0f * inv_ext.x, 511)) | spread3(cell(a.y, lo.y, 512.0f * inv_ext.y, 511)) << 1 |
          spread3(cell(a.z, lo.z, 512.0f * inv_ext.z, 511)) << 2;
  } else {
    const float s = fabsf(b.x) + fabsf(b.y) + fabsf(b.z);
    float u = s > 0.0f ? b.x / s : 0.0f, v = s > 0.0f ? b.y / s : 0.0f;
    if (b.z < 0.0f) {
      const float uu = (1.0f - fabsf(v)) * (u >= 0.0f ? 1.0f : -1.0f);
      v = (1.0f - fabsf(u)) * (v >= 0.0f ? 1.0f : -1.0f);
      u = uu;
    }
    const uint32_t cu = cell(u, -1.0f, 32.0f, 63), cv = cell(v, -1.0f, 32.0f, 63);
    const uint32_t dir = spread3(cu) | spread3(cv) << 1;  // interleaved, 12 bits
    key = (dir & 0xfffu) << 18 | spread3(cell(a.x, lo.x, 64.0f * inv_ext.x, 63)) |
          spread3(cell(a.y, lo.y, 64.0f * inv_ext.y, 63)) << 1 | spread3(cell(a.z, lo.z, 64.0f * inv_ext.z, 63)) << 2;
  }
  keys[i] = key;
  vals[i] = i;
}

}  // namespace

size_t order_scratch_bytes(uint32_t n) {
  size_t temp = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, temp, (uint32_t*)nullptr, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                  (uint32_t*)nullptr, (int)n);
  return 3 * (size_t)n * sizeof(uint32_t) + ((temp + 255) & ~(size_t)255) + 256;
}

namespace {
template <class Src>
cudaError_t order_any(const Src& src, uint32_t n, const float lo[3], const float hi[3], uint32_t kind, uint32_t* order,
                      void* scratch, size_t scratch_bytes, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  if (scratch_bytes < order_scratch_bytes(n)) return cudaErrorInvalidValue;
  uint32_t* keys_in = static_cast<uint32_t*>(scratch);
  uint32_t* keys_out = keys_in + n;
  uint32_t* vals_in = keys_out + n;
  void* temp = reinterpret_cast<void*>((reinterpret_cast<uintptr_t>(vals_in + n) + 255) & ~(uintptr_t)255);
  size_t temp_bytes = scratch_bytes - (static_cast<char*>(temp) - static_cast<char*>(scratch));
  auto inv = [](float a, float b) { return b > a ? 1.0f / (b - a) : 1.0f; };
  k_keys<<<(n + 255) / 256, 256, 0, stream>>>(src, n, make_float3(lo[0], lo[1], lo[2]),
                                              make_float3(inv(lo[0], hi[0]), inv(lo[1], hi[1]), inv(lo[2], hi[2])), kind,
                                              keys_in, vals_in);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys_in, keys_out, vals_in, order, (int)n, 0, 32, stream);
}
}  // namespace

cudaError_t launch_order(const float4* rays, uint32_t n, const float lo[3], const float hi[3], uint32_t kind,
                         uint32_t* order, void* scratch, size_t scratch_bytes, cudaStream_t stream) {
  return order_any(rtk::OneBatch{rays, nullptr, nullptr}, n, lo, hi, kind, order, scratch, scratch_bytes, stream);
}

cudaError_t launch_order_batches(const rtk::BatchEntry* table, uint32_t entries, uint32_t total, const float lo[3],
                                 const float hi[3], uint32_t kind, uint32_t* order, void* scratch, size_t scratch_bytes,
                                 cudaStream_t stream) {
  return order_any(rtk::ManyBatches{table, entries, nullptr}, total, lo, hi, kind, order, scratch, scratch_bytes, stream);
}

}  // namespace rtl
