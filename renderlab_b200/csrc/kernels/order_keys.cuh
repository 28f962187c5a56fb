// Order-preserving integer keys of f32, shared by the device builders: min/max reductions through
// integer atomics, and sort keys that order as f32::total_cmp does.
#pragma once
#include <cstdint>

namespace rtq {

// f32::total_cmp as an unsigned comparison, and back.
__device__ __forceinline__ uint32_t okey(float f) {
  const uint32_t b = __float_as_uint(f);
  return b ^ ((b >> 31) ? 0xffffffffu : 0x80000000u);
}
__device__ __forceinline__ float unkey(uint32_t k) { return __uint_as_float(k ^ ((k >> 31) ? 0x80000000u : 0xffffffffu)); }
// f32::total_cmp as a signed comparison (the host builders' order_key).
__device__ __forceinline__ int32_t order_key(float f) {
  const int32_t x = __float_as_int(f);
  return x ^ (int32_t)(((uint32_t)(x >> 31)) >> 1);
}

}  // namespace rtq
