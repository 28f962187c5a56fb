// Launchers for the PLAIN kernels and the arithmetic self-test.
#include "kernels/bvh2.cuh"
#include "kernels/plain.cuh"
#include "launch.hpp"

namespace rtl {

namespace {
constexpr uint32_t PLAIN_BLOCK = 128;

__global__ void k_selftest(uint32_t* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  volatile float pz = 0.0f, nz = -0.0f, three = 3.0f, two = 2.0f, tiny = 5.877471754e-39f;  // 2^-127, subnormal
  out[0] = __float_as_uint(fminf(nz, pz));
  out[1] = __float_as_uint(fminf(pz, nz));
  out[2] = __float_as_uint(fmaxf(nz, pz));
  out[3] = __float_as_uint(fmaxf(pz, nz));
  out[4] = __float_as_uint(__frcp_rn(three));
  out[5] = __float_as_uint(__fsqrt_rn(two));
  out[6] = __float_as_uint(__frcp_rn(tiny));  // subnormal operand: no flush to zero
  out[7] = __float_as_uint(__fdiv_rn(1.0f, three));
  out[8] = __float_as_uint(__fmul_rn(tiny, 1.0f));
  for (int k = 9; k < 16; ++k) out[k] = 0;
}
}  // namespace

cudaError_t launch_plain(const SceneView& s, uint32_t mode, const float4* rays, void* hits, uint32_t n,
                         rtk::DevStatus* st, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  const dim3 grid((n + PLAIN_BLOCK - 1) / PLAIN_BLOCK), block(PLAIN_BLOCK);
  if (s.layout == 0) {
    if (mode == 0) rtk::k_gi_plain<0><<<grid, block, 0, stream>>>(s.words, rays, hits, n, st);
    else if (mode == 1) rtk::k_gi_plain<1><<<grid, block, 0, stream>>>(s.words, rays, hits, n, st);
    else rtk::k_gi_plain<2><<<grid, block, 0, stream>>>(s.words, rays, hits, n, st);
  } else if (s.layout == 1) {
    if (mode == 0) rtk::k_rs_plain<false><<<grid, block, 0, stream>>>(s.words, rays, hits, n, st);
    else rtk::k_rs_plain<true><<<grid, block, 0, stream>>>(s.words, rays, hits, n, st);
  } else {
    if (mode == 0) rtk::k_rs2_plain<false><<<grid, block, 0, stream>>>(s.words, rays, hits, n, st);
    else rtk::k_rs2_plain<true><<<grid, block, 0, stream>>>(s.words, rays, hits, n, st);
  }
  return cudaGetLastError();
}

cudaError_t launch_selftest(uint32_t* out16, cudaStream_t stream) {
  k_selftest<<<1, 32, 0, stream>>>(out16);
  return cudaGetLastError();
}

}  // namespace rtl
