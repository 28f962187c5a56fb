// FAST kernels: the PLAIN arithmetic (bit-exact) under a scheduled launch.
#include "kernels/plain.cuh"
#include "launch.hpp"

namespace rtl {

cudaError_t launch_fast(const SceneView& s, uint32_t mode, const float4* rays, const uint32_t* order, void* hits,
                        uint32_t n, rtk::DevStatus* st, cudaStream_t stream) {
  (void)s, (void)mode, (void)rays, (void)order, (void)hits, (void)n, (void)st, (void)stream;
  return cudaErrorNotSupported;
}

}  // namespace rtl
