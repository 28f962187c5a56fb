// The GI cell ray producer writing its rays out (the traversal that generates them in its refill
// is launch_fast_cells, kernels_fast.cu).
#include "kernels/cells.cuh"
#include "launch.hpp"

namespace rtl {

namespace {
__global__ void k_cell_rays(const rtk::GiCell* __restrict__ cells, uint32_t items, uint32_t rotate, float4* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= items) return;
  const rtk::Ray r = rtk::gi_cell_ray(cells, i, rotate != 0);
  out[2 * (size_t)i] = make_float4(r.o.x, r.o.y, r.o.z, r.tmin);
  out[2 * (size_t)i + 1] = make_float4(r.d.x, r.d.y, r.d.z, r.tmax);
}
}  // namespace

cudaError_t launch_cell_rays(const void* cells, uint32_t n_cells, uint32_t rotate, float4* rays, cudaStream_t stream) {
  const uint32_t items = n_cells * rtk::GI_DIRECTIONS;
  if (items == 0) return cudaSuccess;
  k_cell_rays<<<(items + 255) / 256, 256, 0, stream>>>(static_cast<const rtk::GiCell*>(cells), items, rotate, rays);
  return cudaGetLastError();
}

}  // namespace rtl
