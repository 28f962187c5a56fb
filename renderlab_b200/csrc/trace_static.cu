// rt_trace_static: the FAST traversal for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc at trace time: an engine that fixes its device memory at
// start-up and forbids allocation in its frame loop, or a renderer that already keeps the packed
// gi_geometry / rl_geometry words in its own device buffer and wants a traversal without creating
// a context (rt_ctx_create allocates its status words and counters). This entry point allocates
// nothing. The FAST kernel's only scratch -- the ray counter its persistent warps take rays from,
// and the device status word its stack-overflow count goes to -- lives in the static device
// array below, 256 bytes that every GPU loading the library holds until the process exits.
//
// Host code may not use `g_static_scratch` as an address: its name on the host is a stand-in.
// The entry point looks up the array's device address once per device, with that device
// current, through cudaGetSymbolAddress, and passes that pointer to the kernel. Every call
// zeroes the counter and status on its stream before the launch and then shares the array with
// every other call, so calls that overlap on the GPU race on it.
//
// Stack overflows: a push onto a full traversal stack is dropped and counted in the array's
// status words, as a context counts it. rt_trace_static_stack_drops reads that count back after
// the call's stream has finished; the next call on the device zeroes it.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/rt_trace.h"
#include "launch.hpp"

namespace {

// word 0: the ray counter; words 16-31: an rtk::DevStatus (stack overflow count)
constexpr uint32_t STATIC_SCRATCH_WORDS = 64;
static __device__ __align__(256) unsigned int g_static_scratch[STATIC_SCRATCH_WORDS];
static_assert(sizeof(rtk::DevStatus) <= 16 * sizeof(unsigned int), "status must fit words 16-31");

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
unsigned int* g_scratch_ptr[MAX_DEVICES] = {};

// The array's device address on the current device (looked up on first use).
cudaError_t scratch_for(int device, unsigned int** out) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[device] = static_cast<unsigned int*>(p);
  }
  *out = g_scratch_ptr[device];
  return cudaSuccess;
}

}  // namespace

extern "C" rt_status rt_trace_static(rt_layout layout, const uint32_t* d_words, size_t n_words, rt_mode mode,
                                     const rt_ray* d_rays, void* d_hits, uint32_t n, void* stream) {
  if ((unsigned)layout > 1u || (unsigned)mode > 2u) return RT_ERR_INVALID_ARG;
  if (n > RT_STATIC_MAX_RAYS) return RT_ERR_INVALID_ARG;  // the ray counter's headroom
  if (n == 0) return RT_OK;
  if (!d_words || !d_rays || !d_hits || n_words < (layout == RT_LAYOUT_GI ? 16u : 8u)) return RT_ERR_INVALID_ARG;
  // rays and words are read in 16-byte loads, hits written as 4-byte words (as rt_trace_ex checks)
  if (reinterpret_cast<uintptr_t>(d_rays) % 16 != 0 || reinterpret_cast<uintptr_t>(d_words) % 16 != 0 ||
      reinterpret_cast<uintptr_t>(d_hits) % 4 != 0)
    return RT_ERR_INVALID_ARG;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= MAX_DEVICES) return RT_ERR_CUDA;
  unsigned int* scratch = nullptr;
  if (scratch_for(device, &scratch) != cudaSuccess) return RT_ERR_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(scratch, 0, STATIC_SCRATCH_WORDS * sizeof(unsigned int), s) != cudaSuccess) return RT_ERR_CUDA;
  rtl::SceneView v{};
  v.layout = (uint32_t)layout;
  v.words = d_words;
  v.n_words = n_words;
  cudaError_t e = rtl::launch_fast(v, (uint32_t)mode, reinterpret_cast<const float4*>(d_rays), nullptr, d_hits, n,
                                   scratch, reinterpret_cast<rtk::DevStatus*>(scratch + 16), s, 8);
  return e == cudaSuccess ? RT_OK : RT_ERR_CUDA;
}

extern "C" rt_status rt_trace_static_stack_drops(void* stream, uint64_t* out) {
  if (!out) return RT_ERR_INVALID_ARG;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= MAX_DEVICES) return RT_ERR_CUDA;
  unsigned int* scratch = nullptr;
  if (scratch_for(device, &scratch) != cudaSuccess) return RT_ERR_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the status words sit at word 16 of the array: DevStatus::stack_drops is their first member
  unsigned long long drops = 0;
  if (cudaMemcpyAsync(&drops, scratch + 16, sizeof drops, cudaMemcpyDeviceToHost, s) != cudaSuccess) return RT_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return RT_ERR_CUDA;
  *out = drops;
  return RT_OK;
}
