// fb_dot_f64_noalloc: an FP64 dot product that never allocates device memory.
//
// Some callers cannot allocate device memory when they need a reduction: processes that hand the
// whole device memory to their own pool allocator at start-up (MPI codes with a fixed per-rank
// memory budget work this way), and loops that must not stall, since cudaMalloc and cudaFree can
// synchronise the device.  fb_dot_f64 allocates its reduction scratch on first use; this variant
// keeps its scratch in a fixed array of this file instead.
//
// The scratch is a file-scope __device__ array: every GPU that loads this file's module holds it
// (NOALLOC_MAX_BLOCKS = 4096 partial sums, 32 KiB, plus a counter and the result) until the process
// exits.  Under CUDA's lazy module loading (the default) the module, and with it the array, is
// loaded by the first use on a device, and that load itself takes device memory.  A caller that
// hands all device memory to its own pool should therefore make one set-up call per device before
// its pool takes the memory: fb_dot_f64_noalloc with n = 0 (x and y may then be null) loads the
// module and the kernel on the current device, resolves the array's address and launches nothing.
// Each block of the kernel reduces NOALLOC_CHUNK = 4096 consecutive elements, so the largest
// accepted vector has 4096 * 4096 = 16,777,216 elements (FB_DOT_NOALLOC_MAX_N); longer vectors are
// rejected with FB_ERR_ARG.  All calls share the one array and it keeps the last
// call's contents: the arrival counter is cleared at the start of every call, and calls that
// overlap on the GPU (concurrent streams, several host threads) race on the array.
#include "fb_common.cuh"

#include <string>

namespace fb
{
  constexpr int NOALLOC_NT = 256;
  constexpr uint32_t NOALLOC_PER_THREAD = 16;
  constexpr uint64_t NOALLOC_CHUNK = uint64_t(NOALLOC_NT) * NOALLOC_PER_THREAD;   // 4096
  constexpr uint32_t NOALLOC_MAX_BLOCKS = 4096;
  static_assert(uint64_t(NOALLOC_MAX_BLOCKS) * NOALLOC_CHUNK == FB_DOT_NOALLOC_MAX_N, "limit in featb200.h");

  struct NoallocScratch
  {
    double partials[NOALLOC_MAX_BLOCKS];
    double result;
    unsigned int counter;
  };

  // The scratch array.  In host code this name is only a stand-in for the device symbol: its
  // device address comes from cudaGetSymbolAddress (noalloc_scratch_ptr below).
  static __device__ __align__(256) NoallocScratch g_noalloc_scratch;

  __global__ void __launch_bounds__(NOALLOC_NT) k_dot_noalloc(const double* __restrict__ x, const double* __restrict__ y,
    uint64_t n, NoallocScratch* sc)
  {
    __shared__ double sh[32];
    const uint64_t base = uint64_t(blockIdx.x) * NOALLOC_CHUNK;
    double s = 0.0;
    #pragma unroll 4
    for(uint32_t k = 0; k < NOALLOC_PER_THREAD; ++k)
    {
      const uint64_t i = base + uint64_t(k) * NOALLOC_NT + threadIdx.x;
      if(i < n)
        s += x[i] * y[i];
    }
    double total;
    if(grid_sum_last<NOALLOC_NT>(s, RedSlot{sc->partials, &sc->counter}, sh, total))
      sc->result = total;
  }

  // Device address of the scratch array in the current context, with that context's device
  // current.  The address is looked up on every call rather than cached per device ordinal: after
  // cudaDeviceReset, or under a context other than the primary one, a cached address would be
  // stale.  Once the module is loaded the lookup allocates nothing.  The kernel's attributes are
  // queried as well, so that under lazy loading the kernel is loaded here, not at its first launch.
  static fb_status noalloc_scratch_ptr(NoallocScratch*& out)
  {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if(e != cudaSuccess)
      return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    cudaFuncAttributes fa;
    e = cudaFuncGetAttributes(&fa, k_dot_noalloc);
    if(e != cudaSuccess)
      return cuda_fail(e, "cudaFuncGetAttributes(k_dot_noalloc)");
    out = static_cast<NoallocScratch*>(p);
    return FB_OK;
  }
} // namespace fb

extern "C" fb_status fb_dot_f64_noalloc(double* result, const double* x, const double* y, uint64_t n, void* stream)
{
  using namespace fb;
  if(!result)
  {
    set_error("dot_noalloc: null result");
    return FB_ERR_ARG;
  }
  if(n > uint64_t(NOALLOC_MAX_BLOCKS) * NOALLOC_CHUNK)
  {
    set_error("dot_noalloc: n = " + std::to_string(n) + " exceeds the maximum of " +
              std::to_string(uint64_t(NOALLOC_MAX_BLOCKS) * NOALLOC_CHUNK) +
              " elements of the fixed scratch array (use fb_dot_f64)");
    return FB_ERR_ARG;
  }
  if(n != 0 && (!x || !y))
  {
    set_error("dot_noalloc: null pointer");
    return FB_ERR_ARG;
  }
  // set-up on the current device (module and kernel loaded, array address resolved); n = 0 stops
  // here, which is the set-up call for callers whose pool takes the device memory afterwards
  NoallocScratch* sc = nullptr;
  fb_status e = noalloc_scratch_ptr(sc);
  if(e != FB_OK)
    return e;
  if(n == 0)
  {
    *result = 0.0;
    return FB_OK;
  }
  cudaStream_t st = as_stream(stream);
  // the array keeps the last call's contents: the arrival counter must start at zero
  FB_CUDA(cudaMemsetAsync(&sc->counter, 0, sizeof(unsigned int), st));
  const unsigned int blocks = (unsigned int)((n + NOALLOC_CHUNK - 1) / NOALLOC_CHUNK);
  k_dot_noalloc<<<blocks, NOALLOC_NT, 0, st>>>(x, y, n, sc);
  FB_LAUNCHED(1);
  double v = 0.0;
  FB_CUDA(cudaMemcpyAsync(&v, &sc->result, sizeof(double), cudaMemcpyDeviceToHost, st));
  FB_CUDA(cudaStreamSynchronize(st));
  *result = v;
  return FB_OK;
}
