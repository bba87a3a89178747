// Shared device/host helpers of the featb200 library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <atomic>
#include <string>

#include "../../include/featb200.h"

namespace fb
{
  // ------------------------------------------------------------------ error reporting
  void set_error(const std::string& msg);
  fb_status cuda_fail(cudaError_t e, const char* what);
  void count_launches(uint64_t n);

#define FB_CUDA(call)                                  \
  do {                                                 \
    cudaError_t fb_e_ = (call);                        \
    if(fb_e_ != cudaSuccess)                           \
      return ::fb::cuda_fail(fb_e_, #call);            \
  } while(0)

#define FB_LAUNCHED(n)                                 \
  do {                                                 \
    cudaError_t fb_e_ = cudaGetLastError();            \
    if(fb_e_ != cudaSuccess)                           \
      return ::fb::cuda_fail(fb_e_, "kernel launch");  \
    ::fb::count_launches(n);                           \
  } while(0)

  inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

  // ------------------------------------------------------------------ value storage types
  // Matrix values are stored as double, float or bf16 (as raw 16-bit words); the arithmetic type
  // of a kernel is double for double storage and float otherwise.
  struct bf16_t { uint16_t bits; };

  template<typename V> struct ValueTraits;
  template<> struct ValueTraits<double> { typedef double acc; };
  template<> struct ValueTraits<float> { typedef float acc; };
  template<> struct ValueTraits<bf16_t> { typedef float acc; };

  __device__ __forceinline__ double to_acc(double v) { return v; }
  __device__ __forceinline__ float to_acc(float v) { return v; }
  __device__ __forceinline__ float to_acc(bf16_t v) { return __uint_as_float(uint32_t(v.bits) << 16); }

  // Arithmetic without FMA contraction, so that every product is rounded before it is added
  // exactly as in the reference's generic C++ loops (no -ffp-contract in its build).
  __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }

  // ------------------------------------------------------------------ programmatic dependent launch
  // A kernel launched with programmatic stream serialisation may be scheduled before its
  // predecessor in the stream has finished; pdl_wait blocks until the predecessor has completed
  // and its writes are visible (a no-op for a kernel launched without the attribute).  No kernel
  // signals its dependents early (griddepcontrol.launch_dependents): the successor is released as
  // the predecessor's blocks exit, so only its launch and its work before pdl_wait overlap.  (An
  // early signal at kernel start was measured faster but gave wrong V-cycles on B200 when FP32
  // sliced-ELL staged passes ran with the single-block tail; the cause was not found.)
  __device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

  // ------------------------------------------------------------------ deterministic reductions
  // Block sum in a fixed order (warp shuffles, then warp 0 over the per-warp partials).
  template<int NT>
  __device__ __forceinline__ double block_sum(double v, double* sh)
  {
    constexpr int NW = NT / 32;
    #pragma unroll
    for(int o = 16; o > 0; o >>= 1)
      v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if(lane == 0)
      sh[warp] = v;
    __syncthreads();
    double t = 0.0;
    if(warp == 0)
    {
      t = (lane < NW) ? sh[lane] : 0.0;
      #pragma unroll
      for(int o = 16; o > 0; o >>= 1)
        t += __shfl_down_sync(0xffffffffu, t, o);
    }
    __syncthreads();
    return t;   // valid in thread 0
  }

  // Grid-wide reduction slot: per-block partials, an arrival counter and the final value.  The
  // last block to arrive sums the partials in block order (deterministic) and resets the counter.
  struct RedSlot
  {
    double* partials;
    unsigned int* counter;
  };

  // Returns true in thread 0 of the last block, with `total` set to the grid sum.
  template<int NT>
  __device__ __forceinline__ bool grid_sum_last(double v, RedSlot slot, double* sh, double& total)
  {
    __shared__ bool am_last;
    double b = block_sum<NT>(v, sh);
    if(threadIdx.x == 0)
    {
      slot.partials[blockIdx.x] = b;
      __threadfence();
      unsigned int prev = atomicAdd(slot.counter, 1u);
      am_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if(!am_last)
      return false;
    __threadfence();
    // the last block sums the partials: each thread a strided subset in order, then a block sum
    double s = 0.0;
    for(unsigned int i = threadIdx.x; i < gridDim.x; i += NT)
      s += ((volatile double*)slot.partials)[i];
    double t = block_sum<NT>(s, sh);
    if(threadIdx.x == 0)
    {
      *slot.counter = 0u;
      total = t;
    }
    return threadIdx.x == 0;
  }

  // Two grid sums at once (partials of b at partials[gridDim.x + block]); true in thread 0 of the
  // last block, with ta, tb set.
  template<int NT>
  __device__ __forceinline__ bool grid_sum2_last(double a, double b, RedSlot slot, double* sh, double& ta, double& tb)
  {
    __shared__ bool am_last;
    const double pa = block_sum<NT>(a, sh);
    const double pb = block_sum<NT>(b, sh);
    if(threadIdx.x == 0)
    {
      slot.partials[blockIdx.x] = pa;
      slot.partials[gridDim.x + blockIdx.x] = pb;
      __threadfence();
      unsigned int prev = atomicAdd(slot.counter, 1u);
      am_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if(!am_last)
      return false;
    __threadfence();
    double sa = 0.0, sb = 0.0;
    for(unsigned int i = threadIdx.x; i < gridDim.x; i += NT)
    {
      sa += ((volatile double*)slot.partials)[i];
      sb += ((volatile double*)slot.partials)[gridDim.x + i];
    }
    const double t1 = block_sum<NT>(sa, sh);
    const double t2 = block_sum<NT>(sb, sh);
    if(threadIdx.x == 0)
    {
      *slot.counter = 0u;
      ta = t1;
      tb = t2;
    }
    return threadIdx.x == 0;
  }

  constexpr double EPS64 = 2.220446049250313080847e-16;
  constexpr float EPS32 = 1.1920928955078125e-7f;
} // namespace fb
