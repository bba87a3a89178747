// SOR and SSOR smoothing sweeps (the preconditioner of the Richardson smoother).
//
// The reference's generic preconditioners (kernel/solver/sor_precond.hpp:179-224,
// kernel/solver/ssor_precond.hpp) sweep the rows in order: forward insertion
//   SOR:  y_i = w (d_i - sum_{j<i} a_ij y_j) / a_ii
//   SSOR: y_i = (d_i - w sum_{j<i} a_ij y_j) / a_ii,   then backward   y_i -= w (sum_{j>i} a_ij y_j) / a_ii
// (sums over the row's stored entries left of the diagonal in stored order, right of it from the
// row's end backwards), then y *= w (2 - w) for SSOR, then the unit filter.  Its CUDA backend
// (kernel/solver/sor_precond.cu:26-41, :294-315; ssor_precond.cu:25-60, :182-230) runs the same
// row formulas colour by colour on a zeroed y.
//
// Here a sweep is a list of colours, each a set of mutually independent rows, run one after the
// other: with the dependency levels of the sequential sweep (fb_setup.cpp, sweep_levels) every row
// sees exactly the values the sequential sweep gives it, so the result equals the reference's
// generic preconditioner bit for bit; with a greedy colouring (greedy_colours) it is the coloured
// sweep of the reference's CUDA backend.  Few colours run one launch each over the grid; many
// colours (dependency levels of a large matrix) run in one block with a barrier between colours.
// Every product and sum is rounded separately and the divisions are IEEE-rounded, as on the host.
#pragma once

#include "fb_common.cuh"

namespace fb
{
  __device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
  __device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }

  // the sweep's matrix: CSR of the full system matrix (Dirichlet rows included: their values take
  // part in the sweep before the filter zeroes them), and each row's diagonal position as the
  // forward (first entry with column >= row) and backward (last entry with column <= row) loops of
  // the reference find it
  template<typename S>
  struct SorCsr
  {
    const uint32_t* rp;
    const uint32_t* col;
    const S* val;
    const uint32_t* posf;
    const uint32_t* posb;
  };

  enum SweepKind { SW_SOR = 0, SW_SSOR_FWD = 1, SW_SSOR_BWD = 2 };

  template<typename S, int KIND>
  __device__ __forceinline__ void sweep_row(const SorCsr<S>& M, const S* __restrict__ in, S* y, uint32_t row, S w)
  {
    if(KIND == SW_SSOR_BWD)
    {
      const uint32_t p = __ldg(M.posb + row);
      S d = S(0);
      for(uint32_t k = __ldg(M.rp + row + 1) - 1u; k > p; --k)
        d = add(d, mul(__ldg(M.val + k), y[__ldg(M.col + k)]));
      y[row] = sub(y[row], div_rn(mul(w, d), __ldg(M.val + p)));
      return;
    }
    const uint32_t p = __ldg(M.posf + row);
    S d = S(0);
    for(uint32_t k = __ldg(M.rp + row); k < p; ++k)
      d = add(d, mul(__ldg(M.val + k), y[__ldg(M.col + k)]));
    if(KIND == SW_SOR)
      y[row] = div_rn(mul(w, sub(in[row], d)), __ldg(M.val + p));
    else
      y[row] = div_rn(sub(in[row], mul(w, d)), __ldg(M.val + p));
  }

  // one colour over the grid: rows[0 .. count)
  template<typename S, int KIND>
  __global__ void __launch_bounds__(NT) k_sweep_colour(SorCsr<S> M, const S* __restrict__ in, S* y,
    const uint32_t* __restrict__ rows, uint32_t count, S w, const Scalars* __restrict__ sc)
  {
    pdl_wait();
    if(gate_closed(sc))
      return;
    const uint32_t k = blockIdx.x * NT + threadIdx.x;
    if(k < count)
      sweep_row<S, KIND>(M, in, y, __ldg(rows + k), w);
  }

  constexpr int SWEEP_BLOCK_NT = 1024;
  constexpr uint32_t SWEEP_LAUNCH_MAX = 16;   // sweeps of at most this many colours launch per colour

  // all colours in one block, a barrier between colours
  template<typename S, int KIND>
  __global__ void __launch_bounds__(SWEEP_BLOCK_NT) k_sweep_block(SorCsr<S> M, const S* __restrict__ in, S* y,
    const uint32_t* __restrict__ order, const uint32_t* __restrict__ cofs, uint32_t ncol, S w,
    const Scalars* __restrict__ sc)
  {
    pdl_wait();
    if(gate_closed(sc))
      return;
    for(uint32_t c = 0; c < ncol; ++c)
    {
      const uint32_t e = __ldg(cofs + c + 1);
      for(uint32_t k = __ldg(cofs + c) + threadIdx.x; k < e; k += SWEEP_BLOCK_NT)
        sweep_row<S, KIND>(M, in, y, __ldg(order + k), w);
      __syncthreads();
    }
  }

  template<typename S>
  __global__ void __launch_bounds__(NT) k_sweep_zero(S* y, uint32_t n, const Scalars* __restrict__ sc)
  {
    pdl_wait();
    if(gate_closed(sc))
      return;
    const uint32_t i = blockIdx.x * NT + threadIdx.x;
    if(i < n)
      y[i] = S(0);
  }

  // the end of one Richardson step with the sweep's result y as the preconditioned defect:
  // cor = F(s y) (s = w (2 - w) for SSOR, else no scaling), out = cor + base (base = null: the
  // smoother's first step, from zero), or out = 0 when the smoother skips (its initial defect norm
  // is zero or not finite)
  template<typename S>
  __global__ void __launch_bounds__(NT) k_sweep_finish(const S* __restrict__ y, const S* base, S* out,
    const uint8_t* __restrict__ dm, const int* __restrict__ skip, S scale, int scaled, uint32_t n,
    const Scalars* __restrict__ sc)
  {
    pdl_wait();
    if(gate_closed(sc))
      return;
    const uint32_t i = blockIdx.x * NT + threadIdx.x;
    if(i >= n)
      return;
    if(*skip)
    {
      out[i] = S(0);
      return;
    }
    S c = scaled ? mul(y[i], scale) : y[i];
    if(__ldg(dm + i))
      c = S(0);
    out[i] = add(c, base ? base[i] : S(0));
  }
} // namespace fb
