// Batched solver: many independent PCG + V-cycle solves of uneven size in one launch per V-cycle
// phase.
//
// Instance j has L_j levels.  Levels are aligned from the coarsest: global level G holds level
// L_j-1-G of every instance with L_j > G, concatenated (each instance's rows padded to a multiple
// of 32, so a warp never spans two instances).  The matrices of a global level are therefore block
// diagonal and every pass of the single-system V-cycle (k_smooth ... k_post2, fb_mg.cu) becomes ONE
// launch over all instances present at that level, using the same per-row bodies (fb_rows.cuh).
// An instance enters the V-cycle at its own top level T_j = L_j-1: its right-hand side there comes
// from its PCG (PCG space = the concatenated top levels), not from a restriction.
//
// Per instance: PCG scalars, stopping test (iterative.hpp:492-507,795-879), Richardson skip flags
// per level, and a status word; converged instances skip all work.  Dot products and norms are
// reduced per warp, summed per instance within the block and added per instance with FP64 atomics;
// the last block to arrive finalises all instances (their summation order is not fixed; results
// agree with single solves to rounding).  System matrices of lexicographically numbered instances
// are held in diagonal storage (values only), as in the single-system solver.
#include "fb_common.cuh"
#include "fb_rows.cuh"
#include "fb_tma.cuh"
#include "fb_setup.h"

#include <algorithm>
#include <map>
#include <mutex>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

namespace fb
{
namespace bt
{
  constexpr int BNT = 256;       // block size of the PCG-space kernels (4 resident per SM: at most 64 registers)
  constexpr int BNT_MAX = 512;   // largest block size the autotuner may pick for the V-cycle passes
  constexpr int BW = BNT / 32;
  constexpr int MAXG = 16;

  struct BScal   // device-resident, per instance arrays of length J
  {
    double *gamma, *gamma_prev, *alpha, *beta, *def_init, *def_cur, *scale, *inv_scale, *acc;
    int *iter, *status, *top;
    int* skip_pre;     // [MAXG * J]
    int* skip_post;    // [MAXG * J]
    unsigned int* arrive;
    int* progress;
    int J;
    double tol_rel, tol_abs, div_rel, div_abs;
    int min_iter, max_iter;
  };

  // per global level, vectors in the V-cycle precision (for the PCG space <-> top level writes)
  template<typename S>
  struct TopPtrs
  {
    S* b[MAXG];
    S* x[MAXG];
    const S* dinv[MAXG];
  };

  __device__ __forceinline__ bool active(const BScal& sc, int j) { return sc.status[j] == FB_SOLVER_PROGRESS; }
  __device__ __forceinline__ bool closed(const BScal& sc) { return *sc.progress <= 0; }

  __device__ __forceinline__ double warp_sum(double v)
  {
    #pragma unroll
    for(int o = 16; o > 0; o >>= 1)
      v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
  }

  // Adds the block's partials per instance to acc[inst] and counts the block in; returns true in
  // warp 0 of the last block of the grid, which then finalises.  A warp's rows belong to one
  // instance (inst < 0: the warp contributes nothing); each run of consecutive warps with the same
  // instance is added by its first warp's lane with one atomic, so the grid's same-address arrival
  // counter takes one atomic per block.  Every thread of the grid must call this.
  __device__ __forceinline__ bool block_arrive(double part, int inst, const BScal& sc)
  {
    __shared__ double ws[BNT_MAX / 32];
    __shared__ int wi[BNT_MAX / 32];
    __shared__ unsigned int prev_s;
    const double s = warp_sum(part);
    const int lane = int(threadIdx.x & 31u), warp = int(threadIdx.x >> 5), nw = int(blockDim.x >> 5);
    if(lane == 0)
    {
      ws[warp] = s;
      wi[warp] = inst;
    }
    __syncthreads();
    if(warp == 0)
    {
      if(lane < nw)
      {
        const int my = wi[lane];
        if(my >= 0 && (lane == 0 || wi[lane - 1] != my))
        {
          double t = 0.0;
          for(int k = lane; k < nw && wi[k] == my; ++k)
            t += ws[k];
          atomicAdd(&sc.acc[my], t);
        }
      }
      __threadfence();
      __syncwarp();
      if(lane == 0)
        prev_s = atomicAdd(sc.arrive, 1u);
    }
    __syncthreads();
    if(prev_s != gridDim.x - 1)
      return false;
    __threadfence();
    return warp == 0;
  }

  // warp 0 of the last block: fin(j, total) for every instance j, accumulators cleared, counter reset
  template<class Fin>
  __device__ __forceinline__ void finalize_all(const BScal& sc, Fin fin)
  {
    const int lane = threadIdx.x & 31;
    for(int j = lane; j < sc.J; j += 32)
    {
      const double tot = atomicAdd(&sc.acc[j], 0.0);
      sc.acc[j] = 0.0;
      fin(j, tot);
    }
    if(lane == 0)
      *sc.arrive = 0u;
  }

  // ---------------------------------------------------------------- V-cycle passes, level G
  template<typename V, typename S>
  __global__ void __launch_bounds__(BNT_MAX) kb_smooth(DCsr<V> A, const S* __restrict__ b, const S* __restrict__ x,
    S* __restrict__ xo, const S* __restrict__ dinv, const uint8_t* __restrict__ dm, const int* __restrict__ sinst,
    const int* __restrict__ skip, BScal sc)
  {
    if(closed(sc))
      return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= A.rows)
      return;
    const int j = __ldg(sinst + (i >> 5));
    if(!active(sc, j))
      return;
    xo[i] = smooth_row<V, S, true>(A, b, x, dinv, dm, skip[j] != 0, i);
  }

  template<typename V, typename S>
  __global__ void __launch_bounds__(BNT_MAX) kb_defect(DCsr<V> A, const S* __restrict__ b, const S* __restrict__ x,
    S* __restrict__ d, const uint8_t* __restrict__ dm, const int* __restrict__ sinst, BScal sc)
  {
    if(closed(sc))
      return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= A.rows)
      return;
    const int j = __ldg(sinst + (i >> 5));
    if(!active(sc, j))
      return;
    d[i] = defect_row<V, S, true>(A, b, x, dm, i);
  }

  // coarse rows of level G-1: rows of instances whose top is G-1 are fed by their PCG: untouched
  template<typename V, typename S>
  __global__ void __launch_bounds__(BNT_MAX) kb_restrict(DCsr<V> R, const S* __restrict__ d, S* __restrict__ bc,
    S* __restrict__ xc, const S* __restrict__ dinvc, const uint8_t* __restrict__ dmc, const int* __restrict__ sinstc,
    int gc, int* __restrict__ skipc, BScal sc)
  {
    if(closed(sc))
      return;
    const uint32_t jr = blockIdx.x * blockDim.x + threadIdx.x;
    int inst = -1;
    double sq = 0.0;
    if(jr < R.rows || (jr & ~31u) < R.rows)
    {
      const int j = __ldg(sinstc + (jr >> 5));
      if(active(sc, j) && sc.top[j] != gc)
      {
        inst = j;
        if(jr < R.rows)
          sq = restrict_row<V, S, true>(R, d, bc, xc, dinvc, dmc, jr);
      }
    }
    if(!xc)
      return;
    if(block_arrive(sq, inst, sc))
      finalize_all(sc, [&](int j, double tot)
      {
        if(active(sc, j) && sc.top[j] > gc)
          skipc[j] = skip_from_norm<S>(sqrt(tot));
      });
  }

  // exact coarse solve per instance: one block per instance
  template<typename S>
  __global__ void __launch_bounds__(BNT) kb_coarse(const S* __restrict__ b, S* __restrict__ x,
    const uint32_t* __restrict__ rowoff, const uint32_t* __restrict__ nrows, const uint32_t* __restrict__ free_off,
    const uint32_t* __restrict__ free_dofs, const uint64_t* __restrict__ inv_off, const double* __restrict__ inv, BScal sc)
  {
    if(closed(sc))
      return;
    const int j = blockIdx.x;
    if(!active(sc, j))
      return;
    const uint32_t r0 = rowoff[j], n = nrows[j];
    const uint32_t f0 = free_off[j], m = free_off[j + 1] - f0;
    coarse_block<S, BNT>(b + r0, x + r0, n, free_dofs + f0, inv + inv_off[j], m);
  }

  template<typename V, typename S>
  __global__ void __launch_bounds__(BNT_MAX) kb_prolong(DCsr<V> P, const S* __restrict__ xc, S* __restrict__ x,
    const uint8_t* __restrict__ dm, const int* __restrict__ sinst, BScal sc)
  {
    if(closed(sc))
      return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= P.rows)
      return;
    const int j = __ldg(sinst + (i >> 5));
    if(!active(sc, j))
      return;
    x[i] = prolong_row<V, S, true>(P, xc, x, dm, i);
  }

  template<typename V, typename S>
  __global__ void __launch_bounds__(BNT_MAX) kb_post1(DCsr<V> A, const S* __restrict__ b, const S* __restrict__ x,
    S* __restrict__ d, S* __restrict__ c, const S* __restrict__ dinv, const uint8_t* __restrict__ dm,
    const int* __restrict__ sinst, int* __restrict__ skip, BScal sc)
  {
    if(closed(sc))
      return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    int inst = -1;
    double sq = 0.0;
    if((i & ~31u) < A.rows)
    {
      const int j = __ldg(sinst + (i >> 5));
      if(active(sc, j))
      {
        inst = j;
        if(i < A.rows)
          sq = post1_row<V, S, true>(A, b, x, d, c, dinv, dm, i);
      }
    }
    if(block_arrive(sq, inst, sc))
      finalize_all(sc, [&](int j, double tot)
      {
        skip[j] = skip_from_norm<S>(sqrt(tot));
      });
  }

  // post-smoothing step k >= 2 at level g; LAST: instances whose top is g write z (PCG space) and
  // r.z -> gamma, beta; the others update x
  template<typename V, typename S, bool LAST>
  __global__ void __launch_bounds__(BNT_MAX) kb_post2(DCsr<V> A, const S* __restrict__ d, const S* __restrict__ c,
    S* __restrict__ co, S* __restrict__ x, double* __restrict__ z, const double* __restrict__ r,
    const int* __restrict__ pcg_base, const S* __restrict__ dinv, const uint8_t* __restrict__ dm,
    const int* __restrict__ sinst, int g, const int* __restrict__ skip, BScal sc)
  {
    typedef typename ValueTraits<V>::acc Ac;
    if(closed(sc))
      return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    int inst = -1;
    double rz = 0.0;
    if((i & ~31u) < A.rows)
    {
      const int j = __ldg(sinst + (i >> 5));
      if(active(sc, j))
      {
        if(i < A.rows)
        {
          const Ac cn = post2_row<V, S, true>(A, d, c, dinv, dm, skip[j] != 0, i);
          if(!LAST)
            co[i] = S(cn);
          else
          {
            const S xn = S(add(Ac(x[i]), cn));
            if(sc.top[j] == g)
            {
              const uint32_t pr = uint32_t(__ldg(pcg_base + (i >> 5))) + (i & 31u);
              const double zi = mul(double(xn), sc.inv_scale[j]);
              z[pr] = zi;
              rz = mul(r[pr], zi);
            }
            else
              x[i] = xn;
          }
        }
        if(LAST && sc.top[j] == g)
          inst = j;
      }
    }
    if(!LAST)
      return;
    if(block_arrive(rz, inst, sc))
      finalize_all(sc, [&](int j, double tot)
      {
        if(active(sc, j) && sc.top[j] == g)
        {
          sc.gamma_prev[j] = sc.gamma[j];
          sc.gamma[j] = tot;
          sc.beta[j] = tot / sc.gamma_prev[j];
        }
      });
  }

  // ---------------------------------------------------------------- staged passes
  // Epilogues of the single-system staged pass (k_tma_pass, fb_tma.cuh) on a global level: the
  // matrix rows stream through shared memory by bulk copies, and each epilogue applies the row body
  // of the one-thread-per-row kernel above (the same arithmetic, so the same values) to the rows of
  // instances in progress.  A row's instance is looked up per warp (instances are padded to whole
  // warps).  Reducing epilogues add each warp's contributions to its instance's accumulator and
  // finish in block_done: one arrival per block; warp 0 of the last block finalises every instance.

  // every lane of a warp calls this for its row (inst < 0: the warp contributes nothing)
  __device__ __forceinline__ void warp_add(double v, int inst, const BScal& sc)
  {
    const double t = warp_sum(v);
    if((threadIdx.x & 31u) == 0 && inst >= 0)
      atomicAdd(&sc.acc[inst], t);
  }

  template<class Fin>
  __device__ __forceinline__ void blocks_done(const BScal& sc, Fin fin)
  {
    __shared__ unsigned int prev_b;
    if((threadIdx.x & 31u) == 0)
      __threadfence();   // this warp's accumulator atomics before the block's arrival
    __syncthreads();
    if(threadIdx.x == 0)
      prev_b = atomicAdd(sc.arrive, 1u);
    __syncthreads();
    if(prev_b != gridDim.x - 1 || threadIdx.x >= 32)
      return;
    __threadfence();
    finalize_all(sc, fin);
  }

  // x' = x + F(D F(b - A x)) (smooth_row); skipped -> 0
  template<typename V, typename S>
  struct BOpSmooth
  {
    typedef typename ValueTraits<V>::acc Ac;
    struct Pre { Ac b, x, di; bool d, on, skip; };
    static constexpr bool REDUCES = false;
    const S* b; const S* x; S* xo; const S* dinv; const uint8_t* dm; const int* sinst; const int* skip; BScal sc;
    __device__ bool closed() const { return bt::closed(sc); }
    __device__ Pre pre(uint32_t i) const
    {
      Pre p{};
      const int j = __ldg(sinst + (i >> 5));
      p.on = active(sc, j);
      if(p.on)
      {
        p.skip = skip[j] != 0;
        p.d = __ldg(dm + i) != 0;
        p.b = Ac(b[i]);
        p.x = Ac(x[i]);
        p.di = Ac(__ldg(dinv + i));
      }
      return p;
    }
    __device__ double operator()(uint32_t i, Ac sum, const Pre& p) const
    {
      if(p.on)
      {
        S out = S(0);
        if(!p.skip)
        {
          const Ac d1 = p.d ? Ac(0) : sub(p.b, sum);
          const Ac c = p.d ? Ac(0) : mul(p.di, d1);
          out = S(add(p.x, c));
        }
        xo[i] = out;
      }
      return 0.0;
    }
    __device__ void finish(double) const {}
  };

  // d = F(b - A x) (defect_row)
  template<typename V, typename S>
  struct BOpDefect
  {
    typedef typename ValueTraits<V>::acc Ac;
    struct Pre { Ac b; bool d, on; };
    static constexpr bool REDUCES = false;
    const S* b; S* dv; const uint8_t* dm; const int* sinst; BScal sc;
    __device__ bool closed() const { return bt::closed(sc); }
    __device__ Pre pre(uint32_t i) const
    {
      Pre p{};
      p.on = active(sc, __ldg(sinst + (i >> 5)));
      if(p.on)
      {
        p.d = __ldg(dm + i) != 0;
        p.b = Ac(b[i]);
      }
      return p;
    }
    __device__ double operator()(uint32_t i, Ac sum, const Pre& p) const
    {
      if(p.on)
        dv[i] = p.d ? S(0) : S(sub(p.b, sum));
      return 0.0;
    }
    __device__ void finish(double) const {}
  };

  // x += F(P x_c) (prolong_row); the gathered vector is the coarse x
  template<typename V, typename S>
  struct BOpProlong
  {
    typedef typename ValueTraits<V>::acc Ac;
    struct Pre { Ac x; bool d, on; };
    static constexpr bool REDUCES = false;
    S* x; const uint8_t* dm; const int* sinst; BScal sc;
    __device__ bool closed() const { return bt::closed(sc); }
    __device__ Pre pre(uint32_t i) const
    {
      Pre p{};
      p.on = active(sc, __ldg(sinst + (i >> 5)));
      if(p.on)
      {
        p.d = __ldg(dm + i) != 0;
        p.x = Ac(x[i]);
      }
      return p;
    }
    __device__ double operator()(uint32_t i, Ac sum, const Pre& p) const
    {
      if(p.on)
      {
        const Ac c = p.d ? Ac(0) : add(sum, Ac(0));
        x[i] = S(add(p.x, c));
      }
      return 0.0;
    }
    __device__ void finish(double) const {}
  };

  // d = F(b - A x), c = F(D d) (post1_calc); per-instance ||d|| -> the post-smoother's skip flag
  template<typename V, typename S>
  struct BOpPost1
  {
    typedef typename ValueTraits<V>::acc Ac;
    struct Pre { Ac b, di; bool d; int j; };
    static constexpr bool REDUCES = false;
    const S* b; S* dv; S* cv; const S* dinv; const uint8_t* dm; const int* sinst; int* skip; BScal sc;
    __device__ bool closed() const { return bt::closed(sc); }
    __device__ Pre pre(uint32_t i) const
    {
      Pre p{};
      const int j = __ldg(sinst + (i >> 5));
      p.j = active(sc, j) ? j : -1;
      if(p.j >= 0)
      {
        p.d = __ldg(dm + i) != 0;
        p.b = Ac(b[i]);
        p.di = Ac(__ldg(dinv + i));
      }
      return p;
    }
    __device__ double operator()(uint32_t i, Ac sum, const Pre& p) const
    {
      double sq = 0.0;
      if(p.j >= 0)
      {
        const Ac d1 = p.d ? Ac(0) : sub(p.b, sum);
        const Ac c1 = p.d ? Ac(0) : mul(p.di, d1);
        dv[i] = S(d1);
        cv[i] = S(add(Ac(0), c1));
        sq = double(d1) * double(d1);
      }
      warp_add(sq, p.j, sc);
      return 0.0;
    }
    __device__ void finish(double) const {}
    __device__ void block_done() const
    {
      int* sk = skip;
      blocks_done(sc, [&](int j, double tot) { sk[j] = skip_from_norm<S>(sqrt(tot)); });
    }
  };

  // post-smoothing step k >= 2 (post2_row) with the gathered c; LAST: x = x + c' (instances whose
  // top is g write z = x * inv_scale and add r.z -> gamma, beta), else c' to co
  template<typename V, typename S, bool LAST>
  struct BOpPost2
  {
    typedef typename ValueTraits<V>::acc Ac;
    struct Pre { Ac d, c, di, x; double r, inv; uint32_t pr; bool dd, skip, top; int j; };
    static constexpr bool REDUCES = false;
    const S* d; const S* c; S* co; S* x; double* z; const double* r; const int* pcg_base; const S* dinv;
    const uint8_t* dm; const int* sinst; int g; const int* skip; BScal sc;
    __device__ bool closed() const { return bt::closed(sc); }
    __device__ Pre pre(uint32_t i) const
    {
      Pre p{};
      const int j = __ldg(sinst + (i >> 5));
      p.j = active(sc, j) ? j : -1;
      if(p.j >= 0)
      {
        p.skip = skip[j] != 0;
        p.dd = __ldg(dm + i) != 0;
        p.d = Ac(d[i]);
        p.c = Ac(c[i]);
        p.di = Ac(__ldg(dinv + i));
        if(LAST)
        {
          p.x = Ac(x[i]);
          p.top = sc.top[j] == g;
          if(p.top)
          {
            p.pr = uint32_t(__ldg(pcg_base + (i >> 5))) + (i & 31u);
            p.r = r[p.pr];
            p.inv = sc.inv_scale[j];
          }
        }
      }
      return p;
    }
    __device__ double operator()(uint32_t i, Ac sum, const Pre& p) const
    {
      double rz = 0.0;
      if(p.j >= 0)
      {
        Ac cn = Ac(0);
        if(!p.skip)
        {
          const Ac dk = p.dd ? Ac(0) : sub(p.d, sum);
          const Ac ck = p.dd ? Ac(0) : mul(p.di, dk);
          cn = add(p.c, ck);
        }
        if(!LAST)
          co[i] = S(cn);
        else
        {
          const S xn = S(add(p.x, cn));
          if(p.top)
          {
            const double zi = mul(double(xn), p.inv);
            z[p.pr] = zi;
            rz = mul(p.r, zi);
          }
          else
            x[i] = xn;
        }
      }
      if(LAST)
        warp_add(rz, p.j >= 0 && p.top ? p.j : -1, sc);
      return 0.0;
    }
    __device__ void finish(double) const {}
    __device__ void block_done() const
    {
      if(!LAST)
        return;
      const BScal& s = sc;
      const int gg = g;
      blocks_done(sc, [&](int j, double tot)
      {
        if(active(s, j) && s.top[j] == gg)
        {
          s.gamma_prev[j] = s.gamma[j];
          s.gamma[j] = tot;
          s.beta[j] = tot / s.gamma_prev[j];
        }
      });
    }
  };

  // b_c = F(R d), sol1_c = F(D_c b_c) (restrict_calc) on coarse rows of instances whose top is not
  // the coarse level; per-instance ||b_c|| -> the coarse pre-smoother's skip flag (xc == null: the
  // coarsest level, no sol1 and no flag)
  template<typename V, typename S>
  struct BOpRestrict
  {
    typedef typename ValueTraits<V>::acc Ac;
    struct Pre { Ac di; bool dc; int j; };
    static constexpr bool REDUCES = false;
    S* bc; S* xc; const S* dinvc; const uint8_t* dmc; const int* sinstc; int gc; int* skipc; BScal sc;
    __device__ bool closed() const { return bt::closed(sc); }
    __device__ Pre pre(uint32_t i) const
    {
      Pre p{};
      const int j = __ldg(sinstc + (i >> 5));
      p.j = (active(sc, j) && sc.top[j] != gc) ? j : -1;
      if(p.j >= 0)
      {
        p.dc = __ldg(dmc + i) != 0;
        if(xc)
          p.di = Ac(__ldg(dinvc + i));
      }
      return p;
    }
    __device__ double operator()(uint32_t i, Ac sum, const Pre& p) const
    {
      double sq = 0.0;
      if(p.j >= 0)
      {
        const Ac v = p.dc ? Ac(0) : add(sum, Ac(0));
        bc[i] = S(v);
        if(xc)
        {
          const Ac c = p.dc ? Ac(0) : mul(p.di, v);
          xc[i] = S(add(Ac(0), c));
        }
        sq = double(v) * double(v);
      }
      if(xc)
        warp_add(sq, p.j, sc);
      return 0.0;
    }
    __device__ void finish(double) const {}
    __device__ void block_done() const
    {
      if(!xc)
        return;
      const BScal& s = sc;
      const int g = gc;
      int* sk = skipc;
      blocks_done(sc, [&](int j, double tot)
      {
        if(active(s, j) && s.top[j] > g)
          sk[j] = skip_from_norm<S>(sqrt(tot));
      });
    }
  };

  // q = F(A p), per-instance q.p -> alpha (FP64, the PCG space)
  struct BOpPcgQ
  {
    struct Pre { double p; bool d; int j; };
    static constexpr bool REDUCES = false;
    double* q; const double* p; const uint8_t* dm; const int* sinst; BScal sc;
    __device__ bool closed() const { return bt::closed(sc); }
    __device__ Pre pre(uint32_t i) const
    {
      Pre r{};
      const int j = __ldg(sinst + (i >> 5));
      r.j = active(sc, j) ? j : -1;
      if(r.j >= 0)
      {
        r.d = dm[i] != 0;
        r.p = p[i];
      }
      return r;
    }
    __device__ double operator()(uint32_t i, double sum, const Pre& pr) const
    {
      double qp = 0.0;
      if(pr.j >= 0)
      {
        const double qv = pr.d ? 0.0 : add(sum, 0.0);
        q[i] = qv;
        qp = mul(qv, pr.p);
      }
      warp_add(qp, pr.j, sc);
      return 0.0;
    }
    __device__ void finish(double) const {}
    __device__ void block_done() const
    {
      const BScal& s = sc;
      blocks_done(sc, [&](int j, double tot)
      {
        if(active(s, j))
          s.alpha[j] = s.gamma[j] / tot;
      });
    }
  };

  // ---------------------------------------------------------------- PCG space
  __device__ __forceinline__ double pow2_inv(double v)
  {
    if(!(v > 0.0) || !isfinite(v))
      return 1.0;
    int e;
    frexp(v, &e);
    return ldexp(1.0, -e);
  }

  __global__ void kb_open(BScal sc)
  {
    for(int j = blockIdx.x * blockDim.x + threadIdx.x; j < sc.J; j += gridDim.x * blockDim.x)
      sc.status[j] = FB_SOLVER_PROGRESS;
    if(blockIdx.x == 0 && threadIdx.x == 0)
      *sc.progress = sc.J;
  }

  __global__ void kb_count(BScal sc, cudaGraphConditionalHandle cond)
  {
    __shared__ int cnt;
    if(threadIdx.x == 0)
      cnt = 0;
    __syncthreads();
    int mine = 0;
    for(int j = threadIdx.x; j < sc.J; j += blockDim.x)
      mine += (sc.status[j] == FB_SOLVER_PROGRESS) ? 1 : 0;
    atomicAdd(&cnt, mine);
    __syncthreads();
    if(threadIdx.x == 0)
    {
      *sc.progress = cnt;
      if(cond)
        cudaGraphSetConditional(cond, cnt > 0 ? 1u : 0u);
    }
  }

  // r = F(rhs - A x), ||r|| -> def_init, status
  __global__ void __launch_bounds__(BNT, 4) kb_pcg_init(DCsr<double> A, const double* __restrict__ rhs,
    const double* __restrict__ x, double* __restrict__ r, const uint8_t* __restrict__ dm, const int* __restrict__ sinst,
    BScal sc)
  {
    const uint32_t i = blockIdx.x * BNT + threadIdx.x;
    int inst = -1;
    double sq = 0.0;
    if((i & ~31u) < A.rows)
    {
      inst = __ldg(sinst + (i >> 5));
      if(i < A.rows)
      {
        const bool dd = dm[i] != 0;
        const double ri = rhs[i];
        const double sum = row_sum<double, double>(A, i, x);
        const double rv = dd ? 0.0 : sub(ri, sum);
        r[i] = rv;
        sq = mul(rv, rv);
      }
    }
    if(block_arrive(sq, inst, sc))
      finalize_all(sc, [&](int j, double tot)
      {
        const double d0 = sqrt(tot);
        sc.def_init[j] = d0;
        sc.def_cur[j] = d0;
        sc.iter[j] = 0;
        sc.gamma[j] = 0.0;
        int st = FB_SOLVER_PROGRESS;
        if(!isfinite(d0))
          st = FB_SOLVER_ABORTED;
        else if(d0 <= EPS64 * EPS64)
          st = FB_SOLVER_SUCCESS;
        sc.status[j] = st;
      });
  }

  // the V-cycle input of every instance at its top level: b = S(r * scale_j), sol1 = F(D .* b);
  // ||b|| -> the top level's pre-smoother skip flag
  template<typename S>
  __global__ void __launch_bounds__(BNT, 4) kb_prep(const double* __restrict__ r, TopPtrs<S> tp,
    const int* __restrict__ mg_base, const uint8_t* __restrict__ dm, const int* __restrict__ sinst, uint32_t n,
    int scale_mode, BScal sc)
  {
    if(closed(sc))
      return;
    const uint32_t i = blockIdx.x * BNT + threadIdx.x;
    int inst = -1;
    double sq = 0.0;
    if((i & ~31u) < n)
    {
      const int j = __ldg(sinst + (i >> 5));
      if(active(sc, j))
      {
        inst = j;
        if(i < n)
        {
          const int g = sc.top[j];
          const double s = scale_mode ? pow2_inv(sc.def_cur[j]) : 1.0;
          const uint32_t mr = uint32_t(__ldg(mg_base + (i >> 5))) + (i & 31u);
          const S b = S(mul(r[i], s));
          tp.b[g][mr] = b;
          const S c = dm[i] ? S(0) : mul(tp.dinv[g][mr], b);
          tp.x[g][mr] = add(S(0), c);
          sq = double(b) * double(b);
        }
      }
    }
    if(block_arrive(sq, inst, sc))
      finalize_all(sc, [&](int j, double tot)
      {
        if(!active(sc, j))
          return;
        const double s = scale_mode ? pow2_inv(sc.def_cur[j]) : 1.0;
        sc.scale[j] = s;
        sc.inv_scale[j] = 1.0 / s;
        sc.skip_pre[sc.top[j] * sc.J + j] = skip_from_norm<S>(sqrt(tot));
      });
  }

  __global__ void __launch_bounds__(BNT, 4) kb_pcg_p(double* __restrict__ p, const double* __restrict__ z,
    const int* __restrict__ sinst, uint32_t n, int first, BScal sc)
  {
    if(closed(sc))
      return;
    const uint32_t i = blockIdx.x * BNT + threadIdx.x;
    if(i >= n)
      return;
    const int j = __ldg(sinst + (i >> 5));
    if(!active(sc, j))
      return;
    p[i] = first ? z[i] : add(mul(p[i], sc.beta[j]), z[i]);
  }

  __global__ void __launch_bounds__(BNT, 4) kb_pcg_q(DCsr<double> A, const double* __restrict__ p, double* __restrict__ q,
    const uint8_t* __restrict__ dm, const int* __restrict__ sinst, BScal sc)
  {
    if(closed(sc))
      return;
    const uint32_t i = blockIdx.x * BNT + threadIdx.x;
    int inst = -1;
    double qp = 0.0;
    if((i & ~31u) < A.rows)
    {
      const int j = __ldg(sinst + (i >> 5));
      if(active(sc, j))
      {
        inst = j;
        if(i < A.rows)
        {
          const bool dd = dm[i] != 0;
          const double pi = p[i];
          const double sum = row_sum<double, double>(A, i, p);
          const double qv = dd ? 0.0 : add(sum, 0.0);
          q[i] = qv;
          qp = mul(qv, pi);
        }
      }
    }
    if(block_arrive(qp, inst, sc))
      finalize_all(sc, [&](int j, double tot)
      {
        if(active(sc, j))
          sc.alpha[j] = sc.gamma[j] / tot;
      });
  }

  // x += alpha p, r -= alpha q, ||r||, stopping test, next V-cycle input at the top level
  template<typename S>
  __global__ void __launch_bounds__(BNT, 4) kb_pcg_x(double* __restrict__ x, double* __restrict__ r,
    const double* __restrict__ p, const double* __restrict__ q, const uint8_t* __restrict__ dm, TopPtrs<S> tp,
    const int* __restrict__ mg_base, const int* __restrict__ sinst, uint32_t n, int scale_mode, BScal sc)
  {
    if(closed(sc))
      return;
    const uint32_t i = blockIdx.x * BNT + threadIdx.x;
    int inst = -1;
    double sq = 0.0;
    if((i & ~31u) < n)
    {
      const int j = __ldg(sinst + (i >> 5));
      if(active(sc, j))
      {
        inst = j;
        if(i < n)
        {
          const double alpha = sc.alpha[j];
          const double s = scale_mode ? pow2_inv(sc.def_cur[j]) : 1.0;
          x[i] = add(x[i], mul(alpha, p[i]));
          const double rv = add(r[i], mul(-alpha, q[i]));
          r[i] = rv;
          const int g = sc.top[j];
          const uint32_t mr = uint32_t(__ldg(mg_base + (i >> 5))) + (i & 31u);
          const S b = S(mul(rv, s));
          tp.b[g][mr] = b;
          const S c = dm[i] ? S(0) : mul(tp.dinv[g][mr], b);
          tp.x[g][mr] = add(S(0), c);
          sq = mul(rv, rv);
        }
      }
    }
    if(block_arrive(sq, inst, sc))
      finalize_all(sc, [&](int j, double tot)
      {
        if(!active(sc, j))
          return;
        const int it = sc.iter[j] + 1;
        const double dc = sqrt(tot);
        const double s = scale_mode ? pow2_inv(sc.def_cur[j]) : 1.0;
        sc.iter[j] = it;
        sc.def_cur[j] = dc;
        int st = FB_SOLVER_PROGRESS;
        if(!isfinite(dc))
          st = FB_SOLVER_ABORTED;
        else if(dc > sc.div_abs || dc > sc.div_rel * sc.def_init[j])
          st = FB_SOLVER_DIVERGED;
        else if(it < sc.min_iter)
          st = FB_SOLVER_PROGRESS;
        else if(dc <= sc.tol_abs && (dc <= sc.tol_rel * sc.def_init[j] || dc <= 0.0))
          st = FB_SOLVER_SUCCESS;
        else if(it >= sc.max_iter)
          st = FB_SOLVER_MAX_ITER;
        sc.status[j] = st;
        sc.scale[j] = s;
        sc.inv_scale[j] = 1.0 / s;
        sc.skip_pre[sc.top[j] * sc.J + j] = skip_from_norm<S>(dc * s);
      });
  }

  __global__ void kb_pack_in(double* __restrict__ dst, const double* __restrict__ src, const int64_t* __restrict__ map,
    uint32_t n)
  {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i < n)
      dst[i] = map[i] >= 0 ? src[map[i]] : 0.0;
  }
  __global__ void kb_pack_out(double* __restrict__ dst, const double* __restrict__ src, const uint32_t* __restrict__ map,
    uint64_t n)
  {
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if(i < n)
      dst[i] = src[map[i]];
  }
} // namespace bt
} // namespace fb

// ==================================================================== host side
struct fb_batch
{
  struct Mat
  {
    uint32_t rows = 0, cols = 0, kw = 0, kmax = 0;
    uint64_t nnz = 0, entries = 0;
    uint32_t* soff = nullptr;
    uint32_t* col = nullptr;
    int16_t* dcol = nullptr;
    int32_t* doff = nullptr;   // diagonal storage: the offsets (no column indices)
    void* val = nullptr;
    double bytes = 0;
  };
  struct GLevel
  {
    uint32_t n = 0;
    Mat A, P, R;          // P: G <- G-1, R: G-1 <- G (G >= 1)
    uint8_t* dm = nullptr;
    void* dinv = nullptr;
    void *b = nullptr, *x = nullptr, *x2 = nullptr, *d = nullptr, *c = nullptr, *c2 = nullptr;
    int* sinst = nullptr;
    int* pcg_base = nullptr;
    std::vector<uint32_t> off;   // per instance row offset (UINT32_MAX: absent)
    int bs = 256;                // rows per block of this level's V-cycle passes (autotuned)
  };
  fb_solver_config cfg;
  int J = 0, NG = 0;
  std::vector<int> top;
  std::vector<GLevel> g;
  std::vector<void*> allocs;
  // PCG space
  uint32_t np = 0;
  Mat Atop;
  uint8_t* dm_top = nullptr;
  int* sinst_top = nullptr;
  int* mg_base_top = nullptr;
  double *x = nullptr, *r = nullptr, *p = nullptr, *q = nullptr, *z = nullptr, *rhs = nullptr;
  std::vector<uint32_t> pcg_off, ntop;
  uint64_t packed = 0;
  int64_t* map_in = nullptr;      // PCG row -> packed index (-1 padding)
  uint32_t* map_out = nullptr;    // packed index -> PCG row
  double *pk_in = nullptr, *pk_out = nullptr;
  // coarse
  uint32_t *c_rowoff = nullptr, *c_nrows = nullptr, *c_free_off = nullptr, *c_free = nullptr;
  uint64_t* c_inv_off = nullptr;
  double* c_inv = nullptr;
  fb::bt::BScal sc{};
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int* err = nullptr;   // a bounded wait of a staged pass expired
  int nsm = 148;
  uint64_t launches_init = 0, launches_body = 0;
  double bytes_init = 0, bytes_body = 0;
};

namespace fb
{
namespace bt
{
  static fb_status bmalloc(fb_batch* s, void** p, size_t bytes)
  {
    cudaError_t e = cudaMalloc(p, bytes + 256);
    if(e != cudaSuccess)
    {
      set_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
      return FB_ERR_NOMEM;
    }
    s->allocs.push_back(*p);
    FB_CUDA(cudaMemset(*p, 0, bytes + 256));
    return FB_OK;
  }

#define BT_TRY(x)                     \
  do {                                \
    fb_status t_ = (x);               \
    if(t_ != FB_OK) return t_;        \
  } while(0)

  template<typename T>
  static fb_status upload_vec(fb_batch* s, T** dst, const std::vector<T>& v)
  {
    BT_TRY(bmalloc(s, (void**)dst, sizeof(T) * std::max<size_t>(1, v.size())));
    if(!v.empty())
      FB_CUDA(cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
    return FB_OK;
  }

  static uint16_t bf16_of(float f)
  {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if((u & 0x7f800000u) == 0x7f800000u)
      return uint16_t(u >> 16) | ((u & 0xffffu) ? 0x40u : 0u);
    u += 0x7fffu + ((u >> 16) & 1u);
    return uint16_t(u >> 16);
  }

  static fb_status upload_mat(fb_batch* s, fb_batch::Mat& d, const HostCsr& M, int prec, const std::vector<uint8_t>* empty,
    bool diag = false)
  {
    const HostSell H = build_sell(M, empty, true, diag);
    const uint32_t ns = (H.rows + 31u) / 32u;
    d.rows = H.rows;
    d.cols = H.cols;
    d.kw = H.kw;
    d.kmax = H.kw;
    for(uint32_t sl = 0; sl + 1 < uint32_t(H.soff.size()); ++sl)
      d.kmax = std::max(d.kmax, (H.soff[sl + 1] - H.soff[sl]) / 32u);
    d.nnz = H.nnz;
    d.entries = H.entries;
    const size_t vb = prec == FB_PREC_F64 ? 8 : (prec == FB_PREC_F32 ? 4 : 2);
    d.bytes = double(H.entries) * double(vb + (!H.doff.empty() ? 0 : (H.narrow ? 2 : 4))) +
              (H.kw ? 0.0 : double(ns + 1) * 4.0);
    BT_TRY(upload_vec(s, &d.soff, H.soff));
    if(!H.doff.empty())
      BT_TRY(upload_vec(s, &d.doff, H.doff));
    else if(H.narrow)
      BT_TRY(upload_vec(s, &d.dcol, H.dcol));
    else
      BT_TRY(upload_vec(s, &d.col, H.col));
    if(prec == FB_PREC_F64)
    {
      double* p = nullptr;
      BT_TRY(upload_vec(s, &p, H.val));
      d.val = p;
    }
    else if(prec == FB_PREC_F32)
    {
      float* p = nullptr;
      BT_TRY(upload_vec(s, &p, std::vector<float>(H.val.begin(), H.val.end())));
      d.val = p;
    }
    else
    {
      std::vector<uint16_t> h(H.val.size());
      for(size_t k = 0; k < h.size(); ++k)
        h[k] = bf16_of(float(H.val[k]));
      uint16_t* p = nullptr;
      BT_TRY(upload_vec(s, &p, h));
      d.val = p;
    }
    return FB_OK;
  }

  constexpr uint32_t STAGED_ROWS = 1000;   // matrices of at least this many rows take the staged passes

  // resident blocks per SM of a staged-pass kernel with `smem` bytes of dynamic shared memory
  static uint32_t staged_resident(const void* kern, size_t smem)
  {
    static std::mutex mu;
    static std::map<std::pair<const void*, size_t>, uint32_t> cache;
    std::lock_guard<std::mutex> g(mu);
    const auto key = std::make_pair(kern, smem);
    const auto it = cache.find(key);
    if(it != cache.end())
      return it->second;
    int nb = 0;
    if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, TMA_NT, smem) != cudaSuccess || nb < 1)
    {
      (void)cudaGetLastError();
      nb = 1;
    }
    cache[key] = uint32_t(nb);
    return uint32_t(nb);
  }

  // dynamic shared memory above 48 KB for every staged-pass instance the batch may launch
  template<typename V, typename S, class Op>
  static fb_status staged_attr()
  {
    const int mx = int(TMA_SMEM_MAX) + 8 * 1024;
    FB_CUDA(cudaFuncSetAttribute(k_tma_pass<V, S, Op, 9, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FB_CUDA(cudaFuncSetAttribute(k_tma_pass<V, S, Op, 9>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FB_CUDA(cudaFuncSetAttribute(k_tma_pass<V, S, Op, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    return FB_OK;
  }
  template<typename V, typename S>
  static fb_status staged_attrs()
  {
    BT_TRY((staged_attr<V, S, BOpSmooth<V, S>>()));
    BT_TRY((staged_attr<V, S, BOpDefect<V, S>>()));
    BT_TRY((staged_attr<V, S, BOpProlong<V, S>>()));
    BT_TRY((staged_attr<V, S, BOpPost1<V, S>>()));
    BT_TRY((staged_attr<V, S, BOpPost2<V, S, true>>()));
    BT_TRY((staged_attr<V, S, BOpPost2<V, S, false>>()));
    BT_TRY((staged_attr<V, S, BOpRestrict<V, S>>()));
    BT_TRY((staged_attr<double, double, BOpPcgQ>()));
    return FB_OK;
  }

  template<typename V> DCsr<V> bview(const fb_batch::Mat& m)
  {
    return DCsr<V>{m.kw ? nullptr : m.soff, m.col, m.dcol, static_cast<const V*>(m.val), m.rows, m.kw, m.doff};
  }

  static unsigned int nblk(uint32_t n) { return std::max(1u, (n + BNT - 1) / BNT); }
  static unsigned int nblk(uint32_t n, int bs) { return std::max(1u, (n + uint32_t(bs) - 1) / uint32_t(bs)); }

  template<typename V, typename S>
  struct BLaunch
  {
    fb_batch* s;
    cudaStream_t st;
    bool dry;
    uint64_t launches = 0;
    double bytes = 0;

    double cb(const fb_batch::Mat& m, double vin, double vout) const
    {
      return m.bytes + double(m.cols) * sizeof(S) + double(m.rows) * sizeof(S) * (vin + vout);
    }

    TopPtrs<S> tops() const
    {
      TopPtrs<S> t;
      std::memset(&t, 0, sizeof(t));
      for(int G = 0; G < s->NG; ++G)
      {
        t.b[G] = (S*)s->g[size_t(G)].b;
        t.x[G] = (S*)s->g[size_t(G)].x;
        t.dinv[G] = (const S*)s->g[size_t(G)].dinv;
      }
      return t;
    }

    // the staged pass serves matrices of at least STAGED_ROWS rows whose stages fit
    static bool use_tma(const fb_batch::Mat& m)
    {
      if(m.rows < STAGED_ROWS || !m.kmax || (m.doff && m.kw != 9))
        return false;
      const uint32_t cb = m.doff ? 0u : (m.dcol ? 2u : 4u);
      return uint64_t(tma_stages<V>()) * tma_stage_bytes<V>(m.kmax, cb) <= TMA_SMEM_MAX;
    }

    // one staged pass (k_tma_pass) over m with gathered vector x and epilogue op: a persistent grid
    // of one wave
    // query_only: look the kernel's residency up (filling the cache outside graph capture), no launch
    template<typename VV, typename XS, class Op>
    void tma(const fb_batch::Mat& m, const void* x, const Op& op, bool query_only = false)
    {
      const uint32_t cb = m.doff ? 0u : (m.dcol ? 2u : 4u);
      const uint32_t nch = (m.rows + TMA_NT - 1) / TMA_NT;
      auto launch = [&](auto kern, size_t sm)
      {
        const uint32_t grid = std::max(1u, std::min(nch, uint32_t(s->nsm) * staged_resident((const void*)kern, sm)));
        if(query_only)
          return;
        kern<<<grid, TMA_NT, sm, st>>>(bview<VV>(m), static_cast<const XS*>(x), m.rows, m.kmax, nullptr, 0u, 0u, 0,
          op, RedSlot{nullptr, nullptr}, s->err);
      };
      if(m.doff)
        launch(k_tma_pass<VV, XS, Op, 9, true>, size_t(tma_stages_dg<VV, true>()) * tma_stage_bytes<VV>(m.kmax, 0u));
      else if(m.kw == 9)
        launch(k_tma_pass<VV, XS, Op, 9>, size_t(tma_stages<VV>()) * tma_stage_bytes<VV>(m.kmax, cb));
      else
        launch(k_tma_pass<VV, XS, Op, 0>, size_t(tma_stages<VV>()) * tma_stage_bytes<VV>(m.kmax, cb));
    }

    // every staged pass the solve launches, looked up once before its launches are captured
    void prime()
    {
      for(int G = 1; G < s->NG; ++G)
      {
        const fb_batch::GLevel& f = s->g[size_t(G)];
        if(use_tma(f.A))
        {
          tma<V, S>(f.A, nullptr, BOpSmooth<V, S>{}, true);
          tma<V, S>(f.A, nullptr, BOpDefect<V, S>{}, true);
          tma<V, S>(f.A, nullptr, BOpPost1<V, S>{}, true);
          tma<V, S>(f.A, nullptr, BOpPost2<V, S, true>{}, true);
          tma<V, S>(f.A, nullptr, BOpPost2<V, S, false>{}, true);
        }
        if(use_tma(f.R))
          tma<V, S>(f.R, nullptr, BOpRestrict<V, S>{}, true);
        if(use_tma(f.P))
          tma<V, S>(f.P, nullptr, BOpProlong<V, S>{}, true);
      }
      if(BLaunch<double, double>::use_tma(s->Atop))
      {
        BLaunch<double, double> d64{s, st, false};
        d64.template tma<double, double>(s->Atop, nullptr, BOpPcgQ{}, true);
      }
    }

    void vcycle()
    {
      const int NG = s->NG;
      const int steps = s->cfg.smooth_steps;
      BScal sc = s->sc;
      std::vector<void*> xcur(static_cast<size_t>(NG));
      for(int G = NG - 1; G >= 1; --G)
      {
        fb_batch::GLevel& f = s->g[size_t(G)];
        fb_batch::GLevel& c = s->g[size_t(G - 1)];
        int* skp = sc.skip_pre + size_t(G) * sc.J;
        void* xa = f.x;
        void* xb = f.x2;
        for(int k = 1; k < steps; ++k)
        {
          if(dry)
            ;
          else if(use_tma(f.A))
            tma<V, S>(f.A, xa, BOpSmooth<V, S>{(const S*)f.b, (const S*)xa, (S*)xb, (const S*)f.dinv, f.dm, f.sinst,
              skp, sc});
          else
            kb_smooth<V, S><<<nblk(f.n, f.bs), f.bs, 0, st>>>(bview<V>(f.A), (const S*)f.b, (const S*)xa, (S*)xb,
              (const S*)f.dinv, f.dm, f.sinst, skp, sc);
          ++launches;
          bytes += cb(f.A, 3, 1);
          std::swap(xa, xb);
        }
        xcur[size_t(G)] = xa;
        if(dry)
          ;
        else if(use_tma(f.A))
          tma<V, S>(f.A, xa, BOpDefect<V, S>{(const S*)f.b, (S*)f.d, f.dm, f.sinst, sc});
        else
          kb_defect<V, S><<<nblk(f.n, f.bs), f.bs, 0, st>>>(bview<V>(f.A), (const S*)f.b, (const S*)xa, (S*)f.d, f.dm,
            f.sinst, sc);
        const bool coarsest = (G - 1 == 0);
        if(dry)
          ;
        else if(use_tma(f.R))
          tma<V, S>(f.R, f.d, BOpRestrict<V, S>{(S*)c.b, coarsest ? (S*)nullptr : (S*)c.x, (const S*)c.dinv, c.dm,
            c.sinst, G - 1, sc.skip_pre + size_t(G - 1) * sc.J, sc});
        else
          kb_restrict<V, S><<<nblk(c.n, c.bs), c.bs, 0, st>>>(bview<V>(f.R), (const S*)f.d, (S*)c.b,
            coarsest ? (S*)nullptr : (S*)c.x, (const S*)c.dinv, c.dm, c.sinst, G - 1,
            sc.skip_pre + size_t(G - 1) * sc.J, sc);
        launches += 2;
        bytes += cb(f.A, 1, 1) + cb(f.R, 0, 3);
      }
      {
        fb_batch::GLevel& c = s->g[0];
        if(!dry)
          kb_coarse<S><<<s->J, BNT, 0, st>>>((const S*)c.b, (S*)c.x, s->c_rowoff, s->c_nrows, s->c_free_off, s->c_free,
            s->c_inv_off, s->c_inv, sc);
        ++launches;
        bytes += double(c.n) * 2 * sizeof(S);
        xcur[0] = c.x;
      }
      for(int G = 1; G < NG; ++G)
      {
        fb_batch::GLevel& f = s->g[size_t(G)];
        void* xf = xcur[size_t(G)];
        int* skq = sc.skip_post + size_t(G) * sc.J;
        if(dry)
          ;
        else
        {
          if(use_tma(f.P))
            tma<V, S>(f.P, xcur[size_t(G - 1)], BOpProlong<V, S>{(S*)xf, f.dm, f.sinst, sc});
          else
            kb_prolong<V, S><<<nblk(f.n, f.bs), f.bs, 0, st>>>(bview<V>(f.P), (const S*)xcur[size_t(G - 1)], (S*)xf,
              f.dm, f.sinst, sc);
          if(use_tma(f.A))
            tma<V, S>(f.A, xf, BOpPost1<V, S>{(const S*)f.b, (S*)f.d, (S*)f.c, (const S*)f.dinv, f.dm, f.sinst, skq,
              sc});
          else
            kb_post1<V, S><<<nblk(f.n, f.bs), f.bs, 0, st>>>(bview<V>(f.A), (const S*)f.b, (const S*)xf, (S*)f.d,
              (S*)f.c, (const S*)f.dinv, f.dm, f.sinst, skq, sc);
        }
        launches += 2;
        bytes += cb(f.P, 1, 1) + cb(f.A, 2, 2);
        void* ca = f.c;
        void* cbuf = f.c2;
        for(int k = 2; k <= steps; ++k)
        {
          const bool last = (k == steps);
          if(dry)
            ;
          else if(use_tma(f.A) && last)
            tma<V, S>(f.A, ca, BOpPost2<V, S, true>{(const S*)f.d, (const S*)ca, (S*)cbuf, (S*)xf, s->z, s->r,
              f.pcg_base, (const S*)f.dinv, f.dm, f.sinst, G, skq, sc});
          else if(use_tma(f.A))
            tma<V, S>(f.A, ca, BOpPost2<V, S, false>{(const S*)f.d, (const S*)ca, (S*)cbuf, (S*)xf, s->z, s->r,
              f.pcg_base, (const S*)f.dinv, f.dm, f.sinst, G, skq, sc});
          else if(last)
            kb_post2<V, S, true><<<nblk(f.n, f.bs), f.bs, 0, st>>>(bview<V>(f.A), (const S*)f.d, (const S*)ca, (S*)cbuf,
              (S*)xf, s->z, s->r, f.pcg_base, (const S*)f.dinv, f.dm, f.sinst, G, skq, sc);
          else
            kb_post2<V, S, false><<<nblk(f.n, f.bs), f.bs, 0, st>>>(bview<V>(f.A), (const S*)f.d, (const S*)ca, (S*)cbuf,
              (S*)xf, s->z, s->r, f.pcg_base, (const S*)f.dinv, f.dm, f.sinst, G, skq, sc);
          ++launches;
          bytes += cb(f.A, 3, 1);
          std::swap(ca, cbuf);
        }
      }
    }

    void init()
    {
      BScal sc = s->sc;
      const bool f64 = s->cfg.precision == FB_PREC_F64;
      if(!dry)
      {
        kb_open<<<4, 256, 0, st>>>(sc);
        kb_pcg_init<<<nblk(s->np), BNT, 0, st>>>(bview<double>(s->Atop), s->rhs, s->x, s->r, s->dm_top, s->sinst_top, sc);
        kb_count<<<1, 256, 0, st>>>(sc, 0);
        kb_prep<S><<<nblk(s->np), BNT, 0, st>>>(s->r, tops(), s->mg_base_top, s->dm_top, s->sinst_top, s->np,
          f64 ? 0 : 1, sc);
      }
      launches += 4;
      bytes += s->Atop.bytes + double(s->np) * 8 * 3 + double(s->np) * (8 + 2 * sizeof(S));
    }

    void tail(bool first, cudaGraphConditionalHandle cond)
    {
      BScal sc = s->sc;
      const bool f64 = s->cfg.precision == FB_PREC_F64;
      if(!dry)
      {
        kb_pcg_p<<<nblk(s->np), BNT, 0, st>>>(s->p, s->z, s->sinst_top, s->np, first ? 1 : 0, sc);
        if(BLaunch<double, double>::use_tma(s->Atop))
        {
          BLaunch<double, double> d64{s, st, false};
          d64.template tma<double, double>(s->Atop, s->p, BOpPcgQ{s->q, s->p, s->dm_top, s->sinst_top, sc});
        }
        else
          kb_pcg_q<<<nblk(s->np), BNT, 0, st>>>(bview<double>(s->Atop), s->p, s->q, s->dm_top, s->sinst_top, sc);
        kb_pcg_x<S><<<nblk(s->np), BNT, 0, st>>>(s->x, s->r, s->p, s->q, s->dm_top, tops(), s->mg_base_top,
          s->sinst_top, s->np, f64 ? 0 : 1, sc);
        kb_count<<<1, 256, 0, st>>>(sc, cond);
      }
      launches += 4;
      bytes += double(s->np) * 8 * 3 + s->Atop.bytes + double(s->np) * 8 * 3 + double(s->np) * (8 * 6 + 2 * sizeof(S));
    }
  };

  // Autotuner: for every global level, the rows per block of its V-cycle passes (64 .. 512, i.e.
  // 2 .. 16 warps of 32 rows) that runs the level's defect pass fastest over all instances present
  // (median of 5 timed launches after 2 untimed ones; the pass writes only the level's defect
  // buffer, which the solve overwrites).  Small levels favour small blocks (more SMs busy), large
  // levels larger ones.
  template<typename V, typename S>
  static fb_status autotune(fb_batch* s)
  {
    cudaStream_t st = s->stream;
    BScal sc = s->sc;
    kb_open<<<4, 256, 0, st>>>(sc);
    FB_LAUNCHED(1);
    const int cand[4] = {64, 128, 256, 512};
    for(int G = 1; G < s->NG; ++G)
    {
      fb_batch::GLevel& f = s->g[size_t(G)];
      float best = 1e30f;
      int pick = 256;
      for(int bs : cand)
      {
        float t[5];
        for(int r = 0; r < 7; ++r)
        {
          FB_CUDA(cudaEventRecord(s->ev0, st));
          // a pass with the per-instance reduction (one arrival per block): it favours larger
          // blocks than a pass without one
          kb_post1<V, S><<<nblk(f.n, bs), bs, 0, st>>>(bview<V>(f.A), (const S*)f.b, (const S*)f.x, (S*)f.d,
            (S*)f.c, (const S*)f.dinv, f.dm, f.sinst, sc.skip_post + size_t(G) * sc.J, sc);
          FB_CUDA(cudaEventRecord(s->ev1, st));
          FB_CUDA(cudaEventSynchronize(s->ev1));
          float ms = 0.f;
          FB_CUDA(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
          if(r >= 2)
            t[r - 2] = ms;
        }
        FB_LAUNCHED(7);
        std::sort(t, t + 5);
        if(t[2] < best * 0.97f)   // a candidate must win by 3% to replace a smaller block size
        {
          best = t[2];
          pick = bs;
        }
      }
      f.bs = pick;
    }
    s->g[0].bs = s->NG > 1 ? s->g[1].bs : 256;
    FB_CUDA(cudaStreamSynchronize(st));
    return FB_OK;
  }

  template<typename V, typename S>
  static fb_status build(fb_batch* s)
  {
    cudaStream_t st = s->stream;
    BT_TRY((staged_attrs<V, S>()));
    if(s->cfg.rows_per_block > 0)
      for(auto& g : s->g)
        g.bs = std::max(32, std::min(BNT_MAX, (s->cfg.rows_per_block + 31) / 32 * 32));
    else
    {
      const fb_status e = autotune<V, S>(s);
      if(e != FB_OK)
        return e;
    }
    {
      BLaunch<V, S> a{s, st, true};
      a.prime();
      a.init();
      a.vcycle();
      a.tail(true, 0);
      s->launches_init = a.launches;
      s->bytes_init = a.bytes;
      BLaunch<V, S> b{s, st, true};
      b.vcycle();
      b.tail(false, 0);
      s->launches_body = b.launches;
      s->bytes_body = b.bytes;
    }
    if(!s->cfg.use_graph)
      return FB_OK;
    FB_CUDA(cudaGraphCreate(&s->graph, 0));
    cudaGraphConditionalHandle cond;
    FB_CUDA(cudaGraphConditionalHandleCreate(&cond, s->graph, 0u, cudaGraphCondAssignDefault));
    FB_CUDA(cudaStreamBeginCaptureToGraph(st, s->graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    {
      BLaunch<V, S> a{s, st, false};
      a.init();
      a.vcycle();
      a.tail(true, cond);
    }
    cudaStreamCaptureStatus cst;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaGraph_t capg = nullptr;
    FB_CUDA(cudaStreamGetCaptureInfo(st, &cst, nullptr, &capg, &deps, &ndeps));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t cnode;
    FB_CUDA(cudaGraphAddNode(&cnode, capg, deps, ndeps, &cp));
    FB_CUDA(cudaStreamUpdateCaptureDependencies(st, &cnode, 1, cudaStreamSetCaptureDependencies));
    cudaGraph_t g_out = nullptr;
    FB_CUDA(cudaStreamEndCapture(st, &g_out));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    FB_CUDA(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    {
      BLaunch<V, S> b{s, st, false};
      b.vcycle();
      b.tail(false, cond);
    }
    cudaGraph_t b_out = nullptr;
    FB_CUDA(cudaStreamEndCapture(st, &b_out));
    FB_CUDA(cudaGraphInstantiate(&s->gexec, s->graph, 0));
    return FB_OK;
  }

  template<typename V, typename S>
  static fb_status run(fb_batch* s)
  {
    cudaStream_t st = s->stream;
    if(s->cfg.use_graph)
    {
      FB_CUDA(cudaGraphLaunch(s->gexec, st));
      return FB_OK;
    }
    BLaunch<V, S> a{s, st, false};
    a.init();
    a.vcycle();
    a.tail(true, 0);
    FB_CUDA(cudaGetLastError());
    while(true)
    {
      int prog = 0;
      FB_CUDA(cudaMemcpyAsync(&prog, s->sc.progress, sizeof(int), cudaMemcpyDeviceToHost, st));
      FB_CUDA(cudaStreamSynchronize(st));
      if(prog <= 0)
        break;
      BLaunch<V, S> b{s, st, false};
      b.vcycle();
      b.tail(false, 0);
      FB_CUDA(cudaGetLastError());
    }
    return FB_OK;
  }

  static fb_status dispatch(fb_batch* s, bool do_build)
  {
    if(s->cfg.precision == FB_PREC_F64)
      return do_build ? build<double, double>(s) : run<double, double>(s);
    if(s->cfg.precision == FB_PREC_F32)
      return do_build ? build<float, float>(s) : run<float, float>(s);
    return do_build ? build<bf16_t, float>(s) : run<bf16_t, float>(s);
  }
} // namespace bt
} // namespace fb

using namespace fb;

extern "C" {

void fb_batch_destroy(fb_batch* s)
{
  if(!s)
    return;
  if(s->gexec) cudaGraphExecDestroy(s->gexec);
  if(s->graph) cudaGraphDestroy(s->graph);
  if(s->ev0) cudaEventDestroy(s->ev0);
  if(s->ev1) cudaEventDestroy(s->ev1);
  if(s->stream) cudaStreamDestroy(s->stream);
  for(void* p : s->allocs)
    cudaFree(p);
  delete s;
}

fb_status fb_batch_rows_per_block(const fb_batch* b, int* rows_per_block, int* num_levels)
{
  if(!b || !num_levels)
  {
    set_error("batch_rows_per_block: bad arguments");
    return FB_ERR_ARG;
  }
  *num_levels = b->NG;
  if(rows_per_block)
    for(int G = 0; G < b->NG; ++G)
      rows_per_block[G] = b->g[size_t(b->NG - 1 - G)].bs;
  return FB_OK;
}

fb_status fb_batch_create(fb_batch** out, int num, fb_hierarchy* const* hs, const fb_solver_config* cfg_in)
{
  if(!out || !hs || num < 1)
  {
    set_error("batch_create: bad arguments");
    return FB_ERR_ARG;
  }
  fb_solver_config cfg;
  if(cfg_in)
    cfg = *cfg_in;
  else
    fb_solver_config_default(&cfg);
  if(cfg.smooth_steps < 2)
  {
    set_error("batch_create: at least 2 smoothing steps");
    return FB_ERR_UNSUPPORTED;
  }
  std::unique_ptr<fb_batch, void (*)(fb_batch*)> s(new fb_batch(), fb_batch_destroy);
  s->cfg = cfg;
  s->J = num;
  const int J = num;
  int NG = 0;
  for(int j = 0; j < J; ++j)
  {
    if(!hs[j] || hs[j]->levels.size() < 2)
    {
      set_error("batch_create: every instance needs a hierarchy of at least 2 levels");
      return FB_ERR_ARG;
    }
    for(const HostLevel& L : hs[j]->levels)
      if(!L.set)
      {
        set_error("batch_create: every level of every instance must be set");
        return FB_ERR_STATE;
      }
    NG = std::max(NG, int(hs[j]->levels.size()));
  }
  if(NG > bt::MAXG)
  {
    set_error("batch_create: too many levels");
    return FB_ERR_UNSUPPORTED;
  }
  s->NG = NG;
  s->top.resize(static_cast<size_t>(J));
  const int prec = cfg.precision;
  const size_t vs = prec == FB_PREC_F64 ? 8 : 4;
  FB_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  FB_CUDA(cudaEventCreate(&s->ev0));
  FB_CUDA(cudaEventCreate(&s->ev1));

  // per instance, per own level: ordering, permuted matrices, masks
  struct Inst
  {
    std::vector<std::vector<uint32_t>> perm, inv;
    std::vector<std::vector<uint8_t>> dm;
  };
  std::vector<Inst> in(static_cast<size_t>(J));
  for(int j = 0; j < J; ++j)
  {
    const fb_hierarchy& h = *hs[j];
    const int L = int(h.levels.size());
    s->top[size_t(j)] = L - 1;
    in[size_t(j)].perm.resize(size_t(L));
    in[size_t(j)].inv.resize(size_t(L));
    in[size_t(j)].dm.resize(size_t(L));
    for(int l = 0; l < L; ++l)
    {
      if(cfg.ordering == FB_ORDER_RCM)
      {
        in[size_t(j)].perm[size_t(l)] = rcm_order(h.levels[size_t(l)].A);
        in[size_t(j)].inv[size_t(l)] = inverse_perm(in[size_t(j)].perm[size_t(l)]);
      }
      const std::vector<uint32_t>& pf = in[size_t(j)].perm[size_t(l)];
      const HostLevel& H = h.levels[size_t(l)];
      in[size_t(j)].dm[size_t(l)].resize(H.A.rows);
      for(uint32_t k = 0; k < H.A.rows; ++k)
        in[size_t(j)].dm[size_t(l)][k] = H.dmask[pf.empty() ? k : pf[k]];
    }
  }
  auto own = [&](int j, int G) { return int(hs[j]->levels.size()) - 1 - G; };   // own level index of global G
  auto r32 = [](uint32_t n) { return (n + 31u) & ~31u; };

  // global levels: offsets, concatenated matrices
  s->g.resize(size_t(NG));
  for(int G = 0; G < NG; ++G)
  {
    fb_batch::GLevel& gl = s->g[size_t(G)];
    gl.off.assign(size_t(J), UINT32_MAX);
    uint32_t n = 0;
    for(int j = 0; j < J; ++j)
    {
      const int l = own(j, G);
      if(l < 0)
        continue;
      gl.off[size_t(j)] = n;
      n += r32(hs[j]->levels[size_t(l)].A.rows);
    }
    gl.n = n;
  }
  std::vector<std::vector<uint8_t>> gdm(static_cast<size_t>(NG));
  for(int G = 0; G < NG; ++G)
  {
    fb_batch::GLevel& gl = s->g[size_t(G)];
    HostCsr A, P, R;
    A.rows = A.cols = gl.n;
    A.rp.assign(size_t(gl.n) + 1, 0);
    std::vector<uint8_t>& dm = gdm[size_t(G)];
    dm.assign(gl.n, 1);
    std::vector<double> dinv(gl.n, 0.0);
    std::vector<int> sinst(gl.n / 32, 0);
    std::vector<int> pcg_base(gl.n / 32, -1);
    const bool has_t = G >= 1;
    if(has_t)
    {
      P.rows = gl.n;
      P.cols = s->g[size_t(G - 1)].n;
      P.rp.assign(size_t(gl.n) + 1, 0);
      R.rows = s->g[size_t(G - 1)].n;
      R.cols = gl.n;
      R.rp.assign(size_t(R.rows) + 1, 0);
    }
    // rows of A and P (level G), in instance order; R rows (level G-1) likewise
    uint32_t row = 0;
    for(int j = 0; j < J; ++j)
    {
      const int l = own(j, G);
      if(l < 0)
        continue;
      const HostLevel& H = hs[j]->levels[size_t(l)];
      const std::vector<uint32_t>& pf = in[size_t(j)].perm[size_t(l)];
      const std::vector<uint32_t>& ivf = in[size_t(j)].inv[size_t(l)];
      const HostCsr Aj = permute(H.A, pf, ivf);
      const std::vector<double> dj = inv_diagonal(Aj, cfg.omega);
      const uint32_t o = gl.off[size_t(j)];
      for(uint32_t r = 0; r < Aj.rows; ++r)
      {
        for(uint32_t k = Aj.rp[r]; k < Aj.rp[r + 1]; ++k)
        {
          A.col.push_back(o + Aj.col[k]);
          A.val.push_back(Aj.val[k]);
        }
        A.rp[size_t(o + r) + 1] = uint32_t(A.col.size());
        dm[o + r] = in[size_t(j)].dm[size_t(l)][r];
        dinv[o + r] = dj[r];
      }
      for(uint32_t r = Aj.rows; r < r32(Aj.rows); ++r)
        A.rp[size_t(o + r) + 1] = uint32_t(A.col.size());
      for(uint32_t sl = o / 32; sl < (o + r32(Aj.rows)) / 32; ++sl)
        sinst[sl] = j;
      if(G == s->top[size_t(j)])
        for(uint32_t sl = o / 32; sl < (o + r32(Aj.rows)) / 32; ++sl)
          pcg_base[sl] = int(sl * 32 - o);   // relative; made absolute with pcg_off below
      if(has_t)
      {
        const int lc = l + 1;   // own coarser level
        const std::vector<uint32_t>& pc = in[size_t(j)].perm[size_t(lc)];
        const std::vector<uint32_t>& ivc = in[size_t(j)].inv[size_t(lc)];
        const HostCsr Pj = permute(H.P, pf, ivc);
        const uint32_t oc = s->g[size_t(G - 1)].off[size_t(j)];
        for(uint32_t r = 0; r < Pj.rows; ++r)
        {
          for(uint32_t k = Pj.rp[r]; k < Pj.rp[r + 1]; ++k)
          {
            P.col.push_back(oc + Pj.col[k]);
            P.val.push_back(Pj.val[k]);
          }
          P.rp[size_t(o + r) + 1] = uint32_t(P.col.size());
        }
        for(uint32_t r = Pj.rows; r < r32(Pj.rows); ++r)
          P.rp[size_t(o + r) + 1] = uint32_t(P.col.size());
      }
      row = o + r32(Aj.rows);
    }
    (void)row;
    if(has_t)
    {
      // R rows live on level G-1: instances in level G-1 order (those present at G have R)
      const fb_batch::GLevel& gc = s->g[size_t(G - 1)];
      for(int j = 0; j < J; ++j)
      {
        const int lc = own(j, G - 1);
        if(lc < 0)
          continue;
        const uint32_t oc = gc.off[size_t(j)];
        const uint32_t nc = hs[j]->levels[size_t(lc)].A.rows;
        const int l = own(j, G);
        if(l >= 0)
        {
          const HostLevel& H = hs[j]->levels[size_t(l)];
          const HostCsr Rj = permute(H.R, in[size_t(j)].perm[size_t(lc)], in[size_t(j)].inv[size_t(l)]);
          const uint32_t o = gl.off[size_t(j)];
          for(uint32_t r = 0; r < Rj.rows; ++r)
          {
            for(uint32_t k = Rj.rp[r]; k < Rj.rp[r + 1]; ++k)
            {
              R.col.push_back(o + Rj.col[k]);
              R.val.push_back(Rj.val[k]);
            }
            R.rp[size_t(oc + r) + 1] = uint32_t(R.col.size());
          }
        }
        else
          for(uint32_t r = 0; r < nc; ++r)
            R.rp[size_t(oc + r) + 1] = uint32_t(R.col.size());
        for(uint32_t r = nc; r < r32(nc); ++r)
          R.rp[size_t(oc + r) + 1] = uint32_t(R.col.size());
      }
    }
    BT_TRY(bt::upload_mat(s.get(), gl.A, A, prec, &dm, cfg.diagonal != 0));
    if(has_t)
    {
      BT_TRY(bt::upload_mat(s.get(), gl.P, P, prec, &dm));
      BT_TRY(bt::upload_mat(s.get(), gl.R, R, prec, &gdm[size_t(G - 1)]));
    }
    BT_TRY(bt::upload_vec(s.get(), &gl.dm, dm));
    if(prec == FB_PREC_F64)
    {
      double* p = nullptr;
      BT_TRY(bt::upload_vec(s.get(), &p, dinv));
      gl.dinv = p;
    }
    else
    {
      float* p = nullptr;
      BT_TRY(bt::upload_vec(s.get(), &p, std::vector<float>(dinv.begin(), dinv.end())));
      gl.dinv = p;
    }
    for(void** v : {&gl.b, &gl.x, &gl.x2, &gl.d, &gl.c, &gl.c2})
      BT_TRY(bt::bmalloc(s.get(), v, vs * size_t(gl.n)));
    BT_TRY(bt::upload_vec(s.get(), &gl.sinst, sinst));
    // pcg_base stays relative until the PCG space exists
    std::vector<int> pb(pcg_base);
    s->g[size_t(G)].pcg_base = nullptr;
    gl.pcg_base = nullptr;
    s->g[size_t(G)].off = gl.off;
    // stash relative bases
    if(true)
    {
      int* d = nullptr;
      BT_TRY(bt::upload_vec(s.get(), &d, pb));
      gl.pcg_base = d;
    }
  }

  // PCG space: concatenated top levels
  s->pcg_off.assign(size_t(J), 0);
  s->ntop.assign(size_t(J), 0);
  uint32_t np = 0;
  for(int j = 0; j < J; ++j)
  {
    s->pcg_off[size_t(j)] = np;
    s->ntop[size_t(j)] = hs[j]->levels[0].A.rows;
    np += r32(s->ntop[size_t(j)]);
  }
  s->np = np;
  {
    HostCsr A;
    A.rows = A.cols = np;
    A.rp.assign(size_t(np) + 1, 0);
    std::vector<uint8_t> dm(np, 1);
    std::vector<int> sinst(np / 32, 0), mgb(np / 32, 0);
    std::vector<int64_t> map_in(np, -1);
    std::vector<uint32_t> map_out;
    uint64_t packed = 0;
    for(int j = 0; j < J; ++j)
    {
      const HostLevel& H = hs[j]->levels[0];
      const std::vector<uint32_t>& pf = in[size_t(j)].perm[0];
      const std::vector<uint32_t>& ivf = in[size_t(j)].inv[0];
      const HostCsr Aj = permute(H.A, pf, ivf);
      const uint32_t o = s->pcg_off[size_t(j)];
      for(uint32_t r = 0; r < Aj.rows; ++r)
      {
        for(uint32_t k = Aj.rp[r]; k < Aj.rp[r + 1]; ++k)
        {
          A.col.push_back(o + Aj.col[k]);
          A.val.push_back(Aj.val[k]);
        }
        A.rp[size_t(o + r) + 1] = uint32_t(A.col.size());
        dm[o + r] = in[size_t(j)].dm[0][r];
        map_in[o + r] = int64_t(packed + (pf.empty() ? r : pf[r]));
      }
      for(uint32_t r = Aj.rows; r < r32(Aj.rows); ++r)
        A.rp[size_t(o + r) + 1] = uint32_t(A.col.size());
      for(uint32_t k = 0; k < Aj.rows; ++k)
        map_out.push_back(o + (ivf.empty() ? k : ivf[k]));
      const uint32_t omg = s->g[size_t(s->top[size_t(j)])].off[size_t(j)];
      for(uint32_t sl = o / 32; sl < (o + r32(Aj.rows)) / 32; ++sl)
      {
        sinst[sl] = j;
        mgb[sl] = int(omg + (sl * 32 - o));
      }
      packed += Aj.rows;
    }
    s->packed = packed;
    BT_TRY(bt::upload_mat(s.get(), s->Atop, A, FB_PREC_F64, &dm, cfg.diagonal != 0));
    BT_TRY(bt::upload_vec(s.get(), &s->dm_top, dm));
    BT_TRY(bt::upload_vec(s.get(), &s->sinst_top, sinst));
    BT_TRY(bt::upload_vec(s.get(), &s->mg_base_top, mgb));
    BT_TRY(bt::upload_vec(s.get(), &s->map_in, map_in));
    BT_TRY(bt::upload_vec(s.get(), &s->map_out, map_out));
    for(double** v : {&s->x, &s->r, &s->p, &s->q, &s->z, &s->rhs})
      BT_TRY(bt::bmalloc(s.get(), (void**)v, 8 * size_t(np)));
    BT_TRY(bt::bmalloc(s.get(), (void**)&s->pk_in, 8 * size_t(packed)));
    BT_TRY(bt::bmalloc(s.get(), (void**)&s->pk_out, 8 * size_t(packed)));
  }
  // absolute PCG bases of the top-level slices of every global level
  for(int G = 0; G < NG; ++G)
  {
    fb_batch::GLevel& gl = s->g[size_t(G)];
    std::vector<int> pb(gl.n / 32, -1);
    for(int j = 0; j < J; ++j)
      if(s->top[size_t(j)] == G && gl.off[size_t(j)] != UINT32_MAX)
      {
        const uint32_t o = gl.off[size_t(j)];
        const uint32_t nj = r32(hs[j]->levels[0].A.rows);
        for(uint32_t sl = o / 32; sl < (o + nj) / 32; ++sl)
          pb[sl] = int(s->pcg_off[size_t(j)] + (sl * 32 - o));
      }
    if(!pb.empty())
      FB_CUDA(cudaMemcpy(gl.pcg_base, pb.data(), sizeof(int) * pb.size(), cudaMemcpyHostToDevice));
  }
  // coarse: per instance exact inverse on its coarsest level (global level 0)
  {
    std::vector<uint32_t> rowoff(static_cast<size_t>(J)), nrows(static_cast<size_t>(J)), free_off(static_cast<size_t>(J) + 1, 0), fr_all;
    std::vector<uint64_t> inv_off(static_cast<size_t>(J) + 1, 0);
    std::vector<double> inv_all;
    for(int j = 0; j < J; ++j)
    {
      const int lc = int(hs[j]->levels.size()) - 1;
      const HostLevel& H = hs[j]->levels[size_t(lc)];
      std::vector<uint32_t> fr;
      std::vector<double> inv;
      coarse_inverse(H.A, H.dmask, fr, inv);
      const std::vector<uint32_t>& ivc = in[size_t(j)].inv[size_t(lc)];
      for(uint32_t& f : fr)
        f = ivc.empty() ? f : ivc[f];
      rowoff[size_t(j)] = s->g[0].off[size_t(j)];
      nrows[size_t(j)] = H.A.rows;
      fr_all.insert(fr_all.end(), fr.begin(), fr.end());
      free_off[size_t(j) + 1] = uint32_t(fr_all.size());
      inv_all.insert(inv_all.end(), inv.begin(), inv.end());
      inv_off[size_t(j) + 1] = inv_all.size();
    }
    BT_TRY(bt::upload_vec(s.get(), &s->c_rowoff, rowoff));
    BT_TRY(bt::upload_vec(s.get(), &s->c_nrows, nrows));
    BT_TRY(bt::upload_vec(s.get(), &s->c_free_off, free_off));
    BT_TRY(bt::upload_vec(s.get(), &s->c_free, fr_all));
    BT_TRY(bt::upload_vec(s.get(), &s->c_inv_off, inv_off));
    BT_TRY(bt::upload_vec(s.get(), &s->c_inv, inv_all));
  }
  // per instance scalars
  {
    bt::BScal& sc = s->sc;
    sc.J = J;
    for(double** v : {&sc.gamma, &sc.gamma_prev, &sc.alpha, &sc.beta, &sc.def_init, &sc.def_cur, &sc.scale,
                      &sc.inv_scale, &sc.acc})
      BT_TRY(bt::bmalloc(s.get(), (void**)v, 8 * size_t(J)));
    BT_TRY(bt::bmalloc(s.get(), (void**)&sc.iter, 4 * size_t(J)));
    BT_TRY(bt::bmalloc(s.get(), (void**)&sc.status, 4 * size_t(J)));
    BT_TRY(bt::upload_vec(s.get(), &sc.top, s->top));
    BT_TRY(bt::bmalloc(s.get(), (void**)&sc.skip_pre, 4 * size_t(bt::MAXG) * J));
    BT_TRY(bt::bmalloc(s.get(), (void**)&sc.skip_post, 4 * size_t(bt::MAXG) * J));
    BT_TRY(bt::bmalloc(s.get(), (void**)&sc.arrive, 64));
    BT_TRY(bt::bmalloc(s.get(), (void**)&sc.progress, 64));
    BT_TRY(bt::bmalloc(s.get(), (void**)&s->err, 64));
    int dev = 0;
    FB_CUDA(cudaGetDevice(&dev));
    FB_CUDA(cudaDeviceGetAttribute(&s->nsm, cudaDevAttrMultiProcessorCount, dev));
    sc.tol_rel = cfg.tol_rel;
    sc.tol_abs = cfg.tol_abs;
    sc.div_rel = 1.0 / EPS64;
    sc.div_abs = 1.0 / (EPS64 * EPS64);
    sc.min_iter = cfg.min_iter;
    sc.max_iter = cfg.max_iter;
  }
  BT_TRY(bt::dispatch(s.get(), true));
  FB_CUDA(cudaDeviceSynchronize());
  *out = s.release();
  return FB_OK;
}

fb_status fb_batch_sizes(const fb_batch* s, uint64_t* top_rows)
{
  if(!s || !top_rows)
  {
    set_error("batch_sizes: bad arguments");
    return FB_ERR_ARG;
  }
  for(int j = 0; j < s->J; ++j)
    top_rows[j] = s->ntop[size_t(j)];
  return FB_OK;
}

static fb_status batch_common(fb_batch* s, fb_solve_info* info)
{
  cudaStream_t st = s->stream;
  FB_CUDA(cudaEventRecord(s->ev0, st));
  BT_TRY(bt::dispatch(s, false));
  FB_CUDA(cudaEventRecord(s->ev1, st));
  const int J = s->J;
  std::vector<int> iter(static_cast<size_t>(J)), status(static_cast<size_t>(J));
  std::vector<double> d0(static_cast<size_t>(J)), d1(static_cast<size_t>(J));
  FB_CUDA(cudaMemcpyAsync(iter.data(), s->sc.iter, 4 * size_t(J), cudaMemcpyDeviceToHost, st));
  FB_CUDA(cudaMemcpyAsync(status.data(), s->sc.status, 4 * size_t(J), cudaMemcpyDeviceToHost, st));
  FB_CUDA(cudaMemcpyAsync(d0.data(), s->sc.def_init, 8 * size_t(J), cudaMemcpyDeviceToHost, st));
  FB_CUDA(cudaMemcpyAsync(d1.data(), s->sc.def_cur, 8 * size_t(J), cudaMemcpyDeviceToHost, st));
  int err = 0;
  FB_CUDA(cudaMemcpyAsync(&err, s->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  FB_CUDA(cudaStreamSynchronize(st));
  if(err)
  {
    FB_CUDA(cudaMemsetAsync(s->err, 0, sizeof(int), st));
    set_error("batch_solve: a bounded wait for staged matrix data expired (results invalid)");
    return FB_ERR_CUDA;
  }
  float ms = 0.f;
  FB_CUDA(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
  int maxit = 0;
  for(int j = 0; j < J; ++j)
    maxit = std::max(maxit, iter[size_t(j)]);
  const uint64_t body = maxit > 1 ? uint64_t(maxit - 1) : 0;
  const uint64_t launches = s->launches_init + body * s->launches_body;
  count_launches(launches);
  if(info)
    for(int j = 0; j < J; ++j)
    {
      info[j].status = status[size_t(j)];
      info[j].iterations = iter[size_t(j)];
      info[j].def_init = d0[size_t(j)];
      info[j].def_final = d1[size_t(j)];
      info[j].solve_ms = double(ms);
      info[j].kernel_launches = launches;
      info[j].bytes_moved = s->bytes_init + double(body) * s->bytes_body;
    }
  return FB_OK;
}

fb_status fb_batch_solve_device(fb_batch* s, double* sol, const double* rhs, void* stream, fb_solve_info* info)
{
  if(!s || !sol || !rhs)
  {
    set_error("batch_solve_device: bad arguments");
    return FB_ERR_ARG;
  }
  cudaStream_t cs = as_stream(stream);
  cudaEvent_t ev;
  FB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  FB_CUDA(cudaEventRecord(ev, cs));
  FB_CUDA(cudaStreamWaitEvent(s->stream, ev, 0));
  const unsigned int gb = unsigned((s->np + 255) / 256);
  bt::kb_pack_in<<<gb, 256, 0, s->stream>>>(s->rhs, rhs, s->map_in, s->np);
  bt::kb_pack_in<<<gb, 256, 0, s->stream>>>(s->x, sol, s->map_in, s->np);
  FB_LAUNCHED(2);
  fb_status e = batch_common(s, info);
  if(e == FB_OK)
  {
    bt::kb_pack_out<<<unsigned((s->packed + 255) / 256), 256, 0, s->stream>>>(sol, s->x, s->map_out, s->packed);
    FB_LAUNCHED(1);
  }
  FB_CUDA(cudaEventRecord(ev, s->stream));
  FB_CUDA(cudaStreamWaitEvent(cs, ev, 0));
  FB_CUDA(cudaStreamSynchronize(s->stream));
  cudaEventDestroy(ev);
  return e;
}

fb_status fb_batch_solve(fb_batch* s, double* sol, const double* rhs, fb_solve_info* info)
{
  if(!s || !sol || !rhs)
  {
    set_error("batch_solve: bad arguments");
    return FB_ERR_ARG;
  }
  FB_CUDA(cudaMemcpyAsync(s->pk_in, rhs, 8 * s->packed, cudaMemcpyHostToDevice, s->stream));
  FB_CUDA(cudaMemcpyAsync(s->pk_out, sol, 8 * s->packed, cudaMemcpyHostToDevice, s->stream));
  FB_CUDA(cudaStreamSynchronize(s->stream));
  BT_TRY(fb_batch_solve_device(s, s->pk_out, s->pk_in, s->stream, info));
  FB_CUDA(cudaMemcpyAsync(sol, s->pk_out, 8 * s->packed, cudaMemcpyDeviceToHost, s->stream));
  FB_CUDA(cudaStreamSynchronize(s->stream));
  return FB_OK;
}

} // extern "C"
