// Solver level: PCG preconditioned by a geometric-multigrid V-cycle, fully device resident.
//
// The V(s,s) cycle with Richardson(1)+Jacobi(omega) smoothing of the reference
// (kernel/solver/multigrid.hpp:1270-2000, kernel/solver/richardson.hpp:160-228,
// kernel/solver/jacobi_precond.hpp:136-165) is executed as a fixed sequence of fused passes, each
// one CSR sweep over one level with its element-wise work folded in (one thread per row, the
// block's slice of the matrix staged in shared memory with 16-byte loads):
//
//   down, level l (rhs b given, sol1 = F(D.*b) written by the producer of b):
//     SMOOTH   (s-1 times)  x' = x + F(D .* F(b - A x))          Richardson steps 2..s
//     DEFECT               d  = F(b - A x)                       MultiGrid defect (equals the
//                                                                 smoother's own last defect)
//     RESTRICT (coarse rows) b_c = F_c(R d), sol1_c = F_c(D_c .* b_c), ||b_c||
//   coarsest: COARSE       x_c = exact inverse on the free DOFs
//   up, level l:
//     PROLONG              x  = x + F(P x_c)
//     POST1                d  = F(b - A x), c = F(D .* d), ||d||  Richardson step 1
//     POST2    (s-1 times) c' = c + F(D .* F(d - A c)); last: x = x + c'
//
// F zeroes Dirichlet rows (UnitFilter::filter_def/filter_cor).  Richardson's trailing defect of the
// post-smoother is never read by the reference and is not computed.  Every product and sum is
// rounded separately (no FMA), and rows are summed in stored entry order, so for FP64 each pass
// reproduces the reference's generic backend bit for bit; only the global dot products and norms
// are summed in a different (tree) order.
//
// PCG (kernel/solver/pcg.hpp:159-286) adds three passes per iteration: Q (q = F(A p), q.p ->
// alpha), X (x += alpha p, r -= alpha q, ||r||, convergence test, next V-cycle input) and P
// (p = z + beta p; r.z and beta come out of the top level's last POST2).  All scalars stay on the
// device; with use_graph the whole solve is one CUDA graph whose loop is a device-side WHILE node.
#include "fb_common.cuh"
#include "fb_rows.cuh"
#include "fb_tma.cuh"
#include "fb_setup.h"
#include <cstddef>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <memory>
#include <vector>

namespace fb
{
  constexpr int NT = 256;   // rows (threads) per block of every pass

  struct Scalars
  {
    double gamma, gamma_prev, alpha, beta;
    double def_init, def_cur;
    double tol_rel, tol_abs, div_rel, div_abs;
    double mg_scale, mg_inv_scale;   // V-cycle input scaling (power of two; 1 in FP64 mode)
    int iter, status, min_iter, max_iter;
  };

  __device__ __forceinline__ bool gate_closed(const Scalars* sc)
  {
    return sc->status != FB_SOLVER_PROGRESS;
  }

  template<typename V, typename S>
  __global__ void __launch_bounds__(NT) k_smooth(DCsr<V> A, const S* __restrict__ b, const S* __restrict__ x,
    S* __restrict__ xo, const S* __restrict__ dinv, const uint8_t* __restrict__ dm, const int* __restrict__ skip,
    const Scalars* __restrict__ sc)
  {
    pdl_wait();
    if(gate_closed(sc))
      return;
    const uint32_t i = blockIdx.x * NT + threadIdx.x;
    if(i >= A.rows)
      return;
    xo[i] = smooth_row<V, S, true>(A, b, x, dinv, dm, *skip != 0, i);
  }

  template<typename V, typename S>
  __global__ void __launch_bounds__(NT) k_defect(DCsr<V> A, const S* __restrict__ b, const S* __restrict__ x,
    S* __restrict__ d, const uint8_t* __restrict__ dm, const Scalars* __restrict__ sc)
  {
    pdl_wait();
    if(gate_closed(sc))
      return;
    const uint32_t i = blockIdx.x * NT + threadIdx.x;
    if(i >= A.rows)
      return;
    d[i] = defect_row<V, S, true>(A, b, x, dm, i);
  }

  // coarse rows: b_c = F_c(R d); with xc: sol1_c = F_c(D_c .* b_c) and ||b_c|| -> skip flag
  template<typename V, typename S>
  __global__ void __launch_bounds__(NT) k_restrict(DCsr<V> R, const S* __restrict__ d, S* __restrict__ bc,
    S* __restrict__ xc, const S* __restrict__ dinvc, const uint8_t* __restrict__ dmc, int* __restrict__ skipc,
    RedSlot slot, const Scalars* __restrict__ sc)
  {
    pdl_wait();
    __shared__ double sh[32];
    if(gate_closed(sc))
      return;
    const uint32_t j = blockIdx.x * NT + threadIdx.x;
    double sq = 0.0;
    if(j < R.rows)
      sq = restrict_row<V, S, true>(R, d, bc, xc, dinvc, dmc, j);
    if(!xc)
      return;
    double total;
    if(grid_sum_last<NT>(sq, slot, sh, total))
      *skipc = skip_from_norm<S>(sqrt(total));
  }

  template<typename S>
  __global__ void __launch_bounds__(NT) k_coarse(const S* __restrict__ b, S* __restrict__ x, uint32_t n,
    const uint32_t* __restrict__ free_dofs, const double* __restrict__ inv, uint32_t m, const Scalars* __restrict__ sc)
  {
    pdl_wait();
    if(gate_closed(sc))
      return;
    coarse_block<S, NT>(b, x, n, free_dofs, inv, m);
  }

  template<typename V, typename S>
  __global__ void __launch_bounds__(NT) k_prolong(DCsr<V> P, const S* __restrict__ xc, S* __restrict__ x,
    const uint8_t* __restrict__ dm, const Scalars* __restrict__ sc)
  {
    pdl_wait();
    if(gate_closed(sc))
      return;
    const uint32_t i = blockIdx.x * NT + threadIdx.x;
    if(i >= P.rows)
      return;
    x[i] = prolong_row<V, S, true>(P, xc, x, dm, i);
  }

  template<typename V, typename S>
  __global__ void __launch_bounds__(NT) k_post1(DCsr<V> A, const S* __restrict__ b, const S* __restrict__ x,
    S* __restrict__ d, S* __restrict__ c, const S* __restrict__ dinv, const uint8_t* __restrict__ dm,
    int* __restrict__ skip, RedSlot slot, const Scalars* __restrict__ sc)
  {
    pdl_wait();
    __shared__ double sh[32];
    if(gate_closed(sc))
      return;
    const uint32_t i = blockIdx.x * NT + threadIdx.x;
    double sq = 0.0;
    if(i < A.rows)
      sq = post1_row<V, S, true>(A, b, x, d, c, dinv, dm, i);
    double total;
    if(grid_sum_last<NT>(sq, slot, sh, total))
      *skip = skip_from_norm<S>(sqrt(total));
  }

  // post-smoothing step k >= 2.  LAST: x += c'.  TOP (with LAST): z = x * inv_scale (FP64), and
  // r.z -> gamma, beta (PCG).
  template<typename V, typename S, bool LAST, bool TOP>
  __global__ void __launch_bounds__(NT) k_post2(DCsr<V> A, const S* __restrict__ d, const S* __restrict__ c,
    S* __restrict__ co, S* __restrict__ x, double* __restrict__ z, const double* __restrict__ r,
    const S* __restrict__ dinv, const uint8_t* __restrict__ dm, const int* __restrict__ skip, RedSlot slot,
    Scalars* __restrict__ sc)
  {
    pdl_wait();
    typedef typename ValueTraits<V>::acc Ac;
    __shared__ double sh[32];
    if(gate_closed(sc))
      return;
    const uint32_t i = blockIdx.x * NT + threadIdx.x;
    const bool skipped = *skip != 0;
    double rz = 0.0;
    if(i < A.rows)
    {
      const Ac cn = post2_row<V, S, true>(A, d, c, dinv, dm, skipped, i);
      if(!LAST)
        co[i] = S(cn);
      else
      {
        const S xn = S(add(Ac(x[i]), cn));
        if(TOP)
        {
          const double zi = mul(double(xn), sc->mg_inv_scale);
          z[i] = zi;
          rz = mul(r[i], zi);
        }
        else
          x[i] = xn;
      }
    }
    if(!(LAST && TOP))
      return;
    double total;
    if(grid_sum_last<NT>(rz, slot, sh, total))
    {
      sc->gamma_prev = sc->gamma;
      sc->gamma = total;
      sc->beta = total / sc->gamma_prev;
    }
  }

  // post-smoothing with a single step: x += c (skip -> x += 0).  TOP as above.
  template<typename S, bool TOP>
  __global__ void __launch_bounds__(NT) k_post_final(const S* __restrict__ c, S* __restrict__ x, double* __restrict__ z,
    const double* __restrict__ r, const int* __restrict__ skip, uint32_t n, RedSlot slot, Scalars* __restrict__ sc)
  {
    pdl_wait();
    typedef S Ac;
    __shared__ double sh[32];
    if(gate_closed(sc))
      return;
    const uint32_t i = blockIdx.x * NT + threadIdx.x;
    double rz = 0.0;
    if(i < n)
    {
      const Ac cn = *skip ? Ac(0) : c[i];
      const S xn = S(add(Ac(x[i]), cn));
      if(TOP)
      {
        const double zi = mul(double(xn), sc->mg_inv_scale);
        z[i] = zi;
        rz = mul(r[i], zi);
      }
      else
        x[i] = xn;
    }
    if(!TOP)
      return;
    double total;
    if(grid_sum_last<NT>(rz, slot, sh, total))
    {
      sc->gamma_prev = sc->gamma;
      sc->gamma = total;
      sc->beta = total / sc->gamma_prev;
    }
  }

  // ------------------------------------------------------------------ adaptive coarse-grid correction
  // MultiGrid::_apply_prol with MultiGridAdaptCGC::MinEnergy / MinDefect (multigrid.hpp:1880-1960):
  // cor = F(P x_c); tmp = F(A cor); w = (d, cor) / (tmp, cor) or (d, tmp) / (tmp, tmp); x += w cor;
  // d += -w tmp; the post-smoother then starts from that defect.  One thread per row.

  // cor = F(P x_c)
  template<typename V, typename S>
  __global__ void __launch_bounds__(NT) k_cgc_prolong(DCsr<V> P, const S* __restrict__ xc, S* __restrict__ cor,
    const uint8_t* __restrict__ dm, const Scalars* __restrict__ sc)
  {
    typedef typename ValueTraits<V>::acc Ac;
    pdl_wait();
    if(gate_closed(sc))
      return;
    const uint32_t i = blockIdx.x * NT + threadIdx.x;
    if(i >= P.rows)
      return;
    const bool d = __ldg(dm + i) != 0;
    const Ac sum = row_sum<V, S, true>(P, i, xc);
    cor[i] = d ? S(0) : S(add(sum, Ac(0)));
  }

  // the two dot products of the step length for row i
  template<int MODE>
  __device__ __forceinline__ void cgc_dots(double d, double c, double t, double& a, double& b)
  {
    if(MODE == FB_CGC_MIN_ENERGY)
    {
      a = d * c;
      b = t * c;
    }
    else
    {
      a = d * t;
      b = t * t;
    }
  }

  // tmp = F(A cor) and w = a / b into *omega
  template<typename V, typename S, int MODE>
  __global__ void __launch_bounds__(NT) k_cgc_apply(DCsr<V> A, const S* __restrict__ cor, const S* __restrict__ d,
    S* __restrict__ tmp, const uint8_t* __restrict__ dm, double* __restrict__ omega, RedSlot slot,
    const Scalars* __restrict__ sc)
  {
    typedef typename ValueTraits<V>::acc Ac;
    __shared__ double sh[32];
    pdl_wait();
    if(gate_closed(sc))
      return;
    const uint32_t i = blockIdx.x * NT + threadIdx.x;
    double a = 0.0, b = 0.0;
    if(i < A.rows)
    {
      const bool dd = __ldg(dm + i) != 0;
      const Ac sum = row_sum<V, S, true>(A, i, cor);
      const S t = dd ? S(0) : S(add(sum, Ac(0)));
      tmp[i] = t;
      cgc_dots<MODE>(double(d[i]), double(cor[i]), double(t), a, b);
    }
    double ta, tb;
    if(grid_sum2_last<NT>(a, b, slot, sh, ta, tb))
      *omega = ta / tb;
  }

  // x += w cor, d += -w tmp
  template<typename S>
  __global__ void __launch_bounds__(NT) k_cgc_update(S* __restrict__ x, const S* __restrict__ cor, S* __restrict__ d,
    const S* __restrict__ tmp, const double* __restrict__ omega, uint32_t n, const Scalars* __restrict__ sc)
  {
    pdl_wait();
    if(gate_closed(sc))
      return;
    const uint32_t i = blockIdx.x * NT + threadIdx.x;
    if(i >= n)
      return;
    const S w = S(*omega);
    x[i] = add(mul(w, cor[i]), x[i]);
    d[i] = add(mul(S(-w), tmp[i]), d[i]);
  }

  // first post-smoothing step from the updated defect: c = F(D .* d), ||d|| -> skip flag
  template<typename S>
  __global__ void __launch_bounds__(NT) k_cgc_post1(const S* __restrict__ d, S* __restrict__ c,
    const S* __restrict__ dinv, const uint8_t* __restrict__ dm, uint32_t n, int* __restrict__ skip, RedSlot slot,
    const Scalars* __restrict__ sc)
  {
    __shared__ double sh[32];
    pdl_wait();
    if(gate_closed(sc))
      return;
    const uint32_t i = blockIdx.x * NT + threadIdx.x;
    double sq = 0.0;
    if(i < n)
    {
      const bool dd = __ldg(dm + i) != 0;
      const S dv = d[i];
      c[i] = dd ? S(0) : add(S(0), mul(__ldg(dinv + i), dv));
      sq = double(dv) * double(dv);
    }
    double total;
    if(grid_sum_last<NT>(sq, slot, sh, total))
      *skip = skip_from_norm<S>(sqrt(total));
  }

  // ------------------------------------------------------------------ TMA-staged pass epilogues
  // Row epilogues for k_tma_pass (fb_tma.cuh); each repeats the arithmetic of the matching row body
  // (fb_rows.cuh) on a row sum computed from the staged chunk, so both paths round identically.
  template<typename V, typename S>
  struct OpSmooth
  {
    typedef typename ValueTraits<V>::acc Ac;
    struct Pre { Ac b, x, di; bool d; };
    static constexpr bool REDUCES = false;
    const S* b; const S* x; S* xo; const S* dinv; const uint8_t* dm; const int* skip; const Scalars* sc;
    __device__ bool closed() const { return gate_closed(sc); }
    __device__ Pre pre(uint32_t i) const { return Pre{Ac(b[i]), Ac(x[i]), Ac(__ldg(dinv + i)), __ldg(dm + i) != 0}; }
    __device__ double operator()(uint32_t i, Ac sum, const Pre& p) const
    {
      S out = S(0);
      if(!*skip)
      {
        const Ac d1 = p.d ? Ac(0) : sub(p.b, sum);
        const Ac c = p.d ? Ac(0) : mul(p.di, d1);
        out = S(add(p.x, c));
      }
      xo[i] = out;
      return 0.0;
    }
    __device__ void finish(double) const {}
  };

  // restriction: b_c = F_c(R d), sol1_c = F_c(D_c .* b_c) (xc != null), ||b_c|| -> the coarse
  // level's pre-smoothing skip flag (restrict_row)
  template<typename V, typename S>
  struct OpRestrict
  {
    typedef typename ValueTraits<V>::acc Ac;
    struct Pre { Ac di; bool d; };
    static constexpr bool REDUCES = true;
    S* bc; S* xc; const S* dinvc; const uint8_t* dmc; int* skip; const Scalars* sc;
    __device__ bool closed() const { return gate_closed(sc); }
    __device__ Pre pre(uint32_t j) const { return Pre{xc ? Ac(__ldg(dinvc + j)) : Ac(0), __ldg(dmc + j) != 0}; }
    __device__ double operator()(uint32_t j, Ac sum, const Pre& p) const
    {
      const Ac v = p.d ? Ac(0) : add(sum, Ac(0));
      bc[j] = S(v);
      if(xc)
      {
        const Ac c = p.d ? Ac(0) : mul(p.di, v);
        xc[j] = S(add(Ac(0), c));
      }
      return double(v) * double(v);
    }
    __device__ void finish(double total) const
    {
      if(xc)
        *skip = skip_from_norm<S>(sqrt(total));
    }
  };

  // prolongation: x += F(P xc) (prolong_row); the pass gathers xc
  template<typename V, typename S>
  struct OpProlong
  {
    typedef typename ValueTraits<V>::acc Ac;
    struct Pre { Ac x; bool d; };
    static constexpr bool REDUCES = false;
    S* x; const uint8_t* dm; const Scalars* sc;
    __device__ bool closed() const { return gate_closed(sc); }
    __device__ Pre pre(uint32_t i) const { return Pre{Ac(x[i]), __ldg(dm + i) != 0}; }
    __device__ double operator()(uint32_t i, Ac sum, const Pre& p) const
    {
      const Ac c = p.d ? Ac(0) : add(sum, Ac(0));
      x[i] = S(add(p.x, c));
      return 0.0;
    }
    __device__ void finish(double) const {}
  };

  template<typename V, typename S>
  struct OpDefect
  {
    typedef typename ValueTraits<V>::acc Ac;
    struct Pre { Ac b; bool d; };
    static constexpr bool REDUCES = false;
    const S* b; S* dv; const uint8_t* dm; const Scalars* sc;
    __device__ bool closed() const { return gate_closed(sc); }
    __device__ Pre pre(uint32_t i) const { return Pre{Ac(b[i]), __ldg(dm + i) != 0}; }
    __device__ double operator()(uint32_t i, Ac sum, const Pre& p) const
    {
      dv[i] = p.d ? S(0) : S(sub(p.b, sum));
      return 0.0;
    }
    __device__ void finish(double) const {}
  };

  template<typename V, typename S>
  struct OpPost1
  {
    typedef typename ValueTraits<V>::acc Ac;
    struct Pre { Ac b, di; bool d; };
    static constexpr bool REDUCES = true;
    const S* b; S* dv; S* cv; const S* dinv; const uint8_t* dm; int* skip; const Scalars* sc;
    __device__ bool closed() const { return gate_closed(sc); }
    __device__ Pre pre(uint32_t i) const { return Pre{Ac(b[i]), Ac(__ldg(dinv + i)), __ldg(dm + i) != 0}; }
    __device__ double operator()(uint32_t i, Ac sum, const Pre& p) const
    {
      const Ac d = p.d ? Ac(0) : sub(p.b, sum);
      dv[i] = S(d);
      const Ac c = p.d ? Ac(0) : mul(p.di, d);
      cv[i] = S(add(Ac(0), c));
      return double(d) * double(d);
    }
    __device__ void finish(double total) const { *skip = skip_from_norm<S>(sqrt(total)); }
  };

  template<typename V, typename S, bool LAST, bool TOP>
  struct OpPost2
  {
    typedef typename ValueTraits<V>::acc Ac;
    struct Pre { Ac d, c, di, x; double r; bool dd; };
    static constexpr bool REDUCES = LAST && TOP;
    const S* dv; const S* cv; S* co; S* x; double* z; const double* r; const S* dinv; const uint8_t* dm;
    const int* skip; Scalars* sc;
    __device__ bool closed() const { return gate_closed(sc); }
    __device__ Pre pre(uint32_t i) const
    {
      return Pre{Ac(dv[i]), Ac(cv[i]), Ac(__ldg(dinv + i)), LAST ? Ac(x[i]) : Ac(0), TOP ? r[i] : 0.0,
                 __ldg(dm + i) != 0};
    }
    __device__ double operator()(uint32_t i, Ac sum, const Pre& p) const
    {
      Ac cn = Ac(0);
      if(!*skip)
      {
        const Ac dk = p.dd ? Ac(0) : sub(p.d, sum);
        const Ac ck = p.dd ? Ac(0) : mul(p.di, dk);
        cn = add(p.c, ck);
      }
      if(!LAST)
      {
        co[i] = S(cn);
        return 0.0;
      }
      const S xn = S(add(p.x, cn));
      if(TOP)
      {
        const double zi = mul(double(xn), sc->mg_inv_scale);
        z[i] = zi;
        return mul(p.r, zi);
      }
      x[i] = xn;
      return 0.0;
    }
    __device__ void finish(double total) const
    {
      sc->gamma_prev = sc->gamma;
      sc->gamma = total;
      sc->beta = total / sc->gamma_prev;
    }
  };

  struct OpPcgQ
  {
    struct Pre { double p; bool d; };
    static constexpr bool REDUCES = true;
    const double* p; double* q; const uint8_t* dm; Scalars* sc;
    __device__ bool closed() const { return gate_closed(sc); }
    __device__ Pre pre(uint32_t i) const { return Pre{p[i], dm[i] != 0}; }
    __device__ double operator()(uint32_t i, double sum, const Pre& pr) const
    {
      const double qv = pr.d ? 0.0 : add(sum, 0.0);
      q[i] = qv;
      return mul(qv, pr.p);
    }
    __device__ void finish(double total) const { sc->alpha = sc->gamma / total; }
  };

  // passes over a level's system matrix (the only matrices kept in diagonal storage)
  template<class Op> struct OnSystem { static constexpr bool value = true; };
  template<typename V, typename S> struct OnSystem<OpRestrict<V, S>> { static constexpr bool value = false; };
  template<typename V, typename S> struct OnSystem<OpProlong<V, S>> { static constexpr bool value = false; };

} // namespace fb

#include "fb_fused.cuh"
#include "fb_stream.cuh"
#include "fb_sor.cuh"

namespace fb
{
  // ------------------------------------------------------------------ coarse-level tail
  // The part of a multigrid cycle below the tail threshold (levels whose row count is at most the
  // threshold, down to the coarsest) in ONE block of TAIL_NT threads: block-stride loops separated
  // by __syncthreads replace one kernel launch per pass.  k_tail runs a V-cycle bottom;
  // k_tail_prog runs a program of cycle events (CycEv, encoded op << 4 | tail level) cut by the host
  // out of the cycle's event list: the F- and W-cycle sub-cycles with their peak smoothing.  The
  // tail's vectors live in shared memory (levels the host placed there; the tail's top level is
  // copied in and its solution copied out), and its matrices, diagonals and masks are
  // bulk-prefetched into L2 when the block starts, so the passes wait on shared memory and L1/L2
  // instead of DRAM.  The row bodies are the grid kernels' own.
  // events of a multigrid cycle (kernel/solver/multigrid.hpp:1350-1440): pre-smoothing steps 2..
  // (step 1 comes with the restriction), defect, restriction to the next coarser level, coarse
  // solve, prolongation from the next coarser level, post-smoothing (also the peak smoother) and
  // the PCG's final post-smoothing, which also forms z and r.z
  // (with adaptive coarse-grid correction: the scaled prolongation, and post-smoothing that starts
  // from the defect it updated)
  enum CycOp : uint8_t { EV_PRE = 0, EV_DEF = 1, EV_RES = 2, EV_CRS = 3, EV_PRO = 4, EV_POST = 5, EV_POST_TOP = 6,
                         EV_PROC = 7, EV_POSTC = 8, EV_POSTC_TOP = 9 };
  struct CycEv { uint8_t op; uint8_t lvl; };   // lvl: the level (restriction, prolongation: the finer one)

  constexpr int TAIL_NT = 320;
  constexpr int MAX_TAIL = 12;
  constexpr int MAX_TAIL_PF = 96;
  constexpr uint32_t TAIL_PF_CHUNK = 32768;
  constexpr size_t TAIL_SMEM_MAX = 200 * 1024;
  constexpr int TAIL_PROG_CHUNK = 1024;

  template<typename V, typename S>
  struct TailLevel
  {
    DCsr<V> A, P, R;       // P: this <- next coarser, R: next coarser <- this
    S *b, *x, *x2, *d, *c, *c2;   // global vectors (used when the level is not in shared memory)
    const S* dinv;
    const uint8_t* dm;
    int* skip_pre;
    int* skip_post;
    uint32_t n;
    uint32_t soff;         // shared-memory offset of the level's six vectors (elements of S)
    uint32_t np;           // padded length of one shared vector
    int in_smem;
  };

  template<typename V, typename S>
  struct TailParams
  {
    TailLevel<V, S> lv[MAX_TAIL];
    int count;             // tail levels including the coarsest
    int steps;
    const uint32_t* free_dofs;
    const double* inv;
    uint32_t m;
    int npf;               // L2 prefetch ranges (16-byte aligned, multiples of 16 bytes)
    int cgc;               // coarse-grid correction (FB_CGC_*), k_tail_prog only
    const void* pf_ptr[MAX_TAIL_PF];
    uint32_t pf_bytes[MAX_TAIL_PF];
  };

  // vector k (0 b, 1 x, 2 x2, 3 d, 4 c, 5 c2) of tail level t
  template<typename V, typename S>
  __device__ __forceinline__ S* tail_vec(const TailParams<V, S>& tp, S* sbase, int t, int k)
  {
    const TailLevel<V, S>& l = tp.lv[t];
    if(l.in_smem)
      return sbase + l.soff + uint32_t(k) * l.np;
    switch(k)
    {
      case 0: return l.b;
      case 1: return l.x;
      case 2: return l.x2;
      case 3: return l.d;
      case 4: return l.c;
      default: return l.c2;
    }
  }

  // SM: every tail level's vectors are in shared memory, so the pointers derive from the shared
  // array alone and the compiler addresses them as shared memory (32-bit, no generic check)
  template<bool SM, typename V, typename S>
  __device__ __forceinline__ S* tail_vec_s(const TailParams<V, S>& tp, S* sbase, int t, int k)
  {
    if(SM)
      return sbase + tp.lv[t].soff + uint32_t(k) * tp.lv[t].np;
    return tail_vec(tp, sbase, t, k);
  }

  template<typename V, typename S, bool SM>
  __global__ void __launch_bounds__(TAIL_NT) k_tail(const __grid_constant__ TailParams<V, S> tp, const Scalars* __restrict__ sc)
  {
    pdl_wait();
    // the parameters in shared memory: the passes index the levels with a run-time level number,
    // which in the parameter space would be constant-cache loads with a dynamic offset
    __shared__ __align__(16) TailParams<V, S> tps;
    {
      typedef TailParams<V, S> TP;
      const uint32_t nw = uint32_t(offsetof(TP, pf_ptr) / 4);
      for(uint32_t k = threadIdx.x; k < nw; k += TAIL_NT)
        reinterpret_cast<uint32_t*>(&tps)[k] = reinterpret_cast<const uint32_t*>(&tp)[k];
    }
    typedef typename ValueTraits<V>::acc Ac;
    extern __shared__ __align__(16) unsigned char tail_smem[];
    __shared__ double sh[32];
    __shared__ int skip_pre_sh[MAX_TAIL];
    __shared__ int skip_post_sh;
    if(gate_closed(sc))
      return;
    S* sbase = reinterpret_cast<S*>(tail_smem);
    // matrix data of all tail levels towards L2, asynchronously
    {
      // thread j issues chunks j, j + TAIL_NT, ... of the flattened chunk list
      uint32_t g = 0;
      for(int r = 0; r < tp.npf; ++r)
      {
        const uint32_t nb = tp.pf_bytes[r];
        for(uint32_t off = 0; off < nb; off += TAIL_PF_CHUNK, ++g)
          if(g % TAIL_NT == threadIdx.x)
          {
            const uint32_t sz = min(TAIL_PF_CHUNK, nb - off);
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;"
                         :: "l"(static_cast<const unsigned char*>(tp.pf_ptr[r]) + off), "r"(sz) : "memory");
          }
      }
    }
    __syncthreads();
    const int cnt = tps.count;
    const int steps = tps.steps;
    // the top level's input: b and sol1 = F(D .* b) written by the restriction above
    if(tps.lv[0].in_smem)
    {
      S* b0 = tail_vec_s<SM>(tps, sbase, 0, 0);
      S* x0 = tail_vec_s<SM>(tps, sbase, 0, 1);
      for(uint32_t i = threadIdx.x; i < tps.lv[0].n; i += TAIL_NT)
      {
        b0[i] = tps.lv[0].b[i];
        x0[i] = tps.lv[0].x[i];
      }
    }
    if(threadIdx.x == 0)
      skip_pre_sh[0] = *(volatile int*)tps.lv[0].skip_pre;
    __syncthreads();
    int xsel[MAX_TAIL];   // 1 or 2: which x buffer holds level t's iterate after pre-smoothing
    for(int t = 0; t + 1 < cnt; ++t)
    {
      const TailLevel<V, S>& f = tps.lv[t];
      const TailLevel<V, S>& c = tps.lv[t + 1];
      const S* fb = tail_vec_s<SM>(tps, sbase, t, 0);
      S* xa = tail_vec_s<SM>(tps, sbase, t, 1);
      S* xb = tail_vec_s<SM>(tps, sbase, t, 2);
      int sel = 1;
      const bool skipped = skip_pre_sh[t] != 0;
      for(int k = 1; k < steps; ++k)
      {
        for(uint32_t i = threadIdx.x; i < f.n; i += TAIL_NT)
          xb[i] = smooth_row<V, S, false>(f.A, fb, xa, f.dinv, f.dm, skipped, i);
        __syncthreads();
        S* tmp = xa;
        xa = xb;
        xb = tmp;
        sel = 3 - sel;
      }
      xsel[t] = sel;
      S* fd = tail_vec_s<SM>(tps, sbase, t, 3);
      for(uint32_t i = threadIdx.x; i < f.n; i += TAIL_NT)
        fd[i] = defect_row<V, S, false>(f.A, fb, xa, f.dm, i);
      __syncthreads();
      const bool coarsest = (t + 2 == cnt);
      S* cbv = tail_vec_s<SM>(tps, sbase, t + 1, 0);
      S* cxv = coarsest ? (S*)nullptr : tail_vec_s<SM>(tps, sbase, t + 1, 1);
      double sq = 0.0;
      for(uint32_t j = threadIdx.x; j < c.n; j += TAIL_NT)
        sq += restrict_row<V, S, false>(f.R, fd, cbv, cxv, c.dinv, c.dm, j);
      const double tot = block_sum<TAIL_NT>(sq, sh);
      if(threadIdx.x == 0 && !coarsest)
      {
        const int sk = skip_from_norm<S>(sqrt(tot));
        skip_pre_sh[t + 1] = sk;
        *(volatile int*)c.skip_pre = sk;
      }
      __syncthreads();
    }
    {
      const TailLevel<V, S>& c = tps.lv[cnt - 1];
      coarse_block<S, TAIL_NT>(tail_vec_s<SM>(tps, sbase, cnt - 1, 0), tail_vec_s<SM>(tps, sbase, cnt - 1, 1), c.n, tps.free_dofs,
        tps.inv, tps.m);
      xsel[cnt - 1] = 1;
      __syncthreads();
    }
    for(int t = cnt - 2; t >= 0; --t)
    {
      const TailLevel<V, S>& f = tps.lv[t];
      S* xf = tail_vec_s<SM>(tps, sbase, t, xsel[t]);
      const S* xc = tail_vec_s<SM>(tps, sbase, t + 1, xsel[t + 1]);
      const S* fb = tail_vec_s<SM>(tps, sbase, t, 0);
      S* fd = tail_vec_s<SM>(tps, sbase, t, 3);
      for(uint32_t i = threadIdx.x; i < f.n; i += TAIL_NT)
        xf[i] = prolong_row<V, S, false>(f.P, xc, xf, f.dm, i);
      __syncthreads();
      S* ca = tail_vec_s<SM>(tps, sbase, t, 4);
      S* cb = tail_vec_s<SM>(tps, sbase, t, 5);
      double sq = 0.0;
      for(uint32_t i = threadIdx.x; i < f.n; i += TAIL_NT)
        sq += post1_row<V, S, false>(f.A, fb, xf, fd, ca, f.dinv, f.dm, i);
      const double tot = block_sum<TAIL_NT>(sq, sh);
      if(threadIdx.x == 0)
      {
        skip_post_sh = skip_from_norm<S>(sqrt(tot));
        *(volatile int*)f.skip_post = skip_post_sh;
      }
      __syncthreads();
      const bool skipped = skip_post_sh != 0;
      if(steps == 1)
      {
        for(uint32_t i = threadIdx.x; i < f.n; i += TAIL_NT)
          xf[i] = S(add(Ac(xf[i]), skipped ? Ac(0) : Ac(ca[i])));
        __syncthreads();
      }
      for(int k = 2; k <= steps; ++k)
      {
        const bool last = (k == steps);
        for(uint32_t i = threadIdx.x; i < f.n; i += TAIL_NT)
        {
          const Ac cn = post2_row<V, S, false>(f.A, fd, ca, f.dinv, f.dm, skipped, i);
          if(last)
            xf[i] = S(add(Ac(xf[i]), cn));
          else
            cb[i] = S(cn);
        }
        __syncthreads();
        S* tmp = ca;
        ca = cb;
        cb = tmp;
      }
    }
    // the top level's solution goes to the global buffer the prolongation above reads
    if(tps.lv[0].in_smem)
    {
      const S* xs = tail_vec_s<SM>(tps, sbase, 0, xsel[0]);
      S* xg = xsel[0] == 1 ? tps.lv[0].x : tps.lv[0].x2;
      for(uint32_t i = threadIdx.x; i < tps.lv[0].n; i += TAIL_NT)
        xg[i] = xs[i];
    }
  }

  // ------------------------------------------------------------------ cluster tail
  // shared state of the tail kernel's interpreter
  struct TailShared
  {
    double sh[32];
    int skip_pre[MAX_TAIL];
    int xsel[MAX_TAIL];    // 1 or 2: which x buffer holds level t's iterate
    int skip_post;
    double omega;          // adaptive coarse-grid correction: the step length
  };

  // The events of k_tail_prog, one function each.  Each ends with its last pass written but not
  // yet synchronised; the interpreter syncs after every event.

  // pre-smoothing steps 2..steps from sol1 in x
  template<typename V, typename S>
  __device__ __forceinline__ void tail_pre(const TailParams<V, S>& tp, S* sbase, int t, TailShared& ts)
  {
    const TailLevel<V, S>& f = tp.lv[t];
    const S* fb = tail_vec(tp, sbase, t, 0);
    S* xa = tail_vec(tp, sbase, t, 1);
    S* xb = tail_vec(tp, sbase, t, 2);
    int sel = 1;
    const bool skipped = ts.skip_pre[t] != 0;
    for(int k = 1; k < tp.steps; ++k)
    {
      for(uint32_t i = threadIdx.x; i < f.n; i += TAIL_NT)
        xb[i] = smooth_row<V, S, false>(f.A, fb, xa, f.dinv, f.dm, skipped, i);
      if(k + 1 < tp.steps)
        __syncthreads();
      S* tmp = xa;
      xa = xb;
      xb = tmp;
      sel = 3 - sel;
    }
    if(threadIdx.x == 0)
      ts.xsel[t] = sel;
  }

  // d = F(b - A x)
  template<typename V, typename S>
  __device__ __forceinline__ void tail_def(const TailParams<V, S>& tp, S* sbase, int t, TailShared& ts)
  {
    const TailLevel<V, S>& f = tp.lv[t];
    const S* fb = tail_vec(tp, sbase, t, 0);
    const S* xa = tail_vec(tp, sbase, t, ts.xsel[t]);
    S* fd = tail_vec(tp, sbase, t, 3);
    for(uint32_t i = threadIdx.x; i < f.n; i += TAIL_NT)
      fd[i] = defect_row<V, S, false>(f.A, fb, xa, f.dm, i);
  }

  // b_{t+1} = F(R d_t), sol1_{t+1}, skip_pre_{t+1}
  template<typename V, typename S>
  __device__ __forceinline__ void tail_res(const TailParams<V, S>& tp, S* sbase, int t, TailShared& ts)
  {
    const TailLevel<V, S>& f = tp.lv[t];
    const TailLevel<V, S>& c = tp.lv[t + 1];
    const S* fd = tail_vec(tp, sbase, t, 3);
    const bool coarsest = (t + 2 == tp.count);
    S* cbv = tail_vec(tp, sbase, t + 1, 0);
    S* cxv = coarsest ? (S*)nullptr : tail_vec(tp, sbase, t + 1, 1);
    double sq = 0.0;
    for(uint32_t j = threadIdx.x; j < c.n; j += TAIL_NT)
      sq += restrict_row<V, S, false>(f.R, fd, cbv, cxv, c.dinv, c.dm, j);
    const double tot = block_sum<TAIL_NT>(sq, ts.sh);
    if(threadIdx.x == 0)
    {
      if(!coarsest)
      {
        const int sk = skip_from_norm<S>(sqrt(tot));
        ts.skip_pre[t + 1] = sk;
        *(volatile int*)c.skip_pre = sk;
      }
      ts.xsel[t + 1] = 1;
    }
  }

  template<typename V, typename S>
  __device__ __forceinline__ void tail_crs(const TailParams<V, S>& tp, S* sbase, TailShared& ts)
  {
    const int cl = tp.count - 1;
    coarse_block<S, TAIL_NT>(tail_vec(tp, sbase, cl, 0), tail_vec(tp, sbase, cl, 1), tp.lv[cl].n, tp.free_dofs,
      tp.inv, tp.m);
    if(threadIdx.x == 0)
      ts.xsel[cl] = 1;
  }

  // x_t += F(P x_{t+1})
  template<typename V, typename S>
  __device__ __forceinline__ void tail_pro(const TailParams<V, S>& tp, S* sbase, int t, TailShared& ts)
  {
    const TailLevel<V, S>& f = tp.lv[t];
    S* xf = tail_vec(tp, sbase, t, ts.xsel[t]);
    const S* xc = tail_vec(tp, sbase, t + 1, ts.xsel[t + 1]);
    for(uint32_t i = threadIdx.x; i < f.n; i += TAIL_NT)
      xf[i] = prolong_row<V, S, false>(f.P, xc, xf, f.dm, i);
  }

  // post-smoothing steps 2..steps (and the single step's update of x) after the first step wrote
  // d, c and the skip flag
  template<typename V, typename S>
  __device__ __forceinline__ void tail_post_rest(const TailParams<V, S>& tp, S* sbase, int t, TailShared& ts)
  {
    typedef typename ValueTraits<V>::acc Ac;
    const TailLevel<V, S>& f = tp.lv[t];
    const int steps = tp.steps;
    S* xf = tail_vec(tp, sbase, t, ts.xsel[t]);
    S* fd = tail_vec(tp, sbase, t, 3);
    S* ca = tail_vec(tp, sbase, t, 4);
    S* cb = tail_vec(tp, sbase, t, 5);
    const bool skipped = ts.skip_post != 0;
    if(steps == 1)
    {
      for(uint32_t i = threadIdx.x; i < f.n; i += TAIL_NT)
        xf[i] = S(add(Ac(xf[i]), skipped ? Ac(0) : Ac(ca[i])));
    }
    for(int k = 2; k <= steps; ++k)
    {
      const bool last = (k == steps);
      for(uint32_t i = threadIdx.x; i < f.n; i += TAIL_NT)
      {
        const Ac cn = post2_row<V, S, false>(f.A, fd, ca, f.dinv, f.dm, skipped, i);
        if(last)
          xf[i] = S(add(Ac(xf[i]), cn));
        else
          cb[i] = S(cn);
      }
      if(!last)
        __syncthreads();
      S* tmp = ca;
      ca = cb;
      cb = tmp;
    }
  }

  // post-smoothing (and the peak smoother) as a correction of x
  template<typename V, typename S>
  __device__ __forceinline__ void tail_post(const TailParams<V, S>& tp, S* sbase, int t, TailShared& ts)
  {
    const TailLevel<V, S>& f = tp.lv[t];
    const S* fb = tail_vec(tp, sbase, t, 0);
    S* xf = tail_vec(tp, sbase, t, ts.xsel[t]);
    S* fd = tail_vec(tp, sbase, t, 3);
    S* ca = tail_vec(tp, sbase, t, 4);
    double sq = 0.0;
    for(uint32_t i = threadIdx.x; i < f.n; i += TAIL_NT)
      sq += post1_row<V, S, false>(f.A, fb, xf, fd, ca, f.dinv, f.dm, i);
    const double tot = block_sum<TAIL_NT>(sq, ts.sh);
    if(threadIdx.x == 0)
    {
      ts.skip_post = skip_from_norm<S>(sqrt(tot));
      *(volatile int*)f.skip_post = ts.skip_post;
    }
    __syncthreads();
    tail_post_rest(tp, sbase, t, ts);
  }

  // adaptive coarse-grid correction (k_cgc_prolong, k_cgc_apply, k_cgc_update in one block)
  template<typename V, typename S>
  __device__ __forceinline__ void tail_proc(const TailParams<V, S>& tp, S* sbase, int t, TailShared& ts)
  {
    typedef typename ValueTraits<V>::acc Ac;
    const TailLevel<V, S>& f = tp.lv[t];
    S* xf = tail_vec(tp, sbase, t, ts.xsel[t]);
    const S* xc = tail_vec(tp, sbase, t + 1, ts.xsel[t + 1]);
    S* fd = tail_vec(tp, sbase, t, 3);
    S* cor = tail_vec(tp, sbase, t, 4);
    S* tmp = tail_vec(tp, sbase, t, 5);
    for(uint32_t i = threadIdx.x; i < f.n; i += TAIL_NT)
    {
      const Ac sum = row_sum<V, S, false>(f.P, i, xc);
      cor[i] = __ldg(f.dm + i) ? S(0) : S(add(sum, Ac(0)));
    }
    __syncthreads();
    double a = 0.0, b = 0.0;
    for(uint32_t i = threadIdx.x; i < f.n; i += TAIL_NT)
    {
      const Ac sum = row_sum<V, S, false>(f.A, i, cor);
      const S tv = __ldg(f.dm + i) ? S(0) : S(add(sum, Ac(0)));
      tmp[i] = tv;
      double pa, pb;
      if(tp.cgc == FB_CGC_MIN_ENERGY)
        cgc_dots<FB_CGC_MIN_ENERGY>(double(fd[i]), double(cor[i]), double(tv), pa, pb);
      else
        cgc_dots<FB_CGC_MIN_DEFECT>(double(fd[i]), double(cor[i]), double(tv), pa, pb);
      a += pa;
      b += pb;
    }
    const double ta = block_sum<TAIL_NT>(a, ts.sh);
    const double tb = block_sum<TAIL_NT>(b, ts.sh);
    if(threadIdx.x == 0)
      ts.omega = ta / tb;
    __syncthreads();
    const S w = S(ts.omega);
    for(uint32_t i = threadIdx.x; i < f.n; i += TAIL_NT)
    {
      xf[i] = add(mul(w, cor[i]), xf[i]);
      fd[i] = add(mul(S(-w), tmp[i]), fd[i]);
    }
  }

  // post-smoothing from the defect updated by tail_proc
  template<typename V, typename S>
  __device__ __forceinline__ void tail_postc(const TailParams<V, S>& tp, S* sbase, int t, TailShared& ts)
  {
    const TailLevel<V, S>& f = tp.lv[t];
    const S* fd = tail_vec(tp, sbase, t, 3);
    S* ca = tail_vec(tp, sbase, t, 4);
    double sq = 0.0;
    for(uint32_t i = threadIdx.x; i < f.n; i += TAIL_NT)
    {
      const S dv = fd[i];
      ca[i] = __ldg(f.dm + i) ? S(0) : add(S(0), mul(__ldg(f.dinv + i), dv));
      sq += double(dv) * double(dv);
    }
    const double tot = block_sum<TAIL_NT>(sq, ts.sh);
    if(threadIdx.x == 0)
    {
      ts.skip_post = skip_from_norm<S>(sqrt(tot));
      *(volatile int*)f.skip_post = ts.skip_post;
    }
    __syncthreads();
    tail_post_rest(tp, sbase, t, ts);
  }

  // The F- and W-cycle tail: the events of one run of the cycle on the tail levels, interpreted.
  // (The V-cycle bottom runs in k_tail above, whose fixed sequence compiles without register
  // spills; this interpreter costs about 0.1 ms per L10 solve more when it runs a V-cycle bottom.)
  template<typename V, typename S>
  __global__ void __launch_bounds__(TAIL_NT) k_tail_prog(const __grid_constant__ TailParams<V, S> tp,
    const uint8_t* __restrict__ prog, int nprog, const Scalars* __restrict__ sc)
  {
    pdl_wait();
    // the parameters in shared memory: the passes index the levels with a run-time level number,
    // which in the parameter space would be constant-cache loads with a dynamic offset
    __shared__ __align__(16) TailParams<V, S> tps;
    {
      typedef TailParams<V, S> TP;
      const uint32_t nw = uint32_t(offsetof(TP, pf_ptr) / 4);
      for(uint32_t k = threadIdx.x; k < nw; k += TAIL_NT)
        reinterpret_cast<uint32_t*>(&tps)[k] = reinterpret_cast<const uint32_t*>(&tp)[k];
    }
    extern __shared__ __align__(16) unsigned char tail_smem[];
    __shared__ TailShared ts;
    __shared__ uint8_t psh[TAIL_PROG_CHUNK];   // the program, a chunk at a time
    if(gate_closed(sc))
      return;
    S* sbase = reinterpret_cast<S*>(tail_smem);
    for(int e = threadIdx.x; e < min(nprog, TAIL_PROG_CHUNK); e += TAIL_NT)
      psh[e] = prog[e];
    // matrix data of all tail levels towards L2, asynchronously
    {
      // thread j issues chunks j, j + TAIL_NT, ... of the flattened chunk list
      uint32_t g = 0;
      for(int r = 0; r < tp.npf; ++r)
      {
        const uint32_t nb = tp.pf_bytes[r];
        for(uint32_t off = 0; off < nb; off += TAIL_PF_CHUNK, ++g)
          if(g % TAIL_NT == threadIdx.x)
          {
            const uint32_t sz = min(TAIL_PF_CHUNK, nb - off);
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;"
                         :: "l"(static_cast<const unsigned char*>(tp.pf_ptr[r]) + off), "r"(sz) : "memory");
          }
      }
    }
    __syncthreads();
    // the top level's input: b and sol1 = F(D .* b) written by the restriction above
    if(tps.lv[0].in_smem)
    {
      S* b0 = tail_vec(tps, sbase, 0, 0);
      S* x0 = tail_vec(tps, sbase, 0, 1);
      for(uint32_t i = threadIdx.x; i < tps.lv[0].n; i += TAIL_NT)
      {
        b0[i] = tps.lv[0].b[i];
        x0[i] = tps.lv[0].x[i];
      }
    }
    if(threadIdx.x == 0)
    {
      ts.skip_pre[0] = *(volatile int*)tps.lv[0].skip_pre;
      ts.xsel[0] = 1;
    }
    __syncthreads();
    for(int e = 0; e < nprog; ++e)
    {
      if(e > 0 && e % TAIL_PROG_CHUNK == 0)
      {
        for(int k = threadIdx.x; k < min(nprog - e, TAIL_PROG_CHUNK); k += TAIL_NT)
          psh[k] = prog[e + k];
        __syncthreads();
      }
      const unsigned ev = psh[e % TAIL_PROG_CHUNK];
      const int op = int(ev >> 4);
      const int t = int(ev & 15u);
      switch(op)
      {
        case EV_PRE: tail_pre(tps, sbase, t, ts); break;
        case EV_DEF: tail_def(tps, sbase, t, ts); break;
        case EV_RES: tail_res(tps, sbase, t, ts); break;
        case EV_CRS: tail_crs(tps, sbase, ts); break;
        case EV_PRO: tail_pro(tps, sbase, t, ts); break;
        case EV_PROC: tail_proc(tps, sbase, t, ts); break;
        case EV_POSTC:
        case EV_POSTC_TOP: tail_postc(tps, sbase, t, ts); break;
        default: tail_post(tps, sbase, t, ts); break;
      }
      __syncthreads();
    }
    // the top level's solution goes to the global buffer the prolongation above reads
    if(tps.lv[0].in_smem)
    {
      const S* xs = tail_vec(tps, sbase, 0, ts.xsel[0]);
      S* xg = ts.xsel[0] == 1 ? tps.lv[0].x : tps.lv[0].x2;
      for(uint32_t i = threadIdx.x; i < tps.lv[0].n; i += TAIL_NT)
        xg[i] = xs[i];
    }
  }

  // The same V-cycle bottom as k_tail, spread over a thread-block cluster of CT_CS blocks (one per
  // SM) so that larger levels fit: rows are dealt out cluster-wide, the passes are separated by the
  // cluster's hardware barrier (release/acquire at cluster scope, so every block sees the vectors
  // the others wrote), and the skip-test norms are summed from per-block partials in block order
  // (deterministic).  The vectors stay in global memory (L2).
  constexpr int CT_NT = 512;
  constexpr int CT_CS = 8;

  __device__ __forceinline__ void cluster_sync_all()
  {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
  }
  __device__ __forceinline__ uint32_t cluster_rank()
  {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
  }

  // cluster-wide sum of one value per thread; `slot` selects this reduction's partials in red[]
  __device__ __forceinline__ double cluster_sum(double v, double* sh, double* __restrict__ red, int slot,
    uint32_t rank)
  {
    const double b = block_sum<CT_NT>(v, sh);
    if(threadIdx.x == 0)
      red[slot * CT_CS + int(rank)] = b;
    cluster_sync_all();
    double t = 0.0;
    #pragma unroll
    for(int r = 0; r < CT_CS; ++r)
      t += *(volatile double*)(red + slot * CT_CS + r);
    return t;
  }

  template<typename V, typename S>
  __global__ void __launch_bounds__(CT_NT) k_ctail(const __grid_constant__ TailParams<V, S> tp,
    const Scalars* __restrict__ sc, double* __restrict__ red)
  {
    typedef typename ValueTraits<V>::acc Ac;
    __shared__ double sh[32];
    __shared__ int skip_pre_sh[MAX_TAIL];
    if(gate_closed(sc))   // the same answer in every block: the gate changes between launches only
      return;
    const uint32_t rank = cluster_rank();
    const uint32_t gt = rank * CT_NT + threadIdx.x;
    constexpr uint32_t GT = uint32_t(CT_CS) * CT_NT;
    // matrix data of all tail levels towards L2: chunk q of the flattened list by thread q % GT
    {
      uint32_t g = 0;
      for(int r = 0; r < tp.npf; ++r)
      {
        const uint32_t nb = tp.pf_bytes[r];
        for(uint32_t off = 0; off < nb; off += TAIL_PF_CHUNK, ++g)
          if(g % GT == gt)
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;"
                         :: "l"(static_cast<const unsigned char*>(tp.pf_ptr[r]) + off),
                            "r"(min(TAIL_PF_CHUNK, nb - off)) : "memory");
      }
    }
    const int cnt = tp.count;
    const int steps = tp.steps;
    if(threadIdx.x == 0)
      skip_pre_sh[0] = *(volatile int*)tp.lv[0].skip_pre;
    __syncthreads();
    int xsel[MAX_TAIL];
    int slot = 0;
    for(int t = 0; t + 1 < cnt; ++t)
    {
      const TailLevel<V, S>& f = tp.lv[t];
      const TailLevel<V, S>& c = tp.lv[t + 1];
      const S* fb = f.b;
      S* xa = f.x;
      S* xb = f.x2;
      int sel = 1;
      const bool skipped = skip_pre_sh[t] != 0;
      for(int k = 1; k < steps; ++k)
      {
        for(uint32_t i = gt; i < f.n; i += GT)
          xb[i] = smooth_row<V, S, false>(f.A, fb, xa, f.dinv, f.dm, skipped, i);
        cluster_sync_all();
        S* tmp = xa;
        xa = xb;
        xb = tmp;
        sel = 3 - sel;
      }
      xsel[t] = sel;
      for(uint32_t i = gt; i < f.n; i += GT)
        f.d[i] = defect_row<V, S, false>(f.A, fb, xa, f.dm, i);
      cluster_sync_all();
      const bool coarsest = (t + 2 == cnt);
      double sq = 0.0;
      for(uint32_t j = gt; j < c.n; j += GT)
        sq += restrict_row<V, S, false>(f.R, f.d, c.b, coarsest ? (S*)nullptr : c.x, c.dinv, c.dm, j);
      const double tot = cluster_sum(sq, sh, red, slot++, rank);
      if(threadIdx.x == 0)
      {
        const int sk = skip_from_norm<S>(sqrt(tot));
        skip_pre_sh[t + 1] = sk;
        if(!coarsest && rank == 0)
          *(volatile int*)c.skip_pre = sk;
      }
      __syncthreads();
    }
    {
      const TailLevel<V, S>& c = tp.lv[cnt - 1];
      if(rank == 0)
        coarse_block<S, CT_NT>(c.b, c.x, c.n, tp.free_dofs, tp.inv, tp.m);
      xsel[cnt - 1] = 1;
      cluster_sync_all();
    }
    for(int t = cnt - 2; t >= 0; --t)
    {
      const TailLevel<V, S>& f = tp.lv[t];
      S* xf = xsel[t] == 1 ? f.x : f.x2;
      const TailLevel<V, S>& cl = tp.lv[t + 1];
      const S* xc = xsel[t + 1] == 1 ? cl.x : cl.x2;
      for(uint32_t i = gt; i < f.n; i += GT)
        xf[i] = prolong_row<V, S, false>(f.P, xc, xf, f.dm, i);
      cluster_sync_all();
      S* ca = f.c;
      S* cb = f.c2;
      double sq = 0.0;
      for(uint32_t i = gt; i < f.n; i += GT)
        sq += post1_row<V, S, false>(f.A, f.b, xf, f.d, ca, f.dinv, f.dm, i);
      const double tot = cluster_sum(sq, sh, red, slot++, rank);
      const int sk = skip_from_norm<S>(sqrt(tot));
      if(threadIdx.x == 0 && rank == 0)
        *(volatile int*)f.skip_post = sk;
      const bool skipped = sk != 0;
      if(steps == 1)
      {
        for(uint32_t i = gt; i < f.n; i += GT)
          xf[i] = S(add(Ac(xf[i]), skipped ? Ac(0) : Ac(ca[i])));
        cluster_sync_all();
      }
      for(int k = 2; k <= steps; ++k)
      {
        const bool last = (k == steps);
        for(uint32_t i = gt; i < f.n; i += GT)
        {
          const Ac cn = post2_row<V, S, false>(f.A, f.d, ca, f.dinv, f.dm, skipped, i);
          if(last)
            xf[i] = S(add(Ac(xf[i]), cn));
          else
            cb[i] = S(cn);
        }
        cluster_sync_all();
        S* tmp = ca;
        ca = cb;
        cb = tmp;
      }
    }
  }

  // ------------------------------------------------------------------ PCG passes (FP64)
  // writes the V-cycle input of the top level: b = S(r * scale) (FP32 modes) and
  // sol1 = F(D .* b); returns the scale used.
  template<typename S>
  __device__ __forceinline__ void mg_input(uint32_t i, double ri, bool dd, double scale, S* __restrict__ bt,
    S* __restrict__ x1, const S* __restrict__ dinv)
  {
    const S b = S(mul(ri, scale));
    if(bt)
      bt[i] = b;
    const S c = dd ? S(0) : mul(dinv[i], b);
    x1[i] = add(S(0), c);
  }

  __device__ __forceinline__ double pow2_near_inverse(double v)
  {
    if(!(v > 0.0) || !isfinite(v))
      return 1.0;
    int e;
    frexp(v, &e);
    return ldexp(1.0, -e);
  }

  // r = F(rhs - A x), ||r|| -> def_init and the status (iterative.hpp:748-771).
  // FP64 mode also writes the V-cycle input (sol1 = F(D .* r), b aliases r).
  template<typename S>
  __global__ void __launch_bounds__(NT) k_pcg_init(DCsr<double> A, const double* __restrict__ rhs,
    const double* __restrict__ x, double* __restrict__ r, const uint8_t* __restrict__ dm, S* __restrict__ x1,
    const S* __restrict__ dinv, int* __restrict__ skip_top, double* __restrict__ hist, RedSlot slot,
    Scalars* __restrict__ sc, cudaGraphConditionalHandle cond)
  {
    pdl_wait();
    __shared__ double sh[32];
    const uint32_t r0 = blockIdx.x * NT;
    const uint32_t i = r0 + threadIdx.x;
    double sq = 0.0;
    if(i < A.rows)
    {
      const bool dd = dm[i] != 0;
      const double ri = rhs[i];
      const double sum = row_sum<double, double>(A, i, x);
      const double rv = dd ? 0.0 : sub(ri, sum);
      r[i] = rv;
      if(x1)
        mg_input<S>(i, rv, dd, 1.0, (S*)nullptr, x1, dinv);
      sq = mul(rv, rv);
    }
    double total;
    if(grid_sum_last<NT>(sq, slot, sh, total))
    {
      const double d0 = sqrt(total);
      sc->def_init = d0;
      sc->def_cur = d0;
      sc->iter = 0;
      sc->gamma = 0.0;
      hist[0] = d0;
      int status = FB_SOLVER_PROGRESS;
      if(!isfinite(d0))
        status = FB_SOLVER_ABORTED;
      else if(d0 <= EPS64 * EPS64)
        status = FB_SOLVER_SUCCESS;
      sc->status = status;
      sc->mg_scale = 1.0;
      sc->mg_inv_scale = 1.0;
      *skip_top = skip_from_norm<double>(d0);
      (void)cond;
    }
  }

  // V-cycle input of the top level from a FP64 vector v, scaled by a power of two near 1/||v||
  // (scale_from_def) or 1.  Computes ||b|| -> skip flag of the top pre-smoother.
  template<typename S>
  __global__ void __launch_bounds__(NT) k_mg_prep(const double* __restrict__ v, S* __restrict__ bt,
    S* __restrict__ x1, const S* __restrict__ dinv, const uint8_t* __restrict__ dm, int* __restrict__ skip_top,
    uint32_t n, int scale_from_def, RedSlot slot, Scalars* __restrict__ sc)
  {
    pdl_wait();
    __shared__ double sh[32];
    if(gate_closed(sc))
      return;
    const double scale = scale_from_def ? pow2_near_inverse(sc->def_cur) : 1.0;
    const uint32_t i = blockIdx.x * NT + threadIdx.x;
    double sq = 0.0;
    if(i < n)
    {
      const double vi = v[i];
      mg_input<S>(i, vi, dm[i] != 0, scale, bt, x1, dinv);
      const double b = double(S(mul(vi, scale)));
      sq = b * b;
    }
    double total;
    if(grid_sum_last<NT>(sq, slot, sh, total))
    {
      sc->mg_scale = scale;
      sc->mg_inv_scale = 1.0 / scale;
      *skip_top = skip_from_norm<S>(sqrt(total));
    }
  }

  // q = F(A p), q.p -> alpha = gamma / (q.p)
  __global__ void __launch_bounds__(NT) k_pcg_q(DCsr<double> A, const double* __restrict__ p, double* __restrict__ q,
    const uint8_t* __restrict__ dm, RedSlot slot, Scalars* __restrict__ sc)
  {
    pdl_wait();
    __shared__ double sh[32];
    if(gate_closed(sc))
      return;
    const uint32_t r0 = blockIdx.x * NT;
    const uint32_t i = r0 + threadIdx.x;
    double qp = 0.0;
    if(i < A.rows)
    {
      const bool dd = dm[i] != 0;
      const double pi = p[i];
      const double sum = row_sum<double, double>(A, i, p);
      const double qv = dd ? 0.0 : add(sum, 0.0);
      q[i] = qv;
      qp = mul(qv, pi);
    }
    double total;
    if(grid_sum_last<NT>(qp, slot, sh, total))
      sc->alpha = sc->gamma / total;
  }

  constexpr int PCGX_U = 4;        // rows per thread in flight in k_pcg_x
  constexpr int PCGX_BPS = 4;      // its resident blocks per SM at 64 registers (grid = one wave)

  // x += alpha p; r -= alpha q; ||r||, stopping test (iterative.hpp:492-507,795-879); the next
  // V-cycle input (FP64: sol1 = F(D .* r); FP32: b = S(r * scale), sol1 = F(D .* b)).
  template<typename S, bool CONVERT>
  __global__ void __launch_bounds__(NT) k_pcg_x(double* __restrict__ x, double* __restrict__ r,
    const double* __restrict__ p, const double* __restrict__ q, const uint8_t* __restrict__ dm, S* __restrict__ bt,
    S* __restrict__ x1, const S* __restrict__ dinv, int* __restrict__ skip_top, double* __restrict__ hist, uint32_t n,
    RedSlot slot, Scalars* __restrict__ sc, cudaGraphConditionalHandle cond)
  {
    pdl_wait();
    __shared__ double sh[32];
    if(gate_closed(sc))
    {
      if(cond && blockIdx.x == 0 && threadIdx.x == 0)
        cudaGraphSetConditional(cond, 0u);
      return;
    }
    const double alpha = sc->alpha;
    const double scale = CONVERT ? pow2_near_inverse(sc->def_cur) : 1.0;
    // grid-stride over the rows, PCGX_U rows per thread in flight: all loads of a group go out
    // before its arithmetic
    const uint32_t stride = gridDim.x * NT;
    double sq = 0.0;
    for(uint32_t i0 = blockIdx.x * NT + threadIdx.x; i0 < n; i0 += PCGX_U * stride)
    {
      double xv[PCGX_U], rv[PCGX_U], pv[PCGX_U], qv[PCGX_U];
      bool dd[PCGX_U];
      #pragma unroll
      for(int u = 0; u < PCGX_U; ++u)
      {
        const uint32_t i = i0 + uint32_t(u) * stride;
        if(i < n)
        {
          xv[u] = x[i];
          rv[u] = r[i];
          pv[u] = p[i];
          qv[u] = q[i];
          dd[u] = dm[i] != 0;
        }
      }
      #pragma unroll
      for(int u = 0; u < PCGX_U; ++u)
      {
        const uint32_t i = i0 + uint32_t(u) * stride;
        if(i < n)
        {
          x[i] = add(xv[u], mul(alpha, pv[u]));
          const double rn = add(rv[u], mul(-alpha, qv[u]));
          r[i] = rn;
          mg_input<S>(i, rn, dd[u], scale, CONVERT ? bt : (S*)nullptr, x1, dinv);
          sq += mul(rn, rn);
        }
      }
    }
    double total;
    if(grid_sum_last<NT>(sq, slot, sh, total))
    {
      const int it = sc->iter + 1;
      const double dc = sqrt(total);
      sc->iter = it;
      sc->def_cur = dc;
      hist[it] = dc;
      int status = FB_SOLVER_PROGRESS;
      if(!isfinite(dc))
        status = FB_SOLVER_ABORTED;
      else if(dc > sc->div_abs || dc > sc->div_rel * sc->def_init)
        status = FB_SOLVER_DIVERGED;
      else if(it < sc->min_iter)
        status = FB_SOLVER_PROGRESS;
      else if(dc <= sc->tol_abs && (dc <= sc->tol_rel * sc->def_init || dc <= 0.0))
        status = FB_SOLVER_SUCCESS;
      else if(it >= sc->max_iter)
        status = FB_SOLVER_MAX_ITER;
      sc->status = status;
      sc->mg_scale = scale;
      sc->mg_inv_scale = 1.0 / scale;
      *skip_top = skip_from_norm<S>(dc * scale);
      if(cond)
        cudaGraphSetConditional(cond, status == FB_SOLVER_PROGRESS ? 1u : 0u);
    }
  }

  // p = z (first) or p = beta p + z (axpy_generic.hpp:34-39 rounding: fl(fl(p*beta) + z))
  __global__ void __launch_bounds__(NT) k_pcg_p(double* __restrict__ p, const double* __restrict__ z, uint32_t n,
    int first, const Scalars* __restrict__ sc)
  {
    pdl_wait();
    if(gate_closed(sc))
      return;
    const uint32_t i = blockIdx.x * NT + threadIdx.x;
    if(i >= n)
      return;
    p[i] = first ? z[i] : add(mul(p[i], sc->beta), z[i]);
  }

  // permutation gathers for the caller <-> device numbering
  __global__ void k_gather(double* __restrict__ out, const double* __restrict__ in, const uint32_t* __restrict__ perm, uint32_t n)
  {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i < n)
      out[i] = in[perm[i]];
  }
  __global__ void k_scatter(double* __restrict__ out, const double* __restrict__ in, const uint32_t* __restrict__ perm, uint32_t n)
  {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i < n)
      out[perm[i]] = in[i];
  }
  __global__ void k_set_status(Scalars* sc, int status)
  {
    sc->status = status;
  }
} // namespace fb

// ==================================================================== host side

namespace fb
{
  struct DevBuf
  {
    void* p = nullptr;
    ~DevBuf() { if(p) cudaFree(p); }
  };

  struct DevMat
  {
    uint32_t rows = 0, cols = 0, nnz = 0;   // nnz: stored entries of non-empty rows
    uint64_t entries = 0;                   // slots including padding
    uint32_t* soff = nullptr;
    uint32_t* col = nullptr;
    int16_t* dcol = nullptr;
    void* val = nullptr;                    // value array in the level's storage type
    size_t smem = 0;
    double bytes = 0;                       // matrix bytes one sweep reads
    uint32_t kw = 0;                        // uniform width (ELL), 0 = sliced
    uint32_t kmax = 0;                      // widest slice's entries per row
    // x windows of the TMA-staged pass: chunk c (TMA_NT rows) reads x[xlo[c] .. xlo[c] + xwin)
    // only; xwin = 0: no window (gathers from global memory)
    uint32_t* xlo = nullptr;
    uint32_t xwin = 0;
    int32_t* doff = nullptr;                // diagonal storage: the diagonals' offsets
  };

  // Grid width W when A is the 9-point operator of a lexicographically numbered W x W vertex grid
  // in diagonal storage with all nine diagonals: every stored entry couples a vertex with itself
  // or one of its eight neighbours (so no entry wraps around a grid line); 0 otherwise.
  static uint32_t grid2d_width(const HostCsr& A, const DevMat& D)
  {
    if(!D.doff || D.kw != 9 || A.rows != A.cols)
      return 0;
    const uint32_t w = uint32_t(std::llround(std::sqrt(double(A.rows))));
    if(w < 3 || uint64_t(w) * w != A.rows)
      return 0;
    for(uint32_t i = 0; i < A.rows; ++i)
    {
      const int x = int(i % w), y = int(i / w);
      for(uint32_t k = A.rp[i]; k < A.rp[i + 1]; ++k)
      {
        const int cx = int(A.col[k] % w), cy = int(A.col[k] / w);
        if(std::abs(cx - x) > 1 || std::abs(cy - y) > 1)
          return 0;
      }
    }
    return w;
  }

  // R (coarse grid (w+1)/2 squared <- fine grid w squared): every stored entry of coarse row
  // (I, J) couples a fine vertex within one step of (2I, 2J)
  static bool restriction_local(const HostCsr& R, uint32_t w)
  {
    if(w % 2 == 0)
      return false;
    const uint32_t wc = (w + 1) / 2;
    if(R.rows != wc * wc || R.cols != w * w)
      return false;
    for(uint32_t j = 0; j < R.rows; ++j)
    {
      const int I = int(j % wc), J = int(j / wc);
      for(uint32_t k = R.rp[j]; k < R.rp[j + 1]; ++k)
      {
        const int cx = int(R.col[k] % w), cy = int(R.col[k] / w);
        if(std::abs(cx - 2 * I) > 1 || std::abs(cy - 2 * J) > 1)
          return false;
      }
    }
    return true;
  }

  // every entry of P's row (x, y) couples the coarse vertex (x / 2 + dx, y / 2 + dy), dx, dy in {0, 1}
  // (integer halves), and the rows have at most FZ_KP entries: the streamed up pass stages the
  // coarse rows y / 2 .. y / 2 + 1 around each fine row
  static bool prolongation_local(const HostCsr& P, uint32_t w)
  {
    if(w % 2 == 0)
      return false;
    const uint32_t wc = (w + 1) / 2;
    if(P.rows != w * w || P.cols != wc * wc)
      return false;
    for(uint32_t i = 0; i < P.rows; ++i)
    {
      const uint32_t x = i % w, y = i / w;
      if(P.rp[i + 1] - P.rp[i] > uint32_t(FZ_KP))
        return false;
      for(uint32_t k = P.rp[i]; k < P.rp[i + 1]; ++k)
      {
        const uint32_t cx = P.col[k] % wc, cy = P.col[k] / wc;
        if(cx < x / 2 || cx > x / 2 + 1 || cy < y / 2 || cy > y / 2 + 1)
          return false;
      }
    }
    return true;
  }

  // tiles of the streamed passes on a W x W level: at most FS_TC_MAX coarse columns, evened out
  // across the grid, and bands of coarse rows sized so that the grid fills one wave of bps blocks
  // per SM
  static FsGeom fs_geom(uint32_t W, int nsm, int bps)
  {
    FsGeom g;
    g.W = int(W);
    g.Wc = int((W + 1) / 2);
    g.ntx = (g.Wc + FS_TC_MAX - 1) / FS_TC_MAX;
    g.TC = (g.Wc + g.ntx - 1) / g.ntx;
    const int nby = std::max(1, std::max(1, nsm) * std::max(1, bps) / g.ntx);
    g.TR = (g.Wc + nby - 1) / nby;
    return g;
  }
  static uint32_t fs_grid(const FsGeom& g) { return uint32_t(g.ntx) * uint32_t((g.Wc + g.TR - 1) / g.TR); }

  // every vertex on the boundary of the w x w grid is a Dirichlet vertex (the streamed passes read
  // the out-of-grid neighbours of boundary rows unguarded and rely on the masks to discard them)
  static bool boundary_dirichlet(const std::vector<uint8_t>& dm, uint32_t w)
  {
    if(w < 2 || dm.size() != size_t(w) * w)
      return false;
    for(uint32_t k = 0; k < w; ++k)
      if(!dm[k] || !dm[size_t(w - 1) * w + k] || !dm[size_t(k) * w] || !dm[size_t(k) * w + w - 1])
        return false;
    return true;
  }

  template<typename V> DCsr<V> view(const DevMat& m)
  {
    return DCsr<V>{m.kw ? nullptr : m.soff, m.col, m.dcol, static_cast<const V*>(m.val), m.rows, m.kw, m.doff};
  }

  struct DevLevel
  {
    uint32_t n = 0;
    DevMat A, P, R;          // MG storage precision
    DevMat A64;              // FP64 top-level matrix for PCG (FP32 modes, level 0 only)
    uint8_t* dm = nullptr;
    void* dinv = nullptr;    // S
    void *b = nullptr, *x = nullptr, *x2 = nullptr, *d = nullptr, *c = nullptr, *c2 = nullptr;
    int* skip_pre = nullptr;
    int* skip_post = nullptr;
    uint32_t gw = 0;         // grid width when the level is a structured 2D grid (fused passes), else 0
    bool fz_down = false;    // the fused down pass applies (structured A and restriction)
    bool fz_up = false;      // the fused up pass applies (structured A)
    bool fs_up = false;      // the streamed up pass applies (also a local prolongation)
    bool fs_ok = false;      // the streamed passes apply (structured, Dirichlet boundary)
  };

  // a level's SOR / SSOR sweep data: the full system matrix in CSR (stored order, Dirichlet rows
  // included), the diagonal positions and the sweeps' colour orders (fb_sor.cuh)
  struct DevSor
  {
    uint32_t *rp = nullptr, *col = nullptr, *posf = nullptr, *posb = nullptr;
    void* val = nullptr;                 // the V-cycle's vector precision
    uint32_t *of = nullptr, *cf = nullptr, *ob = nullptr, *cb = nullptr;   // forward / backward order, offsets
    std::vector<uint32_t> hcf, hcb;      // the offsets on the host (one launch per colour)
    uint64_t nnz = 0;
  };

  // _apply_rest(from, smooth_first) down to level stop: pre-smoothing and defect on every level
  // but `from` when smooth_first is false (its defect is in place), restriction to the next level
  static void ev_down(std::vector<CycEv>& ev, int from, bool smooth_first, int stop)
  {
    for(int l = from; l < stop; ++l)
    {
      if(smooth_first || l > from)
      {
        ev.push_back(CycEv{EV_PRE, uint8_t(l)});
        ev.push_back(CycEv{EV_DEF, uint8_t(l)});
      }
      ev.push_back(CycEv{EV_RES, uint8_t(l)});
    }
  }

  // _apply_prol(to, smooth_last) from level start - 1 up to `to`: prolongation, then
  // post-smoothing except on level `to` when smooth_last is false
  static void ev_up(std::vector<CycEv>& ev, int to, bool smooth_last, int start, bool top, bool cgc)
  {
    for(int l = start - 1; l >= to; --l)
    {
      ev.push_back(CycEv{uint8_t(cgc ? EV_PROC : EV_PRO), uint8_t(l)});
      if(smooth_last || l > to)
      {
        const bool t = top && l == 0;
        ev.push_back(CycEv{uint8_t(cgc ? (t ? EV_POSTC_TOP : EV_POSTC) : (t ? EV_POST_TOP : EV_POST)), uint8_t(l)});
      }
    }
  }

  // _apply_smooth_peak(l): the peak smoother as a correction, then the new defect
  static void ev_peak(std::vector<CycEv>& ev, int l)
  {
    ev.push_back(CycEv{EV_POST, uint8_t(l)});
    ev.push_back(CycEv{EV_DEF, uint8_t(l)});
  }

  // One multigrid cycle over nl levels as events: V = rest(0) + coarse + prol(0); F and W the peak
  // sequences of _apply_cycle_f / _apply_cycle_w (kernel/solver/multigrid.hpp:1356-1440)
  static std::vector<CycEv> cycle_events(int cycle, int nl, bool cgc)
  {
    std::vector<CycEv> ev;
    const int last = nl - 1;
    const CycEv crs{EV_CRS, uint8_t(last)};
    ev_down(ev, 0, true, last);
    ev.push_back(crs);
    if(cycle == FB_CYCLE_F)
    {
      for(int pk = last - 1; pk > 0; --pk)
      {
        ev_up(ev, pk, false, last, false, cgc);
        ev_peak(ev, pk);
        ev_down(ev, pk, false, last);
        ev.push_back(crs);
      }
    }
    else if(cycle == FB_CYCLE_W)
    {
      // the coarse solves number 2^last; before each one after the first, the peak level is the
      // finest level whose counter is still zero below the deepest one that is not
      std::vector<int> cnt(static_cast<size_t>(nl), 0);
      const uint64_t num_cgs = uint64_t(1) << last;
      for(uint64_t cgs = 1; cgs < num_cgs; ++cgs)
      {
        int pk = last;
        while(pk > 0)
          if(cnt[size_t(--pk)] == 0)
            break;
        for(int i = last - 1; i > pk; --i)
          cnt[size_t(i)] = 0;
        ++cnt[size_t(pk)];
        ev_up(ev, pk, false, last, false, cgc);
        ev_peak(ev, pk);
        ev_down(ev, pk, false, last);
        ev.push_back(crs);
      }
    }
    ev_up(ev, 0, true, last, true, cgc);
    return ev;
  }
} // namespace fb

struct fb_solver
{
  fb_solver_config cfg;
  fb_hierarchy* h = nullptr;
  int nlev = 0;
  int vsize = 8;   // bytes per MG vector entry
  std::vector<fb::DevLevel> lv;
  std::vector<void*> allocs;
  std::vector<std::vector<uint32_t>> perms;   // per level; empty = identity
  // coarse
  uint32_t* free_dofs = nullptr;
  double* cinv = nullptr;
  uint32_t nfree = 0;
  // PCG
  double *x = nullptr, *r = nullptr, *p = nullptr, *q = nullptr, *z = nullptr, *rhs = nullptr;
  double *tmp_in = nullptr, *tmp_out = nullptr;
  void* flush = nullptr;   // L2 flush buffer of fb_solver_time_kernel (allocated on first use)
  uint32_t* perm0 = nullptr;
  double* hist = nullptr;
  // fb_solver_update_matrix: per level, the device slot of every caller CSR entry (UINT32_MAX =
  // not stored) and the caller entry of every device row's diagonal; built on first use
  std::vector<uint32_t*> upd_slot, upd_diag;
  fb::Scalars* sc = nullptr;
  fb::RedSlot slot{nullptr, nullptr};
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  cudaGraph_t vgraph = nullptr;
  cudaGraphExec_t vexec = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<fb::DevSor> sor;              // per level (not the coarsest): SOR / SSOR sweep data
  std::vector<fb::CycEv> events;            // one multigrid cycle
  uint8_t* tail_prog = nullptr;             // tail kernel programs: events op << 4 | tail level
  std::vector<uint32_t> seg_off, seg_len;   // program of each tail segment of `events`, in order
  double* cgc_omega = nullptr;   // step length of the adaptive coarse-grid correction
  int max_iter_cap = 0;   // max_iter at creation: the defect history holds max_iter + 2 entries
  void* vc_top = nullptr; // buffer that holds the finest level's result after a standalone V-cycle
  uint32_t slot_cap = 0;  // blocks whose (two) partial sums the reduction slot holds
  int fs_bps_down = 1, fs_bps_up = 1;   // resident blocks per SM of the streamed passes
  int tail_first = -1;    // first level handled by the single-block tail kernel, -1 = none
  int ctail_first = -1;   // first level handled by the cluster tail kernel, -1 = none
  double* cred = nullptr; // cluster tail: per-block partial sums (2 * MAX_TAIL * CT_CS)
  cudaError_t launch_err = cudaSuccess;
  int nsm = 148;          // streaming multiprocessors of the device
  int* err = nullptr;     // device error word (bounded waits that expired)
  uint64_t launches_init = 0, launches_body = 0, launches_vcycle = 0;
  double bytes_init = 0, bytes_body = 0;
  uint64_t counting = 0;
  double counting_bytes = 0;
};

namespace fb
{
  static fb_status dalloc(fb_solver* s, void** p, size_t bytes)
  {
    cudaError_t e = cudaMalloc(p, bytes + 64);
    if(e != cudaSuccess)
    {
      set_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
      return FB_ERR_NOMEM;
    }
    s->allocs.push_back(*p);
    e = cudaMemset(*p, 0, bytes + 64);
    if(e != cudaSuccess)
      return cuda_fail(e, "cudaMemset");
    return FB_OK;
  }

#define FB_TRY(x)                     \
  do {                                \
    fb_status fb_t_ = (x);            \
    if(fb_t_ != FB_OK) return fb_t_;  \
  } while(0)

  static size_t vsize_of(int prec) { return prec == FB_PREC_F64 ? 8 : 4; }
  static size_t valsize_of(int prec) { return prec == FB_PREC_F64 ? 8 : (prec == FB_PREC_F32 ? 4 : 2); }

  static uint16_t to_bf16_rne(float f)
  {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if((u & 0x7f800000u) == 0x7f800000u)
      return uint16_t(u >> 16) | ((u & 0xffffu) ? 0x40u : 0u);
    const uint32_t lsb = (u >> 16) & 1u;
    u += 0x7fffu + lsb;
    return uint16_t(u >> 16);
  }

  // CSR -> the device layout (build_sell), values converted to the storage precision.
  static fb_status upload_mat(fb_solver* s, DevMat& d, const HostCsr& M, int prec, const std::vector<uint8_t>* empty,
                              bool allow_diag = false)
  {
    const HostSell H = build_sell(M, empty, true, allow_diag);
    const uint32_t ns = (H.rows + 31u) / 32u;
    d.rows = H.rows;
    d.cols = H.cols;
    d.nnz = uint32_t(H.nnz);
    d.entries = H.entries;
    d.kw = H.kw;
    d.kmax = H.kw;
    for(uint32_t sl = 0; sl < ns; ++sl)
      d.kmax = std::max(d.kmax, (H.soff[sl + 1] - H.soff[sl]) / 32u);
    const size_t vb = valsize_of(prec);
    const size_t cb = H.narrow ? 2 : 4;
    d.bytes = double(H.entries) * double(vb + (H.doff.empty() ? cb : 0)) + (H.kw ? 0.0 : double(ns + 1) * 4.0);
    if(!H.doff.empty())
    {
      // diagonal storage: values and the offsets only (the grid kernels serve it)
      FB_TRY(dalloc(s, (void**)&d.doff, sizeof(int32_t) * H.doff.size()));
      FB_CUDA(cudaMemcpy(d.doff, H.doff.data(), sizeof(int32_t) * H.doff.size(), cudaMemcpyHostToDevice));
    }
    else
    {
      // column window of every TMA chunk (real entries; narrow padding reads the row itself),
      // start rounded down to 4 entries (16-byte copies for FP32 and FP64 vectors)
      const uint32_t spc = uint32_t(TMA_NT) / 32u;
      const uint32_t nch = (ns + spc - 1) / spc;
      std::vector<uint32_t> lo(std::max<uint32_t>(1, nch), 0u);
      uint32_t wmax = 0;
      for(uint32_t c = 0; c < nch; ++c)
      {
        uint32_t mn = UINT32_MAX, mx = 0;
        for(uint32_t sl = c * spc; sl < std::min(ns, c * spc + spc); ++sl)
        {
          const uint32_t K = (H.soff[sl + 1] - H.soff[sl]) / 32u;
          for(uint32_t lane = 0; lane < 32u; ++lane)
          {
            const uint32_t r = sl * 32u + lane;
            if(r >= H.rows)
              break;
            for(uint32_t k = 0; k < K; ++k)
            {
              const uint64_t e = H.soff[sl] + uint64_t(k) * 32u + lane;
              uint32_t col;
              if(H.narrow)
                col = uint32_t(int64_t(r) + H.dcol[e]);
              else if(H.col[e] == H.cols)
                continue;
              else
                col = H.col[e];
              mn = std::min(mn, col);
              mx = std::max(mx, col);
            }
          }
        }
        if(mn == UINT32_MAX)
          mn = mx = 0;
        lo[c] = mn & ~3u;
        wmax = std::max(wmax, mx + 1 - lo[c]);
      }
      d.xwin = (wmax + 3u) & ~3u;
      if(d.xwin > TMA_XWIN_MAX)
        d.xwin = 0;
      else
      {
        FB_TRY(dalloc(s, (void**)&d.xlo, sizeof(uint32_t) * lo.size()));
        FB_CUDA(cudaMemcpy(d.xlo, lo.data(), sizeof(uint32_t) * lo.size(), cudaMemcpyHostToDevice));
      }
    }
    FB_TRY(dalloc(s, (void**)&d.soff, sizeof(uint32_t) * H.soff.size()));
    FB_CUDA(cudaMemcpy(d.soff, H.soff.data(), sizeof(uint32_t) * H.soff.size(), cudaMemcpyHostToDevice));
    const size_t ne = std::max<size_t>(1, size_t(H.entries));
    if(d.doff)
      ;
    else if(H.narrow)
    {
      FB_TRY(dalloc(s, (void**)&d.dcol, 2 * ne));
      if(H.entries)
        FB_CUDA(cudaMemcpy(d.dcol, H.dcol.data(), 2 * H.entries, cudaMemcpyHostToDevice));
    }
    else
    {
      FB_TRY(dalloc(s, (void**)&d.col, 4 * ne));
      if(H.entries)
        FB_CUDA(cudaMemcpy(d.col, H.col.data(), 4 * H.entries, cudaMemcpyHostToDevice));
    }
    FB_TRY(dalloc(s, &d.val, vb * ne));
    if(H.entries)
    {
      if(prec == FB_PREC_F64)
        FB_CUDA(cudaMemcpy(d.val, H.val.data(), 8 * H.entries, cudaMemcpyHostToDevice));
      else if(prec == FB_PREC_F32)
      {
        std::vector<float> f(H.val.begin(), H.val.end());
        FB_CUDA(cudaMemcpy(d.val, f.data(), 4 * f.size(), cudaMemcpyHostToDevice));
      }
      else
      {
        std::vector<uint16_t> h(H.entries);
        for(size_t k = 0; k < h.size(); ++k)
          h[k] = to_bf16_rne(float(H.val[k]));
        FB_CUDA(cudaMemcpy(d.val, h.data(), 2 * h.size(), cudaMemcpyHostToDevice));
      }
    }
    return FB_OK;
  }

  template<typename S>
  static fb_status upload_vec(fb_solver* s, void** dst, const std::vector<double>& v)
  {
    FB_TRY(dalloc(s, dst, sizeof(S) * std::max<size_t>(1, v.size())));
    std::vector<S> t(v.begin(), v.end());
    FB_CUDA(cudaMemcpy(*dst, t.data(), sizeof(S) * t.size(), cudaMemcpyHostToDevice));
    return FB_OK;
  }

  static fb_status upload_u32(fb_solver* s, uint32_t** dst, const std::vector<uint32_t>& v)
  {
    FB_TRY(dalloc(s, (void**)dst, sizeof(uint32_t) * std::max<size_t>(1, v.size())));
    FB_CUDA(cudaMemcpy(*dst, v.data(), sizeof(uint32_t) * v.size(), cudaMemcpyHostToDevice));
    return FB_OK;
  }

  static unsigned int blocks(uint32_t n) { return std::max(1u, (n + NT - 1) / NT); }

  // Blocks of `kern` (TMA_NT threads, `smem` dynamic shared memory) resident on one SM at once, at
  // most 8 (cached: the occupancy query is made once per kernel and size)
  static uint32_t resident_blocks(const void* kern, size_t smem)
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
    const uint32_t r = uint32_t(std::min(nb, 8));
    cache.emplace(key, r);
    return r;
  }

  // ---------------------------------------------------------------- launch sequences
  template<typename V, typename S>
  struct Launcher
  {
    fb_solver* s;
    cudaStream_t st;
    bool dry = false;          // count launches and bytes only

    // Every kernel of a solve is launched with programmatic stream serialisation (when cfg.pdl):
    // it may be scheduled while its predecessor's last blocks finish, and waits for the
    // predecessor's results in griddepcontrol.wait (pdl_wait; the TMA pass first stages its
    // first chunks of matrix data, which no kernel of a solve writes).
    template<typename... KA, typename... A>
    void go(void (*k)(KA...), dim3 g, dim3 b, size_t smem, A&&... a)
    {
      cudaLaunchConfig_t lc = {};
      lc.gridDim = g;
      lc.blockDim = b;
      lc.dynamicSmemBytes = smem;
      lc.stream = st;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      at[0].val.programmaticStreamSerializationAllowed = 1;
      lc.attrs = at;
      lc.numAttrs = s->cfg.pdl ? 1 : 0;
      const cudaError_t e = cudaLaunchKernelEx(&lc, k, std::forward<A>(a)...);
      if(e != cudaSuccess && s->launch_err == cudaSuccess)
        s->launch_err = e;
    }

    // k_pcg_x: one wave of PCGX_BPS blocks per SM at most
    unsigned int pcgx_grid(uint32_t n) const
    {
      return std::min(blocks(n), unsigned(std::max(1, s->nsm) * PCGX_BPS));
    }

    // column index bytes per entry
    static uint32_t colbytes(const DevMat& m) { return m.doff ? 0u : (m.dcol ? 2u : 4u); }

    bool use_tma_f64(const DevMat& m) const
    {
      if(s->cfg.tma_rows <= 0 || !m.kmax || (m.doff && m.kw != 9 && m.kw != 27) || m.rows < uint32_t(s->cfg.tma_rows))
        return false;
      return uint64_t(tma_stages<double>()) * tma_stage_bytes<double>(m.kmax, colbytes(m)) <= TMA_SMEM_MAX;
    }

    // the TMA-staged pass serves matrices of at least tma_rows rows whose stages fit
    bool use_tma(const DevMat& m) const
    {
      if(s->cfg.tma_rows <= 0 || !m.kmax || (m.doff && m.kw != 9 && m.kw != 27) || m.rows < uint32_t(s->cfg.tma_rows))
        return false;
      return uint64_t(tma_stages<V>()) * tma_stage_bytes<V>(m.kmax, colbytes(m)) <= TMA_SMEM_MAX;
    }
    template<typename VV, typename XS, class Op>
    void tma(const DevMat& m, const void* x, const Op& op)
    {
      // tma_window 1: the x window rides along in shared memory when the stages still fit;
      // 2: it is bulk-prefetched into L2 three chunks ahead; 0: neither
      uint32_t xw = s->cfg.tma_window ? m.xwin : 0u;
      const int xstage = s->cfg.tma_window == 1 ? 1 : 0;
      if(xw && xstage &&
         uint64_t(tma_stages<VV>()) * (tma_stage_bytes<VV>(m.kmax, colbytes(m)) + uint64_t(xw) * sizeof(XS)) >
           TMA_SMEM_MAX)
        xw = 0;
      const uint32_t sb = tma_stage_bytes<VV>(m.kmax, colbytes(m)) + (xstage ? xw * uint32_t(sizeof(XS)) : 0u);
      const size_t smem = size_t(tma_stages<VV>()) * sb;
      const uint32_t padded = (m.rows + 31u) & ~31u;
      const uint32_t nch = (padded + TMA_NT - 1) / TMA_NT;
      // vectors hold cols + 8 entries (dalloc pads 64 bytes): windows end there at the latest
      const uint32_t nxa = (m.cols + 8u) & ~3u;
      // a persistent grid of as many blocks as stay resident together (one wave)
      auto launch = [&](auto kern, const uint32_t* xl, uint32_t xwa, int xs, size_t sm)
      {
        const uint32_t grid = std::max(1u, std::min(nch, uint32_t(s->nsm) * resident_blocks((const void*)kern, sm)));
        go(kern, grid, TMA_NT, sm, view<VV>(m), static_cast<const XS*>(x), padded, m.kmax, xl, xwa, nxa, xs, op,
           s->slot, s->err);
      };
      const size_t smem_dg = size_t(tma_stages_dg<VV, true>()) * sb;
      // diagonal storage of the 2D / 3D Q1 stencils (9 / 27 diagonals); the 2D Q1 stencil in ELL of
      // width 9 runs the fully unrolled row sum
      if constexpr(OnSystem<Op>::value)
        if(m.doff)
        {
          if(m.kw == 9)
            launch(k_tma_pass<VV, XS, Op, 9, true>, nullptr, 0u, 0, smem_dg);
          else
            launch(k_tma_pass<VV, XS, Op, 27, true>, nullptr, 0u, 0, smem_dg);
          return;
        }
      if(m.kw == 9)
        launch(k_tma_pass<VV, XS, Op, 9>, xw ? m.xlo : nullptr, xw, xstage, smem);
      else
        launch(k_tma_pass<VV, XS, Op, 0>, xw ? m.xlo : nullptr, xw, xstage, smem);
    }
    uint64_t launches = 0;
    double bytes = 0;

    DevLevel& L(int i) { return s->lv[size_t(i)]; }

    // algorithmic bytes of one CSR sweep: nnz*(val+idx) + (rows+1)*idx + reads of x + rows*out
    // algorithmic bytes of one sweep: the matrix as stored + gathered vector + row-wise vectors
    double csr_bytes(const DevMat& m, double vec_in, double vec_out)
    {
      return m.bytes + double(m.cols) * sizeof(S) + double(m.rows) * sizeof(S) * (vec_in + vec_out);
    }

    // Shared-memory placement of the tail's vectors (coarsest level first, while the levels fit)
    // and the L2 prefetch list of its matrices, diagonals and masks; returns the dynamic shared
    // memory size.
    size_t tail_layout(TailParams<V, S>& tp, int lt, bool use_smem)
    {
      const int nl = s->nlev;
      uint32_t used = 0;
      for(int l = nl - 1; l >= lt && use_smem; --l)
      {
        TailLevel<V, S>& t = tp.lv[l - lt];
        const uint32_t np = (t.n + 7u) & ~7u;
        if(size_t(used) + 6ull * np * sizeof(S) > TAIL_SMEM_MAX)
          break;
        t.in_smem = 1;
        t.soff = used / uint32_t(sizeof(S));
        t.np = np;
        used += 6u * np * uint32_t(sizeof(S));
      }
      auto pf = [&](const void* p, uint64_t nb)
      {
        if(!p || tp.npf >= MAX_TAIL_PF)
          return;
        const uintptr_t a = reinterpret_cast<uintptr_t>(p);
        const uintptr_t a16 = (a + 15) & ~uintptr_t(15);
        if(nb < (a16 - a) + 16)
          return;
        nb = (nb - (a16 - a)) & ~uint64_t(15);
        tp.pf_ptr[tp.npf] = reinterpret_cast<const void*>(a16);
        tp.pf_bytes[tp.npf] = uint32_t(std::min<uint64_t>(nb, 0xfffffff0ull));
        ++tp.npf;
      };
      auto add_mat = [&](const DevMat& m)
      {
        pf(m.val, m.entries * sizeof(V));
        pf(m.dcol, m.entries * sizeof(int16_t));
        pf(m.col, m.entries * sizeof(uint32_t));
        if(!m.kw && m.soff)
          pf(m.soff, (uint64_t((m.rows + 31) / 32) + 1) * sizeof(uint32_t));
      };
      for(int l = nl - 1; l >= lt; --l)
      {
        const DevLevel& f = L(l);
        add_mat(f.A);
        if(l + 1 < nl)
        {
          add_mat(f.R);
          add_mat(f.P);
        }
        pf(f.dinv, uint64_t(f.n) * sizeof(S));
        pf(f.dm, f.n);
      }
      return used;
    }

    // ---- the pieces of a multigrid cycle (kernel/solver/multigrid.hpp:1350-1440); xcur[l] is the
    // buffer (x or x2) that holds level l's solution

    // pre-smoothing steps k >= 2 of level l (step 1, sol1 = D b, came with the restriction)
    void pre_smooth(int l, std::vector<void*>& xcur)
    {
      DevLevel& f = L(l);
      const int steps = std::max(1, s->cfg.smooth_steps);
      void* xa = f.x;
      void* xb = f.x2;
      for(int k = 1; k < steps; ++k)
      {
        if(dry)
          ;
        else if(use_tma(f.A))
          tma<V, S>(f.A, xa, OpSmooth<V, S>{(const S*)f.b, (const S*)xa, (S*)xb, (const S*)f.dinv, f.dm, f.skip_pre, s->sc});
        else
          go(k_smooth<V, S>, blocks(f.n), NT, f.A.smem, view<V>(f.A), (const S*)f.b, (const S*)xa, (S*)xb,
            (const S*)f.dinv, f.dm, f.skip_pre, s->sc);
        ++launches;
        bytes += csr_bytes(f.A, 3, 1) + f.n;
        std::swap(xa, xb);
      }
      xcur[size_t(l)] = xa;
    }

    // d_l = F(b - A x_l)
    void defect(int l, std::vector<void*>& xcur)
    {
      DevLevel& f = L(l);
      if(dry)
        ;
      else if(use_tma(f.A))
        tma<V, S>(f.A, xcur[size_t(l)], OpDefect<V, S>{(const S*)f.b, (S*)f.d, f.dm, s->sc});
      else
        go(k_defect<V, S>, blocks(f.n), NT, f.A.smem, view<V>(f.A), (const S*)f.b, (const S*)xcur[size_t(l)],
          (S*)f.d, f.dm, s->sc);
      ++launches;
      bytes += csr_bytes(f.A, 1, 1) + f.n;
    }

    // b_{l+1} = F(R d_l), sol1_{l+1} = F(D b_{l+1}) (not on the coarsest level), skip_pre_{l+1}
    void restrict_to(int l)
    {
      const int nl = s->nlev;
      DevLevel& f = L(l);
      DevLevel& c = L(l + 1);
      const bool coarsest = (l + 2 == nl);
      if(dry)
        ;
      else if(use_tma(f.R))
        tma<V, S>(f.R, f.d, OpRestrict<V, S>{(S*)c.b, coarsest ? (S*)nullptr : (S*)c.x, (const S*)c.dinv, c.dm,
          c.skip_pre, s->sc});
      else
        go(k_restrict<V, S>, blocks(c.n), NT, f.R.smem, view<V>(f.R), (const S*)f.d, (S*)c.b,
          coarsest ? (S*)nullptr : (S*)c.x, (const S*)c.dinv, c.dm, c.skip_pre, s->slot, s->sc);
      ++launches;
      bytes += csr_bytes(f.R, 0, coarsest ? 1 : 3) + c.n;
    }

    // exact solve on the coarsest level
    void coarse(std::vector<void*>& xcur)
    {
      const int nl = s->nlev;
      DevLevel& c = L(nl - 1);
      if(!dry) go(k_coarse<S>, 1, NT, 0, (const S*)c.b, (S*)c.x, c.n, s->free_dofs, s->cinv, s->nfree, s->sc);
      ++launches;
      bytes += double(s->nfree) * s->nfree * 8.0 + double(c.n) * 2 * sizeof(S);
      xcur[size_t(nl - 1)] = c.x;
    }

    // x_l += F(P x_{l+1})
    void prolong(int l, std::vector<void*>& xcur)
    {
      DevLevel& f = L(l);
      void* xf = xcur[size_t(l)];
      if(dry)
        ;
      else if(use_tma(f.P))
        tma<V, S>(f.P, xcur[size_t(l + 1)], OpProlong<V, S>{(S*)xf, f.dm, s->sc});
      else
        go(k_prolong<V, S>, blocks(f.n), NT, f.P.smem, view<V>(f.P), (const S*)xcur[size_t(l + 1)], (S*)xf, f.dm,
          s->sc);
      ++launches;
      bytes += csr_bytes(f.P, 1, 1) + f.n;
    }

    // grid sizes of the fused passes of level l
    uint32_t fused_down_grid(int l) const
    {
      const uint32_t t = ((s->lv[size_t(l)].gw + 1) / 2 + FZ_DOWN_TILE - 1) / FZ_DOWN_TILE;
      return t * t;
    }
    uint32_t fused_up_grid(int l) const
    {
      const uint32_t t = (s->lv[size_t(l)].gw + FZ_UP_TILE - 1) / FZ_UP_TILE;
      return t * t;
    }
    // the fused passes apply to levels of at most cfg.fused rows (structured ones, checked at
    // creation) in V(2,2) cycles with the fixed coarse-grid correction
    bool fused_level(int l) const
    {
      return s->cfg.fused > 0 && s->cfg.smoother == FB_SMOOTHER_JACOBI && s->lv[size_t(l)].n <= uint32_t(s->cfg.fused) &&
             s->cfg.cycle == FB_CYCLE_V &&
             s->cfg.adapt_cgc == FB_CGC_FIXED && s->cfg.smooth_steps == 2;
    }

    // pre-smoothing step 2, defect and restriction of level l in one pass (k_fz_down): sol1 in x,
    // the smoothed iterate to x2, b / sol1 / skip flag of level l + 1
    void fused_down(int l, std::vector<void*>& xcur)
    {
      DevLevel& f = L(l);
      DevLevel& c = L(l + 1);
      const bool coarsest = (l + 2 == s->nlev);
      const uint32_t wc = (f.gw + 1) / 2;
      if(!dry)
        go(k_fz_down<V, S>, fused_down_grid(l), FZ_NT, 0, view<V>(f.A), view<V>(f.R), f.gw, wc, (const S*)f.b,
          (const S*)f.x, (S*)f.x2, (const S*)f.dinv, f.dm, (const int*)f.skip_pre, (S*)c.b,
          coarsest ? (S*)nullptr : (S*)c.x, (const S*)c.dinv, c.dm, c.skip_pre, s->slot, (const Scalars*)s->sc);
      ++launches;
      bytes += f.A.bytes + f.R.bytes + double(f.n) * (4.0 * sizeof(S) + 1.0) +
               double(c.n) * ((coarsest ? 1.0 : 3.0) * sizeof(S) + 1.0);
      xcur[size_t(l)] = f.x2;
    }

    // prolongation and both post-smoothing steps of level l in one pass (k_fz_up); the result
    // goes to the level's other x buffer (top: the PCG's z and r.z)
    void fused_up(int l, bool top, std::vector<void*>& xcur)
    {
      DevLevel& f = L(l);
      void* xin = xcur[size_t(l)];
      void* xout = (xin == f.x) ? f.x2 : f.x;
      const S* xc = (const S*)xcur[size_t(l + 1)];
      if(dry)
        ;
      else if(top)
        go(k_fz_up<V, S, true>, fused_up_grid(l), FZ_NT, 0, view<V>(f.A), view<V>(f.P), f.gw, (const S*)xin, xc,
          (S*)nullptr, (const S*)f.b, (const S*)f.dinv, f.dm, f.skip_post, s->z, (const double*)s->r, s->slot, s->sc);
      else
        go(k_fz_up<V, S, false>, fused_up_grid(l), FZ_NT, 0, view<V>(f.A), view<V>(f.P), f.gw, (const S*)xin, xc,
          (S*)xout, (const S*)f.b, (const S*)f.dinv, f.dm, f.skip_post, (double*)nullptr, (const double*)nullptr,
          s->slot, s->sc);
      ++launches;
      bytes += f.A.bytes + f.P.bytes + double(f.P.cols) * sizeof(S) + double(f.n) * (4.0 * sizeof(S) + 1.0) +
               (top ? 16.0 * double(f.n) : 0.0);
      if(!top)
        xcur[size_t(l)] = xout;
    }

    // the streamed passes apply to structured levels above the fused threshold with at least
    // cfg.streamed rows, in the cycles the fused passes serve
    bool stream_level(int l) const
    {
      const uint32_t n = s->lv[size_t(l)].n;
      return s->cfg.streamed > 0 && s->cfg.smoother == FB_SMOOTHER_JACOBI && n >= uint32_t(s->cfg.streamed) &&
             (s->cfg.fused <= 0 || n > uint32_t(s->cfg.fused)) && s->cfg.cycle == FB_CYCLE_V &&
             s->cfg.adapt_cgc == FB_CGC_FIXED && s->cfg.smooth_steps == 2;
    }
    FsGeom stream_geom(int l, bool up) const
    {
      return fs_geom(s->lv[size_t(l)].gw, s->nsm, up ? s->fs_bps_up : s->fs_bps_down);
    }

    // the down pass of level l in its streamed form (k_fs_down); buffers as in fused_down
    void streamed_down(int l, std::vector<void*>& xcur)
    {
      DevLevel& f = L(l);
      DevLevel& c = L(l + 1);
      const bool coarsest = (l + 2 == s->nlev);
      const FsGeom g = stream_geom(l, false);
      if(!dry)
        go(k_fs_down<V, S>, fs_grid(g), FS_NT, FsLay<V, S, false, false>::SMEM, view<V>(f.A), view<V>(f.R), g,
          (const S*)f.b, (const S*)f.x, (S*)f.x2, (const S*)f.dinv, f.dm, (const int*)f.skip_pre, (S*)c.b,
          coarsest ? (S*)nullptr : (S*)c.x, (const S*)c.dinv, c.dm, c.skip_pre, s->slot, s->err,
          (const Scalars*)s->sc);
      ++launches;
      bytes += f.A.bytes + f.R.bytes + double(f.n) * (4.0 * sizeof(S) + 1.0) +
               double(c.n) * ((coarsest ? 1.0 : 3.0) * sizeof(S) + 1.0);
      xcur[size_t(l)] = f.x2;
    }

    // the up pass of level l in its streamed form (k_fs_up); buffers as in fused_up
    void streamed_up(int l, bool top, std::vector<void*>& xcur)
    {
      DevLevel& f = L(l);
      void* xin = xcur[size_t(l)];
      void* xout = (xin == f.x) ? f.x2 : f.x;
      const S* xc = (const S*)xcur[size_t(l + 1)];
      const FsGeom g = stream_geom(l, true);
      if(dry)
        ;
      else if(top)
        go(k_fs_up<V, S, true>, fs_grid(g), FS_NT, FsLay<V, S, true, true>::SMEM, view<V>(f.A), view<V>(f.P), g,
          (const S*)xin, xc, (S*)nullptr, (const S*)f.b, (const S*)f.dinv, f.dm, f.skip_post, s->z,
          (const double*)s->r, s->slot, s->err, s->sc);
      else
        go(k_fs_up<V, S, false>, fs_grid(g), FS_NT, FsLay<V, S, true, false>::SMEM, view<V>(f.A), view<V>(f.P), g,
          (const S*)xin, xc, (S*)xout, (const S*)f.b, (const S*)f.dinv, f.dm, f.skip_post, (double*)nullptr,
          (const double*)nullptr, s->slot, s->err, s->sc);
      ++launches;
      bytes += f.A.bytes + f.P.bytes + double(f.P.cols) * sizeof(S) + double(f.n) * (4.0 * sizeof(S) + 1.0) +
               (top ? 16.0 * double(f.n) : 0.0);
      if(!top)
        xcur[size_t(l)] = xout;
    }

    // adaptive coarse-grid correction of level l: cor = F(P x_{l+1}) in c, tmp = F(A cor) in c2,
    // the step length w, x += w cor, d += -w tmp
    void prolong_cgc(int l, std::vector<void*>& xcur)
    {
      DevLevel& f = L(l);
      void* xf = xcur[size_t(l)];
      if(!dry)
      {
        go(k_cgc_prolong<V, S>, blocks(f.n), NT, f.P.smem, view<V>(f.P), (const S*)xcur[size_t(l + 1)], (S*)f.c, f.dm,
          s->sc);
        if(s->cfg.adapt_cgc == FB_CGC_MIN_ENERGY)
          go(k_cgc_apply<V, S, FB_CGC_MIN_ENERGY>, blocks(f.n), NT, f.A.smem, view<V>(f.A), (const S*)f.c, (const S*)f.d,
            (S*)f.c2, f.dm, s->cgc_omega, s->slot, s->sc);
        else
          go(k_cgc_apply<V, S, FB_CGC_MIN_DEFECT>, blocks(f.n), NT, f.A.smem, view<V>(f.A), (const S*)f.c, (const S*)f.d,
            (S*)f.c2, f.dm, s->cgc_omega, s->slot, s->sc);
        go(k_cgc_update<S>, blocks(f.n), NT, 0, (S*)xf, (const S*)f.c, (S*)f.d, (const S*)f.c2,
          (const double*)s->cgc_omega, f.n, s->sc);
      }
      launches += 3;
      bytes += csr_bytes(f.P, 1, 1) + f.n + csr_bytes(f.A, 2, 1) + f.n + double(f.n) * sizeof(S) * 6;
    }

    // ---- SOR / SSOR smoothing (fb_sor.cuh): each Richardson step sweeps its defect into y and
    // adds the filtered (SSOR: scaled) result to the smoother's iterate

    // out = F(b - A x) with explicit buffers
    void defect_into(int l, const void* b, const void* x, void* out)
    {
      DevLevel& f = L(l);
      if(dry)
        ;
      else if(use_tma(f.A))
        tma<V, S>(f.A, x, OpDefect<V, S>{(const S*)b, (S*)out, f.dm, s->sc});
      else
        go(k_defect<V, S>, blocks(f.n), NT, f.A.smem, view<V>(f.A), (const S*)b, (const S*)x, (S*)out, f.dm, s->sc);
      ++launches;
      bytes += csr_bytes(f.A, 1, 1) + f.n;
    }

    template<int KIND>
    void sweep_colours(const DevSor& q, const uint32_t* order, const uint32_t* dcofs, const std::vector<uint32_t>& hcofs,
      const void* in, void* y)
    {
      const SorCsr<S> M{q.rp, q.col, (const S*)q.val, q.posf, q.posb};
      const S w = S(s->cfg.smoother_omega);
      const uint32_t ncol = uint32_t(hcofs.size()) - 1u;
      if(ncol <= SWEEP_LAUNCH_MAX)
      {
        for(uint32_t c = 0; c < ncol; ++c)
        {
          const uint32_t cnt = hcofs[c + 1] - hcofs[c];
          if(!dry && cnt)
            go(k_sweep_colour<S, KIND>, blocks(cnt), NT, 0, M, (const S*)in, (S*)y, order + hcofs[c], cnt, w,
              (const Scalars*)s->sc);
          launches += cnt ? 1 : 0;
        }
      }
      else
      {
        if(!dry)
          go(k_sweep_block<S, KIND>, 1, SWEEP_BLOCK_NT, 0, M, (const S*)in, (S*)y, order, dcofs, ncol, w,
            (const Scalars*)s->sc);
        ++launches;
      }
    }

    // y = the sweep(s) of the level's smoother applied to `in` (y zeroed first, as the coloured
    // sweeps require)
    void sweep(int l, const void* in, void* y)
    {
      const DevSor& q = s->sor[size_t(l)];
      const uint32_t n = L(l).n;
      if(!dry)
        go(k_sweep_zero<S>, blocks(n), NT, 0, (S*)y, n, (const Scalars*)s->sc);
      ++launches;
      if(s->cfg.smoother == FB_SMOOTHER_SOR)
        sweep_colours<SW_SOR>(q, q.of, q.cf, q.hcf, in, y);
      else
      {
        sweep_colours<SW_SSOR_FWD>(q, q.of, q.cf, q.hcf, in, y);
        sweep_colours<SW_SSOR_BWD>(q, q.ob, q.cb, q.hcb, in, y);
      }
      const double nsw = s->cfg.smoother == FB_SMOOTHER_SOR ? 1.0 : 2.0;
      bytes += nsw * (double(q.nnz) * (4.0 + sizeof(S)) + double(n) * (12.0 + 2.0 * sizeof(S)));
    }

    // out = (skip ? 0 : F(scale * y) + base)
    void sweep_finish(int l, const void* y, const void* base, void* out, const int* skip)
    {
      DevLevel& f = L(l);
      const double w = s->cfg.smoother_omega;
      const bool ssor = s->cfg.smoother == FB_SMOOTHER_SSOR;
      if(!dry)
        go(k_sweep_finish<S>, blocks(f.n), NT, 0, (const S*)y, (const S*)base, (S*)out, f.dm, skip,
          S(ssor ? S(w) * (S(2.0) - S(w)) : S(1)), ssor ? 1 : 0, f.n, (const Scalars*)s->sc);
      ++launches;
      bytes += double(f.n) * ((base ? 3.0 : 2.0) * sizeof(S) + 1.0);
    }

    // pre-smoothing of level l with SOR / SSOR: x_1 = F(M b), x_k = x_{k-1} + F(M F(b - A x_{k-1}))
    void sor_pre(int l, std::vector<void*>& xcur)
    {
      DevLevel& f = L(l);
      const int steps = std::max(1, s->cfg.smooth_steps);
      void* xa = nullptr;
      void* xb = f.x;
      for(int k = 1; k <= steps; ++k)
      {
        const void* in = f.b;
        if(k > 1)
        {
          defect_into(l, f.b, xa, f.d);
          in = f.d;
        }
        sweep(l, in, f.c);
        sweep_finish(l, f.c, xa, xb, f.skip_pre);
        xa = xb;
        xb = (xb == f.x) ? f.x2 : f.x;
      }
      xcur[size_t(l)] = xa;
    }

    // post-smoothing of level l with SOR / SSOR as a correction of x: d = F(b - A x) (with the
    // smoother's skip test), c_1 = F(M d), c_k = c_{k-1} + F(M F(d - A c_{k-1})), x += c
    // (top: the PCG's z and r.z)
    void sor_post(int l, bool top, std::vector<void*>& xcur)
    {
      DevLevel& f = L(l);
      const int steps = std::max(1, s->cfg.smooth_steps);
      void* xf = xcur[size_t(l)];
      void* y = (xf == f.x) ? f.x2 : f.x;
      if(dry)
        ;
      else if(use_tma(f.A))
        tma<V, S>(f.A, xf, OpPost1<V, S>{(const S*)f.b, (S*)f.d, (S*)f.c, (const S*)f.dinv, f.dm, f.skip_post, s->sc});
      else
        go(k_post1<V, S>, blocks(f.n), NT, f.A.smem, view<V>(f.A), (const S*)f.b, (const S*)xf, (S*)f.d, (S*)f.c,
          (const S*)f.dinv, f.dm, f.skip_post, s->slot, s->sc);
      ++launches;
      bytes += csr_bytes(f.A, 2, 2) + f.n;
      void* ca = nullptr;
      void* cb = f.c;
      for(int k = 1; k <= steps; ++k)
      {
        const void* in = f.d;
        if(k > 1)
        {
          defect_into(l, f.d, ca, cb);
          in = cb;
        }
        sweep(l, in, y);
        sweep_finish(l, y, ca, cb, f.skip_post);
        ca = cb;
        cb = (cb == f.c) ? f.c2 : f.c;
      }
      if(!dry)
      {
        if(top)
          go(k_post_final<S, true>, blocks(f.n), NT, 0, (const S*)ca, (S*)xf, s->z, s->r, f.skip_post, f.n, s->slot,
            s->sc);
        else
          go(k_post_final<S, false>, blocks(f.n), NT, 0, (const S*)ca, (S*)xf, nullptr, nullptr, f.skip_post, f.n,
            s->slot, s->sc);
      }
      ++launches;
      bytes += double(f.n) * sizeof(S) * 3;
    }

    // a smoother applied as a correction: d = F(b - A x), c = Richardson-Jacobi(d) from zero, x += c
    // (post-smoothing, and the peak smoother); top: the last step also forms the PCG's z and r.z
    // from_cgc: the defect d was updated by the adaptive coarse-grid correction (no recomputation)
    void post_smooth(int l, bool top, std::vector<void*>& xcur, bool from_cgc = false)
    {
      DevLevel& f = L(l);
      const int steps = std::max(1, s->cfg.smooth_steps);
      void* xf = xcur[size_t(l)];
      if(dry)
        ;
      else if(from_cgc)
        go(k_cgc_post1<S>, blocks(f.n), NT, 0, (const S*)f.d, (S*)f.c, (const S*)f.dinv, f.dm, f.n, f.skip_post, s->slot,
          s->sc);
      else if(use_tma(f.A))
        tma<V, S>(f.A, xf, OpPost1<V, S>{(const S*)f.b, (S*)f.d, (S*)f.c, (const S*)f.dinv, f.dm, f.skip_post, s->sc});
      else
        go(k_post1<V, S>, blocks(f.n), NT, f.A.smem, view<V>(f.A), (const S*)f.b, (const S*)xf, (S*)f.d, (S*)f.c,
          (const S*)f.dinv, f.dm, f.skip_post, s->slot, s->sc);
      ++launches;
      bytes += from_cgc ? double(f.n) * (3 * sizeof(S)) + f.n : csr_bytes(f.A, 2, 2) + f.n;
      void* ca = f.c;
      void* cb = f.c2;
      if(steps == 1)
      {
        if(!dry)
        {
          if(top)
            go(k_post_final<S, true>, blocks(f.n), NT, 0, (const S*)ca, (S*)xf, s->z, s->r, f.skip_post, f.n, s->slot, s->sc);
          else
            go(k_post_final<S, false>, blocks(f.n), NT, 0, (const S*)ca, (S*)xf, nullptr, nullptr, f.skip_post, f.n, s->slot, s->sc);
        }
        ++launches;
        bytes += double(f.n) * sizeof(S) * 3;
      }
      for(int k = 2; k <= steps; ++k)
      {
        const bool last = (k == steps);
        if(dry)
          ;
        else if(use_tma(f.A))
        {
          if(!last)
            tma<V, S>(f.A, ca, OpPost2<V, S, false, false>{(const S*)f.d, (const S*)ca, (S*)cb, (S*)xf, nullptr, nullptr,
              (const S*)f.dinv, f.dm, f.skip_post, s->sc});
          else if(top)
            tma<V, S>(f.A, ca, OpPost2<V, S, true, true>{(const S*)f.d, (const S*)ca, (S*)cb, (S*)xf, s->z, s->r,
              (const S*)f.dinv, f.dm, f.skip_post, s->sc});
          else
            tma<V, S>(f.A, ca, OpPost2<V, S, true, false>{(const S*)f.d, (const S*)ca, (S*)cb, (S*)xf, nullptr, nullptr,
              (const S*)f.dinv, f.dm, f.skip_post, s->sc});
        }
        else if(!last)
          go(k_post2<V, S, false, false>, blocks(f.n), NT, f.A.smem, view<V>(f.A), (const S*)f.d, (const S*)ca,
            (S*)cb, (S*)xf, nullptr, nullptr, (const S*)f.dinv, f.dm, f.skip_post, s->slot, s->sc);
        else if(top)
          go(k_post2<V, S, true, true>, blocks(f.n), NT, f.A.smem, view<V>(f.A), (const S*)f.d, (const S*)ca,
            (S*)cb, (S*)xf, s->z, s->r, (const S*)f.dinv, f.dm, f.skip_post, s->slot, s->sc);
        else
          go(k_post2<V, S, true, false>, blocks(f.n), NT, f.A.smem, view<V>(f.A), (const S*)f.d, (const S*)ca,
            (S*)cb, (S*)xf, nullptr, nullptr, (const S*)f.dinv, f.dm, f.skip_post, s->slot, s->sc);
        ++launches;
        bytes += csr_bytes(f.A, 3, 1) + f.n;
        std::swap(ca, cb);
      }
    }

    // the coarse-level tail kernel (single block or cluster) for the events [e0, e1) of the cycle,
    // which run on levels lt and below; segment `seg` is their program
    void tail(int lt, size_t e0, size_t e1, size_t seg, std::vector<void*>& xcur)
    {
      const int nl = s->nlev;
      const int steps = std::max(1, s->cfg.smooth_steps);
      const bool ctail = s->ctail_first >= 0;
      TailParams<V, S> tp;
      std::memset(&tp, 0, sizeof(tp));
      tp.count = nl - lt;
      tp.steps = steps;
      tp.cgc = s->cfg.adapt_cgc;
      tp.free_dofs = s->free_dofs;
      tp.inv = s->cinv;
      tp.m = s->nfree;
      for(int l = lt; l < nl; ++l)
      {
        DevLevel& f = L(l);
        TailLevel<V, S>& t = tp.lv[l - lt];
        t.A = view<V>(f.A);
        if(l + 1 < nl)
        {
          t.P = view<V>(f.P);
          t.R = view<V>(f.R);
        }
        t.b = (S*)f.b;
        t.x = (S*)f.x;
        t.x2 = (S*)f.x2;
        t.d = (S*)f.d;
        t.c = (S*)f.c;
        t.c2 = (S*)f.c2;
        t.dinv = (const S*)f.dinv;
        t.dm = f.dm;
        t.skip_pre = f.skip_pre;
        t.skip_post = f.skip_post;
        t.n = f.n;
      }
      {
        // algorithmic bytes: the events as the grid kernels would run them
        const bool was_dry = dry;
        const uint64_t nlaunch = launches;
        dry = true;
        run_events(e0, e1, false, -1, xcur);
        dry = was_dry;
        launches = nlaunch;
      }
      xcur[size_t(lt)] = ((steps - 1) % 2) ? L(lt).x2 : L(lt).x;
      const size_t smem = tail_layout(tp, lt, !ctail);
      if(dry)
        ;
      else if(ctail)
      {
        cudaLaunchConfig_t lc = {};
        lc.gridDim = dim3(CT_CS, 1, 1);
        lc.blockDim = dim3(CT_NT, 1, 1);
        lc.dynamicSmemBytes = 0;
        lc.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = CT_CS;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        lc.attrs = at;
        lc.numAttrs = 1;
        const cudaError_t e = cudaLaunchKernelEx(&lc, k_ctail<V, S>, tp, (const Scalars*)s->sc, s->cred);
        if(e != cudaSuccess && s->launch_err == cudaSuccess)
          s->launch_err = e;
      }
      else if(s->cfg.cycle == FB_CYCLE_V && s->cfg.adapt_cgc == FB_CGC_FIXED)
      {
        bool all_smem = true;
        for(int t = 0; t < tp.count; ++t)
          all_smem = all_smem && tp.lv[t].in_smem;
        if(all_smem)
          go(k_tail<V, S, true>, 1, TAIL_NT, smem, tp, s->sc);
        else
          go(k_tail<V, S, false>, 1, TAIL_NT, smem, tp, s->sc);
      }
      else
        go(k_tail_prog<V, S>, 1, TAIL_NT, smem, tp, s->tail_prog + s->seg_off[seg], int(s->seg_len[seg]), s->sc);
      ++launches;
    }

    // the cycle's events [e0, e1) as grid kernels, except the runs on levels lt and below (lt >= 0),
    // which go to the tail kernel one launch each; pcg_top: the final post-smoothing forms z, r.z
    void run_events(size_t e0, size_t e1, bool pcg_top, int lt, std::vector<void*>& xcur)
    {
      const std::vector<CycEv>& ev = s->events;
      size_t seg = 0;
      for(size_t i = e0; i < e1;)
      {
        const CycEv e = ev[i];
        const int l = e.lvl;
        if(lt >= 0 && l >= lt)
        {
          size_t j = i;
          while(j < e1 && ev[j].lvl >= lt)
            ++j;
          tail(lt, i, j, seg++, xcur);
          i = j;
          continue;
        }
        // V(2,2) on a structured level: pre-smoothing, defect and restriction in one pass, and
        // prolongation and post-smoothing in one pass
        // (every fused grid's partial sums fit the reduction slot, which is sized for them)
        if(e.op == EV_PRE && fused_level(l) && L(l).fz_down && fused_down_grid(l) <= s->slot_cap && i + 2 < e1 &&
           ev[i + 1].op == EV_DEF &&
           ev[i + 1].lvl == l && ev[i + 2].op == EV_RES && ev[i + 2].lvl == l)
        {
          fused_down(l, xcur);
          i += 3;
          continue;
        }
        if(e.op == EV_PRO && fused_level(l) && L(l).fz_up && fused_up_grid(l) <= s->slot_cap && i + 1 < e1 &&
           ev[i + 1].lvl == l &&
           (ev[i + 1].op == EV_POST || ev[i + 1].op == EV_POST_TOP))
        {
          fused_up(l, ev[i + 1].op == EV_POST_TOP && pcg_top, xcur);
          i += 2;
          continue;
        }
        // the same on the large structured levels, streamed
        if(e.op == EV_PRE && stream_level(l) && L(l).fs_ok && L(l).fz_down && fs_grid(stream_geom(l, false)) <= s->slot_cap &&
           i + 2 < e1 && ev[i + 1].op == EV_DEF && ev[i + 1].lvl == l && ev[i + 2].op == EV_RES && ev[i + 2].lvl == l)
        {
          streamed_down(l, xcur);
          i += 3;
          continue;
        }
        if(e.op == EV_PRO && stream_level(l) && L(l).fs_ok && L(l).fs_up && fs_grid(stream_geom(l, true)) <= s->slot_cap &&
           i + 1 < e1 && ev[i + 1].lvl == l && (ev[i + 1].op == EV_POST || ev[i + 1].op == EV_POST_TOP))
        {
          streamed_up(l, ev[i + 1].op == EV_POST_TOP && pcg_top, xcur);
          i += 2;
          continue;
        }
        if(s->cfg.smoother != FB_SMOOTHER_JACOBI && (e.op == EV_PRE || e.op == EV_POST || e.op == EV_POST_TOP))
        {
          if(e.op == EV_PRE)
            sor_pre(l, xcur);
          else
            sor_post(l, e.op == EV_POST_TOP && pcg_top, xcur);
          ++i;
          continue;
        }
        switch(e.op)
        {
          case EV_PRE: pre_smooth(l, xcur); break;
          case EV_DEF: defect(l, xcur); break;
          case EV_RES: restrict_to(l); break;
          case EV_CRS: coarse(xcur); break;
          case EV_PRO: prolong(l, xcur); break;
          case EV_POST: post_smooth(l, false, xcur); break;
          case EV_POST_TOP: post_smooth(l, pcg_top, xcur); break;
          case EV_PROC: prolong_cgc(l, xcur); break;
          case EV_POSTC: post_smooth(l, false, xcur, true); break;
          default: post_smooth(l, pcg_top, xcur, true); break;
        }
        ++i;
      }
    }

    // One multigrid cycle from the top level; the top level's b, sol1 and skip_pre are in place.
    void vcycle(bool pcg_top)
    {
      const int nl = s->nlev;
      std::vector<void*> xcur(static_cast<size_t>(nl));
      xcur[0] = L(0).x;
      const int lt = s->ctail_first >= 0 ? s->ctail_first : s->tail_first;
      run_events(0, s->events.size(), pcg_top, lt, xcur);
      if(!dry && !pcg_top)
        s->vc_top = xcur[0];
    }

    const DevMat& A64() { return s->cfg.precision == FB_PREC_F64 ? L(0).A : L(0).A64; }

    void pcg_init()
    {
      DevLevel& t = L(0);
      const bool f64 = s->cfg.precision == FB_PREC_F64;
      const DevMat& A = A64();
      if(!dry) go(k_pcg_init<S>, blocks(t.n), NT, A.smem, view<double>(A), s->rhs, s->x, s->r, t.dm,
        f64 ? (S*)t.x : (S*)nullptr, (const S*)t.dinv, t.skip_pre, s->hist, s->slot, s->sc, 0);
      ++launches;
      bytes += A.bytes + double(t.n) * 8 * 4 + t.n;
      if(!f64)
      {
        if(!dry) go(k_mg_prep<S>, blocks(t.n), NT, 0, s->r, (S*)t.b, (S*)t.x, (const S*)t.dinv, t.dm, t.skip_pre, t.n, 1,
          s->slot, s->sc);
        ++launches;
        bytes += double(t.n) * (8 + 3 * sizeof(S)) + t.n;
      }
    }

    void pcg_tail(bool first, cudaGraphConditionalHandle cond)
    {
      DevLevel& t = L(0);
      const bool f64 = s->cfg.precision == FB_PREC_F64;
      const DevMat& A = A64();
      if(!dry) go(k_pcg_p, blocks(t.n), NT, 0, s->p, s->z, t.n, first ? 1 : 0, s->sc);
      if(dry)
        ;
      else if(use_tma_f64(A))
        tma<double, double>(A, s->p, OpPcgQ{s->p, s->q, t.dm, s->sc});
      else
        go(k_pcg_q, blocks(t.n), NT, A.smem, view<double>(A), s->p, s->q, t.dm, s->slot, s->sc);
      if(dry)
        ;
      else if(f64)
        go(k_pcg_x<S, false>, pcgx_grid(t.n), NT, 0, s->x, s->r, s->p, s->q, t.dm, (S*)nullptr, (S*)t.x,
          (const S*)t.dinv, t.skip_pre, s->hist, t.n, s->slot, s->sc, cond);
      else
        go(k_pcg_x<S, true>, pcgx_grid(t.n), NT, 0, s->x, s->r, s->p, s->q, t.dm, (S*)t.b, (S*)t.x,
          (const S*)t.dinv, t.skip_pre, s->hist, t.n, s->slot, s->sc, cond);
      launches += 3;
      bytes += double(t.n) * 8 * (first ? 2 : 3);                                    // P
      bytes += A.bytes + double(t.n) * 8 * 3 + t.n;                                   // Q
      bytes += double(t.n) * 8 * 6 + double(t.n) * (f64 ? 16 : 12) + t.n;             // X
    }
  };

  // dynamic shared memory of the streamed passes and their resident blocks per SM
  template<typename V, typename S>
  static fb_status fs_occupancy(fb_solver* s)
  {
    typedef FsLay<V, S, false, false> LD;
    typedef FsLay<V, S, true, true> LU;
    typedef FsLay<V, S, true, false> LN;
    FB_CUDA(cudaFuncSetAttribute(k_fs_down<V, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(LD::SMEM)));
    FB_CUDA(cudaFuncSetAttribute(k_fs_up<V, S, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(LU::SMEM)));
    FB_CUDA(cudaFuncSetAttribute(k_fs_up<V, S, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(LN::SMEM)));
    FB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&s->fs_bps_down, k_fs_down<V, S>, FS_NT, LD::SMEM));
    FB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&s->fs_bps_up, k_fs_up<V, S, true>, FS_NT, LU::SMEM));
    s->fs_bps_down = std::max(1, s->fs_bps_down);
    s->fs_bps_up = std::max(1, s->fs_bps_up);
    return FB_OK;
  }

  template<typename V, typename S, class Op>
  static fb_status set_tma_attr_dg(int mx)
  {
    FB_CUDA(cudaFuncSetAttribute(k_tma_pass<V, S, Op, 9, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FB_CUDA(cudaFuncSetAttribute(k_tma_pass<V, S, Op, 27, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    return FB_OK;
  }

  // dynamic shared memory above 48 KB for the TMA-staged passes
  template<typename V, typename S>
  static fb_status set_tma_attrs()
  {
    const int mx = int(TMA_SMEM_MAX) + 8 * 1024;
    FB_CUDA(cudaFuncSetAttribute(k_tma_pass<V, S, OpSmooth<V, S>, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FB_CUDA(cudaFuncSetAttribute(k_tma_pass<V, S, OpSmooth<V, S>, 9>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FB_CUDA(cudaFuncSetAttribute(k_tma_pass<V, S, OpDefect<V, S>, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FB_CUDA(cudaFuncSetAttribute(k_tma_pass<V, S, OpDefect<V, S>, 9>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FB_CUDA(cudaFuncSetAttribute(k_tma_pass<V, S, OpPost1<V, S>, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FB_CUDA(cudaFuncSetAttribute(k_tma_pass<V, S, OpPost1<V, S>, 9>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FB_CUDA(cudaFuncSetAttribute(k_tma_pass<V, S, OpPost2<V, S, false, false>, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FB_CUDA(cudaFuncSetAttribute(k_tma_pass<V, S, OpPost2<V, S, false, false>, 9>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FB_CUDA(cudaFuncSetAttribute(k_tma_pass<V, S, OpPost2<V, S, true, false>, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FB_CUDA(cudaFuncSetAttribute(k_tma_pass<V, S, OpPost2<V, S, true, false>, 9>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FB_CUDA(cudaFuncSetAttribute(k_tma_pass<V, S, OpPost2<V, S, true, true>, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FB_CUDA(cudaFuncSetAttribute(k_tma_pass<V, S, OpPost2<V, S, true, true>, 9>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FB_CUDA(cudaFuncSetAttribute(k_tma_pass<V, S, OpRestrict<V, S>, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FB_CUDA(cudaFuncSetAttribute(k_tma_pass<V, S, OpRestrict<V, S>, 9>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FB_CUDA(cudaFuncSetAttribute(k_tma_pass<V, S, OpProlong<V, S>, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FB_CUDA(cudaFuncSetAttribute(k_tma_pass<V, S, OpProlong<V, S>, 9>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FB_CUDA(cudaFuncSetAttribute(k_tma_pass<double, double, OpPcgQ, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FB_CUDA(cudaFuncSetAttribute(k_tma_pass<double, double, OpPcgQ, 9>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FB_TRY((set_tma_attr_dg<V, S, OpSmooth<V, S>>(mx)));
    FB_TRY((set_tma_attr_dg<V, S, OpDefect<V, S>>(mx)));
    FB_TRY((set_tma_attr_dg<V, S, OpPost1<V, S>>(mx)));
    FB_TRY((set_tma_attr_dg<V, S, OpPost2<V, S, false, false>>(mx)));
    FB_TRY((set_tma_attr_dg<V, S, OpPost2<V, S, true, false>>(mx)));
    FB_TRY((set_tma_attr_dg<V, S, OpPost2<V, S, true, true>>(mx)));
    FB_TRY((set_tma_attr_dg<double, double, OpPcgQ>(mx)));
    FB_CUDA(cudaFuncSetAttribute(k_tail<V, S, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(TAIL_SMEM_MAX)));
    FB_CUDA(cudaFuncSetAttribute(k_tail<V, S, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(TAIL_SMEM_MAX)));
    FB_CUDA(cudaFuncSetAttribute(k_tail_prog<V, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(TAIL_SMEM_MAX)));
    return FB_OK;
  }

  template<typename V, typename S>
  static fb_status build_graphs(fb_solver* s)
  {
    cudaStream_t st = s->stream;
    {
      Launcher<V, S> li{s, st, true};
      li.pcg_init();
      li.vcycle(true);
      li.pcg_tail(true, 0);
      s->launches_init = li.launches;
      s->bytes_init = li.bytes;
      Launcher<V, S> lb{s, st, true};
      lb.vcycle(true);
      lb.pcg_tail(false, 0);
      s->launches_body = lb.launches;
      s->bytes_body = lb.bytes;
      Launcher<V, S> lv{s, st, true};
      lv.vcycle(false);
      s->launches_vcycle = lv.launches + 2;
    }
    if(!s->cfg.use_graph)
      return FB_OK;
    FB_CUDA(cudaGraphCreate(&s->graph, 0));
    cudaGraphConditionalHandle cond;
    FB_CUDA(cudaGraphConditionalHandleCreate(&cond, s->graph, 0u, cudaGraphCondAssignDefault));
    FB_CUDA(cudaStreamBeginCaptureToGraph(st, s->graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    {
      Launcher<V, S> l{s, st, false};
      l.pcg_init();
      l.vcycle(true);
      l.pcg_tail(true, cond);
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
      Launcher<V, S> l{s, st, false};
      l.vcycle(true);
      l.pcg_tail(false, cond);
    }
    cudaGraph_t b_out = nullptr;
    FB_CUDA(cudaStreamEndCapture(st, &b_out));
    FB_CUDA(cudaGraphInstantiate(&s->gexec, s->graph, 0));
    return FB_OK;
  }

  template<typename V, typename S>
  static fb_status run_solve(fb_solver* s)
  {
    cudaStream_t st = s->stream;
    if(s->cfg.use_graph)
    {
      FB_CUDA(cudaGraphLaunch(s->gexec, st));
      FB_CUDA(cudaGetLastError());
      return FB_OK;
    }
    Launcher<V, S> li{s, st, false};
    li.pcg_init();
    li.vcycle(true);
    li.pcg_tail(true, 0);
    FB_LAUNCHED(0);
    while(true)
    {
      Scalars h;
      FB_CUDA(cudaMemcpyAsync(&h, s->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st));
      FB_CUDA(cudaStreamSynchronize(st));
      if(h.status != FB_SOLVER_PROGRESS)
        break;
      Launcher<V, S> lb{s, st, false};
      lb.vcycle(true);
      lb.pcg_tail(false, 0);
      FB_LAUNCHED(0);
    }
    return FB_OK;
  }

  template<typename V, typename S>
  static fb_status run_vcycle(fb_solver* s)
  {
    cudaStream_t st = s->stream;
    DevLevel& t = s->lv[0];
    Launcher<V, S> l{s, st, false};
    // the status gate must be open for the V-cycle passes
    k_set_status<<<1, 1, 0, st>>>(s->sc, FB_SOLVER_PROGRESS);
    // FP64 mode: the top level's b aliases r and is not rewritten
    const bool f64 = s->cfg.precision == FB_PREC_F64;
    k_mg_prep<S><<<blocks(t.n), NT, 0, st>>>(s->r, f64 ? (S*)nullptr : (S*)t.b, (S*)t.x, (const S*)t.dinv, t.dm,
      t.skip_pre, t.n, 0, s->slot, s->sc);
    FB_LAUNCHED(2);
    l.vcycle(false);
    FB_LAUNCHED(l.launches);
    return FB_OK;
  }
} // namespace fb

using namespace fb;

extern "C" {

void fb_solver_config_default(fb_solver_config* c)
{
  if(!c)
    return;
  c->precision = FB_PREC_F64;
  c->ordering = FB_ORDER_NATIVE;
  c->omega = 0.7;
  c->smooth_steps = 2;
  c->tol_rel = 1e-8;
  c->tol_abs = 1.0 / (EPS64 * EPS64);
  c->max_iter = 100;
  c->min_iter = 0;
  c->use_graph = 1;
  c->rows_per_block = 0;
  c->tail_rows = 300;
  c->cluster_rows = 0;
  c->cycle = FB_CYCLE_V;
  c->tma_rows = 1000;
  c->tma_window = 0;
  c->diagonal = 1;
  c->pdl = 1;
  c->adapt_cgc = FB_CGC_FIXED;
  c->fused = 70000;
  c->smoother = FB_SMOOTHER_JACOBI;
  c->smoother_omega = 1.0;
  c->sweep_colouring = FB_SWEEP_SEQUENTIAL;
  c->streamed = 0;
}

fb_status fb_hierarchy_create(fb_hierarchy** out, int num_levels)
{
  if(!out || num_levels < 1 || num_levels > 32)
  {
    set_error("hierarchy_create: bad arguments");
    return FB_ERR_ARG;
  }
  *out = new fb_hierarchy();
  (*out)->levels.resize(size_t(num_levels));
  return FB_OK;
}

void fb_hierarchy_destroy(fb_hierarchy* h) { delete h; }

fb_status fb_hierarchy_set_level(fb_hierarchy* h, int level, const fb_csr_host* A, const uint64_t* filter_idx,
  const double* filter_val, uint64_t nf, const fb_csr_host* P, const fb_csr_host* R)
{
  if(!h || level < 0 || size_t(level) >= h->levels.size() || !A)
  {
    set_error("hierarchy_set_level: bad arguments");
    return FB_ERR_ARG;
  }
  const bool coarsest = size_t(level) + 1 == h->levels.size();
  if(!coarsest && (!P || !R))
  {
    set_error("hierarchy_set_level: P and R are required on every level but the coarsest");
    return FB_ERR_ARG;
  }
  if(A->rows != A->columns)
  {
    set_error("hierarchy_set_level: system matrix is not square");
    return FB_ERR_ARG;
  }
  HostLevel& L = h->levels[size_t(level)];
  std::string e = import_csr(L.A, A->rows, A->columns, A->used_elements, A->row_ptr, A->col_ind, A->val, false);
  if(e.empty() && !coarsest)
  {
    if(P->rows != A->rows || R->columns != A->rows || R->rows != P->columns)
      e = "transfer matrix sizes do not match the system matrix";
    if(e.empty())
      e = import_csr(L.P, P->rows, P->columns, P->used_elements, P->row_ptr, P->col_ind, P->val, true);
    if(e.empty())
      e = import_csr(L.R, R->rows, R->columns, R->used_elements, R->row_ptr, R->col_ind, R->val, true);
  }
  if(!e.empty())
  {
    set_error("hierarchy_set_level: " + e);
    return FB_ERR_ARG;
  }
  L.dmask.assign(A->rows, 0);
  L.fidx.assign(filter_idx, filter_idx + nf);
  L.fval.assign(filter_val ? filter_val : filter_val, filter_val ? filter_val + nf : filter_val);
  for(uint64_t k = 0; k < nf; ++k)
  {
    if(filter_idx[k] >= A->rows)
    {
      set_error("hierarchy_set_level: filter index out of range");
      return FB_ERR_ARG;
    }
    L.dmask[filter_idx[k]] = 1;
  }
  L.set = true;
  return FB_OK;
}

void fb_solver_destroy(fb_solver* s)
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

fb_status fb_solver_create(fb_solver** out, fb_hierarchy* h, const fb_solver_config* cfg_in)
{
  if(!out || !h)
  {
    set_error("solver_create: bad arguments");
    return FB_ERR_ARG;
  }
  for(const HostLevel& L : h->levels)
    if(!L.set)
    {
      set_error("solver_create: every level must be set");
      return FB_ERR_STATE;
    }
  fb_solver_config cfg;
  if(cfg_in)
    cfg = *cfg_in;
  else
    fb_solver_config_default(&cfg);
  if(cfg.precision < FB_PREC_F64 || cfg.precision > FB_PREC_F32_BF16 || cfg.smooth_steps < 1 || cfg.max_iter < 0 ||
     cfg.cycle < FB_CYCLE_V || cfg.cycle > FB_CYCLE_W || cfg.adapt_cgc < FB_CGC_FIXED ||
     cfg.adapt_cgc > FB_CGC_MIN_DEFECT || cfg.smoother < FB_SMOOTHER_JACOBI || cfg.smoother > FB_SMOOTHER_SSOR ||
     (cfg.smoother != FB_SMOOTHER_JACOBI && !(cfg.smoother_omega > 0.0)) || cfg.sweep_colouring < FB_SWEEP_SEQUENTIAL ||
     cfg.sweep_colouring > FB_SWEEP_COLOURED || cfg.streamed < 0)
  {
    set_error("solver_create: bad configuration");
    return FB_ERR_ARG;
  }
  if(cfg.smoother != FB_SMOOTHER_JACOBI && (cfg.adapt_cgc != FB_CGC_FIXED || cfg.ordering != FB_ORDER_NATIVE))
  {
    // a sweep's result depends on the row numbering: it runs in the caller's numbering only
    set_error("solver_create: SOR / SSOR smoothing needs the caller's numbering (FB_ORDER_NATIVE) and the fixed "
              "coarse-grid correction");
    return FB_ERR_UNSUPPORTED;
  }
  std::unique_ptr<fb_solver, void (*)(fb_solver*)> s(new fb_solver(), fb_solver_destroy);
  s->cfg = cfg;
  s->h = h;
  s->nlev = int(h->levels.size());
  const int prec = cfg.precision;
  FB_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  FB_CUDA(cudaEventCreate(&s->ev0));
  FB_CUDA(cudaEventCreate(&s->ev1));

  // orderings (device row k = caller row perm[k])
  s->perms.assign(size_t(s->nlev), std::vector<uint32_t>());
  if(cfg.ordering == FB_ORDER_RCM)
    for(int l = 0; l < s->nlev; ++l)
      s->perms[size_t(l)] = rcm_order(h->levels[size_t(l)].A);

  s->lv.resize(size_t(s->nlev));
  const size_t vs = vsize_of(prec);
  uint32_t max_blocks = 1;
  // Dirichlet masks in device numbering: their rows are stored empty (the filter discards them)
  std::vector<std::vector<uint8_t>> dms(size_t(s->nlev));
  for(int l = 0; l < s->nlev; ++l)
  {
    const HostLevel& H = h->levels[size_t(l)];
    const std::vector<uint32_t>& pf = s->perms[size_t(l)];
    dms[size_t(l)].resize(H.A.rows);
    for(uint32_t k = 0; k < H.A.rows; ++k)
      dms[size_t(l)][k] = H.dmask[pf.empty() ? k : pf[k]];
  }
  for(int l = 0; l < s->nlev; ++l)
  {
    const HostLevel& H = h->levels[size_t(l)];
    DevLevel& D = s->lv[size_t(l)];
    const std::vector<uint32_t>& pf = s->perms[size_t(l)];
    const std::vector<uint32_t> inv_f = pf.empty() ? std::vector<uint32_t>() : inverse_perm(pf);
    D.n = H.A.rows;
    max_blocks = std::max(max_blocks, blocks(D.n));
    HostCsr A = permute(H.A, pf, inv_f);
    FB_TRY(upload_mat(s.get(), D.A, A, prec, &dms[size_t(l)], cfg.diagonal != 0));
    if(l == 0 && prec != FB_PREC_F64)
      FB_TRY(upload_mat(s.get(), D.A64, A, FB_PREC_F64, &dms[size_t(l)], cfg.diagonal != 0));
    if(l + 1 < s->nlev)
    {
      const std::vector<uint32_t>& pc = s->perms[size_t(l + 1)];
      const std::vector<uint32_t> inv_c = pc.empty() ? std::vector<uint32_t>() : inverse_perm(pc);
      FB_TRY(upload_mat(s.get(), D.P, permute(H.P, pf, inv_c), prec, &dms[size_t(l)]));
      FB_TRY(upload_mat(s.get(), D.R, permute(H.R, pc, inv_f), prec, &dms[size_t(l + 1)]));
    }
    if(l + 1 < s->nlev)
    {
      D.gw = grid2d_width(A, D.A);
      D.fz_up = D.gw != 0 && D.P.col && !D.P.dcol && D.P.kmax <= uint32_t(FZ_KP);
      const std::vector<uint32_t>& pc = s->perms[size_t(l + 1)];
      D.fz_down = D.gw != 0 && D.R.col && !D.R.dcol && D.R.kmax <= uint32_t(FZ_KR) &&
                  restriction_local(permute(H.R, pc, inv_f), D.gw);
      D.fs_up = D.fz_up &&
                prolongation_local(permute(H.P, pf, pc.empty() ? std::vector<uint32_t>() : inverse_perm(pc)), D.gw);
      D.fs_ok = D.gw != 0 && boundary_dirichlet(dms[size_t(l)], D.gw);
    }
    const std::vector<uint8_t>& dm = dms[size_t(l)];
    FB_TRY(dalloc(s.get(), (void**)&D.dm, D.n));
    FB_CUDA(cudaMemcpy(D.dm, dm.data(), D.n, cudaMemcpyHostToDevice));
    std::vector<double> dinv = inv_diagonal(A, cfg.omega);
    if(prec == FB_PREC_F64)
      FB_TRY(upload_vec<double>(s.get(), &D.dinv, dinv));
    else
      FB_TRY(upload_vec<float>(s.get(), &D.dinv, dinv));
    for(void** v : {&D.b, &D.x, &D.x2, &D.d, &D.c, &D.c2})
      FB_TRY(dalloc(s.get(), v, vs * D.n));
    FB_TRY(dalloc(s.get(), (void**)&D.skip_pre, 2 * sizeof(int)));
    D.skip_post = D.skip_pre + 1;
    if(l == s->nlev - 1)
    {
      // exact inverse on the caller numbering; free DOFs mapped to device rows
      std::vector<uint32_t> fr;
      std::vector<double> inv;
      coarse_inverse(H.A, H.dmask, fr, inv);
      const std::vector<uint32_t> invp = pf.empty() ? std::vector<uint32_t>() : inverse_perm(pf);
      for(uint32_t& f : fr)
        f = invp.empty() ? f : invp[f];
      s->nfree = uint32_t(fr.size());
      FB_TRY(dalloc(s.get(), (void**)&s->free_dofs, sizeof(uint32_t) * std::max<size_t>(1, fr.size())));
      FB_TRY(dalloc(s.get(), (void**)&s->cinv, sizeof(double) * std::max<size_t>(1, inv.size())));
      if(!fr.empty())
      {
        FB_CUDA(cudaMemcpy(s->free_dofs, fr.data(), sizeof(uint32_t) * fr.size(), cudaMemcpyHostToDevice));
        FB_CUDA(cudaMemcpy(s->cinv, inv.data(), sizeof(double) * inv.size(), cudaMemcpyHostToDevice));
      }
    }
  }
  // FP64 mode: the top level's V-cycle input b aliases the PCG defect r
  const uint32_t n0 = s->lv[0].n;
  FB_TRY(dalloc(s.get(), (void**)&s->x, 8 * size_t(n0)));
  FB_TRY(dalloc(s.get(), (void**)&s->r, 8 * size_t(n0)));
  FB_TRY(dalloc(s.get(), (void**)&s->p, 8 * size_t(n0)));
  FB_TRY(dalloc(s.get(), (void**)&s->q, 8 * size_t(n0)));
  FB_TRY(dalloc(s.get(), (void**)&s->rhs, 8 * size_t(n0)));
  FB_TRY(dalloc(s.get(), (void**)&s->tmp_in, 8 * size_t(n0)));
  FB_TRY(dalloc(s.get(), (void**)&s->tmp_out, 8 * size_t(n0)));
  if(prec == FB_PREC_F64)
  {
    s->lv[0].b = s->r;
    // z is the top level's final solution buffer: POST2 (TOP) writes it directly
    FB_TRY(dalloc(s.get(), (void**)&s->z, 8 * size_t(n0)));
  }
  else
    FB_TRY(dalloc(s.get(), (void**)&s->z, 8 * size_t(n0)));
  if(!s->perms[0].empty())
  {
    FB_TRY(dalloc(s.get(), (void**)&s->perm0, sizeof(uint32_t) * n0));
    FB_CUDA(cudaMemcpy(s->perm0, s->perms[0].data(), sizeof(uint32_t) * n0, cudaMemcpyHostToDevice));
  }
  FB_TRY(dalloc(s.get(), (void**)&s->hist, sizeof(double) * (size_t(cfg.max_iter) + 2)));
  FB_TRY(dalloc(s.get(), (void**)&s->sc, sizeof(Scalars)));
  FB_TRY(dalloc(s.get(), (void**)&s->err, sizeof(int)));
  {
    int dev = 0;
    FB_CUDA(cudaGetDevice(&dev));
    FB_CUDA(cudaDeviceGetAttribute(&s->nsm, cudaDevAttrMultiProcessorCount, dev));
  }
  // the fused passes' grids: ceil(W / 16)^2 (up, 16 x 16 fine tiles) and ceil(Wc / 8)^2 (down,
  // 8 x 8 coarse tiles) blocks, each with two partial sums
  for(int l = 0; l + 1 < s->nlev; ++l)
  {
    const DevLevel& D = s->lv[size_t(l)];
    if(!D.gw)
      continue;
    const uint32_t tu = (D.gw + FZ_UP_TILE - 1) / FZ_UP_TILE, td = ((D.gw + 1) / 2 + FZ_DOWN_TILE - 1) / FZ_DOWN_TILE;
    max_blocks = std::max(max_blocks, std::max(tu * tu, td * td));
  }
  // the streamed passes' grids (tiles sized for the resident blocks of one wave)
  {
    fb_status fe = FB_OK;
    if(prec == FB_PREC_F64)
      fe = fs_occupancy<double, double>(s.get());
    else if(prec == FB_PREC_F32)
      fe = fs_occupancy<float, float>(s.get());
    else
      fe = fs_occupancy<bf16_t, float>(s.get());
    if(fe != FB_OK)
      return fe;
    for(int l = 0; l + 1 < s->nlev; ++l)
    {
      const DevLevel& D = s->lv[size_t(l)];
      if(!D.gw)
        continue;
      max_blocks = std::max(max_blocks, fs_grid(fs_geom(D.gw, s->nsm, s->fs_bps_down)));
      max_blocks = std::max(max_blocks, fs_grid(fs_geom(D.gw, s->nsm, s->fs_bps_up)));
    }
  }
  s->slot_cap = max_blocks;
  FB_TRY(dalloc(s.get(), (void**)&s->slot.partials, sizeof(double) * 2 * (max_blocks + 1)));
  FB_TRY(dalloc(s.get(), (void**)&s->cgc_omega, sizeof(double)));
  FB_TRY(dalloc(s.get(), (void**)&s->slot.counter, sizeof(unsigned int) * 4));
  // SOR / SSOR sweeps: every level but the coarsest gets the full system matrix in CSR (stored
  // order), the diagonal positions and the sweep orders
  if(cfg.smoother != FB_SMOOTHER_JACOBI)
  {
    s->sor.resize(size_t(s->nlev));
    for(int l = 0; l + 1 < s->nlev; ++l)
    {
      const HostCsr& A = h->levels[size_t(l)].A;
      DevSor& q = s->sor[size_t(l)];
      const uint32_t n = A.rows;
      std::vector<uint32_t> posf(n), posb(n);
      for(uint32_t i = 0; i < n; ++i)
      {
        uint32_t k = A.rp[i];
        while(k < A.rp[i + 1] && A.col[k] < i)
          ++k;
        uint32_t kb = A.rp[i + 1];
        while(kb > A.rp[i] && A.col[kb - 1] > i)
          --kb;
        if(k >= A.rp[i + 1] || A.col[k] != i || kb == A.rp[i] || A.col[kb - 1] != i)
        {
          set_error("solver_create: SOR / SSOR smoothing needs every row's diagonal entry, columns sorted");
          return FB_ERR_UNSUPPORTED;
        }
        posf[i] = k;
        posb[i] = kb - 1;
      }
      q.nnz = A.nnz();
      FB_TRY(upload_u32(s.get(), &q.rp, A.rp));
      FB_TRY(upload_u32(s.get(), &q.col, A.col));
      FB_TRY(upload_u32(s.get(), &q.posf, posf));
      FB_TRY(upload_u32(s.get(), &q.posb, posb));
      if(prec == FB_PREC_F64)
        FB_TRY(upload_vec<double>(s.get(), &q.val, A.val));
      else
      {
        // the V-cycle's values: FP32, or BF16-rounded in the BF16-value mode
        std::vector<double> v(A.val);
        if(prec == FB_PREC_F32_BF16)
          for(double& x : v)
          {
            const uint32_t u = uint32_t(to_bf16_rne(float(x))) << 16;
            float f;
            std::memcpy(&f, &u, sizeof(f));
            x = double(f);
          }
        FB_TRY(upload_vec<float>(s.get(), &q.val, v));
      }
      const SweepOrder fw = cfg.sweep_colouring == FB_SWEEP_COLOURED ? greedy_colours(A) : sweep_levels(A, false);
      const SweepOrder bw = cfg.sweep_colouring == FB_SWEEP_COLOURED ? fw : sweep_levels(A, true);
      FB_TRY(upload_u32(s.get(), &q.of, fw.order));
      FB_TRY(upload_u32(s.get(), &q.cf, fw.cofs));
      FB_TRY(upload_u32(s.get(), &q.ob, bw.order));
      FB_TRY(upload_u32(s.get(), &q.cb, bw.cofs));
      q.hcf = fw.cofs;
      q.hcb = bw.cofs;
    }
  }
  // the tail starts at the first level (below the top) with at most tail_rows rows, if it has a
  // coarser level below it (Jacobi smoothing only: the tail kernels run no sweeps)
  s->tail_first = -1;
  s->ctail_first = -1;
  if(cfg.smoother != FB_SMOOTHER_JACOBI)
    ;
  else if(cfg.cluster_rows > 0 && cfg.cycle == FB_CYCLE_V && cfg.adapt_cgc == FB_CGC_FIXED)
    for(int l = 1; l + 1 < s->nlev; ++l)
      if(s->lv[size_t(l)].n <= uint32_t(cfg.cluster_rows))
      {
        s->ctail_first = (s->nlev - l <= MAX_TAIL) ? l : -1;
        break;
      }
  if(s->ctail_first >= 0)
    FB_TRY(dalloc(s.get(), (void**)&s->cred, sizeof(double) * 2 * MAX_TAIL * CT_CS));
  if(cfg.tail_rows > 0 && s->ctail_first < 0 && cfg.smoother == FB_SMOOTHER_JACOBI)
    for(int l = 1; l + 1 < s->nlev; ++l)
      if(s->lv[size_t(l)].n <= uint32_t(cfg.tail_rows))
      {
        s->tail_first = (s->nlev - l <= MAX_TAIL) ? l : -1;
        break;
      }
  // the cycle as events, and the tail kernel's program for each run of events on the tail levels
  // (identical runs share one program)
  s->events = cycle_events(cfg.cycle, s->nlev, cfg.adapt_cgc != FB_CGC_FIXED);
  if(s->tail_first >= 0 && (cfg.cycle != FB_CYCLE_V || cfg.adapt_cgc != FB_CGC_FIXED))
  {
    const int lt = s->tail_first;
    std::vector<uint8_t> progs;
    std::map<std::vector<uint8_t>, uint32_t> seen;
    for(size_t i = 0; i < s->events.size();)
    {
      if(s->events[i].lvl < lt)
      {
        ++i;
        continue;
      }
      std::vector<uint8_t> pg;
      for(; i < s->events.size() && s->events[i].lvl >= lt; ++i)
        pg.push_back(uint8_t((s->events[i].op << 4) | (s->events[i].lvl - lt)));
      auto it = seen.find(pg);
      if(it == seen.end())
      {
        it = seen.emplace(pg, uint32_t(progs.size())).first;
        progs.insert(progs.end(), pg.begin(), pg.end());
      }
      s->seg_off.push_back(it->second);
      s->seg_len.push_back(uint32_t(pg.size()));
    }
    FB_TRY(dalloc(s.get(), (void**)&s->tail_prog, progs.size()));
    FB_CUDA(cudaMemcpy(s->tail_prog, progs.data(), progs.size(), cudaMemcpyHostToDevice));
  }
  Scalars h0;
  std::memset(&h0, 0, sizeof(h0));
  h0.tol_rel = cfg.tol_rel;
  h0.tol_abs = cfg.tol_abs;
  h0.div_rel = 1.0 / EPS64;
  h0.div_abs = 1.0 / (EPS64 * EPS64);
  h0.min_iter = cfg.min_iter;
  h0.max_iter = cfg.max_iter;
  s->max_iter_cap = cfg.max_iter;
  h0.mg_scale = 1.0;
  h0.mg_inv_scale = 1.0;
  FB_CUDA(cudaMemcpy(s->sc, &h0, sizeof(h0), cudaMemcpyHostToDevice));

  fb_status e = FB_OK;
  if(prec == FB_PREC_F64)
    e = set_tma_attrs<double, double>();
  else if(prec == FB_PREC_F32)
    e = set_tma_attrs<float, float>();
  else
    e = set_tma_attrs<bf16_t, float>();
  if(e != FB_OK)
    return e;
  if(prec == FB_PREC_F64)
  {
    e = build_graphs<double, double>(s.get());
  }
  else if(prec == FB_PREC_F32)
  {
    e = build_graphs<float, float>(s.get());
  }
  else
  {
    e = build_graphs<bf16_t, float>(s.get());
  }
  if(e != FB_OK)
    return e;
  FB_CUDA(cudaDeviceSynchronize());
  *out = s.release();
  return FB_OK;
}

} // extern "C"

namespace fb
{
  template<typename V, typename S>
  static fb_status solve_dispatch(fb_solver* s) { return run_solve<V, S>(s); }
  template<typename V, typename S>
  static fb_status vcycle_dispatch(fb_solver* s) { return run_vcycle<V, S>(s); }

} // namespace fb

extern "C" {

static fb_status solve_common(fb_solver* s, fb_solve_info* info)
{
  cudaStream_t st = s->stream;
  const uint32_t n0 = s->lv[0].n;
  FB_CUDA(cudaEventRecord(s->ev0, st));
  fb_status e = FB_OK;
  if(s->cfg.precision == FB_PREC_F64)
    e = solve_dispatch<double, double>(s);
  else if(s->cfg.precision == FB_PREC_F32)
    e = solve_dispatch<float, float>(s);
  else
    e = solve_dispatch<bf16_t, float>(s);
  if(e != FB_OK)
    return e;
  if(s->launch_err != cudaSuccess)
  {
    const cudaError_t le = s->launch_err;
    s->launch_err = cudaSuccess;
    return cuda_fail(le, "cluster tail launch");
  }
  FB_CUDA(cudaEventRecord(s->ev1, st));
  Scalars h;
  int err = 0;
  FB_CUDA(cudaMemcpyAsync(&h, s->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st));
  FB_CUDA(cudaMemcpyAsync(&err, s->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  FB_CUDA(cudaStreamSynchronize(st));
  if(err)
  {
    FB_CUDA(cudaMemsetAsync(s->err, 0, sizeof(int), st));
    set_error("solve: a bounded wait for staged matrix data expired (results invalid)");
    return FB_ERR_CUDA;
  }
  (void)n0;
  count_launches(s->launches_init + (h.iter > 1 ? uint64_t(h.iter - 1) : 0) * s->launches_body);
  if(info)
  {
    info->status = h.status;
    info->iterations = h.iter;
    info->def_init = h.def_init;
    info->def_final = h.def_cur;
    float ms = 0.f;
    FB_CUDA(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    info->solve_ms = double(ms);
    const uint64_t body_runs = h.iter > 1 ? uint64_t(h.iter - 1) : 0;
    info->kernel_launches = s->launches_init + body_runs * s->launches_body;
    info->bytes_moved = s->bytes_init + double(body_runs) * s->bytes_body;
  }
  return FB_OK;
}

// copies a caller-numbered device vector into the device numbering (or plain copy)
static fb_status to_device_order(fb_solver* s, double* dst, const double* src)
{
  const uint32_t n = s->lv[0].n;
  if(s->perm0)
  {
    k_gather<<<blocks(n), NT, 0, s->stream>>>(dst, src, s->perm0, n);
    FB_LAUNCHED(1);
  }
  else
    FB_CUDA(cudaMemcpyAsync(dst, src, 8 * size_t(n), cudaMemcpyDeviceToDevice, s->stream));
  return FB_OK;
}

static fb_status from_device_order(fb_solver* s, double* dst, const double* src)
{
  const uint32_t n = s->lv[0].n;
  if(s->perm0)
  {
    k_scatter<<<blocks(n), NT, 0, s->stream>>>(dst, src, s->perm0, n);
    FB_LAUNCHED(1);
  }
  else
    FB_CUDA(cudaMemcpyAsync(dst, src, 8 * size_t(n), cudaMemcpyDeviceToDevice, s->stream));
  return FB_OK;
}

fb_status fb_solver_solve(fb_solver* s, double* sol, const double* rhs, fb_solve_info* info)
{
  if(!s || !sol || !rhs)
  {
    set_error("solver_solve: bad arguments");
    return FB_ERR_ARG;
  }
  const uint32_t n = s->lv[0].n;
  FB_CUDA(cudaMemcpyAsync(s->tmp_in, rhs, 8 * size_t(n), cudaMemcpyHostToDevice, s->stream));
  FB_TRY(to_device_order(s, s->rhs, s->tmp_in));
  FB_CUDA(cudaMemcpyAsync(s->tmp_in, sol, 8 * size_t(n), cudaMemcpyHostToDevice, s->stream));
  FB_TRY(to_device_order(s, s->x, s->tmp_in));
  FB_TRY(solve_common(s, info));
  FB_TRY(from_device_order(s, s->tmp_out, s->x));
  FB_CUDA(cudaMemcpyAsync(sol, s->tmp_out, 8 * size_t(n), cudaMemcpyDeviceToHost, s->stream));
  FB_CUDA(cudaStreamSynchronize(s->stream));
  return FB_OK;
}

fb_status fb_solver_solve_device(fb_solver* s, double* sol, const double* rhs, void* stream, fb_solve_info* info)
{
  if(!s || !sol || !rhs)
  {
    set_error("solver_solve_device: bad arguments");
    return FB_ERR_ARG;
  }
  cudaStream_t cs = as_stream(stream);
  // order the solver's private stream after the caller's stream, and the caller's after the solve
  cudaEvent_t ev;
  FB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  FB_CUDA(cudaEventRecord(ev, cs));
  FB_CUDA(cudaStreamWaitEvent(s->stream, ev, 0));
  FB_TRY(to_device_order(s, s->rhs, rhs));
  FB_TRY(to_device_order(s, s->x, sol));
  fb_status e = solve_common(s, info);
  if(e == FB_OK)
    e = from_device_order(s, sol, s->x);
  FB_CUDA(cudaEventRecord(ev, s->stream));
  FB_CUDA(cudaStreamWaitEvent(cs, ev, 0));
  FB_CUDA(cudaStreamSynchronize(s->stream));
  cudaEventDestroy(ev);
  return e;
}

fb_status fb_solver_vcycle(fb_solver* s, double* cor, const double* def)
{
  if(!s || !cor || !def)
  {
    set_error("solver_vcycle: bad arguments");
    return FB_ERR_ARG;
  }
  const uint32_t n = s->lv[0].n;
  FB_CUDA(cudaMemcpyAsync(s->tmp_in, def, 8 * size_t(n), cudaMemcpyHostToDevice, s->stream));
  FB_TRY(to_device_order(s, s->r, s->tmp_in));
  fb_status e = FB_OK;
  if(s->cfg.precision == FB_PREC_F64)
    e = vcycle_dispatch<double, double>(s);
  else if(s->cfg.precision == FB_PREC_F32)
    e = vcycle_dispatch<float, float>(s);
  else
    e = vcycle_dispatch<bf16_t, float>(s);
  if(e != FB_OK)
    return e;
  // the top level's solution: the buffer the last post-smoothing step wrote (x or x2 by parity)
  const DevLevel& t = s->lv[0];
  const int steps = std::max(1, s->cfg.smooth_steps);
  void* xtop = s->vc_top ? s->vc_top : (((steps - 1) % 2 == 0) ? t.x : t.x2);
  if(s->cfg.precision == FB_PREC_F64)
    FB_TRY(from_device_order(s, s->tmp_out, (const double*)xtop));
  else
  {
    fb_status ce = fb_convert_f32_to_f64(s->tmp_in, (const float*)xtop, n, s->stream);
    if(ce != FB_OK)
      return ce;
    FB_TRY(from_device_order(s, s->tmp_out, s->tmp_in));
  }
  FB_CUDA(cudaMemcpyAsync(cor, s->tmp_out, 8 * size_t(n), cudaMemcpyDeviceToHost, s->stream));
  FB_CUDA(cudaStreamSynchronize(s->stream));
  return FB_OK;
}

} // extern "C"

namespace fb
{
  // reads n16 16-byte words (L2 fills with clean lines); the sink is written only on a value the
  // data never has, so the loads stay
  __global__ void k_read_sweep(const uint4* __restrict__ p, size_t n16, unsigned int* sink)
  {
    uint32_t acc = 0;
    for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n16; i += size_t(gridDim.x) * blockDim.x)
    {
      const uint4 v = p[i];
      acc ^= v.x ^ v.y ^ v.z ^ v.w;
    }
    if(acc == 0x9e3779b9u)
      atomicAdd(sink, 1u);
  }

  template<typename V, typename S>
  static void time_one(fb_solver* s, int which, cudaStream_t st)
  {
    Launcher<V, S> l{s, st, false};
    const DevLevel& t = s->lv[0];
    const DevMat& A64 = s->cfg.precision == FB_PREC_F64 ? t.A : t.A64;
    if(which == FB_KERNEL_MG_TAIL)
    {
      std::vector<void*> xcur(static_cast<size_t>(s->nlev), nullptr);
      l.tail(s->ctail_first >= 0 ? s->ctail_first : s->tail_first, 0, 0, 0, xcur);
    }
    else if(which == FB_KERNEL_MG_CYCLE)
      l.vcycle(false);
    else if(which == FB_KERNEL_PCG_SPMV)
    {
      if(l.use_tma_f64(A64))
        l.template tma<double, double>(A64, s->p, OpPcgQ{s->p, s->q, t.dm, s->sc});
      else
        k_pcg_q<<<blocks(t.n), NT, A64.smem, st>>>(view<double>(A64), s->p, s->q, t.dm, s->slot, s->sc);
    }
    else if(which == FB_KERNEL_MG_DEFECT)
    {
      if(l.use_tma(t.A))
        l.template tma<V, S>(t.A, t.x, OpDefect<V, S>{(const S*)t.b, (S*)t.d, t.dm, s->sc});
      else
        k_defect<V, S><<<blocks(t.n), NT, t.A.smem, st>>>(view<V>(t.A), (const S*)t.b, (const S*)t.x, (S*)t.d, t.dm,
          s->sc);
    }
    else if(which == FB_KERNEL_MG_SMOOTH)
    {
      if(l.use_tma(t.A))
        l.template tma<V, S>(t.A, t.x, OpSmooth<V, S>{(const S*)t.b, (const S*)t.x, (S*)t.x2, (const S*)t.dinv, t.dm,
          t.skip_pre, s->sc});
      else
        k_smooth<V, S><<<blocks(t.n), NT, t.A.smem, st>>>(view<V>(t.A), (const S*)t.b, (const S*)t.x, (S*)t.x2,
          (const S*)t.dinv, t.dm, t.skip_pre, s->sc);
    }
    else if(which == FB_KERNEL_MG_POST1)
    {
      if(l.use_tma(t.A))
        l.template tma<V, S>(t.A, t.x, OpPost1<V, S>{(const S*)t.b, (S*)t.d, (S*)t.c, (const S*)t.dinv, t.dm,
          t.skip_post, s->sc});
      else
        k_post1<V, S><<<blocks(t.n), NT, t.A.smem, st>>>(view<V>(t.A), (const S*)t.b, (const S*)t.x, (S*)t.d, (S*)t.c,
          (const S*)t.dinv, t.dm, t.skip_post, s->slot, s->sc);
    }
    else if(which == FB_KERNEL_MG_POST2)
    {
      // the finest level's last post-smoothing step as the solve runs it: it also forms z and r.z
      if(l.use_tma(t.A))
        l.template tma<V, S>(t.A, t.c, OpPost2<V, S, true, true>{(const S*)t.d, (const S*)t.c, (S*)t.c2, (S*)t.x, s->z,
          s->r, (const S*)t.dinv, t.dm, t.skip_post, s->sc});
      else
        k_post2<V, S, true, true><<<blocks(t.n), NT, t.A.smem, st>>>(view<V>(t.A), (const S*)t.d, (const S*)t.c,
          (S*)t.c2, (S*)t.x, s->z, s->r, (const S*)t.dinv, t.dm, t.skip_post, s->slot, s->sc);
    }
    else if(which == FB_KERNEL_MG_DOWN)
    {
      std::vector<void*> xcur(static_cast<size_t>(s->nlev), nullptr);
      l.fused_down(0, xcur);
    }
    else if(which == FB_KERNEL_MG_UP)
    {
      // the finest level's pass as the solve runs it: it also forms z and r.z
      std::vector<void*> xcur(static_cast<size_t>(s->nlev), nullptr);
      xcur[0] = t.x2;
      xcur[1] = s->lv[1].x2;
      l.fused_up(0, true, xcur);
    }
    else if(which == FB_KERNEL_MG_SDOWN)
    {
      std::vector<void*> xcur(static_cast<size_t>(s->nlev), nullptr);
      l.streamed_down(0, xcur);
    }
    else if(which == FB_KERNEL_MG_SUP)
    {
      std::vector<void*> xcur(static_cast<size_t>(s->nlev), nullptr);
      xcur[0] = t.x2;
      xcur[1] = s->lv[1].x2;
      l.streamed_up(0, true, xcur);
    }
    else if(which == FB_KERNEL_MG_RESTRICT)
      l.restrict_to(0);
    else if(which == FB_KERNEL_MG_PROLONG)
    {
      std::vector<void*> xcur(static_cast<size_t>(s->nlev), nullptr);
      xcur[0] = t.x;
      xcur[1] = s->lv[1].x;
      l.prolong(0, xcur);
    }
  }

  // algorithmic bytes of one launch of kernel `which` as stored on the device: the matrix as stored,
  // the gathered vector, the row-wise vectors read and written and the Dirichlet mask (the same
  // count the solve's bytes_moved uses); 0 for the multi-pass entries
  template<typename V, typename S>
  static double stored_bytes_one(const fb_solver* s, int which)
  {
    const DevLevel& t = s->lv[0];
    const double n = double(t.n), sx = double(sizeof(S));
    auto csr = [&](const DevMat& m, double vin, double vout)
    {
      return m.bytes + double(m.cols) * sx + double(m.rows) * sx * (vin + vout);
    };
    switch(which)
    {
      case FB_KERNEL_PCG_SPMV:
      {
        const DevMat& A64 = s->cfg.precision == FB_PREC_F64 ? t.A : t.A64;
        return A64.bytes + n * 8.0 * 2.0 + n;
      }
      case FB_KERNEL_MG_DEFECT: return csr(t.A, 1, 1) + n;
      case FB_KERNEL_MG_SMOOTH: return csr(t.A, 3, 1) + n;
      case FB_KERNEL_MG_POST1: return csr(t.A, 2, 2) + n;
      case FB_KERNEL_MG_POST2: return csr(t.A, 3, 1) + n + 16.0 * n;
      case FB_KERNEL_MG_RESTRICT:
      {
        const bool coarsest = s->nlev == 2;
        const double nc = double(s->lv[1].n);
        return t.R.bytes + double(t.R.cols) * sx + nc * sx * (coarsest ? 1.0 : 3.0) + nc;
      }
      case FB_KERNEL_MG_PROLONG: return csr(t.P, 1, 1) + n;
      case FB_KERNEL_MG_DOWN:
      case FB_KERNEL_MG_SDOWN:
      {
        const bool coarsest = s->nlev == 2;
        return t.A.bytes + t.R.bytes + n * (4.0 * sx + 1.0) + double(s->lv[1].n) * ((coarsest ? 1.0 : 3.0) * sx + 1.0);
      }
      case FB_KERNEL_MG_UP:
      case FB_KERNEL_MG_SUP: return t.A.bytes + t.P.bytes + double(t.P.cols) * sx + n * (4.0 * sx + 1.0) + 16.0 * n;
      default: return 0.0;
    }
  }
} // namespace fb

extern "C" {

fb_status fb_solver_time_kernel(fb_solver* s, int which, int reps, int flush_l2, double* avg_ms,
  double* bytes_per_launch)
{
  if(!s || !avg_ms || !bytes_per_launch || reps < 1 || which < FB_KERNEL_PCG_SPMV || which > FB_KERNEL_MG_SUP ||
     (which == FB_KERNEL_MG_DOWN && (s->nlev < 2 || !s->lv[0].fz_down)) ||
     (which == FB_KERNEL_MG_UP && (s->nlev < 2 || !s->lv[0].fz_up)) ||
     (which == FB_KERNEL_MG_SDOWN && (s->nlev < 2 || !s->lv[0].fz_down || !s->lv[0].fs_ok)) ||
     (which == FB_KERNEL_MG_SUP && (s->nlev < 2 || !s->lv[0].fs_up || !s->lv[0].fs_ok)) ||
     (which == FB_KERNEL_MG_TAIL && s->tail_first < 0 && s->ctail_first < 0) ||
     (which >= FB_KERNEL_MG_SMOOTH && s->nlev < 2) ||
     (which >= FB_KERNEL_MG_SMOOTH && (s->tail_first == 0 || s->ctail_first == 0)))
  {
    set_error("solver_time_kernel: bad arguments");
    return FB_ERR_ARG;
  }
  cudaStream_t st = s->stream;
  const DevLevel& t = s->lv[0];
  const bool f64 = s->cfg.precision == FB_PREC_F64;
  // flush: overwrite one 256 MiB half, then read the other (zeroed once) so that the L2 holds clean
  // lines of neither the matrix nor the vectors when the timed launch starts (a write-only flush
  // would leave dirty lines whose write-back lands inside the timed interval)
  const size_t flush_bytes = size_t(256) << 20;
  if(flush_l2 && !s->flush)
  {
    FB_TRY(dalloc(s, &s->flush, 2 * flush_bytes + 256));
    FB_CUDA(cudaMemsetAsync(s->flush, 0, 2 * flush_bytes + 256, st));
  }
  (void)t;
  (void)f64;
  if(s->cfg.precision == FB_PREC_F64)
    *bytes_per_launch = stored_bytes_one<double, double>(s, which);
  else if(s->cfg.precision == FB_PREC_F32)
    *bytes_per_launch = stored_bytes_one<float, float>(s, which);
  else
    *bytes_per_launch = stored_bytes_one<bf16_t, float>(s, which);
  k_set_status<<<1, 1, 0, st>>>(s->sc, FB_SOLVER_PROGRESS);
  FB_LAUNCHED(1);
  double total = 0.0;
  for(int k = 0; k < reps; ++k)
  {
    if(flush_l2)
    {
      unsigned char* f = static_cast<unsigned char*>(s->flush);
      FB_CUDA(cudaMemsetAsync(f, (k + 1) & 0xff, flush_bytes, st));
      k_read_sweep<<<s->nsm * 4, 512, 0, st>>>(reinterpret_cast<const uint4*>(f + flush_bytes), flush_bytes / 16,
        reinterpret_cast<unsigned int*>(f + 2 * flush_bytes));
      FB_LAUNCHED(1);
    }
    FB_CUDA(cudaEventRecord(s->ev0, st));
    // the kernel the solve itself launches for this matrix: TMA-staged pass or per-row kernel
    if(s->cfg.precision == FB_PREC_F64)
      time_one<double, double>(s, which, st);
    else if(s->cfg.precision == FB_PREC_F32)
      time_one<float, float>(s, which, st);
    else
      time_one<bf16_t, float>(s, which, st);
    FB_LAUNCHED(1);
    FB_CUDA(cudaEventRecord(s->ev1, st));
    FB_CUDA(cudaEventSynchronize(s->ev1));
    float ms = 0.f;
    FB_CUDA(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    total += double(ms);
  }
  k_set_status<<<1, 1, 0, st>>>(s->sc, FB_SOLVER_SUCCESS);
  FB_LAUNCHED(1);
  FB_CUDA(cudaStreamSynchronize(st));
  *avg_ms = total / reps;
  return FB_OK;
}

fb_status fb_matrix_storage_plan(const fb_csr_host* M, const uint64_t* empty_rows, uint64_t num_empty, int rcm,
                                 int allow_diag, fb_storage_plan* out)
{
  if(!M || !out || (num_empty && !empty_rows))
  {
    set_error("matrix_storage_plan: bad arguments");
    return FB_ERR_ARG;
  }
  HostCsr A;
  const std::string e = import_csr(A, M->rows, M->columns, M->used_elements, M->row_ptr, M->col_ind, M->val, false);
  if(!e.empty())
  {
    set_error("matrix_storage_plan: " + e);
    return FB_ERR_ARG;
  }
  std::vector<uint8_t> empty(A.rows, 0);
  for(uint64_t k = 0; k < num_empty; ++k)
  {
    if(empty_rows[k] >= A.rows)
    {
      set_error("matrix_storage_plan: empty row out of range");
      return FB_ERR_ARG;
    }
    empty[size_t(empty_rows[k])] = 1;
  }
  if(rcm && A.rows == A.cols)
  {
    const std::vector<uint32_t> perm = rcm_order(A);
    const std::vector<uint32_t> inv = inverse_perm(perm);
    A = permute(A, perm, inv);
    std::vector<uint8_t> ep(A.rows);
    for(uint32_t k = 0; k < A.rows; ++k)
      ep[k] = empty[perm[k]];
    empty.swap(ep);
  }
  const HostSell H = build_sell(A, &empty, true, allow_diag != 0);
  const uint32_t ns = (H.rows + 31u) / 32u;
  uint32_t kmax = H.kw;
  for(uint32_t sl = 0; sl < ns; ++sl)
    kmax = std::max(kmax, (H.soff[sl + 1] - H.soff[sl]) / 32u);
  out->kind = !H.doff.empty() ? 2 : (H.kw ? 1 : 0);
  out->narrow = H.narrow ? 1 : 0;
  out->width = kmax;
  out->diagonals = uint32_t(H.doff.size());
  out->entries = H.entries;
  return FB_OK;
}

fb_status fb_multigrid_cycle_events(int cycle, int adapt_cgc, int num_levels, uint8_t* ops, uint8_t* levels,
                                    uint64_t capacity, uint64_t* count)
{
  if(!count || num_levels < 2 || num_levels > 24 || cycle < FB_CYCLE_V || cycle > FB_CYCLE_W ||
     adapt_cgc < FB_CGC_FIXED || adapt_cgc > FB_CGC_MIN_DEFECT || (capacity && (!ops || !levels)))
  {
    set_error("multigrid_cycle_events: bad arguments");
    return FB_ERR_ARG;
  }
  const std::vector<CycEv> ev = cycle_events(cycle, num_levels, adapt_cgc != FB_CGC_FIXED);
  for(uint64_t i = 0; i < ev.size() && i < capacity; ++i)
  {
    ops[i] = ev[i].op;
    levels[i] = ev[i].lvl;
  }
  *count = ev.size();
  return FB_OK;
}

fb_status fb_solver_level_info(const fb_solver* s, uint64_t* out)
{
  if(!s || !out)
  {
    set_error("solver_level_info: bad arguments");
    return FB_ERR_ARG;
  }
  for(int l = 0; l < s->nlev; ++l)
  {
    out[3 * l + 0] = s->lv[size_t(l)].n;
    out[3 * l + 1] = s->lv[size_t(l)].A.nnz;
    out[3 * l + 2] = s->lv[size_t(l)].P.nnz;
  }
  return FB_OK;
}

} // extern "C"

namespace fb
{
  template<typename V> __device__ __forceinline__ V from_f64(double v);
  template<> __device__ __forceinline__ double from_f64<double>(double v) { return v; }
  template<> __device__ __forceinline__ float from_f64<float>(double v) { return __double2float_rn(v); }
  template<> __device__ __forceinline__ bf16_t from_f64<bf16_t>(double v)
  {
    // FP64 -> FP32 (nearest) -> BF16 (nearest even), as the host upload rounds
    const float f = __double2float_rn(v);
    uint32_t u = __float_as_uint(f);
    bf16_t b;
    if((u & 0x7f800000u) == 0x7f800000u)
      b.bits = uint16_t(u >> 16) | ((u & 0xffffu) ? 0x40u : 0u);
    else
      b.bits = uint16_t((u + 0x7fffu + ((u >> 16) & 1u)) >> 16);
    return b;
  }

  template<typename V>
  __global__ void k_scatter_values(const double* __restrict__ vals, const uint32_t* __restrict__ slot, uint64_t nnz,
    V* __restrict__ dst)
  {
    const uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if(j >= nnz)
      return;
    const uint32_t e = slot[j];
    if(e != 0xffffffffu)
      dst[e] = from_f64<V>(vals[j]);
  }

  // inv_diag = omega / a_ii in FP64, stored in the V-cycle's precision (inv_diagonal + upload_vec)
  template<typename S>
  __global__ void k_update_dinv(const double* __restrict__ vals, const uint32_t* __restrict__ diag, uint32_t n,
    double omega, S* __restrict__ dinv)
  {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if(k >= n)
      return;
    const uint32_t j = diag[k];
    const double a = j == 0xffffffffu ? 0.0 : vals[j];
    dinv[k] = S(omega / a);
  }

  // slot and diagonal maps of level l (see fb_solver::upd_slot)
  static fb_status build_update_maps(fb_solver* s, int l)
  {
    const HostLevel& H = s->h->levels[size_t(l)];
    const std::vector<uint32_t>& pf = s->perms[size_t(l)];
    const std::vector<uint32_t> inv = pf.empty() ? std::vector<uint32_t>() : inverse_perm(pf);
    const HostCsr& A = H.A;
    std::vector<uint8_t> dm(A.rows);
    for(uint32_t k = 0; k < A.rows; ++k)
      dm[k] = H.dmask[pf.empty() ? k : pf[k]];
    const HostSell S = build_sell(permute(A, pf, inv), &dm, true, s->cfg.diagonal != 0);
    std::vector<uint32_t> slot(std::max<size_t>(1, A.col.size()), 0xffffffffu);
    std::vector<uint32_t> diag(std::max<uint32_t>(1, A.rows), 0xffffffffu);
    for(uint32_t r = 0; r < A.rows; ++r)
    {
      const uint32_t k = inv.empty() ? r : inv[r];
      for(uint32_t j = A.rp[r]; j < A.rp[r + 1]; ++j)
      {
        if(A.col[j] == r && diag[k] == 0xffffffffu)
          diag[k] = j;
        if(!dm[k])
          slot[j] = uint32_t(S.slot(k, j - A.rp[r], inv.empty() ? A.col[j] : inv[A.col[j]]));
      }
    }
    uint32_t* ds = nullptr;
    uint32_t* dd = nullptr;
    FB_TRY(dalloc(s, (void**)&ds, sizeof(uint32_t) * slot.size()));
    FB_TRY(dalloc(s, (void**)&dd, sizeof(uint32_t) * diag.size()));
    FB_CUDA(cudaMemcpy(ds, slot.data(), sizeof(uint32_t) * slot.size(), cudaMemcpyHostToDevice));
    FB_CUDA(cudaMemcpy(dd, diag.data(), sizeof(uint32_t) * diag.size(), cudaMemcpyHostToDevice));
    s->upd_slot[size_t(l)] = ds;
    s->upd_diag[size_t(l)] = dd;
    return FB_OK;
  }

  template<typename V, typename S>
  static fb_status update_level(fb_solver* s, int l, const double* vals, cudaStream_t st)
  {
    DevLevel& D = s->lv[size_t(l)];
    const uint64_t nnz = s->h->levels[size_t(l)].A.col.size();
    const uint32_t* slot = s->upd_slot[size_t(l)];
    if(nnz)
    {
      const unsigned g = unsigned((nnz + 255) / 256);
      k_scatter_values<V><<<g, 256, 0, st>>>(vals, slot, nnz, static_cast<V*>(D.A.val));
      if(D.A64.val)
        k_scatter_values<double><<<g, 256, 0, st>>>(vals, slot, nnz, static_cast<double*>(D.A64.val));
    }
    k_update_dinv<S><<<(D.n + 255) / 256, 256, 0, st>>>(vals, s->upd_diag[size_t(l)], D.n, s->cfg.omega,
      static_cast<S*>(D.dinv));
    FB_LAUNCHED(nnz ? (D.A64.val ? 3 : 2) : 1);
    return FB_OK;
  }
} // namespace fb

extern "C" {

fb_status fb_solver_set_tolerances(fb_solver* s, double tol_rel, double tol_abs)
{
  if(!s || !(tol_rel >= 0.0) || !(tol_abs >= 0.0))
  {
    set_error("solver_set_tolerances: bad arguments");
    return FB_ERR_ARG;
  }
  FB_CUDA(cudaStreamSynchronize(s->stream));
  s->cfg.tol_rel = tol_rel;
  s->cfg.tol_abs = tol_abs;
  const double t[2] = {tol_rel, tol_abs};
  static_assert(offsetof(Scalars, tol_abs) == offsetof(Scalars, tol_rel) + sizeof(double), "Scalars layout");
  FB_CUDA(cudaMemcpy(reinterpret_cast<char*>(s->sc) + offsetof(Scalars, tol_rel), t, sizeof(t),
                     cudaMemcpyHostToDevice));
  return FB_OK;
}

fb_status fb_solver_set_iteration_limits(fb_solver* s, int min_iter, int max_iter)
{
  if(!s || min_iter < 0 || max_iter < 0 || max_iter > s->max_iter_cap)
  {
    set_error("solver_set_iteration_limits: bad arguments (max_iter may not exceed the value the solver was created with)");
    return FB_ERR_ARG;
  }
  FB_CUDA(cudaStreamSynchronize(s->stream));
  s->cfg.min_iter = min_iter;
  s->cfg.max_iter = max_iter;
  const int t[2] = {min_iter, max_iter};
  static_assert(offsetof(Scalars, max_iter) == offsetof(Scalars, min_iter) + sizeof(int), "Scalars layout");
  FB_CUDA(cudaMemcpy(reinterpret_cast<char*>(s->sc) + offsetof(Scalars, min_iter), t, sizeof(t),
                     cudaMemcpyHostToDevice));
  return FB_OK;
}

fb_status fb_solver_update_matrix(fb_solver* s, int level, const double* values, void* stream)
{
  if(!s || level < 0 || level >= s->nlev || (!values && !s->h->levels[size_t(level)].A.col.empty()))
  {
    set_error("solver_update_matrix: bad arguments");
    return FB_ERR_ARG;
  }
  if(s->upd_slot.empty())
  {
    s->upd_slot.assign(size_t(s->nlev), nullptr);
    s->upd_diag.assign(size_t(s->nlev), nullptr);
  }
  if(!s->upd_slot[size_t(level)])
    FB_TRY(build_update_maps(s, level));
  cudaStream_t st = as_stream(stream);
  fb_status e;
  if(s->cfg.precision == FB_PREC_F64)
    e = update_level<double, double>(s, level, values, st);
  else if(s->cfg.precision == FB_PREC_F32)
    e = update_level<float, float>(s, level, values, st);
  else
    e = update_level<bf16_t, float>(s, level, values, st);
  if(e != FB_OK)
    return e;
  if(level == s->nlev - 1)
  {
    // the exact coarse inverse from the new values (host Gauss-Jordan, as at creation)
    HostCsr A = s->h->levels[size_t(level)].A;
    if(!A.val.empty())
      FB_CUDA(cudaMemcpyAsync(A.val.data(), values, sizeof(double) * A.val.size(), cudaMemcpyDeviceToHost, st));
    FB_CUDA(cudaStreamSynchronize(st));
    std::vector<uint32_t> fr;
    std::vector<double> inv;
    coarse_inverse(A, s->h->levels[size_t(level)].dmask, fr, inv);
    if(!inv.empty())
      FB_CUDA(cudaMemcpy(s->cinv, inv.data(), sizeof(double) * inv.size(), cudaMemcpyHostToDevice));
  }
  else
    FB_CUDA(cudaStreamSynchronize(st));
  return FB_OK;
}

} // extern "C"
