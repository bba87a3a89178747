// Multi-right-hand-side solver: K = 32 or 64 independent right-hand sides of one multigrid
// hierarchy solved together, each by its own PCG + V-cycle with its own scalars, stopping test and
// smoother skip flags, so every right-hand side follows exactly the single-RHS algorithm
// (kernel/solver/pcg.hpp:188-286, kernel/solver/multigrid.hpp:1270-2000).
//
// Vectors are stored RHS-interleaved, x[row * K + j], the element layout of the reference's
// DenseVectorBlocked<DT, IT, K>.  One warp processes one matrix row for all K right-hand sides
// (K/32 per lane): the row's entries are read once, coalesced, and broadcast by shuffles, and every
// gather of x[col][0..K) is one coalesced K*sizeof(S) access -- the matrix traffic is shared by all
// right-hand sides (the reference's multi-vector CSR kernel, apply.cu:109-135, covers K <= 3).
// With the configuration's `diagonal` set, system matrices of lexicographically numbered Q1 grids
// run in a stencil form instead: values by diagonal, one warp per strip of consecutive rows, each x
// row gathered once for all the strip's rows it enters (strip_rows).  Rows are summed in stored entry order without FMA, per right-hand
// side, as in the single-RHS kernels, in both forms.  Dot products and norms are reduced per block and then with FP64 atomics (their
// summation order is not fixed; results agree with the single-RHS path to rounding).
#include "fb_common.cuh"
#include "fb_setup.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <type_traits>
#include <vector>

namespace fb
{
namespace mr
{
  constexpr int MNT = 256;               // threads per block
  constexpr int MW = MNT / 32;            // warps (rows in flight) per block
  constexpr int KMAX = 64;

  // A matrix in CSR form and, for a system matrix whose stored rows all share one pattern of 9 or
  // 27 column offsets made of triplets (o-1, o, o+1) -- the Q1 stencil of a lexicographically
  // numbered grid -- also in stencil form: dval[k * dn + row] is entry k of the row (zeros for rows
  // stored empty and for the padding up to dn, a multiple of 8), goff[g] the centre offset of
  // triplet g.  nd = 0: CSR only.
  template<typename V>
  struct MCsr
  {
    const uint32_t* rp;
    const uint32_t* col;
    const V* val;
    uint32_t rows;
    const V* dval;
    uint32_t dn;
    int nd;
    int goff[9];
  };

  // rows per warp in the stencil form: the strip's rows share their x gathers (M + 2 row loads per
  // triplet for M rows instead of 3 M); 4 for FP64 values to bound the registers
  template<typename V> struct StripRows { static constexpr int value = sizeof(V) == 8 ? 4 : 8; };

  struct MScal
  {
    double gamma[KMAX], gamma_prev[KMAX], alpha[KMAX], beta[KMAX];
    double def_init[KMAX], def_cur[KMAX], scale[KMAX], inv_scale[KMAX];
    double acc[KMAX];                     // reduction accumulators, zero between passes
    int iter[KMAX], status[KMAX];
    int progress;                         // right-hand sides still in progress
    unsigned int arrive;
    double tol_rel, tol_abs, div_rel, div_abs;
    int min_iter, max_iter;
  };

  __device__ __forceinline__ double shfl_v(double v, int k) { return __shfl_sync(0xffffffffu, v, k); }
  __device__ __forceinline__ float shfl_v(float v, int k) { return __shfl_sync(0xffffffffu, v, k); }
  __device__ __forceinline__ bf16_t shfl_v(bf16_t v, int k)
  {
    bf16_t b;
    b.bits = uint16_t(__shfl_sync(0xffffffffu, uint32_t(v.bits), k));
    return b;
  }
  __device__ __forceinline__ double ldg_m(const double* p) { return __ldg(p); }
  __device__ __forceinline__ float ldg_m(const float* p) { return __ldg(p); }

  __device__ __forceinline__ bool closed(const MScal* sc) { return sc->progress <= 0; }

  // a lane's R consecutive vector entries, in one load where the width allows (8- or 16-byte aligned:
  // the row stride is 32 R entries and the lane offset R entries)
  template<typename S, int R>
  __device__ __forceinline__ void ldg_row(const S* p, S (&v)[R])
  {
    if(R == 2 && sizeof(S) == 4)
    {
      const float2 t = __ldg(reinterpret_cast<const float2*>(p));
      v[0] = S(t.x);
      v[R - 1] = S(t.y);
    }
    else if(R == 2 && sizeof(S) == 8)
    {
      const double2 t = __ldg(reinterpret_cast<const double2*>(p));
      v[0] = S(t.x);
      v[R - 1] = S(t.y);
    }
    else
    {
      #pragma unroll
      for(int r = 0; r < R; ++r)
        v[r] = __ldg(p + r);
    }
  }

  template<typename S> __device__ __forceinline__ double epsq();
  template<> __device__ __forceinline__ double epsq<double>() { return EPS64 * EPS64; }
  template<> __device__ __forceinline__ double epsq<float>() { return double(EPS32) * double(EPS32); }
  template<typename S> __device__ __forceinline__ int skip_of(double nrm)
  {
    return (!isfinite(nrm) || nrm <= epsq<S>()) ? 1 : 0;
  }

  // sum[r] = (A x)[row][lane*R + r], entries in stored order
  template<typename V, typename S, int R>
  __device__ __forceinline__ void mrow(const MCsr<V>& M, uint32_t row, const S* __restrict__ x,
    typename ValueTraits<V>::acc (&sum)[R])
  {
    typedef typename ValueTraits<V>::acc A;
    const int lane = threadIdx.x & 31;
    #pragma unroll
    for(int r = 0; r < R; ++r)
      sum[r] = A(0);
    const uint32_t j0 = __ldg(M.rp + row), j1 = __ldg(M.rp + row + 1);
    for(uint32_t base = j0; base < j1; base += 32)
    {
      const uint32_t cnt = min(32u, j1 - base);
      V v{};
      uint32_t c = 0;
      if(uint32_t(lane) < cnt)
      {
        v = ldg_m(M.val + base + lane);
        c = __ldg(M.col + base + lane);
      }
      // 9 entries per step (the 2D and 3D Q1 rows are 9 and 27 long): their gathers go out together
      #pragma unroll 9
      for(uint32_t k = 0; k < cnt; ++k)
      {
        const A vk = A(shfl_v(v, int(k)));
        const uint32_t ck = __shfl_sync(0xffffffffu, c, int(k));
        const S* xr = x + size_t(ck) * (32 * R) + lane * R;
        S xv[R];
        ldg_row<S, R>(xr, xv);
        #pragma unroll
        for(int r = 0; r < R; ++r)
          sum[r] = add(sum[r], mul(vk, A(xv[r])));
      }
    }
  }

  // the strip's M values of one diagonal (uniform loads: every lane reads the same 16 bytes)
  template<int M>
  __device__ __forceinline__ void ldg_diag(const float* p, float (&v)[M])
  {
    #pragma unroll
    for(int i = 0; i < M; i += 4)
    {
      const float4 t = __ldg(reinterpret_cast<const float4*>(p + i));
      v[i] = t.x;
      v[i + 1] = t.y;
      v[i + 2] = t.z;
      v[i + 3] = t.w;
    }
  }
  template<int M>
  __device__ __forceinline__ void ldg_diag(const double* p, double (&v)[M])
  {
    #pragma unroll
    for(int i = 0; i < M; i += 2)
    {
      const double2 t = __ldg(reinterpret_cast<const double2*>(p + i));
      v[i] = t.x;
      v[i + 1] = t.y;
    }
  }

  // Stencil form, G triplets per row: one warp takes M consecutive rows r0..r0+M-1.  For triplet g
  // the rows need the x rows r0-1+goff[g] .. r0+M+goff[g]; each is loaded once and added to the (up
  // to three) rows whose entry it is.  Row m receives its entries in ascending column order
  // (triplets in order, then o-1, o, o+1), which is the stored CSR order, so every row sum equals
  // mrow's bit for bit.  x rows outside [0, rows) are read only by rows stored empty (their values
  // are zero); they are not loaded.  epi(row, sum) runs for every row < rows.
  template<typename V, typename S, int R, int G, class Epi>
  __device__ __forceinline__ void strip_rows(const MCsr<V>& A, const S* __restrict__ x, Epi& epi)
  {
    typedef typename ValueTraits<V>::acc Ac;
    constexpr int M = StripRows<V>::value;
    constexpr int K = 32 * R;
    const int lane = threadIdx.x & 31;
    const uint32_t n = A.rows;
    const uint32_t nstrips = (n + M - 1) / M;
    for(uint32_t st = blockIdx.x * MW + (threadIdx.x >> 5); st < nstrips; st += gridDim.x * MW)
    {
      const uint32_t r0 = st * M;
      Ac sum[M][R];
      #pragma unroll
      for(int m = 0; m < M; ++m)
        #pragma unroll
        for(int r = 0; r < R; ++r)
          sum[m][r] = Ac(0);
      #pragma unroll
      for(int g = 0; g < G; ++g)
      {
        V v[3][M];
        #pragma unroll
        for(int dx = 0; dx < 3; ++dx)
          ldg_diag<M>(A.dval + size_t(3 * g + dx) * A.dn + r0, v[dx]);
        const int64_t base = int64_t(r0) - 1 + A.goff[g];
        #pragma unroll
        for(int t = 0; t < M + 2; ++t)
        {
          const int64_t xr = base + t;
          S xv[R];
          if(xr >= 0 && xr < int64_t(n))
            ldg_row<S, R>(x + size_t(xr) * K + lane * R, xv);
          else
          {
            #pragma unroll
            for(int r = 0; r < R; ++r)
              xv[r] = S(0);
          }
          #pragma unroll
          for(int m = t - 2; m <= t; ++m)
          {
            if(m < 0 || m >= M)
              continue;
            const Ac vk = Ac(v[t - m][m]);
            #pragma unroll
            for(int r = 0; r < R; ++r)
              sum[m][r] = add(sum[m][r], mul(vk, Ac(xv[r])));
          }
        }
      }
      #pragma unroll
      for(int m = 0; m < M; ++m)
        if(r0 + uint32_t(m) < n)
          epi(r0 + uint32_t(m), sum[m]);
    }
  }

  // epi(row, sum) for every row of A with sum = (A x)[row]: in the stencil form with G = 9 or 3
  // triplets per row, in the CSR form for G = 0.  The form is a template parameter of every matrix
  // pass, so the CSR instances keep the registers (and the resident warps) of the row kernel.
  template<typename V, typename S, int R, int G, class Epi>
  __device__ __forceinline__ void for_rows(const MCsr<V>& A, const S* __restrict__ x, Epi epi)
  {
    typedef typename ValueTraits<V>::acc Ac;
    if constexpr(G > 0)
      strip_rows<V, S, R, G>(A, x, epi);
    else
      for(uint32_t row = blockIdx.x * MW + (threadIdx.x >> 5); row < A.rows; row += gridDim.x * MW)
      {
        Ac sum[R];
        mrow<V, S, R>(A, row, x, sum);
        epi(row, sum);
      }
  }

  // block partials per right-hand side (smem), atomically added to sc->acc; the last block calls
  // fin(j, total) for every j < K and clears the accumulators.  Returns true in the last block.
  template<int R, class Fin>
  __device__ __forceinline__ void reduce_per_rhs(const double (&part)[R], MScal* sc, Fin fin)
  {
    constexpr int K = 32 * R;
    __shared__ double red[MW][K];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    #pragma unroll
    for(int r = 0; r < R; ++r)
      red[warp][lane * R + r] = part[r];
    __syncthreads();
    if(threadIdx.x < K)
    {
      double s = 0.0;
      #pragma unroll
      for(int w = 0; w < MW; ++w)
        s += red[w][threadIdx.x];
      atomicAdd(&sc->acc[threadIdx.x], s);
    }
    __threadfence();
    __syncthreads();
    if(threadIdx.x == 0)
      last = (atomicAdd(&sc->arrive, 1u) == gridDim.x - 1);
    __syncthreads();
    if(!last)
      return;
    __threadfence();
    if(threadIdx.x < K)
    {
      const double tot = atomicAdd(&sc->acc[threadIdx.x], 0.0);
      sc->acc[threadIdx.x] = 0.0;
      fin(int(threadIdx.x), tot);
    }
    if(threadIdx.x == 0)
      sc->arrive = 0u;
  }

#define MR_ROWS(n) \
  for(uint32_t row = blockIdx.x * MW + (threadIdx.x >> 5); row < (n); row += gridDim.x * MW)

  template<typename V, typename S, int R, int G>
  __global__ void __launch_bounds__(MNT) km_smooth(MCsr<V> A, const S* __restrict__ b, const S* __restrict__ x,
    S* __restrict__ xo, const S* __restrict__ dinv, const uint8_t* __restrict__ dm, const int* __restrict__ skip,
    const MScal* __restrict__ sc)
  {
    typedef typename ValueTraits<V>::acc Ac;
    constexpr int K = 32 * R;
    if(closed(sc))
      return;
    const int lane = threadIdx.x & 31;
    for_rows<V, S, R, G>(A, x, [&](uint32_t row, const Ac (&sum)[R])
    {
      const bool d = __ldg(dm + row) != 0;
      const Ac di = Ac(__ldg(dinv + row));
      #pragma unroll
      for(int r = 0; r < R; ++r)
      {
        const size_t e = size_t(row) * K + lane * R + r;
        S out = S(0);
        if(!skip[lane * R + r])
        {
          const Ac d1 = d ? Ac(0) : sub(Ac(b[e]), sum[r]);
          const Ac c = d ? Ac(0) : mul(di, d1);
          out = S(add(Ac(x[e]), c));
        }
        xo[e] = out;
      }
    });
  }

  template<typename V, typename S, int R, int G>
  __global__ void __launch_bounds__(MNT) km_defect(MCsr<V> A, const S* __restrict__ b, const S* __restrict__ x,
    S* __restrict__ dv, const uint8_t* __restrict__ dm, const MScal* __restrict__ sc)
  {
    typedef typename ValueTraits<V>::acc Ac;
    constexpr int K = 32 * R;
    if(closed(sc))
      return;
    const int lane = threadIdx.x & 31;
    for_rows<V, S, R, G>(A, x, [&](uint32_t row, const Ac (&sum)[R])
    {
      const bool d = __ldg(dm + row) != 0;
      #pragma unroll
      for(int r = 0; r < R; ++r)
      {
        const size_t e = size_t(row) * K + lane * R + r;
        dv[e] = d ? S(0) : S(sub(Ac(b[e]), sum[r]));
      }
    });
  }

  template<typename V, typename S, int R>
  __global__ void __launch_bounds__(MNT) km_restrict(MCsr<V> Rm, const S* __restrict__ dv, S* __restrict__ bc,
    S* __restrict__ xc, const S* __restrict__ dinvc, const uint8_t* __restrict__ dmc, int* __restrict__ skipc,
    MScal* __restrict__ sc)
  {
    typedef typename ValueTraits<V>::acc Ac;
    constexpr int K = 32 * R;
    if(closed(sc))
      return;
    const int lane = threadIdx.x & 31;
    double part[R];
    #pragma unroll
    for(int r = 0; r < R; ++r)
      part[r] = 0.0;
    MR_ROWS(Rm.rows)
    {
      Ac sum[R];
      mrow<V, S, R>(Rm, row, dv, sum);
      const bool d = __ldg(dmc + row) != 0;
      #pragma unroll
      for(int r = 0; r < R; ++r)
      {
        const size_t e = size_t(row) * K + lane * R + r;
        const Ac v = d ? Ac(0) : add(sum[r], Ac(0));
        bc[e] = S(v);
        if(xc)
        {
          const Ac c = d ? Ac(0) : mul(Ac(__ldg(dinvc + row)), v);
          xc[e] = S(add(Ac(0), c));
        }
        part[r] += double(v) * double(v);
      }
    }
    if(!xc)
      return;
    reduce_per_rhs<R>(part, sc, [&](int j, double tot) { skipc[j] = skip_of<S>(sqrt(tot)); });
  }

  template<typename S, int R>
  __global__ void __launch_bounds__(1024) km_coarse(const S* __restrict__ b, S* __restrict__ x, uint32_t n,
    const uint32_t* __restrict__ free_dofs, const double* __restrict__ inv, uint32_t m, const MScal* __restrict__ sc)
  {
    constexpr int K = 32 * R;
    if(closed(sc))
      return;
    for(uint32_t i = threadIdx.x; i < n * K; i += 1024)
      x[i] = S(0);
    __syncthreads();
    for(uint32_t idx = threadIdx.x; idx < m * K; idx += 1024)
    {
      const uint32_t i = idx / K, j = idx % K;
      double s = 0.0;
      for(uint32_t l = 0; l < m; ++l)
        s = add(s, mul(__ldg(inv + size_t(i) * m + l), double(b[size_t(__ldg(free_dofs + l)) * K + j])));
      x[size_t(__ldg(free_dofs + i)) * K + j] = S(s);
    }
  }

  template<typename V, typename S, int R>
  __global__ void __launch_bounds__(MNT) km_prolong(MCsr<V> P, const S* __restrict__ xc, S* __restrict__ x,
    const uint8_t* __restrict__ dm, const MScal* __restrict__ sc)
  {
    typedef typename ValueTraits<V>::acc Ac;
    constexpr int K = 32 * R;
    if(closed(sc))
      return;
    const int lane = threadIdx.x & 31;
    MR_ROWS(P.rows)
    {
      Ac sum[R];
      mrow<V, S, R>(P, row, xc, sum);
      const bool d = __ldg(dm + row) != 0;
      #pragma unroll
      for(int r = 0; r < R; ++r)
      {
        const size_t e = size_t(row) * K + lane * R + r;
        const Ac c = d ? Ac(0) : add(sum[r], Ac(0));
        x[e] = S(add(Ac(x[e]), c));
      }
    }
  }

  template<typename V, typename S, int R, int G>
  __global__ void __launch_bounds__(MNT) km_post1(MCsr<V> A, const S* __restrict__ b, const S* __restrict__ x,
    S* __restrict__ dv, S* __restrict__ cv, const S* __restrict__ dinv, const uint8_t* __restrict__ dm,
    int* __restrict__ skip, MScal* __restrict__ sc)
  {
    typedef typename ValueTraits<V>::acc Ac;
    constexpr int K = 32 * R;
    if(closed(sc))
      return;
    const int lane = threadIdx.x & 31;
    double part[R];
    #pragma unroll
    for(int r = 0; r < R; ++r)
      part[r] = 0.0;
    for_rows<V, S, R, G>(A, x, [&](uint32_t row, const Ac (&sum)[R])
    {
      const bool d = __ldg(dm + row) != 0;
      const Ac di = Ac(__ldg(dinv + row));
      #pragma unroll
      for(int r = 0; r < R; ++r)
      {
        const size_t e = size_t(row) * K + lane * R + r;
        const Ac dd = d ? Ac(0) : sub(Ac(b[e]), sum[r]);
        dv[e] = S(dd);
        const Ac c = d ? Ac(0) : mul(di, dd);
        cv[e] = S(add(Ac(0), c));
        part[r] += double(dd) * double(dd);
      }
    });
    reduce_per_rhs<R>(part, sc, [&](int j, double tot) { skip[j] = skip_of<S>(sqrt(tot)); });
  }

  template<typename V, typename S, int R, bool LAST, bool TOP, int G>
  __global__ void __launch_bounds__(MNT) km_post2(MCsr<V> A, const S* __restrict__ dv, const S* __restrict__ cv,
    S* __restrict__ co, S* __restrict__ x, double* __restrict__ z, const double* __restrict__ rr,
    const S* __restrict__ dinv, const uint8_t* __restrict__ dm, const int* __restrict__ skip, MScal* __restrict__ sc)
  {
    typedef typename ValueTraits<V>::acc Ac;
    constexpr int K = 32 * R;
    if(closed(sc))
      return;
    const int lane = threadIdx.x & 31;
    double part[R];
    #pragma unroll
    for(int r = 0; r < R; ++r)
      part[r] = 0.0;
    for_rows<V, S, R, G>(A, cv, [&](uint32_t row, const Ac (&sum)[R])
    {
      const bool d = __ldg(dm + row) != 0;
      const Ac di = Ac(__ldg(dinv + row));
      #pragma unroll
      for(int r = 0; r < R; ++r)
      {
        const int j = lane * R + r;
        const size_t e = size_t(row) * K + j;
        Ac cn = Ac(0);
        if(!skip[j])
        {
          const Ac dk = d ? Ac(0) : sub(Ac(dv[e]), sum[r]);
          const Ac ck = d ? Ac(0) : mul(di, dk);
          cn = add(Ac(cv[e]), ck);
        }
        if(!LAST)
          co[e] = S(cn);
        else
        {
          const S xn = S(add(Ac(x[e]), cn));
          if(TOP)
          {
            const double zi = mul(double(xn), sc->inv_scale[j]);
            z[e] = zi;
            part[r] += mul(rr[e], zi);
          }
          else
            x[e] = xn;
        }
      }
    });
    if(!(LAST && TOP))
      return;
    reduce_per_rhs<R>(part, sc, [&](int j, double tot)
    {
      sc->gamma_prev[j] = sc->gamma[j];
      sc->gamma[j] = tot;
      sc->beta[j] = tot / sc->gamma_prev[j];
    });
  }

  __device__ __forceinline__ double pow2_inv(double v)
  {
    if(!(v > 0.0) || !isfinite(v))
      return 1.0;
    int e;
    frexp(v, &e);
    return ldexp(1.0, -e);
  }

  // r = F(rhs - A x), norms -> def_init, status; FP64 mode: sol1 = F(D .* r)
  template<typename S, int R, int G>
  __global__ void __launch_bounds__(MNT) km_pcg_init(MCsr<double> A, const double* __restrict__ rhs,
    const double* __restrict__ x, double* __restrict__ rr, const uint8_t* __restrict__ dm, S* __restrict__ x1,
    const S* __restrict__ dinv, int* __restrict__ skip_top, MScal* __restrict__ sc)
  {
    constexpr int K = 32 * R;
    const int lane = threadIdx.x & 31;
    double part[R];
    #pragma unroll
    for(int r = 0; r < R; ++r)
      part[r] = 0.0;
    for_rows<double, double, R, G>(A, x, [&](uint32_t row, const double (&sum)[R])
    {
      const bool d = __ldg(dm + row) != 0;
      #pragma unroll
      for(int r = 0; r < R; ++r)
      {
        const size_t e = size_t(row) * K + lane * R + r;
        const double rv = d ? 0.0 : sub(rhs[e], sum[r]);
        rr[e] = rv;
        if(x1)
        {
          const S c = d ? S(0) : mul(__ldg(dinv + row), S(rv));
          x1[e] = add(S(0), c);
        }
        part[r] += mul(rv, rv);
      }
    });
    reduce_per_rhs<R>(part, sc, [&](int j, double tot)
    {
      const double d0 = sqrt(tot);
      sc->def_init[j] = d0;
      sc->def_cur[j] = d0;
      sc->iter[j] = 0;
      sc->gamma[j] = 0.0;
      sc->scale[j] = 1.0;
      sc->inv_scale[j] = 1.0;
      int st = FB_SOLVER_PROGRESS;
      if(!isfinite(d0))
        st = FB_SOLVER_ABORTED;
      else if(d0 <= EPS64 * EPS64)
        st = FB_SOLVER_SUCCESS;
      sc->status[j] = st;
      skip_top[j] = skip_of<double>(d0);
    });
  }

  // number of right-hand sides in progress, computed by a single block after a status update
  __global__ void km_count_progress(MScal* sc, int K, cudaGraphConditionalHandle cond)
  {
    __shared__ int cnt;
    if(threadIdx.x == 0)
      cnt = 0;
    __syncthreads();
    if(int(threadIdx.x) < K && sc->status[threadIdx.x] == FB_SOLVER_PROGRESS)
      atomicAdd(&cnt, 1);
    __syncthreads();
    if(threadIdx.x == 0)
    {
      sc->progress = cnt;
      if(cond)
        cudaGraphSetConditional(cond, cnt > 0 ? 1u : 0u);
    }
  }

  // FP32 modes: b = S(r * scale_j), sol1 = F(D .* b), ||b|| -> skip flags of the top level
  template<typename S, int R>
  __global__ void __launch_bounds__(MNT) km_prep(const double* __restrict__ rr, S* __restrict__ bt,
    S* __restrict__ x1, const S* __restrict__ dinv, const uint8_t* __restrict__ dm, int* __restrict__ skip_top,
    uint32_t n, MScal* __restrict__ sc)
  {
    constexpr int K = 32 * R;
    if(closed(sc))
      return;
    const int lane = threadIdx.x & 31;
    double scale[R], part[R];
    #pragma unroll
    for(int r = 0; r < R; ++r)
    {
      scale[r] = pow2_inv(sc->def_cur[lane * R + r]);
      part[r] = 0.0;
    }
    MR_ROWS(n)
    {
      const bool d = __ldg(dm + row) != 0;
      #pragma unroll
      for(int r = 0; r < R; ++r)
      {
        const size_t e = size_t(row) * K + lane * R + r;
        const S b = S(mul(rr[e], scale[r]));
        bt[e] = b;
        const S c = d ? S(0) : mul(__ldg(dinv + row), b);
        x1[e] = add(S(0), c);
        part[r] += double(b) * double(b);
      }
    }
    reduce_per_rhs<R>(part, sc, [&](int j, double tot)
    {
      const double s = pow2_inv(sc->def_cur[j]);
      sc->scale[j] = s;
      sc->inv_scale[j] = 1.0 / s;
      skip_top[j] = skip_of<S>(sqrt(tot));
    });
  }

  // q = F(A p), q.p -> alpha
  template<int R, int G>
  __global__ void __launch_bounds__(MNT) km_pcg_q(MCsr<double> A, const double* __restrict__ p, double* __restrict__ q,
    const uint8_t* __restrict__ dm, MScal* __restrict__ sc)
  {
    constexpr int K = 32 * R;
    if(closed(sc))
      return;
    const int lane = threadIdx.x & 31;
    double part[R];
    #pragma unroll
    for(int r = 0; r < R; ++r)
      part[r] = 0.0;
    for_rows<double, double, R, G>(A, p, [&](uint32_t row, const double (&sum)[R])
    {
      const bool d = __ldg(dm + row) != 0;
      #pragma unroll
      for(int r = 0; r < R; ++r)
      {
        const size_t e = size_t(row) * K + lane * R + r;
        const double qv = d ? 0.0 : add(sum[r], 0.0);
        q[e] = qv;
        part[r] += mul(qv, p[e]);
      }
    });
    reduce_per_rhs<R>(part, sc, [&](int j, double tot) { sc->alpha[j] = sc->gamma[j] / tot; });
  }

  // per right-hand side still in progress: x += alpha p, r -= alpha q; ||r||, stopping test; the
  // next V-cycle input (FP64: sol1 = F(D .* r); FP32: b = S(r * scale), sol1 = F(D .* b))
  template<typename S, int R, bool CONVERT>
  __global__ void __launch_bounds__(MNT) km_pcg_x(double* __restrict__ x, double* __restrict__ rr,
    const double* __restrict__ p, const double* __restrict__ q, const uint8_t* __restrict__ dm, S* __restrict__ bt,
    S* __restrict__ x1, const S* __restrict__ dinv, int* __restrict__ skip_top, double* __restrict__ hist,
    uint32_t n, int hist_stride, MScal* __restrict__ sc)
  {
    constexpr int K = 32 * R;
    if(closed(sc))
      return;
    const int lane = threadIdx.x & 31;
    double part[R], alpha[R], scale[R];
    bool act[R];
    #pragma unroll
    for(int r = 0; r < R; ++r)
    {
      const int j = lane * R + r;
      act[r] = sc->status[j] == FB_SOLVER_PROGRESS;
      alpha[r] = sc->alpha[j];
      scale[r] = CONVERT ? pow2_inv(sc->def_cur[j]) : 1.0;
      part[r] = 0.0;
    }
    MR_ROWS(n)
    {
      const bool d = __ldg(dm + row) != 0;
      #pragma unroll
      for(int r = 0; r < R; ++r)
      {
        const size_t e = size_t(row) * K + lane * R + r;
        double rv = rr[e];
        if(act[r])
        {
          x[e] = add(x[e], mul(alpha[r], p[e]));
          rv = add(rv, mul(-alpha[r], q[e]));
          rr[e] = rv;
        }
        const S b = S(mul(rv, scale[r]));
        if(CONVERT)
          bt[e] = b;
        const S c = d ? S(0) : mul(__ldg(dinv + row), b);
        x1[e] = add(S(0), c);
        part[r] += mul(rv, rv);
      }
    }
    reduce_per_rhs<R>(part, sc, [&](int j, double tot)
    {
      if(sc->status[j] != FB_SOLVER_PROGRESS)
        return;
      const int it = sc->iter[j] + 1;
      const double dc = sqrt(tot);
      const double s = CONVERT ? pow2_inv(sc->def_cur[j]) : 1.0;
      sc->iter[j] = it;
      sc->def_cur[j] = dc;
      hist[size_t(it) * hist_stride + j] = dc;
      int st = FB_SOLVER_PROGRESS;
      if(!isfinite(dc))
        st = FB_SOLVER_ABORTED;
      else if(dc > sc->div_abs || dc > sc->div_rel * sc->def_init[j])
        st = FB_SOLVER_DIVERGED;
      else if(it < sc->min_iter)
        st = FB_SOLVER_PROGRESS;
      else if(dc <= sc->tol_abs && (dc <= sc->tol_rel * sc->def_init[j] || dc <= 0.0))
        st = FB_SOLVER_SUCCESS;
      else if(it >= sc->max_iter)
        st = FB_SOLVER_MAX_ITER;
      sc->status[j] = st;
      sc->scale[j] = s;
      sc->inv_scale[j] = 1.0 / s;
      skip_top[j] = skip_of<S>(dc * s);
    });
  }

  template<int R>
  __global__ void __launch_bounds__(MNT) km_pcg_p(double* __restrict__ p, const double* __restrict__ z, uint32_t n,
    int first, const MScal* __restrict__ sc)
  {
    constexpr int K = 32 * R;
    if(closed(sc))
      return;
    const int lane = threadIdx.x & 31;
    MR_ROWS(n)
    {
      #pragma unroll
      for(int r = 0; r < R; ++r)
      {
        const int j = lane * R + r;
        const size_t e = size_t(row) * K + j;
        p[e] = first ? z[e] : add(mul(p[e], sc->beta[j]), z[e]);
      }
    }
  }

  __global__ void km_gather_rows(double* __restrict__ out, const double* __restrict__ in, const uint32_t* __restrict__ perm,
    uint32_t n, int K)
  {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if(i < size_t(n) * K)
      out[i] = in[size_t(perm[i / K]) * K + i % K];
  }
  __global__ void km_scatter_rows(double* __restrict__ out, const double* __restrict__ in, const uint32_t* __restrict__ perm,
    uint32_t n, int K)
  {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if(i < size_t(n) * K)
      out[size_t(perm[i / K]) * K + i % K] = in[i];
  }
  __global__ void km_open(MScal* sc, int K)
  {
    if(threadIdx.x == 0)
      sc->progress = K;
  }
} // namespace mr
} // namespace fb

// ==================================================================== host side
struct fb_msolver
{
  fb_solver_config cfg;
  int K = 0, R = 0, nlev = 0;
  struct Mat
  {
    uint32_t rows = 0, cols = 0, nnz = 0;
    uint32_t *rp = nullptr, *col = nullptr;
    void* val = nullptr;
    void* dval = nullptr;                  // stencil form (nd = 9 or 27), see mr::MCsr
    uint32_t dn = 0;
    int nd = 0;
    int goff[9] = {};
  };
  struct Level
  {
    uint32_t n = 0;
    Mat A, P, R, A64;
    uint8_t* dm = nullptr;
    void* dinv = nullptr;
    void *b = nullptr, *x = nullptr, *x2 = nullptr, *d = nullptr, *c = nullptr, *c2 = nullptr;
    int* skip_pre = nullptr;    // [K]
    int* skip_post = nullptr;   // [K]
  };
  std::vector<Level> lv;
  std::vector<void*> allocs;
  std::vector<uint32_t> perm0;
  uint32_t* perm0_d = nullptr;
  uint32_t* free_dofs = nullptr;
  double* cinv = nullptr;
  uint32_t nfree = 0;
  double *x = nullptr, *r = nullptr, *p = nullptr, *q = nullptr, *z = nullptr, *rhs = nullptr;
  double *tin = nullptr, *tout = nullptr, *hist = nullptr;
  fb::mr::MScal* sc = nullptr;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  uint64_t launches_init = 0, launches_body = 0;
  double bytes_init = 0, bytes_body = 0;
  unsigned int grid = 1;
};

namespace fb
{
namespace mr
{
  static fb_status malloc0(fb_msolver* s, void** p, size_t bytes)
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

#define MR_TRY(x)                     \
  do {                                \
    fb_status t_ = (x);               \
    if(t_ != FB_OK) return t_;        \
  } while(0)

  static fb_status upload_stencil(fb_msolver* s, fb_msolver::Mat& d, const std::vector<uint32_t>& rp,
    const std::vector<uint32_t>& col, const std::vector<double>& val, int prec, bool use);

  static fb_status upload(fb_msolver* s, fb_msolver::Mat& d, const HostCsr& M, int prec,
    const std::vector<uint8_t>* empty, bool stencil = false)
  {
    std::vector<uint32_t> rp(size_t(M.rows) + 1, 0), col;
    std::vector<double> val;
    for(uint32_t r = 0; r < M.rows; ++r)
    {
      if(!(empty && (*empty)[r]))
        for(uint32_t j = M.rp[r]; j < M.rp[r + 1]; ++j)
        {
          col.push_back(M.col[j]);
          val.push_back(M.val[j]);
        }
      rp[r + 1] = uint32_t(col.size());
    }
    d.rows = M.rows;
    d.cols = M.cols;
    d.nnz = uint32_t(col.size());
    MR_TRY(malloc0(s, (void**)&d.rp, 4 * rp.size()));
    FB_CUDA(cudaMemcpy(d.rp, rp.data(), 4 * rp.size(), cudaMemcpyHostToDevice));
    const size_t nn = std::max<size_t>(1, col.size());
    MR_TRY(malloc0(s, (void**)&d.col, 4 * nn));
    const size_t vb = prec == FB_PREC_F64 ? 8 : 4;
    MR_TRY(malloc0(s, &d.val, vb * nn));
    if(!col.empty())
    {
      FB_CUDA(cudaMemcpy(d.col, col.data(), 4 * col.size(), cudaMemcpyHostToDevice));
      if(prec == FB_PREC_F64)
        FB_CUDA(cudaMemcpy(d.val, val.data(), 8 * val.size(), cudaMemcpyHostToDevice));
      else
      {
        std::vector<float> f(val.begin(), val.end());
        FB_CUDA(cudaMemcpy(d.val, f.data(), 4 * f.size(), cudaMemcpyHostToDevice));
      }
    }
    return upload_stencil(s, d, rp, col, val, prec, stencil);
  }

  // The stencil form of a system matrix (see MCsr): every stored row has the same column offsets,
  // 9 or 27 of them in triplets (o-1, o, o+1) with increasing centres.  Leaves d.nd = 0 when the
  // pattern does not hold (another numbering, another element) or use is 0.
  static fb_status upload_stencil(fb_msolver* s, fb_msolver::Mat& d, const std::vector<uint32_t>& rp,
    const std::vector<uint32_t>& col, const std::vector<double>& val, int prec, bool use)
  {
    d.nd = 0;
    if(!use)
      return FB_OK;
    std::vector<int64_t> off;
    for(uint32_t r = 0; r < d.rows; ++r)
    {
      const uint32_t len = rp[r + 1] - rp[r];
      if(len == 0)
        continue;
      if(off.empty())
      {
        if(len != 9 && len != 27)
          return FB_OK;
        for(uint32_t j = rp[r]; j < rp[r + 1]; ++j)
          off.push_back(int64_t(col[j]) - int64_t(r));
        for(size_t g = 0; g < off.size() / 3; ++g)
        {
          if(off[3 * g] + 1 != off[3 * g + 1] || off[3 * g + 1] + 1 != off[3 * g + 2])
            return FB_OK;
          if(g > 0 && off[3 * g] <= off[3 * g - 1])
            return FB_OK;
          if(off[3 * g + 1] > INT32_MAX || off[3 * g + 1] < -INT32_MAX)
            return FB_OK;
        }
        continue;
      }
      if(len != off.size())
        return FB_OK;
      for(uint32_t j = rp[r], k = 0; j < rp[r + 1]; ++j, ++k)
        if(int64_t(col[j]) - int64_t(r) != off[k])
          return FB_OK;
    }
    if(off.empty())
      return FB_OK;
    const int nd = int(off.size());
    const uint32_t dn = (d.rows + 7u) & ~7u;
    std::vector<double> dv(size_t(nd) * dn, 0.0);
    for(uint32_t r = 0; r < d.rows; ++r)
      for(uint32_t j = rp[r], k = 0; j < rp[r + 1]; ++j, ++k)
        dv[size_t(k) * dn + r] = val[j];
    const size_t vb = prec == FB_PREC_F64 ? 8 : 4;
    MR_TRY(malloc0(s, &d.dval, vb * dv.size()));
    if(prec == FB_PREC_F64)
      FB_CUDA(cudaMemcpy(d.dval, dv.data(), 8 * dv.size(), cudaMemcpyHostToDevice));
    else
    {
      std::vector<float> f(dv.begin(), dv.end());
      FB_CUDA(cudaMemcpy(d.dval, f.data(), 4 * f.size(), cudaMemcpyHostToDevice));
    }
    d.dn = dn;
    d.nd = nd;
    for(int g = 0; g < nd / 3; ++g)
      d.goff[g] = int(off[size_t(3 * g + 1)]);
    return FB_OK;
  }

  template<typename V> MCsr<V> mv(const fb_msolver::Mat& m)
  {
    MCsr<V> c{m.rp, m.col, static_cast<const V*>(m.val), m.rows, static_cast<const V*>(m.dval), m.dn, m.nd, {}};
    for(int g = 0; g < 9; ++g)
      c.goff[g] = m.goff[g];
    return c;
  }

  template<typename V, typename S, int R>
  struct MLaunch
  {
    fb_msolver* s;
    cudaStream_t st;
    bool dry;
    uint64_t launches = 0;
    double bytes = 0;
    static constexpr int K = 32 * R;

    unsigned int g(uint32_t rows) const
    {
      return std::max(1u, std::min(s->grid, (rows + MW - 1) / MW));
    }
    // blocks of a pass over a system matrix: one warp per row, or per strip in the stencil form
    template<typename W> unsigned int ga(const fb_msolver::Mat& m) const
    {
      constexpr uint32_t M = StripRows<W>::value;
      return g(m.nd ? (m.rows + M - 1) / M : m.rows);
    }
    // matrix bytes read by one pass, as stored
    static double mbytes(const fb_msolver::Mat& m, double vsize)
    {
      if(m.nd)
        return double(m.nd) * m.dn * vsize;
      return double(m.nnz) * (vsize + 4.0) + double(m.rows + 1) * 4.0;
    }
    double mb(const fb_msolver::Mat& m) const { return mbytes(m, sizeof(V)); }
    // f(std::integral_constant<int, G>) with G the stored form of m: 9 or 3 stencil triplets, 0 = CSR
    template<class F> static void by_form(const fb_msolver::Mat& m, F&& f)
    {
      if(m.nd == 27)
        f(std::integral_constant<int, 9>());
      else if(m.nd == 9)
        f(std::integral_constant<int, 3>());
      else
        f(std::integral_constant<int, 0>());
    }
    double vb(uint32_t n, double count) const { return double(n) * K * sizeof(S) * count; }

    void vcycle(bool top_pcg)
    {
      const int nl = s->nlev;
      std::vector<void*> xcur(static_cast<size_t>(nl));
      for(int l = 0; l + 1 < nl; ++l)
      {
        fb_msolver::Level& f = s->lv[size_t(l)];
        fb_msolver::Level& c = s->lv[size_t(l + 1)];
        void* xa = f.x;
        void* xb = f.x2;
        for(int k = 1; k < s->cfg.smooth_steps; ++k)
        {
          if(!dry)
            by_form(f.A, [&](auto gc) {
              km_smooth<V, S, R, decltype(gc)::value><<<ga<V>(f.A), MNT, 0, st>>>(mv<V>(f.A), (const S*)f.b,
                (const S*)xa, (S*)xb, (const S*)f.dinv, f.dm, f.skip_pre, s->sc);
            });
          ++launches;
          bytes += mb(f.A) + vb(f.n, 4);
          std::swap(xa, xb);
        }
        xcur[size_t(l)] = xa;
        if(!dry)
          by_form(f.A, [&](auto gc) {
            km_defect<V, S, R, decltype(gc)::value><<<ga<V>(f.A), MNT, 0, st>>>(mv<V>(f.A), (const S*)f.b,
              (const S*)xa, (S*)f.d, f.dm, s->sc);
          });
        ++launches;
        bytes += mb(f.A) + vb(f.n, 3);
        const bool coarsest = (l + 2 == nl);
        if(!dry)
          km_restrict<V, S, R><<<g(c.n), MNT, 0, st>>>(mv<V>(f.R), (const S*)f.d, (S*)c.b,
            coarsest ? (S*)nullptr : (S*)c.x, (const S*)c.dinv, c.dm, c.skip_pre, s->sc);
        ++launches;
        bytes += mb(f.R) + vb(f.n, 1) + vb(c.n, 2);
      }
      {
        fb_msolver::Level& c = s->lv[size_t(nl - 1)];
        if(!dry)
          km_coarse<S, R><<<1, 1024, 0, st>>>((const S*)c.b, (S*)c.x, c.n, s->free_dofs, s->cinv, s->nfree, s->sc);
        ++launches;
        bytes += double(s->nfree) * s->nfree * 8.0 + vb(c.n, 2);
        xcur[size_t(nl - 1)] = c.x;
      }
      for(int l = nl - 2; l >= 0; --l)
      {
        fb_msolver::Level& f = s->lv[size_t(l)];
        void* xf = xcur[size_t(l)];
        if(!dry)
          km_prolong<V, S, R><<<g(f.n), MNT, 0, st>>>(mv<V>(f.P), (const S*)xcur[size_t(l + 1)], (S*)xf, f.dm, s->sc);
        if(!dry)
          by_form(f.A, [&](auto gc) {
            km_post1<V, S, R, decltype(gc)::value><<<ga<V>(f.A), MNT, 0, st>>>(mv<V>(f.A), (const S*)f.b,
              (const S*)xf, (S*)f.d, (S*)f.c, (const S*)f.dinv, f.dm, f.skip_post, s->sc);
          });
        launches += 2;
        bytes += mb(f.P) + vb(f.n, 2) + vb(s->lv[size_t(l + 1)].n, 1) + mb(f.A) + vb(f.n, 4);
        void* ca = f.c;
        void* cb = f.c2;
        const bool top = top_pcg && l == 0;
        for(int k = 2; k <= s->cfg.smooth_steps; ++k)
        {
          const bool last = (k == s->cfg.smooth_steps);
          if(!dry)
            by_form(f.A, [&](auto gc) {
              constexpr int G = decltype(gc)::value;
              if(!last)
                km_post2<V, S, R, false, false, G><<<ga<V>(f.A), MNT, 0, st>>>(mv<V>(f.A), (const S*)f.d,
                  (const S*)ca, (S*)cb, (S*)xf, nullptr, nullptr, (const S*)f.dinv, f.dm, f.skip_post, s->sc);
              else if(top)
                km_post2<V, S, R, true, true, G><<<ga<V>(f.A), MNT, 0, st>>>(mv<V>(f.A), (const S*)f.d,
                  (const S*)ca, (S*)cb, (S*)xf, s->z, s->r, (const S*)f.dinv, f.dm, f.skip_post, s->sc);
              else
                km_post2<V, S, R, true, false, G><<<ga<V>(f.A), MNT, 0, st>>>(mv<V>(f.A), (const S*)f.d,
                  (const S*)ca, (S*)cb, (S*)xf, nullptr, nullptr, (const S*)f.dinv, f.dm, f.skip_post, s->sc);
            });
          ++launches;
          bytes += mb(f.A) + vb(f.n, 4) + (top && last ? double(f.n) * K * 16.0 : 0.0);
          std::swap(ca, cb);
        }
      }
    }

    const fb_msolver::Mat& A64() { return s->cfg.precision == FB_PREC_F64 ? s->lv[0].A : s->lv[0].A64; }

    void init()
    {
      fb_msolver::Level& t = s->lv[0];
      const bool f64 = s->cfg.precision == FB_PREC_F64;
      if(!dry)
        km_open<<<1, 32, 0, st>>>(s->sc, K);
      if(!dry)
        by_form(A64(), [&](auto gc) {
          km_pcg_init<S, R, decltype(gc)::value><<<ga<double>(A64()), MNT, 0, st>>>(mv<double>(A64()), s->rhs,
            s->x, s->r, t.dm, f64 ? (S*)t.x : (S*)nullptr, (const S*)t.dinv, t.skip_pre, s->sc);
        });
      if(!dry)
        km_count_progress<<<1, 64, 0, st>>>(s->sc, K, 0);
      launches += 3;
      bytes += mbytes(A64(), 8.0) + double(t.n) * K * 8.0 * 3;
      if(!f64)
      {
        if(!dry)
          km_prep<S, R><<<g(t.n), MNT, 0, st>>>(s->r, (S*)t.b, (S*)t.x, (const S*)t.dinv, t.dm, t.skip_pre, t.n, s->sc);
        ++launches;
        bytes += double(t.n) * K * (8.0 + 2 * sizeof(S));
      }
    }

    void tail(bool first, cudaGraphConditionalHandle cond)
    {
      fb_msolver::Level& t = s->lv[0];
      const bool f64 = s->cfg.precision == FB_PREC_F64;
      if(!dry)
      {
        km_pcg_p<R><<<g(t.n), MNT, 0, st>>>(s->p, s->z, t.n, first ? 1 : 0, s->sc);
        by_form(A64(), [&](auto gc) {
          km_pcg_q<R, decltype(gc)::value><<<ga<double>(A64()), MNT, 0, st>>>(mv<double>(A64()), s->p, s->q, t.dm,
            s->sc);
        });
        if(f64)
          km_pcg_x<S, R, false><<<g(t.n), MNT, 0, st>>>(s->x, s->r, s->p, s->q, t.dm, (S*)nullptr, (S*)t.x,
            (const S*)t.dinv, t.skip_pre, s->hist, t.n, K, s->sc);
        else
          km_pcg_x<S, R, true><<<g(t.n), MNT, 0, st>>>(s->x, s->r, s->p, s->q, t.dm, (S*)t.b, (S*)t.x,
            (const S*)t.dinv, t.skip_pre, s->hist, t.n, K, s->sc);
        km_count_progress<<<1, 64, 0, st>>>(s->sc, K, cond);
      }
      launches += 4;
      bytes += double(t.n) * K * 8.0 * 3 + mbytes(A64(), 8.0) + double(t.n) * K * 8.0 * 3 +
               double(t.n) * K * (8.0 * 6 + 2 * sizeof(S));
    }
  };

  template<typename V, typename S, int R>
  static fb_status build(fb_msolver* s)
  {
    cudaStream_t st = s->stream;
    {
      MLaunch<V, S, R> a{s, st, true};
      a.init();
      a.vcycle(true);
      a.tail(true, 0);
      s->launches_init = a.launches;
      s->bytes_init = a.bytes;
      MLaunch<V, S, R> b{s, st, true};
      b.vcycle(true);
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
      MLaunch<V, S, R> a{s, st, false};
      a.init();
      a.vcycle(true);
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
      MLaunch<V, S, R> b{s, st, false};
      b.vcycle(true);
      b.tail(false, cond);
    }
    cudaGraph_t b_out = nullptr;
    FB_CUDA(cudaStreamEndCapture(st, &b_out));
    FB_CUDA(cudaGraphInstantiate(&s->gexec, s->graph, 0));
    return FB_OK;
  }

  template<typename V, typename S, int R>
  static fb_status run(fb_msolver* s)
  {
    cudaStream_t st = s->stream;
    if(s->cfg.use_graph)
    {
      FB_CUDA(cudaGraphLaunch(s->gexec, st));
      return FB_OK;
    }
    MLaunch<V, S, R> a{s, st, false};
    a.init();
    a.vcycle(true);
    a.tail(true, 0);
    FB_CUDA(cudaGetLastError());
    while(true)
    {
      int prog = 0;
      FB_CUDA(cudaMemcpyAsync(&prog, &s->sc->progress, sizeof(int), cudaMemcpyDeviceToHost, st));
      FB_CUDA(cudaStreamSynchronize(st));
      if(prog <= 0)
        break;
      MLaunch<V, S, R> b{s, st, false};
      b.vcycle(true);
      b.tail(false, 0);
      FB_CUDA(cudaGetLastError());
    }
    return FB_OK;
  }

  static fb_status dispatch_build(fb_msolver* s)
  {
    const bool f64 = s->cfg.precision == FB_PREC_F64;
    if(s->R == 1)
      return f64 ? build<double, double, 1>(s) : build<float, float, 1>(s);
    return f64 ? build<double, double, 2>(s) : build<float, float, 2>(s);
  }
  static fb_status dispatch_run(fb_msolver* s)
  {
    const bool f64 = s->cfg.precision == FB_PREC_F64;
    if(s->R == 1)
      return f64 ? run<double, double, 1>(s) : run<float, float, 1>(s);
    return f64 ? run<double, double, 2>(s) : run<float, float, 2>(s);
  }
} // namespace mr
} // namespace fb

using namespace fb;

extern "C" {

void fb_msolver_destroy(fb_msolver* s)
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

fb_status fb_msolver_create(fb_msolver** out, fb_hierarchy* h, const fb_solver_config* cfg_in, int num_rhs)
{
  if(!out || !h || (num_rhs != 32 && num_rhs != 64))
  {
    set_error("msolver_create: bad arguments (num_rhs must be 32 or 64)");
    return FB_ERR_ARG;
  }
  for(const HostLevel& L : h->levels)
    if(!L.set)
    {
      set_error("msolver_create: every level must be set");
      return FB_ERR_STATE;
    }
  fb_solver_config cfg;
  if(cfg_in)
    cfg = *cfg_in;
  else
    fb_solver_config_default(&cfg);
  if(cfg.precision == FB_PREC_F32_BF16 || cfg.smooth_steps < 2 || h->levels.size() < 2)
  {
    set_error("msolver_create: supports FP64 / FP32 V-cycles with at least 2 smoothing steps and 2 levels");
    return FB_ERR_UNSUPPORTED;
  }
  std::unique_ptr<fb_msolver, void (*)(fb_msolver*)> s(new fb_msolver(), fb_msolver_destroy);
  s->cfg = cfg;
  s->K = num_rhs;
  s->R = num_rhs / 32;
  s->nlev = int(h->levels.size());
  const int K = s->K;
  const int prec = cfg.precision;
  const size_t vs = prec == FB_PREC_F64 ? 8 : 4;
  FB_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  FB_CUDA(cudaEventCreate(&s->ev0));
  FB_CUDA(cudaEventCreate(&s->ev1));
  int dev = 0, nsm = 148;
  FB_CUDA(cudaGetDevice(&dev));
  FB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  s->grid = unsigned(nsm) * 8u;

  std::vector<std::vector<uint32_t>> perms(size_t(s->nlev));
  if(cfg.ordering == FB_ORDER_RCM)
    for(int l = 0; l < s->nlev; ++l)
      perms[size_t(l)] = rcm_order(h->levels[size_t(l)].A);
  std::vector<std::vector<uint8_t>> dms(size_t(s->nlev));
  for(int l = 0; l < s->nlev; ++l)
  {
    const HostLevel& H = h->levels[size_t(l)];
    dms[size_t(l)].resize(H.A.rows);
    for(uint32_t k = 0; k < H.A.rows; ++k)
      dms[size_t(l)][k] = H.dmask[perms[size_t(l)].empty() ? k : perms[size_t(l)][k]];
  }
  s->lv.resize(size_t(s->nlev));
  for(int l = 0; l < s->nlev; ++l)
  {
    const HostLevel& H = h->levels[size_t(l)];
    fb_msolver::Level& D = s->lv[size_t(l)];
    const std::vector<uint32_t>& pf = perms[size_t(l)];
    const std::vector<uint32_t> inv_f = pf.empty() ? std::vector<uint32_t>() : inverse_perm(pf);
    D.n = H.A.rows;
    HostCsr A = permute(H.A, pf, inv_f);
    MR_TRY(mr::upload(s.get(), D.A, A, prec, &dms[size_t(l)], cfg.diagonal != 0));
    if(l == 0 && prec != FB_PREC_F64)
      MR_TRY(mr::upload(s.get(), D.A64, A, FB_PREC_F64, &dms[size_t(l)], cfg.diagonal != 0));
    if(l + 1 < s->nlev)
    {
      const std::vector<uint32_t>& pc = perms[size_t(l + 1)];
      const std::vector<uint32_t> inv_c = pc.empty() ? std::vector<uint32_t>() : inverse_perm(pc);
      MR_TRY(mr::upload(s.get(), D.P, permute(H.P, pf, inv_c), prec, &dms[size_t(l)]));
      MR_TRY(mr::upload(s.get(), D.R, permute(H.R, pc, inv_f), prec, &dms[size_t(l + 1)]));
    }
    MR_TRY(mr::malloc0(s.get(), (void**)&D.dm, D.n));
    FB_CUDA(cudaMemcpy(D.dm, dms[size_t(l)].data(), D.n, cudaMemcpyHostToDevice));
    std::vector<double> dinv = inv_diagonal(A, cfg.omega);
    MR_TRY(mr::malloc0(s.get(), &D.dinv, vs * D.n));
    if(prec == FB_PREC_F64)
      FB_CUDA(cudaMemcpy(D.dinv, dinv.data(), 8 * D.n, cudaMemcpyHostToDevice));
    else
    {
      std::vector<float> f(dinv.begin(), dinv.end());
      FB_CUDA(cudaMemcpy(D.dinv, f.data(), 4 * D.n, cudaMemcpyHostToDevice));
    }
    for(void** v : {&D.b, &D.x, &D.x2, &D.d, &D.c, &D.c2})
      MR_TRY(mr::malloc0(s.get(), v, vs * size_t(D.n) * K));
    MR_TRY(mr::malloc0(s.get(), (void**)&D.skip_pre, sizeof(int) * 2 * K));
    D.skip_post = D.skip_pre + K;
    if(l == s->nlev - 1)
    {
      std::vector<uint32_t> fr;
      std::vector<double> inv;
      coarse_inverse(H.A, H.dmask, fr, inv);
      for(uint32_t& f : fr)
        f = inv_f.empty() ? f : inv_f[f];
      s->nfree = uint32_t(fr.size());
      MR_TRY(mr::malloc0(s.get(), (void**)&s->free_dofs, 4 * std::max<size_t>(1, fr.size())));
      MR_TRY(mr::malloc0(s.get(), (void**)&s->cinv, 8 * std::max<size_t>(1, inv.size())));
      if(!fr.empty())
      {
        FB_CUDA(cudaMemcpy(s->free_dofs, fr.data(), 4 * fr.size(), cudaMemcpyHostToDevice));
        FB_CUDA(cudaMemcpy(s->cinv, inv.data(), 8 * inv.size(), cudaMemcpyHostToDevice));
      }
    }
  }
  const size_t n0 = s->lv[0].n;
  for(double** v : {&s->x, &s->r, &s->p, &s->q, &s->z, &s->rhs, &s->tin, &s->tout})
    MR_TRY(mr::malloc0(s.get(), (void**)v, 8 * n0 * K));
  if(prec == FB_PREC_F64)
    s->lv[0].b = s->r;
  if(!perms[0].empty())
  {
    s->perm0 = perms[0];
    MR_TRY(mr::malloc0(s.get(), (void**)&s->perm0_d, 4 * n0));
    FB_CUDA(cudaMemcpy(s->perm0_d, s->perm0.data(), 4 * n0, cudaMemcpyHostToDevice));
  }
  MR_TRY(mr::malloc0(s.get(), (void**)&s->hist, sizeof(double) * (size_t(cfg.max_iter) + 2) * K));
  MR_TRY(mr::malloc0(s.get(), (void**)&s->sc, sizeof(mr::MScal)));
  mr::MScal h0;
  std::memset(&h0, 0, sizeof(h0));
  h0.tol_rel = cfg.tol_rel;
  h0.tol_abs = cfg.tol_abs;
  h0.div_rel = 1.0 / EPS64;
  h0.div_abs = 1.0 / (EPS64 * EPS64);
  h0.min_iter = cfg.min_iter;
  h0.max_iter = cfg.max_iter;
  FB_CUDA(cudaMemcpy(s->sc, &h0, sizeof(h0), cudaMemcpyHostToDevice));
  MR_TRY(mr::dispatch_build(s.get()));
  FB_CUDA(cudaDeviceSynchronize());
  *out = s.release();
  return FB_OK;
}

static fb_status msolve_common(fb_msolver* s, fb_solve_info* info)
{
  cudaStream_t st = s->stream;
  FB_CUDA(cudaEventRecord(s->ev0, st));
  MR_TRY(mr::dispatch_run(s));
  FB_CUDA(cudaEventRecord(s->ev1, st));
  mr::MScal h;
  FB_CUDA(cudaMemcpyAsync(&h, s->sc, sizeof(h), cudaMemcpyDeviceToHost, st));
  FB_CUDA(cudaStreamSynchronize(st));
  float ms = 0.f;
  FB_CUDA(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
  int maxit = 0;
  for(int j = 0; j < s->K; ++j)
    maxit = std::max(maxit, h.iter[j]);
  const uint64_t body = maxit > 1 ? uint64_t(maxit - 1) : 0;
  const uint64_t launches = s->launches_init + body * s->launches_body;
  count_launches(launches);
  if(info)
    for(int j = 0; j < s->K; ++j)
    {
      info[j].status = h.status[j];
      info[j].iterations = h.iter[j];
      info[j].def_init = h.def_init[j];
      info[j].def_final = h.def_cur[j];
      info[j].solve_ms = double(ms);
      info[j].kernel_launches = launches;
      info[j].bytes_moved = s->bytes_init + double(body) * s->bytes_body;
    }
  return FB_OK;
}

static fb_status mperm_in(fb_msolver* s, double* dst, const double* src)
{
  const size_t n = s->lv[0].n, tot = n * size_t(s->K);
  if(s->perm0_d)
  {
    mr::km_gather_rows<<<unsigned((tot + 255) / 256), 256, 0, s->stream>>>(dst, src, s->perm0_d, uint32_t(n), s->K);
    FB_LAUNCHED(1);
  }
  else
    FB_CUDA(cudaMemcpyAsync(dst, src, 8 * tot, cudaMemcpyDeviceToDevice, s->stream));
  return FB_OK;
}

static fb_status mperm_out(fb_msolver* s, double* dst, const double* src)
{
  const size_t n = s->lv[0].n, tot = n * size_t(s->K);
  if(s->perm0_d)
  {
    mr::km_scatter_rows<<<unsigned((tot + 255) / 256), 256, 0, s->stream>>>(dst, src, s->perm0_d, uint32_t(n), s->K);
    FB_LAUNCHED(1);
  }
  else
    FB_CUDA(cudaMemcpyAsync(dst, src, 8 * tot, cudaMemcpyDeviceToDevice, s->stream));
  return FB_OK;
}

fb_status fb_msolver_solve(fb_msolver* s, double* sol, const double* rhs, fb_solve_info* info)
{
  if(!s || !sol || !rhs)
  {
    set_error("msolver_solve: bad arguments");
    return FB_ERR_ARG;
  }
  const size_t tot = size_t(s->lv[0].n) * size_t(s->K);
  FB_CUDA(cudaMemcpyAsync(s->tin, rhs, 8 * tot, cudaMemcpyHostToDevice, s->stream));
  MR_TRY(mperm_in(s, s->rhs, s->tin));
  FB_CUDA(cudaMemcpyAsync(s->tin, sol, 8 * tot, cudaMemcpyHostToDevice, s->stream));
  MR_TRY(mperm_in(s, s->x, s->tin));
  MR_TRY(msolve_common(s, info));
  MR_TRY(mperm_out(s, s->tout, s->x));
  FB_CUDA(cudaMemcpyAsync(sol, s->tout, 8 * tot, cudaMemcpyDeviceToHost, s->stream));
  FB_CUDA(cudaStreamSynchronize(s->stream));
  return FB_OK;
}

fb_status fb_msolver_solve_device(fb_msolver* s, double* sol, const double* rhs, void* stream, fb_solve_info* info)
{
  if(!s || !sol || !rhs)
  {
    set_error("msolver_solve_device: bad arguments");
    return FB_ERR_ARG;
  }
  cudaStream_t cs = as_stream(stream);
  cudaEvent_t ev;
  FB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  FB_CUDA(cudaEventRecord(ev, cs));
  FB_CUDA(cudaStreamWaitEvent(s->stream, ev, 0));
  MR_TRY(mperm_in(s, s->rhs, rhs));
  MR_TRY(mperm_in(s, s->x, sol));
  fb_status e = msolve_common(s, info);
  if(e == FB_OK)
    e = mperm_out(s, sol, s->x);
  FB_CUDA(cudaEventRecord(ev, s->stream));
  FB_CUDA(cudaStreamWaitEvent(cs, ev, 0));
  FB_CUDA(cudaStreamSynchronize(s->stream));
  cudaEventDestroy(ev);
  return e;
}

} // extern "C"
