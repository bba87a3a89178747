// Device views and per-row arithmetic shared by the solvers of this library (single system,
// batched instances): the sliced-ELL / ELL matrix view, the row sum in stored entry order without
// FMA, and the per-row bodies of the V-cycle passes.  Every solver computes a given row with these
// functions, so all of them round identically.
#pragma once

#include "fb_common.cuh"

namespace fb
{
  // ------------------------------------------------------------------ device views
  // Sliced ELL with slices of 32 rows (one warp): slice s holds K_s = (soff[s+1]-soff[s])/32
  // entries per row, entry k of row 32s+lane at soff[s] + 32k + lane, in the row's stored order.
  // Shorter rows are padded with value 0 and a column whose vector entry is always 0 (the zero
  // slot at index `cols`, or the row itself for narrow storage).  Rows whose result the unit
  // filter discards (Dirichlet rows) are stored empty.  Column indices are either absolute u32
  // (`col`) or, for square matrices whose |col - row| fits, int16 offsets from the row (`dcol`).
  // Diagonal storage (`doff`): uniform width kw, entry k of every row on the diagonal doff[k]
  // (column = row + doff[k]; out-of-range columns of padding entries read the row itself), no
  // column indices at all.
  template<typename V>
  struct DCsr
  {
    const uint32_t* soff;   // slice offsets (sliced ELL), or nullptr for uniform width
    const uint32_t* col;    // absolute columns, or nullptr
    const int16_t* dcol;    // column - row, or nullptr
    const V* val;
    uint32_t rows;
    uint32_t kw;            // uniform entries per row (ELL: slice s starts at 32*kw*s), 0 = sliced
    const int32_t* doff = nullptr;   // diagonal offsets (diagonal storage), or nullptr
  };


  __device__ __forceinline__ double ldg_v(const double* p) { return __ldg(p); }
  __device__ __forceinline__ float ldg_v(const float* p) { return __ldg(p); }
  __device__ __forceinline__ bf16_t ldg_v(const bf16_t* p)
  {
    bf16_t b;
    b.bits = __ldg(reinterpret_cast<const unsigned short*>(p));
    return b;
  }

  // Row sum of row `row` in stored entry order; every product and sum rounded separately.  NC:
  // gather the vector through the read-only path (vectors not written by the same kernel).
  template<typename V, typename S, bool NC = true>
  __device__ __forceinline__ typename ValueTraits<V>::acc row_sum(const DCsr<V>& M, uint32_t row, const S* x)
  {
    typedef typename ValueTraits<V>::acc A;
    constexpr uint32_t U = 9;
    const uint32_t sl = row >> 5;
    if(M.kw == U && (M.dcol || M.doff))
    {
      // 2D Q1 stencil, row-relative or diagonal columns: fully unrolled, no width tests
      const uint32_t base = sl * 32u * U + (row & 31u);
      A v[U], xv[U];
      uint32_t c[U];
      #pragma unroll
      for(uint32_t u = 0; u < U; ++u)
      {
        const uint32_t e = base + u * 32u;
        v[u] = to_acc(ldg_v(M.val + e));
        if(M.doff)
        {
          const uint32_t cc = uint32_t(int32_t(row) + __ldg(M.doff + u));
          c[u] = cc < M.rows ? cc : row;
        }
        else
          c[u] = uint32_t(int32_t(row) + int32_t(__ldg(M.dcol + e)));
      }
      #pragma unroll
      for(uint32_t u = 0; u < U; ++u)
        xv[u] = NC ? A(__ldg(x + c[u])) : A(x[c[u]]);
      A sum = A(0);
      #pragma unroll
      for(uint32_t u = 0; u < U; ++u)
        sum = add(sum, mul(v[u], xv[u]));
      return sum;
    }
    uint32_t b0, K;
    if(M.kw)
    {
      // uniform width: the slice start is computed, no dependent load before the entry loads
      K = M.kw;
      b0 = sl * 32u * K;
    }
    else
    {
      b0 = __ldg(M.soff + sl);
      K = (__ldg(M.soff + sl + 1) - b0) >> 5;
    }
    const uint32_t base = b0 + (row & 31u);
    A sum = A(0);
    for(uint32_t k0 = 0; k0 < K; k0 += U)
    {
      A v[U];
      uint32_t c[U];
      #pragma unroll
      for(uint32_t u = 0; u < U; ++u)
        if(k0 + u < K)
        {
          const uint32_t e = base + (k0 + u) * 32u;
          v[u] = to_acc(ldg_v(M.val + e));
          if(M.doff)
          {
            const uint32_t cc = uint32_t(int32_t(row) + __ldg(M.doff + k0 + u));
            c[u] = cc < M.rows ? cc : row;
          }
          else
            c[u] = M.dcol ? uint32_t(int32_t(row) + int32_t(__ldg(M.dcol + e))) : __ldg(M.col + e);
        }
      A xv[U];
      #pragma unroll
      for(uint32_t u = 0; u < U; ++u)
        if(k0 + u < K)
          xv[u] = NC ? A(__ldg(x + c[u])) : A(x[c[u]]);
      #pragma unroll
      for(uint32_t u = 0; u < U; ++u)
        if(k0 + u < K)
          sum = add(sum, mul(v[u], xv[u]));
    }
    return sum;
  }

  template<typename S> __device__ __forceinline__ S eps_sq();
  template<> __device__ __forceinline__ double eps_sq<double>() { return EPS64 * EPS64; }
  template<> __device__ __forceinline__ float eps_sq<float>() { return EPS32 * EPS32; }

  // Richardson's initial-defect test (iterative.hpp:748-771): smooth only if the norm is finite
  // and above eps^2 of the smoother's precision.
  template<typename S>
  __device__ __forceinline__ int skip_from_norm(double nrm)
  {
    return (!isfinite(nrm) || nrm <= double(eps_sq<S>())) ? 1 : 0;
  }

  // ------------------------------------------------------------------ V-cycle passes
  // Per-row bodies shared by the grid kernels (one thread per row) and the single-block tail
  // kernel (block-stride loops), so both produce bitwise identical values.

  // Richardson step k >= 2 of the pre-smoother: x' = x + F(D .* F(b - A x)); skipped -> 0
  template<typename V, typename S, bool NC>
  __device__ __forceinline__ S smooth_row(const DCsr<V>& A, const S* b, const S* x, const S* dinv,
    const uint8_t* dm, bool skipped, uint32_t i)
  {
    typedef typename ValueTraits<V>::acc Ac;
    if(skipped)
      return S(0);
    // row-wise loads first: they do not depend on the row sum's gathers
    const bool d = __ldg(dm + i) != 0;
    const Ac bi = Ac(b[i]), xi = Ac(x[i]), di = Ac(__ldg(dinv + i));
    const Ac sum = row_sum<V, S, NC>(A, i, x);
    const Ac d1 = d ? Ac(0) : sub(bi, sum);
    const Ac c = d ? Ac(0) : mul(di, d1);
    return S(add(xi, c));
  }

  template<typename V, typename S, bool NC>
  __device__ __forceinline__ S defect_row(const DCsr<V>& A, const S* b, const S* x, const uint8_t* dm, uint32_t i)
  {
    typedef typename ValueTraits<V>::acc Ac;
    const bool d = __ldg(dm + i) != 0;
    const Ac bi = Ac(b[i]);
    const Ac sum = row_sum<V, S, NC>(A, i, x);
    return d ? S(0) : S(sub(bi, sum));
  }

  // b_c = F_c(R d) and (with_x) sol1_c = F_c(D_c .* b_c), without stores
  template<typename Ac>
  struct RestrictOut { Ac v, x; };
  template<typename V, typename S, bool NC>
  __device__ __forceinline__ RestrictOut<typename ValueTraits<V>::acc> restrict_calc(const DCsr<V>& R, const S* d,
    bool with_x, const S* dinvc, const uint8_t* dmc, uint32_t j)
  {
    typedef typename ValueTraits<V>::acc Ac;
    const bool dc = __ldg(dmc + j) != 0;
    const Ac di = with_x ? Ac(__ldg(dinvc + j)) : Ac(0);
    const Ac sum = row_sum<V, S, NC>(R, j, d);
    const Ac v = dc ? Ac(0) : add(sum, Ac(0));
    Ac x = Ac(0);
    if(with_x)
    {
      const Ac c = dc ? Ac(0) : mul(di, v);
      x = add(Ac(0), c);
    }
    return RestrictOut<Ac>{v, x};
  }

  // b_c = F_c(R d) and (xc != null) sol1_c = F_c(D_c .* b_c); returns b_c^2
  template<typename V, typename S, bool NC>
  __device__ __forceinline__ double restrict_row(const DCsr<V>& R, const S* d, S* bc, S* xc, const S* dinvc,
    const uint8_t* dmc, uint32_t j)
  {
    const auto o = restrict_calc<V, S, NC>(R, d, xc != nullptr, dinvc, dmc, j);
    bc[j] = S(o.v);
    if(xc)
      xc[j] = S(o.x);
    return double(o.v) * double(o.v);
  }

  // x + F(P xc)
  template<typename V, typename S, bool NC>
  __device__ __forceinline__ S prolong_row(const DCsr<V>& P, const S* xc, const S* x, const uint8_t* dm, uint32_t i)
  {
    typedef typename ValueTraits<V>::acc Ac;
    const bool d = __ldg(dm + i) != 0;
    const Ac xi = Ac(x[i]);
    const Ac sum = row_sum<V, S, NC>(P, i, xc);
    const Ac c = d ? Ac(0) : add(sum, Ac(0));
    return S(add(xi, c));
  }

  // d = F(b - A x), c = F(D .* d), without stores
  template<typename Ac>
  struct Post1Out { Ac d, c; };
  template<typename V, typename S, bool NC>
  __device__ __forceinline__ Post1Out<typename ValueTraits<V>::acc> post1_calc(const DCsr<V>& A, const S* b,
    const S* x, const S* dinv, const uint8_t* dm, uint32_t i)
  {
    typedef typename ValueTraits<V>::acc Ac;
    const bool dd = __ldg(dm + i) != 0;
    const Ac bi = Ac(b[i]), di = Ac(__ldg(dinv + i));
    const Ac sum = row_sum<V, S, NC>(A, i, x);
    const Ac dv = dd ? Ac(0) : sub(bi, sum);
    const Ac cv = dd ? Ac(0) : mul(di, dv);
    return Post1Out<Ac>{dv, add(Ac(0), cv)};
  }

  // d = F(b - A x), c = F(D .* d); returns d^2
  template<typename V, typename S, bool NC>
  __device__ __forceinline__ double post1_row(const DCsr<V>& A, const S* b, const S* x, S* d, S* c, const S* dinv,
    const uint8_t* dm, uint32_t i)
  {
    const auto o = post1_calc<V, S, NC>(A, b, x, dinv, dm, i);
    d[i] = S(o.d);
    c[i] = S(o.c);
    return double(o.d) * double(o.d);
  }

  // post-smoothing step k >= 2: c + F(D .* F(d - A c)); skipped -> 0
  template<typename V, typename S, bool NC>
  __device__ __forceinline__ typename ValueTraits<V>::acc post2_row(const DCsr<V>& A, const S* d, const S* c,
    const S* dinv, const uint8_t* dm, bool skipped, uint32_t i)
  {
    typedef typename ValueTraits<V>::acc Ac;
    if(skipped)
      return Ac(0);
    const bool dd = __ldg(dm + i) != 0;
    const Ac di_ = Ac(d[i]), ci = Ac(c[i]), dv = Ac(__ldg(dinv + i));
    const Ac sum = row_sum<V, S, NC>(A, i, c);
    const Ac dk = dd ? Ac(0) : sub(di_, sum);
    const Ac ck = dd ? Ac(0) : mul(dv, dk);
    return add(ci, ck);
  }

  // exact coarse solve on the free DOFs (FP64 arithmetic whatever S is), one block of NB threads
  template<typename S, int NB>
  __device__ __forceinline__ void coarse_block(const S* b, S* x, uint32_t n, const uint32_t* free_dofs,
    const double* inv, uint32_t m)
  {
    for(uint32_t i = threadIdx.x; i < n; i += NB)
      x[i] = S(0);
    __syncthreads();
    for(uint32_t i = threadIdx.x; i < m; i += NB)
    {
      double s = 0.0;
      for(uint32_t j = 0; j < m; ++j)
        s = add(s, mul(__ldg(inv + size_t(i) * m + j), double(b[__ldg(free_dofs + j)])));
      x[__ldg(free_dofs + i)] = S(s);
    }
  }

} // namespace fb
