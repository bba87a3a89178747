// Fused V-cycle passes for levels on a structured 2D grid (temporal blocking).
//
// A level qualifies when its unknowns are the vertices of a W x W grid numbered lexicographically
// (row i = y * W + x), its system matrix is held in diagonal storage with the nine diagonals of the
// 9-point stencil (offsets -W-1, -W, -W+1, -1, 0, 1, W-1, W, W+1: entry k of a row couples the
// vertex (x + k % 3 - 1, y + k / 3 - 1)), every stored entry couples geometric neighbours, and, for
// the down pass, every entry of its restriction matrix couples the coarse vertex (I, J) with a fine
// vertex within one step of (2I, 2J).  The host checks all of this when the solver is created.
//
// down pass (one launch instead of the pre-smoothing step, the defect and the restriction;
// kernel/solver/multigrid.hpp:1713-1838 with richardson.hpp:187-228): a block owns a square tile
// of coarse vertices.  It loads x (sol1) on the fine region the tile depends on (three
// halo layers), computes the smoothed x2 on that region minus one layer, the defect d on the
// region minus two layers (all in shared memory), restricts d to its coarse vertices with the
// stored restriction rows, and writes x2 of the fine vertices it owns (8 x 8 coarse vertices, 16 x
// 16 fine, per block).
//
// up pass (one launch instead of the prolongation and both post-smoothing steps; multigrid.hpp:
// 1845-2000): a block owns a tile of 16 x 16 fine vertices; x3 = x2 + F(P x_c) on the tile
// plus two layers, d = F(b - A x3) and c = F(D d) on the tile plus one layer, then
// c' = c + F(D F(d - A c)) and x = x3 + c' on the tile.  The post-smoother's skip test needs the
// level-wide defect norm, which is only known at the end: the pass assumes the smoother runs (the
// norm is finite and above eps^2, the case of every non-degenerate solve) and the last block
// rewrites the whole level without the correction if the test says otherwise.  The result goes
// to the level's x buffer, so x2 stays intact for that case.
//
// Every row is computed by the arithmetic of its per-row body in fb_rows.cuh (same operations in
// the same order, products and sums rounded separately), so the fused passes give the unfused
// values bit for bit; a neighbour outside the grid contributes exactly what the unfused row sum
// gets from its zero matrix entry (nothing, for finite vectors).  Each thread evaluates a fixed
// number of rows per phase, branch-free (indices outside the grid are clamped for the loads and
// their results discarded), and issues all its loads before the first phase: those of data that no
// kernel of the solve writes (matrix rows, D^-1, masks) even before griddepcontrol.wait.
//
// The passes serve the levels whose passes are latency-bound (a few hundred thousand rows at
// most): their blocks cut three launches to one, each with a single round of dependent loads.  On
// the largest levels the staged one-pass-per-step kernels stream better than the fused tiles
// (measured), so the solver applies the fusion up to a row threshold.
#pragma once

#include "fb_rows.cuh"

namespace fb
{
  constexpr int FZ_NT = 256;   // threads per block of both passes
  constexpr int FZ_KR = 9;     // entries per restriction row at most (the host checks)
  constexpr int FZ_KP = 4;     // entries per prolongation row at most (the host checks)
  constexpr int FZ_DOWN_TILE = 8;   // coarse tile edge of the down pass (fine 16 x 16 owned)
  constexpr int FZ_UP_TILE = 16;    // fine tile edge of the up pass

  __device__ __forceinline__ int fz_clamp(int v, int w) { return v < 0 ? 0 : (v >= w ? w - 1 : v); }

  // the nine entries of row i in diagonal storage (entry k on the diagonal of stencil point k)
  template<typename V>
  struct FzRow
  {
    typedef typename ValueTraits<V>::acc Ac;
    Ac v[9];
    __device__ __forceinline__ void load(const DCsr<V>& A, uint32_t i)
    {
      const uint32_t base = (i >> 5) * 32u * 9u + (i & 31u);
      #pragma unroll
      for(int k = 0; k < 9; ++k)
        v[k] = to_acc(ldg_v(A.val + base + uint32_t(k) * 32u));
    }
    // row sum in stored order with the gathered vector in a shared tile of row pitch `pitch`;
    // q = the row's own position in the tile
    template<typename S>
    __device__ __forceinline__ Ac sum(const S* tile, int q, int pitch) const
    {
      Ac s = Ac(0);
      #pragma unroll
      for(int k = 0; k < 9; ++k)
        s = add(s, mul(v[k], Ac(tile[q + (k / 3 - 1) * pitch + (k % 3 - 1)])));
      return s;
    }
  };

  // first slot and width of row i of a sliced-ELL / ELL matrix
  template<typename V>
  __device__ __forceinline__ void fz_row_span(const DCsr<V>& M, uint32_t i, uint32_t& base, uint32_t& K)
  {
    uint32_t b0;
    if(M.kw)
    {
      K = M.kw;
      b0 = (i >> 5) * 32u * K;
    }
    else
    {
      b0 = __ldg(M.soff + (i >> 5));
      K = (__ldg(M.soff + (i >> 5) + 1) - b0) >> 5;
    }
    base = b0 + (i & 31u);
  }

  // x + F(P xc) (prolong_row) for a prolongation of at most FZ_KP entries per row, for B rows at
  // once: the row spans, then the entries, then the gathers of all B rows go out together
  template<typename V, typename S, int B>
  __device__ __forceinline__ void fz_prolong_rows(const DCsr<V>& P, const S* __restrict__ xc,
    const S* __restrict__ x, const uint8_t* __restrict__ dm, const uint32_t (&i)[B], S (&out)[B])
  {
    typedef typename ValueTraits<V>::acc Ac;
    uint32_t base[B], K[B];
    bool d[B];
    Ac xi[B];
    #pragma unroll
    for(int k = 0; k < B; ++k)
    {
      fz_row_span(P, i[k], base[k], K[k]);
      d[k] = __ldg(dm + i[k]) != 0;
      xi[k] = Ac(x[i[k]]);
    }
    Ac v[B][FZ_KP];
    uint32_t c[B][FZ_KP];
    #pragma unroll
    for(int k = 0; k < B; ++k)
      #pragma unroll
      for(int u = 0; u < FZ_KP; ++u)
        if(uint32_t(u) < K[k])
        {
          v[k][u] = to_acc(ldg_v(P.val + base[k] + uint32_t(u) * 32u));
          c[k][u] = __ldg(P.col + base[k] + uint32_t(u) * 32u);
        }
    Ac xv[B][FZ_KP];
    #pragma unroll
    for(int k = 0; k < B; ++k)
      #pragma unroll
      for(int u = 0; u < FZ_KP; ++u)
        if(uint32_t(u) < K[k])
          xv[k][u] = Ac(__ldg(xc + c[k][u]));
    #pragma unroll
    for(int k = 0; k < B; ++k)
    {
      Ac sum = Ac(0);
      #pragma unroll
      for(int u = 0; u < FZ_KP; ++u)
        if(uint32_t(u) < K[k])
          sum = add(sum, mul(v[k][u], xv[k][u]));
      const Ac cc = d[k] ? Ac(0) : add(sum, Ac(0));
      out[k] = S(add(xi[k], cc));
    }
  }

  template<typename V, typename S>
  __device__ __forceinline__ S fz_prolong(const DCsr<V>& P, const S* __restrict__ xc, const S* __restrict__ x,
    const uint8_t* __restrict__ dm, uint32_t i)
  {
    const uint32_t ii[1] = {i};
    S o[1];
    fz_prolong_rows<V, S, 1>(P, xc, x, dm, ii, o);
    return o[0];
  }

  // Two grid sums whose totals every thread of the last block receives (the last block then
  // finishes the pass); returns true in all threads of the last block.
  template<int NT>
  __device__ __forceinline__ bool fz_grid_sum2(double a, double b, RedSlot slot, double* sh, double& ta, double& tb)
  {
    __shared__ bool am_last;
    __shared__ double tot[2];
    const double pa = block_sum<NT>(a, sh);
    const double pb = block_sum<NT>(b, sh);
    if(threadIdx.x == 0)
    {
      slot.partials[blockIdx.x] = pa;
      slot.partials[gridDim.x + blockIdx.x] = pb;
      __threadfence();
      const unsigned int prev = atomicAdd(slot.counter, 1u);
      am_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if(!am_last)
      return false;
    __threadfence();
    double sa = 0.0, sb = 0.0;
    for(unsigned int k = threadIdx.x; k < gridDim.x; k += NT)
    {
      sa += ((volatile double*)slot.partials)[k];
      sb += ((volatile double*)slot.partials)[gridDim.x + k];
    }
    const double t1 = block_sum<NT>(sa, sh);
    const double t2 = block_sum<NT>(sb, sh);
    if(threadIdx.x == 0)
    {
      *slot.counter = 0u;
      tot[0] = t1;
      tot[1] = t2;
    }
    __syncthreads();
    ta = tot[0];
    tb = tot[1];
    return true;
  }

  // region geometry: point p of a region of edge E whose first point is the fine vertex (ox, oy)
  struct FzPt
  {
    int gx, gy;
    bool in;
    uint32_t i;   // the row (clamped into the grid)
  };
  template<int E>
  __device__ __forceinline__ FzPt fz_pt(int p, int ox, int oy, int w)
  {
    const int py = p / E, px = p - py * E;
    FzPt r;
    r.gx = ox + px;
    r.gy = oy + py;
    r.in = r.gx >= 0 && r.gx < w && r.gy >= 0 && r.gy < w;
    r.i = uint32_t(fz_clamp(r.gy, w) * w + fz_clamp(r.gx, w));
    return r;
  }

  // the k-th point of this thread in a region of N points (the last one repeated past the end)
  template<int N>
  __device__ __forceinline__ int fz_p(int k) { return min(int(threadIdx.x) + k * FZ_NT, N - 1); }
  template<int N>
  __device__ __forceinline__ bool fz_live(int k) { return int(threadIdx.x) + k * FZ_NT < N; }
  template<int N>
  __host__ __device__ constexpr int fz_per_thread() { return (N + FZ_NT - 1) / FZ_NT; }

  // down pass of level (W x W) into its coarse level (Wc x Wc), one block per 8 x 8 coarse tile;
  // xc == nullptr: the coarse level is the coarsest (no sol1, no skip flag), as in OpRestrict.
  // Everything a block reads that no kernel of the solve writes (the rows of A and R, D^-1, the
  // masks) is loaded before griddepcontrol.wait, so it overlaps the predecessor's end; after the
  // wait one round of loads (sol1, b, the skip flag) precedes three shared-memory phases.
  template<typename V, typename S>
  __global__ void __launch_bounds__(FZ_NT) k_fz_down(DCsr<V> A, DCsr<V> R, uint32_t W, uint32_t Wc,
    const S* __restrict__ b, const S* __restrict__ x, S* __restrict__ x2, const S* __restrict__ dinv,
    const uint8_t* __restrict__ dm, const int* __restrict__ skip, S* __restrict__ bc, S* __restrict__ xc,
    const S* __restrict__ dinvc, const uint8_t* __restrict__ dmc, int* __restrict__ skip_c, RedSlot slot,
    const Scalars* __restrict__ sc)
  {
    typedef typename ValueTraits<V>::acc Ac;
    constexpr int TC = FZ_DOWN_TILE;
    static_assert(TC * TC <= FZ_NT && 4 * TC * TC <= FZ_NT, "one coarse and four fine vertices per thread");
    constexpr int DW = 2 * TC + 1;   // defect region edge (the coarse tile's restriction stencils)
    constexpr int SW = DW + 2;       // smoothed region edge
    constexpr int XW = SW + 2;       // sol1 region edge
    constexpr int NX = fz_per_thread<XW * XW>(), NS = fz_per_thread<SW * SW>(), ND = fz_per_thread<DW * DW>();
    __shared__ S xs[XW * XW];
    __shared__ S x2s[SW * SW];
    __shared__ S ds[DW * DW];
    __shared__ double sh[32];
    const uint32_t tiles_x = (Wc + TC - 1) / TC;
    const int I0 = int(blockIdx.x % tiles_x) * TC;
    const int J0 = int(blockIdx.x / tiles_x) * TC;
    const int fx0 = 2 * I0 - 3, fy0 = 2 * J0 - 3;   // fine origin of the sol1 region
    const int w = int(W);
    // ---- prologue: matrix rows, D^-1 and masks (constant during a solve)
    FzRow<V> as[NS], ad[ND];
    Ac dis[NS];
    bool ms[NS], md[ND];
    uint32_t is_[NS], id_[ND];
    #pragma unroll
    for(int k = 0; k < NS; ++k)
    {
      is_[k] = fz_pt<SW>(fz_p<SW * SW>(k), fx0 + 1, fy0 + 1, w).i;
      as[k].load(A, is_[k]);
      dis[k] = Ac(__ldg(dinv + is_[k]));
      ms[k] = __ldg(dm + is_[k]) != 0;
    }
    #pragma unroll
    for(int k = 0; k < ND; ++k)
    {
      id_[k] = fz_pt<DW>(fz_p<DW * DW>(k), fx0 + 2, fy0 + 2, w).i;
      ad[k].load(A, id_[k]);
      md[k] = __ldg(dm + id_[k]) != 0;
    }
    const int ti = int(threadIdx.x) % TC, tj = int(threadIdx.x) / TC;
    const int I = I0 + ti, J = J0 + tj;
    const bool rown = int(threadIdx.x) < TC * TC && I < int(Wc) && J < int(Wc);
    const uint32_t j = uint32_t(min(J, int(Wc) - 1)) * Wc + uint32_t(min(I, int(Wc) - 1));
    const int centre = (2 * min(J, int(Wc) - 1)) * w + 2 * min(I, int(Wc) - 1);   // the coarse vertex, fine position
    uint32_t rbase, rk;
    fz_row_span(R, j, rbase, rk);
    Ac rv[FZ_KR];
    int rc[FZ_KR];
    #pragma unroll
    for(int u = 0; u < FZ_KR; ++u)
      if(uint32_t(u) < rk)
      {
        rv[u] = to_acc(ldg_v(R.val + rbase + uint32_t(u) * 32u));
        rc[u] = int(__ldg(R.col + rbase + uint32_t(u) * 32u)) - centre;
      }
    const bool dc = __ldg(dmc + j) != 0;
    const Ac dic = xc ? Ac(__ldg(dinvc + j)) : Ac(0);
    // ---- the predecessor's results
    pdl_wait();
    if(gate_closed(sc))
      return;
    S xv[NX];
    #pragma unroll
    for(int k = 0; k < NX; ++k)
      xv[k] = x[fz_pt<XW>(fz_p<XW * XW>(k), fx0, fy0, w).i];
    Ac bs[NS], bd[ND];
    #pragma unroll
    for(int k = 0; k < NS; ++k)
      bs[k] = Ac(b[is_[k]]);
    #pragma unroll
    for(int k = 0; k < ND; ++k)
      bd[k] = Ac(b[id_[k]]);
    const bool skipped = *skip != 0;
    #pragma unroll
    for(int k = 0; k < NX; ++k)
      if(fz_live<XW * XW>(k))
      {
        const int p = fz_p<XW * XW>(k);
        xs[p] = fz_pt<XW>(p, fx0, fy0, w).in ? xv[k] : S(0);
      }
    __syncthreads();
    // pre-smoothing step 2 (smooth_row) on the sol1 region minus one layer
    #pragma unroll
    for(int k = 0; k < NS; ++k)
      if(fz_live<SW * SW>(k))
      {
        const int p = fz_p<SW * SW>(k);
        const int q = (p / SW + 1) * XW + p % SW + 1;
        const Ac sum = as[k].sum(xs, q, XW);
        const Ac d1 = ms[k] ? Ac(0) : sub(bs[k], sum);
        const Ac c = ms[k] ? Ac(0) : mul(dis[k], d1);
        const S out = S(add(Ac(xs[q]), c));
        x2s[p] = (fz_pt<SW>(p, fx0 + 1, fy0 + 1, w).in && !skipped) ? out : S(0);
      }
    __syncthreads();
    // defect (defect_row) on the region minus two layers
    #pragma unroll
    for(int k = 0; k < ND; ++k)
      if(fz_live<DW * DW>(k))
      {
        const int p = fz_p<DW * DW>(k);
        const Ac sum = ad[k].sum(x2s, (p / DW + 1) * SW + p % DW + 1, SW);
        ds[p] = (fz_pt<DW>(p, fx0 + 2, fy0 + 2, w).in && !md[k]) ? S(sub(bd[k], sum)) : S(0);
      }
    __syncthreads();
    // restriction of the tile's coarse vertices (restrict_calc) with the stored rows of R
    double sq = 0.0;
    if(rown)
    {
      const int q0 = (2 * tj + 1) * DW + 2 * ti + 1;   // the coarse vertex in the defect tile
      Ac sum = Ac(0);
      #pragma unroll
      for(int u = 0; u < FZ_KR; ++u)
        if(uint32_t(u) < rk)
        {
          // a stored entry lies within one step of the centre; padding entries (column = the
          // zero slot) contribute the zero they contribute in the unfused sum
          const int diff = rc[u];
          int dy = 0, dx = diff;
          if(diff < -1)
          {
            dy = -1;
            dx = diff + w;
          }
          else if(diff > 1)
          {
            dy = 1;
            dx = diff - w;
          }
          const bool ok = dx >= -1 && dx <= 1;
          sum = add(sum, mul(rv[u], ok ? Ac(ds[q0 + dy * DW + dx]) : Ac(0)));
        }
      const Ac vv = dc ? Ac(0) : add(sum, Ac(0));
      bc[j] = S(vv);
      if(xc)
      {
        const Ac c = dc ? Ac(0) : mul(dic, vv);
        xc[j] = S(add(Ac(0), c));
      }
      sq = double(vv) * double(vv);
    }
    // x2 of the owned fine vertices [2 I0, 2 I0 + 2 TC) x [2 J0, 2 J0 + 2 TC), one per thread
    if(int(threadIdx.x) < 4 * TC * TC)
    {
      const int py = int(threadIdx.x) / (2 * TC), px = int(threadIdx.x) % (2 * TC);
      const int gx = 2 * I0 + px, gy = 2 * J0 + py;
      if(gx < w && gy < w)
        x2[gy * w + gx] = x2s[(py + 2) * SW + px + 2];
    }
    double total;
    if(grid_sum_last<FZ_NT>(sq, slot, sh, total) && xc)
      *skip_c = skip_from_norm<S>(sqrt(total));
  }

  // up pass of a level (W x W) from its coarse solution xcv, one block per 16 x 16 fine tile;
  // TOP: the finest level of the PCG's preconditioner (writes z = x * mg_inv_scale and r.z instead
  // of x).  As in the down pass, the rows of P and A, D^-1 and the masks are loaded before
  // griddepcontrol.wait.
  template<typename V, typename S, bool TOP>
  __global__ void __launch_bounds__(FZ_NT) k_fz_up(DCsr<V> A, DCsr<V> P, uint32_t W, const S* __restrict__ x2,
    const S* __restrict__ xcv, S* __restrict__ xo, const S* __restrict__ b, const S* __restrict__ dinv,
    const uint8_t* __restrict__ dm, int* __restrict__ skip_post, double* __restrict__ z, const double* __restrict__ r,
    RedSlot slot, Scalars* __restrict__ sc)
  {
    typedef typename ValueTraits<V>::acc Ac;
    constexpr int T = FZ_UP_TILE;
    static_assert(T * T <= FZ_NT, "one owned vertex per thread");
    constexpr int CW = T + 2;   // d, c region edge
    constexpr int XW = T + 4;   // x3 region edge
    constexpr int N3 = fz_per_thread<XW * XW>(), NC = fz_per_thread<CW * CW>();
    __shared__ S x3s[XW * XW];
    __shared__ S ds[CW * CW];
    __shared__ S cs[CW * CW];
    __shared__ double sh[32];
    const int w = int(W);
    const uint32_t tiles_x = (W + T - 1) / T;
    const int tx0 = int(blockIdx.x % tiles_x) * T;
    const int ty0 = int(blockIdx.x / tiles_x) * T;
    const int fx0 = tx0 - 2, fy0 = ty0 - 2;
    // ---- prologue: rows of P and A, D^-1, masks
    uint32_t i3[N3], pk[N3], pb[N3];
    bool m3[N3];
    Ac pv[N3][FZ_KP];
    uint32_t pc[N3][FZ_KP];
    #pragma unroll
    for(int k = 0; k < N3; ++k)
    {
      i3[k] = fz_pt<XW>(fz_p<XW * XW>(k), fx0, fy0, w).i;
      fz_row_span(P, i3[k], pb[k], pk[k]);
      m3[k] = __ldg(dm + i3[k]) != 0;
    }
    #pragma unroll
    for(int k = 0; k < N3; ++k)
      #pragma unroll
      for(int u = 0; u < FZ_KP; ++u)
        if(uint32_t(u) < pk[k])
        {
          pv[k][u] = to_acc(ldg_v(P.val + pb[k] + uint32_t(u) * 32u));
          pc[k][u] = __ldg(P.col + pb[k] + uint32_t(u) * 32u);
        }
    FzRow<V> ac[NC], ao;
    Ac dic[NC], dio;
    bool mc[NC], mo;
    uint32_t ic[NC];
    #pragma unroll
    for(int k = 0; k < NC; ++k)
    {
      ic[k] = fz_pt<CW>(fz_p<CW * CW>(k), fx0 + 1, fy0 + 1, w).i;
      ac[k].load(A, ic[k]);
      dic[k] = Ac(__ldg(dinv + ic[k]));
      mc[k] = __ldg(dm + ic[k]) != 0;
    }
    const FzPt go_ = fz_pt<T>(min(int(threadIdx.x), T * T - 1), tx0, ty0, w);
    ao.load(A, go_.i);
    dio = Ac(__ldg(dinv + go_.i));
    mo = __ldg(dm + go_.i) != 0;
    // ---- the predecessor's results
    pdl_wait();
    if(gate_closed(sc))
      return;
    Ac x2v[N3], xg[N3][FZ_KP];
    #pragma unroll
    for(int k = 0; k < N3; ++k)
    {
      x2v[k] = Ac(x2[i3[k]]);
      #pragma unroll
      for(int u = 0; u < FZ_KP; ++u)
        if(uint32_t(u) < pk[k])
          xg[k][u] = Ac(__ldg(xcv + pc[k][u]));
    }
    Ac bc_[NC];
    #pragma unroll
    for(int k = 0; k < NC; ++k)
      bc_[k] = Ac(b[ic[k]]);
    const double ro = TOP ? r[go_.i] : 0.0;
    // prolongation (prolong_row) on the tile plus two layers
    #pragma unroll
    for(int k = 0; k < N3; ++k)
      if(fz_live<XW * XW>(k))
      {
        const int p = fz_p<XW * XW>(k);
        Ac sum = Ac(0);
        #pragma unroll
        for(int u = 0; u < FZ_KP; ++u)
          if(uint32_t(u) < pk[k])
            sum = add(sum, mul(pv[k][u], xg[k][u]));
        const Ac cc = m3[k] ? Ac(0) : add(sum, Ac(0));
        x3s[p] = fz_pt<XW>(p, fx0, fy0, w).in ? S(add(x2v[k], cc)) : S(0);
      }
    __syncthreads();
    // post-smoothing step 1 (post1_calc) on the tile plus one layer; the norm over owned rows
    double sq = 0.0;
    #pragma unroll
    for(int k = 0; k < NC; ++k)
      if(fz_live<CW * CW>(k))
      {
        const int p = fz_p<CW * CW>(k);
        const int py = p / CW, px = p % CW;
        const bool in = fz_pt<CW>(p, fx0 + 1, fy0 + 1, w).in;
        const Ac sum = ac[k].sum(x3s, (py + 1) * XW + px + 1, XW);
        const Ac d1 = mc[k] ? Ac(0) : sub(bc_[k], sum);
        const Ac c1 = mc[k] ? Ac(0) : mul(dic[k], d1);
        ds[p] = in ? S(d1) : S(0);
        cs[p] = in ? S(add(Ac(0), c1)) : S(0);
        if(in && px >= 1 && px <= T && py >= 1 && py <= T)
          sq += double(d1) * double(d1);
      }
    __syncthreads();
    // post-smoothing step 2 (post2_row, not skipped) and the update of the owned row
    double rz = 0.0;
    if(int(threadIdx.x) < T * T)
    {
      const int py = int(threadIdx.x) / T, px = int(threadIdx.x) % T;
      const int q = (py + 1) * CW + px + 1;
      const Ac sum = ao.sum(cs, q, CW);
      const Ac dk = mo ? Ac(0) : sub(Ac(ds[q]), sum);
      const Ac ck = mo ? Ac(0) : mul(dio, dk);
      const Ac cn = add(Ac(cs[q]), ck);
      const S xn = S(add(Ac(x3s[(py + 2) * XW + px + 2]), cn));
      if(go_.in)
      {
        if(TOP)
        {
          const double zi = mul(double(xn), sc->mg_inv_scale);
          z[go_.i] = zi;
          rz = mul(ro, zi);
        }
        else
          xo[go_.i] = xn;
      }
    }
    double tsq, trz;
    if(!fz_grid_sum2<FZ_NT>(sq, rz, slot, sh, tsq, trz))
      return;
    // the last block: the skip test of the post-smoother; when it skips, the level's result is
    // the prolongated x3 without correction (post2_row returns 0 for a skipped smoother)
    const int sk = skip_from_norm<S>(sqrt(tsq));
    if(threadIdx.x == 0)
      *skip_post = sk;
    if(sk)
    {
      const uint32_t n = W * W;
      double rz2 = 0.0;
      for(uint32_t i = threadIdx.x; i < n; i += FZ_NT)
      {
        const S xn = S(add(Ac(fz_prolong<V, S>(P, xcv, x2, dm, i)), Ac(0)));
        if(TOP)
        {
          const double zi = mul(double(xn), sc->mg_inv_scale);
          z[i] = zi;
          rz2 += mul(r[i], zi);
        }
        else
          xo[i] = xn;
      }
      if(TOP)
        trz = block_sum<FZ_NT>(rz2, sh);
    }
    if(TOP && threadIdx.x == 0)
    {
      sc->gamma_prev = sc->gamma;
      sc->gamma = trz;
      sc->beta = trz / sc->gamma_prev;
    }
  }
} // namespace fb
