// Streamed fused V-cycle passes for the large structured 2D levels.
//
// The same two passes as fb_fused.cuh -- down: pre-smoothing step 2 + defect + restriction; up:
// prolongation + both post-smoothing steps (with the PCG's z and r.z on the top level) -- for
// levels too large for the tile-fused form, whose three halo layers around small tiles re-read and
// recompute too much.  A block owns coarse columns [X0, X0 + TC) and coarse rows [Y0, Y0 + TR), i.e.
// the fine vertices [2 X0, 2 X0 + 2 TC) x [2 Y0, 2 Y0 + 2 TR) of the grid, and sweeps them upwards
// in pairs of fine rows (pair q = fine rows 2q - 1 and 2q).  The rows a pair needs from memory
// (the system matrix in diagonal storage, the rows of R or P, the vectors and masks) are copied
// into shared memory by the bulk-copy engine one stage per pair, NR - 1 pairs ahead of the
// threads, each stage completing one mbarrier phase; the intermediate vectors (x2 and d going
// down; x3, d and c going up) live in shared-memory rings of two pairs.  Matrix rows, D^-1 and the
// masks are never written during a solve, so the first stages' copies of them go out before
// griddepcontrol.wait; the vectors written by the predecessor follow the wait.
//
// Step q of the down pass (stages q - 1 and q resident):
//   x2 on fine rows 2q-2, 2q-1     (smooth_row; x1 rows 2q-3 .. 2q)
//   d  on fine rows 2q-3, 2q-2     (defect_row; x2 rows 2q-4 .. 2q-1)
//   b_c, sol1_c on coarse row q-2  (restrict_calc; d rows 2q-5 .. 2q-3)
// Step q of the up pass:
//   x3 on fine rows 2q-1, 2q       (prolong_row; coarse x rows q-1 .. q+1)
//   d, c on fine rows 2q-2, 2q-1   (post1_calc; x3 rows 2q-3 .. 2q)
//   x (or z) on fine rows 2q-3, 2q-2 (post2_row; c rows 2q-4 .. 2q-1)
// A block runs the steps q = Y0 - 1 .. Y0 + TR + 1, so each pass is evaluated on its owned rows and
// on a halo of at most three fine rows and columns.  Every row is computed with the arithmetic of
// its per-row body in fb_rows.cuh (the same operations in the same order, products and sums rounded
// separately), so the results equal the unfused passes bit for bit; grid neighbours outside the
// level contribute zero, as their zero matrix entries do in the unfused sums (every vertex with
// such a neighbour is a Dirichlet vertex, whose result the unit filter discards anyway).  Each
// thread keeps its column offsets for the whole sweep, and every row's staged data is addressed
// through per-row pointers computed once per row and phase; the stencil's neighbours are read
// without bounds tests: the rings hold zeros outside the grid, and a staged row's out-of-grid
// neighbours are read only by Dirichlet vertices, whose values the masks discard.
//
// Requirements (checked by the host): the level is a W x W grid numbered lexicographically with
// its system matrix in diagonal storage (fb_fused.cuh), every vertex on the grid's boundary is a
// Dirichlet vertex, R has at most FZ_KR entries per row, each
// within one fine step of the coarse vertex, and every entry of P's row (x, y) couples the coarse
// vertex (x / 2 + dx, y / 2 + dy) with dx, dy in {0, 1} (integer halves), at most FZ_KP per row.
// Every mbarrier wait is bounded: on expiry the block records the failure in the error word, waits
// (bounded) for its copies still in flight, still takes part in the grid reduction and returns.
#pragma once

#include "fb_fused.cuh"
#include "fb_tma.cuh"

namespace fb
{
  constexpr int FS_NT = 256;        // threads: two fine rows of FS_COLS columns
  constexpr int FS_COLS = 128;
  constexpr int FS_TC_MAX = 61;     // coarse columns of a tile at most: 2 TC + 5 <= FS_COLS - 1

  // tile geometry of one launch
  struct FsGeom
  {
    int W, Wc;       // fine and coarse grid widths
    int TC, TR;      // coarse columns and rows of a tile
    int ntx;         // tiles across the grid
  };

  // stages of a pass (pairs resident: two in use, the rest in flight)
  template<typename V, bool UP>
  __host__ __device__ constexpr int fs_stages() { return sizeof(V) == 8 ? 3 : (UP ? 3 : 4); }

  // shared-memory layout of one stage (byte offsets, every region a multiple of 16 bytes)
  template<typename V, typename S, bool UP, bool TOP>
  struct FsLay
  {
    static constexpr uint32_t SPAN = 2u * FS_TC_MAX + 5u;                  // fine columns of a staged row
    static constexpr uint32_t SL = (SPAN + 31u) / 32u + 1u;                // its diagonal-storage slices
    static constexpr uint32_t AR = SL * 9u * 32u;                          // A entries of a staged row
    static constexpr uint32_t VE = 16u / sizeof(S);                        // vector elements per 16 bytes
    static constexpr uint32_t VW = (SPAN + 2u * VE - 2u + VE - 1u) / VE * VE;
    static constexpr uint32_t MW = (SPAN + 30u + 15u) / 16u * 16u;          // mask bytes of a row
    static constexpr uint32_t DW = (SPAN + 2u + 1u) / 2u * 2u;              // FP64 r of a row
    static constexpr uint32_t RE = ((FS_TC_MAX + 31u) / 32u + 1u) * uint32_t(FZ_KR) * 32u;   // R entries
    static constexpr uint32_t PE = SL * uint32_t(FZ_KP) * 32u;             // P entries of a row
    static constexpr uint32_t CSPAN = FS_TC_MAX + 3u;                      // coarse columns of a staged coarse row
    static constexpr uint32_t CW = (CSPAN + 2u * VE - 2u + VE - 1u) / VE * VE;
    static constexpr uint32_t oA = 0;
    static constexpr uint32_t oB = oA + 2u * AR * uint32_t(sizeof(V));      // b rows
    static constexpr uint32_t oD = oB + 2u * VW * uint32_t(sizeof(S));      // D^-1 rows
    static constexpr uint32_t oX = oD + 2u * VW * uint32_t(sizeof(S));      // x1 (down) / x2 (up) rows
    static constexpr uint32_t oM = oX + 2u * VW * uint32_t(sizeof(S));      // mask rows
    static constexpr uint32_t oTv = oM + 2u * MW;                           // R (down) / P (up) values
    static constexpr uint32_t oTc = oTv + (UP ? 2u * PE : RE) * uint32_t(sizeof(V));   // their columns
    static constexpr uint32_t oC = oTc + (UP ? 2u * PE : RE) * 4u;          // up: coarse x rows q-1 .. q+1
    static constexpr uint32_t oR = oC + (UP ? 3u * CW * uint32_t(sizeof(S)) : 0u);   // up, top level: r rows
    static constexpr uint32_t SO = 16u;                                   // slice offsets of a staged row of R / P
    static constexpr uint32_t oSo = oR + (TOP ? 2u * DW * 8u : 0u);
    static constexpr uint32_t STAGE = oSo + (UP ? 2u : 1u) * SO * 4u;
    static constexpr uint32_t NR = uint32_t(fs_stages<V, UP>());
    static constexpr uint32_t RING = 2u * 2u * uint32_t(FS_COLS) * uint32_t(sizeof(S));   // two pairs of rows
    static constexpr uint32_t NRING = UP ? 3u : 2u;
    static constexpr uint32_t SMEM = NR * STAGE + NRING * RING;
    static_assert(oB % 16u == 0 && oD % 16u == 0 && oX % 16u == 0 && oM % 16u == 0 && oTv % 16u == 0 &&
                  oTc % 16u == 0 && oC % 16u == 0 && oR % 16u == 0 && oSo % 16u == 0 && STAGE % 16u == 0,
                  "16-byte regions");
  };

  // one bulk copy of a stage, described by one lane of the issuing warp (n == 0: no copy)
  struct FsCp
  {
    const void* src;
    uint32_t off;    // destination offset in the stage
    uint32_t n;      // bytes
    int part;        // 1: constant data, 2: the predecessor's vectors
  };

  // The issuing warp (all 32 lanes): lane l holds copy l of a stage.  With mask & 4 the warp sums the
  // stage's bytes and lane 0 arrives on its mbarrier expecting them (before any copy is issued);
  // then every lane issues its copy when its part is selected (mask & part).
  __device__ __forceinline__ void fs_issue_warp(const FsCp& c, unsigned char* st, uint64_t* bar, int mask)
  {
    if(mask & 4)
    {
      uint32_t tot = c.n;
      #pragma unroll
      for(int o = 16; o > 0; o >>= 1)
        tot += __shfl_xor_sync(0xffffffffu, tot, o);
      if((threadIdx.x & 31u) == 0)
        mbar_expect_tx(bar, tot);
      __syncwarp();
    }
    if(c.n && (mask & c.part))
      bulk_g2s(st + c.off, c.src, c.n, bar);
  }

  // first staged column of the block's rows
  __device__ __forceinline__ int fs_c0(int X0) { return max(2 * X0 - 3, 0); }

  // the staged span of fine row y: global rows [g0, g1) (columns [max(2 X0 - 3, 0), min(2 X0 + 2 TC + 2, W)))
  __device__ __forceinline__ void fs_span(const FsGeom& g, int X0, int y, uint32_t& g0, uint32_t& g1)
  {
    g0 = uint32_t(y * g.W + fs_c0(X0));
    g1 = uint32_t(y * g.W + min(2 * X0 + 2 * g.TC + 2, g.W));
  }

  template<uint32_t E>
  __device__ __forceinline__ uint32_t fs_dn(uint32_t v) { return v & ~(E - 1u); }
  template<uint32_t E>
  __device__ __forceinline__ uint32_t fs_up(uint32_t v) { return (v + E - 1u) & ~(E - 1u); }

  // a vector row's range [g0, g1) rounded out to 16 bytes
  template<typename T>
  __device__ __forceinline__ FsCp fs_vec(uint32_t off, const T* v, uint32_t g0, uint32_t g1, int part)
  {
    constexpr uint32_t E = 16u / sizeof(T);
    const uint32_t e0 = fs_dn<E>(g0), e1 = fs_up<E>(g1);
    return FsCp{v + e0, off, (e1 - e0) * uint32_t(sizeof(T)), part};
  }

  // the diagonal-storage slices of global rows [g0, g1)
  template<typename V>
  __device__ __forceinline__ FsCp fs_diag(uint32_t off, const DCsr<V>& A, uint32_t g0, uint32_t g1)
  {
    const uint32_t s0 = g0 >> 5, s1 = (g1 - 1u) >> 5;
    return FsCp{A.val + size_t(s0) * 288u, off, (s1 - s0 + 1u) * 288u * uint32_t(sizeof(V)), 1};
  }

  // first entry of slice s of a sliced-ELL / ELL matrix (from global memory)
  template<typename V>
  __device__ __forceinline__ uint32_t fs_slice_start(const DCsr<V>& M, uint32_t s)
  {
    return M.kw ? s * 32u * M.kw : __ldg(M.soff + s);
  }

  // part `kind` of the sliced-ELL rows [g0, g1) of M whose entries are [e0, e1): 0 the values to
  // voff, 1 the columns to coff, 2 (sliced storage) the slice offsets soff[s0 & ~3 ..] covering
  // soff[s0 .. s1 + 1] to soff_off
  template<typename V>
  __device__ __forceinline__ FsCp fs_ell(int kind, uint32_t voff, uint32_t coff, uint32_t soff_off, const DCsr<V>& M,
    uint32_t g0, uint32_t g1, uint32_t e0, uint32_t e1)
  {
    if(kind == 0)
      return FsCp{M.val + e0, voff, (e1 - e0) * uint32_t(sizeof(V)), 1};
    if(kind == 1)
      return FsCp{M.col + e0, coff, (e1 - e0) * 4u, 1};
    if(M.kw)
      return FsCp{nullptr, 0u, 0u, 1};
    const uint32_t a = (g0 >> 5) & ~3u, e = (((g1 - 1u) >> 5) + 5u) & ~3u;
    return FsCp{M.soff + a, soff_off, (e - a) * 4u, 1};
  }

  // first entry of slice s from the staged slice offsets `so` (which start at slice s0 & ~3)
  template<typename V>
  __device__ __forceinline__ uint32_t fs_sstart(const DCsr<V>& M, const uint32_t* so, uint32_t s0, uint32_t s)
  {
    return M.kw ? s * 32u * M.kw : so[s - (s0 & ~3u)];
  }

  // a staged fine row: pointers to the data of the block's first staged column c0
  template<typename L, typename V, typename S>
  struct FsRowP
  {
    const unsigned char* st;   // the stage of the row's pair
    uint32_t ri;               // 0: the pair's first row (2q - 1), 1: its second (2q)
    uint32_t g0;               // global row of column c0
    const V* a;                // A: column offset o at a[((o + m32) >> 5) * 288 + k * 32 + ((o + m32) & 31)]
    uint32_t m32;
    const S* b;                // vectors: column offset o at [o]
    const S* dv;
    const S* x;
    const uint8_t* m;
    __device__ __forceinline__ const V* arow(int o) const
    {
      const uint32_t u = uint32_t(o) + m32;
      return a + (u >> 5) * 288u + (u & 31u);
    }
  };

  template<typename L, typename V, typename S>
  __device__ __forceinline__ FsRowP<L, V, S> fs_rowp(const unsigned char* sm, int y, int w, int c0, int qb)
  {
    FsRowP<L, V, S> p;
    const int q = (y + 1) >> 1;
    p.st = sm + (uint32_t(q - qb) % L::NR) * L::STAGE;
    p.ri = uint32_t(y + 1) & 1u;
    p.g0 = uint32_t(y * w + c0);
    p.a = reinterpret_cast<const V*>(p.st + L::oA) + p.ri * L::AR;
    p.m32 = p.g0 & 31u;
    const uint32_t mv = p.g0 & (L::VE - 1u);
    p.b = reinterpret_cast<const S*>(p.st + L::oB) + p.ri * L::VW + mv;
    p.dv = reinterpret_cast<const S*>(p.st + L::oD) + p.ri * L::VW + mv;
    p.x = reinterpret_cast<const S*>(p.st + L::oX) + p.ri * L::VW + mv;
    p.m = p.st + L::oM + p.ri * L::MW + (p.g0 & 15u);
    return p;
  }

  // the nine-point row sum in stored order (entry k couples column offset k % 3 - 1 of row k / 3 - 1)
  // with the rows' vectors at xm, x0, xp (each pointing at the row's own column)
  template<typename V, typename S>
  __device__ __forceinline__ typename ValueTraits<V>::acc fs_sum9(const V* ar, const S* xm, const S* x0, const S* xp)
  {
    typedef typename ValueTraits<V>::acc Ac;
    Ac s = Ac(0);
    s = add(s, mul(to_acc(ar[0]), Ac(xm[-1])));
    s = add(s, mul(to_acc(ar[32]), Ac(xm[0])));
    s = add(s, mul(to_acc(ar[64]), Ac(xm[1])));
    s = add(s, mul(to_acc(ar[96]), Ac(x0[-1])));
    s = add(s, mul(to_acc(ar[128]), Ac(x0[0])));
    s = add(s, mul(to_acc(ar[160]), Ac(x0[1])));
    s = add(s, mul(to_acc(ar[192]), Ac(xp[-1])));
    s = add(s, mul(to_acc(ar[224]), Ac(xp[0])));
    s = add(s, mul(to_acc(ar[256]), Ac(xp[1])));
    return s;
  }

  // The rows of R a down-pass stage carries: coarse row q - 2 when the block restricts it; the entry
  // range [e0, e1) of its staged slices (the slice starts are read from global memory, by the
  // issuing lanes, a step before the copy).
  template<typename V>
  __device__ __forceinline__ bool fs_down_rrow(const DCsr<V>& R, const FsGeom& g, int X0, int Y0, int q, uint32_t& j0,
    uint32_t& j1)
  {
    const int yc = q - 2;
    if(yc < Y0 || yc >= min(Y0 + g.TR, g.Wc))
      return false;
    j0 = uint32_t(yc * g.Wc + X0);
    j1 = uint32_t(yc * g.Wc + min(X0 + g.TC, g.Wc));
    return true;
  }

  // the slice starts a lane of the issuing warp needs for stage q (down pass: lanes 10, 11 for R)
  template<typename V>
  __device__ __forceinline__ void fs_down_starts(int lane, const DCsr<V>& R, const FsGeom& g, int X0, int Y0, int q,
    uint32_t& e0, uint32_t& e1)
  {
    uint32_t j0, j1;
    e0 = e1 = 0u;
    if((lane == 10 || lane == 11) && fs_down_rrow(R, g, X0, Y0, q, j0, j1))
    {
      e0 = fs_slice_start(R, j0 >> 5);
      e1 = fs_slice_start(R, ((j1 - 1u) >> 5) + 1u);
    }
  }

  // copy `lane` of stage q of the down pass: rows 2q - 1 and 2q (lanes 0..9: A, D^-1, mask, b, x1
  // of each) and the rows of R of coarse row q - 2 (lanes 10..12: values, columns, slice offsets)
  template<typename V, typename S>
  __device__ __forceinline__ FsCp fs_down_copy(int lane, const DCsr<V>& A, const DCsr<V>& R, const FsGeom& g, int X0,
    int Y0, int q, const S* b, const S* x, const S* dinv, const uint8_t* dm, uint32_t e0, uint32_t e1)
  {
    typedef FsLay<V, S, false, false> L;
    if(lane < 10)
    {
      const int ri = lane / 5, kind = lane % 5;
      const int y = 2 * q - 1 + ri;
      if(y < 0 || y >= g.W)
        return FsCp{nullptr, 0u, 0u, 1};
      uint32_t g0, g1;
      fs_span(g, X0, y, g0, g1);
      const uint32_t vo = uint32_t(ri) * L::VW * uint32_t(sizeof(S));
      switch(kind)
      {
        case 0: return fs_diag(L::oA + uint32_t(ri) * L::AR * uint32_t(sizeof(V)), A, g0, g1);
        case 1: return fs_vec(L::oD + vo, dinv, g0, g1, 1);
        case 2: return fs_vec(L::oM + uint32_t(ri) * L::MW, dm, g0, g1, 1);
        case 3: return fs_vec(L::oB + vo, b, g0, g1, 2);
        default: return fs_vec(L::oX + vo, x, g0, g1, 2);
      }
    }
    uint32_t j0, j1;
    if(lane < 13 && fs_down_rrow(R, g, X0, Y0, q, j0, j1))
    {
      return fs_ell(lane - 10, L::oTv, L::oTc, L::oSo, R, j0, j1, e0, e1);
    }
    return FsCp{nullptr, 0u, 0u, 1};
  }

  // the slice starts a lane of the issuing warp needs for stage q (up pass: the lanes of P's values
  // and columns of each row)
  template<typename V>
  __device__ __forceinline__ void fs_up_starts(int lane, const DCsr<V>& P, const FsGeom& g, int X0, int q,
    uint32_t& e0, uint32_t& e1)
  {
    e0 = e1 = 0u;
    if(lane >= 18)
      return;
    const int ri = lane / 9, kind = lane % 9;
    const int y = 2 * q - 1 + ri;
    if((kind != 3 && kind != 4) || y < 0 || y >= g.W)
      return;
    uint32_t g0, g1;
    fs_span(g, X0, y, g0, g1);
    e0 = fs_slice_start(P, g0 >> 5);
    e1 = fs_slice_start(P, ((g1 - 1u) >> 5) + 1u);
  }

  // copy `lane` of stage q of the up pass: rows 2q - 1 and 2q (lanes 0..17: A, D^-1, mask, P's
  // values, columns and slice offsets, x2, b, on the top level r, of each) and the coarse x rows
  // q - 1 .. q + 1 the prolongation of those rows reads (lanes 18..20)
  template<typename V, typename S, bool TOP>
  __device__ __forceinline__ FsCp fs_up_copy(int lane, const DCsr<V>& A, const DCsr<V>& P, const FsGeom& g, int X0,
    int q, const S* x2, const S* xc, const S* b, const S* dinv, const uint8_t* dm, const double* r, uint32_t e0,
    uint32_t e1)
  {
    typedef FsLay<V, S, true, TOP> L;
    if(lane < 18)
    {
      const int ri = lane / 9, kind = lane % 9;
      const int y = 2 * q - 1 + ri;
      if(y < 0 || y >= g.W)
        return FsCp{nullptr, 0u, 0u, 1};
      uint32_t g0, g1;
      fs_span(g, X0, y, g0, g1);
      const uint32_t vo = uint32_t(ri) * L::VW * uint32_t(sizeof(S));
      const uint32_t po = uint32_t(ri) * L::PE;
      switch(kind)
      {
        case 0: return fs_diag(L::oA + uint32_t(ri) * L::AR * uint32_t(sizeof(V)), A, g0, g1);
        case 1: return fs_vec(L::oD + vo, dinv, g0, g1, 1);
        case 2: return fs_vec(L::oM + uint32_t(ri) * L::MW, dm, g0, g1, 1);
        case 3:
        case 4:
        case 5:
          return fs_ell(kind - 3, L::oTv + po * uint32_t(sizeof(V)), L::oTc + po * 4u,
                        L::oSo + uint32_t(ri) * L::SO * 4u, P, g0, g1, e0, e1);
        case 6: return fs_vec(L::oX + vo, x2, g0, g1, 2);
        case 7: return fs_vec(L::oB + vo, b, g0, g1, 2);
        default:
          return TOP ? fs_vec(L::oR + uint32_t(ri) * L::DW * 8u, r, g0, g1, 2) : FsCp{nullptr, 0u, 0u, 1};
      }
    }
    if(lane < 21)
    {
      const int k = lane - 18, yc = q - 1 + k;
      if(yc < 0 || yc >= g.Wc)
        return FsCp{nullptr, 0u, 0u, 1};
      const uint32_t j0 = uint32_t(yc * g.Wc + max(X0 - 1, 0)), j1 = uint32_t(yc * g.Wc + min(X0 + g.TC + 2, g.Wc));
      return fs_vec(L::oC + uint32_t(k) * L::CW * uint32_t(sizeof(S)), xc, j0, j1, 2);
    }
    return FsCp{nullptr, 0u, 0u, 1};
  }

  // bounded wait for the use-th phase of a stage's mbarrier; false when the limit expired
  __device__ __forceinline__ bool fs_wait(uint64_t* bar, uint32_t use) { return mbar_wait(bar, use & 1u); }

  // end of a sweep: thread 0 waits (bounded) for the copies of the pairs issued but not waited for
  // (steps done .. issued - 1) and records an expired wait; the block then leaves together
  __device__ __forceinline__ void fs_drain(uint64_t* bar, int nr, int done, int issued, bool failed, int* err)
  {
    if(threadIdx.x == 0)
    {
      for(int k = done; k < issued; ++k)
        if(!fs_wait(&bar[k % nr], uint32_t(k / nr)))
        {
          failed = true;
          break;
        }
      if(failed)
        atomicOr(err, 1);
    }
    __syncthreads();
  }

  // Down pass of level (W x W) into its coarse level; xc == nullptr: the coarse level is the
  // coarsest (no sol1, no skip flag), as in OpRestrict.
  template<typename V, typename S>
  __global__ void __launch_bounds__(FS_NT) k_fs_down(DCsr<V> A, DCsr<V> R, FsGeom g, const S* __restrict__ b,
    const S* __restrict__ x, S* __restrict__ x2, const S* __restrict__ dinv, const uint8_t* __restrict__ dm,
    const int* __restrict__ skip, S* __restrict__ bc, S* __restrict__ xc, const S* __restrict__ dinvc,
    const uint8_t* __restrict__ dmc, int* __restrict__ skip_c, RedSlot slot, int* err, const Scalars* __restrict__ sc)
  {
    typedef typename ValueTraits<V>::acc Ac;
    typedef FsLay<V, S, false, false> L;
    typedef FsRowP<L, V, S> RP;
    constexpr int NR = int(L::NR);
    extern __shared__ __align__(128) unsigned char fs_smem[];
    __shared__ __align__(8) uint64_t bar[NR];
    __shared__ double sh[32];
    const int w = g.W;
    const int X0 = int(blockIdx.x % uint32_t(g.ntx)) * g.TC;
    const int Y0 = int(blockIdx.x / uint32_t(g.ntx)) * g.TR;
    const int qb = Y0 - 1, qe = Y0 + g.TR + 1;   // the block's steps (pairs) qb .. qe
    const int nq = qe - qb + 1;
    const int c0 = fs_c0(X0);
    S* x2r = reinterpret_cast<S*>(fs_smem + NR * L::STAGE);   // [4 rows][FS_COLS]: row y at (y + 2) & 3, column 2 X0 - 2 + t
    S* dr = x2r + 4 * FS_COLS;                                 // [4 rows][FS_COLS]: row y at (y + 3) & 3, column 2 X0 - 1 + t
    // warp 0 issues the stages, one copy per lane (e0, e1: the lane's slice starts, read beforehand)
    const int lane = int(threadIdx.x & 31u);
    auto issue = [&](int q, int mask, uint32_t e0, uint32_t e1)
    {
      const int s = (q - qb) % NR;
      const FsCp c = fs_down_copy<V, S>(lane, A, R, g, X0, Y0, q, b, x, dinv, dm, e0, e1);
      fs_issue_warp(c, fs_smem + size_t(s) * L::STAGE, &bar[s], mask);
    };
    auto starts = [&](int q, uint32_t& e0, uint32_t& e1) { fs_down_starts(lane, R, g, X0, Y0, q, e0, e1); };
    if(threadIdx.x == 0)
    {
      for(int s = 0; s < NR; ++s)
        mbar_init(&bar[s], 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    // every slot gets its first pair before the wait for the predecessor (constant data only)
    const int npre = min(NR, nq);
    int issued = npre;   // pairs issued so far (warp 0)
    if(threadIdx.x < 32)
      for(int k = 0; k < npre; ++k)
      {
        uint32_t e0, e1;
        starts(qb + k, e0, e1);
        issue(qb + k, 4 | 1, e0, e1);
      }
    // the thread's columns: x2 at 2 X0 - 2 + t, d at 2 X0 - 1 + t (offsets from c0), owned x2
    const int tid = int(threadIdx.x);
    const int r = tid >> 7, t = tid & (FS_COLS - 1);
    const int cx1 = 2 * X0 - 2 + t, cx2 = cx1 + 1;
    const int o1 = cx1 - c0, o2 = cx2 - c0;
    const bool v1 = t < 2 * g.TC + 3 && cx1 >= 0 && cx1 < w;
    const bool v2 = t < 2 * g.TC + 1 && cx2 >= 0 && cx2 < w;
    const bool own1 = cx1 >= 2 * X0 && cx1 < min(2 * (X0 + g.TC), w);
    const int yo0 = 2 * Y0, yo1 = min(2 * (Y0 + g.TR), w);
    // the restriction's coarse vertex (thread tid < TC) and its constants
    const int X = X0 + tid;
    const bool vr = tid < g.TC && X < g.Wc;
    pdl_wait();
    if(threadIdx.x < 32)
      for(int k = 0; k < npre; ++k)
        issue(qb + k, 2, 0u, 0u);
    const bool closed = gate_closed(sc);
    const bool skipped = closed ? true : (*skip != 0);
    double sq = 0.0;
    bool failed = false;
    int done = 0;   // steps whose stage was waited for
    if(!closed)
      for(int q = qb; q <= qe; ++q, ++done)
      {
        const int s = (q - qb) % NR;
        // the stage refilled at the end of this step: its lanes' slice starts go out now
        const bool refill = q > qb && q - 1 + NR <= qe;
        uint32_t ne0 = 0u, ne1 = 0u;
        if(threadIdx.x < 32 && refill)
          starts(q - 1 + NR, ne0, ne1);
        bool ok = true;
        if(threadIdx.x < 32)
          ok = fs_wait(&bar[s], uint32_t((q - qb) / NR));
        if(__syncthreads_or(!ok))
        {
          failed = true;
          break;
        }
        // pre-smoothing step 2 (smooth_row) on fine row 2q - 2 + r
        if(q >= Y0)
        {
          const int y = 2 * q - 2 + r;
          S out = S(0);
          if(v1 && y >= 0 && y < w && !skipped)
          {
            const RP p0 = fs_rowp<L, V, S>(fs_smem, y, w, c0, qb);
            const RP pm = fs_rowp<L, V, S>(fs_smem, y - 1, w, c0, qb);
            const RP pp = fs_rowp<L, V, S>(fs_smem, y + 1, w, c0, qb);
            const Ac sum = fs_sum9<V, S>(p0.arow(o1), pm.x + o1, p0.x + o1, pp.x + o1);
            const bool dd = p0.m[o1] != 0;
            const Ac d1 = dd ? Ac(0) : sub(Ac(p0.b[o1]), sum);
            const Ac c = dd ? Ac(0) : mul(Ac(p0.dv[o1]), d1);
            out = S(add(Ac(p0.x[o1]), c));
          }
          x2r[((y + 2) & 3) * FS_COLS + t] = out;
          if(own1 && y >= yo0 && y < yo1)
            x2[y * w + cx1] = out;
        }
        __syncthreads();
        // defect (defect_row) on fine row 2q - 3 + r
        if(q >= Y0 + 1)
        {
          const int y = 2 * q - 3 + r;
          S dv = S(0);
          if(v2 && y >= 0 && y < w)
          {
            const RP p0 = fs_rowp<L, V, S>(fs_smem, y, w, c0, qb);
            // the x2 ring's column of d column cx2 - 1 is t
            const Ac sum = fs_sum9<V, S>(p0.arow(o2), x2r + ((y + 1) & 3) * FS_COLS + t + 1,
                                         x2r + ((y + 2) & 3) * FS_COLS + t + 1, x2r + ((y + 3) & 3) * FS_COLS + t + 1);
            if(!p0.m[o2])
              dv = S(sub(Ac(p0.b[o2]), sum));
          }
          dr[((y + 3) & 3) * FS_COLS + t] = dv;
        }
        __syncthreads();
        // restriction (restrict_calc) of coarse row q - 2
        const int yc = q - 2;
        if(vr && yc >= Y0 && yc < min(Y0 + g.TR, g.Wc))
        {
          const unsigned char* st = fs_smem + size_t(s) * L::STAGE;
          const uint32_t j = uint32_t(yc * g.Wc + X);
          const uint32_t s0 = uint32_t(yc * g.Wc + X0) >> 5;
          const uint32_t* so = reinterpret_cast<const uint32_t*>(st + L::oSo);
          const uint32_t e0 = fs_sstart(R, so, s0, s0);
          const uint32_t es = fs_sstart(R, so, s0, j >> 5);
          const uint32_t rk = (fs_sstart(R, so, s0, (j >> 5) + 1u) - es) >> 5;
          const uint32_t base = es - e0 + (j & 31u);
          const V* rv = reinterpret_cast<const V*>(st + L::oTv) + base;
          const uint32_t* rc = reinterpret_cast<const uint32_t*>(st + L::oTc) + base;
          const int centre = 2 * yc * w + 2 * X;
          // d rows 2yc - 1, 2yc, 2yc + 1 at the column of fine 2X (ring column 2 tid + 1)
          const S* dm1 = dr + ((2 * yc + 2) & 3) * FS_COLS + 2 * tid + 1;
          const S* d00 = dr + ((2 * yc + 3) & 3) * FS_COLS + 2 * tid + 1;
          const S* dp1 = dr + ((2 * yc) & 3) * FS_COLS + 2 * tid + 1;
          Ac sum = Ac(0);
          #pragma unroll
          for(int u = 0; u < FZ_KR; ++u)
            if(uint32_t(u) < rk)
            {
              // a stored entry lies within one step of the centre; padding entries (column = the
              // zero slot) contribute the zero they contribute in the unfused sum
              const int diff = int(rc[u * 32]) - centre;
              const int dy = diff < -1 ? -1 : (diff > 1 ? 1 : 0);
              const int dx = diff - dy * w;
              Ac dvv = Ac(0);
              if(dx >= -1 && dx <= 1)
                dvv = Ac((dy < 0 ? dm1 : (dy > 0 ? dp1 : d00))[dx]);
              sum = add(sum, mul(to_acc(rv[u * 32]), dvv));
            }
          const bool dc = __ldg(dmc + j) != 0;
          const Ac vv = dc ? Ac(0) : add(sum, Ac(0));
          bc[j] = S(vv);
          if(xc)
          {
            const Ac c = dc ? Ac(0) : mul(Ac(__ldg(dinvc + j)), vv);
            xc[j] = S(add(Ac(0), c));
          }
          sq += double(vv) * double(vv);
        }
        __syncthreads();
        // every thread is past stage q - 1: refill it with pair q - 1 + NR
        if(threadIdx.x < 32 && refill)
        {
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          issue(q - 1 + NR, 7, ne0, ne1);
          ++issued;
        }
      }
    fs_drain(bar, NR, done, issued, failed, err);
    double total;
    if(grid_sum_last<FS_NT>(sq, slot, sh, total) && xc && !closed)
      *skip_c = skip_from_norm<S>(sqrt(total));
  }

  // Up pass of level (W x W) from its coarse solution xcv; TOP: the finest level of the PCG's
  // preconditioner (writes z = x * mg_inv_scale and r.z instead of x).  The post-smoother's skip
  // test needs the level-wide defect norm, known only at the end: the pass assumes the smoother
  // runs, and the last block rewrites the level without the correction if the test says otherwise
  // (as k_fz_up).  The result goes to xo, so x2 stays intact for that case.
  template<typename V, typename S, bool TOP>
  __global__ void __launch_bounds__(FS_NT) k_fs_up(DCsr<V> A, DCsr<V> P, FsGeom g, const S* __restrict__ x2,
    const S* __restrict__ xcv, S* __restrict__ xo, const S* __restrict__ b, const S* __restrict__ dinv,
    const uint8_t* __restrict__ dm, int* __restrict__ skip_post, double* __restrict__ z, const double* __restrict__ r,
    RedSlot slot, int* err, Scalars* __restrict__ sc)
  {
    typedef typename ValueTraits<V>::acc Ac;
    typedef FsLay<V, S, true, TOP> L;
    typedef FsRowP<L, V, S> RP;
    constexpr int NR = int(L::NR);
    extern __shared__ __align__(128) unsigned char fs_smem[];
    __shared__ __align__(8) uint64_t bar[NR];
    __shared__ double sh[32];
    const int w = g.W;
    const int X0 = int(blockIdx.x % uint32_t(g.ntx)) * g.TC;
    const int Y0 = int(blockIdx.x / uint32_t(g.ntx)) * g.TR;
    const int qb = Y0 - 1, qe = Y0 + g.TR + 1;
    const int nq = qe - qb + 1;
    const int c0 = fs_c0(X0);
    const int yo0 = 2 * Y0, yo1 = min(2 * (Y0 + g.TR), w);   // owned fine rows and columns
    const int xo0 = 2 * X0, xo1 = min(2 * (X0 + g.TC), w);
    S* x3r = reinterpret_cast<S*>(fs_smem + NR * L::STAGE);   // row y at (y + 1) & 3, column 2 X0 - 2 + t
    S* dr = x3r + 4 * FS_COLS;                                 // row y at (y + 2) & 3, column 2 X0 - 1 + t
    S* cr = dr + 4 * FS_COLS;                                  // row y at (y + 2) & 3, column 2 X0 - 1 + t
    // warp 0 issues the stages, one copy per lane (e0, e1: the lane's slice starts, read beforehand)
    const int lane = int(threadIdx.x & 31u);
    auto issue = [&](int q, int mask, uint32_t e0, uint32_t e1)
    {
      const int s = (q - qb) % NR;
      const FsCp c = fs_up_copy<V, S, TOP>(lane, A, P, g, X0, q, x2, xcv, b, dinv, dm, r, e0, e1);
      fs_issue_warp(c, fs_smem + size_t(s) * L::STAGE, &bar[s], mask);
    };
    auto starts = [&](int q, uint32_t& e0, uint32_t& e1) { fs_up_starts(lane, P, g, X0, q, e0, e1); };
    if(threadIdx.x == 0)
    {
      for(int s = 0; s < NR; ++s)
        mbar_init(&bar[s], 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const int npre = min(NR, nq);
    int issued = npre;
    if(threadIdx.x < 32)
      for(int k = 0; k < npre; ++k)
      {
        uint32_t e0, e1;
        starts(qb + k, e0, e1);
        issue(qb + k, 4 | 1, e0, e1);
      }
    // the thread's columns: x3 at 2 X0 - 2 + t, d and c at 2 X0 - 1 + t, the result at 2 X0 + t
    const int tid = int(threadIdx.x);
    const int rr = tid >> 7, t = tid & (FS_COLS - 1);
    const int cx1 = 2 * X0 - 2 + t, cx2 = cx1 + 1, cx3 = cx1 + 2;
    const int o1 = cx1 - c0, o2 = cx2 - c0, o3 = cx3 - c0;
    const bool v1 = t < 2 * g.TC + 4 && cx1 >= 0 && cx1 < w;
    const bool v2 = t < 2 * g.TC + 2 && cx2 >= 0 && cx2 < w;
    const bool own2 = cx2 >= xo0 && cx2 < xo1;
    const bool v3 = t < 2 * g.TC && cx3 < xo1;
    const int cj0 = max(X0 - 1, 0);   // first staged coarse column
    pdl_wait();
    if(threadIdx.x < 32)
      for(int k = 0; k < npre; ++k)
        issue(qb + k, 2, 0u, 0u);
    const bool closed = gate_closed(sc);
    const double inv_scale = TOP && !closed ? sc->mg_inv_scale : 1.0;
    double sq = 0.0, rz = 0.0;
    bool failed = false;
    int done = 0;
    if(!closed)
      for(int q = qb; q <= qe; ++q, ++done)
      {
        const int s = (q - qb) % NR;
        // the stage refilled at the end of this step: its lanes' slice starts go out now
        const bool refill = q > qb && q - 1 + NR <= qe;
        uint32_t ne0 = 0u, ne1 = 0u;
        if(threadIdx.x < 32 && refill)
          starts(q - 1 + NR, ne0, ne1);
        bool ok = true;
        if(threadIdx.x < 32)
          ok = fs_wait(&bar[s], uint32_t((q - qb) / NR));
        if(__syncthreads_or(!ok))
        {
          failed = true;
          break;
        }
        // prolongation (prolong_row) on fine row 2q - 1 + rr
        {
          const int y = 2 * q - 1 + rr;
          S out = S(0);
          if(v1 && y >= 0 && y < w)
          {
            const RP p0 = fs_rowp<L, V, S>(fs_smem, y, w, c0, qb);
            const uint32_t gi = p0.g0 + uint32_t(o1);
            const uint32_t s0 = p0.g0 >> 5;
            const uint32_t* so = reinterpret_cast<const uint32_t*>(p0.st + L::oSo) + p0.ri * L::SO;
            const uint32_t e0 = fs_sstart(P, so, s0, s0);
            const uint32_t es = fs_sstart(P, so, s0, gi >> 5);
            const uint32_t pk = (fs_sstart(P, so, s0, (gi >> 5) + 1u) - es) >> 5;
            const uint32_t base = es - e0 + (gi & 31u);
            const V* pv = reinterpret_cast<const V*>(p0.st + L::oTv) + p0.ri * L::PE + base;
            const uint32_t* pc = reinterpret_cast<const uint32_t*>(p0.st + L::oTc) + p0.ri * L::PE + base;
            // coarse x at (y / 2, x / 2) and (y / 2 + 1, x / 2): staged rows (y / 2) - (q - 1) and one more
            const int ya = y >> 1, xa = cx1 >> 1;
            const S* cxs = reinterpret_cast<const S*>(p0.st + L::oC);
            const uint32_t ma = uint32_t(ya * g.Wc + cj0) & (L::VE - 1u);
            const uint32_t mb = uint32_t((ya + 1) * g.Wc + cj0) & (L::VE - 1u);
            const S* ca = cxs + uint32_t(ya - (q - 1)) * L::CW + ma + uint32_t(xa - cj0);
            const S* cb = cxs + uint32_t(ya + 1 - (q - 1)) * L::CW + mb + uint32_t(xa - cj0);
            const int cbase = ya * g.Wc + xa;
            Ac sum = Ac(0);
            #pragma unroll
            for(int u = 0; u < FZ_KP; ++u)
              if(uint32_t(u) < pk)
              {
                // a stored entry couples (x / 2 + dx, y / 2 + dy), dx, dy in {0, 1}; padding entries
                // (column = the zero slot) contribute the zero they contribute in the unfused sum
                const int diff = int(pc[u * 32]) - cbase;
                const int dy = diff >= g.Wc ? 1 : 0;
                const int dx = diff - dy * g.Wc;
                Ac xv = Ac(0);
                if(diff >= 0 && dx >= 0 && dx <= 1 && diff <= g.Wc + 1)
                  xv = Ac((dy ? cb : ca)[dx]);
                sum = add(sum, mul(to_acc(pv[u * 32]), xv));
              }
            const Ac cc = p0.m[o1] ? Ac(0) : add(sum, Ac(0));
            out = S(add(Ac(p0.x[o1]), cc));
          }
          x3r[((y + 1) & 3) * FS_COLS + t] = out;
        }
        __syncthreads();
        // post-smoothing step 1 (post1_calc) on fine row 2q - 2 + rr
        if(q >= Y0)
        {
          const int y = 2 * q - 2 + rr;
          S dv = S(0), cv = S(0);
          if(v2 && y >= 0 && y < w)
          {
            const RP p0 = fs_rowp<L, V, S>(fs_smem, y, w, c0, qb);
            // the x3 ring's column of column cx2 - 1 is t
            const Ac sum = fs_sum9<V, S>(p0.arow(o2), x3r + (y & 3) * FS_COLS + t + 1,
                                         x3r + ((y + 1) & 3) * FS_COLS + t + 1, x3r + ((y + 2) & 3) * FS_COLS + t + 1);
            const bool dd = p0.m[o2] != 0;
            const Ac d1 = dd ? Ac(0) : sub(Ac(p0.b[o2]), sum);
            const Ac c1 = dd ? Ac(0) : mul(Ac(p0.dv[o2]), d1);
            dv = S(d1);
            cv = S(add(Ac(0), c1));
            if(own2 && y >= yo0 && y < yo1)
              sq += double(d1) * double(d1);
          }
          dr[((y + 2) & 3) * FS_COLS + t] = dv;
          cr[((y + 2) & 3) * FS_COLS + t] = cv;
        }
        __syncthreads();
        // post-smoothing step 2 (post2_row) and the update of the owned fine row 2q - 3 + rr
        if(q >= Y0 + 1)
        {
          const int y = 2 * q - 3 + rr;
          if(v3 && y >= yo0 && y < yo1)
          {
            const RP p0 = fs_rowp<L, V, S>(fs_smem, y, w, c0, qb);
            const uint32_t gi = p0.g0 + uint32_t(o3);
            // the c and d rings' column of column cx3 is t + 1, the x3 ring's t + 2
            const S* c0r = cr + ((y + 2) & 3) * FS_COLS + t + 1;
            const Ac sum = fs_sum9<V, S>(p0.arow(o3), cr + ((y + 1) & 3) * FS_COLS + t + 1, c0r,
                                         cr + ((y + 3) & 3) * FS_COLS + t + 1);
            const bool dd = p0.m[o3] != 0;
            const Ac dk = dd ? Ac(0) : sub(Ac(dr[((y + 2) & 3) * FS_COLS + t + 1]), sum);
            const Ac ck = dd ? Ac(0) : mul(Ac(p0.dv[o3]), dk);
            const Ac cn = add(Ac(c0r[0]), ck);
            const S xn = S(add(Ac(x3r[((y + 1) & 3) * FS_COLS + t + 2]), cn));
            if(TOP)
            {
              const double zi = mul(double(xn), inv_scale);
              z[gi] = zi;
              const double* rv = reinterpret_cast<const double*>(p0.st + L::oR) + p0.ri * L::DW + (p0.g0 & 1u);
              rz += mul(rv[o3], zi);
            }
            else
              xo[gi] = xn;
          }
        }
        __syncthreads();
        if(threadIdx.x < 32 && refill)
        {
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          issue(q - 1 + NR, 7, ne0, ne1);
          ++issued;
        }
      }
    fs_drain(bar, NR, done, issued, failed, err);
    if(closed)
      return;   // every block returns: the reduction is not entered
    double tsq, trz;
    if(!fz_grid_sum2<FS_NT>(sq, rz, slot, sh, tsq, trz))
      return;
    // the last block: the skip test of the post-smoother; when it skips, the level's result is
    // the prolongated x3 without correction (post2_row returns 0 for a skipped smoother)
    const int sk = skip_from_norm<S>(sqrt(tsq));
    if(threadIdx.x == 0)
      *skip_post = sk;
    if(sk)
    {
      const uint32_t n = uint32_t(w) * uint32_t(w);
      double rz2 = 0.0;
      for(uint32_t i = threadIdx.x; i < n; i += FS_NT)
      {
        const S xn = S(add(Ac(fz_prolong<V, S>(P, xcv, x2, dm, i)), Ac(0)));
        if(TOP)
        {
          const double zi = mul(double(xn), inv_scale);
          z[i] = zi;
          rz2 += mul(r[i], zi);
        }
        else
          xo[i] = xn;
      }
      if(TOP)
        trz = block_sum<FS_NT>(rz2, sh);
    }
    if(TOP && threadIdx.x == 0)
    {
      sc->gamma_prev = sc->gamma;
      sc->gamma = trz;
      sc->beta = trz / sc->gamma_prev;
    }
  }
} // namespace fb
