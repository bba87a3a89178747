// TMA-staged row passes over sliced-ELL / ELL matrices.
//
// A persistent block walks over chunks of TMA_NT consecutive rows (TMA_NT/32 slices).  The chunk's
// values and column indices (contiguous in both layouts) are copied into shared memory by the
// bulk-copy engine
// (cp.async.bulk ... mbarrier::complete_tx), NSTAGE chunks ahead of the threads, so the matrix
// stream occupies no registers and stays in flight while the threads gather x from L1/L2 and
// apply the pass's row epilogue.  Every mbarrier wait is bounded: on expiry the kernel records the
// failure in an error word, waits (bounded) for its copies still in flight, and returns.
#pragma once

#include "fb_rows.cuh"

#include <type_traits>
#include <utility>

namespace fb
{
  // Op::block_done() exists: the epilogue finishes each block itself (instead of the grid reduction)
  template<class T, class = void>
  struct HasBlockDone : std::false_type {};
  template<class T>
  struct HasBlockDone<T, std::void_t<decltype(std::declval<const T&>().block_done())>> : std::true_type {};

  constexpr int TMA_NT = 256;          // threads = rows per chunk
  constexpr int TMA_STAGES = 3;   // pipeline depth, at most
  // Stages of a pass over values of type V: FP64 rows are wide, and two stages leave room for
  // more blocks (rows in flight) per SM; measured faster for FP64 on B200, three for FP32/BF16.
  template<typename V>
  __host__ __device__ constexpr int tma_stages() { return sizeof(V) == 8 ? 2 : 3; }
  // Diagonal storage stages values only, and its gathers go out before the wait: two stages leave
  // room for more resident blocks (measured faster for FP32 too).
  template<typename V, bool DG>
  __host__ __device__ constexpr int tma_stages_dg() { return DG ? 2 : tma_stages<V>(); }
  constexpr uint32_t TMA_SPIN = 1u << 22;
  constexpr uint32_t TMA_XWIN_MAX = 8192;              // entries of a staged x window
  constexpr uint64_t TMA_SMEM_MAX = 128u * 1024u;      // dynamic shared memory of all stages

  __device__ __forceinline__ uint32_t smem_u32(const void* p)
  {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
  }

  __device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
  {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
  }

  __device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
  {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
  }

  __device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
  {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
  }

  // bounded wait for the phase with parity `par` of `bar`; false when the limit expired
  __device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t par)
  {
    const uint32_t a = smem_u32(bar);
    for(uint32_t it = 0; it < TMA_SPIN; ++it)
    {
      uint32_t ok;
      asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                   : "=r"(ok) : "r"(a), "r"(par) : "memory");
      if(ok)
        return true;
      if(it > 32)
        __nanosleep(128);
    }
    return false;
  }

  // row sum of a staged row with K entries, entry k at base + 32*k, in stored order; the column
  // is absolute or row-relative.  With a staged window sx of x[x0 .. x0 + xl), the gathers read
  // shared memory; a column outside the window is the zero slot of a padding entry (x = 0).
  // KC > 0: every row of the matrix has exactly KC slots (ELL of width KC), so the loop is fully
  // unrolled without width tests.
  template<typename V, typename S, int KC = 0>
  __device__ __forceinline__ typename ValueTraits<V>::acc staged_row_sum(const V* sv, const int16_t* sd,
    const uint32_t* sc, uint32_t K, uint32_t base, uint32_t row, const S* __restrict__ x, const S* sx,
    uint32_t x0, uint32_t xl)
  {
    typedef typename ValueTraits<V>::acc A;
    if(KC > 0)
    {
      A xv[KC > 0 ? KC : 1];
      #pragma unroll
      for(int u = 0; u < KC; ++u)
      {
        const uint32_t e = base + uint32_t(u) * 32u;
        const uint32_t c = sd ? uint32_t(int32_t(row) + int32_t(sd[e])) : sc[e];
        if(sx)
        {
          const uint32_t o = c - x0;
          xv[u] = o < xl ? A(sx[o]) : A(0);
        }
        else
          xv[u] = A(__ldg(x + c));
      }
      A s = A(0);
      #pragma unroll
      for(int u = 0; u < KC; ++u)
        s = add(s, mul(to_acc(sv[base + uint32_t(u) * 32u]), xv[u]));
      return s;
    }
    constexpr uint32_t U = 9;
    A sum = A(0);
    for(uint32_t k0 = 0; k0 < K; k0 += U)
    {
      A xv[U];
      #pragma unroll
      for(uint32_t u = 0; u < U; ++u)
        if(k0 + u < K)
        {
          const uint32_t e = base + (k0 + u) * 32u;
          const uint32_t c = sd ? uint32_t(int32_t(row) + int32_t(sd[e])) : sc[e];
          if(sx)
          {
            const uint32_t o = c - x0;
            xv[u] = o < xl ? A(sx[o]) : A(0);
          }
          else
            xv[u] = A(__ldg(x + c));
        }
      #pragma unroll
      for(uint32_t u = 0; u < U; ++u)
        if(k0 + u < K)
          sum = add(sum, mul(to_acc(sv[base + (k0 + u) * 32u]), xv[u]));
    }
    return sum;
  }

  // Shared memory bytes of one stage for a matrix of (maximum) width K with cbytes bytes of column
  // index per entry (4 absolute, 2 row-relative, 0 diagonal storage).
  template<typename V>
  __host__ __device__ __forceinline__ uint32_t tma_stage_bytes(uint32_t K, uint32_t cbytes)
  {
    return uint32_t(TMA_NT) * K * uint32_t(sizeof(V) + cbytes);
  }

  // Generic persistent pass: for every row i < A.rows, op(i, sum_i, op.pre(i)) with
  // sum_i = (A x)_i; op returns the row's contribution to an optional grid reduction, finished by
  // op.finish(total) in thread 0 of the last block.  padded_rows = the storage rows (a multiple of
  // 32); kst = the widest slice's entries per row (= A.kw for ELL), which sizes the stages.
  // xlo != null: chunk c reads only x[xlo[c] .. xlo[c] + xw) (xw a multiple of 4 entries; the range
  // ends at nxa, the entries the vector's allocation holds, at the latest).  xstage != 0: that window
  // is staged in shared memory with the chunk; xstage == 0: it is only bulk-prefetched into L2 when
  // the chunk's copies are issued, so the gathers find it there.
  // DG: diagonal storage of width KC: only the values are copied; a row's gathers x[i + doff[k]]
  // depend on no staged data, so they are issued before the wait for the chunk's copies.
  template<typename V, typename S, class Op, int KC = 0, bool DG = false>
  __global__ void __launch_bounds__(TMA_NT) k_tma_pass(DCsr<V> A, const S* __restrict__ x, uint32_t padded_rows,
    uint32_t kst, const uint32_t* __restrict__ xlo, uint32_t xw, uint32_t nxa, int xstage, Op op, RedSlot slot,
    int* err)
  {
    static_assert(!DG || KC > 0, "diagonal storage needs a fixed width");
    typedef typename ValueTraits<V>::acc Ac;
    extern __shared__ __align__(128) unsigned char tma_smem[];
    __shared__ __align__(8) uint64_t bar[TMA_STAGES];
    __shared__ double sh[32];
    constexpr int NS = tma_stages_dg<V, DG>();
    constexpr uint32_t SPC = TMA_NT / 32;   // slices per chunk
    const uint32_t K = A.kw;
    const bool narrow = A.dcol != nullptr;
    const uint32_t cbytes = DG ? 0u : (narrow ? 2u : 4u);
    int32_t doff[DG ? KC : 1];
    if(DG)
    {
      #pragma unroll
      for(int u = 0; u < (DG ? KC : 1); ++u)
        doff[u] = __ldg(A.doff + u);
    }
    const uint32_t mb = tma_stage_bytes<V>(kst, cbytes);
    const uint32_t sb = mb + (xlo && xstage ? xw * uint32_t(sizeof(S)) : 0u);
    const uint32_t nsl = padded_rows / 32u;
    const uint32_t nch = (padded_rows + TMA_NT - 1) / TMA_NT;
    auto issue = [&](uint32_t c, int s)
    {
      uint32_t e0, ne;
      if(K)
      {
        const uint32_t r0 = c * TMA_NT;
        e0 = r0 * K;
        ne = min(uint32_t(TMA_NT), padded_rows - r0) * K;
      }
      else
      {
        e0 = __ldg(A.soff + c * SPC);
        ne = __ldg(A.soff + min(c * SPC + SPC, nsl)) - e0;
      }
      const uint32_t vb = ne * uint32_t(sizeof(V));
      const uint32_t cb = ne * cbytes;
      unsigned char* st = tma_smem + size_t(s) * sb;
      uint32_t x0 = 0, xb = 0;
      if(xlo && ne)
      {
        x0 = __ldg(xlo + c);
        const uint32_t bytes = min(xw, nxa - x0) * uint32_t(sizeof(S));
        if(xstage)
          xb = bytes;
        else
          for(uint32_t o = 0; o < bytes; o += 32768u)
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;"
                         :: "l"(reinterpret_cast<const unsigned char*>(x + x0) + o), "r"(min(32768u, bytes - o))
                         : "memory");
      }
      mbar_expect_tx(&bar[s], vb + cb + xb);
      if(ne == 0)
        return;   // every row of the chunk is empty: the arrival alone completes the phase
      if(xb)
        bulk_g2s(st + mb, x + x0, xb, &bar[s]);
      bulk_g2s(st, A.val + e0, vb, &bar[s]);
      if(DG)
        ;
      else if(narrow)
        bulk_g2s(st + size_t(TMA_NT) * kst * sizeof(V), A.dcol + e0, cb, &bar[s]);
      else
        bulk_g2s(st + size_t(TMA_NT) * kst * sizeof(V), A.col + e0, cb, &bar[s]);
    };
    if(threadIdx.x == 0)
    {
      for(int s = 0; s < NS; ++s)
        mbar_init(&bar[s], 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    // the first chunks' matrix copies do not depend on the preceding kernel (the matrix is never
    // written during a solve): they go out before the wait for the predecessor; a gathered window
    // of x does, so with windows they wait
    auto issue_first = [&]()
    {
      if(threadIdx.x == 0)
        for(int s = 0; s < NS; ++s)
        {
          const uint32_t c = blockIdx.x + uint32_t(s) * gridDim.x;
          if(c < nch)
            issue(c, s);
        }
    };
    if(!xlo)
      issue_first();
    pdl_wait();
    if(xlo)
      issue_first();
    if(op.closed())
    {
      // drain the first copies (bounded) before the block exits
      if(threadIdx.x == 0)
        for(int s = 0; s < NS; ++s)
          if(blockIdx.x + uint32_t(s) * gridDim.x < nch)
            mbar_wait(&bar[s], 0u);
      return;
    }
    double part = 0.0;
    bool failed = false;
    uint32_t it = 0;
    for(uint32_t c = blockIdx.x; c < nch; c += gridDim.x, ++it)
    {
      const int s = int(it % NS);
      const uint32_t par = (it / NS) & 1u;
      const uint32_t i = c * TMA_NT + threadIdx.x;
      // diagonal storage: the row's vector entries and gathers go out before the wait
      Ac xv[DG ? KC : 1];
      typename Op::Pre dpre{};
      if(DG && i < A.rows)
      {
        dpre = op.pre(i);
        #pragma unroll
        for(int u = 0; u < (DG ? KC : 1); ++u)
        {
          const uint32_t cc = uint32_t(int32_t(i) + doff[u]);
          xv[u] = Ac(__ldg(x + (cc < A.rows ? cc : i)));
        }
      }
      // one warp polls the barrier; the others wait in __syncthreads without taking issue slots
      bool ok = true;
      if(threadIdx.x < 32)
        ok = mbar_wait(&bar[s], par);
      if(__syncthreads_or(!ok))   // the whole block leaves together
      {
        failed = true;
        break;
      }
      // every thread is past the previous chunk: refill its stage (NS - 1 chunks ahead)
      if(threadIdx.x == 0 && it > 0)
      {
        const uint32_t c2 = c - gridDim.x + uint32_t(NS) * gridDim.x;
        if(c2 < nch)
        {
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          issue(c2, int((it - 1) % NS));
        }
      }
      const unsigned char* st = tma_smem + size_t(s) * sb;
      const V* sv = reinterpret_cast<const V*>(st);
      const void* scol = st + size_t(TMA_NT) * kst * sizeof(V);
      if(DG)
      {
        if(i < A.rows)
        {
          // entries in stored order (ascending diagonals), each product and sum rounded
          const uint32_t base = (threadIdx.x >> 5) * 32u * uint32_t(KC) + (threadIdx.x & 31u);
          Ac sum = Ac(0);
          #pragma unroll
          for(int u = 0; u < (DG ? KC : 1); ++u)
            sum = add(sum, mul(to_acc(sv[base + uint32_t(u) * 32u]), xv[u]));
          part += op(i, sum, dpre);
        }
      }
      else if(i < A.rows)
      {
        // the row's own vector entries are loaded first; they do not depend on the gathers
        const typename Op::Pre pre = op.pre(i);
        uint32_t kr, base;
        if(K)
        {
          kr = K;
          base = (threadIdx.x >> 5) * 32u * K + (threadIdx.x & 31u);
        }
        else
        {
          const uint32_t sl = i >> 5;
          const uint32_t o = __ldg(A.soff + sl);
          kr = (__ldg(A.soff + sl + 1) - o) >> 5;
          base = o - __ldg(A.soff + c * SPC) + (threadIdx.x & 31u);
        }
        const S* sx = nullptr;
        uint32_t x0 = 0, xl = 0;
        if(xlo && xstage)
        {
          sx = reinterpret_cast<const S*>(st + mb);
          x0 = __ldg(xlo + c);
          xl = min(xw, nxa - x0);
        }
        const auto sum = staged_row_sum<V, S, KC>(sv, narrow ? reinterpret_cast<const int16_t*>(scol) : nullptr,
          narrow ? nullptr : reinterpret_cast<const uint32_t*>(scol), kr, base, i, x, sx, x0, xl);
        part += op(i, sum, pre);
      }
    }
    if(failed)
    {
      // record the expiry, then wait (bounded) for this block's copies still in flight; the block
      // still takes part in the grid reduction below so that its arrival counter completes
      if(threadIdx.x == 0)
      {
        atomicOr(err, 1);
        // copies in flight: chunks it .. it + NS - 1 before the first refill, then one fewer
        const uint32_t pending = it == 0 ? uint32_t(NS) : uint32_t(NS) - 1u;
        for(uint32_t k = 0; k < pending; ++k)
        {
          const uint32_t jt = it + k;
          const uint32_t c = blockIdx.x + jt * gridDim.x;
          if(c < nch)
            mbar_wait(&bar[jt % NS], (jt / NS) & 1u);
        }
      }
      __syncthreads();
    }
    // an epilogue with its own end of block (the batched solver's per-instance reductions): every
    // thread of every block that ran the loop calls it once
    if constexpr(HasBlockDone<Op>::value)
    {
      op.block_done();
      return;
    }
    if(!Op::REDUCES)
      return;
    double total;
    if(grid_sum_last<TMA_NT>(part, slot, sh, total))
      op.finish(total);
  }
} // namespace fb
