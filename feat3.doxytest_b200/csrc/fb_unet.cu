// Learned warm start: a small convolutional U-Net on vertex grids (G = 2^k + 1 points per side)
// that maps (f, log kappa) to an approximation of u, trained on solutions of the FP64 multigrid.
// No counterpart in the reference (its solve path has no learned component).
//
// Network (channels 16/32/64/64, 3x3 "same" convolutions, zero padding):
//   L1 conv 2->16 @G1, ReLU = e1;  S = injection (every other vertex)
//   L2 conv 16->32 @G2 on S(e1), ReLU = e2
//   L3 conv 32->64 @G3 on S(e2), ReLU = e3
//   L4 conv 64->64 @G4 on S(e3), then two more 64->64 convolutions @G4 with dilation 2 and 4
//      (ReLU after each) = e4: the bottleneck sees 15 x 15 of its 17 x 17 points (for G1 = 129), so
//      the prediction can couple the whole domain as the solution operator does
//   L5 conv 128->64 @G3 on [U(e4), e3], ReLU = d3;  U = bilinear vertex upsampling (the Q1
//      prolongation stencil: coincident vertex 1, edge midpoints 1/2 + 1/2, cell centres 4 x 1/4)
//   L6 conv 96->32 @G2 on [U(d3), e2], ReLU = d2
//   L7 conv 48->16 @G1 on [U(d2), e1], ReLU = d1
//   L8 conv 16->1 @G1 on d1 (no activation) = output
// Activations are stored as BF16 in NHWC layout (channels padded to multiples of 8); the
// convolutions are implicit GEMMs on the tensor cores (mma.sync m16n8k16, BF16 operands, FP32
// accumulation); bias, ReLU and the upsampling averages are computed in FP32 and rounded to BF16
// once.  Parameters are FP32 masters (Adam), converted to BF16 GEMM layouts after every update.
//
// Parameter layout (the flat FP32 vector of fb_unet_get_params): per layer, W[co][tap][ci] with
// tap = (dy+1)*3 + (dx+1) (dy along the grid's slow axis), then bias[co].
#include "fb_common.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

namespace fb
{
namespace un
{
  typedef uint16_t bf;

  __device__ __forceinline__ float bf2f(bf v) { return __uint_as_float(uint32_t(v) << 16); }
  __device__ __forceinline__ bf f2bf(float f) { return __bfloat16_as_ushort(__float2bfloat16_rn(f)); }

  constexpr int NLAYER = 10;
  struct LayerDef { int cin, cout, level; bool relu; int dil; };
  // real channel counts; level = resolution index (0 = finest grid); dil = tap spacing
  constexpr LayerDef LAYERS[NLAYER] = {
    {2, 16, 0, true, 1}, {16, 32, 1, true, 1}, {32, 64, 2, true, 1}, {64, 64, 3, true, 1}, {64, 64, 3, true, 2},
    {64, 64, 3, true, 4}, {128, 64, 2, true, 1}, {96, 32, 1, true, 1}, {48, 16, 0, true, 1}, {16, 1, 0, false, 1}};

  __host__ __device__ inline int pad8(int c) { return (c + 7) & ~7; }

  // ------------------------------------------------------------------ tensor-core helpers
  __device__ __forceinline__ uint32_t smem_addr(const void* p)
  {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
  }
  // 16-byte async copy global -> shared; src_bytes 0 fills zeros (halo / padding)
  __device__ __forceinline__ void cp16(void* dst, const void* src, int src_bytes)
  {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" :: "r"(smem_addr(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
  }
  __device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
  template<int N>
  __device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;" :: "n"(N) : "memory"); }

  __device__ __forceinline__ void ldm_x4(uint32_t (&r)[4], const void* p)
  {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(smem_addr(p)));
  }
  __device__ __forceinline__ void ldm_x4_t(uint32_t (&r)[4], const void* p)
  {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(smem_addr(p)));
  }
  __device__ __forceinline__ void ldm_x2_t(uint32_t (&r)[2], const void* p)
  {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];"
                 : "=r"(r[0]), "=r"(r[1]) : "r"(smem_addr(p)));
  }
  __device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
  {
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
  }

  // ------------------------------------------------------------------ implicit-GEMM convolution
  // y[p, n] = act(bias[n] + sum_{tap, c} x[p + off(tap), c] * w[tap*cin + c][n]) for every pixel p of
  // a B x H x W batch (x NHWC with cin channels, cin % 8 == 0; zero outside the grid).  w: kpad x
  // n_ld BF16 (rows >= 9*cin are zero, kpad % 32 == 0).  Output BF16 or FP32 at [p * y_ld + y_off].
  // The same kernel computes the data gradient (x = output gradient, w = flipped transposed weights).
  struct ConvArgs
  {
    const bf* x;
    const bf* w;
    const float* bias;     // nb entries (columns >= nb get no bias)
    void* y;
    int cin, kpad, n, n_ld, nb;
    int B, H, W, dil;
    int y_ld, y_off;
    int relu, out_bf16;
  };

  constexpr int CBM = 128, CBK = 32, CNT = 128;

  template<int BN>
  __global__ void __launch_bounds__(CNT) k_conv(const ConvArgs a)
  {
    constexpr int AST = CBK + 8;          // A row stride (elements): 80 bytes, conflict-free ldmatrix
    constexpr int BST = BN + 8;
    constexpr int NT8 = BN / 8;
    __shared__ __align__(16) bf As[2][CBM * AST];
    __shared__ __align__(16) bf Bs[2][CBK * BST];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int P = a.B * a.H * a.W;
    const int m0 = blockIdx.x * CBM;
    const int n0 = blockIdx.y * BN;
    // this thread's A row (one pixel)
    const int pm = m0 + tid;
    const bool prow = pm < P;
    int pb = 0, py = 0, px = 0;
    if(prow)
    {
      px = pm % a.W;
      const int t = pm / a.W;
      py = t % a.H;
      pb = t / a.H;
    }
    const int K9 = 9 * a.cin;
    auto load = [&](int kt, int buf)
    {
      const int k0 = kt * CBK;
      #pragma unroll
      for(int c = 0; c < CBK / 8; ++c)
      {
        const int k = k0 + c * 8;
        const bf* src = a.x;
        int bytes = 0;
        if(prow && k < K9)
        {
          const int tap = k / a.cin, ci = k - tap * a.cin;
          const int yy = py + (tap / 3 - 1) * a.dil, xx = px + (tap % 3 - 1) * a.dil;
          if(yy >= 0 && yy < a.H && xx >= 0 && xx < a.W)
          {
            src = a.x + ((size_t(pb) * a.H + yy) * a.W + xx) * a.cin + ci;
            bytes = 16;
          }
        }
        cp16(&As[buf][tid * AST + c * 8], src, bytes);
      }
      constexpr int BCH = CBK * BN / 8;   // 16-byte chunks of the B tile
      for(int q = tid; q < BCH; q += CNT)
      {
        const int r = q / (BN / 8), c = q % (BN / 8);
        const int col = n0 + c * 8;
        const bf* src = a.w;
        int bytes = 0;
        if(col < a.n_ld)
        {
          src = a.w + size_t(k0 + r) * a.n_ld + col;
          bytes = 16;
        }
        cp16(&Bs[buf][r * BST + c * 8], src, bytes);
      }
    };
    float acc[2][NT8][4];
    #pragma unroll
    for(int i = 0; i < 2; ++i)
      #pragma unroll
      for(int j = 0; j < NT8; ++j)
        #pragma unroll
        for(int e = 0; e < 4; ++e)
          acc[i][j][e] = 0.f;
    const int nk = a.kpad / CBK;
    load(0, 0);
    cp_commit();
    for(int kt = 0; kt < nk; ++kt)
    {
      const int buf = kt & 1;
      if(kt + 1 < nk)
        load(kt + 1, buf ^ 1);
      cp_commit();
      cp_wait<1>();
      __syncthreads();
      #pragma unroll
      for(int kk = 0; kk < CBK; kk += 16)
      {
        uint32_t af[2][4];
        #pragma unroll
        for(int mt = 0; mt < 2; ++mt)
          ldm_x4(af[mt], &As[buf][(warp * 32 + mt * 16 + (lane & 15)) * AST + kk + (lane >> 4) * 8]);
        #pragma unroll
        for(int nt = 0; nt < NT8; nt += 2)
        {
          if(nt + 1 < NT8)
          {
            uint32_t bfr[4];
            ldm_x4_t(bfr, &Bs[buf][(kk + (lane & 15)) * BST + nt * 8 + (lane >> 4) * 8]);
            #pragma unroll
            for(int mt = 0; mt < 2; ++mt)
            {
              mma16816(acc[mt][nt], af[mt], bfr[0], bfr[1]);
              mma16816(acc[mt][nt + 1], af[mt], bfr[2], bfr[3]);
            }
          }
          else
          {
            uint32_t bfr[2];
            ldm_x2_t(bfr, &Bs[buf][(kk + (lane & 15)) * BST + nt * 8]);
            #pragma unroll
            for(int mt = 0; mt < 2; ++mt)
              mma16816(acc[mt][nt], af[mt], bfr[0], bfr[1]);
          }
        }
      }
      __syncthreads();
    }
    // epilogue: bias, activation, store
    const int g = lane >> 2, tg = lane & 3;
    #pragma unroll
    for(int mt = 0; mt < 2; ++mt)
      #pragma unroll
      for(int h = 0; h < 2; ++h)
      {
        const int row = m0 + warp * 32 + mt * 16 + g + h * 8;
        if(row >= P)
          continue;
        #pragma unroll
        for(int nt = 0; nt < NT8; ++nt)
        {
          const int col = n0 + nt * 8 + tg * 2;
          if(col >= a.n)
            continue;
          float v0 = acc[mt][nt][h * 2 + 0], v1 = acc[mt][nt][h * 2 + 1];
          if(a.bias)
          {
            v0 += col < a.nb ? a.bias[col] : 0.f;
            v1 += col + 1 < a.nb ? a.bias[col + 1] : 0.f;
          }
          if(a.relu)
          {
            v0 = fmaxf(v0, 0.f);
            v1 = fmaxf(v1, 0.f);
          }
          const size_t o = size_t(row) * a.y_ld + a.y_off + col;
          if(a.out_bf16)
          {
            bf* y = static_cast<bf*>(a.y);
            const uint32_t pk = uint32_t(f2bf(v0)) | (uint32_t(f2bf(v1)) << 16);
            *reinterpret_cast<uint32_t*>(y + o) = pk;
          }
          else
          {
            float* y = static_cast<float*>(a.y);
            *reinterpret_cast<float2*>(y + o) = make_float2(v0, v1);
          }
        }
      }
  }

  // ------------------------------------------------------------------ weight gradient
  // part[s][m][j] = sum over the pixels of split s of dy[p, m] * x[p + off(tap_j), c_j] with
  // j = tap*cin + c: M = cout (dy channels, padded to BM), N = 9*cin, K = pixels.
  struct WgradArgs
  {
    const bf* dy;        // [P][m_ld]
    const bf* x;         // [P][cin]
    float* part;         // [splits][m][n] (m < m_real, n < 9*cin)
    int m_ld, m_real, cin;
    int B, H, W, dil;
    int pix_per_split;
  };

  constexpr int WBN = 64, WBK = 32, WNT = 128;

  template<int BM>
  __global__ void __launch_bounds__(WNT) k_wgrad(const WgradArgs a)
  {
    constexpr int AST = BM + 8;     // A stored K-major: [k][m]
    constexpr int BST = WBN + 8;    // B stored [k][n]
    constexpr int MT = BM / 16;
    __shared__ __align__(16) bf As[2][WBK * AST];
    __shared__ __align__(16) bf Bs[2][WBK * BST];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int P = a.B * a.H * a.W;
    const int N9 = 9 * a.cin;
    const int n0 = blockIdx.x * WBN;
    const int p_begin = blockIdx.y * a.pix_per_split;
    const int p_end = min(P, p_begin + a.pix_per_split);
    auto load = [&](int p0, int buf)
    {
      // A: WBK pixels x BM channels of dy
      for(int q = tid; q < WBK * (BM / 8); q += WNT)
      {
        const int r = q / (BM / 8), c = q % (BM / 8);
        const int p = p0 + r;
        const bf* src = a.dy;
        int bytes = 0;
        if(p < p_end && c * 8 < a.m_ld)
        {
          src = a.dy + size_t(p) * a.m_ld + c * 8;
          bytes = 16;
        }
        cp16(&As[buf][r * AST + c * 8], src, bytes);
      }
      // B: WBK pixels x WBN columns of im2col(x)
      for(int q = tid; q < WBK * (WBN / 8); q += WNT)
      {
        const int r = q / (WBN / 8), c = q % (WBN / 8);
        const int p = p0 + r;
        const int j = n0 + c * 8;
        const bf* src = a.x;
        int bytes = 0;
        if(p < p_end && j < N9)
        {
          const int tap = j / a.cin, ci = j - tap * a.cin;
          const int px = p % a.W, t = p / a.W;
          const int py = t % a.H, pb = t / a.H;
          const int yy = py + (tap / 3 - 1) * a.dil, xx = px + (tap % 3 - 1) * a.dil;
          if(yy >= 0 && yy < a.H && xx >= 0 && xx < a.W)
          {
            src = a.x + ((size_t(pb) * a.H + yy) * a.W + xx) * a.cin + ci;
            bytes = 16;
          }
        }
        cp16(&Bs[buf][r * BST + c * 8], src, bytes);
      }
    };
    float acc[MT][2][4];
    #pragma unroll
    for(int i = 0; i < MT; ++i)
      #pragma unroll
      for(int j = 0; j < 2; ++j)
        #pragma unroll
        for(int e = 0; e < 4; ++e)
          acc[i][j][e] = 0.f;
    const int nk = (p_end - p_begin + WBK - 1) / WBK;
    if(nk > 0)
    {
      load(p_begin, 0);
      cp_commit();
    }
    for(int kt = 0; kt < nk; ++kt)
    {
      const int buf = kt & 1;
      if(kt + 1 < nk)
        load(p_begin + (kt + 1) * WBK, buf ^ 1);
      cp_commit();
      cp_wait<1>();
      __syncthreads();
      #pragma unroll
      for(int kk = 0; kk < WBK; kk += 16)
      {
        // B fragments of this warp's 16 columns (two n8 tiles)
        uint32_t bfr[4];
        ldm_x4_t(bfr, &Bs[buf][(kk + (lane & 15)) * BST + warp * 16 + (lane >> 4) * 8]);
        #pragma unroll
        for(int mt = 0; mt < MT; ++mt)
        {
          // A (m x k) from the K-major tile: matrix j covers m-rows (j&1)*8, k-cols (j>>1)*8
          uint32_t af[4];
          const int j = lane >> 3, i = lane & 7;
          ldm_x4_t(af, &As[buf][(kk + (j >> 1) * 8 + i) * AST + mt * 16 + (j & 1) * 8]);
          mma16816(acc[mt][0], af, bfr[0], bfr[1]);
          mma16816(acc[mt][1], af, bfr[2], bfr[3]);
        }
      }
      __syncthreads();
    }
    const int g = lane >> 2, tg = lane & 3;
    float* out = a.part + size_t(blockIdx.y) * a.m_real * N9;
    #pragma unroll
    for(int mt = 0; mt < MT; ++mt)
      #pragma unroll
      for(int h = 0; h < 2; ++h)
      {
        const int m = mt * 16 + g + h * 8;
        if(m >= a.m_real)
          continue;
        #pragma unroll
        for(int nt = 0; nt < 2; ++nt)
        {
          const int n = n0 + warp * 16 + nt * 8 + tg * 2;
          if(n < N9)
            out[size_t(m) * N9 + n] = acc[mt][nt][h * 2 + 0];
          if(n + 1 < N9)
            out[size_t(m) * N9 + n + 1] = acc[mt][nt][h * 2 + 1];
        }
      }
  }

  // grad W[co][tap][ci] (real channels) = sum over splits of part[s][co][tap*cin_pad + ci], in split
  // order; grad b[co] = sum_p dy[p, co] (per-block partial sums, then a fixed-order sum)
  __global__ void k_wgrad_reduce(const float* __restrict__ part, int splits, int m_real, int cin_pad, int cin_real,
    float* __restrict__ gw, int accumulate)
  {
    const int N9 = 9 * cin_pad;
    const int total = m_real * 9 * cin_real;
    for(int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x)
    {
      const int ci = e % cin_real, t = e / cin_real;
      const int tap = t % 9, co = t / 9;
      const size_t j = size_t(co) * N9 + tap * cin_pad + ci;
      float s = 0.f;
      for(int k = 0; k < splits; ++k)
        s += part[size_t(k) * m_real * N9 + j];
      gw[e] = accumulate ? gw[e] + s : s;
    }
  }

  constexpr int BG_NT = 256;
  __global__ void __launch_bounds__(BG_NT) k_bgrad_part(const bf* __restrict__ dy, int P, int ld, int m_real,
    int pix_per_block, float* __restrict__ part)
  {
    // block b sums pixels [b*ppb, (b+1)*ppb) for every channel; threads: channel-major groups
    __shared__ float sh[BG_NT];
    const int p0 = blockIdx.x * pix_per_block, p1 = min(P, p0 + pix_per_block);
    const int groups = BG_NT / 64;   // 64 channels max per pass
    const int c = threadIdx.x % 64, gsub = threadIdx.x / 64;
    float s = 0.f;
    if(c < m_real)
      for(int p = p0 + gsub; p < p1; p += groups)
        s += bf2f(dy[size_t(p) * ld + c]);
    sh[threadIdx.x] = s;
    __syncthreads();
    if(threadIdx.x < 64 && c < m_real)
    {
      float t = 0.f;
      for(int k = 0; k < groups; ++k)
        t += sh[k * 64 + c];
      part[size_t(blockIdx.x) * m_real + c] = t;
    }
  }

  __global__ void k_bgrad_reduce(const float* __restrict__ part, int nblk, int m_real, float* __restrict__ gb,
    int accumulate)
  {
    const int c = threadIdx.x;
    if(c >= m_real)
      return;
    float s = 0.f;
    for(int k = 0; k < nblk; ++k)
      s += part[size_t(k) * m_real + c];
    gb[c] = accumulate ? gb[c] + s : s;
  }

  // ------------------------------------------------------------------ grid transfers and packing
  // NCHW FP32 input (2 channels) -> NHWC BF16 with 8 channels (6 zero)
  __global__ void k_pack_input(const float* __restrict__ in, int B, int G, bf* __restrict__ x)
  {
    const size_t n = size_t(B) * G * G;
    for(size_t p = blockIdx.x * size_t(blockDim.x) + threadIdx.x; p < n; p += size_t(gridDim.x) * blockDim.x)
    {
      const size_t b = p / (size_t(G) * G), r = p % (size_t(G) * G);
      uint32_t w[4] = {0u, 0u, 0u, 0u};
      w[0] = uint32_t(f2bf(in[(b * 2 + 0) * G * G + r])) | (uint32_t(f2bf(in[(b * 2 + 1) * G * G + r])) << 16);
      *reinterpret_cast<uint4*>(x + p * 8) = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }

  // injection: coarse (i, j) = fine (2i, 2j); C channels, 8 at a time
  __global__ void k_subsample(const bf* __restrict__ f, int B, int Gf, int C, bf* __restrict__ c)
  {
    const int Gc = (Gf + 1) / 2, C8 = C / 8;
    const size_t n = size_t(B) * Gc * Gc * C8;
    for(size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x)
    {
      const int ch = int(e % C8);
      const size_t p = e / C8;
      const int x = int(p % Gc), y = int((p / Gc) % Gc);
      const size_t b = p / (size_t(Gc) * Gc);
      const size_t src = ((b * Gf + 2 * y) * Gf + 2 * x) * C + ch * 8;
      *reinterpret_cast<uint4*>(c + p * C + ch * 8) = *reinterpret_cast<const uint4*>(f + src);
    }
  }

  // out[:, :, :, 0:Cu] = U(coarse) (bilinear vertex upsampling, FP32 average rounded once),
  // out[:, :, :, Cu:Cu+Cs] = skip
  __global__ void k_upsample_cat(const bf* __restrict__ coarse, int Cu, const bf* __restrict__ skip, int Cs, int B,
    int Gf, bf* __restrict__ out)
  {
    const int Gc = (Gf + 1) / 2, Ct = Cu + Cs;
    const size_t n = size_t(B) * Gf * Gf * Ct;
    for(size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x)
    {
      const int ch = int(e % Ct);
      const size_t p = e / Ct;
      const int x = int(p % Gf), y = int((p / Gf) % Gf);
      const size_t b = p / (size_t(Gf) * Gf);
      bf v;
      if(ch >= Cu)
        v = skip[p * Cs + (ch - Cu)];
      else
      {
        const int y0 = y >> 1, x0 = x >> 1, y1 = y0 + (y & 1), x1 = x0 + (x & 1);
        const bf* cb = coarse + b * size_t(Gc) * Gc * Cu + ch;
        const float a00 = bf2f(cb[(size_t(y0) * Gc + x0) * Cu]);
        const float a01 = bf2f(cb[(size_t(y0) * Gc + x1) * Cu]);
        const float a10 = bf2f(cb[(size_t(y1) * Gc + x0) * Cu]);
        const float a11 = bf2f(cb[(size_t(y1) * Gc + x1) * Cu]);
        v = f2bf(((a00 + a01) + (a10 + a11)) * 0.25f);
      }
      out[e] = v;
    }
  }

  // adjoint of U for channel range [c0, c0+C) of a fine gradient (FP32, row stride ld):
  // gc(i, j) = sum_{dy,dx in -1..1} w(dy) w(dx) gf(2i+dy, 2j+dx) (in-grid points), w(0) = 1,
  // w(+-1) = 1/2; the four corner products of a cell centre carry 1/4 each.  Then dpre = mask(post)
  // * gc as BF16 ([B][Gc][Gc][C]).
  __global__ void k_upsample_bwd_mask(const float* __restrict__ gf, int ld, int c0, int C, int B, int Gf,
    const bf* __restrict__ post, bf* __restrict__ dpre)
  {
    const int Gc = (Gf + 1) / 2;
    const size_t n = size_t(B) * Gc * Gc * C;
    for(size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x)
    {
      const int ch = int(e % C);
      const size_t p = e / C;
      const int x = int(p % Gc), y = int((p / Gc) % Gc);
      const size_t b = p / (size_t(Gc) * Gc);
      float s = 0.f;
      for(int dy = -1; dy <= 1; ++dy)
      {
        const int yf = 2 * y + dy;
        if(yf < 0 || yf >= Gf)
          continue;
        for(int dx = -1; dx <= 1; ++dx)
        {
          const int xf = 2 * x + dx;
          if(xf < 0 || xf >= Gf)
            continue;
          const float w = (dy == 0 ? 1.f : 0.5f) * (dx == 0 ? 1.f : 0.5f);
          s += w * gf[((b * Gf + yf) * Gf + xf) * ld + c0 + ch];
        }
      }
      dpre[e] = f2bf(bf2f(post[e]) > 0.f ? s : 0.f);
    }
  }

  // dpre = mask(post) * (g1[p, c1+c] (optional) + (even-even p ? g2[p/2 coarse, c] : 0) (optional))
  __global__ void k_grad_mask(const bf* __restrict__ post, int C, int B, int G, const float* __restrict__ g1, int ld1,
    int c1, const float* __restrict__ g2, int ld2, bf* __restrict__ dpre)
  {
    const int Gc = (G + 1) / 2;
    const size_t n = size_t(B) * G * G * C;
    for(size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x)
    {
      const int ch = int(e % C);
      const size_t p = e / C;
      float s = 0.f;
      if(g1)
        s += g1[p * ld1 + c1 + ch];
      if(g2)
      {
        const int x = int(p % G), y = int((p / G) % G);
        if(!(x & 1) && !(y & 1))
        {
          const size_t b = p / (size_t(G) * G);
          s += g2[((b * Gc + y / 2) * Gc + x / 2) * ld2 + ch];
        }
      }
      dpre[e] = f2bf(bf2f(post[e]) > 0.f ? s : 0.f);
    }
  }

  // output gradient (FP32 [B][G][G]) -> BF16 [P][8], channel 0
  __global__ void k_pack_dout(const float* __restrict__ g, size_t P, bf* __restrict__ dy)
  {
    for(size_t p = blockIdx.x * size_t(blockDim.x) + threadIdx.x; p < P; p += size_t(gridDim.x) * blockDim.x)
      *reinterpret_cast<uint4*>(dy + p * 8) = make_uint4(uint32_t(f2bf(g[p])), 0u, 0u, 0u);
  }

  // output [P][8] FP32 channel 0 -> [B][G][G]
  __global__ void k_unpack_out(const float* __restrict__ y, size_t P, float* __restrict__ out)
  {
    for(size_t p = blockIdx.x * size_t(blockDim.x) + threadIdx.x; p < P; p += size_t(gridDim.x) * blockDim.x)
      out[p] = y[p * 8];
  }

  // FP32 master -> BF16 GEMM layouts: forward wf[tap*cin_pad + ci][co] (kpad x cout_pad) and data
  // gradient wd[t*cout_pad + co][ci] = W[co][8-t][ci] (kpad_d x cin_pad)
  __global__ void k_prep_weights(const float* __restrict__ W, int cin, int cout, int cin_pad, int cout_pad, int kpad,
    int kpad_d, bf* __restrict__ wf, bf* __restrict__ wd)
  {
    const int nf = kpad * cout_pad, nd = kpad_d * cin_pad;
    for(int e = blockIdx.x * blockDim.x + threadIdx.x; e < nf + nd; e += gridDim.x * blockDim.x)
    {
      if(e < nf)
      {
        const int co = e % cout_pad, k = e / cout_pad;
        const int tap = k / cin_pad, ci = k % cin_pad;
        float v = 0.f;
        if(tap < 9 && ci < cin && co < cout)
          v = W[(co * 9 + tap) * cin + ci];
        wf[e] = f2bf(v);
      }
      else if(wd)
      {
        const int f = e - nf;
        const int ci = f % cin_pad, k = f / cin_pad;
        const int t = k / cout_pad, co = k % cout_pad;
        float v = 0.f;
        if(t < 9 && ci < cin && co < cout)
          v = W[(co * 9 + (8 - t)) * cin + ci];
        wd[f] = f2bf(v);
      }
    }
  }

  // Adam (Kingma & Ba 2015, Algorithm 1) on the FP32 masters
  __global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
    size_t n, float lr, float b1, float b2, float eps, float c1, float c2)
  {
    for(size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    {
      const float gi = g[i];
      const float mi = b1 * m[i] + (1.f - b1) * gi;
      const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
      m[i] = mi;
      v[i] = vi;
      p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
  }

  // loss = sum (y - t)^2 / n over [n]; grad = 2 (y - t) / n (per-block partials, fixed-order sum)
  constexpr int MSE_NT = 256;
  __global__ void __launch_bounds__(MSE_NT) k_mse(const float* __restrict__ y, const float* __restrict__ t, size_t n,
    float* __restrict__ grad, double* __restrict__ part)
  {
    __shared__ double sh[32];
    double s = 0.0;
    const float inv = 1.f / float(n);
    for(size_t i = blockIdx.x * size_t(MSE_NT) + threadIdx.x; i < n; i += size_t(gridDim.x) * MSE_NT)
    {
      const float d = y[i] - t[i];
      if(grad)
        grad[i] = 2.f * d * inv;
      s += double(d) * double(d);
    }
    const double tot = block_sum<MSE_NT>(s, sh);
    if(threadIdx.x == 0)
      part[blockIdx.x] = tot;
  }
  __global__ void k_mse_final(const double* __restrict__ part, int nb, size_t n, double* __restrict__ loss)
  {
    double s = 0.0;
    for(int k = 0; k < nb; ++k)
      s += part[k];
    *loss = s / double(n);
  }
} // namespace un
} // namespace fb

using namespace fb;
using namespace fb::un;

struct fb_unet
{
  int G[4] = {0, 0, 0, 0};
  int max_batch = 0;
  size_t nparam = 0;
  size_t woff[NLAYER], boff[NLAYER];
  int cin_pad[NLAYER], cout_pad[NLAYER], kpad[NLAYER], kpad_d[NLAYER];
  std::vector<void*> allocs;
  float *param = nullptr, *grad = nullptr, *adam_m = nullptr, *adam_v = nullptr;
  bf* wf[NLAYER] = {};
  bf* wd[NLAYER] = {};
  // activations (BF16 NHWC): x8 (input), e1..e4, s1..s3, c3, c2, c1, d3, d2, d1
  bf *x8 = nullptr, *e[4] = {}, *s[3] = {}, *c[3] = {}, *d[3] = {};
  bf* b4[2] = {};              // bottleneck: outputs of the dilation-2 and dilation-4 convolutions
  float* yout = nullptr;       // [P1][8] FP32 pre-activation output of L8
  // backward scratch: BF16 output gradient and pre-activation gradient (one layer at a time);
  // FP32 data gradients of the concatenated inputs (dc1 @G1 48 ch, dc2 @G2 96, dc3 @G3 128) and of
  // the other inputs (gs: d1, then s3, s2, s1 in turn)
  bf *dy8 = nullptr, *dpre = nullptr;
  float* dc[3] = {};
  float* gs = nullptr;
  float* wpart = nullptr;
  size_t wpart_n = 0;
  float* bpart = nullptr;
  size_t bpart_n = 0;
  double* mse_part = nullptr;
  double* mse_loss = nullptr;
  bool weights_ready = false;
};

namespace
{
  fb_status ualloc(fb_unet* u, void** p, size_t bytes)
  {
    FB_CUDA(cudaMalloc(p, std::max<size_t>(bytes, 256)));
    u->allocs.push_back(*p);
    return FB_OK;
  }
#define UN_TRY(x)                      \
  do {                                 \
    fb_status t_ = (x);                \
    if(t_ != FB_OK) return t_;         \
  } while(0)

  unsigned grid_for(size_t n, int nt = 256)
  {
    return unsigned(std::min<size_t>(std::max<size_t>((n + nt - 1) / nt, 1), 148 * 16));
  }

  fb_status prep_weights(fb_unet* u, cudaStream_t st)
  {
    for(int l = 0; l < NLAYER; ++l)
    {
      const LayerDef& L = LAYERS[l];
      const int nf = u->kpad[l] * u->cout_pad[l] + (u->wd[l] ? u->kpad_d[l] * u->cin_pad[l] : 0);
      k_prep_weights<<<grid_for(size_t(nf)), 256, 0, st>>>(u->param + u->woff[l], L.cin, L.cout, u->cin_pad[l],
        u->cout_pad[l], u->kpad[l], u->kpad_d[l], u->wf[l], u->wd[l]);
    }
    FB_LAUNCHED(NLAYER);
    u->weights_ready = true;
    return FB_OK;
  }

  // y = conv(x) of layer l at grid G (B images); bf16 output with ReLU or FP32 without
  fb_status conv_fwd(fb_unet* u, int l, const bf* x, int B, int G, void* y, int y_ld, bool out_bf16, bool relu,
    cudaStream_t st)
  {
    ConvArgs a;
    a.x = x;
    a.w = u->wf[l];
    a.bias = u->param + u->boff[l];
    a.y = y;
    a.cin = u->cin_pad[l];
    a.kpad = u->kpad[l];
    a.n = u->cout_pad[l];
    a.n_ld = u->cout_pad[l];
    a.nb = LAYERS[l].cout;
    a.B = B;
    a.dil = LAYERS[l].dil;
    a.H = G;
    a.W = G;
    a.y_ld = y_ld;
    a.y_off = 0;
    a.relu = relu ? 1 : 0;
    a.out_bf16 = out_bf16 ? 1 : 0;
    const int P = B * G * G;
    const int bn = std::min(64, a.n);
    dim3 grid((P + CBM - 1) / CBM, (a.n + bn - 1) / bn);
    switch(bn)
    {
      case 8: k_conv<8><<<grid, CNT, 0, st>>>(a); break;
      case 16: k_conv<16><<<grid, CNT, 0, st>>>(a); break;
      case 32: k_conv<32><<<grid, CNT, 0, st>>>(a); break;
      default: k_conv<64><<<grid, CNT, 0, st>>>(a); break;
    }
    FB_LAUNCHED(1);
    return FB_OK;
  }

  // data gradient of layer l: gx[p][ci] (FP32, ci < cin_pad) from dpre [P][cout_pad]
  fb_status conv_bwd_data(fb_unet* u, int l, const bf* dpre, int B, int G, float* gx, cudaStream_t st)
  {
    ConvArgs a;
    a.x = dpre;
    a.w = u->wd[l];
    a.bias = nullptr;
    a.y = gx;
    a.cin = u->cout_pad[l];
    a.kpad = u->kpad_d[l];
    a.n = u->cin_pad[l];
    a.n_ld = u->cin_pad[l];
    a.nb = 0;
    a.B = B;
    a.dil = LAYERS[l].dil;
    a.H = G;
    a.W = G;
    a.y_ld = u->cin_pad[l];
    a.y_off = 0;
    a.relu = 0;
    a.out_bf16 = 0;
    const int P = B * G * G;
    const int bn = std::min(64, a.n);
    dim3 grid((P + CBM - 1) / CBM, (a.n + bn - 1) / bn);
    switch(bn)
    {
      case 8: k_conv<8><<<grid, CNT, 0, st>>>(a); break;
      case 16: k_conv<16><<<grid, CNT, 0, st>>>(a); break;
      case 32: k_conv<32><<<grid, CNT, 0, st>>>(a); break;
      default: k_conv<64><<<grid, CNT, 0, st>>>(a); break;
    }
    FB_LAUNCHED(1);
    return FB_OK;
  }

  // weight and bias gradients of layer l from dpre [P][cout_pad] and its input x [P][cin_pad]
  fb_status conv_bwd_weight(fb_unet* u, int l, const bf* dpre, const bf* x, int B, int G, int acc, cudaStream_t st)
  {
    const LayerDef& L = LAYERS[l];
    const int P = B * G * G;
    const int N9 = 9 * u->cin_pad[l];
    const int ntile = (N9 + WBN - 1) / WBN;
    // splits: about 4 waves of 148 SMs, at least 64 pixels each
    int splits = std::max(1, std::min((148 * 8) / ntile, (P + 63) / 64));
    const int pps = ((P + splits - 1) / splits + WBK - 1) / WBK * WBK;
    splits = (P + pps - 1) / pps;
    const size_t need = size_t(splits) * L.cout * N9;
    if(need > u->wpart_n)
    {
      set_error("unet: weight-gradient scratch too small");
      return FB_ERR_STATE;
    }
    WgradArgs a;
    a.dy = dpre;
    a.x = x;
    a.part = u->wpart;
    a.m_ld = u->cout_pad[l];
    a.m_real = L.cout;
    a.cin = u->cin_pad[l];
    a.B = B;
    a.H = G;
    a.W = G;
    a.dil = L.dil;
    a.pix_per_split = pps;
    dim3 grid(ntile, splits);
    const int bm = u->cout_pad[l] <= 16 ? 16 : (u->cout_pad[l] <= 32 ? 32 : 64);
    switch(bm)
    {
      case 16: k_wgrad<16><<<grid, WNT, 0, st>>>(a); break;
      case 32: k_wgrad<32><<<grid, WNT, 0, st>>>(a); break;
      default: k_wgrad<64><<<grid, WNT, 0, st>>>(a); break;
    }
    const int tot = L.cout * 9 * L.cin;
    k_wgrad_reduce<<<grid_for(size_t(tot)), 256, 0, st>>>(u->wpart, splits, L.cout, u->cin_pad[l], L.cin,
      u->grad + u->woff[l], acc);
    const int ppb = 2048;
    const int nblk = (P + ppb - 1) / ppb;
    if(size_t(nblk) * L.cout > u->bpart_n)
    {
      set_error("unet: bias-gradient scratch too small");
      return FB_ERR_STATE;
    }
    k_bgrad_part<<<nblk, BG_NT, 0, st>>>(dpre, P, u->cout_pad[l], L.cout, ppb, u->bpart);
    k_bgrad_reduce<<<1, 64, 0, st>>>(u->bpart, nblk, L.cout, u->grad + u->boff[l], acc);
    FB_LAUNCHED(4);
    return FB_OK;
  }
} // namespace

extern "C" {

fb_status fb_unet_create(fb_unet** out, int grid, int max_batch)
{
  if(!out || max_batch < 1 || grid < 9 || ((grid - 1) & 7) != 0 || ((grid - 1) & (grid - 2)) != 0)
  {
    set_error("unet_create: grid must be 2^k + 1 (k >= 3), max_batch >= 1");
    return FB_ERR_ARG;
  }
  std::unique_ptr<fb_unet> u(new fb_unet());
  u->max_batch = max_batch;
  u->G[0] = grid;
  for(int i = 1; i < 4; ++i)
    u->G[i] = (u->G[i - 1] + 1) / 2;
  size_t off = 0;
  for(int l = 0; l < NLAYER; ++l)
  {
    const LayerDef& L = LAYERS[l];
    u->woff[l] = off;
    off += size_t(L.cout) * 9 * L.cin;
    u->boff[l] = off;
    off += size_t(L.cout);
    u->cin_pad[l] = pad8(L.cin);
    u->cout_pad[l] = pad8(L.cout);
    u->kpad[l] = (9 * u->cin_pad[l] + CBK - 1) / CBK * CBK;
    u->kpad_d[l] = (9 * u->cout_pad[l] + CBK - 1) / CBK * CBK;
  }
  u->nparam = off;
  fb_unet* p = u.get();
  auto fail = [&](fb_status e) { for(void* a : p->allocs) cudaFree(a); return e; };
  fb_status e;
#define UN_A(ptr, bytes) do { e = ualloc(p, (void**)&(ptr), (bytes)); if(e != FB_OK) return fail(e); } while(0)
  UN_A(p->param, sizeof(float) * off);
  UN_A(p->grad, sizeof(float) * off);
  UN_A(p->adam_m, sizeof(float) * off);
  UN_A(p->adam_v, sizeof(float) * off);
  FB_CUDA(cudaMemset(p->param, 0, sizeof(float) * off));
  FB_CUDA(cudaMemset(p->grad, 0, sizeof(float) * off));
  FB_CUDA(cudaMemset(p->adam_m, 0, sizeof(float) * off));
  FB_CUDA(cudaMemset(p->adam_v, 0, sizeof(float) * off));
  for(int l = 0; l < NLAYER; ++l)
  {
    UN_A(p->wf[l], sizeof(bf) * p->kpad[l] * p->cout_pad[l]);
    if(l > 0)
      UN_A(p->wd[l], sizeof(bf) * p->kpad_d[l] * p->cin_pad[l]);
  }
  const size_t B = size_t(max_batch);
  auto pix = [&](int lv) { return B * size_t(p->G[lv]) * p->G[lv]; };
  UN_A(p->x8, sizeof(bf) * pix(0) * 8);
  const int ech[4] = {16, 32, 64, 64};
  for(int i = 0; i < 4; ++i)
    UN_A(p->e[i], sizeof(bf) * pix(i) * ech[i]);
  for(int i = 0; i < 3; ++i)
    UN_A(p->s[i], sizeof(bf) * pix(i + 1) * ech[i]);
  for(int i = 0; i < 2; ++i)
    UN_A(p->b4[i], sizeof(bf) * pix(3) * 64);
  // c[0] = [U(d2), e1] @G1 (48), c[1] = [U(d3), e2] @G2 (96), c[2] = [U(e4), e3] @G3 (128)
  UN_A(p->c[0], sizeof(bf) * pix(0) * 48);
  UN_A(p->c[1], sizeof(bf) * pix(1) * 96);
  UN_A(p->c[2], sizeof(bf) * pix(2) * 128);
  // d[0] = d1 @G1 (16), d[1] = d2 @G2 (32), d[2] = d3 @G3 (64)
  UN_A(p->d[0], sizeof(bf) * pix(0) * 16);
  UN_A(p->d[1], sizeof(bf) * pix(1) * 32);
  UN_A(p->d[2], sizeof(bf) * pix(2) * 64);
  UN_A(p->yout, sizeof(float) * pix(0) * 8);
  UN_A(p->dy8, sizeof(bf) * pix(0) * 8);
  // largest dpre: G1 x 16 or G2 x 32 or G3 x 64 channels
  size_t dmax = std::max(std::max(pix(0) * 16, pix(1) * 32), std::max(pix(2) * 64, pix(3) * 64));
  UN_A(p->dpre, sizeof(bf) * dmax);
  UN_A(p->dc[0], sizeof(float) * pix(0) * 48);
  UN_A(p->dc[1], sizeof(float) * pix(1) * 96);
  UN_A(p->dc[2], sizeof(float) * pix(2) * 128);
  UN_A(p->gs, sizeof(float) * std::max(std::max(pix(0) * 16, pix(3) * 64), std::max(pix(2) * 32, pix(1) * 16)));
  p->wpart_n = size_t(148) * 8 * 64 * WBN;   // splits * cout * 9 cin_pad <= (1184 / ntile) * 64 * ntile * WBN
  UN_A(p->wpart, sizeof(float) * p->wpart_n);
  p->bpart_n = (pix(0) + 2047) / 2048 * 64 + 64;
  UN_A(p->bpart, sizeof(float) * p->bpart_n);
  UN_A(p->mse_part, sizeof(double) * 1024);
  UN_A(p->mse_loss, sizeof(double));
#undef UN_A
  *out = u.release();
  return FB_OK;
}

void fb_unet_destroy(fb_unet* u)
{
  if(!u)
    return;
  for(void* a : u->allocs)
    cudaFree(a);
  delete u;
}

fb_status fb_unet_num_params(const fb_unet* u, uint64_t* n)
{
  if(!u || !n)
  {
    set_error("unet_num_params: bad arguments");
    return FB_ERR_ARG;
  }
  *n = u->nparam;
  return FB_OK;
}

fb_status fb_unet_set_params(fb_unet* u, const float* host)
{
  if(!u || !host)
  {
    set_error("unet_set_params: bad arguments");
    return FB_ERR_ARG;
  }
  FB_CUDA(cudaMemcpy(u->param, host, sizeof(float) * u->nparam, cudaMemcpyHostToDevice));
  FB_CUDA(cudaMemset(u->adam_m, 0, sizeof(float) * u->nparam));
  FB_CUDA(cudaMemset(u->adam_v, 0, sizeof(float) * u->nparam));
  UN_TRY(prep_weights(u, 0));
  FB_CUDA(cudaDeviceSynchronize());
  return FB_OK;
}

fb_status fb_unet_get_params(const fb_unet* u, float* host)
{
  if(!u || !host)
  {
    set_error("unet_get_params: bad arguments");
    return FB_ERR_ARG;
  }
  FB_CUDA(cudaDeviceSynchronize());
  FB_CUDA(cudaMemcpy(host, u->param, sizeof(float) * u->nparam, cudaMemcpyDeviceToHost));
  return FB_OK;
}

fb_status fb_unet_get_grads(const fb_unet* u, float* host)
{
  if(!u || !host)
  {
    set_error("unet_get_grads: bad arguments");
    return FB_ERR_ARG;
  }
  FB_CUDA(cudaDeviceSynchronize());
  FB_CUDA(cudaMemcpy(host, u->grad, sizeof(float) * u->nparam, cudaMemcpyDeviceToHost));
  return FB_OK;
}

// in: DEVICE [batch][2][G][G] FP32 (f, log kappa, already scaled); out: DEVICE [batch][G][G] FP32
fb_status fb_unet_forward(fb_unet* u, const float* in, float* out, int batch, void* stream)
{
  if(!u || !in || !out || batch < 1 || batch > u->max_batch || !u->weights_ready)
  {
    set_error("unet_forward: bad arguments (or parameters not set)");
    return FB_ERR_ARG;
  }
  cudaStream_t st = as_stream(stream);
  const int B = batch;
  const int* G = u->G;
  const size_t P0 = size_t(B) * G[0] * G[0];
  k_pack_input<<<grid_for(P0), 256, 0, st>>>(in, B, G[0], u->x8);
  FB_LAUNCHED(1);
  UN_TRY(conv_fwd(u, 0, u->x8, B, G[0], u->e[0], 16, true, true, st));
  const int ech[4] = {16, 32, 64, 64};
  for(int i = 0; i < 3; ++i)
  {
    const size_t nc = size_t(B) * G[i + 1] * G[i + 1] * (ech[i] / 8);
    k_subsample<<<grid_for(nc), 256, 0, st>>>(u->e[i], B, G[i], ech[i], u->s[i]);
    FB_LAUNCHED(1);
    UN_TRY(conv_fwd(u, i + 1, u->s[i], B, G[i + 1], u->e[i + 1], ech[i + 1], true, true, st));
  }
  // bottleneck: dilation 2 and 4
  UN_TRY(conv_fwd(u, 4, u->e[3], B, G[3], u->b4[0], 64, true, true, st));
  UN_TRY(conv_fwd(u, 5, u->b4[0], B, G[3], u->b4[1], 64, true, true, st));
  // decoder
  {
    const size_t n3 = size_t(B) * G[2] * G[2] * 128;
    k_upsample_cat<<<grid_for(n3), 256, 0, st>>>(u->b4[1], 64, u->e[2], 64, B, G[2], u->c[2]);
    FB_LAUNCHED(1);
    UN_TRY(conv_fwd(u, 6, u->c[2], B, G[2], u->d[2], 64, true, true, st));
    const size_t n2 = size_t(B) * G[1] * G[1] * 96;
    k_upsample_cat<<<grid_for(n2), 256, 0, st>>>(u->d[2], 64, u->e[1], 32, B, G[1], u->c[1]);
    FB_LAUNCHED(1);
    UN_TRY(conv_fwd(u, 7, u->c[1], B, G[1], u->d[1], 32, true, true, st));
    const size_t n1 = size_t(B) * G[0] * G[0] * 48;
    k_upsample_cat<<<grid_for(n1), 256, 0, st>>>(u->d[1], 32, u->e[0], 16, B, G[0], u->c[0]);
    FB_LAUNCHED(1);
    UN_TRY(conv_fwd(u, 8, u->c[0], B, G[0], u->d[0], 16, true, true, st));
    UN_TRY(conv_fwd(u, 9, u->d[0], B, G[0], u->yout, 8, false, false, st));
  }
  k_unpack_out<<<grid_for(P0), 256, 0, st>>>(u->yout, P0, out);
  FB_LAUNCHED(1);
  return FB_OK;
}

// Gradients of the parameters for d loss / d out = dout (DEVICE [batch][G][G] FP32) at the
// activations of the last fb_unet_forward (same batch).  accumulate != 0 adds to the stored gradients.
fb_status fb_unet_backward(fb_unet* u, const float* dout, int batch, int accumulate, void* stream)
{
  if(!u || !dout || batch < 1 || batch > u->max_batch)
  {
    set_error("unet_backward: bad arguments");
    return FB_ERR_ARG;
  }
  cudaStream_t st = as_stream(stream);
  const int B = batch;
  const int* G = u->G;
  const int acc = accumulate ? 1 : 0;
  const size_t P0 = size_t(B) * G[0] * G[0];
  auto n_at = [&](int lv, int C) { return size_t(B) * G[lv] * G[lv] * C; };
  // L8 (input d1): dy8 = dout
  k_pack_dout<<<grid_for(P0), 256, 0, st>>>(dout, P0, u->dy8);
  FB_LAUNCHED(1);
  UN_TRY(conv_bwd_weight(u, 9, u->dy8, u->d[0], B, G[0], acc, st));
  UN_TRY(conv_bwd_data(u, 9, u->dy8, B, G[0], u->gs, st));                       // d1 grad [P0][16]
  // L7 (input c1 = [U(d2), e1]): dpre = mask(d1) * gs
  k_grad_mask<<<grid_for(n_at(0, 16)), 256, 0, st>>>(u->d[0], 16, B, G[0], u->gs, 16, 0, nullptr, 0, u->dpre);
  FB_LAUNCHED(1);
  UN_TRY(conv_bwd_weight(u, 8, u->dpre, u->c[0], B, G[0], acc, st));
  UN_TRY(conv_bwd_data(u, 8, u->dpre, B, G[0], u->dc[0], st));                   // dc1 [P0][48]
  // L6 (input c2 = [U(d3), e2]): dpre = mask(d2) * U^T(dc1[:, 0:32])
  k_upsample_bwd_mask<<<grid_for(n_at(1, 32)), 256, 0, st>>>(u->dc[0], 48, 0, 32, B, G[0], u->d[1], u->dpre);
  FB_LAUNCHED(1);
  UN_TRY(conv_bwd_weight(u, 7, u->dpre, u->c[1], B, G[1], acc, st));
  UN_TRY(conv_bwd_data(u, 7, u->dpre, B, G[1], u->dc[1], st));                   // dc2 [P1][96]
  // L5 (input c3 = [U(e4), e3]): dpre = mask(d3) * U^T(dc2[:, 0:64])
  k_upsample_bwd_mask<<<grid_for(n_at(2, 64)), 256, 0, st>>>(u->dc[1], 96, 0, 64, B, G[1], u->d[2], u->dpre);
  FB_LAUNCHED(1);
  UN_TRY(conv_bwd_weight(u, 6, u->dpre, u->c[2], B, G[2], acc, st));
  UN_TRY(conv_bwd_data(u, 6, u->dpre, B, G[2], u->dc[2], st));                   // dc3 [P2][128]
  // bottleneck, dilation 4 (input b4[0]): dpre = mask(e4) * U^T(dc3[:, 0:64])
  k_upsample_bwd_mask<<<grid_for(n_at(3, 64)), 256, 0, st>>>(u->dc[2], 128, 0, 64, B, G[2], u->b4[1], u->dpre);
  FB_LAUNCHED(1);
  UN_TRY(conv_bwd_weight(u, 5, u->dpre, u->b4[0], B, G[3], acc, st));
  UN_TRY(conv_bwd_data(u, 5, u->dpre, B, G[3], u->gs, st));                      // b4[0] grad [P3][64]
  // bottleneck, dilation 2 (input e4a = e[3])
  k_grad_mask<<<grid_for(n_at(3, 64)), 256, 0, st>>>(u->b4[0], 64, B, G[3], u->gs, 64, 0, nullptr, 0, u->dpre);
  FB_LAUNCHED(1);
  UN_TRY(conv_bwd_weight(u, 4, u->dpre, u->e[3], B, G[3], acc, st));
  UN_TRY(conv_bwd_data(u, 4, u->dpre, B, G[3], u->gs, st));                      // e[3] grad [P3][64]
  // L4 (input s3 = S(e3))
  k_grad_mask<<<grid_for(n_at(3, 64)), 256, 0, st>>>(u->e[3], 64, B, G[3], u->gs, 64, 0, nullptr, 0, u->dpre);
  FB_LAUNCHED(1);
  UN_TRY(conv_bwd_weight(u, 3, u->dpre, u->s[2], B, G[3], acc, st));
  UN_TRY(conv_bwd_data(u, 3, u->dpre, B, G[3], u->gs, st));                      // s3 grad [P3][64]
  // L3 (input s2): dpre = mask(e3) * (dc3[:, 64:128] + S^T(gs))
  k_grad_mask<<<grid_for(n_at(2, 64)), 256, 0, st>>>(u->e[2], 64, B, G[2], u->dc[2], 128, 64, u->gs, 64, u->dpre);
  FB_LAUNCHED(1);
  UN_TRY(conv_bwd_weight(u, 2, u->dpre, u->s[1], B, G[2], acc, st));
  UN_TRY(conv_bwd_data(u, 2, u->dpre, B, G[2], u->gs, st));                      // s2 grad [P2][32]
  // L2 (input s1): dpre = mask(e2) * (dc2[:, 64:96] + S^T(gs))
  k_grad_mask<<<grid_for(n_at(1, 32)), 256, 0, st>>>(u->e[1], 32, B, G[1], u->dc[1], 96, 64, u->gs, 32, u->dpre);
  FB_LAUNCHED(1);
  UN_TRY(conv_bwd_weight(u, 1, u->dpre, u->s[0], B, G[1], acc, st));
  UN_TRY(conv_bwd_data(u, 1, u->dpre, B, G[1], u->gs, st));                      // s1 grad [P1][16]
  // L1 (input x8): dpre = mask(e1) * (dc1[:, 32:48] + S^T(gs))
  k_grad_mask<<<grid_for(n_at(0, 16)), 256, 0, st>>>(u->e[0], 16, B, G[0], u->dc[0], 48, 32, u->gs, 16, u->dpre);
  FB_LAUNCHED(1);
  UN_TRY(conv_bwd_weight(u, 0, u->dpre, u->x8, B, G[0], acc, st));
  return FB_OK;
}

// Adam step on the FP32 masters with the stored gradients (step t >= 1 for the bias corrections),
// then the BF16 GEMM copies.
fb_status fb_unet_adam(fb_unet* u, float lr, float beta1, float beta2, float eps, int t, void* stream)
{
  if(!u || t < 1)
  {
    set_error("unet_adam: bad arguments");
    return FB_ERR_ARG;
  }
  cudaStream_t st = as_stream(stream);
  const float c1 = 1.f - std::pow(beta1, float(t)), c2 = 1.f - std::pow(beta2, float(t));
  k_adam<<<grid_for(u->nparam), 256, 0, st>>>(u->param, u->grad, u->adam_m, u->adam_v, u->nparam, lr, beta1, beta2,
    eps, c1, c2);
  FB_LAUNCHED(1);
  return prep_weights(u, st);
}

// Mean squared error over n entries (DEVICE arrays): *loss (DEVICE double) = sum (y - t)^2 / n;
// grad (DEVICE, may be NULL) = 2 (y - t) / n.
fb_status fb_unet_mse(fb_unet* u, const float* y, const float* t, uint64_t n, float* grad, double* loss, void* stream)
{
  if(!u || !y || !t || !loss || n == 0)
  {
    set_error("unet_mse: bad arguments");
    return FB_ERR_ARG;
  }
  cudaStream_t st = as_stream(stream);
  const int nb = int(std::min<uint64_t>(1024, (n + MSE_NT - 1) / MSE_NT));
  k_mse<<<nb, MSE_NT, 0, st>>>(y, t, size_t(n), grad, u->mse_part);
  k_mse_final<<<1, 1, 0, st>>>(u->mse_part, nb, size_t(n), loss);
  FB_LAUNCHED(2);
  return FB_OK;
}

} // extern "C"
