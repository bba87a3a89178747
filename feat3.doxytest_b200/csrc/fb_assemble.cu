// Q1 assembly on the uniformly refined unit square (and, for the Laplacian, the unit cube), on
// the device: the set-up step before the
// solve path (the reference assembles on the host: kernel/assembly/domain_assembler_helpers.hpp,
// kernel/assembly/common_operators.hpp:36, common_functionals.hpp:33, with the 3x3 Gauss rule that
// "auto-degree:5" selects).  Vertices are numbered lexicographically ((2^L+1)^2 of them); the
// stiffness values are written in the row-sorted 9-point CSR pattern of fb_q1_pattern_2d.
//
// kappa = exp(g), g(x, y) = s * sum_{i,j} (xi_ij cos t + eta_ij sin t) / (kx_i^2 + ky_j^2),
// t = 2 pi (kx_i x + ky_j y), kx = ky = -K/2 .. K/2-1 (the (0,0) mode excluded); f = sum of
// Gaussians a * exp(-|x - c|^2 / (2 w^2)).  Pass 1 computes every cell's 4x4 element matrix and
// 4 load contributions (one thread per cell); pass 2 sums them per matrix entry / vertex (one
// thread per vertex, cells in ascending index order), so no atomics are needed and the result is
// deterministic.
#include "fb_common.cuh"

#include <cmath>
#include <vector>

namespace fb
{
namespace as
{
  struct Ref
  {
    double xq[3], wq[3];
    double val[9][4];       // phi_v at quad point q
    double gg[9][4][4];     // grad phi_u . grad phi_v at q (reference element)
  };
  __constant__ Ref c_ref;

  // g at (x, y) by the separable sum: h_i = sum_j c_ij e^{2 pi i ky_j y}, g = s sum_i Re(h_i e^{2 pi i kx_i x})
  __device__ double field(double x, double y, int K, const double* __restrict__ xi, const double* __restrict__ eta,
    double s)
  {
    const double tp = 6.283185307179586476925286766559;
    double acc = 0.0;
    for(int i = 0; i < K; ++i)
    {
      const double kx = double(i - K / 2);
      double hr = 0.0, hi = 0.0;
      for(int j = 0; j < K; ++j)
      {
        const double ky = double(j - K / 2);
        const double den = kx * kx + ky * ky;
        if(den == 0.0)
          continue;
        double sy, cy;
        sincos(tp * ky * y, &sy, &cy);
        const double a = __ldg(xi + i * K + j) / den, b = __ldg(eta + i * K + j) / den;
        hr += a * cy + b * sy;
        hi += a * sy - b * cy;
      }
      double sx, cx;
      sincos(tp * kx * x, &sx, &cx);
      acc += hr * cx - hi * sx;
    }
    return s * acc;
  }

  // Separable tables of the field at the quadrature coordinates (3 per cell and direction, index
  // 3*cell + q): ex[t][i] = e^{2 pi i kx_i x_t} and hy[t][i] = sum_j c_ij e^{2 pi i ky_j y_t}, so that
  // g(x_t, y_u) = s * sum_i Re(ex[t][i] * hy[u][i]): K complex products per point instead of K^2
  // sine/cosine pairs.
  __global__ void k_field_tables(int N, double h, int K, const double* __restrict__ xi,
    const double* __restrict__ eta, double2* __restrict__ ex, double2* __restrict__ hy)
  {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if(e >= 3 * N * K)
      return;
    const double tp = 6.283185307179586476925286766559;
    const int i = e % K, t = e / K;
    const double c = (double(t / 3) + (1.0 + c_ref.xq[t % 3]) / 2.0) * h;   // x_t = y_t
    const double kx = double(i - K / 2);
    double sx, cx;
    sincos(tp * kx * c, &sx, &cx);
    ex[e] = make_double2(cx, sx);
    double hr = 0.0, hi = 0.0;
    for(int j = 0; j < K; ++j)
    {
      const double ky = double(j - K / 2);
      const double den = kx * kx + ky * ky;
      if(den == 0.0)
        continue;
      double sy, cy;
      sincos(tp * ky * c, &sy, &cy);
      const double a = __ldg(xi + i * K + j) / den, b = __ldg(eta + i * K + j) / den;
      hr += a * cy + b * sy;
      hi += a * sy - b * cy;
    }
    hy[e] = make_double2(hr, hi);
  }

  // per cell: the 4x4 element matrix (kappa-weighted) and the 4 load-vector contributions
  __global__ void k_cells(int N, double h, int K, const double2* __restrict__ ex, const double2* __restrict__ hy,
    double s, int ng, const double* __restrict__ gauss, double* __restrict__ ke, double* __restrict__ fe)
  {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if(c >= N * N)
      return;
    const int cx = c % N, cy = c / N;
    double kq[9], fq[9];
    for(int qy = 0; qy < 3; ++qy)
      for(int qx = 0; qx < 3; ++qx)
      {
        const int q = qx * 3 + qy;   // reference order: x index slowest (meshgrid "ij" over (x, y))
        const double x = (double(cx) + (1.0 + c_ref.xq[qx]) / 2.0) * h;
        const double y = (double(cy) + (1.0 + c_ref.xq[qy]) / 2.0) * h;
        double kv = 1.0;
        if(K > 0 && ke)
        {
          const double2* exr = ex + size_t(cx * 3 + qx) * K;
          const double2* hyr = hy + size_t(cy * 3 + qy) * K;
          double g = 0.0;
          for(int i = 0; i < K; ++i)
          {
            const double2 a = __ldg(exr + i), b = __ldg(hyr + i);
            g += b.x * a.x - b.y * a.y;
          }
          kv = exp(s * g);
        }
        kq[q] = kv;
        double f = 0.0;
        for(int g = 0; g < ng && fe; ++g)
        {
          const double dx = x - gauss[4 * g + 0], dy = y - gauss[4 * g + 1], w = gauss[4 * g + 2];
          f += gauss[4 * g + 3] * exp(-(dx * dx + dy * dy) / (2.0 * w * w));
        }
        fq[q] = f;
      }
    if(ke)
      for(int a = 0; a < 4; ++a)
        for(int b = 0; b < 4; ++b)
        {
          double v = 0.0;
          for(int q = 0; q < 9; ++q)
            v += kq[q] * (c_ref.wq[q / 3] * c_ref.wq[q % 3]) * c_ref.gg[q][a][b];
          ke[size_t(c) * 16 + a * 4 + b] = v;
        }
    if(fe)
      for(int a = 0; a < 4; ++a)
      {
        double v = 0.0;
        for(int q = 0; q < 9; ++q)
          v += fq[q] * (c_ref.wq[q / 3] * c_ref.wq[q % 3]) * c_ref.val[q][a];
        fe[size_t(c) * 4 + a] = (h / 2.0) * (h / 2.0) * v;
      }
  }

  // per vertex: stiffness row (sorted neighbours) and load entry, summing cells in ascending order
  __global__ void k_vertices(int N, const double* __restrict__ ke, const double* __restrict__ fe,
    const uint64_t* __restrict__ rp, double* __restrict__ vals, double* __restrict__ rhs)
  {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    const int n1 = N + 1;
    if(v >= n1 * n1)
      return;
    const int ix = v % n1, iy = v / n1;
    if(vals)
    {
      uint64_t pos = rp[v];
      for(int dy = -1; dy <= 1; ++dy)
        for(int dx = -1; dx <= 1; ++dx)
        {
          const int jx = ix + dx, jy = iy + dy;
          if(jx < 0 || jy < 0 || jx > N || jy > N)
            continue;
          double s = 0.0;
          for(int cy = max(max(iy, jy) - 1, 0); cy <= min(min(iy, jy), N - 1); ++cy)
            for(int cx = max(max(ix, jx) - 1, 0); cx <= min(min(ix, jx), N - 1); ++cx)
            {
              const int a = (ix - cx) + 2 * (iy - cy);
              const int b = (jx - cx) + 2 * (jy - cy);
              s += ke[(size_t(cy) * N + cx) * 16 + a * 4 + b];
            }
          vals[pos++] = s;
        }
    }
    if(rhs)
    {
      double s = 0.0;
      for(int cy = max(iy - 1, 0); cy <= min(iy, N - 1); ++cy)
        for(int cx = max(ix - 1, 0); cx <= min(ix, N - 1); ++cx)
          s += fe[(size_t(cy) * N + cx) * 4 + (ix - cx) + 2 * (iy - cy)];
      const bool boundary = ix == 0 || iy == 0 || ix == N || iy == N;
      rhs[v] = boundary ? 0.0 : s;
    }
  }

  // f and g (= log kappa) at the vertices of level L (lexicographic, x fastest)
  __global__ void k_sample(int N, int K, const double* __restrict__ xi, const double* __restrict__ eta, double s,
    int ng, const double* __restrict__ gauss, double* __restrict__ fv, double* __restrict__ gv)
  {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    const int n1 = N + 1;
    if(v >= n1 * n1)
      return;
    const double h = 1.0 / N;
    const double x = double(v % n1) * h, y = double(v / n1) * h;
    if(gv)
      gv[v] = K > 0 ? field(x, y, K, xi, eta, s) : 0.0;
    if(fv)
    {
      double f = 0.0;
      for(int g = 0; g < ng; ++g)
      {
        const double dx = x - gauss[4 * g + 0], dy = y - gauss[4 * g + 1], w = gauss[4 * g + 2];
        f += gauss[4 * g + 3] * exp(-(dx * dx + dy * dy) / (2.0 * w * w));
      }
      fv[v] = f;
    }
  }

  // Q1 prolongation level-1 -> level on the lexicographic vertices: fine vertex (ix, iy) takes
  // coarse (ix/2, iy/2) with weight 1 per even coordinate and the two neighbours (i-1)/2, (i+1)/2
  // with 1/2 each per odd coordinate; entries in ascending coarse index.  The row pointer is in
  // closed form: cnt(i) = 1 + (i odd), sum_{j<i} cnt(j) = i + i/2.
  __global__ void k_prolongation(int Nf, uint64_t* __restrict__ rp, uint64_t* __restrict__ col,
    double* __restrict__ val)
  {
    const int n1 = Nf + 1, nc1 = Nf / 2 + 1;
    const uint64_t v = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if(v >= uint64_t(n1) * n1)
      return;
    const int ix = int(v % n1), iy = int(v / n1);
    const uint64_t W = uint64_t(n1 + Nf / 2);
    const int cx = 1 + (ix & 1), cy = 1 + (iy & 1);
    const uint64_t off = uint64_t(iy + iy / 2) * W + uint64_t(cy) * uint64_t(ix + ix / 2);
    rp[v] = off;
    if(v + 1 == uint64_t(n1) * n1)
      rp[v + 1] = off + uint64_t(cx) * cy;
    const int x0 = ix / 2, y0 = iy / 2;   // odd i: (i-1)/2 and (i+1)/2 = x0, x0 + 1
    uint64_t e = off;
    for(int b = 0; b < cy; ++b)
      for(int a = 0; a < cx; ++a)
      {
        col[e] = uint64_t(y0 + b) * nc1 + uint64_t(x0 + a);
        val[e] = (cx == 2 ? 0.5 : 1.0) * (cy == 2 ? 0.5 : 1.0);
        ++e;
      }
  }

  // ---------------------------------------------------------------- 3D (unit cube, hexahedra)
  // Trilinear Q1 on [-1,1]^3 with the 3x3x3 Gauss rule (q = 9 qx + 3 qy + qz), local vertex
  // v = bx + 2 by + 4 bz; the Laplace element matrix is the same for every cell (h/2 times the
  // reference one), so only the load vector needs per-cell work.
  struct Ref3
  {
    double xq[3], wq[3];
    double val[27][8];      // phi_v at quad point q
    double kloc[8][8];      // element stiffness of the reference element scaled to cells of size h = 1
  };
  __constant__ Ref3 c_ref3;

  // per cell: the 8 load-vector contributions of a sum of Gaussians (rows c_x, c_y, c_z, w, a)
  __global__ void k_cells3(int N, double h, int ng, const double* __restrict__ gauss, double* __restrict__ fe)
  {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if(c >= (long long)N * N * N)
      return;
    const int cx = int(c % N), cy = int((c / N) % N), cz = int(c / ((long long)N * N));
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for(int qx = 0; qx < 3; ++qx)
      for(int qy = 0; qy < 3; ++qy)
        for(int qz = 0; qz < 3; ++qz)
        {
          const int q = qx * 9 + qy * 3 + qz;
          const double x = (double(cx) + (1.0 + c_ref3.xq[qx]) / 2.0) * h;
          const double y = (double(cy) + (1.0 + c_ref3.xq[qy]) / 2.0) * h;
          const double z = (double(cz) + (1.0 + c_ref3.xq[qz]) / 2.0) * h;
          double f = 0.0;
          for(int g = 0; g < ng; ++g)
          {
            const double dx = x - gauss[5 * g + 0], dy = y - gauss[5 * g + 1], dz = z - gauss[5 * g + 2];
            const double w = gauss[5 * g + 3];
            f += gauss[5 * g + 4] * exp(-(dx * dx + dy * dy + dz * dz) / (2.0 * w * w));
          }
          const double wf = f * (c_ref3.wq[qx] * c_ref3.wq[qy] * c_ref3.wq[qz]);
          for(int a = 0; a < 8; ++a)
            acc[a] += wf * c_ref3.val[q][a];
        }
    const double sc = (h / 2.0) * (h / 2.0) * (h / 2.0);
    for(int a = 0; a < 8; ++a)
      fe[size_t(c) * 8 + a] = sc * acc[a];
  }

  // per vertex: the 27-point stiffness row (sorted neighbours) and the load entry, cells in
  // ascending index order
  __global__ void k_vertices3(int N, double h, const double* __restrict__ fe, const uint64_t* __restrict__ rp,
    double* __restrict__ vals, double* __restrict__ rhs)
  {
    const long long n1 = N + 1;
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if(v >= n1 * n1 * n1)
      return;
    const int ix = int(v % n1), iy = int((v / n1) % n1), iz = int(v / (n1 * n1));
    if(vals)
    {
      uint64_t pos = rp[v];
      for(int dz = -1; dz <= 1; ++dz)
        for(int dy = -1; dy <= 1; ++dy)
          for(int dx = -1; dx <= 1; ++dx)
          {
            const int jx = ix + dx, jy = iy + dy, jz = iz + dz;
            if(jx < 0 || jy < 0 || jz < 0 || jx > N || jy > N || jz > N)
              continue;
            double s = 0.0;
            for(int cz = max(max(iz, jz) - 1, 0); cz <= min(min(iz, jz), N - 1); ++cz)
              for(int cy = max(max(iy, jy) - 1, 0); cy <= min(min(iy, jy), N - 1); ++cy)
                for(int cx = max(max(ix, jx) - 1, 0); cx <= min(min(ix, jx), N - 1); ++cx)
                {
                  const int a = (ix - cx) + 2 * (iy - cy) + 4 * (iz - cz);
                  const int b = (jx - cx) + 2 * (jy - cy) + 4 * (jz - cz);
                  s += h * c_ref3.kloc[a][b];
                }
            vals[pos++] = s;
          }
    }
    if(rhs)
    {
      double s = 0.0;
      for(int cz = max(iz - 1, 0); cz <= min(iz, N - 1); ++cz)
        for(int cy = max(iy - 1, 0); cy <= min(iy, N - 1); ++cy)
          for(int cx = max(ix - 1, 0); cx <= min(ix, N - 1); ++cx)
            s += fe[((size_t(cz) * N + cy) * N + cx) * 8 + (ix - cx) + 2 * (iy - cy) + 4 * (iz - cz)];
      const bool boundary = ix == 0 || iy == 0 || iz == 0 || ix == N || iy == N || iz == N;
      rhs[v] = boundary ? 0.0 : s;
    }
  }

  // Q1 prolongation level-1 -> level on the lexicographic vertices of the cube: per direction an
  // even fine coordinate takes coarse i/2 (weight 1), an odd one (i-1)/2 and (i+1)/2 (1/2 each);
  // entries in ascending coarse index.  Row pointer in closed form with S(i) = i + i/2 the entries
  // of the coordinates before i on one line and W = S(N + 1).
  __global__ void k_prolongation3(int Nf, uint64_t* __restrict__ rp, uint64_t* __restrict__ col,
    double* __restrict__ val)
  {
    const uint64_t n1 = uint64_t(Nf) + 1, nc1 = uint64_t(Nf) / 2 + 1;
    const uint64_t v = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if(v >= n1 * n1 * n1)
      return;
    const uint64_t ix = v % n1, iy = (v / n1) % n1, iz = v / (n1 * n1);
    const uint64_t W = n1 + uint64_t(Nf) / 2;
    const uint64_t cx = 1 + (ix & 1), cy = 1 + (iy & 1), cz = 1 + (iz & 1);
    const uint64_t off = (iz + iz / 2) * W * W + cz * (iy + iy / 2) * W + cz * cy * (ix + ix / 2);
    rp[v] = off;
    if(v + 1 == n1 * n1 * n1)
      rp[v + 1] = off + cx * cy * cz;
    const uint64_t x0 = ix / 2, y0 = iy / 2, z0 = iz / 2;
    uint64_t e = off;
    for(uint64_t c = 0; c < cz; ++c)
      for(uint64_t b = 0; b < cy; ++b)
        for(uint64_t a = 0; a < cx; ++a)
        {
          col[e] = ((z0 + c) * nc1 + (y0 + b)) * nc1 + (x0 + a);
          val[e] = (cx == 2 ? 0.5 : 1.0) * (cy == 2 ? 0.5 : 1.0) * (cz == 2 ? 0.5 : 1.0);
          ++e;
        }
  }

  static bool ref3_ready[64] = {};
  static fb_status upload_ref3()
  {
    int dev = 0;
    FB_CUDA(cudaGetDevice(&dev));
    if(dev >= 0 && dev < 64 && ref3_ready[dev])
      return FB_OK;
    Ref3 r;
    const double g = std::sqrt(3.0 / 5.0);
    const double xs[3] = {-g, 0.0, g}, ws[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
    for(int k = 0; k < 3; ++k)
    {
      r.xq[k] = xs[k];
      r.wq[k] = ws[k];
    }
    double gr[27][8][3];
    for(int qx = 0; qx < 3; ++qx)
      for(int qy = 0; qy < 3; ++qy)
        for(int qz = 0; qz < 3; ++qz)
        {
          const int q = qx * 9 + qy * 3 + qz;
          const double p[3] = {xs[qx], xs[qy], xs[qz]};
          for(int v = 0; v < 8; ++v)
          {
            double f[3], sg[3];
            for(int d = 0; d < 3; ++d)
            {
              sg[d] = ((v >> d) & 1) ? 1.0 : -1.0;
              f[d] = 1.0 + p[d] * sg[d];
            }
            r.val[q][v] = f[0] * f[1] * f[2] / 8.0;
            gr[q][v][0] = sg[0] * f[1] * f[2] / 8.0;
            gr[q][v][1] = sg[1] * f[0] * f[2] / 8.0;
            gr[q][v][2] = sg[2] * f[0] * f[1] / 8.0;
          }
        }
    // (h/2)^3 (2/h)^2 = h/2: the reference element's matrix times 1/2, times h in the vertex kernel
    for(int a = 0; a < 8; ++a)
      for(int b = 0; b < 8; ++b)
      {
        double s = 0.0;
        for(int qx = 0; qx < 3; ++qx)
          for(int qy = 0; qy < 3; ++qy)
            for(int qz = 0; qz < 3; ++qz)
            {
              const int q = qx * 9 + qy * 3 + qz;
              const double gg = gr[q][a][0] * gr[q][b][0] + gr[q][a][1] * gr[q][b][1] + gr[q][a][2] * gr[q][b][2];
              s += ws[qx] * ws[qy] * ws[qz] * gg;
            }
        r.kloc[a][b] = 0.5 * s;
      }
    FB_CUDA(cudaMemcpyToSymbol(c_ref3, &r, sizeof(Ref3)));
    if(dev >= 0 && dev < 64)
      ref3_ready[dev] = true;
    return FB_OK;
  }

  static bool ref_ready[64] = {};
  static fb_status upload_ref()
  {
    int dev = 0;
    FB_CUDA(cudaGetDevice(&dev));
    if(dev >= 0 && dev < 64 && ref_ready[dev])
      return FB_OK;
    Ref r;
    const double g = std::sqrt(3.0 / 5.0);
    const double xs[3] = {-g, 0.0, g}, ws[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
    for(int k = 0; k < 3; ++k)
    {
      r.xq[k] = xs[k];
      r.wq[k] = ws[k];
    }
    for(int qx = 0; qx < 3; ++qx)
      for(int qy = 0; qy < 3; ++qy)
      {
        const int q = qx * 3 + qy;
        double gr[4][2];
        for(int v = 0; v < 4; ++v)
        {
          const double sx = (v & 1) ? 1.0 : -1.0, sy = (v & 2) ? 1.0 : -1.0;
          const double fx = 1.0 + xs[qx] * sx, fy = 1.0 + xs[qy] * sy;
          r.val[q][v] = fx * fy / 4.0;
          gr[v][0] = sx * fy / 4.0;
          gr[v][1] = sy * fx / 4.0;
        }
        for(int a = 0; a < 4; ++a)
          for(int b = 0; b < 4; ++b)
            r.gg[q][a][b] = gr[a][0] * gr[b][0] + gr[a][1] * gr[b][1];
      }
    FB_CUDA(cudaMemcpyToSymbol(c_ref, &r, sizeof(Ref)));
    if(dev >= 0 && dev < 64)
      ref_ready[dev] = true;
    return FB_OK;
  }
} // namespace as
} // namespace fb

using namespace fb;

extern "C" {

fb_status fb_q1_pattern_2d(int level, uint64_t* nnz_out, uint64_t* row_ptr, uint64_t* col_ind)
{
  if(level < 0 || level > 13 || !nnz_out)
  {
    set_error("q1_pattern_2d: bad arguments");
    return FB_ERR_ARG;
  }
  const int N = 1 << level, n1 = N + 1;
  uint64_t pos = 0;
  if(row_ptr)
    row_ptr[0] = 0;
  for(int iy = 0; iy <= N; ++iy)
    for(int ix = 0; ix <= N; ++ix)
    {
      for(int dy = -1; dy <= 1; ++dy)
        for(int dx = -1; dx <= 1; ++dx)
        {
          const int jx = ix + dx, jy = iy + dy;
          if(jx < 0 || jy < 0 || jx > N || jy > N)
            continue;
          if(col_ind)
            col_ind[pos] = uint64_t(jy) * n1 + jx;
          ++pos;
        }
      if(row_ptr)
        row_ptr[uint64_t(iy) * n1 + ix + 1] = pos;
    }
  *nnz_out = pos;
  return FB_OK;
}

fb_status fb_q1_assemble_2d(int level, int kmodes, const double* xi, const double* eta, double s, int ngauss,
  const double* gauss, const uint64_t* row_ptr, double* values, double* rhs, void* stream)
{
  if(level < 0 || level > 13 || kmodes < 0 || kmodes > 64 || (kmodes && (!xi || !eta)) ||
     (ngauss && !gauss) || (values && !row_ptr) || (!values && !rhs))
  {
    set_error("q1_assemble_2d: bad arguments");
    return FB_ERR_ARG;
  }
  fb_status e = as::upload_ref();
  if(e != FB_OK)
    return e;
  const int N = 1 << level;
  const double h = 1.0 / N;
  cudaStream_t st = as_stream(stream);
  double *ke = nullptr, *fe = nullptr;
  double2 *ex = nullptr, *hy = nullptr;
  const int K = values ? kmodes : 0;
  if(values)
    FB_CUDA(cudaMallocAsync((void**)&ke, sizeof(double) * 16 * size_t(N) * N, st));
  if(rhs)
    FB_CUDA(cudaMallocAsync((void**)&fe, sizeof(double) * 4 * size_t(N) * N, st));
  if(K)
  {
    FB_CUDA(cudaMallocAsync((void**)&ex, sizeof(double2) * 3 * size_t(N) * K, st));
    FB_CUDA(cudaMallocAsync((void**)&hy, sizeof(double2) * 3 * size_t(N) * K, st));
    as::k_field_tables<<<(3 * N * K + 127) / 128, 128, 0, st>>>(N, h, K, xi, eta, ex, hy);
    FB_LAUNCHED(1);
  }
  const int cells = N * N, verts = (N + 1) * (N + 1);
  as::k_cells<<<(cells + 127) / 128, 128, 0, st>>>(N, h, K, ex, hy, s, rhs ? ngauss : 0, gauss, ke, fe);
  as::k_vertices<<<(verts + 255) / 256, 256, 0, st>>>(N, ke, fe, row_ptr, values, rhs);
  FB_LAUNCHED(2);
  if(ke)
    FB_CUDA(cudaFreeAsync(ke, st));
  if(fe)
    FB_CUDA(cudaFreeAsync(fe, st));
  if(ex)
    FB_CUDA(cudaFreeAsync(ex, st));
  if(hy)
    FB_CUDA(cudaFreeAsync(hy, st));
  FB_CUDA(cudaStreamSynchronize(st));
  return FB_OK;
}

fb_status fb_q1_prolongation_2d(int level, uint64_t* nnz, uint64_t* row_ptr, uint64_t* col_ind, double* values,
  void* stream)
{
  if(level < 1 || level > 13 || !nnz)
  {
    set_error("q1_prolongation_2d: bad arguments");
    return FB_ERR_ARG;
  }
  const uint64_t Nf = uint64_t(1) << level, n1 = Nf + 1;
  const uint64_t cnt = n1 + Nf / 2;   // x-entries per fine row
  *nnz = cnt * cnt;
  if(!row_ptr && !col_ind && !values)
    return FB_OK;
  if(!row_ptr || !col_ind || !values)
  {
    set_error("q1_prolongation_2d: row_ptr, col_ind and values are all needed");
    return FB_ERR_ARG;
  }
  cudaStream_t st = as_stream(stream);
  as::k_prolongation<<<unsigned((n1 * n1 + 255) / 256), 256, 0, st>>>(int(Nf), row_ptr, col_ind, values);
  FB_LAUNCHED(1);
  FB_CUDA(cudaStreamSynchronize(st));
  return FB_OK;
}

fb_status fb_q1_pattern_3d(int level, uint64_t* nnz_out, uint64_t* row_ptr, uint64_t* col_ind)
{
  if(level < 0 || level > 8 || !nnz_out)
  {
    set_error("q1_pattern_3d: bad arguments");
    return FB_ERR_ARG;
  }
  const int64_t N = int64_t(1) << level, n1 = N + 1;
  uint64_t pos = 0;
  if(row_ptr)
    row_ptr[0] = 0;
  for(int64_t iz = 0; iz <= N; ++iz)
    for(int64_t iy = 0; iy <= N; ++iy)
      for(int64_t ix = 0; ix <= N; ++ix)
      {
        for(int64_t dz = -1; dz <= 1; ++dz)
          for(int64_t dy = -1; dy <= 1; ++dy)
            for(int64_t dx = -1; dx <= 1; ++dx)
            {
              const int64_t jx = ix + dx, jy = iy + dy, jz = iz + dz;
              if(jx < 0 || jy < 0 || jz < 0 || jx > N || jy > N || jz > N)
                continue;
              if(col_ind)
                col_ind[pos] = uint64_t((jz * n1 + jy) * n1 + jx);
              ++pos;
            }
        if(row_ptr)
          row_ptr[uint64_t((iz * n1 + iy) * n1 + ix) + 1] = pos;
      }
  *nnz_out = pos;
  return FB_OK;
}

fb_status fb_q1_assemble_3d(int level, int ngauss, const double* gauss, const uint64_t* row_ptr, double* values,
  double* rhs, void* stream)
{
  if(level < 0 || level > 8 || (ngauss && !gauss) || ngauss < 0 || (values && !row_ptr) || (!values && !rhs))
  {
    set_error("q1_assemble_3d: bad arguments");
    return FB_ERR_ARG;
  }
  fb_status e = as::upload_ref3();
  if(e != FB_OK)
    return e;
  const int N = 1 << level;
  const double h = 1.0 / N;
  cudaStream_t st = as_stream(stream);
  double* fe = nullptr;
  const long long cells = (long long)N * N * N, verts = (long long)(N + 1) * (N + 1) * (N + 1);
  if(rhs)
  {
    FB_CUDA(cudaMallocAsync((void**)&fe, sizeof(double) * 8 * size_t(cells), st));
    as::k_cells3<<<unsigned((cells + 127) / 128), 128, 0, st>>>(N, h, ngauss, gauss, fe);
    FB_LAUNCHED(1);
  }
  as::k_vertices3<<<unsigned((verts + 255) / 256), 256, 0, st>>>(N, h, fe, row_ptr, values, rhs);
  FB_LAUNCHED(1);
  if(fe)
    FB_CUDA(cudaFreeAsync(fe, st));
  FB_CUDA(cudaStreamSynchronize(st));
  return FB_OK;
}

fb_status fb_q1_prolongation_3d(int level, uint64_t* nnz, uint64_t* row_ptr, uint64_t* col_ind, double* values,
  void* stream)
{
  if(level < 1 || level > 8 || !nnz)
  {
    set_error("q1_prolongation_3d: bad arguments");
    return FB_ERR_ARG;
  }
  const uint64_t Nf = uint64_t(1) << level, n1 = Nf + 1;
  const uint64_t cnt = n1 + Nf / 2;   // entries per fine line
  *nnz = cnt * cnt * cnt;
  if(!row_ptr && !col_ind && !values)
    return FB_OK;
  if(!row_ptr || !col_ind || !values)
  {
    set_error("q1_prolongation_3d: row_ptr, col_ind and values are all needed");
    return FB_ERR_ARG;
  }
  cudaStream_t st = as_stream(stream);
  as::k_prolongation3<<<unsigned((n1 * n1 * n1 + 255) / 256), 256, 0, st>>>(int(Nf), row_ptr, col_ind, values);
  FB_LAUNCHED(1);
  FB_CUDA(cudaStreamSynchronize(st));
  return FB_OK;
}

fb_status fb_q1_sample_2d(int level, int kmodes, const double* xi, const double* eta, double s, int ngauss,
  const double* gauss, double* f, double* g, void* stream)
{
  if(level < 0 || level > 13 || kmodes < 0 || kmodes > 64 || (kmodes && g && (!xi || !eta)) ||
     (ngauss && f && !gauss) || (!f && !g))
  {
    set_error("q1_sample_2d: bad arguments");
    return FB_ERR_ARG;
  }
  const int N = 1 << level, verts = (N + 1) * (N + 1);
  cudaStream_t st = as_stream(stream);
  as::k_sample<<<(verts + 255) / 256, 256, 0, st>>>(N, kmodes, xi, eta, s, f ? ngauss : 0, gauss, f, g);
  FB_LAUNCHED(1);
  FB_CUDA(cudaStreamSynchronize(st));
  return FB_OK;
}

} // extern "C"
