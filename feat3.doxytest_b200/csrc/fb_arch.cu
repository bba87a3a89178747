// Op-level seam: replacements of the reference's LAFEM::Arch backend kernels on raw device
// pointers (kernel/lafem/arch/*.hpp).  Each entry point enqueues on the caller's stream and, like
// the reference's *_cuda functions (which end in cudaDeviceSynchronize), returns after the work
// is done.
#include "fb_common.cuh"

#include <mutex>
#include <string>
#include <unordered_map>

namespace fb
{
  static thread_local std::string g_err;
  static std::atomic<uint64_t> g_launches{0};

  void set_error(const std::string& msg) { g_err = msg; }
  fb_status cuda_fail(cudaError_t e, const char* what)
  {
    g_err = std::string(what) + ": " + cudaGetErrorString(e);
    return FB_ERR_CUDA;
  }
  void count_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

  // ------------------------------------------------------------------ CSR apply
  // One thread per row; the block's slice of col_ind/val is staged in shared memory with
  // coalesced loads, then each thread sums its row in stored order with separately rounded
  // products and sums (bitwise equal to Apply::csr_generic, apply_generic.hpp:58-66).  Blocks
  // whose slice exceeds the staging capacity read their rows from global memory directly.
  constexpr int APPLY_NT = 256;
  constexpr int APPLY_CAP = 3072;   // staged entries per block

  template<typename DT, typename IT>
  __global__ void __launch_bounds__(APPLY_NT) k_apply_csr(DT* __restrict__ r, DT a, const DT* __restrict__ x,
    DT b, const DT* y, const DT* __restrict__ val, const IT* __restrict__ col, const IT* __restrict__ rp,
    uint64_t rows, bool use_y)
  {
    __shared__ DT s_val[APPLY_CAP];
    __shared__ uint32_t s_col[APPLY_CAP];
    const uint64_t r0 = uint64_t(blockIdx.x) * APPLY_NT;
    const uint64_t row = r0 + threadIdx.x;
    const uint64_t rend = (r0 + APPLY_NT < rows) ? r0 + APPLY_NT : rows;
    const uint64_t s0 = uint64_t(rp[r0]);
    const uint64_t s1 = uint64_t(rp[rend]);
    const bool staged = (s1 - s0) <= uint64_t(APPLY_CAP);
    if(staged)
    {
      for(uint64_t k = threadIdx.x; k < s1 - s0; k += APPLY_NT)
      {
        s_val[k] = val[s0 + k];
        s_col[k] = uint32_t(col[s0 + k]);
      }
      __syncthreads();
    }
    if(row >= rows)
      return;
    const uint64_t j0 = uint64_t(rp[row]), j1 = uint64_t(rp[row + 1]);
    DT sum = DT(0);
    if(staged)
    {
      for(uint64_t j = j0 - s0; j < j1 - s0; ++j)
        sum = add(sum, mul(s_val[j], x[s_col[j]]));
    }
    else
    {
      for(uint64_t j = j0; j < j1; ++j)
        sum = add(sum, mul(val[j], x[col[j]]));
    }
    const DT yv = use_y ? y[row] : DT(0);
    r[row] = add(mul(sum, a), mul(b, yv));
  }

  // transposed: r = a * (b/a * r0 + A^T x), r0 = y or 0 (apply_generic.hpp:38-55); the scatter
  // uses atomics, so its summation order differs from the sequential reference loop.
  template<typename DT>
  __global__ void k_scale_init(DT* r, const DT* y, DT ba, uint64_t n, bool use_y)
  {
    for(uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
      r[i] = mul(ba, use_y ? y[i] : DT(0));
  }
  template<typename DT, typename IT>
  __global__ void k_apply_csr_t(DT* r, const DT* __restrict__ x, const DT* __restrict__ val,
    const IT* __restrict__ col, const IT* __restrict__ rp, uint64_t rows)
  {
    for(uint64_t row = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; row < rows; row += uint64_t(gridDim.x) * blockDim.x)
    {
      const DT xv = x[row];
      for(uint64_t j = uint64_t(rp[row]); j < uint64_t(rp[row + 1]); ++j)
        atomicAdd(&r[col[j]], mul(val[j], xv));
    }
  }
  template<typename DT>
  __global__ void k_scale_inplace(DT* r, DT a, uint64_t n)
  {
    for(uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
      r[i] = mul(a, r[i]);
  }

  static unsigned int grid_for(uint64_t n, int nt, unsigned int cap = 148u * 16u)
  {
    uint64_t g = (n + uint64_t(nt) - 1) / uint64_t(nt);
    if(g < 1) g = 1;
    if(g > cap) g = cap;
    return (unsigned int)g;
  }

  template<typename DT, typename IT>
  static fb_status apply_csr(DT* r, DT a, const DT* x, DT b, const DT* y, const DT* val, const IT* col,
    const IT* rp, uint64_t rows, uint64_t cols, uint64_t nnz, int transposed, void* stream)
  {
    const DT eps = sizeof(DT) == 8 ? DT(EPS64) : DT(EPS32);
    const uint64_t nout = transposed ? cols : rows;
    if(!r || !rp || (nnz && (!x || !val || !col)))
    {
      set_error("apply_csr: null pointer");
      return FB_ERR_ARG;
    }
    if(r == x)
    {
      set_error("apply_csr: r must not alias x");
      return FB_ERR_ARG;
    }
    cudaStream_t st = as_stream(stream);
    const bool use_y = !(fabs(double(b)) < double(eps));
    if(use_y && !y)
    {
      set_error("apply_csr: y is null");
      return FB_ERR_ARG;
    }
    if(nout == 0)
      return FB_OK;
    if(!transposed)
    {
      if(rows == 0)
        return FB_OK;
      unsigned int g = (unsigned int)((rows + APPLY_NT - 1) / APPLY_NT);
      k_apply_csr<DT, IT><<<g, APPLY_NT, 0, st>>>(r, a, x, b, y, val, col, rp, rows, use_y);
      FB_LAUNCHED(1);
    }
    else
    {
      k_scale_init<DT><<<grid_for(cols, 256), 256, 0, st>>>(r, y, b / a, cols, use_y);
      k_apply_csr_t<DT, IT><<<grid_for(rows, 256), 256, 0, st>>>(r, x, val, col, rp, rows);
      k_scale_inplace<DT><<<grid_for(cols, 256), 256, 0, st>>>(r, a, cols);
      FB_LAUNCHED(3);
    }
    FB_CUDA(cudaStreamSynchronize(st));
    return FB_OK;
  }

  // ------------------------------------------------------------------ BLAS-1
  template<typename DT>
  __global__ void k_axpy(DT* r, DT a, const DT* x, const DT* y, uint64_t n)
  {
    for(uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
      r[i] = add(mul(a, x[i]), y[i]);
  }
  template<typename DT>
  __global__ void k_cprod(DT* r, const DT* x, const DT* y, uint64_t n)
  {
    for(uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
      r[i] = mul(x[i], y[i]);
  }
  template<typename DT>
  __global__ void k_cinv(DT* r, const DT* x, DT s, uint64_t n)
  {
    for(uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
      r[i] = s / x[i];
  }
  template<typename DT>
  __global__ void k_scale(DT* r, const DT* x, DT s, uint64_t n)
  {
    for(uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
      r[i] = mul(x[i], s);
  }

  template<typename DT>
  __global__ void k_set_memory(DT* r, DT v, uint64_t n)
  {
    for(uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
      r[i] = v;
  }
  // one thread per row: every entry of the row scaled by the row's factor
  template<typename DT, typename IT>
  __global__ void k_scale_rows(DT* r, const DT* a, const IT* rp, const DT* x, uint64_t rows)
  {
    for(uint64_t row = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; row < rows; row += uint64_t(gridDim.x) * blockDim.x)
    {
      const DT s = x[row];
      for(uint64_t k = uint64_t(rp[row]); k < uint64_t(rp[row + 1]); ++k)
        r[k] = mul(a[k], s);
    }
  }

  // Dot products reduce in FP64 per thread (grid-stride), per block, then in the last block over
  // the block partials in block order: deterministic for a given launch shape.
  constexpr int RED_NT = 256;
  constexpr unsigned int RED_MAX_BLOCKS = 148u * 8u;

  template<typename DT>
  __global__ void __launch_bounds__(RED_NT) k_dot(const DT* __restrict__ x, const DT* __restrict__ y, uint64_t n,
    RedSlot slot, double* out)
  {
    __shared__ double sh[32];
    double s = 0.0;
    for(uint64_t i = blockIdx.x * uint64_t(RED_NT) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * RED_NT)
      s += double(x[i]) * double(y[i]);
    double total;
    if(grid_sum_last<RED_NT>(s, slot, sh, total))
      *out = total;
  }

  // Per-device scratch of the reductions: block partials, the arrival counter and the result.
  struct RedScratch
  {
    double* partials = nullptr;
    unsigned int* counter = nullptr;
    double* result = nullptr;
  };

  static fb_status red_scratch(RedScratch*& out)
  {
    static std::mutex mu;
    static std::unordered_map<int, RedScratch> per_dev;
    int dev = 0;
    FB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    auto it = per_dev.find(dev);
    if(it == per_dev.end())
    {
      RedScratch s;
      void* p = nullptr;
      FB_CUDA(cudaMalloc(&p, RED_MAX_BLOCKS * sizeof(double) + 256));
      s.partials = static_cast<double*>(p);
      s.result = reinterpret_cast<double*>(static_cast<char*>(p) + RED_MAX_BLOCKS * sizeof(double));
      s.counter = reinterpret_cast<unsigned int*>(static_cast<char*>(p) + RED_MAX_BLOCKS * sizeof(double) + 128);
      FB_CUDA(cudaMemset(s.counter, 0, sizeof(unsigned int)));
      it = per_dev.emplace(dev, s).first;
    }
    out = &it->second;
    return FB_OK;
  }

  template<typename DT>
  static fb_status dot(double& result, const DT* x, const DT* y, uint64_t n, void* stream)
  {
    if(n == 0)
    {
      result = 0.0;
      return FB_OK;
    }
    if(!x || !y)
    {
      set_error("dot: null pointer");
      return FB_ERR_ARG;
    }
    RedScratch* rs = nullptr;
    fb_status e = red_scratch(rs);
    if(e != FB_OK)
      return e;
    cudaStream_t st = as_stream(stream);
    k_dot<DT><<<grid_for(n, RED_NT, RED_MAX_BLOCKS), RED_NT, 0, st>>>(x, y, n, RedSlot{rs->partials, rs->counter}, rs->result);
    FB_LAUNCHED(1);
    FB_CUDA(cudaMemcpyAsync(&result, rs->result, sizeof(double), cudaMemcpyDeviceToHost, st));
    FB_CUDA(cudaStreamSynchronize(st));
    return FB_OK;
  }

  // ------------------------------------------------------------------ filters, diagonal, convert
  template<typename DT, typename IT>
  __global__ void k_filter_rhs(DT* v, const DT* vals, const IT* idx, uint64_t ue)
  {
    for(uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < ue; i += uint64_t(gridDim.x) * blockDim.x)
      v[idx[i]] = vals[i];
  }
  template<typename DT, typename IT>
  __global__ void k_filter_def(DT* v, const IT* idx, uint64_t ue)
  {
    for(uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < ue; i += uint64_t(gridDim.x) * blockDim.x)
      v[idx[i]] = DT(0);
  }
  template<typename IT>
  __global__ void k_diagonal(IT* diag, const IT* col, const IT* rp, uint64_t rows)
  {
    for(uint64_t row = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; row < rows; row += uint64_t(gridDim.x) * blockDim.x)
    {
      IT pos = rp[rows];
      for(IT j = rp[row]; j < rp[row + 1]; ++j)
        if(uint64_t(col[j]) == row)
        {
          pos = j;
          break;
        }
      diag[row] = pos;
    }
  }
  template<typename D, typename S>
  __global__ void k_convert(D* d, const S* s, uint64_t n)
  {
    for(uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
      d[i] = D(s[i]);
  }
} // namespace fb

using namespace fb;

#define FB_ELEMENTWISE(KERNEL, N, ...)                                                     \
  do {                                                                                     \
    if((N) == 0) return FB_OK;                                                             \
    cudaStream_t st_ = as_stream(stream);                                                  \
    KERNEL<<<grid_for((N), 256), 256, 0, st_>>>(__VA_ARGS__);                              \
    FB_LAUNCHED(1);                                                                        \
    FB_CUDA(cudaStreamSynchronize(st_));                                                   \
    return FB_OK;                                                                          \
  } while(0)

extern "C" {

const char* fb_last_error(void) { return fb::g_err.c_str(); }
const char* fb_version(void) { return "featb200 0.1 (sm_100a)"; }
uint64_t fb_kernel_launch_count(void) { return fb::g_launches.load(); }

fb_status fb_apply_csr_f64_u64(double* r, double a, const double* x, double b, const double* y,
  const double* val, const uint64_t* col_ind, const uint64_t* row_ptr, uint64_t rows, uint64_t columns,
  uint64_t used_elements, int transposed, void* stream)
{
  return apply_csr<double, uint64_t>(r, a, x, b, y, val, col_ind, row_ptr, rows, columns, used_elements, transposed, stream);
}
fb_status fb_apply_csr_f64_u32(double* r, double a, const double* x, double b, const double* y,
  const double* val, const uint32_t* col_ind, const uint32_t* row_ptr, uint64_t rows, uint64_t columns,
  uint64_t used_elements, int transposed, void* stream)
{
  return apply_csr<double, uint32_t>(r, a, x, b, y, val, col_ind, row_ptr, rows, columns, used_elements, transposed, stream);
}
fb_status fb_apply_csr_f32_u64(float* r, float a, const float* x, float b, const float* y,
  const float* val, const uint64_t* col_ind, const uint64_t* row_ptr, uint64_t rows, uint64_t columns,
  uint64_t used_elements, int transposed, void* stream)
{
  return apply_csr<float, uint64_t>(r, a, x, b, y, val, col_ind, row_ptr, rows, columns, used_elements, transposed, stream);
}
fb_status fb_apply_csr_f32_u32(float* r, float a, const float* x, float b, const float* y,
  const float* val, const uint32_t* col_ind, const uint32_t* row_ptr, uint64_t rows, uint64_t columns,
  uint64_t used_elements, int transposed, void* stream)
{
  return apply_csr<float, uint32_t>(r, a, x, b, y, val, col_ind, row_ptr, rows, columns, used_elements, transposed, stream);
}

fb_status fb_axpy_f64(double* r, double a, const double* x, const double* y, uint64_t n, void* stream)
{
  if(n && (!r || !x || !y)) { set_error("axpy: null pointer"); return FB_ERR_ARG; }
  FB_ELEMENTWISE(k_axpy<double>, n, r, a, x, y, n);
}
fb_status fb_axpy_f32(float* r, float a, const float* x, const float* y, uint64_t n, void* stream)
{
  if(n && (!r || !x || !y)) { set_error("axpy: null pointer"); return FB_ERR_ARG; }
  FB_ELEMENTWISE(k_axpy<float>, n, r, a, x, y, n);
}

fb_status fb_dot_f64(double* result, const double* x, const double* y, uint64_t n, void* stream)
{
  if(!result) { set_error("dot: null result"); return FB_ERR_ARG; }
  double v = 0.0;
  fb_status e = dot<double>(v, x, y, n, stream);
  if(e == FB_OK) *result = v;
  return e;
}
fb_status fb_dot_f32(float* result, const float* x, const float* y, uint64_t n, void* stream)
{
  if(!result) { set_error("dot: null result"); return FB_ERR_ARG; }
  double v = 0.0;
  fb_status e = dot<float>(v, x, y, n, stream);
  if(e == FB_OK) *result = float(v);
  return e;
}
fb_status fb_norm2_f64(double* result, const double* x, uint64_t n, void* stream)
{
  if(!result) { set_error("norm2: null result"); return FB_ERR_ARG; }
  double v = 0.0;
  fb_status e = dot<double>(v, x, x, n, stream);
  if(e == FB_OK) *result = sqrt(v);
  return e;
}
fb_status fb_norm2_f32(float* result, const float* x, uint64_t n, void* stream)
{
  if(!result) { set_error("norm2: null result"); return FB_ERR_ARG; }
  double v = 0.0;
  fb_status e = dot<float>(v, x, x, n, stream);
  if(e == FB_OK) *result = float(sqrt(v));
  return e;
}

fb_status fb_component_product_f64(double* r, const double* x, const double* y, uint64_t n, void* stream)
{
  if(n && (!r || !x || !y)) { set_error("component_product: null pointer"); return FB_ERR_ARG; }
  FB_ELEMENTWISE(k_cprod<double>, n, r, x, y, n);
}
fb_status fb_component_product_f32(float* r, const float* x, const float* y, uint64_t n, void* stream)
{
  if(n && (!r || !x || !y)) { set_error("component_product: null pointer"); return FB_ERR_ARG; }
  FB_ELEMENTWISE(k_cprod<float>, n, r, x, y, n);
}
fb_status fb_component_invert_f64(double* r, const double* x, double s, uint64_t n, void* stream)
{
  if(n && (!r || !x)) { set_error("component_invert: null pointer"); return FB_ERR_ARG; }
  FB_ELEMENTWISE(k_cinv<double>, n, r, x, s, n);
}
fb_status fb_component_invert_f32(float* r, const float* x, float s, uint64_t n, void* stream)
{
  if(n && (!r || !x)) { set_error("component_invert: null pointer"); return FB_ERR_ARG; }
  FB_ELEMENTWISE(k_cinv<float>, n, r, x, s, n);
}
fb_status fb_scale_f64(double* r, const double* x, double s, uint64_t n, void* stream)
{
  if(n && (!r || !x)) { set_error("scale: null pointer"); return FB_ERR_ARG; }
  FB_ELEMENTWISE(k_scale<double>, n, r, x, s, n);
}
fb_status fb_scale_f32(float* r, const float* x, float s, uint64_t n, void* stream)
{
  if(n && (!r || !x)) { set_error("scale: null pointer"); return FB_ERR_ARG; }
  FB_ELEMENTWISE(k_scale<float>, n, r, x, s, n);
}

fb_status fb_unit_filter_rhs_f64_u64(double* v, const double* vals, const uint64_t* idx, uint64_t ue, void* stream)
{
  if(ue && (!v || !vals || !idx)) { set_error("filter_rhs: null pointer"); return FB_ERR_ARG; }
  FB_ELEMENTWISE((k_filter_rhs<double, uint64_t>), ue, v, vals, idx, ue);
}
fb_status fb_unit_filter_def_f64_u64(double* v, const uint64_t* idx, uint64_t ue, void* stream)
{
  if(ue && (!v || !idx)) { set_error("filter_def: null pointer"); return FB_ERR_ARG; }
  FB_ELEMENTWISE((k_filter_def<double, uint64_t>), ue, v, idx, ue);
}
fb_status fb_unit_filter_rhs_f32_u32(float* v, const float* vals, const uint32_t* idx, uint64_t ue, void* stream)
{
  if(ue && (!v || !vals || !idx)) { set_error("filter_rhs: null pointer"); return FB_ERR_ARG; }
  FB_ELEMENTWISE((k_filter_rhs<float, uint32_t>), ue, v, vals, idx, ue);
}
fb_status fb_unit_filter_def_f32_u32(float* v, const uint32_t* idx, uint64_t ue, void* stream)
{
  if(ue && (!v || !idx)) { set_error("filter_def: null pointer"); return FB_ERR_ARG; }
  FB_ELEMENTWISE((k_filter_def<float, uint32_t>), ue, v, idx, ue);
}

fb_status fb_diagonal_csr_u64(uint64_t* diag, const uint64_t* col_ind, const uint64_t* row_ptr, uint64_t rows, void* stream)
{
  if(rows && (!diag || !col_ind || !row_ptr)) { set_error("diagonal: null pointer"); return FB_ERR_ARG; }
  FB_ELEMENTWISE(k_diagonal<uint64_t>, rows, diag, col_ind, row_ptr, rows);
}

fb_status fb_set_memory_f64(double* r, double value, uint64_t n, void* stream)
{
  if(n && !r) { set_error("set_memory: null pointer"); return FB_ERR_ARG; }
  FB_ELEMENTWISE(k_set_memory<double>, n, r, value, n);
}
fb_status fb_set_memory_f32(float* r, float value, uint64_t n, void* stream)
{
  if(n && !r) { set_error("set_memory: null pointer"); return FB_ERR_ARG; }
  FB_ELEMENTWISE(k_set_memory<float>, n, r, value, n);
}
fb_status fb_set_memory_u64(uint64_t* r, uint64_t value, uint64_t n, void* stream)
{
  if(n && !r) { set_error("set_memory: null pointer"); return FB_ERR_ARG; }
  FB_ELEMENTWISE(k_set_memory<uint64_t>, n, r, value, n);
}
fb_status fb_set_memory_u32(uint32_t* r, uint32_t value, uint64_t n, void* stream)
{
  if(n && !r) { set_error("set_memory: null pointer"); return FB_ERR_ARG; }
  FB_ELEMENTWISE(k_set_memory<uint32_t>, n, r, value, n);
}

fb_status fb_scale_rows_csr_f64_u64(double* r, const double* val, const uint64_t* row_ptr, const double* x,
                                    uint64_t rows, void* stream)
{
  if(rows && (!r || !val || !row_ptr || !x)) { set_error("scale_rows: null pointer"); return FB_ERR_ARG; }
  FB_ELEMENTWISE((k_scale_rows<double, uint64_t>), rows, r, val, row_ptr, x, rows);
}

fb_status fb_convert_f64_to_f32(float* dst, const double* src, uint64_t n, void* stream)
{
  if(n && (!dst || !src)) { set_error("convert: null pointer"); return FB_ERR_ARG; }
  FB_ELEMENTWISE((k_convert<float, double>), n, dst, src, n);
}
fb_status fb_convert_f32_to_f64(double* dst, const float* src, uint64_t n, void* stream)
{
  if(n && (!dst || !src)) { set_error("convert: null pointer"); return FB_ERR_ARG; }
  FB_ELEMENTWISE((k_convert<double, float>), n, dst, src, n);
}

} // extern "C"
