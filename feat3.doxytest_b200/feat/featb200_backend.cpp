// FEAT's CUDA backend entry points implemented on libfeatb200.
//
// A FEAT build with FEAT_HAVE_CUDA compiles this file INSTEAD of kernel/util/cuda_util.cu and the
// kernel/lafem/arch/*.cu files of the ops below, and links libfeatb200.so.  FEAT's dispatch is left
// as it is: with Backend::set_preferred_backend(PreferredBackend::cuda) every container op of the
// solve path (kernel/backend.hpp:55-92, BACKEND_SKELETON_*) lands here, on the managed memory that
// MemoryPool allocates (kernel/util/memory_pool.hpp:79-104).  Like FEAT's own CUDA backend, every op
// returns after the device finished it (each of FEAT's *_cuda functions ends in
// cudaDeviceSynchronize), so host code may read the containers right after the call; failures throw
// FEAT's InternalError with the library's message.
//
// Entry points (FEAT declaration -> library call):
//   Util::cuda_malloc_managed / cuda_free / cuda_copy / cuda_synchronize   (kernel/util/cuda_util.hpp)
//                                  -> cudaMallocManaged / cudaFree / cudaMemcpy / cudaDeviceSynchronize
//   Util::cuda_set_memory<DT>      -> fb_set_memory_*          (cuda_util.cu:202-219)
//   Util::cuda_convert<DT1, DT2>   -> fb_convert_*             (cuda_util.cu:228-262)
//   Arch::Apply::csr_cuda          -> fb_apply_csr_*           (apply.hpp:240, apply.cu:176-261)
//   Arch::Axpy::value_cuda         -> fb_axpy_*                (axpy.hpp:53, axpy.cu:18-75)
//   Arch::DotProduct::value_cuda   -> fb_dot_*                 (dot_product.hpp:53, dot_product.cu:21-61)
//   Arch::Norm2::value_cuda        -> fb_norm2_*               (norm.hpp:53, norm.cu:20-59)
//   Arch::Scale::value_cuda        -> fb_scale_*               (scale.hpp:54)
//   Arch::ComponentProduct::value_cuda -> fb_component_product_* (component_product.hpp:53)
//   Arch::ComponentInvert::value_cuda  -> fb_component_invert_*  (component_invert.hpp:50)
//   Arch::UnitFilter::filter_rhs_cuda / filter_def_cuda -> fb_unit_filter_* (unit_filter.hpp:67-70)
//   Arch::Diagonal::csr_cuda       -> fb_diagonal_csr_u64      (diagonal.hpp:43)
//   Arch::ScaleRows::csr_cuda      -> fb_scale_rows_csr_f64_u64 (scale_row_col.hpp:52)
#include <kernel/base_header.hpp>
#include <kernel/util/cuda_util.hpp>
#include <kernel/util/exception.hpp>
#include <kernel/lafem/arch/apply.hpp>
#include <kernel/lafem/arch/axpy.hpp>
#include <kernel/lafem/arch/dot_product.hpp>
#include <kernel/lafem/arch/norm.hpp>
#include <kernel/lafem/arch/scale.hpp>
#include <kernel/lafem/arch/component_product.hpp>
#include <kernel/lafem/arch/component_invert.hpp>
#include <kernel/lafem/arch/unit_filter.hpp>
#include <kernel/lafem/arch/diagonal.hpp>
#include <kernel/lafem/arch/scale_row_col.hpp>

#include <cuda_runtime_api.h>
#include <featb200.h>

#include <cstdint>
#include <string>
#include <type_traits>

static_assert(sizeof(FEAT::Index) == sizeof(std::uint64_t), "this binding expects 64-bit FEAT::Index");

namespace
{
  // a failed library call becomes FEAT's InternalError; a successful one is complete on return
  inline void fb_check(fb_status st, const char* what)
  {
    if(st != FB_OK)
      throw FEAT::InternalError(what, __FILE__, __LINE__, std::string("libfeatb200: ") + fb_last_error());
  }

  inline void cuda_check(cudaError_t e, const char* what)
  {
    if(e != cudaSuccess)
      throw FEAT::InternalError(what, __FILE__, __LINE__, std::string("CUDA: ") + cudaGetErrorString(e));
  }

  // a type combination FEAT's headers reference but the library does not provide: fails loudly
  [[noreturn]] inline void unsupported(const char* what)
  {
    throw FEAT::InternalError(what, __FILE__, __LINE__, "libfeatb200 provides no kernel for this value/index type");
  }

  inline const std::uint64_t* u64(const unsigned long* p) { return reinterpret_cast<const std::uint64_t*>(p); }
  inline std::uint64_t* u64(unsigned long* p) { return reinterpret_cast<std::uint64_t*>(p); }
  inline const std::uint32_t* u32(const unsigned int* p) { return reinterpret_cast<const std::uint32_t*>(p); }

  // overloads per value / index type
  inline fb_status fbx_set_memory(double* p, double v, std::uint64_t n) { return fb_set_memory_f64(p, v, n, nullptr); }
  inline fb_status fbx_set_memory(float* p, float v, std::uint64_t n) { return fb_set_memory_f32(p, v, n, nullptr); }
  inline fb_status fbx_set_memory(unsigned long* p, unsigned long v, std::uint64_t n)
  { return fb_set_memory_u64(u64(p), std::uint64_t(v), n, nullptr); }
  inline fb_status fbx_set_memory(unsigned int* p, unsigned int v, std::uint64_t n)
  { return fb_set_memory_u32(reinterpret_cast<std::uint32_t*>(p), std::uint32_t(v), n, nullptr); }

  inline fb_status fbx_convert(float* d, const double* s, std::uint64_t n) { return fb_convert_f64_to_f32(d, s, n, nullptr); }
  inline fb_status fbx_convert(double* d, const float* s, std::uint64_t n) { return fb_convert_f32_to_f64(d, s, n, nullptr); }

  inline fb_status fbx_apply(double* r, double a, const double* x, double b, const double* y, const double* val,
    const unsigned long* col, const unsigned long* rp, std::uint64_t rows, std::uint64_t cols, std::uint64_t nnz, int tr)
  { return fb_apply_csr_f64_u64(r, a, x, b, y, val, u64(col), u64(rp), rows, cols, nnz, tr, nullptr); }
  inline fb_status fbx_apply(double* r, double a, const double* x, double b, const double* y, const double* val,
    const unsigned int* col, const unsigned int* rp, std::uint64_t rows, std::uint64_t cols, std::uint64_t nnz, int tr)
  { return fb_apply_csr_f64_u32(r, a, x, b, y, val, u32(col), u32(rp), rows, cols, nnz, tr, nullptr); }
  inline fb_status fbx_apply(float* r, float a, const float* x, float b, const float* y, const float* val,
    const unsigned long* col, const unsigned long* rp, std::uint64_t rows, std::uint64_t cols, std::uint64_t nnz, int tr)
  { return fb_apply_csr_f32_u64(r, a, x, b, y, val, u64(col), u64(rp), rows, cols, nnz, tr, nullptr); }
  inline fb_status fbx_apply(float* r, float a, const float* x, float b, const float* y, const float* val,
    const unsigned int* col, const unsigned int* rp, std::uint64_t rows, std::uint64_t cols, std::uint64_t nnz, int tr)
  { return fb_apply_csr_f32_u32(r, a, x, b, y, val, u32(col), u32(rp), rows, cols, nnz, tr, nullptr); }

  inline fb_status fbx_axpy(double* r, double a, const double* x, const double* y, std::uint64_t n)
  { return fb_axpy_f64(r, a, x, y, n, nullptr); }
  inline fb_status fbx_axpy(float* r, float a, const float* x, const float* y, std::uint64_t n)
  { return fb_axpy_f32(r, a, x, y, n, nullptr); }
  inline fb_status fbx_dot(double* out, const double* x, const double* y, std::uint64_t n)
  { return fb_dot_f64(out, x, y, n, nullptr); }
  inline fb_status fbx_dot(float* out, const float* x, const float* y, std::uint64_t n)
  { return fb_dot_f32(out, x, y, n, nullptr); }
  inline fb_status fbx_norm2(double* out, const double* x, std::uint64_t n) { return fb_norm2_f64(out, x, n, nullptr); }
  inline fb_status fbx_norm2(float* out, const float* x, std::uint64_t n) { return fb_norm2_f32(out, x, n, nullptr); }
  inline fb_status fbx_scale(double* r, const double* x, double s, std::uint64_t n) { return fb_scale_f64(r, x, s, n, nullptr); }
  inline fb_status fbx_scale(float* r, const float* x, float s, std::uint64_t n) { return fb_scale_f32(r, x, s, n, nullptr); }
  inline fb_status fbx_cprod(double* r, const double* x, const double* y, std::uint64_t n)
  { return fb_component_product_f64(r, x, y, n, nullptr); }
  inline fb_status fbx_cprod(float* r, const float* x, const float* y, std::uint64_t n)
  { return fb_component_product_f32(r, x, y, n, nullptr); }
  inline fb_status fbx_cinv(double* r, const double* x, double s, std::uint64_t n)
  { return fb_component_invert_f64(r, x, s, n, nullptr); }
  inline fb_status fbx_cinv(float* r, const float* x, float s, std::uint64_t n)
  { return fb_component_invert_f32(r, x, s, n, nullptr); }
  inline fb_status fbx_filter_rhs(double* v, const double* e, const unsigned long* idx, std::uint64_t ue)
  { return fb_unit_filter_rhs_f64_u64(v, e, u64(idx), ue, nullptr); }
  inline fb_status fbx_filter_def(double* v, const unsigned long* idx, std::uint64_t ue)
  { return fb_unit_filter_def_f64_u64(v, u64(idx), ue, nullptr); }
  inline fb_status fbx_filter_rhs(float* v, const float* e, const unsigned int* idx, std::uint64_t ue)
  { return fb_unit_filter_rhs_f32_u32(v, e, u32(idx), ue, nullptr); }
  inline fb_status fbx_filter_def(float* v, const unsigned int* idx, std::uint64_t ue)
  { return fb_unit_filter_def_f32_u32(v, u32(idx), ue, nullptr); }
} // namespace

namespace FEAT
{
  namespace Util
  {
    // launch-shape settings of FEAT's own kernels; the library sizes its launches itself, so they
    // are recorded and otherwise unused
    Index cuda_blocksize_misc = 256;
    Index cuda_blocksize_reduction = 256;
    Index cuda_blocksize_spmv = 256;
    Index cuda_blocksize_axpy = 256;

    void cuda_set_blocksize(Index misc, Index reduction, Index spmv, Index axpy)
    {
      cuda_blocksize_misc = misc;
      cuda_blocksize_reduction = reduction;
      cuda_blocksize_spmv = spmv;
      cuda_blocksize_axpy = axpy;
    }

    void cuda_set_device(const int device) { cuda_check(cudaSetDevice(device), __func__); }

    void cuda_check_last_error() { cuda_check(cudaGetLastError(), __func__); }

    void* cuda_get_device_pointer(void* host)
    {
      void* d = nullptr;
      cuda_check(cudaHostGetDevicePointer(&d, host, 0), __func__);
      return d;
    }

    void* cuda_malloc_managed(const Index bytes)
    {
      void* p = nullptr;
      cuda_check(cudaMallocManaged(&p, bytes), __func__);
      return p;
    }

    void cuda_free(void* address)
    {
      if(address != nullptr)
        cuda_check(cudaFree(address), __func__);
    }

    // one device per process: rank modulo the GPUs of the node (cuda_util.cu:100-111); the
    // library needs managed-memory support for FEAT's containers
    void cuda_initialize(int rank, int /*ranks_per_node*/, int /*ranks_per_uma*/, int gpus_per_node)
    {
      const int device = gpus_per_node > 0 ? rank % gpus_per_node : 0;
      cuda_check(cudaSetDevice(device), __func__);
      int mm = 0;
      cuda_check(cudaDeviceGetAttribute(&mm, cudaDevAttrManagedMemory, device), __func__);
      if(mm != 1)
        throw InternalError(__func__, __FILE__, __LINE__, "selected CUDA device does not support managed memory");
    }

    void cuda_finalize() { cuda_check(cudaDeviceSynchronize(), __func__); }

    void cuda_synchronize() { cuda_check(cudaDeviceSynchronize(), __func__); }

    void cuda_reset_device() { cuda_check(cudaDeviceReset(), __func__); }

    void cuda_copy(void* dest, const void* src, const Index bytes)
    {
      cuda_check(cudaMemcpy(dest, src, bytes, cudaMemcpyDefault), __func__);
    }

    void cuda_reset_algos() {}

    template<typename DT_>
    void cuda_set_memory(DT_* address, const DT_ val, const Index count)
    {
      fb_check(fbx_set_memory(address, val, count), __func__);
    }

    template<typename DT1_, typename DT2_>
    void cuda_convert(DT1_* dest, const DT2_* src, const Index count)
    {
      fb_check(fbx_convert(dest, src, count), __func__);
    }

    template void cuda_set_memory<double>(double*, const double, const Index);
    template void cuda_set_memory<float>(float*, const float, const Index);
    template void cuda_set_memory<unsigned long>(unsigned long*, const unsigned long, const Index);
    template void cuda_set_memory<unsigned int>(unsigned int*, const unsigned int, const Index);
    template void cuda_convert<float, double>(float*, const double*, const Index);
    template void cuda_convert<double, float>(double*, const float*, const Index);
  } // namespace Util

  namespace LAFEM
  {
    namespace Arch
    {
      template<typename DT_, typename IT_>
      void Apply::csr_cuda(DT_* r, const DT_ a, const DT_* const x, const DT_ b, const DT_* const y,
        const DT_* const val, const IT_* const col_ind, const IT_* const row_ptr, const Index rows,
        const Index columns, const Index used_elements, const bool transposed)
      {
        fb_check(fbx_apply(r, a, x, b, y, val, col_ind, row_ptr, rows, columns, used_elements, transposed ? 1 : 0), __func__);
      }
      template void Apply::csr_cuda<double, unsigned long>(double*, const double, const double* const, const double,
        const double* const, const double* const, const unsigned long* const, const unsigned long* const, const Index,
        const Index, const Index, const bool);
      template void Apply::csr_cuda<double, unsigned int>(double*, const double, const double* const, const double,
        const double* const, const double* const, const unsigned int* const, const unsigned int* const, const Index,
        const Index, const Index, const bool);
      template void Apply::csr_cuda<float, unsigned long>(float*, const float, const float* const, const float,
        const float* const, const float* const, const unsigned long* const, const unsigned long* const, const Index,
        const Index, const Index, const bool);
      template void Apply::csr_cuda<float, unsigned int>(float*, const float, const float* const, const float,
        const float* const, const float* const, const unsigned int* const, const unsigned int* const, const Index,
        const Index, const Index, const bool);

      template<typename DT_>
      void Axpy::value_cuda(DT_* r, const DT_ a, const DT_* const x, const DT_* const y, const Index size)
      {
        fb_check(fbx_axpy(r, a, x, y, size), __func__);
      }
      template void Axpy::value_cuda<double>(double*, const double, const double* const, const double* const, const Index);
      template void Axpy::value_cuda<float>(float*, const float, const float* const, const float* const, const Index);

      template<typename DT_>
      DT_ DotProduct::value_cuda(const DT_* const x, const DT_* const y, const Index size)
      {
        DT_ out = DT_(0);
        fb_check(fbx_dot(&out, x, y, size), __func__);
        return out;
      }
      template double DotProduct::value_cuda<double>(const double* const, const double* const, const Index);
      template float DotProduct::value_cuda<float>(const float* const, const float* const, const Index);

      template<typename DT_>
      DT_ Norm2::value_cuda(const DT_* const x, const Index size)
      {
        DT_ out = DT_(0);
        fb_check(fbx_norm2(&out, x, size), __func__);
        return out;
      }
      template double Norm2::value_cuda<double>(const double* const, const Index);
      template float Norm2::value_cuda<float>(const float* const, const Index);

      template<typename DT_>
      void Scale::value_cuda(DT_* r, const DT_* const x, const DT_ s, const Index size)
      {
        fb_check(fbx_scale(r, x, s, size), __func__);
      }
      template void Scale::value_cuda<double>(double*, const double* const, const double, const Index);
      template void Scale::value_cuda<float>(float*, const float* const, const float, const Index);

      template<typename DT_>
      void ComponentProduct::value_cuda(DT_* r, const DT_* const x, const DT_* const y, const Index size)
      {
        fb_check(fbx_cprod(r, x, y, size), __func__);
      }
      template void ComponentProduct::value_cuda<double>(double*, const double* const, const double* const, const Index);
      template void ComponentProduct::value_cuda<float>(float*, const float* const, const float* const, const Index);

      template<typename DT_>
      void ComponentInvert::value_cuda(DT_* r, const DT_* const x, const DT_ s, const Index size)
      {
        fb_check(fbx_cinv(r, x, s, size), __func__);
      }
      template void ComponentInvert::value_cuda<double>(double*, const double* const, const double, const Index);
      template void ComponentInvert::value_cuda<float>(float*, const float* const, const float, const Index);

      // (double, u64) and (float, u32): the library's index types per value type
      template<typename DT_, typename IT_>
      void UnitFilter::filter_rhs_cuda(DT_* v, const DT_* const sv_elements, const IT_* const sv_indices, const Index ue)
      {
        if constexpr((std::is_same_v<DT_, double> && std::is_same_v<IT_, unsigned long>) ||
                     (std::is_same_v<DT_, float> && std::is_same_v<IT_, unsigned int>))
          fb_check(fbx_filter_rhs(v, sv_elements, sv_indices, ue), __func__);
        else
          unsupported(__func__);
      }
      template<typename DT_, typename IT_>
      void UnitFilter::filter_def_cuda(DT_* v, const IT_* const sv_indices, const Index ue)
      {
        if constexpr((std::is_same_v<DT_, double> && std::is_same_v<IT_, unsigned long>) ||
                     (std::is_same_v<DT_, float> && std::is_same_v<IT_, unsigned int>))
          fb_check(fbx_filter_def(v, sv_indices, ue), __func__);
        else
          unsupported(__func__);
      }
      template void UnitFilter::filter_rhs_cuda<double, unsigned long>(double*, const double* const,
        const unsigned long* const, const Index);
      template void UnitFilter::filter_def_cuda<double, unsigned long>(double*, const unsigned long* const, const Index);
      template void UnitFilter::filter_rhs_cuda<float, unsigned int>(float*, const float* const,
        const unsigned int* const, const Index);
      template void UnitFilter::filter_def_cuda<float, unsigned int>(float*, const unsigned int* const, const Index);

      template<typename IT_>
      void Diagonal::csr_cuda(IT_* diag, const IT_* const col_ind, const IT_* const row_ptr, const Index rows)
      {
        if constexpr(std::is_same_v<IT_, unsigned long>)
          fb_check(fb_diagonal_csr_u64(u64(diag), u64(col_ind), u64(row_ptr), rows, nullptr), __func__);
        else
          unsupported(__func__);
      }
      template void Diagonal::csr_cuda<unsigned long>(unsigned long*, const unsigned long* const,
        const unsigned long* const, const Index);

      template<typename DT_, typename IT_>
      void ScaleRows::csr_cuda(DT_* r, const DT_* const a, const IT_* const /*col_ind*/, const IT_* const row_ptr,
        const DT_* const x, const Index rows, const Index, const Index)
      {
        if constexpr(std::is_same_v<DT_, double> && std::is_same_v<IT_, unsigned long>)
          fb_check(fb_scale_rows_csr_f64_u64(r, a, u64(row_ptr), x, rows, nullptr), __func__);
        else
          unsupported(__func__);
      }
      template void ScaleRows::csr_cuda<double, unsigned long>(double*, const double* const, const unsigned long* const,
        const unsigned long* const, const double* const, const Index, const Index, const Index);
    } // namespace Arch
  } // namespace LAFEM
} // namespace FEAT
