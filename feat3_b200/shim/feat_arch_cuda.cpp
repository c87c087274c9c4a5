// FEAT3-side binding of the LAFEM arch layer for Mem::CUDA onto libfeat3_b200.
//
// A FEAT3 build compiles this file in place of its own CUDA backend sources of these
// operations (kernel/lafem/arch/{apply,axpy,dot_product,norm,component_product,
// component_invert,scale,diagonal,unit_filter}.cu) and links libfeat3_b200.so. It defines the
// static member templates that the reference's headers declare for Mem::CUDA and instantiates
// them for float and double and for both of FEAT3's index types (unsigned int, and the default
// Index = unsigned long, kernel/base_header.hpp:95-97), so SparseMatrixCSR/SparseMatrixELL::apply,
// DenseVector::axpy/dot/norm2/component_product/..., UnitFilter and the solver templates above
// them run on the sm_100a kernels without edits.
//
// Semantics kept from the reference:
//  * every call is issued on the legacy default stream, the stream the reference uses;
//  * DotProduct / Norm2 return the value to the host, so they synchronise, as the reference's
//    host-pointer-mode cuBLAS calls do (kernel/lafem/arch/dot_product.cu:24-64, norm.cu:24-60);
//  * a non-zero status of the library becomes the reference's InternalError
//    (kernel/util/exception.hpp:96-139), thrown on the caller's side of the C ABI.
// The 64-bit index overloads read the caller's arrays as they are; nothing is allocated.
#include <kernel/lafem/arch/apply.hpp>
#include <kernel/lafem/arch/axpy.hpp>
#include <kernel/lafem/arch/component_invert.hpp>
#include <kernel/lafem/arch/component_product.hpp>
#include <kernel/lafem/arch/diagonal.hpp>
#include <kernel/lafem/arch/dot_product.hpp>
#include <kernel/lafem/arch/norm.hpp>
#include <kernel/lafem/arch/scale.hpp>
#include <kernel/lafem/arch/unit_filter.hpp>
#include <kernel/util/exception.hpp>
#include <kernel/util/string.hpp>

#include <feat3_b200.h>

#include <type_traits>

static_assert(std::is_same<unsigned long, uint64_t>::value, "FEAT3's Index must be the library's 64-bit index");

namespace FEAT
{
  namespace LAFEM
  {
    namespace Arch
    {
      namespace
      {
        inline void fb_status(int st, const char* func, const char* file, int line)
        {
          if(st != FB_OK)
            throw InternalError(func, file, line, "feat3_b200 call failed with status " + stringify(st));
        }
#define FB_SHIM(call) fb_status((call), __func__, __FILE__, __LINE__)

        // value type x index type -> entry point
        inline int csr_fw(double* r, double a, const double* x, double b, const double* y, const double* v,
                          const unsigned int* c, const unsigned int* p, Index m, Index n, Index z, bool t)
        { return fb_csr_apply_f64(r, a, x, b, y, v, c, p, m, n, z, t ? 1 : 0, nullptr); }
        inline int csr_fw(float* r, float a, const float* x, float b, const float* y, const float* v,
                          const unsigned int* c, const unsigned int* p, Index m, Index n, Index z, bool t)
        { return fb_csr_apply_f32(r, a, x, b, y, v, c, p, m, n, z, t ? 1 : 0, nullptr); }
        inline int csr_fw(double* r, double a, const double* x, double b, const double* y, const double* v,
                          const unsigned long* c, const unsigned long* p, Index m, Index n, Index z, bool t)
        { return fb_csr_apply_f64_u64(r, a, x, b, y, v, c, p, m, n, z, t ? 1 : 0, nullptr); }
        inline int csr_fw(float* r, float a, const float* x, float b, const float* y, const float* v,
                          const unsigned long* c, const unsigned long* p, Index m, Index n, Index z, bool t)
        { return fb_csr_apply_f32_u64(r, a, x, b, y, v, c, p, m, n, z, t ? 1 : 0, nullptr); }

        inline int ell_fw(double* r, double a, const double* x, double b, const double* y, const double* v,
                          const unsigned int* c, const unsigned int* cs, const unsigned int* cl, Index C, Index m)
        { return fb_ell_apply_f64(r, a, x, b, y, v, c, cs, cl, C, m, nullptr); }
        inline int ell_fw(float* r, float a, const float* x, float b, const float* y, const float* v,
                          const unsigned int* c, const unsigned int* cs, const unsigned int* cl, Index C, Index m)
        { return fb_ell_apply_f32(r, a, x, b, y, v, c, cs, cl, C, m, nullptr); }
        inline int ell_fw(double* r, double a, const double* x, double b, const double* y, const double* v,
                          const unsigned long* c, const unsigned long* cs, const unsigned long* cl, Index C, Index m)
        { return fb_ell_apply_f64_u64(r, a, x, b, y, v, c, cs, cl, C, m, nullptr); }
        inline int ell_fw(float* r, float a, const float* x, float b, const float* y, const float* v,
                          const unsigned long* c, const unsigned long* cs, const unsigned long* cl, Index C, Index m)
        { return fb_ell_apply_f32_u64(r, a, x, b, y, v, c, cs, cl, C, m, nullptr); }

        inline int diag_csr_fw(double* d, const double* v, const unsigned int* c, const unsigned int* p, Index m)
        { return fb_diagonal_csr_f64(d, v, c, p, m, nullptr); }
        inline int diag_csr_fw(float* d, const float* v, const unsigned int* c, const unsigned int* p, Index m)
        { return fb_diagonal_csr_f32(d, v, c, p, m, nullptr); }
        inline int diag_csr_fw(double* d, const double* v, const unsigned long* c, const unsigned long* p, Index m)
        { return fb_diagonal_csr_f64_u64(d, v, c, p, m, nullptr); }
        inline int diag_csr_fw(float* d, const float* v, const unsigned long* c, const unsigned long* p, Index m)
        { return fb_diagonal_csr_f32_u64(d, v, c, p, m, nullptr); }

        inline int diag_ell_fw(double* d, const double* v, const unsigned int* c, const unsigned int* cs,
                               const unsigned int* cl, Index C, Index m)
        { return fb_diagonal_ell_f64(d, v, c, cs, cl, C, m, nullptr); }
        inline int diag_ell_fw(float* d, const float* v, const unsigned int* c, const unsigned int* cs,
                               const unsigned int* cl, Index C, Index m)
        { return fb_diagonal_ell_f32(d, v, c, cs, cl, C, m, nullptr); }
        inline int diag_ell_fw(double* d, const double* v, const unsigned long* c, const unsigned long* cs,
                               const unsigned long* cl, Index C, Index m)
        { return fb_diagonal_ell_f64_u64(d, v, c, cs, cl, C, m, nullptr); }
        inline int diag_ell_fw(float* d, const float* v, const unsigned long* c, const unsigned long* cs,
                               const unsigned long* cl, Index C, Index m)
        { return fb_diagonal_ell_f32_u64(d, v, c, cs, cl, C, m, nullptr); }

        inline int rhs_fw(double* v, const double* e, const unsigned int* i, Index n)
        { return fb_unit_filter_rhs_f64(v, e, i, n, nullptr); }
        inline int rhs_fw(float* v, const float* e, const unsigned int* i, Index n)
        { return fb_unit_filter_rhs_f32(v, e, i, n, nullptr); }
        inline int rhs_fw(double* v, const double* e, const unsigned long* i, Index n)
        { return fb_unit_filter_rhs_f64_u64(v, e, i, n, nullptr); }
        inline int rhs_fw(float* v, const float* e, const unsigned long* i, Index n)
        { return fb_unit_filter_rhs_f32_u64(v, e, i, n, nullptr); }
        inline int def_fw(double* v, const unsigned int* i, Index n) { return fb_unit_filter_def_f64(v, i, n, nullptr); }
        inline int def_fw(float* v, const unsigned int* i, Index n) { return fb_unit_filter_def_f32(v, i, n, nullptr); }
        inline int def_fw(double* v, const unsigned long* i, Index n) { return fb_unit_filter_def_f64_u64(v, i, n, nullptr); }
        inline int def_fw(float* v, const unsigned long* i, Index n) { return fb_unit_filter_def_f32_u64(v, i, n, nullptr); }

        inline int axpy_fw(double* r, double a, const double* x, const double* y, Index n)
        { return fb_axpy_f64(r, a, x, y, n, nullptr); }
        inline int axpy_fw(float* r, float a, const float* x, const float* y, Index n)
        { return fb_axpy_f32(r, a, x, y, n, nullptr); }
        inline int dot_fw(const double* x, const double* y, Index n, double* out) { return fb_dot_f64_sync(x, y, n, out, nullptr); }
        inline int dot_fw(const float* x, const float* y, Index n, double* out) { return fb_dot_f32_sync(x, y, n, out, nullptr); }
        inline int norm_fw(const double* x, Index n, double* out) { return fb_norm2_f64_sync(x, n, out, nullptr); }
        inline int norm_fw(const float* x, Index n, double* out) { return fb_norm2_f32_sync(x, n, out, nullptr); }
        inline int cprod_fw(double* r, const double* x, const double* y, Index n)
        { return fb_component_product_f64(r, x, y, n, nullptr); }
        inline int cprod_fw(float* r, const float* x, const float* y, Index n)
        { return fb_component_product_f32(r, x, y, n, nullptr); }
        inline int cinv_fw(double* r, const double* x, double s, Index n) { return fb_component_invert_f64(r, x, s, n, nullptr); }
        inline int cinv_fw(float* r, const float* x, float s, Index n) { return fb_component_invert_f32(r, x, s, n, nullptr); }
        inline int scale_fw(double* r, const double* x, double s, Index n) { return fb_scale_f64(r, x, s, n, nullptr); }
        inline int scale_fw(float* r, const float* x, float s, Index n) { return fb_scale_f32(r, x, s, n, nullptr); }
      } // namespace

      // ---- Apply (kernel/lafem/arch/apply.hpp:271-296)
      template <typename DT_>
      void Apply<Mem::CUDA>::csr(DT_ * r, const DT_ a, const DT_ * const x, const DT_ b, const DT_ * const y,
                                 const DT_ * const val, const unsigned int * const col_ind,
                                 const unsigned int * const row_ptr, const Index rows, const Index columns,
                                 const Index used_elements, const bool transposed)
      {
        FB_SHIM(csr_fw(r, a, x, b, y, val, col_ind, row_ptr, rows, columns, used_elements, transposed));
      }

      template <typename DT_>
      void Apply<Mem::CUDA>::csr(DT_ * r, const DT_ a, const DT_ * const x, const DT_ b, const DT_ * const y,
                                 const DT_ * const val, const unsigned long * const col_ind,
                                 const unsigned long * const row_ptr, const Index rows, const Index columns,
                                 const Index used_elements, const bool transposed)
      {
        FB_SHIM(csr_fw(r, a, x, b, y, val, col_ind, row_ptr, rows, columns, used_elements, transposed));
      }

      template <typename DT_, typename IT_>
      void Apply<Mem::CUDA>::ell(DT_ * r, const DT_ a, const DT_ * const x, const DT_ b, const DT_ * const y,
                                 const DT_ * const val, const IT_ * const col_ind, const IT_ * const cs,
                                 const IT_ * const cl, const Index C, const Index rows)
      {
        FB_SHIM(ell_fw(r, a, x, b, y, val, col_ind, cs, cl, C, rows));
      }

      template void Apply<Mem::CUDA>::csr(float *, const float, const float * const, const float, const float * const,
        const float * const, const unsigned int * const, const unsigned int * const, const Index, const Index, const Index, const bool);
      template void Apply<Mem::CUDA>::csr(double *, const double, const double * const, const double, const double * const,
        const double * const, const unsigned int * const, const unsigned int * const, const Index, const Index, const Index, const bool);
      template void Apply<Mem::CUDA>::csr(float *, const float, const float * const, const float, const float * const,
        const float * const, const unsigned long * const, const unsigned long * const, const Index, const Index, const Index, const bool);
      template void Apply<Mem::CUDA>::csr(double *, const double, const double * const, const double, const double * const,
        const double * const, const unsigned long * const, const unsigned long * const, const Index, const Index, const Index, const bool);
      template void Apply<Mem::CUDA>::ell(float *, const float, const float * const, const float, const float * const,
        const float * const, const unsigned int * const, const unsigned int * const, const unsigned int * const, const Index, const Index);
      template void Apply<Mem::CUDA>::ell(double *, const double, const double * const, const double, const double * const,
        const double * const, const unsigned int * const, const unsigned int * const, const unsigned int * const, const Index, const Index);
      template void Apply<Mem::CUDA>::ell(float *, const float, const float * const, const float, const float * const,
        const float * const, const unsigned long * const, const unsigned long * const, const unsigned long * const, const Index, const Index);
      template void Apply<Mem::CUDA>::ell(double *, const double, const double * const, const double, const double * const,
        const double * const, const unsigned long * const, const unsigned long * const, const unsigned long * const, const Index, const Index);

      // ---- Axpy, DotProduct, Norm2, ComponentProduct, ComponentInvert, Scale
      template <typename DT_>
      void Axpy<Mem::CUDA>::dv(DT_ * r, const DT_ a, const DT_ * const x, const DT_ * const y, const Index size)
      {
        FB_SHIM(axpy_fw(r, a, x, y, size));
      }

      template <typename DT_>
      DT_ DotProduct<Mem::CUDA>::value(const DT_ * const x, const DT_ * const y, const Index size)
      {
        double out = 0.0;
        FB_SHIM(dot_fw(x, y, size, &out));
        return DT_(out);
      }

      template <typename DT_>
      DT_ Norm2<Mem::CUDA>::value(const DT_ * const x, const Index size)
      {
        double out = 0.0;
        FB_SHIM(norm_fw(x, size, &out));
        return DT_(out);
      }

      template <typename DT_>
      void ComponentProduct<Mem::CUDA>::value(DT_ * r, const DT_ * const x, const DT_ * const y, const Index size)
      {
        FB_SHIM(cprod_fw(r, x, y, size));
      }

      template <typename DT_>
      void ComponentInvert<Mem::CUDA>::value(DT_ * r, const DT_ * const x, const DT_ s, const Index size)
      {
        FB_SHIM(cinv_fw(r, x, s, size));
      }

      template <typename DT_>
      void Scale<Mem::CUDA>::value(DT_ * r, const DT_ * const x, const DT_ s, const Index size)
      {
        FB_SHIM(scale_fw(r, x, s, size));
      }

      template void Axpy<Mem::CUDA>::dv(float *, const float, const float * const, const float * const, const Index);
      template void Axpy<Mem::CUDA>::dv(double *, const double, const double * const, const double * const, const Index);
      template float DotProduct<Mem::CUDA>::value(const float * const, const float * const, const Index);
      template double DotProduct<Mem::CUDA>::value(const double * const, const double * const, const Index);
      template float Norm2<Mem::CUDA>::value(const float * const, const Index);
      template double Norm2<Mem::CUDA>::value(const double * const, const Index);
      template void ComponentProduct<Mem::CUDA>::value(float *, const float * const, const float * const, const Index);
      template void ComponentProduct<Mem::CUDA>::value(double *, const double * const, const double * const, const Index);
      template void ComponentInvert<Mem::CUDA>::value(float *, const float * const, const float, const Index);
      template void ComponentInvert<Mem::CUDA>::value(double *, const double * const, const double, const Index);
      template void Scale<Mem::CUDA>::value(float *, const float * const, const float, const Index);
      template void Scale<Mem::CUDA>::value(double *, const double * const, const double, const Index);

      // ---- Diagonal (kernel/lafem/arch/diagonal.hpp:69-80) and UnitFilter (unit_filter.hpp:74-81)
      template <typename DT_, typename IT_>
      void Diagonal<Mem::CUDA>::csr(DT_ * diag, const DT_ * const val, const IT_ * const col_ind,
                                    const IT_ * const row_ptr, const Index rows)
      {
        FB_SHIM(diag_csr_fw(diag, val, col_ind, row_ptr, rows));
      }

      template <typename DT_, typename IT_>
      void Diagonal<Mem::CUDA>::ell(DT_ * diag, const DT_ * const val, const IT_ * const col_ind,
                                    const IT_ * const cs, const IT_ * const cl, const Index C, const Index rows)
      {
        FB_SHIM(diag_ell_fw(diag, val, col_ind, cs, cl, C, rows));
      }

      template <typename DT_, typename IT_>
      void UnitFilter<Mem::CUDA>::filter_rhs(DT_ * v, const DT_ * const sv_elements, const IT_ * const sv_indices,
                                             const Index ue)
      {
        FB_SHIM(rhs_fw(v, sv_elements, sv_indices, ue));
      }

      template <typename DT_, typename IT_>
      void UnitFilter<Mem::CUDA>::filter_def(DT_ * v, const IT_ * const sv_indices, const Index ue)
      {
        FB_SHIM(def_fw(v, sv_indices, ue));
      }

#define FB_SHIM_IT(DT, IT) \
      template void Diagonal<Mem::CUDA>::csr(DT *, const DT * const, const IT * const, const IT * const, const Index); \
      template void Diagonal<Mem::CUDA>::ell(DT *, const DT * const, const IT * const, const IT * const, \
                                             const IT * const, const Index, const Index); \
      template void UnitFilter<Mem::CUDA>::filter_rhs(DT *, const DT * const, const IT * const, const Index); \
      template void UnitFilter<Mem::CUDA>::filter_def(DT *, const IT * const, const Index);
      FB_SHIM_IT(float, unsigned int)
      FB_SHIM_IT(double, unsigned int)
      FB_SHIM_IT(float, unsigned long)
      FB_SHIM_IT(double, unsigned long)
#undef FB_SHIM_IT
#undef FB_SHIM
    } // namespace Arch
  } // namespace LAFEM
} // namespace FEAT
