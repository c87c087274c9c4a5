// SELL-C-sigma (C = 32) and CSR kernel family of the multigrid driver.
//
// One warp owns one chunk of 32 rows; slot j of the chunk holds the j-th entry of each of
// its 32 rows, so every value/column load of a warp is one contiguous 32-element segment
// (256 B for FP64 values, 128 B for u32 columns or FP32 values, 64 B for FP16 values).
// The kernels are grid-stride over chunks with a grid sized to the resident capacity of the
// 148 SMs, and finish with an "epilogue" functor that fuses what follows the product in the
// reference's operator sequence (defect, Jacobi update, filter, dot products).
#pragma once
#include "fb_common.cuh"

namespace fb {

// ------------------------------------------------------------------ value loads
template<typename VT> struct ValLoad;
template<> struct ValLoad<double> { __device__ __forceinline__ static double ld(const double* p) { return __ldg(p); } };
template<> struct ValLoad<float>  { __device__ __forceinline__ static float ld(const float* p) { return __ldg(p); } };
template<> struct ValLoad<__half> { __device__ __forceinline__ static float ld(const __half* p) { return __half2float(__ldg(p)); } };

// streaming (evict-first) loads for the matrix streams, which are touched once per product
__device__ __forceinline__ uint32_t ld_stream(const uint32_t* p) { return __ldcs(p); }
__device__ __forceinline__ double ld_stream(const double* p) { return __ldcs(p); }
__device__ __forceinline__ float ld_stream(const float* p) { return __ldcs(p); }
__device__ __forceinline__ float ld_stream(const __half* p) {
  unsigned short u = __ldcs(reinterpret_cast<const unsigned short*>(p));
  return __half2float(__ushort_as_half(u));
}

struct SellView {
  uint32_t nchunks;
  uint32_t rows;
  const uint32_t* cs;    // nchunks+1 chunk starts (entries)
  const uint32_t* cl;    // nchunks chunk lengths (slots)
  const uint32_t* col;   // column per entry
  const void* val;       // values (double / float / __half)
  const uint32_t* perm;  // slot row -> matrix row (nullptr = identity)
  float scale;           // FP16 storage: a_ij = scale * h_ij (1 otherwise)
};

__device__ __forceinline__ bool masked(const uint32_t* mask, uint32_t row) {
  return mask && ((__ldg(mask + (row >> 5)) >> (row & 31)) & 1u);
}

// skip predicate of the Richardson smoother: its initial defect norm is not finite or
// <= eps^2 (kernel/solver/iterative.hpp:744-766); sumsq = squared norm in FP64
template<typename T>
__device__ __forceinline__ bool smoother_skip(const double* sumsq) {
  if (!sumsq) return false;
  const double v = *((volatile const double*)sumsq);
  const double nrm = sqrt(v);
  const double e = double(eps_of<T>());
  return !(isfinite(nrm)) || nrm <= e * e;
}

// ------------------------------------------------------------------ epilogues
// r = a*s + b*y
template<typename T>
struct EpiAxpby {
  static constexpr bool kReduce = false;
  T* r; const T* y; T a, b; bool use_y;
  __device__ __forceinline__ double operator()(uint32_t row, T s) const {
    r[row] = use_y ? (s * a) + (b * y[row]) : s * a;
    return 0.0;
  }
};

// def = filter_def(rhs - A x); optional ||def||^2 and FP32 copy of def
template<typename T, bool RED, bool LOW>
struct EpiDefect {
  static constexpr bool kReduce = RED;
  T* def; const T* rhs; const uint32_t* mask; float* def32;
  __device__ __forceinline__ double operator()(uint32_t row, T s) const {
    T d = rhs[row] - s;
    if (masked(mask, row)) d = T(0);
    def[row] = d;
    if (LOW) def32[row] = float(d);
    return RED ? double(d) * double(d) : 0.0;
  }
};

// one damped-Jacobi Richardson step on the level system (fused defect + update):
//   out = x + omega * filter_cor(invd o (rhs - A x)); skip => out = s0 (0 if s0 == nullptr)
// reduction: ||filter_def(rhs - A x)||^2 (initial defect of the smoother, post-smoothing)
template<typename T, bool RED>
struct EpiJacobi {
  static constexpr bool kReduce = RED;
  const T* x; const T* rhs; const T* invd; T* out; const T* s0; const uint32_t* mask;
  const double* skip_src; T omega;
  __device__ __forceinline__ double operator()(uint32_t row, T s) const {
    if (smoother_skip<T>(skip_src)) {
      out[row] = s0 ? s0[row] : T(0);
      return 0.0;
    }
    const T d = rhs[row] - s;
    if (masked(mask, row)) {
      out[row] = x[row];
      return 0.0;
    }
    const T t = invd[row] * d;
    out[row] = omega * t + x[row];
    return RED ? double(d) * double(d) : 0.0;
  }
};

// PCG direction product: q = filter_def(A p), reduction q . p
template<typename T>
struct EpiPcgQ {
  static constexpr bool kReduce = true;
  T* q; const T* p; const uint32_t* mask;
  __device__ __forceinline__ double operator()(uint32_t row, T s) const {
    const T v = masked(mask, row) ? T(0) : s;
    q[row] = v;
    return double(v) * double(p[row]);
  }
};

// restriction: rhs_c = filter_def(R d); ||rhs_c||^2; first pre-smoothing step from zero
//   sol1 = omega * filter_cor(invd o rhs_c)   (written only when sol1 != nullptr)
template<typename T>
struct EpiRestrict {
  static constexpr bool kReduce = true;
  T* rhs; T* sol1; const T* invd; const uint32_t* mask; T omega;
  __device__ __forceinline__ double operator()(uint32_t row, T s) const {
    const bool m = masked(mask, row);
    const T v = m ? T(0) : s;
    rhs[row] = v;
    if (sol1) sol1[row] = m ? T(0) : omega * (invd[row] * v);
    return double(v) * double(v);
  }
};

// prolongation + coarse-grid correction: sol += 1 * filter_cor(P sol_c)
template<typename T>
struct EpiProlong {
  static constexpr bool kReduce = false;
  T* sol; const uint32_t* mask;
  __device__ __forceinline__ double operator()(uint32_t row, T s) const {
    if (!masked(mask, row)) sol[row] = T(1) * s + sol[row];
    return 0.0;
  }
};

// ------------------------------------------------------------------ SELL kernel
// AT = accumulation type (double for FP64 values, float otherwise)
template<typename VT, typename XT, typename AT, typename Epi, int UNROLL>
__global__ void __launch_bounds__(256) k_sell(SellView A, const XT* __restrict__ x, Epi epi,
                                              double* ws, unsigned* counter, double* red_out) {
  __shared__ double sh[8];
  const int lane = threadIdx.x & 31;
  const uint32_t wpb = blockDim.x >> 5;
  const VT* __restrict__ val = static_cast<const VT*>(A.val);
  double acc = 0.0;
  for (uint32_t c = blockIdx.x * wpb + (threadIdx.x >> 5); c < A.nchunks; c += gridDim.x * wpb) {
    const uint32_t beg = __ldg(A.cs + c) + lane;
    const uint32_t len = __ldg(A.cl + c);
    AT sum = AT(0);
    uint32_t j = 0;
    for (; j + UNROLL <= len; j += UNROLL) {
      uint32_t cc[UNROLL];
      AT vv[UNROLL];
#pragma unroll
      for (int u = 0; u < UNROLL; ++u) {
        cc[u] = ld_stream(A.col + beg + (j + u) * 32u);
        vv[u] = AT(ld_stream(val + beg + (j + u) * 32u));
      }
#pragma unroll
      for (int u = 0; u < UNROLL; ++u) sum += vv[u] * AT(__ldg(x + cc[u]));
    }
    for (; j < len; ++j) {
      const uint32_t cc = ld_stream(A.col + beg + j * 32u);
      sum += AT(ld_stream(val + beg + j * 32u)) * AT(__ldg(x + cc));
    }
    const uint32_t srow = c * 32u + lane;
    if (srow < A.rows) {
      const uint32_t row = A.perm ? __ldg(A.perm + srow) : srow;
      if (sizeof(VT) == 2) sum *= AT(A.scale);
      acc += epi(row, sum);
    }
  }
  if (Epi::kReduce) {
    const double blk = block_sum<256>(acc, sh);
    reduce_finish<256>(blk, ws, counter, red_out, sh, false);
  }
}

// ------------------------------------------------------------------ CSR kernel (transfers)
struct CsrView {
  uint32_t rows;
  const uint32_t* rp;
  const uint32_t* col;
  const void* val;
};

template<typename VT, typename XT, typename AT, typename Epi, int G>
__global__ void __launch_bounds__(256) k_csr_epi(CsrView A, const XT* __restrict__ x, Epi epi,
                                                 double* ws, unsigned* counter, double* red_out) {
  __shared__ double sh[8];
  const VT* __restrict__ val = static_cast<const VT*>(A.val);
  const int sub = threadIdx.x % G;
  const uint32_t gpb = blockDim.x / G;
  double acc = 0.0;
  const uint32_t stride = gridDim.x * gpb;
  // all threads of a sub-group run the same trip count, so the shuffles are convergent
  for (uint32_t rb = blockIdx.x * gpb; rb < A.rows; rb += stride) {
    const uint32_t row = rb + threadIdx.x / G;
    AT sum = AT(0);
    if (row < A.rows) {
      const uint32_t end = __ldg(A.rp + row + 1);
      for (uint32_t k = __ldg(A.rp + row) + sub; k < end; k += G)
        sum += AT(ValLoad<VT>::ld(val + k)) * AT(__ldg(x + __ldg(A.col + k)));
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o, G);
    if (sub == 0 && row < A.rows) acc += epi(row, sum);
  }
  if (Epi::kReduce) {
    const double blk = block_sum<256>(acc, sh);
    reduce_finish<256>(blk, ws, counter, red_out, sh, false);
  }
}

}  // namespace fb
