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

// one element global -> shared without a register round trip (cp.async, sm_80+): a warp's
// whole staging pass is in flight at once; complete with cp_async_wait_all() + a barrier
template<typename T>
__device__ __forceinline__ void cp_async_elem(T* smem_dst, const T* gsrc) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "cp.async element of 4 or 8 bytes");
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst));
  if constexpr (sizeof(T) == 4) asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(gsrc) : "memory");
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }


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

// FP16 values of two slots per 4-byte load (the FP16 storage interleaves each chunk's slot pairs)
__device__ __forceinline__ float2 ld_stream_pair(const __half* p) {
  const unsigned u = __ldcs(reinterpret_cast<const unsigned*>(p));
  return __half22float2(*reinterpret_cast<const __half2*>(&u));
}

struct SellView {
  uint32_t nchunks;
  uint32_t rows;
  const uint32_t* cs;    // nchunks+1 chunk starts (entries)
  const uint32_t* cl;    // nchunks chunk lengths (slots)
  const uint32_t* col;   // column per entry
  const void* val;       // values (double / float / __half; FP16: slot pairs interleaved, see k_sell)
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
// reduction: RED: ||filter_def(rhs - A x)||^2 (initial defect of the smoother, post-smoothing);
// DOT: out . rhs (the last post-smoothing step of the finest level, whose result is the
// preconditioned defect z and whose rhs is the outer defect r: PCG's r . z)
template<typename T, bool RED, bool DOT = false>
struct EpiJacobi {
  static constexpr bool kReduce = RED || DOT;
  const T* x; const T* rhs; const T* invd; T* out; const T* s0; const uint32_t* mask;
  const double* skip_src; T omega;
  __device__ __forceinline__ double operator()(uint32_t row, T s) const {
    // every input is loaded before out is stored (a load after the store would wait behind it)
    const T b = rhs[row];
    if (smoother_skip<T>(skip_src)) {
      const T o = s0 ? s0[row] : T(0);
      out[row] = o;
      return DOT ? double(o) * double(b) : 0.0;
    }
    const T d = b - s;
    if (masked(mask, row)) {
      const T o = x[row];
      out[row] = o;
      return DOT ? double(o) * double(b) : 0.0;
    }
    const T t = invd[row] * d;
    const T o = omega * t + x[row];
    out[row] = o;
    return RED ? double(d) * double(d) : (DOT ? double(o) * double(b) : 0.0);
  }
};

// The same step for the matrix-free tiled kernel on a Q1 lattice, which forms the inverse
// diagonal of a tile row from the cell coefficients it already holds: a_vv = kr[0] * (sum of
// k over the row's 8 cells), so invd = wd / sum with wd = omega_jac / kr[0] (one streamed
// vector less). Rows outside the tiles use the stored invd.
template<typename T, bool RED = false, bool DOT = false>
struct EpiJacobiK : EpiJacobi<T, RED, DOT> {
  T wd;
};

// PCG direction product: q = filter_def(A p), reduction q . p
// (p may be stored in FP32 when the outer solver keeps its search direction in FP32; the product
// and q stay in T)
template<typename T, typename PT = T>
struct EpiPcgQ {
  static constexpr bool kReduce = true;
  T* q; const PT* p; const uint32_t* mask;
  __device__ __forceinline__ double operator()(uint32_t row, T s) const {
    const T v = masked(mask, row) ? T(0) : s;
    // p's value is loaded before q is stored: a load after the store could not be moved ahead
    // of it (q might alias p as far as the compiler knows) and would wait behind it
    const PT pr = __ldg(p + row);
    q[row] = v;
    return double(v) * double(pr);
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
    const T id = sol1 ? __ldg(invd + row) : T(0);  // loaded before the stores (as in EpiPcgQ)
    rhs[row] = v;
    if (sol1) sol1[row] = m ? T(0) : omega * (id * v);
    return double(v) * double(v);
  }
  // the same with the row's inverse diagonal already loaded (id; any value when sol1 is null)
  __device__ __forceinline__ double with_invd(uint32_t row, T s, T id) const {
    const bool m = masked(mask, row);
    const T v = m ? T(0) : s;
    rhs[row] = v;
    if (sol1) sol1[row] = m ? T(0) : omega * (id * v);
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

// ------------------------------------------------------------------ epilogue operands ahead
// The row inputs of an epilogue, loaded before the row's products are formed (at the start of
// its chunk), so that their latency overlaps the products' loads instead of following them; the
// arithmetic is the epilogue's own. Epilogues without a specialisation load nothing ahead, and
// neither do the kernels that measured slower with it: the FP64 and FP32 SELL steps (926 -> 991
// and 652 -> 659 us per Jacobi step at 257^3) and the FP64 stencil Jacobi step (647 -> 656 us,
// EpiPreIf<false, ...>). Measured faster: the FP32 packed stencil step 365 -> 349 us, the FP64
// stencil PCG-q 656 -> 639 us, the FP16 SELL step 527 -> 520 us.
template<typename Epi>
struct EpiPreNone {
  struct type {};
  __device__ __forceinline__ static type load(const Epi&, uint32_t) { return {}; }
  template<typename S>
  __device__ __forceinline__ static double apply(const Epi& e, uint32_t row, S s, const type&) {
    return e(row, s);
  }
};
template<typename Epi> struct EpiPre : EpiPreNone<Epi> {};
template<bool ON, typename Epi> using EpiPreIf = typename std::conditional<ON, EpiPre<Epi>, EpiPreNone<Epi>>::type;

template<typename T, bool RED, bool DOT>
struct EpiPre<EpiJacobi<T, RED, DOT>> {
  using E = EpiJacobi<T, RED, DOT>;
  struct type { T b, id, xr; bool m; };
  __device__ __forceinline__ static type load(const E& e, uint32_t row) {
    return {e.rhs[row], e.invd ? e.invd[row] : T(0), e.x ? e.x[row] : T(0), masked(e.mask, row)};
  }
  __device__ __forceinline__ static double apply(const E& e, uint32_t row, T s, const type& p) {
    if (smoother_skip<T>(e.skip_src)) {
      const T o = e.s0 ? e.s0[row] : T(0);
      e.out[row] = o;
      return DOT ? double(o) * double(p.b) : 0.0;
    }
    const T d = p.b - s;
    if (p.m) {
      e.out[row] = p.xr;
      return DOT ? double(p.xr) * double(p.b) : 0.0;
    }
    const T t = p.id * d;
    const T o = e.omega * t + p.xr;
    e.out[row] = o;
    return RED ? double(d) * double(d) : (DOT ? double(o) * double(p.b) : 0.0);
  }
};

template<typename T, bool RED, bool LOW>
struct EpiPre<EpiDefect<T, RED, LOW>> {
  using E = EpiDefect<T, RED, LOW>;
  struct type { T b; bool m; };
  __device__ __forceinline__ static type load(const E& e, uint32_t row) { return {e.rhs[row], masked(e.mask, row)}; }
  __device__ __forceinline__ static double apply(const E& e, uint32_t row, T s, const type& p) {
    T d = p.b - s;
    if (p.m) d = T(0);
    e.def[row] = d;
    if (LOW) e.def32[row] = float(d);
    return RED ? double(d) * double(d) : 0.0;
  }
};

template<typename T, typename PT>
struct EpiPre<EpiPcgQ<T, PT>> {
  using E = EpiPcgQ<T, PT>;
  struct type { PT pr; bool m; };
  __device__ __forceinline__ static type load(const E& e, uint32_t row) { return {__ldg(e.p + row), masked(e.mask, row)}; }
  __device__ __forceinline__ static double apply(const E& e, uint32_t row, T s, const type& p) {
    const T v = p.m ? T(0) : s;
    e.q[row] = v;
    return double(v) * double(p.pr);
  }
};

// out = filter(s): the prolongated correction (filter_cor) or A times it (filter_def) of the
// adaptive coarse-grid correction (both filters zero the Dirichlet entries)
template<typename T>
struct EpiFiltered {
  static constexpr bool kReduce = false;
  T* out; const uint32_t* mask;
  __device__ __forceinline__ double operator()(uint32_t row, T s) const {
    out[row] = masked(mask, row) ? T(0) : s;
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
    if constexpr (sizeof(VT) == 2) {
      // FP16: slots 2p and 2p+1 of a chunk are stored interleaved (entry cs + 64p + 2 lane + (j & 1)),
      // so one 4-byte load per lane brings both values; an odd last slot keeps the plain layout.
      // The products are summed in slot order, as in the plain form. The row and its epilogue
      // operands are loaded ahead of the products (EpiPre).
      const uint32_t srow = c * 32u + lane;
      const bool has = srow < A.rows;
      const uint32_t row = has ? (A.perm ? __ldg(A.perm + srow) : srow) : 0u;
      const typename EpiPre<Epi>::type pre = has ? EpiPre<Epi>::load(epi, row) : typename EpiPre<Epi>::type{};
      const VT* vpair = val + (beg - lane) + 2u * lane;
      for (; j + 2 <= len; j += 2) {
        const uint32_t c0 = ld_stream(A.col + beg + j * 32u), c1 = ld_stream(A.col + beg + (j + 1) * 32u);
        const float2 v = ld_stream_pair(vpair + j * 32u);
        sum += AT(v.x) * AT(__ldg(x + c0));
        sum += AT(v.y) * AT(__ldg(x + c1));
      }
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
      if (has) {
        sum *= AT(A.scale);
        acc += EpiPre<Epi>::apply(epi, row, sum, pre);
      }
      continue;
    }
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

namespace fb {

// ------------------------------------------------------------------ stencil SELL
// SELL-32 with implicit column indices for lattice matrices whose every row has the
// same stencil of S neighbour offsets (Q1 on a structured grid: S = 9 in 2D, 27 in 3D).
// Slot j of row r holds a(r, r + off[j]) (0 where the neighbour does not exist), stored
// chunk-major like SELL: val[(c*S + j)*32 + lane]. No column-index stream is read: the
// neighbour index is computed, so the x loads are independent of any other load.
template<int S>
struct StencilView {
  uint32_t rows, nchunks;
  const void* val;
  float scale;
  int32_t off[S];
};

template<typename VT, typename XT, typename AT, typename Epi, int S, int G>
__global__ void __launch_bounds__(256) k_stencil(StencilView<S> A, const XT* __restrict__ x, Epi epi,
                                                 double* ws, unsigned* counter, double* red_out) {
  __shared__ double sh[8];
  const int lane = threadIdx.x & 31;
  const uint32_t wpb = blockDim.x >> 5;
  const VT* __restrict__ val = static_cast<const VT*>(A.val);
  const int32_t last = int32_t(A.rows) - 1;  // rows < 2^31 (checked when the hierarchy is built)
  double acc = 0.0;
  for (uint32_t c = blockIdx.x * wpb + (threadIdx.x >> 5); c < A.nchunks; c += gridDim.x * wpb) {
    const int32_t row0 = int32_t(c) * 32;
    const int32_t row = row0 + lane;
    const VT* vp = val + size_t(c) * S * 32 + lane;
    using Pre = EpiPreIf<std::is_same<Epi, EpiPcgQ<AT, XT>>::value, Epi>;
    const typename Pre::type pre = row <= last ? Pre::load(epi, uint32_t(row)) : typename Pre::type{};
    // warp-uniform: every neighbour of every row of the chunk lies inside the vector
    const bool inside = row0 + A.off[0] >= 0 && row0 + 31 + A.off[S - 1] <= last;
    AT sum = AT(0);
    if (inside) {
      const XT* xr = x + row;
#pragma unroll
      for (int j0 = 0; j0 < S; j0 += G) {
        AT vv[G], xx[G];
#pragma unroll
        for (int u = 0; u < G; ++u)
          if (j0 + u < S) {
            vv[u] = AT(ld_stream(vp + (j0 + u) * 32));
            xx[u] = AT(__ldg(xr + A.off[j0 + u]));
          }
#pragma unroll
        for (int u = 0; u < G; ++u)
          if (j0 + u < S) sum += vv[u] * xx[u];
      }
    } else {
#pragma unroll
      for (int j0 = 0; j0 < S; j0 += G) {
        AT vv[G], xx[G];
#pragma unroll
        for (int u = 0; u < G; ++u)
          if (j0 + u < S) {
            int32_t col = row + A.off[j0 + u];
            col = col < 0 ? 0 : (col > last ? last : col);
            vv[u] = AT(ld_stream(vp + (j0 + u) * 32));
            xx[u] = AT(__ldg(x + col));
          }
#pragma unroll
        for (int u = 0; u < G; ++u)
          if (j0 + u < S) sum += vv[u] * xx[u];
      }
    }
    if (row <= last) {
      if (sizeof(VT) == 2) sum *= AT(A.scale);
      acc += Pre::apply(epi, uint32_t(row), sum, pre);
    }
  }
  if (Epi::kReduce) {
    const double blk = block_sum<256>(acc, sh);
    reduce_finish<256>(blk, ws, counter, red_out, sh, false);
  }
}

// Packed stencil storage for 2- and 4-byte values: every lane reads 8 bytes per load, i.e.
// W = 8 / sizeof(value) consecutive slots of its row: val[((c*G + g)*32 + lane)*W + e] holds
// slot j = g*W + e (G = ceil(S/W); slots j >= S hold 0). A warp load is 256 contiguous bytes.
template<typename VT> struct Pack8;
// raw(): the 8 bytes as loaded; cvt(): their values as FP32 (ld = cvt(raw))
template<> struct Pack8<__half> {
  static constexpr int W = 4;
  __device__ __forceinline__ static uint2 raw(const __half* p) { return __ldcs(reinterpret_cast<const uint2*>(p)); }
  __device__ __forceinline__ static void cvt(uint2 w, float* v) {
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&w.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&w.y));
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
  }
  __device__ __forceinline__ static void ld(const __half* p, float* v) { cvt(raw(p), v); }
};
template<> struct Pack8<float> {
  static constexpr int W = 2;
  __device__ __forceinline__ static uint2 raw(const float* p) { return __ldcs(reinterpret_cast<const uint2*>(p)); }
  __device__ __forceinline__ static void cvt(uint2 w, float* v) {
    v[0] = __uint_as_float(w.x);
    v[1] = __uint_as_float(w.y);
  }
  __device__ __forceinline__ static void ld(const float* p, float* v) { cvt(raw(p), v); }
};

// slot j's neighbour offset on a lattice of CM1 points per side (slot j = (dz+1)*9 + (dy+1)*3 +
// (dx+1) in 3D, (dy+1)*3 + (dx+1) in 2D): a compile-time constant, so that the gathers of a chunk
// whose neighbours all lie inside the vector take it as an immediate address offset
template<int S, int CM1>
__host__ __device__ constexpr int32_t lattice_off(int j) {
  return S == 27 ? ((j / 9 - 1) * CM1 + (j / 3 % 3 - 1)) * CM1 + (j % 3 - 1) : (j / 3 - 1) * CM1 + (j % 3 - 1);
}

// CM1 > 0: the lattice size as a compile-time constant (the launcher checks that the stored
// offsets are those of lattice_off); 0: offsets from the view
template<typename VT, typename Epi, int S, int CM1 = 0>
__global__ void __launch_bounds__(256, 4) k_stencil_packed(StencilView<S> A, const float* __restrict__ x, Epi epi,
                                                           double* ws, unsigned* counter, double* red_out) {
  constexpr int W = Pack8<VT>::W;
  constexpr int G = (S + W - 1) / W;
  __shared__ double sh[8];
  const int lane = threadIdx.x & 31;
  const uint32_t wpb = blockDim.x >> 5;
  const VT* __restrict__ val = static_cast<const VT*>(A.val);
  const int32_t last = int32_t(A.rows) - 1;
  auto off = [&](int j) -> int32_t {
    if constexpr (CM1 > 0) return lattice_off<S, CM1>(j);
    else return A.off[j];
  };
  double acc = 0.0;
  for (uint32_t c = blockIdx.x * wpb + (threadIdx.x >> 5); c < A.nchunks; c += gridDim.x * wpb) {
    const int32_t row0 = int32_t(c) * 32;
    const int32_t row = row0 + lane;
    const VT* vp = val + (size_t(c) * G * 32 + lane) * W;
    const typename EpiPre<Epi>::type pre =
        row <= last ? EpiPre<Epi>::load(epi, uint32_t(row)) : typename EpiPre<Epi>::type{};
    const bool inside = row0 + off(0) >= 0 && row0 + 31 + off(S - 1) <= last;
    float sum = 0.0f;
    if (inside) {
      const float* xr = x + row;
#pragma unroll
      for (int g = 0; g < G; ++g) {
        float v[W];
        Pack8<VT>::ld(vp + g * 32 * W, v);
#pragma unroll
        for (int e = 0; e < W; ++e)
          if (g * W + e < S) sum += v[e] * __ldg(xr + off(g * W + e));
      }
    } else {
#pragma unroll
      for (int g = 0; g < G; ++g) {
        float v[W];
        Pack8<VT>::ld(vp + g * 32 * W, v);
#pragma unroll
        for (int e = 0; e < W; ++e) {
          const int j = g * W + e;
          if (j < S) {
            int32_t col = row + off(j);
            col = col < 0 ? 0 : (col > last ? last : col);
            sum += v[e] * __ldg(x + col);
          }
        }
      }
    }
    if (row <= last) {
      if (sizeof(VT) == 2) sum *= A.scale;
      acc += EpiPre<Epi>::apply(epi, uint32_t(row), sum, pre);
    }
  }
  if (Epi::kReduce) {
    const double blk = block_sum<256>(acc, sh);
    reduce_finish<256>(blk, ws, counter, red_out, sh, false);
  }
}

// ------------------------------------------------------------------ matrix-free Q1 operator
// y = A(k) x for a structured Q1 level without reading a matrix: A(k) = sum_e k_e K_e with
// K_e = (h/2)^(dim-2) K_ref, K_ref the unit-coefficient element matrix of [-1,1]^dim. Local
// vertex a of a cell has bit d set when it lies at the upper end of the cell in direction d.
// On the cube, K_ref[a][b] depends only on a xor b (a reflection of the cube maps vertex a
// to vertex 0 and keeps the Laplacian), so kr[r] = (h/2)^(dim-2) K_ref[0][r] carries the
// whole element matrix. Row i sums over the (up to 2^dim) cells around lattice point i;
// cells outside the domain are skipped, so boundary rows equal the assembled matrix rows.
template<typename T, int DIM>
struct MfView {
  uint32_t rows, nchunks;
  uint32_t M1;          // lattice points per side (= cells per side + 1)
  const T* k;           // per-cell coefficient, lexicographic (nullptr = 1)
  uint64_t ne;          // number of cells
  unsigned long long* err;  // debugging aid: first out-of-range index is recorded here (nullptr = off)
  T kr[1 << DIM];
  int32_t off[DIM == 3 ? 27 : 9];  // neighbour offsets, slot j = (dz+1)*9 + (dy+1)*3 + (dx+1)
};

template<typename T, typename Epi, int DIM>
__global__ void __launch_bounds__(256) k_mf_q1(MfView<T, DIM> A, const T* __restrict__ x, Epi epi,
                                               double* ws, unsigned* counter, double* red_out) {
  constexpr int S = DIM == 3 ? 27 : 9;
  constexpr int NE = 1 << DIM;
  pdl_wait();
  __shared__ double sh[8];
  const int lane = threadIdx.x & 31;
  const uint32_t wpb = blockDim.x >> 5;
  const int32_t last = int32_t(A.rows) - 1;
  const int32_t M1 = int32_t(A.M1), N = M1 - 1;
  double acc = 0.0;
  if (A.err) {
    const uint64_t m1 = A.M1;
    const uint64_t want = DIM == 3 ? m1 * m1 * m1 : m1 * m1;
    const uint64_t nc = DIM == 3 ? uint64_t(N) * N * N : uint64_t(N) * N;
    if (want != A.rows || (A.k && nc != A.ne) || A.nchunks != (A.rows + 31) / 32) {
      atomicCAS(A.err, 0ull, 3ull << 62);
      return;
    }
  }
  for (uint32_t c = blockIdx.x * wpb + (threadIdx.x >> 5); c < A.nchunks; c += gridDim.x * wpb) {
    const int32_t row0 = int32_t(c) * 32;
    const int32_t row = row0 + lane;
    const bool inside = row0 + A.off[0] >= 0 && row0 + 31 + A.off[S - 1] <= last;
    T xv[S];
#pragma unroll
    for (int j = 0; j < S; ++j) {
      int32_t col = row + A.off[j];
      if (!inside) col = col < 0 ? 0 : (col > last ? last : col);
      if (A.err && uint32_t(col) > uint32_t(last)) {
        atomicCAS(A.err, 0ull, (1ull << 62) | (uint64_t(uint32_t(row)) << 8) | uint64_t(j));
        col = 0;
      }
      xv[j] = __ldg(x + col);
    }
    const int32_t rr = row <= last ? row : last;
    const int32_t X = rr % M1;
    const int32_t t = rr / M1;
    const int32_t Y = DIM == 3 ? t % M1 : t;
    const int32_t Z = DIM == 3 ? t / M1 : 0;
    T s = T(0);
#pragma unroll
    for (int e = 0; e < NE; ++e) {
      // cell (X-1+ox, Y-1+oy, Z-1+oz); the row's vertex in it is a = (1-ox, 1-oy, 1-oz)
      const int ox = e & 1, oy = (e >> 1) & 1, oz = (e >> 2) & 1;
      const int a = (1 - ox) | ((1 - oy) << 1) | (DIM == 3 ? (1 - oz) << 2 : 0);
      const int32_t ex = X - 1 + ox, ey = Y - 1 + oy, ez = DIM == 3 ? Z - 1 + oz : 0;
      const bool valid = uint32_t(ex) < uint32_t(N) && uint32_t(ey) < uint32_t(N) &&
                         (DIM == 2 || uint32_t(ez) < uint32_t(N));
      int64_t eidx = valid ? int64_t(ex) + int64_t(N) * (ey + int64_t(N) * ez) : 0;
      if (A.err && A.k && uint64_t(eidx) >= A.ne) {
        atomicCAS(A.err, 0ull, (2ull << 62) | (uint64_t(uint32_t(row)) << 8) | uint64_t(e));
        eidx = 0;
      }
      T ke = A.k ? __ldg(A.k + eidx) : T(1);
      ke = valid ? ke : T(0);
      T in = T(0);
#pragma unroll
      for (int b = 0; b < NE; ++b) {
        const int dx = ox - 1 + (b & 1), dy = oy - 1 + ((b >> 1) & 1);
        const int dz = DIM == 3 ? oz - 1 + ((b >> 2) & 1) : 0;
        const int j = DIM == 3 ? (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1) : (dy + 1) * 3 + (dx + 1);
        in += A.kr[a ^ b] * xv[j];
      }
      s += ke * in;
    }
    if (row <= last) acc += epi(uint32_t(row), s);
  }
  pdl_trigger();
  if (Epi::kReduce) {
    const double blk = block_sum<256>(acc, sh);
    reduce_finish<256>(blk, ws, counter, red_out, sh, false);
  }
}

// FP64 stencil array [c][j][lane] -> packed 8-byte layout of VT (scaled by inv for FP16)
template<typename VT>
__global__ void k_stencil_pack(VT* dst, const double* __restrict__ src, uint32_t nchunks, int S, double inv) {
  constexpr int W = Pack8<VT>::W;
  const int G = (S + W - 1) / W;
  const uint64_t total = uint64_t(nchunks) * G * 32 * W;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < total; i += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t e = i % W, lane = (i / W) % 32, g = (i / (32 * W)) % G, c = i / (uint64_t(32) * W * G);
    const uint64_t j = g * W + e;
    const double v = j < uint64_t(S) ? src[(c * S + j) * 32 + lane] * inv : 0.0;
    dst[i] = VT(v);
  }
}

// ------------------------------------------------------------------ matrix-free Q1 transfers
// Nested Q1 interpolation on lexicographic lattices: fine coordinate X takes coarse X/2
// (weight 1) when even, (X-1)/2 and (X+1)/2 (weight 1/2 each) when odd; P is the tensor
// product, R = P^T. Terms are summed in ascending coarse (resp. fine) index order.
struct Q1Transfer {
  int dim;
  uint32_t Mf1, Mc1;   // lattice points per side, fine and coarse
  uint32_t nf, nc;
};

// launched on a (ceil(M1/32), ceil(M1/8), M1 or 1) grid of 32x8 blocks: no index division.
// Every fine point reads the 2^dim coarse corners around it with independent loads; for an
// even coordinate both corners coincide and the second carries weight 0, so the terms and
// their order are those of the CSR row (plus exact zeros).
template<typename T, typename Epi>
__global__ void __launch_bounds__(256) k_prol_q1(Q1Transfer g, const T* __restrict__ xc, Epi epi) {
  const uint32_t X = blockIdx.x * 32 + threadIdx.x, Y = blockIdx.y * 8 + threadIdx.y, Z = blockIdx.z;
  if (X >= g.Mf1 || Y >= g.Mf1) return;
  const uint32_t i = X + g.Mf1 * (Y + g.Mf1 * Z);
  const uint32_t cx0 = X >> 1, cx1 = (X + 1) >> 1, cy0 = Y >> 1, cy1 = (Y + 1) >> 1;
  const uint32_t cz0 = Z >> 1, cz1 = (Z + 1) >> 1;
  const T w = ((X & 1) ? T(0.5) : T(1)) * ((Y & 1) ? T(0.5) : T(1)) * ((Z & 1) ? T(0.5) : T(1));
  const T wx1 = (X & 1) ? w : T(0), wy1 = (Y & 1) ? T(1) : T(0), wz1 = (Z & 1) ? T(1) : T(0);
  const size_t r00 = (size_t(cz0) * g.Mc1 + cy0) * g.Mc1, r01 = (size_t(cz0) * g.Mc1 + cy1) * g.Mc1;
  T v[8];
  v[0] = xc[r00 + cx0]; v[1] = xc[r00 + cx1];
  v[2] = xc[r01 + cx0]; v[3] = xc[r01 + cx1];
  if (g.dim == 3) {
    const size_t r10 = (size_t(cz1) * g.Mc1 + cy0) * g.Mc1, r11 = (size_t(cz1) * g.Mc1 + cy1) * g.Mc1;
    v[4] = xc[r10 + cx0]; v[5] = xc[r10 + cx1];
    v[6] = xc[r11 + cx0]; v[7] = xc[r11 + cx1];
  }
  T s = T(0);
  s += w * v[0];
  s += wx1 * v[1];
  s += (wy1 * w) * v[2];
  s += (wy1 * wx1) * v[3];
  if (g.dim == 3) {
    s += (wz1 * w) * v[4];
    s += (wz1 * wx1) * v[5];
    s += (wz1 * wy1 * w) * v[6];
    s += (wz1 * wy1 * wx1) * v[7];
  }
  epi(i, s);
}

// launched on a (ceil(Mc1/32), ceil(Mc1/8), Mc1 or 1) grid of 32x8 blocks; the 3^dim fine
// neighbours are read with independent loads (indices clamped, weight 0 outside the lattice)
template<typename T, typename Epi>
__global__ void __launch_bounds__(256) k_rest_q1(Q1Transfer g, const T* __restrict__ xf, Epi epi,
                                                 double* ws, unsigned* counter, double* red_out) {
  __shared__ double sh[8];
  const int X = int(blockIdx.x * 32 + threadIdx.x), Y = int(blockIdx.y * 8 + threadIdx.y), Z = int(blockIdx.z);
  double acc = 0.0;
  if (X < int(g.Mc1) && Y < int(g.Mc1)) {
    const uint32_t i = uint32_t(X) + g.Mc1 * (uint32_t(Y) + g.Mc1 * uint32_t(Z));
    const int F = int(g.Mf1) - 1;
    const int Fz = g.dim == 3 ? F : 0;
    int fx[3], fy[3], fz[3];
    T wx[3], wy[3], wz[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int ox = 2 * X + d - 1, oy = 2 * Y + d - 1, oz = 2 * Z + d - 1;
      const T wd = d == 1 ? T(1) : T(0.5);
      wx[d] = (ox < 0 || ox > F) ? T(0) : wd;
      wy[d] = (oy < 0 || oy > F) ? T(0) : wd;
      wz[d] = (g.dim == 3) ? ((oz < 0 || oz > Fz) ? T(0) : wd) : (d == 1 ? T(1) : T(0));
      fx[d] = ox < 0 ? 0 : (ox > F ? F : ox);
      fy[d] = oy < 0 ? 0 : (oy > F ? F : oy);
      fz[d] = oz < 0 ? 0 : (oz > Fz ? Fz : oz);
    }
    T v[27];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const T* row = xf + (size_t(fz[a]) * g.Mf1 + fy[b]) * g.Mf1;
#pragma unroll
        for (int c = 0; c < 3; ++c) v[(a * 3 + b) * 3 + c] = (g.dim == 3 || a == 1) ? row[fx[c]] : T(0);
      }
    T s = T(0);
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c) s += (wx[c] * wy[b] * wz[a]) * v[(a * 3 + b) * 3 + c];
    acc = epi(i, s);
  }
  if (Epi::kReduce) {
    const uint32_t tid = threadIdx.x + blockDim.x * threadIdx.y;
    const double blk = block_sum_tid<256>(acc, sh, tid);
    const uint32_t nblk = gridDim.x * gridDim.y * gridDim.z;
    const uint32_t bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    reduce_finish_nd<256>(blk, ws, counter, red_out, sh, bid, nblk);
  }
}

// 3D restriction with the fine block staged in shared memory: a block owns 32 x 8 x CZ coarse
// points and first loads the (65 x 17 x (2 CZ + 1)) fine values around them with coalesced
// loads (indices clamped; a clamped value always meets weight 0), then every thread forms CZ
// coarse rows from shared memory. Terms and their order are those of k_rest_q1.
// Launched on a (ceil(Mc1/32), ceil(Mc1/8), ceil(Mc1/CZ)) grid of 256 threads.
//
// bmask (structured levels, the filter is the lattice boundary): the grid covers the coarse
// indices 0..Mc1-2 per axis only, so no block exists for the last plane, line or column alone
// (2^l + 1 points per side). Those rows are filtered, hence zero; the threads next to them write
// them without any fine data.
template<typename T, int CZ>
__global__ void __launch_bounds__(256) k_rest_q1_tile(Q1Transfer g, const T* __restrict__ xf, EpiRestrict<T> epi,
                                                      double* ws, unsigned* counter, double* red_out, int bmask) {
  constexpr int SX = 65, SY = 17, SZ = 2 * CZ + 1;
  pdl_wait();
  __shared__ T sm[SZ][SY][SX];
  __shared__ double sh[8];
  const int X0 = int(blockIdx.x) * 32, Y0 = int(blockIdx.y) * 8, Z0 = int(blockIdx.z) * CZ;
  const int F = int(g.Mf1) - 1;
  const int fx0 = 2 * X0 - 1, fy0 = 2 * Y0 - 1, fz0 = 2 * Z0 - 1;
  // one warp per fine line segment of 65 values (no index division), all copies in flight
  const int lane = threadIdx.x & 31, wrp = threadIdx.x >> 5;
  for (int r = wrp; r < SY * SZ; r += 8) {
    const int ly = r % SY, lz = r / SY;
    int fy = fy0 + ly, fz = fz0 + lz;
    fy = fy < 0 ? 0 : (fy > F ? F : fy);
    fz = fz < 0 ? 0 : (fz > F ? F : fz);
    const T* line = xf + (size_t(fz) * g.Mf1 + fy) * g.Mf1;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int lx = lane + 32 * k;
      if (lx < SX) {
        int fx = fx0 + lx;
        fx = fx < 0 ? 0 : (fx > F ? F : fx);
        cp_async_elem(&sm[lz][ly][lx], line + fx);
      }
    }
  }
  cp_async_wait_all();
  __syncthreads();
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int X = X0 + tx, Y = Y0 + ty;
  double acc = 0.0;
  if (X < int(g.Mc1) && Y < int(g.Mc1)) {
    T wx[3], wy[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int ox = 2 * X + d - 1, oy = 2 * Y + d - 1;
      const T wd = d == 1 ? T(1) : T(0.5);
      wx[d] = (ox < 0 || ox > F) ? T(0) : wd;
      wy[d] = (oy < 0 || oy > F) ? T(0) : wd;
    }
    T wxy[3][3];
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int c = 0; c < 3; ++c) wxy[b][c] = wx[c] * wy[b];
#pragma unroll
    for (int cz = 0; cz < CZ; ++cz) {
      const int Z = Z0 + cz;
      if (Z >= int(g.Mc1)) break;
      T wz[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const int oz = 2 * Z + d - 1;
        wz[d] = (oz < 0 || oz > F) ? T(0) : (d == 1 ? T(1) : T(0.5));
      }
      // the weights are powers of two: wxy * wz equals wx * wy * wz exactly
      T s = T(0);
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
          for (int c = 0; c < 3; ++c) s += (wxy[b][c] * wz[a]) * sm[2 * cz + a][2 * ty + b][2 * tx + c];
      const uint32_t i = uint32_t(X) + g.Mc1 * (uint32_t(Y) + g.Mc1 * uint32_t(Z));
      acc += epi(i, s);
    }
    if (bmask) {
      // the boundary rows beyond the grid: X = Mc1-1 / Y = Mc1-1 next to this thread, and the
      // plane Z = Mc1-1 above the last block
      const int E = int(g.Mc1) - 1;
      const bool ex = X == E - 1 && E == 32 * int(gridDim.x);
      const bool ey = Y == E - 1 && E == 8 * int(gridDim.y);
      const bool ez = int(blockIdx.z) == int(gridDim.z) - 1 && E == CZ * int(gridDim.z);
      if (ex || ey || ez) {
        const int nz = ez ? CZ + 1 : CZ;
        for (int cz = 0; cz < nz; ++cz) {
          const int Z = cz < CZ ? Z0 + cz : E;
          if (Z > E) break;
          for (int q = 0; q < 4; ++q) {
            const bool qx = q & 1, qy = q & 2;
            if ((qx && !ex) || (qy && !ey)) continue;
            if (!qx && !qy && Z != E) continue;  // the thread's own row: formed above
            const uint32_t i = uint32_t(qx ? E : X) + g.Mc1 * (uint32_t(qy ? E : Y) + g.Mc1 * uint32_t(Z));
            acc += epi(i, T(0));
          }
        }
      }
    }
  }
  const double blk = block_sum<256>(acc, sh);
  const uint32_t nblk = gridDim.x * gridDim.y * gridDim.z;
  const uint32_t bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  reduce_finish_nd<256>(blk, ws, counter, red_out, sh, bid, nblk);
}

// 3D prolongation + coarse-grid correction with the coarse block in shared memory: a block
// owns 32 x 8 x FZ fine points; every thread first loads the FZ iterate values of its fine
// column (in flight together), the block loads the 17 x 5 x (FZ/2+1) coarse values behind the
// tile, then every thread forms its FZ corrections. `bmask` (structured levels): the filter is
// the lattice boundary, evaluated from coordinates instead of read. Terms and their order are
// those of k_prol_q1. Launched on a (ceil(Mf1/32), ceil(Mf1/8), ceil(Mf1/FZ)) grid of 256 threads.
template<typename T, int FZ>
__global__ void __launch_bounds__(256) k_prol_q1_tile(Q1Transfer g, const T* __restrict__ xc, T* __restrict__ sol,
                                                      const uint32_t* __restrict__ mask, int bmask) {
  static_assert(FZ % 2 == 0, "slabs start on even planes");
  constexpr int CX = 17, CY = 5, CZ = FZ / 2 + 1;
  pdl_wait();
  __shared__ T cm[CZ][CY][CX];
  const uint32_t X0 = blockIdx.x * 32, Y0 = blockIdx.y * 8, Z0 = blockIdx.z * FZ;
  const uint32_t cx0 = X0 >> 1, cy0 = Y0 >> 1, cz0 = Z0 >> 1;
  const uint32_t Cm = g.Mc1 - 1;
  // this thread's iterate column first: its loads are in flight while the coarse block arrives
  const uint32_t tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const uint32_t X = X0 + tx, Y = Y0 + ty;
  const bool act = X < g.Mf1 && Y < g.Mf1;
  const size_t plane = size_t(g.Mf1) * g.Mf1;
  const size_t i0 = act ? X + size_t(g.Mf1) * (Y + size_t(g.Mf1) * Z0) : 0;
  T old[FZ];
#pragma unroll
  for (int z = 0; z < FZ; ++z) old[z] = (act && Z0 + z < g.Mf1) ? sol[i0 + z * plane] : T(0);
  {
    // one warp per coarse line segment of 17 values
    const int lane = threadIdx.x & 31, wrp = threadIdx.x >> 5;
    for (int r = wrp; r < CY * CZ; r += 8) {
      const int ly = r % CY, lz = r / CY;
      if (lane < CX) {
        const uint32_t cx = min(cx0 + lane, Cm), cy = min(cy0 + ly, Cm), cz = min(cz0 + lz, Cm);
        cp_async_elem(&cm[lz][ly][lane], xc + (size_t(cz) * g.Mc1 + cy) * g.Mc1 + cx);
      }
    }
  }
  cp_async_wait_all();
  __syncthreads();
  pdl_trigger();
  if (!act) return;
  const bool bxy = X == 0 || X == g.Mf1 - 1 || Y == 0 || Y == g.Mf1 - 1;
  const uint32_t lx0 = (X >> 1) - cx0, lx1 = ((X + 1) >> 1) - cx0;
  const uint32_t ly0 = (Y >> 1) - cy0, ly1 = ((Y + 1) >> 1) - cy0;
  const T hx = (X & 1) ? T(0.5) : T(1), hy = (Y & 1) ? T(0.5) : T(1);
  const T wy1 = (Y & 1) ? T(1) : T(0);
  // the correction of plane z of the slab
  auto corr = [&](int z) {
    const T w = hx * hy * ((z & 1) ? T(0.5) : T(1));
    const T wx1 = (X & 1) ? w : T(0);
    const T wz1 = (z & 1) ? T(1) : T(0);
    const int q0 = z >> 1, q1 = (z + 1) >> 1;
    T s = T(0);
    s += w * cm[q0][ly0][lx0];
    s += wx1 * cm[q0][ly0][lx1];
    s += (wy1 * w) * cm[q0][ly1][lx0];
    s += (wy1 * wx1) * cm[q0][ly1][lx1];
    s += (wz1 * w) * cm[q1][ly0][lx0];
    s += (wz1 * wx1) * cm[q1][ly0][lx1];
    s += (wz1 * wy1 * w) * cm[q1][ly1][lx0];
    s += (wz1 * wy1 * wx1) * cm[q1][ly1][lx1];
    return s;
  };
  if (bmask && Z0 > 0 && Z0 + FZ < g.Mf1) {
    // every plane of the slab is interior: the filter is the column's own test, no branch per row
    if (bxy) return;
#pragma unroll
    for (int z = 0; z < FZ; ++z) sol[i0 + z * plane] = T(1) * corr(z) + old[z];
    return;
  }
#pragma unroll
  for (int z = 0; z < FZ; ++z) {
    if (Z0 + z >= g.Mf1) break;
    const size_t i = i0 + z * plane;
    bool msk;
    if (bmask) msk = bxy || Z0 + z == 0 || Z0 + z == g.Mf1 - 1;
    else msk = mask ? ((__ldg(mask + (i >> 5)) >> (i & 31)) & 1u) : false;
    const T s = corr(z);
    if (!msk) sol[i] = T(1) * s + old[z];
  }
}

}  // namespace fb
