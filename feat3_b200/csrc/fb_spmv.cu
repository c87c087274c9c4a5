// Sparse matrix-vector products of the operator layer:
//   * CSR  r = b*y + a*A*x   (sub-warp per row, width picked from the mean row length)
//   * CSR  r = b*y + a*A^T*x (scatter with FP64/FP32 atomics)
//   * FEAT SELL-C ("ELL") r = b*y + a*A*x (thread per row, chunk-major coalesced streams)
// Each takes 32-bit (IT = uint32_t) or 64-bit (IT = uint64_t, FEAT's default Index) index
// arrays as they are; the 64-bit forms read the caller's arrays directly, no narrowing copy.
#include "fb_common.cuh"

namespace fb {

template<typename T, int G, typename IT>
__global__ void __launch_bounds__(256) k_csr(T* r, T a, const T* __restrict__ x, T b, const T* y,
                                             const T* __restrict__ val, const IT* __restrict__ col,
                                             const IT* __restrict__ rp, uint64_t rows, bool use_y) {
  const uint64_t gid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  const uint64_t row = gid / G;
  const int sub = threadIdx.x % G;
  if (row >= rows) return;  // whole sub-group exits together (G divides 32)
  const IT beg = rp[row], end = rp[row + 1];
  T sum(0);
  for (IT k = beg + sub; k < end; k += G) sum += val[k] * x[col[k]];
  const unsigned mask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1)));
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(mask, sum, o, G);
  if (sub == 0) {
    const T prev = use_y ? y[row] : T(0);
    r[row] = use_y ? (sum * a) + (b * prev) : sum * a;
  }
}

template<typename T>
__global__ void k_scale_copy(T* r, const T* y, T b, uint64_t n, bool use_y) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    r[i] = use_y ? b * y[i] : T(0);
}

template<typename T, typename IT>
__global__ void k_csr_t(T* r, T a, const T* __restrict__ x, const T* __restrict__ val,
                        const IT* __restrict__ col, const IT* __restrict__ rp, uint64_t rows) {
  const uint64_t gid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  const uint64_t row = gid / 8;
  const int sub = threadIdx.x % 8;
  if (row >= rows) return;
  const T xa = a * x[row];
  for (IT k = rp[row] + sub; k < rp[row + 1]; k += 8) atomicAdd(&r[col[k]], val[k] * xa);
}

template<typename T, typename IT>
__global__ void __launch_bounds__(256) k_ell(T* r, T a, const T* __restrict__ x, T b, const T* y,
                                             const T* __restrict__ val, const IT* __restrict__ col,
                                             const IT* __restrict__ cs, const IT* __restrict__ cl,
                                             uint32_t C, uint64_t rows, bool use_y) {
  const uint64_t row = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  if (row >= rows) return;
  const uint64_t c = row / C;
  const IT lane = IT(row % C);
  const IT base = cs[c] + lane, len = cl[c];
  T sum(0);
#pragma unroll 4
  for (IT j = 0; j < len; ++j) {
    const IT k = base + j * IT(C);
    sum += val[k] * x[col[k]];
  }
  const T prev = use_y ? y[row] : T(0);
  r[row] = use_y ? (sum * a) + (b * prev) : sum * a;
}

template<typename T, typename IT>
int csr_apply(T* r, T a, const T* x, T b, const T* y, const T* val, const IT* col, const IT* rp,
              uint64_t rows, uint64_t cols, uint64_t nnz, int transposed, cudaStream_t s) {
  const bool use_y = std::fabs(b) >= eps_of<T>();
  const uint64_t nout = transposed ? cols : rows;
  if (nout == 0) return FB_OK;
  if (!r || (use_y && !y) || (rows && (!rp || (nnz && (!val || !col || !x))))) return FB_ERR_INVALID;
  // sizes must fit the index type (rows and columns are indices, nnz a row-pointer value)
  const uint64_t lim = sizeof(IT) == 4 ? 0xffffffffull : ~0ull;
  if (rows > lim || cols > lim || nnz > lim) return FB_ERR_INVALID;
  if (transposed) {
    k_scale_copy<T><<<grid_for(nout, 256) > 16u * kSMs ? 16u * kSMs : grid_for(nout, 256), 256, 0, s>>>(r, y, b, nout, use_y);
    FB_CHECK_LAUNCH();
    if (rows && nnz) {
      k_csr_t<T, IT><<<grid_for(rows * 8, 256), 256, 0, s>>>(r, a, x, val, col, rp, rows);
      FB_CHECK_LAUNCH();
    }
    return FB_OK;
  }
  const double avg = rows ? double(nnz) / double(rows) : 0.0;
  if (avg <= 4.0)       k_csr<T, 2, IT><<<grid_for(rows * 2, 256), 256, 0, s>>>(r, a, x, b, y, val, col, rp, rows, use_y);
  else if (avg <= 8.0)  k_csr<T, 4, IT><<<grid_for(rows * 4, 256), 256, 0, s>>>(r, a, x, b, y, val, col, rp, rows, use_y);
  else if (avg <= 32.0) k_csr<T, 8, IT><<<grid_for(rows * 8, 256), 256, 0, s>>>(r, a, x, b, y, val, col, rp, rows, use_y);
  else if (avg <= 64.0) k_csr<T, 16, IT><<<grid_for(rows * 16, 256), 256, 0, s>>>(r, a, x, b, y, val, col, rp, rows, use_y);
  else                  k_csr<T, 32, IT><<<grid_for(rows * 32, 256), 256, 0, s>>>(r, a, x, b, y, val, col, rp, rows, use_y);
  FB_CHECK_LAUNCH();
  return FB_OK;
}

template<typename T, typename IT>
int ell_apply(T* r, T a, const T* x, T b, const T* y, const T* val, const IT* col, const IT* cs,
              const IT* cl, uint64_t C, uint64_t rows, cudaStream_t s) {
  const bool use_y = std::fabs(b) >= eps_of<T>();
  if (rows == 0) return FB_OK;
  if (!r || (use_y && !y) || !val || !col || !cs || !cl || !x || C == 0 || C > 1024 || rows > 0xffffffffull)
    return FB_ERR_INVALID;
  k_ell<T, IT><<<grid_for(rows, 256), 256, 0, s>>>(r, a, x, b, y, val, col, cs, cl, uint32_t(C), rows, use_y);
  FB_CHECK_LAUNCH();
  return FB_OK;
}

template<typename T, typename IT>
__global__ void k_diag_csr(T* d, const T* __restrict__ val, const IT* __restrict__ col,
                           const IT* __restrict__ rp, uint64_t rows) {
  const uint64_t row = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  if (row >= rows) return;
  T v(0);
  for (IT k = rp[row]; k < rp[row + 1]; ++k)
    if (col[k] == row) { v = val[k]; break; }
  d[row] = v;
}

template<typename T, typename IT>
__global__ void k_diag_ell(T* d, const T* __restrict__ val, const IT* __restrict__ col,
                           const IT* __restrict__ cs, const IT* __restrict__ cl, uint32_t C, uint64_t rows) {
  const uint64_t row = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  if (row >= rows) return;
  const uint64_t c = row / C;
  const IT base = cs[c] + IT(row % C);
  T v(0);
  for (IT j = 0; j < cl[c]; ++j) {
    const IT k = base + j * IT(C);
    if (col[k] == row && val[k] != T(0)) { v = val[k]; break; }
  }
  d[row] = v;
}

template<typename T, typename IT>
int diag_csr(T* d, const T* val, const IT* col, const IT* rp, uint64_t rows, cudaStream_t s) {
  if (rows == 0) return FB_OK;
  if (!d || !val || !col || !rp) return FB_ERR_INVALID;
  k_diag_csr<T, IT><<<grid_for(rows, 256), 256, 0, s>>>(d, val, col, rp, rows);
  FB_CHECK_LAUNCH();
  return FB_OK;
}

template<typename T, typename IT>
int diag_ell(T* d, const T* val, const IT* col, const IT* cs, const IT* cl, uint64_t C, uint64_t rows,
             cudaStream_t s) {
  if (rows == 0) return FB_OK;
  if (!d || !val || !col || !cs || !cl || C == 0 || C > 1024) return FB_ERR_INVALID;
  k_diag_ell<T, IT><<<grid_for(rows, 256), 256, 0, s>>>(d, val, col, cs, cl, uint32_t(C), rows);
  FB_CHECK_LAUNCH();
  return FB_OK;
}

}  // namespace fb

using namespace fb;
#define ST(s) ((cudaStream_t)(s))

extern "C" {

int fb_csr_apply_f64(double* r, double a, const double* x, double b, const double* y, const double* val,
                     const uint32_t* col, const uint32_t* rp, uint64_t rows, uint64_t cols, uint64_t nnz,
                     int transposed, fb_stream_t s) {
  return csr_apply<double, uint32_t>(r, a, x, b, y, val, col, rp, rows, cols, nnz, transposed, ST(s));
}
int fb_csr_apply_f32(float* r, float a, const float* x, float b, const float* y, const float* val,
                     const uint32_t* col, const uint32_t* rp, uint64_t rows, uint64_t cols, uint64_t nnz,
                     int transposed, fb_stream_t s) {
  return csr_apply<float, uint32_t>(r, a, x, b, y, val, col, rp, rows, cols, nnz, transposed, ST(s));
}
int fb_csr_apply_f64_u64(double* r, double a, const double* x, double b, const double* y, const double* val,
                         const uint64_t* col, const uint64_t* rp, uint64_t rows, uint64_t cols, uint64_t nnz,
                         int transposed, fb_stream_t s) {
  return csr_apply<double, uint64_t>(r, a, x, b, y, val, col, rp, rows, cols, nnz, transposed, ST(s));
}
int fb_csr_apply_f32_u64(float* r, float a, const float* x, float b, const float* y, const float* val,
                         const uint64_t* col, const uint64_t* rp, uint64_t rows, uint64_t cols, uint64_t nnz,
                         int transposed, fb_stream_t s) {
  return csr_apply<float, uint64_t>(r, a, x, b, y, val, col, rp, rows, cols, nnz, transposed, ST(s));
}
int fb_ell_apply_f64(double* r, double a, const double* x, double b, const double* y, const double* val,
                     const uint32_t* col, const uint32_t* cs, const uint32_t* cl, uint64_t C, uint64_t rows,
                     fb_stream_t s) {
  return ell_apply<double, uint32_t>(r, a, x, b, y, val, col, cs, cl, C, rows, ST(s));
}
int fb_ell_apply_f32(float* r, float a, const float* x, float b, const float* y, const float* val,
                     const uint32_t* col, const uint32_t* cs, const uint32_t* cl, uint64_t C, uint64_t rows,
                     fb_stream_t s) {
  return ell_apply<float, uint32_t>(r, a, x, b, y, val, col, cs, cl, C, rows, ST(s));
}
int fb_ell_apply_f64_u64(double* r, double a, const double* x, double b, const double* y, const double* val,
                         const uint64_t* col, const uint64_t* cs, const uint64_t* cl, uint64_t C, uint64_t rows,
                         fb_stream_t s) {
  return ell_apply<double, uint64_t>(r, a, x, b, y, val, col, cs, cl, C, rows, ST(s));
}
int fb_ell_apply_f32_u64(float* r, float a, const float* x, float b, const float* y, const float* val,
                         const uint64_t* col, const uint64_t* cs, const uint64_t* cl, uint64_t C, uint64_t rows,
                         fb_stream_t s) {
  return ell_apply<float, uint64_t>(r, a, x, b, y, val, col, cs, cl, C, rows, ST(s));
}
int fb_diagonal_csr_f64(double* d, const double* val, const uint32_t* col, const uint32_t* rp, uint64_t rows,
                        fb_stream_t s) {
  return diag_csr<double, uint32_t>(d, val, col, rp, rows, ST(s));
}
int fb_diagonal_csr_f32(float* d, const float* val, const uint32_t* col, const uint32_t* rp, uint64_t rows,
                        fb_stream_t s) {
  return diag_csr<float, uint32_t>(d, val, col, rp, rows, ST(s));
}
int fb_diagonal_csr_f64_u64(double* d, const double* val, const uint64_t* col, const uint64_t* rp, uint64_t rows,
                            fb_stream_t s) {
  return diag_csr<double, uint64_t>(d, val, col, rp, rows, ST(s));
}
int fb_diagonal_csr_f32_u64(float* d, const float* val, const uint64_t* col, const uint64_t* rp, uint64_t rows,
                            fb_stream_t s) {
  return diag_csr<float, uint64_t>(d, val, col, rp, rows, ST(s));
}
int fb_diagonal_ell_f64(double* d, const double* val, const uint32_t* col, const uint32_t* cs, const uint32_t* cl,
                        uint64_t C, uint64_t rows, fb_stream_t s) {
  return diag_ell<double, uint32_t>(d, val, col, cs, cl, C, rows, ST(s));
}
int fb_diagonal_ell_f32(float* d, const float* val, const uint32_t* col, const uint32_t* cs, const uint32_t* cl,
                        uint64_t C, uint64_t rows, fb_stream_t s) {
  return diag_ell<float, uint32_t>(d, val, col, cs, cl, C, rows, ST(s));
}
int fb_diagonal_ell_f64_u64(double* d, const double* val, const uint64_t* col, const uint64_t* cs, const uint64_t* cl,
                            uint64_t C, uint64_t rows, fb_stream_t s) {
  return diag_ell<double, uint64_t>(d, val, col, cs, cl, C, rows, ST(s));
}
int fb_diagonal_ell_f32_u64(float* d, const float* val, const uint64_t* col, const uint64_t* cs, const uint64_t* cl,
                            uint64_t C, uint64_t rows, fb_stream_t s) {
  return diag_ell<float, uint64_t>(d, val, col, cs, cl, C, rows, ST(s));
}

}  // extern "C"
