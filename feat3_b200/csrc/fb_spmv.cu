// Sparse matrix-vector products of the operator layer:
//   * CSR  r = b*y + a*A*x   (sub-warp per row, width picked from the mean row length)
//   * CSR  r = b*y + a*A^T*x (scatter with FP64/FP32 atomics)
//   * FEAT SELL-C ("ELL") r = b*y + a*A*x (thread per row, chunk-major coalesced streams)
#include "fb_common.cuh"

namespace fb {

template<typename T, int G>
__global__ void __launch_bounds__(256) k_csr(T* r, T a, const T* __restrict__ x, T b, const T* y,
                                             const T* __restrict__ val, const uint32_t* __restrict__ col,
                                             const uint32_t* __restrict__ rp, uint64_t rows, bool use_y) {
  const uint64_t gid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  const uint64_t row = gid / G;
  const int sub = threadIdx.x % G;
  if (row >= rows) return;  // whole sub-group exits together (G divides 32)
  const uint32_t beg = rp[row], end = rp[row + 1];
  T sum(0);
  for (uint32_t k = beg + sub; k < end; k += G) sum += val[k] * x[col[k]];
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

template<typename T>
__global__ void k_csr_t(T* r, T a, const T* __restrict__ x, const T* __restrict__ val,
                        const uint32_t* __restrict__ col, const uint32_t* __restrict__ rp, uint64_t rows) {
  const uint64_t gid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  const uint64_t row = gid / 8;
  const int sub = threadIdx.x % 8;
  if (row >= rows) return;
  const T xa = a * x[row];
  for (uint32_t k = rp[row] + sub; k < rp[row + 1]; k += 8) atomicAdd(&r[col[k]], val[k] * xa);
}

template<typename T>
__global__ void __launch_bounds__(256) k_ell(T* r, T a, const T* __restrict__ x, T b, const T* y,
                                             const T* __restrict__ val, const uint32_t* __restrict__ col,
                                             const uint32_t* __restrict__ cs, const uint32_t* __restrict__ cl,
                                             uint32_t C, uint64_t rows, bool use_y) {
  const uint64_t row = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  if (row >= rows) return;
  const uint64_t c = row / C;
  const uint32_t lane = uint32_t(row % C);
  const uint32_t base = cs[c] + lane, len = cl[c];
  T sum(0);
#pragma unroll 4
  for (uint32_t j = 0; j < len; ++j) {
    const uint32_t k = base + j * C;
    sum += val[k] * x[col[k]];
  }
  const T prev = use_y ? y[row] : T(0);
  r[row] = use_y ? (sum * a) + (b * prev) : sum * a;
}

template<typename T>
int csr_apply(T* r, T a, const T* x, T b, const T* y, const T* val, const uint32_t* col, const uint32_t* rp,
              uint64_t rows, uint64_t cols, uint64_t nnz, int transposed, cudaStream_t s) {
  const bool use_y = std::fabs(b) >= eps_of<T>();
  const uint64_t nout = transposed ? cols : rows;
  if (nout == 0) return FB_OK;
  if (!r || (use_y && !y) || (rows && (!rp || (nnz && (!val || !col || !x))))) return FB_ERR_INVALID;
  if (rows > 0xffffffffull || cols > 0xffffffffull || nnz > 0xffffffffull) return FB_ERR_INVALID;
  if (transposed) {
    k_scale_copy<T><<<grid_for(nout, 256) > 16u * kSMs ? 16u * kSMs : grid_for(nout, 256), 256, 0, s>>>(r, y, b, nout, use_y);
    FB_CHECK_LAUNCH();
    if (rows && nnz) {
      k_csr_t<T><<<grid_for(rows * 8, 256), 256, 0, s>>>(r, a, x, val, col, rp, rows);
      FB_CHECK_LAUNCH();
    }
    return FB_OK;
  }
  const double avg = rows ? double(nnz) / double(rows) : 0.0;
  if (avg <= 4.0)       k_csr<T, 2><<<grid_for(rows * 2, 256), 256, 0, s>>>(r, a, x, b, y, val, col, rp, rows, use_y);
  else if (avg <= 8.0)  k_csr<T, 4><<<grid_for(rows * 4, 256), 256, 0, s>>>(r, a, x, b, y, val, col, rp, rows, use_y);
  else if (avg <= 32.0) k_csr<T, 8><<<grid_for(rows * 8, 256), 256, 0, s>>>(r, a, x, b, y, val, col, rp, rows, use_y);
  else if (avg <= 64.0) k_csr<T, 16><<<grid_for(rows * 16, 256), 256, 0, s>>>(r, a, x, b, y, val, col, rp, rows, use_y);
  else                  k_csr<T, 32><<<grid_for(rows * 32, 256), 256, 0, s>>>(r, a, x, b, y, val, col, rp, rows, use_y);
  FB_CHECK_LAUNCH();
  return FB_OK;
}

template<typename T>
int ell_apply(T* r, T a, const T* x, T b, const T* y, const T* val, const uint32_t* col, const uint32_t* cs,
              const uint32_t* cl, uint64_t C, uint64_t rows, cudaStream_t s) {
  const bool use_y = std::fabs(b) >= eps_of<T>();
  if (rows == 0) return FB_OK;
  if (!r || (use_y && !y) || !val || !col || !cs || !cl || !x || C == 0 || C > 1024 || rows > 0xffffffffull)
    return FB_ERR_INVALID;
  k_ell<T><<<grid_for(rows, 256), 256, 0, s>>>(r, a, x, b, y, val, col, cs, cl, uint32_t(C), rows, use_y);
  FB_CHECK_LAUNCH();
  return FB_OK;
}

template<typename T>
__global__ void k_diag_csr(T* d, const T* __restrict__ val, const uint32_t* __restrict__ col,
                           const uint32_t* __restrict__ rp, uint64_t rows) {
  const uint64_t row = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  if (row >= rows) return;
  T v(0);
  for (uint32_t k = rp[row]; k < rp[row + 1]; ++k)
    if (col[k] == row) { v = val[k]; break; }
  d[row] = v;
}

template<typename T>
__global__ void k_diag_ell(T* d, const T* __restrict__ val, const uint32_t* __restrict__ col,
                           const uint32_t* __restrict__ cs, const uint32_t* __restrict__ cl, uint32_t C, uint64_t rows) {
  const uint64_t row = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  if (row >= rows) return;
  const uint64_t c = row / C;
  const uint32_t base = cs[c] + uint32_t(row % C);
  T v(0);
  for (uint32_t j = 0; j < cl[c]; ++j) {
    const uint32_t k = base + j * C;
    if (col[k] == row && val[k] != T(0)) { v = val[k]; break; }
  }
  d[row] = v;
}

}  // namespace fb

using namespace fb;
#define ST(s) ((cudaStream_t)(s))

extern "C" {

int fb_csr_apply_f64(double* r, double a, const double* x, double b, const double* y, const double* val,
                     const uint32_t* col, const uint32_t* rp, uint64_t rows, uint64_t cols, uint64_t nnz,
                     int transposed, fb_stream_t s) {
  return csr_apply<double>(r, a, x, b, y, val, col, rp, rows, cols, nnz, transposed, ST(s));
}
int fb_csr_apply_f32(float* r, float a, const float* x, float b, const float* y, const float* val,
                     const uint32_t* col, const uint32_t* rp, uint64_t rows, uint64_t cols, uint64_t nnz,
                     int transposed, fb_stream_t s) {
  return csr_apply<float>(r, a, x, b, y, val, col, rp, rows, cols, nnz, transposed, ST(s));
}
int fb_ell_apply_f64(double* r, double a, const double* x, double b, const double* y, const double* val,
                     const uint32_t* col, const uint32_t* cs, const uint32_t* cl, uint64_t C, uint64_t rows,
                     fb_stream_t s) {
  return ell_apply<double>(r, a, x, b, y, val, col, cs, cl, C, rows, ST(s));
}
int fb_ell_apply_f32(float* r, float a, const float* x, float b, const float* y, const float* val,
                     const uint32_t* col, const uint32_t* cs, const uint32_t* cl, uint64_t C, uint64_t rows,
                     fb_stream_t s) {
  return ell_apply<float>(r, a, x, b, y, val, col, cs, cl, C, rows, ST(s));
}
int fb_diagonal_csr_f64(double* d, const double* val, const uint32_t* col, const uint32_t* rp, uint64_t rows,
                        fb_stream_t s) {
  if (rows == 0) return FB_OK;
  if (!d || !val || !col || !rp) return FB_ERR_INVALID;
  k_diag_csr<double><<<grid_for(rows, 256), 256, 0, ST(s)>>>(d, val, col, rp, rows);
  FB_CHECK_LAUNCH();
  return FB_OK;
}
int fb_diagonal_csr_f32(float* d, const float* val, const uint32_t* col, const uint32_t* rp, uint64_t rows,
                        fb_stream_t s) {
  if (rows == 0) return FB_OK;
  if (!d || !val || !col || !rp) return FB_ERR_INVALID;
  k_diag_csr<float><<<grid_for(rows, 256), 256, 0, ST(s)>>>(d, val, col, rp, rows);
  FB_CHECK_LAUNCH();
  return FB_OK;
}
int fb_diagonal_ell_f64(double* d, const double* val, const uint32_t* col, const uint32_t* cs, const uint32_t* cl,
                        uint64_t C, uint64_t rows, fb_stream_t s) {
  if (rows == 0) return FB_OK;
  if (!d || !val || !col || !cs || !cl || C == 0) return FB_ERR_INVALID;
  k_diag_ell<double><<<grid_for(rows, 256), 256, 0, ST(s)>>>(d, val, col, cs, cl, uint32_t(C), rows);
  FB_CHECK_LAUNCH();
  return FB_OK;
}

}  // extern "C"
