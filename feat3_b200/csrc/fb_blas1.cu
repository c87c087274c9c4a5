// Vector kernels of the operator layer: axpy, dot, norm2, component product/invert,
// scale, unit filter, precision conversion, fill. HBM-bound; grid-stride loops with
// 16-byte vector accesses where the pointers allow it.
#include "fb_common.cuh"

#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <vector>

namespace fb {

// ------------------------------------------------------------------ workspace (per device)
namespace {
std::mutex g_ws_mtx;
std::vector<Workspace*> g_ws;  // indexed by device ordinal
}

int workspace_get(Workspace** out) {
  int dev = 0;
  FB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_ws_mtx);
  if ((int)g_ws.size() <= dev) g_ws.resize(dev + 1, nullptr);
  if (!g_ws[dev]) {
    Workspace* w = new Workspace();
    if (cudaMalloc(&w->partials, sizeof(double) * kRedBlocks) != cudaSuccess ||
        cudaMalloc(&w->counter, sizeof(unsigned) * 8) != cudaSuccess ||
        cudaMalloc(&w->result, sizeof(double) * 8) != cudaSuccess ||
        cudaMallocHost(&w->host_result, sizeof(double) * 8) != cudaSuccess) {
      delete w;
      return FB_ERR_ALLOC;
    }
    // one-time initialisation, complete before any stream (blocking or not) can use the counter
    if (cudaMemset(w->counter, 0, sizeof(unsigned) * 8) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
      return FB_ERR_CUDA;
    g_ws[dev] = w;
  }
  *out = g_ws[dev];
  return FB_OK;
}

bool debug_enabled() {
  static int on = -1;
  if (on < 0) { const char* e = std::getenv("FB_DEBUG"); on = (e && e[0] == '1') ? 1 : 0; }
  return on == 1;
}

bool pdl_enabled() {
  static int on = -1;
  if (on < 0) { const char* e = std::getenv("FB_PDL"); on = (e && e[0] == '1') ? 1 : 0; }
  return on == 1;
}

bool check_enabled() {
  static int on = -1;
  if (on < 0) { const char* e = std::getenv("FB_CHECK"); on = ((e && e[0] == '1') || debug_enabled()) ? 1 : 0; }
  return on == 1;
}

cudaError_t debug_sync(cudaStream_t s, const char* file, int line) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) return cudaSuccess;
  cudaError_t e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) std::fprintf(stderr, "feat3_b200: %s after the launch at %s:%d\n", cudaGetErrorString(e), file, line);
  return e;
}

void debug_report(cudaError_t e, const char* what, const char* file, int line) {
  std::fprintf(stderr, "feat3_b200: %s returned %s at %s:%d\n", what, cudaGetErrorString(e), file, line);
}

// ------------------------------------------------------------------ elementwise kernels
template<typename T>
__global__ void k_axpy(T* __restrict__ r, T a, const T* __restrict__ x, const T* __restrict__ y, uint64_t n) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    r[i] = a * x[i] + y[i];
}
template<typename T>
__global__ void k_copy(T* __restrict__ r, const T* __restrict__ x, uint64_t n) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    r[i] = x[i];
}
template<typename T>
__global__ void k_cprod(T* __restrict__ r, const T* __restrict__ x, const T* __restrict__ y, uint64_t n) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    r[i] = x[i] * y[i];
}
template<typename T>
__global__ void k_cinv(T* __restrict__ r, const T* __restrict__ x, T s, uint64_t n) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    r[i] = s / x[i];
}
template<typename T>
__global__ void k_scale(T* __restrict__ r, const T* __restrict__ x, T s, uint64_t n) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    r[i] = s * x[i];
}
template<typename T>
__global__ void k_set(T* __restrict__ r, T v, uint64_t n) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    r[i] = v;
}
template<typename D, typename S>
__global__ void k_convert(D* __restrict__ r, const S* __restrict__ x, uint64_t n) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    r[i] = D(x[i]);
}
template<typename T, typename IT>
__global__ void k_filter_rhs(T* __restrict__ v, const T* __restrict__ sv, const IT* __restrict__ idx, uint64_t ue) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < ue; i += uint64_t(gridDim.x) * blockDim.x)
    v[idx[i]] = sv[i];
}
template<typename T, typename IT>
__global__ void k_filter_def(T* __restrict__ v, const IT* __restrict__ idx, uint64_t ue) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < ue; i += uint64_t(gridDim.x) * blockDim.x)
    v[idx[i]] = T(0);
}

// dot / sum of squares, FP64 accumulation, deterministic finish
template<typename T, bool SQUARE, bool SQRT>
__global__ void __launch_bounds__(kRedThreads) k_dot(const T* __restrict__ x, const T* __restrict__ y, uint64_t n,
                                                     double* ws, unsigned* counter, double* out) {
  __shared__ double sh[kRedThreads / 32];
  double acc = 0.0;
  for (uint64_t i = blockIdx.x * uint64_t(kRedThreads) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * kRedThreads) {
    const double a = double(x[i]);
    acc += SQUARE ? a * a : a * double(y[i]);
  }
  double blk = block_sum<kRedThreads>(acc, sh);
  reduce_finish<kRedThreads>(blk, ws, counter, out, sh, SQRT);
}

constexpr int kEW = 256;
inline unsigned ew_grid(uint64_t n) {
  unsigned g = grid_for(n, kEW);
  return g > 16u * kSMs ? 16u * kSMs : g;
}

template<typename T>
int axpy(T* r, T a, const T* x, const T* y, uint64_t n, cudaStream_t s) {
  if (n == 0) return FB_OK;
  if (!r || !y || (!x && std::fabs(double(a)) >= double(eps_of<T>()))) return FB_ERR_INVALID;
  if (std::fabs(a) < eps_of<T>()) {
    if (r == y) return FB_OK;
    k_copy<T><<<ew_grid(n), kEW, 0, s>>>(r, y, n);
  } else {
    k_axpy<T><<<ew_grid(n), kEW, 0, s>>>(r, a, x, y, n);
  }
  FB_CHECK_LAUNCH();
  return FB_OK;
}

template<typename T, bool SQUARE, bool SQRT>
int reduce(const T* x, const T* y, uint64_t n, double* result, cudaStream_t s) {
  if (!result || (n > 0 && (!x || (!SQUARE && !y)))) return FB_ERR_INVALID;
  Workspace* ws = nullptr;
  FB_TRY(workspace_get(&ws));
  unsigned g = grid_for(n, kRedThreads);
  if (g > unsigned(kRedBlocks)) g = kRedBlocks;
  k_dot<T, SQUARE, SQRT><<<g, kRedThreads, 0, s>>>(x, y, n, ws->partials, ws->counter, result);
  FB_CHECK_LAUNCH();
  return FB_OK;
}

template<typename T, bool SQUARE, bool SQRT>
int reduce_sync(const T* x, const T* y, uint64_t n, double* host_result, cudaStream_t s) {
  if (!host_result) return FB_ERR_INVALID;
  Workspace* ws = nullptr;
  FB_TRY(workspace_get(&ws));
  FB_TRY((reduce<T, SQUARE, SQRT>(x, y, n, ws->result, s)));
  FB_CUDA(cudaMemcpyAsync(ws->host_result, ws->result, sizeof(double), cudaMemcpyDeviceToHost, s));
  FB_CUDA(cudaStreamSynchronize(s));
  *host_result = *ws->host_result;
  return FB_OK;
}

template<typename K, typename... A>
int launch_ew(K kern, uint64_t n, cudaStream_t s, A... args) {
  if (n == 0) return FB_OK;
  kern<<<ew_grid(n), kEW, 0, s>>>(args...);
  FB_CHECK_LAUNCH();
  return FB_OK;
}

}  // namespace fb

using namespace fb;
#define ST(s) ((cudaStream_t)(s))

extern "C" {

int fb_axpy_f64(double* r, double a, const double* x, const double* y, uint64_t n, fb_stream_t s) { return axpy<double>(r, a, x, y, n, ST(s)); }
int fb_axpy_f32(float* r, float a, const float* x, const float* y, uint64_t n, fb_stream_t s) { return axpy<float>(r, a, x, y, n, ST(s)); }

int fb_dot_f64(const double* x, const double* y, uint64_t n, double* res, fb_stream_t s) { return reduce<double, false, false>(x, y, n, res, ST(s)); }
int fb_dot_f32(const float* x, const float* y, uint64_t n, double* res, fb_stream_t s) { return reduce<float, false, false>(x, y, n, res, ST(s)); }
int fb_dot_f64_sync(const double* x, const double* y, uint64_t n, double* h, fb_stream_t s) { return reduce_sync<double, false, false>(x, y, n, h, ST(s)); }
int fb_dot_f32_sync(const float* x, const float* y, uint64_t n, double* h, fb_stream_t s) { return reduce_sync<float, false, false>(x, y, n, h, ST(s)); }
int fb_norm2_f64(const double* x, uint64_t n, double* res, fb_stream_t s) { return reduce<double, true, true>(x, x, n, res, ST(s)); }
int fb_norm2_f32(const float* x, uint64_t n, double* res, fb_stream_t s) { return reduce<float, true, true>(x, x, n, res, ST(s)); }
int fb_norm2_f64_sync(const double* x, uint64_t n, double* h, fb_stream_t s) { return reduce_sync<double, true, true>(x, x, n, h, ST(s)); }
int fb_norm2_f32_sync(const float* x, uint64_t n, double* h, fb_stream_t s) { return reduce_sync<float, true, true>(x, x, n, h, ST(s)); }

int fb_component_product_f64(double* r, const double* x, const double* y, uint64_t n, fb_stream_t s) {
  if (n && (!r || !x || !y)) return FB_ERR_INVALID;
  return launch_ew(k_cprod<double>, n, ST(s), r, x, y, n);
}
int fb_component_product_f32(float* r, const float* x, const float* y, uint64_t n, fb_stream_t s) {
  if (n && (!r || !x || !y)) return FB_ERR_INVALID;
  return launch_ew(k_cprod<float>, n, ST(s), r, x, y, n);
}
int fb_component_invert_f64(double* r, const double* x, double sc, uint64_t n, fb_stream_t s) {
  if (n && (!r || !x)) return FB_ERR_INVALID;
  return launch_ew(k_cinv<double>, n, ST(s), r, x, sc, n);
}
int fb_component_invert_f32(float* r, const float* x, float sc, uint64_t n, fb_stream_t s) {
  if (n && (!r || !x)) return FB_ERR_INVALID;
  return launch_ew(k_cinv<float>, n, ST(s), r, x, sc, n);
}
int fb_scale_f64(double* r, const double* x, double sc, uint64_t n, fb_stream_t s) {
  if (n && (!r || !x)) return FB_ERR_INVALID;
  return launch_ew(k_scale<double>, n, ST(s), r, x, sc, n);
}
int fb_scale_f32(float* r, const float* x, float sc, uint64_t n, fb_stream_t s) {
  if (n && (!r || !x)) return FB_ERR_INVALID;
  return launch_ew(k_scale<float>, n, ST(s), r, x, sc, n);
}
int fb_unit_filter_rhs_f64(double* v, const double* sv, const uint32_t* idx, uint64_t ue, fb_stream_t s) {
  if (ue && (!v || !sv || !idx)) return FB_ERR_INVALID;
  return launch_ew(k_filter_rhs<double, uint32_t>, ue, ST(s), v, sv, idx, ue);
}
int fb_unit_filter_def_f64(double* v, const uint32_t* idx, uint64_t ue, fb_stream_t s) {
  if (ue && (!v || !idx)) return FB_ERR_INVALID;
  return launch_ew(k_filter_def<double, uint32_t>, ue, ST(s), v, idx, ue);
}
int fb_unit_filter_rhs_f32(float* v, const float* sv, const uint32_t* idx, uint64_t ue, fb_stream_t s) {
  if (ue && (!v || !sv || !idx)) return FB_ERR_INVALID;
  return launch_ew(k_filter_rhs<float, uint32_t>, ue, ST(s), v, sv, idx, ue);
}
int fb_unit_filter_def_f32(float* v, const uint32_t* idx, uint64_t ue, fb_stream_t s) {
  if (ue && (!v || !idx)) return FB_ERR_INVALID;
  return launch_ew(k_filter_def<float, uint32_t>, ue, ST(s), v, idx, ue);
}
int fb_unit_filter_rhs_f64_u64(double* v, const double* sv, const uint64_t* idx, uint64_t ue, fb_stream_t s) {
  if (ue && (!v || !sv || !idx)) return FB_ERR_INVALID;
  return launch_ew(k_filter_rhs<double, uint64_t>, ue, ST(s), v, sv, idx, ue);
}
int fb_unit_filter_def_f64_u64(double* v, const uint64_t* idx, uint64_t ue, fb_stream_t s) {
  if (ue && (!v || !idx)) return FB_ERR_INVALID;
  return launch_ew(k_filter_def<double, uint64_t>, ue, ST(s), v, idx, ue);
}
int fb_unit_filter_rhs_f32_u64(float* v, const float* sv, const uint64_t* idx, uint64_t ue, fb_stream_t s) {
  if (ue && (!v || !sv || !idx)) return FB_ERR_INVALID;
  return launch_ew(k_filter_rhs<float, uint64_t>, ue, ST(s), v, sv, idx, ue);
}
int fb_unit_filter_def_f32_u64(float* v, const uint64_t* idx, uint64_t ue, fb_stream_t s) {
  if (ue && (!v || !idx)) return FB_ERR_INVALID;
  return launch_ew(k_filter_def<float, uint64_t>, ue, ST(s), v, idx, ue);
}
int fb_convert_f64_to_f32(float* d, const double* x, uint64_t n, fb_stream_t s) {
  if (n && (!d || !x)) return FB_ERR_INVALID;
  return launch_ew(k_convert<float, double>, n, ST(s), d, x, n);
}
int fb_convert_f32_to_f64(double* d, const float* x, uint64_t n, fb_stream_t s) {
  if (n && (!d || !x)) return FB_ERR_INVALID;
  return launch_ew(k_convert<double, float>, n, ST(s), d, x, n);
}
int fb_set_f64(double* d, double v, uint64_t n, fb_stream_t s) {
  if (n && !d) return FB_ERR_INVALID;
  return launch_ew(k_set<double>, n, ST(s), d, v, n);
}
int fb_set_f32(float* d, float v, uint64_t n, fb_stream_t s) {
  if (n && !d) return FB_ERR_INVALID;
  return launch_ew(k_set<float>, n, ST(s), d, v, n);
}

const char* fb_version(void) { return "feat3_b200 0.1 (sm_100a)"; }

}  // extern "C"
