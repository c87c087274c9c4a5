// Dot product that allocates nothing, for callers that cannot call cudaMalloc.
//
// Some callers cannot allocate device memory at the moment they need a reduction. For example,
// code that runs under an external memory manager that owns every allocation, code that must not
// trigger allocation while another library holds the device's memory budget, or an embedding
// that forbids allocation after start-up. fb_dot_f64 draws its partial-sum buffer from a
// per-device workspace that it allocates on first use. This variant runs the same reduction
// kernel with its scratch in a fixed, file-scope device array instead, so no call ever
// allocates or frees device or host memory.
#include "fb_common.cuh"

#include <mutex>

namespace fb {

// the same reduction kernel as fb_dot_f64 (fb_blas1.cu): FP64 accumulation, fixed-order finish
template<typename T>
__global__ void __launch_bounds__(kRedThreads) k_dot_noalloc(const T* __restrict__ x, const T* __restrict__ y,
                                                             uint64_t n, double* ws, unsigned* counter, double* out) {
  __shared__ double sh[kRedThreads / 32];
  double acc = 0.0;
  for (uint64_t i = blockIdx.x * uint64_t(kRedThreads) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * kRedThreads)
    acc += double(x[i]) * double(y[i]);
  const double blk = block_sum<kRedThreads>(acc, sh);
  reduce_finish<kRedThreads>(blk, ws, counter, out, sh, false);
}

// Scratch of the no-allocation entry point: one partial sum per CTA plus the CTA-arrival
// counter. 32 KiB + 256 B on every GPU that loads the library, held until the process exits.
constexpr int kNoallocMaxPartials = FB_NOALLOC_DOT_MAX_CTAS;
static __device__ __align__(256) double g_noalloc_partials[kNoallocMaxPartials];
static __device__ __align__(256) unsigned g_noalloc_counter[64];

namespace {
struct NoallocSymbols {
  double* partials = nullptr;
  unsigned* counter = nullptr;
};
constexpr int kMaxDevices = 64;
std::mutex g_mtx;
NoallocSymbols g_sym[kMaxDevices];
bool g_ready[kMaxDevices] = {false};

// Device addresses of the scratch arrays on the current device. In host code the array names
// are host-side stand-ins, not device addresses, so they are looked up once per device with
// that device current. This set-up happens inside the first call on each device.
int noalloc_symbols(NoallocSymbols* out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return FB_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_mtx);
  if (!g_ready[dev]) {
    NoallocSymbols s;
    if (cudaGetSymbolAddress((void**)&s.partials, g_noalloc_partials) != cudaSuccess) return FB_ERR_CUDA;
    if (cudaGetSymbolAddress((void**)&s.counter, g_noalloc_counter) != cudaSuccess) return FB_ERR_CUDA;
    g_sym[dev] = s;
    g_ready[dev] = true;
  }
  *out = g_sym[dev];
  return FB_OK;
}
}  // namespace

}  // namespace fb

using namespace fb;

extern "C" {

int fb_dot_f64_noalloc(const double* x, const double* y, uint64_t n, double* result, fb_stream_t stream) {
  if (!result || (n > 0 && (!x || !y))) return FB_ERR_INVALID;
  // one partial sum per CTA; each CTA covers FB_NOALLOC_DOT_ELEMS_PER_CTA elements
  const uint64_t per_cta = FB_NOALLOC_DOT_ELEMS_PER_CTA;
  const uint64_t grid = n == 0 ? 1 : (n + per_cta - 1) / per_cta;
  if (n > FB_NOALLOC_DOT_MAX_N || grid > uint64_t(kNoallocMaxPartials)) return FB_ERR_TOO_LARGE;
  NoallocSymbols s;
  FB_TRY(noalloc_symbols(&s));
  cudaStream_t st = (cudaStream_t)stream;
  // the arrival counter must start at zero; the partial sums are overwritten before use
  FB_CUDA(cudaMemsetAsync(s.counter, 0, sizeof(unsigned), st));
  k_dot_noalloc<double><<<unsigned(grid), kRedThreads, 0, st>>>(x, y, n, s.partials, s.counter, result);
  FB_CHECK_LAUNCH();
  return FB_OK;
}

}  // extern "C"
