// Shared device/host helpers of the feat3_b200 sm_100a kernels.
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <stdint.h>
#include <cmath>

#include "../../include/feat3_b200.h"

namespace fb {

constexpr int kSMs = 148;            // B200: 2 dies x 74 SMs
constexpr int kWarp = 32;
constexpr int kRedBlocks = 4 * kSMs; // reduction grid: 4 resident CTAs per SM
constexpr int kRedThreads = 256;

// FB_DEBUG=1 in the environment: synchronise after every launch of the multigrid driver
// and report the source line of a failing launch (debugging aid; never on by default)
bool debug_enabled();
// FB_CHECK=1 (implied by FB_DEBUG=1): kernels with self-checks record out-of-range indices
// instead of using them; the record is reported when the solve ends
bool check_enabled();
cudaError_t debug_sync(cudaStream_t s, const char* file, int line);
void debug_report(cudaError_t e, const char* what, const char* file, int line);

// Programmatic dependent launch: kernels of the solve path may be scheduled while their
// predecessor in the stream finishes. Every kernel launched that way starts with pdl_wait()
// (returns once the predecessor has completed and its writes are visible; a no-op for a
// normal launch), and signals pdl_trigger() when the rest of its work no longer delays the
// launch of its successor. Off by default (no gain measured on the graph-replayed solve);
// FB_PDL=1 in the environment turns the attribute on.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
bool pdl_enabled();

// map a CUDA error onto the C-ABI status
inline int cuda_status(cudaError_t e) { return e == cudaSuccess ? FB_OK : FB_ERR_CUDA; }
#define FB_CHECK_LAUNCH() do { cudaError_t _e = cudaGetLastError(); if (_e != cudaSuccess) return FB_ERR_CUDA; } while (0)
#define FB_TRY(x) do { int _s = (x); if (_s != FB_OK) return _s; } while (0)
#define FB_CUDA(x)                                                                       \
  do {                                                                                   \
    cudaError_t _e = (x);                                                                \
    if (_e != cudaSuccess) {                                                             \
      if (fb::debug_enabled()) fb::debug_report(_e, #x, __FILE__, __LINE__);             \
      return FB_ERR_CUDA;                                                                \
    }                                                                                    \
  } while (0)


inline unsigned grid_for(uint64_t n, int threads, int per_thread = 1) {
  uint64_t g = (n + uint64_t(threads) * per_thread - 1) / (uint64_t(threads) * per_thread);
  if (g < 1) g = 1;
  if (g > 0x7fffffffull) g = 0x7fffffffull;
  return unsigned(g);
}

template<typename T> __host__ __device__ constexpr T eps_of();
template<> __host__ __device__ constexpr double eps_of<double>() { return 2.220446049250313e-16; }
template<> __host__ __device__ constexpr float eps_of<float>() { return 1.1920928955078125e-07f; }

// ---------------------------------------------------------------------------------------
// deterministic two-stage reduction: every CTA writes one partial, the last CTA to finish
// sums the partials in index order and writes the scalar. `ws` = [partials (gridDim)],
// `counter` = one u32 that must be 0 before the launch; the last CTA resets it to 0.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template<int THREADS>
__device__ __forceinline__ double block_sum(double v, double* sh /* THREADS/32 */) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = 0.0;
  if (wid == 0) {
    r = (lane < THREADS / 32) ? sh[lane] : 0.0;
    r = warp_sum(r);
  }
  return r;  // valid in thread 0
}

// block sum for 2D/3D blocks: `tid` = flattened thread index; result valid in tid 0
template<int THREADS>
__device__ __forceinline__ double block_sum_tid(double v, double* sh, uint32_t tid) {
  v = warp_sum(v);
  const int lane = tid & 31, wid = tid >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = 0.0;
  if (wid == 0) {
    r = (lane < THREADS / 32) ? sh[lane] : 0.0;
    r = warp_sum(r);
  }
  return r;
}

// Finish a reduction: thread 0 of every CTA passes its CTA partial. Returns true in the one
// thread (of the last CTA) that wrote `*out` (the final sum, optionally transformed).
// The partials buffer and counter live in `ws`/`counter`.
template<int THREADS>
__device__ __forceinline__ bool reduce_finish(double blk, double* ws, unsigned* counter, double* out,
                                              double* sh, bool take_sqrt = false) {
  __shared__ bool am_last;
  if (threadIdx.x == 0) {
    ws[blockIdx.x] = blk;
    __threadfence();
    unsigned t = atomicAdd(counter, 1u);
    am_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  double v = 0.0;
  // fixed order: thread t sums partials t, t+THREADS, ... (L2 loads, free to overlap)
#pragma unroll 4
  for (unsigned i = threadIdx.x; i < gridDim.x; i += THREADS) v += __ldcg(ws + i);
  v = block_sum<THREADS>(v, sh);
  if (threadIdx.x == 0) {
    *out = take_sqrt ? sqrt(v) : v;
    *counter = 0u;
  }
  return threadIdx.x == 0;
}

// the same finish for 2D/3D grids: `bid` = linear block index, `nblk` = number of blocks
template<int THREADS>
__device__ __forceinline__ bool reduce_finish_nd(double blk, double* ws, unsigned* counter, double* out,
                                                 double* sh, uint32_t bid, uint32_t nblk) {
  __shared__ bool am_last;
  const uint32_t tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  if (tid == 0) {
    ws[bid] = blk;
    __threadfence();
    unsigned t = atomicAdd(counter, 1u);
    am_last = (t == nblk - 1);
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  double v = 0.0;
#pragma unroll 4
  for (uint32_t i = tid; i < nblk; i += THREADS) v += __ldcg(ws + i);
  // block_sum indexes by threadIdx.x: flatten is equivalent for 1D-flattened warps
  v = warp_sum(v);
  const int lane = tid & 31, wid = tid >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  if (wid == 0) {
    double r = (lane < THREADS / 32) ? sh[lane] : 0.0;
    r = warp_sum(r);
    if (lane == 0) { *out = r; *counter = 0u; }
  }
  return tid == 0;
}

// per-device library workspace for the stand-alone reductions of the operator C-ABI
struct Workspace {
  double* partials = nullptr;   // kRedBlocks doubles
  unsigned* counter = nullptr;  // one counter per concurrent reduction slot
  double* result = nullptr;     // device scalar used by the *_sync host-returning variants
  double* host_result = nullptr;
};
int workspace_get(Workspace** ws);

}  // namespace fb
